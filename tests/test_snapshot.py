"""Snapshot output and checkpoints on the CPU (no device needed): the VTK
writer against the reference's own writer (examples/common/vtk_writer.hpp),
the binary VTK form, and the checkpoint format's round trip and integrity
checks."""
import json
import os
import struct

import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gcm():
    import gridcalc_b200
    return gridcalc_b200


def test_vtk_ascii_is_the_reference_file(gcm, tmp_path):
    """Golden file written by the reference: signed zero, extremes,
    subnormals, non-finite values, 17 significant digits."""
    golden = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))
    vals, h = golden["vtk/values"], golden["vtk/h"]
    g = gcm.Grid(vals.shape[2], vals.shape[1], vals.shape[0], *h)
    path = tmp_path / "ours.vtk"
    gcm.write_vtk(vals, g, str(path), "psi")
    with open(os.path.join(HERE, "golden", "reference_snapshot.vtk"), "rb") as f:
        assert path.read_bytes() == f.read()


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
def test_vtk_ascii_matches_live_reference(gcm, tmp_path):
    ref = oracle_lib.reference()
    rng = np.random.default_rng(5)
    for shape, h, name in (((11, 23, 37), (0.1, 1.0 / 3.0, 2.5), "psi"), ((1, 64, 64), (1.0, 1.0, 1.0), "u")):
        f = rng.standard_normal(shape) * 10.0 ** rng.integers(-5, 6, size=shape)
        ref.write_vtk(f, str(tmp_path / "ref.vtk"), name, h)
        gcm.write_vtk(f, gcm.Grid(shape[2], shape[1], shape[0], *h), str(tmp_path / "ours.vtk"), name)
        assert (tmp_path / "ours.vtk").read_bytes() == (tmp_path / "ref.vtk").read_bytes()


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
@settings(max_examples=200, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow,
                                                                   HealthCheck.function_scoped_fixture])
@given(data=st.data())
def test_vtk_ascii_matches_live_reference_random(gcm, tmp_path, data):
    """Any double (signed zeros, subnormals, infinities, NaNs of either sign,
    extreme exponents), any spacing and field name: the same bytes as the
    reference writer."""
    ref = oracle_lib.reference()
    shape = tuple(data.draw(st.integers(1, 5)) for _ in range(3))
    h = tuple(data.draw(st.floats(1e-9, 1e9)) for _ in range(3))
    name = data.draw(st.text(alphabet="abcdefghijklmnopqrstuvwxyz_0123456789", min_size=1, max_size=10))
    vals = data.draw(st.lists(st.floats(allow_nan=True, allow_infinity=True, width=64),
                              min_size=int(np.prod(shape)), max_size=int(np.prod(shape))))
    f = np.array(vals, dtype=np.float64).reshape(shape)
    ref.write_vtk(f, str(tmp_path / "ref.vtk"), name, h)
    gcm.write_vtk(f, gcm.Grid(shape[2], shape[1], shape[0], *h), str(tmp_path / "ours.vtk"), name)
    assert (tmp_path / "ours.vtk").read_bytes() == (tmp_path / "ref.vtk").read_bytes()


def test_vtk_binary_and_float_fields(gcm, tmp_path):
    rng = np.random.default_rng(6)
    f = rng.standard_normal((3, 5, 7))
    g = gcm.Grid(7, 5, 3, 0.5, 0.5, 2.0)
    gcm.write_vtk(f, g, str(tmp_path / "a.vtk"), "psi")
    gcm.write_vtk(f, g, str(tmp_path / "b.vtk"), "psi", binary=True)
    a = (tmp_path / "a.vtk").read_bytes()
    b = (tmp_path / "b.vtk").read_bytes()
    head_a = a.split(b"LOOKUP_TABLE default\n")[0]
    head_b, body = b.split(b"LOOKUP_TABLE default\n")
    assert head_b == head_a.replace(b"\nASCII\n", b"\nBINARY\n")
    assert np.array_equal(np.frombuffer(body[:-1], dtype=">f8").reshape(f.shape), f) and body[-1:] == b"\n"
    # float fields are written as the doubles they convert to
    f32 = f.astype(np.float32)
    gcm.write_vtk(f32, g, str(tmp_path / "c.vtk"), "psi")
    gcm.write_vtk(f32.astype(np.float64), g, str(tmp_path / "d.vtk"), "psi")
    assert (tmp_path / "c.vtk").read_bytes() == (tmp_path / "d.vtk").read_bytes()


def test_vtk_open_failure_message(gcm, tmp_path):
    g = gcm.Grid(2, 2, 1)
    with pytest.raises(ValueError, match="cannot open") as ei:
        gcm.write_vtk(np.zeros((1, 2, 2)), g, str(tmp_path / "no" / "such" / "dir.vtk"))
    assert ei.value.status == "GC_ERR_IO"


@pytest.mark.parametrize("dtype,comps", [(np.float64, 1), (np.float32, 1), (np.float64, 3)])
def test_checkpoint_round_trip(gcm, tmp_path, dtype, comps):
    rng = np.random.default_rng(7)
    g = gcm.Grid(9, 8, 7, 0.1, 0.2, 0.3)
    shape = g.shape if comps == 1 else (comps,) + g.shape
    f = rng.standard_normal(shape).astype(dtype)
    meta = {"step": 1234, "t": 12.34, "kappa": 0.7, "note": "ψ"}
    path = str(tmp_path / "state.gcb")
    gcm.save_checkpoint(f, g, path, meta)
    grid, dts, c, mlen = gcm.checkpoint_info(path)
    assert grid == g and dts == ("f64" if dtype == np.float64 else "f32") and c == comps
    back, grid2, meta2 = gcm.load_checkpoint(path)
    assert back.dtype == dtype and back.shape == shape and np.array_equal(back, f)
    assert meta2 == meta and grid2 == g
    raw = open(path, "rb").read()
    assert raw[:8] == b"GCB200CK" and len(raw) == 80 + mlen + f.nbytes
    assert struct.unpack_from("<I", raw, 8) == (2,)          # version 2: whole-file checksum
    assert struct.unpack_from("<4i", raw, 16) == (9, 8, 7, comps)
    assert json.loads(raw[80:80 + mlen].decode()) == meta
    assert not os.path.exists(path + ".part")


def test_checkpoint_integrity_checks(gcm, tmp_path):
    g = gcm.Grid(4, 4, 4)
    f = np.arange(64.0).reshape(g.shape)
    path = tmp_path / "c.gcb"
    gcm.save_checkpoint(f, g, str(path), {"step": 1})
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "flip.gcb"
    raw2 = bytearray(raw)
    raw2[-9] ^= 0x01                       # one bit of the data
    bad.write_bytes(bytes(raw2))
    with pytest.raises(ValueError, match="checksum") as ei:
        gcm.load_checkpoint(str(bad))
    assert ei.value.status == "GC_ERR_IO"
    (tmp_path / "short.gcb").write_bytes(bytes(raw[:-8]))
    with pytest.raises(ValueError, match="truncated"):
        gcm.load_checkpoint(str(tmp_path / "short.gcb"))
    (tmp_path / "magic.gcb").write_bytes(b"XXXXXXXX" + bytes(raw[8:]))
    with pytest.raises(ValueError, match="not a gridcalc_b200 checkpoint"):
        gcm.load_checkpoint(str(tmp_path / "magic.gcb"))
    raw3 = bytearray(raw)
    struct.pack_into("<i", raw3, 16, 5)    # nx no longer matches the data size
    (tmp_path / "hdr.gcb").write_bytes(bytes(raw3))
    with pytest.raises(ValueError, match="inconsistent header"):
        gcm.checkpoint_info(str(tmp_path / "hdr.gcb"))
    with pytest.raises(ValueError, match="cannot open"):
        gcm.checkpoint_info(str(tmp_path / "missing.gcb"))


# --- checkpoint integrity, random cases ----------------------------------------

_M64 = (1 << 64) - 1


def _checksum64(data: bytes) -> int:
    """The format's 64-bit multiply-rotate checksum, restated (test only)."""
    h = 0x9E3779B97F4A7C15 ^ len(data)
    for i in range(0, len(data), 8):
        w = int.from_bytes(data[i:i + 8].ljust(8, b"\0"), "little")
        h ^= (w * 0xFF51AFD7ED558CCD) & _M64
        h = ((((h << 27) | (h >> 37)) & _M64) * 0x9E3779B97F4A7C15 + 0x52DCE729) & _M64
    h ^= h >> 33
    h = (h * 0xC4CEB9FE1A85EC53) & _M64
    return h ^ (h >> 29)


_META = st.dictionaries(st.text(min_size=1, max_size=8), st.one_of(
    st.integers(-10 ** 12, 10 ** 12), st.floats(allow_nan=False, allow_infinity=False), st.text(max_size=12)),
    max_size=4)


@settings(max_examples=80, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow,
                                                                   HealthCheck.function_scoped_fixture])
@given(data=st.data(), dtype=st.sampled_from([np.float64, np.float32]), comps=st.sampled_from([1, 3]),
       meta=_META)
def test_checkpoint_random_round_trip_and_any_bit_flip(gcm, tmp_path, data, dtype, comps, meta):
    """Any grid, dtype, component count and JSON metadata round-trips
    exactly; a single flipped bit anywhere in the file (header, metadata or
    data) makes the load fail instead of returning altered values."""
    n = [data.draw(st.integers(1, 6)) for _ in range(3)]
    h = [data.draw(st.floats(1e-3, 1e3)) for _ in range(3)]
    g = gcm.Grid(n[0], n[1], n[2], *h)
    shape = g.shape if comps == 1 else (comps,) + g.shape
    f = np.random.default_rng(sum(n)).standard_normal(shape).astype(dtype)
    path = str(tmp_path / "r.gcb")
    gcm.save_checkpoint(f, g, path, meta)
    back, g2, m2 = gcm.load_checkpoint(path)
    assert np.array_equal(back, f) and g2 == g and m2 == meta
    raw = bytearray(open(path, "rb").read())
    bit = data.draw(st.integers(0, 8 * len(raw) - 1))
    raw[bit // 8] ^= 1 << (bit % 8)
    bad = tmp_path / "flipped.gcb"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        gcm.load_checkpoint(str(bad))


def test_checkpoint_version_1_still_read(gcm, tmp_path):
    """A version-1 file (its checksum covers the data only) loads unchanged."""
    g = gcm.Grid(5, 4, 3, 0.5, 0.25, 2.0)
    f = np.random.default_rng(3).standard_normal(g.shape)
    path = tmp_path / "v2.gcb"
    gcm.save_checkpoint(f, g, str(path), {"step": 7})
    raw = bytearray(path.read_bytes())
    mlen = struct.unpack_from("<Q", raw, 64)[0]
    struct.pack_into("<I", raw, 8, 1)
    struct.pack_into("<Q", raw, 72, _checksum64(bytes(raw[80 + mlen:])))
    old = tmp_path / "v1.gcb"
    old.write_bytes(bytes(raw))
    back, g2, meta = gcm.load_checkpoint(str(old))
    assert np.array_equal(back, f) and g2 == g and meta == {"step": 7}
    raw[-1] ^= 0x80                           # its data checksum still guards the data
    old.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        gcm.load_checkpoint(str(old))

