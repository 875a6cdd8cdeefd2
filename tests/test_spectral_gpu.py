"""Spectral (FFT) derivatives on the GPU against the reference's PocketFFT
path (spectral/Derivatives.hpp): golden vectors from the reference itself and
the live reference build where present, to rounding; exactness on
band-limited fields; the path as the large-N oracle for order-6 stencils."""
import math
import os

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu

COUNTS = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (2, 1, 1), (0, 3, 0), (2, 2, 0), (1, 1, 1), (4, 0, 0),
          (0, 0, 3)]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", torch.float64)


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _close(got, want, rel=1e-12):
    scale = max(float(np.max(np.abs(want))), 1.0)
    return float(np.max(np.abs(got - want))) <= rel * scale


def test_golden_vectors(gc):
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz"))
    for name in ("aniso3d", "flat2d", "cube7"):
        f, h = golden[f"{name}/f"], tuple(golden[f"{name}/h"])
        g = gc.Grid(f.shape[2], f.shape[1], f.shape[0], *h)
        x = _dev(f)
        assert _close(_host(gc.spectral_laplacian(x, g)), golden[f"{name}/spectral_laplacian"]), name
        assert _close(_host(gc.spectral_biharmonic(x, g)), golden[f"{name}/spectral_biharmonic"]), name
        assert _close(_host(gc.spectral_gradient(x, g)), golden[f"{name}/spectral_gradient"]), name
        for c in COUNTS:
            assert _close(_host(gc.spectral_partial(x, g, c)), golden[f"{name}/spectral_partial{c[0]}{c[1]}{c[2]}"]), \
                (name, c)


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
def test_live_reference_all_counts(gc):
    """Every count triple with total order <= 4, even and odd extents (the
    Nyquist rule), 2-D and 3-D, anisotropic spacing."""
    ref = oracle_lib.reference()
    rng = np.random.default_rng(12)
    for shape, h in (((6, 8, 10), (0.3, 0.7, 1.1)), ((1, 16, 20), (1.0, 0.5, 1.0)), ((5, 9, 7), (1.0, 1.0, 2.0))):
        f = rng.standard_normal(shape)
        g = gc.Grid(shape[2], shape[1], shape[0], *h)
        x = _dev(f)
        for ax in range(5):
            for ay in range(5 - ax):
                for az in range(5 - ax - ay):
                    want = ref.spectral("partial", f, h, (ax, ay, az))
                    assert _close(_host(gc.spectral_partial(x, g, (ax, ay, az))), want), (shape, ax, ay, az)
        assert _close(_host(gc.spectral_gradient(x, g)), ref.spectral("gradient", f, h))
        assert _close(_host(gc.spectral_laplacian(x, g)), ref.spectral("laplacian", f, h))


def _modes(n, seed):
    """A band-limited field on [0, 2 pi)^3 (|k| <= 6) with its exact x and
    mixed (x, y) derivatives."""
    import torch
    rng = np.random.default_rng(seed)
    x = torch.arange(n, device="cuda", dtype=torch.float64) * (2 * math.pi / n)
    z, y, xx = torch.meshgrid(x, x, x, indexing="ij")
    f = torch.zeros_like(z)
    fx = torch.zeros_like(z)
    fxy = torch.zeros_like(z)
    for _ in range(12):
        k = rng.integers(-6, 7, size=3)
        a, phi = rng.standard_normal(), rng.uniform(0, 2 * math.pi)
        arg = k[0] * xx + k[1] * y + k[2] * z + phi
        f += a * torch.cos(arg)
        fx -= a * k[0] * torch.sin(arg)
        fxy -= a * k[0] * k[1] * torch.cos(arg)
    return f.contiguous(), fx, fxy


def test_exact_on_band_limited_fields(gc):
    n = 48
    f, fx, fxy = _modes(n, 3)
    h = 2 * math.pi / n
    g = gc.Grid(n, n, n, h, h, h)
    assert float((gc.spectral_partial(f, g, (1, 0, 0)) - fx).abs().max()) < 1e-11
    assert float((gc.spectral_partial(f, g, (1, 1, 0)) - fxy).abs().max()) < 1e-10
    assert float((gc.spectral_gradient(f, g)[0] - fx).abs().max()) < 1e-11


def test_large_n_oracle_for_order6(gc):
    """The intended use: the order-6 stencil Laplacian converges to the
    spectral one at slope 6 (48^3 -> 96^3)."""
    import torch
    errs = []
    for n in (48, 96):
        x = torch.arange(n, device="cuda", dtype=torch.float64) * (2 * math.pi / n)
        z, y, xx = torch.meshgrid(x, x, x, indexing="ij")
        f = (torch.sin(2 * xx + y) * torch.cos(3 * z) + 0.5 * torch.cos(xx - 2 * y + z)).contiguous()
        h = 2 * math.pi / n
        g = gc.Grid(n, n, n, h, h, h)
        lap6 = gc.laplacian(f, g, 6)
        spec = gc.spectral_laplacian(f, g)
        errs.append(float((lap6 - spec).abs().max()))
    slope = math.log2(errs[0] / errs[1])
    assert 5.5 < slope < 6.5, errs


def test_rejections(gc):
    import torch
    g = gc.Grid(8, 8, 8)
    with pytest.raises(ValueError, match="double") as ei:
        gc.spectral_laplacian(torch.zeros((8, 8, 8), device="cuda", dtype=torch.float32), g)
    assert ei.value.status == "GC_ERR_UNSUPPORTED"
    with pytest.raises(ValueError, match="Nx = 1"):
        gc.spectral_laplacian(torch.zeros((8, 8, 1), device="cuda", dtype=torch.float64), gc.Grid(1, 8, 8))
    with pytest.raises(ValueError, match="0..8"):
        gc.spectral_partial(torch.zeros((8, 8, 8), device="cuda", dtype=torch.float64), g, (9, 0, 0))


def test_two_contexts_on_two_streams_same_shape(gc):
    """Each context keeps its own FFT plans bound to its own stream: two
    contexts transforming the same shape at the same time, on two streams,
    give exactly what one context gives alone (shared plans would let one
    context's transform run on the other's stream and share its work area)."""
    import torch
    n = 96
    g = gc.Grid(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n)
    rng = np.random.default_rng(3)
    fields = [_dev(rng.standard_normal((n, n, n))) for _ in range(2)]
    want = [_host(gc.spectral_laplacian(f, g)) for f in fields]
    streams = [torch.cuda.Stream() for _ in range(2)]
    ctxs = [gc.Context(0, s.cuda_stream) for s in streams]
    outs = [torch.empty_like(f) for f in fields]
    for rep in range(4):
        for j in range(2):
            with torch.cuda.stream(streams[j]):
                gc.spectral_laplacian(fields[j], g, out=outs[j], ctx=ctxs[j])
        torch.cuda.synchronize()
        for j in range(2):
            assert np.array_equal(outs[j].cpu().numpy(), want[j]), (rep, j)
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("shape", [(64, 64, 64), (1, 2, 4096), (1, 3, 6000), (2, 96, 50)])
def test_own_transform_lengths(gc, shape):
    """The library's transforms at lengths the golden grids do not reach:
    power-of-two lines (radix-2, up to 4096 with the line beyond 48 KB of
    shared memory) and long non-power-of-two lines (direct DFT, 6000), against
    torch's double-precision FFT of the same field."""
    import torch
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    nz, ny, nx = shape
    h = (0.5, 0.25, 1.0)
    g = gc.Grid(nx, ny, nz, *h)
    x = _dev(f)
    ft = torch.from_numpy(f)
    kx = torch.fft.rfftfreq(nx, d=h[0], dtype=torch.float64) * 2 * np.pi   # (torch's default dtype is float32)
    ky = torch.fft.fftfreq(ny, d=h[1], dtype=torch.float64) * 2 * np.pi
    kz = torch.fft.fftfreq(nz, d=h[2], dtype=torch.float64) * 2 * np.pi
    k2 = kx[None, None, :] ** 2 + ky[None, :, None] ** 2 + kz[:, None, None] ** 2
    want = torch.fft.irfftn(-k2 * torch.fft.rfftn(ft), s=shape).numpy()
    assert _close(_host(gc.spectral_laplacian(x, g)), want), shape
    # d/dx: the Nyquist mode of an even axis is zeroed for an odd count
    mult = 1j * kx[None, None, :]
    if nx % 2 == 0:
        mult = mult.clone()
        mult[..., -1] = 0
    want_dx = torch.fft.irfftn(mult * torch.fft.rfftn(ft), s=shape).numpy()
    assert _close(_host(gc.spectral_partial(x, g, (1, 0, 0))), want_dx), shape
