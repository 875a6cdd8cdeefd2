"""ctypes access to the CPU oracle (test infrastructure).

``oracle/liboracle.so`` is the plain-C restatement of the reference hot path
(oracle/gc_oracle.c); ``oracle/_ref/libgcref.so`` is the reference headers
themselves compiled from the reference tree (present only where that tree was
available at build time).  Only tests, the smoke check and the benchmark's
CPU-baseline leg use this module; it is never on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libgcref.so")

_P = C.POINTER(C.c_double)
_d = C.c_double
_i = C.c_int


# Per-axis derivative counts (x, y, z) of the reference's 31 named partials
# (diff/MixedPartial.hpp, ThirdOrder.hpp, FourthOrder.hpp), with their names.
PARTIAL_NAMES = {
    (2, 0, 0): "dxx", (0, 2, 0): "dyy", (0, 0, 2): "dzz", (1, 1, 0): "dxy", (1, 0, 1): "dxz", (0, 1, 1): "dyz",
    (3, 0, 0): "d3dx3", (0, 3, 0): "d3dy3", (0, 0, 3): "d3dz3", (2, 1, 0): "d3dx2dy", (1, 2, 0): "d3dxdy2",
    (2, 0, 1): "d3dx2dz", (1, 0, 2): "d3dxdz2", (0, 2, 1): "d3dy2dz", (0, 1, 2): "d3dydz2", (1, 1, 1): "d3dxdydz",
    (4, 0, 0): "d4dx4", (0, 4, 0): "d4dy4", (0, 0, 4): "d4dz4", (3, 1, 0): "d4dx3dy", (1, 3, 0): "d4dxdy3",
    (3, 0, 1): "d4dx3dz", (1, 0, 3): "d4dxdz3", (0, 3, 1): "d4dy3dz", (0, 1, 3): "d4dydz3", (2, 2, 0): "d4dx2dy2",
    (2, 0, 2): "d4dx2dz2", (0, 2, 2): "d4dy2dz2", (2, 1, 1): "d4dx2dydz", (1, 2, 1): "d4dxdy2dz",
    (1, 1, 2): "d4dxdydz2",
}
PARTIALS = list(PARTIAL_NAMES)


def _ensure_built() -> None:
    src = os.path.join(ORACLE_DIR, "gc_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "liboracle.so"], check=True)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


class _Instr(C.Structure):
    """One integrand-program instruction (gc_instr / oc_instr layout)."""
    _fields_ = [("op", C.c_int16), ("dst", C.c_int16), ("a", C.c_int16), ("b", C.c_int16), ("value", C.c_double)]


class _Lib:
    """Common numpy front end over either library (prefix oc_ or ref_)."""

    def __init__(self, path: str, prefix: str):
        self.lib = C.CDLL(path)
        self.p = prefix
        for nm in ("integrate", "ch_free_energy", "ch_gradient_energy", "ch_mean"):
            getattr(self.lib, prefix + nm).restype = _d
        err = getattr(self.lib, prefix + "last_error")
        err.restype = C.c_char_p

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def error(self) -> str:
        return self._f("last_error")().decode()

    def _g(self, shape, h):
        nz, ny, nx = shape
        return (nx, ny, nz, _d(h[0]), _d(h[1]), _d(h[2]))

    def _rc(self, rc):
        if rc != 0:
            raise ValueError(self.error())

    def op(self, name: str, order: int, f: np.ndarray, h=(1.0, 1.0, 1.0)) -> np.ndarray:
        """laplacian / gradient / divergence / biharmonic on an (nz, ny, nx)
        array (vector fields: (3, nz, ny, nx)); gradient_vec maps a vector
        field to a (3, 3, nz, ny, nx) matrix field M[row, col] = d_col v_row
        and divergence_mat maps such a matrix field back to a vector field."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        shape = f.shape[-3:]
        out_shape = {"gradient": (3,) + shape, "gradient_vec": (3, 3) + shape,
                     "divergence_mat": (3,) + shape}.get(name, shape)
        out = np.zeros(out_shape)
        self._rc(self._f(name)(order, *self._g(shape, h), _ptr(f), _ptr(out)))
        return out

    def mixed(self, counts, order: int, f: np.ndarray, h=(1.0, 1.0, 1.0)) -> np.ndarray:
        """d^(ax+ay+az) f / dx^ax dy^ay dz^az on an (nz, ny, nx) array."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(f.shape)
        ax, ay, az = counts
        self._rc(self._f("mixed")(ax, ay, az, order, *self._g(f.shape, h), _ptr(f), _ptr(out)))
        return out

    def evaluate_program(self, components: int, arity: int, instr, field, h=(1.0, 1.0, 1.0),
                         kahan=False) -> float:
        """func::evaluate with the callable given as a register program
        (rows op, dst, a, b, value); field (nz, ny, nx) or (3, nz, ny, nx)."""
        field = np.ascontiguousarray(field, dtype=np.float64)
        rows = [_Instr(int(o), int(d), int(a), int(b), float(v)) for o, d, a, b, v in instr]
        arr = (_Instr * len(rows))(*rows)
        out = C.c_double()
        self._rc(self._f("evaluate_program")(components, arity, *self._g(field.shape[-3:], h), _ptr(field), arr,
                                             len(rows), int(kahan), C.byref(out)))
        return out.value

    def cell_laplacian(self, psi, D, h=(1.0, 1.0, 1.0)):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        D = np.ascontiguousarray(D, dtype=np.float64)
        out = np.zeros(psi.shape)
        if self.p == "oc_":
            bad = C.c_int64(-1)
            self._rc(self._f("cell_laplacian")(*self._g(psi.shape, h), _ptr(psi), _ptr(D), _ptr(out), C.byref(bad)))
        else:
            self._rc(self._f("cell_laplacian")(*self._g(psi.shape, h), _ptr(psi), _ptr(D), _ptr(out)))
        return out

    def integrate(self, f, h=(1.0, 1.0, 1.0), kahan=False) -> float:
        f = np.ascontiguousarray(f, dtype=np.float64)
        return self._f("integrate")(*self._g(f.shape, h), _ptr(f), int(kahan))

    def ch_rhs(self, order, M, kappa, psi, h=(1.0, 1.0, 1.0)):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        out = np.zeros(psi.shape)
        self._rc(self._f("ch_rhs")(order, _d(M), _d(kappa), *self._g(psi.shape, h), _ptr(psi), _ptr(out)))
        return out

    def ch_integrate(self, order, M, kappa, psi, dt, n_steps, rk4=True, h=(1.0, 1.0, 1.0)):
        psi = np.array(psi, dtype=np.float64, order="C", copy=True)
        self._rc(self._f("ch_integrate")(order, _d(M), _d(kappa), *self._g(psi.shape, h), _ptr(psi),
                                         _d(dt), n_steps, int(rk4)))
        return psi

    def ch_free_energy(self, psi, kappa, h=(1.0, 1.0, 1.0)) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return self._f("ch_free_energy")(*self._g(psi.shape, h), _ptr(psi), _d(kappa))

    def ch_gradient_energy(self, psi, h=(1.0, 1.0, 1.0)) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return self._f("ch_gradient_energy")(*self._g(psi.shape, h), _ptr(psi))

    def ch_mean(self, psi, h=(1.0, 1.0, 1.0)) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return self._f("ch_mean")(*self._g(psi.shape, h), _ptr(psi))

    def diffuse_const(self, psi, D, dt, n_steps, rk4=True, h=(1.0, 1.0, 1.0)):
        psi = np.array(psi, dtype=np.float64, order="C", copy=True)
        self._rc(self._f("diffuse_const")(*self._g(psi.shape, h), _ptr(psi), _d(D), _d(dt), n_steps, int(rk4)))
        return psi

    def diffuse_fvm(self, psi, D, dt, n_steps, rk4=True, h=(1.0, 1.0, 1.0)):
        psi = np.array(psi, dtype=np.float64, order="C", copy=True)
        D = np.ascontiguousarray(D, dtype=np.float64)
        self._rc(self._f("diffuse_fvm")(*self._g(psi.shape, h), _ptr(psi), _ptr(D), _d(dt), n_steps, int(rk4)))
        return psi


class Oracle(_Lib):
    def __init__(self):
        _ensure_built()
        super().__init__(ORACLE_SO, "oc_")
        self.lib.oc_sum_pairwise.restype = _d
        self.lib.oc_sum_neumaier.restype = _d
        self.lib.oc_d_max_face.restype = _d

    def weights(self, kind: int, order: int):
        buf = (C.c_double * 17)()
        r = self.lib.oc_weights(kind, order, buf)
        return None if r < 0 else np.array(buf[: 2 * r + 1])

    def sum_pairwise(self, x) -> float:
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.oc_sum_pairwise(_ptr(x), C.c_size_t(x.size))

    def sum_neumaier(self, x) -> float:
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.oc_sum_neumaier(_ptr(x), C.c_size_t(x.size))

    def d_max_face(self, D) -> float:
        D = np.ascontiguousarray(D, dtype=np.float64)
        nz, ny, nx = D.shape
        return self.lib.oc_d_max_face(nx, ny, nz, _ptr(D))


class Reference(_Lib):
    def __init__(self):
        super().__init__(REF_SO, "ref_")

    def spectral(self, op: str, f, h=(1.0, 1.0, 1.0), counts=(0, 0, 0)):
        """spectral/Derivatives.hpp through PocketFFT: op 'partial' (counts
        0..4 each), 'laplacian', 'biharmonic' or 'gradient' (3 planes)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        code = {"partial": 0, "laplacian": 1, "biharmonic": 2, "gradient": 3}[op]
        out = np.zeros(((3,) if op == "gradient" else ()) + f.shape)
        self._rc(self.lib.ref_spectral(code, *counts, *self._g(f.shape, h), _ptr(f), _ptr(out)))
        return out

    def write_vtk(self, f, path: str, name: str, h=(1.0, 1.0, 1.0)) -> None:
        """examples/common/vtk_writer.hpp: the reference's ASCII snapshot file."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._rc(self.lib.ref_write_vtk(*self._g(f.shape, h), _ptr(f), path.encode(), name.encode()))

    def make_random_ic(self, shape, seed: int, amplitude: float, h=(1.0, 1.0, 1.0)):
        out = np.zeros(shape)
        self.lib.ref_make_random_ic(*self._g(shape, h), C.c_uint64(seed), _d(amplitude), _ptr(out))
        return out

    def uniform_draws(self, seed: int, amplitude: float, n: int) -> np.ndarray:
        """makeRandomIc's draws before the mean subtraction (std::mt19937_64 +
        std::uniform_real_distribution of the C++ library this was built with)."""
        out = np.zeros(n)
        self.lib.ref_uniform_draws(C.c_uint64(seed), _d(amplitude), C.c_size_t(n), _ptr(out))
        return out


def oracle() -> Oracle:
    return Oracle()


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def reference() -> Reference:
    return Reference()


# CPU flags each x86-64 micro-architecture level needs (x86-64 psABI).
_LEVEL_FLAGS = {
    "v4": {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl", "avx2", "fma", "bmi2"},
    "v3": {"avx", "avx2", "fma", "bmi1", "bmi2", "movbe", "f16c", "abm", "xsave"},
}


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def timing_reference():
    """The reference build for the timed CPU baseline: the release build
    (-O3 -DNDEBUG) for the highest x86-64 level this CPU supports, else the
    parity build.  Returns (library, description)."""
    flags = _cpu_flags()
    for level in ("v4", "v3"):
        path = os.path.join(ORACLE_DIR, "_ref", f"libgcref_{level}.so")
        if os.path.exists(path) and _LEVEL_FLAGS[level] <= flags:
            lib = Reference.__new__(Reference)
            _Lib.__init__(lib, path, "ref_")
            return lib, f"reference headers, g++ -O3 -DNDEBUG -march=x86-64-{level}"
    if reference_available():
        return reference(), "reference headers, g++ -O3 -DNDEBUG -ffp-contract=off (parity build)"
    return oracle(), "C port of the reference (oracle/gc_oracle.c), gcc -O2"
