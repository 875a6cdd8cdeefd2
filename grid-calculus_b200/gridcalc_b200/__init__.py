"""Python mirror of the gridcalc hot-path API over the gridcalc_b200 C ABI.

The reference (gridcalc 0.15.1) is header-only C++; its C++ drop-in lives in
``grid-calculus_b200/include/gridcalc``.  This module exposes the same
functions to Python callers (the tests and the benchmark) with the same names,
argument meaning and error behaviour: a violated precondition raises
``ValueError`` (the reference throws ``std::invalid_argument``) carrying the
library's message.

Device memory is a ``torch.Tensor`` on a CUDA device (float64 or float32,
contiguous, i-fastest: shape ``(nz, ny, nx)``).  Every computation runs in
``libgridcalc_b200.so``; there is no CPU path, and importing this module
fails if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

from . import integrand
from . import integrand as _integrand
from .integrand import maximum, minimum, sqrt

__all__ = [
    "lib", "Grid", "Context", "context", "GcError", "F64", "F32",
    "Pairwise", "Kahan", "RK4", "ExplicitEuler", "CahnHilliardRhs",
    "laplacian", "gradient", "divergence", "biharmonic", "d4", "cell_laplacian",
    "integrate", "evaluate", "ch_rhs", "ch_integrate", "diffuse", "diffuse_fvm",
    "d_max_face", "version", "ChBatch", "Corrector", "corrector_init_params", "ch_rkc",
    "rkc_stability_bound", "partial", "PARTIALS", "sqrt", "minimum", "maximum", "program_struct", "integrand_program",
    "write_vtk", "save_checkpoint", "checkpoint_info", "load_checkpoint", "Snapshotter",
    "spectral_partial", "spectral_laplacian", "spectral_biharmonic", "spectral_gradient", "check_finite",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libgridcalc_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"gridcalc_b200: {LIB_PATH} is missing; build it with "
        "`python grid-calculus_b200/build.py` (there is no CPU fallback)")

lib = C.CDLL(LIB_PATH)

F64, F32 = 0, 1
GC_OK = 0
STATUS = {
    0: "GC_OK", 1: "GC_ERR_INVALID_ARG", 2: "GC_ERR_AXIS_EXTENT", 3: "GC_ERR_GRID_MISMATCH",
    4: "GC_ERR_NONPOSITIVE_D", 5: "GC_ERR_CFL", 6: "GC_ERR_CUDA", 7: "GC_ERR_TIMEOUT",
    8: "GC_ERR_NONFINITE", 9: "GC_ERR_UNSUPPORTED", 10: "GC_ERR_IO",
}


class gc_grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double)]


class gc_ch_params(C.Structure):
    _fields_ = [("mobility", C.c_double), ("kappa", C.c_double), ("order", C.c_int32)]


class gc_integrand(C.Structure):
    _fields_ = [("kind", C.c_int32), ("kappa", C.c_double)]


_vp, _gp, _i32, _dbl = C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_double
_SIGS = {
    "gc_context_create": [C.POINTER(C.c_void_p), _i32, _vp],
    "gc_context_destroy": [_vp],
    "gc_synchronize": [_vp],
    "gc_selftest_bounded_wait": [_vp, C.c_int64],
    "gc_malloc": [_vp, C.c_size_t, C.POINTER(C.c_void_p)],
    "gc_free": [_vp, _vp],
    "gc_memcpy_h2d": [_vp, _vp, _vp, C.c_size_t],
    "gc_memcpy_d2h": [_vp, _vp, _vp, C.c_size_t],
    "gc_laplacian": [_vp, _gp, _i32, _i32, _vp, _vp],
    "gc_gradient": [_vp, _gp, _i32, _i32, _vp, _vp],
    "gc_divergence": [_vp, _gp, _i32, _i32, _vp, _vp],
    "gc_biharmonic": [_vp, _gp, _i32, _i32, _vp, _vp],
    "gc_cell_laplacian": [_vp, _gp, _i32, _vp, _vp, _vp, C.POINTER(C.c_int64)],
    "gc_integrate": [_vp, _gp, _i32, _vp, _i32, C.POINTER(C.c_double)],
    "gc_evaluate": [_vp, _gp, _i32, _vp, C.POINTER(gc_integrand), _i32, C.POINTER(C.c_double)],
    "gc_ch_rhs": [_vp, _gp, _i32, C.POINTER(gc_ch_params), _vp, _vp],
    "gc_ch_integrate": [_vp, _gp, _i32, C.POINTER(gc_ch_params), _vp, _dbl, _i32, _i32],
    "gc_diffuse": [_vp, _gp, _i32, _vp, _dbl, _dbl, _i32, _i32],
    "gc_diffuse_fvm": [_vp, _gp, _i32, _vp, _vp, _dbl, _i32, _i32, C.POINTER(C.c_int64)],
    "gc_d_max_face": [_vp, _gp, _i32, _vp, C.POINTER(C.c_double)],
    "gc_ch_rkc": [_vp, _gp, _i32, C.POINTER(gc_ch_params), _vp, _dbl, C.c_int32, C.c_int32],
    "gc_partial": [_vp, _gp, _i32, _i32, _i32, _i32, _i32, _vp, _vp],
    "gc_gradient_vec": [_vp, _gp, _i32, _i32, _vp, _vp],
    "gc_divergence_mat": [_vp, _gp, _i32, _i32, _vp, _vp],
}


class gc_ch_member(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("mobility", C.c_double),
                ("kappa", C.c_double), ("dt", C.c_double)]


_SIGS.update({
    "gc_ch_batch_create": [_vp, C.c_int32, C.POINTER(gc_ch_member), C.c_int32, _i32, C.POINTER(C.c_void_p)],
    "gc_ch_batch_destroy": [_vp],
    "gc_ch_batch_offsets": [_vp, C.POINTER(C.c_int64)],
    "gc_ch_batch_state": [_vp, C.POINTER(C.c_void_p)],
    "gc_ch_batch_run": [_vp, C.c_int32],
    "gc_ch_batch_diagnostics": [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "gc_ch_batch_autotune": [_vp, C.c_int32, C.c_char_p, C.c_char_p, C.c_size_t],
    "gc_ch_batch_set_shape": [_vp, C.c_int32],
})
for _name, _args in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = C.c_int
lib.gc_last_error.restype = C.c_char_p
lib.gc_last_error.argtypes = []
lib.gc_version.restype = C.c_char_p
lib.gc_rkc_stability_bound.restype = C.c_double
lib.gc_rkc_stability_bound.argtypes = [C.c_int32]
lib.gc_status_string.restype = C.c_char_p
lib.gc_status_string.argtypes = [C.c_int]


class GcError(ValueError):
    """A precondition the reference enforces with std::invalid_argument, or a
    device error.  ``status`` is the gc_status name."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = STATUS.get(status, str(status))


def _check(status: int) -> None:
    if status != GC_OK:
        raise GcError(status, lib.gc_last_error().decode())


def version() -> str:
    return lib.gc_version().decode()


@dataclass(frozen=True)
class Grid:
    """core::Grid (core/Grid.hpp:28-148): extents and per-axis cell size."""
    nx: int
    ny: int
    nz: int
    hx: float = 1.0
    hy: float = 1.0
    hz: float = 1.0

    def __post_init__(self):
        if self.nx <= 0 or self.ny <= 0 or self.nz <= 0:
            raise ValueError(f"Grid: extents (Nx, Ny, Nz) must be > 0; got ({self.nx}, {self.ny}, {self.nz})")
        if not (self.hx > 0 and self.hy > 0 and self.hz > 0):
            raise ValueError(f"Grid: cell_size components must be > 0; got ({self.hx}, {self.hy}, {self.hz})")

    @property
    def size(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self) -> tuple:
        return (self.nz, self.ny, self.nx)

    @property
    def cell_volume(self) -> float:
        return self.hx * self.hy * self.hz

    def c(self) -> gc_grid:
        return gc_grid(self.nx, self.ny, self.nz, self.hx, self.hy, self.hz)


OPT_CLUSTER_STEPPING = 0
OPT_FUSED_STEP = 1
lib.gc_context_set_option.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
lib.gc_context_set_option.restype = C.c_int


class Context:
    """A gc_context: one CUDA stream plus cached scratch and graphs."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        _check(lib.gc_context_create(C.byref(h), device, stream))
        self.handle = h
        self.device = device

    def synchronize(self) -> None:
        _check(lib.gc_synchronize(self.handle))

    def set_cluster_stepping(self, enabled: bool) -> None:
        """GC_OPT_CLUSTER_STEPPING: small 2-D grids advance in one
        cluster-resident launch (off by default: the fused step kernel is
        faster on B200)."""
        _check(lib.gc_context_set_option(self.handle, OPT_CLUSTER_STEPPING, int(bool(enabled))))

    def set_fused_step(self, enabled: bool) -> None:
        """GC_OPT_FUSED_STEP: 2-D double RK4 at order 2 runs one fused kernel
        per step (default) or the four stage kernels."""
        _check(lib.gc_context_set_option(self.handle, OPT_FUSED_STEP, int(bool(enabled))))

    def close(self) -> None:
        if self.handle:
            lib.gc_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Context | None = None


def context() -> Context:
    """The module's default context on the current CUDA device, bound to
    torch's current stream."""
    global _default
    if _default is None:
        import torch
        # Enqueue on torch's current stream so that tensors produced by torch
        # are complete before our kernels read them (stream order).
        _default = Context(torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
    return _default


# --- tags ---------------------------------------------------------------
class Pairwise:  # func::Pairwise
    code = 0


class Kahan:  # func::Kahan
    code = 1


class RK4:  # solve::RK4
    code = 1
    diffusionCFLLimit = 0.6963


class ExplicitEuler:  # solve::ExplicitEuler
    code = 0
    diffusionCFLLimit = 0.5


@dataclass(frozen=True)
class CahnHilliardRhs:
    """Device RHS functor M lap(-psi + psi^3 - kappa lap psi)
    (examples/common/cahn_hilliard.hpp:38-59) at Laplacian order 2, 4 or 6."""
    mobility: float = 1.0
    kappa: float = 1.0
    order: int = 2

    def c(self) -> gc_ch_params:
        return gc_ch_params(self.mobility, self.kappa, self.order)


# --- helpers ------------------------------------------------------------
def _dtype_code(t) -> int:
    import torch
    if t.dtype == torch.float64:
        return F64
    if t.dtype == torch.float32:
        return F32
    raise ValueError(f"gridcalc_b200: fields must be float64 or float32, got {t.dtype}")


def _dtype_code_of(dtype) -> int:
    """The gc_dtype code of a torch dtype."""
    import torch
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise ValueError(f"gridcalc_b200: fields must be float64 or float32, got {dtype}")


def _require(t, grid: Grid, comps: int = 1):
    if not t.is_cuda:
        raise ValueError("gridcalc_b200: fields must live on a CUDA device")
    if not t.is_contiguous():
        raise ValueError("gridcalc_b200: fields must be contiguous")
    if t.numel() != comps * grid.size:
        raise ValueError(f"gridcalc_b200: field has {t.numel()} values, grid needs {comps * grid.size}")


def _ctx(ctx):
    return (ctx or context()).handle


def _empty_like_grid(t, grid: Grid, comps: int = 1):
    import torch
    shape = grid.shape if comps == 1 else (comps,) + grid.shape
    return torch.empty(shape, dtype=t.dtype, device=t.device)


# --- diff:: -------------------------------------------------------------
def laplacian(field, grid: Grid, order: int = 2, out=None, ctx=None):
    """diff::laplacian<Order> (diff/Laplacian.hpp:44-75)."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    _check(lib.gc_laplacian(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), order,
                            field.data_ptr(), out.data_ptr()))
    return out


def _matrix_like_grid(t, grid: Grid):
    import torch
    return torch.empty((3, 3) + grid.shape, dtype=t.dtype, device=t.device)


def gradient(field, grid: Grid, order: int = 2, out=None, ctx=None):
    """diff::gradient<Order>, overloaded on the field's rank like the
    reference.  Scalar -> vector (diff/Gradient.hpp:43-74): out has shape
    (3, nz, ny, nx).  Vector (3 * cells values) -> matrix
    (diff/Gradient.hpp:100-137): out has shape (3, 3, nz, ny, nx) with
    out[row, col] = d_col v_row."""
    if field.numel() == 3 * grid.size and grid.size > 0:
        _require(field, grid, 3)
        out = _matrix_like_grid(field, grid) if out is None else out
        _require(out, grid, 9)
        _check(lib.gc_gradient_vec(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), order,
                                   field.data_ptr(), out.data_ptr()))
        return out
    _require(field, grid)
    out = _empty_like_grid(field, grid, 3) if out is None else out
    _check(lib.gc_gradient(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), order,
                           field.data_ptr(), out.data_ptr()))
    return out


def divergence(vfield, grid: Grid, order: int = 2, out=None, ctx=None):
    """diff::divergence<Order>, overloaded on the field's rank like the
    reference.  Vector -> scalar (diff/Divergence.hpp:43-74).  Matrix
    (9 * cells values, [row, col] planes) -> vector
    (diff/Divergence.hpp:100-135): out[row] = sum over col of d_col M[row, col]."""
    if vfield.numel() == 9 * grid.size and grid.size > 0:
        _require(vfield, grid, 9)
        out = _empty_like_grid(vfield, grid, 3) if out is None else out
        _require(out, grid, 3)
        _check(lib.gc_divergence_mat(_ctx(ctx), C.byref(grid.c()), _dtype_code(vfield), order,
                                     vfield.data_ptr(), out.data_ptr()))
        return out
    _require(vfield, grid, 3)
    out = _empty_like_grid(vfield, grid) if out is None else out
    _check(lib.gc_divergence(_ctx(ctx), C.byref(grid.c()), _dtype_code(vfield), order,
                             vfield.data_ptr(), out.data_ptr()))
    return out


def partial(field, grid: Grid, counts, order: int = 2, out=None, ctx=None):
    """diff::detail::mixedDerivative<ax, ay, az, Order>
    (diff/detail/MultiIndexDerivative.hpp:96-137): d^(ax+ay+az) f /
    dx^ax dy^ay dz^az, counts (ax, ay, az) each 0..4."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    ax, ay, az = counts
    _check(lib.gc_partial(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), order, ax, ay, az,
                          field.data_ptr(), out.data_ptr()))
    return out


# The reference's 31 named partials (diff/MixedPartial.hpp, ThirdOrder.hpp,
# FourthOrder.hpp) by their per-axis derivative counts.
PARTIALS = {
    "dxx": (2, 0, 0), "dyy": (0, 2, 0), "dzz": (0, 0, 2), "dxy": (1, 1, 0), "dxz": (1, 0, 1), "dyz": (0, 1, 1),
    "d3dx3": (3, 0, 0), "d3dy3": (0, 3, 0), "d3dz3": (0, 0, 3), "d3dx2dy": (2, 1, 0), "d3dxdy2": (1, 2, 0),
    "d3dx2dz": (2, 0, 1), "d3dxdz2": (1, 0, 2), "d3dy2dz": (0, 2, 1), "d3dydz2": (0, 1, 2), "d3dxdydz": (1, 1, 1),
    "d4dx4": (4, 0, 0), "d4dy4": (0, 4, 0), "d4dz4": (0, 0, 4), "d4dx3dy": (3, 1, 0), "d4dxdy3": (1, 3, 0),
    "d4dx3dz": (3, 0, 1), "d4dxdz3": (1, 0, 3), "d4dy3dz": (0, 3, 1), "d4dydz3": (0, 1, 3),
    "d4dx2dy2": (2, 2, 0), "d4dx2dz2": (2, 0, 2), "d4dy2dz2": (0, 2, 2), "d4dx2dydz": (2, 1, 1),
    "d4dxdy2dz": (1, 2, 1), "d4dxdydz2": (1, 1, 2),
}


def _named_partial(name, counts):
    def op(field, grid: Grid, order: int = 2, out=None, ctx=None):
        return partial(field, grid, counts, order, out, ctx)
    op.__name__ = name
    op.__doc__ = f"diff::{name}<Order>: d^{sum(counts)} f / dx^{counts[0]} dy^{counts[1]} dz^{counts[2]}."
    return op


for _pname, _pcounts in PARTIALS.items():
    globals()[_pname] = _named_partial(_pname, _pcounts)


def biharmonic(field, grid: Grid, order: int = 2, out=None, ctx=None):
    """diff::biharmonic<Order> (diff/Biharmonic.hpp:48-104)."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    _check(lib.gc_biharmonic(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), order,
                             field.data_ptr(), out.data_ptr()))
    return out


d4 = biharmonic  # diff::d4 (diff/Biharmonic.hpp:116-119)


# --- fvm:: --------------------------------------------------------------
def cell_laplacian(psi, D, grid: Grid, out=None, ctx=None):
    """fvm::cellLaplacian (fvm/CellLaplacian.hpp:91-143)."""
    _require(psi, grid)
    _require(D, grid)
    if D.dtype != psi.dtype:
        raise ValueError("gridcalc_b200: psi and D must share a dtype")
    out = _empty_like_grid(psi, grid) if out is None else out
    bad = C.c_int64(-1)
    _check(lib.gc_cell_laplacian(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), psi.data_ptr(),
                                 D.data_ptr(), out.data_ptr(), C.byref(bad)))
    return out


# --- func:: -------------------------------------------------------------
def integrate(field, grid: Grid, tag=Pairwise, ctx=None) -> float:
    """func::integrate(field, Pairwise|Kahan) (func/Integrate.hpp:116-135)."""
    _require(field, grid)
    r = C.c_double()
    _check(lib.gc_integrate(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                            tag.code, C.byref(r)))
    return r.value


INTEGRANDS = {"psi": 0, "psi_squared": 1, "ch_free_energy": 2, "grad_squared": 3}


class gc_instr(C.Structure):
    _fields_ = [("op", C.c_int16), ("dst", C.c_int16), ("a", C.c_int16), ("b", C.c_int16), ("value", C.c_double)]


class gc_program(C.Structure):
    _fields_ = [("components", C.c_int32), ("arity", C.c_int32), ("n_instr", C.c_int32), ("reserved", C.c_int32),
                ("instr", gc_instr * _integrand.MAX_INSTR)]


lib.gc_evaluate_program.argtypes = [_vp, _gp, _i32, _vp, C.POINTER(gc_program), _i32, C.POINTER(C.c_double)]
lib.gc_evaluate_program.restype = C.c_int


lib.gc_integrand_program.argtypes = [C.POINTER(gc_integrand), C.POINTER(gc_program)]
lib.gc_integrand_program.restype = C.c_int


def integrand_program(name: str, kappa: float = 0.0) -> "_integrand.Program":
    """The program evaluate(field, grid, name) runs for a named hot-path
    integrand, as an integrand.Program (no GPU work)."""
    out = gc_program()
    _check(lib.gc_integrand_program(C.byref(gc_integrand(INTEGRANDS[name], kappa)), C.byref(out)))
    rows = [(int(i.op), int(i.dst), int(i.a), int(i.b), float(i.value)) for i in out.instr[:out.n_instr]]
    return _integrand.Program(out.components, out.arity, rows)


def program_struct(prog: "_integrand.Program") -> gc_program:
    """The C layout of a traced integrand program."""
    p = gc_program(prog.components, prog.arity, len(prog.instr), 0)
    for k, (op, dst, a, b, value) in enumerate(prog.instr):
        p.instr[k] = gc_instr(op, dst, a, b, value)
    return p


def evaluate(field, grid: Grid, integrand, kappa: float = 0.0, tag=Pairwise, ctx=None) -> float:
    """func::evaluate(field, f, tag).

    f may be a Python callable, like the reference's callable
    (func/Functional.hpp:88-148 for a scalar psi: f(psi), f(psi, grad),
    f(psi, grad, lap), f(psi, grad, lap, bih); :183-220 for a vector field of
    3 * cells values: f(u), f(u, M) with M[row, col] = d_col u_row).  It is
    traced once into a device program (gridcalc_b200.integrand) and the
    integrand is formed and reduced on the GPU.  A traced
    ``integrand.Program`` is accepted as well, and the hot-path integrands
    by name: 'psi', 'psi_squared', 'ch_free_energy' (-psi^2/2 + psi^4/4 +
    kappa/2 |grad psi|^2) and 'grad_squared'."""
    if isinstance(integrand, str):
        _require(field, grid)
        f = gc_integrand(INTEGRANDS[integrand], kappa)
        r = C.c_double()
        _check(lib.gc_evaluate(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                               C.byref(f), tag.code, C.byref(r)))
        return r.value
    comps = 3 if grid.size > 0 and field.numel() == 3 * grid.size else 1
    is_program = hasattr(integrand, "instr") and hasattr(integrand, "arity") and hasattr(integrand, "components")
    prog = integrand if is_program else _integrand.trace(integrand, comps)
    if prog.components != comps:
        raise ValueError(f"gridcalc_b200: program is for {prog.components} component(s), field has {comps}")
    _require(field, grid, comps)
    p = program_struct(prog)
    r = C.c_double()
    _check(lib.gc_evaluate_program(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                                   C.byref(p), tag.code, C.byref(r)))
    return r.value


# --- solve:: ------------------------------------------------------------
def ch_rhs(psi, grid: Grid, rhs: CahnHilliardRhs, out=None, ctx=None):
    """One evaluation of the Cahn-Hilliard RHS (cahn_hilliard.hpp:38-59)."""
    _require(psi, grid)
    out = _empty_like_grid(psi, grid) if out is None else out
    _check(lib.gc_ch_rhs(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), C.byref(rhs.c()),
                         psi.data_ptr(), out.data_ptr()))
    return out


def ch_rkc(psi, grid: Grid, rhs: CahnHilliardRhs, dt: float, n_steps: int, stages: int, ctx=None):
    """n_steps damped RKC2 steps of dt with `stages` stages, psi in place (no
    reference counterpart: the base step of the learned coarse step)."""
    _require(psi, grid)
    _check(lib.gc_ch_rkc(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), C.byref(rhs.c()),
                         psi.data_ptr(), dt, n_steps, stages))
    return psi


def rkc_stability_bound(stages: int) -> float:
    """beta(s): RKC2 is stable for dt * lambda_max <= beta(s)."""
    return lib.gc_rkc_stability_bound(stages)


lib.gc_ch_cluster_ctas.argtypes = [C.POINTER(gc_grid), C.c_int, C.c_int32, C.c_int]
lib.gc_ch_cluster_ctas.restype = C.c_int32


def ch_cluster_ctas(grid: Grid, dtype, order: int, tag=RK4) -> int:
    """CTAs of the cluster-resident launch ch_integrate uses for this grid
    (0: the grid does not fit; the per-stage kernels run)."""
    return lib.gc_ch_cluster_ctas(C.byref(grid.c()), _dtype_code_of(dtype), order, tag.code)


def ch_integrate(psi, grid: Grid, rhs: CahnHilliardRhs, dt: float, n_steps: int, tag=RK4, ctx=None):
    """solve::integrate(psi, rhs, dt, n_steps, RK4|ExplicitEuler)
    (solve/RK4.hpp:99-154) with the device Cahn-Hilliard RHS; psi in place."""
    _require(psi, grid)
    _check(lib.gc_ch_integrate(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), C.byref(rhs.c()),
                               psi.data_ptr(), dt, n_steps, tag.code))
    return psi


def diffuse(psi, grid: Grid, D, dt: float, n_steps: int, tag=ExplicitEuler, ctx=None):
    """solve::diffuse (solve/Diffusion.hpp:89-216): D a float (constant) or a
    field (FVM, harmonic-mean faces); psi advanced in place."""
    _require(psi, grid)
    if isinstance(D, (int, float)):
        _check(lib.gc_diffuse(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), psi.data_ptr(),
                              float(D), dt, n_steps, tag.code))
    else:
        _require(D, grid)
        if D.dtype != psi.dtype:
            raise ValueError("gridcalc_b200: psi and D must share a dtype")
        bad = C.c_int64(-1)
        _check(lib.gc_diffuse_fvm(_ctx(ctx), C.byref(grid.c()), _dtype_code(psi), psi.data_ptr(),
                                  D.data_ptr(), dt, n_steps, tag.code, C.byref(bad)))
    return psi


diffuse_fvm = diffuse


def d_max_face(D, grid: Grid, ctx=None) -> float:
    """Largest harmonic-mean face D (solve/Diffusion.hpp:187-207)."""
    _require(D, grid)
    r = C.c_double()
    _check(lib.gc_d_max_face(_ctx(ctx), C.byref(grid.c()), _dtype_code(D), D.data_ptr(), C.byref(r)))
    return r.value


class ChBatch:
    """Batched Cahn-Hilliard ensemble (gc_ch_batch_*): independent 2-D members
    of uneven size, each with its own mobility, kappa and dt, advanced
    together.  `members` is a list of (nx, ny, mobility, kappa, dt)."""

    def __init__(self, members, order: int = 4, dtype=None, ctx=None):
        import torch
        dtype = dtype or torch.float32
        self.ctx = ctx or context()
        self.dtype = dtype
        self.members = [tuple(m) for m in members]
        arr = (gc_ch_member * len(members))(*[gc_ch_member(int(a), int(b), float(c), float(d), float(e))
                                              for a, b, c, d, e in self.members])
        h = C.c_void_p()
        _check(lib.gc_ch_batch_create(self.ctx.handle, len(members), arr, order,
                                      F64 if dtype == torch.float64 else F32, C.byref(h)))
        self.handle = h
        offs = (C.c_int64 * (len(members) + 1))()
        _check(lib.gc_ch_batch_offsets(h, offs))
        self.offsets = list(offs)
        ptr = C.c_void_p()
        _check(lib.gc_ch_batch_state(h, C.byref(ptr)))
        self.state_ptr = ptr.value

    def set_member(self, i: int, values) -> None:
        """Copies a (ny, nx) host or device array into member i."""
        import torch
        t = torch.as_tensor(values, dtype=self.dtype).contiguous()
        n = self.members[i][0] * self.members[i][1]
        assert t.numel() == n
        esize = t.element_size()
        dst = self.state_ptr + self.offsets[i] * esize
        host = t.cpu().contiguous()
        _check(lib.gc_memcpy_h2d(self.ctx.handle, dst, host.data_ptr(), n * esize))
        self.ctx.synchronize()

    def get_member(self, i: int):
        """Member i as a (ny, nx) float64 numpy array."""
        import numpy as np
        import torch
        nx, ny = self.members[i][0], self.members[i][1]
        out = torch.empty((ny, nx), dtype=self.dtype)
        esize = out.element_size()
        _check(lib.gc_memcpy_d2h(self.ctx.handle, out.data_ptr(), self.state_ptr + self.offsets[i] * esize,
                                 nx * ny * esize))
        return out.double().numpy()

    def run(self, n_steps: int) -> None:
        _check(lib.gc_ch_batch_run(self.handle, n_steps))

    FUSED = 4   # GC_BATCH_FUSED: the fused four-stage kernel
    SHAPES = ("32x16x4", "64x8x4", "64x16x4", "64x32x8")   # the stage kernels' tiles, 0..3

    def set_shape(self, shape: int) -> None:
        """Selects a tile shape: 0..3 the stage kernels' tiles (SHAPES),
        FUSED the four-stage kernel (orders 2 and 4)."""
        _check(lib.gc_ch_batch_set_shape(self.handle, shape))

    def diagnostics(self):
        """(mass, free_energy) per member, FP64 (reference convention)."""
        n = len(self.members)
        m = (C.c_double * n)()
        f = (C.c_double * n)()
        _check(lib.gc_ch_batch_diagnostics(self.handle, m, f))
        return list(m), list(f)

    def autotune(self, steps_per_trial: int = 8, cache_path: str | None = None) -> str:
        buf = C.create_string_buffer(4096)
        _check(lib.gc_ch_batch_autotune(self.handle, steps_per_trial,
                                        cache_path.encode() if cache_path else None, buf, 4096))
        return buf.value.decode()

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.gc_ch_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class gc_corrector_policy(C.Structure):
    _fields_ = [("dt_fine", C.c_double), ("fine_per_coarse", C.c_int32),
                ("residual_tol", C.c_double), ("energy_tol", C.c_double), ("energy_rtol", C.c_double),
                ("try_base", C.c_int32)]


class gc_corrector_stats(C.Structure):
    _fields_ = [("accepted", C.c_int64), ("fallbacks", C.c_int64), ("rejected_energy", C.c_int64),
                ("rejected_residual", C.c_int64), ("accepted_base", C.c_int64), ("last_residual", C.c_double)]


for _name, _args in {
    "gc_corrector_create": [_vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)],
    "gc_corrector_destroy": [_vp],
    "gc_corrector_set_params": [_vp, C.POINTER(C.c_float), C.c_int32, C.c_float],
    "gc_corrector_get_params": [_vp, C.POINTER(C.c_float), C.c_int32],
    "gc_corrector_set_base": [_vp, C.c_void_p, C.c_double, C.c_int32],
    "gc_corrector_set_loss": [_vp, C.c_int32],
    "gc_corrector_forward": [_vp, C.c_int32, _i32, _vp, _vp],
    "gc_corrector_gradient": [_vp, C.c_int32, _i32, _vp, _vp, C.POINTER(C.c_float), C.POINTER(C.c_double)],
    "gc_corrector_train_step": [_vp, C.c_int32, _i32, _vp, _vp, C.c_float, C.POINTER(C.c_double)],
    "gc_corrector_advance": [_vp, _gp, C.POINTER(gc_ch_params), _vp, C.c_int32,
                             C.POINTER(gc_corrector_policy), C.POINTER(gc_corrector_stats)],
}.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = C.c_int
lib.gc_corrector_num_params.restype = C.c_int32
lib.gc_corrector_num_params.argtypes = []

CORRECTOR_LAYERS, CORRECTOR_CHANNELS = 6, 32
# Default relative free-energy tolerance of the accept/reject judge: a rise
# of F by one part in 1e10 per coarse step is accepted.  It is far above the
# FP64 round-off of F's sum (about cells x 1e-16 x the mean density, 1e-16 of
# |F|) and far below the 1e-3 free-energy error target (1250 coarse steps to
# t = 200 could add at most 1.25e-7 of |F|).
ENERGY_RTOL = 1e-10


def corrector_init_params(seed: int = 0, last_scale: float = 0.1, inputs: int = 1):
    """He-normal initial parameters (FP32) for the corrector: per layer
    W[9][32 in][32 out] then b[32]; the first layer sees `inputs` input
    channels (1: c alone; 3: c and the two base-step features)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n_c = CORRECTOR_CHANNELS
    out = []
    for layer in range(CORRECTOR_LAYERS):
        fan_in = 9 * (inputs if layer == 0 else n_c)
        w = rng.standard_normal((9, n_c, n_c)) * np.sqrt(2.0 / fan_in)
        if layer == 0:
            w[:, inputs:, :] = 0.0
        if layer == CORRECTOR_LAYERS - 1:
            w *= last_scale
            w[:, :, 1:] = 0.0
        out.append(w.ravel())
        out.append(np.zeros(n_c))
    return np.concatenate(out).astype(np.float32)


class Corrector:
    """Learned coarse-step corrector (gc_corrector_*): 6-layer periodic 3x3
    CNN, BF16 on tensor cores, trained by the library's own kernels."""

    def __init__(self, height: int, width: int, max_batch: int = 1, ctx=None):
        self.ctx = ctx or context()
        self.shape = (height, width)
        h = C.c_void_p()
        _check(lib.gc_corrector_create(self.ctx.handle, height, width, max_batch, C.byref(h)))
        self.handle = h
        self.n_params = lib.gc_corrector_num_params()
        self.s_out = 0.05
        self._base = None       # (mobility, kappa, order, dt_coarse, stages) of set_base
        self._normalized = None  # set_loss

    def set_params(self, params, s_out: float = 0.05) -> None:
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.n_params
        self.s_out = s_out
        _check(lib.gc_corrector_set_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size, s_out))

    def get_params(self):
        import numpy as np
        p = np.empty(self.n_params, dtype=np.float32)
        _check(lib.gc_corrector_get_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def set_base(self, rhs: "CahnHilliardRhs | None", dt_coarse: float = 0.16, stages: int = 6) -> None:
        """Coarse step B(c) + delta over one RKC2 step B of dt_coarse with
        `stages` stages (the network sees B's increment and error indicator);
        None turns the base step off (coarse step c + delta)."""
        _check(lib.gc_corrector_set_base(self.handle, C.byref(rhs.c()) if rhs is not None else None,
                                         dt_coarse, stages))
        self._base = None if rhs is None else (rhs.mobility, rhs.kappa, rhs.order, dt_coarse, stages)

    def set_loss(self, normalized: bool) -> None:
        """normalized: weight each training sample by 1 / mean((target - s)^2),
        s = B(c) with a base step else c."""
        _check(lib.gc_corrector_set_loss(self.handle, 1 if normalized else 0))
        self._normalized = bool(normalized)

    def save(self, path: str, meta: dict | None = None) -> None:
        """Writes the FP32 master parameters (the BF16 tensor-core copies are
        derived from them) as a checkpoint file, with s_out, the base step and
        the loss setting in its metadata."""
        info = dict(meta or {})
        info.update({"kind": "corrector", "n_params": self.n_params, "s_out": self.s_out,
                     "base": list(self._base) if self._base else None, "normalized_loss": self._normalized})
        save_checkpoint(self.get_params(), Grid(self.n_params, 1, 1), path, info)

    def load(self, path: str) -> dict:
        """Restores parameters (and the base step / loss setting when the file
        records them) written by save(); returns the file's metadata."""
        params, _, meta = load_checkpoint(path)
        if meta.get("kind") != "corrector" or meta.get("n_params") != self.n_params:
            raise ValueError(f"gridcalc_b200: {path} does not hold parameters of this corrector")
        self.set_params(params.reshape(-1), s_out=meta["s_out"])
        if meta.get("base"):
            m, k, o, dt_c, st = meta["base"]
            self.set_base(CahnHilliardRhs(m, k, int(o)), dt_c, int(st))
        if meta.get("normalized_loss") is not None:
            self.set_loss(meta["normalized_loss"])
        return meta

    def forward(self, c):
        """Coarse-step increment (B(c) - c + delta with a base step, else the
        zero-mean correction delta) for a (B, H, W) float32/float64 CUDA tensor."""
        import torch
        c = c.contiguous()
        out = torch.empty(c.shape, dtype=torch.float32, device=c.device)
        _check(lib.gc_corrector_forward(self.handle, c.shape[0], _dtype_code(c), c.data_ptr(), out.data_ptr()))
        return out

    def gradient(self, c, target):
        """(gradient, loss) for (B, H, W) CUDA tensors c, target of one dtype."""
        import numpy as np
        if c.dtype != target.dtype:
            raise ValueError("gridcalc_b200: c and target must share a dtype")
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_double()
        _check(lib.gc_corrector_gradient(self.handle, c.shape[0], _dtype_code(c), c.contiguous().data_ptr(),
                                         target.contiguous().data_ptr(),
                                         g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return g, loss.value

    def train_step(self, c, target, lr: float) -> float:
        if c.dtype != target.dtype:
            raise ValueError("gridcalc_b200: c and target must share a dtype")
        loss = C.c_double()
        _check(lib.gc_corrector_train_step(self.handle, c.shape[0], _dtype_code(c), c.contiguous().data_ptr(),
                                           target.contiguous().data_ptr(), lr, C.byref(loss)))
        return loss.value

    def advance(self, psi, grid: Grid, rhs: "CahnHilliardRhs", n_coarse: int, dt_fine: float = 0.01,
                fine_per_coarse: int = 16, residual_tol: float = 0.05, energy_tol: float = 0.0,
                energy_rtol: float = ENERGY_RTOL, try_base: bool = True):
        """n_coarse learned coarse steps of psi (in place), each accepted when
        F rises by at most energy_tol + energy_rtol |F| and the trapezoid
        residual is at most residual_tol; a rejected step is taken by the
        base step alone when that passes the same test (try_base, with a base
        step set), else by plain RK4 steps.  Returns the counts, with the
        network's rejections by cause."""
        pol = gc_corrector_policy(dt_fine, fine_per_coarse, residual_tol, energy_tol, energy_rtol, int(try_base))
        st = gc_corrector_stats()
        _check(lib.gc_corrector_advance(self.handle, C.byref(grid.c()), C.byref(rhs.c()), psi.data_ptr(),
                                        n_coarse, C.byref(pol), C.byref(st)))
        return {"accepted": st.accepted, "fallbacks": st.fallbacks, "rejected_energy": st.rejected_energy,
                "rejected_residual": st.rejected_residual, "accepted_base": st.accepted_base,
                "last_residual": st.last_residual}

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.gc_corrector_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- snapshot output and checkpoints (examples/common/vtk_writer.hpp:34) ---
lib.gc_write_vtk.argtypes = [C.POINTER(gc_grid), C.c_int, C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
lib.gc_write_checkpoint.argtypes = [C.POINTER(gc_grid), C.c_int, C.c_int32, C.c_void_p, C.c_char_p, C.c_char_p]
lib.gc_checkpoint_info.argtypes = [C.c_char_p, C.POINTER(gc_grid), C.POINTER(C.c_int), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_size_t)]
lib.gc_read_checkpoint.argtypes = [C.c_char_p, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t]
lib.gc_load_checkpoint.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t]
lib.gc_snapshotter_create.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
lib.gc_snapshot_vtk.argtypes = [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
lib.gc_snapshot_checkpoint.argtypes = [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_int32, C.c_void_p, C.c_char_p,
                                       C.c_char_p]
lib.gc_snapshotter_flush.argtypes = [C.c_void_p]
lib.gc_snapshotter_destroy.argtypes = [C.c_void_p]
for _f in ("gc_write_vtk", "gc_write_checkpoint", "gc_checkpoint_info", "gc_read_checkpoint", "gc_load_checkpoint",
           "gc_snapshotter_create", "gc_snapshot_vtk", "gc_snapshot_checkpoint", "gc_snapshotter_flush",
           "gc_snapshotter_destroy"):
    getattr(lib, _f).restype = C.c_int


def _host_array(field):
    import numpy as np
    a = field.detach().cpu().numpy() if hasattr(field, "detach") else np.asarray(field)
    a = np.ascontiguousarray(a)
    if a.dtype == np.float64:
        return a, F64
    if a.dtype == np.float32:
        return a, F32
    raise ValueError(f"gridcalc_b200: fields must be float64 or float32, got {a.dtype}")


def _components(n: int, grid: Grid) -> int:
    if n % grid.size:
        raise ValueError(f"gridcalc_b200: field has {n} values, not a multiple of the grid's {grid.size}")
    return n // grid.size


def write_vtk(field, grid: Grid, path: str, name: str = "psi", binary: bool = False) -> None:
    """gridcalc::examples::writeVtkStructuredPoints (examples/common/vtk_writer.hpp:34):
    the reference's ASCII file byte for byte, or the same header with
    big-endian doubles (binary=True).  field: numpy array or tensor."""
    a, dt = _host_array(field)
    if a.size != grid.size:
        raise ValueError(f"gridcalc_b200: field has {a.size} values, grid needs {grid.size}")
    _check(lib.gc_write_vtk(C.byref(grid.c()), dt, a.ctypes.data, os.fsencode(path), name.encode(), int(binary)))


def save_checkpoint(field, grid: Grid, path: str, meta: dict | None = None) -> None:
    """Writes a checkpoint (header, JSON metadata, the field's planes)."""
    import json
    a, dt = _host_array(field)
    _check(lib.gc_write_checkpoint(C.byref(grid.c()), dt, _components(a.size, grid), a.ctypes.data,
                                   os.fsencode(path), json.dumps(meta or {}).encode()))


def checkpoint_info(path: str):
    """(Grid, 'f64' | 'f32', components, metadata length) of a checkpoint."""
    g, dt, comps, mlen = gc_grid(), C.c_int(), C.c_int32(), C.c_size_t()
    _check(lib.gc_checkpoint_info(os.fsencode(path), C.byref(g), C.byref(dt), C.byref(comps), C.byref(mlen)))
    return Grid(g.nx, g.ny, g.nz, g.hx, g.hy, g.hz), ("f64" if dt.value == F64 else "f32"), comps.value, mlen.value


def load_checkpoint(path: str, device=None, ctx=None):
    """Reads a checkpoint: (field, Grid, metadata dict).  device None: a numpy
    array; a CUDA device: a tensor filled on the context's stream."""
    import json
    import numpy as np
    grid, dts, comps, mlen = checkpoint_info(path)
    shape = grid.shape if comps == 1 else (comps,) + grid.shape
    meta = C.create_string_buffer(mlen + 1)
    if device is None:
        a = np.empty(shape, dtype=np.float64 if dts == "f64" else np.float32)
        _check(lib.gc_read_checkpoint(os.fsencode(path), a.ctypes.data, a.nbytes, meta, mlen + 1))
        return a, grid, json.loads(meta.value.decode() or "{}")
    import torch
    t = torch.empty(shape, dtype=torch.float64 if dts == "f64" else torch.float32, device=device)
    _check(lib.gc_load_checkpoint(_ctx(ctx), os.fsencode(path), t.data_ptr(), t.numel() * t.element_size(), meta,
                                  mlen + 1))
    return t, grid, json.loads(meta.value.decode() or "{}")


class Snapshotter:
    """Snapshots of device fields that overlap the computation: each call
    copies the field into a device slot on the context's stream and
    returns; the slot reaches pinned host memory on a copy stream and a
    writer thread writes the file.  ``flush()`` waits for every file."""

    def __init__(self, depth: int = 2, ctx=None):
        self._ctx = ctx or context()
        self.handle = C.c_void_p()
        _check(lib.gc_snapshotter_create(self._ctx.handle, depth, C.byref(self.handle)))

    def vtk(self, field, grid: Grid, path: str, name: str = "psi", binary: bool = False) -> None:
        _require(field, grid)
        _check(lib.gc_snapshot_vtk(self.handle, C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                                   os.fsencode(path), name.encode(), int(binary)))

    def checkpoint(self, field, grid: Grid, path: str, meta: dict | None = None) -> None:
        import json
        if not field.is_cuda or not field.is_contiguous():
            raise ValueError("gridcalc_b200: snapshots take contiguous CUDA tensors")
        _check(lib.gc_snapshot_checkpoint(self.handle, C.byref(grid.c()), _dtype_code(field),
                                          _components(field.numel(), grid), field.data_ptr(), os.fsencode(path),
                                          json.dumps(meta or {}).encode()))

    def flush(self) -> None:
        _check(lib.gc_snapshotter_flush(self.handle))

    def close(self) -> None:
        if self.handle:
            h, self.handle = self.handle, C.c_void_p()
            _check(lib.gc_snapshotter_destroy(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            if self.handle:
                lib.gc_snapshotter_destroy(self.handle)
        except Exception:
            pass


# --- spectral derivatives (spectral/Derivatives.hpp) ----------------------
for _f, _args in (("gc_spectral_partial", [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p]),
                  ("gc_spectral_laplacian", [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_void_p, C.c_void_p]),
                  ("gc_spectral_biharmonic", [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_void_p, C.c_void_p]),
                  ("gc_spectral_gradient", [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_void_p, C.c_void_p])):
    getattr(lib, _f).argtypes = _args
    getattr(lib, _f).restype = C.c_int


def spectral_partial(field, grid: Grid, counts, out=None, ctx=None):
    """spectral::partial<ax, ay, az> (spectral/Derivatives.hpp:78-134): the
    FFT derivative d^(ax+ay+az) f / dx^ax dy^ay dz^az of a float64 field."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    ax, ay, az = counts
    _check(lib.gc_spectral_partial(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), ax, ay, az, field.data_ptr(),
                                   out.data_ptr()))
    return out


def spectral_laplacian(field, grid: Grid, out=None, ctx=None):
    """spectral::laplacian (spectral/Derivatives.hpp:144-172)."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    _check(lib.gc_spectral_laplacian(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                                     out.data_ptr()))
    return out


def spectral_biharmonic(field, grid: Grid, out=None, ctx=None):
    """spectral::biharmonic (spectral/Derivatives.hpp:175-204)."""
    _require(field, grid)
    out = _empty_like_grid(field, grid) if out is None else out
    _check(lib.gc_spectral_biharmonic(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                                      out.data_ptr()))
    return out


def spectral_gradient(field, grid: Grid, out=None, ctx=None):
    """spectral::gradient (spectral/Derivatives.hpp:207-240); out (3, nz, ny, nx)."""
    _require(field, grid)
    out = _empty_like_grid(field, grid, 3) if out is None else out
    _check(lib.gc_spectral_gradient(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), field.data_ptr(),
                                    out.data_ptr()))
    return out


# --- non-finite detection ----------------------------------------------------
lib.gc_check_finite.argtypes = [C.c_void_p, C.POINTER(gc_grid), C.c_int, C.c_int32, C.c_void_p,
                                C.POINTER(C.c_int64)]
lib.gc_check_finite.restype = C.c_int


def check_finite(field, grid: Grid, ctx=None) -> None:
    """Raises GcError (status GC_ERR_NONFINITE, the message naming the value
    and its cell) when the device field holds a NaN or an infinity."""
    if not field.is_cuda or not field.is_contiguous():
        raise ValueError("gridcalc_b200: fields must be contiguous CUDA tensors")
    first = C.c_int64(-1)
    _check(lib.gc_check_finite(_ctx(ctx), C.byref(grid.c()), _dtype_code(field), _components(field.numel(), grid),
                               field.data_ptr(), C.byref(first)))


# --- seeded initial condition (makeRandomIc) ---------------------------------
lib.gc_random_ic.argtypes = [C.POINTER(gc_grid), C.c_uint64, C.c_double, C.c_int32, C.c_void_p]
lib.gc_random_ic.restype = C.c_int


def random_ic(grid: Grid, seed: int, amplitude: float, subtract_mean: bool = True):
    """makeRandomIc (examples/common/cahn_hilliard.hpp:85-103): one draw per
    cell of uniform_real_distribution(-amplitude, amplitude) over
    mt19937_64(seed), in flat index order, the mean subtracted (or, with
    subtract_mean=False, the raw draws: 0 plus i.i.d. uniform noise).
    Returns a host float64 array of shape (nz, ny, nx)."""
    import numpy as np
    out = np.empty(grid.shape, dtype=np.float64)
    _check(lib.gc_random_ic(C.byref(grid.c()), C.c_uint64(seed), float(amplitude), int(bool(subtract_mean)),
                            out.ctypes.data))
    return out
