"""GPU parity of the stencil operators against the CPU oracle and the
reference golden vectors.

Bar: double results are bit-identical to the oracle (which is bit-identical
to the reference); float results are within a stated relative L2 of the
double oracle; order 6 (no reference counterpart) is pinned by analytic
derivatives and a convergence slope.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")
OPS = ("laplacian", "gradient", "divergence", "biharmonic")
# Float storage: relative L2 error of the float result against the double
# oracle on N(0,1) inputs (stencil cancellation amplifies float rounding).
F32_TOL = {"laplacian": 2e-6, "gradient": 1e-6, "divergence": 1e-6, "biharmonic": 5e-6}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_op(gc, op, order, arr, grid, dtype):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr)).to("cuda", dtype)
    out = getattr(gc, op)(t, grid, order)
    torch.cuda.synchronize()
    return out.double().cpu().numpy()


def grid_of(gc, shape, h):
    nz, ny, nx = shape
    return gc.Grid(nx, ny, nz, *h)


def radius(op, order):
    return {"laplacian": order // 2, "gradient": order // 2, "divergence": order // 2,
            "biharmonic": order // 2 + 1}[op]


SHAPES = [((8, 10, 12), (0.3, 0.25, 0.5)), ((1, 9, 17), (1.0, 1.0, 1.0)),
          ((7, 20, 33), (1.0, 1.0, 1.0)), ((24, 40, 70), (0.1, 0.2, 0.3)), ((1, 65, 130), (1.0, 1.0, 1.0)),
          ((9, 1, 11), (1.0, 1.0, 1.0)),
          ((96, 20, 36), (0.5, 0.4, 0.3))]   # several z chunks per column of the 3-D plane ring


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("order", [2, 4, 6])
def test_f64_bit_exact_vs_oracle(gc, oracle, op, order):
    import torch
    rng = np.random.default_rng(100 + order)
    for shape, h in SHAPES:
        r = radius(op, order)
        if any(1 < n < 2 * r + 1 for n in shape):
            continue
        src = rng.standard_normal((3,) + shape if op == "divergence" else shape)
        want = oracle.op(op, order, src, h)
        got = run_op(gc, op, order, src, grid_of(gc, shape, h), torch.float64)
        assert np.array_equal(got, want), (op, order, shape, np.abs(got - want).max())


def test_f64_golden_vectors(gc):
    import torch
    golden = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in golden.files if k.endswith("/f")})
    for g in names:
        f, v, h = golden[f"{g}/f"], golden[f"{g}/v"], tuple(golden[f"{g}/h"])
        grid = grid_of(gc, f.shape, h)
        for order in (2, 4):
            for op, src in (("laplacian", f), ("gradient", f), ("divergence", v), ("biharmonic", f)):
                got = run_op(gc, op, order, src, grid, torch.float64)
                assert np.array_equal(got, golden[f"{g}/{op}{order}"]), (g, op, order)


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("order", [2, 4, 6])
def test_f32_within_tolerance(gc, oracle, op, order):
    import torch
    rng = np.random.default_rng(200 + order)
    shape, h = (24, 40, 70), (0.1, 0.2, 0.3)
    src = rng.standard_normal((3,) + shape if op == "divergence" else shape)
    src32 = src.astype(np.float32).astype(np.float64)  # same input values for both sides
    want = oracle.op(op, order, src32, h)
    got = run_op(gc, op, order, src32, grid_of(gc, shape, h), torch.float32)
    err = rel_l2(got, want)
    assert err < F32_TOL[op] * (3 if order == 6 else 1), (op, order, err)


def _analytic_modes(n, kx=1, ky=2, kz=3):
    h = 2 * np.pi / n
    x = np.arange(n) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.sin(kx * X) * np.cos(ky * Y) * np.sin(kz * Z)
    k2 = kx * kx + ky * ky + kz * kz
    t = lambda a: np.ascontiguousarray(a.transpose(2, 1, 0))
    return t(f), t(-k2 * f), t(k2 * k2 * f), h


@pytest.mark.parametrize("op", ["laplacian", "biharmonic"])
def test_order6_vs_analytic_slope(gc, op):
    import torch
    errs = []
    ns = (32, 64)
    for n in ns:
        f, lap, bih, h = _analytic_modes(n)
        got = run_op(gc, op, 6, f, gc.Grid(n, n, n, h, h, h), torch.float64)
        errs.append(np.abs(got - (lap if op == "laplacian" else bih)).max())
    slope = math.log(errs[0] / errs[1]) / math.log(ns[1] / ns[0])
    assert abs(slope - 6) < 0.5, (errs, slope)


def test_laplacian_eigenfunction_accuracy(gc):
    """test/laplacian_test.cpp:40-64: sin sin sin at N=32, order 2, rel max
    error below 1.5e-2."""
    import torch
    n = 32
    h = 2 * np.pi / n
    x = np.arange(n) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.ascontiguousarray((np.sin(X) * np.sin(Y) * np.sin(Z)).transpose(2, 1, 0))
    got = run_op(gc, "laplacian", 2, f, gc.Grid(n, n, n, h, h, h), torch.float64)
    assert np.abs(got + 3 * f).max() / np.abs(3 * f).max() < 1.5e-2


@pytest.mark.parametrize("axis,shape", [("x", (8, 8, 2)), ("y", (8, 3, 8)), ("z", (4, 8, 8))])
def test_axis_extent_error(gc, axis, shape):
    import torch
    t = torch.zeros(shape, dtype=torch.float64, device="cuda")
    nz, ny, nx = shape
    with pytest.raises(ValueError, match=f"axis {axis}") as ei:
        gc.laplacian(t, gc.Grid(nx, ny, nz), 4)
    assert ei.value.status == "GC_ERR_AXIS_EXTENT"


def test_degenerate_axes_allowed(gc, oracle):
    """N == 1 is a degenerate axis (diff/detail/PreconditionAxisExtent.hpp:64-67)."""
    import torch
    rng = np.random.default_rng(5)
    for shape in ((1, 1, 16), (1, 12, 1), (10, 1, 1)):
        f = rng.standard_normal(shape)
        for order in (2, 4, 6):
            got = run_op(gc, "laplacian", order, f, grid_of(gc, shape, (1, 1, 1)), torch.float64)
            assert np.array_equal(got, oracle.op("laplacian", order, f)), (shape, order)


def test_large_f64_vs_analytic_and_oracle(gc, oracle):
    """A 128^3 grid: bit-exact against the oracle for laplacian order 4."""
    import torch
    n = 128
    rng = np.random.default_rng(9)
    f = rng.standard_normal((n, n, n))
    got = run_op(gc, "laplacian", 4, f, gc.Grid(n, n, n, 1 / n, 1 / n, 1 / n), torch.float64)
    want = oracle.op("laplacian", 4, f, (1 / n, 1 / n, 1 / n))
    assert np.array_equal(got, want)
