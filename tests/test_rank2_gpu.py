"""Rank-2 gradient (Vec3d -> Mat3d, diff/Gradient.hpp:100-137) and
rank-lowering divergence (Mat3d -> Vec3d, diff/Divergence.hpp:100-135) on
the GPU: double results bit-identical to the oracle and to the reference's
golden vectors, float within stated tolerance, and the reference suite's
known-answer checks (test/vector_tensor_test.cpp) restated on the device."""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = [((9, 10, 12), (0.3, 0.25, 0.5)), ((1, 9, 17), (1.0, 1.0, 1.0)), ((8, 8, 40), (0.5, 1.0, 2.0)),
         ((40, 12, 10), (1.0, 1.0, 1.0)), ((33, 34, 35), (0.7, 0.9, 1.1))]


def _dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def _grid(gc, shape, h):
    return gc.Grid(shape[-1], shape[-2], shape[-3], *h)


@pytest.mark.parametrize("order", [2, 4, 6])
def test_bit_exact_vs_oracle(gc, oracle, order):
    rng = np.random.default_rng(13 + order)
    for shape, h in GRIDS:
        r = order // 2
        if any(1 < n < 2 * r + 1 for n in shape):
            continue
        g = _grid(gc, shape, h)
        v = rng.standard_normal((3,) + shape)
        m = rng.standard_normal((3, 3) + shape)
        got = _host(gc.gradient(_dev(v), g, order))
        assert got.shape == (3, 3) + shape
        assert np.array_equal(got, oracle.op("gradient_vec", order, v, h)), (shape, order)
        got = _host(gc.divergence(_dev(m), g, order))
        assert got.shape == (3,) + shape
        assert np.array_equal(got, oracle.op("divergence_mat", order, m, h)), (shape, order)


def test_golden_vectors(gc):
    """Outputs of the reference itself (tests/golden/make_golden.py)."""
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz"))
    for name in ("aniso3d", "flat2d", "cube7"):
        v, m, h = golden[f"{name}/v"], golden[f"{name}/m"], tuple(golden[f"{name}/h"])
        g = _grid(gc, v.shape, h)
        for order in (2, 4):
            assert np.array_equal(_host(gc.gradient(_dev(v), g, order)), golden[f"{name}/gradient_vec{order}"])
            assert np.array_equal(_host(gc.divergence(_dev(m), g, order)), golden[f"{name}/divergence_mat{order}"])


def test_float32_within_tolerance(gc, oracle):
    import torch
    rng = np.random.default_rng(5)
    shape, h = (20, 24, 28), (0.5, 0.25, 1.0)
    g = _grid(gc, shape, h)
    v = rng.standard_normal((3,) + shape)
    m = rng.standard_normal((3, 3) + shape)
    for order in (2, 4, 6):
        want = oracle.op("gradient_vec", order, v, h)
        got = _host(gc.gradient(_dev(v, torch.float32), g, order))
        # float32 tap sums: a few ulps of the largest term, scaled by 1/h
        assert np.max(np.abs(got - want)) <= 2e-5 * np.max(np.abs(want)), order
        want = oracle.op("divergence_mat", order, m, h)
        got = _host(gc.divergence(_dev(m, torch.float32), g, order))
        assert np.max(np.abs(got - want)) <= 2e-5 * np.max(np.abs(want)), order


def test_out_buffers_and_stream_order(gc, oracle):
    """Caller-provided outputs are written in place; the two rank-2 calls
    compose on one stream (div(grad v) without a host sync in between)."""
    import torch
    rng = np.random.default_rng(9)
    shape, h = (10, 11, 12), (1.0, 1.0, 1.0)
    g = _grid(gc, shape, h)
    v = rng.standard_normal((3,) + shape)
    M = torch.empty((3, 3) + shape, dtype=torch.float64, device="cuda")
    out = torch.empty((3,) + shape, dtype=torch.float64, device="cuda")
    gc.gradient(_dev(v), g, 4, out=M)
    gc.divergence(M, g, 4, out=out)
    want = oracle.op("divergence_mat", 4, oracle.op("gradient_vec", 4, v, h), h)
    assert np.array_equal(_host(out), want)


def _sample(N, fn, comps):
    h = 2 * math.pi / N
    ax = np.arange(N) * h
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    return np.stack([c for c in fn(x, y, z)]).reshape((comps,) + (N, N, N)), h, (x, y, z)


def test_kat_linear_fields_exact_in_interior(gc):
    """MatGradientTest.OnLinearField / MatDivergenceTest.OnLinearField."""
    a, b, c = 1.5, -0.5, 2.25
    N = 8
    v, h, (x, y, z) = _sample(N, lambda x, y, z: (a * x, b * y, c * z), 3)
    g = gc.Grid(N, N, N, h, h, h)
    M = _host(gc.gradient(_dev(v), g))[:, :, 1:-1, 1:-1, 1:-1]
    want = np.diag([a, b, c])
    assert np.max(np.abs(M - want[:, :, None, None, None])) < 1e-12
    mat = np.zeros((3, 3, N, N, N))
    mat[0, 0], mat[1, 1], mat[2, 2] = a * x, b * y, c * z
    d = _host(gc.divergence(_dev(mat), g))[:, 1:-1, 1:-1, 1:-1]
    assert np.max(np.abs(d - np.array([a, b, c])[:, None, None, None])) < 1e-12


def test_kat_index_convention(gc):
    """MatGradientTest.IndexConvention: v = (sin y, 0, 0) -> only M(0, 1) = cos y."""
    N = 32
    v, h, (x, y, z) = _sample(N, lambda x, y, z: (np.sin(y), 0 * x, 0 * x), 3)
    M = _host(gc.gradient(_dev(v), gc.Grid(N, N, N, h, h, h)))
    k0, j0, i0 = 5, 11, 7
    assert abs(M[0, 1, k0, j0, i0] - math.cos(j0 * h)) < 1e-2
    others = [M[r, c, k0, j0, i0] for r in range(3) for c in range(3) if (r, c) != (0, 1)]
    assert max(abs(o) for o in others) < 1e-12


def _mat_grad_err(gc, N, order):
    v, h, (x, y, z) = _sample(N, lambda x, y, z: (np.sin(x), np.sin(y), np.sin(z)), 3)
    M = _host(gc.gradient(_dev(v), gc.Grid(N, N, N, h, h, h), order))
    ref = np.zeros_like(M)
    ref[0, 0], ref[1, 1], ref[2, 2] = np.cos(x), np.cos(y), np.cos(z)
    return np.max(np.abs(M - ref))


def _mat_div_err(gc, N):
    def field(x, y, z):
        return (np.sin(x), np.sin(y), np.sin(z), np.cos(2 * x), np.cos(2 * y), np.cos(2 * z),
                np.sin(x) * np.cos(y), np.sin(y) * np.cos(z), np.sin(z) * np.cos(x))
    m, h, (x, y, z) = _sample(N, field, 9)
    d = _host(gc.divergence(_dev(m.reshape((3, 3, N, N, N))), gc.Grid(N, N, N, h, h, h)))
    ref = np.stack([np.cos(x) + np.cos(y) + np.cos(z),
                    -2 * np.sin(2 * x) - 2 * np.sin(2 * y) - 2 * np.sin(2 * z),
                    np.cos(x) * np.cos(y) + np.cos(y) * np.cos(z) + np.cos(z) * np.cos(x)])
    return np.max(np.abs(d - ref))


def _div_grad_err(gc, N):
    fn = lambda x, y, z: (np.sin(x) * np.cos(y), np.sin(y) * np.cos(z), np.sin(z) * np.cos(x))  # noqa: E731
    v, h, _ = _sample(N, fn, 3)
    g = gc.Grid(N, N, N, h, h, h)
    lap = _host(gc.divergence(gc.gradient(_dev(v), g), g))
    return np.max(np.abs(lap + 2 * v))


@pytest.mark.parametrize("err", ["grad", "div", "divgrad"])
def test_kat_convergence_order2(gc, err):
    """MatGradientTest / MatDivergenceTest.ConvergenceOrder2 and
    VectorIdentityTest.DivergenceOfGradientEqualsLaplacian: slopes in [1.7, 2.3]."""
    f = {"grad": lambda N: _mat_grad_err(gc, N, 2), "div": lambda N: _mat_div_err(gc, N),
         "divgrad": lambda N: _div_grad_err(gc, N)}[err]
    e16, e32, e64 = f(16), f(32), f(64)
    for s in (math.log2(e16 / e32), math.log2(e32 / e64)):
        assert 1.7 < s < 2.3, (err, e16, e32, e64)


def test_kat_order4_tighter(gc):
    """MatGradientTest.Order4IsTighterThanOrder2."""
    assert _mat_grad_err(gc, 32, 4) < _mat_grad_err(gc, 32, 2) / 5.0


def test_kat_hessian_symmetric_and_trace(gc):
    """VectorIdentityTest.HessianIsSymmetric and TraceOfGradientEqualsDivergence
    (the trace sums the same three rounded terms in the same order as the
    vector divergence, so the two agree bit for bit here)."""
    N = 32
    h = 2 * math.pi / N
    g = gc.Grid(N, N, N, h, h, h)
    (phi,), _, _ = _sample(N, lambda x, y, z: (np.sin(x) * np.cos(y) * np.sin(z),), 1)
    H = _host(gc.gradient(gc.gradient(_dev(phi), g), g))
    assert max(np.max(np.abs(H[0, 1] - H[1, 0])), np.max(np.abs(H[0, 2] - H[2, 0])),
               np.max(np.abs(H[1, 2] - H[2, 1]))) < 1e-12
    fn = lambda x, y, z: (np.sin(x) * np.cos(y), np.sin(y) * np.cos(z), np.sin(z) * np.cos(x))  # noqa: E731
    v, _, _ = _sample(N, fn, 3)
    M = _host(gc.gradient(_dev(v), g))
    tr = (M[0, 0] + M[1, 1]) + M[2, 2]
    assert np.array_equal(tr, _host(gc.divergence(_dev(v), g)))


@pytest.mark.parametrize("axis,shape", [("x", (8, 8, 2)), ("y", (8, 3, 8)), ("z", (4, 8, 8))])
def test_axis_extent_error(gc, axis, shape):
    """stencil_axis_extent_test.cpp: the rank-2 forms apply the first-derivative radius per axis."""
    g = _grid(gc, shape, (1.0, 1.0, 1.0))
    with pytest.raises(ValueError, match=f"axis {axis}") as ei:
        gc.gradient(_dev(np.zeros((3,) + shape)), g, 6)
    assert ei.value.status == "GC_ERR_AXIS_EXTENT"
    with pytest.raises(ValueError, match=f"axis {axis}"):
        gc.divergence(_dev(np.zeros((3, 3) + shape)), g, 6)
