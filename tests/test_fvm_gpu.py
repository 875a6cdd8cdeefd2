"""FVM cell Laplacian and the diffusion drivers on the GPU against the oracle
(bit-identical in double) plus the reference's known answers and error
contracts (test/fvm_cell_laplacian_test.cpp, test/fvm_grid_mismatch_test.cpp,
test/diffusion_test.cpp, test/heterogeneous_diffusion_test.cpp)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def grid_of(gc, shape, h=(1.0, 1.0, 1.0)):
    nz, ny, nx = shape
    return gc.Grid(nx, ny, nz, *h)


def test_cell_laplacian_golden(gc):
    golden = np.load(GOLDEN)
    for name in sorted({k.split("/")[0] for k in golden.files if k.endswith("/f")}):
        f, D, h = golden[f"{name}/f"], golden[f"{name}/D"], tuple(golden[f"{name}/h"])
        got = host(gc.cell_laplacian(dev(f), dev(D), grid_of(gc, f.shape, h)))
        assert np.array_equal(got, golden[f"{name}/cell_laplacian"]), name


@pytest.mark.parametrize("shape", [(1, 50, 70), (20, 33, 40), (9, 1, 12)])
def test_cell_laplacian_bit_exact(gc, oracle, shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    D = np.exp(rng.standard_normal(shape))
    h = (0.5, 0.7, 1.1)
    got = host(gc.cell_laplacian(dev(f), dev(D), grid_of(gc, shape, h)))
    assert np.array_equal(got, oracle.cell_laplacian(f, D, h))


def test_harmonic_mean_known_answer(gc):
    psi = dev(np.array([0.0, 1.0, 1.0, 0.0]).reshape(1, 1, 4))
    D = dev(np.array([1.0, 4.0, 4.0, 1.0]).reshape(1, 1, 4))
    out = host(gc.cell_laplacian(psi, D, gc.Grid(4, 1, 1))).ravel()
    np.testing.assert_allclose(out, [1.6, -1.6, -1.6, 1.6], rtol=4 * np.finfo(float).eps)


def test_constant_d_matches_scaled_laplacian(gc):
    """test/fvm_cell_laplacian_test.cpp:30-70: constant D gives c * lap."""
    rng = np.random.default_rng(2)
    shape = (16, 16, 16)
    f = rng.standard_normal(shape)
    g = grid_of(gc, shape, (0.5, 0.5, 0.5))
    a = host(gc.cell_laplacian(dev(f), dev(np.full(shape, 2.5)), g))
    b = host(gc.laplacian(dev(f), g, 2))
    assert np.abs(a - 2.5 * b).max() <= 1e-12 * np.abs(b).max()


def test_nonpositive_d_names_flat_index(gc):
    g = gc.Grid(8, 8, 8)
    D = np.ones(g.shape)
    D[4, 3, 2] = 0.0
    D[6, 0, 0] = -1.0
    with pytest.raises(ValueError, match="flat index 282") as ei:
        gc.cell_laplacian(dev(np.zeros(g.shape)), dev(D), g)
    assert ei.value.status == "GC_ERR_NONPOSITIVE_D"
    with pytest.raises(ValueError, match="solve::diffuse"):
        gc.diffuse(dev(np.zeros(g.shape)), g, dev(D), 0.001, 1, gc.ExplicitEuler)


def test_diffuse_golden(gc):
    golden = np.load(GOLDEN)
    u0, D = golden["diff/u0"], golden["diff/D"]
    g = grid_of(gc, u0.shape)
    t = dev(u0)
    gc.diffuse(t, g, dev(D), 0.05, 10, gc.RK4)
    assert np.array_equal(host(t), golden["diff/fvm_rk4"])
    t = dev(u0)
    gc.diffuse(t, g, dev(D), 0.05, 10, gc.ExplicitEuler)
    assert np.array_equal(host(t), golden["diff/fvm_euler"])
    t = dev(u0)
    gc.diffuse(t, g, 0.7, 0.05, 10, gc.RK4)
    assert np.array_equal(host(t), golden["diff/const_rk4"])


@pytest.mark.parametrize("steps", [1, 64, 101])
def test_diffuse_fvm_bit_exact(gc, oracle, steps):
    rng = np.random.default_rng(steps)
    shape = (16, 24, 20)
    u0 = rng.random(shape)
    D = np.exp(0.5 * rng.standard_normal(shape))
    dmax = oracle.d_max_face(D)
    dt = 0.5 * 0.6963 / (dmax * 3.0)
    t = dev(u0)
    gc.diffuse(t, grid_of(gc, shape), dev(D), dt, steps, gc.RK4)
    assert np.array_equal(host(t), oracle.diffuse_fvm(u0, D, dt, steps))


def test_diffuse_fvm_float32_mass_and_error(gc, oracle):
    """FP32 storage, FP64 mass: mass drift after 200 RK4 steps and error
    against the FP64 oracle, stated as bounds."""
    import torch
    rng = np.random.default_rng(77)
    shape = (32, 32, 32)
    u0 = rng.random(shape).astype(np.float32).astype(np.float64)
    D = np.exp(0.5 * rng.standard_normal(shape)).astype(np.float32).astype(np.float64)
    dt = 0.5 * 0.6963 / (oracle.d_max_face(D) * 3.0)
    g = grid_of(gc, shape)
    t = dev(u0, torch.float32)
    m0 = gc.integrate(t, g, gc.Kahan)
    gc.diffuse(t, g, dev(D, torch.float32), dt, 200, gc.RK4)
    m1 = gc.integrate(t, g, gc.Kahan)
    assert abs(m1 - m0) / abs(m0) < 1e-5
    want = oracle.diffuse_fvm(u0, D, dt, 200)
    err = np.linalg.norm(host(t) - want) / np.linalg.norm(want)
    assert err < 1e-5, err


def test_cfl_violation(gc):
    g = gc.Grid(8, 8, 8)
    t = dev(np.zeros(g.shape))
    with pytest.raises(ValueError, match="solve::diffuse") as ei:
        gc.diffuse(t, g, 1.0, 0.5, 1, gc.RK4)
    assert ei.value.status == "GC_ERR_CFL"
    with pytest.raises(ValueError, match="solve::diffuse"):
        gc.diffuse(t, g, dev(np.full(g.shape, 3.0)), 0.5, 1, gc.RK4)


def test_diffusion_decay_rate(gc):
    """test/diffusion_test.cpp:46-71: sin x sin y sin z decays as exp(-3 D t)."""
    n = 32
    h = 2 * np.pi / n
    x = np.arange(n) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.ascontiguousarray((np.sin(X) * np.sin(Y) * np.sin(Z)).transpose(2, 1, 0))
    D, dt, steps = 0.5, 0.01, 100
    t = dev(f)
    gc.diffuse(t, gc.Grid(n, n, n, h, h, h), D, dt, steps, gc.RK4)
    ratio = host(t).max() / f.max()
    assert abs(ratio - np.exp(-3 * D * dt * steps)) < 5e-3
