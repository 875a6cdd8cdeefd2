"""The cluster-resident integrator (one launch of a thread-block cluster for
all steps, state in shared memory) against the oracle and against the
per-stage kernels.

The plain method exactly as configured: 128 x 128, FP64, order 2,
M = kappa = 1, dt = 0.01, 2000 RK4 steps from the reference's own initial
condition generator (mt19937_64, seed 42, U[-0.05, 0.05], no mean
subtraction): bit-identical to the oracle at steps 1, 10, 100 and 2000, and
so are the free energy and the mass.  Then grids around the cluster's
capacity, uneven slabs, every order, Euler, non-unit spacing / M / kappa,
degenerate axes, and float against the double oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def cluster_path(gc):
    """The cluster-resident path is opt-in: on for every test here."""
    ctx = gc.context()
    ctx.set_cluster_stepping(True)
    yield
    ctx.set_cluster_stepping(False)


def dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def test_config1_reference_ic_bit_exact(gc, oracle):
    import torch
    g = gc.Grid(128, 128, 1)
    assert gc.ch_cluster_ctas(g, torch.float64, 2) > 0
    psi0 = gc.random_ic(g, 42, 0.05, subtract_mean=False)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    t = dev(psi0)
    cpu = psi0.copy()
    done = 0
    for target in (1, 10, 100, 2000):
        gc.ch_integrate(t, g, rhs, 0.01, target - done, gc.RK4)
        cpu = oracle.ch_integrate(2, 1.0, 1.0, cpu, 0.01, target - done)
        done = target
        assert np.array_equal(host(t), cpu), target
        assert gc.evaluate(t, g, "ch_free_energy", kappa=1.0) == oracle.ch_free_energy(cpu, 1.0)
        assert gc.integrate(t, g) == oracle.integrate(cpu)


def _ic(shape, seed):
    rng = np.random.default_rng(seed)
    return 0.05 * (2.0 * rng.random(shape) - 1.0)


@pytest.mark.parametrize("nx,ny", [(128, 128), (240, 240), (56, 40), (33, 17), (100, 129), (7, 9), (1, 64),
                                   (64, 1), (300, 8)])
@pytest.mark.parametrize("order", [2, 4, 6])
def test_shapes_orders_bit_exact(gc, oracle, nx, ny, order):
    import torch
    R = order // 2
    if 2 <= nx <= 2 * R or 2 <= ny <= 2 * R:
        pytest.skip("axis extent rejected by requireAxisExtent")
    g = gc.Grid(nx, ny, 1)
    if gc.ch_cluster_ctas(g, torch.float64, order) == 0:
        pytest.skip("does not fit one cluster")
    psi0 = _ic((1, ny, nx), 31 * order + nx + ny)
    dt = {2: 0.01, 4: 0.005, 6: 0.004}[order]
    rhs = gc.CahnHilliardRhs(1.0, 1.0, order)
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 25, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 1.0, 1.0, psi0, dt, 25))
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt / 2, 7, gc.ExplicitEuler)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 1.0, 1.0, psi0, dt / 2, 7, rk4=False))


@pytest.mark.parametrize("order", [2, 4])
def test_non_unit_spacing_mobility_kappa(gc, oracle, order):
    h = (0.9, 1.2, 1.0)
    g = gc.Grid(90, 70, 1, *h)
    psi0 = _ic((1, 70, 90), 5 + order)
    rhs = gc.CahnHilliardRhs(0.8, 1.3, order)
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, 0.002, 13, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.3, psi0, 0.002, 13, h=h))


def test_same_as_stage_kernels(gc):
    """The cluster launch and the per-stage kernels give the same double
    trajectory (order 4: the fused step kernel does not take it), on one
    context switched between the two paths."""
    import torch
    g = gc.Grid(160, 144, 1)
    psi0 = _ic((1, 144, 160), 77)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 4)
    ctx = gc.Context(0, torch.cuda.current_stream().cuda_stream)
    ctx.set_cluster_stepping(True)
    a, b = dev(psi0), dev(psi0)
    gc.ch_integrate(a, g, rhs, 0.005, 40, gc.RK4, ctx=ctx)
    ctx.set_cluster_stepping(False)
    ctx.set_fused_step(False)
    gc.ch_integrate(b, g, rhs, 0.005, 40, gc.RK4, ctx=ctx)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    ctx.close()


def test_float_against_double_oracle(gc, oracle):
    import torch
    g = gc.Grid(200, 200, 1)
    assert gc.ch_cluster_ctas(g, torch.float32, 4) > 0
    psi0 = _ic((1, 200, 200), 9)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 4)
    t = dev(psi0, torch.float32)
    gc.ch_integrate(t, g, rhs, 0.005, 200, gc.RK4)
    want = oracle.ch_integrate(4, 1.0, 1.0, psi0.astype(np.float32).astype(np.float64), 0.005, 200)
    err = np.linalg.norm(host(t) - want) / np.linalg.norm(want)
    assert err < 1e-5, err   # FP32 storage and stencils over 200 steps
