"""The fused RK4 step kernel (all four stages of a step on a tile with an
8-cell halo in shared memory; one launch per step) against the oracle, bit
for bit: grids with TMA-loaded interior tiles and wrapped edge tiles, partial
last tiles, each of its four tile shapes (32 x 8 and 32 x 16 on grids that
64 x 16 tiles would not spread over every SM, 64 x 16, 64 x 28 on large
grids), the
smallest grid it takes, non-unit spacing / mobility / kappa, step counts
across graph replays; and against the four stage kernels on a larger grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", torch.float64)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture
def ctx(gc):
    """A context with the cluster-resident path off, so that every grid here
    takes the fused step kernel."""
    import torch
    c = gc.Context(0, torch.cuda.current_stream().cuda_stream)
    c.set_cluster_stepping(False)
    yield c
    c.close()


@pytest.mark.parametrize("shape", [(1, 44, 80), (1, 100, 160), (1, 131, 250), (1, 300, 400), (1, 87, 82),
                                   (1, 64, 1030), (1, 33, 48), (1, 40, 50), (1, 128, 128), (1, 256, 256),
                                   (1, 512, 512), (1, 520, 600)])
@pytest.mark.parametrize("steps", [1, 17, 40])
def test_fused_bit_exact(gc, oracle, ctx, shape, steps):
    rng = np.random.default_rng(shape[1] * 7 + shape[2] + steps)
    psi0 = 0.05 * (2.0 * rng.random(shape) - 1.0)
    g = gc.Grid(shape[2], shape[1], 1)
    t = dev(psi0)
    gc.ch_integrate(t, g, gc.CahnHilliardRhs(1.0, 1.0, 2), 0.01, steps, gc.RK4, ctx=ctx)
    assert np.array_equal(host(t), oracle.ch_integrate(2, 1.0, 1.0, psi0, 0.01, steps))
    ctx.synchronize()  # a timed-out TMA wait, if any, is reported here


def test_fused_non_unit(gc, oracle, ctx):
    h = (0.9, 1.2, 1.0)
    rng = np.random.default_rng(5)
    psi0 = 0.3 + 0.05 * (2.0 * rng.random((1, 120, 200)) - 1.0)
    g = gc.Grid(200, 120, 1, *h)
    t = dev(psi0)
    gc.ch_integrate(t, g, gc.CahnHilliardRhs(0.8, 1.3, 2), 0.004, 21, gc.RK4, ctx=ctx)
    assert np.array_equal(host(t), oracle.ch_integrate(2, 0.8, 1.3, psi0, 0.004, 21, h=h))


def test_fused_equals_stage_kernels_large(gc, ctx):
    """A 2048^2 grid (the largest the fused kernel takes): 50 steps equal the
    stage kernels bit for bit."""
    import torch
    n = 2048
    g = gc.Grid(n, n, 1)
    psi0 = torch.from_numpy(gc.random_ic(g, 3, 0.05, subtract_mean=False)).cuda()
    a, b = psi0.clone(), psi0.clone()
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    gc.ch_integrate(a, g, rhs, 0.01, 50, gc.RK4, ctx=ctx)
    ctx.set_fused_step(False)
    gc.ch_integrate(b, g, rhs, 0.01, 50, gc.RK4, ctx=ctx)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
