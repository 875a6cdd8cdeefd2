"""Cahn-Hilliard time stepping on the GPU against the oracle.

The double path is bit-identical to the reference: RHS, RK4 and explicit
Euler trajectories (golden vectors from the reference, plus the oracle on
the plain-method workload: 128 x 128, dt = 0.01, 2000 RK4 steps).  The float
path is compared with the double oracle and its error is stated in the
assertion.  Physics acceptance follows test/cahn_hilliard_test.cpp:101-184.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["cluster", "fused", "stages"])
def stepping_path(request, gc):
    """Every test runs three times: with small 2-D grids in one
    cluster-resident launch (and larger 2-D double order-2 grids one fused
    kernel per RK4 step), with the default paths (the fused step kernel for
    every 2-D double order-2 grid), and with the four stage kernels forced."""
    ctx = gc.context()
    ctx.set_cluster_stepping(request.param == "cluster")
    ctx.set_fused_step(request.param != "stages")
    yield request.param
    ctx.set_cluster_stepping(False)
    ctx.set_fused_step(True)

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


def uniform_ic(shape, seed, amp=0.05, mean=0.0):
    """The plain-method initial condition: mean + U[-amp, amp] i.i.d.,
    generated once on the host and fed identically to both sides."""
    rng = np.random.default_rng(seed)
    return mean + amp * (2.0 * rng.random(shape) - 1.0)


def test_rhs_golden(gc):
    golden = np.load(GOLDEN)
    for name in sorted({k.split("/")[0] for k in golden.files if k.endswith("/f")}):
        f, h = golden[f"{name}/f"], tuple(golden[f"{name}/h"])
        for order in (2, 4):
            got = host(gc.ch_rhs(dev(0.1 * f), grid_of(gc, f.shape, h), gc.CahnHilliardRhs(1.3, 0.7, order)))
            assert np.array_equal(got, golden[f"{name}/ch_rhs{order}"]), (name, order)


def test_trajectories_golden(gc):
    golden = np.load(GOLDEN)
    psi0 = golden["ch2d/psi0"]
    g = grid_of(gc, psi0.shape)
    for order in (2, 4):
        t = dev(psi0)
        gc.ch_integrate(t, g, gc.CahnHilliardRhs(1.0, 1.0, order), 0.01, 40, gc.RK4)
        assert np.array_equal(host(t), golden[f"ch2d/rk4_order{order}"]), order
        t = dev(psi0)
        gc.ch_integrate(t, g, gc.CahnHilliardRhs(1.0, 1.0, order), 0.005, 40, gc.ExplicitEuler)
        assert np.array_equal(host(t), golden[f"ch2d/euler_order{order}"]), order
    p3 = golden["ch3d/psi0"]
    t = dev(p3)
    gc.ch_integrate(t, grid_of(gc, p3.shape), gc.CahnHilliardRhs(1.0, 0.5, 2), 0.005, 20, gc.RK4)
    assert np.array_equal(host(t), golden["ch3d/rk4_order2"])


def test_plain_method_128_bit_exact(gc, oracle):
    """128 x 128, M = kappa = 1, order 2, dt = 0.01, 2000 RK4 steps, FP64:
    every 500 steps the state is bit-identical to the oracle, and so are the
    free energy in the double-well form F_ref + V/4 and the mass."""
    shape = (1, 128, 128)
    psi0 = uniform_ic(shape, 42)
    g = grid_of(gc, shape)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    t = dev(psi0)
    cpu = psi0.copy()
    mass0 = gc.integrate(t, g, gc.Kahan)
    for _ in range(4):
        gc.ch_integrate(t, g, rhs, 0.01, 500, gc.RK4)
        cpu = oracle.ch_integrate(2, 1.0, 1.0, cpu, 0.01, 500)
        assert np.array_equal(host(t), cpu)
        assert gc.evaluate(t, g, "ch_free_energy", kappa=1.0) == oracle.ch_free_energy(cpu, 1.0)
    assert abs(gc.integrate(t, g, gc.Kahan) - mass0) < 1e-10


@pytest.mark.parametrize("order", [2, 4, 6])
@pytest.mark.parametrize("steps", [1, 3, 66, 131])
def test_rk4_orders_and_step_counts(gc, oracle, order, steps):
    """Odd counts and counts beyond one captured graph (64 steps) exercise
    graph replay, direct leftover steps and the final buffer copy."""
    shape = (1, 40, 56)
    psi0 = uniform_ic(shape, order * 100 + steps)
    dt = {2: 0.01, 4: 0.005, 6: 0.004}[order]
    t = dev(psi0)
    gc.ch_integrate(t, grid_of(gc, shape), gc.CahnHilliardRhs(1.0, 1.0, order), dt, steps, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 1.0, 1.0, psi0, dt, steps))


@pytest.mark.parametrize("shape", [(1, 200, 266), (1, 97, 300), (1, 131, 250), (1, 64, 66)])
@pytest.mark.parametrize("order", [2, 4, 6])
def test_2d_tma_tiles_interior_edge_partial(gc, oracle, shape, order):
    """Even-width 2-D grids large enough for interior tiles take the
    TMA-pipelined kernel (interior tiles by TMA, edge and partial tiles by
    wrapped loads); odd widths take the strip kernel.  Both must stay
    bit-identical, for RK4 (all four stage kinds) and Euler, and over enough
    steps that every CTA processes several tiles."""
    psi0 = uniform_ic(shape, 7 * order + shape[2])
    dt = {2: 0.01, 4: 0.005, 6: 0.004}[order]
    rhs = gc.CahnHilliardRhs(1.0, 1.0, order)
    g = grid_of(gc, shape)
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 18, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 1.0, 1.0, psi0, dt, 18))
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt / 2, 5, gc.ExplicitEuler)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 1.0, 1.0, psi0, dt / 2, 5, rk4=False))
    gc.context().synchronize()  # reports a timed-out device wait, if any


@pytest.mark.parametrize("shape", [(1, 36, 260), (1, 37, 130), (1, 70, 132), (1, 41, 382)])
@pytest.mark.parametrize("order", [2, 4])
def test_2d_edges_non_unit(gc, oracle, shape, order):
    """Small even-width grids (the one-column TMA kernel): heights and widths
    at or just above a staged region's, a narrow last tile, and anisotropic
    spacing with M, kappa != 1 (no unit shortcuts); RK4 and Euler."""
    h = (0.9, 1.2, 1.0)
    psi0 = uniform_ic(shape, 11 * order + shape[1])
    dt = {2: 0.004, 4: 0.002}[order]
    rhs = gc.CahnHilliardRhs(0.8, 1.3, order)
    g = grid_of(gc, shape, h)
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 12, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.3, psi0, dt, 12, h=h))
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 4, gc.ExplicitEuler)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.3, psi0, dt, 4, rk4=False, h=h))


@pytest.mark.parametrize("order", [2, 4])
def test_2d_two_column_large_grid(gc, oracle, order):
    """Grids large enough for the two-column kernel (at least ten rounds of
    its tiles per persistent CTA: 126 x 32 tiles in two 512-thread CTAs per
    SM at order 2, 124 x 16 in three 256-thread CTAs at order 4), with a
    partial last tile in x and in y and non-unit h, M, kappa; RK4 (its three
    RHS stages) and Euler, bit-identical to the oracle."""
    import math
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    nx = 4094                                   # even; last tile 62 (order 2) / 2 (order 4) columns
    tx, ty, slots = (126, 32, 2 * sms) if order == 2 else (124, 16, 3 * sms)
    rows = math.ceil(10 * slots / math.ceil(nx / tx))
    shape = (1, (rows - 1) * ty + ty // 2 + 1, nx)   # last tile row partly filled
    h = (0.9, 1.2, 1.0)
    psi0 = uniform_ic(shape, 3 + order)
    dt = {2: 0.004, 4: 0.002}[order]
    rhs = gc.CahnHilliardRhs(0.8, 1.3, order)
    g = grid_of(gc, shape, h)
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 2, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.3, psi0, dt, 2, h=h))
    t = dev(psi0)
    gc.ch_integrate(t, g, rhs, dt, 1, gc.ExplicitEuler)
    assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.3, psi0, dt, 1, rk4=False, h=h))


def test_2d_state_buffer_off_16_byte_boundary(gc, oracle):
    """A state field starting 8 bytes past a 16-byte boundary cannot be a TMA
    source or a 16-byte store target: the stage launches take the plain
    kernels for it, and the result is the same bits."""
    import torch
    shape = (1, 96, 260)
    psi0 = uniform_ic(shape, 5)
    flat = torch.empty(psi0.size + 1, dtype=torch.float64, device="cuda")
    t = flat[1:].view(shape)
    assert t.data_ptr() % 16 == 8
    t.copy_(dev(psi0))
    gc.ch_integrate(t, grid_of(gc, shape), gc.CahnHilliardRhs(1.0, 1.0, 2), 0.01, 10, gc.RK4)
    assert np.array_equal(host(t), oracle.ch_integrate(2, 1.0, 1.0, psi0, 0.01, 10))


def test_3d_and_anisotropic(gc, oracle):
    shape = (12, 10, 14)
    h = (0.9, 1.1, 1.3)
    psi0 = uniform_ic(shape, 8)
    for order, dt in ((2, 0.01), (4, 0.004)):
        t = dev(psi0)
        gc.ch_integrate(t, grid_of(gc, shape, h), gc.CahnHilliardRhs(0.8, 1.2, order), dt, 25, gc.RK4)
        assert np.array_equal(host(t), oracle.ch_integrate(order, 0.8, 1.2, psi0, dt, 25, h=h)), order


def test_float32_error_vs_double_oracle(gc, oracle):
    """FP32 storage and stencils: error against the FP64 oracle after 1000
    steps of the plain method at 128 x 128 (t = 10), stated as relative L2."""
    import torch
    shape = (1, 128, 128)
    psi0 = uniform_ic(shape, 42).astype(np.float32).astype(np.float64)
    t = dev(psi0, torch.float32)
    g = grid_of(gc, shape)
    gc.ch_integrate(t, g, gc.CahnHilliardRhs(1.0, 1.0, 2), 0.01, 1000, gc.RK4)
    want = oracle.ch_integrate(2, 1.0, 1.0, psi0, 0.01, 1000)
    got = host(t)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 1e-3, err
    f_gpu = gc.evaluate(t, g, "ch_free_energy", kappa=1.0)
    f_ref = oracle.ch_free_energy(want, 1.0)
    v4 = g.size * g.cell_volume / 4.0
    assert abs((f_gpu + v4) - (f_ref + v4)) / abs(f_ref + v4) < 1e-3


@pytest.mark.parametrize("shape,order", [((1, 96, 130), 2), ((1, 96, 130), 4), ((1, 40, 134), 6),
                                         ((1, 40, 127), 2), ((1, 33, 71), 4), ((1, 24, 10), 2), ((1, 20, 16), 4)])
def test_float32_tile_paths_vs_double_oracle(gc, oracle, shape, order):
    """Float runs two columns per thread on even widths and one otherwise;
    both, with edge and partial tiles and grids narrower than a tile, stay
    within 1e-4 relative L2 of the FP64 oracle over 200 RK4 steps."""
    import torch
    psi0 = uniform_ic(shape, 7).astype(np.float32).astype(np.float64)
    t = dev(psi0, torch.float32)
    dt = {2: 0.01, 4: 0.006, 6: 0.005}[order]
    gc.ch_integrate(t, grid_of(gc, shape), gc.CahnHilliardRhs(0.9, 1.1, order), dt, 200, gc.RK4)
    want = oracle.ch_integrate(order, 0.9, 1.1, psi0, dt, 200)
    err = np.linalg.norm(host(t) - want) / np.linalg.norm(want)
    assert err < 1e-4, err


@pytest.mark.parametrize("width", [130, 127])
def test_float32_rkc_and_euler_vs_double(gc, width):
    """The RKC2 stages and the Euler step in float (two-column and one-column
    tiles) against the same library steps in double."""
    import torch
    shape = (1, 48, width)
    psi0 = uniform_ic(shape, 9).astype(np.float32).astype(np.float64)
    g = grid_of(gc, shape)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    for run in (lambda x: gc.ch_rkc(x, g, rhs, 0.16, 10, 6),
                lambda x: gc.ch_integrate(x, g, rhs, 0.01, 50, gc.ExplicitEuler)):
        a, b = dev(psi0, torch.float32), dev(psi0)
        run(a)
        run(b)
        err = float(torch.linalg.norm(a.double() - b) / torch.linalg.norm(b))
        assert err < 1e-5, err


def test_acceptance_3d_coarsening(gc, oracle):
    """test/cahn_hilliard_test.cpp:95-184 restated: 24^3, dt = 0.02,
    kappa = 0.5, amplitude 0.1 (mean removed), snapshots after 0, 500, 1000,
    1500 and 2500 RK4 steps: F non-increasing (tolerance 1e-6 |F0| + 1e-9),
    the gradient energy drops by more than 3 % between the last two
    snapshots, the mean moves by less than 1e-10; and the final state is
    bit-identical to the oracle."""
    shape = (24, 24, 24)
    psi0 = uniform_ic(shape, 42, amp=0.1)
    psi0 -= psi0.mean()
    g = grid_of(gc, shape)
    t = dev(psi0)
    rhs = gc.CahnHilliardRhs(1.0, 0.5, 2)
    vol = g.size * g.cell_volume
    F = [gc.evaluate(t, g, "ch_free_energy", kappa=0.5)]
    E = [gc.evaluate(t, g, "grad_squared")]
    m0 = gc.evaluate(t, g, "psi") / vol
    for seg in (500, 500, 500, 1000):
        gc.ch_integrate(t, g, rhs, 0.02, seg, gc.RK4)
        F.append(gc.evaluate(t, g, "ch_free_energy", kappa=0.5))
        E.append(gc.evaluate(t, g, "grad_squared"))
    tol = 1e-6 * abs(F[0]) + 1e-9
    assert all(b <= a + tol for a, b in zip(F, F[1:])), F
    assert (E[3] - E[4]) / E[3] > 0.03, E
    assert abs(gc.evaluate(t, g, "psi") / vol - m0) < 1e-10
    assert np.array_equal(host(t), oracle.ch_integrate(2, 1.0, 0.5, psi0, 0.02, 2500))


def test_constant_field_zero_rhs(gc):
    """test/cahn_hilliard_test.cpp:47-58."""
    g = gc.Grid(16, 16, 16)
    t = dev(np.full(g.shape, 0.3))
    out = host(gc.ch_rhs(t, g, gc.CahnHilliardRhs(1.0, 1.0, 2)))
    assert np.abs(out).max() < 1e-12


def test_errors(gc):
    g = gc.Grid(16, 16, 1)
    t = dev(np.zeros(g.shape))
    with pytest.raises(ValueError, match="n_steps must be >= 0"):
        gc.ch_integrate(t, g, gc.CahnHilliardRhs(), 0.01, -1, gc.RK4)
    with pytest.raises(ValueError, match="dt must be >= 0"):
        gc.ch_integrate(t, g, gc.CahnHilliardRhs(), -0.01, 1, gc.RK4)
    with pytest.raises(ValueError, match="axis x"):
        gc.ch_integrate(dev(np.zeros((1, 16, 4))), gc.Grid(4, 16, 1), gc.CahnHilliardRhs(order=4), 0.01, 1)
