"""Known-answer and property checks restated from the reference's own test
suite, run through the C ABI on the GPU (each cites the test it restates):
RK4's temporal order and its CFL stability gap, the order-4 Laplacian's
convergence and accuracy over order 2, the biharmonic of a Fourier mode,
conservation of the Cahn-Hilliard right-hand side, and positivity, L2
decay and mass conservation of heterogeneous FVM diffusion."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def test_rk4_temporal_order_and_stability_gap(gc):
    """test/integrator_test.cpp (analytic decay, order 4, stability gap): a
    Fourier mode of the discrete heat equation decays as exp(-D mu t); the
    RK4 error shrinks ~16x when dt halves; dt at the CFL bound runs, beyond
    it the driver refuses with the reference's message."""
    n, m, D = 32, 3, 1.0
    h = 1.0 / n
    g = gc.Grid(n, 1, 1, h, 1.0, 1.0)
    x = np.arange(n) * h
    f0 = np.cos(2 * np.pi * m * x).reshape(1, 1, n)
    mu = 4.0 / h ** 2 * math.sin(math.pi * m / n) ** 2      # exact symbol of the order-2 Laplacian
    T = 2e-3
    errs = []
    for steps in (8, 16, 32):
        t = dev(f0)
        gc.diffuse(t, g, D, T / steps, steps, gc.RK4)
        errs.append(np.abs(host(t) - f0 * math.exp(-D * mu * T)).max())
    assert 14.0 < errs[0] / errs[1] < 18.0 and 14.0 < errs[1] / errs[2] < 18.0, errs
    dt_max = 0.6963 / (D * (1 / h ** 2 + 1 + 1))   # RK4 limit on D dt (1/hx^2 + 1/hy^2 + 1/hz^2)
    t = dev(f0)
    gc.diffuse(t, g, D, 0.999 * dt_max, 4, gc.RK4)
    assert np.isfinite(host(t)).all()
    with pytest.raises(gc.GcError) as e:
        gc.diffuse(dev(f0), g, D, 1.01 * dt_max, 4, gc.RK4)
    assert e.value.status == "GC_ERR_CFL" and "solve::diffuse" in str(e.value)


def test_order4_laplacian_convergence_and_accuracy(gc):
    """test/higher_order_test.cpp:104-235: the order-4 Laplacian converges with
    slope 4 and is at least 10x more accurate than order 2 at N = 32."""
    import torch
    errs = {2: [], 4: []}
    sizes = (16, 32, 64)
    for n in sizes:
        h = 1.0 / n
        x = np.arange(n) * h
        f = np.sin(2 * np.pi * x).reshape(1, 1, n)
        exact = -(2 * np.pi) ** 2 * f
        g = gc.Grid(n, 1, 1, h, 1.0, 1.0)
        for order in (2, 4):
            got = host(gc.laplacian(dev(f, torch.float64), g, order))
            errs[order].append(np.abs(got - exact).max())
    slope4 = math.log(errs[4][0] / errs[4][2]) / math.log(sizes[2] / sizes[0])
    slope2 = math.log(errs[2][0] / errs[2][2]) / math.log(sizes[2] / sizes[0])
    assert 3.7 < slope4 < 4.3 and 1.8 < slope2 < 2.2, (slope2, slope4)
    assert errs[4][1] * 10 < errs[2][1]


@pytest.mark.parametrize("order", [2, 4])
def test_biharmonic_of_a_fourier_mode(gc, order):
    """test/phase_8_test.cpp:272-357: the biharmonic of cos(k.x) is |k|^4 cos(k.x)
    up to the stencil's truncation (order 2 / 4 convergence), mixed terms
    included (a 2-D mode)."""
    import torch
    errs = []
    for n in (16, 32, 64):
        h = 1.0 / n
        x = np.arange(n) * h
        X, Y = np.meshgrid(x, x, indexing="xy")
        f = np.cos(2 * np.pi * (2 * X + Y)).reshape(1, n, n)
        k4 = ((2 * np.pi) ** 2 * (4 + 1)) ** 2
        got = host(gc.biharmonic(dev(f, torch.float64), gc.Grid(n, n, 1, h, h, 1.0), order))
        errs.append(np.abs(got - k4 * f).max() / k4)
    slope = math.log(errs[0] / errs[2]) / math.log(4)
    assert abs(slope - order) < 0.4, (errs, slope)


def test_ch_rhs_is_conservative(gc):
    """test/cahn_hilliard_test.cpp:60-78: the right-hand side sums to zero
    (|sum| < 1e-10 max |rhs| n) on a random field, 2-D and 3-D, orders 2/4/6."""
    rng = np.random.default_rng(4)
    for shape in ((1, 48, 40), (12, 16, 20)):
        psi = rng.uniform(-1, 1, shape)
        g = gc.Grid(shape[2], shape[1], shape[0])
        for order in (2, 4, 6):
            if shape[0] > 1 and shape[0] <= order:
                continue
            r = host(gc.ch_rhs(dev(psi), g, gc.CahnHilliardRhs(1.0, 1.3, order)))
            assert abs(r.sum()) < 1e-10 * np.abs(r).max() * r.size, (shape, order)


def test_fvm_diffusion_positivity_l2_decay_mass(gc):
    """test/heterogeneous_diffusion_test.cpp:88-115 and
    fvm_diffusion_acceptance_test.cpp:95-179: with a positive field and a
    heterogeneous positive D, RK4 FVM diffusion keeps the field positive,
    makes its L2 norm non-increasing and conserves mass to 1e-10."""
    rng = np.random.default_rng(8)
    n = 24
    g = gc.Grid(n, n, n)
    u0 = 1.0 + rng.random((n, n, n))
    D = np.exp(0.5 * rng.standard_normal((n, n, n)))
    Dt = dev(D)
    dmax = gc.d_max_face(Dt, g)
    dt = 0.5 * 0.6963 / (dmax * 3 * 4)
    t = dev(u0)
    m0 = float(u0.sum())
    l2 = [float(np.linalg.norm(u0))]
    for _ in range(5):
        gc.diffuse(t, g, Dt, dt, 20, gc.RK4)
        u = host(t)
        assert u.min() > 0
        l2.append(float(np.linalg.norm(u)))
    assert all(b <= a * (1 + 1e-14) for a, b in zip(l2, l2[1:])), l2
    assert abs(u.sum() - m0) / m0 < 1e-10
