"""RKC2 base step of the learned coarse step: coefficients and stability
(CPU), the library's device step bit for bit against the CPU restatement
driven by the oracle's Cahn-Hilliard RHS, second-order convergence and
stability far beyond the RK4 limit (GPU)."""
import numpy as np
import pytest

import rkc_ref


@pytest.mark.parametrize("s", [2, 3, 5, 8, 16])
def test_rkc_second_order_and_stable_interval(s):
    c = rkc_ref.coeffs(s)
    for z in (1e-3, -1e-3, -1e-2):
        R = rkc_ref.stability_polynomial(s, z)
        assert abs(R - (1 + z + z * z / 2)) < 0.2 * abs(z) ** 3 + 1e-15   # second order
    zz = np.linspace(-c["beta"], 0.0, 1001)
    assert max(abs(rkc_ref.stability_polynomial(s, z)) for z in zz) <= 1.0 + 1e-12
    assert 0.49 * s * s <= c["beta"] <= 0.66 * s * s


def test_library_bound_matches_restatement():
    import ctypes as C
    from test_abi import LIB
    lib = C.CDLL(LIB)
    lib.gc_rkc_stability_bound.restype = C.c_double
    lib.gc_rkc_stability_bound.argtypes = [C.c_int32]
    for s in (2, 3, 4, 5, 6, 8, 10, 16, 64):
        assert lib.gc_rkc_stability_bound(s) == rkc_ref.coeffs(s)["beta"]
    assert lib.gc_rkc_stability_bound(1) == 0.0 and lib.gc_rkc_stability_bound(65) == 0.0


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    return 0.05 * (2 * rng.random(shape) - 1)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,order,s", [((1, 40, 48), 2, 5), ((1, 40, 48), 4, 3), ((1, 33, 37), 2, 2),
                                           ((12, 12, 16), 2, 4), ((12, 12, 16), 4, 6)])
def test_rkc_bit_identical_to_restatement(gc, oracle, shape, order, s):
    import torch
    psi0 = _field(shape, 11 + s)
    t = torch.from_numpy(psi0.copy()).cuda()
    g = gc.Grid(shape[2], shape[1], shape[0])
    dt = 0.5 * rkc_ref.coeffs(s)["beta"] / (80.0 if shape[0] == 1 else 120.0)
    gc.ch_rkc(t, g, gc.CahnHilliardRhs(1.0, 1.0, order), dt, 3, s)
    want = psi0.copy()
    for _ in range(3):
        want = rkc_ref.step(lambda y: oracle.ch_rhs(order, 1.0, 1.0, y), want, dt, s)
    assert np.array_equal(t.cpu().numpy(), want)


@pytest.mark.gpu
def test_rkc_second_order_convergence_and_stability(gc, oracle):
    """Against 64 fine RK4 steps per step: error ratio ~4 when dt halves; at
    dt = 0.16 (beyond RK4's limit ~0.035 on this 2-D order-2 grid) six stages
    stay bounded while RK4 at that dt blows up."""
    import torch
    size = 64
    g = gc.Grid(size, size, 1)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    c = torch.from_numpy(_field((1, size, size), 3)).cuda()
    gc.ch_integrate(c, g, rhs, 0.01, 1500, gc.RK4)   # past the spinodal stage: a smooth pattern
    errs = []
    for dt in (0.04, 0.02, 0.01):
        ref = c.clone()
        gc.ch_integrate(ref, g, rhs, dt / 64, 64 * int(round(0.16 / dt)), gc.RK4)
        x = c.clone()
        gc.ch_rkc(x, g, rhs, dt, int(round(0.16 / dt)), 6)
        errs.append(float(torch.linalg.norm(x - ref) / torch.linalg.norm(ref - c)))
    assert 3.0 < errs[0] / errs[1] < 5.0 and 3.0 < errs[1] / errs[2] < 5.0, errs
    x = c.clone()
    gc.ch_rkc(x, g, rhs, 0.16, 200, 6)
    assert bool(torch.isfinite(x).all()) and float(x.abs().max()) < 1.5
    y = c.clone()
    gc.ch_integrate(y, g, rhs, 0.16, 50, gc.RK4)
    assert not bool(torch.isfinite(y).all()) or float(y.abs().max()) > 10.0
