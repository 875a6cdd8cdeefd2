"""Random cases on the GPU against the oracle (hypothesis): grids with
degenerate and regular axes, anisotropic spacings, orders 2, 4 and 6, every
stencil operator and the Cahn-Hilliard integrators; double results must be
bit-identical to the oracle's."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

pytestmark = pytest.mark.gpu

_AXIS = st.one_of(st.just(1), st.integers(9, 40))   # valid for every radius up to 4
_H = st.floats(0.3, 2.0, allow_nan=False)
_OPS = ["laplacian", "gradient", "divergence", "biharmonic", "gradient_vec", "divergence_mat", "partial",
        "cell_laplacian"]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", torch.float64)


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


@settings(max_examples=40, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(data=st.data(), name=st.sampled_from(_OPS), order=st.sampled_from([2, 4, 6]))
def test_random_operators(gc, oracle, data, name, order):
    shape = (data.draw(_AXIS), data.draw(_AXIS), data.draw(_AXIS))
    h = (data.draw(_H), data.draw(_H), data.draw(_H))
    g = gc.Grid(shape[2], shape[1], shape[0], *h)
    rng = np.random.default_rng(data.draw(st.integers(0, 2 ** 32 - 1)))
    f = rng.standard_normal(shape)
    if name in ("laplacian", "gradient", "biharmonic"):
        got = _host(getattr(gc, name)(_dev(f), g, order))
        want = oracle.op(name, order, f, h)
    elif name in ("divergence", "gradient_vec"):
        v = rng.standard_normal((3,) + shape)
        got = _host(gc.divergence(_dev(v), g, order) if name == "divergence" else gc.gradient(_dev(v), g, order))
        want = oracle.op(name, order, v, h)
    elif name == "divergence_mat":
        m = rng.standard_normal((3, 3) + shape)
        got = _host(gc.divergence(_dev(m), g, order))
        want = oracle.op(name, order, m, h)
    elif name == "partial":
        counts = data.draw(st.tuples(st.integers(0, 4), st.integers(0, 4), st.integers(0, 4))
                           .filter(lambda c: 1 <= sum(c) <= 4))
        got = _host(gc.partial(_dev(f), g, counts, order))
        want = oracle.mixed(counts, order, f, h)
    else:
        D = np.exp(rng.standard_normal(shape))
        got = _host(gc.cell_laplacian(_dev(f), _dev(D), g))
        want = oracle.cell_laplacian(f, D, h)
    assert np.array_equal(got, want), (name, order, shape, h)


@settings(max_examples=25, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(data=st.data(), order=st.sampled_from([2, 4, 6]), rk4=st.booleans())
def test_random_cahn_hilliard(gc, oracle, data, order, rk4):
    """2-D grids of random (odd and even) widths, so that the strip, the
    TMA and the plain kernels all occur, and small 3-D grids."""
    if data.draw(st.booleans()):
        shape = (1, data.draw(st.integers(9, 300)), data.draw(st.integers(9, 300)))
    else:
        shape = (data.draw(st.integers(9, 24)), data.draw(st.integers(9, 24)), data.draw(st.integers(9, 24)))
    h = (data.draw(_H), data.draw(_H), 1.0 if shape[0] == 1 else data.draw(_H))
    M, kappa = data.draw(_H), data.draw(_H)
    steps = data.draw(st.integers(1, 20))
    rng = np.random.default_rng(data.draw(st.integers(0, 2 ** 32 - 1)))
    psi0 = 0.05 * (2.0 * rng.random(shape) - 1.0)
    dt = 2e-3 * min(h) ** 4 / (M * max(kappa, 1.0))
    t = _dev(psi0)
    gc.ch_integrate(t, gc.Grid(shape[2], shape[1], shape[0], *h), gc.CahnHilliardRhs(M, kappa, order), dt, steps,
                    gc.RK4 if rk4 else gc.ExplicitEuler)
    want = oracle.ch_integrate(order, M, kappa, psi0, dt, steps, rk4=rk4, h=h)
    assert np.array_equal(_host(t), want), (shape, order, rk4, steps)
