"""The CPU oracle is pinned before it is trusted.

1. Against golden vectors produced by the reference itself
   (tests/golden/reference_vectors.npz, made by tests/golden/make_golden.py):
   every operator, integral, RHS and trajectory must be bit-identical.
2. Against the live reference build (oracle/_ref, when present) on fresh
   seeded inputs.
3. Against the known-answer tests of the reference's own test suite,
   restated here (weights, harmonic-mean flux, unit-field volume, error
   message contracts).
4. Order 6 (no reference counterpart): Taylor-moment conditions of the
   tables and the convergence slope against analytic derivatives.
"""
import math
import os

import numpy as np
import pytest

import oracle_lib

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _grids(golden):
    names = sorted({k.split("/")[0] for k in golden.files if k.endswith("/f")})
    return names


# --- 1. golden vectors ----------------------------------------------------
def test_oracle_matches_reference_golden_operators(oracle, golden):
    for g in _grids(golden):
        f, v, D, h = golden[f"{g}/f"], golden[f"{g}/v"], golden[f"{g}/D"], tuple(golden[f"{g}/h"])
        for order in (2, 4):
            for op, src in (("laplacian", f), ("gradient", f), ("divergence", v), ("biharmonic", f)):
                got = oracle.op(op, order, src, h)
                assert np.array_equal(got, golden[f"{g}/{op}{order}"]), (g, op, order)
            got = oracle.ch_rhs(order, 1.3, 0.7, 0.1 * f, h)
            assert np.array_equal(got, golden[f"{g}/ch_rhs{order}"]), (g, "ch_rhs", order)
            assert np.array_equal(oracle.op("gradient_vec", order, v, h), golden[f"{g}/gradient_vec{order}"])
            assert np.array_equal(oracle.op("divergence_mat", order, golden[f"{g}/m"], h),
                                  golden[f"{g}/divergence_mat{order}"])
        assert np.array_equal(oracle.cell_laplacian(f, D, h), golden[f"{g}/cell_laplacian"])
        assert oracle.integrate(f, h, kahan=False) == float(golden[f"{g}/integrate_pairwise"])
        assert oracle.integrate(f, h, kahan=True) == float(golden[f"{g}/integrate_kahan"])
        assert oracle.ch_free_energy(f, 0.8, h) == float(golden[f"{g}/free_energy"])
        assert oracle.ch_gradient_energy(f, h) == float(golden[f"{g}/gradient_energy"])
        assert oracle.ch_mean(f, h) == float(golden[f"{g}/mean"])


def test_oracle_matches_reference_golden_partials(oracle, golden):
    """diff/detail/MultiIndexDerivative.hpp: the 31 named partials, bit for bit."""
    for name, order in (("aniso3d", 4), ("flat2d", 2)):   # the cases tests/golden/make_golden.py stores
        f, h = golden[f"{name}/f"], tuple(golden[f"{name}/h"])
        for c in oracle_lib.PARTIALS:
            got = oracle.mixed(c, order, f, h)
            assert np.array_equal(got, golden[f"{name}/partial{c[0]}{c[1]}{c[2]}_{order}"]), (name, c, order)


def test_oracle_matches_reference_golden_trajectories(oracle, golden):
    psi0 = golden["ch2d/psi0"]
    for order in (2, 4):
        assert np.array_equal(oracle.ch_integrate(order, 1.0, 1.0, psi0, 0.01, 40, rk4=True),
                              golden[f"ch2d/rk4_order{order}"])
        assert np.array_equal(oracle.ch_integrate(order, 1.0, 1.0, psi0, 0.005, 40, rk4=False),
                              golden[f"ch2d/euler_order{order}"])
    assert np.array_equal(oracle.ch_integrate(2, 1.0, 0.5, golden["ch3d/psi0"], 0.005, 20, rk4=True),
                          golden["ch3d/rk4_order2"])
    u0, D = golden["diff/u0"], golden["diff/D"]
    assert np.array_equal(oracle.diffuse_fvm(u0, D, 0.05, 10, rk4=True), golden["diff/fvm_rk4"])
    assert np.array_equal(oracle.diffuse_fvm(u0, D, 0.05, 10, rk4=False), golden["diff/fvm_euler"])
    assert np.array_equal(oracle.diffuse_const(u0, 0.7, 0.05, 10, rk4=True), golden["diff/const_rk4"])


# --- 2. live reference ----------------------------------------------------
@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
def test_oracle_matches_live_reference(oracle):
    ref = oracle_lib.reference()
    rng = np.random.default_rng(7)
    for shape, h in (((5, 13, 11), (0.7, 1.1, 0.9)), ((1, 31, 29), (1.0, 1.0, 1.0)), ((9, 1, 10), (1.0, 1.0, 1.0))):
        f = rng.standard_normal(shape)
        v = rng.standard_normal((3,) + shape)
        for order in (2, 4):
            for op, src in (("laplacian", f), ("gradient", f), ("divergence", v), ("biharmonic", f)):
                r = 2 if op == "biharmonic" and order == 2 else (3 if op == "biharmonic" else order // 2)
                if any(1 < n < 2 * r + 1 for n in shape):
                    continue
                assert np.array_equal(oracle.op(op, order, src, h), ref.op(op, order, src, h)), (shape, op, order)
            if not any(1 < n < order + 1 for n in shape):
                m = rng.standard_normal((3, 3) + shape)
                assert np.array_equal(oracle.op("gradient_vec", order, v, h), ref.op("gradient_vec", order, v, h))
                assert np.array_equal(oracle.op("divergence_mat", order, m, h), ref.op("divergence_mat", order, m, h))
        x = rng.standard_normal(4097)
        g = x.reshape(1, 1, -1)
        assert oracle.integrate(g) == ref.integrate(g)
        assert oracle.integrate(g, kahan=True) == ref.integrate(g, kahan=True)
    psi = ref.make_random_ic((1, 32, 32), 42, 0.05)
    a = oracle.ch_integrate(2, 1.0, 1.0, psi, 0.01, 100)
    b = ref.ch_integrate(2, 1.0, 1.0, psi, 0.01, 100)
    assert np.array_equal(a, b)


# --- 3. known answers from the reference test suite -----------------------
def test_weight_tables_match_reference_headers(oracle):
    # stencil/CentralDifference.hpp:41-74, FirstDerivative.hpp:51-86,
    # ThirdDerivative.hpp:49-84, FourthDerivative.hpp:49-83
    assert np.array_equal(oracle.weights(2, 2), [1.0, -2.0, 1.0])
    assert np.array_equal(oracle.weights(2, 4), [-1 / 12, 4 / 3, -5 / 2, 4 / 3, -1 / 12])
    assert np.array_equal(oracle.weights(1, 2), [-0.5, 0.0, 0.5])
    assert np.array_equal(oracle.weights(1, 4), [1 / 12, -2 / 3, 0.0, 2 / 3, -1 / 12])
    assert np.array_equal(oracle.weights(3, 2), [-0.5, 1.0, 0.0, -1.0, 0.5])
    assert np.array_equal(oracle.weights(3, 4), [1 / 8, -1.0, 13 / 8, 0.0, -13 / 8, 1.0, -1 / 8])
    assert np.array_equal(oracle.weights(4, 2), [1.0, -4.0, 6.0, -4.0, 1.0])
    assert np.array_equal(oracle.weights(4, 4), [-1 / 6, 2.0, -13 / 2, 28 / 3, -13 / 2, 2.0, -1 / 6])


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
@pytest.mark.parametrize("order", [2, 4, 6])
def test_weight_tables_taylor_moments(oracle, kind, order):
    """sum_m w_m m^q / q! = [q == kind] for q < kind + order (the stencil is
    exact on polynomials of that degree); checked in exact rational arithmetic
    for the order-6 tables, which have no reference counterpart."""
    from fractions import Fraction
    w = oracle.weights(kind, order)
    r = (len(w) - 1) // 2
    offs = range(-r, r + 1)
    wf = [Fraction(x).limit_denominator(1000) for x in w]
    for q in range(kind + order):
        s = sum(wm * Fraction(m) ** q for wm, m in zip(wf, offs)) / math.factorial(q)
        assert s == (1 if q == kind else 0), (kind, order, q, s)


def test_fvm_harmonic_mean_known_answer(oracle):
    # test/fvm_cell_laplacian_test.cpp:90-120: D = [1,4,4,1], psi = [0,1,1,0]
    psi = np.array([0.0, 1.0, 1.0, 0.0]).reshape(1, 1, 4)
    D = np.array([1.0, 4.0, 4.0, 1.0]).reshape(1, 1, 4)
    out = oracle.cell_laplacian(psi, D).ravel()
    np.testing.assert_allclose(out, [1.6, -1.6, -1.6, 1.6], rtol=4 * np.finfo(float).eps)


def test_integrate_unit_field_is_volume(oracle):
    # test/integrate_test.cpp:31-47
    ones = np.ones((4, 16, 8))
    h = (0.25, 0.125, 0.5)
    vol = (8 * 0.25) * (16 * 0.125) * (4 * 0.5)
    assert oracle.integrate(ones, h) == pytest.approx(vol, rel=4e-16)
    assert oracle.integrate(ones, h, kahan=True) == pytest.approx(vol, rel=4e-16)


@pytest.mark.parametrize("axis,shape", [("x", (8, 8, 2)), ("y", (8, 3, 8)), ("z", (4, 8, 8))])
def test_axis_extent_message(oracle, axis, shape):
    # test/stencil_axis_extent_test.cpp:214-245: the message names the axis
    with pytest.raises(ValueError, match=f"axis {axis}"):
        oracle.op("laplacian", 4, np.zeros(shape))


def test_cfl_and_positive_d_messages(oracle):
    u = np.zeros((4, 4, 4))
    with pytest.raises(ValueError, match="solve::diffuse"):
        oracle.diffuse_const(u, 1.0, 1.0, 1, rk4=True)
    D = np.ones((4, 4, 4))
    D[1, 2, 3] = 0.0
    with pytest.raises(ValueError, match="flat index"):
        oracle.cell_laplacian(u, D)


# --- 4. order 6 ----------------------------------------------------------
def _analytic(n):
    h = 2 * np.pi / n
    x = np.arange(n) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.sin(X) * np.cos(2 * Y) * np.sin(Z)
    lap = -(1 + 4 + 1) * f
    bih = (1 + 4 + 1) ** 2 * f
    return f.transpose(2, 1, 0).copy(), lap.transpose(2, 1, 0).copy(), bih.transpose(2, 1, 0).copy(), h


@pytest.mark.parametrize("op,expect", [("laplacian", 6), ("biharmonic", 6)])
def test_order6_convergence_slope(oracle, op, expect):
    errs = []
    ns = (16, 32)
    for n in ns:
        f, lap, bih, h = _analytic(n)
        got = oracle.op(op, 6, f, (h, h, h))
        ref = lap if op == "laplacian" else bih
        errs.append(np.abs(got - ref).max())
    slope = math.log(errs[0] / errs[1]) / math.log(ns[1] / ns[0])
    assert abs(slope - expect) < 0.5, (errs, slope)


# --- 2b. live reference, random cases -----------------------------------------
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

_AXIS = st.one_of(st.just(1), st.integers(7, 11))   # valid for every stencil radius up to 3
_H = st.floats(0.3, 2.0, allow_nan=False)
_OPS = ["laplacian", "gradient", "divergence", "biharmonic", "gradient_vec", "divergence_mat", "mixed",
        "cell_laplacian", "ch_rhs", "ch_rk4", "ch_euler", "diffuse_const", "diffuse_fvm", "integrate"]


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
@settings(max_examples=150, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(data=st.data(), name=st.sampled_from(_OPS), order=st.sampled_from([2, 4]))
def test_oracle_matches_live_reference_random(oracle, data, name, order):
    """Random grids (degenerate and regular axes), spacings, orders and
    coefficients: every path function of the oracle gives the reference's
    own result (compiled from its headers) bit for bit."""
    ref = oracle_lib.reference()
    shape = (data.draw(_AXIS), data.draw(_AXIS), data.draw(_AXIS))
    h = (data.draw(_H), data.draw(_H), data.draw(_H))
    rng = np.random.default_rng(data.draw(st.integers(0, 2 ** 32 - 1)))
    f = rng.standard_normal(shape)

    def same(a, b):
        assert np.array_equal(a, b, equal_nan=True), (name, order, shape, h)

    if name in ("laplacian", "gradient", "biharmonic"):
        same(oracle.op(name, order, f, h), ref.op(name, order, f, h))
    elif name in ("divergence", "gradient_vec"):
        v = rng.standard_normal((3,) + shape)
        same(oracle.op(name, order, v, h), ref.op(name, order, v, h))
    elif name == "divergence_mat":
        m = rng.standard_normal((3, 3) + shape)
        same(oracle.op(name, order, m, h), ref.op(name, order, m, h))
    elif name == "mixed":
        counts = data.draw(st.tuples(st.integers(0, 4), st.integers(0, 4), st.integers(0, 4))
                           .filter(lambda c: 2 <= sum(c) <= 4))
        same(oracle.mixed(counts, order, f, h), ref.mixed(counts, order, f, h))
    elif name == "cell_laplacian":
        D = np.exp(rng.standard_normal(shape))
        same(oracle.cell_laplacian(f, D, h), ref.cell_laplacian(f, D, h))
    elif name == "ch_rhs":
        M, kappa = data.draw(_H), data.draw(_H)
        same(oracle.ch_rhs(order, M, kappa, 0.1 * f, h), ref.ch_rhs(order, M, kappa, 0.1 * f, h))
    elif name in ("ch_rk4", "ch_euler"):
        M, kappa = data.draw(_H), data.draw(_H)
        dt = 1e-3 * min(h) ** 4
        rk4 = name == "ch_rk4"
        same(oracle.ch_integrate(order, M, kappa, 0.1 * f, dt, 3, rk4=rk4, h=h),
             ref.ch_integrate(order, M, kappa, 0.1 * f, dt, 3, rk4=rk4, h=h))
    elif name == "diffuse_const":
        D = data.draw(_H)
        dt = 0.05 * min(h) ** 2 / D
        rk4 = data.draw(st.booleans())
        same(oracle.diffuse_const(f, D, dt, 3, rk4=rk4, h=h), ref.diffuse_const(f, D, dt, 3, rk4=rk4, h=h))
    elif name == "diffuse_fvm":
        D = np.exp(0.5 * rng.standard_normal(shape))
        dt = 0.05 * min(h) ** 2 / float(D.max())
        rk4 = data.draw(st.booleans())
        same(oracle.diffuse_fvm(f, D, dt, 3, rk4=rk4, h=h), ref.diffuse_fvm(f, D, dt, 3, rk4=rk4, h=h))
    else:
        x = rng.standard_normal(data.draw(st.integers(1, 5000))).reshape(1, 1, -1)
        assert oracle.integrate(x, h) == ref.integrate(x, h)
        assert oracle.integrate(x, h, kahan=True) == ref.integrate(x, h, kahan=True)
