"""func::evaluate with general callables on the GPU (gc_evaluate_program):
every arity of the reference's scalar and Vec3d forms
(func/Functional.hpp:88-148, :183-220), double results bit-identical to the
oracle and to the reference's golden values, float storage bit-identical to
the oracle on the same float values, the compensated tag within a stated
tolerance, and the host-side rules (extent order, malformed programs)."""
import ctypes as C
import os

import numpy as np
import pytest

import integrand_cases as IC

pytestmark = pytest.mark.gpu

GRIDS = [((9, 10, 12), (0.3, 0.25, 0.5)), ((1, 9, 17), (1.0, 1.0, 1.0)), ((8, 8, 40), (0.5, 1.0, 2.0)),
         ((33, 34, 35), (0.7, 0.9, 1.1)), ((5, 5, 5), (1.0, 1.0, 1.0))]


def _dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


def _grid(gc, shape, h):
    return gc.Grid(shape[-1], shape[-2], shape[-3], *h)


@pytest.mark.parametrize("name", list(IC.CASES))
def test_bit_exact_vs_oracle(gc, oracle, name):
    comps, fn = IC.CASES[name]
    prog = IC.program(name)
    rng = np.random.default_rng(sum(map(ord, name)))
    for shape, h in GRIDS:
        field = rng.standard_normal(shape if comps == 1 else (3,) + shape)
        want = oracle.evaluate_program(comps, prog.arity, prog.instr, field, h)
        assert gc.evaluate(_dev(field), _grid(gc, shape, h), fn) == want, (name, shape)
        # A traced Program is accepted as it is.
        assert gc.evaluate(_dev(field), _grid(gc, shape, h), prog) == want


def test_golden_values(gc):
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz"))
    from gridcalc_b200 import integrand
    for g in ("aniso3d", "flat2d", "cube7"):
        f, v, h = golden[f"{g}/f"], golden[f"{g}/v"], tuple(golden[f"{g}/h"])
        for name in IC.CASES:
            comps, arity = (int(x) for x in golden[f"program/{name}_shape"])
            prog = integrand.Program(comps, arity, [tuple(r) for r in golden[f"program/{name}"]])
            prog.instr = [(int(o), int(d), int(a), int(b), float(val)) for o, d, a, b, val in prog.instr]
            src = f if comps == 1 else v
            got = gc.evaluate(_dev(src), _grid(gc, src.shape, h), prog)
            assert got == float(golden[f"{g}/evaluate_{name}"]), (g, name)


def test_float_storage_is_exact_on_float_values(gc, oracle):
    """Float fields are promoted to double on load, so the result is the
    oracle's on the float-rounded values, bit for bit."""
    import torch
    rng = np.random.default_rng(2)
    shape, h = (20, 24, 28), (0.5, 0.25, 1.0)
    for name, (comps, fn) in IC.CASES.items():
        field = rng.standard_normal(shape if comps == 1 else (3,) + shape).astype(np.float32)
        prog = IC.program(name)
        want = oracle.evaluate_program(comps, prog.arity, prog.instr, field.astype(np.float64), h)
        assert gc.evaluate(_dev(field, torch.float32), _grid(gc, shape, h), fn) == want, name


def test_kahan_tag_within_tolerance(gc, oracle):
    """The device compensated sum is deterministic but not the reference's
    sequential Neumaier order: agreement to a few ulps of the sum of |f|."""
    rng = np.random.default_rng(4)
    shape, h = (40, 48, 56), (1.0, 1.0, 1.0)
    for name, (comps, fn) in IC.CASES.items():
        field = rng.standard_normal(shape if comps == 1 else (3,) + shape)
        prog = IC.program(name)
        want = oracle.evaluate_program(comps, prog.arity, prog.instr, field, h, kahan=True)
        got = gc.evaluate(_dev(field), _grid(gc, shape, h), fn, tag=gc.Kahan)
        # Both sums are compensated: their error is a few ulps of the result.
        assert abs(got - want) <= 1e-13 * abs(want) + 1e-15, name
        assert got == gc.evaluate(_dev(field), _grid(gc, shape, h), fn, tag=gc.Kahan)   # deterministic


def test_program_matches_fixed_integrand_at_scale(gc):
    """At 256^3 the recorded free energy equals the dedicated device
    integrand (same operations, same pairwise tree), bit for bit."""
    import torch
    n = 256
    g = gc.Grid(n, n, n, 0.5, 0.5, 0.5)
    psi = 0.1 * torch.randn((n, n, n), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    a = gc.evaluate(psi, g, lambda p, d: -0.5 * p * p + 0.25 * p * p * p * p + 0.5 * 0.7 * d.squaredNorm())
    b = gc.evaluate(psi, g, "ch_free_energy", kappa=0.7)
    assert a == b


def test_extent_checks_follow_the_reference_order(gc, oracle):
    """Arity 4 checks the gradient (radius 1) before the biharmonic
    (radius 2): on nx = 4, ny = 2 the reference reports axis y."""
    shape = (8, 2, 4)
    f = np.zeros(shape)
    fn = lambda p, g, lap, bih: bih  # noqa: E731
    with pytest.raises(ValueError, match="axis y") as ei:
        gc.evaluate(_dev(f), _grid(gc, shape, (1.0, 1.0, 1.0)), fn)
    assert ei.value.status == "GC_ERR_AXIS_EXTENT"
    prog = IC.integrand.trace(fn)
    with pytest.raises(ValueError, match="axis y"):
        oracle.evaluate_program(1, 4, prog.instr, f)
    # arity 1 needs no neighbours: any extent
    assert gc.evaluate(_dev(f), _grid(gc, shape, (1.0, 1.0, 1.0)), lambda p: p * p) == 0.0


def _raw(gc, comps, arity, rows):
    p = gc.gc_program(comps, arity, len(rows), 0)
    for k, r in enumerate(rows):
        p.instr[k] = gc.gc_instr(*r)
    return p


@pytest.mark.parametrize("comps,arity,rows,msg", [
    (1, 1, [(11, 0, 0, 0, 0.0)], "unknown opcode"),
    (1, 1, [(2, 0, 1, 2, 0.0)], "read before it is written"),
    (1, 1, [(1, 0, 1, 0, 0.0)], "not available at arity"),
    (3, 1, [(1, 0, 3, 0, 0.0)], "not available at arity"),
    (1, 5, [(0, 0, 0, 0, 1.0)], "arity"),
    (2, 1, [(0, 0, 0, 0, 1.0)], "components"),
    (1, 1, [], "n_instr"),
    (1, 1, [(0, 32, 0, 0, 1.0)], "destination"),
])
def test_malformed_programs_are_rejected(gc, comps, arity, rows, msg):
    shape = (4, 4, 4)
    field = _dev(np.zeros((3,) + shape if comps == 3 else shape))
    p = _raw(gc, comps, arity, rows)
    r = C.c_double()
    st = gc.lib.gc_evaluate_program(gc.context().handle, C.byref(_grid(gc, shape, (1, 1, 1)).c()), gc.F64,
                                    field.data_ptr(), C.byref(p), 0, C.byref(r))
    assert gc.STATUS[st] == "GC_ERR_INVALID_ARG"
    assert msg in gc.lib.gc_last_error().decode()


def test_non_finite_values_propagate_like_the_reference(gc, oracle):
    """An infinite value: the zero-weight centre tap of the gradient gives
    0 * inf = NaN in the reference's sum, and so here; a value-only
    integrand keeps the infinity."""
    import math
    shape, h = (6, 7, 8), (1.0, 1.0, 1.0)
    f = np.random.default_rng(8).standard_normal(shape)
    f[3, 4, 5] = np.inf
    g = _grid(gc, shape, h)
    grad_only = lambda p, d: d[0] * d[0]  # noqa: E731
    want = oracle.evaluate_program(1, 2, IC.integrand.trace(grad_only).instr, f, h)
    got = gc.evaluate(_dev(f), g, grad_only)
    assert math.isnan(want) and math.isnan(got)
    assert gc.evaluate(_dev(f), g, lambda p: p) == oracle.evaluate_program(1, 1, IC.integrand.trace(lambda p: p).instr, f, h) == math.inf


from hypothesis import HealthCheck, assume, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402


@settings(max_examples=20, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(data=st.data(), arity=st.integers(1, 4))
def test_random_integrands_bit_exact_vs_oracle(gc, oracle, data, arity):
    """Random expressions over every opcode and input (each a new NVRTC
    compile): the device result is the oracle's, bit for bit, non-finite
    field values included."""
    tree = data.draw(IC.random_tree({1: 1, 2: 4, 3: 5, 4: 6}[arity]))
    fn = IC.tree_callable(tree, arity)
    try:
        prog = IC.integrand.trace(fn)
    except (ZeroDivisionError, ValueError):
        assume(False)
    rng = np.random.default_rng(len(prog.instr) + 17 * arity)
    shape, h = (9, 11, 13), (0.5, 0.75, 1.25)
    field = rng.standard_normal(shape)
    if data.draw(st.integers(0, 4)) == 0:
        field[4, 5, 6] = data.draw(st.sampled_from([np.inf, -np.inf, np.nan]))
    want = oracle.evaluate_program(1, prog.arity, prog.instr, field, h)
    got = gc.evaluate(_dev(field), _grid(gc, shape, h), prog)
    assert got == want or (np.isnan(got) and np.isnan(want)), (prog.instr, got, want)
