"""Integrand programs on the CPU: the oracle's func::evaluate against the
reference's golden values, the recorder (gridcalc_b200.integrand) against
the Python callables it records, and its error rules."""
import os

import numpy as np
import pytest

import integrand_cases as IC

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")
I = IC.integrand


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _inputs(oracle, name, field, h):
    """The callable's arguments at every cell, from the oracle's order-2
    derivative fields (the reference's defaults)."""
    comps, fn = IC.CASES[name]
    arity = I.arity_of(fn)
    if comps == 1:
        ins = [field]
        if arity >= 2:
            ins += list(oracle.op("gradient", 2, field, h))
        if arity >= 3:
            ins.append(oracle.op("laplacian", 2, field, h))
        if arity >= 4:
            ins.append(oracle.op("biharmonic", 2, field, h))
        return ins
    ins = list(field)
    if arity >= 2:
        M = oracle.op("gradient_vec", 2, field, h)
        ins += [M[r, c] for r in range(3) for c in range(3)]
    return ins


def _call(name, ins):
    comps, fn = IC.CASES[name]
    arity = I.arity_of(fn)
    if comps == 1:
        args = [ins[0], I.SymVec3(ins[1:4]) if arity >= 2 else None, ins[4] if arity >= 3 else None,
                ins[5] if arity >= 4 else None][:arity]
    else:
        args = [I.SymVec3(ins[0:3]), I.SymMat3([ins[3 + 3 * r: 6 + 3 * r] for r in range(3)]) if arity >= 2 else None][:arity]
    return fn(*args)


def test_oracle_matches_reference_golden_evaluate(oracle, golden):
    """func::evaluate (func/Functional.hpp:88-220): the oracle's value equals
    the reference's for every arity, scalar and vector, both tags."""
    for g in ("aniso3d", "flat2d", "cube7"):
        f, v, h = golden[f"{g}/f"], golden[f"{g}/v"], tuple(golden[f"{g}/h"])
        for name in IC.CASES:
            rows = golden[f"program/{name}"]
            comps, arity = (int(x) for x in golden[f"program/{name}_shape"])
            src = f if comps == 1 else v
            assert oracle.evaluate_program(comps, arity, rows, src, h) == float(golden[f"{g}/evaluate_{name}"])
            assert oracle.evaluate_program(comps, arity, rows, src, h, kahan=True) == \
                float(golden[f"{g}/evaluate_{name}_kahan"])


def test_golden_programs_are_the_recorders(golden):
    for name in IC.CASES:
        prog = IC.program(name)
        assert np.array_equal(IC.rows(prog), golden[f"program/{name}"]), name
        assert [prog.components, prog.arity] == list(golden[f"program/{name}_shape"])


def test_program_equals_callable_bit_for_bit(oracle):
    """The recorded program run on arrays gives exactly what the Python
    callable gives on them (both IEEE double, operation by operation), and
    the oracle's integral of it is the oracle's evaluate."""
    rng = np.random.default_rng(11)
    shape, h = (6, 7, 9), (0.3, 0.7, 1.1)
    for name, (comps, _) in IC.CASES.items():
        field = rng.standard_normal(shape if comps == 1 else (3,) + shape)
        ins = _inputs(oracle, name, field, h)
        direct = np.asarray(_call(name, ins), dtype=np.float64) * np.ones(shape)
        prog = IC.program(name)
        via = I.interpret(prog, ins) * np.ones(shape)
        assert np.array_equal(direct, via), name
        assert oracle.integrate(direct, h) == oracle.evaluate_program(comps, prog.arity, prog.instr, field, h), name


def test_recorded_free_energy_is_the_reference_free_energy(oracle, golden):
    """examples/common/cahn_hilliard.hpp:64-68 written as a callable."""
    prog = I.trace(lambda p, g: -0.5 * p * p + 0.25 * p * p * p * p + 0.5 * 0.8 * g.squaredNorm())
    for g in ("aniso3d", "cube7"):
        f, h = golden[f"{g}/f"], tuple(golden[f"{g}/h"])
        assert oracle.evaluate_program(1, 2, prog.instr, f, h) == float(golden[f"{g}/free_energy"])


def test_constant_and_reuse():
    prog = I.trace(lambda p: 3.0)
    assert prog.instr == [(0, prog.instr[0][1], 0, 0, 3.0)]
    # A long chain reuses registers: 121 instructions on a handful of registers.
    def chain(p):
        acc = p
        for k in range(40):
            acc = acc * 0.5 + p
        return acc
    prog = I.trace(chain)
    assert len(prog) == 1 + 40 * 3 and max(r[1] for r in prog.instr) < 4


def test_recorder_errors():
    with pytest.raises(TypeError, match=r"\*\*"):
        I.trace(lambda p: p ** 2)
    with pytest.raises(TypeError, match="minimum/maximum"):
        I.trace(lambda p: p if p > 0 else -p)
    with pytest.raises(TypeError, match="truth value"):
        I.trace(lambda p: p and 1.0)
    with pytest.raises(TypeError, match="1..4"):
        I.trace(lambda a, b, c, d, e: a)
    with pytest.raises(TypeError, match="1..2"):
        I.trace(lambda u, M, x: u[0], 3)

    def wide(p):
        xs = [p * float(k + 2) for k in range(40)]   # all live before the sum
        acc = xs[0]
        for x in xs[1:]:
            acc = acc + x
        return acc
    with pytest.raises(ValueError, match="live"):
        I.trace(wide)

    def long(p):
        acc = p
        for _ in range(70):
            acc = acc * p + 1.0
        return acc
    with pytest.raises(ValueError, match="instructions"):
        I.trace(long)


def test_oracle_rejects_inputs_beyond_arity(oracle):
    f = np.zeros((4, 4, 4))
    with pytest.raises(ValueError, match="beyond the arity"):
        oracle.evaluate_program(1, 1, [(1, 0, 1, 0, 0.0)], f)


def test_generated_sources_compile_for_sm100a():
    """The CUDA source gc_evaluate_program generates for every recorded case
    (both storage types) compiles under NVRTC for sm_100a with the options
    the library uses (evaluate.cu); no GPU is needed to compile."""
    import ctypes as C
    import gridcalc_b200 as gc
    nv = C.CDLL("/usr/local/cuda/lib64/libnvrtc.so.12")
    gc.lib.gc_program_source.restype = C.c_size_t
    gc.lib.gc_program_source.argtypes = [C.POINTER(gc.gc_program), C.c_int, C.c_char_p, C.c_size_t]
    opts = (C.c_char_p * 3)(b"--gpu-architecture=sm_100a", b"--fmad=false", b"-std=c++17")
    for name, (comps, fn) in IC.CASES.items():
        p = gc.program_struct(gc.integrand.trace(fn, comps))
        for dt in (gc.F64, gc.F32):
            n = gc.lib.gc_program_source(C.byref(p), dt, None, 0)
            buf = C.create_string_buffer(n)
            assert gc.lib.gc_program_source(C.byref(p), dt, buf, n) == n
            src = buf.value
            assert (b"#define GC_T double" if dt == gc.F64 else b"#define GC_T float") in src
            # The variant for fields whose offsets fit 32 bits and whose cell
            # pairs are aligned prepends two defines.
            for variant in (src, b"#define GC_IDX32 1\n#define GC_PAIRS 1\n" + src):
                h = C.c_void_p()
                assert nv.nvrtcCreateProgram(C.byref(h), variant, b"gc_integrand.cu", 0, None, None) == 0
                rc = nv.nvrtcCompileProgram(h, 3, opts)
                size = C.c_size_t()
                nv.nvrtcGetProgramLogSize(h, C.byref(size))
                log = C.create_string_buffer(size.value)
                nv.nvrtcGetProgramLog(h, log)
                nv.nvrtcDestroyProgram(C.byref(h))
                assert rc == 0, (name, dt, log.value.decode())
    bad = gc.gc_program(1, 1, 1, 0)
    bad.instr[0] = gc.gc_instr(2, 0, 0, 0, 0.0)   # reads a register never written
    assert gc.lib.gc_program_source(C.byref(bad), gc.F64, None, 0) == 0


def test_named_integrands_are_the_reference_expressions(oracle, golden):
    """gc_evaluate runs its named integrands as built-in programs
    (gc_integrand_program).  They are instruction for instruction what the
    recorder makes of the reference's expressions (cahn_hilliard.hpp:64-77,
    heterogeneous_diffusion.hpp:82), and the oracle running them gives the
    reference's golden energies; no GPU is needed."""
    import gridcalc_b200 as gc
    for kappa in (0.8, 1.0, 0.35):
        assert gc.integrand_program("ch_free_energy", kappa).instr == I.trace(
            lambda p, g: -0.5 * p * p + 0.25 * p * p * p * p + (0.5 * kappa) * g.squaredNorm()).instr
    assert gc.integrand_program("grad_squared").instr == I.trace(lambda p, g: g.squaredNorm()).instr
    assert gc.integrand_program("psi_squared").instr == I.trace(lambda p: p * p).instr
    assert gc.integrand_program("psi").instr == I.trace(lambda p: p).instr
    for g in ("aniso3d", "cube7"):
        f, h = golden[f"{g}/f"], tuple(golden[f"{g}/h"])
        fe = gc.integrand_program("ch_free_energy", 0.8)
        assert oracle.evaluate_program(1, fe.arity, fe.instr, f, h) == float(golden[f"{g}/free_energy"])
        ge = gc.integrand_program("grad_squared")
        assert oracle.evaluate_program(1, ge.arity, ge.instr, f, h) == float(golden[f"{g}/gradient_energy"])
    with pytest.raises(KeyError):
        gc.integrand_program("elastic")
    bad = gc.gc_program()
    assert gc.STATUS[gc.lib.gc_integrand_program(gc.C.byref(gc.gc_integrand(7, 0.0)), gc.C.byref(bad))] == \
        "GC_ERR_INVALID_ARG"


# --- random integrands (property test) --------------------------------------
from hypothesis import HealthCheck, assume, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402


@settings(max_examples=250, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(data=st.data(), arity=st.integers(1, 4))
def test_random_integrands_record_exactly(oracle, data, arity):
    """Random expressions over every opcode and every input of the arity:
    the recorded program computes exactly what the Python callable computes
    on the same arrays (bit for bit, non-finite values included), and the
    oracle's func::evaluate of the program is the integral of those values."""
    n_inputs = {1: 1, 2: 4, 3: 5, 4: 6}[arity]
    tree = data.draw(IC.random_tree(n_inputs))
    fn = IC.tree_callable(tree, arity)
    try:
        prog = I.trace(fn)
    except (ZeroDivisionError, ValueError):   # a constant subexpression divides by zero / too large
        assume(False)
    rng = np.random.default_rng(len(prog.instr))
    shape, h = (5, 6, 7), (0.5, 0.75, 1.25)
    field = rng.standard_normal(shape)
    if data.draw(st.integers(0, 4)) == 0:
        field[2, 3, 4] = data.draw(st.sampled_from([np.inf, -np.inf, np.nan]))
    ins = [field]
    if arity >= 2:
        ins += list(oracle.op("gradient", 2, field, h))
    if arity >= 3:
        ins.append(oracle.op("laplacian", 2, field, h))
    if arity >= 4:
        ins.append(oracle.op("biharmonic", 2, field, h))
    with np.errstate(all="ignore"):
        direct = np.asarray(fn(*([ins[0], I.SymVec3(ins[1:4]), *(ins[4:])][:arity])), dtype=np.float64) * np.ones(shape)
        via = np.asarray(I.interpret(prog, ins), dtype=np.float64) * np.ones(shape)
    assert np.array_equal(direct.view(np.uint64), via.view(np.uint64))
    got = oracle.evaluate_program(1, prog.arity, prog.instr, field, h)
    want = oracle.integrate(direct, h)
    assert got == want or (np.isnan(got) and np.isnan(want))
