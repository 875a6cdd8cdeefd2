"""Integrands for the func::evaluate parity tests and golden vectors: Python
callables of every arity the reference's evaluate accepts
(func/Functional.hpp:88-148 scalar, :183-220 vector), traced into device
programs by the package's recorder (loaded from its file, so no GPU library
is needed to build the programs)."""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The package's own recorder module, shared with the package when both are
# imported (so symbols and programs are the same classes on either side).
if "gridcalc_b200.integrand" in sys.modules:
    integrand = sys.modules["gridcalc_b200.integrand"]
else:
    _spec = importlib.util.spec_from_file_location(
        "gridcalc_b200.integrand", os.path.join(ROOT, "grid-calculus_b200", "gridcalc_b200", "integrand.py"))
    integrand = importlib.util.module_from_spec(_spec)
    sys.modules["gridcalc_b200.integrand"] = integrand
    _spec.loader.exec_module(integrand)
sqrt, minimum, maximum = integrand.sqrt, integrand.minimum, integrand.maximum

# name -> (components, callable)
CASES = {
    "s1_cubic": (1, lambda p: p * p * p - 0.5 * p),
    "s2_free_energy": (1, lambda p, g: -0.5 * p * p + 0.25 * p * p * p * p + 0.5 * 0.7 * g.squaredNorm()),
    "s3_mixed": (1, lambda p, g, lap: p * lap + g[0] * g[1] - abs(lap) / (1.0 + p * p)),
    "s4_all": (1, lambda p, g, lap, bih: maximum(p, 0.0) * bih + minimum(lap, g[2]) + sqrt(1.0 + p * p) + g.norm()),
    "v1_norm": (3, lambda u: u.squaredNorm() + u[0] * u[2]),
    "v2_elastic": (3, lambda u, M: 0.8 * M.doubleContract(M) + 0.5 * 1.3 * M.trace() * M.trace() - u.dot(u)),
}


def program(name):
    comps, fn = CASES[name]
    return integrand.trace(fn, comps)


def rows(prog):
    """The program as an (n, 5) array of (op, dst, a, b, value)."""
    import numpy as np
    return np.array(prog.instr, dtype=np.float64).reshape(-1, 5)


# --- random expression trees for the property tests ---------------------------
_UNARY = ("neg", "abs", "sqrt")
_BINARY = ("add", "sub", "mul", "div", "min", "max")


def random_tree(n_inputs):
    """A hypothesis strategy: expression trees over inputs 0..n_inputs-1 and
    non-zero constants, with every unary and binary opcode."""
    from hypothesis import strategies as st
    leaf = st.one_of(st.tuples(st.just("in"), st.integers(0, n_inputs - 1)),
                     st.tuples(st.just("c"), st.floats(-4.0, 4.0, allow_nan=False).filter(lambda v: v != 0.0)))
    return st.recursive(leaf, lambda kids: st.one_of(
        st.tuples(st.sampled_from(_UNARY), kids),
        st.tuples(st.sampled_from(_BINARY), kids, kids)), max_leaves=12)


def eval_tree(node, ins):
    """The expression over scalars, Sym values or arrays alike: the same
    Python callable is recorded and run directly."""
    kind = node[0]
    if kind == "in":
        return ins[node[1]]
    if kind == "c":
        return node[1]
    a = eval_tree(node[1], ins)
    if kind == "neg":
        return -a
    if kind == "abs":
        return abs(a)
    if kind == "sqrt":
        return sqrt(abs(a))
    b = eval_tree(node[2], ins)
    return {"add": lambda: a + b, "sub": lambda: a - b, "mul": lambda: a * b, "div": lambda: a / b,
            "min": lambda: minimum(a, b), "max": lambda: maximum(a, b)}[kind]()


def tree_callable(tree, arity):
    """The tree as a callable of the given arity (psi, grad, lap, bih)."""
    if arity == 1:
        return lambda p: eval_tree(tree, [p])
    if arity == 2:
        return lambda p, g: eval_tree(tree, [p, g[0], g[1], g[2]])
    if arity == 3:
        return lambda p, g, lap: eval_tree(tree, [p, g[0], g[1], g[2], lap])
    return lambda p, g, lap, bih: eval_tree(tree, [p, g[0], g[1], g[2], lap, bih])
