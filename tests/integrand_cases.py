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
