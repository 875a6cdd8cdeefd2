"""Integrand programs: a Python callable for func::evaluate turned into the
straight-line register program the device evaluates (gc_program in
gridcalc_b200.h).

The reference calls a host callable per cell (func/Functional.hpp:88-148
for a scalar psi with arity 1..4, :183-220 for a Vec3d field with arity
1..2).  Here the callable is called once, on symbolic arguments; the
operations it performs on them are recorded in order and become device
instructions.  Python's float arithmetic is IEEE double with correct
rounding, as are the device's + - * / and sqrt, so the device integrand is
the value the callable itself would return at every cell, bit for bit.

Supported on symbols: + - * / (either side a number), unary - and abs(),
``sqrt``, ``minimum`` / ``maximum`` (std::min / std::max semantics); vectors
index with ``v[i]`` and offer ``dot``, ``squaredNorm``, ``norm``; matrices
index with ``M[row, col]`` (M(row, col) = d_col u_row) and offer ``trace``,
``squaredNorm`` and ``doubleContract``.  Sums inside these helpers follow
the reference's Eigen types: component order, left to right.
"""
from __future__ import annotations

import inspect
import math
from dataclasses import dataclass, field

MAX_INSTR = 128
REGS = 32

OPC = {"const": 0, "input": 1, "add": 2, "sub": 3, "mul": 4, "div": 5, "neg": 6, "abs": 7, "sqrt": 8,
       "min": 9, "max": 10}

# Input numbers (gridcalc_b200.h GC_IN_*).
PSI, GRAD_X, GRAD_Y, GRAD_Z, LAP, BIH = 0, 1, 2, 3, 4, 5
U_X, U_Y, U_Z, DU = 0, 1, 2, 3


class _Trace:
    def __init__(self):
        self.nodes: list[tuple] = []      # (op, args, payload)
        self.inputs: dict[int, int] = {}

    def add(self, op, args=(), payload=0.0) -> "Sym":
        self.nodes.append((op, tuple(args), payload))
        return Sym(self, len(self.nodes) - 1)

    def input(self, k: int) -> "Sym":
        if k not in self.inputs:
            self.inputs[k] = self.add("input", (), k).id
        return Sym(self, self.inputs[k])


class Sym:
    """A double-valued quantity of one cell."""
    __slots__ = ("t", "id")
    __array_ufunc__ = None   # numpy scalars defer to the reflected operators

    def __init__(self, t: _Trace, node: int):
        self.t, self.id = t, node

    def _lift(self, x) -> "Sym":
        if isinstance(x, Sym):
            if x.t is not self.t:
                raise ValueError("integrand: symbols from different traces")
            return x
        if isinstance(x, bool) or not isinstance(x, (int, float)):
            raise TypeError(f"integrand: unsupported operand {type(x).__name__}")
        return self.t.add("const", (), float(x))

    def _bin(self, op, other, rev=False):
        o = self._lift(other)
        return self.t.add(op, (o.id, self.id) if rev else (self.id, o.id))

    def __add__(self, o): return self._bin("add", o)
    def __radd__(self, o): return self._bin("add", o, True)
    def __sub__(self, o): return self._bin("sub", o)
    def __rsub__(self, o): return self._bin("sub", o, True)
    def __mul__(self, o): return self._bin("mul", o)
    def __rmul__(self, o): return self._bin("mul", o, True)
    def __truediv__(self, o): return self._bin("div", o)
    def __rtruediv__(self, o): return self._bin("div", o, True)
    def __neg__(self): return self.t.add("neg", (self.id,))
    def __pos__(self): return self
    def __abs__(self): return self.t.add("abs", (self.id,))

    def __pow__(self, o):
        raise TypeError("integrand: ** is not supported (its rounding is the C library's); multiply instead")

    def __bool__(self):
        raise TypeError("integrand: a symbolic value has no truth value; use minimum/maximum")

    def _cmp(self, o):
        raise TypeError("integrand: comparisons cannot be recorded; use minimum/maximum")

    __lt__ = __le__ = __gt__ = __ge__ = _cmp

    def __float__(self):
        raise TypeError("integrand: a symbolic value has no float value")


def _is_array(x) -> bool:
    return hasattr(x, "__array__") and not isinstance(x, float)


def sqrt(x):
    """Correctly rounded square root (std::sqrt); also on numbers and numpy arrays."""
    if isinstance(x, Sym):
        return x.t.add("sqrt", (x.id,))
    if _is_array(x):
        import numpy as np
        return np.sqrt(x)
    return math.sqrt(x)


def minimum(a, b):
    """std::min(a, b): b if b < a else a; also on numbers and numpy arrays."""
    s = a if isinstance(a, Sym) else b
    if isinstance(s, Sym):
        return s.t.add("min", (s._lift(a).id, s._lift(b).id))
    if _is_array(a) or _is_array(b):
        import numpy as np
        return np.where(b < a, b, a)
    return b if b < a else a


def maximum(a, b):
    """std::max(a, b): b if a < b else a; also on numbers and numpy arrays."""
    s = a if isinstance(a, Sym) else b
    if isinstance(s, Sym):
        return s.t.add("max", (s._lift(a).id, s._lift(b).id))
    if _is_array(a) or _is_array(b):
        import numpy as np
        return np.where(a < b, b, a)
    return b if a < b else a


def _sum_sq(xs):
    acc = xs[0] * xs[0]
    for x in xs[1:]:
        acc = acc + x * x
    return acc


class SymVec3:
    """Vec3d of one cell (Eigen::Vector3d)."""

    def __init__(self, comps):
        self.c = list(comps)

    def __getitem__(self, i):
        return self.c[i]

    def __call__(self, i):
        return self.c[i]

    def dot(self, o: "SymVec3"):
        return (self.c[0] * o.c[0] + self.c[1] * o.c[1]) + self.c[2] * o.c[2]

    def squaredNorm(self):  # noqa: N802 (Eigen's name)
        return _sum_sq(self.c)

    def norm(self):
        return sqrt(self.squaredNorm())


class SymMat3:
    """Mat3d of one cell (Eigen::Matrix3d), M[row, col]."""

    def __init__(self, entries):
        self.m = [list(r) for r in entries]

    def __getitem__(self, rc):
        r, c = rc
        return self.m[r][c]

    def __call__(self, r, c):
        return self.m[r][c]

    def trace(self):
        return (self.m[0][0] + self.m[1][1]) + self.m[2][2]

    def _storage_sum(self, o: "SymMat3"):
        # Eigen's coefficient-wise sum: storage (column-major) order from 0.0.
        acc = 0.0
        for c in range(3):
            for r in range(3):
                acc = acc + self.m[r][c] * o.m[r][c]
        return acc

    def squaredNorm(self):  # noqa: N802 (Eigen's name)
        return self._storage_sum(self)

    def doubleContract(self, o: "SymMat3"):  # noqa: N802
        """A : B = (A.array() * B.array()).sum() (tensor/Contraction.hpp:88-101)."""
        return self._storage_sum(o)


@dataclass
class Program:
    components: int
    arity: int
    instr: list = field(default_factory=list)   # (op, dst, a, b, value)

    def __len__(self):
        return len(self.instr)


def arity_of(fn) -> int:
    """Number of positional parameters without defaults (the callable's arity)."""
    sig = inspect.signature(fn)
    n = 0
    for p in sig.parameters.values():
        if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD) and p.default is p.empty:
            n += 1
        elif p.kind == p.VAR_POSITIONAL:
            raise TypeError("integrand: *args callables have no fixed arity")
    return n


def trace(fn, components: int = 1, arity: int | None = None) -> Program:
    """Record fn on symbolic arguments.  Scalar fields (components 1) call
    fn(psi[, grad[, lap[, bih]]]); vector fields (components 3) call
    fn(u[, M])."""
    if components not in (1, 3):
        raise ValueError("integrand: components must be 1 (scalar) or 3 (vector)")
    arity = arity_of(fn) if arity is None else arity
    top = 4 if components == 1 else 2
    if not 1 <= arity <= top:
        raise TypeError(f"integrand: a {'scalar' if components == 1 else 'vector'} integrand takes 1..{top} "
                        f"arguments, got {arity}")
    t = _Trace()
    if components == 1:
        args = [t.input(PSI), SymVec3([t.input(GRAD_X), t.input(GRAD_Y), t.input(GRAD_Z)]), t.input(LAP),
                t.input(BIH)][:arity]
    else:
        args = [SymVec3([t.input(U_X + c) for c in range(3)]),
                SymMat3([[t.input(DU + 3 * r + c) for c in range(3)] for r in range(3)])][:arity]
    out = fn(*args)
    if not isinstance(out, Sym):
        if isinstance(out, (int, float)) and not isinstance(out, bool):
            out = t.add("const", (), float(out))
        else:
            raise TypeError(f"integrand: the callable must return a number, got {type(out).__name__}")
    return Program(components, arity, _allocate(t, out.id))


def _allocate(t: _Trace, root: int) -> list:
    """Emit the nodes the result depends on, in trace order, on at most REGS
    registers (a register is reused once its value has had its last read)."""
    live = set()
    stack = [root]
    while stack:
        k = stack.pop()
        if k in live:
            continue
        live.add(k)
        stack.extend(t.nodes[k][1])
    order = sorted(live)
    last = {}
    for pos, k in enumerate(order):
        for a in t.nodes[k][1]:
            last[a] = pos
    last[root] = len(order)
    free = list(range(REGS - 1, -1, -1))
    reg = {}
    out = []
    for pos, k in enumerate(order):
        op, args, payload = t.nodes[k]
        srcs = [reg[a] for a in args]
        for a in set(args):
            if last[a] == pos:
                free.append(reg[a])
        if not free:
            raise ValueError(f"integrand: more than {REGS} values live at once")
        dst = free.pop()
        reg[k] = dst
        a = int(payload) if op == "input" else (srcs[0] if srcs else 0)
        b = srcs[1] if len(srcs) > 1 else 0
        out.append((OPC[op], dst, a, b, float(payload) if op == "const" else 0.0))
    if len(out) > MAX_INSTR:
        raise ValueError(f"integrand: {len(out)} instructions, at most {MAX_INSTR}")
    return out


def interpret(prog: Program, inputs):
    """Run the program on arrays of inputs (numpy or floats) with Python /
    numpy double arithmetic: the program's meaning, for tests."""
    import numpy as np
    r = [None] * REGS
    for op, dst, a, b, value in prog.instr:
        if op == 0:
            v = value
        elif op == 1:
            v = inputs[a]
        elif op == 2:
            v = r[a] + r[b]
        elif op == 3:
            v = r[a] - r[b]
        elif op == 4:
            v = r[a] * r[b]
        elif op == 5:
            v = r[a] / r[b]
        elif op == 6:
            v = -r[a]
        elif op == 7:
            v = np.abs(r[a])
        elif op == 8:
            v = np.sqrt(r[a])
        elif op == 9:
            v = np.where(r[b] < r[a], r[b], r[a])
        else:
            v = np.where(r[a] < r[b], r[b], r[a])
        r[dst] = v
    return r[prog.instr[-1][1]]
