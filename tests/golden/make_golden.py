"""Generates tests/golden/reference_vectors.npz from the reference itself.

Runs the reference gridcalc headers, compiled from the reference tree into
oracle/_ref/libgcref.so by oracle/Makefile, on small seeded inputs and stores
inputs and outputs.  The fixtures pin the CPU oracle (oracle/gc_oracle.c) and
the GPU kernels on machines where the reference tree is absent.

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import integrand_cases  # noqa: E402
import oracle_lib  # noqa: E402

PARTIALS = oracle_lib.PARTIALS
# Grids and orders the partials are stored for (all 31 each).
PARTIAL_CASES = [("aniso3d", 4), ("flat2d", 2)]

# Count triples the spectral partial is stored for.
SPECTRAL_COUNTS = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (2, 1, 1), (0, 3, 0), (2, 2, 0), (1, 1, 1),
                   (4, 0, 0), (0, 0, 3)]

# (name, shape (nz, ny, nx), h)
GRIDS = [
    ("aniso3d", (8, 10, 12), (0.3, 0.25, 0.5)),
    ("flat2d", (1, 9, 17), (1.0, 1.0, 1.0)),
    ("cube7", (7, 7, 7), (1.0, 0.5, 2.0)),
]


def main() -> None:
    ref = oracle_lib.reference()
    rng = np.random.default_rng(20261203)
    # Matrix fields draw from their own stream so the earlier arrays keep their values.
    rng_mat = np.random.default_rng(20261204)
    out: dict[str, np.ndarray] = {}
    for name, shape, h in GRIDS:
        f = rng.standard_normal(shape)
        v = rng.standard_normal((3,) + shape)
        D = np.exp(0.5 * rng.standard_normal(shape))
        out[f"{name}/f"] = f
        out[f"{name}/v"] = v
        out[f"{name}/D"] = D
        m = rng_mat.standard_normal((3, 3) + shape)
        out[f"{name}/m"] = m
        out[f"{name}/h"] = np.array(h)
        for order in (2, 4):
            out[f"{name}/laplacian{order}"] = ref.op("laplacian", order, f, h)
            out[f"{name}/gradient{order}"] = ref.op("gradient", order, f, h)
            out[f"{name}/divergence{order}"] = ref.op("divergence", order, v, h)
            out[f"{name}/biharmonic{order}"] = ref.op("biharmonic", order, f, h)
            out[f"{name}/ch_rhs{order}"] = ref.ch_rhs(order, 1.3, 0.7, 0.1 * f, h)
            out[f"{name}/gradient_vec{order}"] = ref.op("gradient_vec", order, v, h)
            out[f"{name}/divergence_mat{order}"] = ref.op("divergence_mat", order, m, h)
        out[f"{name}/cell_laplacian"] = ref.cell_laplacian(f, D, h)
        out[f"{name}/integrate_pairwise"] = np.array(ref.integrate(f, h, kahan=False))
        out[f"{name}/integrate_kahan"] = np.array(ref.integrate(f, h, kahan=True))
        out[f"{name}/free_energy"] = np.array(ref.ch_free_energy(f, 0.8, h))
        out[f"{name}/gradient_energy"] = np.array(ref.ch_gradient_energy(f, h))
        out[f"{name}/mean"] = np.array(ref.ch_mean(f, h))
        # func::evaluate with callables of every arity (tests/integrand_cases.py).
        for cname, (comps, _) in integrand_cases.CASES.items():
            prog = integrand_cases.program(cname)
            src = f if comps == 1 else v
            out[f"{name}/evaluate_{cname}"] = np.array(ref.evaluate_program(comps, prog.arity, prog.instr, src, h))
            out[f"{name}/evaluate_{cname}_kahan"] = np.array(
                ref.evaluate_program(comps, prog.arity, prog.instr, src, h, kahan=True))
        # The reference's spectral (PocketFFT) derivatives.
        out[f"{name}/spectral_laplacian"] = ref.spectral("laplacian", f, h)
        out[f"{name}/spectral_biharmonic"] = ref.spectral("biharmonic", f, h)
        out[f"{name}/spectral_gradient"] = ref.spectral("gradient", f, h)
        for c in SPECTRAL_COUNTS:
            out[f"{name}/spectral_partial{c[0]}{c[1]}{c[2]}"] = ref.spectral("partial", f, h, c)
        for pname, porder in PARTIAL_CASES:
            if pname == name:
                for c in PARTIALS:
                    out[f"{name}/partial{c[0]}{c[1]}{c[2]}_{porder}"] = ref.mixed(c, porder, f, h)

    # Cahn-Hilliard trajectories on a 2-D grid (h = 1, stable dt).
    psi0 = 0.05 * (2.0 * rng.random((1, 24, 24)) - 1.0)
    out["ch2d/psi0"] = psi0
    for order in (2, 4):
        out[f"ch2d/rk4_order{order}"] = ref.ch_integrate(order, 1.0, 1.0, psi0, 0.01, 40, rk4=True)
        out[f"ch2d/euler_order{order}"] = ref.ch_integrate(order, 1.0, 1.0, psi0, 0.005, 40, rk4=False)
    psi3 = 0.05 * (2.0 * rng.random((8, 8, 8)) - 1.0)
    out["ch3d/psi0"] = psi3
    out["ch3d/rk4_order2"] = ref.ch_integrate(2, 1.0, 0.5, psi3, 0.005, 20, rk4=True)

    # Diffusion drivers.
    u0 = rng.random((6, 8, 10))
    Dh = np.exp(0.3 * rng.standard_normal((6, 8, 10)))
    out["diff/u0"] = u0
    out["diff/D"] = Dh
    out["diff/fvm_rk4"] = ref.diffuse_fvm(u0, Dh, 0.05, 10, rk4=True)
    out["diff/fvm_euler"] = ref.diffuse_fvm(u0, Dh, 0.05, 10, rk4=False)
    out["diff/const_rk4"] = ref.diffuse_const(u0, 0.7, 0.05, 10, rk4=True)

    # The reference initial-condition generator (mt19937_64, mean removed).
    out["ic/seed42_16x16"] = ref.make_random_ic((1, 16, 16), 42, 0.05)

    # The programs those values were computed with (rows op, dst, a, b, value).
    for cname in integrand_cases.CASES:
        prog = integrand_cases.program(cname)
        out[f"program/{cname}"] = integrand_cases.rows(prog)
        out[f"program/{cname}_shape"] = np.array([prog.components, prog.arity])

    # A snapshot written by the reference's VTK writer, with values that pin
    # its number formatting (signed zero, extremes, non-finite, inexact decimals).
    vals = np.concatenate([rng.standard_normal(48),
                           [-0.0, 0.0, 1e-300, -1e300, 0.1, 1.0 / 3.0, 2.0 ** -1074, np.inf, -np.inf, np.nan,
                            123456789012345678.0, 5e-324]])
    snap = vals.reshape(3, 4, 5)
    out["vtk/values"] = snap
    out["vtk/h"] = np.array([0.3, 0.25, 0.5])
    ref.write_vtk(snap, os.path.join(HERE, "reference_snapshot.vtk"), "psi", (0.3, 0.25, 0.5))

    path = os.path.join(HERE, "reference_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
