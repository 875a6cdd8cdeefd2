"""GPU func::integrate / func::evaluate against the oracle.

The pairwise tag reproduces the reference's recursive pairwise tree, so the
double result must be bit-identical for every length (the tree shape
changes with n: base cases of 33..64 values, uneven splits).  The Kahan tag
is a different (parallel, compensated) summation order: it must agree with
the reference's sequential Neumaier sum to a few ulp of sum |x|, and be
deterministic.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float64)


LENGTHS = [1, 2, 63, 64, 65, 127, 128, 129, 1000, 4097, 8191, 8192, 8193, 16385, 100003,
           1 << 20, (1 << 20) + 7, 3 * (1 << 18) + 5]


@pytest.mark.parametrize("n", LENGTHS)
def test_pairwise_bit_exact(gc, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) * 10.0 ** rng.uniform(-3, 3, n)
    g = gc.Grid(n, 1, 1, 0.5, 0.25, 2.0)
    got = gc.integrate(dev(x), g, gc.Pairwise)
    want = oracle.integrate(x.reshape(1, 1, n), (0.5, 0.25, 2.0))
    assert got == want, (n, got, want)


def test_pairwise_bit_exact_large(gc, oracle):
    n = 256 ** 3
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n)
    got = gc.integrate(dev(x), gc.Grid(256, 256, 256, 1 / 256, 1 / 256, 1 / 256), gc.Pairwise)
    want = oracle.integrate(x.reshape(256, 256, 256), (1 / 256,) * 3)
    assert got == want


@pytest.mark.parametrize("n", [1, 100, 8193, (1 << 20) + 7])
def test_kahan_close_and_deterministic(gc, oracle, n):
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal(n)
    g = gc.Grid(n, 1, 1)
    a = gc.integrate(dev(x), g, gc.Kahan)
    b = gc.integrate(dev(x), g, gc.Kahan)
    assert a == b
    want = oracle.integrate(x.reshape(1, 1, n), kahan=True)
    assert abs(a - want) <= 4 * np.finfo(float).eps * np.abs(x).sum() + 1e-300


def test_float32_storage_promoted(gc, oracle):
    import torch
    rng = np.random.default_rng(11)
    x32 = rng.standard_normal(123457).astype(np.float32)
    g = gc.Grid(123457, 1, 1)
    got = gc.integrate(dev(x32, torch.float32), g, gc.Pairwise)
    want = oracle.integrate(x32.astype(np.float64).reshape(1, 1, -1))
    assert got == want


def test_unit_field_volume(gc):
    """test/integrate_test.cpp:31-47."""
    g = gc.Grid(8, 16, 4, 0.25, 0.125, 0.5)
    ones = np.ones(g.shape)
    vol = (8 * 0.25) * (16 * 0.125) * (4 * 0.5)
    assert gc.integrate(dev(ones), g, gc.Pairwise) == vol
    assert gc.integrate(dev(ones), g, gc.Kahan) == vol


def test_energies_bit_exact_golden(gc):
    golden = np.load(GOLDEN)
    for name in sorted({k.split("/")[0] for k in golden.files if k.endswith("/f")}):
        f, h = golden[f"{name}/f"], tuple(golden[f"{name}/h"])
        nz, ny, nx = f.shape
        g = gc.Grid(nx, ny, nz, *h)
        t = dev(f)
        assert gc.integrate(t, g) == float(golden[f"{name}/integrate_pairwise"])
        assert gc.evaluate(t, g, "ch_free_energy", kappa=0.8) == float(golden[f"{name}/free_energy"])
        assert gc.evaluate(t, g, "grad_squared") == float(golden[f"{name}/gradient_energy"])
        vol_total = f.size * g.cell_volume
        assert gc.evaluate(t, g, "psi") / vol_total == float(golden[f"{name}/mean"])


def test_fixed_integrands_psi_squared_and_float(gc, oracle):
    """The remaining hot-path integrands of func::evaluate: psi^2
    (heterogeneous_diffusion.hpp:82) is the pairwise integral of the rounded
    squares; float fields are promoted to double per cell, so 'psi' and
    'psi_squared' on a float field are the oracle's values on the promoted
    values; the Kahan tag agrees to a few ulps and is deterministic."""
    import torch
    rng = np.random.default_rng(23)
    shape, h = (7, 33, 65), (0.5, 0.25, 2.0)
    f = rng.standard_normal(shape)
    g = gc.Grid(shape[2], shape[1], shape[0], *h)
    assert gc.evaluate(dev(f), g, "psi_squared") == oracle.integrate(f * f, h)
    f32 = f.astype(np.float32)
    p32 = f32.astype(np.float64)
    t32 = dev(f32, torch.float32)
    assert gc.evaluate(t32, g, "psi") == oracle.integrate(p32, h)
    assert gc.evaluate(t32, g, "psi_squared") == oracle.integrate(p32 * p32, h)
    for name in ("psi_squared", "ch_free_energy", "grad_squared"):
        a = gc.evaluate(dev(f), g, name, kappa=0.6, tag=gc.Kahan)
        b = gc.evaluate(dev(f), g, name, kappa=0.6)
        assert a == gc.evaluate(dev(f), g, name, kappa=0.6, tag=gc.Kahan)
        assert abs(a - b) <= 1e-13 * abs(b), name


def test_energies_bit_exact_large(gc, oracle):
    rng = np.random.default_rng(21)
    f = 0.3 * rng.standard_normal((1, 512, 384))
    g = gc.Grid(384, 512, 1)
    t = dev(f)
    assert gc.evaluate(t, g, "ch_free_energy", kappa=1.0) == oracle.ch_free_energy(f, 1.0)
    assert gc.evaluate(t, g, "grad_squared") == oracle.ch_gradient_energy(f)


def test_d_max_face(gc, oracle):
    rng = np.random.default_rng(4)
    D = np.exp(rng.standard_normal((12, 17, 20)))
    g = gc.Grid(20, 17, 12)
    assert gc.d_max_face(dev(D), g) == oracle.d_max_face(D)
