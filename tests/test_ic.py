"""The product's seeded initial condition (gc_random_ic) against the
reference's makeRandomIc (examples/common/cahn_hilliard.hpp:85-103).

Pinned three ways: the golden vector generated from the reference build
(ic/seed42_16x16), the reference build itself on several grids, seeds and
amplitudes (mean subtracted), and the standard library's mt19937_64 +
uniform_real_distribution draws (the raw draws the workload's "0 plus
i.i.d. uniform noise" initial condition uses).  No GPU work.
"""
import numpy as np
import pytest

import gridcalc_b200 as gc
import oracle_lib


def test_golden_seed42():
    want = np.load(oracle_lib.ROOT + "/tests/golden/reference_vectors.npz")["ic/seed42_16x16"]
    got = gc.random_ic(gc.Grid(16, 16, 1), 42, 0.05)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("shape,seed,amp", [((1, 128, 128), 42, 0.05), ((7, 5, 3), 0, 1.0),
                                            ((1, 1, 1), 2**64 - 1, 0.3), ((4, 33, 17), 123456789, 1e-3)])
def test_mean_subtracted_vs_reference(shape, seed, amp):
    ref = oracle_lib.reference()
    nz, ny, nx = shape
    want = ref.make_random_ic(shape, seed, amp)
    got = gc.random_ic(gc.Grid(nx, ny, nz), seed, amp)
    assert np.array_equal(got, want)


@pytest.mark.skipif(not oracle_lib.reference_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("seed,amp", [(42, 0.05), (5489, 1.0), (7, 0.4)])
def test_raw_draws_vs_standard_library(seed, amp):
    ref = oracle_lib.reference()
    n = 128 * 128 + 700   # crosses many 312-word refills
    want = ref.uniform_draws(seed, amp, n)
    got = gc.random_ic(gc.Grid(n, 1, 1), seed, amp, subtract_mean=False).ravel()
    assert np.array_equal(got, want)
    assert np.all(np.abs(got) <= amp)


def test_raw_draws_range_and_mean():
    g = gc.Grid(256, 256, 1)
    raw = gc.random_ic(g, 42, 0.05, subtract_mean=False)
    assert raw.min() >= -0.05 and raw.max() < 0.05
    assert abs(raw.mean()) < 1e-3
    sub = gc.random_ic(g, 42, 0.05)
    assert abs(sub.sum()) < 1e-12
    # the reference's mean: a sequential sum (np.cumsum adds in order) over n
    assert np.array_equal(sub, raw - np.cumsum(raw.ravel())[-1] / raw.size)


def test_errors():
    with pytest.raises(gc.GcError):
        gc.random_ic(gc.Grid(4, 4, 1), 1, float("nan"))
    with pytest.raises(gc.GcError):
        gc.random_ic(gc.Grid(4, 4, 1), 1, -1.0)
