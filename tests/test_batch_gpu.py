"""Batched Cahn-Hilliard ensemble: members of uneven size, each with its own
kappa, mobility and dt.  In double the ensemble runs the same tile
arithmetic as the single-grid path, so every member must be bit-identical
to the oracle run on that member alone; in float the error against the
double oracle is bounded; per-member FP64 mass and free energy agree with
the oracle; the autotuner picks a shape and records it in a JSON cache."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [  # (nx, ny, mobility, kappa, dt)
    (16, 16, 1.0, 1.0, 0.004), (80, 48, 1.0, 0.5, 0.008), (64, 64, 0.7, 2.0, 0.002),
    (33, 17, 1.0, 1.3, 0.003), (144, 96, 1.0, 0.9, 0.005), (1, 40, 1.0, 1.0, 0.004),
]


def stable_dt(kappa, order=4):
    lam = 2 * (16 / 3 if order == 4 else 4.0)
    return 0.5 * 2.7853 / (lam * (kappa * lam + 2))


def ics(members, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny, *_ in members:
        cbar = rng.uniform(-0.4, 0.4)
        out.append(cbar + 0.05 * (2 * rng.random((ny, nx)) - 1))
    return out


@pytest.mark.parametrize("shape", [2, 4], ids=["stage_kernels", "fused"])
@pytest.mark.parametrize("order", [2, 4])
def test_f64_ensemble_bit_exact_per_member(gc, oracle, order, shape):
    """Both kernels (four stage launches per step, or the fused four-stage
    launch) give every double member bit for bit the oracle's result."""
    import torch
    b = gc.ChBatch(MEMBERS, order=order, dtype=torch.float64)
    b.set_shape(shape)
    init = ics(MEMBERS)
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    b.run(37)
    for i, (nx, ny, mob, kap, dt) in enumerate(MEMBERS):
        want = oracle.ch_integrate(order, mob, kap, init[i].reshape(1, ny, nx), dt, 37)
        assert np.array_equal(b.get_member(i), want.reshape(ny, nx)), i
    b.close()


@pytest.mark.parametrize("shape", [2, 4], ids=["stage_kernels", "fused"])
def test_f32_ensemble_error_and_diagnostics(gc, oracle, shape):
    import torch
    members = [(nx, ny, 1.0, kap, stable_dt(kap)) for nx, ny, kap in
               [(64, 64, 0.5), (96, 80, 1.2), (128, 128, 2.0), (48, 112, 0.8)]]
    b = gc.ChBatch(members, order=4, dtype=torch.float32)
    b.set_shape(shape)
    init = [c.astype(np.float32).astype(np.float64) for c in ics(members, seed=11)]
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    steps = 300
    b.run(steps)
    mass, energy = b.diagnostics()
    for i, (nx, ny, mob, kap, dt) in enumerate(members):
        want = oracle.ch_integrate(4, mob, kap, init[i].reshape(1, ny, nx), dt, steps)
        got = b.get_member(i).reshape(1, ny, nx)
        l2 = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert l2 < 1e-4, (i, l2)
        f_ref = oracle.ch_free_energy(want, kap)
        v4 = nx * ny / 4.0
        # double-well form F + V/4 (f = (c^2 - 1)^2 / 4)
        assert abs((energy[i] + v4) - (f_ref + v4)) / abs(f_ref + v4) < 1e-4, (i, energy[i], f_ref)
        m_ref = float(init[i].sum())
        assert abs(mass[i] - m_ref) < 1e-6 * nx * ny, (i, mass[i], m_ref)  # mean drift < 1e-6
    b.close()


def test_f32_ensemble_with_odd_width_member(gc, oracle):
    """One odd-width member sends the float ensemble down the one-column
    tiles; every member still within 1e-4 of the FP64 oracle."""
    import torch
    members = [(nx, ny, 1.0, kap, stable_dt(kap)) for nx, ny, kap in [(64, 48, 0.7), (33, 40, 1.1), (96, 17, 1.5)]]
    b = gc.ChBatch(members, order=4, dtype=torch.float32)
    init = [c.astype(np.float32).astype(np.float64) for c in ics(members, seed=5)]
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    b.run(150)
    for i, (nx, ny, mob, kap, dt) in enumerate(members):
        want = oracle.ch_integrate(4, mob, kap, init[i].reshape(1, ny, nx), dt, 150)
        l2 = np.linalg.norm(b.get_member(i).reshape(1, ny, nx) - want) / np.linalg.norm(want)
        assert l2 < 1e-4, (i, l2)
    b.close()


def test_diagnostics_match_oracle_f64(gc, oracle):
    import torch
    b = gc.ChBatch(MEMBERS[:5], order=4, dtype=torch.float64)
    init = ics(MEMBERS[:5], seed=5)
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    mass, energy = b.diagnostics()
    for i, (nx, ny, mob, kap, dt) in enumerate(MEMBERS[:5]):
        c = init[i].reshape(1, ny, nx)
        assert abs(mass[i] - oracle.integrate(c)) <= 1e-13 * np.abs(c).sum()
        f = oracle.ch_free_energy(c, kap)
        assert abs(energy[i] - f) <= 1e-13 * max(1.0, abs(f))
    b.close()


def test_autotune_and_cache(gc, oracle, tmp_path):
    import torch
    members = [(nx, nx, 1.0, 1.0, stable_dt(1.0)) for nx in (64, 96, 160, 256)]
    b = gc.ChBatch(members, order=4, dtype=torch.float32)
    init = ics(members, seed=2)
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    cache = str(tmp_path / "tune.json")
    report = json.loads(b.autotune(steps_per_trial=4, cache_path=cache))
    assert set(report["trials_ms_per_step"]) == {"32x16x4", "64x8x4", "64x16x4", "64x32x8", "fused64x32"}
    assert report["choice"] in report["trials_ms_per_step"]
    # tuning restored the state
    assert np.array_equal(b.get_member(2), init[2].astype(np.float32).astype(np.float64))
    cached = json.loads(open(cache).read())
    assert len(cached) == 1
    b2 = gc.ChBatch(members, order=4, dtype=torch.float32)
    assert json.loads(b2.autotune(steps_per_trial=4, cache_path=cache))["cached"] is True
    b.close()
    b2.close()


@pytest.mark.parametrize("shape", [2, 4], ids=["stage_kernels", "fused"])
def test_large_members(gc, oracle, shape):
    """Members at the top of the ensemble's size range (512^2 and 640 x 576):
    in double bit-identical to the oracle after 20 steps; in float, after
    1000 steps at each member's stable dt, within 1e-4 (L2) and 1e-5 (free
    energy) of the FP64 solution from the same FP32-rounded start (the plain
    FP64 path, itself bit-identical to the oracle)."""
    import torch
    members = [(512, 512, 1.0, 1.0, stable_dt(1.0)), (96, 80, 1.0, 1.7, stable_dt(1.7)),
               (640, 576, 1.0, 0.6, stable_dt(0.6))]
    init = ics(members, seed=21)
    b = gc.ChBatch(members, order=4, dtype=torch.float64)
    b.set_shape(shape)
    for i, c0 in enumerate(init):
        b.set_member(i, c0)
    b.run(20)
    for i in (0, 2):
        nx, ny, mob, kap, dt = members[i]
        want = oracle.ch_integrate(4, mob, kap, init[i].reshape(1, ny, nx), dt, 20)
        assert np.array_equal(b.get_member(i), want.reshape(ny, nx)), i
    b.close()
    b = gc.ChBatch(members, order=4, dtype=torch.float32)
    b.set_shape(shape)
    start = [c.astype(np.float32).astype(np.float64) for c in init]
    for i, c0 in enumerate(start):
        b.set_member(i, c0)
    b.run(1000)
    _, energy = b.diagnostics()
    for i, (nx, ny, mob, kap, dt) in enumerate(members):
        g = gc.Grid(nx, ny, 1)
        want = torch.from_numpy(start[i].reshape(1, ny, nx)).cuda()
        gc.ch_integrate(want, g, gc.CahnHilliardRhs(mob, kap, 4), dt, 1000, gc.RK4)
        got = torch.from_numpy(b.get_member(i).reshape(1, ny, nx)).cuda().double()
        l2 = float(torch.linalg.norm(got - want) / torch.linalg.norm(want))
        assert l2 < 1e-4, (i, l2)
        v4 = nx * ny / 4.0
        f_ref = gc.evaluate(want, g, "ch_free_energy", kappa=kap) + v4
        assert abs(energy[i] + v4 - f_ref) / abs(f_ref) < 1e-5, (i, energy[i] + v4, f_ref)
    b.close()


def test_shape_selection_errors(gc):
    """The fused shape covers orders 2 and 4 only; shapes outside 0..4 are
    rejected."""
    import torch
    b = gc.ChBatch([(32, 32, 1.0, 1.0, 0.001)], order=6, dtype=torch.float32)
    with pytest.raises(gc.GcError) as ei:
        b.set_shape(gc.ChBatch.FUSED)
    assert ei.value.status == "GC_ERR_UNSUPPORTED"
    with pytest.raises(gc.GcError) as ei:
        b.set_shape(5)
    assert ei.value.status == "GC_ERR_INVALID_ARG"
    b.set_shape(3)
    b.run(2)
    b.close()
