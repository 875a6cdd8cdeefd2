"""Learned coarse-step workflow for 2-D Cahn-Hilliard (kappa = M = 1).

The coarse step of dt = 0.16 is one RKC2 step (6 stages, stable far beyond
RK4's limit) plus the network's correction of that step's error: B(c) +
delta(c, B(c)).  Trajectories come from the plain GPU solver (FP64 RK4,
dt = 0.01); training pairs are (c(t), c(t + 16 dt)) taken on the fly along
each trajectory, in FP64, and the network is trained by the library's own
kernels (Corrector.train_step) on the per-sample normalised loss.
Evaluation runs held-out seeds to t_end -- plain fine RK4 (the reference and
the "plain form" timing), the learned coarse step, and the same coarse step
without the network (the RKC2 base alone) -- each coarse scheme with the
plain-RK4 fallback, and reports the relative L2 error, the free-energy error
(f = (c^2 - 1)^2 / 4 convention: F + V/4), the fallback rate and the
speedup.  Initial data: c = cbar + U[-0.05, 0.05] with cbar ~ U[-0.3, 0.3],
one seeded numpy generator per trajectory.
"""
from __future__ import annotations

import time

import numpy as np

from . import (ENERGY_RTOL, CahnHilliardRhs, Corrector, Grid, RK4, ch_integrate, ch_rhs, ch_rkc,
               corrector_init_params, evaluate)

DT_FINE = 0.01
FINE_PER_COARSE = 16
BASE_STAGES = 6   # RKC2 stages: beta(6) = 22.9 >= 0.16 x 80 (spectral radius, 2-D order 2, |c| <= 1) x 1.7


def initial_condition(seed: int, size: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    cbar = rng.uniform(-0.3, 0.3)
    return cbar + 0.05 * (2.0 * rng.random((size, size)) - 1.0)


def train(net: Corrector, seeds, size: int = 512, fine_steps: int = 5000, batch: int = 16,
          lr: float = 2e-3, lr_final: float = 2e-4, log=None) -> dict:
    """Trains on trajectories of `fine_steps` fine steps for each seed, `batch`
    trajectories at a time; one Adam step per coarse interval."""
    import torch
    g = Grid(size, size, 1)
    rhs = CahnHilliardRhs(1.0, 1.0, 2)
    seeds = list(seeds)
    groups = [seeds[i:i + batch] for i in range(0, len(seeds), batch)]
    iters_per_group = fine_steps // FINE_PER_COARSE
    total = iters_per_group * len(groups)
    losses, k = [], 0
    t_data = t_train = 0.0
    for grp in groups:
        states = torch.from_numpy(np.stack([initial_condition(s, size) for s in grp])).cuda()
        for _ in range(iters_per_group):
            t0 = time.perf_counter()
            inp = states.clone()
            for b in range(states.shape[0]):
                ch_integrate(states[b], g, rhs, DT_FINE, FINE_PER_COARSE, RK4)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            frac = k / max(total - 1, 1)
            rate = lr * (lr_final / lr) ** frac
            losses.append(net.train_step(inp, states, rate))
            t2 = time.perf_counter()
            t_data += t1 - t0
            t_train += t2 - t1
            k += 1
            if log and k % 100 == 0:
                log(f"train iter {k}/{total} loss {losses[-1]:.3e}")
    return {"iterations": k, "trajectories": len(seeds), "fine_steps": fine_steps, "batch": batch,
            "loss_first": losses[0], "loss_last": float(np.mean(losses[-10:])),
            "seconds_data": t_data, "seconds_train": t_train}


def trapezoid_residual(c0, c1, g: Grid, rhs: CahnHilliardRhs, dt: float) -> float:
    """|(c1 - c0)/dt - (f(c0) + f(c1))/2| / |(f(c0) + f(c1))/2| with f the
    Cahn-Hilliard RHS: the acceptance test of gc_corrector_advance."""
    import torch
    fm = 0.5 * (ch_rhs(c0, g, rhs) + ch_rhs(c1, g, rhs))
    return float(torch.linalg.norm((c1 - c0) / dt - fm) / torch.linalg.norm(fm))


def residual_profile(net: Corrector, seeds, size: int = 512, times=(2.0, 10.0, 50.0, 100.0, 200.0)) -> dict:
    """At several times: the trapezoid residual of the true coarse pair
    (c(t), c(t + 16 dt)), of the base step alone and of the learned step,
    and the one-step errors |step - true| / |true - c| of both."""
    import torch
    g = Grid(size, size, 1)
    rhs = CahnHilliardRhs(1.0, 1.0, 2)
    dtc = DT_FINE * FINE_PER_COARSE
    rows = []
    for s in seeds:
        c = torch.from_numpy(initial_condition(s, size)).cuda()
        t_now = 0.0
        for t in times:
            n = int(round((t - t_now) / DT_FINE))
            ch_integrate(c, g, rhs, DT_FINE, n, RK4)
            t_now = t
            nxt = c.clone()
            ch_integrate(nxt, g, rhs, DT_FINE, FINE_PER_COARSE, RK4)
            base = c.clone()
            ch_rkc(base, g, rhs, dtc, 1, BASE_STAGES)
            cand = c + net.forward(c[None]).double()[0]
            step = torch.linalg.norm(nxt - c)
            rows.append({"seed": s, "t": t,
                         "residual_true": trapezoid_residual(c, nxt, g, rhs, dtc),
                         "residual_base": trapezoid_residual(c, base, g, rhs, dtc),
                         "residual_net": trapezoid_residual(c, cand, g, rhs, dtc),
                         "step_err_base": float(torch.linalg.norm(base - nxt) / step),
                         "step_err_net": float(torch.linalg.norm(cand - nxt) / step)})
    return {"rows": rows}


def _free_energy_baseline(psi, g: Grid) -> float:
    return evaluate(psi, g, "ch_free_energy", kappa=1.0) + g.size * g.cell_volume / 4.0


def evaluate_heldout(schemes, seeds, size: int = 512, t_end: float = 200.0, energy_tol: float = 0.0,
                     energy_rtol: float = ENERGY_RTOL) -> dict:
    """schemes: list of (name, corrector, residual_tol[, try_base]).  Per seed the plain
    fine RK4 reference runs once; every scheme advances the same initial
    state by coarse steps with the plain-RK4 fallback and is compared with
    it at t_end.  Fallbacks are also counted by cause (the proposal raised F
    beyond energy_tol + energy_rtol |F|, or its residual exceeded the
    scheme's tolerance; a proposal can fail both)."""
    import torch
    g = Grid(size, size, 1)
    rhs = CahnHilliardRhs(1.0, 1.0, 2)
    n_fine = int(round(t_end / DT_FINE))
    n_coarse = n_fine // FINE_PER_COARSE
    t_fine = 0.0
    schemes = [tuple(sc) + (True,) if len(sc) == 3 else tuple(sc) for sc in schemes]
    rec = {sc[0]: {"l2": [], "ferr": [], "acc": 0, "fb": 0, "rej_e": 0, "rej_r": 0, "acc_b": 0, "t": 0.0}
           for sc in schemes}
    for s in seeds:
        c0 = torch.from_numpy(initial_condition(s, size)).cuda()
        ref = c0.clone()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ch_integrate(ref, g, rhs, DT_FINE, n_coarse * FINE_PER_COARSE, RK4)
        torch.cuda.synchronize()
        t_fine += time.perf_counter() - t0
        fr = _free_energy_baseline(ref, g)
        for name, net, tol, try_base in schemes:
            r = rec[name]
            x = c0.clone()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            st = net.advance(x, g, rhs, n_coarse, DT_FINE, FINE_PER_COARSE, tol, energy_tol, energy_rtol, try_base)
            torch.cuda.synchronize()
            r["t"] += time.perf_counter() - t1
            r["acc"] += st["accepted"]
            r["fb"] += st["fallbacks"]
            r["rej_e"] += st["rejected_energy"]
            r["rej_r"] += st["rejected_residual"]
            r["acc_b"] += st["accepted_base"]
            r["l2"].append(float(torch.linalg.norm(x - ref) / torch.linalg.norm(ref)))
            r["ferr"].append(abs(_free_energy_baseline(x, g) - fr) / abs(fr))
    cells_steps = len(seeds) * size * size * n_coarse * FINE_PER_COARSE
    out = {"seeds": len(seeds), "t_end": t_end, "coarse_steps_per_scheme": n_coarse * len(seeds),
           "energy_tol": energy_tol, "energy_rtol": energy_rtol,
           "plain_mcell_steps": cells_steps / t_fine / 1e6, "schemes": {}}
    for name, _, tol, try_base in schemes:
        r = rec[name]
        total = r["acc"] + r["acc_b"] + r["fb"]
        out["schemes"][name] = {
            "residual_tol": tol, "try_base": try_base, "accepted": r["acc"], "accepted_base": r["acc_b"],
            "fallbacks": r["fb"], "fallback_rate": r["fb"] / max(total, 1),
            "rejected_energy": r["rej_e"], "rejected_residual": r["rej_r"],
            "l2_err_mean": float(np.mean(r["l2"])), "l2_err_max": float(np.max(r["l2"])),
            "f_err_mean": float(np.mean(r["ferr"])), "f_err_max": float(np.max(r["ferr"])),
            "mcell_steps_equiv": cells_steps / r["t"] / 1e6, "speedup_vs_plain": t_fine / r["t"]}
    return out


def new_corrector(size: int, batch: int, seed: int = 0, zero: bool = False) -> Corrector:
    """A corrector over the RKC2 base step, trained on the per-sample
    normalised loss.  zero: all-zero parameters, i.e. the base step alone."""
    net = Corrector(size, size, max_batch=batch)
    p = corrector_init_params(seed=seed, last_scale=0.1, inputs=3)
    net.set_params(np.zeros_like(p) if zero else p, s_out=1.0)
    net.set_base(CahnHilliardRhs(1.0, 1.0, 2), DT_FINE * FINE_PER_COARSE, BASE_STAGES)
    net.set_loss(True)
    return net
