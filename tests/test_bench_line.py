"""bench.py's headline line must stay short (the driver keeps only the tail
of stdout): the form summaries it carries are checked on synthetic form
results, and a failing form is reported in one short entry."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_form_summaries_are_short():
    b = _bench()
    ops = {"f64_512": {k: {"frac": 0.123456789} for k in ("laplacian2", "gradient2", "divergence2", "biharmonic2",
                                                          "integrate", "evaluate_free_energy", "laplacian4")},
           "f32_512": {"laplacian2": {"frac": 0.3}}}
    scheme = {"speedup_vs_plain": 0.8619075162930939, "fallback_rate": 0.0073375, "l2_err_max": 0.000221999,
              "f_err_max": 2.50159e-06}
    forms = {
        "config1": {"Mcell-steps/s": 1776.123456, "cpu_baseline": {"value": 9.3265966}, "mass_drift": -7.7e-14,
                    "F_every_100_steps": [4096.0] * 21},
        "operators": {"results": ops},
        "fvm": {"Mcell-steps/s": 36840.5, "frac": 0.38241, "mass_drift_rel": 2.685e-09},
        "batched": {"Mcell-steps/s": 39330.2, "frac": 0.3122, "speedup_vs_plain_f32": 6.596,
                    "speedup_vs_plain_f64": 8.402, "accuracy": {"l2_err_max": 2.5e-6, "f_err_max": 1.4e-6}},
        "learned": {"train": {"trajectories": 512}, "eval": {"seeds": 64, "schemes": {
            "learned_tol0.003": scheme, "learned_tol0.01": scheme, "base_only_tol0.003": scheme,
            "base_only_tol0.01": scheme}}},
    }
    summary = {k: b.form_summary(k, v) for k, v in forms.items()}
    assert len(json.dumps(summary)) < 900, len(json.dumps(summary))
    assert set(summary["learned"]) == {"traj", "seeds", "learned", "base_only"}


def test_failing_form_is_one_short_entry():
    b = _bench()
    s = b.form_summary("batched", {"error": "RuntimeError: " + "x" * 5000})
    assert len(json.dumps(s)) < 200
