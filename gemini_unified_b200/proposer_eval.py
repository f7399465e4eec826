"""Evaluation of the learned step/order proposer on a whole workload.

    python -m gemini_unified_b200.proposer_eval --workload body_waves [--slab 64] [--out eval.json]

Runs the fast FP64 solver over every frequency of the workload, slab by slab,
three ways: without the proposer, with its order targets, and with its order
targets and initial steps.  It prints one JSON record with, per way:
* device solve time, summed over the slabs;
* accepted and rejected steps, and extrapolation attempts per accepted step;
* lane use of the lockstep phase kernels (instrumentation counters): lanes
  integrating per warp trip, and lanes computing per extrapolation attempt;
* items that ended with a non-zero status (step below the minimum, 200,000
  steps);
and the spectral difference of each proposer run against the run without it,
relative to each (node, spectrum) spectrum's peak in its frequency, over the
items both runs solved.  The proposer only moves the step sequence; the error
control still accepts or rejects every step.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import configs, model as M
from . import proposer
from .fk import GEM_BACKEND_GPU_FAST, GeminiFK

WAYS = (("without", 0), ("order", proposer.USE_ORDER), ("order+steps", proposer.USE_ORDER | proposer.USE_STEP))


def evaluate(workload: str, slab: int = 64, weights: str = proposer.WEIGHTS, margin: float = 0.1, jf=None):
    w = configs.WORKLOADS[workload]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    ctx = {}
    for name, use in WAYS:
        fk = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
        if use:
            proposer.enable(fk, weights, use, margin)
        fk.instrument(True)
        ctx[name] = fk
    tot = {name: dict(solve_ms=0.0, steps_ok=0, steps_rej=0, attempts=0, failed=0, trips=np.zeros(3),
                      lanes=np.zeros(3), att_iter=np.zeros(3), att_lanes=np.zeros(3)) for name, _ in WAYS}
    err = {name: 0.0 for name, use in WAYS if use}
    items = 0
    lo, hi = jf if jf else (g.nf1, g.nf2)
    for a in range(lo, hi + 1, slab):
        b = min(a + slab - 1, hi)
        koff = np.concatenate([[0], np.cumsum(g.nwn[a - 1: b])])
        out = {}
        for name, _ in WAYS:
            fk = ctx[name]
            _, _, g64, st = fk.run(w.params, jre, a, b, f32=False, f64=True, raise_on_failure=False)
            s = fk.stats()
            prof, _ = fk.instrument_read()
            t = tot[name]
            t["solve_ms"] += s["solve_ms"]
            t["steps_ok"] += int(s["steps_ok"]); t["steps_rej"] += int(s["steps_rej"])
            t["attempts"] += int(s["attempts"])
            t["failed"] += int(np.count_nonzero(st))
            for ph in range(3):
                t["trips"][ph] += float(prof[8 * ph]); t["lanes"][ph] += float(prof[8 * ph + 1])
                t["att_iter"][ph] += float(prof[8 * ph + 2]); t["att_lanes"][ph] += float(prof[8 * ph + 3])
            out[name] = (g64, st)
        ref, st0 = out["without"]
        items += ref.shape[2]
        for name in err:
            got, st1 = out[name]
            ok = (st0 == 0) & (st1 == 0)
            for jf in range(a, b + 1):
                k0, k1 = int(koff[jf - a]), int(koff[jf - a + 1])
                sel = np.nonzero(ok[k0:k1])[0] + k0
                if not len(sel):
                    continue
                r = ref[:, :, sel]
                scale = np.nanmax(np.abs(r), axis=-1, keepdims=True)
                d = np.abs(got[:, :, sel] - r) / np.maximum(scale, 1e-300)
                err[name] = max(err[name], float(np.nanmax(d)))
    res = {"workload": workload, "jf": [int(lo), int(hi)], "frequencies": int(hi - lo + 1), "items": int(items),
           "lmax": int(g.nwn.max() - 1), "weights": weights, "margin": margin, "ways": {}}
    for name, _ in WAYS:
        t = tot[name]
        res["ways"][name] = {
            "solve_ms": t["solve_ms"], "steps_ok": t["steps_ok"], "steps_rej": t["steps_rej"],
            "attempts_per_step": t["attempts"] / max(1, t["steps_ok"] + t["steps_rej"]),
            "failed_items": t["failed"],
            "lanes_integrating_per_trip": (t["lanes"] / np.maximum(t["trips"], 1) / 32).round(4).tolist(),
            "lanes_per_attempt": (t["att_lanes"] / np.maximum(t["att_iter"], 1) / 32).round(4).tolist(),
        }
    base = res["ways"]["without"]["solve_ms"]
    for name in err:
        res["ways"][name]["speedup"] = base / res["ways"][name]["solve_ms"]
        res["ways"][name]["spectral_diff_vs_without"] = err[name]
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="body_waves", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--slab", type=int, default=64)
    ap.add_argument("--weights", default=proposer.WEIGHTS)
    ap.add_argument("--margin", type=float, default=0.1)
    ap.add_argument("--out", default="")
    ap.add_argument("--jf", default="", help="first:last frequency index (default: the whole band)")
    a = ap.parse_args(argv)
    res = evaluate(a.workload, a.slab, a.weights, a.margin, tuple(int(x) for x in a.jf.split(":")) if a.jf else None)
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
