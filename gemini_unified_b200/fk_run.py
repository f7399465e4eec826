"""Compute the FK spectra of one frequency slab of a named workload on the GPU.

    python -m gemini_unified_b200.fk_run --workload batched_fk --jf 404:411 --backend 2 --repeat 2

The command-line counterpart of computeGreenFKSpectraForSynthetics for a slab
of frequencies (all wavenumbers, all external nodes); prints one JSON line with
the run's counters and times.  Used for profiling a slab of the batched
configuration (its highest frequencies carry the most work per frequency).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import configs, model as M
from .fk import GeminiFK


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batched_fk", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--jf", default="", help="first:last frequency index (1-based, inclusive); default all")
    ap.add_argument("--backend", type=int, default=2, choices=[1, 2], help="1 plain FP64, 2 fast FP64")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    w = configs.WORKLOADS[a.workload]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    lo, hi = (g.nf1, g.nf2) if not a.jf else (int(x) for x in a.jf.split(":"))
    if not (g.nf1 <= lo <= hi <= g.nf2):
        raise SystemExit("frequency range %d:%d outside %d:%d" % (lo, hi, g.nf1, g.nf2))
    fk = GeminiFK(m, ex, backend=a.backend)
    for _ in range(a.repeat):
        _, _, _, st = fk.run(w.params, jre, lo, hi, f32=True, f64=False)
    s = fk.stats()
    print(json.dumps({"workload": a.workload, "jf": [lo, hi], "backend": a.backend, "items": int(s["items"]),
                      "failed": int(np.count_nonzero(st)), "solve_ms": s["solve_ms"],
                      "solves_per_s": s["items"] / s["solve_ms"] * 1e3, "steps_ok": int(s["steps_ok"]),
                      "steps_rej": int(s["steps_rej"]), "attempts": int(s["attempts"]), "flops": int(s["flops"])}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
