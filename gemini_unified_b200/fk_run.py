"""Compute the FK spectra of one frequency slab of a named workload on the GPU.

    python -m gemini_unified_b200.fk_run --workload batched_fk --jf 404:411 --backend 2 --repeat 2

The command-line counterpart of computeGreenFKSpectraForSynthetics for a slab
of frequencies (all wavenumbers, all external nodes); prints one JSON line with
the run's counters and times.  Used for profiling a slab of the batched
configuration (its highest frequencies carry the most work per frequency).

    python -m gemini_unified_b200.fk_run --workload batched_fk --jf 392:411 --aski all --repeat 2

``--aski`` runs the FK spectra of computeGreenFKSpectraForASKI instead: the
given source nodes ("all" or a comma list of 1-based indices, the receiver
node added if missing) plus the force at the receiver, as one set run
(gem_fk_run_aski), then, for comparison, as one gem_fk_run_dsv per source.
Both times are wall-clock times of the blocking calls on device buffers.
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import json
import time

import numpy as np

from . import configs, model as M
from .fk import GeminiFK, fk_params_c, lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batched_fk", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--jf", default="", help="first:last frequency index (1-based, inclusive); default all")
    ap.add_argument("--backend", type=int, default=2, choices=[1, 2], help="1 plain FP64, 2 fast FP64")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--aski", default="", help="source nodes of the ASKI spectra: 'all' or a comma list")
    ap.add_argument("--sched", default="", help="schedule index per phase (toroidal,spheroidal,adjoint), "
                    "see fk.SCHEDULES; default: the library's")
    ap.add_argument("--defer", default="", help="bookkeeping deferral index per phase, see fk.DEFERRALS")
    ap.add_argument("--queue", default="", help="queue granularity index per phase, see fk.GRANULARITIES")
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
    if a.sched:
        fk.schedule_set([int(x) for x in a.sched.split(",")])
    if a.defer:
        fk.defer_set([int(x) for x in a.defer.split(",")])
    if a.queue:
        fk.queue_set([int(x) for x in a.queue.split(",")])
    if a.aski:
        return aski(fk, w, ex, jre, lo, hi, a)
    best = None
    for _ in range(a.repeat):
        _, _, _, st = fk.run(w.params, jre, lo, hi, f32=True, f64=False)
        s = fk.stats()
        if best is None or s["solve_ms"] < best["solve_ms"]:
            best = s
    s = best
    print(json.dumps({"workload": a.workload, "jf": [lo, hi], "backend": a.backend, "items": int(s["items"]),
                      "schedule": fk.schedule(), "defer": fk.defer(), "queue": fk.queue(),
                      "phase_ms": [round(float(x), 3) for x in s["phase_ms"]],
                      "failed": int(np.count_nonzero(st)), "solve_ms": s["solve_ms"],
                      "solves_per_s": s["items"] / s["solve_ms"] * 1e3, "steps_ok": int(s["steps_ok"]),
                      "steps_rej": int(s["steps_rej"]), "attempts": int(s["attempts"]), "flops": int(s["flops"])}))
    return 0


def aski(fk, w, ex, jre, lo, hi, a):
    """Time the ASKI FK spectra of the slab: one set run against one DSV run per source."""
    import torch
    jsnod = list(range(1, ex.nnod + 1)) if a.aski == "all" else [int(x) for x in a.aski.split(",")]
    if jre not in jsnod:
        jsnod.append(jre)
    js = np.ascontiguousarray(jsnod, np.int32)
    g = M.frequency_grid(w.params, fk.model.rearth)
    nkf = int(g.nwn[lo - 1: hi].sum())
    nsp_m = M.nsp_dsv(w.params.source_type)
    ntot = ex.nnod * nkf * (len(js) * nsp_m + M.nsp_dsv("FORCE"))
    dre = torch.zeros(ntot, dtype=torch.float32, device="cuda")
    dim = torch.zeros(ntot, dtype=torch.float32, device="cuda")
    dst = torch.zeros(nkf, dtype=torch.int32, device="cuda")
    pc = fk_params_c(w.params, jre)
    t_set = []
    for _ in range(a.repeat):
        torch.cuda.synchronize()
        t = time.perf_counter()
        rc = lib().gem_fk_run_aski_device(fk._h, ctypes.byref(pc), len(js), js.ctypes.data_as(ctypes.c_void_p), lo,
                                          hi, dre.data_ptr(), dim.data_ptr(), None, dst.data_ptr(), None)
        torch.cuda.synchronize()
        t_set.append(time.perf_counter() - t)
        if rc:
            raise SystemExit(lib().gem_last_error(fk._h).decode())
    failed = int((dst != 0).sum().item())
    force = fk_params_c(dataclasses.replace(w.params, source_type="FORCE"), jre)
    t_node = []
    for _ in range(a.repeat):
        torch.cuda.synchronize()
        t = time.perf_counter()
        off = 0
        for b in range(len(js) + 1):
            q = force if b == len(js) else fk_params_c(w.params, int(js[b]))
            rc = lib().gem_fk_run_dsv_device(fk._h, ctypes.byref(q), lo, hi, dre.data_ptr() + 4 * off,
                                             dim.data_ptr() + 4 * off, None, dst.data_ptr(), None)
            if rc:
                raise SystemExit(lib().gem_last_error(fk._h).decode())
            off += ex.nnod * nkf * (M.nsp_dsv("FORCE") if b == len(js) else nsp_m)
        torch.cuda.synchronize()
        t_node.append(time.perf_counter() - t)
    print(json.dumps({"workload": a.workload, "jf": [lo, hi], "backend": a.backend, "degrees": nkf,
                      "sources": len(js) + 1, "nodes": ex.nnod, "failed": failed,
                      "set_run_s": round(min(t_set), 4), "per_source_runs_s": round(min(t_node), 4),
                      "solves_per_s_per_source": round(nkf * (len(js) + 1) / min(t_set))}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
