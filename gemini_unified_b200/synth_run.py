"""Seismograms of many stations from one node's FK spectra on the GPU.

    python -m gemini_unified_b200.synth_run --workload batched_fk --repeat 3

The command-line counterpart of computeSyntheticSeismograms for moment-tensor
sources (all stations of the workload, six unit moment tensors).  The FK
spectra are seeded synthetic coefficients with the shape of the workload's
spectra: amplitudes log-normal with log10|c| ~ N(-3, 1) clipped to [-6, 0]
and uniform phases (``fk_coefficients``).  Prints one JSON line with the
device time per run.
"""
from __future__ import annotations

import argparse
import ctypes
import json

import numpy as np

from . import configs, model as M
from .fk import FrequencyTime, lib, synth_params


def fk_coefficients(nsp: int, nkf: int, seed: int = 2024):
    """float32 (re, im) spectra [nsp, nkf]: log-normal amplitudes, uniform phases."""
    rng = np.random.default_rng(seed)
    amp = 10.0 ** np.clip(rng.normal(-3.0, 1.0, size=(nsp, nkf)), -6.0, 0.0)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(nsp, nkf))
    return (amp * np.cos(ph)).astype(np.float32), (amp * np.sin(ph)).astype(np.float32)


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batched_fk", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--stations", type=int, default=0, help="first N stations only (0 = all)")
    a = ap.parse_args(argv)
    w = configs.WORKLOADS[a.workload]
    m = w.model()
    g = M.frequency_grid(w.params, m.rearth)
    nsp = M.nsp_for(w.params)
    gr, gi = fk_coefficients(nsp, int(g.nkfmax))
    theta, phi, propdir = w.stations()
    if a.stations:
        theta, phi, propdir = theta[: a.stations], phi[: a.stations], propdir[: a.stations]
    theta, phi, propdir = (np.ascontiguousarray(x) for x in (theta, phi, propdir))
    mt = np.ascontiguousarray(configs.unit_moment_tensors(), np.float64)
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs)
    nwn = np.ascontiguousarray(g.nwn, np.int32)
    ctx = FrequencyTime()
    d_gr = torch.from_numpy(gr).cuda()
    d_gi = torch.from_numpy(gi).cuda()
    out = torch.empty((len(theta), len(mt), 3, w.nsamp), dtype=torch.float32, device="cuda")
    L = lib()
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    ms = []
    for _ in range(a.repeat):
        rc = L.gem_synth_run_device(ctx._h, ctypes.byref(sp), p(nwn), d_gr.data_ptr(), d_gi.data_ptr(), len(theta),
                                    p(theta), p(phi), p(propdir), len(mt), p(mt), out.data_ptr(), None)
        if rc >= 2:
            raise SystemExit(L.gem_last_error(ctx._h).decode())
        from .fk import Stats
        s = Stats()
        L.gem_stats_get(ctx._h, ctypes.byref(s))
        ms.append(s.synth_ms)
    ntr = len(theta) * len(mt)
    print(json.dumps({"workload": a.workload, "stations": len(theta), "moment_tensors": len(mt), "traces": ntr,
                      "nsamp": w.nsamp, "synth_ms": ms, "traces_per_s": ntr / (min(ms) / 1e3),
                      "finite": bool(torch.isfinite(out).all().item())}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
