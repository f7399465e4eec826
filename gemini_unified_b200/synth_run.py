"""Seismograms of many stations from one node's FK spectra on the GPU.

    python -m gemini_unified_b200.synth_run --workload batched_fk --repeat 3

The command-line counterpart of computeSyntheticSeismograms (all stations of
the workload; six unit moment tensors, or with ``--source FORCE`` three unit
forces Fr, Ft, Ff).  The FK
spectra are seeded synthetic coefficients with the shape of the workload's
spectra: amplitudes log-normal with log10|c| ~ N(-3, 1) clipped to [-6, 0]
and uniform phases (``fk_coefficients``), or, with ``--fkfile PATH --node JR``,
the spectra of node JR of an FK-spectra file (HDF5, the reference's layout;
its frequency grid replaces the workload's, as readMetaGreenFKSpectra and
readDataNodeGreenFKSpectra give it to computeSyntheticSeismograms).  Prints
one JSON line with the device time per run.
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
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
    ap.add_argument("--backend", type=int, default=2, choices=[1, 2],
                    help="1 FP64 degree sums, 2 sliced-integer tensor-core degree sums")
    ap.add_argument("--check", action="store_true", help="also run the FP64 form and report the relative error")
    ap.add_argument("--source", default="MOMENT", choices=["MOMENT", "FORCE"])
    ap.add_argument("--fkfile", default="", help="FK-spectra file (HDF5) to take the spectra from")
    ap.add_argument("--node", type=int, default=0, help="external node of the file (1-based; default the deepest)")
    a = ap.parse_args(argv)
    w = configs.WORKLOADS[a.workload]
    m = w.model()
    g = M.frequency_grid(w.params, m.rearth)
    params = dataclasses.replace(w.params, source_type=a.source)
    nsp = M.nsp_for(params)
    if a.fkfile:
        from .fkfile import FKFile
        with FKFile(a.fkfile) as f:
            g = f.grid()
            gr, gi = f.read_node(a.node or 1)
            if f.meta.nsp != nsp:
                raise SystemExit("the file holds %d spectra per node, the %s source needs %d" % (f.meta.nsp, a.source,
                                                                                                 nsp))
    else:
        gr, gi = fk_coefficients(nsp, int(g.nkfmax))
    theta, phi, propdir = w.stations()
    if a.stations:
        theta, phi, propdir = theta[: a.stations], phi[: a.stations], propdir[: a.stations]
    theta, phi, propdir = (np.ascontiguousarray(x) for x in (theta, phi, propdir))
    mt = np.ascontiguousarray(configs.unit_moment_tensors() if a.source == "MOMENT" else np.eye(3), np.float64)
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs, global_=w.params.global_, rearth=m.rearth,
                      source_type=a.source)
    nwn = np.ascontiguousarray(g.nwn, np.int32)
    d_gr = torch.from_numpy(gr).cuda()
    d_gi = torch.from_numpy(gi).cuda()
    L = lib()
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)

    def run(backend, repeat):
        from .fk import Stats
        ctx = FrequencyTime(backend=backend)
        out = torch.empty((len(theta), len(mt), 3, w.nsamp), dtype=torch.float32, device="cuda")
        ms = []
        for _ in range(repeat):
            rc = L.gem_synth_run_device(ctx._h, ctypes.byref(sp), p(nwn), d_gr.data_ptr(), d_gi.data_ptr(),
                                        len(theta), p(theta), p(phi), p(propdir), len(mt), p(mt), out.data_ptr(), None)
            if rc >= 2:
                raise SystemExit(L.gem_last_error(ctx._h).decode())
            s = Stats()
            L.gem_stats_get(ctx._h, ctypes.byref(s))
            ms.append(s.synth_ms)
        return out, ms

    out, ms = run(a.backend, a.repeat)
    ntr = len(theta) * len(mt)
    res = {"workload": a.workload, "backend": a.backend, "source": a.source, "stations": len(theta), "sources": len(mt),
           "traces": ntr, "nsamp": w.nsamp, "synth_ms": ms, "traces_per_s": ntr / (min(ms) / 1e3),
           "finite": bool(torch.isfinite(out).all().item())}
    if a.check:
        ref, ms_ref = run(1, 1)
        res.update(trace_errors(out, ref))
        res["fp64_synth_ms"] = ms_ref[0]
    print(json.dumps(res))
    return 0


def trace_errors(got, ref) -> dict:
    """Relative L2 error of every 1-component trace (float64 norms) and of the whole set."""
    import torch
    g = got.double().reshape(-1, got.shape[-1])
    r = ref.double().reshape(-1, ref.shape[-1])
    scale = 1.0 / r.abs().max()
    g, r = g * scale, r * scale
    num = torch.linalg.vector_norm(g - r, dim=1)
    den = torch.linalg.vector_norm(r, dim=1)
    rel = (num / den).cpu().numpy()
    return {"rel_l2_trace_max": float(rel.max()), "rel_l2_trace_median": float(np.median(rel)),
            "rel_l2_all": float((torch.linalg.vector_norm(g - r) / torch.linalg.vector_norm(r)).item())}


if __name__ == "__main__":
    raise SystemExit(main())
