"""Synthetics for SPECFEM coupling at many boundary points of one node on the GPU.

    python -m gemini_unified_b200.coupling_run --workload batched_fk --points 1000 --repeat 3

The command-line counterpart of the boundary-point loops of
computeSyntheticsForSpecfemCoupling (computeSynthetics and computeTension for
every point of one node).  The DSV spectra with radial derivatives come from
gem_fk_run_dsv for a moment source (or with ``--source FORCE`` a force) at the
workload's receiver node, evaluated at its deepest node.  The boundary points
are seeded: distances uniform in 5..90 degrees, azimuths uniform, unit normals
of random direction.  The node's complex elastic constants are fixed values of
a crustal solid.  Prints one JSON line with the device time per run of the
spectra form and of the time-series form.
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import json

import numpy as np

from . import configs, model as M
from .fk import GEM_BACKEND_GPU_FAST, CouplingParams, GeminiFK, lib

ELCON = np.array([1.1e11 + 1e8j, 1.2e11 + 1e8j, 4e10, 4.5e10 + 5e7j, 4.4e10, 0, 0])
MOMENT = np.array([1.0, -0.4, 0.7, 0.3, -0.5, 0.2])
FORCE = np.array([0.8, -0.3, 0.6])


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batched_fk", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--points", type=int, default=1000)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--source", default="MOMENT", choices=["MOMENT", "FORCE"])
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--backend", type=int, default=2, choices=[1, 2],
                    help="1 FP64 degree sums, 2 sliced-integer tensor-core degree sums")
    ap.add_argument("--check", action="store_true", help="also run the FP64 form and report the difference")
    a = ap.parse_args(argv)
    w = configs.WORKLOADS[a.workload]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    params = dataclasses.replace(w.params, source_type=a.source)
    istyp = 1 if a.source == "MOMENT" else 0
    fk = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    gre, gim, _, st = fk.run_dsv(params, jre, g.nf1, g.nf2, f64=False)
    ctxs = {2: fk, 1: GeminiFK(m, ex)}
    if np.any(st != 0):
        raise SystemExit("DSV spectra: %d items failed" % int(np.sum(st != 0)))
    nsp, nkf = gre.shape[1], gre.shape[2]
    rng = np.random.default_rng(a.seed)
    npts = a.points
    delta = np.radians(rng.uniform(5.0, 90.0, npts))
    xi = np.radians(rng.uniform(-180.0, 180.0, npts))
    nrm = rng.normal(size=(npts, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    zel = np.tile(ELCON, (g.nf2, 1))
    src = np.ascontiguousarray(MOMENT if istyp else FORCE)
    nsamp = 1 << int(np.ceil(np.log2(2 * g.nf2)))
    dt = 1.0 / (nsamp * g.df)
    dgr = torch.from_numpy(np.ascontiguousarray(gre[0])).cuda()
    dgi = torch.from_numpy(np.ascontiguousarray(gim[0])).cuda()
    nwn = np.ascontiguousarray(g.nwn, np.int32)
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    res = {"workload": a.workload, "source": a.source, "points": npts, "frequencies": g.nf2 - g.nf1 + 1,
           "degrees": nkf, "nsamp": nsamp, "backend": a.backend}
    outs = {}
    for spectra, be in ((1, a.backend), (0, a.backend)) + (((1, 1),) if a.check else ()):
        cp = CouplingParams(nf1=g.nf1, nf2=g.nf2, nwnmax=g.nwnmax, nkfmax=nkf, nsp=nsp, df=g.df, sigma=g.sigma,
                            re=ex.r[0], nsamp=nsamp, dt=dt, tred=0.0, order_highpass=2, fc_highpass=0.002,
                            order_lowpass=4, fc_lowpass=0.8 * g.nf2 * g.df, thetas=0.3, phis=1.0, thetac=0.5,
                            phic=1.2, spectra=spectra, istyp=istyp)
        n = npts * 6 * (2 * g.nf2 if spectra else nsamp)
        out = torch.zeros(n, dtype=torch.float64 if spectra else torch.float32, device="cuda")
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(a.repeat):
            torch.cuda.synchronize()
            t0.record()
            rc = lib().gem_coupling_run_device(ctxs[be]._h, ctypes.byref(cp), P(nwn), dgr.data_ptr(), dgi.data_ptr(),
                                               P(zel), P(src), npts, P(delta), P(xi), P(nrm),
                                               out.data_ptr() if spectra else None,
                                               None if spectra else out.data_ptr(), None)
            t1.record()
            torch.cuda.synchronize()
            if rc:
                raise SystemExit(lib().gem_last_error(ctxs[be]._h).decode())
            ms.append(t0.elapsed_time(t1))
        tag = ("spectra" if spectra else "traces") + ("" if be == a.backend else "_fp64")
        res[tag + "_ms"] = round(min(ms), 3)
        res["finite_" + tag] = bool(torch.isfinite(out).all().item())
        outs[tag] = out
    if a.check:   # largest difference relative to each (point, component) spectrum's peak
        got = outs["spectra"].view(npts, 6, g.nf2, 2)
        ref = outs["spectra_fp64"].view(npts, 6, g.nf2, 2)
        mag = torch.sqrt((ref ** 2).sum(-1))
        scale = mag.amax(dim=2, keepdim=True).clamp_min(1e-300)
        res["spectra_rel_diff_fp64"] = float((torch.sqrt(((got - ref) ** 2).sum(-1)) / scale).max().item())
    print(json.dumps(res))


if __name__ == "__main__":
    main()
