"""ctypes binding of libgemini_fk.so: FK spectra on the GPU.

The host-side counterpart of computeGreenFKSpectraForSynthetics
(f90/computeGreenFKSpectraForSynthetics.f90): load the earth model and the
external nodes once, then compute the FK spectra gf(iwn, isp, node) of any
frequency slab in one call.  There is no CPU path: without the CUDA library
or a GPU every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from .model import (ExternalRadialNodes, FKParams, GeminiError, NodeEarthModel, aski_nf1, fk_params_c,
                    frequency_grid, nsp_dsv, nsp_for)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libgemini_fk.so")

GEM_BACKEND_GPU_FP64 = 1
GEM_BACKEND_GPU_FAST = 2
# solver schedules (include/gemini_fk.h): threads per block and whether the 4-
# and 5-variable systems keep their half- and end-step matrices (fast backend)
SCHEDULES = [(384, False), (512, False), (256, False), (384, True), (512, True), (256, True)]
NSCHED = len(SCHEDULES)
# bookkeeping deferrals (lanes waiting, steps waited)
DEFERRALS = [(1, 0), (8, 6), (16, 10), (32, 24), (32, 48), (32, 1000000)]
NDEFER = len(DEFERRALS)
# queue granularities: (positions a lane reserves per fetch, positions of the
# runs the warps of a block share; 0: none)
GRANULARITIES = [(1, 0), (2, 0), (4, 0), (1, 1024)]
NGRAN = len(GRANULARITIES)
STATUS_TEXT = {0: "ok", 1: "step size smaller than minimum", 2: "maximum number of steps reached",
               3: "continued fraction did not converge", 4: "node/discontinuity bookkeeping",
               5: "non-finite value", 7: "ocean receiver or source not supported"}


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("steps_ok", "steps_rej", "attempts", "sysmats", "matvecs", "flops", "items", "failed")] + \
               [("solve_ms", ctypes.c_double), ("prep_ms", ctypes.c_double), ("synth_ms", ctypes.c_double),
                ("phase_flops", ctypes.c_int64 * 3), ("phase_ms", ctypes.c_double * 3)]

    def asdict(self):
        return {n: (list(getattr(self, n)) if n.startswith("phase") else getattr(self, n)) for n, _ in self._fields_}


_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library; raise loudly when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GeminiError("libgemini_fk.so is not built (python -m gemini_unified_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p
        L.gem_ctx_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
        L.gem_ctx_destroy.argtypes = [vp]
        L.gem_ctx_destroy.restype = None
        L.gem_last_error.argtypes = [vp]
        L.gem_last_error.restype = ctypes.c_char_p
        L.gem_model_load.argtypes = [vp, vp]
        L.gem_nodes_set.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.gem_fk_grid.argtypes = [vp, vp, ip, ip, ip, ip, vp, ctypes.c_int]
        L.gem_fk_run.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
        L.gem_fk_run_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp]
        L.gem_fk_run_dsv.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
        L.gem_fk_run_dsv_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp]
        L.gem_fk_run_aski.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
        L.gem_coupling_run.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp, vp]
        L.gem_coupling_run_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp, vp, vp]
        L.gem_fk_run_aski_device.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp,
                                             vp]
        L.gem_stats_get.argtypes = [vp, ctypes.POINTER(Stats)]
        L.gem_fk_graph_build.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
        L.gem_fk_graph_launch.argtypes = [vp, vp]
        L.gem_synth_run.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp]
        L.gem_synth_run_device.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, vp]
        L.gem_synth_run_opts.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, vp]
        L.gem_synth_run_device_opts.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp,
                                                vp, vp]
        L.gem_ifft_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, vp]
        L.gem_ifft_run_device.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, vp, vp]
        L.gem_steplog.argtypes = [vp, ctypes.c_longlong]
        L.gem_steplog_read.argtypes = [vp, vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
        L.gem_order_target.argtypes = [vp, ctypes.c_int]
        L.gem_tc_wait_limit.argtypes = [vp, ctypes.c_longlong]
        L.gem_ray_table.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int), vp, vp, vp, vp]
        L.gem_travel_times.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_int, vp, vp, vp]
        L.gem_fk_schedule_set.argtypes = [vp, vp]
        L.gem_fk_schedule_get.argtypes = [vp, vp]
        L.gem_fk_autotune.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.gem_fk_defer_set.argtypes = [vp, vp]
        L.gem_fk_defer_get.argtypes = [vp, vp]
        L.gem_fk_queue_set.argtypes = [vp, vp]
        L.gem_fk_queue_get.argtypes = [vp, vp]
        L.gem_instrument.argtypes = [vp, ctypes.c_int]
        L.gem_instrument_read.argtypes = [vp, vp, vp, ctypes.POINTER(ctypes.c_int)]
        _lib = L
    return _lib


# one Bulirsch-Stoer step attempt of the step log (StepRec, 32 bytes)
STEP_DTYPE = np.dtype([("x", "<f8"), ("h", "<f8"), ("k", "<i4"), ("lgy", "<f4"), ("nl", "<i2"), ("sys", "i1"),
                       ("result", "i1"), ("phase", "<i2"), ("nstep", "<i2")])
assert STEP_DTYPE.itemsize == 32


class CouplingParams(ctypes.Structure):
    """C layout of ``gem_coupling_params`` (include/gemini_fk.h)."""
    _fields_ = [("nf1", ctypes.c_int), ("nf2", ctypes.c_int), ("nwnmax", ctypes.c_int),
                ("nkfmax", ctypes.c_longlong), ("nsp", ctypes.c_int), ("df", ctypes.c_double),
                ("sigma", ctypes.c_double), ("re", ctypes.c_double), ("nsamp", ctypes.c_int),
                ("dt", ctypes.c_double), ("tred", ctypes.c_double), ("order_highpass", ctypes.c_int),
                ("fc_highpass", ctypes.c_double), ("order_lowpass", ctypes.c_int), ("fc_lowpass", ctypes.c_double),
                ("thetas", ctypes.c_double), ("phis", ctypes.c_double), ("thetac", ctypes.c_double),
                ("phic", ctypes.c_double), ("spectra", ctypes.c_int), ("istyp", ctypes.c_int)]

    def __init__(self, **kw):
        kw.setdefault("istyp", 1)
        super().__init__(**kw)


class SynthParams(ctypes.Structure):
    """C layout of ``gem_synth_params`` (include/gemini_fk.h)."""

    _fields_ = [("nf1", ctypes.c_int), ("nf2", ctypes.c_int), ("nwnmax", ctypes.c_int),
                ("nkfmax", ctypes.c_longlong), ("nsp", ctypes.c_int), ("istyp", ctypes.c_int),
                ("global_", ctypes.c_int), ("df", ctypes.c_double), ("sigma", ctypes.c_double),
                ("nsamp", ctypes.c_int), ("dt", ctypes.c_double), ("velocity", ctypes.c_int),
                ("tred", ctypes.c_double), ("order_highpass", ctypes.c_int), ("fc_highpass", ctypes.c_double),
                ("order_lowpass", ctypes.c_int), ("fc_lowpass", ctypes.c_double), ("dwn", ctypes.c_double),
                ("rearth", ctypes.c_double)]


class StationOpts(ctypes.Structure):
    """C layout of ``gem_synth_station_opts`` (include/gemini_fk.h)."""

    _fields_ = [("tred", ctypes.c_void_p), ("nsamp_true", ctypes.c_void_p), ("stafilter", ctypes.c_void_p),
                ("nstf", ctypes.c_int), ("tanf_stf", ctypes.c_double), ("stf", ctypes.c_void_p)]


def synth_params(grid, nsp, nsamp, dt, filspecs, velocity=False, tred=0.0, global_=1,
                 rearth=6371000.0, source_type="MOMENT") -> SynthParams:
    """Parameters as computeSyntheticSeismograms reads them back from the FK file:
    df, sigma, dwn and the earth radius are stored as float32
    (computeGreenFKSpectraForSynthetics.f90:261-263).  source_type "MOMENT"
    (istyp 1, sources are moment tensors) or "FORCE" (istyp 0, single forces)."""
    f32 = lambda v: float(np.float32(v))
    istyp = {"FORCE": 0, "MOMENT": 1}[source_type]
    return SynthParams(grid.nf1, grid.nf2, int(grid.nwnmax), int(grid.nkfmax), nsp, istyp, int(global_), f32(grid.df),
                       f32(grid.sigma), int(nsamp), float(dt), 1 if velocity else 0, float(tred),
                       int(round(filspecs[0])), float(filspecs[1]), int(round(filspecs[2])), float(filspecs[3]),
                       f32(grid.dwn), f32(rearth))


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class FrequencyTime:
    """Batched transformFrequencyTime (f90/frequencyTime.f90:55-113) on one GPU."""

    def __init__(self, device: int = 0, backend: int = GEM_BACKEND_GPU_FP64):
        self._h = ctypes.c_void_p()
        rc = lib().gem_ctx_create(device, backend, ctypes.byref(self._h))
        if rc != 0 or not self._h:
            raise GeminiError("gem_ctx_create failed (no CUDA device %d)" % device)
        self.warning = None

    def _check(self, rc: int):
        self.warning = lib().gem_last_error(self._h).decode() if rc == 1 else None
        if rc >= 2:
            raise GeminiError(lib().gem_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            lib().gem_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def run(self, nf1: int, nf2: int, df: float, sigma: float, sp: np.ndarray, nsamp: int, dt: float) -> np.ndarray:
        """sp: complex [ntr, ldsp >= nf2] (column j is frequency j*df) -> float32 [ntr, nsamp]."""
        sp = np.ascontiguousarray(sp, np.complex128)
        ntr, ld = sp.shape
        ts = np.zeros((ntr, nsamp), np.float32)
        self._check(lib().gem_ifft_run(self._h, nf1, nf2, df, sigma, ntr, _ptr(sp), ld, nsamp, dt, _ptr(ts)))
        return ts

    def run_device(self, nf1, nf2, df, sigma, ntr, d_sp: int, ldsp: int, nsamp, dt, d_ts: int, stream: int = 0):
        """Same on device buffers (integer device pointers)."""
        return self._check(lib().gem_ifft_run_device(self._h, nf1, nf2, df, sigma, ntr, d_sp, ldsp, nsamp, dt,
                                                     d_ts, stream or None))


class GeminiFK:
    """One GPU context with an earth model and external radial nodes loaded."""

    def __init__(self, model: NodeEarthModel, nodes: ExternalRadialNodes, device: int = 0,
                 backend: int = GEM_BACKEND_GPU_FP64):
        self._h = ctypes.c_void_p()
        rc = lib().gem_ctx_create(device, backend, ctypes.byref(self._h))
        if rc != 0 or not self._h:
            raise GeminiError("gem_ctx_create failed (no CUDA device %d or unsupported backend)" % device)
        self.model, self.nodes = model, nodes
        self._desc = model.desc()
        self._check(lib().gem_model_load(self._h, ctypes.byref(self._desc)))
        self._r = np.ascontiguousarray(nodes.r, np.float64)
        self._s = np.ascontiguousarray(nodes.state, np.int32)
        self._l = np.ascontiguousarray(nodes.layer, np.int32)
        self._check(lib().gem_nodes_set(self._h, len(self._r), _ptr(self._r), _ptr(self._s), _ptr(self._l)))

    def _check(self, rc: int):
        if rc >= 2:
            raise GeminiError(lib().gem_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            lib().gem_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def grid(self, params: FKParams, jre: int):
        pc = fk_params_c(params, jre)
        nf1, nf2, nwnmax, nsp = (ctypes.c_int() for _ in range(4))
        cap = 1 << 20
        nwn = np.zeros(cap, np.int32)
        self._check(lib().gem_fk_grid(self._h, ctypes.byref(pc), ctypes.byref(nf1), ctypes.byref(nf2),
                                      ctypes.byref(nwnmax), ctypes.byref(nsp), _ptr(nwn), cap))
        return nf1.value, nf2.value, nwnmax.value, nsp.value, nwn[: nf2.value].copy()

    def run(self, params: FKParams, jre: int, jf_first: int, jf_last: int, f32: bool = True,
            f64: bool = True, raise_on_failure: bool = True, out=None):
        """FK spectra of frequencies jf_first..jf_last.

        Returns (gfre, gfim, gf64, status) with gf arrays shaped
        (nnod, nsp, nkf) -- the transpose view of the Fortran (nkf, nsp, nnod)
        layout -- and status per wavenumber-frequency index k.  out: optional
        caller-owned float32 (gfre, gfim) arrays of that shape (for example in
        pinned memory) that receive the float32 spectra.
        """
        grid = frequency_grid(params, self.model.rearth)
        nkf = int(grid.nwn[jf_first - 1: jf_last].sum())
        nsp = nsp_for(params)
        nnod = self.nodes.nnod
        pc = fk_params_c(params, jre)
        if out is not None and f32:
            gre, gim = out
            for a in (gre, gim):
                if a.dtype != np.float32 or a.shape != (nnod, nsp, nkf) or not a.flags.c_contiguous:
                    raise GeminiError("out arrays must be C-contiguous float32 of shape %s" % ((nnod, nsp, nkf),))
        else:
            gre = np.zeros((nnod, nsp, nkf), np.float32) if f32 else None
            gim = np.zeros((nnod, nsp, nkf), np.float32) if f32 else None
        g64 = np.zeros((nnod, nsp, nkf), np.complex128) if f64 else None
        status = np.zeros(nkf, np.int32)
        rc = lib().gem_fk_run(self._h, ctypes.byref(pc), jf_first, jf_last, _ptr(gre), _ptr(gim), _ptr(g64),
                              _ptr(status))
        if rc >= 2 and (raise_on_failure or not np.any(status)):
            raise GeminiError(lib().gem_last_error(self._h).decode())
        return gre, gim, g64, status

    def run_dsv(self, params: FKParams, jsrc: int, jf_first: int, jf_last: int, f32: bool = True,
                f64: bool = True, raise_on_failure: bool = True):
        """DSV spectra with radial derivatives of a source at node jsrc (type
        params.source_type), the body of the source-node loop of
        computeGreenFKSpectraForASKI.f90:451-541.  Returns (gfre, gfim, gf64,
        status) shaped (nnod, nsp, nkf) with nsp = nsp_dsv(source type): U, V
        for each spheroidal jump, then dU/dr, dV/dr, then W and dW/dr."""
        grid = frequency_grid(params, self.model.rearth)
        nkf = int(grid.nwn[jf_first - 1: jf_last].sum())
        nsp = nsp_dsv(params.source_type)
        nnod = self.nodes.nnod
        pc = fk_params_c(params, jsrc)
        gre = np.zeros((nnod, nsp, nkf), np.float32) if f32 else None
        gim = np.zeros((nnod, nsp, nkf), np.float32) if f32 else None
        g64 = np.zeros((nnod, nsp, nkf), np.complex128) if f64 else None
        status = np.zeros(nkf, np.int32)
        rc = lib().gem_fk_run_dsv(self._h, ctypes.byref(pc), jf_first, jf_last, _ptr(gre), _ptr(gim), _ptr(g64),
                                  _ptr(status))
        if rc >= 2 and (raise_on_failure or not np.any(status)):
            raise GeminiError(lib().gem_last_error(self._h).decode())
        return gre, gim, g64, status

    def aski_spectra(self, params: FKParams, jsnod, jre: int, jf_first: int, jf_last: int, f32: bool = True,
                     f64: bool = True, raise_on_failure: bool = True):
        """The FK spectra of computeGreenFKSpectraForASKI for frequencies
        jf_first..jf_last in one call (gem_fk_run_aski): the minors once over the
        source-node range, then the DSV spectra of each source node in jsnod
        (type params.source_type) and of a force at the receiver node jre, which
        must be among the source nodes (:196-209).  Returns a list of (gfre,
        gfim, gf64, status) shaped (nnod, nsp, nkf), the force last, as the
        program's files <DSVBASENAME>.<type>.<js> hold them."""
        jsnod = np.ascontiguousarray([int(j) for j in jsnod], np.int32)
        if jre not in list(jsnod):
            raise GeminiError("receiver node must also be a source node")
        if jf_first < aski_nf1(params):
            raise GeminiError("frequency index %d below the first ASKI frequency %d" % (jf_first, aski_nf1(params)))
        grid = frequency_grid(params, self.model.rearth)
        nkf = int(grid.nwn[jf_first - 1: jf_last].sum())
        nnod = self.nodes.nnod
        nsp_m, nsp_f = nsp_dsv(params.source_type), nsp_dsv("FORCE")
        ntot = nnod * nkf * (len(jsnod) * nsp_m + nsp_f)
        gre = np.zeros(ntot, np.float32) if f32 else None
        gim = np.zeros(ntot, np.float32) if f32 else None
        g64 = np.zeros(ntot, np.complex128) if f64 else None
        status = np.zeros(nkf, np.int32)
        pc = fk_params_c(params, jre)
        rc = lib().gem_fk_run_aski(self._h, ctypes.byref(pc), len(jsnod), _ptr(jsnod), jf_first, jf_last, _ptr(gre),
                                   _ptr(gim), _ptr(g64), _ptr(status))
        if rc >= 2 and (raise_on_failure or not np.any(status)):
            raise GeminiError(lib().gem_last_error(self._h).decode())
        out, off = [], 0
        for b in range(len(jsnod) + 1):
            nsp = nsp_f if b == len(jsnod) else nsp_m
            n = nnod * nsp * nkf
            blk = [None if a is None else a[off:off + n].reshape(nnod, nsp, nkf) for a in (gre, gim, g64)]
            out.append((blk[0], blk[1], blk[2], status))
            off += n
        return out

    def run_device(self, params: FKParams, jre: int, jf_first: int, jf_last: int, gfre=None, gfim=None,
                   gf64=None, status=None, stream: int = 0):
        """Same on caller-provided device buffers (integer device pointers)."""
        pc = fk_params_c(params, jre)
        self._check(lib().gem_fk_run_device(self._h, ctypes.byref(pc), jf_first, jf_last, gfre, gfim, gf64,
                                            status, stream or None))

    def graph_build(self, params: FKParams, jre: int, jf_first: int, jf_last: int, gfre=None, gfim=None,
                    gf64=None, status=None):
        """Capture the device work of a slab into a CUDA graph (device output pointers as in run_device)."""
        pc = fk_params_c(params, jre)
        self._check(lib().gem_fk_graph_build(self._h, ctypes.byref(pc), jf_first, jf_last, gfre, gfim, gf64, status))

    def graph_launch(self, stream: int = 0):
        """Replay the captured slab on a stream (asynchronous)."""
        self._check(lib().gem_fk_graph_launch(self._h, stream or None))

    def synthetics(self, sp: SynthParams, nwn, gfkr, gfki, theta, phi, propdir, mt, tred=None, nsamp_true=None,
                   stafilter=None, stf=None, tanf_stf=0.0):
        """Seismograms of all stations x sources: float32 [nsta, nsrc, 3 (Z,N,E), nsamp].

        gfkr/gfki: float32 FK spectra of the source node, shaped (nsp, nkfmax).
        mt: moment tensors (nsrc, 6) for sp.istyp 1, forces (nsrc, 3) as
        (Fr, Ft, Ff) for sp.istyp 0.  Per-station options of the station loop
        (gem_synth_station_opts): tred [nsta] reduction times, nsamp_true [nsta]
        samples kept, stafilter complex [nsta, 3, nf2], stf float32 source wavelet
        whose first sample is at tanf_stf."""
        keep = []
        opts = None
        if tred is not None or nsamp_true is not None or stafilter is not None or stf is not None:
            conv = lambda a, t: None if a is None else np.ascontiguousarray(a, t)
            arrs = [conv(tred, np.float64), conv(nsamp_true, np.int32), conv(stafilter, np.complex128),
                    conv(stf, np.float32)]
            keep += arrs
            opts = StationOpts(_ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), 0 if arrs[3] is None else len(arrs[3]),
                               float(tanf_stf), _ptr(arrs[3]))
        gr = np.ascontiguousarray(gfkr, np.float32); gi = np.ascontiguousarray(gfki, np.float32)
        nwn = np.ascontiguousarray(nwn, np.int32)
        th = np.ascontiguousarray(theta, np.float64); ph = np.ascontiguousarray(phi, np.float64)
        pd = np.ascontiguousarray(propdir, np.float64)
        mt = np.ascontiguousarray(mt, np.float64).reshape(-1, 6 if sp.istyp == 1 else 3)
        out = np.zeros((len(th), len(mt), 3, sp.nsamp), np.float32)
        if opts is None:
            self._check(lib().gem_synth_run(self._h, ctypes.byref(sp), _ptr(nwn), _ptr(gr), _ptr(gi), len(th),
                                            _ptr(th), _ptr(ph), _ptr(pd), len(mt), _ptr(mt), _ptr(out)))
        else:
            self._check(lib().gem_synth_run_opts(self._h, ctypes.byref(sp), _ptr(nwn), _ptr(gr), _ptr(gi), len(th),
                                                 _ptr(th), _ptr(ph), _ptr(pd), len(mt), _ptr(mt),
                                                 ctypes.byref(opts), _ptr(out)))
        return out

    def coupling(self, cp: CouplingParams, nwn, gr, gi, zelcon, mt, delta, xi, nrm):
        """Synthetics for SPECFEM coupling (gem_coupling_run) at boundary points
        of one node: gr/gi float32 (nsp, nkfmax) DSV spectra with derivatives,
        zelcon complex [nf2, 7].  Returns complex spectra [npts, 6, nf2] when
        cp.spectra, else float32 traces [npts, 6, nsamp] (velocity x, y, z,
        traction x, y, z in the box frame)."""
        gr = np.ascontiguousarray(gr, np.float32)
        gi = np.ascontiguousarray(gi, np.float32)
        nwn = np.ascontiguousarray(nwn, np.int32)
        zel = np.ascontiguousarray(zelcon, np.complex128)
        mt = np.ascontiguousarray(mt, np.float64)
        delta = np.ascontiguousarray(delta, np.float64)
        xi = np.ascontiguousarray(xi, np.float64)
        nrm = np.ascontiguousarray(nrm, np.float64)
        npts = len(delta)
        if gr.shape != (cp.nsp, cp.nkfmax) or gi.shape != gr.shape or zel.shape != (cp.nf2, 7) or \
                nrm.shape != (npts, 3) or len(xi) != npts or len(nwn) < cp.nf2 or len(mt) != (6 if cp.istyp else 3):
            raise GeminiError("coupling: inconsistent input shapes")
        spec = np.zeros((npts, 6, cp.nf2), np.complex128) if cp.spectra else None
        tr = None if cp.spectra else np.zeros((npts, 6, cp.nsamp), np.float32)
        self._check(lib().gem_coupling_run(self._h, ctypes.byref(cp), _ptr(nwn), _ptr(gr), _ptr(gi), _ptr(zel),
                                           _ptr(mt), npts, _ptr(delta), _ptr(xi), _ptr(nrm), _ptr(spec), _ptr(tr)))
        return spec if cp.spectra else tr

    def schedule(self):
        """Schedule index per phase (toroidal, spheroidal, adjoint); see SCHEDULES."""
        s = (ctypes.c_int * 3)()
        self._check(lib().gem_fk_schedule_get(self._h, s))
        return [int(x) for x in s]

    def schedule_set(self, sched):
        s = (ctypes.c_int * 3)(*[int(x) for x in sched])
        self._check(lib().gem_fk_schedule_set(self._h, s))

    def defer(self):
        """Bookkeeping deferral index per phase; see DEFERRALS."""
        s = (ctypes.c_int * 3)()
        self._check(lib().gem_fk_defer_get(self._h, s))
        return [int(x) for x in s]

    def defer_set(self, defer):
        s = (ctypes.c_int * 3)(*[int(x) for x in defer])
        self._check(lib().gem_fk_defer_set(self._h, s))

    def queue(self):
        """Queue granularity index per phase; see GRANULARITIES."""
        s = (ctypes.c_int * 3)()
        self._check(lib().gem_fk_queue_get(self._h, s))
        return [int(x) for x in s]

    def queue_set(self, gran):
        s = (ctypes.c_int * 3)(*[int(x) for x in gran])
        self._check(lib().gem_fk_queue_set(self._h, s))

    def autotune(self, params: FKParams, jre: int, jf_first: int = 0, jf_last: int = 0, repeats: int = 1):
        """Pick per phase the fastest schedule, then the fastest bookkeeping
        deferral, then the fastest queue granularity, on frequencies
        jf_first..jf_last (default: the top quarter of the band, which holds
        about 44% of the solves).  Returns {"schedule": [tor, sph, adj],
        "defer": [...], "queue": [...], "ms": (NSCHED + NDEFER + NGRAN, 3)
        phase times}."""
        if not jf_first:
            grid = frequency_grid(params, self.model.rearth)
            jf_last = grid.nf2
            jf_first = max(grid.nf1, grid.nf2 - (grid.nf2 - grid.nf1 + 1) // 4)
        pc = fk_params_c(params, jre)
        ms = np.zeros(3 * (NSCHED + NDEFER + NGRAN), np.float32)
        s = (ctypes.c_int * 3)()
        d = (ctypes.c_int * 3)()
        self._check(lib().gem_fk_autotune(self._h, ctypes.byref(pc), int(jf_first), int(jf_last), int(repeats),
                                          _ptr(ms), s, d))
        return {"schedule": [int(x) for x in s], "defer": [int(x) for x in d], "queue": self.queue(),
                "ms": ms.reshape(NSCHED + NDEFER + NGRAN, 3), "jf": [int(jf_first), int(jf_last)]}

    def ray_table(self, stype: str = "P", attmode: int = 3, eps: float = 1e-6, drtp: float = 10000.0,
                  rtmax: float = 0.0):
        """Travel-time table by ray tracing (computeTravelTimeTable): returns
        (rtp [ntp], slowness [ntp], table float32 [ntp, nnod, 2] of (Delta, T)).
        rtmax defaults to the radius of the top node."""
        if not rtmax:
            rtmax = float(self.nodes.r[-1])
        cap = int((rtmax - self.model.roc) / drtp) + 2
        n = ctypes.c_int()
        rtp = np.zeros(cap); slow = np.zeros(cap)
        table = np.zeros((cap, self.nodes.nnod, 2), np.float32)
        status = np.zeros(cap, np.int32)
        self._check(lib().gem_ray_table(self._h, {"P": 0, "S": 1}[stype], int(attmode), float(eps), float(drtp),
                                        float(rtmax), cap, ctypes.byref(n), _ptr(rtp), _ptr(slow), _ptr(table),
                                        _ptr(status)))
        k = n.value
        return rtp[:k], slow[:k], table[:k]

    def travel_times(self, rtp, slowness, table, rs, re, delta, tele=True):
        """Travel times (s) of the table (float32 as stored) for source radius rs and
        receivers at radii re and distances delta (rad) (getTravelTimes)."""
        rnod = np.ascontiguousarray(self.nodes.r, np.float32)
        rtp = np.ascontiguousarray(rtp, np.float32); sl = np.ascontiguousarray(slowness, np.float32)
        tb = np.ascontiguousarray(table, np.float32)
        re = np.ascontiguousarray(np.broadcast_to(re, np.shape(delta)), np.float64)
        de = np.ascontiguousarray(delta, np.float64)
        tt = np.zeros(len(de))
        self._check(lib().gem_travel_times(self._h, len(rnod), len(rtp), _ptr(rnod), _ptr(rtp), _ptr(sl), _ptr(tb),
                                           1 if tele else 0, float(rs), len(de), _ptr(re), _ptr(de), _ptr(tt)))
        return tt

    def order_target(self, k: int):
        """Attempt the step-size control aims at (fast backend; 3..7, 0 restores the reference's 6)."""
        self._check(lib().gem_order_target(self._h, int(k)))

    def tc_wait_limit(self, ns: int):
        """Time limit in ns of each pipeline wait of the tensor-core degree sums (0 restores 1 s);
        a wait that runs out makes the synthetics call fail with GeminiError."""
        self._check(lib().gem_tc_wait_limit(self._h, int(ns)))

    def steplog(self, capacity: int):
        """Record every step attempt of the following runs (capacity records; 0 = off)."""
        self._check(lib().gem_steplog(self._h, int(capacity)))

    def steplog_read(self, capacity: int) -> np.ndarray:
        out = np.zeros(capacity, STEP_DTYPE)
        n = ctypes.c_longlong()
        self._check(lib().gem_steplog_read(self._h, _ptr(out), capacity, ctypes.byref(n)))
        return out[: min(n.value, capacity)]

    def instrument(self, enable: bool = True):
        self._check(lib().gem_instrument(self._h, 1 if enable else 0))

    def instrument_read(self):
        prof = np.zeros(32, np.uint64)
        ns = np.zeros(2 * 148 * 64, np.uint64)
        nw = ctypes.c_int()
        self._check(lib().gem_instrument_read(self._h, _ptr(prof), _ptr(ns), ctypes.byref(nw)))
        return prof, ns[: 2 * nw.value].reshape(-1, 2)

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().gem_stats_get(self._h, ctypes.byref(s)))
        return s.asdict()
