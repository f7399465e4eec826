"""ctypes binding of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
module.  It checks the CUDA product path; nothing in gemini_unified_b200 may
import it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("steps_ok", "steps_rej", "attempts", "sysmats", "matvecs", "flops")]

    def asdict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def build() -> str:
    srcs = [os.path.join(HERE, f) for f in ("oracle_fk.cpp", "oracle_synth.cpp", "oracle_core.h")]
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        L = _lib
        vp = ctypes.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create_nodes.restype = vp
        L.oracle_destroy.argtypes = [vp]
        L.oracle_nnod.argtypes = [vp]
        L.oracle_nodes.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_node_index.argtypes = [vp, ctypes.c_double]
        L.oracle_spline.argtypes = [vp, ctypes.c_double, ctypes.c_int] + [ctypes.c_void_p] * 4
        L.oracle_start_radius.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oracle_start_radius.restype = ctypes.c_double
        L.oracle_bottom_iv.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_propagate.argtypes = ([vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_void_p] * 3)
        L.oracle_nwn.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_fk_frequency.argtypes = [vp, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_dsv_frequency.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_legendre.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        L.oracle_coupling.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_double] * 3 +
                                      [ctypes.c_void_p] * 3 + [ctypes.c_double, ctypes.c_int] + [ctypes.c_double] * 5 +
                                      [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_int] + [ctypes.c_void_p] * 3)
        L.oracle_fft.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_wavenumber_integrals.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p]
        L.oracle_synthetics_bessel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        L.oracle_freq_time.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_void_p]
        L.oracle_wavenumber_integrals_src.argtypes = [ctypes.c_int] + L.oracle_wavenumber_integrals.argtypes
        L.oracle_degree_sums_force.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_synthetics_src.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 4
                                            + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int] + [ctypes.c_void_p] * 3
                                            + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_void_p])
        L.oracle_synthetics_opts.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 4
                                             + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_int] + [ctypes.c_void_p] * 3
                                             + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_double] + [ctypes.c_void_p] * 3
                                             + [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_void_p])
        L.oracle_ray_table.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_degree_sums.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_synthetics.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_void_p]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One earth model + external node set, as the FK driver holds them."""

    def __init__(self, model, nodes):
        self._desc = model.desc()
        self.model = model
        r = np.ascontiguousarray(nodes.r, dtype=np.float64)
        s = np.ascontiguousarray(nodes.state, dtype=np.int32)
        l = np.ascontiguousarray(nodes.layer, dtype=np.int32)
        self.h = lib().oracle_create_nodes(ctypes.byref(self._desc), len(r), _p(r), _p(s), _p(l))
        if not self.h:
            raise RuntimeError("oracle_create_nodes failed")

    @classmethod
    def from_blocks(cls, model, nnodb, drb, shift, rearth):
        self = cls.__new__(cls)
        self._desc = model.desc()
        self.model = model
        nb = np.ascontiguousarray(nnodb, dtype=np.int32)
        dr = np.ascontiguousarray(drb, dtype=np.float64)
        self.h = lib().oracle_create(ctypes.byref(self._desc), len(nb), _p(nb), _p(dr),
                                     ctypes.c_double(shift), ctypes.c_double(rearth))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        return self

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def ray_table(self, stype, attmode, eps, drtp, rtmax, cap, nnod):
        """computeTravelTimeTable: (ntp, rtp, slowness, table float32 [ntp, nnod, 2], status)."""
        n = ctypes.c_int()
        rtp = np.zeros(cap); slow = np.zeros(cap)
        table = np.zeros((cap, nnod, 2), np.float32); st = np.zeros(cap, np.int32)
        rc = lib().oracle_ray_table(self.h, {"P": 0, "S": 1}[stype], attmode, eps, drtp, rtmax, cap, ctypes.byref(n),
                                    _p(rtp), _p(slow), _p(table), _p(st))
        k = n.value
        return rc, rtp[:k], slow[:k], table[:k], st[:k]

    def nodes(self):
        n = lib().oracle_nnod(self.h)
        r = np.zeros(n); s = np.zeros(n, np.int32); l = np.zeros(n, np.int32)
        lib().oracle_nodes(self.h, _p(r), _p(s), _p(l))
        return r, s, l

    def spline(self, f, attmode):
        nk = self.model.nk
        ro = np.zeros(nk); ro2 = np.zeros(nk); el = np.zeros(nk * 14); el2 = np.zeros(nk * 14)
        rc = lib().oracle_spline(self.h, ctypes.c_double(f), attmode, _p(ro), _p(ro2), _p(el), _p(el2))
        if rc:
            raise RuntimeError("spline failed")
        return ro, ro2, el.view(np.complex128).reshape(nk, 7), el2.view(np.complex128).reshape(nk, 7)

    def start_radius(self, f, attmode, wn, tor):
        return lib().oracle_start_radius(self.h, ctypes.c_double(f), attmode, ctypes.c_double(wn), int(tor))

    def bottom_iv(self, f, attmode, omim, dll1, r, kind):
        """Start vector of an upward integration at r (kind 0 toroidal, 1 minors), its
        initial step and the status of the continued fractions (initialValues.f90:202-416)."""
        y = np.zeros(4 if kind == 0 else 10)
        htry = ctypes.c_double()
        rc = lib().oracle_bottom_iv(self.h, f, attmode, omim, dll1, r, int(kind), _p(y), ctypes.byref(htry))
        return y.view(np.complex128), htry.value, rc

    def propagate(self, f, attmode, omim, dll1, sys, x1, x2, htry, eps, y0):
        """y(x2) of system sys (0 minors, 3 toroidal, 4 adjoint solid) from y(x1) = y0, as
        y1 * 10**lgnorm (propagateOde.f90:132-331); returns (y1, lgnorm, status)."""
        y0 = np.ascontiguousarray(y0, np.complex128)
        y1 = np.zeros_like(y0)
        lg = ctypes.c_double()
        rc = lib().oracle_propagate(self.h, f, attmode, omim, dll1, int(sys), x1, x2, htry, eps,
                                    _p(y0.view(np.float64)), _p(y1.view(np.float64)), ctypes.byref(lg))
        return y1, lg.value, rc

    def nwn(self, pc):
        cap = 1 << 16
        nwn = np.zeros(cap, np.int32)
        nf1 = ctypes.c_int(); nf2 = ctypes.c_int()
        rc = lib().oracle_nwn(self.h, ctypes.byref(pc), ctypes.byref(nf1), ctypes.byref(nf2), _p(nwn), cap)
        if rc:
            raise RuntimeError("oracle_nwn failed")
        return nf1.value, nf2.value, nwn[: nf2.value].copy()

    def fk_frequency(self, pc, jf, nwn, nsp, iwn_lo=1, iwn_hi=1 << 30):
        """FK spectra of one frequency: complex128 [nnod, nsp, nwn] plus per-iwn status and stats."""
        nnod = lib().oracle_nnod(self.h)
        gf = np.zeros(nwn * nsp * nnod * 2)
        status = np.zeros(nwn, np.int32)
        st = Stats()
        rc = lib().oracle_fk_frequency(self.h, ctypes.byref(pc), jf, nwn, _p(gf), _p(status), ctypes.byref(st),
                                       iwn_lo, iwn_hi)
        if rc < 0:
            raise RuntimeError("oracle_fk_frequency: unsupported configuration")
        if rc != nsp:
            raise RuntimeError(f"nsp mismatch {rc} != {nsp}")
        g = gf.view(np.complex128).reshape(nnod, nsp, nwn)
        return g, status, st.asdict()

    def dsv_frequency(self, pc, jsnod, jf, nwn, iwn_lo=1, iwn_hi=1 << 30):
        """DSV spectra with radial derivatives of one frequency for the source
        nodes jsnod (type pc.istyp) and a force at pc.jre, as the ASKI FK driver
        computes them: a list of complex128 [nnod, nsp_js, nwn], one per source
        (the force last), plus per-iwn status and stats."""
        nnod = lib().oracle_nnod(self.h)
        js = np.ascontiguousarray(jsnod, np.int32)
        ns = len(js)
        gf = np.zeros((ns + 1) * nwn * 20 * nnod * 2)
        nsp = np.zeros(ns + 1, np.int32)
        status = np.zeros(nwn, np.int32)
        st = Stats()
        rc = lib().oracle_dsv_frequency(self.h, ctypes.byref(pc), _p(js), ns, jf, nwn, _p(gf), _p(nsp), _p(status),
                                        ctypes.byref(st), iwn_lo, iwn_hi)
        if rc < 0:
            raise RuntimeError("oracle_dsv_frequency: unsupported configuration")
        blocks = gf.view(np.complex128).reshape(ns + 1, -1)
        out = [blocks[j, :nwn * int(nsp[j]) * nnod].reshape(nnod, int(nsp[j]), nwn) for j in range(ns + 1)]
        return out, status, st.asdict()


def legendre(lmax, theta):
    out = np.zeros(5 * 3 * (lmax + 1))
    lib().oracle_legendre(lmax, ctypes.c_double(theta), _p(out))
    return out.reshape(5, 3, lmax + 1)


def fft(x, y, n, is_):
    x = np.ascontiguousarray(x, np.float64).copy(); y = np.ascontiguousarray(y, np.float64).copy()
    lib().oracle_fft(n, is_, _p(x), _p(y))
    return x, y


def freq_time(nf1, nf2, df, sigma, sp, nsamp, dt):
    """transformFrequencyTime of each row of sp (complex [ntr, ldsp >= nf2]).
    Returns (float32 [ntr, nsamp], level 0 ok / 1 decimation warning)."""
    sp = np.ascontiguousarray(sp, np.complex128)
    ntr, ld = sp.shape
    ts = np.zeros((ntr, nsamp), np.float32)
    rc = lib().oracle_freq_time(nf1, nf2, df, sigma, ntr, _p(sp), ld, nsamp, dt, _p(ts))
    if rc >= 2:
        raise RuntimeError("oracle_freq_time: invalid sizes")
    return ts, rc


def wavenumber_integrals(nf1, nf2, nwn, nwnmax, gr, gi, dwn, rearth, x):
    """The 14 moment wavenumber integrals (regional mode): complex [nsta, nf2, 14]; x in m."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    x = np.ascontiguousarray(x, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    hd = np.zeros(len(x) * nf2 * 14 * 2)
    rc = lib().oracle_wavenumber_integrals(nf1, nf2, _p(nwn), nwnmax, nkf, nsp, _p(gr), _p(gi), dwn, rearth, len(x),
                                           _p(x), _p(hd))
    if rc:
        raise RuntimeError("oracle_wavenumber_integrals failed")
    return hd.view(np.complex128).reshape(len(x), nf2, 14)


def synthetics_bessel(nf1, nf2, nwn, nwnmax, df, sigma, dwn, rearth, gr, gi, theta, phi, propdir, mt, filspecs,
                      velocity, tred, nsamp, dt):
    """Synthetics of the regional mode; theta = distance / rearth.  float32 [nsta, nmt, 3, nsamp]."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64); ph = np.ascontiguousarray(phi, np.float64)
    pd = np.ascontiguousarray(propdir, np.float64); mt = np.ascontiguousarray(mt, np.float64).reshape(-1, 6)
    fs = np.ascontiguousarray(filspecs, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    out = np.zeros((len(th), len(mt), 3, nsamp), np.float32)
    rc = lib().oracle_synthetics_bessel(nf1, nf2, _p(nwn), nwnmax, df, sigma, dwn, rearth, nkf, nsp, _p(gr), _p(gi),
                                        len(th), _p(th), _p(ph), _p(pd), len(mt), _p(mt), _p(fs), int(velocity),
                                        tred, nsamp, dt, _p(out))
    if rc:
        raise RuntimeError("oracle_synthetics_bessel failed (%d)" % rc)
    return out


def degree_sums(nf1, nf2, nwn, nwnmax, gr, gi, theta):
    """gr/gi: float32 [nsp, nkfmax] (row per spectrum).  Returns complex [nsta, nf2, 14]."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    hd = np.zeros(len(th) * nf2 * 14 * 2)
    rc = lib().oracle_degree_sums(nf1, nf2, _p(nwn), nwnmax, nkf, nsp, _p(gr), _p(gi), len(th), _p(th), _p(hd))
    if rc:
        raise RuntimeError("oracle_degree_sums failed")
    return hd.view(np.complex128).reshape(len(th), nf2, 14)


def synthetics(nf1, nf2, nwn, nwnmax, df, sigma, gr, gi, theta, phi, propdir, mt, filspecs,
               velocity, tred, nsamp, dt):
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64); ph = np.ascontiguousarray(phi, np.float64)
    pd = np.ascontiguousarray(propdir, np.float64)
    mt = np.ascontiguousarray(mt, np.float64).reshape(-1, 6)
    fs = np.ascontiguousarray(filspecs, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    tr = np.zeros(len(th) * len(mt) * 3 * nsamp, np.float32)
    rc = lib().oracle_synthetics(nf1, nf2, _p(nwn), nwnmax, df, sigma, nkf, nsp, _p(gr), _p(gi), len(th),
                                 _p(th), _p(ph), _p(pd), len(mt), _p(mt), _p(fs), int(velocity), tred,
                                 nsamp, dt, _p(tr))
    if rc:
        raise RuntimeError("oracle_synthetics failed")
    return tr.reshape(len(th), len(mt), 3, nsamp)


def force_degree_sums(nf1, nf2, nwn, nwnmax, gr, gi, theta):
    """The 7 force degree sums: gr/gi float32 [nsp >= 5, nkfmax].  complex [nsta, nf2, 7]."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    hd = np.zeros(len(th) * nf2 * 7 * 2)
    rc = lib().oracle_degree_sums_force(nf1, nf2, _p(nwn), nwnmax, nkf, nsp, _p(gr), _p(gi), len(th), _p(th), _p(hd))
    if rc:
        raise RuntimeError("oracle_degree_sums_force failed")
    return hd.view(np.complex128).reshape(len(th), nf2, 7)


def force_wavenumber_integrals(nf1, nf2, nwn, nwnmax, gr, gi, dwn, rearth, x):
    """The 7 force wavenumber integrals (regional mode): complex [nsta, nf2, 7]; x in m."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    x = np.ascontiguousarray(x, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    hd = np.zeros(len(x) * nf2 * 7 * 2)
    rc = lib().oracle_wavenumber_integrals_src(0, nf1, nf2, _p(nwn), nwnmax, nkf, nsp, _p(gr), _p(gi), dwn, rearth,
                                               len(x), _p(x), _p(hd))
    if rc:
        raise RuntimeError("oracle_wavenumber_integrals_src failed")
    return hd.view(np.complex128).reshape(len(x), nf2, 7)


def synthetics_src(source_type, global_, nf1, nf2, nwn, nwnmax, df, sigma, dwn, rearth, gr, gi, theta, phi, propdir,
                   src, filspecs, velocity, tred, nsamp, dt):
    """Synthetics of either source type ("MOMENT": src (nsrc, 6); "FORCE": src (nsrc, 3)
    as Fr, Ft, Ff) and either mode (global_ 1 degree sums, 0 wavenumber integrals at
    distance theta * rearth).  float32 [nsta, nsrc, 3, nsamp]."""
    istyp = {"FORCE": 0, "MOMENT": 1}[source_type]
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64); ph = np.ascontiguousarray(phi, np.float64)
    pd = np.ascontiguousarray(propdir, np.float64)
    src = np.ascontiguousarray(src, np.float64).reshape(-1, 6 if istyp == 1 else 3)
    fs = np.ascontiguousarray(filspecs, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    out = np.zeros((len(th), len(src), 3, nsamp), np.float32)
    rc = lib().oracle_synthetics_src(istyp, int(global_), nf1, nf2, _p(nwn), nwnmax, df, sigma, dwn, rearth, nkf, nsp,
                                     _p(gr), _p(gi), len(th), _p(th), _p(ph), _p(pd), len(src), _p(src), _p(fs),
                                     int(velocity), tred, nsamp, dt, _p(out))
    if rc:
        raise RuntimeError("oracle_synthetics_src failed (%d)" % rc)
    return out


def synthetics_opts(source_type, global_, nf1, nf2, nwn, nwnmax, df, sigma, dwn, rearth, gr, gi, theta, phi, propdir,
                    src, filspecs, velocity, tred, nsamp, dt, tred_sta=None, nstrue=None, stafilter=None, stf=None,
                    tanf_stf=0.0):
    """synthetics_src with the station loop's per-station options: tred_sta [nsta] reduction
    times, nstrue [nsta] samples kept (later samples 0), stafilter complex [nsta, 3, nf2],
    stf float32 [nstf] source wavelet starting at tanf_stf (computeSyntheticSeismograms.f90:344-397)."""
    istyp = {"FORCE": 0, "MOMENT": 1}[source_type]
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkf = gr.shape
    th = np.ascontiguousarray(theta, np.float64); ph = np.ascontiguousarray(phi, np.float64)
    pd = np.ascontiguousarray(propdir, np.float64)
    src = np.ascontiguousarray(src, np.float64).reshape(-1, 6 if istyp == 1 else 3)
    fs = np.ascontiguousarray(filspecs, np.float64)
    nwn = np.ascontiguousarray(nwn, np.int32)
    ts = None if tred_sta is None else np.ascontiguousarray(tred_sta, np.float64)
    nt = None if nstrue is None else np.ascontiguousarray(nstrue, np.int32)
    sf = None if stafilter is None else np.ascontiguousarray(stafilter, np.complex128)
    w = None if stf is None else np.ascontiguousarray(stf, np.float32)
    out = np.zeros((len(th), len(src), 3, nsamp), np.float32)
    rc = lib().oracle_synthetics_opts(istyp, int(global_), nf1, nf2, _p(nwn), nwnmax, df, sigma, dwn, rearth, nkf, nsp,
                                      _p(gr), _p(gi), len(th), _p(th), _p(ph), _p(pd), len(src), _p(src), _p(fs),
                                      int(velocity), tred, _p(ts), _p(nt), _p(sf), 0 if w is None else len(w),
                                      float(tanf_stf), _p(w), nsamp, dt, _p(out))
    if rc:
        raise RuntimeError("oracle_synthetics_opts failed (%d)" % rc)
    return out


def coupling(nf1, nf2, nwn, nwnmax, gr, gi, df, sigma, re, zelcon, mt, filspecs, tred, nsamp, dt, thetas, phis,
             thetac, phic, delta, xi, nrm, spectra=False, debug=False, istyp=1):
    """SPECFEM-coupling synthetics at boundary points
    (computeSyntheticsForSpecfemCoupling.f90:677-793).  gr/gi: float32 DSV
    spectra with derivatives of the points' node, shape (nsp, nkfmax), nsp >= 20
    for a moment tensor mt[6] (istyp 1), >= 10 for a force mt[3] (istyp 0);
    zelcon: complex [nf2, 7] elastic constants of the node per frequency.
    Returns (spectra complex [npts, 6, nf2] or None, traces float32 [npts, 6,
    nsamp] or None, debug complex [npts, nf2, 4, 3] or None)."""
    gr = np.ascontiguousarray(gr, np.float32); gi = np.ascontiguousarray(gi, np.float32)
    nsp, nkfmax = gr.shape
    nwn = np.ascontiguousarray(nwn, np.int32)
    zel = np.ascontiguousarray(zelcon, np.complex128).reshape(-1)
    mt = np.ascontiguousarray(mt, np.float64); fs = np.ascontiguousarray(filspecs, np.float64)
    delta = np.ascontiguousarray(delta, np.float64); xi = np.ascontiguousarray(xi, np.float64)
    nrm = np.ascontiguousarray(nrm, np.float64).reshape(-1)
    npts = len(delta)
    spec = np.zeros(npts * 6 * nf2, np.complex128) if spectra else None
    tr = None if spectra else np.zeros(npts * 6 * nsamp, np.float32)
    dbg = np.zeros(npts * nf2 * 12, np.complex128) if debug else None
    rc = lib().oracle_coupling(istyp, nf1, nf2, _p(nwn), nwnmax, nkfmax, nsp, _p(gr), _p(gi), df, sigma, re, _p(zel),
                               _p(mt), _p(fs), tred, nsamp, dt, thetas, phis, thetac, phic, npts, _p(delta), _p(xi),
                               _p(nrm), 1 if spectra else 0, _p(spec), _p(tr), _p(dbg))
    if rc:
        raise RuntimeError("oracle_coupling: level %d" % rc)
    return (None if spec is None else spec.reshape(npts, 6, nf2),
            None if tr is None else tr.reshape(npts, 6, nsamp),
            None if dbg is None else dbg.reshape(npts, nf2, 4, 3))

