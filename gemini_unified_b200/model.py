"""Earth model, external radial nodes and frequency/wavenumber grid.

Host-side mirror of the reference's model and node set-up, which runs once per
job and feeds the GPU library through flat arrays:

* :func:`load_node_model` reads a GEMINI JSON node model exactly as
  ``createNodeEarthmodel`` does (f90/nodeEarthmodel.f90:98-257), including the
  number parser of the bundled fson library (fson/fson.f90:327-414), which
  builds a real from ``integral + digits / 10**ndigits`` rather than by
  correctly rounded conversion.
* :class:`ExternalRadialNodes` mirrors createExternalRadialNodes and
  splitNodesAtDiscosExternalRadialNodes (f90/externalRadialNodes.f90:82-156,
  337-418): blocks of equidistant nodes below the (shifted) surface, plus one
  node just below and one just above every model interface above the deepest
  node.
* :func:`frequency_grid` mirrors the frequency / wavenumber set-up of
  computeGreenFKSpectraForSynthetics (f90/computeGreenFKSpectraForSynthetics.f90:
  186-236): df = 1/TLEN, sigma = 5 df, nf1..nf2 and nwn(jf).
"""
from __future__ import annotations

import ctypes
import dataclasses
import json
import math
from typing import List, Optional, Sequence

import numpy as np

# mathConstants.f90:34 -- the "double" pi literal has no d0 exponent, so it is
# pi rounded to single precision, then widened.
PI_F = float(np.float32(3.141592653589793))
TWO_PI_F = 2.0 * PI_F
EPS_D = float(np.finfo(np.float64).eps)

ATTENUATION_MODES = {
    "ELASTIC": 0,
    "ATTENUATION_ONLY": 1,
    "DISPERSION_ONLY": 2,
    "ATTENUATION_AND_DISPERSION": 3,
}
SOURCE_TYPES = {"FORCE": 0, "MOMENT": 1}


class GeminiError(RuntimeError):
    """Error with the reference's level-2 semantics (fatal for the caller)."""


# --------------------------------------------------------------------------
#  fson number semantics
# --------------------------------------------------------------------------
def _pow10(k: int) -> float:
    """10**k as gfortran's integer power (repeated squaring; exact to 10**22)."""
    n = abs(k)
    x, y = 10.0, 1.0
    while n:
        if n & 1:
            y *= x
        x *= x
        n >>= 1
    return 1.0 / y if k < 0 else y


def fson_number(text: str):
    """Parse a JSON number the way fson's parse_number does (fson.f90:327-414).

    Integers stay integers.  Reals are ``integral + frac_digits/10**ndigits``
    (two roundings), times ``10**exp`` when an exponent is present, negated
    last.
    """
    s = text.strip()
    neg = s.startswith("-")
    if neg:
        s = s[1:]
    mant, exp_part = s, None
    for ch in "eE":
        if ch in s:
            mant, exp_part = s.split(ch, 1)
            break
    if "." in mant:
        ipart, fpart = mant.split(".", 1)
    else:
        ipart, fpart = mant, None
    integral = int(ipart) if ipart else 0
    if fpart is None and exp_part is None:
        return -integral if neg else integral
    frac = 0.0
    if fpart is not None and fpart != "":
        frac = float(int(fpart)) / _pow10(len(fpart))
    frac = frac + float(integral)
    if exp_part is not None:
        frac = frac * _pow10(int(exp_part))
    return -frac if neg else frac


def _fson_loads(text: str):
    return json.loads(text, parse_float=fson_number, parse_int=fson_number)


# --------------------------------------------------------------------------
#  Node earth model
# --------------------------------------------------------------------------
class ModelDesc(ctypes.Structure):
    """C layout of ``gem_model_desc`` (include/gemini_fk.h)."""

    _fields_ = [
        ("fref", ctypes.c_double), ("rearth", ctypes.c_double),
        ("ric", ctypes.c_double), ("roc", ctypes.c_double),
        ("aniflag", ctypes.c_int), ("fsflag", ctypes.c_int), ("equidis", ctypes.c_int),
        ("nlay", ctypes.c_int), ("nk", ctypes.c_int), ("nic", ctypes.c_int), ("noc", ctypes.c_int),
        ("iflso", ctypes.POINTER(ctypes.c_int)), ("iktop", ctypes.POINTER(ctypes.c_int)),
        ("rb", ctypes.POINTER(ctypes.c_double)),
        ("depth", ctypes.POINTER(ctypes.c_double)), ("ro", ctypes.POINTER(ctypes.c_double)),
        ("vpv", ctypes.POINTER(ctypes.c_double)), ("vph", ctypes.POINTER(ctypes.c_double)),
        ("vsv", ctypes.POINTER(ctypes.c_double)), ("vsh", ctypes.POINTER(ctypes.c_double)),
        ("eta", ctypes.POINTER(ctypes.c_double)), ("qk", ctypes.POINTER(ctypes.c_double)),
        ("qm", ctypes.POINTER(ctypes.c_double)),
    ]


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


@dataclasses.dataclass
class NodeEarthModel:
    """Node earth model as read by createNodeEarthmodel (nodeEarthmodel.f90:98-257).

    Arrays are 0-based copies of the reference's 1-based arrays.
    """

    fref: float
    rearth: float
    ric: float
    roc: float
    aniflag: int
    fsflag: int
    equidis: int
    nlay: int
    nk: int
    nic: int
    noc: int
    iflso: np.ndarray
    iktop: np.ndarray
    rb: np.ndarray
    depth: np.ndarray
    ro: np.ndarray
    vpv: np.ndarray
    vph: np.ndarray
    vsv: np.ndarray
    vsh: np.ndarray
    eta: np.ndarray
    qk: np.ndarray
    qm: np.ndarray
    name: str = ""

    # ---- derived quantities exactly as the reference forms them
    @property
    def rk(self) -> np.ndarray:
        return self.rearth - self.depth                    # nodeEarthmodel.f90:175

    @property
    def ikbot(self) -> np.ndarray:
        b = np.zeros(self.nlay, dtype=np.int32)            # :165-166
        b[1:] = self.iktop[:-1] + 1
        return b

    @property
    def rhs(self) -> float:
        return float(self.rb[0])

    def layer_index(self, r: float):
        """getLayerIndexNodeEarthmodel (nodeEarthmodel.f90:599-607): (nl, top), 1-based nl."""
        nl = locate(r, self.rb) + 1
        top = 1 if abs(r / self.rb[min(nl, self.nlay) - 1] - 1.0) < EPS_D else 0
        return nl, top

    def desc(self) -> ModelDesc:
        """Flat C description; the returned object keeps its arrays alive."""
        self._keep = [np.ascontiguousarray(a) for a in (
            self.iflso.astype(np.int32), self.iktop.astype(np.int32), self.rb, self.depth, self.ro,
            self.vpv, self.vph, self.vsv, self.vsh, self.eta, self.qk, self.qm)]
        k = self._keep
        return ModelDesc(self.fref, self.rearth, self.ric, self.roc, self.aniflag, self.fsflag,
                         self.equidis, self.nlay, self.nk, self.nic, self.noc,
                         _iptr(k[0]), _iptr(k[1]), _dptr(k[2]), _dptr(k[3]), _dptr(k[4]),
                         _dptr(k[5]), _dptr(k[6]), _dptr(k[7]), _dptr(k[8]), _dptr(k[9]),
                         _dptr(k[10]), _dptr(k[11]))

    def isotropic(self) -> "NodeEarthModel":
        """Isotropic derivative of a TI model: PV -> P, SV -> S, eta = 1."""
        return dataclasses.replace(self, aniflag=0, vph=self.vpv.copy(), vsh=self.vsv.copy(),
                                   eta=np.ones_like(self.eta), name=self.name + "-iso")


def _as_int_bool(v) -> int:
    if isinstance(v, bool):
        return 1 if v else 0
    return int(v)


def load_node_model(path: str) -> NodeEarthModel:
    """Read a GEMINI JSON node model (nodeEarthmodel.f90:98-257)."""
    with open(path) as fh:
        d = _fson_loads(fh.read())
    return node_model_from_dict(d, name=path)


def _layer_tops(d: dict):
    """Layer-top radii (key radius_upper_layer_boundary_m, nodeEarthmodel.f90:152).

    Older model files (earthmodels/ak135q.json, the fixture of the reference's
    model-reader test) name the key ``..._km`` and use km throughout; the values
    are taken as they are, so that test's radii (in km) come out unchanged.
    The reference itself stops with "Unable to resolve path" on such files.
    """
    if "radius_upper_layer_boundary_m" in d:
        return d["radius_upper_layer_boundary_m"]
    if "radius_upper_layer_boundary_km" in d:
        return d["radius_upper_layer_boundary_km"]
    raise GeminiError("Unable to resolve path: radius_upper_layer_boundary_m")


def node_model_from_dict(d: dict, name: str = "") -> NodeEarthModel:
    np_ = d["node_properties"]
    nlay = int(d["num_layers"])
    nk = int(d["num_nodes"])
    aniflag = _as_int_bool(d["anisotropic"])
    f64 = lambda v: np.asarray([float(x) for x in v], dtype=np.float64)
    if aniflag == 0:
        vpv = f64(np_["P-velocity"]); vph = vpv.copy()
        vsv = f64(np_["S-velocity"]); vsh = vsv.copy()
        eta = np.ones(nk)
    else:
        vpv = f64(np_["PV-velocity"]); vph = f64(np_["PH-velocity"])
        vsv = f64(np_["SV-velocity"]); vsh = f64(np_["SH-velocity"])
        eta = f64(np_["eta"])
    iflso = np.asarray([int(x) for x in d["isfluid"]], dtype=np.int32)
    fsflag = _as_int_bool(d["full_space"])
    if iflso[nlay - 1] == 1 and fsflag == 1:
        raise GeminiError("Full space and ocean is not allowed!!")
    m = NodeEarthModel(
        fref=float(d["reference_frequency_hz"]), rearth=float(d["earth_radius"]),
        ric=float(d["radius_inner_core"]), roc=float(d["radius_outer_core"]),
        aniflag=aniflag, fsflag=fsflag, equidis=_as_int_bool(d["equidistant_nodes"]),
        nlay=nlay, nk=nk, nic=int(d["layer_inner_core"]), noc=int(d["layer_outer_core"]),
        iflso=iflso, iktop=np.asarray([int(x) for x in d["index_upper_boundary"]], dtype=np.int32),
        rb=f64(_layer_tops(d)), depth=f64(np_["depth"]),
        ro=f64(np_["density"]), vpv=vpv, vph=vph, vsv=vsv, vsh=vsh, eta=eta,
        qk=f64(np_["Qkappa"]), qm=f64(np_["Qmu"]), name=name)
    if len(m.rb) != nlay or len(m.iktop) != nlay or len(m.depth) != nk:
        raise GeminiError("Inconsistent dimension of model parameters")
    return m


def _natural_spline_y2(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Second derivatives of the natural cubic spline through (x, y) from the
    tridiagonal system of cubicSpline.f90:74-109 (first and last rows set the
    end second derivatives to zero), solved by elimination."""
    n = len(x)
    if n <= 2:
        return np.zeros(n)
    lo, di, up, rhs = np.zeros(n), np.ones(n), np.zeros(n), np.zeros(n)
    for j in range(1, n - 1):
        lo[j] = (x[j] - x[j - 1]) / 6.0
        di[j] = (x[j + 1] - x[j - 1]) / 3.0
        up[j] = (x[j + 1] - x[j]) / 6.0
        rhs[j] = (y[j + 1] - y[j]) / (x[j + 1] - x[j]) - (y[j] - y[j - 1]) / (x[j] - x[j - 1])
    for j in range(1, n):              # forward elimination (rows 0 and n-1 are y2 = 0)
        w = lo[j] / di[j - 1]
        di[j] -= w * up[j - 1]
        rhs[j] -= w * rhs[j - 1]
    y2 = np.zeros(n)
    y2[n - 1] = rhs[n - 1] / di[n - 1]
    for j in range(n - 2, -1, -1):
        y2[j] = (rhs[j] - up[j] * y2[j + 1]) / di[j]
    return y2


def node_elastic_constants(m: NodeEarthModel, nodes: "ExternalRadialNodes"):
    """Density, inverse Q (kappa, mu) and the seven elastic constants A, C, F,
    L, N, kappa, mu at the external nodes, from the model's splines at the
    reference frequency in ELASTIC mode -- what elasticConstantsExternalRadialNodes
    (externalRadialNodes.f90:423-435) stores with the nodes.  ELASTIC mode
    (nodeEarthmodel.f90:302-306) makes the constants real; the layer-1
    halfspace is constant, the other layers are natural cubic splines over
    their knots (splineEarthmodelCoefficients.f90:46-94,118-162).

    Returns ro [nnod], qinv [nnod, 2], elcon complex [nnod, 7]."""
    nk = m.nk
    vph = m.vph if m.aniflag else m.vpv
    vsh = m.vsh if m.aniflag else m.vsv
    eta = m.eta if m.aniflag else np.ones(nk)
    qinv = np.stack([1.0 / m.qk, np.maximum(1.0 / m.qm, 0.0)], axis=1)     # nodeEarthmodel.f90:206-214
    el = np.zeros((nk, 7))
    for j in range(nk):   # complexElasticVTIConstants (complexElasticConstants.f90:48-106) without attenuation
        ro, alfv, alfh, betv, beth, et = m.ro[j], m.vpv[j], vph[j], m.vsv[j], vsh[j], eta[j]
        if betv > float(np.float32(1e-6)):
            epa, epc, epn, epl = ro * alfh * alfh, ro * alfv * alfv, ro * beth * beth, ro * betv * betv
            epf = et * (epa - 2.0 * epl)
            kappa = (epc + 4.0 * epa - 4.0 * epn + 4.0 * epf) / 9.0
            mue = (epc + epa + 6.0 * epl + 5.0 * epn - 2.0 * epf) / 15.0
            el[j] = [epa, epc, epf, epl, epn, kappa, mue]
        else:
            kappa = ro * alfv * alfv
            el[j] = [kappa, kappa, kappa, 0.0, 0.0, kappa, 0.0]
    rk = m.rk
    iktop = m.iktop.astype(int)           # 1-based knot index of each layer's top
    ikbot = m.ikbot.astype(int)
    fields = np.concatenate([m.ro[:, None], qinv, el], axis=1)   # 10 splined quantities per knot
    y2 = np.zeros_like(fields)
    for nl in range(2, m.nlay + 1):
        j1, j2 = ikbot[nl - 1] - 1, iktop[nl - 1]       # 0-based slice of the layer's knots
        for q in range(fields.shape[1]):
            y2[j1:j2, q] = _natural_spline_y2(rk[j1:j2], fields[j1:j2, q])
    out = np.zeros((nodes.nnod, fields.shape[1]))
    for i in range(nodes.nnod):
        r, nl = float(nodes.r[i]), int(nodes.layer[i])
        if nl == 1:
            out[i] = fields[iktop[0] - 1]
            continue
        j1, j2 = iktop[nl - 2] + 1, iktop[nl - 1]      # 1-based knot range of the layer
        if j2 - j1 == 1:
            j = j1
        else:
            j = j1 - 1
            jr = j2 + 1
            while jr - j > 1:
                mid = (j + jr) // 2
                if r > rk[mid - 1]:
                    j = mid
                else:
                    jr = mid
            j = max(j, j1)
            j = min(j, j2 - 1)
        x1, x2 = rk[j - 1], rk[j]
        h = x2 - x1
        a = (x2 - r) / h
        b = 1.0 - a
        v = a * fields[j - 1] + b * fields[j]
        if j2 - j1 > 1:
            v = v + h * h * a * (a * a - 1.0) / 6.0 * y2[j - 1] + h * h * b * (b * b - 1.0) / 6.0 * y2[j]
        out[i] = v
    return out[:, 0], out[:, 1:3], out[:, 3:].astype(np.complex128)


def property_at_node(m: NodeEarthModel, prop: str, i: int) -> float:
    """getPropertyNodeEarthmodel (nodeEarthmodel.f90:570-590): single-precision result, 1-based i."""
    src = {"node_radius": m.rk, "vp": m.vpv, "vs": m.vsv, "rho": m.ro}.get(prop)
    if src is None:
        return float(np.float32(999999.0))
    return float(np.float32(src[i - 1]))


# --------------------------------------------------------------------------
#  locate (locatePoint.f90:72-101)
# --------------------------------------------------------------------------
def locate(xx: float, x: Sequence[float]) -> int:
    """Index j (0..n) with x(j) < xx <= x(j+1) for 1-based ascending x.

    A one-element array takes the "descending" branch, exactly as the
    reference does.
    """
    n = len(x)
    lidx, ridx = 0, n + 1
    asc = x[n - 1] > x[0]
    while ridx - lidx > 1:
        midx = (lidx + ridx) // 2
        if asc:
            if xx > x[midx - 1]:
                lidx = midx
            else:
                ridx = midx
        else:
            if xx > x[midx - 1]:
                ridx = midx
            else:
                lidx = midx
    return lidx


# --------------------------------------------------------------------------
#  External radial nodes
# --------------------------------------------------------------------------
@dataclasses.dataclass
class ExternalRadialNodes:
    rearth: float
    r: np.ndarray        # radii (ascending)
    state: np.ndarray    # 1 fluid, 0 solid
    layer: np.ndarray    # 1-based layer index

    @property
    def nnod(self) -> int:
        return len(self.r)

    @classmethod
    def from_blocks(cls, model: NodeEarthModel, nnod_blocks: Sequence[int],
                    dr_blocks: Sequence[float], shift: float, rearth: float) -> "ExternalRadialNodes":
        """createExternalRadialNodes (externalRadialNodes.f90:82-156)."""
        nnod = int(sum(nnod_blocks)) + 1
        prn = np.zeros(nnod)
        prn[nnod - 1] = rearth - shift
        n = nnod
        for nb, dr in zip(nnod_blocks, dr_blocks):
            for i in range(1, nb + 1):
                prn[n - i - 1] = prn[n - 1] - i * float(dr)
            n -= nb
        if np.any(prn < 0.0):
            raise GeminiError("Negative radii, check your input")
        return cls.split(model, prn, rearth)

    @classmethod
    def split(cls, model: NodeEarthModel, prn: np.ndarray, rearth: float) -> "ExternalRadialNodes":
        """splitNodesAtDiscosExternalRadialNodes (externalRadialNodes.f90:337-418)."""
        rb = model.rb
        L = model.nlay
        nnod = len(prn)
        drmin = rb[L - 1] * 1.e-4
        r, st, ly = [], [], []
        ne = 0
        for ib in range(1, L + 1):
            n = locate(rb[ib - 1], prn)
            if n == 0:
                continue
            iflso = int(model.iflso[ib - 1])
            for k in range(ne, n):
                r.append(prn[k]); ly.append(ib); st.append(iflso)
            if n >= nnod:
                break
            up = abs(prn[n] - rb[ib - 1]) < drmin        # prn(n+1)
            lo = abs(prn[n - 1] - rb[ib - 1]) < drmin    # prn(n)
            if up and lo:
                raise GeminiError("External nodes too close to each other, use bigger spacing")
            if up:
                r.append(rb[ib - 1] - drmin * 0.5); ly.append(ib); st.append(iflso)
                if n + 1 < nnod:
                    r.append(rb[ib - 1] + drmin * 0.5); ly.append(ib + 1); st.append(int(model.iflso[ib]))
                    ne = n + 1
                else:
                    ne = n
            elif lo:
                r[-1] = rb[ib - 1] - drmin * 0.5; ly[-1] = ib; st[-1] = iflso
                r.append(rb[ib - 1] + drmin * 0.5); ly.append(ib + 1); st.append(int(model.iflso[ib]))
                ne = n
            else:
                ne = n
                r.append(rb[ib - 1] - drmin * 0.5); ly.append(ib); st.append(iflso)
                r.append(rb[ib - 1] + drmin * 0.5); ly.append(ib + 1); st.append(int(model.iflso[ib]))
        return cls(rearth, np.asarray(r, dtype=np.float64), np.asarray(st, dtype=np.int32),
                   np.asarray(ly, dtype=np.int32))

    def node_index(self, rs: float) -> int:
        """getNodeIdxFromRadiusExternalRadialNodes (externalRadialNodes.f90:547-559), 1-based."""
        jr = locate(rs, self.r)
        if jr == 0:
            jr = 1
        if jr < self.nnod:
            if abs(rs - self.r[jr - 1]) > abs(rs - self.r[jr]):
                jr += 1
        return jr


# --------------------------------------------------------------------------
#  FK parameters and frequency grid
# --------------------------------------------------------------------------
@dataclasses.dataclass
class FKParams:
    """Parfile keys of computeGreenFKSpectraForSynthetics used on the hot path."""

    tlen: float
    fmax: float
    p1lim: float
    p2lim: float
    frac: float = 0.0
    xlen: float = 1.0e6
    eps: float = 1.0e-5
    global_: int = 1
    attmode: str = "ATTENUATION_AND_DISPERSION"
    source_type: str = "MOMENT"
    stressflag: bool = False
    fmin: float = 0.0


class FKParamsC(ctypes.Structure):
    """C layout of ``gem_fk_params`` (include/gemini_fk.h)."""

    _fields_ = [
        ("tlen", ctypes.c_double), ("fmax", ctypes.c_double), ("fmin", ctypes.c_double),
        ("p1lim", ctypes.c_double), ("p2lim", ctypes.c_double), ("frac", ctypes.c_double),
        ("xlen", ctypes.c_double), ("eps", ctypes.c_double),
        ("global_", ctypes.c_int), ("attmode", ctypes.c_int), ("istyp", ctypes.c_int),
        ("stressflag", ctypes.c_int), ("jre", ctypes.c_int),
    ]


def fk_params_c(p: FKParams, jre: int) -> FKParamsC:
    if p.attmode not in ATTENUATION_MODES:
        raise GeminiError("Invalid attenuation mode")
    if p.source_type not in SOURCE_TYPES:
        raise GeminiError("Invalid source type")
    return FKParamsC(p.tlen, p.fmax, p.fmin, p.p1lim, p.p2lim, p.frac, p.xlen, p.eps,
                     p.global_, ATTENUATION_MODES[p.attmode], SOURCE_TYPES[p.source_type],
                     1 if p.stressflag else 0, jre)


@dataclasses.dataclass
class FrequencyGrid:
    df: float
    sigma: float
    nf1: int
    nf2: int
    nwn: np.ndarray          # [nf2], nwn[jf-1]; zero below nf1
    nwnmax: int
    dwn: float

    @property
    def nkfmax(self) -> int:
        return int(self.nwn.sum())

    def offsets(self) -> np.ndarray:
        """Offset of frequency jf's slab in the FK file: sum(nwn(1:jf-1))."""
        return np.concatenate([[0], np.cumsum(self.nwn)])[:-1]


def _nint(x: float) -> int:
    """Fortran NINT: round half away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def frequency_grid(p: FKParams, rearth: float) -> FrequencyGrid:
    """computeGreenFKSpectraForSynthetics.f90:186-236."""
    df = 1.0 / p.tlen
    nf2 = _nint(p.fmax / df) + 1
    nf1 = max(_nint(p.fmin / df), 2)
    ommax = TWO_PI_F * (nf2 - 1) * df
    sigma = 5.0 * df
    dwn = TWO_PI_F / p.xlen
    wnmax = 0.5 * ommax * (p.p1lim + p.p2lim) / (1.0 - p.frac)
    nwnmax = int(wnmax / dwn) + 1
    if p.global_ == 1:
        nwnmax = _nint(wnmax * rearth - 0.5) + 1
    nwn = np.zeros(nf2, dtype=np.int32)
    for jf in range(nf1, nf2 + 1):
        f = (jf - 1) * df
        omre = 2.0 * PI_F * f
        if f <= 0.5 * (nf2 - 1) * df:
            wn2 = omre * p.p1lim + p.frac * wnmax
        else:
            wn2 = 0.5 * ommax * (p.p1lim + p.p2lim) + (omre - ommax) * p.p2lim + p.frac * wnmax
        if p.global_ == 1:
            nwn[jf - 1] = _nint(wn2 * rearth - 0.5) + 1
        else:
            nwn[jf - 1] = int(wn2 / dwn) + 1
    return FrequencyGrid(df, sigma, nf1, nf2, nwn, nwnmax, dwn)


def nsp_dsv(source_type: str) -> int:
    """Spectra per node of the DSV spectra with radial derivatives (U, V, dU/dr,
    dV/dr per spheroidal jump, W, dW/dr per toroidal jump) of a source in the
    solid (computeGreenFKSpectraForASKI.f90:231-233,306-328)."""
    njsph, njtor = (2, 1) if source_type == "FORCE" else (4, 2)
    return 4 * njsph + 2 * njtor


def aski_nf1(p: FKParams) -> int:
    """First frequency index of the ASKI FK program, max(nint(fmin/df), 1) + 1
    (computeGreenFKSpectraForASKI.f90:218-220); the rest of its grid is that of
    the synthetics program."""
    return max(_nint(p.fmin / (1.0 / p.tlen)), 1) + 1


def nsp_for(p: FKParams) -> int:
    """Number of FK spectra per node for a receiver in the solid (:274-313)."""
    njsph, njtor = (2, 1) if p.source_type == "FORCE" else (4, 2)
    if p.stressflag:
        return 4 * njsph + 2 * njtor
    return 2 * njsph + njtor
