"""Concrete inputs of the benchmark / parity workloads.

Each workload is the parfile-equivalent of computeGreenFKSpectraForSynthetics
(templates/parfile_gfksyn_si) plus the synthetics geometry.  All inputs are
synthetic and deterministic; the earth model is the reference's PREM node
model (no ocean, SI units) made isotropic (PV -> P, SV -> S, eta = 1).

* ``global_small``  -- 51 frequencies to 0.05 Hz (df = 1/1024), l <= ~700,
  ~18k (omega, l) solves, source at 10 km depth, receiver at the surface;
  50 epicentral distances 1..170 deg, 6 unit moment tensors, 2048 samples
  at dt = 0.5 s.
* ``batched_fk``    -- 410 frequencies to 0.2 Hz (df = 1/2048), slowness
  4.0e-4 s/m (l <= ~3205, ~658k solves), 20 source depths 5..700 km plus the
  surface receiver.
* ``regional``      -- regional (flat, Bessel) mode: an 8-layer crust over a
  homogeneous halfspace (``regional_crust``), 512 frequencies to 5 Hz (df =
  1/102.4 s), slowness 1/1600 s/m and XLEN 2560 km (nwn <= ~8000 wavenumbers,
  ~2M solves), 24 source depths 1..24 km, receiver at the surface; 2000
  distances 1..200 km, 2048 samples at dt = 0.05 s.  (Source depths 0.5 km
  apart cannot straddle a crustal boundary: the node splitting of
  externalRadialNodes.f90:337-418 rejects two nodes within R 1e-4 = 637 m of
  one discontinuity.)
* ``regional_small`` -- the same to 1 Hz (103 frequencies, nwn <= 1601, ~82k
  solves) at 20 distances: the parity case of the regional mode.
* ``body_waves``    -- global body waves to 0.5 Hz (df = 1/2048, 1024
  frequencies), slowness 4.0e-4 s/m (l <= ~8006, ~4.1M solves), source at
  10 km depth, receiver at the surface: the evaluation workload of the learned
  step/order proposer.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Sequence

import numpy as np

from .model import ExternalRadialNodes, FKParams, NodeEarthModel, load_node_model, node_model_from_dict

MODEL_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                         "models")


def prem(isotropic: bool = True) -> NodeEarthModel:
    m = load_node_model(os.path.join(MODEL_DIR, "prem-no-ocean_si.json"))
    return m.isotropic() if isotropic else m


# crust of the regional model, top to bottom: thickness (km), vs (km/s), Q_mu
CRUST = [(1.0, 2.0, 100.0), (2.0, 2.4, 150.0), (2.0, 2.8, 200.0), (3.0, 3.1, 250.0), (3.0, 3.4, 300.0),
         (4.0, 3.6, 400.0), (5.0, 3.8, 500.0), (5.0, 4.0, 550.0)]
HALFSPACE = (4.6, 600.0)   # vs (km/s), Q_mu


def regional_crust(rearth: float = 6371000.0) -> NodeEarthModel:
    """Node model of the regional configuration: a homogeneous halfspace sphere
    (layer 1) below 8 crustal layers 1..5 km thick (25 km, boundaries at whole
    kilometres), vs 2.0 -> 4.0 km/s,
    vp = 1.73 vs, density from Gardner's rule rho = 1740 vp^0.25 (vp in km/s,
    rho in kg/m^3), Q_mu 100 -> 600, Q_kappa 57823; isotropic, no fluid layer.
    Each crustal layer is constant between its two knots."""
    layers = [(None, HALFSPACE[0], HALFSPACE[1])] + list(reversed(CRUST))   # bottom to top
    depth, vs, qm, tops, iktop = [], [], [], [], []
    z = sum(t for t, _, _ in CRUST) * 1000.0
    depth.append(z); vs.append(HALFSPACE[0]); qm.append(HALFSPACE[1])      # halfspace: one knot
    tops.append(rearth - z); iktop.append(1)
    for th, v, q in layers[1:]:
        ztop = z - th * 1000.0
        depth += [z, ztop]; vs += [v, v]; qm += [q, q]
        tops.append(rearth - ztop); iktop.append(len(depth))
        z = ztop
    vs_ms = [1000.0 * v for v in vs]
    vp_ms = [1.73 * v for v in vs_ms]
    rho = [1740.0 * (vp / 1000.0) ** 0.25 for vp in vp_ms]
    n = len(depth)
    d = {"reference_frequency_hz": 1.0, "anisotropic": False, "earth_radius": rearth, "full_space": 0,
         "equidistant_nodes": 1, "num_layers": len(layers), "num_nodes": n, "layer_inner_core": 0,
         "layer_outer_core": 0, "radius_inner_core": 0.0, "radius_outer_core": 0.0,
         "radius_upper_layer_boundary_m": tops, "isfluid": [0] * len(layers), "index_upper_boundary": iktop,
         "node_properties": {"depth": depth, "density": rho, "P-velocity": vp_ms, "S-velocity": vs_ms,
                             "Qkappa": [57823.0] * n, "Qmu": qm}}
    return node_model_from_dict(d, name="regional_crust")


@dataclasses.dataclass
class Workload:
    name: str
    params: FKParams
    nnod_blocks: List[int]
    dr_blocks: List[float]
    shift: float
    rec_radius: float
    isotropic: bool = True
    # synthetics
    ndist: int = 50
    dist_deg: tuple = (1.0, 170.0)
    azimuth_deg: float = 30.0
    nsamp: int = 2048
    dt: float = 0.5
    filspecs: tuple = (2.0, 0.002, 4.0, 0.04)
    dist_km: tuple = ()       # regional mode: distances in km instead of dist_deg
    crust: bool = False       # regional crustal model instead of PREM

    def model(self) -> NodeEarthModel:
        return regional_crust() if self.crust else prem(self.isotropic)

    def nodes(self, model: NodeEarthModel) -> ExternalRadialNodes:
        return ExternalRadialNodes.from_blocks(model, self.nnod_blocks, self.dr_blocks, self.shift,
                                               model.rearth)

    def stations(self):
        """(theta [rad], phi [rad], propdir [rad]) for a source at the north pole.

        With the source at the pole, the azimuth seen from the source is phi and
        the propagation direction at the receiver (from south over east) is phi
        as well (eventStationGeometry.f90:38-70 with ev_colat = 0).
        """
        d2r = np.pi / 180.0
        if self.dist_km:   # epicentral distance in radians of the model's radius
            theta = np.linspace(self.dist_km[0], self.dist_km[1], self.ndist) * 1000.0 / self.model().rearth
        else:
            theta = np.linspace(self.dist_deg[0], self.dist_deg[1], self.ndist) * d2r
        phi = np.full(self.ndist, self.azimuth_deg * d2r)
        return theta, phi, phi.copy()


def unit_moment_tensors() -> np.ndarray:
    """Six unit moment tensors (Mrr, Mtt, Mff, Mrt, Mrf, Mtf)."""
    return np.eye(6)


GLOBAL_SMALL = Workload(
    name="global_small",
    params=FKParams(tlen=1024.0, fmax=0.05, p1lim=3.5e-4, p2lim=3.5e-4, frac=0.0, eps=1.0e-5),
    nnod_blocks=[1], dr_blocks=[10000.0], shift=0.0, rec_radius=6371000.0,
    ndist=50, nsamp=2048, dt=0.5)

BATCHED_FK = Workload(
    name="batched_fk",
    params=FKParams(tlen=2048.0, fmax=0.2, p1lim=4.0e-4, p2lim=4.0e-4, frac=0.0, eps=1.0e-5),
    nnod_blocks=[1, 19], dr_blocks=[5000.0, 695000.0 / 19.0], shift=0.0, rec_radius=6371000.0,
    ndist=4000, dist_deg=(0.5, 179.5), nsamp=8192, dt=0.25)

BODY_WAVES = Workload(
    name="body_waves",
    params=FKParams(tlen=2048.0, fmax=0.5, p1lim=4.0e-4, p2lim=4.0e-4, frac=0.0, eps=1.0e-5),
    nnod_blocks=[1], dr_blocks=[10000.0], shift=0.0, rec_radius=6371000.0,
    ndist=50, nsamp=4096, dt=0.25)

REGIONAL = Workload(
    name="regional",
    params=FKParams(tlen=102.4, fmax=5.0, p1lim=1.0 / 1600.0, p2lim=1.0 / 1600.0, frac=0.0, xlen=2.56e6,
                    eps=1.0e-5, global_=0),
    nnod_blocks=[24], dr_blocks=[1000.0], shift=0.0, rec_radius=6371000.0, crust=True,
    ndist=2000, dist_km=(1.0, 200.0), nsamp=2048, dt=0.05, filspecs=(2.0, 0.05, 4.0, 3.0))

REGIONAL_SMALL = dataclasses.replace(
    REGIONAL, name="regional_small",
    params=dataclasses.replace(REGIONAL.params, fmax=1.0), ndist=20, filspecs=(2.0, 0.05, 4.0, 0.8))

WORKLOADS = {w.name: w for w in (GLOBAL_SMALL, BATCHED_FK, BODY_WAVES, REGIONAL, REGIONAL_SMALL)}
