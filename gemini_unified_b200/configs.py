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

from .model import ExternalRadialNodes, FKParams, NodeEarthModel, load_node_model

MODEL_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                         "models")


def prem(isotropic: bool = True) -> NodeEarthModel:
    m = load_node_model(os.path.join(MODEL_DIR, "prem-no-ocean_si.json"))
    return m.isotropic() if isotropic else m


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

    def model(self) -> NodeEarthModel:
        return prem(self.isotropic)

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

WORKLOADS = {w.name: w for w in (GLOBAL_SMALL, BATCHED_FK, BODY_WAVES)}
