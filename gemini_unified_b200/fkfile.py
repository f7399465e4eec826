"""The FK-spectra file between computeGreenFKSpectraForSynthetics and
computeSyntheticSeismograms, written and read in the reference's HDF5 layout.

Layout (computeGreenFKSpectraForSynthetics.f90:242-343,508-519;
greenFKSpectra.f90:71-167; externalRadialNodes.f90:209-324).  The reference
writes from Fortran, whose array dimensions HDF5 stores in reverse order, so a
Fortran array (nkfmax, nsp, nnod) is the HDF5 dataspace [nnod][nsp][nkfmax] --
exactly the library's FK output layout (k fastest):

* root attribute ``identity``: fdate() string of the run;
* root attribute ``dataSpecificIntegers``: int32 [istyp, ncsph, nctor, njsph, njtor];
* ``earthModelName``, ``attenuationMode``: scalar fixed-length strings;
* ``reals``: float32 [rearth, re, sigma, df, dwn, fref];
* ``integers``: int32 [nf1, nf2, nkfmax, nwnmax, dsvstep = 2, derivflag = 0,
  numtasks, global];
* ``numberOfWavenumbersForFrequency``: int32 nwn(1:nf2);
* group ``externalNodes``: ``rearth`` float32 [1], ``radii`` float32 [nnod],
  ``state``, ``layer`` int32 [nnod], ``density`` float32 [nnod],
  ``inverseQ`` float32 [nnod][2], ``realElcon`` and ``imagElcon`` float32
  [nnod][7] (the model at the reference frequency, ELASTIC mode);
* ``GreenFKSpectraReal`` and ``GreenFKSpectraImag``: float32 [nnod][nsp][nkfmax].

A writer lays out the metadata and allocates both spectra datasets at once;
each frequency slab is then written where the reference's independent MPI-IO
writes put it (offset sum(nwn(1:jf-1)) along k), so slabs may arrive in any
order, as the ranks of the reference deliver them.
"""
from __future__ import annotations

import dataclasses
import os
import time
from typing import Optional

import numpy as np

from . import h5file
from .model import (ExternalRadialNodes, FKParams, FrequencyGrid, NodeEarthModel, frequency_grid,
                    node_elastic_constants, nsp_for)


@dataclasses.dataclass
class FKFileMeta:
    """What readMetaGreenFKSpectra (greenFKSpectra.f90:71-137) takes from the file."""
    identity: str
    earth_model_name: str
    attenuation_mode: str
    rearth: float
    re: float
    sigma: float
    df: float
    dwn: float
    fref: float
    nf1: int
    nf2: int
    nkfmax: int
    nwnmax: int
    dsvstep: int
    derivflag: int
    numtasks: int
    global_: int
    nwn: np.ndarray
    istyp: int
    ncsph: int
    nctor: int
    njsph: int
    njtor: int
    nsp: int
    nnod: int
    node_radii: np.ndarray
    node_state: np.ndarray
    node_layer: np.ndarray
    node_density: np.ndarray
    node_qinv: np.ndarray
    node_elcon: np.ndarray

    def dsvmask(self) -> np.ndarray:
        """Components present (greenFKSpectra.f90:117-133): U R V S UP VP W T WP."""
        m = np.array([1, 0, 1, 0, 0, 0, 1, 0, 0])
        if self.derivflag == 1:
            m[[4, 5, 8]] = 1
        if self.dsvstep == 1:
            m[[1, 3, 7]] = 1
        if self.ncsph == 2:
            m[3] = 0
        if self.nctor == 0:
            m[[6, 7, 8]] = 0
        return m

    def position(self, isp: int, jsp: int) -> int:
        """1-based index of spectrum (component isp 1..9, jump jsp) in the nsp
        dimension (positionDataGreenFKSpectra, greenFKSpectra.f90:204-212)."""
        m = self.dsvmask()
        if isp <= 6:
            return int(m[:isp - 1].sum()) * self.njsph + jsp
        return int(m[:6].sum()) * self.njsph + int(m[6:isp - 1].sum()) * self.njtor + jsp


def fdate() -> str:
    """The date string of Fortran's fdate(), as the reference stamps its files."""
    t = time.localtime()
    return time.strftime("%a %b ", t) + "%2d" % t.tm_mday + time.strftime(" %H:%M:%S %Y", t)


class FKFileWriter:
    """Writes the FK-spectra file of one run: the metadata at creation, the
    spectra frequency slab by frequency slab (write_slab), in any order."""

    def __init__(self, path: str, model: NodeEarthModel, nodes: ExternalRadialNodes, params: FKParams, jre: int,
                 earth_model_name: str = "", numtasks: int = 1, identity: Optional[str] = None):
        g = frequency_grid(params, model.rearth)
        self.grid: FrequencyGrid = g
        self.nsp = nsp_for(params)
        self.nnod = nodes.nnod
        self.nkfmax = int(g.nkfmax)
        self.koff = np.concatenate([[0], np.cumsum(np.asarray(g.nwn[g.nf1 - 1: g.nf2], np.int64))])
        istyp = 0 if params.source_type == "FORCE" else 1
        receiver_in_fluid = int(nodes.state[jre - 1]) == 1
        ncsph, nctor = (2, 0) if receiver_in_fluid else (4, 2)
        njsph, njtor = (2, 1) if istyp == 0 else (4, 2)
        ro, qinv, elcon = node_elastic_constants(model, nodes)
        f32, i32 = np.float32, np.int32
        w = h5file.H5Writer(path)
        w.set_attr("/", "identity", identity if identity is not None else fdate())
        w.create_string("earthModelName", earth_model_name or model.name or "model")
        w.create_string("attenuationMode", params.attmode)
        w.create_dataset("reals", np.array([model.rearth, nodes.r[jre - 1], g.sigma, g.df, g.dwn, model.fref], f32))
        w.create_group("externalNodes")
        w.create_dataset("externalNodes/rearth", np.array([model.rearth], f32))
        w.create_dataset("externalNodes/radii", np.asarray(nodes.r, f32))
        w.create_dataset("externalNodes/state", np.asarray(nodes.state, i32))
        w.create_dataset("externalNodes/layer", np.asarray(nodes.layer, i32))
        w.create_dataset("externalNodes/density", np.asarray(ro, f32))
        w.create_dataset("externalNodes/inverseQ", np.asarray(qinv, f32))
        w.create_dataset("externalNodes/realElcon", np.asarray(elcon.real, f32))
        w.create_dataset("externalNodes/imagElcon", np.asarray(elcon.imag, f32))
        w.create_dataset("numberOfWavenumbersForFrequency", np.asarray(g.nwn[: g.nf2], i32))
        w.create_dataset("integers", np.array([g.nf1, g.nf2, self.nkfmax, g.nwnmax, 2, 0, numtasks, params.global_], i32))
        w.set_attr("/", "dataSpecificIntegers", np.array([istyp, ncsph, nctor, njsph, njtor], i32))
        shape = (self.nnod, self.nsp, self.nkfmax)
        w.create_dataset("GreenFKSpectraReal", shape=shape, dtype="<f4")
        w.create_dataset("GreenFKSpectraImag", shape=shape, dtype="<f4")
        w.close()
        self._off = {"re": w.data_offset("GreenFKSpectraReal"), "im": w.data_offset("GreenFKSpectraImag")}
        self._fd = os.open(path, os.O_RDWR)

    def write_slab(self, jf_first: int, jf_last: int, gfre, gfim) -> None:
        """float32 spectra of frequencies jf_first..jf_last, shaped (nnod, nsp, nkf of
        the slab) -- the C view of the library's Fortran (nkf, nsp, nnod) output."""
        g = self.grid
        if not (g.nf1 <= jf_first <= jf_last <= g.nf2):
            raise ValueError("frequencies %d..%d outside %d..%d" % (jf_first, jf_last, g.nf1, g.nf2))
        k0, k1 = int(self.koff[jf_first - g.nf1]), int(self.koff[jf_last - g.nf1 + 1])
        for key, a in (("re", gfre), ("im", gfim)):
            a = np.ascontiguousarray(a, np.float32)
            if a.shape != (self.nnod, self.nsp, k1 - k0):
                raise ValueError("slab shape %s, expected %s" % (a.shape, (self.nnod, self.nsp, k1 - k0)))
            for n in range(self.nnod):
                for isp in range(self.nsp):
                    pos = self._off[key] + 4 * ((n * self.nsp + isp) * self.nkfmax + k0)
                    os.pwrite(self._fd, a[n, isp].tobytes(), pos)

    def close(self) -> None:
        if self._fd is not None:
            os.fsync(self._fd)
            os.close(self._fd)
            self._fd = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class FKFile:
    """Read access to an FK-spectra file (readMetaGreenFKSpectra,
    readDataNodeGreenFKSpectra: greenFKSpectra.f90:71-167)."""

    def __init__(self, path: str):
        self.h5 = h5file.H5Reader(path)
        f = self.h5
        s = lambda name: bytes(f[name].read().item()).decode("ascii")
        reals = f["reals"].read()
        ints = f["integers"].read()
        dsi = f.attrs["dataSpecificIntegers"]
        ex = f["externalNodes"]
        spec = f["GreenFKSpectraReal"]
        self.meta = FKFileMeta(
            identity=bytes(f.attrs["identity"].item()).decode("ascii"), earth_model_name=s("earthModelName"),
            attenuation_mode=s("attenuationMode"), rearth=float(reals[0]), re=float(reals[1]),
            sigma=float(reals[2]), df=float(reals[3]), dwn=float(reals[4]), fref=float(reals[5]),
            nf1=int(ints[0]), nf2=int(ints[1]), nkfmax=int(ints[2]), nwnmax=int(ints[3]), dsvstep=int(ints[4]),
            derivflag=int(ints[5]), numtasks=int(ints[6]), global_=int(ints[7]),
            nwn=f["numberOfWavenumbersForFrequency"].read(), istyp=int(dsi[0]), ncsph=int(dsi[1]),
            nctor=int(dsi[2]), njsph=int(dsi[3]), njtor=int(dsi[4]), nsp=int(spec.shape[1]),
            nnod=int(spec.shape[0]), node_radii=ex["radii"].read(), node_state=ex["state"].read(),
            node_layer=ex["layer"].read(), node_density=ex["density"].read(), node_qinv=ex["inverseQ"].read(),
            node_elcon=ex["realElcon"].read() + 1j * ex["imagElcon"].read())
        if spec.shape[2] != self.meta.nkfmax:
            raise h5file.H5FormatError("spectra extent %d differs from nkfmax %d" % (spec.shape[2], self.meta.nkfmax))

    def grid(self) -> FrequencyGrid:
        """The frequency grid of the file (its float32 df, sigma and dwn, as the
        reference's synthetics program reads them)."""
        m = self.meta
        nwn = np.zeros(m.nf2, np.int64)
        nwn[: len(m.nwn)] = m.nwn
        return FrequencyGrid(m.df, m.sigma, m.nf1, m.nf2, nwn, m.nwnmax, m.dwn)

    def read_node(self, jr: int):
        """(gfkr, gfki) float32 (nsp, nkfmax) of external node jr (1-based)."""
        if not 1 <= jr <= self.meta.nnod:
            raise ValueError("node %d outside 1..%d" % (jr, self.meta.nnod))
        return (self.h5["GreenFKSpectraReal"].read_rows(jr - 1, 1)[0],
                self.h5["GreenFKSpectraImag"].read_rows(jr - 1, 1)[0])

    def close(self):
        self.h5.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
