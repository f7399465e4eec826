"""FK spectra to seismograms on several GPUs: frequency-sharded FK spectra, one
all-gather of the source node's spectra, station-sharded seismograms.

The reference splits the frequencies of computeGreenFKSpectraForSynthetics
over its MPI ranks (computeGreenFKSpectraForSynthetics.f90:361-387), each rank
writes its frequencies' slabs of the FK file (:508-519), and
computeSyntheticSeismograms reads the whole band of one source node from that
file before its station loop (computeSyntheticSeismograms.f90:290).  Here the
file in between is replaced by one collective:

1. each rank computes the FK spectra of its frequencies, all nodes, on its GPU
   (``fk_fn``);
2. the float32 spectra of the source node, (re, im) x nsp x (this rank's
   wavenumber-frequency columns), are padded to the widest rank and exchanged
   with one ``all_gather`` (NCCL over NVLink on GPUs, gloo on CPUs); every rank
   copies each rank's columns to their place in the full (nsp, nkfmax) slab --
   exact copies, so the slab equals a single-rank run bit for bit;
3. each rank computes the seismograms of its share of the stations from the
   full slab (``synth_fn``); no further exchange is needed, since the inverse
   FFT of a trace only needs that trace's spectrum.

The frequency split is either contiguous blocks of about equal cost, one FK
launch per rank (the default: on a GPU one large launch keeps the persistent
solver busy), or the reference's zig-zag order (``partition="zigzag"``, one
launch per contiguous run).  Nothing here issues TMA loads or multicast.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np


def zigzag(nf1: int, nf2: int, rank: int, size: int) -> List[int]:
    """Frequencies of one rank in the reference's order (computeGreenFKSpectraForSynthetics.f90:361-387)."""
    nf = nf2 - nf1 + 1
    npart = nf // size + (1 if nf % size else 0)
    out, jfe = [], nf2
    for k in range(1, npart + 1):
        jf = jfe - rank if k % 2 == 1 else jfe + rank - size + 1
        jfe -= size
        if jf < nf1:
            break
        out.append(jf)
    return sorted(out)


def contiguous_runs(js: Sequence[int]) -> List[Tuple[int, int]]:
    """Runs (first, last) of consecutive frequency indices."""
    runs, start, prev = [], None, None
    for a in js:
        if start is None:
            start = prev = a
        elif a == prev + 1:
            prev = a
        else:
            runs.append((start, prev))
            start = prev = a
    if start is not None:
        runs.append((start, prev))
    return runs


def frequency_cost(nwn: np.ndarray, jf: int) -> float:
    """Cost model of one frequency: its number of degrees times the number of
    wavelengths along a radial path (steps of a quarter wavelength,
    initialValues.f90:226), both growing with the frequency."""
    return float(nwn[jf - 1]) * float(max(jf - 1, 1))


def cost_blocks(nwn: np.ndarray, nf1: int, nf2: int, size: int) -> List[List[Tuple[int, int]]]:
    """Contiguous frequency blocks of about equal cost, one per rank.  Every rank
    gets at least one frequency while they last; ranks beyond the number of
    frequencies get none."""
    n = nf2 - nf1 + 1
    cum = np.cumsum([frequency_cost(nwn, j) for j in range(nf1, nf2 + 1)])
    bounds = [0]
    for r in range(1, size):
        e = int(np.searchsorted(cum, cum[-1] * r / size, side="left")) + 1
        lo = min(bounds[-1] + 1, n)
        hi = max(n - (size - r), lo)
        bounds.append(min(max(e, lo), hi))
    bounds.append(n)
    return [[(nf1 + bounds[r], nf1 + bounds[r + 1] - 1)] if bounds[r + 1] > bounds[r] else []
            for r in range(size)]


def partition_runs(nwn: np.ndarray, nf1: int, nf2: int, size: int, partition: str = "blocks"):
    """Frequency runs (first, last) of every rank."""
    if partition == "blocks":
        return cost_blocks(nwn, nf1, nf2, size)
    if partition == "zigzag":
        return [contiguous_runs(zigzag(nf1, nf2, r, size)) for r in range(size)]
    raise ValueError("partition must be 'blocks' or 'zigzag'")


class SlabPartition:
    """Which wavenumber-frequency columns k of the (nsp, nkfmax) slab each rank
    computes: k of (jf, iwn) = sum(nwn[nf1-1 : jf-1]) + iwn - 1."""

    def __init__(self, nwn: np.ndarray, nf1: int, nf2: int, runs_per_rank):
        self.nf1, self.nf2 = nf1, nf2
        self.koff = np.concatenate([[0], np.cumsum(np.asarray(nwn[nf1 - 1: nf2], np.int64))])
        self.nkf = int(self.koff[-1])
        self.runs = [list(r) for r in runs_per_rank]
        self.cols = []
        for runs in self.runs:
            parts = [np.arange(self.koff[a - nf1], self.koff[b - nf1 + 1], dtype=np.int64) for a, b in runs]
            self.cols.append(np.concatenate(parts) if parts else np.zeros(0, np.int64))
        self.width = max(1, max(len(c) for c in self.cols))
        allc = np.sort(np.concatenate(self.cols))
        if not np.array_equal(allc, np.arange(self.nkf)):
            raise ValueError("the ranks' frequency runs must cover every frequency exactly once")


def all_gather_slab(local, part: SlabPartition, rank: int, group=None):
    """All ranks' columns into the full slab.

    local: tensor (..., len(part.cols[rank])) of this rank's columns in
    part.cols[rank] order.  Returns (..., part.nkf) on local's device.  One
    all_gather of the padded local tensor; the placement is exact copies."""
    import torch
    import torch.distributed as dist
    size = dist.get_world_size(group)
    n = len(part.cols[rank])
    if local.shape[-1] != n:
        raise ValueError("rank %d holds %d columns, the partition gives it %d" % (rank, local.shape[-1], n))
    pad = torch.zeros(tuple(local.shape[:-1]) + (part.width,), dtype=local.dtype, device=local.device)
    pad[..., :n] = local
    bufs = [torch.empty_like(pad) for _ in range(size)]
    dist.all_gather(bufs, pad, group=group)
    full = torch.empty(tuple(local.shape[:-1]) + (part.nkf,), dtype=local.dtype, device=local.device)
    for r in range(size):
        c = part.cols[r]
        if len(c):
            full[..., torch.as_tensor(c, device=local.device)] = bufs[r][..., :len(c)]
    return full


def station_share(nsta: int, rank: int, size: int) -> np.ndarray:
    """Station indices of one rank (round robin: near and far stations on every rank)."""
    return np.arange(nsta)[rank::size]


def fk_to_traces(rank: int, size: int, nwn: np.ndarray, nf1: int, nf2: int, nsp: int, node: int, nsta: int,
                 fk_fn: Callable, synth_fn: Callable, partition: str = "blocks", group=None, device="cpu"):
    """The three stages on this rank.

    fk_fn(jf_first, jf_last) -> (re, im): float32 tensors (nnod, nsp, nkf of the
    run), the FK spectra of every node for frequencies jf_first..jf_last.
    synth_fn(gre, gim, stations) -> traces of the given station indices from
    the full (nsp, nkfmax) float32 slab of the source node.
    node: 1-based source node; device: where the exchange buffers live (the
    GPU for NCCL).  Returns (traces of this rank's stations, their indices, the
    full (2, nsp, nkfmax) slab)."""
    import torch
    runs = partition_runs(nwn, nf1, nf2, size, partition)
    part = SlabPartition(nwn, nf1, nf2, runs)
    pieces = []
    for a, b in part.runs[rank]:
        re, im = fk_fn(a, b)
        pieces.append(torch.stack([re[node - 1], im[node - 1]]))
    if pieces:
        local = torch.cat(pieces, dim=-1)
    else:   # a rank without frequencies still takes part in the collective
        local = torch.zeros((2, nsp, 0), dtype=torch.float32, device=device)
    full = all_gather_slab(local, part, rank, group)
    sta = station_share(nsta, rank, size)
    traces = synth_fn(full[0], full[1], sta)
    return traces, sta, full


class GpuStages:
    """fk_fn and synth_fn of fk_to_traces on one GPU through the library's
    device entry points (gem_fk_run_device, gem_synth_run_device): buffers stay
    in HBM, and the slab exchange runs over NCCL."""

    def __init__(self, model, nodes, params, jre: int, synth_params, stations, mt, device: int = 0,
                 backend: int = 2, stream=None):
        import torch
        from .fk import GeminiFK
        from .model import frequency_grid, nsp_for
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.fk = GeminiFK(model, nodes, device=device, backend=backend)
        self.params, self.jre = params, jre
        self.grid = frequency_grid(params, model.rearth)
        self.nsp = nsp_for(params)
        self.nnod = nodes.nnod
        self.sp = synth_params
        self.theta, self.phi, self.propdir = (np.ascontiguousarray(a, np.float64) for a in stations)
        self.mt = np.ascontiguousarray(mt, np.float64)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.dev)

    def fk_fn(self, a: int, b: int):
        torch = self.torch
        nkf = int(self.grid.nwn[a - 1: b].sum())
        re = torch.empty((self.nnod, self.nsp, nkf), dtype=torch.float32, device=self.dev)
        im = torch.empty_like(re)
        st = torch.empty(nkf, dtype=torch.int32, device=self.dev)
        self.fk.run_device(self.params, self.jre, a, b, gfre=re.data_ptr(), gfim=im.data_ptr(), status=st.data_ptr(),
                           stream=self.stream.cuda_stream)
        if int(st.abs().sum()) != 0:
            raise RuntimeError("failed (omega, l) items in frequencies %d..%d" % (a, b))
        return re, im

    def synth_fn(self, gre, gim, sta):
        import ctypes
        from .fk import lib
        torch = self.torch
        th, ph, pd = (np.ascontiguousarray(x[sta]) for x in (self.theta, self.phi, self.propdir))
        out = torch.empty((len(sta), len(self.mt), 3, self.sp.nsamp), dtype=torch.float32, device=self.dev)
        if len(sta) == 0:
            return out
        gre, gim = gre.contiguous(), gim.contiguous()
        nwn = np.ascontiguousarray(self.grid.nwn, np.int32)
        p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
        self.fk._check(lib().gem_synth_run_device(self.fk._h, ctypes.byref(self.sp), p(nwn), gre.data_ptr(),
                                                  gim.data_ptr(), len(sta), p(th), p(ph), p(pd), len(self.mt),
                                                  p(self.mt), out.data_ptr(), ctypes.c_void_p(self.stream.cuda_stream)))
        return out
