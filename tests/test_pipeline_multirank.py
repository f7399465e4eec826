"""The multi-GPU FK-to-seismogram pipeline's exchange on two gloo ranks (CPU).

gemini_unified_b200.pipeline splits the frequencies over the ranks, gathers
the source node's float32 FK spectra of all frequencies with one all_gather,
and splits the stations.  Here both ranks run the same code with the CPU
oracle as the FK and seismogram stages, on a small global case (12
frequencies to 0.012 Hz, l <= ~150).  The gathered slab must equal the
single-process slab bit for bit, and each rank's traces the single-process
traces of its stations, for both frequency partitions (cost-balanced blocks
and the reference's zig-zag)."""
import dataclasses
import os
import socket

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M
from gemini_unified_b200 import pipeline as P


def _case():
    w = configs.WORKLOADS["global_small"]
    params = dataclasses.replace(w.params, fmax=0.012)
    m = w.model()
    ex = w.nodes(m)
    return w, params, m, ex


class _OracleStages:
    """FK and seismogram stages on the CPU oracle, shaped like the GPU stages."""

    def __init__(self):
        import oracle
        from gemini_unified_b200.fk import synth_params
        self.w, self.params, m, ex = _case()
        self.jre = ex.node_index(self.w.rec_radius)
        self.node = ex.node_index(m.rearth - 10000.0)
        self.g = M.frequency_grid(self.params, m.rearth)
        self.nsp = M.nsp_for(self.params)
        self.o = oracle.Oracle(m, ex)
        self.pc = M.fk_params_c(self.params, self.jre)
        self.sp = synth_params(self.g, self.nsp, self.w.nsamp, self.w.dt, self.w.filspecs)
        th, ph, pd = self.w.stations()
        sel = slice(0, 50, 8)   # 7 stations 1..170 degrees
        self.theta, self.phi, self.propdir = th[sel], ph[sel], pd[sel]
        self.mt = configs.unit_moment_tensors()[[0, 3]]

    def fk_fn(self, a, b):
        import torch
        spec = np.concatenate([self.o.fk_frequency(self.pc, jf, int(self.g.nwn[jf - 1]), self.nsp)[0]
                               for jf in range(a, b + 1)], axis=2)
        return torch.from_numpy(spec.real.astype(np.float32)), torch.from_numpy(spec.imag.astype(np.float32))

    def synth_fn(self, gre, gim, sta):
        import oracle
        import torch
        tr = oracle.synthetics(self.g.nf1, self.g.nf2, self.g.nwn, self.g.nwnmax, self.sp.df, self.sp.sigma,
                               gre.numpy(), gim.numpy(), self.theta[sta], self.phi[sta], self.propdir[sta], self.mt,
                               self.w.filspecs, False, 0.0, self.w.nsamp, self.w.dt)
        return torch.from_numpy(tr)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, size, port, partition, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=120))
    S = _OracleStages()
    traces, sta, full = P.fk_to_traces(rank, size, S.g.nwn, S.g.nf1, S.g.nf2, S.nsp, S.node, len(S.theta),
                                       S.fk_fn, S.synth_fn, partition=partition)
    out.put((rank, traces.numpy(), sta, full.numpy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.fixture(scope="module")
def single():
    """The single-process run: FK spectra of the whole band, traces of every station."""
    S = _OracleStages()
    re, im = S.fk_fn(S.g.nf1, S.g.nf2)
    full = np.stack([re[S.node - 1].numpy(), im[S.node - 1].numpy()])
    import torch
    traces = S.synth_fn(torch.from_numpy(full[0]), torch.from_numpy(full[1]), np.arange(len(S.theta))).numpy()
    return full, traces


@pytest.mark.parametrize("partition", ["blocks", "zigzag"])
def test_two_ranks_reproduce_the_single_process_run_bit_for_bit(single, partition):
    import torch.multiprocessing as mp
    full1, traces1 = single
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, partition, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seen = np.zeros(len(traces1), int)
    for rank, tr, sta, full in res:
        assert np.array_equal(full.view(np.uint32), full1.view(np.uint32))   # NaN positions included
        assert np.array_equal(tr.view(np.uint32), traces1[sta].view(np.uint32))
        seen[sta] += 1
    assert np.all(seen == 1)


@pytest.mark.parametrize("size", [1, 2, 3, 4, 8])
def test_cost_blocks_cover_the_band_once_and_balance_the_cost(size):
    w = configs.WORKLOADS["batched_fk"]
    g = M.frequency_grid(w.params, w.model().rearth)
    runs = P.cost_blocks(g.nwn, g.nf1, g.nf2, size)
    part = P.SlabPartition(g.nwn, g.nf1, g.nf2, runs)   # raises unless every column is covered once
    assert part.nkf == int(g.nkfmax)
    assert all(len(r) == 1 for r in runs)               # one FK launch per rank
    cost = [sum(P.frequency_cost(g.nwn, j) for a, b in r for j in range(a, b + 1)) for r in runs]
    assert max(cost) <= 1.03 * np.mean(cost)


def test_more_ranks_than_frequencies_leave_ranks_without_work():
    nwn = np.arange(1, 8)
    runs = P.cost_blocks(nwn, 2, 5, 6)
    assert [len(r) for r in runs] == [1, 1, 1, 1, 0, 0]
    P.SlabPartition(nwn, 2, 5, runs)
