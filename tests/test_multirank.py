"""Host logic of the multi-GPU path, on the CPU.

bench.py splits the frequencies over the ranks in the reference's zig-zag
order (computeGreenFKSpectraForSynthetics.f90:361-387), splits the stations of
the seismogram leg round-robin, and reduces times with a maximum over ranks.
These tests check the split on its own and run two gloo ranks through the same
reductions."""
import os
import socket

import numpy as np
import pytest

import bench
from gemini_unified_b200 import configs, model as M


def _grid():
    w = configs.WORKLOADS["batched_fk"]
    return M.frequency_grid(w.params, w.model().rearth)


@pytest.mark.parametrize("size", [1, 2, 3, 4, 8])
def test_zigzag_covers_every_frequency_once_and_balances_cost(size):
    g = _grid()
    parts = [bench.zigzag(g.nf1, g.nf2, r, size) for r in range(size)]
    allf = sorted(f for p in parts for f in p)
    assert allf == list(range(g.nf1, g.nf2 + 1))
    # the work of a frequency grows with its number of degrees: the zig-zag keeps ranks within 2 %
    work = [int(g.nwn[np.array(p) - 1].sum()) for p in parts]
    assert max(work) <= 1.02 * np.mean(work)
    for p in parts:
        runs = bench.contiguous_runs(p)
        assert sum(b - a + 1 for a, b in runs) == len(p)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, size, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size)
    g = _grid()
    cover = torch.zeros(g.nf2 + 1, dtype=torch.int64)
    for f in bench.zigzag(g.nf1, g.nf2, rank, size):
        cover[f] += 1
    dist.all_reduce(cover)
    w = configs.WORKLOADS["batched_fk"]
    theta, _, _ = w.stations()
    sta = torch.zeros(len(theta), dtype=torch.int64)
    sta[np.arange(len(theta))[slice(rank, None, size)]] = 1
    dist.all_reduce(sta)
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((cover.tolist(), int(sta.min()), int(sta.max()), float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_all_work_and_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cover, smin, smax, tmax = res
    g = _grid()
    assert all(c == 1 for c in cover[g.nf1:]) and sum(cover[:g.nf1]) == 0
    assert smin == smax == 1
    assert tmax == 11.0
