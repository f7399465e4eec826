"""GPU against the CPU oracle at the benchmark's own configurations.

* Batched FK spectra (410 frequencies to 0.2 Hz, l <= 3205, 37 nodes): the
  whole band on the GPU, both builds, against the oracle on a seeded sample of
  two (omega, l) items per frequency (820 items, every frequency, all nodes).
  The plain build must agree to 1e-10 and the fast build to 1e-8 relative to
  the largest value of each spectrum (node, component) of the item's
  frequency, with identical NaN positions (the l = 0 V components).
* Degree sums of the tensor-core configuration (seeded log-normal FK
  coefficients of the batched grid's shape, l <= 3205, 8192 samples): 66
  stations including 0.5, 90 and 179.5 degrees (the near-antipodal one cancels
  the degree sum by five orders of magnitude), all six moment tensors, both
  sum forms, against the oracle's station loop: FP64 form to 1e-7 relative L2
  per trace, mixed form to the seismogram bar 1e-5.
* Regional FK spectra at the top frequency (5 Hz, nwn = 8001): a seeded sample
  of the wavenumbers, both builds, as for the batched configuration.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
RTOL_PLAIN = 1e-10
RTOL_FAST = 1e-8
RTOL_TRACE = {1: 1e-7, 2: 1e-5}


def _oracle_items(o, pc, g, nsp, items):
    """Oracle spectra [nnod, nsp] and status of single (jf, iwn) items, threads over items."""
    def one(it):
        jf, iwn = it
        spec, status, _ = o.fk_frequency(pc, jf, int(g.nwn[jf - 1]), nsp, iwn, iwn)
        return spec[:, :, iwn - 1].copy(), int(status[iwn - 1])
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as pool:
        return list(pool.map(one, items))


def _check_items(fk, w, jre, g, nsp, sample, refs, rtol, slab=41):
    """Run the band in slabs of frequencies and compare the sampled items, each
    relative to the largest value of every spectrum of its frequency."""
    by_jf = {}
    for (jf, iwn), r in zip(sample, refs):
        by_jf.setdefault(jf, []).append((iwn, r))
    jfs = sorted(by_jf)
    worst = 0.0
    for a in range(jfs[0], jfs[-1] + 1, slab):
        b = min(a + slab - 1, jfs[-1])
        _, _, g64, st = fk.run(w.params, jre, a, b, f32=False)
        assert np.all(st == 0)
        off = 0
        for jf in range(a, b + 1):
            n = int(g.nwn[jf - 1])
            blk = g64[:, :, off:off + n]
            scale = np.nanmax(np.abs(blk), axis=-1)
            for iwn, (ref, sto) in by_jf.get(jf, []):
                assert sto == 0
                got = blk[:, :, iwn - 1]
                assert np.array_equal(np.isnan(got), np.isnan(ref)), (jf, iwn)
                ok = ~np.isnan(ref)
                err = np.abs(got - ref)[ok] / np.maximum(scale[ok], 1e-300)
                if err.size:
                    worst = max(worst, float(err.max()))
            off += n
    assert worst <= rtol, worst
    return worst


@pytest.fixture(scope="module")
def batched(gpu):
    import oracle
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    assert ex.nnod == 37 and g.nf2 - g.nf1 + 1 == 410
    rng = np.random.default_rng(8)
    sample = [(jf, int(iwn)) for jf in range(g.nf1, g.nf2 + 1)
              for iwn in rng.choice(np.arange(1, int(g.nwn[jf - 1]) + 1), size=2, replace=False)]
    nsp = M.nsp_for(w.params)
    refs = _oracle_items(oracle.Oracle(m, ex), M.fk_params_c(w.params, jre), g, nsp, sample)
    return w, m, ex, jre, g, nsp, sample, refs


@pytest.mark.parametrize("backend", [1, 2])
def test_batched_fk_sample_over_every_frequency(batched, backend):
    from gemini_unified_b200.fk import GeminiFK
    w, m, ex, jre, g, nsp, sample, refs = batched
    assert len(sample) == 820 and len({jf for jf, _ in sample}) == 410
    worst = _check_items(GeminiFK(m, ex, backend=backend), w, jre, g, nsp, sample, refs,
                         RTOL_PLAIN if backend == 1 else RTOL_FAST)
    print("backend %d: worst relative error over %d items %.2e" % (backend, len(sample), worst))


@pytest.fixture(scope="module")
def sums_config(gpu):
    """Stations, seeded coefficients and the oracle's traces of the tensor-core configuration."""
    import oracle
    from gemini_unified_b200.fk import synth_params
    from gemini_unified_b200.synth_run import fk_coefficients
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    g = M.frequency_grid(w.params, m.rearth)
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)   # df and sigma float32-rounded, as the reference stores them
    assert int(g.nwn.max()) - 1 >= 3200 and w.nsamp == 8192
    gr, gi = fk_coefficients(10, int(g.nkfmax))
    d2r = np.pi / 180.0
    dist = np.concatenate([[0.5, 90.0, 179.5], np.linspace(1.0, 179.0, 63)])
    rng = np.random.default_rng(21)
    theta = np.ascontiguousarray(dist * d2r)
    phi = np.ascontiguousarray(rng.uniform(0.0, 2.0 * np.pi, dist.size))
    propdir = np.ascontiguousarray(phi + rng.uniform(-0.2, 0.2, dist.size))
    mt = configs.unit_moment_tensors()

    def one(i):
        return oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta[i:i + 1], phi[i:i + 1],
                                 propdir[i:i + 1], mt, w.filspecs, False, 0.0, w.nsamp, w.dt)
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as pool:
        ref = np.concatenate(list(pool.map(one, range(dist.size))), axis=0)
    return w, m, g, sp, gr, gi, theta, phi, propdir, mt, ref


@pytest.mark.parametrize("backend", [1, 2])
def test_tensor_core_sums_configuration_matches_oracle(sums_config, backend):
    from gemini_unified_b200.fk import GeminiFK
    w, m, g, sp, gr, gi, theta, phi, propdir, mt, ref = sums_config
    ex = w.nodes(m)
    got = GeminiFK(m, ex, backend=backend).synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    assert got.shape == ref.shape == (66, 6, 3, 8192)
    assert np.all(np.isfinite(got))
    scale = 1.0 / np.abs(ref).max()
    a = got.astype(np.float64).reshape(-1, w.nsamp) * scale
    b = ref.astype(np.float64).reshape(-1, w.nsamp) * scale
    num, den = np.linalg.norm(a - b, axis=1), np.linalg.norm(b, axis=1)
    assert np.all(den > 0)
    rel = num / den
    print("backend %d: trace rel L2 max %.2e median %.2e; antipodal station %.2e" %
          (backend, rel.max(), np.median(rel), rel.reshape(66, -1)[2].max()))
    assert rel.max() <= RTOL_TRACE[backend]


@pytest.mark.parametrize("backend", [1, 2])
def test_regional_top_frequency_matches_oracle(gpu, backend):
    import oracle
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["regional"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    jf = g.nf2
    n = int(g.nwn[jf - 1])
    assert n >= 8000
    rng = np.random.default_rng(5)
    # wn = 0 (iwn = 1) is not computed in the regional mode
    iwns = sorted({2, 3, n // 2, n} | set(int(i) for i in rng.choice(np.arange(4, n), size=28, replace=False)))
    sample = [(jf, i) for i in iwns]
    nsp = M.nsp_for(w.params)
    refs = _oracle_items(oracle.Oracle(m, ex), M.fk_params_c(w.params, jre), g, nsp, sample)
    worst = _check_items(GeminiFK(m, ex, backend=backend), w, jre, g, nsp, sample, refs,
                         RTOL_PLAIN if backend == 1 else RTOL_FAST)
    print("backend %d: worst relative error over %d wavenumbers of %g Hz %.2e" % (backend, len(sample),
                                                                                   (jf - 1) * g.df, worst))


def test_pipeline_stages_on_one_rank_equal_the_direct_calls(gpu):
    """The GPU stages of the multi-GPU pipeline (gemini_unified_b200.pipeline.GpuStages)
    through a one-rank NCCL group: FK spectra into device buffers, the all-gather, and
    the device seismogram entry point give the direct host calls' traces bit for bit
    (FP64 form, global configuration)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    from gemini_unified_b200 import pipeline as P
    from gemini_unified_b200.fk import GeminiFK, synth_params
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    nsp = M.nsp_for(w.params)
    src = ex.node_index(m.rearth - 10000.0)
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs)
    stations = w.stations()
    mt = configs.unit_moment_tensors()[[0, 5]]
    s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
    try:
        st = P.GpuStages(m, ex, w.params, jre, sp, stations, mt, device=0, backend=1)
        traces, sta, full = P.fk_to_traces(0, 1, g.nwn, g.nf1, g.nf2, nsp, src, len(stations[0]), st.fk_fn,
                                           st.synth_fn, device=torch.device("cuda", 0))
        torch.cuda.synchronize()
        got, slab = traces.cpu().numpy(), full.cpu().numpy()
    finally:
        dist.destroy_process_group()
    fk = GeminiFK(m, ex)
    gre, gim, _, _ = fk.run(w.params, jre, g.nf1, g.nf2, f64=False)
    assert np.array_equal(slab[0].view(np.uint32), gre[src - 1].view(np.uint32))
    assert np.array_equal(slab[1].view(np.uint32), gim[src - 1].view(np.uint32))
    ref = fk.synthetics(sp, g.nwn, gre[src - 1], gim[src - 1], *stations, mt)
    assert np.array_equal(np.arange(len(stations[0])), sta)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
