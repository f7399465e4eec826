"""GPU parity of the FK solver against the CPU oracle (through the C ABI).

Tolerance: the FP64 solver repeats the reference's arithmetic operation by
operation (no FMA contraction); its spectra must agree with the oracle to
1e-10 relative to the largest value of each spectrum (the bar for the FP64
path is 1e-8), with identical NaN positions (l = 0 V components)."""
import dataclasses

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _cmp(a, b):
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    ok = ~na
    scale = np.abs(b[ok]).max()
    return np.abs(a[ok] - b[ok]).max() / scale


@pytest.fixture(scope="module")
def small(gpu):
    import oracle
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    return w, m, ex, jre, GeminiFK(m, ex), oracle.Oracle(m, ex)


@pytest.fixture(scope="module")
def small_ref(small):
    """Oracle spectra of every frequency of the global configuration (threads over frequencies)."""
    import concurrent.futures as cf
    import os
    w, m, ex, jre, fk, o = small
    g = M.frequency_grid(w.params, m.rearth)
    pc = M.fk_params_c(w.params, jre)
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as pool:
        refs = list(pool.map(lambda jf: o.fk_frequency(pc, jf, int(g.nwn[jf - 1]), 10)[0], range(g.nf1, g.nf2 + 1)))
    return g, refs


def test_global_small_all_frequencies(small, small_ref):
    """Every frequency of the 51-frequency global configuration, all 18169 solves."""
    w, m, ex, jre, fk, o = small
    g, refs = small_ref
    gre, gim, g64, st = fk.run(w.params, jre, g.nf1, g.nf2)
    assert np.all(st == 0)
    off = 0
    worst = 0.0
    for jf in range(g.nf1, g.nf2 + 1):
        n = int(g.nwn[jf - 1])
        ref = refs[jf - g.nf1]
        got = g64[:, :, off:off + n]
        worst = max(worst, _cmp(got, ref))
        # float32 outputs are the rounded FP64 values
        fin = ~np.isnan(ref)
        assert np.array_equal(gre[:, :, off:off + n][fin], got.real[fin].astype(np.float32))
        off += n
    assert worst <= RTOL


def test_batched_highest_frequency_sample(gpu):
    import oracle
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    jf = g.nf2
    n = int(g.nwn[jf - 1])
    fk = GeminiFK(m, ex)
    _, _, g64, st = fk.run(w.params, jre, jf, jf, f32=False)
    assert np.all(st == 0)
    o = oracle.Oracle(m, ex)
    pc = M.fk_params_c(w.params, jre)
    for iwn in (1, 2, 17, 400, 1601, 3000, n):
        ref, sto, _ = o.fk_frequency(pc, jf, n, 10, iwn, iwn)
        a, b = g64[:, :, iwn - 1], ref[:, :, iwn - 1]
        if iwn == 1:
            assert np.array_equal(np.isnan(a), np.isnan(b))
            ok = ~np.isnan(b)
            a, b = a[ok], b[ok]
        assert np.abs(a - b).max() <= RTOL * np.abs(b).max()


def test_deterministic_and_device_api(small):
    import torch
    w, m, ex, jre, fk, o = small
    _, _, a, _ = fk.run(w.params, jre, 30, 34, f32=False)
    _, _, b, _ = fk.run(w.params, jre, 30, 34, f32=False)
    assert np.array_equal(np.nan_to_num(a, nan=1.0), np.nan_to_num(b, nan=1.0))
    g = M.frequency_grid(w.params, m.rearth)
    nkf = int(g.nwn[29:34].sum())
    d64 = torch.zeros((ex.nnod, 10, nkf, 2), dtype=torch.float64, device="cuda")
    dst = torch.ones(nkf, dtype=torch.int32, device="cuda")
    fk.run_device(w.params, jre, 30, 34, gf64=d64.data_ptr(), status=dst.data_ptr())
    torch.cuda.synchronize()
    c = torch.view_as_complex(d64).cpu().numpy()
    assert np.array_equal(np.nan_to_num(a, nan=1.0), np.nan_to_num(c, nan=1.0))
    assert int(dst.abs().sum()) == 0


def test_fault_injection_min_step_status(small):
    """An unreachable accuracy: every item ends with status 1 (step size below
    minimum), the call returns an error, nothing hangs."""
    from gemini_unified_b200.model import GeminiError
    w, m, ex, jre, fk, o = small
    bad = dataclasses.replace(w.params, eps=1e-30)
    with pytest.raises(GeminiError):
        fk.run(bad, jre, 3, 3)
    _, _, _, st = fk.run(bad, jre, 3, 3, raise_on_failure=False)
    assert np.all(st[1:] == 1)


def test_rejects_invalid_inputs(small):
    from gemini_unified_b200.model import GeminiError
    w, m, ex, jre, fk, o = small
    with pytest.raises(GeminiError):
        fk.run(w.params, jre, 1, 3)          # below nf1
    with pytest.raises(GeminiError):
        fk.run(w.params, ex.nnod + 5, 3, 3)  # receiver node out of range


# The fast build contracts products into FMAs, evaluates the splines from a
# per-interval Horner table and replaces divisions by reciprocals: rounding
# differs from the reference's, so its bar is the FP64 spectral bar itself,
# 1e-8 relative to the largest value of each spectrum (node, component).
RTOL_FAST = 1e-8


def _cmp_per_spectrum(a, b):
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    err = np.where(na, 0.0, np.abs(a - b))
    scale = np.nanmax(np.where(na, 0.0, np.abs(b)), axis=-1, keepdims=True)
    return float((err / np.maximum(scale, 1e-300)).max())


def test_fast_backend_global_small(small, small_ref):
    """Fast build against the oracle on every solve of the global configuration."""
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST
    w, m, ex, jre, _, o = small
    g, refs = small_ref
    fast = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    _, _, g64, st = fast.run(w.params, jre, g.nf1, g.nf2, f32=False)
    assert np.all(st == 0)
    ref = np.concatenate(refs, axis=2)
    assert _cmp_per_spectrum(g64, ref) <= RTOL_FAST


def test_fast_backend_batched_slab(gpu):
    """Fast against plain on a slab of the batched configuration's top frequencies."""
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    plain = GeminiFK(m, ex)
    fast = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    _, _, a, sa = plain.run(w.params, jre, g.nf2 - 3, g.nf2, f32=False)
    _, _, b, sb = fast.run(w.params, jre, g.nf2 - 3, g.nf2, f32=False)
    assert np.all(sa == 0) and np.all(sb == 0)
    assert _cmp_per_spectrum(b, a) <= RTOL_FAST


@pytest.mark.parametrize("istyp,stress", [(0, 0), (1, 1), (0, 1)])
@pytest.mark.parametrize("backend", [1, 2])
def test_force_source_and_stress_outputs(small, istyp, stress, backend):
    """Force sources (nsp 5, or 10 with stresses) and moment sources with
    stresses (nsp 20) against the oracle, on three frequencies of the global
    configuration; plain build to the parity bar, fast build to the FP64 bar."""
    from gemini_unified_b200.fk import GeminiFK
    w, m, ex, jre, _, o = small
    params = dataclasses.replace(w.params, source_type="FORCE" if istyp == 0 else "MOMENT", stressflag=bool(stress))
    nsp = M.nsp_for(params)
    assert nsp == {(0, 0): 5, (1, 1): 20, (0, 1): 10}[(istyp, stress)]
    g = M.frequency_grid(params, m.rearth)
    fk = GeminiFK(m, ex, backend=backend)
    _, _, g64, st = fk.run(params, jre, 20, 22, f32=False)
    assert np.all(st == 0) and g64.shape[1] == nsp
    pc = M.fk_params_c(params, jre)
    ref = np.concatenate([o.fk_frequency(pc, jf, int(g.nwn[jf - 1]), nsp)[0] for jf in (20, 21, 22)], axis=2)
    assert _cmp_per_spectrum(g64, ref) <= (RTOL if backend == 1 else RTOL_FAST)


def test_graph_replay_matches_direct_run(small):
    """The captured launch sequence of a slab gives the direct run's spectra and
    status bit for bit, on two replays; a later direct run invalidates it."""
    import torch
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST
    from gemini_unified_b200.model import GeminiError
    w, m, ex, jre, _, o = small
    g = M.frequency_grid(w.params, m.rearth)
    for backend in (1, GEM_BACKEND_GPU_FAST):
        fk = GeminiFK(m, ex, backend=backend)
        _, _, ref, st = fk.run(w.params, jre, 20, 30, f32=False)
        nkf = int(g.nwn[19:30].sum())
        d64 = torch.empty((ex.nnod, 10, nkf, 2), dtype=torch.float64, device="cuda")
        dst = torch.empty(nkf, dtype=torch.int32, device="cuda")
        fk.graph_build(w.params, jre, 20, 30, gf64=d64.data_ptr(), status=dst.data_ptr())
        for _ in range(2):
            d64.fill_(7.0)
            fk.graph_launch()
            torch.cuda.synchronize()
            got = torch.view_as_complex(d64).cpu().numpy()
            assert np.array_equal(np.nan_to_num(got, nan=1.0), np.nan_to_num(ref, nan=1.0))
            assert int(dst.abs().sum()) == 0
        fk.run(w.params, jre, 3, 3, f32=False)
        with pytest.raises(GeminiError):
            fk.graph_launch()


def test_every_schedule_gives_identical_spectra(small):
    """Block size, matrix caching and the bookkeeping deferral change the time
    only: every schedule and deferral of both backends gives the default's
    spectra bit for bit."""
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST, NDEFER, NGRAN, NSCHED
    from gemini_unified_b200.model import GeminiError
    w, m, ex, jre, _, o = small
    for backend in (1, GEM_BACKEND_GPU_FAST):
        fk = GeminiFK(m, ex, backend=backend)
        assert fk.schedule() == [1, 0, 1] and fk.defer() == [4, 4, 4]
        _, _, ref, st = fk.run(w.params, jre, 40, 52, f32=False)
        assert np.all(st == 0)
        same = lambda got: np.array_equal(np.nan_to_num(got, nan=1.0), np.nan_to_num(ref, nan=1.0))
        for s in range(NSCHED):
            fk.schedule_set([s, s, s])
            _, _, got, st = fk.run(w.params, jre, 40, 52, f32=False)
            assert np.all(st == 0) and same(got), (backend, "schedule", s)
        for d in range(NDEFER):
            fk.defer_set([d, d, d])
            _, _, got, st = fk.run(w.params, jre, 40, 52, f32=False)
            assert np.all(st == 0) and same(got), (backend, "deferral", d)
        assert fk.queue() == [0, 0, 0]
        for q in range(NGRAN):
            fk.queue_set([q, q, q])
            _, _, got, st = fk.run(w.params, jre, 40, 52, f32=False)
            assert np.all(st == 0) and same(got), (backend, "queue granularity", q)
        with pytest.raises(GeminiError):
            fk.queue_set([0, NGRAN, 0])
        with pytest.raises(GeminiError):
            fk.schedule_set([0, NSCHED, 0])
        with pytest.raises(GeminiError):
            fk.defer_set([NDEFER, 0, 0])


def test_autotune_keeps_the_fastest_schedule(small):
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST, NDEFER, NGRAN, NSCHED
    w, m, ex, jre, _, o = small
    for backend, ncand in ((1, 3), (GEM_BACKEND_GPU_FAST, NSCHED)):
        fk = GeminiFK(m, ex, backend=backend)
        r = fk.autotune(w.params, jre, 44, 52)
        ms = r["ms"]
        assert ms.shape == (NSCHED + NDEFER + NGRAN, 3)
        assert np.all(ms[:ncand] > 0) and np.all(ms[ncand:NSCHED] == -1) and np.all(ms[NSCHED:] > 0)
        for ph in range(3):
            assert r["schedule"][ph] == int(np.argmin(ms[:ncand, ph]))
            assert r["defer"][ph] == int(np.argmin(ms[NSCHED:NSCHED + NDEFER, ph]))
            assert r["queue"][ph] == int(np.argmin(ms[NSCHED + NDEFER:, ph]))
        assert fk.schedule() == r["schedule"] and fk.defer() == r["defer"] and fk.queue() == r["queue"]
        _, _, g64, st = fk.run(w.params, jre, 44, 52, f32=False)
        assert np.all(st == 0)


@pytest.mark.parametrize("corrupt", ["knots_not_monotone", "nan_velocity", "inf_density"])
def test_corrupted_model_is_rejected(small, corrupt):
    """A corrupted earth model is refused on the host when it is loaded, with an
    error and no kernel launched: knot depths that do not increase monotonically,
    or non-finite values."""
    from gemini_unified_b200.fk import GeminiFK
    from gemini_unified_b200.model import GeminiError
    w, m, ex, jre, fk, o = small
    bad = dataclasses.replace(m, depth=m.depth.copy(), vpv=m.vpv.copy(), ro=m.ro.copy())
    if corrupt == "knots_not_monotone":
        k = len(bad.depth) // 2
        bad.depth[k], bad.depth[k + 1] = bad.depth[k + 1] + 1000.0, bad.depth[k]
    elif corrupt == "nan_velocity":
        bad.vpv[3] = np.nan
    else:
        bad.ro[5] = np.inf
    with pytest.raises(GeminiError):
        GeminiFK(bad, ex)
    # the context that loaded the good model still runs
    _, _, g64, st = fk.run(w.params, jre, 3, 3, f32=False)
    assert np.all(st == 0)


def test_batched_run_with_resume_matches_one_call(small, tmp_path):
    """fk_batches over the whole band in batches of 16 frequencies, on the GPU, gives
    the float32 spectra of one call for the whole band; a second run computes nothing."""
    from gemini_unified_b200 import fk_batches
    w, m, ex, jre, fk, o = small
    g = M.frequency_grid(w.params, m.rearth)
    res = fk_batches.run(fk, w.params, jre, str(tmp_path), 16)
    assert all(c for _, c in res)
    gre, gim, st = fk_batches.load(str(tmp_path))
    ref_re, ref_im, _, ref_st = fk.run(w.params, jre, g.nf1, g.nf2, f64=False)
    np.testing.assert_array_equal(st, ref_st)
    np.testing.assert_array_equal(np.nan_to_num(gre, nan=1.0), np.nan_to_num(ref_re, nan=1.0))
    np.testing.assert_array_equal(np.nan_to_num(gim, nan=1.0), np.nan_to_num(ref_im, nan=1.0))
    assert not any(c for _, c in fk_batches.run(fk, w.params, jre, str(tmp_path), 16))


def test_plain_form_against_regression_vectors(small):
    """The parity form against the committed oracle vectors (frequencies 8 and 30):
    the same bar as against the live oracle, 1e-10 of each spectrum's largest value."""
    import os
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_fk_global_small.npz"))
    w, m, ex, jre, fk, o = small
    g = M.frequency_grid(w.params, m.rearth)
    for jf in (8, 30):
        _, _, g64, st = fk.run(w.params, jre, jf, jf, f32=False)
        ref = gold["jf%d" % jf]
        assert np.all(st == gold["status%d" % jf])
        assert g64.shape == ref.shape
        assert _cmp(g64, ref) <= 1e-10
