"""GPU synthetics (degree sums, filters, rotation, inverse FFT) against the
CPU oracle on the same float32 FK spectra.  The FP64 sums run as tiled
matrix products, so the summation order differs from the reference's loop,
and the traces are float32 (one rounding flip is 6e-8 relative): traces must
agree to 1e-7 relative L2 per trace (the seismogram bar is 1e-5)."""
import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu


def _rel(got, ref, nsamp):
    """Per-trace L2 error and norm in float64 (the traces are ~1e-20 m: float32 squares underflow)."""
    scale = 1.0 / np.abs(ref).max()
    g = got.astype(np.float64).reshape(-1, nsamp) * scale
    r = ref.astype(np.float64).reshape(-1, nsamp) * scale
    return np.linalg.norm(g - r, axis=1), np.linalg.norm(r, axis=1)


@pytest.fixture(scope="module")
def fkdata(gpu):
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    fk = GeminiFK(m, ex)
    gre, gim, _, st = fk.run(w.params, jre, g.nf1, g.nf2, f64=False)
    src = ex.node_index(m.rearth - 10000.0)    # source at 10 km depth
    return w, m, ex, g, fk, gre[src - 1], gim[src - 1]


def test_synthetics_match_oracle(fkdata):
    import oracle
    from gemini_unified_b200.fk import synth_params
    w, m, ex, g, fk, gr, gi = fkdata
    theta, phi, propdir = w.stations()
    mt = configs.unit_moment_tensors()
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    got = fk.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    ref = oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta, phi, propdir, mt,
                            w.filspecs, False, 0.0, w.nsamp, w.dt)
    assert got.shape == ref.shape == (50, 6, 3, 2048)
    assert np.all(np.isfinite(got))
    num, den = _rel(got, ref, w.nsamp)
    assert np.all(den > 0)
    assert np.max(num / den) <= 1e-7


def test_synthetics_velocity_and_shift(fkdata):
    import oracle
    from gemini_unified_b200.fk import synth_params
    w, m, ex, g, fk, gr, gi = fkdata
    theta, phi, propdir = w.stations()
    theta, phi, propdir = theta[::10], phi[::10] + 0.3, propdir[::10] + 0.1
    mt = np.array([[1.0, -0.5, -0.5, 0.3, -0.2, 0.7]])
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs, velocity=True, tred=20.0)
    got = fk.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    ref = oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta, phi, propdir, mt,
                            w.filspecs, True, 20.0, w.nsamp, w.dt)
    num, den = _rel(got, ref, w.nsamp)
    assert np.all(den > 0)
    assert np.max(num / den) <= 1e-7


# The mixed-precision form (fast backend) computes the degree sums on the
# tensor cores from 7-bit integer slices of both operands with exact INT32
# accumulation, and its inverse FFT uses exact twiddles; its seismograms must
# agree with the FP64 form to 1e-5 relative L2 per trace.
RTOL_MIXED = 1e-5


def test_mixed_precision_synthetics_against_fp64(fkdata):
    import oracle
    from gemini_unified_b200.fk import FrequencyTime, GEM_BACKEND_GPU_FAST, GeminiFK, synth_params
    w, m, ex, g, fk, gr, gi = fkdata
    theta, phi, propdir = w.stations()
    mt = configs.unit_moment_tensors()
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    fast = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    got = fast.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    ref = oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta, phi, propdir, mt,
                            w.filspecs, False, 0.0, w.nsamp, w.dt)
    assert np.all(np.isfinite(got))
    num, den = _rel(got, ref, w.nsamp)
    assert np.max(num / den) <= RTOL_MIXED


def test_mixed_precision_synthetics_many_stations(gpu):
    """Seeded log-normal FK coefficients of the batched configuration's shape
    (10 spectra x 658,944 wavenumber-frequency samples, l <= 3205) at 600
    stations: several tiles in every dimension of the tensor-core products."""
    from gemini_unified_b200.fk import GEM_BACKEND_GPU_FAST, GEM_BACKEND_GPU_FP64, GeminiFK, synth_params
    from gemini_unified_b200.synth_run import fk_coefficients
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    g = M.frequency_grid(w.params, m.rearth)
    gr, gi = fk_coefficients(10, int(g.nkfmax))
    theta, phi, propdir = w.stations()
    sel = slice(0, 4000, 7)   # 572 stations over 0.5..179.5 deg
    theta, phi, propdir = theta[sel], phi[sel], propdir[sel]
    mt = configs.unit_moment_tensors()[[0, 3, 5]]
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    ref = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FP64).synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    got = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST).synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    assert np.all(np.isfinite(got))
    num, den = _rel(got, ref, w.nsamp)
    assert np.max(num / den) <= RTOL_MIXED


def test_tensor_core_wait_limit_reports_error(fkdata):
    """Failure detection of the tensor-core sums, without a GPU fault: with a
    pipeline wait limit of 1 ns the first wait of a tile that is not complete
    already runs out, the kernel drains its own copies and products, frees its
    tensor memory and returns, and the call fails with GEM_ERROR.  The context
    stays usable: with the default limit restored the same call matches the
    oracle."""
    import oracle
    from gemini_unified_b200.fk import GEM_BACKEND_GPU_FAST, GeminiError, GeminiFK, synth_params
    w, m, ex, g, fk, gr, gi = fkdata
    theta, phi, propdir = w.stations()
    theta, phi, propdir = theta[::10], phi[::10], propdir[::10]
    mt = configs.unit_moment_tensors()[:2]
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    fast = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    fast.tc_wait_limit(1)
    with pytest.raises(GeminiError, match="timed out"):
        fast.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    fast.tc_wait_limit(0)
    got = fast.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    ref = oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta, phi, propdir, mt,
                            w.filspecs, False, 0.0, w.nsamp, w.dt)
    num, den = _rel(got, ref, w.nsamp)
    assert np.max(num / den) <= RTOL_MIXED


@pytest.mark.parametrize("backend", [1, 2])
def test_station_options_match_oracle(fkdata, backend):
    """Per-station reduction times (as AUTOMATIC_TIMESHIFT sets them), samples kept per
    station, station filters and a source wavelet (computeSyntheticSeismograms.f90:344-397,
    463-484) against the oracle's station loop."""
    import oracle
    from gemini_unified_b200.fk import GeminiFK, synth_params
    w, m, ex, g, fk, gr, gi = fkdata
    theta, phi, propdir = w.stations()
    theta, phi, propdir = theta[::5], phi[::5] + 0.4, propdir[::5] - 0.2
    nsta = len(theta)
    rng = np.random.default_rng(7)
    mt = configs.unit_moment_tensors()[[0, 3, 5]]
    tred = 30.0 + 4.0 * np.arange(nsta)
    nstrue = np.full(nsta, w.nsamp, np.int32); nstrue[::3] = w.nsamp - 500
    sf = (1.0 + 0.2 * rng.standard_normal((nsta, 3, g.nf2))) * np.exp(1j * 0.3 * rng.standard_normal((nsta, 3, g.nf2)))
    tt = np.arange(40) * w.dt
    stf = (np.exp(-((tt - 8.0) / 3.0) ** 2)).astype(np.float32)
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    got = GeminiFK(m, ex, backend=backend).synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt, tred=tred,
                                                       nsamp_true=nstrue, stafilter=sf, stf=stf, tanf_stf=-4.0)
    ref = oracle.synthetics_opts("MOMENT", 1, g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, 0.0, m.rearth, gr, gi,
                                 theta, phi, propdir, mt, w.filspecs, False, 0.0, w.nsamp, w.dt, tred_sta=tred,
                                 nstrue=nstrue, stafilter=sf, stf=stf, tanf_stf=-4.0)
    assert np.all(np.isfinite(got))
    for s in range(0, nsta, 3):
        assert np.all(got[s, :, :, nstrue[s]:] == 0)
    num, den = _rel(got, ref, w.nsamp)
    assert np.all(den > 0)
    assert np.max(num / den) <= (1e-7 if backend == 1 else RTOL_MIXED)


@pytest.mark.parametrize("backend", [1, 2])
def test_pinned_output_overlaps_station_groups(gpu, backend):
    """Into pinned host memory the host entry point computes the stations in groups
    and copies each group's traces while the next one runs.  The FP64 form gives the
    single-pass traces bit for bit (every station's sums and transforms are its own);
    the mixed form's degree scales span the stations of a call, so it agrees to its
    seismogram bar."""
    import ctypes
    import torch
    from gemini_unified_b200.fk import GeminiFK, lib, synth_params, _ptr
    from gemini_unified_b200.synth_run import fk_coefficients
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    g = M.frequency_grid(w.params, m.rearth)
    gr, gi = fk_coefficients(10, int(g.nkfmax))
    theta, phi, propdir = w.stations()
    sel = slice(0, 4000, 3)   # 1334 stations: four groups
    theta, phi, propdir = (np.ascontiguousarray(a[sel]) for a in (theta, phi, propdir))
    mt = np.ascontiguousarray(configs.unit_moment_tensors()[[0, 4]], np.float64)
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    fk = GeminiFK(m, ex, backend=backend)
    ref = fk.synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, mt)
    out = torch.zeros(ref.shape, dtype=torch.float32, pin_memory=True).numpy()
    nwn = np.ascontiguousarray(g.nwn, np.int32)
    for _ in range(2):
        out[:] = 0
        fk._check(lib().gem_synth_run(fk._h, ctypes.byref(sp), _ptr(nwn), _ptr(gr), _ptr(gi), len(theta), _ptr(theta),
                                      _ptr(phi), _ptr(propdir), len(mt), _ptr(mt), _ptr(out)))
        if backend == 1:
            np.testing.assert_array_equal(out, ref)
        else:
            num, den = _rel(out, ref, w.nsamp)
            assert np.max(num / den) <= RTOL_MIXED
