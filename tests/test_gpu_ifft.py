"""GPU batched inverse FFT (transformFrequencyTime) against the CPU oracle.

The kernel runs the reference's radix-2 transform in FP64 with its twiddle
angles; the twiddles come from the device's sincos and the series are rounded
to float32, so traces must agree to 1e-7 relative L2 per series."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL_L2 = 1e-7

CASES = [
    # nf1, nf2, df, nsamp, dt: the global configuration's series, a decimated
    # series, the 8192-sample series of the batched configuration, a 512-sample
    # one, a 4096-sample one, an 8192-sample one with a band of 1496 bins, and
    # 4096 samples decimated by 2 from an 8192-point transform (the fast form's
    # table path for the output factors)
    (2, 52, 1.0 / 1024, 2048, 0.5),
    (3, 300, 1.0 / 1024, 256, 4.0),
    (2, 411, 1.0 / 2048, 8192, 0.25),
    (2, 200, 1.0 / 512, 512, 1.0),
    (2, 300, 1.0 / 1024, 4096, 0.25),
    (5, 1500, 1.0 / 2048, 8192, 0.25),
    (2, 3000, 1.0 / 2048, 4096, 0.5),
]


def _spectra(ntr, ld, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((ntr, ld)) + 1j * rng.standard_normal((ntr, ld))


@pytest.fixture(scope="module")
def ft(gpu):
    from gemini_unified_b200.fk import FrequencyTime
    return FrequencyTime()


@pytest.mark.parametrize("case", CASES)
def test_ifft_matches_oracle(ft, case):
    import oracle
    nf1, nf2, df, nsamp, dt = case
    sigma = 5 * df
    sp = _spectra(37, nf2 + 3, nf2)
    ref, level = oracle.freq_time(nf1, nf2, df, sigma, sp, nsamp, dt)
    got = ft.run(nf1, nf2, df, sigma, sp, nsamp, dt)
    assert (ft.warning is not None) == (level == 1)
    err = np.linalg.norm((got - ref).astype(np.float64), axis=1) / np.linalg.norm(ref.astype(np.float64), axis=1)
    assert err.max() <= RTOL_L2


def test_ifft_device_api_and_leading_dimension(ft):
    import torch
    import oracle
    nf1, nf2, df, nsamp, dt = CASES[0]
    sp = _spectra(5, 80, 3)
    ref, _ = oracle.freq_time(nf1, nf2, df, 0.0, sp, nsamp, dt)
    d_sp = torch.from_numpy(sp.view(np.float64).copy()).cuda()
    d_ts = torch.zeros((5, nsamp), dtype=torch.float32, device="cuda")
    ft.run_device(nf1, nf2, df, 0.0, 5, d_sp.data_ptr(), 80, nsamp, dt, d_ts.data_ptr())
    torch.cuda.synchronize()
    got = d_ts.cpu().numpy()
    err = np.linalg.norm((got - ref).astype(np.float64), axis=1) / np.linalg.norm(ref.astype(np.float64), axis=1)
    assert err.max() <= RTOL_L2


def test_ifft_rejects_invalid_sizes(ft):
    from gemini_unified_b200.model import GeminiError
    sp = _spectra(2, 60, 0)
    with pytest.raises(GeminiError):
        ft.run(2, 52, 1.0 / 1024, 0.0, sp, 2048, 0.3)       # nsamp*dt*df != 1
    with pytest.raises(GeminiError):
        ft.run(2, 52, 1.0 / 1024, 0.0, sp, 16384, 1.0 / 16)  # FFT length above 8192
    with pytest.raises(GeminiError):
        ft.run(2, 61, 1.0 / 1024, 0.0, sp, 2048, 0.5)       # nf2 beyond the leading dimension


def _exact(nf1, nf2, df, sigma, sp, nsamp, dt):
    """transformFrequencyTime with an exact inverse DFT (numpy, FP64)."""
    ns = max(nsamp, 2 ** (int(np.ceil(np.log2(np.float32(nf2)))) + 1))
    ndec = 1 if ns == nsamp else int(round(dt / (1.0 / (df * ns))))
    X = np.zeros((sp.shape[0], ns // 2 + 1), complex)
    X[:, nf1 - 1:nf2] = sp[:, nf1 - 1:nf2]
    x = np.fft.irfft(X, n=ns) * ns
    dts = dt / ndec
    return x[:, ::ndec][:, :nsamp] * df * np.exp(sigma * dts * np.arange(nsamp))


@pytest.mark.parametrize("case", CASES)
def test_fast_ifft_exact_and_reference(case):
    """Fast form (real output from a half-length complex transform): within
    float32 rounding of the exact inverse DFT, and within the 1e-5 seismogram
    bar of the reference's transform (whose twiddles use single-precision pi)."""
    import oracle
    from gemini_unified_b200.fk import FrequencyTime, GEM_BACKEND_GPU_FAST
    nf1, nf2, df, nsamp, dt = case
    sigma = 5 * df
    sp = _spectra(29, nf2 + 2, nf2 + 7)
    got = FrequencyTime(backend=GEM_BACKEND_GPU_FAST).run(nf1, nf2, df, sigma, sp, nsamp, dt).astype(np.float64)
    ex = _exact(nf1, nf2, df, sigma, sp, nsamp, dt)
    assert (np.linalg.norm(got - ex, axis=1) / np.linalg.norm(ex, axis=1)).max() <= RTOL_L2
    ref, _ = oracle.freq_time(nf1, nf2, df, sigma, sp, nsamp, dt)
    ref = ref.astype(np.float64)
    assert (np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)).max() <= 1e-5
