"""Self-consistency checks of the CPU oracle (no reference golden data exists
for the FK hot path: the reference's regression data refseis/ is not shipped)."""
import numpy as np
import pytest

import oracle
from gemini_unified_b200 import configs, model as M


def test_legendre_against_scipy():
    sp = pytest.importorskip("scipy.special")
    lmax = 60
    for theta in (0.3, 1.2, 2.9):
        t = oracle.legendre(lmax, theta)
        ls = np.arange(lmax + 1)
        x = np.cos(theta)
        for m in range(3):
            ref = sp.lpmv(m, ls, x) * (-1) ** m          # reference omits the Condon-Shortley sign
            got = t[0, m]
            mask = ls >= m
            assert np.allclose(got[mask], ref[mask], rtol=1e-10, atol=1e-12 * np.abs(ref[mask]).max())
        # dP/dtheta by central differences
        eps = 1e-6
        tp, tm = oracle.legendre(lmax, theta + eps), oracle.legendre(lmax, theta - eps)
        fd = (tp[0] - tm[0]) / (2 * eps)
        assert np.allclose(t[1], fd, rtol=1e-5, atol=1e-6 * np.abs(fd).max())
        # P/sin(theta) for m >= 1
        assert np.allclose(t[2, 1:, 1:], t[0, 1:, 1:] / np.sin(theta), rtol=1e-13)


def test_legendre_poles():
    t = oracle.legendre(10, 0.0)
    ls = np.arange(11)
    assert np.allclose(t[0, 0], 1.0)                         # P_l(1) = 1
    assert np.allclose(t[1, 1], 0.5 * ls * (ls + 1))         # legendreFunctions.f90:113


def test_fft_against_numpy():
    n = 8
    N = 1 << n
    rng = np.random.default_rng(1)
    x = rng.standard_normal(N); y = rng.standard_normal(N)
    ox, oy = oracle.fft(x, y, n, +1)
    ref = np.fft.ifft(x + 1j * y) * N                         # sum x_k exp(+2 pi i nk/N)
    got = ox + 1j * oy
    # twiddles use pi rounded to single precision (fourierTransform.f90:128)
    assert np.max(np.abs(got - ref)) < 1e-4 * np.max(np.abs(ref))
    dx, dy = oracle.fft(np.eye(1, N, 0)[0], np.zeros(N), n, +1)
    assert np.all(dx == 1.0) and np.all(dy == 0.0)


def _spectra(ntr, ld, nf1, nf2, seed):
    rng = np.random.default_rng(seed)
    sp = rng.standard_normal((ntr, ld)) + 1j * rng.standard_normal((ntr, ld))
    sp[:, :nf1 - 1] = 7.0    # outside nf1..nf2: must be ignored
    sp[:, nf2:] = -3.0
    return sp


def test_freq_time_against_numpy():
    """transformFrequencyTime: Hermitian completion of bins nf1..nf2, inverse
    DFT, times df * exp(sigma t); with and without decimation."""
    df = 1.0 / 1024
    sigma = 5 * df
    for nf1, nf2, nsamp, dt, ndec in ((2, 52, 2048, 0.5, 1), (3, 300, 256, 4.0, 4)):
        sp = _spectra(3, nf2 + 5, nf1, nf2, nf2)
        ts, level = oracle.freq_time(nf1, nf2, df, sigma, sp, nsamp, dt)
        ns = max(nsamp, 2 ** (int(np.ceil(np.log2(nf2))) + 1))
        X = np.zeros((3, ns), complex)
        X[:, nf1 - 1:nf2] = sp[:, nf1 - 1:nf2]
        full = np.fft.irfft(X[:, : ns // 2 + 1], n=ns) * ns    # Re of the Hermitian sum
        t = np.arange(nsamp) * (dt / ndec)                      # the reference's exp(sigma*dts) per output sample
        ref = full[:, ::ndec][:, :nsamp] * df * np.exp(sigma * t)
        err = np.linalg.norm(ts - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert err.max() < 1e-5                                 # twiddles use single-precision pi
        assert level == (1 if ndec > 1 else 0)


def test_freq_time_rejects_inconsistent_sampling():
    sp = _spectra(1, 60, 2, 52, 0)
    with pytest.raises(RuntimeError):
        oracle.freq_time(2, 52, 1.0 / 1024, 0.0, sp, 2048, 0.3)     # nsamp*dt*df != 1
    with pytest.raises(RuntimeError):
        oracle.freq_time(2, 52, 1.0 / 1024, 0.0, sp, 4096, 0.5)     # nsamp*dt beyond 1/df


def test_degree_sums_against_direct_formula():
    """harmonicDegreeSums.f90:231-351 evaluated independently in numpy."""
    rng = np.random.default_rng(7)
    nf1, nf2 = 2, 4
    nwn = np.array([0, 30, 41, 52], np.int32)
    nkf = int(nwn.sum())
    gr = rng.standard_normal((10, nkf)).astype(np.float32)
    gi = rng.standard_normal((10, nkf)).astype(np.float32)
    theta = np.array([0.4, 2.0])
    hd = oracle.degree_sums(nf1, nf2, nwn, 52, gr, gi, theta)
    PI_F = M.PI_F
    defs = [(0, 0, 0, 0.0, 0), (0, 0, 0, 0.0, 1), (0, 1, 1, 2.0, 2), (0, 2, 2, 2.0, 3), (1, 0, 1, 0.0, 4),
            (1, 0, 1, 0.0, 5), (1, 1, 1, 2.0, 6), (1, 2, 2, 2.0, 7), (2, 1, 1, 2.0, 8), (2, 2, 2, 4.0, 9),
            (1, 1, 1, 2.0, 8), (1, 2, 2, -2.0, 9), (2, 1, 1, 2.0, 6), (2, 2, 2, -4.0, 7)]
    for it, th in enumerate(theta):
        tab = oracle.legendre(51, th)
        off = 0
        for jf in range(nf1, nf2 + 1):
            n = int(nwn[jf - 1]); lmax = n - 1
            l = np.arange(n)
            jt = max(1, min(int(np.floor(lmax * 0.8 + 0.5)), lmax))
            c1 = lmax * 0.2 * 2.0 / PI_F; c2 = 0.8 / 0.2 * 0.5 * PI_F
            tap = np.where(l < jt, 1.0, np.cos(l / c1 - c2) ** 2)
            for k, (kind, m, l0, fac, col) in enumerate(defs):
                g = gr[col, off:off + n].astype(np.float64) + 1j * gi[col, off:off + n]
                T = tab[kind, m, :n]
                w = np.ones(n) if fac == 0.0 else fac / np.maximum(l * (l + 1), 1)
                terms = T * w * g * (2 * l + 1) / (4 * PI_F) * tap
                ref = terms[l0:].sum()
                assert abs(hd[it, jf - 1, k] - ref) <= 1e-12 * max(1.0, np.abs(terms).sum())
            off += n


@pytest.fixture(scope="module")
def small():
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    return w, m, ex, jre, oracle.Oracle(m, ex)


def test_fk_deterministic_and_status(small):
    w, m, ex, jre, o = small
    pc = M.fk_params_c(w.params, jre)
    g1, s1, st1 = o.fk_frequency(pc, 6, 71, 10)
    g2, s2, st2 = o.fk_frequency(pc, 6, 71, 10)
    assert np.array_equal(s1, np.zeros_like(s1))
    assert np.array_equal(np.nan_to_num(g1, nan=7.0), np.nan_to_num(g2, nan=7.0)) and st1 == st2
    # l = 0 V-components are NaN in the reference too: bgout(3,1) = -f*bgin(2,4)/elp1 with elp1 = 0
    assert np.all(np.isnan(g1[:, 4:8, 0])) and not np.any(np.isnan(g1[:, :4, :]))


def test_fk_accuracy_convergence(small):
    """Spectra at ACCURACY 1e-5 and 1e-7 agree to O(1e-5) (the integrator's own error)."""
    w, m, ex, jre, o = small
    import dataclasses
    p_lo = M.fk_params_c(w.params, jre)
    p_hi = M.fk_params_c(dataclasses.replace(w.params, eps=1e-7), jre)
    a, _, _ = o.fk_frequency(p_lo, 12, 161, 10, 2, 161)
    b, _, _ = o.fk_frequency(p_hi, 12, 161, 10, 2, 161)
    u, v = a[jre - 1, :, 1:], b[jre - 1, :, 1:]
    rel = np.linalg.norm(u - v) / np.linalg.norm(v)
    assert rel < 1e-3


def test_fk_fault_injection_min_step(small):
    """An unreachable accuracy makes every step fail down to the minimum step size
    (integrationStep.f90:176-180): status 1, no hang."""
    w, m, ex, jre, o = small
    import dataclasses
    pc = M.fk_params_c(dataclasses.replace(w.params, eps=1e-30), jre)
    g, st, _ = o.fk_frequency(pc, 3, 23, 10, 3, 5)
    assert np.all(st[2:5] == 1)


def test_proposer_mlp_gradient_against_finite_differences():
    """The FP64 restatement of the proposer network: its reverse-mode gradient
    agrees with central differences of its loss."""
    import proposer_mlp
    rng = np.random.default_rng(11)
    w = rng.normal(0, 0.3, proposer_mlp.NPARAM)
    x = rng.normal(0, 1, (40, proposer_mlp.NF))
    y = rng.normal(0, 1, (40, proposer_mlp.NO))
    mask = (rng.random((40, proposer_mlp.NO)) > 0.3).astype(float)
    _, g = proposer_mlp.loss_and_grad(w, x, y, mask)
    for i in rng.choice(proposer_mlp.NPARAM, 25, replace=False):
        e = np.zeros_like(w); e[i] = 1e-6
        fd = (proposer_mlp.loss_and_grad(w + e, x, y, mask)[0] - proposer_mlp.loss_and_grad(w - e, x, y, mask)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_wavenumber_integral_of_an_analytic_spectrum():
    """Trapezoid + Filon + Neumann end terms of momentWavenumberIntegrals on
    G(k) = exp(-a k): int k exp(-a k) J0(k x) dk = a / (a^2 + x^2)^(3/2).  The
    rule is second order in x dk: its error falls 4x when dk halves."""
    a, re = 20000.0, 6371000.0

    def rel_err(n, x):
        dwn = 40.0 / a / n
        gr = np.zeros((10, n), np.float32)
        gr[0] = np.exp(-a * np.arange(n) * dwn)
        hd = oracle.wavenumber_integrals(2, 2, np.array([0, n], np.int32), n, gr, np.zeros_like(gr), dwn, re, [x])
        got = hd[0, 1, 0].real / (re * re / (2 * np.float32(np.pi)))
        return got / (a / (a * a + x * x) ** 1.5) - 1.0, x * dwn

    for x in (5000.0, 50000.0, 200000.0):
        e1, xdk = rel_err(8000, x)
        e2, _ = rel_err(16000, x)
        assert abs(e1) < 2.0 * xdk * xdk
        if abs(e1) > 1e-5:
            assert 3.5 < e1 / e2 < 4.5


def test_bessel_functions_of_the_oracle_against_scipy():
    sp = pytest.importorskip("scipy.special")
    # the oracle's integral of a single wavenumber sample isolates J at that point
    n, dwn, x, re = 64, 1e-5, 123456.0, 6371000.0
    for j in (5, 20, 40):
        gr = np.zeros((10, n), np.float32); gi = np.zeros_like(gr)
        gr[:, j - 1] = 1.0
        hd = oracle.wavenumber_integrals(2, 2, np.array([0, n], np.int32), n, gr, gi, dwn, re, [x])
        k = (j - 1) * dwn
        taper_w = hd[0, 1, 0].real / (re * re / (2 * np.float32(np.pi))) / (k * sp.j0(k * x))
        # integral 1 (k J0) and integral 3 (2/re J1) share the sample's weight
        ratio = hd[0, 1, 2].real / hd[0, 1, 0].real
        assert abs(ratio - (2.0 / re * sp.j1(k * x)) / (k * sp.j0(k * x))) < 1e-9 * abs(ratio) + 1e-12
        assert np.isfinite(taper_w)


# Each force sum or integral uses a table kind and an FK spectrum that one
# moment sum also uses, with the factor 2/l(l+1) or its negative
# (harmonicDegreeSums.f90:110-171 against :297-351, wavenumberIntegrals.f90:160-168
# against :259-274): with the moment spectra filled from the force spectra
# (moment column 0, 2, 4, 6, 8 <- force column 0..4) force sum k equals
# sign x moment sum MATE[k].
FORCE_MATE = [(0, 1.0), (2, -1.0), (4, 1.0), (6, -1.0), (8, -1.0), (10, 1.0), (12, 1.0)]


def _force_and_moment_slabs(nwn, seed):
    rng = np.random.default_rng(seed)
    nkf = int(nwn.sum())
    fr = rng.standard_normal((5, nkf)).astype(np.float32)
    fi = rng.standard_normal((5, nkf)).astype(np.float32)
    mr = np.zeros((10, nkf), np.float32); mi = np.zeros_like(mr)
    mr[0::2] = fr; mi[0::2] = fi
    return fr, fi, mr, mi


def test_force_degree_sums_against_moment_sums():
    nwn = np.array([0, 40, 48, 56, 64], np.int32)
    fr, fi, mr, mi = _force_and_moment_slabs(nwn, 5)
    theta = [0.05, 0.7, 2.9]
    f = oracle.force_degree_sums(2, 5, nwn, 64, fr, fi, theta)
    m = oracle.degree_sums(2, 5, nwn, 64, mr, mi, theta)
    for k, (km, sg) in enumerate(FORCE_MATE):
        a, b = f[:, 1:, k], sg * m[:, 1:, km]   # the two loops round in their own order
        assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


def test_force_wavenumber_integrals_against_moment_integrals():
    nwn = np.array([0, 400, 480, 560, 640], np.int32)
    fr, fi, mr, mi = _force_and_moment_slabs(nwn, 6)
    x = [3000.0, 40000.0, 250000.0]   # trapezoid only, both rules, mostly Filon
    f = oracle.force_wavenumber_integrals(2, 5, nwn, 640, fr, fi, 2e-6, 6371000.0, x)
    m = oracle.wavenumber_integrals(2, 5, nwn, 640, mr, mi, 2e-6, 6371000.0, x)
    for k, (km, sg) in enumerate(FORCE_MATE):
        a, b = f[:, 1:, k], sg * m[:, 1:, km]
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_force_synthetics_are_linear_in_the_force():
    """Traces of (Fr, Ft, Ff) equal the sum of the traces of its components
    (singleFrequencyDisplacement.f90:35-46 is linear), in both modes."""
    nwn = np.array([0, 60, 64, 64, 64, 64, 64, 64], np.int32)
    fr, fi, _, _ = _force_and_moment_slabs(nwn, 7)
    theta, phi, propdir = [0.02, 0.4], [0.3, 2.0], [0.1, -0.7]
    F = np.array([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0], [0.5, -2.0, 1.5]])
    for glob in (1, 0):
        tr = oracle.synthetics_src("FORCE", glob, 2, 8, nwn, 64, 1.0 / 256, 0.002, 2e-5, 6371000.0, fr, fi, theta, phi,
                                   propdir, F, [2, 0.005, 4, 0.06], 0, 0.0, 256, 1.0).astype(np.float64)
        comb = 0.5 * tr[:, 0] - 2.0 * tr[:, 1] + 1.5 * tr[:, 2]
        assert np.abs(tr).max() > 0
        assert np.abs(tr[:, 3] - comb).max() <= 1e-5 * np.abs(comb).max()


def _station_case():
    nwn = np.array([0, 60, 64, 64, 64, 64, 64, 64], np.int32)
    rng = np.random.default_rng(11)
    gr = rng.standard_normal((10, int(nwn.sum()))).astype(np.float32)
    gi = rng.standard_normal((10, int(nwn.sum()))).astype(np.float32)
    mt = np.array([[1.0, -0.5, -0.5, 0.3, -0.2, 0.7]])
    args = dict(nf1=2, nf2=8, nwn=nwn, nwnmax=64, df=1.0 / 256, sigma=0.002, dwn=2e-5, rearth=6371000.0, gr=gr, gi=gi,
                theta=[0.02, 0.4, 1.3], phi=[0.3, 2.0, 4.0], propdir=[0.1, -0.7, 2.5], src=mt,
                filspecs=[2, 0.005, 4, 0.06], velocity=0, nsamp=256, dt=1.0)
    return args


def test_station_options_default_to_the_plain_station_loop():
    a = _station_case()
    ref = oracle.synthetics_src("MOMENT", 1, tred=5.0, **a)
    got = oracle.synthetics_opts("MOMENT", 1, tred=0.0, tred_sta=[5.0, 5.0, 5.0], nstrue=[256] * 3,
                                 stafilter=np.ones((3, 3, 8), np.complex128), **a)
    np.testing.assert_array_equal(got, ref)


def test_station_filter_scales_and_samples_are_cut():
    a = _station_case()
    ref = oracle.synthetics_src("MOMENT", 1, tred=0.0, **a).astype(np.float64)
    sf = np.ones((3, 3, 8), np.complex128)
    sf[1, 2, :] = 2.0   # station 1, third component (before rotation) doubled
    got = oracle.synthetics_opts("MOMENT", 1, tred=0.0, stafilter=sf, nstrue=[256, 200, 100], **a).astype(np.float64)
    np.testing.assert_array_equal(got[0], ref[0])
    assert np.all(got[1, :, :, 200:] == 0) and np.all(got[2, :, :, 100:] == 0)
    np.testing.assert_array_equal(got[2, :, :, :100], ref[2, :, :, :100])
    # the transverse component before rotation is doubled: Z is unchanged, N and E change
    np.testing.assert_array_equal(got[1, :, 0, :200], ref[1, :, 0, :200])
    assert np.abs(got[1, :, 1:, :200] - ref[1, :, 1:, :200]).max() > 0


def test_source_wavelet_convolution_against_a_direct_loop():
    """convolveWithSourceWavelet as written in the reference: f(k) = sum over the wavelet
    of dt * u(k - n + nhm + 1) * stf(n), nhm samples of it before t = 0, rounded to
    single precision after every term."""
    a = _station_case()
    stf = np.array([0.1, 0.5, 1.0, 0.4, -0.2, 0.05], np.float32)
    tanf = -2.0
    plain = oracle.synthetics_opts("MOMENT", 1, tred=0.0, nstrue=[256, 180, 256], **a)
    got = oracle.synthetics_opts("MOMENT", 1, tred=0.0, nstrue=[256, 180, 256], stf=stf, tanf_stf=tanf, **a)
    nhm = int(np.floor(abs(tanf) / a["dt"] + 0.5))
    for s, nd in ((0, 256), (1, 180)):
        for c in range(3):
            u = plain[s, 0, c]
            for k in (1, 2, 3, 50, nd - 2, nd):
                acc = np.float32(0.0)
                for n in range(max(1, k - nd + nhm + 1), min(k + nhm, len(stf)) + 1):
                    j = n - nhm
                    acc = np.float32(float(acc) + (a["dt"] * float(u[k - j])) * float(stf[n - 1]))
                assert got[s, 0, c, k - 1] == acc


def test_ray_table_slowness_is_the_travel_time_slope():
    """Along the surface node, T(p) and Delta(p) of the rays obey dT/dDelta = p
    (computeTravelTimeTable's table; the ray parameter is the slope of the
    travel-time curve)."""
    m = configs.WORKLOADS["batched_fk"].model()
    ex = configs.WORKLOADS["batched_fk"].nodes(m)
    o = oracle.Oracle(m, ex)
    rc, rtp, slow, tab, st = o.ray_table("P", 3, 1e-6, 20000.0, float(ex.r[-1]), 400, ex.nnod)
    assert rc == 0 and np.all(st == 0) and len(rtp) == int(int(ex.r[-1] - m.roc) / 20000.0 + 1)
    # lower-mantle turning points (the upper mantle's discontinuities fold the curve)
    low = rtp <= 5600000.0
    d = tab[low, -1, 0].astype(np.float64); t = tab[low, -1, 1].astype(np.float64)
    assert np.all(np.diff(d) < 0) and np.all(np.diff(t) < 0)   # deeper turning points go farther
    slope = np.diff(t) / np.diff(d)
    pm = 0.5 * (slow[low][1:] + slow[low][:-1])
    assert np.abs(slope / pm - 1.0).max() < 2e-3
    # the deepest ray grazes the core-mantle boundary near 98 degrees (two legs)
    assert 95.0 < 2 * np.degrees(d[0]) < 101.0


def test_oracle_reproduces_its_regression_vectors():
    """The committed oracle FK spectra of frequencies 8 and 30 of the global
    configuration (tests/golden/make_fixtures.py --oracle): bit for bit."""
    import os
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_fk_global_small.npz"))
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    o = oracle.Oracle(m, ex)
    pc = M.fk_params_c(w.params, jre)
    for jf in (8, 30):
        spec, status, _ = o.fk_frequency(pc, jf, int(g.nwn[jf - 1]), M.nsp_for(w.params))
        np.testing.assert_array_equal(status, gold["status%d" % jf])
        np.testing.assert_array_equal(np.nan_to_num(spec, nan=1.0), np.nan_to_num(gold["jf%d" % jf], nan=1.0))
