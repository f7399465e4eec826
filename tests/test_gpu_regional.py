"""Regional (flat-earth, Bessel) mode on the GPU against the CPU oracle.

FK spectra: the FP64 solver in the reference's operation order, 1e-10 relative
to each spectrum's largest value, as in the global mode.  Synthetics: the
wavenumber integrals (trapezoid below kx = 3, Filon above, Neumann end terms;
wavenumberIntegrals.f90:320-475) run as the degree sums do; the Bessel and
Neumann functions come from CUDA's j0/j1/y0/y1 on the GPU and the C library in
the oracle, so the FP64 form's traces must agree to 1e-7 relative L2 per trace.
The mixed-precision form (sliced-integer tensor-core sums, radix-16 FFT with
exact twiddles where the reference's use single-precision pi) is held to the
seismogram bar, 1e-5 per trace."""
import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
RTOL = 1e-10
RTOL_TRACE = {1: 1e-7, 2: 1e-5}


@pytest.fixture(scope="module")
def regional(gpu):
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["regional_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    fk = GeminiFK(m, ex)
    gre, gim, g64, st = fk.run(w.params, jre, g.nf1, g.nf2)
    assert np.all(st == 0)
    return w, m, ex, jre, g, gre, gim, g64


def test_regional_fk_spectra_match_oracle(regional):
    import oracle
    w, m, ex, jre, g, gre, gim, g64 = regional
    o = oracle.Oracle(m, ex)
    pc = M.fk_params_c(w.params, jre)
    koff = np.concatenate([[0], np.cumsum(g.nwn[g.nf1 - 1: g.nf2])])
    for jf in (g.nf1, 40, g.nf2):
        n = int(g.nwn[jf - 1])
        for iwn in (2, 3, n // 3, n // 2 + 1, n):
            ref, sto, _ = o.fk_frequency(pc, jf, n, 10, iwn, iwn)
            assert sto[iwn - 1] == 0
            a = g64[:, :, koff[jf - g.nf1] + iwn - 1]
            b = ref[:, :, iwn - 1]
            assert np.abs(a - b).max() <= RTOL * np.abs(b).max()
    # wn = 0 (iwn = 1) is not computed in the regional mode and stays zero
    assert np.all(g64[:, :, 0] == 0)


@pytest.mark.parametrize("backend", [1, 2])
def test_regional_synthetics_match_oracle(regional, backend):
    import oracle
    from gemini_unified_b200.fk import GeminiFK, synth_params
    w, m, ex, jre, g, gre, gim, g64 = regional
    src = ex.node_index(m.rearth - 10000.0)
    theta, phi, propdir = w.stations()
    mt = configs.unit_moment_tensors()
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs, global_=0, rearth=m.rearth)
    got = GeminiFK(m, ex, backend=backend).synthetics(sp, g.nwn, gre[src - 1], gim[src - 1], theta, phi, propdir, mt)
    ref = oracle.synthetics_bessel(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, sp.dwn, sp.rearth, gre[src - 1],
                                   gim[src - 1], theta, phi, propdir, mt, w.filspecs, False, 0.0, w.nsamp, w.dt)
    assert got.shape == ref.shape == (20, 6, 3, w.nsamp)
    assert np.all(np.isfinite(got))
    scale = 1.0 / np.abs(ref).max()
    a = got.astype(np.float64).reshape(-1, w.nsamp) * scale
    b = ref.astype(np.float64).reshape(-1, w.nsamp) * scale
    rel = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    print("backend %d: trace rel L2 max %.2e median %.2e" % (backend, rel.max(), np.median(rel)))
    assert rel.max() <= RTOL_TRACE[backend]
