"""Single-force sources (istyp 0) on the GPU against the CPU oracle, in the
global (degree sums, harmonicDegreeSums.f90:110-171) and the regional
(wavenumber integrals, wavenumberIntegrals.f90:122-250) mode: the 5 force FK
spectra of the solver, the 7 force sums or integrals, the force displacement
(singleFrequencyDisplacement.f90:35-46), filters, rotation and inverse FFT.
Per-trace relative L2 bars as for moment tensors: 1e-7 for the FP64 form, the
seismogram bar 1e-5 for the mixed-precision form."""
import dataclasses

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
RTOL_TRACE = {1: 1e-7, 2: 1e-5}
FORCES = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.6, -0.3, 0.8]])


def _force_fk(name):
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS[name]
    m = w.model()
    ex = w.nodes(m)
    params = dataclasses.replace(w.params, source_type="FORCE")
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(params, m.rearth)
    assert M.nsp_for(params) == 5
    gre, gim, _, st = GeminiFK(m, ex).run(params, jre, g.nf1, g.nf2, f64=False)
    assert np.all(st == 0)
    src = ex.node_index(m.rearth - 10000.0)
    return w, m, ex, g, gre[src - 1], gim[src - 1]


@pytest.fixture(scope="module")
def global_force(gpu):
    return _force_fk("global_small")


@pytest.fixture(scope="module")
def regional_force(gpu):
    return _force_fk("regional_small")


def _trace_rel(got, ref, nsamp):
    scale = 1.0 / np.abs(ref).max()
    a = got.astype(np.float64).reshape(-1, nsamp) * scale
    b = ref.astype(np.float64).reshape(-1, nsamp) * scale
    num, den = np.linalg.norm(a - b, axis=1), np.linalg.norm(b, axis=1)
    # a trace that is zero by symmetry (transverse motion of a vertical force)
    # must come out zero on both sides
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


@pytest.mark.parametrize("mode", ["global", "regional"])
@pytest.mark.parametrize("backend", [1, 2])
def test_force_synthetics_match_oracle(global_force, regional_force, mode, backend):
    import oracle
    from gemini_unified_b200.fk import GeminiFK, synth_params
    w, m, ex, g, gr, gi = global_force if mode == "global" else regional_force
    glob = 1 if mode == "global" else 0
    theta, phi, propdir = w.stations()
    sp = synth_params(g, 5, w.nsamp, w.dt, w.filspecs, global_=glob, rearth=m.rearth, source_type="FORCE")
    got = GeminiFK(m, ex, backend=backend).synthetics(sp, g.nwn, gr, gi, theta, phi, propdir, FORCES)
    ref = oracle.synthetics_src("FORCE", glob, g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, sp.dwn, sp.rearth, gr,
                                gi, theta, phi, propdir, FORCES, w.filspecs, False, 0.0, w.nsamp, w.dt)
    assert got.shape == ref.shape == (len(theta), 4, 3, w.nsamp)
    assert np.all(np.isfinite(got))
    assert np.abs(ref).max() > 0
    rel = _trace_rel(got, ref, w.nsamp)
    print("%s backend %d: trace rel L2 max %.2e median %.2e" % (mode, backend, rel.max(), np.median(rel)))
    assert rel.max() <= RTOL_TRACE[backend]


def test_force_synthetics_reject_moment_spectra_count(global_force):
    from gemini_unified_b200.fk import GeminiFK, synth_params
    from gemini_unified_b200.model import GeminiError
    w, m, ex, g, gr, gi = global_force
    theta, phi, propdir = w.stations()
    sp = synth_params(g, 4, w.nsamp, w.dt, w.filspecs, source_type="FORCE")
    with pytest.raises(GeminiError, match="5 force spectra"):
        GeminiFK(m, ex).synthetics(sp, g.nwn, gr[:4], gi[:4], theta, phi, propdir, FORCES)
