"""GPU parity of the DSV spectra with radial derivatives (the FK spectra of
computeGreenFKSpectraForASKI.f90) against the CPU oracle, through the C ABI
(gem_fk_run_dsv per source node, gem_fk_run_aski for a set of them).

Tolerances as for the synthetics FK spectra: the FP64 build agrees with the
oracle to 1e-10 relative to the largest value of the compared spectra, the
fast build to 1e-8.  gem_fk_run_dsv integrates the minors for one source
node, gem_fk_run_aski once over the node range as the reference does; the two
agree to round-off."""
import dataclasses

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
RTOL = 1e-10
RTOL_FAST = 1e-8
JF1, JF2 = 28, 31


def _rel(a, b):
    assert np.all(np.isfinite(a)) and np.all(np.isfinite(b))
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def aski(gpu):
    import oracle
    from gemini_unified_b200.fk import GeminiFK
    w = dataclasses.replace(configs.GLOBAL_SMALL, nnod_blocks=[4], dr_blocks=[10000.0])
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    return w, m, ex, jre, g, GeminiFK(m, ex), oracle.Oracle(m, ex)


def _oracle_single(o, w, g, src, force):
    """Oracle spectra of one source node over JF1..JF2, as (nnod, nsp, nkf)."""
    blocks = []
    for jf in range(JF1, JF2 + 1):
        out, st, _ = o.dsv_frequency(M.fk_params_c(w.params, src), [src], jf, int(g.nwn[jf - 1]))
        assert np.all(st == 0)
        blocks.append(out[1] if force else out[0])
    return np.concatenate(blocks, axis=2)


@pytest.mark.parametrize("src", [1, 5, 8, 11])
def test_dsv_moment_and_force_match_oracle(aski, src):
    """Moment source at an interior, the deepest and the surface node, and the
    force at the same node: every degree of four frequencies, 20 and 10 spectra
    per node at all 11 nodes."""
    w, m, ex, jre, g, fk, o = aski
    for force in (False, True):
        p = dataclasses.replace(w.params, source_type="FORCE") if force else w.params
        gre, gim, g64, st = fk.run_dsv(p, src, JF1, JF2)
        assert np.all(st == 0)
        assert g64.shape[1] == (10 if force else 20)
        ref = _oracle_single(o, w, g, src, force)
        assert _rel(g64, ref) <= RTOL, (src, force)
        assert np.array_equal(gre, g64.real.astype(np.float32))
        assert np.array_equal(gim, g64.imag.astype(np.float32))


def test_aski_spectra_match_the_reference_node_range_run(aski):
    """aski_spectra (one set run: minors over the node range, then every source
    node and the force at the receiver) against the oracle's restatement of
    the program's loop."""
    w, m, ex, jre, g, fk, o = aski
    srcs = [1, 5, 8, jre]
    jf = 40
    res = fk.aski_spectra(w.params, srcs, jre, jf, jf, f32=False)
    ref, st, _ = o.dsv_frequency(M.fk_params_c(w.params, jre), srcs, jf, int(g.nwn[jf - 1]))
    assert np.all(st == 0) and len(res) == len(ref) == len(srcs) + 1
    for (_, _, a, sa), b in zip(res, ref):
        assert np.all(sa == 0)
        assert _rel(a, b) <= RTOL


@pytest.mark.parametrize("source_type", ["MOMENT", "FORCE"])
def test_aski_set_run_equals_per_node_runs(aski, source_type):
    """One set run (minors once over the node range 1..11) against one
    gem_fk_run_dsv per source node: equal to round-off (the minors' final
    normalisation differs between the two ranges)."""
    w, m, ex, jre, g, fk, o = aski
    p = dataclasses.replace(w.params, source_type=source_type)
    srcs = [1, 3, 6, 9, jre]
    res = fk.aski_spectra(p, srcs, jre, JF1, JF2, f32=False)
    force = dataclasses.replace(w.params, source_type="FORCE")
    for (_, _, a, sa), (s, q) in zip(res, [(s, p) for s in srcs] + [(jre, force)]):
        assert np.all(sa == 0)
        _, _, b, sb = fk.run_dsv(q, s, JF1, JF2, f32=False)
        assert a.shape == b.shape
        assert _rel(a, b) <= 1e-12, s


def test_dsv_fast_backend(aski):
    from gemini_unified_b200.fk import GeminiFK, GEM_BACKEND_GPU_FAST
    w, m, ex, jre, g, fk, o = aski
    fast = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    for src in (1, jre):
        _, _, a, sa = fast.run_dsv(w.params, src, JF1, JF2, f32=False)
        _, _, b, sb = fk.run_dsv(w.params, src, JF1, JF2, f32=False)
        assert np.all(sa == 0) and np.all(sb == 0)
        assert _rel(a, b) <= RTOL_FAST
    for (_, _, a, sa), (_, _, b, sb) in zip(fast.aski_spectra(w.params, [1, 6, jre], jre, JF1, JF2, f32=False),
                                            fk.aski_spectra(w.params, [1, 6, jre], jre, JF1, JF2, f32=False)):
        assert np.all(sa == 0) and np.all(sb == 0)
        assert _rel(a, b) <= RTOL_FAST


def test_synthetics_spectra_unchanged_after_a_dsv_run(aski):
    """The DSV mode lasts one call: the next plain run on the context gives the
    synthetics program's spectra again."""
    w, m, ex, jre, g, fk, o = aski
    jf = 20
    n = int(g.nwn[jf - 1])
    fk.run_dsv(w.params, 5, jf, jf)
    fk.aski_spectra(w.params, [2, 7, jre], jre, jf, jf)
    _, _, got, st = fk.run(w.params, jre, jf, jf, f32=False)
    ref, sto, _ = o.fk_frequency(M.fk_params_c(w.params, jre), jf, n, M.nsp_for(w.params))
    assert np.all(st == 0) and got.shape == ref.shape
    ok = ~np.isnan(ref)
    assert np.array_equal(np.isnan(got), ~ok)
    assert np.abs(got[ok] - ref[ok]).max() <= RTOL * np.abs(ref[ok]).max()


def test_dsv_rejects_fluid_nodes_and_bad_source_sets(aski):
    from gemini_unified_b200.fk import GeminiFK
    from gemini_unified_b200.model import ExternalRadialNodes, GeminiError
    w, m, ex, jre, g, fk, o = aski
    with pytest.raises(GeminiError):
        fk.aski_spectra(w.params, [1, 5], jre, 10, 10)              # receiver not among the sources
    with pytest.raises(GeminiError):
        fk.aski_spectra(w.params, [1, jre], jre, 1, 1)              # below the first frequency
    core = ExternalRadialNodes.split(m, np.array([3.0e6, 6.331e6, 6.371e6]), m.rearth)
    assert 1 in list(core.state)
    fkc = GeminiFK(m, core)
    top = core.node_index(w.rec_radius)
    with pytest.raises(GeminiError, match="fluid"):
        fkc.run_dsv(w.params, top, 10, 10)


def test_dsv_regional_mode_matches_oracle(gpu):
    """Regional (wavenumber) mode on the 8-layer crust: a moment source at an
    interior node and the force at the receiver, against the oracle's loop over
    the node range."""
    import oracle
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["regional_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    jf = 40
    srcs = [3, 12, jre]
    res = GeminiFK(m, ex).aski_spectra(w.params, srcs, jre, jf, jf, f32=False)
    ref, st, _ = oracle.Oracle(m, ex).dsv_frequency(M.fk_params_c(w.params, jre), srcs, jf, int(g.nwn[jf - 1]))
    assert np.all(st == 0)
    for (_, _, a, sa), b in zip(res, ref):
        assert np.all(sa == 0)
        assert np.all(a[:, :, 0] == 0)          # wavenumber 0 stays zero in the regional mode
        assert _rel(a, b) <= RTOL
