"""CPU checks of the oracle's DSV spectra with radial derivatives, the FK
spectra of computeGreenFKSpectraForASKI.f90 (source-node loop :451-541,
derivatives dsvDerivatives.f90:39-72).

The reference's tests hold no vectors for this program, so the restatement is
pinned by three properties:
* reciprocity -- the field at the receiver node of a source at node n equals
  the synthetics program's spectrum of a source at n seen at the receiver
  (reciprocity.f90), to the integration accuracy;
* the radial derivatives agree with finite differences of the field between
  two nodes of one layer to the O(h^2) error of the difference;
* the program's single minors integration over the node range gives the same
  spectra as one run per source node to round-off (the GPU path runs one per
  source node).
"""
import dataclasses

import numpy as np
import pytest

import oracle
from gemini_unified_b200 import configs, model as M

JF = 30          # 0.0283 Hz
IWN_HI = 120     # degrees 0..119 keep each oracle call to a fraction of a second


@pytest.fixture(scope="module")
def aski():
    w = dataclasses.replace(configs.GLOBAL_SMALL, nnod_blocks=[4], dr_blocks=[10000.0])
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    o = oracle.Oracle(m, ex)
    g = M.frequency_grid(w.params, m.rearth)
    return w, m, ex, jre, o, int(g.nwn[JF - 1])


def test_dsv_layout_and_status(aski):
    w, m, ex, jre, o, n = aski
    out, st, _ = o.dsv_frequency(M.fk_params_c(w.params, jre), [1, jre], JF, n, 1, IWN_HI)
    assert np.all(st == 0)
    assert [a.shape for a in out] == [(ex.nnod, 20, n), (ex.nnod, 20, n), (ex.nnod, 10, n)]
    for a in out:
        assert np.all(np.isfinite(a))
        assert np.all(a[..., IWN_HI:] == 0)          # degrees outside the requested range stay zero
        assert np.abs(a[..., 1:IWN_HI]).max() > 0


def test_dsv_rejects_a_receiver_outside_the_source_nodes(aski):
    w, m, ex, jre, o, n = aski
    with pytest.raises(RuntimeError):
        o.dsv_frequency(M.fk_params_c(w.params, jre), [1, 2], JF, n, 1, 4)


def test_dsv_spectra_obey_reciprocity(aski):
    """U, V and W at the receiver of a moment source at node s against the
    synthetics program's spectra of a source at s (degree 0 excluded: its V
    spectra are NaN there)."""
    w, m, ex, jre, o, n = aski
    pc = M.fk_params_c(w.params, jre)
    srcs = [1, 2, 5, 8, 10]
    out, st, _ = o.dsv_frequency(pc, srcs + [jre], JF, n, 1, IWN_HI)
    syn, sts, _ = o.fk_frequency(pc, JF, n, M.nsp_for(w.params), 1, IWN_HI)
    assert np.all(st == 0) and np.all(sts == 0)
    for i, s in enumerate(srcs):
        a = out[i][jre - 1][:, 1:IWN_HI]
        b = syn[s - 1][:, 1:IWN_HI]
        uv = np.abs(a[0:8] - b[0:8]).max() / np.abs(b[0:8]).max()
        ww = np.abs(a[16:18] - b[8:10]).max() / np.abs(b[8:10]).max()
        assert uv < 1e-4 and ww < 1e-4, (s, uv, ww)


def test_dsv_derivatives_match_finite_differences(aski):
    """(g(r2) - g(r1)) / (r2 - r1) against the mean of the derivatives at the two
    deepest nodes (10 km apart in one layer) for a source at the surface node."""
    w, m, ex, jre, o, n = aski
    assert ex.layer[0] == ex.layer[1]
    out, st, _ = o.dsv_frequency(M.fk_params_c(w.params, jre), [jre], JF, n, 1, IWN_HI)
    h = ex.r[1] - ex.r[0]
    for a, nj, nt in ((out[0], 4, 2), (out[1], 2, 1)):
        pairs = [(0, 2 * nj), (nj, 3 * nj), (4 * nj, 4 * nj + nt)]
        for iv, idv in pairs:
            k = nt if iv == 4 * nj else nj
            fd = (a[1, iv:iv + k, 1:IWN_HI] - a[0, iv:iv + k, 1:IWN_HI]) / h
            tr = 0.5 * (a[1, idv:idv + k, 1:IWN_HI] + a[0, idv:idv + k, 1:IWN_HI])
            assert np.abs(fd - tr).max() / np.abs(tr).max() < 0.03


def test_dsv_node_range_equals_single_source_runs(aski):
    w, m, ex, jre, o, n = aski
    srcs = [1, 5, 8, jre]
    rng, st, _ = o.dsv_frequency(M.fk_params_c(w.params, jre), srcs, JF, n, 1, IWN_HI)
    for i, s in enumerate(srcs):
        one, _, _ = o.dsv_frequency(M.fk_params_c(w.params, s), [s], JF, n, 1, IWN_HI)
        assert np.abs(one[0] - rng[i]).max() <= 1e-13 * np.abs(rng[i]).max()
    one, _, _ = o.dsv_frequency(M.fk_params_c(w.params, jre), [jre], JF, n, 1, IWN_HI)
    assert np.abs(one[1] - rng[-1]).max() <= 1e-13 * np.abs(rng[-1]).max()


def test_aski_first_frequency():
    p = configs.GLOBAL_SMALL.params
    assert M.aski_nf1(p) == 2
    assert M.aski_nf1(dataclasses.replace(p, fmin=5.0 / 1024.0)) == 6
    assert M.frequency_grid(dataclasses.replace(p, fmin=5.0 / 1024.0), 6371000.0).nf1 == 5
    assert M.nsp_dsv("MOMENT") == 20 and M.nsp_dsv("FORCE") == 10


def test_dsv_spectra_obey_reciprocity_in_the_regional_mode():
    """The same reciprocity in the regional (wavenumber) mode on the 8-layer crust:
    U, V and W at the receiver of moment sources at two crustal nodes against the
    synthetics program's spectra of those sources (wavenumbers 2..299)."""
    w = configs.WORKLOADS["regional_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    jf, hi = 40, 300
    n = int(g.nwn[jf - 1])
    o = oracle.Oracle(m, ex)
    pc = M.fk_params_c(w.params, jre)
    out, st, _ = o.dsv_frequency(pc, [3, 12, jre], jf, n, 1, hi)
    syn, sts, _ = o.fk_frequency(pc, jf, n, M.nsp_for(w.params), 1, hi)
    assert np.all(st == 0) and np.all(sts == 0)
    for i, s in enumerate([3, 12]):
        a = out[i][jre - 1][:, 1:hi]
        b = syn[s - 1][:, 1:hi]
        assert np.abs(a[0:8] - b[0:8]).max() / np.abs(b[0:8]).max() < 5e-4, s
        assert np.abs(a[16:18] - b[8:10]).max() / np.abs(b[8:10]).max() < 5e-4, s
