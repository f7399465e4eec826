"""CPU checks of the oracle's SPECFEM-coupling synthetics
(computeSyntheticsForSpecfemCoupling.f90:677-793): the 42 degree sums with
derivatives, strain, stress, rotations and traction.

The reference holds no vectors for this program; the restatement is pinned by
properties of its parts, for moment and force sources:
* the theta and phi derivatives (moment sums 29-42, force sums 15-21, and the
  phi-derivative formulas) against central differences of the displacement in
  distance and azimuth;
* the radial derivatives (moment sums 15-28, force sums 8-14) against finite
  differences of the
  displacement between two nodes 10 km apart;
* the rotations to the box frame keep the length of the displacement vector,
  and the traction of a symmetric stress satisfies n2 . t(n1) = n1 . t(n2).
"""
import dataclasses

import numpy as np
import pytest

import oracle
from gemini_unified_b200 import configs, model as M

JF = 30
MT = np.array([1.0, -0.4, 0.7, 0.3, -0.5, 0.2])
FORCE = np.array([0.8, -0.3, 0.6])
FS = [2.0, 0.002, 4.0, 0.04]
ZEL = [1.1e11 + 1e8j, 1.2e11 + 1e8j, 4e10, 4.5e10 + 5e7j, 4.4e10, 0, 0]


@pytest.fixture(scope="module")
def dsv():
    w = dataclasses.replace(configs.GLOBAL_SMALL, nnod_blocks=[4], dr_blocks=[10000.0])
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    n = int(g.nwn[JF - 1])
    out, st, _ = oracle.Oracle(m, ex).dsv_frequency(M.fk_params_c(w.params, jre), [jre], JF, n)
    assert np.all(st == 0)
    nwn = np.zeros(JF, np.int32)
    nwn[JF - 1] = n
    zel = np.tile(np.array(ZEL, complex), (JF, 1))
    return ex, g, n, nwn, out, zel


def _run(dsv, node, d, x, nrm=(0.0, 0.0, 1.0), istyp=1):
    ex, g, n, nwn, out, zel = dsv
    gm = out[0] if istyp == 1 else out[1]          # moment source, or the force at the same node
    gr = gm[node - 1].real.astype(np.float32)
    gi = gm[node - 1].imag.astype(np.float32)
    src = MT if istyp == 1 else FORCE
    return oracle.coupling(JF, JF, nwn, n, gr, gi, g.df, g.sigma, ex.r[node - 1], zel, src, FS, 0.0, 2048, 0.5,
                           0.1, 0.2, 0.3, 0.4, [d], [x], [list(nrm)], spectra=True, debug=True, istyp=istyp)


@pytest.mark.parametrize("istyp", [1, 0])
def test_theta_and_phi_derivatives_against_central_differences(dsv, istyp):
    ex = dsv[0]
    d0, x0, h = np.radians(30.0), np.radians(40.0), 1e-4
    _, _, D = _run(dsv, 1, d0, x0, istyp=istyp)
    ut, uf = D[0, JF - 1, 2], D[0, JF - 1, 3]
    _, _, Dp = _run(dsv, 1, d0 + h, x0, istyp=istyp)
    _, _, Dm = _run(dsv, 1, d0 - h, x0, istyp=istyp)
    fd = (Dp[0, JF - 1, 0] - Dm[0, JF - 1, 0]) / (2 * h) / ex.r[0]
    assert np.abs(fd - ut).max() / np.abs(ut).max() < 1e-3        # O((h l)^2) with l <= 396
    _, _, Dp = _run(dsv, 1, d0, x0 + h, istyp=istyp)
    _, _, Dm = _run(dsv, 1, d0, x0 - h, istyp=istyp)
    fd = (Dp[0, JF - 1, 0] - Dm[0, JF - 1, 0]) / (2 * h) / (ex.r[0] * np.sin(d0))
    assert np.abs(fd - uf).max() / np.abs(uf).max() < 1e-6


@pytest.mark.parametrize("istyp", [1, 0])
def test_radial_derivative_against_two_nodes(dsv, istyp):
    ex = dsv[0]
    d0, x0 = np.radians(30.0), np.radians(40.0)
    _, _, D1 = _run(dsv, 1, d0, x0, istyp=istyp)
    _, _, D2 = _run(dsv, 2, d0, x0, istyp=istyp)
    fd = (D2[0, JF - 1, 0] - D1[0, JF - 1, 0]) / (ex.r[1] - ex.r[0])
    tr = 0.5 * (D2[0, JF - 1, 1] + D1[0, JF - 1, 1])
    assert np.abs(fd - tr).max() / np.abs(tr).max() < 0.02


def test_rotation_keeps_length_and_traction_is_symmetric(dsv):
    d0, x0 = np.radians(55.0), np.radians(-120.0)
    S, _, D = _run(dsv, 3, d0, x0)
    u = D[0, JF - 1, 0]
    assert abs(np.sum(np.abs(S[0, :3, JF - 1]) ** 2) - np.sum(np.abs(u) ** 2)) <= 1e-12 * np.sum(np.abs(u) ** 2)
    n1, n2 = np.array([0.3, -0.5, 0.8]), np.array([-0.7, 0.2, 0.4])
    t1 = _run(dsv, 3, d0, x0, n1)[0][0, 3:, JF - 1]
    t2 = _run(dsv, 3, d0, x0, n2)[0][0, 3:, JF - 1]
    assert abs(n2 @ t1 - n1 @ t2) <= 1e-12 * max(abs(n2 @ t1), 1e-300)
    assert np.abs(t1).max() > 0
