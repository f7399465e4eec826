"""Travel-time table by ray tracing (computeTravelTimeTable.f90:160-226) on the GPU
against the CPU oracle, and the table lookup (travelTimes.f90:105-260) against a
restatement here.  The ray integrator repeats the reference's operations in FP64
without FMA contraction on both sides, and the table is float32 as the reference
stores it, so the tables must agree to float32 rounding."""
import numpy as np
import pytest

from gemini_unified_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rays(gpu):
    from gemini_unified_b200.fk import GeminiFK
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    fk = GeminiFK(m, ex)
    return m, ex, fk


@pytest.mark.parametrize("stype", ["P", "S"])
def test_ray_table_matches_oracle(rays, stype):
    import oracle
    m, ex, fk = rays
    rtp, slow, tab = fk.ray_table(stype, attmode=3, eps=1e-6, drtp=20000.0)
    rc, rtp_o, slow_o, tab_o, st = oracle.Oracle(m, ex).ray_table(stype, 3, 1e-6, 20000.0, float(ex.r[-1]), 400,
                                                                  ex.nnod)
    assert rc == 0 and np.all(st == 0)
    assert len(rtp) == len(rtp_o) == 145
    np.testing.assert_array_equal(rtp, rtp_o)
    assert np.abs(slow / slow_o - 1.0).max() <= 1e-14
    assert np.abs(tab - tab_o).max() <= 1e-6 * np.abs(tab_o).max()
    assert np.all(tab[:, -1, 1] > 0)


def _locate(xx, a):
    """locate (locatePoint.f90:72-101) on a[0..n-1] as a 1-based array: 0..n."""
    n = len(a)
    lo, hi = 0, n + 1
    asc = a[n - 1] > a[0]
    while hi - lo > 1:
        mid = (lo + hi) // 2
        gt = xx > a[mid - 1]
        if asc:
            lo, hi = (mid, hi) if gt else (lo, mid)
        else:
            lo, hi = (lo, mid) if gt else (mid, hi)
    return lo


def _tele_time(rnod, rtp, slow, tab, rs, re, din):
    """getTravelTimes for a TELE table and a distance inside the table's range."""
    def legs(r):   # node interval of radius r and its interpolation weights
        j = _locate(np.float32(r), rnod)
        j = min(max(j, 1), len(rnod) - 1)
        a = (float(rnod[j]) - r) / float(np.float32(rnod[j] - rnod[j - 1]))
        return j, a, 1.0 - a
    js, as_, bs = legs(rs)
    je, ae, be = legs(re)
    jtps, jtpr = _locate(np.float32(rs), rtp), _locate(np.float32(re), rtp)
    n = min(jtps, jtpr)
    D = tab[:n, :, 0].astype(np.float64); T = tab[:n, :, 1].astype(np.float64)
    dv = as_ * D[:, js - 1] + bs * D[:, js] + ae * D[:, je - 1] + be * D[:, je]
    tv = as_ * T[:, js - 1] + bs * T[:, js] + ae * T[:, je - 1] + be * T[:, je] - slow[:n].astype(np.float64) * dv
    jd = _locate(din, dv)
    ad = (dv[jd] - din) / (dv[jd] - dv[jd - 1])
    bd = 1.0 - ad
    tau = ad * tv[jd - 1] + bd * tv[jd]
    p = ad * float(slow[jd - 1]) + bd * float(slow[jd])
    return tau + p * din


def test_travel_time_lookup(rays):
    m, ex, fk = rays
    rtp, slow, tab = fk.ray_table("P", attmode=3, eps=1e-6, drtp=20000.0)
    rnod = ex.r.astype(np.float32)
    rtp32, slow32 = rtp.astype(np.float32), slow.astype(np.float32)
    rs, re = float(ex.r[5]), float(ex.r[-1])
    deg = np.linspace(35.0, 90.0, 41)
    tt = fk.travel_times(rtp32, slow32, tab, rs, re, np.radians(deg), tele=True)
    ref = np.array([_tele_time(rnod, rtp32, slow32, tab, rs, re, d) for d in np.radians(deg)])
    assert np.abs(tt - ref).max() <= 1e-9 * ref.max()
    assert np.all(np.diff(tt) > 0)                          # later arrivals farther away
    assert 500.0 < tt[np.argmin(np.abs(deg - 60.0))] < 700.0   # a P wave near 60 degrees (s)
