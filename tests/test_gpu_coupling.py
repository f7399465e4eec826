"""GPU parity of the synthetics for SPECFEM coupling (gem_coupling_run) with
the CPU oracle (computeSyntheticsForSpecfemCoupling.f90:677-793).

Both sides take the same float32 DSV spectra with radial derivatives (from
gem_fk_run_dsv, a moment source or a force at the surface node) at the node of
the boundary points.  In the FP64 form the degree sums run in FP64 on both sides
and differ only in the order of the additions: spectra must agree to 1e-9
relative to the largest value of each (point, component) spectrum.  The mixed
form (fast backend) runs the 13 products on the tensor cores as sliced-INT8
integer products (42 bits of each operand, exact INT32 accumulation): its
spectra must agree to 1e-8.  Time series are float32 and must agree to 1e-6
relative to the largest sample of each series in both forms."""
import dataclasses

import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu
NPTS = 16
MT = np.array([1.0, -0.4, 0.7, 0.3, -0.5, 0.2])
FORCE = np.array([0.8, -0.3, 0.6])
FS = (2.0, 0.002, 4.0, 0.04)


@pytest.fixture(scope="module")
def case(gpu):
    from gemini_unified_b200.fk import GEM_BACKEND_GPU_FAST, GeminiFK
    w = dataclasses.replace(configs.GLOBAL_SMALL, nnod_blocks=[4], dr_blocks=[10000.0])
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    fk = GeminiFK(m, ex)
    gre, gim, _, st = fk.run_dsv(w.params, jre, g.nf1, g.nf2, f64=False)
    fre, fim, _, sf = fk.run_dsv(dataclasses.replace(w.params, source_type="FORCE"), jre, g.nf1, g.nf2, f64=False)
    assert np.all(st == 0) and np.all(sf == 0)
    rng = np.random.default_rng(7)
    delta = np.radians(np.linspace(10.0, 80.0, NPTS))
    xi = np.radians(rng.uniform(-180.0, 180.0, NPTS))
    nrm = rng.normal(size=(NPTS, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    f = np.arange(g.nf2) * g.df
    base = np.array([1.1e11 + 1e8j, 1.2e11 + 1e8j, 4e10, 4.5e10 + 5e7j, 4.4e10, 0, 0])
    zel = base[None, :] * (1.0 + 0.01 * f[:, None])
    node = 1
    return dict(w=w, g=g, fk=fk, fast=GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST), gr={1: gre[node - 1], 0: fre[node - 1]}, gi={1: gim[node - 1], 0: fim[node - 1]},
                re=ex.r[node - 1], delta=delta, xi=xi, nrm=nrm, zel=zel, nkf=gre.shape[2])


def _params(c, spectra, istyp=1):
    from gemini_unified_b200.fk import CouplingParams
    g = c["g"]
    return CouplingParams(nf1=g.nf1, nf2=g.nf2, nwnmax=g.nwnmax, nkfmax=c["nkf"], nsp=20 if istyp else 10,
                          df=g.df, sigma=g.sigma, istyp=istyp,
                          re=c["re"], nsamp=2048, dt=0.5, tred=0.0, order_highpass=int(FS[0]), fc_highpass=FS[1],
                          order_lowpass=int(FS[2]), fc_lowpass=FS[3], thetas=0.35, phis=1.1, thetac=0.6,
                          phic=1.4, spectra=1 if spectra else 0)


def _oracle(c, spectra, istyp=1):
    import oracle
    g = c["g"]
    return oracle.coupling(g.nf1, g.nf2, g.nwn, g.nwnmax, c["gr"][istyp], c["gi"][istyp], g.df, g.sigma, c["re"],
                           c["zel"], MT if istyp else FORCE, FS, 0.0, 2048, 0.5, 0.35, 1.1, 0.6, 1.4, c["delta"],
                           c["xi"], c["nrm"], spectra=spectra, istyp=istyp)


def _gpu(c, spectra, istyp=1, backend=1):
    return c["fk" if backend == 1 else "fast"].coupling(_params(c, spectra, istyp), c["g"].nwn, c["gr"][istyp], c["gi"][istyp], c["zel"],
                            MT if istyp else FORCE, c["delta"], c["xi"], c["nrm"])


@pytest.mark.parametrize("backend", [1, 2])
@pytest.mark.parametrize("istyp", [1, 0])
def test_coupling_spectra_match_oracle(case, istyp, backend):
    got = _gpu(case, True, istyp, backend)
    ref = _oracle(case, True, istyp)[0]
    assert got.shape == ref.shape == (NPTS, 6, case["g"].nf2)
    scale = np.abs(ref).max(axis=2, keepdims=True)
    assert np.all(scale > 0)
    err = (np.abs(got - ref) / scale).max()
    print("backend %d istyp %d: spectra %.2e" % (backend, istyp, err))
    assert err <= (1e-9 if backend == 1 else 1e-8)


@pytest.mark.parametrize("backend", [1, 2])
@pytest.mark.parametrize("istyp", [1, 0])
def test_coupling_time_series_match_oracle(case, istyp, backend):
    got = _gpu(case, False, istyp, backend)
    ref = _oracle(case, False, istyp)[1]
    assert got.shape == ref.shape == (NPTS, 6, 2048)
    scale = np.abs(ref).max(axis=2, keepdims=True)
    assert np.all(scale > 0)
    assert (np.abs(got.astype(np.float64) - ref) / scale).max() <= 1e-6


def test_coupling_rejects_spectra_without_derivatives(case):
    from gemini_unified_b200.model import GeminiError
    p = _params(case, True)
    p.nsp = 10
    with pytest.raises(GeminiError, match="derivatives"):
        case["fk"].coupling(p, case["g"].nwn, case["gr"][1][:10], case["gi"][1][:10], case["zel"], MT,
                            case["delta"], case["xi"], case["nrm"])
