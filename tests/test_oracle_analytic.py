"""The oracle's radial integrations against closed forms in a homogeneous sphere.

These checks pin the oracle outside its own code: the closed forms come from
the elastic equations of a homogeneous, isotropic, anelastic sphere, not from
the reference.  With complex moduli L = N = mu, C = A = lambda + 2 mu, F =
lambda, density rho and complex frequency omega (omre + i omim), the
solutions regular at the centre are spherical Bessel functions j_nu of order
nu, nu (nu + 1) = dll1, at k_a = omega sqrt(rho / C) (P) and k_b = omega
sqrt(rho / L) (S):

* toroidal: W = j_nu(k_b r), T = L (W' - W / r);
* spheroidal, in the variables (U, R, V, S) of radial displacement, radial
  traction, horizontal displacement and tangential traction: from the P
  potential U = k_a j_nu'(k_a r), V = j_nu(k_a r) / r; from the S potential
  U = dll1 j_nu(k_b r) / r, V = j_nu(k_b r) / r + k_b j_nu'(k_b r); and
  R = C U' + F (2 U - dll1 V) / r, S = L (V' - V / r + U / r);
* the spheroidal minors m_ij = w_i^P w_j^S - w_j^P w_i^S (the second-order
  minors of the basis solutions); the 5-variable system carries
  (m12, m13, m14, m23, m24), and m34 = -m12 / dll1 for the regular pair.

The checks:

* the start vectors of the upward integrations (toroidalBottomInitialValues,
  minorsBottomInitialValues, initialValues.f90:202-416, evaluated with
  continued fractions converged to 1e-6) are parallel to the closed forms;
* starting from the closed form at r0, one propagation of the toroidal and
  minors systems (propagateOde.f90:132-331 with the Bulirsch-Stoer step of
  complexBulirschStep.f90:111-359 and the system matrices of
  toroidalOdeSystem.f90:81-102 and minorsOdeSystem.f90:77-126) reproduces the
  closed form at r1 in amplitude and direction, to the integration accuracy;
* the adjoint solid system (solidtOdeSystem.f90:77-114) keeps z . w constant
  for the closed-form forward solutions w.

Closed forms use mpmath at 30 digits.
"""
import mpmath as mp
import numpy as np
import pytest

from gemini_unified_b200.model import ExternalRadialNodes, node_model_from_dict

RE = 6371000.0
R_INNER = 2000000.0    # top of the homogeneous innermost layer (a second, constant layer lies above)
VP, VS, RHO, QMU, QKAPPA = 8000.0, 4500.0, 3300.0, 600.0, 57823.0
ATTMODE = 1           # attenuation and dispersion, as the FK loop runs it
F = 0.05              # Hz
OMIM = -5.0 / 1024.0  # imaginary part of the complex frequency (-sigma of df = 1/1024)
PI_F32 = float(np.float32(np.pi))   # the reference's default-REAL pi


def homogeneous_sphere():
    d = {"reference_frequency_hz": 1.0, "anisotropic": False, "earth_radius": RE, "full_space": 0,
         "equidistant_nodes": 1, "num_layers": 2, "num_nodes": 3, "layer_inner_core": 0, "layer_outer_core": 0,
         "radius_inner_core": 0.0, "radius_outer_core": 0.0, "radius_upper_layer_boundary_m": [R_INNER, RE],
         "isfluid": [0, 0], "index_upper_boundary": [1, 3],
         "node_properties": {"depth": [RE - R_INNER, RE - R_INNER, 0.0], "density": [RHO] * 3,
                             "P-velocity": [VP] * 3, "S-velocity": [VS] * 3, "Qkappa": [QKAPPA] * 3,
                             "Qmu": [QMU] * 3}}
    return node_model_from_dict(d, name="homogeneous_sphere")


@pytest.fixture(scope="module")
def sphere():
    import oracle
    m = homogeneous_sphere()
    ex = ExternalRadialNodes.from_blocks(m, [1], [10000.0], 0.0, RE)
    o = oracle.Oracle(m, ex)
    _, _, el, _ = o.spline(F, ATTMODE)
    A, C, Fm, L, N = (complex(v) for v in el[2, :5])
    assert abs(A - C) <= 1e-12 * abs(C) and abs(L - N) <= 1e-12 * abs(L)   # isotropic
    assert np.allclose(el[0, :5], el[2, :5], rtol=1e-14)                    # homogeneous
    om = mp.mpc(2.0 * PI_F32 * F, OMIM)
    return o, {"om": om, "ro": mp.mpf(RHO), "C": mp.mpc(C), "F": mp.mpc(Fm), "L": mp.mpc(L)}


mp.mp.dps = 30


def _sph(nu, z):
    """j_nu(z), j_nu'(z), j_nu''(z) for complex z and real order nu."""
    j = mp.sqrt(mp.pi / (2 * z)) * mp.besselj(nu + 0.5, z)
    j1 = mp.sqrt(mp.pi / (2 * z)) * mp.besselj(nu + 1.5, z)
    jp = nu / z * j - j1
    jpp = -(2 / z) * jp - (1 - nu * (nu + 1) / z ** 2) * j
    return j, jp, jpp


def toroidal(r, p, dll1):
    nu = -0.5 + mp.sqrt(0.25 + dll1)
    kb = p["om"] * mp.sqrt(p["ro"] / p["L"])
    j, jp, _ = _sph(nu, kb * r)
    return [j, p["L"] * (kb * jp - j / r)]


def solid(r, p, dll1):
    """(U, R, V, S) of the P and S solutions regular at the centre."""
    nu = -0.5 + mp.sqrt(0.25 + dll1)
    C, Fm, L = p["C"], p["F"], p["L"]
    ka = p["om"] * mp.sqrt(p["ro"] / C)
    kb = p["om"] * mp.sqrt(p["ro"] / L)
    out = []
    j, jp, jpp = _sph(nu, ka * r)
    U, Up, V, Vp = ka * jp, ka ** 2 * jpp, j / r, ka * jp / r - j / r ** 2
    out.append([U, C * Up + Fm * (2 * U - dll1 * V) / r, V, L * (Vp - V / r + U / r)])
    j, jp, jpp = _sph(nu, kb * r)
    U, Up = dll1 * j / r, dll1 * (kb * jp / r - j / r ** 2)
    V, Vp = j / r + kb * jp, kb * jp / r - j / r ** 2 + kb ** 2 * jpp
    out.append([U, C * Up + Fm * (2 * U - dll1 * V) / r, V, L * (Vp - V / r + U / r)])
    return out


def minors(r, p, dll1):
    wP, wS = solid(r, p, dll1)
    m = lambda i, j: wP[i] * wS[j] - wP[j] * wS[i]
    return [m(0, 1), m(0, 2), m(0, 3), m(1, 2), m(1, 3)], m(2, 3)


def _c(v):
    return np.array([complex(x) for x in v])


def _direction_error(a, b):
    """Distance between the complex directions of two vectors."""
    k = int(np.argmax(np.abs(b)))
    a, b = a / a[k], b / b[k]
    return float(np.abs(a - b).max() / np.abs(b).max())


# (dll1, r0, r1): start below the turning point of the S waves (where the start
# values use the Bessel-ratio fraction) and integrate into the oscillating part;
# the second case starts in the homogeneous innermost layer and crosses its top
CASES = [(300.0 * 301.0, 3.0e6, 6.0e6), (30.0 * 31.0 + 0.37, 1.5e6, 6.2e6)]


@pytest.mark.parametrize("dll1,r0,r1", CASES)
def test_closed_forms_satisfy_the_minor_relation(sphere, dll1, r0, r1):
    _, p = sphere
    for r in (r0, r1):
        m5, m34 = minors(r, p, dll1)
        assert abs(m34 + m5[0] / dll1) <= 1e-20 * abs(m34)


@pytest.mark.parametrize("dll1,r0,r1", CASES)
def test_start_vectors_are_the_regular_solutions(sphere, dll1, r0, r1):
    o, p = sphere
    yt, htry, rc = o.bottom_iv(F, ATTMODE, OMIM, dll1, r0, 0)
    assert rc == 0 and htry > 0
    assert _direction_error(yt, _c(toroidal(r0, p, dll1))) <= 1e-5
    ym, _, rc = o.bottom_iv(F, ATTMODE, OMIM, dll1, r0, 1)
    assert rc == 0
    assert _direction_error(ym, _c(minors(r0, p, dll1)[0])) <= 1e-5


@pytest.mark.parametrize("dll1,r0,r1", CASES)
def test_propagation_reproduces_the_closed_forms(sphere, dll1, r0, r1):
    """Amplitude and direction at r1 from the exact values at r0, at the integration
    accuracies 1e-5 (the configurations' ACCURACY), 1e-7 and 1e-9.  The error accumulates
    over the steps of the path: 15-90 eps over 3000 km at l = 300, up to 500 eps over the
    4700 km (about 70 S wavelengths) at l = 30 (measured).  The bar is 1000 eps, and the
    error must fall by at least 100x from eps 1e-5 to 1e-9: the integration converges to
    the closed form."""
    o, p = sphere
    for sys, form in ((3, lambda r: toroidal(r, p, dll1)), (0, lambda r: minors(r, p, dll1)[0])):
        y0 = _c(form(r0))
        ref = [mp.mpc(v) for v in form(r1)]
        errs = []
        for eps in (1e-5, 1e-7, 1e-9):
            y1, lg, rc = o.propagate(F, ATTMODE, OMIM, dll1, sys, r0, r1, 1.0e4, eps, y0)
            assert rc == 0
            # y(r1) = y1 10^lg, compared in mpmath
            scale = mp.mpf(10) ** mp.mpf(lg)
            got = [mp.mpc(complex(v)) * scale for v in y1]
            err = float(max(abs(g - r) for g, r in zip(got, ref)) / max(abs(r) for r in ref))
            assert err <= 1000 * eps, (sys, eps, err)
            errs.append(err)
        assert errs[2] <= errs[0] / 100, (sys, errs)


def test_adjoint_system_keeps_the_pairing_with_forward_solutions(sphere):
    """z' = -A^T z and w' = A w give d(z.w)/dr = 0: integrate the adjoint solid system
    downward from r1 and compare z.w at r0 with z.w at r1 for both regular solutions.
    Going down, z grows by some 35 orders of magnitude, so z.w is a difference of large
    terms; its error is measured against the largest term at either end (measured: 4 eps
    for the P solution, below eps for the S solution), and it must converge with eps."""
    o, p = sphere
    dll1, r0, r1 = 300.0 * 301.0, 4.5e6, 6.0e6
    rng = np.random.default_rng(3)
    z1 = rng.standard_normal(4) + 1j * rng.standard_normal(4)
    w0, w1 = solid(r0, p, dll1), solid(r1, p, dll1)
    errs = []
    for eps in (1e-5, 1e-9):
        z0, lg, rc = o.propagate(F, ATTMODE, OMIM, dll1, 4, r1, r0, -1.0e4, eps, z1)
        assert rc == 0
        scale = mp.mpf(10) ** mp.mpf(lg)
        for k in range(2):
            t0 = [mp.mpc(complex(z)) * scale * w for z, w in zip(z0, w0[k])]
            t1 = [mp.mpc(complex(z)) * w for z, w in zip(z1, w1[k])]
            terms = max(max(abs(t) for t in t0), max(abs(t) for t in t1))
            err = float(abs(sum(t0) - sum(t1)) / terms)
            assert err <= 10 * eps, (k, eps, err)
            errs.append(err)
    assert errs[2] <= errs[0] / 100 and errs[3] <= errs[1] / 100, errs
