"""Pins of the descriptor's building blocks against independent implementations.

The soap_turbo source is absent from the reference tree, so the descriptor's
values cannot be compared with the reference; what can be pinned is every
mathematical ingredient, against scipy and exact polynomial integration:
the orthonormal poly3 basis, the real spherical harmonics, the smeared angular
factor and the Gaussian radial projection, and each analytic derivative by
finite differences.
"""
import numpy as np
import pytest
from scipy import integrate, special

from _util import O
from turbogap_b200.hypers import SoapTurboHypers, carbon_hypers


def test_poly3_basis_is_orthonormal_gram_schmidt():
    """phi_n = rc^-1/2 t^3 sum_j W[n,j] t^j, t=(rc-x)/rc: orthonormal on [0, rc] and
    spanning (rc - x)^(alpha+2), alpha = 1..alpha_max, in Gram-Schmidt order."""
    from fractions import Fraction
    for amax in (4, 8):
        W = O.poly3_W(amax)
        # W[n] = sqrt(2n+7) * integer coefficients: recover them and integrate exactly
        C = [[int(round(W[n, j] / np.sqrt(2 * n + 7))) for j in range(amax)] for n in range(amax)]
        for n in range(amax):
            assert np.allclose(np.array(C[n]) * np.sqrt(2 * n + 7), W[n], rtol=1e-15, atol=0)
        for a in range(amax):
            for b in range(amax):
                # int_0^1 t^6 (sum_i C_ai t^i)(sum_j C_bj t^j) dt
                g = sum(Fraction(C[a][i] * C[b][j], i + j + 7)
                        for i in range(amax) for j in range(amax))
                want = Fraction(1, 2 * a + 7) if a == b else Fraction(0)
                assert g == want, (a, b)
        # triangular: phi_n has no t^j for j > n (Gram-Schmidt of t^3, t^4, ...)
        assert np.all(np.triu(W, 1) == 0)


def test_real_ylm_matches_scipy_and_gradient():
    rng = np.random.default_rng(1)
    L = 8
    for _ in range(20):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        Y, dY = O.real_ylm(L, u, with_grad=True)
        theta = np.arccos(u[2])
        phi = np.arctan2(u[1], u[0])
        for l in range(L + 1):
            for m in range(-l, l + 1):
                # scipy: complex Y_l^m with Condon-Shortley phase
                ya = special.sph_harm_y(l, abs(m), theta, phi)
                cs = (-1) ** abs(m)
                if m == 0:
                    ref = ya.real
                elif m > 0:
                    ref = np.sqrt(2) * cs * ya.real
                else:
                    ref = np.sqrt(2) * cs * ya.imag
                assert abs(Y[l * l + l + m] - ref) < 1e-12
        # tangential gradient vs finite differences on the sphere
        eps = 1e-6
        for q in range(3):
            e = np.zeros(3)
            e[q] = eps
            up = (u + e) / np.linalg.norm(u + e)
            um = (u - e) / np.linalg.norm(u - e)
            fd = (O.real_ylm(L, up) - O.real_ylm(L, um)) / (2 * eps)
            an = dY[:, q] - (dY @ u) * u[q]
            assert np.abs(fd - an).max() < 1e-6


def test_angular_factor_is_smeared_legendre_expansion():
    """a_l(r) = 4 pi e^-k i_l(k), k = r^2/sigma_t^2: the Legendre coefficients of the
    angular Gaussian exp(-r^2 (1 - cos g)/sigma_t^2)."""
    h = carbon_hypers()
    hc = O.HypersC(h)
    for r in (0.7, 1.5, 2.6, 3.5):
        a, da = O.angular(hc, 0, r)
        k = r * r / 0.25
        ref = 4 * np.pi * np.exp(-k) * special.spherical_in(np.arange(9), k)
        assert np.allclose(a, ref, rtol=1e-12, atol=1e-300)
        # same coefficients by direct projection of the angular Gaussian
        for l in (0, 3, 8):
            f = lambda c: np.exp(-k * (1 - c)) * special.eval_legendre(l, c)
            proj = integrate.quad(f, -1, 1, epsabs=1e-14)[0] * (2 * l + 1) / 2
            assert abs(proj * 4 * np.pi / (2 * l + 1) - a[l]) < 1e-10 * max(1, abs(a[l]))
        e = 1e-6
        fd = (O.angular(hc, 0, r + e)[0] - O.angular(hc, 0, r - e)[0]) / (2 * e)
        assert np.abs(fd - da).max() < 1e-6


@pytest.mark.parametrize("re_", [0, 1, 2])
@pytest.mark.parametrize("srs", [0.0, 0.1])
def test_radial_projection_matches_quadrature(re_, srs):
    """R~_n(r) = w(r) int_0^rc phi_n(x) x^re exp(-(x-r)^2/(2 sigma_r(r)^2)) dx."""
    h = SoapTurboHypers(species_z=[1], alpha_max=[8], radial_enhancement=re_,
                        atom_sigma_r_scaling=[srs], amplitude_scaling=[1.5])
    hc = O.HypersC(h)
    rc, W = 3.7, O.poly3_W(8)

    def phi(n, x):
        t = (rc - x) / rc
        return rc ** -0.5 * t ** 3 * np.polyval(W[n][::-1], t)

    for r in (0.0, 1.1, 2.3, 3.4):
        R, dR = O.radial(hc, 0, r, self_pair=(r == 0.0))
        sig = 0.5 * (1 + srs * r)
        if r == 0.0:
            w = 1.0  # central atom: global_scaling * central_weight
        else:
            x = r / rc
            w = (1 - 3 * x * x + 2 * x ** 3) ** 1.5
            if r > 3.2:
                t = (r - 3.2) / 0.5
                w *= np.exp(-4 * t * t / (1 - t * t))
        for n in range(8):
            f = lambda xx: phi(n, xx) * xx ** re_ * np.exp(-(xx - r) ** 2 / (2 * sig ** 2))
            ref = w * integrate.quad(f, 0, rc, epsabs=1e-13, limit=200)[0]
            assert abs(R[n] - ref) < 1e-9, (n, r)
        if r > 0:
            # d/dr under the integral (w' from the closed form), by quadrature
            dsig = 0.5 * srs
            x = r / rc
            P = 1 - 3 * x * x + 2 * x ** 3
            dw = 1.5 * P ** 0.5 * (-6 * x + 6 * x * x) / rc
            if r > 3.2:
                t = (r - 3.2) / 0.5
                fc = np.exp(-4 * t * t / (1 - t * t))
                dw = dw * fc + P ** 1.5 * fc * (-4) * (2 * t / (1 - t * t) ** 2) / 0.5
            for n in range(8):
                g = lambda xx: (phi(n, xx) * xx ** re_ * np.exp(-(xx - r) ** 2 / (2 * sig ** 2)))
                dg = lambda xx: g(xx) * ((xx - r) / sig ** 2 + (xx - r) ** 2 * dsig / sig ** 3)
                ref = dw * integrate.quad(g, 0, rc, epsabs=1e-13, limit=200)[0] + \
                    w * integrate.quad(dg, 0, rc, epsabs=1e-13, limit=200)[0]
                assert abs(dR[n] - ref) < 1e-8, (n, r)


def test_radial_vanishes_smoothly_at_cutoff():
    hc = O.HypersC(carbon_hypers())
    for r in (3.7, 3.8):
        R, dR = O.radial(hc, 0, r)
        assert np.all(R == 0) and np.all(dR == 0)
    R, dR = O.radial(hc, 0, 3.699)
    assert np.abs(R).max() < 1e-30 and np.abs(dR).max() < 1e-26
