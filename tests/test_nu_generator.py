"""CPU: the COOL_EOS table generator (harm_nu.cuh, host build) against the
mathematics it evaluates.

The generator restates the reference's Fortran abundance() and its modules.
No Fortran compiler exists here, so its output is not compared with the
reference's ("parity unpinned"); these tests pin its pieces instead:
 - the Gauss-Legendre and Gauss-Laguerre rules against roots and weights
   computed in 30-digit arithmetic (mpmath);
 - the generalised Fermi-Dirac integrals against 30-digit adaptive
   quadrature of their definition and against the closed form at eta = 0,
   theta = 0: F_k(0) = Gamma(k+1) (1 - 2^-k) zeta(k+1);
 - the node values against bounds the physics fixes: 3/2 p <= e <= 3 p for a
   mixture of ideal and relativistic gases, pairs, photons and trapped
   neutrinos in the radiation-dominated limit, charge neutrality, and
   fractions in [0, 1].
"""
import math

import mpmath as mp
import numpy as np
import pytest

import harm_cool_b200 as hc
from harm_cool_b200 import eos_tables as et

mp.mp.dps = 30
KS = (0.5, 1.5, 2.5, 3.5)


@pytest.fixture(scope="module")
def lib(harm_lib):
    return harm_lib


def test_quadrature_rules_match_30_digit_roots(lib):
    r = hc.nu_rules()
    for n, (x, w) in ((20, r["l20"]), (40, r["l40"])):
        for xi, wi in zip(x, w):
            t = mp.findroot(lambda s: mp.legendre(n, s), mp.mpf(xi))
            dp = n * (t * mp.legendre(n, t) - mp.legendre(n - 1, t)) / (t * t - 1)
            assert abs(xi / float(t) - 1) <= 2.3e-16
            assert abs(wi / float(2 / ((1 - t * t) * dp * dp)) - 1) <= 4.5e-16
        assert abs(2 * w.sum() - 2) < 1e-14
    x, w = r["g20"]
    for xi, wi in zip(x, w):
        t = mp.findroot(lambda s: mp.laguerre(20, 0, s), mp.mpf(xi))
        want = mp.exp(t) * t / (21 ** 2 * mp.laguerre(21, 0, t) ** 2)
        assert abs(xi / float(t) - 1) <= 2.3e-16
        assert abs(wi / float(want) - 1) <= 4.5e-16


def _fermi_mp(k, eta, theta):
    """30-digit adaptive quadrature, split at the integrand's scales: powers of
    two, eta +- powers of two, and 2/theta where the relativistic factor bends"""
    if eta < 0:  # e^eta times an integrand of order one
        f = lambda x: x ** k * mp.sqrt(1 + theta * x / 2) / (mp.exp(x) + mp.exp(eta))
        scale = mp.exp(eta)
    else:
        f = lambda x: x ** k * mp.sqrt(1 + theta * x / 2) / (mp.exp(x - eta) + 1)
        scale = 1
    pts = {mp.mpf(0), mp.inf}
    for e in range(-3, 8):
        pts.add(mp.mpf(2) ** e)
        for c in (eta - mp.mpf(2) ** e, eta + mp.mpf(2) ** e):
            if c > 0:
                pts.add(c)
    if theta > 0:
        for c in (0.1, 1, 10):
            pts.add(c * 2 / theta)
    return scale * mp.quad(f, sorted(pts))


@pytest.mark.parametrize("eta", [-60.0, -1.0, 0.0, 5.0, 100.0, 1e4])
def test_fermi_integrals_against_quadrature_of_their_definition(lib, eta):
    """Aparicio's four-interval 20-point scheme: within 1e-15 where the
    relativity parameter is small (theta <= 1e-3: all nucleons, and electrons
    below ~0.5 MeV), 2e-10 at its worst (theta ~ 1e3 and eta <~ 10, where
    sqrt(1 + theta x / 2) bends inside the first interval)."""
    thetas = np.array([0.0, 1e-6, 1e-3, 1.0, 1e3, 1e6])
    F = hc.nu_fermi(np.full(len(thetas), eta), thetas)
    for i, th in enumerate(thetas):
        tol = 1e-14 if th <= 1e-3 else 5e-10
        for m, k in enumerate(KS):
            want = float(_fermi_mp(mp.mpf(k), mp.mpf(eta), mp.mpf(th)))
            assert abs(F[i, m] / want - 1) <= tol, (eta, th, k, F[i, m], want)


def test_fermi_integrals_closed_form_at_zero():
    """F_k(0, 0) = Gamma(k+1) (1 - 2^-k) zeta(k+1); F_1/2(0) = 0.678093895..."""
    F = hc.nu_fermi(np.zeros(1), np.zeros(1))[0]
    for m, k in enumerate(KS):
        want = float(mp.gamma(k + 1) * (1 - mp.mpf(2) ** -k) * mp.zeta(k + 1))
        assert abs(F[m] / want - 1) <= 1e-14
    assert abs(F[0] - 0.6780938951531) < 1e-12


def test_fermi_integrals_limits():
    """non-degenerate: F_k -> Gamma(k+1) e^eta; degenerate: F_k -> eta^(k+1) / (k+1)
    (plus the Sommerfeld term pi^2/6 k eta^(k-1))"""
    F = hc.nu_fermi(np.array([-40.0, 1e4]), np.zeros(2))
    for m, k in enumerate(KS):
        assert abs(F[0, m] / (math.gamma(k + 1) * math.exp(-40.0)) - 1) < 1e-15 * 10
        eta = 1e4
        som = eta ** (k + 1) / (k + 1) + math.pi ** 2 / 6 * k * eta ** (k - 1)
        assert abs(F[1, m] / som - 1) < 1e-12


def _xnuc(nb, kt):
    """free-nucleon mass fraction (Popham et al. 1999), capped to [0, 1]"""
    rho10, t11 = nb * 1.66e5, kt * 1.16059e-1
    return min(max(295.5 / rho10 ** 0.75 * t11 ** 1.125 * math.exp(-0.8209 / t11), 0.0), 1.0)


@pytest.fixture(scope="module")
def nodes(lib):
    """rho 1e4..1e14 g/cm^3 at T of 1e8 K (no free nucleons) and 3e9..1e12 K,
    at two radii; the band of a few 1e8 K, where each node costs ~0.3 s on one
    core, is left to the GPU tests"""
    R, T = np.meshgrid([1e4, 1e7, 1e10, 1e12, 1e14], [1e8, 3e9, 3e10, 3e11, 1e12], indexing="ij")
    rho = np.concatenate([R.ravel(), R.ravel()])
    temp = np.concatenate([T.ravel(), T.ravel()])
    hd = np.concatenate([np.full(R.size, et.hdfac(6.0)), np.full(R.size, et.hdfac(40.0))])
    return rho, temp, hd, hc.nu_abundance(rho, temp, hd)


def test_energy_between_ideal_and_relativistic_gas(nodes):
    rho, T, hd, a = nodes
    assert np.all(a["p"] > 0) and np.all(a["e"] > 0)
    ratio = a["e"] / a["p"]
    assert np.all(ratio >= 1.5 * (1 - 1e-12)) and np.all(ratio <= 3.0 * (1 + 1e-12)), ratio


def test_radiation_dominated_limit(nodes):
    """At 1e12 K and 1e4 g/cm^3 photons, relativistic pairs (7/4 of the photons'
    pressure) and the trapped neutrinos (7/8 (b1 + b2), b in [0, 1]) carry the
    pressure: p / p_photon in [2.75, 4.5]"""
    rho, T, hd, a = nodes
    kt = 1e12 / 1.16059e10
    p_gamma = math.pi ** 2 / 45 * kt ** 4 / 197.3269718 ** 3 * 1.6021772e33
    sel = (rho == 1e4) & (T == 1e12)
    r = a["p"][sel] / p_gamma
    assert np.all(r >= 2.75 * (1 - 1e-3)) and np.all(r <= 4.5 * (1 + 1e-3)), r


def test_fractions_and_charge_neutrality(nodes):
    """Either n_e- - n_e+ = n_p + n_e0 (the protons and the electrons of helium)
    to the electron solve's tolerance, or the electron degeneracy was capped at 0
    (eeta, number_den.f90:325-327) and the net electron density is that of
    eta = 0, below n_p + n_e0.  The first check allows for the rounding of
    n_e- - n_e+ where pairs outnumber the net electrons (by 1e8 at 1e12 K and
    1e4 g/cm^3)."""
    rho, T, hd, a = nodes
    assert np.all((a["xp"] >= 0) & (a["xp"] <= 1))
    assert np.all(a["nee"] >= 0) and np.all(a["nep"] >= 0)
    pi, hbc, me = float(np.float32(math.pi)), float(np.float32(197.3269718)), 0.510998910
    n_eq = n_cap = 0
    for k in range(len(rho)):
        nb, kt = rho[k] / 1.66e15, T[k] / 1.16059e10
        x = _xnuc(nb, kt)
        ne = nb * x * a["xp"][k] + abs(1 - x) * nb / 2
        nl = a["nee"][k] - a["nep"][k]
        beta = kt / me
        c = math.sqrt(2.0) / pi ** 2 * (me / hbc) ** 3 * beta ** 1.5
        F = hc.nu_fermi(np.array([0.0, -2.0 / beta]), np.array([beta, beta]))
        n0 = c * (F[0, 0] + beta * F[0, 1]) - c * (F[1, 0] + beta * F[1, 1])
        if abs(nl - ne) <= 1e-8 * ne + 1e-13 * (a["nee"][k] + a["nep"][k]):
            n_eq += 1
        else:
            assert abs(nl / n0 - 1) <= 1e-12 and n0 < ne, (rho[k], T[k], nl, ne, n0)
            n_cap += 1
    assert n_eq >= 10 and n_cap >= 10


def test_neutrino_terms_at_high_temperature(nodes):
    rho, T, hd, a = nodes
    hot = T >= 3e9
    assert np.all(a["qnu"][hot] > 0) and np.all(a["tau"][hot] > 0)
    # a larger scale height (the outer radius) is optically thicker
    n = len(rho) // 2
    assert np.all(a["tau"][n:][hot[n:]] >= a["tau"][:n][hot[:n]])


def test_threads_do_not_change_the_values(nodes):
    rho, T, hd, a = nodes
    b = hc.nu_abundance(rho[::7], T[::7], hd[::7], threads=1)
    for k in a:
        assert np.array_equal(a[k][::7], b[k], equal_nan=True), k
