"""The COOL_EOS table generator on the device (harm_nu_tables, harm_nu.cu)
against the same restatement of abundance() on the host (harm_nu_host.cpp).

The two builds run the same source; they differ in the libm they call (CUDA's
exp, log and pow against glibc's, a few ulps apart), and the Newton solves
inside abundance() stop at a tolerance of 1e-8 relative, so the tables agree
to that tolerance rather than bit for bit.
"""
import numpy as np
import pytest

import harm_cool_b200 as hc
from harm_cool_b200 import eos_tables as et

pytestmark = pytest.mark.gpu


def _nodes():
    """rho 1e4..1e14 g/cm^3 and T 1e8..1e12 K, 9 x 9 log-spaced, at two radii"""
    R, T = np.meshgrid(np.logspace(4, 14, 9), np.logspace(8, 12, 9), indexing="ij")
    rho = np.concatenate([R.ravel(), R.ravel()])
    temp = np.concatenate([T.ravel(), T.ravel()])
    hd = np.concatenate([np.full(R.size, et.hdfac(6.0)), np.full(R.size, et.hdfac(40.0))])
    return rho, temp, hd


def test_device_nodes_match_the_host():
    rho, T, hd = _nodes()
    h = hc.nu_abundance(rho, T, hd)
    d = hc.nu_abundance(rho, T, hd, device=0)
    for k, tol in (("e", 1e-8), ("p", 1e-8), ("nee", 1e-8), ("qnu", 1e-8), ("tau", 1e-8)):
        scale = np.abs(h[k]) + 1e-300
        rel = np.abs(d[k] - h[k]) / scale
        print(k, "max rel %.2e median %.2e" % (rel.max(), np.median(rel)))
        assert rel.max() <= tol, (k, rho[rel.argmax()], T[rel.argmax()], d[k][rel.argmax()], h[k][rel.argmax()])
    assert np.abs(d["xp"] - h["xp"]).max() <= 1e-8


def test_tables_pack_the_nodes_as_calc_cache_val():
    """values[t][i][j] = e, p, Qnu, tau, Yee at rho = x[i], T = y[j], HdFac[t]
    (cooleos.c:171-194), cut into several launches"""
    xa, ya = et.log_axis(7, 1e5, 1e13), et.log_axis(6, 2e8, 5e11)
    hd = np.array([et.hdfac(8.0), et.hdfac(30.0)])
    val, ms = hc.nu_tables(xa, ya, hd, slice_nodes=37)
    assert ms > 0
    R, T = np.meshgrid(xa, ya, indexing="ij")
    for t in range(2):
        a = hc.nu_abundance(R.ravel(), T.ravel(), hd[t], device=0)
        want = np.stack([a["e"], a["p"], a["qnu"], a["tau"], (a["nee"] - a["nep"]) / (R.ravel() / 1.66e15)], axis=1)
        np.testing.assert_array_equal(val[t].reshape(-1, 5), want)
