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


def test_tables_filled_on_demand_give_the_run_on_complete_tables():
    """A 16x16 COOL_EOS torus (1e11 g/cm^3 scale) on 24x24 generator tables over
    rho 1e4-1e14, T 1e8-1e12: filling the nodes as the run reads them
    (eos_tables.on_demand, which marks NaN reads with harm_eos_track_missing)
    ends in the state, flags and temperature guesses of the same 6 steps on
    complete tables, bit for bit, having computed fewer nodes."""
    pr = hc.torus_problem(16, 16, 1, a=0.6, rin=4.0, rmax=11.8, beta=50.0)
    grid = dict(nx=24, ny=24, rho=(1.e4, 1.e14), T=(1.e8, 1.e12), gam=pr.params.gam)
    xa, ya, val, consts, info = et.physical_tables(et.zone_radii(pr), **grid)
    for c in (consts,):
        c["rho_unit"] = 1.e11
        c["u_unit"] = c["p_unit"] = 1.e11 * et.CL * et.CL

    def run(eos):
        ctx = hc.Context(pr)
        ctx.init_torus()
        ctx.set_eos(eos)
        ctx.run(1)
        ctx.run(5)
        p, fl = ctx.get_prims(with_flags=True)
        out = (p, fl, ctx.eos_guess(), ctx.diag()["fail_code"])
        ctx.close()
        return out

    E = hc.Eos(xa, ya, val, consts)
    full = run(E)
    E.close()
    lazy, how, have = et.on_demand(run, xa, ya, consts, margin=2)
    print("on demand:", how["passes"], "passes,", how["nodes"], "of", how["nodes_total"], "nodes")
    assert how["nodes"] < how["nodes_total"] and how["nodes"] == have.sum()
    assert full[3] == 0 and lazy[3] == 0
    for a, b in zip(full[:3], lazy[:3]):
        assert np.array_equal(a, b)
