"""CPU: the oracle and the library's host set-up against fixtures made by the reference.

The fixtures (tests/golden/make_golden.py) hold the reference's own state
after init() and after 1, 2 and 5 steps; the oracle must reproduce them bit
for bit, and the library's host grid code must reproduce the reference's
geometry bit for bit (sha256 of every array)."""
import hashlib

import numpy as np
import pytest

from helpers import active, full_state, load_fixture, make_oracle, problem_from_fixture

CFGS = ["t2d", "t3d"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("cfg", CFGS)
def test_host_geometry_bitexact(cfg, harm_lib):
    fx = load_fixture(cfg)
    pr = problem_from_fixture(fx)
    for k in (1, 2, 3):
        assert pr.params.dx[k] == float(fx["par_dx%d" % k])
        assert pr.params.startx[k] == float(fx["par_startx%d" % k])
    for name, arr in pr.geometry.items():
        assert sha(arr) == str(fx["sha_" + name]), name


@pytest.mark.parametrize("cfg", CFGS)
def test_oracle_steps_bitexact(cfg, harm_lib, oracle_built):
    fx = load_fixture(cfg)
    pr = problem_from_fixture(fx)
    o = make_oracle(pr)
    o.p[...] = full_state(pr, fx["p0"])
    o.pflag[...] = full_state(pr, fx["pflag0"])
    o.set_time(*fx["t0"])
    done = 0
    for n in (1, 2, 5):
        while done < n:
            assert o.step() == 0
            done += 1
        np.testing.assert_array_equal(active(pr, o.p), fx["p%d" % n])
        np.testing.assert_array_equal(active(pr, o.pflag), fx["pflag%d" % n])
        assert o.time() == tuple(fx["t%d" % n])
        d = o.diag()
        assert d["fail_code"] == 0
        vals = [d[k] for k in ("mdot", "edot", "ldot", "mdot_in", "mdot_out", "mass_curr", "mass_in", "mass_out")]
        np.testing.assert_array_equal(np.array(vals), fx["diag%d" % n])


def test_oracle_inversions_kat(oracle_built):
    """Utoprim_2d and the two isentropic fall-backs against the reference's outputs."""
    from oracle.pyoracle import oracle_lib
    import ctypes
    fx = load_fixture("t2d")
    pr = problem_from_fixture(fx)
    kat = dict(np.load(__import__("os").path.join(__import__("helpers").GOLDEN, "kat_u2p.npz")))
    lib = oracle_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    g = pr.geometry
    gam = float(kat["gam"])
    for which, name in ((0, "2d"), (1, "vsq2fix1"), (2, "fix1")):
        for t in range(len(kat["U"])):
            i, j = (int(v) for v in kat["ij"][t])
            U = kat["U"][t].copy()
            prim = kat["guess"][t].copy()
            gcov = np.ascontiguousarray(g["gcov"][i, j, 3])
            gcon = np.ascontiguousarray(g["gcon"][i, j, 3])
            args = [gam, U.ctypes.data_as(dp), gcov.ctypes.data_as(dp), gcon.ctypes.data_as(dp),
                    float(g["gdet"][i, j, 3]), prim.ctypes.data_as(dp)]
            if which == 0:
                r = lib.ora_utoprim_2d(*args)
            elif which == 1:
                r = lib.ora_utoprim_1dvsq2fix1(*args, float(g["katm"][i]))
            else:
                r = lib.ora_utoprim_1dfix1(*args, float(g["katm"][i]))
            assert r == kat["ret_" + name][t], (name, t)
            np.testing.assert_array_equal(prim, kat["prim_" + name][t])
