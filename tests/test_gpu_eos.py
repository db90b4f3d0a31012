"""GPU: the device run-time COOL_EOS (harm_eos_batch) against the oracle's
restatement of cooleos.c/cache4d.c/akima.c/mnewt.h, bit for bit, on the tables
the reference's COOL_EOS build makes (oracle/eos_standin.c as generator), and
against the reference's own outputs in tests/golden/eos_ce2d.npz."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables(oracle_built):
    from oracle.pyoracle import standin_tables
    f = np.load(os.path.join(GOLDEN, "eos_ce2d.npz"))
    startx1, dx1, R0, gam = f["grid"]
    return standin_tables(startx1, dx1, R0, int(f["sn1"]), gam), f


@pytest.fixture(scope="module")
def dev(harm_lib, tables):
    import harm_cool_b200 as hc
    T, _ = tables
    e = hc.Eos(T.xa, T.ya, T.val, T.consts)
    yield e
    e.close()


def _same(a, b):
    return (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))


@pytest.mark.parametrize("what", ["pressure", "dpdu", "dpdrho"])
def test_device_eos_matches_reference_fixture(what, dev, tables):
    _, f = tables
    v, lt = dev.batch(what, f["tab"], f["rho0"], f["u"], f["lastT"])
    ok = _same(v, f[what])
    assert ok.all(), np.flatnonzero(~ok)[:10]
    assert _same(lt, f[what + "_lastT"]).all()


@pytest.mark.parametrize("seed", [11, 12])
def test_device_eos_matches_oracle(seed, dev, tables):
    from oracle.pyoracle import OracleEos
    from golden.make_golden import eos_inputs
    T, _ = tables
    O = OracleEos(T)
    tab, rho0, u, lastT = eos_inputs(np.random.default_rng(seed), T.ntab, 50000)
    for what in ("pressure", "dpdu", "dpdrho"):
        a, la = dev.batch(what, tab, rho0, u, lastT)
        b, lb = O.batch(what, tab, rho0, u, lastT)
        ok = _same(a, b)
        assert ok.all(), (what, np.flatnonzero(~ok)[:10])
        assert _same(la, lb).all(), what


def test_device_eos_guesses_chain_like_the_reference(dev, tables):
    """Calls that share one guess in sequence (InitCache_CoolEOS's LastT) give what
    the oracle gives for the same sequence."""
    from oracle.pyoracle import OracleEos
    T, _ = tables
    O = OracleEos(T)
    rng = np.random.default_rng(5)
    t0 = 0.0
    tg, to = t0, t0
    for k in range(50):
        rho0 = 10 ** rng.uniform(-6, 1)
        u = rho0 * 10 ** rng.uniform(-4, 0)
        a, la = dev.batch("pressure", [7], [rho0], [u], [tg])
        b, lb = O.batch("pressure", [7], [rho0], [u], [to])
        assert _same(a, b).all() and _same(la, lb).all(), k
        tg, to = la[0], lb[0]


def test_device_eos_rejects_bad_tables(harm_lib, tables):
    import harm_cool_b200 as hc
    T, _ = tables
    with pytest.raises(hc.HarmError):
        hc.Eos(T.xa[::-1], T.ya, T.val, T.consts)
    e = hc.Eos(T.xa, T.ya, T.val, T.consts)
    with pytest.raises(hc.HarmError):
        e.batch("pressure", [T.ntab], [1.0], [1.0], [0.0])
    e.close()


# mixed precision: tables, Akima windows and the T solve in FP32, against the
# FP64 oracle from the same guesses.  Both solves stop at a residual of 1e-6 in
# e, so the FP64 pressure itself depends on its starting guess at about that
# level; the FP32 pressure is held to 2e-5 relative where both solved from the
# table.
P32_TOL = 2e-5


def test_device_eos_fp32_against_fp64_oracle(dev, tables):
    from oracle.pyoracle import OracleEos
    from golden.make_golden import eos_inputs
    T, _ = tables
    O = OracleEos(T)
    tab, rho0, u, lastT = eos_inputs(np.random.default_rng(21), T.ntab, 50000)
    a, la = dev.batch("pressure", tab, rho0, u, lastT, mixed=True)
    b, lb = O.batch("pressure", tab, rho0, u, lastT)
    gam = T.consts["gam"]
    gl_a = a == (gam - 1.) * u
    gl_b = b == (gam - 1.) * u
    both = ~gl_a & ~gl_b & (u > 0)
    rel = np.abs(a[both] / b[both] - 1.)
    print("FP32 EOS: %d table solves, max rel %.2e, median %.2e; branch agreement %.5f"
          % (both.sum(), rel.max(), np.median(rel), np.mean(gl_a == gl_b)))
    assert both.sum() > 20000
    assert rel.max() <= P32_TOL
    # the fall-backs (outside the table, e < 0) are the FP64 path's, exactly
    out = (rho0 * T.consts["rho_unit"] < T.consts["rho_min"]) | (rho0 * T.consts["rho_unit"] > T.consts["rho_max"])
    assert np.array_equal(a[out], b[out])
    assert np.mean(gl_a == gl_b) > 0.99
    # the temperatures agree to the solve tolerance
    trel = np.abs(la[both] / lb[both] - 1.)
    assert trel.max() <= 1e-4, trel.max()


def test_fp32_refused_for_tables_beyond_float_range(harm_lib, tables):
    """Values spanning more than float's exponent range: the FP64 path still
    serves them, the FP32 path is refused (no silent overflow)."""
    import harm_cool_b200 as hc
    T, _ = tables
    v = T.val.copy()
    v[0, 0, 0, 0] = 1e-300        # e spans far more than 2^240
    e = hc.Eos(T.xa, T.ya, v, T.consts)
    a, _ = e.batch("pressure", [5], [1.0], [1e-2], [0.0])
    assert np.isfinite(a).all()
    with pytest.raises(hc.HarmError):
        e.batch("pressure", [5], [1.0], [1e-2], [0.0], mixed=True)
    e.close()
