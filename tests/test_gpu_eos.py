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
