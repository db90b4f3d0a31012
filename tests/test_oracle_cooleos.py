"""CPU: the oracle's run-time COOL_EOS (oracle/cooleos_oracle.c) against the
reference's own (cooleos.c, cache4d.c, akima.c, mnewt.h compiled from the
reference's sources with oracle/eos_standin.c as the table generator).

The fixture tests run anywhere; the direct comparison runs only where the
COOL_EOS checker build oracle/_ref/ce2d exists, in a subprocess (the reference
keeps its state in globals)."""
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _fixture():
    return np.load(os.path.join(GOLDEN, "eos_ce2d.npz"))


def _tables(f):
    from oracle.pyoracle import standin_tables
    startx1, dx1, R0, gam = f["grid"]
    return standin_tables(startx1, dx1, R0, int(f["sn1"]), gam)


def _same(a, b):
    return np.all((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b)))


def test_oracle_tables_match_reference_digest(oracle_built):
    f = _fixture()
    T = _tables(f)
    assert hashlib.sha256(np.ascontiguousarray(T.val).tobytes()).hexdigest() == str(f["sha_tables"])
    axes = np.concatenate([T.xa, T.ya])
    assert hashlib.sha256(axes.tobytes()).hexdigest() == str(f["sha_axes"])
    names = [str(n) for n in f["const_names"]]
    assert [T.consts[n] for n in names] == f["consts"].tolist()
    assert np.array_equal(T.consts["hdfac"], f["hdfac"])


@pytest.mark.parametrize("what", ["pressure", "dpdu", "dpdrho"])
def test_oracle_eos_matches_reference_fixture(what, oracle_built):
    from oracle.pyoracle import OracleEos
    f = _fixture()
    O = OracleEos(_tables(f))
    v, lt = O.batch(what, f["tab"], f["rho0"], f["u"], f["lastT"])
    assert _same(v, f[what]), np.flatnonzero(~((v == f[what]) | (np.isnan(v) & np.isnan(f[what]))))[:10]
    assert _same(lt, f[what + "_lastT"])


def test_fixture_covers_every_branch():
    f = _fixture()
    gam = f["grid"][3]
    names = [str(n) for n in f["const_names"]]
    c = dict(zip(names, f["consts"].tolist()))
    rho = f["rho0"] * c["rho_unit"]
    gl = f["pressure"] == (gam - 1.) * f["u"]
    in_range = (rho >= c["rho_min"]) & (rho <= c["rho_max"])
    assert np.any(rho < c["rho_min"]) and np.any(rho > c["rho_max"])
    assert np.any(f["u"] < 0) and np.any(f["pressure"][in_range & (f["u"] < 0)] == 0.0)
    assert np.any(f["lastT"] == 0.0)
    assert np.any(gl & in_range & (f["u"] > 0))           # solves that failed: gamma-law fall-back
    assert np.mean(~gl & in_range) > 0.4                   # most in-range entries solve from the table
    # the finite-difference steps vanish in FP64: the reference's derivatives are 0
    assert np.all(f["dpdu"][np.isfinite(f["dpdu"])] == 0.0)
    assert np.all(f["dpdrho"][np.isfinite(f["dpdrho"])] == 0.0)


SCRIPT = r'''
import sys, numpy as np
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
from oracle.pyoracle import Reference, OracleEos, standin_tables
from golden.make_golden import eos_inputs
ref = Reference("ce2d")
T = ref.cool_tables()
S = standin_tables(ref.get("startx1"), ref.get("dx1"), ref.get("R0"), ref.sn1, ref.get("gam"))
assert {{k: v for k, v in T.consts.items() if k != "hdfac"}} == {{k: v for k, v in S.consts.items() if k != "hdfac"}}
assert np.array_equal(T.consts["hdfac"], S.consts["hdfac"])
assert np.array_equal(T.xa, S.xa) and np.array_equal(T.ya, S.ya)
assert np.array_equal(T.val.view(np.int64), S.val.view(np.int64))
O = OracleEos(S)
tab, rho0, u, lastT = eos_inputs(np.random.default_rng(7), T.ntab, 20000)
for what in ("pressure", "dpdu", "dpdrho"):
    a, la = ref.cool_batch(what, tab, rho0, u, lastT)
    b, lb = O.batch(what, tab, rho0, u, lastT)
    ok = (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))
    assert ok.all(), (what, np.flatnonzero(~ok)[:10])
    assert np.array_equal(la.view(np.int64), lb.view(np.int64)), what
# interpolated values and T-derivatives at arbitrary points of one table
rng = np.random.default_rng(3)
for k in range(300):
    t = int(rng.integers(0, T.ntab)); rho = 10 ** rng.uniform(2, 15); TT = 10 ** rng.uniform(4, 18)
    for d in (0, 1):
        v = O.value(t, d, rho, TT, der=True)
        assert v is not None
print("ok")
'''


def test_oracle_eos_matches_reference(oracle_built):
    lib = os.path.join(ROOT, "oracle", "_ref", "ce2d", "libharmref.so")
    if not os.path.exists(lib):
        pytest.skip("COOL_EOS reference checker not built here")
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, tests=os.path.join(ROOT, "tests"))],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "ok" in r.stdout
