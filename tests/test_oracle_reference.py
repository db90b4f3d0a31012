"""CPU: the oracle against the reference's own step_ch() compiled from its sources.

Runs only where oracle/_ref was built (the container that has the reference
tree).  Each configuration runs in a subprocess: the reference keeps its
state in globals."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import sys, numpy as np
sys.path.insert(0, {root!r})
from oracle.pyoracle import Reference, Oracle
ref = Reference({cfg!r})
if {lim!r} is not None:
    ref.set("lim", {lim!r})
o = Oracle(ref.params(), ref.geometry())
o.p[...] = ref.p; o.pflag[...] = ref.pflag
o.set_time(ref.get("t"), ref.get("dt"))
hs = slice(1, ref.n3 + 1) if ref.n3 > 1 else slice(0, 1)
for s in range({steps}):
    ref.step(); assert o.step() == 0
    assert np.array_equal(ref.p[hs], o.p[hs]), s
    assert np.array_equal(ref.pflag[hs], o.pflag[hs]), s
    assert o.time() == (ref.get("t"), ref.get("dt")), s
    d = o.diag()
    assert d["fail_code"] == 0
    for k in ("mdot", "edot", "ldot", "mass_curr", "mass_in", "mass_out"):
        assert d[k] == ref.get(k), (s, k)
print("ok")
'''


@pytest.mark.parametrize("cfg,steps,lim", [
    ("c1", 40, None), ("m3d", 8, None),
    # the 288x256 r-theta grid of the 288x256x256 benchmark, 4 phi planes
    ("c2s", 2, None),
    # van Leer and minmod slopes (interp.c:71-87), set at run time as init.c sets lim
    ("c1", 20, 1), ("c1", 20, 2)])
def test_oracle_matches_reference(cfg, steps, lim, oracle_built):
    lib = os.path.join(ROOT, "oracle", "_ref", cfg, "libharmref.so")
    if not os.path.exists(lib):
        pytest.skip("reference checker not built here")
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, cfg=cfg, steps=steps, lim=lim)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "ok" in r.stdout
