"""The drop-in: the reference's own host program (main.c's init path, init.c,
diag.c, ...) with harm_cool_b200/shim/harm_gpu.cpp linked in place of
step_ch.c, bounds.c, fixup.c and utoprim_2d.c, so that its step_ch(),
bound_prim(), fixup(), set_Katm() and Utoprim_2d() run on the GPU.  The state
after init() (whose fixup()/bound_prim() calls go to the GPU too) and after 1,
2 and 5 step_ch() calls must equal the reference's CPU run bit for bit
(tests/golden/t2d.npz, t3d.npz, made from the unmodified reference); the
mass diagnostic, a sum over the grid, to 1e-13."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu

SCRIPT = r'''
import sys, numpy as np
sys.path.insert(0, {root!r})
from oracle.pyoracle import Reference
fx = dict(np.load({fixture!r}))
ref = Reference({cfg!r})
hs = slice(1, ref.n3 + 1) if ref.n3 > 1 else slice(0, 1)
assert np.array_equal(ref.p[hs], fx["p0"]), "after init()"
assert np.array_equal(ref.pflag[hs], fx["pflag0"]), "pflag after init()"
assert (ref.get("t"), ref.get("dt")) == tuple(fx["t0"])
done = 0
for n in (1, 2, 5):
    while done < n:
        ref.step()
        done += 1
    assert np.array_equal(ref.p[hs], fx["p%d" % n]), n
    assert np.array_equal(ref.pflag[hs], fx["pflag%d" % n]), n
    assert (ref.get("t"), ref.get("dt")) == tuple(fx["t%d" % n]), n
    # a sum over the grid, added in another order on the device
    assert abs(ref.get("mass_curr") - fx["diag%d" % n][5]) <= 1e-13 * abs(fx["diag%d" % n][5]), n
if ref.n3 == 1:
    # Utoprim_2d() through the shim on the reference's known answers
    kat = dict(np.load({kat!r}))
    for U, (i, j), guess, r, want in zip(kat["U"], kat["ij"], kat["guess"], kat["ret_2d"], kat["prim_2d"]):
        pr = guess.copy()
        got = ref.lib.ref_utoprim_2d(U.ctypes.data_as(ref_dp), int(i), int(j), pr.ctypes.data_as(ref_dp))
        assert got == r
        if r == 0:
            assert np.array_equal(pr, want), (i, j)
print("ok")
'''


@pytest.mark.parametrize("cfg,fixture", [("g2d", "t2d"), ("g3d", "t3d")])
def test_reference_host_steps_through_the_shim(cfg, fixture, harm_lib):
    lib = os.path.join(ROOT, "oracle", "_ref", cfg, "libharmref.so")
    if not os.path.exists(lib):
        pytest.skip("drop-in build not made here (needs the reference tree)")
    script = SCRIPT.format(root=ROOT, cfg=cfg, fixture=os.path.join(ROOT, "tests", "golden", fixture + ".npz"),
                           kat=os.path.join(ROOT, "tests", "golden", "kat_u2p.npz"))
    script = script.replace("ref_dp", "__import__('ctypes').POINTER(__import__('ctypes').c_double)")
    r = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "ok" in r.stdout
