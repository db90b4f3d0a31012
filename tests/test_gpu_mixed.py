"""GPU: the mixed-precision step against the FP64 step on the same torus.

The mixed path evaluates the face reconstruction, face states, wave speeds and
Lax-Friedrichs fluxes in FP32 and keeps the connection source, the flux
divergence, the accumulation of U, the Noble inversion and the floors in
FP64.  Its contract is a density L1 error of at most 1e-4 (relative to the
mean |rho|) after 1000 steps against FP64; the L1 errors of u, the
velocities and the fields are printed beside it.  The FP64 GPU path is itself
bit-identical to the oracle (test_gpu_parity), so it stands in for the oracle
over runs too long for the CPU."""
import numpy as np
import pytest

from helpers import NAMES, active, l1_groups, l1_rel, make_oracle

pytestmark = pytest.mark.gpu
L1_RHO_1000 = 1e-4


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _pair(hc, pr):
    a = hc.Context(pr)
    a.init_torus()
    b = hc.Context(pr)
    b.init_torus()
    b.set_precision(hc.Context.MIXED)
    return a, b


def _report(tag, l1, grouped=None):
    print(tag, " ".join("%s=%.3e" % (n, v) for n, v in zip(NAMES, l1)))
    if grouped:
        print("    grouped:", " ".join("%s=%.3e" % kv for kv in grouped.items()))


def test_mixed_2d_1000_steps_density_l1(hc):
    pr = hc.torus_problem(128, 128, 1)
    a, b = _pair(hc, pr)
    done = 0
    for n in (1, 100, 1000):
        a.run(n - done)
        b.run(n - done)
        done = n
        pa, pb = active(pr, a.get_prims()), active(pr, b.get_prims())
        assert np.all(np.isfinite(pb))
        l1 = l1_rel(pb, pa)
        _report("mixed vs FP64, 128x128, %d steps:" % n, l1, l1_groups(pb, pa))
    assert l1[0] <= L1_RHO_1000, l1
    assert b.diag()["fail_code"] == 0
    # the same number of steps advances the same simulated time to FP32 accuracy
    ta, tb = a.time()[0], b.time()[0]
    assert abs(ta - tb) <= 1e-4 * ta, (ta, tb)
    a.close()
    b.close()


def test_mixed_3d_steps_track_fp64(hc):
    pr = hc.torus_problem(48, 48, 16)
    a, b = _pair(hc, pr)
    a.run(200)
    b.run(200)
    pa, pb = active(pr, a.get_prims()), active(pr, b.get_prims())
    l1 = l1_rel(pb, pa)
    _report("mixed vs FP64, 48x48x16, 200 steps:", l1, l1_groups(pb, pa))
    assert l1[0] <= L1_RHO_1000, l1
    assert b.diag()["fail_code"] == 0


def test_mixed_one_step_against_oracle(hc, oracle_built):
    """One mixed step from the same state as the oracle's FP64 step: the
    per-step error of the FP32 face fluxes, at FP32 round-off scale."""
    pr = hc.torus_problem(64, 64, 1)
    ctx = hc.Context(pr)
    ctx.init_torus()
    p0, f0 = ctx.get_prims(with_flags=True)
    o = make_oracle(pr)
    o.p[...] = p0
    o.pflag[...] = f0
    o.set_time(*ctx.time())
    ctx.set_precision(hc.Context.MIXED)
    ctx.run(1)
    assert o.step() == 0
    g = active(pr, ctx.get_prims())
    c = active(pr, o.p)
    l1 = l1_rel(g, c)
    _report("mixed vs oracle, 64x64, 1 step:", l1)
    assert l1[0] <= 1e-6, l1
