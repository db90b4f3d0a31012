"""GPU: the failure paths, without faulting or hanging the GPU.

The reference meets bad zones by failing inversions (repaired by
fixup_utoprim), and ends the run with exit(11) when dt falls below 1e-9
(step_ch.c:126-129).  A torus whose inversions fail in many zones and a dt
set too small on the host drive those paths; the device's handling is
compared with the oracle's: the same flags, the same repaired state bit for
bit, and an error status in place of the exit, after which the context stops
advancing until the host resets its time."""
import numpy as np
import pytest

from helpers import active, make_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _pair(hc, pr, steps=3):
    ctx = hc.Context(pr)
    ctx.init_torus()
    ctx.run(steps)
    p, fl = ctx.get_prims(with_flags=True)
    o = make_oracle(pr)
    o.p[...] = p
    o.pflag[...] = fl
    o.set_time(*ctx.time())
    d = ctx.diag()
    o.set_mass(d["mass_in"], d["mass_out"])
    return ctx, o, p, fl


@pytest.mark.parametrize("shape", [(96, 64, 1), (192, 128, 1)])
def test_failure_heavy_torus_matches_oracle(shape, hc, oracle_built):
    """A torus (a=0.1945, Rmax=9.45, beta=187: one of the seeded ensemble's
    draws) whose inversions fail in many zones every step: the isentropic
    fall-backs, the floors and fixup_utoprim's repairs (wavefronts beyond 512
    failures) must give the oracle's state and flags bit for bit."""
    pr = hc.torus_problem(*shape, a=0.1945427836190702, rmax=9.453765228095609, beta=186.68974421644967)
    ctx, o, p, fl = _pair(hc, pr, steps=2)
    repaired = []
    for _ in range(2):
        ctx.step_ch()
        assert o.step() == 0
        ctx.sync()
        g, gf = ctx.get_prims(with_flags=True)
        np.testing.assert_array_equal(active(pr, g), active(pr, o.p))
        np.testing.assert_array_equal(active(pr, gf), active(pr, o.pflag))
        # after fixup_utoprim the flags read 0 on the zones it repaired
        a = active(pr, gf)[:, 2:-2, 2:-2]
        repaired.append(int((a == 0).sum()))
    assert ctx.diag()["fail_code"] == o.diag()["fail_code"] == 0
    print("repaired zones per step", shape, repaired)
    assert max(repaired) > 0


def test_tiny_dt_stops_the_run_with_an_error(hc, oracle_built):
    """Where the reference calls exit(11) the device records HARM_E_DT and
    later steps do nothing; the host restores the run by setting the time."""
    pr = hc.torus_problem(32, 32, 1)
    ctx, o, p, fl = _pair(hc, pr)
    t, dt = ctx.time()
    ctx.set_time(t, 1e-10)
    o.set_time(t, 1e-10)
    with pytest.raises(hc.HarmError) as e:
        ctx.run(1)
    assert e.value.code == -11
    assert o.step() == 11
    # the step the reference took before exiting, bit for bit
    np.testing.assert_array_equal(active(pr, ctx.get_prims()), active(pr, o.p))
    frozen = ctx.get_prims()
    with pytest.raises(hc.HarmError):
        ctx.run(3)                                 # halted: nothing advances
    np.testing.assert_array_equal(ctx.get_prims(), frozen)
    ctx.set_time(t, dt)                            # the host restarts the clock
    ctx.run(2)
    assert np.any(ctx.get_prims() != frozen)
