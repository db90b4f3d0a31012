"""GPU: tracer particles (tracers.c) against the reference's own tracer lists
and against the oracle.

Tracer positions follow the reference's arithmetic (the kernels are built with
-fmad=false), so the comparisons are bit for bit.  The reference erases
retired tracers; the device keeps them with a status, so the fixture
comparisons are over the active tracers, and the statuses are compared with
the oracle, which keeps them the same way."""
import numpy as np
import pytest

from helpers import full_state, load_fixture, make_oracle, problem_from_fixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _as_dict(ids, X):
    return {tuple(i): x for i, x in zip(ids.tolist(), X)}


def _same_active(ids, X, st, ids_ref, X_ref):
    m = st == 0
    a, b = _as_dict(ids[m], X[m]), _as_dict(ids_ref, X_ref)
    assert set(a) == set(b), (len(a), len(b))
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=str(k))


@pytest.mark.parametrize("cfg", ["r2d", "r3d"])
def test_tracers_match_reference(cfg, hc, oracle_built):
    fx = load_fixture("tracers_" + cfg)
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p0"]), full_state(pr, fx["pflag0"]))
    ctx.set_time(*fx["t0"])
    o = make_oracle(pr)
    o.p[...] = full_state(pr, fx["p0"])
    o.pflag[...] = full_state(pr, fx["pflag0"])
    o.set_time(*fx["t0"])
    R0, hslope = float(fx["par_R0"]), float(fx["par_hslope"])
    n = ctx.tracers_init()
    o.tracers_init(R0, hslope)
    ids, X, st = ctx.tracers()
    assert n == len(fx["tr_ids0"])
    np.testing.assert_array_equal(ids, fx["tr_ids0"])   # same loop order as init_tracers()
    np.testing.assert_array_equal(X, fx["tr_X0"])
    done = 0
    for step in (1, 2, 5, 6, 10, 30):
        while done < step:
            ctx.step_ch()
            assert o.step() == 0
            done += 1
            if done == 5:
                ctx.sync()
                _same_active(*ctx.tracers(), fx["tr_ids5"], fx["tr_X5"])
                ctx.tracers_put(fx["cu_ids"], fx["cu_X"])
                o.tracers_put(fx["cu_ids"], fx["cu_X"], R0, hslope)
        ctx.sync()
        ids, X, st = ctx.tracers()
        if step < 5:
            _same_active(ids, X, st, fx["tr_ids%d" % step], fx["tr_X%d" % step])
        elif step > 5:
            _same_active(ids, X, st, fx["cu_ids%d" % step], fx["cu_X%d" % step])
            oi, oX, ost = o.tracers()
            np.testing.assert_array_equal(ids, oi)
            np.testing.assert_array_equal(st, ost)
            np.testing.assert_array_equal(X, oX)
    assert ctx.diag()["fail_code"] == 0


def test_tracers_128x128_follow_oracle(hc, oracle_built):
    pr = hc.torus_problem(128, 128, 1)
    ctx = hc.Context(pr)
    ctx.init_torus()
    p0, f0 = ctx.get_prims(with_flags=True)
    o = make_oracle(pr)
    o.p[...] = p0
    o.pflag[...] = f0
    o.set_time(*ctx.time())
    n = ctx.tracers_init()
    assert n == o.tracers_init(pr.grid.R0, pr.grid.hslope)
    assert n > 1000
    X_init = ctx.tracers()[1]
    ctx.run(60)                     # graph replay with the tracer kernel in it
    for _ in range(60):
        assert o.step() == 0
    ids, X, st = ctx.tracers()
    oi, oX, ost = o.tracers()
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(st, ost)
    np.testing.assert_array_equal(X, oX)
    # the tracers did move
    assert (st == 0).sum() > 0
    assert np.abs(X[st == 0] - X_init[st == 0]).max() > 1e-3
