"""CPU: the oracle's tracer restatement against the reference's own tracers.c.

The fixtures in tests/golden/tracers_<config>.npz hold the tracer list of the
reference compiled from its sources (TRACERSDUMP on): after init_tracers(),
after 1, 2 and 5 steps, and for a seeded custom list (tracers near the inner
radius, beyond the outer tracer radius, outside the grid) carried from step 5
to step 30.  The reference erases retired tracers from its list; the oracle
keeps them with a status, so the comparison is over the active ones."""
import numpy as np
import pytest

from helpers import load_fixture, make_oracle, full_state, problem_from_fixture


def _active(ids, X, st):
    m = st == 0
    return ids[m], X[m]


def _as_dict(ids, X):
    return {tuple(i): x for i, x in zip(ids.tolist(), X)}


def _same(ids_a, X_a, ids_b, X_b):
    a, b = _as_dict(ids_a, X_a), _as_dict(ids_b, X_b)
    assert set(a) == set(b), (len(a), len(b), sorted(set(a) ^ set(b))[:5])
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=str(k))


@pytest.mark.parametrize("cfg", ["r2d", "r3d"])
def test_oracle_tracers_match_reference(cfg, oracle_built, harm_lib):
    fx = load_fixture("tracers_" + cfg)
    pr = problem_from_fixture(fx)
    o = make_oracle(pr)
    o.p[...] = full_state(pr, fx["p0"])
    o.pflag[...] = full_state(pr, fx["pflag0"])
    o.set_time(*fx["t0"])
    R0, hslope = float(fx["par_R0"]), float(fx["par_hslope"])
    n = o.tracers_init(R0, hslope)
    ids, X, st = o.tracers()
    assert n == len(fx["tr_ids0"])
    _same(ids, X, fx["tr_ids0"], fx["tr_X0"])
    done = 0
    for step in (1, 2, 5, 6, 10, 30):
        while done < step:
            assert o.step() == 0
            done += 1
            if done == 5:
                _same(*_active(*o.tracers()), fx["tr_ids5"], fx["tr_X5"])
                o.tracers_put(fx["cu_ids"], fx["cu_X"], R0, hslope)
        if step < 5:
            _same(*_active(*o.tracers()), fx["tr_ids%d" % step], fx["tr_X%d" % step])
        elif step > 5:
            _same(*_active(*o.tracers()), fx["cu_ids%d" % step], fx["cu_X%d" % step])
    ids, X, st = o.tracers()
    # the custom list exercises the retirements: dropped, fell in, left (and in 3D the jet)
    kinds = set(st.tolist())
    assert {-1, 0, 1, 2} <= kinds, kinds
    if pr.params.n3 > 1:
        assert 3 in kinds, kinds
