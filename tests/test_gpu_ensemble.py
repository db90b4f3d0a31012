"""GPU: ensembles of independent tori, tile shapes and the tile autotuner.

An ensemble step must advance every member exactly as a step of that member
alone would: the members' step sequences are parallel branches of one CUDA
graph and share no data, and a zone's arithmetic does not depend on the tile
shape.  So every comparison here is bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _members(hc, seed):
    probs = [p for p, _ in hc.ensemble_problems(5, seed=seed, sizes=(32, 48, 64))]
    probs.append(hc.torus_problem(16, 16, 4, a=0.5, rmax=11.0, beta=50.0))   # a 3D member too
    return probs


def _fresh(hc, pr, mixed=False, tile=None):
    c = hc.Context(pr)
    c.init_torus()
    if mixed:
        c.set_precision(hc.Context.MIXED)
    if tile:
        c.set_tile(*tile)
    return c


@pytest.mark.parametrize("mixed", [False, True])
def test_ensemble_step_equals_solo_steps(hc, mixed):
    probs = _members(hc, seed=3)
    tiles = [None, (64, 2), (16, 8), None, (128, 1), None]
    ens_ctx = [_fresh(hc, pr, mixed, t) for pr, t in zip(probs, tiles)]
    ens = hc.Ensemble(ens_ctx)
    ens.run(40)
    for pr, t, ce in zip(probs, tiles, ens_ctx):
        solo = _fresh(hc, pr, mixed, t)
        solo.run(40)
        a, fa = ce.get_prims(with_flags=True)
        b, fb = solo.get_prims(with_flags=True)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(fa, fb)
        assert ce.time() == solo.time()
        assert ce.diag()["fail_code"] == 0
        solo.close()
    # members keep their own dt: once the Courant limit binds (after the
    # initial ramp of 1.3x per step), differently sized grids step differently
    assert len({c.time()[1] for c in ens_ctx}) > 1
    # a member changed after binding is re-captured at the next run
    ens_ctx[0].set_tile(64, 2)
    ens.run(2)
    ens.close()


def test_tile_shape_does_not_change_results(hc):
    pr = hc.torus_problem(40, 36, 4)
    ref = _fresh(hc, pr)
    ref.run(5)
    for tile in [(64, 2), (16, 8), (128, 1), (8, 16)]:
        c = _fresh(hc, pr, tile=tile)
        c.run(5)
        np.testing.assert_array_equal(c.get_prims(), ref.get_prims())
        assert c.time() == ref.time()
        c.close()


def test_autotune_keeps_the_state(hc):
    pr = hc.torus_problem(64, 64, 1)
    c = _fresh(hc, pr)
    c.run(3)
    p0, f0 = c.get_prims(with_flags=True)
    t0 = c.time()
    d0 = c.diag()
    tile = c.autotune_tile(steps=2)
    assert tile in [(32, 4), (64, 2), (16, 8), (128, 1)]
    assert c.tile() == tile
    p1, f1 = c.get_prims(with_flags=True)
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(f0, f1)
    assert c.time() == t0
    assert c.diag()["mass_in"] == d0["mass_in"]
    # and the run continues exactly as an untuned one
    other = _fresh(hc, pr)
    other.run(5)
    c.run(2)
    np.testing.assert_array_equal(c.get_prims(), other.get_prims())
