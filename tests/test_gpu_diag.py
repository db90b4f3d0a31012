"""GPU: diag()'s integrals and div B on the device, against the oracle and
the reference's printed values.  Each zone's U and |div B| follow the
reference's arithmetic, so divbmax and its zone agree exactly; the sums add up
in another order, within 1e-13 relative."""
import numpy as np
import pytest

from helpers import full_state, load_fixture, make_oracle, problem_from_fixture

pytestmark = pytest.mark.gpu
TOL_SUM = 1e-13


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _agree(g, o):
    for k in ("rmed", "pp", "e"):
        assert abs(g[k] - o[k]) <= TOL_SUM * abs(o[k]), (k, g[k], o[k])
    assert g["divbmax"] == o["divbmax"]
    assert g["imax"] == o["imax"]


@pytest.mark.parametrize("cfg", ["t2d", "t3d"])
def test_diag_matches_reference_print(cfg, hc, oracle_built):
    fx = load_fixture(cfg)
    ref = load_fixture("diag_" + cfg)
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p5"]), full_state(pr, fx["pflag5"]))
    g = ctx.integrals()
    o = make_oracle(pr)
    o.p[...] = full_state(pr, fx["p5"])
    _agree(g, o.diag_integrals())
    assert float("%.5g" % g["rmed"]) == ref["printed"][0]
    assert float("%.6g" % g["divbmax"]) == ref["printed"][3]
    assert g["imax"] == ref["imax"].tolist()


@pytest.mark.parametrize("shape,steps", [((128, 128, 1), 50), ((48, 48, 16), 20)])
def test_diag_follows_oracle_after_steps(shape, steps, hc, oracle_built):
    pr = hc.torus_problem(*shape)
    ctx = hc.Context(pr)
    ctx.init_torus()
    ctx.run(steps)
    p = ctx.get_prims()
    o = make_oracle(pr)
    o.p[...] = p
    _agree(ctx.integrals(), o.diag_integrals())
