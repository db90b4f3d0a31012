"""CPU: the oracle's restatement of diag()'s integrals against the reference.

The reference prints the integrals with 5 significant digits (ener.out,
diag.c:317) and divbmax with 6 (the LOG line, diag.c:314); the zone of
divbmax is printed exactly.  Fixtures: tests/golden/diag_<config>.npz, from
diag(INIT_OUT) on the state after 5 steps (the p5 of <config>.npz)."""
import numpy as np
import pytest

from helpers import full_state, load_fixture, make_oracle, problem_from_fixture


def printed(x, digits):
    return float("%.*g" % (digits, x))


@pytest.mark.parametrize("cfg", ["t2d", "t3d"])
def test_oracle_diag_matches_reference(cfg, oracle_built, harm_lib):
    fx = load_fixture(cfg)
    ref = load_fixture("diag_" + cfg)
    pr = problem_from_fixture(fx)
    o = make_oracle(pr)
    o.p[...] = full_state(pr, fx["p5"])
    d = o.diag_integrals()
    rmed, pp, e, divbmax = ref["printed"]
    assert printed(d["rmed"], 5) == rmed
    assert printed(d["pp"], 5) == pp
    assert printed(d["e"], 5) == e
    assert printed(d["divbmax"], 6) == divbmax
    assert d["imax"] == ref["imax"].tolist()
