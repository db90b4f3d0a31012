"""CPU: the host-side table builder (harm_cool_b200.eos_tables) lays out the
reference's table grid and HdFac (SetupCache_CoolEOS, cooleos.c:825-992) exactly
as the reference's code computes them, and its synthetic generator agrees with
the checker build's stand-in (oracle/eos_standin.c) to rounding."""
import numpy as np

import harm_cool_b200 as hc
from harm_cool_b200 import eos_tables


def test_axes_hdfac_and_constants_match_the_reference_layout(oracle_built):
    from oracle.pyoracle import standin_tables
    pr = hc.torus_problem(32, 32, 1, a=0.6, rin=4.0, rmax=11.8, beta=50.0)
    xa, ya, val, c = eos_tables.build_tables(eos_tables.zone_radii(pr), gam=pr.params.gam)
    S = standin_tables(pr.params.startx[1], pr.params.dx[1], pr.grid.R0, pr.params.n1 + 4, pr.params.gam)
    assert np.array_equal(xa, S.xa) and np.array_equal(ya, S.ya)
    assert np.array_equal(c["hdfac"], S.consts["hdfac"])
    for k in hc.EOS_CONSTANTS + ("l_unit",):
        assert c[k] == S.consts[k], k
    # the same ideal gas plus radiation, formed in numpy instead of C
    np.testing.assert_allclose(val, S.val, rtol=1e-14, atol=0)


def test_table_shape_and_ranges():
    radii = np.array([3.0, 5.0, 8.0])
    xa, ya, val, c = eos_tables.build_tables(radii, nx=20, ny=30, rho=(1e4, 1e14), T=(1e8, 1e12))
    assert val.shape == (3, 20, 30, 5)
    assert xa[0] == 1e4 and abs(xa[-1] / 1e14 - 1) < 1e-12
    assert ya[0] == 1e8 and abs(ya[-1] / 1e12 - 1) < 1e-12
    assert np.all(np.diff(xa) > 0) and np.all(np.diff(ya) > 0)
    assert np.all(val[..., 0] > 0) and np.all(val[..., 1] > 0)
    np.testing.assert_allclose(val[..., 4], 0.5)          # Yee of the stand-in
    assert c["rho_min"] == 1e4 and c["t_max"] == 1e12


def test_on_demand_loop_fills_what_the_run_reads():
    """eos_tables.on_demand with a stand-in table object and filler: a run that
    reads a chain of nodes, each revealed only once the previous one holds a
    value (as a temperature solve walks the table), is repeated until it reads
    no NaN; each pass computes the nodes read as NaN and a margin around them,
    no node twice, and the last run is returned."""
    import numpy as np
    xa, ya = np.arange(10.), np.arange(12.)
    consts = {"hdfac": np.ones(2)}
    path = [(0, 2, 3), (0, 5, 3), (1, 5, 9), (1, 8, 1)]
    filled = []

    class FakeEos:
        def __init__(self, xa, ya, val, consts):
            self.val = val.copy()
            self.marks = np.zeros(val.shape[:3], dtype=bool)

        def track_missing(self):
            pass

        def missing(self):
            return self.marks

        def close(self):
            pass

    def run(eos):
        # walk the path until the first node that is not computed yet
        for t, i, j in path:
            if np.isnan(eos.val[t, i, j, 0]):
                eos.marks[t, i, j] = True
                return "stopped"
        return "complete"

    def fill(val, xa, ya, hd, mask, device):
        val[mask] = 1.0
        filled.append(int(mask.sum()))
        return int(mask.sum()), 0.0

    result, info, have = eos_tables.on_demand(run, xa, ya, consts, margin=1, make_eos=FakeEos, fill=fill)
    assert result == "complete"
    assert info["passes"] == len(path) + 1 and info["nodes"] == sum(filled) == have.sum()
    for t, i, j in path:
        assert have[t, i, j]
    # margin 1: the cross around each node, within the table
    assert have[0, 1:4, 3].all() and have[0, 2, 2:5].all() and not have[0, 0, 0]
