"""GPU: the ASCII dump (dump() with HDFDUMP 0, dump.c:1710-2047) written from the
device state against the reference's own dump of the same state: the header
line, and every zone line through its sha256 (tests/golden/dump_*.npz,
cool_ce2d.npz).  Zone lines hold the coordinates, primitives, cooling values,
div B, the four-vectors, wave speeds, sqrt(-g), |v| and the gamma = 4/3 sound
speed, radial velocity and Mach number, all printed with %32.22e, so equal
digests mean the same values bit for bit."""
import hashlib

import numpy as np
import pytest

from helpers import full_state, load_fixture, problem_from_fixture

pytestmark = pytest.mark.gpu
FIELDS = ("t", "N1", "N23", "startx1", "startx23", "dx1", "dx23", "tf", "nstep", "a", "gam", "cour", "DTd", "DTl",
          "DTi", "DTr", "dump_cnt", "image_cnt", "rdump_cnt", "dt", "lim", "failed", "Rin", "Rout", "hslope", "R0")
INTS = {"N1", "N23", "nstep", "DTr", "dump_cnt", "image_cnt", "rdump_cnt", "lim", "failed"}
OWNED = {"t", "N1", "N23", "startx1", "startx23", "dx1", "dx23", "dt"}   # the context's own


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _fields(header):
    vals = header.split()
    return {k: (int(v) if k in INTS else float(v)) for k, v in zip(FIELDS, vals) if k not in OWNED}


def _check(path, header, sha):
    lines = open(path).read().split("\n")
    assert lines[-1] == ""
    assert lines[0] == header
    zl = lines[1:-1]
    assert len(zl) == len(sha)
    bad = [k for k, l in enumerate(zl) if hashlib.sha256(l.encode()).hexdigest() != sha[k]]
    assert not bad, (len(bad), bad[:5], zl[bad[0]][:300])


@pytest.mark.parametrize("cfg", ["t2d", "t3d"])
def test_dump_matches_reference(cfg, hc, tmp_path):
    fx = load_fixture(cfg)
    dm = load_fixture("dump_" + cfg)
    header = dm["header"].tobytes().decode()
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p5"]), full_state(pr, fx["pflag5"]))
    ctx.set_time(*fx["t5"])
    path = str(tmp_path / "dump")
    ctx.dump_write(path, **_fields(header))
    _check(path, header, dm["sha"])
    ctx.close()


@pytest.mark.parametrize("cfg", ["ce2d", "ce3d"])
def test_cool_dump_matches_reference(cfg, hc, tmp_path, oracle_built):
    from oracle.pyoracle import standin_tables
    fx = load_fixture("cool_" + cfg)
    T = standin_tables(float(fx["par_startx1"]), float(fx["par_dx1"]), float(fx["par_R0"]), int(fx["n"][0]) + 4,
                       float(fx["par_gam"]))
    eos = hc.Eos(T.xa, T.ya, T.val, T.consts)
    header = fx["dump_header"].tobytes().decode()
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.set_eos(eos)
    ctx.put_prims(full_state(pr, fx["p12"]), full_state(pr, fx["pflag12"]))
    ctx.set_time(*fx["t12"])
    ctx.put_eos_guess(fx["lastT_after_diag"])
    path = str(tmp_path / "dump")
    ctx.dump_write(path, **_fields(header))
    _check(path, header, fx["dump_sha"])
    g = ctx.eos_guess()
    assert np.array_equal(g.view(np.int64), fx["lastT_after_dump"].view(np.int64))
    ctx.close()
    eos.close()
