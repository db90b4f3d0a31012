"""GPU: restart files in the reference's format, against files written by the
reference's own restart_write() (tests/golden/restart_<config>.npz, after 5
steps).  Written from the device, the file matches the reference's text
byte for byte, except where the reference prints uninitialised stat() sizes
(ener.out's and each tracer file's) and, in 3D, the phi ghost planes, which
hold stale copies in the reference and periodic copies here.  Read into the
device, the reference's file gives back its state exactly."""
import os

import numpy as np
import pytest

from helpers import full_state, load_fixture, problem_from_fixture

pytestmark = pytest.mark.gpu
HEADER = ("n1", "n2", "n3", "t", "tf", "nstep", "a", "gam", "cour", "DTd", "DTl", "DTi", "DTr", "dump_cnt",
          "image_cnt", "rdump_cnt", "dt", "lim", "failed", "Rin", "Rout", "hslope", "R0", "mass_start",
          "mass_in", "mass_out", "tdump", "timage", "tlog", "defcon", "nfailed", "Rbr", "cyl_R0", "cyl_Th0")
INTS = {"n1", "n2", "n3", "nstep", "DTr", "dump_cnt", "image_cnt", "rdump_cnt", "lim", "failed", "nfailed"}


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


def _ref_text(cfg):
    return load_fixture("restart_" + cfg)["text"].tobytes().decode()


def _header_fields(text):
    vals = text.split("\n")[0].split()
    return {k: (int(v) if k in INTS else float(v)) for k, v in zip(HEADER, vals)}


def _context(hc, cfg):
    """The reference's state after 5 steps, on the device."""
    fx = load_fixture("tracers_" + cfg if cfg.startswith("r") else cfg)
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p5"]), full_state(pr, fx["pflag5"]))
    ctx.set_time(*fx["t5"])
    return fx, pr, ctx


def test_restart_write_matches_reference_2d_with_tracers(hc, tmp_path):
    ref = _ref_text("r2d")
    fx, pr, ctx = _context(hc, "r2d")
    ctx.set_mass(*fx["mass5"])
    ctx.tracers_put(fx["tr_ids5"], fx["tr_X5"])
    h = _header_fields(ref)
    body_end = ref.rstrip().split("\n")[-1]       # the line with ener.out's size and the tracers
    ener_size = int(body_end.split()[0])
    fields = {k: v for k, v in h.items() if k not in ("n1", "n2", "n3", "t", "dt", "mass_in", "mass_out")}
    path = str(tmp_path / "rdump")
    ctx.restart_write(path, ener_size=ener_size, **fields)
    ours = open(path).read()
    a, b = ours.split("\n"), ref.split("\n")
    assert len(a) == len(b)
    assert a[:-1] == b[:-1]                       # header and every cell, byte for byte
    # last line: ener.out size, tracer radii, count, then per tracer i j h X0..X3 size
    ta, tb = a[-1].split(), b[-1].split()
    assert len(ta) == len(tb)
    per = 8
    n = int(tb[9])
    assert ta[1:10] == tb[1:10]
    for k in range(n):
        ra, rb = ta[10 + per * k:10 + per * (k + 1)], tb[10 + per * k:10 + per * (k + 1)]
        assert ra[:7] == rb[:7], k                # labels and X; the size field is a stat() result


def test_restart_write_matches_reference_3d(hc, tmp_path):
    ref = _ref_text("t3d")
    fx, pr, ctx = _context(hc, "t3d")
    ctx.set_mass(*fx["diag5"][6:8])
    h = _header_fields(ref)
    fields = {k: v for k, v in h.items() if k not in ("n1", "n2", "n3", "t", "dt", "mass_in", "mass_out")}
    path = str(tmp_path / "rdump")
    ctx.restart_write(path, ener_size=int(ref.rstrip().split("\n")[-1].split()[0]), **fields)
    ours = open(path).read().split("\n")
    refl = ref.split("\n")
    assert ours[0] == refl[0]
    sn3, sn1, sn2 = pr.shape
    cells = np.arange(sn3 * sn1 * sn2).reshape(pr.shape)
    for c in cells[1:-1].ravel():                 # the active phi planes, every r and theta cell
        assert ours[1 + c] == refl[1 + c], c


@pytest.mark.parametrize("cfg", ["r2d", "t3d"])
def test_restart_read_gives_the_reference_state(cfg, hc, tmp_path):
    ref = _ref_text(cfg)
    path = tmp_path / "rdump"
    path.write_text(ref)
    fx = load_fixture("tracers_" + cfg if cfg.startswith("r") else cfg)
    pr = problem_from_fixture(fx)
    ctx = hc.Context(pr)
    ctx.init_torus()                              # something else in the context first
    hd = ctx.restart_read(str(path))
    p = ctx.get_prims()
    act = slice(1, -1) if pr.params.n3 > 1 else slice(None)
    np.testing.assert_array_equal(p[act], fx["p5"])
    assert ctx.time() == (fx["t5"][0], fx["t5"][1])
    assert hd["nstep"] == 5
    if cfg.startswith("r"):
        ids, X, st = ctx.tracers()
        np.testing.assert_array_equal(ids, fx["tr_ids5"])
        np.testing.assert_array_equal(X, fx["tr_X5"])
        assert np.all(st == 0)
    # and the run continues from there exactly as the reference's uninterrupted run did
    if cfg == "r2d":
        ctx.run(1)
        np.testing.assert_array_equal(ctx.get_prims()[act], fx["p6"])
