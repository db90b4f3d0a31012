"""GPU: the COOL_EOS step (step_ch() with the run-time EOS and Utoprim_5d)
against the reference's own COOL_EOS build, through tests/golden/cool_ce2d.npz.

The reference's loops visit zones one after another and each zone's EOS calls
continue from the temperature guess its previous call left; the device keeps
that chain per zone (and seeds the first step row by row), so the FP64 result
is expected bit for bit: primitives, flags, t, dt and the guesses.  The tables
are the ones the reference's build makes (oracle/eos_standin.c in place of its
Fortran generator), rebuilt by the oracle and checked against the reference's
digest in test_oracle_cooleos."""
import numpy as np
import pytest

from helpers import active, full_state, load_fixture, problem_from_fixture

pytestmark = pytest.mark.gpu
STEPS = (1, 2, 5, 12)


@pytest.fixture(scope="module")
def hc(harm_lib):
    import harm_cool_b200
    return harm_cool_b200


@pytest.fixture(scope="module", params=["ce2d", "ce3d"])
def fx(request):
    return load_fixture("cool_" + request.param)


@pytest.fixture(scope="module")
def eos(hc, fx, oracle_built):
    from oracle.pyoracle import standin_tables
    T = standin_tables(float(fx["par_startx1"]), float(fx["par_dx1"]), float(fx["par_R0"]),
                       int(fx["n"][0]) + 4, float(fx["par_gam"]))
    e = hc.Eos(T.xa, T.ya, T.val, T.consts)
    yield e
    e.close()


def _problem(hc, fx):
    pr = problem_from_fixture(fx)
    pr.torus = hc.TorusSpec(4.0, 11.8, 1.e-3, 50.0)   # the torus of init.c:108-117
    return pr


def _bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def test_cool_init_matches_reference(hc, fx):
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.init_torus()
    p = ctx.get_prims()
    assert _bits_equal(active(pr, p), fx["p0"])
    assert ctx.time() == tuple(fx["t0"])
    ctx.close()


def _compare(pr, ctx, fx, n):
    p, fl = ctx.get_prims(with_flags=True)
    g = active(pr, p)
    ok = g.view(np.int64) == fx["p%d" % n].view(np.int64)
    assert ok.all(), (n, int((~ok).sum()), np.argwhere(~ok)[:5].tolist())
    assert np.array_equal(active(pr, fl), fx["pflag%d" % n]), n
    assert ctx.time() == tuple(fx["t%d" % n]), n
    assert _bits_equal(ctx.eos_guess(), fx["lastT%d" % n]), n
    # the diagnostics are device reductions in another summation order
    d = ctx.diag()
    assert d["fail_code"] == 0
    for k, name in enumerate(("mdot", "edot", "ldot")):
        ref = fx["diag%d" % n][k]
        assert abs(d[name] - ref) <= 1e-12 * max(abs(ref), 1e-300), (n, name, d[name], ref)
    ref = fx["diag%d" % n][5]
    assert abs(d["mass_curr"] - ref) <= 1e-13 * abs(ref), n


def test_cool_steps_match_reference(hc, fx, eos):
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p0"]), full_state(pr, fx["pflag0"]))
    ctx.set_time(*fx["t0"])
    ctx.set_eos(eos)
    assert not ctx.eos_guess().any()
    done = 0
    for n in STEPS:
        ctx.run(n - done)     # the first call runs the seeding step, then the graph
        done = n
        _compare(pr, ctx, fx, n)
    ctx.close()


def test_cool_step_by_step_matches_run(hc, fx, eos):
    """harm_step_ch one step at a time (no graph) gives the same states."""
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.put_prims(full_state(pr, fx["p0"]), full_state(pr, fx["pflag0"]))
    ctx.set_time(*fx["t0"])
    ctx.set_eos(eos)
    for _ in range(5):
        ctx.step_ch()
    ctx.sync()
    _compare(pr, ctx, fx, 5)
    ctx.close()


def test_cool_resume_from_saved_guesses(hc, fx, eos):
    """State and guesses of step 5 put back: steps 6..12 as the reference."""
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.set_eos(eos)
    ctx.put_prims(full_state(pr, fx["p5"]), full_state(pr, fx["pflag5"]))
    ctx.set_time(*fx["t5"])
    ctx.set_mass(*fx["diag5"][6:8])
    ctx.put_eos_guess(fx["lastT5"])
    ctx.run(7)
    _compare(pr, ctx, fx, 12)
    ctx.close()


def test_utoprim_5d_matches_reference_kat(hc, fx, eos):
    n = len(fx["u5_ret"])
    prim = np.ascontiguousarray(fx["u5_guess"].copy())
    ret, lt = eos.utoprim_5d(fx["u5_U"], fx["u5_gcov"].reshape(n, 16), fx["u5_gcon"].reshape(n, 16), fx["u5_gdet"],
                             fx["u5_hij"][:, 1], fx["u5_lastT"], prim)
    assert np.array_equal(ret, fx["u5_ret"])
    assert _bits_equal(prim, fx["u5_prim"])
    assert _bits_equal(lt, fx["u5_lastT_after"])


def test_cool_context_rules(hc, fx, eos):
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.init_torus()
    ctx.set_eos(eos)
    with pytest.raises(hc.HarmError):
        ctx.autotune_tile(steps=1)      # the tile autotuner times the gamma-law step
    small = hc.Context(hc.torus_problem(pr.params.n1 + 8, 16, 1))
    with pytest.raises(hc.HarmError):
        small.set_eos(eos)      # 8 more radial indices than tables
    ctx.set_eos(None)           # back to the gamma-law step
    ctx.run(2)
    assert ctx.diag()["fail_code"] == 0
    small.close()
    ctx.close()


def test_cool_mixed_tracks_fp64(hc, eos):
    """The COOL_EOS step with the face physics' EOS calls in FP32 against the FP64
    COOL_EOS step: density L1 within 1e-4 after 300 steps of a 64x64 torus."""
    from harm_cool_b200 import eos_tables
    pr = hc.torus_problem(64, 64, 1, a=0.6, rin=4.0, rmax=11.8, beta=50.0)
    xa, ya, val, consts = eos_tables.build_tables(eos_tables.zone_radii(pr), gam=pr.params.gam)
    E = hc.Eos(xa, ya, val, consts)
    a = hc.Context(pr)
    a.init_torus()
    a.set_eos(E)
    b = hc.Context(pr)
    b.init_torus()
    b.set_precision(hc.Context.MIXED)
    b.set_eos(E)
    for n in (1, 300):
        a.run(n if n == 1 else n - 1)
        b.run(n if n == 1 else n - 1)
    pa, pb = a.get_prims(), b.get_prims()
    assert np.all(np.isfinite(pb))
    from helpers import l1_groups, l1_rel
    l1 = l1_rel(pb, pa)
    print("COOL_EOS mixed vs FP64, 64x64, 300 steps:", l1_groups(pb, pa))
    assert l1[0] <= 1e-4, l1
    assert b.diag()["fail_code"] == 0
    a.close()
    b.close()
    E.close()


def test_cool_restart_matches_reference(hc, fx, eos, tmp_path):
    """restart_write() of a COOL_EOS run ends with every zone's temperature guess
    (restart_write_CoolEOS, cooleos.c:996-1013): the device's file matches the
    reference's after 5 steps, and reading the reference's file continues the
    run exactly (steps 6..12)."""
    from test_gpu_restart import _header_fields
    ref = fx["restart5"].tobytes().decode()
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.set_eos(eos)
    ctx.put_prims(full_state(pr, fx["p5"]), full_state(pr, fx["pflag5"]))
    ctx.set_time(*fx["t5"])
    ctx.set_mass(*fx["diag5"][6:8])
    ctx.put_eos_guess(fx["lastT5"])
    h = _header_fields(ref)
    fields = {k: v for k, v in h.items() if k not in ("n1", "n2", "n3", "t", "dt", "mass_in", "mass_out")}
    refl = ref.split("\n")
    tail = refl[-1].split()
    path = str(tmp_path / "rdump")
    ctx.restart_write(path, ener_size=int(tail[0]), **fields)
    ours = open(path).read().split("\n")
    assert ours[0] == refl[0]
    # every cell of the active phi planes (in 3D the reference's phi ghost planes
    # hold stale exchange copies, this writer periodic ones)
    cells = np.arange(int(np.prod(pr.shape))).reshape(pr.shape)
    act = cells[1:-1] if pr.params.n3 > 1 else cells
    for c in act.ravel():
        assert ours[1 + c] == refl[1 + c], c
    assert ours[-1].split()[1:] == tail[1:]      # the guesses, as the reference prints them
    ctx.close()
    path2 = tmp_path / "rdump_ref"
    path2.write_text(ref)
    c2 = hc.Context(pr)
    c2.set_eos(eos)
    c2.init_torus()
    c2.restart_read(str(path2))
    assert np.array_equal(active(pr, c2.get_prims()), fx["p5"])
    assert _bits_equal(c2.eos_guess(), fx["lastT5"])
    c2.run(7)
    assert _bits_equal(active(pr, c2.get_prims()), fx["p12"])
    assert _bits_equal(c2.eos_guess(), fx["lastT12"])
    c2.close()


def test_cool_diag_matches_reference(hc, fx, eos):
    """diag() with COOL_EOS on the state after 12 steps: the integrals and the
    neutrino luminosities as ener.out prints them (diag.c:316-320: %10.5g for
    t, rmed, pp, e; %15.8g for lnu, lnu_rho, lnu_rho_2, lnu2), divbmax and its
    zone, and the guesses diag() leaves (bit for bit: its InitCache, primtoU and
    CoolVal calls move them)."""
    pr = _problem(hc, fx)
    ctx = hc.Context(pr)
    ctx.set_eos(eos)
    ctx.put_prims(full_state(pr, fx["p12"]), full_state(pr, fx["pflag12"]))
    ctx.set_time(*fx["t12"])
    ctx.put_eos_guess(fx["lastT12"])
    ctx.run(0)
    d = ctx.integrals()
    ener = fx["diag_cool_ener"]
    for k, name in ((1, "rmed"), (2, "pp"), (3, "e")):
        assert float("%10.5g" % d[name]) == ener[k], (name, d[name], ener[k])
    for k, name in ((9, "lnu"), (10, "lnu_rho"), (11, "lnu_rho_2"), (12, "lnu2")):
        assert float("%15.8g" % d[name]) == ener[k], (name, d[name], ener[k])
    divb = fx["diag_cool_divb"]
    assert float("%g" % d["divbmax"]) == divb[0]
    assert d["imax"] == [int(v) for v in divb[1:]]
    assert _bits_equal(ctx.eos_guess(), fx["lastT_after_diag"])
    ctx.close()
