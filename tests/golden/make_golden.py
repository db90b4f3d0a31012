"""Generate the golden fixtures in tests/golden/ from the HARM-COOL reference.

Run in a container that has the reference sources (it builds and imports
oracle/_ref/<config>/libharmref.so, the reference compiled from its own C
files).  Fixtures hold only generated numbers:
  <config>.npz  run parameters, sha256 of the reference's geometry arrays,
                the primitives and flags after init() and after 1, 2 and 5
                calls of step_ch(), with t, dt and the diagnostics.
  kat_u2p.npz   Utoprim_2d / Utoprim_1dvsq2fix1 / Utoprim_1dfix1 inputs and
                outputs on perturbed zones of the 2D torus.
  diag_<config>.npz  diag(INIT_OUT)'s printed integrals and divbmax with its
                zone, on the state after 5 steps.
  restart_<config>.npz  restart_write()'s file after 5 steps, as text.
  tracers_<config>.npz  the reference's tracer particles (tracers.c) after
                init_tracers() and after steps, and a seeded custom tracer
                list carried through 25 more steps.
  eos_<config>.npz  the run-time COOL_EOS of a COOL_EOS build: digests of its
                tables, pressure/dpdu/dpdrho on seeded entries.
  cool_<config>.npz  step_ch() of a COOL_EOS build: states, flags, times and
                temperature guesses after init() and steps; the restart file
                after 5 steps; diag() and dump() after 12 steps with the guesses
                they leave; Utoprim_5d known answers.
  dump_<config>.npz  dump()'s ASCII dump after 5 steps: header line and the
                sha256 of every zone line.
Each configuration runs in its own process: the reference keeps its state in
globals.
"""
import ctypes
import hashlib
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
STEPS = (1, 2, 5)
SCALARS = ("mdot", "edot", "ldot", "mdot_in", "mdot_out", "mass_curr", "mass_in", "mass_out")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def one_config(cfg):
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    hs = slice(1, ref.n3 + 1) if ref.n3 > 1 else slice(0, 1)
    g = ref.geometry()
    out = {"n": np.array([ref.n1, ref.n2, ref.n3])}
    for name in ("a", "gam", "cour", "defcon", "tf", "Rin", "Rout", "hslope", "R0",
                 "dx1", "dx2", "dx3", "startx1", "startx2", "startx3"):
        out["par_" + name] = np.array(ref.get(name))
    for k, v in g.items():
        out["sha_" + k] = np.array(sha(v))
    out["p0"] = ref.p[hs].copy()
    out["pflag0"] = ref.pflag[hs].copy()
    out["t0"] = np.array([ref.get("t"), ref.get("dt")])
    done = 0
    for n in STEPS:
        while done < n:
            ref.step()
            done += 1
        out["p%d" % n] = ref.p[hs].copy()
        out["pflag%d" % n] = ref.pflag[hs].copy()
        out["t%d" % n] = np.array([ref.get("t"), ref.get("dt")])
        out["diag%d" % n] = np.array([ref.get(s) for s in SCALARS])
    np.savez_compressed(os.path.join(HERE, cfg + ".npz"), **out)


def custom_tracers(ref, rng, n=240):
    """A seeded tracer set over the whole grid, with tracers close to the inner
    radius (they fall in), beyond the outer tracer radius inside and outside the
    theta window (they leave as out and jet), and a few outside the grid (the
    search fails and they are dropped)."""
    import math
    sx = [0., ref.get("startx1"), ref.get("startx2"), ref.get("startx3")]
    dx = [0., ref.get("dx1"), ref.get("dx2"), ref.get("dx3")]
    n1, n2, n3 = ref.n1, ref.n2, ref.n3
    R0, hslope = ref.get("R0"), ref.get("hslope")
    x1lo, x1hi = sx[1] - 0.5 * dx[1], sx[1] + (n1 + 0.5) * dx[1]
    x2lo, x2hi = sx[2] - 0.5 * dx[2], sx[2] + (n2 + 0.5) * dx[2]
    x3hi = sx[3] + n3 * dx[3]
    rout_t = 0.8 * (math.exp(sx[1] + n1 * dx[1]) + R0)
    X = []
    for k in range(n):
        kind = k % 6
        x2 = rng.uniform(x2lo, x2hi)
        x3 = rng.uniform(sx[3], x3hi) if n3 > 1 else 0.
        if kind == 0:     # near the inner tracer radius
            x1 = sx[1] - 0.5 * dx[1] + rng.uniform(1e-6, 2e-2)
        elif kind == 1:   # beyond the outer tracer radius
            x1 = math.log(rout_t - R0) + rng.uniform(1e-6, 0.5 * dx[1])
        elif kind == 2:   # outside the grid (dropped by the search)
            x1 = x1lo - rng.uniform(0.1, 1.) * dx[1] if rng.random() < 0.5 else x1hi + rng.uniform(1., 2.) * dx[1]
        else:
            x1 = rng.uniform(sx[1], sx[1] + n1 * dx[1])
        X.append((x1, x2, x3))
    ids = np.array([(1000 + k, 0, 0) for k in range(n)], dtype=np.int32)
    return ids, np.array(X)


def tracer_config(cfg):
    """The reference's tracers (tracers.c, TRACERSDUMP on): init_tracers() after
    init, the list after 1, 2 and 5 steps, then a custom seeded list set after
    step 5 and read back after steps 6, 10 and 30."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    hs = slice(1, ref.n3 + 1) if ref.n3 > 1 else slice(0, 1)
    out = {"n": np.array([ref.n1, ref.n2, ref.n3])}
    for name in ("a", "gam", "cour", "defcon", "tf", "Rin", "Rout", "hslope", "R0",
                 "dx1", "dx2", "dx3", "startx1", "startx2", "startx3"):
        out["par_" + name] = np.array(ref.get(name))
    out["p0"] = ref.p[hs].copy()
    out["pflag0"] = ref.pflag[hs].copy()
    out["t0"] = np.array([ref.get("t"), ref.get("dt")])
    out["tr_ids0"], out["tr_X0"] = ref.tracers()
    done = 0
    for nstep in (1, 2, 5, 6, 10, 30):
        while done < nstep:
            ref.step()
            done += 1
            if done == 5:
                out["p5"] = ref.p[hs].copy()
                out["pflag5"] = ref.pflag[hs].copy()
                out["t5"] = np.array([ref.get("t"), ref.get("dt")])
                out["mass5"] = np.array([ref.get("mass_in"), ref.get("mass_out")])
                out["tr_ids5"], out["tr_X5"] = ref.tracers()
                ids, X = custom_tracers(ref, np.random.default_rng(7 + ref.n3))
                out["cu_ids"], out["cu_X"] = ids, X
                ref.set_tracers(ids, X)
        if nstep < 5:
            out["tr_ids%d" % nstep], out["tr_X%d" % nstep] = ref.tracers()
        elif nstep > 5:
            out["cu_ids%d" % nstep], out["cu_X%d" % nstep] = ref.tracers()
            out["p%d" % nstep] = ref.p[hs].copy()
    np.savez_compressed(os.path.join(HERE, "tracers_" + cfg + ".npz"), **out)


def diag_config(cfg):
    """diag(INIT_OUT) of the reference after 5 steps (the state of <cfg>.npz's p5):
    the printed integrals and divbmax with its zone."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    for _ in range(5):
        ref.step()
    d = ref.diag_init()
    np.savez_compressed(os.path.join(HERE, "diag_" + cfg + ".npz"),
                        printed=np.array([d["rmed"], d["pp"], d["e"], d["divbmax"]]),
                        imax=np.array(d["imax"], dtype=np.int32))


def restart_config(cfg):
    """restart_write() of the reference after 5 steps (the state of
    <cfg>.npz's p5, or tracers_<cfg>.npz's for a configuration with tracers):
    the file's text."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    for _ in range(5):
        ref.step()
    text = ref.restart_write()
    np.savez_compressed(os.path.join(HERE, "restart_" + cfg + ".npz"),
                        text=np.frombuffer(text.encode(), dtype=np.uint8))


def kat_u2p():
    sys.path.insert(0, ROOT)
    import ctypes
    from oracle.pyoracle import Reference
    ref = Reference("t2d")
    lib = ref.lib
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ref_prim_to_U.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp]
    lib.ref_utoprim_fix.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, ctypes.c_int]
    g = ref.geometry()
    rng = np.random.default_rng(20261203)
    rows = []
    p = ref.p[0]
    for t in range(256):
        i = int(rng.integers(2, ref.n1 + 2))
        j = int(rng.integers(2, ref.n2 + 2))
        pr = p[i, j].copy()
        U = np.zeros(8)
        lib.ref_prim_to_U(pr.ctypes.data_as(dp), i, j, U.ctypes.data_as(dp))
        mode = t % 4
        if mode == 1:      # small perturbation of the conserved state
            U[:5] *= 1. + 1e-3 * rng.standard_normal(5)
        elif mode == 2:    # large perturbation, some inversions fail
            U[:5] *= 1. + 0.5 * rng.standard_normal(5)
        elif mode == 3:    # perturbed guess
            pr[:5] *= 1. + 0.05 * rng.standard_normal(5)
        if t == 5:
            U[0] = -abs(U[0])  # the U[0] <= 0 early return
        rows.append((i, j, U.copy(), pr.copy()))
    n = len(rows)
    ij = np.array([(r[0], r[1]) for r in rows], dtype=np.int32)
    U = np.array([r[2] for r in rows])
    guess = np.array([r[3] for r in rows])
    res = {"ij": ij, "U": U, "guess": guess, "gam": np.array(ref.get("gam"))}
    for which, name in ((0, "2d"), (1, "vsq2fix1"), (2, "fix1")):
        out = guess.copy()
        ret = np.zeros(n, dtype=np.int32)
        for t in range(n):
            Ut = U[t].copy()
            pt = out[t]
            ptr = pt.ctypes.data_as(dp)
            i, j = int(ij[t, 0]), int(ij[t, 1])
            if which == 0:
                ret[t] = lib.ref_utoprim_2d(Ut.ctypes.data_as(dp), i, j, ptr)
            else:
                ret[t] = lib.ref_utoprim_fix(Ut.ctypes.data_as(dp), i, j, ptr, g["katm"][i], which)
        res["prim_" + name] = out
        res["ret_" + name] = ret
    np.savez_compressed(os.path.join(HERE, "kat_u2p.npz"), **res)


def dump_digest(text):
    """A dump's header line, the sha256 of every zone line and the first two lines."""
    lines = text.split("\n")
    assert lines[-1] == ""
    zl = lines[1:-1]
    return {"header": np.frombuffer(lines[0].encode(), dtype=np.uint8),
            "sha": np.array([hashlib.sha256(l.encode()).hexdigest() for l in zl]),
            "first": np.frombuffer("\n".join(zl[:2]).encode(), dtype=np.uint8)}


def dump_config(cfg):
    """dump() (the ASCII dump, dump.c:1710-2047) of the state after 5 steps."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference, _QuietStdout
    ref = Reference(cfg)
    with _QuietStdout():
        for _ in range(5):
            ref.step()
    np.savez_compressed(os.path.join(HERE, "dump_%s.npz" % cfg), **dump_digest(ref.dump()))


def eos_inputs(rng, ntab, n):
    """Seeded (table, rho0, u, T guess) entries over the run-time EOS's branches:
    table range, gamma-law below rhoMin / above rhoMax, e < 0, no guess yet
    (LastT == 0), solves that fail at the top of the T range."""
    tab = rng.integers(0, ntab, n)
    rho0 = 10 ** rng.uniform(-11, 4, n)
    u = rho0 * 10 ** rng.uniform(-9, 8, n) * np.where(rng.uniform(size=n) < 0.05, -1.0, 1.0)
    lastT = np.where(rng.uniform(size=n) < 0.3, 0.0, 10 ** rng.uniform(4.0, 17.9, n))
    return tab.astype(np.int32), rho0, u, lastT


def eos_config(cfg):
    """The reference's run-time EOS (COOL_EOS checker build, oracle/eos_standin.c
    as the table generator): its tables' digest and pressure, dp/du, dp/drho with
    the guesses they leave, on seeded entries."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    T = ref.cool_tables()
    out = {"grid": np.array([ref.get("startx1"), ref.get("dx1"), ref.get("R0"), ref.get("gam")]),
           "sn1": np.array(ref.sn1), "sha_tables": np.array(sha(T.val)),
           "sha_axes": np.array(sha(np.concatenate([T.xa, T.ya]))),
           "consts": np.array([T.consts[k] for k in sorted(T.consts) if k != "hdfac"]),
           "const_names": np.array(sorted(k for k in T.consts if k != "hdfac")),
           "hdfac": T.consts["hdfac"]}
    tab, rho0, u, lastT = eos_inputs(np.random.default_rng(2024), T.ntab, 3000)
    out.update(tab=tab, rho0=rho0, u=u, lastT=lastT)
    for what in ("pressure", "dpdu", "dpdrho"):
        v, lt = ref.cool_batch(what, tab, rho0, u, lastT)
        out[what] = v
        out[what + "_lastT"] = lt
    np.savez_compressed(os.path.join(HERE, "eos_%s.npz" % cfg), **out)


COOL_STEPS = (1, 2, 5, 12)


def cool_config(cfg):
    """step_ch() with COOL_EOS on (COOL_EOS checker build): the state, flags,
    times and temperature guesses after init() and after 1, 2, 5, 12 steps; then
    Utoprim_5d known answers on perturbed zones of the last state."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    ref = Reference(cfg)
    hs = slice(1, ref.n3 + 1) if ref.n3 > 1 else slice(0, 1)
    out = {"n": np.array([ref.n1, ref.n2, ref.n3])}
    for name in ("a", "gam", "cour", "defcon", "tf", "Rin", "Rout", "hslope", "R0",
                 "dx1", "dx2", "dx3", "startx1", "startx2", "startx3"):
        out["par_" + name] = np.array(ref.get(name))
    out["p0"] = ref.p[hs].copy()
    out["pflag0"] = ref.pflag[hs].copy()
    out["t0"] = np.array([ref.get("t"), ref.get("dt")])
    out["lastT0"] = ref.cool_lastT()
    done = 0
    from oracle.pyoracle import _QuietStdout
    for n in COOL_STEPS:
        with _QuietStdout():
            while done < n:
                ref.step()
                done += 1
        out["p%d" % n] = ref.p[hs].copy()
        out["pflag%d" % n] = ref.pflag[hs].copy()
        out["t%d" % n] = np.array([ref.get("t"), ref.get("dt")])
        out["lastT%d" % n] = ref.cool_lastT()
        out["diag%d" % n] = np.array([ref.get(s) for s in SCALARS])
        if n == 5:
            with _QuietStdout():
                out["restart5"] = np.frombuffer(ref.restart_write().encode(), dtype=np.uint8)
    # diag(INIT_OUT) on the state after the last step: ener.out's integrals and
    # COOL_EOS luminosities (diag.c:316-320), and the guesses diag() leaves
    with _QuietStdout():
        dg = ref.diag_init()
    out["diag_cool_ener"] = np.array(dg["ener"])
    out["diag_cool_divb"] = np.array([dg["divbmax"]] + dg["imax"])
    out["lastT_after_diag"] = ref.cool_lastT()
    # then dump(), which moves the guesses too
    dd = dump_digest(ref.dump())
    out.update({"dump_" + k: v for k, v in dd.items()})
    out["lastT_after_dump"] = ref.cool_lastT()
    # Utoprim_5d on perturbed states of active zones, each with its own guess
    rng = np.random.default_rng(55)
    last = ref.cool_lastT()
    p = ref.p[hs].copy()
    g = ref.geometry()
    rows = []
    for k in range(240):
        h = 0 if ref.n3 == 1 else int(rng.integers(1, ref.n3 + 1))
        i = int(rng.integers(2, ref.n1 + 2))
        j = int(rng.integers(2, ref.n2 + 2))
        pz = p[h - (1 if ref.n3 > 1 else 0), i, j].copy()
        pert = pz.copy()
        pert[:5] *= 1.0 + 1e-3 * rng.uniform(-1, 1, 5)
        U, _ = ref.cool_prim_to_U(pert, h, i, j, last[h, i, j])
        r, res, lt = ref.utoprim_5d(U, h, i, j, pz, last[h, i, j])
        rows.append((h, i, j, U, pz, last[h, i, j], r, res, lt))
    out["u5_hij"] = np.array([r[:3] for r in rows], dtype=np.int32)
    out["u5_U"] = np.array([r[3] for r in rows])
    out["u5_guess"] = np.array([r[4] for r in rows])
    out["u5_lastT"] = np.array([r[5] for r in rows])
    out["u5_ret"] = np.array([r[6] for r in rows], dtype=np.int32)
    out["u5_prim"] = np.array([r[7] for r in rows])
    out["u5_lastT_after"] = np.array([r[8] for r in rows])
    out["u5_gcov"] = np.array([g["gcov"][r[1], r[2], 3] for r in rows])
    out["u5_gcon"] = np.array([g["gcon"][r[1], r[2], 3] for r in rows])
    out["u5_gdet"] = np.array([g["gdet"][r[1], r[2], 3] for r in rows])
    np.savez_compressed(os.path.join(HERE, "cool_%s.npz" % cfg), **out)


def adjoint_config(cfg, m=16, seed=3, nsteps=10):
    """Central differences, taken on the reference's own step, of J = the change
    of mass_in (diag.c:578) over nsteps steps with respect to the amplitudes of
    the seeded density modes of harm_cool_b200.adjoint.Modes, and J at zero
    amplitudes: the check of the device adjoint's dJ/dA_m.  h = 1e-9: the
    atmosphere sits within ~1e-7 of its density floor, and a larger step
    straddles the floor's kink (fixup.c:142-187)."""
    sys.path.insert(0, ROOT)
    from oracle.pyoracle import Reference
    from harm_cool_b200.adjoint import Modes
    ref = Reference(cfg)
    assert ref.n3 == 1 and ref.n1 == ref.n2
    p0 = ref.p.copy()
    t0, dt0 = ref.get("t"), ref.get("dt")
    modes = Modes(ref.n1, ref.n2, m=m, seed=seed)

    def J(amps):
        ref.p[...] = p0
        ref.set("t", t0)
        ref.set("dt", dt0)
        modes.apply(ref.p, amps)
        ref.lib.ref_bound_prim(ref.p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        m0 = ref.get("mass_in")
        for _ in range(nsteps):
            ref.step()
        return ref.get("mass_in") - m0

    J0 = J(np.zeros(m))
    h = 1e-9
    fd = np.zeros(m)
    for k in range(m):
        a = np.zeros(m)
        a[k] = h
        jp = J(a)
        a[k] = -h
        fd[k] = (jp - J(a)) / (2 * h)
    np.savez_compressed(os.path.join(HERE, "adjoint_%s.npz" % cfg), setup=np.array([ref.n1, m, seed, nsteps]),
                        J=np.array(J0), fd=fd)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        if sys.argv[1] == "kat":
            kat_u2p()
        elif sys.argv[1].startswith("restart_"):
            restart_config(sys.argv[1][len("restart_"):])
        elif sys.argv[1].startswith("diag_"):
            diag_config(sys.argv[1][len("diag_"):])
        elif sys.argv[1].startswith("tracers_"):
            tracer_config(sys.argv[1][len("tracers_"):])
        elif sys.argv[1].startswith("eos_"):
            eos_config(sys.argv[1][len("eos_"):])
        elif sys.argv[1].startswith("cool_"):
            cool_config(sys.argv[1][len("cool_"):])
        elif sys.argv[1].startswith("dump_"):
            dump_config(sys.argv[1][len("dump_"):])
        elif sys.argv[1].startswith("adjoint_"):
            adjoint_config(sys.argv[1][len("adjoint_"):])
        else:
            one_config(sys.argv[1])
        sys.exit(0)
    sys.path.insert(0, ROOT)
    from oracle import build_ref
    for cfg in ("t2d", "t3d", "r2d", "r3d", "ce2d", "ce3d"):
        build_ref.build_config(cfg, force=True)
    for arg in ("t2d", "t3d", "kat", "tracers_r2d", "tracers_r3d", "diag_t2d", "diag_t3d",
                "restart_r2d", "restart_t3d", "eos_ce2d", "cool_ce2d", "cool_ce3d", "dump_t2d", "dump_t3d", "adjoint_t2d"):
        subprocess.run([sys.executable, os.path.abspath(__file__), arg], check=True,
                       stderr=subprocess.DEVNULL)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
