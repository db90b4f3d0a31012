"""Generate the golden fixtures in tests/golden/ from the HARM-COOL reference.

Run in a container that has the reference sources (it builds and imports
oracle/_ref/<config>/libharmref.so, the reference compiled from its own C
files).  Fixtures hold only generated numbers:
  <config>.npz  run parameters, sha256 of the reference's geometry arrays,
                the primitives and flags after init() and after 1, 2 and 5
                calls of step_ch(), with t, dt and the diagnostics.
  kat_u2p.npz   Utoprim_2d / Utoprim_1dvsq2fix1 / Utoprim_1dfix1 inputs and
                outputs on perturbed zones of the 2D torus.
Each configuration runs in its own process: the reference keeps its state in
globals.
"""
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


if __name__ == "__main__":
    if len(sys.argv) > 1:
        if sys.argv[1] == "kat":
            kat_u2p()
        else:
            one_config(sys.argv[1])
        sys.exit(0)
    sys.path.insert(0, ROOT)
    from oracle import build_ref
    for cfg in ("t2d", "t3d"):
        build_ref.build_config(cfg, force=True)
    for arg in ("t2d", "t3d", "kat"):
        subprocess.run([sys.executable, os.path.abspath(__file__), arg], check=True,
                       stderr=subprocess.DEVNULL)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
