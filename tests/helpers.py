"""Shared helpers: problems from the golden fixtures, oracle set-up, comparisons."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
NAMES = ("rho", "u", "u1", "u2", "u3", "B1", "B2", "B3")


def load_fixture(cfg):
    return dict(np.load(os.path.join(GOLDEN, cfg + ".npz")))


def problem_from_fixture(fx):
    """The fixture's run rebuilt with the library's host set-up code."""
    import harm_cool_b200 as hc
    n1, n2, n3 = (int(v) for v in fx["n"])
    pr = hc.torus_problem(n1, n2, n3, a=float(fx["par_a"]), gam=float(fx["par_gam"]),
                          cour=float(fx["par_cour"]), hslope=float(fx["par_hslope"]),
                          Rout=float(fx["par_Rout"]), R0=float(fx["par_R0"]), tf=float(fx["par_tf"]))
    return pr


def full_state(pr, active):
    """Embed active phi planes in an array of the reference's full shape."""
    p = np.zeros(pr.shape + active.shape[3:], dtype=active.dtype)
    if pr.params.n3 > 1:
        p[1:-1] = active
    else:
        p[:] = active
    return p


def active(pr, full):
    return full[1:-1] if pr.params.n3 > 1 else full


def make_oracle(pr):
    from oracle.pyoracle import Oracle, make_params
    prm = pr.params
    op = make_params(prm.n1, prm.n2, prm.n3, prm.a, prm.gam, prm.cour, list(prm.dx), list(prm.startx),
                     defcon=prm.defcon, tf=prm.tf, lim=prm.lim)
    return Oracle(op, pr.geometry)


def field_rel_err(a, b):
    """Per primitive: max |a-b| over the grid divided by max |b| over the grid."""
    out = []
    for k in range(8):
        scale = np.max(np.abs(b[..., k]))
        out.append(float(np.max(np.abs(a[..., k] - b[..., k])) / scale) if scale > 0 else
                   float(np.max(np.abs(a[..., k]))))
    return np.array(out)


def l1_rel(a, b):
    out = []
    for k in range(8):
        scale = np.mean(np.abs(b[..., k]))
        out.append(float(np.mean(np.abs(a[..., k] - b[..., k])) / scale) if scale > 0 else 0.)
    return np.array(out)


def l1_groups(a, b):
    """L1 of (a-b) relative to the L1 of b for rho, u, the velocity vector and the
    field vector."""
    out = {}
    for n, ks in (("rho", [0]), ("u", [1]), ("v", [2, 3, 4]), ("B", [5, 6, 7])):
        s = np.sum(np.abs(b[..., ks]))
        out[n] = float(np.sum(np.abs(a[..., ks] - b[..., ks])) / s) if s > 0 else 0.
    return out
