"""Gradients of the time-integrated horizon accretion through the discrete adjoint.

The device adjoint (Context.adjoint_mass_in, harm_adjoint_mass_in) returns, for
K steps of the 2D gamma-law step, J -- the mass that crosses the inner radial
boundary meanwhile, the reference's mass_in (diag.c:578) -- and dJ/dp0, the
gradient with respect to every cell of the initial primitive state.  This
module puts parameters in front of it:

    theta = (rmax, beta, A_1 .. A_M)

rmax and beta are the torus' pressure-maximum radius and plasma beta (init.c:
108-116); A_m are the amplitudes of M seeded smooth perturbation modes of the
density, rho <- rho (1 + sum_m A_m phi_m), applied after init() to the active
zones, after which bound_prim() fills the ghosts again.  The reference
perturbs u with white noise (init.c:266-274) and has no such modes; they are
this module's own, defined on the zone indices so that any code holding the
same state array applies them identically.  The spin a is not a parameter
here: it moves the grid's inner edge (Rin = 0.98 r_H(a), init.c:125) and with
it every metric entry, whose derivatives the adjoint does not carry.

dJ/dtheta_k = sum over cells of dJ/dp0 * dp0/dtheta_k, with dp0/dtheta_k the
central difference of the initial state (init + modes + bound_prim, which are
cheap) and dJ/dp0 from one adjoint sweep for all parameters together.
"""
import numpy as np

RHO = 0  # density slot of a primitive record (decs.h:190)


class Modes:
    """M smooth modes phi_m(i, j) = sin(pi k1 x1 + phase) sin(pi k2 x2) on the
    active zones, x1 = (i - istart + 0.5)/N1, x2 = (j - jstart + 0.5)/N2, with
    k1, k2 in 1..4 and the phase drawn from a seeded generator; they vanish
    towards the poles."""

    def __init__(self, n1, n2, m=16, seed=0):
        rng = np.random.default_rng(seed)
        self.k1 = rng.integers(1, 5, size=m)
        self.k2 = rng.integers(1, 5, size=m)
        self.phase = rng.uniform(0.0, 2.0 * np.pi, size=m)
        x1 = (np.arange(n1) + 0.5) / n1
        x2 = (np.arange(n2) + 0.5) / n2
        self.phi = np.stack([np.outer(np.sin(np.pi * self.k1[q] * x1 + self.phase[q]), np.sin(np.pi * self.k2[q] * x2))
                             for q in range(m)])

    @property
    def m(self):
        return len(self.phi)

    def apply(self, p, amps, h=0, istart=2, jstart=2):
        """rho <- rho (1 + sum_m A_m phi_m) on the active zones of plane h of a
        p[h][i][j][NPR] array, in place."""
        n1, n2 = self.phi.shape[1:]
        f = 1.0 + np.tensordot(np.asarray(amps, dtype=np.float64), self.phi, axes=1)
        p[h, istart:istart + n1, jstart:jstart + n2, RHO] *= f
        return p


def initial_state(ctx, modes, rmax, beta, amps):
    """init() with the given torus, the modes applied, ghosts filled: the state
    resident on the context and returned in get_prims' layout."""
    pr = ctx.problem
    pr.torus.rmax, pr.torus.beta = rmax, beta
    ctx.init_torus()
    p = ctx.get_prims()
    modes.apply(p, amps)
    ctx.bound_prim(p)
    ctx.put_prims(p)
    return p


def mass_in_gradient(ctx, modes, rmax, beta, amps, nsteps, checkpoint_every=10, rel_step=1e-6):
    """J and dJ/dtheta, theta = (rmax, beta, A_1..A_M), through one adjoint sweep.

    Returns (J, grad, info): info holds dJ/dp0 and the device times (ms) of the
    forward pass and of the reverse sweep."""
    amps = np.asarray(amps, dtype=np.float64)
    theta = np.concatenate([[rmax, beta], amps])
    dp = []
    for k in range(len(theta)):
        h = rel_step * max(abs(theta[k]), 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        pp = initial_state(ctx, modes, tp[0], tp[1], tp[2:])
        pm = initial_state(ctx, modes, tm[0], tm[1], tm[2:])
        dp.append((pp - pm) / (2.0 * h))
    initial_state(ctx, modes, rmax, beta, amps)
    J, lam, ms = ctx.adjoint_mass_in(nsteps, checkpoint_every)
    grad = np.array([np.sum(lam * d) for d in dp])
    return J, grad, {"dJ_dp0": lam, "ms": ms}


def mass_in(ctx, modes, rmax, beta, amps, nsteps):
    """J alone: the forward steps from the parameters' initial state."""
    initial_state(ctx, modes, rmax, beta, amps)
    m0 = ctx.diag()["mass_in"]
    for _ in range(nsteps):
        ctx.step_ch()
    ctx.sync()
    return ctx.diag()["mass_in"] - m0
