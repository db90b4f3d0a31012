"""The discrete adjoint of the 2D gamma-law step (harm_adjoint_mass_in) against
central differences of the step itself.

J is the mass that crosses the inner radial boundary during K steps (mass_in,
diag.c:578).  The step is bit-identical to the reference's, so a central
difference of the device step is a central difference of the reference code;
tests/golden/adjoint_t2d.npz also holds differences taken on the reference
itself (make_golden.py).  Tolerance: 1e-4 relative to the largest component
of the gradient compared.

Step of the differences: h = 1e-9 relative.  The torus' atmosphere sits within
~1e-7 (relative) of its density floor, which fixup() re-applies every step, so
a difference with h = 1e-6 straddles the floor's kink in many zones and
averages a slope of 1 with a slope of 0; the adjoint gives the derivative of
the branch the step took, which the smaller step resolves.
"""
import os

import numpy as np
import pytest

import harm_cool_b200 as hc
from harm_cool_b200 import adjoint as ad

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-4
H = 1e-9


def _context(n1, n2):
    return hc.Context(hc.torus_problem(n1, n2, 1))


def _mass_in_from(ctx, p, nsteps):
    ctx.init_torus()  # t, dt and the counters as at the start
    ctx.put_prims(p)
    m0 = ctx.diag()["mass_in"]
    for _ in range(nsteps):
        ctx.step_ch()
    ctx.sync()
    return ctx.diag()["mass_in"] - m0


def _smooth_direction(shape, seed):
    """a smooth random field per primitive on the active zones of plane 0"""
    rng = np.random.default_rng(seed)
    _, sn1, sn2, _ = shape
    n1, n2 = sn1 - 4, sn2 - 4
    x1 = (np.arange(n1) + 0.5) / n1
    x2 = (np.arange(n2) + 0.5) / n2
    v = np.zeros(shape)
    for k in range(8):
        f = np.zeros((n1, n2))
        for _ in range(3):
            a, b = rng.integers(1, 5, size=2)
            f += rng.normal() * np.outer(np.sin(np.pi * a * x1 + rng.uniform(0, 6.28)), np.sin(np.pi * b * x2))
        v[0, 2:2 + n1, 2:2 + n2, k] = f
    return v


@pytest.mark.parametrize("nsteps,every", [(6, 4), (12, 5)])
def test_state_direction_against_central_difference(nsteps, every):
    ctx = _context(48, 48)
    ctx.init_torus()
    p0 = ctx.get_prims()
    v = _smooth_direction(p0.shape, seed=nsteps)
    # perturbations relative to each cell's own value (velocities and fields:
    # plus a thousandth of their scale on the grid, many start at zero)
    scale = np.array([np.abs(p0[..., k]).max() for k in range(8)])
    v *= np.abs(p0) + 1e-3 * scale * (np.arange(8) >= 2)
    J, lam, ms = ctx.adjoint_mass_in(nsteps, every)
    # the context has advanced: J again by the plain steps
    J0 = _mass_in_from(ctx, p0, nsteps)
    assert J == J0
    h = H
    Jp = _mass_in_from(ctx, p0 + h * v, nsteps)
    Jm = _mass_in_from(ctx, p0 - h * v, nsteps)
    fd = (Jp - Jm) / (2 * h)
    ad_ = float(np.sum(lam * v))
    assert abs(ad_ - fd) <= TOL * abs(fd), (ad_, fd)


def test_checkpoint_spacing_does_not_change_the_gradient():
    """one segment recorded on the forward pass (9), full segments of odd and
    even length replayed from graphs (3, 2, 4), partial last segments (2, 4)"""
    ctx = _context(32, 32)
    ctx.init_torus()
    p0 = ctx.get_prims()
    J1, l1, _ = ctx.adjoint_mass_in(9, 9)
    for every in (2, 3, 4):
        ctx.init_torus()
        ctx.put_prims(p0)
        J2, l2, _ = ctx.adjoint_mass_in(9, every)
        assert J1 == J2
        np.testing.assert_allclose(l2, l1, rtol=1e-12, atol=1e-12 * np.abs(l1).max())


def test_parameter_gradient_against_central_difference():
    """dJ/d(rmax, beta, A_1..A_16) on a 48x48 torus over 10 steps"""
    ctx = _context(48, 48)
    modes = ad.Modes(48, 48, m=16, seed=3)
    amps = np.zeros(16)
    J, g, info = ad.mass_in_gradient(ctx, modes, 12.0, 100.0, amps, 10, checkpoint_every=4, rel_step=H)
    theta = np.concatenate([[12.0, 100.0], amps])
    fd = np.zeros_like(g)
    for k in range(len(theta)):
        h = H * max(abs(theta[k]), 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd[k] = (ad.mass_in(ctx, modes, tp[0], tp[1], tp[2:], 10) - ad.mass_in(ctx, modes, tm[0], tm[1], tm[2:], 10)) / (2 * h)
    scale = np.abs(fd).max()
    assert scale > 0
    np.testing.assert_allclose(g, fd, rtol=0, atol=TOL * scale)


def test_rmax_and_beta_gradients_once_the_torus_reaches_the_inner_boundary():
    """dJ/drmax and dJ/dbeta over a window long enough for the torus's own matter
    to reach the inner boundary: 64x64 torus, K = 800 steps (t ~ 35 M),
    checkpoint every 100.  Over the 10 to 50 steps of the other tests only the
    atmosphere flows in and both are exactly zero.  The central differences are
    noisy here: the atmosphere sits at its density floor, whose kink a difference
    straddles in some zones, and the differences spread by about 1e-3 (rmax) and
    a few percent (beta) between h = 3e-9 and 1e-7.  So the adjoint is checked
    against the median difference over those steps, to 2e-3 for rmax and 2e-2
    for beta; beyond about 1500 steps the flow turns chaotic and neither the
    differences nor the derivative mean anything."""
    n, K = 64, 800
    ctx = _context(n, n)
    modes = ad.Modes(n, n, m=2, seed=0)
    amps = np.zeros(2)
    J, g, info = ad.mass_in_gradient(ctx, modes, 12.0, 100.0, amps, K, checkpoint_every=100, rel_step=1e-7)
    theta = np.array([12.0, 100.0])
    fd = np.zeros((4, 2))
    for a, hr in enumerate((1e-7, 3e-8, 1e-8, 3e-9)):
        for k in range(2):
            h = hr * theta[k]
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            fd[a, k] = (ad.mass_in(ctx, modes, tp[0], tp[1], amps, K) - ad.mass_in(ctx, modes, tm[0], tm[1], amps, K)) / (2 * h)
    med = np.median(fd, axis=0)
    print("K = %d: adjoint dJ/drmax %.6e dJ/dbeta %.6e; central differences" % (K, g[0], g[1]), fd.tolist())
    # clearly non-zero: the torus's matter reaches the boundary within the window
    assert abs(med[0]) > 1e-5 and abs(med[1]) > 1e-9
    assert abs(g[0] - med[0]) <= 2e-3 * abs(med[0]), (g[0], med[0])
    assert abs(g[1] - med[1]) <= 2e-2 * abs(med[1]), (g[1], med[1])


def test_against_reference_central_differences(oracle_built):
    """dJ/dA_m against central differences taken on the reference's own step
    (32x32 torus, 10 steps; fixture written by make_golden.py).  Over these
    steps Utoprim_1dvsq2fix1 rescues failed inversions (the oracle counts
    them), so the fall-back adjoint (ift_fallback) is part of what matches."""
    f = np.load(os.path.join(HERE, "golden", "adjoint_t2d.npz"))
    n, m, seed, nsteps = (int(x) for x in f["setup"])
    ctx = _context(n, n)
    modes = ad.Modes(n, n, m=m, seed=seed)
    ad.initial_state(ctx, modes, 12.0, 100.0, np.zeros(m))
    drift, rescued1, rescued2 = _oracle_branches(ctx.problem, ctx.get_prims(), ctx.time(), nsteps)
    print("fall-back rescues %d + %d, drift-frame floors %d" % (rescued1, rescued2, drift))
    assert rescued1 > 0
    J, g, _ = ad.mass_in_gradient(ctx, modes, 12.0, 100.0, np.zeros(m), nsteps, checkpoint_every=4, rel_step=H)
    assert J == f["J"]
    fd = f["fd"]
    np.testing.assert_allclose(g[2:], fd, rtol=0, atol=TOL * np.abs(fd).max())


def test_refusals():
    ctx3 = hc.Context(hc.torus_problem(16, 16, 4))
    ctx3.init_torus()
    with pytest.raises(hc.HarmError):
        ctx3.adjoint_mass_in(2, 1)
    ctx = _context(16, 16)
    ctx.init_torus()
    ctx.set_precision(hc.Context.MIXED)
    with pytest.raises(hc.HarmError):
        ctx.adjoint_mass_in(2, 1)


class _MassInFunction:
    """J(theta) as a torch.autograd.Function over the device adjoint: the test
    harness's thin wrapper (the library itself has no torch dependency)."""

    @staticmethod
    def make(ctx, modes, nsteps, every):
        import torch

        class MassIn(torch.autograd.Function):
            @staticmethod
            def forward(fctx, theta):
                th = theta.detach().cpu().numpy()
                J, g, _ = ad.mass_in_gradient(ctx, modes, th[0], th[1], th[2:], nsteps, every, rel_step=H)
                fctx.save_for_backward(torch.as_tensor(g, dtype=theta.dtype))
                return theta.new_tensor(J)

            @staticmethod
            def backward(fctx, gout):
                (g,) = fctx.saved_tensors
                return gout * g

        return MassIn.apply


def test_torch_autograd_wrapper():
    torch = pytest.importorskip("torch")
    ctx = _context(32, 32)
    modes = ad.Modes(32, 32, m=16, seed=3)
    f = _MassInFunction.make(ctx, modes, 6, 3)
    theta = torch.tensor([12.0, 100.0] + [0.0] * 16, dtype=torch.float64, requires_grad=True)
    J = f(theta)
    (g,) = torch.autograd.grad(J, theta)
    J2, g2, _ = ad.mass_in_gradient(ctx, modes, 12.0, 100.0, np.zeros(16), 6, 3, rel_step=H)
    assert float(J.detach()) == J2
    # atomic accumulation order may move the last bits between two sweeps
    np.testing.assert_allclose(g.numpy(), g2, rtol=1e-10, atol=1e-10 * np.abs(g2).max())


def _oracle_branches(pr, p0, t_dt, nsteps):
    """The oracle's counts of floors in the drift frame and of inversions rescued
    by Utoprim_1dvsq2fix1 and Utoprim_1dfix1 over nsteps from p0: the device
    step takes the same branches bit for bit, so these are the paths the
    adjoint of the same steps goes through."""
    from helpers import make_oracle
    o = make_oracle(pr)
    o.p[...] = p0
    o.pflag[...] = 0
    o.set_time(*t_dt)
    o.branch_counts(reset=True)
    for _ in range(nsteps):
        o.step()
    return o.branch_counts(reset=True)


def test_repaired_zones_against_central_difference(oracle_built):
    """A 3x3 block of strong radial field six zones from the inner boundary
    makes the inversion fail in 8 zones of the first step, and fixup_utoprim
    repairs them from their neighbours with corner and last-resort stencils
    (fixup.c:432-538): the adjoint replays those repairs and transposes them,
    and the failed inversions keep their guess.  The same steps floor zones in
    the drift frame (fixup_vjp) and rescue inversions with Utoprim_1dvsq2fix1
    (ift_fallback), as the oracle's branch counts show.  (With the block against the
    boundary, J itself is rough at the inversion tolerance, ~1e-10 relative,
    and no central difference resolves a slope there.)"""
    n, i0 = 48, 8
    ctx = _context(n, n)
    ctx.init_torus()
    p0 = ctx.get_prims()
    blk = (0, slice(i0, i0 + 3), slice(2 + n // 2 - 1, 2 + n // 2 + 2), 5)
    p0[blk] = 1e3 * np.abs(p0[..., 5]).max()
    ctx.init_torus()
    ctx.put_prims(p0)
    ctx.step_ch()
    ctx.sync()
    _, fl = ctx.get_prims(with_flags=True)
    assert np.sum(fl[0, 2:n + 2, 2:n + 2] != 1) > 0  # the step repaired zones
    v = _smooth_direction(p0.shape, seed=7)
    scale = np.array([np.abs(p0[..., k]).max() for k in range(8)])
    v *= np.abs(p0) + 1e-3 * scale * (np.arange(8) >= 2)
    ctx.init_torus()
    ctx.put_prims(p0)
    drift, rescued1, rescued2 = _oracle_branches(ctx.problem, p0, ctx.time(), 4)
    print("drift-frame floors %d, fall-back rescues %d + %d" % (drift, rescued1, rescued2))
    assert drift > 0 and rescued1 > 0  # the floors' drift frame and ift_fallback are exercised
    J, lam, _ = ctx.adjoint_mass_in(4, 3)
    assert J == _mass_in_from(ctx, p0, 4)
    fd = (_mass_in_from(ctx, p0 + H * v, 4) - _mass_in_from(ctx, p0 - H * v, 4)) / (2 * H)
    ad_ = float(np.sum(lam * v))
    assert abs(ad_ - fd) <= TOL * abs(fd), (ad_, fd)
