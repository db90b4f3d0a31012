"""Host-side construction of the run-time COOL_EOS tables.

The reference builds one table per radial index when it starts
(SetupCache_CoolEOS, cooleos.c:825-992): a 72 x 72 grid, logarithmic in rho
(1e2..1e15 g/cm^3) and T (1e4..1e18 K), whose nodes hold e, p, Qnu, tau and Yee
from its Fortran EOS and neutrino-rate code, abundance() (abundance.f90:6-243),
called with the table's HdFac (the disc scale-height factor at the zone's
radius, cooleos.c:945-960) through calc_cache_val (cooleos.c:171-194).  The
tables are built once on the host and then uploaded (harm_cool_b200.Eos).

build_tables() lays out the grid and HdFac exactly as the reference does and
takes the generator as a function; ideal_gas_radiation() is a synthetic
stand-in (no neutrino physics: placeholder power laws for Qnu and tau).
physical_tables() fills the same layout from the library's restatement of
abundance() (harm_nu.cuh), every node computed on the GPU; on_demand() computes
only the nodes a run reads, as the reference's cache does.
"""
import math

import numpy as np

# cooleos.c:83-135 (CGS)
GNEWT = 6.6742867e-8
MSUN = 1.9892e33
KBOL = 1.3e-16
CL = 2.99792458e10
MP, ME, MN, MHE = 1.67262163783e-24, 9.10956e-28, 1.67492729e-24, 6.6465e-24
MAV = (MP + MN + 2. * ME + MHE) / 5.
M_BLH = 3. * MSUN
BHS = 0.6
L_UNIT = GNEWT * M_BLH / (CL * CL)
RHO_SCALE = 1.5e-5
M_UNIT = RHO_SCALE * MSUN
RHO_UNIT = M_UNIT / (L_UNIT * L_UNIT * L_UNIT)
U_UNIT = RHO_UNIT * CL * CL * 1.0
P_UNIT = U_UNIT


def constants(gam, rho=(1.e2, 1.e15), T=(1.e4, 1.e18)):
    """The unit and range constants harm_cool_b200.Eos takes."""
    return {"rho_unit": RHO_UNIT, "u_unit": U_UNIT, "p_unit": P_UNIT, "kbol": KBOL, "mav": MAV, "cl": CL,
            "rho_min": rho[0], "rho_max": rho[1], "t_min": T[0], "t_max": T[1], "hh": 1.0e-6, "gam": gam,
            "l_unit": L_UNIT}


def log_axis(n, lo, hi):
    """Cache4d::setindices, LOGARITHMIC (cache4d.c:336-343)."""
    delta = (math.log10(hi) - math.log10(lo)) / (n - 1)
    return np.array([10.0 ** (math.log10(lo) + delta * r) for r in range(n)])


def hdfac(r):
    """HdFac of the table at radius r (cooleos.c:945-960)."""
    omega = CL * CL * CL / GNEWT / M_BLH / (BHS + r ** 1.5)
    return 1.0 / omega


def zone_radii(problem):
    """Radius of the zone centre of every radial index 0..N1+3 (coord() and
    bl_coord() on the modified Kerr-Schild grid)."""
    p, g = problem.params, problem.grid
    return np.array([math.exp(p.startx[1] + ((i - 2) + 0.5) * p.dx[1]) + g.R0 for i in range(p.n1 + 4)])


def ideal_gas_radiation(rho, T, hd):
    """Synthetic stand-in for abundance(): nucleons and electrons as ideal gases
    (Ye = 1/2) plus black-body radiation; returns e, p, Qnu, tau, xnee, xnep."""
    kB, mu, arad = 1.380649e-16, 1.66053907e-24, 7.5657e-15
    nb = rho / mu
    pgas = 1.5 * nb * kB * T
    prad = arad * T ** 4 / 3.0
    qnu = 1.0e-39 * rho * T ** 3
    return (1.5 * pgas + 3.0 * prad, pgas + prad, qnu, 1.0e-10 * qnu * hd,
            0.5 * rho / 1.66e15, np.zeros_like(rho))


def build_tables(radii, generator=ideal_gas_radiation, nx=72, ny=72, rho=(1.e2, 1.e15), T=(1.e4, 1.e18),
                 gam=4. / 3.):
    """Tables for the given radial indices: (xaxis, yaxis, values[ntab][nx][ny][5],
    constants with each table's HdFac), values packed as calc_cache_val packs them
    (cooleos.c:171-194)."""
    xa, ya = log_axis(nx, *rho), log_axis(ny, *T)
    R, TT = np.meshgrid(xa, ya, indexing="ij")
    val = np.zeros((len(radii), nx, ny, 5))
    for t, r in enumerate(radii):
        e, p, qnu, tau, xnee, xnep = generator(R, TT, hdfac(r))
        val[t, ..., 0], val[t, ..., 1], val[t, ..., 2], val[t, ..., 3] = e, p, qnu, tau
        val[t, ..., 4] = (xnee - xnep) / (R / 1.66e15)
    c = constants(gam, rho, T)
    c["hdfac"] = np.array([hdfac(r) for r in radii])
    return xa, ya, val, c


def physical_tables(radii, nx=72, ny=72, rho=(1.e2, 1.e15), T=(1.e4, 1.e18), gam=4. / 3., device=0):
    """Tables of the library's abundance() (harm_cool_b200.nu_tables, on the
    GPU), every node computed, laid out as build_tables() lays them out:
    (xaxis, yaxis, values, constants, info); info gives the nodes and the
    device time.  on_demand() computes only the nodes a run reads."""
    from . import nu_tables
    xa, ya = log_axis(nx, *rho), log_axis(ny, *T)
    hd = np.array([hdfac(r) for r in radii])
    val, ms = nu_tables(xa, ya, hd, device=device)
    c = constants(gam, rho, T)
    c["hdfac"] = hd
    nodes = len(radii) * nx * ny
    return xa, ya, val, c, {"nodes": nodes, "device_ms": ms, "nodes_per_s": nodes / (ms / 1e3)}


def fill_nodes(val, xa, ya, hd, mask, device=0):
    """Compute the nodes where mask is set ([ntab][nx][ny]) with the library's
    abundance() on the GPU and write them into val, packed as calc_cache_val
    packs them; returns (nodes, device seconds)."""
    from . import nu_abundance
    import time
    t, i, j = np.nonzero(mask)
    if len(t) == 0:
        return 0, 0.0
    rho = xa[i]
    t0 = time.perf_counter()
    a = nu_abundance(rho, ya[j], hd[t], device=device)
    s = time.perf_counter() - t0
    val[t, i, j, 0], val[t, i, j, 1], val[t, i, j, 2], val[t, i, j, 3] = a["e"], a["p"], a["qnu"], a["tau"]
    val[t, i, j, 4] = (a["nee"] - a["nep"]) / (rho / 1.66e15)
    return len(t), s


def on_demand(run, xa, ya, consts, margin=2, max_passes=40, device=0, make_eos=None, fill=None):
    """A run on tables filled as it reads them, the way the reference's cache
    fills its nodes.  run(eos) makes a fresh run on the given tables and
    returns its result.  Every node starts as NaN; after each run the nodes it
    read as NaN, with margin nodes around them in rho and T, are computed on
    the GPU, and the run starts again.  The first run that reads no NaN node
    read only computed nodes, so it is the run on complete tables.  Returns its
    result, a summary of the passes and the mask of computed nodes.
    make_eos(xa, ya, val, consts) and fill(val, xa, ya, hd, mask, device) stand
    in for harm_cool_b200.Eos and fill_nodes (tests drive the loop with them)."""
    if make_eos is None:
        from . import Eos as make_eos
    fill = fill_nodes if fill is None else fill
    hd = np.asarray(consts["hdfac"])
    val = np.full((len(hd), len(xa), len(ya), 5), np.nan)
    have = np.zeros(val.shape[:3], dtype=bool)
    passes = []
    for _ in range(max_passes):
        eos = make_eos(xa, ya, val, consts)
        eos.track_missing()
        result = run(eos)
        miss = eos.missing()
        eos.close()
        if not miss.any():
            info = {"passes": len(passes) + 1, "nodes": int(have.sum()), "nodes_total": int(have.size),
                    "generation_s": sum(p[1] for p in passes), "per_pass": passes}
            return result, info, have
        grow = miss.copy()
        for _ in range(margin):
            g = grow.copy()
            g[:, 1:, :] |= grow[:, :-1, :]
            g[:, :-1, :] |= grow[:, 1:, :]
            g[:, :, 1:] |= grow[:, :, :-1]
            g[:, :, :-1] |= grow[:, :, 1:]
            grow = g
        grow &= ~have
        n, s = fill(val, xa, ya, hd, grow, device)
        have |= grow
        passes.append((n, s))
    raise RuntimeError("tables still missing nodes after %d passes" % max_passes)
