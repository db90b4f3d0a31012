"""harm_cool_b200: HARM-COOL's per-zone GRMHD update (the step_ch() path) on B200.

The Python layer is a thin host-side mirror of the reference's calling
surface -- step_ch(), bound_prim(), fixup(), fixup_utoprim(), Utoprim_2d()
(decs.h:548-608) -- over the C ABI in include/harm_b200.h.  All compute runs
in libharm_b200.so's sm_100a kernels; there is no CPU path: without the
library or without a B200 every compute call raises.

Arrays use the reference's layouts: primitives p[SN3][SN1][SN2][8] float64,
pflag int8 [SN3][SN1][SN2], geometry as set_grid() builds it.
"""
import ctypes
import math
import os

import numpy as np

__all__ = ["HarmError", "Params", "GridSpec", "TorusSpec", "Diag", "Problem", "Context", "Ensemble", "Eos",
           "torus_problem", "set_points", "set_grid", "set_katm", "utoprim_2d_batch", "library",
           "NPR", "NPG"]

NPR, NPG = 8, 5
HERE = os.path.dirname(os.path.abspath(__file__))
# HARM_B200_LIB names another build of the library (a variant built for comparison)
LIB_PATH = os.environ.get("HARM_B200_LIB") or os.path.join(HERE, "libharm_b200.so")


class HarmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("harm_b200 error %d: %s" % (code, msg))
        self.code = code


class Params(ctypes.Structure):
    """harm_params: run parameters (decs.h:263-283, init.c:104-125)."""
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int), ("lim", ctypes.c_int),
                ("a", ctypes.c_double), ("gam", ctypes.c_double), ("cour", ctypes.c_double),
                ("defcon", ctypes.c_double), ("tf", ctypes.c_double),
                ("dx", ctypes.c_double * 4), ("startx", ctypes.c_double * 4)]


class GridSpec(ctypes.Structure):
    """harm_grid_spec: modified Kerr-Schild grid (coord.c:61-81, 202-262)."""
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("a", ctypes.c_double), ("Rin", ctypes.c_double), ("Rout", ctypes.c_double),
                ("R0", ctypes.c_double), ("hslope", ctypes.c_double)]


class TorusSpec(ctypes.Structure):
    """harm_torus_spec: Fishbone-Moncrief torus (init.c:70-160)."""
    _fields_ = [("rin", ctypes.c_double), ("rmax", ctypes.c_double), ("kappa", ctypes.c_double),
                ("beta", ctypes.c_double)]


class RestartHeader(ctypes.Structure):
    """harm_restart_header: the reference's restart header (restart.c:103-136)."""
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("t", ctypes.c_double), ("tf", ctypes.c_double), ("nstep", ctypes.c_int),
                ("a", ctypes.c_double), ("gam", ctypes.c_double), ("cour", ctypes.c_double),
                ("DTd", ctypes.c_double), ("DTl", ctypes.c_double), ("DTi", ctypes.c_double),
                ("DTr", ctypes.c_int), ("dump_cnt", ctypes.c_int), ("image_cnt", ctypes.c_int),
                ("rdump_cnt", ctypes.c_int), ("dt", ctypes.c_double), ("lim", ctypes.c_int),
                ("failed", ctypes.c_int), ("Rin", ctypes.c_double), ("Rout", ctypes.c_double),
                ("hslope", ctypes.c_double), ("R0", ctypes.c_double), ("mass_start", ctypes.c_double),
                ("mass_in", ctypes.c_double), ("mass_out", ctypes.c_double), ("tdump", ctypes.c_double),
                ("timage", ctypes.c_double), ("tlog", ctypes.c_double), ("defcon", ctypes.c_double),
                ("nfailed", ctypes.c_int), ("Rbr", ctypes.c_double), ("cyl_R0", ctypes.c_double),
                ("cyl_Th0", ctypes.c_double), ("ener_size", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Integrals(ctypes.Structure):
    """harm_integrals: diag()'s sums and the largest div B (diag.c:113-230)."""
    _fields_ = [("mass", ctypes.c_double), ("ang_mom", ctypes.c_double), ("energy", ctypes.c_double),
                ("divbmax", ctypes.c_double), ("imax", ctypes.c_int * 3),
                ("lnu", ctypes.c_double), ("lnu_rho", ctypes.c_double), ("lnu_rho_2", ctypes.c_double),
                ("lnu2", ctypes.c_double)]


class Diag(ctypes.Structure):
    """harm_diag: per-step diagnostics (diag.c:437-580) and the first failure."""
    _fields_ = [("mdot", ctypes.c_double), ("edot", ctypes.c_double), ("ldot", ctypes.c_double),
                ("mdot_in", ctypes.c_double), ("mdot_out", ctypes.c_double),
                ("mass_curr", ctypes.c_double), ("mass_in", ctypes.c_double),
                ("mass_out", ctypes.c_double), ("ndt", ctypes.c_double),
                ("fail_code", ctypes.c_int), ("fail_h", ctypes.c_int), ("fail_i", ctypes.c_int),
                ("fail_j", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


EOS_CONSTANTS = ("rho_unit", "u_unit", "p_unit", "kbol", "mav", "cl", "rho_min", "rho_max",
                 "t_min", "t_max", "hh", "gam")


class EosDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("ntab", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in EOS_CONSTANTS] + [("l_unit", ctypes.c_double)]


_DP = ctypes.POINTER(ctypes.c_double)
_BP = ctypes.POINTER(ctypes.c_byte)
_lib = None

# every symbol include/harm_b200.h declares, with its ctypes signature
_SIGNATURES = {
    "harm_last_error": (ctypes.c_char_p, []),
    "harm_set_points": (ctypes.c_int, [ctypes.POINTER(GridSpec), _DP, _DP]),
    "harm_set_grid": (ctypes.c_int, [ctypes.POINTER(GridSpec), _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
    "harm_set_katm": (ctypes.c_int, [ctypes.POINTER(GridSpec), ctypes.c_double, _DP, _DP]),
    "harm_create": (ctypes.c_int, [ctypes.POINTER(Params), _DP, _DP, _DP, _DP, _DP, _DP, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "harm_destroy": (None, [ctypes.c_void_p]),
    "harm_init_torus": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GridSpec), ctypes.POINTER(TorusSpec)]),
    "harm_put_prims": (ctypes.c_int, [ctypes.c_void_p, _DP, _BP]),
    "harm_get_prims": (ctypes.c_int, [ctypes.c_void_p, _DP, _BP]),
    "harm_set_time": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]),
    "harm_get_time": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP]),
    "harm_set_mass": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]),
    "harm_get_diag": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Diag)]),
    "harm_set_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "harm_step_ch": (ctypes.c_int, [ctypes.c_void_p]),
    "harm_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "harm_step_ch_host": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "harm_run_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _DP]),
    "harm_adjoint_mass_in": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _DP, _DP, _DP]),
    "harm_step_ch_host_timed": (ctypes.c_int, [ctypes.c_void_p, _DP, ctypes.c_int, _DP]),
    "harm_run_host": (ctypes.c_int, [ctypes.c_void_p, _DP, ctypes.c_int]),
    "harm_time_kernels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _DP]),
    "harm_fixup": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_bound_prim": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_fixup_utoprim": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_fixup1zone": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, ctypes.POINTER(ctypes.c_int), _DP, _BP]),
    "harm_utoprim_2d_batch": (ctypes.c_int, [_DP, _DP, _DP, _DP, _DP, ctypes.POINTER(ctypes.c_int),
                                             ctypes.c_long, ctypes.c_double]),
    "harm_utoprim_fix_batch": (ctypes.c_int, [ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP, ctypes.POINTER(ctypes.c_int),
                                              ctypes.c_long, ctypes.c_double]),
    "harm_pow_batch": (ctypes.c_int, [ctypes.c_int, _DP, _DP, _DP, ctypes.c_long]),
    "harm_restart_write": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RestartHeader), ctypes.POINTER(GridSpec),
                                          ctypes.c_char_p]),
    "harm_restart_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(GridSpec),
                                         ctypes.POINTER(RestartHeader)]),
    "harm_diag_integrals": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Integrals)]),
    "harm_tracers_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GridSpec), ctypes.POINTER(ctypes.c_long)]),
    "harm_tracers_put": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GridSpec), ctypes.POINTER(ctypes.c_int), _DP,
                                        ctypes.c_long]),
    "harm_tracers_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]),
    "harm_tracers_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), _DP, _BP]),
    "harm_set_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "harm_get_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "harm_autotune_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    "harm_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "harm_ensemble_destroy": (None, [ctypes.c_void_p]),
    "harm_ensemble_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "harm_ensemble_run_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _DP]),
    "harm_utoprim_2d_batch_noalloc": (ctypes.c_int, [_DP, _DP, _DP, _DP, _DP, ctypes.POINTER(ctypes.c_int),
                                                     ctypes.c_long, ctypes.c_double]),
    "harm_eos_create": (ctypes.c_int, [ctypes.POINTER(EosDesc), _DP, _DP, _DP, _DP,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "harm_eos_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "harm_eos_track_missing": (ctypes.c_int, [ctypes.c_void_p]),
    "harm_eos_missing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "harm_eos_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                      ctypes.POINTER(ctypes.c_int), _DP, _DP, _DP, _DP]),
    "harm_utoprim_5d_batch": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, _DP, _DP, ctypes.POINTER(ctypes.c_int), _DP,
                                             _DP, ctypes.POINTER(ctypes.c_int), ctypes.c_long]),
    "harm_set_eos": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "harm_dump_write": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RestartHeader), ctypes.POINTER(GridSpec),
                                       ctypes.c_char_p]),
    "harm_get_eos_guess": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_put_eos_guess": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "harm_fp64_peak": (ctypes.c_int, [ctypes.c_int, _DP]),
    "harm_div_check": (ctypes.c_int, [ctypes.c_int, ctypes.c_long, ctypes.c_ulonglong,
                                      ctypes.POINTER(ctypes.c_ulonglong)]),
    "harm_pow_check": (ctypes.c_int, [ctypes.c_int, ctypes.c_long, ctypes.c_ulonglong,
                                      ctypes.POINTER(ctypes.c_ulonglong)]),
    "harm_nu_rules": (ctypes.c_int, [_DP]),
    "harm_nu_fermi": (ctypes.c_int, [_DP, _DP, ctypes.c_long, _DP]),
    "harm_nu_abundance": (ctypes.c_int, [_DP, _DP, _DP, ctypes.c_long, ctypes.c_int, _DP]),
    "harm_nu_abundance_dev": (ctypes.c_int, [ctypes.c_int, _DP, _DP, _DP, ctypes.c_long, _DP]),
    "harm_nu_tables": (ctypes.c_int, [ctypes.c_int, _DP, ctypes.c_int, _DP, ctypes.c_int, _DP, ctypes.c_int,
                                      ctypes.c_long, _DP, ctypes.POINTER(ctypes.c_float)]),
}


def library():
    """Load libharm_b200.so (built in-tree by harm_cool_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HarmError(-3, "libharm_b200.so is not built; run harm_cool_b200.build.build()")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def fp64_peak(device=0):
    """Measured FP64 pipe rates of the device: DFMA, DADD and DMUL thread
    instructions per second, IEEE divisions and reciprocals per second."""
    out = np.zeros(5)
    _check(library().harm_fp64_peak(device, _dp(out)))
    return {"dfma_inst_per_s": out[0], "dadd_inst_per_s": out[1], "dmul_inst_per_s": out[2],
            "ddiv_per_s": out[3], "drcp_per_s": out[4]}


def utoprim_fix_batch(which, U, gcov, gcon, gdet, K, prim, gam):
    """Utoprim_1dvsq2fix1 (which 1) or Utoprim_1dfix1 (which 2) over zones; prim
    (the guess) is updated in place; returns the reference's return codes."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    gcov = np.ascontiguousarray(gcov, dtype=np.float64)
    gcon = np.ascontiguousarray(gcon, dtype=np.float64)
    gdet = np.ascontiguousarray(gdet, dtype=np.float64)
    K = np.ascontiguousarray(K, dtype=np.float64)
    assert prim.flags["C_CONTIGUOUS"] and prim.dtype == np.float64
    ret = np.zeros(len(U), dtype=np.int32)
    _check(library().harm_utoprim_fix_batch(which, _dp(U), _dp(gcov), _dp(gcon), _dp(gdet), _dp(K), _dp(prim),
                                            ret.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(U), gam))
    return ret


def pow_batch(x, y, device=0):
    """The device's correctly rounded x**y (the fall-back inversions' power)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros_like(x)
    _check(library().harm_pow_batch(device, _dp(x), _dp(y), _dp(out), len(x)))
    return out


def div_check(n, seed=1, device=0):
    """The library's shared-divisor division against IEEE division on the device:
    (samples that differ, near-midpoint samples drawn)."""
    c = (ctypes.c_ulonglong * 2)()
    _check(library().harm_div_check(device, n, seed, c))
    return int(c[0]), int(c[1])


def nu_rules():
    """The quadrature rules of the COOL_EOS generator: 20- and 40-point
    Gauss-Legendre (positive abscissae, weights) and 20-point Gauss-Laguerre
    (abscissae, weights times e^x)."""
    out = np.zeros(100)
    _check(library().harm_nu_rules(_dp(out)))
    return {"l20": (out[0:10], out[10:20]), "l40": (out[20:40], out[40:60]), "g20": (out[60:80], out[80:100])}


def nu_fermi(eta, theta):
    """F_k(eta, theta) for k = 1/2, 3/2, 5/2, 7/2 (host): shape (n, 4)."""
    eta = np.ascontiguousarray(eta, dtype=np.float64).ravel()
    theta = np.ascontiguousarray(np.broadcast_to(theta, eta.shape), dtype=np.float64)
    F = np.zeros((len(eta), 4))
    _check(library().harm_nu_fermi(_dp(eta), _dp(theta), len(eta), _dp(F)))
    return F


_NU_FIELDS = ("e", "p", "qnu", "tau", "nee", "nep", "xp")


def nu_abundance(rho, T, hdfac, threads=0, device=None):
    """abundance() at the given nodes, on the host's cores (device None) or on a
    GPU: a dict of arrays e, p (erg/cm^3), qnu (erg/cm^2/s), tau, nee, nep
    (fm^-3) and xp (proton fraction of the free nucleons)."""
    rho, T, hdfac = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in np.broadcast_arrays(rho, T, hdfac))
    out = np.zeros((len(rho), 7))
    if device is None:
        _check(library().harm_nu_abundance(_dp(rho), _dp(T), _dp(hdfac), len(rho), threads, _dp(out)))
    else:
        _check(library().harm_nu_abundance_dev(device, _dp(rho), _dp(T), _dp(hdfac), len(rho), _dp(out)))
    return {k: out[:, i].copy() for i, k in enumerate(_NU_FIELDS)}


def nu_tables(xaxis, yaxis, hdfac, device=0, slice_nodes=0):
    """Every node of the per-radius tables on the GPU: values[ntab][nx][ny][5]
    (e, p, Qnu, tau, Yee) and the build's device time in ms."""
    xaxis = np.ascontiguousarray(xaxis, dtype=np.float64)
    yaxis = np.ascontiguousarray(yaxis, dtype=np.float64)
    hdfac = np.ascontiguousarray(hdfac, dtype=np.float64)
    val = np.zeros((len(hdfac), len(xaxis), len(yaxis), 5))
    ms = ctypes.c_float(0.)
    _check(library().harm_nu_tables(device, _dp(xaxis), len(xaxis), _dp(yaxis), len(yaxis), _dp(hdfac), len(hdfac),
                                     slice_nodes, _dp(val), ctypes.byref(ms)))
    return val, ms.value


def pow_check(n, seed=1, device=0):
    """The fall-back inversions' cube-root power against the general one on the
    device: (samples that differ, samples left to the general path)."""
    c = (ctypes.c_ulonglong * 2)()
    _check(library().harm_pow_check(device, n, seed, c))
    return int(c[0]), int(c[1])


def _check(rc):
    if rc != 0:
        raise HarmError(rc, library().harm_last_error().decode())
    return rc


def _dp(a):
    return a.ctypes.data_as(_DP)


def _shape3(n1, n2, n3):
    return (n3 + 2 if n3 > 1 else 1, n1 + 4, n2 + 4)


# ---------------------------------------------------------------------------
# host-side grid set-up (no GPU needed)

def set_points(gs):
    dx = (ctypes.c_double * 4)()
    sx = (ctypes.c_double * 4)()
    _check(library().harm_set_points(ctypes.byref(gs), dx, sx))
    return list(dx), list(sx)


def set_grid(gs, dx, sx):
    """Geometry of the 2D (r, theta) grid, reference layout (main.c:413-520)."""
    sn1, sn2 = gs.n1 + 4, gs.n2 + 4
    g = {"gcov": np.zeros((sn1, sn2, NPG, 4, 4)), "gcon": np.zeros((sn1, sn2, NPG, 4, 4)),
         "gdet": np.zeros((sn1, sn2, NPG)), "conn": np.zeros((sn1, sn2, 4, 4, 4)),
         "coords": np.zeros((sn1, sn2, 4))}
    cdx = (ctypes.c_double * 4)(*dx)
    csx = (ctypes.c_double * 4)(*sx)
    _check(library().harm_set_grid(ctypes.byref(gs), cdx, csx, _dp(g["gcov"]), _dp(g["gcon"]),
                                   _dp(g["gdet"]), _dp(g["conn"]), _dp(g["coords"])))
    return g


def set_katm(gs, gam, coords):
    katm = np.zeros(gs.n1 + 4)
    _check(library().harm_set_katm(ctypes.byref(gs), gam, _dp(np.ascontiguousarray(coords)), _dp(katm)))
    return katm


class Problem:
    """Everything init() fixes before the first step: parameters, grid, torus, geometry."""

    def __init__(self, params, grid, torus, geometry):
        self.params, self.grid, self.torus, self.geometry = params, grid, torus, geometry

    @property
    def shape(self):
        return _shape3(self.params.n1, self.params.n2, self.params.n3)

    @property
    def zones(self):
        return self.params.n1 * self.params.n2 * self.params.n3


def torus_problem(n1, n2, n3, a=0.9375, rin=6.0, rmax=12.0, beta=100.0, kappa=1.e-3, gam=4. / 3.,
                  cour=0.9, hslope=0.3, Rout=100.0, R0=0.0, tf=20000.0, lim=0):
    """The reference's torus set-up (init.c:70-160) for a given grid and torus.

    Defaults are the benchmark torus: a=0.9375, rin=6, rmax=12, beta=100,
    kappa=1e-3, gamma=4/3, hslope=0.3, Rout=100, inner radius 0.98 r_horizon."""
    Rin = 0.98 * (1. + math.sqrt(1. - a * a))
    gs = GridSpec(n1, n2, n3, a, Rin, Rout, R0, hslope)
    dx, sx = set_points(gs)
    geom = set_grid(gs, dx, sx)
    geom["katm"] = set_katm(gs, gam, geom["coords"])
    p = Params()
    p.n1, p.n2, p.n3, p.lim = n1, n2, n3, lim
    p.a, p.gam, p.cour, p.defcon, p.tf = a, gam, cour, 1.0, tf
    for k in range(4):
        p.dx[k] = dx[k]
        p.startx[k] = sx[k]
    return Problem(p, gs, TorusSpec(rin, rmax, kappa, beta), geom)


def utoprim_2d_batch(U, gcov, gcon, gdet, prim, gam):
    """Utoprim_2d() (utoprim_2d.c:126) on the device for n independent zones.

    prim holds the guess on entry and the result on exit; returns the
    reference's return codes."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    gcov = np.ascontiguousarray(gcov, dtype=np.float64)
    gcon = np.ascontiguousarray(gcon, dtype=np.float64)
    gdet = np.ascontiguousarray(gdet, dtype=np.float64)
    assert prim.flags["C_CONTIGUOUS"] and prim.dtype == np.float64
    n = U.shape[0]
    ret = np.zeros(n, dtype=np.int32)
    _check(library().harm_utoprim_2d_batch(_dp(U), _dp(gcov), _dp(gcon), _dp(gdet), _dp(prim),
                                           ret.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, gam))
    return ret


class Eos:
    """Run-time COOL_EOS tables on the device (the reference's per-radius cacheT
    tables, SetupCache_CoolEOS, cooleos.c:825-992) and batch calls of
    pressure_rho0_u_CoolEOS / dpdu_calc_CoolEOS / dpdrho_calc_CoolEOS.

    xaxis[nx] (rho, g/cm^3), yaxis[ny] (T, K), values[ntab][nx][ny][5] with
    e, p, Qnu, tau, Yee per node, consts: the unit and range constants named in
    EOS_CONSTANTS, and for the cooling diagnostics "l_unit" and "hdfac" (each
    table's HdFac)."""

    WHAT = {"pressure": 0, "dpdu": 1, "dpdrho": 2}

    def __init__(self, xaxis, yaxis, values, consts):
        self.xaxis = np.ascontiguousarray(xaxis, dtype=np.float64)
        self.yaxis = np.ascontiguousarray(yaxis, dtype=np.float64)
        v = np.ascontiguousarray(values, dtype=np.float64)
        ntab, nx, ny, nd = v.shape
        if nd != 5 or nx != len(self.xaxis) or ny != len(self.yaxis):
            raise ValueError("values must be [ntab][nx][ny][5]")
        d = EosDesc(nx=nx, ny=ny, ntab=ntab, l_unit=float(consts.get("l_unit", 0.0)),
                    **{k: float(consts[k]) for k in EOS_CONSTANTS})
        hd = consts.get("hdfac")
        hd = None if hd is None else np.ascontiguousarray(hd, dtype=np.float64)
        if hd is not None and len(hd) != ntab:
            raise ValueError("hdfac needs one value per table")
        h = ctypes.c_void_p()
        _check(library().harm_eos_create(ctypes.byref(d), _dp(self.xaxis), _dp(self.yaxis), _dp(v),
                                         _dp(hd) if hd is not None else None, ctypes.byref(h)))
        self.h = h
        self.ntab, self.consts = ntab, dict(consts)

    def batch(self, what, tab, rho0, u, lastT, mixed=False):
        """One call per entry, each from its own temperature guess; returns
        (values, guesses after).  mixed: interpolation and T solve in FP32."""
        tab = np.ascontiguousarray(tab, dtype=np.int32)
        rho0 = np.ascontiguousarray(rho0, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        lt = np.array(lastT, dtype=np.float64)
        out = np.zeros(len(tab))
        _check(library().harm_eos_batch(self.h, self.WHAT[what], 1 if mixed else 0, len(tab),
                                        tab.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(rho0), _dp(u),
                                        _dp(lt), _dp(out)))
        return out, lt

    def pressure(self, tab, rho0, u, lastT):
        return self.batch("pressure", tab, rho0, u, lastT)

    def track_missing(self):
        """Mark the NaN nodes that table reads meet from now on (before set_eos)."""
        _check(library().harm_eos_track_missing(self.h))

    def missing(self):
        """The marked nodes: bool [ntab][nx][ny]."""
        m = np.zeros((self.ntab, len(self.xaxis), len(self.yaxis)), dtype=np.uint8)
        _check(library().harm_eos_missing(self.h, m.ctypes.data))
        return m.astype(bool)

    def utoprim_5d(self, U, gcov, gcon, gdet, tab, lastT, prim):
        """Utoprim_5d (utoprim_5d.c:179) for n independent zones with tables tab[n]
        and guesses lastT[n]; prim holds the guess on entry and the result on
        exit.  Returns (codes, guesses after)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        gcov = np.ascontiguousarray(gcov, dtype=np.float64)
        gcon = np.ascontiguousarray(gcon, dtype=np.float64)
        gdet = np.ascontiguousarray(gdet, dtype=np.float64)
        tab = np.ascontiguousarray(tab, dtype=np.int32)
        lt = np.array(lastT, dtype=np.float64)
        assert prim.flags["C_CONTIGUOUS"] and prim.dtype == np.float64
        n = U.shape[0]
        ret = np.zeros(n, dtype=np.int32)
        _check(library().harm_utoprim_5d_batch(self.h, _dp(U), _dp(gcov), _dp(gcon), _dp(gdet),
                                               tab.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(lt), _dp(prim),
                                               ret.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n))
        return ret, lt

    def close(self):
        if getattr(self, "h", None):
            library().harm_eos_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# device context

class Context:
    """One grid's state resident on one GPU, driven like the reference's globals."""

    def __init__(self, problem, device=0):
        self.problem = problem
        self.lib = library()
        g = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in problem.geometry.items()}
        self._geom = g
        h = ctypes.c_void_p()
        _check(self.lib.harm_create(ctypes.byref(problem.params), _dp(g["gcov"]), _dp(g["gcon"]),
                                    _dp(g["gdet"]), _dp(g["conn"]), _dp(g["coords"]), _dp(g["katm"]),
                                    device, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.harm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return self.problem.shape

    def init_torus(self):
        """init() (init.c:70-472): the torus, resident on the device; t=0, dt=1e-5."""
        pr = self.problem
        _check(self.lib.harm_init_torus(self.h, ctypes.byref(pr.grid), ctypes.byref(pr.torus)))

    def put_prims(self, p, pflag=None):
        p = np.ascontiguousarray(p, dtype=np.float64)
        assert p.shape == self.shape + (NPR,)
        fl = None
        if pflag is not None:
            pflag = np.ascontiguousarray(pflag, dtype=np.int8)
            fl = pflag.ctypes.data_as(_BP)
        _check(self.lib.harm_put_prims(self.h, _dp(p), fl))

    def get_prims(self, with_flags=False):
        p = np.empty(self.shape + (NPR,))
        fl = np.empty(self.shape, dtype=np.int8) if with_flags else None
        _check(self.lib.harm_get_prims(self.h, _dp(p), fl.ctypes.data_as(_BP) if with_flags else None))
        return (p, fl) if with_flags else p

    def set_time(self, t, dt):
        _check(self.lib.harm_set_time(self.h, t, dt))

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.harm_get_time(self.h, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def set_mass(self, mass_in, mass_out):
        _check(self.lib.harm_set_mass(self.h, mass_in, mass_out))

    def diag(self):
        d = Diag()
        _check(self.lib.harm_get_diag(self.h, ctypes.byref(d)))
        return d.as_dict()

    FP64, MIXED = 0, 1

    def set_precision(self, mode):
        """Context.FP64 (default, bit-compatible with the reference) or Context.MIXED."""
        _check(self.lib.harm_set_precision(self.h, mode))

    def set_eos(self, eos):
        """Step with COOL_EOS on the given Eos tables (one per radial index,
        N1+4 of them); None goes back to the gamma-law step."""
        _check(self.lib.harm_set_eos(self.h, eos.h if eos is not None else None))
        self._eos = eos  # the tables must outlive the attachment

    def eos_guess(self):
        """The per-zone temperature guesses _aLastT[SN3][SN1][SN2] (cooleos.c:69)."""
        a = np.zeros(self.shape)
        _check(self.lib.harm_get_eos_guess(self.h, _dp(a)))
        return a

    def put_eos_guess(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape
        _check(self.lib.harm_put_eos_guess(self.h, _dp(a)))

    def step_ch(self):
        """One full step (step_ch.c:90-140), asynchronous; see sync()."""
        _check(self.lib.harm_step_ch(self.h))

    def run(self, nsteps):
        """nsteps steps replayed from one captured CUDA graph; synchronises."""
        _check(self.lib.harm_run(self.h, nsteps))

    def run_timed(self, nsteps):
        """run() with the device time of the nsteps graph launches, in ms."""
        ms = ctypes.c_double()
        _check(self.lib.harm_run_timed(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def step_ch_host_timed(self, p, nsteps):
        """run_host() timed on the device, in ms."""
        assert p.flags["C_CONTIGUOUS"] and p.dtype == np.float64 and p.shape == self.shape + (NPR,)
        ms = ctypes.c_double()
        _check(self.lib.harm_step_ch_host_timed(self.h, _dp(p), nsteps, ctypes.byref(ms)))
        return ms.value

    KERNELS = ("flux", "update", "bound_prim", "fixup_utoprim", "diag")

    def time_kernels(self, reps=5):
        """Average device ms per launch of each step kernel, launched on its own."""
        ms = (ctypes.c_double * len(self.KERNELS))()
        _check(self.lib.harm_time_kernels(self.h, reps, ms))
        return dict(zip(self.KERNELS, list(ms)))

    def sync(self):
        _check(self.lib.harm_sync(self.h))

    def restart_write(self, path, **fields):
        """restart_write(): the state in the reference's restart format; header fields
        the device does not own come from `fields` (defaults: this problem's parameters,
        zeros elsewhere)."""
        pr = self.problem
        hd = RestartHeader()
        hd.tf, hd.a, hd.gam, hd.cour = pr.params.tf, pr.params.a, pr.params.gam, pr.params.cour
        hd.lim, hd.defcon = pr.params.lim, pr.params.defcon
        hd.Rin, hd.Rout, hd.hslope, hd.R0 = pr.grid.Rin, pr.grid.Rout, pr.grid.hslope, pr.grid.R0
        hd.Rbr = -1.0
        for k, v in fields.items():
            setattr(hd, k, v)
        _check(self.lib.harm_restart_write(self.h, ctypes.byref(hd), ctypes.byref(pr.grid), path.encode()))

    def dump_write(self, path, **fields):
        """dump(): the reference's ASCII dump of the state; header fields as for
        restart_write()."""
        pr = self.problem
        hd = RestartHeader()
        hd.tf, hd.a, hd.gam, hd.cour = pr.params.tf, pr.params.a, pr.params.gam, pr.params.cour
        hd.lim, hd.defcon = pr.params.lim, pr.params.defcon
        hd.Rin, hd.Rout, hd.hslope, hd.R0 = pr.grid.Rin, pr.grid.Rout, pr.grid.hslope, pr.grid.R0
        hd.Rbr = -1.0
        for k, v in fields.items():
            setattr(hd, k, v)
        _check(self.lib.harm_dump_write(self.h, ctypes.byref(hd), ctypes.byref(pr.grid), path.encode()))

    def adjoint_mass_in(self, nsteps, checkpoint_every=10):
        """Discrete adjoint of nsteps steps (2D gamma-law FP64 step): runs them from
        the current state and returns (J, grad, ms) -- J the mass that crossed the
        inner boundary (the change of mass_in, diag.c:578), grad = dJ/dp of the state
        at the call in get_prims' layout, ms the device time of the forward pass and
        of the reverse sweep."""
        J = ctypes.c_double()
        grad = np.zeros(self.shape + (NPR,))
        ms = (ctypes.c_double * 2)()
        _check(self.lib.harm_adjoint_mass_in(self.h, nsteps, checkpoint_every, ctypes.byref(J), _dp(grad), ms))
        return J.value, grad, (ms[0], ms[1])

    def restart_read(self, path):
        """restart_init(): state, time, mass counters and tracers from a restart file."""
        hd = RestartHeader()
        _check(self.lib.harm_restart_read(self.h, path.encode(), ctypes.byref(self.problem.grid), ctypes.byref(hd)))
        return hd.as_dict()

    def integrals(self):
        """diag()'s integrals: mass, angular momentum, energy, divbmax and its zone."""
        d = Integrals()
        _check(self.lib.harm_diag_integrals(self.h, ctypes.byref(d)))
        return {"rmed": d.mass, "pp": d.ang_mom, "e": d.energy, "divbmax": d.divbmax, "imax": list(d.imax),
                "lnu": d.lnu, "lnu_rho": d.lnu_rho, "lnu_rho_2": d.lnu_rho_2, "lnu2": d.lnu2}

    # tracer particles (tracers.c)
    def tracers_init(self):
        """init_tracers(): a tracer at every zone centre with rho > RHOMIN; returns the count."""
        n = ctypes.c_long()
        _check(self.lib.harm_tracers_init(self.h, ctypes.byref(self.problem.grid), ctypes.byref(n)))
        return n.value

    def tracers_put(self, ids, X):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        X = np.ascontiguousarray(X, dtype=np.float64)
        _check(self.lib.harm_tracers_put(self.h, ctypes.byref(self.problem.grid),
                                         ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(X), len(ids)))

    def tracers(self):
        """(ids[n][3], X[n][3], status[n]) of every tracer, retired ones included."""
        n = ctypes.c_long()
        _check(self.lib.harm_tracers_count(self.h, ctypes.byref(n)))
        n = n.value
        ids = np.zeros((n, 3), dtype=np.int32)
        X = np.zeros((n, 3))
        st = np.zeros(n, dtype=np.int8)
        if n:
            _check(self.lib.harm_tracers_get(self.h, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(X),
                                             st.ctypes.data_as(_BP)))
        return ids, X, st

    def set_tile(self, bx, by):
        """Threads per block of the face and zone kernels (bx theta x by r, 128 in all)."""
        _check(self.lib.harm_set_tile(self.h, bx, by))

    def tile(self):
        bx, by = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.harm_get_tile(self.h, ctypes.byref(bx), ctypes.byref(by)))
        return bx.value, by.value

    def autotune_tile(self, steps=3):
        """Time each candidate tile on this state (restored afterwards); keep the fastest."""
        bx, by = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.harm_autotune_tile(self.h, steps, ctypes.byref(bx), ctypes.byref(by)))
        return bx.value, by.value

    def step_ch_host(self, p):
        """step_ch() on a host primitive array, in place (upload, step, download)."""
        assert p.flags["C_CONTIGUOUS"] and p.dtype == np.float64 and p.shape == self.shape + (NPR,)
        _check(self.lib.harm_step_ch_host(self.h, _dp(p)))

    def run_host(self, p, nsteps):
        """nsteps of step_ch_host() on p in place, each step's upload overlapped
        with the previous step's download (harm_run_host)."""
        assert p.flags["C_CONTIGUOUS"] and p.dtype == np.float64 and p.shape == self.shape + (NPR,)
        _check(self.lib.harm_run_host(self.h, _dp(p), nsteps))

    def _on_array(self, fn, pv):
        assert pv.flags["C_CONTIGUOUS"] and pv.dtype == np.float64 and pv.shape == self.shape + (NPR,)
        _check(fn(self.h, _dp(pv)))
        return pv

    def fixup(self, pv):
        """fixup() (fixup.c:51-60) on a host array, in place."""
        return self._on_array(self.lib.harm_fixup, pv)

    def bound_prim(self, pv):
        """bound_prim() (bounds.c:54-331) on a host array, in place."""
        return self._on_array(self.lib.harm_bound_prim, pv)

    def fixup_utoprim(self, pv, pflag=None):
        """fixup_utoprim() (fixup.c:432-538) on a host array, in place; pflag, if
        given, replaces the device's failure flags first."""
        if pflag is not None:
            cur = self.get_prims()
            self.put_prims(cur, pflag)
        return self._on_array(self.lib.harm_fixup_utoprim, pv)


class Ensemble:
    """Independent grids on one GPU advanced together: one CUDA graph launch per
    ensemble step, each member stepping with its own dt (harm_ensemble_*)."""

    def __init__(self, contexts):
        self.lib = library()
        self.members = list(contexts)
        arr = (ctypes.c_void_p * len(self.members))(*[c.h for c in self.members])
        h = ctypes.c_void_p()
        _check(self.lib.harm_ensemble_create(arr, len(self.members), ctypes.byref(h)))
        self.h = h

    def run(self, nsteps):
        _check(self.lib.harm_ensemble_run(self.h, nsteps))

    def run_timed(self, nsteps):
        ms = ctypes.c_double()
        _check(self.lib.harm_ensemble_run_timed(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.harm_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ensemble_problems(n, seed=0, sizes=(96, 128, 192, 256), a_range=(0.0, 0.98), rmax_range=(9.0, 14.0),
                      beta_range=(30.0, 300.0)):
    """n seeded 2D tori for an ensemble run: N1 and N2 drawn independently from
    sizes, spin a, pressure-maximum radius Rmax and plasma beta drawn uniformly;
    the rest as the benchmark torus (rin=6, gamma=4/3, kappa=1e-3, hslope=0.3,
    Rout=100, grid inner radius 0.98 r_horizon).  Returns [(problem, draw)]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        n1 = int(rng.choice(sizes))
        n2 = int(rng.choice(sizes))
        a = float(rng.uniform(*a_range))
        rmax = float(rng.uniform(*rmax_range))
        beta = float(rng.uniform(*beta_range))
        out.append((torus_problem(n1, n2, 1, a=a, rmax=rmax, beta=beta),
                    {"n1": n1, "n2": n2, "a": a, "rmax": rmax, "beta": beta}))
    return out
