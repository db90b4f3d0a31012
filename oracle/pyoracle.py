"""ctypes bindings for the CPU oracle and for the reference checker build.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NPR, NPG = 8, 5


class OraParams(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("lim", ctypes.c_int), ("a", ctypes.c_double), ("gam", ctypes.c_double),
                ("cour", ctypes.c_double), ("defcon", ctypes.c_double), ("tf", ctypes.c_double),
                ("dx", ctypes.c_double * 4), ("startx", ctypes.c_double * 4)]


class OraDiag(ctypes.Structure):
    _fields_ = [("mdot", ctypes.c_double), ("edot", ctypes.c_double), ("ldot", ctypes.c_double),
                ("mdot_in", ctypes.c_double), ("mdot_out", ctypes.c_double),
                ("mass_curr", ctypes.c_double), ("mass_in", ctypes.c_double),
                ("mass_out", ctypes.c_double), ("ndt", ctypes.c_double),
                ("fail_code", ctypes.c_int), ("fail_h", ctypes.c_int), ("fail_i", ctypes.c_int),
                ("fail_j", ctypes.c_int)]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


_oracle_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        path = os.path.join(HERE, "_build", "libharm_oracle.so")
        if not os.path.exists(path):
            from . import build_oracle  # noqa: F401  (package import when available)
        lib = ctypes.CDLL(path)
        lib.ora_create.restype = ctypes.c_void_p
        lib.ora_create.argtypes = [ctypes.POINTER(OraParams)] + [ctypes.POINTER(ctypes.c_double)] * 6
        for name in ("ora_p", "ora_ph"):
            getattr(lib, name).restype = ctypes.POINTER(ctypes.c_double)
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        lib.ora_flux.restype = ctypes.POINTER(ctypes.c_double)
        lib.ora_flux.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ora_pflag.restype = ctypes.POINTER(ctypes.c_byte)
        lib.ora_pflag.argtypes = [ctypes.c_void_p]
        lib.ora_destroy.argtypes = [ctypes.c_void_p]
        lib.ora_step_ch.argtypes = [ctypes.c_void_p]
        lib.ora_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        lib.ora_get_time.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double)]
        lib.ora_set_mass.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        lib.ora_get_diag.argtypes = [ctypes.c_void_p, ctypes.POINTER(OraDiag)]
        for name in ("ora_fixup", "ora_bound_prim", "ora_fixup_utoprim"):
            getattr(lib, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ora_utoprim_2d.argtypes = [ctypes.c_double, dp, dp, dp, ctypes.c_double, dp]
        lib.ora_utoprim_1dvsq2fix1.argtypes = [ctypes.c_double, dp, dp, dp, ctypes.c_double, dp,
                                               ctypes.c_double]
        lib.ora_utoprim_1dfix1.argtypes = [ctypes.c_double, dp, dp, dp, ctypes.c_double, dp,
                                           ctypes.c_double]
        lib.ora_face_flux.argtypes = [ctypes.c_double, ctypes.c_int, dp, dp, dp, dp,
                                      ctypes.c_double, dp, dp]
        ip = ctypes.POINTER(ctypes.c_int)
        lib.ora_tracers_geometry.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        lib.ora_tracers_init.restype = ctypes.c_long
        lib.ora_tracers_init.argtypes = [ctypes.c_void_p]
        lib.ora_tracers_put.argtypes = [ctypes.c_void_p, ip, dp, ctypes.c_long]
        lib.ora_tracers_count.restype = ctypes.c_long
        lib.ora_tracers_count.argtypes = [ctypes.c_void_p]
        lib.ora_tracers_get.argtypes = [ctypes.c_void_p, ip, dp, ctypes.POINTER(ctypes.c_byte)]
        lib.ora_diag_integrals.argtypes = [ctypes.c_void_p, dp, ip]
        _oracle_lib = lib
    return _oracle_lib


def make_params(n1, n2, n3, a, gam, cour, dx, startx, defcon=1.0, tf=20000.0, lim=0):
    p = OraParams()
    p.n1, p.n2, p.n3, p.lim = n1, n2, n3, lim
    p.a, p.gam, p.cour, p.defcon, p.tf = a, gam, cour, defcon, tf
    for k in range(4):
        p.dx[k] = dx[k]
        p.startx[k] = startx[k]
    return p


def shape3(n1, n2, n3):
    return (n3 + 2 if n3 > 1 else 1, n1 + 4, n2 + 4)


class Oracle:
    """One oracle state: prims, fluxes and flags in the reference layout."""

    def __init__(self, params, geom):
        self.lib = oracle_lib()
        self.params = params
        self.geom = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in geom.items()}
        g = self.geom
        self.h = self.lib.ora_create(ctypes.byref(params), _dp(g["gcov"]), _dp(g["gcon"]),
                                     _dp(g["gdet"]), _dp(g["conn"]), _dp(g["coords"]),
                                     _dp(g["katm"]))
        if not self.h:
            raise ValueError("oracle rejected the grid size")
        s3 = shape3(params.n1, params.n2, params.n3)
        n = s3[0] * s3[1] * s3[2]
        self.p = np.ctypeslib.as_array(self.lib.ora_p(self.h), shape=(n * NPR,)).reshape(s3 + (NPR,))
        self.ph = np.ctypeslib.as_array(self.lib.ora_ph(self.h), shape=(n * NPR,)).reshape(s3 + (NPR,))
        self.pflag = np.ctypeslib.as_array(self.lib.ora_pflag(self.h), shape=(n,)).reshape(s3)

    def flux(self, d):
        s3 = self.p.shape
        n = s3[0] * s3[1] * s3[2] * NPR
        return np.ctypeslib.as_array(self.lib.ora_flux(self.h, d), shape=(n,)).reshape(s3)

    def set_time(self, t, dt):
        self.lib.ora_set_time(self.h, t, dt)

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        self.lib.ora_get_time(self.h, ctypes.byref(t), ctypes.byref(dt))
        return t.value, dt.value

    def set_mass(self, mass_in, mass_out):
        self.lib.ora_set_mass(self.h, mass_in, mass_out)

    def diag(self):
        d = OraDiag()
        self.lib.ora_get_diag(self.h, ctypes.byref(d))
        return {f: getattr(d, f) for f, _ in OraDiag._fields_}

    def step(self):
        return self.lib.ora_step_ch(self.h)

    def branch_counts(self, reset=True):
        """floors in the drift frame, inversions rescued by Utoprim_1dvsq2fix1 and by
        Utoprim_1dfix1, since the last reset (process-wide counts)"""
        out = (ctypes.c_long * 3)()
        self.lib.ora_branch_counts(out, 1 if reset else 0)
        return list(out)

    def diag_integrals(self):
        """diag()'s sums (mass, angular momentum, energy), divbmax and its zone."""
        out = np.zeros(4)
        imax = np.zeros(3, dtype=np.int32)
        self.lib.ora_diag_integrals(self.h, _dp(out), imax.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return {"rmed": out[0], "pp": out[1], "e": out[2], "divbmax": out[3], "imax": imax.tolist()}

    # tracer particles (tracers.c)
    def tracers_init(self, R0, hslope):
        self.lib.ora_tracers_geometry(self.h, R0, hslope)
        return self.lib.ora_tracers_init(self.h)

    def tracers_put(self, ids, X, R0, hslope):
        self.lib.ora_tracers_geometry(self.h, R0, hslope)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        X = np.ascontiguousarray(X, dtype=np.float64)
        self.lib.ora_tracers_put(self.h, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(X), len(ids))

    def tracers(self):
        """(ids[n][3], X[n][3], status[n]) for every tracer, retired ones included."""
        n = self.lib.ora_tracers_count(self.h)
        ids = np.zeros((n, 3), dtype=np.int32)
        X = np.zeros((n, 3))
        st = np.zeros(n, dtype=np.int8)
        self.lib.ora_tracers_get(self.h, ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(X),
                                 st.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)))
        return ids, X, st

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.ora_destroy(self.h)
        except Exception:
            pass


EOS_CONSTANTS = ("rho_unit", "u_unit", "p_unit", "kbol", "mav", "cl", "rho_min", "rho_max",
                 "t_min", "t_max", "hh", "gam")


class OraEos(ctypes.Structure):
    _fields_ = ([("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nd", ctypes.c_int), ("ntab", ctypes.c_int),
                 ("xa", ctypes.POINTER(ctypes.c_double)), ("ya", ctypes.POINTER(ctypes.c_double)),
                 ("val", ctypes.POINTER(ctypes.c_double))]
                + [(n, ctypes.c_double) for n in EOS_CONSTANTS])


class EosTables:
    """Run-time COOL_EOS tables: rho axis xa[nx], T axis ya[ny], values
    val[ntab][nx][ny][nd] (e, p, Qnu, tau, Yee per node, cooleos.c:32-37) and the
    unit and range constants (cooleos.c:83-135, 840-940) as a dict."""

    def __init__(self, xa, ya, val, consts):
        self.xa = np.ascontiguousarray(xa, dtype=np.float64)
        self.ya = np.ascontiguousarray(ya, dtype=np.float64)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.consts = dict(consts)
        self.ntab, self.nx, self.ny, self.nd = self.val.shape

    def struct(self):
        e = OraEos(nx=self.nx, ny=self.ny, nd=self.nd, ntab=self.ntab, xa=_dp(self.xa), ya=_dp(self.ya),
                   val=_dp(self.val), **{k: float(self.consts[k]) for k in EOS_CONSTANTS})
        e._keep = self
        return e


class OracleEos:
    """The CPU restatement of the run-time EOS (cooleos_oracle.c) on given tables."""

    WHAT = {"pressure": 0, "dpdu": 1, "dpdrho": 2}

    def __init__(self, tables):
        self.lib = oracle_lib()
        self.tables = tables
        self.s = tables.struct()

    def batch(self, what, tab, rho0, u, lastT):
        """what in pressure/dpdu/dpdrho, one call per entry in order; returns
        (out, lastT after)."""
        tab = np.ascontiguousarray(tab, dtype=np.int32)
        rho0 = np.ascontiguousarray(rho0, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        lt = np.array(lastT, dtype=np.float64)
        out = np.zeros(len(tab))
        self.lib.ora_eos_batch(ctypes.byref(self.s), self.WHAT[what], ctypes.c_long(len(tab)),
                               tab.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(rho0), _dp(u), _dp(lt),
                               _dp(out))
        return out, lt

    def value(self, tab, d, rho, T, der=False):
        v, dv = ctypes.c_double(), ctypes.c_double()
        ok = self.lib.ora_eos_value(ctypes.byref(self.s), tab, d, ctypes.c_double(rho), ctypes.c_double(T),
                                    ctypes.byref(v), ctypes.byref(dv) if der else None)
        if not ok:
            return None
        return (v.value, dv.value) if der else v.value


def standin_tables(startx1, dx1, R0, sn1, gam, nx=72, ny=72, rho=(1.e2, 1.e15), T=(1.e4, 1.e18)):
    """The tables SetupCache_CoolEOS builds (cooleos.c:825-992) for radial indices
    0..sn1-1 of a grid, with oracle/eos_standin.c as the generator, and the unit
    and range constants: what the COOL_EOS checker build computes."""
    lib = oracle_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ora_eos_hdfac.restype = ctypes.c_double
    lib.ora_eos_hdfac.argtypes = [ctypes.c_double]
    lib.ora_zone_r.restype = ctypes.c_double
    lib.ora_zone_r.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.ora_eos_axis.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
    lib.ora_eos_fill.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double, dp]
    lib.ora_eos_constants.argtypes = [ctypes.c_double, dp]
    xa, ya = np.zeros(nx), np.zeros(ny)
    lib.ora_eos_axis(nx, rho[0], rho[1], _dp(xa))
    lib.ora_eos_axis(ny, T[0], T[1], _dp(ya))
    val = np.zeros((sn1, nx, ny, 5))
    hdfac = np.zeros(sn1)
    for i in range(sn1):
        hdfac[i] = lib.ora_eos_hdfac(lib.ora_zone_r(startx1, dx1, R0, i))
        lib.ora_eos_fill(nx, ny, _dp(xa), _dp(ya), hdfac[i], _dp(val[i]))
    c = np.zeros(len(EOS_CONSTANTS))
    lib.ora_eos_constants(gam, _dp(c))
    consts = dict(zip(EOS_CONSTANTS, c.tolist()))
    consts["rho_min"], consts["rho_max"], consts["t_min"], consts["t_max"] = rho[0], rho[1], T[0], T[1]
    # L_UNIT = GNEWT M_BLH / CL^2 (cooleos.c:109), the same operations as the C
    consts["l_unit"] = 6.6742867e-8 * (3. * 1.9892e33) / (2.99792458e10 * 2.99792458e10)
    consts["hdfac"] = hdfac
    return EosTables(xa, ya, val, consts)


class _QuietStdout:
    """Silence file descriptor 1 (the reference prints progress on stdout)."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        fd = os.open(os.devnull, os.O_WRONLY)
        os.dup2(fd, 1)
        os.close(fd)

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)


class Reference:
    """The reference's own step_ch() (oracle/_ref/<config>/libharmref.so).

    One configuration per process: the reference keeps its state in globals."""

    def __init__(self, config):
        path = os.path.join(HERE, "_ref", config, "libharmref.so")
        self.lib = lib = ctypes.CDLL(path)
        lib.ref_get.restype = ctypes.c_double
        lib.ref_get.argtypes = [ctypes.c_char_p]
        lib.ref_set.argtypes = [ctypes.c_char_p, ctypes.c_double]
        lib.ref_ptr.restype = ctypes.c_void_p
        lib.ref_ptr.argtypes = [ctypes.c_char_p]
        lib.ref_utoprim_2d.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
        lib.ref_time_steps.restype = ctypes.c_double
        if hasattr(lib, "ref_tracers_count"):
            lib.ref_tracers_count.restype = ctypes.c_long
        lib.ref_init()
        d = (ctypes.c_int * 16)()
        lib.ref_dims(d)
        self.n1, self.n2, self.n3, self.sn1, self.sn2, self.sn3 = d[0], d[1], d[2], d[3], d[4], d[5]
        s3 = (self.sn3, self.sn1, self.sn2)
        self.p = self._arr("p", s3 + (NPR,))
        self.ph = self._arr("ph", s3 + (NPR,))
        self.pflag = np.ctypeslib.as_array(
            ctypes.cast(lib.ref_ptr(b"pflag"), ctypes.POINTER(ctypes.c_byte)), shape=s3)

    def _arr(self, name, shape, dtype=ctypes.c_double):
        ptr = ctypes.cast(self.lib.ref_ptr(name.encode()), ctypes.POINTER(dtype))
        return np.ctypeslib.as_array(ptr, shape=shape)

    def get(self, name):
        return self.lib.ref_get(name.encode())

    def restart_write(self):
        """restart_write(): the reference's restart file, as text."""
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            os.mkdir(os.path.join(d, "dumps"))
            if self.lib.ref_restart_write(d.encode()) != 0:
                raise RuntimeError("restart_write failed")
            return open(os.path.join(d, "dumps", "rdump1.0_1x1x1")).read()

    def restart_init(self, text):
        """restart_init() from the given restart file text; re-binds the arrays."""
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            os.mkdir(os.path.join(d, "dumps"))
            with open(os.path.join(d, "dumps", "rdump1.0_1x1x1"), "w") as f:
                f.write(text)
            if self.lib.ref_restart_init(d.encode()) != 0:
                raise RuntimeError("restart_init failed")
        s3 = (self.sn3, self.sn1, self.sn2)
        self.p = self._arr("p", s3 + (NPR,))
        self.ph = self._arr("ph", s3 + (NPR,))
        self.pflag = np.ctypeslib.as_array(
            ctypes.cast(self.lib.ref_ptr(b"pflag"), ctypes.POINTER(ctypes.c_byte)), shape=s3)

    def dump(self):
        """dump() (dump.c:1710-2047): the reference's ASCII dump of the state, as text."""
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "dump")
            with _QuietStdout():
                if self.lib.ref_dump(path.encode()) != 0:
                    raise RuntimeError("dump failed")
            return open(path).read()

    def diag_init(self):
        """diag(INIT_OUT): (rmed, pp, e) as ener.out prints them (%10.5g), divbmax as the
        LOG line prints it (%g) and its zone (i, j, h from 0) (diag.c:312-326)."""
        import re
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            os.mkdir(os.path.join(d, "dumps"))
            if self.lib.ref_diag_init(d.encode()) != 0:
                raise RuntimeError("diag(INIT_OUT) failed")
            ener = open(os.path.join(d, "ener.out")).read().split()
            log = open(os.path.join(d, "diag_stderr.txt")).read()
        m = re.search(r"divbmax:\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(\S+)", log)
        return {"rmed": float(ener[1]), "pp": float(ener[2]), "e": float(ener[3]),
                "divbmax": float(m.group(4)), "imax": [int(m.group(1)), int(m.group(2)), int(m.group(3))],
                "ener": [float(v) for v in ener]}

    def tracers(self):
        """The reference's tracer list (tracers.c:24): ids[n][3] = (i, j, h), X[n][3]."""
        n = self.lib.ref_tracers_count()
        ids = np.zeros((n, 3), dtype=np.int32)
        X = np.zeros((n, 3))
        self.lib.ref_tracers_get(ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return ids, X

    def set_tracers(self, ids, X):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        X = np.ascontiguousarray(X, dtype=np.float64)
        self.lib.ref_tracers_set(ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_long(len(ids)))

    def set(self, name, value):
        return self.lib.ref_set(name.encode(), float(value))

    def geometry(self):
        g2 = (self.sn1, self.sn2)
        return {"gcov": self._arr("gcov", g2 + (NPG, 4, 4)).copy(),
                "gcon": self._arr("gcon", g2 + (NPG, 4, 4)).copy(),
                "gdet": self._arr("gdet", g2 + (NPG,)).copy(),
                "conn": self._arr("conn", g2 + (4, 4, 4)).copy(),
                "coords": self._arr("coords", g2 + (4,)).copy(),
                "katm": self._arr("Katm", (self.sn1,)).copy()}

    def params(self):
        g = self.get
        return make_params(self.n1, self.n2, self.n3, g("a"), g("gam"), g("cour"),
                           [0.0, g("dx1"), g("dx2"), g("dx3")],
                           [0.0, g("startx1"), g("startx2"), g("startx3")],
                           defcon=g("defcon"), tf=g("tf"), lim=int(g("lim")))

    def step(self):
        self.lib.ref_step()

    # run-time COOL_EOS (COOL_EOS checker builds only; oracle/cool_hooks.inc)
    def cool_constants(self):
        c = np.zeros(len(EOS_CONSTANTS) + 1)
        self.lib.ref_cool_constants(_dp(c))
        return dict(zip(EOS_CONSTANTS + ("l_unit",), c.tolist()))

    def cool_tables(self):
        """Every node of every per-radius table, computed by the reference's own
        table fill, as EosTables."""
        d = (ctypes.c_int * 4)()
        self.lib.ref_cool_dims(d)
        nx, ny, nd, ntab = d[0], d[1], d[2], d[3]
        xa, ya = np.zeros(nx), np.zeros(ny)
        val = np.zeros((ntab, nx, ny, nd))
        hdfac = np.zeros(ntab)
        hd = ctypes.c_double()
        with _QuietStdout():
            for i in range(ntab):
                self.lib.ref_cool_table(i, _dp(xa), _dp(ya), _dp(val[i]), ctypes.byref(hd))
                hdfac[i] = hd.value
        consts = self.cool_constants()
        consts["hdfac"] = hdfac
        return EosTables(xa, ya, val, consts)

    def cool_batch(self, what, tab, rho0, u, lastT):
        """pressure/dpdu/dpdrho through the reference's own functions, one call per
        entry in order, each entry with its own guess; returns (out, lastT after)."""
        fn = {"pressure": self.lib.ref_cool_pressure, "dpdu": self.lib.ref_cool_dpdu,
              "dpdrho": self.lib.ref_cool_dpdrho}[what]
        fn.restype = ctypes.c_double
        fn.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        out = np.zeros(len(tab))
        lt = np.array(lastT, dtype=np.float64)
        with _QuietStdout():
            for k in range(len(tab)):
                t = ctypes.c_double(lt[k])
                out[k] = fn(int(tab[k]), float(rho0[k]), float(u[k]), ctypes.byref(t))
                lt[k] = t.value
        return out, lt

    def cool_lastT(self):
        a = np.zeros((self.sn3, self.sn1, self.sn2))
        self.lib.ref_cool_lastT_get(_dp(a))
        return a

    def set_cool_lastT(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.lib.ref_cool_lastT_set(_dp(a))

    def cool_prim_to_U(self, pr, h, i, j, lastT):
        """primtoU at zone (h, i, j) with the zone's guess; returns (U, lastT after)."""
        pr = np.array(pr, dtype=np.float64)
        U = np.zeros(NPR)
        t = ctypes.c_double(lastT)
        with _QuietStdout():
            self.lib.ref_cool_prim_to_U(_dp(pr), h, i, j, _dp(U), ctypes.byref(t))
        return U, t.value

    def utoprim_5d(self, U, h, i, j, prim, lastT):
        """Utoprim_5d at zone (h, i, j) entered as advance() enters it; returns
        (code, prim after, lastT after)."""
        U = np.array(U, dtype=np.float64)
        pr = np.array(prim, dtype=np.float64)
        t = ctypes.c_double(lastT)
        with _QuietStdout():
            r = self.lib.ref_utoprim_5d(_dp(U), h, i, j, _dp(pr), ctypes.byref(t))
        return r, pr, t.value
