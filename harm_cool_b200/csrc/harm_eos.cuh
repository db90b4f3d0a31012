// Run-time COOL_EOS on the device: the reference's per-radius (rho, T) tables,
// Akima interpolation on a window of 3 or 4 nodes per axis, the Newton solve
// for T and the pressure with its gamma-law fall-backs.
//
// Reference: pressure_rho0_u_CoolEOS (cooleos.c:314-444), the residual and its
// derivative (cooleos.c:198-300), mnewtc<1> (mnewt.h:105-205),
// Cache4d::getvalues in SPLINE mode (cache4d.c:863-1134) with calcbox
// (cache4d.c:408-439) and dvec_bracket (akima.c:314-336), interpolate_akima
// (akima.c:9-161), spline_akima_der (akima.c:259-298), dpdu_calc_CoolEOS and
// dpdrho_calc_CoolEOS (cooleos.c:667-741).  Built with -fmad=false and every
// expression in the reference's order, the FP64 results are the reference's bit
// for bit.  Two changes that cannot alter a result:
//  * an Akima window's cubic is formed only for the interval the evaluation
//    selects (the reference forms all of them and uses one);
//  * the Newton loop stops when a step is refused (the reference repeats the
//    identical pass until its 300 iterations are spent).
// The temperature guess that the reference keeps per zone behind the global
// LastT pointer (InitCache_CoolEOS, cooleos.c:770-807) travels in an EosCursor.
// A cursor remembers its last call: a call with bit-identical arguments that
// starts from the guess the last call left returns the last result, which is
// what the reference computes for it (a converged guess passes the residual test
// at once; a failed solve left the guess unchanged and fails the same way).
#pragma once
#include <math_constants.h>

#include <cstdint>

namespace harm {

// value planes of a table set (cooleos.c:32-37)
enum { EOS_E = 0, EOS_P = 1, EOS_QNU = 2, EOS_TAU = 3, EOS_YEE = 4, EOS_ND = 5 };

struct EosDev {
  int nx, ny, ntab;
  const double *xa, *ya;   // rho axis [nx], T axis [ny]
  const double *val;       // [EOS_ND][ntab][nx][ny]
  double rho_unit, u_unit, p_unit, kbol, mav, cl;
  double rho_min, rho_max, t_min, t_max, hh, gam;
  // FP32 copies for the mixed-precision interpolation: axes, and e and p
  // scaled by powers of two (se, sp) into the float range; f32 = 0 when the
  // tables do not fit
  int f32;
  const float *xa32, *ya32, *e32, *p32;  // [ntab][nx][ny] each
  double se, sp;
  // CoolVal_rho0_u_CoolEOS: each table's HdFac (cooleos.c:945-960, null when not
  // given) and L_UNIT
  const double *hdfac;
  double l_unit;
  // [ntab][nx][ny]: set to 1 where a table read (FP64, or FP32 of the mixed
  // path) met a NaN node (tables filled on demand leave the nodes not yet
  // generated NaN); null when not tracked
  unsigned char *miss;
};

// record the NaN nodes of a loaded row of n nodes, table tab, rho node x, T nodes from y0
template <int N, class T>
__device__ __forceinline__ void eos_note_missing(const EosDev &E, int tab, int x, int y0, const T *ys)
{
  if (!E.miss) return;
#pragma unroll
  for (int k = 0; k < N; k++)
    if (ys[k] != ys[k]) E.miss[((long)tab * E.nx + x) * E.ny + y0 + k] = 1;
}

// the cubic of interval i (akima.c:115-135): its left node, value, slope and
// the two higher coefficients
struct AkimaCubic {
  double xi, yi, si, c1, c2;
  __device__ __forceinline__ double at(double t) const
  {
    const double u = t - xi;
    return yi + si * u + c1 * u * u + c2 * u * u * u;
  }
};

// The T-direction cubics of one value plane's window, one per rho row, kept
// while the window (table, rho window, T window) and each row's interval stay
// the same: a cubic depends on nothing else, so a kept one is the one the
// reference forms again.
struct AkimaRowCache {
  int tab, x0, y0, sx, sy;  // tab < 0: empty
  int iv[4];                // each row's interval (-1: none kept)
  AkimaCubic c[4];
};

struct EosCursor {
  int tab;          // radial index of the table (cacheT[i])
  double T;         // the zone's temperature guess (*LastT)
  bool memo, m_f32;
  double m_rho, m_u, m_p, m_T;
  bool keep;             // keep cubics between evaluations
  AkimaRowCache ce, cp;  // cubics of the e and p windows last used
};

// a cursor on table tab with guess T, nothing remembered
__device__ __forceinline__ EosCursor eos_cursor(int tab, double T, bool keep = true)
{
  EosCursor c;
  c.tab = tab;
  c.T = T;
  c.memo = false;
  c.m_f32 = false;
  c.keep = keep;
  c.ce.tab = -1;
  c.cp.tab = -1;
  return c;
}

__device__ __forceinline__ bool same_bits(double a, double b)
{
  return __double_as_longlong(a) == __double_as_longlong(b);
}

// calcbox(SPLINE) of dvec_bracket: window [lo, lo + n - 1] of 3 or 4 nodes.  The
// bracket is the smallest k in [1, n-2] with v < x[k], else n-1 (1-based left
// index); a bisection over the increasing axis finds the same k.
__device__ __forceinline__ void eos_window(int n, const double *__restrict__ x, double v, int &lo, int &cnt)
{
  int a = 1, b = n - 1;  // answer in [a, b]; b = n - 1 when no node qualifies
  while (a < b) {
    int m = (a + b) >> 1;
    if (v < __ldg(x + m)) b = m;
    else a = m + 1;
  }
  const int left = a;  // 1-based left end of the bracket; the right end is left + 1
  int l0 = left - 2, r0 = left + 1;  // 0-based: one node below and one above the bracket
  if (l0 < 0) l0 = 0;
  if (r0 >= n) r0 = n - 1;
  lo = l0;
  cnt = r0 - l0 + 1;
}

// Akima node derivative from the four slopes around the node (akima.c:96-113)
__device__ __forceinline__ double akima_node(double t0, double t1, double t2, double t3)
{
  double d0 = t3 - t2;
  if (d0 < 0.0) d0 *= -1.0;
  double d1 = t1 - t0;
  if (d1 < 0.0) d1 *= -1.0;
  if ((d0 + d1) < 1e-9) return 0.5 * (t1 + t2);
  return (d0 * t1 + d1 * t2) / (d0 + d1);
}

// slopes of an Akima window of SI nodes with the two extrapolated intervals on
// each side (akima.c:34-94): mm[0..SI+2]
template <int SI>
__device__ __forceinline__ void akima_slopes(const double *x, const double *y, double *mm)
{
#pragma unroll
  for (int k = 0; k < SI - 1; k++) mm[k + 2] = (y[k + 1] - y[k]) / (x[k + 1] - x[k]);
  double xl1 = x[0] + x[1] - x[2];
  double xl0 = xl1 + x[0] - x[1];
  double yl1 = (x[0] - xl1) * (mm[3] - 2.0 * mm[2]) + y[0];
  mm[1] = (y[0] - yl1) / (x[0] - xl1);
  double yl0 = (xl1 - xl0) * (mm[2] - 2.0 * mm[1]) + yl1;
  mm[0] = (yl1 - yl0) / (xl1 - xl0);
  double xr2 = x[SI - 1] + x[SI - 2] - x[SI - 3];
  double xr3 = xr2 + x[SI - 1] - x[SI - 2];
  double yr2 = (2.0 * mm[SI] - mm[SI - 1]) * (xr2 - x[SI - 1]) + y[SI - 1];
  mm[SI + 1] = (yr2 - y[SI - 1]) / (xr2 - x[SI - 1]);
  double yr3 = (2.0 * mm[SI + 1] - mm[SI]) * (xr3 - xr2) + yr2;
  mm[SI + 2] = (yr3 - yr2) / (xr3 - xr2);
}

// the interval interpolate_akima's search selects for t (akima.c:140-152)
template <int SI>
__device__ __forceinline__ int akima_interval(const double *x, double t)
{
  int i = (t > x[1]) ? 1 : 0;
  if (SI == 4 && t > x[2]) i = 2;
  return i;
}

template <int SI>
__device__ __forceinline__ AkimaCubic akima_cubic(const double *x, const double *y, const double *mm, int i)
{
  double xi = x[0], xi1 = x[1], yi = y[0], yi1 = y[1];
  double a0 = mm[0], a1 = mm[1], a2 = mm[2], a3 = mm[3], a4 = mm[4];
  if (i >= 1) { xi = x[1]; xi1 = x[2]; yi = y[1]; yi1 = y[2]; a0 = mm[1]; a1 = mm[2]; a2 = mm[3]; a3 = mm[4]; a4 = mm[5]; }
  if (SI == 4 && i >= 2) { xi = x[2]; xi1 = x[3]; yi = y[2]; yi1 = y[3]; a0 = mm[2]; a1 = mm[3]; a2 = mm[4]; a3 = mm[5]; a4 = mm[6]; }
  const double si = akima_node(a0, a1, a2, a3), si1 = akima_node(a1, a2, a3, a4);
  const double d0 = xi1 - xi;
  const double d1 = yi1 - yi;
  const double t2 = d1 / d0;
  AkimaCubic c;
  c.xi = xi;
  c.yi = yi;
  c.si = si;
  c.c1 = (3.0 * t2 - 2.0 * si - si1) / d0;
  c.c2 = (si + si1 - 2.0 * t2) / (d0 * d0);
  return c;
}

// one Akima window: the value at t (akima.c:137-158), and with DER the central
// difference of spline_akima_der (h = t * 1e-6).  Points that fall in the same
// interval share its cubic, formed once.
template <int SI, bool DER>
__device__ __forceinline__ void akima_window(const double *x, const double *y, double t, double &v, double &dv)
{
  double mm[SI + 3];
  akima_slopes<SI>(x, y, mm);
  const int i = akima_interval<SI>(x, t);
  const AkimaCubic c = akima_cubic<SI>(x, y, mm, i);
  v = c.at(t);
  if (DER) {
    const double h = t * 1.0E-6;
    const double tm = t - h, tp = t + h;
    const int im = akima_interval<SI>(x, tm), ip = akima_interval<SI>(x, tp);
    const double vm = im == i ? c.at(tm) : akima_cubic<SI>(x, y, mm, im).at(tm);
    const double vp = ip == i ? c.at(tp) : akima_cubic<SI>(x, y, mm, ip).at(tp);
    dv = (vp - vm) / (2.0 * h);
  }
}

// getvalues at (rho, T) for one value plane: Akima along T on each rho row of
// the window, then along rho (cache4d.c:1086-1127).  With a cache, a row whose
// T-interval is the one kept reuses its cubic.
template <int SX, int SY, bool DER>
__device__ __noinline__ void eos_value_w(const EosDev &E, const double *__restrict__ plane, int tab, int x0, int y0,
                                         double rho, double T, double &val, double &der, AkimaRowCache *cache)
{
  double xw[SX], yw[SY], row[SX], rowd[SX];
#pragma unroll
  for (int k = 0; k < SX; k++) xw[k] = __ldg(E.xa + x0 + k);
#pragma unroll
  for (int k = 0; k < SY; k++) yw[k] = __ldg(E.ya + y0 + k);
  if (cache && !(cache->tab == tab && cache->x0 == x0 && cache->y0 == y0 && cache->sx == SX && cache->sy == SY)) {
    cache->tab = tab;
    cache->x0 = x0;
    cache->y0 = y0;
    cache->sx = SX;
    cache->sy = SY;
#pragma unroll
    for (int r = 0; r < 4; r++) cache->iv[r] = -1;
  }
  const int i = akima_interval<SY>(yw, T);
  // spline_akima_der's points (akima.c:259-298)
  const double h = T * 1.0E-6;
  const double tm = T - h, tp = T + h;
  const int im = DER ? akima_interval<SY>(yw, tm) : i, ip = DER ? akima_interval<SY>(yw, tp) : i;
#pragma unroll
  for (int r = 0; r < SX; r++) {
    const double *src = plane + (long)(x0 + r) * E.ny + y0;
    double ys[SY], mm[SY + 3];
    bool have = false;
    AkimaCubic c;
    if (cache && cache->iv[r] == i) {
      c = cache->c[r];
    } else {
#pragma unroll
      for (int k = 0; k < SY; k++) ys[k] = __ldg(src + k);
      eos_note_missing<SY>(E, tab, x0 + r, y0, ys);
      akima_slopes<SY>(yw, ys, mm);
      have = true;
      c = akima_cubic<SY>(yw, ys, mm, i);
      if (cache) {
        cache->c[r] = c;
        cache->iv[r] = i;
      }
    }
    row[r] = c.at(T);
    if (DER) {
      if ((im != i || ip != i) && !have) {
#pragma unroll
        for (int k = 0; k < SY; k++) ys[k] = __ldg(src + k);
        eos_note_missing<SY>(E, tab, x0 + r, y0, ys);
        akima_slopes<SY>(yw, ys, mm);
      }
      const double vm = im == i ? c.at(tm) : akima_cubic<SY>(yw, ys, mm, im).at(tm);
      const double vp = ip == i ? c.at(tp) : akima_cubic<SY>(yw, ys, mm, ip).at(tp);
      rowd[r] = (vp - vm) / (2.0 * h);
    }
  }
  double unused;
  akima_window<SX, false>(xw, row, rho, val, unused);
  if (DER) akima_window<SX, false>(xw, rowd, rho, der, unused);
}

// returns false outside the table (the reference's getvalues returns 0 there
// without writing its outputs, cache4d.c:899-911)
template <bool DER>
__device__ __forceinline__ bool eos_value(const EosDev &E, int tab, int d, double rho, int x0, int sx, double T,
                                          double &val, double &der, AkimaRowCache *cache = nullptr)
{
  if (!(T >= __ldg(E.ya)) || !(T <= __ldg(E.ya + E.ny - 1))) return false;
  int y0, sy;
  eos_window(E.ny, E.ya, T, y0, sy);
  const double *plane = E.val + ((long)d * E.ntab + tab) * E.nx * E.ny;
  if (sx == 4) {
    if (sy == 4) eos_value_w<4, 4, DER>(E, plane, tab, x0, y0, rho, T, val, der, cache);
    else eos_value_w<4, 3, DER>(E, plane, tab, x0, y0, rho, T, val, der, cache);
  } else {
    if (sy == 4) eos_value_w<3, 4, DER>(E, plane, tab, x0, y0, rho, T, val, der, cache);
    else eos_value_w<3, 3, DER>(E, plane, tab, x0, y0, rho, T, val, der, cache);
  }
  return true;
}

__device__ __forceinline__ bool eos_rho_window(const EosDev &E, double rho, int &x0, int &sx)
{
  if (!(rho >= __ldg(E.xa)) || !(rho <= __ldg(E.xa + E.nx - 1))) return false;
  eos_window(E.nx, E.xa, rho, x0, sx);
  return true;
}

// mnewtc<1>(300, x, 1e-6, minx, maxx) on (e - e(rho, T)) / e; returns berr
static __device__ __noinline__ double eos_newton_T(const EosDev &E, int tab, double rho, bool rho_in, int x0, int sx,
                                            double e, double &x, double minx, double maxx, AkimaRowCache *ce)
{
  double best = x, besterr = 1.0E100;
  for (int k = 1; k <= 300; k++) {
    double ecur = CUDART_NAN, dcur = CUDART_NAN;
    if (rho_in) {
      double v, dv;
      if (eos_value<true>(E, tab, EOS_E, rho, x0, sx, x, v, dv, ce)) { ecur = v; dcur = dv; }
    }
    const double F = (e - ecur) / e;
    const double D = -dcur / e;
    double bet = -F;
    double errf = 0.0;
    errf += fabs(bet);
    if (errf <= 1.0E-6) return errf;
    if (errf < besterr) { besterr = errf; best = x; }
    if (fabs(D) > 0.0) bet = bet / D;
    const double nv = x + bet;
    if (nv >= minx && nv <= maxx && nv != x) x = nv;
    else break;
  }
  x = best;
  return besterr;
}

// pressure_rho0_u_CoolEOS (cooleos.c:314-444) with the guess in c.T
static __device__ __noinline__ double eos_pressure(const EosDev &E, EosCursor &c, double rho0, double u)
{
  if (c.memo && !c.m_f32 && same_bits(rho0, c.m_rho) && same_bits(u, c.m_u) && same_bits(c.T, c.m_T))
    return c.m_p;
  const double rho = rho0 * E.rho_unit;
  const double e = u * E.u_unit;
  const double hh = E.hh;
  double p;
  if (c.T == 0.0) {
    const double corrfact = 1.0;
    c.T = (E.gam - 1.) * u / rho0 / E.kbol * E.mav * E.cl * E.cl * corrfact;
    if (c.T < E.t_min * (1.0 + hh)) c.T = E.t_min * (1.0 + hh);
  }
  if (rho < E.rho_min) p = (E.gam - 1.) * u;
  else if (rho > E.rho_max) p = (E.gam - 1.) * u;
  else if (e < 0.0) p = 0.0;
  else {
    const double minx = E.t_min * (1.0 + hh), maxx = E.t_max * (1.0 - hh);
    int x0 = 0, sx = 4;
    const bool rho_in = eos_rho_window(E, rho, x0, sx);
    double x = c.T;
    const double berr = eos_newton_T(E, c.tab, rho, rho_in, x0, sx, e, x, minx, maxx, c.keep ? &c.ce : nullptr);
    if (berr > 1.0E-6) p = (E.gam - 1.) * u;
    else {
      double v = CUDART_NAN, unused;
      if (rho_in) {
        double w;
        if (eos_value<false>(E, c.tab, EOS_P, rho, x0, sx, x, w, unused, c.keep ? &c.cp : nullptr)) v = w;
      }
      c.T = x;
      p = v / E.p_unit;
    }
  }
  c.memo = true;
  c.m_f32 = false;
  c.m_rho = rho0;
  c.m_u = u;
  c.m_p = p;
  c.m_T = c.T;
  return p;
}

// the cooling values of CoolVal_rho0_u_CoolEOS (decs.h:251-258)
enum { COOL_LAMBDA_SIM = 0, COOL_P = 1, COOL_Hd = 2, COOL_Qnu = 3, COOL_Tau = 4, COOL_T = 5, COOL_Yee = 6,
       NCOOLVAL = 7 };

// CoolVal_rho0_u_CoolEOS (cooleos.c:479-662): p, T, the disc scale height, the
// neutrino emissivity and cooling rate, tau and Yee at (rho0, u) of the zone at
// radius r, with the zone's guess in c.T.  Unlike the pressure it has no e < 0
// branch, and it tests the table range before setting a first guess.
static __device__ __noinline__ void eos_coolval(const EosDev &E, EosCursor &c, double rho0, double u, double r,
                                                double *cv)
{
  const double SMALL_ = 1.e-20;
  const double rho = rho0 * E.rho_unit;
  const double e = u * E.u_unit;
  const double hh = E.hh;
  const double HdFac = E.hdfac[c.tab];
  bool gamma_law = rho < E.rho_min || rho > E.rho_max;
  double x = 0.;
  int x0 = 0, sx = 4;
  bool rho_in = false;
  if (!gamma_law) {
    if (c.T == 0.0) {
      const double corrfact = 1.0;
      c.T = (E.gam - 1.) * u / rho0 / E.kbol * E.mav * E.cl * E.cl * corrfact;
      if (c.T < E.t_min * (1.0 + hh)) c.T = E.t_min * (1.0 + hh);
    }
    const double minx = E.t_min * (1.0 + hh), maxx = E.t_max * (1.0 - hh);
    rho_in = eos_rho_window(E, rho, x0, sx);
    x = c.T;
    const double berr = eos_newton_T(E, c.tab, rho, rho_in, x0, sx, e, x, minx, maxx, c.keep ? &c.ce : nullptr);
    gamma_law = berr > 1.0E-6;
  }
  c.memo = false;
  if (gamma_law) {
    cv[COOL_P] = (E.gam - 1.) * u;
    cv[COOL_LAMBDA_SIM] = SMALL_;
    cv[COOL_Qnu] = SMALL_;
    const double Hd = HdFac * E.cl * sqrt(cv[COOL_P] * E.p_unit / (rho * E.cl * E.cl + e));
    cv[COOL_Hd] = Hd / E.l_unit;
    cv[COOL_T] = (E.gam - 1.) * u / rho0 / E.kbol * E.mav * E.cl * E.cl;
    cv[COOL_Tau] = 0.0;
    cv[COOL_Yee] = 0.0;
    return;
  }
  double val[EOS_ND];
#pragma unroll
  for (int d = 0; d < EOS_ND; d++) {
    double v = CUDART_NAN, unused;
    if (rho_in) {
      double w;
      if (eos_value<false>(E, c.tab, d, rho, x0, sx, x, w, unused)) v = w;
    }
    val[d] = v;
  }
  c.T = x;
  const double Hd = HdFac * E.cl * sqrt(val[EOS_P] / (rho * E.cl * E.cl + val[EOS_E]));
  const double Hdisk = 0.5 * r * E.l_unit;
  const double lambda_cgs = val[EOS_QNU] / Hdisk;
  cv[COOL_LAMBDA_SIM] = lambda_cgs / (E.rho_unit * E.cl * E.cl * E.cl / E.l_unit);
  cv[COOL_Hd] = Hd / E.l_unit;
  cv[COOL_Qnu] = val[EOS_QNU] / (E.rho_unit * E.cl * E.cl * E.cl / E.l_unit);
  cv[COOL_P] = val[EOS_P] / E.p_unit;
  cv[COOL_T] = x;
  cv[COOL_Tau] = val[EOS_TAU] > 0 ? val[EOS_TAU] : 0.0;
  cv[COOL_Yee] = val[EOS_YEE];
}

// dpdu_calc_CoolEOS (cooleos.c:667-704)
__device__ __forceinline__ double eos_dpdu(const EosDev &E, EosCursor &c, double rho0, double u)
{
  const double h = u * E.hh / E.u_unit;
  const double uP = u + h;
  double uM = u - h;
  if (uM > 0) {
    const double pP = eos_pressure(E, c, rho0, uP);
    const double pM = eos_pressure(E, c, rho0, uM);
    return (pP - pM) / (2.0 * h);
  }
  uM = u;
  const double pP = eos_pressure(E, c, rho0, uP);
  const double pM = eos_pressure(E, c, rho0, uM);
  return (pP - pM) / (h);
}

// dpdrho_calc_CoolEOS (cooleos.c:706-741)
__device__ __forceinline__ double eos_dpdrho(const EosDev &E, EosCursor &c, double rho0, double u)
{
  const double h = rho0 * E.hh / E.rho_unit;
  const double rhoP = rho0 + h;
  double rhoM = rho0 - h;
  if (rhoM > 0) {
    const double pP = eos_pressure(E, c, rhoP, u);
    const double pM = eos_pressure(E, c, rhoM, u);
    return (pP - pM) / (2.0 * h);
  }
  rhoM = rho0;
  const double pP = eos_pressure(E, c, rhoP, u);
  const double pM = eos_pressure(E, c, rhoM, u);
  return (pP - pM) / (h);
}

// ---------------------------------------------------------------------------
// Mixed precision: the same solve with the tables, the Akima windows and the
// Newton iteration in float.  Differences from the FP64 path, all within its
// 1e-6 solve tolerance: e and p are scaled by powers of two into the float
// range; an Akima node derivative is formed as a weighted mean (the FP64
// form's products overflow float); the T-derivative of e is the derivative of
// the interpolating cubic instead of spline_akima_der's central difference,
// which float cannot resolve at h = T * 1e-6.  The branches (table range,
// e < 0) and the gamma-law fall-backs are the FP64 path's, and a solve that
// float cannot bring to the tolerance is redone in FP64, so that a zone falls
// back to the gamma law only where the FP64 path does (but for solves that
// FP64 fails and float passes).

__device__ __forceinline__ void eos_window_f(int n, const float *__restrict__ x, float v, int &lo, int &cnt)
{
  int a = 1, b = n - 1;
  while (a < b) {
    int m = (a + b) >> 1;
    if (v < __ldg(x + m)) b = m;
    else a = m + 1;
  }
  int l0 = a - 2, r0 = a + 1;
  if (l0 < 0) l0 = 0;
  if (r0 >= n) r0 = n - 1;
  lo = l0;
  cnt = r0 - l0 + 1;
}

__device__ __forceinline__ float akima_node_f(float t0, float t1, float t2, float t3)
{
  const float d0 = fabsf(t3 - t2), d1 = fabsf(t1 - t0);
  const float s = d0 + d1;
  if (!(s >= 1e-30f)) return 0.5f * (t1 + t2);
  const float w = __fdividef(d0, s);
  return __fmaf_rn(w, t1 - t2, t2);
}

template <int SI>
__device__ __forceinline__ void akima_slopes_f(const float *x, const float *y, float *mm)
{
#pragma unroll
  for (int k = 0; k < SI - 1; k++) mm[k + 2] = __fdividef(y[k + 1] - y[k], x[k + 1] - x[k]);
  const float xl1 = x[0] + x[1] - x[2];
  const float xl0 = xl1 + x[0] - x[1];
  const float yl1 = __fmaf_rn(x[0] - xl1, mm[3] - 2.f * mm[2], y[0]);
  mm[1] = __fdividef(y[0] - yl1, x[0] - xl1);
  const float yl0 = __fmaf_rn(xl1 - xl0, mm[2] - 2.f * mm[1], yl1);
  mm[0] = __fdividef(yl1 - yl0, xl1 - xl0);
  const float xr2 = x[SI - 1] + x[SI - 2] - x[SI - 3];
  const float xr3 = xr2 + x[SI - 1] - x[SI - 2];
  const float yr2 = __fmaf_rn(2.f * mm[SI] - mm[SI - 1], xr2 - x[SI - 1], y[SI - 1]);
  mm[SI + 1] = __fdividef(yr2 - y[SI - 1], xr2 - x[SI - 1]);
  const float yr3 = __fmaf_rn(2.f * mm[SI + 1] - mm[SI], xr3 - xr2, yr2);
  mm[SI + 2] = __fdividef(yr3 - yr2, xr3 - xr2);
}

// value (and with DER the derivative) of the cubic of the interval t falls in
template <int SI, bool DER>
__device__ __forceinline__ void akima_window_f(const float *x, const float *y, float t, float &v, float &dv)
{
  float mm[SI + 3];
  akima_slopes_f<SI>(x, y, mm);
  int i = (t > x[1]) ? 1 : 0;
  if (SI == 4 && t > x[2]) i = 2;
  float xi = x[0], xi1 = x[1], yi = y[0], yi1 = y[1];
  float a0 = mm[0], a1 = mm[1], a2 = mm[2], a3 = mm[3], a4 = mm[4];
  if (i >= 1) { xi = x[1]; xi1 = x[2]; yi = y[1]; yi1 = y[2]; a0 = mm[1]; a1 = mm[2]; a2 = mm[3]; a3 = mm[4]; a4 = mm[5]; }
  if (SI == 4 && i >= 2) { xi = x[2]; xi1 = x[3]; yi = y[2]; yi1 = y[3]; a0 = mm[2]; a1 = mm[3]; a2 = mm[4]; a3 = mm[5]; a4 = mm[6]; }
  const float si = akima_node_f(a0, a1, a2, a3), si1 = akima_node_f(a1, a2, a3, a4);
  const float d0 = xi1 - xi;
  const float rd = __fdividef(1.f, d0);
  const float t2 = (yi1 - yi) * rd;
  const float c1 = (3.f * t2 - 2.f * si - si1) * rd;
  const float c2 = (si + si1 - 2.f * t2) * rd * rd;
  const float u = t - xi;
  v = __fmaf_rn(__fmaf_rn(__fmaf_rn(c2, u, c1), u, si), u, yi);
  if (DER) dv = __fmaf_rn(__fmaf_rn(3.f * c2, u, 2.f * c1), u, si);
}

template <int SX, int SY, bool DER>
__device__ __noinline__ void eos_value_wf(const EosDev &E, const float *__restrict__ plane, int tab, int x0, int y0,
                                          float rho, float T, float &val, float &der)
{
  float xw[SX], yw[SY], row[SX], rowd[SX];
#pragma unroll
  for (int k = 0; k < SX; k++) xw[k] = __ldg(E.xa32 + x0 + k);
#pragma unroll
  for (int k = 0; k < SY; k++) yw[k] = __ldg(E.ya32 + y0 + k);
#pragma unroll
  for (int r = 0; r < SX; r++) {
    const float *src = plane + (long)(x0 + r) * E.ny + y0;
    float ys[SY];
#pragma unroll
    for (int k = 0; k < SY; k++) ys[k] = __ldg(src + k);
    eos_note_missing<SY>(E, tab, x0 + r, y0, ys);
    float d = 0.f;
    akima_window_f<SY, DER>(yw, ys, T, row[r], d);
    rowd[r] = d;
  }
  float unused;
  akima_window_f<SX, false>(xw, row, rho, val, unused);
  if (DER) akima_window_f<SX, false>(xw, rowd, rho, der, unused);
}

template <bool DER>
__device__ __forceinline__ bool eos_value_f(const EosDev &E, int tab, const float *planes, float rho, int x0, int sx,
                                            float T, float &val, float &der)
{
  if (!(T >= __ldg(E.ya32)) || !(T <= __ldg(E.ya32 + E.ny - 1))) return false;
  int y0, sy;
  eos_window_f(E.ny, E.ya32, T, y0, sy);
  const float *plane = planes + (long)tab * E.nx * E.ny;
  if (sx == 4) {
    if (sy == 4) eos_value_wf<4, 4, DER>(E, plane, tab, x0, y0, rho, T, val, der);
    else eos_value_wf<4, 3, DER>(E, plane, tab, x0, y0, rho, T, val, der);
  } else {
    if (sy == 4) eos_value_wf<3, 4, DER>(E, plane, tab, x0, y0, rho, T, val, der);
    else eos_value_wf<3, 3, DER>(E, plane, tab, x0, y0, rho, T, val, der);
  }
  return true;
}

// mnewtc<1>'s iteration in float; returns berr
static __device__ __noinline__ float eos_newton_T_f(const EosDev &E, int tab, float rho, bool rho_in, int x0, int sx,
                                                    float e, float &x, float minx, float maxx)
{
  float best = x, besterr = 1.0e30f;
  for (int k = 1; k <= 300; k++) {
    float ecur = CUDART_NAN_F, dcur = CUDART_NAN_F;
    if (rho_in) {
      float v, dv;
      if (eos_value_f<true>(E, tab, E.e32, rho, x0, sx, x, v, dv)) { ecur = v; dcur = dv; }
    }
    const float re = __fdividef(1.f, e);
    const float F = (e - ecur) * re;
    const float D = -dcur * re;
    float bet = -F;
    const float errf = fabsf(bet);
    if (errf <= 1.0e-6f) return errf;
    if (errf < besterr) { besterr = errf; best = x; }
    if (fabsf(D) > 0.f) bet = bet / D;
    const float nv = x + bet;
    if (nv >= minx && nv <= maxx && nv != x) x = nv;
    else break;
  }
  x = best;
  return besterr;
}

// pressure_rho0_u_CoolEOS with the interpolation and the solve in float
static __device__ __noinline__ double eos_pressure_f(const EosDev &E, EosCursor &c, double rho0, double u)
{
  if (c.memo && c.m_f32 && same_bits(rho0, c.m_rho) && same_bits(u, c.m_u) && same_bits(c.T, c.m_T)) return c.m_p;
  const double rho = rho0 * E.rho_unit;
  const double e = u * E.u_unit;
  const double hh = E.hh;
  double p;
  if (c.T == 0.0) {
    c.T = (E.gam - 1.) * u / rho0 / E.kbol * E.mav * E.cl * E.cl;
    if (c.T < E.t_min * (1.0 + hh)) c.T = E.t_min * (1.0 + hh);
  }
  if (rho < E.rho_min) p = (E.gam - 1.) * u;
  else if (rho > E.rho_max) p = (E.gam - 1.) * u;
  else if (e < 0.0) p = 0.0;
  else {
    const float minx = (float)(E.t_min * (1.0 + hh)), maxx = (float)(E.t_max * (1.0 - hh));
    const float rf = (float)rho;
    int x0 = 0, sx = 4;
    bool rho_in = rf >= __ldg(E.xa32) && rf <= __ldg(E.xa32 + E.nx - 1);
    if (rho_in) eos_window_f(E.nx, E.xa32, rf, x0, sx);
    float x = (float)c.T;
    const float berr = eos_newton_T_f(E, c.tab, rf, rho_in, x0, sx, (float)(e * E.se), x, minx, maxx);
    if (!(berr <= 1.0e-6f)) {
      // float could not reach the tolerance: the FP64 solve decides, so the
      // table-or-gamma-law branch is the FP64 path's
      p = eos_pressure(E, c, rho0, u);
    } else {
      float v = CUDART_NAN_F, unused;
      if (rho_in) {
        float w;
        if (eos_value_f<false>(E, c.tab, E.p32, rf, x0, sx, x, w, unused)) v = w;
      }
      c.T = (double)x;
      p = (double)v / E.sp / E.p_unit;
    }
  }
  c.memo = true;
  c.m_f32 = true;
  c.m_rho = rho0;
  c.m_u = u;
  c.m_p = p;
  c.m_T = c.T;
  return p;
}

// dpdu_calc_CoolEOS and dpdrho_calc_CoolEOS over the float solve
__device__ __forceinline__ double eos_dpdu_f(const EosDev &E, EosCursor &c, double rho0, double u)
{
  const double h = u * E.hh / E.u_unit;
  const double uP = u + h;
  double uM = u - h;
  if (uM > 0) return (eos_pressure_f(E, c, rho0, uP) - eos_pressure_f(E, c, rho0, uM)) / (2.0 * h);
  uM = u;
  const double pP = eos_pressure_f(E, c, rho0, uP);
  return (pP - eos_pressure_f(E, c, rho0, uM)) / (h);
}

__device__ __forceinline__ double eos_dpdrho_f(const EosDev &E, EosCursor &c, double rho0, double u)
{
  const double h = rho0 * E.hh / E.rho_unit;
  const double rhoP = rho0 + h;
  double rhoM = rho0 - h;
  if (rhoM > 0) return (eos_pressure_f(E, c, rhoP, u) - eos_pressure_f(E, c, rhoM, u)) / (2.0 * h);
  rhoM = rho0;
  const double pP = eos_pressure_f(E, c, rhoP, u);
  return (pP - eos_pressure_f(E, c, rhoM, u)) / (h);
}

}  // namespace harm
