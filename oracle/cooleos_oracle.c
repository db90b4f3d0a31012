/*
 * CPU restatement of the reference's run-time COOL_EOS (TEST INFRASTRUCTURE ONLY:
 * the checker for the device EOS, never the product).
 *
 * What it restates, step for step:
 *  - Cache4d::getvalues in SPLINE mode with a fixed z index (cache4d.c:863-1134):
 *    the interpolation window of calcbox (cache4d.c:408-439) around the bracket of
 *    dvec_bracket (akima.c:314-336) on each axis, Akima along T for every rho row
 *    of the window, then Akima along rho;
 *  - interpolate_akima (akima.c:9-161): slopes, two extrapolated points on each
 *    side, Akima node derivatives, cubic coefficients, evaluation; and
 *    spline_akima_der's central difference with h = T * 1e-6 (akima.c:259-298);
 *  - the one-dimensional Newton solve mnewtc<1> (mnewt.h:105-205) with the
 *    residual (e - e(rho, T)) / e and its derivative (cooleos.c:230-300);
 *  - pressure_rho0_u_CoolEOS (cooleos.c:314-444), dpdu_calc_CoolEOS and
 *    dpdrho_calc_CoolEOS (cooleos.c:667-741).
 *
 * One behaviour is defined here where the reference has none: when the first
 * temperature of a solve lies outside the table (a guess carried in from outside
 * [TMin, TMax]), getvalues returns without writing its outputs (cache4d.c:899-911)
 * and the reference goes on with uninitialised stack values.  Here the residual is
 * NaN, so the solve makes no step and ends in the gamma-law fall-back
 * (cooleos.c:408-427) with the guess unchanged.
 */
#include <math.h>
#include <string.h>

#include "harm_oracle.h"

/* dvec_bracket (akima.c:314-336): 1-based bracket of v in x[0..n-1] */
static void bracket(int n, const double *x, double v, int *left, int *right)
{
  for (int i = 2; i <= n - 1; i++)
    if (v < x[i - 1]) { *left = i - 1; *right = i; return; }
  *left = n - 1;
  *right = n;
}

/* calcbox in SPLINE mode (cache4d.c:408-439): 0-based window [lo, hi] */
static void window(int n, const double *x, double v, int *lo, int *hi)
{
  int l, r;
  bracket(n, x, v, &l, &r);
  l -= 2;  /* one node below the 0-based bracket */
  /* r: one node above the 0-based bracket */
  if (l < 0) l = 0;
  if (r >= n) r = n - 1;
  *lo = l;
  *hi = r;
}

/* interpolate_akima (akima.c:9-161) on si <= 4 points (x[k], y[k*ys]), evaluated at
   nout points t[] */
static void akima(int si, const double *x, const double *y, int ys, int nout, const double *t, double *out)
{
  /* mm[0], mm[1]: slopes of the two extrapolated intervals on the left; mm[k+2],
     k = 0..si-2: slopes of the data; mm[si+1], mm[si+2]: extrapolated on the right */
  double mm[7], s[4], c0[3], c1[3], c2[3];
  for (int k = 0; k < si - 1; k++) mm[k + 2] = (y[(k + 1) * ys] - y[k * ys]) / (x[k + 1] - x[k]);
  double xl1 = x[0] + x[1] - x[2];
  double xl0 = xl1 + x[0] - x[1];
  double yl1 = (x[0] - xl1) * (mm[3] - 2.0 * mm[2]) + y[0];
  mm[1] = (y[0] - yl1) / (x[0] - xl1);
  double yl0 = (xl1 - xl0) * (mm[2] - 2.0 * mm[1]) + yl1;
  mm[0] = (yl1 - yl0) / (xl1 - xl0);
  double xa = x[si - 2], xb = x[si - 1], yb = y[(si - 1) * ys];
  double xr2 = xb + xa - x[si - 3];
  double xr3 = xr2 + xb - xa;
  double yr2 = (2.0 * mm[si] - mm[si - 1]) * (xr2 - xb) + yb;
  mm[si + 1] = (yr2 - yb) / (xr2 - xb);
  double yr3 = (2.0 * mm[si + 1] - mm[si]) * (xr3 - xr2) + yr2;
  mm[si + 2] = (yr3 - yr2) / (xr3 - xr2);
  /* node derivatives from the four slopes around each node */
  for (int k = 0; k < si; k++) {
    double t0 = mm[k], t1 = mm[k + 1], t2 = mm[k + 2], t3 = mm[k + 3];
    double d0 = t3 - t2;
    if (d0 < 0.0) d0 *= -1.0;
    double d1 = t1 - t0;
    if (d1 < 0.0) d1 *= -1.0;
    if ((d0 + d1) < 1e-9) s[k] = 0.5 * (t1 + t2);
    else s[k] = (d0 * t1 + d1 * t2) / (d0 + d1);
  }
  /* the cubic of each interval an evaluation can select */
  for (int k = 0; k < si - 1; k++) {
    double d0 = x[k + 1] - x[k];
    double d1 = y[(k + 1) * ys] - y[k * ys];
    double t2 = d1 / d0;
    c0[k] = y[k * ys];
    c1[k] = (3.0 * t2 - 2.0 * s[k] - s[k + 1]) / d0;
    c2[k] = (s[k] + s[k + 1] - 2.0 * t2) / (d0 * d0);
  }
  for (int o = 0; o < nout; o++) {
    int i = -1, pos = 0;
    while (t[o] > x[pos] && i < si - 2) { pos++; i++; }
    if (i < 0) i = 0;
    double u = t[o] - x[i];
    out[o] = c0[i] + s[i] * u + c1[i] * u * u + c2[i] * u * u * u;
  }
}

/* Cache4d::getvalues(rho, T, 0, SPLINE, val, der, 0, mask) for one value index d
   (cache4d.c:863-1134); returns 0 outside the table */
static int table_value(const OraEos *E, int tab, int d, double rho, double T, double *val, double *der)
{
  const int nx = E->nx, ny = E->ny, nd = E->nd;
  if (rho < E->xa[0] || rho > E->xa[nx - 1] || T < E->ya[0] || T > E->ya[ny - 1]) return 0;
  int x0, x1, y0, y1;
  window(nx, E->xa, rho, &x0, &x1);
  window(ny, E->ya, T, &y0, &y1);
  double row[4], rowd[4];
  for (int r = 0; r <= x1 - x0; r++) {
    const double *v = E->val + (((size_t)tab * nx + x0 + r) * ny + y0) * nd + d;
    if (der) {
      /* spline_akima_der (akima.c:259-298) */
      const double h = T * 1.0E-6;
      double tt[3] = {T - h, T, T + h}, o[3];
      akima(y1 - y0 + 1, E->ya + y0, v, nd, 3, tt, o);
      row[r] = o[1];
      rowd[r] = (o[2] - o[0]) / (2.0 * h);
    } else {
      akima(y1 - y0 + 1, E->ya + y0, v, nd, 1, &T, &row[r]);
    }
  }
  akima(x1 - x0 + 1, E->xa + x0, row, 1, 1, &rho, val);
  if (der) akima(x1 - x0 + 1, E->xa + x0, rowd, 1, 1, &rho, der);
  return 1;
}

/* residual (e - e(rho, T)) / e and its derivative (cooleos.c:230-300) */
static void residual(const OraEos *E, int tab, double rho, double e, double T, double *F, double *D)
{
  double ecur, dcur;
  if (!table_value(E, tab, ORA_EOS_E, rho, T, &ecur, &dcur)) { ecur = NAN; dcur = NAN; }
  *F = (e - ecur) / e;
  *D = -dcur / e;
}

/* mnewtc<1>(300, x, 1e-6, minx, maxx, ..., nlos = 1) (mnewt.h:105-205) */
static double newton_T(const OraEos *E, int tab, double rho, double e, double *x, double minx, double maxx)
{
  double best = *x, besterr = 1.0E100;
  for (int k = 1; k <= 300; k++) {
    double F, D;
    residual(E, tab, rho, e, *x, &F, &D);
    double bet = -F;
    double errf = 0.0;
    errf += fabs(bet);
    if (errf <= 1.0E-6) return errf;
    if (errf < besterr) { besterr = errf; best = *x; }
    /* ludcmp<1> refuses a matrix whose largest |entry| is not above 0 (NaN
       included); lubksb<1> then divides by the pivot */
    if (fabs(D) > 0.0) bet = bet / D;
    double nv = *x + bet;
    if (nv >= minx && nv <= maxx && nv != *x) *x = nv;
    else break;  /* x unchanged: every later pass repeats this one */
  }
  *x = best;
  return besterr;
}

double ora_eos_pressure(const OraEos *E, int tab, double rho0, double u, double *lastT)
{
  const double rho = rho0 * E->rho_unit;
  const double e = u * E->u_unit;
  const double hh = E->hh;
  if (*lastT == 0.0) {
    const double corrfact = 1.0;
    *lastT = (E->gam - 1.) * u / rho0 / E->kbol * E->mav * E->cl * E->cl * corrfact;
    if (*lastT < E->t_min * (1.0 + hh)) *lastT = E->t_min * (1.0 + hh);
  }
  if (rho < E->rho_min) return (E->gam - 1.) * u;
  if (rho > E->rho_max) return (E->gam - 1.) * u;
  if (e < 0.0) return 0.0;
  const double minx = E->t_min * (1.0 + hh), maxx = E->t_max * (1.0 - hh);
  double x = *lastT;
  double berr = newton_T(E, tab, rho, e, &x, minx, maxx);
  if (berr > 1.0E-6) return (E->gam - 1.) * u;
  double p;
  if (!table_value(E, tab, ORA_EOS_P, rho, x, &p, NULL)) p = NAN;
  *lastT = x;
  return p / E->p_unit;
}

double ora_eos_dpdu(const OraEos *E, int tab, double rho0, double u, double *lastT)
{
  double h = u * E->hh / E->u_unit;
  double uP = u + h, uM = u - h;
  if (uM > 0) {
    double pP = ora_eos_pressure(E, tab, rho0, uP, lastT);
    double pM = ora_eos_pressure(E, tab, rho0, uM, lastT);
    return (pP - pM) / (2.0 * h);
  }
  uM = u;
  double pP = ora_eos_pressure(E, tab, rho0, uP, lastT);
  double pM = ora_eos_pressure(E, tab, rho0, uM, lastT);
  return (pP - pM) / (h);
}

double ora_eos_dpdrho(const OraEos *E, int tab, double rho0, double u, double *lastT)
{
  double h = rho0 * E->hh / E->rho_unit;
  double rhoP = rho0 + h, rhoM = rho0 - h;
  if (rhoM > 0) {
    double pP = ora_eos_pressure(E, tab, rhoP, u, lastT);
    double pM = ora_eos_pressure(E, tab, rhoM, u, lastT);
    return (pP - pM) / (2.0 * h);
  }
  rhoM = rho0;
  double pP = ora_eos_pressure(E, tab, rhoP, u, lastT);
  double pM = ora_eos_pressure(E, tab, rhoM, u, lastT);
  return (pP - pM) / (h);
}

/* batch forms for the ctypes caller: one call per entry, in order, each with its
   own guess in lastT[n] (in and out) */
void ora_eos_batch(const OraEos *E, int what, long n, const int *tab, const double *rho0, const double *u,
                   double *lastT, double *out)
{
  for (long k = 0; k < n; k++) {
    if (what == 0) out[k] = ora_eos_pressure(E, tab[k], rho0[k], u[k], &lastT[k]);
    else if (what == 1) out[k] = ora_eos_dpdu(E, tab[k], rho0[k], u[k], &lastT[k]);
    else out[k] = ora_eos_dpdrho(E, tab[k], rho0[k], u[k], &lastT[k]);
  }
}

/* the table value d at (rho, T) by the reference's interpolation (0 outside) */
int ora_eos_value(const OraEos *E, int tab, int d, double rho, double T, double *val, double *der)
{
  return table_value(E, tab, d, rho, T, val, der);
}

/* ---- the tables themselves: SetupCache_CoolEOS (cooleos.c:825-992) with the
   stand-in generator of eos_standin.c in place of abundance_ ---- */

void abundance_(double *rho, double *T, double *HdFac, double *e, double *p, double *Qnu, double *tau,
                double *xnee, double *xnep);

/* unit and range constants (cooleos.c:83-135, 840-940, 849-855) */
void ora_eos_constants(double gam, double *o)
{
  const double GNEWT = 6.6742867e-8, MSUN = 1.9892e33, KBOL = 1.3e-16, CL = 2.99792458e10;
  const double MP = 1.67262163783e-24, ME = 9.10956e-28, MN = 1.67492729e-24, MHE = 6.6465e-24;
  const double MAV = (MP + MN + 2. * ME + MHE) / 5.;
  const double M_BLH = 3. * MSUN;
  const double L_UNIT = GNEWT * M_BLH / (CL * CL);
  const double RHO_SCALE = 1.5e-5, USCALE = 1.0;
  const double M_UNIT = RHO_SCALE * MSUN;
  const double RHO_UNIT = M_UNIT / (L_UNIT * L_UNIT * L_UNIT);
  const double U_UNIT = RHO_UNIT * CL * CL * USCALE;
  o[0] = RHO_UNIT; o[1] = U_UNIT; o[2] = U_UNIT; o[3] = KBOL; o[4] = MAV; o[5] = CL;
  o[6] = 1.e2; o[7] = 1.e15; o[8] = 1.e4; o[9] = 1.e18; o[10] = 1.0E-6; o[11] = gam;
}

/* Cache4d::setindices, LOGARITHMIC axis (cache4d.c:336-343) */
void ora_eos_axis(int n, double min, double max, double *v)
{
  double delta = (log10(max) - log10(min)) / (n - 1);
  for (int r = 0; r < n; r++) v[r] = pow(10.0, log10(min) + delta * r);
}

/* HdFac of the table of a zone at radius r (cooleos.c:945-960) */
double ora_eos_hdfac(double r)
{
  const double GNEWT = 6.6742867e-8, MSUN = 1.9892e33, CL = 2.99792458e10;
  const double M_BLH = 3. * MSUN, bhs = 0.6;
  double cs = 1.0;
  double omega = CL * CL * CL / GNEWT / M_BLH / (bhs + pow(r, 1.5));
  return cs / omega;
}

/* every node of one table through calc_cache_val (cooleos.c:171-194):
   val[nx][ny][5] */
void ora_eos_fill(int nx, int ny, const double *xa, const double *ya, double hdfac, double *val)
{
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++) {
      double ro = xa[ix], te = ya[iy], hd = hdfac;
      double e, p, Qnu, tau, xnee, xnep;
      abundance_(&ro, &te, &hd, &e, &p, &Qnu, &tau, &xnee, &xnep);
      double *v = val + ((size_t)ix * ny + iy) * 5;
      v[0] = e; v[1] = p; v[2] = Qnu; v[3] = tau; v[4] = (xnee - xnep) / (ro / 1.66e15);
    }
}

/* the radius of the zone centre of radial index i (coord(), bl_coord() of
   coord.c for the modified Kerr-Schild grid), as SetupCache_CoolEOS takes it */
double ora_zone_r(double startx1, double dx1, double R0, int i)
{
  return exp(startx1 + ((i - 2) + 0.5) * dx1) + R0;
}
