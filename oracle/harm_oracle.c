/*
 * CPU oracle for the HARM-COOL step_ch() path (see harm_oracle.h).
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 *
 * Restated from the reference's gamma-law single-rank code path; every
 * function names the reference lines it follows.  Expression order matches
 * the reference so results agree bit for bit when built with
 * -ffp-contract=off.  Where the reference calls fail() and exits
 * (diag.c:381-397), the oracle records the first such event in its diag
 * block and carries on with the value the reference assigns just before the
 * call; parity is only defined on runs that record none.
 */
#include "harm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NPR 8
#define NDIM 4
#define NPG 5
enum { RHO, UU, U1, U2, U3, B1, B2, B3 };
enum { FACE1, FACE2, CORN, CENT, FACE3 };
enum { MC, VANL, MINM };

/* the <math.h> values the reference uses (not declared under -std=c99) */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_PI_2
#define M_PI_2 1.57079632679489661923
#endif

/* decs.h:127-158 */
#define RHOMIN (1.e-6)
#define UUMIN (1.e-8)
#define RHOMINLIMIT (1.e-20)
#define UUMINLIMIT (1.e-20)
#define POWRHO (2.0)
#define BSQORHOMAX (50.)
#define BSQOUMAX (2500.)
#define UORHOMAX (50.)
#define SMALL (1.e-20)
#define GAMMAMAX (50.)
#define SAFE (1.3)
#define POLEFIX_ROWS 2 /* decs.h:91-95, 3D only */

/* u2p_defs.h:79-99 */
#define MAX_NEWT_ITER 30
#define NEWT_TOL 1.0e-10
#define MIN_NEWT_TOL 1.0e-10
#define EXTRA_NEWT_ITER 2
#define NEWT_TOL2 1.0e-15
#define W_TOO_BIG 1.e20
#define UTSQ_TOO_BIG 1.e20
#define FAIL_VAL 1.e30

/* failure codes, decs.h:232-238 */
#define FAIL_VCHAR_DISCR 2
#define FAIL_COEFF_NEG 3
#define FAIL_COEFF_SUP 4
#define FAIL_GAMMA 5

typedef struct {
  double gcov[NDIM][NDIM];
  double gcon[NDIM][NDIM];
  double g;
} geom_t;

typedef struct {
  double ucon[NDIM], ucov[NDIM], bcon[NDIM], bcov[NDIM];
} state_t;

struct ora_state {
  ora_params prm;
  int sn1, sn2, sn3;
  int istart, istop, jstart, jstop, hstart, hstop;
  double *p, *ph, *dq, *F1, *F2, *F3, *e1, *e2, *e3;
  signed char *pflag;
  double *gcov, *gcon, *gdet, *conn, *coords, *katm;
  double t, dt;
  ora_diag d;
  /* current zone, for the failure record (metric.c:269-272) */
  int ch, ci, cj;
  /* tracer particles (tracers.c:19-35): labels, code coordinates X1..X3,
     status (0 active, 1 fell in, 2 left inside the theta window, 3 left in
     the jet, -1 dropped by the search); R0 and hslope for bl_coord() */
  long ntr;
  int *tr_ids;
  double *tr_X;
  signed char *tr_st;
  double R0, hslope;
};

/* ------------------------------------------------------------------ */
/* indexing                                                             */

static size_t zidx(const ora_state *s, int h, int i, int j)
{
  return ((size_t)h * s->sn1 + i) * s->sn2 + j;
}
#define PV(s, arr, h, i, j) ((arr) + zidx(s, h, i, j) * NPR)

static void fail(ora_state *s, int code)
{
  if (s && s->d.fail_code == 0) {
    s->d.fail_code = code; s->d.fail_h = s->ch; s->d.fail_i = s->ci; s->d.fail_j = s->cj;
  }
}

/* metric.c:257-273 */
static void get_geometry(ora_state *s, int h, int i, int j, int loc, geom_t *g)
{
  size_t b = ((size_t)i * s->sn2 + j) * NPG + loc;
  memcpy(g->gcov, s->gcov + b * 16, sizeof(g->gcov));
  memcpy(g->gcon, s->gcon + b * 16, sizeof(g->gcon));
  g->g = s->gdet[b];
  s->ch = h; s->ci = i; s->cj = j;
}

static void geom_from(const double *gcov, const double *gcon, double gdet, geom_t *g)
{
  memcpy(g->gcov, gcov, sizeof(g->gcov));
  memcpy(g->gcon, gcon, sizeof(g->gcon));
  g->g = gdet;
}

/* ------------------------------------------------------------------ */
/* physics: phys.c, metric.c                                            */

/* metric.c:210-231 */
static void lower(const double *ucon, const geom_t *g, double *ucov)
{
  for (int m = 0; m < 4; m++)
    ucov[m] = g->gcov[m][0] * ucon[0] + g->gcov[m][1] * ucon[1] + g->gcov[m][2] * ucon[2]
              + g->gcov[m][3] * ucon[3];
}

/* metric.c:234-255 */
static void raise_(const double *ucov, const geom_t *g, double *ucon)
{
  for (int m = 0; m < 4; m++)
    ucon[m] = g->gcon[m][0] * ucov[0] + g->gcon[m][1] * ucov[1] + g->gcon[m][2] * ucov[2]
              + g->gcon[m][3] * ucov[3];
}

static double dot4(const double *a, const double *b)
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* phys.c:300-324 */
static int gamma_calc(const double *pr, const geom_t *g, double *gamma)
{
  double qsq = g->gcov[1][1] * pr[U1] * pr[U1] + g->gcov[2][2] * pr[U2] * pr[U2]
               + g->gcov[3][3] * pr[U3] * pr[U3]
               + 2. * (g->gcov[1][2] * pr[U1] * pr[U2] + g->gcov[1][3] * pr[U1] * pr[U3]
                       + g->gcov[2][3] * pr[U2] * pr[U3]);
  if (qsq < 0.) {
    if (fabs(qsq) > 1.E-10) { *gamma = 1.; return 1; }
    qsq = 1.E-10;
  }
  *gamma = sqrt(1. + qsq);
  return 0;
}

/* phys.c:232-252 */
static void ucon_calc(ora_state *s, const double *pr, const geom_t *g, double *ucon)
{
  double alpha = 1. / sqrt(-g->gcon[0][0]);
  double beta[NDIM], gamma;
  for (int j = 1; j < 4; j++) beta[j] = g->gcon[0][j] * alpha * alpha;
  if (gamma_calc(pr, g, &gamma)) fail(s, FAIL_GAMMA);
  ucon[0] = gamma / alpha;
  for (int j = 1; j < 4; j++) ucon[j] = pr[U1 + j - 1] - gamma * beta[j] / alpha;
}

/* phys.c:108-117 */
static void bcon_calc(const double *pr, const double *ucon, const double *ucov, double *bcon)
{
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  for (int j = 1; j < 4; j++) bcon[j] = (pr[B1 - 1 + j] + bcon[0] * ucon[j]) / ucon[0];
}

/* phys.c:219-229 */
static void get_state(ora_state *s, const double *pr, const geom_t *g, state_t *q)
{
  ucon_calc(s, pr, g, q->ucon);
  lower(q->ucon, g, q->ucov);
  bcon_calc(pr, q->ucon, q->ucov, q->bcon);
  lower(q->bcon, g, q->bcov);
}

/* phys.c:143-161 */
static void mhd_calc(double gam, const double *pr, int dir, const state_t *q, double *mhd)
{
  double r = pr[RHO], u = pr[UU];
  double P = (gam - 1.) * u;
  double w = P + r + u;
  double bsq = dot4(q->bcon, q->bcov);
  double eta = w + bsq;
  double ptot = P + 0.5 * bsq;
  for (int j = 0; j < 4; j++)
    mhd[j] = eta * q->ucon[dir] * q->ucov[j] + ptot * (dir == j ? 1. : 0.)
             - q->bcon[dir] * q->bcov[j];
}

/* phys.c:59-96 */
static void primtoflux(double gam, const double *pr, const state_t *q, int dir, const geom_t *g,
                       double *flux)
{
  double mhd[NDIM];
  flux[RHO] = pr[RHO] * q->ucon[dir];
  mhd_calc(gam, pr, dir, q, mhd);
  flux[UU] = mhd[0] + flux[RHO];
  flux[U1] = mhd[1];
  flux[U2] = mhd[2];
  flux[U3] = mhd[3];
  flux[B1] = q->bcon[1] * q->ucon[dir] - q->bcon[dir] * q->ucon[1];
  flux[B2] = q->bcon[2] * q->ucon[dir] - q->bcon[dir] * q->ucon[2];
  flux[B3] = q->bcon[3] * q->ucon[dir] - q->bcon[dir] * q->ucon[3];
  for (int k = 0; k < NPR; k++) flux[k] *= g->g;
}

/* phys.c:337-476 (gamma-law branch) */
static void vchar(ora_state *s, double gam, const double *pr, const state_t *q, const geom_t *g,
                  int js, double *vmax, double *vmin)
{
  double Acov[NDIM] = {0., 0., 0., 0.}, Bcov[NDIM] = {0., 0., 0., 0.}, Acon[NDIM], Bcon[NDIM];
  Acov[js] = 1.;
  raise_(Acov, g, Acon);
  Bcov[0] = 1.;
  raise_(Bcov, g, Bcon);
  double bsq = dot4(q->bcon, q->bcov);
  double rho = pr[RHO], u = pr[UU];
  double EF = rho + gam * u;
  double EE = bsq + EF;
  double va2 = bsq / EE;
  double cs2 = gam * (gam - 1.) * u / EF;
  double cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.) { fail(s, FAIL_COEFF_NEG); cms2 = SMALL; }
  if (cms2 > 1.) { fail(s, FAIL_COEFF_SUP); cms2 = 1.; }
  double Asq = dot4(Acon, Acov), Bsq = dot4(Bcon, Bcov);
  double Au = dot4(Acov, q->ucon), Bu = dot4(Bcov, q->ucon), AB = dot4(Acon, Bcov);
  double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  double A = Bu2 - (Bsq + Bu2) * cms2;
  double B = 2. * (AuBu - (AB + AuBu) * cms2);
  double C = Au2 - (Asq + Au2) * cms2;
  double discr = B * B - 4. * A * C;
  if ((discr < 0.0) && (discr > -1.e-10)) discr = 0.0;
  else if (discr < -1.e-10) { fail(s, FAIL_VCHAR_DISCR); discr = 0.; }
  discr = sqrt(discr);
  double vp = -(-B + discr) / (2. * A);
  double vm = -(-B - discr) / (2. * A);
  if (vp > vm) { *vmax = vp; *vmin = vm; }
  else { *vmax = vm; *vmin = vp; }
}

/* phys.c:165-207; conn is this zone's [4][4][4] block */
static void source(ora_state *s, double gam, const double *ph, const geom_t *g, const double *conn,
                   double *dU)
{
  double mhd[NDIM][NDIM];
  state_t q;
  get_state(s, ph, g, &q);
  for (int d = 0; d < 4; d++) mhd_calc(gam, ph, d, &q, mhd[d]);
  for (int k = 0; k < NPR; k++) dU[k] = 0.;
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) {
      dU[UU] += mhd[j][k] * conn[(k * 4 + 0) * 4 + j];
      dU[U1] += mhd[j][k] * conn[(k * 4 + 1) * 4 + j];
      dU[U2] += mhd[j][k] * conn[(k * 4 + 2) * 4 + j];
      dU[U3] += mhd[j][k] * conn[(k * 4 + 3) * 4 + j];
    }
  for (int k = 0; k < NPR; k++) dU[k] *= g->g;
}

/* interp.c:49-93 */
static double slope_lim(int lim, double y1, double y2, double y3)
{
  double Dqm, Dqp, Dqc, s;
  if (lim == MC) {
    Dqm = 2. * (y2 - y1);
    Dqp = 2. * (y3 - y2);
    Dqc = 0.5 * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    if (fabs(Dqm) < fabs(Dqp) && fabs(Dqm) < fabs(Dqc)) return Dqm;
    if (fabs(Dqp) < fabs(Dqc)) return Dqp;
    return Dqc;
  }
  if (lim == VANL) {
    Dqm = (y2 - y1);
    Dqp = (y3 - y2);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    return 2. * s / (Dqm + Dqp);
  }
  Dqm = (y2 - y1);
  Dqp = (y3 - y2);
  s = Dqm * Dqp;
  if (s <= 0.) return 0.;
  if (fabs(Dqm) < fabs(Dqp)) return Dqm;
  return Dqp;
}

/* ------------------------------------------------------------------ */
/* conserved -> primitive inversions                                    */

/* the reference keeps these in file-scope globals (utoprim_1dfix1.c:78-80);
   here they live in one context per call */
typedef struct {
  double gam;
  double Bsq, QdotBsq, Qtsq, Qdotn, D, K_atm;
  double W_for_gnr2, rho_for_gnr2, W_for_gnr2_old, rho_for_gnr2_old;
} u2p_t;

/* u2p_util.c:176-199 */
static void raise_g(const double *vcov, const double gcon[4][4], double *vcon)
{
  for (int i = 0; i < NDIM; i++) {
    vcon[i] = 0.;
    for (int j = 0; j < NDIM; j++) vcon[i] += gcon[i][j] * vcov[j];
  }
}
static void lower_g(const double *vcon, const double gcov[4][4], double *vcov)
{
  for (int i = 0; i < NDIM; i++) {
    vcov[i] = 0.;
    for (int j = 0; j < NDIM; j++) vcov[i] += gcov[i][j] * vcon[j];
  }
}
/* u2p_util.c:208-219 */
static void ncov_calc(const double gcon[4][4], double *ncov)
{
  double lapse = sqrt(-1. / gcon[0][0]);
  ncov[0] = -lapse;
  for (int i = 1; i < NDIM; i++) ncov[i] = 0.;
}

/* scalars shared by the three inversions (utoprim_2d.c:229-262) */
static void u2p_scalars(u2p_t *c, const double *U, const double gcov[4][4], const double gcon[4][4],
                        double *Bcon, double *Qcon, double *ncon, double *QdotB)
{
  double Bcov[NDIM], Qcov[NDIM], ncov[NDIM], Qsq;
  Bcon[0] = 0.;
  for (int i = 1; i < 4; i++) Bcon[i] = U[B1 + i - 1];
  lower_g(Bcon, gcov, Bcov);
  for (int i = 0; i < 4; i++) Qcov[i] = U[UU + i];
  raise_g(Qcov, gcon, Qcon);
  c->Bsq = 0.;
  for (int i = 1; i < 4; i++) c->Bsq += Bcon[i] * Bcov[i];
  *QdotB = 0.;
  for (int i = 0; i < 4; i++) *QdotB += Qcov[i] * Bcon[i];
  c->QdotBsq = *QdotB * *QdotB;
  ncov_calc(gcon, ncov);
  raise_g(ncov, gcon, ncon);
  c->Qdotn = Qcon[0] * ncov[0];
  Qsq = 0.;
  for (int i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  c->Qtsq = Qsq + c->Qdotn * c->Qdotn;
  c->D = U[RHO];
}

/* utoprim_2d.c:269-282: returns 1 and the sq of u-tilde, or 0 on failure */
static int utsq_guess(const double gcov[4][4], const double *prim, double *utsq_out)
{
  double utsq = 0.;
  for (int i = 1; i < 4; i++)
    for (int j = 1; j < 4; j++) utsq += gcov[i][j] * prim[U1 + i - 1] * prim[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 0;
  *utsq_out = utsq;
  return 1;
}

static double vsq_calc(const u2p_t *c, double W)
{
  double Wsq = W * W;
  double Xsq = (c->Bsq + W) * (c->Bsq + W);
  return (Wsq * c->Qtsq + c->QdotBsq * (c->Bsq + 2. * W)) / (Wsq * Xsq);
}

/* utoprim_2d.c:394-405 */
static double x1_of_x0(const u2p_t *c, double x0)
{
  double vsq = fabs(vsq_calc(c, x0));
  return (vsq > 1.) ? (1.0 - 1.e-15) : vsq;
}

/* utoprim_2d.c:416-431 */
static void validate_x_2d(double x[2], const double x0[2])
{
  x[0] = fabs(x[0]);
  x[0] = (x[0] > W_TOO_BIG) ? x0[0] : x[0];
  x[1] = (x[1] < 0.) ? 0. : x[1];
  x[1] = (x[1] > 1.) ? (1. - 1.e-15) : x[1];
}

/* utoprim_2d.c:562-624 with the gamma-law EOS of :645-678 */
static void func_vsq(const u2p_t *c, const double x[2], double dx[2], double *f, double *df)
{
  double GAMMA = c->gam, Bsq = c->Bsq, QdotBsq = c->QdotBsq, Qtsq = c->Qtsq, Qdotn = c->Qdotn,
         D = c->D;
  double W = x[0], vsq = x[1], Wsq = W * W;
  double gtmp = 1. - vsq;
  double p_tmp = (GAMMA - 1.) * (W * gtmp - D * sqrt(gtmp)) / GAMMA;
  double dPdW = (GAMMA - 1.) * (1. - vsq) / GAMMA;
  double dPdvsq = (GAMMA - 1.) * (0.5 * D / sqrt(1. - vsq) - W) / GAMMA;
  double t2 = -0.5 * Bsq + dPdvsq;
  double t3 = Bsq + W;
  double t4 = t3 * t3;
  double t9 = 1. / Wsq;
  double t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
  double t16 = QdotBsq * t9;
  double t18 = -Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  double t21 = 1. / t3;
  double t23 = 1. / W;
  double t24 = t16 * t23;
  double t25 = -1.0 + dPdW - t24;
  double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  double t36 = 1. / t35;
  dx[0] = -(t2 * t11 + t4 * t18) * t21 * t36;
  double t40 = (vsq + t24) * t3;
  dx[1] = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
  double r0 = t11, r1 = t18;
  *df = -r0 * r0 - r1 * r1;
  *f = -0.5 * (*df);
}

/* utoprim_2d.c:442-541 */
static int gnr_2d(const u2p_t *c, double x[2])
{
  double f = 1., df = 1., dx[2], x_old[2], errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    func_vsq(c, x, dx, &f, &df);
    x_old[0] = x[0]; x_old[1] = x[1];
    x[0] += dx[0]; x[1] += dx[1];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    errx += (x[1] == 0.) ? fabs(dx[1]) : fabs(dx[1] / x[1]);
    validate_x_2d(x, x_old);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df)) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

/* utoprim_2d.c:219-362 */
static int u2p_body_2d(u2p_t *c, const double *U, const double gcov[4][4], const double gcon[4][4],
                       double *prim)
{
  double Bcon[NDIM], Qcon[NDIM], ncon[NDIM], QdotB, utsq;
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  u2p_scalars(c, U, gcov, gcon, Bcon, Qcon, ncon, &QdotB);
  if (!utsq_guess(gcov, prim, &utsq)) return 2;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c->D / gamma;
  double u = prim[UU];
  double p = (c->gam - 1.) * u;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c->Bsq) - c->QdotBsq * (2. * W_last + c->Bsq))
          <= W_last * W_last * (c->Qtsq - c->Bsq * c->Bsq))
         && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  double x[2];
  x[0] = fabs(W_last);
  x[1] = x1_of_x0(c, W_last);
  int retval = gnr_2d(c, x);
  double W = x[0], vsq = x[1];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c->D * gtmp;
  w = W * (1. - vsq);
  p = (c->gam - 1.) * (w - rho0) / c->gam;
  u = w - (rho0 + p);
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  double Qtcon[NDIM];
  for (int i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * c->Qdotn;
  for (int i = 1; i < 4; i++) prim[U1 + i - 1] = gamma / (W + c->Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  return 0;
}

/* the U/prim rescaling that wraps every inversion (utoprim_2d.c:126-176) */
typedef int (*u2p_body_fn)(u2p_t *, const double *, const double[4][4], const double[4][4], double *);

static int u2p_wrap(u2p_t *c, u2p_body_fn body, const double *U, const double gcov[4][4],
                    const double gcon[4][4], double gdet, double *prim)
{
  double U_tmp[NPR], prim_tmp[NPR];
  for (int i = B1; i <= B3; i++) prim[i] = U[i] / gdet;
  if (U[0] <= 0.) return -100;
  double alpha = 1.0 / sqrt(-gcon[0][0]);
  U_tmp[RHO] = alpha * U[RHO] / gdet;
  U_tmp[UU] = alpha * (U[UU] - U[RHO]) / gdet;
  for (int i = U1; i <= U3; i++) U_tmp[i] = alpha * U[i] / gdet;
  for (int i = B1; i <= B3; i++) U_tmp[i] = alpha * U[i] / gdet;
  for (int i = 0; i < B1; i++) prim_tmp[i] = prim[i];
  for (int i = B1; i <= B3; i++) prim_tmp[i] = alpha * prim[i];
  int ret = body(c, U_tmp, gcov, gcon, prim_tmp);
  if (ret == 0)
    for (int i = 0; i < B1; i++) prim[i] = prim_tmp[i];
  return ret;
}

/* Branch counts for the tests (ora_branch_counts): [0] floors that took the
   drift-frame branch, [1] inversions that Utoprim_1dvsq2fix1 rescued, [2]
   inversions that Utoprim_1dfix1 rescued.  They show which paths a test state
   exercises; the device step takes the same branches bit for bit. */
long ora_counts[3];

void ora_branch_counts(long *out, int reset)
{
  for (int k = 0; k < 3; k++) {
    out[k] = ora_counts[k];
    if (reset) ora_counts[k] = 0;
  }
}

/* --- Utoprim_1dvsq2fix1 (utoprim_1dvsq2fix1.c) --- */

/* :583-606 */
static double W_of_vsq_fix(const u2p_t *c, double vsq, double *p, double *rho, double *u)
{
  double gtmp = (1. - vsq);
  *rho = c->D * sqrt(gtmp);
  *p = c->K_atm * pow(*rho, c->gam);
  *u = *p / (c->gam - 1.);
  return (*rho + *u + *p) / gtmp;
}

/* :615-622 */
static double dWdvsq_calc(double GAMMA, double vsq, double rho, double p)
{
  return (GAMMA * (2. - GAMMA) * p + (GAMMA - 1.) * rho) / (2. * (GAMMA - 1.) * (1. - vsq) * (1. - vsq));
}

/* :541-566 */
static void func_1d_gnr(const u2p_t *c, const double *x, double *dx, double *f, double *df)
{
  double p, rho, u, vsq = x[0];
  double W = W_of_vsq_fix(c, vsq, &p, &rho, &u);
  double Wsq = W * W, W3 = W * Wsq;
  double dWdvsq = dWdvsq_calc(c->gam, vsq, rho, p);
  double fact_tmp = (c->Bsq + W);
  double r0 = c->Qtsq - vsq * fact_tmp * fact_tmp + c->QdotBsq * (c->Bsq + 2. * W) / Wsq;
  double j00 = -fact_tmp * (fact_tmp + 2. * dWdvsq * (vsq + c->QdotBsq / W3));
  dx[0] = -r0 / j00;
  *f = 0.5 * r0 * r0;
  *df = -2. * (*f);
}

/* :373-380 */
static void validate_x_1d(double *x, const double *x0)
{
  double small = 1.e-10;
  x[0] = (x[0] >= 1.0) ? (0.5 * (x0[0] + 1.)) : x[0];
  x[0] = (x[0] < -small) ? (0.5 * x0[0]) : x[0];
  x[0] = fabs(x[0]);
}

/* :395-492 */
static int gnr_vsq2fix1(const u2p_t *c, double *x)
{
  double f = 1., df = 1., dx[1], x_old[1], errx = 1., W = 0., W_old, p, rho, u;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    func_1d_gnr(c, x, dx, &f, &df);
    x_old[0] = x[0];
    x[0] += dx[0];
    validate_x_1d(x, x_old);
    W_old = W;
    W = W_of_vsq_fix(c, x[0], &p, &rho, &u);
    errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
    errx += (x[0] == 0.) ? fabs(x[0] - x_old[0]) : fabs((x[0] - x_old[0]) / x[0]);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df)) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

/* :222-356 */
static int u2p_body_vsq2fix1(u2p_t *c, const double *U, const double gcov[4][4],
                             const double gcon[4][4], double *prim)
{
  double Bcon[NDIM], Qcon[NDIM], ncon[NDIM], QdotB, utsq, p, rho0, u;
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  u2p_scalars(c, U, gcov, gcon, Bcon, Qcon, ncon, &QdotB);
  if (!utsq_guess(gcov, prim, &utsq)) return 2;
  double gammasq = 1. + utsq;
  double x[1];
  x[0] = 1. - 1. / gammasq;
  int retval = gnr_vsq2fix1(c, x);
  if (retval != 0) return retval * 100 + 1;
  double vsq = x[0];
  if ((vsq >= 1.) || (vsq < 0.)) return 4;
  double W = W_of_vsq_fix(c, vsq, &p, &rho0, &u);
  double gtmp = sqrt(1. - vsq);
  double gamma = 1. / gtmp;
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  double Qtcon[NDIM];
  for (int i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * c->Qdotn;
  for (int i = 1; i < 4; i++) prim[U1 + i - 1] = gamma / (W + c->Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  return 0;
}

/* --- Utoprim_1dfix1 (utoprim_1dfix1.c) --- */

/* :818-838 */
static void func_gnr2_rho(const u2p_t *c, const double *x, double *dx, double *f, double *df)
{
  double GAMMA = c->gam;
  double A = c->D * c->D;
  double B0 = A * GAMMA * c->K_atm;
  double B = B0 / (GAMMA - 1.);
  double rho = x[0];
  double W = c->W_for_gnr2;
  double C = pow(rho, GAMMA - 1.);
  double r0 = rho * W - A - B * C;
  double j00 = W - B0 * C / rho;
  dx[0] = -r0 / j00;
  *f = 0.5 * r0 * r0;
  *df = -2. * (*f);
}

/* :601-697 */
static int gnr2(const u2p_t *c, double *x)
{
  double f = 1., df = 1., dx[1], errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    func_gnr2_rho(c, x, dx, &f, &df);
    x[0] += dx[0];
    errx = 0.;
    errx += (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    errx /= 1. * 1;
    x[0] = fabs(x[0]);
    /* the reference's extra-iteration switch stays off here (:667-669) */
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL2) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

/* :721-771 */
static void func_1d_orig1(u2p_t *c, const double *x, double *dx, double *f, double *df)
{
  double GAMMA = c->gam, K_atm = c->K_atm, Bsq = c->Bsq, QdotBsq = c->QdotBsq, Qtsq = c->Qtsq;
  double W = x[0], x_rho[1], rho_g;
  int ntries = 0;
  c->W_for_gnr2_old = c->W_for_gnr2;
  c->W_for_gnr2 = W;
  rho_g = x_rho[0] = c->rho_for_gnr2;
  while (gnr2(c, x_rho) && (ntries++ < 10)) {
    rho_g *= 10.;
    x_rho[0] = rho_g;
  }
  c->rho_for_gnr2_old = c->rho_for_gnr2;
  double rho = c->rho_for_gnr2 = x_rho[0];
  double Dc = c->D;
  double t1 = Dc * Dc, t2 = QdotBsq * t1, t3 = t2 * Bsq, t5 = Bsq * Bsq, t8 = t1 * Bsq,
         t10 = t1 * W, t21 = W * W, t23 = rho * rho, t26 = 1. / t1;
  double r0 = (t3 + (2.0 * t2 + ((Qtsq - t5) * t1 + (-2.0 * t8 - t10) * W) * W) * W
               + (t5 + (2.0 * Bsq + W) * W) * t21 * t23) * t26 / t21;
  double t29 = t1 * t1, t30 = QdotBsq * t29, t32 = GAMMA * K_atm, t33 = pow(rho, 1.0 * GAMMA),
         t34 = t32 * t33, t38 = t23 * t33, t51 = GAMMA * t1 * K_atm * t33, t67 = t21 * W;
  double j00 = -2.0 * (t30 * Bsq * t34
                       + (t30 * t34 + ((-t38 * Bsq * t32 + Bsq * GAMMA * t1 * K_atm * t33) * t1
                                       + (-t38 * GAMMA * K_atm + t51) * t1 * W) * t21) * W
                       + ((-t3 + (-t2 + (-t8 - t10) * t21) * W) * W + (-t5 - Bsq * W) * t67 * t23) * t23)
               * t26 / (t51 - W * t23) / t67;
  dx[0] = -r0 / j00;
  *f = 0.5 * r0 * r0;
  *df = -2. * (*f);
}

/* :500-595 */
static int gnr_fix1(u2p_t *c, double *x)
{
  double f = 1., df = 1., dx[1], errx = 1.;
  const double Bsq = c->Bsq, QdotBsq = c->QdotBsq, Qtsq = c->Qtsq;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    func_1d_orig1(c, x, dx, &f, &df);
    x[0] += dx[0];
    int i_increase = 0;
    while (((x[0] * x[0] * x[0] * (x[0] + 2. * Bsq) - QdotBsq * (2. * x[0] + Bsq))
            <= x[0] * x[0] * (Qtsq - Bsq * Bsq))
           && (i_increase < 10)) {
      x[0] -= (1. * i_increase) * dx[0] / 10.;
      i_increase++;
    }
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    x[0] = fabs(x[0]);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

/* :223-367 */
static int u2p_body_fix1(u2p_t *c, const double *U, const double gcov[4][4], const double gcon[4][4],
                         double *prim)
{
  double Bcon[NDIM], Qcon[NDIM], ncon[NDIM], QdotB, utsq;
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  u2p_scalars(c, U, gcov, gcon, Bcon, Qcon, ncon, &QdotB);
  if (!utsq_guess(gcov, prim, &utsq)) return 2;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c->D / gamma;
  double p = c->K_atm * pow(rho0, c->gam);
  double u = p / (c->gam - 1.);
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c->Bsq) - c->QdotBsq * (2. * W_last + c->Bsq))
          <= W_last * W_last * (c->Qtsq - c->Bsq * c->Bsq))
         && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  c->W_for_gnr2 = c->W_for_gnr2_old = W_last;
  c->rho_for_gnr2 = c->rho_for_gnr2_old = rho0;
  double x[1] = {W_last};
  int retval = gnr_fix1(c, x);
  double W = x[0];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  double vsq = vsq_calc(c, W);
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c->D * gtmp;
  p = c->K_atm * pow(rho0, c->gam);
  u = p / (c->gam - 1.);
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  double Qtcon[NDIM];
  for (int i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * c->Qdotn;
  for (int i = 1; i < 4; i++) prim[U1 + i - 1] = gamma / (W + c->Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  for (int i = B1; i <= B3; i++) prim[i] = U[i];
  return 0;
}

int ora_utoprim_2d(double gam, const double U[8], const double *gcov, const double *gcon,
                   double gdet, double *prim)
{
  u2p_t c = {0};
  c.gam = gam;
  return u2p_wrap(&c, u2p_body_2d, U, (const double(*)[4])gcov, (const double(*)[4])gcon, gdet, prim);
}

int ora_utoprim_1dvsq2fix1(double gam, const double U[8], const double *gcov,
                           const double *gcon, double gdet, double *prim, double K)
{
  u2p_t c = {0};
  c.gam = gam;
  c.K_atm = K;
  int r = u2p_wrap(&c, u2p_body_vsq2fix1, U, (const double(*)[4])gcov, (const double(*)[4])gcon,
                   gdet, prim);
  return r;
}

int ora_utoprim_1dfix1(double gam, const double U[8], const double *gcov, const double *gcon,
                       double gdet, double *prim, double K)
{
  u2p_t c = {0};
  c.gam = gam;
  c.K_atm = K;
  return u2p_wrap(&c, u2p_body_fix1, U, (const double(*)[4])gcov, (const double(*)[4])gcon, gdet, prim);
}

/* ------------------------------------------------------------------ */
/* floors: fixup.c                                                      */

/* fixup.c:117-140 (BL branch) */
static void get_rho_u_floor(double gam, double r, double *rho_floor, double *u_floor)
{
  double rhoscal = pow(r, -POWRHO);
  double uuscal = pow(rhoscal, gam);
  double rhoflr = RHOMIN * rhoscal;
  double uuflr = UUMIN * uuscal;
  if (rhoflr < RHOMINLIMIT) rhoflr = RHOMINLIMIT;
  if (uuflr < UUMINLIMIT) uuflr = UUMINLIMIT;
  *rho_floor = rhoflr;
  *u_floor = uuflr;
}

/* phys.c:273-297 */
static void ut_calc_3vel(const double *vcon, const geom_t *g, double *ut)
{
  double AA = g->gcov[0][0];
  double BB = 2. * (g->gcov[0][1] * vcon[1] + g->gcov[0][2] * vcon[2] + g->gcov[0][3] * vcon[3]);
  double CC = g->gcov[1][1] * vcon[1] * vcon[1] + g->gcov[2][2] * vcon[2] * vcon[2]
              + g->gcov[3][3] * vcon[3] * vcon[3]
              + 2. * (g->gcov[1][2] * vcon[1] * vcon[2] + g->gcov[1][3] * vcon[1] * vcon[3]
                      + g->gcov[2][3] * vcon[2] * vcon[3]);
  double DD = -1. / (AA + BB + CC);
  double one_over_alpha_sq = -g->gcon[0][0];
  if (DD < one_over_alpha_sq) DD = one_over_alpha_sq;
  *ut = sqrt(DD);
}

/* phys.c:255-270 */
static void ucon_to_utcon(const double *ucon, const geom_t *g, double *utcon)
{
  double alpha = 1. / sqrt(-g->gcon[0][0]);
  double beta[NDIM];
  for (int j = 1; j < 4; j++) beta[j] = g->gcon[0][j] * alpha * alpha;
  double gamma = alpha * ucon[0];
  utcon[0] = 0;
  for (int j = 1; j < 4; j++) utcon[j] = ucon[j] + gamma * beta[j] / alpha;
}

/* fixup.c:142-383 (DRIFT_FLOOR=1, DOKTOT=0) */
static void fixup1zone(ora_state *s, int h, int i, int j, double *pv)
{
  double gam = s->prm.gam;
  double pv_prefloor[NPR], rhoflr, uuflr, gamma, f;
  geom_t g;
  state_t q;
  for (int k = 0; k < NPR; k++) pv_prefloor[k] = pv[k];
  double r = s->coords[((size_t)i * s->sn2 + j) * 4 + 1];
  get_rho_u_floor(gam, r, &rhoflr, &uuflr);
  get_geometry(s, h, i, j, CENT, &g);
  get_state(s, pv, &g, &q);
  double bsq = dot4(q.bcon, q.bcov);
  if (rhoflr < bsq / BSQORHOMAX) rhoflr = bsq / BSQORHOMAX;
  if (uuflr < bsq / BSQOUMAX) uuflr = bsq / BSQOUMAX;
  if (rhoflr < pv[UU] / UORHOMAX) rhoflr = pv[UU] / UORHOMAX;
  int dofloor = 0;
  if (pv[RHO] < rhoflr) { pv[RHO] = rhoflr; dofloor = 1; }
  if (pv[UU] < uuflr) { pv[UU] = uuflr; dofloor = 1; }
  double trans;
  if (dofloor && (trans = 10. * bsq / (pv[RHO] < pv[UU] ? pv[RHO] : pv[UU]) - 1.) > 0.) {
    ora_counts[0]++;
    if (trans > 1.) trans = 1.;
    double betapar = -q.bcon[0] / ((bsq + SMALL) * q.ucon[0]);
    double betasq = betapar * betapar * bsq;
    double betasqmax = 1. - 1. / (GAMMAMAX * GAMMAMAX);
    if (betasq > betasqmax) betasq = betasqmax;
    double gdr = 1. / sqrt(1 - betasq);
    double ucondr[NDIM], Bcon[NDIM], Bcov[NDIM], vcon[NDIM], ucon[NDIM], utcon[NDIM], ut;
    for (int k = 0; k < NDIM; k++) ucondr[k] = gdr * (q.ucon[k] + betapar * q.bcon[k]);
    Bcon[0] = 0.;
    for (int k = 1; k < NDIM; k++) Bcon[k] = pv[B1 - 1 + k];
    lower(Bcon, &g, Bcov);
    double udotB = dot4(q.ucon, Bcov);
    double Bsq = dot4(Bcon, Bcov);
    double B = sqrt(Bsq);
    double wold = pv_prefloor[RHO] + pv_prefloor[UU] * gam;
    double QdotB = udotB * wold * q.ucon[0];
    double wnew = pv[RHO] + pv[UU] * gam;
    double x = 2. * QdotB / (B * wnew * ucondr[0] + SMALL);
    double vpar = x / (ucondr[0] * (1. + sqrt(1. + x * x)));
    double one_over_ucondr_t = 1. / ucondr[0];
    vcon[0] = 1.;
    for (int k = 1; k < NDIM; k++) vcon[k] = vpar * Bcon[k] / (B + SMALL) + ucondr[k] * one_over_ucondr_t;
    ut_calc_3vel(vcon, &g, &ut);
    for (int k = 0; k < NDIM; k++) ucon[k] = ut * vcon[k];
    ucon_to_utcon(ucon, &g, utcon);
    for (int k = 1; k < NDIM; k++) pv[k + UU] = utcon[k] * trans + pv_prefloor[k + UU] * (1. - trans);
  }
  if (gamma_calc(pv, &g, &gamma)) {
    s->pflag[zidx(s, h, i, j)] = -33;
  } else if (gamma > GAMMAMAX) {
    f = sqrt((GAMMAMAX * GAMMAMAX - 1.) / (gamma * gamma - 1.));
    pv[U1] *= f;
    pv[U2] *= f;
    pv[U3] *= f;
  }
}

/* ------------------------------------------------------------------ */
/* loops                                                               */

/* ZLOOP / ZSLOOP bounds for one rank (decs.h:455-494) */
#define HLO(s, m) ((s)->prm.n3 == 1 ? 0 : (s)->hstart + (m))
#define HHI(s, m) ((s)->prm.n3 == 1 ? 0 : (s)->hstop + (m))
#define ZSLOOP(s, hs, he, is, ie, js, je)                                    \
  for (int h = HLO(s, hs); h <= HHI(s, he); h++)                            \
    for (int i = (s)->istart + (is); i <= (s)->istop + (ie); i++)           \
      for (int j = (s)->jstart + (js); j <= (s)->jstop + (je); j++)
#define ZLOOP(s) ZSLOOP(s, 0, 0, 0, 0, 0, 0)

/* the phi self-exchange of one whole plane (mpi.c:284-321 slices, hsize=1) */
static void copy_plane(ora_state *s, double *arr, int ncomp, int hdst, int hsrc)
{
  size_t n = (size_t)s->sn1 * s->sn2 * ncomp;
  memcpy(arr + (size_t)hdst * n, arr + (size_t)hsrc * n, n * sizeof(double));
}

/* fixup.c:51-60 */
void ora_fixup(ora_state *s, double *pv)
{
  ZLOOP(s) fixup1zone(s, h, i, j, PV(s, pv, h, i, j));
}

/* bounds.c:333-378 */
static void inflow_check(ora_state *s, double *pr, int h, int i, int j, int type)
{
  geom_t g;
  double ucon[NDIM], gamma;
  get_geometry(s, h, i, j, CENT, &g);
  ucon_calc(s, pr, &g, ucon);
  if (((ucon[1] > 0.) && (type == 0)) || ((ucon[1] < 0.) && (type == 1))) {
    if (gamma_calc(pr, &g, &gamma)) fail(s, FAIL_GAMMA);
    pr[U1] /= gamma;
    pr[U2] /= gamma;
    pr[U3] /= gamma;
    double alpha = 1. / sqrt(-g.gcon[0][0]);
    double beta1 = g.gcon[0][1] * alpha * alpha;
    pr[U1] = beta1 / alpha;
    double vsq = 0.;
    for (int a = 1; a < NDIM; a++)
      for (int b = 1; b < NDIM; b++) vsq += g.gcov[a][b] * pr[U1 + a - 1] * pr[U1 + b - 1];
    if (fabs(vsq) < 1.e-13) vsq = 1.e-13;
    if (vsq >= 1.) vsq = 1. - 1. / (GAMMAMAX * GAMMAMAX);
    gamma = 1. / sqrt(1. - vsq);
    pr[U1] *= gamma;
    pr[U2] *= gamma;
    pr[U3] *= gamma;
  }
}

/* opposite-phi plane of h on one rank (mpi.c:374-386 with hsize=1) */
static int opposite_h(int n3, int h)
{
  int oxx = (h + n3 / 2 == n3) ? n3 : ((h + n3 / 2) % n3);
  return oxx;
}

/* bounds.c:54-331 and the polefix of :381-436 */
void ora_bound_prim(ora_state *s, double *prim)
{
  signed char *pflag = s->pflag;
  int n3 = s->prm.n3;
  /* inner and outer radial: copy */
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart; j <= s->jstop; j++) {
      for (int k = 0; k < NPR; k++) {
        PV(s, prim, h, s->istart - 1, j)[k] = PV(s, prim, h, s->istart, j)[k];
        PV(s, prim, h, s->istart - 2, j)[k] = PV(s, prim, h, s->istart, j)[k];
      }
      pflag[zidx(s, h, s->istart - 1, j)] = pflag[zidx(s, h, s->istart, j)];
      pflag[zidx(s, h, s->istart - 2, j)] = pflag[zidx(s, h, s->istart, j)];
    }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart; j <= s->jstop; j++) {
      for (int k = 0; k < NPR; k++) {
        PV(s, prim, h, s->istop + 1, j)[k] = PV(s, prim, h, s->istop, j)[k];
        PV(s, prim, h, s->istop + 2, j)[k] = PV(s, prim, h, s->istop, j)[k];
      }
      pflag[zidx(s, h, s->istop + 1, j)] = pflag[zidx(s, h, s->istop, j)];
      pflag[zidx(s, h, s->istop + 2, j)] = pflag[zidx(s, h, s->istop, j)];
    }
  if (n3 > 1) {
    /* polefix (bounds.c:381-436), POLEFIX=2 in 3D */
    const int jref = POLEFIX_ROWS;
    for (int h = s->hstart; h <= s->hstop; h++)
      for (int i = s->istart - 2; i <= s->istop + 2; i++)
        for (int jj = 0; jj < jref; jj++)
          for (int k = 0; k < NPR; k++) {
            if (k == B1 || k == B2 || k == B3) continue;
            if (k == U2)
              PV(s, prim, h, i, s->jstart + jj)[k] =
                  (jj + 0.5) / (jref + 0.5) * PV(s, prim, h, i, s->jstart + jref)[k];
            else
              PV(s, prim, h, i, s->jstart + jj)[k] = PV(s, prim, h, i, s->jstart + jref)[k];
          }
    for (int h = s->hstart; h <= s->hstop; h++)
      for (int i = s->istart - 2; i <= s->istop + 2; i++)
        for (int jj = 0; jj < jref; jj++)
          for (int k = 0; k < NPR; k++) {
            if (k == B1 || k == B2 || k == B3) continue;
            if (k == U2)
              PV(s, prim, h, i, s->jstop - jj)[k] =
                  (jj + 0.5) / (jref + 0.5) * PV(s, prim, h, i, s->jstop - jref)[k];
            else
              PV(s, prim, h, i, s->jstop - jj)[k] = PV(s, prim, h, i, s->jstop - jref)[k];
          }
    /* polar ghosts from the opposite-phi plane, staged through dq (bounds.c:156-250) */
    double *dq = s->dq;
    for (int h = s->hstart; h <= s->hstop; h++)
      for (int i = s->istart - 2; i <= s->istop + 2; i++) {
        for (int k = 0; k < NPR; k++) {
          PV(s, dq, h, i, s->jstart - 1)[k] = PV(s, prim, h, i, s->jstart)[k];
          PV(s, dq, h, i, s->jstart - 2)[k] = PV(s, prim, h, i, s->jstart + 1)[k];
        }
        pflag[zidx(s, h, i, s->jstart - 1)] = pflag[zidx(s, h, i, s->jstart)];
        pflag[zidx(s, h, i, s->jstart - 2)] = pflag[zidx(s, h, i, s->jstart + 1)];
      }
    for (int h = s->hstart; h <= s->hstop; h++)
      for (int i = s->istart - 2; i <= s->istop + 2; i++) {
        for (int k = 0; k < NPR; k++) {
          PV(s, dq, h, i, s->jstop + 1)[k] = PV(s, prim, h, i, s->jstop)[k];
          PV(s, dq, h, i, s->jstop + 2)[k] = PV(s, prim, h, i, s->jstop - 1)[k];
        }
        pflag[zidx(s, h, i, s->jstop + 1)] = pflag[zidx(s, h, i, s->jstop)];
        pflag[zidx(s, h, i, s->jstop + 2)] = pflag[zidx(s, h, i, s->jstop - 1)];
      }
    for (int h = s->hstart; h <= s->hstop; h++) {
      int ho = opposite_h(n3, h);
      for (int i = s->istart - 2; i <= s->istop + 2; i++)
        for (int k = 0; k < NPR; k++) {
          PV(s, prim, h, i, s->jstart - 2)[k] = PV(s, dq, ho, i, s->jstart - 2)[k];
          PV(s, prim, h, i, s->jstart - 1)[k] = PV(s, dq, ho, i, s->jstart - 1)[k];
        }
    }
    for (int h = s->hstart; h <= s->hstop; h++) {
      int ho = opposite_h(n3, h);
      for (int i = s->istart - 2; i <= s->istop + 2; i++)
        for (int k = 0; k < NPR; k++) {
          PV(s, prim, h, i, s->jstop + 1)[k] = PV(s, dq, ho, i, s->jstop + 1)[k];
          PV(s, prim, h, i, s->jstop + 2)[k] = PV(s, dq, ho, i, s->jstop + 2)[k];
        }
    }
  } else {
    /* 2D: reflect (bounds.c:279-300) */
    for (int i = s->istart - 2; i <= s->istop + 2; i++) {
      for (int k = 0; k < NPR; k++) {
        PV(s, prim, 0, i, s->jstart - 1)[k] = PV(s, prim, 0, i, s->jstart)[k];
        PV(s, prim, 0, i, s->jstart - 2)[k] = PV(s, prim, 0, i, s->jstart + 1)[k];
      }
      pflag[zidx(s, 0, i, s->jstart - 1)] = pflag[zidx(s, 0, i, s->jstart)];
      pflag[zidx(s, 0, i, s->jstart - 2)] = pflag[zidx(s, 0, i, s->jstart + 1)];
    }
    for (int i = s->istart - 2; i <= s->istop + 2; i++) {
      for (int k = 0; k < NPR; k++) {
        PV(s, prim, 0, i, s->jstop + 1)[k] = PV(s, prim, 0, i, s->jstop)[k];
        PV(s, prim, 0, i, s->jstop + 2)[k] = PV(s, prim, 0, i, s->jstop - 1)[k];
      }
      pflag[zidx(s, 0, i, s->jstop + 1)] = pflag[zidx(s, 0, i, s->jstop)];
      pflag[zidx(s, 0, i, s->jstop + 2)] = pflag[zidx(s, 0, i, s->jstop - 1)];
    }
  }
  /* U2, B2 antisymmetric across the poles (bounds.c:253-275, 302-319) */
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istart - 2; i <= s->istop + 2; i++) {
      for (int j = s->jstart - 2; j < s->jstart; j++) {
        PV(s, prim, h, i, j)[U2] *= -1.;
        PV(s, prim, h, i, j)[B2] *= -1.;
      }
    }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istart - 2; i <= s->istop + 2; i++) {
      for (int j = s->jstop + 1; j <= s->jstop + 2; j++) {
        PV(s, prim, h, i, j)[U2] *= -1.;
        PV(s, prim, h, i, j)[B2] *= -1.;
      }
    }
  /* no inflow through the radial boundaries (bounds.c:321-329) */
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istart - 2; i <= s->istart - 1; i++)
      for (int j = s->jstart - 2; j <= s->jstop + 2; j++) inflow_check(s, PV(s, prim, h, i, j), h, i, j, 0);
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istop + 1; i <= s->istop + 2; i++)
      for (int j = s->jstart - 2; j <= s->jstop + 2; j++) inflow_check(s, PV(s, prim, h, i, j), h, i, j, 1);
}

/* fixup.c:432-538 (FIXUPAVG=1) */
void ora_fixup_utoprim(ora_state *s, double *pv)
{
  signed char *pflag = s->pflag;
  ZSLOOP(s, 0, 0, -2, 2, -2, 2) pflag[zidx(s, h, i, j)] = !pflag[zidx(s, h, i, j)];
  ZLOOP(s) {
    if (pflag[zidx(s, h, i, j)] == 0) {
#define PF(di, dj) (pflag[zidx(s, h, i + (di), j + (dj))] != 0)
#define Q(di, dj, k) PV(s, pv, h, i + (di), j + (dj))[k]
      int pf1 = PF(-1, 1), pf2 = PF(0, 1), pf3 = PF(1, 1), pf8 = PF(-1, 0), pf4 = PF(1, 0),
          pf7 = PF(-1, -1), pf6 = PF(0, -1), pf5 = PF(1, -1);
      double *z = PV(s, pv, h, i, j);
      if (pf2 && pf4 && pf6 && pf8) {
        for (int k = 0; k < B1; k++) z[k] = 0.25 * (Q(0, 1, k) + Q(0, -1, k) + Q(-1, 0, k) + Q(1, 0, k));
      } else if (pf1 && pf3 && pf5 && pf7) {
        for (int k = 0; k < B1; k++) z[k] = 0.25 * (Q(1, 1, k) + Q(1, -1, k) + Q(-1, 1, k) + Q(-1, -1, k));
      } else {
        for (int k = RHO; k <= UU; k++)
          z[k] = 0.5 * (0.25 * (Q(0, 1, k) + Q(0, -1, k) + Q(-1, 0, k) + Q(1, 0, k))
                        + 0.25 * (Q(1, 1, k) + Q(1, -1, k) + Q(-1, 1, k) + Q(-1, -1, k)));
        z[U1] = z[U2] = z[U3] = 0.;
      }
#undef PF
#undef Q
      pflag[zidx(s, h, i, j)] = 0;
      fixup1zone(s, h, i, j, z);
    }
  }
}

/* ------------------------------------------------------------------ */
/* fluxes                                                              */

/* one face: step_ch.c:429-473 with HLLF=0, LAXF=1 */
static void face_flux(ora_state *s, double gam, int dir, const double *p_l, const double *p_r,
                      const geom_t *g, double *F, double *ctop_out)
{
  state_t sl, sr;
  double F_l[NPR], F_r[NPR], U_l[NPR], U_r[NPR], cmax_l, cmin_l, cmax_r, cmin_r;
  get_state(s, p_l, g, &sl);
  get_state(s, p_r, g, &sr);
  primtoflux(gam, p_l, &sl, dir, g, F_l);
  primtoflux(gam, p_l, &sl, 0, g, U_l);
  vchar(s, gam, p_l, &sl, g, dir, &cmax_l, &cmin_l);
  primtoflux(gam, p_r, &sr, dir, g, F_r);
  primtoflux(gam, p_r, &sr, 0, g, U_r);
  vchar(s, gam, p_r, &sr, g, dir, &cmax_r, &cmin_r);
  double t1 = 0. > cmax_l ? 0. : cmax_l;
  double cmax = fabs(t1 > cmax_r ? t1 : cmax_r);
  double t2 = 0. > -cmin_l ? 0. : -cmin_l;
  double cmin = fabs(t2 > -cmin_r ? t2 : -cmin_r);
  double ctop = cmax > cmin ? cmax : cmin;
  for (int k = 0; k < NPR; k++)
    F[k] = 0.0 * ((cmax * F_l[k] + cmin * F_r[k] - cmax * cmin * (U_r[k] - U_l[k])) / (cmax + cmin + SMALL))
           + 1.0 * (0.5 * (F_l[k] + F_r[k] - ctop * (U_r[k] - U_l[k])));
  *ctop_out = ctop;
}

void ora_face_flux(double gam, int dir, const double pl[8], const double pr[8],
                   const double *gcov, const double *gcon, double gdet,
                   double F[8], double *ctop)
{
  geom_t g;
  geom_from(gcov, gcon, gdet, &g);
  face_flux(NULL, gam, dir, pl, pr, &g, F, ctop);
}

/* step_ch.c:331-504 */
static double fluxcalc(ora_state *s, double *pr, double *F, int dir, int fullstep)
{
  int hdel = dir == 3, idel = dir == 1, jdel = dir == 2;
  int face = dir == 1 ? FACE1 : dir == 2 ? FACE2 : FACE3;
  double gam = s->prm.gam;
  double *dq = s->dq;
  ZSLOOP(s, 0, 0, -1, 1, -1, 1) {
    for (int k = 0; k < NPR; k++)
      PV(s, dq, h, i, j)[k] = slope_lim(s->prm.lim, PV(s, pr, h - hdel, i - idel, j - jdel)[k],
                                        PV(s, pr, h, i, j)[k], PV(s, pr, h + hdel, i + idel, j + jdel)[k]);
  }
  if (hdel) copy_plane(s, dq, NPR, s->hstart - 1, s->hstop);
  double ndt = 1.e9;
  ZSLOOP(s, 0, 0, -hdel - jdel, 1, -hdel - idel, 1) {
    double *Fz = PV(s, F, h, i, j);
    if (dir == 2 && (j == s->jstart || j == s->jstop + 1)) {
      for (int k = 0; k < NPR; k++) Fz[k] = 0.;
      continue;
    }
    double p_l[NPR], p_r[NPR], ctop;
    const double *pm = PV(s, pr, h - hdel, i - idel, j - jdel), *dqm = PV(s, dq, h - hdel, i - idel, j - jdel);
    const double *pz = PV(s, pr, h, i, j), *dqz = PV(s, dq, h, i, j);
    for (int k = 0; k < NPR; k++) {
      p_l[k] = pm[k] + 0.5 * dqm[k];
      p_r[k] = pz[k] - 0.5 * dqz[k];
    }
    geom_t g;
    get_geometry(s, h, i, j, face, &g);
    face_flux(s, gam, dir, p_l, p_r, &g, Fz, &ctop);
    if (fullstep && i >= s->istart && i <= s->istop && j >= s->jstart && j <= s->jstop) {
      double dtij = s->prm.cour * s->prm.dx[dir] / ctop;
      if (dtij < ndt) ndt = dtij;
    }
  }
  return ndt;
}

/* coord.c:264-324 */
static void fix_flux(ora_state *s)
{
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istart - 1; i <= s->istop + 1; i++) {
      PV(s, s->F1, h, i, s->jstart - 1)[B2] = -PV(s, s->F1, h, i, s->jstart)[B2];
      if (s->prm.n3 > 1) PV(s, s->F3, h, i, s->jstart - 1)[B2] = -PV(s, s->F3, h, i, s->jstart)[B2];
      for (int k = 0; k < NPR; k++) PV(s, s->F2, h, i, s->jstart)[k] = 0.;
    }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int i = s->istart - 1; i <= s->istop + 1; i++) {
      PV(s, s->F1, h, i, s->jstop + 1)[B2] = -PV(s, s->F1, h, i, s->jstop)[B2];
      if (s->prm.n3 > 1) PV(s, s->F3, h, i, s->jstop + 1)[B2] = -PV(s, s->F3, h, i, s->jstop)[B2];
      for (int k = 0; k < NPR; k++) PV(s, s->F2, h, i, s->jstop + 1)[k] = 0.;
    }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart - 2; j <= s->jstop + 2; j++)
      if (PV(s, s->F1, h, s->istart, j)[RHO] > 0) PV(s, s->F1, h, s->istart, j)[RHO] = 0;
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart - 2; j <= s->jstop + 2; j++)
      if (PV(s, s->F1, h, s->istop + 1, j)[RHO] < 0) PV(s, s->F1, h, s->istop + 1, j)[RHO] = 0;
}

#define E(arr, h, i, j) (arr)[zidx(s, h, i, j)]

/* step_ch.c:514-629 (N3 <= 2) */
static void flux_ct_2d(ora_state *s)
{
  double *F1 = s->F1, *F2 = s->F2, *emf = s->e1;
  ZSLOOP(s, 0, 0, 0, 1, 0, 1)
  E(emf, h, i, j) = 0.25 * (PV(s, F1, h, i, j)[B2] + PV(s, F1, h, i, j - 1)[B2] - PV(s, F2, h, i, j)[B1]
                            - PV(s, F2, h, i - 1, j)[B1]);
  ZSLOOP(s, 0, 0, 0, 1, 0, 0) {
    PV(s, F1, h, i, j)[B1] = 0.;
    PV(s, F1, h, i, j)[B2] = 0.5 * (E(emf, h, i, j) + E(emf, h, i, j + 1));
  }
  ZSLOOP(s, 0, 0, 0, 0, 0, 1) {
    PV(s, F2, h, i, j)[B1] = -0.5 * (E(emf, h, i, j) + E(emf, h, i + 1, j));
    PV(s, F2, h, i, j)[B2] = 0.;
  }
}

/* step_ch.c:726-798 (N3 > 2), with the phi self-exchanges it makes */
static void flux_ct_3d(ora_state *s)
{
  double *F1 = s->F1, *F2 = s->F2, *F3 = s->F3, *e1 = s->e1, *e2 = s->e2, *e3 = s->e3;
  copy_plane(s, F1, NPR, s->hstart - 1, s->hstop);
  copy_plane(s, F2, NPR, s->hstart - 1, s->hstop);
  ZSLOOP(s, 0, 0, 0, 1, 0, 1) {
    E(e1, h, i, j) = 0.25 * ((PV(s, F2, h, i, j)[B3] + PV(s, F2, h - 1, i, j)[B3])
                             - (PV(s, F3, h, i, j)[B2] + PV(s, F3, h, i, j - 1)[B2]));
    E(e2, h, i, j) = 0.25 * ((PV(s, F3, h, i, j)[B1] + PV(s, F3, h, i - 1, j)[B1])
                             - (PV(s, F1, h, i, j)[B3] + PV(s, F1, h - 1, i, j)[B3]));
    E(e3, h, i, j) = 0.25 * ((PV(s, F1, h, i, j)[B2] + PV(s, F1, h, i, j - 1)[B2])
                             - (PV(s, F2, h, i, j)[B1] + PV(s, F2, h, i - 1, j)[B1]));
  }
  copy_plane(s, e1, 1, s->hstop + 1, s->hstart);
  copy_plane(s, e2, 1, s->hstop + 1, s->hstart);
  ZSLOOP(s, 0, 0, 0, 1, 0, 0) {
    PV(s, F1, h, i, j)[B1] = 0.;
    PV(s, F1, h, i, j)[B2] = 0.5 * (E(e3, h, i, j) + E(e3, h, i, j + 1));
    PV(s, F1, h, i, j)[B3] = -0.5 * (E(e2, h, i, j) + E(e2, h + 1, i, j));
  }
  ZSLOOP(s, 0, 0, 0, 0, 0, 1) {
    PV(s, F2, h, i, j)[B1] = -0.5 * (E(e3, h, i, j) + E(e3, h, i + 1, j));
    PV(s, F2, h, i, j)[B2] = 0.;
    PV(s, F2, h, i, j)[B3] = 0.5 * (E(e1, h, i, j) + E(e1, h + 1, i, j));
  }
  ZSLOOP(s, 0, 0, 0, 0, 0, 0) {
    PV(s, F3, h, i, j)[B1] = 0.5 * (E(e2, h, i, j) + E(e2, h, i + 1, j));
    PV(s, F3, h, i, j)[B2] = -0.5 * (E(e1, h, i, j) + E(e1, h, i, j + 1));
    PV(s, F3, h, i, j)[B3] = 0.;
  }
}

/* diag.c:437-465 */
static void diag_flux(ora_state *s)
{
  double dx2 = s->prm.dx[2], dx3 = s->prm.dx[3];
  s->d.mdot = s->d.edot = s->d.ldot = 0.;
  s->d.mdot_in = s->d.mdot_out = 0.;
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart; j <= s->jstop; j++) {
      const double *F = PV(s, s->F1, h, s->istart, j);
      s->d.mdot += F[RHO] * dx2 * dx3;
      s->d.edot -= (F[UU] - F[RHO]) * dx2 * dx3;
      s->d.ldot += F[U3] * dx2 * dx3;
    }
}

/* diag.c:477-580 with MDOTTYPE NEU_AGA_GHOST1 */
static void diag_mass(ora_state *s, double Dt)
{
  double dx1 = s->prm.dx[1], dx2 = s->prm.dx[2], dx3 = s->prm.dx[3];
  geom_t g;
  double ucon[NDIM];
  s->d.mass_curr = 0.;
  s->d.mdot_in = s->d.mdot_out = 0.;
  ZLOOP(s) {
    double gd = s->gdet[((size_t)i * s->sn2 + j) * NPG + CENT];
    s->d.mass_curr += PV(s, s->p, h, i, j)[RHO] * gd * dx1 * dx2 * dx3;
  }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart; j <= s->jstop; j++) {
      int i = s->istart - 1;
      get_geometry(s, h, i, j, CENT, &g);
      ucon_calc(s, PV(s, s->p, h, i, j), &g, ucon);
      s->d.mdot_in += PV(s, s->p, h, i, j)[RHO] * ucon[1] * g.g * dx2 * dx3;
    }
  for (int h = HLO(s, 0); h <= HHI(s, 0); h++)
    for (int j = s->jstart; j <= s->jstop; j++) {
      int i = s->istop + 1;
      get_geometry(s, h, i, j, CENT, &g);
      ucon_calc(s, PV(s, s->p, h, i, j), &g, ucon);
      s->d.mdot_out -= PV(s, s->p, h, i, j)[RHO] * ucon[1] * g.g * dx2 * dx3;
    }
  s->d.mass_in += s->d.mdot_in * Dt;
  s->d.mass_out += s->d.mdot_out * Dt;
}

/* step_ch.c:153-318 */
double ora_advance(ora_state *s, double *pi, double *pb, double Dt, double *pf, int fullstep)
{
  double gam = s->prm.gam;
  int n3 = s->prm.n3;
  double ndt1, ndt2, ndt3 = 0.;
  if (pf != pi) ZLOOP(s) memcpy(PV(s, pf, h, i, j), PV(s, pi, h, i, j), NPR * sizeof(double));
  if (n3 > 2) {
    copy_plane(s, pb, NPR, s->hstart - 1, s->hstop);
    copy_plane(s, pb, NPR, s->hstop + 1, s->hstart);
  }
  ndt1 = fluxcalc(s, pb, s->F1, 1, fullstep);
  ndt2 = fluxcalc(s, pb, s->F2, 2, fullstep);
  if (n3 > 2) ndt3 = fluxcalc(s, pb, s->F3, 3, fullstep);
  fix_flux(s);
  if (n3 > 2) flux_ct_3d(s); else flux_ct_2d(s);
  if (fullstep) diag_flux(s);
  if (n3 > 1) copy_plane(s, s->F3, NPR, s->hstop + 1, s->hstart);

  double dx1 = s->prm.dx[1], dx2 = s->prm.dx[2], dx3 = s->prm.dx[3];
  ZLOOP(s) {
    geom_t g;
    double U[NPR], dU[NPR];
    state_t q;
    get_geometry(s, h, i, j, CENT, &g);
    const double *conn = s->conn + ((size_t)i * s->sn2 + j) * 64;
    source(s, gam, PV(s, pb, h, i, j), &g, conn, dU);
    get_state(s, PV(s, pi, h, i, j), &g, &q);
    primtoflux(gam, PV(s, pi, h, i, j), &q, 0, &g, U);
    for (int k = 0; k < NPR; k++) {
      double a1 = PV(s, s->F1, h, i + 1, j)[k] - PV(s, s->F1, h, i, j)[k];
      double a2 = PV(s, s->F2, h, i, j + 1)[k] - PV(s, s->F2, h, i, j)[k];
      if (n3 > 2) {
        double a3 = PV(s, s->F3, h + 1, i, j)[k] - PV(s, s->F3, h, i, j)[k];
        U[k] += Dt * (-(a1) / dx1 - (a2) / dx2 - (a3) / dx3 + dU[k]);
      } else {
        U[k] += Dt * (-(a1) / dx1 - (a2) / dx2 + dU[k]);
      }
    }
    double *pz = PV(s, pf, h, i, j);
    signed char *fl = &s->pflag[zidx(s, h, i, j)];
    *fl = (signed char)ora_utoprim_2d(gam, U, &g.gcov[0][0], &g.gcon[0][0], g.g, pz);
    if (*fl) {
      double kappa = s->katm[i];
      *fl = (signed char)ora_utoprim_1dvsq2fix1(gam, U, &g.gcov[0][0], &g.gcon[0][0], g.g, pz, kappa);
      if (!*fl) ora_counts[1]++;
      else {
        *fl = (signed char)ora_utoprim_1dfix1(gam, U, &g.gcov[0][0], &g.gcon[0][0], g.g, pz, kappa);
        if (!*fl) ora_counts[2]++;
      }
    }
  }
  if (n3 > 2) return s->prm.defcon * 1. / (1. / ndt1 + 1. / ndt2 + 1. / ndt3);
  return s->prm.defcon * 1. / (1. / ndt1 + 1. / ndt2);
}

/* step_ch.c:90-140 */
/* ------------------------------------------------------------------ */
/* tracer particles (tracers.c)                                         */

/* coord() (metric.c:62-115) for the CENT and FACE3 locations, single rank */
static void coord_x(const ora_state *s, int h, int i, int j, int loc, double *X)
{
  i -= 2;
  j -= 2;
  h -= s->prm.n3 > 1 ? 1 : 0;
  X[0] = 1.;
  X[1] = s->prm.startx[1] + (i + 0.5) * s->prm.dx[1];
  X[2] = s->prm.startx[2] + (j + 0.5) * s->prm.dx[2];
  if (loc == FACE3 || s->prm.n3 <= 2) X[3] = s->prm.startx[3] + h * s->prm.dx[3];
  else X[3] = s->prm.startx[3] + (h + 0.5) * s->prm.dx[3];
}

/* search_tracer() (tracers.c:39-98): the zone below the tracer along each axis */
static int search_tracer(const ora_state *s, const double *XX, int *hh, int *ii, int *jj)
{
  double Xl[4], Xr[4];
  int ok;
  coord_x(s, s->hstart, s->istart - 1, s->jstart - 1, CENT, Xl);
  if (XX[1] < Xl[1] || XX[2] < Xl[2]) return 0;
  *hh = 0;
  ok = 0;
  for (int i = s->istart - 1; i <= s->istop; i++) {
    coord_x(s, s->hstart, i, s->jstart, CENT, Xl);
    coord_x(s, s->hstart, i + 1, s->jstart, CENT, Xr);
    if (XX[1] >= Xl[1] && XX[1] < Xr[1]) { *ii = i; ok = 1; break; }
  }
  if (!ok) return 0;
  ok = 0;
  for (int j = s->jstart - 1; j <= s->jstop; j++) {
    coord_x(s, s->hstart, s->istart, j, CENT, Xl);
    coord_x(s, s->hstart, s->istart, j + 1, CENT, Xr);
    if (XX[2] >= Xl[2] && XX[2] < Xr[2]) { *jj = j; ok = 1; break; }
  }
  if (!ok) return 0;
  if (s->prm.n3 > 2) {
    ok = 0;
    for (int h = s->hstart; h <= s->hstop; h++) {
      coord_x(s, h, s->istart, s->jstart, FACE3, Xl);
      coord_x(s, h + 1, s->istart, s->jstart, FACE3, Xr);
      if (XX[3] >= Xl[3] && XX[3] < Xr[3]) { *hh = h; ok = 1; break; }
    }
    if (!ok) return 0;
  }
  return 1;
}

/* ucon_fun() (tracers.c:257-269): u^mu with the spatial parts divided by u^t */
static void ucon_fun(ora_state *s, int h, int i, int j, double *ucon)
{
  geom_t g;
  get_geometry(s, h, i, j, CENT, &g);
  ucon_calc(s, PV(s, s->p, h, i, j), &g, ucon);
  ucon[1] /= ucon[0];
  ucon[2] /= ucon[0];
  ucon[3] /= ucon[0];
}

/* linear_interpolation() (tracers.c:193-254) of ucon_fun, VALDIM = 4 */
static void interp_ucon(ora_state *s, const double *tX, int hh, int ii, int jj, double *val)
{
  const int WPH = s->prm.n3 > 2 ? 2 : 1;
  double XX[2][2][2][4], valt[2][2][2][4], tmp1[2][2][4], tmp2[2][4];
  for (int l3 = 0; l3 < WPH; l3++)
    for (int l1 = 0; l1 < 2; l1++)
      for (int l2 = 0; l2 < 2; l2++) {
        coord_x(s, hh + l3, ii + l1, jj + l2, CENT, XX[l3][l1][l2]);
        ucon_fun(s, hh + l3, ii + l1, jj + l2, valt[l3][l1][l2]);
      }
  for (int l3 = 0; l3 < WPH; l3++)
    for (int l1 = 0; l1 < 2; l1++) {
      double T1 = 1.0 / (XX[l3][l1][1][2] - XX[l3][l1][0][2]);
      double T2 = tX[2] - XX[l3][l1][0][2];
      for (int k = 0; k < 4; k++) {
        double ypval = (valt[l3][l1][1][k] - valt[l3][l1][0][k]) * T1;
        tmp1[l3][l1][k] = valt[l3][l1][0][k] + T2 * ypval;
      }
    }
  for (int l3 = 0; l3 < WPH; l3++) {
    double T1 = 1.0 / (XX[l3][1][1][1] - XX[l3][0][0][1]);
    double T2 = tX[1] - XX[l3][0][0][1];
    for (int k = 0; k < 4; k++) {
      double ypval = (tmp1[l3][1][k] - tmp1[l3][0][k]) * T1;
      tmp2[l3][k] = tmp1[l3][0][k] + T2 * ypval;
    }
  }
  if (WPH == 1) {
    for (int k = 0; k < 4; k++) val[k] = tmp2[0][k];
  } else {
    double T1 = 1.0 / (XX[1][1][1][3] - XX[0][0][0][3]);
    double T2 = tX[3] - XX[0][0][0][3];
    for (int k = 0; k < 4; k++) {
      double ypval = (tmp2[1][k] - tmp2[0][k]) * T1;
      val[k] = tmp2[0][k] + T2 * ypval;
    }
  }
}

/* bl_coord() (coord.c:61-124) with gammie_coords, Rbr < 0, COORDSINGFIX */
static void bl_coord_rth(const ora_state *s, const double *X, double *r, double *th)
{
  *r = exp(X[1]) + s->R0;
  double t = M_PI_2 * (1. + X[2]) + ((1. - s->hslope) / 2.) * sin(M_PI * (1. + X[2]));
  if (fabs(t) < 1.E-20) t = t >= 0 ? 1.E-20 : -1.E-20;
  if (fabs(M_PI - t) < 1.E-20) t = t >= M_PI ? M_PI + 1.E-20 : M_PI - 1.E-20;
  *th = t;
}

/* update_tracers() (tracers.c:298-429), one rank: move each active tracer by
   the interpolated u^i/u^t over Dt, then retire those that fell in or left */
static void update_tracers(ora_state *s, double Dt)
{
  const double Rin = exp(s->prm.startx[1] - 0.5 * s->prm.dx[1]) + s->R0;           /* :121 */
  const double Rout = 0.8 * (exp(s->prm.startx[1] + s->prm.n1 * s->prm.dx[1]) + s->R0);
  const double thmin = 0.02 * M_PI, thmax = 0.98 * M_PI;
  /* the phi-periodic ghost plane the interpolation reads (tracers.c:313-318) */
  if (s->prm.n3 > 2)
    memcpy(PV(s, s->p, s->hstop + 1, 0, 0), PV(s, s->p, s->hstart, 0, 0),
           (size_t)s->sn1 * s->sn2 * NPR * sizeof(double));
  for (long k = 0; k < s->ntr; k++) {
    if (s->tr_st[k]) continue;
    double X[4] = {0., s->tr_X[3 * k], s->tr_X[3 * k + 1], s->tr_X[3 * k + 2]};
    int hh, ii, jj;
    if (!search_tracer(s, X, &hh, &ii, &jj)) { s->tr_st[k] = -1; continue; }
    double ucon[4];
    interp_ucon(s, X, hh, ii, jj, ucon);
    for (int m = 1; m < 4; m++) X[m] += ucon[m] * Dt;
    double r, th;
    bl_coord_rth(s, X, &r, &th);
    for (int m = 1; m < 4; m++) s->tr_X[3 * k + m - 1] = X[m];
    if (r < Rin || th < 0 || th > M_PI) s->tr_st[k] = 1;
    else if (r >= Rout) s->tr_st[k] = (th >= thmin && th <= thmax) ? 2 : 3;
  }
  if (s->prm.n3 > 2)  /* tracers.c:385-408: back into [0, 2 pi] */
    for (long k = 0; k < s->ntr; k++) {
      if (s->tr_st[k]) continue;
      double *x3 = &s->tr_X[3 * k + 2];
      if (*x3 < 0.) *x3 += 2. * M_PI;
      else if (*x3 > 2. * M_PI) *x3 -= 2. * M_PI;
    }
}

static void tracers_alloc(ora_state *s, long n)
{
  free(s->tr_ids); free(s->tr_X); free(s->tr_st);
  s->ntr = n;
  s->tr_ids = (int *)calloc(3 * (size_t)(n ? n : 1), sizeof(int));
  s->tr_X = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
  s->tr_st = (signed char *)calloc((size_t)(n ? n : 1), 1);
}

void ora_tracers_geometry(ora_state *s, double R0, double hslope)
{
  s->R0 = R0;
  s->hslope = hslope;
}

/* init_tracers() (tracers.c:109-188): one tracer per zone centre whose zone
   (found by the search) has rho > RHOMIN, in h, i, j loop order */
long ora_tracers_init(ora_state *s)
{
  const int n1 = s->prm.n1, n2 = s->prm.n2, n3 = s->prm.n3;
  long cnt = 0;
  int *ids = (int *)malloc(3 * sizeof(int) * (size_t)n1 * n2 * n3);
  double *X = (double *)malloc(3 * sizeof(double) * (size_t)n1 * n2 * n3);
  for (int h = 0; h < n3; h++)
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n2; j++) {
        double tX[4] = {0., s->prm.startx[1] + (i + 0.5) * s->prm.dx[1],
                        s->prm.startx[2] + (j + 0.5) * s->prm.dx[2], s->prm.startx[3] + h * s->prm.dx[3]};
        int hh, ii, jj;
        if (search_tracer(s, tX, &hh, &ii, &jj) && PV(s, s->p, hh, ii, jj)[RHO] > RHOMIN) {
          ids[3 * cnt] = i; ids[3 * cnt + 1] = j; ids[3 * cnt + 2] = h;
          X[3 * cnt] = tX[1]; X[3 * cnt + 1] = tX[2]; X[3 * cnt + 2] = tX[3];
          cnt++;
        }
      }
  ora_tracers_put(s, ids, X, cnt);
  free(ids);
  free(X);
  return cnt;
}

void ora_tracers_put(ora_state *s, const int *ids, const double *X, long n)
{
  tracers_alloc(s, n);
  memcpy(s->tr_ids, ids, 3 * sizeof(int) * (size_t)n);
  memcpy(s->tr_X, X, 3 * sizeof(double) * (size_t)n);
}

long ora_tracers_count(const ora_state *s) { return s->ntr; }

void ora_tracers_get(const ora_state *s, int *ids, double *X, signed char *status)
{
  memcpy(ids, s->tr_ids, 3 * sizeof(int) * (size_t)s->ntr);
  memcpy(X, s->tr_X, 3 * sizeof(double) * (size_t)s->ntr);
  memcpy(status, s->tr_st, (size_t)s->ntr);
}

/* ------------------------------------------------------------------ */
/* diag() integrals and the divergence of B (diag.c:113-230)            */

void ora_diag_integrals(ora_state *s, double *out4, int *imax)
{
  const double dx1 = s->prm.dx[1], dx2 = s->prm.dx[2], dx3 = s->prm.dx[3];
  const double dV = dx1 * dx2 * dx3;  /* main.c:427 */
  double pp = 0., e = 0., rmed = 0., divbmax = 0.;
  imax[0] = imax[1] = imax[2] = 0;
  /* the phi ghost plane below the first one (diag.c:121-129: plane hstop -> plane 0) */
  if (s->prm.n3 > 2)
    memcpy(PV(s, s->p, 0, 0, 0), PV(s, s->p, s->hstop, 0, 0), (size_t)s->sn1 * s->sn2 * NPR * sizeof(double));
  for (int h = s->hstart; h <= s->hstop; h++)
    for (int i = s->istart; i <= s->istop; i++)
      for (int j = s->jstart; j <= s->jstop; j++) {
        geom_t g;
        state_t q;
        double U[NPR], divb;
        get_geometry(s, h, i, j, CENT, &g);
        get_state(s, PV(s, s->p, h, i, j), &g, &q);
        primtoflux(s->prm.gam, PV(s, s->p, h, i, j), &q, 0, &g, U);
        rmed += U[RHO] * dV;
        pp += U[U3] * dV;
        e += U[UU] * dV;
#define P_(hh, ii, jj, k) PV(s, s->p, hh, ii, jj)[k]
#define G_(ii, jj) s->gdet[((size_t)(ii) * s->sn2 + (jj)) * NPG + CENT]
        if (s->prm.n3 > 2) {
          divb = fabs(0.25 * (P_(h, i, j, B1) * G_(i, j) + P_(h - 1, i, j, B1) * G_(i, j)
                              + P_(h, i, j - 1, B1) * G_(i, j - 1) + P_(h - 1, i, j - 1, B1) * G_(i, j - 1)
                              - P_(h, i - 1, j, B1) * G_(i - 1, j) - P_(h - 1, i - 1, j, B1) * G_(i - 1, j)
                              - P_(h, i - 1, j - 1, B1) * G_(i - 1, j - 1)
                              - P_(h - 1, i - 1, j - 1, B1) * G_(i - 1, j - 1)) / dx1
                      + 0.25 * (P_(h, i, j, B2) * G_(i, j) + P_(h - 1, i, j, B2) * G_(i, j)
                                + P_(h, i - 1, j, B2) * G_(i - 1, j) + P_(h - 1, i - 1, j, B2) * G_(i - 1, j)
                                - P_(h, i, j - 1, B2) * G_(i, j - 1) - P_(h - 1, i, j - 1, B2) * G_(i, j - 1)
                                - P_(h, i - 1, j - 1, B2) * G_(i - 1, j - 1)
                                - P_(h - 1, i - 1, j - 1, B2) * G_(i - 1, j - 1)) / dx2
                      + 0.25 * (P_(h, i, j, B3) * G_(i, j) + P_(h, i - 1, j, B3) * G_(i - 1, j)
                                + P_(h, i, j - 1, B3) * G_(i, j - 1) + P_(h, i - 1, j - 1, B3) * G_(i - 1, j - 1)
                                - P_(h - 1, i, j, B3) * G_(i, j) - P_(h - 1, i - 1, j, B3) * G_(i - 1, j)
                                - P_(h - 1, i, j - 1, B3) * G_(i, j - 1)
                                - P_(h - 1, i - 1, j - 1, B3) * G_(i - 1, j - 1)) / dx3);
        } else {
          divb = fabs(0.5 * (P_(h, i, j, B1) * G_(i, j) + P_(h, i, j - 1, B1) * G_(i, j - 1)
                             - P_(h, i - 1, j, B1) * G_(i - 1, j) - P_(h, i - 1, j - 1, B1) * G_(i - 1, j - 1)) / dx1
                      + 0.5 * (P_(h, i, j, B2) * G_(i, j) + P_(h, i - 1, j, B2) * G_(i - 1, j)
                               - P_(h, i, j - 1, B2) * G_(i, j - 1) - P_(h, i - 1, j - 1, B2) * G_(i - 1, j - 1)) / dx2);
        }
#undef P_
#undef G_
        if (divb > divbmax) {
          imax[0] = i - 2;
          imax[1] = j - 2;
          imax[2] = s->prm.n3 == 1 ? 0 : h - 1;
          divbmax = divb;
        }
      }
  out4[0] = rmed;
  out4[1] = pp;
  out4[2] = e;
  out4[3] = divbmax;
}

int ora_step_ch(ora_state *s)
{
  double ndt;
  ora_advance(s, s->p, s->p, 0.5 * s->dt, s->ph, 0);
  ora_fixup(s, s->ph);
  ora_bound_prim(s, s->ph);
  ora_fixup_utoprim(s, s->ph);
  ora_bound_prim(s, s->ph);
  ndt = ora_advance(s, s->p, s->ph, s->dt, s->p, 1);
  ora_fixup(s, s->p);
  ora_bound_prim(s, s->p);
  ora_fixup_utoprim(s, s->p);
  ora_bound_prim(s, s->p);
  diag_mass(s, s->dt);
  if (s->ntr) update_tracers(s, s->dt);  /* step_ch.c:121-123 */
  s->d.ndt = ndt;
  if (s->dt < 1.e-9) return 11;
  s->t += s->dt;
  if (ndt > SAFE * s->dt) ndt = SAFE * s->dt;
  s->dt = ndt;
  if (s->t + s->dt > s->prm.tf) s->dt = s->prm.tf - s->t;
  return 0;
}

/* ------------------------------------------------------------------ */
/* state management                                                    */

ora_state *ora_create(const ora_params *prm, const double *gcov, const double *gcon,
                      const double *gdet, const double *conn, const double *coords,
                      const double *katm)
{
  if (prm->n1 < 4 || prm->n2 < 8 || prm->n3 < 1 || (prm->n3 > 1 && (prm->n3 % 2 || prm->n3 < 4)))
    return NULL;
  ora_state *s = (ora_state *)calloc(1, sizeof(ora_state));
  s->prm = *prm;
  s->sn1 = prm->n1 + 4;
  s->sn2 = prm->n2 + 4;
  s->sn3 = prm->n3 > 1 ? prm->n3 + 2 : 1;
  s->istart = 2; s->istop = prm->n1 + 1;
  s->jstart = 2; s->jstop = prm->n2 + 1;
  s->hstart = prm->n3 > 1 ? 1 : 0; s->hstop = prm->n3 > 1 ? prm->n3 : 0;
  size_t nz = (size_t)s->sn3 * s->sn1 * s->sn2, ng = (size_t)s->sn1 * s->sn2;
  s->p = (double *)calloc(nz * NPR, sizeof(double));
  s->ph = (double *)calloc(nz * NPR, sizeof(double));
  s->dq = (double *)calloc(nz * NPR, sizeof(double));
  s->F1 = (double *)calloc(nz * NPR, sizeof(double));
  s->F2 = (double *)calloc(nz * NPR, sizeof(double));
  s->F3 = (double *)calloc(nz * NPR, sizeof(double));
  s->e1 = (double *)calloc(nz, sizeof(double));
  s->e2 = (double *)calloc(nz, sizeof(double));
  s->e3 = (double *)calloc(nz, sizeof(double));
  s->pflag = (signed char *)calloc(nz, 1);
  s->gcov = (double *)malloc(ng * NPG * 16 * sizeof(double));
  s->gcon = (double *)malloc(ng * NPG * 16 * sizeof(double));
  s->gdet = (double *)malloc(ng * NPG * sizeof(double));
  s->conn = (double *)malloc(ng * 64 * sizeof(double));
  s->coords = (double *)malloc(ng * 4 * sizeof(double));
  s->katm = (double *)malloc(s->sn1 * sizeof(double));
  memcpy(s->gcov, gcov, ng * NPG * 16 * sizeof(double));
  memcpy(s->gcon, gcon, ng * NPG * 16 * sizeof(double));
  memcpy(s->gdet, gdet, ng * NPG * sizeof(double));
  memcpy(s->conn, conn, ng * 64 * sizeof(double));
  memcpy(s->coords, coords, ng * 4 * sizeof(double));
  memcpy(s->katm, katm, s->sn1 * sizeof(double));
  return s;
}

void ora_destroy(ora_state *s)
{
  if (!s) return;
  free(s->p); free(s->ph); free(s->dq); free(s->F1); free(s->F2); free(s->F3);
  free(s->e1); free(s->e2); free(s->e3); free(s->pflag);
  free(s->gcov); free(s->gcon); free(s->gdet); free(s->conn); free(s->coords); free(s->katm);
  free(s->tr_ids); free(s->tr_X); free(s->tr_st);
  free(s);
}

double *ora_p(ora_state *s) { return s->p; }
double *ora_ph(ora_state *s) { return s->ph; }
signed char *ora_pflag(ora_state *s) { return s->pflag; }
double *ora_flux(ora_state *s, int dir) { return dir == 1 ? s->F1 : dir == 2 ? s->F2 : s->F3; }
void ora_set_time(ora_state *s, double t, double dt) { s->t = t; s->dt = dt; }
void ora_get_time(const ora_state *s, double *t, double *dt) { *t = s->t; *dt = s->dt; }
void ora_set_mass(ora_state *s, double mass_in, double mass_out) { s->d.mass_in = mass_in; s->d.mass_out = mass_out; }
void ora_get_diag(const ora_state *s, ora_diag *d) { *d = s->d; }
