// Device physics of the HARM-COOL zone update, one zone (or face) per thread.
//
// Every routine keeps the reference's floating-point expression order, and
// the library is built with -fmad=false, so with the IEEE division and
// square root of sm_100 the FP64 results reproduce the reference's SSE2
// results bit for bit.  Two things differ by construction:
//  * metric entries that are structurally zero in modified Kerr-Schild
//    coordinates (g_{t theta}, g_{r theta}, g_{theta phi} and their inverse
//    counterparts) are not stored, so the x*0 terms the reference adds are
//    skipped -- this can only change the sign of an exactly-zero result;
//  * the isentropic fall-back inversions raise densities to the adiabatic
//    index with pow_cr (harm_pow.cuh), the correctly rounded power, where the
//    reference calls the host libm's pow(), correctly rounded in all but rare
//    cases.
#pragma once
#include <cstdint>

#include "harm_pow.cuh"

namespace harm {

enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4, B1 = 5, B2 = 6, B3 = 7 };

// decs.h:127-158, u2p_defs.h:79-99
constexpr double RHOMIN = 1.e-6, UUMIN = 1.e-8;
constexpr double BSQORHOMAX = 50., BSQOUMAX = 2500., UORHOMAX = 50.;
constexpr double SMALL = 1.e-20, GAMMAMAX = 50., SAFE = 1.3;
constexpr int MAX_NEWT_ITER = 30, EXTRA_NEWT_ITER = 2;
constexpr double NEWT_TOL = 1.0e-10, MIN_NEWT_TOL = 1.0e-10, NEWT_TOL2 = 1.0e-15;
constexpr double W_TOO_BIG = 1.e20, UTSQ_TOO_BIG = 1.e20, FAIL_VAL = 1.e30;

// failure codes (decs.h:232-238)
enum { FAIL_VCHAR_DISCR = 2, FAIL_COEFF_NEG = 3, FAIL_COEFF_SUP = 4, FAIL_GAMMA = 5 };

// Non-zero metric entries at one location: gcov is symmetric, gcon is not
// bit-symmetric (it comes from an LU inverse), both vanish in the
// (t,theta), (r,theta), (theta,phi) slots.
struct Geo {
  double v00, v01, v03, v11, v13, v22, v33;                      // gcov
  double n00, n01, n03, n10, n11, n13, n22, n30, n31, n33;       // gcon
  double g;                                                      // sqrt(-det g)
  double alpha;  // 1/sqrt(-g^tt), as ucon_calc and the inversion form it (phys.c:238)
  double ialpha; // 1/alpha rounded to nearest: the divisor of div_rn for alpha
  double ig;     // 1/g rounded to nearest (zone centres; where g = 0 it is not used)
};
constexpr int GEO_N = 21;

// ---------------------------------------------------------------------------
// Division by a divisor that many divisions share.
//
// The step divides by the same few numbers again and again: the lapse alpha
// (ucon_calc), sqrt(-g) (the inversion's rescaling), the cell widths (the flux
// divergence), the adiabatic index (the Noble pressure), u^t (bcon_calc).  An
// IEEE double division costs about 14 FP64 issue slots on sm_100; with
// y = 1/b rounded to nearest formed once, div_rn returns the same correctly
// rounded quotient in 6:
//  * q = a y is within two ulps of a/b, and one FMA correction
//    q + (a - b q) y (Markstein, IBM J. Res. Dev. 34:111-119, 1990) brings it
//    within one ulp: q is then a faithful quotient;
//  * for a faithful q the remainder r = a - b q is a double, so fma(-q, b, a)
//    forms it exactly (Boldo and Daumas, ARITH-16, 2003);
//  * a/b = q + r/b, so q is the nearest double to a/b exactly when |r| is
//    below b times half the gap between q and its neighbour on the side of a/b
//    (a power of two, so that product is exact); otherwise the neighbour is.
//    a/b is never halfway between two doubles, so there is no tie.
// y must be RN(1/b).  Divisors other than b > 0 in [2^-60, 2^61), and
// numerators outside [2^-800, 2^800] in magnitude (subnormal, huge, inf, NaN),
// take the IEEE division; a zero numerator gives a y, the signed zero a/b is.
__device__ __forceinline__ double div_rn(double a, double b, double y)
{
#if HARM_STEP_MIXED
  // the mixed-precision step: the reciprocal multiply, within an ulp of a/b
  // (that step answers for its L1 accuracy against the FP64 step, not for bits)
  return a * y;
#endif
  const long long ia = __double_as_longlong(a);
  const unsigned ea = (unsigned)(ia >> 52) & 0x7ffu;
  const unsigned eb = (unsigned)(__double_as_longlong(b) >> 52) & 0xfffu;  // sign bit included
  const bool okb = eb - 963u <= 120u;                                      // b > 0, 2^-60 <= b < 2^61
  if (!okb || ea - 223u > 1600u) return (okb && (ia << 1) == 0) ? a * y : a / b;
  double q = a * y;
  double r = fma(-q, b, a);
  q = fma(r, y, q);
  r = fma(-q, b, a);
  long long iq = __double_as_longlong(q);
  const bool up = (r > 0.) == (q > 0.);                     // |a/b| > |q|
  const int eq = (int)((iq >> 52) & 0x7ff);
  // half the gap to the neighbour towards a/b: a quarter ulp below a power of two
  const int eh = eq - 53 - ((!up && (iq & 0xfffffffffffffLL) == 0) ? 1 : 0);
  const double hb = __longlong_as_double((long long)eh << 52) * b;
  if (fabs(r) > hb) {
    iq += up ? 1 : -1;
    q = __longlong_as_double(iq);
  }
  return q;
}

// div_rn for a divisor formed at run time: its reciprocal is one IEEE division,
// worth it from two quotients on; divisors outside [2^-60, 2^60] divide directly
__device__ __forceinline__ bool div_rn_ok(double b)
{
  const unsigned eb = (unsigned)(__double_as_longlong(b) >> 52) & 0xfffu;  // sign bit included
  return eb - 963u <= 120u;                                                 // b > 0, 2^-60 <= b < 2^61
}

// a/b for the step's scalar type: div_rn for double, plain division for the
// adjoint's dual numbers (whose value part is the same correctly rounded quotient)
template <class R>
__device__ __forceinline__ R div_by(const R &a, double b, double y)
{
  return a / b;
}
template <>
__device__ __forceinline__ double div_by<double>(const double &a, double b, double y)
{
  return div_rn(a, b, y);
}

// geometry planes: [GEO_N][ng], entry e of point gi at G[e*ng + gi]
__device__ __forceinline__ void load_geo(const double *__restrict__ G, long ng, long gi, Geo &q)
{
  q.v00 = __ldg(G + 0 * ng + gi); q.v01 = __ldg(G + 1 * ng + gi); q.v03 = __ldg(G + 2 * ng + gi);
  q.v11 = __ldg(G + 3 * ng + gi); q.v13 = __ldg(G + 4 * ng + gi); q.v22 = __ldg(G + 5 * ng + gi);
  q.v33 = __ldg(G + 6 * ng + gi);
  q.n00 = __ldg(G + 7 * ng + gi); q.n01 = __ldg(G + 8 * ng + gi); q.n03 = __ldg(G + 9 * ng + gi);
  q.n10 = __ldg(G + 10 * ng + gi); q.n11 = __ldg(G + 11 * ng + gi); q.n13 = __ldg(G + 12 * ng + gi);
  q.n22 = __ldg(G + 13 * ng + gi); q.n30 = __ldg(G + 14 * ng + gi); q.n31 = __ldg(G + 15 * ng + gi);
  q.n33 = __ldg(G + 16 * ng + gi); q.g = __ldg(G + 17 * ng + gi);
  q.alpha = __ldg(G + 18 * ng + gi);
  q.ialpha = __ldg(G + 19 * ng + gi);
  q.ig = __ldg(G + 20 * ng + gi);
}

// The routines below that the discrete adjoint linearises are templates on
// the scalar type R: double for the step itself, a forward-mode dual number
// (harm_dual.cuh) for the adjoint's local Jacobians.  The double
// instantiation is the reference's expression order unchanged.
template <class R>
struct StateT {
  R ucon[4], ucov[4], bcon[4], bcov[4];
};
using State = StateT<double>;

// lower() (metric.c:210-231)
template <class R>
__device__ __forceinline__ void lower(const R *u, const Geo &q, R *d)
{
  d[0] = q.v00 * u[0] + q.v01 * u[1] + q.v03 * u[3];
  d[1] = q.v01 * u[0] + q.v11 * u[1] + q.v13 * u[3];
  d[2] = q.v22 * u[2];
  d[3] = q.v03 * u[0] + q.v13 * u[1] + q.v33 * u[3];
}

template <class R>
__device__ __forceinline__ R dot4(const R *a, const R *b)
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

// gamma_calc() (phys.c:300-324); returns 1 on failure
template <class R>
__device__ __forceinline__ int gamma_calc(const R *pr, const Geo &q, R &gamma)
{
  R qsq = q.v11 * pr[U1] * pr[U1] + q.v22 * pr[U2] * pr[U2] + q.v33 * pr[U3] * pr[U3]
               + 2. * (q.v13 * pr[U1] * pr[U3]);
  if (qsq < 0.) {
    if (fabs(qsq) > 1.E-10) { gamma = 1.; return 1; }
    qsq = 1.E-10;
  }
  gamma = sqrt(1. + qsq);
  return 0;
}

// ucon_calc() (phys.c:232-252); sets *fail on a gamma failure
template <class R>
__device__ __forceinline__ void ucon_calc(const R *pr, const Geo &q, R *ucon, int *fail)
{
  const double alpha = q.alpha;
  double b1 = q.n01 * alpha * alpha, b3 = q.n03 * alpha * alpha;
  R gamma;
  if (gamma_calc(pr, q, gamma)) *fail = FAIL_GAMMA;
  ucon[0] = div_by(gamma, alpha, q.ialpha);
  ucon[1] = pr[U1] - div_by(gamma * b1, alpha, q.ialpha);
  // the reference's pr[U2] - gamma * b2 / alpha with b2 = g^{t theta} alpha^2 = 0*alpha*alpha:
  // gamma * (+0) / alpha is +0 for finite gamma and NaN otherwise, and so is
  // gamma - gamma, which takes two operations instead of a division
  ucon[2] = pr[U2] - (gamma - gamma);
  ucon[3] = pr[U3] - div_by(gamma * b3, alpha, q.ialpha);
}

// bcon_calc() (phys.c:108-117)
template <class R>
__device__ __forceinline__ void bcon_calc(const R *pr, const R *ucon, const R *ucov, R *bcon)
{
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  bcon[1] = (pr[B1] + bcon[0] * ucon[1]) / ucon[0];
  bcon[2] = (pr[B2] + bcon[0] * ucon[2]) / ucon[0];
  bcon[3] = (pr[B3] + bcon[0] * ucon[3]) / ucon[0];
}
// the double form: three quotients by u^t share one reciprocal
template <>
__device__ __forceinline__ void bcon_calc<double>(const double *pr, const double *ucon, const double *ucov,
                                                  double *bcon)
{
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  const double u0 = ucon[0];
  if (div_rn_ok(u0)) {
    const double y = 1. / u0;
    bcon[1] = div_rn(pr[B1] + bcon[0] * ucon[1], u0, y);
    bcon[2] = div_rn(pr[B2] + bcon[0] * ucon[2], u0, y);
    bcon[3] = div_rn(pr[B3] + bcon[0] * ucon[3], u0, y);
  } else {
    bcon[1] = (pr[B1] + bcon[0] * ucon[1]) / u0;
    bcon[2] = (pr[B2] + bcon[0] * ucon[2]) / u0;
    bcon[3] = (pr[B3] + bcon[0] * ucon[3]) / u0;
  }
}

// get_state() (phys.c:219-229)
template <class R>
__device__ __forceinline__ void get_state(const R *pr, const Geo &q, StateT<R> &s, int *fail)
{
  ucon_calc(pr, q, s.ucon, fail);
  lower(s.ucon, q, s.ucov);
  bcon_calc(pr, s.ucon, s.ucov, s.bcon);
  lower(s.bcon, q, s.bcov);
}

// mhd_calc() (phys.c:143-161): one row T^dir_nu of the stress tensor
template <class R>
__device__ __forceinline__ void mhd_calc(double gam, const R *pr, int dir, const StateT<R> &s, R *mhd)
{
  R r = pr[RHO], u = pr[UU];
  R P = (gam - 1.) * u;
  R w = P + r + u;
  R bsq = dot4(s.bcon, s.bcov);
  R eta = w + bsq;
  R ptot = P + 0.5 * bsq;
#pragma unroll
  for (int j = 0; j < 4; j++)
    mhd[j] = eta * s.ucon[dir] * s.ucov[j] + ptot * (dir == j ? 1. : 0.) - s.bcon[dir] * s.bcov[j];
}

// primtoflux() (phys.c:59-96)
template <class R>
__device__ __forceinline__ void primtoflux(double gam, const R *pr, const StateT<R> &s, int dir, double g, R *flux)
{
  R mhd[4];
  flux[RHO] = pr[RHO] * s.ucon[dir];
  mhd_calc(gam, pr, dir, s, mhd);
  flux[UU] = mhd[0] + flux[RHO];
  flux[U1] = mhd[1];
  flux[U2] = mhd[2];
  flux[U3] = mhd[3];
  flux[B1] = s.bcon[1] * s.ucon[dir] - s.bcon[dir] * s.ucon[1];
  flux[B2] = s.bcon[2] * s.ucon[dir] - s.bcon[dir] * s.ucon[2];
  flux[B3] = s.bcon[3] * s.ucon[dir] - s.bcon[dir] * s.ucon[3];
#pragma unroll
  for (int k = 0; k < 8; k++) flux[k] *= g;
}

// gcon[m][js] and gcon[0][js] for the wave-speed quadratic
__device__ __forceinline__ double gcon_diag(const Geo &q, int js)
{
  return js == 1 ? q.n11 : js == 2 ? q.n22 : q.n33;
}
__device__ __forceinline__ double gcon_t(const Geo &q, int js)
{
  return js == 1 ? q.n01 : js == 2 ? 0. : q.n03;
}

// vchar() (phys.c:337-476, gamma-law): with A = e^js and B = e^t the
// contractions reduce to metric entries: A.A = g^{js js}, B.B = g^{tt},
// A.u = u^js, B.u = u^t, A.B = g^{t js}
template <class R>
__device__ __forceinline__ void vchar(double gam, const R *pr, const StateT<R> &s, const Geo &q, int js, R &vmax,
                                      R &vmin, int *fail)
{
  R bsq = dot4(s.bcon, s.bcov);
  R rho = pr[RHO], u = pr[UU];
  R EF = rho + gam * u;
  R EE = bsq + EF;
  R va2 = bsq / EE;
  R cs2 = gam * (gam - 1.) * u / EF;
  R cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.) { *fail = FAIL_COEFF_NEG; cms2 = SMALL; }
  if (cms2 > 1.) { *fail = FAIL_COEFF_SUP; cms2 = 1.; }
  double Asq = gcon_diag(q, js), Bsq = q.n00;
  R Au = s.ucon[js], Bu = s.ucon[0];
  double AB = gcon_t(q, js);
  R Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  R A = Bu2 - (Bsq + Bu2) * cms2;
  R B = 2. * (AuBu - (AB + AuBu) * cms2);
  R C = Au2 - (Asq + Au2) * cms2;
  R discr = B * B - 4. * A * C;
  if ((discr < 0.0) && (discr > -1.e-10)) discr = 0.0;
  else if (discr < -1.e-10) { *fail = FAIL_VCHAR_DISCR; discr = 0.; }
  discr = sqrt(discr);
  R vp = -(-B + discr) / (2. * A);
  R vm = -(-B - discr) / (2. * A);
  if (vp > vm) { vmax = vp; vmin = vm; }
  else { vmax = vm; vmin = vp; }
}

// The local Lax-Friedrichs flux of one face (step_ch.c:431-473, HLLF = 0 and
// LAXF = 1 at :66-67): lf_flux combines the two sides' fluxes F^dir, conserved
// variables U and wave speeds into F and the face's wave speed ctop;
// face_side evaluates one side; face_flux is both sides and the combination.
template <class R>
__device__ __forceinline__ void lf_flux(const R *Fl, const R *Ul, const R &cmaxl, const R &cminl, const R *Fr,
                                        const R *Ur, const R &cmaxr, const R &cminr, R *F, R &ctop)
{
  R t1 = 0. > cmaxl ? R(0.) : cmaxl;
  R cmax = fabs(t1 > cmaxr ? t1 : cmaxr);
  R t2 = 0. > -cminl ? R(0.) : -cminl;
  R cmin = fabs(t2 > -cminr ? t2 : -cminr);
  ctop = cmax > cmin ? cmax : cmin;
#pragma unroll
  for (int k = 0; k < 8; k++) F[k] = 0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k]));
}

template <int DIR, class R>
__device__ __forceinline__ void face_side(double gam, const R *p, const Geo &q, R *F, R *U, R &cmax, R &cmin,
                                          int *fail)
{
  StateT<R> s;
  get_state(p, q, s, fail);
  primtoflux(gam, p, s, DIR, q.g, F);
  primtoflux(gam, p, s, 0, q.g, U);
  vchar(gam, p, s, q, DIR, cmax, cmin, fail);
}

template <int DIR, class R>
__device__ __forceinline__ void face_flux(double gam, const R *pl, const R *pr, const Geo &q, R *F, R &ctop,
                                          int *fail)
{
  StateT<R> s;
  R Fl[8], Ul[8], cmaxl, cminl, cmaxr, cminr;
  get_state(pl, q, s, fail);
  primtoflux(gam, pl, s, DIR, q.g, Fl);
  primtoflux(gam, pl, s, 0, q.g, Ul);
  vchar(gam, pl, s, q, DIR, cmaxl, cminl, fail);
  get_state(pr, q, s, fail);
  {
    R Fr[8], Ur[8];
    primtoflux(gam, pr, s, DIR, q.g, Fr);
    primtoflux(gam, pr, s, 0, q.g, Ur);
    vchar(gam, pr, s, q, DIR, cmaxr, cminr, fail);
    lf_flux(Fl, Ul, cmaxl, cminl, Fr, Ur, cmaxr, cminr, F, ctop);
  }
}

// source() (phys.c:165-207); conn stored as [k][min(nu,j)][max(nu,j)]
__device__ __forceinline__ int conn_slot(int k, int a, int b)
{
  int lo = a < b ? a : b, hi = a < b ? b : a;
  // pairs (lo,hi) with lo <= hi in row order: 00 01 02 03 11 12 13 22 23 33
  int pair = lo == 0 ? hi : lo == 1 ? 3 + hi : lo == 2 ? 5 + hi : 9;
  return k * 10 + pair;
}

template <class R>
__device__ __forceinline__ void source_of_state(double gam, const R *pb, const StateT<R> &s, const Geo &q,
                                                const double *__restrict__ conn, long ng, long gi, R *dU)
{
  R mhd[4][4];
#pragma unroll
  for (int d = 0; d < 4; d++) mhd_calc(gam, pb, d, s, mhd[d]);
#pragma unroll
  for (int k = 0; k < 8; k++) dU[k] = 0.;
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      dU[UU] += mhd[j][k] * __ldg(conn + conn_slot(k, 0, j) * ng + gi);
      dU[U1] += mhd[j][k] * __ldg(conn + conn_slot(k, 1, j) * ng + gi);
      dU[U2] += mhd[j][k] * __ldg(conn + conn_slot(k, 2, j) * ng + gi);
      dU[U3] += mhd[j][k] * __ldg(conn + conn_slot(k, 3, j) * ng + gi);
    }
#pragma unroll
  for (int k = 0; k < 8; k++) dU[k] *= q.g;
}

// slope_lim() (interp.c:49-93)
template <class R>
__device__ __forceinline__ R slope_lim(int lim, R y1, R y2, R y3)
{
  R Dqm, Dqp, s;
  if (lim == 0) {
    Dqm = 2. * (y2 - y1);
    Dqp = 2. * (y3 - y2);
    R Dqc = 0.5 * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= 0.) return R(0.);
    if (fabs(Dqm) < fabs(Dqp) && fabs(Dqm) < fabs(Dqc)) return Dqm;
    if (fabs(Dqp) < fabs(Dqc)) return Dqp;
    return Dqc;
  }
  Dqm = (y2 - y1);
  Dqp = (y3 - y2);
  s = Dqm * Dqp;
  if (s <= 0.) return R(0.);
  if (lim == 1) return 2. * s / (Dqm + Dqp);
  if (fabs(Dqm) < fabs(Dqp)) return Dqm;
  return Dqp;
}

// ---------------------------------------------------------------------------
// conserved -> primitive (utoprim_2d.c, utoprim_1dvsq2fix1.c, utoprim_1dfix1.c)

struct U2P {
  double gam, igam, Bsq, QdotBsq, Qtsq, Qdotn, D, K_atm;
  double W_for_gnr2, rho_for_gnr2;
};

// utoprim_2d.c:229-262 with the u2p_util.c lower_g/raise_g/ncov_calc
__device__ __forceinline__ void u2p_scalars(U2P &c, const double *U, const Geo &q, double *Bcon, double *Qcon,
                                            double *ncon, double &QdotB)
{
  double Bcov[4], Qcov[4], ncov0;
  Bcon[0] = 0.;
  Bcon[1] = U[B1]; Bcon[2] = U[B2]; Bcon[3] = U[B3];
  lower(Bcon, q, Bcov);
  Qcov[0] = U[UU]; Qcov[1] = U[U1]; Qcov[2] = U[U2]; Qcov[3] = U[U3];
  Qcon[0] = q.n00 * Qcov[0] + q.n01 * Qcov[1] + q.n03 * Qcov[3];
  Qcon[1] = q.n10 * Qcov[0] + q.n11 * Qcov[1] + q.n13 * Qcov[3];
  Qcon[2] = q.n22 * Qcov[2];
  Qcon[3] = q.n30 * Qcov[0] + q.n31 * Qcov[1] + q.n33 * Qcov[3];
  c.Bsq = Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3];
  QdotB = Qcov[0] * Bcon[0] + Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  c.QdotBsq = QdotB * QdotB;
  double lapse = sqrt(-1. / q.n00);
  ncov0 = -lapse;
  ncon[0] = q.n00 * ncov0;
  ncon[1] = q.n10 * ncov0;
  ncon[2] = 0. * ncov0;
  ncon[3] = q.n30 * ncov0;
  c.Qdotn = Qcon[0] * ncov0;
  double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
  c.D = U[RHO];
}

// utoprim_2d.c:269-282
__device__ __forceinline__ bool utsq_guess(const Geo &q, const double *prim, double &utsq)
{
  double a = prim[U1], b = prim[U2], d = prim[U3];
  // the reference's double loop over (i, j) in 1..3, zero terms dropped
  utsq = q.v11 * a * a + q.v13 * a * d + q.v22 * b * b + q.v13 * d * a + q.v33 * d * d;
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  return !(utsq < 0. || utsq > UTSQ_TOO_BIG);
}

__device__ __forceinline__ double vsq_calc(const U2P &c, double W)
{
  double Wsq = W * W;
  double Xsq = (c.Bsq + W) * (c.Bsq + W);
  return (Wsq * c.Qtsq + c.QdotBsq * (c.Bsq + 2. * W)) / (Wsq * Xsq);
}

// utoprim_2d.c:562-624 with the gamma-law EOS (:645-678)
__device__ __forceinline__ void func_vsq(const U2P &c, const double *x, double *dx, double &f, double &df)
{
  const double GAMMA = c.gam, Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qtsq = c.Qtsq, Qdotn = c.Qdotn, D = c.D;
  double W = x[0], vsq = x[1], Wsq = W * W;
  double gtmp = 1. - vsq;
  double p_tmp = div_rn((GAMMA - 1.) * (W * gtmp - D * sqrt(gtmp)), GAMMA, c.igam);
  double dPdW = div_rn((GAMMA - 1.) * (1. - vsq), GAMMA, c.igam);
  double dPdvsq = div_rn((GAMMA - 1.) * (0.5 * D / sqrt(1. - vsq) - W), GAMMA, c.igam);
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
  df = -t11 * t11 - t18 * t18;
  f = -0.5 * df;
}

// utoprim_2d.c:442-541
__device__ __forceinline__ int gnr_2d(const U2P &c, double *x)
{
  double f = 1., df = 1., dx[2], x0, x1, errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    func_vsq(c, x, dx, f, df);
    x0 = x[0];
    x1 = x[1];
    (void)x1;
    x[0] += dx[0];
    x[1] += dx[1];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    errx += (x[1] == 0.) ? fabs(dx[1]) : fabs(dx[1] / x[1]);
    // validate_x (utoprim_2d.c:416-431)
    x[0] = fabs(x[0]);
    x[0] = (x[0] > W_TOO_BIG) ? x0 : x[0];
    x[1] = (x[1] < 0.) ? 0. : x[1];
    x[1] = (x[1] > 1.) ? (1. - 1.e-15) : x[1];
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df)) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

// the shared tail: prims from W, v^2 (utoprim_2d.c:346-353)
__device__ __forceinline__ void u2p_velocities(const U2P &c, const double *Qcon, const double *ncon,
                                               const double *Bcon, double QdotB, double W, double gamma,
                                               double *prim)
{
#pragma unroll
  for (int i = 1; i < 4; i++) {
    double Qt = Qcon[i] + ncon[i] * c.Qdotn;
    prim[U1 + i - 1] = gamma / (W + c.Bsq) * (Qt + QdotB * Bcon[i] / W);
  }
}

// utoprim_2d.c:219-362 on the rescaled U
// the mixed path's two-phase Newton solve (harm_phys32.cuh)
__device__ __forceinline__ int gnr_2d_mixed(const U2P &c, double *x);

template <bool MIXED = false>
__device__ __forceinline__ int u2p_body_2d(U2P &c, const double *U, const Geo &q, double *prim)
{
  double Bcon[4], Qcon[4], ncon[4], QdotB, utsq;
  u2p_scalars(c, U, q, Bcon, Qcon, ncon, QdotB);
  if (!utsq_guess(q, prim, utsq)) return 2;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c.D / gamma;
  double u = prim[UU];
  double p = (c.gam - 1.) * u;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq))
          <= W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq))
         && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  double x[2];
  x[0] = fabs(W_last);
  double vsq0 = fabs(vsq_calc(c, W_last));
  x[1] = (vsq0 > 1.) ? (1.0 - 1.e-15) : vsq0;
  int retval;
  if constexpr (MIXED) retval = gnr_2d_mixed(c, x);
  else retval = gnr_2d(c, x);
  double W = x[0], vsq = x[1];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c.D * gtmp;
  w = W * (1. - vsq);
  p = div_rn((c.gam - 1.) * (w - rho0), c.gam, c.igam);
  u = w - (rho0 + p);
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  u2p_velocities(c, Qcon, ncon, Bcon, QdotB, W, gamma, prim);
  return 0;
}

// ---- Utoprim_1dvsq2fix1 (utoprim_1dvsq2fix1.c) ----

__device__ __forceinline__ double W_of_vsq_fix(const U2P &c, double vsq, double &p, double &rho, double &u)
{
  double gtmp = (1. - vsq);
  rho = c.D * sqrt(gtmp);
  p = c.K_atm * pow_cr(rho, c.gam);
  u = p / (c.gam - 1.);
  return (rho + u + p) / gtmp;
}

static __device__ __noinline__ int u2p_body_vsq2fix1(U2P &c, const double *U, const Geo &q, double *prim)
{
  double Bcon[4], Qcon[4], ncon[4], QdotB, utsq, p, rho0, u;
  u2p_scalars(c, U, q, Bcon, Qcon, ncon, QdotB);
  if (!utsq_guess(q, prim, utsq)) return 2;
  double gammasq = 1. + utsq;
  double x = 1. - 1. / gammasq;
  // general_newton_raphson (utoprim_1dvsq2fix1.c:395-492) with func_1d_gnr (:541-566)
  const double GAMMA = c.gam;
  double f = 1., df = 1., errx = 1., W = 0., W_old;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    if (x != x) return 201;  // as in Utoprim_1dfix1 below: NaN to the end, then failure 201
    double pp, rr, uu;
    double Wc = W_of_vsq_fix(c, x, pp, rr, uu);
    double Wsq = Wc * Wc, W3 = Wc * Wsq;
    double dWdvsq = (GAMMA * (2. - GAMMA) * pp + (GAMMA - 1.) * rr) / (2. * (GAMMA - 1.) * (1. - x) * (1. - x));
    double fact_tmp = (c.Bsq + Wc);
    double r0 = c.Qtsq - x * fact_tmp * fact_tmp + c.QdotBsq * (c.Bsq + 2. * Wc) / Wsq;
    double j00 = -fact_tmp * (fact_tmp + 2. * dWdvsq * (x + c.QdotBsq / W3));
    double dx = -r0 / j00;
    f = 0.5 * r0 * r0;
    df = -2. * f;
    double x_old = x;
    x += dx;
    x = (x >= 1.0) ? (0.5 * (x_old + 1.)) : x;
    x = (x < -1.e-10) ? (0.5 * x_old) : x;
    x = fabs(x);
    W_old = W;
    W = W_of_vsq_fix(c, x, pp, rr, uu);
    errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
    errx += (x == 0.) ? fabs(x - x_old) : fabs((x - x_old) / x);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  int retval = 0;
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  if (retval != 0) return retval * 100 + 1;
  double vsq = x;
  if ((vsq >= 1.) || (vsq < 0.)) return 4;
  double Wf = W_of_vsq_fix(c, vsq, p, rho0, u);
  double gtmp = sqrt(1. - vsq);
  double gamma = 1. / gtmp;
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  u2p_velocities(c, Qcon, ncon, Bcon, QdotB, Wf, gamma, prim);
  return 0;
}

// ---- Utoprim_1dfix1 (utoprim_1dfix1.c) ----

// gnr2 with func_gnr2_rho (:601-697, :818-838)
static __device__ __noinline__ int gnr2_rho(const U2P &c, double &x)
{
  const double GAMMA = c.gam;
  double f = 1., df = 1., errx = 1.;
  int n_iter = 0;
  bool keep = true;
  while (keep) {
    // a NaN iterate stays NaN through every remaining trial, and the solve
    // then ends in failure (2) with x NaN: return that now
    if (x != x) return 2;
    double A = c.D * c.D;
    double B0 = A * GAMMA * c.K_atm;
    double B = B0 / (GAMMA - 1.);
    double rho = x;
    double W = c.W_for_gnr2;
    double C = pow_cr(rho, GAMMA - 1.);
    double r0 = rho * W - A - B * C;
    double j00 = W - B0 * C / rho;
    double dx = -r0 / j00;
    f = 0.5 * r0 * r0;
    df = -2. * f;
    x += dx;
    errx = 0.;
    errx += (x == 0.) ? fabs(dx) : fabs(dx / x);
    errx /= 1. * 1;
    x = fabs(x);
    if (((fabs(errx) <= NEWT_TOL2)) || (n_iter >= (MAX_NEWT_ITER - 1))) keep = false;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x)) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

// func_1d_orig1 (:721-771)
static __device__ __noinline__ void func_1d_orig1(U2P &c, double W, double &dx, double &f, double &df)
{
  const double GAMMA = c.gam, K_atm = c.K_atm, Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qtsq = c.Qtsq;
  c.W_for_gnr2 = W;
  double rho_g, x_rho;
  rho_g = x_rho = c.rho_for_gnr2;
  int ntries = 0;
  while (gnr2_rho(c, x_rho) && (ntries++ < 10)) {
    rho_g *= 10.;
    x_rho = rho_g;
  }
  double rho = c.rho_for_gnr2 = x_rho;
  double Dc = c.D;
  double t1 = Dc * Dc, t2 = QdotBsq * t1, t3 = t2 * Bsq, t5 = Bsq * Bsq, t8 = t1 * Bsq, t10 = t1 * W,
         t21 = W * W, t23 = rho * rho, t26 = 1. / t1;
  double r0 = (t3 + (2.0 * t2 + ((Qtsq - t5) * t1 + (-2.0 * t8 - t10) * W) * W) * W
               + (t5 + (2.0 * Bsq + W) * W) * t21 * t23) * t26 / t21;
  double t29 = t1 * t1, t30 = QdotBsq * t29, t32 = GAMMA * K_atm, t33 = pow_cr(rho, 1.0 * GAMMA), t34 = t32 * t33,
         t38 = t23 * t33, t51 = GAMMA * t1 * K_atm * t33, t67 = t21 * W;
  double j00 = -2.0 * (t30 * Bsq * t34
                       + (t30 * t34 + ((-t38 * Bsq * t32 + Bsq * GAMMA * t1 * K_atm * t33) * t1
                                       + (-t38 * GAMMA * K_atm + t51) * t1 * W) * t21) * W
                       + ((-t3 + (-t2 + (-t8 - t10) * t21) * W) * W + (-t5 - Bsq * W) * t67 * t23) * t23)
               * t26 / (t51 - W * t23) / t67;
  dx = -r0 / j00;
  f = 0.5 * r0 * r0;
  df = -2. * f;
}

static __device__ __noinline__ int u2p_body_fix1(U2P &c, const double *U, const Geo &q, double *prim)
{
  double Bcon[4], Qcon[4], ncon[4], QdotB, utsq;
  u2p_scalars(c, U, q, Bcon, Qcon, ncon, QdotB);
  if (!utsq_guess(q, prim, utsq)) return 2;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = c.D / gamma;
  double p = c.K_atm * pow_cr(rho0, c.gam);
  double u = p / (c.gam - 1.);
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq))
          <= W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq))
         && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  c.W_for_gnr2 = W_last;
  c.rho_for_gnr2 = rho0;
  // general_newton_raphson (utoprim_1dfix1.c:500-595)
  double x = W_last, f = 1., df = 1., errx = 1.;
  const double Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qtsq = c.Qtsq;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    // once W is NaN every remaining trial gives NaN, and the inversion ends in
    // failure 201 with prim untouched: return that now (c is the caller's
    // scratch and is discarded)
    if (x != x) return 201;
    double dx;
    func_1d_orig1(c, x, dx, f, df);
    x += dx;
    int inc = 0;
    while (((x * x * x * (x + 2. * Bsq) - QdotBsq * (2. * x + Bsq)) <= x * x * (Qtsq - Bsq * Bsq)) && (inc < 10)) {
      x -= (1. * inc) * dx / 10.;
      inc++;
    }
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER)
        || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  int retval = 0;
  if (!isfinite(f) || !isfinite(df) || !isfinite(x)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  double W = x;
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  double vsq = vsq_calc(c, W);
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c.D * gtmp;
  p = c.K_atm * pow_cr(rho0, c.gam);
  u = p / (c.gam - 1.);
  if ((rho0 <= 0.) || (u <= 0.)) return 5;
  prim[RHO] = rho0;
  prim[UU] = u;
  u2p_velocities(c, Qcon, ncon, Bcon, QdotB, W, gamma, prim);
  return 0;
}

// the U and prim rescaling around every inversion (utoprim_2d.c:126-176);
// which: 0 Utoprim_2d, 1 Utoprim_1dvsq2fix1, 2 Utoprim_1dfix1
template <int which, bool MIXED = false>
__device__ __forceinline__ int utoprim(double gam, double K, const double *U, const Geo &q, double *prim)
{
  double Ut[8], pt[8];
  prim[B1] = div_rn(U[B1], q.g, q.ig);
  prim[B2] = div_rn(U[B2], q.g, q.ig);
  prim[B3] = div_rn(U[B3], q.g, q.ig);
  if (U[0] <= 0.) return -100;
  const double alpha = q.alpha;
  Ut[RHO] = div_rn(alpha * U[RHO], q.g, q.ig);
  Ut[UU] = div_rn(alpha * (U[UU] - U[RHO]), q.g, q.ig);
#pragma unroll
  for (int i = U1; i <= B3; i++) Ut[i] = div_rn(alpha * U[i], q.g, q.ig);
#pragma unroll
  for (int i = 0; i < B1; i++) pt[i] = prim[i];
#pragma unroll
  for (int i = B1; i <= B3; i++) pt[i] = alpha * prim[i];
  U2P c;
  c.gam = gam;
  c.igam = 1. / gam;
  c.K_atm = K;
  int ret;
  if (which == 0) ret = u2p_body_2d<MIXED>(c, Ut, q, pt);
  else if (which == 1) ret = u2p_body_vsq2fix1(c, Ut, q, pt);
  else ret = u2p_body_fix1(c, Ut, q, pt);
  if (ret == 0) {
#pragma unroll
    for (int i = 0; i < B1; i++) prim[i] = pt[i];
  }
  return ret;
}

// ---------------------------------------------------------------------------
// floors (fixup.c:142-383) with precomputed radial floors rho_flr, u_flr
// (get_rho_u_floor, fixup.c:117-140, evaluated on the host with the same pow)

// phys.c:273-297
template <class R>
__device__ __forceinline__ R ut_calc_3vel(const R *v, const Geo &q)
{
  double AA = q.v00;
  R BB = 2. * (q.v01 * v[1] + q.v03 * v[3]);
  R CC = q.v11 * v[1] * v[1] + q.v22 * v[2] * v[2] + q.v33 * v[3] * v[3] + 2. * (q.v13 * v[1] * v[3]);
  R DD = -1. / (AA + BB + CC);
  double one_over_alpha_sq = -q.n00;
  if (DD < one_over_alpha_sq) DD = one_over_alpha_sq;
  return sqrt(DD);
}

// returns true if the zone's pflag must be set to -33 (gamma failure)
template <class R>
static __device__ bool fixup1zone(double gam, double rho_floor, double uu_floor, const Geo &q, R *pv, int *fail)
{
  R pre[8];
#pragma unroll
  for (int k = 0; k < 8; k++) pre[k] = pv[k];
  StateT<R> s;
  get_state(pv, q, s, fail);
  R bsq = dot4(s.bcon, s.bcov);
  R rhoflr = rho_floor, uuflr = uu_floor;
  if (rhoflr < bsq / BSQORHOMAX) rhoflr = bsq / BSQORHOMAX;
  if (uuflr < bsq / BSQOUMAX) uuflr = bsq / BSQOUMAX;
  if (rhoflr < pv[UU] / UORHOMAX) rhoflr = pv[UU] / UORHOMAX;
  bool dofloor = false;
  if (pv[RHO] < rhoflr) { pv[RHO] = rhoflr; dofloor = true; }
  if (pv[UU] < uuflr) { pv[UU] = uuflr; dofloor = true; }
  R trans;
  if (dofloor && (trans = 10. * bsq / (pv[RHO] < pv[UU] ? pv[RHO] : pv[UU]) - 1.) > 0.) {
    if (trans > 1.) trans = 1.;
    R betapar = -s.bcon[0] / ((bsq + SMALL) * s.ucon[0]);
    R betasq = betapar * betapar * bsq;
    double betasqmax = 1. - 1. / (GAMMAMAX * GAMMAMAX);
    if (betasq > betasqmax) betasq = betasqmax;
    R gdr = 1. / sqrt(1 - betasq);
    R ucondr[4], Bcon[4], Bcov[4], vcon[4], ucon[4];
#pragma unroll
    for (int k = 0; k < 4; k++) ucondr[k] = gdr * (s.ucon[k] + betapar * s.bcon[k]);
    Bcon[0] = 0.;
    Bcon[1] = pv[B1]; Bcon[2] = pv[B2]; Bcon[3] = pv[B3];
    lower(Bcon, q, Bcov);
    R udotB = dot4(s.ucon, Bcov);
    R Bsq = dot4(Bcon, Bcov);
    R B = sqrt(Bsq);
    R wold = pre[RHO] + pre[UU] * gam;
    R QdotB = udotB * wold * s.ucon[0];
    R wnew = pv[RHO] + pv[UU] * gam;
    R x = 2. * QdotB / (B * wnew * ucondr[0] + SMALL);
    R vpar = x / (ucondr[0] * (1. + sqrt(1. + x * x)));
    R one_over_ucondr_t = 1. / ucondr[0];
    vcon[0] = 1.;
#pragma unroll
    for (int k = 1; k < 4; k++) vcon[k] = vpar * Bcon[k] / (B + SMALL) + ucondr[k] * one_over_ucondr_t;
    R ut = ut_calc_3vel(vcon, q);
#pragma unroll
    for (int k = 0; k < 4; k++) ucon[k] = ut * vcon[k];
    // ucon_to_utcon (phys.c:255-270)
    const double alpha = q.alpha;
    R gm = alpha * ucon[0];
    double be[4] = {0., q.n01 * alpha * alpha, 0. * alpha * alpha, q.n03 * alpha * alpha};
#pragma unroll
    for (int k = 1; k < 4; k++) {
      R utc = ucon[k] + gm * be[k] / alpha;
      pv[k + UU] = utc * trans + pre[k + UU] * (1. - trans);
    }
  }
  R gamma;
  if (gamma_calc(pv, q, gamma)) return true;
  if (gamma > GAMMAMAX) {
    R f = sqrt((GAMMAMAX * GAMMAMAX - 1.) / (gamma * gamma - 1.));
    pv[U1] *= f;
    pv[U2] *= f;
    pv[U3] *= f;
  }
  return false;
}

// inflow_check() (bounds.c:333-378)
template <class R>
__device__ __forceinline__ void inflow_check(R *pr, const Geo &q, int type, int *fail)
{
  R ucon[4];
  ucon_calc(pr, q, ucon, fail);
  if (((ucon[1] > 0.) && (type == 0)) || ((ucon[1] < 0.) && (type == 1))) {
    R gamma;
    if (gamma_calc(pr, q, gamma)) *fail = FAIL_GAMMA;
    pr[U1] /= gamma;
    pr[U2] /= gamma;
    pr[U3] /= gamma;
    const double alpha = q.alpha;
    double beta1 = q.n01 * alpha * alpha;
    pr[U1] = beta1 / alpha;
    R a = pr[U1], b = pr[U2], d = pr[U3];
    R vsq = q.v11 * a * a + q.v13 * a * d + q.v22 * b * b + q.v13 * d * a + q.v33 * d * d;
    if (fabs(vsq) < 1.e-13) vsq = 1.e-13;
    if (vsq >= 1.) vsq = 1. - 1. / (GAMMAMAX * GAMMAMAX);
    gamma = 1. / sqrt(1. - vsq);
    pr[U1] *= gamma;
    pr[U2] *= gamma;
    pr[U3] *= gamma;
  }
}

}  // namespace harm
