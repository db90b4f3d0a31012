// FP32 face-flux physics of the mixed-precision step: the same formulas as
// harm_phys.cuh (phys.c:59-476, interp.c:49-93) evaluated in float on an
// FP32 copy of the face metric.  Only the reconstruction, the face states,
// their fluxes and the magnetosonic speeds use it; everything that feeds the
// conserved update's accumulation and the inversion stays FP64.
#pragma once
#include "harm_phys.cuh"

namespace harm {

struct GeoF {
  float v00, v01, v03, v11, v13, v22, v33;
  float n00, n01, n03, n10, n11, n13, n22, n30, n31, n33;
  float g;
};

__device__ __forceinline__ void load_geo_f(const float *__restrict__ G, long ng, long gi, GeoF &q)
{
  q.v00 = __ldg(G + 0 * ng + gi); q.v01 = __ldg(G + 1 * ng + gi); q.v03 = __ldg(G + 2 * ng + gi);
  q.v11 = __ldg(G + 3 * ng + gi); q.v13 = __ldg(G + 4 * ng + gi); q.v22 = __ldg(G + 5 * ng + gi);
  q.v33 = __ldg(G + 6 * ng + gi);
  q.n00 = __ldg(G + 7 * ng + gi); q.n01 = __ldg(G + 8 * ng + gi); q.n03 = __ldg(G + 9 * ng + gi);
  q.n10 = __ldg(G + 10 * ng + gi); q.n11 = __ldg(G + 11 * ng + gi); q.n13 = __ldg(G + 12 * ng + gi);
  q.n22 = __ldg(G + 13 * ng + gi); q.n30 = __ldg(G + 14 * ng + gi); q.n31 = __ldg(G + 15 * ng + gi);
  q.n33 = __ldg(G + 16 * ng + gi); q.g = __ldg(G + 17 * ng + gi);
}

struct StateF {
  float ucon[4], ucov[4], bcon[4], bcov[4];
};

__device__ __forceinline__ void lower_f(const float *u, const GeoF &q, float *d)
{
  d[0] = q.v00 * u[0] + q.v01 * u[1] + q.v03 * u[3];
  d[1] = q.v01 * u[0] + q.v11 * u[1] + q.v13 * u[3];
  d[2] = q.v22 * u[2];
  d[3] = q.v03 * u[0] + q.v13 * u[1] + q.v33 * u[3];
}

__device__ __forceinline__ float dot4f(const float *a, const float *b)
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

// get_state() in float; alpha = 1/sqrt(-g^tt), gamma from the relative 4-velocity
__device__ __forceinline__ void get_state_f(const float *pr, const GeoF &q, StateF &s, int *fail)
{
  const float ialpha = sqrtf(-q.n00);  // 1/alpha
  float qsq = q.v11 * pr[U1] * pr[U1] + q.v22 * pr[U2] * pr[U2] + q.v33 * pr[U3] * pr[U3]
              + 2.f * (q.v13 * pr[U1] * pr[U3]);
  if (qsq < 0.f) {
    if (fabsf(qsq) > 1.E-10f) *fail = FAIL_GAMMA;
    qsq = 1.E-10f;
  }
  const float gamma = sqrtf(1.f + qsq);
  // u^t = gamma/alpha, u^i = utilde^i - gamma beta^i / alpha with beta^i = g^{ti} alpha^2
  s.ucon[0] = gamma * ialpha;
  const float ga = gamma / ialpha;  // gamma * alpha
  s.ucon[1] = pr[U1] - ga * q.n01;
  s.ucon[2] = pr[U2];
  s.ucon[3] = pr[U3] - ga * q.n03;
  lower_f(s.ucon, q, s.ucov);
  s.bcon[0] = pr[B1] * s.ucov[1] + pr[B2] * s.ucov[2] + pr[B3] * s.ucov[3];
  const float iut = 1.f / s.ucon[0];
  s.bcon[1] = (pr[B1] + s.bcon[0] * s.ucon[1]) * iut;
  s.bcon[2] = (pr[B2] + s.bcon[0] * s.ucon[2]) * iut;
  s.bcon[3] = (pr[B3] + s.bcon[0] * s.ucon[3]) * iut;
  lower_f(s.bcon, q, s.bcov);
}

// primtoflux() for direction dir and (dir = 0) the conserved variables, sharing b^2
template <int DIR>
__device__ __forceinline__ void fluxes_f(float gam, const float *pr, const StateF &s, float g, float *F, float *U,
                                         float &bsq_out)
{
  const float r = pr[RHO], u = pr[UU];
  const float P = (gam - 1.f) * u;
  const float w = P + r + u;
  const float bsq = dot4f(s.bcon, s.bcov);
  const float eta = w + bsq;
  const float ptot = P + 0.5f * bsq;
  bsq_out = bsq;
  // direction DIR
  F[RHO] = g * (r * s.ucon[DIR]);
  {
    const float eu = eta * s.ucon[DIR], bd = s.bcon[DIR];
    const float m0 = eu * s.ucov[0] - bd * s.bcov[0];
    F[UU] = g * (m0 + r * s.ucon[DIR]);
    F[U1] = g * (eu * s.ucov[1] + (DIR == 1 ? ptot : 0.f) - bd * s.bcov[1]);
    F[U2] = g * (eu * s.ucov[2] + (DIR == 2 ? ptot : 0.f) - bd * s.bcov[2]);
    F[U3] = g * (eu * s.ucov[3] + (DIR == 3 ? ptot : 0.f) - bd * s.bcov[3]);
    F[B1] = g * (s.bcon[1] * s.ucon[DIR] - bd * s.ucon[1]);
    F[B2] = g * (s.bcon[2] * s.ucon[DIR] - bd * s.ucon[2]);
    F[B3] = g * (s.bcon[3] * s.ucon[DIR] - bd * s.ucon[3]);
  }
  // time component (conserved variables)
  {
    const float eu = eta * s.ucon[0], bd = s.bcon[0];
    U[RHO] = g * (r * s.ucon[0]);
    U[UU] = g * (eu * s.ucov[0] + ptot - bd * s.bcov[0] + r * s.ucon[0]);
    U[U1] = g * (eu * s.ucov[1] - bd * s.bcov[1]);
    U[U2] = g * (eu * s.ucov[2] - bd * s.bcov[2]);
    U[U3] = g * (eu * s.ucov[3] - bd * s.bcov[3]);
    U[B1] = g * (s.bcon[1] * s.ucon[0] - bd * s.ucon[1]);
    U[B2] = g * (s.bcon[2] * s.ucon[0] - bd * s.ucon[2]);
    U[B3] = g * (s.bcon[3] * s.ucon[0] - bd * s.ucon[3]);
  }
}

// vchar() in float (phys.c:337-476, gamma-law)
template <int DIR>
__device__ __forceinline__ void vchar_f(float gam, const float *pr, const StateF &s, const GeoF &q, float bsq,
                                        float &vmax, float &vmin, int *fail)
{
  const float rho = pr[RHO], u = pr[UU];
  const float EF = rho + gam * u;
  const float EE = bsq + EF;
  const float va2 = bsq / EE;
  const float cs2 = gam * (gam - 1.f) * u / EF;
  float cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.f) { *fail = FAIL_COEFF_NEG; cms2 = 1.e-20f; }
  if (cms2 > 1.f) { *fail = FAIL_COEFF_SUP; cms2 = 1.f; }
  const float Asq = DIR == 1 ? q.n11 : DIR == 2 ? q.n22 : q.n33;
  const float Bsq = q.n00;
  const float Au = s.ucon[DIR], Bu = s.ucon[0];
  const float AB = DIR == 1 ? q.n01 : DIR == 2 ? 0.f : q.n03;
  const float Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  const float A = Bu2 - (Bsq + Bu2) * cms2;
  const float B = 2.f * (AuBu - (AB + AuBu) * cms2);
  const float C = Au2 - (Asq + Au2) * cms2;
  float discr = B * B - 4.f * A * C;
  if (discr < 0.f) discr = 0.f;
  discr = sqrtf(discr);
  const float i2a = 0.5f / A;
  const float vp = (B - discr) * i2a;
  const float vm = (B + discr) * i2a;
  vmax = fmaxf(vp, vm);
  vmin = fminf(vp, vm);
}

__device__ __forceinline__ float slope_lim_f(int lim, float y1, float y2, float y3)
{
  float Dqm, Dqp, s;
  if (lim == 0) {
    Dqm = 2.f * (y2 - y1);
    Dqp = 2.f * (y3 - y2);
    const float Dqc = 0.5f * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= 0.f) return 0.f;
    if (fabsf(Dqm) < fabsf(Dqp) && fabsf(Dqm) < fabsf(Dqc)) return Dqm;
    if (fabsf(Dqp) < fabsf(Dqc)) return Dqp;
    return Dqc;
  }
  Dqm = (y2 - y1);
  Dqp = (y3 - y2);
  s = Dqm * Dqp;
  if (s <= 0.f) return 0.f;
  if (lim == 1) return 2.f * s / (Dqm + Dqp);
  if (fabsf(Dqm) < fabsf(Dqp)) return Dqm;
  return Dqp;
}

// the local Lax-Friedrichs flux of one face in float
template <int DIR>
__device__ __forceinline__ void face_flux_f(float gam, const float *pl, const float *pr, const GeoF &q, float *F,
                                            float &ctop, int *fail)
{
  StateF s;
  float Fl[8], Ul[8], Fr[8], Ur[8], bsq, cmaxl, cminl, cmaxr, cminr;
  get_state_f(pl, q, s, fail);
  fluxes_f<DIR>(gam, pl, s, q.g, Fl, Ul, bsq);
  vchar_f<DIR>(gam, pl, s, q, bsq, cmaxl, cminl, fail);
  get_state_f(pr, q, s, fail);
  fluxes_f<DIR>(gam, pr, s, q.g, Fr, Ur, bsq);
  vchar_f<DIR>(gam, pr, s, q, bsq, cmaxr, cminr, fail);
  const float cmax = fabsf(fmaxf(fmaxf(0.f, cmaxl), cmaxr));
  const float cmin = fabsf(fmaxf(fmaxf(0.f, -cminl), -cminr));
  ctop = fmaxf(cmax, cmin);
#pragma unroll
  for (int k = 0; k < 8; k++) F[k] = 0.5f * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k]));
}

// ---------------------------------------------------------------------------
// the mixed path's zone update

// relative Newton step at which the float phase hands over to FP64
constexpr float F32_NEWT_TOL = 1.e-5f;

// source() (phys.c:165-207) in float: dU_nu = sqrt(-g) T^kappa_lambda
// Gamma^lambda_{nu kappa}, on an FP32 copy of the connection (stored as
// [k][min(nu,j)][max(nu,j)] like the FP64 planes); used away from the horizon
__device__ __forceinline__ void source_f(float gam, const float *pr, const GeoF &q, const float *__restrict__ conn,
                                         long ng, long gi, double *dU, int *fail)
{
  StateF s;
  get_state_f(pr, q, s, fail);
  const float r = pr[RHO], u = pr[UU];
  const float P = (gam - 1.f) * u;
  const float bsq = dot4f(s.bcon, s.bcov);
  const float eta = P + r + u + bsq;
  const float ptot = P + 0.5f * bsq;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float t = eta * s.ucon[j] * s.ucov[k] + (j == k ? ptot : 0.f) - s.bcon[j] * s.bcov[k];
#pragma unroll
      for (int nu = 0; nu < 4; nu++) {
        const int lo = nu < j ? nu : j, hi = nu < j ? j : nu;
        const int pair = lo == 0 ? hi : lo == 1 ? 3 + hi : lo == 2 ? 5 + hi : 9;
        acc[nu] += t * __ldg(conn + (long)(k * 10 + pair) * ng + gi);
      }
    }
#pragma unroll
  for (int k = 0; k < 8; k++) dU[k] = 0.;
  dU[UU] = (double)(acc[0] * q.g);
  dU[U1] = (double)(acc[1] * q.g);
  dU[U2] = (double)(acc[2] * q.g);
  dU[U3] = (double)(acc[3] * q.g);
}

// func_vsq() (utoprim_2d.c:562-624, gamma-law) in float: the Newton step only
__device__ __forceinline__ float newton_step_f(float GAMMA, float Bsq, float QdotBsq, float Qtsq, float Qdotn, float D,
                                               float W, float vsq, float &dW, float &dv)
{
  const float Wsq = W * W;
  const float gtmp = 1.f - vsq;
  const float sg = sqrtf(gtmp);
  const float p_tmp = (GAMMA - 1.f) * (W * gtmp - D * sg) / GAMMA;
  const float dPdW = (GAMMA - 1.f) * gtmp / GAMMA;
  const float dPdvsq = (GAMMA - 1.f) * (0.5f * D / sg - W) / GAMMA;
  const float t2 = -0.5f * Bsq + dPdvsq;
  const float t3 = Bsq + W;
  const float t4 = t3 * t3;
  const float t9 = 1.f / Wsq;
  const float t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.f * W) * t9;
  const float t16 = QdotBsq * t9;
  const float t18 = -Qdotn - 0.5f * Bsq * (1.f + vsq) + 0.5f * t16 - W + p_tmp;
  const float t21 = 1.f / t3;
  const float t23 = 1.f / W;
  const float t24 = t16 * t23;
  const float t25 = -1.f + dPdW - t24;
  const float t35 = t25 * t3 + (Bsq - 2.f * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  const float t36 = 1.f / t35;
  dW = -(t2 * t11 + t4 * t18) * t21 * t36;
  dv = -(-t25 * t11 - 2.f * (vsq + t24) * t3 * t18) * t21 * t36;
  return t11 * t11 + t18 * t18;
}

// The 2D Newton solve of the mixed path: Newton steps in float from the
// reference's starting point until the relative step falls below 1e-5, then
// FP64 Newton steps (the residual and Jacobian of func_vsq, the reference's
// validate_x clamps) until it falls below NEWT_TOL.  When the float phase
// converged and the first FP64 step is itself below 1e-5 -- it confirms the
// float answer to that accuracy, and a Newton step from there squares the
// error -- that step ends the solve.  Falls back to the FP64 solve from the
// start when the float phase leaves the finite range.
__device__ __forceinline__ int gnr_2d_mixed(const U2P &c, double *x)
{
  float W = (float)x[0], vsq = (float)x[1];
  const float G = (float)c.gam, Bsq = (float)c.Bsq, QB = (float)c.QdotBsq, Qt = (float)c.Qtsq, Qn = (float)c.Qdotn,
              D = (float)c.D;
  bool ok = isfinite(W) && isfinite(vsq) && W > 0.f;
  bool f32_conv = false;
  for (int n = 0; n < MAX_NEWT_ITER && ok; n++) {
    float dW, dv;
    newton_step_f(G, Bsq, QB, Qt, Qn, D, W, vsq, dW, dv);
    const float W0 = W;
    W += dW;
    vsq += dv;
    float errx = (W == 0.f) ? fabsf(dW) : fabsf(dW / W);
    errx += (vsq == 0.f) ? fabsf(dv) : fabsf(dv / vsq);
    W = fabsf(W);
    W = (W > 1.e20f) ? W0 : W;
    vsq = vsq < 0.f ? 0.f : vsq;
    vsq = vsq > 1.f ? 1.f - 1.e-7f : vsq;
    ok = isfinite(W) && isfinite(vsq) && W > 0.f;
    if (errx <= F32_NEWT_TOL) {
      f32_conv = ok;
      break;
    }
  }
  if (ok) {
    x[0] = (double)W;
    x[1] = (double)vsq;
  }
  double f = 1., df = 1., dx[2], errx = 1.;
  for (int n = 0; n < MAX_NEWT_ITER; n++) {
    func_vsq(c, x, dx, f, df);
    const double x0 = x[0];
    x[0] += dx[0];
    x[1] += dx[1];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    errx += (x[1] == 0.) ? fabs(dx[1]) : fabs(dx[1] / x[1]);
    x[0] = fabs(x[0]);
    x[0] = (x[0] > W_TOO_BIG) ? x0 : x[0];
    x[1] = (x[1] < 0.) ? 0. : x[1];
    x[1] = (x[1] > 1.) ? (1. - 1.e-15) : x[1];
    if (fabs(errx) <= NEWT_TOL) break;
    if (n == 0 && f32_conv && errx <= (double)F32_NEWT_TOL) {
      errx = 0.;
      break;
    }
  }
  if (!isfinite(f) || !isfinite(df)) return 2;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

}  // namespace harm
