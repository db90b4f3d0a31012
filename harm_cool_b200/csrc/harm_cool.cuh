// Zone physics of the COOL_EOS step: the stress tensor, fluxes, wave speeds
// and source with the run-time EOS pressure, and the 5D Newton inversion
// Utoprim_5d with its analytic Jacobian.
//
// Reference: mhd_calc_CoolEOS and the COOL_EOS branches of primtoflux,
// source and vchar (phys.c:47-207, 337-476); Utoprim_5d and its helpers
// (utoprim_5d.c:179-982) over the u2p_util.c routines (u2p_util.c:50-340).
// As in harm_phys.cuh, metric entries that vanish in modified Kerr-Schild
// coordinates are not stored and the x*0 terms are not added; every other
// operation keeps the reference's order, and the unit is built with
// -fmad=false.
#pragma once
#include "harm_eos.cuh"

namespace harm {

// ---------------------------------------------------------------------------
// fluxes, wave speeds and source with the run-time EOS (phys.c)

// mhd_calc_CoolEOS (phys.c:122-141)
__device__ __forceinline__ void mhd_calc_cool(double r, double u, double P, int dir, const State &s, double *mhd)
{
  double w = P + r + u;
  double bsq = dot4(s.bcon, s.bcov);
  double eta = w + bsq;
  double ptot = P + 0.5 * bsq;
#pragma unroll
  for (int j = 0; j < 4; j++)
    mhd[j] = eta * s.ucon[dir] * s.ucov[j] + ptot * (dir == j ? 1. : 0.) - s.bcon[dir] * s.bcov[j];
}

// the EOS calls of the face physics: FP64 (the reference's arithmetic) or the
// mixed-precision interpolation
template <bool F32>
__device__ __forceinline__ double face_pressure(const EosDev &E, EosCursor &c, double rho, double u)
{
  return F32 ? eos_pressure_f(E, c, rho, u) : eos_pressure(E, c, rho, u);
}

// primtoflux() with COOL_EOS (phys.c:59-96)
template <bool F32 = false>
__device__ __forceinline__ void primtoflux_cool(const EosDev &E, EosCursor &c, const double *pr, const State &s,
                                                int dir, double g, double *flux)
{
  double mhd[4];
  flux[RHO] = pr[RHO] * s.ucon[dir];
  {
    const double rho = pr[RHO], u = pr[UU];
    const double p = face_pressure<F32>(E, c, rho, u);
    mhd_calc_cool(rho, u, p, dir, s, mhd);
  }
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

// vchar() with COOL_EOS and COOL_EOS_SIMPLECS 0 (phys.c:337-476): the sound
// speed of Ibanez et al. from dp/drho and dp/de; no fail() on the clamps
template <bool F32 = false>
__device__ __forceinline__ void vchar_cool(const EosDev &E, EosCursor &c, const double *pr, const State &s,
                                           const Geo &q, int js, double &vmax, double &vmin, int *fail)
{
  double bsq = dot4(s.bcon, s.bcov);
  double rho = pr[RHO], u = pr[UU];
  double p = face_pressure<F32>(E, c, rho, u);
  double EF = rho + u + p;
  double EE = bsq + EF;
  double va2 = bsq / EE;
  double cs2;
  {
    double e = u / rho;
    double enthalpy = 1.0 + e + p / rho;
    double dpdrho = F32 ? eos_dpdrho_f(E, c, rho, u) : eos_dpdrho(E, c, rho, u);
    double dpde = (F32 ? eos_dpdu_f(E, c, rho, u) : eos_dpdu(E, c, rho, u)) * rho;
    cs2 = (dpdrho + p / rho / rho * dpde) / enthalpy;
  }
  double cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < SMALL) cms2 = SMALL;
  if (cms2 > 1.) cms2 = 1.;
  double Asq = gcon_diag(q, js), Bsq = q.n00;
  double Au = s.ucon[js], Bu = s.ucon[0], AB = gcon_t(q, js);
  double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  double A = Bu2 - (Bsq + Bu2) * cms2;
  double B = 2. * (AuBu - (AB + AuBu) * cms2);
  double C = Au2 - (Asq + Au2) * cms2;
  double discr = B * B - 4. * A * C;
  if ((discr < 0.0) && (discr > -1.e-10)) discr = 0.0;
  else if (discr < -1.e-10) { *fail = FAIL_VCHAR_DISCR; discr = 0.; }
  discr = sqrt(discr);
  double vp = -(-B + discr) / (2. * A);
  double vm = -(-B - discr) / (2. * A);
  if (vp > vm) { vmax = vp; vmin = vm; }
  else { vmax = vm; vmin = vp; }
}

// ---------------------------------------------------------------------------
// u2p_util.c routines (metric from a Geo)

// ucon_calc_g (u2p_util.c:152-176)
__device__ __forceinline__ void ucon_calc_g(const double *pr, const Geo &q, double *ucon)
{
  double a = 0.;
  a += q.v11 * pr[U1] * pr[U1];
  a += q.v13 * pr[U1] * pr[U3];
  a += q.v22 * pr[U2] * pr[U2];
  a += q.v13 * pr[U3] * pr[U1];
  a += q.v33 * pr[U3] * pr[U3];
  a = fabs(a);
  double gamma = sqrt(1. + a);
  double lapse = sqrt(-1. / q.n00);
  ucon[0] = 0. - lapse * gamma * q.n00;
  ucon[1] = pr[U1] - lapse * gamma * q.n01;
  ucon[2] = pr[U2] - lapse * gamma * 0.;
  ucon[3] = pr[U3] - lapse * gamma * q.n03;
}

// bcon_calc_g (u2p_util.c:241-259), ncov = (-lapse, 0, 0, 0)
__device__ __forceinline__ void bcon_calc_g(const double *pr, const double *ucon, const double *ucov, double ncov0,
                                            double *bcon)
{
  double Bc1 = -ncov0 * pr[B1], Bc2 = -ncov0 * pr[B2], Bc3 = -ncov0 * pr[B3];
  double udB = 0.;
  udB += ucov[0] * 0.;
  udB += ucov[1] * Bc1;
  udB += ucov[2] * Bc2;
  udB += ucov[3] * Bc3;
  double gamma = -ucon[0] * ncov0;
  bcon[0] = (0. + ucon[0] * udB) / gamma;
  bcon[1] = (Bc1 + ucon[1] * udB) / gamma;
  bcon[2] = (Bc2 + ucon[2] * udB) / gamma;
  bcon[3] = (Bc3 + ucon[3] * udB) / gamma;
}

// gamma_calc_g (u2p_util.c:277-300); returns 1 (gamma untouched) for utsq < -1e-10
__device__ __forceinline__ int gamma_calc_g(const double *pr, const Geo &q, double &gamma)
{
  double utsq = q.v11 * pr[U1] * pr[U1] + q.v22 * pr[U2] * pr[U2] + q.v33 * pr[U3] * pr[U3]
                + 2. * (0. * pr[U1] * pr[U2] + q.v13 * pr[U1] * pr[U3] + 0. * pr[U2] * pr[U3]);
  if (utsq < 0.0) {
    if (fabs(utsq) > 1.E-10) return 1;
    else utsq = fabs(utsq);
  }
  gamma = sqrt(1. + utsq);
  return 0;
}

// primtoU_g with COOL_EOS (u2p_util.c:80-140)
static __device__ __noinline__ void primtoU_g_cool(const EosDev &E, EosCursor &c, const double *prim, const Geo &q, double *U)
{
  double ucon[4], ucov[4], bcon[4], bcov[4];
  const double alpha = 1.0 / sqrt(-q.n00);
  ucon_calc_g(prim, q, ucon);
  lower(ucon, q, ucov);
  const double ncov0 = -sqrt(-1. / q.n00);
  const double gamma = -ncov0 * ucon[0];
  bcon_calc_g(prim, ucon, ucov, ncov0, bcon);
  lower(bcon, q, bcov);
  double n_dot_b = 0.;
  n_dot_b += ncov0 * bcon[0];
  n_dot_b += 0. * bcon[1];
  n_dot_b += 0. * bcon[2];
  n_dot_b += 0. * bcon[3];
  double bsq = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++) bsq += bcov[i] * bcon[i];
  const double rho0 = prim[RHO], u = prim[UU];
  const double p = eos_pressure(E, c, rho0, u);
  const double w = rho0 + u + p;
  U[RHO] = ucon[0] * rho0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const double ncovi = i == 0 ? ncov0 : 0.;
    U[UU + i] = gamma * (w + bsq) * ucov[i] - (p + bsq / 2.) * ncovi + n_dot_b * bcov[i];
    U[UU + i] /= alpha;
  }
  U[UU] = U[UU] + U[RHO];
  U[B1] = prim[B1];
  U[B2] = prim[B2];
  U[B3] = prim[B3];
#pragma unroll
  for (int i = 0; i < 8; i++) U[i] *= q.g;
}

// full gcov[j][k] of a Geo (structural zeros as 0.)
__device__ __forceinline__ double gcov_at(const Geo &q, int j, int k)
{
  const int a = j < k ? j : k, b = j < k ? k : j;
  if (a == 0) return b == 0 ? q.v00 : b == 1 ? q.v01 : b == 3 ? q.v03 : 0.;
  if (a == 1) return b == 1 ? q.v11 : b == 3 ? q.v13 : 0.;
  if (a == 2) return b == 2 ? q.v22 : 0.;
  return q.v33;
}

// ---------------------------------------------------------------------------
// Utoprim_5d (utoprim_5d.c:179-982)

constexpr double U5_TOL_RESID = 1.e-4;
constexpr double U5_NUMEPSILON = 2.2204460492503131e-16;

// dudp_calc_g (utoprim_5d.c:409-528): Am = dU(1-5)/dp(1-5)
static __device__ __noinline__ void dudp_calc_g(const EosDev &E, EosCursor &c, const double *pr, const Geo &q,
                                         double Am[5][5])
{
  double ucon[4], ucov[4], bcon[4], bcov[4];
  double tempA[5][5];
#pragma unroll
  for (int j = 0; j < 5; j++)
#pragma unroll
    for (int k = 0; k < 5; k++) tempA[j][k] = Am[j][k] = 0.;
  ucon_calc_g(pr, q, ucon);
  lower(ucon, q, ucov);
  const double ncov0 = -sqrt(-1. / q.n00);
  bcon_calc_g(pr, ucon, ucov, ncov0, bcon);
  lower(bcon, q, bcov);
  const double bsq = dot4(bcon, bcov);
  // dutdui_calc_g (:563-570)
  double dutdui[4];
  dutdui[0] = 0.;
#pragma unroll
  for (int j = 1; j < 4; j++) dutdui[j] = -ucov[j] / ucov[0];
  // dbtdui_calc_g (:572-585)
  double dbtdui[4];
  {
    double Bv[4] = {0., pr[B1], pr[B2], pr[B3]}, Bcov[4];
    lower(Bv, q, Bcov);
    dbtdui[0] = 0.;
#pragma unroll
    for (int j = 1; j < 4; j++) dbtdui[j] = Bcov[j] + Bcov[0] * dutdui[j];
  }
  // dbiduj_calc_g (:587-602)
  double dbiduj[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 0; k < 4; k++) dbiduj[j][k] = 0.;
#pragma unroll
  for (int j = 1; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++) dbiduj[j][k] = -bcon[j] * dutdui[k] / ucon[0] + ucon[j] * dbtdui[k] / ucon[0];
#pragma unroll
  for (int j = 1; j < 4; j++) dbiduj[j][j] += bcon[0] / ucon[0];
#pragma unroll
  for (int j = 1; j < 4; j++) dbiduj[0][j] = dbtdui[j];
  // dbsqdui_calc_g (:604-613)
  double dbsqdui[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    dbsqdui[j] = 0.;
#pragma unroll
    for (int k = 0; k < 4; k++) dbsqdui[j] += 2. * bcov[k] * dbiduj[k][j];
  }
  // dudduu_calc_g (:615-620) and dbdiduj_calc_g (:625-631), spatial k
  double dudduu[4][4], dbdiduj[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++) {
      dudduu[j][k] = gcov_at(q, j, k) + gcov_at(q, j, 0) * dutdui[k];
      double s = 0.;
#pragma unroll
      for (int l = 0; l < 4; l++) s += gcov_at(q, j, l) * dbiduj[l][k];
      dbdiduj[j][k] = s;
    }
  const double eta = pr[RHO] + pr[UU] + eos_pressure(E, c, pr[RHO], pr[UU]) + bsq;
  Am[RHO][RHO] = ucon[0];
  const double dpdrho = eos_dpdrho(E, c, pr[RHO], pr[UU]);
#pragma unroll
  for (int j = 0; j < 4; j++) Am[UU + j][RHO] = (1.0 + dpdrho) * ucon[0] * ucov[j] + (j == 0 ? 1. : 0.) * dpdrho;
  Am[RHO][UU] = 0.0;
  const double dpdu = eos_dpdu(E, c, pr[RHO], pr[UU]);
#pragma unroll
  for (int j = 0; j < 4; j++) Am[UU + j][UU] = (1.0 + dpdu) * ucon[0] * ucov[j] + (j == 0 ? 1. : 0.) * dpdu;
#pragma unroll
  for (int j = 1; j < 4; j++) Am[RHO][U1 + j - 1] = pr[RHO] * dutdui[j];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int k = 1; k < 4; k++)
      Am[UU + j][U1 + k - 1] = dbsqdui[k] * ucon[0] * ucov[j] + eta * (dutdui[k] * ucov[j] + ucon[0] * dudduu[j][k])
                               + (j == 0 ? 1. : 0.) * 0.5 * dbsqdui[k] - (dbtdui[k] * bcov[j] + bcon[0] * dbdiduj[j][k]);
#pragma unroll
  for (int k = 0; k < 5; k++) Am[UU][k] += Am[RHO][k];
  // dgdvi_calc_g (:531-544); gamma is left unset by a failing gamma_calc_g in
  // the reference, NaN here
  double gamma = CUDART_NAN;
  gamma_calc_g(pr, q, gamma);
  double dgdvi[4];
#pragma unroll
  for (int j = 1; j < 4; j++) {
    dgdvi[j] = 0.;
#pragma unroll
    for (int k = 1; k < 4; k++) dgdvi[j] += 1.0 / gamma * gcov_at(q, j, k) * pr[U1 + k - 1];
  }
  // duidvj_calc_g (:546-561), spatial rows
  double duidvj[4][4];
  {
    const double alpha = 1.0 / sqrt(-q.n00);
    const double betacon[4] = {0., q.n01 * alpha * alpha, 0. * alpha * alpha, q.n03 * alpha * alpha};
#pragma unroll
    for (int j = 1; j < 4; j++)
#pragma unroll
      for (int k = 1; k < 4; k++) duidvj[j][k] = (j == k ? 1. : 0.) - betacon[j] / alpha * dgdvi[k];
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    tempA[i][RHO] = Am[i][RHO];
    tempA[i][UU] = Am[i][UU];
  }
#pragma unroll
  for (int i = 0; i < 5; i++)
#pragma unroll
    for (int j = 1; j < 4; j++)
#pragma unroll
      for (int l = 1; l <= 3; l++) tempA[RHO + i][U1 + j - 1] += Am[RHO + i][U1 + l - 1] * duidvj[l][j];
#pragma unroll
  for (int i = 0; i < 5; i++)
#pragma unroll
    for (int j = 0; j < 5; j++) Am[i][j] = tempA[i][j] * q.g;
}

// LU_decompose (utoprim_5d.c:657-829): Crout with implicit partial pivoting;
// max_row carries over between columns as in the reference
__device__ __forceinline__ int lu_decompose5(double A[5][5], int permute[5])
{
  const double absmin = 1e-30;
  double row_norm[5];
  int max_row = 0;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    double absmax = 0.;
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double m = fabs(A[i][j]);
      if (m > absmax) absmax = m;
    }
    if (absmax == 0.) return 1;
    row_norm[i] = 1. / absmax;
  }
#pragma unroll
  for (int j = 0; j < 5; j++) {
#pragma unroll
    for (int i = 0; i < j; i++)
#pragma unroll
      for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
    double absmax = 0.0;
#pragma unroll
    for (int i = j; i < 5; i++) {
#pragma unroll
      for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
      double m = fabs(A[i][j]) * row_norm[i];
      if (m >= absmax) { absmax = m; max_row = i; }
    }
    if (max_row != j) {
      if ((j == 3) && (A[j][j + 1] == 0.)) {
        max_row = j;
      } else {
        // (max_row < j only when a column held no comparable entry and the
        // previous column's choice carried over)
#pragma unroll
        for (int r = 0; r < 5; r++)
          if (r != j && r == max_row) {
#pragma unroll
            for (int k = 0; k < 5; k++) { double t = A[j][k]; A[j][k] = A[r][k]; A[r][k] = t; }
            row_norm[r] = row_norm[j];
          }
      }
    }
    permute[j] = max_row;
    if (A[j][j] == 0.) A[j][j] = absmin;
    if (j != 4) {
      double t = 1. / A[j][j];
#pragma unroll
      for (int i = j + 1; i < 5; i++) A[i][j] *= t;
    }
  }
  return 0;
}

// LU_substitution (utoprim_5d.c:832-880)
__device__ __forceinline__ void lu_substitute5(const double A[5][5], double B[5], const int permute[5])
{
#pragma unroll
  for (int i = 0; i < 5; i++) {
    double t = 0.;
#pragma unroll
    for (int r = 0; r < 5; r++) if (r == permute[i]) t = B[r];
#pragma unroll
    for (int r = 0; r < 5; r++) if (r == permute[i]) B[r] = B[i];
#pragma unroll
    for (int j = i - 1; j >= 0; j--) t -= A[i][j] * B[j];
    B[i] = t;
  }
#pragma unroll
  for (int i = 4; i >= 0; i--) {
#pragma unroll
    for (int j = i + 1; j < 5; j++) B[i] -= A[i][j] * B[j];
    B[i] /= A[i][i];
  }
}

struct U5Target {
  double U[8];
};

// func_5d (utoprim_5d.c:250-365): residual, its norm f and df, and the Newton step
static __device__ __noinline__ void func_5d(const EosDev &E, EosCursor &c, const U5Target &T, const Geo &q,
                                     const double *prguess, double *dxm, double &f, double &df)
{
  double pr[8], U_curr[8], Am[5][5], beta[5];
  int permute[5] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 5; i++) pr[i] = prguess[i];
#pragma unroll
  for (int i = 5; i < 8; i++) pr[i] = T.U[i] / q.g;
  primtoU_g_cool(E, c, pr, q, U_curr);
  dudp_calc_g(E, c, pr, q, Am);
  double norm = 0.0;
  int numnormterms = 0;
#pragma unroll
  for (int j = 0; j < 5; j++)
#pragma unroll
    for (int k = 0; k < 5; k++)
      if (Am[j][k] > U5_NUMEPSILON) {
        norm += fabs(Am[j][k]);
        numnormterms++;
      }
  norm = ((double)(numnormterms)) / (norm);
#pragma unroll
  for (int j = 0; j < 5; j++)
#pragma unroll
    for (int k = 0; k < 5; k++) Am[j][k] *= (norm);
  double residnorm;
  df = residnorm = 0.;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const double resid = U_curr[k] - T.U[k];
    beta[k] = -resid * (norm);
    residnorm = 0.5 * (fabs(U_curr[k]) + fabs(T.U[k]));
    residnorm = (residnorm == 0.) ? 1. : 1. / residnorm;
    df -= residnorm * resid * resid;
  }
  f = -0.5 * (df);
#pragma unroll
  for (int i = 0; i < 5; i++) dxm[i] = beta[i];
  lu_decompose5(Am, permute);
  lu_substitute5(Am, dxm, permute);
}

// calc_errx_5d with COOL_EOS (utoprim_5d.c:372-392)
__device__ __forceinline__ void calc_errx_5d(const EosDev &E, EosCursor &c, const Geo &q, const double *x,
                                             double &W, double &vsq)
{
  const double v1 = x[U1], v2 = x[U2], v3 = x[U3];
  vsq = 0.;
  vsq += q.v11 * v1 * v1;
  vsq += q.v13 * v1 * v3;
  vsq += q.v22 * v2 * v2;
  vsq += q.v13 * v3 * v1;
  vsq += q.v33 * v3 * v3;
  const double gsqtmp = 1. + vsq;
  vsq /= gsqtmp;
  W = gsqtmp * (x[UU] + x[RHO] + eos_pressure(E, c, x[RHO], x[UU]));
}

// Utoprim_5d (utoprim_5d.c:179-245) with general_newton_raphson (:887-982)
static __device__ __noinline__ int utoprim_5d(const EosDev &E, EosCursor &c, const double *U, const Geo &q, double *prim)
{
  U5Target T;
#pragma unroll
  for (int k = 0; k < 8; k++) T.U[k] = U[k];
#pragma unroll
  for (int k = B1; k <= B3; k++) prim[k] = U[k] / q.g;
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = prim[k];
  // general_newton_raphson(x, 5, func_5d)
  double errx = 1., f = 1., df = 1.;
  int i_extra = 0, doing_extra = 0;
  double vsq = 0., W = 0., W_old = 0.;
  int n_iter = 0;
  bool keep_iterating = true;
  while (keep_iterating) {
    double dx[5];
    func_5d(E, c, T, q, x, dx, f, df);
#pragma unroll
    for (int id = 0; id < 5; id++) x[id] += dx[id];
    W_old = W;
    calc_errx_5d(E, c, q, x, W, vsq);
    errx = (W == 0.) ? fabs(W - W_old) : fabs((W - W_old) / W);
    if ((fabs(errx) <= NEWT_TOL) && (f <= U5_TOL_RESID) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0))
      doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep_iterating = false;
    n_iter++;
  }
  int ret;
  if (!isfinite(f) || !isfinite(df)) ret = 2;
  else if ((fabs(errx) > MIN_NEWT_TOL) || (f > U5_TOL_RESID)) ret = 1;
  else ret = 0;
  if (ret) return 100 * ret + 1;
  if ((x[RHO] < 0.0) || (x[UU] < 0.0)) return 5;
  double gamma_tmp;
  if (gamma_calc_g(x, q, gamma_tmp) == 1) return 4;
#pragma unroll
  for (int k = 0; k < 8; k++) prim[k] = x[k];
  return 0;
}

}  // namespace harm
