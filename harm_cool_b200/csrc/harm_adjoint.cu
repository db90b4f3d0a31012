// Discrete adjoint of K steps of step_ch() (2D, gamma-law, FP64).
//
// Objective: the mass that crosses the inner radial boundary during the K
// steps, J = sum_n dt^n din^n -- the reference's mass_in (diag.c:578,
// mass_in += mdot_in*Dt), din^n = sum_j rho u^1 sqrt(-g) dx2 dx3 over the
// inner ghost row of the step's result (diag_mass, MDOTTYPE NEU_AGA_GHOST1,
// diag.c:486-515).  Output: dJ/dp of the state the K steps start from, every
// cell of every primitive (ghost cells included, since the first step's
// stencils read them).
//
// Method.  The state p^n of every checkpoint_every-th step is kept on a forward
// pass; the reverse sweep recomputes each segment from its checkpoint with the
// step's own kernels (exact::launch_step_rec), keeping the intermediates of
// every step (StepRec), and then walks the steps backwards.  The recomputation
// of one segment runs on the context's stream while the next is reversed on
// another.  Each part of a step is transposed where it is linear (flux-CT
// averaging, the flux divergence, bound_prim copies, fixup_utoprim stencils).
// The face fluxes (get_state, primtoflux, vchar and the Lax-Friedrichs
// combination), primtoU, the connection source and fixup()'s floors (outside
// its drift-frame branch) are differentiated by hand in reverse mode.  The
// limiter, inflow_check(), the objective, the drift-frame floors and the
// fall-back inversions are linearised with forward-mode dual numbers
// (harm_dual.cuh).  Limiter branches, clamps and the wave-speed choice are
// frozen at the forward's.  The inversion is differentiated through its
// converged solution by the implicit-function theorem: Utoprim_2d's Newton
// residuals vanish at the converged (W, v^2), so its adjoint is a transposed
// 2x2 solve; the isentropic fall-backs replace primtoU's energy row by their
// constraint u = K rho^gam/(gam-1), an 8x8 solve.  A zone whose inversion
// failed keeps its guess (the step's p^n) and U[B]/gdet.  The time step is
// part of the chain: dt^{n+1} = min(ndt, 1.3 dt^n) with ndt = defcon/(1/n1 +
// 1/n2) and n_d the Courant minimum over the corrector's faces
// (step_ch.c:126-137, 477-484), so the face that set each minimum gets the
// adjoint of its wave speed.
//
// Every kernel of the reverse sweep reads recorded values only.  The values
// the dual numbers carry, and those the reverse-mode routines recompute, are
// the step's own (the same IEEE operations), so every branch the
// linearisation takes is the branch the step took.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "harm_common.cuh"
#include "harm_bound.cuh"
#include "harm_dual.cuh"

namespace harm {
namespace adj {

constexpr int FU_THREADS = 1024;
enum { ERR_FAILS = 1, ERR_SINGULAR = 2 };

using D8 = Dual<8>;

// the adjoint's scalar chain through the time step, kept on the device
struct AdjScalars {
  double lam_dt_next;  // dJ/d dt^{n+1} (all later steps)
  double ln[2];        // adjoints of the corrector's Courant minima n1, n2
  double lDt[2];       // dJ/dDt of the predictor's and the corrector's update
  int claim[2];        // the face that set each minimum has been found
};

// before step n's reverse (run by k_adj_din_bound): dt^{n+1} = min(ndt, 1.3 dt^n),
// ndt = defcon / (1/n1 + 1/n2) (step_ch.c:126-137); sa is the run state before
// k_finalize, sb after
__device__ __forceinline__ void adj_dt_pre(const DevScalars *sa, const DevScalars *sb, double defcon, AdjScalars *a)
{
  const double dt = sa->dt, ndt = sb->ndt;
  const double n1 = __longlong_as_double((long long)sa->ndt_bits[0]);
  const double n2 = __longlong_as_double((long long)sa->ndt_bits[1]);
  const double lam_ndt = ndt > SAFE * dt ? 0. : a->lam_dt_next;
  const double S = 1. / n1 + 1. / n2;
  a->ln[0] = lam_ndt * defcon / (n1 * n1) / (S * S);
  a->ln[1] = lam_ndt * defcon / (n2 * n2) / (S * S);
  a->lDt[0] = a->lDt[1] = 0.;
  a->claim[0] = a->claim[1] = 0;
}

// after it: dJ/d dt^n = din^n (J = sum dt din) + the ramp + both updates' Dt
__global__ void k_adj_dt_post(const DevScalars *sa, const DevScalars *sb, AdjScalars *a)
{
  const double dt = sa->dt, ndt = sb->ndt;
  double l = sb->mdot_in + 0.5 * a->lDt[0] + a->lDt[1];
  if (ndt > SAFE * dt) l += SAFE * a->lam_dt_next;
  a->lam_dt_next = l;
}

// ---------------------------------------------------------------------------
// objective: dt^n * din^n on the inner ghost row of p^{n+1} (diag.c:499)

// the seed of one inner ghost cell (i = istart - 1, active j), weight w = dt^n
__device__ __forceinline__ void din_seed(const Grid &G, const double *__restrict__ P, const double *__restrict__ geo,
                                         double *lam, int j, double w)
{
  const int i = G.istart - 1;
  const long c = cidx(G, 0, i, j);
  D8 pr[8];
#pragma unroll
  for (int k = 0; k < 8; k++) pr[k] = D8::seed(P[k * G.nc + c], k);
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, (long)i * G.sn2 + j, q);
  D8 ucon[4];
  int fail = 0;
  ucon_calc(pr, q, ucon, &fail);
  D8 term = pr[RHO] * ucon[1] * q.g * G.dx2 * G.dx3;
#pragma unroll
  for (int k = 0; k < 8; k++) lam[k * G.nc + c] += w * term.d[k];
}

// ---------------------------------------------------------------------------
// bound_prim (bounds.c:54-331) transposed: each ghost cell's adjoint goes to
// the active cell it was copied from, through the sign flips and
// inflow_check(); the ghost's own adjoint ends (its old value was overwritten).
// X holds the values bound_prim copied (its active cells).

__device__ __forceinline__ void bound_rev_cell(const Grid &G, const double *__restrict__ X,
                                               const double *__restrict__ geo, double *lam, int t)
{
  BoundCell b = bound_cell(G, t, 4);
  const int i = b.i, j = b.j;
  const bool rghost = i < G.istart || i > G.istop;
  const int ci = i < G.istart ? G.istart : (i > G.istop ? G.istop : i);
  int js = j;
  bool flip = false;
  if (j >= G.jstart && j <= G.jstop) {
    if (!rghost) return;
  } else {
    const bool low = j < G.jstart;
    js = low ? (j == G.jstart - 1 ? G.jstart : G.jstart + 1) : (j == G.jstop + 1 ? G.jstop : G.jstop - 1);
    flip = true;
  }
  const long c = cidx(G, 0, i, j), cs = cidx(G, 0, ci, js);
  double lg[8], lv[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    lg[k] = lam[k * G.nc + c];
    lam[k * G.nc + c] = 0.;
  }
  if (rghost) {
    D8 v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      double s = X[k * G.nc + cs];
      if (flip && (k == U2 || k == B2)) s *= -1.;
      v[k] = D8::seed(s, k);
    }
    Geo q;
    load_geo(geo_at(geo, G, L_CENT), G.ng, (long)i * G.sn2 + j, q);
    int fail = 0;
    inflow_check(v, q, i < G.istart ? 0 : 1, &fail);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      double s = 0.;
#pragma unroll
      for (int o = 0; o < 8; o++) s += lg[o] * v[o].d[k];
      lv[k] = s;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) lv[k] = lg[k];
  }
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double s = (flip && (k == U2 || k == B2)) ? -lv[k] : lv[k];
    if (s != 0.) atomicAdd(&lam[k * G.nc + cs], s);
  }
}

__global__ void k_adj_bound(Grid G, const double *__restrict__ X, const double *__restrict__ geo, double *lam)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 4 * G.sn2 + 4 * (G.sn1 - 4)) bound_rev_cell(G, X, geo, lam, t);
}

// The start of one step's reverse: the time step's chain (adj_dt_pre), the
// objective's seed dt^n d(rho u^1 sqrt(-g))/dp on the inner ghost row of the
// step's result P, and the transpose of the bound_prim that produced those
// ghosts -- each ghost cell seeded and transposed by the same thread.
__global__ void k_adj_din_bound(Grid G, const double *__restrict__ P, const double *__restrict__ geo, double *lam,
                                const DevScalars *sa, const DevScalars *sb, AdjScalars *as)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) adj_dt_pre(sa, sb, G.defcon, as);
  if (t >= 4 * G.sn2 + 4 * (G.sn1 - 4)) return;
  const BoundCell b = bound_cell(G, t, 4);
  if (b.i == G.istart - 1 && b.j >= G.jstart && b.j <= G.jstop) din_seed(G, P, geo, lam, b.j, sa->dt);
  bound_rev_cell(G, P, geo, lam, t);
}

// ---------------------------------------------------------------------------
// fixup_utoprim (fixup.c:432-538) transposed.  One block: the failed zones of
// the half step (pflag != 0 after the first bound_prim) are listed in loop
// order, the repairs are replayed on a working copy exactly as the step made
// them (each stencil chosen from the flags as earlier repairs left them), and
// then undone in reverse order, so a last-resort average that read an earlier
// repair passes its adjoint on to that repair's stencil.  The kernel then
// transposes the bound_prim that came before the repairs (the repairs may
// read ghost cells).  Without a repair the ghosts' adjoint is already zero
// (the later bound_prim's transpose cleared it), so that bound_prim's
// transpose has nothing to do either: the kernel returns at once when the
// count of failed zones the recomputed step kept (nfail) is zero.

__global__ void __launch_bounds__(FU_THREADS) k_adj_fixup_bound(Grid G, const double *__restrict__ X1,
                                                                  const signed char *__restrict__ fl1,
                                                                  const double *__restrict__ geo,
                                                                  const double *__restrict__ floors, double *W,
                                                                  signed char *Wf, int *list, double *vbuf,
                                                                  signed char *kinds, double *lam, int *err,
                                                                  const int *__restrict__ nfail)
{
  __shared__ int cnt[FU_THREADS];
  __shared__ int nsh;
  const int tid = threadIdx.x;
  // the step's fixup_utoprim met no failed zone (its count, kept by the recomputation)
  if (*nfail == 0) return;
  const long nact = (long)G.n1 * G.n2;
  const long per = (nact + FU_THREADS - 1) / FU_THREADS;
  const long a0 = tid * per, a1 = a0 + per < nact ? a0 + per : nact;
  int m = 0;
  for (long t = a0; t < a1; t++) {
    const int i = G.istart + (int)(t / G.n2), j = G.jstart + (int)(t % G.n2);
    if (fl1[cidx(G, 0, i, j)] != 0) m++;
  }
  cnt[tid] = m;
  __syncthreads();
  if (tid == 0) {
    int s = 0;
    for (int k = 0; k < FU_THREADS; k++) {
      const int v = cnt[k];
      cnt[k] = s;
      s += v;
    }
    nsh = s;
  }
  __syncthreads();
  const int n = nsh;
  if (n == 0) return;
  if (n > FAIL_CAP) {
    if (tid == 0) atomicOr(err, ERR_FAILS);
    return;
  }
  int o = cnt[tid];
  for (long t = a0; t < a1; t++) {
    const int i = G.istart + (int)(t / G.n2), j = G.jstart + (int)(t % G.n2);
    const long c = cidx(G, 0, i, j);
    if (fl1[c] != 0) list[o++] = (int)c;
  }
  for (long c = tid; c < G.nc; c += FU_THREADS) {
#pragma unroll
    for (int k = 0; k < 8; k++) W[k * G.nc + c] = X1[k * G.nc + c];
    Wf[c] = (signed char)(!fl1[c]);  // k_fu_flip
  }
  __syncthreads();
  if (tid == 0) {
    const double *gC = geo_at(geo, G, L_CENT);
    for (int t = 0; t < n; t++) {
      const long c = list[t];
      const int kind = stencil_kind(G, Wf, c);
      double v[8];
      repair_zone(G, W, c, kind, v);
      for (int k = 0; k < 8; k++) vbuf[(long)t * 8 + k] = v[k];
      kinds[t] = (signed char)kind;
      const int i = (int)((c / G.sn2) % G.sn1), j = (int)(c % G.sn2);
      const long gi = (long)i * G.sn2 + j;
      Geo q;
      load_geo(gC, G.ng, gi, q);
      int fail = 0;
      const bool g33 = fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail);
      for (int k = 0; k < 8; k++) W[k * G.nc + c] = v[k];
      Wf[c] = g33 ? (signed char)-33 : (signed char)0;
    }
    const long s = G.sn2;
    for (int t = n - 1; t >= 0; t--) {
      const long c = list[t];
      const int kind = kinds[t];
      const int i = (int)((c / G.sn2) % G.sn1), j = (int)(c % G.sn2);
      const long gi = (long)i * G.sn2 + j;
      Geo q;
      load_geo(gC, G.ng, gi, q);
      D8 v[8];
      for (int k = 0; k < 8; k++) v[k] = D8::seed(vbuf[(long)t * 8 + k], k);
      int fail = 0;
      fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail);
      double lo[8], lv[8];
      for (int k = 0; k < 8; k++) lo[k] = lam[k * G.nc + c];
      for (int k = 0; k < 8; k++) {
        double a = 0.;
        for (int r = 0; r < 8; r++) a += lo[r] * v[r].d[k];
        lv[k] = a;
      }
      // the repair keeps the zone's fields and replaces the rest
      for (int k = 0; k < 8; k++) lam[k * G.nc + c] = k >= B1 ? lv[k] : 0.;
      if (kind == 0) {
        for (int k = 0; k < B1; k++) {
          double *L = lam + k * G.nc;
          const double a = 0.25 * lv[k];
          L[c + 1] += a; L[c - 1] += a; L[c - s] += a; L[c + s] += a;
        }
      } else if (kind == 1) {
        for (int k = 0; k < B1; k++) {
          double *L = lam + k * G.nc;
          const double a = 0.25 * lv[k];
          L[c + s + 1] += a; L[c + s - 1] += a; L[c - s + 1] += a; L[c - s - 1] += a;
        }
      } else {
        for (int k = RHO; k <= UU; k++) {
          double *L = lam + k * G.nc;
          const double a = 0.5 * 0.25 * lv[k];
          L[c + 1] += a; L[c - 1] += a; L[c - s] += a; L[c + s] += a;
          L[c + s + 1] += a; L[c + s - 1] += a; L[c - s + 1] += a; L[c - s - 1] += a;
        }
      }
    }
  }
  __syncthreads();
  // the bound_prim before the repairs, transposed
  for (int t = tid; t < 4 * G.sn2 + 4 * (G.sn1 - 4); t += FU_THREADS) bound_rev_cell(G, X1, geo, lam, t);
}

// ---------------------------------------------------------------------------
// Reverse mode, differentiated by hand, of the state routines the update and
// the face fluxes use.  Values are recomputed with the step's own routines, so
// every clamp and selection takes the step's branch; a clamped quantity passes
// no derivative.

// adjoints of get_state's outputs and of the primitives read directly
struct StateAdj {
  double uc[4], ucv[4], bc[4], bcv[4], rho, u, bsq;
};

__device__ __forceinline__ void adj_zero(StateAdj &a)
{
#pragma unroll
  for (int k = 0; k < 4; k++) a.uc[k] = a.ucv[k] = a.bc[k] = a.bcv[k] = 0.;
  a.rho = a.u = a.bsq = 0.;
}

// one row T^d_j of mhd_calc (phys.c:143-161), given its adjoint am[j]; eta is
// the row's rho + u + p + b^2
__device__ __forceinline__ void mhd_rev(double gam, const StateT<double> &s, double eta, int d, const double *am,
                                        StateAdj &a)
{
  double aeta = 0.;
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    aeta += am[jj] * s.ucon[d] * s.ucov[jj];
    a.uc[d] += am[jj] * eta * s.ucov[jj];
    a.ucv[jj] += am[jj] * eta * s.ucon[d];
    a.bc[d] -= am[jj] * s.bcov[jj];
    a.bcv[jj] -= am[jj] * s.bcon[d];
  }
  const double aptot = am[d];  // ptot = p + b^2/2 on the diagonal
  a.bsq += aeta + 0.5 * aptot;
  a.rho += aeta;
  a.u += aeta + (gam - 1.) * (aeta + aptot);  // eta and ptot through p = (gam - 1) u
}

// primtoflux for direction d (phys.c:59-96), given the adjoint af of its result
__device__ __forceinline__ void flux_rev(double gam, const double *p, const Geo &q, const StateT<double> &s,
                                         double eta, int d, const double *af, StateAdj &a)
{
  double f[8];
#pragma unroll
  for (int k = 0; k < 8; k++) f[k] = af[k] * q.g;
  const double f0 = f[RHO] + f[UU];  // F[UU] = T^d_t + F[RHO]
  a.rho += f0 * s.ucon[d];
  a.uc[d] += f0 * p[RHO];
  mhd_rev(gam, s, eta, d, f + UU, a);
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {  // F[B_i] = b^i u^d - b^d u^i
    const double fb = f[B1 + ii - 1];
    a.bc[ii] += fb * s.ucon[d];
    a.uc[d] += fb * s.bcon[ii];
    a.bc[d] -= fb * s.ucon[ii];
    a.uc[ii] -= fb * s.bcon[d];
  }
}

// get_state (phys.c:219-252, 108-117, metric.c:210-231) and b^2 reversed:
// the primitives' adjoint ap
__device__ __forceinline__ void state_rev(const double *p, const Geo &q, const StateT<double> &s, StateAdj &a,
                                          double *ap)
{
  // b^2 = b^mu b_mu
#pragma unroll
  for (int k = 0; k < 4; k++) {
    a.bc[k] += a.bsq * s.bcov[k];
    a.bcv[k] += a.bsq * s.bcon[k];
  }
  // b_mu = lower(b^mu)
  a.bc[0] += q.v00 * a.bcv[0] + q.v01 * a.bcv[1] + q.v03 * a.bcv[3];
  a.bc[1] += q.v01 * a.bcv[0] + q.v11 * a.bcv[1] + q.v13 * a.bcv[3];
  a.bc[2] += q.v22 * a.bcv[2];
  a.bc[3] += q.v03 * a.bcv[0] + q.v13 * a.bcv[1] + q.v33 * a.bcv[3];
  // b^i = (B^i + b^t u^i) / u^t, b^t = B^i u_i
  double aBf[3], abt = a.bc[0];
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {
    aBf[ii - 1] = a.bc[ii] / s.ucon[0];
    abt += a.bc[ii] * s.ucon[ii] / s.ucon[0];
    a.uc[ii] += a.bc[ii] * s.bcon[0] / s.ucon[0];
    a.uc[0] -= a.bc[ii] * s.bcon[ii] / s.ucon[0];
  }
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {
    aBf[ii - 1] += abt * s.ucov[ii];
    a.ucv[ii] += abt * p[B1 + ii - 1];
  }
  // u_mu = lower(u^mu)
  a.uc[0] += q.v00 * a.ucv[0] + q.v01 * a.ucv[1] + q.v03 * a.ucv[3];
  a.uc[1] += q.v01 * a.ucv[0] + q.v11 * a.ucv[1] + q.v13 * a.ucv[3];
  a.uc[2] += q.v22 * a.ucv[2];
  a.uc[3] += q.v03 * a.ucv[0] + q.v13 * a.ucv[1] + q.v33 * a.ucv[3];
  // u^t = gamma / alpha, u^i = w^i - gamma beta^i / alpha (beta^2 = 0),
  // gamma = sqrt(1 + qsq) unless gamma_calc clamps qsq
  const double w1 = p[U1], w2 = p[U2], w3 = p[U3];
  const double qsq = q.v11 * w1 * w1 + q.v22 * w2 * w2 + q.v33 * w3 * w3 + 2. * (q.v13 * w1 * w3);
  const double alpha = q.alpha, b1 = q.n01 * alpha * alpha, b3 = q.n03 * alpha * alpha;
  const double gamma = s.ucon[0] * alpha;
  const double agam = a.uc[0] / alpha - a.uc[1] * b1 / alpha - a.uc[3] * b3 / alpha;
  const double aq = qsq < 0. ? 0. : agam * 0.5 / gamma;
  ap[RHO] = a.rho;
  ap[UU] = a.u;
  ap[U1] = a.uc[1] + aq * (2. * q.v11 * w1 + 2. * q.v13 * w3);
  ap[U2] = a.uc[2] + aq * 2. * q.v22 * w2;
  ap[U3] = a.uc[3] + aq * (2. * q.v33 * w3 + 2. * q.v13 * w1);
  ap[B1] = aBf[0];
  ap[B2] = aBf[1];
  ap[B3] = aBf[2];
}

// ---------------------------------------------------------------------------
// the inversion and fixup() of one zone (k_invert) transposed

// x with A^T x = b, A[o][k] row-major 8x8; Gaussian elimination with partial pivoting
__device__ bool solve8t(const double (*A)[8], const double *b, double *x)
{
  double M[8][9];
  for (int r = 0; r < 8; r++) {
    for (int c = 0; c < 8; c++) M[r][c] = A[c][r];
    M[r][8] = b[r];
  }
  for (int col = 0; col < 8; col++) {
    int piv = col;
    double best = fabs(M[col][col]);
    for (int r = col + 1; r < 8; r++)
      if (fabs(M[r][col]) > best) { best = fabs(M[r][col]); piv = r; }
    if (!(best > 0.)) return false;
    if (piv != col)
      for (int c = col; c < 9; c++) { double t = M[col][c]; M[col][c] = M[piv][c]; M[piv][c] = t; }
    for (int r = col + 1; r < 8; r++) {
      const double f = M[r][col] / M[col][col];
      for (int c = col; c < 9; c++) M[r][c] -= f * M[col][c];
    }
  }
  for (int r = 7; r >= 0; r--) {
    double s = M[r][8];
    for (int c = r + 1; c < 8; c++) s -= M[r][c] * x[c];
    x[r] = s / M[r][r];
  }
  return true;
}

// The adjoint of Utoprim_2d's result with respect to U (utoprim_2d.c:126-624),
// through the implicit-function theorem on its own two-variable Newton
// system: the residuals r1 = t11, r2 = t18 of func_vsq (utoprim_2d.c:562-624,
// gamma-law :645-678) vanish at the converged (W, v^2), which the returned
// primitives give back (rho = D sqrt(1 - v^2), u = (w - rho)/gam,
// W = w / (1 - v^2)).  lz: adjoint of the returned primitives z; lu: adjoint
// of the conserved variables U.
__device__ __forceinline__ void u2p_ift_rev(double gam, const double *U, const double *z, const Geo &q,
                                            const double *lz, double *lu)
{
  // the rescaled U and the scalars the inversion forms from it (utoprim_2d.c:126-176, 229-262)
  const double alpha = q.alpha, f = alpha / q.g;
  double Ut[8];
  Ut[RHO] = alpha * U[RHO] / q.g;
  Ut[UU] = alpha * (U[UU] - U[RHO]) / q.g;
#pragma unroll
  for (int k = U1; k <= B3; k++) Ut[k] = alpha * U[k] / q.g;
  U2P c;
  c.gam = gam;
  c.K_atm = 0.;
  double Bcon[4], Qcon[4], ncon[4], QdotB;
  u2p_scalars(c, Ut, q, Bcon, Qcon, ncon, QdotB);
  const double Bsq = c.Bsq, QdotBsq = c.QdotBsq, Qdotn = c.Qdotn, D = c.D;
  const double Qcov[4] = {Ut[UU], Ut[U1], Ut[U2], Ut[U3]};
  const double ncov0 = -sqrt(-1. / q.n00);
  // the converged W and v^2
  const double rho = z[RHO], u = z[UU];
  const double gtmp = rho / D, om = gtmp * gtmp, vsq = 1. - om, w = gam * u + rho, W = w / om;
  const double gamma = 1. / gtmp, WB = W + Bsq;
  double aD = 0., aW = 0., av = 0., aBsq = 0., aQdotB = 0., aQdotn = 0., agamma = 0.;
  double aQcon[4] = {0., 0., 0., 0.}, aBc[4] = {0., 0., 0., 0.};
  // u^i = gamma / (W + B^2) (Qt^i + (Q.B) B^i / W), Qt^i = Q^i + n^i (Q.n)  (u2p_velocities)
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {
    const double Qt = Qcon[ii] + ncon[ii] * Qdotn;
    const double X = Qt + QdotB * Bcon[ii] / W;
    const double ui = gamma / WB * X;
    const double a = lz[U1 + ii - 1];
    agamma += a * X / WB;
    aW -= a * ui / WB;
    aBsq -= a * ui / WB;
    const double aX = a * gamma / WB;
    aQcon[ii] += aX;
    aQdotn += aX * ncon[ii];
    aQdotB += aX * Bcon[ii] / W;
    aBc[ii] += aX * QdotB / W;
    aW -= aX * QdotB * Bcon[ii] / (W * W);
  }
  // u = (w - rho) / gam, rho = D gtmp, w = W (1 - v^2), gamma = 1 / gtmp, gtmp = sqrt(1 - v^2)
  const double aw = lz[UU] / gam, arho = lz[RHO] - lz[UU] / gam;
  aD += arho * gtmp;
  const double agtmp = arho * D - agamma / om;
  aW += aw * om;
  av -= aw * W + agtmp * 0.5 / gtmp;
  // implicit-function theorem: J^T mu = (aW, av), then a_theta = -(mu1 dr1/dtheta + mu2 dr2/dtheta)
  const double W2 = W * W, W3 = W2 * W;
  const double r1W = -2. * vsq * WB + 2. * QdotBsq / W2 - 2. * QdotBsq * (Bsq + 2. * W) / W3;
  const double r1v = -WB * WB;
  const double r2W = -QdotBsq / W3 - 1. + (gam - 1.) * om / gam;
  const double r2v = -0.5 * Bsq + (gam - 1.) * (0.5 * D / gtmp - W) / gam;
  const double det = r1W * r2v - r2W * r1v;
  const double mu1 = (aW * r2v - r2W * av) / det, mu2 = (r1W * av - r1v * aW) / det;
  const double aQtsq = -mu1;
  aBsq -= mu1 * (-2. * vsq * WB + QdotBsq / W2) - mu2 * 0.5 * (1. + vsq);
  const double aQdotBsq = -(mu1 * (Bsq + 2. * W) / W2 + mu2 * 0.5 / W2);
  aQdotn += mu2;
  aD += mu2 * (gam - 1.) * gtmp / gam;
  // Qtsq = Q.Q + (Q.n)^2, Q.n = Q^t n_t, (Q.B)^2
  aQdotB += 2. * QdotB * aQdotBsq;
  aQdotn += 2. * Qdotn * aQtsq;
  double aQcov[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    aQcov[m] = aQtsq * Qcon[m];
    aQcon[m] += aQtsq * Qcov[m];
  }
  aQcon[0] += aQdotn * ncov0;
  // Q^mu = g^{mu nu} Q_nu
  aQcov[0] += q.n00 * aQcon[0] + q.n10 * aQcon[1] + q.n30 * aQcon[3];
  aQcov[1] += q.n01 * aQcon[0] + q.n11 * aQcon[1] + q.n31 * aQcon[3];
  aQcov[2] += q.n22 * aQcon[2];
  aQcov[3] += q.n03 * aQcon[0] + q.n13 * aQcon[1] + q.n33 * aQcon[3];
  // Q.B = Q_i B^i and B^2 = B^i B_i (B^t = 0)
  const double Bcov[4] = {0., q.v11 * Bcon[1] + q.v13 * Bcon[3], q.v22 * Bcon[2], q.v13 * Bcon[1] + q.v33 * Bcon[3]};
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {
    aQcov[ii] += aQdotB * Bcon[ii];
    aBc[ii] += aQdotB * Qcov[ii] + 2. * aBsq * Bcov[ii];
  }
  // back to U: D = Ut[RHO], Q_t = Ut[UU], Q_i = Ut[U_i], B^i = Ut[B_i]; the fields' own prim[B] = U[B]/gdet
  lu[RHO] = f * (aD - aQcov[0]);
  lu[UU] = f * aQcov[0];
#pragma unroll
  for (int ii = 1; ii < 4; ii++) {
    lu[UU + ii] = f * aQcov[ii];
    lu[B1 + ii - 1] = f * aBc[ii] + lz[B1 + ii - 1] / q.g;
  }
}

// fixup1zone (fixup.c:142-383) reversed by hand where its drift-frame branch
// is not taken: the density and energy floors (each the largest of the radial
// floor, b^2 / BSQORHOMAX or BSQOUMAX, and for the density u / UORHOMAX) and
// the Lorentz-factor limit.  lz = (d fixup1zone / dz)^T lo.  Returns false,
// leaving lz alone, where the drift-frame branch applies.
__device__ __forceinline__ bool fixup_rev(double gam, double rho_floor, double uu_floor, const Geo &q,
                                          const double *z, const double *lo, double *lz)
{
  StateT<double> s;
  int fail = 0;
  get_state(z, q, s, &fail);
  const double bsq = dot4(s.bcon, s.bcov);
  double rflr = rho_floor, uflr = uu_floor;
  int rsrc = 0, usrc = 0;  // 0: the radial floor, 1: b^2, 2 (density only): u
  if (rflr < bsq / BSQORHOMAX) { rflr = bsq / BSQORHOMAX; rsrc = 1; }
  if (uflr < bsq / BSQOUMAX) { uflr = bsq / BSQOUMAX; usrc = 1; }
  if (rflr < z[UU] / UORHOMAX) { rflr = z[UU] / UORHOMAX; rsrc = 2; }
  const bool rfl = z[RHO] < rflr, ufl = z[UU] < uflr;
  const double r1 = rfl ? rflr : z[RHO], u1 = ufl ? uflr : z[UU];
  if ((rfl || ufl) && 10. * bsq / (r1 < u1 ? r1 : u1) - 1. > 0.) return false;
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = lo[k];
  // the Lorentz-factor limit: w^i -> f w^i, f = sqrt((GAMMAMAX^2 - 1) / qsq)
  const double w1 = z[U1], w2 = z[U2], w3 = z[U3];
  const double qsq = q.v11 * w1 * w1 + q.v22 * w2 * w2 + q.v33 * w3 * w3 + 2. * (q.v13 * w1 * w3);
  if (qsq >= 0. && sqrt(1. + qsq) > GAMMAMAX) {
    const double f = sqrt((GAMMAMAX * GAMMAMAX - 1.) / qsq);
    const double S = (a[U1] * w1 + a[U2] * w2 + a[U3] * w3) * (-0.5 * f / qsq);
    a[U1] = f * a[U1] + S * (2. * q.v11 * w1 + 2. * q.v13 * w3);
    a[U2] = f * a[U2] + S * 2. * q.v22 * w2;
    a[U3] = f * a[U3] + S * (2. * q.v33 * w3 + 2. * q.v13 * w1);
  }
  // the floors
  double absq = 0.;
  const double arho = a[RHO], auu = a[UU];
  if (rfl) {
    a[RHO] = 0.;
    if (rsrc == 1) absq += arho / BSQORHOMAX;
  }
  if (ufl) {
    a[UU] = 0.;
    if (usrc == 1) absq += auu / BSQOUMAX;
  }
  if (rfl && rsrc == 2) a[UU] += arho / UORHOMAX;
  if (absq != 0.) {
    StateAdj sa;
    adj_zero(sa);
    sa.bsq = absq;
    double ab[8];
    state_rev(z, q, s, sa, ab);
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] += ab[k];
  }
#pragma unroll
  for (int k = 0; k < 8; k++) lz[k] = a[k];
  return true;
}

// lz = (d fixup1zone / dz)^T lo for a zone the floors changed (dual numbers;
// out of line: most zones are left alone and skip it)
static __device__ __noinline__ void fixup_vjp(double gam, double rho_floor, double uu_floor, const Geo &q,
                                              const double *z, const double *lo, double *lz)
{
  D8 v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = D8::seed(z[k], k);
  int fail = 0;
  fixup1zone(gam, rho_floor, uu_floor, q, v, &fail);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double a = 0.;
#pragma unroll
    for (int o = 0; o < 8; o++) a += lo[o] * v[o].d[k];
    lz[k] = a;
  }
}

// A fall-back inversion's adjoint (Utoprim_1dvsq2fix1 / Utoprim_1dfix1 solve with
// u = K rho^gam / (gam - 1) in place of the energy equation): the
// implicit-function theorem on primtoU with that row replaced, an 8x8 solve.
// Rare, so kept out of line.
static __device__ __noinline__ bool ift_fallback(double gam, double K, const double *z, const Geo &q,
                                                 const double *lz, double *lu)
{
  double M[8][8];
  {
    D8 v[8], Uo[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = D8::seed(z[k], k);
    StateT<D8> s;
    int fail = 0;
    get_state(v, q, s, &fail);
    primtoflux(gam, v, s, 0, q.g, Uo);
#pragma unroll
    for (int o = 0; o < 8; o++)
#pragma unroll
      for (int k = 0; k < 8; k++) M[o][k] = Uo[o].d[k];
  }
#pragma unroll
  for (int k = 0; k < 8; k++) M[UU][k] = 0.;
  M[UU][UU] = 1.;
  M[UU][RHO] = -K * gam * pow(z[RHO], gam - 1.) / (gam - 1.);
  const bool ok = solve8t(M, lz, lu);
  lu[UU] = 0.;
  return ok;
}

// lamf: adjoint of the half step's output pf (its active cells are consumed);
// lamU: adjoint of the conserved variables the update formed; lampi: adjoint of
// the inversion's guess pi (a failed zone keeps it).  Zr, wz: the inversion's
// output before fixup() and which inversion gave it, as the step recorded them.
__global__ void __launch_bounds__(128) k_adj_invert(Grid G, const double *__restrict__ Ub,
                                                    const double *__restrict__ Zr,
                                                    const signed char *__restrict__ wz,
                                                    const double *__restrict__ geo, const double *__restrict__ floors,
                                                    const double *__restrict__ katm, double *lamf, double *lamU,
                                                    double *lampi, int *err)
{
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, 0, i, j);
  const long gi = (long)i * G.sn2 + j;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double z[8];
#pragma unroll
  for (int k = 0; k < 8; k++) z[k] = Zr[k * G.nc + c];
  const int w = wz[c];
  const int flag = w < 0, which = w < 0 ? 0 : w;
  const double K = katm[i];
  double lo[8], lz[8], lu[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    lo[k] = lamf[k * G.nc + c];
    lamf[k * G.nc + c] = 0.;
  }
  {
    // fixup() leaves most zones alone: there its Jacobian is the identity
    double v0[8];
    bool same = true;
#pragma unroll
    for (int k = 0; k < 8; k++) v0[k] = z[k];
    int fail = 0;
    fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v0, &fail);
#pragma unroll
    for (int k = 0; k < 8; k++) same &= v0[k] == z[k];
    if (same) {
#pragma unroll
      for (int k = 0; k < 8; k++) lz[k] = lo[k];
    } else if (!fixup_rev(G.gam, floors[gi], floors[G.ng + gi], q, z, lo, lz)) {
      fixup_vjp(G.gam, floors[gi], floors[G.ng + gi], q, z, lo, lz);
    }
  }
  if (flag == 0 && which == 0) {
    double U[8];
#pragma unroll
    for (int k = 0; k < 8; k++) U[k] = Ub[k * G.nc + c];
    u2p_ift_rev(G.gam, U, z, q, lz, lu);
  } else if (flag == 0) {
    if (!ift_fallback(G.gam, K, z, q, lz, lu)) {
      atomicOr(err, ERR_SINGULAR);
#pragma unroll
      for (int k = 0; k < 8; k++) lu[k] = 0.;
    }
  } else {
#pragma unroll
    for (int k = 0; k < B1; k++) {
      lampi[k * G.nc + c] += lz[k];
      lu[k] = 0.;
    }
#pragma unroll
    for (int k = B1; k < 8; k++) lu[k] = lz[k] / q.g;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) lamU[k * G.nc + c] = lu[k];
}

// source() (phys.c:165-207) reversed: dU_nu = g sum_{j,k} T^j_k conn[k][nu][j]
// for nu = t..phi in U[UU..U3]; w * lu is the adjoint of dU
__device__ __forceinline__ void source_rev(double gam, const Geo &q, const StateT<double> &s, double eta,
                                           const double *__restrict__ conn, long ng, long gi, const double *lu,
                                           double w, StateAdj &a)
{
#pragma unroll
  for (int jj = 0; jj < 4; jj++) {
    double am[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double x = 0.;
#pragma unroll
      for (int nu = 0; nu < 4; nu++) x += lu[UU + nu] * __ldg(conn + conn_slot(k, nu, jj) * ng + gi);
      am[k] = w * q.g * x;
    }
    mhd_rev(gam, s, eta, jj, am, a);
  }
}

// ---------------------------------------------------------------------------
// the update (k_cons: primtoU, source, flux-CT, flux divergence) transposed

// adjoint of one corner EMF (step_ch.c:546-547) onto the raw face fluxes,
// through fix_flux's polar reflection of F1[B2] (coord.c:284-301)
__device__ __forceinline__ void add_f1b2(const Grid &G, int i, int j, double a, double *lamF1)
{
  if (j == G.jstart - 1) atomicAdd(&lamF1[B2 * G.nc + cidx(G, 0, i, G.jstart)], -a);
  else if (j == G.jstop + 1) atomicAdd(&lamF1[B2 * G.nc + cidx(G, 0, i, G.jstop)], -a);
  else atomicAdd(&lamF1[B2 * G.nc + cidx(G, 0, i, j)], a);
}

__device__ __forceinline__ void emf_adjoint(const Grid &G, int i, int j, double l, double *lamF1, double *lamF2)
{
  if (l == 0.) return;
  const double a = 0.25 * l;
  add_f1b2(G, i, j, a, lamF1);
  add_f1b2(G, i, j - 1, a, lamF1);
  atomicAdd(&lamF2[B1 * G.nc + cidx(G, 0, i, j)], -a);
  atomicAdd(&lamF2[B1 * G.nc + cidx(G, 0, i - 1, j)], -a);
}

// U = primtoU(pi) + Dt (-dF1/dx1 - dF2/dx2 + source(pb)) (step_ch.c:247-263);
// FULL: the corrector (pi = p^n, pb = ph), whose source at ph is
// k_adj_source's, else the predictor (pi = pb = p^n)
template <bool FULL>
__global__ void __launch_bounds__(128) k_adj_cons(Grid G, const double *__restrict__ pi,
                                                  const double *__restrict__ Ub, const double *__restrict__ F1rho,
                                                  const double *__restrict__ geo, const double *__restrict__ conn,
                                                  const double *__restrict__ lamU, double *lampi, double *lamF1,
                                                  double *lamF2, const DevScalars *sa, AdjScalars *as)
{
  const double Dt = FULL ? sa->dt : 0.5 * sa->dt;
  double *lamDt = &as->lDt[FULL ? 1 : 0];
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  double lDt = 0.;
  if (i <= G.istop && j <= G.jstop) {
    const long c = cidx(G, 0, i, j);
    const long gi = (long)i * G.sn2 + j;
    Geo q;
    load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
    double lu[8], P0[8];
#pragma unroll
    for (int k = 0; k < 8; k++) lu[k] = lamU[k * G.nc + c];
    int fail = 0;
    {
      // primtoU at pi and, in the predictor (pi = pb), the source at the same state
      double pz[8];
#pragma unroll
      for (int k = 0; k < 8; k++) pz[k] = pi[k * G.nc + c];
      StateT<double> s;
      get_state(pz, q, s, &fail);
      primtoflux(G.gam, pz, s, 0, q.g, P0);
      const double eta = (G.gam - 1.) * pz[UU] + pz[RHO] + pz[UU] + dot4(s.bcon, s.bcov);
      StateAdj a;
      adj_zero(a);
      flux_rev(G.gam, pz, q, s, eta, 0, lu, a);
      if (!FULL) source_rev(G.gam, q, s, eta, conn, G.ng, gi, lu, Dt, a);
      double li[8];
      state_rev(pz, q, s, a, li);
#pragma unroll
      for (int k = 0; k < 8; k++) lampi[k * G.nc + c] += li[k];
    }
    // dU/dDt = (U - primtoU(pi)) / Dt, the step's own flux divergence plus source
#pragma unroll
    for (int o = 0; o < 8; o++) lDt += lu[o] * ((Ub[o * G.nc + c] - P0[o]) / Dt);

    // the zone's processed face fluxes
    const double a1 = Dt / G.dx1, a2 = Dt / G.dx2;
    double g1m[8], g1p[8], g2m[8], g2p[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      g1m[k] = lu[k] * a1;
      g1p[k] = -lu[k] * a1;
      g2m[k] = lu[k] * a2;
      g2p[k] = -lu[k] * a2;
    }
    // no inflow of mass through the radial boundaries (coord.c:307-321)
    if (i == G.istart && F1rho[cidx(G, 0, i, j)] > 0) g1m[RHO] = 0.;
    if (i == G.istop && F1rho[cidx(G, 0, i + 1, j)] < 0) g1p[RHO] = 0.;
    const long c1p = cidx(G, 0, i + 1, j), c2p = cidx(G, 0, i, j + 1);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      if (k == B1 || k == B2) continue;
      atomicAdd(&lamF1[k * G.nc + c], g1m[k]);
      atomicAdd(&lamF1[k * G.nc + c1p], g1p[k]);
      atomicAdd(&lamF2[k * G.nc + c], g2m[k]);
      atomicAdd(&lamF2[k * G.nc + c2p], g2p[k]);
    }
    // flux-CT (step_ch.c:514-629): f1m[B2] = (eA+eB)/2, f1p[B2] = (eC+eD)/2,
    // f2m[B1] = -(eA+eC)/2, f2p[B1] = -(eB+eD)/2 with the corner EMFs
    // A (i,j), B (i,j+1), C (i+1,j), D (i+1,j+1)
    emf_adjoint(G, i, j, 0.5 * g1m[B2] - 0.5 * g2m[B1], lamF1, lamF2);
    emf_adjoint(G, i, j + 1, 0.5 * g1m[B2] - 0.5 * g2p[B1], lamF1, lamF2);
    emf_adjoint(G, i + 1, j, 0.5 * g1p[B2] - 0.5 * g2m[B1], lamF1, lamF2);
    emf_adjoint(G, i + 1, j + 1, 0.5 * g1p[B2] - 0.5 * g2p[B1], lamF1, lamF2);
  }
  __shared__ double red[4];
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  double v = warp_sum(lDt);
  if ((t & 31) == 0) red[t >> 5] = v;
  __syncthreads();
  if (t == 0) atomicAdd(lamDt, (red[0] + red[1]) + (red[2] + red[3]));
}

// the corrector's source at pb = ph (its part of k_cons), reversed: the adjoint
// of ph gets dt (d source / d ph)^T lamU; runs beside k_adj_cons<true>
__global__ void __launch_bounds__(128) k_adj_source(Grid G, const double *__restrict__ pb,
                                                    const double *__restrict__ geo, const double *__restrict__ conn,
                                                    const double *__restrict__ lamU, double *lampb,
                                                    const DevScalars *sa)
{
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, 0, i, j);
  const long gi = (long)i * G.sn2 + j;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double lu[8], pz[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    lu[k] = lamU[k * G.nc + c];
    pz[k] = pb[k * G.nc + c];
  }
  StateT<double> s;
  int fail = 0;
  get_state(pz, q, s, &fail);
  const double eta = (G.gam - 1.) * pz[UU] + pz[RHO] + pz[UU] + dot4(s.bcon, s.bcov);
  StateAdj a;
  adj_zero(a);
  source_rev(G.gam, q, s, eta, conn, G.ng, gi, lu, sa->dt, a);
  double lb[8];
  state_rev(pz, q, s, a, lb);
#pragma unroll
  for (int k = 0; k < 8; k++) lampb[k * G.nc + c] += lb[k];
}

// ---------------------------------------------------------------------------
// the face fluxes (k_flux: limited face states, LF flux) transposed

// face_side (harm_phys.cuh: get_state, primtoflux for DIR and for t, vchar
// (phys.c:337-476)) reversed: given the side's state s (get_state of p) and the
// adjoints of its outputs aF (F^DIR), aU (F^t), acx (vmax) and acn (vmin), the
// adjoint of the side's primitives
template <int DIR>
__device__ __forceinline__ void face_side_rev(double gam, const double *p, const Geo &q, const StateT<double> &s,
                                              const double *aF, const double *aU, double acx, double acn, double *ap)
{
  const double rho = p[RHO], u = p[UU];
  const double bsq = dot4(s.bcon, s.bcov);

  // vchar, values as it forms them
  const double EF = rho + gam * u, EE = bsq + EF, va2 = bsq / EE, cs2 = gam * (gam - 1.) * u / EF;
  double cms2 = cs2 + va2 - cs2 * va2;
  bool clive = true;
  if (cms2 < 0.) { cms2 = SMALL; clive = false; }
  if (cms2 > 1.) { cms2 = 1.; clive = false; }
  const double Asq = gcon_diag(q, DIR), Bsq = q.n00, AB = gcon_t(q, DIR);
  const double Au = s.ucon[DIR], Bu = s.ucon[0];
  const double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  const double A = Bu2 - (Bsq + Bu2) * cms2;
  const double B = 2. * (AuBu - (AB + AuBu) * cms2);
  const double C = Au2 - (Asq + Au2) * cms2;
  double discr = B * B - 4. * A * C;
  const bool dlive = !(discr < 0.);
  if (!dlive) discr = 0.;
  const double dd = sqrt(discr);
  const double vp = -(-B + dd) / (2. * A), vm = -(-B - dd) / (2. * A);

  // vchar reversed: vmax, vmin -> A, B, C -> u^DIR, u^t, cms2 -> rho, u, b^2
  StateAdj a;
  adj_zero(a);
  const double avp = vp > vm ? acx : acn, avm = vp > vm ? acn : acx;
  double aA = -(avp * vp + avm * vm) / A;
  double aB = (avp + avm) / (2. * A);
  const double adisc = (dlive && dd > 0.) ? ((avm - avp) / (2. * A)) * 0.5 / dd : 0.;
  aB += 2. * B * adisc;
  aA += -4. * C * adisc;
  const double aC = -4. * A * adisc;
  a.uc[DIR] += aC * 2. * Au * (1. - cms2) + aB * 2. * (1. - cms2) * Bu;
  a.uc[0] += aA * 2. * Bu * (1. - cms2) + aB * 2. * (1. - cms2) * Au;
  const double acms = clive ? -aA * (Bsq + Bu2) - aB * 2. * (AB + AuBu) - aC * (Asq + Au2) : 0.;
  const double acs2 = acms * (1. - va2), ava2 = acms * (1. - cs2);
  a.u += acs2 * gam * (gam - 1.) / EF;
  double aEF = -acs2 * cs2 / EF;
  const double aEE = -ava2 * va2 / EE;
  a.bsq += ava2 / EE + aEE;
  aEF += aEE;
  a.rho += aEF;
  a.u += gam * aEF;

  // the two fluxes, then the state
  const double eta = (gam - 1.) * u + rho + u + bsq;
  flux_rev(gam, p, q, s, eta, DIR, aF, a);
  flux_rev(gam, p, q, s, eta, 0, aU, a);
  state_rev(p, q, s, a, ap);
}

// FULL: the corrector, whose Courant minimum n_d (recorded) gets adjoint
// as->ln.  Two lanes per face, one per side of the Lax-Friedrichs flux; they
// swap their sides' values and each reverses its own side.
template <int DIR, bool FULL>
__global__ void __launch_bounds__(128) k_adj_flux(Grid G, const double *__restrict__ pb,
                                                  const double *__restrict__ geo,
                                                  const double *__restrict__ lamF, double *lamp,
                                                  const DevScalars *sa, AdjScalars *as,
                                                  const double *__restrict__ ctrec)
{
  using D4 = Dual<4>;
  const int side = threadIdx.x & 1, lane = threadIdx.x & 31;
  const unsigned pmask = 0x3u << (lane & ~1);
  const int j = (DIR == 2 ? G.jstart : G.jstart - 1) + blockIdx.x * (blockDim.x >> 1) + (threadIdx.x >> 1);
  const int i = (DIR == 1 ? G.istart : G.istart - 1) + blockIdx.y;
  if (i > G.istop + 1 || j > G.jstop + 1) return;
  if (DIR == 2 && (j == G.jstart || j == G.jstop + 1)) return;  // polar faces carry no flux
  const long c = cidx(G, 0, i, j);
  double lF[8];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    lF[k] = lamF[k * G.nc + c];
    any |= lF[k] != 0.;
  }
  const bool act = FULL && i >= G.istart && i <= G.istop && j >= G.jstart && j <= G.jstop;
  const double lnd = FULL ? as->ln[DIR - 1] : 0.;
  const double nmin = FULL ? __longlong_as_double((long long)sa->ndt_bits[DIR - 1]) : 0.;
  const double dxd = DIR == 1 ? G.dx1 : G.dx2;
  if (!any && !(act && lnd != 0.)) return;  // the same for both lanes of the face
  // a face without flux adjoint matters only if it set the Courant minimum
  // (its wave speed as the recomputed step kept it)
  if (FULL && !any && !(G.cour * dxd / ctrec[(DIR - 1) * G.nc + c] == nmin)) return;
  const long o1 = DIR == 1 ? c - 2 * G.sn2 : c - 2, o2 = DIR == 1 ? c - G.sn2 : c - 1,
             o3 = DIR == 1 ? c + G.sn2 : c + 1;
  // limited face states (interp.c:49-93); the derivatives of this lane's side
  // in (p[-2], p[-1], p[0], p[+1])
  double ps[8], dlim[8][4];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const double *P = pb + k * G.nc;
    D4 a = D4::seed(P[o1], 0), b = D4::seed(P[o2], 1), z = D4::seed(P[c], 2), e = D4::seed(P[o3], 3);
    D4 v = side ? z - 0.5 * slope_lim(G.lim, b, z, e) : b + 0.5 * slope_lim(G.lim, a, b, z);
    ps[k] = v.v;
#pragma unroll
    for (int m = 0; m < 4; m++) dlim[k][m] = v.d[m];
  }
  Geo q;
  load_geo(geo_at(geo, G, DIR == 1 ? L_FACE1 : L_FACE2), G.ng, (long)i * G.sn2 + j, q);
  // this side's state, conserved variables and wave speeds (face_side without F^DIR)
  int f0 = 0;
  StateT<double> ss;
  get_state(ps, q, ss, &f0);
  double Us[8], cxs, cns, Uo[8];
  primtoflux(G.gam, ps, ss, 0, q.g, Us);
  vchar(G.gam, ps, ss, q, DIR, cxs, cns, &f0);
#pragma unroll
  for (int k = 0; k < 8; k++) Uo[k] = __shfl_xor_sync(pmask, Us[k], 1);
  const double cxo = __shfl_xor_sync(pmask, cxs, 1), cno = __shfl_xor_sync(pmask, cns, 1);
  const double *Ul = side ? Uo : Us, *Ur = side ? Us : Uo;
  const double cxl = side ? cxo : cxs, cnl = side ? cno : cns, cxr = side ? cxs : cxo, cnr = side ? cns : cno;
  // lf_flux's wave speed and the branches it takes
  const double t1 = 0. > cxl ? 0. : cxl;
  const double cmv = t1 > cxr ? t1 : cxr, cmax = fabs(cmv);
  const double t2 = 0. > -cnl ? 0. : -cnl;
  const double cnv = t2 > -cnr ? t2 : -cnr, cmin = fabs(cnv);
  const double ctop = cmax > cmin ? cmax : cmin;
  // the face that set the Courant minimum gets the adjoint of its wave speed
  double lct = 0.;
  if (act && lnd != 0.) {
    int win = 0;
    if (side == 0 && G.cour * dxd / ctop == nmin) win = atomicCAS(&as->claim[DIR - 1], 0, 1) == 0;
    win = __shfl_sync(pmask, win, lane & ~1);
    if (win) lct = -lnd * nmin / ctop;
  }
  if (!any && lct == 0.) return;
  // lf_flux reversed: F = (Fl + Fr - ctop (Ur - Ul)) / 2
  double act_ = lct;
#pragma unroll
  for (int k = 0; k < 8; k++) act_ -= 0.5 * lF[k] * (Ur[k] - Ul[k]);
  const double acmv = cmax > cmin ? (cmv < 0. ? -act_ : act_) : 0.;
  const double acnv = cmax > cmin ? 0. : (cnv < 0. ? -act_ : act_);
  double acxl = 0., acxr = 0., acnl = 0., acnr = 0.;
  if (t1 > cxr) {
    if (!(0. > cxl)) acxl = acmv;
  } else {
    acxr = acmv;
  }
  if (t2 > -cnr) {
    if (!(0. > -cnl)) acnl = -acnv;
  } else {
    acnr = -acnv;
  }
  double aF[8], aU[8], ap[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    aF[k] = 0.5 * lF[k];
    aU[k] = (side ? -0.5 : 0.5) * ctop * lF[k];
  }
  face_side_rev<DIR>(G.gam, ps, q, ss, aF, aU, side ? acxr : acxl, side ? acnr : acnl, ap);
  // and through the limiter onto the four cells
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double *L = lamp + k * G.nc;
    const double la = ap[k] * dlim[k][0], lb = ap[k] * dlim[k][1], lz = ap[k] * dlim[k][2],
                 le = ap[k] * dlim[k][3];
    if (la != 0.) atomicAdd(L + o1, la);
    if (lb != 0.) atomicAdd(L + o2, lb);
    if (lz != 0.) atomicAdd(L + c, lz);
    if (le != 0.) atomicAdd(L + o3, le);
  }
}

// ---------------------------------------------------------------------------
// host side

struct DevBuf {
  std::vector<void *> ptrs;
  ~DevBuf()
  {
    for (void *p : ptrs) cudaFree(p);
  }
  template <class T>
  T *get(size_t n)
  {
    void *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T *)p;
  }
};

static int run_adjoint(Ctx *x, int nsteps, int every, double *J, double *grad, double *ms)
{
  const Grid &G = x->G;
  const size_t nc = (size_t)G.nc, pl = 8 * nc;
  // the dual-number kernels keep up to ~2.3 KB per thread in local memory
  size_t stack = 0;
  CK(cudaDeviceGetLimit(&stack, cudaLimitStackSize));
  if (stack < 4096) CK(cudaDeviceSetLimit(cudaLimitStackSize, 4096));
  // the caller's stack limit again on every return (after B's buffers are freed)
  struct RestoreStack {
    size_t s;
    bool on;
    ~RestoreStack()
    {
      if (on) cudaDeviceSetLimit(cudaLimitStackSize, s);
    }
  } restore_stack{stack, stack < 4096};
  const int nseg = (nsteps + every - 1) / every;
  const int nrec = every < nsteps ? every : nsteps;
  DevBuf B;
  // checkpoints; per-step records of a segment, twice (segments alternate
  // between the two sets, so one is recomputed while the other is reversed);
  // the run state of every step; the adjoint state
  double *ck = B.get<double>(pl * nseg);
  DevScalars *cks = B.get<DevScalars>(nseg + 1);
  double *pend = B.get<double>(pl);
  DevScalars *scall = B.get<DevScalars>(2 * (size_t)nsteps);
  double *recp[2], *recd[2];
  signed char *recf[2];
  DevScalars *recs[2];
  int *recn[2];
  for (int b = 0; b < 2; b++) {
    recp[b] = B.get<double>(pl * (nrec + 1));
    recd[b] = B.get<double>((size_t)nrec * (7 * pl + 4 * nc));
    recf[b] = B.get<signed char>((size_t)nrec * 4 * nc);
    recs[b] = B.get<DevScalars>((size_t)nrec * 2);
    recn[b] = B.get<int>((size_t)nrec * 2);
    if (!recp[b] || !recd[b] || !recf[b] || !recs[b] || !recn[b])
      return fail_with(HARM_E_CUDA, "device memory for the adjoint");
  }
  double *lam = B.get<double>(6 * pl);  // next, cur, ph, U, F1, F2
  double *W = B.get<double>(pl);
  signed char *Wf = B.get<signed char>(nc);
  int *list = B.get<int>(FAIL_CAP);
  double *vbuf = B.get<double>((size_t)FAIL_CAP * 8);
  signed char *kinds = B.get<signed char>(FAIL_CAP);
  int *err = B.get<int>(1);
  AdjScalars *as = B.get<AdjScalars>(1);
  if (!ck || !cks || !pend || !scall || !lam || !W || !Wf || !list || !vbuf || !kinds || !err || !as)
    return fail_with(HARM_E_CUDA, "device memory for the adjoint");
  std::vector<StepRec> rec[2];
  for (int b = 0; b < 2; b++) {
    rec[b].resize(nrec);
    for (int r = 0; r < nrec; r++) {
      double *d = recd[b] + (size_t)r * (7 * pl + 4 * nc);
      StepRec &s = rec[b][r];
      s.X1[0] = d; s.X1[1] = d + pl; s.Ub[0] = d + 2 * pl; s.Ub[1] = d + 3 * pl; s.ph = d + 4 * pl;
      s.Z[0] = d + 5 * pl; s.Z[1] = d + 6 * pl;
      s.F1rho[0] = d + 7 * pl; s.F1rho[1] = d + 7 * pl + nc; s.ctop = d + 7 * pl + 2 * nc;
      s.fl1[0] = recf[b] + (size_t)r * 4 * nc; s.fl1[1] = s.fl1[0] + nc;
      s.wz[0] = s.fl1[0] + 2 * nc; s.wz[1] = s.fl1[0] + 3 * nc;
      s.sc[0] = recs[b] + 2 * r; s.sc[1] = recs[b] + 2 * r + 1;
      s.nfail[0] = recn[b] + 2 * r; s.nfail[1] = recn[b] + 2 * r + 1;
    }
  }
  // the adjoint of the state after the step being undone (A) and before it (B)
  double *const A = lam, *const Bl = lam + pl, *lh = lam + 2 * pl, *lU = lam + 3 * pl, *lF1 = lam + 4 * pl,
                *lF2 = lam + 5 * pl;
  // the context's stream runs the forward pass and the recomputation, rs the
  // reverse sweep
  cudaStream_t st = x->stream, rs = nullptr, fs = nullptr;
  CK(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking));
  cudaEvent_t e0, e1, e2, efwd, erec[2], erev[2];  // timing; forward done; records ready; reverse done
  cudaEvent_t efork[2], ejoin[2];                   // the two face directions, side by side
  cudaEvent_t ecf, ecj;                             // the corrector's update and source, side by side
  struct Guard {
    cudaStream_t s, f;
    std::vector<cudaEvent_t> e;
    ~Guard()
    {
      for (cudaEvent_t v : e) cudaEventDestroy(v);
      if (s) cudaStreamDestroy(s);
      if (f) cudaStreamDestroy(f);
    }
  } guard{rs, nullptr, {}};
  CK(cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking));
  guard.f = fs;
  for (cudaEvent_t *e : {&e0, &e1, &e2}) {
    CK(cudaEventCreate(e));
    guard.e.push_back(*e);
  }
  for (cudaEvent_t *e :
       {&efwd, &erec[0], &erec[1], &erev[0], &erev[1], &efork[0], &efork[1], &ejoin[0], &ejoin[1], &ecf, &ecj}) {
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    guard.e.push_back(*e);
  }
  struct Graph {
    cudaGraphExec_t e = nullptr;
    ~Graph() { if (e) cudaGraphExecDestroy(e); }
  };
  auto capture = [&](Graph &g, auto &&body) -> int {
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = body();
    cudaError_t e = cudaStreamEndCapture(st, &gr);
    if (rc) return rc;
    if (e != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&g.e, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    return HARM_OK;
  };
  const size_t pb = pl * sizeof(double);
  // one segment's steps, recorded into set b (recomputation): states before
  // each step and after the last
  auto record = [&](int b, int len) -> int {
    for (int r = 0; r < len; r++) {
      CK(cudaMemcpyAsync(recp[b] + (size_t)r * pl, x->p, pb, cudaMemcpyDeviceToDevice, st));
      int rc = exact::launch_step_rec(x, rec[b][r]);
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(recp[b] + (size_t)len * pl, x->p, pb, cudaMemcpyDeviceToDevice, st));
    return HARM_OK;
  };

  const dim3 tile(32, 4);
  const dim3 zg((G.n2 + 31) / 32, (G.n1 + 3) / 4, 1);
  // face kernels: 64 faces along theta per block, two lanes each; one r row per block
  const dim3 ftile(128, 1);
  const dim3 g1((G.n2 + 2 + 63) / 64, G.n1 + 1, 1);
  const dim3 g2((G.n2 + 1 + 63) / 64, G.n1 + 2, 1);
  const int nbc = 4 * G.sn2 + 4 * (G.sn1 - 4);
  // the reverse of one segment of len steps recorded in set b, on stream q:
  // the adjoint of its last state in A on entry, of its first state in A on
  // exit, B zero both times
  auto reverse = [&](int b, int len, cudaStream_t q) -> int {
    double *lnext = A, *lcur = Bl;
    for (int r = len - 1; r >= 0; r--) {
      const StepRec &R = rec[b][r];
      const DevScalars *sa = R.sc[0], *sb = R.sc[1];
      const double *pn = recp[b] + (size_t)r * pl, *pnext = recp[b] + (size_t)(r + 1) * pl;
      // the time step's chain, the objective's seed on the step's result, and
      // the corrector's bound_prim, fixup_utoprim, bound_prim, inversion, update, fluxes
      k_adj_din_bound<<<(nbc + 127) / 128, 128, 0, q>>>(G, pnext, x->geo, lnext, sa, sb, as);
      k_adj_fixup_bound<<<1, FU_THREADS, 0, q>>>(G, R.X1[1], R.fl1[1], x->geo, x->floors, W, Wf, list, vbuf, kinds,
                                                lnext, err, R.nfail[1]);
      k_adj_invert<<<zg, tile, 0, q>>>(G, R.Ub[1], R.Z[1], R.wz[1], x->geo, x->floors, x->katm, lnext, lU, lcur,
                                       err);
      CK(cudaMemsetAsync(lF1, 0, 2 * pb, q));
      // primtoU(p^n) and the face fluxes' adjoints beside the source at ph (fs)
      CK(cudaEventRecord(ecf, q));
      CK(cudaStreamWaitEvent(fs, ecf, 0));
      k_adj_cons<true><<<zg, tile, 0, q>>>(G, pn, R.Ub[1], R.F1rho[1], x->geo, x->conn, lU, lcur, lF1, lF2, sa, as);
      k_adj_source<<<zg, tile, 0, fs>>>(G, R.ph, x->geo, x->conn, lU, lh, sa);
      CK(cudaEventRecord(ecj, fs));
      CK(cudaStreamWaitEvent(q, ecj, 0));
      // the two directions run side by side (fs), each adding into the state adjoint
      CK(cudaEventRecord(efork[0], q));
      CK(cudaStreamWaitEvent(fs, efork[0], 0));
      k_adj_flux<1, true><<<g1, ftile, 0, q>>>(G, R.ph, x->geo, lF1, lh, sa, as, R.ctop);
      k_adj_flux<2, true><<<g2, ftile, 0, fs>>>(G, R.ph, x->geo, lF2, lh, sa, as, R.ctop);
      CK(cudaEventRecord(ejoin[0], fs));
      CK(cudaStreamWaitEvent(q, ejoin[0], 0));
      // predictor, from p^n into ph
      k_adj_bound<<<(nbc + 127) / 128, 128, 0, q>>>(G, R.ph, x->geo, lh);
      k_adj_fixup_bound<<<1, FU_THREADS, 0, q>>>(G, R.X1[0], R.fl1[0], x->geo, x->floors, W, Wf, list, vbuf, kinds,
                                                lh, err, R.nfail[0]);
      k_adj_invert<<<zg, tile, 0, q>>>(G, R.Ub[0], R.Z[0], R.wz[0], x->geo, x->floors, x->katm, lh, lU, lcur, err);
      CK(cudaMemsetAsync(lF1, 0, 2 * pb, q));
      k_adj_cons<false><<<zg, tile, 0, q>>>(G, pn, R.Ub[0], R.F1rho[0], x->geo, x->conn, lU, lcur, lF1, lF2, sa,
                                            as);
      CK(cudaEventRecord(efork[1], q));
      CK(cudaStreamWaitEvent(fs, efork[1], 0));
      k_adj_flux<1, false><<<g1, ftile, 0, q>>>(G, pn, x->geo, lF1, lcur, sa, as, nullptr);
      k_adj_flux<2, false><<<g2, ftile, 0, fs>>>(G, pn, x->geo, lF2, lcur, sa, as, nullptr);
      CK(cudaEventRecord(ejoin[1], fs));
      CK(cudaStreamWaitEvent(q, ejoin[1], 0));
      k_adj_dt_post<<<1, 1, 0, q>>>(sa, sb, as);
      CK(cudaGetLastError());
      // the adjoint of p^n becomes the next (earlier) step's output adjoint
      double *t = lnext;
      lnext = lcur;
      lcur = t;
      CK(cudaMemsetAsync(lcur, 0, pb, q));
      CK(cudaMemsetAsync(lh, 0, pb, q));
    }
    if (lnext != A) {
      CK(cudaMemcpyAsync(A, lnext, pb, cudaMemcpyDeviceToDevice, q));
      CK(cudaMemsetAsync(lnext, 0, pb, q));
    }
    return HARM_OK;
  };

  CK(cudaMemsetAsync(err, 0, sizeof(int), st));
  CK(cudaMemsetAsync(as, 0, sizeof(AdjScalars), st));
  CK(cudaMemsetAsync(lam, 0, 6 * pb, st));
  const int last0 = (nseg - 1) * every, lastlen = nsteps - last0, blast = (nseg - 1) & 1;
  Graph gstep, grec[2], grev[2];
  int rc = capture(gstep, [&] { return exact::launch_step(x); });
  if (rc) return rc;
  for (int b = 0; b < 2; b++) {
    if (nseg > 1) {
      rc = capture(grec[b], [&] { return record(b, every); });
      if (rc) return rc;
    }
    rc = capture(grev[b], [&] { return reverse(b, every, st); });
    if (rc) return rc;
  }
  // the run state recorded with segment seg's steps, kept for the checks at the end
  auto keep_scalars = [&](int seg, int len) -> int {
    CK(cudaMemcpyAsync(scall + 2 * (size_t)seg * every, recs[seg & 1], 2 * (size_t)len * sizeof(DevScalars),
                       cudaMemcpyDeviceToDevice, st));
    return HARM_OK;
  };

  // forward pass: a checkpoint every `every` steps; the last segment is
  // recorded on the way, so it needs no recomputation
  CK(cudaEventRecord(e0, st));
  for (int seg = 0; seg < nseg; seg++) {
    CK(cudaMemcpyAsync(ck + (size_t)seg * pl, x->p, pb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(cks + seg, x->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, st));
    if (seg < nseg - 1) {
      for (int r = 0; r < every; r++) CK(cudaGraphLaunch(gstep.e, st));
    } else if (lastlen == every && nseg > 1) {
      CK(cudaGraphLaunch(grec[blast].e, st));
    } else {
      rc = record(blast, lastlen);
      if (rc) return rc;
    }
  }
  CK(cudaEventRecord(e1, st));
  rc = keep_scalars(nseg - 1, lastlen);
  if (rc) return rc;
  CK(cudaMemcpyAsync(pend, x->p, pb, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(cks + nseg, x->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, st));
  CK(cudaEventRecord(efwd, st));
  DevScalars s0, s1;
  CK(cudaMemcpyAsync(&s0, cks, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&s1, cks + nseg, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (s1.fail_code || s1.halted)
    return fail_with(HARM_E_ADJOINT, "the forward steps failed (fail code " + std::to_string(s1.fail_code) + ")");
  *J = s1.mass_in - s0.mass_in;

  // reverse sweep, segment by segment from the last; each segment's reverse
  // (rs) overlaps the recomputation of the segment before it (st)
  CK(cudaStreamWaitEvent(rs, efwd, 0));
  for (int seg = nseg - 1; seg >= 0; seg--) {
    const int b = seg & 1, len = seg == nseg - 1 ? lastlen : every;
    if (seg < nseg - 1) CK(cudaStreamWaitEvent(rs, erec[b], 0));
    if (len == every) {
      CK(cudaGraphLaunch(grev[b].e, rs));
    } else {
      rc = reverse(b, len, rs);
      if (rc) return rc;
    }
    CK(cudaEventRecord(erev[b], rs));
    if (seg > 0) {
      // recompute segment seg - 1 into the other set, once the reverse that
      // last read that set (segment seg + 1's) is done
      const int bp = (seg - 1) & 1;
      if (seg + 1 <= nseg - 1) CK(cudaStreamWaitEvent(st, erev[bp], 0));
      CK(cudaMemcpyAsync(x->p, ck + (size_t)(seg - 1) * pl, pb, cudaMemcpyDeviceToDevice, st));
      CK(cudaMemcpyAsync(x->sc, cks + seg - 1, sizeof(DevScalars), cudaMemcpyDeviceToDevice, st));
      CK(cudaGraphLaunch(grec[bp].e, st));
      rc = keep_scalars(seg - 1, every);
      if (rc) return rc;
      CK(cudaEventRecord(erec[bp], st));
    }
  }
  CK(cudaEventRecord(e2, rs));
  CK(cudaStreamWaitEvent(st, e2, 0));
  int herr = 0;
  std::vector<DevScalars> hs(2 * (size_t)nsteps);
  CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hs.data(), scall, hs.size() * sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int n = 0; n < nsteps; n++) {
    const DevScalars &sa = hs[2 * n], &sb = hs[2 * n + 1];
    if (sb.fail_code) return fail_with(HARM_E_ADJOINT, "a recomputed step failed");
    if (sb.dt != (sb.ndt > SAFE * sa.dt ? SAFE * sa.dt : sb.ndt))
      return fail_with(HARM_E_ARG, "the steps reach tf: the adjoint needs dt = min(ndt, 1.3 dt) throughout");
  }
  if (herr & ERR_FAILS)
    return fail_with(HARM_E_ADJOINT, "more failed inversions in a half step than the adjoint lists");
  if (herr & ERR_SINGULAR)
    return fail_with(HARM_E_ADJOINT, "a singular primtoU Jacobian in the adjoint of an inversion");
  if (ms) {
    float a, b;
    CK(cudaEventElapsedTime(&a, e0, e1));
    CK(cudaEventElapsedTime(&b, e1, e2));
    ms[0] = a;
    ms[1] = b;
  }
  rc = get_prims(x, A, grad, nullptr);
  if (rc) return rc;
  // leave the context where the forward pass ended
  CK(cudaMemcpyAsync(x->p, pend, pb, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(x->sc, cks + nseg, sizeof(DevScalars), cudaMemcpyDeviceToDevice, st));
  CK(cudaStreamSynchronize(st));
  return HARM_OK;
}

}  // namespace adj
}  // namespace harm

extern "C" int harm_adjoint_mass_in(harm_ctx *h, int nsteps, int checkpoint_every, double *J, double *grad,
                                    double *ms)
{
  using namespace harm;
  if (!h || !J || !grad) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  if (nsteps < 1 || checkpoint_every < 1) return fail_with(HARM_E_ARG, "nsteps and checkpoint_every must be >= 1");
  if (x->G.n3 != 1) return fail_with(HARM_E_ARG, "the adjoint covers the 2D step (N3 = 1)");
  if (x->cool) return fail_with(HARM_E_ARG, "the adjoint covers the gamma-law step, not COOL_EOS");
  if (x->mode != HARM_FP64) return fail_with(HARM_E_ARG, "the adjoint runs on the FP64 step");
  if (x->ntr) return fail_with(HARM_E_ARG, "the adjoint's recomputation would move the tracers again: detach them");
  return adj::run_adjoint(x, nsteps, checkpoint_every, J, grad, ms);
}
