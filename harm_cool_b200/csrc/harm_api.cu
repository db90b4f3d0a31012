// Kernels shared by both precision variants (boundaries, failure repair,
// diagnostics, layout conversion, set-up helpers) and the C ABI of
// libharm_b200.  Built with -fmad=false.
//
// Device layout.  The reference keeps each primitive array as
// p[SN3][SN1][SN2][8] on the host.  On the device every array is stored
// plane by plane (structure of arrays), X[k][h][i][j] with j fastest, so a
// warp reading one variable of 32 neighbouring theta zones reads 256
// contiguous bytes.  Only the N3 active phi planes are stored: the
// reference's two phi ghost planes are exact copies of planes N3 and 1 made by
// MPI self-exchange (step_ch.c:183-198, 222-230, mpi.c:284-321), so here the
// phi index simply wraps.  Geometry is axisymmetric and stored once per
// (r, theta) point, 18 planes per face location (harm_phys.cuh) plus 40
// connection planes and two floor planes.
//
// One step (step_ch.c:90-140) is, on one stream and without host sync:
//   predictor : k_flux x3, k_update(dt/2) [flux-CT, source, inversion, floors],
//               k_bound, k_fu_flip, k_fu_fix, k_bound
//   corrector : k_flux x3 (+Courant minima), k_update(dt), k_diag_flux,
//               k_bound, k_fu_flip, k_fu_fix, k_bound
//   k_diag_mass, k_finalize (diagnostic sums, next dt)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "harm_common.cuh"
#include "harm_bound.cuh"

namespace harm {

// ---------------------------------------------------------------------------
// boundary conditions (bounds.c:54-331, polefix :381-436)
//
// Each thread owns one cell that bound_prim writes and computes its final
// value directly from cells that bound_prim never writes, so no ordering is
// needed: radial ghosts copy the edge zone, polefix rows copy row jstart+2
// (linear ramp for U2, fields untouched), polar ghosts reflect (2D) or take
// the opposite-phi plane (3D), U2 and B2 flip sign across the pole, and the
// radial ghosts finally get inflow_check().

template <bool THREE_D>
__global__ void k_bound(Grid G, double *P, signed char *pflag, const double *__restrict__ geo, DevScalars *sc)
{
  if (sc->halted) return;
  const int nrow = THREE_D ? 8 : 4;
  const int ncell = 4 * G.sn2 + nrow * (G.sn1 - 4);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  if (t >= ncell) return;
  BoundCell b = bound_cell(G, t, nrow);
  const int i = b.i, j = b.j;
  double v[8];
  signed char fl;
  const bool rghost = i < G.istart || i > G.istop;
  const int ci = i < G.istart ? G.istart : (i > G.istop ? G.istop : i);
  if (j >= G.jstart && j <= G.jstop) {
    if (!rghost && !THREE_D) return;  // nothing to do (2D rows only list ghosts)
    polefixed<THREE_D>(G, P, h, i, j, v);
    fl = pflag[cidx(G, h, ci, j)];
  } else {
    // polar ghosts: source row and plane
    const bool low = j < G.jstart;
    const int js = low ? (j == G.jstart - 1 ? G.jstart : G.jstart + 1) : (j == G.jstop + 1 ? G.jstop : G.jstop - 1);
    const int hs = THREE_D ? (h + G.n3 / 2) % G.n3 : h;  // opposite-phi plane (mpi.c:374-386)
    polefixed<THREE_D>(G, P, hs, i, js, v);
    v[U2] *= -1.;
    v[B2] *= -1.;
    fl = pflag[cidx(G, h, ci, js)];
  }
  if (rghost) {
    Geo q;
    load_geo(geo_at(geo, G, L_CENT), G.ng, (long)i * G.sn2 + j, q);
    int fail = 0;
    inflow_check(v, q, i < G.istart ? 0 : 1, &fail);
    if (fail) record_fail(sc, fail, h + (THREE_D ? 1 : 0), i, j);
  }
  const long c = cidx(G, h, i, j);
  if (THREE_D && !rghost && j >= G.jstart && j <= G.jstop) {
#pragma unroll
    for (int k = 0; k < 5; k++) P[k * G.nc + c] = v[k];  // polefix leaves the fields alone
    return;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) P[k * G.nc + c] = v[k];
  pflag[c] = fl;
}

// ---------------------------------------------------------------------------
// fixup_utoprim() (fixup.c:432-538)
//
// The reference flips pflag over all (i, j) of the active phi planes and
// then repairs failed zones in loop order, in place.  Repairs from the edge
// or corner stencils read only good zones, which the repair never changes;
// the last-resort average reads every neighbour and so sees earlier repairs.
// k_fu_flip flips the flags and lists the failed zones.  For a few failures
// k_fu_fix sorts the list into loop order, precomputes the stencil repairs in
// parallel and then replays the whole list in order on one thread,
// recomputing any zone whose stencil choice changed or that needs the
// last-resort average.  For many failures k_fu_wave repairs them in
// wavefronts instead: a repair reads only its own phi plane, and within a
// plane zone (i, j) depends only on (i-1, j-1..j+1) and (i, j-1), all on
// earlier lines 2i + j = const, so each plane is one block that sweeps those
// lines in order with a barrier between them -- the loop order's results.

__global__ void k_fu_flip(Grid G, signed char *pflag, int *list, DevScalars *sc)
{
  if (sc->halted) return;
  const long n = G.nc;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    signed char f = pflag[c];
    signed char nf = (signed char)(!f);
    pflag[c] = nf;
    if (nf == 0) {
      int j = (int)(c % G.sn2), i = (int)((c / G.sn2) % G.sn1);
      if (i >= G.istart && i <= G.istop && j >= G.jstart && j <= G.jstop) {
        int slot = atomicAdd(&sc->nfail, 1);
        if (slot < FAIL_CAP) list[slot] = (int)c;
        else sc->fail_overflow = 1;
      }
    }
  }
}

__device__ __forceinline__ void cell_hij(const Grid &G, long c, int &h, int &i, int &j)
{
  j = (int)(c % G.sn2);
  i = (int)((c / G.sn2) % G.sn1);
  h = (int)(c / ((long)G.sn2 * G.sn1));
}

__global__ void __launch_bounds__(NTHR_FIX) k_fu_fix(Grid G, double *P, signed char *pflag, int *list, double *fixbuf,
                                                     const double *__restrict__ geo, const double *__restrict__ floors,
                                                     DevScalars *sc)
{
  if (sc->halted) return;
  __shared__ int keys[FIX_LIST_MAX];
  __shared__ signed char kinds[FIX_LIST_MAX];
  __shared__ int gfail;
  const int n = sc->nfail;
  if (n == 0) return;
  if (n > FIX_LIST_MAX || sc->fail_overflow) return;  // k_fu_wave's case
  const int tid = threadIdx.x;
  if (tid == 0) gfail = 0;
  const double *gC = geo_at(geo, G, L_CENT);
  {
    // bitonic sort of the failed cells into loop order
    int m = 1;
    while (m < n) m <<= 1;
    for (int t = tid; t < m; t += blockDim.x) keys[t] = t < n ? list[t] : 0x7fffffff;
    __syncthreads();
    for (int size = 2; size <= m; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = tid; t < m; t += blockDim.x) {
          int u = t ^ stride;
          if (u > t) {
            bool up = (t & size) == 0;
            int a = keys[t], b = keys[u];
            if ((a > b) == up) { keys[t] = b; keys[u] = a; }
          }
        }
        __syncthreads();
      }
    // parallel: stencil repairs from the flags as they stand now
    for (int t = tid; t < n; t += blockDim.x) {
      long c = keys[t];
      int kind = stencil_kind(G, pflag, c);
      kinds[t] = (signed char)kind;
      if (kind < 2) {
        double v[8];
        repair_zone(G, P, c, kind, v);
        int h, i, j;
        cell_hij(G, c, h, i, j);
        long gi = (long)i * G.sn2 + j;
        Geo q;
        load_geo(gC, G.ng, gi, q);
        int fail = 0;
        bool g33 = fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail);
        if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
        if (g33) kinds[t] = (signed char)(kinds[t] | 4);
        for (int k = 0; k < 8; k++) fixbuf[(long)t * 8 + k] = v[k];
      }
    }
    __syncthreads();
    // in order, one thread
    if (tid == 0) {
      for (int t = 0; t < n; t++) {
        long c = keys[t];
        int kind = stencil_kind(G, pflag, c);
        int pre = kinds[t] & 3;
        double v[8];
        bool g33;
        int h, i, j;
        cell_hij(G, c, h, i, j);
        if (kind == pre && kind < 2) {
          for (int k = 0; k < 8; k++) v[k] = fixbuf[(long)t * 8 + k];
          g33 = (kinds[t] & 4) != 0;
        } else {
          repair_zone(G, P, c, kind, v);
          long gi = (long)i * G.sn2 + j;
          Geo q;
          load_geo(gC, G.ng, gi, q);
          int fail = 0;
          g33 = fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail);
          if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
        }
        for (int k = 0; k < 8; k++) P[k * G.nc + c] = v[k];
        pflag[c] = g33 ? (signed char)-33 : (signed char)0;
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    sc->nfail = 0;
    sc->fail_overflow = 0;
  }
}

// many failures: one block per phi plane, wavefronts 2i + j in order
__global__ void __launch_bounds__(256) k_fu_wave(Grid G, double *P, signed char *pflag,
                                                 const double *__restrict__ geo, const double *__restrict__ floors,
                                                 DevScalars *sc)
{
  if (sc->halted) return;
  const int n = sc->nfail;
  if (n == 0) return;  // none, or k_fu_fix has repaired them
  const int h = blockIdx.x;
  const double *gC = geo_at(geo, G, L_CENT);
  const int w0 = 2 * G.istart + G.jstart, w1 = 2 * G.istop + G.jstop;
  for (int w = w0; w <= w1; w++) {
    // i such that j = w - 2i lies in [jstart, jstop]
    int ilo = (w - G.jstop + 1) / 2, ihi = (w - G.jstart) / 2;
    if (ilo < G.istart) ilo = G.istart;
    if (ihi > G.istop) ihi = G.istop;
    for (int i = ilo + (int)threadIdx.x; i <= ihi; i += blockDim.x) {
      const int j = w - 2 * i;
      const long c = cidx(G, h, i, j);
      if (pflag[c] != 0) continue;
      double v[8];
      repair_zone(G, P, c, stencil_kind(G, pflag, c), v);
      const long gi = (long)i * G.sn2 + j;
      Geo q;
      load_geo(gC, G.ng, gi, q);
      int fail = 0;
      bool g33 = fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail);
      if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
      for (int k = 0; k < 8; k++) P[k * G.nc + c] = v[k];
      pflag[c] = g33 ? (signed char)-33 : (signed char)0;
    }
    __syncthreads();
  }
  // the last block to finish clears the counters for the next call
  __shared__ bool last;
  __threadfence();
  if (threadIdx.x == 0) last = atomicAdd(&sc->wave_done, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    sc->wave_done = 0;
    sc->nfail = 0;
    sc->fail_overflow = 0;
  }
}

// ---------------------------------------------------------------------------
// diag_mass() (diag.c:477-580, MDOTTYPE NEU_AGA_GHOST1) partial sums

__global__ void __launch_bounds__(256) k_diag_mass(Grid G, const double *__restrict__ P, const double *__restrict__ geo,
                                                   double *partials, int nparts, DevScalars *sc)
{
  if (sc->halted) return;
  const double *gC = geo_at(geo, G, L_CENT);
  double m = 0., din = 0., dout = 0.;
  const long nact = (long)G.n3 * G.n1 * G.n2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nact; t += (long)gridDim.x * blockDim.x) {
    int j = G.jstart + (int)(t % G.n2);
    int i = G.istart + (int)((t / G.n2) % G.n1);
    int h = (int)(t / ((long)G.n2 * G.n1));
    long gi = (long)i * G.sn2 + j;
    m += P[RHO * G.nc + cidx(G, h, i, j)] * __ldg(gC + 17 * G.ng + gi) * G.dx1 * G.dx2 * G.dx3;
  }
  const long nrad = (long)G.n3 * G.n2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < 2 * nrad; t += (long)gridDim.x * blockDim.x) {
    bool inner = t < nrad;
    long u = inner ? t : t - nrad;
    int j = G.jstart + (int)(u % G.n2), h = (int)(u / G.n2);
    int i = inner ? G.istart - 1 : G.istop + 1;
    long c = cidx(G, h, i, j);
    double pr[8];
    for (int k = 0; k < 8; k++) pr[k] = P[k * G.nc + c];
    Geo q;
    load_geo(gC, G.ng, (long)i * G.sn2 + j, q);
    double ucon[4];
    int fail = 0;
    ucon_calc(pr, q, ucon, &fail);
    if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
    double term = pr[RHO] * ucon[1] * q.g * G.dx2 * G.dx3;
    if (inner) din += term;
    else dout -= term;
  }
  __shared__ double red[3][8];
  m = warp_sum(m);
  din = warp_sum(din);
  dout = warp_sum(dout);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = m; red[1][w] = din; red[2][w] = dout; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0., b = 0., d = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) { a += red[0][k]; b += red[1][k]; d += red[2][k]; }
    partials[blockIdx.x] = a;
    partials[nparts + blockIdx.x] = b;
    partials[2 * nparts + blockIdx.x] = d;
  }
}

// sums of the partials, mass counters, and the next time step (step_ch.c:119-137)
__global__ void k_finalize(Grid G, const double *partials, int nparts, DevScalars *sc)
{
  if (sc->halted) return;
  __shared__ double red[3][32];
  double a = 0., b = 0., d = 0.;
  for (int t = threadIdx.x; t < nparts; t += blockDim.x) {
    a += partials[t];
    b += partials[nparts + t];
    d += partials[2 * nparts + t];
  }
  a = warp_sum(a);
  b = warp_sum(b);
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = b; red[2][threadIdx.x >> 5] = d; }
  __syncthreads();
  if (threadIdx.x != 0) return;
  a = b = d = 0.;
  for (int k = 0; k < (int)(blockDim.x >> 5); k++) { a += red[0][k]; b += red[1][k]; d += red[2][k]; }
  double dt = sc->dt;
  sc->mass_curr = a;
  sc->mdot_in = b;
  sc->mdot_out = d;
  sc->mass_in += b * dt;
  sc->mass_out += d * dt;
  double n1 = __longlong_as_double((long long)sc->ndt_bits[0]);
  double n2 = __longlong_as_double((long long)sc->ndt_bits[1]);
  double n3 = __longlong_as_double((long long)sc->ndt_bits[2]);
  double ndt = G.n3 > 2 ? G.defcon * 1. / (1. / n1 + 1. / n2 + 1. / n3) : G.defcon * 1. / (1. / n1 + 1. / n2);
  sc->ndt = ndt;
  const unsigned long long big = (unsigned long long)__double_as_longlong(1.e9);
  sc->ndt_bits[0] = sc->ndt_bits[1] = sc->ndt_bits[2] = big;
  if (dt < 1.e-9) {
    sc->err = HARM_E_DT;
    sc->halted = 1;
    return;
  }
  double t = sc->t + dt;
  if (ndt > SAFE * dt) ndt = SAFE * dt;
  dt = ndt;
  if (t + dt > G.tf) dt = G.tf - t;
  sc->t = t;
  sc->dt = dt;
  if (sc->fail_code) sc->halted = 1;
}

// ---------------------------------------------------------------------------
// layout conversion between the host's p[h][i][j][8] and device planes

__global__ void k_from_host(Grid G, int h0, const double *__restrict__ A, double *P, const signed char *fa,
                            signed char *pflag)
{
  const long n = G.nc;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    long hc = c + (long)h0 * G.sn1 * G.sn2;  // cell in the host array (skips the phi ghost plane)
#pragma unroll
    for (int k = 0; k < 8; k++) P[k * n + c] = A[hc * 8 + k];
    if (fa) pflag[c] = fa[hc];
  }
}

__global__ void k_to_host(Grid G, int h0, const double *__restrict__ P, double *A, const signed char *pflag,
                          signed char *fa)
{
  // host planes: h0 ghost + n3 active + h0 ghost; ghosts are the periodic copies
  const long plane = (long)G.sn1 * G.sn2;
  const long nh = (long)(G.n3 + 2 * h0) * plane;
  for (long hc = blockIdx.x * (long)blockDim.x + threadIdx.x; hc < nh; hc += (long)gridDim.x * blockDim.x) {
    long hh = hc / plane, r = hc % plane;
    long hd = hh - h0;
    if (hd < 0) hd += G.n3;
    if (hd >= G.n3) hd -= G.n3;
    long c = hd * plane + r;
#pragma unroll
    for (int k = 0; k < 8; k++) A[hc * 8 + k] = P[k * G.nc + c];
    if (fa) fa[hc] = pflag[c];
  }
}

// fixup() alone over the active zones (harm_fixup)
__global__ void k_fixup(Grid G, double *P, signed char *pflag, const double *__restrict__ geo,
                        const double *__restrict__ floors, DevScalars *sc)
{
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, h, i, j), gi = (long)i * G.sn2 + j;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double v[8];
  for (int k = 0; k < 8; k++) v[k] = P[k * G.nc + c];
  int fail = 0;
  if (fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail)) pflag[c] = -33;
  if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
  for (int k = 0; k < 8; k++) P[k * G.nc + c] = v[k];
}

// Utoprim_2d over independent zones (harm_utoprim_2d_batch)
__global__ void k_utoprim_batch(const double *U, const double *gcov, const double *gcon, const double *gdet,
                                double *prim, int *ret, long n, double gam)
{
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double *a = gcov + t * 16, *b = gcon + t * 16;
  Geo q;
  q.v00 = a[0]; q.v01 = a[1]; q.v03 = a[3]; q.v11 = a[5]; q.v13 = a[7]; q.v22 = a[10]; q.v33 = a[15];
  q.n00 = b[0]; q.n01 = b[1]; q.n03 = b[3]; q.n10 = b[4]; q.n11 = b[5]; q.n13 = b[7]; q.n22 = b[10];
  q.n30 = b[12]; q.n31 = b[13]; q.n33 = b[15];
  q.alpha = 1. / sqrt(-q.n00);
  q.g = gdet[t];
  q.ialpha = 1. / q.alpha;
  q.ig = 1. / q.g;
  double u[8], p[8];
  for (int k = 0; k < 8; k++) { u[k] = U[t * 8 + k]; p[k] = prim[t * 8 + k]; }
  ret[t] = utoprim<0>(gam, 0., u, q, p);
  for (int k = 0; k < 8; k++) prim[t * 8 + k] = p[k];
}

// Utoprim_1dvsq2fix1 (which 1) or Utoprim_1dfix1 (which 2) over independent zones
__global__ void k_utoprim_fix_batch(int which, const double *U, const double *gcov, const double *gcon,
                                    const double *gdet, const double *K, double *prim, int *ret, long n, double gam)
{
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double *a = gcov + t * 16, *b = gcon + t * 16;
  Geo q;
  q.v00 = a[0]; q.v01 = a[1]; q.v03 = a[3]; q.v11 = a[5]; q.v13 = a[7]; q.v22 = a[10]; q.v33 = a[15];
  q.n00 = b[0]; q.n01 = b[1]; q.n03 = b[3]; q.n10 = b[4]; q.n11 = b[5]; q.n13 = b[7]; q.n22 = b[10];
  q.n30 = b[12]; q.n31 = b[13]; q.n33 = b[15];
  q.alpha = 1. / sqrt(-q.n00);
  q.g = gdet[t];
  q.ialpha = 1. / q.alpha;
  q.ig = 1. / q.g;
  double u[8], p[8];
  for (int k = 0; k < 8; k++) { u[k] = U[t * 8 + k]; p[k] = prim[t * 8 + k]; }
  ret[t] = which == 1 ? utoprim<1>(gam, K[t], u, q, p) : utoprim<2>(gam, K[t], u, q, p);
  for (int k = 0; k < 8; k++) prim[t * 8 + k] = p[k];
}

__global__ void k_pow_batch(const double *x, const double *y, double *out, long n)
{
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) out[t] = pow_cr(x[t], y[t]);
}

// torus set-up: b^2 maximum over the active zones, and the field rescaling (init.c:368-403)
__global__ void k_bsq_max(Grid G, const double *__restrict__ P, const double *__restrict__ geo, DevScalars *sc)
{
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, h, i, j), gi = (long)i * G.sn2 + j;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double v[8];
  for (int k = 0; k < 8; k++) v[k] = P[k * G.nc + c];
  State s;
  int fail = 0;
  get_state(v, q, s, &fail);
  double bsq = dot4(s.bcon, s.bcov);
  if (bsq > 0.) atomicMax(&sc->bsq_bits, (unsigned long long)__double_as_longlong(bsq));
}

__global__ void k_scale_field(Grid G, double *P, double norm)
{
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, h, i, j);
  P[B1 * G.nc + c] *= norm;
  P[B2 * G.nc + c] *= norm;
}

// ---------------------------------------------------------------------------
// host side

thread_local std::string g_err;

int fail_with(int code, const std::string &msg)
{
  g_err = msg;
  return code;
}

int launch_bound(Ctx *x, double *P)
{
  const Grid &G = x->G;
  const int nrow = G.n3 > 1 ? 8 : 4;
  const int ncell = 4 * G.sn2 + nrow * (G.sn1 - 4);
  dim3 grid((ncell + 127) / 128, G.n3);
  if (G.n3 > 1) k_bound<true><<<grid, 128, 0, x->stream>>>(G, P, x->pflag, x->geo, x->sc);
  else k_bound<false><<<grid, 128, 0, x->stream>>>(G, P, x->pflag, x->geo, x->sc);
  return HARM_OK;
}

int launch_fixup_utoprim(Ctx *x, double *P, int *nfail_out)
{
  const Grid &G = x->G;
  k_fu_flip<<<148 * 8, 256, 0, x->stream>>>(G, x->pflag, x->fail_list, x->sc);
  // the number of failed zones, kept for the discrete adjoint before the repair clears it
  if (nfail_out) CK(cudaMemcpyAsync(nfail_out, &x->sc->nfail, sizeof(int), cudaMemcpyDeviceToDevice, x->stream));
  k_fu_fix<<<1, NTHR_FIX, 0, x->stream>>>(G, P, x->pflag, x->fail_list, x->fix_buf, x->geo, x->floors, x->sc);
  k_fu_wave<<<G.n3, 256, 0, x->stream>>>(G, P, x->pflag, x->geo, x->floors, x->sc);
  return HARM_OK;
}

// diag_mass(), update_tracers() and the next dt (step_ch.c:119-137)
void launch_mass(Ctx *x)
{
  k_diag_mass<<<x->nparts, 256, 0, x->stream>>>(x->G, x->p, x->geo, x->partials, x->nparts, x->sc);
  if (x->ntr) launch_tracers(x);
  k_finalize<<<1, 1024, 0, x->stream>>>(x->G, x->partials, x->nparts, x->sc);
}

void invalidate_graph(Ctx *x)
{
  if (x->graph_exec) {
    cudaGraphExecDestroy(x->graph_exec);
    x->graph_exec = nullptr;
  }
}

int launch_step(Ctx *x)
{
  if (x->cool) return cool_launch_step(x);
  return x->mode == HARM_MIXED ? mixed::launch_step(x) : exact::launch_step(x);
}

// structural checks on the host geometry: the device stores only the
// non-zero, independent entries
bool geometry_layout_ok(const Dims &d, const double *gcov, const double *gcon, const double *conn, std::string &why)
{
  static const int zero_slots[6][2] = {{0, 2}, {1, 2}, {2, 0}, {2, 1}, {2, 3}, {3, 2}};
  for (long c = 0; c < d.plane(); c++)
    for (int loc = 0; loc < 5; loc++) {
      const double *a = gcov + (c * 5 + loc) * 16, *b = gcon + (c * 5 + loc) * 16;
      for (auto &z : zero_slots)
        if (a[z[0] * 4 + z[1]] != 0. || b[z[0] * 4 + z[1]] != 0.) { why = "metric entry expected to vanish is non-zero"; return false; }
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
          if (a[m * 4 + n] != a[n * 4 + m]) { why = "gcov not symmetric"; return false; }
    }
  for (long c = 0; c < d.plane(); c++)
    for (int k = 0; k < 4; k++)
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
          if (conn[c * 64 + k * 16 + a * 4 + b] != conn[c * 64 + k * 16 + b * 4 + a]) {
            why = "connection not symmetric in its lower indices";
            return false;
          }
  return true;
}

}  // namespace harm

using namespace harm;

namespace harm {
int launch_step(Ctx *x);
}


extern "C" const char *harm_last_error(void) { return g_err.c_str(); }

extern "C" int harm_create(const harm_params *prm, const double *gcov, const double *gcon, const double *gdet,
                           const double *conn, const double *coords, const double *katm, int device,
                           harm_ctx **out)
{
  if (!prm || !gcov || !gcon || !gdet || !conn || !coords || !katm || !out) return fail_with(HARM_E_ARG, "null argument");
  if (!valid_grid(prm->n1, prm->n2, prm->n3)) return fail_with(HARM_E_ARG, "grid must have n1>=4, n2>=8, n3==1 or even n3>=4");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
    return fail_with(HARM_E_NODEV, "no CUDA device");
  cudaDeviceProp dp;
  CK(cudaGetDeviceProperties(&dp, device));
  if (dp.major != 10) return fail_with(HARM_E_NODEV, "the library is compiled for sm_100a (B200)");
  Dims d = make_dims(prm->n1, prm->n2, prm->n3);
  std::string why;
  if (!geometry_layout_ok(d, gcov, gcon, conn, why)) return fail_with(HARM_E_ARG, why);
  CK(cudaSetDevice(device));
  harm_ctx *h = new harm_ctx();
  Ctx *x = &h->x;
  std::memset(x, 0, sizeof(Ctx));
  x->D = d;
  x->prm = *prm;
  x->device = device;
  Grid &G = x->G;
  G.n1 = d.n1; G.n2 = d.n2; G.n3 = d.n3; G.sn1 = d.sn1; G.sn2 = d.sn2;
  G.istart = d.istart; G.istop = d.istop; G.jstart = d.jstart; G.jstop = d.jstop;
  G.ng = (long)d.sn1 * d.sn2;
  G.nc = (long)d.n3 * G.ng;
  G.lim = prm->lim;
  G.gam = prm->gam; G.cour = prm->cour; G.defcon = prm->defcon; G.tf = prm->tf;
  G.dx1 = prm->dx[1]; G.dx2 = prm->dx[2]; G.dx3 = prm->dx[3];
  G.idx1 = 1. / G.dx1; G.idx2 = 1. / G.dx2; G.idx3 = 1. / G.dx3;
  // the mixed path keeps the connection source in FP64 within 2 r_H of the
  // black hole (r from the Boyer-Lindquist coordinates of the zone centres)
  {
    const double rH = 1. + sqrt(1. - prm->a * prm->a);
    G.isrc32 = G.istop + 1;
    for (int i = G.istart; i <= G.istop; i++)
      if (coords[((long)i * d.sn2 + G.jstart) * 4 + 1] >= 2. * rH) { G.isrc32 = i; break; }
  }
  x->nparts = 148 * 4;
  x->tbx = 32;
  x->tby = 4;
  auto al = [&](void **p, size_t b) -> int { CK(cudaMalloc(p, b)); return HARM_OK; };
  const size_t st = 8 * G.nc * sizeof(double);
  int rc = HARM_OK;
  rc |= al((void **)&x->p, st);
  rc |= al((void **)&x->ph, st);
  rc |= al((void **)&x->F1, st);
  rc |= al((void **)&x->F2, st);
  rc |= al((void **)&x->F3, d.n3 > 1 ? st : 8);
  rc |= al((void **)&x->pflag, G.nc);
  rc |= al((void **)&x->geo, 4 * GEO_N * G.ng * sizeof(double));
  rc |= al((void **)&x->conn, 40 * G.ng * sizeof(double));
  rc |= al((void **)&x->floors, 2 * G.ng * sizeof(double));
  rc |= al((void **)&x->katm, d.sn1 * sizeof(double));
  rc |= al((void **)&x->stage, (size_t)8 * d.cells() * sizeof(double));
  rc |= al((void **)&x->stage_flag, d.cells());
  rc |= al((void **)&x->fail_list, FAIL_CAP * sizeof(int));
  rc |= al((void **)&x->fix_buf, FAIL_CAP * 8 * sizeof(double));
  rc |= al((void **)&x->partials, 3 * x->nparts * sizeof(double));
  rc |= al((void **)&x->sc, sizeof(DevScalars));
  rc |= al((void **)&x->Ubuf, st);
  rc |= al((void **)&x->emf, 3 * G.nc * sizeof(double));
  rc |= al((void **)&x->coolgeo, 2 * G.ng * sizeof(double));
  if (rc != HARM_OK) { harm_destroy(h); return HARM_E_CUDA; }
  if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) { harm_destroy(h); return fail_with(HARM_E_CUDA, "stream"); }
  // geometry planes
  std::vector<double> hg((size_t)4 * GEO_N * G.ng), hc((size_t)40 * G.ng), hf((size_t)2 * G.ng);
  static const int locs[4] = {0 /*FACE1*/, 1 /*FACE2*/, 4 /*FACE3*/, 3 /*CENT*/};
  for (int L = 0; L < 4; L++)
    for (long c = 0; c < G.ng; c++) {
      const double *a = gcov + (c * 5 + locs[L]) * 16, *b = gcon + (c * 5 + locs[L]) * 16;
      const double alpha = 1. / sqrt(-b[0]), g = gdet[c * 5 + locs[L]];
      const double vals[GEO_N] = {a[0], a[1], a[3], a[5], a[7], a[10], a[15],
                                  b[0], b[1], b[3], b[4], b[5], b[7], b[10], b[12], b[13], b[15],
                                  g, alpha, 1. / alpha, 1. / g};
      for (int e = 0; e < GEO_N; e++) hg[((size_t)L * GEO_N + e) * G.ng + c] = vals[e];
    }
  for (long c = 0; c < G.ng; c++)
    for (int k = 0; k < 4; k++)
      for (int lo = 0; lo < 4; lo++)
        for (int hi = lo; hi < 4; hi++) {
          int pair = lo == 0 ? hi : lo == 1 ? 3 + hi : lo == 2 ? 5 + hi : 9;
          hc[(size_t)(k * 10 + pair) * G.ng + c] = conn[c * 64 + k * 16 + lo * 4 + hi];
        }
  // radial floors get_rho_u_floor() (fixup.c:117-140), evaluated on the host
  radial_floors(coords, prm->gam, G.ng, hf.data());
  // zone-centre r and |r tan theta| (get_coord, metric.c:446-458; diag.c:238-242)
  std::vector<double> hcg((size_t)2 * G.ng);
  for (long c = 0; c < G.ng; c++) {
    const double r = coords[c * 4 + 1], th = coords[c * 4 + 2];
    hcg[c] = r;
    hcg[G.ng + c] = fabs(r * tan(th));
  }
  DevScalars s0;
  std::memset(&s0, 0, sizeof(s0));
  unsigned long long big;
  double b9 = 1.e9;
  std::memcpy(&big, &b9, 8);
  s0.ndt_bits[0] = s0.ndt_bits[1] = s0.ndt_bits[2] = big;
  s0.dt = 1.e-5;
  if (cudaMemcpy(x->geo, hg.data(), hg.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->conn, hc.data(), hc.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->floors, hf.data(), hf.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->coolgeo, hcg.data(), hcg.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->katm, katm, d.sn1 * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(x->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(x->p, 0, st) != cudaSuccess || cudaMemset(x->ph, 0, st) != cudaSuccess ||
      cudaMemset(x->F1, 0, st) != cudaSuccess || cudaMemset(x->F2, 0, st) != cudaSuccess ||
      cudaMemset(x->pflag, 0, G.nc) != cudaSuccess) {
    harm_destroy(h);
    return fail_with(HARM_E_CUDA, "upload");
  }
  *out = h;
  return HARM_OK;
}

extern "C" void harm_destroy(harm_ctx *h)
{
  if (!h) return;
  Ctx *x = &h->x;
  if (x->graph_exec) cudaGraphExecDestroy(x->graph_exec);
  void *ptrs[] = {x->p, x->ph, x->F1, x->F2, x->F3, x->pflag, x->geo, x->conn, x->floors, x->katm,
                  x->stage, x->stage_flag, x->fail_list, x->fix_buf, x->partials, x->sc,
                  x->F1f, x->F2f, x->F3f, x->geo32, x->conn32, x->Ubuf, x->emf, x->trX, x->trids, x->trst,
                  x->lastT, x->coolgeo, x->cooldiag};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (x->pinned) cudaFreeHost(x->pinned);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete h;
}

static int put_prims(Ctx *x, const double *p, const signed char *pflag, double *dst)
{
  const Dims &d = x->D;
  const int h0 = d.n3 > 1 ? 1 : 0;
  const size_t nb = (size_t)8 * d.cells() * sizeof(double);
  CK(cudaMemcpyAsync(x->stage, p, nb, cudaMemcpyHostToDevice, x->stream));
  if (pflag) CK(cudaMemcpyAsync(x->stage_flag, pflag, d.cells(), cudaMemcpyHostToDevice, x->stream));
  k_from_host<<<148 * 8, 256, 0, x->stream>>>(x->G, h0, x->stage, dst, pflag ? x->stage_flag : nullptr, x->pflag);
  CK(cudaGetLastError());
  return HARM_OK;
}

int harm::get_prims(Ctx *x, const double *src, double *p, signed char *pflag)
{
  const Dims &d = x->D;
  const int h0 = d.n3 > 1 ? 1 : 0;
  k_to_host<<<148 * 8, 256, 0, x->stream>>>(x->G, h0, src, x->stage, x->pflag, pflag ? x->stage_flag : nullptr);
  CK(cudaGetLastError());
  const size_t nb = (size_t)8 * d.cells() * sizeof(double);
  if (p) CK(cudaMemcpyAsync(p, x->stage, nb, cudaMemcpyDeviceToHost, x->stream));
  if (pflag) CK(cudaMemcpyAsync(pflag, x->stage_flag, d.cells(), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return HARM_OK;
}

extern "C" int harm_put_prims(harm_ctx *h, const double *p, const signed char *pflag)
{
  if (!h || !p) return fail_with(HARM_E_ARG, "null argument");
  int rc = put_prims(&h->x, p, pflag, h->x.p);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->x.stream));
  return HARM_OK;
}

extern "C" int harm_get_prims(harm_ctx *h, double *p, signed char *pflag)
{
  if (!h || (!p && !pflag)) return fail_with(HARM_E_ARG, "null argument");
  return get_prims(&h->x, h->x.p, p, pflag);
}

static int read_scalars(Ctx *x, DevScalars *s)
{
  CK(cudaMemcpyAsync(s, x->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return HARM_OK;
}

static int write_scalars(Ctx *x, const DevScalars *s)
{
  CK(cudaMemcpyAsync(x->sc, s, sizeof(DevScalars), cudaMemcpyHostToDevice, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return HARM_OK;
}

extern "C" int harm_set_time(harm_ctx *h, double t, double dt)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  DevScalars s;
  int rc = read_scalars(&h->x, &s);
  if (rc) return rc;
  s.t = t;
  s.dt = dt;
  s.err = 0;
  s.halted = 0;
  s.fail_code = 0;
  return write_scalars(&h->x, &s);
}

extern "C" int harm_get_time(harm_ctx *h, double *t, double *dt)
{
  if (!h || !t || !dt) return fail_with(HARM_E_ARG, "null argument");
  DevScalars s;
  int rc = read_scalars(&h->x, &s);
  if (rc) return rc;
  *t = s.t;
  *dt = s.dt;
  return HARM_OK;
}

extern "C" int harm_set_mass(harm_ctx *h, double mass_in, double mass_out)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  DevScalars s;
  int rc = read_scalars(&h->x, &s);
  if (rc) return rc;
  s.mass_in = mass_in;
  s.mass_out = mass_out;
  return write_scalars(&h->x, &s);
}

extern "C" int harm_get_diag(harm_ctx *h, harm_diag *d)
{
  if (!h || !d) return fail_with(HARM_E_ARG, "null argument");
  DevScalars s;
  int rc = read_scalars(&h->x, &s);
  if (rc) return rc;
  d->mdot = s.mdot; d->edot = s.edot; d->ldot = s.ldot;
  d->mdot_in = s.mdot_in; d->mdot_out = s.mdot_out; d->mass_curr = s.mass_curr;
  d->mass_in = s.mass_in; d->mass_out = s.mass_out; d->ndt = s.ndt;
  d->fail_code = s.fail_code; d->fail_h = s.fail_h; d->fail_i = s.fail_i; d->fail_j = s.fail_j;
  return HARM_OK;
}

namespace harm {
int sync_status(Ctx *x)
{
  CK(cudaStreamSynchronize(x->stream));
  CK(cudaGetLastError());
  DevScalars s;
  int rc = read_scalars(x, &s);
  if (rc) return rc;
  if (s.err) return fail_with(s.err, "dt < 1e-9 (the reference exits with code 11)");
  return HARM_OK;
}
}  // namespace harm

extern "C" int harm_sync(harm_ctx *h)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  return sync_status(&h->x);
}

extern "C" int harm_set_precision(harm_ctx *h, int mode)
{
  if (!h || (mode != HARM_FP64 && mode != HARM_MIXED)) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  if (x->cool && mode == HARM_MIXED && !x->eos.f32) return fail_with(HARM_E_ARG, "table values span more than float holds");
  if (mode == HARM_MIXED && !x->F1f) {
    const Grid &G = x->G;
    const size_t fb = 8 * G.nc * sizeof(float);
    CK(cudaMalloc(&x->F1f, fb));
    CK(cudaMalloc(&x->F2f, fb));
    CK(cudaMalloc(&x->F3f, G.n3 > 1 ? fb : 8));
    CK(cudaMalloc(&x->geo32, (size_t)4 * GEO_N * G.ng * sizeof(float)));
    CK(cudaMalloc(&x->conn32, (size_t)40 * G.ng * sizeof(float)));
    // FP32 copies of the metric at FACE1, FACE2, FACE3, CENT and of the connection
    std::vector<double> hg((size_t)4 * GEO_N * G.ng);
    std::vector<float> hf(hg.size());
    CK(cudaMemcpy(hg.data(), x->geo, hg.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < hg.size(); k++) hf[k] = (float)hg[k];
    CK(cudaMemcpy(x->geo32, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<double> hc((size_t)40 * G.ng);
    std::vector<float> hcf(hc.size());
    CK(cudaMemcpy(hc.data(), x->conn, hc.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < hc.size(); k++) hcf[k] = (float)hc[k];
    CK(cudaMemcpy(x->conn32, hcf.data(), hcf.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (mode != x->mode && x->graph_exec) {
    cudaGraphExecDestroy(x->graph_exec);
    x->graph_exec = nullptr;
  }
  x->mode = mode;
  return HARM_OK;
}

extern "C" int harm_step_ch(harm_ctx *h)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  return launch_step(&h->x);
}

extern "C" int harm_run(harm_ctx *h, int nsteps)
{
  if (!h || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  if (x->cool && x->cool_seed) {
    // the seeding step runs outside the graph, which holds the ordinary step
    if (nsteps == 0) return HARM_OK;
    int rc = launch_step(x);
    if (rc) return rc;
    nsteps--;
  }
  if (!x->graph_exec) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch_step(x);
    cudaError_t e = cudaStreamEndCapture(x->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&x->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
  }
  for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(x->graph_exec, x->stream));
  return harm_sync(h);
}

extern "C" int harm_step_ch_host(harm_ctx *h, double *p)
{
  if (!h || !p) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  int rc = put_prims(x, p, nullptr, x->p);
  if (rc) return rc;
  rc = launch_step(x);
  if (rc) return rc;
  return get_prims(x, x->p, p, nullptr);
}

// the per-array entry points: upload into the half-step buffer, run, download
static int on_host_array(harm_ctx *h, double *pv, int which)
{
  if (!h || !pv) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  int rc = put_prims(x, pv, nullptr, x->ph);
  if (rc) return rc;
  const Grid &G = x->G;
  if (which == 0) {
    k_fixup<<<zone_grid(G), dim3(32, 4), 0, x->stream>>>(G, x->ph, x->pflag, x->geo, x->floors, x->sc);
  } else if (which == 1) {
    launch_bound(x, x->ph);
  } else {
    launch_fixup_utoprim(x, x->ph);
  }
  CK(cudaGetLastError());
  return get_prims(x, x->ph, pv, nullptr);
}

// fixup1zone() (fixup.c:142-383) at listed zones of the context's grid
__global__ void k_fixup_zones(Grid G, long n, const int *__restrict__ hij, double *pv, signed char *flag,
                              const double *__restrict__ geo, const double *__restrict__ floors, DevScalars *sc)
{
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int h = hij[3 * t], i = hij[3 * t + 1], j = hij[3 * t + 2];
  const long gi = (long)i * G.sn2 + j;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double v[8];
  for (int k = 0; k < 8; k++) v[k] = pv[8 * t + k];
  int fail = 0;
  flag[t] = fixup1zone(G.gam, floors[gi], floors[G.ng + gi], q, v, &fail) ? -33 : 0;
  if (fail) record_fail(sc, fail, h, i, j);
  for (int k = 0; k < 8; k++) pv[8 * t + k] = v[k];
}

extern "C" int harm_fixup1zone(harm_ctx *h, long n, const int *hij, double *pv, signed char *flag)
{
  if (!h || !hij || !pv || !flag || n < 0) return fail_with(HARM_E_ARG, "harm_fixup1zone: bad arguments");
  if (n == 0) return HARM_OK;
  Ctx *x = &h->x;
  const Grid &G = x->G;
  for (long t = 0; t < n; t++) {
    const int hh = hij[3 * t], i = hij[3 * t + 1], j = hij[3 * t + 2];
    if (hh < 0 || hh >= x->D.sn3 || i < 0 || i >= G.sn1 || j < 0 || j >= G.sn2)
      return fail_with(HARM_E_ARG, "harm_fixup1zone: zone outside the grid");
  }
  CK(cudaSetDevice(x->device));
  int *dh = nullptr;
  double *dp = nullptr;
  signed char *df = nullptr;
  CK(cudaMalloc(&dh, 3 * n * sizeof(int)));
  CK(cudaMalloc(&dp, 8 * n * sizeof(double)));
  CK(cudaMalloc(&df, n));
  int rc = HARM_OK;
  if (cudaMemcpyAsync(dh, hij, 3 * n * sizeof(int), cudaMemcpyHostToDevice, x->stream) != cudaSuccess ||
      cudaMemcpyAsync(dp, pv, 8 * n * sizeof(double), cudaMemcpyHostToDevice, x->stream) != cudaSuccess)
    rc = fail_with(HARM_E_CUDA, "harm_fixup1zone: upload");
  if (rc == HARM_OK) {
    k_fixup_zones<<<(unsigned)((n + 127) / 128), 128, 0, x->stream>>>(G, n, dh, dp, df, x->geo, x->floors, x->sc);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(pv, dp, 8 * n * sizeof(double), cudaMemcpyDeviceToHost, x->stream) != cudaSuccess ||
        cudaMemcpyAsync(flag, df, n, cudaMemcpyDeviceToHost, x->stream) != cudaSuccess ||
        cudaStreamSynchronize(x->stream) != cudaSuccess)
      rc = fail_with(HARM_E_CUDA, "harm_fixup1zone: launch");
  }
  cudaFree(dh);
  cudaFree(dp);
  cudaFree(df);
  return rc;
}

extern "C" int harm_fixup(harm_ctx *h, double *pv) { return on_host_array(h, pv, 0); }
extern "C" int harm_bound_prim(harm_ctx *h, double *pv) { return on_host_array(h, pv, 1); }
extern "C" int harm_fixup_utoprim(harm_ctx *h, double *pv) { return on_host_array(h, pv, 2); }

extern "C" int harm_utoprim_2d_batch(const double *U, const double *gcov, const double *gcon, const double *gdet,
                                     double *prim, int *ret, long n, double gam)
{
  if (!U || !gcov || !gcon || !gdet || !prim || !ret || n < 0) return fail_with(HARM_E_ARG, "null argument");
  if (n == 0) return HARM_OK;
  // device copies, freed on every return
  struct Buffers {
    double *dU = nullptr, *da = nullptr, *db = nullptr, *dg = nullptr, *dp = nullptr;
    int *dr = nullptr;
    ~Buffers() { cudaFree(dU); cudaFree(da); cudaFree(db); cudaFree(dg); cudaFree(dp); cudaFree(dr); }
  } B;
  double *&dU = B.dU, *&da = B.da, *&db = B.db, *&dg = B.dg, *&dp = B.dp;
  int *&dr = B.dr;
  CK(cudaMalloc(&dU, n * 8 * 8));
  CK(cudaMalloc(&da, n * 16 * 8));
  CK(cudaMalloc(&db, n * 16 * 8));
  CK(cudaMalloc(&dg, n * 8));
  CK(cudaMalloc(&dp, n * 8 * 8));
  CK(cudaMalloc(&dr, n * sizeof(int)));
  CK(cudaMemcpy(dU, U, n * 64, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(da, gcov, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(db, gcon, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dg, gdet, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dp, prim, n * 64, cudaMemcpyHostToDevice));
  k_utoprim_batch<<<(unsigned)((n + 127) / 128), 128>>>(dU, da, db, dg, dp, dr, n, gam);
  CK(cudaGetLastError());
  CK(cudaMemcpy(prim, dp, n * 64, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ret, dr, n * sizeof(int), cudaMemcpyDeviceToHost));
  return HARM_OK;
}

extern "C" int harm_utoprim_fix_batch(int which, const double *U, const double *gcov, const double *gcon,
                                      const double *gdet, const double *K, double *prim, int *ret, long n, double gam)
{
  if ((which != 1 && which != 2) || !U || !gcov || !gcon || !gdet || !K || !prim || !ret || n < 0)
    return fail_with(HARM_E_ARG, "harm_utoprim_fix_batch: bad arguments");
  if (n == 0) return HARM_OK;
  struct Buffers {
    double *dU = nullptr, *da = nullptr, *db = nullptr, *dg = nullptr, *dk = nullptr, *dp = nullptr;
    int *dr = nullptr;
    ~Buffers() { cudaFree(dU); cudaFree(da); cudaFree(db); cudaFree(dg); cudaFree(dk); cudaFree(dp); cudaFree(dr); }
  } B;
  CK(cudaMalloc(&B.dU, n * 8 * 8));
  CK(cudaMalloc(&B.da, n * 16 * 8));
  CK(cudaMalloc(&B.db, n * 16 * 8));
  CK(cudaMalloc(&B.dg, n * 8));
  CK(cudaMalloc(&B.dk, n * 8));
  CK(cudaMalloc(&B.dp, n * 8 * 8));
  CK(cudaMalloc(&B.dr, n * sizeof(int)));
  CK(cudaMemcpy(B.dU, U, n * 64, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.da, gcov, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.db, gcon, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.dg, gdet, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.dk, K, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.dp, prim, n * 64, cudaMemcpyHostToDevice));
  k_utoprim_fix_batch<<<(unsigned)((n + 127) / 128), 128>>>(which, B.dU, B.da, B.db, B.dg, B.dk, B.dp, B.dr, n, gam);
  CK(cudaGetLastError());
  CK(cudaMemcpy(prim, B.dp, n * 64, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ret, B.dr, n * sizeof(int), cudaMemcpyDeviceToHost));
  return HARM_OK;
}

extern "C" int harm_pow_batch(int device, const double *x, const double *y, double *out, long n)
{
  if (!x || !y || !out || n < 0) return fail_with(HARM_E_ARG, "harm_pow_batch: bad arguments");
  if (n == 0) return HARM_OK;
  CK(cudaSetDevice(device));
  struct Buffers {
    double *dx = nullptr, *dy = nullptr, *dz = nullptr;
    ~Buffers() { cudaFree(dx); cudaFree(dy); cudaFree(dz); }
  } B;
  CK(cudaMalloc(&B.dx, n * 8));
  CK(cudaMalloc(&B.dy, n * 8));
  CK(cudaMalloc(&B.dz, n * 8));
  CK(cudaMemcpy(B.dx, x, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.dy, y, n * 8, cudaMemcpyHostToDevice));
  k_pow_batch<<<(unsigned)((n + 127) / 128), 128>>>(B.dx, B.dy, B.dz, n);
  CK(cudaGetLastError());
  CK(cudaMemcpy(out, B.dz, n * 8, cudaMemcpyDeviceToHost));
  return HARM_OK;
}

// init(): torus fields on the host, floors and boundaries on the device, the
// loop potential on the host, its normalisation on the device (init.c:70-472)
extern "C" int harm_init_torus(harm_ctx *h, const harm_grid_spec *g, const harm_torus_spec *tor)
{
  if (!h || !g || !tor) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Dims &d = x->D;
  if (g->n1 != d.n1 || g->n2 != d.n2 || g->n3 != d.n3) return fail_with(HARM_E_ARG, "grid spec does not match the context");
  const size_t ncell = (size_t)d.cells();
  std::vector<double> p(ncell * 8, 0.), gcov, gcon((size_t)d.plane() * 80), gdet((size_t)d.plane() * 5);
  // the torus velocity transform needs the CENT inverse metric; recompute the grid on the host
  {
    std::vector<double> gv((size_t)d.plane() * 80), cn((size_t)d.plane() * 64), co((size_t)d.plane() * 4);
    int rc = harm_set_grid(g, x->prm.dx, x->prm.startx, gv.data(), gcon.data(), gdet.data(), cn.data(), co.data());
    if (rc) return rc;
    gcov.swap(gv);
  }
  double rhomax, umax;
  torus_hydro(*g, x->prm, *tor, gcov.data(), gcon.data(), p.data(), &rhomax, &umax);
  for (int hh = d.hstart; hh <= d.hstop; hh++)
    for (int i = d.istart; i <= d.istop; i++)
      for (int j = d.jstart; j <= d.jstop; j++) {
        double *pz = p.data() + (((size_t)hh * d.sn1 + i) * d.sn2 + j) * 8;
        pz[0] /= rhomax;
        pz[1] /= rhomax;
      }
  umax /= rhomax;
  int rc = harm_put_prims(h, p.data(), nullptr);
  if (rc) return rc;
  const Grid &G = x->G;
  k_fixup<<<zone_grid(G), dim3(32, 4), 0, x->stream>>>(G, x->p, x->pflag, x->geo, x->floors, x->sc);
  launch_bound(x, x->p);
  rc = get_prims(x, x->p, p.data(), nullptr);
  if (rc) return rc;
  torus_field(d, x->prm, gdet.data(), p.data());
  rc = harm_put_prims(h, p.data(), nullptr);
  if (rc) return rc;
  DevScalars s;
  rc = read_scalars(x, &s);
  if (rc) return rc;
  s.bsq_bits = 0;
  rc = write_scalars(x, &s);
  if (rc) return rc;
  k_bsq_max<<<zone_grid(G), dim3(32, 4), 0, x->stream>>>(G, x->p, x->geo, x->sc);
  rc = read_scalars(x, &s);
  if (rc) return rc;
  double bsq_max;
  std::memcpy(&bsq_max, &s.bsq_bits, 8);
  double beta_act = (x->prm.gam - 1.) * umax / (0.5 * bsq_max);
  double norm = sqrt(beta_act / tor->beta);
  k_scale_field<<<zone_grid(G), dim3(32, 4), 0, x->stream>>>(G, x->p, norm);
  k_fixup<<<zone_grid(G), dim3(32, 4), 0, x->stream>>>(G, x->p, x->pflag, x->geo, x->floors, x->sc);
  launch_bound(x, x->p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(x->stream));
  // main(): t = 0, dt = 1e-5 (init.c:122-123), mass counters from zero
  rc = read_scalars(x, &s);
  if (rc) return rc;
  s.t = 0.;
  s.dt = 1.e-5;
  s.mass_in = s.mass_out = 0.;
  s.fail_code = 0;
  s.err = 0;
  s.halted = 0;
  return write_scalars(x, &s);
}

// ---------------------------------------------------------------------------
// device-timed entry points

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair()
  {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

extern "C" int harm_run_timed(harm_ctx *h, int nsteps, double *ms)
{
  if (!h || !ms || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  int rc = harm_run(h, 0);  // capture the graph outside the timed region
  if (rc) return rc;
  if (!x->graph_exec) return fail_with(HARM_E_ARG, "COOL_EOS: run the seeding step before timing");
  EventPair e;
  CK(cudaEventCreate(&e.a));
  CK(cudaEventCreate(&e.b));
  CK(cudaEventRecord(e.a, x->stream));
  for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(x->graph_exec, x->stream));
  CK(cudaEventRecord(e.b, x->stream));
  CK(cudaEventSynchronize(e.b));
  float f;
  CK(cudaEventElapsedTime(&f, e.a, e.b));
  *ms = f;
  return harm_sync(h);
}

// nsteps of (upload p, step, download into p), the state passing through the
// host array between steps, as nsteps calls of harm_step_ch_host move it.
// The copies run on two streams of their own, cut into chunks: the upload of
// chunk c for step s+1 waits only for the download of chunk c of step s, so
// the two directions of the link carry the two copies at once.  Both copies
// go through the staging buffer, chunk by chunk in the same order, and the
// layout kernels wait for a whole copy.  *ms (may be NULL): the device time
// from the first upload to the last download.
static int run_host(Ctx *x, double *p, int nsteps, double *ms)
{
  const int h0 = x->D.n3 > 1 ? 1 : 0;
  const size_t nb = (size_t)8 * x->D.cells() * sizeof(double);
  constexpr int C = 16;
  const size_t chunk = ((nb / C + 4095) / 4096) * 4096;
  struct Res {
    cudaStream_t up = nullptr, dn = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr, ready = nullptr, uploaded = nullptr, done = nullptr, dc[C] = {};
    ~Res()
    {
      for (cudaEvent_t e : dc)
        if (e) cudaEventDestroy(e);
      for (cudaEvent_t e : {t0, t1, ready, uploaded, done})
        if (e) cudaEventDestroy(e);
      if (up) cudaStreamDestroy(up);
      if (dn) cudaStreamDestroy(dn);
    }
  } r;
  CK(cudaStreamCreateWithFlags(&r.up, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&r.dn, cudaStreamNonBlocking));
  CK(cudaEventCreate(&r.t0));
  CK(cudaEventCreate(&r.t1));
  for (cudaEvent_t *e : {&r.ready, &r.uploaded, &r.done}) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (cudaEvent_t &e : r.dc) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaEventRecord(r.t0, x->stream));
  CK(cudaStreamWaitEvent(r.up, r.t0, 0));
  for (int s = 0; s < nsteps; s++) {
    for (int c = 0; c < C; c++) {
      const size_t off = c * chunk;
      if (off >= nb) break;
      if (s > 0) CK(cudaStreamWaitEvent(r.up, r.dc[c], 0));
      CK(cudaMemcpyAsync((char *)x->stage + off, (const char *)p + off, nb - off < chunk ? nb - off : chunk,
                         cudaMemcpyHostToDevice, r.up));
    }
    CK(cudaEventRecord(r.uploaded, r.up));
    CK(cudaStreamWaitEvent(x->stream, r.uploaded, 0));
    k_from_host<<<148 * 8, 256, 0, x->stream>>>(x->G, h0, x->stage, x->p, nullptr, x->pflag);
    CK(cudaGetLastError());
    int rc = launch_step(x);
    if (rc) return rc;
    k_to_host<<<148 * 8, 256, 0, x->stream>>>(x->G, h0, x->p, x->stage, x->pflag, nullptr);
    CK(cudaGetLastError());
    CK(cudaEventRecord(r.ready, x->stream));
    CK(cudaStreamWaitEvent(r.dn, r.ready, 0));
    for (int c = 0; c < C; c++) {
      const size_t off = c * chunk;
      if (off >= nb) break;
      CK(cudaMemcpyAsync((char *)p + off, (const char *)x->stage + off, nb - off < chunk ? nb - off : chunk,
                         cudaMemcpyDeviceToHost, r.dn));
      CK(cudaEventRecord(r.dc[c], r.dn));
    }
  }
  CK(cudaEventRecord(r.done, r.dn));
  CK(cudaStreamWaitEvent(x->stream, r.done, 0));
  CK(cudaEventRecord(r.t1, x->stream));
  CK(cudaEventSynchronize(r.t1));
  if (ms) {
    float f;
    CK(cudaEventElapsedTime(&f, r.t0, r.t1));
    *ms = f;
  }
  return HARM_OK;
}

extern "C" int harm_run_host(harm_ctx *h, double *p, int nsteps)
{
  if (!h || !p || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  int rc = run_host(&h->x, p, nsteps, nullptr);
  if (rc) return rc;
  return harm_sync(h);
}

extern "C" int harm_step_ch_host_timed(harm_ctx *h, double *p, int nsteps, double *ms)
{
  if (!h || !p || !ms || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  int rc = run_host(&h->x, p, nsteps, ms);
  if (rc) return rc;
  return harm_sync(h);
}

extern "C" int harm_time_kernels(harm_ctx *h, int reps, double *ms)
{
  if (!h || !ms || reps < 1) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  if (x->cool) return cool_time_kernels(x, reps, ms);
  return x->mode == HARM_MIXED ? mixed::time_kernels(x, reps, ms) : exact::time_kernels(x, reps, ms);
}

// ---------------------------------------------------------------------------
// tile shapes and their autotuner

static bool tile_ok(int bx, int by) { return bx >= 8 && by >= 1 && bx * by == 128 && (bx & 7) == 0; }


extern "C" int harm_set_tile(harm_ctx *h, int bx, int by)
{
  if (!h || !tile_ok(bx, by)) return fail_with(HARM_E_ARG, "tile must be bx x by = 128 threads, bx a multiple of 8");
  Ctx *x = &h->x;
  if (x->tbx != bx || x->tby != by) invalidate_graph(x);
  x->tbx = bx;
  x->tby = by;
  return HARM_OK;
}

extern "C" int harm_get_tile(harm_ctx *h, int *bx, int *by)
{
  if (!h || !bx || !by) return fail_with(HARM_E_ARG, "null argument");
  *bx = h->x.tbx;
  *by = h->x.tby;
  return HARM_OK;
}

// Times `steps` ordinary steps per candidate tile, each trial from the same
// saved state (primitives, flags, run scalars), and keeps the fastest; the
// state is restored afterwards, so the run continues as if untouched.
extern "C" int harm_autotune_tile(harm_ctx *h, int steps, int *bx, int *by)
{
  if (!h || steps < 1) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  if (x->cool) return fail_with(HARM_E_ARG, "the tile autotuner is for the gamma-law step");
  static const int cand[][2] = {{32, 4}, {64, 2}, {16, 8}, {128, 1}};
  const size_t pb = (size_t)8 * x->G.nc * sizeof(double);
  DevScalars s0;
  int rc = read_scalars(x, &s0);
  if (rc) return rc;
  CK(cudaMemcpyAsync(x->stage, x->p, pb, cudaMemcpyDeviceToDevice, x->stream));
  CK(cudaMemcpyAsync(x->stage_flag, x->pflag, x->G.nc, cudaMemcpyDeviceToDevice, x->stream));
  const int keep_x = x->tbx, keep_y = x->tby;
  EventPair e;
  CK(cudaEventCreate(&e.a));
  CK(cudaEventCreate(&e.b));
  float best = -1.f;
  int bi = 0;
  for (int c = 0; c < 4; c++) {
    x->tbx = cand[c][0];
    x->tby = cand[c][1];
    rc = launch_step(x);  // warm-up, from the saved state
    if (!rc) {
      CK(cudaEventRecord(e.a, x->stream));
      for (int s = 0; s < steps && !rc; s++) rc = launch_step(x);
      CK(cudaEventRecord(e.b, x->stream));
      CK(cudaEventSynchronize(e.b));
      float f;
      CK(cudaEventElapsedTime(&f, e.a, e.b));
      if (best < 0.f || f < best) { best = f; bi = c; }
    }
    // back to the saved state for the next candidate (and for the caller)
    CK(cudaMemcpyAsync(x->p, x->stage, pb, cudaMemcpyDeviceToDevice, x->stream));
    CK(cudaMemcpyAsync(x->pflag, x->stage_flag, x->G.nc, cudaMemcpyDeviceToDevice, x->stream));
    int wr = write_scalars(x, &s0);
    if (wr) return wr;
    if (rc) {
      x->tbx = keep_x;
      x->tby = keep_y;
      return rc;
    }
  }
  invalidate_graph(x);
  x->tbx = cand[bi][0];
  x->tby = cand[bi][1];
  if (bx) *bx = x->tbx;
  if (by) *by = x->tby;
  return sync_status(x);
}

// ---------------------------------------------------------------------------
// ensembles: independent grids advanced together by one graph launch per step

struct harm_ensemble {
  std::vector<Ctx *> members;
  std::vector<int> mode, tbx, tby;  // member settings the graph was captured with
  std::vector<long> ntr;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
};

static void ensemble_free(harm_ensemble *e)
{
  if (e->exec) cudaGraphExecDestroy(e->exec);
  for (cudaEvent_t v : e->join) if (v) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

extern "C" int harm_ensemble_create(harm_ctx *const *members, int n, harm_ensemble **out)
{
  if (!members || n < 1 || !out) return fail_with(HARM_E_ARG, "bad argument");
  for (int k = 0; k < n; k++) {
    if (!members[k]) return fail_with(HARM_E_ARG, "null member");
    if (members[k]->x.cool) return fail_with(HARM_E_ARG, "ensembles hold gamma-law members");
    if (members[k]->x.device != members[0]->x.device) return fail_with(HARM_E_ARG, "members on different devices");
    for (int m = 0; m < k; m++)
      if (members[m] == members[k]) return fail_with(HARM_E_ARG, "a context appears twice");
  }
  harm_ensemble *e = new harm_ensemble();
  e->device = members[0]->x.device;
  for (int k = 0; k < n; k++) e->members.push_back(&members[k]->x);
  e->mode.assign(n, -1);
  e->tbx.assign(n, 0);
  e->tby.assign(n, 0);
  e->ntr.assign(n, -1);
  e->join.assign(n, nullptr);
  if (cudaSetDevice(e->device) != cudaSuccess || cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
    ensemble_free(e);
    return fail_with(HARM_E_CUDA, "ensemble stream");
  }
  for (int k = 0; k < n; k++)
    if (cudaEventCreateWithFlags(&e->join[k], cudaEventDisableTiming) != cudaSuccess) {
      ensemble_free(e);
      return fail_with(HARM_E_CUDA, "ensemble events");
    }
  *out = e;
  return HARM_OK;
}

extern "C" void harm_ensemble_destroy(harm_ensemble *e)
{
  if (e) ensemble_free(e);
}

// (Re)capture when a member's precision or tile changed since the last capture.
static int ensemble_graph(harm_ensemble *e)
{
  bool same = e->exec != nullptr;
  for (size_t k = 0; k < e->members.size() && same; k++) {
    const Ctx *x = e->members[k];
    same = x->mode == e->mode[k] && x->tbx == e->tbx[k] && x->tby == e->tby[k] && x->ntr == e->ntr[k];
  }
  if (same) return HARM_OK;
  if (e->exec) {
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  CK(cudaSetDevice(e->device));
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HARM_OK;
  cudaError_t ce = cudaEventRecord(e->fork, e->stream);
  for (size_t k = 0; k < e->members.size() && ce == cudaSuccess && rc == HARM_OK; k++) {
    Ctx *x = e->members[k];
    ce = cudaStreamWaitEvent(x->stream, e->fork, 0);
    if (ce == cudaSuccess) rc = launch_step(x);
    if (ce == cudaSuccess && rc == HARM_OK) ce = cudaEventRecord(e->join[k], x->stream);
    if (ce == cudaSuccess && rc == HARM_OK) ce = cudaStreamWaitEvent(e->stream, e->join[k], 0);
    e->mode[k] = x->mode;
    e->tbx[k] = x->tbx;
    e->tby[k] = x->tby;
    e->ntr[k] = x->ntr;
  }
  cudaError_t ee = cudaStreamEndCapture(e->stream, &g);
  if (rc) return rc;
  if (ce != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("ensemble capture: ") + cudaGetErrorString(ce));
  if (ee != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("ensemble capture: ") + cudaGetErrorString(ee));
  ce = cudaGraphInstantiate(&e->exec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("ensemble instantiate: ") + cudaGetErrorString(ce));
  return HARM_OK;
}

static int ensemble_status(harm_ensemble *e)
{
  CK(cudaStreamSynchronize(e->stream));
  for (Ctx *x : e->members) {
    int rc = sync_status(x);
    if (rc) return rc;
  }
  return HARM_OK;
}

extern "C" int harm_ensemble_run(harm_ensemble *e, int nsteps)
{
  if (!e || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  int rc = ensemble_graph(e);
  if (rc) return rc;
  for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(e->exec, e->stream));
  return ensemble_status(e);
}

extern "C" int harm_ensemble_run_timed(harm_ensemble *e, int nsteps, double *ms)
{
  if (!e || !ms || nsteps < 0) return fail_with(HARM_E_ARG, "bad argument");
  int rc = ensemble_graph(e);
  if (rc) return rc;
  EventPair ev;
  CK(cudaEventCreate(&ev.a));
  CK(cudaEventCreate(&ev.b));
  CK(cudaEventRecord(ev.a, e->stream));
  for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(e->exec, e->stream));
  CK(cudaEventRecord(ev.b, e->stream));
  CK(cudaEventSynchronize(ev.b));
  float f;
  CK(cudaEventElapsedTime(&f, ev.a, ev.b));
  *ms = f;
  return ensemble_status(e);
}
