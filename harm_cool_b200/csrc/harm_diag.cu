// diag()'s integrals and the divergence of B on the device (diag.c:113-230):
// the sums of U[RHO], U[U3] and U[UU] times dV over the active zones, and the
// largest |div B| in its flux-CT form with the first zone (in the reference's
// h, i, j loop order) where it occurs.  The host reads these at its LOG
// cadence instead of downloading the state.  Built with -fmad=false: every
// zone's U and div B follow the reference's arithmetic; only the order in
// which the sums add up differs (block partials, then a fixed order on the
// host).
#include <vector>

#include "harm_common.cuh"
#include "harm_cool.cuh"

namespace harm {
namespace {

__device__ __forceinline__ double P_(const Grid &G, const double *P, int k, int h, int i, int j)
{
  return __ldg(P + k * G.nc + cidx(G, h, i, j));
}

// |div B| at zone (h, i, j) of device plane h, corner-centred (diag.c:140-200)
__device__ double divb_zone(const Grid &G, const double *P, const double *gd, int h, int i, int j)
{
  const long s = G.sn2;
  const long c = (long)i * s + j;
  const double g00 = __ldg(gd + c), g01 = __ldg(gd + c - 1), g10 = __ldg(gd + c - s), g11 = __ldg(gd + c - s - 1);
  if (G.n3 > 2) {
    const int m = hwrap(G, h - 1);
    return fabs(0.25 * (P_(G, P, B1, h, i, j) * g00 + P_(G, P, B1, m, i, j) * g00
                        + P_(G, P, B1, h, i, j - 1) * g01 + P_(G, P, B1, m, i, j - 1) * g01
                        - P_(G, P, B1, h, i - 1, j) * g10 - P_(G, P, B1, m, i - 1, j) * g10
                        - P_(G, P, B1, h, i - 1, j - 1) * g11 - P_(G, P, B1, m, i - 1, j - 1) * g11) / G.dx1
                + 0.25 * (P_(G, P, B2, h, i, j) * g00 + P_(G, P, B2, m, i, j) * g00
                          + P_(G, P, B2, h, i - 1, j) * g10 + P_(G, P, B2, m, i - 1, j) * g10
                          - P_(G, P, B2, h, i, j - 1) * g01 - P_(G, P, B2, m, i, j - 1) * g01
                          - P_(G, P, B2, h, i - 1, j - 1) * g11 - P_(G, P, B2, m, i - 1, j - 1) * g11) / G.dx2
                + 0.25 * (P_(G, P, B3, h, i, j) * g00 + P_(G, P, B3, h, i - 1, j) * g10
                          + P_(G, P, B3, h, i, j - 1) * g01 + P_(G, P, B3, h, i - 1, j - 1) * g11
                          - P_(G, P, B3, m, i, j) * g00 - P_(G, P, B3, m, i - 1, j) * g10
                          - P_(G, P, B3, m, i, j - 1) * g01 - P_(G, P, B3, m, i - 1, j - 1) * g11) / G.dx3);
  }
  return fabs(0.5 * (P_(G, P, B1, h, i, j) * g00 + P_(G, P, B1, h, i, j - 1) * g01
                     - P_(G, P, B1, h, i - 1, j) * g10 - P_(G, P, B1, h, i - 1, j - 1) * g11) / G.dx1
              + 0.5 * (P_(G, P, B2, h, i, j) * g00 + P_(G, P, B2, h, i - 1, j) * g10
                       - P_(G, P, B2, h, i, j - 1) * g01 - P_(G, P, B2, h, i - 1, j - 1) * g11) / G.dx2);
}

__device__ __forceinline__ void zone_of(const Grid &G, long t, int &h, int &i, int &j)
{
  j = G.jstart + (int)(t % G.n2);
  i = G.istart + (int)((t / G.n2) % G.n1);
  h = (int)(t / ((long)G.n2 * G.n1));
}

// per block: the three sums; per zone: |div B| into the running maximum
__global__ void __launch_bounds__(256) k_diag_int(Grid G, const double *__restrict__ P,
                                                  const double *__restrict__ geo, double *partials, int nparts,
                                                  DevScalars *sc)
{
  const double *gC = geo_at(geo, G, L_CENT);
  const double *gd = gC + 17 * G.ng;  // sqrt(-g) at CENT
  const double dV = G.dx1 * G.dx2 * G.dx3;
  double m = 0., l = 0., e = 0., dmax = 0.;
  const long nact = (long)G.n3 * G.n1 * G.n2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nact; t += (long)gridDim.x * blockDim.x) {
    int h, i, j;
    zone_of(G, t, h, i, j);
    const long c = cidx(G, h, i, j);
    double pr[8], U[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pr[k] = __ldg(P + k * G.nc + c);
    Geo q;
    load_geo(gC, G.ng, (long)i * G.sn2 + j, q);
    State s;
    int fail = 0;
    get_state(pr, q, s, &fail);
    primtoflux(G.gam, pr, s, 0, q.g, U);
    m += U[RHO] * dV;
    l += U[U3] * dV;
    e += U[UU] * dV;
    dmax = fmax(dmax, divb_zone(G, P, gd, h, i, j));
  }
  __shared__ double red[3][8];
  m = warp_sum(m);
  l = warp_sum(l);
  e = warp_sum(e);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][w] = m;
    red[1][w] = l;
    red[2][w] = e;
    if (dmax > 0.) atomicMax(&sc->divb_bits, (unsigned long long)__double_as_longlong(dmax));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0., b = 0., d = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) { a += red[0][k]; b += red[1][k]; d += red[2][k]; }
    partials[blockIdx.x] = a;
    partials[nparts + blockIdx.x] = b;
    partials[2 * nparts + blockIdx.x] = d;
  }
}

// the first zone in loop order (h, i, j) whose |div B| equals the maximum
__global__ void __launch_bounds__(256) k_divb_loc(Grid G, const double *__restrict__ P,
                                                  const double *__restrict__ geo, DevScalars *sc)
{
  const double *gd = geo_at(geo, G, L_CENT) + 17 * G.ng;
  const unsigned long long best = sc->divb_bits;
  const long nact = (long)G.n3 * G.n1 * G.n2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nact; t += (long)gridDim.x * blockDim.x) {
    int h, i, j;
    zone_of(G, t, h, i, j);
    const double v = divb_zone(G, P, gd, h, i, j);
    if (v > 0. && (unsigned long long)__double_as_longlong(v) == best) atomicMin(&sc->divb_loc, (long long)t);
  }
}

// ---------------------------------------------------------------------------
// COOL_EOS (diag.c:137-251): per zone InitCache_CoolEOS, primtoU with the run-time
// EOS and CoolVal_rho0_u_CoolEOS, which move the zone's guess; the sums of
// U[RHO], U[U3], U[UU] dV, Lambda sqrt(-g), Lambda sqrt(-g) rho and
// sqrt(-g) rho; each zone's Hd and Qnu for the per-row lnu2.

constexpr int NCOOLSUM = 6;

__device__ __forceinline__ void cool_zone(const Grid &G, const double *__restrict__ P, const double *__restrict__ gC,
                                          const EosDev &E, double *lastT, const double *__restrict__ rcent,
                                          double *hdq, int h, int i, int j, double *acc)
{
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  double pr[8], U[8];
#pragma unroll
  for (int k = 0; k < 8; k++) pr[k] = __ldg(P + k * G.nc + c);
  Geo q;
  load_geo(gC, G.ng, gi, q);
  double T = lastT[c];
  if (T == 0.0 && j > G.jstart) T = lastT[c - 1];
  EosCursor cur = eos_cursor(i, T);
  State s;
  int fail = 0;
  get_state(pr, q, s, &fail);
  primtoflux_cool(E, cur, pr, s, 0, q.g, U);
  double cv[NCOOLVAL];
  eos_coolval(E, cur, pr[RHO], pr[UU], __ldg(rcent + gi), cv);
  lastT[c] = cur.T;
  hdq[c] = cv[COOL_Hd];
  hdq[G.nc + c] = cv[COOL_Qnu];
  const double dV = G.dx1 * G.dx2 * G.dx3;
  acc[0] += U[RHO] * dV;
  acc[1] += U[U3] * dV;
  acc[2] += U[UU] * dV;
  acc[3] += cv[COOL_LAMBDA_SIM] * q.g;
  acc[4] += cv[COOL_LAMBDA_SIM] * q.g * pr[RHO];
  acc[5] += q.g * pr[RHO];
}

__device__ __forceinline__ void block_sums(double *acc, double *partials, int nparts)
{
  __shared__ double red[NCOOLSUM][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NCOOLSUM; k++) {
    const double v = warp_sum(acc[k]);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NCOOLSUM) {
    double a = 0.;
    for (int m = 0; m < (int)(blockDim.x >> 5); m++) a += red[threadIdx.x][m];
    partials[threadIdx.x * nparts + blockIdx.x] = a;
  }
}

// one thread per zone (every zone has a guess), or with ROWS one thread per
// (phi, r) row walking theta in order (zones without a guess take their
// neighbour's, as the reference's loop order gives them)
template <bool ROWS>
__global__ void __launch_bounds__(256) k_diag_cool(Grid G, const double *__restrict__ P,
                                                   const double *__restrict__ geo, EosDev E, double *lastT,
                                                   const double *__restrict__ rcent, double *hdq, double *partials,
                                                   int nparts)
{
  const double *gC = geo_at(geo, G, L_CENT);
  double acc[NCOOLSUM] = {0., 0., 0., 0., 0., 0.};
  if (ROWS) {
    const long row = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (row < (long)G.n3 * G.n1) {
      const int h = (int)(row / G.n1), i = G.istart + (int)(row % G.n1);
      for (int j = G.jstart; j <= G.jstop; j++) cool_zone(G, P, gC, E, lastT, rcent, hdq, h, i, j, acc);
    }
  } else {
    const long nact = (long)G.n3 * G.n1 * G.n2;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nact; t += (long)gridDim.x * blockDim.x) {
      int h, i, j;
      zone_of(G, t, h, i, j);
      cool_zone(G, P, gC, E, lastT, rcent, hdq, h, i, j, acc);
    }
  }
  block_sums(acc, partials, nparts);
}

// lnu2 (diag.c:225-249), one thread per (phi, r) row: the mean Hd over theta
// from the equator, the first theta from there where |r tan theta| reaches it,
// and Qnu sqrt(-g) there
__global__ void k_lnu2_rows(Grid G, const double *__restrict__ geo, const double *__restrict__ rtan,
                            const double *__restrict__ hdq, double *rows)
{
  const long row = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (row >= (long)G.n3 * G.n1) return;
  const int h = (int)(row / G.n1), i = G.istart + (int)(row % G.n1);
  const double *gd = geo_at(geo, G, L_CENT) + 17 * G.ng;
  double Hd_avg = 0.0;
  for (int j = G.jstart + G.n2 / 2; j <= G.jstop; j++) Hd_avg += hdq[cidx(G, h, i, j)];
  Hd_avg /= G.n2 / 2;
  int j;
  for (j = G.jstart + G.n2 / 2; j <= G.jstop; j++)
    if (Hd_avg <= __ldg(rtan + (long)i * G.sn2 + j)) break;
  if (j > G.jstop) j = G.jstop;
  rows[row] = hdq[G.nc + cidx(G, h, i, j)] * __ldg(gd + (long)i * G.sn2 + j);
}

}  // namespace

int cool_integrals(Ctx *x, harm_integrals *out)
{
  const Grid &G = x->G;
  const long nrows = (long)G.n3 * G.n1;
  const int rblocks = (int)((nrows + 255) / 256);
  const int np = x->nparts > rblocks ? x->nparts : rblocks;
  if (!x->cooldiag) {
    // [Hd, Qnu][nc], the block partials [6][np], the rows' lnu2 [nrows]
    CK(cudaMalloc(&x->cooldiag, ((size_t)2 * G.nc + (size_t)NCOOLSUM * np + nrows) * sizeof(double)));
  }
  double *hdq = x->cooldiag, *part = hdq + 2 * G.nc, *rows = part + (size_t)NCOOLSUM * np;
  CK(cudaMemsetAsync(part, 0, (size_t)NCOOLSUM * np * sizeof(double), x->stream));
  if (x->cool_seed)
    k_diag_cool<true><<<rblocks, 256, 0, x->stream>>>(G, x->p, x->geo, x->eos, x->lastT, x->coolgeo, hdq, part, np);
  else
    k_diag_cool<false><<<x->nparts, 256, 0, x->stream>>>(G, x->p, x->geo, x->eos, x->lastT, x->coolgeo, hdq, part,
                                                          np);
  k_lnu2_rows<<<rblocks, 256, 0, x->stream>>>(G, x->geo, x->coolgeo + G.ng, hdq, rows);
  CK(cudaGetLastError());
  std::vector<double> hp((size_t)NCOOLSUM * np + nrows);
  CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  double s[NCOOLSUM] = {0., 0., 0., 0., 0., 0.};
  for (int k = 0; k < NCOOLSUM; k++)
    for (int b = 0; b < np; b++) s[k] += hp[(size_t)k * np + b];
  double lnu2 = 0.;
  for (long r = 0; r < nrows; r++) lnu2 += hp[(size_t)NCOOLSUM * np + r];  // the reference's (h, i) order
  out->mass = s[0];
  out->ang_mom = s[1];
  out->energy = s[2];
  out->lnu = s[3];
  out->lnu_rho = s[4] / s[5];
  out->lnu_rho_2 = s[5];
  out->lnu2 = lnu2;
  return HARM_OK;
}

}  // namespace harm

using namespace harm;

extern "C" int harm_diag_integrals(harm_ctx *h, harm_integrals *out)
{
  if (!h || !out) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Grid &G = x->G;
  // clear the running maximum and location (fields of the device scalars)
  const unsigned long long zero = 0ull;
  const long long far = 0x7fffffffffffffffll;
  CK(cudaMemcpyAsync(&x->sc->divb_bits, &zero, sizeof(zero), cudaMemcpyHostToDevice, x->stream));
  CK(cudaMemcpyAsync(&x->sc->divb_loc, &far, sizeof(far), cudaMemcpyHostToDevice, x->stream));
  k_diag_int<<<x->nparts, 256, 0, x->stream>>>(G, x->p, x->geo, x->partials, x->nparts, x->sc);
  k_divb_loc<<<x->nparts, 256, 0, x->stream>>>(G, x->p, x->geo, x->sc);
  CK(cudaGetLastError());
  std::vector<double> part(3 * (size_t)x->nparts);
  unsigned long long bits = 0;
  long long loc = 0;
  CK(cudaMemcpyAsync(part.data(), x->partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaMemcpyAsync(&bits, &x->sc->divb_bits, sizeof(bits), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaMemcpyAsync(&loc, &x->sc->divb_loc, sizeof(loc), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  double s3[3] = {0., 0., 0.};
  for (int k = 0; k < 3; k++)
    for (int b = 0; b < x->nparts; b++) s3[k] += part[(size_t)k * x->nparts + b];
  out->mass = s3[0];
  out->ang_mom = s3[1];
  out->energy = s3[2];
  out->lnu = out->lnu_rho = out->lnu_rho_2 = out->lnu2 = 0.;
  if (x->cool) {
    if (!x->eos.hdfac) return fail_with(HARM_E_ARG, "COOL_EOS diagnostics need each table's HdFac");
    const int rc = cool_integrals(x, out);
    if (rc) return rc;
  }
  double dmax = 0.;
  std::memcpy(&dmax, &bits, sizeof(dmax));
  out->divbmax = dmax;
  if (bits == 0) {
    out->imax[0] = out->imax[1] = out->imax[2] = 0;
  } else {
    out->imax[0] = (int)((loc / G.n2) % G.n1);
    out->imax[1] = (int)(loc % G.n2);
    out->imax[2] = G.n3 == 1 ? 0 : (int)(loc / ((long long)G.n2 * G.n1));
  }
  return HARM_OK;
}
