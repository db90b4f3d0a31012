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

}  // namespace
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
