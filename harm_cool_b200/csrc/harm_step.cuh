// Kernels of one step that differ between the FP64 path and the mixed path:
// the face fluxes, the update with flux-CT, and the flux diagnostics.
// Included by harm_exact.cu (HARM_STEP_MIXED 0) and harm_mixed.cu (HARM_STEP_MIXED 1),
// each inside its own namespace.
//
// FP64 path: everything in double, built with -fmad=false, bit-compatible
// with the reference.  Mixed path: slopes, face states, the face metric,
// get_state/primtoflux/vchar and the Lax-Friedrichs flux in float; face
// fluxes stored as float; the flux divergence, flux-CT averaging, the
// connection source, U accumulation, the Noble inversion and the floors in
// double.
#pragma once
#include "harm_common.cuh"
#if HARM_STEP_MIXED
#include "harm_phys32.cuh"
#endif

// Resident blocks of 128 threads per SM that the register allocation must
// allow, per kernel.  The kernels are bound by the latency of dependent FP64
// instructions, so more resident warps beat the few spills the tighter
// register budgets cost; each variant sets values measured best on a B200.
#ifndef HARM_FLUX_MINB
#define HARM_FLUX_MINB 1
#endif
#ifndef HARM_CONS_MINB
#define HARM_CONS_MINB 1
#endif
#ifndef HARM_INV_MINB
#define HARM_INV_MINB 1
#endif
// phi planes each block sweeps, for the flux and for the zone kernels:
// consecutive planes of one (r, theta) tile reuse its geometry and (for the
// phi-direction fluxes) its stencil from L1
#ifndef HARM_HB_FLUX
#define HARM_HB_FLUX 1
#endif
#ifndef HARM_HB_ZONE
#define HARM_HB_ZONE 4
#endif

namespace harm {
namespace HARM_VARIANT {

// blocks of tile.x (theta) by tile.y (r) zones, HARM_HB_ZONE phi planes each
inline dim3 zone_grid_hb(const Grid &G, dim3 tile)
{
  return dim3((G.n2 + tile.x - 1) / tile.x, (G.n1 + tile.y - 1) / tile.y, (G.n3 + HARM_HB_ZONE - 1) / HARM_HB_ZONE);
}

#if HARM_STEP_MIXED
using flux_t = float;
#else
using flux_t = double;
#endif


// faces of direction DIR per theta row and rows per phi plane (step_ch.c:407)
template <int DIR>
__host__ __device__ __forceinline__ int faces_per_row(const Grid &G) { return DIR == 2 ? G.n2 + 1 : G.n2 + 2; }
template <int DIR>
__host__ __device__ __forceinline__ int face_rows(const Grid &G) { return DIR == 1 ? G.n1 + 1 : G.n1 + 2; }

// One thread per face of direction DIR.  Face ranges (step_ch.c:407): dir 1
// i in [istart, istop+1], j in [jstart-1, jstop+1]; dir 2 i in [istart-1,
// istop+1], j in [jstart, jstop+1] (the polar faces jstart and jstop+1 carry
// no flux, :412-416); dir 3 i in [istart-1, istop+1], j in [jstart-1, jstop+1].
// REC (the discrete adjoint's recomputation): also keep the wave speed of every
// face that takes part in the Courant minimum, in ctrec[(DIR - 1) nc + cell].
template <int DIR, bool FULL, bool REC = false>
__global__ void __launch_bounds__(128, HARM_FLUX_MINB) k_flux(Grid G, const double *__restrict__ pb, flux_t *__restrict__ F,
                                              const double *__restrict__ geo, const float *__restrict__ geo32,
                                              DevScalars *sc, double *__restrict__ ctrec)
{
  if (sc->halted) return;
  // faces of one phi plane numbered row by row (theta fastest), 128 per block,
  // so that only the plane's last warp has idle lanes
  const int nj = faces_per_row<DIR>(G);
  const int f = blockIdx.x * 128 + threadIdx.y * blockDim.x + threadIdx.x;
  const int j = (DIR == 2 ? G.jstart : G.jstart - 1) + f % nj;
  const int i = (DIR == 1 ? G.istart : G.istart - 1) + f / nj;
  const int h0 = blockIdx.z * HARM_HB_FLUX, h1 = min(G.n3, h0 + HARM_HB_FLUX);
  double dtmin = 1.e9;
  const bool in = i <= G.istop + 1;
  if (in) for (int h = h0; h < h1; h++) {
    const long c = cidx(G, h, i, j);
    if (DIR == 2 && (j == G.jstart || j == G.jstop + 1)) {
#pragma unroll
      for (int k = 0; k < 8; k++) F[k * G.nc + c] = 0.;
    } else {
      long o1, o2, o3;  // zone-2d, zone-d, zone+d
      if (DIR == 1) { o1 = c - 2 * G.sn2; o2 = c - G.sn2; o3 = c + G.sn2; }
      else if (DIR == 2) { o1 = c - 2; o2 = c - 1; o3 = c + 1; }
      else {
        o1 = cidx(G, hwrap(G, h - 2), i, j);
        o2 = cidx(G, hwrap(G, h - 1), i, j);
        o3 = cidx(G, hwrap(G, h + 1), i, j);
      }
#if HARM_STEP_MIXED
      float pl[8], pr[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const double *P = pb + k * G.nc;
        float a = (float)__ldg(P + o1), b = (float)__ldg(P + o2), z = (float)__ldg(P + c), e = (float)__ldg(P + o3);
        pl[k] = b + 0.5f * slope_lim_f(G.lim, a, b, z);
        pr[k] = z - 0.5f * slope_lim_f(G.lim, b, z, e);
      }
      GeoF q;
      load_geo_f(geo32 + (long)(DIR - 1) * GEO_N * G.ng, G.ng, (long)i * G.sn2 + j, q);
      float Fz[8], ctopf;
      int fail = 0;
      face_flux_f<DIR>((float)G.gam, pl, pr, q, Fz, ctopf, &fail);
      const double ctop = (double)ctopf;
#else
      double pl[8], pr[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const double *P = pb + k * G.nc;
        double a = __ldg(P + o1), b = __ldg(P + o2), z = __ldg(P + c), e = __ldg(P + o3);
        pl[k] = b + 0.5 * slope_lim(G.lim, a, b, z);
        pr[k] = z - 0.5 * slope_lim(G.lim, b, z, e);
      }
      Geo q;
      load_geo(geo_at(geo, G, DIR == 1 ? L_FACE1 : DIR == 2 ? L_FACE2 : L_FACE3), G.ng, (long)i * G.sn2 + j, q);
      double Fz[8], ctop;
      int fail = 0;
      face_flux<DIR>(G.gam, pl, pr, q, Fz, ctop, &fail);
#endif
#pragma unroll
      for (int k = 0; k < 8; k++) F[k * G.nc + c] = Fz[k];
      if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
      if (FULL && i >= G.istart && i <= G.istop && j >= G.jstart && j <= G.jstop) {
        const double dxd = DIR == 1 ? G.dx1 : DIR == 2 ? G.dx2 : G.dx3;
        dtmin = fmin(dtmin, G.cour * dxd / ctop);
        if (REC) ctrec[(DIR - 1) * G.nc + c] = ctop;
      }
    }
  }
  if (FULL) {
    __shared__ double red[4];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    double v = warp_min(dtmin);
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    if (t == 0) {
      v = fmin(fmin(red[0], red[1]), fmin(red[2], red[3]));
      if (v < 1.e9) atomicMin(&sc->ndt_bits[DIR - 1], (unsigned long long)__double_as_longlong(v));
    }
  }
}


// ctrec (the adjoint's recomputation of a corrector): keep the direction-1
// and -2 faces' wave speeds there
template <bool FULL>
void launch_flux(const Grid &G, dim3 b, cudaStream_t st, const double *pb, flux_t *F1, flux_t *F2, flux_t *F3,
                 const double *geo, const float *geo32, DevScalars *sc, double *ctrec = nullptr)
{
  const int gz = (G.n3 + HARM_HB_FLUX - 1) / HARM_HB_FLUX;
  // 128 faces per block whatever the tile's shape
  dim3 g1((faces_per_row<1>(G) * face_rows<1>(G) + 127) / 128, 1, gz);
  dim3 g2((faces_per_row<2>(G) * face_rows<2>(G) + 127) / 128, 1, gz);
  dim3 g3((faces_per_row<3>(G) * face_rows<3>(G) + 127) / 128, 1, gz);
#if !HARM_STEP_MIXED
  if (FULL && ctrec) {
    // ctrec holds directions 1 and 2 (the adjoint that reads it is 2D); a 3D
    // step still gets its phi fluxes, without a record
    k_flux<1, true, true><<<g1, b, 0, st>>>(G, pb, F1, geo, geo32, sc, ctrec);
    k_flux<2, true, true><<<g2, b, 0, st>>>(G, pb, F2, geo, geo32, sc, ctrec);
    if (G.n3 > 1) k_flux<3, true><<<g3, b, 0, st>>>(G, pb, F3, geo, geo32, sc, nullptr);
    return;
  }
#endif
  k_flux<1, FULL><<<g1, b, 0, st>>>(G, pb, F1, geo, geo32, sc, nullptr);
  k_flux<2, FULL><<<g2, b, 0, st>>>(G, pb, F2, geo, geo32, sc, nullptr);
  if (G.n3 > 1) k_flux<3, FULL><<<g3, b, 0, st>>>(G, pb, F3, geo, geo32, sc, nullptr);
}

// ---------------------------------------------------------------------------
// update (step_ch.c:237-306) fused with flux_ct (step_ch.c:514-629, 726-798),
// the flux boundary fixes (coord.c:264-324) and fixup() (fixup.c:51-60)

struct Flux {
  const flux_t *F1, *F2, *F3;
  Grid G;
  __device__ double raw(int d, int k, int h, int i, int j) const
  {
    const flux_t *F = d == 1 ? F1 : d == 2 ? F2 : F3;
    return (double)__ldg(F + k * G.nc + cidx(G, h, i, j));
  }
  // B-component of a raw face flux after fix_flux's polar reflection
  // (coord.c:284-301): F1,F3[B2] at jstart-1 / jstop+1 mirror jstart / jstop
  __device__ double rawB2(int d, int h, int i, int j) const
  {
    if (j == G.jstart - 1) return -raw(d, B2, h, i, G.jstart);
    if (j == G.jstop + 1) return -raw(d, B2, h, i, G.jstop);
    return raw(d, B2, h, i, j);
  }
  // 2D EMF (step_ch.c:546-547)
  __device__ double emf2(int i, int j) const
  {
    return 0.25 * (rawB2(1, 0, i, j) + rawB2(1, 0, i, j - 1) - raw(2, B1, 0, i, j) - raw(2, B1, 0, i - 1, j));
  }
  // 3D EMFs (step_ch.c:754-764); h-1 wraps (phi periodic)
  __device__ double e1(int h, int i, int j) const
  {
    int hm = hwrap(G, h - 1);
    return 0.25 * ((raw(2, B3, h, i, j) + raw(2, B3, hm, i, j)) - (rawB2(3, h, i, j) + rawB2(3, h, i, j - 1)));
  }
  __device__ double e2(int h, int i, int j) const
  {
    int hm = hwrap(G, h - 1);
    return 0.25 * ((raw(3, B1, h, i, j) + raw(3, B1, h, i - 1, j)) - (raw(1, B3, h, i, j) + raw(1, B3, hm, i, j)));
  }
  __device__ double e3(int h, int i, int j) const
  {
    return 0.25 * ((rawB2(1, h, i, j) + rawB2(1, h, i, j - 1)) - (raw(2, B1, h, i, j) + raw(2, B1, h, i - 1, j)));
  }
};

template <bool THREE_D>
__device__ void zone_fluxes(const Flux &FX, int h, int i, int j, double *f1m, double *f1p, double *f2m,
                            double *f2p, double *f3m, double *f3p)
{
  const Grid &G = FX.G;
  const int hp = THREE_D ? hwrap(G, h + 1) : 0;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    f1m[k] = FX.raw(1, k, h, i, j);
    f1p[k] = FX.raw(1, k, h, i + 1, j);
    f2m[k] = FX.raw(2, k, h, i, j);
    f2p[k] = FX.raw(2, k, h, i, j + 1);
    if (THREE_D) {
      f3m[k] = FX.raw(3, k, h, i, j);
      f3p[k] = FX.raw(3, k, hp, i, j);
    }
  }
  // no inflow of mass through the radial boundaries (coord.c:307-321)
  if (i == G.istart && f1m[RHO] > 0) f1m[RHO] = 0;
  if (i + 1 == G.istop + 1 && f1p[RHO] < 0) f1p[RHO] = 0;
  if (!THREE_D) {
    double eA = FX.emf2(i, j), eB = FX.emf2(i, j + 1), eC = FX.emf2(i + 1, j), eD = FX.emf2(i + 1, j + 1);
    f1m[B1] = 0.;
    f1m[B2] = 0.5 * (eA + eB);
    f1m[B3] = FX.raw(1, B3, 0, i, j);
    f1p[B1] = 0.;
    f1p[B2] = 0.5 * (eC + eD);
    f1p[B3] = FX.raw(1, B3, 0, i + 1, j);
    f2m[B1] = -0.5 * (eA + eC);
    f2m[B2] = 0.;
    f2m[B3] = FX.raw(2, B3, 0, i, j);
    f2p[B1] = -0.5 * (eB + eD);
    f2p[B2] = 0.;
    f2p[B3] = FX.raw(2, B3, 0, i, j + 1);
  } else {
    double e3a = FX.e3(h, i, j), e3b = FX.e3(h, i, j + 1), e3c = FX.e3(h, i + 1, j), e3d = FX.e3(h, i + 1, j + 1);
    double e2a = FX.e2(h, i, j), e2b = FX.e2(hp, i, j), e2c = FX.e2(h, i + 1, j), e2d = FX.e2(hp, i + 1, j);
    double e1a = FX.e1(h, i, j), e1b = FX.e1(hp, i, j), e1c = FX.e1(h, i, j + 1), e1d = FX.e1(hp, i, j + 1);
    f1m[B1] = 0.;
    f1m[B2] = 0.5 * (e3a + e3b);
    f1m[B3] = -0.5 * (e2a + e2b);
    f1p[B1] = 0.;
    f1p[B2] = 0.5 * (e3c + e3d);
    f1p[B3] = -0.5 * (e2c + e2d);
    f2m[B1] = -0.5 * (e3a + e3c);
    f2m[B2] = 0.;
    f2m[B3] = 0.5 * (e1a + e1b);
    f2p[B1] = -0.5 * (e3b + e3d);
    f2p[B2] = 0.;
    f2p[B3] = 0.5 * (e1c + e1d);
    f3m[B1] = 0.5 * (e2a + e2c);
    f3m[B2] = -0.5 * (e1a + e1c);
    f3m[B3] = 0.;
    f3p[B1] = 0.5 * (e2b + e2d);
    f3p[B2] = -0.5 * (e1b + e1d);
    f3p[B3] = 0.;
  }
}

// flux_ct's corner EMFs (step_ch.c:514-629 in 2D, 726-798 in 3D), each
// formed once from the raw face fluxes, for the update of the four zones that
// share the corner: emf[2 nc + cell] e3 (2D: the one EMF), and in 3D emf[cell]
// e1, emf[nc + cell] e2.  Corners i in [istart, istop+1], j in [jstart,
// jstop+1], every phi plane.
template <bool THREE_D>
__global__ void __launch_bounds__(128) k_emf(Grid G, const flux_t *__restrict__ F1, const flux_t *__restrict__ F2,
                                             const flux_t *__restrict__ F3, double *__restrict__ emf, DevScalars *sc)
{
  if (sc->halted) return;
  const int nj = G.n2 + 1;
  const int f = blockIdx.x * 128 + threadIdx.x;
  const int j = G.jstart + f % nj, i = G.istart + f / nj;
  if (i > G.istop + 1) return;
  const int h = blockIdx.z;
  const Flux FX{F1, F2, F3, G};
  const long c = cidx(G, h, i, j);
  if (THREE_D) {
    emf[c] = FX.e1(h, i, j);
    emf[G.nc + c] = FX.e2(h, i, j);
    emf[2 * G.nc + c] = FX.e3(h, i, j);
  } else {
    emf[2 * G.nc + c] = FX.emf2(i, j);
  }
}

// The flux divergence of the update (step_ch.c:247-263) one conserved
// component at a time, U[k] += Dt (-dF1/dx1 - dF2/dx2 [- dF3/dx3] + dU[k]), with
// the same face fluxes zone_fluxes forms (the no-inflow mass-flux fix, and the
// field components rebuilt from the corner EMFs of flux_ct, read from k_emf's
// planes), so only one component's six face values are live at a time.
template <bool THREE_D>
__device__ __forceinline__ void flux_update(const Flux &FX, const double *__restrict__ emf, int h, int i, int j,
                                            double Dt, const double *dU, double *U)
{
  const Grid &G = FX.G;
  const int hp = THREE_D ? hwrap(G, h + 1) : 0;
  auto upd = [&](int k, double f1m, double f1p, double f2m, double f2p, double f3m, double f3p) {
#if HARM_STEP_MIXED
    const double idx1 = 1. / G.dx1, idx2 = 1. / G.dx2, idx3 = 1. / G.dx3;
    if (THREE_D)
      U[k] += Dt * (-(f1p - f1m) * idx1 - (f2p - f2m) * idx2 - (f3p - f3m) * idx3 + dU[k]);
    else
      U[k] += Dt * (-(f1p - f1m) * idx1 - (f2p - f2m) * idx2 + dU[k]);
#else
    if (THREE_D)
      U[k] += Dt * (-div_rn(f1p - f1m, G.dx1, G.idx1) - div_rn(f2p - f2m, G.dx2, G.idx2)
                    - div_rn(f3p - f3m, G.dx3, G.idx3) + dU[k]);
    else
      U[k] += Dt * (-div_rn(f1p - f1m, G.dx1, G.idx1) - div_rn(f2p - f2m, G.dx2, G.idx2) + dU[k]);
#endif
  };
#pragma unroll
  for (int k = 0; k < 5; k++) {
    double f1m = FX.raw(1, k, h, i, j), f1p = FX.raw(1, k, h, i + 1, j);
    if (k == RHO) {
      // no inflow of mass through the radial boundaries (coord.c:307-321)
      if (i == G.istart && f1m > 0) f1m = 0;
      if (i + 1 == G.istop + 1 && f1p < 0) f1p = 0;
    }
    const double f2m = FX.raw(2, k, h, i, j), f2p = FX.raw(2, k, h, i, j + 1);
    const double f3m = THREE_D ? FX.raw(3, k, h, i, j) : 0., f3p = THREE_D ? FX.raw(3, k, hp, i, j) : 0.;
    upd(k, f1m, f1p, f2m, f2p, f3m, f3p);
  }
  const double *E1 = emf, *E2 = emf + G.nc, *E3 = emf + 2 * G.nc;
  if (!THREE_D) {
    const double eA = __ldg(E3 + cidx(G, 0, i, j)), eB = __ldg(E3 + cidx(G, 0, i, j + 1));
    const double eC = __ldg(E3 + cidx(G, 0, i + 1, j)), eD = __ldg(E3 + cidx(G, 0, i + 1, j + 1));
    upd(B1, 0., 0., -0.5 * (eA + eC), -0.5 * (eB + eD), 0., 0.);
    upd(B2, 0.5 * (eA + eB), 0.5 * (eC + eD), 0., 0., 0., 0.);
    upd(B3, FX.raw(1, B3, 0, i, j), FX.raw(1, B3, 0, i + 1, j), FX.raw(2, B3, 0, i, j), FX.raw(2, B3, 0, i, j + 1),
        0., 0.);
  } else {
    const double e3a = __ldg(E3 + cidx(G, h, i, j)), e3b = __ldg(E3 + cidx(G, h, i, j + 1));
    const double e3c = __ldg(E3 + cidx(G, h, i + 1, j)), e3d = __ldg(E3 + cidx(G, h, i + 1, j + 1));
    const double e2a = __ldg(E2 + cidx(G, h, i, j)), e2b = __ldg(E2 + cidx(G, hp, i, j));
    const double e2c = __ldg(E2 + cidx(G, h, i + 1, j)), e2d = __ldg(E2 + cidx(G, hp, i + 1, j));
    upd(B1, 0., 0., -0.5 * (e3a + e3c), -0.5 * (e3b + e3d), 0.5 * (e2a + e2c), 0.5 * (e2b + e2d));
    const double e1a = __ldg(E1 + cidx(G, h, i, j)), e1b = __ldg(E1 + cidx(G, hp, i, j));
    const double e1c = __ldg(E1 + cidx(G, h, i, j + 1)), e1d = __ldg(E1 + cidx(G, hp, i, j + 1));
    upd(B2, 0.5 * (e3a + e3b), 0.5 * (e3c + e3d), 0., 0., -0.5 * (e1a + e1c), -0.5 * (e1b + e1d));
    upd(B3, -0.5 * (e2a + e2b), -0.5 * (e2c + e2d), 0.5 * (e1a + e1b), 0.5 * (e1c + e1d), 0., 0.);
  }
}

__device__ void source(double gam, const double *pb, const Geo &q, const double *__restrict__ conn, long ng, long gi,
                       double *dU, int *fail)
{
  State s;
  get_state(pb, q, s, fail);
  source_of_state(gam, pb, s, q, conn, ng, gi, dU);
}

// The zone update (step_ch.c:237-306) in two launches, so that each holds
// fewer registers and more warps stay resident to cover FP64 latency:
// k_cons forms U -- flux_ct (step_ch.c:514-629, 726-798), the flux boundary
// fixes (coord.c:264-324), source() (phys.c:165-207), primtoU of pi and the
// flux divergence (step_ch.c:247-263) -- into Ub; k_invert runs Utoprim_2d
// with the isentropic fall-backs (step_ch.c:265-300) and fixup()
// (fixup.c:142-383).  The order of every floating-point operation is the
// reference's.
template <bool FULL, bool THREE_D>
__global__ void __launch_bounds__(128, HARM_CONS_MINB) k_cons(Grid G, const double *__restrict__ pi,
                                                              const double *__restrict__ pb,
                                                              const flux_t *__restrict__ F1,
                                                              const flux_t *__restrict__ F2,
                                                              const flux_t *__restrict__ F3,
                                                              const double *__restrict__ geo,
                                                              const double *__restrict__ conn,
                                                              const float *__restrict__ geo32,
                                                              const float *__restrict__ conn32,
                                                              const double *__restrict__ emf,
                                                              double *__restrict__ Ub, DevScalars *sc)
{
  if (sc->halted) return;
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > G.istop || j > G.jstop) return;
  const double Dt = FULL ? sc->dt : 0.5 * sc->dt;
  const int h0 = blockIdx.z * HARM_HB_ZONE, h1 = min(G.n3, h0 + HARM_HB_ZONE);
  for (int h = h0; h < h1; h++) {
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  int fail = 0;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double dU[8], U[8];
#if HARM_STEP_MIXED
  if (i >= G.isrc32) {
    // away from the horizon: the connection source in float (harm_phys32.cuh)
    float pf32[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pf32[k] = (float)__ldg(pb + k * G.nc + c);
    GeoF qf;
    load_geo_f(geo32 + (long)L_CENT * GEO_N * G.ng, G.ng, gi, qf);
    source_f((float)G.gam, pf32, qf, conn32, G.ng, gi, dU, &fail);
    double pz[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pz[k] = __ldg(pi + k * G.nc + c);
    State s;
    get_state(pz, q, s, &fail);
    primtoflux(G.gam, pz, s, 0, q.g, U);
  } else
#endif
  if (!FULL) {
    // the predictor advances from pi == pb (advance(p, p, ...), step_ch.c:101):
    // one state serves both source() and primtoU()
    double pz[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pz[k] = __ldg(pb + k * G.nc + c);
    State s;
    get_state(pz, q, s, &fail);
    source_of_state(G.gam, pz, s, q, conn, G.ng, gi, dU);
    primtoflux(G.gam, pz, s, 0, q.g, U);
  } else {
    {
      double pbz[8];
#pragma unroll
      for (int k = 0; k < 8; k++) pbz[k] = __ldg(pb + k * G.nc + c);
      source(G.gam, pbz, q, conn, G.ng, gi, dU, &fail);
    }
    double pz[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pz[k] = __ldg(pi + k * G.nc + c);
    State s;
    get_state(pz, q, s, &fail);
    primtoflux(G.gam, pz, s, 0, q.g, U);
  }
  flux_update<THREE_D>(Flux{F1, F2, F3, G}, emf, h, i, j, Dt, dU, U);
#pragma unroll
  for (int k = 0; k < 8; k++) Ub[k * G.nc + c] = U[k];
  if (fail) record_fail(sc, fail, h + (THREE_D ? 1 : 0), i, j);
  }
}

// the isentropic fall-backs (step_ch.c:277-300), kept out of line: most
// zones never take them, and inlined they crowd the kernel's hot code out of
// the instruction cache
static __device__ __noinline__ int inversion_fallbacks(double gam, double kap, const double *U, const Geo &q,
                                                       double *pz)
{
  int flag = utoprim<1>(gam, kap, U, q, pz);
  if (flag) flag = utoprim<2>(gam, kap, U, q, pz);
  return flag;
}

// REC: also keep the inversion's output before fixup() and which inversion
// gave it (zrec, wrec), for the discrete adjoint's recomputation
template <bool REC>
__global__ void __launch_bounds__(128, HARM_INV_MINB) k_invert(Grid G, const double *__restrict__ pi,
                                                               const double *__restrict__ Ub,
                                                               double *__restrict__ pf,
                                                               signed char *__restrict__ pflag,
                                                               const double *__restrict__ geo,
                                                               const double *__restrict__ floors,
                                                               const double *__restrict__ katm, DevScalars *sc,
                                                               double *__restrict__ zrec,
                                                               signed char *__restrict__ wrec)
{
  if (sc->halted) return;
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > G.istop || j > G.jstop) return;
  const int h0 = blockIdx.z * HARM_HB_ZONE, h1 = min(G.n3, h0 + HARM_HB_ZONE);
  for (int h = h0; h < h1; h++) {
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  int fail = 0;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double U[8], pz[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    U[k] = __ldg(Ub + k * G.nc + c);
    pz[k] = __ldg(pi + k * G.nc + c);
  }
  int flag = utoprim<0, (bool)HARM_STEP_MIXED>(G.gam, 0., U, q, pz);
  if (REC) {
    int which = 0;
    if (flag) {
      which = 1;
      flag = utoprim<1>(G.gam, __ldg(katm + i), U, q, pz);
      if (flag) {
        which = 2;
        flag = utoprim<2>(G.gam, __ldg(katm + i), U, q, pz);
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) zrec[k * G.nc + c] = pz[k];
    wrec[c] = (signed char)(flag ? -1 : which);
  } else if (flag) {
    flag = inversion_fallbacks(G.gam, __ldg(katm + i), U, q, pz);
  }
  signed char fl = (signed char)flag;
  if (fixup1zone(G.gam, __ldg(floors + gi), __ldg(floors + G.ng + gi), q, pz, &fail)) fl = -33;
#pragma unroll
  for (int k = 0; k < 8; k++) pf[k * G.nc + c] = pz[k];
  pflag[c] = fl;
  if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
  }
}

// diag_flux() (diag.c:437-465): sums over the inner radial face, after the
// mass-flux fix; one block, fixed summation order
__global__ void k_diag_flux(Grid G, const flux_t *__restrict__ F1, DevScalars *sc)
{
  if (sc->halted) return;
  __shared__ double red[3][32];
  double m = 0., e = 0., l = 0.;
  const long n = (long)G.n3 * G.n2;
  for (long t = threadIdx.x; t < n; t += blockDim.x) {
    int h = (int)(t / G.n2), j = G.jstart + (int)(t % G.n2);
    long c = cidx(G, h, G.istart, j);
    double fr = (double)F1[RHO * G.nc + c];
    if (fr > 0) fr = 0;
    m += fr * G.dx2 * G.dx3;
    e += ((double)F1[UU * G.nc + c] - fr) * G.dx2 * G.dx3;
    l += (double)F1[U3 * G.nc + c] * G.dx2 * G.dx3;
  }
  m = warp_sum(m);
  e = warp_sum(e);
  l = warp_sum(l);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = m;
    red[1][threadIdx.x >> 5] = e;
    red[2][threadIdx.x >> 5] = l;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int nw = blockDim.x >> 5;
    double a = threadIdx.x < nw ? red[0][threadIdx.x] : 0.;
    double b = threadIdx.x < nw ? red[1][threadIdx.x] : 0.;
    double d = threadIdx.x < nw ? red[2][threadIdx.x] : 0.;
    a = warp_sum(a);
    b = warp_sum(b);
    d = warp_sum(d);
    if (threadIdx.x == 0) {
      sc->mdot = a;
      sc->edot = -b;
      sc->ldot = d;
    }
  }
}


// ---------------------------------------------------------------------------
// one step of this variant

struct Bufs {
  flux_t *F1, *F2, *F3;
};

inline Bufs bufs(Ctx *x)
{
#if HARM_STEP_MIXED
  return Bufs{x->F1f, x->F2f, x->F3f};
#else
  return Bufs{x->F1, x->F2, x->F3};
#endif
}

template <bool FULL>
void launch_update(Ctx *x, const double *pi, const double *pb, double *pf, double *zrec = nullptr,
                   signed char *wrec = nullptr)
{
  const Grid &G = x->G;
  Bufs B = bufs(x);
  const dim3 tile(x->tbx, x->tby);
  const dim3 zg = zone_grid_hb(G, tile);
  const dim3 eg(((G.n2 + 1) * (G.n1 + 1) + 127) / 128, 1, G.n3);
  if (G.n3 > 1) {
    k_emf<true><<<eg, 128, 0, x->stream>>>(G, B.F1, B.F2, B.F3, x->emf, x->sc);
    k_cons<FULL, true><<<zg, tile, 0, x->stream>>>(G, pi, pb, B.F1, B.F2, B.F3, x->geo, x->conn, x->geo32,
                                                   x->conn32, x->emf, x->Ubuf, x->sc);
  } else {
    k_emf<false><<<eg, 128, 0, x->stream>>>(G, B.F1, B.F2, B.F3, x->emf, x->sc);
    k_cons<FULL, false><<<zg, tile, 0, x->stream>>>(G, pi, pb, B.F1, B.F2, B.F3, x->geo, x->conn, x->geo32,
                                                    x->conn32, x->emf, x->Ubuf, x->sc);
  }
#if !HARM_STEP_MIXED
  if (zrec)
    k_invert<true><<<zg, tile, 0, x->stream>>>(G, pi, x->Ubuf, pf, x->pflag, x->geo, x->floors, x->katm, x->sc,
                                               zrec, wrec);
  else
#endif
    k_invert<false><<<zg, tile, 0, x->stream>>>(G, pi, x->Ubuf, pf, x->pflag, x->geo, x->floors, x->katm, x->sc,
                                                nullptr, nullptr);
}

// advance() + fixup + bound_prim + fixup_utoprim + bound_prim (step_ch.c:101-117)
template <bool FULL>
void launch_half(Ctx *x, const double *pi, const double *pb, double *pf)
{
  Bufs B = bufs(x);
  launch_flux<FULL>(x->G, dim3(x->tbx, x->tby), x->stream, pb, B.F1, B.F2, B.F3, x->geo, x->geo32, x->sc);
  launch_update<FULL>(x, pi, pb, pf);
  if (FULL) k_diag_flux<<<1, 1024, 0, x->stream>>>(x->G, B.F1, x->sc);
  launch_bound(x, pf);
  launch_fixup_utoprim(x, pf);
  launch_bound(x, pf);
}

int launch_step(Ctx *x)
{
  launch_half<false>(x, x->p, x->p, x->ph);
  launch_half<true>(x, x->p, x->ph, x->p);
  launch_mass(x);
  CK(cudaGetLastError());
  return HARM_OK;
}

#if !HARM_STEP_MIXED
// launch_half and launch_step as above, also keeping what the discrete adjoint
// reads back (StepRec); the same kernels in the same order, so the recomputed
// step is the step
template <bool FULL>
static void launch_half_rec(Ctx *x, const double *pi, const double *pb, double *pf, const StepRec &r)
{
  const int s = FULL ? 1 : 0;
  const size_t nc = (size_t)x->G.nc;
  Bufs B = bufs(x);
  launch_flux<FULL>(x->G, dim3(x->tbx, x->tby), x->stream, pb, B.F1, B.F2, B.F3, x->geo, x->geo32, x->sc,
                    FULL ? r.ctop : nullptr);
  cudaMemcpyAsync(r.F1rho[s], B.F1 + RHO * nc, nc * sizeof(double), cudaMemcpyDeviceToDevice, x->stream);
  launch_update<FULL>(x, pi, pb, pf, r.Z[s], r.wz[s]);
  cudaMemcpyAsync(r.Ub[s], x->Ubuf, 8 * nc * sizeof(double), cudaMemcpyDeviceToDevice, x->stream);
  if (FULL) k_diag_flux<<<1, 1024, 0, x->stream>>>(x->G, B.F1, x->sc);
  launch_bound(x, pf);
  cudaMemcpyAsync(r.X1[s], pf, 8 * nc * sizeof(double), cudaMemcpyDeviceToDevice, x->stream);
  cudaMemcpyAsync(r.fl1[s], x->pflag, nc, cudaMemcpyDeviceToDevice, x->stream);
  launch_fixup_utoprim(x, pf, r.nfail[s]);
  launch_bound(x, pf);
}

int launch_step_rec(Ctx *x, const StepRec &r)
{
  launch_half_rec<false>(x, x->p, x->p, x->ph, r);
  cudaMemcpyAsync(r.ph, x->ph, 8 * (size_t)x->G.nc * sizeof(double), cudaMemcpyDeviceToDevice, x->stream);
  launch_half_rec<true>(x, x->p, x->ph, x->p, r);
  // the corrector's Courant minima, before k_finalize resets them
  cudaMemcpyAsync(r.sc[0], x->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, x->stream);
  launch_mass(x);
  cudaMemcpyAsync(r.sc[1], x->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, x->stream);
  CK(cudaGetLastError());
  return HARM_OK;
}
#endif

// reps ordinary steps, one kernel at a time with an event after each, so
// every kernel is timed inside the sequence it runs in; slots: flux, update,
// bound_prim, fixup_utoprim, diagnostics
int time_kernels(Ctx *x, int reps, double *ms)
{
  const Grid &G = x->G;
  Bufs B = bufs(x);
  const int nev = 16;
  cudaEvent_t ev[nev];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  double acc[HARM_NKERNELS] = {0, 0, 0, 0, 0};
  for (int r = 0; r < reps; r++) {
    int e = 0, slot[nev];
    CK(cudaEventRecord(ev[e++], x->stream));
    for (int half = 0; half < 2; half++) {
      const bool full = half == 1;
      double *pi = x->p, *pb = full ? x->ph : x->p, *pf = full ? x->p : x->ph;
      const dim3 tile(x->tbx, x->tby);
      if (full) launch_flux<true>(G, tile, x->stream, pb, B.F1, B.F2, B.F3, x->geo, x->geo32, x->sc);
      else launch_flux<false>(G, tile, x->stream, pb, B.F1, B.F2, B.F3, x->geo, x->geo32, x->sc);
      slot[e] = 0; CK(cudaEventRecord(ev[e++], x->stream));
      if (full) launch_update<true>(x, pi, pb, pf);
      else launch_update<false>(x, pi, pb, pf);
      slot[e] = 1; CK(cudaEventRecord(ev[e++], x->stream));
      if (full) {
        k_diag_flux<<<1, 1024, 0, x->stream>>>(G, B.F1, x->sc);
        slot[e] = 4; CK(cudaEventRecord(ev[e++], x->stream));
      }
      launch_bound(x, pf);
      slot[e] = 2; CK(cudaEventRecord(ev[e++], x->stream));
      launch_fixup_utoprim(x, pf);
      slot[e] = 3; CK(cudaEventRecord(ev[e++], x->stream));
      launch_bound(x, pf);
      slot[e] = 2; CK(cudaEventRecord(ev[e++], x->stream));
    }
    launch_mass(x);
    slot[e] = 4; CK(cudaEventRecord(ev[e++], x->stream));
    CK(cudaEventSynchronize(ev[e - 1]));
    for (int k = 1; k < e; k++) {
      float f;
      CK(cudaEventElapsedTime(&f, ev[k - 1], ev[k]));
      acc[slot[k]] += f;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  const double per_step[HARM_NKERNELS] = {2, 2, 4, 2, 1};
  for (int k = 0; k < HARM_NKERNELS; k++) ms[k] = acc[k] / (reps * per_step[k]);
  return sync_status(x);
}

}  // namespace HARM_VARIANT
}  // namespace harm
