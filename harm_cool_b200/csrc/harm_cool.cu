// The COOL_EOS step (decs.h:110 COOL_EOS 1): step_ch() with the run-time EOS
// pressure in the face fluxes, wave speeds, source and primtoU, and Utoprim_5d
// in place of Utoprim_2d and its isentropic fall-backs (step_ch.c:241-300,
// 437-441).  FP64, built with -fmad=false: the reference's results bit for bit.
// In mixed precision the EOS calls of the face fluxes, the wave speeds, the
// source and primtoU interpolate and solve in FP32; Utoprim_5d, whose 5D Newton
// needs its pressure to 1e-10, stays FP64, as does all other arithmetic.
//
// The temperature guess of each zone (_aLastT[SN3][SN1][SN2], cooleos.c:69,
// 836) lives in Ctx::lastT.  The reference runs its loops one zone after
// another, and every EOS call of a face or zone continues from the guess the
// previous call on the same zone index left (InitCache_CoolEOS,
// cooleos.c:770-807, points LastT at the face's or zone's entry).  Each thread
// here makes the calls of one face or zone in the reference's order, and the
// launches keep the reference's loop order (fluxes in r, theta, phi, then the
// update), so each zone's chain of guesses is the reference's.  The one
// exception is a zone's first call: with no guess yet, InitCache_CoolEOS copies
// the guess of the theta neighbour j-1, which the same loop has just set.  A
// step that may meet such zones runs its face launches with one thread per
// (phi, r) row walking theta in order (the seeding step); after one step every
// zone the loops visit holds a guess and the launches go back to one thread per
// face.
#define HARM_VARIANT cool
#define HARM_STEP_MIXED 0
// resident blocks of 128 threads per SM that the COOL_EOS kernels' register
// budgets must allow (measured on a B200: 3 for the faces, 168 registers, is
// 3 % faster than 1; the update kernels lose with more than 1)
#ifndef HARM_COOL_FLUX_MINB
#define HARM_COOL_FLUX_MINB 3
#endif
#ifndef HARM_COOL_CONS_MINB
#define HARM_COOL_CONS_MINB 1
#endif
#ifndef HARM_COOL_INV_MINB
#define HARM_COOL_INV_MINB 1
#endif
#define HARM_FLUX_MINB 1
#define HARM_CONS_MINB 1
#define HARM_INV_MINB 1
#include "harm_step.cuh"
#include "harm_cool.cuh"

namespace harm {
namespace cool {

// InitCache_CoolEOS (cooleos.c:770-807): the cursor of zone (h, i, j), tables of
// radial index i; a zone without a guess takes its theta neighbour's
__device__ __forceinline__ EosCursor init_cache(const Grid &G, double *lastT, int h, int i, int j)
{
  const long z = cidx(G, h, i, j);
  double T = lastT[z];
  if (T == 0.0 && j > G.jstart) T = lastT[z - 1];
  return eos_cursor(i, T);
}

template <int DIR, bool F32>
__device__ __forceinline__ void face_flux_cool(const EosDev &E, EosCursor &c, const double *pl, const double *pr,
                                               const Geo &q, double *F, double &ctop, int *fail)
{
  State s;
  double Fl[8], Ul[8], cmaxl, cminl, cmaxr, cminr;
  get_state(pl, q, s, fail);
  primtoflux_cool<F32>(E, c, pl, s, DIR, q.g, Fl);
  primtoflux_cool<F32>(E, c, pl, s, 0, q.g, Ul);
  vchar_cool<F32>(E, c, pl, s, q, DIR, cmaxl, cminl, fail);
  get_state(pr, q, s, fail);
  double Fr[8], Ur[8];
  primtoflux_cool<F32>(E, c, pr, s, DIR, q.g, Fr);
  primtoflux_cool<F32>(E, c, pr, s, 0, q.g, Ur);
  vchar_cool<F32>(E, c, pr, s, q, DIR, cmaxr, cminr, fail);
  double t1 = 0. > cmaxl ? 0. : cmaxl;
  double cmax = fabs(t1 > cmaxr ? t1 : cmaxr);
  double t2 = 0. > -cminl ? 0. : -cminl;
  double cmin = fabs(t2 > -cminr ? t2 : -cminr);
  ctop = cmax > cmin ? cmax : cmin;
#pragma unroll
  for (int k = 0; k < 8; k++) F[k] = 0.5 * (Fl[k] + Fr[k] - ctop * (Ur[k] - Ul[k]));
}

// one face of direction DIR (step_ch.c:407-487); returns the Courant limit of
// an active face, 1e9 otherwise
template <int DIR, bool FULL, bool F32>
__device__ __noinline__ double one_face(const Grid &G, const double *__restrict__ pb, double *__restrict__ F,
                                        const double *__restrict__ geo, const EosDev &E, double *lastT,
                                        DevScalars *sc, int h, int i, int j)
{
  const long c = cidx(G, h, i, j);
  if (DIR == 2 && (j == G.jstart || j == G.jstop + 1)) {
#pragma unroll
    for (int k = 0; k < 8; k++) F[k * G.nc + c] = 0.;
    return 1.e9;
  }
  long o1, o2, o3;
  if (DIR == 1) { o1 = c - 2 * G.sn2; o2 = c - G.sn2; o3 = c + G.sn2; }
  else if (DIR == 2) { o1 = c - 2; o2 = c - 1; o3 = c + 1; }
  else {
    o1 = cidx(G, hwrap(G, h - 2), i, j);
    o2 = cidx(G, hwrap(G, h - 1), i, j);
    o3 = cidx(G, hwrap(G, h + 1), i, j);
  }
  double pl[8], pr[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const double *P = pb + k * G.nc;
    double a = P[o1], b = P[o2], z = P[c], e = P[o3];
    pl[k] = b + 0.5 * slope_lim(G.lim, a, b, z);
    pr[k] = z - 0.5 * slope_lim(G.lim, b, z, e);
  }
  Geo q;
  load_geo(geo_at(geo, G, DIR == 1 ? L_FACE1 : DIR == 2 ? L_FACE2 : L_FACE3), G.ng, (long)i * G.sn2 + j, q);
  EosCursor cur = init_cache(G, lastT, h, i, j);
  double Fz[8], ctop;
  int fail = 0;
  face_flux_cool<DIR, F32>(E, cur, pl, pr, q, Fz, ctop, &fail);
  lastT[c] = cur.T;
#pragma unroll
  for (int k = 0; k < 8; k++) F[k * G.nc + c] = Fz[k];
  if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
  if (FULL && i >= G.istart && i <= G.istop && j >= G.jstart && j <= G.jstop) {
    const double dxd = DIR == 1 ? G.dx1 : DIR == 2 ? G.dx2 : G.dx3;
    return G.cour * dxd / ctop;
  }
  return 1.e9;
}

template <bool FULL>
__device__ __forceinline__ void reduce_dt(DevScalars *sc, int dir, double dtmin)
{
  if (!FULL) return;
  __shared__ double red[4];
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  double v = warp_min(dtmin);
  if ((t & 31) == 0) red[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    v = fmin(fmin(red[0], red[1]), fmin(red[2], red[3]));
    if (v < 1.e9) atomicMin(&sc->ndt_bits[dir - 1], (unsigned long long)__double_as_longlong(v));
  }
}

// one thread per face; face ranges as k_flux's
template <int DIR, bool FULL, bool F32>
__global__ void __launch_bounds__(128, HARM_COOL_FLUX_MINB) k_flux_cool(Grid G, const double *__restrict__ pb, double *__restrict__ F,
                                                   const double *__restrict__ geo, EosDev E, double *lastT,
                                                   DevScalars *sc)
{
  if (sc->halted) return;
  const int j = (DIR == 2 ? G.jstart : G.jstart - 1) + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (DIR == 1 ? G.istart : G.istart - 1) + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  double dtmin = 1.e9;
  if ((i <= G.istop + 1) && (j <= G.jstop + 1))
    dtmin = one_face<DIR, FULL, F32>(G, pb, F, geo, E, lastT, sc, h, i, j);
  reduce_dt<FULL>(sc, DIR, dtmin);
}

// the seeding form: one thread per (phi, r) row, theta faces in the
// reference's order (j innermost, step_ch.c:407)
template <int DIR, bool FULL, bool F32>
__global__ void __launch_bounds__(128) k_flux_cool_rows(Grid G, const double *__restrict__ pb, double *__restrict__ F,
                                                        const double *__restrict__ geo, EosDev E, double *lastT,
                                                        DevScalars *sc)
{
  if (sc->halted) return;
  const int i = (DIR == 1 ? G.istart : G.istart - 1) + blockIdx.x * blockDim.x + threadIdx.x;
  const int h = blockIdx.y;
  double dtmin = 1.e9;
  if (i <= G.istop + 1)
    for (int j = (DIR == 2 ? G.jstart : G.jstart - 1); j <= G.jstop + 1; j++)
      dtmin = fmin(dtmin, one_face<DIR, FULL, F32>(G, pb, F, geo, E, lastT, sc, h, i, j));
  reduce_dt<FULL>(sc, DIR, dtmin);
}

template <bool FULL, bool F32>
void launch_flux_cool_p(Ctx *x, const double *pb, bool rows)
{
  const Grid &G = x->G;
  const EosDev &E = x->eos;
  if (rows) {
    const dim3 b(128, 1);
    k_flux_cool_rows<1, FULL, F32><<<dim3((G.n1 + 1 + 127) / 128, G.n3), b, 0, x->stream>>>(G, pb, x->F1, x->geo, E,
                                                                                            x->lastT, x->sc);
    k_flux_cool_rows<2, FULL, F32><<<dim3((G.n1 + 2 + 127) / 128, G.n3), b, 0, x->stream>>>(G, pb, x->F2, x->geo, E,
                                                                                            x->lastT, x->sc);
    if (G.n3 > 1)
      k_flux_cool_rows<3, FULL, F32><<<dim3((G.n1 + 2 + 127) / 128, G.n3), b, 0, x->stream>>>(
          G, pb, x->F3, x->geo, E, x->lastT, x->sc);
    return;
  }
  const dim3 b(x->tbx, x->tby);
  dim3 g1((G.n2 + 2 + b.x - 1) / b.x, (G.n1 + 1 + b.y - 1) / b.y, G.n3);
  dim3 g2((G.n2 + 1 + b.x - 1) / b.x, (G.n1 + 2 + b.y - 1) / b.y, G.n3);
  dim3 g3((G.n2 + 2 + b.x - 1) / b.x, (G.n1 + 2 + b.y - 1) / b.y, G.n3);
  k_flux_cool<1, FULL, F32><<<g1, b, 0, x->stream>>>(G, pb, x->F1, x->geo, E, x->lastT, x->sc);
  k_flux_cool<2, FULL, F32><<<g2, b, 0, x->stream>>>(G, pb, x->F2, x->geo, E, x->lastT, x->sc);
  if (G.n3 > 1) k_flux_cool<3, FULL, F32><<<g3, b, 0, x->stream>>>(G, pb, x->F3, x->geo, E, x->lastT, x->sc);
}

// the face physics' EOS calls in FP32 in mixed precision, FP64 otherwise
template <bool FULL>
void launch_flux_cool(Ctx *x, const double *pb, bool rows)
{
  if (x->mode == HARM_MIXED) launch_flux_cool_p<FULL, true>(x, pb, rows);
  else launch_flux_cool_p<FULL, false>(x, pb, rows);
}

// source() with COOL_EOS (phys.c:165-207)
template <bool F32>
__device__ __noinline__ void source_cool(const EosDev &E, EosCursor &c, const double *pb, const State &s, const Geo &q,
                                         const double *__restrict__ conn, long ng, long gi, double *dU)
{
  double mhd[4][4];
  {
    const double rho = pb[RHO], u = pb[UU];
    const double p = face_pressure<F32>(E, c, rho, u);
#pragma unroll
    for (int d = 0; d < 4; d++) mhd_calc_cool(rho, u, p, d, s, mhd[d]);
  }
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

// the update's first half (step_ch.c:241-263): source(pb), primtoU(pi) and the
// flux divergence, with flux-CT and the flux boundary fixes, into Ub.  F32 (mixed
// precision): the source's and primtoU's pressures from the FP32 interpolation
// (all else FP64, the accumulation of U included)
template <bool FULL, bool THREE_D, bool F32>
__global__ void __launch_bounds__(128, HARM_COOL_CONS_MINB) k_cons_cool(Grid G, const double *__restrict__ pi, const double *__restrict__ pb,
                                                   const double *__restrict__ F1, const double *__restrict__ F2,
                                                   const double *__restrict__ F3, const double *__restrict__ geo,
                                                   const double *__restrict__ conn, EosDev E, double *lastT,
                                                   double *__restrict__ Ub, DevScalars *sc)
{
  if (sc->halted) return;
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  if (i > G.istop || j > G.jstop) return;
  const double Dt = FULL ? sc->dt : 0.5 * sc->dt;
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  int fail = 0;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  EosCursor cur = init_cache(G, lastT, h, i, j);
  double dU[8], U[8];
  {
    double pbz[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pbz[k] = pb[k * G.nc + c];
    State s;
    get_state(pbz, q, s, &fail);
    source_cool<F32>(E, cur, pbz, s, q, conn, G.ng, gi, dU);
  }
  {
    double pz[8];
#pragma unroll
    for (int k = 0; k < 8; k++) pz[k] = pi[k * G.nc + c];
    State s;
    get_state(pz, q, s, &fail);
    primtoflux_cool<F32>(E, cur, pz, s, 0, q.g, U);
  }
  lastT[c] = cur.T;
  {
    Flux FX{F1, F2, F3, G};
    double f1m[8], f1p[8], f2m[8], f2p[8], f3m[8], f3p[8];
    zone_fluxes<THREE_D>(FX, h, i, j, f1m, f1p, f2m, f2p, f3m, f3p);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      if (THREE_D)
        U[k] += Dt * (-div_rn(f1p[k] - f1m[k], G.dx1, G.idx1) - div_rn(f2p[k] - f2m[k], G.dx2, G.idx2)
                      - div_rn(f3p[k] - f3m[k], G.dx3, G.idx3) + dU[k]);
      else
        U[k] += Dt * (-div_rn(f1p[k] - f1m[k], G.dx1, G.idx1) - div_rn(f2p[k] - f2m[k], G.dx2, G.idx2) + dU[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 8; k++) Ub[k * G.nc + c] = U[k];
  if (fail) record_fail(sc, fail, h + (THREE_D ? 1 : 0), i, j);
}

// the update's second half (step_ch.c:265-268) and fixup() (fixup.c:51-60):
// Utoprim_5d from the guess pi, no isentropic fall-backs under COOL_EOS
__global__ void __launch_bounds__(128, HARM_COOL_INV_MINB) k_invert_cool(Grid G, const double *__restrict__ pi,
                                                     const double *__restrict__ Ub, double *__restrict__ pf,
                                                     signed char *__restrict__ pflag, const double *__restrict__ geo,
                                                     const double *__restrict__ floors, EosDev E, double *lastT,
                                                     DevScalars *sc)
{
  if (sc->halted) return;
  const int j = G.jstart + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = G.istart + blockIdx.y * blockDim.y + threadIdx.y;
  const int h = blockIdx.z;
  if (i > G.istop || j > G.jstop) return;
  const long c = cidx(G, h, i, j);
  const long gi = (long)i * G.sn2 + j;
  int fail = 0;
  Geo q;
  load_geo(geo_at(geo, G, L_CENT), G.ng, gi, q);
  double U[8], pz[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    U[k] = Ub[k * G.nc + c];
    pz[k] = pi[k * G.nc + c];
  }
  EosCursor cur = init_cache(G, lastT, h, i, j);
  int flag = utoprim_5d(E, cur, U, q, pz);
  lastT[c] = cur.T;
  signed char fl = (signed char)flag;
  if (fixup1zone(G.gam, __ldg(floors + gi), __ldg(floors + G.ng + gi), q, pz, &fail)) fl = -33;
#pragma unroll
  for (int k = 0; k < 8; k++) pf[k * G.nc + c] = pz[k];
  pflag[c] = fl;
  if (fail) record_fail(sc, fail, h + (G.n3 > 1 ? 1 : 0), i, j);
}

template <bool FULL, bool THREE_D, bool F32>
void launch_cons_cool_p(Ctx *x, const double *pi, const double *pb, dim3 zg, dim3 tile)
{
  k_cons_cool<FULL, THREE_D, F32><<<zg, tile, 0, x->stream>>>(x->G, pi, pb, x->F1, x->F2, x->F3, x->geo, x->conn,
                                                              x->eos, x->lastT, x->Ubuf, x->sc);
}

template <bool FULL>
void launch_cons_cool(Ctx *x, const double *pi, const double *pb, dim3 zg, dim3 tile)
{
  const bool f32 = x->mode == HARM_MIXED;
  if (x->G.n3 > 1) {
    if (f32) launch_cons_cool_p<FULL, true, true>(x, pi, pb, zg, tile);
    else launch_cons_cool_p<FULL, true, false>(x, pi, pb, zg, tile);
  } else {
    if (f32) launch_cons_cool_p<FULL, false, true>(x, pi, pb, zg, tile);
    else launch_cons_cool_p<FULL, false, false>(x, pi, pb, zg, tile);
  }
}

template <bool FULL>
void launch_half(Ctx *x, const double *pi, const double *pb, double *pf, bool rows)
{
  const Grid &G = x->G;
  launch_flux_cool<FULL>(x, pb, rows);
  const dim3 tile(x->tbx, x->tby);
  const dim3 zg((G.n2 + tile.x - 1) / tile.x, (G.n1 + tile.y - 1) / tile.y, G.n3);
  launch_cons_cool<FULL>(x, pi, pb, zg, tile);
  k_invert_cool<<<zg, tile, 0, x->stream>>>(G, pi, x->Ubuf, pf, x->pflag, x->geo, x->floors, x->eos, x->lastT,
                                            x->sc);
  if (FULL) k_diag_flux<<<1, 1024, 0, x->stream>>>(G, x->F1, x->sc);
  launch_bound(x, pf);
  launch_fixup_utoprim(x, pf);
  launch_bound(x, pf);
}

}  // namespace cool

// the COOL_EOS step; the first step after the guesses were reset seeds them
int cool_launch_step(Ctx *x)
{
  const bool rows = x->cool_seed;
  cool::launch_half<false>(x, x->p, x->p, x->ph, rows);
  cool::launch_half<true>(x, x->p, x->ph, x->p, false);
  launch_mass(x);
  x->cool_seed = false;
  CK(cudaGetLastError());
  return HARM_OK;
}

// Utoprim_5d over independent zones, each with its table index and guess
__global__ void k_utoprim_5d_batch(EosDev E, const double *U, const double *gcov, const double *gcon,
                                   const double *gdet, const int *tab, double *lastT, double *prim, int *ret, long n)
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
  EosCursor c = eos_cursor(tab[t], lastT[t]);
  ret[t] = utoprim_5d(E, c, u, q, p);
  lastT[t] = c.T;
  for (int k = 0; k < 8; k++) prim[t * 8 + k] = p[k];
}

}  // namespace harm

using namespace harm;

extern "C" int harm_set_eos(harm_ctx *h, const harm_eos *eos)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  Ctx *x = &h->x;
  if (!eos) {
    if (x->cool) invalidate_graph(x);
    x->cool = false;
    return HARM_OK;
  }
  if (eos->device != x->device) return fail_with(HARM_E_ARG, "EOS tables on another device");
  if (eos->d.ntab != x->G.sn1) return fail_with(HARM_E_ARG, "COOL_EOS needs one table per radial index (N1+4)");
  if (x->mode == HARM_MIXED && !eos->d.f32) return fail_with(HARM_E_ARG, "table values span more than float holds");
  if (!x->lastT) {
    CK(cudaMalloc(&x->lastT, (size_t)x->G.nc * sizeof(double)));
    CK(cudaMemsetAsync(x->lastT, 0, (size_t)x->G.nc * sizeof(double), x->stream));
    x->cool_seed = true;
  }
  invalidate_graph(x);
  x->eos = eos->d;
  x->cool = true;
  return HARM_OK;
}

// the guesses in the reference's layout [SN3][SN1][SN2]; the phi ghost planes
// of a 3D grid hold no guess (the loops never visit them)
extern "C" int harm_get_eos_guess(harm_ctx *h, double *lastT)
{
  if (!h || !lastT) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  if (!x->cool) return fail_with(HARM_E_ARG, "no EOS tables attached");
  const Grid &G = x->G;
  const int g3 = G.n3 > 1 ? 1 : 0;
  const size_t plane = (size_t)G.sn1 * G.sn2;
  CK(cudaStreamSynchronize(x->stream));
  for (size_t k = 0; k < plane * (G.n3 + 2 * g3); k++) lastT[k] = 0.;
  CK(cudaMemcpy(lastT + g3 * plane, x->lastT, (size_t)G.nc * sizeof(double), cudaMemcpyDeviceToHost));
  return HARM_OK;
}

extern "C" int harm_put_eos_guess(harm_ctx *h, const double *lastT)
{
  if (!h || !lastT) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  if (!x->cool) return fail_with(HARM_E_ARG, "no EOS tables attached");
  const Grid &G = x->G;
  const size_t plane = (size_t)G.sn1 * G.sn2;
  CK(cudaStreamSynchronize(x->stream));
  CK(cudaMemcpy(x->lastT, lastT + (G.n3 > 1 ? plane : 0), (size_t)G.nc * sizeof(double), cudaMemcpyHostToDevice));
  x->cool_seed = true;  // zones without a guess take their neighbour's, in order
  invalidate_graph(x);
  return HARM_OK;
}

extern "C" int harm_utoprim_5d_batch(const harm_eos *eos, const double *U, const double *gcov, const double *gcon,
                                     const double *gdet, const int *tab, double *lastT, double *prim, int *ret,
                                     long n)
{
  if (!eos || !U || !gcov || !gcon || !gdet || !tab || !lastT || !prim || !ret || n < 0)
    return fail_with(HARM_E_ARG, "null argument");
  for (long k = 0; k < n; k++)
    if (tab[k] < 0 || tab[k] >= eos->d.ntab) return fail_with(HARM_E_ARG, "table index out of range");
  if (n == 0) return HARM_OK;
  struct Buffers {
    double *U = nullptr, *a = nullptr, *b = nullptr, *g = nullptr, *T = nullptr, *p = nullptr;
    int *t = nullptr, *r = nullptr;
    ~Buffers() { cudaFree(U); cudaFree(a); cudaFree(b); cudaFree(g); cudaFree(T); cudaFree(p); cudaFree(t); cudaFree(r); }
  } B;
  CK(cudaMalloc(&B.U, n * 64));
  CK(cudaMalloc(&B.a, n * 128));
  CK(cudaMalloc(&B.b, n * 128));
  CK(cudaMalloc(&B.g, n * 8));
  CK(cudaMalloc(&B.T, n * 8));
  CK(cudaMalloc(&B.p, n * 64));
  CK(cudaMalloc(&B.t, n * sizeof(int)));
  CK(cudaMalloc(&B.r, n * sizeof(int)));
  CK(cudaMemcpy(B.U, U, n * 64, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.a, gcov, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.b, gcon, n * 128, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.g, gdet, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.T, lastT, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.p, prim, n * 64, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.t, tab, n * sizeof(int), cudaMemcpyHostToDevice));
  k_utoprim_5d_batch<<<(unsigned)((n + 127) / 128), 128>>>(eos->d, B.U, B.a, B.b, B.g, B.t, B.T, B.p, B.r, n);
  CK(cudaGetLastError());
  CK(cudaMemcpy(prim, B.p, n * 64, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ret, B.r, n * sizeof(int), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(lastT, B.T, n * 8, cudaMemcpyDeviceToHost));
  return HARM_OK;
}

namespace harm {

// reps ordinary COOL_EOS steps, one launch group at a time with an event after
// each (slots as the gamma-law variants': flux, update, bound_prim,
// fixup_utoprim, diagnostics); the seeding step, if pending, runs first, untimed
int cool_time_kernels(Ctx *x, int reps, double *ms)
{
  if (x->cool_seed) {
    int rc = cool_launch_step(x);
    if (rc) return rc;
  }
  const Grid &G = x->G;
  const int nev = 16;
  cudaEvent_t ev[nev];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  double acc[HARM_NKERNELS] = {0, 0, 0, 0, 0};
  const dim3 tile(x->tbx, x->tby);
  const dim3 zg((G.n2 + tile.x - 1) / tile.x, (G.n1 + tile.y - 1) / tile.y, G.n3);
  for (int r = 0; r < reps; r++) {
    int e = 0, slot[nev];
    CK(cudaEventRecord(ev[e++], x->stream));
    for (int half = 0; half < 2; half++) {
      const bool full = half == 1;
      double *pi = x->p, *pb = full ? x->ph : x->p, *pf = full ? x->p : x->ph;
      if (full) cool::launch_flux_cool<true>(x, pb, false);
      else cool::launch_flux_cool<false>(x, pb, false);
      slot[e] = 0; CK(cudaEventRecord(ev[e++], x->stream));
      if (full) cool::launch_cons_cool<true>(x, pi, pb, zg, tile);
      else cool::launch_cons_cool<false>(x, pi, pb, zg, tile);
      cool::k_invert_cool<<<zg, tile, 0, x->stream>>>(G, pi, x->Ubuf, pf, x->pflag, x->geo, x->floors, x->eos,
                                                      x->lastT, x->sc);
      slot[e] = 1; CK(cudaEventRecord(ev[e++], x->stream));
      if (full) {
        cool::k_diag_flux<<<1, 1024, 0, x->stream>>>(G, x->F1, x->sc);
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

}  // namespace harm
