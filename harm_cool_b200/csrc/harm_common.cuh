// Types and helpers shared by the CUDA translation units of libharm_b200.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "harm_b200.h"
#include "harm_eos.cuh"
#include "harm_phys.cuh"
#include "host_setup.h"

namespace harm {

// ---------------------------------------------------------------------------
// device-side run state

struct DevScalars {
  double t, dt;
  unsigned long long ndt_bits[3];  // per-direction Courant minima (bits of positive doubles)
  double mdot, edot, ldot, mdot_in, mdot_out, mass_curr, mass_in, mass_out, ndt;
  double bsq_max;                  // torus set-up only
  unsigned long long bsq_bits;
  int fail_code, fail_h, fail_i, fail_j;
  int err;                         // HARM_E_DT when dt < 1e-9
  int halted;                      // set after a failure: later steps do nothing
  int nfail, fail_overflow;        // failed zones met by the current fixup_utoprim
  int wave_done;                   // blocks of k_fu_wave finished (reset by the last)
  unsigned long long divb_bits;    // diagnostics: bits of max |div B| (a positive double)
  long long divb_loc;              // and its first zone in loop order
};

// Problem description passed by value to every kernel.
struct Grid {
  int n1, n2, n3, sn1, sn2;
  int istart, istop, jstart, jstop;
  long ng;   // sn1*sn2, points per geometry plane
  long nc;   // n3*sn1*sn2, cells per state plane
  int lim;
  double gam, cour, defcon, tf;
  double dx1, dx2, dx3;
  double idx1, idx2, idx3;  // 1/dx rounded to nearest: the divisors of div_rn in the flux divergence
  int isrc32;  // mixed path: first radial index whose connection source runs in float (r >= 2 r_H)
};

// tracer particles (tracers.c): the grid as the reference's coord() and
// bl_coord() see it, in the reference's own indices (h from 1 in 3D)
struct TrParams {
  double sx1, sx2, sx3, dx1, dx2, dx3;
  double R0, hslope, Rin, Rout, thmin, thmax;
  int n3, istart, istop, jstart, jstop, hstart, hstop;
};

constexpr int FAIL_CAP = 8192;     // failed zones listed by k_fu_flip
constexpr int FIX_LIST_MAX = 512;  // up to this many, repaired through the sorted list
constexpr int NTHR_FIX = 1024;

struct Ctx {
  Grid G;
  Dims D;
  harm_params prm;
  int device;
  cudaStream_t stream;
  double *p, *ph;                // [8][nc]
  double *F1, *F2, *F3;          // [8][nc]
  signed char *pflag;            // [nc]
  double *geo;                   // [4 locations][GEO_N][ng]: FACE1, FACE2, FACE3, CENT
  double *conn;                  // [40][ng]
  double *floors;                // [2][ng]
  double *katm;                  // [sn1]
  double *stage;                 // [8*nc] host-layout staging
  signed char *stage_flag;       // [sn3*sn1*sn2]
  int *fail_list;                // [FAIL_CAP]
  double *fix_buf;               // [FAIL_CAP*8]
  double *partials;              // [3][nparts]
  int nparts;
  DevScalars *sc;
  cudaGraphExec_t graph_exec;
  int graph_steps;
  double *pinned;                // pinned host buffer for the host-array entry points
  size_t pinned_bytes;
  int mode;                      // HARM_FP64 or HARM_MIXED
  float *F1f, *F2f, *F3f;        // mixed mode: FP32 face fluxes [8][nc]
  float *geo32;                  // mixed mode: FP32 geometry [4 locations][GEO_N][ng]
  float *conn32;                 // mixed mode: FP32 connection [40][ng]
  double *Ubuf;                  // conserved variables between the two update launches [8][nc]
  double *emf;                   // flux_ct's corner EMFs e1, e2, e3 [3][nc] (k_emf)
  int tbx, tby;                  // tile of the zone and face kernels: theta x r threads, 128 in all
  long ntr;                      // tracer particles
  double *trX;                   // [3][ntr] code coordinates X1, X2, X3
  int *trids;                    // [ntr][3] labels (i, j, h)
  signed char *trst;             // [ntr] 0 active, 1 in, 2 out, 3 jet, -1 dropped
  TrParams trp;
  bool cool;                     // COOL_EOS step with the run-time EOS below
  EosDev eos;                    // the attached tables (owned by the caller's harm_eos)
  double *lastT;                 // [nc] per-zone temperature guesses (_aLastT)
  bool cool_seed;                // the next step may meet zones without a guess
  double *coolgeo;               // [2][ng] r and |r tan theta| at zone centres (diag.c:225-249)
  double *cooldiag;              // COOL_EOS diagnostics scratch (harm_diag.cu)
};

__device__ __forceinline__ void record_fail(DevScalars *sc, int code, int h, int i, int j)
{
  if (atomicCAS(&sc->fail_code, 0, code) == 0) {
    sc->fail_h = h;
    sc->fail_i = i;
    sc->fail_j = j;
  }
}

__device__ __forceinline__ long cidx(const Grid &G, int h, int i, int j)
{
  return ((long)h * G.sn1 + i) * G.sn2 + j;
}

__device__ __forceinline__ int hwrap(const Grid &G, int h)
{
  return h < 0 ? h + G.n3 : (h >= G.n3 ? h - G.n3 : h);
}

// geometry location slots on the device
enum { L_FACE1 = 0, L_FACE2 = 1, L_FACE3 = 2, L_CENT = 3 };

__device__ __forceinline__ const double *geo_at(const double *geo, const Grid &G, int loc)
{
  return geo + (long)loc * GEO_N * G.ng;
}

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}


__device__ __forceinline__ float warp_minf(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// host helpers (harm_api.cu)

extern thread_local std::string g_err;
int fail_with(int code, const std::string &msg);

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return ::harm::fail_with(HARM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

inline dim3 zone_grid(const Grid &G) { return dim3((G.n2 + 31) / 32, (G.n1 + 3) / 4, G.n3); }

// What the discrete adjoint (harm_adjoint.cu) keeps of one recomputed step;
// index 0 is the predictor, 1 the corrector.  Device pointers, [8][nc] planes
// unless noted.
struct StepRec {
  double *X1[2];                 // the inversion's output after the first bound_prim
  double *Ub[2];                 // the conserved variables the update formed
  double *Z[2];                  // the inversion's output before fixup()
  signed char *wz[2];            // which inversion gave it: 0 Utoprim_2d, 1 and 2 the fall-backs, -1 none [nc]
  double *F1rho[2];              // raw radial mass flux [nc] (the no-inflow fix reads its sign)
  double *ctop;                  // the corrector's face wave speeds, directions 1 and 2 [2][nc]
  signed char *fl1[2];           // pflag after the first bound_prim [nc]
  int *nfail[2];                 // the failed zones fixup_utoprim then met (device int)
  double *ph;                    // the predictor's final state
  DevScalars *sc[2];             // the run state before k_finalize (the corrector's Courant minima) and after
};

// kernels shared by both precisions (harm_api.cu)
int launch_bound(Ctx *x, double *P);
int get_prims(Ctx *x, const double *src, double *p, signed char *pflag);  // device planes -> host layout
int launch_fixup_utoprim(Ctx *x, double *P, int *nfail_out = nullptr);
void launch_mass(Ctx *x);
int sync_status(Ctx *x);

void launch_tracers(Ctx *x);     // update_tracers() (harm_tracers.cu)
int cool_launch_step(Ctx *x);    // the COOL_EOS step (harm_cool.cu)
int cool_time_kernels(Ctx *x, int reps, double *ms);
void invalidate_graph(Ctx *x);   // a captured step no longer matches the context

// one step and the per-kernel timing of each precision variant
namespace exact {
int launch_step(Ctx *x);
int launch_step_rec(Ctx *x, const StepRec &r);  // launch_step, keeping r
int time_kernels(Ctx *x, int reps, double *ms);
}
namespace mixed {
int launch_step(Ctx *x);
int time_kernels(Ctx *x, int reps, double *ms);
}

}  // namespace harm

struct harm_ctx {
  harm::Ctx x;
};

struct harm_eos {
  harm::EosDev d;
  double *axes = nullptr;  // xa[nx] then ya[ny]
  double *vals = nullptr;  // [EOS_ND][ntab][nx][ny]
  float *f32 = nullptr;    // xa32[nx], ya32[ny], e32 and p32 [ntab][nx][ny]
  unsigned char *miss = nullptr;  // [ntab][nx][ny] NaN nodes read (harm_eos_track_missing)
  int device = 0;
};
