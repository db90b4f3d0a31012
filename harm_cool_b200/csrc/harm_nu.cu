// The COOL_EOS table generator on the device: abundance() (harm_nu.cuh) at
// every node of the per-radius (rho, T) tables, one warp per node.
//
// The reference fills the same tables lazily on the host, node by node, with
// six worker threads calling its Fortran abundance_() (cooleos.c:171-194,
// 805-820; cache4d.c) and caches them in files.  Here every node of every
// table is computed in one pass before the run.  A node is a nest of Newton
// solves whose trials evaluate Fermi and rate integrals by Gauss quadrature,
// in FP64; its cost varies by four orders of magnitude with the temperature
// (where free nucleons are a trace, at a few 1e8 K, the proton-fraction solve
// runs all 200 of its trials, each over three nested solves).  A thread per
// node would leave a warp waiting on its slowest lane and run each
// quadrature's terms one after another; a warp per node keeps its lanes on
// one control flow and spreads the terms of every quadrature over them
// (lane_sum, harm_nu.cuh).
//
// Six blocks of four warps per SM (80 registers a thread): the warps' long
// FP64 latency chains (exp, log, division) need that many to keep the FP64
// pipe busy; measured 1.13x faster than four blocks at 128 registers, which
// were 1.44x faster than three at 168.
//
// Tables are launched one per kernel over several streams without waiting in
// between, so the blocks of a table still on its slowest nodes share the SMs
// with the next tables' blocks.  Every loop in the physics has a fixed trip
// count or the 200-trial cap of the Newton solver, so every warp ends.
#include "harm_b200.h"
#include "harm_common.cuh"
#include "harm_nu.cuh"

#include <cuda_runtime.h>

#include <vector>

namespace harm {
namespace nu {
const Rules *host_rules();

__constant__ Rules c_rules;

// the quadrature rules into shared memory: the lanes of a warp read different
// nodes of a rule at once, which the constant cache would serialise
__device__ __forceinline__ void load_rules(Rules &R)
{
  for (int q = threadIdx.x; q < (int)(sizeof(Rules) / sizeof(double)); q += blockDim.x)
    reinterpret_cast<double *>(&R)[q] = reinterpret_cast<const double *>(&c_rules)[q];
  __syncthreads();
}

// node k of the slice [k0, k0 + n) on warp k - k0, with k = (t ny + j) nx + i
// for table t, T index j and rho index i; values packed as calc_cache_val
// packs them (cooleos.c:171-194) at values[t][i][j]: e, p, Qnu, tau,
// Yee = (n_e- - n_e+) / n_b
__global__ void __launch_bounds__(128, 6) k_tables(const double *xaxis, int nx, const double *yaxis, int ny,
                                                const double *hdfac, long k0, long n, double *values)
{
  __shared__ Rules R;
  load_rules(R);
  const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;  // whole warps: the lanes of a node stay together
  const long k = k0 + w;
  const int i = (int)(k % nx);
  const long tj = k / nx;
  const int j = (int)(tj % ny), t = (int)(tj / ny);
  const double rho = xaxis[i];
  const Abundance a = abundance(R, rho, yaxis[j], hdfac[t]);
  if ((threadIdx.x & 31) == 0) {
    double *v = values + 5 * (((long)t * nx + i) * ny + j);
    v[0] = a.e;
    v[1] = a.p;
    v[2] = a.qnu;
    v[3] = a.tau;
    v[4] = (a.nee - a.nep) / (rho / 1.66e15);
  }
}

// abundance() at a list of nodes, a warp per node, for checks against the host
__global__ void __launch_bounds__(128, 6) k_nodes(const double *rho, const double *T, const double *hdfac, long n,
                                               double *out)
{
  __shared__ Rules R;
  load_rules(R);
  const long k = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= n) return;
  const Abundance a = abundance(R, rho[k], T[k], hdfac[k]);
  if ((threadIdx.x & 31) == 0) {
    double *o = out + 7 * k;
    o[0] = a.e;
    o[1] = a.p;
    o[2] = a.qnu;
    o[3] = a.tau;
    o[4] = a.nee;
    o[5] = a.nep;
    o[6] = a.xp;
  }
}

static int upload_rules(int device)
{
  static int done[64];
  if (device < 0 || device >= 64) return fail_with(HARM_E_ARG, "harm_nu: bad device");
  if (done[device]) return HARM_OK;
  const Rules *R = host_rules();
  if (!R) return fail_with(HARM_E_ARG, "harm_nu: quadrature root search failed");
  CK(cudaMemcpyToSymbol(c_rules, R, sizeof(Rules)));
  done[device] = 1;
  return HARM_OK;
}

// device buffers freed on every return path
struct DevBufs {
  std::vector<void *> p;
  ~DevBufs()
  {
    for (void *q : p) cudaFree(q);
  }
  template <class T>
  cudaError_t alloc(T **ptr, size_t count)
  {
    void *q = nullptr;
    const cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e == cudaSuccess) p.push_back(q);
    *ptr = (T *)q;
    return e;
  }
};

}  // namespace nu
}  // namespace harm

using namespace harm;

extern "C" int harm_nu_tables(int device, const double *xaxis, int nx, const double *yaxis, int ny,
                              const double *hdfac, int ntab, long slice, double *values, float *ms)
{
  if (nx <= 0 || ny <= 0 || ntab <= 0 || !xaxis || !yaxis || !hdfac || !values)
    return fail_with(HARM_E_ARG, "harm_nu_tables: bad arguments");
  CK(cudaSetDevice(device));
  int rc = nu::upload_rules(device);
  if (rc != HARM_OK) return rc;
  const long n = (long)nx * ny * ntab;
  if (slice <= 0) slice = (long)nx * ny;  // a table per launch
  nu::DevBufs b;
  double *dx, *dy, *dh, *dv;
  CK(b.alloc(&dx, nx));
  CK(b.alloc(&dy, ny));
  CK(b.alloc(&dh, ntab));
  CK(b.alloc(&dv, 5 * n));
  CK(cudaMemcpy(dx, xaxis, nx * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dy, yaxis, ny * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dh, hdfac, ntab * sizeof(double), cudaMemcpyHostToDevice));
  // slices on NS streams, each stream's first slice after e0 and e1 after
  // every stream's last; streams and events released on every return path
  constexpr int NS = 8;
  struct Res {
    cudaStream_t st[NS] = {};
    cudaEvent_t e0 = nullptr, e1 = nullptr, done[NS] = {};
    ~Res()
    {
      for (int s = 0; s < NS; s++) {
        if (done[s]) cudaEventDestroy(done[s]);
        if (st[s]) cudaStreamDestroy(st[s]);
      }
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } r;
  CK(cudaEventCreate(&r.e0));
  CK(cudaEventCreate(&r.e1));
  for (int s = 0; s < NS; s++) {
    CK(cudaStreamCreateWithFlags(&r.st[s], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&r.done[s], cudaEventDisableTiming));
  }
  CK(cudaDeviceSynchronize());
  CK(cudaEventRecord(r.e0, r.st[0]));
  for (int s = 1; s < NS; s++) CK(cudaStreamWaitEvent(r.st[s], r.e0, 0));
  int q = 0;
  for (long k0 = 0; k0 < n; k0 += slice, q = (q + 1) % NS) {
    const long m = (n - k0 < slice) ? n - k0 : slice;
    nu::k_tables<<<(unsigned)((m + 3) / 4), 128, 0, r.st[q]>>>(dx, nx, dy, ny, dh, k0, m, dv);
    CK(cudaGetLastError());
  }
  for (int s = 1; s < NS; s++) {
    CK(cudaEventRecord(r.done[s], r.st[s]));
    CK(cudaStreamWaitEvent(r.st[0], r.done[s], 0));
  }
  CK(cudaEventRecord(r.e1, r.st[0]));
  CK(cudaEventSynchronize(r.e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, r.e0, r.e1));
  if (ms) *ms = t;
  CK(cudaMemcpy(values, dv, 5 * n * sizeof(double), cudaMemcpyDeviceToHost));
  return HARM_OK;
}

extern "C" int harm_nu_abundance_dev(int device, const double *rho, const double *T, const double *hdfac, long n,
                                     double *out)
{
  if (n <= 0 || !rho || !T || !hdfac || !out) return fail_with(HARM_E_ARG, "harm_nu_abundance_dev: bad arguments");
  CK(cudaSetDevice(device));
  int rc = nu::upload_rules(device);
  if (rc != HARM_OK) return rc;
  nu::DevBufs b;
  double *dr, *dt, *dh, *dout;
  CK(b.alloc(&dr, n));
  CK(b.alloc(&dt, n));
  CK(b.alloc(&dh, n));
  CK(b.alloc(&dout, 7 * n));
  CK(cudaMemcpy(dr, rho, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dt, T, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dh, hdfac, n * sizeof(double), cudaMemcpyHostToDevice));
  nu::k_nodes<<<(unsigned)((n + 3) / 4), 128>>>(dr, dt, dh, n, dout);
  CK(cudaGetLastError());
  CK(cudaMemcpy(out, dout, 7 * n * sizeof(double), cudaMemcpyDeviceToHost));
  return HARM_OK;
}
