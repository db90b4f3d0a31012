// Measured FP64 pipe peaks of the device, for the FP64 roofline of the step
// kernels.  The step is built with -fmad=false, so its arithmetic reaches the
// FP64 pipe as separate DADD and DMUL instructions (one flop each), plus the
// DFMA sequences of IEEE division and square root; the roofline that bounds it
// is therefore the pipe's instruction rate, measured here for each kind, next
// to the DFMA flop rate (two flops per instruction).
//
// Each kernel runs 8 independent dependency chains per thread over a grid of
// 8 blocks of 256 threads per SM, long enough (tens of ms) for CUDA events to
// time it; the result is stored only under a condition the inputs never meet,
// so nothing is optimised away.
#include <cuda_runtime.h>

#include "harm_common.cuh"

namespace harm {

constexpr int PEAK_CHAINS = 8;

template <int OP>
__global__ void __launch_bounds__(256) k_fp64_peak(int iters, double a, double b, double *sink)
{
  double x[PEAK_CHAINS];
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; c++) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) {
      if (OP == 0) x[c] = fma(x[c], a, b);   // DFMA
      else if (OP == 1) x[c] = x[c] + b;     // DADD
      else if (OP == 2) x[c] = x[c] * a;     // DMUL
      else if (OP == 3) x[c] = x[c] / a;     // IEEE division
      else x[c] = __drcp_rn(x[c]);           // IEEE reciprocal
    }
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; c++) s += x[c];
  if (s == 1234.5678) sink[threadIdx.x] = s;
}

template <int OP>
static int time_peak(int sms, int iters, double *rate)
{
  const dim3 grid(8 * sms), block(256);
  double *sink = nullptr;
  CK(cudaMalloc(&sink, 256 * sizeof(double)));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // a = 1 - 2^-30 keeps the products and quotients far from overflow and underflow
  const double a = 1.0 - 9.313225746154785e-10, b = 1e-12;
  k_fp64_peak<OP><<<grid, block>>>(iters / 8, a, b, sink);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    CK(cudaEventRecord(e0));
    k_fp64_peak<OP><<<grid, block>>>(iters, a, b, sink);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float ms;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  *rate = (double)grid.x * block.x * PEAK_CHAINS * (double)iters / (best * 1e-3);
  return HARM_OK;
}

// ---------------------------------------------------------------------------
// div_rn (harm_phys.cuh) against the IEEE division on this device

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long &s)
{
  unsigned long long z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// a double with a random significand, the given unbiased exponent and sign
__device__ __forceinline__ double make_double(unsigned long long mant, int e, bool neg)
{
  return __longlong_as_double((long long)(((unsigned long long)neg << 63) |
                                          ((unsigned long long)(e + 1023) << 52) | (mant & 0xfffffffffffffULL)));
}

// Each sample draws a divisor b (significand random or all ones, exponent in
// [-60, 60]) and a numerator a: either random (exponent in [-820, 820],
// zeros, signed zeros, subnormals, infinities and NaNs among them) or built
// so that a/b lies within a few ulps of 2^-54 of a midpoint between two
// doubles, where the last correction decides.  counts[0]: samples whose
// div_rn differs in any bit from a / b; counts[1]: near-midpoint samples.
__global__ void k_div_check(long n, unsigned long long seed, unsigned long long *counts)
{
  unsigned long long bad = 0, mid = 0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    unsigned long long s = seed ^ (0x632be59bd9b4e019ULL * (unsigned long long)(t + 1));
    const unsigned long long r0 = splitmix64(s), r1 = splitmix64(s), r2 = splitmix64(s), r3 = splitmix64(s);
    const int eb = (int)(r0 % 121) - 60;
    const double b = make_double((r0 >> 8) % 5 == 0 ? ~0ULL : r1, eb, false);
    const double y = 1. / b;
    double a;
    const int mode = (int)(r2 % 16);
    if (mode < 8) {
      a = make_double(r3, (int)((r2 >> 8) % 1641) - 820, (r2 >> 20) & 1);
    } else if (mode < 14) {
      // q random; a = b (q + half an ulp of q) rounded: a/b is within about an ulp
      // of a (times 2^-53 relative) of that midpoint
      const double q = make_double(r3, (int)((r2 >> 8) % 121) - 60, (r2 >> 20) & 1);
      const double hulp = __longlong_as_double((long long)((((__double_as_longlong(q) >> 52) & 0x7ff) - 53)) << 52);
      const double p = b * q, e = fma(b, q, -p);
      a = p + (e + b * ((r2 >> 21) & 1 ? hulp : -hulp));
      mid++;
    } else {
      const int k = (int)((r2 >> 8) % 6);
      const double sp[6] = {0., -0., 4.9e-324, 1e300, __longlong_as_double(0x7ff0000000000000LL),
                            __longlong_as_double(0x7ff8000000000000LL)};
      a = sp[k] * ((r2 >> 20) & 1 ? -1. : 1.);
    }
    const double d0 = a / b, d1 = div_rn(a, b, y);
    if (__double_as_longlong(d0) != __double_as_longlong(d1) && !(d0 != d0 && d1 != d1)) bad++;
  }
  atomicAdd(&counts[0], bad);
  atomicAdd(&counts[1], mid);
}

// pow_third (harm_pow.cuh) against the general double-double path pow_dd:
// x with a random significand and an exponent in [-700, 699], y = RN(4/3) or
// RN(4/3) - 1.  counts[0]: samples where pow_third decided and differs from
// pow_dd in any bit; counts[1]: samples it left to pow_dd.
__global__ void k_pow_check(long n, unsigned long long seed, unsigned long long *counts)
{
  unsigned long long bad = 0, undecided = 0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    unsigned long long s = seed ^ (0x632be59bd9b4e019ULL * (unsigned long long)(t + 1));
    const unsigned long long r0 = splitmix64(s), r1 = splitmix64(s);
    const double x = make_double(r1, (int)(r0 % 1400) - 700, false);
    const double y = (r0 >> 32) & 1 ? 1.3333333333333333 : 0.33333333333333326;
    double f;
    if (pow_third(x, y, f)) {
      const double g = pow_dd(x, y);
      if (__double_as_longlong(f) != __double_as_longlong(g)) bad++;
    } else {
      undecided++;
    }
  }
  atomicAdd(&counts[0], bad);
  atomicAdd(&counts[1], undecided);
}

}  // namespace harm

extern "C" int harm_pow_check(int device, long n, unsigned long long seed, unsigned long long *counts)
{
  using namespace harm;
  if (!counts || n < 0) return fail_with(HARM_E_ARG, "harm_pow_check: bad arguments");
  CK(cudaSetDevice(device));
  unsigned long long *d = nullptr;
  CK(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  CK(cudaMemset(d, 0, 2 * sizeof(unsigned long long)));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  k_pow_check<<<8 * sms, 256>>>(n, seed, d);
  CK(cudaGetLastError());
  CK(cudaMemcpy(counts, d, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return HARM_OK;
}

extern "C" int harm_div_check(int device, long n, unsigned long long seed, unsigned long long *counts)
{
  using namespace harm;
  if (!counts || n < 0) return fail_with(HARM_E_ARG, "harm_div_check: bad arguments");
  CK(cudaSetDevice(device));
  unsigned long long *d = nullptr;
  CK(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  CK(cudaMemset(d, 0, 2 * sizeof(unsigned long long)));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  k_div_check<<<8 * sms, 256>>>(n, seed, d);
  CK(cudaGetLastError());
  CK(cudaMemcpy(counts, d, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return HARM_OK;
}

extern "C" int harm_fp64_peak(int device, double *out)
{
  using namespace harm;
  if (!out) return fail_with(HARM_E_ARG, "harm_fp64_peak: null output");
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  int rc;
  if ((rc = time_peak<0>(sms, 16384, &out[0])) != HARM_OK) return rc;
  if ((rc = time_peak<1>(sms, 16384, &out[1])) != HARM_OK) return rc;
  if ((rc = time_peak<2>(sms, 16384, &out[2])) != HARM_OK) return rc;
  if ((rc = time_peak<3>(sms, 2048, &out[3])) != HARM_OK) return rc;
  if ((rc = time_peak<4>(sms, 2048, &out[4])) != HARM_OK) return rc;
  return HARM_OK;
}
