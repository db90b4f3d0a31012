// harm_utoprim_2d_batch_noalloc: the batched Utoprim_2d inversion with its
// device working memory in a fixed array inside this library, so that a call
// allocates and frees nothing.
//
// Who needs this.  harm_utoprim_2d_batch stages the caller's host arrays in
// device buffers that it allocates and frees on every call.  Some hosts of
// this code cannot do that:
//   * a simulation that sized its resident state to the GPU's memory (a
//     288x256x256 FP64 run with its fluxes and geometry), or that hands all
//     device memory to another allocator up front (a caching allocator such
//     as PyTorch's), has no room left for new allocations in mid-run;
//   * cudaFree waits for the whole device to go idle, so a host that re-inverts
//     a few zones (restart, repair of failed zones) while the step pipeline runs
//     on other streams would stall that pipeline on every call.
// This entry point copies into, runs on and copies out of the array below.
//
// Limits.  At most HARM_U2P_NOALLOC_MAX zones per call; larger batches are
// rejected with HARM_E_ARG before any device work.  Every GPU that loads the
// library holds the array (about 6.2 MiB) until the process exits.  All calls
// on a device share the one array, and it keeps the last call's contents:
// two calls whose work overlaps on the GPU (for example from two host threads
// at once) race and corrupt each other's results.  Each call writes every
// slot that its kernel reads before the kernel runs, and the kernel writes
// every return code, so nothing has to start at zero.
//
// Set-up.  Host code cannot use the array's name as a device address: on the
// host it names a stand-in object, and a kernel given that address would
// fault or read the wrong memory.  The first call on each device therefore
// asks the runtime for the array's device address (cudaGetSymbolAddress, with
// that device current) and creates one non-blocking stream for the calls
// (so they do not serialise with the host's blocking streams), and keeps both
// for later calls.  Make that first call before any stream capture is begun on
// the device.  Both belong to the device's primary context: a host that
// resets the device (cudaDeviceReset) after the first call must not call this
// entry point again in that process.
#include <mutex>

#include "harm_common.cuh"

namespace harm {
namespace {

constexpr long kMax = HARM_U2P_NOALLOC_MAX;
// doubles per zone: U 8, gcov 16, gcon 16, gdet 1, prim 8; then one int per zone
constexpr long kOffU = 0, kOffCov = 8 * kMax, kOffCon = 24 * kMax, kOffDet = 40 * kMax, kOffPrim = 41 * kMax,
               kOffRet = 49 * kMax, kDoubles = 49 * kMax + kMax / 2;

static __device__ __align__(256) double g_u2p_scratch[kDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices];          // device address of g_u2p_scratch, per device
cudaStream_t g_stream[kMaxDevices];   // the calls' stream, per device

int scratch_address(double **out, cudaStream_t *st)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail_with(HARM_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_u2p_scratch);
    if (e != cudaSuccess)
      return fail_with(HARM_E_CUDA, std::string("cudaGetSymbolAddress(g_u2p_scratch): ") + cudaGetErrorString(e));
    cudaStream_t s = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail_with(HARM_E_CUDA, std::string("cudaStreamCreateWithFlags: ") + cudaGetErrorString(e));
    g_stream[dev] = s;
    g_addr[dev] = static_cast<double *>(p);
  }
  *out = g_addr[dev];
  *st = g_stream[dev];
  return HARM_OK;
}

// the same per-zone work as k_utoprim_batch, on operands laid out in the
// fixed array at the offsets above
__global__ void k_utoprim_batch_fixed(double *S, long n, double gam)
{
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double *a = S + kOffCov + t * 16, *b = S + kOffCon + t * 16;
  Geo q;
  q.v00 = a[0]; q.v01 = a[1]; q.v03 = a[3]; q.v11 = a[5]; q.v13 = a[7]; q.v22 = a[10]; q.v33 = a[15];
  q.n00 = b[0]; q.n01 = b[1]; q.n03 = b[3]; q.n10 = b[4]; q.n11 = b[5]; q.n13 = b[7]; q.n22 = b[10];
  q.n30 = b[12]; q.n31 = b[13]; q.n33 = b[15];
  q.alpha = 1. / sqrt(-q.n00);
  q.g = S[kOffDet + t];
  q.ialpha = 1. / q.alpha;
  q.ig = 1. / q.g;
  double u[8], p[8];
  for (int k = 0; k < 8; k++) { u[k] = S[kOffU + t * 8 + k]; p[k] = S[kOffPrim + t * 8 + k]; }
  reinterpret_cast<int *>(S + kOffRet)[t] = utoprim<0>(gam, 0., u, q, p);
  for (int k = 0; k < 8; k++) S[kOffPrim + t * 8 + k] = p[k];
}

}  // namespace
}  // namespace harm

using namespace harm;

extern "C" int harm_utoprim_2d_batch_noalloc(const double *U, const double *gcov, const double *gcon,
                                             const double *gdet, double *prim, int *ret, long n, double gam)
{
  if (!U || !gcov || !gcon || !gdet || !prim || !ret || n < 0) return fail_with(HARM_E_ARG, "null argument");
  if (n > kMax)
    return fail_with(HARM_E_ARG, "harm_utoprim_2d_batch_noalloc: " + std::to_string(n) +
                                     " zones exceed its fixed device buffer of HARM_U2P_NOALLOC_MAX = " +
                                     std::to_string(kMax) + " zones; split the batch");
  if (n == 0) return HARM_OK;
  double *S = nullptr;
  cudaStream_t st = nullptr;
  int rc = scratch_address(&S, &st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(S + kOffU, U, n * 8 * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(S + kOffCov, gcov, n * 16 * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(S + kOffCon, gcon, n * 16 * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(S + kOffDet, gdet, n * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(S + kOffPrim, prim, n * 8 * sizeof(double), cudaMemcpyHostToDevice, st));
  k_utoprim_batch_fixed<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, n, gam);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(prim, S + kOffPrim, n * 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(ret, S + kOffRet, n * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return HARM_OK;
}
