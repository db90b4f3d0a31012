// Run-time COOL_EOS tables on the device and the batch entry points
// (harm_eos_create, harm_eos_batch).  The tables are the ones the reference
// builds once per radial index on the host (SetupCache_CoolEOS,
// cooleos.c:825-992): the caller builds them the same way and hands them over.
#include <cmath>
#include <vector>

#include "harm_common.cuh"
#include "harm_eos.cuh"

namespace harm {

__global__ void k_eos_batch(EosDev E, int what, int f32, long n, const int *__restrict__ tab,
                            const double *__restrict__ rho0, const double *__restrict__ u, double *__restrict__ lastT,
                            double *__restrict__ out)
{
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  EosCursor c = eos_cursor(tab[k], lastT[k]);
  double r;
  if (f32) {
    if (what == HARM_EOS_PRESSURE) r = eos_pressure_f(E, c, rho0[k], u[k]);
    else if (what == HARM_EOS_DPDU) r = eos_dpdu_f(E, c, rho0[k], u[k]);
    else r = eos_dpdrho_f(E, c, rho0[k], u[k]);
  } else {
    if (what == HARM_EOS_PRESSURE) r = eos_pressure(E, c, rho0[k], u[k]);
    else if (what == HARM_EOS_DPDU) r = eos_dpdu(E, c, rho0[k], u[k]);
    else r = eos_dpdrho(E, c, rho0[k], u[k]);
  }
  out[k] = r;
  lastT[k] = c.T;
}

// the power of two that centres a plane's magnitudes (log scale) in the float
// range; 0 when they span more than float can hold.  NaN nodes (tables filled
// on demand, nodes not computed yet) stay NaN in the copy and do not count.
static double f32_scale(const std::vector<double> &v, size_t off, size_t n)
{
  double lo = 0., hi = 0.;
  for (size_t k = 0; k < n; k++) {
    double a = fabs(v[off + k]);
    if (a != a) continue;
    if (!(a < 1e308)) return 0.;
    if (a > 0. && (lo == 0. || a < lo)) lo = a;
    if (a > hi) hi = a;
  }
  if (hi == 0.) return 1.;
  int elo, ehi;
  frexp(lo, &elo);
  frexp(hi, &ehi);
  if (ehi - elo > 240) return 0.;
  return ldexp(1.0, -(elo + ehi) / 2);
}

}  // namespace harm

using harm::fail_with;

extern "C" int harm_eos_create(const harm_eos_desc *dsc, const double *xaxis, const double *yaxis,
                               const double *values, const double *hdfac, harm_eos **out)
{
  if (!dsc || !xaxis || !yaxis || !values || !out) return fail_with(HARM_E_ARG, "null argument");
  *out = nullptr;
  if (dsc->nx < 3 || dsc->ny < 3 || dsc->ntab < 1) return fail_with(HARM_E_ARG, "tables need 3 or more nodes per axis");
  for (int k = 1; k < dsc->nx; k++)
    if (!(xaxis[k] > xaxis[k - 1])) return fail_with(HARM_E_ARG, "rho axis not increasing");
  for (int k = 1; k < dsc->ny; k++)
    if (!(yaxis[k] > yaxis[k - 1])) return fail_with(HARM_E_ARG, "T axis not increasing");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  // the EOS calls nest deeper than the default 1 KiB per-thread stack of this
  // process's context (Utoprim_5d -> Jacobian -> pressure -> T solve -> table)
  size_t stack = 0;
  CK(cudaDeviceGetLimit(&stack, cudaLimitStackSize));
  if (stack < 4096) CK(cudaDeviceSetLimit(cudaLimitStackSize, 4096));
  harm_eos *e = new harm_eos();
  e->device = dev;
  const long nx = dsc->nx, ny = dsc->ny, nt = dsc->ntab, plane = nx * ny;
  // reference node order [ntab][nx][ny][5] -> one plane per value [5][ntab][nx][ny]
  std::vector<double> v((size_t)harm::EOS_ND * nt * plane);
  for (long t = 0; t < nt; t++)
    for (long q = 0; q < plane; q++)
      for (int d = 0; d < harm::EOS_ND; d++)
        v[((size_t)d * nt + t) * plane + q] = values[((size_t)t * plane + q) * harm::EOS_ND + d];
  // axes, then each table's HdFac when given
  cudaError_t err = cudaMalloc(&e->axes, (nx + ny + nt) * sizeof(double));
  if (err == cudaSuccess) err = cudaMalloc(&e->vals, v.size() * sizeof(double));
  if (err == cudaSuccess) err = cudaMemcpy(e->axes, xaxis, nx * sizeof(double), cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->axes + nx, yaxis, ny * sizeof(double), cudaMemcpyHostToDevice);
  if (err == cudaSuccess && hdfac)
    err = cudaMemcpy(e->axes + nx + ny, hdfac, nt * sizeof(double), cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(e->vals, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
  // float copies of the axes and of the e and p planes, scaled into range
  const size_t np = (size_t)nt * plane;
  const double se = harm::f32_scale(v, (size_t)harm::EOS_E * np, np);
  const double sp = harm::f32_scale(v, (size_t)harm::EOS_P * np, np);
  const bool f32 = se > 0. && sp > 0.;
  if (f32 && err == cudaSuccess) {
    std::vector<float> f(nx + ny + 2 * np);
    for (long k = 0; k < nx; k++) f[k] = (float)xaxis[k];
    for (long k = 0; k < ny; k++) f[nx + k] = (float)yaxis[k];
    for (size_t k = 0; k < np; k++) {
      f[nx + ny + k] = (float)(v[(size_t)harm::EOS_E * np + k] * se);
      f[nx + ny + np + k] = (float)(v[(size_t)harm::EOS_P * np + k] * sp);
    }
    err = cudaMalloc(&e->f32, f.size() * sizeof(float));
    if (err == cudaSuccess) err = cudaMemcpy(e->f32, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (err != cudaSuccess) {
    cudaFree(e->axes);
    cudaFree(e->vals);
    cudaFree(e->f32);
    delete e;
    return fail_with(HARM_E_CUDA, std::string("EOS tables: ") + cudaGetErrorString(err));
  }
  harm::EosDev &d = e->d;
  d.f32 = f32 ? 1 : 0;
  d.xa32 = f32 ? e->f32 : nullptr;
  d.ya32 = f32 ? e->f32 + nx : nullptr;
  d.e32 = f32 ? e->f32 + nx + ny : nullptr;
  d.p32 = f32 ? e->f32 + nx + ny + np : nullptr;
  d.se = se;
  d.sp = sp;
  d.nx = dsc->nx;
  d.ny = dsc->ny;
  d.ntab = dsc->ntab;
  d.xa = e->axes;
  d.ya = e->axes + nx;
  d.val = e->vals;
  d.rho_unit = dsc->rho_unit;
  d.u_unit = dsc->u_unit;
  d.p_unit = dsc->p_unit;
  d.kbol = dsc->kbol;
  d.mav = dsc->mav;
  d.cl = dsc->cl;
  d.rho_min = dsc->rho_min;
  d.rho_max = dsc->rho_max;
  d.t_min = dsc->t_min;
  d.t_max = dsc->t_max;
  d.hh = dsc->hh;
  d.gam = dsc->gam;
  d.hdfac = hdfac ? e->axes + nx + ny : nullptr;
  d.l_unit = dsc->l_unit;
  d.miss = nullptr;
  *out = e;
  return HARM_OK;
}

extern "C" int harm_eos_destroy(harm_eos *e)
{
  if (!e) return HARM_OK;
  cudaFree(e->axes);
  cudaFree(e->vals);
  cudaFree(e->f32);
  cudaFree(e->miss);
  delete e;
  return HARM_OK;
}

extern "C" int harm_eos_track_missing(harm_eos *e)
{
  if (!e) return fail_with(HARM_E_ARG, "null argument");
  const size_t n = (size_t)e->d.ntab * e->d.nx * e->d.ny;
  if (!e->miss) CK(cudaMalloc(&e->miss, n));
  CK(cudaMemset(e->miss, 0, n));
  e->d.miss = e->miss;
  return HARM_OK;
}

extern "C" int harm_eos_missing(const harm_eos *e, unsigned char *out)
{
  if (!e || !out) return fail_with(HARM_E_ARG, "null argument");
  if (!e->miss) return fail_with(HARM_E_ARG, "missing nodes are not tracked (harm_eos_track_missing)");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(out, e->miss, (size_t)e->d.ntab * e->d.nx * e->d.ny, cudaMemcpyDeviceToHost));
  return HARM_OK;
}

extern "C" int harm_eos_batch(harm_eos *e, int what, int precision, long n, const int *tab, const double *rho0,
                              const double *u, double *lastT, double *out)
{
  if (!e || !tab || !rho0 || !u || !lastT || !out || n < 0) return fail_with(HARM_E_ARG, "null argument");
  if (what != HARM_EOS_PRESSURE && what != HARM_EOS_DPDU && what != HARM_EOS_DPDRHO)
    return fail_with(HARM_E_ARG, "unknown EOS quantity");
  if (precision != HARM_FP64 && precision != HARM_MIXED) return fail_with(HARM_E_ARG, "bad precision");
  if (precision == HARM_MIXED && !e->d.f32) return fail_with(HARM_E_ARG, "table values span more than float holds");
  for (long k = 0; k < n; k++)
    if (tab[k] < 0 || tab[k] >= e->d.ntab) return fail_with(HARM_E_ARG, "table index out of range");
  if (n == 0) return HARM_OK;
  struct Buffers {
    int *t = nullptr;
    double *r = nullptr, *uu = nullptr, *T = nullptr, *o = nullptr;
    ~Buffers() { cudaFree(t); cudaFree(r); cudaFree(uu); cudaFree(T); cudaFree(o); }
  } B;
  CK(cudaMalloc(&B.t, n * sizeof(int)));
  CK(cudaMalloc(&B.r, n * sizeof(double)));
  CK(cudaMalloc(&B.uu, n * sizeof(double)));
  CK(cudaMalloc(&B.T, n * sizeof(double)));
  CK(cudaMalloc(&B.o, n * sizeof(double)));
  CK(cudaMemcpy(B.t, tab, n * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.r, rho0, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.uu, u, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(B.T, lastT, n * sizeof(double), cudaMemcpyHostToDevice));
  harm::k_eos_batch<<<(unsigned)((n + 127) / 128), 128>>>(e->d, what, precision == HARM_MIXED, n, B.t, B.r, B.uu,
                                                           B.T, B.o);
  CK(cudaGetLastError());
  CK(cudaMemcpy(out, B.o, n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(lastT, B.T, n * sizeof(double), cudaMemcpyDeviceToHost));
  return HARM_OK;
}
