// Tracer particles (tracers.c) on the device: one thread per tracer moves it
// by the interpolated coordinate velocity u^i/u^t over the step's dt and
// retires it when it falls in or leaves, as update_tracers() does
// (tracers.c:298-429) after diag_mass (step_ch.c:121-123).  The reference
// keeps a std::vector and erases retired tracers; here every tracer keeps its
// slot and a status (0 active, 1 fell in, 2 left inside the theta window, 3
// left in the jet, -1 dropped because the search found no zone), so the list
// needs no compaction and stays in its original order.  The per-tracer dump
// files and their renames (dump_one_tracer, tracers.c:468-510) are host I/O
// and are not reproduced: the status says where a retired tracer went.
// Built with -fmad=false, so positions follow the reference's arithmetic.
#include <vector>

#include "harm_common.cuh"

namespace harm {
namespace {

// coord() (metric.c:62-115), CENT and FACE3, single rank
__host__ __device__ inline void tr_coord(const TrParams &T, int h, int i, int j, bool face3, double *X)
{
  i -= 2;
  j -= 2;
  h -= T.n3 > 1 ? 1 : 0;
  X[1] = T.sx1 + (i + 0.5) * T.dx1;
  X[2] = T.sx2 + (j + 0.5) * T.dx2;
  X[3] = (face3 || T.n3 <= 2) ? T.sx3 + h * T.dx3 : T.sx3 + (h + 0.5) * T.dx3;
}

// search_tracer() (tracers.c:39-98): linear scans, as the reference does
__host__ __device__ inline bool tr_search(const TrParams &T, const double *XX, int &hh, int &ii, int &jj)
{
  double Xl[4], Xr[4];
  tr_coord(T, T.hstart, T.istart - 1, T.jstart - 1, false, Xl);
  if (XX[1] < Xl[1] || XX[2] < Xl[2]) return false;
  hh = 0;
  bool ok = false;
  for (int i = T.istart - 1; i <= T.istop && !ok; i++) {
    tr_coord(T, T.hstart, i, T.jstart, false, Xl);
    tr_coord(T, T.hstart, i + 1, T.jstart, false, Xr);
    if (XX[1] >= Xl[1] && XX[1] < Xr[1]) { ii = i; ok = true; }
  }
  if (!ok) return false;
  ok = false;
  for (int j = T.jstart - 1; j <= T.jstop && !ok; j++) {
    tr_coord(T, T.hstart, T.istart, j, false, Xl);
    tr_coord(T, T.hstart, T.istart, j + 1, false, Xr);
    if (XX[2] >= Xl[2] && XX[2] < Xr[2]) { jj = j; ok = true; }
  }
  if (!ok) return false;
  if (T.n3 > 2) {
    ok = false;
    for (int h = T.hstart; h <= T.hstop && !ok; h++) {
      tr_coord(T, h, T.istart, T.jstart, true, Xl);
      tr_coord(T, h + 1, T.istart, T.jstart, true, Xr);
      if (XX[3] >= Xl[3] && XX[3] < Xr[3]) { hh = h; ok = true; }
    }
    if (!ok) return false;
  }
  return true;
}

// ucon_fun() (tracers.c:257-269) at reference zone (h, i, j); device planes wrap in phi
__device__ inline void tr_ucon(const Grid &G, const double *__restrict__ P, const double *__restrict__ gC, int h,
                               int i, int j, double *ucon, int *fail)
{
  const int hd = G.n3 > 1 ? hwrap(G, h - 1) : 0;
  const long c = cidx(G, hd, i, j);
  double pr[8];
#pragma unroll
  for (int k = 0; k < 8; k++) pr[k] = __ldg(P + k * G.nc + c);
  Geo q;
  load_geo(gC, G.ng, (long)i * G.sn2 + j, q);
  ucon_calc(pr, q, ucon, fail);
  ucon[1] /= ucon[0];
  ucon[2] /= ucon[0];
  ucon[3] /= ucon[0];
}

__global__ void __launch_bounds__(128) k_tracers(Grid G, TrParams T, const double *__restrict__ P,
                                                 const double *__restrict__ geo, double *X, signed char *st, long n,
                                                 DevScalars *sc)
{
  if (sc->halted) return;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n || st[t] != 0) return;
  const double Dt = sc->dt;
  const double *gC = geo_at(geo, G, L_CENT);
  double tX[4] = {0., X[t], X[n + t], X[2 * n + t]};
  int hh, ii, jj;
  if (!tr_search(T, tX, hh, ii, jj)) {
    st[t] = -1;
    return;
  }
  // linear_interpolation() (tracers.c:193-254) of ucon_fun, theta, then r, then phi
  const int WPH = T.n3 > 2 ? 2 : 1;
  double tmp2[2][4];
  int fail = 0;
  for (int l3 = 0; l3 < WPH; l3++) {
    double tmp1[2][4];
    double r00 = 0., r11 = 0.;  // XX[l3][0][0][RR] and XX[l3][1][1][RR]
    for (int l1 = 0; l1 < 2; l1++) {
      double Xa[4], Xb[4], va[4], vb[4];
      tr_coord(T, hh + l3, ii + l1, jj, false, Xa);
      tr_coord(T, hh + l3, ii + l1, jj + 1, false, Xb);
      tr_ucon(G, P, gC, hh + l3, ii + l1, jj, va, &fail);
      tr_ucon(G, P, gC, hh + l3, ii + l1, jj + 1, vb, &fail);
      const double T1 = 1.0 / (Xb[2] - Xa[2]);
      const double T2 = tX[2] - Xa[2];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double ypval = (vb[k] - va[k]) * T1;
        tmp1[l1][k] = va[k] + T2 * ypval;
      }
      if (l1 == 0) r00 = Xa[1];
      else r11 = Xb[1];
    }
    const double T1 = 1.0 / (r11 - r00);
    const double T2 = tX[1] - r00;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double ypval = (tmp1[1][k] - tmp1[0][k]) * T1;
      tmp2[l3][k] = tmp1[0][k] + T2 * ypval;
    }
  }
  double ucon[4];
  if (WPH == 1) {
#pragma unroll
    for (int k = 0; k < 4; k++) ucon[k] = tmp2[0][k];
  } else {
    double Xa[4], Xb[4];
    tr_coord(T, hh, ii, jj, false, Xa);              // XX[0][0][0]
    tr_coord(T, hh + 1, ii + 1, jj + 1, false, Xb);  // XX[1][1][1]
    const double T1 = 1.0 / (Xb[3] - Xa[3]);
    const double T2 = tX[3] - Xa[3];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double ypval = (tmp2[1][k] - tmp2[0][k]) * T1;
      ucon[k] = tmp2[0][k] + T2 * ypval;
    }
  }
  if (fail) record_fail(sc, fail, hh, ii, jj);
  for (int k = 1; k < 4; k++) tX[k] += ucon[k] * Dt;
  // bl_coord() (coord.c:61-124): gammie_coords with COORDSINGFIX
  const double r = exp(tX[1]) + T.R0;
  double th = M_PI_2 * (1. + tX[2]) + ((1. - T.hslope) / 2.) * sin(M_PI * (1. + tX[2]));
  if (fabs(th) < 1.E-20) th = th >= 0 ? 1.E-20 : -1.E-20;
  if (fabs(M_PI - th) < 1.E-20) th = th >= M_PI ? M_PI + 1.E-20 : M_PI - 1.E-20;
  signed char s = 0;
  if (r < T.Rin || th < 0 || th > M_PI) s = 1;
  else if (r >= T.Rout) s = (th >= T.thmin && th <= T.thmax) ? 2 : 3;
  // back into [0, 2 pi] for those that stay (tracers.c:385-408)
  if (s == 0 && T.n3 > 2) {
    if (tX[3] < 0.) tX[3] += 2. * M_PI;
    else if (tX[3] > 2. * M_PI) tX[3] -= 2. * M_PI;
  }
  X[t] = tX[1];
  X[n + t] = tX[2];
  X[2 * n + t] = tX[3];
  st[t] = s;
}

TrParams tr_params(const Ctx *x, const harm_grid_spec &g)
{
  const harm_params &p = x->prm;
  TrParams T;
  T.sx1 = p.startx[1]; T.sx2 = p.startx[2]; T.sx3 = p.startx[3];
  T.dx1 = p.dx[1]; T.dx2 = p.dx[2]; T.dx3 = p.dx[3];
  T.R0 = g.R0;
  T.hslope = g.hslope;
  // init_tracers() (tracers.c:118-123)
  T.Rin = exp(p.startx[1] - 0.5 * p.dx[1]) + g.R0;
  T.Rout = 0.8 * (exp(p.startx[1] + p.n1 * p.dx[1]) + g.R0);
  T.thmin = 0.02 * M_PI;
  T.thmax = 0.98 * M_PI;
  T.n3 = p.n3;
  T.istart = 2; T.istop = p.n1 + 1;
  T.jstart = 2; T.jstop = p.n2 + 1;
  T.hstart = p.n3 > 1 ? 1 : 0; T.hstop = p.n3 > 1 ? p.n3 : 0;
  return T;
}

int tr_upload(Ctx *x, const int *ids, const double *X, long n)
{
  cudaFree(x->trX);
  cudaFree(x->trids);
  cudaFree(x->trst);
  x->trX = nullptr;
  x->trids = nullptr;
  x->trst = nullptr;
  x->ntr = 0;
  invalidate_graph(x);
  if (n == 0) return HARM_OK;
  CK(cudaMalloc(&x->trX, 3 * n * sizeof(double)));
  CK(cudaMalloc(&x->trids, 3 * n * sizeof(int)));
  CK(cudaMalloc(&x->trst, n));
  std::vector<double> planes(3 * (size_t)n);
  for (long k = 0; k < n; k++)
    for (int m = 0; m < 3; m++) planes[m * (size_t)n + k] = X[3 * k + m];
  CK(cudaMemcpy(x->trX, planes.data(), planes.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(x->trids, ids, 3 * n * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemset(x->trst, 0, n));
  x->ntr = n;
  return HARM_OK;
}

}  // namespace

void launch_tracers(Ctx *x)
{
  const long n = x->ntr;
  k_tracers<<<(unsigned)((n + 127) / 128), 128, 0, x->stream>>>(x->G, x->trp, x->p, x->geo, x->trX, x->trst, n,
                                                                 x->sc);
}

}  // namespace harm

using namespace harm;

extern "C" int harm_tracers_init(harm_ctx *h, const harm_grid_spec *g, long *count)
{
  if (!h || !g) return fail_with(HARM_E_ARG, "null argument");
  Ctx *x = &h->x;
  const Grid &G = x->G;
  const TrParams T = tr_params(x, *g);
  // the density of every cell (plane RHO of the device state)
  std::vector<double> rho(G.nc);
  CK(cudaStreamSynchronize(x->stream));
  CK(cudaMemcpy(rho.data(), x->p, G.nc * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<int> ids;
  std::vector<double> X;
  // init_tracers() (tracers.c:153-180): zone centres in h, i, j order
  for (int hz = 0; hz < G.n3; hz++)
    for (int i = 0; i < G.n1; i++)
      for (int j = 0; j < G.n2; j++) {
        double tX[4] = {0., T.sx1 + (i + 0.5) * T.dx1, T.sx2 + (j + 0.5) * T.dx2, T.sx3 + hz * T.dx3};
        int hh, ii, jj;
        if (!tr_search(T, tX, hh, ii, jj)) continue;
        const int hd = G.n3 > 1 ? (hh - 1) % G.n3 : 0;
        if (rho[((size_t)hd * G.sn1 + ii) * G.sn2 + jj] > RHOMIN) {
          ids.insert(ids.end(), {i, j, hz});
          X.insert(X.end(), {tX[1], tX[2], tX[3]});
        }
      }
  x->trp = T;
  int rc = tr_upload(x, ids.data(), X.data(), (long)ids.size() / 3);
  if (rc) return rc;
  if (count) *count = x->ntr;
  return HARM_OK;
}

extern "C" int harm_tracers_put(harm_ctx *h, const harm_grid_spec *g, const int *ids, const double *X, long n)
{
  if (!h || !g || n < 0 || (n > 0 && (!ids || !X))) return fail_with(HARM_E_ARG, "bad argument");
  Ctx *x = &h->x;
  CK(cudaStreamSynchronize(x->stream));
  x->trp = tr_params(x, *g);
  return tr_upload(x, ids, X, n);
}

extern "C" int harm_tracers_count(harm_ctx *h, long *n)
{
  if (!h || !n) return fail_with(HARM_E_ARG, "null argument");
  *n = h->x.ntr;
  return HARM_OK;
}

extern "C" int harm_tracers_get(harm_ctx *h, int *ids, double *X, signed char *status)
{
  if (!h) return fail_with(HARM_E_ARG, "null context");
  Ctx *x = &h->x;
  const long n = x->ntr;
  CK(cudaStreamSynchronize(x->stream));
  if (n == 0) return HARM_OK;
  if (ids) CK(cudaMemcpy(ids, x->trids, 3 * n * sizeof(int), cudaMemcpyDeviceToHost));
  if (X) {
    std::vector<double> planes(3 * (size_t)n);
    CK(cudaMemcpy(planes.data(), x->trX, planes.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (long k = 0; k < n; k++)
      for (int m = 0; m < 3; m++) X[3 * k + m] = planes[m * (size_t)n + k];
  }
  if (status) CK(cudaMemcpy(status, x->trst, n, cudaMemcpyDeviceToHost));
  return HARM_OK;
}
