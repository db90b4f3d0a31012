// Cell enumeration of bound_prim() and the repair stencils of
// fixup_utoprim(), shared by the step's kernels (harm_api.cu) and by the
// discrete adjoint that transposes them (harm_adjoint.cu).
#pragma once
#include "harm_common.cuh"

namespace harm {

struct BoundCell { int i, j; };

__device__ __forceinline__ BoundCell bound_cell(const Grid &G, int t, int nrow)
{
  // columns i in {0,1,sn1-2,sn1-1} with every j, then rows with i in [2, sn1-3]
  const int ncol = 4 * G.sn2;
  BoundCell b;
  if (t < ncol) {
    int col = t / G.sn2;
    b.i = col < 2 ? col : G.sn1 - 4 + col;
    b.j = t % G.sn2;
  } else {
    int u = t - ncol;
    int row = u / (G.sn1 - 4);
    b.i = 2 + u % (G.sn1 - 4);
    // rows: 0,1,sn2-2,sn2-1 then (3D) jstart, jstart+1, jstop-1, jstop
    b.j = row < 2 ? row : row < 4 ? G.sn2 - 4 + row : (row == 4 ? G.jstart : row == 5 ? G.jstart + 1
                                                                       : row == 6 ? G.jstop - 1 : G.jstop);
    (void)nrow;
  }
  return b;
}

// value after the radial copy and (3D) polefix, for any column i, active row j
template <bool THREE_D>
__device__ __forceinline__ void polefixed(const Grid &G, const double *P, int h, int i, int j, double *v)
{
  const int ci = i < G.istart ? G.istart : (i > G.istop ? G.istop : i);
  const long c = cidx(G, h, ci, j);
  int jj = -1, jref = -1;
  if (THREE_D) {
    if (j == G.jstart) { jj = 0; jref = G.jstart + 2; }
    else if (j == G.jstart + 1) { jj = 1; jref = G.jstart + 2; }
    else if (j == G.jstop) { jj = 0; jref = G.jstop - 2; }
    else if (j == G.jstop - 1) { jj = 1; jref = G.jstop - 2; }
  }
  if (jj >= 0) {
    // bound_x2dn/up_polefix (bounds.c:381-436): fields kept, U2 ramped, the rest copied
    const long cr = cidx(G, h, ci, jref);
#pragma unroll
    for (int k = 0; k < 5; k++) {
      double r = P[k * G.nc + cr];
      v[k] = (k == U2) ? (jj + 0.5) / (2 + 0.5) * r : r;
    }
#pragma unroll
    for (int k = 5; k < 8; k++) v[k] = P[k * G.nc + c];
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = P[k * G.nc + c];
  }
}

// 0: edge average, 1: corner average, 2: last resort (fixup.c:491-530)
__device__ __forceinline__ int stencil_kind(const Grid &G, const signed char *pflag, long c)
{
  const long s = G.sn2;
  bool pf2 = pflag[c + 1] != 0, pf4 = pflag[c + s] != 0, pf6 = pflag[c - 1] != 0, pf8 = pflag[c - s] != 0;
  bool pf1 = pflag[c - s + 1] != 0, pf3 = pflag[c + s + 1] != 0, pf5 = pflag[c + s - 1] != 0,
       pf7 = pflag[c - s - 1] != 0;
  if (pf2 && pf4 && pf6 && pf8) return 0;
  if (pf1 && pf3 && pf5 && pf7) return 1;
  return 2;
}

static __device__ void repair_zone(const Grid &G, const double *P, long c, int kind, double *v)
{
  const long s = G.sn2;
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = P[k * G.nc + c];
  if (kind == 0) {
    for (int k = 0; k < B1; k++) {
      const double *X = P + k * G.nc;
      v[k] = 0.25 * (X[c + 1] + X[c - 1] + X[c - s] + X[c + s]);
    }
  } else if (kind == 1) {
    for (int k = 0; k < B1; k++) {
      const double *X = P + k * G.nc;
      v[k] = 0.25 * (X[c + s + 1] + X[c + s - 1] + X[c - s + 1] + X[c - s - 1]);
    }
  } else {
    for (int k = RHO; k <= UU; k++) {
      const double *X = P + k * G.nc;
      v[k] = 0.5 * (0.25 * (X[c + 1] + X[c - 1] + X[c - s] + X[c + s])
                    + 0.25 * (X[c + s + 1] + X[c + s - 1] + X[c - s + 1] + X[c - s - 1]));
    }
    v[U1] = v[U2] = v[U3] = 0.;
  }
}

}  // namespace harm
