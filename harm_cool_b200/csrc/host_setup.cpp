// Host-side grid set-up and initial torus fields for libharm_b200.
//
// The reference computes its geometry once on the host (set_grid,
// main.c:413-520) and the step path only reads it; this file is the
// equivalent host code for callers that do not link the reference's own
// host program.  The connection and the coordinate Jacobian are finite
// differences (metric.c:158-207, 373-426), so the arithmetic below keeps the
// reference's expression order: the same glibc gives the same bits.
#include "host_setup.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace harm {

namespace {

enum { FACE1 = 0, FACE2 = 1, CORN = 2, CENT = 3, FACE3 = 4 };
enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4, B1 = 5, B2 = 6, B3 = 7 };

const double DELTA = 1.e-5;       // metric.c:158
const double SINGSMALL = 1.E-20;  // decs.h:164
const double RHOMIN = 1.e-6, UUMIN = 1.e-8, RHOMINLIMIT = 1.e-20, UUMINLIMIT = 1.e-20;
const double SMALL = 1.e-20;

struct Grid {
  Dims d;
  double dx[4], sx[4];
  double a, R0, hslope;
};

// coord() for one rank (metric.c:62-115)
void coord(const Grid &G, int h, int i, int j, int loc, double *X)
{
  i -= 2;
  j -= 2;
  h -= G.d.n3 > 1 ? 1 : 0;
  const bool phc = G.d.n3 > 2;
  X[0] = 1.;
  if (loc == FACE1) {
    X[1] = G.sx[1] + i * G.dx[1];
    X[2] = G.sx[2] + (j + 0.5) * G.dx[2];
    X[3] = phc ? G.sx[3] + (h + 0.5) * G.dx[3] : G.sx[3] + h * G.dx[3];
  } else if (loc == FACE2) {
    X[1] = G.sx[1] + (i + 0.5) * G.dx[1];
    X[2] = G.sx[2] + j * G.dx[2];
    X[3] = phc ? G.sx[3] + (h + 0.5) * G.dx[3] : G.sx[3] + h * G.dx[3];
  } else if (loc == FACE3) {
    X[1] = G.sx[1] + (i + 0.5) * G.dx[1];
    X[2] = G.sx[2] + (j + 0.5) * G.dx[2];
    X[3] = G.sx[3] + h * G.dx[3];
  } else if (loc == CENT) {
    X[1] = G.sx[1] + (i + 0.5) * G.dx[1];
    X[2] = G.sx[2] + (j + 0.5) * G.dx[2];
    X[3] = phc ? G.sx[3] + (h + 0.5) * G.dx[3] : G.sx[3] + h * G.dx[3];
  } else {
    X[1] = G.sx[1] + i * G.dx[1];
    X[2] = G.sx[2] + j * G.dx[2];
    X[3] = G.sx[3] + h * G.dx[3];
  }
}

// modified Kerr-Schild -> Boyer-Lindquist map with the polar-axis guard
// (coord.c:61-81 with Rbr < 0, coord.c:84-108 with COORDSINGFIX)
void bl_coord_vec(const Grid &G, const double *X, double *V)
{
  V[0] = X[0];
  V[1] = exp(X[1]) + G.R0;
  V[2] = M_PI_2 * (1. + X[2]) + ((1. - G.hslope) / 2.) * sin(M_PI * (1. + X[2]));
  V[3] = X[3];
  if (fabs(V[2]) < SINGSMALL) {
    if (V[2] >= 0) V[2] = SINGSMALL;
    if (V[2] < 0) V[2] = -SINGSMALL;
  }
  if (fabs(M_PI - V[2]) < SINGSMALL) {
    if (V[2] >= M_PI) V[2] = M_PI + SINGSMALL;
    if (V[2] < M_PI) V[2] = M_PI - SINGSMALL;
  }
}

// Jacobian d(r,theta,phi)/d(X) by central differences (metric.c:373-426)
void dxdxp_func(const Grid &G, const double *X, double dxdxp[4][4])
{
  double Xh[4], Xl[4], Vh[4], Vl[4];
  for (int k = 0; k < 4; k++) {
    for (int l = 0; l < 4; l++) Xh[l] = X[l];
    for (int l = 0; l < 4; l++) Xl[l] = X[l];
    Xh[k] += DELTA;
    Xl[k] -= DELTA;
    bl_coord_vec(G, Xh, Vh);
    bl_coord_vec(G, Xl, Vl);
    for (int j = 0; j < 4; j++) dxdxp[j][k] = (Vh[j] - Vl[j]) / (Xh[k] - Xl[k]);
  }
}

// Kerr-Schild metric in the code coordinates (coord.c:128-199)
void gcov_func(const Grid &G, const double *X, double gcovp[4][4])
{
  double gcov[4][4], dxdxp[4][4], V[4];
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) gcov[j][k] = gcovp[j][k] = 0.;
  bl_coord_vec(G, X, V);
  const double r = V[1], th = V[2], a = G.a;
  const double cth = cos(th);
  const double sth = sin(th);
  const double s2 = sth * sth;
  const double rho2 = r * r + a * a * cth * cth;
  dxdxp_func(G, X, dxdxp);
  gcov[0][0] = (-1. + 2. * r / rho2);
  gcov[0][1] = (2. * r / rho2);
  gcov[0][3] = (-2. * a * r * s2 / rho2);
  gcov[1][0] = gcov[0][1];
  gcov[1][1] = (1. + 2. * r / rho2);
  gcov[1][3] = (-a * s2 * (1. + 2. * r / rho2));
  gcov[2][2] = rho2;
  gcov[3][0] = gcov[0][3];
  gcov[3][1] = gcov[1][3];
  gcov[3][3] = s2 * (rho2 + a * a * s2 * (1. + 2. * r / rho2));
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      gcovp[i][j] = 0;
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++) gcovp[i][j] += gcov[k][l] * dxdxp[k][i] * dxdxp[l][j];
    }
}

// Crout LU with implicit partial pivoting (lu.c:114-275)
int lu_decompose(double A[4][4], int permute[4])
{
  const double absmin = 1.e-30;
  double row_norm[4], absmax, maxtemp;
  int max_row = 0;
  const int n = 4;
  for (int i = 0; i < n; i++) {
    absmax = 0.;
    for (int j = 0; j < n; j++) {
      maxtemp = fabs(A[i][j]);
      if (maxtemp > absmax) absmax = maxtemp;
    }
    if (absmax == 0.) return 1;
    row_norm[i] = 1. / absmax;
  }
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < j; i++)
      for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
    absmax = 0.0;
    for (int i = j; i < n; i++) {
      for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
      maxtemp = fabs(A[i][j]) * row_norm[i];
      if (maxtemp >= absmax) {
        absmax = maxtemp;
        max_row = i;
      }
    }
    if (max_row != j) {
      if ((j == (n - 2)) && (A[j][j + 1] == 0.)) {
        max_row = j;
      } else {
        for (int k = 0; k < n; k++) {
          maxtemp = A[j][k];
          A[j][k] = A[max_row][k];
          A[max_row][k] = maxtemp;
        }
        row_norm[max_row] = row_norm[j];
      }
    }
    permute[j] = max_row;
    if (A[j][j] == 0.) A[j][j] = absmin;
    if (j != (n - 1)) {
      maxtemp = 1. / A[j][j];
      for (int i = (j + 1); i < n; i++) A[i][j] *= maxtemp;
    }
  }
  return 0;
}

// forward/backward substitution (lu.c:288-323)
void lu_substitution(const double A[4][4], double B[4], const int permute[4])
{
  const int n = 4;
  for (int i = 0; i < n; i++) {
    double tmpvar = B[permute[i]];
    B[permute[i]] = B[i];
    for (int j = (i - 1); j >= 0; j--) tmpvar -= A[i][j] * B[j];
    B[i] = tmpvar;
  }
  for (int i = (n - 1); i >= 0; i--) {
    for (int j = (i + 1); j < n; j++) B[i] -= A[i][j] * B[j];
    B[i] /= A[i][i];
  }
}

// sqrt|det g| from the LU diagonal (metric.c:118-138)
double gdet_func(const double gcov[4][4])
{
  double tmp[4][4];
  int permute[4];
  std::memcpy(tmp, gcov, sizeof(tmp));
  lu_decompose(tmp, permute);
  double detg = 1.;
  for (int j = 0; j < 4; j++) detg *= tmp[j][j];
  return sqrt(fabs(detg));
}

// inverse by LU, column by column (lu.c:60-90)
int invert_matrix(const double Am[4][4], double Aminv[4][4])
{
  double Amtmp[4][4], dxm[4];
  int permute[4];
  std::memcpy(Amtmp, Am, sizeof(Amtmp));
  if (lu_decompose(Amtmp, permute) != 0) return 1;
  for (int i = 0; i < 4; i++) {
    for (int j = 0; j < 4; j++) dxm[j] = 0.;
    dxm[i] = 1.;
    lu_substitution(Amtmp, dxm, permute);
    for (int j = 0; j < 4; j++) Aminv[j][i] = dxm[j];
  }
  return 0;
}

// connection by central differences of the metric (metric.c:161-207)
void conn_func(const Grid &G, const double *X, const double gcon[4][4], double conn[4][4][4])
{
  double tmp[4][4][4], Xh[4], Xl[4], gh[4][4], gl[4][4];
  for (int k = 0; k < 4; k++) {
    for (int l = 0; l < 4; l++) Xh[l] = X[l];
    for (int l = 0; l < 4; l++) Xl[l] = X[l];
    Xh[k] += DELTA;
    Xl[k] -= DELTA;
    gcov_func(G, Xh, gh);
    gcov_func(G, Xl, gl);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) conn[i][j][k] = (gh[i][j] - gl[i][j]) / (Xh[k] - Xl[k]);
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) tmp[i][j][k] = 0.5 * (conn[j][i][k] + conn[k][i][j] - conn[k][j][i]);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) {
        conn[i][j][k] = 0.;
        for (int l = 0; l < 4; l++) conn[i][j][k] += gcon[i][l] * tmp[l][j][k];
      }
}

bool fill_grid(const harm_grid_spec *g, const double *dx, const double *sx, Grid *G)
{
  if (!g || !valid_grid(g->n1, g->n2, g->n3)) return false;
  G->d = make_dims(g->n1, g->n2, g->n3);
  for (int k = 0; k < 4; k++) {
    G->dx[k] = dx ? dx[k] : 0.;
    G->sx[k] = sx ? sx[k] : 0.;
  }
  G->a = g->a;
  G->R0 = g->R0;
  G->hslope = g->hslope;
  return true;
}

// Boyer-Lindquist metric pieces used to build the torus velocity (metric.c:297-366)
void bl_gcov_func(double a, double r, double th, double gcov[4][4])
{
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 4; k++) gcov[j][k] = 0.;
  double sth = fabs(sin(th));
  double s2 = sth * sth;
  double cth = cos(th);
  double a2 = a * a;
  double r2 = r * r;
  double DD = 1. - 2. / r + a2 / r2;
  double mu = 1. + a2 * cth * cth / r2;
  gcov[0][0] = -(1. - 2. / (r * mu));
  gcov[0][3] = -2. * a * s2 / (r * mu);
  gcov[3][0] = gcov[0][3];
  gcov[1][1] = mu / DD;
  gcov[2][2] = r2 * mu;
  gcov[3][3] = r2 * sth * sth * (1. + a2 / r2 + 2. * a2 * s2 / (r2 * r * mu));
}

// init.c:557-567
double lfish_calc(double a, double r)
{
  return (((pow(a, 2) - 2. * a * sqrt(r) + pow(r, 2))
           * ((-2. * a * r * (pow(a, 2) - 2. * a * sqrt(r) + pow(r, 2))) / sqrt(2. * a * sqrt(r) + (-3. + r) * r)
              + ((a + (-2. + r) * sqrt(r)) * (pow(r, 3) + pow(a, 2) * (2. + r))) / sqrt(1 + (2. * a) / pow(r, 1.5) - 3. / r)))
          / (pow(r, 3) * sqrt(2. * a * sqrt(r) + (-3. + r) * r) * (pow(a, 2) + (-2. + r) * r)));
}

// seeded KISS generator, one draw in [0, 1] (random.c:17-45)
double kiss_uniform(unsigned int z, unsigned int w, unsigned int jsr, unsigned int jcong)
{
  z = 36969u * (z & 65535u) + (z >> 16);
  w = 18000u * (w & 65535u) + (w >> 16);
  unsigned int mwc = (z << 16) + w;
  jsr ^= (jsr << 17);
  jsr ^= (jsr >> 13);
  jsr ^= (jsr << 5);
  jcong = 69069u * jcong + 1234567u;
  unsigned int kiss = (mwc ^ jcong) + jsr;
  double u = ((double)(kiss)) / 0xFFFFFFFF;
  return 0.0 + (1.0 - 0.0) * u;
}

}  // namespace

bool valid_grid(int n1, int n2, int n3)
{
  if (n1 < 4 || n2 < 8 || n3 < 1) return false;
  if (n3 > 1 && (n3 < 4 || n3 % 2)) return false;
  return true;
}

Dims make_dims(int n1, int n2, int n3)
{
  Dims d;
  d.n1 = n1; d.n2 = n2; d.n3 = n3;
  d.sn1 = n1 + 4; d.sn2 = n2 + 4; d.sn3 = n3 > 1 ? n3 + 2 : 1;
  d.istart = 2; d.istop = n1 + 1; d.jstart = 2; d.jstop = n2 + 1;
  d.hstart = n3 > 1 ? 1 : 0; d.hstop = n3 > 1 ? n3 : 0;
  return d;
}

// init.c:161-268 and coord_transform() (init.c:479-555)
void torus_hydro(const harm_grid_spec &gs, const harm_params &prm, const harm_torus_spec &tor,
                 const double *gcovA, const double *gconA, double *p, double *rhomax_out, double *umax_out)
{
  Grid G;
  fill_grid(&gs, prm.dx, prm.startx, &G);
  const Dims &d = G.d;
  const double a = prm.a, gam = prm.gam, rin = tor.rin, kappa = tor.kappa;
  const double l = lfish_calc(a, tor.rmax);
  double rhomax = 0., umax = 0.;
  // Everything but the seeded perturbation of u is independent of phi (the
  // metric is axisymmetric and dx^3/dX^3 is exactly 1), so the fields are
  // evaluated once per (r, theta) and the perturbation per zone.
  const long plane = (long)d.sn1 * d.sn2;
  std::vector<double> ubase(plane, 0.);
  std::vector<char> in_torus(plane, 0);
  {
    const int h = d.hstart;
    for (int i = d.istart; i <= d.istop; i++)
      for (int j = d.jstart; j <= d.jstop; j++) {
        double X[4], V[4];
        coord(G, h, i, j, CENT, X);
        bl_coord_vec(G, X, V);
        const double r = V[1], th = V[2];
        double sth = sin(th);
        double cth = cos(th);
        double DD = r * r - 2. * r + a * a;
        double AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth;
        double SS = r * r + a * a * cth * cth;
        double thin = M_PI / 2.;
        double sthin = sin(thin);
        double cthin = cos(thin);
        double DDin = rin * rin - 2. * rin + a * a;
        double AAin = (rin * rin + a * a) * (rin * rin + a * a) - DDin * a * a * sthin * sthin;
        double SSin = rin * rin + a * a * cthin * cthin;
        double lnh;
        if (r >= rin) {
          lnh = 0.5 * log((1. + sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * sth * AA * sth))) / (SS * DD / AA))
                - 0.5 * sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * AA * sth * sth))
                - 2. * a * r * l / AA
                - (0.5 * log((1. + sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin)))
                             / (SSin * DDin / AAin))
                   - 0.5 * sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin))
                   - 2. * a * rin * l / AAin);
        } else {
          lnh = 1.;
        }
        double *pz = p + (((long)h * d.sn1 + i) * d.sn2 + j) * 8;
        if (lnh < SMALL || r < rin) {
          pz[RHO] = 1.e-7 * RHOMIN;
          pz[UU] = 1.e-7 * UUMIN;
          pz[U1] = 0.;
          pz[U2] = 0.;
          pz[U3] = 0.;
        } else {
          double hm1 = exp(lnh) - 1.;
          double rho = pow(hm1 * (gam - 1.) / (kappa * gam), 1. / (gam - 1.));
          double u = kappa * pow(rho, gam) / (gam - 1.);
          double expm2chi = SS * SS * DD / (AA * AA * sth * sth);
          double up1 = sqrt((-1. + sqrt(1. + 4. * l * l * expm2chi)) / 2.);
          double up = 2. * a * r * sqrt(1. + up1 * up1) / sqrt(AA * SS * DD) + sqrt(SS / AA) * up1 / sth;
          pz[RHO] = rho;
          if (rho > rhomax) rhomax = rho;
          ubase[(long)i * d.sn2 + j] = u;
          in_torus[(long)i * d.sn2 + j] = 1;
          if (u > umax && r >= rin) umax = u;
          // coord_transform(): BL 4-velocity -> KS -> modified KS relative 4-velocity
          double ucon[4], gbl[4][4], trans[4][4], tmp[4];
          ucon[1] = 0.;
          ucon[2] = 0.;
          ucon[3] = up;
          double thb = th;
          if (thb < 0) thb *= -1.;
          if (thb > M_PI) thb = 2. * M_PI - thb;
          bl_gcov_func(a, r, thb, gbl);
          double A_ = gbl[0][0];
          double B_ = 2. * (gbl[0][1] * ucon[1] + gbl[0][2] * ucon[2] + gbl[0][3] * ucon[3]);
          double C_ = 1. + gbl[1][1] * ucon[1] * ucon[1] + gbl[2][2] * ucon[2] * ucon[2]
                      + gbl[3][3] * ucon[3] * ucon[3]
                      + 2. * (gbl[1][2] * ucon[1] * ucon[2] + gbl[1][3] * ucon[1] * ucon[3]
                              + gbl[2][3] * ucon[2] * ucon[3]);
          double discr = B_ * B_ - 4. * A_ * C_;
          ucon[0] = (-B_ - sqrt(discr)) / (2. * A_);
          for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) trans[m][n] = 0.;
          for (int m = 0; m < 4; m++) trans[m][m] = 1.;
          trans[0][1] = 2. * r / (r * r - 2. * r + a * a);
          trans[3][1] = a / (r * r - 2. * r + a * a);
          for (int m = 0; m < 4; m++) tmp[m] = 0.;
          for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) tmp[m] += trans[m][n] * ucon[n];
          for (int m = 0; m < 4; m++) ucon[m] = tmp[m];
          double dxdxp[4][4], dxpdx[4][4], uconp[4];
          X[0] = 1;
          dxdxp_func(G, X, dxdxp);
          invert_matrix(dxdxp, dxpdx);
          for (int m = 0; m < 4; m++) {
            uconp[m] = 0;
            for (int n = 0; n < 4; n++) uconp[m] += dxpdx[m][n] * ucon[n];
          }
          // ucon_to_utcon() with the CENT metric of this zone (phys.c:255-270)
          const double *gc = gconA + (((long)i * d.sn2 + j) * 5 + CENT) * 16;
          (void)gcovA;
          double alpha = 1. / sqrt(-gc[0]);
          double gamma = alpha * uconp[0];
          double utcon[4];
          for (int m = 1; m < 4; m++) {
            double beta = gc[m] * alpha * alpha;
            utcon[m] = uconp[m] + gamma * beta / alpha;
          }
          pz[U1] = utcon[1];
          pz[U2] = utcon[2];
          pz[U3] = utcon[3];
        }
        pz[B1] = 0.;
        pz[B2] = 0.;
        pz[B3] = 0.;
      }
  }
  for (int h = d.hstart; h <= d.hstop; h++) {
    if (h == d.hstart) continue;
    std::memcpy(p + (long)h * plane * 8, p + (long)d.hstart * plane * 8, plane * 8 * sizeof(double));
  }
  for (int h = d.hstart; h <= d.hstop; h++)
    for (int i = d.istart; i <= d.istop; i++)
      for (int j = d.jstart; j <= d.jstop; j++) {
        const long c = (long)i * d.sn2 + j;
        if (!in_torus[c]) continue;
        unsigned int ii = i - 2, jj = j - 2, hh = d.n3 == 1 ? 0 : h - 1;
        unsigned int s = hh * ii * jj + ii * jj + jj;
        p[((long)h * plane + c) * 8 + UU] =
            ubase[c] * (1. + 4.e-2 * (kiss_uniform(12345 + s, 65435 + s, 34221 + s, 43543 + s) - 0.5));
      }
  *rhomax_out = rhomax;
  *umax_out = umax;
}

// init.c:327-368
void torus_field(const Dims &d, const harm_params &prm, const double *gdet, double *p)
{
  const long pl = d.plane();
  double *A = new double[pl];
  for (int h = d.hstart; h <= d.hstop; h++) {
    double *ph = p + (long)h * pl * 8;
    for (long c = 0; c < pl; c++) A[c] = 0.;
    for (int i = d.istart; i <= d.istop + 1; i++)
      for (int j = d.jstart; j <= d.jstop + 1; j++) {
        double rho_av = 0.25 * (ph[((long)i * d.sn2 + j) * 8 + RHO] + ph[((long)(i - 1) * d.sn2 + j) * 8 + RHO]
                                + ph[((long)i * d.sn2 + j - 1) * 8 + RHO]
                                + ph[((long)(i - 1) * d.sn2 + j - 1) * 8 + RHO]);
        double q = rho_av / 1. - 0.2;
        if (q > 0.) A[(long)i * d.sn2 + j] = q;
      }
    for (int i = d.istart; i <= d.istop; i++)
      for (int j = d.jstart; j <= d.jstop; j++) {
        double g = gdet[((long)i * d.sn2 + j) * 5 + CENT];
        const double a00 = A[(long)i * d.sn2 + j], a01 = A[(long)i * d.sn2 + j + 1];
        const double a10 = A[(long)(i + 1) * d.sn2 + j], a11 = A[(long)(i + 1) * d.sn2 + j + 1];
        double *pz = ph + ((long)i * d.sn2 + j) * 8;
        pz[B1] = -(a00 - a01 + a10 - a11) / (2. * prm.dx[2] * g);
        pz[B2] = (a00 + a01 - a10 - a11) / (2. * prm.dx[1] * g);
        pz[B3] = 0.;
      }
  }
  delete[] A;
}

void radial_floors(const double *coords, double gam, long n, double *out)
{
  for (long c = 0; c < n; c++) {
    const double r = coords[c * 4 + 1];
    double rhoscal = pow(r, -2.0);
    double uuscal = pow(rhoscal, gam);
    double rhoflr = RHOMIN * rhoscal;
    double uuflr = UUMIN * uuscal;
    if (rhoflr < RHOMINLIMIT) rhoflr = RHOMINLIMIT;
    if (uuflr < UUMINLIMIT) uuflr = UUMINLIMIT;
    out[c] = rhoflr;
    out[n + c] = uuflr;
  }
}

}  // namespace harm

// ---------------------------------------------------------------------------
// C ABI

using namespace harm;

extern "C" int harm_set_points(const harm_grid_spec *g, double dx[4], double startx[4])
{
  if (!g || !dx || !startx || !valid_grid(g->n1, g->n2, g->n3) || !(g->Rin > g->R0) || !(g->Rout > g->Rin))
    return HARM_E_ARG;
  const double x1max = log(g->Rout - g->R0);
  startx[0] = 0.;
  startx[1] = log(g->Rin - g->R0);
  startx[2] = -1.;
  startx[3] = 0.;
  dx[0] = 0.;
  dx[1] = (x1max - startx[1]) / g->n1;
  dx[2] = 2. / g->n2;
  dx[3] = 2. * M_PI / g->n3;
  return HARM_OK;
}

extern "C" int harm_set_grid(const harm_grid_spec *g, const double dx[4], const double startx[4],
                             double *gcov, double *gcon, double *gdet, double *conn, double *coords)
{
  Grid G;
  if (!fill_grid(g, dx, startx, &G) || !gcov || !gcon || !gdet || !conn || !coords) return HARM_E_ARG;
  const Dims &d = G.d;
  const int h = d.n3 > 1 ? 1 : 0;
  for (int i = 0; i < d.sn1; ++i)
    for (int j = 0; j < d.sn2; ++j) {
      const long c = (long)i * d.sn2 + j;
      double X[4], V[4];
      static const int order[5] = {CENT, CORN, FACE1, FACE2, FACE3};
      for (int o = 0; o < 5; o++) {
        const int loc = order[o];
        double(*gv)[4] = (double(*)[4])(gcov + (c * 5 + loc) * 16);
        double(*gn)[4] = (double(*)[4])(gcon + (c * 5 + loc) * 16);
        coord(G, h, i, j, loc, X);
        gcov_func(G, X, gv);
        gdet[c * 5 + loc] = gdet_func(gv);
        invert_matrix(gv, gn);
        if (loc == CENT) {
          conn_func(G, X, gn, (double(*)[4][4])(conn + c * 64));
          bl_coord_vec(G, X, V);
          for (int k = 0; k < 4; k++) coords[c * 4 + k] = V[k];
        }
      }
    }
  return HARM_OK;
}

extern "C" int harm_set_katm(const harm_grid_spec *g, double gam, const double *coords, double *katm)
{
  if (!g || !coords || !katm || !valid_grid(g->n1, g->n2, g->n3)) return HARM_E_ARG;
  const Dims d = make_dims(g->n1, g->n2, g->n3);
  // fixup1zone() on rho = u = -1, v = B = 0 at theta index 0 reduces to the
  // radial floor (fixup.c:117-187), and Katm = (gam-1) u_floor / rho_floor^gam
  for (int i = 0; i < d.sn1; i++) katm[i] = 0.;
  for (int i = d.istart; i <= d.istop; i++) {
    const double r = coords[((long)i * d.sn2 + 0) * 4 + 1];
    double rhoscal = pow(r, -2.0);
    double uuscal = pow(rhoscal, gam);
    double rhoflr = RHOMIN * rhoscal;
    double uuflr = UUMIN * uuscal;
    if (rhoflr < RHOMINLIMIT) rhoflr = RHOMINLIMIT;
    if (uuflr < UUMINLIMIT) uuflr = UUMINLIMIT;
    katm[i] = (gam - 1.) * uuflr / pow(rhoflr, gam);
  }
  return HARM_OK;
}
