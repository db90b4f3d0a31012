// The equation of state and neutrino rates behind HARM-COOL's COOL_EOS
// tables: nucleons, electron-positron pairs, helium, radiation and trapped
// neutrinos in beta equilibrium, at a given baryon density, temperature and
// disc scale-height factor.  A restatement of the reference's Fortran table
// generator, abundance() (abundance.f90:6-243), and of the routines it
// calls, written once for the host and the device:
//
//   abundance.f90:6-243       abundance()        node values e, p, Qnu, tau, n_e-, n_e+
//   chem_eq.f90:49-191        chem_eq, eqnucl, nuclear, funcnb, neutrino
//   chem_eq.f90:193-431       the rate integrands func1k .. func3r
//   chem_eq.f90:433-490       rtbis_funcnb (Newton on funcnb)
//   number_den.f90:26-397     fxnn, fxnp, neta, peta, eeta, lepton
//   eos.f90:32-183            eos_npe, eos_rad, eos_neu, eos_he
//   accretion.f90:24-117      xnuc, h_dep, opt_dep, b_neu
//   neu_rate.f90:30-261       pair, urca, func1 .. func3, brem, plasmon
//   gauss_integral.f90:26-219 the 40-point Gauss-Legendre and 20-point
//                             Gauss-Laguerre rules of the rate integrals
//   gauss_integral.f90:241-438 dfermi and its integrands
//   mnewtf.f90:94-150         mnewt, for one unknown
//
// Units are the reference's: densities in fm^-3, energies and temperatures
// in MeV, until abundance() converts e and p to erg cm^-3.
//
// Code size.  Each Newton solver and each rate routine is kept out of line
// (HNU_NOINLINE) and exists once in the kernel, the Fermi integrals have one
// copy of their term code per number of indices, whatever the number of sets
// a call asks for, and a lane's loop over its quadrature terms stays rolled:
// inlined at every call site and unrolled, the kernel outgrew the instruction
// cache and its warps waited on instruction fetch more than on anything else.
//
// One node, one warp.  A node is a nest of Newton solves whose every trial
// evaluates Fermi integrals or rate integrals by Gauss quadrature.  All 32
// lanes of a warp run the node's scalar code together, with the same values,
// and split each quadrature's terms between them (lane_sum): lane l adds
// terms l, l + 32, ... and a butterfly over the lanes combines the partial
// sums, so that every lane holds the same sum and the control flow stays
// uniform.  The quadratures a Newton trial needs at x, x + dx and x - dx, or
// that a routine needs for several species, go into one such sum.  The host
// build runs the 32 lanes one after another and the same butterfly, so both
// builds add the terms in the same order.
//
// Fidelity.  The reference is gfortran code; no Fortran compiler exists
// here, so this restatement is not compared with its output.  It keeps the
// reference's formulae, their order of operations and its constants, and
// three properties of the Fortran that move results at the 1e-8 level:
//  - literals written without a kind (3.1415926535897932, 197.3269718e0,
//    5.6e-5, 0.557, 13.8, 2.0/3.0, 1./3.) are single precision in Fortran;
//    they appear here as float literals (HNU_F);
//  - arguments pass by reference: h_dep() scales its caller's p and e, and
//    opt_dep() zeroes its caller's b1 before b_neu() sets it again;
//  - mnewt() with one unknown: a zero or NaN derivative skips the solve and
//    steps by the residual itself (ludcmp's singular branch).
// What differs in the last bits only: integer powers are products and
// x**1.5-style powers are pow(); the Fermi kernels take x^k as
// x^(k-1/2) sqrt(x) and fold each interval's half-length into the weights;
// quadrature terms are summed in the lane order above rather than node by
// node; and the emissivities of the trapping iteration are evaluated once
// (they do not depend on its unknowns).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define HNU __host__ __device__ __forceinline__
#define HNU_NOINLINE static __host__ __device__ __noinline__
#else
#define HNU inline
#define HNU_NOINLINE static
#endif

// a Fortran default-real literal, as the real(8) value it converts to
#define HNU_F(x) ((double)(x##f))

namespace harm {
namespace nu {

// const_mod.f90
constexpr double PI = HNU_F(3.1415926535897932);
constexpr double HC = HNU_F(197.3269718);  // MeV fm
constexpr double SIGMASB = HNU_F(5.6e-5);
constexpr double XME = 0.510998910, XMP = 938.272013, XMN = 939.56536;  // MeV

// Quadrature rules.  Abscissae and weights are computed on the host by
// harm_nu_rules() (harm_nu_host.cpp) from the definitions of the rules; the
// Gauss-Laguerre weights carry the factor e^x, as the integrands include the
// weight function.
struct Rules {
  double l20x[10], l20w[10];  // 20-point Gauss-Legendre on (-1, 1): positive abscissae
  double l40x[20], l40w[20];  // 40-point Gauss-Legendre on (-1, 1): positive abscissae
  double g20x[20], g20w[20];  // 20-point Gauss-Laguerre on (0, inf)
};

HNU double sq(double x) { return x * x; }
HNU double cube(double x) { return x * x * x; }

// ---------------------------------------------------------------------------
// Sums over the lanes of a warp
// ---------------------------------------------------------------------------

// Combine the lanes' partial sums: out[a] = the sum over lanes of part[a].  The
// butterfly adds, on lanes l and l ^ d, the same two partial sums, so all lanes
// end equal.  On the host, part holds the 32 lanes' partials, [32][NA].
template <int NA>
HNU void lane_reduce(double *part, double *out)
{
#if defined(__CUDA_ARCH__)
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
#pragma unroll
    for (int a = 0; a < NA; a++) part[a] += __shfl_xor_sync(0xffffffffu, part[a], d);
#pragma unroll
  for (int a = 0; a < NA; a++) out[a] = part[a];
#else
  // lane 0's butterfly: at distance d it adds lane d's partial, which holds the
  // same sums over lanes d .. 2d-1 that lanes 0 .. d-1 hold over 0 .. d-1
  for (int d = 16; d > 0; d >>= 1)
    for (int l = 0; l < d; l++)
      for (int a = 0; a < NA; a++) part[l * NA + a] = part[l * NA + a] + part[(l + d) * NA + a];
  for (int a = 0; a < NA; a++) out[a] = part[a];
#endif
}

// out[a] = sum over terms e < NTERM of what term(e, acc) adds to acc[a], for
// NA accumulators: lane l takes terms l, l + 32, ... in that order.  The
// loop over a lane's terms stays rolled: one copy of the term's code.
template <int NA, int NTERM, class Term>
HNU void lane_sum(const Term &term, double *out)
{
#if defined(__CUDA_ARCH__)
  const int l = threadIdx.x & 31;
  double part[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) part[a] = 0.0;
#pragma unroll 1
  for (int e = l; e < NTERM; e += 32) term(e, part);
  lane_reduce<NA>(part, out);
#else
  double part[32 * NA];
  for (int l = 0; l < 32; l++) {
    for (int a = 0; a < NA; a++) part[l * NA + a] = 0.0;
    for (int e = l; e < NTERM; e += 32) term(e, part + l * NA);
  }
  lane_reduce<NA>(part, out);
#endif
}

// ---------------------------------------------------------------------------
// Generalised Fermi-Dirac integrals
//   F_k(eta, theta) = int_0^inf x^k sqrt(1 + theta x / 2) / (e^(x - eta) + 1) dx
// for k = 1/2, 3/2, 5/2, 7/2, by Aparicio's four-interval quadrature (ApJS 117,
// 627, 1998) as in dfermi (gauss_integral.f90:241-349): 20-point
// Gauss-Legendre on [0, sqrt(s1)] in z = sqrt(x), on [s1, s2] and [s2, s3], and
// 20-point Gauss-Laguerre on [s3, inf), with breakpoints that follow eta.
// ---------------------------------------------------------------------------

// the intervals of one (eta, theta): centres and half-lengths of the three
// Gauss-Legendre pieces (the first in z) and the start of the tail
struct FdSpan {
  double eta, theta, c[3], h[3], s3;
};

HNU FdSpan fd_span(double eta, double theta)
{
  // breakpoint fit of Aparicio (1998)
  const double d = 3.3609, sg = 9.1186e-2;
  const double a1 = 6.7774, b1 = 1.1418, c1 = 2.9826;
  const double a2 = 3.7601, b2 = 9.3719e-2, c2 = 2.1063e-2, d2 = 3.1084e1, e2 = 1.0056;
  const double a3 = 7.5669, b3 = 1.1695, c3 = 7.5416e-1, d3 = 6.6558, e3 = -1.2819e-1;
  const double eta1 = sg * (eta - d);
  const double xi = (eta1 <= 5.0e1) ? log(1.0 + exp(eta1)) / sg : eta - d;
  const double xi2 = xi * xi;
  const double x1 = (a1 + b1 * xi + c1 * xi2) / (1.0 + c1 * xi);
  const double x2 = (a2 + b2 * xi + c2 * d2 * xi2) / (1.0 + e2 * xi + c2 * xi2);
  const double x3 = (a3 + b3 * xi + c3 * d3 * xi2) / (1.0 + e3 * xi + c3 * xi2);
  const double s1 = x1 - x2, s2 = x1, s3 = x1 + x3, s12 = sqrt(s1);
  FdSpan s;
  s.eta = eta;
  s.theta = theta;
  s.c[0] = 0.5 * s12;
  s.h[0] = 0.5 * s12;
  s.c[1] = 0.5 * (s1 + s2);
  s.h[1] = 0.5 * (s2 - s1);
  s.c[2] = 0.5 * (s2 + s3);
  s.h[2] = 0.5 * (s3 - s2);
  s.s3 = s3;
  return s;
}

// The 80 terms of one Fermi integral set of NK indices: terms r / 20 = 0, 1,
// 2 are the Gauss-Legendre intervals, node (r % 20) / 2 on the side
// (r % 20) & 1; piece 3 is the Gauss-Laguerre node r % 20.  The integrands
// are fdfunc1 and, in z = sqrt(x), fdfunc2 (gauss_integral.f90:354-438), with
// the overflow guard at x - eta = 100.
template <int NK>
struct FdTerms {
  const Rules &R;
  const FdSpan &S;
  HNU void operator()(int r, double *a) const
  {
    const int piece = r / 20, q = r % 20;
    double x, w;
    if (piece < 3) {
      const int j = q >> 1;
      const double c = piece == 0 ? S.c[0] : (piece == 1 ? S.c[1] : S.c[2]);
      const double h = piece == 0 ? S.h[0] : (piece == 1 ? S.h[1] : S.h[2]);
      x = c + ((q & 1) ? -h : h) * R.l20x[j];
      w = R.l20w[j] * h;
    } else {
      x = S.s3 + R.g20x[q];
      w = R.g20w[q];
    }
    if (piece == 0) {  // z = x here: 2 z^(2k+1) sqrt(1 + theta z^2 / 2) / (e^(z^2 - eta) + 1)
      const double zsq = x * x;
      const double dxst = sqrt(1.0 + 0.5 * zsq * S.theta);
      const double g = (zsq - S.eta < 1.0e2) ? dxst / (exp(zsq - S.eta) + 1.0) : dxst * exp(S.eta - zsq);
      double zk = zsq;
#pragma unroll
      for (int k = 0; k < NK; k++) {
        a[k] += 2.0 * zk * g * w;
        zk *= zsq;
      }
    } else {
      const double dxst = sqrt(1.0 + 0.5 * x * S.theta);
      const double g = (x - S.eta < 1.0e2) ? dxst / (exp(x - S.eta) + 1.0) : dxst * exp(S.eta - x);
      double xk = sqrt(x);
#pragma unroll
      for (int k = 0; k < NK; k++) {
        a[k] += xk * g * w;
        xk *= x;
      }
    }
  }
};

// F[m NK + k] = F_{k+1/2}(eta[m], theta[m]) for m < M <= 32.  On the device
// lane m works out the intervals of set m and hands them to the other lanes:
// the same function of the same arguments, so the same bits, for a fraction
// of the instructions.  The sets go one after another through one copy of the
// term code; lane l adds terms l, l + 32, l + 64 of each set into that set's
// partials, which the butterfly then combines.
template <int NK>
HNU_NOINLINE void fermi_sets(const Rules &R, int M, const double *eta, const double *theta, double *F)
{
#if defined(__CUDA_ARCH__)
  const int l = threadIdx.x & 31;
  double e = eta[0], th = theta[0];
#pragma unroll 1
  for (int q = 1; q < M; q++)
    if (l == q) {
      e = eta[q];
      th = theta[q];
    }
  const FdSpan mine = fd_span(e, th);
#pragma unroll 1
  for (int m = 0; m < M; m++) {
    FdSpan S;
    S.eta = __shfl_sync(0xffffffffu, mine.eta, m);
    S.theta = __shfl_sync(0xffffffffu, mine.theta, m);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      S.c[q] = __shfl_sync(0xffffffffu, mine.c[q], m);
      S.h[q] = __shfl_sync(0xffffffffu, mine.h[q], m);
    }
    S.s3 = __shfl_sync(0xffffffffu, mine.s3, m);
    double part[NK];
#pragma unroll
    for (int a = 0; a < NK; a++) part[a] = 0.0;
    const FdTerms<NK> t{R, S};
#pragma unroll 1
    for (int r = l; r < 80; r += 32) t(r, part);
    lane_reduce<NK>(part, F + m * NK);
  }
#else
  for (int m = 0; m < M; m++) {
    const FdSpan S = fd_span(eta[m], theta[m]);
    const FdTerms<NK> t{R, S};
    double part[32 * NK];
    for (int l = 0; l < 32; l++) {
      for (int a = 0; a < NK; a++) part[l * NK + a] = 0.0;
      for (int r = l; r < 80; r += 32) t(r, part + l * NK);
    }
    lane_reduce<NK>(part, F + m * NK);
  }
#endif
}

template <int M, int NK>
HNU void fermi(const Rules &R, const double *eta, const double *theta, double *F)
{
  static_assert(M <= 32, "one lane per set");
  fermi_sets<NK>(R, M, eta, theta, F);
}

// ---------------------------------------------------------------------------
// Number densities (number_den.f90)
// ---------------------------------------------------------------------------

// c in n = c (F_1/2 + beta F_3/2) for fermions of mass m (MeV) and
// beta = kt / m: sqrt2/pi^2 (m/hc)^3 beta^1.5 (eq. 20; fxnn, fxnp, lepton)
HNU double density_coef(double m, double beta) { return sqrt(2.0) / sq(PI) * cube(m / HC) * pow(beta, 1.5); }

// the density of nucleons with beta = kt / m and coefficient c at
// degeneracies eta[0..2] (fxnn, fxnp)
HNU void fermion_density3(const Rules &R, double beta, double c, const double *eta, double *n)
{
  const double th[3] = {beta, beta, beta};
  double F[3 * 2];
  fermi<3, 2>(R, eta, th, F);
  for (int i = 0; i < 3; i++) n[i] = c * (F[2 * i] + beta * F[2 * i + 1]);
}

// electrons and positrons at electron degeneracies etae[0..N), beta = kt / m_e
// and density coefficient c (lepton, number_den.f90:374-395): nl = n_e- - n_e+,
// and the two densities
template <int N>
HNU void lepton_bc(const Rules &R, double beta, double c, const double *etae, double *nl, double *nee,
                   double *nep)
{
  double eta[2 * N], th[2 * N];
  for (int i = 0; i < N; i++) {
    eta[2 * i] = etae[i];
    eta[2 * i + 1] = -etae[i] - 2.0 / beta;
    th[2 * i] = th[2 * i + 1] = beta;
  }
  double F[2 * N * 2];
  fermi<2 * N, 2>(R, eta, th, F);
  for (int i = 0; i < N; i++) {
    const double ne = c * (F[4 * i] + beta * F[4 * i + 1]);
    const double np = c * (F[4 * i + 2] + beta * F[4 * i + 3]);
    if (nee) nee[i] = ne;
    if (nep) nep[i] = np;
    nl[i] = ne - np;
  }
}

template <int N>
HNU void lepton(const Rules &R, double kt, const double *etae, double *nl, double *nee, double *nep)
{
  const double beta = kt / XME;
  lepton_bc<N>(R, beta, density_coef(XME, beta), etae, nl, nee, nep);
}

// mnewt (mnewtf.f90:108-150) with one unknown and the central-difference
// Jacobian of the usrfun_* routines: solve G(x) = target from x, up to 200
// trials, stopping when |G(x) - target| <= tolf or the step is <= 1e-20.
// g(xs, ys) evaluates G at x, x + xacc and x - xacc together.
template <class G3>
HNU double newton1(const G3 &g, double x, double target, double tolf)
{
  for (int k = 0; k < 200; k++) {
    double xacc = fabs(x) * 1.0e-8;
    if (xacc < 1.0e-50) xacc = 1.0e-50;
    const double xs[3] = {x, x + xacc, x - xacc};
    double ys[3];
    g(xs, ys);
    const double f = target - ys[0];
    const double fp = target - ys[1];
    const double fm = target - ys[2];
    const double fjac = (fp - fm) / (2.0 * xacc);
    double dx = -f;
    if (fabs(dx) <= tolf) return x;
    if (fabs(fjac) > 0.) dx = dx / fjac;  // else ludcmp finds it singular: the step is the residual
    const double xn = x + dx;
    if (fabs(dx) <= 1.0e-20) return xn;
    // x is the whole state of the iteration: once a step leaves it unchanged,
    // every later trial repeats that step, and the 200th returns this x
    if (xn == x && signbit(xn) == signbit(x)) return x;
    x = xn;
  }
  return x;
}

HNU double newton_tol(double n)
{
  const double tol = 1.0e-8 * n;
  return tol < 1.0e-50 ? 1.0e-50 : tol;
}

// the densities a Newton solve evaluates, with beta and the density
// coefficient (a pow()) worked out once per solve
struct FermionN3 {
  const Rules &R;
  double beta, c;
  HNU FermionN3(const Rules &r, double m, double kt) : R(r), beta(kt / m), c(density_coef(m, kt / m)) {}
  HNU void operator()(const double *x, double *y) const { fermion_density3(R, beta, c, x, y); }
};
struct LeptonN3 {
  const Rules &R;
  double beta, c;
  HNU LeptonN3(const Rules &r, double kt) : R(r), beta(kt / XME), c(density_coef(XME, kt / XME)) {}
  HNU void operator()(const double *x, double *y) const { lepton_bc<3>(R, beta, c, x, y, nullptr, nullptr); }
};

// degeneracy of neutrons and protons of density n (neta, peta): Newton from -10
HNU_NOINLINE double neta(const Rules &R, double kt, double n)
{
  return newton1(FermionN3(R, XMN, kt), -10.0, n, newton_tol(n));
}
HNU_NOINLINE double peta(const Rules &R, double kt, double n)
{
  return newton1(FermionN3(R, XMP, kt), -10.0, n, newton_tol(n));
}

// electron degeneracy for the net lepton density n (eeta): Newton from m_e/kt,
// capped at 0
HNU_NOINLINE double eeta(const Rules &R, double kt, double n)
{
  const double e = newton1(LeptonN3(R, kt), 0.510998910 / kt, n, newton_tol(n));
  return e > 0.0 ? 0.0 : e;
}

// ---------------------------------------------------------------------------
// Equations of state (eos.f90), e and p in MeV fm^-3
// ---------------------------------------------------------------------------

// nucleons and pairs (eos_npe, eos.f90:32-112): for each fermion species
// p = cp (F_3/2 + beta/2 F_5/2), e = 3/2 cp (F_3/2 + beta F_5/2),
// cp = 2/3 sqrt2/pi^2 (m/hc)^3 m beta^2.5; the positrons count only where the
// electron density is positive
HNU_NOINLINE void eos_npe(const Rules &R, double kt, double etan, double etap, double etae, double nee, double *e,
                 double *p)
{
  const double mass[4] = {XME, XME, XMP, XMN};
  const double eta[4] = {etae, -etae - 2.0 / (kt / XME), etap, etan};
  double th[4];
  for (int s = 0; s < 4; s++) th[s] = kt / mass[s];
  double F[4 * 3];
  fermi<4, 3>(R, eta, th, F);  // F_1/2 is computed and unused
  double ps[4], es[4];
  for (int s = 0; s < 4; s++) {
    const double m = mass[s], beta = th[s];
    const double cp = (double)(2.0f / 3.0f) * sqrt(2.0) / sq(PI) * cube(m / HC) * m * pow(beta, 2.5);
    const double ce = 3.0 / 2.0 * cp;
    ps[s] = cp * (F[3 * s + 1] + 0.5 * beta * F[3 * s + 2]);
    es[s] = ce * (F[3 * s + 1] + beta * F[3 * s + 2]);
  }
  if (nee <= 0.0) ps[1] = es[1] = 0.0;
  *p = ps[0] + ps[1] + ps[2] + ps[3];
  *e = es[0] + es[1] + es[2] + es[3];
}

// black-body radiation (eos_rad) and trapped neutrinos with blocking b1, b2 (eos_neu)
HNU double p_rad(double kt) { return PI * PI / 15.0 * kt * cube(kt / HC) / 3.0; }
HNU double p_neu(double kt, double b1, double b2)
{
  return 7.0 / 8.0 * (b1 + b2) * PI * PI / 15.0 * kt * cube(kt / HC) / 3.0;
}

// helium nuclei as an ideal gas, dropped where the Sackur-Tetrode entropy is
// not positive (eos_he)
HNU void eos_he(double kt, double nhe, double *e, double *p)
{
  *e = *p = 0.0;
  if (nhe <= 0.0) return;
  const double mhe = 3755.6740;
  const double s = nhe * (2.5 + 1.5 * log(mhe * kt / sq(HC) / 2.0 / PI) - log(nhe));
  if (s <= 0.0) return;
  *e = 1.5 * nhe * kt;
  *p = nhe * kt;
}

// ---------------------------------------------------------------------------
// The disc (accretion.f90)
// ---------------------------------------------------------------------------

// mass fraction of free nucleons (Popham et al. 1999) (xnuc)
HNU double xnuc(double nb, double kt)
{
  const double rho10 = nb * 1.66e5;
  const double t11 = kt * 1.16059e-1;
  double x = 295.5 / pow(rho10, 0.75) * pow(t11, 1.125) * exp(-0.8209 / t11);
  if (x > 1.0) x = 1.0;
  if (x < 0.0) x = 0.0;
  return x;
}

// scale height HdFac * c_s (h_dep); p and e come back in erg cm^-3, as the
// Fortran routine rescales its caller's arguments
HNU double h_dep(double hdfac, double nb, double &p, double &e)
{
  const double CC = 2.99792458e10;
  const double rho = nb * 1.66e15;
  p = p * 1.6021772e33;
  e = e * 1.6021772e33;
  double cs = CC * sqrt(p / (rho * CC * CC + e));
  if (cs > CC) cs = CC;
  return hdfac * cs;
}

// ---------------------------------------------------------------------------
// Neutrino emissivities, erg cm^-3 s^-1 (neu_rate.f90)
// ---------------------------------------------------------------------------

// e+ e- annihilation into electron and into mu (= tau) neutrinos (pair)
HNU void pair(const Rules &R, double kt, double etae, double *ev1, double *ev2)
{
  const double QC = 1.023e23;
  const double beta = kt / 0.510998910;
  double cv = 2.0 * 0.23 + 0.5, ca = 0.5;
  const double cv1e = cv * cv + ca * ca, cv2e = cv * cv - ca * ca;
  cv = 2.0 * 0.23 - 0.5;
  ca = -0.5;
  const double cv1m = cv * cv + ca * ca, cv2m = cv * cv - ca * ca;
  const double eta[2] = {etae, -etae - 2.0 / beta}, th[2] = {beta, beta};
  double F[2 * 4];
  fermi<2, 4>(R, eta, th, F);
  const double *G = F;
  const double u_1 = G[0], u0 = G[0] + beta * G[1], u1 = G[0] + 2.0 * beta * G[1] + beta * beta * G[2];
  const double u2 = G[0] + 3.0 * beta * G[1] + 3.0 * beta * beta * G[2] + cube(beta) * G[3];
  G = F + 4;
  const double f_1 = G[0], f0 = G[0] + beta * G[1], f1 = G[0] + 2.0 * beta * G[1] + beta * beta * G[2];
  const double f2 = G[0] + 3.0 * beta * G[1] + 3.0 * beta * beta * G[2] + cube(beta) * G[3];
  const double a = 8.0 * (f1 * u2 + f2 * u1) - 2.0 * (f_1 * u2 + f2 * u_1) + 7.0 * (f0 * u1 + f1 * u0) +
                   5.0 * (f0 * u_1 + f_1 * u0);
  const double b = f0 * (u1 + u_1) + (f_1 + f1) * u0;
  const double pre = QC / (36.0 * PI) * (2.0 / (sq(PI) * sq(PI))) * cube(beta);
  *ev1 = pre * (cv1e * a + 9.0 * cv2e * b);
  *ev2 = pre * (cv1m * a + 9.0 * cv2m * b);
}

// The weak-rate integrands: x sqrt(x^2 - 1/beta^2) (q -+ x)^POW times an
// electron or positron occupation and a neutrino blocking factor, over the
// electron energy x in units of kt.  K selects the reaction: 1 n -> p e nu~
// on [1/beta, q]; 2 p e- -> n nu and 3 n e+ -> p nu~ on [x0, inf).  KIND 0:
// the |1 - b1 f| blocking (func1..3, func1k..3k); 1: |b1 f| absorption
// (func1r..3r).
template <int K, int KIND, int POW>
HNU double rate(double x, double kt, double eta, double b1)
{
  const double beta = kt / XME;
  const double q = (XMN - XMP) / kt;
  double xe, en;
  if (K == 1) {
    xe = KIND == 0 ? eta - (x - 1.0 / beta) : (x - 1.0 / beta) - eta;
    en = q - x;
  } else if (K == 2) {
    xe = KIND == 0 ? -eta + (x - 1.0 / beta) : +eta - (x - 1.0 / beta);
    en = x - q;
  } else {
    xe = KIND == 0 ? -eta + (x - 1.0 / beta) : eta - (x - 1.0 / beta);
    en = x + q;
  }
  const double f1 = 1.0 / (exp(xe) + 1.0);
  const double ex = K == 1 ? exp(q - x) : (K == 2 ? exp(x - q) : exp(x + q));
  const double f2 = KIND == 0 ? fabs(1.0 - b1 / (ex + 1.0)) : fabs(b1 / (ex + 1.0));
  const double enp = POW == 3 ? en * en * en : en * en;
  return x * sqrt(x * x - 1.0 / (beta * beta)) * enp * f1 * f2;
}

// The rate integrals of one routine as 80 terms: 0..39 the 40-point
// Gauss-Legendre rule on [a, b] = [m_e, m_n - m_p] / kt for reaction 1
// (gauss_legendre, gauss_integral.f90:118-219: node e / 2 on the side e & 1,
// centre c and half-length h), 40..59 the 20-point Gauss-Laguerre rule from
// (m_n - m_p) / kt for reaction 2 and 60..79 from m_e / kt for reaction 3
// (gauss_laguerre, gauss_integral.f90:26-113, scale 1).  RK: also the
// absorption integrands of neutrino() (chem_eq.f90), into accumulators 3..5.
// The Legendre sums still take the half-length factor.
template <int POW, bool RK>
struct RateTerms {
  const Rules &R;
  double kt, etae, etaep, b1, c, h;
  HNU void operator()(int e, double *acc) const
  {
    if (e < 40) {
      const int j = e >> 1;
      const double x = c + ((e & 1) ? -h : h) * R.l40x[j];
      acc[0] += rate<1, 0, POW>(x, kt, etae, b1) * R.l40w[j];
      if (RK) acc[3] += rate<1, 1, POW>(x, kt, etae, b1) * R.l40w[j];
    } else if (e < 60) {
      const int j = e - 40;
      const double x = (XMN - XMP) / kt + 1.0 * R.g20x[j];
      acc[1] += rate<2, 0, POW>(x, kt, etae, b1) * R.g20w[j];
      if (RK) acc[4] += rate<2, 1, POW>(x, kt, etae, b1) * R.g20w[j];
    } else {
      const int j = e - 60;
      const double x = XME / kt + 1.0 * R.g20x[j];
      acc[2] += rate<3, 0, POW>(x, kt, etaep, b1) * R.g20w[j];
      if (RK) acc[5] += rate<3, 1, POW>(x, kt, etaep, b1) * R.g20w[j];
    }
  }
};

// URCA emissivities without blocking (urca, neu_rate.f90:110-160):
// n -> p e nu~ (evn), p e- -> n nu (evep), n e+ -> p nu~ (even)
HNU void urca(const Rules &R, double kt, double nn, double np, double etae, double etaep, double *evep,
              double *even, double *evn)
{
  const double t11 = kt * 1.16059e-1;
  const double t6 = cube(t11) * cube(t11);
  const double a = XME / kt, b = (XMN - XMP) / kt, h = 0.5 * (b - a);
  double I[3];
  lane_sum<3, 80>(RateTerms<3, false>{R, kt, etae, etaep, 0.0, 0.5 * (a + b), h}, I);
  *evn = 1.14473926e37 * t6 * nn * (I[0] * h);
  *evep = 1.14473926e37 * t6 * np * (I[1] * 1.0);
  *even = 1.14473926e37 * t6 * nn * (I[2] * 1.0);
}

// nucleon-nucleon bremsstrahlung (brem) and plasmon decay (plasmon)
HNU double brem(double nb, double kt)
{
  const double rho10 = nb * 1.66e5, t11 = kt * 1.16059e-1;
  return 3.35e27 * (rho10 * rho10) * pow(t11, 5.5);
}
HNU double plasmon(double kt, double etae)
{
  const double t11 = kt * 1.16059e-1;
  const double eta = etae + 0.510998910 / kt;
  const double gp = 5.565e-2 * sqrt((sq(PI) + 3.0 * sq(eta)) / 3.0);
  const double t9 = sq(sq(t11)) * sq(sq(t11)) * t11;
  return 1.5e32 * t9 * (cube(gp) * cube(gp)) * exp(-gp) * (1.0 + gp) * (2.0 + sq(gp) / (1.0 + gp));
}

// Emissivities of electron neutrinos (qe) and of one heavy-lepton flavour
// (qo), erg cm^-3 s^-1, as opt_dep sums them (accretion.f90:65-84): pairs,
// URCA without blocking, bremsstrahlung and plasmons.  None depends on the
// scale height or the blocking factors, so the ten trapping iterations of
// abundance() and funcnb(), which the reference runs through opt_dep() with
// the same arguments each time, take them from one evaluation.
struct Emission {
  double qe, qo;
};

HNU_NOINLINE Emission emission(const Rules &R, double kt, double nnucl, double nn, double np, double etae,
                                double etaep)
{
  double ev1, ev2, evep, even, evn;
  pair(R, kt, etae, &ev1, &ev2);
  urca(R, kt, nn, np, etae, etaep, &evep, &even, &evn);
  const double evbrem = brem(nnucl, kt);
  const double evpl = plasmon(kt, etae);
  return {ev1 + evep + even + evn + evbrem / 3.0 + evpl, ev2 + evbrem / 3.0};
}

// absorption and scattering optical depths over the scale height hd
// (opt_dep, accretion.f90:65-100)
HNU void opt_dep(const Emission &q, double hd, double kt, double nn, double np, double *ta1, double *ta2,
                 double *ts)
{
  const double t11 = kt * 1.16059e-1;
  const double xl = 5.67051e39 * 4.0 * 7.0 / 8.0 * (sq(t11) * sq(t11));
  *ta1 = q.qe * hd / xl;
  *ta2 = q.qo * hd / xl;
  const double cv = (double)(0.5f + 2.0f * 0.23f);
  const double alph = 1.25, xme = 0.510998910;
  const double csn = (1.0 + 5.0 * sq(alph)) / 24.0;
  const double csp = (4.0 * sq(cv - 1.0) + 5.0 * sq(alph)) / 24.0;
  const double tsn = csn * 1.76e-5 * nn * hd * HNU_F(13.8) * sq(kt / xme);
  const double tsp = csp * 1.76e-5 * np * hd * HNU_F(13.8) * sq(kt / xme);
  *ts = tsn + tsp;
}

// blocking factors of electron and heavy-lepton neutrinos (b_neu)
HNU void b_neu(double ta1, double ta2, double ts, double *b1, double *b2)
{
  const double te = ta1 + ts, tt = ta2 + ts, r3 = sqrt(3.0);
  const double third = (double)(1.0f / 3.0f);
  *b1 = (te / 2.0 + 1.0 / r3) / (te / 2.0 + 1.0 / r3 + third / ta1);
  *b2 = (tt / 2.0 + 1.0 / r3) / (tt / 2.0 + 1.0 / r3 + third / ta2);
  if (ta1 <= 0.0 || ta2 <= 0.0) *b1 = *b2 = 0.0;
}

// ---------------------------------------------------------------------------
// Chemical equilibrium (chem_eq.f90)
// ---------------------------------------------------------------------------

// the state shared by funcnb's evaluations (the Fortran common block /nucl/)
struct Nucl {
  double nnucl, kt, ne0, hdfac, nb0;
};

// the net rate of the six neutron-proton reactions, relative to p e- -> n nu,
// with neutrino blocking b1 (neutrino, chem_eq.f90:194-253)
HNU_NOINLINE double net_rate(const Rules &R, double b1, double kt, double nn, double np, double etae)
{
  const double etaep = -etae - 2.0 * XME / kt;
  const double t11 = kt * 1.16059e-1;
  const double t5 = sq(t11) * sq(t11) * t11;
  if (nn < 0.0) nn = 0.0;
  if (np < 0.0) np = 0.0;
  const double a = XME / kt, b = (XMN - XMP) / kt, h = 0.5 * (b - a);
  double I[6];
  lane_sum<6, 80>(RateTerms<2, true>{R, kt, etae, etaep, b1, 0.5 * (a + b), h}, I);
  const double evn = 2.03813046e35 * t5 * nn * (I[0] * h + I[3] * h);
  const double evep = 2.03813046e35 * t5 * np * (I[1] * 1.0 + I[4] * 1.0);
  const double even = 2.03813046e35 * t5 * nn * (I[2] * 1.0 + I[5] * 1.0);
  if (fabs(evep) < 1.0e-80) return (evep - even - evn) / (fabs(evep) + 1.0e-80);
  return (evep - even - evn) / fabs(evep);
}

// degeneracies of the nucleons for proton fraction xp (nuclear)
HNU void nuclear(const Rules &R, double kt, double nb, double xp, double *etan, double *etap)
{
  double np = nb * xp, nn = nb - np;
  if (np <= 0.0) np = 0.0;
  *etap = peta(R, kt, np);
  if (nn <= 0.0) nn = 0.0;
  *etan = neta(R, kt, nn);
}

// the energy balance of the gas at proton fraction xp, with the neutrino
// trapping iterated ten times (funcnb, chem_eq.f90:140-192)
HNU_NOINLINE double funcnb(const Rules &R, const Nucl &c, double xp)
{
  const double beta = c.kt / XME;
  double etan, etap;
  nuclear(R, c.kt, c.nnucl, xp, &etan, &etap);
  const double nhe = c.ne0 / 2.0;
  const double np = c.nnucl * xp, nn = c.nnucl - np;
  const double ne = c.nnucl * xp + c.ne0;
  const double etae = eeta(R, c.kt, ne);
  const double etaep = -etae - 2.0 / beta;
  double b1 = 0.0, b2 = 0.0, nl, nee, nep;
  lepton<1>(R, c.kt, &etae, &nl, &nee, &nep);
  double e, p, ehe, phe;
  eos_npe(R, c.kt, etan, etap, etae, nee, &e, &p);
  const double pr = p_rad(c.kt), er = 3.0 * pr;
  eos_he(c.kt, nhe, &ehe, &phe);
  const double p1 = p + pr + phe, e1 = e + er + ehe;
  const Emission q = emission(R, c.kt, c.nnucl, nn, np, etae, etaep);
  for (int i = 0; i < 10; i++) {
    const double pneu = p_neu(c.kt, b1, b2);
    double pp = p1 + pneu, ee = e1 + 3.0 * pneu;
    const double hd = h_dep(c.hdfac, c.nb0, pp, ee);
    double ta1, ta2, ts;
    opt_dep(q, hd, c.kt, nn, np, &ta1, &ta2, &ts);
    b_neu(ta1, ta2, ts, &b1, &b2);
  }
  return net_rate(R, b1, c.kt, nn, np, etae);
}

struct FuncNb3 {
  const Rules &R;
  const Nucl &c;
  HNU void operator()(const double *x, double *y) const
  {
    for (int i = 0; i < 3; i++) y[i] = funcnb(R, c, x[i]);
  }
};

struct Abundance {
  double e, p, qnu, tau, nee, nep;  // erg cm^-3, erg cm^-3, erg cm^-2 s^-1, -, fm^-3, fm^-3
  double xp;                        // proton fraction of the free nucleons
};

// abundance() at density rho (g cm^-3), temperature T (K) and scale-height
// factor hdfac (abundance.f90:6-243, with chem_eq and eqnucl, chem_eq.f90:49-102)
HNU_NOINLINE Abundance abundance(const Rules &R, double rho, double T, double hdfac)
{
  const double nb = rho / 1.66e15;
  const double kt = T / 1.16059e10;
  const double beta = kt / XME;
  const double xn = xnuc(nb, kt);
  const double nnuc = nb * xn;
  const double nhe = (nb - nnuc) / 4.0;

  // eqnucl: the proton fraction by Newton on funcnb from 1/2, kept in [0, 1]
  const Nucl c{nb * xn, kt, fabs(1.0 - xn) * nb / 2.0, hdfac, nb};
  double xp = newton1(FuncNb3{R, c}, (1.0 - 0.0) / 2.0, 0.0, newton_tol(c.nnucl));
  if (xp < 0.0) xp = 0.0;
  if (xp > 1.0) xp = 1.0;
  double etan, etap;
  nuclear(R, kt, c.nnucl, xp, &etan, &etap);
  const double np = c.nnucl * xp, nn = c.nnucl - np;
  const double etae = eeta(R, kt, np + c.ne0);

  const double etaep = -etae - 2.0 / beta;
  Abundance a;
  double nl;
  lepton<1>(R, kt, &etae, &nl, &a.nee, &a.nep);
  double enucl, pnucl, ehe, phe;
  eos_npe(R, kt, etan, etap, etae, a.nee, &enucl, &pnucl);
  const double prad = p_rad(kt), erad = 3.0 * prad;
  eos_he(kt, nhe, &ehe, &phe);
  const double p1 = pnucl + prad + phe, e1 = enucl + erad + ehe;
  double b1 = 0.0, b2 = 0.0, ta1 = 0.0, ta2 = 0.0, ts = 0.0;
  const Emission q = emission(R, kt, nnuc, nn, np, etae, etaep);
  for (int i = 0; i < 10; i++) {
    const double pneu = p_neu(kt, b1, b2);
    double p = p1 + pneu, e = e1 + 3.0 * pneu;
    const double hd = h_dep(hdfac, nb, p, e);
    opt_dep(q, hd, kt, nn, np, &ta1, &ta2, &ts);
    b_neu(ta1, ta2, ts, &b1, &b2);
  }
  const double pneu = p_neu(kt, b1, b2), eneu = 3.0 * pneu;
  const double T4 = sq(T) * sq(T);
  a.qnu = 7.0 / 8.0 * SIGMASB * T4 / 0.75 *
          (1. / (0.5 * ta1 + 0.5 * ts + HNU_F(0.557) + HNU_F(0.3) / ta1) +
           1. / (0.5 * ta2 + 0.5 * ts + HNU_F(0.557) + HNU_F(0.3) / ta2));
  a.tau = ts + ta1 + ta2;
  a.p = (pnucl + prad + pneu + phe) * 1.6021772e33;
  a.e = (enucl + erad + eneu + ehe) * 1.6021772e33;
  a.xp = xp;
  return a;
}

}  // namespace nu
}  // namespace harm
