// Host side of the COOL_EOS table generator (harm_nu.cuh): the quadrature
// rules, and abundance() over a list of nodes on the host's cores.
//
// harm_nu_abundance() is the library's counterpart of the reference's
// Fortran entry point abundance_() (abundance.f90:6-243, bound from C++ at
// cooleos.c:58-59 and called per table node by calc_cache_val,
// cooleos.c:171-194); harm_nu_tables() (harm_nu.cu) builds whole tables on
// the device.
#include "harm_b200.h"
#include "harm_nu.cuh"

#include <math.h>

#include <atomic>
#include <string>
#include <thread>
#include <vector>

namespace harm {
int fail_with(int code, const std::string &msg);

namespace nu {

namespace {

// Legendre polynomial P_n(x) by the three-term recurrence, and P_{n-1}(x)
void legendre(int n, long double x, long double *pn, long double *pn1)
{
  long double p0 = 1.0L, p1 = x;
  for (int k = 1; k < n; k++) {
    const long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pn1 = p0;
}

// Laguerre polynomial L_n(x) by the three-term recurrence
long double laguerre(int n, long double x)
{
  long double l0 = 1.0L, l1 = 1.0L - x;
  if (n == 0) return l0;
  for (int k = 1; k < n; k++) {
    const long double l2 = ((2 * k + 1 - x) * l1 - k * l0) / (k + 1);
    l0 = l1;
    l1 = l2;
  }
  return l1;
}

// the zeros of f on (lo, hi), bracketed by sign changes on a grid of m steps
// and refined by bisection to the last bit of long double
template <class F>
std::vector<long double> zeros(const F &f, long double lo, long double hi, int m)
{
  std::vector<long double> z;
  long double a = lo, fa = f(a);
  for (int s = 1; s <= m; s++) {
    const long double b = lo + (hi - lo) * s / m, fb = f(b);
    if ((fa < 0) != (fb < 0)) {
      long double u = a, v = b, fu = fa;
      for (int it = 0; it < 200; it++) {
        const long double c = 0.5L * (u + v);
        if (c <= u || c >= v) break;
        const long double fc = f(c);
        if ((fc < 0) == (fu < 0)) {
          u = c;
          fu = fc;
        } else {
          v = c;
        }
      }
      z.push_back(0.5L * (u + v));
    }
    a = b;
    fa = fb;
  }
  return z;
}

// n-point Gauss-Legendre: the n/2 positive abscissae in increasing order and
// their weights 2 / ((1 - x^2) P_n'(x)^2)
bool gauss_legendre(int n, double *x, double *w)
{
  auto P = [n](long double t) {
    long double pn, pn1;
    legendre(n, t, &pn, &pn1);
    return pn;
  };
  const std::vector<long double> z = zeros(P, 0.0L, 1.0L, 200000);
  if ((int)z.size() != n / 2) return false;
  for (int i = 0; i < n / 2; i++) {
    const long double t = z[i];
    long double pn, pn1;
    legendre(n, t, &pn, &pn1);
    const long double dp = n * (t * pn - pn1) / (t * t - 1.0L);
    x[i] = (double)t;
    w[i] = (double)(2.0L / ((1.0L - t * t) * dp * dp));
  }
  return true;
}

// n-point Gauss-Laguerre (weight e^-x on (0, inf)): abscissae and e^x times
// the weights x / ((n+1)^2 L_{n+1}(x)^2)
bool gauss_laguerre(int n, double *x, double *w)
{
  auto L = [n](long double t) { return laguerre(n, t); };
  const std::vector<long double> z = zeros(L, 1.0e-6L, 4.0L * n + 2.0L, 400000);
  if ((int)z.size() != n) return false;
  for (int i = 0; i < n; i++) {
    const long double t = z[i];
    const long double l1 = laguerre(n + 1, t);
    x[i] = (double)t;
    w[i] = (double)(expl(t) * t / ((long double)(n + 1) * (n + 1) * l1 * l1));
  }
  return true;
}

}  // namespace

// the rules, computed once; null if a root search came up short
const Rules *host_rules()
{
  static Rules r;
  static const bool ok = gauss_legendre(20, r.l20x, r.l20w) && gauss_legendre(40, r.l40x, r.l40w) &&
                         gauss_laguerre(20, r.g20x, r.g20w);
  return ok ? &r : nullptr;
}

}  // namespace nu
}  // namespace harm

using namespace harm;

extern "C" int harm_nu_rules(double *out)
{
  if (!out) return fail_with(HARM_E_ARG, "harm_nu_rules: null output");
  const nu::Rules *R = nu::host_rules();
  if (!R) return fail_with(HARM_E_ARG, "harm_nu_rules: quadrature root search failed");
  const double *src = &R->l20x[0];
  for (size_t i = 0; i < sizeof(nu::Rules) / sizeof(double); i++) out[i] = src[i];
  return HARM_OK;
}

extern "C" int harm_nu_fermi(const double *eta, const double *theta, long n, double *F)
{
  if (n < 0 || (n > 0 && (!eta || !theta || !F))) return fail_with(HARM_E_ARG, "harm_nu_fermi: bad arguments");
  const nu::Rules *R = nu::host_rules();
  if (!R) return fail_with(HARM_E_ARG, "harm_nu_fermi: quadrature root search failed");
  for (long i = 0; i < n; i++) nu::fermi<1, 4>(*R, eta + i, theta + i, F + 4 * i);
  return HARM_OK;
}

extern "C" int harm_nu_abundance(const double *rho, const double *T, const double *hdfac, long n, int threads,
                                 double *out)
{
  if (n < 0 || (n > 0 && (!rho || !T || !hdfac || !out)))
    return fail_with(HARM_E_ARG, "harm_nu_abundance: bad arguments");
  const nu::Rules *Rp = nu::host_rules();
  if (!Rp) return fail_with(HARM_E_ARG, "harm_nu_abundance: quadrature root search failed");
  const nu::Rules &R = *Rp;
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads < 1) threads = 1;
  if (threads > n) threads = (int)(n > 0 ? n : 1);
  std::atomic<long> next(0);
  auto work = [&] {
    for (long i; (i = next.fetch_add(1)) < n;) {
      const nu::Abundance a = nu::abundance(R, rho[i], T[i], hdfac[i]);
      double *o = out + 7 * i;
      o[0] = a.e;
      o[1] = a.p;
      o[2] = a.qnu;
      o[3] = a.tau;
      o[4] = a.nee;
      o[5] = a.nep;
      o[6] = a.xp;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; t++) pool.emplace_back(work);
  work();
  for (auto &t : pool) t.join();
  return HARM_OK;
}
