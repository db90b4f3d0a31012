// x^y rounded to nearest, for the isentropic fall-back inversions.
//
// The reference's fall-backs (utoprim_1dvsq2fix1.c, utoprim_1dfix1.c) raise
// densities to the adiabatic index with the host libm's pow(), which returns
// the correctly rounded power except in rare cases within a tiny fraction of
// an ulp of a rounding boundary.  CUDA's pow() is accurate to about two ulps,
// so a fall-back zone could land one ulp away from the reference.  pow_cr
// evaluates exp(y ln x) in double-double arithmetic (relative error near
// 2^-95) and rounds once, which gives the correctly rounded power whenever
// the exact value is not within about 2^-42 ulp of a boundary.
//
// Double-double arithmetic: Dekker's exact product by FMA and Knuth's
// two-sum (the QD library's algorithms, Hida, Li and Bailey, 2001).
// ln m for m in [1/sqrt2, sqrt2) by the series 2 atanh s, s = (m-1)/(m+1),
// |s| <= 0.1716 (21 terms reach 2^-107); exp r by r = k ln2 + r', Taylor
// series of r'/1024 (8 terms) squared ten times.  The constants are 1/(2k+1),
// 1/n! and ln 2 split into the nearest double and the nearest double to the
// remainder.  The two exponents of the gamma = 4/3 law take a cheaper path
// through the cube root (pow_third), which gives the same rounded results.
#pragma once

namespace harm {

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD dd_two_sum(double a, double b)
{
  const double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b)
{
  const double s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b)
{
  DD s = dd_two_sum(a.hi, b.hi);
  const DD t = dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DD dd_mul(DD a, DD b)
{
  const double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return dd_fast_two_sum(p, e);
}
__device__ __forceinline__ DD dd_mul_d(DD a, double b)
{
  const double p = a.hi * b;
  double e = fma(a.hi, b, -p);
  e += a.lo * b;
  return dd_fast_two_sum(p, e);
}
__device__ __forceinline__ DD dd_div(DD a, DD b)
{
  const double q1 = a.hi / b.hi;
  DD r = dd_add(a, dd_mul_d(b, -q1));
  const double q2 = r.hi / b.hi;
  r = dd_add(r, dd_mul_d(b, -q2));
  const double q3 = r.hi / b.hi;
  return dd_add(dd_fast_two_sum(q1, q2), DD{q3, 0.});
}

__device__ __forceinline__ DD dd_ln2() { return {0.6931471805599453, 2.3190468138462996e-17}; }

// ln x for finite x > 0
__device__ __forceinline__ DD dd_log(double x)
{
  // 1/(2k+1), k = 0..21
  const double io_hi[22] = {1.0, 0.3333333333333333, 0.2, 0.14285714285714285, 0.1111111111111111,
                            0.09090909090909091, 0.07692307692307693, 0.06666666666666667, 0.058823529411764705,
                            0.05263157894736842, 0.047619047619047616, 0.043478260869565216, 0.04,
                            0.037037037037037035, 0.034482758620689655, 0.03225806451612903,
                            0.030303030303030304, 0.02857142857142857, 0.02702702702702703, 0.02564102564102564,
                            0.024390243902439025, 0.023255813953488372};
  const double io_lo[22] = {0.0, 1.850371707708594e-17, -1.1102230246251566e-17, 7.93016446160826e-18,
                            6.1679056923619804e-18, -2.523234146875356e-18, -4.270088556250602e-18,
                            9.251858538542971e-19, 8.163404592832033e-19, 2.921639538487254e-18,
                            2.64338815386942e-18, 1.206764157201257e-18, -8.326672684688674e-19,
                            2.05596856412066e-18, 4.785444071660157e-19, 8.953411488912552e-19,
                            -8.410780489584519e-19, 8.921435019309293e-19, -1.50030138462859e-18,
                            8.896017825522087e-19, -8.46206573647223e-19, 3.2273925134452225e-19};
  int e;
  double m = frexp(x, &e);  // x = m 2^e, m in [1/2, 1)
  if (m < 0.7071067811865476) {
    m *= 2.;
    e -= 1;
  }
  const DD s = dd_div(DD{m - 1., 0.}, dd_two_sum(m, 1.));  // m - 1 is exact for m in [1/2, 2]
  const DD s2 = dd_mul(s, s);
  DD t{io_hi[21], io_lo[21]};
#pragma unroll 1
  for (int k = 20; k >= 0; k--) t = dd_add(dd_mul(t, s2), DD{io_hi[k], io_lo[k]});
  return dd_add(dd_mul_d(dd_ln2(), (double)e), dd_mul(dd_mul_d(s, 2.), t));
}

// e^z for |z.hi| <= 700, as a double-double before the scaling by 2^k
__device__ __forceinline__ double dd_exp_rn(DD z)
{
  // 1/n!, n = 0..8
  const double if_hi[9] = {1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664, 0.008333333333333333,
                           0.001388888888888889, 0.0001984126984126984, 2.48015873015873e-05};
  const double if_lo[9] = {0.0, 0.0, 0.0, 9.25185853854297e-18, 2.3129646346357427e-18, 1.1564823173178714e-19,
                           -5.300543954373577e-20, 1.7209558293420705e-22, 2.1511947866775882e-23};
  const double k = rint(z.hi * 1.4426950408889634);
  DD r = dd_add(z, dd_mul_d(dd_ln2(), -k));
  r.hi *= 0.0009765625;  // 2^-10, exact
  r.lo *= 0.0009765625;
  DD t{if_hi[8], if_lo[8]};
#pragma unroll 1
  for (int n = 7; n >= 0; n--) t = dd_add(dd_mul(t, r), DD{if_hi[n], if_lo[n]});
#pragma unroll 1
  for (int q = 0; q < 10; q++) t = dd_mul(t, t);
  return ldexp(t.hi, (int)k);  // t.hi is t rounded to nearest; the scaling is exact
}

// x^y for the exponents of the gamma = 4/3 law, y = RN(4/3) and RN(4/3) - 1,
// which the fall-back inversions raise densities to in their inner loops.
// Both are k/3 + d with k = 4 or 1 and the same offset d = -2^-52/3 exactly
// (4/3 rounds down by a third of an ulp), so
//   x^y = (x^(1/3))^k (1 + d ln x + (d ln x)^2/2 + ...),  |d ln x| < 5.2e-14.
// The cube root is cbrt(x) refined by one Newton step with its residual
// x - c^3 formed in double-double: the step squares cbrt's relative error
// (below 2^-51), and the residual and the correction are good to 2^-101.
// With the product by x and the first-order term, the double-double result
// is within 2^-88 of x^y.  It is returned rounded when every value within
// 2^-84 of it rounds the same way, and the exact x^y, within 2^-88, is one of
// them; otherwise (about once in 2^31 draws) the caller takes the general
// path.  Arguments: 2^-700 <= x <= 2^700, so that the result and its ulp are
// normal doubles.
__device__ __forceinline__ bool pow_third(double x, double y, double &out)
{
  int k;
  if (y == 1.3333333333333333) k = 4;          // RN(4/3)
  else if (y == 0.33333333333333326) k = 1;    // RN(4/3) - 1, exact
  else return false;
  if (!(x >= 0x1p-700 && x <= 0x1p700)) return false;
  const double c0 = cbrt(x);
  // c0^3 = q + q_lo to 2^-104; x - q is exact (q is within a factor 2 of x)
  const double s = c0 * c0, s_lo = fma(c0, c0, -s);
  const double q = s * c0, q_lo = fma(s, c0, -q) + s_lo * c0;
  const double r = (x - q) - q_lo;
  const DD c = dd_fast_two_sum(c0, r / (3.0 * s));
  const DD P = (k == 4) ? dd_mul_d(c, x) : c;
  const double t = -(0x1p-52 / 3.0) * log(x);  // d ln x
  const DD v = dd_add(P, DD{P.hi * t, 0.});
  // v.hi is v rounded, |v.lo| <= half an ulp of v.hi; the spacing below a power
  // of two is half the spacing above
  const long long b = __double_as_longlong(v.hi);
  const double ulp = __longlong_as_double((((b >> 52) & 0x7ff) - 52) << 52);
  const double half = (v.lo < 0. && (b & 0xfffffffffffffLL) == 0) ? 0.25 * ulp : 0.5 * ulp;
  if (fabs(v.lo) + v.hi * 0x1p-84 < half) {
    out = v.hi;
    return true;
  }
  return false;
}

// x^y rounded to nearest for finite x > 0 and finite y with |y ln x| <= 700;
// every other case (zero, negative, infinite or NaN arguments, over- and
// underflow) goes to pow().  pow_dd is the general path; pow_cr tries
// pow_third first.
__device__ __forceinline__ double pow_dd(double x, double y)
{
  if (!(x > 0.) || !isfinite(x) || !isfinite(y)) return pow(x, y);
  if (y == 0.) return 1.;
  const DD z = dd_mul_d(dd_log(x), y);
  if (!(fabs(z.hi) <= 700.)) return pow(x, y);
  return dd_exp_rn(z);
}

static __device__ __noinline__ double pow_cr(double x, double y)
{
  double r;
  if (pow_third(x, y, r)) return r;
  return pow_dd(x, y);
}

}  // namespace harm
