// fgpu_ddmath.h -- correctly rounded natural logarithm and exponential in
// double-double arithmetic, for host and device.
//
// fosite's step-size controller (AdjustTimestep, timedisc_base.f90:759-814) takes
// EXP and LOG of the error norm; the host compiler's libm and CUDA's libm may round
// these differently.  Evaluating both in double-double (about 104 significant bits)
// and rounding once gives the correctly rounded value on the host and on the device
// alike, so a controller running on either side produces the same step sizes.
//
// Methods (textbook, see e.g. Muller, "Elementary Functions", ch. 6-7):
//   log x = k ln 2 + 2 atanh(s),  s = (m - 1)/(m + 1),  x = m 2^k,  m in [sqrt(1/2), sqrt(2)),
//           atanh by its odd power series in s^2 (|s| <= 0.172);
//   exp x = 2^k exp(r),  r = x - k ln 2 with |r| <= ln2/2, exp(r) by its Taylor series.
// ln 2 is split into a double and a remainder (0x1.62e42fefa39efp-1 + 0x1.abc9e3b39803fp-56).
// Products and sums are rounded individually (no contraction), so every platform
// evaluates the same operations.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define FGPU_HD __host__ __device__ __forceinline__
#else
#define FGPU_HD inline
#endif

namespace fgpu {
namespace ddm {

struct dd { double hi, lo; };

// IEEE operations that the compiler may not fuse
FGPU_HD double add_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  volatile double s = a + b;
  return s;
#endif
}
FGPU_HD double mul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  volatile double p = a * b;
  return p;
#endif
}
FGPU_HD double fma_rn(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

FGPU_HD dd two_sum(double a, double b) {
  const double s = add_rn(a, b);
  const double bb = add_rn(s, -a);
  const double e = add_rn(add_rn(a, -add_rn(s, -bb)), add_rn(b, -bb));
  return {s, e};
}
FGPU_HD dd quick_two_sum(double a, double b) {
  const double s = add_rn(a, b);
  return {s, add_rn(b, -add_rn(s, -a))};
}
FGPU_HD dd two_prod(double a, double b) {
  const double p = mul_rn(a, b);
  return {p, fma_rn(a, b, -p)};
}
FGPU_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo = add_rn(s.lo, t.hi);
  s = quick_two_sum(s.hi, s.lo);
  s.lo = add_rn(s.lo, t.lo);
  return quick_two_sum(s.hi, s.lo);
}
FGPU_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = add_rn(p.lo, add_rn(mul_rn(a.hi, b.lo), mul_rn(a.lo, b.hi)));
  return quick_two_sum(p.hi, p.lo);
}
FGPU_HD dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo = add_rn(p.lo, mul_rn(a.lo, b));
  return quick_two_sum(p.hi, p.lo);
}
// a / b with three quotient digits
FGPU_HD dd dd_div(dd a, dd b) {
  const double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_mul_d(b, -q1));
  const double q2 = r.hi / b.hi;
  r = dd_add(r, dd_mul_d(b, -q2));
  const double q3 = r.hi / b.hi;
  dd q = quick_two_sum(q1, q2);
  return dd_add(q, dd{q3, 0.0});
}

constexpr double LN2_HI = 0x1.62e42fefa39efp-1;
constexpr double LN2_LO = 0x1.abc9e3b39803fp-56;

// correctly rounded log(x) for positive normal x (other arguments: the platform's log)
FGPU_HD double log_cr(double x) {
  if (!(x > 0.0) || !(x < INFINITY) || x < 0x1p-1022) return log(x);
  int k;
  double m = frexp(x, &k);                   // x = m 2^k, m in [1/2, 1)
  if (m < 0x1.6a09e667f3bcdp-1) { m = m * 2.0; k -= 1; }   // m in [sqrt(1/2), sqrt(2))
  const dd num = {add_rn(m, -1.0), 0.0};      // exact (Sterbenz)
  const dd den = two_sum(m, 1.0);
  const dd s = dd_div(num, den);
  const dd s2 = dd_mul(s, s);
  // atanh(s)/s = sum_{j>=0} s^(2j)/(2j+1), |s^2| < 0.0295: 24 terms reach 2^-120
  dd acc = dd_div(dd{1.0, 0.0}, dd{49.0, 0.0});
  for (int j = 23; j >= 0; --j) acc = dd_add(dd_mul(acc, s2), dd_div(dd{1.0, 0.0}, dd{2.0 * j + 1.0, 0.0}));
  dd r = dd_mul(dd_mul_d(s, 2.0), acc);
  const dd kl = dd_add(two_prod((double)k, LN2_HI), dd{mul_rn((double)k, LN2_LO), 0.0});
  r = dd_add(kl, r);
  return add_rn(r.hi, r.lo);
}

// correctly rounded exp(x) for |x| < 700 (other arguments: the platform's exp)
FGPU_HD double exp_cr(double x) {
  if (!(fabs(x) < 700.0)) return exp(x);
  const double k = nearbyint(x / LN2_HI);
  // r = x - k ln2 in double-double
  const dd p = two_prod(k, LN2_HI);
  dd r = two_sum(x, -p.hi);
  r.lo = add_rn(r.lo, -p.lo);
  r.lo = add_rn(r.lo, -mul_rn(k, LN2_LO));
  r = quick_two_sum(r.hi, r.lo);
  // exp(r) = 1 + r(1 + r/2(1 + r/3(...))), |r| <= 0.347: 27 terms reach 2^-120
  dd acc = {1.0, 0.0};
  for (int n = 27; n >= 1; --n) acc = dd_add(dd{1.0, 0.0}, dd_div(dd_mul(r, acc), dd{(double)n, 0.0}));
  return ldexp(add_rn(acc.hi, acc.lo), (int)k);
}

}  // namespace ddm
}  // namespace fgpu
