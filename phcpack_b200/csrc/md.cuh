// md.cuh -- multiple-double arithmetic on the device (sm_100a).
//
// Number formats as in PHCpack src/GPU/Norms: double-double (hi, lo),
// quad-double and octo-double (four and eight limbs, decreasing
// significance), stored limb-interleaved.  Complex numbers store the real limbs, then the
// imaginary limbs.
//
// Every floating-point operation goes through __dadd_rn / __dsub_rn /
// __dmul_rn / __fma_rn, so nvcc can neither contract an add and a multiply
// into an FMA nor reassociate: the error-free transformations stay exact.
// The one intended FMA is two_prod, whose error term a*b - p is exact when
// computed by a single fused multiply-add (it replaces the Dekker split of
// Norms/double_double_gpufun.cu:158-193; both are exact).
//
// Algorithms: two_sum (Knuth), quick_two_sum (Dekker); dd add/mul/div as in
// the QD library of Hida, Li and Bailey (Norms/double_double_gpufun.cu:17-260);
// qd add/mul as limb-wise accumulation with error propagation and a final
// renormalisation (the baileyAdd_fast / baileyMul_fast scheme of CAMPARY,
// Norms/quad_double_gpufun.cu:209,313), written as unrolled loops.
#pragma once
#include <cuda_runtime.h>

namespace md {

#define MD_INL __device__ __forceinline__

MD_INL double add(double a, double b) { return __dadd_rn(a, b); }
MD_INL double sub(double a, double b) { return __dsub_rn(a, b); }
MD_INL double mul(double a, double b) { return __dmul_rn(a, b); }

MD_INL double two_sum(double a, double b, double &e) {
  double s = add(a, b);
  double bb = sub(s, a);
  e = add(sub(a, sub(s, bb)), sub(b, bb));
  return s;
}
MD_INL double quick_two_sum(double a, double b, double &e) {
  double s = add(a, b);
  e = sub(b, sub(s, a));
  return s;
}
MD_INL double two_prod(double a, double b, double &e) {
  double p = mul(a, b);
  e = __fma_rn(a, b, -p);
  return p;
}

// ------------------------------------------------------------- dd
struct dd {
  double hi, lo;
};
MD_INL dd mk(double h, double l) { dd r; r.hi = h; r.lo = l; return r; }

MD_INL dd operator+(dd a, dd b) {
  double s2, t2;
  double s1 = two_sum(a.hi, b.hi, s2);
  double t1 = two_sum(a.lo, b.lo, t2);
  s2 = add(s2, t1);
  s1 = quick_two_sum(s1, s2, s2);
  s2 = add(s2, t2);
  dd r;
  r.hi = quick_two_sum(s1, s2, r.lo);
  return r;
}
MD_INL dd operator-(dd a) { return mk(-a.hi, -a.lo); }
MD_INL dd operator-(dd a, dd b) { return a + (-b); }
MD_INL dd operator*(dd a, dd b) {
  double p2;
  double p1 = two_prod(a.hi, b.hi, p2);
  p2 = __fma_rn(a.hi, b.lo, p2);
  p2 = __fma_rn(a.lo, b.hi, p2);
  dd r;
  r.hi = quick_two_sum(p1, p2, r.lo);
  return r;
}
MD_INL dd mul_d(dd a, double b) {
  double p2;
  double p1 = two_prod(a.hi, b, p2);
  p2 = __fma_rn(a.lo, b, p2);
  dd r;
  r.hi = quick_two_sum(p1, p2, r.lo);
  return r;
}
MD_INL dd operator/(dd a, dd b) {
  double q1 = __ddiv_rn(a.hi, b.hi);
  dd r = a - mul_d(b, q1);
  double q2 = __ddiv_rn(r.hi, b.hi);
  r = r - mul_d(b, q2);
  double q3 = __ddiv_rn(r.hi, b.hi);
  dd q;
  q.hi = quick_two_sum(q1, q2, q.lo);
  return q + mk(q3, 0.0);
}
// Karp's square root: sqrt(a) = a*x + (a - (a*x)^2)*x/2 with x ~ 1/sqrt(a)
MD_INL dd sqrt(dd a) {
  if (a.hi == 0.0 && a.lo == 0.0) return mk(0.0, 0.0);
  if (a.hi < 0.0) return mk(-1.0, 0.0);
  double x = __ddiv_rn(1.0, __dsqrt_rn(a.hi));
  double ax = mul(a.hi, x);
  dd axsq = mk(ax, 0.0) * mk(ax, 0.0);
  dd y = a - axsq;
  dd r;
  r.hi = two_sum(ax, mul(mul(y.hi, x), 0.5), r.lo);
  return r;
}
MD_INL double lead(dd a) { return a.hi; }
MD_INL bool is_zero(dd a) { return a.hi == 0.0 && a.lo == 0.0; }

// ------------------------------------------------------------- qd
struct qd {
  double x[4];
};
MD_INL qd mkq(double a, double b, double c, double d) { qd r; r.x[0] = a; r.x[1] = b; r.x[2] = c; r.x[3] = d; return r; }

// five overlapping terms (decreasing magnitude) -> four-term expansion
MD_INL qd renorm5(double f0, double f1, double f2, double f3, double f4) {
  double e1, e2, e3, e4;
  double s = quick_two_sum(f3, f4, e4);
  s = quick_two_sum(f2, s, e3);
  s = quick_two_sum(f1, s, e2);
  double e0 = quick_two_sum(f0, s, e1);
  const double f[5] = {e0, e1, e2, e3, e4};
  // top-down pass: emit a component whenever the running sum leaves a
  // non-zero error; components are placed by predicated selects so the
  // result stays in registers
  double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
  int k = 0;
  double acc = f[0];
#pragma unroll
  for (int i = 1; i <= 4; ++i) {
    double e;
    double t = quick_two_sum(acc, f[i], e);
    if (e != 0.0 && k < 4) {
      r0 = (k == 0) ? t : r0;
      r1 = (k == 1) ? t : r1;
      r2 = (k == 2) ? t : r2;
      r3 = (k == 3) ? t : r3;
      ++k;
      acc = e;
    } else {
      acc = t;
    }
  }
  if (k < 4 && acc != 0.0) {
    r0 = (k == 0) ? acc : r0;
    r1 = (k == 1) ? acc : r1;
    r2 = (k == 2) ? acc : r2;
    r3 = (k == 3) ? acc : r3;
  }
  return mkq(r0, r1, r2, r3);
}

MD_INL void accum(double &f1, double &f2, double &f3, double &f4, int lvl, double v) {
  if (lvl <= 1) f1 = two_sum(f1, v, v);
  if (lvl <= 2) f2 = two_sum(f2, v, v);
  if (lvl <= 3) f3 = two_sum(f3, v, v);
  f4 = add(f4, v);
}

MD_INL qd operator+(const qd &a, const qd &b) {
  double e;
  double f0, f1, f2, f3, f4 = 0.0;
  f3 = two_sum(a.x[3], b.x[3], e);
  f4 = add(f4, e);
  f2 = two_sum(a.x[2], b.x[2], e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  f1 = two_sum(a.x[1], b.x[1], e);
  f2 = two_sum(f2, e, e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  f0 = two_sum(a.x[0], b.x[0], e);
  f1 = two_sum(f1, e, e);
  f2 = two_sum(f2, e, e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  return renorm5(f0, f1, f2, f3, f4);
}
MD_INL qd operator-(const qd &a) { return mkq(-a.x[0], -a.x[1], -a.x[2], -a.x[3]); }
MD_INL qd operator-(const qd &a, const qd &b) { return a + (-b); }

MD_INL qd operator*(const qd &a, const qd &b) {
  double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0, f4;
  double e, p;
  // order-4 terms in plain arithmetic
  f4 = mul(a.x[1], b.x[3]);
  f4 = __fma_rn(a.x[2], b.x[2], f4);
  f4 = __fma_rn(a.x[3], b.x[1], f4);
  // order 3
  p = two_prod(a.x[0], b.x[3], e); f4 = add(f4, e); f3 = add(f3, p);
  p = two_prod(a.x[1], b.x[2], e); f4 = add(f4, e); f3 = two_sum(f3, p, e); f4 = add(f4, e);
  p = two_prod(a.x[2], b.x[1], e); f4 = add(f4, e); f3 = two_sum(f3, p, e); f4 = add(f4, e);
  p = two_prod(a.x[3], b.x[0], e); f4 = add(f4, e); f3 = two_sum(f3, p, e); f4 = add(f4, e);
  // order 2
  f2 = two_prod(a.x[0], b.x[2], e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  p = two_prod(a.x[1], b.x[1], e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  f2 = two_sum(f2, p, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  p = two_prod(a.x[2], b.x[0], e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  f2 = two_sum(f2, p, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  // order 1
  f1 = two_prod(a.x[0], b.x[1], e); f2 = two_sum(f2, e, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  p = two_prod(a.x[1], b.x[0], e); f2 = two_sum(f2, e, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  f1 = two_sum(f1, p, e); f2 = two_sum(f2, e, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  // order 0
  f0 = two_prod(a.x[0], b.x[0], e);
  f1 = two_sum(f1, e, e); f2 = two_sum(f2, e, e); f3 = two_sum(f3, e, e); f4 = add(f4, e);
  return renorm5(f0, f1, f2, f3, f4);
}
MD_INL qd mul_d(const qd &a, double b) {
  double e;
  double f0, f1, f2, f3, f4 = 0.0;
  f3 = two_prod(a.x[3], b, e);
  f4 = add(f4, e);
  f2 = two_prod(a.x[2], b, e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  f1 = two_prod(a.x[1], b, e);
  f2 = two_sum(f2, e, e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  f0 = two_prod(a.x[0], b, e);
  f1 = two_sum(f1, e, e);
  f2 = two_sum(f2, e, e);
  f3 = two_sum(f3, e, e);
  f4 = add(f4, e);
  return renorm5(f0, f1, f2, f3, f4);
}
MD_INL qd operator/(const qd &a, const qd &b) {
  double q0 = __ddiv_rn(a.x[0], b.x[0]);
  qd r = a - mul_d(b, q0);
  double q1 = __ddiv_rn(r.x[0], b.x[0]);
  r = r - mul_d(b, q1);
  double q2 = __ddiv_rn(r.x[0], b.x[0]);
  r = r - mul_d(b, q2);
  double q3 = __ddiv_rn(r.x[0], b.x[0]);
  r = r - mul_d(b, q3);
  double q4 = __ddiv_rn(r.x[0], b.x[0]);
  return renorm5(q0, q1, q2, q3, q4);
}
MD_INL qd sqrt(const qd &a) {
  if (a.x[0] == 0.0 && a.x[1] == 0.0 && a.x[2] == 0.0 && a.x[3] == 0.0) return mkq(0.0, 0.0, 0.0, 0.0);
  if (a.x[0] < 0.0) return mkq(-1.0, 0.0, 0.0, 0.0);
  dd s = sqrt(mk(a.x[0], a.x[1]));
  qd b = mkq(s.hi, s.lo, 0.0, 0.0);
  qd z = b * b + a;
  z = z / b;
  return mkq(mul(z.x[0], 0.5), mul(z.x[1], 0.5), mul(z.x[2], 0.5), mul(z.x[3], 0.5));
}
MD_INL double lead(const qd &a) { return a.x[0]; }
MD_INL bool is_zero(const qd &a) { return a.x[0] == 0.0 && a.x[1] == 0.0 && a.x[2] == 0.0 && a.x[3] == 0.0; }

// ------------------------------------------------------------- od
// Octo-double: eight limbs, decreasing significance.  Add, multiply and
// divide generalise the qd scheme above to eight limbs: limb-wise (add) or
// order-wise (multiply: all products a_i b_j with i + j = p by two_prod for
// p < 8, plainly for p = 8) accumulation with the errors cascaded into the
// lower-order accumulators, a ninth accumulator for the rest, and a
// renormalisation of the nine terms: the scheme of the reference's
// octo-doubles (Norms/octo_double_functions.cpp, CAMPARY's
// baileyAdd/Mul_fast<8,8,8>), except that the order-8 products are summed
// by fused multiply-adds.
struct od {
  double x[8];
};
MD_INL od mko(double a) {
  od r;
#pragma unroll
  for (int i = 0; i < 8; ++i) r.x[i] = 0.0;
  r.x[0] = a;
  return r;
}

// nine overlapping terms (decreasing magnitude) -> eight-term expansion
MD_INL od renorm9(const double (&f)[9]) {
  double e[9];
  double s = quick_two_sum(f[7], f[8], e[8]);
#pragma unroll
  for (int i = 6; i >= 0; --i) s = quick_two_sum(f[i], s, e[i + 1]);
  e[0] = s;
  od r = mko(0.0);
  int k = 0;
  double acc = e[0];
#pragma unroll
  for (int i = 1; i <= 8; ++i) {
    double err;
    const double t = quick_two_sum(acc, e[i], err);
    if (err != 0.0 && k < 8) {
#pragma unroll
      for (int j = 0; j < 8; ++j) r.x[j] = (k == j) ? t : r.x[j];
      ++k;
      acc = err;
    } else {
      acc = t;
    }
  }
  if (k < 8 && acc != 0.0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) r.x[j] = (k == j) ? acc : r.x[j];
  }
  return r;
}

// v added at accumulator level lvl, its rounding errors cascaded down
MD_INL void accum9(double (&f)[9], int lvl, double v) {
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (j >= lvl) f[j] = two_sum(f[j], v, v);
  f[8] = add(f[8], v);
}

MD_INL od operator+(const od &a, const od &b) {
  double f[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) f[j] = 0.0;
#pragma unroll
  for (int i = 7; i >= 0; --i) {
    double e;
    f[i] = two_sum(a.x[i], b.x[i], e);
    accum9(f, i + 1, e);
  }
  return renorm9(f);
}
MD_INL od operator-(const od &a) {
  od r;
#pragma unroll
  for (int i = 0; i < 8; ++i) r.x[i] = -a.x[i];
  return r;
}
MD_INL od operator-(const od &a, const od &b) { return a + (-b); }

MD_INL od operator*(const od &a, const od &b) {
  double f[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) f[j] = 0.0;
  // order-8 terms in plain arithmetic
  f[8] = mul(a.x[1], b.x[7]);
#pragma unroll
  for (int i = 2; i < 8; ++i) f[8] = __fma_rn(a.x[i], b.x[8 - i], f[8]);
#pragma unroll
  for (int p = 7; p >= 0; --p) {
#pragma unroll
    for (int i = 0; i <= p; ++i) {
      double e;
      const double q = two_prod(a.x[i], b.x[p - i], e);
      accum9(f, p + 1, e);
      accum9(f, p, q);
    }
  }
  return renorm9(f);
}
MD_INL od mul_d(const od &a, double b) {
  double f[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) f[j] = 0.0;
#pragma unroll
  for (int i = 7; i >= 0; --i) {
    double e;
    f[i] = two_prod(a.x[i], b, e);
    accum9(f, i + 1, e);
  }
  return renorm9(f);
}
MD_INL od operator/(const od &a, const od &b) {
  double q[9];
  od r = a;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    q[i] = __ddiv_rn(r.x[0], b.x[0]);
    if (i < 8) r = r - mul_d(b, q[i]);
  }
  return renorm9(q);
}
MD_INL double lead(const od &a) { return a.x[0]; }
MD_INL bool is_zero(const od &a) {
  bool z = true;
#pragma unroll
  for (int i = 0; i < 8; ++i) z = z && a.x[i] == 0.0;
  return z;
}

// ------------------------------------------------------------- double
MD_INL double mul_d(double a, double b) { return mul(a, b); }
MD_INL double lead(double a) { return a; }
MD_INL bool is_zero(double a) { return a == 0.0; }

// ------------------------------------------------------------- traits
template <class R> struct real_traits;
template <> struct real_traits<double> {
  static const int limbs = 1;
  MD_INL static double zero() { return 0.0; }
  MD_INL static double one() { return 1.0; }
  MD_INL static double from(double a) { return a; }
  MD_INL static double add(double a, double b) { return __dadd_rn(a, b); }
  MD_INL static double sub(double a, double b) { return __dsub_rn(a, b); }
  MD_INL static double mul(double a, double b) { return __dmul_rn(a, b); }
  MD_INL static double div(double a, double b) { return __ddiv_rn(a, b); }
  MD_INL static double sqrt(double a) { return __dsqrt_rn(a); }
  MD_INL static double neg(double a) { return -a; }
};
template <> struct real_traits<dd> {
  static const int limbs = 2;
  MD_INL static dd zero() { return mk(0.0, 0.0); }
  MD_INL static dd one() { return mk(1.0, 0.0); }
  MD_INL static dd from(double a) { return mk(a, 0.0); }
  MD_INL static dd add(dd a, dd b) { return a + b; }
  MD_INL static dd sub(dd a, dd b) { return a - b; }
  MD_INL static dd mul(dd a, dd b) { return a * b; }
  MD_INL static dd div(dd a, dd b) { return a / b; }
  MD_INL static dd sqrt(dd a) { return md::sqrt(a); }
  MD_INL static dd neg(dd a) { return -a; }
};
template <> struct real_traits<qd> {
  static const int limbs = 4;
  MD_INL static qd zero() { return mkq(0.0, 0.0, 0.0, 0.0); }
  MD_INL static qd one() { return mkq(1.0, 0.0, 0.0, 0.0); }
  MD_INL static qd from(double a) { return mkq(a, 0.0, 0.0, 0.0); }
  MD_INL static qd add(const qd &a, const qd &b) { return a + b; }
  MD_INL static qd sub(const qd &a, const qd &b) { return a - b; }
  MD_INL static qd mul(const qd &a, const qd &b) { return a * b; }
  MD_INL static qd div(const qd &a, const qd &b) { return a / b; }
  MD_INL static qd sqrt(const qd &a) { return md::sqrt(a); }
  MD_INL static qd neg(const qd &a) { return -a; }
};
template <> struct real_traits<od> {
  static const int limbs = 8;
  MD_INL static od zero() { return mko(0.0); }
  MD_INL static od one() { return mko(1.0); }
  MD_INL static od from(double a) { return mko(a); }
  MD_INL static od add(const od &a, const od &b) { return a + b; }
  MD_INL static od sub(const od &a, const od &b) { return a - b; }
  MD_INL static od mul(const od &a, const od &b) { return a * b; }
  MD_INL static od div(const od &a, const od &b) { return a / b; }
  MD_INL static od neg(const od &a) { return -a; }
};

// ------------------------------------------------------------- complex
template <class R> struct cx {
  R re, im;
};

// Real or complex number in precision R, with the operations the kernels
// use.  num<R, false> is R itself; num<R, true> is cx<R>.
template <class R, bool C> struct num;

template <class R> struct num<R, false> {
  typedef R T;
  typedef R real;
  static const bool is_complex = false;
  typedef real_traits<R> tr;
  static const int width = tr::limbs;
  MD_INL static T zero() { return tr::zero(); }
  MD_INL static T one() { return tr::one(); }
  MD_INL static T from(double a) { return tr::from(a); }
  MD_INL static T add(const T &a, const T &b) { return tr::add(a, b); }
  MD_INL static T sub(const T &a, const T &b) { return tr::sub(a, b); }
  MD_INL static T mul(const T &a, const T &b) { return tr::mul(a, b); }
  MD_INL static T neg(const T &a) { return tr::neg(a); }
  MD_INL static T conj(const T &a) { return a; }
  MD_INL static T scale(const T &a, const R &b) { return tr::mul(a, b); }
  MD_INL static T scale_d(const T &a, double b) { return md::mul_d(a, b); }
  MD_INL static R norm2(const T &a) { return tr::mul(a, a); }
  MD_INL static T div(const T &a, const T &b) { return tr::div(a, b); }
  MD_INL static double lead(const T &a) { return fabs(md::lead(a)); }
  MD_INL static double mag(const T &a) { return fabs(md::lead(a)); }
  MD_INL static double re_lead(const T &a) { return md::lead(a); }
};

template <class R> struct num<R, true> {
  typedef cx<R> T;
  typedef R real;
  static const bool is_complex = true;
  typedef real_traits<R> tr;
  static const int width = 2 * tr::limbs;
  MD_INL static T mkc(const R &a, const R &b) { T r; r.re = a; r.im = b; return r; }
  MD_INL static T zero() { return mkc(tr::zero(), tr::zero()); }
  MD_INL static T one() { return mkc(tr::one(), tr::zero()); }
  MD_INL static T from(double a) { return mkc(tr::from(a), tr::zero()); }
  MD_INL static T add(const T &a, const T &b) { return mkc(tr::add(a.re, b.re), tr::add(a.im, b.im)); }
  MD_INL static T sub(const T &a, const T &b) { return mkc(tr::sub(a.re, b.re), tr::sub(a.im, b.im)); }
  MD_INL static T mul(const T &a, const T &b) {
    return mkc(tr::sub(tr::mul(a.re, b.re), tr::mul(a.im, b.im)), tr::add(tr::mul(a.im, b.re), tr::mul(a.re, b.im)));
  }
  MD_INL static T neg(const T &a) { return mkc(tr::neg(a.re), tr::neg(a.im)); }
  MD_INL static T conj(const T &a) { return mkc(a.re, tr::neg(a.im)); }
  MD_INL static T scale(const T &a, const R &b) { return mkc(tr::mul(a.re, b), tr::mul(a.im, b)); }
  MD_INL static T scale_d(const T &a, double b) { return mkc(md::mul_d(a.re, b), md::mul_d(a.im, b)); }
  MD_INL static R norm2(const T &a) { return tr::add(tr::mul(a.re, a.re), tr::mul(a.im, a.im)); }
  MD_INL static T div(const T &a, const T &b) {
    R d = norm2(b);
    T n = mul(a, conj(b));
    return mkc(tr::div(n.re, d), tr::div(n.im, d));
  }
  // |re| + |im| of the leading limbs, the 1-norm PHCpack uses in its skip
  // rules (Newton/dbl_onenorms_host.cpp:20)
  MD_INL static double lead(const T &a) { return fabs(md::lead(a.re)) + fabs(md::lead(a.im)); }
  MD_INL static double mag(const T &a) { return hypot(md::lead(a.re), md::lead(a.im)); }
  MD_INL static double re_lead(const T &a) { return md::lead(a.re); }
};

// ------------------------------------------------------------- memory
// A number of width W doubles is moved as W/2 double2 (W even) or one double.
MD_INL void ldr(const double *p, double &a) { a = p[0]; }
MD_INL void ldr(const double *p, dd &a) {
  double2 v = *reinterpret_cast<const double2 *>(p);
  a.hi = v.x; a.lo = v.y;
}
MD_INL void ldr(const double *p, qd &a) {
  double2 v0 = reinterpret_cast<const double2 *>(p)[0];
  double2 v1 = reinterpret_cast<const double2 *>(p)[1];
  a.x[0] = v0.x; a.x[1] = v0.y; a.x[2] = v1.x; a.x[3] = v1.y;
}
MD_INL void str(double *p, const double &a) { p[0] = a; }
MD_INL void str(double *p, const dd &a) { *reinterpret_cast<double2 *>(p) = make_double2(a.hi, a.lo); }
MD_INL void str(double *p, const qd &a) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(a.x[0], a.x[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(a.x[2], a.x[3]);
}
MD_INL void ldr(const double *p, od &a) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double2 v = reinterpret_cast<const double2 *>(p)[i];
    a.x[2 * i] = v.x;
    a.x[2 * i + 1] = v.y;
  }
}
MD_INL void str(double *p, const od &a) {
#pragma unroll
  for (int i = 0; i < 4; ++i) reinterpret_cast<double2 *>(p)[i] = make_double2(a.x[2 * i], a.x[2 * i + 1]);
}
template <class R> MD_INL void ldn(const double *p, R &a) { ldr(p, a); }
template <class R> MD_INL void ldn(const double *p, cx<R> &a) {
  ldr(p, a.re);
  ldr(p + real_traits<R>::limbs, a.im);
}
template <class R> MD_INL void stn(double *p, const R &a) { str(p, a); }
template <class R> MD_INL void stn(double *p, const cx<R> &a) {
  str(p, a.re);
  str(p + real_traits<R>::limbs, a.im);
}

// warp shuffles of whole numbers
MD_INL double shfl_xor(double a, int m) { return __shfl_xor_sync(0xffffffffu, a, m); }
MD_INL dd shfl_xor(dd a, int m) { return mk(shfl_xor(a.hi, m), shfl_xor(a.lo, m)); }
MD_INL qd shfl_xor(const qd &a, int m) {
  return mkq(shfl_xor(a.x[0], m), shfl_xor(a.x[1], m), shfl_xor(a.x[2], m), shfl_xor(a.x[3], m));
}
MD_INL od shfl_xor(const od &a, int m) {
  od r;
#pragma unroll
  for (int i = 0; i < 8; ++i) r.x[i] = shfl_xor(a.x[i], m);
  return r;
}
template <class R> MD_INL cx<R> shfl_xor(const cx<R> &a, int m) {
  cx<R> r;
  r.re = shfl_xor(a.re, m);
  r.im = shfl_xor(a.im, m);
  return r;
}
MD_INL double shfl(double a, int src) { return __shfl_sync(0xffffffffu, a, src); }
MD_INL dd shfl(dd a, int s) { return mk(shfl(a.hi, s), shfl(a.lo, s)); }
MD_INL qd shfl(const qd &a, int s) { return mkq(shfl(a.x[0], s), shfl(a.x[1], s), shfl(a.x[2], s), shfl(a.x[3], s)); }
MD_INL od shfl(const od &a, int s) {
  od r;
#pragma unroll
  for (int i = 0; i < 8; ++i) r.x[i] = shfl(a.x[i], s);
  return r;
}
template <class R> MD_INL cx<R> shfl(const cx<R> &a, int s) {
  cx<R> r;
  r.re = shfl(a.re, s);
  r.im = shfl(a.im, s);
  return r;
}

}  // namespace md
