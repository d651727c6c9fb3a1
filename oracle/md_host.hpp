// md_host.hpp -- host multiple-double arithmetic for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  This header belongs to the oracle: it is the
// checker that the CUDA path is compared against, never the product.
//
// Number formats follow PHCpack's src/GPU/Norms conventions:
//   dd = (hi, lo)                  -- double_double_functions.cpp
//   qd = (hihi, lohi, hilo, lolo)  -- quad_double_functions.cpp
// stored limb-interleaved in memory (limb 0 first, decreasing significance).
//
// Algorithms are the published error-free transformations:
//   two_sum (Knuth), quick_two_sum (Dekker), two_prod by one fused
//   multiply-add (exact, so it agrees in value with the Dekker split that
//   Norms/double_double_functions.cpp:158-193 uses);
//   dd add/mul/div/sqrt of Hida, Li and Bailey's QD library
//   (double_double_functions.cpp:24-260);
//   qd add/mul as the limb-by-limb accumulation with a final
//   renormalisation that CAMPARY calls baileyAdd_fast / baileyMul_fast
//   (quad_double_functions.cpp:209,313), written here as loops.
// Compile with -ffp-contract=off: the transformations are only exact when
// the compiler does not fuse or reassociate.
#pragma once
#include <cmath>

namespace orc {

static inline double two_sum(double a, double b, double *e) {
  double s = a + b;
  double bb = s - a;
  *e = (a - (s - bb)) + (b - bb);
  return s;
}
static inline double quick_two_sum(double a, double b, double *e) {
  double s = a + b;
  *e = b - (s - a);
  return s;
}
static inline double two_diff(double a, double b, double *e) {
  double s = a - b;
  double bb = s - a;
  *e = (a - (s - bb)) - (b + bb);
  return s;
}
static inline double two_prod(double a, double b, double *e) {
  double p = a * b;
  *e = std::fma(a, b, -p);
  return p;
}

// ---------------------------------------------------------------- dd
struct dd {
  double hi, lo;
  dd() : hi(0.0), lo(0.0) {}
  dd(double h) : hi(h), lo(0.0) {}
  dd(double h, double l) : hi(h), lo(l) {}
};

static inline dd operator+(const dd &a, const dd &b) {
  double s2, t2;
  double s1 = two_sum(a.hi, b.hi, &s2);
  double t1 = two_sum(a.lo, b.lo, &t2);
  s2 += t1;
  s1 = quick_two_sum(s1, s2, &s2);
  s2 += t2;
  double lo;
  double hi = quick_two_sum(s1, s2, &lo);
  return dd(hi, lo);
}
static inline dd operator-(const dd &a) { return dd(-a.hi, -a.lo); }
static inline dd operator-(const dd &a, const dd &b) { return a + (-b); }
static inline dd operator*(const dd &a, const dd &b) {
  double p2;
  double p1 = two_prod(a.hi, b.hi, &p2);
  p2 += (a.hi * b.lo + a.lo * b.hi);
  double lo;
  double hi = quick_two_sum(p1, p2, &lo);
  return dd(hi, lo);
}
static inline dd mul_d(const dd &a, double b) {
  double p2;
  double p1 = two_prod(a.hi, b, &p2);
  p2 += a.lo * b;
  double lo;
  double hi = quick_two_sum(p1, p2, &lo);
  return dd(hi, lo);
}
static inline dd operator/(const dd &a, const dd &b) {
  double q1 = a.hi / b.hi;
  dd r = a - mul_d(b, q1);
  double q2 = r.hi / b.hi;
  r = r - mul_d(b, q2);
  double q3 = r.hi / b.hi;
  double lo;
  double hi = quick_two_sum(q1, q2, &lo);
  return dd(hi, lo) + dd(q3);
}
static inline dd sqrt(const dd &a) {
  if (a.hi == 0.0 && a.lo == 0.0) return dd(0.0);
  if (a.hi < 0.0) return dd(-1.0);  // same sentinel as the reference
  double x = 1.0 / std::sqrt(a.hi);
  double ax = a.hi * x;
  dd y = a - dd(ax) * dd(ax);
  double lo;
  double hi = two_sum(ax, y.hi * x * 0.5, &lo);
  return dd(hi, lo);
}
static inline double to_double(const dd &a) { return a.hi + a.lo; }
static inline double lead(const dd &a) { return a.hi; }
static inline bool is_zero(const dd &a) { return a.hi == 0.0 && a.lo == 0.0; }
static inline dd abs(const dd &a) { return a.hi < 0.0 ? -a : a; }

// ---------------------------------------------------------------- qd
struct qd {
  double x[4];
  qd() { x[0] = x[1] = x[2] = x[3] = 0.0; }
  qd(double a) { x[0] = a; x[1] = x[2] = x[3] = 0.0; }
  qd(double a, double b, double c, double d) { x[0] = a; x[1] = b; x[2] = c; x[3] = d; }
  qd(const dd &a) { x[0] = a.hi; x[1] = a.lo; x[2] = x[3] = 0.0; }
};

// Renormalise five overlapping terms f[0..4] (decreasing magnitude) into a
// non-overlapping four-term expansion: a bottom-up quick_two_sum pass,
// then a top-down pass that keeps only non-zero components
// (quad_double_functions.cpp:11-150, written as a loop).
static inline qd renorm5(const double *in) {
  double f[5];
  double s = in[4];
  for (int i = 3; i >= 0; --i) s = quick_two_sum(in[i], s, &f[i + 1]);
  f[0] = s;
  double r[4] = {0.0, 0.0, 0.0, 0.0};
  int k = 0;
  double acc = f[0];
  for (int i = 1; i <= 4 && k < 4; ++i) {
    double e;
    double t = quick_two_sum(acc, f[i], &e);
    if (e != 0.0) {
      r[k++] = t;
      acc = e;
    } else {
      acc = t;
    }
  }
  if (k < 4 && acc != 0.0) r[k++] = acc;
  return qd(r[0], r[1], r[2], r[3]);
}

// add `v` into f[lvl..3], carrying each rounding error to the next level
// and dropping the final error into f[4]
static inline void accumulate(double *f, int lvl, double v) {
  for (int j = lvl; j < 4; ++j) f[j] = two_sum(f[j], v, &v);
  f[4] += v;
}

static inline qd operator+(const qd &a, const qd &b) {
  double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int k = 3; k >= 0; --k) {
    double e;
    f[k] = two_sum(a.x[k], b.x[k], &e);
    accumulate(f, k + 1, e);
  }
  return renorm5(f);
}
static inline qd operator-(const qd &a) { return qd(-a.x[0], -a.x[1], -a.x[2], -a.x[3]); }
static inline qd operator-(const qd &a, const qd &b) { return a + (-b); }
static inline qd operator*(const qd &a, const qd &b) {
  double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  f[4] = a.x[1] * b.x[3] + a.x[2] * b.x[2] + a.x[3] * b.x[1];
  for (int k = 3; k >= 0; --k) {
    for (int i = 0; i <= k; ++i) {
      double e;
      double p = two_prod(a.x[i], b.x[k - i], &e);
      accumulate(f, k + 1 <= 4 ? k + 1 : 4, e);
      accumulate(f, k, p);
    }
  }
  return renorm5(f);
}
static inline qd mul_d(const qd &a, double b) {
  double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int k = 3; k >= 0; --k) {
    double e;
    double p = two_prod(a.x[k], b, &e);
    accumulate(f, k + 1, e);
    accumulate(f, k, p);
  }
  return renorm5(f);
}
static inline qd operator/(const qd &a, const qd &b) {
  double q[5];
  qd r = a;
  for (int i = 0; i < 4; ++i) {
    q[i] = r.x[0] / b.x[0];
    r = r - mul_d(b, q[i]);
  }
  q[4] = r.x[0] / b.x[0];
  return renorm5(q);
}
static inline qd sqrt(const qd &a) {
  if (a.x[0] == 0.0 && a.x[1] == 0.0 && a.x[2] == 0.0 && a.x[3] == 0.0) return qd(0.0);
  if (a.x[0] < 0.0) return qd(-1.0);
  dd s = sqrt(dd(a.x[0], a.x[1]));
  qd b(s);
  // one Newton step: (b^2 + a) / (2 b)
  qd z = b * b + a;
  z = z / b;
  return qd(z.x[0] * 0.5, z.x[1] * 0.5, z.x[2] * 0.5, z.x[3] * 0.5);
}
static inline double to_double(const qd &a) { return a.x[0] + a.x[1]; }
static inline double lead(const qd &a) { return a.x[0]; }
static inline bool is_zero(const qd &a) { return a.x[0] == 0.0 && a.x[1] == 0.0 && a.x[2] == 0.0 && a.x[3] == 0.0; }
static inline qd abs(const qd &a) { return a.x[0] < 0.0 ? -a : a; }

// ---------------------------------------------------------------- od
// Octo-double: the qd scheme above on eight limbs (nine accumulators, the
// order-8 products summed plainly), the scheme of the reference's
// octo-doubles (odf_add, odf_mul, odf_mul_od_d, odf_div and odf_fast_renorm
// of Norms/octo_double_functions.cpp, CAMPARY's baileyAdd/Mul_fast<8,8,8>)
// written as loops.  The device code (phcpack_b200/csrc/md.cuh) sums the
// order-8 products by fused multiply-adds.
struct od {
  double x[8];
  od() { for (int i = 0; i < 8; ++i) x[i] = 0.0; }
  od(double a) { x[0] = a; for (int i = 1; i < 8; ++i) x[i] = 0.0; }
  od(const dd &a) { x[0] = a.hi; x[1] = a.lo; for (int i = 2; i < 8; ++i) x[i] = 0.0; }
  od(const qd &a) { for (int i = 0; i < 4; ++i) x[i] = a.x[i]; for (int i = 4; i < 8; ++i) x[i] = 0.0; }
};

static inline od renorm9(const double *in) {
  double f[9];
  double s = in[8];
  for (int i = 7; i >= 0; --i) s = quick_two_sum(in[i], s, &f[i + 1]);
  f[0] = s;
  od r;
  int k = 0;
  double acc = f[0];
  for (int i = 1; i <= 8; ++i) {
    double e;
    const double t = quick_two_sum(acc, f[i], &e);
    if (e != 0.0 && k < 8) {
      r.x[k++] = t;
      acc = e;
    } else {
      acc = t;
    }
  }
  if (k < 8 && acc != 0.0) r.x[k] = acc;
  return r;
}

static inline void accumulate9(double *f, int lvl, double v) {
  for (int j = lvl; j < 8; ++j) f[j] = two_sum(f[j], v, &v);
  f[8] += v;
}

static inline od operator+(const od &a, const od &b) {
  double f[9] = {0.0};
  for (int k = 7; k >= 0; --k) {
    double e;
    f[k] = two_sum(a.x[k], b.x[k], &e);
    accumulate9(f, k + 1, e);
  }
  return renorm9(f);
}
static inline od operator-(const od &a) {
  od r;
  for (int i = 0; i < 8; ++i) r.x[i] = -a.x[i];
  return r;
}
static inline od operator-(const od &a, const od &b) { return a + (-b); }
static inline od operator*(const od &a, const od &b) {
  double f[9] = {0.0};
  f[8] = a.x[1] * b.x[7];
  for (int i = 2; i < 8; ++i) f[8] += a.x[i] * b.x[8 - i];
  for (int k = 7; k >= 0; --k)
    for (int i = 0; i <= k; ++i) {
      double e;
      const double p = two_prod(a.x[i], b.x[k - i], &e);
      accumulate9(f, k + 1, e);
      accumulate9(f, k, p);
    }
  return renorm9(f);
}
static inline od mul_d(const od &a, double b) {
  double f[9] = {0.0};
  for (int k = 7; k >= 0; --k) {
    double e;
    f[k] = two_prod(a.x[k], b, &e);
    accumulate9(f, k + 1, e);
  }
  return renorm9(f);
}
static inline od operator/(const od &a, const od &b) {
  double q[9];
  od r = a;
  for (int i = 0; i < 9; ++i) {
    q[i] = r.x[0] / b.x[0];
    if (i < 8) r = r - mul_d(b, q[i]);
  }
  return renorm9(q);
}
static inline double to_double(const od &a) { return a.x[0] + a.x[1]; }
static inline double lead(const od &a) { return a.x[0]; }
static inline bool is_zero(const od &a) {
  for (int i = 0; i < 8; ++i)
    if (a.x[i] != 0.0) return false;
  return true;
}
static inline od abs(const od &a) { return a.x[0] < 0.0 ? -a : a; }

// ------------------------------------------------------- plain double
static inline double sqrt(double a) { return std::sqrt(a); }
static inline double abs(double a) { return std::fabs(a); }
static inline double mul_d(double a, double b) { return a * b; }
static inline double to_double(double a) { return a; }
static inline double lead(double a) { return a; }
static inline bool is_zero(double a) { return a == 0.0; }

// ------------------------------------------------------- limbs
template <class R> struct limbs;
template <> struct limbs<double> { static const int n = 1; };
template <> struct limbs<dd> { static const int n = 2; };
template <> struct limbs<qd> { static const int n = 4; };
template <> struct limbs<od> { static const int n = 8; };

static inline void load(const double *p, double &a) { a = p[0]; }
static inline void load(const double *p, dd &a) { a.hi = p[0]; a.lo = p[1]; }
static inline void load(const double *p, qd &a) { for (int i = 0; i < 4; ++i) a.x[i] = p[i]; }
static inline void load(const double *p, od &a) { for (int i = 0; i < 8; ++i) a.x[i] = p[i]; }
static inline void store(double *p, const double &a) { p[0] = a; }
static inline void store(double *p, const dd &a) { p[0] = a.hi; p[1] = a.lo; }
static inline void store(double *p, const qd &a) { for (int i = 0; i < 4; ++i) p[i] = a.x[i]; }
static inline void store(double *p, const od &a) { for (int i = 0; i < 8; ++i) p[i] = a.x[i]; }

// ------------------------------------------------------- complex
template <class R> struct cx {
  R re, im;
  cx() : re(0.0), im(0.0) {}
  cx(const R &r) : re(r), im(0.0) {}
  cx(const R &r, const R &i) : re(r), im(i) {}
};
template <class R> static inline cx<R> operator+(const cx<R> &a, const cx<R> &b) { return cx<R>(a.re + b.re, a.im + b.im); }
template <class R> static inline cx<R> operator-(const cx<R> &a, const cx<R> &b) { return cx<R>(a.re - b.re, a.im - b.im); }
template <class R> static inline cx<R> operator-(const cx<R> &a) { return cx<R>(-a.re, -a.im); }
template <class R> static inline cx<R> operator*(const cx<R> &a, const cx<R> &b) {
  return cx<R>(a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im);
}
template <class R> static inline cx<R> conj(const cx<R> &a) { return cx<R>(a.re, -a.im); }
template <class R> static inline cx<R> mul_d(const cx<R> &a, double b) { return cx<R>(mul_d(a.re, b), mul_d(a.im, b)); }
template <class R> static inline R norm2(const cx<R> &a) { return a.re * a.re + a.im * a.im; }
template <class R> static inline cx<R> operator/(const cx<R> &a, const cx<R> &b) {
  R d = norm2(b);
  cx<R> n = a * conj(b);
  return cx<R>(n.re / d, n.im / d);
}
template <class R> static inline double lead(const cx<R> &a) { return std::fabs(lead(a.re)) + std::fabs(lead(a.im)); }
template <class R> static inline bool is_zero(const cx<R> &a) { return is_zero(a.re) && is_zero(a.im); }

template <class R> struct limbs<cx<R> > { static const int n = 2 * limbs<R>::n; };
template <class R> static inline void load(const double *p, cx<R> &a) { load(p, a.re); load(p + limbs<R>::n, a.im); }
template <class R> static inline void store(double *p, const cx<R> &a) { store(p, a.re); store(p + limbs<R>::n, a.im); }

// scalar traits used by the templated algorithms
template <class T> struct real_of { typedef T type; };
template <class R> struct real_of<cx<R> > { typedef R type; };
template <class T> struct is_cx { static const bool v = false; };
template <class R> struct is_cx<cx<R> > { static const bool v = true; };

static inline double conj(double a) { return a; }
static inline dd conj(const dd &a) { return a; }
static inline qd conj(const qd &a) { return a; }
static inline od conj(const od &a) { return a; }
static inline double norm2(double a) { return a * a; }
static inline dd norm2(const dd &a) { return a * a; }
static inline qd norm2(const qd &a) { return a * a; }
static inline od norm2(const od &a) { return a * a; }

}  // namespace orc
