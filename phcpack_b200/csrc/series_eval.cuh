// series_eval.cuh -- warp-level truncated power series products and the
// monomial / polynomial evaluation-differentiation built on them.
//
// The convolution z_k = sum_{i<=k} x_i y_{k-i}, k = 0..d, is the hot loop of
// PHCpack's Convolutions and Polynomials (dbl2_convolutions_kernels.cu:92,
// dbl2_polynomials_kernels.cu:25), where one thread owns one coefficient and
// thread k does k+1 of the d+1 padded steps.  Here one warp computes one
// product: coefficients k and d-k are paired (together d+2 terms), and the
// two lanes of a pair split those terms in halves, so every lane does
// ceil((d+2)/2) steps; one shuffle exchange adds the halves.  Series live
// in shared memory, limb-interleaved.
#pragma once
#include "md.cuh"

namespace phc {

// lane mapping of a degree-deg product, deg+1 <= 32
struct lanemap {
  int p, h, k1, k2, t0, t1, partner, steps;
  bool valid;  // this lane owns output coefficient kout()
  __device__ __forceinline__ lanemap(int deg, int lane) {
    const int n1 = deg + 1;
    const int np = (n1 + 1) >> 1;
    const bool active = lane < 2 * np;
    p = active ? lane % np : 0;
    h = active ? lane / np : 0;
    k1 = p;
    k2 = deg - p;
    const int nt = (k1 == k2) ? (p + 1) : (deg + 2);
    const int half = (nt + 1) >> 1;
    t0 = (h == 0) ? 0 : half;
    t1 = (h == 0) ? half : nt;
    if (!active) t0 = t1 = 0;
    partner = active ? (h == 0 ? lane + np : lane - np) : lane;
    steps = ((deg + 2) + 1) >> 1;
    valid = active && !(h == 1 && k1 == k2);
  }
  __device__ __forceinline__ int kout() const { return h == 0 ? k1 : k2; }
};

template <class N>
struct wser {
  typedef typename N::T T;
  static const int W = N::width;

  // z = x*y (x, y series in shared memory); returns the coefficient this
  // lane owns (m.valid) at index m.kout().  All 32 lanes must call it.
  // Compiled once and called (not inlined at its many call sites): the
  // evaluation kernel is bound by instruction fetch when every call site
  // carries its own copy of the loop.
  static __device__ __noinline__ T conv(const double *x, const double *y, const lanemap &m) {
    T a1 = N::zero(), a2 = N::zero();
    for (int s = 0; s < m.steps; ++s) {
      const int t = m.t0 + s;
      if (t < m.t1) {
        const bool first = (t <= m.p);
        const int i = first ? t : t - (m.p + 1);
        const int j = (first ? m.k1 : m.k2) - i;
        T xi, yj;
        md::ldn(x + i * W, xi);
        md::ldn(y + j * W, yj);
        const T pr = N::mul(xi, yj);
        T a = first ? a1 : a2;
        a = N::add(a, pr);
        if (first) a1 = a; else a2 = a;
      }
    }
    const T o1 = md::shfl(a1, m.partner);
    const T o2 = md::shfl(a2, m.partner);
    return (m.h == 0) ? N::add(a1, o1) : N::add(a2, o2);
  }

  // dst[k] = z (shared memory), then make it visible to the warp
  static __device__ __forceinline__ void put(double *dst, const T &z, const lanemap &m) {
    if (m.valid) md::stn(dst + m.kout() * W, z);
    __syncwarp();
  }
  static __device__ __forceinline__ void prod(const double *x, const double *y, double *z, const lanemap &m) {
    const T r = conv(x, y, m);
    __syncwarp();  // z may alias a buffer other lanes still read
    put(z, r, m);
  }
  // row[k] += e*z in global memory (lane-owned coefficient); the first
  // contribution to a row (first == true) is stored without reading it
  static __device__ __forceinline__ void acc_global(double *row, const T &z, const lanemap &m, int e, bool first) {
    if (m.valid) {
      const T zz = (e > 1) ? N::scale_d(z, (double)e) : z;
      if (first) {
        md::stn(row + m.kout() * W, zz);
      } else {
        T v;
        md::ldn(row + m.kout() * W, v);
        md::stn(row + m.kout() * W, N::add(v, zz));
      }
    }
  }
  // row[k] += e*src[k] for a series src in shared memory, lane k
  static __device__ __forceinline__ void acc_series(double *row, const double *src, int n1, int e, bool first) {
    const int lane = threadIdx.x & 31;
    if (lane < n1) {
      T z;
      md::ldn(src + lane * W, z);
      if (e > 1) z = N::scale_d(z, (double)e);
      if (first) {
        md::stn(row + lane * W, z);
      } else {
        T v;
        md::ldn(row + lane * W, v);
        md::stn(row + lane * W, N::add(v, z));
      }
    }
  }
};

// Shared-memory series slots a warp needs for monomials of up to maxvar
// variables: the coefficient, a temporary, f_0..f_{k-2}, b_0..b_{k-3}.
__host__ __device__ inline int warp_slots(int maxvar) {
  int s = 2 * maxvar - 1;
  return s < 3 ? 3 : s;
}

// Value and gradient of one polynomial of a system, accumulated by one warp
// into out (dim+1 series in global memory; row dim is the value).  The
// value is accumulated in registers (each lane its coefficients) and
// written once.  A gradient row is stored at its first contribution and
// read, added to and written back only after that (a 64-bit mask records
// the rows 0..63 written so far; rows from 64 on are zeroed first and
// always accumulated); rows no monomial reached are zeroed at the end.
//
// Per monomial: the common-factor method of Newton/dbl2_systems_host.cpp:
// 18-110 (coefficient <- x^(e-1) * coefficient, derivative j scaled by e_j),
// then the forward/backward/cross products of
// Convolutions/dbl2_monomials_host.cpp:4-22 (CPU_dbl2_evaldiff, :175).
template <class N>
__device__ void warp_poly_evaldiff(int dim, int deg, int maxvar, int m0, int m1, const int *__restrict__ nvr,
                                   const int *__restrict__ idx, const int *__restrict__ exps,
                                   const double *__restrict__ cst, const double *__restrict__ cff,
                                   const double *X,  // shared: dim series
                                   double *scr,      // shared: warp_slots(maxvar) series
                                   double *out) {
  typedef typename N::T T;
  const int W = N::width;
  const int n1 = deg + 1;
  const int S = n1 * W;  // doubles per series
  const int lane = threadIdx.x & 31;
  const lanemap m(deg, lane);
  typedef wser<N> ws;

  // rows past the first 64 start at zero (the mask covers rows 0..63)
  for (int r = 64; r < dim; ++r)
    if (lane < n1) md::stn(out + r * S + lane * W, N::zero());
  unsigned long long written = 0ull;  // gradient rows stored so far (uniform over the warp)
  auto first_touch = [&](int r) {
    if (r >= 64) return false;
    const bool f = !((written >> r) & 1ull);
    written |= 1ull << r;
    return f;
  };
  // the value starts at the constant series, lane-owned coefficients
  T vacc = N::zero();
  if (m.valid) md::ldn(cst + m.kout() * W, vacc);
  double *C = scr;
  double *Tm = scr + S;
  double *F = scr + 2 * S;                 // f_0 .. f_{k-2}
  double *B = scr + (1 + maxvar) * S;      // b_0 .. b_{k-3}

  for (int mon = m0; mon < m1; ++mon) {
    const int k = nvr[mon];
    const int *ix = idx + mon * maxvar;
    const int *ex = exps + mon * maxvar;
    // a malformed monomial (variable count, index or exponent out of range)
    // is skipped rather than read out of bounds; the host entry points
    // reject such supports before any launch
    bool ok = (k >= 1 && k <= maxvar);
    for (int v = 0; ok && v < k; ++v) ok = (ix[v] >= 0 && ix[v] < dim && ex[v] >= 1);
    if (!ok) continue;
    if (lane < n1) {
      T c;
      md::ldn(cff + (long)mon * S + lane * W, c);
      md::stn(C + lane * W, c);
    }
    __syncwarp();
    // common factors: C <- x_v^(e_v - 1) * C
    for (int v = 0; v < k; ++v) {
      const int e = ex[v];
      for (int r = 1; r < e; ++r) {
        ws::prod(X + ix[v] * S, C, Tm, m);
        double *t = C; C = Tm; Tm = t;
      }
    }
    if (k == 1) {
      const T z = ws::conv(X + ix[0] * S, C, m);
      if (m.valid) vacc = N::add(vacc, z);
      ws::acc_series(out + ix[0] * S, C, n1, ex[0], first_touch(ix[0]));
    } else if (k == 2) {
      ws::prod(X + ix[0] * S, X + ix[1] * S, Tm, m);
      T z = ws::conv(Tm, C, m);
      if (m.valid) vacc = N::add(vacc, z);
      z = ws::conv(C, X + ix[0] * S, m);
      ws::acc_global(out + ix[1] * S, z, m, ex[1], first_touch(ix[1]));
      z = ws::conv(C, X + ix[1] * S, m);
      ws::acc_global(out + ix[0] * S, z, m, ex[0], first_touch(ix[0]));
    } else {
      // forward products f_i = f_{i-1} x_i, f_0 = c x_0
      ws::prod(C, X + ix[0] * S, F, m);
      for (int i = 1; i < k - 1; ++i) ws::prod(F + (i - 1) * S, X + ix[i] * S, F + i * S, m);
      T z = ws::conv(F + (k - 2) * S, X + ix[k - 1] * S, m);
      if (m.valid) vacc = N::add(vacc, z);
      ws::acc_series(out + ix[k - 1] * S, F + (k - 2) * S, n1, ex[k - 1], first_touch(ix[k - 1]));
      // backward products b_0 = x_{k-1} x_{k-2}, b_i = b_{i-1} x_{k-2-i}
      ws::prod(X + ix[k - 1] * S, X + ix[k - 2] * S, B, m);
      for (int i = 1; i < k - 2; ++i) ws::prod(B + (i - 1) * S, X + ix[k - 2 - i] * S, B + i * S, m);
      // b_{k-3} <- b_{k-3} * c : derivative in x_0
      z = ws::conv(B + (k - 3) * S, C, m);
      __syncwarp();
      ws::put(B + (k - 3) * S, z, m);
      ws::acc_series(out + ix[0] * S, B + (k - 3) * S, n1, ex[0], first_touch(ix[0]));
      // cross products: derivative in x_j, 1 <= j <= k-2
      if (k == 3) {
        z = ws::conv(F, X + ix[2] * S, m);
        ws::acc_global(out + ix[1] * S, z, m, ex[1], first_touch(ix[1]));
      } else {
        for (int i = 0; i < k - 3; ++i) {
          z = ws::conv(F + i * S, B + (k - 4 - i) * S, m);
          ws::acc_global(out + ix[i + 1] * S, z, m, ex[i + 1], first_touch(ix[i + 1]));
        }
        z = ws::conv(F + (k - 3) * S, X + ix[k - 1] * S, m);
        ws::acc_global(out + ix[k - 2] * S, z, m, ex[k - 2], first_touch(ix[k - 2]));
      }
    }
    __syncwarp();
  }
  // the value, and zeros in the rows no monomial reached
  if (m.valid) md::stn(out + dim * S + m.kout() * W, vacc);
  for (int r = 0; r < dim && r < 64; ++r)
    if (!((written >> r) & 1ull) && lane < n1) md::stn(out + r * S + lane * W, N::zero());
}

// ------------------------------------------------------- degrees 32..191
// Series longer than a warp: each lane owns the coefficients k = lane,
// lane + 32, ... of a product, each formed in the reference's order
// x_0 y_k + x_1 y_{k-1} + ... + x_k y_0 (CPU_dbl2_product,
// Convolutions/dbl2_convolutions_host.cpp:7); the lanes of a 32-coefficient
// chunk differ by at most 32 terms.  Compiled once and called.
template <class N>
__device__ __noinline__ typename N::T conv_at(const double *x, const double *y, int k) {
  typedef typename N::T T;
  const int W = N::width;
  T a = N::zero();
  for (int i = 0; i <= k; ++i) {
    T xi, yj;
    md::ldn(x + i * W, xi);
    md::ldn(y + (k - i) * W, yj);
    a = N::add(a, N::mul(xi, yj));
  }
  return a;
}

// warp_poly_evaldiff for deg + 1 > 32 coefficients: the same monomial
// method and the same outputs; the value accumulates in a series of the
// warp's scratch (slot warp_slots(maxvar)), the products go through the
// scratch coefficient by coefficient.
template <class N>
__device__ void warp_poly_evaldiff_big(int dim, int deg, int maxvar, int m0, int m1, const int *__restrict__ nvr,
                                       const int *__restrict__ idx, const int *__restrict__ exps,
                                       const double *__restrict__ cst, const double *__restrict__ cff,
                                       const double *X,  // dim series (shared memory or global)
                                       double *scr,      // shared: warp_slots(maxvar) + 1 series
                                       double *out) {
  typedef typename N::T T;
  const int W = N::width;
  const int n1 = deg + 1;
  const int S = n1 * W;
  const int lane = threadIdx.x & 31;
  for (int r = 64; r < dim; ++r)
    for (int k = lane; k < n1; k += 32) md::stn(out + r * S + k * W, N::zero());
  unsigned long long written = 0ull;
  auto first_touch = [&](int r) {
    if (r >= 64) return false;
    const bool f = !((written >> r) & 1ull);
    written |= 1ull << r;
    return f;
  };
  double *C = scr;
  double *Tm = scr + S;
  double *F = scr + 2 * S;                 // f_0 .. f_{k-2}
  double *B = scr + (1 + maxvar) * S;      // b_0 .. b_{k-3}
  double *Vs = scr + warp_slots(maxvar) * S;  // the value
  for (int k = lane; k < n1; k += 32) {
    T c;
    md::ldn(cst + k * W, c);
    md::stn(Vs + k * W, c);
  }
  // z = x y into the scratch series z (z is neither x nor y)
  auto prod = [&](const double *x, const double *y, double *z) {
    for (int k = lane; k < n1; k += 32) md::stn(z + k * W, conv_at<N>(x, y, k));
    __syncwarp();
  };
  auto add_value = [&](const double *x, const double *y) {
    for (int k = lane; k < n1; k += 32) {
      const T z = conv_at<N>(x, y, k);
      T v;
      md::ldn(Vs + k * W, v);
      md::stn(Vs + k * W, N::add(v, z));
    }
  };
  // row += e x y (global memory; the first contribution is stored)
  auto acc_prod = [&](double *row, const double *x, const double *y, int e, bool first) {
    for (int k = lane; k < n1; k += 32) {
      T z = conv_at<N>(x, y, k);
      if (e > 1) z = N::scale_d(z, (double)e);
      if (first) {
        md::stn(row + k * W, z);
      } else {
        T v;
        md::ldn(row + k * W, v);
        md::stn(row + k * W, N::add(v, z));
      }
    }
  };
  // row += e src (src a scratch series)
  auto acc_src = [&](double *row, const double *src, int e, bool first) {
    for (int k = lane; k < n1; k += 32) {
      T z;
      md::ldn(src + k * W, z);
      if (e > 1) z = N::scale_d(z, (double)e);
      if (first) {
        md::stn(row + k * W, z);
      } else {
        T v;
        md::ldn(row + k * W, v);
        md::stn(row + k * W, N::add(v, z));
      }
    }
  };

  for (int mon = m0; mon < m1; ++mon) {
    const int k = nvr[mon];
    const int *ix = idx + mon * maxvar;
    const int *ex = exps + mon * maxvar;
    bool ok = (k >= 1 && k <= maxvar);
    for (int v = 0; ok && v < k; ++v) ok = (ix[v] >= 0 && ix[v] < dim && ex[v] >= 1);
    if (!ok) continue;
    for (int c = lane; c < n1; c += 32) {
      T v;
      md::ldn(cff + (long)mon * S + c * W, v);
      md::stn(C + c * W, v);
    }
    __syncwarp();
    // common factors: C <- x_v^(e_v - 1) * C
    for (int v = 0; v < k; ++v)
      for (int r = 1; r < ex[v]; ++r) {
        prod(X + ix[v] * S, C, Tm);
        double *t = C; C = Tm; Tm = t;
      }
    if (k == 1) {
      add_value(X + ix[0] * S, C);
      acc_src(out + ix[0] * S, C, ex[0], first_touch(ix[0]));
    } else if (k == 2) {
      prod(X + ix[0] * S, X + ix[1] * S, Tm);
      add_value(Tm, C);
      acc_prod(out + ix[1] * S, C, X + ix[0] * S, ex[1], first_touch(ix[1]));
      acc_prod(out + ix[0] * S, C, X + ix[1] * S, ex[0], first_touch(ix[0]));
    } else {
      prod(C, X + ix[0] * S, F);
      for (int i = 1; i < k - 1; ++i) prod(F + (i - 1) * S, X + ix[i] * S, F + i * S);
      add_value(F + (k - 2) * S, X + ix[k - 1] * S);
      acc_src(out + ix[k - 1] * S, F + (k - 2) * S, ex[k - 1], first_touch(ix[k - 1]));
      prod(X + ix[k - 1] * S, X + ix[k - 2] * S, B);
      for (int i = 1; i < k - 2; ++i) prod(B + (i - 1) * S, X + ix[k - 2 - i] * S, B + i * S);
      prod(B + (k - 3) * S, C, Tm);  // b_{k-3} c: the derivative in x_0
      acc_src(out + ix[0] * S, Tm, ex[0], first_touch(ix[0]));
      if (k == 3) {
        acc_prod(out + ix[1] * S, F, X + ix[2] * S, ex[1], first_touch(ix[1]));
      } else {
        for (int i = 0; i < k - 3; ++i)
          acc_prod(out + ix[i + 1] * S, F + i * S, B + (k - 4 - i) * S, ex[i + 1], first_touch(ix[i + 1]));
        acc_prod(out + ix[k - 2] * S, F + (k - 3) * S, X + ix[k - 1] * S, ex[k - 2], first_touch(ix[k - 2]));
      }
    }
    __syncwarp();
  }
  for (int k = lane; k < n1; k += 32) {
    T v;
    md::ldn(Vs + k * W, v);
    md::stn(out + dim * S + k * W, v);
  }
  for (int r = 0; r < dim && r < 64; ++r)
    if (!((written >> r) & 1ull))
      for (int k = lane; k < n1; k += 32) md::stn(out + r * S + k * W, N::zero());
}

}  // namespace phc
