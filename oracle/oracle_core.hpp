// oracle_core.hpp -- templated CPU restatement of PHCpack's multiple-double
// power-series hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker the CUDA kernels are compared
// against.  Nothing in the product links or calls this code.
//
// Every routine cites the reference routine whose arithmetic it restates
// (paths relative to PHCpack's src/GPU).  T is the scalar type: double, dd,
// qd or cx<...> of those.  Arrays are flat and limb-interleaved: a series of
// degree d is (d+1) consecutive numbers, each limbs<T>::n doubles.
#pragma once
#include <vector>
#include <cstring>
#include "md_host.hpp"

namespace orc {

template <class T> static inline T ld(const double *p, long i) {
  T a;
  load(p + i * limbs<T>::n, a);
  return a;
}
template <class T> static inline void st(double *p, long i, const T &a) { store(p + i * limbs<T>::n, a); }

// z = x*y truncated at degree deg.
// Convolutions/dbl2_convolutions_host.cpp:7 (CPU_dbl2_product): z[k] starts
// at x[0]*y[k] and accumulates x[i]*y[k-i] for i = 1..k.
template <class T> static void conv(int deg, const T *x, const T *y, T *z) {
  for (int k = 0; k <= deg; ++k) {
    T acc = x[0] * y[k];
    for (int i = 1; i <= k; ++i) acc = acc + x[i] * y[k - i];
    z[k] = acc;
  }
}

// Value and gradient of cff * x[idx[0]] * ... * x[idx[nvr-1]] (distinct
// variables), by forward, backward and cross products.
// Convolutions/dbl2_monomials_host.cpp:4-22 (algorithm), :28 (CPU_dbl2_speel)
// and :175 (CPU_dbl2_evaldiff).  out[v] receives the derivative series with
// respect to variable idx[v] (v < nvr) and out[nvr] the value.
template <class T>
static void monomial_evaldiff(int nvr, int deg, const int *idx, const T *cff,
                              const std::vector<const T *> &x, std::vector<std::vector<T> > &out) {
  const int n1 = deg + 1;
  for (int v = 0; v <= nvr; ++v) out[v].assign(n1, T());
  if (nvr == 1) {
    conv(deg, x[idx[0]], cff, out[1].data());
    for (int i = 0; i < n1; ++i) out[0][i] = cff[i];
    return;
  }
  if (nvr == 2) {
    std::vector<T> t(n1);
    conv(deg, x[idx[0]], x[idx[1]], t.data());
    conv(deg, t.data(), cff, out[2].data());
    conv(deg, cff, x[idx[0]], out[1].data());
    conv(deg, cff, x[idx[1]], out[0].data());
    return;
  }
  std::vector<std::vector<T> > f(nvr, std::vector<T>(n1)), b(nvr - 2, std::vector<T>(n1)),
      c(nvr - 2, std::vector<T>(n1));
  conv(deg, cff, x[idx[0]], f[0].data());
  for (int i = 1; i < nvr; ++i) conv(deg, f[i - 1].data(), x[idx[i]], f[i].data());
  conv(deg, x[idx[nvr - 1]], x[idx[nvr - 2]], b[0].data());
  for (int i = 1; i < nvr - 2; ++i) conv(deg, b[i - 1].data(), x[idx[nvr - 2 - i]], b[i].data());
  {
    std::vector<T> t(n1);
    conv(deg, b[nvr - 3].data(), cff, t.data());
    b[nvr - 3] = t;
  }
  if (nvr == 3) {
    conv(deg, f[0].data(), x[idx[2]], c[0].data());
  } else {
    for (int i = 0; i < nvr - 3; ++i) conv(deg, f[i].data(), b[nvr - 4 - i].data(), c[i].data());
    conv(deg, f[nvr - 3].data(), x[idx[nvr - 1]], c[nvr - 3].data());
  }
  out[nvr] = f[nvr - 1];
  out[nvr - 1] = f[nvr - 2];
  out[0] = b[nvr - 3];
  for (int k = 1; k < nvr - 1; ++k) out[k] = c[k - 1];
}

// One polynomial p = cst + sum_m cff_m * prod_j x[idx_mj]^exp_mj at a
// vector of series.  Exponents > 1 use the common-factor method of
// Newton/dbl2_systems_host.cpp:18-110: cff <- x^(e-1) * cff by repeated
// series products, the distinct-variable monomial evaluation above, then
// derivative j scaled by e_j.  Monomials are accumulated as in
// Polynomials/dbl2_polynomials_host.cpp:259 (CPU_dbl2_poly_evaldiff):
// output row dim starts at cst, rows 0..dim-1 at zero.
// out: (dim+1) series, row `dim` the value, row j the derivative in x_j.
template <class T>
static void poly_evaldiff(int dim, int deg, int nbr, const int *nvr, const int *idx, const int *exps,
                          int maxvar, const T *cst, const T *cff, const T *input, T *out) {
  const int n1 = deg + 1;
  std::vector<const T *> x(dim);
  for (int j = 0; j < dim; ++j) x[j] = input + (long)j * n1;
  for (int i = 0; i < n1; ++i) out[(long)dim * n1 + i] = cst[i];
  for (int j = 0; j < dim; ++j)
    for (int i = 0; i < n1; ++i) out[(long)j * n1 + i] = T();
  std::vector<std::vector<T> > mon(maxvar + 1);
  std::vector<T> c(n1), t(n1);
  for (int m = 0; m < nbr; ++m) {
    const int k = nvr[m];
    const int *ix = idx + (long)m * maxvar;
    const int *ex = exps + (long)m * maxvar;
    for (int i = 0; i < n1; ++i) c[i] = cff[(long)m * n1 + i];
    bool common = false;
    for (int v = 0; v < k; ++v)
      for (int e = 1; e < ex[v]; ++e) {
        conv(deg, x[ix[v]], c.data(), t.data());
        c = t;
        common = true;
      }
    monomial_evaldiff(k, deg, ix, c.data(), x, mon);
    if (common)
      for (int v = 0; v < k; ++v)
        for (int i = 0; i < n1; ++i) mon[v][i] = mul_d(mon[v][i], (double)ex[v]);
    for (int i = 0; i < n1; ++i) out[(long)dim * n1 + i] = out[(long)dim * n1 + i] + mon[k][i];
    for (int v = 0; v < k; ++v)
      for (int i = 0; i < n1; ++i) out[(long)ix[v] * n1 + i] = out[(long)ix[v] * n1 + i] + mon[v][i];
  }
}

// ------------------------------------------------------------------ QR
// Householder vector and beta for x[0..n-1], v[0] = 1.
// Matrices/dbl2_factorizations.cpp:374 (real) and :436 (complex): the real
// case takes v0 = x0 - mu or -sigma/(x0 + mu); the complex case scales mu
// by the phase of x0 so that R has diagonal mu*x0/|x0|.
template <class T>
static void house(int n, const T *x, T *v, typename real_of<T>::type *beta) {
  typedef typename real_of<T>::type R;
  R sigma(0.0);
  v[0] = T(R(1.0));
  for (int i = 1; i < n; ++i) {
    sigma = sigma + norm2(x[i]);
    v[i] = x[i];
  }
  if (is_zero(sigma)) {
    *beta = R(0.0);
    return;
  }
  T v0 = T();
  if constexpr (is_cx<T>::v) {
    R sq0 = norm2(x[0]);
    R rad0 = sqrt(sq0);
    R mu = sqrt(sq0 + sigma);
    if (is_zero(rad0)) {
      v0 = T(-mu);
    } else {
      mu = mu / rad0;
      v0 = T(x[0].re - mu * x[0].re, x[0].im - mu * x[0].im);
    }
  } else {
    R mu = sqrt(x[0] * x[0] + sigma);
    if (lead(x[0]) <= 0.0)
      v0 = x[0] - mu;
    else
      v0 = -(sigma / (x[0] + mu));
  }
  R v0sq = norm2(v0);
  *beta = mul_d(v0sq / (sigma + v0sq), 2.0);
  if constexpr (is_cx<T>::v) {
    T inv0(v0.re / v0sq, -(v0.im / v0sq));
    for (int i = 1; i < n; ++i) v[i] = v[i] * inv0;
  } else {
    for (int i = 1; i < n; ++i) v[i] = v[i] / v0;
  }
  v[0] = T(R(1.0));
}

// R <- (I - beta v v^H) R on rows k.., columns k..ncols-1.
// Matrices/dbl2_factorizations.cpp:534 (real), :567 (complex).
template <class T>
static void left_update(int nrows, int ncols, int k, T *Rm, int ldr, const T *v,
                        const typename real_of<T>::type &beta) {
  std::vector<T> w(ncols - k);
  for (int j = k; j < ncols; ++j) {
    T acc = T();
    for (int i = k; i < nrows; ++i) acc = acc + conj(Rm[(long)i * ldr + j]) * v[i - k];
    w[j - k] = T(acc) * T(beta);
  }
  for (int i = k; i < nrows; ++i)
    for (int j = k; j < ncols; ++j) Rm[(long)i * ldr + j] = Rm[(long)i * ldr + j] - v[i - k] * conj(w[j - k]);
}

// Blocked Householder QR with WY accumulation, A = Q R, Q is nrows x nrows,
// R is nrows x ncols (row-major), ncols = szt*nbt.
// Matrices/dbl2_baqr_host.cpp:728 (CPU_dbl2_blocked_houseqr): per tile, the
// szt reflectors are applied to the panel column by column, then
// W = -B (I + W Y^H) Y column by column (:13 VB_to_W), the trailing columns
// get R <- R + Y W^H R (:169 leftRupdate, skipped for the last tile) and
// Q <- Q + Q W Y^H (:417 rightQupdate).
template <class T>
static void blocked_houseqr(int nrows, int ncols, int szt, int nbt, const T *A, T *Q, T *Rm) {
  typedef typename real_of<T>::type Rt;
  for (int i = 0; i < nrows; ++i) {
    for (int j = 0; j < nrows; ++j) Q[(long)i * nrows + j] = T();
    Q[(long)i * nrows + i] = T(Rt(1.0));
    for (int j = 0; j < ncols; ++j) Rm[(long)i * ncols + j] = A[(long)i * ncols + j];
  }
  std::vector<T> x(nrows), v(nrows);
  std::vector<Rt> B(szt);
  std::vector<std::vector<T> > Y(szt, std::vector<T>(nrows)), W(szt, std::vector<T>(nrows));
  for (int k = 0; k < nbt; ++k) {
    const int rowoff = k * szt;
    const int rowdim = nrows - rowoff;
    for (int L = 0; L < szt; ++L) {
      const int col = k * szt + L;
      const int endcol = (k + 1) * szt;
      const int nrc = nrows - col;
      for (int i = col; i < nrows; ++i) x[i - col] = Rm[(long)i * ncols + col];
      Rt beta;
      house(nrc, x.data(), v.data(), &beta);
      left_update(nrows, endcol, col, Rm, ncols, v.data(), beta);
      B[L] = beta;
      for (int i = 0; i < L; ++i) Y[L][i] = T();
      for (int i = 0; i < nrc; ++i) Y[L][i + L] = v[i];
    }
    // W from B and Y (Matrices/dbl2_baqr_host.cpp:13)
    for (int i = 0; i < rowdim; ++i) W[0][i] = -(T(B[0]) * Y[0][i]);
    std::vector<T> p(szt);
    for (int j = 1; j < szt; ++j) {
      for (int kk = 0; kk < j; ++kk) {
        T acc = T();
        for (int i = 0; i < rowdim; ++i) acc = acc + conj(Y[kk][i]) * Y[j][i];
        p[kk] = acc;
      }
      for (int i = 0; i < rowdim; ++i) {
        T z = T();
        for (int kk = 0; kk < j; ++kk) z = z + W[kk][i] * p[kk];
        z = z + Y[j][i];
        W[j][i] = -(T(B[j]) * z);
      }
    }
    if (k < nbt - 1) {  // R <- R + Y W^H R on the trailing columns
      const int coloff = (k + 1) * szt;
      const int coldim = ncols - coloff;
      std::vector<T> YWH((long)rowdim * rowdim), prd((long)rowdim * coldim);
      for (int i = 0; i < rowdim; ++i)
        for (int j = 0; j < rowdim; ++j) {
          T acc = T();
          for (int kk = 0; kk < szt; ++kk) acc = acc + Y[kk][i] * conj(W[kk][j]);
          YWH[(long)i * rowdim + j] = acc;
        }
      for (int i = 0; i < rowdim; ++i)
        for (int j = 0; j < coldim; ++j) {
          T acc = T();
          for (int kk = 0; kk < rowdim; ++kk) acc = acc + YWH[(long)i * rowdim + kk] * Rm[(long)(rowoff + kk) * ncols + coloff + j];
          prd[(long)i * coldim + j] = acc;
        }
      for (int i = 0; i < rowdim; ++i)
        for (int j = 0; j < coldim; ++j)
          Rm[(long)(rowoff + i) * ncols + coloff + j] = Rm[(long)(rowoff + i) * ncols + coloff + j] + prd[(long)i * coldim + j];
    }
    {  // Q <- Q + Q W Y^H on columns rowoff..
      std::vector<T> WYH((long)rowdim * rowdim), prd((long)nrows * rowdim);
      for (int i = 0; i < rowdim; ++i)
        for (int j = 0; j < rowdim; ++j) {
          T acc = T();
          for (int kk = 0; kk < szt; ++kk) acc = acc + W[kk][i] * conj(Y[kk][j]);
          WYH[(long)i * rowdim + j] = acc;
        }
      for (int i = 0; i < nrows; ++i)
        for (int j = 0; j < rowdim; ++j) {
          T acc = T();
          for (int kk = 0; kk < rowdim; ++kk) acc = acc + Q[(long)i * nrows + rowoff + kk] * WYH[(long)kk * rowdim + j];
          prd[(long)i * rowdim + j] = acc;
        }
      for (int i = 0; i < nrows; ++i)
        for (int j = 0; j < rowdim; ++j)
          Q[(long)i * nrows + rowoff + j] = Q[(long)i * nrows + rowoff + j] + prd[(long)i * rowdim + j];
    }
  }
}

// Unblocked Householder QR, Matrices/dbl2_factorizations.cpp:723
// (CPU_dbl2_factors_houseqr), used by the host least-squares head.
template <class T>
static void houseqr(int nrows, int ncols, const T *A, T *Q, T *Rm) {
  typedef typename real_of<T>::type Rt;
  for (int i = 0; i < nrows; ++i) {
    for (int j = 0; j < nrows; ++j) Q[(long)i * nrows + j] = T();
    Q[(long)i * nrows + i] = T(Rt(1.0));
    for (int j = 0; j < ncols; ++j) Rm[(long)i * ncols + j] = A[(long)i * ncols + j];
  }
  std::vector<T> x(nrows), v(nrows), w(nrows);
  for (int k = 0; k < ncols; ++k) {
    if (nrows - k <= 0) break;
    for (int i = k; i < nrows; ++i) x[i - k] = Rm[(long)i * ncols + k];
    Rt beta;
    house(nrows - k, x.data(), v.data(), &beta);
    left_update(nrows, ncols, k, Rm, ncols, v.data(), beta);
    // Q <- Q (I - beta v v^H), dbl2_factorizations.cpp:629/:662
    for (int i = 0; i < nrows; ++i) {
      T acc = T();
      for (int j = k; j < nrows; ++j) acc = acc + Q[(long)i * nrows + j] * v[j - k];
      w[i] = acc * T(beta);
    }
    for (int i = 0; i < nrows; ++i)
      for (int j = k; j < nrows; ++j) Q[(long)i * nrows + j] = Q[(long)i * nrows + j] - w[i] * conj(v[j - k]);
  }
}

// x = U^{-1} b by back substitution, Matrices/dbl2_factorizations.cpp:121.
template <class T> static void backward(int dim, const T *U, int ldu, const T *b, T *x) {
  for (int i = dim - 1; i >= 0; --i) {
    T acc = b[i];
    for (int j = dim - 1; j > i; --j) acc = acc - U[(long)i * ldu + j] * x[j];
    x[i] = acc / U[(long)i * ldu + i];
  }
}

// Tiled back substitution, Matrices/dbl2_tabs_host.cpp:147
// (CPU_dbl2_upper_tiled_solver).  Like the reference it overwrites the
// diagonal tiles of U with their inverses and b with the updated right hand
// sides.
template <class T> static void upper_tiled_solver(int dim, int szt, int nbt, T *U, T *b, T *x) {
  typedef typename real_of<T>::type Rt;
  std::vector<T> Tt((long)szt * szt), inv((long)szt * szt), e(szt), col(szt), wb(szt);
  auto invert_tile = [&](int idx) {
    for (int i = 0; i < szt; ++i)
      for (int j = 0; j < szt; ++j) Tt[(long)i * szt + j] = U[(long)(idx + i) * dim + idx + j];
    for (int j = 0; j < szt; ++j) {
      for (int i = 0; i < szt; ++i) e[i] = T();
      e[j] = T(Rt(1.0));
      backward(szt, Tt.data(), szt, e.data(), col.data());
      for (int i = 0; i < szt; ++i) inv[(long)i * szt + j] = col[i];
    }
    for (int i = 0; i < szt; ++i)
      for (int j = 0; j < szt; ++j) U[(long)(idx + i) * dim + idx + j] = inv[(long)i * szt + j];
  };
  int idx = (nbt - 1) * szt;
  invert_tile(idx);
  for (int i = 0; i < szt; ++i) {
    T acc = T();
    for (int j = 0; j < szt; ++j) acc = acc + inv[(long)i * szt + j] * b[idx + j];
    x[idx + i] = acc;
  }
  for (int k = nbt - 1; k > 0; --k) {
    idx -= szt;
    invert_tile(idx);
    for (int L = 0; L < k; ++L) {
      const int r = L * szt;
      for (int i = 0; i < szt; ++i) {
        T acc = T();
        for (int j = 0; j < szt; ++j) acc = acc + U[(long)(r + i) * dim + idx + szt + j] * x[idx + szt + j];
        b[r + i] = b[r + i] - acc;
      }
    }
    for (int i = 0; i < szt; ++i) {
      T acc = T();
      for (int j = 0; j < szt; ++j) acc = acc + inv[(long)i * szt + j] * b[idx + j];
      wb[i] = acc;
    }
    for (int i = 0; i < szt; ++i) x[idx + i] = wb[i];
  }
}

// ----------------------------------------------- block Toeplitz solve
// max_i of |hi limb| (complex: |re|+|im|): Newton/dbl_onenorms_host.cpp:9,20
template <class T> static double maxnorm(int dim, const T *v) {
  double r = 0.0;
  for (int i = 0; i < dim; ++i) {
    double a = is_cx<T>::v ? lead(v[i]) : std::fabs(lead(v[i]));
    if (a > r) r = a;
  }
  return r;
}

// x = R^{-1} Q^H b, Matrices/dbl2_factorizations.cpp:823 (factors_qrbs)
template <class T> static void qrbs(int n, const T *Q, const T *Rm, const T *b, T *x, T *w) {
  for (int i = 0; i < n; ++i) {
    T acc = T();
    for (int j = 0; j < n; ++j) acc = acc + conj(Q[(long)j * n + i]) * b[j];
    w[i] = acc;
  }
  backward(n, Rm, n, w, x);
}

// Skip thresholds of the reference's least-squares solvers:
// Newton/dbl_bals_host.cpp:36,199 (double: |b_0| + 1 == 1 for the head,
// 1e-15 in the tail), dbl2_bals_host.cpp:43,254 (1e-28), dbl4_bals_host.cpp:51,335
// (1e-56).
template <class T> static double skip_tol() {
  const int L = limbs<typename real_of<T>::type>::n;
  return L == 1 ? 1.0e-15 : (L == 2 ? 1.0e-28 : 1.0e-56);
}
template <class T> static bool head_tiny(double nrm) {
  const int L = limbs<typename real_of<T>::type>::n;
  return L == 1 ? (nrm + 1.0 == 1.0) : (nrm < skip_tol<T>());
}

struct bals_state {
  int zeroQ, noqr, upidx, bsidx, newtail;
};

// Solve sum_{j<=k} A_j x_{k-j} = b_k, k = 0..degp1-1 (A_j dim x dim).
// Newton/dbl2_bals_host.cpp:479 (CPU_dbl2_qrbs_solve) with the head at :15
// and the tail at :228, including the skip rules: no QR when |b_0| < 1e-28
// unless zeroQ, no update with x_{i-1} when |x_{i-1}| < 1e-28, no back
// substitution (x_i = 0) when |b_i| < 1e-28 (thresholds per precision in
// skip_tol).  rhs is overwritten.
template <class T>
static void bals_solve(int dim, int degp1, int tailidx, const T *mat, T *rhs, T *sol, T *Q, T *Rm,
                       bals_state *st) {
  const long nn = (long)dim * dim;
  std::vector<T> w(dim);
  if (!(st->noqr && !st->zeroQ)) {
    double nrm = maxnorm(dim, rhs);
    if (head_tiny<T>(nrm)) st->noqr = st->zeroQ ? 0 : 1;
    if (!st->noqr) {
      houseqr(dim, dim, mat, Q, Rm);
      st->zeroQ = 0;
      qrbs(dim, Q, Rm, rhs, sol, w.data());
    }
  }
  if (degp1 > 1) {
    int skipup = 0, skipbs = 0;
    bool first = true;
    st->newtail = degp1;
    for (int i = tailidx; i < degp1; ++i) {
      const T *xi = sol + (long)(i - 1) * dim;
      if (maxnorm(dim, xi) < skip_tol<T>()) {
        ++skipup;
      } else {
        for (int j = i; j < degp1; ++j) {
          const T *Aj = mat + (long)(j - i + 1) * nn;
          T *wj = rhs + (long)j * dim;
          for (int k = 0; k < dim; ++k) {
            T acc = wj[k];
            for (int L = 0; L < dim; ++L) acc = acc - Aj[(long)k * dim + L] * xi[L];
            wj[k] = acc;
          }
        }
      }
      T *x = sol + (long)i * dim;
      T *b = rhs + (long)i * dim;
      if (maxnorm(dim, b) < skip_tol<T>()) {
        ++skipbs;
        for (int j = 0; j < dim; ++j) x[j] = T();
      } else {
        if (first) {
          st->newtail = i;
          first = false;
        }
        qrbs(dim, Q, Rm, b, x, w.data());
      }
    }
    st->upidx = skipup;
    st->bsidx = skipbs;
  }
}

}  // namespace orc
