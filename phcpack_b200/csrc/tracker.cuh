// tracker.cuh -- CTA-level building blocks of the path tracker: evaluation
// of a homotopy h(x, t) = sum_terms (a + b t) x^e and its Jacobian at a
// vector of power series in s = t - t0, the small dense solves, the Pade
// approximants and the conversions between precisions.
#pragma once
#include "md.cuh"
#include "dense.cuh"

namespace phc {

static const int kTrackThreads = 128;
static const int kTrackKmax = 16;   // largest series degree of the predictor

// Homotopy systems, flat (see include/phc_b200.h, phc_track):
struct TrackDev {
  int nsys, maxvar, maxdim;
  const int *dim;        // [nsys]
  const int *mono_off;   // [nsys+1] distinct monomials of system s
  const int *mono_nvr;   // [nmono]
  const int *mono_idx;   // [nmono*maxvar]
  const int *mono_exp;   // [nmono*maxvar]
  const int *eq_off;     // [nsys+1] equations of system s
  const int *term_off;   // [neq+1]  terms of equation e
  const int *term_mono;  // [nterm]  global monomial id
  const double *term_a;  // [nterm*2] complex double
  const double *term_b;  // [nterm*2]
  const int *jg_off;     // [neq*maxdim+1] Jacobian gather lists per (equation, variable)
  const int *jg_term;    // [njg] term id
  const int *jg_slot;    // [njg] slot of the variable in the term's monomial
};

// Tracking parameters (include/phc_b200.h, phc_track: ipar and dpar)
struct TrackParDev {
  int deg, numdeg, dendeg, nit, corsteps, maxsteps, refine_steps, step_mode;
  double pbeta, alpha, maxsize, minsize, tolres, epsilon, restol, learn_scale;
};

// conversions between number types (complex only)
template <class A, class B> struct conv_num;
template <class R> struct conv_num<md::num<R, true>, md::num<R, true> > {
  __device__ __forceinline__ static md::cx<R> go(const md::cx<R> &a) { return a; }
};
template <> struct conv_num<md::num<md::dd, true>, md::num<double, true> > {
  __device__ __forceinline__ static md::cx<double> go(const md::cx<md::dd> &a) {
    md::cx<double> r;
    r.re = __dadd_rn(a.re.hi, a.re.lo);
    r.im = __dadd_rn(a.im.hi, a.im.lo);
    return r;
  }
};
template <> struct conv_num<md::num<double, true>, md::num<md::dd, true> > {
  __device__ __forceinline__ static md::cx<md::dd> go(const md::cx<double> &a) {
    md::cx<md::dd> r;
    r.re = md::mk(a.re, 0.0);
    r.im = md::mk(a.im, 0.0);
    return r;
  }
};
template <> struct conv_num<md::num<md::dd, true>, md::num<md::qd, true> > {
  __device__ __forceinline__ static md::cx<md::qd> go(const md::cx<md::dd> &a) {
    md::cx<md::qd> r;
    r.re = md::mkq(a.re.hi, a.re.lo, 0.0, 0.0);
    r.im = md::mkq(a.im.hi, a.im.lo, 0.0, 0.0);
    return r;
  }
};
template <> struct conv_num<md::num<md::qd, true>, md::num<md::dd, true> > {
  __device__ __forceinline__ static md::cx<md::dd> go(const md::cx<md::qd> &a) {
    md::cx<md::dd> r;
    r.re = md::mk(a.re.x[0], a.re.x[1]);
    r.im = md::mk(a.im.x[0], a.im.x[1]);
    return r;
  }
};

template <class N>
__device__ __forceinline__ typename N::T cnum(double re, double im) {
  typename N::T r = N::from(re);
  r.im = N::tr::from(im);
  return r;
}

// Evaluate the homotopy of system s at the series x (n series of degree w,
// leading dimension xld numbers per variable) and t = t0 + s:
//   h[i*(w+1)+k]        value series of equation i,
//   J[(k*n + i)*n + j]  Jacobian series (when J != nullptr).
// V, G: shared staging for the distinct monomials, nm*(w+1) and
// nm*maxvar*(w+1) numbers.
// Phase 1: one thread per distinct monomial computes its value and its
// partials (exponent included) by the common-factor method and products of
// the distinct variables.  Phase 2: one thread per output coefficient
// gathers the coefficient series (a + b t0) + b s times the monomial series
// over the terms of its equation (value) or over the Jacobian gather list
// of its (equation, variable) pair.
template <class N>
__device__ void hom_eval_cta(const TrackDev &S, int s, int w, double t0, const double *x, int xld, double *V,
                             double *G, double *h, double *J) {
  typedef typename N::T T;
  const int W = N::width;
  const int n = S.dim[s];
  const int n1 = w + 1;
  const int m0 = S.mono_off[s];
  const int nm = S.mono_off[s + 1] - m0;
  const int mv = S.maxvar;
  for (int m = threadIdx.x; m < nm; m += blockDim.x) {
    const int gm = m0 + m;
    const int k = S.mono_nvr[gm];
    const int *ix = S.mono_idx + (long)gm * mv;
    const int *ex = S.mono_exp + (long)gm * mv;
    T F[kTrackKmax + 1], acc[kTrackKmax + 1];
    bool unitF = true;
    for (int i = 0; i < n1; ++i) F[i] = (i == 0) ? N::one() : N::zero();
    for (int v = 0; v < k; ++v)
      for (int e = 1; e < ex[v]; ++e) {
        const double *xv = x + (long)ix[v] * xld * W;
        for (int kk = w; kk >= 0; --kk) {  // in place: F[kk] only needs F[<= kk]
          T a = N::zero();
          for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xv, i), F[kk - i]));
          F[kk] = a;
        }
        unitF = false;
      }
    double *Vm = V + (long)m * n1 * W;
    double *Gm = G + (long)m * mv * n1 * W;
    if (k == 0) {
      for (int i = 0; i < n1; ++i) stn_at<N>(Vm, i, F[i]);
      continue;
    }
    for (int v = 0; v < k; ++v) {
      for (int i = 0; i < n1; ++i) acc[i] = F[i];
      bool unit = unitF;
      for (int u = 0; u < k; ++u) {
        if (u == v) continue;
        const double *xu = x + (long)ix[u] * xld * W;
        if (unit) {
          for (int i = 0; i < n1; ++i) acc[i] = ldn_at<N>(xu, i);
          unit = false;
        } else {
          for (int kk = w; kk >= 0; --kk) {
            T a = N::zero();
            for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xu, i), acc[kk - i]));
            acc[kk] = a;
          }
        }
      }
      if (v == 0) {
        const double *x0 = x + (long)ix[0] * xld * W;
        for (int kk = 0; kk < n1; ++kk) {
          T a = N::zero();
          for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(x0, i), acc[kk - i]));
          stn_at<N>(Vm, kk, a);
        }
      }
      const double e = (double)ex[v];
      for (int i = 0; i < n1; ++i) stn_at<N>(Gm + (long)v * n1 * W, i, e == 1.0 ? acc[i] : N::scale_d(acc[i], e));
    }
  }
  __syncthreads();
  const int e0 = S.eq_off[s];
  const int nval = n * n1;
  const int njac = J ? n * n * n1 : 0;
  for (int it = threadIdx.x; it < nval + njac; it += blockDim.x) {
    T acc = N::zero();
    if (it < nval) {
      const int i = it / n1, kk = it % n1;
      for (int tr = S.term_off[e0 + i]; tr < S.term_off[e0 + i + 1]; ++tr) {
        const T a = cnum<N>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
        const T b = cnum<N>(S.term_b[2 * tr], S.term_b[2 * tr + 1]);
        const T c0 = N::add(a, N::scale_d(b, t0));
        const double *Vm = V + (long)(S.term_mono[tr] - m0) * n1 * W;
        acc = N::add(acc, N::mul(c0, ldn_at<N>(Vm, kk)));
        if (kk > 0) acc = N::add(acc, N::mul(b, ldn_at<N>(Vm, kk - 1)));
      }
      stn_at<N>(h, (long)i * n1 + kk, acc);
    } else {
      const int r = it - nval;
      const int kk = r / (n * n), i = (r / n) % n, j = r % n;
      const int g = (e0 + i) * S.maxdim + j;
      for (int q = S.jg_off[g]; q < S.jg_off[g + 1]; ++q) {
        const int tr = S.jg_term[q];
        const T a = cnum<N>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
        const T b = cnum<N>(S.term_b[2 * tr], S.term_b[2 * tr + 1]);
        const T c0 = N::add(a, N::scale_d(b, t0));
        const double *Gm = G + ((long)(S.term_mono[tr] - m0) * mv + S.jg_slot[q]) * n1 * W;
        acc = N::add(acc, N::mul(c0, ldn_at<N>(Gm, kk)));
        if (kk > 0) acc = N::add(acc, N::mul(b, ldn_at<N>(Gm, kk - 1)));
      }
      stn_at<N>(J, ((long)kk * n + i) * n + j, acc);
    }
  }
  __syncthreads();
}

// Q <- Q (I - beta v v^H) on columns c..n-1 of the n x n matrix Q
// (Matrices/dbl2_factorizations.cpp:629/:662)
template <class N>
__device__ void block_apply_reflector_right(int n, int c, double *Q, dense_smem &S) {
  typedef typename N::T T;
  typedef typename N::real R;
  typedef md::num<R, false> RN;
  const R beta = ldn_at<RN>(S.misc, 0);
  if (md::is_zero(beta)) return;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T acc = N::zero();
    for (int j = c; j < n; ++j) acc = N::add(acc, N::mul(ldn_at<N>(Q, (long)i * n + j), ldn_at<N>(S.v, j - c)));
    stn_at<N>(S.w, i, N::scale(acc, beta));
  }
  __syncthreads();
  const int nc = n - c;
  for (int t = threadIdx.x; t < n * nc; t += blockDim.x) {
    const int i = t / nc, j = c + t % nc;
    const long o = (long)i * n + j;
    stn_at<N>(Q, o, N::sub(ldn_at<N>(Q, o), N::mul(ldn_at<N>(S.w, i), N::conj(ldn_at<N>(S.v, j - c)))));
  }
  __syncthreads();
}

// Householder QR of the n x n matrix in Rm (overwritten by R), Q formed
// explicitly, then Minv = R^{-1} (upper triangular inverse).  Unblocked:
// the systems the tracker solves are small.
template <class N>
__device__ void small_qr(int n, double *Q, double *Rm, double *Rinv, dense_smem &S) {
  for (int t = threadIdx.x; t < n * n; t += blockDim.x)
    stn_at<N>(Q, t, (t / n == t % n) ? N::one() : N::zero());
  __syncthreads();
  for (int c = 0; c < n; ++c) {
    block_house<N>(n - c, Rm + (long)c * n * N::width + (long)c * N::width, n, S);
    block_apply_reflector<N>(n, n, c, n, Rm, S);
    block_apply_reflector_right<N>(n, c, Q, S);
  }
  block_invert_tiles<N>(n, n, Rm, n, Rinv);
}

// y = M b, M n x n, one thread per row
template <class N>
__device__ void cta_matvec(int n, const double *M, const double *b, double *y) {
  typedef typename N::T T;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T acc = N::zero();
    for (int j = 0; j < n; ++j) acc = N::add(acc, N::mul(ldn_at<N>(M, (long)i * n + j), ldn_at<N>(b, j)));
    stn_at<N>(y, i, acc);
  }
  __syncthreads();
}

// y = M^H b
template <class N>
__device__ void cta_matvec_h(int n, const double *M, const double *b, double *y) {
  typedef typename N::T T;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T acc = N::zero();
    for (int j = 0; j < n; ++j) acc = N::add(acc, N::mul(N::conj(ldn_at<N>(M, (long)j * n + i)), ldn_at<N>(b, j)));
    stn_at<N>(y, i, acc);
  }
  __syncthreads();
}

}  // namespace phc
