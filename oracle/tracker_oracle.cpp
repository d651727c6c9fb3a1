// tracker_oracle.cpp -- CPU restatement of the series-Pade path tracker.
//
// TEST INFRASTRUCTURE ONLY: the checker of the GPU tracker and the CPU
// baseline of bench.py.  Never part of the product path.
//
// The reference's series-Pade tracker is Ada code (not compilable here):
//   Curves/predictor_corrector_trackers.adb:51-77  Track_One_Path
//   Curves/predictor_corrector_loops.adb:37-85     Predictor_Corrector_Loop
//   Curves/standard_predictor_convolutions.adb:1142-1185 LU_Prediction,
//                                              :958-993   Predictor_Feedback
//   Curves/standard_rational_approximations.ads:67-145 Pade, Evaluate
//   Math_Lib/Circuits/convergence_radius_estimates.adb:138,354 Fabry
//   Solutions/standard_mixed_residuals.adb:472 Mixed_Residual
//   Curves/homotopy_continuation_parameters.adb:6-24 defaults
// restated here on top of this oracle's multiple-double arithmetic.  What is
// restated and what is left out:
//  * predictor: the Taylor series of the path in s = t - t0 to degree K,
//    x_k = -J_0^{-1} [h(x_0 + ... + x_{k-1} s^{k-1})]_k one degree at a
//    time (the fixed point of LU_Prediction's Newton on power series, with
//    J_0 factored once and applied as its inverse); [L/M] Pade approximant
//    per component; pole step
//    pbeta * r with r the smallest Fabry radius |c_{K-3}/c_{K-2}| (offset 2
//    as in Newton_Fabry);
//  * the curvature step (Hesse_Pade, Curves/dobldobl_predictor_convolutions
//    .adb:383-406): eta = 2 sigma_min(J) / |(sigma_max(H_1), ...,
//    sigma_max(H_n))|_2 at the current point (Distance,
//    Curves/singular_values_of_hessians.adb:190-211), the step
//    (cbeta eta / |Pade error estimates|_2)^(1/K) (Step_Distance,
//    Curves/series_and_predictors.adb:813-825; Solution_Error,
//    Curves/homotopy_pade_approximants.adb:687-754); the singular values in
//    complex double by one-sided Jacobi rotations to convergence;
//  * step = the smallest of the pole step, the curvature step and maxsize,
//    counted as pole, curvature or maxsize step (Minimum,
//    Curves/three_way_minima.adb:48-62); a step reaching 1 - minsize goes to
//    t = 1 (Bounded_Update, three_way_minima.adb:96-109);
//  * step_mode bit 2 (double predictor): J_0 inverted by Householder QR
//    (qr_inverse) instead of LU;
//  * step_mode bit 1: the learned proposal plain step * exp(network(features))
//    (the BF16 network of the model buffer, evaluated in float in the
//    device's order of operations); a proposal whose feedback or corrector
//    fails is redone with the plain step;
//  * predictor feedback: halve the step until the mixed residual of the
//    Pade prediction is below alpha (fail below minsize);
//  * corrector: at most corsteps LU Newton steps at the new t (LU_Newton_Steps,
//    Curves/corrector_convolutions.adb:1193-1224), residuals in double-double,
//    the Jacobian and its solve in the predictor's precision, converged when
//    max |dx_i| <= tolres, followed by one extra step; on failure halve the
//    step and re-evaluate the Pade approximant (fail below minsize);
//  * stop when |1 - t| < epsilon; refine the endpoint at t = 1 and classify
//    success when the max-norm residual is at most restol.
// The homotopy is h(x, t) = sum_terms ((1 - t) a + t b) x^e, which is
// (1 - t) gamma q(x) + t p(x) with a = gamma c_q, b = c_p
// (Path/Path_GPU/eval_coef.cu:27-28).
#include <vector>
#include <thread>
#include <atomic>
#include <cmath>
#include <algorithm>
#include <cstring>
#include <utility>
#include "oracle_core.hpp"

using namespace orc;

namespace {

struct TrackSys {
  int nsys, maxvar;
  const int *dim;       // [nsys]
  const int *mono_off;  // [nsys+1], global monomial ids
  const int *mono_nvr;  // [nmono]
  const int *mono_idx;  // [nmono*maxvar]
  const int *mono_exp;  // [nmono*maxvar]
  const int *eq_off;    // [nsys+1], global equation ids
  const int *term_off;  // [neq+1]
  const int *term_mono; // [nterm]
  const double *term_a; // [nterm*2] complex double
  const double *term_b; // [nterm*2]
};

struct TrackPar {
  int deg, numdeg, dendeg, nit, corsteps, maxsteps, refine_steps, step_mode;
  double pbeta, alpha, maxsize, minsize, tolres, epsilon, restol, learn_scale, cbeta;
  const unsigned char *model;  // the learned step's model buffer (step_mode 1)
};

template <class R> static cx<R> cplx(double re, double im) { return cx<R>(R(re), R(im)); }

template <class T> struct is_double { static const bool v = false; };
template <> struct is_double<cx<double> > { static const bool v = true; };

// Evaluate h and, when jac != nullptr, J at a vector of series x (dim
// series of degree w) at t = t0 + s: value series h[i][k], Jacobian series
// jac[k][i][j].  Per distinct monomial: common factor, then products of the
// distinct variables (the reference's common-factor + Speelpenning method
// restated for a monomial without coefficient); per term the coefficient
// series c0 + c1 s, c1 = b - a, c0 = a + t0 c1, multiplies the monomial and
// its partials.
template <class T>
static void hom_eval(const TrackSys &S, int s, int w, double t0, const std::vector<std::vector<T> > &x,
                     std::vector<std::vector<T> > &h, std::vector<T> *jac) {
  typedef typename real_of<T>::type R;
  const int n = S.dim[s];
  const int n1 = w + 1;
  const int m0 = S.mono_off[s], m1 = S.mono_off[s + 1];
  const int nm = m1 - m0;
  // V[m] value, G[m][v] partial w.r.t. slot v (exponent included)
  std::vector<std::vector<T> > V(nm, std::vector<T>(n1));
  std::vector<std::vector<std::vector<T> > > G(nm);
  std::vector<T> tmp(n1), acc(n1);
  for (int m = 0; m < nm; ++m) {
    const int gm = m0 + m;
    const int k = S.mono_nvr[gm];
    const int *ix = S.mono_idx + (long)gm * S.maxvar;
    const int *ex = S.mono_exp + (long)gm * S.maxvar;
    std::vector<T> F(n1);
    F[0] = T(R(1.0));
    for (int v = 0; v < k; ++v)
      for (int e = 1; e < ex[v]; ++e) {
        conv(w, x[ix[v]].data(), F.data(), tmp.data());
        F = tmp;
      }
    G[m].assign(k, std::vector<T>(n1));
    if (k == 0) {
      V[m] = F;
      continue;
    }
    // partial v = F * prod_{u != v} x_u ; value = partial_0 * x_0
    for (int v = 0; v < k; ++v) {
      acc = F;
      for (int u = 0; u < k; ++u) {
        if (u == v) continue;
        conv(w, acc.data(), x[ix[u]].data(), tmp.data());
        acc = tmp;
      }
      if (v == 0) conv(w, acc.data(), x[ix[0]].data(), V[m].data());
      for (int i = 0; i < n1; ++i) G[m][v][i] = mul_d(acc[i], (double)ex[v]);
    }
  }
  h.assign(n, std::vector<T>(n1));
  if (jac) jac->assign((long)n1 * n * n, T());
  const int e0 = S.eq_off[s];
  for (int i = 0; i < n; ++i) {
    const int eq = e0 + i;
    for (int tr = S.term_off[eq]; tr < S.term_off[eq + 1]; ++tr) {
      const int m = S.term_mono[tr] - m0;
      const T a = cplx<R>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
      const T b = cplx<R>(S.term_b[2 * tr], S.term_b[2 * tr + 1]) - a;  // d/dt
      const T c0 = a + b * T(R(t0));
      for (int kk = 0; kk < n1; ++kk) {
        T v = c0 * V[m][kk];
        if (kk > 0) v = v + b * V[m][kk - 1];
        h[i][kk] = h[i][kk] + v;
      }
      if (jac) {
        const int gm = m0 + m;
        const int k = S.mono_nvr[gm];
        const int *ix = S.mono_idx + (long)gm * S.maxvar;
        for (int vv = 0; vv < k; ++vv) {
          const int j = ix[vv];
          for (int kk = 0; kk < n1; ++kk) {
            T v = c0 * G[m][vv][kk];
            if (kk > 0) v = v + b * G[m][vv][kk - 1];
            T &dst = (*jac)[((long)kk * n + i) * n + j];
            dst = dst + v;
          }
        }
      }
    }
  }
}

// |h_i| evaluated with |coefficients(t)| at |x| (real, in double), for the
// mixed residual of Solutions/standard_mixed_residuals.adb:472
template <class T>
static void hom_abs_eval(const TrackSys &S, int s, double t, const std::vector<double> &ax, std::vector<double> &r) {
  const int n = S.dim[s];
  r.assign(n, 0.0);
  const int e0 = S.eq_off[s];
  for (int i = 0; i < n; ++i)
    for (int tr = S.term_off[e0 + i]; tr < S.term_off[e0 + i + 1]; ++tr) {
      const int gm = S.term_mono[tr];
      const double cr = std::fma(S.term_b[2 * tr] - S.term_a[2 * tr], t, S.term_a[2 * tr]);
      const double ci = std::fma(S.term_b[2 * tr + 1] - S.term_a[2 * tr + 1], t, S.term_a[2 * tr + 1]);
      double v = std::hypot(cr, ci);
      for (int u = 0; u < S.mono_nvr[gm]; ++u)
        v *= std::pow(ax[S.mono_idx[(long)gm * S.maxvar + u]], S.mono_exp[(long)gm * S.maxvar + u]);
      r[i] += v;
    }
}

template <class R> static double cabs(const cx<R> &a) { return std::hypot(to_double(a.re), to_double(a.im)); }

// LU factorization with partial pivoting and its solves: lufac and lusolve
// of Math_Lib/Reduction/standard_complex_linear_solvers.adb:123-178 and
// :552-583 (LINPACK zgefa/zgesl).  The pivot of column k is the first row of
// largest |re| + |im| (leading limbs); the multipliers -a_ik / a_kk are
// stored below the diagonal.  Where lusolve divides by u_kk, the back
// substitution here multiplies by dinv[k] = 1 / u_kk formed during the
// factorization (NaN for a zero pivot), as the GPU tracker does.
template <class T> struct lu_solver {
  typedef typename real_of<T>::type R;
  int n = 0, info = 0;
  std::vector<T> a, dinv;
  std::vector<int> ipvt;
  void factor(int n_, const std::vector<T> &A) {
    n = n_;
    a.assign(A.begin(), A.begin() + (long)n * n);
    dinv.assign(n, T());
    ipvt.assign(n, 0);
    info = 0;
    for (int k = 0; k < n; ++k) {
      int ell = k;
      double smax = lead(a[(long)k * n + k]);
      if (std::isnan(smax)) smax = INFINITY;
      for (int i = k + 1; i < n; ++i) {
        double v = lead(a[(long)i * n + k]);
        if (std::isnan(v)) v = INFINITY;
        if (v > smax) { smax = v; ell = i; }
      }
      ipvt[k] = ell;
      if (smax == 0.0) {
        if (info == 0) info = k + 1;
        dinv[k] = T(R(NAN));
        continue;
      }
      if (ell != k)
        for (int j = k; j < n; ++j) std::swap(a[(long)ell * n + j], a[(long)k * n + j]);
      const T inv = T(R(1.0)) / a[(long)k * n + k];
      dinv[k] = inv;
      const T temp = -inv;
      for (int i = k + 1; i < n; ++i) a[(long)i * n + k] = temp * a[(long)i * n + k];
      for (int i = k + 1; i < n; ++i)
        for (int j = k + 1; j < n; ++j) a[(long)i * n + j] = a[(long)i * n + j] + a[(long)k * n + j] * a[(long)i * n + k];
    }
  }
  // x = A^{-1} b (x may alias b)
  void solve(const T *b, T *x) const {
    if (x != b) for (int i = 0; i < n; ++i) x[i] = b[i];
    for (int k = 0; k < n - 1; ++k) {
      const int ell = ipvt[k];
      const T t = x[ell];
      if (ell != k) { x[ell] = x[k]; x[k] = t; }
      for (int i = k + 1; i < n; ++i) x[i] = x[i] + t * a[(long)i * n + k];
    }
    for (int kb = n - 1; kb >= 0; --kb) {
      x[kb] = x[kb] * dinv[kb];
      const T t = x[kb];
      for (int j = 0; j < kb; ++j) x[j] = x[j] - t * a[(long)j * n + kb];
    }
  }
  // M = A^{-1}, row-major, column by column
  void inverse(std::vector<T> &M) const {
    M.assign((long)n * n, T());
    std::vector<T> col(n);
    for (int c = 0; c < n; ++c) {
      for (int i = 0; i < n; ++i) col[i] = (i == c) ? T(R(1.0)) : T();
      solve(col.data(), col.data());
      for (int i = 0; i < n; ++i) M[(long)i * n + c] = col[i];
    }
  }
};

// M = A^{-1} by Householder QR (step_mode bit 2 of the double predictor),
// the operations in the order of the GPU's warp_qrinverse: column k takes
// sigma = sum_{i>k} |a_ik|^2, nu = sqrt(|a_kk|^2 + sigma), phase phi =
// a_kk/|a_kk| (1 for a_kk = 0), v = (a_kk + phi nu, a_{k+1,k}, ...), tau =
// 2/|v|^2, r_kk = -phi nu, then a_j -= tau v (v^H a_j) for j > k; M = Q^H
// from the identity, then R X = M by back substitution.
static void qr_inverse(int n, const std::vector<cx<double> > &A0, std::vector<cx<double> > &M) {
  typedef cx<double> T;
  typedef double R;
  std::vector<T> a(A0.begin(), A0.begin() + (long)n * n), vk(n);
  std::vector<R> tau(n, R(0.0));
  for (int k = 0; k < n; ++k) {
    R sig = R(0.0);
    for (int i = k + 1; i < n; ++i) sig = sig + norm2(a[(long)i * n + k]);
    const T xk = a[(long)k * n + k];
    const R a2 = norm2(xk);
    const R nu = std::sqrt(a2 + sig);
    T v0, rkk;
    R t = R(0.0);
    if (nu != R(0.0)) {
      T phi = T(R(1.0));
      if (a2 != R(0.0)) {
        const R ab = std::sqrt(a2);
        phi = T(xk.re / ab, xk.im / ab);
      }
      v0 = T(xk.re + phi.re * nu, xk.im + phi.im * nu);
      t = R(2.0) / (norm2(v0) + sig);
      rkk = T(-(phi.re * nu), -(phi.im * nu));
    }
    vk[k] = v0;
    tau[k] = t;
    a[(long)k * n + k] = rkk;
    for (int j = k + 1; j < n; ++j) {
      T w = conj(v0) * a[(long)k * n + j];
      for (int i = k + 1; i < n; ++i) w = w + conj(a[(long)i * n + k]) * a[(long)i * n + j];
      w = T(w.re * t, w.im * t);
      a[(long)k * n + j] = a[(long)k * n + j] - v0 * w;
      for (int i = k + 1; i < n; ++i) a[(long)i * n + j] = a[(long)i * n + j] - a[(long)i * n + k] * w;
    }
  }
  M.assign((long)n * n, T());
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) M[(long)i * n + c] = (i == c) ? T(R(1.0)) : T();
    for (int k = 0; k < n; ++k) {
      const R t = tau[k];
      if (t == R(0.0)) continue;
      const T v0 = vk[k];
      T w = conj(v0) * M[(long)k * n + c];
      for (int i = k + 1; i < n; ++i) w = w + conj(a[(long)i * n + k]) * M[(long)i * n + c];
      w = T(w.re * t, w.im * t);
      M[(long)k * n + c] = M[(long)k * n + c] - v0 * w;
      for (int i = k + 1; i < n; ++i) M[(long)i * n + c] = M[(long)i * n + c] - a[(long)i * n + k] * w;
    }
    for (int i = n - 1; i >= 0; --i) {
      T acc = M[(long)i * n + c];
      for (int j = i + 1; j < n; ++j) acc = acc - a[(long)i * n + j] * M[(long)j * n + c];
      M[(long)i * n + c] = acc / a[(long)i * n + i];
    }
  }
}

// The predictor's Taylor series: x[i] series of degree K, on entry the
// constant terms hold the current point.  x_k = -J_0^{-1} [h(x truncated
// below degree k)]_k for k = 1..K, with J_0 factored once by lufac and
// applied as its inverse; the fixed point of Newton's method on power series
// (LU_Prediction, Curves/standard_predictor_convolutions.adb:1142-1185)
// computed one degree at a time, as the GPU tracker does.
template <class T>
static void taylor_series(const TrackSys &S, int s, const TrackPar &P, double t0, std::vector<std::vector<T> > &x) {
  const int n = S.dim[s];
  const int K = P.deg;
  std::vector<std::vector<T> > h;
  std::vector<T> jac, M, r(n);
  lu_solver<T> lu;
  {
    std::vector<std::vector<T> > x0(n, std::vector<T>(1));
    for (int i = 0; i < n; ++i) x0[i][0] = x[i][0];
    hom_eval(S, s, 0, t0, x0, h, &jac);
    bool by_qr = false;
    if constexpr (is_double<T>::v) {
      by_qr = (P.step_mode & 2) != 0;
      if (by_qr) qr_inverse(n, jac, M);
    }
    if (!by_qr) {
      lu.factor(n, jac);
      lu.inverse(M);
    }
  }
  for (int k = 1; k <= K; ++k) {
    std::vector<std::vector<T> > xw(n, std::vector<T>(k + 1));
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < k; ++j) xw[i][j] = x[i][j];
    hom_eval<T>(S, s, k, t0, xw, h, nullptr);
    for (int i = 0; i < n; ++i) r[i] = h[i][k];
    for (int i = 0; i < n; ++i) {
      T acc = T();
      for (int j = 0; j < n; ++j) acc = acc + M[(long)i * n + j] * r[j];
      x[i][k] = -acc;
    }
  }
}

// [L/M] Pade approximant of the series c[0..L+M]: denominator from
// sum_{j=1..M} c_{L+i-j} q_j = -c_{L+i}, i = 1..M, by Gaussian elimination
// with partial pivoting; numerator p_i = sum_{j<=min(i,M)} q_j c_{i-j}
// (Curves/standard_rational_approximations.ads:67-100).  A singular
// denominator system falls back to the Taylor polynomial (q = 1, p = c).
template <class T>
static bool pade(int L, int M, const std::vector<T> &c, std::vector<T> &p, std::vector<T> &q) {
  typedef typename real_of<T>::type R;
  q.assign(M + 1, T());
  q[0] = T(R(1.0));
  p.assign(L + M + 1, T());
  bool ok = true;
  if (M > 0) {
    std::vector<T> A((long)M * M), b(M);
    for (int i = 1; i <= M; ++i) {
      for (int j = 1; j <= M; ++j) {
        const int k = L + i - j;
        A[(i - 1) * M + (j - 1)] = k >= 0 ? c[k] : T();
      }
      b[i - 1] = -c[L + i];
    }
    for (int col = 0; col < M && ok; ++col) {
      int piv = col;
      double best = cabs(A[col * M + col]);
      for (int r = col + 1; r < M; ++r)
        if (cabs(A[r * M + col]) > best) { best = cabs(A[r * M + col]); piv = r; }
      if (best == 0.0) { ok = false; break; }
      if (piv != col) {
        for (int j = 0; j < M; ++j) std::swap(A[piv * M + j], A[col * M + j]);
        std::swap(b[piv], b[col]);
      }
      for (int r = col + 1; r < M; ++r) {
        const T f = A[r * M + col] / A[col * M + col];
        for (int j = col; j < M; ++j) A[r * M + j] = A[r * M + j] - f * A[col * M + j];
        b[r] = b[r] - f * b[col];
      }
    }
    if (ok) {
      for (int i = M - 1; i >= 0; --i) {
        T acc = b[i];
        for (int j = i + 1; j < M; ++j) acc = acc - A[i * M + j] * q[j + 1];
        q[i + 1] = acc / A[i * M + i];
      }
    }
  }
  if (!ok) {
    q.assign(M + 1, T());
    q[0] = T(R(1.0));
    for (int i = 0; i <= L + M; ++i) p[i] = c[i];
    return false;
  }
  for (int i = 0; i <= L; ++i) {
    T acc = T();
    for (int j = 0; j <= std::min(i, M); ++j) acc = acc + q[j] * c[i - j];
    p[i] = acc;
  }
  for (int i = L + 1; i <= L + M; ++i) p[i] = T();
  return true;
}

template <class T> static T horner(const std::vector<T> &a, int deg, const T &z) {
  T acc = a[deg];
  for (int i = deg - 1; i >= 0; --i) acc = acc * z + a[i];
  return acc;
}

// conversions between the precisions (round to nearest double; widen exactly)
template <class PT, class CT> static void convert(const CT &a, PT &b);
template <> void convert(const cx<dd> &a, cx<double> &b) { b = cx<double>(a.re.hi + a.re.lo, a.im.hi + a.im.lo); }
template <> void convert(const cx<dd> &a, cx<dd> &b) { b = a; }
template <> void convert(const cx<double> &a, cx<double> &b) { b = a; }
template <> void convert(const cx<double> &a, cx<dd> &b) { b = cx<dd>(dd(a.re), dd(a.im)); }
template <> void convert(const cx<double> &a, cx<qd> &b) { b = cx<qd>(qd(a.re), qd(a.im)); }
template <> void convert(const cx<dd> &a, cx<qd> &b) { b = cx<qd>(qd(a.re), qd(a.im)); }
template <> void convert(const cx<qd> &a, cx<qd> &b) { b = a; }
template <> void convert(const cx<dd> &a, cx<od> &b) { b = cx<od>(od(a.re), od(a.im)); }
template <> void convert(const cx<od> &a, cx<od> &b) { b = a; }
// end points are written as complex quad-doubles, or octo-doubles for an
// octo-double refinement
template <class RT> struct out_num { typedef cx<qd> type; };
template <> struct out_num<cx<od> > { typedef cx<od> type; };

// Newton at a point (the corrector / refinement), returns converged:
// LU_Newton_Steps (Curves/corrector_convolutions.adb:1193-1224) with h in
// precision T and the Jacobian, its LU and the solve in precision JT (T, or
// double in the precision-split tracker, as on the GPU); x += dx in T.
template <class T, class JT>
static bool point_newton(const TrackSys &S, int s, double t, std::vector<T> &x, int maxit, double tol, int extra,
                         double *lastdx) {
  const int n = S.dim[s];
  std::vector<std::vector<T> > xs(n, std::vector<T>(1)), h;
  std::vector<std::vector<JT> > xj(n, std::vector<JT>(1)), hj;
  std::vector<JT> jac, dx(n);
  lu_solver<JT> lu;
  bool conv = false;
  int extra_left = extra;
  *lastdx = 1e300;
  for (int it = 0; it < maxit + extra; ++it) {
    if (it >= maxit && !conv) break;
    for (int i = 0; i < n; ++i) {
      xs[i][0] = x[i];
      convert(x[i], xj[i][0]);
    }
    hom_eval<T>(S, s, 0, t, xs, h, nullptr);
    hom_eval(S, s, 0, t, xj, hj, &jac);
    lu.factor(n, jac);
    for (int i = 0; i < n; ++i) {
      convert(h[i][0], dx[i]);
      dx[i] = -dx[i];
    }
    lu.solve(dx.data(), dx.data());
    if (lu.info != 0) {  // singular Jacobian: x unchanged, not converged
      *lastdx = INFINITY;
      return false;
    }
    double m = 0.0;
    for (int i = 0; i < n; ++i) {
      T d;
      convert(dx[i], d);
      x[i] = x[i] + d;
      const double a = cabs(dx[i]);
      m = (a > m || std::isnan(a)) ? a : m;
    }
    *lastdx = m;
    if (std::isnan(m)) return false;
    if (conv) {
      if (--extra_left <= 0) break;
    } else if (m <= tol) {
      conv = true;
      if (extra_left <= 0) break;
    }
  }
  return conv;
}

template <class T> static double maxres(const TrackSys &S, int s, double t, const std::vector<T> &x) {
  const int n = S.dim[s];
  std::vector<std::vector<T> > xs(n, std::vector<T>(1)), h;
  for (int i = 0; i < n; ++i) xs[i][0] = x[i];
  hom_eval<T>(S, s, 0, t, xs, h, nullptr);
  double r = 0.0;
  for (int i = 0; i < n; ++i) r = std::max(r, cabs(h[i][0]));
  return r;
}


struct PathOut {
  int status, nsteps, nreject, nbpole, nbhess, nbmaxm;
  double t, residual;
};

// ------------------------------------------------------ curvature step
// Extreme singular values (smallest, largest) of the n x n complex matrix A
// (row-major, real and imaginary parts) by one-sided Jacobi rotations of
// its columns (Hestenes) until every pair is orthogonal to 1e-15 relative.
static std::pair<double, double> singular_extremes(int n, std::vector<cx<double> > A) {
  for (int sweep = 0; sweep < 80; ++sweep) {
    bool rotated = false;
    for (int p = 0; p + 1 < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double al = 0.0, be = 0.0, gr = 0.0, gi = 0.0;
        for (int r = 0; r < n; ++r) {
          const cx<double> &ap = A[(long)r * n + p], &aq = A[(long)r * n + q];
          al += ap.re * ap.re + ap.im * ap.im;
          be += aq.re * aq.re + aq.im * aq.im;
          gr += ap.re * aq.re + ap.im * aq.im;
          gi += ap.re * aq.im - ap.im * aq.re;
        }
        const double g = std::hypot(gr, gi);
        if (!(g > 1e-15 * std::sqrt(al) * std::sqrt(be))) continue;
        rotated = true;
        const double zeta = (be - al) / (2.0 * g);
        const double tt = (zeta < 0.0 ? -1.0 : 1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + tt * tt), sn = c * tt;
        const double pr = gr / g, pi = gi / g;
        for (int r = 0; r < n; ++r) {
          const cx<double> ap = A[(long)r * n + p], aq = A[(long)r * n + q];
          const cx<double> aqt(pr * aq.re + pi * aq.im, pr * aq.im - pi * aq.re);
          A[(long)r * n + p] = cx<double>(c * ap.re - sn * aqt.re, c * ap.im - sn * aqt.im);
          A[(long)r * n + q] = cx<double>(sn * ap.re + c * aqt.re, sn * ap.im + c * aqt.im);
        }
      }
    if (!rotated) break;
  }
  double smin = INFINITY, smax = 0.0;
  for (int j = 0; j < n; ++j) {
    double s2 = 0.0;
    for (int r = 0; r < n; ++r) s2 += A[(long)r * n + j].re * A[(long)r * n + j].re + A[(long)r * n + j].im * A[(long)r * n + j].im;
    smin = std::min(smin, std::sqrt(s2));
    smax = std::max(smax, std::sqrt(s2));
  }
  return std::make_pair(smin, smax);
}

// ------------------------------------------------------ learned step
// Features of a predictor step and the network's forward pass, in the
// operations and order of the device (phcpack_b200/csrc/mlp.cuh:
// track_features, mlp_forward_cta).
static void step_features(int n, int K, double t, double plain_step, const std::vector<double> &mag, float *f) {
  const double tiny = 1e-300;
  for (int q = 0; q < 8; ++q) {
    const int k = (q + 1 <= K) ? q + 1 : K;
    double mx = 0.0, rmin = 1e300;
    for (int i = 0; i < n; ++i) {
      const double a = mag[(long)i * (K + 1) + k], b = mag[(long)i * (K + 1) + k - 1];
      mx = std::fmax(mx, a);
      if (a > 0.0) rmin = std::fmin(rmin, b / a);
    }
    const double rt = (mx > 0.0) ? -std::log(mx + tiny) / k : 30.0;
    const double rr = (rmin < 1e299) ? std::log(rmin + tiny) : 30.0;
    f[q] = (float)std::fmin(std::fmax(rt, -30.0), 30.0);
    f[8 + q] = (float)std::fmin(std::fmax(rr, -30.0), 30.0);
  }
  for (int q = 0; q < 4; ++q) {
    const int k = q <= K ? q : K;
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = std::fmax(mx, mag[(long)i * (K + 1) + k]);
    f[20 + q] = (float)std::fmin(std::fmax(std::log(mx + tiny), -60.0), 60.0);
  }
  f[16] = (float)std::log(plain_step + tiny);
  f[17] = (float)t;
  f[18] = (float)std::log(std::fmax(1.0 - t, 1e-16));
  f[19] = (float)std::log((double)n);
}

static float bf16_to_float(unsigned short h) {
  const unsigned int u = (unsigned int)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// The network 24 -> 128 -> 128 -> 1 of a model buffer (float mean[24],
// inv_std[24], b1[128], b2[128], b3[4], pad[4], then BF16 W1[128][24],
// W2[128][128], W3[128]); the output clipped to [-3, 3].
static float mlp_forward(const unsigned char *model, const float *feat) {
  const float *fl = reinterpret_cast<const float *>(model);
  const float *mean = fl, *inv_std = fl + 24, *b1 = fl + 48, *b2 = fl + 176, *b3 = fl + 304;
  const unsigned short *h = reinterpret_cast<const unsigned short *>(fl + 312);
  const unsigned short *W1 = h, *W2 = h + 128 * 24, *W3 = h + 128 * 24 + 128 * 128;
  float h1[128], c[128];
  for (int j = 0; j < 128; ++j) {
    float a = b1[j];
    for (int i = 0; i < 24; ++i) a = std::fmaf(bf16_to_float(W1[j * 24 + i]), (feat[i] - mean[i]) * inv_std[i], a);
    h1[j] = std::fmax(a, 0.0f);
  }
  for (int j = 0; j < 128; ++j) {
    float a = b2[j];
    for (int i = 0; i < 128; ++i) a = std::fmaf(bf16_to_float(W2[j * 128 + i]), h1[i], a);
    c[j] = bf16_to_float(W3[j]) * std::fmax(a, 0.0f);
  }
  float red[4];
  for (int w = 0; w < 4; ++w) {  // the butterfly of __shfl_xor_sync within each warp
    float v[32];
    for (int l = 0; l < 32; ++l) v[l] = c[32 * w + l];
    for (int o = 16; o > 0; o >>= 1) {
      float u[32];
      for (int l = 0; l < 32; ++l) u[l] = v[l] + v[l ^ o];
      for (int l = 0; l < 32; ++l) v[l] = u[l];
    }
    red[w] = v[0];
  }
  const float out = b3[0] + red[0] + red[1] + red[2] + red[3];
  return std::fmin(std::fmax(out, -3.0f), 3.0f);
}

// The pieces of the step size that need the point's Hessians, Jacobian and
// Pade error estimates (defined after the end-game helpers below).
template <class T>
static double curvature_step(const TrackSys &S, int s, const TrackPar &P, double t,
                             const std::vector<std::vector<T> > &xs, const std::vector<std::vector<T> > &num,
                             const std::vector<std::vector<T> > &den, const std::vector<int> &pdeg,
                             const std::vector<int> &qdeg);

// Track one path.  PT: predictor numbers, CT: corrector numbers, RT:
// refinement numbers.
template <class PT, class CT, class RT>
static PathOut track_path(const TrackSys &S, int s, const TrackPar &P, const double *x0, double *xend) {
  const int n = S.dim[s];
  const int K = P.deg;
  PathOut o{0, 0, 0, 0, 0, 0, 0.0, 0.0};
  std::vector<CT> x(n);
  for (int i = 0; i < n; ++i) convert(cx<double>(x0[2 * i], x0[2 * i + 1]), x[i]);
  double t = 0.0, dxn;
  point_newton<CT, PT>(S, s, 0.0, x, P.corsteps, P.tolres, 1, &dxn);
  std::vector<std::vector<PT> > xs(n, std::vector<PT>(K + 1));
  std::vector<std::vector<PT> > num(n), den(n);
  std::vector<CT> xc(n);
  std::vector<PT> xp(n);
  std::vector<double> ax(n), rabs, mag((size_t)n * (K + 1));
  std::vector<int> pdeg(n), qdeg(n);
  const bool use_model = (P.step_mode & 1) && P.model != nullptr;
  bool failed = false;
  int k;
  for (k = 0; k < P.maxsteps; ++k) {
    for (int i = 0; i < n; ++i) {
      xs[i].assign(K + 1, PT());
      convert(x[i], xs[i][0]);
    }
    taylor_series(S, s, P, t, xs);
    double r = 1e300;
    bool rfail = true;
    for (int i = 0; i < n; ++i) {
      const bool ok = pade(P.numdeg, P.dendeg, xs[i], num[i], den[i]);
      pdeg[i] = ok ? P.numdeg : K;  // the fallback is the Taylor polynomial
      qdeg[i] = ok ? P.dendeg : 0;
      const double cden = cabs(xs[i][K - 2]);
      if (cden != 0.0) {
        const double ri = cabs(xs[i][K - 3]) / cden;
        if (ri < r) r = ri;
        rfail = false;
      }
      for (int q = 0; q <= K; ++q) mag[(size_t)i * (K + 1) + q] = cabs(xs[i][q]);
    }
    const double pole_step = rfail ? P.maxsize : P.pbeta * r;
    const double curv_step = curvature_step(S, s, P, t, xs, num, den, pdeg, qdeg);
    double plain_step;
    if (pole_step < curv_step) {
      if (pole_step < P.maxsize) { plain_step = pole_step; ++o.nbpole; }
      else { plain_step = P.maxsize; ++o.nbmaxm; }
    } else {
      if (curv_step < P.maxsize) { plain_step = curv_step; ++o.nbhess; }
      else { plain_step = P.maxsize; ++o.nbmaxm; }
    }
    if (std::isnan(plain_step)) plain_step = 0.0;
    double step = plain_step;
    bool learned = false;
    if (use_model) {
      float feat[24];
      step_features(n, K, t, plain_step, mag, feat);
      const float lr = mlp_forward(P.model, feat);
      const double prop = plain_step * std::exp((double)lr) * P.learn_scale;
      if (prop > P.minsize && prop == prop) {
        step = std::fmin(prop, P.maxsize);
        learned = true;
      }
    }
    auto predict = [&](double st) {
      const PT z = PT(typename real_of<PT>::type(st));
      for (int i = 0; i < n; ++i) xp[i] = horner(num[i], pdeg[i], z) / horner(den[i], qdeg[i], z);
    };
    bool accepted = false;
    for (int attempt = 0; attempt < 2 && !accepted; ++attempt) {
      if (attempt == 1) {  // the learned proposal was rejected: the plain step
        if (!learned) break;
        learned = false;
        step = plain_step;
      }
      if (t + step >= 1.0 - P.minsize) step = 1.0 - t;  // Bounded_Update
      if (!(step > 0.0)) {
        if (learned) continue;
        failed = true;
        break;
      }
      // predictor feedback on the mixed residual
      bool ok = false;
      for (int h = 0; h < 64; ++h) {
        predict(step);
        std::vector<std::vector<PT> > xs0(n, std::vector<PT>(1)), hv;
        for (int i = 0; i < n; ++i) {
          xs0[i][0] = xp[i];
          ax[i] = cabs(xp[i]);
        }
        hom_eval<PT>(S, s, 0, t + step, xs0, hv, nullptr);
        hom_abs_eval<PT>(S, s, t + step, ax, rabs);
        double mixres = 0.0;
        for (int i = 0; i < n; ++i) mixres += cabs(hv[i][0]) / (rabs[i] + 1.0);
        mixres /= n;
        if (mixres < P.alpha) { ok = true; break; }
        step *= 0.5;
        ++o.nreject;
        if (step < P.minsize) break;
      }
      if (!ok) {
        if (learned) continue;
        failed = true;
        break;
      }
      // corrector with step halving
      bool cok = false;
      for (int h = 0; h < 64; ++h) {
        for (int i = 0; i < n; ++i) convert(xp[i], xc[i]);
        if (point_newton<CT, PT>(S, s, t + step, xc, P.corsteps, P.tolres, 1, &dxn)) { cok = true; break; }
        ++o.nreject;
        if (learned) break;
        step *= 0.5;
        if (step < P.minsize) break;
        predict(step);
      }
      if (cok) { accepted = true; break; }
      if (learned) continue;
      failed = true;
      break;
    }
    if (failed || !accepted) { failed = true; break; }
    x = xc;
    t += step;
    if (std::fabs(1.0 - t) < P.epsilon) { ++k; break; }
  }
  o.nsteps = k;
  o.t = t;
  std::vector<RT> xr(n);
  for (int i = 0; i < n; ++i) convert(x[i], xr[i]);
  if (!failed && std::fabs(1.0 - t) < P.epsilon) {
    point_newton<RT, RT>(S, s, 1.0, xr, P.refine_steps, 0.0, 0, &dxn);
    o.residual = maxres(S, s, 1.0, xr);
    o.status = (o.residual <= P.restol) ? 0 : 3;
  } else {
    o.residual = maxres(S, s, t, xr);
    o.status = failed ? 1 : 2;
  }
  typedef typename out_num<RT>::type XT;
  for (int i = 0; i < n; ++i) {
    XT q;
    convert(xr[i], q);
    store(xend + (long)i * limbs<XT>::n, q);
  }
  return o;
}

// ---------------------------------------------------------------- end game
// The end-game diagnostics at a point (x, t) of the homotopy, restated:
// Newton at the point, the Taylor series of the path to degree K, Fabry's
// ratio over the components (Newton_Fabry,
// Curves/dobldobl_fabry_on_homotopy.adb:30-83; Fabry,
// Circuits/convergence_radius_estimates.adb:138-163,392-425), the Pade error
// estimates (Solution_Error_Estimate, Threshold_Index,
// Curves/homotopy_pade_approximants.adb:558-568,717-754), and the Jacobian
// and the Hessians in complex double, whose singular values the caller
// computes (Distance, Curves/singular_values_of_hessians.adb:190-211).

// a + 1 == 1 in the working precision (Is_Zero,
// Circuits/convergence_radius_estimates.adb:8-20)
template <class R> static bool negligible(const R &a) {
  double u[8], v[8];
  store(u, R(1.0) + a);
  store(v, R(1.0));
  for (int l = 0; l < limbs<R>::n; ++l)
    if (u[l] != v[l]) return false;
  return true;
}
template <class R> static bool negligible(const cx<R> &z) { return negligible(z.re) && negligible(z.im); }

template <class R> static bool less_limbs(const R &a, const R &b) {
  double u[8], v[8];
  store(u, a);
  store(v, b);
  for (int l = 0; l < limbs<R>::n; ++l)
    if (u[l] != v[l]) return u[l] < v[l];
  return false;
}

template <class T>
static void fabry_one(const std::vector<T> &c, int K, int off, T &z, double &e, bool &fail) {
  fail = negligible(c[K - off]);
  if (fail) return;
  const double nm1 = (double)(K - 1);
  if (off == 0) {
    z = c[K - 1] / c[K];
    e = negligible(c[K - 1]) ? 1.0 : cabs(z - c[K - 2] / c[K - 1]) * nm1;
  } else {
    z = c[K - 1 - off] / c[K - off];
    e = negligible(c[K]) ? 1.0 : cabs(z - c[K - 1] / c[K]) * nm1;
  }
}

template <class T>
static double pade_error(const std::vector<T> &c, int K, const std::vector<T> &p, int pdeg, const std::vector<T> &q,
                         int qdeg) {
  typedef typename real_of<T>::type R;
  const int endidx = std::min(pdeg + qdeg + 2, K);
  int top = -1;
  for (int i = endidx; i >= 0; --i)
    if (cabs(c[i]) > 1e-5) { top = i; break; }
  T res = T(R(1.0));
  if (top >= 0) {
    res = c[top];
    for (int i = 1; i <= qdeg && i <= top; ++i) res = res + q[i] * c[top - i];
    if (top <= pdeg) res = p[top] - res;
  }
  const double a = cabs(res);
  return a < 1e-5 ? 1.0 : a;
}

template <class R> static double lead_of(const R &a) { double u[8]; store(u, a); return u[0]; }

// J[i][j] = dh_i/dx_j and H[i][j][k] = d^2 h_i / dx_j dx_k at (x, t), complex
// double, row-major (real, imaginary) pairs with ld numbers per row
static void jacobian_hessians(const TrackSys &S, int s, double t, const std::vector<cx<double> > &x, int ld,
                              double *J, double *H) {
  const int n = S.dim[s];
  std::fill(J, J + 2L * ld * ld, 0.0);
  std::fill(H, H + 2L * ld * ld * ld, 0.0);
  for (int i = 0; i < n; ++i) {
    const int eq = S.eq_off[s] + i;
    for (int tr = S.term_off[eq]; tr < S.term_off[eq + 1]; ++tr) {
      const int gm = S.term_mono[tr];
      const int nv = S.mono_nvr[gm];
      const int *ix = S.mono_idx + (long)gm * S.maxvar, *ex = S.mono_exp + (long)gm * S.maxvar;
      const cx<double> c(std::fma(S.term_b[2 * tr] - S.term_a[2 * tr], t, S.term_a[2 * tr]),
                         std::fma(S.term_b[2 * tr + 1] - S.term_a[2 * tr + 1], t, S.term_a[2 * tr + 1]));
      for (int u = 0; u < nv; ++u) {
        // first partial
        cx<double> a = mul_d(c, (double)ex[u]);
        for (int w = 0; w < nv; ++w)
          for (int e = ex[w] - (w == u); e > 0; --e) a = a * x[ix[w]];
        J[2 * ((long)i * ld + ix[u])] += a.re;
        J[2 * ((long)i * ld + ix[u]) + 1] += a.im;
        for (int v = 0; v < nv; ++v) {
          const double mult = u == v ? (double)ex[u] * (ex[u] - 1) : (double)ex[u] * ex[v];
          if (mult == 0.0) continue;
          cx<double> b = mul_d(c, mult);
          for (int w = 0; w < nv; ++w)
            for (int e = ex[w] - (w == u) - (w == v); e > 0; --e) b = b * x[ix[w]];
          const long o = 2 * (((long)i * ld + ix[u]) * ld + ix[v]);
          H[o] += b.re;
          H[o + 1] += b.im;
        }
      }
    }
  }
}

// The curvature step at the predictor's point (Hesse_Pade): the Jacobian
// and the Hessians of the equations at (x_0, t) in complex double, eta =
// 2 sigma_min(J) / |(sigma_max(H_1), ..., sigma_max(H_n))|_2, and
// (cbeta eta / |Pade error estimates|_2)^(1/K).
template <class T>
static double curvature_step(const TrackSys &S, int s, const TrackPar &P, double t,
                             const std::vector<std::vector<T> > &xs, const std::vector<std::vector<T> > &num,
                             const std::vector<std::vector<T> > &den, const std::vector<int> &pdeg,
                             const std::vector<int> &qdeg) {
  const int n = S.dim[s];
  const int K = P.deg;
  std::vector<cx<double> > xd(n);
  for (int i = 0; i < n; ++i) xd[i] = cx<double>(lead_of(xs[i][0].re), lead_of(xs[i][0].im));
  std::vector<double> J(2L * n * n), H(2L * n * n * n);
  jacobian_hessians(S, s, t, xd, n, J.data(), H.data());
  std::vector<cx<double> > A((size_t)n * n);
  for (long q = 0; q < (long)n * n; ++q) A[q] = cx<double>(J[2 * q], J[2 * q + 1]);
  const double smin = singular_extremes(n, A).first;
  double hsum = 0.0;
  for (int i = 0; i < n; ++i) {
    for (long q = 0; q < (long)n * n; ++q) A[q] = cx<double>(H[2 * ((long)i * n * n + q)], H[2 * ((long)i * n * n + q) + 1]);
    const double sm = singular_extremes(n, A).second;
    hsum += sm * sm;
  }
  const double eta = hsum > 0.0 ? 2.0 * smin / std::sqrt(hsum) : INFINITY;
  double perr = 0.0;
  for (int i = 0; i < n; ++i) {
    const double pe = pade_error(xs[i], K, num[i], pdeg[i], den[i], qdeg[i]);
    perr += pe * pe;
  }
  return std::pow(P.cbeta * eta / std::sqrt(perr), 1.0 / K);
}

struct DiagOut {
  int fail, status;
  double zre, zim, radius, err, padenorm, lastdx;
};

template <class T>
static DiagOut diag_point(const TrackSys &S, int s, const int *ipar, const double *dpar, const double *xp, int xlimbs,
                          double t, int ld, double *series, double *J, double *H) {
  typedef typename real_of<T>::type R;
  const int n = S.dim[s];
  const int K = ipar[0], L = ipar[1], M = ipar[2], off = ipar[3], nsteps = ipar[4];
  const int LP = limbs<R>::n;
  DiagOut o{1, 0, 0.0, 0.0, INFINITY, 0.0, 0.0, 0.0};
  std::vector<T> x(n);
  for (int i = 0; i < n; ++i) {
    double re[8] = {0}, im[8] = {0};
    for (int l = 0; l < LP && l < xlimbs; ++l) {
      re[l] = xp[(long)i * 2 * xlimbs + l];
      im[l] = xp[(long)i * 2 * xlimbs + xlimbs + l];
    }
    load(re, x[i].re);
    load(im, x[i].im);
  }
  bool conv = true;
  if (nsteps > 0) conv = point_newton<T, T>(S, s, t, x, nsteps, dpar[0], 1, &o.lastdx);
  std::vector<cx<double> > xd(n);
  for (int i = 0; i < n; ++i) xd[i] = cx<double>(lead_of(x[i].re), lead_of(x[i].im));
  jacobian_hessians(S, s, t, xd, ld, J, H);
  std::vector<std::vector<T> > xs(n, std::vector<T>(K + 1));
  for (int i = 0; i < n; ++i) xs[i][0] = x[i];
  {
    std::vector<std::vector<T> > x0(n, std::vector<T>(1)), h;
    std::vector<T> jac;
    for (int i = 0; i < n; ++i) x0[i][0] = x[i];
    hom_eval(S, s, 0, t, x0, h, &jac);
    lu_solver<T> lu;
    lu.factor(n, jac);
    if (lu.info != 0) {
      o.status = 1;
      o.padenorm = std::sqrt((double)n);
    }
  }
  if (o.status == 0) {
    TrackPar P{};
    P.deg = K;
    taylor_series(S, s, P, t, xs);
    int best = -1;
    R rbest = R(0.0);
    double pn = 0.0;
    for (int i = 0; i < n; ++i) {
      T z;
      double e = 0.0;
      bool fail = true;
      fabry_one(xs[i], K, off, z, e, fail);
      if (!fail) {
        const R ri = norm2(z);
        if (best < 0 || less_limbs(ri, rbest)) {
          best = i;
          rbest = ri;
          o.zre = lead_of(z.re);
          o.zim = lead_of(z.im);
          o.radius = cabs(z);
          o.err = e;
        }
      }
      std::vector<T> p, q;
      int pd = L, qd = M;
      if (!pade(L, M, xs[i], p, q)) {  // the fallback: the Taylor polynomial of degree K
        p = xs[i];
        pd = K;
        qd = 0;
      }
      const double pe = pade_error(xs[i], K, p, pd, q, qd);
      pn += pe * pe;
    }
    o.padenorm = std::sqrt(pn);
    o.fail = best < 0 ? 1 : 0;
    o.status = conv ? 0 : 2;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k <= K; ++k) store(series + ((long)i * (K + 1) + k) * 2 * LP, xs[i][k]);
  return o;
}

}  // namespace

extern "C" {

// Track npaths paths with nthreads host threads.  pmode: predictor
// precision (1 double, 2 double-double); rmode: refinement precision
// (2 dd, 4 qd, 8 od; 1 with pmode 1: all in double, corrector included);
// the corrector is double-double otherwise; step_mode 1 with a
// model buffer: the learned step.  ipar and dpar as in phc_track (dpar[8]
// = cbeta).  x0: start points, maxdim complex doubles per path; xend:
// maxdim complex quad-doubles per path (octo-doubles for rmode 8; lower
// limbs zero below the refinement precision); info: per path status,
// nsteps, nreject, nbpole, nbhess, nbmaxm; dinfo: per path t, residual.
int orc_track(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr, const int *mono_idx,
              const int *mono_exp, const int *eq_off, const int *term_off, const int *term_mono,
              const double *term_a, const double *term_b, int npaths, const int *path_sys, int maxdim,
              const double *x0, const int *ipar, const double *dpar, int pmode, int rmode, int step_mode,
              const void *model, int nthreads, double *xend, int *info, double *dinfo) {
  TrackSys S{nsys, maxvar, dim, mono_off, mono_nvr, mono_idx, mono_exp, eq_off, term_off, term_mono, term_a, term_b};
  TrackPar P;
  P.deg = ipar[0]; P.numdeg = ipar[1]; P.dendeg = ipar[2]; P.nit = ipar[3];
  P.corsteps = ipar[4]; P.maxsteps = ipar[5]; P.refine_steps = ipar[6];
  P.pbeta = dpar[0]; P.alpha = dpar[1]; P.maxsize = dpar[2]; P.minsize = dpar[3];
  P.tolres = dpar[4]; P.epsilon = dpar[5]; P.restol = dpar[6];
  P.learn_scale = dpar[7] > 0.0 ? dpar[7] : 1.0;
  P.cbeta = dpar[8];
  P.step_mode = step_mode;
  P.model = (step_mode & 1) ? static_cast<const unsigned char *>(model) : nullptr;
  if (P.numdeg + P.dendeg != P.deg || P.deg < 3 || !(P.cbeta > 0.0)) return -1;
  if (step_mode < 0 || step_mode > 3 || ((step_mode & 2) && pmode != 1)) return -1;
  // rmode 1 (with pmode 1): everything in double, the FP64 run the
  // multiple-double results are compared with
  if ((pmode != 1 && pmode != 2) || (rmode != 1 && rmode != 2 && rmode != 4 && rmode != 8)) return -1;
  if (rmode == 1 && pmode != 1) return -1;
  std::atomic<int> next(0);
  auto work = [&]() {
    for (;;) {
      const int p = next.fetch_add(1);
      if (p >= npaths) return;
      const int s = path_sys[p];
      PathOut o;
      double *xe = xend + (long)p * maxdim * (rmode == 8 ? 16 : 8);
      const double *xs = x0 + (long)p * maxdim * 2;
      if (rmode == 1) o = track_path<cx<double>, cx<double>, cx<double> >(S, s, P, xs, xe);
      else if (pmode == 1 && rmode == 2) o = track_path<cx<double>, cx<dd>, cx<dd> >(S, s, P, xs, xe);
      else if (pmode == 1 && rmode == 4) o = track_path<cx<double>, cx<dd>, cx<qd> >(S, s, P, xs, xe);
      else if (pmode == 1) o = track_path<cx<double>, cx<dd>, cx<od> >(S, s, P, xs, xe);
      else if (rmode == 2) o = track_path<cx<dd>, cx<dd>, cx<dd> >(S, s, P, xs, xe);
      else if (rmode == 4) o = track_path<cx<dd>, cx<dd>, cx<qd> >(S, s, P, xs, xe);
      else o = track_path<cx<dd>, cx<dd>, cx<od> >(S, s, P, xs, xe);
      int *io = info + 6L * p;
      io[0] = o.status;
      io[1] = o.nsteps;
      io[2] = o.nreject;
      io[3] = o.nbpole;
      io[4] = o.nbhess;
      io[5] = o.nbmaxm;
      dinfo[2 * p] = o.t;
      dinfo[2 * p + 1] = o.residual;
    }
  };
  if (nthreads <= 1) {
    work();
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(work);
    for (auto &x : th) x.join();
  }
  return 0;
}


// End-game diagnostics of npaths points (restating phc_series_diagnostics
// but for the singular values): per point x at xpt (maxdim complex numbers of
// xlimbs limbs per part) and t = tpt[p]; ipar: deg, numdeg, dendeg, offset,
// newton_steps; dpar: tolres; pmode 1, 2 or 4.  Out per point: series
// (maxdim x (deg+1) complex numbers in the working precision), dout (z re,
// z im, radius, Fabry error, Pade error norm, last Newton |dx|), iout (fail,
// status), J (maxdim^2 complex doubles, row-major) and H (maxdim^3 complex
// doubles: equation, row, column).
int orc_series_diagnostics(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                           const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                           const int *term_mono, const double *term_a, const double *term_b, int npaths,
                           const int *path_sys, int maxdim, const double *xpt, int xlimbs, const double *tpt,
                           const int *ipar, const double *dpar, int pmode, double *series, double *dout, int *iout,
                           double *J, double *H) {
  TrackSys S{nsys, maxvar, dim, mono_off, mono_nvr, mono_idx, mono_exp, eq_off, term_off, term_mono, term_a, term_b};
  const int K = ipar[0];
  if (pmode != 1 && pmode != 2 && pmode != 4) return -1;
  if (K < 3 || ipar[1] + ipar[2] > K || ipar[3] < 0 || ipar[3] > K - 2) return -1;
  for (int p = 0; p < npaths; ++p) {
    const int s = path_sys[p];
    const double *xp = xpt + (long)p * maxdim * 2 * xlimbs;
    double *se = series + (long)p * maxdim * (K + 1) * 2 * pmode;
    double *Jp = J + 2L * p * maxdim * maxdim, *Hp = H + 2L * p * maxdim * maxdim * maxdim;
    DiagOut o;
    if (pmode == 1) o = diag_point<cx<double> >(S, s, ipar, dpar, xp, xlimbs, tpt[p], maxdim, se, Jp, Hp);
    else if (pmode == 2) o = diag_point<cx<dd> >(S, s, ipar, dpar, xp, xlimbs, tpt[p], maxdim, se, Jp, Hp);
    else o = diag_point<cx<qd> >(S, s, ipar, dpar, xp, xlimbs, tpt[p], maxdim, se, Jp, Hp);
    double *d = dout + 6L * p;
    d[0] = o.zre; d[1] = o.zim; d[2] = o.radius; d[3] = o.err; d[4] = o.padenorm; d[5] = o.lastdx;
    iout[2 * p] = o.fail;
    iout[2 * p + 1] = o.status;
  }
  return 0;
}

}  // extern "C"
