// tracker.cuh -- CTA-level building blocks of the path tracker: evaluation
// of a homotopy h(x, t) = sum_terms ((1 - t) a + t b) x^e and its Jacobian at a
// vector of power series in s = t - t0, the small dense solves, the Pade
// approximants and the conversions between precisions.
#pragma once
#include "md.cuh"
#include "dense.cuh"

namespace phc {

// The large CTA-level routines are inlined at every call site (a routine
// shared by several kernel instantiations would otherwise become a call,
// with registers spilled around it); TRACK_OUTLINE=1 compiles them as calls
// instead (less code for the instruction cache).
//
// Loops stay rolled (#pragma unroll 1 on every loop of the tracker without
// a pragma of its own).  Seven paths share an SM, each in another phase of
// a step, so the code of all phases competes for the SM's instruction
// cache: with the compiler's unrolled copies of the loops over terms,
// monomials, rows and degrees the hot code of one kernel exceeded 400 KB,
// the instruction cache hit 60 % of its requests and warps stalled on
// instruction fetch about as often as on barriers; rolled, the same steps
// (bit for bit) take two thirds of the time on the 1024-path workload.
#ifndef TRACK_OUTLINE
#define TRACK_OUTLINE 0
#endif
#if TRACK_OUTLINE
#define TRACK_FN __noinline__
#else
#define TRACK_FN __forceinline__
#endif

static const int kTrackThreads = 128;
static const int kTrackKmax = 16;   // largest series degree of the predictor

// Thread numbering of the tracker's CTA.  The first warp of the numbering
// does the serial parts of a step (pivots, the point solves, the scalar
// decisions).  Warps are spread over an SM's four sub-partitions by their
// hardware slot (%warpid mod 4) and a CTA takes consecutive slots, so with
// threadIdx.x the first warps of all CTAs on an SM would queue on one
// sub-partition.  Each CTA instead numbers its threads from a lead warp
// picked by its slot: ctid() is threadIdx.x rotated by whole warps (lanes
// and warp membership unchanged).  track_pick_lead sets the rotation once
// per CTA; blockDim.x == kTrackThreads.
__shared__ int track_rot;

__device__ __forceinline__ int ctid() { return (threadIdx.x + track_rot) & (kTrackThreads - 1); }

__device__ __forceinline__ void track_pick_lead() {
  __shared__ int slot[kTrackThreads / 32];
  const int nw = kTrackThreads / 32;
  if ((threadIdx.x & 31) == 0) {
    unsigned w;
    asm volatile("mov.u32 %0, %%warpid;" : "=r"(w));
    slot[threadIdx.x >> 5] = (int)w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int mn = slot[0];
    #pragma unroll 1
    for (int v = 1; v < nw; ++v) mn = min(mn, slot[v]);
    const int want = (mn / nw) & 3;
    int lead = 0;
    #pragma unroll 1
    for (int v = nw - 1; v >= 0; --v)
      if ((slot[v] & 3) == want) lead = v;
    track_rot = (kTrackThreads - 32 * lead) & (kTrackThreads - 1);
  }
  __syncthreads();
}

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
  const int *jg_slot;    // [njg] >= 0: slot of the variable in the term's monomial (staged partial);
                         // -1: the partial is 1; -2: it is 2 x_j; -3-l: it is x_l
  int gstaged;           // some gather entry needs a staged partial
};

// A monomial of total degree <= 2 has partial derivatives that are a
// variable's series, 2 x_j or 1: they are read in place, not staged.
__host__ __device__ inline bool simple_monomial(int k, const int *ex) {
  return (k == 1 && ex[0] >= 1 && ex[0] <= 2) || (k == 2 && ex[0] == 1 && ex[1] == 1);
}

// Tracking parameters (include/phc_b200.h, phc_track: ipar and dpar)
struct TrackParDev {
  int deg, numdeg, dendeg, nit, corsteps, maxsteps, refine_steps, step_mode;
  double pbeta, alpha, maxsize, minsize, tolres, epsilon, restol, learn_scale, cbeta;
};

// Words per path of the tracker's info output: status, steps, rejected
// steps, and the times the step was the pole step, the curvature step and
// maxsize (nbpole, nbhess, nbmaxm of the reference's Minimum).
static const int kTrackInfo = 6;

// Parameters of the end-game diagnostics (include/phc_b200.h,
// phc_series_diagnostics: ipar and dpar)
struct DiagParDev {
  int deg, numdeg, dendeg, offset, newton_steps;
  double tolres, beta2;
};
static const int kDiagOut = 10;  // doubles per point in dout

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
template <> struct conv_num<md::num<md::dd, true>, md::num<md::od, true> > {
  __device__ __forceinline__ static md::cx<md::od> go(const md::cx<md::dd> &a) {
    md::cx<md::od> r;
    r.re = md::mko(a.re.hi);
    r.re.x[1] = a.re.lo;
    r.im = md::mko(a.im.hi);
    r.im.x[1] = a.im.lo;
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
//   h[i*(w+1)+k]        value series of equation i, in precision N,
//   J[(k*n + i)*n + j]  Jacobian series (when J != nullptr), in precision
//                       JN (N, or double for a Newton step whose linear
//                       solve runs in double).
// V, G: shared staging for the distinct monomials, nm*(w+1) and
// nm*maxvar*(w+1) numbers; G is written only when S.gstaged and J is wanted
// (monomials of total degree <= 2 stage no partials).
// Phase 1: one thread per distinct monomial computes its value and its
// partials (exponent included) by the common-factor method and products of
// the distinct variables.  Phase 2: the coefficient series c0 + c1 s, with
// c1 = b - a and c0 = a + t0 c1 (exactly b at t0 = 1 in double-double),
// times the monomial series, summed over the terms of an equation (one warp
// per equation, lanes over the terms, shuffle reductions) or over the
// Jacobian gather list of an (equation, variable) pair (one thread per
// pair); KC coefficients at a time, so that each term's data is loaded once
// per KC coefficients.
template <class N, int KC = 1, class JN = N>
__device__ TRACK_FN void hom_eval_cta(const TrackDev &S, int s, int w, double t0, const double *x, int xld, double *V,
                             double *G, double *h, double *J) {
  typedef typename N::T T;
  typedef typename JN::T JT;
  const int W = N::width;
  const int n = S.dim[s];
  const int n1 = w + 1;
  const int m0 = S.mono_off[s];
  const int nm = S.mono_off[s + 1] - m0;
  const int mv = S.maxvar;
  const bool stage = S.gstaged && J != nullptr;
  #pragma unroll 1
  for (int m = ctid(); m < nm; m += blockDim.x) {
    const int gm = m0 + m;
    const int k = S.mono_nvr[gm];
    const int *ix = S.mono_idx + (long)gm * mv;
    const int *ex = S.mono_exp + (long)gm * mv;
    if (k >= 1 && simple_monomial(k, ex)) {
      // value only: x_j, x_j^2 or x_j x_l (the partials are read in place)
      double *Vm = V + (long)m * n1 * W;
      const double *xa = x + (long)ix[0] * xld * W;
      const double *xb = (k == 2) ? x + (long)ix[1] * xld * W : xa;
      if (k == 1 && ex[0] == 1) {
        #pragma unroll 1
        for (int i = 0; i < n1; ++i) stn_at<N>(Vm, i, ldn_at<N>(xa, i));
      } else {
        #pragma unroll 1
        for (int kk = 0; kk < n1; ++kk) {
          T a = N::zero();
          #pragma unroll 1
          for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xa, i), ldn_at<N>(xb, kk - i)));
          stn_at<N>(Vm, kk, a);
        }
      }
      continue;
    }
    T F[kTrackKmax + 1], acc[kTrackKmax + 1];
    bool unitF = true;
    #pragma unroll 1
    for (int i = 0; i < n1; ++i) F[i] = (i == 0) ? N::one() : N::zero();
    #pragma unroll 1
    for (int v = 0; v < k; ++v)
      #pragma unroll 1
      for (int e = 1; e < ex[v]; ++e) {
        const double *xv = x + (long)ix[v] * xld * W;
        #pragma unroll 1
        for (int kk = w; kk >= 0; --kk) {  // in place: F[kk] only needs F[<= kk]
          T a = N::zero();
          #pragma unroll 1
          for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xv, i), F[kk - i]));
          F[kk] = a;
        }
        unitF = false;
      }
    double *Vm = V + (long)m * n1 * W;
    double *Gm = G + (long)m * mv * n1 * W;
    if (k == 0) {
      #pragma unroll 1
      for (int i = 0; i < n1; ++i) stn_at<N>(Vm, i, F[i]);
      continue;
    }
    #pragma unroll 1
    for (int v = 0; v < (stage ? k : 1); ++v) {
      #pragma unroll 1
      for (int i = 0; i < n1; ++i) acc[i] = F[i];
      bool unit = unitF;
      #pragma unroll 1
      for (int u = 0; u < k; ++u) {
        if (u == v) continue;
        const double *xu = x + (long)ix[u] * xld * W;
        if (unit) {
          #pragma unroll 1
          for (int i = 0; i < n1; ++i) acc[i] = ldn_at<N>(xu, i);
          unit = false;
        } else {
          #pragma unroll 1
          for (int kk = w; kk >= 0; --kk) {
            T a = N::zero();
            #pragma unroll 1
            for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xu, i), acc[kk - i]));
            acc[kk] = a;
          }
        }
      }
      if (v == 0) {
        const double *x0 = x + (long)ix[0] * xld * W;
        #pragma unroll 1
        for (int kk = 0; kk < n1; ++kk) {
          T a = N::zero();
          #pragma unroll 1
          for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(x0, i), acc[kk - i]));
          stn_at<N>(Vm, kk, a);
        }
      }
      if (!stage) continue;
      const double e = (double)ex[v];
      #pragma unroll 1
      for (int i = 0; i < n1; ++i) stn_at<N>(Gm + (long)v * n1 * W, i, e == 1.0 ? acc[i] : N::scale_d(acc[i], e));
    }
  }
  __syncthreads();
  const int e0 = S.eq_off[s];
  const int lane = ctid() & 31, warp = ctid() >> 5, nw = blockDim.x >> 5;
  #pragma unroll 1
  for (int i = warp; i < n; i += nw) {
    const int tb = S.term_off[e0 + i], te = S.term_off[e0 + i + 1];
    #pragma unroll 1
    for (int k0 = 0; k0 < n1; k0 += KC) {
      T acc[KC];
#pragma unroll
      for (int r = 0; r < KC; ++r) acc[r] = N::zero();
      #pragma unroll 1
      for (int tr = tb + lane; tr < te; tr += 32) {
        const T a = cnum<N>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
        const T b = N::sub(cnum<N>(S.term_b[2 * tr], S.term_b[2 * tr + 1]), a);  // d/dt
        const T c0 = N::add(a, N::scale_d(b, t0));
        const double *Vm = V + (long)(S.term_mono[tr] - m0) * n1 * W;
        T prev = k0 > 0 ? ldn_at<N>(Vm, k0 - 1) : N::zero();
#pragma unroll
        for (int r = 0; r < KC; ++r) {
          const int kk = k0 + r;
          if (kk < n1) {
            const T v = ldn_at<N>(Vm, kk);
            acc[r] = N::add(acc[r], N::mul(c0, v));
            if (kk > 0) acc[r] = N::add(acc[r], N::mul(b, prev));
            prev = v;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < KC; ++r)
        if (k0 + r < n1) {
          const T sum = warp_sum<N>(acc[r]);
          if (lane == 0) stn_at<N>(h, (long)i * n1 + k0 + r, sum);
        }
    }
  }
  if (J != nullptr) {
    #pragma unroll 1
    for (int it = ctid(); it < n * n; it += blockDim.x) {
      const int i = it / n, j = it % n;
      const int g = (e0 + i) * S.maxdim + j;
      const int qb = S.jg_off[g], qe = S.jg_off[g + 1];
      #pragma unroll 1
      for (int k0 = 0; k0 < n1; k0 += KC) {
        JT acc[KC];
#pragma unroll
        for (int r = 0; r < KC; ++r) acc[r] = JN::zero();
        #pragma unroll 1
        for (int q = qb; q < qe; ++q) {
          const int tr = S.jg_term[q];
          const int sl = S.jg_slot[q];
          const JT a = cnum<JN>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
          const JT b = JN::sub(cnum<JN>(S.term_b[2 * tr], S.term_b[2 * tr + 1]), a);  // d/dt
          const JT c0 = JN::add(a, JN::scale_d(b, t0));
          // the partial's series: staged (sl >= 0), the constant 1 (-1),
          // 2 x_j (-2) or x_l (-3-l)
          const double *gp = nullptr;
          if (sl >= 0) gp = G + ((long)(S.term_mono[tr] - m0) * mv + sl) * n1 * W;
          else if (sl <= -2) gp = x + (long)((sl == -2) ? j : -sl - 3) * xld * W;
          auto gload = [&](int kk) -> JT {
            if (gp == nullptr) return kk == 0 ? JN::one() : JN::zero();
            const JT v = conv_num<N, JN>::go(ldn_at<N>(gp, kk));
            return sl == -2 ? JN::add(v, v) : v;
          };
          JT prev = k0 > 0 ? gload(k0 - 1) : JN::zero();
#pragma unroll
          for (int r = 0; r < KC; ++r) {
            const int kk = k0 + r;
            if (kk < n1) {
              const JT v = gload(kk);
              acc[r] = JN::add(acc[r], JN::mul(c0, v));
              if (kk > 0) acc[r] = JN::add(acc[r], JN::mul(b, prev));
              prev = v;
            }
          }
        }
#pragma unroll
        for (int r = 0; r < KC; ++r)
          if (k0 + r < n1) stn_at<JN>(J, ((long)(k0 + r) * n + i) * n + j, acc[r]);
      }
    }
  }
  __syncthreads();
}

// Coefficient k >= 1 of the homotopy at a series truncated below degree k:
// with x_k, x_{k+1}, ... zero in x (n series, leading dimension xld numbers),
//   r[i] = [h_i(x(s), t0 + s)]_k,
// which, as h is polynomial, leaves out exactly the term J_0 x_k, so that
// x_k = -J_0^{-1} r (the recursion for Taylor coefficients of the path).
// V2: shared staging of two numbers per distinct monomial, its series
// coefficients k-1 and k.  Phase 1: one thread per monomial; phase 2: one
// warp per equation, lanes over its terms.
template <class N>
__device__ TRACK_FN void hom_coef_cta(const TrackDev &S, int s, int k, double t0, const double *x, int xld, double *V2,
                             double *r) {
  typedef typename N::T T;
  const int W = N::width;
  const int n = S.dim[s];
  const int m0 = S.mono_off[s];
  const int nm = S.mono_off[s + 1] - m0;
  const int mv = S.maxvar;
  #pragma unroll 1
  for (int m = ctid(); m < nm; m += blockDim.x) {
    const int gm = m0 + m;
    const int kv = S.mono_nvr[gm];
    const int *ix = S.mono_idx + (long)gm * mv;
    const int *ex = S.mono_exp + (long)gm * mv;
    T c1 = N::zero(), c2 = N::zero();  // coefficients k-1 and k
    if (kv == 0) {
      if (k == 1) c1 = N::one();
    } else if (simple_monomial(kv, ex)) {
      const double *xa = x + (long)ix[0] * xld * W;
      const double *xb = (kv == 2) ? x + (long)ix[1] * xld * W : xa;
      if (kv == 1 && ex[0] == 1) {
        c1 = ldn_at<N>(xa, k - 1);
        c2 = ldn_at<N>(xa, k);
      } else {
        #pragma unroll 1
        for (int i = 0; i <= k - 1; ++i) c1 = N::add(c1, N::mul(ldn_at<N>(xa, i), ldn_at<N>(xb, k - 1 - i)));
        #pragma unroll 1
        for (int i = 0; i <= k; ++i) c2 = N::add(c2, N::mul(ldn_at<N>(xa, i), ldn_at<N>(xb, k - i)));
      }
    } else {
      T F[kTrackKmax + 1];
      #pragma unroll 1
      for (int i = 0; i <= k; ++i) F[i] = (i == 0) ? N::one() : N::zero();
      #pragma unroll 1
      for (int v = 0; v < kv; ++v)
        #pragma unroll 1
        for (int e = 0; e < ex[v]; ++e) {
          const double *xv = x + (long)ix[v] * xld * W;
          #pragma unroll 1
          for (int kk = k; kk >= 0; --kk) {  // in place: F[kk] only needs F[<= kk]
            T a = N::zero();
            #pragma unroll 1
            for (int i = 0; i <= kk; ++i) a = N::add(a, N::mul(ldn_at<N>(xv, i), F[kk - i]));
            F[kk] = a;
          }
        }
      c1 = F[k - 1];
      c2 = F[k];
    }
    stn_at<N>(V2, 2L * m, c1);
    stn_at<N>(V2, 2L * m + 1, c2);
  }
  __syncthreads();
  const int e0 = S.eq_off[s];
  const int lane = ctid() & 31, warp = ctid() >> 5, nw = blockDim.x >> 5;
  #pragma unroll 1
  for (int i = warp; i < n; i += nw) {
    T acc = N::zero();
    #pragma unroll 1
    for (int tr = S.term_off[e0 + i] + lane; tr < S.term_off[e0 + i + 1]; tr += 32) {
      const T a = cnum<N>(S.term_a[2 * tr], S.term_a[2 * tr + 1]);
      const T b = N::sub(cnum<N>(S.term_b[2 * tr], S.term_b[2 * tr + 1]), a);  // d/dt
      const T c0 = N::add(a, N::scale_d(b, t0));
      const long mm = 2L * (S.term_mono[tr] - m0);
      acc = N::add(acc, N::mul(c0, ldn_at<N>(V2, mm + 1)));
      acc = N::add(acc, N::mul(b, ldn_at<N>(V2, mm)));
    }
    acc = warp_sum<N>(acc);
    if (lane == 0) stn_at<N>(r, i, acc);
  }
  __syncthreads();
}

// Exact maximum over the warp of values that are non-negative (or -1 for
// none, read as 0): doubles >= 0 order as their bit patterns, so two 32-bit
// max reductions (redux.sync), over the high words and then over the low
// words of the lanes that hold the largest high word, give the maximum
// (two instructions in place of five rounds of shuffles).
__device__ __forceinline__ double warp_max_nonneg(double v) {
  const unsigned hi = (v >= 0.0) ? (unsigned)__double2hiint(v) : 0u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned lo = (v >= 0.0 && hi == mhi) ? (unsigned)__double2loint(v) : 0u;
  const unsigned mlo = __reduce_max_sync(0xffffffffu, lo);
  return __hiloint2double((int)mhi, (int)mlo);
}

// LU factorization with partial pivoting of the n x n matrix A (row-major,
// shared memory, n <= 32), in place: lufac of
// Math_Lib/Reduction/standard_complex_linear_solvers.adb:123-178 (LINPACK's
// zgefa).  Column k pivots on the first row of largest |re| + |im| (leading
// limbs), rows k and ell swap in columns k..n-1, and the multipliers
// -a_ik / a_kk overwrite column k below the diagonal.  Besides ipvt the
// reciprocals dinv[k] = 1 / u_kk are kept for the back substitution (NaN
// for a zero pivot).  One warp alone, no CTA barrier (the other warps of the
// CTA stay free).  Per column: lane i (k <= i < n) holds a_ik and forms its
// reciprocal while the warp finds the largest candidate (warp_max_nonneg
// and one ballot), so that 1 / a_kk is a shuffle away once the pivot row is
// known; the rows swap (lanes over the columns); the (n-k-1)^2 entries of
// the trailing update are spread over the lanes, each lane forming the
// multiplier of its entry's row from column k; the multipliers are stored
// last, a lane per row.  Every entry sees zgefa's operations in their order
// (the results do not depend on the lane layout).  Called by all lanes of
// the warp; returns info to every lane: 0, or k + 1 for the first column k
// without a nonzero pivot.
template <class N>
__device__ TRACK_FN int warp_lufac(int n, double *A, int *ipvt, double *dinv) {
  typedef typename N::T T;
  const int lane = threadIdx.x & 31;
  int info = 0;
  #pragma unroll 1
  for (int k = 0; k < n; ++k) {
    const bool cand = lane >= k && lane < n;
    T a = N::zero();
    double v = -1.0;
    if (cand) {
      a = ldn_at<N>(A, (long)lane * n + k);
      v = N::lead(a);
      if (!(v == v)) v = INFINITY;  // a NaN pivot candidate reads as infinity
    }
    const T r = cand ? N::div(N::one(), a) : N::zero();
    // the largest value, then the first row that holds it (one ballot)
    const double mx = warp_max_nonneg(v);
    const unsigned hold = __ballot_sync(0xffffffffu, cand && v == mx);
    const int ix = hold ? __ffs(hold) - 1 : n;
    const int ell = ix < n ? ix : n - 1;
    if (lane == 0) ipvt[k] = ell;
    if (mx == 0.0) {
      if (info == 0) info = k + 1;  // this column is already triangularized
      if (lane == 0) stn_at<N>(dinv, k, N::from(NAN));
      __syncwarp();
      continue;
    }
    const T inv = md::shfl(r, ell);
    if (lane == 0) stn_at<N>(dinv, k, inv);
    if (ell != k)
      #pragma unroll 1
      for (int j = k + lane; j < n; j += 32) {
        const T t = ldn_at<N>(A, (long)ell * n + j);
        stn_at<N>(A, (long)ell * n + j, ldn_at<N>(A, (long)k * n + j));
        stn_at<N>(A, (long)k * n + j, t);
      }
    // lane i's entry of column k after the swap (row ell holds the old row k)
    const T ak = md::shfl(a, k);
    const T ai = (lane == ell) ? ak : a;
    const T ninv = N::neg(inv);
    __syncwarp();
    // trailing update: entry (k+1+i, k+1+j) of the m x m block at e = i m + j
    const int m = n - k - 1;
    if (m > 0) {
      int i = lane / m, j = lane - (lane / m) * m;
      const int qi = 32 / m, qj = 32 - (32 / m) * m;
      #pragma unroll 1
      for (int e = lane; e < m * m; e += 32) {
        const long o = (long)(k + 1 + i) * n + (k + 1 + j);
        const T mik = N::mul(ninv, ldn_at<N>(A, (long)(k + 1 + i) * n + k));
        stn_at<N>(A, o, N::add(ldn_at<N>(A, o), N::mul(ldn_at<N>(A, (long)k * n + k + 1 + j), mik)));
        i += qi;
        j += qj;
        if (j >= m) {
          j -= m;
          ++i;
        }
      }
    }
    __syncwarp();
    // column k is not read again by this factorization
    if (lane > k && lane < n) stn_at<N>(A, (long)lane * n + k, N::mul(ninv, ai));
  }
  __syncwarp();
  return info;
}

// Solve A x = b with the factors of warp_lufac: lusolve of
// standard_complex_linear_solvers.adb:552-583 (row interchanges applied in
// order with the multipliers, then back substitution), except that the back
// substitution multiplies by dinv[k] = 1 / u_kk where lusolve divides.
// Called by one warp alone, lane i passing b_i (n <= 32, lanes >= n pass
// zero); returns x_i in lane i.
template <class N>
__device__ typename N::T warp_lusolve(int n, const double *A, const int *ipvt, const double *dinv,
                                      typename N::T v) {
  typedef typename N::T T;
  const int lane = threadIdx.x & 31;
  // lane k's reciprocal pivot dinv[k], read once before the substitutions
  // (off the dependent chain of the back substitution)
  const T dl = (lane < n) ? ldn_at<N>(dinv, lane) : N::zero();
  #pragma unroll 1
  for (int k = 0; k < n - 1; ++k) {  // L y = P b
    const int ell = ipvt[k];
    const T t = md::shfl(v, ell);
    const T bk = md::shfl(v, k);
    if (lane == ell) v = bk;
    if (lane == k) v = t;
    if (lane > k && lane < n) v = N::add(v, N::mul(t, ldn_at<N>(A, (long)lane * n + k)));
  }
  #pragma unroll 1
  for (int kb = n - 1; kb >= 0; --kb) {  // U x = y
    if (lane == kb) v = N::mul(v, dl);
    const T t = md::shfl(v, kb);
    if (lane < kb) v = N::sub(v, N::mul(t, ldn_at<N>(A, (long)lane * n + kb)));
  }
  return v;
}

// M = A^{-1} from the factors of warp_lufac by one warp: lusolve applied to
// the columns e_c of the identity, all columns at once, each substitution
// step spread over the lanes (every entry sees the same operations in the
// same order as a column-by-column solve; an entry's row and column follow
// from the previous pass's by adding 32 = qi n + qc, without divisions).
// Called by all lanes of one warp; the caller synchronises before M is read
// by other warps.
template <class N>
__device__ TRACK_FN void warp_luinverse(int n, const double *A, const int *ipvt, const double *dinv, double *M) {
  typedef typename N::T T;
  const int lane = threadIdx.x & 31;
  const int i0 = lane / n, c0 = lane - (lane / n) * n;  // entry e = i n + c of lane's first pass
  const int qi = 32 / n, qc = 32 - (32 / n) * n;
  auto next = [&](int &i, int &c) {
    i += qi;
    c += qc;
    if (c >= n) {
      c -= n;
      ++i;
    }
  };
  {
    int i = i0, c = c0;
    #pragma unroll 1
    for (int e = lane; e < n * n; e += 32) {
      stn_at<N>(M, e, (i == c) ? N::one() : N::zero());
      next(i, c);
    }
  }
  __syncwarp();
  #pragma unroll 1
  for (int k = 0; k < n - 1; ++k) {  // L y = P e_c
    const int ell = ipvt[k];
    if (ell != k)
      #pragma unroll 1
      for (int c = lane; c < n; c += 32) {
        const T t = ldn_at<N>(M, (long)ell * n + c);
        stn_at<N>(M, (long)ell * n + c, ldn_at<N>(M, (long)k * n + c));
        stn_at<N>(M, (long)k * n + c, t);
      }
    __syncwarp();
    const int m = n - k - 1;
    int i = i0, c = c0;
    #pragma unroll 1
    for (int e = lane; e < m * n; e += 32) {
      const long o = (long)(k + 1 + i) * n + c;
      stn_at<N>(M, o, N::add(ldn_at<N>(M, o), N::mul(ldn_at<N>(M, (long)k * n + c), ldn_at<N>(A, (long)(k + 1 + i) * n + k))));
      next(i, c);
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int kb = n - 1; kb >= 0; --kb) {  // U x = y
    #pragma unroll 1
    for (int c = lane; c < n; c += 32)
      stn_at<N>(M, (long)kb * n + c, N::mul(ldn_at<N>(M, (long)kb * n + c), ldn_at<N>(dinv, kb)));
    __syncwarp();
    int j = i0, c = c0;
    #pragma unroll 1
    for (int e = lane; e < kb * n; e += 32) {
      const long o = (long)j * n + c;
      stn_at<N>(M, o, N::sub(ldn_at<N>(M, o), N::mul(ldn_at<N>(M, (long)kb * n + c), ldn_at<N>(A, (long)j * n + kb))));
      next(j, c);
    }
    __syncwarp();
  }
}

// M = A^{-1} by Householder QR, for the predictor's J_0 in complex double
// (step_mode bit 2: the predictor's solves by QR instead of LU).  Column k:
// sigma = sum_{i>k} |a_ik|^2, nu = sqrt(|a_kk|^2 + sigma), phase phi =
// a_kk / |a_kk| (1 for a_kk = 0), reflector I - tau v v^H with v = (a_kk +
// phi nu, a_{k+1,k}, ...) and tau = 2 / |v|^2, r_kk = -phi nu; the other
// columns j > k get a_j -= tau v (v^H a_j).  Then M = Q^H (the reflectors
// applied to the identity in order) and R X = M by back substitution.  A
// holds R on and above the diagonal and v below it on return; vk, tau: n
// numbers of N and n reals of scratch (shared memory).  One warp: lane 0
// forms each reflector, the lanes then own the columns (each column's sums
// run over the rows in order), so the operations and their order are those
// of a column-by-column solve.  A zero column leaves r_kk = 0 (tau = 0) and
// the inverse infinite or NaN, as a zero pivot of the LU does.
template <class N>
__device__ TRACK_FN void warp_qrinverse(int n, double *A, double *M, double *vk, double *tau) {
  typedef typename N::T T;
  typedef typename N::real R;
  typedef typename N::tr tr;
  const int lane = threadIdx.x & 31;
  #pragma unroll 1
  for (int k = 0; k < n; ++k) {
    if (lane == 0) {
      R sig = tr::zero();
      #pragma unroll 1
      for (int i = k + 1; i < n; ++i) sig = tr::add(sig, N::norm2(ldn_at<N>(A, (long)i * n + k)));
      const T xk = ldn_at<N>(A, (long)k * n + k);
      const R a2 = N::norm2(xk);
      const R nu = tr::sqrt(tr::add(a2, sig));
      T v0 = N::zero(), rkk = N::zero();
      R t = tr::zero();
      if (nu != tr::zero()) {
        T phi = N::one();
        if (a2 != tr::zero()) {
          const R ab = tr::sqrt(a2);
          phi = N::mkc(tr::div(xk.re, ab), tr::div(xk.im, ab));
        }
        v0 = N::mkc(tr::add(xk.re, tr::mul(phi.re, nu)), tr::add(xk.im, tr::mul(phi.im, nu)));
        t = tr::div(tr::from(2.0), tr::add(N::norm2(v0), sig));
        rkk = N::mkc(tr::neg(tr::mul(phi.re, nu)), tr::neg(tr::mul(phi.im, nu)));
      }
      stn_at<N>(vk, k, v0);
      tau[k] = t;
      stn_at<N>(A, (long)k * n + k, rkk);
    }
    __syncwarp();
    const T v0 = ldn_at<N>(vk, k);
    const R t = tau[k];
    #pragma unroll 1
    for (int j = k + 1 + lane; j < n; j += 32) {  // lanes over the columns to the right
      T w = N::mul(N::conj(v0), ldn_at<N>(A, (long)k * n + j));
      #pragma unroll 1
      for (int i = k + 1; i < n; ++i)
        w = N::add(w, N::mul(N::conj(ldn_at<N>(A, (long)i * n + k)), ldn_at<N>(A, (long)i * n + j)));
      w = N::mkc(tr::mul(w.re, t), tr::mul(w.im, t));
      stn_at<N>(A, (long)k * n + j, N::sub(ldn_at<N>(A, (long)k * n + j), N::mul(v0, w)));
      #pragma unroll 1
      for (int i = k + 1; i < n; ++i)
        stn_at<N>(A, (long)i * n + j, N::sub(ldn_at<N>(A, (long)i * n + j), N::mul(ldn_at<N>(A, (long)i * n + k), w)));
    }
    __syncwarp();
  }
  // M = Q^H = H_{n-1} ... H_0 I, lanes over the columns
  #pragma unroll 1
  for (int c = lane; c < n; c += 32) {
    #pragma unroll 1
    for (int i = 0; i < n; ++i) stn_at<N>(M, (long)i * n + c, i == c ? N::one() : N::zero());
    #pragma unroll 1
    for (int k = 0; k < n; ++k) {
      const R t = tau[k];
      if (t == tr::zero()) continue;
      const T v0 = ldn_at<N>(vk, k);
      T w = N::mul(N::conj(v0), ldn_at<N>(M, (long)k * n + c));
      #pragma unroll 1
      for (int i = k + 1; i < n; ++i)
        w = N::add(w, N::mul(N::conj(ldn_at<N>(A, (long)i * n + k)), ldn_at<N>(M, (long)i * n + c)));
      w = N::mkc(tr::mul(w.re, t), tr::mul(w.im, t));
      stn_at<N>(M, (long)k * n + c, N::sub(ldn_at<N>(M, (long)k * n + c), N::mul(v0, w)));
      #pragma unroll 1
      for (int i = k + 1; i < n; ++i)
        stn_at<N>(M, (long)i * n + c, N::sub(ldn_at<N>(M, (long)i * n + c), N::mul(ldn_at<N>(A, (long)i * n + k), w)));
    }
    // R X = Q^H, column c
    #pragma unroll 1
    for (int i = n - 1; i >= 0; --i) {
      T acc = ldn_at<N>(M, (long)i * n + c);
      #pragma unroll 1
      for (int j = i + 1; j < n; ++j) acc = N::sub(acc, N::mul(ldn_at<N>(A, (long)i * n + j), ldn_at<N>(M, (long)j * n + c)));
      stn_at<N>(M, (long)i * n + c, N::div(acc, ldn_at<N>(A, (long)i * n + i)));
    }
  }
  __syncwarp();
}

// ------------------------------------------------------------ singular values
// The curvature step of the predictor needs the smallest singular value of
// the Jacobian and the largest of each Hessian at the current point
// (Hesse_Pade, Curves/dobldobl_predictor_convolutions.adb:383-406; the
// reference computes full SVDs with LINPACK's zsvdc, Math_Lib/Matrices/
// dobldobl_complex_singular_values.adb).  Here one warp finds the two
// extreme singular values of an n x n complex matrix: Householder
// bidiagonalization (Golub and Kahan), then bisection with Sturm counts on
// the 2n x 2n zero-diagonal tridiagonal form of the real bidiagonal (its
// eigenvalues are +-sigma_i), 33-way per round (one trial point per lane).

__device__ __forceinline__ double2 cx_conj_mul(double2 a, double2 b) {  // conj(a) b
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}
__device__ __forceinline__ double2 cx_mul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double warp_sum_d(double a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  return a;
}

// Number of eigenvalues below x of the 2n x 2n symmetric tridiagonal with
// zero diagonal and off-diagonals c_0 = d_0, c_1 = e_0, c_2 = d_1, ...,
// c_{2n-2} = d_{n-1} (d held by lane k as dk, e as ek): the sign changes of
// its leading principal minors p_m = -x p_{m-1} - c_{m-1}^2 p_{m-2} (a zero
// minor takes the sign opposite to its predecessor), rescaled by powers of
// two to stay in range.  Every lane passes its own x.
static __device__ int gk_count(int n, double dk, double ek, double x) {
  double pm2 = 1.0, pm1 = -x;
  int cnt = pm1 < 0.0 ? 1 : 0;
  bool neg = pm1 < 0.0 || pm1 == 0.0;  // sign of p_{m-1} (a zero counts as a change)
  #pragma unroll 1
  for (int m = 1; m < 2 * n; ++m) {
    const int k = (m - 1) >> 1;
    const double c = __shfl_sync(0xffffffffu, (m - 1) & 1 ? ek : dk, k);
    const double p = fma(-x, pm1, -(c * c) * pm2);
    const bool pn = (p == 0.0) ? !neg : p < 0.0;
    cnt += (pn != neg) ? 1 : 0;
    neg = pn;
    pm2 = pm1;
    pm1 = p;
    const double s = fmax(fabs(pm1), fabs(pm2));
    if (s > 0x1p+500) {
      pm1 *= 0x1p-500;
      pm2 *= 0x1p-500;
    } else if (s < 0x1p-500 && s > 0.0) {
      pm1 *= 0x1p+500;
      pm2 *= 0x1p+500;
    }
  }
  return cnt;
}

// The eigenvalue of the Golub-Kahan form in (lo, hi] where the count first
// reaches target: 33-way bisection until hi - lo <= 2^-52 hi (at most 30
// rounds); the decisions are uniform over the warp.
static __device__ double gk_bisect(int n, double dk, double ek, double lo, double hi, int target) {
  const int lane = threadIdx.x & 31;
  #pragma unroll 1
  for (int round = 0; round < 30 && hi - lo > 0x1p-52 * hi; ++round) {
    const double x = lo + (hi - lo) * (double)(lane + 1) * (1.0 / 33.0);
    const unsigned m = __ballot_sync(0xffffffffu, gk_count(n, dk, ek, x) >= target);
    if (m == 0u) {
      lo = __shfl_sync(0xffffffffu, x, 31);
    } else {
      const int l = __ffs(m) - 1;
      const double xh = __shfl_sync(0xffffffffu, x, l);
      const double xl = __shfl_sync(0xffffffffu, x, l > 0 ? l - 1 : 0);
      if (l > 0) lo = xl;
      hi = xh;
    }
  }
  return hi;
}

// Extreme singular values (x: smallest, y: largest) of the n x n complex
// matrix A (column-major, shared memory, n <= 32; destroyed).  want: 1 the
// smallest, 2 the largest, 3 both (the other is returned as 0).  One warp,
// all lanes; a matrix with a non-finite entry gives (0, inf).
static __device__ double2 warp_singular_extremes(int n, double2 *A, int want) {
  const int lane = threadIdx.x & 31;
  double amax = 0.0;
  #pragma unroll 1
  for (int q = lane; q < n * n; q += 32) {
    const double2 a = A[q];
    const double m = fmax(fabs(a.x), fabs(a.y));
    amax = (m == m) ? fmax(amax, m) : INFINITY;
  }
  amax = warp_max(amax);
  if (amax == 0.0) return make_double2(0.0, 0.0);
  if (!(amax < INFINITY)) return make_double2(0.0, INFINITY);
  // scale by a power of two: the largest |entry| in [1, 2)
  int ex;
  frexp(amax, &ex);
  const double sc = ldexp(1.0, 1 - ex);
  #pragma unroll 1
  for (int q = lane; q < n * n; q += 32) A[q] = make_double2(A[q].x * sc, A[q].y * sc);
  __syncwarp();
  double dk = 0.0, ek = 0.0;  // lane k keeps d_k and e_k of the bidiagonal
  #pragma unroll 1
  for (int k = 0; k < n; ++k) {
    // left reflector on column k, rows k..n-1 (lanes over the rows)
    const double2 x = (lane >= k && lane < n) ? A[(long)k * n + lane] : make_double2(0.0, 0.0);
    const double s2 = warp_sum_d(lane > k && lane < n ? x.x * x.x + x.y * x.y : 0.0);
    const double2 xk = make_double2(__shfl_sync(0xffffffffu, x.x, k), __shfl_sync(0xffffffffu, x.y, k));
    const double ak = hypot(xk.x, xk.y);
    const double nrm = sqrt(fma(ak, ak, s2));
    if (lane == k) dk = nrm;
    if (s2 > 0.0) {
      // v = x - alpha e_k, alpha = -(x_k / |x_k|) |x|; tau = 2 / v^H v
      const double2 ph = ak > 0.0 ? make_double2(xk.x / ak, xk.y / ak) : make_double2(1.0, 0.0);
      const double vk = ak + nrm;
      const double tau = 2.0 / fma(vk, vk, s2);
      __syncwarp();
      if (lane == k) A[(long)k * n + k] = make_double2(ph.x * vk, ph.y * vk);
      __syncwarp();
      #pragma unroll 1
      for (int j = k + 1 + lane; j < n; j += 32) {  // lanes over the columns to the right
        double2 w = make_double2(0.0, 0.0);
        #pragma unroll 1
        for (int r = k; r < n; ++r) {
          const double2 p = cx_conj_mul(A[(long)k * n + r], A[(long)j * n + r]);
          w.x += p.x;
          w.y += p.y;
        }
        w = make_double2(w.x * tau, w.y * tau);
        #pragma unroll 1
        for (int r = k; r < n; ++r) {
          const double2 p = cx_mul(A[(long)k * n + r], w);
          A[(long)j * n + r] = make_double2(A[(long)j * n + r].x - p.x, A[(long)j * n + r].y - p.y);
        }
      }
      __syncwarp();
    }
    if (k + 1 >= n) break;
    // right reflector on row k, columns k+1..n-1 (lanes over the columns)
    const double2 y = (lane > k && lane < n) ? A[(long)lane * n + k] : make_double2(0.0, 0.0);
    const double t2 = warp_sum_d(lane > k + 1 && lane < n ? y.x * y.x + y.y * y.y : 0.0);
    const double2 yk = make_double2(__shfl_sync(0xffffffffu, y.x, k + 1), __shfl_sync(0xffffffffu, y.y, k + 1));
    const double bk = hypot(yk.x, yk.y);
    const double nr = sqrt(fma(bk, bk, t2));
    if (lane == k) ek = nr;
    if (t2 > 0.0) {
      // A <- A (I - tau conj(u) u^T) with u = y - beta e_{k+1}, beta = -(y_{k+1} / |y_{k+1}|) |y|
      const double2 ph = bk > 0.0 ? make_double2(yk.x / bk, yk.y / bk) : make_double2(1.0, 0.0);
      const double uk = bk + nr;
      const double tau = 2.0 / fma(uk, uk, t2);
      __syncwarp();
      if (lane == k) A[(long)(k + 1) * n + k] = make_double2(ph.x * uk, ph.y * uk);
      __syncwarp();
      #pragma unroll 1
      for (int r = k + 1 + lane; r < n; r += 32) {  // lanes over the rows below
        double2 z = make_double2(0.0, 0.0);
        #pragma unroll 1
        for (int c = k + 1; c < n; ++c) {
          const double2 p = cx_conj_mul(A[(long)c * n + k], A[(long)c * n + r]);
          z.x += p.x;
          z.y += p.y;
        }
        z = make_double2(z.x * tau, z.y * tau);
        #pragma unroll 1
        for (int c = k + 1; c < n; ++c) {
          const double2 p = cx_mul(z, A[(long)c * n + k]);
          A[(long)c * n + r] = make_double2(A[(long)c * n + r].x - p.x, A[(long)c * n + r].y - p.y);
        }
      }
      __syncwarp();
    }
  }
  double smin = 0.0, smax = 0.0;
  if (want & 2) {
    // sigma_max in [max entry of the bidiagonal, Gershgorin bound of the GK form]
    const double ekm = __shfl_up_sync(0xffffffffu, ek, 1);
    const double em = lane > 0 ? ekm : 0.0;
    double lo = lane < n ? fmax(dk, ek) : 0.0, hi = lane < n ? dk + fmax(ek, em) : 0.0;
    lo = warp_max(lo);
    hi = warp_max(hi);
    smax = gk_bisect(n, dk, ek, lo, hi, 2 * n) / sc;
  }
  if (want & 1) {
    // sigma_min in (0, min |d_k|] (a triangular matrix's smallest singular
    // value is at most its smallest diagonal entry)
    double hi = lane < n ? dk : INFINITY;
    #pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) hi = fmin(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    smin = hi > 0.0 ? gk_bisect(n, dk, ek, 0.0, hi, n + 1) / sc : 0.0;
  }
  return make_double2(smin, smax);
}

// Hessian of equation i of system s at (x, t) in complex double, column-
// major n x n in H; x: n complex doubles.  Lane j builds row j from the
// Jacobian gather list of (equation i, variable j): a partial that is a
// constant contributes nothing, 2 x_j gives 2c on the diagonal, x_l gives
// c at column l, and a staged partial of a monomial of degree >= 3 the
// second derivatives of c x^e by the common factors.  Deterministic: every
// cell has one writer and a fixed order.  One warp, n <= 32.
static __device__ void warp_hessian_rows(const TrackDev &S, int s, int i, int n, double t, const double2 *x, double2 *H) {
  const int j = threadIdx.x & 31;
  #pragma unroll 1
  for (int l = 0; l < n && j < n; ++l) H[(long)l * n + j] = make_double2(0.0, 0.0);
  if (j < n) {
    const int g = (S.eq_off[s] + i) * S.maxdim + j;
    #pragma unroll 1
    for (int q = S.jg_off[g]; q < S.jg_off[g + 1]; ++q) {
      const int tr = S.jg_term[q], sl = S.jg_slot[q];
      if (sl == -1) continue;
      // the coefficient (1 - t) a + t b
      const double2 c = make_double2(fma(S.term_b[2 * tr] - S.term_a[2 * tr], t, S.term_a[2 * tr]),
                                     fma(S.term_b[2 * tr + 1] - S.term_a[2 * tr + 1], t, S.term_a[2 * tr + 1]));
      if (sl == -2) {
        double2 &h = H[(long)j * n + j];
        h = make_double2(h.x + 2.0 * c.x, h.y + 2.0 * c.y);
      } else if (sl <= -3) {
        double2 &h = H[(long)(-sl - 3) * n + j];
        h = make_double2(h.x + c.x, h.y + c.y);
      } else {
        const int gm = S.term_mono[tr];
        const int nv = S.mono_nvr[gm];
        const int *ix = S.mono_idx + (long)gm * S.maxvar;
        const int *ex = S.mono_exp + (long)gm * S.maxvar;
        #pragma unroll 1
        for (int u = 0; u < nv; ++u) {
          const double mult = u == sl ? (double)ex[u] * (ex[u] - 1) : (double)ex[u] * ex[sl];
          if (mult == 0.0) continue;
          double2 acc = make_double2(c.x * mult, c.y * mult);
          #pragma unroll 1
          for (int w = 0; w < nv; ++w)
            #pragma unroll 1
            for (int e = ex[w] - (w == u) - (w == sl); e > 0; --e) acc = cx_mul(acc, x[ix[w]]);
          double2 &h = H[(long)ix[u] * n + j];
          h = make_double2(h.x + acc.x, h.y + acc.y);
        }
      }
    }
  }
  __syncwarp();
}

// |error estimate| of one component's Pade approximant (numerator degree
// pdeg, denominator degree qdeg): at the last index top <= min(pdeg + qdeg
// + 2, K) with |c_top| > 1e-5, the coefficient of the series times the
// denominator, subtracted from the numerator's when top <= pdeg; 1 when no
// coefficient passes the threshold or the estimate is below 1e-5
// (Solution_Error_Estimate and Threshold_Index,
// Curves/homotopy_pade_approximants.adb:558-568,717-754).
template <class N>
__device__ double pade_error_one(const double *c, int K, const double *num, int pdeg, const double *den, int qdeg) {
  typedef typename N::T T;
  const int endidx = min(pdeg + qdeg + 2, K);
  int top = -1;
  #pragma unroll 1
  for (int i = endidx; i >= 0; --i)
    if (N::mag(ldn_at<N>(c, i)) > 1e-5) {
      top = i;
      break;
    }
  T res = N::one();
  if (top >= 0) {
    res = ldn_at<N>(c, top);
    #pragma unroll 1
    for (int i = 1; i <= qdeg && i <= top; ++i) res = N::add(res, N::mul(ldn_at<N>(den, i), ldn_at<N>(c, top - i)));
    if (top <= pdeg) res = N::sub(ldn_at<N>(num, top), res);
  }
  const double a = N::mag(res);
  return a < 1e-5 ? 1.0 : a;
}

// y = M b, M n x n, one thread per row
template <class N>
__device__ void cta_matvec(int n, const double *M, const double *b, double *y) {
  typedef typename N::T T;
  #pragma unroll 1
  for (int i = ctid(); i < n; i += blockDim.x) {
    T acc = N::zero();
    #pragma unroll 1
    for (int j = 0; j < n; ++j) acc = N::add(acc, N::mul(ldn_at<N>(M, (long)i * n + j), ldn_at<N>(b, j)));
    stn_at<N>(y, i, acc);
  }
  __syncthreads();
}

// Shared-memory layout of a path's CTA (in doubles)
struct TrackLayout {
  long xs, V, G, hs, J0, M, r, num, den, xp, xc, hc, Jc, Vc, Gc, red, piv, dinv, feat, mag, degs, hbuf, svd, xd, sv,
      part, padw, xa, qrw, total;
};

// Matrices of the singular-value jobs of a predictor step: one per warp
// (the Hessians) and one for the Jacobian.
static const int kSvdSlots = kTrackThreads / 32 + 1;

__host__ __device__ inline TrackLayout track_layout(int n, int K, int M, int nm, int mv, int Wp, int Wr, int gst) {
  TrackLayout L;
  long o = 0;
  auto take = [&](long doubles) {
    long r = o;
    o += (doubles + 1) & ~1L;  // keep 16-byte alignment
    return r;
  };
  const long K1 = K + 1;
  // state that lives through a whole step
  L.xs = take(n * K1 * Wp);
  L.xc = take(n * Wr);
  L.num = take(n * K1 * Wp);
  L.den = take(n * (M + 1) * Wp);
  L.xp = take(n * Wp);
  const int Wm = Wp > Wr ? Wp : Wr;
  L.red = take(32 * Wm);
  L.piv = take(24);  // 32 pivot rows and the info word, as ints
  L.dinv = take(n * Wm);
  L.feat = take(32);
  L.mag = take(n * K1);
  L.degs = take(n);
  L.hbuf = take(2 * 128 + 8);
  L.svd = take((long)kSvdSlots * n * n * 2);  // complex doubles
  L.xd = take(2L * n);
  L.sv = take(n + 2);
  L.xa = take(n);  // |x_i| of the predicted point (mixed residual)
  L.qrw = take(3L * n);  // the predictor's Householder scratch (2n doubles of v_kk, n of tau)
  // scratch of the Taylor series and the predictor feedback ...
  const long ov = o;
  L.V = take(nm * 2 * Wp);  // two coefficients per monomial (point evaluations use one)
  L.G = take(gst ? nm * mv * Wp : 0);  // only monomials of degree >= 3 stage partials
  L.hs = take(n * Wp);
  L.J0 = take(n * n * Wp);
  L.M = take(n * n * Wp);
  L.r = take(n * Wp);
  L.padw = take((long)n * (M * M + 2 * M + 1) * Wp);  // the Pade systems (pade_one_ws)
  const long pend = o;
  // ... overlaid by the scratch of the corrector and the refinement, which
  // run after the Pade approximants are formed
  o = ov;
  L.hc = take(n * Wr);
  L.Jc = take(n * n * Wr);
  L.Vc = take(nm * Wr);
  L.Gc = take(gst ? nm * mv * Wr : 0);
  // partial residuals of the split corrector (double predictor, no staged
  // partials): one complex double-double per residual thread
  L.part = take(Wp == 2 && !gst ? (kTrackThreads - 32) * 4 : 0);
  L.total = o > pend ? o : pend;
  return L;
}

// Newton at a point in precision N (the corrector and the refinement):
// LU_Newton_Steps of Curves/corrector_convolutions.adb:1193-1224 restated:
// each step evaluates h(x) in precision N and J(x) in precision JN (N, or
// double in the precision-split tracker: Newton with a double Jacobian and
// a residual in N still converges to the accuracy of N, each step gaining
// about 16 digits near the solution), factors J by warp_lufac and solves
// J dx = -h(x) (a singular Jacobian ends the steps unconverged, x
// unchanged); converged when max |dx| <= tol, then extra more steps.  x
// (shared, n numbers of precision N) is updated in place; lastdx: the last
// max |dx|.
template <class N, class JN>
__device__ TRACK_FN bool point_newton(const TrackDev &S, int s, int n, double t, double *x, double *h, double *Jm, double *Vc,
                             double *Gc, int *piv, double *dinv, double *red, int maxit, double tol, int extra,
                             double *lastdx) {
  bool conv = false;
  int extra_left = extra;
  *lastdx = 1e300;
  #pragma unroll 1
  for (int it = 0; it < maxit + extra; ++it) {
    if (it >= maxit && !conv) break;
    hom_eval_cta<N, 1, JN>(S, s, 0, t, x, 1, Vc, Gc, h, Jm);
    if (ctid() < 32) {
      const int lane = ctid();
      const int info = warp_lufac<JN>(n, Jm, piv, dinv);
      typename JN::T b = JN::zero();
      if (lane < n) b = JN::neg(conv_num<N, JN>::go(ldn_at<N>(h, lane)));
      const typename JN::T v = warp_lusolve<JN>(n, Jm, piv, dinv, b);
      double m = 0.0;
      if (lane < n) {
        m = JN::mag(v);
        if (!(m == m)) m = INFINITY;
        if (info == 0) stn_at<N>(x, lane, N::add(ldn_at<N>(x, lane), conv_num<JN, N>::go(v)));
      }
      m = warp_max_nonneg(m);
      if (lane == 0) red[0] = info ? INFINITY : m;
    }
    __syncthreads();
    const double m = red[0];
    __syncthreads();
    *lastdx = m;
    if (!(m <= 1e300)) return false;
    if (conv) {
      if (--extra_left <= 0) break;
    } else if (m <= tol) {
      conv = true;
      if (extra_left <= 0) break;
    }
  }
  return conv;
}

// Compensated sum (Sum2 of Ogita, Rump and Oishi, 2005) of products of a
// double and a double-double: two error-free transformations per product,
// the rounding errors gathered in e; s + e carries about double-double
// accuracy.
struct sum2 {
  double s, e;
  __device__ __forceinline__ void zero() {
    s = 0.0;
    e = 0.0;
  }
  __device__ __forceinline__ void add_prod(double a, const md::dd &v) {
    double ep, es;
    const double p = md::two_prod(a, v.hi, ep);
    s = md::two_sum(s, p, es);
    e = __fma_rn(a, v.lo, md::add(e, md::add(es, ep)));
  }
  __device__ __forceinline__ md::dd value() const {
    md::dd r;
    r.hi = md::two_sum(s, e, r.lo);
    return r;
  }
};

// Barrier of the three residual warps of the split corrector (named
// barrier 1; the lead warp does not take part).
__device__ __forceinline__ void residual_warps_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kTrackThreads - 32) : "memory");
}

// First of the G residual threads that work on equation i when the n
// equations (ci terms before equation i, T terms in all) share them in
// proportion to their terms, each at least one: strictly increasing in i,
// from 0 at i = 0 to G at i = n.
__device__ __forceinline__ int eq_first_thread(int i, int n, int G, int ci, int T) {
  return i + (T > 0 ? (int)((long long)(G - n) * ci / T) : 0);
}

// The corrector's Newton steps with a double Jacobian (the precision-split
// tracker, for systems that stage no partials): the same steps, tests and
// results as point_newton<N, double> (Curves/corrector_convolutions.adb
// :1193-1224, LU_Newton_Steps), with the work of an iteration split over
// the CTA.  First all threads evaluate J(x) in complex double from the
// Jacobian gather lists at the double copy xj of x (one entry per thread)
// and the values x^e of the system's distinct monomials in double-double
// (into V, one monomial per thread).  Then the lead warp factors J while
// the other three warps form h(x, t): the terms of each equation go to a
// group of threads (in proportion to the terms, eq_first_thread), each
// thread accumulates P = sum b x^e and Q = sum a x^e with compensated sums,
// its share of h is Q + t (P - Q), and the first thread of the group adds
// the shares in order.  Last the lead warp solves, updates x (n numbers of
// N, double-double, in shared memory) and xj.  V: the distinct monomials,
// numbers of N; part: (kTrackThreads - 32) numbers of N.
template <class N>
__device__ TRACK_FN bool point_newton_split(const TrackDev &S, int s, int n, double t, double *x, double *h,
                                            double *Jm, double2 *xj, double *V, double *part, int *piv,
                                            double *dinv, double *red, int maxit, double tol, int extra,
                                            double *lastdx) {
  typedef md::num<double, true> JN;
  typedef typename N::T T;
  const int G = kTrackThreads - 32;
  const int e0 = S.eq_off[s];
  const int m0 = S.mono_off[s], nm = S.mono_off[s + 1] - m0;
  const int tb0 = S.term_off[e0], nterm = S.term_off[e0 + n] - tb0;
  // residual thread ri: equation req, position rk in a group of rg threads
  const int ri = ctid() - 32;
  int req = 0, rk = 0, rg = 1;
  if (ri >= 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (eq_first_thread(mid, n, G, S.term_off[e0 + mid] - tb0, nterm) <= ri) lo = mid;
      else hi = mid - 1;
    }
    req = lo;
    const int f0 = eq_first_thread(lo, n, G, S.term_off[e0 + lo] - tb0, nterm);
    const int f1 = lo + 1 < n ? eq_first_thread(lo + 1, n, G, S.term_off[e0 + lo + 1] - tb0, nterm) : G;
    rk = ri - f0;
    rg = f1 - f0;
  }
  auto to_d2 = [](const T &v) {
    return make_double2(__dadd_rn(v.re.hi, v.re.lo), __dadd_rn(v.im.hi, v.im.lo));
  };
  if (ctid() < n) xj[ctid()] = to_d2(ldn_at<N>(x, ctid()));
  __syncthreads();
  bool conv = false;
  int extra_left = extra;
  int info = 0;
  *lastdx = 1e300;
  #pragma unroll 1
  for (int it = 0; it < maxit + extra; ++it) {
    if (it >= maxit && !conv) break;
    // J(x) in complex double, one entry per thread
    #pragma unroll 1
    for (int e = ctid(); e < n * n; e += kTrackThreads) {
      const int i = e / n, j = e % n;
      const int g = (e0 + i) * S.maxdim + j;
      double2 acc = make_double2(0.0, 0.0);
      #pragma unroll 1
      for (int q = S.jg_off[g]; q < S.jg_off[g + 1]; ++q) {
        const int tr = S.jg_term[q], sl = S.jg_slot[q];
        const double ar = S.term_a[2 * tr], ai = S.term_a[2 * tr + 1];
        const double2 c = make_double2(fma(S.term_b[2 * tr] - ar, t, ar), fma(S.term_b[2 * tr + 1] - ai, t, ai));
        double2 v;
        if (sl == -1) v = make_double2(1.0, 0.0);
        else if (sl == -2) v = make_double2(2.0 * xj[j].x, 2.0 * xj[j].y);
        else v = xj[-sl - 3];
        acc.x = fma(c.x, v.x, fma(-c.y, v.y, acc.x));
        acc.y = fma(c.x, v.y, fma(c.y, v.x, acc.y));
      }
      reinterpret_cast<double2 *>(Jm)[e] = acc;
    }
    // the distinct monomials x^e in double-double, one per thread
    #pragma unroll 1
    for (int m = ctid(); m < nm; m += kTrackThreads) {
      const int gm = m0 + m;
      const int nv = S.mono_nvr[gm];
      const int *ix = S.mono_idx + (long)gm * S.maxvar;
      const int *ex = S.mono_exp + (long)gm * S.maxvar;
      T v = N::one();
      bool unit = true;
      #pragma unroll 1
      for (int u = 0; u < nv; ++u) {
        const T xu = ldn_at<N>(x, ix[u]);
        #pragma unroll 1
        for (int q = 0; q < ex[u]; ++q) {
          v = unit ? xu : N::mul(v, xu);
          unit = false;
        }
      }
      stn_at<N>(V, m, v);
    }
    __syncthreads();
    if (ctid() < 32) {
      info = warp_lufac<JN>(n, Jm, piv, dinv);
    } else {
      sum2 pr, pi, qr, qi;
      pr.zero(); pi.zero(); qr.zero(); qi.zero();
      #pragma unroll 1
      for (int tr = S.term_off[e0 + req] + rk; tr < S.term_off[e0 + req + 1]; tr += rg) {
        const T v = ldn_at<N>(V, S.term_mono[tr] - m0);
        const double ar = S.term_a[2 * tr], ai = S.term_a[2 * tr + 1];
        const double br = S.term_b[2 * tr], bi = S.term_b[2 * tr + 1];
        pr.add_prod(br, v.re);
        pr.add_prod(-bi, v.im);
        pi.add_prod(br, v.im);
        pi.add_prod(bi, v.re);
        qr.add_prod(ar, v.re);
        qr.add_prod(-ai, v.im);
        qi.add_prod(ar, v.im);
        qi.add_prod(ai, v.re);
      }
      T P, Q;
      P.re = pr.value();
      P.im = pi.value();
      Q.re = qr.value();
      Q.im = qi.value();
      stn_at<N>(part, ri, N::add(Q, N::scale_d(N::sub(P, Q), t)));
      residual_warps_sync();
      if (rk == 0) {
        T acc = ldn_at<N>(part, ri);
        #pragma unroll 1
        for (int k = 1; k < rg; ++k) acc = N::add(acc, ldn_at<N>(part, ri + k));
        stn_at<N>(h, req, acc);
      }
    }
    __syncthreads();
    if (ctid() < 32) {
      const int lane = ctid();
      typename JN::T b = JN::zero();
      if (lane < n) b = JN::neg(conv_num<N, JN>::go(ldn_at<N>(h, lane)));
      const typename JN::T v = warp_lusolve<JN>(n, Jm, piv, dinv, b);
      double m = 0.0;
      if (lane < n) {
        m = JN::mag(v);
        if (!(m == m)) m = INFINITY;
        if (info == 0) {
          const T xn = N::add(ldn_at<N>(x, lane), conv_num<JN, N>::go(v));
          stn_at<N>(x, lane, xn);
          xj[lane] = to_d2(xn);
        }
      }
      m = warp_max_nonneg(m);
      if (lane == 0) red[0] = info ? INFINITY : m;
    }
    __syncthreads();
    const double m = red[0];
    __syncthreads();
    *lastdx = m;
    if (!(m <= 1e300)) return false;
    if (conv) {
      if (--extra_left <= 0) break;
    } else if (m <= tol) {
      conv = true;
      if (extra_left <= 0) break;
    }
  }
  return conv;
}

// Pade [L/M] of component i's series c (K+1 numbers), Gaussian elimination
// with partial pivoting on the M x M system; Taylor fallback when singular.
// Curves/standard_rational_approximations.ads:67-100.  Returns the numerator
// degree used (L, or K for the fallback); the denominator degree is M or 0.
template <class N>
__device__ TRACK_FN int pade_one(int L, int M, int K, const double *c, double *num, double *den) {
  typedef typename N::T T;
  T A[kTrackKmax * kTrackKmax / 4 + 16], b[kTrackKmax / 2 + 8], q[kTrackKmax / 2 + 9];
  bool ok = true;
  #pragma unroll 1
  for (int i = 1; i <= M; ++i) {
    #pragma unroll 1
    for (int j = 1; j <= M; ++j) {
      const int k = L + i - j;
      A[(i - 1) * M + (j - 1)] = k >= 0 ? ldn_at<N>(c, k) : N::zero();
    }
    b[i - 1] = N::neg(ldn_at<N>(c, L + i));
  }
  #pragma unroll 1
  for (int col = 0; col < M && ok; ++col) {
    int piv = col;
    double best = N::mag(A[col * M + col]);
    #pragma unroll 1
    for (int r = col + 1; r < M; ++r) {
      const double m = N::mag(A[r * M + col]);
      if (m > best) { best = m; piv = r; }
    }
    if (!(best > 0.0)) { ok = false; break; }
    if (piv != col) {
      #pragma unroll 1
      for (int j = 0; j < M; ++j) { T tt = A[piv * M + j]; A[piv * M + j] = A[col * M + j]; A[col * M + j] = tt; }
      T tt = b[piv]; b[piv] = b[col]; b[col] = tt;
    }
    #pragma unroll 1
    for (int r = col + 1; r < M; ++r) {
      const T f = N::div(A[r * M + col], A[col * M + col]);
      #pragma unroll 1
      for (int j = col; j < M; ++j) A[r * M + j] = N::sub(A[r * M + j], N::mul(f, A[col * M + j]));
      b[r] = N::sub(b[r], N::mul(f, b[col]));
    }
  }
  q[0] = N::one();
  if (ok) {
    #pragma unroll 1
    for (int i = M - 1; i >= 0; --i) {
      T acc = b[i];
      #pragma unroll 1
      for (int j = i + 1; j < M; ++j) acc = N::sub(acc, N::mul(A[i * M + j], q[j + 1]));
      q[i + 1] = N::div(acc, A[i * M + i]);
    }
    #pragma unroll 1
    for (int i = 0; i <= M; ++i) stn_at<N>(den, i, q[i]);
    #pragma unroll 1
    for (int i = 0; i <= L; ++i) {
      T acc = N::zero();
      #pragma unroll 1
      for (int j = 0; j <= (i < M ? i : M); ++j) acc = N::add(acc, N::mul(q[j], ldn_at<N>(c, i - j)));
      stn_at<N>(num, i, acc);
    }
    return L;
  }
  stn_at<N>(den, 0, N::one());
  #pragma unroll 1
  for (int i = 0; i <= K; ++i) stn_at<N>(num, i, ldn_at<N>(c, i));
  return K;
}

// pade_one with the M x M system, its right hand side and the denominator in
// shared memory (w: M*M + 2*M + 1 numbers of N) instead of per-thread local
// arrays: the same operations in the same order, so the same results.  In
// the tracker's CTA the local arrays of the threads that form the
// approximants outgrow the L1 cache left beside the shared memory of eight
// paths, and every access of the elimination would go to L2.
template <class N>
__device__ TRACK_FN int pade_one_ws(int L, int M, int K, const double *c, double *num, double *den, double *w) {
  typedef typename N::T T;
  const int W = N::width;
  double *A = w, *b = w + (long)M * M * W, *q = w + (long)(M * M + M) * W;
  auto a_at = [&](int i, int j) { return ldn_at<N>(A, (long)i * M + j); };
  bool ok = true;
  #pragma unroll 1
  for (int i = 1; i <= M; ++i) {
    #pragma unroll 1
    for (int j = 1; j <= M; ++j) {
      const int k = L + i - j;
      stn_at<N>(A, (long)(i - 1) * M + (j - 1), k >= 0 ? ldn_at<N>(c, k) : N::zero());
    }
    stn_at<N>(b, i - 1, N::neg(ldn_at<N>(c, L + i)));
  }
  #pragma unroll 1
  for (int col = 0; col < M && ok; ++col) {
    int piv = col;
    double best = N::mag(a_at(col, col));
    #pragma unroll 1
    for (int r = col + 1; r < M; ++r) {
      const double m = N::mag(a_at(r, col));
      if (m > best) { best = m; piv = r; }
    }
    if (!(best > 0.0)) { ok = false; break; }
    if (piv != col) {
      #pragma unroll 1
      for (int j = 0; j < M; ++j) {
        const T tt = a_at(piv, j);
        stn_at<N>(A, (long)piv * M + j, a_at(col, j));
        stn_at<N>(A, (long)col * M + j, tt);
      }
      const T tt = ldn_at<N>(b, piv);
      stn_at<N>(b, piv, ldn_at<N>(b, col));
      stn_at<N>(b, col, tt);
    }
    const T acc = a_at(col, col);
    const T bc = ldn_at<N>(b, col);
    #pragma unroll 1
    for (int r = col + 1; r < M; ++r) {
      const T f = N::div(a_at(r, col), acc);
      #pragma unroll 1
      for (int j = col; j < M; ++j) stn_at<N>(A, (long)r * M + j, N::sub(a_at(r, j), N::mul(f, a_at(col, j))));
      stn_at<N>(b, r, N::sub(ldn_at<N>(b, r), N::mul(f, bc)));
    }
  }
  stn_at<N>(q, 0, N::one());
  if (ok) {
    #pragma unroll 1
    for (int i = M - 1; i >= 0; --i) {
      T acc = ldn_at<N>(b, i);
      #pragma unroll 1
      for (int j = i + 1; j < M; ++j) acc = N::sub(acc, N::mul(a_at(i, j), ldn_at<N>(q, j + 1)));
      stn_at<N>(q, i + 1, N::div(acc, a_at(i, i)));
    }
    #pragma unroll 1
    for (int i = 0; i <= M; ++i) stn_at<N>(den, i, ldn_at<N>(q, i));
    #pragma unroll 1
    for (int i = 0; i <= L; ++i) {
      T acc = N::zero();
      #pragma unroll 1
      for (int j = 0; j <= (i < M ? i : M); ++j) acc = N::add(acc, N::mul(ldn_at<N>(q, j), ldn_at<N>(c, i - j)));
      stn_at<N>(num, i, acc);
    }
    return L;
  }
  stn_at<N>(den, 0, N::one());
  #pragma unroll 1
  for (int i = 0; i <= K; ++i) stn_at<N>(num, i, ldn_at<N>(c, i));
  return K;
}

}  // namespace phc
