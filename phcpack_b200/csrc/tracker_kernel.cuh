// tracker_kernel.cuh -- batched series-Pade path tracking on the GPU: the
// kernel and its launch, compiled in two units (tracker.cu for the
// double-double predictor, tracker_fp64.cu for the double predictor of the
// precision-split tracker) so that they build in parallel.
//
// A persistent kernel: each CTA repeatedly takes the next path from an
// on-device work queue (one atomicAdd; no waiting on other CTAs) and tracks
// it from t = 0 to t = 1, so paths of uneven length balance across the SMs;
// a batch that fits in one wave maps CTA b to path b instead.
// Per step (the Ada Predictor_Corrector_Loop, predictor_corrector_loops.adb
// :37-85, restated):
//   predictor, in PN precision (double or double-double):
//     the Taylor series of the path in s = t - t0 to degree K, one
//     coefficient at a time with the LU of J_0 (factored and J_0^{-1}
//     formed once per predictor step);
//     [L/M] Pade approximant per component; pole step pbeta * r, r the
//     smallest Fabry radius |c_{K-3}/c_{K-2}|; step <= maxsize, cut at t = 1;
//     predictor feedback: halve until the mixed residual < alpha;
//   corrector: at most corsteps LU Newton steps with residuals and updates
//     in double-double and the Jacobian and its solve in PN precision,
//     converged when max |dx| <= tolres, plus one extra step; on failure
//     halve the step;
//   the step size comes from a learned model when one is given (step_mode
//     bit 1): a proposal whose corrector fails is rejected and the step is
//     redone with the plain pole step; step_mode bit 2 (double predictor):
//     J_0 is inverted by Householder QR instead of LU;
//   at t = 1: refinement in RN precision (double-, quad- or octo-double) and
//     classification by the max-norm residual.
// Every loop is bounded (maxsteps, halvings down to minsize); nothing waits.
#pragma once
#include "common.cuh"
#include "tracker.cuh"
#include "mlp.cuh"
#include "../../include/phc_b200.h"

#ifndef TRACK_MINB
#define TRACK_MINB 8
#endif

namespace phc {


template <class N>
__device__ double cta_maxmag(int n, const double *v, double *red) {
  double a = 0.0;
  #pragma unroll 1
  for (int i = ctid(); i < n; i += blockDim.x) {
    const double m = N::mag(ldn_at<N>(v, i));
    a = (m != m) ? INFINITY : fmax(a, m);  // a NaN reads as infinity
  }
  return block_max(a, red);
}

// max_i |h_i(x, t)| at a point, in precision N
template <class N>
__device__ double point_residual(const TrackDev &S, int s, int n, double t, const double *x, double *h, double *Vc,
                                 double *Gc, double *red) {
  hom_eval_cta<N>(S, s, 0, t, x, 1, Vc, Gc, h, nullptr);
  return cta_maxmag<N>(n, h, red);
}

template <class N>
__device__ typename N::T horner(const double *a, int deg, const typename N::T &z) {
  typename N::T acc = ldn_at<N>(a, deg);
  #pragma unroll 1
  for (int i = deg - 1; i >= 0; --i) acc = N::add(N::mul(acc, z), ldn_at<N>(a, i));
  return acc;
}

// Evaluate the Pade approximants at step st into xp, and return the mixed
// residual (1/n) sum_i |h_i(xp, t+st)| / (|h|_i(|xp|, t+st) + 1) of
// Solutions/standard_mixed_residuals.adb:472, where |h| has the moduli of
// the coefficients at t+st.  Predictor_Feedback,
// Curves/standard_predictor_convolutions.adb:958-993.
template <class PN>
__device__ TRACK_FN double pade_mixres(const TrackDev &S, int s, int n, int K, int dendeg, double t, double st,
                              const double *num, const double *den, const int *degs, double *xp, double *xa,
                              double *V, double *G, double *hs, double *red) {
  const int Wp = PN::width;
  #pragma unroll 1
  for (int i = ctid(); i < n; i += blockDim.x) {
    const typename PN::T z = PN::from(st);
    const typename PN::T nv = horner<PN>(num + (long)i * (K + 1) * Wp, degs[2 * i], z);
    const typename PN::T dv = horner<PN>(den + (long)i * (dendeg + 1) * Wp, degs[2 * i + 1], z);
    const typename PN::T xi = PN::div(nv, dv);
    stn_at<PN>(xp, i, xi);
    xa[i] = PN::mag(xi);
  }
  __syncthreads();
  hom_eval_cta<PN>(S, s, 0, t + st, xp, 1, V, G, hs, nullptr);
  // one warp per equation, lanes over its terms
  const int lane = ctid() & 31, warp = ctid() >> 5, nw = blockDim.x >> 5;
  double part = 0.0;
  #pragma unroll 1
  for (int i = warp; i < n; i += nw) {
    double ab = 0.0;
    const int eq = S.eq_off[s] + i;
    #pragma unroll 1
    for (int tr = S.term_off[eq] + lane; tr < S.term_off[eq + 1]; tr += 32) {
      const int gm = S.term_mono[tr];
      // |(1 - t') a + t' b| at t' = t + st
      double v = hypot(fma(S.term_b[2 * tr] - S.term_a[2 * tr], t + st, S.term_a[2 * tr]),
                       fma(S.term_b[2 * tr + 1] - S.term_a[2 * tr + 1], t + st, S.term_a[2 * tr + 1]));
      #pragma unroll 1
      for (int u = 0; u < S.mono_nvr[gm]; ++u) {
        const double xu = xa[S.mono_idx[(long)gm * S.maxvar + u]];
        #pragma unroll 1
        for (int e = 0; e < S.mono_exp[(long)gm * S.maxvar + u]; ++e) v *= xu;
      }
      ab += v;
    }
    #pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) ab += __shfl_xor_sync(0xffffffffu, ab, o);
    if (lane == 0) part += PN::mag(ldn_at<PN>(hs, i)) / (ab + 1.0);
  }
  return block_sum<md::num<double, false> >(part, red) / n;
}

// The corrector's Newton steps at t (x: n numbers of CN in shared memory):
// the split form of point_newton_split when the predictor is in double and
// the system stages no partials, point_newton otherwise.
template <class CN, class PN>
__device__ TRACK_FN bool corrector_newton(const TrackDev &S, int s, int n, double t, double *x, double *sm,
                                          const TrackLayout &L, int *piv, double *dinv, double *red, int maxit,
                                          double tol, int extra, double *lastdx) {
  if constexpr (PN::width == 2 && CN::width == 4) {
    if (!S.gstaged)
      return point_newton_split<CN>(S, s, n, t, x, sm + L.hc, sm + L.Jc, reinterpret_cast<double2 *>(sm + L.xd),
                                    sm + L.Vc, sm + L.part, piv, dinv, red, maxit, tol, extra, lastdx);
  }
  return point_newton<CN, PN>(S, s, n, t, x, sm + L.hc, sm + L.Jc, sm + L.Vc, sm + L.Gc, piv, dinv, red, maxit, tol,
                              extra, lastdx);
}

// Track the paths of one CTA.  PN: predictor numbers, CN: corrector
// (double-double), RN: refinement.  Output per path: xend (maxdim complex
// quad-doubles), info (status, steps, rejected), dinfo (t, residual).
// Resident CTAs per SM asked of the compiler (a register budget): 8 for the
// precision-split tracker (double predictor, double-double refinement), whose
// shared memory per path is small enough for 8 paths per SM; 1 otherwise.
// The WIDE variant of the split tracker asks for one CTA fewer (72 registers
// per thread instead of 64: fewer spills, each step a little faster); a batch
// that fits on the GPU in one wave at that occupancy is launched with it.
template <class PN, class RN, bool WIDE>
struct track_min_blocks {
  static const bool split = PN::width <= 2 && RN::width <= 4;
  static const int value = split ? (WIDE ? TRACK_MINB - 1 : TRACK_MINB) : 1;
};

template <class PN, class CN, class RN, bool WIDE>
__global__ void __launch_bounds__(kTrackThreads, (track_min_blocks<PN, RN, WIDE>::value))
    k_track(TrackDev S, TrackParDev P, int npaths, int path_begin, const int *__restrict__ path_sys,
            const double *__restrict__ x0, int *queue, const float *__restrict__ model, double *__restrict__ xend,
            int *__restrict__ info, double *__restrict__ dinfo, float *__restrict__ log, int log_cap,
            int *__restrict__ log_count) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int cur;
  const int K = P.deg;
  const int Wp = PN::width, Wr = RN::width;
  const int n_max = S.maxdim;
  int nm_max = 0;
  #pragma unroll 1
  for (int s = 0; s < S.nsys; ++s) nm_max = max(nm_max, S.mono_off[s + 1] - S.mono_off[s]);
  const TrackLayout L = track_layout(n_max, K, P.dendeg, nm_max, S.maxvar, Wp, Wr, S.gstaged);
  double *red = sm + L.red;
  int *piv = reinterpret_cast<int *>(sm + L.piv);
  double *dinv = sm + L.dinv;
  track_pick_lead();
  int next_static = blockIdx.x;
  #pragma unroll 1
  for (;;) {
    if (queue) {
      if (ctid() == 0) cur = atomicAdd(queue, 1);
      __syncthreads();
    } else {
      if (ctid() == 0) cur = next_static;
      __syncthreads();
      next_static += gridDim.x;
    }
    const int p = cur;
    __syncthreads();
    if (p >= npaths) break;
    const int path = path_begin + p;
    const int s = path_sys[path];
    const int n = S.dim[s];
    double *xc = sm + L.xc;
    // start point, refined at t = 0
    #pragma unroll 1
    for (int i = ctid(); i < n; i += blockDim.x) {
      const double *z = x0 + ((long)path * n_max + i) * 2;
      stn_at<CN>(xc, i, cnum<CN>(z[0], z[1]));
    }
    __syncthreads();
    double t = 0.0, dxn;
    corrector_newton<CN, PN>(S, s, n, 0.0, xc, sm, L, piv, dinv, red, P.corsteps, P.tolres, 1, &dxn);
    int status = 2, nsteps = 0, nrej = 0, nbpole = 0, nbhess = 0, nbmaxm = 0;
    bool failed = false;
    #pragma unroll 1
    for (int step_it = 0; step_it < P.maxsteps; ++step_it) {
      // ---------------- predictor: the Taylor series of the path in PN
      // x(s) = x_0 + x_1 s + ... + x_K s^K solves h(x(s), t + s) = 0 to
      // degree K.  Its coefficients follow one degree at a time from the
      // LU of J_0 = dh/dx at the point: x_k = -J_0^{-1} [h(x_0 + ... +
      // x_{k-1} s^{k-1}, t + s)]_k.  This is the fixed point that Newton's
      // method on power series (LU_Prediction,
      // Curves/standard_predictor_convolutions.adb:1142-1185, J_0 factored
      // once by lufac) converges to, computed without the Jacobian series:
      // K coefficient evaluations and K products with J_0^{-1}.
      double *xs = sm + L.xs;
      #pragma unroll 1
      for (int t2 = ctid(); t2 < n * (K + 1); t2 += blockDim.x) {
        const int i = t2 / (K + 1), k = t2 % (K + 1);
        typename PN::T v = PN::zero();
        if (k == 0) v = conv_num<CN, PN>::go(ldn_at<CN>(xc, i));
        stn_at<PN>(xs, t2, v);
      }
      __syncthreads();
      hom_eval_cta<PN>(S, s, 0, t, xs, K + 1, sm + L.V, sm + L.G, sm + L.hs, sm + L.J0);
      // the Jacobian and the point in complex double for the singular values
      double2 *svd = reinterpret_cast<double2 *>(sm + L.svd);
      double2 *xd = reinterpret_cast<double2 *>(sm + L.xd);
      double *sv = sm + L.sv;
      #pragma unroll 1
      for (int q = ctid(); q < n * n; q += blockDim.x) {
        const typename PN::T v = ldn_at<PN>(sm + L.J0, q);
        svd[(long)(kSvdSlots - 1) * n * n + q] = make_double2(md::lead(v.re), md::lead(v.im));
      }
      #pragma unroll 1
      for (int i = ctid(); i < n; i += blockDim.x) {
        const typename PN::T v = ldn_at<PN>(xs, (long)i * (K + 1));
        xd[i] = make_double2(md::lead(v.re), md::lead(v.im));
      }
      __syncthreads();
      // the lead warp factors J_0 and forms its inverse; meanwhile the other
      // warps form the Hessians at the point and their Frobenius norms, upper
      // bounds of their largest singular values (sv[i] = |H_i|_F^2)
      if (ctid() < 32) {
        bool by_qr = false;  // step_mode bit 2: J_0 by Householder QR (double predictor)
        if constexpr (PN::width == 2) {
          by_qr = (P.step_mode & 2) != 0;
          if (by_qr) warp_qrinverse<PN>(n, sm + L.J0, sm + L.M, sm + L.qrw, sm + L.qrw + 2 * n);
        }
        if (!by_qr) {
          warp_lufac<PN>(n, sm + L.J0, piv, dinv);
          warp_luinverse<PN>(n, sm + L.J0, piv, dinv, sm + L.M);
        }
      } else {
        const int hw = (ctid() >> 5), nhw = kTrackThreads / 32 - 1;
        #pragma unroll 1
        for (int i = hw - 1; i < n; i += nhw) {
          double2 *H = svd + (long)hw * n * n;
          warp_hessian_rows(S, s, i, n, t, xd, H);
          double f = 0.0;
          #pragma unroll 1
          for (int q = ctid() & 31; q < n * n; q += 32) f = fma(H[q].x, H[q].x, fma(H[q].y, H[q].y, f));
          f = warp_sum_d(f);
          if ((ctid() & 31) == 0) sv[i] = f;
        }
      }
      __syncthreads();
      #pragma unroll 1
      for (int k = 1; k <= K; ++k) {
        hom_coef_cta<PN>(S, s, k, t, xs, K + 1, sm + L.V, sm + L.r);
        #pragma unroll 1
        for (int i = ctid(); i < n; i += blockDim.x) {
          typename PN::T acc = PN::zero();
          #pragma unroll 1
          for (int j = 0; j < n; ++j)
            acc = PN::add(acc, PN::mul(ldn_at<PN>(sm + L.M, (long)i * n + j), ldn_at<PN>(sm + L.r, j)));
          stn_at<PN>(xs, (long)i * (K + 1) + k, PN::neg(acc));
        }
        __syncthreads();
      }
      // ---------------- Pade, the pole step and the curvature step
      int pdeg_i = 0, qdeg_i = 0;
      double rmin = 1e300, perr2 = 0.0;
      double *num = sm + L.num, *den = sm + L.den;
      #pragma unroll 1
      for (int i = ctid(); i < n; i += blockDim.x) {
        const double *ci = xs + (long)i * (K + 1) * Wp;
        double *numi = num + (long)i * (K + 1) * Wp, *deni = den + (long)i * (P.dendeg + 1) * Wp;
        pdeg_i = pade_one_ws<PN>(P.numdeg, P.dendeg, K, ci, numi, deni,
                                 sm + L.padw + (long)i * (P.dendeg * P.dendeg + 2 * P.dendeg + 1) * Wp);
        qdeg_i = (pdeg_i == P.numdeg) ? P.dendeg : 0;
        const double pe = pade_error_one<PN>(ci, K, numi, pdeg_i, deni, qdeg_i);
        perr2 = fma(pe, pe, perr2);
        const double cd = PN::mag(ldn_at<PN>(ci, K - 2));
        if (cd != 0.0) rmin = fmin(rmin, PN::mag(ldn_at<PN>(ci, K - 3)) / cd);
        double *mg = sm + L.mag + (long)i * (K + 1);
        #pragma unroll 1
        for (int k = 0; k <= K; ++k) mg[k] = PN::mag(ldn_at<PN>(ci, k));
      }
      // per-component Pade degrees go to shared memory for the evaluations
      int *degs = reinterpret_cast<int *>(sm + L.degs);
      if (ctid() < n) {
        degs[2 * ctid()] = pdeg_i;
        degs[2 * ctid() + 1] = qdeg_i;
      }
      const double r = block_min(rmin, red);
      const double perr = sqrt(block_sum<md::num<double, false> >(perr2, red));
      const bool rfail = !(r < 1e299);
      const double pole_step = rfail ? P.maxsize : P.pbeta * r;
      // Hesse_Pade (Curves/dobldobl_predictor_convolutions.adb:383-406):
      // eta = 2 sigma_min(J) / |(sigma_max(H_1), ..., sigma_max(H_n))|_2
      // (Distance), the curvature step (cbeta eta / |Pade errors|_2)^(1/K)
      // (Step_Distance, Curves/series_and_predictors.adb:813-825).
      // sigma_min(J) >= 1 / |J^{-1}|_F and sigma_max(H_i) <= |H_i|_F bound
      // eta, and so the curvature step, from below; when that bound is
      // already above min(pole step, maxsize) the curvature step cannot be
      // the smallest and the minimum below takes the same branch with it as
      // with +inf, so the singular values are computed only otherwise (a 1 %
      // margin covers the rounding of the bounds).
      double mf2 = 0.0;
      #pragma unroll 1
      for (int q = ctid(); q < n * n; q += blockDim.x) {
        const double a = PN::mag(ldn_at<PN>(sm + L.M, q));
        mf2 = fma(a, a, mf2);
      }
      mf2 = block_sum<md::num<double, false> >(mf2, red);
      double hf2 = 0.0;
      #pragma unroll 1
      for (int i = 0; i < n; ++i) hf2 += sv[i];
      const double cap = fmin(pole_step, P.maxsize);
      double curv_step = INFINITY;
      bool exact = hf2 > 0.0;  // all Hessians zero: eta and the curvature step are +inf
      if (exact && mf2 > 0.0 && mf2 < INFINITY && hf2 < INFINITY) {
        const double curv_lo = pow(P.cbeta * (2.0 / sqrt(mf2 * hf2)) / perr, 1.0 / K);
        exact = !(curv_lo > 1.01 * cap);
      }
      if (exact) {
        // the singular values, a job per warp: job i < n the largest of the
        // Hessian of equation i, job n the smallest of the Jacobian (its copy
        // from before the LU); every thread has read the norms in sv
        __syncthreads();
        #pragma unroll 1
        for (int job = ctid() >> 5; job <= n; job += kTrackThreads / 32) {
          if (job < n) {
            double2 *H = svd + (long)(ctid() >> 5) * n * n;
            warp_hessian_rows(S, s, job, n, t, xd, H);
            const double2 e = warp_singular_extremes(n, H, 2);
            if ((ctid() & 31) == 0) sv[job] = e.y;
          } else {
            const double2 e = warp_singular_extremes(n, svd + (long)(kSvdSlots - 1) * n * n, 1);
            if ((ctid() & 31) == 0) sv[n] = e.x;
          }
        }
        __syncthreads();
        double hsum = 0.0;
        #pragma unroll 1
        for (int i = 0; i < n; ++i) hsum = fma(sv[i], sv[i], hsum);
        const double eta = hsum > 0.0 ? 2.0 * sv[n] / sqrt(hsum) : INFINITY;
        curv_step = pow(P.cbeta * eta / perr, 1.0 / K);
        __syncthreads();
      }
      // the smallest of the pole step, the curvature step and maxsize
      // (Minimum, Curves/three_way_minima.adb:48-62, with its counts)
      double plain_step;
      if (pole_step < curv_step) {
        if (pole_step < P.maxsize) { plain_step = pole_step; ++nbpole; }
        else { plain_step = P.maxsize; ++nbmaxm; }
      } else {
        if (curv_step < P.maxsize) { plain_step = curv_step; ++nbhess; }
        else { plain_step = P.maxsize; ++nbmaxm; }
      }
      if (!(plain_step == plain_step)) plain_step = 0.0;  // a NaN curvature step
      double step = plain_step;
      bool learned = false;
      float *feat = reinterpret_cast<float *>(sm + L.feat);
      if (((P.step_mode & 1) && model != nullptr) || log != nullptr) {
        track_features(ctid(), n, K, t, plain_step, sm + L.mag, feat);
        __syncthreads();
      }
      if ((P.step_mode & 1) && model != nullptr) {
        const float lr = mlp_forward_cta(model, feat, reinterpret_cast<float *>(sm + L.hbuf));
        const double prop = plain_step * exp((double)lr) * P.learn_scale;
        if (prop > P.minsize && prop == prop) {
          step = fmin(prop, P.maxsize);
          learned = true;
        }
      }
      const double step0 = step;
      bool accepted = false;
      #pragma unroll 1
      for (int attempt = 0; attempt < 2 && !accepted; ++attempt) {
        if (attempt == 1) {
          // the learned proposal was rejected: redo the step with the plain one
          if (!learned) break;
          learned = false;
          step = plain_step;
        }
        // Bounded_Update (Curves/three_way_minima.adb:96-109): a step that
        // comes within minsize of t = 1 goes to t = 1
        if (t + step >= 1.0 - P.minsize) step = 1.0 - t;
        if (!(step > 0.0)) {  // a zero curvature step (singular Jacobian)
          if (learned) continue;
          failed = true;
          break;
        }
        // predictor feedback on the mixed residual
        double *xp = sm + L.xp;
        bool ok = false;
        #pragma unroll 1
        for (int h = 0; h < 64; ++h) {
          const double mixres = pade_mixres<PN>(S, s, n, K, P.dendeg, t, step, num, den, degs, xp, sm + L.xa,
                                                sm + L.V, sm + L.G, sm + L.hs, red);
          if (mixres < P.alpha) { ok = true; break; }
          step *= 0.5;
          ++nrej;
          if (step < P.minsize) break;
        }
        if (!ok) {
          if (learned) continue;  // the plain step gets its own feedback
          failed = true;
          break;
        }
        // corrector with step halving
        bool cok = false;
        #pragma unroll 1
        for (int h = 0; h < 64; ++h) {
          #pragma unroll 1
          for (int i = ctid(); i < n; i += blockDim.x)
            stn_at<CN>(xc, i, conv_num<PN, CN>::go(ldn_at<PN>(xp, i)));
          __syncthreads();
          if (corrector_newton<CN, PN>(S, s, n, t + step, xc, sm, L, piv, dinv, red, P.corsteps, P.tolres, 1,
                                       &dxn)) {
            cok = true;
            break;
          }
          ++nrej;
          if (learned) break;  // rejected proposal: retry with the plain step
          step *= 0.5;
          if (step < P.minsize) break;
          #pragma unroll 1
          for (int i = ctid(); i < n; i += blockDim.x) {
            const typename PN::T z = PN::from(step);
            const int pd = degs[2 * i], qd = degs[2 * i + 1];
            stn_at<PN>(xp, i, PN::div(horner<PN>(num + (long)i * (K + 1) * Wp, pd, z),
                                      horner<PN>(den + (long)i * (P.dendeg + 1) * Wp, qd, z)));
          }
          __syncthreads();
        }
        if (cok) { accepted = true; break; }
        if (learned) continue;  // rejected proposal: redo with the plain step
        failed = true;
        break;
      }
      if (failed || !accepted) { failed = true; break; }
      // training log: features, accepted step, plain step, proposal, t and
      // the largest probed step (plain step times 1.5, 2, 3, 4, 6, at most
      // maxsize and 1 - t) whose Pade prediction still passes the feedback
      if (log != nullptr) {
        double best = step;
        const double mults[5] = {1.5, 2.0, 3.0, 4.0, 6.0};
        #pragma unroll 1
        for (int q = 0; q < 5; ++q) {
          double sp = fmin(plain_step * mults[q], P.maxsize);
          if (t + sp > 1.0) sp = 1.0 - t;
          if (sp <= best) continue;
          const double mr = pade_mixres<PN>(S, s, n, K, P.dendeg, t, sp, num, den, degs, sm + L.xp, sm + L.xa,
                                            sm + L.V, sm + L.G, sm + L.hs, red);
          if (mr < P.alpha) best = sp;
        }
        if (ctid() == 0) {
          const int slot = atomicAdd(log_count, 1);
          if (slot < log_cap) {
            float *f = log + (long)slot * 32;
            #pragma unroll 1
            for (int q = 0; q < 24; ++q) f[q] = feat[q];
            f[24] = (float)step;
            f[25] = (float)plain_step;
            f[26] = (float)step0;
            f[27] = (float)t;
            f[28] = (float)best;
            #pragma unroll 1
            for (int q = 29; q < 32; ++q) f[q] = 0.0f;
          }
        }
      }
      t += step;
      ++nsteps;
      if (fabs(1.0 - t) < P.epsilon) { status = 0; break; }
    }
    // ---------------- refinement and classification
    double *xr = sm + L.xc;  // reuse the corrector slots at the refinement width
    // xc holds CN numbers: widen in place from the top (RN width >= CN width)
    if (RN::width != CN::width) {  // n <= blockDim.x: one number per thread
      typename CN::T v = CN::zero();
      if (ctid() < n) v = ldn_at<CN>(xc, ctid());
      __syncthreads();
      if (ctid() < n) stn_at<RN>(xr, ctid(), conv_num<CN, RN>::go(v));
      __syncthreads();
    }
    double res;
    if (!failed && status == 0) {
      point_newton<RN, RN>(S, s, n, 1.0, xr, sm + L.hc, sm + L.Jc, sm + L.Vc, sm + L.Gc, piv, dinv, red, P.refine_steps,
                       0.0, 0, &dxn);
      res = point_residual<RN>(S, s, n, 1.0, xr, sm + L.hc, sm + L.Vc, sm + L.Gc, red);
      status = (res <= P.restol) ? 0 : 3;
    } else {
      res = point_residual<RN>(S, s, n, t, xr, sm + L.hc, sm + L.Vc, sm + L.Gc, red);
      status = failed ? 1 : 2;
    }
    // end points as complex quad-doubles (octo-doubles for an octo-double
    // refinement), lower limbs zero below the refinement precision
    const int XL = RN::tr::limbs > 4 ? 8 : 4;
    #pragma unroll 1
    for (int q = ctid(); q < n_max * 2 * XL; q += blockDim.x) {
      const int i = q / (2 * XL), c = q % (2 * XL);
      double v = 0.0;
      if (i < n) {
        const int lim = RN::tr::limbs;
        const int part = c / XL, limb = c % XL;
        if (limb < lim) v = xr[(long)i * RN::width + part * lim + limb];
      }
      xend[((long)path * n_max) * 2 * XL + q] = v;
    }
    if (ctid() == 0) {
      int *io = info + (long)kTrackInfo * path;
      io[0] = status;
      io[1] = nsteps;
      io[2] = nrej;
      io[3] = nbpole;
      io[4] = nbhess;
      io[5] = nbmaxm;
      dinfo[2 * path] = t;
      dinfo[2 * path + 1] = res;
    }
    __syncthreads();
  }
}


}  // namespace phc

namespace phc {

long track_smem_bytes(int maxdim, int K, int M, int nmono_max, int maxvar, int pmode, int rmode, int gst);

template <class PN, class CN, class RN>
static int track_launch(const TrackDev &S, const TrackParDev &P, int nmono_max, int npaths, const int *path_sys,
                        const double *x0, const void *model, double *xend, int *info, double *dinfo, float *log,
                        int log_cap, int *log_count, int *queue, int one_per_launch, cudaStream_t st) {
  const long smem = track_smem_bytes(S.maxdim, P.deg, P.dendeg, nmono_max, S.maxvar, PN::tr::limbs, RN::tr::limbs, S.gstaged);
  if (smem > 227 * 1024) {
    set_error("track: %ld bytes of shared memory needed (dim %d, degree %d, %d monomials)", smem, S.maxdim, P.deg,
              nmono_max);
    return PHC_ERR_LIMIT;
  }
  auto kern = k_track<PN, CN, RN, false>;
  PHC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const float *mdl = reinterpret_cast<const float *>(model);
  if (one_per_launch) {
    // the plain arrangement: one launch (one CTA) per path, back to back
    #pragma unroll 1
    for (int p = 0; p < npaths; ++p) {
      kern<<<1, kTrackThreads, smem, st>>>(S, P, 1, p, path_sys, x0, nullptr, mdl, xend, info, dinfo, log, log_cap,
                                           log_count);
      PHC_CHECK_LAUNCH();
    }
    return PHC_OK;
  }
  int dev = 0, nsm = 148, per = 1;
  PHC_CUDA(cudaGetDevice(&dev));
  PHC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  PHC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kTrackThreads, smem));
  if (per < 1) per = 1;
  if constexpr (track_min_blocks<PN, RN, true>::split) {
    // one wave at the lower occupancy: take the variant with more registers
    // (the autotuner's choice when it made one: 1 narrow, 2 wide)
    auto wide = k_track<PN, CN, RN, true>;
    PHC_CUDA(cudaFuncSetAttribute(wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_w = 0;
    PHC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_w, wide, kTrackThreads, smem));
    const int variant = tune_get(kTuneTrackVariant);
    const bool take_wide = variant == 2 || (variant == 0 && (long)npaths <= (long)nsm * per_w);
    if (per_w >= 1 && take_wide) {
      kern = wide;
      per = per_w;
    }
  }
  // paths tracked at once per SM: all the resident CTAs the occupancy allows,
  // or fewer when the autotuner found that faster (fewer paths share an SM's
  // issue slots; the work queue hands the rest out as paths finish)
  const int cap = tune_get(kTuneTrackPerSM);
  if (cap > 0 && cap < per) per = cap;
  long grid = (long)nsm * per;
  if (grid > npaths) grid = npaths;
  if (grid < 1) return PHC_OK;
  // a batch that fits in one wave: CTA b tracks path b (the queue would
  // balance nothing, and the fixed mapping makes the launch time steadier);
  // otherwise the work queue hands out the paths as CTAs finish theirs
  int *q = grid >= npaths ? nullptr : queue;
  if (q) PHC_CUDA(cudaMemsetAsync(q, 0, sizeof(int), st));
  kern<<<(unsigned)grid, kTrackThreads, smem, st>>>(S, P, npaths, 0, path_sys, x0, q, mdl, xend, info, dinfo, log,
                                                     log_cap, log_count);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

}  // namespace phc
