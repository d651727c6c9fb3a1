// diagnostics.cu -- end-game diagnostics at points of the homotopy, batched
// on the GPU: the series of the path at a point and its Fabry ratio (the
// nearest singular point in t), the Hessian distance to the nearest singular
// solution, and the curvature step of the Pade predictor.
#include "common.cuh"
#include "tracker.cuh"
#include "../../include/phc_b200.h"

namespace phc {

// End-game diagnostics at points of the homotopy: the series of the path
// at (x, t) and its Fabry ratio (Newton_Fabry,
// Curves/dobldobl_fabry_on_homotopy.adb:30-83; Fabry,
// Circuits/convergence_radius_estimates.adb:138-163,392-425), and the
// Hessian distance to the nearest singular solution with the curvature step
// of the Pade predictor (Distance and Hesse_Pade,
// Curves/dobldobl_predictor_convolutions.adb:368-406; Solution_Error_Estimate
// and Threshold_Index, Curves/homotopy_pade_approximants.adb:558-568,717-754;
// Step_Distance, Curves/series_and_predictors.adb:813-825).  One CTA per
// point.

// a + 1 == 1 in the working precision (Is_Zero,
// Circuits/convergence_radius_estimates.adb:8-20)
template <class N>
__device__ bool md_negligible(const typename N::real &a) {
  typedef typename N::tr tr;
  __align__(16) double u[8], v[8];
  md::str(u, tr::add(tr::one(), a));
  md::str(v, tr::one());
  for (int l = 0; l < tr::limbs; ++l)
    if (u[l] != v[l]) return false;
  return true;
}

template <class N>
__device__ bool cx_negligible(const typename N::T &z) {
  return md_negligible<N>(z.re) && md_negligible<N>(z.im);
}

// a < b for normalised multiple doubles: the limbs compared in order
template <class N>
__device__ bool md_less(const typename N::real &a, const typename N::real &b) {
  __align__(16) double u[8], v[8];
  md::str(u, a);
  md::str(v, b);
  for (int l = 0; l < N::tr::limbs; ++l)
    if (u[l] != v[l]) return u[l] < v[l];
  return false;
}

// Fabry's ratio of one component's series c[0..K]: z = c[K-1-off]/c[K-off];
// the error estimate compares it with the next ratio, times K - 1.
template <class N>
__device__ void fabry_one(const double *c, int K, int off, typename N::T &z, double &e, bool &fail) {
  typedef typename N::T T;
  const T cl = ldn_at<N>(c, K - off);
  fail = cx_negligible<N>(cl);
  if (fail) return;
  const double nm1 = (double)(K - 1);
  if (off == 0) {
    const T c1 = ldn_at<N>(c, K - 1);
    z = N::div(c1, cl);
    e = cx_negligible<N>(c1) ? 1.0 : N::mag(N::sub(z, N::div(ldn_at<N>(c, K - 2), c1))) * nm1;
  } else {
    const T cK = ldn_at<N>(c, K);
    z = N::div(ldn_at<N>(c, K - 1 - off), cl);
    e = cx_negligible<N>(cK) ? 1.0 : N::mag(N::sub(z, N::div(ldn_at<N>(c, K - 1), cK))) * nm1;
  }
}

// One CTA per point: Newton at (x, t), the Taylor series to degree K, Fabry
// over the components, the Pade error estimates, and the extreme singular
// values of the Jacobian and of the n Hessians (a job per warp, the warp
// routines of the tracker's curvature step).
template <class PN>
__global__ void __launch_bounds__(kTrackThreads, 1)
    k_series_diag(TrackDev S, DiagParDev D, int npaths, const int *__restrict__ path_sys,
                  const double *__restrict__ xpt, int xlimbs, const double *__restrict__ tpt,
                  double *__restrict__ series, double *__restrict__ dout, int *__restrict__ iout) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int sinfo;
  typedef typename PN::T T;
  typedef typename PN::real R;
  const int K = D.deg, Wp = PN::width, LP = PN::tr::limbs;
  const int n_max = S.maxdim;
  int nm_max = 0;
  for (int s = 0; s < S.nsys; ++s) nm_max = max(nm_max, S.mono_off[s + 1] - S.mono_off[s]);
  const TrackLayout L = track_layout(n_max, K, D.dendeg, nm_max, S.maxvar, Wp, Wp, S.gstaged);
  double2 *svd = reinterpret_cast<double2 *>(sm + L.svd);  // kSvdSlots matrices of n_max^2
  double *sv = sm + L.sv;                                   // n_max + 1 singular values
  double *red = sm + L.red;
  int *piv = reinterpret_cast<int *>(sm + L.piv);
  double *dinv = sm + L.dinv;
  track_pick_lead();
  const int path = blockIdx.x;
  if (path >= npaths) return;
  const int s = path_sys[path];
  const int n = S.dim[s];
  const double t = tpt[path];
  const int lane = ctid() & 31, warp = ctid() >> 5;
  // the point, its limbs truncated or padded to the working precision
  double *xc = sm + L.xc;
  for (int q = ctid(); q < n * Wp; q += blockDim.x) {
    const int i = q / Wp, l = q % Wp, part = l / LP, limb = l % LP;
    const double *src = xpt + ((long)path * n_max + i) * 2 * xlimbs + part * xlimbs;
    xc[q] = limb < xlimbs ? src[limb] : 0.0;
  }
  __syncthreads();
  double dxn = 0.0;
  bool conv = true;
  if (D.newton_steps > 0)
    conv = point_newton<PN, PN>(S, s, n, t, xc, sm + L.hc, sm + L.Jc, sm + L.Vc, sm + L.Gc, piv, dinv, red,
                                D.newton_steps, D.tolres, 1, &dxn);
  // the series, x_0 the point
  double *xs = sm + L.xs;
  for (int q = ctid(); q < n * (K + 1); q += blockDim.x) {
    const int i = q / (K + 1), k = q % (K + 1);
    stn_at<PN>(xs, q, k == 0 ? ldn_at<PN>(xc, i) : PN::zero());
  }
  double2 *xd = reinterpret_cast<double2 *>(sm + L.xd);
  for (int i = ctid(); i < n; i += blockDim.x) {
    const T v = ldn_at<PN>(xc, i);
    xd[i] = make_double2(md::lead(v.re), md::lead(v.im));
  }
  __syncthreads();
  hom_eval_cta<PN>(S, s, 0, t, xs, K + 1, sm + L.V, sm + L.G, sm + L.hs, sm + L.J0);
  double2 *Jd = svd + (long)(kSvdSlots - 1) * n * n;
  for (int q = ctid(); q < n * n; q += blockDim.x) {
    const T v = ldn_at<PN>(sm + L.J0, q);
    Jd[q] = make_double2(md::lead(v.re), md::lead(v.im));
  }
  __syncthreads();
  if (ctid() < 32) {
    const int info = warp_lufac<PN>(n, sm + L.J0, piv, dinv);
    if (info == 0) warp_luinverse<PN>(n, sm + L.J0, piv, dinv, sm + L.M);
    if (ctid() == 0) sinfo = info;
  }
  __syncthreads();
  const bool singular = sinfo != 0;
  if (!singular) {
    for (int k = 1; k <= K; ++k) {
      hom_coef_cta<PN>(S, s, k, t, xs, K + 1, sm + L.V, sm + L.r);
      for (int i = ctid(); i < n; i += blockDim.x) {
        T acc = PN::zero();
        for (int j = 0; j < n; ++j)
          acc = PN::add(acc, PN::mul(ldn_at<PN>(sm + L.M, (long)i * n + j), ldn_at<PN>(sm + L.r, j)));
        stn_at<PN>(xs, (long)i * (K + 1) + k, PN::neg(acc));
      }
      __syncthreads();
    }
  }
  // Fabry and the Pade error estimates, a component per lane of the lead warp
  double *zk = sm + L.hs;  // n numbers
  double *mg = sm + L.mag;  // e, fail flag and Pade error per component
  if (ctid() < 32) {
    if (lane < n && !singular) {
      const double *ci = xs + (long)lane * (K + 1) * Wp;
      T z = PN::zero();
      double e = 0.0;
      bool fail = true;
      fabry_one<PN>(ci, K, D.offset, z, e, fail);
      stn_at<PN>(zk, lane, z);
      mg[lane] = e;
      mg[n + lane] = fail ? 1.0 : 0.0;
      double *num = sm + L.num + (long)lane * (K + 1) * Wp;
      double *den = sm + L.den + (long)lane * (D.dendeg + 1) * Wp;
      const int pd = pade_one<PN>(D.numdeg, D.dendeg, K, ci, num, den);
      mg[2 * n + lane] = pade_error_one<PN>(ci, K, num, pd, den, pd == D.numdeg ? D.dendeg : 0);
    } else if (lane < n) {
      mg[lane] = 0.0;
      mg[n + lane] = 1.0;
      mg[2 * n + lane] = 1.0;
    }
  }
  __syncthreads();
  // singular values: job j < n the Hessian of equation j (largest), job n
  // the Jacobian (smallest)
  for (int j = warp; j <= n; j += kTrackThreads / 32) {
    double2 *A = j < n ? svd + (long)warp * n * n : Jd;
    if (j < n) warp_hessian_rows(S, s, j, n, t, xd, A);
    const double2 mm = warp_singular_extremes(n, A, j < n ? 2 : 1);
    if (lane == 0) sv[j] = j < n ? mm.y : mm.x;
  }
  __syncthreads();
  if (ctid() == 0) {
    // the component of smallest radius, the first on ties
    int best = -1;
    R rbest = PN::tr::zero();
    for (int i = 0; i < n; ++i) {
      if (mg[n + i] != 0.0) continue;
      const R ri = PN::norm2(ldn_at<PN>(zk, i));
      if (best < 0 || md_less<PN>(ri, rbest)) {
        best = i;
        rbest = ri;
      }
    }
    double *o = dout + (long)path * kDiagOut;
    if (best >= 0) {
      const T z = ldn_at<PN>(zk, best);
      o[0] = md::lead(z.re);
      o[1] = md::lead(z.im);
      o[2] = PN::mag(z);
      o[3] = mg[best];
    } else {
      o[0] = o[1] = o[3] = 0.0;
      o[2] = INFINITY;
    }
    double hn = 0.0, pn = 0.0;
    for (int i = 0; i < n; ++i) {
      hn += sv[i] * sv[i];
      pn += mg[2 * n + i] * mg[2 * n + i];
    }
    hn = sqrt(hn);
    pn = sqrt(pn);
    const double eta = hn > 0.0 ? 2.0 * sv[n] / hn : INFINITY;
    o[4] = sv[n];
    o[5] = hn;
    o[6] = eta;
    o[7] = pn;
    o[8] = pow(D.beta2 * eta / pn, 1.0 / K);
    o[9] = dxn;
    iout[2 * path] = best < 0 ? 1 : 0;
    iout[2 * path + 1] = singular ? 1 : (conv ? 0 : 2);
  }
  if (series != nullptr) {
    double *dst = series + (long)path * n_max * (K + 1) * Wp;
    for (int q = ctid(); q < n * (K + 1) * Wp; q += blockDim.x) dst[q] = xs[q];
  }
}

}  // namespace phc

namespace phc {

long diag_smem_bytes(int maxdim, int K, int M, int nmono_max, int maxvar, int pmode, int gst) {
  const int W = 2 * pmode;
  const TrackLayout L = track_layout(maxdim, K, M, nmono_max, maxvar, W, W, gst);
  return L.total * (long)sizeof(double);
}

// The checks of the precision, the dimension, the degrees and the limbs of
// the points.
int diag_check(const DiagParDev &D, int pmode, int maxdim, int xlimbs) {
  PHC_REQUIRE(pmode == 1 || pmode == 2 || pmode == 4, "series_diagnostics: precision %d not in {1,2,4}", pmode);
  PHC_REQUIRE(maxdim >= 1 && maxdim <= 32, "series_diagnostics: dimension %d not in [1,32]", maxdim);
  PHC_REQUIRE(xlimbs == 1 || xlimbs == 2 || xlimbs == 4 || xlimbs == 8,
              "series_diagnostics: xlimbs %d not in {1,2,4,8}", xlimbs);
  PHC_REQUIRE(D.deg >= 3 && D.deg <= kTrackKmax && D.numdeg >= 0 && D.dendeg >= 0 && D.dendeg <= 8 &&
                  D.numdeg + D.dendeg <= D.deg,
              "series_diagnostics: need 3 <= deg <= %d, numdeg + dendeg <= deg, dendeg <= 8", kTrackKmax);
  PHC_REQUIRE(D.offset >= 0 && D.offset <= D.deg - 2, "series_diagnostics: offset %d not in [0, deg-2]", D.offset);
  PHC_REQUIRE(D.newton_steps >= 0 && D.newton_steps <= 64, "series_diagnostics: newton_steps %d not in [0,64]",
              D.newton_steps);
  return PHC_OK;
}

template <class PN>
static int diag_launch(const TrackDev &S, const DiagParDev &D, int nmono_max, int npaths, const int *path_sys,
                       const double *xpt, int xlimbs, const double *tpt, double *series, double *dout, int *iout,
                       cudaStream_t st) {
  const long smem = diag_smem_bytes(S.maxdim, D.deg, D.dendeg, nmono_max, S.maxvar, PN::tr::limbs, S.gstaged);
  if (smem > 227 * 1024) {
    set_error("series_diagnostics: %ld bytes of shared memory needed (dim %d, degree %d, %d monomials)", smem,
              S.maxdim, D.deg, nmono_max);
    return PHC_ERR_LIMIT;
  }
  auto kern = k_series_diag<PN>;
  PHC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)npaths, kTrackThreads, smem, st>>>(S, D, npaths, path_sys, xpt, xlimbs, tpt, series, dout, iout);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

int series_diag(const TrackDev &S, const DiagParDev &D, int nmono_max, int npaths, const int *path_sys,
                const double *xpt, int xlimbs, const double *tpt, int pmode, double *series, double *dout, int *iout,
                cudaStream_t st) {
  const int bad = diag_check(D, pmode, S.maxdim, xlimbs);
  if (bad) return bad;
  if (npaths == 0) return PHC_OK;
  typedef md::num<double, true> Z1;
  typedef md::num<md::dd, true> Z2;
  typedef md::num<md::qd, true> Z4;
  if (pmode == 1)
    return diag_launch<Z1>(S, D, nmono_max, npaths, path_sys, xpt, xlimbs, tpt, series, dout, iout, st);
  if (pmode == 2)
    return diag_launch<Z2>(S, D, nmono_max, npaths, path_sys, xpt, xlimbs, tpt, series, dout, iout, st);
  return diag_launch<Z4>(S, D, nmono_max, npaths, path_sys, xpt, xlimbs, tpt, series, dout, iout, st);
}

}  // namespace phc
