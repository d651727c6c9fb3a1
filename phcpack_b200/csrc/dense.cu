// dense.cu -- batched kernels of the Matrices and Newton layers: blocked
// Householder QR, tiled back substitution and the block-Toeplitz least
// squares solve, one CTA per instance.
#include "common.cuh"
#include "dense.cuh"

namespace phc {

static const int kDenseThreads = 256;

// per-instance workspace (doubles); the split tensor-core products need
// ozaki_work_doubles more
__host__ __device__ inline long dense_stride(int n, int szt, int W, bool oz) {
  return dense_work_numbers(n, szt) * W + (oz ? ozaki_work_doubles(n, ozaki_slices<md::qd>::s) : 0);
}

template <class N, bool OZ>
__global__ void __launch_bounds__(kDenseThreads)
    k_blocked_houseqr(int n, int ncols, int szt, const double *__restrict__ A, double *__restrict__ Q,
                      double *__restrict__ Rm, double *__restrict__ work, int stage) {
  extern __shared__ __align__(16) double sm[];
  const int W = N::width;
  const long inst = blockIdx.x;
  dense_smem S = carve<N>(sm, n, szt);
  const double *a = A + inst * n * ncols * W;
  double *q = Q + inst * n * n * W;
  double *r = Rm + inst * n * ncols * W;
  double *wk = work + inst * dense_stride(n, szt, W, OZ);
  // the WY panels and the column panel of R in shared memory when staged
  double *ywpt = stage ? sm + dense_smem_doubles(n, szt, W) : wk;
  double *panel = stage ? ywpt + 4L * n * szt * W : nullptr;
  for (long t = threadIdx.x; t < (long)n * ncols * W; t += blockDim.x) r[t] = a[t];
  __syncthreads();
  block_houseqr<N, OZ>(n, ncols, szt, q, r, ywpt, wk + dense_work_numbers(n, szt) * W, S, panel);
}

// Like Matrices/dbl2_tabs_kernels.cu:952 (GPU_dbl2_upper_tiled_solver): b is
// overwritten by the updated right hand sides and the diagonal tiles of U by
// their inverses.
template <class N>
__global__ void __launch_bounds__(kDenseThreads)
    k_upper_tiled_solver(int dim, int szt, double *__restrict__ U, double *__restrict__ b, double *__restrict__ x,
                         double *__restrict__ work) {
  const int W = N::width;
  const long inst = blockIdx.x;
  double *u = U + inst * dim * dim * W;
  double *bb = b + inst * dim * W;
  double *xx = x + inst * dim * W;
  double *tinv = work + inst * (long)dim * szt * W;
  block_invert_tiles<N>(dim, szt, u, dim, tinv);
  block_tiled_backsub<N>(dim, szt, u, dim, tinv, bb, xx);
  const int nbt = dim / szt;
  for (int t = threadIdx.x; t < nbt * szt * szt; t += blockDim.x) {
    const int tile = t / (szt * szt), i = (t / szt) % szt, j = t % szt;
    stn_at<N>(u, (long)(tile * szt + i) * dim + tile * szt + j, ldn_at<N>(tinv, t));
  }
}

// Block lower-triangular Toeplitz least squares, one instance per CTA:
// Newton/dbl2_bals_kernels.cu:554 (GPU_dbl2_bals_solve) with the head at
// :108 and the tail at dbl2_tail_kernels.cu:154; skip rules of
// Newton/dbl2_bals_host.cpp:15,228 (no QR when |b_0| < 1e-28 unless zeroQ,
// no update with a solution block below 1e-28, no back substitution for a
// right hand side below 1e-28; 1e-15 and 1e-56 in double and quad-double).
// flags per instance: zeroQ, noqr, upidx, bsidx, newtail; with tailidx < 0
// the tail starts at the instance's flags[4].
template <class N, bool OZ>
__global__ void __launch_bounds__(kDenseThreads)
    k_bals_solve(int n, int degp1, int szt, int tailidx, const double *__restrict__ mat, double *__restrict__ rhs,
                 double *__restrict__ sol, double *__restrict__ Q, double *__restrict__ Rm, int *__restrict__ flags,
                 double *__restrict__ work, int stage) {
  extern __shared__ __align__(16) double sm[];
  typedef typename N::T T;
  const int W = N::width;
  const long inst = blockIdx.x;
  dense_smem S = carve<N>(sm, n, szt);
  const long nn = (long)n * n;
  const double *A = mat + inst * degp1 * nn * W;
  double *b = rhs + inst * degp1 * n * W;
  double *x = sol + inst * degp1 * n * W;
  double *q = Q + inst * nn * W;
  double *r = Rm + inst * nn * W;
  int *fl = flags + inst * 5;
  double *wk = work + inst * dense_stride(n, szt, W, OZ);
  // staged: the WY panels, the column panel of R and then the inverted
  // diagonal tiles of R in shared memory
  double *ywpt = stage ? sm + dense_smem_doubles(n, szt, W) : wk;
  double *panel = stage ? ywpt + 4L * n * szt * W : nullptr;
  double *tinv = stage ? panel : wk + 4L * n * szt * W;
  int zeroQ = fl[0], noqr = fl[1];
  const int tail0 = max(1, tailidx >= 0 ? tailidx : fl[4]);
  bool tinv_ok = false;
  if (!(noqr && !zeroQ)) {
    const double nrm = block_maxnorm<N>(n, b, S.red);
    if (head_tiny<N>(nrm)) {
      noqr = zeroQ ? 0 : 1;
      if (noqr)
        for (int i = threadIdx.x; i < n; i += blockDim.x) stn_at<N>(x, i, N::zero());
    }
    if (!noqr) {
      for (long t = threadIdx.x; t < nn * W; t += blockDim.x) r[t] = A[t];
      __syncthreads();
      block_houseqr<N, OZ>(n, n, szt, q, r, ywpt, wk + dense_work_numbers(n, szt) * W, S, panel);
      zeroQ = 0;
      block_invert_tiles<N>(n, szt, r, n, tinv);
      tinv_ok = true;
      block_qhb<N>(n, q, b, S.w);
      block_tiled_backsub<N>(n, szt, r, n, tinv, S.w, S.x);
      for (int i = threadIdx.x; i < n; i += blockDim.x) stn_at<N>(x, i, ldn_at<N>(S.x, i));
      __syncthreads();
    }
  }
  int up = 0, bs = 0, newtail = tail0;
  if (degp1 > 1) {
    if (!tinv_ok) block_invert_tiles<N>(n, szt, r, n, tinv);
    bool first = true;
    newtail = degp1;
    for (int i = tail0; i < degp1; ++i) {
      const double *xp = x + (long)(i - 1) * n * W;
      double nrm = block_maxnorm<N>(n, xp, S.red);
      if (nrm < skip_tol<N>()) {
        ++up;
      } else {
        for (int l = threadIdx.x; l < n; l += blockDim.x) stn_at<N>(S.x, l, ldn_at<N>(xp, l));
        __syncthreads();
        block_tail_update<N>(n, degp1, i, A, b, S.x);
      }
      const double *bi = b + (long)i * n * W;
      nrm = block_maxnorm<N>(n, bi, S.red);
      double *xi = x + (long)i * n * W;
      if (nrm < skip_tol<N>()) {
        ++bs;
        for (int l = threadIdx.x; l < n; l += blockDim.x) stn_at<N>(xi, l, N::zero());
        __syncthreads();
      } else {
        if (first) {
          newtail = i;
          first = false;
        }
        block_qhb<N>(n, q, bi, S.w);
        block_tiled_backsub<N>(n, szt, r, n, tinv, S.w, S.x);
        for (int l = threadIdx.x; l < n; l += blockDim.x) stn_at<N>(xi, l, ldn_at<N>(S.x, l));
        __syncthreads();
      }
    }
  }
  if (threadIdx.x == 0) {
    fl[0] = zeroQ;
    fl[1] = noqr;
    if (degp1 > 1) {
      fl[2] = up;
      fl[3] = bs;
    }
    fl[4] = newtail;
  }
}

// Stage the WY panels and the column panel of R in shared memory?  Only on
// request (knob 3 of phc_tune_set = 2) and when they fit: the staged kernel
// runs one CTA per SM where the unstaged one runs two, and on the
// quad-double least squares of dimension 64 (tile 16) it measured 38 %
// slower (65.1 against 47.3 ms for 512 instances); the autotuner times both.
static bool dense_stage(int n, int szt, int W) {
  const long staged = dense_smem_doubles_staged(n, szt, W) * (long)sizeof(double);
  return tune_get(kTuneDenseStage) == 2 && staged <= 227L * 1024 - 1024;
}

template <class N>
static int qr_launch(int ninst, int n, int ncols, int szt, const double *A, double *Q, double *R, double *work,
                     cudaStream_t st, bool oz) {
  const int stage = dense_stage(n, szt, N::width) ? 1 : 0;
  const long smem = (stage ? dense_smem_doubles_staged(n, szt, N::width) : dense_smem_doubles(n, szt, N::width)) *
                    (long)sizeof(double);
  auto kern = oz ? k_blocked_houseqr<N, true> : k_blocked_houseqr<N, false>;
  PHC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<ninst, kDenseThreads, smem, st>>>(n, ncols, szt, A, Q, R, work, stage);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

// The residual of the linearised power-series system, one instance per CTA
// and one thread per entry (i, L), tailidx <= i < degp1:
//   res_i[L] = rhs_i[L] - sum_{j=0}^{i-tailidx} sum_k A_j[L][k] sol_{i-j}[k],
// in the order of Newton/dbl2_bals_host.cpp:548-600 (CPU_dbl2_linear_residue;
// complex numbers :602-680: re -= Are xre, re += Aim xim, im -= Are xim,
// im -= Aim xre, each product rounded before it is added).  resmax: prec
// doubles per instance, the magnitudes of the limbs of the first entry (in
// the order of i, then L) with the largest |leading limb| (|re| + |im| for
// complex numbers, limb by limb), zero when every entry is zero.
template <class N>
__device__ __forceinline__ void residue_dec(typename N::T &r, const typename N::T &a, const typename N::T &x) {
  if constexpr (N::is_complex) {
    typedef typename N::tr tr;
    r.re = tr::sub(r.re, tr::mul(a.re, x.re));
    r.re = tr::add(r.re, tr::mul(a.im, x.im));
    r.im = tr::sub(r.im, tr::mul(a.re, x.im));
    r.im = tr::sub(r.im, tr::mul(a.im, x.re));
  } else {
    r = N::sub(r, N::mul(a, x));
  }
}

template <class N>
__global__ void __launch_bounds__(kDenseThreads)
    k_linear_residue(int n, int degp1, int tailidx, const double *__restrict__ mat, const double *__restrict__ rhs,
                     const double *__restrict__ sol, double *__restrict__ res, double *__restrict__ resmax) {
  typedef typename N::T T;
  const int W = N::width;
  const int limbs = N::tr::limbs;
  const long inst = blockIdx.x;
  const double *A = mat + inst * (long)degp1 * n * n * W;
  const double *b = rhs + inst * (long)degp1 * n * W;
  const double *x = sol + inst * (long)degp1 * n * W;
  double *r = res + inst * (long)degp1 * n * W;
  const int cnt = (degp1 - tailidx) * n;
  double best = 0.0;
  int bidx = -1;
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int i = tailidx + e / n, L = e % n;
    T acc = ldn_at<N>(b, (long)i * n + L);
    for (int j = 0; j <= i - tailidx; ++j) {
      const double *Aj = A + (long)j * n * n * W;
      const double *xj = x + (long)(i - j) * n * W;
      for (int k = 0; k < n; ++k) residue_dec<N>(acc, ldn_at<N>(Aj, (long)L * n + k), ldn_at<N>(xj, k));
    }
    stn_at<N>(r, (long)i * n + L, acc);
    const double v = N::lead(acc);
    if (v > best) {  // a NaN is never taken, as in the reference
      best = v;
      bidx = e;
    }
  }
  __shared__ double sv[kDenseThreads];
  __shared__ int si[kDenseThreads];
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bidx;
  __syncthreads();
  for (int o = kDenseThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double v2 = sv[threadIdx.x + o];
      const int i2 = si[threadIdx.x + o];
      const double v1 = sv[threadIdx.x];
      const int i1 = si[threadIdx.x];
      if (i2 >= 0 && (i1 < 0 || v2 > v1 || (v2 == v1 && i2 < i1))) {
        sv[threadIdx.x] = v2;
        si[threadIdx.x] = i2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < limbs) {
    const int l = threadIdx.x, e = si[0];
    double m = 0.0;
    if (e >= 0) {
      const double *p = r + ((long)(tailidx + e / n) * n + e % n) * W;
      m = N::is_complex ? fabs(p[l]) + fabs(p[limbs + l]) : fabs(p[l]);
    }
    resmax[inst * limbs + l] = m;
  }
}

template <class N>
static int residue_launch(int ninst, int n, int degp1, int tailidx, const double *mat, const double *rhs,
                          const double *sol, double *res, double *resmax, cudaStream_t st) {
  k_linear_residue<N><<<ninst, kDenseThreads, 0, st>>>(n, degp1, tailidx, mat, rhs, sol, res, resmax);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

template <class N>
static int tabs_launch(int ninst, int dim, int szt, double *U, double *b, double *x, double *work, cudaStream_t st) {
  k_upper_tiled_solver<N><<<ninst, kDenseThreads, 0, st>>>(dim, szt, U, b, x, work);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

template <class N>
static int bals_launch(int ninst, int n, int degp1, int szt, int tailidx, const double *mat, double *rhs, double *sol,
                       double *Q, double *R, int *flags, double *work, cudaStream_t st, bool oz) {
  const int stage = dense_stage(n, szt, N::width) ? 1 : 0;
  const long smem = (stage ? dense_smem_doubles_staged(n, szt, N::width) : dense_smem_doubles(n, szt, N::width)) *
                    (long)sizeof(double);
  auto kern = oz ? k_bals_solve<N, true> : k_bals_solve<N, false>;
  PHC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<ninst, kDenseThreads, smem, st>>>(n, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work, stage);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

#define PHC_DISPATCH(prec, cplx, CALL)                 \
  do {                                                 \
    if (!(cplx)) {                                     \
      if ((prec) == 1) { typedef md::num<double, false> N; return CALL; } \
      if ((prec) == 2) { typedef md::num<md::dd, false> N; return CALL; } \
      { typedef md::num<md::qd, false> N; return CALL; } \
    } else {                                           \
      if ((prec) == 1) { typedef md::num<double, true> N; return CALL; } \
      if ((prec) == 2) { typedef md::num<md::dd, true> N; return CALL; } \
      { typedef md::num<md::qd, true> N; return CALL; } \
    }                                                  \
  } while (0)

long dense_work_doubles(int prec, int cplx, int n, int szt) {
  return dense_work_numbers(n, szt) * width_of(prec, cplx);
}

int blocked_houseqr(int prec, int cplx, int ninst, int n, int ncols, int szt, const double *A, double *Q, double *R,
                    double *work, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "blocked_houseqr: precision %d", prec);
  PHC_REQUIRE(n >= 1 && szt >= 1 && ncols % szt == 0 && ncols <= n && ncols >= 1, "blocked_houseqr: need ncols = szt*nbt <= n");
  if (ninst == 0) return PHC_OK;
  PHC_DISPATCH(prec, cplx, qr_launch<N>(ninst, n, ncols, szt, A, Q, R, work, st, false));
}

long dense_work_doubles_wy(int prec, int cplx, int n, int szt, int wy) {
  return dense_stride(n, szt, width_of(prec, cplx), wy != 0 && !cplx);
}

int blocked_houseqr_wy(int prec, int cplx, int ninst, int n, int ncols, int szt, const double *A, double *Q,
                       double *R, double *work, int wy, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "blocked_houseqr: precision %d", prec);
  PHC_REQUIRE(n >= 1 && n <= 64 && szt >= 1 && ncols % szt == 0 && ncols <= n && ncols >= 1,
              "blocked_houseqr: need ncols = szt*nbt <= n <= 64 with the tensor-core products");
  if (ninst == 0) return PHC_OK;
  PHC_DISPATCH(prec, cplx, qr_launch<N>(ninst, n, ncols, szt, A, Q, R, work, st, wy != 0 && !cplx));
}

int upper_tiled_solver(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x, double *work,
                       cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "upper_tiled_solver: precision %d", prec);
  PHC_REQUIRE(dim >= 1 && szt >= 1 && dim % szt == 0, "upper_tiled_solver: need dim = szt*nbt");
  if (ninst == 0) return PHC_OK;
  PHC_DISPATCH(prec, cplx, tabs_launch<N>(ninst, dim, szt, U, b, x, work, st));
}

int bals_solve(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat, double *rhs,
               double *sol, double *Q, double *R, int *flags, double *work, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "bals_solve: precision %d", prec);
  PHC_REQUIRE(n >= 1 && szt >= 1 && n % szt == 0 && degp1 >= 1, "bals_solve: need n = szt*nbt, degp1 >= 1");
  PHC_REQUIRE(tailidx != 0 && tailidx <= degp1, "bals_solve: tailidx %d not in [1, degp1=%d] (or < 0: per instance)", tailidx, degp1);
  if (ninst == 0) return PHC_OK;
  PHC_DISPATCH(prec, cplx, bals_launch<N>(ninst, n, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work, st, false));
}

int bals_solve_wy(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat,
                  double *rhs, double *sol, double *Q, double *R, int *flags, double *work, int wy, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "bals_solve: precision %d", prec);
  PHC_REQUIRE(n >= 1 && n <= 64 && szt >= 1 && n % szt == 0 && degp1 >= 1,
              "bals_solve: need n = szt*nbt <= 64 with the tensor-core products, degp1 >= 1");
  PHC_REQUIRE(tailidx != 0 && tailidx <= degp1, "bals_solve: tailidx %d not in [1, degp1=%d] (or < 0: per instance)", tailidx, degp1);
  if (ninst == 0) return PHC_OK;
  PHC_DISPATCH(prec, cplx,
               bals_launch<N>(ninst, n, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work, st, wy != 0 && !cplx));
}

int linear_residue(int prec, int cplx, int ninst, int n, int degp1, int tailidx, const double *mat, const double *rhs,
                   const double *sol, double *res, double *resmax, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec), "linear_residue: precision %d", prec);
  PHC_REQUIRE(n >= 1 && degp1 >= 1 && tailidx >= 0 && tailidx <= degp1,
              "linear_residue: need dim >= 1, degp1 >= 1, 0 <= tailidx <= degp1");
  if (ninst == 0) return PHC_OK;
  PHC_REQUIRE(mat && rhs && sol && res && resmax, "linear_residue: null pointer");
  PHC_DISPATCH(prec, cplx, residue_launch<N>(ninst, n, degp1, tailidx, mat, rhs, sol, res, resmax, st));
}

}  // namespace phc
