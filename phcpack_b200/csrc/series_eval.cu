// series_eval.cu -- batched evaluation and differentiation of polynomial
// systems at truncated power series (the Polynomials layer of PHCpack's GPU
// code, Polynomials/dbl2_polynomials_kernels.cu:1577, batched over systems).
//
// Grid: one CTA per (system, group of up to 8 polynomials); one warp per
// polynomial.  The CTA stages the system's input series in shared memory
// (coalesced 16-byte loads), each warp keeps its monomial's forward and
// backward products in its own shared-memory slots and accumulates the
// polynomial's value and gradient rows in the output buffer, which it owns.
#include "common.cuh"
#include "series_eval.cuh"

namespace phc {

static const int kMaxWarpsPerBlock = 8;
static const int kMaxSmem = 227 * 1024;

template <class N>
__global__ void __launch_bounds__(kMaxWarpsPerBlock * 32)
    k_system_evaldiff(int dim, int deg, int maxvar, int wpb, int stage, const int *__restrict__ mon_off,
                      const int *__restrict__ nvr, const int *__restrict__ idx, const int *__restrict__ exps,
                      const double *__restrict__ cst, const double *__restrict__ cff,
                      const double *__restrict__ input, double *__restrict__ output) {
  extern __shared__ __align__(16) double sm[];
  const int W = N::width;
  const int S = (deg + 1) * W;
  const int bps = (dim + wpb - 1) / wpb;
  const int s = blockIdx.x / bps;
  const int p0 = (blockIdx.x % bps) * wpb;
  const double *xin = input + (long)s * dim * S;
  const double *X = xin;
  double *scr = sm;
  if (stage) {
    double *Xs = sm;
    const int n = dim * S;
    if ((W & 1) == 0) {
      const double2 *src = reinterpret_cast<const double2 *>(xin);
      double2 *dst = reinterpret_cast<double2 *>(Xs);
      for (int i = threadIdx.x; i < n / 2; i += blockDim.x) dst[i] = src[i];
    } else {
      for (int i = threadIdx.x; i < n; i += blockDim.x) Xs[i] = xin[i];
    }
    X = Xs;
    scr = sm + ((n + 1) & ~1);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  const int p = p0 + warp;
  if (p >= dim) return;
  scr += (long)warp * warp_slots(maxvar) * S;
  const long sp = (long)s * dim + p;
  warp_poly_evaldiff<N>(dim, deg, maxvar, mon_off[sp], mon_off[sp + 1], nvr, idx, exps, cst + sp * S, cff, X, scr,
                        output + sp * (dim + 1) * S);
}

// Degrees 32..191: the same grid, warp_poly_evaldiff_big, one more scratch
// series per warp (the value); the inputs are staged in shared memory when
// they fit beside the scratch and read from global memory otherwise.
template <class N>
__global__ void __launch_bounds__(kMaxWarpsPerBlock * 32)
    k_system_evaldiff_big(int dim, int deg, int maxvar, int wpb, int stage, const int *__restrict__ mon_off,
                          const int *__restrict__ nvr, const int *__restrict__ idx, const int *__restrict__ exps,
                          const double *__restrict__ cst, const double *__restrict__ cff,
                          const double *__restrict__ input, double *__restrict__ output) {
  extern __shared__ __align__(16) double sm[];
  const int W = N::width;
  const int S = (deg + 1) * W;
  const int bps = (dim + wpb - 1) / wpb;
  const int s = blockIdx.x / bps;
  const int p0 = (blockIdx.x % bps) * wpb;
  const double *xin = input + (long)s * dim * S;
  const double *X = xin;
  double *scr = sm;
  if (stage) {
    double *Xs = sm;
    const int n = dim * S;
    for (int i = threadIdx.x; i < n; i += blockDim.x) Xs[i] = xin[i];
    X = Xs;
    scr = sm + ((n + 1) & ~1);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  const int p = p0 + warp;
  if (p >= dim) return;
  scr += (long)warp * (warp_slots(maxvar) + 1) * S;
  const long sp = (long)s * dim + p;
  warp_poly_evaldiff_big<N>(dim, deg, maxvar, mon_off[sp], mon_off[sp + 1], nvr, idx, exps, cst + sp * S, cff, X,
                            scr, output + sp * (dim + 1) * S);
}

template <class N>
static int launch_system(int nsys, int dim, int deg, int maxvar, const int *mon_off, const int *nvr, const int *idx,
                         const int *exps, const double *cst, const double *cff, const double *input, double *output,
                         cudaStream_t stream) {
  const int W = N::width;
  const int S = (deg + 1) * W;
  const bool big = deg > 31;  // series longer than a warp: k_system_evaldiff_big
  // one warp per polynomial, up to 8 per CTA; monomials with many variables
  // need many scratch series per warp, so fewer warps share a CTA when the
  // shared memory would not hold the scratch of 8; the inputs are staged in
  // shared memory when they fit beside the scratch
  const long per_warp = (long)(warp_slots(maxvar) + (big ? 1 : 0)) * S * sizeof(double);
  const long xs = (long)((dim * S + 1) & ~1) * sizeof(double);
  int wpb = dim < kMaxWarpsPerBlock ? dim : kMaxWarpsPerBlock;
  const int tuned = tune_get(kTuneEvalWarps);  // warps per CTA chosen by the autotuner
  if (tuned > 0) wpb = tuned < dim ? tuned : dim;
  while (wpb > 1 && (long)wpb * per_warp > kMaxSmem) --wpb;
  const long scr = (long)wpb * per_warp;
  int stage = (scr + xs) <= 200 * 1024;
  const long smem = scr + (stage ? xs : 0);
  if (smem > kMaxSmem) {
    set_error("system_evaldiff: %ld bytes of shared memory needed (maxvar %d, degree %d)", smem, maxvar, deg);
    return PHC_ERR_LIMIT;
  }
  auto kern = big ? k_system_evaldiff_big<N> : k_system_evaldiff<N>;
  PHC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int bps = (dim + wpb - 1) / wpb;
  const long grid = (long)nsys * bps;
  kern<<<(unsigned)grid, wpb * 32, smem, stream>>>(dim, deg, maxvar, wpb, stage, mon_off, nvr, idx, exps, cst, cff,
                                                   input, output);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

int system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off, const int *nvr,
                    const int *idx, const int *exps, const double *cst, const double *cff, const double *input,
                    double *output, cudaStream_t stream) {
  PHC_REQUIRE(prec_ok(prec), "system_evaldiff: precision %d not in {1,2,4}", prec);
  PHC_REQUIRE(nsys >= 0 && dim >= 1 && deg >= 0 && maxvar >= 1, "system_evaldiff: bad sizes");
  if (deg > 191) {
    set_error("system_evaldiff: degree %d > 191", deg);
    return PHC_ERR_LIMIT;
  }
  if (nsys == 0) return PHC_OK;
  PHC_REQUIRE(mon_off && nvr && idx && exps && cst && cff && input && output, "system_evaldiff: null pointer");
#define PHC_SYS(R, C) \
  return launch_system<md::num<R, C> >(nsys, dim, deg, maxvar, mon_off, nvr, idx, exps, cst, cff, input, output, stream)
  if (!cplx) {
    if (prec == 1) PHC_SYS(double, false);
    if (prec == 2) PHC_SYS(md::dd, false);
    PHC_SYS(md::qd, false);
  } else {
    if (prec == 1) PHC_SYS(double, true);
    if (prec == 2) PHC_SYS(md::dd, true);
    PHC_SYS(md::qd, true);
  }
#undef PHC_SYS
}

}  // namespace phc
