// newton.cu -- one step of Newton's method on power series for a batch of
// systems (row / polynomial form): evaluate and differentiate at the current
// series, linearise (matrix series -> series of matrices, rhs = -f), solve
// the block-Toeplitz least-squares problem, update the series.
//
// Newton/dbl2_newton_method.cpp:429 (dbl2_row_newton_qrstep) and :134
// (dbl2_update_newton_qrstep), Newton/dbl2_systems_host.cpp:709
// (dbl2_map_evaldiff_output), Newton/dbl2_newton_testers.cpp:116
// (dbl2_update_series).  Four launches, all device-resident and capturable
// in one CUDA graph; the reference copies every intermediate to the host.
#include "common.cuh"
#include "dense.cuh"

namespace phc {

int system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off, const int *nvr,
                    const int *idx, const int *exps, const double *cst, const double *cff, const double *input,
                    double *output, cudaStream_t stream);
int bals_solve(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat, double *rhs,
               double *sol, double *Q, double *R, int *flags, double *work, cudaStream_t st);
long dense_work_doubles(int prec, int cplx, int n, int szt);

// series stored with capacity maxdeg+1 per variable; the working degree is
// deg <= maxdeg.  Packs the working prefix of every series (and of cst and
// cff) into contiguous degree-deg arrays.
__global__ void k_pack_series(long nseries, int W, int deg, int maxdeg, const double *__restrict__ src,
                              double *__restrict__ dst) {
  const long S = (long)(deg + 1) * W, Smax = (long)(maxdeg + 1) * W;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nseries * S; t += (long)gridDim.x * blockDim.x) {
    const long s = t / S, r = t % S;
    dst[t] = src[s * Smax + r];
  }
}

// output[s][i][j][k] (j = dim: value) -> jac[s][k][i][j], rhs[s][k][i] = -value
__global__ void k_linearize(int nsys, int dim, int deg, int W, const double *__restrict__ out,
                            double *__restrict__ jac, double *__restrict__ rhs) {
  const int n1 = deg + 1;
  const long per = (long)dim * (dim + 1) * n1;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)nsys * per; t += (long)gridDim.x * blockDim.x) {
    const long s = t / per;
    const long r = t % per;
    const int i = (int)(r / ((dim + 1) * n1));
    const int j = (int)((r / n1) % (dim + 1));
    const int k = (int)(r % n1);
    const double *src = out + t * W;
    if (j < dim) {
      double *dst = jac + ((((s * n1 + k) * dim + i) * dim) + j) * W;
      for (int c = 0; c < W; ++c) dst[c] = src[c];
    } else {
      double *dst = rhs + ((s * n1 + k) * dim + i) * W;
      for (int c = 0; c < W; ++c) dst[c] = -src[c];
    }
  }
}

// x[s][i][j] += dx[s][j][i] for j >= newtail - 1 (per system), in the
// precision of N
template <class N>
__global__ void k_update_series(int nsys, int dim, int deg, int maxdeg, const int *__restrict__ flags,
                                const double *__restrict__ sol, double *__restrict__ series) {
  const int n1 = deg + 1;
  const long per = (long)dim * n1;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)nsys * per; t += (long)gridDim.x * blockDim.x) {
    const long s = t / per;
    const int i = (int)((t % per) / n1), j = (int)(t % n1);
    if (j < flags[s * 5 + 4] - 1) continue;
    double *xp = series + ((s * dim + i) * (long)(maxdeg + 1) + j) * N::width;
    const double *dp = sol + ((s * n1 + j) * (long)dim + i) * N::width;
    typename N::T a, b;
    md::ldn(xp, a);
    md::ldn(dp, b);
    md::stn(xp, N::add(a, b));
  }
}

static unsigned grid_for(long n, int threads) {
  long g = (n + threads - 1) / threads;
  if (g > 148L * 32) g = 148L * 32;
  return (unsigned)(g < 1 ? 1 : g);
}

long newton_work_doubles(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, long nmon) {
  const long W = width_of(prec, cplx);
  const long n1 = deg + 1;
  const long packed = (long)nsys * dim * n1 * W * 2 + nmon * n1 * W;  // input, cst, cff
  const long out = (long)nsys * dim * (dim + 1) * n1 * W;
  const long jac = (long)nsys * n1 * dim * dim * W;
  const long vec = (long)nsys * n1 * dim * W * 2;  // rhs, sol
  const long bals = (long)nsys * dense_work_doubles(prec, cplx, dim, szt);
  (void)maxdeg;
  return packed + out + jac + vec + bals + 64;
}

int newton_step(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, int maxvar, const int *mon_off,
                long nmon, const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                double *series, double *Q, double *R, int *flags, double *work, cudaStream_t st) {
  PHC_REQUIRE(prec_ok(prec) && nsys >= 0 && dim >= 1 && deg >= 0 && deg <= maxdeg, "newton_step: bad sizes");
  PHC_REQUIRE(dim % szt == 0, "newton_step: dim %d not a multiple of the tile size %d", dim, szt);
  if (nsys == 0) return PHC_OK;
  const long W = width_of(prec, cplx);
  const long n1 = deg + 1;
  double *p = work;
  double *xin = p;  p += (long)nsys * dim * n1 * W;
  double *cs = p;   p += (long)nsys * dim * n1 * W;
  double *cf = p;   p += nmon * n1 * W;
  double *out = p;  p += (long)nsys * dim * (dim + 1) * n1 * W;
  double *jac = p;  p += (long)nsys * n1 * dim * dim * W;
  double *rhs = p;  p += (long)nsys * n1 * dim * W;
  double *sol = p;  p += (long)nsys * n1 * dim * W;
  double *bw = p;
  const int T = 256;
  k_pack_series<<<grid_for((long)nsys * dim * n1 * W, T), T, 0, st>>>((long)nsys * dim, (int)W, deg, maxdeg, series, xin);
  k_pack_series<<<grid_for((long)nsys * dim * n1 * W, T), T, 0, st>>>((long)nsys * dim, (int)W, deg, maxdeg, cst, cs);
  if (nmon > 0)
    k_pack_series<<<grid_for(nmon * n1 * W, T), T, 0, st>>>(nmon, (int)W, deg, maxdeg, cff, cf);
  PHC_CHECK_LAUNCH();
  int rc = system_evaldiff(prec, cplx, nsys, dim, deg, maxvar, mon_off, nvr, idx, exps, cs, cf, xin, out, st);
  if (rc) return rc;
  k_linearize<<<grid_for((long)nsys * dim * (dim + 1) * n1, T), T, 0, st>>>(nsys, dim, deg, (int)W, out, jac, rhs);
  PHC_CHECK_LAUNCH();
  PHC_CUDA(cudaMemsetAsync(sol, 0, (size_t)nsys * n1 * dim * W * sizeof(double), st));
  rc = bals_solve(prec, cplx, nsys, dim, (int)n1, szt, -1, jac, rhs, sol, Q, R, flags, bw, st);
  if (rc) return rc;
#define PHC_UPD(R_, C_)                                                                                         \
  k_update_series<md::num<R_, C_> ><<<grid_for((long)nsys * dim * n1, T), T, 0, st>>>(nsys, dim, deg, maxdeg, \
                                                                                      flags, sol, series)
  if (!cplx) {
    if (prec == 1) PHC_UPD(double, false);
    else if (prec == 2) PHC_UPD(md::dd, false);
    else PHC_UPD(md::qd, false);
  } else {
    if (prec == 1) PHC_UPD(double, true);
    else if (prec == 2) PHC_UPD(md::dd, true);
    else PHC_UPD(md::qd, true);
  }
#undef PHC_UPD
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

}  // namespace phc
