// capi.cu -- the C ABI of the library (declared in include/phc_b200.h).
//
// Device entry points take device pointers and a cudaStream_t (passed as
// void*) and return an int status: 0 ok, > 0 a count of failed items, < 0 an
// error whose text phc_last_error() returns.  *_host variants take host
// arrays, stage them on the device and copy the results back, like the
// reference's GPU_* host drivers do.
#include <cstring>
#include <string>
#include <mutex>
#include <atomic>
#include "common.cuh"
#include "../../include/phc_b200.h"

namespace phc {

static thread_local char g_err[512] = {0};

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char *get_error() { return g_err; }

int system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off, const int *nvr,
                    const int *idx, const int *exps, const double *cst, const double *cff, const double *input,
                    double *output, cudaStream_t stream);

long dense_work_doubles(int prec, int cplx, int n, int szt);
int blocked_houseqr(int prec, int cplx, int ninst, int n, int ncols, int szt, const double *A, double *Q, double *R,
                    double *work, cudaStream_t st);
int upper_tiled_solver(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x, double *work,
                       cudaStream_t st);
int bals_solve(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat, double *rhs,
               double *sol, double *Q, double *R, int *flags, double *work, cudaStream_t st);

int linear_residue(int prec, int cplx, int ninst, int n, int degp1, int tailidx, const double *mat, const double *rhs,
                   const double *sol, double *res, double *resmax, cudaStream_t st);

long newton_work_doubles(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, long nmon);
int newton_step(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, int maxvar, const int *mon_off,
                long nmon, const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                double *series, double *Q, double *R, int *flags, double *work, cudaStream_t st);

// device scratch owned for the duration of one host call
// Two streams that start after the work already on a caller's stream and
// that the caller's stream waits for at the end (join); without pipelining
// the caller's stream is used alone.
struct StreamPair {
  cudaStream_t q[2] = {nullptr, nullptr};
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  cudaStream_t base = nullptr;
  bool two = false;
  ~StreamPair() {
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    for (auto &s : q)
      if (s) cudaStreamDestroy(s);
  }
  int make(cudaStream_t st, bool pipelined) {
    base = st;
    two = pipelined;
    if (!two) return PHC_OK;
    for (auto &e : ev) PHC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PHC_CUDA(cudaEventRecord(ev[0], st));
    for (auto &s : q) {
      PHC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      PHC_CUDA(cudaStreamWaitEvent(s, ev[0], 0));
    }
    return PHC_OK;
  }
  cudaStream_t get(int c) const { return two ? q[c & 1] : base; }
  int join(cudaStream_t st) {
    if (!two) return PHC_OK;
    for (int i = 0; i < 2; ++i) {
      PHC_CUDA(cudaEventRecord(ev[1 + i], q[i]));
      PHC_CUDA(cudaStreamWaitEvent(st, ev[1 + i], 0));
    }
    return PHC_OK;
  }
};

struct dbuf {
  void *p = nullptr;
  ~dbuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      set_error("cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
      p = nullptr;
      return PHC_ERR_CUDA;
    }
    return PHC_OK;
  }
};

static std::atomic<int> g_tune[kTuneKnobs];

int tune_get(int knob) { return (knob >= 0 && knob < kTuneKnobs) ? g_tune[knob].load() : 0; }

}  // namespace phc

using namespace phc;

extern "C" {

const char *phc_last_error(void) { return get_error(); }

int phc_tune_set(int knob, int value) {
  PHC_REQUIRE(knob >= 0 && knob < kTuneKnobs, "tune_set: knob %d not in 0..%d", knob, kTuneKnobs - 1);
  PHC_REQUIRE(value >= 0, "tune_set: value %d < 0", value);
  if (knob == kTuneEvalWarps) PHC_REQUIRE(value <= 8, "tune_set: warps per CTA %d > 8", value);
  if (knob == kTuneTrackVariant) PHC_REQUIRE(value <= 2, "tune_set: tracker variant %d not in 0..2", value);
  if (knob == kTuneTrackPerSM) PHC_REQUIRE(value <= 32, "tune_set: paths per SM %d > 32", value);
  if (knob == kTuneDenseStage) PHC_REQUIRE(value <= 2, "tune_set: staging %d not in 0..2", value);
  g_tune[knob].store(value);
  return PHC_OK;
}

int phc_tune_get(int knob) {
  PHC_REQUIRE(knob >= 0 && knob < kTuneKnobs, "tune_get: knob %d not in 0..%d", knob, kTuneKnobs - 1);
  return g_tune[knob].load();
}

int phc_abi_version(void) { return PHC_ABI_VERSION; }

int phc_system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                        const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                        const double *input, double *output, void *stream) {
  return system_evaldiff(prec, cplx, nsys, dim, deg, maxvar, mon_off, nvr, idx, exps, cst, cff, input, output,
                         (cudaStream_t)stream);
}

int phc_system_evaldiff_host(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                             const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                             const double *input, double *output, void *stream) {
  PHC_REQUIRE(prec_ok(prec) && nsys >= 0 && dim >= 1 && deg >= 0 && maxvar >= 1, "system_evaldiff_host: bad sizes");
  if (nsys == 0) return PHC_OK;
  const long W = width_of(prec, cplx);
  const long S = (deg + 1) * W;
  const long npoly = (long)nsys * dim;
  const long nmon = mon_off[npoly];
  const size_t b_off = (npoly + 1) * sizeof(int), b_nvr = nmon * sizeof(int), b_idx = nmon * maxvar * sizeof(int);
  const size_t b_cst = npoly * S * sizeof(double), b_cff = nmon * S * sizeof(double);
  const size_t b_in = npoly * S * sizeof(double), b_out = npoly * (dim + 1) * S * sizeof(double);
  auto al = [](size_t n) { return (n + 255) & ~size_t(255); };
  const size_t total = al(b_off) + al(b_nvr) + 2 * al(b_idx) + al(b_cst) + al(b_cff) + al(b_in) + al(b_out);
  dbuf buf;
  int rc = buf.alloc(total);
  if (rc) return rc;
  char *p = (char *)buf.p;
  int *d_off = (int *)p; p += al(b_off);
  int *d_nvr = (int *)p; p += al(b_nvr);
  int *d_idx = (int *)p; p += al(b_idx);
  int *d_exp = (int *)p; p += al(b_idx);
  double *d_cst = (double *)p; p += al(b_cst);
  double *d_cff = (double *)p; p += al(b_cff);
  double *d_in = (double *)p; p += al(b_in);
  double *d_out = (double *)p;
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(d_off, mon_off, b_off, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_nvr, nvr, b_nvr, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_idx, idx, b_idx, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_exp, exps, b_idx, cudaMemcpyHostToDevice, st));
  // The systems in chunks on two streams: the copies of one chunk in and
  // of another out overlap the evaluation of a third.  A chunk's
  // coefficients are the contiguous rows of its monomials; the kernel
  // indexes monomials globally and everything else from the chunk's start.
  const int nchunk = nsys >= 64 ? 8 : 1;
  StreamPair sp;
  rc = sp.make(st, nchunk > 1);
  if (rc) return rc;
  for (int c = 0; c < nchunk; ++c) {
    cudaStream_t q = sp.get(c);
    const long s0 = (long)nsys * c / nchunk, s1 = (long)nsys * (c + 1) / nchunk;
    if (s1 == s0) continue;
    const long r0 = s0 * dim, r1 = s1 * dim;
    const long m0 = mon_off[r0], m1 = mon_off[r1];
    PHC_CUDA(cudaMemcpyAsync(d_cst + r0 * S, cst + r0 * S, (r1 - r0) * S * sizeof(double), cudaMemcpyHostToDevice, q));
    PHC_CUDA(cudaMemcpyAsync(d_cff + m0 * S, cff + m0 * S, (m1 - m0) * S * sizeof(double), cudaMemcpyHostToDevice, q));
    PHC_CUDA(cudaMemcpyAsync(d_in + r0 * S, input + r0 * S, (r1 - r0) * S * sizeof(double), cudaMemcpyHostToDevice, q));
    rc = system_evaldiff(prec, cplx, (int)(s1 - s0), dim, deg, maxvar, d_off + r0, d_nvr, d_idx, d_exp, d_cst + r0 * S,
                         d_cff, d_in + r0 * S, d_out + r0 * (dim + 1) * S, q);
    if (rc) return rc;
    PHC_CUDA(cudaMemcpyAsync(output + r0 * (dim + 1) * S, d_out + r0 * (dim + 1) * S,
                             (r1 - r0) * (dim + 1) * S * sizeof(double), cudaMemcpyDeviceToHost, q));
  }
  rc = sp.join(st);
  if (rc) return rc;
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

long long phc_dense_workspace_bytes(int prec, int cplx, int n, int szt) {
  if (!prec_ok(prec) || n < 1 || szt < 1) return -1;
  return (long long)dense_work_doubles(prec, cplx, n, szt) * (long long)sizeof(double);
}

int phc_blocked_houseqr(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A, double *Q,
                        double *R, double *work, void *stream) {
  return blocked_houseqr(prec, cplx, ninst, nrows, ncols, szt, A, Q, R, work, (cudaStream_t)stream);
}

int phc_upper_tiled_solver(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x,
                           double *work, void *stream) {
  return upper_tiled_solver(prec, cplx, ninst, dim, szt, U, b, x, work, (cudaStream_t)stream);
}

int phc_bals_solve(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                   double *rhs, double *sol, double *Q, double *R, int *flags, double *work, void *stream) {
  return bals_solve(prec, cplx, ninst, dim, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work,
                    (cudaStream_t)stream);
}

}  // extern "C"

// ---- host-buffer variants: stage, run, copy back, synchronise
namespace {
struct staged {
  dbuf buf;
  char *p = nullptr;
  size_t used = 0, cap = 0;
  int alloc(size_t n) {
    cap = n;
    int rc = buf.alloc(n);
    p = (char *)buf.p;
    return rc;
  }
  template <class X> X *take(size_t count) {
    size_t b = (count * sizeof(X) + 255) & ~size_t(255);
    X *r = (X *)(p + used);
    used += b;
    return r;
  }
};
inline size_t al(size_t n) { return (n + 255) & ~size_t(255); }
}  // namespace

extern "C" {

int phc_blocked_houseqr_host(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A,
                             double *Q, double *R, void *stream) {
  PHC_REQUIRE(prec_ok(prec) && ninst >= 0 && nrows >= 1 && szt >= 1, "blocked_houseqr_host: bad sizes");
  if (ninst == 0) return PHC_OK;
  const size_t W = width_of(prec, cplx);
  const size_t nA = (size_t)ninst * nrows * ncols * W, nQ = (size_t)ninst * nrows * nrows * W;
  const size_t nw = (size_t)ninst * dense_work_doubles(prec, cplx, nrows, szt);
  staged s;
  int rc = s.alloc(al(nA * 8) + al(nQ * 8) + al(nA * 8) + al(nw * 8));
  if (rc) return rc;
  double *dA = s.take<double>(nA), *dQ = s.take<double>(nQ), *dR = s.take<double>(nA), *dW = s.take<double>(nw);
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(dA, A, nA * 8, cudaMemcpyHostToDevice, st));
  rc = blocked_houseqr(prec, cplx, ninst, nrows, ncols, szt, dA, dQ, dR, dW, st);
  if (rc) return rc;
  PHC_CUDA(cudaMemcpyAsync(Q, dQ, nQ * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(R, dR, nA * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

int phc_upper_tiled_solver_host(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x,
                                void *stream) {
  PHC_REQUIRE(prec_ok(prec) && ninst >= 0 && dim >= 1 && szt >= 1, "upper_tiled_solver_host: bad sizes");
  if (ninst == 0) return PHC_OK;
  const size_t W = width_of(prec, cplx);
  const size_t nU = (size_t)ninst * dim * dim * W, nb = (size_t)ninst * dim * W;
  const size_t nw = (size_t)ninst * dim * szt * W;
  staged s;
  int rc = s.alloc(al(nU * 8) + 2 * al(nb * 8) + al(nw * 8));
  if (rc) return rc;
  double *dU = s.take<double>(nU), *db = s.take<double>(nb), *dx = s.take<double>(nb), *dW = s.take<double>(nw);
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(dU, U, nU * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(db, b, nb * 8, cudaMemcpyHostToDevice, st));
  rc = upper_tiled_solver(prec, cplx, ninst, dim, szt, dU, db, dx, dW, st);
  if (rc) return rc;
  PHC_CUDA(cudaMemcpyAsync(U, dU, nU * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(b, db, nb * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(x, dx, nb * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

int phc_bals_solve_host(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                        double *rhs, double *sol, double *Q, double *R, int *flags, void *stream) {
  PHC_REQUIRE(prec_ok(prec) && ninst >= 0 && dim >= 1 && szt >= 1 && degp1 >= 1, "bals_solve_host: bad sizes");
  if (ninst == 0) return PHC_OK;
  const size_t W = width_of(prec, cplx);
  const size_t nm = (size_t)ninst * degp1 * dim * dim * W, nb = (size_t)ninst * degp1 * dim * W;
  const size_t nq = (size_t)ninst * dim * dim * W, nf = (size_t)ninst * 5;
  const size_t nw = (size_t)ninst * dense_work_doubles(prec, cplx, dim, szt);
  staged s;
  int rc = s.alloc(al(nm * 8) + 2 * al(nb * 8) + 2 * al(nq * 8) + al(nf * 4) + al(nw * 8));
  if (rc) return rc;
  double *dm = s.take<double>(nm), *db = s.take<double>(nb), *dx = s.take<double>(nb);
  double *dQ = s.take<double>(nq), *dR = s.take<double>(nq);
  int *df = s.take<int>(nf);
  double *dW = s.take<double>(nw);
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(dm, mat, nm * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(db, rhs, nb * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(dx, sol, nb * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(dQ, Q, nq * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(dR, R, nq * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(df, flags, nf * 4, cudaMemcpyHostToDevice, st));
  rc = bals_solve(prec, cplx, ninst, dim, degp1, szt, tailidx, dm, db, dx, dQ, dR, df, dW, st);
  if (rc) return rc;
  PHC_CUDA(cudaMemcpyAsync(rhs, db, nb * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(sol, dx, nb * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(Q, dQ, nq * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(R, dR, nq * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(flags, df, nf * 4, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

int phc_linear_residue(int prec, int cplx, int ninst, int dim, int degp1, int tailidx, const double *mat,
                       const double *rhs, const double *sol, double *res, double *resmax, void *stream) {
  return linear_residue(prec, cplx, ninst, dim, degp1, tailidx, mat, rhs, sol, res, resmax, (cudaStream_t)stream);
}

int phc_linear_residue_host(int prec, int cplx, int ninst, int dim, int degp1, int tailidx, const double *mat,
                            const double *rhs, const double *sol, double *res, double *resmax, void *stream) {
  PHC_REQUIRE(prec_ok(prec) && ninst >= 0 && dim >= 1 && degp1 >= 1 && tailidx >= 0 && tailidx <= degp1,
              "linear_residue_host: bad sizes");
  if (ninst == 0) return PHC_OK;
  PHC_REQUIRE(mat && rhs && sol && res && resmax, "linear_residue_host: null pointer");
  const size_t W = width_of(prec, cplx);
  const size_t nm = (size_t)ninst * degp1 * dim * dim * W, nb = (size_t)ninst * degp1 * dim * W;
  const size_t nr = (size_t)ninst * prec;
  staged s;
  int rc = s.alloc(al(nm * 8) + 3 * al(nb * 8) + al(nr * 8));
  if (rc) return rc;
  double *dm = s.take<double>(nm), *db = s.take<double>(nb), *dx = s.take<double>(nb), *dr = s.take<double>(nb);
  double *dmax = s.take<double>(nr);
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(dm, mat, nm * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(db, rhs, nb * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(dx, sol, nb * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(dr, res, nb * 8, cudaMemcpyHostToDevice, st));  // rows below tailidx stay as they are
  rc = linear_residue(prec, cplx, ninst, dim, degp1, tailidx, dm, db, dx, dr, dmax, st);
  if (rc) return rc;
  PHC_CUDA(cudaMemcpyAsync(res, dr, nb * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(resmax, dmax, nr * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ Newton
extern "C" {

long long phc_newton_workspace_bytes(int prec, int cplx, int nsys, int dim, int deg, int szt, long long nmon) {
  if (!prec_ok(prec) || nsys < 0 || dim < 1 || deg < 0 || szt < 1) return -1;
  return (long long)newton_work_doubles(prec, cplx, nsys, dim, deg, deg, szt, (long)nmon) * 8;
}

int phc_newton_step(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, int maxvar,
                    const int *mon_off, long long nmon, const int *nvr, const int *idx, const int *exps,
                    const double *cst, const double *cff, double *series, double *Q, double *R, int *flags,
                    double *work, void *stream) {
  return newton_step(prec, cplx, nsys, dim, deg, maxdeg, szt, maxvar, mon_off, (long)nmon, nvr, idx, exps, cst, cff,
                     series, Q, R, flags, work, (cudaStream_t)stream);
}

// Newton's method on power series for a batch of systems, host arrays in and
// out, the loop of Newton/dbl2_newton_method.cpp:1455-1492: at most nsteps
// steps; schedule 0 keeps the working degree at deg, schedule 1 follows the
// reference's 0, 1, 2, 4, 7, 11, ... (wrkdeg += 1 + wrkdeg/2, capped at deg)
// and stops once every system's tail index reached deg.  series: nsys*dim
// series of degree deg (updated in place); flags: 5 ints per system out.
int phc_newton_host(int prec, int cplx, int nsys, int dim, int deg, int szt, int maxvar, const int *mon_off,
                    const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                    double *series, int nsteps, int schedule, int *flags, void *stream) {
  PHC_REQUIRE(prec_ok(prec) && nsys >= 0 && dim >= 1 && deg >= 0 && szt >= 1 && dim % szt == 0,
              "newton_host: bad sizes");
  if (nsys == 0) return PHC_OK;
  const size_t W = width_of(prec, cplx);
  const long npoly = (long)nsys * dim;
  const long nmon = mon_off[npoly];
  const size_t S = (size_t)(deg + 1) * W;
  const size_t nwork = (size_t)newton_work_doubles(prec, cplx, nsys, dim, deg, deg, szt, nmon);
  staged s;
  int rc = s.alloc(al((npoly + 1) * 4) + al(nmon * 4) + 2 * al(nmon * maxvar * 4) + 2 * al(npoly * S * 8) +
                   al(nmon * S * 8) + 2 * al((size_t)nsys * dim * dim * W * 8) + al(nsys * 20) + al(nwork * 8));
  if (rc) return rc;
  int *d_off = s.take<int>(npoly + 1), *d_nvr = s.take<int>(nmon);
  int *d_idx = s.take<int>(nmon * maxvar), *d_exp = s.take<int>(nmon * maxvar);
  double *d_cst = s.take<double>(npoly * S), *d_ser = s.take<double>(npoly * S), *d_cff = s.take<double>(nmon * S);
  double *d_Q = s.take<double>((size_t)nsys * dim * dim * W), *d_R = s.take<double>((size_t)nsys * dim * dim * W);
  int *d_fl = s.take<int>((size_t)nsys * 5);
  double *d_w = s.take<double>(nwork);
  cudaStream_t st = (cudaStream_t)stream;
  PHC_CUDA(cudaMemcpyAsync(d_off, mon_off, (npoly + 1) * 4, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_nvr, nvr, nmon * 4, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_idx, idx, nmon * maxvar * 4, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_exp, exps, nmon * maxvar * 4, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_cst, cst, npoly * S * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_cff, cff, nmon * S * 8, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_ser, series, npoly * S * 8, cudaMemcpyHostToDevice, st));
  for (long i = 0; i < nsys; ++i) {
    flags[5 * i + 0] = 1;  // zeroQ
    flags[5 * i + 1] = 0;  // noqr
    flags[5 * i + 2] = 0;
    flags[5 * i + 3] = 0;
    flags[5 * i + 4] = 1;  // tail index
  }
  PHC_CUDA(cudaMemcpyAsync(d_fl, flags, (size_t)nsys * 20, cudaMemcpyHostToDevice, st));
  int wrkdeg = schedule ? 0 : deg;
  for (int step = 0; step < nsteps; ++step) {
    rc = newton_step(prec, cplx, nsys, dim, wrkdeg, deg, szt, maxvar, d_off, nmon, d_nvr, d_idx, d_exp, d_cst, d_cff,
                     d_ser, d_Q, d_R, d_fl, d_w, st);
    if (rc) return rc;
    if (schedule) {
      PHC_CUDA(cudaMemcpyAsync(flags, d_fl, (size_t)nsys * 20, cudaMemcpyDeviceToHost, st));
      PHC_CUDA(cudaStreamSynchronize(st));
      bool done = true;
      for (long i = 0; i < nsys; ++i) done = done && flags[5 * i + 4] >= deg;
      if (done) break;
      wrkdeg = wrkdeg + 1 + wrkdeg / 2;
      if (wrkdeg > deg) wrkdeg = deg;
    }
  }
  PHC_CUDA(cudaMemcpyAsync(series, d_ser, npoly * S * 8, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaMemcpyAsync(flags, d_fl, (size_t)nsys * 20, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

}  // extern "C"
