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

// device scratch owned for the duration of one host call
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

}  // namespace phc

using namespace phc;

extern "C" {

const char *phc_last_error(void) { return get_error(); }

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
  PHC_CUDA(cudaMemcpyAsync(d_cst, cst, b_cst, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_cff, cff, b_cff, cudaMemcpyHostToDevice, st));
  PHC_CUDA(cudaMemcpyAsync(d_in, input, b_in, cudaMemcpyHostToDevice, st));
  rc = system_evaldiff(prec, cplx, nsys, dim, deg, maxvar, d_off, d_nvr, d_idx, d_exp, d_cst, d_cff, d_in, d_out, st);
  if (rc) return rc;
  PHC_CUDA(cudaMemcpyAsync(output, d_out, b_out, cudaMemcpyDeviceToHost, st));
  PHC_CUDA(cudaStreamSynchronize(st));
  return PHC_OK;
}

}  // extern "C"
