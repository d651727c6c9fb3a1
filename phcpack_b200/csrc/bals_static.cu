// bals_static.cu -- the block-Toeplitz least-squares solve without any
// allocation: its workspace is a fixed array in device memory that the
// library owns for the lifetime of the process.
//
// Who needs this: callers that cannot let a library call cudaMalloc or
// cudaFree, namely latency-critical callers that cannot afford the
// device-wide synchronisation cudaFree implies, frameworks that hand all
// device memory to their own allocator and account for every byte, and code
// that must not allocate at all once it has been set up.  They
// pass inputs and outputs (device memory they own) and get the workspace
// from here.
//
// Limits and rules:
//  * the workspace holds kBalsStaticDoubles doubles (8 MiB); a call whose
//    ninst * phc_dense_workspace_bytes(prec, cplx, dim, szt) exceeds it is
//    rejected with PHC_ERR_LIMIT and an explanation;
//  * every GPU that loads the library reserves these 8 MiB until the process
//    exits;
//  * all calls share the one array, so calls that overlap on the GPU (other
//    streams, other host threads) race: serialise them;
//  * the array keeps the previous call's contents; the solver writes every
//    workspace entry before reading it (reflector panels, products and the
//    inverted tiles of R), so nothing needs clearing between calls;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress, with that device current; make that first call
//    before any stream capture begins.
#include <mutex>
#include "common.cuh"
#include "../../include/phc_b200.h"

namespace phc {

long dense_work_doubles(int prec, int cplx, int n, int szt);
int bals_solve(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat, double *rhs,
               double *sol, double *Q, double *R, int *flags, double *work, cudaStream_t st);

static const long kBalsStaticDoubles = 1L << 20;  // 8 MiB
static __device__ __align__(256) double g_bals_scratch[kBalsStaticDoubles];

static const int kMaxDevices = 64;
static double *g_bals_scratch_ptr[kMaxDevices] = {nullptr};
static std::mutex g_bals_scratch_lock;

// Device address of this device's array (host code must not use the
// symbol itself: on the host it names a stand-in, not device memory).  The
// address is looked up once per device and kept for the life of the
// process, so the library must not be used across a reset of the device
// (cudaDeviceReset or a new primary context), which would leave it stale.
static int bals_scratch_address(double **out) {
  int dev = 0;
  PHC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("bals_solve_static: device %d beyond the %d supported", dev, kMaxDevices);
    return PHC_ERR_LIMIT;
  }
  std::lock_guard<std::mutex> g(g_bals_scratch_lock);
  if (g_bals_scratch_ptr[dev] == nullptr) {
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_bals_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("bals_solve_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return PHC_ERR_CUDA;
    }
    g_bals_scratch_ptr[dev] = p;
  }
  *out = g_bals_scratch_ptr[dev];
  return PHC_OK;
}

}  // namespace phc

using namespace phc;

extern "C" {

long long phc_bals_solve_static_capacity_bytes(void) { return (long long)kBalsStaticDoubles * (long long)sizeof(double); }

int phc_bals_solve_static(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                          double *rhs, double *sol, double *Q, double *R, int *flags, void *stream) {
  PHC_REQUIRE(prec_ok(prec), "bals_solve_static: precision %d not in {1,2,4}", prec);
  PHC_REQUIRE(ninst >= 0 && dim >= 1 && szt >= 1 && dim % szt == 0 && degp1 >= 1,
              "bals_solve_static: need ninst >= 0, dim = szt*nbt, degp1 >= 1");
  const long need = (long)ninst * dense_work_doubles(prec, cplx, dim, szt);
  if (need > kBalsStaticDoubles) {
    set_error("bals_solve_static: %d instances of dimension %d (tile %d) need %ld bytes of workspace, more than the "
              "%ld bytes of the static array; split the batch or use phc_bals_solve with your own workspace",
              ninst, dim, szt, need * (long)sizeof(double), kBalsStaticDoubles * (long)sizeof(double));
    return PHC_ERR_LIMIT;
  }
  double *work = nullptr;
  int rc = bals_scratch_address(&work);
  if (rc) return rc;
  if (ninst == 0) return PHC_OK;
  return bals_solve(prec, cplx, ninst, dim, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work,
                    (cudaStream_t)stream);
}

}  // extern "C"
