// capi_wy.cu -- C ABI of the blocked QR and block-Toeplitz solve with a
// choice of how the WY trailing products run (include/phc_b200.h).
#include "common.cuh"
#include "../../include/phc_b200.h"

namespace phc {
long dense_work_doubles_wy(int prec, int cplx, int n, int szt, int wy);
int blocked_houseqr_wy(int prec, int cplx, int ninst, int n, int ncols, int szt, const double *A, double *Q,
                       double *R, double *work, int wy, cudaStream_t st);
int bals_solve_wy(int prec, int cplx, int ninst, int n, int degp1, int szt, int tailidx, const double *mat,
                  double *rhs, double *sol, double *Q, double *R, int *flags, double *work, int wy, cudaStream_t st);
}  // namespace phc

using namespace phc;

extern "C" {

long long phc_dense_workspace_bytes_wy(int prec, int cplx, int n, int szt, int wy) {
  if (!prec_ok(prec) || n < 1 || szt < 1) return -1;
  return (long long)dense_work_doubles_wy(prec, cplx, n, szt, wy) * (long long)sizeof(double);
}

int phc_blocked_houseqr_wy(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A, double *Q,
                           double *R, double *work, int wy, void *stream) {
  return blocked_houseqr_wy(prec, cplx, ninst, nrows, ncols, szt, A, Q, R, work, wy, (cudaStream_t)stream);
}

int phc_bals_solve_wy(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                      double *rhs, double *sol, double *Q, double *R, int *flags, double *work, int wy, void *stream) {
  return bals_solve_wy(prec, cplx, ninst, dim, degp1, szt, tailidx, mat, rhs, sol, Q, R, flags, work, wy,
                       (cudaStream_t)stream);
}

}  // extern "C"
