// ref_shim_matrices.cu -- PHCpack's device entry points of the blocked
// Householder QR and the tiled back substitution, with the reference's
// exact signatures, implemented on this library's C ABI:
//   GPU_dbl2_blocked_houseqr, GPU_cmplx2_blocked_houseqr
//       Matrices/dbl2_baqr_kernels.h:2479, :2540          (SHIM_BAQR2)
//   GPU_dbl4_blocked_houseqr, GPU_cmplx4_blocked_houseqr
//       Matrices/dbl4_baqr_kernels.h:3668, :3739          (SHIM_BAQR4)
//   GPU_dbl2_upper_inverse, GPU_cmplx2_upper_inverse,
//   GPU_dbl2_upper_tiled_solver, GPU_cmplx2_upper_tiled_solver
//       Matrices/dbl2_tabs_kernels.h:309, :330, :358, :392 (SHIM_TABS2)
//
// TEST INFRASTRUCTURE: the recipes of oracle/Makefile compile this file once
// per family (the macro in parentheses) against the reference's own header,
// so that any difference in the signatures fails to compile, and link it, in
// place of the reference's dbl2_baqr_kernels.cu, dbl4_baqr_kernels.cu or
// dbl2_tabs_kernels.cu, with the reference's unchanged test programs
// Matrices/test_dbl2_baqr.cpp, test_dbl4_baqr.cpp and test_dbl2_tabs.cpp
// and their host sources (read in place, output into oracle/_ref).  The
// reference's testers then check this library's factors and solutions with
// their own CPU code and probes.  The same functions are the binding a
// maintainer would add to PHCpack in place of its kernels.
//
// The reference's per-limb arrays (hi, lo; re, im), rows of row-major
// matrices, become the library's limb-interleaved row-major numbers; the
// per-kernel times of the reference's many launches are reported as one
// kernel time (in the first time argument, the others zero) and the
// reference's operation counts are not kept (zero).
#include <chrono>
#include <cstdio>
#include <vector>
#if defined(SHIM_BAQR2)
#include "dbl2_baqr_kernels.h"
#elif defined(SHIM_BAQR4)
#include "dbl4_baqr_kernels.h"
#elif defined(SHIM_TABS2)
#include "dbl2_tabs_kernels.h"
#endif
#include "phc_b200.h"

namespace {

// matrix of nrows x ncols numbers of W limbs from W row-pointer arrays
std::vector<double> pack(int nrows, int ncols, int W, double **const *parts) {
  std::vector<double> v((size_t)nrows * ncols * W);
  for (int i = 0; i < nrows; ++i)
    for (int j = 0; j < ncols; ++j)
      for (int l = 0; l < W; ++l) v[((size_t)i * ncols + j) * W + l] = parts[l][i][j];
  return v;
}

void unpack(const std::vector<double> &v, int nrows, int ncols, int W, double **const *parts) {
  for (int i = 0; i < nrows; ++i)
    for (int j = 0; j < ncols; ++j)
      for (int l = 0; l < W; ++l) parts[l][i][j] = v[((size_t)i * ncols + j) * W + l];
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void report(int rc, const char *name) {
  if (rc < 0) std::fprintf(stderr, "%s: %s\n", name, phc_last_error());
}

#if defined(SHIM_BAQR2) || defined(SHIM_BAQR4)
// A = Q R of one matrix; A, Q, R given as W limb arrays each.
void houseqr(int prec, int cplx, int nrows, int ncols, int szt, double **const *A, double **const *Q,
             double **const *R, double *lapms[10], double *walltimesec, long long *cnt[4], const char *name) {
  const int W = prec * (cplx ? 2 : 1);
  std::vector<double> a = pack(nrows, ncols, W, A);
  std::vector<double> q((size_t)nrows * nrows * W), r((size_t)nrows * ncols * W);
  const auto t0 = std::chrono::steady_clock::now();
  report(phc_blocked_houseqr_host(prec, cplx, 1, nrows, ncols, szt, a.data(), q.data(), r.data(), nullptr), name);
  const double secs = seconds_since(t0);
  unpack(q, nrows, nrows, W, Q);
  unpack(r, nrows, ncols, W, R);
  for (int k = 0; k < 10; ++k) *lapms[k] = k == 0 ? secs * 1e3 : 0.0;
  *walltimesec = secs;
  for (int k = 0; k < 4; ++k) *cnt[k] = 0;
}
#endif

#if defined(SHIM_TABS2)
std::vector<double> pack_vec(int n, int W, double *const *parts) {
  std::vector<double> v((size_t)n * W);
  for (int i = 0; i < n; ++i)
    for (int l = 0; l < W; ++l) v[(size_t)i * W + l] = parts[l][i];
  return v;
}

void unpack_vec(const std::vector<double> &v, int n, int W, double *const *parts) {
  for (int i = 0; i < n; ++i)
    for (int l = 0; l < W; ++l) parts[l][i] = v[(size_t)i * W + l];
}

// U x = b by the tiled solver: U's diagonal tiles become their inverses and
// b the updated right hand sides, as in the reference.
void tiled(int cplx, int dim, int szt, double **const *U, double *const *b, double *const *x, double *lapms[4],
           double *walltimesec, long long *cnt[3], const char *name) {
  const int W = cplx ? 4 : 2;
  std::vector<double> u = pack(dim, dim, W, U), bb = pack_vec(dim, W, b), xx((size_t)dim * W);
  const auto t0 = std::chrono::steady_clock::now();
  report(phc_upper_tiled_solver_host(2, cplx, 1, dim, szt, u.data(), bb.data(), xx.data(), nullptr), name);
  const double secs = seconds_since(t0);
  unpack(u, dim, dim, W, U);
  unpack_vec(bb, dim, W, b);
  unpack_vec(xx, dim, W, x);
  for (int k = 0; k < 4; ++k) *lapms[k] = k == 3 ? secs * 1e3 : 0.0;
  *walltimesec = secs;
  for (int k = 0; k < 3; ++k) *cnt[k] = 0;
}

// the inverse of an upper triangular U: the solver with one tile of size
// dim overwrites U with its inverse
void inverse(int cplx, int dim, double **const *U, double **const *invU, double *lapms, double *walltimesec,
             const char *name) {
  const int W = cplx ? 4 : 2;
  std::vector<double> u = pack(dim, dim, W, U), b((size_t)dim * W, 0.0), x((size_t)dim * W);
  const auto t0 = std::chrono::steady_clock::now();
  report(phc_upper_tiled_solver_host(2, cplx, 1, dim, dim, u.data(), b.data(), x.data(), nullptr), name);
  const double secs = seconds_since(t0);
  unpack(u, dim, dim, W, invU);
  *lapms = secs * 1e3;
  *walltimesec = secs;
}
#endif

}  // namespace

#if defined(SHIM_BAQR2)
void GPU_dbl2_blocked_houseqr(int nrows, int ncols, int szt, int nbt, double **Ahi, double **Alo, double **Qhi,
                              double **Qlo, double **Rhi, double **Rlo, double *houselapms, double *RTvlapms,
                              double *tileRlapms, double *vb2Wlapms, double *WYTlapms, double *QWYTlapms,
                              double *Qaddlapms, double *YWTlapms, double *YWTClapms, double *Raddlapms,
                              double *walltimesec, long long int *addcnt, long long int *mulcnt,
                              long long int *divcnt, long long int *sqrtcnt, bool verbose) {
  (void)nbt; (void)verbose;
  double **A[2] = {Ahi, Alo}, **Q[2] = {Qhi, Qlo}, **R[2] = {Rhi, Rlo};
  double *t[10] = {houselapms, RTvlapms, tileRlapms, vb2Wlapms, WYTlapms, QWYTlapms, Qaddlapms, YWTlapms,
                   YWTClapms, Raddlapms};
  long long *c[4] = {addcnt, mulcnt, divcnt, sqrtcnt};
  houseqr(2, 0, nrows, ncols, szt, A, Q, R, t, walltimesec, c, "GPU_dbl2_blocked_houseqr");
}

void GPU_cmplx2_blocked_houseqr(int nrows, int ncols, int szt, int nbt, double **Arehi, double **Arelo,
                                double **Aimhi, double **Aimlo, double **Qrehi, double **Qrelo, double **Qimhi,
                                double **Qimlo, double **Rrehi, double **Rrelo, double **Rimhi, double **Rimlo,
                                double *houselapms, double *RHvlapms, double *tileRlapms, double *vb2Wlapms,
                                double *WYHlapms, double *QWYHlapms, double *Qaddlapms, double *YWHlapms,
                                double *YWHClapms, double *Raddlapms, double *walltimesec, long long int *addcnt,
                                long long int *mulcnt, long long int *divcnt, long long int *sqrtcnt, bool verbose) {
  (void)nbt; (void)verbose;
  double **A[4] = {Arehi, Arelo, Aimhi, Aimlo}, **Q[4] = {Qrehi, Qrelo, Qimhi, Qimlo};
  double **R[4] = {Rrehi, Rrelo, Rimhi, Rimlo};
  double *t[10] = {houselapms, RHvlapms, tileRlapms, vb2Wlapms, WYHlapms, QWYHlapms, Qaddlapms, YWHlapms,
                   YWHClapms, Raddlapms};
  long long *c[4] = {addcnt, mulcnt, divcnt, sqrtcnt};
  houseqr(2, 1, nrows, ncols, szt, A, Q, R, t, walltimesec, c, "GPU_cmplx2_blocked_houseqr");
}
#endif

#if defined(SHIM_BAQR4)
void GPU_dbl4_blocked_houseqr(int nrows, int ncols, int szt, int nbt, double **Ahihi, double **Alohi,
                              double **Ahilo, double **Alolo, double **Qhihi, double **Qlohi, double **Qhilo,
                              double **Qlolo, double **Rhihi, double **Rlohi, double **Rhilo, double **Rlolo,
                              double *houselapms, double *RTvlapms, double *tileRlapms, double *vb2Wlapms,
                              double *WYTlapms, double *QWYTlapms, double *Qaddlapms, double *YWTlapms,
                              double *YWTClapms, double *Raddlapms, double *walltimesec, long long int *addcnt,
                              long long int *mulcnt, long long int *divcnt, long long int *sqrtcnt, bool verbose) {
  (void)nbt; (void)verbose;
  double **A[4] = {Ahihi, Alohi, Ahilo, Alolo}, **Q[4] = {Qhihi, Qlohi, Qhilo, Qlolo};
  double **R[4] = {Rhihi, Rlohi, Rhilo, Rlolo};
  double *t[10] = {houselapms, RTvlapms, tileRlapms, vb2Wlapms, WYTlapms, QWYTlapms, Qaddlapms, YWTlapms,
                   YWTClapms, Raddlapms};
  long long *c[4] = {addcnt, mulcnt, divcnt, sqrtcnt};
  houseqr(4, 0, nrows, ncols, szt, A, Q, R, t, walltimesec, c, "GPU_dbl4_blocked_houseqr");
}

void GPU_cmplx4_blocked_houseqr(int nrows, int ncols, int szt, int nbt, double **Arehihi, double **Arelohi,
                                double **Arehilo, double **Arelolo, double **Aimhihi, double **Aimlohi,
                                double **Aimhilo, double **Aimlolo, double **Qrehihi, double **Qrelohi,
                                double **Qrehilo, double **Qrelolo, double **Qimhihi, double **Qimlohi,
                                double **Qimhilo, double **Qimlolo, double **Rrehihi, double **Rrelohi,
                                double **Rrehilo, double **Rrelolo, double **Rimhihi, double **Rimlohi,
                                double **Rimhilo, double **Rimlolo, double *houselapms, double *RHvlapms,
                                double *tileRlapms, double *vb2Wlapms, double *WYHlapms, double *QWYHlapms,
                                double *Qaddlapms, double *YWHlapms, double *YWHClapms, double *Raddlapms,
                                double *walltimesec, long long int *addcnt, long long int *mulcnt,
                                long long int *divcnt, long long int *sqrtcnt, bool verbose) {
  (void)nbt; (void)verbose;
  double **A[8] = {Arehihi, Arelohi, Arehilo, Arelolo, Aimhihi, Aimlohi, Aimhilo, Aimlolo};
  double **Q[8] = {Qrehihi, Qrelohi, Qrehilo, Qrelolo, Qimhihi, Qimlohi, Qimhilo, Qimlolo};
  double **R[8] = {Rrehihi, Rrelohi, Rrehilo, Rrelolo, Rimhihi, Rimlohi, Rimhilo, Rimlolo};
  double *t[10] = {houselapms, RHvlapms, tileRlapms, vb2Wlapms, WYHlapms, QWYHlapms, Qaddlapms, YWHlapms,
                   YWHClapms, Raddlapms};
  long long *c[4] = {addcnt, mulcnt, divcnt, sqrtcnt};
  houseqr(4, 1, nrows, ncols, szt, A, Q, R, t, walltimesec, c, "GPU_cmplx4_blocked_houseqr");
}
#endif

#if defined(SHIM_TABS2)
void GPU_dbl2_upper_inverse(int dim, double **Uhi, double **Ulo, double **invUhi, double **invUlo, double *lapms,
                            double *walltimesec) {
  double **U[2] = {Uhi, Ulo}, **V[2] = {invUhi, invUlo};
  inverse(0, dim, U, V, lapms, walltimesec, "GPU_dbl2_upper_inverse");
}

void GPU_cmplx2_upper_inverse(int dim, double **Urehi, double **Urelo, double **Uimhi, double **Uimlo,
                              double **invUrehi, double **invUrelo, double **invUimhi, double **invUimlo,
                              double *lapms, double *walltimesec) {
  double **U[4] = {Urehi, Urelo, Uimhi, Uimlo}, **V[4] = {invUrehi, invUrelo, invUimhi, invUimlo};
  inverse(1, dim, U, V, lapms, walltimesec, "GPU_cmplx2_upper_inverse");
}

void GPU_dbl2_upper_tiled_solver(int dim, int szt, int nbt, double **Uhi, double **Ulo, double *bhi, double *blo,
                                 double *xhi, double *xlo, double *invlapms, double *mullapms, double *sublapms,
                                 double *totlapms, double *walltimesec, long long int *addcnt,
                                 long long int *mulcnt, long long int *divcnt) {
  (void)nbt;
  double **U[2] = {Uhi, Ulo};
  double *b[2] = {bhi, blo}, *x[2] = {xhi, xlo};
  double *t[4] = {invlapms, mullapms, sublapms, totlapms};
  long long *c[3] = {addcnt, mulcnt, divcnt};
  tiled(0, dim, szt, U, b, x, t, walltimesec, c, "GPU_dbl2_upper_tiled_solver");
}

void GPU_cmplx2_upper_tiled_solver(int dim, int szt, int nbt, double **Urehi, double **Urelo, double **Uimhi,
                                   double **Uimlo, double *brehi, double *brelo, double *bimhi, double *bimlo,
                                   double *xrehi, double *xrelo, double *ximhi, double *ximlo, double *invlapms,
                                   double *mullapms, double *sublapms, double *totlapms, double *walltimesec,
                                   long long int *addcnt, long long int *mulcnt, long long int *divcnt) {
  (void)nbt;
  double **U[4] = {Urehi, Urelo, Uimhi, Uimlo};
  double *b[4] = {brehi, brelo, bimhi, bimlo}, *x[4] = {xrehi, xrelo, ximhi, ximlo};
  double *t[4] = {invlapms, mullapms, sublapms, totlapms};
  long long *c[3] = {addcnt, mulcnt, divcnt};
  tiled(1, dim, szt, U, b, x, t, walltimesec, c, "GPU_cmplx2_upper_tiled_solver");
}
#endif
