// ref_shim_newton.cu -- the device entry points of PHCpack's Newton layer,
// with the reference's exact signatures, implemented on this library's C ABI:
//   GPU_dbl2_bals_solve                      Newton/dbl2_bals_kernels.h:255
//   GPU_cmplx2_bals_solve                    Newton/dbl2_bals_kernels.h:313
//   GPU_dbl2_linear_residue                  Newton/dbl2_tail_kernels.h:164
//   GPU_cmplx2_linear_residue                Newton/dbl2_tail_kernels.h:199
//   GPU_dbl2_evaluate_monomials              Newton/dbl2_systems_kernels.h:409
//   GPU_cmplx2vectorized_evaluate_monomials  Newton/dbl2_systems_kernels.h:541
//   GPU_dbl2_evaluate_columns                Newton/dbl2_systems_kernels.h:625
//   GPU_cmplx2_evaluate_columns              Newton/dbl2_systems_kernels.h:668
// and, compiled with -DSHIM_NEWTON4, their quad double twins GPU_dbl4_* and
// GPU_cmplx4_* (Newton/dbl4_bals_kernels.h:353, :431; dbl4_tail_kernels.h
// :244, :295; dbl4_systems_kernels.h).
//
// TEST INFRASTRUCTURE: the recipe of oracle/Makefile (target `shim`) compiles
// this file against the reference's own headers and links it, together
// with ref_shim_polynomials.cu, in place of the reference's
// dbl2_bals_kernels.cu, dbl2_tail_kernels.cu, dbl2_systems_kernels.cu,
// dbl2_baqr_kernels.cu, dbl2_tabs_kernels.cu and dbl2_polynomials_kernels.cu
// (their dbl4 twins for the quad double build), with the reference's
// unchanged Newton test program Newton/test_dbl2_newton.cpp
// (test_dbl4_newton.cpp) and its host sources, read in place, output into
// oracle/_ref.  In its mode 2 the reference's tester runs every Newton step
// on the host and through these entry points and prints the sums of the
// differences of the evaluated systems, Jacobians, right hand sides, Q, R,
// updated right hand sides, solutions and series.
//
// Mapping onto the library:
//  * bals_solve -> phc_bals_solve_host with one instance; the reference's
//    zeroQ, noqr, upidx, bsidx, newtail are the library's five flags, with
//    the same skip rules (dbl2_bals_kernels.cu:596-810).
//  * linear_residue -> phc_linear_residue_host.
//  * evaluate_monomials: polynomial i of the system is monomial i; one
//    phc_system_evaldiff_host call evaluates a batch of two systems, the
//    monomials themselves (value and the derivatives scaled by the
//    exponents) and, to return the evaluated common factors in cff as the
//    reference does (dbl2_systems_kernels.cu:855-878), the monomials
//    cff[i] * prod x_j^(e_j - 1) over the exponents e_j > 1.  Like the
//    reference, only rows idx[i][*] and dim of output[i] are written.
//  * evaluate_columns: polynomial j sums the monomials of all columns with
//    nvr[c][j] > 0, the last polynomial carries the constant -1
//    (dbl2_systems_kernels.cu:1291); funval and the linearised Jacobian come
//    from that system, and the workspace output holds, as in the reference,
//    the evaluation of the last column that has a monomial in equation j.
// Timings are wall-clock seconds of the library call (copies included);
// the bals_solve time is reported as QR time and the operation counts of the
// residual are the multiplications and additions of its definition.
#include <chrono>
#include <cstdio>
#include <vector>
#if defined(SHIM_NEWTON4)
#include "dbl4_bals_kernels.h"
#include "dbl4_tail_kernels.h"
#include "dbl4_systems_kernels.h"
#else
#include "dbl2_bals_kernels.h"
#include "dbl2_tail_kernels.h"
#include "dbl2_systems_kernels.h"
#endif
#include "phc_b200.h"

namespace {

typedef std::chrono::steady_clock clk;

double secs_since(clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); }

// vector of n numbers from limb arrays: limb l of number k at [k*W + l]
void pack(std::vector<double> &dst, size_t at, int n, int W, double *const *parts) {
  for (int k = 0; k < n; ++k)
    for (int l = 0; l < W; ++l) dst[at + (size_t)k * W + l] = parts[l][k];
}

void unpack(const std::vector<double> &src, size_t at, int n, int W, double *const *parts) {
  for (int k = 0; k < n; ++k)
    for (int l = 0; l < W; ++l) parts[l][k] = src[at + (size_t)k * W + l];
}

// rows of an n x m matrix given as limb arrays of row pointers
void pack_rows(std::vector<double> &dst, size_t at, int n, int m, int W, double **const *rows) {
  for (int i = 0; i < n; ++i) {
    double *r[8];
    for (int l = 0; l < W; ++l) r[l] = rows[l][i];
    pack(dst, at + (size_t)i * m * W, m, W, r);
  }
}

void unpack_rows(const std::vector<double> &src, size_t at, int n, int m, int W, double **const *rows) {
  for (int i = 0; i < n; ++i) {
    double *r[8];
    for (int l = 0; l < W; ++l) r[l] = rows[l][i];
    unpack(src, at + (size_t)i * m * W, m, W, r);
  }
}

void pack_mats(std::vector<double> &dst, int degp1, int dim, int W, double ***const *mat) {
  const size_t nn = (size_t)dim * dim * W;
  for (int k = 0; k < degp1; ++k) {
    double **mk[8];
    for (int l = 0; l < W; ++l) mk[l] = mat[l][k];
    pack_rows(dst, k * nn, dim, dim, W, mk);
  }
}

void report(int rc, const char *name) {
  if (rc < 0) std::fprintf(stderr, "%s: %s\n", name, phc_last_error());
}

void bals(int prec, int cplx, int dim, int degp1, int szt, int tailidx, double ***const *mat, double **const *Q,
          double **const *R, double **const *rhs, double **const *sol, bool *zeroQ, bool *noqr, int *upidx,
          int *bsidx, int *newtail, double *totqrlapsedms, const char *name) {
  const int W = prec * (cplx ? 2 : 1);
  const size_t nn = (size_t)dim * dim * W, nv = (size_t)dim * W;
  std::vector<double> m(degp1 * nn), b(degp1 * nv), x(degp1 * nv), q(nn), r(nn);
  pack_mats(m, degp1, dim, W, mat);
  pack_rows(b, 0, degp1, dim, W, rhs);
  pack_rows(x, 0, degp1, dim, W, sol);
  pack_rows(q, 0, dim, dim, W, Q);
  pack_rows(r, 0, dim, dim, W, R);
  int flags[5] = {*zeroQ ? 1 : 0, *noqr ? 1 : 0, 0, 0, tailidx};
  const auto t0 = clk::now();
  const int rc = phc_bals_solve_host(prec, cplx, 1, dim, degp1, szt, tailidx, m.data(), b.data(), x.data(),
                                     q.data(), r.data(), flags, nullptr);
  *totqrlapsedms += secs_since(t0) * 1e3;
  report(rc, name);
  unpack_rows(b, 0, degp1, dim, W, rhs);
  unpack_rows(x, 0, degp1, dim, W, sol);
  unpack_rows(q, 0, dim, dim, W, Q);
  unpack_rows(r, 0, dim, dim, W, R);
  *zeroQ = flags[0] != 0;
  *noqr = flags[1] != 0;
  *upidx = flags[2];
  *bsidx = flags[3];
  *newtail = flags[4];
}

// resmax: prec pointers, the limbs of the largest residual entry
void residue(int prec, int cplx, int dim, int degp1, int tailidx, double ***const *mat, double **const *rhs,
             double **const *sol, double **const *resvec, double *const *resmax, double *lapms, long long *add,
             long long *mul, const char *name) {
  const int W = prec * (cplx ? 2 : 1);
  const size_t nn = (size_t)dim * dim * W, nv = (size_t)dim * W;
  std::vector<double> m(degp1 * nn), b(degp1 * nv), x(degp1 * nv), res(degp1 * nv), rmax(prec);
  pack_mats(m, degp1, dim, W, mat);
  pack_rows(b, 0, degp1, dim, W, rhs);
  pack_rows(x, 0, degp1, dim, W, sol);
  pack_rows(res, 0, degp1, dim, W, resvec);
  const auto t0 = clk::now();
  const int rc = phc_linear_residue_host(prec, cplx, 1, dim, degp1, tailidx, m.data(), b.data(), x.data(),
                                         res.data(), rmax.data(), nullptr);
  *lapms = secs_since(t0) * 1e3;
  report(rc, name);
  unpack_rows(res, 0, degp1, dim, W, resvec);
  for (int l = 0; l < prec; ++l) *resmax[l] = rmax[l];
  // res_i = rhs_i - sum_{j=0}^{i-tailidx} A_j sol_{i-j}: dim^2 products and
  // sums per matrix-vector product, one subtraction per entry
  long long prods = 0;
  for (int i = tailidx; i < degp1; ++i) prods += (long long)(i - tailidx + 1) * dim * dim;
  *mul += prods;
  *add += prods + (long long)(degp1 - tailidx) * dim;
}

// A batch of systems for phc_system_evaldiff_host, built one polynomial at
// a time (polynomials in system order, monomials in polynomial order).
struct Batch {
  int prec, W, dim, deg, maxvar = 1, nsys = 0;
  std::vector<int> mon_off{0}, nvr, idx, exps;
  std::vector<std::vector<int>> vars, pows;
  std::vector<double> cff, cst, input;
  Batch(int prec_, int W_, int dim_, int deg_) : prec(prec_), W(W_), dim(dim_), deg(deg_) {}
  size_t series() const { return (size_t)(deg + 1) * W; }
  void monomial(const int *v, const int *e, int k, double *const *c) {
    vars.emplace_back(v, v + k);
    pows.emplace_back(e, e + k);
    maxvar = k > maxvar ? k : maxvar;
    const size_t at = cff.size();
    cff.resize(at + series());
    pack(cff, at, deg + 1, W, c);
  }
  void end_polynomial() { mon_off.push_back((int)vars.size()); }
  // the system's input series (limb arrays of dim rows) and zero constants
  void end_system(double **const *input_rows) {
    const size_t at = input.size();
    input.resize(at + dim * series());
    pack_rows(input, at, dim, deg + 1, W, input_rows);
    cst.resize(input.size(), 0.0);
    ++nsys;
  }
  // run; returns the output, dim+1 series per polynomial
  std::vector<double> run(int cplx, double *ms, const char *name) {
    const size_t nm = vars.size() > 0 ? vars.size() : 1;
    nvr.assign(nm, 0);
    idx.assign(nm * maxvar, 0);
    exps.assign(nm * maxvar, 0);
    for (size_t m = 0; m < vars.size(); ++m) {
      nvr[m] = (int)vars[m].size();
      for (size_t j = 0; j < vars[m].size(); ++j) {
        idx[m * maxvar + j] = vars[m][j];
        exps[m * maxvar + j] = pows[m][j];
      }
    }
    if (cff.empty()) cff.assign(series(), 0.0);
    std::vector<double> out((size_t)nsys * dim * (dim + 1) * series(), 0.0);
    const auto t0 = clk::now();
    const int rc = phc_system_evaldiff_host(prec, cplx, nsys, dim, deg, maxvar, mon_off.data(), nvr.data(),
                                            idx.data(), exps.data(), cst.data(), cff.data(), input.data(),
                                            out.data(), nullptr);
    *ms += secs_since(t0) * 1e3;
    report(rc, name);
    return out;
  }
  // series r of polynomial p of system s in the output
  size_t at(int s, int p, int r) const { return (((size_t)s * dim + p) * (dim + 1) + r) * series(); }
};

void evaluate_monomials(int prec, int cplx, int dim, int deg, const int *nvr, int *const *idx, int *const *exp,
                        const int *nbrfac, int *const *expfac, double **const *cff, double **const *input,
                        double ***const *output, double *totcnvlapsedms, const char *name) {
  const int W = prec * (cplx ? 2 : 1), n1 = deg + 1;
  Batch B(prec, W, dim, deg);
  auto cff_of = [&](int i, double **c) {
    for (int l = 0; l < W; ++l) c[l] = cff[l][i];
  };
  // system 0: the monomials
  for (int i = 0; i < dim; ++i) {
    double *c[8];
    cff_of(i, c);
    B.monomial(idx[i], exp[i], nvr[i], c);
    B.end_polynomial();
  }
  B.end_system(input);
  // system 1: the common factors cff[i] * prod x^(e-1), e > 1
  for (int i = 0; i < dim; ++i) {
    if (nbrfac[i] > 0) {
      std::vector<int> v, e;
      for (int j = 0; j < nvr[i]; ++j)
        if (expfac[i][j] > 0) {
          v.push_back(idx[i][j]);
          e.push_back(expfac[i][j]);
        }
      if (!v.empty()) {
        double *c[8];
        cff_of(i, c);
        B.monomial(v.data(), e.data(), (int)v.size(), c);
      }
    }
    B.end_polynomial();
  }
  B.end_system(input);
  const std::vector<double> out = B.run(cplx, totcnvlapsedms, name);
  for (int i = 0; i < dim; ++i) {
    auto put_row = [&](int r) {
      double *o[8];
      for (int l = 0; l < W; ++l) o[l] = output[l][i][r];
      unpack(out, B.at(0, i, r), n1, W, o);
    };
    for (int j = 0; j < nvr[i]; ++j) put_row(idx[i][j]);
    put_row(dim);
    if (nbrfac[i] > 0 && B.mon_off[dim + i + 1] > B.mon_off[dim + i]) {
      double *c[8];
      cff_of(i, c);
      unpack(out, B.at(1, i, dim), n1, W, c);
    }
  }
}

void evaluate_columns(int prec, int cplx, int dim, int deg, int nbrcol, int *const *nvr, int **const *idx,
                      double ***const *cff, double **const *input, double ***const *output,
                      double **const *funval, double ***const *jacval, double *totcnvlapsedms, const char *name) {
  const int W = prec * (cplx ? 2 : 1), n1 = deg + 1;
  Batch B(prec, W, dim, deg);
  std::vector<int> ones(dim > 0 ? dim : 1, 1);
  std::vector<int> last(dim, -1);  // last column with a monomial in equation j
  for (int j = 0; j < dim; ++j) {
    for (int c = 0; c < nbrcol; ++c)
      if (nvr[c][j] > 0) {
        double *cf[8];
        for (int l = 0; l < W; ++l) cf[l] = cff[l][c][j];
        B.monomial(idx[c][j], ones.data(), nvr[c][j], cf);
        last[j] = c;
      }
    B.end_polynomial();
  }
  B.end_system(input);
  for (int j = 0; j < dim; ++j) {
    const int c = last[j];
    if (c >= 0) {
      double *cf[8];
      for (int l = 0; l < W; ++l) cf[l] = cff[l][c][j];
      B.monomial(idx[c][j], ones.data(), nvr[c][j], cf);
    }
    B.end_polynomial();
  }
  B.end_system(input);
  // the constant -1 of the last equation (system 0)
  B.cst[(size_t)(dim - 1) * B.series()] = -1.0;
  const std::vector<double> out = B.run(cplx, totcnvlapsedms, name);
  for (int j = 0; j < dim; ++j) {
    double *f[8];
    for (int l = 0; l < W; ++l) f[l] = funval[l][j];
    unpack(out, B.at(0, j, dim), n1, W, f);
    for (int v = 0; v < dim; ++v)
      for (int L = 0; L < n1; ++L)
        for (int l = 0; l < W; ++l) jacval[l][L][j][v] = out[B.at(0, j, v) + (size_t)L * W + l];
    const int c = last[j];
    if (c >= 0) {
      auto put_row = [&](int r) {
        double *o[8];
        for (int l = 0; l < W; ++l) o[l] = output[l][j][r];
        unpack(out, B.at(1, j, r), n1, W, o);
      };
      for (int k = 0; k < nvr[c][j]; ++k) put_row(idx[c][j][k]);
      put_row(dim);
    }
  }
}

}  // namespace

#if !defined(SHIM_NEWTON4)

void GPU_dbl2_bals_solve(int dim, int degp1, int szt, int nbt, int tailidx, double ***mathi, double ***matlo,
                         double **Qhi, double **Qlo, double **Rhi, double **Rlo, double **rhshi, double **rhslo,
                         double **solhi, double **sollo, bool *zeroQ, bool *noqr, int *upidx, int *bsidx,
                         int *newtail, double *totqrlapsedms, double *totqtblapsedms, double *totbslapsedms,
                         double *totupdlapsedms, int vrblvl) {
  (void)nbt; (void)totqtblapsedms; (void)totbslapsedms; (void)totupdlapsedms; (void)vrblvl;
  double ***mat[2] = {mathi, matlo};
  double **Q[2] = {Qhi, Qlo}, **R[2] = {Rhi, Rlo}, **rhs[2] = {rhshi, rhslo}, **sol[2] = {solhi, sollo};
  bals(2, 0, dim, degp1, szt, tailidx, mat, Q, R, rhs, sol, zeroQ, noqr, upidx, bsidx, newtail, totqrlapsedms,
       "GPU_dbl2_bals_solve");
}

void GPU_cmplx2_bals_solve(int dim, int degp1, int szt, int nbt, int tailidx, double ***matrehi, double ***matrelo,
                           double ***matimhi, double ***matimlo, double **Qrehi, double **Qrelo, double **Qimhi,
                           double **Qimlo, double **Rrehi, double **Rrelo, double **Rimhi, double **Rimlo,
                           double **rhsrehi, double **rhsrelo, double **rhsimhi, double **rhsimlo, double **solrehi,
                           double **solrelo, double **solimhi, double **solimlo, bool *zeroQ, bool *noqr, int *upidx,
                           int *bsidx, int *newtail, double *totqrlapsedms, double *totqtblapsedms,
                           double *totbslapsedms, double *totupdlapsedms, int vrblvl) {
  (void)nbt; (void)totqtblapsedms; (void)totbslapsedms; (void)totupdlapsedms; (void)vrblvl;
  double ***mat[4] = {matrehi, matrelo, matimhi, matimlo};
  double **Q[4] = {Qrehi, Qrelo, Qimhi, Qimlo}, **R[4] = {Rrehi, Rrelo, Rimhi, Rimlo};
  double **rhs[4] = {rhsrehi, rhsrelo, rhsimhi, rhsimlo}, **sol[4] = {solrehi, solrelo, solimhi, solimlo};
  bals(2, 1, dim, degp1, szt, tailidx, mat, Q, R, rhs, sol, zeroQ, noqr, upidx, bsidx, newtail, totqrlapsedms,
       "GPU_cmplx2_bals_solve");
}

void GPU_dbl2_linear_residue(int dim, int degp1, int szt, int nbt, int tailidx, double ***mathi, double ***matlo,
                             double **rhshi, double **rhslo, double **solhi, double **sollo, double **resvechi,
                             double **resveclo, double *resmaxhi, double *resmaxlo, double *lapms, long long *add,
                             long long *mul, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***mat[2] = {mathi, matlo};
  double **rhs[2] = {rhshi, rhslo}, **sol[2] = {solhi, sollo}, **res[2] = {resvechi, resveclo};
  double *resmax[2] = {resmaxhi, resmaxlo};
  residue(2, 0, dim, degp1, tailidx, mat, rhs, sol, res, resmax, lapms, add, mul, "GPU_dbl2_linear_residue");
}

void GPU_cmplx2_linear_residue(int dim, int degp1, int szt, int nbt, int tailidx, double ***matrehi,
                               double ***matrelo, double ***matimhi, double ***matimlo, double **rhsrehi,
                               double **rhsrelo, double **rhsimhi, double **rhsimlo, double **solrehi,
                               double **solrelo, double **solimhi, double **solimlo, double **resvecrehi,
                               double **resvecrelo, double **resvecimhi, double **resvecimlo, double *resmaxhi,
                               double *resmaxlo, double *lapms, long long *add, long long *mul, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***mat[4] = {matrehi, matrelo, matimhi, matimlo};
  double **rhs[4] = {rhsrehi, rhsrelo, rhsimhi, rhsimlo}, **sol[4] = {solrehi, solrelo, solimhi, solimlo};
  double **res[4] = {resvecrehi, resvecrelo, resvecimhi, resvecimlo};
  double *resmax[2] = {resmaxhi, resmaxlo};
  residue(2, 1, dim, degp1, tailidx, mat, rhs, sol, res, resmax, lapms, add, mul, "GPU_cmplx2_linear_residue");
}

void GPU_dbl2_evaluate_monomials(int dim, int deg, int szt, int nbt, int *nvr, int **idx, int **exp, int *nbrfac,
                                 int **expfac, double **cffhi, double **cfflo, double *acchi, double *acclo,
                                 double **inputhi, double **inputlo, double ***outputhi, double ***outputlo,
                                 double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)acchi; (void)acclo; (void)vrblvl;
  double **cff[2] = {cffhi, cfflo}, **in[2] = {inputhi, inputlo};
  double ***out[2] = {outputhi, outputlo};
  evaluate_monomials(2, 0, dim, deg, nvr, idx, exp, nbrfac, expfac, cff, in, out, totcnvlapsedms,
                     "GPU_dbl2_evaluate_monomials");
}

void GPU_cmplx2vectorized_evaluate_monomials(int dim, int deg, int szt, int nbt, int *nvr, int **idx, int **exp,
                                             int *nbrfac, int **expfac, double **cffrehi, double **cffrelo,
                                             double **cffimhi, double **cffimlo, double *accrehi, double *accrelo,
                                             double *accimhi, double *accimlo, double **inputrehi,
                                             double **inputrelo, double **inputimhi, double **inputimlo,
                                             double ***outputrehi, double ***outputrelo, double ***outputimhi,
                                             double ***outputimlo, double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)accrehi; (void)accrelo; (void)accimhi; (void)accimlo; (void)vrblvl;
  double **cff[4] = {cffrehi, cffrelo, cffimhi, cffimlo};
  double **in[4] = {inputrehi, inputrelo, inputimhi, inputimlo};
  double ***out[4] = {outputrehi, outputrelo, outputimhi, outputimlo};
  evaluate_monomials(2, 1, dim, deg, nvr, idx, exp, nbrfac, expfac, cff, in, out, totcnvlapsedms,
                     "GPU_cmplx2vectorized_evaluate_monomials");
}

void GPU_dbl2_evaluate_columns(int dim, int deg, int nbrcol, int szt, int nbt, int **nvr, int ***idx,
                               double ***cffhi, double ***cfflo, double **inputhi, double **inputlo,
                               double ***outputhi, double ***outputlo, double **funvalhi, double **funvallo,
                               double ***jacvalhi, double ***jacvallo, double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***cff[2] = {cffhi, cfflo}, ***out[2] = {outputhi, outputlo}, ***jac[2] = {jacvalhi, jacvallo};
  double **in[2] = {inputhi, inputlo}, **fun[2] = {funvalhi, funvallo};
  evaluate_columns(2, 0, dim, deg, nbrcol, nvr, idx, cff, in, out, fun, jac, totcnvlapsedms,
                   "GPU_dbl2_evaluate_columns");
}

void GPU_cmplx2_evaluate_columns(int dim, int deg, int nbrcol, int szt, int nbt, int **nvr, int ***idx,
                                 double ***cffrehi, double ***cffrelo, double ***cffimhi, double ***cffimlo,
                                 double **inputrehi, double **inputrelo, double **inputimhi, double **inputimlo,
                                 double ***outputrehi, double ***outputrelo, double ***outputimhi,
                                 double ***outputimlo, double **funvalrehi, double **funvalrelo,
                                 double **funvalimhi, double **funvalimlo, double ***jacvalrehi,
                                 double ***jacvalrelo, double ***jacvalimhi, double ***jacvalimlo,
                                 double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***cff[4] = {cffrehi, cffrelo, cffimhi, cffimlo};
  double ***out[4] = {outputrehi, outputrelo, outputimhi, outputimlo};
  double ***jac[4] = {jacvalrehi, jacvalrelo, jacvalimhi, jacvalimlo};
  double **in[4] = {inputrehi, inputrelo, inputimhi, inputimlo};
  double **fun[4] = {funvalrehi, funvalrelo, funvalimhi, funvalimlo};
  evaluate_columns(2, 1, dim, deg, nbrcol, nvr, idx, cff, in, out, fun, jac, totcnvlapsedms,
                   "GPU_cmplx2_evaluate_columns");
}

#else  // quad double: the dbl4 / cmplx4 twins

void GPU_dbl4_bals_solve(int dim, int degp1, int szt, int nbt, int tailidx, double ***mathihi, double ***matlohi,
                         double ***mathilo, double ***matlolo, double **Qhihi, double **Qlohi, double **Qhilo,
                         double **Qlolo, double **Rhihi, double **Rlohi, double **Rhilo, double **Rlolo,
                         double **rhshihi, double **rhslohi, double **rhshilo, double **rhslolo, double **solhihi,
                         double **sollohi, double **solhilo, double **sollolo, bool *zeroQ, bool *noqr, int *upidx,
                         int *bsidx, int *newtail, double *totqrlapsedms, double *totqtblapsedms,
                         double *totbslapsedms, double *totupdlapsedms, int vrblvl) {
  (void)nbt; (void)totqtblapsedms; (void)totbslapsedms; (void)totupdlapsedms; (void)vrblvl;
  double ***mat[4] = {mathihi, matlohi, mathilo, matlolo};
  double **Q[4] = {Qhihi, Qlohi, Qhilo, Qlolo}, **R[4] = {Rhihi, Rlohi, Rhilo, Rlolo};
  double **rhs[4] = {rhshihi, rhslohi, rhshilo, rhslolo}, **sol[4] = {solhihi, sollohi, solhilo, sollolo};
  bals(4, 0, dim, degp1, szt, tailidx, mat, Q, R, rhs, sol, zeroQ, noqr, upidx, bsidx, newtail, totqrlapsedms,
       "GPU_dbl4_bals_solve");
}

void GPU_cmplx4_bals_solve(int dim, int degp1, int szt, int nbt, int tailidx, double ***matrehihi,
                           double ***matrelohi, double ***matrehilo, double ***matrelolo, double ***matimhihi,
                           double ***matimlohi, double ***matimhilo, double ***matimlolo, double **Qrehihi,
                           double **Qrelohi, double **Qrehilo, double **Qrelolo, double **Qimhihi, double **Qimlohi,
                           double **Qimhilo, double **Qimlolo, double **Rrehihi, double **Rrelohi, double **Rrehilo,
                           double **Rrelolo, double **Rimhihi, double **Rimlohi, double **Rimhilo, double **Rimlolo,
                           double **rhsrehihi, double **rhsrelohi, double **rhsrehilo, double **rhsrelolo,
                           double **rhsimhihi, double **rhsimlohi, double **rhsimhilo, double **rhsimlolo,
                           double **solrehihi, double **solrelohi, double **solrehilo, double **solrelolo,
                           double **solimhihi, double **solimlohi, double **solimhilo, double **solimlolo,
                           bool *zeroQ, bool *noqr, int *upidx, int *bsidx, int *newtail, double *totqrlapsedms,
                           double *totqtblapsedms, double *totbslapsedms, double *totupdlapsedms, int vrblvl) {
  (void)nbt; (void)totqtblapsedms; (void)totbslapsedms; (void)totupdlapsedms; (void)vrblvl;
  double ***mat[8] = {matrehihi, matrelohi, matrehilo, matrelolo, matimhihi, matimlohi, matimhilo, matimlolo};
  double **Q[8] = {Qrehihi, Qrelohi, Qrehilo, Qrelolo, Qimhihi, Qimlohi, Qimhilo, Qimlolo};
  double **R[8] = {Rrehihi, Rrelohi, Rrehilo, Rrelolo, Rimhihi, Rimlohi, Rimhilo, Rimlolo};
  double **rhs[8] = {rhsrehihi, rhsrelohi, rhsrehilo, rhsrelolo, rhsimhihi, rhsimlohi, rhsimhilo, rhsimlolo};
  double **sol[8] = {solrehihi, solrelohi, solrehilo, solrelolo, solimhihi, solimlohi, solimhilo, solimlolo};
  bals(4, 1, dim, degp1, szt, tailidx, mat, Q, R, rhs, sol, zeroQ, noqr, upidx, bsidx, newtail, totqrlapsedms,
       "GPU_cmplx4_bals_solve");
}

void GPU_dbl4_linear_residue(int dim, int degp1, int szt, int nbt, int tailidx, double ***mathihi,
                             double ***matlohi, double ***mathilo, double ***matlolo, double **rhshihi,
                             double **rhslohi, double **rhshilo, double **rhslolo, double **solhihi,
                             double **sollohi, double **solhilo, double **sollolo, double **resvechihi,
                             double **resveclohi, double **resvechilo, double **resveclolo, double *resmaxhihi,
                             double *resmaxlohi, double *resmaxhilo, double *resmaxlolo, double *lapms,
                             long long *add, long long *mul, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***mat[4] = {mathihi, matlohi, mathilo, matlolo};
  double **rhs[4] = {rhshihi, rhslohi, rhshilo, rhslolo}, **sol[4] = {solhihi, sollohi, solhilo, sollolo};
  double **res[4] = {resvechihi, resveclohi, resvechilo, resveclolo};
  double *resmax[4] = {resmaxhihi, resmaxlohi, resmaxhilo, resmaxlolo};
  residue(4, 0, dim, degp1, tailidx, mat, rhs, sol, res, resmax, lapms, add, mul, "GPU_dbl4_linear_residue");
}

void GPU_cmplx4_linear_residue(int dim, int degp1, int szt, int nbt, int tailidx, double ***matrehihi,
                               double ***matrelohi, double ***matrehilo, double ***matrelolo, double ***matimhihi,
                               double ***matimlohi, double ***matimhilo, double ***matimlolo, double **rhsrehihi,
                               double **rhsrelohi, double **rhsrehilo, double **rhsrelolo, double **rhsimhihi,
                               double **rhsimlohi, double **rhsimhilo, double **rhsimlolo, double **solrehihi,
                               double **solrelohi, double **solrehilo, double **solrelolo, double **solimhihi,
                               double **solimlohi, double **solimhilo, double **solimlolo, double **resvecrehihi,
                               double **resvecrelohi, double **resvecrehilo, double **resvecrelolo,
                               double **resvecimhihi, double **resvecimlohi, double **resvecimhilo,
                               double **resvecimlolo, double *resmaxhihi, double *resmaxlohi, double *resmaxhilo,
                               double *resmaxlolo, double *lapms, long long *add, long long *mul, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***mat[8] = {matrehihi, matrelohi, matrehilo, matrelolo, matimhihi, matimlohi, matimhilo, matimlolo};
  double **rhs[8] = {rhsrehihi, rhsrelohi, rhsrehilo, rhsrelolo, rhsimhihi, rhsimlohi, rhsimhilo, rhsimlolo};
  double **sol[8] = {solrehihi, solrelohi, solrehilo, solrelolo, solimhihi, solimlohi, solimhilo, solimlolo};
  double **res[8] = {resvecrehihi, resvecrelohi, resvecrehilo, resvecrelolo,
                     resvecimhihi, resvecimlohi, resvecimhilo, resvecimlolo};
  double *resmax[4] = {resmaxhihi, resmaxlohi, resmaxhilo, resmaxlolo};
  residue(4, 1, dim, degp1, tailidx, mat, rhs, sol, res, resmax, lapms, add, mul, "GPU_cmplx4_linear_residue");
}

void GPU_dbl4_evaluate_monomials(int dim, int deg, int szt, int nbt, int *nvr, int **idx, int **exp, int *nbrfac,
                                 int **expfac, double **cffhihi, double **cfflohi, double **cffhilo,
                                 double **cfflolo, double *acchihi, double *acclohi, double *acchilo,
                                 double *acclolo, double **inputhihi, double **inputlohi, double **inputhilo,
                                 double **inputlolo, double ***outputhihi, double ***outputlohi,
                                 double ***outputhilo, double ***outputlolo, double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)acchihi; (void)acclohi; (void)acchilo; (void)acclolo; (void)vrblvl;
  double **cff[4] = {cffhihi, cfflohi, cffhilo, cfflolo}, **in[4] = {inputhihi, inputlohi, inputhilo, inputlolo};
  double ***out[4] = {outputhihi, outputlohi, outputhilo, outputlolo};
  evaluate_monomials(4, 0, dim, deg, nvr, idx, exp, nbrfac, expfac, cff, in, out, totcnvlapsedms,
                     "GPU_dbl4_evaluate_monomials");
}

void GPU_cmplx4vectorized_evaluate_monomials(
    int dim, int deg, int szt, int nbt, int *nvr, int **idx, int **exp, int *nbrfac, int **expfac,
    double **cffrehihi, double **cffrelohi, double **cffrehilo, double **cffrelolo, double **cffimhihi,
    double **cffimlohi, double **cffimhilo, double **cffimlolo, double *accrehihi, double *accrelohi,
    double *accrehilo, double *accrelolo, double *accimhihi, double *accimlohi, double *accimhilo,
    double *accimlolo, double **inputrehihi, double **inputrelohi, double **inputrehilo, double **inputrelolo,
    double **inputimhihi, double **inputimlohi, double **inputimhilo, double **inputimlolo,
    double ***outputrehihi, double ***outputrelohi, double ***outputrehilo, double ***outputrelolo,
    double ***outputimhihi, double ***outputimlohi, double ***outputimhilo, double ***outputimlolo,
    double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  (void)accrehihi; (void)accrelohi; (void)accrehilo; (void)accrelolo;
  (void)accimhihi; (void)accimlohi; (void)accimhilo; (void)accimlolo;
  double **cff[8] = {cffrehihi, cffrelohi, cffrehilo, cffrelolo, cffimhihi, cffimlohi, cffimhilo, cffimlolo};
  double **in[8] = {inputrehihi, inputrelohi, inputrehilo, inputrelolo,
                    inputimhihi, inputimlohi, inputimhilo, inputimlolo};
  double ***out[8] = {outputrehihi, outputrelohi, outputrehilo, outputrelolo,
                      outputimhihi, outputimlohi, outputimhilo, outputimlolo};
  evaluate_monomials(4, 1, dim, deg, nvr, idx, exp, nbrfac, expfac, cff, in, out, totcnvlapsedms,
                     "GPU_cmplx4vectorized_evaluate_monomials");
}

void GPU_dbl4_evaluate_columns(int dim, int deg, int nbrcol, int szt, int nbt, int **nvr, int ***idx,
                               double ***cffhihi, double ***cfflohi, double ***cffhilo, double ***cfflolo,
                               double **inputhihi, double **inputlohi, double **inputhilo, double **inputlolo,
                               double ***outputhihi, double ***outputlohi, double ***outputhilo,
                               double ***outputlolo, double **funvalhihi, double **funvallohi, double **funvalhilo,
                               double **funvallolo, double ***jacvalhihi, double ***jacvallohi,
                               double ***jacvalhilo, double ***jacvallolo, double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***cff[4] = {cffhihi, cfflohi, cffhilo, cfflolo};
  double ***out[4] = {outputhihi, outputlohi, outputhilo, outputlolo};
  double ***jac[4] = {jacvalhihi, jacvallohi, jacvalhilo, jacvallolo};
  double **in[4] = {inputhihi, inputlohi, inputhilo, inputlolo};
  double **fun[4] = {funvalhihi, funvallohi, funvalhilo, funvallolo};
  evaluate_columns(4, 0, dim, deg, nbrcol, nvr, idx, cff, in, out, fun, jac, totcnvlapsedms,
                   "GPU_dbl4_evaluate_columns");
}

void GPU_cmplx4_evaluate_columns(
    int dim, int deg, int nbrcol, int szt, int nbt, int **nvr, int ***idx, double ***cffrehihi,
    double ***cffrelohi, double ***cffrehilo, double ***cffrelolo, double ***cffimhihi, double ***cffimlohi,
    double ***cffimhilo, double ***cffimlolo, double **inputrehihi, double **inputrelohi, double **inputrehilo,
    double **inputrelolo, double **inputimhihi, double **inputimlohi, double **inputimhilo, double **inputimlolo,
    double ***outputrehihi, double ***outputrelohi, double ***outputrehilo, double ***outputrelolo,
    double ***outputimhihi, double ***outputimlohi, double ***outputimhilo, double ***outputimlolo,
    double **funvalrehihi, double **funvalrelohi, double **funvalrehilo, double **funvalrelolo,
    double **funvalimhihi, double **funvalimlohi, double **funvalimhilo, double **funvalimlolo,
    double ***jacvalrehihi, double ***jacvalrelohi, double ***jacvalrehilo, double ***jacvalrelolo,
    double ***jacvalimhihi, double ***jacvalimlohi, double ***jacvalimhilo, double ***jacvalimlolo,
    double *totcnvlapsedms, int vrblvl) {
  (void)szt; (void)nbt; (void)vrblvl;
  double ***cff[8] = {cffrehihi, cffrelohi, cffrehilo, cffrelolo, cffimhihi, cffimlohi, cffimhilo, cffimlolo};
  double ***out[8] = {outputrehihi, outputrelohi, outputrehilo, outputrelolo,
                      outputimhihi, outputimlohi, outputimhilo, outputimlolo};
  double ***jac[8] = {jacvalrehihi, jacvalrelohi, jacvalrehilo, jacvalrelolo,
                      jacvalimhihi, jacvalimlohi, jacvalimhilo, jacvalimlolo};
  double **in[8] = {inputrehihi, inputrelohi, inputrehilo, inputrelolo,
                    inputimhihi, inputimlohi, inputimhilo, inputimlolo};
  double **fun[8] = {funvalrehihi, funvalrelohi, funvalrehilo, funvalrelolo,
                     funvalimhihi, funvalimlohi, funvalimhilo, funvalimlolo};
  evaluate_columns(4, 1, dim, deg, nbrcol, nvr, idx, cff, in, out, fun, jac, totcnvlapsedms,
                   "GPU_cmplx4_evaluate_columns");
}

#endif
