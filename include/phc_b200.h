/* phc_b200.h -- C ABI of the B200 multiple-double power-series library.
 *
 * Conventions shared by every entry point:
 *   - prec is the number of limbs: 1 (double), 2 (double-double),
 *     4 (quad-double); cplx != 0 selects complex numbers.
 *   - Numbers are stored limb-interleaved: a real number is prec consecutive
 *     doubles (most significant first), a complex number 2*prec doubles
 *     (real limbs, then imaginary limbs).  A truncated power series of
 *     degree deg is deg+1 consecutive numbers.  Matrices are row-major.
 *   - Plain entry points take DEVICE pointers and a cudaStream_t passed as
 *     void* (NULL = legacy default stream); they enqueue work and return
 *     without synchronising.  *_host entry points take HOST pointers, stage
 *     the data on the device, run, copy the results back and synchronise,
 *     like the reference's GPU_* host drivers.
 *   - Return value: 0 ok, > 0 a count of failed items (e.g. paths that did
 *     not converge), < 0 an error: -1 bad argument, -2 CUDA error,
 *     -3 size beyond a kernel limit, -4 a bounded device wait gave up.
 *     phc_last_error() returns the text of the last error on this thread.
 *
 * Reference interfaces replaced (paths relative to PHCpack's src/GPU) are
 * named above each declaration.
 */
#ifndef PHC_B200_H
#define PHC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PHC_ABI_VERSION 1

const char *phc_last_error(void);
int phc_abi_version(void);

/* Evaluation and differentiation of a batch of nsys polynomial systems of
 * dimension dim at a vector of power series truncated at degree deg.
 *
 * Replaces Polynomials/dbl2_polynomials_kernels.h GPU_dbl2_poly_evaldiff
 * (body at dbl2_polynomials_kernels.cu:1577), its cmplx2 / dbl4 / cmplx4
 * twins, and the monomial-form Newton/dbl2_systems_kernels.cu:848
 * GPU_dbl2_evaluate_monomials (exponents > 1 by the common-factor method),
 * batched over systems and polynomials in one launch.
 *
 * Supports: polynomial p of system s owns monomials
 *   mon_off[s*dim+p] .. mon_off[s*dim+p+1]-1   (mon_off has nsys*dim+1 entries);
 * monomial m has nvr[m] distinct variables idx[m*maxvar + j] with exponents
 * exps[m*maxvar + j] >= 1, j < nvr[m].
 * cst:    nsys*dim constant series;  cff: one coefficient series per monomial;
 * input:  nsys*dim input series (system s, variable j);
 * output: nsys*dim*(dim+1) series; polynomial (s,p) occupies dim+1 series,
 *         series j < dim the derivative with respect to x_j, series dim the
 *         value (the reference's output[dim] convention).
 * Limit: deg <= 31. */
int phc_system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                        const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                        const double *input, double *output, void *stream);
int phc_system_evaldiff_host(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                             const int *nvr, const int *idx, const int *exps, const double *cst,
                             const double *cff, const double *input, double *output, void *stream);

/* ---------------------------------------------------------------- Matrices
 * Batched dense linear algebra, one instance per CTA.  The device entry
 * points take a workspace of ninst * phc_dense_workspace_bytes(...) bytes
 * (WY panels, products, inverted diagonal tiles of R).
 */
long long phc_dense_workspace_bytes(int prec, int cplx, int n, int szt);

/* A = Q R for ninst matrices A (nrows x ncols, ncols = szt*nbt <= nrows),
 * Q nrows x nrows, R nrows x ncols.  Replaces Matrices/dbl2_baqr_kernels.h
 * GPU_dbl2_blocked_houseqr (body at dbl2_baqr_kernels.cu:3520) and its
 * cmplx2 / dbl4 / cmplx4 twins: Householder reflectors in PHCpack's
 * convention, applied per column inside a tile, then the WY trailing updates
 * R += Y (W^H R) and Q += (Q W) Y^H. */
int phc_blocked_houseqr(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A, double *Q,
                        double *R, double *work, void *stream);
int phc_blocked_houseqr_host(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A,
                             double *Q, double *R, void *stream);

/* x = U^{-1} b for ninst upper triangular U (dim = szt*nbt) by inverting the
 * diagonal tiles and block back substitution.  Replaces
 * Matrices/dbl2_tabs_kernels.h GPU_dbl2_upper_tiled_solver (body at
 * dbl2_tabs_kernels.cu:952); like it, overwrites the diagonal tiles of U
 * with their inverses and b with the updated right hand sides.  work: dim*szt
 * numbers per instance. */
int phc_upper_tiled_solver(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x,
                           double *work, void *stream);
int phc_upper_tiled_solver_host(int prec, int cplx, int ninst, int dim, int szt, double *U, double *b, double *x,
                                void *stream);

/* ------------------------------------------------------------------ Newton
 * Block lower-triangular Toeplitz least squares sum_{j<=k} A_j x_{k-j} = b_k,
 * k < degp1, for ninst instances (mat: degp1 matrices dim x dim; rhs, sol:
 * degp1 vectors of dim; Q, R: dim x dim).  Replaces
 * Newton/dbl2_bals_kernels.cu:554 GPU_dbl2_bals_solve (head :108, tail
 * dbl2_tail_kernels.cu:154) and twins, with the reference's skip rules.
 * flags: 5 ints per instance, in/out: zeroQ, noqr, upidx, bsidx, newtail.
 * tailidx >= 1 starts the tail there for every instance; tailidx < 0 takes
 * each instance's flags[4].  rhs is overwritten. */
int phc_bals_solve(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                   double *rhs, double *sol, double *Q, double *R, int *flags, double *work, void *stream);
int phc_bals_solve_host(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                        double *rhs, double *sol, double *Q, double *R, int *flags, void *stream);

/* One Newton step on power series for nsys systems (row form) at working
 * degree deg <= maxdeg: evaluate and differentiate (phc_system_evaldiff),
 * linearise (matrix series -> series of matrices, rhs = -f), solve
 * (phc_bals_solve with each system's tail index in flags[4]), update
 * x[i][j] += dx[j][i] for j >= newtail - 1.  series, cst, cff are stored with
 * capacity maxdeg+1 per series.  Replaces Newton/dbl2_newton_method.h:406
 * dbl2_row_newton_qrstep (GPU mode) and its cmplx / dbl4 twins.  work:
 * phc_newton_workspace_bytes(...) bytes.  flags start at zeroQ=1, noqr=0,
 * tail=1. */
long long phc_newton_workspace_bytes(int prec, int cplx, int nsys, int dim, int deg, int szt, long long nmon);
int phc_newton_step(int prec, int cplx, int nsys, int dim, int deg, int maxdeg, int szt, int maxvar,
                    const int *mon_off, long long nmon, const int *nvr, const int *idx, const int *exps,
                    const double *cst, const double *cff, double *series, double *Q, double *R, int *flags,
                    double *work, void *stream);
/* The Newton loop of Newton/dbl2_newton_method.cpp:1455-1492 on host
 * arrays: nsteps steps, schedule 0 = fixed degree deg, 1 = the reference's
 * working-degree schedule with its stop rule. */
int phc_newton_host(int prec, int cplx, int nsys, int dim, int deg, int szt, int maxvar, const int *mon_off,
                    const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                    double *series, int nsteps, int schedule, int *flags, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PHC_B200_H */
