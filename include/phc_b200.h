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

#ifdef __cplusplus
}
#endif

#endif /* PHC_B200_H */
