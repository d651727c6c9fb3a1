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

#define PHC_ABI_VERSION 2

const char *phc_last_error(void);
int phc_abi_version(void);

/* Launch-shape knobs, process-wide, set by the autotuner
 * (phcpack_b200/autotune.py); value 0 restores the built-in rule.  No
 * counterpart in the reference, whose launch shapes are fixed at compile
 * time or passed per call.
 *   knob 0: polynomials (warps) per CTA of phc_system_evaldiff, 1..8
 *           (the rule: min(dim, 8), fewer when the scratch needs it);
 *   knob 1: variant of the split tracker's kernel, 1 the 64-register one
 *           (8 paths per SM), 2 the 72-register one (7 paths per SM) (the
 *           rule: 2 when the batch fits in one wave at 7 per SM);
 *   knob 2: paths the tracker runs at once per SM, 1..32, at most what the
 *           occupancy allows (the rule: that maximum); the work queue hands
 *           out the other paths as paths finish;
 *   knob 3: blocked QR and least squares: 2 stages the WY panels and the
 *           column panel of R in shared memory when they fit (one CTA per
 *           SM), 0 or 1 keeps them in global memory (the rule: global).
 * phc_tune_get returns the value (>= 0) or an error. */
int phc_tune_set(int knob, int value);
int phc_tune_get(int knob);

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
 * Limit: deg <= 191 (the reference's largest degree); series of up to 32
 * coefficients take one warp per product, longer ones a lane per
 * coefficient (k, k + 32, ...). */
int phc_system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                        const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                        const double *input, double *output, void *stream);
/* The host entry copies the systems in, evaluates and copies out in chunks
 * on two streams; the copies overlap the evaluation only when the host
 * arrays are pinned (cudaHostAlloc / cudaHostRegister): with pageable
 * memory each copy out blocks the issuing thread and the chunks run one
 * after another. */
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

/* The residual of the linearised power-series system: for tailidx <= i <
 * degp1, res_i = rhs_i - sum_{j=0}^{i-tailidx} A_j sol_{i-j} (rows i <
 * tailidx of res are left as they are), for ninst instances laid out as in
 * phc_bals_solve; resmax: prec doubles per instance, the per-limb
 * magnitudes of the entry of res with the largest leading limb (|re| + |im|
 * for complex numbers), as the reference's resmaxhi, resmaxlo.  Replaces
 * Newton/dbl2_tail_kernels.h GPU_dbl2_linear_residue (body at
 * dbl2_tail_kernels.cu:383, host twin dbl2_bals_host.cpp:548) and twins. */
int phc_linear_residue(int prec, int cplx, int ninst, int dim, int degp1, int tailidx, const double *mat,
                       const double *rhs, const double *sol, double *res, double *resmax, void *stream);
int phc_linear_residue_host(int prec, int cplx, int ninst, int dim, int degp1, int tailidx, const double *mat,
                            const double *rhs, const double *sol, double *res, double *resmax, void *stream);

/* The same QR and least-squares solve with a choice of how the four WY
 * trailing products of each tile (R += Y (W^T C), Q += (Q W^T) Y) run:
 * wy = 0 on the CUDA cores in multiple-double arithmetic (as above), wy = 1
 * as Ozaki-split products on the FP64 tensor cores (mma.sync m8n8k4 f64):
 * each operand cut into 21-bit slices on per-row / per-column exponent
 * grids so that every slice product and every inner sum is exact, the sums
 * of equal order added into the multiple-double result.  wy = 1 applies to
 * real numbers with dim <= 64 (complex numbers keep the CUDA-core products).
 * The products of Matrices/dbl2_baqr_kernels.cu:2872-3444 (dbl2_small_WYT,
 * _QWYT, _Qupdate, _YWTC, _R_add_YWTC) in the reference run one thread per
 * entry on CUDA cores.  Workspace: ninst * phc_dense_workspace_bytes_wy(...). */
long long phc_dense_workspace_bytes_wy(int prec, int cplx, int n, int szt, int wy);
int phc_blocked_houseqr_wy(int prec, int cplx, int ninst, int nrows, int ncols, int szt, const double *A, double *Q,
                           double *R, double *work, int wy, void *stream);
int phc_bals_solve_wy(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
                      double *rhs, double *sol, double *Q, double *R, int *flags, double *work, int wy, void *stream);

/* phc_bals_solve without any allocation.  No counterpart in the reference:
 * this entry point is for callers that cannot let a library call cudaMalloc
 * or cudaFree (latency-critical callers that cannot afford cudaFree's
 * device-wide synchronisation, frameworks whose own allocator owns and
 * accounts for all device memory, code that must not allocate once it has
 * been set up).
 * Same arguments and results as phc_bals_solve minus the workspace, which
 * is a static device array of phc_bals_solve_static_capacity_bytes() bytes
 * (8 MiB, held by every GPU that loads the library until exit); larger
 * requests fail with -3.  All calls share that array: calls that overlap on
 * the GPU race and must be serialised.  The first call on a device looks up
 * the array's address and should come before any stream capture; the
 * address is kept for the process, so do not use the library across a
 * device reset (cudaDeviceReset). */
long long phc_bals_solve_static_capacity_bytes(void);
int phc_bals_solve_static(int prec, int cplx, int ninst, int dim, int degp1, int szt, int tailidx, const double *mat,
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

/* ------------------------------------------------------------------ Track
 * Batched series-Pade path tracking of homotopies
 *   h(x, t) = sum over terms ((1 - t) a + t b) x^e,  t from 0 to 1,
 * which is (1 - t) gamma q(x) + t p(x) with a = gamma c_q, b = c_p (the
 * form of Path/Path_GPU/eval_coef.cu:27-28; at t = 1 the target's
 * coefficients are used exactly).
 * Replaces the tracker behind the Ada/phcpy C interface:
 * Ada/PHCtoC/gpumanypaths_dd.h:27 gpumanypaths_dd (and _d, _qd), whose
 * internal GPU_Path_mult (Path/Path_GPU/path_gpu.h:38) tracks many paths and
 * returns per-path success flags, with the algorithm of the Ada series-Pade
 * tracker (Curves/predictor_corrector_trackers.adb:51).
 *
 * Systems: nsys systems; system s has dim[s] variables and equations;
 *   distinct monomials mono_off[s] .. mono_off[s+1]-1, monomial m has
 *   mono_nvr[m] (0 = the constant 1) distinct variables mono_idx[m*maxvar+v]
 *   with exponents mono_exp[m*maxvar+v];
 *   equations eq_off[s] .. eq_off[s+1]-1 (dim[s] of them), equation e has
 *   terms term_off[e] .. term_off[e+1]-1, term r is ((1 - t) a + t b) times monomial
 *   term_mono[r] (global id), a = term_a[2r] + i term_a[2r+1], b likewise.
 * Jacobian gather lists (from phc_track_prepare): for (equation e, variable
 *   j) the entries jg_off[e*maxdim+j] .. jg_off[e*maxdim+j+1]-1 of jg_term,
 *   jg_slot.  A slot >= 0 is the variable's place in the term's monomial
 *   (the partial is staged in shared memory); for monomials of total degree
 *   <= 2 the partial is read in place: -1 the constant 1, -2 the series
 *   2 x_j, -3-l the series x_l.  phc_track_prepare returns the number of
 *   staged entries; pass it as gstaged to phc_track and phc_track_smem_bytes
 *   (0 drops the staging buffer from shared memory).
 * Paths: path p belongs to system path_sys[p] and starts at x0 (maxdim complex
 *   doubles per path).
 * ipar: deg (series degree K), numdeg (L), dendeg (M), nit (>= 1; the
 *   reference's number of Newton steps on the series, unused: the Taylor
 *   coefficients are computed one degree at a time, the fixed point those
 *   steps approach), corsteps, maxsteps, refine_steps.
 * dpar: pbeta, alpha, maxsize, minsize, tolres, epsilon, restol (endpoint
 *   residual bound), learn_scale (multiplies learned proposals; 0 = 1),
 *   cbeta (the curvature step's factor, beta2; 0.005 in the reference's
 *   defaults, Curves/homotopy_continuation_parameters.adb:13).
 * Step rule per predictor step (LU_Prediction,
 *   Curves/standard_predictor_convolutions.adb:1170-1184, with Hesse_Pade as
 *   in Curves/dobldobl_predictor_convolutions.adb:383-406): the smallest of
 *   the pole step pbeta * r (r the smallest Fabry radius |c_{K-3}/c_{K-2}|;
 *   maxsize when no component has a radius), the curvature step
 *   (cbeta eta / |Pade errors|_2)^(1/K) with eta = 2 sigma_min(J) /
 *   |(sigma_max(H_1), ..., sigma_max(H_n))|_2 at the current point, and
 *   maxsize; a step that reaches 1 - minsize goes to t = 1 (Bounded_Update).
 * pmode: 1 (double) or 2 (double-double), the precision of the predictor
 *   and of the corrector's Jacobian and linear solves; the corrector's
 *   residuals and updates are double-double; rmode: refinement precision 2,
 *   4 (quad-double) or 8 (octo-double), all of its arithmetic.
 * step_mode: bit 1 (value 1) with a model (phc_mlp_*) uses the learned step
 *   proposer; a proposal whose feedback or corrector fails is redone with
 *   the plain step.  Bit 2 (value 2, pmode 1 only): the predictor inverts
 *   J_0 by Householder QR in double (the reflectors of the reference's
 *   complex convention, applied column by column) instead of LU, the QR
 *   solve of the power-series Newton step (Newton/dbl2_newton_method.cpp
 *   :429) in the predictor's double precision.
 * Output per path: xend maxdim complex quad-doubles, octo-doubles for rmode
 *   8 (lower limbs zero below rmode), info[6p..6p+5] = status (0 success,
 *   1 step below minsize, 2 maxsteps reached, 3 endpoint residual above
 *   restol), steps, rejected steps, and how often the step was the pole
 *   step, the curvature step and maxsize (the reference's nbpole, nbhess,
 *   nbmaxm); dinfo[2p..2p+1] = final t, endpoint residual.
 * log: when not NULL, each accepted step appends 32 floats (24 features,
 *   accepted step, plain step, proposed step, t, largest probed step that
 *   passes the feedback) up to log_cap records;
 *   *log_count counts them.  queue: one device int (the work-queue counter).
 * one_per_launch != 0 tracks one path per launch (one CTA), back to back:
 *   the plain arrangement the batched kernel is measured against. */
long long phc_track_gather_count(int nsys, const int *mono_off, const int *mono_nvr, const int *eq_off,
                                 const int *term_off, const int *term_mono);
int phc_track_prepare(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                      const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                      const int *term_mono, int maxdim, int *jg_off, int *jg_term, int *jg_slot);
long long phc_track_smem_bytes(int maxdim, int deg, int dendeg, int nmono_max, int maxvar, int pmode, int rmode,
                               int gstaged);
int phc_track(int nsys, const int *dim, int maxvar, int maxdim, int nmono_max, const int *mono_off,
              const int *mono_nvr, const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
              const int *term_mono, const double *term_a, const double *term_b, const int *jg_off,
              const int *jg_term, const int *jg_slot, int gstaged, int npaths, const int *path_sys,
              const double *x0, const int *ipar, const double *dpar, int pmode, int rmode, int step_mode,
              const void *model, double *xend, int *info, double *dinfo, float *log, int log_cap, int *log_count,
              int *queue, int one_per_launch, void *stream);
/* Host arrays in and out; returns the number of paths not classified as
 * success (>= 0) or an error (< 0).  The device buffer and a pinned staging
 * buffer are kept per device between calls (grown when needed; inputs go
 * over in one copy, outputs back in one); calls are serialised;
 * phc_track_host_release() frees the buffers. */
int phc_track_host(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                   const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                   const int *term_mono, const double *term_a, const double *term_b, int npaths,
                   const int *path_sys, const double *x0, const int *ipar, const double *dpar, int pmode, int rmode,
                   int step_mode, const void *model, double *xend, int *info, double *dinfo, void *stream);
void phc_track_host_release(void);

/* ------------------------------------------- the tracker's drop-in entry
 * gpumanypaths_d, gpumanypaths_dd, gpumanypaths_qd replace the functions of
 * the same names and signatures in Ada/PHCtoC/gpumanypaths_d.h,
 * gpumanypaths_dd.h:27 and gpumanypaths_qd.h (bodies gpumanypaths_dd.cpp
 * :18-62), which phcpy calls as py2c_gpu_manypaths_dd(mode, verbose,
 * regamma, imgamma) (Mod/phcpy2cpath_dd.cpp:4593).  Like them, they read
 * the target system p, the start system q and the start solutions from the
 * containers, track every path of (1 - t) gamma q + t p with gamma =
 * regamma + i imgamma, and write the end points back into the solution
 * container.  mode: 0 (CPU and GPU in the reference; here the GPU, whose
 * end points the reference writes back in this mode too), 1 (CPU only:
 * refused, -1, as this library tracks on the GPU), 2 (GPU); verbose > 0
 * prints what the reference prints.  Returns 0 when the paths were tracked
 * (per-path status in the container), < 0 on an error.  End points are
 * refined in double-double (_d, _dd) or quad-double (_qd); the tracker is
 * phc_track_host with the parameters of phc_container_set_parameters
 * (default: degree 8, [4/4] Pade, the reference's step rules).
 *
 * The containers: PHCpack keeps the systems and solutions in its Ada
 * containers (syscon, solcon), which need the Ada runtime; this library
 * keeps its own with the same content.  A system of neq polynomials in
 * nvar variables: polynomial i has nterms[i] terms; term r (the terms of
 * all polynomials in order) has the exponents exps[r*nvar .. r*nvar+nvar-1]
 * and the complex coefficient cff[2r] + i cff[2r+1] (rounded to double, as
 * the tracker's coefficients are doubles).  Solutions: coordinate j of
 * solution s has the limbs doubles per part (1, 2 or 4) at
 * sols[((s*nvar + j)*2 + part)*limbs + l], part 0 real and 1 imaginary; start
 * solutions are rounded to double.  After tracking, get_solutions gives the
 * end points with t, the status (0 success, 1 step below minsize, 2
 * maxsteps, 3 residual above restol) and the endpoint residual per
 * solution (any of its output pointers may be NULL). */
int phc_container_set_target(int neq, int nvar, const int *nterms, const int *exps, const double *cff);
int phc_container_set_start(int neq, int nvar, const int *nterms, const int *exps, const double *cff);
int phc_container_set_solutions(int nsols, int nvar, int limbs, const double *sols);
int phc_container_number_of_solutions(int *nsols);
/* the number of variables of the solutions (else of the target), 0 when empty */
int phc_container_dimension(int *nvar);
int phc_container_get_solutions(int limbs, double *sols, double *t, int *status, double *res);
/* ipar[7] and dpar[9] as in phc_track */
int phc_container_set_parameters(const int *ipar, const double *dpar);
void phc_container_clear(void);
int gpumanypaths_d(int mode, int verbose, double regamma, double imgamma);
int gpumanypaths_dd(int mode, int verbose, double regamma, double imgamma);
int gpumanypaths_qd(int mode, int verbose, double regamma, double imgamma);

/* The mixed volume of the Newton polytopes of a square system in n
 * variables (the BKK bound on its isolated roots with nonzero coordinates):
 * the method of MixedVol, Ada Root_Counts/MixedVol/mixedvol_algorithm.adb
 * (mv, the C code mixed_volume1.c, relation_table1.c, one_level_lp1.c):
 * random lifting from seed, the mixed cells of the induced subdivision by a
 * depth-first search with LP feasibility tests, the volume the sum of
 * |det| over the cells.  Support i has counts[i] exponent vectors of n ints,
 * stored support after support in pts.  cells (may be NULL): up to
 * max_cells cells, each n pairs (p_i, q_i) of point indices within the
 * supports; *ncells (may be NULL): the number of mixed cells.  Host code
 * only (no device work).  Returns the mixed volume (>= 0) or an error. */
long long phc_mixed_volume(int n, const int *counts, const int *pts, unsigned long long seed, int max_cells,
                           int *cells, long long *ncells);

/* End-game diagnostics at points (x, t) of the homotopies of phc_track: the
 * Newton-Fabry convergence radius of the path's series and the Hessian
 * distance to the nearest singular solution, with the curvature step of the
 * Pade predictor.  Replaces, batched over points:
 *   Newton_Fabry      Ada Deformations/Curves/dobldobl_fabry_on_homotopy.adb:30-83
 *   Fabry             Ada Math_Lib/Circuits/convergence_radius_estimates.adb:138-163,392-425
 *   Distance          Ada Deformations/Curves/singular_values_of_hessians.adb:190-211
 *   Hesse_Pade        Ada Deformations/Curves/dobldobl_predictor_convolutions.adb:368-406
 *   Step_Distance     Ada Deformations/Curves/series_and_predictors.adb:813-825
 * Systems: the device arrays of phc_track (gather lists from
 *   phc_track_prepare).  Point p lies on system path_sys[p] at t = tpt[p]
 *   with x at xpt: maxdim complex numbers per point, xlimbs doubles per part
 *   (the real limbs, then the imaginary limbs; xlimbs 1, 2, 4 or 8, so that
 *   start points (1) and the end points of phc_track (4, or 8 after an
 *   octo-double refinement) are read as they are).
 * ipar: deg K (3..16, the degree of the series), numdeg L and dendeg M
 *   (L + M <= K, M <= 8: the Pade approximant of the curvature step),
 *   offset (0..K-2: the Fabry ratio is c_{K-1-offset} / c_{K-offset}; 1 in
 *   Newton_Fabry), newton_steps (0..64 Newton steps at t before the series;
 *   0 = none).
 * dpar: tolres (Newton's bound on max |dx|), beta2 (factor of the curvature
 *   step; 0.005 in the reference's defaults).
 * pmode: 1, 2 or 4: double, double-double or quad-double for Newton, the
 *   series, Fabry and Pade; the Jacobian and the Hessians are rounded to
 *   double for their singular values (one-sided Jacobi).
 * Outputs per point: series (may be NULL): maxdim x (K+1) complex numbers
 *   in the working precision (2 * pmode doubles each: real limbs, then
 *   imaginary limbs); dout (10 doubles): z (real, imaginary; the singular
 *   point is at t + z), the radius |z|, Fabry's error estimate,
 *   sigma_min(J), the 2-norm of the Hessians' largest singular values, eta =
 *   2 sigma_min(J) / that norm (+inf when every Hessian is zero), the 2-norm
 *   of the Pade error estimates, the curvature step (beta2 eta / that
 *   norm)^(1/K), Newton's last max |dx|; iout (2 ints): 1 when Fabry fails
 *   (every component's c_{K-offset} is negligible, or no series), and the
 *   status: 0, 1 (singular Jacobian at the point: no series) or 2 (Newton did
 *   not reach tolres).  Device pointers; no counterpart of this batching in
 *   the reference, which runs these one solution at a time on the host. */
int phc_series_diagnostics(int nsys, const int *dim, int maxvar, int maxdim, int nmono_max, const int *mono_off,
                           const int *mono_nvr, const int *mono_idx, const int *mono_exp, const int *eq_off,
                           const int *term_off, const int *term_mono, const double *term_a, const double *term_b,
                           const int *jg_off, const int *jg_term, const int *jg_slot, int gstaged, int npaths,
                           const int *path_sys, const double *xpt, int xlimbs, const double *tpt, const int *ipar,
                           const double *dpar, int pmode, double *series, double *dout, int *iout, void *stream);
/* Host arrays in and out (the same arguments; the gather lists are built
 * here); allocates and frees its device memory per call. */
int phc_series_diagnostics_host(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                                const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                                const int *term_mono, const double *term_a, const double *term_b, int npaths,
                                const int *path_sys, const double *xpt, int xlimbs, const double *tpt,
                                const int *ipar, const double *dpar, int pmode, double *series, double *dout,
                                int *iout);
/* ------------------------------------------------------- learned step size
 * No counterpart in the reference (its trackers use the ratio / Pade pole
 * and curvature steps only).  A 24 -> 128 -> 128 -> 1 ReLU network predicts
 * log(accepted step / pole step) from 24 features of the predictor's series
 * (phcpack_b200/csrc/mlp.cuh).  Model buffer: FP32 normalisation and biases,
 * BF16 weights, phc_mlp_model_bytes() bytes, 16-byte aligned (phc_track
 * checks).  Training keeps FP32 master
 * parameters (phc_mlp_param_count() floats: W1[128][24], b1[128],
 * W2[128][128], b2[128], W3[128], b3) and Adam moments of the same size. */
long long phc_mlp_model_bytes(void);
long long phc_mlp_param_count(void);
/* params + normalisation (24 means, 24 inverse deviations) -> model buffer */
int phc_mlp_pack(const float *params, const float *mean, const float *inv_std, void *model, void *stream);
/* out[b] = network(X[b]) for nb samples of 24 floats */
int phc_mlp_forward(const void *model, int nb, const float *X, float *out, void *stream);
/* grad += d/dparams of the mean squared error over (X, y); loss += that error */
int phc_mlp_grad(const void *model, int nb, const float *X, const float *y, float *grad, float *loss, void *stream);
/* one Adam step (t >= 1) on params from grad, which is cleared */
int phc_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                 int t, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PHC_B200_H */
