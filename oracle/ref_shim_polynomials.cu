// ref_shim_polynomials.cu -- PHCpack's device entry points for the
// evaluation and differentiation of one polynomial at power series, with
// the reference's exact signatures, implemented on this library's C ABI:
//   GPU_dbl2_poly_evaldiff               Polynomials/dbl2_polynomials_kernels.h:812
//   GPU_cmplx2_poly_evaldiff             Polynomials/dbl2_polynomials_kernels.h:870
//   GPU_cmplx2vectorized_poly_evaldiff   Polynomials/dbl2_polynomials_kernels.h:960
// and, compiled with -DSHIM_POLY4, their quad double twins GPU_dbl4_*,
// GPU_cmplx4_* and GPU_cmplx4vectorized_poly_evaldiff
// (Polynomials/dbl4_polynomials_kernels.h:1173, :1254, :1397).
//
// TEST INFRASTRUCTURE: the recipe of oracle/Makefile (target `shim`) compiles
// this file against the reference's own header, so that any difference in
// the signatures fails to compile, and links it, in place of the
// reference's dbl2_polynomials_kernels.cu, with the reference's unchanged
// test program Polynomials/test_dbl2_polynomials.cpp and its host sources
// (read in place, output into oracle/_ref).  The reference's own tester then
// compares this library's results with its CPU code.  The same file is the
// binding a maintainer would add to PHCpack in place of its own kernels.
//
// The reference's per-limb arrays (hi, lo; re, im) become the library's
// limb-interleaved numbers; the polynomial is polynomial 0 of a one-system
// batch whose other polynomials are empty; the job lists of the reference's
// layered launches are not needed (one fused launch) and are ignored, and
// the convolution and addition times are reported together as the
// convolution time.
#include <chrono>
#include <cstdio>
#include <vector>
#if defined(SHIM_POLY4)
#include "dbl4_polynomials_kernels.h"
#else
#include "dbl2_polynomials_kernels.h"
#endif
#include "phc_b200.h"

namespace {

struct Supports {
  int maxvar = 1;
  std::vector<int> mon_off, nvr, idx, exps;
};

Supports supports(int dim, int nbr, const int *nvr, int *const *idx) {
  Supports s;
  for (int m = 0; m < nbr; ++m) s.maxvar = nvr[m] > s.maxvar ? nvr[m] : s.maxvar;
  s.mon_off.assign(dim + 1, nbr);
  s.mon_off[0] = 0;
  const int nm = nbr > 0 ? nbr : 1;
  s.nvr.assign(nm, 0);
  s.idx.assign((size_t)nm * s.maxvar, 0);
  s.exps.assign((size_t)nm * s.maxvar, 0);
  for (int m = 0; m < nbr; ++m) {
    s.nvr[m] = nvr[m];
    for (int j = 0; j < nvr[m]; ++j) {
      s.idx[(size_t)m * s.maxvar + j] = idx[m][j];
      s.exps[(size_t)m * s.maxvar + j] = 1;  // the reference's monomials are products of distinct variables
    }
  }
  return s;
}

// limb-interleaved copies: number k of a series gets W doubles
void put(std::vector<double> &dst, size_t at, int n1, int W, const double *const *parts) {
  for (int k = 0; k < n1; ++k)
    for (int l = 0; l < W; ++l) dst[at + (size_t)k * W + l] = parts[l][k];
}

void get(const std::vector<double> &src, size_t at, int n1, int W, double *const *parts) {
  for (int k = 0; k < n1; ++k)
    for (int l = 0; l < W; ++l) parts[l][k] = src[at + (size_t)k * W + l];
}

// Evaluate and differentiate; pl[q][l] are the limb arrays of quantity q
// (constant, coefficients, inputs, outputs) in the order of the limbs.
void evaldiff(int prec, int cplx, int dim, int nbr, int deg, const int *nvr, int *const *idx, double *const *cst,
              double **const *cff, double **const *input, double **const *output, double *cnvlapms,
              double *addlapms, double *elapsedms, double *walltimesec, const char *name) {
  const int W = prec * (cplx ? 2 : 1), n1 = deg + 1;
  const Supports s = supports(dim, nbr, nvr, idx);
  std::vector<double> c((size_t)dim * n1 * W, 0.0), f((size_t)(nbr > 0 ? nbr : 1) * n1 * W, 0.0);
  std::vector<double> x((size_t)dim * n1 * W), out((size_t)dim * (dim + 1) * n1 * W, 0.0);
  put(c, 0, n1, W, cst);
  for (int m = 0; m < nbr; ++m) {
    const double *pm[8];
    for (int l = 0; l < W; ++l) pm[l] = cff[l][m];
    put(f, (size_t)m * n1 * W, n1, W, pm);
  }
  for (int v = 0; v < dim; ++v) {
    const double *pv[8];
    for (int l = 0; l < W; ++l) pv[l] = input[l][v];
    put(x, (size_t)v * n1 * W, n1, W, pv);
  }
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = phc_system_evaldiff_host(prec, cplx, 1, dim, deg, s.maxvar, s.mon_off.data(), s.nvr.data(),
                                          s.idx.data(), s.exps.data(), c.data(), f.data(), x.data(), out.data(),
                                          nullptr);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) std::fprintf(stderr, "%s: %s\n", name, phc_last_error());
  for (int r = 0; r <= dim; ++r) {
    double *pr[8];
    for (int l = 0; l < W; ++l) pr[l] = output[l][r];
    get(out, (size_t)r * n1 * W, n1, W, pr);
  }
  *cnvlapms = secs * 1e3;
  *addlapms = 0.0;
  *elapsedms = secs * 1e3;
  *walltimesec = secs;
}

}  // namespace

#if !defined(SHIM_POLY4)

void GPU_dbl2_poly_evaldiff(int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *csthi, double *cstlo,
                            double **cffhi, double **cfflo, double **inputhi, double **inputlo, double **outputhi,
                            double **outputlo, ConvolutionJobs cnvjobs, AdditionJobs addjobs, double *cnvlapms,
                            double *addlapms, double *elapsedms, double *walltimesec, int vrblvl) {
  (void)BS; (void)cnvjobs; (void)addjobs; (void)vrblvl;
  double *cst[2] = {csthi, cstlo};
  double **cff[2] = {cffhi, cfflo}, **in[2] = {inputhi, inputlo}, **out[2] = {outputhi, outputlo};
  evaldiff(2, 0, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_dbl2_poly_evaldiff");
}

void GPU_cmplx2_poly_evaldiff(int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *cstrehi,
                              double *cstrelo, double *cstimhi, double *cstimlo, double **cffrehi, double **cffrelo,
                              double **cffimhi, double **cffimlo, double **inputrehi, double **inputrelo,
                              double **inputimhi, double **inputimlo, double **outputrehi, double **outputrelo,
                              double **outputimhi, double **outputimlo, ConvolutionJobs cnvjobs,
                              AdditionJobs addjobs, double *cnvlapms, double *addlapms, double *elapsedms,
                              double *walltimesec, int vrblvl) {
  (void)BS; (void)cnvjobs; (void)addjobs; (void)vrblvl;
  double *cst[4] = {cstrehi, cstrelo, cstimhi, cstimlo};
  double **cff[4] = {cffrehi, cffrelo, cffimhi, cffimlo};
  double **in[4] = {inputrehi, inputrelo, inputimhi, inputimlo};
  double **out[4] = {outputrehi, outputrelo, outputimhi, outputimlo};
  evaldiff(2, 1, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_cmplx2_poly_evaldiff");
}

void GPU_cmplx2vectorized_poly_evaldiff(int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *cstrehi,
                                        double *cstrelo, double *cstimhi, double *cstimlo, double **cffrehi,
                                        double **cffrelo, double **cffimhi, double **cffimlo, double **inputrehi,
                                        double **inputrelo, double **inputimhi, double **inputimlo,
                                        double **outputrehi, double **outputrelo, double **outputimhi,
                                        double **outputimlo, ComplexConvolutionJobs cnvjobs,
                                        ComplexIncrementJobs incjobs, ComplexAdditionJobs addjobs, double *cnvlapms,
                                        double *addlapms, double *elapsedms, double *walltimesec, int vrblvl) {
  (void)BS; (void)cnvjobs; (void)incjobs; (void)addjobs; (void)vrblvl;
  double *cst[4] = {cstrehi, cstrelo, cstimhi, cstimlo};
  double **cff[4] = {cffrehi, cffrelo, cffimhi, cffimlo};
  double **in[4] = {inputrehi, inputrelo, inputimhi, inputimlo};
  double **out[4] = {outputrehi, outputrelo, outputimhi, outputimlo};
  evaldiff(2, 1, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_cmplx2vectorized_poly_evaldiff");
}

#else  // quad double: Polynomials/dbl4_polynomials_kernels.h:1173, :1254, :1397

void GPU_dbl4_poly_evaldiff(int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *csthihi,
                            double *cstlohi, double *csthilo, double *cstlolo, double **cffhihi, double **cfflohi,
                            double **cffhilo, double **cfflolo, double **inputhihi, double **inputlohi,
                            double **inputhilo, double **inputlolo, double **outputhihi, double **outputlohi,
                            double **outputhilo, double **outputlolo, ConvolutionJobs cnvjobs, AdditionJobs addjobs,
                            double *cnvlapms, double *addlapms, double *elapsedms, double *walltimesec,
                            int vrblvl) {
  (void)BS; (void)cnvjobs; (void)addjobs; (void)vrblvl;
  double *cst[4] = {csthihi, cstlohi, csthilo, cstlolo};
  double **cff[4] = {cffhihi, cfflohi, cffhilo, cfflolo};
  double **in[4] = {inputhihi, inputlohi, inputhilo, inputlolo};
  double **out[4] = {outputhihi, outputlohi, outputhilo, outputlolo};
  evaldiff(4, 0, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_dbl4_poly_evaldiff");
}

void GPU_cmplx4_poly_evaldiff(
    int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *cstrehihi, double *cstrelohi,
    double *cstrehilo, double *cstrelolo, double *cstimhihi, double *cstimlohi, double *cstimhilo,
    double *cstimlolo, double **cffrehihi, double **cffrelohi, double **cffrehilo, double **cffrelolo,
    double **cffimhihi, double **cffimlohi, double **cffimhilo, double **cffimlolo, double **inputrehihi,
    double **inputrelohi, double **inputrehilo, double **inputrelolo, double **inputimhihi, double **inputimlohi,
    double **inputimhilo, double **inputimlolo, double **outputrehihi, double **outputrelohi,
    double **outputrehilo, double **outputrelolo, double **outputimhihi, double **outputimlohi,
    double **outputimhilo, double **outputimlolo, ConvolutionJobs cnvjobs, AdditionJobs addjobs, double *cnvlapms,
    double *addlapms, double *elapsedms, double *walltimesec, int vrblvl) {
  (void)BS; (void)cnvjobs; (void)addjobs; (void)vrblvl;
  double *cst[8] = {cstrehihi, cstrelohi, cstrehilo, cstrelolo, cstimhihi, cstimlohi, cstimhilo, cstimlolo};
  double **cff[8] = {cffrehihi, cffrelohi, cffrehilo, cffrelolo, cffimhihi, cffimlohi, cffimhilo, cffimlolo};
  double **in[8] = {inputrehihi, inputrelohi, inputrehilo, inputrelolo,
                    inputimhihi, inputimlohi, inputimhilo, inputimlolo};
  double **out[8] = {outputrehihi, outputrelohi, outputrehilo, outputrelolo,
                     outputimhihi, outputimlohi, outputimhilo, outputimlolo};
  evaldiff(4, 1, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_cmplx4_poly_evaldiff");
}

void GPU_cmplx4vectorized_poly_evaldiff(
    int BS, int dim, int nbr, int deg, int *nvr, int **idx, double *cstrehihi, double *cstrelohi,
    double *cstrehilo, double *cstrelolo, double *cstimhihi, double *cstimlohi, double *cstimhilo,
    double *cstimlolo, double **cffrehihi, double **cffrelohi, double **cffrehilo, double **cffrelolo,
    double **cffimhihi, double **cffimlohi, double **cffimhilo, double **cffimlolo, double **inputrehihi,
    double **inputrelohi, double **inputrehilo, double **inputrelolo, double **inputimhihi, double **inputimlohi,
    double **inputimhilo, double **inputimlolo, double **outputrehihi, double **outputrelohi,
    double **outputrehilo, double **outputrelolo, double **outputimhihi, double **outputimlohi,
    double **outputimhilo, double **outputimlolo, ComplexConvolutionJobs cnvjobs, ComplexIncrementJobs incjobs,
    ComplexAdditionJobs addjobs, double *cnvlapms, double *addlapms, double *elapsedms, double *walltimesec,
    int vrblvl) {
  (void)BS; (void)cnvjobs; (void)incjobs; (void)addjobs; (void)vrblvl;
  double *cst[8] = {cstrehihi, cstrelohi, cstrehilo, cstrelolo, cstimhihi, cstimlohi, cstimhilo, cstimlolo};
  double **cff[8] = {cffrehihi, cffrelohi, cffrehilo, cffrelolo, cffimhihi, cffimlohi, cffimhilo, cffimlolo};
  double **in[8] = {inputrehihi, inputrelohi, inputrehilo, inputrelolo,
                    inputimhihi, inputimlohi, inputimhilo, inputimlolo};
  double **out[8] = {outputrehihi, outputrelohi, outputrehilo, outputrelolo,
                     outputimhihi, outputimlohi, outputimhilo, outputimlolo};
  evaldiff(4, 1, dim, nbr, deg, nvr, idx, cst, cff, in, out, cnvlapms, addlapms, elapsedms, walltimesec,
           "GPU_cmplx4vectorized_poly_evaldiff");
}

#endif
