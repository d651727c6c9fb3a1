// tracker_fp64.cu -- the launches of the precision-split tracker (double
// predictor and corrector Jacobian, double-double corrector residuals) with
// double-, quad- or octo-double refinement; the kernel is in
// tracker_kernel.cuh.
#include "tracker_kernel.cuh"

namespace phc {

int track_fp64(const TrackDev &S, const TrackParDev &P, int nmono_max, int npaths, const int *path_sys,
               const double *x0, int rmode, const void *model, double *xend, int *info, double *dinfo, float *log,
               int log_cap, int *log_count, int *queue, int one_per_launch, cudaStream_t st) {
  typedef md::num<double, true> Z1;
  typedef md::num<md::dd, true> Z2;
  typedef md::num<md::qd, true> Z4;
  typedef md::num<md::od, true> Z8;
  if (rmode == 8)
    return track_launch<Z1, Z2, Z8>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                    log_count, queue, one_per_launch, st);
  if (rmode == 2)
    return track_launch<Z1, Z2, Z2>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                    log_count, queue, one_per_launch, st);
  return track_launch<Z1, Z2, Z4>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                  log_count, queue, one_per_launch, st);
}

}  // namespace phc
