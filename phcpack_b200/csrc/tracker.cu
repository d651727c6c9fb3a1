// tracker.cu -- the path tracker's entry (the checks and the dispatch over
// the precisions) and the launches with the double-double predictor; the
// kernel is in tracker_kernel.cuh, the double-predictor launches in
// tracker_fp64.cu.
#include "tracker_kernel.cuh"

namespace phc {

int track_fp64(const TrackDev &S, const TrackParDev &P, int nmono_max, int npaths, const int *path_sys,
               const double *x0, int rmode, const void *model, double *xend, int *info, double *dinfo, float *log,
               int log_cap, int *log_count, int *queue, int one_per_launch, cudaStream_t st);

long track_smem_bytes(int maxdim, int K, int M, int nmono_max, int maxvar, int pmode, int rmode, int gst) {
  const int Wp = 2 * pmode, Wr = 2 * rmode;
  return track_layout(maxdim, K, M, nmono_max, maxvar, Wp, Wr, gst).total * (long)sizeof(double);
}

// The checks of the modes, the dimension and the series and Pade degrees.
int track_check(const TrackParDev &P, int pmode, int rmode, int maxdim) {
  PHC_REQUIRE(pmode == 1 || pmode == 2, "track: predictor precision %d not in {1,2}", pmode);
  PHC_REQUIRE(rmode == 2 || rmode == 4 || rmode == 8, "track: refinement precision %d not in {2,4,8}", rmode);
  PHC_REQUIRE(maxdim >= 1 && maxdim <= 32, "track: dimension %d not in [1,32]", maxdim);
  PHC_REQUIRE(P.deg >= 3 && P.deg <= kTrackKmax && P.numdeg + P.dendeg == P.deg && P.dendeg <= 8 && P.nit >= 1,
              "track: need 3 <= deg = numdeg + dendeg <= %d, dendeg <= 8", kTrackKmax);
  PHC_REQUIRE(P.cbeta > 0.0 && P.cbeta < INFINITY, "track: cbeta %g is not positive", P.cbeta);
  PHC_REQUIRE(P.step_mode >= 0 && P.step_mode <= 3, "track: step_mode %d not in 0..3", P.step_mode);
  PHC_REQUIRE(!(P.step_mode & 2) || pmode == 1, "track: the QR predictor (step_mode bit 2) needs pmode 1");
  return PHC_OK;
}

int track(const TrackDev &S, const TrackParDev &P, int nmono_max, int npaths, const int *path_sys, const double *x0,
          int pmode, int rmode, const void *model, double *xend, int *info, double *dinfo, float *log, int log_cap,
          int *log_count, int *queue, int one_per_launch, cudaStream_t st) {
  const int bad = track_check(P, pmode, rmode, S.maxdim);
  if (bad) return bad;
  PHC_REQUIRE(queue != nullptr || one_per_launch, "track: the batched launch needs a queue counter");
  PHC_REQUIRE(model == nullptr || (reinterpret_cast<unsigned long long>(model) & 15) == 0, "track: the model buffer is not 16-byte aligned");
  if (npaths == 0) return PHC_OK;
  if (pmode == 1)
    return track_fp64(S, P, nmono_max, npaths, path_sys, x0, rmode, model, xend, info, dinfo, log, log_cap, log_count,
                      queue, one_per_launch, st);
  typedef md::num<md::dd, true> Z2;
  typedef md::num<md::qd, true> Z4;
  typedef md::num<md::od, true> Z8;
  if (rmode == 8)
    return track_launch<Z2, Z2, Z8>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                    log_count, queue, one_per_launch, st);
  if (rmode == 2)
    return track_launch<Z2, Z2, Z2>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                    log_count, queue, one_per_launch, st);
  return track_launch<Z2, Z2, Z4>(S, P, nmono_max, npaths, path_sys, x0, model, xend, info, dinfo, log, log_cap,
                                  log_count, queue, one_per_launch, st);
}

}  // namespace phc
