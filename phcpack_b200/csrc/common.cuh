// common.cuh -- shared host-side helpers of the CUDA library.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>

namespace phc {

// Status codes of the C ABI: 0 ok, > 0 count of failed items (paths that
// did not converge and similar), < 0 errors.
enum {
  PHC_OK = 0,
  PHC_ERR_ARG = -1,       // bad size, precision or pointer
  PHC_ERR_CUDA = -2,      // a CUDA call failed
  PHC_ERR_LIMIT = -3,     // size beyond a documented kernel limit
  PHC_ERR_TIMEOUT = -4,   // a bounded device-side wait gave up
};

void set_error(const char *fmt, ...);
const char *get_error();

#define PHC_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      ::phc::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,           \
                       cudaGetErrorString(e_));                             \
      return ::phc::PHC_ERR_CUDA;                                           \
    }                                                                       \
  } while (0)

#define PHC_CHECK_LAUNCH()                                                  \
  do {                                                                      \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess) {                                                \
      ::phc::set_error("%s:%d launch: %s", __FILE__, __LINE__,              \
                       cudaGetErrorString(e_));                             \
      return ::phc::PHC_ERR_CUDA;                                           \
    }                                                                       \
  } while (0)

#define PHC_REQUIRE(cond, ...)                                              \
  do {                                                                      \
    if (!(cond)) {                                                          \
      ::phc::set_error(__VA_ARGS__);                                        \
      return ::phc::PHC_ERR_ARG;                                            \
    }                                                                       \
  } while (0)

inline int width_of(int prec, int cplx) { return prec * (cplx ? 2 : 1); }
// Launch-shape knobs set by the autotuner (phc_tune_set); 0 leaves the
// built-in rule.
enum { kTuneEvalWarps = 0, kTuneTrackVariant = 1, kTuneTrackPerSM = 2, kTuneDenseStage = 3, kTuneKnobs = 4 };
int tune_get(int knob);
inline bool prec_ok(int prec) { return prec == 1 || prec == 2 || prec == 4; }

}  // namespace phc
