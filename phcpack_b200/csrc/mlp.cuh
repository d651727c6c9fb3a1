// mlp.cuh -- the learned step-size proposer: features of a predictor step
// and the CTA-wide BF16 inference used inside the tracker.
//
// Model: 24 -> 128 -> 128 -> 1, ReLU hidden layers, BF16 weights, FP32
// biases, accumulation and feature normalisation.  It predicts the log of
// the ratio of an accepted step to the plain pole step; the proposal is
// pole_step * exp(out), clipped to [e^-3, e^3] times the pole step.
#pragma once
#include <cuda_bf16.h>

namespace phc {

static const int kMlpIn = 24, kMlpH = 128;

// Byte layout of a model buffer (16-byte aligned pieces):
//   float mean[24], inv_std[24], b1[128], b2[128], b3[4], pad[4]   (1248 B)
//   bf16  W1[128][24], W2[128][128], W3[128]
struct MlpView {
  const float *mean, *inv_std, *b1, *b2, *b3;
  const __nv_bfloat16 *W1, *W2, *W3;
};
__host__ __device__ inline long mlp_float_count() { return 24 + 24 + 128 + 128 + 4 + 4; }
__host__ __device__ inline long mlp_bf16_count() { return 128L * 24 + 128L * 128 + 128; }
__host__ __device__ inline long mlp_model_bytes() { return mlp_float_count() * 4 + mlp_bf16_count() * 2; }

__host__ __device__ inline MlpView mlp_view(const void *base) {
  MlpView v;
  const float *f = reinterpret_cast<const float *>(base);
  v.mean = f;
  v.inv_std = f + 24;
  v.b1 = f + 48;
  v.b2 = f + 176;
  v.b3 = f + 304;
  const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(f + mlp_float_count());
  v.W1 = h;
  v.W2 = h + 128 * 24;
  v.W3 = h + 128 * 24 + 128 * 128;
  return v;
}

// Features of one predictor step: from the magnitudes mag[i*(K+1)+k] of the
// series coefficients of the n components, the current t and the pole step.
//   f[0..7]   log of the root-test radius (max_i |c_ik|)^(-1/k), k = 1..8
//   f[8..15]  log of the ratio radius min_i |c_i,k-1| / |c_ik|, k = 1..8
//   f[16..19] log pole step, t, log(1 - t), log n
//   f[20..23] log max_i |c_ik| for k = 0..3
// Orders beyond K repeat the last one.  Every thread of the CTA calls it
// with its number tid; threads 0..12 compute a share each.
__device__ __forceinline__ void track_features(int tid, int n, int K, double t, double pole_step, const double *mag,
                                      float *f) {
  const double tiny = 1e-300;
  if (tid < 8) {
    const int q = tid;
    const int k = (q + 1 <= K) ? q + 1 : K;
    double mx = 0.0, rmin = 1e300;
    #pragma unroll 1
    for (int i = 0; i < n; ++i) {
      const double a = mag[i * (K + 1) + k], b = mag[i * (K + 1) + k - 1];
      mx = fmax(mx, a);
      if (a > 0.0) rmin = fmin(rmin, b / a);
    }
    double rt = (mx > 0.0) ? -log(mx + tiny) / k : 30.0;
    double rr = (rmin < 1e299) ? log(rmin + tiny) : 30.0;
    f[q] = (float)fmin(fmax(rt, -30.0), 30.0);
    f[8 + q] = (float)fmin(fmax(rr, -30.0), 30.0);
  } else if (tid < 12) {
    const int q = tid - 8;
    const int k = q <= K ? q : K;
    double mx = 0.0;
    #pragma unroll 1
    for (int i = 0; i < n; ++i) mx = fmax(mx, mag[i * (K + 1) + k]);
    f[20 + q] = (float)fmin(fmax(log(mx + tiny), -60.0), 60.0);
  } else if (tid == 12) {
    f[16] = (float)log(pole_step + tiny);
    f[17] = (float)t;
    f[18] = (float)log(fmax(1.0 - t, 1e-16));
    f[19] = (float)log((double)n);
  }
}

// CTA-wide forward pass for one sample (every thread of the block calls
// it; blockDim.x >= 128).  hbuf: shared scratch of 2*128 floats + 8.
// Returns log(step / pole_step) to every thread.
__device__ __forceinline__ float mlp_forward_cta(const void *model, const float *feat, float *hbuf) {
  const MlpView M = mlp_view(model);
  const int j = threadIdx.x;
  float *h1 = hbuf, *h2 = hbuf + kMlpH, *red = hbuf + 2 * kMlpH;
  // rows of W1 and W2 read 8 weights (16 bytes) at a time; the sums keep
  // the order i = 0, 1, ... (the model buffer is 16-byte aligned)
  if (j < kMlpH) {
    float a = M.b1[j];
    const uint4 *w = reinterpret_cast<const uint4 *>(M.W1 + j * kMlpIn);
    #pragma unroll 1
    for (int c = 0; c < kMlpIn / 8; ++c) {
      const uint4 u = __ldg(w + c);
      const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = 8 * c + r;
        a = fmaf(__bfloat162float(e[r]), (feat[i] - M.mean[i]) * M.inv_std[i], a);
      }
    }
    h1[j] = fmaxf(a, 0.0f);
  }
  __syncthreads();
  float contrib = 0.0f;
  if (j < kMlpH) {
    float a = M.b2[j];
    const uint4 *w = reinterpret_cast<const uint4 *>(M.W2 + j * kMlpH);
    #pragma unroll 1
    for (int c = 0; c < kMlpH / 8; ++c) {
      const uint4 u = __ldg(w + c);
      const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
      for (int r = 0; r < 8; ++r) a = fmaf(__bfloat162float(e[r]), h1[8 * c + r], a);
    }
    h2[j] = fmaxf(a, 0.0f);
    contrib = __bfloat162float(M.W3[j]) * h2[j];
  }
  // sum over the 4 warps of the first 128 threads
  #pragma unroll 1
  for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
  if ((j & 31) == 0 && j < kMlpH) red[j >> 5] = contrib;
  __syncthreads();
  float out = M.b3[0] + red[0] + red[1] + red[2] + red[3];
  __syncthreads();
  return fminf(fmaxf(out, -3.0f), 3.0f);
}

}  // namespace phc
