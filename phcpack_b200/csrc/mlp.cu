// mlp.cu -- training and batched inference of the learned step proposer
// (24 -> 128 -> 128 -> 1, ReLU), hand-written.
//
// Parameters live in FP32 (master copy, Adam moments); every training step
// first rounds them to the BF16 model buffer the tracker reads (mlp.cuh),
// and the forward and backward passes use exactly those BF16 weights with
// FP32 accumulation, so the gradients are those of the deployed network.
// One CTA of 128 threads takes a chunk of samples; thread j owns hidden
// unit j in both layers, keeps its rows of dW1 and dW2 in shared memory
// across the chunk, and adds them to the global gradient once at the end.
#include <cuda_bf16.h>
#include "common.cuh"
#include "mlp.cuh"
#include "../../include/phc_b200.h"

namespace phc {

// FP32 parameter vector layout (also the gradient and Adam moment layout):
//   W1[128][24], b1[128], W2[128][128], b2[128], W3[128], b3[1]
static const long kP_W1 = 0, kP_b1 = kP_W1 + 128 * 24, kP_W2 = kP_b1 + 128, kP_b2 = kP_W2 + 128 * 128,
                  kP_W3 = kP_b2 + 128, kP_b3 = kP_W3 + 128, kP_total = kP_b3 + 1;

// master FP32 parameters + normalisation -> the BF16 model buffer
__global__ void k_mlp_pack(const float *__restrict__ P, const float *__restrict__ mean,
                           const float *__restrict__ inv_std, unsigned char *__restrict__ model) {
  float *f = reinterpret_cast<float *>(model);
  __nv_bfloat16 *h = reinterpret_cast<__nv_bfloat16 *>(f + mlp_float_count());
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 128 * 24 + 128 * 128 + 128 + 312;
       i += gridDim.x * blockDim.x) {
    if (i < 24) {
      f[i] = mean[i];
      f[24 + i] = inv_std[i];
    } else if (i < 24 + 128) {
      f[48 + (i - 24)] = P[kP_b1 + (i - 24)];
    } else if (i < 24 + 256) {
      f[176 + (i - 152)] = P[kP_b2 + (i - 152)];
    } else if (i < 24 + 256 + 8) {
      const int q = i - 280;
      f[304 + q] = (q == 0) ? P[kP_b3] : 0.0f;
    } else if (i >= 312) {
      const int q = i - 312;
      if (q < 128 * 24)
        h[q] = __float2bfloat16_rn(P[kP_W1 + q]);
      else if (q < 128 * 24 + 128 * 128)
        h[q] = __float2bfloat16_rn(P[kP_W2 + (q - 128 * 24)]);
      else
        h[q] = __float2bfloat16_rn(P[kP_W3 + (q - 128 * 24 - 128 * 128)]);
    }
  }
}

// Batched inference: out[b] = network(X[b]) (log step ratio, unclipped)
__global__ void __launch_bounds__(128) k_mlp_forward(const unsigned char *__restrict__ model, int nb,
                                                     const float *__restrict__ X, float *__restrict__ out) {
  __shared__ float h1[128], red[4];
  __shared__ float xs[24];
  const MlpView M = mlp_view(model);
  const int j = threadIdx.x;
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {
    if (j < 24) xs[j] = (X[(long)b * 24 + j] - M.mean[j]) * M.inv_std[j];
    __syncthreads();
    float a = M.b1[j];
    for (int i = 0; i < 24; ++i) a = fmaf(__bfloat162float(M.W1[j * 24 + i]), xs[i], a);
    h1[j] = fmaxf(a, 0.0f);
    __syncthreads();
    a = M.b2[j];
    for (int i = 0; i < 128; ++i) a = fmaf(__bfloat162float(M.W2[j * 128 + i]), h1[i], a);
    float c = __bfloat162float(M.W3[j]) * fmaxf(a, 0.0f);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((j & 31) == 0) red[j >> 5] = c;
    __syncthreads();
    if (j == 0) out[b] = M.b3[0] + red[0] + red[1] + red[2] + red[3];
    __syncthreads();
  }
}

// Forward + backward of the mean squared error over nb samples (X, y),
// gradients added into G (FP32, kP_total), loss into *loss.
__global__ void __launch_bounds__(128) k_mlp_grad(const unsigned char *__restrict__ model, int nb,
                                                  const float *__restrict__ X, const float *__restrict__ y,
                                                  float *__restrict__ G, float *__restrict__ loss) {
  extern __shared__ float smf[];
  float *dW2 = smf;                 // 128 x 128
  float *dW1 = dW2 + 128 * 128;     // 128 x 24
  float *h1 = dW1 + 128 * 24;       // 128
  float *g2 = h1 + 128;             // 128
  float *xs = g2 + 128;             // 24 (+8)
  float *red = xs + 32;             // 8
  const MlpView M = mlp_view(model);
  const int j = threadIdx.x;
  for (int i = j; i < 128 * 128; i += 128) dW2[i] = 0.0f;
  for (int i = j; i < 128 * 24; i += 128) dW1[i] = 0.0f;
  float db1 = 0.0f, db2 = 0.0f, dW3 = 0.0f, db3 = 0.0f, lsum = 0.0f;
  const float w3 = __bfloat162float(M.W3[j]);
  __syncthreads();
  const int chunk = (nb + gridDim.x - 1) / gridDim.x;
  const int b0 = blockIdx.x * chunk, b1 = min(nb, b0 + chunk);
  for (int b = b0; b < b1; ++b) {
    if (j < 24) xs[j] = (X[(long)b * 24 + j] - M.mean[j]) * M.inv_std[j];
    __syncthreads();
    float a = M.b1[j];
    for (int i = 0; i < 24; ++i) a = fmaf(__bfloat162float(M.W1[j * 24 + i]), xs[i], a);
    const float z1 = a;
    h1[j] = fmaxf(z1, 0.0f);
    __syncthreads();
    a = M.b2[j];
    for (int i = 0; i < 128; ++i) a = fmaf(__bfloat162float(M.W2[j * 128 + i]), h1[i], a);
    const float z2 = a, hj2 = fmaxf(z2, 0.0f);
    float c = w3 * hj2;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((j & 31) == 0) red[j >> 5] = c;
    __syncthreads();
    const float out = M.b3[0] + red[0] + red[1] + red[2] + red[3];
    const float g = 2.0f * (out - y[b]) / (float)nb;  // d(mean squared error)/d out
    if (j == 0) {
      lsum += (out - y[b]) * (out - y[b]);
      db3 += g;
    }
    dW3 += g * hj2;
    const float gz2 = (z2 > 0.0f) ? g * w3 : 0.0f;
    g2[j] = gz2;
    db2 += gz2;
    for (int i = 0; i < 128; ++i) dW2[j * 128 + i] += gz2 * h1[i];
    __syncthreads();
    // back through W2 to hidden layer 1: column j of W2
    float gh1 = 0.0f;
    for (int i = 0; i < 128; ++i) gh1 = fmaf(__bfloat162float(M.W2[i * 128 + j]), g2[i], gh1);
    const float gz1 = (z1 > 0.0f) ? gh1 : 0.0f;
    db1 += gz1;
    for (int i = 0; i < 24; ++i) dW1[j * 24 + i] += gz1 * xs[i];
    __syncthreads();
  }
  for (int i = j; i < 128 * 128; i += 128) atomicAdd(&G[kP_W2 + i], dW2[i]);
  for (int i = j; i < 128 * 24; i += 128) atomicAdd(&G[kP_W1 + i], dW1[i]);
  atomicAdd(&G[kP_b1 + j], db1);
  atomicAdd(&G[kP_b2 + j], db2);
  atomicAdd(&G[kP_W3 + j], dW3);
  if (j == 0) {
    atomicAdd(&G[kP_b3], db3);
    atomicAdd(loss, lsum / (float)nb);
  }
}

// Adam on the FP32 master parameters (Kingma and Ba), gradients cleared.
__global__ void k_mlp_adam(float *__restrict__ P, float *__restrict__ G, float *__restrict__ m, float *__restrict__ v,
                           float lr, float beta1, float beta2, float eps, int t) {
  const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < kP_total; i += (long)gridDim.x * blockDim.x) {
    const float g = G[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * g;
    const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    G[i] = 0.0f;
  }
}

}  // namespace phc

using namespace phc;

extern "C" {

long long phc_mlp_param_count(void) { return kP_total; }

int phc_mlp_pack(const float *params, const float *mean, const float *inv_std, void *model, void *stream) {
  PHC_REQUIRE(params && mean && inv_std && model, "mlp_pack: null pointer");
  k_mlp_pack<<<64, 256, 0, (cudaStream_t)stream>>>(params, mean, inv_std, (unsigned char *)model);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

int phc_mlp_forward(const void *model, int nb, const float *X, float *out, void *stream) {
  PHC_REQUIRE(nb >= 0 && model && X && out, "mlp_forward: bad arguments");
  if (nb == 0) return PHC_OK;
  const int grid = nb < 148 * 8 ? nb : 148 * 8;
  k_mlp_forward<<<grid, 128, 0, (cudaStream_t)stream>>>((const unsigned char *)model, nb, X, out);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

int phc_mlp_grad(const void *model, int nb, const float *X, const float *y, float *grad, float *loss, void *stream) {
  PHC_REQUIRE(nb >= 1 && model && X && y && grad && loss, "mlp_grad: bad arguments");
  const long smem = (128L * 128 + 128 * 24 + 128 + 128 + 32 + 8) * sizeof(float);
  PHC_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int grid = (nb + 63) / 64;
  if (grid > 148) grid = 148;
  k_mlp_grad<<<grid, 128, smem, (cudaStream_t)stream>>>((const unsigned char *)model, nb, X, y, grad, loss);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

int phc_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                 int t, void *stream) {
  PHC_REQUIRE(params && grad && m && v && t >= 1, "mlp_adam: bad arguments");
  k_mlp_adam<<<40, 512, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, beta1, beta2, eps, t);
  PHC_CHECK_LAUNCH();
  return PHC_OK;
}

}  // extern "C"
