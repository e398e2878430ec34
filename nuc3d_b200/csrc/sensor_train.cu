// sensor_train.cu -- training of the face smoothness sensor (19 -> 32 -> 32 -> 1 MLP,
// ReLU, one logit) on the GPU: forward, loss and backward, and Adam.
//
// Parameters, FP32, in this order (kSensorParams floats):
//   W1 [32][19], b1 [32], W2 [32][32], b2 [32], W3 [32], b3 [1]
// The forward pass rounds the features, the weights and the hidden activations to BF16
// (round to nearest even), as the tensor-core inference in the sweep does; gradients pass
// those roundings unchanged (straight through) and accumulate in FP32.
// Loss: binary cross entropy on the logit, positives weighted by pos_weight, averaged
// over the n samples of the call.  No counterpart in the reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "nuc3d_gpu.h"

namespace {

constexpr int IN = 19, H = 32;
constexpr int OW1 = 0, OB1 = OW1 + H * IN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H,
              OB3 = OW3 + H, NPAR = OB3 + 1;
static_assert(NPAR == NUC3D_SENSOR_PARAMS, "parameter layout");
constexpr int TS = 64;  // samples per CTA tile

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float softplus(float z) {
  return z > 0.0f ? z + log1pf(expf(-z)) : log1pf(expf(z));
}

// One tile of TS samples: activations in shared memory, weight gradients summed over the
// tile and added to grad; the tile's loss is added to *loss.
__global__ void __launch_bounds__(256)
mlp_loss_grad_kernel(const float *__restrict__ prm, const float *__restrict__ x,
                     const unsigned char *__restrict__ y, int n, float pos_weight, float inv_n,
                     float *__restrict__ grad, float *__restrict__ loss, float *__restrict__ logits) {
  __shared__ float sW[NPAR];
  __shared__ float sx[TS][IN + 1], sh1[TS][H + 1], sh2[TS][H + 1], sd1[TS][H + 1], sd2[TS][H + 1];
  __shared__ float sz[TS], sdz[TS];
  const int s0 = blockIdx.x * TS;
  for (int i = threadIdx.x; i < NPAR; i += blockDim.x) sW[i] = bf(prm[i]);
  for (int i = threadIdx.x; i < TS * IN; i += blockDim.x) {
    const int s = i / IN, k = i % IN;
    sx[s][k] = (s0 + s < n) ? bf(x[(long long)(s0 + s) * IN + k]) : 0.0f;
  }
  __syncthreads();
  // layer 1
  for (int i = threadIdx.x; i < TS * H; i += blockDim.x) {
    const int s = i / H, j = i % H;
    float a = sW[OB1 + j];
    for (int k = 0; k < IN; ++k) a += sW[OW1 + j * IN + k] * sx[s][k];
    sh1[s][j] = bf(fmaxf(a, 0.0f));
  }
  __syncthreads();
  // layer 2
  for (int i = threadIdx.x; i < TS * H; i += blockDim.x) {
    const int s = i / H, j = i % H;
    float a = sW[OB2 + j];
    for (int k = 0; k < H; ++k) a += sW[OW2 + j * H + k] * sh1[s][k];
    sh2[s][j] = bf(fmaxf(a, 0.0f));
  }
  __syncthreads();
  // logit, loss and d(loss)/d(logit)
  if (threadIdx.x < TS) {
    const int s = threadIdx.x;
    float z = sW[OB3];
    for (int k = 0; k < H; ++k) z += sW[OW3 + k] * sh2[s][k];
    sz[s] = z;
    float dz = 0.0f, l = 0.0f;
    if (s0 + s < n) {
      const float t = y[s0 + s] ? 1.0f : 0.0f;
      const float sig = 1.0f / (1.0f + expf(-z));
      l = (pos_weight * t * softplus(-z) + (1.0f - t) * softplus(z)) * inv_n;
      dz = ((1.0f - t) * sig - pos_weight * t * (1.0f - sig)) * inv_n;
      if (logits) logits[s0 + s] = z;
    }
    sdz[s] = dz;
    // tile loss: warp sums, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((s & 31) == 0) atomicAdd(loss, l);
  }
  __syncthreads();
  // back through layer 3 and the ReLU of layer 2
  for (int i = threadIdx.x; i < TS * H; i += blockDim.x) {
    const int s = i / H, j = i % H;
    sd2[s][j] = sh2[s][j] > 0.0f ? sdz[s] * sW[OW3 + j] : 0.0f;
  }
  __syncthreads();
  // back through layer 2 and the ReLU of layer 1
  for (int i = threadIdx.x; i < TS * H; i += blockDim.x) {
    const int s = i / H, k = i % H;
    float a = 0.0f;
    for (int j = 0; j < H; ++j) a += sd2[s][j] * sW[OW2 + j * H + k];
    sd1[s][k] = sh1[s][k] > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  // parameter gradients: sums over the tile's samples
  for (int p = threadIdx.x; p < NPAR; p += blockDim.x) {
    float g = 0.0f;
    if (p < OB1) {
      const int j = p / IN, k = p % IN;
      for (int s = 0; s < TS; ++s) g += sd1[s][j] * sx[s][k];
    } else if (p < OW2) {
      for (int s = 0; s < TS; ++s) g += sd1[s][p - OB1];
    } else if (p < OB2) {
      const int j = (p - OW2) / H, k = (p - OW2) % H;
      for (int s = 0; s < TS; ++s) g += sd2[s][j] * sh1[s][k];
    } else if (p < OW3) {
      for (int s = 0; s < TS; ++s) g += sd2[s][p - OB2];
    } else if (p < OB3) {
      for (int s = 0; s < TS; ++s) g += sdz[s] * sh2[s][p - OW3];
    } else {
      for (int s = 0; s < TS; ++s) g += sdz[s];
    }
    atomicAdd(grad + p, g);
  }
}

__global__ void adam_kernel(float *__restrict__ prm, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int np, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

extern "C" {

int nuc3d_sensor_loss_grad(const float *params, const float *feat, const unsigned char *label,
                           long long n, float pos_weight, float *grad, float *loss, float *logits,
                           void *stream) {
  if (!params || !feat || !label || !grad || !loss || n <= 0) return NUC3D_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(grad, 0, NPAR * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(loss, 0, sizeof(float), st);
  if (e != cudaSuccess) return NUC3D_ECUDA;
  const long long tiles = (n + TS - 1) / TS;
  if (tiles > 0x7fffffffLL) return NUC3D_EINVAL;
  mlp_loss_grad_kernel<<<(unsigned)tiles, 256, 0, st>>>(params, feat, label, (int)n, pos_weight,
                                                        1.0f / (float)n, grad, loss, logits);
  return cudaGetLastError() == cudaSuccess ? NUC3D_OK : NUC3D_ECUDA;
}

int nuc3d_sensor_adam(float *params, const float *grad, float *m, float *v, float lr, float beta1,
                      float beta2, float eps, int step, void *stream) {
  if (!params || !grad || !m || !v || step < 1) return NUC3D_EINVAL;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<(NPAR + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grad, m, v, NPAR, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? NUC3D_OK : NUC3D_ECUDA;
}

}  // extern "C"
