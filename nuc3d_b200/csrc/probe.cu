// probe.cu -- device measurements that are not part of the solver ABI
// (exported from libnuc3d_probe.so):
//   nuc3d_probe_fp64_tflops  FP64 peak, measured with a dependent-FMA microbenchmark.
//     The NUC3d path is plain FP64 (no tensor cores), so its compute roof is measured
//     here: every thread runs 8 independent DFMA chains, enough CTAs to fill all SMs
//     several times over, timed with CUDA events.
//   nuc3d_probe_qdiv         the throughput build's division next to IEEE division on
//     the same operands, for the accuracy test of the former.
//   nuc3d_probe_crpow        the energy reset's double-double pow (cr_pow), for the test
//     that pins its bits to the oracle's.
#include <cuda_runtime.h>

#define NUC3D_NS fast
#define NUC3D_FAST 1
#include "physics.cuh"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_loop(double *out, int iters, double b, double c) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == 1234.5678) out[blockIdx.x] = s;  // never true; keeps the chains alive
}

__global__ void qdiv_pairs(const double *a, const double *b, double *q_fast, double *q_ieee,
                           long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    q_fast[i] = nuc3d::fast::qdiv(a[i], b[i]);
    q_ieee[i] = a[i] / b[i];
  }
}

__global__ void crpow_pairs(const double *x, const double *y, double *r, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = nuc3d::fast::cr_pow(x[i], y[i]);
}

}  // namespace

extern "C" {

// r[i] = cr_pow(x[i], y[i]) on the device; host arrays of n doubles.  Returns 0 or a CUDA
// error code.
int nuc3d_probe_crpow(int device, const double *x, const double *y, double *r, long long n) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  double *d = nullptr;
  const size_t bytes = (size_t)n * sizeof(double);
  if ((e = cudaMalloc(&d, 3 * bytes)) != cudaSuccess) return (int)e;
  cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(d + n, y, bytes, cudaMemcpyHostToDevice);
  crpow_pairs<<<296, 256>>>(d, d + n, d + 2 * n, n);
  e = cudaMemcpy(r, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

// q_fast[i] = the throughput build's a[i] / b[i], q_ieee[i] = IEEE a[i] / b[i]; host arrays
// of n doubles.  Returns 0 or a CUDA error code.
int nuc3d_probe_qdiv(int device, const double *a, const double *b, double *q_fast, double *q_ieee,
                     long long n) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return (int)e;
  double *d = nullptr;
  const size_t bytes = (size_t)n * sizeof(double);
  if ((e = cudaMalloc(&d, 4 * bytes)) != cudaSuccess) return (int)e;
  cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(d + n, b, bytes, cudaMemcpyHostToDevice);
  qdiv_pairs<<<1184, 256>>>(d, d + n, d + 2 * n, d + 3 * n, n);
  cudaMemcpy(q_fast, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  e = cudaMemcpy(q_ieee, d + 3 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

// Returns sustained FP64 TFLOP/s (FMA = 2 flops) over `reps` launches, or a negative
// CUDA error code.
double nuc3d_probe_fp64_tflops(int device, int reps) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double *out = nullptr;
  if (cudaMalloc(&out, 1 << 20) != cudaSuccess) return -2.0;
  const int blocks = sms * 16, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dfma_loop<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0);
  for (int r = 0; r < reps; ++r) dfma_loop<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return -3.0;
  const double flops = 2.0 * kChains * (double)iters * threads * blocks * reps;
  return flops / (ms * 1e-3) / 1e12;
}

}  // extern "C"
