// Workload statistics of a plan and an FP64 throughput probe, used by the benchmark to
// express kernel times as fractions of a roofline.
#include <cuda_runtime.h>

#include <cmath>

#include "executor.h"

namespace hankel {

// out[0]  sum over asymptotic boxes of sources (nj)
// out[1]  sum over asymptotic boxes of targets (ni)
// out[2]  FFT cells (sum of n2; entries 2-4, 8, 9 in units of NLP-term vectors)
// out[3]  sum of nj * W (spreading taps per vector)
// out[4]  sum of ni * W (interpolation taps per vector)
// out[5]  direct-box pairs (sum of ni * nj)
// out[6]  local boxes: sum of nj
// out[7]  local boxes: sum of ni
// out[8]  FFT cells read by interpolation (sum of n2 / sigma + W)
// out[9]  FFT flops per vector (sum of 5 n2 log2 n2)
// out[10] expansion terms per column (NLP)
// out[11] local expansion terms (K_loc + 1)
// out[12] asymptotic boxes oversampled below sigma = 2
// out[13] 1 if the asymptotic boxes run in FP32 (mixed precision), else 0
// out[14] modelled worst-case error of the asymptotic boxes in FP32, per unit ||c||_1
// out[15] planning ms: grid validation and box partition
// out[16] planning ms: work lists
// out[17] planning ms: device tables and uploads
// out[18] 1 when the box partition ran on the device
// out[19] bytes of the source records (first cell, W weights, nlp factors per box source)
// out[20] bytes of the target records (first cell, weights, nlp factors per box target)
void plan_stats(const DevicePlan& D, double* out, int n) {
  double s[21] = {0};
  const double e = D.mixed_asy ? 4.0 : 8.0;  // bytes of the arithmetic type
  // Per-vector sums (entries 2-4, 8, 9) count a box with fewer expansion terms than the
  // plan's NLP in proportion (nlp / NLP), so that multiplying by NLP * B gives the work.
  for (const AsyBoxD& b : D.asyb) {
    double nj = b.j1 - b.j0 + 1, ni = b.i1 - b.i0 + 1;
    const AsyClass& K = D.classes[b.cls];
    const double f = D.NLP > 0 ? (double)b.nlp / (double)D.NLP : 1.0;
    s[0] += nj;
    s[1] += ni;
    s[2] += f * b.n2;
    s[3] += f * nj * K.W;
    s[4] += f * ni * K.W;
    s[8] += f * std::min((double)b.n2, b.n2 / K.sigma + K.W);
    s[9] += f * 5.0 * b.n2 * std::log2((double)b.n2);
    const double we = D.mixed_asy ? ((K.W + 3) & ~3) : ((K.W + 1) & ~1);  // padded target weights
    s[19] += nj * (4.0 + e * K.W + 2.0 * e * b.nlp);
    s[20] += ni * (4.0 + e * we + 2.0 * e * b.nlp);
    if (K.sigma != 2.0) s[12] += 1.0;
  }
  for (const HBox& b : D.dir_boxes) s[5] += (double)(b.i1 - b.i0 + 1) * (double)(b.j1 - b.j0 + 1);
  for (const HBox& b : D.asy_direct) s[5] += (double)(b.i1 - b.i0 + 1) * (double)(b.j1 - b.j0 + 1);
  for (const HBox& b : D.loc_boxes) {
    s[6] += b.j1 - b.j0 + 1;
    s[7] += b.i1 - b.i0 + 1;
  }
  s[10] = D.NLP;
  s[11] = D.KL1;
  s[13] = D.mixed_asy ? 1.0 : 0.0;
  s[14] = D.fp32_err;
  s[15] = D.plan_ms[0];
  s[16] = D.plan_ms[1];
  s[17] = D.plan_ms[2];
  s[18] = D.partition_on_device;
  for (int i = 0; i < n && i < 21; ++i) out[i] = s[i];
}

namespace {
__global__ void k_fp64_fma(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keeps the loop alive
}
// Packed two-lane FP32 multiply-add (fma.rn.f32x2), the instruction the single-precision
// asymptotic kernels issue.
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
  unsigned long long d;
  asm volatile("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__global__ void k_fp32_fma(float* out, int iters, float a, float b) {
  const unsigned long long pa = (unsigned long long)__float_as_uint(a) | ((unsigned long long)__float_as_uint(a) << 32);
  const unsigned long long pb = (unsigned long long)__float_as_uint(b) | ((unsigned long long)__float_as_uint(b) << 32);
  unsigned long long x[8];
#pragma unroll
  for (int q = 0; q < 8; ++q)
    x[q] = (unsigned long long)__float_as_uint((float)(threadIdx.x + q)) |
           ((unsigned long long)__float_as_uint((float)(threadIdx.x + 2 * q)) << 32);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = ffma2(x[q], pa, pb);
  }
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += __uint_as_float((unsigned)(x[q] & 0xffffffffull)) + __uint_as_float((unsigned)(x[q] >> 32));
  if (s == 12345.678f) out[0] = s;  // keeps the loop alive
}

template <class Launch>
int time_probe(Launch launch, float* ms_out) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch(64);  // warm up
  cudaEventRecord(e0);
  launch(4096);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_out = ms;
  return (cudaGetLastError() != cudaSuccess || ms <= 0.f) ? NUFHT_E_CUDA : 0;
}
}  // namespace

int fp32_peak(double* tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float* d = nullptr;
  if (cudaMalloc(&d, sizeof(float)) != cudaSuccess) return NUFHT_E_CUDA;
  const int blocks = sms * 8, threads = 256;
  float ms = 0.f;
  int rc = time_probe([&](int it) { k_fp32_fma<<<blocks, threads>>>(d, it, 0.999999f, 1e-9f); }, &ms);
  cudaFree(d);
  if (rc) return rc;
  // 8 chains x 2 lanes x 2 flops per packed FMA
  *tflops = 2.0 * 2.0 * 8.0 * 4096.0 * blocks * threads / (ms * 1e-3) / 1e12;
  return 0;
}

int fp64_peak(double* tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return NUFHT_E_CUDA;
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp64_fma<<<blocks, threads>>>(d, 64, 0.999999, 1e-9);  // warm up
  cudaEventRecord(e0);
  k_fp64_fma<<<blocks, threads>>>(d, iters, 0.999999, 1e-9);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return NUFHT_E_CUDA;
  double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return 0;
}

}  // namespace hankel
