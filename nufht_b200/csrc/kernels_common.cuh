// Helpers shared by the executor's kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>

#include "executor.h"

namespace hankel {

// d += a * b for one 8 x 8 x 4 FP64 tensor-core tile (DMMA): lane q holds A[q/4][q%4],
// B[q%4][q/4] and D[q/4][2(q%4)], D[q/4][2(q%4)+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

#define NUFHT_CUDA_TRY(expr)                                                               \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess) {                                                               \
      std::fprintf(stderr, "nufht_b200: %s failed: %s\n", #expr, cudaGetErrorString(_e));  \
      return NUFHT_E_CUDA;                                                                 \
    }                                                                                      \
  } while (0)

#define NUFHT_LAUNCH_CHECK()                                                               \
  do {                                                                                     \
    g_launch_counter.fetch_add(1, std::memory_order_relaxed);                              \
    cudaError_t _e = cudaGetLastError();                                                   \
    if (_e != cudaSuccess) {                                                               \
      std::fprintf(stderr, "nufht_b200: kernel launch failed: %s\n", cudaGetErrorString(_e)); \
      return NUFHT_E_CUDA;                                                                 \
    }                                                                                      \
  } while (0)

// Exponential-of-semicircle kernel in grid units, support |u| < W/2.
__device__ __forceinline__ double es_kernel(double u, double inv_half_w, double beta) {
  double z = u * inv_half_w;
  double s = 1.0 - z * z;
  return s > 0.0 ? exp(beta * (sqrt(s) - 1.0)) : 0.0;
}

// Fourier transform of the kernel, int psi(u) cos(om u) du, by Gauss-Legendre quadrature.
__device__ __forceinline__ double es_hat(const AsyConst& P, double om) {
  double s = 0.0;
  for (int q = 0; q < P.nq; ++q) s += P.qwpsi[q] * cos(om * P.qx[q]);
  return 2.0 * s;
}

// Asynchronous global -> shared copies (cp.async, completed by cp_async_wait_all).
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

}  // namespace hankel
