// Direct boxes: g[i,t] += sum_j c[j,t] J_nu(k_i r_j)  (src/expansions.c:78-97).
// One Bessel value per (i, j) pair, reused across BT batch columns held in registers.
// Tall boxes map one thread to a target; thin boxes (few targets, many sources) give each
// target `lanes` threads that split the sources and combine with warp shuffles.
#pragma once

#include "bessel.cuh"
#include "kernels_common.cuh"

namespace hankel {

constexpr int kDirThreads = 128;
constexpr int kDirSources = 1024;  // sources per work item
constexpr int kDirChunk = 64;      // sources staged in shared memory per round
constexpr int kThinDirect = 16;    // asymptotic boxes this thin (sources or targets) are summed directly

// At least 4 CTAs per SM (registers capped at 128 a thread): the Bessel recurrences are
// latency chains, and the extra warps hide them better than the registers the compiler
// would otherwise keep (measured on B200: direct phase 3.33 -> 2.88 ms at the 1e6-point
// workload).
template <int BT>
__global__ void __launch_bounds__(kDirThreads, 4) k_dir(
    const double* __restrict__ rs, const double* __restrict__ ws, const double* __restrict__ cs,
    int ld_cs, double* __restrict__ gs, int ld_gs, int B, const DirItem* __restrict__ items,
    int nu2, double sgn) {
  const DirItem it = items[blockIdx.x];
  const int t0 = blockIdx.y * BT;
  const int tid = threadIdx.x;
  const int L = it.lanes;
  const int ti = tid / L, lane = tid - ti * L;
  const bool valid = ti < it.ni;
  const double k = valid ? ws[it.i0 + ti] : 0.0;
  __shared__ double s_r[kDirChunk];
  __shared__ double s_c[BT * kDirChunk];  // [column][source]
  double acc[BT];
#pragma unroll
  for (int q = 0; q < BT; ++q) acc[q] = 0.0;
  for (int s0 = 0; s0 < it.nj; s0 += kDirChunk) {
    const int ns = min(kDirChunk, it.nj - s0);
    for (int s = tid; s < ns; s += kDirThreads) s_r[s] = rs[it.j0 + s0 + s];
    for (int e = tid; e < kDirChunk * BT; e += kDirThreads) {
      int tt = e / kDirChunk, s = e - tt * kDirChunk;
      s_c[e] = (s < ns && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    if (valid) {
      // Two independent Bessel evaluations per step for instruction-level parallelism.
      int s = lane;
      for (; s + L < ns; s += 2 * L) {
        double Ja = bessel_j(nu2, k * s_r[s]);
        double Jb = bessel_j(nu2, k * s_r[s + L]);
#pragma unroll
        for (int q = 0; q < BT; ++q) {
          acc[q] = fma(s_c[q * kDirChunk + s], Ja, acc[q]);
          acc[q] = fma(s_c[q * kDirChunk + s + L], Jb, acc[q]);
        }
      }
      if (s < ns) {
        double J = bessel_j(nu2, k * s_r[s]);
#pragma unroll
        for (int q = 0; q < BT; ++q) acc[q] = fma(s_c[q * kDirChunk + s], J, acc[q]);
      }
    }
    __syncthreads();
  }
  for (int off = L >> 1; off > 0; off >>= 1) {
#pragma unroll
    for (int q = 0; q < BT; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
  }
  if (valid && lane == 0) {
#pragma unroll
    for (int q = 0; q < BT; ++q)
      if (t0 + q < B) atomicAdd(&gs[(size_t)(t0 + q) * ld_gs + it.i0 + ti], sgn * acc[q]);
  }
}

__global__ void k_besselj(int nu2, const double* __restrict__ x, double* __restrict__ out,
                          long count) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) out[e] = bessel_j(nu2, x[e]);
}

}  // namespace hankel
