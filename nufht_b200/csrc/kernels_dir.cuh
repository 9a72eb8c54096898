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

// Plan-time table of J_nu on [0, nint): on each unit interval [a, a+1) the Chebyshev
// coefficients of degree < kJTabCoefs in t = 2 (x - a) - 1, from J_nu at the interval's
// Chebyshev-Gauss nodes (the exact evaluation of bessel.cuh).  J_nu and all its derivatives
// are bounded by 1 on the real line, so the coefficients of a unit interval fall below 1e-20
// by degree 15; evaluation is one Clenshaw sum instead of a recurrence over the order (about
// 250 steps of Miller's algorithm at order 100 near the transition region).
constexpr int kJTabCoefs = 16;
constexpr int kJTabMaxIntervals = 4096;

__global__ void k_build_jtable(int nu2, double* __restrict__ tab, int nint) {
  __shared__ double f[kJTabCoefs];
  const int a = blockIdx.x, j = threadIdx.x;
  if (a >= nint) return;
  const double tj = cos(M_PI * (j + 0.5) / kJTabCoefs);
  f[j] = bessel_j(nu2, (double)a + 0.5 * (tj + 1.0));
  __syncthreads();
  double c = 0.0;
  for (int q = 0; q < kJTabCoefs; ++q) c += f[q] * cos(M_PI * j * (q + 0.5) / kJTabCoefs);
  c *= 2.0 / kJTabCoefs;
  if (j == 0) c *= 0.5;
  tab[(size_t)a * kJTabCoefs + j] = c;
}

__device__ __forceinline__ double jtab_eval(const double* __restrict__ tab, double x) {
  const int a = (int)x;
  const double t = 2.0 * (x - (double)a) - 1.0, t2 = 2.0 * t;
  const double2* c2 = reinterpret_cast<const double2*>(tab + (size_t)a * kJTabCoefs);
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int k = kJTabCoefs / 2 - 1; k >= 0; --k) {
    const double2 cc = __ldg(c2 + k);
    double bn = fma(t2, b1, cc.y - b2);  // coefficient 2k + 1
    b2 = b1;
    b1 = bn;
    if (k > 0) {
      bn = fma(t2, b1, cc.x - b2);  // coefficient 2k
      b2 = b1;
      b1 = bn;
    } else {
      return fma(t, b1, cc.x - b2);
    }
  }
  return 0.0;
}

// J_nu(x) from the table where it covers x, else directly.
__device__ __forceinline__ double bessel_j_dir(int nu2, double x, const double* __restrict__ tab, int nint) {
  return (tab != nullptr && x < (double)nint) ? jtab_eval(tab, x) : bessel_j(nu2, x);
}

// At least 4 CTAs per SM (registers capped at 128 a thread): the Bessel recurrences are
// latency chains, and the extra warps hide them better than the registers the compiler
// would otherwise keep (measured on B200: direct phase 3.33 -> 2.88 ms at the 1e6-point
// workload).
template <int BT>
__global__ void __launch_bounds__(kDirThreads, 4) k_dir(
    const double* __restrict__ rs, const double* __restrict__ ws, const double* __restrict__ cs,
    int ld_cs, double* __restrict__ gs, int ld_gs, int B, const DirItem* __restrict__ items,
    int nu2, double sgn, const double* __restrict__ jtab, int jtab_n) {
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
        double Ja = bessel_j_dir(nu2, k * s_r[s], jtab, jtab_n);
        double Jb = bessel_j_dir(nu2, k * s_r[s + L], jtab, jtab_n);
#pragma unroll
        for (int q = 0; q < BT; ++q) {
          acc[q] = fma(s_c[q * kDirChunk + s], Ja, acc[q]);
          acc[q] = fma(s_c[q * kDirChunk + s + L], Jb, acc[q]);
        }
      }
      if (s < ns) {
        double J = bessel_j_dir(nu2, k * s_r[s], jtab, jtab_n);
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
