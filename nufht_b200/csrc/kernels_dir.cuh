// Direct boxes: g[i,t] += sum_j c[j,t] J_nu(k_i r_j)  (src/expansions.c:78-97).
// One Bessel value per (i, j) pair, reused across the batch columns.  k_dir (the default)
// keeps BT columns in registers per thread: tall boxes map one thread to a target, thin boxes
// (few targets, many sources) give each target `lanes` threads that split the sources and
// combine with warp shuffles.  k_dir_mma (NUFHT_B200_DIR_MMA=1) evaluates tiles of Bessel
// values and multiplies them by the coefficients on the FP64 tensor cores.
#pragma once

#include "bessel.cuh"
#include "kernels_common.cuh"

namespace hankel {

constexpr int kDirThreads = 128;
constexpr int kDirSources = 1024;  // sources per work item
constexpr int kDirChunk = 64;      // sources per shared-memory stage (two stages in flight)
static_assert(kDirChunk % 64 == 0, "a stage must hold whole pairs of steps of up to 32 lanes");
constexpr int kThinDirect = 16;    // asymptotic boxes this thin (sources or targets) are summed directly

// Plan-time table of J_nu on [0, nint): on each unit interval [a, a+1) the Chebyshev
// coefficients of degree < kJTabCoefs in t = 2 (x - a) - 1, from J_nu at the interval's
// Chebyshev-Gauss nodes (the exact evaluation of bessel.cuh).  J_nu and all its derivatives
// are bounded by 1 on the real line, so the coefficients of a unit interval fall below 1e-20
// by degree 15; evaluation is one Clenshaw sum (16 multiply-adds on 128 bytes that the
// sorted arguments of a thread keep in L1) instead of a recurrence over the order (about 250
// steps of Miller's algorithm at order 100 near the transition region) or Hankel's
// expansion with up to 34 terms (order 0 from x = 17).
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
  // Two stages of kDirChunk sources: radii and the BT columns of c ([column][source]), filled
  // by asynchronous copies while the CTA sums the other stage.
  __shared__ __align__(16) double s_r[2][kDirChunk];
  __shared__ __align__(16) double s_c[2][BT * kDirChunk];
  double acc[BT];
#pragma unroll
  for (int q = 0; q < BT; ++q) acc[q] = 0.0;
  auto stage = [&](int b, int s0) {
    const int ns = min(kDirChunk, it.nj - s0);
    for (int s = tid; s < kDirChunk; s += kDirThreads) {
      if (s < ns) cp_async8(&s_r[b][s], rs + it.j0 + s0 + s);
      else s_r[b][s] = 0.0;
    }
    for (int e = tid; e < kDirChunk * BT; e += kDirThreads) {
      const int tt = e / kDirChunk, s = e - tt * kDirChunk;
      if (s < ns && t0 + tt < B) cp_async8(&s_c[b][e], cs + (size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s);
      else s_c[b][e] = 0.0;
    }
    cp_async_commit();
  };
  stage(0, 0);
  int b = 0;
  for (int s0 = 0; s0 < it.nj; s0 += kDirChunk) {
    const int ns = min(kDirChunk, it.nj - s0);
    cp_async_wait_all();  // this thread's copies of stage b have landed
    __syncthreads();      // all copies of stage b visible; stage b ^ 1 no longer read
    if (s0 + kDirChunk < it.nj) stage(b ^ 1, s0 + kDirChunk);
    const double* cr = s_r[b];
    const double* cc = s_c[b];
    if (valid) {
      // Two independent Bessel evaluations per step for instruction-level parallelism.  The
      // stage length is a multiple of 2 L, so each thread visits its sources in the same
      // order whatever the stage length.
      int s = lane;
      for (; s + L < ns; s += 2 * L) {
        double Ja = bessel_j_dir(nu2, k * cr[s], jtab, jtab_n);
        double Jb = bessel_j_dir(nu2, k * cr[s + L], jtab, jtab_n);
#pragma unroll
        for (int q = 0; q < BT; ++q) {
          acc[q] = fma(cc[q * kDirChunk + s], Ja, acc[q]);
          acc[q] = fma(cc[q * kDirChunk + s + L], Jb, acc[q]);
        }
      }
      if (s < ns) {
        double J = bessel_j_dir(nu2, k * cr[s], jtab, jtab_n);
#pragma unroll
        for (int q = 0; q < BT; ++q) acc[q] = fma(cc[q * kDirChunk + s], J, acc[q]);
      }
    }
    b ^= 1;
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

// Direct boxes on the FP64 tensor cores.  Per chunk of SC sources the CTA evaluates the
// Bessel tile J[i][s] = J_nu(k_i r_s) of its targets into shared memory (ROWS x SC = 2048
// independent evaluations, 16 per thread, so their latency chains overlap), then adds
// J (ROWS x SC) times c (SC x 8 NTN columns) with mma.sync.m8n8k4.f64 (DMMA) tiles: the B
// multiply-adds per pair leave the FP64 pipe, which keeps only the Bessel evaluation.  ROWS =
// 64 (items of up to 64 targets; warps own pairs of m-tiles) or 16 (thin boxes, up to 16
// targets and 128 sources per chunk; the warps split the k-steps and each adds its partial
// sums).  Shared-memory rows of SC + 4 doubles (== 4 mod 16) keep the fragment loads free of
// bank conflicts.
constexpr int kDirMmaTile = 2048;  // Bessel values per chunk
constexpr int kDirMmaSources = 1024;  // sources per work item

template <int ROWS>
struct DirMmaSmem {
  static constexpr int SC = kDirMmaTile / ROWS;  // sources per chunk
  static constexpr int LD = SC + 4;              // row stride of J and c (doubles)
  static constexpr size_t bytes(int BT) { return sizeof(double) * ((size_t)(ROWS + BT) * LD + SC + ROWS); }
};

template <int ROWS, int NTN>
__global__ void __launch_bounds__(128, 4) k_dir_mma(
    const double* __restrict__ rs, const double* __restrict__ ws, const double* __restrict__ cs,
    int ld_cs, double* __restrict__ gs, int ld_gs, int B, const DirItem* __restrict__ items,
    int nu2, double sgn, const double* __restrict__ jtab, int jtab_n) {
  using S = DirMmaSmem<ROWS>;
  constexpr int SC = S::SC, LD = S::LD;
  constexpr int BT = 8 * NTN;
  constexpr int MG = ROWS / 16;  // groups of two m-tiles
  constexpr int WK = 4 / MG;     // warps sharing one group (splitting the k-steps)
  const DirItem it = items[blockIdx.x];
  const int t0 = blockIdx.y * BT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int mg = warp / WK, kp = warp - mg * WK;
  const int MT = (it.ni + 7) >> 3;  // m-tiles holding targets
  extern __shared__ __align__(16) double dsm[];
  double* s_J = dsm;                 // [ROWS][LD]
  double* s_c = s_J + ROWS * LD;     // [BT][LD]: column-major tile of c
  double* s_r = s_c + BT * LD;       // [SC]
  double* s_k = s_r + SC;            // [ROWS]
  for (int i = tid; i < ROWS; i += 128) s_k[i] = i < it.ni ? ws[it.i0 + i] : 0.0;
  double acc[2][NTN][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NTN; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  const int rows = MT * 8;
  for (int s0 = 0; s0 < it.nj; s0 += SC) {
    const int ns = min(SC, it.nj - s0);
    __syncthreads();  // the previous chunk's tiles are consumed (and s_k is visible)
    for (int s = tid; s < SC; s += 128) s_r[s] = s < ns ? rs[it.j0 + s0 + s] : 0.0;
    for (int e = tid; e < BT * SC; e += 128) {
      const int tt = e / SC, s = e - tt * SC;
      s_c[tt * LD + s] = (s < ns && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    // the Bessel tile: rows of the item's targets only (rows * SC is a multiple of 256), zeros
    // past its targets and sources; two independent evaluations per step, both straight-line
    // (an unused slot evaluates at x = 1 and is discarded) so that their chains overlap
    const int nev = rows * SC;
    for (int e = tid; e < nev; e += 256) {
      const int e2 = e + 128;
      const int ia = e / SC, sa = e - ia * SC;
      const int ib = e2 / SC, sb = e2 - ib * SC;
      const bool va = ia < it.ni && sa < ns, vb = ib < it.ni && sb < ns;
      const double xa = va ? s_k[ia] * s_r[sa] : 1.0, xb = vb ? s_k[ib] * s_r[sb] : 1.0;
      const double Ja = bessel_j_dir(nu2, xa, jtab, jtab_n);
      const double Jb = bessel_j_dir(nu2, xb, jtab, jtab_n);
      s_J[ia * LD + sa] = va ? Ja : 0.0;
      s_J[ib * LD + sb] = vb ? Jb : 0.0;
    }
    __syncthreads();
    // J x c on DMMA tiles: this warp's two m-tiles, all NTN n-tiles, its share of the k-steps
#pragma unroll 2
    for (int ks = kp; ks < SC / 4; ks += WK) {
      const int k0 = ks * 4;
      double a[2], b[NTN];
#pragma unroll
      for (int q = 0; q < 2; ++q) a[q] = s_J[((mg * 2 + q) * 8 + (lane >> 2)) * LD + k0 + (lane & 3)];
#pragma unroll
      for (int q = 0; q < NTN; ++q) b[q] = s_c[(q * 8 + (lane >> 2)) * LD + k0 + (lane & 3)];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (mg * 2 + q >= MT) continue;
#pragma unroll
        for (int p = 0; p < NTN; ++p) dmma884(acc[q][p][0], acc[q][p][1], a[q], b[p]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int i = (mg * 2 + q) * 8 + (lane >> 2);
    if (i >= it.ni) continue;
#pragma unroll
    for (int p = 0; p < NTN; ++p)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = t0 + p * 8 + 2 * (lane & 3) + h;
        if (t < B) atomicAdd(&gs[(size_t)t * ld_gs + it.i0 + i], sgn * acc[q][p][h]);
      }
  }
}

__global__ void k_besselj(int nu2, const double* __restrict__ x, double* __restrict__ out,
                          long count) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) out[e] = bessel_j(nu2, x[e]);
}

}  // namespace hankel
