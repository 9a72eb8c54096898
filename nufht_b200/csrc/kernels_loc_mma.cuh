// Local boxes on the FP64 tensor cores: the two contractions of the Wimp expansion
// (src/expansions.c:212-337) as warp-level DMMA products (mma.sync.aligned.m8n8k4 with
// FP64 operands and accumulators; sm_100a executes them on its FP64 tensor pipe).
//
//   projection  C[l,t] = sum_j T_l(r_j / r_end) c[j,t]      (K+1) x nj  times  nj x B
//   evaluation  g[i,t] += sum_l b_l(k_i r_end / 2) C[l,t]     ni x (K+1)  times  (K+1) x B
//
// Both stage their left operand in shared memory (the Chebyshev table of a source chunk; the
// Bessel table J_0..J_maxo of a tile of targets, from which b_l is formed while the fragment
// is loaded) and keep 8 x 8 output tiles in registers.  Shared-memory row strides are chosen
// == 4 (mod 16) doubles so that the fragment loads of a half-warp (4 rows x 4 consecutive
// columns) fall in distinct banks.
#pragma once

#include "kernels_loc.cuh"

namespace hankel {


__host__ __device__ constexpr int round8(int v) { return (v + 7) & ~7; }
// Smallest stride >= v with stride == 4 (mod 16).
__host__ __device__ constexpr int stride4(int v) { return v + ((4 - v) % 16 + 16) % 16; }

constexpr int kLocMmaWarps = kLocThreads / 32;

// Shared-memory layout of k_loc_proj_mma (doubles): the table T[MB][TS] of the CTA's block
// of orders, then c[chunk][BS] of its block of columns.
struct LocProjMma {
  int MB, BT, TS, BS, chunk;
  __host__ __device__ size_t doubles() const { return (size_t)MB * TS + (size_t)chunk * BS; }
};
inline LocProjMma loc_proj_mma_layout(int MB, int BT, int chunk) {
  LocProjMma L;
  L.MB = MB;
  L.BT = BT;
  L.chunk = chunk;
  L.TS = stride4(chunk);
  L.BS = stride4(round8(BT));
  return L;
}

// Projection of one source chunk item onto the Chebyshev polynomials.  CTA (item, order block
// ob, column block) covers orders [ob MB, ob MB + MB) and BT columns: it fills only its own
// orders of the table (segments seeded with cos(m theta), see k_loc_proj) and reuses every
// table entry for all BT columns.  Warp w owns the output tiles w, w + 8, ... (at most NT) of the
// (MB/8) x (BT/8) tile grid, strided (tile = w + 8 q): a warp's tiles share their n-tile.
template <int NT>
__global__ void __launch_bounds__(kLocThreads) k_loc_proj_mma(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    const LocBoxD* __restrict__ boxes, const ProjItem* __restrict__ items, int KL1, int odd,
    double* __restrict__ partial, LocProjMma L) {
  const ProjItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int lb = blockIdx.y * L.MB;               // first order of the block
  const int nl = min(L.MB, KL1 - lb);             // orders of the block
  const int t0 = blockIdx.z * L.BT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sT = reinterpret_cast<double*>(smem_raw);  // [MB][TS]
  double* sC = sT + (size_t)L.MB * L.TS;               // [chunk][BS]
  const int chunk = L.chunk;
  const int nnt = round8(L.BT) >> 3;
  const int ntiles = (round8(nl) >> 3) * nnt;
  double acc[NT][2];
  int a_off[NT], b_off[NT];  // this lane's fragment offsets of each tile (-1: no tile)
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    acc[q][0] = acc[q][1] = 0.0;
    const int tile = warp + q * kLocMmaWarps;
    const int mt = tile / nnt, nt = tile - mt * nnt;
    a_off[q] = tile < ntiles ? mt * 8 * L.TS : -1;
    b_off[q] = nt * 8;
  }
  // orders of the block past KL1 (padding to whole m-tiles) stay zero
  for (int e = tid; e < (L.MB - nl) * L.TS; e += blockDim.x) sT[(size_t)nl * L.TS + e] = 0.0;
  const double inv_end = bx.r_end > 0.0 ? 1.0 / bx.r_end : 0.0;
  const int nseg = (nl + kLocSeg - 1) / kLocSeg;
  const int ar = lane >> 2, ac = lane & 3;
  for (int s0 = 0; s0 < it.nj; s0 += chunk) {
    const int ns = min(chunk, it.nj - s0);
    __syncthreads();  // previous chunk consumed
    for (int e = tid; e < nseg * chunk; e += blockDim.x) {
      const int sg = e / chunk, s = e - sg * chunk;
      const int la = sg * kLocSeg, le = min(nl, la + kLocSeg);  // block-relative orders
      if (s < ns) {
        double x = rs[it.j0 + s0 + s] * inv_end;
        x = fmin(fmax(x, -1.0), 1.0);
        const double th = acos(x);
        const int m0 = odd ? 2 * (lb + la) + 1 : 2 * (lb + la);  // degree of order lb + la
        double tp = cos((double)(m0 - 2) * th);
        double tc = cos((double)m0 * th);
        const double two_t2 = 2.0 * (2.0 * x * x - 1.0);
        for (int l = la; l < le; ++l) {
          sT[(size_t)l * L.TS + s] = (odd || lb + l > 0) ? 2.0 * tc : tc;
          const double tn = two_t2 * tc - tp;
          tp = tc;
          tc = tn;
        }
      } else {
        for (int l = la; l < le; ++l) sT[(size_t)l * L.TS + s] = 0.0;
      }
    }
    for (int e = tid; e < chunk * L.BS; e += blockDim.x) {
      const int s = e / L.BS, tt = e - s * L.BS;
      sC[e] = (s < ns && tt < L.BT && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    // sources outer, tiles inner: the warp's NT accumulator chains advance together, and
    // consecutive tiles of a warp reuse the left fragment of their m-tile
    for (int k0 = 0; k0 < chunk; k0 += 4) {
      const double* pa = sT + (size_t)ar * L.TS + k0 + ac;
      const double* pb = sC + (size_t)(k0 + ac) * L.BS + ar;
      int b_cur = -1;
      double b = 0.0;
#pragma unroll
      for (int q = 0; q < NT; ++q) {
        if (a_off[q] >= 0) {  // warp-uniform
          if (b_off[q] != b_cur) {  // constant over q when the n-tile count divides 8
            b_cur = b_off[q];
            b = pb[b_cur];
          }
          dmma884(acc[q][0], acc[q][1], pa[a_off[q]], b);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    const int tile = warp + q * kLocMmaWarps;
    if (tile >= ntiles) continue;
    const int mt = tile / nnt, nt = tile - mt * nnt;
    const int l = lb + mt * 8 + (lane >> 2);
    const int tt = nt * 8 + 2 * (lane & 3);
#pragma unroll
    for (int h = 0; h < 2; ++h)
      if (l < KL1 && tt + h < L.BT && t0 + tt + h < B)
        partial[((size_t)blockIdx.x * KL1 + l) * B + t0 + tt + h] = acc[q][h];
  }
}

// Evaluation: each CTA takes one item (<= kLocTargets targets of one box) in tiles of TI
// targets.  Per tile, TI threads run Miller's recurrence for J_0 .. J_maxo at
// z = k r_end / 2 into a shared table (one row per target); then the warps form
// b_l = J_{l0+odd+l} J_{|l-l0|} (-1)^{max(l-l0,0)} while loading the left fragments and
// multiply by the box's coefficients C, staged kLocMmaK orders x 64 columns at a time.
constexpr int kLocMmaK = 64;     // orders of C staged per round
constexpr int kLocMmaCols = 64;  // columns per pass over a tile
struct LocEvalMma {
  int TI, JS, CS;
  __host__ __device__ size_t doubles() const { return (size_t)TI * JS + (size_t)kLocMmaK * CS; }
};
inline LocEvalMma loc_eval_mma_layout(int TI, int maxo) {
  LocEvalMma L;
  L.TI = TI;
  L.JS = stride4(maxo + 1);
  L.CS = stride4(kLocMmaCols);
  return L;
}

// Unnormalised J_0(z) .. J_nmax(z) into row[0..nmax] by Miller's downward recurrence (as
// bessel_j_orders, bessel.cuh) and the factor 1/S that normalises them (S = f_0 + 2 sum of
// the even-order values).  The recurrence starts above nmax, so it writes every entry; the
// caller scales each factor by 1/S as it forms the products (unnormalised values reach 1e250,
// so their products would overflow).
__device__ __forceinline__ double miller_rows_unnormalised(int nmax, double z, double* row) {
  // Orders far above z underflow: |J_n(z)| <= (z/2)^n / n!, below 1e-300 from some n_eff on.
  // Those entries are zero (their products with |J| <= 1 are below FP64's range), and the
  // recurrence starts above n_eff instead of nmax -- at small z a start at nmax would grow by
  // ~2n/z per step and rescale the whole row every few dozen steps.
  int neff = nmax;
  if (z < (double)nmax) {
    const double lz = log(0.5 * z);
    auto lbound = [&](int n) { return (double)n * lz - lgamma((double)n + 1.0); };
    int lo = max(1, (int)ceil(z)), hi = nmax;
    if (lo < hi && lbound(hi) < -700.0) {
      while (lo < hi) {  // smallest n in [lo, hi] with bound < e^-700
        const int mid = (lo + hi) >> 1;
        if (lbound(mid) < -700.0) hi = mid;
        else lo = mid + 1;
      }
      neff = lo;
    }
  }
  for (int i = neff + 1; i <= nmax; ++i) row[i] = 0.0;
  nmax = neff;
  int M = nmax;
  if ((double)M < z) M = (int)ceil(z);
  const int N = miller_start(M);
  const double tox = 2.0 / z;
  double fkp1 = 0.0, fk = 1e-30, sum = 0.0;
  for (int k = N; k > 0; --k) {
    const double fkm1 = ((double)k * tox) * fk - fkp1;
    fkp1 = fk;
    fk = fkm1;
    if (fabs(fk) > 1e250) {
      fk *= 1e-250;
      fkp1 *= 1e-250;
      sum *= 1e-250;
      for (int i = k; i <= nmax; ++i) row[i] *= 1e-250;
    }
    const int km1 = k - 1;
    if (km1 <= nmax) row[km1] = fk;
    if (km1 > 0 && (km1 & 1) == 0) sum += fk;
  }
  return 1.0 / (2.0 * sum + fk);
}

template <int TI>
__global__ void __launch_bounds__(kLocThreads) k_loc_eval_mma(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const LocBoxD* __restrict__ boxes, const EvalItem* __restrict__ items,
    const double* __restrict__ cheb, int K, int nu_int, double sgn, LocEvalMma L) {
  constexpr int MT = TI / 8;                       // m-tiles per target tile
  constexpr int NTN = kLocMmaCols / 8;             // n-tiles per column pass
  constexpr int NTW = (MT * NTN + kLocMmaWarps - 1) / kLocMmaWarps;  // tiles per warp
  const EvalItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int KL1 = K + 1;
  const int l0 = nu_int / 2, odd = nu_int & 1;
  const int maxo = l0 + K + odd;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ar = lane >> 2, ac = lane & 3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sJ = reinterpret_cast<double*>(smem_raw);  // [TI][JS]
  double* sC = sJ + (size_t)TI * L.JS;                 // [kLocMmaK][CS]
  __shared__ double s_scale[TI];                       // 1 / S per target of the tile
  const double* cbox = cheb + (size_t)it.box * KL1 * B;
  // Warp w owns tiles w NTW .. w NTW + NTW - 1 of the MT x NTN tile grid (row-major), so
  // consecutive tiles of a warp share their m-tile and the left fragment.
  const int tile0 = warp * NTW;
  for (int i0 = 0; i0 < it.ni; i0 += TI) {
    __syncthreads();  // previous tile's table consumed
    if (tid < TI) {
      double* row = sJ + (size_t)tid * L.JS;
      const int i = it.i0 + i0 + tid;
      const double z = i0 + tid < it.ni ? ws[i] * bx.r_end / 2.0 : 0.0;
      if (z < 1e-30) {
        for (int q = 0; q <= maxo; ++q) row[q] = 0.0;
        row[0] = 1.0;
        s_scale[tid] = 1.0;
      } else {
        s_scale[tid] = miller_rows_unnormalised(maxo, z, row);
      }
    }
    for (int cb = 0; cb < B; cb += kLocMmaCols) {
      const int ncol = min(kLocMmaCols, B - cb);
      double acc[NTW][2];
#pragma unroll
      for (int q = 0; q < NTW; ++q) acc[q][0] = acc[q][1] = 0.0;
      for (int kc = 0; kc < KL1; kc += kLocMmaK) {
        const int kn = min(kLocMmaK, KL1 - kc);
        const int kn4 = (kn + 3) & ~3, nc8 = round8(ncol);
        __syncthreads();  // table written / previous coefficients consumed
        for (int e = tid; e < kn4 * nc8; e += blockDim.x) {
          const int l = e / nc8, t = e - l * nc8;
          sC[(size_t)l * L.CS + t] = (l < kn && t < ncol) ? cbox[(size_t)(kc + l) * B + cb + t] : 0.0;
        }
        __syncthreads();
        for (int k0 = 0; k0 < kn; k0 += 4) {
          const int l = kc + k0 + ac;  // order of this lane's left element
          const int lo = l > l0 ? l - l0 : l0 - l;
          const bool neg = l > l0 && ((l - l0) & 1);
          const double* bl = sC + (size_t)(k0 + ac) * L.CS + ar;
          int mt_cur = -1;
          double a = 0.0;
#pragma unroll
          for (int q = 0; q < NTW; ++q) {
            const int tile = tile0 + q;
            if (tile < MT * NTN) {
              const int mt = tile / NTN, nt = tile - mt * NTN;
              if (mt != mt_cur) {  // warp-uniform
                mt_cur = mt;
                a = 0.0;
                if (l < KL1) {
                  const double* jrow = sJ + (size_t)(mt * 8 + ar) * L.JS;
                  const double iv = s_scale[mt * 8 + ar];
                  a = (jrow[l0 + odd + l] * iv) * (jrow[lo] * iv);
                  if (neg) a = -a;
                }
              }
              if (nt * 8 < ncol) dmma884(acc[q][0], acc[q][1], a, bl[nt * 8]);
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NTW; ++q) {
        const int tile = tile0 + q;
        if (tile >= MT * NTN) continue;
        const int mt = tile / NTN, nt = tile - mt * NTN;
        const int ii = i0 + mt * 8 + ar;
        const int tt = nt * 8 + 2 * ac;
        if (ii >= it.ni) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (tt + h < ncol) atomicAdd(&gs[(size_t)(cb + tt + h) * ld_gs + it.i0 + ii], sgn * acc[q][h]);
      }
    }
  }
}

}  // namespace hankel
