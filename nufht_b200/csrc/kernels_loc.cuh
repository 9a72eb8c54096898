// Local boxes: the Wimp expansion (src/expansions.c:212-337)
//   g[i,t] += sum_{l=0}^{K} b_l(k_i r_end / 2) C[l,t],
//   C[l,t]  = sum_j T_l(r_j / r_end) c[j,t],
// with T_l = eps_l T_{2l} (even nu; eps_0 = 1, else 2) or 2 T_{2l+1} (odd nu) and
// b_l(z) = J_{l0+odd+l}(z) J_{|l-l0|}(z) (-1)^{max(l-l0,0)}, l0 = nu/2 rounded down.
#pragma once

#include "bessel.cuh"
#include "kernels_common.cuh"

namespace hankel {

constexpr int kLocSources = 2048;  // sources per projection work item
constexpr int kLocChunk = 64;      // sources staged per round, at most
constexpr int kLocTargets = 128;   // targets per evaluation CTA
constexpr int kLocThreads = 256;   // threads of a projection CTA
constexpr int kLocMaxNL = 40;      // expansion orders per projection thread, at most
constexpr int kLocSeg = 32;        // expansion orders per thread when filling the table

// Partial projections over one source chunk.  The table T_l(x_s) of a chunk is filled in
// segments of kLocSeg orders, all threads at once: a thread takes one (segment, source)
// pair, seeds it with cos(m theta) (x = cos theta) for its first two polynomial degrees and
// steps with T_{m+2} = 2 T_2(x) T_m - T_{m-2} (the degrees of one parity; stable for
// |x| <= 1), so a Wimp degree in the hundreds costs no long serial recurrence.  Thread
// (l_out, t_out) owns column t0 + t_out and the orders l_out + q LS, q < NL (LS =
// kLocThreads / BT): NL = 1 for the usual degrees, up to kLocMaxNL for the degrees of very
// large orders, which keeps BT (columns per CTA, each CTA refilling the table) large.
// `chunk` (even) sources are staged per round so that the KL1 x chunk table fits in shared
// memory.
template <int NL>
__global__ void __launch_bounds__(kLocThreads) k_loc_proj(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    const LocBoxD* __restrict__ boxes, const ProjItem* __restrict__ items, int KL1, int odd,
    double* __restrict__ partial, int BT, int chunk) {
  const ProjItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int t0 = blockIdx.y * BT;
  const int tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sT = reinterpret_cast<double*>(smem_raw);  // [KL1][chunk]
  double* sC = sT + (size_t)KL1 * chunk;              // [chunk][BT]
  const int LS = kLocThreads / BT;
  const int l_out = tid / BT, t_out = tid - l_out * BT;
  double acc[NL];
#pragma unroll
  for (int q = 0; q < NL; ++q) acc[q] = 0.0;
  // A box whose sources all sit at r = 0 has r_end = 0; then only the l = 0 term survives
  // (J_l(0) = 0 for l >= 1) and any x works.  The reference divides by zero there.
  const double inv_end = bx.r_end > 0.0 ? 1.0 / bx.r_end : 0.0;
  const int nseg = (KL1 + kLocSeg - 1) / kLocSeg;
  for (int s0 = 0; s0 < it.nj; s0 += chunk) {
    const int ns = min(chunk, it.nj - s0);
    for (int e = tid; e < nseg * chunk; e += blockDim.x) {
      const int sg = e / chunk, s = e - sg * chunk;
      const int l0 = sg * kLocSeg, l1 = min(KL1, l0 + kLocSeg);
      if (s < ns) {
        double x = rs[it.j0 + s0 + s] * inv_end;
        x = fmin(fmax(x, -1.0), 1.0);
        const double th = acos(x);
        const int m0 = odd ? 2 * l0 + 1 : 2 * l0;  // degree of order l0
        double tp = cos((double)(m0 - 2) * th);     // T_{m0-2} (T_{-n} = T_n)
        double tc = cos((double)m0 * th);           // T_{m0}
        const double two_t2 = 2.0 * (2.0 * x * x - 1.0);
        for (int l = l0; l < l1; ++l) {
          sT[(size_t)l * chunk + s] = (odd || l > 0) ? 2.0 * tc : tc;
          const double tn = two_t2 * tc - tp;
          tp = tc;
          tc = tn;
        }
      } else {
        for (int l = l0; l < l1; ++l) sT[(size_t)l * chunk + s] = 0.0;
      }
    }
    for (int e = tid; e < chunk * BT; e += blockDim.x) {
      int tt = e / chunk, s = e - tt * chunk;
      sC[s * BT + tt] = (s < ns && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    // Sources in pairs: one coefficient load per source serves all NL orders, one 16-byte
    // table load two multiply-adds (chunk is even, so every pair is 16-byte aligned).
    const int ns2 = ns & ~1;
    for (int s = 0; s < ns2; s += 2) {
      const double c0 = sC[s * BT + t_out], c1 = sC[(s + 1) * BT + t_out];
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const int l = l_out + q * LS;
        if (l < KL1) {
          const double2 tv = *reinterpret_cast<const double2*>(sT + (size_t)l * chunk + s);
          acc[q] = fma(tv.x, c0, acc[q]);
          acc[q] = fma(tv.y, c1, acc[q]);
        }
      }
    }
    if (ns & 1) {
      const double c0 = sC[ns2 * BT + t_out];
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const int l = l_out + q * LS;
        if (l < KL1) acc[q] = fma(sT[(size_t)l * chunk + ns2], c0, acc[q]);
      }
    }
    __syncthreads();
  }
  if (t0 + t_out < B) {
#pragma unroll
    for (int q = 0; q < NL; ++q) {
      const int l = l_out + q * LS;
      if (l < KL1) partial[((size_t)blockIdx.x * KL1 + l) * B + t0 + t_out] = acc[q];
    }
  }
}

__global__ void k_loc_reduce(const LocBoxD* __restrict__ boxes, int nbox, int KL1, int B,
                             const double* __restrict__ partial, double* __restrict__ cheb) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long tot = (long long)nbox * KL1 * B;
  if (e >= tot) return;
  int b = (int)(e / ((long long)KL1 * B));
  int rem = (int)(e - (long long)b * KL1 * B);
  const LocBoxD bx = boxes[b];
  double s = 0.0;
  for (int q = 0; q < bx.nitems; ++q) s += partial[(size_t)(bx.item0 + q) * KL1 * B + rem];
  cheb[e] = s;
}

constexpr int kLocEvalCols = 16;  // columns accumulated in registers per evaluation pass

// Evaluation at the box's targets: J_0 .. J_maxo at z = k r_end / 2 by Miller's algorithm
// (local array of MAXO + 1 values per thread), then g[i,t] += sum_l b_l C[l,t] with
// b_l = J_{l0+odd+l} J_{|l-l0|} (-1)^{max(l-l0,0)}.  The coefficients C of the box are
// staged in shared memory for BTC columns at a time (the rows padded by kLocEvalCols
// values); each b_l, formed from two reads of the local array, feeds kLocEvalCols columns
// held in registers, so large Wimp degrees do not re-read the array once per column.
template <int MAXO>
__global__ void __launch_bounds__(kLocTargets) k_loc_eval(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const LocBoxD* __restrict__ boxes, const EvalItem* __restrict__ items,
    const double* __restrict__ cheb, int K, int nu_int, double sgn, int BTC) {
  const EvalItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int KL1 = K + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s_cheb = reinterpret_cast<double*>(smem_raw);  // [KL1][BTC]
  const int tid = threadIdx.x;
  const bool has = tid < it.ni;
  const int i = it.i0 + (has ? tid : 0);
  const int l0 = nu_int / 2, odd = nu_int & 1;
  const int maxo = l0 + K + odd;
  double J[MAXO + 1];
  if (has) {
    double z = ws[i] * bx.r_end / 2.0;
    if (z < 1e-30) {
      for (int q = 0; q <= maxo; ++q) J[q] = 0.0;
      J[0] = 1.0;
    } else {
      bessel_j_orders(maxo, z, J);
    }
  }
  for (int tb = 0; tb < B; tb += BTC) {
    const int nt = min(BTC, B - tb);
    __syncthreads();
    for (int e = tid; e < KL1 * nt; e += blockDim.x) {
      int l = e / nt, tt = e - l * nt;
      s_cheb[l * BTC + tt] = cheb[((size_t)it.box * KL1 + l) * B + tb + tt];
    }
    __syncthreads();
    if (!has) continue;
    for (int tc = 0; tc < nt; tc += kLocEvalCols) {
      double acc[kLocEvalCols];
#pragma unroll
      for (int u = 0; u < kLocEvalCols; ++u) acc[u] = 0.0;
      for (int l = 0; l <= K; ++l) {
        int lo = l > l0 ? l - l0 : l0 - l;
        double v = J[l0 + odd + l] * J[lo];
        if (l > l0 && ((l - l0) & 1)) v = -v;
        const double* row = s_cheb + l * BTC + tc;  // the padding covers row[u] past BTC
#pragma unroll
        for (int u = 0; u < kLocEvalCols; ++u) acc[u] = fma(v, row[u], acc[u]);
      }
      const int nu_c = min(kLocEvalCols, nt - tc);
      for (int u = 0; u < nu_c; ++u) atomicAdd(&gs[(size_t)(tb + tc + u) * ld_gs + i], sgn * acc[u]);
    }
  }
}

}  // namespace hankel
