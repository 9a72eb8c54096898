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
constexpr int kLocChunk = 64;      // sources staged per round
constexpr int kLocTargets = 128;   // targets per evaluation CTA

// Partial projections over one source chunk; Chebyshev polynomials by the three-term
// recurrence T_{n+1} = 2 x T_n - T_{n-1}.
__global__ void __launch_bounds__(256) k_loc_proj(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    const LocBoxD* __restrict__ boxes, const ProjItem* __restrict__ items, int KL1, int odd,
    double* __restrict__ partial, int BT) {
  const ProjItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int t0 = blockIdx.y * BT;
  const int tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sT = reinterpret_cast<double*>(smem_raw);  // [KL1][kLocChunk]
  double* sC = sT + KL1 * kLocChunk;                  // [kLocChunk][BT]
  const int l_out = tid / BT, t_out = tid - l_out * BT;
  const bool has_out = l_out < KL1;
  double acc = 0.0;
  // A box whose sources all sit at r = 0 has r_end = 0; then only the l = 0 term survives
  // (J_l(0) = 0 for l >= 1) and any x works.  The reference divides by zero there.
  const double inv_end = bx.r_end > 0.0 ? 1.0 / bx.r_end : 0.0;
  for (int s0 = 0; s0 < it.nj; s0 += kLocChunk) {
    const int ns = min(kLocChunk, it.nj - s0);
    for (int s = tid; s < kLocChunk; s += blockDim.x) {
      if (s < ns) {
        double x = rs[it.j0 + s0 + s] * inv_end;
        x = fmin(fmax(x, -1.0), 1.0);
        double tm1 = 1.0, tc = x;  // T_{n-1}, T_n as n advances
        int l = 0;
        for (int nn = 0; l < KL1; ++nn) {
          double Tn;
          if (nn == 0) {
            Tn = 1.0;
          } else if (nn == 1) {
            Tn = x;
          } else {
            double tn = 2.0 * x * tc - tm1;
            tm1 = tc;
            tc = tn;
            Tn = tn;
          }
          int order = odd ? 2 * l + 1 : 2 * l;
          if (nn == order) {
            sT[l * kLocChunk + s] = odd ? 2.0 * Tn : (l == 0 ? Tn : 2.0 * Tn);
            ++l;
          }
        }
      } else {
        for (int l = 0; l < KL1; ++l) sT[l * kLocChunk + s] = 0.0;
      }
    }
    for (int e = tid; e < kLocChunk * BT; e += blockDim.x) {
      int tt = e / kLocChunk, s = e - tt * kLocChunk;
      sC[s * BT + tt] =
          (s < ns && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    if (has_out) {
      const double* Tl = sT + l_out * kLocChunk;
#pragma unroll 8
      for (int s = 0; s < kLocChunk; ++s) acc = fma(Tl[s], sC[s * BT + t_out], acc);
    }
    __syncthreads();
  }
  if (has_out && t0 + t_out < B)
    partial[((size_t)blockIdx.x * KL1 + l_out) * B + t0 + t_out] = acc;
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

template <int MAXO>
__global__ void __launch_bounds__(kLocTargets) k_loc_eval(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const LocBoxD* __restrict__ boxes, const EvalItem* __restrict__ items,
    const double* __restrict__ cheb, int K, int nu_int, double sgn) {
  const EvalItem it = items[blockIdx.x];
  const LocBoxD bx = boxes[it.box];
  const int KL1 = K + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s_cheb = reinterpret_cast<double*>(smem_raw);  // [KL1][B]
  for (int e = threadIdx.x; e < KL1 * B; e += blockDim.x)
    s_cheb[e] = cheb[(size_t)it.box * KL1 * B + e];
  __syncthreads();
  const int tid = threadIdx.x;
  if (tid >= it.ni) return;
  const int i = it.i0 + tid;
  const int l0 = nu_int / 2, odd = nu_int & 1;
  const int maxo = l0 + K + odd;
  double J[MAXO + 1];
  double z = ws[i] * bx.r_end / 2.0;
  if (z < 1e-30) {
    for (int q = 0; q <= maxo; ++q) J[q] = 0.0;
    J[0] = 1.0;
  } else {
    bessel_j_orders(maxo, z, J);
  }
  double bl[MAXO + 1];
  for (int l = 0; l <= K; ++l) {
    int lo = l > l0 ? l - l0 : l0 - l;
    double v = J[l0 + odd + l] * J[lo];
    if (l > l0 && ((l - l0) & 1)) v = -v;
    bl[l] = v;
  }
  for (int t = 0; t < B; ++t) {
    double acc = 0.0;
    for (int l = 0; l <= K; ++l) acc = fma(bl[l], s_cheb[l * B + t], acc);
    atomicAdd(&gs[(size_t)t * ld_gs + i], sgn * acc);
  }
}

}  // namespace hankel
