// Asymptotic boxes: Hankel's large-argument expansion (src/expansions.c:483-559) evaluated
// with a type-3 NUFFT written for this executor.
//
// For one box with sources r in [C - X, C + X] and targets k in [D - S, D + S] every one
// of the NLP = 2 (K + 1) expansion terms and every batch column t is a transform
//   F_{lp,t}(k) = sum_j c[j,t] (rref / r_j)^{lp+1/2} exp(i k r_j),   lp = 2l + p,
// whose target factor is sqrt(2/pi) (-1)^l a_lp (k rref)^{-(lp+1/2)}; rref (the box's
// smallest radius) keeps both factors bounded.  Stage 1 spreads
// a_j exp(i D (r_j - C)) with the exponential-of-semicircle kernel psi onto cells l h,
// h = pi / (sigma S); stage 2 divides by psi-hat, zero-pads to n2 >= sigma (2 half + 1) and
// runs a backward FFT (cuFFT); stage 3 interpolates at u = (k - D) h n2 / (2 pi) and
// multiplies by exp(i (phi + k C)) / psi-hat((k - D) h) and the target factor.  Terms with
// p = 0 add Re, p = 1 subtract Im (src/expansions.c:520-557); both are written as
// Re(mu F) with mu rotated by i for p = 1.
//
// T is the arithmetic and grid-storage type of stages 1-3: double (plain FP64) or float
// (mixed precision).  Cell indices, source and target phases, the deconvolution tables and
// the final combination into g stay in FP64 in both.
//
// Workspace layout: box b owns n2 * V contiguous complex values, vector v = t * NLP + lp
// at offset cell_off * V + v * n2 (one contiguous FFT input per vector).
#pragma once

#include <climits>

#include "kernels_common.cuh"

namespace hankel {

constexpr int kSpreadTile = 16;     // cells owned by one mode-0 spreading CTA
constexpr int kSpreadChunk = 64;    // sources staged in shared memory per round
constexpr int kChunkSources = 2048; // sources per mode-1 work item, at most
constexpr int kTileMaxSources = 4096;
constexpr int kInterpTile = 128;    // targets per interpolation CTA
constexpr int kInterpChunk = 32;    // targets per shared-memory round

// Window capacity (cells) of a spreading CTA for kernel width W.
__host__ __device__ constexpr int spread_window(int W) { return W + 8 > kSpreadTile ? W + 8 : kSpreadTile; }
// Vectors per interpolating thread for kernel width W.
__host__ __device__ constexpr int interp_vpt(int W) { return W <= 12 ? 2 : 1; }

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

template <typename T>
__device__ __forceinline__ typename Cplx<T>::type cmake(T x, T y) {
  typename Cplx<T>::type v;
  v.x = x;
  v.y = y;
  return v;
}

// Exponential-of-semicircle kernel in the arithmetic type.
__device__ __forceinline__ double es_kernel_t(double u, double ihw, double beta) { return es_kernel(u, ihw, beta); }
__device__ __forceinline__ float es_kernel_t(float u, float ihw, float beta) {
  float z = u * ihw;
  float s = 1.0f - z * z;
  return s > 0.0f ? expf(beta * (sqrtf(s) - 1.0f)) : 0.0f;
}

// Shared-memory layout of k_asy_spread (byte offsets, each region 16-byte aligned); the
// host sizes the launch with the same function.
struct SpreadSmem {
  size_t win, wc, ph, u, rho, c, l0, total;
};
__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }
template <typename T>
__host__ __device__ inline SpreadSmem spread_smem(int W, int VCTA, int NLP, int BT, bool windowed) {
  SpreadSmem L{};
  size_t c2 = 2 * sizeof(T);
  L.win = 0;
  L.wc = align16(L.win + (windowed ? (size_t)spread_window(W) * (VCTA + 1) * c2 : 0));
  L.ph = align16(L.wc + (size_t)kSpreadChunk * W * c2);
  L.u = align16(L.ph + (size_t)kSpreadChunk * 16);
  L.rho = align16(L.u + (size_t)kSpreadChunk * 8);
  L.c = align16(L.rho + (size_t)kSpreadChunk * NLP * sizeof(T));
  L.l0 = align16(L.c + (size_t)BT * (kSpreadChunk + 1) * sizeof(T));
  L.total = align16(L.l0 + (size_t)kSpreadChunk * 4);
  return L;
}

// Plan-time tables: 1/psi-hat(2 pi l / n2) for each box cell l, and
// exp(i (phi + k C)) / psi-hat((k - D) h) for each box target.
__global__ void k_asy_setup_cells(const AsyBoxD* __restrict__ boxes, AsyConst P,
                                  double* __restrict__ corr) {
  const AsyBoxD bx = boxes[blockIdx.y];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * bx.half + 1; c += gridDim.x * blockDim.x) {
    int l = c - bx.half;
    corr[bx.corr_off + c] = 1.0 / es_hat(P, 2.0 * M_PI * (double)l / (double)bx.n2);
  }
}

__global__ void k_asy_setup_targets(const double* __restrict__ ws, const AsyBoxD* __restrict__ boxes,
                                    AsyConst P, double2* __restrict__ post) {
  const AsyBoxD bx = boxes[blockIdx.y];
  const int ni = bx.i1 - bx.i0 + 1;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ni; q += gridDim.x * blockDim.x) {
    double k = ws[bx.i0 + q];
    double inv_hat = 1.0 / es_hat(P, (k - bx.D) * bx.h);
    double sn, cn;
    sincos(k * bx.C, &sn, &cn);
    double er = cn * P.cos_phi - sn * P.sin_phi, ei = sn * P.cos_phi + cn * P.sin_phi;
    post[bx.post_off + q] = make_double2(er * inv_hat, ei * inv_hat);
  }
}

// Stage 1.  Thread (tl, lp) of the CTA owns term lp of column t0 + tl (vector
// v = t0 * NLP + tid).  Sources are sorted, so those whose kernel support starts at the
// same cell accumulate in registers; the accumulators go, once per cell change, to a
// shared window of the CTA's own cells (WINDOWED: mode-0 tiles, written with plain stores
// at the end) or straight to the pre-zeroed grid with atomic adds (mode-1 source chunks of
// dense boxes, where cell changes are rare).  The source phase exp(i D x) is folded into
// complex kernel weights staged once per source.
template <typename T, int W, bool WINDOWED>
__global__ void __launch_bounds__(256) k_asy_spread(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    typename Cplx<T>::type* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const SpreadItem* __restrict__ items, const double* __restrict__ corr, AsyConst P, int BT,
    int V_total) {
  using C2 = typename Cplx<T>::type;
  constexpr int SCP = kSpreadChunk + 1;  // padded row of the staged coefficients
  const SpreadItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int VCTA = blockDim.x;
  const int WP = VCTA + 1;  // padded window row
  const int tid = threadIdx.x;
  const int tl = tid / NLP, lp = tid - tl * NLP;
  const int t0 = blockIdx.y * BT;
  const int v0 = t0 * NLP;
  const int nv = min(VCTA, V_total - v0);  // valid vectors of this CTA
  const bool active = tid < nv;
  C2* gbox = grid + (size_t)bx.cell_off * (size_t)V_total;
  const int nc = it.ncell;

  if (WINDOWED && it.mode == 2) {  // zero padding of the FFT input: threads along cells
    for (int e = tid; e < nc * nv; e += VCTA) {
      int vv = e / nc, cell = e - vv * nc;
      gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = cmake<T>(0, 0);
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SpreadSmem L = spread_smem<T>(W, VCTA, NLP, BT, WINDOWED);
  C2* win = reinterpret_cast<C2*>(smem_raw + L.win);       // [WIN][WP]
  C2* s_wc = reinterpret_cast<C2*>(smem_raw + L.wc);       // [SCH][W]
  double2* s_ph = reinterpret_cast<double2*>(smem_raw + L.ph);  // [SCH]
  double* s_u = reinterpret_cast<double*>(smem_raw + L.u);  // [SCH]
  T* s_rho = reinterpret_cast<T*>(smem_raw + L.rho);        // [SCH][NLP]
  T* s_c = reinterpret_cast<T*>(smem_raw + L.c);            // [BT][SCP]
  int* s_l0 = reinterpret_cast<int*>(smem_raw + L.l0);      // [SCH]

  if (WINDOWED)
    for (int cell = 0; cell < nc; ++cell) win[cell * WP + tid] = cmake<T>(0, 0);
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;
  C2 acc[W];
#pragma unroll
  for (int q = 0; q < W; ++q) acc[q] = cmake<T>(0, 0);
  int cur = INT_MIN;

  auto flush = [&](int c0) {
    if (WINDOWED) {
#pragma unroll
      for (int q = 0; q < W; ++q) {
        int cell = c0 + q - it.l_start;
        if (cell >= 0 && cell < nc) {
          C2 w2 = win[cell * WP + tid];
          w2.x += acc[q].x;
          w2.y += acc[q].y;
          win[cell * WP + tid] = w2;
        }
        acc[q] = cmake<T>(0, 0);
      }
    } else {
#pragma unroll
      for (int q = 0; q < W; ++q) {
        int l = c0 + q;
        if (active && l >= -bx.half && l <= bx.half && (acc[q].x != (T)0 || acc[q].y != (T)0)) {
          T c = (T)corr[bx.corr_off + l + bx.half];
          int idx = l < 0 ? l + bx.n2 : l;
          T* dst = reinterpret_cast<T*>(gbox + (size_t)(v0 + tid) * bx.n2 + idx);
          atomicAdd(dst, acc[q].x * c);
          atomicAdd(dst + 1, acc[q].y * c);
        }
        acc[q] = cmake<T>(0, 0);
      }
    }
  };

  for (int s0 = it.js; s0 < it.je; s0 += kSpreadChunk) {
    const int ns = min(kSpreadChunk, it.je - s0);
    __syncthreads();  // previous round's staging fully consumed
    // Per-source quantities, spread over all threads of the CTA.
    for (int s = tid; s < ns; s += VCTA) {
      double r = rs[s0 + s];
      double x = r - bx.C;
      double u = x / bx.h;
      s_u[s] = u;
      s_l0[s] = (int)ceil(u - 0.5 * W);
      double sn, cn;
      sincos(bx.D * x, &sn, &cn);
      s_ph[s] = make_double2(cn, sn);
    }
    for (int e = tid; e < ns * NLP; e += VCTA) {
      int s = e / NLP, q = e - s * NLP;
      double r = rs[s0 + s];
      double rho = 0.0;
      if (r > 0.0) {  // (rref / r)^(q + 1/2); sources at r = 0 contribute nothing
        double ir = bx.rref / r;
        rho = sqrt(ir);
        for (int z = 0; z < q; ++z) rho *= ir;
      }
      s_rho[e] = (T)rho;
    }
    for (int e = tid; e < ns * BT; e += VCTA) {
      int tt = e / ns, s = e - tt * ns;
      s_c[tt * SCP + s] = (T)((t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + s0 + s] : 0.0);
    }
    __syncthreads();
    for (int e = tid; e < ns * W; e += VCTA) {
      int s = e / W, q = e - s * W;
      T w = es_kernel_t((T)((double)(s_l0[s] + q) - s_u[s]), ihw, beta);
      double2 ph = s_ph[s];
      s_wc[e] = cmake<T>(w * (T)ph.x, w * (T)ph.y);
    }
    __syncthreads();
    for (int s = 0; s < ns; ++s) {
      int l0 = s_l0[s];
      if (l0 != cur) {
        if (cur != INT_MIN) flush(cur);
        cur = l0;
      }
      T a = s_c[tl * SCP + s] * s_rho[s * NLP + lp];
#pragma unroll
      for (int q = 0; q < W; ++q) {
        C2 wc = s_wc[s * W + q];
        acc[q].x = fma(wc.x, a, acc[q].x);
        acc[q].y = fma(wc.y, a, acc[q].y);
      }
    }
  }
  if (cur != INT_MIN) flush(cur);
  if (!WINDOWED) return;
  __syncthreads();
  // Transposed write-out of the CTA's own cells: consecutive threads take consecutive
  // cells of one vector.
  for (int e = tid; e < nc * nv; e += VCTA) {
    int vv = e / nc, cell = e - vv * nc;
    C2 val = win[cell * WP + vv];
    T c = (T)corr[bx.corr_off + it.l_start + cell + bx.half];
    gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = cmake<T>(val.x * c, val.y * c);
  }
}

// Stage 3.  Thread tid owns term lp = tid % NLP of the VPT columns t0 + tid / NLP + u BTH
// and interpolates them at each target, keeping a sliding window of W grid values per
// vector in registers; the NLP terms of a column are summed (in FP64) through padded
// shared memory and added to g.
template <typename T, int W, int VPT>
__global__ void __launch_bounds__(256) k_asy_interp(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const typename Cplx<T>::type* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const InterpItem* __restrict__ items, const double2* __restrict__ post, AsyConst P, int BTH,
    int V_total, double sgn) {
  using C2 = typename Cplx<T>::type;
  const InterpItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int VCTA = blockDim.x;
  const int VV = VCTA * VPT;
  const int YP = VV + 1;  // padded row of the per-target results
  const int BT = BTH * VPT;
  const int tid = threadIdx.x;
  const int tl = tid / NLP, lp = tid - tl * NLP;
  const int t0 = blockIdx.y * BT;
  bool active[VPT];
#pragma unroll
  for (int u = 0; u < VPT; ++u) active[u] = t0 + tl + u * BTH < B;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s_mu = reinterpret_cast<double2*>(smem_raw);          // [KC][NLP]
  double* s_y = reinterpret_cast<double*>(s_mu + kInterpChunk * NLP);  // [KC][YP]
  T* s_wt = reinterpret_cast<T*>(s_y + kInterpChunk * YP);       // [KC][W]
  int* s_q0 = reinterpret_cast<int*>(s_wt + kInterpChunk * W);   // [KC]

  const int n2 = bx.n2;
  const C2* row[VPT];
#pragma unroll
  for (int u = 0; u < VPT; ++u)
    row[u] = grid + (size_t)bx.cell_off * (size_t)V_total + (size_t)(t0 * NLP + tid + u * VCTA) * (size_t)n2;
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;
  const double u_scale = bx.h * (double)n2 / (2.0 * M_PI);
  C2 g[VPT][W];
  int gq = INT_MIN;

  for (int k0 = it.ks; k0 < it.ke; k0 += kInterpChunk) {
    const int nk = min(kInterpChunk, it.ke - k0);
    for (int e = tid; e < nk * W; e += VCTA) {
      int kk = e / W, q = e - kk * W;
      double u = (ws[k0 + kk] - bx.D) * u_scale;
      int q0 = (int)ceil(u - 0.5 * W);
      if (q == 0) s_q0[kk] = q0;
      s_wt[kk * W + q] = es_kernel_t((T)(u - (double)(q0 + q)), ihw, beta);
    }
    for (int e = tid; e < nk * NLP; e += VCTA) {
      int kk = e / NLP, q = e - kk * NLP;
      double k = ws[k0 + kk];
      double2 ps = post[bx.post_off + (k0 + kk - bx.i0)];
      // coef_q (k rref)^{-(q + 1/2)}
      double kr = k * bx.rref;
      double pw = 1.0 / sqrt(kr), ik = 1.0 / kr;
      for (int e2 = 0; e2 < q; ++e2) pw *= ik;
      double sc = P.coef[q] * pw;
      double mr = sc * ps.x, mi = sc * ps.y;
      s_mu[kk * NLP + q] = (q & 1) ? make_double2(-mi, mr) : make_double2(mr, mi);
    }
    __syncthreads();
    for (int kk = 0; kk < nk; ++kk) {
      int q0 = s_q0[kk];
      if (q0 != gq) {
        if (q0 == gq + 1) {
          int idx = q0 + W - 1;
          idx = idx < 0 ? idx + n2 : (idx >= n2 ? idx - n2 : idx);
#pragma unroll
          for (int u = 0; u < VPT; ++u) {
#pragma unroll
            for (int q = 0; q < W - 1; ++q) g[u][q] = g[u][q + 1];
            g[u][W - 1] = active[u] ? row[u][idx] : cmake<T>(0, 0);
          }
        } else {
#pragma unroll
          for (int q = 0; q < W; ++q) {
            int idx = q0 + q;
            idx = idx < 0 ? idx + n2 : (idx >= n2 ? idx - n2 : idx);
#pragma unroll
            for (int u = 0; u < VPT; ++u) g[u][q] = active[u] ? row[u][idx] : cmake<T>(0, 0);
          }
        }
        gq = q0;
      }
      T tr[VPT], ti[VPT];
#pragma unroll
      for (int u = 0; u < VPT; ++u) tr[u] = ti[u] = (T)0;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        T w = s_wt[kk * W + q];
#pragma unroll
        for (int u = 0; u < VPT; ++u) {
          tr[u] = fma(w, g[u][q].x, tr[u]);
          ti[u] = fma(w, g[u][q].y, ti[u]);
        }
      }
      double2 mu = s_mu[kk * NLP + lp];
#pragma unroll
      for (int u = 0; u < VPT; ++u)
        s_y[kk * YP + tid + u * VCTA] = mu.x * (double)tr[u] - mu.y * (double)ti[u];
    }
    __syncthreads();
    for (int e = tid; e < nk * BT; e += VCTA) {
      int tt = e / nk, kk = e - tt * nk;
      if (t0 + tt < B) {
        // column tt lives in vectors (tt % BTH) * NLP + q + (tt / BTH) * VCTA
        const int base = (tt % BTH) * NLP + (tt / BTH) * VCTA;
        double s = 0.0;
        for (int q = 0; q < NLP; ++q) s += s_y[kk * YP + base + q];
        atomicAdd(&gs[(size_t)(t0 + tt) * ld_gs + k0 + kk], sgn * s);
      }
    }
    __syncthreads();
  }
}

}  // namespace hankel
