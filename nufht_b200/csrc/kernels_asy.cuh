// Asymptotic boxes: Hankel's large-argument expansion (src/expansions.c:483-559) evaluated
// with a type-3 NUFFT written for this executor.
//
// For one box with sources r in [C - X, C + X] and targets k in [D - S, D + S] every one
// of the NLP = 2 (K + 1) expansion terms and every batch column t is a transform
//   F_{lp,t}(k) = sum_j c[j,t] r_j^{-(lp+1/2)} exp(i k r_j),   lp = 2l + p.
// Stage 1 spreads a_j exp(i D (r_j - C)) with the exponential-of-semicircle kernel psi onto
// cells l h, h = pi / (sigma S); stage 2 divides by psi-hat, zero-pads to
// n2 >= sigma (2 half + 1) and runs a backward FFT (cuFFT); stage 3 interpolates at
// u = (k - D) h n2 / (2 pi) and multiplies by exp(i (phi + k C)) / psi-hat((k - D) h) and
// by the expansion's target factor sqrt(2/pi) (-1)^l a_lp k^{-(lp+1/2)}.  Terms with
// p = 0 add Re, p = 1 subtract Im (src/expansions.c:520-557); both are written as
// Re(mu F) with mu rotated by i for p = 1.
//
// Workspace layout: box b owns n2 * V contiguous complex values, vector v = t * NLP + lp
// at offset cell_off * V + v * n2 (one contiguous FFT input per vector).
#pragma once

#include <climits>

#include "kernels_common.cuh"

namespace hankel {

constexpr int kSpreadTile = 16;     // cells owned by one mode-0 spreading CTA
constexpr int kSpreadChunk = 32;    // sources staged in shared memory per round
constexpr int kChunkSources = 2048; // sources per mode-1 work item, at most
constexpr int kTileMaxSources = 4096;
constexpr int kInterpTile = 128;    // targets per interpolation CTA
constexpr int kInterpChunk = 32;    // targets per shared-memory round

// Window capacity (cells) of a spreading CTA for kernel width W.
__host__ __device__ constexpr int spread_window(int W) { return W + 8 > kSpreadTile ? W + 8 : kSpreadTile; }

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

// Stage 1.  Thread (tl, lp) of the CTA owns expansion term lp of column t0 + tl, i.e.
// vector v = t0 * NLP + tid.  Sources are sorted, so those whose kernel support starts at
// the same cell accumulate in registers and reach the shared window once per cell change.
// The window rows are padded by one element so that the transposed write-out (threads
// along cells) is free of bank conflicts.
template <int W>
__global__ void __launch_bounds__(256) k_asy_spread(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    double2* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const SpreadItem* __restrict__ items, const double* __restrict__ corr, AsyConst P, int BT,
    int V_total) {
  constexpr int WIN = spread_window(W);
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
  const int nv = min(VCTA, V_total - v0);  // vectors of this CTA
  const bool active = tid < nv;
  double2* gbox = grid + (size_t)bx.cell_off * (size_t)V_total;
  const int nc = it.ncell;

  if (it.mode == 2) {  // zero padding of the FFT input: threads along cells
    for (int e = tid; e < nc * nv; e += VCTA) {
      int vv = e / nc, cell = e - vv * nc;
      gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = make_double2(0.0, 0.0);
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* win = reinterpret_cast<double2*>(smem_raw);                 // [WIN][WP]
  double* s_w = reinterpret_cast<double*>(win + WIN * WP);            // [SCH][W]
  double2* s_ph = reinterpret_cast<double2*>(s_w + kSpreadChunk * W); // [SCH]
  double* s_rho = reinterpret_cast<double*>(s_ph + kSpreadChunk);     // [SCH][NLP]
  double* s_c = s_rho + kSpreadChunk * NLP;                            // [BT][SCP]
  double* s_u = s_c + BT * SCP;                                        // [SCH]
  int* s_l0 = reinterpret_cast<int*>(s_u + kSpreadChunk);              // [SCH]

  for (int cell = 0; cell < nc; ++cell) win[cell * WP + tid] = make_double2(0.0, 0.0);
  const double ihw = 2.0 / (double)W;
  double2 acc[W];
#pragma unroll
  for (int q = 0; q < W; ++q) acc[q] = make_double2(0.0, 0.0);
  int cur = INT_MIN;

  auto flush = [&](int c0) {
#pragma unroll
    for (int q = 0; q < W; ++q) {
      int cell = c0 + q - it.l_start;
      if (cell >= 0 && cell < nc) {
        double2 w2 = win[cell * WP + tid];
        w2.x += acc[q].x;
        w2.y += acc[q].y;
        win[cell * WP + tid] = w2;
      }
      acc[q] = make_double2(0.0, 0.0);
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
      double rho = 1.0 / sqrt(r), ir = 1.0 / r;
      for (int z = 0; z < q; ++z) rho *= ir;
      s_rho[e] = rho;
    }
    for (int e = tid; e < ns * BT; e += VCTA) {
      int tt = e / ns, s = e - tt * ns;
      s_c[tt * SCP + s] = (t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + s0 + s] : 0.0;
    }
    __syncthreads();
    for (int e = tid; e < ns * W; e += VCTA) {
      int s = e / W, q = e - s * W;
      s_w[e] = es_kernel((double)(s_l0[s] + q) - s_u[s], ihw, P.beta);
    }
    __syncthreads();
    if (active) {
      for (int s = 0; s < ns; ++s) {
        int l0 = s_l0[s];
        if (l0 != cur) {
          if (cur != INT_MIN) flush(cur);
          cur = l0;
        }
        double a = s_c[tl * SCP + s] * s_rho[s * NLP + lp];
        double2 ph = s_ph[s];
        double ar = a * ph.x, ai = a * ph.y;
#pragma unroll
        for (int q = 0; q < W; ++q) {
          double w = s_w[s * W + q];
          acc[q].x = fma(w, ar, acc[q].x);
          acc[q].y = fma(w, ai, acc[q].y);
        }
      }
    }
  }
  if (active && cur != INT_MIN) flush(cur);
  __syncthreads();
  // Transposed write-out: consecutive threads take consecutive cells of one vector.
  if (it.mode == 0) {
    // Plain stores: this CTA owns cells [l_start, l_start + ncell) of the box.
    for (int e = tid; e < nc * nv; e += VCTA) {
      int vv = e / nc, cell = e - vv * nc;
      double2 val = win[cell * WP + vv];
      double c = corr[bx.corr_off + it.l_start + cell + bx.half];
      gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = make_double2(val.x * c, val.y * c);
    }
  } else {
    // Atomic adds into the (pre-zeroed) grid of a dense box.
    for (int e = tid; e < nc * nv; e += VCTA) {
      int vv = e / nc, cell = e - vv * nc;
      int l = it.l_start + cell;
      if (l < -bx.half || l > bx.half) continue;
      double2 val = win[cell * WP + vv];
      if (val.x == 0.0 && val.y == 0.0) continue;
      double c = corr[bx.corr_off + l + bx.half];
      int idx = l < 0 ? l + bx.n2 : l;
      double* dst = reinterpret_cast<double*>(gbox + (size_t)(v0 + vv) * bx.n2 + idx);
      atomicAdd(dst, val.x * c);
      atomicAdd(dst + 1, val.y * c);
    }
  }
}

// Stage 3.  Thread (tl, lp) interpolates vector v = t0 * NLP + tid at each target, keeping
// a sliding window of W grid values in registers; the NLP terms of a column are summed
// through shared memory and added to g.
template <int W>
__global__ void __launch_bounds__(256) k_asy_interp(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const double2* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const InterpItem* __restrict__ items, const double2* __restrict__ post, AsyConst P, int BT,
    int V_total, double sgn) {
  const InterpItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int VCTA = blockDim.x;
  const int tid = threadIdx.x;
  const int tl = tid / NLP, lp = tid - tl * NLP;
  const int t0 = blockIdx.y * BT;
  const bool active = (tl < BT) && (t0 + tl < B);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s_mu = reinterpret_cast<double2*>(smem_raw);                // [KC][NLP]
  double* s_wt = reinterpret_cast<double*>(s_mu + kInterpChunk * NLP); // [KC][W]
  double* s_y = s_wt + kInterpChunk * W;                                // [KC][VCTA]
  int* s_q0 = reinterpret_cast<int*>(s_y + kInterpChunk * VCTA);        // [KC]

  const int n2 = bx.n2;
  const double2* row =
      grid + (size_t)bx.cell_off * (size_t)V_total + (size_t)(t0 * NLP + tid) * (size_t)n2;
  const double ihw = 2.0 / (double)W;
  const double u_scale = bx.h * (double)n2 / (2.0 * M_PI);
  double2 g[W];
  int gq = INT_MIN;

  for (int k0 = it.ks; k0 < it.ke; k0 += kInterpChunk) {
    const int nk = min(kInterpChunk, it.ke - k0);
    for (int e = tid; e < nk * W; e += VCTA) {
      int kk = e / W, q = e - kk * W;
      double u = (ws[k0 + kk] - bx.D) * u_scale;
      int q0 = (int)ceil(u - 0.5 * W);
      if (q == 0) s_q0[kk] = q0;
      s_wt[kk * W + q] = es_kernel(u - (double)(q0 + q), ihw, P.beta);
    }
    for (int e = tid; e < nk * NLP; e += VCTA) {
      int kk = e / NLP, q = e - kk * NLP;
      double k = ws[k0 + kk];
      double2 ps = post[bx.post_off + (k0 + kk - bx.i0)];
      // coef_q k^{-(q + 1/2)}
      double pw = 1.0 / sqrt(k), ik = 1.0 / k;
      for (int e2 = 0; e2 < q; ++e2) pw *= ik;
      double sc = P.coef[q] * pw;
      double mr = sc * ps.x, mi = sc * ps.y;
      s_mu[kk * NLP + q] = (q & 1) ? make_double2(-mi, mr) : make_double2(mr, mi);
    }
    __syncthreads();
    if (active) {
      for (int kk = 0; kk < nk; ++kk) {
        int q0 = s_q0[kk];
        if (q0 != gq) {
          if (q0 == gq + 1) {
#pragma unroll
            for (int q = 0; q < W - 1; ++q) g[q] = g[q + 1];
            int idx = q0 + W - 1;
            idx = idx < 0 ? idx + n2 : (idx >= n2 ? idx - n2 : idx);
            g[W - 1] = row[idx];
          } else {
#pragma unroll
            for (int q = 0; q < W; ++q) {
              int idx = q0 + q;
              idx = idx < 0 ? idx + n2 : (idx >= n2 ? idx - n2 : idx);
              g[q] = row[idx];
            }
          }
          gq = q0;
        }
        double tr = 0.0, ti = 0.0;
#pragma unroll
        for (int q = 0; q < W; ++q) {
          double w = s_wt[kk * W + q];
          tr = fma(w, g[q].x, tr);
          ti = fma(w, g[q].y, ti);
        }
        double2 mu = s_mu[kk * NLP + lp];
        s_y[kk * VCTA + tid] = mu.x * tr - mu.y * ti;
      }
    }
    __syncthreads();
    for (int e = tid; e < nk * BT; e += VCTA) {
      int tt = e / nk, kk = e - tt * nk;
      if (t0 + tt < B) {
        double s = 0.0;
        for (int q = 0; q < NLP; ++q) s += s_y[kk * VCTA + tt * NLP + q];
        atomicAdd(&gs[(size_t)(t0 + tt) * ld_gs + k0 + kk], sgn * s);
      }
    }
    __syncthreads();
  }
}

}  // namespace hankel
