// GPU executor of the batched NUFHT on B200 (sm_100a).
//
// A device plan holds device copies of the sorted grids rs (sources) and ws (targets),
// the reference's box partition turned into flat work lists, and a device workspace.
// One transform g = H c runs as a fixed sequence of kernels on one stream:
//
//   local boxes      k_loc_proj   -> k_loc_reduce -> k_loc_eval
//   asymptotic boxes k_asy_spread -> cuFFT (Z2Z, one batched call per FFT length)
//                                 -> k_asy_interp
//   direct boxes     k_dir
//
// The asymptotic boxes evaluate Hankel's expansion (src/expansions.c:483-559) with a
// type-3 NUFFT written here: all 2(K_asy+1) expansion terms and all batch columns of a
// box share one spreading pass and one interpolation pass.  Spreading and interpolation
// use the exponential-of-semicircle kernel of Barnett, Magland & af Klinteberg (2019);
// the inner uniform transform is cuFFT.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "bessel.cuh"
#include "executor.h"

namespace hankel {

std::atomic<long long> g_launch_counter{0};

namespace {

constexpr int kSigma = 2;         // oversampling of both type-3 stages
constexpr int kSpreadTile = 16;   // grid cells owned by one spreading CTA
constexpr int kSpreadChunk = 32;  // sources staged in shared memory at a time
constexpr int kInterpTile = 128;  // targets per interpolation CTA
constexpr int kInterpChunk = 8;   // targets per shared-memory round
constexpr int kDirTargets = 128;  // targets per direct CTA (one per thread)
constexpr int kDirSources = 1024; // sources per direct work item
constexpr int kDirChunk = 64;     // sources staged at a time
constexpr int kLocSources = 2048; // sources per projection work item
constexpr int kLocChunk = 64;
constexpr int kLocTargets = 128;

#define NUFHT_CUDA_TRY(expr)                                                          \
  do {                                                                                \
    cudaError_t _e = (expr);                                                          \
    if (_e != cudaSuccess) {                                                          \
      std::fprintf(stderr, "nufht_b200: %s failed: %s\n", #expr, cudaGetErrorString(_e)); \
      return NUFHT_E_CUDA;                                                            \
    }                                                                                 \
  } while (0)

#define NUFHT_LAUNCH_CHECK()                                                          \
  do {                                                                                \
    g_launch_counter.fetch_add(1, std::memory_order_relaxed);                         \
    cudaError_t _e = cudaGetLastError();                                              \
    if (_e != cudaSuccess) {                                                          \
      std::fprintf(stderr, "nufht_b200: kernel launch failed: %s\n", cudaGetErrorString(_e)); \
      return NUFHT_E_CUDA;                                                            \
    }                                                                                 \
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

// ----------------------------------------------------------------------------------
// Asymptotic boxes, stage 1: spread.  One CTA owns kSpreadTile consecutive grid cells of
// one box for BT batch columns; thread (tl, lp) owns expansion term lp of column t0+tl.
// Sources arrive sorted, so all sources whose kernel support starts at the same cell are
// accumulated in registers and flushed to the shared window once per cell change.
// ----------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) k_asy_spread(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    double2* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const SpreadItem* __restrict__ items, AsyConst P, int BT, int V_total) {
  const SpreadItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int VCTA = blockDim.x;
  const int tid = threadIdx.x;
  const int tl = tid / NLP, lp = tid - tl * NLP;
  const int t0 = blockIdx.y * BT;
  const bool active = (tl < BT) && (t0 + tl < B);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* win = reinterpret_cast<double2*>(smem_raw);                  // [TC][VCTA]
  double* s_w = reinterpret_cast<double*>(win + kSpreadTile * VCTA);   // [SCH][W]
  double2* s_ph = reinterpret_cast<double2*>(s_w + kSpreadChunk * W);  // [SCH]
  double* s_rho = reinterpret_cast<double*>(s_ph + kSpreadChunk);      // [SCH][NLP]
  double* s_c = s_rho + kSpreadChunk * NLP;                             // [SCH][BT]
  double* s_corr = s_c + kSpreadChunk * BT;                             // [TC]
  int* s_l0 = reinterpret_cast<int*>(s_corr + kSpreadTile);             // [SCH]

  for (int e = tid; e < kSpreadTile * VCTA; e += VCTA) win[e] = make_double2(0.0, 0.0);
  if (tid < it.ncell) {
    s_corr[tid] = it.padding ? 0.0
                             : 1.0 / es_hat(P, 2.0 * M_PI * (double)(it.l_start + tid) /
                                                   (double)bx.n2);
  }
  const double inv_h = 1.0 / bx.h;
  const double ihw = 2.0 / (double)W;
  double2 acc[W];
#pragma unroll
  for (int q = 0; q < W; ++q) acc[q] = make_double2(0.0, 0.0);
  int cur = INT_MIN;
  __syncthreads();

  auto flush = [&](int c0) {
#pragma unroll
    for (int q = 0; q < W; ++q) {
      int cell = c0 + q - it.l_start;
      if (cell >= 0 && cell < it.ncell) {
        double2 v = win[cell * VCTA + tid];
        v.x += acc[q].x;
        v.y += acc[q].y;
        win[cell * VCTA + tid] = v;
      }
      acc[q] = make_double2(0.0, 0.0);
    }
  };

  for (int s0 = it.js; s0 < it.je; s0 += kSpreadChunk) {
    const int ns = min(kSpreadChunk, it.je - s0);
    for (int s = tid; s < ns; s += VCTA) {
      double r = rs[s0 + s];
      double x = r - bx.C;
      double u = x / bx.h;
      int l0 = (int)ceil(u - 0.5 * W);
      s_l0[s] = l0;
#pragma unroll
      for (int q = 0; q < W; ++q) s_w[s * W + q] = es_kernel((double)(l0 + q) - u, ihw, P.beta);
      double sn, cn;
      sincos(bx.D * x, &sn, &cn);
      s_ph[s] = make_double2(cn, sn);
      double rho = 1.0 / sqrt(r), ir = 1.0 / r;
      for (int q = 0; q < NLP; ++q) {
        s_rho[s * NLP + q] = rho;
        rho *= ir;
      }
    }
    for (int e = tid; e < ns * BT; e += VCTA) {
      int tt = e / ns, s = e - tt * ns;
      s_c[s * BT + tt] = (t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + s0 + s] : 0.0;
    }
    __syncthreads();
    if (active) {
      for (int s = 0; s < ns; ++s) {
        int l0 = s_l0[s];
        if (l0 != cur) {
          if (cur != INT_MIN) flush(cur);
          cur = l0;
        }
        double a = s_c[s * BT + tl] * s_rho[s * NLP + lp];
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
    __syncthreads();
  }
  if (active && cur != INT_MIN) flush(cur);
  __syncthreads();
  (void)inv_h;
  // Write the tile, deconvolved for the second stage, to the FFT input.
  const size_t box_base = (size_t)bx.cell_off * (size_t)V_total;
  const int nc = it.ncell;
  for (int e = tid; e < nc * VCTA; e += VCTA) {
    int vv = e / nc, cell = e - vv * nc;
    int v = t0 * NLP + vv;
    if (v < V_total && (vv / NLP) < BT) {
      double2 val = win[cell * VCTA + vv];
      double c = s_corr[cell];
      grid[box_base + (size_t)v * bx.n2 + it.fft_start + cell] = make_double2(val.x * c, val.y * c);
    }
  }
}

// ----------------------------------------------------------------------------------
// Asymptotic boxes, stage 3: interpolate the FFT output at the targets and add the
// phase-rotated, scaled expansion terms to g.
// ----------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) k_asy_interp(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const double2* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const InterpItem* __restrict__ items, AsyConst P, int BT, int V_total, double sgn) {
  const InterpItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int VCTA = blockDim.x;
  const int tid = threadIdx.x;
  const int tl = tid / NLP, lp = tid - tl * NLP;
  const int t0 = blockIdx.y * BT;
  const bool active = (tl < BT) && (t0 + tl < B);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s_mu = reinterpret_cast<double2*>(smem_raw);          // [KC][NLP]
  double* s_wt = reinterpret_cast<double*>(s_mu + kInterpChunk * NLP);  // [KC][W]
  double* s_y = s_wt + kInterpChunk * W;                          // [KC][VCTA]
  int* s_q0 = reinterpret_cast<int*>(s_y + kInterpChunk * VCTA);  // [KC]

  const int n2 = bx.n2;
  const double2* row =
      grid + (size_t)bx.cell_off * (size_t)V_total + (size_t)(t0 * NLP + tid) * (size_t)n2;
  const double ihw = 2.0 / (double)W;
  const double u_scale = bx.h * (double)n2 / (2.0 * M_PI);
  double2 g[W];
  int gq = INT_MIN;

  for (int k0 = it.ks; k0 < it.ke; k0 += kInterpChunk) {
    const int nk = min(kInterpChunk, it.ke - k0);
    if (tid < nk) {
      double k = ws[k0 + tid];
      double th = (k - bx.D) * bx.h;
      double u = (k - bx.D) * u_scale;
      int q0 = (int)ceil(u - 0.5 * W);
      s_q0[tid] = q0;
#pragma unroll
      for (int q = 0; q < W; ++q) s_wt[tid * W + q] = es_kernel(u - (double)(q0 + q), ihw, P.beta);
      double inv_hat = 1.0 / es_hat(P, th);
      double sn, cn;
      sincos(k * bx.C, &sn, &cn);
      // e^{i(phi + k C)}
      double er = cn * P.cos_phi - sn * P.sin_phi, ei = sn * P.cos_phi + cn * P.sin_phi;
      double pw = inv_hat / sqrt(k), ik = 1.0 / k;
      for (int q = 0; q < NLP; ++q) {
        double sc = P.coef[q] * pw;
        double mr = sc * er, mi = sc * ei;
        // odd terms contribute -Im(mu T) = Re(i mu T)
        s_mu[tid * NLP + q] = (q & 1) ? make_double2(-mi, mr) : make_double2(mr, mi);
        pw *= ik;
      }
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
            idx %= n2;
            if (idx < 0) idx += n2;
            g[W - 1] = row[idx];
          } else {
#pragma unroll
            for (int q = 0; q < W; ++q) {
              int idx = (q0 + q) % n2;
              if (idx < 0) idx += n2;
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

// ----------------------------------------------------------------------------------
// Direct boxes: g[i,t] += sum_j c[j,t] J_nu(k_i r_j), one Bessel value per (i, j) pair
// reused across BT columns held in registers (src/expansions.c:78-97).
// ----------------------------------------------------------------------------------
template <int BT>
__global__ void __launch_bounds__(kDirTargets) k_dir(
    const double* __restrict__ rs, const double* __restrict__ ws, const double* __restrict__ cs,
    int ld_cs, double* __restrict__ gs, int ld_gs, int B, const DirItem* __restrict__ items,
    int nu2, double sgn) {
  const DirItem it = items[blockIdx.x];
  const int t0 = blockIdx.y * BT;
  const int tid = threadIdx.x;
  const bool valid = tid < it.ni;
  const double k = valid ? ws[it.i0 + tid] : 0.0;
  __shared__ double s_r[kDirChunk];
  __shared__ double s_c[kDirChunk * BT];
  double acc[BT];
#pragma unroll
  for (int q = 0; q < BT; ++q) acc[q] = 0.0;
  for (int s0 = 0; s0 < it.nj; s0 += kDirChunk) {
    const int ns = min(kDirChunk, it.nj - s0);
    for (int s = tid; s < ns; s += blockDim.x) s_r[s] = rs[it.j0 + s0 + s];
    for (int e = tid; e < kDirChunk * BT; e += blockDim.x) {
      int tt = e / kDirChunk, s = e - tt * kDirChunk;
      s_c[s * BT + tt] =
          (s < ns && t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + it.j0 + s0 + s] : 0.0;
    }
    __syncthreads();
    if (valid) {
      for (int s = 0; s < ns; ++s) {
        double J = bessel_j(nu2, k * s_r[s]);
#pragma unroll
        for (int q = 0; q < BT; ++q) acc[q] = fma(s_c[s * BT + q], J, acc[q]);
      }
    }
    __syncthreads();
  }
  if (valid) {
#pragma unroll
    for (int q = 0; q < BT; ++q)
      if (t0 + q < B) atomicAdd(&gs[(size_t)(t0 + q) * ld_gs + it.i0 + tid], sgn * acc[q]);
  }
}

// ----------------------------------------------------------------------------------
// Local boxes (src/expansions.c:212-337).
// k_loc_proj: partial Chebyshev projections C[l,t] = sum_j T_l(r_j / r_end) c[j,t] over
// one source chunk, with T_l = eps_l T_{2l} (even nu) or 2 T_{2l+1} (odd nu), evaluated
// by the Chebyshev three-term recurrence.
// ----------------------------------------------------------------------------------
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
  const double inv_end = 1.0 / bx.r_end;
  for (int s0 = 0; s0 < it.nj; s0 += kLocChunk) {
    const int ns = min(kLocChunk, it.nj - s0);
    for (int s = tid; s < kLocChunk; s += blockDim.x) {
      if (s < ns) {
        double x = rs[it.j0 + s0 + s] * inv_end;
        x = fmin(fmax(x, -1.0), 1.0);
        double tm1 = 1.0, tc = x;  // T_0, T_1
        int l = 0;
        int order = 0;
        // Walk T_n upward, storing the orders used by the expansion.
        double Tn = 1.0;
        for (int nn = 0; l < KL1; ++nn) {
          if (nn == 0) Tn = 1.0;
          else if (nn == 1) Tn = x;
          else {
            double tn = 2.0 * x * tc - tm1;
            tm1 = tc;
            tc = tn;
            Tn = tn;
          }
          order = odd ? 2 * l + 1 : 2 * l;
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

// Bessel products b_l(z) = J_{l0+odd+l}(z) J_{|l-l0|}(z) (-1)^{max(l-l0,0)}, z = k r_end / 2,
// then g[i,t] += sum_l b_l C[l,t]  (src/expansions.c:280-336).
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
  // b_l overwrites J[l] in place is not possible (indices overlap); keep a second array.
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

__global__ void k_besselj(int nu2, const double* __restrict__ x, double* __restrict__ out,
                          long count) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) out[e] = bessel_j(nu2, x[e]);
}

template <typename T>
int upload(const std::vector<T>& h, T** d) {
  *d = nullptr;
  if (h.empty()) return 0;
  NUFHT_CUDA_TRY(cudaMalloc((void**)d, h.size() * sizeof(T)));
  NUFHT_CUDA_TRY(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

int nice_fft_len(long long n) {
  // Smallest 2^a 3^b 5^c 7^d >= n.
  long long best = LLONG_MAX;
  for (long long p2 = 1; p2 < 4 * n + 16; p2 *= 2)
    for (long long p3 = p2; p3 < 4 * n + 16; p3 *= 3)
      for (long long p5 = p3; p5 < 4 * n + 16; p5 *= 5)
        for (long long p7 = p5; p7 < 4 * n + 16; p7 *= 7)
          if (p7 >= n && p7 < best) best = p7;
  return (int)best;
}

void gauss_legendre(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

double host_es(double u, int W, double beta) {
  double z = 2.0 * u / W;
  double s = 1.0 - z * z;
  return s > 0.0 ? std::exp(beta * (std::sqrt(s) - 1.0)) : 0.0;
}

}  // namespace

// ------------------------------------------------------------------------------------
// Plan construction.
// ------------------------------------------------------------------------------------
int spread_width_for_tol(double tol) {
  int w = (int)std::ceil(std::log10(1.0 / tol)) + 1;
  return std::min(std::max(w, 2), 16);
}

void DevicePlan::build_lists() {
  const double* rs = h_rs.data();
  const double* ws = h_ws.data();
  // ---- local boxes
  locb.clear(); proj.clear(); eval.clear();
  KL1 = P.K_loc + 1;
  for (size_t b = 0; b < loc_boxes.size(); ++b) {
    const HBox& hb = loc_boxes[b];
    LocBoxD d;
    d.i0 = hb.i0; d.ni = hb.i1 - hb.i0 + 1; d.j0 = hb.j0; d.nj = hb.j1 - hb.j0 + 1;
    d.r_end = rs[hb.j1];
    d.item0 = (int)proj.size();
    for (int j = hb.j0; j <= hb.j1; j += kLocSources)
      proj.push_back({(int)b, j, std::min(kLocSources, hb.j1 - j + 1)});
    d.nitems = (int)proj.size() - d.item0;
    for (int i = hb.i0; i <= hb.i1; i += kLocTargets)
      eval.push_back({(int)b, i, std::min(kLocTargets, hb.i1 - i + 1)});
    locb.push_back(d);
  }
  // ---- direct boxes
  dir.clear();
  for (const HBox& hb : dir_boxes)
    for (int i = hb.i0; i <= hb.i1; i += kDirTargets)
      for (int j = hb.j0; j <= hb.j1; j += kDirSources)
        dir.push_back({i, std::min(kDirTargets, hb.i1 - i + 1), j, std::min(kDirSources, hb.j1 - j + 1)});
  // ---- asymptotic boxes
  asyb.clear(); spread.clear(); interp.clear(); groups.clear();
  W = spread_width_for_tol(P.tol);
  const double beta = 2.30 * W;
  std::vector<AsyBoxD> tmp;
  for (const HBox& hb : asy_boxes) {
    AsyBoxD d;
    d.i0 = hb.i0; d.i1 = hb.i1; d.j0 = hb.j0; d.j1 = hb.j1;
    double rlo = rs[hb.j0], rhi = rs[hb.j1], klo = ws[hb.i0], khi = ws[hb.i1];
    d.C = 0.5 * (rlo + rhi);
    double X = 0.5 * (rhi - rlo);
    d.D = 0.5 * (klo + khi);
    double S = 0.5 * (khi - klo);
    double Smin = 1e-12 * std::max(std::fabs(d.D), 1.0);
    if (S < Smin) S = Smin;
    d.h = M_PI / ((double)kSigma * S);
    long long half = (long long)std::ceil(X / d.h + 0.5 * W);
    long long L1 = 2 * half + 1;
    d.half = (int)half;
    d.n2 = nice_fft_len(std::max<long long>((long long)kSigma * L1, 2 * kSpreadTile));
    tmp.push_back(d);
  }
  std::vector<int> order(tmp.size());
  for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tmp[a].n2 < tmp[b].n2; });
  long long off = 0;
  for (int q : order) {
    AsyBoxD d = tmp[q];
    d.cell_off = off;
    off += d.n2;
    if (groups.empty() || groups.back().n2 != d.n2)
      groups.push_back({d.n2, (int)asyb.size(), 0, d.cell_off});
    groups.back().nbox++;
    asyb.push_back(d);
  }
  total_cells = off;
  for (size_t b = 0; b < asyb.size(); ++b) {
    const AsyBoxD& d = asyb[b];
    auto l0_of = [&](int j) {
      double x = rs[j] - d.C;
      double u = x / d.h;
      return (long long)std::ceil(u - 0.5 * W);
    };
    // first source index in [j0, j1+1) with l0 >= lo
    auto first_ge = [&](long long lo) {
      int a = d.j0, c = d.j1 + 1;
      while (a < c) {
        int mid = a + (c - a) / 2;
        if (l0_of(mid) >= lo) c = mid;
        else a = mid + 1;
      }
      return a;
    };
    auto add_tile = [&](int l_start, int ncell, int fft_start) {
      SpreadItem s;
      s.box = (int)b; s.l_start = l_start; s.ncell = ncell; s.fft_start = fft_start; s.padding = 0;
      s.js = first_ge((long long)l_start - W);
      s.je = first_ge((long long)l_start + ncell + 1);
      spread.push_back(s);
    };
    for (int l = 0; l <= d.half; l += kSpreadTile)
      add_tile(l, std::min(kSpreadTile, d.half - l + 1), l);
    for (int l = -1; l >= -d.half; l -= kSpreadTile) {
      int lo = std::max(l - kSpreadTile + 1, -d.half);
      add_tile(lo, l - lo + 1, d.n2 + lo);
    }
    for (int f = d.half + 1; f <= d.n2 - d.half - 1; f += kSpreadTile) {
      SpreadItem s;
      s.box = (int)b; s.l_start = 0; s.fft_start = f; s.ncell = std::min(kSpreadTile, d.n2 - d.half - f);
      s.js = s.je = 0; s.padding = 1;
      spread.push_back(s);
    }
    for (int i = d.i0; i <= d.i1; i += kInterpTile)
      interp.push_back({(int)b, i, std::min(i + kInterpTile, d.i1 + 1)});
  }
  // ---- constants of the asymptotic evaluation
  AsyConst& A = ac;
  std::memset(&A, 0, sizeof(A));
  A.NLP = 2 * (P.K_asy + 1);
  A.beta = beta;
  double anu = std::fabs(P.nu);
  double ph = M_PI * (-anu / 2.0 - 0.25);
  A.cos_phi = std::cos(ph);
  A.sin_phi = std::sin(ph);
  double s2p = std::sqrt(2.0 / M_PI);
  for (int lp = 0; lp < A.NLP && lp < kMaxNLP; ++lp) {
    int l = lp / 2;
    A.coef[lp] = s2p * ((l & 1) ? -1.0 : 1.0) * P.asy_coef[lp];
  }
  A.nq = std::min(2 * W + 16, kMaxQuad);
  double gx[kMaxQuad], gw[kMaxQuad];
  gauss_legendre(A.nq, gx, gw);
  for (int q = 0; q < A.nq; ++q) {
    A.qx[q] = (gx[q] + 1.0) * 0.25 * W;
    A.qwpsi[q] = gw[q] * 0.25 * W * host_es(A.qx[q], W, beta);
  }
}

int DevicePlan::upload_all() {
  NUFHT_CUDA_TRY(cudaSetDevice(device));
  NUFHT_CUDA_TRY(cudaMalloc((void**)&d_rs, sizeof(double) * (size_t)m));
  NUFHT_CUDA_TRY(cudaMalloc((void**)&d_ws, sizeof(double) * (size_t)n));
  NUFHT_CUDA_TRY(cudaMemcpy(d_rs, h_rs.data(), sizeof(double) * m, cudaMemcpyHostToDevice));
  NUFHT_CUDA_TRY(cudaMemcpy(d_ws, h_ws.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  int rc;
  if ((rc = upload(locb, &d_locb)) || (rc = upload(proj, &d_proj)) || (rc = upload(eval, &d_eval)) ||
      (rc = upload(dir, &d_dir)) || (rc = upload(asyb, &d_asyb)) || (rc = upload(spread, &d_spread)) ||
      (rc = upload(interp, &d_interp)))
    return rc;
  return 0;
}

DevicePlan::~DevicePlan() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  for (auto& kv : fft_plans) cufftDestroy(kv.second);
  cudaFree(d_rs); cudaFree(d_ws); cudaFree(d_locb); cudaFree(d_proj); cudaFree(d_eval);
  cudaFree(d_dir); cudaFree(d_asyb); cudaFree(d_spread); cudaFree(d_interp);
  cudaFree(d_grid); cudaFree(d_partial); cudaFree(d_cheb); cudaFree(d_fft_work);
  cudaFree(d_stage_c); cudaFree(d_stage_g);
  if (prev >= 0) cudaSetDevice(prev);
}

int DevicePlan::ensure_workspace(int B) {
  if (B <= ws_B) return 0;
  cudaFree(d_grid); cudaFree(d_partial); cudaFree(d_cheb); cudaFree(d_fft_work);
  d_grid = nullptr; d_partial = nullptr; d_cheb = nullptr; d_fft_work = nullptr;
  for (auto& kv : fft_plans) cufftDestroy(kv.second);
  fft_plans.clear();
  ws_B = 0;
  size_t bytes = 0;
  const long long V = (long long)ac.NLP * B;
  if (!asyb.empty()) {
    size_t g = (size_t)total_cells * (size_t)V * sizeof(double2);
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_grid, g));
    bytes += g;
    size_t need = 0;
    for (const FftGroup& gr : groups) {
      cufftHandle h;
      if (cufftCreate(&h) != CUFFT_SUCCESS) return NUFHT_E_CUDA;
      cufftSetAutoAllocation(h, 0);
      int nn = gr.n2;
      long long batch = (long long)gr.nbox * V;
      if (batch > INT_MAX) return NUFHT_E_TOO_LARGE;
      size_t wsz = 0;
      if (cufftMakePlanMany(h, 1, &nn, nullptr, 1, nn, nullptr, 1, nn, CUFFT_Z2Z, (int)batch, &wsz) !=
          CUFFT_SUCCESS) {
        cufftDestroy(h);
        std::fprintf(stderr, "nufht_b200: cufftMakePlanMany failed (n=%d batch=%lld)\n", nn, batch);
        return NUFHT_E_CUDA;
      }
      need = std::max(need, wsz);
      fft_plans[gr.n2] = h;
    }
    if (need) {
      NUFHT_CUDA_TRY(cudaMalloc(&d_fft_work, need));
      bytes += need;
    }
    for (auto& kv : fft_plans) cufftSetWorkArea(kv.second, d_fft_work);
  }
  if (!locb.empty()) {
    size_t p = (size_t)proj.size() * KL1 * B * sizeof(double);
    size_t c = (size_t)locb.size() * KL1 * B * sizeof(double);
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_partial, p));
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_cheb, c));
    bytes += p + c;
  }
  ws_B = B;
  ws_bytes = bytes;
  return 0;
}

namespace {

template <int W>
int launch_asy(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B,
               cudaStream_t st, double sgn) {
  const AsyConst& A = D.ac;
  const int NLP = A.NLP;
  int BT = std::max(1, std::min(256 / NLP, 32));
  BT = std::min(BT, B);
  const int VCTA = NLP * BT;
  const int V_total = NLP * B;
  const int ngy = (B + BT - 1) / BT;
  size_t sm_spread = sizeof(double2) * kSpreadTile * VCTA + sizeof(double) * kSpreadChunk * W +
                     sizeof(double2) * kSpreadChunk + sizeof(double) * kSpreadChunk * NLP +
                     sizeof(double) * kSpreadChunk * BT + sizeof(double) * kSpreadTile +
                     sizeof(int) * kSpreadChunk;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_asy_spread<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_asy_interp<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  dim3 g1((unsigned)D.spread.size(), (unsigned)ngy);
  k_asy_spread<W><<<g1, VCTA, sm_spread, st>>>(D.d_rs, cs, ld_cs, B, D.d_grid, D.d_asyb,
                                               D.d_spread, A, BT, V_total);
  NUFHT_LAUNCH_CHECK();
  for (const FftGroup& gr : D.groups) {
    cufftHandle h = D.fft_plans[gr.n2];
    cufftSetStream(h, st);
    double2* p = D.d_grid + (size_t)gr.cell_off * (size_t)V_total;
    if (cufftExecZ2Z(h, (cufftDoubleComplex*)p, (cufftDoubleComplex*)p, CUFFT_INVERSE) != CUFFT_SUCCESS)
      return NUFHT_E_CUDA;
  }
  size_t sm_interp = sizeof(double2) * kInterpChunk * NLP + sizeof(double) * kInterpChunk * W +
                     sizeof(double) * kInterpChunk * VCTA + sizeof(int) * kInterpChunk;
  dim3 g2((unsigned)D.interp.size(), (unsigned)ngy);
  k_asy_interp<W><<<g2, VCTA, sm_interp, st>>>(D.d_ws, gs, ld_gs, B, D.d_grid, D.d_asyb,
                                               D.d_interp, A, BT, V_total, sgn);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

template <int BT>
int launch_dir(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B,
               cudaStream_t st, double sgn) {
  dim3 g((unsigned)D.dir.size(), (unsigned)((B + BT - 1) / BT));
  k_dir<BT><<<g, kDirTargets, 0, st>>>(D.d_rs, D.d_ws, cs, ld_cs, gs, ld_gs, B, D.d_dir, D.nu2, sgn);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

template <int MAXO>
int launch_loc_eval(DevicePlan& D, double* gs, int ld_gs, int B, cudaStream_t st, double sgn) {
  size_t sm = sizeof(double) * D.KL1 * B;
  if (sm > 48 * 1024)
    cudaFuncSetAttribute(k_loc_eval<MAXO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_loc_eval<MAXO><<<(unsigned)D.eval.size(), kLocTargets, sm, st>>>(
      D.d_ws, gs, ld_gs, B, D.d_locb, D.d_eval, D.d_cheb, D.P.K_loc, D.nu2 / 2, sgn);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

}  // namespace

int DevicePlan::run(const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
                    bool zero_output) {
  NUFHT_CUDA_TRY(cudaSetDevice(device));
  int rc = ensure_workspace(B);
  if (rc) return rc;
  if (zero_output)
    NUFHT_CUDA_TRY(cudaMemset2DAsync(gs, sizeof(double) * (size_t)ld_gs, 0, sizeof(double) * (size_t)n, B, st));
  const double sgn = sign;
  // ---- local boxes
  if (!locb.empty()) {
    int BT = 32;
    while (BT > 1 && KL1 * BT > 256) BT >>= 1;
    BT = std::min(BT, B);
    dim3 g((unsigned)proj.size(), (unsigned)((B + BT - 1) / BT));
    size_t sm = sizeof(double) * (KL1 * kLocChunk + kLocChunk * BT);
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_proj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_loc_proj<<<g, 256, sm, st>>>(d_rs, cs, ld_cs, B, d_locb, d_proj, KL1, (nu2 / 2) & 1, d_partial, BT);
    NUFHT_LAUNCH_CHECK();
    long long tot = (long long)locb.size() * KL1 * B;
    k_loc_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_locb, (int)locb.size(), KL1, B, d_partial, d_cheb);
    NUFHT_LAUNCH_CHECK();
    int maxo = (nu2 / 2) / 2 + P.K_loc + ((nu2 / 2) & 1);
    if (maxo <= 64) rc = launch_loc_eval<64>(*this, gs, ld_gs, B, st, sgn);
    else if (maxo <= 160) rc = launch_loc_eval<160>(*this, gs, ld_gs, B, st, sgn);
    else if (maxo <= 512) rc = launch_loc_eval<512>(*this, gs, ld_gs, B, st, sgn);
    else return NUFHT_E_TOO_LARGE;
    if (rc) return rc;
  }
  // ---- asymptotic boxes
  if (!asyb.empty()) {
    if (ac.NLP > kMaxNLP) return NUFHT_E_TOO_LARGE;
    switch (W) {
      case 2: rc = launch_asy<2>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 3: rc = launch_asy<3>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 4: rc = launch_asy<4>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 5: rc = launch_asy<5>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 6: rc = launch_asy<6>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 7: rc = launch_asy<7>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 8: rc = launch_asy<8>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 9: rc = launch_asy<9>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 10: rc = launch_asy<10>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 11: rc = launch_asy<11>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 12: rc = launch_asy<12>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 13: rc = launch_asy<13>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 14: rc = launch_asy<14>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      case 15: rc = launch_asy<15>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
      default: rc = launch_asy<16>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn); break;
    }
    if (rc) return rc;
  }
  // ---- direct boxes
  if (!dir.empty()) {
    if (B >= 32) rc = launch_dir<32>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    else if (B >= 16) rc = launch_dir<16>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    else if (B >= 8) rc = launch_dir<8>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    else if (B >= 4) rc = launch_dir<4>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    else rc = launch_dir<1>(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    if (rc) return rc;
  }
  return 0;
}

int run_besselj(double nu, const double* x, double* out, long count, cudaStream_t st) {
  double anu = std::fabs(nu);
  int nu2 = (int)std::llround(2.0 * anu);
  if (std::fabs(2.0 * anu - nu2) > 1e-12) return -2;
  if ((nu2 & 1) == 0 && nu2 / 2 > 200) return -2;
  if ((nu2 & 1) && nu2 > 19) return -2;
  if (count <= 0) return 0;
  k_besselj<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(nu2, x, out, count);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

}  // namespace hankel
