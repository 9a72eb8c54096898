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
// Workspace layout: box b (with NLP expansion terms) owns n2 * NLP * B contiguous complex
// values from cell_off * B (cell_off = the sum of n2 * NLP over the boxes before it); vector
// v = t * NLP + lp starts at v * n2 within them (one contiguous FFT input per vector).
#pragma once

#include <climits>
#include <cstdlib>

#include "kernels_common.cuh"

namespace hankel {

constexpr int kSpreadTile = 32;     // cells owned by one mode-0 spreading CTA
constexpr int kMinFft = 32;         // smallest FFT length of a box
constexpr int kSpreadChunk = 64;    // sources staged in shared memory per round, at most
constexpr int kChunkSources = 2048; // sources per mode-1 work item, at most
constexpr int kTileMaxSources = 2048;  // sources of a mode-0 tile, at most (denser boxes: mode 1)
constexpr int kInterpTile = 128;    // targets per interpolation CTA
constexpr int kInterpChunk = 32;    // targets per shared-memory round

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

// Work split of the spreading and interpolation CTAs.  Thread (tl, g) owns LPT
// consecutive expansion terms lp = g LPT .. g LPT + LPT - 1 of column t0 + tl, so every
// kernel weight read from shared memory feeds 2 LPT multiply-adds (register blocking).
// NG = NLP / LPT threads per column, BT columns per CTA.
struct AsyShape {
  int LPT, NG, BT, threads, ngy, V_total;
};

// Staged kernel weights per source and per target (real), padded so that every row is read
// with 16-byte shared-memory loads.
template <typename T>
__host__ __device__ constexpr int spread_we(int W) { return sizeof(T) == 4 ? (W + 3) & ~3 : (W + 1) & ~1; }
template <typename T>
__host__ __device__ constexpr int interp_we(int W) { return sizeof(T) == 4 ? (W + 3) & ~3 : (W + 1) & ~1; }

__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Shared-memory layout of k_asy_spread: two buffers (the chunk being walked and the next one,
// filled by asynchronous copies), each with the chunk's first cells, run ends, weights (rows
// of WE real values), amplitude factors (rows of NLP complex values) and coefficients (rows of
// BTP columns); byte offsets, each region 16-byte aligned.  The host sizes the launch with
// the same function.
struct SpreadSmem {
  size_t l0, end, w, p, c, buf, total;
};
template <typename T>
__host__ __device__ inline SpreadSmem spread_smem(int W, int NLP, int BTP, int SCH) {
  SpreadSmem L{};
  const size_t c2 = 2 * sizeof(T);
  L.l0 = 0;
  L.end = align16(L.l0 + (size_t)SCH * 4);
  L.w = align16(L.end + (size_t)SCH * 4);
  L.p = align16(L.w + (size_t)SCH * spread_we<T>(W) * sizeof(T));
  L.c = align16(L.p + (size_t)SCH * NLP * c2);
  L.buf = align16(L.c + (size_t)SCH * BTP * sizeof(T));
  L.total = 2 * L.buf;
  return L;
}
// Coefficient row of a spreading CTA in shared memory: BT columns rounded up to 16 bytes.
template <typename T>
__host__ __device__ constexpr int spread_btp(int BT) { return sizeof(T) == 4 ? (BT + 3) & ~3 : (BT + 1) & ~1; }

// Index one past the run of equal values that contains a[s] in the non-decreasing a[0, n).
__device__ __forceinline__ int run_end(const int* a, int n, int s) {
  const int v = a[s];
  int lo = s + 1, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] > v) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Shared-memory layout of k_asy_interp: the per-thread partial sums of a chunk of targets,
// then two buffers (the chunk being walked and the next one, filled by asynchronous copies of
// the target records), each with the chunk's factors mu, weights, first cells and run ends.
struct InterpSmem {
  size_t y, buf0, mu, wt, q0, end, buf, total;
};
template <typename T>
__host__ __device__ inline InterpSmem interp_smem(int W, int NLP, int threads) {
  InterpSmem L{};
  L.y = 0;
  L.buf0 = align16((size_t)kInterpChunk * (threads + 1) * sizeof(T));
  L.mu = 0;
  L.wt = align16(L.mu + (size_t)kInterpChunk * NLP * 2 * sizeof(T));
  L.q0 = align16(L.wt + (size_t)kInterpChunk * interp_we<T>(W) * sizeof(T));
  L.end = align16(L.q0 + (size_t)kInterpChunk * 4);
  L.buf = align16(L.end + (size_t)kInterpChunk * 4);
  L.total = L.buf0 + 2 * L.buf;
  return L;
}

// Plan-time table: 1/psi-hat(2 pi l / n2) for each box cell l.
static __global__ void k_asy_setup_cells(const AsyBoxD* __restrict__ boxes, AsyConst P,
                                  double* __restrict__ corr) {
  const AsyBoxD bx = boxes[blockIdx.y];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * bx.half + 1; c += gridDim.x * blockDim.x) {
    int l = c - bx.half;
    corr[bx.corr_off + c] = 1.0 / es_hat(P, 2.0 * M_PI * (double)l / (double)bx.n2);
  }
}

// Plan-time target records of stage 3 (k_asy_interp), per box and target i: the first cell
// q0 of its stencil at post_off + (i - i0), its W kernel weights at tw_off + (i - i0) WE
// (zeros after W), and its NLP factors
//   mu_lp = coef_lp (k rref)^-(lp + 1/2) exp(i (phi + k C)) / psi-hat((k - D) h)
// (rotated by i for odd lp) at tm_off + (i - i0) NLP, computed in FP64 and rounded to the
// arithmetic type; the weights are evaluated in that type at the FP64 offset u - (q0 + e).
template <typename T>
__global__ void k_asy_target_records(const double* __restrict__ ws, const AsyBoxD* __restrict__ boxes, AsyConst P,
                                     int W, int* __restrict__ tq0, T* __restrict__ tw,
                                     typename Cplx<T>::type* __restrict__ tmu) {
  const AsyBoxD bx = boxes[blockIdx.y];
  const int ni = bx.i1 - bx.i0 + 1;
  const int WE = interp_we<T>(W);
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;
  const double u_scale = bx.h * (double)bx.n2 / (2.0 * M_PI);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ni; q += gridDim.x * blockDim.x) {
    const double k = ws[bx.i0 + q];
    const double uu = (k - bx.D) * u_scale;
    const int q0 = (int)ceil(uu - 0.5 * W);
    tq0[bx.post_off + q] = q0;
    for (int e = 0; e < WE; ++e)
      tw[bx.tw_off + (long long)q * WE + e] = e < W ? es_kernel_t((T)(uu - (double)(q0 + e)), ihw, beta) : (T)0;
    const double inv_hat = 1.0 / es_hat(P, (k - bx.D) * bx.h);
    double sn, cn;
    sincos(k * bx.C, &sn, &cn);
    const double psx = (cn * P.cos_phi - sn * P.sin_phi) * inv_hat;
    const double psy = (sn * P.cos_phi + cn * P.sin_phi) * inv_hat;
    const double ik = 1.0 / (k * bx.rref);
    double pw = sqrt(ik);
    for (int lp = 0; lp < bx.nlp; ++lp, pw *= ik) {
      const double sc = P.coef[lp] * pw;
      const double mr = sc * psx, mi = sc * psy;
      tmu[bx.tm_off + (long long)q * bx.nlp + lp] = (lp & 1) ? cmake<T>((T)-mi, (T)mr) : cmake<T>((T)mr, (T)mi);
    }
  }
}

// Real weights of one source or target from shared memory (16-byte loads).
template <int WE>
__device__ __forceinline__ void load_weights(const float* src, float (&w)[WE]) {
  const float4* p = reinterpret_cast<const float4*>(src);
#pragma unroll
  for (int q = 0; q < WE / 4; ++q) {
    float4 v = p[q];
    w[4 * q] = v.x;
    w[4 * q + 1] = v.y;
    w[4 * q + 2] = v.z;
    w[4 * q + 3] = v.w;
  }
}
template <int WE>
__device__ __forceinline__ void load_weights(const double* src, double (&w)[WE]) {
  const double2* p = reinterpret_cast<const double2*>(src);
#pragma unroll
  for (int q = 0; q < WE / 2; ++q) {
    double2 v = p[q];
    w[2 * q] = v.x;
    w[2 * q + 1] = v.y;
  }
}

// acc += w * a for complex w and real a: one packed two-lane FMA in single precision
// (__ffma2_rn, FFMA2 on sm_100 and later), two FMAs in double.
__device__ __forceinline__ void cfma(float2& acc, float2 w, float a) { acc = __ffma2_rn(w, make_float2(a, a), acc); }
__device__ __forceinline__ void cfma(double2& acc, double2 w, double a) {
  acc.x = fma(w.x, a, acc.x);
  acc.y = fma(w.y, a, acc.y);
}

__device__ __forceinline__ void grid_atomic_add(float2* p, float2 v) {
  atomicAdd(p, v);  // one vector reduction (sm_90 and later)
}
__device__ __forceinline__ void grid_atomic_add(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

// Plan-time source records of stage 1 (k_asy_spread), per box and source j: first cell of
// the kernel support at rec_off + (j - j0), W real weights psi(l0 + q - u) / psi-hat(l0 + q)
// at recw_off + (j - j0) W, and NLP complex factors (rref / r)^(lp + 1/2) exp(i D (r - C))
// at recp_off + (j - j0) NLP (the source phase is the same for all taps, so it rides with
// the amplitude).  The weights and the first cell follow from the same FP64 position
// u = (r - C) / h as the cell tables; the kernel value is evaluated in the arithmetic type,
// the factors in FP64 and rounded.
template <typename T>
__global__ void k_asy_records(const double* __restrict__ rs, const AsyBoxD* __restrict__ boxes, AsyConst P, int W,
                              const double* __restrict__ corr, int* __restrict__ rl0, T* __restrict__ rw,
                              typename Cplx<T>::type* __restrict__ rp) {
  const AsyBoxD bx = boxes[blockIdx.y];
  const int nj = bx.j1 - bx.j0 + 1;
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nj; q += gridDim.x * blockDim.x) {
    const double r = rs[bx.j0 + q];
    const double x = r - bx.C;
    const double u = x / bx.h;
    const int l0 = (int)ceil(u - 0.5 * W);
    rl0[bx.rec_off + q] = l0;
    double sn, cn;
    sincos(bx.D * x, &sn, &cn);
    for (int e = 0; e < W; ++e) {
      const int cell = l0 + e;
      rw[bx.recw_off + (long long)q * W + e] =
          (cell >= -bx.half && cell <= bx.half)
              ? es_kernel_t((T)((double)cell - u), ihw, beta) * (T)corr[bx.corr_off + cell + bx.half]
              : (T)0;
    }
    const double ir = r > 0.0 ? bx.rref / r : 0.0;  // sources at r = 0 contribute nothing
    double pw = sqrt(ir);
    for (int lp = 0; lp < bx.nlp; ++lp, pw *= ir)
      rp[bx.recp_off + (long long)q * bx.nlp + lp] = cmake<T>((T)(pw * cn), (T)(pw * sn));
  }
}

// ct[j * ldct + t] = cs[t * ld_cs + j] in the arithmetic type (zero for t >= B): 32 x 32
// tiles through shared memory, coalesced on both sides.
template <typename T>
__global__ void __launch_bounds__(256) k_pack_coefficients(const double* __restrict__ cs, int ld_cs, int B, int m,
                                                           T* __restrict__ ct, int ldct) {
  __shared__ double tile[32][33];
  const int j0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int t = t0 + ty, j = j0 + threadIdx.x;
    tile[ty][threadIdx.x] = (t < B && j < m) ? cs[(size_t)t * ld_cs + j] : 0.0;
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int j = j0 + ty, t = t0 + threadIdx.x;
    if (j < m && t < ldct) ct[(size_t)j * ldct + t] = (T)tile[threadIdx.x][ty];
  }
}

// Stage 1.  Everything about a source except its coefficients is fixed when the plan is
// made, so the plan keeps, per (box, source) pair (k_asy_records): the first cell l0 of its
// kernel support, its W complex weights psi(l0 + q - u) exp(i D x) / psi-hat(l0 + q) (zero
// outside [-half, half]) and its NLP amplitude factors (rref / r)^(lp + 1/2).  A transform packs
// its coefficients source-major in the arithmetic type (k_pack_coefficients), and a spreading
// CTA copies its sources' records and coefficients to shared memory in chunks of SCH sources
// with cp.async, the next chunk in flight while the current one is walked.
//
// Sources are sorted, so l0 never decreases.  The CTA walks the cells in order; at cell c it
// adds every source with l0 == c into W register accumulators per vector, then cell c is final
// and leaves.  The accumulators form a ring indexed (position + tap) mod W, and the walk is
// unrolled W times so that every ring index is a compile-time constant: no register moves as
// the window advances.  TILE items (mode 0) own their cells and store each one exactly once,
// zeros where no source reaches; the source chunks of dense boxes (mode 1) add their cells
// atomically to the pre-zeroed grid.  Empty stretches between sources are skipped once the
// ring is empty.
template <typename T, int W, int LPT, bool TILE>
__global__ void __launch_bounds__(256) k_asy_spread(
    const T* __restrict__ ct, int ldct, int B, typename Cplx<T>::type* __restrict__ grid,
    const AsyBoxD* __restrict__ boxes, const SpreadItem* __restrict__ items, const int* __restrict__ rl0,
    const T* __restrict__ rw, const typename Cplx<T>::type* __restrict__ rp, int NLP, int BT, int V_total,
    int SCH) {
  using C2 = typename Cplx<T>::type;
  constexpr int WE = spread_we<T>(W);
  constexpr int PER16 = 16 / (int)sizeof(T);  // values per 16-byte copy
  const SpreadItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NG = NLP / LPT;
  const int nthr = blockDim.x;
  const int VCTA = BT * NLP;
  const int tid = threadIdx.x;
  const int tl = tid / NG, g = tid - tl * NG;
  const int t0 = blockIdx.y * BT;
  const int v0 = t0 * NLP;
  const int vloc = tl * NLP + g * LPT;  // first of this thread's vectors within the CTA
  const bool active = tl < BT && t0 + tl < B;
  C2* gbox = grid + (size_t)bx.cell_off * (size_t)B;
  const int nc = it.ncell;

  if (TILE && it.mode == 2) {  // zero padding of the FFT input: threads along cells
    const int nv = min(VCTA, V_total - v0);
    for (int e = tid; e < nc * nv; e += nthr) {
      int vv = e / nc, cell = e - vv * nc;
      gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = cmake<T>(0, 0);
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int BTP = spread_btp<T>(BT);
  const SpreadSmem L = spread_smem<T>(W, NLP, BTP, SCH);
  const int nsrc = it.je - it.js;
  const int jr0 = it.js - bx.j0;  // first source of the item within its box

  // Copies of the item's sources [s0, s0 + ns) into buffer b (one commit group).
  auto issue = [&](int b, int s0, int ns) {
    unsigned char* base = smem_raw + (size_t)b * L.buf;
    int* d_l0 = reinterpret_cast<int*>(base + L.l0);
    T* d_w = reinterpret_cast<T*>(base + L.w);
    C2* d_p = reinterpret_cast<C2*>(base + L.p);
    T* d_c = reinterpret_cast<T*>(base + L.c);
    const int js = jr0 + s0;
    for (int s = tid; s < ns; s += nthr) cp_async4(d_l0 + s, rl0 + bx.rec_off + js + s);
    const T* gw = rw + bx.recw_off + (long long)js * W;
    for (int e = tid; e < ns * W; e += nthr) {
      const int s = e / W, q = e - s * W;
      if constexpr (sizeof(T) == 4) cp_async4(d_w + s * WE + q, gw + e);
      else cp_async8(d_w + s * WE + q, gw + e);
    }
    const C2* gp = rp + bx.recp_off + (long long)js * NLP;
    for (int e = tid; e < ns * NLP; e += nthr) {
      if constexpr (sizeof(T) == 4) cp_async8(d_p + e, gp + e);
      else cp_async16(d_p + e, gp + e);
    }
    // coefficients: BTP columns per source in 16-byte pieces (ldct and t0 are multiples of 4;
    // pieces past the packed row are columns >= B, whose threads store nothing)
    const int npc = BTP / PER16;
    const T* gc = ct + (size_t)(it.js + s0) * ldct + t0;
    for (int e = tid; e < ns * npc; e += nthr) {
      const int s = e / npc, q = e - s * npc;
      if (t0 + q * PER16 < ldct) cp_async16(d_c + s * BTP + q * PER16, gc + (size_t)s * ldct + q * PER16);
    }
    cp_async_commit();
  };
  const int* s_l0 = nullptr;
  int* s_end = nullptr;
  const T* s_w = nullptr;
  const C2* s_p = nullptr;
  const T* s_c = nullptr;
  auto point = [&](int b) {
    unsigned char* base = smem_raw + (size_t)b * L.buf;
    s_l0 = reinterpret_cast<const int*>(base + L.l0);
    s_end = reinterpret_cast<int*>(base + L.end);
    s_w = reinterpret_cast<const T*>(base + L.w);
    s_p = reinterpret_cast<const C2*>(base + L.p);
    s_c = reinterpret_cast<const T*>(base + L.c);
  };

  C2 acc[LPT][W];
#pragma unroll
  for (int u = 0; u < LPT; ++u)
#pragma unroll
    for (int q = 0; q < W; ++q) acc[u][q] = cmake<T>(0, 0);

  // Tiles write every cell they own exactly once, in increasing order: cells the walk skips
  // (no source support) get zeros.  zc = first owned cell not written yet.
  int zc = it.l_start;
  auto zero_to = [&](int upto) {  // zeros for owned cells [zc, upto)
    if (!TILE) return;
    const int hi = min(upto, it.l_start + nc);
    if (active)
      for (int cc = max(zc, it.l_start); cc < hi; ++cc) {
        const int idx = it.fft_start + (cc - it.l_start);
#pragma unroll
        for (int u = 0; u < LPT; ++u) gbox[(size_t)(v0 + vloc + u) * bx.n2 + idx] = cmake<T>(0, 0);
      }
    zc = max(zc, hi);
  };

  if (nsrc > 0) {
    int s0 = 0;  // item-relative first source of the current chunk
    int ns = min(SCH, nsrc);
    int cur = 0;
    issue(0, 0, ns);
    if (ns < nsrc) issue(1, ns, min(SCH, nsrc - ns));
    cp_async_wait_all();
    __syncthreads();
    point(0);
    for (int s = tid; s < ns; s += nthr) s_end[s] = run_end(s_l0, ns, s);
    __syncthreads();
    int sp = 0;
    // first cell and run end of source sp, kept in registers (loaded when sp moves, so that
    // the loads overlap the work before the next test)
    int ln = s_l0[0], en = s_end[0];
    int c = ln;
    // last cell to visit: the last source's support end, or the tile's end
    int c_end = rl0[bx.rec_off + jr0 + nsrc - 1] + W - 1;
    if (TILE) c_end = min(c_end, it.l_start + nc - 1);
    int last = INT_MIN / 2;  // cell of the latest source added
    bool done = c > c_end;
    while (!done) {
#pragma unroll
      for (int jj = 0; jj < W; ++jj) {
        // sources whose support starts at cell c (ring position jj)
        for (;;) {
          if (sp < ns && ln == c) {
            const int e = en;
            if (e < ns) {
              ln = s_l0[e];
              en = s_end[e];
            }
            if (tl < BT) {
              auto add = [&](int s) {
                const T cv = s_c[s * BTP + tl];
                T wt[WE];
                load_weights<WE>(s_w + s * WE, wt);
#pragma unroll
                for (int u = 0; u < LPT; ++u) {
                  const C2 pp = s_p[s * NLP + g * LPT + u];
                  const C2 a = cmake<T>(cv * pp.x, cv * pp.y);  // complex amplitude of the source
#pragma unroll
                  for (int q = 0; q < W; ++q) cfma(acc[u][(jj + q) % W], a, wt[q]);
                }
              };
#pragma unroll 1
              for (int s = sp; s < e; ++s) add(s);
            }
            last = c;
            sp = e;
          }
          if (sp < ns || s0 + ns >= nsrc) break;
          // the next chunk (already in flight) becomes current; the buffer just released
          // takes the one after it
          cp_async_wait_all();
          __syncthreads();
          cur ^= 1;
          s0 += ns;
          ns = min(SCH, nsrc - s0);
          point(cur);
          for (int s = tid; s < ns; s += nthr) s_end[s] = run_end(s_l0, ns, s);
          if (s0 + ns < nsrc) issue(cur ^ 1, s0 + ns, min(SCH, nsrc - s0 - ns));
          __syncthreads();
          sp = 0;
          ln = s_l0[0];
          en = s_end[0];
        }
        // cell c is final
        if (active) {
          if (TILE) {
            const int cl = c - it.l_start;
            if (cl >= 0 && cl < nc) {
              // the CTA owns the cell: zeros for the owned cells skipped before it, then the cell
              zero_to(c);
              zc = c + 1;
              const int idx = it.fft_start + cl;
#pragma unroll
              for (int u = 0; u < LPT; ++u) gbox[(size_t)(v0 + vloc + u) * bx.n2 + idx] = acc[u][jj];
            }
          } else if (c >= -bx.half && c <= bx.half) {
            const int idx = c < 0 ? c + bx.n2 : c;
#pragma unroll
            for (int u = 0; u < LPT; ++u) {
              const C2 v = acc[u][jj];
              if (v.x != (T)0 || v.y != (T)0) grid_atomic_add(gbox + (size_t)(v0 + vloc + u) * bx.n2 + idx, v);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < LPT; ++u) acc[u][jj] = cmake<T>(0, 0);
        if (c >= c_end) {
          done = true;
          break;
        }
        // Past the ring's last non-empty cell the next source's cell can be jumped to: all
        // accumulators are zero, so any ring position may stand for it.
        const int nxt = sp < ns ? ln : INT_MAX;
        if (c >= last + W - 1 && nxt != INT_MAX && nxt > c + 1) c = nxt;
        else ++c;
      }
    }
  }
  zero_to(INT_MAX);  // owned cells after the walk (or all of them when no source reaches the tile)
}

// Stage 3.  Thread (tl, g) owns terms g LPT .. g LPT + LPT - 1 of column t0 + tl.  The target
// records (k_asy_target_records) are copied to shared memory in chunks of kInterpChunk with
// cp.async, the next chunk in flight while the current one is walked.  Targets are sorted, so
// the first cell q0 of their stencil never decreases; the CTA walks the cells in order with a
// ring of R = W + 1 grid values per vector in registers (the stencil plus one cell fetched a
// step ahead); the walk is unrolled R times, which makes every ring index a compile-time
// constant.  Each thread combines its terms with the per-target factors mu and leaves its
// partial sum in shared memory; at the end of each chunk of targets the NG partials of a
// column are added in FP64 and atomically into g, consecutive threads taking consecutive
// targets of a column.  (Warp shuffles for the partial sums measured slower on B200.)
template <typename T, int W, int LPT>
__global__ void __launch_bounds__(256) k_asy_interp(
    double* __restrict__ gs, int ld_gs, int B, const typename Cplx<T>::type* __restrict__ grid,
    const AsyBoxD* __restrict__ boxes, const InterpItem* __restrict__ items, const int* __restrict__ tq0,
    const T* __restrict__ tw, const typename Cplx<T>::type* __restrict__ tmu, int NLP, int BT, double sgn) {
  using C2 = typename Cplx<T>::type;
  constexpr int WE = interp_we<T>(W);
  constexpr int R = W + 1;
  constexpr int PER16 = 16 / (int)sizeof(T);  // values per 16-byte copy
  const InterpItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NG = NLP / LPT;
  const int nthr = blockDim.x;
  const int YP = nthr + 1;  // padded row of the per-target partial sums
  const int tid = threadIdx.x;
  const int tl = tid / NG, g = tid - tl * NG;
  const int t0 = blockIdx.y * BT;
  const bool active = tl < BT && t0 + tl < B;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InterpSmem L = interp_smem<T>(W, NLP, nthr);
  T* s_y = reinterpret_cast<T*>(smem_raw + L.y);  // [KC][YP]: per-thread partial sums (already in T)
  const C2* s_mu = nullptr;  // [KC][NLP]
  const T* s_wt = nullptr;   // [KC][WE]
  const int* s_q0 = nullptr; // [KC]
  int* s_end = nullptr;      // [KC]: end of the equal-q0 run
  auto point = [&](int b) {
    unsigned char* base = smem_raw + L.buf0 + (size_t)b * L.buf;
    s_mu = reinterpret_cast<const C2*>(base + L.mu);
    s_wt = reinterpret_cast<const T*>(base + L.wt);
    s_q0 = reinterpret_cast<const int*>(base + L.q0);
    s_end = reinterpret_cast<int*>(base + L.end);
  };
  // Copies of the records of targets [k0, k0 + nk) into buffer b (one commit group).
  auto issue = [&](int b, int k0, int nk) {
    unsigned char* base = smem_raw + L.buf0 + (size_t)b * L.buf;
    C2* d_mu = reinterpret_cast<C2*>(base + L.mu);
    T* d_wt = reinterpret_cast<T*>(base + L.wt);
    int* d_q0 = reinterpret_cast<int*>(base + L.q0);
    const int q = k0 - bx.i0;
    for (int kk = tid; kk < nk; kk += nthr) cp_async4(d_q0 + kk, tq0 + bx.post_off + q + kk);
    const T* gw = tw + bx.tw_off + (long long)q * WE;  // rows of WE values: 16-byte pieces
    for (int e = tid; e < nk * WE / PER16; e += nthr) cp_async16(d_wt + e * PER16, gw + e * PER16);
    const C2* gm = tmu + bx.tm_off + (long long)q * NLP;
    for (int e = tid; e < nk * NLP; e += nthr) {
      if constexpr (sizeof(T) == 4) cp_async8(d_mu + e, gm + e);
      else cp_async16(d_mu + e, gm + e);
    }
    cp_async_commit();
  };

  const int n2 = bx.n2;
  const C2* row[LPT];
#pragma unroll
  for (int u = 0; u < LPT; ++u)
    row[u] = grid + (size_t)bx.cell_off * (size_t)B +
             (size_t)(active ? (t0 + tl) * NLP + g * LPT + u : 0) * (size_t)n2;

  auto fetch = [&](int cell, int u) -> C2 {
    int idx = cell < 0 ? cell + n2 : (cell >= n2 ? cell - n2 : cell);
    return active ? row[u][idx] : cmake<T>(0, 0);
  };

  // Sum the NG partials of each column and add them to g (all threads).
  auto flush = [&](int k0, int nk) {
    __syncthreads();
    for (int e = tid; e < nk * BT; e += nthr) {
      int tt = e / nk, kk = e - tt * nk;
      if (t0 + tt < B) {
        double sum = 0.0;
        for (int q = 0; q < NG; ++q) sum += (double)s_y[kk * YP + tt * NG + q];
        atomicAdd(&gs[(size_t)(t0 + tt) * ld_gs + k0 + kk], sgn * sum);
      }
    }
  };

  if (it.ke <= it.ks) return;
  int k0 = it.ks;
  int nk = min(kInterpChunk, it.ke - k0);
  int cur = 0;
  issue(0, k0, nk);
  if (k0 + nk < it.ke) issue(1, k0 + nk, min(kInterpChunk, it.ke - k0 - nk));
  cp_async_wait_all();
  __syncthreads();
  point(0);
  for (int kk = tid; kk < nk; kk += nthr) s_end[kk] = run_end(s_q0, nk, kk);
  __syncthreads();
  int kp = 0;
  // first cell and run end of target kp, kept in registers (loaded when kp moves, so that
  // the loads overlap the work before the next test)
  int qn = s_q0[0], en = s_end[0];
  int c = qn;
  C2 gw[LPT][R];
#pragma unroll
  for (int q = 0; q < R; ++q)
#pragma unroll
    for (int u = 0; u < LPT; ++u) gw[u][q] = fetch(c + q, u);
  bool done = false;
  while (!done) {
#pragma unroll
    for (int jj = 0; jj < R; ++jj) {
      // targets whose stencil starts at cell c (ring position jj)
      for (;;) {
        if (kp < nk && qn == c) {
          const int e = en;
          if (e < nk) {
            qn = s_q0[e];
            en = s_end[e];
          }
          if (tl < BT) {
#pragma unroll 1
            for (int k = kp; k < e; ++k) {
              T wt[WE];
              load_weights<WE>(s_wt + k * WE, wt);
              T y = (T)0;
#pragma unroll
              for (int u = 0; u < LPT; ++u) {
                C2 f = cmake<T>(0, 0);
#pragma unroll
                for (int q = 0; q < W; ++q) cfma(f, gw[u][(jj + q) % R], wt[q]);
                const C2 mu = s_mu[k * NLP + g * LPT + u];
                y = fma(mu.x, f.x, y);
                y = fma(-mu.y, f.y, y);
              }
              s_y[k * YP + tid] = y;
            }
          }
          kp = e;
        }
        if (kp < nk) break;
        flush(k0, nk);
        if (k0 + nk >= it.ke) {
          done = true;
          break;
        }
        // the next chunk (already in flight) becomes current; the buffer just released takes
        // the one after it
        cp_async_wait_all();
        __syncthreads();  // partial sums read, current buffer released, copies visible
        cur ^= 1;
        k0 += nk;
        nk = min(kInterpChunk, it.ke - k0);
        point(cur);
        for (int kk = tid; kk < nk; kk += nthr) s_end[kk] = run_end(s_q0, nk, kk);
        if (k0 + nk < it.ke) issue(cur ^ 1, k0 + nk, min(kInterpChunk, it.ke - k0 - nk));
        __syncthreads();
        kp = 0;
        qn = s_q0[0];
        en = s_end[0];
      }
      if (done) break;
      // advance to the next target's cell; ring position jj + 1 stands for it
      const int nxt = qn;
      if (nxt == c + 1) {
        // the slot of cell c takes cell c + R (one cell ahead of the next stencil)
#pragma unroll
        for (int u = 0; u < LPT; ++u) gw[u][jj] = fetch(c + R, u);
        c = nxt;
      } else {
        // a jump: refill the ring in its canonical order and restart at position 0 (one
        // refill sequence in the code instead of one per ring position)
#pragma unroll
        for (int q = 0; q < R; ++q)
#pragma unroll
          for (int u = 0; u < LPT; ++u) gw[u][q] = fetch(nxt + q, u);
        c = nxt;
        break;
      }
    }
  }
}

}  // namespace hankel
