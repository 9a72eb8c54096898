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

constexpr int kSpreadTile = 16;     // cells owned by one mode-0 spreading CTA at 8 or more terms
constexpr int kMinFft = 32;         // smallest FFT length of a box
constexpr int kSpreadChunk = 64;    // sources staged in shared memory per round
constexpr int kChunkSources = 2048; // sources per mode-1 work item, at most
constexpr int kTileMaxSources = 4096;
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
// kernel weight read from shared memory feeds 2 LPT multiply-adds (register blocking), and
// the LPT source amplitudes (rref / r)^(lp + 1/2) c follow from one staged value by
// multiplications with rref / r.  NG = NLP / LPT threads per column, BT columns per CTA.
struct AsyShape {
  int LPT, NG, BT, threads, ngy, V_total;
};

// Cells of a mode-0 spreading tile (AsyConst::tile_cells, chosen per kernel class at plan
// time): 16 at 6 or more expansion terms, 32 at 2 or 4 (whose CTAs have one term per thread,
// NLP / 1 threads per column), or NUFHT_B200_TILE_CELLS_SMALL for 2 and 4 terms.  A window
// (cells x (vectors + 1) complex values, when tiles write through shared memory) of these
// sizes stays near 16 KB for 2 and 4 terms and 33 KB for 8.
inline int spread_tile_cells(int nlp) {
  static const int small = [] {
    const char* e = std::getenv("NUFHT_B200_TILE_CELLS_SMALL");
    const int v = e ? std::atoi(e) : 0;
    return (v >= 8 && v <= 256) ? v : 2 * kSpreadTile;
  }();
  return nlp >= 6 ? kSpreadTile : small;
}

// Staged kernel weights per source (complex) and per target (real), padded so that every
// row is read with 16-byte shared-memory loads.
template <typename T>
__host__ __device__ constexpr int spread_we(int W) { return sizeof(T) == 4 ? (W + 1) & ~1 : W; }
template <typename T>
__host__ __device__ constexpr int interp_we(int W) { return sizeof(T) == 4 ? (W + 3) & ~3 : (W + 1) & ~1; }

__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Shared-memory layout of k_asy_spread (byte offsets, each region 16-byte aligned); the
// host sizes the launch with the same function.
struct SpreadSmem {
  size_t win, wc, rq, c, u, ph, l0, end, total;
};
template <typename T>
__host__ __device__ inline SpreadSmem spread_smem(int W, int VCTA, int NG, int BT, bool windowed, int tile_cells) {
  SpreadSmem L{};
  const size_t c2 = 2 * sizeof(T);
  L.win = 0;
  L.wc = align16(L.win + (windowed ? (size_t)tile_cells * (VCTA + 1) * c2 : 0));
  L.rq = align16(L.wc + (size_t)kSpreadChunk * spread_we<T>(W) * c2);
  L.c = align16(L.rq + (size_t)kSpreadChunk * NG * c2);
  L.u = align16(L.c + (size_t)BT * (kSpreadChunk + 1) * sizeof(T));
  L.ph = align16(L.u + (size_t)kSpreadChunk * sizeof(double));
  L.l0 = align16(L.ph + (size_t)kSpreadChunk * c2);
  L.end = align16(L.l0 + (size_t)kSpreadChunk * 4);
  L.total = align16(L.end + (size_t)kSpreadChunk * 4);
  return L;
}

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

// Shared-memory layout of k_asy_interp.
struct InterpSmem {
  size_t mu, y, wt, q0, end, uu, total;
};
template <typename T>
__host__ __device__ inline InterpSmem interp_smem(int W, int NLP, int threads) {
  InterpSmem L{};
  L.mu = 0;
  L.y = align16(L.mu + (size_t)kInterpChunk * NLP * 2 * sizeof(T));
  L.wt = align16(L.y + (size_t)kInterpChunk * (threads + 1) * sizeof(T));
  L.q0 = align16(L.wt + (size_t)kInterpChunk * interp_we<T>(W) * sizeof(T));
  L.end = align16(L.q0 + (size_t)kInterpChunk * 4);
  L.uu = align16(L.end + (size_t)kInterpChunk * 4);
  L.total = align16(L.uu + (size_t)kInterpChunk * sizeof(double));
  return L;
}

// Plan-time tables: 1/psi-hat(2 pi l / n2) for each box cell l, and
// exp(i (phi + k C)) / psi-hat((k - D) h) for each box target.
static __global__ void k_asy_setup_cells(const AsyBoxD* __restrict__ boxes, AsyConst P,
                                  double* __restrict__ corr) {
  const AsyBoxD bx = boxes[blockIdx.y];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * bx.half + 1; c += gridDim.x * blockDim.x) {
    int l = c - bx.half;
    corr[bx.corr_off + c] = 1.0 / es_hat(P, 2.0 * M_PI * (double)l / (double)bx.n2);
  }
}

static __global__ void k_asy_setup_targets(const double* __restrict__ ws, const AsyBoxD* __restrict__ boxes,
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

// Weights of one source or target from shared memory (16-byte loads).
template <int WE>
__device__ __forceinline__ void load_weights(const float2* src, float2 (&w)[WE]) {
  const float4* p = reinterpret_cast<const float4*>(src);
#pragma unroll
  for (int q = 0; q < WE / 2; ++q) {
    float4 v = p[q];
    w[2 * q] = make_float2(v.x, v.y);
    w[2 * q + 1] = make_float2(v.z, v.w);
  }
}
template <int WE>
__device__ __forceinline__ void load_weights(const double2* src, double2 (&w)[WE]) {
#pragma unroll
  for (int q = 0; q < WE; ++q) w[q] = src[q];
}
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

// Stage 1.  Sources are sorted, so the first cell l0 of their kernel support never
// decreases.  The CTA walks the cells c in order; at cell c it adds every source with
// l0 == c into W register accumulators per vector, then cell c is final and leaves.  The
// accumulators form a ring indexed (position + tap) mod W, and the walk is unrolled W times
// so that every ring index is a compile-time constant: no register moves as the window
// advances.  A finished cell goes to a shared window of the CTA's own cells (WINDOWED,
// mode-0 tiles; written to the grid with coalesced stores at the end) or is added
// atomically to the pre-zeroed grid (mode-1 source chunks of dense boxes).  Empty stretches
// between sources are skipped once the ring is empty.  The source phase exp(i D x) is folded
// into complex kernel weights staged once per source.
template <typename T, int W, int LPT, bool WINDOWED, bool DIRECT = false>
__global__ void __launch_bounds__(256) k_asy_spread(
    const double* __restrict__ rs, const double* __restrict__ cs, int ld_cs, int B,
    typename Cplx<T>::type* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const SpreadItem* __restrict__ items, const double* __restrict__ corr, AsyConst P, int BT,
    int V_total) {
  using C2 = typename Cplx<T>::type;
  constexpr int SCP = kSpreadChunk + 1;  // padded row of the staged coefficients
  constexpr int WE = spread_we<T>(W);
  const SpreadItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int NG = NLP / LPT;
  const int nthr = blockDim.x;
  const int VCTA = BT * NLP;
  const int WP = VCTA + 1;  // padded window row
  const int tid = threadIdx.x;
  const int tl = tid / NG, g = tid - tl * NG;
  const int t0 = blockIdx.y * BT;
  const int v0 = t0 * NLP;
  const int nv = min(VCTA, V_total - v0);  // valid vectors of this CTA
  const int vloc = tl * NLP + g * LPT;     // first of this thread's vectors within the CTA
  const bool active = tl < BT && t0 + tl < B;
  C2* gbox = grid + (size_t)bx.cell_off * (size_t)B;
  const int nc = it.ncell;

  if (WINDOWED && it.mode == 2) {  // zero padding of the FFT input: threads along cells
    for (int e = tid; e < nc * nv; e += nthr) {
      int vv = e / nc, cell = e - vv * nc;
      gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = cmake<T>(0, 0);
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TC = P.tile_cells;
  const SpreadSmem L = spread_smem<T>(W, VCTA, NG, BT, WINDOWED && !DIRECT, TC);
  C2* win = reinterpret_cast<C2*>(smem_raw + L.win);        // [TC][WP]
  C2* s_wc = reinterpret_cast<C2*>(smem_raw + L.wc);        // [SCH][WE]
  C2* s_rq = reinterpret_cast<C2*>(smem_raw + L.rq);        // [SCH][NG]: (rho of term g LPT, rref / r)
  T* s_c = reinterpret_cast<T*>(smem_raw + L.c);            // [BT][SCP]
  double* s_u = reinterpret_cast<double*>(smem_raw + L.u);  // [SCH]
  C2* s_ph = reinterpret_cast<C2*>(smem_raw + L.ph);        // [SCH]: exp(i D x)
  int* s_l0 = reinterpret_cast<int*>(smem_raw + L.l0);      // [SCH]
  int* s_end = reinterpret_cast<int*>(smem_raw + L.end);    // [SCH]: end of the equal-l0 run

  if (WINDOWED && !DIRECT)
    for (int e = tid; e < TC * WP; e += nthr) win[e] = cmake<T>(0, 0);
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;

  // Stage sources [s0, s0 + ns) (all threads; barriers on both sides).
  auto stage = [&](int s0, int ns) {
    __syncthreads();  // previous round fully consumed
    for (int s = tid; s < ns; s += nthr) {
      double r = rs[s0 + s];
      double x = r - bx.C;
      double u = x / bx.h;
      s_u[s] = u;
      s_l0[s] = (int)ceil(u - 0.5 * W);
      double sn, cn;
      sincos(bx.D * x, &sn, &cn);
      s_ph[s] = cmake<T>((T)cn, (T)sn);
      double ir = r > 0.0 ? bx.rref / r : 0.0;  // sources at r = 0 contribute nothing
      double rho = sqrt(ir);
      for (int q = 0; q < NG; ++q) {
        s_rq[s * NG + q] = cmake<T>((T)rho, (T)ir);
        for (int z = 0; z < LPT; ++z) rho *= ir;
      }
    }
    for (int e = tid; e < ns * BT; e += nthr) {
      int tt = e / ns, s = e - tt * ns;
      s_c[tt * SCP + s] = (T)((t0 + tt < B) ? cs[(size_t)(t0 + tt) * ld_cs + s0 + s] : 0.0);
    }
    __syncthreads();
    // complex weights psi(l - u) exp(i D x) / psi-hat(cell l): the deconvolution factor of the
    // target cell is folded in here (loaded in parallel with the other weights), so finished
    // cells are stored as they are
    for (int e = tid; e < ns * WE; e += nthr) {
      int s = e / WE, q = e - s * WE;
      const int cell = s_l0[s] + q;
      T w = (q < W && cell >= -bx.half && cell <= bx.half)
                ? es_kernel_t((T)((double)cell - s_u[s]), ihw, beta) * (T)corr[bx.corr_off + cell + bx.half]
                : (T)0;
      C2 ph = s_ph[s];
      s_wc[e] = cmake<T>(w * ph.x, w * ph.y);
    }
    for (int s = tid; s < ns; s += nthr) s_end[s] = run_end(s_l0, ns, s);
    __syncthreads();
  };

  C2 acc[LPT][W];
#pragma unroll
  for (int u = 0; u < LPT; ++u)
#pragma unroll
    for (int q = 0; q < W; ++q) acc[u][q] = cmake<T>(0, 0);

  // DIRECT tiles write every cell they own exactly once, in increasing order: cells the walk
  // skips (no source support) get zeros.  zc = first owned cell not written yet.
  int zc = it.l_start;
  auto zero_to = [&](int upto) {  // zeros for owned cells [zc, upto)
    if (!(WINDOWED && DIRECT)) return;
    const int hi = min(upto, it.l_start + nc);
    if (active)
      for (int cc = max(zc, it.l_start); cc < hi; ++cc) {
        const int idx = it.fft_start + (cc - it.l_start);
#pragma unroll
        for (int u = 0; u < LPT; ++u) gbox[(size_t)(v0 + vloc + u) * bx.n2 + idx] = cmake<T>(0, 0);
      }
    zc = max(zc, hi);
  };

  if (it.je > it.js) {
    int s0 = it.js;
    int ns = min(kSpreadChunk, it.je - s0);
    stage(s0, ns);
    int sp = 0;
    int c = s_l0[0];
    // last cell to visit: the last source's support end, or the tile's end
    int c_end;
    {
      double ul = (rs[it.je - 1] - bx.C) / bx.h;
      c_end = (int)ceil(ul - 0.5 * W) + W - 1;
      if (WINDOWED) c_end = min(c_end, it.l_start + nc - 1);
    }
    int last = INT_MIN / 2;  // cell of the latest source added
    bool done = c > c_end;
    while (!done) {
#pragma unroll
      for (int jj = 0; jj < W; ++jj) {
        // sources whose support starts at cell c (ring position jj)
        for (;;) {
          if (sp < ns && s_l0[sp] == c) {
            // the run of sources with l0 == c in this chunk: a known trip count, two
            // sources per step so that the shared loads of both issue together
            const int e = s_end[sp];
            if (tl < BT) {
              auto add = [&](int s) {
                const C2 rq = s_rq[s * NG + g];
                T a = s_c[tl * SCP + s] * rq.x;
                C2 wc[WE];
                load_weights<WE>(s_wc + s * WE, wc);
#pragma unroll
                for (int u = 0; u < LPT; ++u) {
#pragma unroll
                  for (int q = 0; q < W; ++q) cfma(acc[u][(jj + q) % W], wc[q], a);
                  a *= rq.y;
                }
              };
#pragma unroll 1
              for (int s = sp; s < e; ++s) add(s);
            }
            last = c;
            sp = e;
          }
          if (sp < ns || s0 + ns >= it.je) break;
          s0 += ns;
          ns = min(kSpreadChunk, it.je - s0);
          stage(s0, ns);
          sp = 0;
        }
        // cell c is final
        if (active) {
          if (WINDOWED) {
            const int cl = c - it.l_start;
            if (cl >= 0 && cl < nc) {
              if (DIRECT) {
                // the CTA owns the cell: zeros for the owned cells skipped before it, then
                // the cell scaled by 1/psi-hat, for each vector
                zero_to(c);
                zc = c + 1;
                const int idx = it.fft_start + cl;
#pragma unroll
                for (int u = 0; u < LPT; ++u) gbox[(size_t)(v0 + vloc + u) * bx.n2 + idx] = acc[u][jj];
              } else {
#pragma unroll
                for (int u = 0; u < LPT; ++u) win[cl * WP + vloc + u] = acc[u][jj];
              }
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
        const int nxt = sp < ns ? s_l0[sp] : INT_MAX;
        if (c >= last + W - 1 && nxt != INT_MAX && nxt > c + 1) c = nxt;
        else ++c;
      }
    }
  }
  zero_to(INT_MAX);  // owned cells after the walk (or all of them when no source reaches the tile)
  if (!WINDOWED || DIRECT) return;
  __syncthreads();
  // Transposed write-out of the CTA's own cells: consecutive threads take consecutive
  // cells of one vector.
  for (int e = tid; e < nc * nv; e += nthr) {
    int vv = e / nc, cell = e - vv * nc;
    gbox[(size_t)(v0 + vv) * bx.n2 + it.fft_start + cell] = win[cell * WP + vv];
  }
}

// Stage 3.  Thread (tl, g) owns terms g LPT .. g LPT + LPT - 1 of column t0 + tl.  Targets
// are sorted, so the first cell q0 of their stencil never decreases; the CTA walks the cells
// in order with a ring of R = W + 1 grid values per vector in registers (the stencil plus one
// cell fetched a step ahead); the walk is unrolled R times, which makes every ring index a
// compile-time constant.  Each thread combines its terms with the per-target factors mu
// (rounded to the arithmetic type from their FP64 values) and leaves its partial sum in
// shared memory; at the end of each chunk of targets the NG partials of a column are added
// in FP64 and atomically into g, consecutive threads taking consecutive targets of a column.
// (Warp shuffles for the partial sums measured slower on B200.)
template <typename T, int W, int LPT>
__global__ void __launch_bounds__(256) k_asy_interp(
    const double* __restrict__ ws, double* __restrict__ gs, int ld_gs, int B,
    const typename Cplx<T>::type* __restrict__ grid, const AsyBoxD* __restrict__ boxes,
    const InterpItem* __restrict__ items, const double2* __restrict__ post, AsyConst P, int BT,
    int V_total, double sgn) {
  using C2 = typename Cplx<T>::type;
  constexpr int WE = interp_we<T>(W);
  constexpr int R = W + 1;
  const InterpItem it = items[blockIdx.x];
  const AsyBoxD bx = boxes[it.box];
  const int NLP = P.NLP;
  const int NG = NLP / LPT;
  const int nthr = blockDim.x;
  const int YP = nthr + 1;  // padded row of the per-target partial sums
  const int tid = threadIdx.x;
  const int tl = tid / NG, g = tid - tl * NG;
  const int t0 = blockIdx.y * BT;
  const bool active = tl < BT && t0 + tl < B;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const InterpSmem L = interp_smem<T>(W, NLP, nthr);
  C2* s_mu = reinterpret_cast<C2*>(smem_raw + L.mu);        // [KC][NLP]
  T* s_y = reinterpret_cast<T*>(smem_raw + L.y);  // [KC][YP]: per-thread partial sums (already in T)
  T* s_wt = reinterpret_cast<T*>(smem_raw + L.wt);          // [KC][WE]
  int* s_q0 = reinterpret_cast<int*>(smem_raw + L.q0);      // [KC]
  int* s_end = reinterpret_cast<int*>(smem_raw + L.end);    // [KC]: end of the equal-q0 run
  double* s_uu = reinterpret_cast<double*>(smem_raw + L.uu);  // [KC]: target position in cells

  const int n2 = bx.n2;
  const C2* row[LPT];
#pragma unroll
  for (int u = 0; u < LPT; ++u)
    row[u] = grid + (size_t)bx.cell_off * (size_t)B +
             (size_t)(active ? (t0 + tl) * NLP + g * LPT + u : 0) * (size_t)n2;
  const T ihw = (T)(2.0 / (double)W);
  const T beta = (T)P.beta;
  const double u_scale = bx.h * (double)n2 / (2.0 * M_PI);

  auto fetch = [&](int cell, int u) -> C2 {
    int idx = cell < 0 ? cell + n2 : (cell >= n2 ? cell - n2 : cell);
    return active ? row[u][idx] : cmake<T>(0, 0);
  };

  // Stage targets [k0, k0 + nk) (all threads; barriers on both sides).
  auto stage = [&](int k0, int nk) {
    __syncthreads();
    // per target (one thread each): stencil start, and the NLP factors
    // mu_q = coef_q (k rref)^{-(q + 1/2)} exp(i (phi + k C)) / psi-hat, rotated by i for odd q,
    // with one square root and one reciprocal per target
    for (int kk = tid; kk < nk; kk += nthr) {
      const double k = ws[k0 + kk];
      const double uu = (k - bx.D) * u_scale;
      s_uu[kk] = uu;
      s_q0[kk] = (int)ceil(uu - 0.5 * W);
      const double2 ps = post[bx.post_off + (k0 + kk - bx.i0)];
      const double kr = k * bx.rref;
      const double ik = 1.0 / kr;
      double pw = sqrt(ik);
      for (int q = 0; q < NLP; ++q, pw *= ik) {
        const double sc = P.coef[q] * pw;
        const double mr = sc * ps.x, mi = sc * ps.y;
        s_mu[kk * NLP + q] = (q & 1) ? cmake<T>((T)-mi, (T)mr) : cmake<T>((T)mr, (T)mi);
      }
    }
    __syncthreads();
    // kernel weights over all (target, tap) pairs
    for (int e = tid; e < nk * WE; e += nthr) {
      const int kk = e / WE, q = e - kk * WE;
      s_wt[e] = q < W ? es_kernel_t((T)(s_uu[kk] - (double)(s_q0[kk] + q)), ihw, beta) : (T)0;
    }
    for (int kk = tid; kk < nk; kk += nthr) s_end[kk] = run_end(s_q0, nk, kk);
    __syncthreads();
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
  stage(k0, nk);
  int kp = 0;
  int c = s_q0[0];
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
        if (kp < nk && s_q0[kp] == c) {
          const int e = s_end[kp];
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
        k0 += nk;
        nk = min(kInterpChunk, it.ke - k0);
        stage(k0, nk);
        kp = 0;
      }
      if (done) break;
      // advance to the next target's cell; ring position jj + 1 stands for it
      const int nxt = s_q0[kp];
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
