// Device planner: the reference's box partition (generate_boxes / split_box,
// src/fast_hankel_nufht.c:498-744) computed on the GPU from device-resident sorted grids,
// with the same boxes in the same order as the host planner (planner.cpp) and the reference.
//
// The reference's first-element-above-threshold scans (find_first_*, :454-466) are binary
// searches here (the grids are non-decreasing, the thresholds z / k and z / r monotone).  The
// recursive split of the direct region runs level-synchronously: per level one kernel gives
// every direct box a warp whose lanes evaluate the ten candidate rows of split_box in
// parallel (the first candidate with the largest local + asymptotic area wins, as in the
// reference), and one single-CTA kernel turns the per-box child counts into offsets (block
// scan) and writes the children in box order.  Nothing returns to the host between levels;
// the final reclassification of small boxes into direct ones is one more scan, and only the
// box lists are copied back.  Input validation (finite, non-negative, non-decreasing) is a
// device reduction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "kernels_common.cuh"
#include "nufht_internal.h"

namespace hankel {
namespace {

constexpr int kScanThreads = 1024;

// First index with a[index] > thr in the non-decreasing a[0, len), or -1.
__device__ __forceinline__ int d_first_greater(const double* __restrict__ a, int len, double thr) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = lo + ((hi - lo) >> 1);
    if (a[mid] > thr) hi = mid;
    else lo = mid + 1;
  }
  return lo == len ? -1 : lo;
}

struct PartState {
  int n_dir;    // direct boxes of the current level
  int n_loc;    // local boxes so far
  int n_asy;    // asymptotic boxes so far
  int overflow; // a list outgrew its buffer
};

// Split decisions of one level: warp w takes box w (grid-stride); lanes 0..9 evaluate the
// candidate rows of split_box.  Per box: split flag, split row/column and child counts.
__global__ void k_split_level(const double* __restrict__ rs, int m, const double* __restrict__ ws, double z,
                              int min_dim_prod, const HBox* __restrict__ dir, const PartState* __restrict__ st,
                              int4* __restrict__ dec) {
  const int nd = st->n_dir;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nd; w += warps) {
    const HBox b = dir[w];
    const long long d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
    if (!(d1 * d2 > 4LL * (long long)min_dim_prod)) {
      if (lane == 0) dec[w] = make_int4(0, 0, 0, 0);  // kept: no split
      continue;
    }
    // candidate rows: round(i0 + t (i1 - i0)), t = k/9, consecutive duplicates dropped
    int cand = -1;
    bool fresh = false;
    if (lane < 10) {
      if (b.i1 <= b.i0) {
        cand = b.i0;
        fresh = lane == 0;
      } else {
        auto row = [&](int k) {
          // the same rounding as the host: no fused multiply-add
          const double t = (double)k / 9.0;
          int idx = (int)llround(__dadd_rn((double)b.i0, __dmul_rn(t, (double)(b.i1 - b.i0))));
          return min(max(idx, b.i0), b.i1);
        };
        cand = row(lane);
        fresh = lane == 0 || cand != row(lane - 1);
      }
    }
    long long v = -1;
    if (fresh) {
      const int j = d_first_greater(rs, m, z / ws[cand]);
      v = 0;
      if (j >= 0)
        v = (long long)(cand - b.i0 + 1) * (long long)(j - b.j0 + 1) +
            (long long)(b.i1 - cand + 1) * (long long)(b.j1 - j + 1);
    }
    // first lane with the largest value (the reference keeps the first strict maximum)
    long long best = v;
    int bl = fresh ? lane : 32;
    for (int off = 16; off > 0; off >>= 1) {
      const long long ov = __shfl_xor_sync(0xffffffffu, best, off);
      const int ol = __shfl_xor_sync(0xffffffffu, bl, off);
      if (ov > best || (ov == best && ol < bl)) {
        best = ov;
        bl = ol;
      }
    }
    const int is = __shfl_sync(0xffffffffu, cand, bl & 31);
    if (lane == 0) {
      int js = d_first_greater(rs, m, z / ws[is]);
      if (js < 0) js = b.j0;
      dec[w] = make_int4(1, is, js, 0);
    }
  }
}

// Exclusive block scan of one int per thread (kScanThreads threads); returns the total.
__device__ int block_scan(int v, int* s_tmp, int* out_excl) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  int x = v;
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) s_tmp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = lane < (kScanThreads >> 5) ? s_tmp[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, off);
      if (lane >= off) s += y;
    }
    s_tmp[lane] = s;  // inclusive prefix of the warp totals
  }
  __syncthreads();
  const int warp_base = wid > 0 ? s_tmp[wid - 1] : 0;
  *out_excl = warp_base + x - v;
  const int total = s_tmp[(kScanThreads >> 5) - 1];
  __syncthreads();
  return total;
}

// Children of one level in box order: for a split box (i0..i1, j0..j1) at (is, js) the
// reference appends loc (i0, is-1, j0, js-1) and direct (i0, is-1, js, j1) when is > i0, then
// asy (is, i1, js, j1) and direct (is, i1, j0, js-1); a kept box is carried over.
__global__ void __launch_bounds__(kScanThreads) k_emit_level(const HBox* __restrict__ dir, const int4* __restrict__ dec,
                                                           PartState* st, HBox* __restrict__ next, int cap_dir,
                                                           HBox* __restrict__ loc, int cap_loc, HBox* __restrict__ asy,
                                                           int cap_asy) {
  __shared__ int s_tmp[32];
  __shared__ int s_base[3];
  const int nd = st->n_dir;
  if (threadIdx.x == 0) {
    s_base[0] = 0;
    s_base[1] = st->n_loc;
    s_base[2] = st->n_asy;
  }
  __syncthreads();
  for (int c0 = 0; c0 < nd; c0 += kScanThreads) {
    const int w = c0 + threadIdx.x;
    HBox b{0, 0, 0, 0};
    int4 d = make_int4(0, 0, 0, 0);
    if (w < nd) {
      b = dir[w];
      d = dec[w];
    }
    const bool split = w < nd && d.x;
    const bool has_low = split && d.y > b.i0;
    const int n_next = w < nd ? (split ? (has_low ? 2 : 1) : 1) : 0;
    const int n_loc = has_low ? 1 : 0;
    const int n_asy = split ? 1 : 0;
    int o_next, o_loc, o_asy;
    const int t_next = block_scan(n_next, s_tmp, &o_next);
    const int t_loc = block_scan(n_loc, s_tmp, &o_loc);
    const int t_asy = block_scan(n_asy, s_tmp, &o_asy);
    const int pn = s_base[0] + o_next, pl = s_base[1] + o_loc, pa = s_base[2] + o_asy;
    if (w < nd) {
      const bool fits = pn + n_next <= cap_dir && pl + n_loc <= cap_loc && pa + n_asy <= cap_asy;
      if (!fits) {
        st->overflow = 1;
      } else if (!split) {
        next[pn] = b;
      } else {
        const int is = d.y, js = d.z;
        int q = pn;
        if (has_low) {
          loc[pl] = HBox{b.i0, is - 1, b.j0, js - 1};
          next[q++] = HBox{b.i0, is - 1, js, b.j1};
        }
        asy[pa] = HBox{is, b.i1, js, b.j1};
        next[q] = HBox{is, b.i1, b.j0, js - 1};
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_base[0] += t_next;
      s_base[1] += t_loc;
      s_base[2] += t_asy;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st->n_dir = min(s_base[0], cap_dir);
    st->n_loc = min(s_base[1], cap_loc);
    st->n_asy = min(s_base[2], cap_asy);
  }
}

// Final reclassification (generate_boxes, :719-741): local boxes thinner than Kthr and
// asymptotic boxes with area below min_dim_prod join the direct list, in that order after
// the last level's direct boxes.  Writes the final lists (loc, asy, dir) and their counts.
__global__ void __launch_bounds__(kScanThreads) k_classify(const HBox* __restrict__ loc, const HBox* __restrict__ asy,
                                                         const HBox* __restrict__ dir, const PartState* __restrict__ st,
                                                         int Kthr, int min_dim_prod, HBox* __restrict__ out_loc,
                                                         HBox* __restrict__ out_asy, HBox* __restrict__ out_dir,
                                                         int* __restrict__ counts) {
  __shared__ int s_tmp[32];
  __shared__ int s_nl, s_na, s_nd;
  const int nl = st->n_loc, na = st->n_asy, nd = st->n_dir;
  if (threadIdx.x == 0) {
    s_nl = 0;
    s_na = 0;
    s_nd = nd;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nd; e += kScanThreads) out_dir[e] = dir[e];
  for (int pass = 0; pass < 2; ++pass) {
    const HBox* src = pass == 0 ? loc : asy;
    const int ns = pass == 0 ? nl : na;
    HBox* keep = pass == 0 ? out_loc : out_asy;
    for (int c0 = 0; c0 < ns; c0 += kScanThreads) {
      const int w = c0 + threadIdx.x;
      HBox b{0, 0, 0, 0};
      bool to_dir = false;
      if (w < ns) {
        b = src[w];
        const int d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
        to_dir = pass == 0 ? min(d1, d2) < Kthr
                           : (long long)d1 * (long long)d2 < (long long)min_dim_prod;
      }
      int o_dir, o_keep;
      const int t_dir = block_scan(w < ns && to_dir ? 1 : 0, s_tmp, &o_dir);
      const int t_keep = block_scan(w < ns && !to_dir ? 1 : 0, s_tmp, &o_keep);
      if (w < ns) {
        if (to_dir) out_dir[s_nd + o_dir] = b;
        else keep[(pass == 0 ? s_nl : s_na) + o_keep] = b;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s_nd += t_dir;
        if (pass == 0) s_nl += t_keep;
        else s_na += t_keep;
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    counts[0] = s_nl;
    counts[1] = s_na;
    counts[2] = s_nd;
  }
}

// The rectangle's boundary indices (generate_boxes, :608-640): out = {i0, i1, j0, j1}.
__global__ void k_bounds(const double* __restrict__ rs, int m, const double* __restrict__ ws, int n, double z,
                         int* __restrict__ out) {
  if (threadIdx.x != 0) return;
  const int i0 = d_first_greater(ws, n, z / rs[m - 1]);
  int i1;
  if (m == 1) {
    i1 = i0 == -1 ? -1 : i0 - 1;
  } else {
    const int idx = d_first_greater(ws, n, z / rs[0]);
    i1 = idx == -1 ? n - 1 : idx - 1;
  }
  const int j0 = d_first_greater(rs, m, z / ws[n - 1]);
  int j1;
  if (n == 1) {
    j1 = j0 == -1 ? -1 : j0 - 1;
  } else {
    const int idx = d_first_greater(rs, m, z / ws[0]);
    j1 = idx == -1 ? m - 1 : idx - 1;
  }
  out[0] = i0;
  out[1] = i1;
  out[2] = j0;
  out[3] = j1;
}

// flags |= 1 when a[0, len) is not finite, non-negative and non-decreasing.
__global__ void k_check_grid(const double* __restrict__ a, long len, int* __restrict__ flag) {
  bool bad = false;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) {
    const double v = a[i];
    if (!isfinite(v) || v < 0.0 || (i > 0 && v < a[i - 1])) bad = true;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)); }
};

}  // namespace

int device_check_grid(const double* d_a, int len, cudaStream_t st) {
  DevBuf<int> flag;
  NUFHT_CUDA_TRY(flag.alloc(1));
  NUFHT_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  const int blocks = std::max(1, std::min(148 * 4, (len + 255) / 256));
  k_check_grid<<<blocks, 256, 0, st>>>(d_a, len, flag.p);
  NUFHT_LAUNCH_CHECK();
  int h = 0;
  NUFHT_CUDA_TRY(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  NUFHT_CUDA_TRY(cudaStreamSynchronize(st));
  return h ? -1 : 0;
}

namespace {

// Initial state of the partition (generate_boxes, :608-657) from the boundary indices
// {i0, i1, j0, j1}: the local and asymptotic strips around the direct region and the direct
// region itself as the first level's only box; out_flags[0] = 1 when the rectangle is all
// local, 2 all asymptotic, 3 when m == 1 or n == 1 (strips only).
__global__ void k_init_partition(const int* __restrict__ bnd, int m, int n, PartState* st, HBox* dir, HBox* loc,
                                 HBox* asy, int* out_flags) {
  if (threadIdx.x != 0) return;
  const int i0 = bnd[0], i1 = bnd[1], j0 = bnd[2], j1 = bnd[3];
  int nl = 0, na = 0, flag = 0;
  if (i0 == -1) {
    loc[nl++] = HBox{0, n - 1, 0, m - 1};
    flag = 1;
  } else if (i1 < 0) {
    asy[na++] = HBox{0, n - 1, 0, m - 1};
    flag = 2;
  } else {
    if (i0 > 0) loc[nl++] = HBox{0, i0 - 1, 0, m - 1};
    if (j0 > 0) loc[nl++] = HBox{i0, n - 1, 0, j0 - 1};
    if (i1 < n - 1) asy[na++] = HBox{i1 + 1, n - 1, 0, m - 1};
    if (j1 < m - 1) asy[na++] = HBox{0, i1, j1 + 1, m - 1};
    if (m == 1 || n == 1) flag = 3;
  }
  dir[0] = HBox{i0, i1, j0, j1};
  st->n_dir = flag ? 0 : 1;
  st->n_loc = nl;
  st->n_asy = na;
  st->overflow = 0;
  out_flags[0] = flag;
}

}  // namespace

int device_make_boxes(const double* d_rs, int m, const double* d_ws, int n, double z, int max_levels,
                      int min_dim_prod, int Kthr, HBoxes* out, cudaStream_t st, int* bad_grid) {
  out->loc.clear();
  out->asy.clear();
  out->dir.clear();
  if (bad_grid) *bad_grid = 0;
  if (n <= 0 || m <= 0) return 0;
  if (max_levels <= 0) {
    const int mn = std::min(n, m);
    const double ratio = (double)mn * (double)mn / (double)min_dim_prod;
    max_levels = ratio < 1.0 ? 0 : (int)std::floor(std::log2(ratio));
    if (max_levels < 0) max_levels = 0;
  }
  // One device arena per attempt: the state and small counters, then the box lists.  The lists
  // start at 64K boxes each (far above the partitions of the workloads seen: about a thousand
  // boxes at 1e6 x 1e6) and grow 16-fold when one overflowed.
  for (long cap = 1L << 16;; cap *= 16) {
    if (cap > (1L << 28)) {
      std::fprintf(stderr, "nufht_b200: device planner box lists too long\n");
      return NUFHT_E_TOO_LARGE;
    }
    const size_t head = 256;  // PartState, bounds, flags, counts
    const size_t nb = (size_t)cap;
    DevBuf<unsigned char> arena;
    NUFHT_CUDA_TRY(arena.alloc(head + sizeof(HBox) * nb * 8 + sizeof(int4) * nb));
    unsigned char* a = arena.p;
    PartState* dSt = reinterpret_cast<PartState*>(a);
    int* dBnd = reinterpret_cast<int*>(a + 64);      // 4 ints
    int* dFlag = reinterpret_cast<int*>(a + 96);     // [0] trivial-rectangle flag, [1] bad rs, [2] bad ws
    int* dCnt = reinterpret_cast<int*>(a + 128);     // final counts
    HBox* dA = reinterpret_cast<HBox*>(a + head);
    HBox* dB = dA + nb;
    HBox* dLoc = dB + nb;
    HBox* dAsy = dLoc + nb;
    HBox* oLoc = dAsy + nb;
    HBox* oAsy = oLoc + nb;
    HBox* oDir = oAsy + nb;  // 2 nb: the last level's boxes plus reclassified ones
    int4* dDec = reinterpret_cast<int4*>(oDir + 2 * nb);
    NUFHT_CUDA_TRY(cudaMemsetAsync(dFlag, 0, 3 * sizeof(int), st));
    if (bad_grid) {
      const int br = std::max(1, std::min(148 * 4, (m + 255) / 256)), bw = std::max(1, std::min(148 * 4, (n + 255) / 256));
      k_check_grid<<<br, 256, 0, st>>>(d_rs, m, dFlag + 1);
      NUFHT_LAUNCH_CHECK();
      k_check_grid<<<bw, 256, 0, st>>>(d_ws, n, dFlag + 2);
      NUFHT_LAUNCH_CHECK();
    }
    k_bounds<<<1, 32, 0, st>>>(d_rs, m, d_ws, n, z, dBnd);
    NUFHT_LAUNCH_CHECK();
    k_init_partition<<<1, 32, 0, st>>>(dBnd, m, n, dSt, dA, dLoc, dAsy, dFlag);
    NUFHT_LAUNCH_CHECK();
    HBox* cur = dA;
    HBox* nxt = dB;
    for (int lev = 0; lev < max_levels; ++lev) {
      k_split_level<<<148 * 4, 256, 0, st>>>(d_rs, m, d_ws, z, min_dim_prod, cur, dSt, dDec);
      NUFHT_LAUNCH_CHECK();
      k_emit_level<<<1, kScanThreads, 0, st>>>(cur, dDec, dSt, nxt, (int)cap, dLoc, (int)cap, dAsy, (int)cap);
      NUFHT_LAUNCH_CHECK();
      std::swap(cur, nxt);
    }
    k_classify<<<1, kScanThreads, 0, st>>>(dLoc, dAsy, cur, dSt, Kthr, min_dim_prod, oLoc, oAsy, oDir, dCnt);
    NUFHT_LAUNCH_CHECK();
    struct {
      PartState s;    // offset 0
      int pad[20];
      int flag[3];    // offset 96
      int pad2[5];
      int cnt[3];     // offset 128
    } h;
    static_assert(sizeof(PartState) == 16 && sizeof(h) == 140, "arena layout");
    NUFHT_CUDA_TRY(cudaMemcpyAsync(&h, a, sizeof(h), cudaMemcpyDeviceToHost, st));
    NUFHT_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.flag[1] || h.flag[2]) {
      if (bad_grid) *bad_grid = h.flag[1] ? 1 : 2;
      return 0;
    }
    if (h.s.overflow) continue;
    const int cl = h.flag[0] == 0 ? h.cnt[0] : h.s.n_loc;
    const int ca = h.flag[0] == 0 ? h.cnt[1] : h.s.n_asy;
    const int cd = h.flag[0] == 0 ? h.cnt[2] : 0;
    const HBox* sl = h.flag[0] == 0 ? oLoc : dLoc;
    const HBox* sa = h.flag[0] == 0 ? oAsy : dAsy;
    out->loc.resize(cl);
    out->asy.resize(ca);
    out->dir.resize(cd);
    if (cl) NUFHT_CUDA_TRY(cudaMemcpyAsync(out->loc.data(), sl, sizeof(HBox) * cl, cudaMemcpyDeviceToHost, st));
    if (ca) NUFHT_CUDA_TRY(cudaMemcpyAsync(out->asy.data(), sa, sizeof(HBox) * ca, cudaMemcpyDeviceToHost, st));
    if (cd) NUFHT_CUDA_TRY(cudaMemcpyAsync(out->dir.data(), oDir, sizeof(HBox) * cd, cudaMemcpyDeviceToHost, st));
    NUFHT_CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
  }
}

}  // namespace hankel
