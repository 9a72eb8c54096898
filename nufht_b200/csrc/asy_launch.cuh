// Launchers of the asymptotic-box kernels (spread, FFT, interpolation) for one arithmetic
// type; included by asy_f32.cu and asy_f64.cu, one instantiation each, so that the two
// precisions compile in parallel.
#pragma once

#include <cufft.h>

#include <algorithm>
#include <cstdlib>

#include "executor.h"
#include "kernels_asy.cuh"

namespace hankel {
namespace {

AsyShape asy_shape(int NLP, int B, int LPT) {
  AsyShape L;
  L.LPT = LPT;
  L.NG = NLP / LPT;
  // columns per CTA: up to 32, a multiple of 4 (16-byte pieces of the packed coefficients)
  int cap = std::max(4, std::min(256 / L.NG, 32) & ~3);
  L.BT = std::min(cap, B);
  L.threads = L.BT * L.NG;
  L.V_total = NLP * B;
  L.ngy = (B + L.BT - 1) / L.BT;
  return L;
}

// Sources per shared-memory round of spreading (NUFHT_B200_SPREAD_CHUNK, 16..64, default 64).
inline int spread_chunk() {
  static const int v = [] {
    const char* e = std::getenv("NUFHT_B200_SPREAD_CHUNK");
    const int q = e ? std::atoi(e) : kSpreadChunk;
    return (q >= 16 && q <= kSpreadChunk) ? q : kSpreadChunk;
  }();
  return v;
}

template <typename T, int W, int LPT, bool TILE>
int launch_spread_kind(DevicePlan& D, const AsyClass& K, int item0, int nitems, int B, cudaStream_t st) {
  if (nitems == 0) return 0;
  using C2 = typename Cplx<T>::type;
  const AsyShape L = asy_shape(K.ac.NLP, B, LPT);
  const int sch = spread_chunk();
  const size_t sm = spread_smem<T>(W, K.ac.NLP, spread_btp<T>(L.BT), sch).total;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_asy_spread<T, W, LPT, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    attr_set = true;
  }
  dim3 g((unsigned)nitems, (unsigned)L.ngy);
  k_asy_spread<T, W, LPT, TILE><<<g, L.threads, sm, st>>>(
      static_cast<const T*>(D.d_ct), D.ldct, B, static_cast<C2*>(D.d_grid), D.d_asyb, D.d_spread + item0,
      D.d_rec_l0, static_cast<const T*>(D.d_rec_w), static_cast<const C2*>(D.d_rec_p), K.ac.NLP, L.BT, L.V_total,
      sch);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

// Tiles (and the zero padding) own their cells; the source chunks of dense boxes add theirs
// atomically.
template <typename T, int W, int LPT>
int launch_spread_lpt(DevicePlan& D, const AsyClass& K, int B, cudaStream_t st) {
  int rc = launch_spread_kind<T, W, LPT, true>(D, K, K.spread0, K.nspread, B, st);
  if (rc) return rc;
  return launch_spread_kind<T, W, LPT, false>(D, K, K.spreadA0, K.nspreadA, B, st);
}

template <typename T, int W, int LPT>
int launch_interp_lpt(DevicePlan& D, const AsyClass& K, double* gs, int ld_gs, int B, cudaStream_t st,
                      double sgn) {
  const AsyShape L = asy_shape(K.ac.NLP, B, LPT);
  size_t sm = interp_smem<T>(W, K.ac.NLP, L.threads).total;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_asy_interp<T, W, LPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    attr_set = true;
  }
  dim3 g((unsigned)K.ninterp, (unsigned)L.ngy);
  using C2 = typename Cplx<T>::type;
  k_asy_interp<T, W, LPT><<<g, L.threads, sm, st>>>(gs, ld_gs, B, static_cast<const C2*>(D.d_grid), D.d_asyb,
                                                    D.d_interp + K.interp0, D.d_tq0, static_cast<const T*>(D.d_tw),
                                                    static_cast<const C2*>(D.d_tmu), K.ac.NLP, L.BT, sgn);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

// Terms per thread (register blocking): LPT = 2, or 1 in double precision for windows wider
// than 10 (register budget) and for classes of at most 4 terms (so that a CTA keeps at least
// two warps' worth of threads, NLP / LPT per column); NLP = 2 (K + 1) is even.
// NUFHT_B200_SPREAD_LPT_SMALL=2 / NUFHT_B200_INTERP_LPT_SMALL=2 keep two terms per thread for
// the classes of at most 4 terms in spreading / interpolation.
inline int lpt_small(bool interp) {
  static const int vs = [] {
    const char* e = std::getenv("NUFHT_B200_SPREAD_LPT_SMALL");
    return (e && e[0] == '2') ? 2 : 1;
  }();
  static const int vi = [] {
    const char* e = std::getenv("NUFHT_B200_INTERP_LPT_SMALL");
    return (e && e[0] == '2') ? 2 : 1;
  }();
  return interp ? vi : vs;
}

template <typename T>
int build_records_t(DevicePlan& D) {
  using C2 = typename Cplx<T>::type;
  if (D.asyb.empty()) return 0;
  const size_t b0 = sizeof(int) * (size_t)D.total_rec, b1 = sizeof(T) * (size_t)D.total_recw,
               b2 = sizeof(C2) * (size_t)D.total_recp;
  const size_t b3 = sizeof(int) * (size_t)D.total_post, b4 = sizeof(T) * (size_t)D.total_tw,
               b5 = sizeof(C2) * (size_t)D.total_tm;
  NUFHT_CUDA_TRY(cudaMalloc((void**)&D.d_rec_l0, b0));
  NUFHT_CUDA_TRY(cudaMalloc(&D.d_rec_w, b1));
  NUFHT_CUDA_TRY(cudaMalloc(&D.d_rec_p, b2));
  NUFHT_CUDA_TRY(cudaMalloc((void**)&D.d_tq0, b3));
  NUFHT_CUDA_TRY(cudaMalloc(&D.d_tw, b4));
  NUFHT_CUDA_TRY(cudaMalloc(&D.d_tmu, b5));
  D.rec_bytes = b0 + b1 + b2 + b3 + b4 + b5;
  for (size_t q0 = 0; q0 < D.asyb.size();) {
    size_t q1 = q0;
    while (q1 < D.asyb.size() && D.asyb[q1].cls == D.asyb[q0].cls && q1 - q0 < 65535) ++q1;
    const AsyClass& K = D.classes[D.asyb[q0].cls];
    k_asy_records<T><<<dim3(64, (unsigned)(q1 - q0)), 256>>>(D.d_rs, D.d_asyb + q0, K.ac, K.W, D.d_corr,
                                                              D.d_rec_l0, static_cast<T*>(D.d_rec_w),
                                                              static_cast<C2*>(D.d_rec_p));
    NUFHT_LAUNCH_CHECK();
    k_asy_target_records<T><<<dim3(64, (unsigned)(q1 - q0)), 256>>>(D.d_ws, D.d_asyb + q0, K.ac, K.W, D.d_tq0,
                                                                     static_cast<T*>(D.d_tw),
                                                                     static_cast<C2*>(D.d_tmu));
    NUFHT_LAUNCH_CHECK();
    q0 = q1;
  }
  return 0;
}

template <typename T, int W>
int launch_spread(DevicePlan& D, const AsyClass& K, int B, cudaStream_t st) {
  if constexpr (sizeof(T) == 8 && W > 10) return launch_spread_lpt<T, W, 1>(D, K, B, st);
  else if (K.ac.NLP <= 4 && lpt_small(false) == 1) return launch_spread_lpt<T, W, 1>(D, K, B, st);
  else return launch_spread_lpt<T, W, 2>(D, K, B, st);
}


template <typename T, int W>
int launch_interp(DevicePlan& D, const AsyClass& K, double* gs, int ld_gs, int B, cudaStream_t st, double sgn) {
  if (K.ninterp == 0) return 0;
  if constexpr (sizeof(T) == 8 && W > 10) return launch_interp_lpt<T, W, 1>(D, K, gs, ld_gs, B, st, sgn);
  else if (K.ac.NLP <= 4 && lpt_small(true) == 1) return launch_interp_lpt<T, W, 1>(D, K, gs, ld_gs, B, st, sgn);
  else return launch_interp_lpt<T, W, 2>(D, K, gs, ld_gs, B, st, sgn);
}

#define NUFHT_W_DISPATCH(FN, T, Wv, ...)          \
  switch (Wv) {                                   \
    case 2: rc = FN<T, 2>(__VA_ARGS__); break;    \
    case 3: rc = FN<T, 3>(__VA_ARGS__); break;    \
    case 4: rc = FN<T, 4>(__VA_ARGS__); break;    \
    case 5: rc = FN<T, 5>(__VA_ARGS__); break;    \
    case 6: rc = FN<T, 6>(__VA_ARGS__); break;    \
    case 7: rc = FN<T, 7>(__VA_ARGS__); break;    \
    case 8: rc = FN<T, 8>(__VA_ARGS__); break;    \
    case 9: rc = FN<T, 9>(__VA_ARGS__); break;    \
    case 10: rc = FN<T, 10>(__VA_ARGS__); break;  \
    case 11: rc = FN<T, 11>(__VA_ARGS__); break;  \
    case 12: rc = FN<T, 12>(__VA_ARGS__); break;  \
    case 13: rc = FN<T, 13>(__VA_ARGS__); break;  \
    case 14: rc = FN<T, 14>(__VA_ARGS__); break;  \
    case 15: rc = FN<T, 15>(__VA_ARGS__); break;  \
    default: rc = FN<T, 16>(__VA_ARGS__); break;  \
  }

template <typename T>
int exec_fft(const FftGroup& gr, T* grid, int B, cudaStream_t st) {
  using C2 = typename Cplx<T>::type;
  cufftSetStream(gr.plan, st);
  C2* p = reinterpret_cast<C2*>(grid) + (size_t)gr.cell_off * B;
  cufftResult fr;
  if (sizeof(T) == 8)
    fr = cufftExecZ2Z(gr.plan, (cufftDoubleComplex*)p, (cufftDoubleComplex*)p, CUFFT_INVERSE);
  else
    fr = cufftExecC2C(gr.plan, (cufftComplex*)p, (cufftComplex*)p, CUFFT_INVERSE);
  return fr == CUFFT_SUCCESS ? 0 : NUFHT_E_CUDA;
}

// The asymptotic boxes.  Each kernel class owns disjoint grid rows, so in the concurrent
// form every class runs its own pipeline -- spreading, the FFTs of its groups,
// interpolation -- on its stream slot, with one fork and one join for all of them (small
// classes and small FFT groups overlap the large ones instead of waiting at phase
// boundaries).  With phase timing on (D.serial) the three phases run one after the other on
// the caller's stream, so that each phase's device time can be read.
template <typename T>
int run_asy_t(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
              double sgn) {
  using C2 = typename Cplx<T>::type;
  int rc = 0;
  C2* grid = static_cast<C2*>(D.d_grid);
  if (!D.serial) {
    if (D.chunk_cell_end > D.chunk_cell_begin)
      NUFHT_CUDA_TRY(cudaMemsetAsync(grid + (size_t)D.chunk_cell_begin * B, 0,
                                     sizeof(C2) * (size_t)(D.chunk_cell_end - D.chunk_cell_begin) * B, st));
    {
      dim3 g((unsigned)((D.m + 31) / 32), (unsigned)((D.ldct + 31) / 32));
      k_pack_coefficients<T><<<g, dim3(32, 8), 0, st>>>(cs, ld_cs, B, D.m, static_cast<T*>(D.d_ct), D.ldct);
      NUFHT_LAUNCH_CHECK();
    }
    int used[DevicePlan::kAuxStreams];
    int nu = 0;
    for (int q = 0; q < DevicePlan::kAuxStreams - 2; ++q) {
      bool any = false;
      for (const AsyClass& K : D.classes) any = any || K.slot == q;
      if (any) used[nu++] = 2 + q;
    }
    if ((rc = fork_streams(D, st, used, nu))) return rc;
    for (int c = 0; c < (int)D.classes.size(); ++c) {
      const AsyClass& K = D.classes[c];
      if (K.slot < 0) continue;
      const cudaStream_t s = D.aux[2 + K.slot];
      if (K.nspread + K.nspreadA > 0) {
        NUFHT_W_DISPATCH(launch_spread, T, K.W, D, K, B, s);
        if (rc) return rc;
      }
      for (const FftGroup& gr : D.groups)
        if (gr.cls == c && (rc = exec_fft<T>(gr, reinterpret_cast<T*>(grid), B, s))) return rc;
      NUFHT_W_DISPATCH(launch_interp, T, K.W, D, K, gs, ld_gs, B, s, sgn);
      if (rc) return rc;
    }
    return join_streams(D, st, used, nu);
  }
  {
    PhaseScope ps(kPhaseSpread, st);
    if (D.chunk_cell_end > D.chunk_cell_begin)
      NUFHT_CUDA_TRY(cudaMemsetAsync(grid + (size_t)D.chunk_cell_begin * B, 0,
                                     sizeof(C2) * (size_t)(D.chunk_cell_end - D.chunk_cell_begin) * B, st));
    {  // coefficients source-major in the arithmetic type
      dim3 g((unsigned)((D.m + 31) / 32), (unsigned)((D.ldct + 31) / 32));
      k_pack_coefficients<T><<<g, dim3(32, 8), 0, st>>>(cs, ld_cs, B, D.m, static_cast<T*>(D.d_ct), D.ldct);
      NUFHT_LAUNCH_CHECK();
    }
    // the classes' boxes own disjoint grid ranges: their launches run concurrently
    int used[DevicePlan::kAuxStreams];
    int nu = 0;
    for (const AsyClass& K : D.classes) {
      if (K.nspread + K.nspreadA == 0) continue;
      if (nu < DevicePlan::kAuxStreams - 2) {
        used[nu] = 2 + nu;
        ++nu;
      }
    }
    if ((rc = fork_streams(D, st, used, nu))) return rc;
    int q = 0;
    for (const AsyClass& K : D.classes) {
      if (K.nspread + K.nspreadA == 0) continue;
      cudaStream_t cs_st = D.serial ? st : D.aux[used[q++ % nu]];
      NUFHT_W_DISPATCH(launch_spread, T, K.W, D, K, B, cs_st);
      if (rc) return rc;
    }
    if ((rc = join_streams(D, st, used, nu))) return rc;
  }
  {
    PhaseScope ps(kPhaseFft, st);
    for (const FftGroup& gr : D.groups)
      if ((rc = exec_fft<T>(gr, reinterpret_cast<T*>(grid), B, st))) return rc;
  }
  {
    PhaseScope ps(kPhaseInterp, st);
    // the classes add into g with atomics: their launches run concurrently
    int used[DevicePlan::kAuxStreams];
    int nu = 0;
    for (const AsyClass& K : D.classes) {
      if (K.ninterp == 0) continue;
      if (nu < DevicePlan::kAuxStreams - 2) {
        used[nu] = 2 + nu;
        ++nu;
      }
    }
    if ((rc = fork_streams(D, st, used, nu))) return rc;
    int q = 0;
    for (const AsyClass& K : D.classes) {
      if (K.ninterp == 0) continue;
      cudaStream_t cs_st = D.serial ? st : D.aux[used[q++ % nu]];
      NUFHT_W_DISPATCH(launch_interp, T, K.W, D, K, gs, ld_gs, B, cs_st, sgn);
      if (rc) return rc;
    }
    if ((rc = join_streams(D, st, used, nu))) return rc;
  }
  return 0;
}

}  // namespace
}  // namespace hankel
