// Allocation-free entry point: the local (Wimp) expansion of one box, with all of its
// scratch memory -- the work lists, the per-chunk partial Chebyshev projections and the
// projected coefficients -- in a fixed device array defined in this file instead of memory
// from cudaMalloc.
//
// For callers that cannot allocate device memory at call time: code running inside an
// application's own memory pool or allocator budget, real-time loops that forbid
// allocation after start-up, and library hosts that only hand out pre-sized buffers.
//
// Limits and behaviour:
//   * the scratch array holds kNoAllocScratchBytes (4 MiB) on every GPU that loads this
//     library, for the life of the process;
//   * a call needs about ceil(m/2048) * (K+1) * batch * 8 bytes of partial sums, plus
//     12 bytes per 2048 sources and per 128 targets of work lists; larger calls are
//     rejected with NUFHT_E_TOO_LARGE before anything runs;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call before any
//     stream capture;
//   * every call on a device shares the same array: calls whose kernels overlap on the GPU
//     (different streams, or different host threads) race and corrupt each other's
//     results; serialise them.  Each call rewrites every part of the array it reads, so
//     nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "executor.h"
#include "kernels_common.cuh"

namespace hankel {

constexpr size_t kNoAllocScratchBytes = 4u << 20;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocLocSources = 2048;  // sources per projection item (as the plan path)
constexpr int kNoAllocLocTargets = 128;   // targets per evaluation item (as the plan path)

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
int noalloc_scratch(unsigned char** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return NUFHT_E_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return NUFHT_E_TOO_LARGE;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "nufht_b200: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return NUFHT_E_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return 0;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Work lists of a single local box covering sources [0, m) and targets [0, n).
__global__ void k_noalloc_loc_items(const double* __restrict__ rs, int m, int n, LocBoxD* box,
                                    ProjItem* proj, int nproj, EvalItem* eval, int neval) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0) {
    LocBoxD b;
    b.i0 = 0;
    b.ni = n;
    b.j0 = 0;
    b.nj = m;
    b.r_end = rs[m - 1];
    b.item0 = 0;
    b.nitems = nproj;
    *box = b;
  }
  if (e < nproj) {
    int j = e * kNoAllocLocSources;
    proj[e] = ProjItem{0, j, min(kNoAllocLocSources, m - j)};
  }
  if (e < neval) {
    int i = e * kNoAllocLocTargets;
    eval[e] = EvalItem{0, i, min(kNoAllocLocTargets, n - i)};
  }
}

// Device memory of the current device (or managed memory, which any device can reach).
bool on_current_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace
}  // namespace hankel

extern "C" int nufht_b200_add_loc_batch_noalloc(double* gs, double nu, const double* rs, const double* cs,
                                                 const double* ws, int m, int n, int K, int batch, int ld_cs,
                                                 int ld_gs, void* stream) {
  using namespace hankel;
  if (!gs || !rs || !cs || !ws || m <= 0 || n <= 0 || batch <= 0 || K < 0) return -400;
  if (ld_cs < m || ld_gs < n) return -401;
  if (!is_integer(nu) || std::fabs(nu) > 200.0) return -2;
  // Every buffer, and the stream, must belong to the current device: the kernels and the
  // scratch array used are the current device's.
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return NUFHT_E_CUDA;
  if (!on_current_device(gs, dev) || !on_current_device(rs, dev) || !on_current_device(cs, dev) ||
      !on_current_device(ws, dev))
    return -400;
  if (stream) {
    int sdev = -1;
    if (cudaStreamGetDevice((cudaStream_t)stream, &sdev) != cudaSuccess) {
      cudaGetLastError();
      return -400;
    }
    if (sdev != dev) return -400;
  }
  const int nu_int = (int)std::llround(std::fabs(nu));
  // J_{-n} = (-1)^n J_n: odd negative orders add the negated expansion.
  const double sgn = (nu < 0.0 && (nu_int & 1)) ? -1.0 : 1.0;
  const int KL1 = K + 1;
  if (KL1 > 256 || nu_int / 2 + K + (nu_int & 1) > 512) return NUFHT_E_TOO_LARGE;
  const int nproj = (m + kNoAllocLocSources - 1) / kNoAllocLocSources;
  const int neval = (n + kNoAllocLocTargets - 1) / kNoAllocLocTargets;
  size_t off_box = 0;
  size_t off_proj = align256(off_box + sizeof(LocBoxD));
  size_t off_eval = align256(off_proj + sizeof(ProjItem) * (size_t)nproj);
  size_t off_part = align256(off_eval + sizeof(EvalItem) * (size_t)neval);
  size_t off_cheb = align256(off_part + sizeof(double) * (size_t)nproj * KL1 * batch);
  size_t total = off_cheb + sizeof(double) * (size_t)KL1 * batch;
  if (total > kNoAllocScratchBytes) return NUFHT_E_TOO_LARGE;
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  LocBoxD* d_box = reinterpret_cast<LocBoxD*>(base + off_box);
  ProjItem* d_proj = reinterpret_cast<ProjItem*>(base + off_proj);
  EvalItem* d_eval = reinterpret_cast<EvalItem*>(base + off_eval);
  double* d_part = reinterpret_cast<double*>(base + off_part);
  double* d_cheb = reinterpret_cast<double*>(base + off_cheb);
  int nitems = nproj > neval ? nproj : neval;
  k_noalloc_loc_items<<<(unsigned)((nitems + 255) / 256), 256, 0, st>>>(rs, m, n, d_box, d_proj, nproj, d_eval,
                                                                         neval);
  g_launch_counter.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return NUFHT_E_CUDA;
  return run_loc_box(rs, ws, cs, ld_cs, gs, ld_gs, batch, d_box, d_proj, nproj, d_eval, neval, d_part, d_cheb, K,
                     nu_int, sgn, st);
}
