// Transposes between the executor's column-major batches (column t of a matrix at p + t * ld)
// and row-major ones (row j at p + j * ld: a C-order (rows, batch) array), on the GPU, so
// that callers holding C-order arrays need no host-side copy.
#include "executor.h"
#include "kernels_common.cuh"

namespace hankel {
namespace {

constexpr int kTile = 32;

// out[c * ldo + r] = in[r * ldi + c] for r < rows, c < cols, through a padded shared tile:
// both the loads (along c) and the stores (along r) are coalesced.
__global__ void k_transpose(const double* __restrict__ in, int ldi, double* __restrict__ out, int ldo, int rows,
                            int cols) {
  __shared__ double tile[kTile][kTile + 1];
  const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  for (int y = threadIdx.y; y < kTile; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[y][threadIdx.x] = in[(size_t)r * ldi + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < kTile; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * ldo + r] = tile[threadIdx.x][y];
  }
}

}  // namespace

int transpose_f64(const double* in, int ldi, double* out, int ldo, int rows, int cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return 0;
  const long long gy = (cols + kTile - 1) / kTile;
  if (gy > 65535) return NUFHT_E_TOO_LARGE;
  dim3 grid((unsigned)((rows + kTile - 1) / kTile), (unsigned)gy);
  k_transpose<<<grid, dim3(kTile, 8), 0, st>>>(in, ldi, out, ldo, rows, cols);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

}  // namespace hankel
