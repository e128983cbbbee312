// Periodic geometry on the device: minimum-image pair vectors and the
// overlap test (src/bdsim/clib/bead.c:27-260).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

// rij[a][b] = minimg(r_b - r_a) for a < b and its negation for a > b
// (bead.c:27-95).  One thread per ordered pair (a < b), grid-stride.
__global__ void pointer_matrix_kernel(const double* __restrict__ pos, int n, double L,
                                      double* __restrict__ rij) {
  long long npairs = (long long)n * (n - 1) / 2;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j;
    pair_from_linear(p, i, j);  // i > j
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = pbg_min_image(pos[3 * i + c] - pos[3 * j + c], L);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      rij[3 * (long long)i + 3 * (long long)j * n + c] = d[c];
      rij[3 * (long long)j + 3 * (long long)i * n + c] = -d[c];
    }
  }
}

// Any non-bonded overlapping pair sets *flag.  conn (N*N int32) may be null.
__global__ void overlap_kernel(const double* __restrict__ pos, const double* __restrict__ radii,
                               int n, double L, double thr, const int* __restrict__ conn,
                               int* __restrict__ flag) {
  long long npairs = (long long)n * (n - 1) / 2;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j;
    pair_from_linear(p, i, j);
    if (conn && conn[j + (long long)n * i]) continue;
    if (pair_overlaps(pos, radii, i, j, L, thr)) {
      atomicOr(flag, 1);
      return;
    }
  }
}

int launch_pointer_matrix(const double* pos, int n, double L, double* rij, cudaStream_t st) {
  if (n < 2) return PBG_OK;
  long long npairs = (long long)n * (n - 1) / 2;
  int blocks = (int)std::min<long long>((npairs + 255) / 256, 148LL * 16);
  pointer_matrix_kernel<<<blocks, 256, 0, st>>>(pos, n, L, rij);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_overlap(const double* pos, const double* radii, int n, double L, double thr,
                   const int* conn, int* flag, cudaStream_t st) {
  PBG_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
  if (n < 2) return PBG_OK;
  long long npairs = (long long)n * (n - 1) / 2;
  int blocks = (int)std::min<long long>((npairs + 255) / 256, 148LL * 8);
  overlap_kernel<<<blocks, 256, 0, st>>>(pos, radii, n, L, thr, conn, flag);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
