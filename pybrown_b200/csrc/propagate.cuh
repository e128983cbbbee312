// Launchers of the position-update kernels (propagate.cu).
#pragma once

#include "common.cuh"

namespace pbg {

// Row-vector dot products of the matrix-vector kernels: one warp per row,
// each lane takes 16-byte chunks of the row (4 FP32 or 2 FP64 values; rows
// start on 16-byte boundaries because ld is a multiple of 64) at a stride of
// 32 chunks, four chunks in flight at a time, so that enough bytes are
// outstanding per SM to keep HBM busy.  Columns j >= jend are skipped (the
// vector x is not read there).  Per lane the terms are summed in increasing
// j; the lanes' sums are combined by a fixed shuffle tree: the result does
// not depend on scheduling.  term(j, a_j) is the product the caller wants.
template <typename T> struct Chunk;
template <> struct Chunk<float> {
  static constexpr int W = 4;
  using V = float4;
  static __device__ __forceinline__ void get(const V& v, double out[4]) {
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
  }
};
template <> struct Chunk<double> {
  static constexpr int W = 2;
  using V = double2;
  static __device__ __forceinline__ void get(const V& v, double out[2]) {
    out[0] = v.x; out[1] = v.y;
  }
};

template <typename T, typename F>
__device__ __forceinline__ double row_dot(const T* __restrict__ a, int jend, F term) {
  using C = Chunk<T>;
  constexpr int W = C::W, U = 4;
  const int lane = threadIdx.x & 31;
  const int nchunks = (jend + W - 1) / W;
  const typename C::V* av = reinterpret_cast<const typename C::V*>(a);
  double s = 0.0;
  for (int c0 = lane; c0 < nchunks; c0 += 32 * U) {
    typename C::V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (c0 + 32 * u < nchunks) v[u] = __ldg(av + c0 + 32 * u);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = c0 + 32 * u;
      if (c < nchunks) {
        double e[W];
        C::get(v[u], e);
#pragma unroll
        for (int q = 0; q < W; ++q)
          if (c * W + q < jend) s += term(c * W + q, e[q]);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

int launch_gemv_scaled(const void* A, int ld, int n, int precision, const double* x, double c,
                       double* y, cudaStream_t st);
int launch_gemv_diff(const void* A, const void* A0, int ld, int n, int precision, const double* x,
                     double c, double* y, cudaStream_t st);
int launch_trmv_lower(const void* B, int ld, int n, int precision, const double* x, double* y,
                      cudaStream_t st);
int launch_scale2(const double* in, double s1, double s2, int n, double* out, cudaStream_t st);
int launch_translate(double* pos, const double* v, int n, bool negate, cudaStream_t st);
int launch_wrap(double* pos, int n3, double L, cudaStream_t st);
int launch_drift_combine(const double* Dy, const double* Bxi, const double* ddet, double c2, int n,
                         double* drift, cudaStream_t st);
// Solves B^T y = rhs (B lower, order ld, padded); invdiag are the inverted
// diagonal tiles left by the Cholesky workspace; rhs, r_work, y have ld entries.
// With flags (ld / 64 ints of scratch) and err, one cooperative data-flow
// launch when its ld / 64 CTAs fit on the device (a wait that gives up sets
// *err = -1); otherwise, or with null flags, one launch per block row.
int launch_trsv_upper(const void* B, int ld, int precision, const void* invdiag, const double* rhs,
                      double* r_work, double* y, int* flags, int* err, cudaStream_t st);

}  // namespace pbg
