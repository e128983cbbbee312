// Position-update kernels (src/bdsim/pyBrown/box.py:202-389, 614-617):
// deterministic step (dt/kBT) D F, stochastic step sqrt(2 dt) B xi, the
// midpoint drift terms, translation and the keep-in-box wrap.
//
// Matrix-vector products are HBM-bound: one warp per row, 16-byte loads with
// four in flight per lane (row_dot), FP64 accumulation, fixed shuffle tree
// (so a result does not depend on scheduling).  B is lower triangular and
// only its lower part is read.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "propagate.cuh"

namespace pbg {

namespace {

// y_i = sum_j fl(c * A_ij) x_j  (box.py:356: dt / kBT * D @ F).
template <typename T>
__global__ void gemv_scaled_kernel(const T* __restrict__ A, int ld, int n, const double* __restrict__ x,
                                   double c, double* __restrict__ y) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  const double s = row_dot(A + (size_t)row * ld, n, [&](int j, double a) { return (c * a) * x[j]; });
  if (lane == 0) y[row] = s;
}

// y_i = sum_j fl(c * (A_ij - A0_ij)) x_j  (box.py:306: m dt/(2 kBT) (D - D0) @ F).
template <typename T>
__global__ void gemv_diff_kernel(const T* __restrict__ A, const T* __restrict__ A0, int ld, int n,
                                 const double* __restrict__ x, double c, double* __restrict__ y) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  const T* a0 = A0 + (size_t)row * ld;
  const double s = row_dot(A + (size_t)row * ld, n,
                           [&](int j, double a) { return (c * (a - (double)a0[j])) * x[j]; });
  if (lane == 0) y[row] = s;
}

// y_i = sum_{j <= i} B_ij x_j  (box.py:371: B @ N with B lower triangular).
template <typename T>
__global__ void trmv_lower_kernel(const T* __restrict__ B, int ld, int n, const double* __restrict__ x,
                                  double* __restrict__ y) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  const double s = row_dot(B + (size_t)row * ld, row + 1, [&](int j, double b) { return b * x[j]; });
  if (lane == 0) y[row] = s;
}

// out = (in * s1) * s2, the evaluation order of box.py:356,371
// (X = M @ v * sqrt(2 dt) * mult).
__global__ void scale2_kernel(const double* __restrict__ in, double s1, double s2, int n,
                              double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (in[i] * s1) * s2;
}

// pos += v (Bead.translate, bead.py:92-101; all beads mobile).
__global__ void translate_kernel(double* __restrict__ pos, const double* __restrict__ v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pos[i] += v[i];
}

// pos -= v, written as pos += (-v) like _stochastic_step(mult=-1).
__global__ void untranslate_kernel(double* __restrict__ pos, const double* __restrict__ v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pos[i] += -v[i];
}

__global__ void wrap_kernel(double* __restrict__ pos, int n3, double L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) pos[i] = pbg_wrap(pos[i], L);
}

// drift = (c2 * (D' y - B0 xi)) + ddet, with y = B0^{-T} xi (box.py:306-312).
__global__ void drift_combine_kernel(const double* __restrict__ Dy, const double* __restrict__ Bxi,
                                     const double* __restrict__ ddet, double c2, int n,
                                     double* __restrict__ drift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) drift[i] = c2 * (Dy[i] - Bxi[i]) + ddet[i];
}

// One step of the blocked back substitution B^T y = rhs (B lower, upper system):
// block row I: y_I = inv(B_II)^T r_I (every CTA recomputes it), then
// r_K -= B_IK^T y_I for K < I, one CTA per K tile.
template <typename T>
__global__ void __launch_bounds__(256) trsv_upper_step_kernel(const T* __restrict__ B, int ld, int I,
                                                              const T* __restrict__ invdiag,
                                                              double* __restrict__ r, double* __restrict__ y) {
  __shared__ double s_y[PBG_TILE];
  __shared__ double s_r[PBG_TILE];
  const int tid = threadIdx.x;
  const int nb = PBG_TILE;
  if (tid < nb) s_r[tid] = r[I * nb + tid];
  __syncthreads();
  // y_I[c] = sum_k invL[k][c] r_I[k]  (inv(B_II)^T r_I)
  const T* D = invdiag + (size_t)I * nb * nb;
  if (tid < nb) {
    double s = 0.0;
    for (int k = tid; k < nb; ++k) s += (double)D[k * nb + tid] * s_r[k];
    s_y[tid] = s;
  }
  __syncthreads();
  if (blockIdx.x == 0 && tid < nb) y[I * nb + tid] = s_y[tid];
  const int K = blockIdx.x;  // tiles K < I
  if (K >= I) return;
  // r_K[c] -= sum_k B[I*nb + k][K*nb + c] y_I[k]
  if (tid < nb) {
    double s = 0.0;
    const T* b = B + (size_t)I * nb * ld + (size_t)K * nb + tid;
    for (int k = 0; k < nb; ++k) s += (double)b[(size_t)k * ld] * s_y[k];
    r[K * nb + tid] -= s;
  }
}

__device__ __forceinline__ int trsv_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void trsv_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr long long TRSV_SPIN_LIMIT = 1LL << 24;

// The whole back substitution B^T y = rhs in one launch: CTA K owns block row
// K of the upper system.  For I = nt-1 down to K+1 (the fixed order of the
// per-step launches) it waits for y_I to be published, then accumulates
// B_IK^T y_I; the tile B_IK for the next I is already in registers while it
// waits.  Thread (c, g) (c = tid % 64, g = tid / 64) sums rows 16g .. 16g+15
// of column c; the four partial sums meet in a fixed order, so the result
// does not depend on scheduling.  Then y_K = inv(B_KK)^T r_K from the
// inverted diagonal tile (staged in shared memory at the start, before any
// wait), stored, and flags[K] released.  All CTAs are co-resident (cooperative
// launch).  A wait that gives up after spin_limit polls sets *err = -1 and
// the CTA still publishes (y_K then NaN), so no other CTA waits on it.
template <typename T>
__global__ void __launch_bounds__(256) trsv_upper_df_kernel(const T* __restrict__ B, int ld, int nt,
                                                            const T* __restrict__ invdiag,
                                                            const double* __restrict__ rhs, double* y,
                                                            int* flags, int* err, long long spin_limit) {
  constexpr int nb = PBG_TILE, G = 4, R = nb / G;
  __shared__ T s_d[nb * nb];
  __shared__ double s_part[G][nb];
  __shared__ double s_r[nb];
  __shared__ int s_ok;
  const int tid = threadIdx.x, c = tid % nb, g = tid / nb;
  const int K = nt - 1 - (int)blockIdx.x;  // the first CTAs scheduled start the chain
  const T* D = invdiag + (size_t)K * nb * nb;
  for (int e = tid; e < nb * nb; e += blockDim.x) s_d[e] = D[e];
  const double r0 = tid < nb ? rhs[(size_t)K * nb + tid] : 0.0;
  if (tid == 0) s_ok = 1;
  // column c of B_IK, rows 16g .. 16g+15
  auto load_tile = [&](int I, T (&v)[R]) {
    const T* b = B + ((size_t)I * nb + g * R) * ld + (size_t)K * nb + c;
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = b[(size_t)j * ld];
  };
  T nxt[R];
  double acc = 0.0;
  if (nt - 1 > K) load_tile(nt - 1, nxt);
  for (int I = nt - 1; I > K; --I) {
    T cur[R];
#pragma unroll
    for (int j = 0; j < R; ++j) cur[j] = nxt[j];
    if (I - 1 > K) load_tile(I - 1, nxt);
    if (tid == 0) {
      long long it = 0;
      while (trsv_ld_acquire(flags + I) == 0)
        if (++it > spin_limit) {
          atomicExch(err, -1);
          s_ok = 0;
          break;
        }
    }
    __syncthreads();
    double yv[R];
#pragma unroll
    for (int j = 0; j < R; ++j) yv[j] = __ldcg(y + (size_t)I * nb + g * R + j);
#pragma unroll
    for (int j = 0; j < R; ++j) acc += (double)cur[j] * yv[j];
  }
  s_part[g][c] = acc;
  __syncthreads();
  if (tid < nb) s_r[tid] = r0 - ((s_part[0][tid] + s_part[1][tid]) + (s_part[2][tid] + s_part[3][tid]));
  __syncthreads();
  // y_K[c] = sum_{k >= c} invL[k][c] r_K[k]
  double q = 0.0;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int k = g * R + j;
    if (k >= c) q += (double)s_d[k * nb + c] * s_r[k];
  }
  s_part[g][c] = q;
  __syncthreads();
  if (tid < nb) {
    const double v = (s_part[0][tid] + s_part[1][tid]) + (s_part[2][tid] + s_part[3][tid]);
    y[(size_t)K * nb + tid] = s_ok ? v : __longlong_as_double(0x7ff8000000000000LL);
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) trsv_st_release(flags + K, 1);
}

inline int rows_grid(int n) { return (n * 32 + 255) / 256; }
inline int vec_grid(int n) { return (n + 255) / 256; }

}  // namespace

int launch_gemv_scaled(const void* A, int ld, int n, int precision, const double* x, double c,
                       double* y, cudaStream_t st) {
  if (precision == PBG_PREC_FP64)
    gemv_scaled_kernel<double><<<rows_grid(n), 256, 0, st>>>((const double*)A, ld, n, x, c, y);
  else
    gemv_scaled_kernel<float><<<rows_grid(n), 256, 0, st>>>((const float*)A, ld, n, x, c, y);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_gemv_diff(const void* A, const void* A0, int ld, int n, int precision, const double* x,
                     double c, double* y, cudaStream_t st) {
  if (precision == PBG_PREC_FP64)
    gemv_diff_kernel<double><<<rows_grid(n), 256, 0, st>>>((const double*)A, (const double*)A0, ld, n, x, c, y);
  else
    gemv_diff_kernel<float><<<rows_grid(n), 256, 0, st>>>((const float*)A, (const float*)A0, ld, n, x, c, y);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_trmv_lower(const void* B, int ld, int n, int precision, const double* x, double* y,
                      cudaStream_t st) {
  if (precision == PBG_PREC_FP64)
    trmv_lower_kernel<double><<<rows_grid(n), 256, 0, st>>>((const double*)B, ld, n, x, y);
  else
    trmv_lower_kernel<float><<<rows_grid(n), 256, 0, st>>>((const float*)B, ld, n, x, y);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_scale2(const double* in, double s1, double s2, int n, double* out, cudaStream_t st) {
  scale2_kernel<<<vec_grid(n), 256, 0, st>>>(in, s1, s2, n, out);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_translate(double* pos, const double* v, int n, bool negate, cudaStream_t st) {
  if (negate) untranslate_kernel<<<vec_grid(n), 256, 0, st>>>(pos, v, n);
  else translate_kernel<<<vec_grid(n), 256, 0, st>>>(pos, v, n);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_wrap(double* pos, int n3, double L, cudaStream_t st) {
  wrap_kernel<<<vec_grid(n3), 256, 0, st>>>(pos, n3, L);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_drift_combine(const double* Dy, const double* Bxi, const double* ddet, double c2, int n,
                         double* drift, cudaStream_t st) {
  drift_combine_kernel<<<vec_grid(n), 256, 0, st>>>(Dy, Bxi, ddet, c2, n, drift);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

namespace {

// CTAs of trsv_upper_df_kernel<T> that fit on the current device at once.
template <typename T>
int trsv_df_capacity() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  if (!cached[dev]) {
    int bps = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, trsv_upper_df_kernel<T>, 256, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 0;
    cached[dev] = std::max(1, bps * sms);
  }
  return cached[dev];
}

template <typename T>
int launch_trsv_df(const T* B, int ld, const T* invdiag, const double* rhs, double* y, int* flags, int* err,
                   cudaStream_t st) {
  const int nt = ld / PBG_TILE;
  PBG_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)nt * sizeof(int), st));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nt);
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PBG_CUDA_TRY(cudaLaunchKernelEx(&cfg, trsv_upper_df_kernel<T>, B, ld, nt, invdiag, rhs, y, flags, err,
                                  TRSV_SPIN_LIMIT));
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace

int launch_trsv_upper(const void* B, int ld, int precision, const void* invdiag, const double* rhs,
                      double* r_work, double* y, int* flags, int* err, cudaStream_t st) {
  const int nt = ld / PBG_TILE;
  if (flags && err) {
    if (precision == PBG_PREC_FP64 && nt <= trsv_df_capacity<double>())
      return launch_trsv_df((const double*)B, ld, (const double*)invdiag, rhs, y, flags, err, st);
    if (precision != PBG_PREC_FP64 && nt <= trsv_df_capacity<float>())
      return launch_trsv_df((const float*)B, ld, (const float*)invdiag, rhs, y, flags, err, st);
  }
  PBG_CUDA_TRY(cudaMemcpyAsync(r_work, rhs, (size_t)ld * sizeof(double), cudaMemcpyDeviceToDevice, st));
  for (int I = nt - 1; I >= 0; --I) {
    const int grid = I > 0 ? I : 1;
    if (precision == PBG_PREC_FP64)
      trsv_upper_step_kernel<double><<<grid, 256, 0, st>>>((const double*)B, ld, I, (const double*)invdiag, r_work, y);
    else
      trsv_upper_step_kernel<float><<<grid, 256, 0, st>>>((const float*)B, ld, I, (const float*)invdiag, r_work, y);
    PBG_CHECK_LAUNCH();
  }
  return PBG_OK;
}

}  // namespace pbg
