// Dense SPD factorisations on sm_100a: lower Cholesky factor (numpy.linalg.cholesky
// at src/bdsim/pyBrown/box.py:554) and SPD inverse (numpy.linalg.inv at
// box.py:514,524,537, done here through the Cholesky factor).
//
// Storage: row-major, leading dimension ld (a multiple of 64), order padded to
// ld with an identity block so every 64 x 64 tile is full.  Right-looking
// tiled algorithm, one kernel per stage of each panel:
//   potrf_diag  -- one CTA factors the diagonal tile in FP64 and forms the
//                  inverse of the factor (for the panel solve);
//   trsm_panel  -- one CTA per tile below it: L_ik = A_ik * inv(L_kk)^T;
//   syrk_update -- one CTA per trailing lower tile: A_ij -= L_ik L_jk^T.
// In the mixed precision path the matrix is FP32 and the diagonal tiles are
// still factored and inverted in FP64.
#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

namespace {

constexpr int NB = PBG_TILE;  // 64
constexpr int THREADS = 256;
constexpr int KC = 32;        // k-chunk staged in shared memory

template <typename T>
__device__ __forceinline__ T* tile_ptr(T* A, int ld, int ti, int tj) {
  return A + (size_t)ti * NB * ld + (size_t)tj * NB;
}

// acc[4][4] += A_tile (64 x K, row-major, lda) * B_tile(64 x K)^T for the
// 4 x 4 block of rows 4*ty.., cols 4*tx.. (ty, tx in 0..15).
template <typename T>
__device__ void tile_gemm_nt(const T* __restrict__ Ag, int lda, const T* __restrict__ Bg, int ldb,
                             int K, T acc[4][4], T* sA, T* sB) {
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  for (int k0 = 0; k0 < K; k0 += KC) {
    // stage as [k][row] so that a thread's 4 rows are contiguous
    for (int t = tid; t < NB * KC; t += THREADS) {
      const int r = t / KC, k = t % KC;
      sA[k * (NB + 4) + r] = Ag[(size_t)r * lda + k0 + k];
      sB[k * (NB + 4) + r] = Bg[(size_t)r * ldb + k0 + k];
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < KC; ++k) {
      T a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = sA[k * (NB + 4) + 4 * ty + u];
        b[u] = sB[k * (NB + 4) + 4 * tx + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
}

// Factor diagonal tile k in FP64; write L_kk (upper part zeroed) and
// inv(L_kk) into invL (64 x 64, row-major).  info: 1 + first bad row.
template <typename T>
__global__ void __launch_bounds__(THREADS) potrf_diag_kernel(T* __restrict__ A, int ld, int k, int n,
                                                            T* __restrict__ invL, int* __restrict__ info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double (*L)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(smem_raw);
  double (*X)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(smem_raw + sizeof(double) * NB * (NB + 1));
  const int tid = threadIdx.x;
  T* Akk = tile_ptr(A, ld, k, k);
  for (int t = tid; t < NB * NB; t += THREADS) {
    const int r = t / NB, c = t % NB;
    L[r][c] = c <= r ? (double)Akk[(size_t)r * ld + c] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < NB; ++j) {
    if (tid == 0) {
      const double d = L[j][j];
      if (!(d > 0.0)) {
        const int row = k * NB + j;
        if (row < n) atomicCAS(info, 0, row + 1);
      }
      L[j][j] = sqrt(d);
    }
    __syncthreads();
    const double d = L[j][j];
    for (int i = j + 1 + tid; i < NB; i += THREADS) L[i][j] /= d;
    __syncthreads();
    // trailing lower update: elements (i, c), j < c <= i
    const int m = NB - 1 - j;
    for (int t = tid; t < m * m; t += THREADS) {
      const int i = j + 1 + t / m, c = j + 1 + t % m;
      if (c <= i) L[i][c] -= L[i][j] * L[c][j];
    }
    __syncthreads();
  }
  // inverse of the lower factor: 4 threads per column, forward substitution
  {
    const int col = tid / 4, part = tid % 4;
    for (int i = 0; i < NB; ++i) {
      double s = 0.0;
      if (i > col)
        for (int kk = col + part; kk < i; kk += 4) s += L[i][kk] * X[kk][col];
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if (part == 0) {
        if (i < col) X[i][col] = 0.0;
        else if (i == col) X[i][col] = 1.0 / L[i][i];
        else X[i][col] = -s / L[i][i];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int t = tid; t < NB * NB; t += THREADS) {
    const int r = t / NB, c = t % NB;
    Akk[(size_t)r * ld + c] = (T)(c <= r ? L[r][c] : 0.0);
    invL[t] = (T)X[r][c];
  }
}

// L_ik = A_ik * inv(L_kk)^T for tile rows i = k+1+blockIdx.x.
template <typename T>
__global__ void __launch_bounds__(THREADS) trsm_panel_kernel(T* __restrict__ A, int ld, int k,
                                                            const T* __restrict__ invL) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + KC * (NB + 4);
  const int i = k + 1 + blockIdx.x;
  T acc[4][4] = {};
  T* Aik = tile_ptr(A, ld, i, k);
  // invL is lower triangular: row r of inv(L_kk)^T ... use B = invL (64 x 64), C = A_ik * invL^T
  tile_gemm_nt<T>(Aik, ld, invL, NB, NB, acc, sA, sB);
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  __syncthreads();
  for (int u = 0; u < 4; ++u)
    for (int v = 0; v < 4; ++v) Aik[(size_t)(4 * ty + u) * ld + 4 * tx + v] = acc[u][v];
}

// A_ij -= L_ik L_jk^T for all k < j <= i.
template <typename T>
__global__ void __launch_bounds__(THREADS) syrk_update_kernel(T* __restrict__ A, int ld, int k) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + KC * (NB + 4);
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) ++I;
  while (I * (I + 1) / 2 > b) --I;
  const int J = b - I * (I + 1) / 2;
  const int i = k + 1 + I, j = k + 1 + J;
  T acc[4][4] = {};
  tile_gemm_nt<T>(tile_ptr(A, ld, i, k), ld, tile_ptr(A, ld, j, k), ld, NB, acc, sA, sB);
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  T* Cij = tile_ptr(A, ld, i, j);
  for (int u = 0; u < 4; ++u)
    for (int v = 0; v < 4; ++v) Cij[(size_t)(4 * ty + u) * ld + 4 * tx + v] -= acc[u][v];
}

template <typename T>
__global__ void pad_identity_kernel(T* A, int n, int ld) {
  const long long total = (long long)ld * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / ld), c = (int)(t % ld);
    if (r >= n || c >= n) A[t] = (T)(r == c ? 1.0 : 0.0);
  }
}

// ---- SPD inverse helpers (FP64) ------------------------------------------

// X_i = inv(L_ii) * (E_i - sum_{k<i} L_ik X_k) for block row i of X = inv(L),
// one CTA per 64-column tile c <= i.  E_i is the identity block row.
__global__ void __launch_bounds__(THREADS) trtri_row_kernel(const double* __restrict__ L, int ld, int i,
                                                           const double* __restrict__ invdiag,
                                                           double* __restrict__ X, int ldx) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sA = reinterpret_cast<double*>(smem);
  double* sB = sA + KC * (NB + 4);
  double* sT = sB + KC * (NB + 4);  // 64 x 65 temp
  const int c = blockIdx.x;         // column tile, c <= i
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  double acc[4][4] = {};
  // acc = sum_{k=c}^{i-1} L_ik X_kc ; X_kc is 64x64 row-major: need B^T form, so
  // accumulate with an explicit transpose-free loop.
  for (int kt = c; kt < i; ++kt) {
    const double* Lik = L + (size_t)i * NB * ld + (size_t)kt * NB;
    const double* Xkc = X + (size_t)kt * NB * ldx + (size_t)c * NB;
    for (int k0 = 0; k0 < NB; k0 += KC) {
      for (int t = tid; t < NB * KC; t += THREADS) {
        const int r = t / KC, kk = t % KC;
        sA[kk * (NB + 4) + r] = Lik[(size_t)r * ld + k0 + kk];       // A[r][k]
      }
      for (int t = tid; t < NB * KC; t += THREADS) {
        const int kk = t / NB, col = t % NB;
        sB[kk * (NB + 4) + col] = Xkc[(size_t)(k0 + kk) * ldx + col];  // B[k][col]
      }
      __syncthreads();
      for (int kk = 0; kk < KC; ++kk) {
        double a[4], b[4];
        for (int u = 0; u < 4; ++u) {
          a[u] = sA[kk * (NB + 4) + 4 * ty + u];
          b[u] = sB[kk * (NB + 4) + 4 * tx + u];
        }
        for (int u = 0; u < 4; ++u)
          for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
      }
      __syncthreads();
    }
  }
  // T = E_ic - acc
  for (int u = 0; u < 4; ++u)
    for (int v = 0; v < 4; ++v) {
      const int r = 4 * ty + u, col = 4 * tx + v;
      sT[r * (NB + 1) + col] = (i == c && r == col ? 1.0 : 0.0) - acc[u][v];
    }
  __syncthreads();
  // X_ic = invdiag_i * T
  const double* D = invdiag + (size_t)i * NB * NB;
  for (int u = 0; u < 4; ++u)
    for (int v = 0; v < 4; ++v) {
      const int r = 4 * ty + u, col = 4 * tx + v;
      double s = 0.0;
      for (int kk = 0; kk <= r; ++kk) s += D[r * NB + kk] * sT[kk * (NB + 1) + col];
      X[(size_t)(i * NB + r) * ldx + c * NB + col] = s;
    }
}

// inv(A) = X^T X with X = inv(L) lower: (X^T X)_ij = sum_{k >= max(i,j)} X_ki X_kj.
// One CTA per lower output tile (I >= J); writes both (I,J) and (J,I).
__global__ void __launch_bounds__(THREADS) lauum_kernel(const double* __restrict__ X, int ldx, int nt,
                                                       double* __restrict__ A, int ld) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sA = reinterpret_cast<double*>(smem);
  double* sB = sA + KC * (NB + 4);
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) ++I;
  while (I * (I + 1) / 2 > b) --I;
  const int J = b - I * (I + 1) / 2;
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  double acc[4][4] = {};
  for (int kt = I; kt < nt; ++kt) {
    const double* XkI = X + (size_t)kt * NB * ldx + (size_t)I * NB;
    const double* XkJ = X + (size_t)kt * NB * ldx + (size_t)J * NB;
    for (int k0 = 0; k0 < NB; k0 += KC) {
      for (int t = tid; t < NB * KC; t += THREADS) {
        const int kk = t / NB, col = t % NB;
        sA[kk * (NB + 4) + col] = XkI[(size_t)(k0 + kk) * ldx + col];
        sB[kk * (NB + 4) + col] = XkJ[(size_t)(k0 + kk) * ldx + col];
      }
      __syncthreads();
      for (int kk = 0; kk < KC; ++kk) {
        double a[4], bb[4];
        for (int u = 0; u < 4; ++u) {
          a[u] = sA[kk * (NB + 4) + 4 * ty + u];
          bb[u] = sB[kk * (NB + 4) + 4 * tx + u];
        }
        for (int u = 0; u < 4; ++u)
          for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * bb[v];
      }
      __syncthreads();
    }
  }
  for (int u = 0; u < 4; ++u)
    for (int v = 0; v < 4; ++v) {
      const int r = I * NB + 4 * ty + u, c = J * NB + 4 * tx + v;
      A[(size_t)r * ld + c] = acc[u][v];
      A[(size_t)c * ld + r] = acc[u][v];
    }
}

}  // namespace

int launch_pad_identity(void* A, int n, int ld, int precision, cudaStream_t st) {
  if (n >= ld) return PBG_OK;
  const long long total = (long long)ld * ld;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
  if (precision == PBG_PREC_FP64) pad_identity_kernel<double><<<blocks, 256, 0, st>>>((double*)A, n, ld);
  else pad_identity_kernel<float><<<blocks, 256, 0, st>>>((float*)A, n, ld);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// Workspace: one 64 x 64 tile for inv(L_kk) per diagonal tile (kept so the
// SPD inverse can reuse them).
size_t cholesky_work_bytes(int ld, int precision) {
  const size_t es = precision == PBG_PREC_FP64 ? 8 : 4;
  return (size_t)(ld / NB) * NB * NB * es;
}

constexpr size_t POTRF_SMEM = 2 * sizeof(double) * NB * (NB + 1);

int launch_cholesky_ws(void* A, int n, int ld, int precision, int* info, void* work, cudaStream_t st) {
  if (ld % NB != 0 || n > ld || n < 0) return PBG_ERR_ARG;
  static bool attr_done = false;
  if (!attr_done) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(potrf_diag_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)POTRF_SMEM));
    PBG_CUDA_TRY(cudaFuncSetAttribute(potrf_diag_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)POTRF_SMEM));
    attr_done = true;
  }
  if (precision == PBG_PREC_FP64) {
    const int nt = ld / NB;
    double* W = (double*)work;
    double* Ad = (double*)A;
    const size_t smem = 2 * KC * (NB + 4) * sizeof(double);
    PBG_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
    for (int k = 0; k < nt; ++k) {
      potrf_diag_kernel<double><<<1, THREADS, POTRF_SMEM, st>>>(Ad, ld, k, n, W + (size_t)k * NB * NB, info);
      PBG_CHECK_LAUNCH();
      const int m = nt - k - 1;
      if (m == 0) break;
      trsm_panel_kernel<double><<<m, THREADS, smem, st>>>(Ad, ld, k, W + (size_t)k * NB * NB);
      PBG_CHECK_LAUNCH();
      syrk_update_kernel<double><<<m * (m + 1) / 2, THREADS, smem, st>>>(Ad, ld, k);
      PBG_CHECK_LAUNCH();
    }
    return PBG_OK;
  }
  const int nt = ld / NB;
  float* W = (float*)work;
  float* Af = (float*)A;
  const size_t smem = 2 * KC * (NB + 4) * sizeof(float);
  PBG_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
  for (int k = 0; k < nt; ++k) {
    potrf_diag_kernel<float><<<1, THREADS, POTRF_SMEM, st>>>(Af, ld, k, n, W + (size_t)k * NB * NB, info);
    PBG_CHECK_LAUNCH();
    const int m = nt - k - 1;
    if (m == 0) break;
    trsm_panel_kernel<float><<<m, THREADS, smem, st>>>(Af, ld, k, W + (size_t)k * NB * NB);
    PBG_CHECK_LAUNCH();
    syrk_update_kernel<float><<<m * (m + 1) / 2, THREADS, smem, st>>>(Af, ld, k);
    PBG_CHECK_LAUNCH();
  }
  return PBG_OK;
}

size_t spd_inverse_work_bytes(int ld) {
  // inv(L_kk) tiles + X = inv(L) (ld x ld)
  return cholesky_work_bytes(ld, PBG_PREC_FP64) + (size_t)ld * ld * sizeof(double);
}

int launch_spd_inverse(double* A, int n, int ld, int* info, void* work, cudaStream_t st) {
  const int nt = ld / NB;
  double* W = (double*)work;
  double* X = W + (size_t)nt * NB * NB;
  int rc = launch_cholesky_ws(A, n, ld, PBG_PREC_FP64, info, W, st);
  if (rc != PBG_OK) return rc;
  const size_t smem_t = (2 * KC * (NB + 4) + NB * (NB + 1)) * sizeof(double);
  PBG_CUDA_TRY(cudaFuncSetAttribute(trtri_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t));
  PBG_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)ld * ld * sizeof(double), st));
  for (int i = 0; i < nt; ++i) {
    trtri_row_kernel<<<i + 1, THREADS, smem_t, st>>>(A, ld, i, W, X, ld);
    PBG_CHECK_LAUNCH();
  }
  const size_t smem = 2 * KC * (NB + 4) * sizeof(double);
  lauum_kernel<<<nt * (nt + 1) / 2, THREADS, smem, st>>>(X, ld, nt, A, ld);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
