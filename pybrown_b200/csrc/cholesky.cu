// Dense SPD factorisations on sm_100a: lower Cholesky factor (numpy.linalg.cholesky
// at src/bdsim/pyBrown/box.py:554) and SPD inverse (numpy.linalg.inv at
// box.py:514,524,537, done here through the Cholesky factor).
//
// Storage: row-major, leading dimension ld (a multiple of 64), order padded to
// ld with an identity block so every 64 x 64 tile is full.  The factorisation
// itself is the data-flow kernel of cholesky_df.cu; this file adds the SPD
// inverse inv(A) = inv(L)^T inv(L): block-row triangular inversion (trtri_row)
// then the symmetric product (lauum), both tiled FP64 kernels.
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

// Workspace: [inv(L_kk) tiles, nt x 64 x 64][data-flow scratch].
size_t cholesky_work_bytes(int ld, int precision) {
  const size_t es = precision == PBG_PREC_FP64 ? 8 : 4;
  return (size_t)(ld / NB) * NB * NB * es + df_work_bytes(ld);
}

// Factors A in place with the data-flow kernel and leaves the inverted
// diagonal tiles of the factor at the start of `work` (used by the SPD inverse
// and the triangular solve of the midpoint scheme).
int launch_cholesky_ws(void* A, int n, int ld, int precision, int* info, void* work, cudaStream_t st) {
  if (ld % NB != 0 || n > ld || n < 0) return PBG_ERR_ARG;
  const size_t es = precision == PBG_PREC_FP64 ? 8 : 4;
  unsigned char* inv_tiles = static_cast<unsigned char*>(work);
  unsigned char* df = inv_tiles + (size_t)(ld / NB) * NB * NB * es;
  return launch_cholesky_df(A, n, ld, precision, info, inv_tiles, df, st);
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
