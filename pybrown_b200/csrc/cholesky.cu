// Dense SPD factorisations on sm_100a: lower Cholesky factor (numpy.linalg.cholesky
// at src/bdsim/pyBrown/box.py:554) and SPD inverse (numpy.linalg.inv at
// box.py:514,524,537, done here through the Cholesky factor).
//
// Storage: row-major, leading dimension ld (a multiple of 64), order padded to
// ld with an identity block so every 64 x 64 tile is full.  The factorisation
// itself is the data-flow kernel of cholesky_df.cu; this file adds the SPD
// inverse inv(A) = inv(L)^T inv(L): triangular inversion level by level
// (recursive doubling on the block structure), then the symmetric product,
// both on the tensor cores (FP64 DMMA tile products, cholesky_df.cu).
#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

namespace {

constexpr int NB = PBG_TILE;  // 64

template <typename T>
__global__ void pad_identity_kernel(T* A, int n, int ld) {
  const long long total = (long long)ld * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / ld), c = (int)(t % ld);
    if (r >= n || c >= n) A[t] = (T)(r == c ? 1.0 : 0.0);
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

// Workspace: the factorisation's (inv(L_kk) tiles, data-flow scratch), then
// X = inv(L) (ld x ld) from the next 256-byte boundary.
static size_t spd_x_offset(int ld) { return (cholesky_work_bytes(ld, PBG_PREC_FP64) + 255) / 256 * 256; }

size_t spd_inverse_work_bytes(int ld) { return spd_x_offset(ld) + (size_t)ld * ld * sizeof(double); }

// inv(A) = X^T X with X = inv(L): one data-flow launch factors A and forms
// X's off-diagonal tiles, then X's diagonal tiles and the symmetric product.
int launch_spd_inverse(double* A, int n, int ld, int* info, void* work, cudaStream_t st) {
  const int nt = ld / NB;
  unsigned char* w = static_cast<unsigned char*>(work);
  double* inv = reinterpret_cast<double*>(w);
  double* X = reinterpret_cast<double*>(w + spd_x_offset(ld));
  int rc = launch_cholesky_df(A, n, ld, PBG_PREC_FP64, info, inv, w + (size_t)nt * NB * NB * sizeof(double), st, X);
  if (rc != PBG_OK) return rc;
  if ((rc = launch_trtri_diag(inv, X, ld, PBG_PREC_FP64, st))) return rc;
  return launch_lauum_tc(X, ld, 1.0, false, A, PBG_PREC_FP64, st);
}

}  // namespace pbg
