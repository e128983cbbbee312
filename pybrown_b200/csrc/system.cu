// Device-resident simulation state and one Box.propagate step
// (src/bdsim/pyBrown/box.py:150-389, 486-556) on sm_100a.
//
// A pbg_system owns, in HBM, every per-system tensor of the reference's Box:
// positions, radii, bond matrix, force, D, B and (lubrication modes) Mff, Rff,
// R, plus the midpoint copies.  The step protocol mirrors the reference's
// control flow one to one; the host supplies the Gaussian vector of each move
// attempt (RandomState order) and learns whether it was accepted.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "propagate.cuh"
#include "system.cuh"

namespace pbg {

namespace {

template <typename T>
__global__ void copy_lower_pad_kernel(const T* __restrict__ src, T* __restrict__ dst, int n, int ld) {
  const long long total = (long long)ld * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / ld), c = (int)(t % ld);
    T v;
    if (r < n && c < n) v = c <= r ? src[t] : (T)0;
    else v = (T)(r == c ? 1 : 0);
    dst[t] = v;
  }
}

__global__ void scale_matrix_kernel(double* __restrict__ A, int n, int ld, double s) {
  const long long total = (long long)n * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % ld);
    if (c < n) A[t] = s * A[t];
  }
}

template <typename T>
__global__ void cast_matrix_kernel(const double* __restrict__ src, T* __restrict__ dst, long long total) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    dst[t] = (T)src[t];
}

template <typename T>
__global__ void export_matrix_kernel(const T* __restrict__ src, int n, int ld, int lower_only,
                                     double* __restrict__ dst) {
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    dst[t] = (lower_only && c > r) ? 0.0 : (double)src[(size_t)r * ld + c];
  }
}

inline int grid_for(long long total) { return (int)std::min<long long>((total + 255) / 256, 148LL * 16); }

// ---- mixed lubricated path -------------------------------------------------
// R = Rff (FP32 -> FP64), every element of the padded matrix.
__global__ void widen_matrix_kernel(const float* __restrict__ src, double* __restrict__ dst, long long total) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    dst[t] = (double)src[t];
}

// F = J R J rounded to FP32, J the reversal of all ld indices (the identity
// padding moves to the leading rows and columns).
__global__ void reverse_narrow_kernel(const double* __restrict__ R, int ld, float* __restrict__ F) {
  const long long total = (long long)ld * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    F[t] = (float)R[total - 1 - t];
}

// res = b - R x in FP64 (one warp per row: 16-byte loads, four in flight per
// lane, fixed shuffle tree; row_dot).
__global__ void residual_kernel(const double* __restrict__ R, int ld, int n, const double* __restrict__ b,
                                const double* __restrict__ x, double* __restrict__ res) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  const double s = row_dot(R + (size_t)row * ld, n, [&](int j, double r) { return r * x[j]; });
  if (lane == 0) res[row] = b[row] - s;
}

// x += y ; out = c (a - b)
__global__ void add_vec_kernel(double* __restrict__ x, const double* __restrict__ y, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += y[i];
}
// out[i] = c in[ld-1-i] (J, the reversal of all ld indices, times c)
__global__ void reverse_scale_kernel(const double* __restrict__ in, int ld, double c, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ld) out[i] = c * in[ld - 1 - i];
}
__global__ void diff_scaled_kernel(const double* __restrict__ a, const double* __restrict__ b, double c, int n,
                                   double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = c * (a[i] - b[i]);
}

}  // namespace

template <typename F>
static int sys_alloc(void** p, size_t bytes, F&&) {
  if (bytes == 0) {
    *p = nullptr;
    return PBG_OK;
  }
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    pbg_set_error_message("cudaMalloc of %zu bytes failed", bytes);
    return PBG_ERR_NOMEM;
  }
  return PBG_OK;
}

#define SYS_ALLOC(ptr, bytes)                                                     \
  do {                                                                            \
    int _rc = sys_alloc((void**)&(ptr), (bytes), 0);                              \
    if (_rc != PBG_OK) {                                                          \
      destroy_system(s);                                                          \
      return _rc;                                                                 \
    }                                                                             \
  } while (0)

void destroy_system(pbg_system* s) {
  if (!s) return;
  free_interactions(s);
  free_immobile(s);
  void* ptrs[] = {s->pos,  s->pos_snap, s->radii, s->conn,  s->force, s->D,     s->B,    s->D0,
                  s->Mff,  s->Rff,      s->R,     s->Mff0,  s->Rff0,  s->R0,    s->FX,   s->U,
                  s->BX,   s->ddet,     s->y,     s->rwork, s->Dy,    s->drift, s->xi,   s->phase,
                  s->chol_work, s->inv_work, s->dflags, s->div, s->sol, s->sol0, s->res, s->corr,
                  s->G,    s->tflags};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (s->hflags) cudaFreeHost(s->hflags);
  if (s->hpos) cudaFreeHost(s->hpos);
  if (s->run_exec) cudaGraphExecDestroy(s->run_exec);
  if (s->d_run) cudaFree(s->d_run);
  if (s->h_run) cudaFreeHost(s->h_run);
  if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
  if (s->cap_stream2) cudaStreamDestroy(s->cap_stream2);
  delete s;
}

int create_system(const pbg_params* prm, pbg_system** out) {
  if (!prm || !out) return PBG_ERR_ARG;
  const pbg_params& p = *prm;
  if (p.n_beads <= 0 || !(p.box_length > 0) || p.hydrodynamics < PBG_HI_NONE ||
      p.hydrodynamics > PBG_HI_RPY_SMITH_LUB || (p.precision != PBG_PREC_FP64 && p.precision != PBG_PREC_MIXED) ||
      (p.propagation_scheme != PBG_SCHEME_ERMAK && p.propagation_scheme != PBG_SCHEME_MIDPOINT) ||
      (p.propagation_scheme == PBG_SCHEME_MIDPOINT && !(p.m_midpoint != 0.0))) {
    pbg_set_error_message("invalid pbg_params");
    return PBG_ERR_ARG;
  }
  pbg_system* s = new pbg_system();
  s->p = p;
  s->N = p.n_beads;
  s->n = 3 * p.n_beads;
  s->ld = pbg_round_up(s->n, PBG_TILE);
  s->lub = p.hydrodynamics == PBG_HI_RPY_LUB || p.hydrodynamics == PBG_HI_RPY_SMITH_LUB;
  s->smith = p.hydrodynamics == PBG_HI_RPY_SMITH || p.hydrodynamics == PBG_HI_RPY_SMITH_LUB;
  // Lubrication modes with precision "mixed": FP32 far-field mobility and its
  // tensor-core inverse, FP64 resistance matrix R, FP32 D and B from the
  // tensor-core inverse of J R J, FP64-refined solves with R.
  s->mlub = s->lub && p.precision == PBG_PREC_MIXED;
  s->prec = p.precision;
  s->es = s->prec == PBG_PREC_FP64 ? sizeof(double) : sizeof(float);
  const size_t ff_es = s->mlub ? sizeof(float) : sizeof(double);
  const size_t N = s->N, ld = s->ld;
  const size_t mat = ld * ld;
  if (s->smith) {
    int rc = get_ewald_tables(p.ewald_alpha, p.ewald_real, p.ewald_imag, &s->tables);
    if (rc != PBG_OK) {
      delete s;
      return rc;
    }
  }
  SYS_ALLOC(s->pos, N * 3 * sizeof(double));
  SYS_ALLOC(s->pos_snap, N * 3 * sizeof(double));
  SYS_ALLOC(s->radii, N * sizeof(double));
  SYS_ALLOC(s->force, ld * sizeof(double));
  SYS_ALLOC(s->D, mat * s->es);
  SYS_ALLOC(s->B, mat * s->es);
  if (p.propagation_scheme == PBG_SCHEME_MIDPOINT) SYS_ALLOC(s->D0, mat * s->es);
  if (s->lub) {
    SYS_ALLOC(s->Mff, mat * ff_es);
    SYS_ALLOC(s->Rff, mat * ff_es);
    SYS_ALLOC(s->R, mat * sizeof(double));
    if (p.propagation_scheme == PBG_SCHEME_MIDPOINT) {
      SYS_ALLOC(s->Mff0, mat * ff_es);
      SYS_ALLOC(s->Rff0, mat * ff_es);
      SYS_ALLOC(s->R0, mat * sizeof(double));
    }
    SYS_ALLOC(s->inv_work, s->mlub ? tc_inverse_work_bytes(s->ld) : spd_inverse_work_bytes(s->ld));
    if (s->mlub && p.propagation_scheme == PBG_SCHEME_MIDPOINT) SYS_ALLOC(s->G, mat * sizeof(float));
  }
  double** vecs[] = {&s->FX, &s->U,  &s->BX,   &s->ddet, &s->y,   &s->rwork, &s->Dy,
                     &s->drift, &s->xi, &s->sol, &s->sol0, &s->res, &s->corr};
  for (double** v : vecs) SYS_ALLOC(*v, ld * sizeof(double));
  if (s->smith) SYS_ALLOC(s->phase, phase_scratch_bytes(s->N, s->tables, s->prec));
  SYS_ALLOC(s->chol_work, cholesky_work_bytes(s->ld, s->prec));
  SYS_ALLOC(s->dflags, 8 * sizeof(int));
  SYS_ALLOC(s->tflags, (ld / PBG_TILE) * sizeof(int));
  if (cudaMallocHost((void**)&s->hflags, 8 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    destroy_system(s);
    return PBG_ERR_NOMEM;
  }
  // Zero every vector once so the padding entries stay zero forever.
  for (double** v : vecs)
    if (cudaMemset(*v, 0, ld * sizeof(double)) != cudaSuccess) {
      destroy_system(s);
      return PBG_ERR_CUDA;
    }
  cudaMemset(s->force, 0, ld * sizeof(double));
  cudaMemset(s->dflags, 0, 8 * sizeof(int));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    destroy_system(s);
    return PBG_ERR_CUDA;
  }
  *out = s;
  return PBG_OK;
}

int system_set_state(pbg_system* s, const double* pos, const double* radii, const int* conn, cudaStream_t st) {
  const size_t N = s->N;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->pos, pos, N * 3 * sizeof(double), cudaMemcpyDefault, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(s->radii, radii, N * sizeof(double), cudaMemcpyDefault, st));
  if (conn) {
    if (!s->conn) {
      if (cudaMalloc((void**)&s->conn, N * N * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return PBG_ERR_NOMEM;
      }
    }
    PBG_CUDA_TRY(cudaMemcpyAsync(s->conn, conn, N * N * sizeof(int), cudaMemcpyDefault, st));
  } else if (s->conn) {
    cudaFree(s->conn);
    s->conn = nullptr;
  }
  s->have_state = true;
  if (s->p.hydrodynamics == PBG_HI_NONE) return build_nohi(s, st);
  return PBG_OK;
}

// nohi (box.py:488-490, 548-550): D = kBT 1e19 / 6 / pi / a / eta on the
// diagonal, B = sqrt(D); kept as diagonal matrices so every other code path
// is shared.
int build_nohi(pbg_system* s, cudaStream_t st) {
  std::vector<double> radii(s->N);
  PBG_CUDA_TRY(cudaMemcpyAsync(radii.data(), s->radii, s->N * sizeof(double), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  const size_t ld = s->ld;
  std::vector<double> D(ld * ld, 0.0), B(ld * ld, 0.0);
  for (size_t k = 0; k < ld; ++k) {
    if (k < (size_t)s->n) {
      const double d = s->p.kBT * 1e19 / 6 / PBG_PI / radii[k / 3] / s->p.viscosity;
      D[k * ld + k] = d;
      B[k * ld + k] = std::sqrt(d);
    } else {
      D[k * ld + k] = B[k * ld + k] = 1.0;
    }
  }
  if (s->prec == PBG_PREC_FP64) {
    PBG_CUDA_TRY(cudaMemcpyAsync(s->D, D.data(), ld * ld * sizeof(double), cudaMemcpyHostToDevice, st));
    PBG_CUDA_TRY(cudaMemcpyAsync(s->B, B.data(), ld * ld * sizeof(double), cudaMemcpyHostToDevice, st));
  } else {
    std::vector<float> Df(D.begin(), D.end()), Bf(B.begin(), B.end());
    PBG_CUDA_TRY(cudaMemcpyAsync(s->D, Df.data(), ld * ld * sizeof(float), cudaMemcpyHostToDevice, st));
    PBG_CUDA_TRY(cudaMemcpyAsync(s->B, Bf.data(), ld * ld * sizeof(float), cudaMemcpyHostToDevice, st));
  }
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  return PBG_OK;
}

static PairSource pair_source(const pbg_system* s) {
  PairSource src;
  src.pos = s->pos;
  src.pairs = nullptr;
  src.n = s->N;
  src.L = s->p.box_length;
  return src;
}

// box.py:486-528.  fill_B: the step factors this D next (decompose), so the
// build also writes D's lower triangle into B.
int compute_Dff(pbg_system* s, cudaStream_t st, bool fill_B) {
  const pbg_params& p = s->p;
  const bool smith = s->smith;
  const PairSource src = pair_source(s);
  int rc;
  if (!s->lub) {
    const double scale = p.kBT * 1e19 / p.viscosity;
    // when this step factors D, the build also writes D's lower triangle into
    // B (the factorisation's input), so decompose needs no copy
    void* lower = fill_B ? s->B : nullptr;
    rc = launch_rpy_tensor(src, s->pos, s->radii, smith, s->tables, scale, s->prec, s->D, s->ld, s->phase, st,
                           lower);
    if (rc) return rc;
    if ((rc = launch_pad_identity(s->D, s->n, s->ld, s->prec, st))) return rc;
    if (lower) {
      if ((rc = launch_pad_identity(s->B, s->n, s->ld, s->prec, st))) return rc;
      s->b_holds_lower_D = true;
    }
    return PBG_OK;
  }
  const double scale = 1e19 / p.viscosity;
  if (s->mlub) {
    // Mff in FP32, Rff = inv(Mff) on the tensor cores (a copy is factored)
    rc = launch_rpy_tensor(src, s->pos, s->radii, smith, s->tables, scale, PBG_PREC_MIXED, s->Mff, s->ld, s->phase,
                           st);
    if (rc) return rc;
    rc = launch_pad_identity(s->Mff, s->n, s->ld, PBG_PREC_MIXED, st);
    if (rc) return rc;
    const TcInverseWork w = tc_inverse_work(s->inv_work, s->ld);
    PBG_CUDA_TRY(cudaMemcpyAsync(w.F, s->Mff, (size_t)s->ld * s->ld * sizeof(float), cudaMemcpyDeviceToDevice, st));
    s->work_holds_R = false;
    if ((rc = tc_factor_invert(s->ld, s->dflags + 2, s->inv_work, st))) return rc;
    return tc_lauum(w.X, s->ld, 1.0f, false, (float*)s->Rff, s->dflags + 2, st);
  }
  rc = launch_rpy_tensor(src, s->pos, s->radii, smith, s->tables, scale, PBG_PREC_FP64, s->Mff, s->ld, s->phase, st);
  if (rc) return rc;
  rc = launch_pad_identity(s->Mff, s->n, s->ld, PBG_PREC_FP64, st);
  if (rc) return rc;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->Rff, s->Mff, (size_t)s->ld * s->ld * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return launch_spd_inverse(s->Rff, s->n, s->ld, s->dflags + 2, s->inv_work, st);
}

// Mixed lubricated path: G = chol(J R J) and X = inv(G) on the tensor cores
// (FP32 chain, 3xTF32 updates on the tensor cores, X formed in the same launch);
// then inv(R) = J X^T X J.
static int factor_reversed_R(pbg_system* s, int* info, cudaStream_t st) {
  const TcInverseWork w = tc_inverse_work(s->inv_work, s->ld);
  const long long total = (long long)s->ld * s->ld;
  reverse_narrow_kernel<<<grid_for(total), 256, 0, st>>>(s->R, s->ld, w.F);
  PBG_CHECK_LAUNCH();
  int rc = tc_factor_invert(s->ld, info, s->inv_work, st);
  s->work_holds_R = rc == PBG_OK;
  return rc;
}

// box.py:533-541: R = C eta / 1e19 + Rff ; D = kBT inv(R).
int compute_Dtot(pbg_system* s, cudaStream_t st) {
  const pbg_params& p = s->p;
  if (s->mlub) {
    const long long total = (long long)s->ld * s->ld;
    widen_matrix_kernel<<<grid_for(total), 256, 0, st>>>((const float*)s->Rff, s->R, total);
    PBG_CHECK_LAUNCH();
    int rc = launch_lubrication_add(pair_source(s), s->radii, p.lubrication_cutoff, p.cichocki_correction,
                                    p.viscosity / 1e19, s->R, s->ld, st);
    if (rc) return rc;
    if ((rc = factor_reversed_R(s, s->dflags + 3, st))) return rc;
    const TcInverseWork w = tc_inverse_work(s->inv_work, s->ld);
    return tc_lauum(w.X, s->ld, (float)p.kBT, true, (float*)s->D, s->dflags + 3, st);
  }
  const size_t bytes = (size_t)s->ld * s->ld * sizeof(double);
  PBG_CUDA_TRY(cudaMemcpyAsync(s->R, s->Rff, bytes, cudaMemcpyDeviceToDevice, st));
  int rc = launch_lubrication_add(pair_source(s), s->radii, p.lubrication_cutoff, p.cichocki_correction,
                                  p.viscosity / 1e19, s->R, s->ld, st);
  if (rc) return rc;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->D, s->R, bytes, cudaMemcpyDeviceToDevice, st));
  rc = launch_spd_inverse((double*)s->D, s->n, s->ld, s->dflags + 3, s->inv_work, st);
  if (rc) return rc;
  scale_matrix_kernel<<<grid_for((long long)s->n * s->ld), 256, 0, st>>>((double*)s->D, s->n, s->ld, p.kBT);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// box.py:546-556: B = chol(D), lower.
int decompose(pbg_system* s, cudaStream_t st) {
  if (s->p.hydrodynamics == PBG_HI_NONE) return PBG_OK;
  if (s->mlub) {
    // chol(kBT inv(R)) = sqrt(kBT) J G^{-T} J: read off X = inv(G), no second factorisation
    int rc;
    if (!s->work_holds_R && (rc = factor_reversed_R(s, s->dflags + 1, st))) return rc;
    const TcInverseWork w = tc_inverse_work(s->inv_work, s->ld);
    if ((rc = tc_reversed_factor(w.X, w.F, s->ld, std::sqrt(s->p.kBT), (float*)s->B, (float*)s->chol_work, st)))
      return rc;
    // keep G for the midpoint's inv(B0^T) xi
    if (s->p.propagation_scheme == PBG_SCHEME_MIDPOINT) {
      PBG_CUDA_TRY(cudaMemcpyAsync(s->G, w.F, (size_t)s->ld * s->ld * sizeof(float), cudaMemcpyDeviceToDevice, st));
      s->g_valid = true;
    }
    return PBG_OK;
  }
  if (!s->b_holds_lower_D) {
    const long long total = (long long)s->ld * s->ld;
    if (s->prec == PBG_PREC_FP64)
      copy_lower_pad_kernel<double><<<grid_for(total), 256, 0, st>>>((const double*)s->D, (double*)s->B, s->n, s->ld);
    else
      copy_lower_pad_kernel<float><<<grid_for(total), 256, 0, st>>>((const float*)s->D, (float*)s->B, s->n, s->ld);
    PBG_CHECK_LAUNCH();
  }
  s->b_holds_lower_D = false;  // the factorisation overwrites it
  return launch_cholesky_ws(s->B, s->n, s->ld, s->prec, s->dflags + 1, s->chol_work, st);
}

static int overlap_check(pbg_system* s, cudaStream_t st, bool* overlap) {
  *overlap = false;
  if (!s->p.check_overlaps) return PBG_OK;
  int rc = launch_overlap(s->pos, s->radii, s->N, s->p.box_length, s->p.overlap_treshold, s->conn, s->dflags, st);
  if (rc) return rc;
  if ((rc = overlap_immobile(s, s->dflags, st))) return rc;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->hflags, s->dflags, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  *overlap = s->hflags[0] != 0;
  return PBG_OK;
}

// Mixed lubricated path: x = R^{-1} b from the FP32 D = kBT inv(R) with one
// step of iterative refinement against the FP64 R:
//   x0 = D b / kBT,  x = x0 + D (b - R x0) / kBT  (residual in FP64).
static int refined_solve(pbg_system* s, const void* D, const double* R, const double* b, double* x,
                         cudaStream_t st) {
  const int n = s->n;
  const double c = 1.0 / s->p.kBT;
  int rc = launch_gemv_scaled(D, s->ld, n, s->prec, b, c, x, st);
  if (rc) return rc;
  residual_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(R, s->ld, n, b, x, s->res);
  PBG_CHECK_LAUNCH();
  if ((rc = launch_gemv_scaled(D, s->ld, n, s->prec, s->res, c, s->corr, st))) return rc;
  add_vec_kernel<<<(n + 255) / 256, 256, 0, st>>>(x, s->corr, n);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// Deterministic step (box.py:353-362): pos += ((dt/kBT) D @ F) * mult.
static int deterministic_step(pbg_system* s, const void* D, double mult, cudaStream_t st) {
  if (s->mlub) {
    // (dt/kBT) D F = dt R^{-1} F, by the refined solve
    int rc = refined_solve(s, D, s->R, step_force(s), s->sol, st);
    if (rc) return rc;
    if ((rc = launch_scale2(s->sol, s->dt, mult, s->n, s->FX, st))) return rc;
    return launch_translate(s->pos, s->FX, s->n, false, st);
  }
  // F = 0: every term of ((dt/kBT) D F) mult is +-0 and pos + (+-0) = pos
  if (!s->ff && s->force_zero) return PBG_OK;
  int rc = launch_gemv_scaled(D, s->ld, s->n, s->prec, step_force(s), s->dt / s->p.kBT, s->FX, st);
  if (rc) return rc;
  rc = launch_scale2(s->FX, 1.0, mult, s->n, s->FX, st);
  if (rc) return rc;
  return launch_translate(s->pos, s->FX, s->n, false, st);
}

// Stochastic step (box.py:366-375) from U = B @ xi: pos += (U sqrt(2 dt)) * mult.
static int stochastic_step(pbg_system* s, double mult, cudaStream_t st) {
  int rc = launch_scale2(s->U, std::sqrt(2 * s->dt), mult, s->n, s->BX, st);
  if (rc) return rc;
  return launch_translate(s->pos, s->BX, s->n, false, st);
}

// ---- divergence of the lubricated D (box.py:560-610) ----------------------
__global__ void neg_rowsum_kernel(const double* __restrict__ D, int n, int ld, double* __restrict__ out) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int c = lane; c < n; c += 32) s += D[(size_t)row * ld + c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = -s;
}

__global__ void add_row_kernel(const double* __restrict__ D, int m, int n, int ld, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] += D[(size_t)m * ld + k];
}

__global__ void add_scalar_kernel(double* p, int idx, double v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) p[idx] = p[idx] + v;
}

__global__ void div_apply_kernel(double* __restrict__ div, int n, double eps, double dt, double* __restrict__ pos) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double d = div[k] / eps;
  div[k] = d;
  pos[k] += d * dt;
}

int set_divergence(pbg_system* s, bool on) {
  if (on && s->mlub) {
    pbg_set_error_message("the divergence term needs precision fp64 in the lubrication modes");
    return PBG_ERR_ARG;
  }
  if (on && !s->div) {
    const size_t mat = (size_t)s->ld * s->ld;
    bool ok = cudaMalloc(&s->div, s->ld * sizeof(double)) == cudaSuccess;
    if (ok && !s->D0) ok = cudaMalloc(&s->D0, mat * s->es) == cudaSuccess;
    if (ok && s->lub && !s->Mff0) ok = cudaMalloc(&s->Mff0, mat * sizeof(double)) == cudaSuccess;
    if (ok && s->lub && !s->Rff0) ok = cudaMalloc(&s->Rff0, mat * sizeof(double)) == cudaSuccess;
    if (ok && s->lub && !s->R0) ok = cudaMalloc(&s->R0, mat * sizeof(double)) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      pbg_set_error_message("out of device memory for the divergence term");
      return PBG_ERR_NOMEM;
    }
  }
  s->divergence = on;
  return PBG_OK;
}

// After the deterministic step of the Ermak scheme in the lubrication modes
// (box.py:211-215): div = (sum over coordinates m of row m of D at the
// position moved by eps in m, minus the row sums of D) / eps, by forward
// differences with eps = 1e-7 (box.py:560-610), then pos += div dt.  The
// matrices of the step are restored afterwards.
static int divergence_step(pbg_system* s, cudaStream_t st) {
  const double eps = 0.0000001;
  const int n = s->n, ld = s->ld;
  const size_t bytes = (size_t)ld * ld * s->es, bytes64 = (size_t)ld * ld * sizeof(double);
  PBG_CUDA_TRY(cudaMemcpyAsync(s->D0, s->D, bytes, cudaMemcpyDeviceToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(s->Mff0, s->Mff, bytes64, cudaMemcpyDeviceToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(s->Rff0, s->Rff, bytes64, cudaMemcpyDeviceToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(s->R0, s->R, bytes64, cudaMemcpyDeviceToDevice, st));
  neg_rowsum_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>((const double*)s->D, n, ld, s->div);
  PBG_CHECK_LAUNCH();
  int rc;
  for (int m = 0; m < n; ++m) {
    add_scalar_kernel<<<1, 32, 0, st>>>(s->pos, m, eps);
    PBG_CHECK_LAUNCH();
    if (s->build_Dff && (rc = compute_Dff(s, st, false))) return rc;
    if (s->build_Dnf && (rc = compute_Dtot(s, st))) return rc;
    add_row_kernel<<<(n + 255) / 256, 256, 0, st>>>((const double*)s->D, m, n, ld, s->div);
    PBG_CHECK_LAUNCH();
    add_scalar_kernel<<<1, 32, 0, st>>>(s->pos, m, -eps);
    PBG_CHECK_LAUNCH();
  }
  std::swap(s->D, s->D0);
  std::swap(s->Mff, s->Mff0);
  std::swap(s->Rff, s->Rff0);
  std::swap(s->R, s->R0);
  div_apply_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->div, n, eps, s->dt, s->pos);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int step_begin(pbg_system* s, double dt, int build_Dff, int build_Dnf, int chol, cudaStream_t st) {
  if (!s->have_state) {
    pbg_set_error_message("pbg_step_begin before pbg_set_state");
    return PBG_ERR_STATE;
  }
  s->dt = dt;
  s->build_Dff = build_Dff;
  s->build_Dnf = build_Dnf;
  s->cholesky = chol;
  s->attempts = 0;
  int rc;
  if (s->p.hydrodynamics != PBG_HI_NONE) {
    if (build_Dff && (rc = compute_Dff(s, st, chol && !s->lub))) return rc;
    if (s->lub && build_Dnf && (rc = compute_Dtot(s, st))) return rc;
    if (chol && (rc = decompose(s, st))) return rc;
  }
  // box.py:186: forces at the step-start positions, after the matrices.
  if ((rc = compute_forces(s, st))) return rc;
  const double mult = s->p.propagation_scheme == PBG_SCHEME_MIDPOINT ? 1.0 / s->p.m_midpoint : 1.0;
  if ((rc = deterministic_step(s, s->D, mult, st))) return rc;
  if (s->divergence && s->lub && s->p.propagation_scheme == PBG_SCHEME_ERMAK && (rc = divergence_step(s, st)))
    return rc;
  s->in_step = true;
  return PBG_OK;
}

// Midpoint rebuild at the predicted positions (box.py:291-304); the
// step-start matrices move to the *0 buffers.  The midpoint Cholesky factor is
// discarded by the reference (box.py:316), so it is not formed.
static int midpoint_rebuild(pbg_system* s, cudaStream_t st) {
  const size_t bytes = (size_t)s->ld * s->ld * s->es;
  const size_t bytes64 = (size_t)s->ld * s->ld * sizeof(double);
  const size_t bytes_ff = s->mlub ? (size_t)s->ld * s->ld * sizeof(float) : bytes64;
  std::swap(s->D, s->D0);
  if (s->lub) {
    std::swap(s->Mff, s->Mff0);
    std::swap(s->Rff, s->Rff0);
    std::swap(s->R, s->R0);
  }
  int rc;
  if (s->p.hydrodynamics == PBG_HI_NONE) {
    PBG_CUDA_TRY(cudaMemcpyAsync(s->D, s->D0, bytes, cudaMemcpyDeviceToDevice, st));
    return PBG_OK;
  }
  if (s->build_Dff) {
    if ((rc = compute_Dff(s, st, false))) return rc;
  } else {
    PBG_CUDA_TRY(cudaMemcpyAsync(s->D, s->D0, bytes, cudaMemcpyDeviceToDevice, st));
    if (s->lub) {
      PBG_CUDA_TRY(cudaMemcpyAsync(s->Mff, s->Mff0, bytes_ff, cudaMemcpyDeviceToDevice, st));
      PBG_CUDA_TRY(cudaMemcpyAsync(s->Rff, s->Rff0, bytes_ff, cudaMemcpyDeviceToDevice, st));
    }
  }
  if (s->lub) {
    if (s->build_Dnf) {
      if ((rc = compute_Dtot(s, st))) return rc;
    } else {
      PBG_CUDA_TRY(cudaMemcpyAsync(s->R, s->R0, bytes64, cudaMemcpyDeviceToDevice, st));
      if (s->build_Dff) {
        // D keeps the step-start value when the lubrication build is skipped.
        PBG_CUDA_TRY(cudaMemcpyAsync(s->D, s->D0, bytes, cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  return PBG_OK;
}

static void midpoint_restore(pbg_system* s) {
  s->work_holds_R = false;  // the workspace holds the midpoint R's factor
  std::swap(s->D, s->D0);
  if (s->lub) {
    std::swap(s->Mff, s->Mff0);
    std::swap(s->Rff, s->Rff0);
    std::swap(s->R, s->R0);
  }
}

// Mixed lubricated path, midpoint scheme: y = inv(B0^T) xi = J G J xi / sqrt(kBT)
// by one triangular product with the FP32 factor G of J R0 J (instead of the
// blocked triangular solve with B0).
static int midpoint_y_from_G(pbg_system* s, cudaStream_t st) {
  const int ld = s->ld, g = (ld + 255) / 256;
  reverse_scale_kernel<<<g, 256, 0, st>>>(s->xi, ld, 1.0, s->res);
  PBG_CHECK_LAUNCH();
  int rc = launch_trmv_lower(s->G, ld, ld, PBG_PREC_MIXED, s->res, s->corr, st);
  if (rc) return rc;
  reverse_scale_kernel<<<g, 256, 0, st>>>(s->corr, ld, 1.0 / std::sqrt(s->p.kBT), s->y);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int step_attempt(pbg_system* s, const double* xi, int* accepted, cudaStream_t st) {
  if (!s->in_step) {
    pbg_set_error_message("pbg_step_attempt outside a step");
    return PBG_ERR_STATE;
  }
  s->attempts++;
  const int n = s->n;
  int rc;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->xi, xi, n * sizeof(double), cudaMemcpyDefault, st));
  if ((rc = launch_trmv_lower(s->B, s->ld, n, s->prec, s->xi, s->U, st))) return rc;
  bool overlap = false;
  if (s->p.propagation_scheme == PBG_SCHEME_ERMAK) {
    // box.py:219-248
    if ((rc = stochastic_step(s, 1.0, st))) return rc;
    if ((rc = overlap_check(s, st, &overlap))) return rc;
    if (overlap) {
      if ((rc = stochastic_step(s, -1.0, st))) return rc;
      *accepted = 0;
    } else {
      *accepted = 1;
    }
    return PBG_OK;
  }
  // Midpoint (box.py:272-347).
  const double m = s->p.m_midpoint;
  if ((rc = stochastic_step(s, 1.0 / m, st))) return rc;
  if ((rc = overlap_check(s, st, &overlap))) return rc;
  if (overlap) {
    if ((rc = stochastic_step(s, -1.0 / m, st))) return rc;
    *accepted = 0;
    return PBG_OK;
  }
  if ((rc = midpoint_rebuild(s, st))) return rc;
  // deterministic drift m dt / (2 kBT) (D' - D0) @ F; in the mixed lubricated
  // path (m dt / 2) (R'^{-1} F - R0^{-1} F) by refined solves
  if (s->mlub) {
    if ((rc = refined_solve(s, s->D, s->R, step_force(s), s->sol, st))) return rc;
    if ((rc = refined_solve(s, s->D0, s->R0, step_force(s), s->sol0, st))) return rc;
    diff_scaled_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->sol, s->sol0, m * s->dt / 2, n, s->ddet);
    PBG_CHECK_LAUNCH();
  } else if ((rc = launch_gemv_diff(s->D, s->D0, s->ld, n, s->prec, step_force(s), m * s->dt / (2 * s->p.kBT),
                                    s->ddet, st))) {
    return rc;
  }
  // stochastic drift m/2 sqrt(2 dt) (D' inv(B0^T) - B0) @ xi = c2 (D' y - B0 xi), B0^T y = xi
  if (s->mlub && s->g_valid) {
    if ((rc = midpoint_y_from_G(s, st))) return rc;
  } else if ((rc = launch_trsv_upper(s->B, s->ld, s->prec, s->chol_work, s->xi, s->rwork, s->y, s->tflags,
                                       s->dflags + 4, st))) {
    return rc;
  }
  if (s->mlub) {
    // B0 xi = D0 y, so the drift is c2 kBT (R'^{-1} y - R0^{-1} y): both terms
    // by refined solves, so that the FP32 rounding of B0 does not enter the
    // difference (c2 = 50 sqrt(2 dt) at m = 100 amplifies any mismatch)
    if ((rc = refined_solve(s, s->D, s->R, s->y, s->sol, st))) return rc;
    if ((rc = refined_solve(s, s->D0, s->R0, s->y, s->sol0, st))) return rc;
    const double c2 = m / 2 * std::sqrt(2 * s->dt);
    diff_scaled_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->sol, s->sol0, c2 * s->p.kBT, n, s->drift);
    PBG_CHECK_LAUNCH();
    add_vec_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->drift, s->ddet, n);
    PBG_CHECK_LAUNCH();
  } else {
    if ((rc = launch_gemv_scaled(s->D, s->ld, n, s->prec, s->y, 1.0, s->Dy, st))) return rc;
    if ((rc = launch_drift_combine(s->Dy, s->U, s->ddet, m / 2 * std::sqrt(2 * s->dt), n, s->drift, st))) return rc;
  }
  midpoint_restore(s);
  if ((rc = deterministic_step(s, s->D, 1.0 - 1.0 / m, st))) return rc;
  if ((rc = stochastic_step(s, 1.0 - 1.0 / m, st))) return rc;
  if ((rc = launch_translate(s->pos, s->drift, n, false, st))) return rc;
  if ((rc = overlap_check(s, st, &overlap))) return rc;
  if (overlap) {
    if ((rc = deterministic_step(s, s->D, -(1.0 - 1.0 / m), st))) return rc;
    if ((rc = stochastic_step(s, -1.0, st))) return rc;
    if ((rc = launch_translate(s->pos, s->drift, n, true, st))) return rc;
    *accepted = 0;
  } else {
    *accepted = 1;
  }
  return PBG_OK;
}

int step_end(pbg_system* s, cudaStream_t st, double* pos_out) {
  if (!s->in_step) {
    pbg_set_error_message("pbg_step_end outside a step");
    return PBG_ERR_STATE;
  }
  s->in_step = false;
  int rc = launch_wrap(s->pos, s->n, s->p.box_length, st);
  if (rc) return rc;
  const size_t pos_bytes = (size_t)s->N * 3 * sizeof(double);
  if (pos_out && !s->hpos && cudaMallocHost((void**)&s->hpos, pos_bytes) != cudaSuccess) {
    cudaGetLastError();
    s->hpos = nullptr;
    pbg_set_error_message("cudaMallocHost of the position staging buffer failed");
    return PBG_ERR_NOMEM;
  }
  if (pos_out) PBG_CUDA_TRY(cudaMemcpyAsync(s->hpos, s->pos, pos_bytes, cudaMemcpyDeviceToHost, st));
  // surface factorisation failures of this step
  PBG_CUDA_TRY(cudaMemcpyAsync(s->hflags, s->dflags, 5 * sizeof(int), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  if (pos_out) std::memcpy(pos_out, s->hpos, pos_bytes);
  if (s->hflags[4] < 0) {
    PBG_CUDA_TRY(cudaMemsetAsync(s->dflags + 4, 0, sizeof(int), st));
    pbg_set_error_message("a device-wide wait in the back substitution gave up");
    return PBG_ERR_BARRIER;
  }
  if (s->hflags[1] < 0 || s->hflags[2] < 0 || s->hflags[3] < 0) {
    pbg_set_error_message("a device-wide wait in the factorisation gave up");
    return PBG_ERR_BARRIER;
  }
  if (s->hflags[1] || s->hflags[2] || s->hflags[3]) {
    pbg_set_error_message("matrix not positive definite (cholesky info %d, inverse info %d/%d)",
                          s->hflags[1], s->hflags[2], s->hflags[3]);
    return PBG_ERR_NOT_SPD;
  }
  return PBG_OK;
}

// ---- device-side steps of pbg_run -----------------------------------------
// With the noise pool in device memory and the Ermak scheme (no lubrication,
// no divergence term), a step runs
// without the host between its attempts: the step start, then rounds of
// {xi = the pool's next n draws, U = B xi, the move, the overlap test, the
// undo of a rejected move, the bookkeeping} until a move is accepted, the
// attempts reach max_move_attempts or the pool runs out, then the wrap.  The
// same kernels run either one by one (the host reads the round's verdict) or,
// from the second step with the same flags, dt and force state, as one CUDA
// graph whose attempt rounds sit under a conditional WHILE node.  Every
// arithmetic step is the host-driven one's, so the trajectories are equal bit
// for bit.

static bool device_accessible(const void* p);

namespace {

struct RunDev {
  const double* pool;
  long long pool_len;
  long long used;  // draws consumed in this pbg_run call
  int attempts;    // of the current step
  int status;      // 0, RUN_NOISE or RUN_ATTEMPTS
  int rounds;      // attempt rounds of the current step
  int more;        // the current step's move was rejected and is tried again
  int flags[4];    // the step's copy of dflags (overlap, factorisation infos)
};
constexpr int RUN_NOISE = 1, RUN_ATTEMPTS = 2;

__global__ void run_step_init_kernel(RunDev* r) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    r->attempts = 0;
    r->rounds = 0;
    r->more = 1;
  }
}

// xi = the pool's next n draws; zeros once the pool has run out (the move is
// then nothing and the round ends the run).
__global__ void run_gather_kernel(const RunDev* __restrict__ r, int n, double* __restrict__ xi) {
  const long long used = r->used;
  const bool ok = used + n <= r->pool_len;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    xi[i] = ok ? r->pool[used + i] : 0.0;
}

// The undo of a rejected move, pos += (U sqrt(2 dt)) * (-1): the arithmetic of
// the host-driven undo (scale2 with mult = -1, then translate), each product
// and sum rounded on its own (no contraction into an FMA).
__global__ void run_undo_kernel(double* __restrict__ pos, const double* __restrict__ U, double s1, int n,
                                const int* __restrict__ overlap) {
  if (!*overlap) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pos[i] = __dadd_rn(pos[i], __dmul_rn(__dmul_rn(U[i], s1), -1.0));
}

// The round's bookkeeping: the draws consumed, the attempt counted, and
// whether another round follows (the WHILE node's condition when captured).
__global__ void run_round_update_kernel(RunDev* r, int n, int max_att, const int* __restrict__ overlap,
                                        cudaGraphConditionalHandle handle, int use_handle) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int more = 0;
  if (r->used + n > r->pool_len) {
    r->status = RUN_NOISE;
  } else {
    r->used += n;
    const int a = ++r->attempts;
    if (*overlap) {
      if (a >= max_att) r->status = RUN_ATTEMPTS;
      else more = 1;
    }
  }
  ++r->rounds;
  r->more = more;
  if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

}  // namespace

// One round of attempts (six kernels and the overlap flag's reset).
static int enqueue_run_round(pbg_system* s, cudaStream_t st, cudaGraphConditionalHandle handle, int use_handle) {
  const int n = s->n;
  RunDev* r = static_cast<RunDev*>(s->d_run);
  run_gather_kernel<<<(n + 255) / 256, 256, 0, st>>>(r, n, s->xi);
  PBG_CHECK_LAUNCH();
  int rc = launch_trmv_lower(s->B, s->ld, n, s->prec, s->xi, s->U, st);
  if (rc) return rc;
  if ((rc = stochastic_step(s, 1.0, st))) return rc;
  if ((rc = launch_overlap(s->pos, s->radii, s->N, s->p.box_length, s->p.overlap_treshold, s->conn, s->dflags,
                           st)))
    return rc;
  if ((rc = overlap_immobile(s, s->dflags, st))) return rc;
  run_undo_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->pos, s->U, std::sqrt(2 * s->dt), n, s->dflags);
  PBG_CHECK_LAUNCH();
  run_round_update_kernel<<<1, 32, 0, st>>>(r, n, std::max(1, s->p.max_move_attempts), s->dflags, handle,
                                             use_handle);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// The start of a step: the step-start snapshot of the positions, the matrices
// and the deterministic move (step_begin), the round state.
static int enqueue_run_start(pbg_system* s, double dt, int bDff, int bDnf, int chol, cudaStream_t st) {
  const size_t pos_bytes = (size_t)s->N * 3 * sizeof(double);
  PBG_CUDA_TRY(cudaMemcpyAsync(s->pos_snap, s->pos, pos_bytes, cudaMemcpyDeviceToDevice, st));
  int rc = step_begin(s, dt, bDff, bDnf, chol, st);
  if (rc) return rc;
  run_step_init_kernel<<<1, 32, 0, st>>>(static_cast<RunDev*>(s->d_run));
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// The end of a step: the wrap and the step's report to pinned host memory.
static int enqueue_run_tail(pbg_system* s, cudaStream_t st) {
  int rc = launch_wrap(s->pos, s->n, s->p.box_length, st);
  if (rc) return rc;
  RunDev* r = static_cast<RunDev*>(s->d_run);
  PBG_CUDA_TRY(cudaMemcpyAsync(r->flags, s->dflags, 4 * sizeof(int), cudaMemcpyDeviceToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(s->h_run, s->d_run, sizeof(RunDev), cudaMemcpyDeviceToHost, st));
  return PBG_OK;
}

void drop_run_graph(pbg_system* s) {
  if (s->run_exec) cudaGraphExecDestroy(s->run_exec);
  s->run_exec = nullptr;
  s->run_key = -1;
}

// Captures start + WHILE{round} + tail into s->run_exec.  A refusal by the
// driver leaves run_refused set (steps then run their kernels one by one).
static int capture_run_step(pbg_system* s, double dt, int bDff, int bDnf, int chol) {
  if (!s->cap_stream) PBG_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
  if (!s->cap_stream2) PBG_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_stream2, cudaStreamNonBlocking));
  const long long l0 = pbg_launch_count();
  auto refuse = [&](cudaGraph_t g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    const long long k = pbg_launch_count() - l0;  // nothing ran
    pbg_count_launches(-k);
    pbg_count_host_calls(-k);
    s->in_step = false;
    s->run_refused = true;
    return PBG_OK;
  };
  if (cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) return refuse(nullptr);
  int rc = enqueue_run_start(s, dt, bDff, bDnf, chol, s->cap_stream);
  const long long fixed0 = pbg_launch_count() - l0;
  bool ok = rc == PBG_OK;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle handle = 0;
  cudaGraphNodeParams cp = {};
  if (ok) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    ok = cudaStreamGetCaptureInfo(s->cap_stream, &cs, nullptr, &g, &deps, &ndeps) == cudaSuccess &&
         cs == cudaStreamCaptureStatusActive &&
         cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNode_t wnode = nullptr;
    if (ok) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&wnode, g, deps, ndeps, &cp) == cudaSuccess &&
           cudaStreamUpdateCaptureDependencies(s->cap_stream, &wnode, 1, cudaStreamSetCaptureDependencies) ==
               cudaSuccess;
    }
    if (ok) {
      ok = cudaStreamBeginCaptureToGraph(s->cap_stream2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed) == cudaSuccess;
      if (ok) {
        const long long r0 = pbg_launch_count();
        rc = enqueue_run_round(s, s->cap_stream2, handle, 1);
        s->run_round_kernels = pbg_launch_count() - r0;
        cudaGraph_t body = nullptr;
        ok = cudaStreamEndCapture(s->cap_stream2, &body) == cudaSuccess && rc == PBG_OK;
      }
    }
  }
  const long long before_tail = pbg_launch_count();
  if (ok) ok = enqueue_run_tail(s, s->cap_stream) == PBG_OK;
  const long long tail = pbg_launch_count() - before_tail;
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(s->cap_stream, &graph);
  if (!ok || end != cudaSuccess || !graph) return refuse(graph);
  const cudaError_t inst = cudaGraphInstantiate(&s->run_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) {
    s->run_exec = nullptr;
    return refuse(nullptr);
  }
  s->run_fixed_kernels = fixed0 + tail;
  const long long k = pbg_launch_count() - l0;  // nothing ran yet
  pbg_count_launches(-k);
  pbg_count_host_calls(-k);
  s->in_step = false;  // the capture went through step_begin without running it
  return PBG_OK;
}

// pbg_run's steps on the device (see above); the pool is device memory.
// Outcomes and rollbacks are those of the host-driven loop below.
static int run_device(pbg_system* s, long long j0, int n_steps, double dt, int diff_freq, int lub_freq,
                      int chol_freq, const double* pool, long long pool_len, cudaStream_t st) {
  const size_t pos_bytes = (size_t)s->N * 3 * sizeof(double);
  if (!s->d_run) {
    if (cudaMalloc(&s->d_run, sizeof(RunDev)) != cudaSuccess) {
      cudaGetLastError();
      s->d_run = nullptr;
      pbg_set_error_message("cudaMalloc of the run state failed");
      return PBG_ERR_NOMEM;
    }
    if (cudaMallocHost(&s->h_run, sizeof(RunDev)) != cudaSuccess) {
      cudaGetLastError();
      s->h_run = nullptr;
      pbg_set_error_message("cudaMallocHost of the run report failed");
      return PBG_ERR_NOMEM;
    }
  }
  RunDev* h = static_cast<RunDev*>(s->h_run);
  *h = RunDev{};
  h->pool = pool;
  h->pool_len = pool_len;
  PBG_CUDA_TRY(cudaMemcpyAsync(s->d_run, h, sizeof(RunDev), cudaMemcpyHostToDevice, st));
  int rc = PBG_OK;
  for (int k = 0; k < n_steps; ++k) {
    const long long j = j0 + k;
    const int bDff = j % diff_freq == 0, bDnf = j % lub_freq == 0, chol = j % chol_freq == 0;
    const long long key = bDff | (bDnf << 1) | (chol << 2) | ((long long)s->force_zero << 3) |
                          ((long long)s->ff << 4) | ((long long)s->M << 5);
    if (key != s->run_key || dt != s->run_key_dt) {
      drop_run_graph(s);
      s->run_key = key;
      s->run_key_dt = dt;
      s->run_key_repeats = 0;
    }
    ++s->run_key_repeats;
    if (!s->run_exec && !s->run_refused && s->run_key_repeats >= 2 && (rc = capture_run_step(s, dt, bDff, bDnf, chol)))
      break;
    if (s->run_exec) {
      PBG_CUDA_TRY(cudaGraphLaunch(s->run_exec, st));
      PBG_CUDA_TRY(cudaStreamSynchronize(st));
      pbg_count_launches(s->run_fixed_kernels + s->run_round_kernels * h->rounds);
      pbg_count_host_calls(1);
    } else {
      if ((rc = enqueue_run_start(s, dt, bDff, bDnf, chol, st))) break;
      do {  // the rounds driven from the host: the same kernels, the verdict read after each
        if ((rc = enqueue_run_round(s, st, 0, 0))) break;
        PBG_CUDA_TRY(cudaMemcpyAsync(h, s->d_run, sizeof(RunDev), cudaMemcpyDeviceToHost, st));
        PBG_CUDA_TRY(cudaStreamSynchronize(st));
      } while (h->more);
      if (rc) break;
      if ((rc = enqueue_run_tail(s, st))) break;
      PBG_CUDA_TRY(cudaStreamSynchronize(st));
    }
    s->in_step = false;
    if (h->status) {
      PBG_CUDA_TRY(cudaMemcpyAsync(s->pos, s->pos_snap, pos_bytes, cudaMemcpyDeviceToDevice, st));
      PBG_CUDA_TRY(cudaStreamSynchronize(st));
      if (h->status == RUN_NOISE) {
        pbg_set_error_message("pbg_run: the noise pool ran out in step %lld", j);
        rc = PBG_ERR_NOISE;
      } else {
        pbg_set_error_message("maximal number of move attempts exceeded in step %lld", j);
        rc = PBG_ERR_ATTEMPTS;
      }
      break;
    }
    // factorisation failures of this step, as step_end reports them
    for (int q = 0; q < 4; ++q) s->hflags[q] = h->flags[q];
    if (h->flags[1] < 0 || h->flags[2] < 0 || h->flags[3] < 0) {
      pbg_set_error_message("a device-wide wait in the factorisation gave up");
      rc = PBG_ERR_BARRIER;
      break;
    }
    if (h->flags[1] || h->flags[2] || h->flags[3]) {
      pbg_set_error_message("matrix not positive definite (cholesky info %d, inverse info %d/%d)", h->flags[1],
                            h->flags[2], h->flags[3]);
      rc = PBG_ERR_NOT_SPD;
      break;
    }
    s->report.steps_done++;
    s->report.draws_consumed = h->used;
    s->report.last_attempts = h->attempts;
    s->report.max_attempts = std::max(s->report.max_attempts, h->attempts);
  }
  s->in_step = false;
  return rc;
}

// Steps j0 .. j0+n_steps-1 of BD.py:177 with the noise taken in order from
// `pool`: the protocol of Box.propagate (box.py:150-250) with the pool in
// place of RandomState.  A step that runs out of noise or of move attempts
// (box.py:248) is rolled back to its start positions and ends the run.
int run(pbg_system* s, long long j0, int n_steps, double dt, int diff_freq, int lub_freq, int chol_freq,
        const double* pool, long long pool_len, cudaStream_t st) {
  s->report = pbg_step_report{};
  if (n_steps < 0 || diff_freq <= 0 || lub_freq <= 0 || chol_freq <= 0 || pool_len < 0 || (!pool && n_steps > 0)) {
    pbg_set_error_message("invalid pbg_run arguments");
    return s->report.status = PBG_ERR_ARG;
  }
  if (s->in_step) {
    pbg_set_error_message("pbg_run inside a step");
    return s->report.status = PBG_ERR_STATE;
  }
  if (n_steps > 0 && s->p.propagation_scheme == PBG_SCHEME_ERMAK && !s->lub && !s->divergence &&
      device_accessible(pool))
    return s->report.status = run_device(s, j0, n_steps, dt, diff_freq, lub_freq, chol_freq, pool, pool_len, st);
  const int n = s->n;
  const size_t pos_bytes = (size_t)s->N * 3 * sizeof(double);
  long long used = 0;
  int rc = PBG_OK;
  for (int k = 0; k < n_steps; ++k) {
    const long long j = j0 + k;
    PBG_CUDA_TRY(cudaMemcpyAsync(s->pos_snap, s->pos, pos_bytes, cudaMemcpyDeviceToDevice, st));
    if ((rc = step_begin(s, dt, j % diff_freq == 0, j % lub_freq == 0, j % chol_freq == 0, st))) break;
    int accepted = 0, attempts = 0;
    while (!accepted) {
      if (used + n > pool_len) {
        pbg_set_error_message("pbg_run: the noise pool ran out in step %lld", j);
        rc = PBG_ERR_NOISE;
        break;
      }
      if ((rc = step_attempt(s, pool + used, &accepted, st))) break;
      used += n;
      ++attempts;
      if (!accepted && attempts >= s->p.max_move_attempts) {
        pbg_set_error_message("maximal number of move attempts exceeded in step %lld", j);
        rc = PBG_ERR_ATTEMPTS;
        break;
      }
    }
    if (rc) {
      s->in_step = false;
      PBG_CUDA_TRY(cudaMemcpyAsync(s->pos, s->pos_snap, pos_bytes, cudaMemcpyDeviceToDevice, st));
      break;
    }
    if ((rc = step_end(s, st))) break;
    s->report.steps_done++;
    s->report.draws_consumed = used;
    s->report.last_attempts = attempts;
    s->report.max_attempts = std::max(s->report.max_attempts, attempts);
  }
  s->report.status = rc;
  return rc;
}

template <typename T>
__global__ void import_matrix_kernel(const double* __restrict__ src, int n, int ld, T* __restrict__ dst) {
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    dst[(size_t)r * ld + c] = (T)src[t];
  }
}

// True if `p` can be dereferenced by a kernel (device or managed memory).
static bool device_accessible(const void* p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Accepts host or device memory: host input is staged through a
// stream-ordered device buffer.
int system_set_matrix(pbg_system* s, int which, const double* in, cudaStream_t st) {
  void* dst = nullptr;
  int prec = PBG_PREC_FP64;
  switch (which) {
    case PBG_MAT_D: dst = s->D; prec = s->prec; break;
    case PBG_MAT_B: dst = s->B; prec = s->prec; break;
    case PBG_MAT_MFF: dst = s->Mff; prec = s->mlub ? PBG_PREC_MIXED : PBG_PREC_FP64; break;
    case PBG_MAT_RFF: dst = s->Rff; prec = s->mlub ? PBG_PREC_MIXED : PBG_PREC_FP64; break;
    case PBG_MAT_R: dst = s->R; break;
    default: return PBG_ERR_ARG;
  }
  if (!dst) return PBG_ERR_ARG;
  const size_t bytes = (size_t)s->n * s->n * sizeof(double);
  const double* src = in;
  void* stage = nullptr;
  if (!device_accessible(in)) {
    PBG_CUDA_TRY(cudaMallocAsync(&stage, bytes, st));
    PBG_CUDA_TRY(cudaMemcpyAsync(stage, in, bytes, cudaMemcpyHostToDevice, st));
    src = (const double*)stage;
  }
  int rc = launch_pad_identity(dst, s->n, s->ld, prec, st);
  if (rc == PBG_OK) {
    const long long total = (long long)s->n * s->n;
    if (prec == PBG_PREC_FP64)
      import_matrix_kernel<double><<<grid_for(total), 256, 0, st>>>(src, s->n, s->ld, (double*)dst);
    else
      import_matrix_kernel<float><<<grid_for(total), 256, 0, st>>>(src, s->n, s->ld, (float*)dst);
    if (cudaGetLastError() != cudaSuccess) rc = PBG_ERR_CUDA;
    else pbg_count_launch();
  }
  if (stage) {
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
    PBG_CUDA_TRY(cudaFreeAsync(stage, st));
  }
  if (which == PBG_MAT_R) s->work_holds_R = false;
  if (which == PBG_MAT_B) s->g_valid = false;  // inv(B0^T) xi then comes from the explicit B
  return rc;
}

int system_get_matrix(pbg_system* s, int which, double* out, cudaStream_t st) {
  const void* src = nullptr;
  int prec = PBG_PREC_FP64, lower = 0;
  switch (which) {
    case PBG_MAT_D: src = s->D; prec = s->prec; break;
    case PBG_MAT_B: src = s->B; prec = s->prec; lower = 1; break;
    case PBG_MAT_MFF: src = s->Mff; prec = s->mlub ? PBG_PREC_MIXED : PBG_PREC_FP64; break;
    case PBG_MAT_RFF: src = s->Rff; prec = s->mlub ? PBG_PREC_MIXED : PBG_PREC_FP64; break;
    case PBG_MAT_R: src = s->R; break;
    default: return PBG_ERR_ARG;
  }
  if (!src) return PBG_ERR_ARG;
  const size_t bytes = (size_t)s->n * s->n * sizeof(double);
  double* dst = out;
  void* stage = nullptr;
  const bool host = !device_accessible(out);
  if (host) {
    PBG_CUDA_TRY(cudaMallocAsync(&stage, bytes, st));
    dst = (double*)stage;
  }
  const long long total = (long long)s->n * s->n;
  if (prec == PBG_PREC_FP64)
    export_matrix_kernel<double><<<grid_for(total), 256, 0, st>>>((const double*)src, s->n, s->ld, lower, dst);
  else
    export_matrix_kernel<float><<<grid_for(total), 256, 0, st>>>((const float*)src, s->n, s->ld, lower, dst);
  PBG_CHECK_LAUNCH();
  if (host) {
    PBG_CUDA_TRY(cudaMemcpyAsync(out, stage, bytes, cudaMemcpyDeviceToHost, st));
    PBG_CUDA_TRY(cudaFreeAsync(stage, st));
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return PBG_OK;
}

}  // namespace pbg
