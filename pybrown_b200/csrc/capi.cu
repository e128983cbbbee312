// extern "C" entry points of libpybrown_b200.so (declared in include/pybrown_b200.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>

#include "common.cuh"
#include "kernels.cuh"
#include "propagate.cuh"
#include "system.cuh"

namespace {

thread_local std::string g_last_error;

cudaStream_t legacy_stream() {
  // One private stream for the reference-ABI calls (they are synchronous).
  static std::once_flag once;
  static cudaStream_t st = nullptr;
  std::call_once(once, [] { cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking); });
  return st;
}

// The stream-ordered pool of this process keeps freed memory instead of
// returning it to the driver at every synchronisation (which made each
// scratch allocation a fresh mapping); set once per device.
void keep_pool_memory() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  cudaGetLastError();
  done[dev] = true;
}

// Device scratch for the reference-ABI calls, stream-ordered.
struct DevBuf {
  void* p = nullptr;
  cudaStream_t st;
  explicit DevBuf(cudaStream_t s) : st(s) {}
  int alloc(size_t bytes) {
    keep_pool_memory();
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, st) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      pbg_set_error_message("cudaMallocAsync of %zu bytes failed", bytes);
      return PBG_ERR_NOMEM;
    }
    return PBG_OK;
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

void report_legacy_failure(const char* fn, int rc) {
  fprintf(stderr, "pybrown_b200: %s failed (%d): %s\n", fn, rc, g_last_error.c_str());
}

#define LEGACY_TRY(fn, expr)              \
  do {                                    \
    int _rc = (expr);                     \
    if (_rc != PBG_OK) {                  \
      report_legacy_failure(fn, _rc);     \
      return;                             \
    }                                     \
  } while (0)

#define LEGACY_TRY_RET(fn, expr, val)     \
  do {                                    \
    int _rc = (expr);                     \
    if (_rc != PBG_OK) {                  \
      report_legacy_failure(fn, _rc);     \
      return (val);                       \
    }                                     \
  } while (0)

int h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  PBG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  return PBG_OK;
}
int d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  PBG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
  return PBG_OK;
}
int sync(cudaStream_t st) {
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  return PBG_OK;
}

// Shared body of RPY_M_matrix / RPY_Smith_M_matrix: packed pair vectors in,
// 3N x 3N out (the reference stores M[I + J*3N]; M is symmetric).
int legacy_rpy(double* as, double* pointers, int N, bool smith, double L, double alpha, int m_max,
               int n_max, double* M) {
  if (N <= 0) return PBG_OK;
  cudaStream_t st = legacy_stream();
  const pbg::EwaldTables* t = nullptr;
  if (smith) {
    int rc = pbg::get_ewald_tables(alpha, m_max, n_max, &t);
    if (rc) return rc;
  }
  const size_t n3 = 3 * (size_t)N, npairs = (size_t)N * (N - 1) / 2;
  DevBuf d_as(st), d_pairs(st), d_pos(st), d_M(st), d_phase(st);
  int rc;
  if ((rc = d_as.alloc(N * sizeof(double))) || (rc = d_pairs.alloc(3 * npairs * sizeof(double))) ||
      (rc = d_pos.alloc(3 * (size_t)N * sizeof(double))) || (rc = d_M.alloc(n3 * n3 * sizeof(double))) ||
      (rc = d_phase.alloc(pbg::phase_scratch_bytes(N, t, PBG_PREC_FP64))))
    return rc;
  if ((rc = h2d(d_as.p, as, N * sizeof(double), st))) return rc;
  if (npairs && (rc = h2d(d_pairs.p, pointers, 3 * npairs * sizeof(double), st))) return rc;
  // The reference fills only the entries it computes (free space leaves the
  // off-diagonal entries of the diagonal blocks untouched): start from M.
  if ((rc = h2d(d_M.p, M, n3 * n3 * sizeof(double), st))) return rc;
  if ((rc = pbg::launch_positions_from_pairs(d_pairs.as<double>(), N, d_pos.as<double>(), st))) return rc;
  pbg::PairSource src{nullptr, npairs ? d_pairs.as<double>() : nullptr, N, L};
  if (!npairs) src.pos = d_pos.as<double>();
  if ((rc = pbg::launch_rpy_tensor(src, d_pos.as<double>(), d_as.as<double>(), smith, t, 1.0, PBG_PREC_FP64,
                                   d_M.p, (int)n3, d_phase.p, st)))
    return rc;
  if ((rc = d2h(M, d_M.p, n3 * n3 * sizeof(double), st))) return rc;
  return sync(st);
}

}  // namespace

void pbg_record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  g_last_error = buf;
}

static std::atomic<long long> g_launches{0};     // kernels run
static std::atomic<long long> g_host_calls{0};   // launch calls made by the host (kernels and graphs)

void pbg_count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  g_host_calls.fetch_add(1, std::memory_order_relaxed);
}
void pbg_count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void pbg_count_host_calls(long long n) { g_host_calls.fetch_add(n, std::memory_order_relaxed); }

void pbg_set_error_message(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

extern "C" {

const char* pbg_last_error(void) { return g_last_error.c_str(); }

int pbg_version(void) { return 10000; }

long long pbg_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

long long pbg_host_launch_count(void) { return g_host_calls.load(std::memory_order_relaxed); }

// ------------------------------------------------------------------ tier 1

void RPY_M_matrix(double* as, double* pointers, int number_of_beads, double* M_matrix) {
  LEGACY_TRY("RPY_M_matrix", legacy_rpy(as, pointers, number_of_beads, false, 1.0, 0, 0, 0, M_matrix));
}

void RPY_Smith_M_matrix(double* as, double* pointers, double box_length, double alpha, int m_max, int n_max,
                        int number_of_beads, double* M_matrix) {
  LEGACY_TRY("RPY_Smith_M_matrix",
             legacy_rpy(as, pointers, number_of_beads, true, box_length, alpha, m_max, n_max, M_matrix));
}

void JO_2B_R_matrix(double ai, double aj, double rx, double ry, double rz, double* R_matrix) {
  cudaStream_t st = legacy_stream();
  DevBuf d(st);
  LEGACY_TRY("JO_2B_R_matrix", d.alloc(18 * sizeof(double)));
  LEGACY_TRY("JO_2B_R_matrix", pbg::launch_jo_pair(ai, aj, rx, ry, rz, d.as<double>(), st));
  LEGACY_TRY("JO_2B_R_matrix", d2h(R_matrix, d.p, 18 * sizeof(double), st));
  LEGACY_TRY("JO_2B_R_matrix", sync(st));
}

void JO_R_lubrication_correction_matrix(double* as, double* pointers, int number_of_beads, double cutoff_distance,
                                        int cichocki_correction, double* correction_matrix) {
  const int N = number_of_beads;
  if (N < 2) return;
  cudaStream_t st = legacy_stream();
  const size_t n3 = 3 * (size_t)N, npairs = (size_t)N * (N - 1) / 2;
  DevBuf d_as(st), d_pairs(st), d_C(st);
  const char* fn = "JO_R_lubrication_correction_matrix";
  LEGACY_TRY(fn, d_as.alloc(N * sizeof(double)));
  LEGACY_TRY(fn, d_pairs.alloc(3 * npairs * sizeof(double)));
  LEGACY_TRY(fn, d_C.alloc(n3 * n3 * sizeof(double)));
  LEGACY_TRY(fn, h2d(d_as.p, as, N * sizeof(double), st));
  LEGACY_TRY(fn, h2d(d_pairs.p, pointers, 3 * npairs * sizeof(double), st));
  LEGACY_TRY(fn, h2d(d_C.p, correction_matrix, n3 * n3 * sizeof(double), st));
  pbg::PairSource src{nullptr, d_pairs.as<double>(), N, 0.0};
  LEGACY_TRY(fn, pbg::launch_lubrication_add(src, d_as.as<double>(), cutoff_distance, cichocki_correction, 1.0,
                                             d_C.as<double>(), (int)n3, st));
  LEGACY_TRY(fn, d2h(correction_matrix, d_C.p, n3 * n3 * sizeof(double), st));
  LEGACY_TRY(fn, sync(st));
}

void pointer_pbc_matrix(double* positions, int number_of_beads, double box_length, double* pointers) {
  const int N = number_of_beads;
  if (N < 1) return;
  cudaStream_t st = legacy_stream();
  DevBuf d_pos(st), d_rij(st);
  const char* fn = "pointer_pbc_matrix";
  const size_t nr = 3 * (size_t)N * N;
  LEGACY_TRY(fn, d_pos.alloc(3 * (size_t)N * sizeof(double)));
  LEGACY_TRY(fn, d_rij.alloc(nr * sizeof(double)));
  LEGACY_TRY(fn, h2d(d_pos.p, positions, 3 * (size_t)N * sizeof(double), st));
  LEGACY_TRY(fn, h2d(d_rij.p, pointers, nr * sizeof(double), st));  // diagonal left as given
  LEGACY_TRY(fn, pbg::launch_pointer_matrix(d_pos.as<double>(), N, box_length, d_rij.as<double>(), st));
  LEGACY_TRY(fn, d2h(pointers, d_rij.p, nr * sizeof(double), st));
  LEGACY_TRY(fn, sync(st));
}

void pointer_immobile_pbc_matrix(double* positions_mobile, double* positions_immobile, int number_of_mobile,
                                 int number_of_immobile, double box_length, double* pointers) {
  // Immobile beads sit outside the hydrodynamic hot path; this export keeps the
  // ABI complete with the reference's semantics (bead.c:99-158).
  for (int j = 0; j < number_of_immobile; j++)
    for (int i = 0; i < number_of_mobile; i++)
      for (int c = 0; c < 3; c++)
        pointers[3 * j + 3 * i * number_of_immobile + c] =
            pbg_min_image(positions_immobile[3 * j + c] - positions_mobile[3 * i + c], box_length);
}

int check_overlaps(double* positions, double* as, int number_of_beads, double box_length, double overlap_treshold,
                   int* connection_matrix) {
  const int N = number_of_beads;
  if (N < 2) return 0;
  cudaStream_t st = legacy_stream();
  DevBuf d_pos(st), d_as(st), d_conn(st), d_flag(st);
  const char* fn = "check_overlaps";
  LEGACY_TRY_RET(fn, d_pos.alloc(3 * (size_t)N * sizeof(double)), 0);
  LEGACY_TRY_RET(fn, d_as.alloc(N * sizeof(double)), 0);
  LEGACY_TRY_RET(fn, d_conn.alloc((size_t)N * N * sizeof(int)), 0);
  LEGACY_TRY_RET(fn, d_flag.alloc(sizeof(int)), 0);
  LEGACY_TRY_RET(fn, h2d(d_pos.p, positions, 3 * (size_t)N * sizeof(double), st), 0);
  LEGACY_TRY_RET(fn, h2d(d_as.p, as, N * sizeof(double), st), 0);
  LEGACY_TRY_RET(fn, h2d(d_conn.p, connection_matrix, (size_t)N * N * sizeof(int), st), 0);
  LEGACY_TRY_RET(fn, pbg::launch_overlap(d_pos.as<double>(), d_as.as<double>(), N, box_length, overlap_treshold,
                                         d_conn.as<int>(), d_flag.as<int>(), st), 0);
  int flag = 0;
  LEGACY_TRY_RET(fn, d2h(&flag, d_flag.p, sizeof(int), st), 0);
  LEGACY_TRY_RET(fn, sync(st), 0);
  return flag ? 1 : 0;
}

// ------------------------------------------------------------------ tier 2: stateless

int pbg_dev_pointer_matrix(const double* pos, int n_beads, double box_length, double* rij, void* stream) {
  return pbg::launch_pointer_matrix(pos, n_beads, box_length, rij, (cudaStream_t)stream);
}

int pbg_dev_rpy_matrix(const double* pos, const double* radii, int n_beads, double box_length, double scale,
                       double* M, int ld, void* stream) {
  if (n_beads < 0 || ld < 3 * n_beads) return PBG_ERR_ARG;
  pbg::PairSource src{pos, nullptr, n_beads, box_length};
  return pbg::launch_rpy_tensor(src, pos, radii, false, nullptr, scale, PBG_PREC_FP64, M, ld, nullptr,
                                (cudaStream_t)stream);
}

int pbg_dev_smith_matrix(const double* pos, const double* radii, int n_beads, double box_length, double alpha,
                         int m_max, int n_max, double scale, int precision, void* M, int ld, void* stream) {
  if (n_beads < 0 || ld < 3 * n_beads || (precision != PBG_PREC_FP64 && precision != PBG_PREC_MIXED))
    return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const pbg::EwaldTables* t = nullptr;
  int rc = pbg::get_ewald_tables(alpha, m_max, n_max, &t);
  if (rc) return rc;
  DevBuf phase(st);
  if ((rc = phase.alloc(pbg::phase_scratch_bytes(n_beads, t, precision)))) return rc;
  pbg::PairSource src{pos, nullptr, n_beads, box_length};
  return pbg::launch_rpy_tensor(src, pos, radii, true, t, scale, precision, M, ld, phase.p, st);
}

int pbg_dev_lubrication_add(const double* pos, const double* radii, int n_beads, double box_length, double cutoff,
                            int cichocki, double scale, double* M, int ld, void* stream) {
  if (n_beads < 0 || ld < 3 * n_beads) return PBG_ERR_ARG;
  pbg::PairSource src{pos, nullptr, n_beads, box_length};
  return pbg::launch_lubrication_add(src, radii, cutoff, cichocki, scale, M, ld, (cudaStream_t)stream);
}

int pbg_dev_check_overlaps(const double* pos, const double* radii, int n_beads, double box_length, double threshold,
                           const int* conn, int* flag_dev, void* stream) {
  return pbg::launch_overlap(pos, radii, n_beads, box_length, threshold, conn, flag_dev, (cudaStream_t)stream);
}

int pbg_dev_cholesky(void* A, int n, int ld, int precision, int* info_dev, void* stream) {
  if (ld % PBG_TILE || n > ld || n < 0 ||
      (precision != PBG_PREC_FP64 && precision != PBG_PREC_MIXED && precision != PBG_PREC_MIXED_FP64_DIAG))
    return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = pbg::launch_pad_identity(A, n, ld, precision, st);
  if (rc) return rc;
  DevBuf work(st);
  if ((rc = work.alloc(pbg::cholesky_work_bytes(ld, precision)))) return rc;
  return pbg::launch_cholesky_ws(A, n, ld, precision, info_dev, work.p, st);
}

int pbg_dev_spd_inverse(double* A, int n, int ld, int* info_dev, void* stream) {
  if (ld % PBG_TILE || n > ld || n < 0) return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = pbg::launch_pad_identity(A, n, ld, PBG_PREC_FP64, st);
  if (rc) return rc;
  DevBuf work(st);
  if ((rc = work.alloc(pbg::spd_inverse_work_bytes(ld)))) return rc;
  return pbg::launch_spd_inverse(A, n, ld, info_dev, work.p, st);
}

// ------------------------------------------------------------------ tier 2: system

int pbg_create(const pbg_params* params, pbg_system** out) { return pbg::create_system(params, out); }

int pbg_destroy(pbg_system* sys) {
  pbg::destroy_system(sys);
  return PBG_OK;
}

int pbg_set_state(pbg_system* sys, const double* pos, const double* radii, const int* conn, void* stream) {
  if (!sys || !pos || !radii) return PBG_ERR_ARG;
  pbg::drop_run_graph(sys);
  return pbg::system_set_state(sys, pos, radii, conn, (cudaStream_t)stream);
}

int pbg_set_divergence(pbg_system* sys, int on) {
  if (!sys) return PBG_ERR_ARG;
  pbg::drop_run_graph(sys);
  return pbg::set_divergence(sys, on != 0);
}

int pbg_set_positions(pbg_system* sys, const double* pos, void* stream) {
  if (!sys || !pos) return PBG_ERR_ARG;
  if (!sys->have_state) {
    pbg_set_error_message("pbg_set_positions before pbg_set_state");
    return PBG_ERR_STATE;
  }
  PBG_CUDA_TRY(cudaMemcpyAsync(sys->pos, pos, sys->N * 3 * sizeof(double), cudaMemcpyDefault, (cudaStream_t)stream));
  return PBG_OK;
}

int pbg_set_immobile(pbg_system* sys, int n_immobile, const double* pos, const double* radii, const int* order,
                     const int* conn_mi, void* stream) {
  if (!sys) return PBG_ERR_ARG;
  pbg::drop_run_graph(sys);
  return pbg::set_immobile(sys, n_immobile, pos, radii, order, conn_mi, (cudaStream_t)stream);
}

int pbg_set_interactions(pbg_system* sys, const pbg_interactions* desc) {
  if (!sys) return PBG_ERR_ARG;
  pbg::drop_run_graph(sys);
  return pbg::set_interactions(sys, desc);
}

int pbg_get_energy(pbg_system* sys, double* energy_host, void* stream) {
  if (!sys || !energy_host) return PBG_ERR_ARG;
  if (!sys->energy) {
    *energy_host = 0.0;
    return PBG_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  PBG_CUDA_TRY(cudaMemcpyAsync(energy_host, sys->energy, sizeof(double), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  return PBG_OK;
}

int pbg_get_force(pbg_system* sys, double* force_host, void* stream) {
  if (!sys || !force_host) return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  PBG_CUDA_TRY(cudaMemcpyAsync(force_host, pbg::step_force(sys), sys->n * sizeof(double), cudaMemcpyDefault, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  return PBG_OK;
}

int pbg_set_force(pbg_system* sys, const double* force, void* stream) {
  if (!sys) return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  bool zero = true;
  if (!force) {
    PBG_CUDA_TRY(cudaMemsetAsync(sys->force, 0, sys->ld * sizeof(double), st));
  } else {
    PBG_CUDA_TRY(cudaMemcpyAsync(sys->force, force, sys->n * sizeof(double), cudaMemcpyDefault, st));
    // a force in host memory is checked here: an all-zero one lets the step
    // skip D F, whose result would be zero bit for bit
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, force) == cudaSuccess &&
        (at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeUnregistered)) {
      for (int i = 0; i < sys->n && zero; ++i) zero = force[i] == 0.0;
    } else {
      cudaGetLastError();
      zero = false;
    }
  }
  sys->force_zero = zero;
  return PBG_OK;
}

int pbg_get_positions(pbg_system* sys, double* pos_out, void* stream) {
  if (!sys || !pos_out) return PBG_ERR_ARG;
  PBG_CUDA_TRY(cudaMemcpyAsync(pos_out, sys->pos, sys->n * sizeof(double), cudaMemcpyDefault, (cudaStream_t)stream));
  return PBG_OK;
}

int pbg_get_matrix(pbg_system* sys, int which, double* out, void* stream) {
  if (!sys || !out) return PBG_ERR_ARG;
  return pbg::system_get_matrix(sys, which, out, (cudaStream_t)stream);
}

int pbg_set_matrix(pbg_system* sys, int which, const double* src, void* stream) {
  if (!sys || !src) return PBG_ERR_ARG;
  return pbg::system_set_matrix(sys, which, src, (cudaStream_t)stream);
}

int pbg_step_begin(pbg_system* sys, double dt, int build_Dff, int build_Dnf, int cholesky, void* stream) {
  if (!sys) return PBG_ERR_ARG;
  return pbg::step_begin(sys, dt, build_Dff, build_Dnf, cholesky, (cudaStream_t)stream);
}

int pbg_step_attempt(pbg_system* sys, const double* xi, int* accepted_host, void* stream) {
  if (!sys || !xi || !accepted_host) return PBG_ERR_ARG;
  return pbg::step_attempt(sys, xi, accepted_host, (cudaStream_t)stream);
}

int pbg_step_end(pbg_system* sys, void* stream) {
  if (!sys) return PBG_ERR_ARG;
  return pbg::step_end(sys, (cudaStream_t)stream);
}

int pbg_step_finish(pbg_system* sys, double* pos_host, void* stream) {
  if (!sys || !pos_host) return PBG_ERR_ARG;
  return pbg::step_end(sys, (cudaStream_t)stream, pos_host);
}

int pbg_run(pbg_system* sys, long long j0, int n_steps, double dt, int diff_freq, int lub_freq, int chol_freq,
            const double* pool, long long pool_len, void* stream) {
  if (!sys) return PBG_ERR_ARG;
  return pbg::run(sys, j0, n_steps, dt, diff_freq, lub_freq, chol_freq, pool, pool_len, (cudaStream_t)stream);
}

int pbg_run_report(pbg_system* sys, pbg_step_report* out, void* stream) {
  (void)stream;
  if (!sys || !out) return PBG_ERR_ARG;
  *out = sys->report;
  return PBG_OK;
}

}  // extern "C"
