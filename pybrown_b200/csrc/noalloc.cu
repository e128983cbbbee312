// Allocation-free variant of the Smith-Ewald RPY tensor build.
//
// pbg_dev_smith_matrix takes its scratch (the per-bead reciprocal-space phase
// tables) from the stream-ordered pool and its lattice tables from a cached
// cudaMalloc.  Some callers cannot allow either: an application whose memory
// manager has already claimed all device memory, or a step loop that must not
// run into the implicit device-wide synchronisation of cudaMalloc/cudaFree
// while other streams are busy.  pbg_dev_smith_matrix_noalloc does the same
// computation with every byte of scratch in one file-scope device array of
// fixed size, so it never allocates.  Every GPU that loads the library holds
// this array until the process exits.
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace pbg {
namespace {

// Capacities of the shared scratch array.
constexpr int NOALLOC_MAX_REAL = 4096;       // real-space images, |m|_1 <= ewald_real
constexpr int NOALLOC_MAX_RECIP = 2048;      // half of the n != 0 vectors, |n|_1 <= ewald_imag
constexpr size_t NOALLOC_PHASE_BYTES = 4u << 20;  // n_beads * n_recip * 16 bytes at most
constexpr size_t NOALLOC_REAL_BYTES = (size_t)NOALLOC_MAX_REAL * 4 * sizeof(double);
constexpr size_t NOALLOC_RECIP_BYTES = (size_t)NOALLOC_MAX_RECIP * 8 * sizeof(double);
constexpr size_t NOALLOC_RECIP_F_BYTES = (size_t)NOALLOC_MAX_RECIP * 8 * sizeof(float);
constexpr size_t NOALLOC_BYTES = NOALLOC_REAL_BYTES + NOALLOC_RECIP_BYTES + NOALLOC_RECIP_F_BYTES + NOALLOC_PHASE_BYTES;

// Layout: [real images][reciprocal table FP64][reciprocal table FP32][phase tables].
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch, looked up once per device (in host
// code the symbol name is only a host-side handle, not a device address).
std::mutex g_addr_mu;
void* g_addr[64] = {};

int scratch_address(void** out) {
  int dev = 0;
  PBG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    pbg_set_error_message("pbg_dev_smith_matrix_noalloc: device ordinal %d out of range", dev);
    return PBG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      pbg_record_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      return PBG_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return PBG_OK;
}

// Lattice tables of (alpha, m_max, n_max) in the layout of the Ewald tile
// kernel: images (mx, my, mz, 0) in the L1-ball loop order of the reference
// (src/bdsim/clib/diff_tensor.c:675-683), half of the n vectors with weights
// (nx, ny, nz, P, R, S, 0, 0) doubled for the -n partner, and the
// a-independent lattice sums of the self block (diff_tensor.c:652-849).
void host_tables(double alpha, int m_max, int n_max, std::vector<double>& real, std::vector<double>& recip,
                 double self_O[6], double self_Q[6]) {
  for (int mx = -m_max; mx <= m_max; ++mx)
    for (int my = -(m_max - std::abs(mx)); my <= m_max - std::abs(mx); ++my)
      for (int mz = -(m_max - std::abs(mx) - std::abs(my)); mz <= m_max - std::abs(mx) - std::abs(my); ++mz) {
        const double v[4] = {(double)mx, (double)my, (double)mz, 0.0};
        real.insert(real.end(), v, v + 4);
      }
  const double kk = PBG_PI * PBG_PI / (alpha * alpha);
  for (int nx = -n_max; nx <= n_max; ++nx)
    for (int ny = -(n_max - std::abs(nx)); ny <= n_max - std::abs(nx); ++ny)
      for (int nz = -(n_max - std::abs(nx) - std::abs(ny)); nz <= n_max - std::abs(nx) - std::abs(ny); ++nz) {
        if (!(nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0))) continue;
        const double nl2 = nx * nx + ny * ny + nz * nz;
        const double e = std::exp(-kk * nl2);
        const double P = 2.0 * (2.0 / PBG_PI) / nl2 * e;
        const double R = P * (1.0 + kk * nl2) / nl2;
        const double S = 2.0 * 4 * PBG_PI * e / nl2;
        const double v[8] = {(double)nx, (double)ny, (double)nz, P, R, S, 0.0, 0.0};
        recip.insert(recip.end(), v, v + 8);
      }
  // self-block lattice sums, a-independent part
  const double sqrt_pi = std::sqrt(PBG_PI), alpha2 = alpha * alpha, alpha3 = alpha * alpha2;
  for (int c = 0; c < 6; ++c) self_O[c] = self_Q[c] = 0.0;
  for (size_t q = 0; q < real.size(); q += 4) {
    const double mx = real[q], my = real[q + 1], mz = real[q + 2];
    if (mx == 0 && my == 0 && mz == 0) continue;
    const double mm[6] = {mx * mx, my * my, mz * mz, mx * my, mx * mz, my * mz};
    const double l2 = mm[0] + mm[1] + mm[2], l = std::sqrt(l2), l3 = l2 * l, l5 = l3 * l2;
    const double ec = std::erfc(alpha * l), e = std::exp(-alpha2 * l2);
    const double o_fn[6] = {(1 + mm[0] / l2) / l, (1 + mm[1] / l2) / l, (1 + mm[2] / l2) / l,
                            mm[3] / l3, mm[4] / l3, mm[5] / l3};
    const double q_fn[6] = {(1 - 3 * mm[0] / l2) / l3, (1 - 3 * mm[1] / l2) / l3, (1 - 3 * mm[2] / l2) / l3,
                            -3 * mm[3] / l5, -3 * mm[4] / l5, -3 * mm[5] / l5};
    const double w_o = 2 * alpha / sqrt_pi * e / l2;
    const double am = alpha * l;
    const double w_q1 = std::erfc(am) + 2 / sqrt_pi * am * e;
    const double w_q2 = 2 / sqrt_pi * 2 * alpha3 * e / l2;
    for (int c = 0; c < 6; ++c) {
      self_O[c] += ec * o_fn[c] + w_o * mm[c];
      self_Q[c] += w_q1 * q_fn[c] - w_q2 * mm[c];
    }
  }
  for (int nx = -n_max; nx <= n_max; ++nx)
    for (int ny = -(n_max - std::abs(nx)); ny <= n_max - std::abs(nx); ++ny)
      for (int nz = -(n_max - std::abs(nx) - std::abs(ny)); nz <= n_max - std::abs(nx) - std::abs(ny); ++nz) {
        if (!nx && !ny && !nz) continue;
        const double nl2 = nx * nx + ny * ny + nz * nz;
        const double mm[6] = {(double)nx * nx, (double)ny * ny, (double)nz * nz,
                              (double)nx * ny, (double)nx * nz, (double)ny * nz};
        const double w = 2.0 / PBG_PI / nl2 * std::exp(-kk * nl2);
        const double t = 1.0 / nl2 + kk;
        for (int c = 0; c < 3; ++c) self_O[c] += w * (1.0 - t * mm[c]);
        for (int c = 3; c < 6; ++c) self_O[c] += w * (-t * mm[c]);
        const double wq = 4 * PBG_PI * std::exp(-kk * nl2) / nl2;
        for (int c = 0; c < 6; ++c) self_Q[c] += wq * mm[c];
      }
}

}  // namespace
}  // namespace pbg

extern "C" int pbg_dev_smith_matrix_noalloc(const double* pos, const double* radii, int n_beads,
                                            double box_length, double alpha, int m_max, int n_max,
                                            double scale, int precision, void* M, int ld, void* stream) {
  using namespace pbg;
  if (n_beads < 0 || ld < 3 * n_beads || (precision != PBG_PREC_FP64 && precision != PBG_PREC_MIXED) ||
      m_max < 0 || n_max < 0 || !(alpha > 0) || !(box_length > 0)) {
    pbg_set_error_message("pbg_dev_smith_matrix_noalloc: invalid arguments");
    return PBG_ERR_ARG;
  }
  if (n_beads == 0) return PBG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<double> real, recip;
  EwaldTables t;
  host_tables(alpha, m_max, n_max, real, recip, t.self_O, t.self_Q);
  t.alpha = alpha;
  t.m_max = m_max;
  t.n_max = n_max;
  t.n_real = (int)(real.size() / 4);
  t.n_recip = (int)(recip.size() / 8);
  const size_t elem = precision == PBG_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t phase_bytes = (size_t)n_beads * t.n_recip * elem;
  if (t.n_real > NOALLOC_MAX_REAL || t.n_recip > NOALLOC_MAX_RECIP || phase_bytes > NOALLOC_PHASE_BYTES) {
    pbg_set_error_message(
        "pbg_dev_smith_matrix_noalloc: size beyond the fixed scratch (%d images of max %d, %d reciprocal "
        "vectors of max %d, %zu phase bytes of max %zu)",
        t.n_real, NOALLOC_MAX_REAL, t.n_recip, NOALLOC_MAX_RECIP, phase_bytes, NOALLOC_PHASE_BYTES);
    return PBG_ERR_ARG;
  }
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char* b = static_cast<unsigned char*>(base);
  t.d_real = reinterpret_cast<double*>(b);
  t.d_recip = reinterpret_cast<double*>(b + NOALLOC_REAL_BYTES);
  t.d_recip_f = reinterpret_cast<float*>(b + NOALLOC_REAL_BYTES + NOALLOC_RECIP_BYTES);
  void* phase = b + NOALLOC_REAL_BYTES + NOALLOC_RECIP_BYTES + NOALLOC_RECIP_F_BYTES;
  std::vector<float> recip_f(recip.begin(), recip.end());
  // Pageable host sources: the copies are staged before the calls return, so
  // the local vectors may go out of scope afterwards.
  PBG_CUDA_TRY(cudaMemcpyAsync(t.d_real, real.data(), real.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  if (!recip.empty()) {
    PBG_CUDA_TRY(cudaMemcpyAsync(t.d_recip, recip.data(), recip.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    PBG_CUDA_TRY(cudaMemcpyAsync(t.d_recip_f, recip_f.data(), recip_f.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  }
  PairSource src{pos, nullptr, n_beads, box_length};
  return launch_rpy_tensor(src, pos, radii, true, &t, scale, precision, M, ld, phase, st);
}
