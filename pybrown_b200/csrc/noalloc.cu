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
#include <algorithm>
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

// Host-to-device copy through kernel parameters: the launch itself carries
// the values, so nothing is staged in pageable memory and the host does not
// wait for the stream.  Each launch moves up to TABLE_CHUNK doubles (within
// the 4 KB classic parameter limit); `dst_f`, if set, also receives them
// rounded to float.
constexpr int TABLE_CHUNK = 480;
struct TableChunk {
  double v[TABLE_CHUNK];
  int count;
};

__global__ void fill_table_kernel(TableChunk c, double* dst, float* dst_f) {
  for (int t = threadIdx.x; t < c.count; t += blockDim.x) {
    dst[t] = c.v[t];
    if (dst_f) dst_f[t] = (float)c.v[t];
  }
}

int upload_table(const std::vector<double>& src, double* dst, float* dst_f, cudaStream_t st) {
  TableChunk c;
  for (size_t off = 0; off < src.size(); off += TABLE_CHUNK) {
    c.count = (int)std::min<size_t>(TABLE_CHUNK, src.size() - off);
    std::copy(src.begin() + off, src.begin() + off + c.count, c.v);
    fill_table_kernel<<<1, 128, 0, st>>>(c, dst + off, dst_f ? dst_f + off : nullptr);
    PBG_CHECK_LAUNCH();
  }
  return PBG_OK;
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
  // Sizes are checked from the closed-form lattice counts before any table
  // is built, so an oversized ewald_real / ewald_imag is refused at once.
  // (Beyond 64 the counts exceed both capacities anyway.)
  const long long n_real = m_max > 64 ? (1LL << 40) : lattice_points_l1(m_max);
  const long long n_recip = n_max > 64 ? (1LL << 40) : (lattice_points_l1(n_max) - 1) / 2;
  const size_t elem = precision == PBG_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const long double phase_bytes = (long double)n_beads * (long double)n_recip * (long double)elem;
  if (n_real > NOALLOC_MAX_REAL || n_recip > NOALLOC_MAX_RECIP || phase_bytes > (long double)NOALLOC_PHASE_BYTES) {
    pbg_set_error_message(
        "pbg_dev_smith_matrix_noalloc: size beyond the fixed scratch (%lld images of max %d, %lld reciprocal "
        "vectors of max %d, %.0Lf phase bytes of max %zu)",
        n_real, NOALLOC_MAX_REAL, n_recip, NOALLOC_MAX_RECIP, phase_bytes, NOALLOC_PHASE_BYTES);
    return PBG_ERR_ARG;
  }
  if (n_beads == 0) return PBG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  std::vector<double> real, recip;
  EwaldTables t;
  build_lattice_tables(alpha, m_max, n_max, real, recip, t.self_O, t.self_Q);
  t.alpha = alpha;
  t.m_max = m_max;
  t.n_max = n_max;
  t.n_real = (int)(real.size() / 4);
  t.n_recip = (int)(recip.size() / 8);
  unsigned char* b = static_cast<unsigned char*>(base);
  t.d_real = reinterpret_cast<double*>(b);
  t.d_recip = reinterpret_cast<double*>(b + NOALLOC_REAL_BYTES);
  t.d_recip_f = reinterpret_cast<float*>(b + NOALLOC_REAL_BYTES + NOALLOC_RECIP_BYTES);
  void* phase = b + NOALLOC_REAL_BYTES + NOALLOC_RECIP_BYTES + NOALLOC_RECIP_F_BYTES;
  // The tables are rewritten by every call (stream-ordered before the kernels
  // that read them); the phase tables are fully written by the phase kernel.
  rc = upload_table(real, t.d_real, nullptr, st);
  if (rc) return rc;
  rc = upload_table(recip, t.d_recip, t.d_recip_f, st);
  if (rc) return rc;
  PairSource src{pos, nullptr, n_beads, box_length};
  return launch_rpy_tensor(src, pos, radii, true, &t, scale, precision, M, ld, phase, st);
}
