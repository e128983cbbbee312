// Batched replicas: many independent BD systems with hydrodynamic
// interactions (rpy / rpy_smith, Ermak-McCammon scheme) advanced together.
//
// Every replica follows Box.propagate (src/bdsim/pyBrown/box.py:150-250) on
// its own positions, radii, box and noise stream, exactly as a single system
// would: D from the RPY (or Smith-Ewald RPY) tensor, B = chol(D), the
// deterministic step (dt/kBT) D F, then attempts of the stochastic step
// sqrt(2 dt) B xi that are undone on a bead overlap and redrawn.
//
// Each replica owns its device buffers (allocated when it is added).  The
// per-replica descriptors and work lists that the kernels read are rebuilt
// only when the membership changes, so replicas can join and leave between
// steps while the others keep their state on the device.  One step is a
// fixed sequence of launches over all replicas: phase tables and Ewald tiles
// (one work list), the padded copy into B, one cooperative data-flow Cholesky
// over every replica's tiles (left-looking on the tcgen05 tensor cores in the
// mixed precision, right-looking DMMA tile tasks in FP64), then the
// per-replica vector kernels (replica = blockIdx.y).  Replicas never interact, and each one's arithmetic does not
// depend on which other replicas share the batch.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "propagate.cuh"
#include "pybrown_b200.h"

namespace pbg {

// The stream-ordered pool keeps freed replica memory for the next replica
// instead of returning it to the driver at every synchronisation.
inline void batch_pool_keep() {
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

struct BatchReplica {
  pbg_params p;
  int N = 0, n = 0, ld = 0, nt = 0;
  double scale = 0;  // kBT 1e19 / eta: D = scale * M (box.py:498)
  double *pos = nullptr, *radii = nullptr, *force = nullptr, *U = nullptr, *xi = nullptr;
  void *D = nullptr, *B = nullptr, *invdiag = nullptr, *phase = nullptr;
  bool has_force = false;
  unsigned long long seed = 0, draws = 0;
  // this replica's Cholesky task list on the device (built once, when added)
  int4* tasks = nullptr;
  std::vector<int> seg_start;
};

// One piece of a merged task list: `count` tasks of replica `replica`.
struct GatherSeg {
  const int4* src;
  long long dst;
  int count, replica;
};

// What the vector kernels need of one replica.
struct BatchDev {
  double* pos;
  const double* radii;
  const double* force;
  double* U;
  double* xi;
  const void* D;
  void* B;
  double L, thr, kBT;
  int N, n, ld, check, has_force, pad;
};

}  // namespace pbg

struct pbg_batch {
  int precision = PBG_PREC_MIXED;
  int hydrodynamics = PBG_HI_RPY_SMITH;
  double alpha = 0;
  int m_max = 0, n_max = 0;
  const pbg::EwaldTables* tables = nullptr;
  std::vector<pbg::BatchReplica*> slots;
  // active replicas (slot ids) in the order of the device arrays
  std::vector<int> active;
  bool dirty = true;
  double dt = 0;
  bool in_step = false;
  // device arrays of the current membership
  pbg::BatchDev* d_reps = nullptr;
  void* d_rpy = nullptr;
  int4* d_ework = nullptr;
  int n_ework = 0;
  pbg::CholRep* d_chol = nullptr;
  int4* d_tasks = nullptr;
  int ntasks = 0;
  pbg::GatherSeg* d_segs = nullptr;
  int4* d_eparts = nullptr;  // per replica: tiles per edge, offset in the Ewald work list
  // capacities (bytes) of the grow-only arrays above
  size_t cap_reps = 0, cap_rpy = 0, cap_ework = 0, cap_chol = 0, cap_tasks = 0, cap_segs = 0, cap_eparts = 0,
         cap_flags = 0;
  int* d_flags = nullptr;  // [4 ctl][per replica: upd nt^2, fin nt^2][R infos]
  size_t flag_ints = 0;
  int* d_info = nullptr;
  int* d_ovl = nullptr;
  unsigned char* d_mask = nullptr;
  unsigned long long* d_stream = nullptr;  // [R][2]: seed, draws of each noise stream
  int* h_ovl = nullptr;  // pinned, read after a stream synchronisation
  int* h_info = nullptr;
  std::vector<unsigned char> mask;  // of the last upload, active order
  size_t cap = 0;  // capacity of the per-replica device/pinned arrays
  int max_n = 0;
  // Schedule of the batched factorisation (pbg_batch_autotune): the order in
  // which the replicas' task segments are merged, and the resident CTAs per
  // SM (0 = as many as fit).  Neither changes any result.
  int merge_order = PBG_MERGE_LARGER_FIRST;
  int ctas_per_sm = 0;
  bool have_D = false;  // a step has built D (the autotuner factors it)
  // CUDA graph of the deterministic part of a step (Ewald build, copy into
  // B, the persistent factorisation, the deterministic move), captured once a
  // step repeats with the same membership and flags, replayed afterwards.
  cudaStream_t cap_stream = nullptr;   // private non-blocking stream for the capture
  cudaGraphExec_t begin_exec = nullptr;
  long long begin_kernels = 0;         // kernel launches inside the graph
  int key_build = -1, key_chol = -1, key_force = -1;
  double key_dt = 0;
  int key_repeats = 0;                 // steps in a row with the current key
  bool graph_refused = false;          // the driver refused the capture: direct launches
  // Whole steps on the device (pbg_batch_step): the start, the rounds of
  // attempts under a conditional WHILE node and the wrap, as one graph.
  cudaStream_t cap_stream2 = nullptr;  // captures the loop body
  cudaGraphExec_t step_exec = nullptr;
  long long step_fixed_kernels = 0;    // kernels of one replay besides the rounds
  int* d_att = nullptr;                // [R] attempts of this step (inside d_flags)
  int* d_words = nullptr;              // [4]: any replica still moving, error bits, rounds, 0
  int* d_maxatt = nullptr;             // [cap] max_move_attempts per replica
  int* h_step = nullptr;               // pinned: infos, attempts, words of the last step
  bool streams_on_device = false;      // d_stream holds every replica's (seed, draws)
  bool host_draws_stale = false;       // ... and the host copies are behind it
};

namespace pbg {

namespace {

// B = lower(D) with the identity beyond n and zeros above the diagonal.
template <typename T>
__global__ void batch_copy_lower_kernel(const BatchDev* __restrict__ reps) {
  const BatchDev& r = reps[blockIdx.y];
  const T* src = static_cast<const T*>(r.D);
  T* dst = static_cast<T*>(r.B);
  const int n = r.n, ld = r.ld;
  const long long total = (long long)ld * ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / ld), col = (int)(t % ld);
    T v;
    if (row < n && col < n) v = col <= row ? src[t] : (T)0;
    else v = (T)(row == col ? 1 : 0);
    dst[t] = v;
  }
}

// The padding rows of B's lower triangle: identity (rows n .. ld-1, columns
// up to the diagonal).  The rest of the lower triangle comes from the Ewald
// build; nothing reads B above the diagonal.
template <typename T>
__global__ void batch_pad_lower_kernel(const BatchDev* __restrict__ reps) {
  const BatchDev& r = reps[blockIdx.y];
  T* dst = static_cast<T*>(r.B);
  const int n = r.n, ld = r.ld;
  const long long total = (long long)(ld - n) * ld;
  for (long long t = threadIdx.x; t < total; t += blockDim.x) {
    const int row = n + (int)(t / ld), col = (int)(t % ld);
    if (col <= row) dst[(size_t)row * ld + col] = (T)(row == col ? 1 : 0);
  }
}

// Deterministic step (box.py:353-362) for replicas with a force:
// pos += ((dt/kBT) D @ F * 1) * 1, one warp per row.
template <typename T>
__global__ void batch_det_kernel(const BatchDev* __restrict__ reps, double dt) {
  const BatchDev& r = reps[blockIdx.y];
  if (!r.has_force) return;
  const T* D = static_cast<const T*>(r.D);
  const double c = dt / r.kBT;
  const double* F = r.force;
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < r.n; row += gridDim.x * warps) {
    const double s = row_dot(D + (size_t)row * r.ld, r.n, [&](int j, double a) { return (c * a) * F[j]; });
    // the displacement waits in U until every row is done (see batch_det_move)
    if (lane == 0) r.U[row] = (s * 1.0) * 1.0;
  }
}

__global__ void batch_det_move_kernel(const BatchDev* __restrict__ reps) {
  const BatchDev& r = reps[blockIdx.y];
  if (!r.has_force) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) r.pos[i] += r.U[i];
}

// U = B xi for the masked replicas (box.py:371; B lower triangular).
template <typename T>
__global__ void batch_trmv_kernel(const BatchDev* __restrict__ reps, const unsigned char* __restrict__ mask) {
  if (!mask[blockIdx.y]) return;
  const BatchDev& r = reps[blockIdx.y];
  const T* B = static_cast<const T*>(r.B);
  const double* xi = r.xi;
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < r.n; row += gridDim.x * warps) {
    const double s = row_dot(B + (size_t)row * r.ld, row + 1, [&](int j, double b) { return b * xi[j]; });
    if (lane == 0) r.U[row] = s;
  }
}

// Stochastic step (box.py:366-375): pos += (U sqrt(2 dt)) * mult, for the
// masked replicas; with `undo`, only those whose overlap flag is set.
__global__ void batch_move_kernel(const BatchDev* __restrict__ reps, const unsigned char* __restrict__ mask,
                                  const int* __restrict__ ovl, double s1, double mult, int undo) {
  if (!mask[blockIdx.y]) return;
  if (undo && !ovl[blockIdx.y]) return;
  const BatchDev& r = reps[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x)
    r.pos[i] += (r.U[i] * s1) * mult;
}

// Overlap test of the masked replicas (bead.c:169-218), no bonded pairs.
__global__ void batch_overlap_kernel(const BatchDev* __restrict__ reps, const unsigned char* __restrict__ mask,
                                     int* __restrict__ ovl) {
  if (!mask[blockIdx.y]) return;
  const BatchDev& r = reps[blockIdx.y];
  if (!r.check) return;
  const long long npairs = (long long)r.N * (r.N - 1) / 2;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    if (ovl[blockIdx.y]) return;
    int i, j;
    pair_from_linear(p, i, j);
    if (pair_overlaps(r.pos, r.radii, i, j, r.L, r.thr)) {
      atomicOr(ovl + blockIdx.y, 1);
      return;
    }
  }
}

__global__ void batch_wrap_kernel(const BatchDev* __restrict__ reps) {
  const BatchDev& r = reps[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x)
    r.pos[i] = pbg_wrap(r.pos[i], r.L);
}

// Counter-based normal variates for a replica's noise stream: Philox-4x32-10
// (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011) keyed by the replica's seed, counter = pair index of the draw,
// and the Box-Muller transform of two 53-bit uniforms.  Draw d of a stream
// depends only on (seed, d), never on the other replicas of the batch.
__device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
  const uint32_t hi0 = __umulhi(m0, c[0]), lo0 = m0 * c[0];
  const uint32_t hi1 = __umulhi(m1, c[2]), lo1 = m1 * c[2];
  const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
  c[0] = n0;
  c[1] = lo1;
  c[2] = n2;
  c[3] = lo0;
}

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
  const unsigned long long v = ((unsigned long long)hi << 32 | lo) >> 11;
  return ((double)v + 0.5) * (1.0 / 9007199254740992.0);  // (0, 1)
}

__global__ void batch_noise_kernel(const BatchDev* __restrict__ reps, const unsigned char* __restrict__ mask,
                                   const unsigned long long* __restrict__ streams) {
  if (!mask[blockIdx.y]) return;
  const BatchDev& r = reps[blockIdx.y];
  const unsigned long long seed = streams[2 * blockIdx.y], base = streams[2 * blockIdx.y + 1] / 2;  // even
  const int pairs = (r.n + 1) / 2;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < pairs; q += gridDim.x * blockDim.x) {
    const unsigned long long ctr = base + (unsigned long long)q;
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = u53(c[0], c[1]), u2 = u53(c[2], c[3]);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    r.xi[2 * q] = rad * cs;
    if (2 * q + 1 < r.n) r.xi[2 * q + 1] = rad * sn;
  }
}

// Start of the attempt rounds of a device step: every replica moves; the
// attempt counts and the step words are cleared.
__global__ void batch_round_init_kernel(int R, unsigned char* __restrict__ mask, int* __restrict__ att,
                                        int* __restrict__ words) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < R; q += gridDim.x * blockDim.x) {
    mask[q] = 1;
    att[q] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x < 4) words[threadIdx.x] = 0;
}

// End of one round of attempts (one block): each moving replica has taken one
// more attempt and consumed 3N draws (rounded up to even) of its stream; it
// stops when its move was accepted (already undone otherwise) or when it has
// used max_move_attempts (error bit ATTEMPTS, as box.py:248 asserts).
// words[0] = whether any replica still moves; inside the step's graph the
// WHILE node's condition is set to it, and a round cap bounds every launch.
constexpr int BATCH_ROUND_CAP = 4096;
__global__ void batch_round_update_kernel(const BatchDev* __restrict__ reps, int R, unsigned char* __restrict__ mask,
                                          const int* __restrict__ ovl, int* __restrict__ att,
                                          const int* __restrict__ maxatt, unsigned long long* __restrict__ streams,
                                          int* __restrict__ words, cudaGraphConditionalHandle handle,
                                          int use_handle) {
  int moving = 0;
  for (int q = threadIdx.x; q < R; q += blockDim.x) {
    if (!mask[q]) continue;
    const int n = reps[q].n;
    const int a = att[q] + 1;
    att[q] = a;
    streams[2 * q + 1] += (unsigned long long)(n + (n & 1));
    if (!ovl[q]) {
      mask[q] = 0;
    } else if (a >= maxatt[q]) {
      mask[q] = 0;
      atomicOr(words + 1, (int)PBG_DEV_ERR_ATTEMPTS);
    } else {
      moving = 1;
    }
  }
  const int any = __syncthreads_or(moving);
  if (threadIdx.x == 0) {
    const int rounds = words[2] + 1;
    words[2] = rounds;
    words[0] = any;
    if (use_handle) cudaGraphSetConditional(handle, (any && rounds % BATCH_ROUND_CAP != 0) ? 1u : 0u);
  }
}

inline size_t elem_size(int precision) { return precision == PBG_PREC_FP64 ? 8 : 4; }

// Replica buffers come from the stream-ordered pool on the legacy default
// stream: allocation and release are ordered after the batch's earlier work
// on that stream (and on every blocking stream) and need no device-wide sync.
void free_replica(BatchReplica* r) {
  if (!r) return;
  void* bufs[] = {r->pos, r->radii, r->force, r->U, r->xi, r->D, r->B, r->invdiag, r->phase, r->tasks};
  for (void* p : bufs)
    if (p) cudaFreeAsync(p, 0);
  delete r;
}

bool pool_alloc(void* p, size_t bytes) {
  return cudaMallocAsync(static_cast<void**>(p), bytes, 0) == cudaSuccess;
}

template <typename P>
void free_dev(P*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// Device array of at least `bytes`, kept between rebuilds (grow only).
template <typename P>
int ensure(P*& p, size_t& cap, size_t bytes) {
  if (bytes <= cap && p) return PBG_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const size_t want = std::max<size_t>(bytes + bytes / 4, 256);
  if (cudaMalloc((void**)&p, want) != cudaSuccess) {
    cudaGetLastError();
    pbg_set_error_message("out of device memory for the batch descriptors (%zu bytes)", want);
    return PBG_ERR_NOMEM;
  }
  cap = want;
  return PBG_OK;
}

// Merged task list: copies every segment and writes its replica index.
__global__ void gather_tasks_kernel(const GatherSeg* __restrict__ segs, int nseg, int4* __restrict__ out) {
  for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
    const GatherSeg g = segs[s];
    for (int t = threadIdx.x; t < g.count; t += blockDim.x) {
      int4 v = g.src[t];
      v.x = (v.x & 7) | (g.replica << 3);
      out[g.dst + t] = v;
    }
  }
}

// Ewald work list: replica q's lower-triangle bead tiles (I, J), I >= J, in
// row order, at parts[q].y; parts[q].x = tiles per edge.
__global__ void ewald_work_kernel(const int4* __restrict__ parts, int4* __restrict__ out) {
  const int q = blockIdx.y;
  const int T = parts[q].x;
  const long long off = parts[q].y;
  const int total = T * (T + 1) / 2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    while (I * (I + 1) / 2 > t) --I;
    out[off + t] = make_int4(q, I, t - I * (I + 1) / 2, 0);
  }
}

// After device steps the device streams are ahead of the host's draw
// counts: copy them back (active order) before anything reads or changes
// them on the host or reorders the replicas.
int pull_draws(pbg_batch* b) {
  if (!b->host_draws_stale) return PBG_OK;
  const int R = (int)b->active.size();
  std::vector<unsigned long long> h(2 * (size_t)R);
  if (R) PBG_CUDA_TRY(cudaMemcpy(h.data(), b->d_stream, h.size() * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost));
  for (int q = 0; q < R; ++q) {
    BatchReplica* r = b->slots[b->active[q]];
    if (r) r->draws = h[2 * q + 1];
  }
  b->host_draws_stale = false;
  b->streams_on_device = false;
  return PBG_OK;
}

// Uploads every replica's (seed, draws) in the active order, unless the
// device copy is current.
int push_streams(pbg_batch* b, cudaStream_t st) {
  if (b->streams_on_device) return PBG_OK;
  const int R = (int)b->active.size();
  std::vector<unsigned long long> streams(2 * (size_t)R);
  for (int q = 0; q < R; ++q) {
    const BatchReplica* r = b->slots[b->active[q]];
    streams[2 * q] = r->seed;
    streams[2 * q + 1] = r->draws;
  }
  // pageable source: staged before the call returns
  if (R) PBG_CUDA_TRY(cudaMemcpyAsync(b->d_stream, streams.data(), streams.size() * sizeof(unsigned long long),
                                      cudaMemcpyHostToDevice, st));
  b->streams_on_device = true;
  return PBG_OK;
}

void drop_graphs(pbg_batch* b) {
  if (b->begin_exec) {
    cudaGraphExecDestroy(b->begin_exec);
    b->begin_exec = nullptr;
  }
  if (b->step_exec) {
    cudaGraphExecDestroy(b->step_exec);
    b->step_exec = nullptr;
  }
}

// Rebuilds the device descriptors and work lists of the current membership:
// small per-replica descriptors from the host, the task and tile work lists
// assembled on the device from each replica's cached list.
int rebuild(pbg_batch* b, cudaStream_t st) {
  int rc0 = pull_draws(b);
  if (rc0) return rc0;
  b->streams_on_device = false;
  drop_graphs(b);
  b->key_repeats = 0;
  b->key_build = -1;
  b->active.clear();
  for (int s = 0; s < (int)b->slots.size(); ++s)
    if (b->slots[s]) b->active.push_back(s);
  const int R = (int)b->active.size();
  b->n_ework = b->ntasks = 0;
  if ((size_t)R > b->cap || !b->d_ovl) {
    // the kernels of earlier steps on this stream may still read the old
    // arrays: the stream-ordered frees wait for them, the host buffers are
    // released once the stream has drained
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
    for (void* p : {(void*)b->d_ovl, (void*)b->d_mask, (void*)b->d_stream, (void*)b->d_maxatt})
      if (p) PBG_CUDA_TRY(cudaFreeAsync(p, st));
    b->d_ovl = nullptr;
    b->d_mask = nullptr;
    b->d_stream = nullptr;
    b->d_maxatt = nullptr;
    if (b->h_ovl) cudaFreeHost(b->h_ovl);
    if (b->h_info) cudaFreeHost(b->h_info);
    if (b->h_step) cudaFreeHost(b->h_step);
    b->h_ovl = b->h_info = b->h_step = nullptr;
    b->cap = std::max<size_t>(2 * R, 16);
    PBG_CUDA_TRY(cudaMallocAsync((void**)&b->d_ovl, b->cap * sizeof(int), st));
    PBG_CUDA_TRY(cudaMallocAsync((void**)&b->d_mask, b->cap, st));
    PBG_CUDA_TRY(cudaMallocAsync((void**)&b->d_stream, 2 * b->cap * sizeof(unsigned long long), st));
    PBG_CUDA_TRY(cudaMallocAsync((void**)&b->d_maxatt, b->cap * sizeof(int), st));
    PBG_CUDA_TRY(cudaMallocHost(&b->h_ovl, b->cap * sizeof(int)));
    PBG_CUDA_TRY(cudaMallocHost(&b->h_info, b->cap * sizeof(int)));
    PBG_CUDA_TRY(cudaMallocHost(&b->h_step, (2 * b->cap + 4) * sizeof(int)));
  }
  b->max_n = 0;
  if (R == 0) {
    b->dirty = false;
    return PBG_OK;
  }
  // grow-only arrays: the kernels of earlier steps must be done with them
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<BatchDev> reps(R);
  std::vector<unsigned char> rpy(R * rpy_batch_arg_bytes());
  std::vector<int4> eparts(R);
  size_t flag_ints = 4, n_ework = 0, ntasks = 0;
  std::vector<size_t> flag_off(R);
  int max_seg = 0;
  for (int q = 0; q < R; ++q) {
    const BatchReplica* r = b->slots[b->active[q]];
    flag_off[q] = flag_ints;
    flag_ints += 2 * (size_t)r->nt * r->nt;
    b->max_n = std::max(b->max_n, r->n);
    const int T = (r->N + 15) / 16;
    eparts[q] = make_int4(T, (int)n_ework, 0, 0);
    n_ework += (size_t)T * (T + 1) / 2;
    ntasks += r->seg_start.empty() ? 0 : r->seg_start.back();
    max_seg = std::max(max_seg, (int)r->seg_start.size() - 1);
  }
  // after the per-replica flags: the infos, the attempt counts and the step
  // words, contiguous so that one copy reports a step
  const size_t info_off = flag_ints;
  flag_ints += 2 * (size_t)R + 4;
  b->flag_ints = flag_ints;
  int rc;
  if ((rc = ensure(b->d_flags, b->cap_flags, flag_ints * sizeof(int)))) return rc;
  b->d_info = b->d_flags + info_off;
  b->d_att = b->d_info + R;
  b->d_words = b->d_att + R;
  std::vector<CholRep> chol(R);
  const bool smith = b->hydrodynamics == PBG_HI_RPY_SMITH;
  for (int q = 0; q < R; ++q) {
    BatchReplica* r = b->slots[b->active[q]];
    BatchDev& d = reps[q];
    d.pos = r->pos;
    d.radii = r->radii;
    d.force = r->force;
    d.U = r->U;
    d.xi = r->xi;
    d.D = r->D;
    d.B = r->B;
    d.L = r->p.box_length;
    d.thr = r->p.overlap_treshold;
    d.kBT = r->p.kBT;
    d.N = r->N;
    d.n = r->n;
    d.ld = r->ld;
    d.check = r->p.check_overlaps;
    d.has_force = r->has_force;
    d.pad = 0;
    rpy_batch_arg(r->pos, r->radii, r->N, r->p.box_length, smith, b->tables, r->scale, r->D, r->B, r->ld, r->phase,
                  rpy.data() + q * rpy_batch_arg_bytes());
    CholRep& c = chol[q];
    c.A = r->B;
    c.invdiag = r->invdiag;
    c.upd = b->d_flags + flag_off[q];
    c.fin = c.upd + (size_t)r->nt * r->nt;
    c.info = b->d_info + q;
    c.ld = r->ld;
    c.n = r->n;
    c.nt = r->nt;
    c.pad = 0;
  }
  // Merge order of the replicas' task segments (see cholesky_df.cu): by
  // segment number with larger matrices first (default), in the order the
  // replicas were added, smaller first, replica after replica (all of one
  // replica's segments, larger replicas first), or larger first in chunks of
  // replicas whose matrices fit a byte budget, chunk after chunk.  Each replica's own
  // segments keep their order in every policy, so every task still depends
  // only on earlier tasks.
  std::vector<int> order(R);
  for (int q = 0; q < R; ++q) order[q] = q;
  if (b->merge_order != PBG_MERGE_ADDED) {
    const bool larger = b->merge_order != PBG_MERGE_SMALLER_FIRST;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      const int nx = b->slots[b->active[x]]->nt, ny = b->slots[b->active[y]]->nt;
      return larger ? nx > ny : nx < ny;
    });
  }
  std::vector<GatherSeg> segs;
  long long dst = 0;
  auto push_seg = [&](int q, int sg) {
    const BatchReplica* r = b->slots[b->active[q]];
    if (sg + 1 >= (int)r->seg_start.size()) return;
    const int count = r->seg_start[sg + 1] - r->seg_start[sg];
    if (count <= 0) return;
    segs.push_back(GatherSeg{r->tasks + r->seg_start[sg], dst, count, q});
    dst += count;
  };
  if (b->merge_order == PBG_MERGE_REPLICA_MAJOR) {
    for (int q : order)
      for (int sg = 0; sg < max_seg; ++sg) push_seg(q, sg);
  } else if (b->merge_order >= PBG_MERGE_CHUNK_32M) {
    // chunks of consecutive (larger-first) replicas within the byte budget
    const size_t budget = (size_t)32 << (20 + (b->merge_order - PBG_MERGE_CHUNK_32M));
    const size_t es = b->precision == PBG_PREC_FP64 ? 8 : 4;
    for (size_t c0 = 0; c0 < order.size();) {
      size_t c1 = c0, bytes = 0;
      do {
        const BatchReplica* r = b->slots[b->active[order[c1]]];
        bytes += (size_t)r->ld * r->ld * es;
        ++c1;
      } while (c1 < order.size() && bytes + (size_t)b->slots[b->active[order[c1]]]->ld *
                                                b->slots[b->active[order[c1]]]->ld * es <= budget);
      for (int sg = 0; sg < max_seg; ++sg)
        for (size_t q = c0; q < c1; ++q) push_seg(order[q], sg);
      c0 = c1;
    }
  } else {
    for (int sg = 0; sg < max_seg; ++sg)
      for (int q : order) push_seg(q, sg);
  }
  if ((rc = ensure(b->d_reps, b->cap_reps, R * sizeof(BatchDev))) ||
      (rc = ensure(b->d_rpy, b->cap_rpy, rpy.size())) ||
      (rc = ensure(b->d_ework, b->cap_ework, n_ework * sizeof(int4))) ||
      (rc = ensure(b->d_chol, b->cap_chol, R * sizeof(CholRep))) ||
      (rc = ensure(b->d_tasks, b->cap_tasks, std::max<size_t>(ntasks, 1) * sizeof(int4))) ||
      (rc = ensure(b->d_segs, b->cap_segs, std::max<size_t>(segs.size(), 1) * sizeof(GatherSeg))) ||
      (rc = ensure(b->d_eparts, b->cap_eparts, R * sizeof(int4))))
    return rc;
  // pageable sources: each copy is staged before the call returns
  PBG_CUDA_TRY(cudaMemcpyAsync(b->d_reps, reps.data(), R * sizeof(BatchDev), cudaMemcpyHostToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(b->d_rpy, rpy.data(), rpy.size(), cudaMemcpyHostToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(b->d_chol, chol.data(), R * sizeof(CholRep), cudaMemcpyHostToDevice, st));
  PBG_CUDA_TRY(cudaMemcpyAsync(b->d_eparts, eparts.data(), R * sizeof(int4), cudaMemcpyHostToDevice, st));
  std::vector<int> maxatt(R);
  for (int q = 0; q < R; ++q) maxatt[q] = std::max(1, b->slots[b->active[q]]->p.max_move_attempts);
  PBG_CUDA_TRY(cudaMemcpyAsync(b->d_maxatt, maxatt.data(), R * sizeof(int), cudaMemcpyHostToDevice, st));
  if (!segs.empty()) {
    PBG_CUDA_TRY(cudaMemcpyAsync(b->d_segs, segs.data(), segs.size() * sizeof(GatherSeg), cudaMemcpyHostToDevice,
                                 st));
    gather_tasks_kernel<<<(int)std::min<size_t>(segs.size(), 148 * 16), 256, 0, st>>>(b->d_segs, (int)segs.size(),
                                                                                      b->d_tasks);
    PBG_CHECK_LAUNCH();
  }
  ewald_work_kernel<<<dim3(8, R), 256, 0, st>>>(b->d_eparts, b->d_ework);
  PBG_CHECK_LAUNCH();
  b->n_ework = (int)n_ework;
  b->ntasks = (int)dst;
  b->dirty = false;
  return PBG_OK;
}

inline dim3 rows_grid(const pbg_batch* b, int per_block) {
  const int x = std::max(1, std::min(64, (b->max_n + per_block - 1) / per_block));
  return dim3(x, (unsigned)b->active.size());
}

// Copies the host mask (indexed by slot, or all when null) to the device in
// the order of the active replicas.  Returns the number of masked replicas.
// Small uploads go from pageable memory: the copy is staged before the call
// returns, so the host vectors can change right away.
int upload_mask(pbg_batch* b, const unsigned char* mask, cudaStream_t st, int* count) {
  const int R = (int)b->active.size();
  b->mask.assign(R, 0);
  int c = 0;
  for (int q = 0; q < R; ++q) {
    b->mask[q] = mask ? (mask[b->active[q]] ? 1 : 0) : 1;
    c += b->mask[q];
  }
  *count = c;
  if (R) PBG_CUDA_TRY(cudaMemcpyAsync(b->d_mask, b->mask.data(), R, cudaMemcpyHostToDevice, st));
  return PBG_OK;
}

}  // namespace
}  // namespace pbg

using namespace pbg;

extern "C" {

PBG_API int pbg_batch_create(const pbg_params* tmpl, pbg_batch** out) {
  if (!tmpl || !out) return PBG_ERR_ARG;
  if (tmpl->hydrodynamics != PBG_HI_RPY && tmpl->hydrodynamics != PBG_HI_RPY_SMITH) {
    pbg_set_error_message("batched replicas support the rpy and rpy_smith hydrodynamics");
    return PBG_ERR_ARG;
  }
  if (tmpl->precision != PBG_PREC_FP64 && tmpl->precision != PBG_PREC_MIXED) return PBG_ERR_ARG;
  if (tmpl->propagation_scheme != PBG_SCHEME_ERMAK) {
    pbg_set_error_message("batched replicas support the ermak propagation scheme");
    return PBG_ERR_ARG;
  }
  auto* b = new pbg_batch();
  b->precision = tmpl->precision;
  b->hydrodynamics = tmpl->hydrodynamics;
  if (b->hydrodynamics == PBG_HI_RPY_SMITH) {
    b->alpha = tmpl->ewald_alpha;
    b->m_max = tmpl->ewald_real;
    b->n_max = tmpl->ewald_imag;
    int rc = get_ewald_tables(b->alpha, b->m_max, b->n_max, &b->tables);
    if (rc) {
      delete b;
      return rc;
    }
  }
  *out = b;
  return PBG_OK;
}

PBG_API int pbg_batch_destroy(pbg_batch* b) {
  if (!b) return PBG_OK;
  cudaDeviceSynchronize();
  for (auto* r : b->slots) free_replica(r);
  free_dev(b->d_reps);
  free_dev(b->d_rpy);
  free_dev(b->d_ework);
  free_dev(b->d_chol);
  free_dev(b->d_tasks);
  free_dev(b->d_segs);
  free_dev(b->d_eparts);
  free_dev(b->d_flags);
  free_dev(b->d_ovl);
  free_dev(b->d_mask);
  free_dev(b->d_stream);
  free_dev(b->d_maxatt);
  if (b->h_ovl) cudaFreeHost(b->h_ovl);
  if (b->h_info) cudaFreeHost(b->h_info);
  if (b->h_step) cudaFreeHost(b->h_step);
  drop_graphs(b);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->cap_stream2) cudaStreamDestroy(b->cap_stream2);
  delete b;
  return PBG_OK;
}

PBG_API int pbg_cholesky_task_list(int nt, int precision, int* tasks, int cap, int* seg, int seg_cap, int* n_tasks,
                                   int* n_segs) {
  if (nt < 1 || !tasks || !seg || !n_tasks || !n_segs) return PBG_ERR_ARG;
  std::vector<int4> list;
  std::vector<int> starts;
  cholesky_replica_tasks(nt, precision, list, starts);
  *n_tasks = (int)list.size();
  *n_segs = (int)starts.size();
  if ((int)list.size() > cap || (int)starts.size() > seg_cap) return PBG_ERR_ARG;
  for (size_t t = 0; t < list.size(); ++t) {
    tasks[4 * t + 0] = list[t].x;
    tasks[4 * t + 1] = list[t].y;
    tasks[4 * t + 2] = list[t].z;
    tasks[4 * t + 3] = list[t].w;
  }
  for (size_t q = 0; q < starts.size(); ++q) seg[q] = starts[q];
  return PBG_OK;
}

// Device bytes a replica of n_beads takes in a batch of this precision.
PBG_API long long pbg_batch_footprint(int precision, int hydrodynamics, int ewald_imag, int n_beads) {
  const long long n = 3LL * n_beads, ld = (n + PBG_TILE - 1) / PBG_TILE * PBG_TILE, nt = ld / PBG_TILE;
  const long long es = elem_size(precision);
  long long n_recip = 0;
  if (hydrodynamics == PBG_HI_RPY_SMITH)
    for (int x = -ewald_imag; x <= ewald_imag; ++x)
      for (int y = -ewald_imag; y <= ewald_imag; ++y)
        for (int z = -ewald_imag; z <= ewald_imag; ++z)
          if (std::abs(x) + std::abs(y) + std::abs(z) <= ewald_imag && (x || y || z)) ++n_recip;
  n_recip /= 2;
  return 2 * ld * ld * es + nt * PBG_TILE * PBG_TILE * es + (long long)n_beads * n_recip * 2 * es +
         (4 * ld + 4 * n_beads) * 8 + 2 * nt * nt * 4;
}

PBG_API int pbg_batch_add(pbg_batch* b, const pbg_params* p, const double* pos, const double* radii, int* slot) {
  if (!b || !p || !pos || !radii || !slot || p->n_beads <= 0 || !(p->box_length > 0) || !(p->kBT > 0) ||
      !(p->viscosity > 0))
    return PBG_ERR_ARG;
  if (b->in_step) {
    pbg_set_error_message("pbg_batch_add inside a step");
    return PBG_ERR_STATE;
  }
  int prc = pull_draws(b);
  if (prc) return prc;
  auto* r = new BatchReplica();
  r->p = *p;
  r->N = p->n_beads;
  r->n = 3 * r->N;
  r->ld = (r->n + PBG_TILE - 1) / PBG_TILE * PBG_TILE;
  r->nt = r->ld / PBG_TILE;
  r->scale = p->kBT * 1e19 / p->viscosity;
  const size_t es = elem_size(b->precision), ld = r->ld;
  batch_pool_keep();
  bool ok = pool_alloc(&r->pos, r->n * sizeof(double)) && pool_alloc(&r->radii, r->N * sizeof(double)) &&
            pool_alloc(&r->force, ld * sizeof(double)) && pool_alloc(&r->U, ld * sizeof(double)) &&
            pool_alloc(&r->xi, ld * sizeof(double)) && pool_alloc(&r->D, ld * ld * es) &&
            pool_alloc(&r->B, ld * ld * es) && pool_alloc(&r->invdiag, (size_t)r->nt * PBG_TILE * PBG_TILE * es);
  const size_t ph = phase_scratch_bytes(r->N, b->tables, b->precision);
  if (ok && ph) ok = pool_alloc(&r->phase, ph);
  std::vector<int4> tasks;
  cholesky_replica_tasks(r->nt, b->precision, tasks, r->seg_start);
  if (ok && !tasks.empty()) {
    ok = pool_alloc(&r->tasks, tasks.size() * sizeof(int4)) &&
         cudaMemcpyAsync(r->tasks, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice, 0) ==
             cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    free_replica(r);
    pbg_set_error_message("out of device memory adding a replica of %d beads", p->n_beads);
    return PBG_ERR_NOMEM;
  }
  cudaMemsetAsync(r->force, 0, ld * sizeof(double), 0);
  cudaMemsetAsync(r->U, 0, ld * sizeof(double), 0);
  cudaMemsetAsync(r->xi, 0, ld * sizeof(double), 0);
  // ordered on the legacy stream after the allocations; a pageable source is
  // staged before the call returns
  PBG_CUDA_TRY(cudaMemcpyAsync(r->pos, pos, r->n * sizeof(double), cudaMemcpyDefault, 0));
  PBG_CUDA_TRY(cudaMemcpyAsync(r->radii, radii, r->N * sizeof(double), cudaMemcpyDefault, 0));
  int s = 0;
  while (s < (int)b->slots.size() && b->slots[s]) ++s;
  if (s == (int)b->slots.size()) b->slots.push_back(nullptr);
  b->slots[s] = r;
  b->dirty = true;
  *slot = s;
  return PBG_OK;
}

static BatchReplica* slot_of(pbg_batch* b, int slot) {
  if (!b || slot < 0 || slot >= (int)b->slots.size()) return nullptr;
  return b->slots[slot];
}

PBG_API int pbg_batch_remove(pbg_batch* b, int slot) {
  BatchReplica* r = slot_of(b, slot);
  if (!r) return PBG_ERR_ARG;
  if (b->in_step) {
    pbg_set_error_message("pbg_batch_remove inside a step");
    return PBG_ERR_STATE;
  }
  int rc = pull_draws(b);
  if (rc) return rc;
  free_replica(r);
  b->slots[slot] = nullptr;
  b->dirty = true;
  return PBG_OK;
}

PBG_API int pbg_batch_slots(pbg_batch* b) { return b ? (int)b->slots.size() : 0; }

PBG_API int pbg_batch_set_positions(pbg_batch* b, int slot, const double* pos) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !pos) return PBG_ERR_ARG;
  PBG_CUDA_TRY(cudaMemcpy(r->pos, pos, r->n * sizeof(double), cudaMemcpyDefault));
  return PBG_OK;
}

PBG_API int pbg_batch_get_positions(pbg_batch* b, int slot, double* out) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !out) return PBG_ERR_ARG;
  PBG_CUDA_TRY(cudaMemcpy(out, r->pos, r->n * sizeof(double), cudaMemcpyDefault));
  return PBG_OK;
}

// Stream-ordered copy of one replica's positions into `out` (pinned host
// memory for the copy to be asynchronous); the caller waits on the stream.
PBG_API int pbg_batch_get_positions_async(pbg_batch* b, int slot, double* out, void* stream) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !out) return PBG_ERR_ARG;
  PBG_CUDA_TRY(cudaMemcpyAsync(out, r->pos, r->n * sizeof(double), cudaMemcpyDefault, (cudaStream_t)stream));
  return PBG_OK;
}

PBG_API int pbg_batch_set_force(pbg_batch* b, int slot, const double* F) {
  BatchReplica* r = slot_of(b, slot);
  if (!r) return PBG_ERR_ARG;
  if (F) PBG_CUDA_TRY(cudaMemcpy(r->force, F, r->n * sizeof(double), cudaMemcpyDefault));
  else PBG_CUDA_TRY(cudaMemset(r->force, 0, r->n * sizeof(double)));
  if (r->has_force != (F != nullptr)) b->dirty = true;
  r->has_force = F != nullptr;
  return PBG_OK;
}

// Noise for the next attempt of one replica (3N normals, host or device memory).
PBG_API int pbg_batch_set_noise(pbg_batch* b, int slot, const double* xi) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !xi) return PBG_ERR_ARG;
  PBG_CUDA_TRY(cudaMemcpy(r->xi, xi, r->n * sizeof(double), cudaMemcpyDefault));
  return PBG_OK;
}

PBG_API int pbg_batch_set_seed(pbg_batch* b, int slot, unsigned long long seed, unsigned long long draws) {
  BatchReplica* r = slot_of(b, slot);
  if (!r) return PBG_ERR_ARG;
  int rc = pull_draws(b);
  if (rc) return rc;
  r->seed = seed;
  r->draws = draws + (draws & 1);
  b->streams_on_device = false;
  return PBG_OK;
}

PBG_API int pbg_batch_get_draws(pbg_batch* b, int slot, unsigned long long* draws) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !draws) return PBG_ERR_ARG;
  int rc = pull_draws(b);
  if (rc) return rc;
  *draws = r->draws;
  return PBG_OK;
}

// Fills the masked replicas' noise from their counter-based streams and
// advances each stream by 3N draws (rounded up to even).
PBG_API int pbg_batch_fill_noise(pbg_batch* b, const unsigned char* mask, void* stream) {
  if (!b) return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (b->dirty && (rc = rebuild(b, st))) return rc;
  const int R = (int)b->active.size();
  if (!R) return PBG_OK;
  int count = 0;
  if ((rc = upload_mask(b, mask, st, &count))) return rc;
  if (!count) return PBG_OK;
  // the stream positions of this fill (the host counts are authoritative here)
  if ((rc = pull_draws(b))) return rc;
  b->streams_on_device = false;
  if ((rc = push_streams(b, st))) return rc;
  batch_noise_kernel<<<rows_grid(b, 512), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_stream);
  PBG_CHECK_LAUNCH();
  for (int q = 0; q < R; ++q)
    if (b->mask[q]) {
      BatchReplica* r = b->slots[b->active[q]];
      r->draws += (unsigned long long)(r->n + (r->n & 1));
    }
  b->streams_on_device = false;  // the device copy is now behind the host counts
  return PBG_OK;
}

// The device work of a step's start: D (build_D), B = chol(D) (cholesky) of
// every replica and the deterministic move of the replicas with a force.
static int enqueue_begin(pbg_batch* b, double dt, int build_D, int cholesky, bool any_force, cudaStream_t st) {
  const int R = (int)b->active.size();
  const bool f64 = b->precision == PBG_PREC_FP64;
  const bool smith = b->hydrodynamics == PBG_HI_RPY_SMITH;
  int rc;
  // a step that builds and factors D has the Ewald build write D's lower
  // triangle into B as well; only B's padding rows are then set here
  if (build_D && (rc = launch_rpy_batch(b->precision, smith, b->tables, b->d_rpy, b->d_ework, b->n_ework, R,
                                        cholesky != 0, st)))
    return rc;
  if (cholesky) {
    if (build_D) {
      const dim3 g(1, R);
      if (f64) batch_pad_lower_kernel<double><<<g, 256, 0, st>>>(b->d_reps);
      else batch_pad_lower_kernel<float><<<g, 256, 0, st>>>(b->d_reps);
    } else {
      const dim3 g(64, R);
      if (f64) batch_copy_lower_kernel<double><<<g, 256, 0, st>>>(b->d_reps);
      else batch_copy_lower_kernel<float><<<g, 256, 0, st>>>(b->d_reps);
    }
    PBG_CHECK_LAUNCH();
    PBG_CUDA_TRY(cudaMemsetAsync(b->d_flags, 0, b->flag_ints * sizeof(int), st));
    if ((rc = launch_cholesky_batch(b->precision, b->d_chol, b->d_tasks, b->ntasks, b->d_flags, b->ctas_per_sm, st)))
      return rc;
  }
  if (any_force) {
    if (f64) batch_det_kernel<double><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, dt);
    else batch_det_kernel<float><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, dt);
    PBG_CHECK_LAUNCH();
    batch_det_move_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps);
    PBG_CHECK_LAUNCH();
  }
  return PBG_OK;
}

// Captures enqueue_begin into b->begin_exec on the private stream.  A refusal
// by the driver (capture or instantiation) leaves graph_refused set and the
// step runs its launches directly; any other error is returned.
static int capture_begin(pbg_batch* b, double dt, int build_D, int cholesky, bool any_force) {
  if (!b->cap_stream) PBG_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  const long long l0 = pbg_launch_count();
  if (cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    b->graph_refused = true;
    return PBG_OK;
  }
  int rc = enqueue_begin(b, dt, build_D, cholesky, any_force, b->cap_stream);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->cap_stream, &graph);
  const long long kernels = pbg_launch_count() - l0;
  pbg_count_launches(-kernels);  // nothing ran yet
  pbg_count_host_calls(-kernels);
  if (rc != PBG_OK || end != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    b->graph_refused = true;
    return PBG_OK;
  }
  const cudaError_t inst = cudaGraphInstantiate(&b->begin_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) {
    cudaGetLastError();
    b->begin_exec = nullptr;
    b->graph_refused = true;
    return PBG_OK;
  }
  b->begin_kernels = kernels;
  return PBG_OK;
}

// Builds D (build_D) and B = chol(D) (cholesky) of every replica and applies
// the deterministic step of the replicas with a force.  The second and later
// steps with the same membership, flags and dt replay one CUDA graph.
PBG_API int pbg_batch_step_begin(pbg_batch* b, double dt, int build_D, int cholesky, void* stream) {
  if (!b || !(dt > 0)) return PBG_ERR_ARG;
  if (b->in_step) {
    pbg_set_error_message("pbg_batch_step_begin inside a step");
    return PBG_ERR_STATE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (b->dirty && (rc = rebuild(b, st))) return rc;
  b->dt = dt;
  const int R = (int)b->active.size();
  if (!R) {
    b->in_step = true;
    return PBG_OK;
  }
  bool any_force = false;
  for (int s : b->active) any_force = any_force || b->slots[s]->has_force;
  const bool same = b->key_build == build_D && b->key_chol == cholesky && b->key_force == (int)any_force &&
                    b->key_dt == dt;
  if (!same) {
    if (b->begin_exec) {
      cudaGraphExecDestroy(b->begin_exec);
      b->begin_exec = nullptr;
    }
    b->key_build = build_D;
    b->key_chol = cholesky;
    b->key_force = (int)any_force;
    b->key_dt = dt;
    b->key_repeats = 0;
  }
  ++b->key_repeats;
  if (!b->begin_exec && !b->graph_refused && b->key_repeats >= 2 &&
      (rc = capture_begin(b, dt, build_D, cholesky, any_force)))
    return rc;
  if (b->begin_exec) {
    PBG_CUDA_TRY(cudaGraphLaunch(b->begin_exec, st));
    pbg_count_launches(b->begin_kernels);
    pbg_count_host_calls(1);
  } else if ((rc = enqueue_begin(b, dt, build_D, cholesky, any_force, st))) {
    return rc;
  }
  if (build_D) b->have_D = true;
  b->in_step = true;
  return PBG_OK;
}

// One round of attempts of the replicas still moving (mask): their noise,
// U = B xi, the move, the overlap test, the undo of the rejected moves and
// the round's bookkeeping (batch_round_update_kernel).  Six kernels.
static int enqueue_round(pbg_batch* b, cudaStream_t st, cudaGraphConditionalHandle handle, int use_handle) {
  const int R = (int)b->active.size();
  const bool f64 = b->precision == PBG_PREC_FP64;
  const double s1 = std::sqrt(2 * b->dt);
  batch_noise_kernel<<<rows_grid(b, 512), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_stream);
  PBG_CHECK_LAUNCH();
  if (f64) batch_trmv_kernel<double><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, b->d_mask);
  else batch_trmv_kernel<float><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, b->d_mask);
  PBG_CHECK_LAUNCH();
  batch_move_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl, s1, 1.0, 0);
  PBG_CHECK_LAUNCH();
  PBG_CUDA_TRY(cudaMemsetAsync(b->d_ovl, 0, R * sizeof(int), st));
  batch_overlap_kernel<<<dim3(64, R), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl);
  PBG_CHECK_LAUNCH();
  batch_move_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl, s1, -1.0, 1);
  PBG_CHECK_LAUNCH();
  batch_round_update_kernel<<<1, 1024, 0, st>>>(b->d_reps, R, b->d_mask, b->d_ovl, b->d_att, b->d_maxatt,
                                                 b->d_stream, b->d_words, handle, use_handle);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}
constexpr int ROUND_KERNELS = 6;

// The wrap into the box and the step's report (infos, attempts, words) into
// pinned host memory.
static int enqueue_step_tail(pbg_batch* b, cudaStream_t st) {
  const int R = (int)b->active.size();
  batch_wrap_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps);
  PBG_CHECK_LAUNCH();
  PBG_CUDA_TRY(cudaMemcpyAsync(b->h_step, b->d_info, (2 * (size_t)R + 4) * sizeof(int), cudaMemcpyDeviceToHost, st));
  return PBG_OK;
}

static int enqueue_round_init(pbg_batch* b, cudaStream_t st) {
  const int R = (int)b->active.size();
  batch_round_init_kernel<<<(R + 255) / 256, 256, 0, st>>>(R, b->d_mask, b->d_att, b->d_words);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

// Captures a whole device step into b->step_exec: the start (enqueue_begin),
// the round initialisation, a conditional WHILE node whose body is one round
// (its last kernel sets the condition), and the tail.  A refusal by the
// driver leaves graph_refused set (direct launches from then on).
static int capture_step(pbg_batch* b, double dt, int build_D, int cholesky, bool any_force) {
  if (!b->cap_stream) PBG_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  if (!b->cap_stream2) PBG_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream2, cudaStreamNonBlocking));
  const long long l0 = pbg_launch_count();
  auto refuse = [&](cudaGraph_t g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    const long long k = pbg_launch_count() - l0;  // nothing ran
    pbg_count_launches(-k);
    pbg_count_host_calls(-k);
    b->graph_refused = true;
    return PBG_OK;
  };
  if (cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) return refuse(nullptr);
  int rc = enqueue_begin(b, dt, build_D, cholesky, any_force, b->cap_stream);
  if (rc == PBG_OK) rc = enqueue_round_init(b, b->cap_stream);
  const long long fixed0 = pbg_launch_count() - l0;
  bool ok = rc == PBG_OK;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle handle = 0;
  cudaGraphNodeParams cp = {};
  if (ok) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    ok = cudaStreamGetCaptureInfo(b->cap_stream, &cs, nullptr, &g, &deps, &ndeps) == cudaSuccess &&
         cs == cudaStreamCaptureStatusActive &&
         cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNode_t wnode = nullptr;
    if (ok) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&wnode, g, deps, ndeps, &cp) == cudaSuccess &&
           cudaStreamUpdateCaptureDependencies(b->cap_stream, &wnode, 1, cudaStreamSetCaptureDependencies) ==
               cudaSuccess;
    }
    if (ok) {
      ok = cudaStreamBeginCaptureToGraph(b->cap_stream2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed) == cudaSuccess;
      if (ok) {
        rc = enqueue_round(b, b->cap_stream2, handle, 1);
        cudaGraph_t body = nullptr;
        ok = cudaStreamEndCapture(b->cap_stream2, &body) == cudaSuccess && rc == PBG_OK;
      }
    }
  }
  if (ok) ok = enqueue_step_tail(b, b->cap_stream) == PBG_OK;
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->cap_stream, &graph);
  if (!ok || end != cudaSuccess || !graph) return refuse(graph);
  const cudaError_t inst = cudaGraphInstantiate(&b->step_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) {
    b->step_exec = nullptr;
    return refuse(nullptr);
  }
  // kernels per replay besides the rounds: the start, the initialisation and the wrap
  b->step_fixed_kernels = fixed0 + 1;
  const long long k = pbg_launch_count() - l0;  // nothing ran yet
  pbg_count_launches(-k);
  pbg_count_host_calls(-k);
  return PBG_OK;
}

// 1 while the start of a step (or, with pbg_batch_step, the whole step)
// replays a CUDA graph, 0 while it launches its kernels directly, -1 if the
// driver refused the capture.
PBG_API int pbg_batch_graph_state(pbg_batch* b) {
  if (!b) return 0;
  return b->graph_refused ? -1 : ((b->begin_exec || b->step_exec) ? 1 : 0);
}

// A whole step of every replica with device noise (see the header).
PBG_API int pbg_batch_step(pbg_batch* b, double dt, int build_D, int cholesky, int* status, int* attempts,
                           void* stream) {
  if (!b || !(dt > 0)) return PBG_ERR_ARG;
  if (b->in_step) {
    pbg_set_error_message("pbg_batch_step inside a step");
    return PBG_ERR_STATE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (b->dirty && (rc = rebuild(b, st))) return rc;
  const int R = (int)b->active.size();
  if (!R) return PBG_OK;
  if ((rc = push_streams(b, st))) return rc;
  b->dt = dt;
  bool any_force = false;
  for (int s : b->active) any_force = any_force || b->slots[s]->has_force;
  const bool same = b->key_build == build_D && b->key_chol == cholesky && b->key_force == (int)any_force &&
                    b->key_dt == dt;
  if (!same) {
    drop_graphs(b);
    b->key_build = build_D;
    b->key_chol = cholesky;
    b->key_force = (int)any_force;
    b->key_dt = dt;
    b->key_repeats = 0;
  }
  ++b->key_repeats;
  if (!b->step_exec && !b->graph_refused && b->key_repeats >= 2 &&
      (rc = capture_step(b, dt, build_D, cholesky, any_force)))
    return rc;
  const int* words = b->h_step + 2 * R;
  if (b->step_exec) {
    PBG_CUDA_TRY(cudaGraphLaunch(b->step_exec, st));
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
    pbg_count_launches(b->step_fixed_kernels + (long long)ROUND_KERNELS * words[2]);
    pbg_count_host_calls(1);
  } else {
    if ((rc = enqueue_begin(b, dt, build_D, cholesky, any_force, st)) || (rc = enqueue_round_init(b, st)))
      return rc;
  }
  // rounds launched from the host: all of them without a graph, or those
  // beyond the graph's round cap
  int* h_words = b->h_step + 2 * R;
  bool more = !b->step_exec;
  if (b->step_exec && words[0]) {
    more = true;
  }
  while (more) {
    if ((rc = enqueue_round(b, st, 0, 0))) return rc;
    PBG_CUDA_TRY(cudaMemcpyAsync(h_words, b->d_words, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
    more = h_words[0] != 0;
  }
  if (!b->step_exec || words[0]) {
    // not replayed, or rounds were added: the tail runs here
    if ((rc = enqueue_step_tail(b, st))) return rc;
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
  }
  b->have_D = b->have_D || build_D;
  b->streams_on_device = true;
  b->host_draws_stale = true;
  int worst = 0;
  for (int q = 0; q < R; ++q) {
    const int slot = b->active[q];
    if (status) status[slot] = b->h_step[q];
    if (attempts) attempts[slot] = b->h_step[R + q];
    if (b->h_step[q] < 0) worst = -1;
    else if (b->h_step[q] > 0 && worst == 0) worst = 1;
  }
  if (words[1] & PBG_DEV_ERR_ATTEMPTS) {
    pbg_set_error_message("maximal number of move attempts exceeded in a batched step");
    return PBG_ERR_ATTEMPTS;
  }
  if (worst < 0) {
    pbg_set_error_message("a device-wide wait in the batched factorisation gave up");
    return PBG_ERR_BARRIER;
  }
  if (worst > 0) {
    pbg_set_error_message("a replica's diffusion matrix is not positive definite");
    return PBG_ERR_NOT_SPD;
  }
  return PBG_OK;
}

PBG_API int pbg_batch_step_attempt(pbg_batch* b, const unsigned char* mask, unsigned char* accepted, void* stream) {
  if (!b) return PBG_ERR_ARG;
  if (!b->in_step) {
    pbg_set_error_message("pbg_batch_step_attempt outside a step");
    return PBG_ERR_STATE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int R = (int)b->active.size();
  if (!R) return PBG_OK;
  int count = 0, rc;
  if ((rc = upload_mask(b, mask, st, &count))) return rc;
  if (!count) return PBG_OK;
  const bool f64 = b->precision == PBG_PREC_FP64;
  const double s1 = std::sqrt(2 * b->dt);
  if (f64) batch_trmv_kernel<double><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, b->d_mask);
  else batch_trmv_kernel<float><<<rows_grid(b, 8), 256, 0, st>>>(b->d_reps, b->d_mask);
  PBG_CHECK_LAUNCH();
  batch_move_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl, s1, 1.0, 0);
  PBG_CHECK_LAUNCH();
  PBG_CUDA_TRY(cudaMemsetAsync(b->d_ovl, 0, R * sizeof(int), st));
  batch_overlap_kernel<<<dim3(64, R), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl);
  PBG_CHECK_LAUNCH();
  batch_move_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps, b->d_mask, b->d_ovl, s1, -1.0, 1);
  PBG_CHECK_LAUNCH();
  PBG_CUDA_TRY(cudaMemcpyAsync(b->h_ovl, b->d_ovl, R * sizeof(int), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  if (accepted)
    for (int q = 0; q < R; ++q)
      if (b->mask[q]) accepted[b->active[q]] = b->h_ovl[q] ? 0 : 1;
  return PBG_OK;
}

// Wraps every replica into its box and reports the factorisation status of
// the step: status[slot] (host, optional) = 0, or the first non-positive
// pivot (1-based), or -1 when a wait of the factorisation gave up.
PBG_API int pbg_batch_step_end(pbg_batch* b, int* status, void* stream) {
  if (!b) return PBG_ERR_ARG;
  if (!b->in_step) {
    pbg_set_error_message("pbg_batch_step_end outside a step");
    return PBG_ERR_STATE;
  }
  b->in_step = false;
  cudaStream_t st = (cudaStream_t)stream;
  const int R = (int)b->active.size();
  if (!R) return PBG_OK;
  batch_wrap_kernel<<<rows_grid(b, 256), 256, 0, st>>>(b->d_reps);
  PBG_CHECK_LAUNCH();
  PBG_CUDA_TRY(cudaMemcpyAsync(b->h_info, b->d_info, R * sizeof(int), cudaMemcpyDeviceToHost, st));
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  int worst = 0;
  for (int q = 0; q < R; ++q) {
    if (status) status[b->active[q]] = b->h_info[q];
    if (b->h_info[q] < 0) worst = -1;
    else if (b->h_info[q] > 0 && worst == 0) worst = 1;
  }
  if (worst < 0) {
    pbg_set_error_message("a device-wide wait in the batched factorisation gave up");
    return PBG_ERR_BARRIER;
  }
  if (worst > 0) {
    pbg_set_error_message("a replica's diffusion matrix is not positive definite");
    return PBG_ERR_NOT_SPD;
  }
  return PBG_OK;
}

// D or B (which = PBG_MAT_D / PBG_MAT_B) of one replica as a 3N x 3N FP64
// row-major host array.
PBG_API int pbg_batch_set_schedule(pbg_batch* b, int merge_order, int ctas_per_sm) {
  if (!b || merge_order < PBG_MERGE_LARGER_FIRST || merge_order >= PBG_MERGE_ORDERS || ctas_per_sm < 0)
    return PBG_ERR_ARG;
  if (b->in_step) {
    pbg_set_error_message("pbg_batch_set_schedule inside a step");
    return PBG_ERR_STATE;
  }
  if (merge_order != b->merge_order) b->dirty = true;
  b->merge_order = merge_order;
  b->ctas_per_sm = ctas_per_sm;
  return PBG_OK;
}

// Times the copy of D into B and the batched factorisation under each
// schedule.  Refactoring the current D reproduces the current B bit for bit
// (every tile's arithmetic is fixed by the task order of its replica).
PBG_API int pbg_batch_autotune(pbg_batch* b, int reps, int* best, float* ms, void* stream) {
  if (!b || reps < 1 || !best) return PBG_ERR_ARG;
  if (b->in_step || !b->have_D) {
    pbg_set_error_message("pbg_batch_autotune needs a completed step and must be called between steps");
    return PBG_ERR_STATE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int R = (int)b->active.size();
  const bool f64 = b->precision == PBG_PREC_FP64;
  int max_ctas = 1, sms = 0;
  if (R) {
    const int rr = cholesky_batch_residency(b->precision, &max_ctas, &sms);
    if (rr) return rr;
  }
  max_ctas = std::min(max_ctas, 2);
  if (ms)
    for (int c = 0; c < 2 * PBG_MERGE_ORDERS; ++c) ms[c] = -1.0f;
  const int old_order = b->merge_order, old_ctas = b->ctas_per_sm;
  float best_ms = -1.0f;
  best[0] = old_order;
  best[1] = old_ctas;
  cudaEvent_t e0, e1;
  PBG_CUDA_TRY(cudaEventCreate(&e0));
  PBG_CUDA_TRY(cudaEventCreate(&e1));
  int rc = PBG_OK;
  for (int order = PBG_MERGE_LARGER_FIRST; order < PBG_MERGE_ORDERS && rc == PBG_OK && R; ++order) {
    for (int ctas = 1; ctas <= max_ctas && rc == PBG_OK; ++ctas) {
      b->merge_order = order;
      b->ctas_per_sm = ctas;
      b->dirty = true;
      if ((rc = rebuild(b, st))) break;
      float total = 0.0f;
      for (int r = 0; r <= reps && rc == PBG_OK; ++r) {  // the first run is a warm-up
        if (cudaEventRecord(e0, st) != cudaSuccess) { rc = PBG_ERR_CUDA; break; }
        const dim3 g(64, R);
        if (f64) batch_copy_lower_kernel<double><<<g, 256, 0, st>>>(b->d_reps);
        else batch_copy_lower_kernel<float><<<g, 256, 0, st>>>(b->d_reps);
        if (cudaGetLastError() != cudaSuccess) { rc = PBG_ERR_CUDA; break; }
        pbg_count_launch();
        if (cudaMemsetAsync(b->d_flags, 0, b->flag_ints * sizeof(int), st) != cudaSuccess) { rc = PBG_ERR_CUDA; break; }
        if ((rc = launch_cholesky_batch(b->precision, b->d_chol, b->d_tasks, b->ntasks, b->d_flags, ctas, st))) break;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) { rc = PBG_ERR_CUDA; break; }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (r) total += t;
      }
      if (rc != PBG_OK) break;
      const float mean = total / reps;
      if (ms) ms[order * 2 + ctas - 1] = mean;
      if (best_ms < 0.0f || mean < best_ms) {
        best_ms = mean;
        best[0] = order;
        best[1] = ctas;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->merge_order = rc == PBG_OK ? best[0] : old_order;
  b->ctas_per_sm = rc == PBG_OK ? best[1] : old_ctas;
  b->dirty = true;
  if (rc == PBG_OK) {
    // surface a failed factorisation like a step would
    PBG_CUDA_TRY(cudaMemcpyAsync(b->h_info, b->d_info, R * sizeof(int), cudaMemcpyDeviceToHost, st));
    PBG_CUDA_TRY(cudaStreamSynchronize(st));
    for (int q = 0; q < R; ++q)
      if (b->h_info[q] != 0) {
        pbg_set_error_message("factorisation failed during autotuning (replica %d, info %d)", q, b->h_info[q]);
        return b->h_info[q] < 0 ? PBG_ERR_BARRIER : PBG_ERR_NOT_SPD;
      }
  }
  return rc;
}

// Factors a copy of one replica's current D with the single-matrix kernel
// (the batch's precision) and returns its status in *info (0, a 1-based
// non-positive pivot, or -1): after a failed batched step, tells a matrix
// that is not positive definite from a factorisation that failed on a good
// one.  B and the replica's state are left as they are.
PBG_API int pbg_batch_check_factor(pbg_batch* b, int slot, int* info, void* stream) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !info) return PBG_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t es = elem_size(b->precision), ld = r->ld;
  void *A = nullptr, *work = nullptr;
  int* dinfo = nullptr;
  const size_t wbytes = cholesky_work_bytes(r->ld, b->precision);
  if (cudaMallocAsync(&A, ld * ld * es, st) != cudaSuccess || cudaMallocAsync(&work, wbytes, st) != cudaSuccess ||
      cudaMallocAsync((void**)&dinfo, sizeof(int), st) != cudaSuccess) {
    cudaGetLastError();
    if (A) cudaFreeAsync(A, st);
    if (work) cudaFreeAsync(work, st);
    pbg_set_error_message("out of device memory checking a replica's factorisation");
    return PBG_ERR_NOMEM;
  }
  int rc = PBG_OK;
  if (cudaMemcpyAsync(A, r->D, ld * ld * es, cudaMemcpyDeviceToDevice, st) != cudaSuccess) rc = PBG_ERR_CUDA;
  if (rc == PBG_OK) rc = launch_pad_identity(A, r->n, r->ld, b->precision, st);
  if (rc == PBG_OK) rc = launch_cholesky_ws(A, r->n, r->ld, b->precision, dinfo, work, st);
  int h = 0;
  if (rc == PBG_OK && (cudaMemcpyAsync(&h, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                       cudaStreamSynchronize(st) != cudaSuccess))
    rc = PBG_ERR_CUDA;
  cudaFreeAsync(A, st);
  cudaFreeAsync(work, st);
  cudaFreeAsync(dinfo, st);
  *info = h;
  return rc;
}

PBG_API int pbg_batch_get_matrix(pbg_batch* b, int slot, int which, double* out) {
  BatchReplica* r = slot_of(b, slot);
  if (!r || !out || (which != PBG_MAT_D && which != PBG_MAT_B)) return PBG_ERR_ARG;
  const size_t es = elem_size(b->precision), ld = r->ld;
  std::vector<unsigned char> h(ld * ld * es);
  PBG_CUDA_TRY(cudaMemcpy(h.data(), which == PBG_MAT_D ? r->D : r->B, h.size(), cudaMemcpyDeviceToHost));
  for (int i = 0; i < r->n; ++i)
    for (int j = 0; j < r->n; ++j) {
      double v;
      if (es == 8) v = reinterpret_cast<const double*>(h.data())[(size_t)i * ld + j];
      else v = reinterpret_cast<const float*>(h.data())[(size_t)i * ld + j];
      if (which == PBG_MAT_B && j > i) v = 0.0;
      out[(size_t)i * r->n + j] = v;
    }
  return PBG_OK;
}

}  // extern "C"
