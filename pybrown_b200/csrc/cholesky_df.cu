// Data-flow tiled Cholesky factorisation on sm_100a (the factor of
// numpy.linalg.cholesky at src/bdsim/pyBrown/box.py:554).
//
// Single matrix: one persistent kernel, all CTAs co-resident (cooperative
// launch), one CTA per SM.  The 64 x 64 tiles of the lower triangle are
// processed as tasks:
//   F(k)     diagonal tile k: its last update (column k-1), then the
//            factorisation by 8-column panels (each 8 x 8 pivot block
//            factored in registers, rank-8 trailing updates by the other
//            warps) and the explicit inverse inv(L_kk);
//   S(i, k)  tile (i, k) below the diagonal: its last update, then
//            L_ik = A_ik inv(L_kk)^T as one tile product;
//   U(i,j,k) trailing update A_ij -= L_ik L_jk^T (j >= k+2): FP64 DMMA
//            (mma.sync m8n8k4 f64) in the FP64 path; in the mixed path
//            3xTF32 split products (hi*hi + hi*lo + lo*hi) on the tcgen05
//            tensor cores, up to four rows per task, accumulated in TMEM
//            (tc_tile.cuh).
// The FP64 path factors and inverts the diagonal tiles in FP64; the mixed
// path (FP32 matrix) does both in FP32 on the chain CTA (run_chain_f32), or
// in FP64 rounded to FP32 on store (PBG_PREC_MIXED_FP64_DIAG).
//
// The critical path of the factorisation is F(0), S(1,0), F(1), S(2,1), ...:
// block 0 (the chain CTA) runs exactly that sequence and keeps what one step
// hands to the next in shared memory (L(k, k-1) for the update of F(k) and
// S(k+1, k); inv(L_kk) for S(k+1, k)), so the chain never waits on a round
// trip through L2.  The other CTAs take the remaining tasks in a fixed order
// from an atomic counter: S(., 0), then for each k the solves S(i, k+1)
// (i >= k+3) and the updates U(., ., k), the update that gates the next panel
// first; the last update of the chain's next solve S(k+2, k+1) leads the list
// for panel k.  With an output X (the SPD inverse) the same list also forms
// X = inv(L) (XG / XZ tasks).  Every task depends only on chain tasks and on
// tasks earlier in the list, so with all CTAs resident the lowest unfinished
// task can always run.
//
// Batches of independent matrices: FP64 right-looking tile tasks
// (chol_batch_kernel<double>); mixed left-looking tasks that accumulate a
// whole K range on the tcgen05 tensor cores (chol_batch_ll_kernel).
//
// Dependencies are tracked per tile (per row in the left-looking batch):
// upd counts applied updates, fin marks final L tiles.  Waits spin on these
// flags with a bounded iteration count; on expiry the kernel raises an abort
// flag, marks info = -1 and every CTA returns.  Tile data written by other
// CTAs is read with L2-coherent loads (ld.global.cg, cp.async.cg).
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_tile.cuh"

namespace pbg {

namespace {

constexpr int NB = 64;
constexpr int THREADS = 256;
constexpr int TILE_PER_THREAD = 64 * 64 / THREADS;  // elements of a 64 x 64 tile per thread
constexpr int LDA = NB + 4;   // staged tile row (bank-conflict-free fragment and row loads)
constexpr long long SPIN_LIMIT = 1LL << 24;

// TASK_U2 / TASK_U3 / TASK_U4: U(i, j, k) .. U(i+r-1, j, k) as one task (they
// share L_jk).  Groups of three and four rows only in the FP32 single-matrix
// list, whose update tasks run on the tcgen05 tensor cores.
enum : int { TASK_F = 0, TASK_S = 1, TASK_U = 2, TASK_I = 3, TASK_U2 = 4, TASK_U3 = 5, TASK_U4 = 6 };
// XG / XZ: the tasks that form X = inv(L) in the same list (single-matrix
// lists of an SPD inverse only; see inverse_update / inverse_finish).
enum : int { TASK_XG = 7, TASK_XZ = 8 };

struct DFArgs {
  void* A;
  int ld, n, nt, ntasks;
  const int4* tasks;
  int* ctl;      // [0] next task, [1] abort, [2] spin failures
  int* upd;      // nt * nt
  int* fin;      // nt * nt
  int* info;
  void* invdiag; // nt * 64 * 64 (T): inv(L_kk), row-major tiles
  unsigned* err;
  long long spin_limit;  // polls before a wait gives up
  void* X;       // or null: X = inv(L) is formed too (off-diagonal tiles of the ld x ld matrix)
  int* xupd;     // nt * nt: terms applied to X's tile (i, j)
  int* xfin;     // nt * nt: X's tile (i, j) final
};

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

#ifdef PBG_TASK_TRACE
// Optional per-task timeline (build with -DPBG_TASK_TRACE): for task t,
// [fetch, waits done, end] in globaltimer ns and the SM id.  The chain tasks
// F(k), S(k+1, k) take the slots ntasks + 2k, ntasks + 2k + 1.
__device__ long long g_task_trace[4 * 65536];
__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int smid() {
  int s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return s;
}
#define TRACE(slot, t) \
  if (threadIdx.x == 0 && (t) < 65536) g_task_trace[4 * (t) + (slot)] = (slot) == 3 ? smid() : gtimer()
// Phase totals of the left-looking batch workers: per CTA, 16 slots of
// clock64 cycles or counts (see ll_task).
__device__ long long g_ll_prof[1024 * 16];
#define LLPROF(slot, v) \
  if (threadIdx.x == 0 && blockIdx.x < 1024) g_ll_prof[blockIdx.x * 16 + (slot)] += (v)
#define LLCLK() clock64()
// Finer timeline of the FP32 chain: 8 stamps per panel k.
__device__ long long g_chain_trace[8 * 1024];
#define CTRACE(k, slot) \
  if (threadIdx.x == 0 && (k) < 1024) g_chain_trace[8 * (k) + (slot)] = gtimer()
#else
#define TRACE(slot, t)
#define CTRACE(k, slot)
#define LLPROF(slot, v) ((void)(v))
#define LLCLK() 0LL
#endif

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }

// Warp 0 waits until every flags[q] >= targets[q] (count <= 9, bounded);
// returns false if the run was aborted.  Lane q polls flag q, so one round
// costs one L2 round trip whatever the count.  The acquire loads followed by
// the CTA barrier order every thread's later reads after the producers'
// release.
__device__ bool wait_all(const DFArgs& a, const int* const* flags, const int* targets, int count, int* s_ok) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int* flag = nullptr;
    int target = 0;
#pragma unroll
    for (int q = 0; q < 9; ++q)  // compile-time indices: the arrays stay in registers
      if (q < count && q == lane) {
        flag = flags[q];
        target = targets[q];
      }
    bool done = flag == nullptr;
    int ok = 1;
    for (long long it = 0;; ++it) {
      if (!done) done = ld_acquire(flag) >= target;
      if (__all_sync(0xffffffffu, done)) break;
      // the abort flag is polled every 16th round, so a round costs one L2 trip
      if ((it & 15) == 15) {
        const int ab = __shfl_sync(0xffffffffu, lane == 0 ? ld_acquire(a.ctl + 1) : 0, 0);
        if (ab) {
          ok = 0;
          break;
        }
      }
      if (it + 1 > a.spin_limit) {
        if (lane == 0) {
          atomicExch(a.ctl + 1, 1);
          atomicAdd(a.ctl + 2, 1);
          atomicOr(a.err, PBG_DEV_ERR_BARRIER);
          atomicCAS(a.info, 0, -1);  // -1: the factorisation gave up waiting
        }
        ok = 0;
        break;
      }
      if (it > 256) __nanosleep(200);
    }
    if (lane == 0) *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__device__ __forceinline__ bool wait_geq(const DFArgs& a, const int* flag, int target, int* s_ok) {
  return wait_all(a, &flag, &target, 1, s_ok);
}

// The CTA barrier makes every thread's tile stores happen-before thread 0's
// release store (release is cumulative), so no separate fence is needed.
__device__ __forceinline__ void publish(int* flag, int value) {
  __syncthreads();
  if (threadIdx.x == 0) st_release(flag, value);
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <typename T>
__device__ __forceinline__ T* tile(const DFArgs& a, int i, int j) {
  return reinterpret_cast<T*>(a.A) + (size_t)i * NB * a.ld + (size_t)j * NB;
}

// Row-major asynchronous copy of a 64 x 64 tile into smem rows of `lds`
// elements, 16 bytes per cp.async (all issued before any wait).  The caller
// waits with cp_async_wait_all() and a barrier.
template <typename T>
__device__ __forceinline__ void stage_async(const T* g, int ld, T* s, int lds) {
  constexpr int per_row = NB * (int)sizeof(T) / 16;  // 16-byte chunks per row
  constexpr int elems = 16 / (int)sizeof(T);
#pragma unroll
  for (int q = 0; q < NB * per_row / THREADS; ++q) {
    const int t = threadIdx.x + q * THREADS;
    const int r = t / per_row, c = (t % per_row) * elems;
    cp_async16(s + r * lds + c, g + (size_t)r * ld + c);
  }
}

// Asynchronous copy of `count` contiguous T (count * sizeof(T) a multiple of 16).
template <typename T>
__device__ __forceinline__ void copy_async(const T* g, T* s, int count) {
  constexpr int elems = 16 / (int)sizeof(T);
  for (int t = threadIdx.x; t < count / elems; t += THREADS) cp_async16(s + t * elems, g + t * elems);
}

// 16-byte shared-memory loads of N consecutive T (p 16-byte aligned).
template <int N>
__device__ __forceinline__ void lds_vec(const float* p, float (&v)[N]) {
#pragma unroll
  for (int q = 0; q < N; q += 4) {
    const float4 x = *reinterpret_cast<const float4*>(p + q);
    v[q] = x.x; v[q + 1] = x.y; v[q + 2] = x.z; v[q + 3] = x.w;
  }
}
template <int N>
__device__ __forceinline__ void lds_vec(const double* p, double (&v)[N]) {
#pragma unroll
  for (int q = 0; q < N; q += 2) {
    const double2 x = *reinterpret_cast<const double2*>(p + q);
    v[q] = x.x; v[q + 1] = x.y;
  }
}

// Row-major copy of a 64 x 64 smem tile (rows of `lds`) to global, 16 bytes per store.
template <typename T>
__device__ __forceinline__ void store_tile(const T* s, int lds, T* g, int ld) {
  constexpr int elems = 16 / (int)sizeof(T);
  constexpr int per_row = NB / elems;
#pragma unroll
  for (int q = 0; q < NB * per_row / THREADS; ++q) {
    const int t = threadIdx.x + q * THREADS;
    const int r = t / per_row, c = (t % per_row) * elems;
    *reinterpret_cast<float4*>(g + (size_t)r * ld + c) = *reinterpret_cast<const float4*>(s + r * lds + c);
  }
}

// ---------------------------------------------------------------- tile GEMM
// Accumulator layout: 16 elements per thread; warp w owns rows 16*(w/2).. and
// columns 32*(w%2).. of the 64 x 64 tile.  Each thread holds two rows
// (row(rs), rs = 0, 1) times eight columns (col(cs), cs = 0..7); idx(rs, cs)
// is the element's place in the accumulator array.
__device__ __forceinline__ int acc_row(int rs) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  return 16 * (w >> 1) + 8 * rs + (lane >> 2);
}
__device__ __forceinline__ int acc_col(int cs) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  return 32 * (w & 1) + 8 * (cs >> 1) + 2 * (lane & 3) + (cs & 1);
}

template <typename T> struct TileMMA;

template <> struct TileMMA<double> {
  // mma.m8n8k4 f64: 2 m-tiles x 4 n-tiles of 8 x 8, 2 accumulators each.
  static __device__ __forceinline__ int idx(int rs, int cs) { return rs * 8 + cs; }
  // acc -= A B^T with A, B (64 x 64, rows = output row / column, cols = k) in smem.
  static __device__ __forceinline__ void sub(const double* sA, const double* sB, double acc[16]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1), g = lane >> 2, t = lane & 3;
#pragma unroll 4
    for (int k0 = 0; k0 < NB; k0 += 4) {
      double a[2], b[4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) a[mt] = -sA[(m0 + 8 * mt + g) * LDA + k0 + t];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) b[nt] = sB[(n0 + 8 * nt + g) * LDA + k0 + t];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          double& c0 = acc[(mt * 4 + nt) * 2];
          double& c1 = acc[(mt * 4 + nt) * 2 + 1];
          asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                       : "+d"(c0), "+d"(c1)
                       : "d"(a[mt]), "d"(b[nt]));
        }
    }
  }
};


__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

template <> struct TileMMA<float> {
  // mma.m16n8k8 tf32: 1 m-tile of 16 x 4 n-tiles of 8, 4 accumulators each.
  // The product A B^T is accumulated from zero in its own registers and
  // subtracted from acc at the end: the tensor cores' accumulation rounds at
  // the magnitude of the product, not of the tile it updates, and acc takes
  // one FP32 rounding per product (accumulating into acc directly made the
  // factor's error grow with the number of panels, to 9e-6 at order 3072).
  static __device__ __forceinline__ int idx(int rs, int cs) { return (cs >> 1) * 4 + rs * 2 + (cs & 1); }
  static __device__ __forceinline__ void sub(const float* sA, const float* sB, float acc[16]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1), g = lane >> 2, t = lane & 3;
    float prod[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) prod[e] = 0.0f;
#pragma unroll 2
    for (int k0 = 0; k0 < NB; k0 += 8) {
      // split the A fragment and the B fragments into tf32 hi + lo
      unsigned ah[4], al[4];
      {
        const float v[4] = {sA[(m0 + g) * LDA + k0 + t], sA[(m0 + g + 8) * LDA + k0 + t],
                            sA[(m0 + g) * LDA + k0 + t + 4], sA[(m0 + g + 8) * LDA + k0 + t + 4]};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ah[q] = to_tf32(v[q]);
          al[q] = to_tf32(v[q] - __uint_as_float(ah[q]));
        }
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const float v0 = sB[(n0 + 8 * nt + g) * LDA + k0 + t];
        const float v1 = sB[(n0 + 8 * nt + g) * LDA + k0 + t + 4];
        const unsigned bh0 = to_tf32(v0), bh1 = to_tf32(v1);
        const unsigned bl0 = to_tf32(v0 - __uint_as_float(bh0)), bl1 = to_tf32(v1 - __uint_as_float(bh1));
        float* c = prod + 4 * nt;
#define PBG_TF32_MMA(A0, A1, A2, A3, B0, B1)                                                        \
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, " \
               "{%8,%9}, {%0,%1,%2,%3};"                                                            \
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])                                     \
               : "r"(A0), "r"(A1), "r"(A2), "r"(A3), "r"(B0), "r"(B1))
        PBG_TF32_MMA(al[0], al[1], al[2], al[3], bh0, bh1);
        PBG_TF32_MMA(ah[0], ah[1], ah[2], ah[3], bl0, bl1);
        PBG_TF32_MMA(ah[0], ah[1], ah[2], ah[3], bh0, bh1);
#undef PBG_TF32_MMA
      }
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] -= prod[e];
  }
};

template <typename T>
__device__ __forceinline__ void load_acc(const T* g, int ld, T acc[16]) {
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) acc[TileMMA<T>::idx(rs, cs)] = ldcg(g + (size_t)acc_row(rs) * ld + acc_col(cs));
}

template <typename T>
__device__ __forceinline__ void store_acc(T* g, int ld, const T acc[16]) {
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) g[(size_t)acc_row(rs) * ld + acc_col(cs)] = acc[TileMMA<T>::idx(rs, cs)];
}

// Loads tile (i, j) into acc and applies update U(i, j, k): the two staged L
// tiles are copied asynchronously while the accumulator loads are in flight.
template <typename T>
__device__ __forceinline__ void load_and_update(const DFArgs& a, int i, int j, int k, T acc[16], T* sA, T* sB) {
  stage_async(tile<T>(a, i, k), a.ld, sA, LDA);
  if (i != j) stage_async(tile<T>(a, j, k), a.ld, sB, LDA);
  load_acc(tile<T>(a, i, j), a.ld, acc);
  cp_async_wait_all();
  __syncthreads();
  TileMMA<T>::sub(sA, i != j ? sB : sA, acc);
  __syncthreads();
}

// ---------------------------------------------------------------- F(k)
template <typename T>
__device__ __forceinline__ T rsqrt_t(T x);
// 1/sqrt(x) for the FP64 pivots: the PTX rsqrt.approx.ftz.f64 estimate
// refined by two Newton-Raphson steps y <- y + y (1 - x y^2) / 2, which
// converge quadratically to full precision (measured <= 1.24 ulp over
// [1e-30, 1e30] against a long-double reference; the library call measured
// about 100 cycles more per pivot inside the pivot-block code).  For positive
// normal x: subnormals are flushed to zero and x <= 0 gives inf or NaN, which
// the factorisation reports as a non-positive pivot before it is used.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = fma(0.5 * y, fma(-x * y, y, 1.0), y);
  return fma(0.5 * y, fma(-x * y, y, 1.0), y);
}
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt_nr(x); }


// Panel strip row length: 8 values padded so that 16-byte row loads and the
// tensor-core fragment loads of eight different rows hit distinct banks.
template <typename T> struct Strip { static constexpr int PB = sizeof(T) == 8 ? 10 : 12; };

// Shared memory of factor_tile besides Lk and X: two panel strips
// (alternating; reused as scratch by the inversion), the reciprocal pivots.
template <typename T>
constexpr int factor_smem_elems() { return 2 * NB * Strip<T>::PB + NB; }

// Rank-8 update acc -= Pr Pc^T of the calling warp's 16 x 32 block on the
// tensor cores, Pr / Pc rows = the block's rows / columns of the panel strip
// P (8 values each).  Strip rows below `lo` are read as zero, so columns
// before the trailing part (and rows above it) are left unchanged.
__device__ __forceinline__ void strip_update(const double* P, int lo, double acc[16]) {
  constexpr int PB = Strip<double>::PB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1), g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < 8; k0 += 4) {
    double a[2], b[4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int r = m0 + 8 * mt + g;
      a[mt] = r >= lo ? -P[r * PB + k0 + t] : 0.0;
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int c = n0 + 8 * nt + g;
      b[nt] = c >= lo ? P[c * PB + k0 + t] : 0.0;
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        double& c0 = acc[(mt * 4 + nt) * 2];
        double& c1 = acc[(mt * 4 + nt) * 2 + 1];
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(c0), "+d"(c1)
                     : "d"(a[mt]), "d"(b[nt]));
      }
  }
}

// One warp's output tile D = A B of a small smem product on the tensor cores:
// A rows with stride lda (k contiguous), B k-major rows with stride ldb, K a
// multiple of 4: an 8 x 8 FP64 tile (mma m8n8k4), lane holds D[g][2t + h].
// (The diagonal tiles are inverted in FP64 in both paths.)
struct WarpTile64 {
  static constexpr int TM = 8;
  static __device__ __forceinline__ void mma(const double* A, int lda, const double* B, int ldb, int K, double d[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    d[0] = d[1] = 0.0;
    for (int k0 = 0; k0 < K; k0 += 4) {
      const double a = A[g * lda + k0 + t], b = B[(k0 + t) * ldb + g];
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(d[0]), "+d"(d[1])
                   : "d"(a), "d"(b));
    }
  }
  // element q of the lane's part of D: row, column within the tile
  static __device__ __forceinline__ int row(int q) { return (threadIdx.x & 31) >> 2; }
  static __device__ __forceinline__ int col(int q) { return 2 * (threadIdx.x & 3) + (q & 1); }
  static constexpr int NQ = 2;
};

// The FP32 counterpart on the FMA pipe (the FP32 chain inverts its diagonal
// tiles in FP32): lane (g, t) forms D[g][2t], D[g][2t + 1] as K-term dot
// products in ascending k.
struct WarpTile32 {
  static constexpr int TM = 8;
  static __device__ __forceinline__ void mma(const float* A, int lda, const float* B, int ldb, int K, float d[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float d0 = 0.0f, d1 = 0.0f;
#pragma unroll 8
    for (int k0 = 0; k0 < K; k0 += 4) {
      const float4 a4 = *reinterpret_cast<const float4*>(A + g * lda + k0);
      const float av[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float2 b = *reinterpret_cast<const float2*>(B + (k0 + q) * ldb + 2 * t);
        d0 = fmaf(av[q], b.x, d0);
        d1 = fmaf(av[q], b.y, d1);
      }
    }
    d[0] = d0;
    d[1] = d1;
  }
  static __device__ __forceinline__ int row(int q) { return (threadIdx.x & 31) >> 2; }
  static __device__ __forceinline__ int col(int q) { return 2 * (threadIdx.x & 3) + (q & 1); }
  static constexpr int NQ = 2;
};

template <typename T> struct WarpTileOf;
template <> struct WarpTileOf<double> { using type = WarpTile64; };
template <> struct WarpTileOf<float> { using type = WarpTile32; };

// Inverse of the lower-triangular L_kk (in Lk, [64][LDA], zero above the
// diagonal) into X ([64][LDA]), with Rinv[j] = 1 / L_jj and scratch Tm
// (>= 32 x 36 T).  The eight 8 x 8 diagonal blocks are inverted by forward
// substitution (warp b, lane c < 8 owns column c of block b); then three
// doubling levels s = 8, 16, 32 fill the off-diagonal blocks:
//   inv([L11 0; L21 L22]) = [X11 0; -X22 (L21 X11) X22],  X_ii = inv(L_ii),
// each level two dependent block products: by one short dot product per
// thread at s = 8, by warp tensor-core tiles at s = 16 and 32.
template <typename T>
__device__ __forceinline__ void invert_factor(const T* Lk, const T* Rinv, T* X, T* Tm) {
  using WT = typename WarpTileOf<T>::type;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (lane < 8) {
    const T* D = Lk + 8 * warp * LDA + 8 * warp;
    const T* R = Rinv + 8 * warp;
    T x[8];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
      T sacc = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q < ii && q >= lane) sacc += D[ii * LDA + q] * x[q];
      x[ii] = ii < lane ? T(0) : (ii == lane ? R[ii] : -sacc * R[ii]);
    }
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) X[(8 * warp + ii) * LDA + 8 * warp + lane] = x[ii];
  }
  // blocks above the block diagonal are zero
  for (int t = tid; t < NB * NB; t += THREADS) {
    const int r = t >> 6, c = t & 63;
    if ((c >> 3) > (r >> 3)) X[r * LDA + c] = T(0);
  }
  __syncthreads();
  // s = 8: four 8 x 8 products per phase, one output per thread
  {
    const int m = tid >> 6, rr = (tid >> 3) & 7, cc = tid & 7, b0 = 16 * m;
    T v = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) v += Lk[(b0 + 8 + rr) * LDA + b0 + q] * X[(b0 + q) * LDA + b0 + cc];
    Tm[m * 64 + rr * 8 + cc] = v;
    __syncthreads();
    T u = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) u += X[(b0 + 8 + rr) * LDA + b0 + 8 + q] * Tm[m * 64 + q * 8 + cc];
    X[(b0 + 8 + rr) * LDA + b0 + cc] = -u;
    __syncthreads();
  }
#pragma unroll
  for (int s = 16; s < NB; s *= 2) {
    const int ldt = s + 4;                              // Tm row stride
    const int tiles_r = s / WT::TM, tiles = (NB / (2 * s)) * tiles_r * (s / 8);
    // Tm = L21 X11 for every 2s x 2s diagonal block
    for (int q = warp; q < tiles; q += THREADS / 32) {
      const int m = q / (tiles_r * (s / 8)), tr = (q / (s / 8)) % tiles_r, tc = q % (s / 8), b0 = 2 * s * m;
      T d[4];
      WT::mma(Lk + (b0 + s + tr * WT::TM) * LDA + b0, LDA, X + b0 * LDA + b0 + 8 * tc, LDA, s, d);
      T* o = Tm + m * s * ldt + tr * WT::TM * ldt + 8 * tc;
#pragma unroll
      for (int e = 0; e < WT::NQ; ++e) o[WT::row(e) * ldt + WT::col(e)] = d[e];
    }
    __syncthreads();
    // X21 = -X22 Tm
    for (int q = warp; q < tiles; q += THREADS / 32) {
      const int m = q / (tiles_r * (s / 8)), tr = (q / (s / 8)) % tiles_r, tc = q % (s / 8), b0 = 2 * s * m;
      T d[4];
      WT::mma(X + (b0 + s + tr * WT::TM) * LDA + b0 + s, LDA, Tm + m * s * ldt + 8 * tc, ldt, s, d);
      T* o = X + (b0 + s + tr * WT::TM) * LDA + b0 + 8 * tc;
#pragma unroll
      for (int e = 0; e < WT::NQ; ++e) o[WT::row(e) * LDA + WT::col(e)] = -d[e];
    }
    __syncthreads();
  }
}

// inv(L_kk) from Lk ([64][LDA], zero above the diagonal) and Rinv = 1 / L_jj
// into X, then to the global invdiag array as S.  Scratch: Tm (>= 32 x 36).
template <typename T, typename S>
__device__ __forceinline__ void store_inverse(const DFArgs& a, int k, const T* Lk, const T* Rinv, T* X, T* Tm) {
  invert_factor(Lk, Rinv, X, Tm);
  S* inv = reinterpret_cast<S*>(a.invdiag) + (size_t)k * NB * NB;
  if constexpr (sizeof(S) == sizeof(T)) {
    store_tile(X, LDA, inv, NB);
  } else {
    for (int t = threadIdx.x; t < NB * NB; t += THREADS) inv[t] = (S)X[(t >> 6) * LDA + (t & 63)];
  }
}

// The eight 8 x 8 diagonal blocks of inv(L) (L in Lk, Rinv = 1 / L_jj) into
// XL[b][i][c] (8 x 8 x 8 doubles): warp b, lane c < 8 solves column c by
// forward substitution.  The caller orders XL's readers after a CTA barrier.
__device__ __forceinline__ void leaf_inverses(const double* Lk, const double* Rinv, double* XL) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane < 8) {
    const double* D = Lk + 8 * warp * LDA + 8 * warp;
    const double* R = Rinv + 8 * warp;
    double x[8];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
      double sacc = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q < ii && q >= lane) sacc += D[ii * LDA + q] * x[q];
      x[ii] = ii < lane ? 0.0 : (ii == lane ? R[ii] : -sacc * R[ii]);
    }
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) XL[warp * 64 + ii * 8 + lane] = x[ii];
  }
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// C <- C inv(L)^T for the 64 x 64 tile C (T, [64][LDA] smem) by blocked
// forward substitution in FP64 on the tensor cores: warp w owns rows
// 8w .. 8w+7 and, for each 8-column block j,
//   W_j = (C_j - W_{<j} L_{j,<j}^T) inv(L_jj)^T,
// where W ([64][LDA] doubles) holds the rows in FP64 (W may alias C when T
// is double).  L: [64][LDA] doubles, XL: leaf_inverses.  Only warp-level
// synchronisation: every warp reads its own rows, L and XL.
template <typename T>
__device__ __forceinline__ void trsm_rows(const double* L, const double* XL, T* C, double* W) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = 8 * warp;
  if constexpr (sizeof(T) != sizeof(double)) {
#pragma unroll 4
    for (int e = lane; e < 8 * NB; e += 32) W[(r0 + (e >> 6)) * LDA + (e & 63)] = (double)C[(r0 + (e >> 6)) * LDA + (e & 63)];
    __syncwarp();
  }
  double* Wr = W + r0 * LDA;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c0 = 8 * j;
    // the update's operands first, then its 2j products on four accumulators
    double av[14], bv[14];
    const double* Lj = L + (c0 + g) * LDA;
#pragma unroll
    for (int q = 0; q < 2 * j; ++q) {
      av[q] = -Wr[g * LDA + 4 * q + t];
      bv[q] = Lj[4 * q + t];
    }
    double d[4][2] = {{Wr[g * LDA + c0 + 2 * t], Wr[g * LDA + c0 + 2 * t + 1]}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int q = 0; q < 2 * j; ++q) dmma(d[q & 3], av[q], bv[q]);
    __syncwarp();
    Wr[g * LDA + c0 + 2 * t] = (d[0][0] + d[1][0]) + (d[2][0] + d[3][0]);
    Wr[g * LDA + c0 + 2 * t + 1] = (d[0][1] + d[1][1]) + (d[2][1] + d[3][1]);
    __syncwarp();
    // times inv(L_jj)^T: B[k][n] = XL[j][n][k]
    double e0[2] = {0.0, 0.0}, e1[2] = {0.0, 0.0};
    const double a0 = Wr[g * LDA + c0 + t], a1 = Wr[g * LDA + c0 + 4 + t];
    const double b0 = XL[j * 64 + g * 8 + t], b1 = XL[j * 64 + g * 8 + 4 + t];
    dmma(e0, a0, b0);
    dmma(e1, a1, b1);
    __syncwarp();
    Wr[g * LDA + c0 + 2 * t] = e0[0] + e1[0];
    Wr[g * LDA + c0 + 2 * t + 1] = e0[1] + e1[1];
    __syncwarp();
  }
  if constexpr (sizeof(T) != sizeof(double)) {
#pragma unroll 4
    for (int e = lane; e < 8 * NB; e += 32) C[(r0 + (e >> 6)) * LDA + (e & 63)] = (T)W[(r0 + (e >> 6)) * LDA + (e & 63)];
  }
}

// Factor the 64 x 64 tile held in acc (already fully updated) in T arithmetic,
// by eight 8-column panels.  Per panel p (columns c0 = 8p .. c0+7):
//  1. the owners copy the panel's column strip (rows >= c0) to shared memory;
//  2. warps 0 and 1 each factor the 8 x 8 diagonal block -- every lane holds
//     the whole block and factors it in its own registers, so the pivot chain
//     is rsqrt -> multiply -> FMA with no shuffles -- and then each lane
//     solves one strip row below it against the block (L_r = A_r L_pp^-T);
//  3. every owner takes its final strip values back, and the warps whose
//     16 x 32 block has trailing elements apply the rank-8 update on the
//     tensor cores (strip_update).
// Two CTA barriers per panel (the strips alternate between two buffers).
// Then L_kk (upper triangle zeroed) goes to global memory and to Lk
// ([64][LDA] smem), and its inverse is formed in X ([64][LDA] smem) and
// written to the global invdiag array.  Ends with a CTA barrier.
// T is the arithmetic, S the type of the matrix in global memory (the mixed
// path factors its FP32 diagonal tiles in FP64 and stores them rounded).
// Optional early fetch of the chain's next solve input during F(k): at the
// start of the last panel, if *flag >= target, the tile src is staged into dst
// ([64][LDA]) with cp.async and *ready is set (read after the tile's final
// barrier).
template <typename S>
struct SolveInput {
  const int* flag;
  int target;
  const S* src;
  int ld;
  S* dst;
  int* ready;
};

template <typename T, typename S = T, bool INVERSE = true>
__device__ __forceinline__ void factor_tile(const DFArgs& a, int k, T acc[16], T* fs, T* Lk, T* X,
                                            const SolveInput<S>* pre = nullptr) {
  constexpr int PB = Strip<T>::PB;
  T* Rinv = fs + 2 * NB * PB;  // [64] 1 / L_jj
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = 16 * (warp >> 1), n0 = 32 * (warp & 1);
#pragma unroll 1
  for (int p = 0; p < 8; ++p) {
    const int c0 = 8 * p;
    T* P = fs + (p & 1) * NB * PB;
    // this panel's columns are the accumulator column pair (c0 - n0) / 8 of
    // the warps with n0 <= c0 < n0 + 32
    const bool owner = c0 >= n0 && c0 < n0 + 32;
    const int pair = (c0 - n0) >> 3;
    if (owner) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q == pair)
#pragma unroll
          for (int rs = 0; rs < 2; ++rs)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int r = acc_row(rs), cs = 2 * q + h;
              if (r >= c0) P[r * PB + acc_col(cs) - c0] = acc[TileMMA<T>::idx(rs, cs)];
            }
    }
    // warp 7 has no trailing update in the last panel: it polls the flag
    // before the barrier, takes the value after it and stages the tile
    int pre_v = 0;
    if (pre && p == 7 && tid == 32 * 7) pre_v = ld_acquire(pre->flag);
    __syncthreads();
    if (pre && p == 7 && warp == 7) {
      const int v = __shfl_sync(0xffffffffu, pre_v, 0);
      __syncwarp();  // lane 0's acquire orders the other lanes' copies
      const bool go = v >= pre->target;
      if (go) {
        constexpr int per_row = NB * (int)sizeof(S) / 16, elems = 16 / (int)sizeof(S);
        for (int c = lane; c < NB * per_row; c += 32) {
          const int r = c / per_row, cc = (c % per_row) * elems;
          cp_async16(pre->dst + r * LDA + cc, pre->src + (size_t)r * pre->ld + cc);
        }
      }
      if (lane == 0) *pre->ready = go ? 1 : 0;
    }
    if (warp < 2) {
      // the diagonal block, in every lane (upper entries are not used)
      T l[8][8];
#pragma unroll
      for (int i = 0; i < 8; ++i) lds_vec(P + (c0 + i) * PB, l[i]);
      const int r0 = c0 + 8 + 32 * warp + lane;
      const bool v0 = r0 < NB;
      T x0[8];
      if (v0) lds_vec(P + r0 * PB, x0);
      else
#pragma unroll
        for (int c = 0; c < 8; ++c) x0[c] = T(0);
      // right-looking 8 x 8 Cholesky; a non-positive pivot is recorded and
      // reported after the block
      int bad = -1;
      T rinv[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const T d = l[j][j];
        if (!(d > T(0)) && bad < 0) bad = j;
        const T rs = rsqrt_t<T>(d);
        rinv[j] = rs;
        l[j][j] = d * rs;
#pragma unroll
        for (int i = j + 1; i < 8; ++i) l[i][j] *= rs;
#pragma unroll
        for (int i = j + 1; i < 8; ++i)
#pragma unroll
          for (int c = j + 1; c <= i; ++c) l[i][c] -= l[i][j] * l[c][j];
      }
      // the strip row below the block: x = a L_pp^-T by forward substitution
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        x0[j] *= rinv[j];
#pragma unroll
        for (int c = j + 1; c < 8; ++c) x0[c] -= x0[j] * l[c][j];
      }
      if (v0)
#pragma unroll
        for (int c = 0; c < 8; ++c) P[r0 * PB + c] = x0[c];
      if (warp == 0 && lane == 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
          for (int c = 0; c < 8; ++c) P[(c0 + i) * PB + c] = c <= i ? l[i][c] : T(0);
          Rinv[c0 + i] = rinv[i];
        }
        if (bad >= 0 && k * NB + c0 + bad < a.n) atomicCAS(a.info, 0, k * NB + c0 + bad + 1);
      }
    }
    __syncthreads();
    // final values of this panel's strip back into the accumulators
    if (owner) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q == pair)
#pragma unroll
          for (int rs = 0; rs < 2; ++rs)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int r = acc_row(rs), cs = 2 * q + h;
              if (r >= c0) acc[TileMMA<T>::idx(rs, cs)] = P[r * PB + acc_col(cs) - c0];
            }
    }
    // trailing elements (c >= c0 + 8, r >= c) exist in this warp's block?
    const int lo = c0 + 8;
    if (m0 + 15 >= lo && m0 + 15 >= n0 && n0 + 31 >= lo) strip_update(P, lo, acc);
    // no barrier here: the next panel writes the other strip buffer, and the
    // two barriers of that panel separate these reads from its next reuse
  }
  S* g = tile<S>(a, k, k);
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) {
      const int r = acc_row(rs), c = acc_col(cs);
      const T v = c <= r ? acc[TileMMA<T>::idx(rs, cs)] : T(0);
      g[(size_t)r * a.ld + c] = (S)v;
      Lk[r * LDA + c] = v;
    }
  __syncthreads();
  if constexpr (INVERSE) store_inverse<T, S>(a, k, Lk, Rinv, X, fs);
}

// acc = -(acc + ...) helpers for S: acc = C inv(L_kk)^T with C, X in smem.
template <typename T>
__device__ __forceinline__ void solve_by_inverse(const T* C, const T* X, T acc[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = T(0);
  TileMMA<T>::sub(C, X, acc);  // acc = -C X^T
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = -acc[e];
}

template <typename T>
__device__ __forceinline__ void smem_to_acc(const T* s, T acc[16]) {
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) acc[TileMMA<T>::idx(rs, cs)] = s[acc_row(rs) * LDA + acc_col(cs)];
}

template <typename T>
__device__ __forceinline__ void acc_to_smem(const T acc[16], T* s) {
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) s[acc_row(rs) * LDA + acc_col(cs)] = acc[TileMMA<T>::idx(rs, cs)];
}

// ---------------------------------------------------------------- FP32 chain
// The mixed path's chain CTA factors, inverts and solves in FP32: the
// diagonal tiles of a well-conditioned FP32 matrix lose nothing to FP32
// pivots that FP32 storage and the 3xTF32 updates have not already cost,
// while every step of the panel chain gets shorter (MUFU rsqrt instead of
// a refined FP64 rsqrt, FP32 FMA latency, no FP64 conversion).

// Named barriers (0 is __syncthreads): arrive does not wait; both order the
// calling threads' earlier shared-memory accesses before the barrier completes.
// Whole warps call them; __syncwarp first reconverges a warp after divergent
// code (the barrier instructions are warp-aligned).
__device__ __forceinline__ void bar_arrive(int id, int count) {
  __syncwarp();
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_wait(int id, int count) {
  __syncwarp();
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// T[r][c] -= sum_q T[r][c0+q] T[c][c0+q] (q = 0..7, in order): the rank-8
// update of one trailing element with the factored panel c0..c0+7.
__device__ __forceinline__ void panel_update(float* T, int r, int c, int c0) {
  const float4 a0 = *reinterpret_cast<const float4*>(T + r * LDA + c0);
  const float4 a1 = *reinterpret_cast<const float4*>(T + r * LDA + c0 + 4);
  const float4 b0 = *reinterpret_cast<const float4*>(T + c * LDA + c0);
  const float4 b1 = *reinterpret_cast<const float4*>(T + c * LDA + c0 + 4);
  float v = T[r * LDA + c];
  v = fmaf(-a0.x, b0.x, v);
  v = fmaf(-a0.y, b0.y, v);
  v = fmaf(-a0.z, b0.z, v);
  v = fmaf(-a0.w, b0.w, v);
  v = fmaf(-a1.x, b1.x, v);
  v = fmaf(-a1.y, b1.y, v);
  v = fmaf(-a1.z, b1.z, v);
  v = fmaf(-a1.w, b1.w, v);
  T[r * LDA + c] = v;
}

// F(k) of the FP32 chain on the tile T (smem [64][LDA]: lower triangle valid
// with every update applied; the caller's writes end with a CTA barrier).
// Eight 8-column panels.  Warp 0 factors panel p -- the 8 x 8 pivot block in
// every lane's registers (the pivot chain is rsqrt -> multiply -> FMA) and
// the strip rows below it (L_r = A_r L_pp^-T, one row per lane) -- while
// warps 1-7 apply the rank-8 update of panel p-1 to the trailing lower
// triangle: first the eight columns of panel p+1 (look-ahead), then the
// rest.  Named barrier 1: panel p factored (warp 0 arrives, warps 1-7
// wait); named barrier 2: panel p+1's columns updated (warps 1-7 arrive,
// warp 0 waits).  The update of panel p's columns (c0..c0+7) by warps 1-7 and
// warp 0's work on them never overlap, nor do the look-ahead and the rest.
// Returns after a CTA barrier with L_kk in T's lower triangle (the upper one
// as it was) and Rinv[j] = 1 / L_jj.  A non-positive (or NaN) pivot is
// recorded in info.
__device__ __forceinline__ void factor_tile_f32(const DFArgs& a, int k, float* T, float* Rinv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
#pragma unroll 1
    for (int p = 0; p < 8; ++p) {
      const int c0 = 8 * p;
      if (p > 0) bar_wait(2, THREADS);
      float l[8][8];
#pragma unroll
      for (int i = 0; i < 8; ++i) lds_vec(T + (c0 + i) * LDA + c0, l[i]);
      int bad = -1;
      float rinv[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float d = l[j][j];
        // a pivot below the smallest normal float (or NaN) is reported like a
        // non-positive one; the MUFU estimate (rel. error < 2^-22) is FP32 accurate
        if (!(d >= 1.17549435e-38f) && bad < 0) bad = j;
        float rs;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rs) : "f"(d));
        rinv[j] = rs;
        l[j][j] = d * rs;
#pragma unroll
        for (int i = j + 1; i < 8; ++i) l[i][j] *= rs;
#pragma unroll
        for (int i = j + 1; i < 8; ++i)
#pragma unroll
          for (int c = j + 1; c <= i; ++c) l[i][c] = fmaf(-l[i][j], l[c][j], l[i][c]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = c0 + 8 + lane + 32 * h;
        if (r < NB) {
          float x[8];
          lds_vec(T + r * LDA + c0, x);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            x[j] *= rinv[j];
#pragma unroll
            for (int c = j + 1; c < 8; ++c) x[c] = fmaf(-x[j], l[c][j], x[c]);
          }
          *reinterpret_cast<float4*>(T + r * LDA + c0) = make_float4(x[0], x[1], x[2], x[3]);
          *reinterpret_cast<float4*>(T + r * LDA + c0 + 4) = make_float4(x[4], x[5], x[6], x[7]);
        }
      }
      if (lane < 8) {  // lane i writes row c0 + i of the pivot block (zero above the diagonal) and 1 / L_ii
        float row[8], rv = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; ++c) row[c] = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (i == lane) {
#pragma unroll
            for (int c = 0; c <= i; ++c) row[c] = l[i][c];
            rv = rinv[i];
          }
        *reinterpret_cast<float4*>(T + (c0 + lane) * LDA + c0) = make_float4(row[0], row[1], row[2], row[3]);
        *reinterpret_cast<float4*>(T + (c0 + lane) * LDA + c0 + 4) = make_float4(row[4], row[5], row[6], row[7]);
        Rinv[c0 + lane] = rv;
      }
      if (lane == 0 && bad >= 0 && k * NB + c0 + bad < a.n) atomicCAS(a.info, 0, k * NB + c0 + bad + 1);
      bar_arrive(1, THREADS);
    }
  } else {
    const int t = threadIdx.x - 32, nthr = THREADS - 32;
#pragma unroll 1
    for (int p = 0; p < 8; ++p) {
      const int c0 = 8 * p;
      bar_wait(1, THREADS);
      if (p == 7) break;
      // look-ahead: the columns c0+8 .. c0+15 of panel p+1, rows below them
      for (int e = t; e < (NB - c0 - 8) * 8; e += nthr) {
        const int r = c0 + 8 + (e >> 3), c = c0 + 8 + (e & 7);
        if (c <= r) panel_update(T, r, c, c0);
      }
      bar_arrive(2, THREADS);
      // the rest of the trailing triangle, columns >= c0 + 16 and rows >= the
      // column: thread t takes columns c0 + 16 + (t & 15) + 16 m of the rows
      // c0 + 16 + (t >> 4) + 14 q (no integer division); each row's panel
      // values are loaded once
      const int cl = t & 15;
      for (int r = c0 + 16 + (t >> 4); r < NB; r += nthr / 16) {
        const float4 a0 = *reinterpret_cast<const float4*>(T + r * LDA + c0);
        const float4 a1 = *reinterpret_cast<const float4*>(T + r * LDA + c0 + 4);
        for (int c = c0 + 16 + cl; c <= r; c += 16) {
          const float4 b0 = *reinterpret_cast<const float4*>(T + c * LDA + c0);
          const float4 b1 = *reinterpret_cast<const float4*>(T + c * LDA + c0 + 4);
          float v = T[r * LDA + c];
          v = fmaf(-a0.x, b0.x, v);
          v = fmaf(-a0.y, b0.y, v);
          v = fmaf(-a0.z, b0.z, v);
          v = fmaf(-a0.w, b0.w, v);
          v = fmaf(-a1.x, b1.x, v);
          v = fmaf(-a1.y, b1.y, v);
          v = fmaf(-a1.z, b1.z, v);
          v = fmaf(-a1.w, b1.w, v);
          T[r * LDA + c] = v;
        }
      }
    }
  }
  __syncthreads();
}

// L_kk from T (zero above the diagonal) into tile (k, k) of the factor and
// inv(L_kk) from X into invdiag, 16 bytes per store.
__device__ __forceinline__ void store_factor_inverse(const DFArgs& a, int k, const float* T, const float* X) {
  float* g = tile<float>(a, k, k);
  float* inv = reinterpret_cast<float*>(a.invdiag) + (size_t)k * NB * NB;
#pragma unroll
  for (int q = 0; q < NB * NB / 4 / THREADS; ++q) {
    const int e = threadIdx.x + q * THREADS, r = e >> 4, c = (e & 15) * 4;
    float4 v = *reinterpret_cast<const float4*>(T + r * LDA + c);
    if (c + 1 > r) v.y = 0.0f;
    if (c + 2 > r) v.z = 0.0f;
    if (c + 3 > r) v.w = 0.0f;
    if (c > r) v.x = 0.0f;
    *reinterpret_cast<float4*>(g + (size_t)r * a.ld + c) = v;
    *reinterpret_cast<float4*>(inv + r * NB + c) = *reinterpret_cast<const float4*>(X + r * LDA + c);
  }
}

// Shared memory of an FP32 factor task: the tile, its inverse, the inversion
// scratch (32 x 36) and 1 / L_jj.
constexpr size_t factor_task_f32_smem_bytes() { return sizeof(float) * (2 * NB * LDA + 32 * 36 + NB); }

// F(k) as a list task of the batched mixed factorisation: the updated tile
// (acc) factored and inverted in FP32 exactly as the FP32 chain does, L_kk
// and inv(L_kk) stored; the caller publishes.  smem is free on entry.
__device__ __forceinline__ void factor_task_f32(const DFArgs& a, int k, const float acc[16], unsigned char* smem) {
  float* T = reinterpret_cast<float*>(smem);
  float* X = T + NB * LDA;
  float* Tm = X + NB * LDA;
  float* Rinv = Tm + 32 * 36;
  acc_to_smem(acc, T);
  __syncthreads();
  factor_tile_f32(a, k, T, Rinv);
  invert_factor<float>(T, Rinv, X, Tm);
  store_factor_inverse(a, k, T, X);
}

// Shared memory of the FP32 chain: five [64][LDA] float tiles (the tile
// being factored, inv(L_kk), the solve's input, the previous solve's
// result, the prefetched next diagonal tile), the inversion scratch
// (32 x 36) and 1 / L_jj.
constexpr size_t chain_f32_smem_bytes() { return sizeof(float) * (5 * NB * LDA + 32 * 36 + NB); }

// The FP32 chain CTA: for k = 0, 1, ...
//   A_kk after its updates by the workers, minus L(k,k-1) L(k,k-1)^T (3xTF32
//   on the tensor cores; L(k,k-1) is still in shared memory);
//   F(k) (factor_tile_f32), inv(L_kk) (FP32, on the FMA pipe) -- L_kk goes to
//   the factor and inv(L_kk) to invdiag, published as fin(k,k) = 2 for the
//   workers' solves (no I(k) tasks in this list);
//   S(k+1,k) = A(k+1,k) inv(L_kk)^T (3xTF32), kept in shared memory for the
//   next step and published as fin(k+1,k) = 1.
// The solve's input is fetched during F(k) when its last update is already
// done, and the next diagonal tile during S(k+1,k) when its worker updates
// are.
__device__ void run_chain_f32(const DFArgs& a, unsigned char* smem, int* s_ok) {
  __shared__ int s_pf[2];  // [0] next diagonal tile fetched, [1] solve input fetched
  float* T = reinterpret_cast<float*>(smem);
  float* X = T + NB * LDA;
  float* Cn = X + NB * LDA;
  float* Lp = Cn + NB * LDA;
  float* sA = Lp + NB * LDA;
  float* Tm = sA + NB * LDA;
  float* Rinv = Tm + 32 * 36;
  const int nt = a.nt;
  bool pf_diag = false;
  for (int k = 0; k < nt; ++k) {
    float acc[16];
    TRACE(0, a.ntasks + 2 * k);
    TRACE(3, a.ntasks + 2 * k);
    CTRACE(k, 7);
    if (k > 0) {
      if (pf_diag) {
        cp_async_wait_all();
        __syncthreads();
        smem_to_acc(sA, acc);
      } else {
        if (!wait_geq(a, a.upd + k * nt + k, k - 1, s_ok)) return;
        load_acc(tile<float>(a, k, k), a.ld, acc);
      }
      TileMMA<float>::sub(Lp, Lp, acc);
    } else {
      load_acc(tile<float>(a, 0, 0), a.ld, acc);
    }
    acc_to_smem(acc, T);
    if (threadIdx.x == 0) s_pf[1] = k + 1 < nt && ld_acquire(a.upd + (k + 1) * nt + k) >= k;
    __syncthreads();
    // thread 0's acquire and the barrier order the early fetch after the updates
    const bool have_in = s_pf[1] != 0;
    if (have_in) stage_async(tile<float>(a, k + 1, k), a.ld, Cn, LDA);
    TRACE(1, a.ntasks + 2 * k);
    CTRACE(k, 0);
    factor_tile_f32(a, k, T, Rinv);
    CTRACE(k, 1);
    invert_factor<float>(T, Rinv, X, Tm);
    CTRACE(k, 2);
    store_factor_inverse(a, k, T, X);
    publish(a.fin + k * nt + k, 2);
    CTRACE(k, 3);
    TRACE(2, a.ntasks + 2 * k);
    if (k + 1 == nt) return;
    TRACE(0, a.ntasks + 2 * k + 1);
    TRACE(3, a.ntasks + 2 * k + 1);
    if (!have_in) {
      if (!wait_geq(a, a.upd + (k + 1) * nt + k, k, s_ok)) return;
      stage_async(tile<float>(a, k + 1, k), a.ld, Cn, LDA);
    }
    if (threadIdx.x == 0) s_pf[0] = ld_acquire(a.upd + (k + 1) * nt + k + 1) >= k;
    cp_async_wait_all();
    __syncthreads();
    pf_diag = s_pf[0] != 0;
    if (pf_diag) stage_async(tile<float>(a, k + 1, k + 1), a.ld, sA, LDA);
    TRACE(1, a.ntasks + 2 * k + 1);
    CTRACE(k, 4);
    solve_by_inverse(Cn, X, acc);
    CTRACE(k, 5);
    acc_to_smem(acc, Lp);
    __syncthreads();
    store_tile(Lp, LDA, tile<float>(a, k + 1, k), a.ld);
    publish(a.fin + (k + 1) * nt + k, 1);
    CTRACE(k, 6);
    TRACE(2, a.ntasks + 2 * k + 1);
  }
}

// Shared memory of the chain CTA: four T tiles Cp, Cn, X, sA ([64][LDA]
// each) and the FP64 factor scratch -- in the FP64 path X holds L_kk from F(k)
// to S(k+1, k); in the mixed path two more FP64 tiles (L_kk, the FP64 rows of
// the solve) come first.  Every piece is a multiple of 16 bytes, so each
// starts 16-byte aligned.
template <typename T>
constexpr size_t chain_smem_bytes() {
  return sizeof(T) * 4 * NB * LDA + (sizeof(T) == 8 ? 0 : sizeof(double) * 2 * NB * LDA) +
         sizeof(double) * factor_smem_elems<double>();
}

// The chain CTA: F(0), S(1, 0), F(1), S(2, 1), ... with L(k, k-1) and the
// FP64 L_kk kept in shared memory from one task to the next.  F(k) does not
// form inv(L_kk) (a worker task I(k) does, for the other solves of column k);
// S(k+1, k) is a blocked forward substitution against L_kk (trsm_rows).  The
// last update of S(k+1, k) (with panel k-1) is a worker task that runs during
// F(k); while S(k+1, k) runs, the next diagonal tile is prefetched into
// shared memory if its updates by the workers are already complete.
template <typename T>
__device__ void run_chain(const DFArgs& a, unsigned char* smem, int* s_ok) {
  __shared__ int s_pf;
  T* Cp = reinterpret_cast<T*>(smem);  // L(k, k-1), the previous solve's result
  T* Cn = Cp + NB * LDA;               // this step's solve input / result L(k+1, k)
  T* X = Cn + NB * LDA;                // FP64 path: L_kk
  T* sA = X + NB * LDA;                // prefetched A_kk
  double* Lk64;  // L_kk in FP64, F(k) to S(k+1, k)
  double* W64;   // FP64 rows of the solve (the mixed path; the FP64 path solves in Cn)
  double* fs64;  // factor scratch; its strip area holds the leaf inverses during S
  if constexpr (sizeof(T) == 8) {
    Lk64 = reinterpret_cast<double*>(X);
    W64 = nullptr;
    fs64 = reinterpret_cast<double*>(sA + NB * LDA);
  } else {
    Lk64 = reinterpret_cast<double*>(sA + NB * LDA);
    W64 = Lk64 + NB * LDA;
    fs64 = W64 + NB * LDA;
  }
  double* Rinv64 = fs64 + 2 * NB * Strip<double>::PB;
  double* XL = fs64;
  __shared__ int s_in;  // A(k+1, k) staged into Cn during F(k)
  const int nt = a.nt;
  bool pf = false;  // A_kk prefetched into sA
  for (int k = 0; k < nt; ++k) {
    T acc[16];
    const SolveInput<T> pre{a.upd + (k + 1) * nt + k, k, tile<T>(a, k + 1, k), a.ld, Cn, &s_in};
    const SolveInput<T>* ppre = k + 1 < nt ? &pre : nullptr;
    // F(k): A_kk after updates 0 .. k-2 (other CTAs), minus L(k,k-1) L(k,k-1)^T
    TRACE(0, a.ntasks + 2 * k);
    TRACE(3, a.ntasks + 2 * k);
    if (k > 0) {
      if (pf) {
        cp_async_wait_all();
        __syncthreads();
        smem_to_acc(sA, acc);
      } else {
        if (!wait_geq(a, a.upd + k * nt + k, k - 1, s_ok)) return;
        load_acc(tile<T>(a, k, k), a.ld, acc);
      }
      TileMMA<T>::sub(Cp, Cp, acc);  // Cp is complete: the last solve ended with a barrier
    } else {
      load_acc(tile<T>(a, 0, 0), a.ld, acc);
    }
    TRACE(1, a.ntasks + 2 * k);
    if constexpr (sizeof(T) == 8) {
      factor_tile<double, double, false>(a, k, acc, fs64, Lk64, nullptr, ppre);
    } else {
      double acc64[16];
#pragma unroll
      for (int rs = 0; rs < 2; ++rs)
#pragma unroll
        for (int cs = 0; cs < 8; ++cs)
          acc64[TileMMA<double>::idx(rs, cs)] = (double)acc[TileMMA<float>::idx(rs, cs)];
      factor_tile<double, float, false>(a, k, acc64, fs64, Lk64, nullptr, ppre);
    }
    publish(a.fin + k * nt + k, 1);
    TRACE(2, a.ntasks + 2 * k);
    if (k + 1 == nt) {
      // the last inverse has no solve task after it: form it here
      double* X64 = sizeof(T) == 8 ? reinterpret_cast<double*>(Cn) : W64;
      store_inverse<double, T>(a, k, Lk64, Rinv64, X64, fs64);
      publish(a.fin + k * nt + k, 2);
      return;
    }
    // S(k+1, k): A(k+1,k) after updates 0 .. k-1 (other CTAs), times inv(L_kk)^T
    TRACE(0, a.ntasks + 2 * k + 1);
    TRACE(3, a.ntasks + 2 * k + 1);
    const bool have_in = s_in != 0;
    if (have_in) cp_async_wait_all();
    if (threadIdx.x == 0) s_pf = ld_acquire(a.upd + (k + 1) * nt + k + 1) >= k;
    leaf_inverses(Lk64, Rinv64, XL);
    if (k > 0 && !have_in) {
      if (!wait_geq(a, a.upd + (k + 1) * nt + k, k, s_ok)) return;
    } else {
      __syncthreads();
    }
    // thread 0's acquire and the barrier order the prefetch after the updates
    pf = s_pf != 0;
    if (pf) stage_async(tile<T>(a, k + 1, k + 1), a.ld, sA, LDA);
    if (!have_in) {
      load_acc(tile<T>(a, k + 1, k), a.ld, acc);
      acc_to_smem(acc, Cn);
    }
    TRACE(1, a.ntasks + 2 * k + 1);
    __syncthreads();  // each warp solves rows that other warps stored
    if constexpr (sizeof(T) == 8) trsm_rows<T>(Lk64, XL, Cn, reinterpret_cast<double*>(Cn));
    else trsm_rows<T>(Lk64, XL, Cn, W64);
    __syncthreads();
    store_tile(Cn, LDA, tile<T>(a, k + 1, k), a.ld);
    publish(a.fin + (k + 1) * nt + k, 1);
    TRACE(2, a.ntasks + 2 * k + 1);
    T* t = Cp;
    Cp = Cn;
    Cn = t;
  }
}

// U(i, j, k) with every tile moved by 16-byte copies: the target tile is
// staged into sC with cp.async together with L_ik, L_jk (instead of per-thread
// 4-byte loads), updated in registers, and written back through sC with
// 16-byte stores.  sC: a third [64][LDA] tile.
template <typename T>
__device__ __forceinline__ void update_tile(const DFArgs& a, int i, int j, int k, T acc[16], T* sA, T* sB, T* sC) {
  stage_async(tile<T>(a, i, k), a.ld, sA, LDA);
  if (i != j) stage_async(tile<T>(a, j, k), a.ld, sB, LDA);
  stage_async(tile<T>(a, i, j), a.ld, sC, LDA);
  cp_async_wait_all();
  __syncthreads();
  smem_to_acc(sC, acc);
  TileMMA<T>::sub(sA, i != j ? sB : sA, acc);
  acc_to_smem(acc, sC);  // each thread rewrites the elements it read
  __syncthreads();
  store_tile(sC, LDA, tile<T>(a, i, j), a.ld);
}

// U(i, j, k) and U(i+1, j, k) together: five tiles (L_ik, L_jk, L_{i+1,k} and
// both targets) staged with 16-byte copies in one round, two accumulators
// against the shared L_jk, one round of 16-byte stores.  s: five [64][LDA]
// T tiles.
template <typename T>
__device__ __forceinline__ void update_tile_pair(const DFArgs& a, int i, int j, int k, T acc[16], T* s) {
  T* sA1 = s;
  T* sB = sA1 + NB * LDA;
  T* sC1 = sB + NB * LDA;
  T* sA2 = sC1 + NB * LDA;
  T* sC2 = sA2 + NB * LDA;
  if (i != j) stage_async(tile<T>(a, i, k), a.ld, sA1, LDA);
  stage_async(tile<T>(a, j, k), a.ld, sB, LDA);
  stage_async(tile<T>(a, i + 1, k), a.ld, sA2, LDA);
  stage_async(tile<T>(a, i, j), a.ld, sC1, LDA);
  stage_async(tile<T>(a, i + 1, j), a.ld, sC2, LDA);
  cp_async_wait_all();
  __syncthreads();
  T acc2[16];
  smem_to_acc(sC1, acc);
  smem_to_acc(sC2, acc2);
  TileMMA<T>::sub(i != j ? sA1 : sB, sB, acc);
  TileMMA<T>::sub(sA2, sB, acc2);
  acc_to_smem(acc, sC1);  // each thread rewrites the elements it read
  acc_to_smem(acc2, sC2);
  __syncthreads();
  store_tile(sC1, LDA, tile<T>(a, i, j), a.ld);
  store_tile(sC2, LDA, tile<T>(a, i + 1, j), a.ld);
}

// ---------------------------------------------------------------- tcgen05 updates
// The FP32 lists' update tasks run on the 5th-generation tensor cores: a task
// U(i .. i+rows-1, j, k) (rows <= 4, sharing L_jk) splits L_jk and the rows'
// L_ik into TF32 hi / lo halves in swizzled shared memory, one thread issues
// P = L_ik L_jk^T as 3xTF32 MMAs (M = 128: two row tiles per MMA, N = 64,
// K = 64) into TMEM accumulators (from zero), and the warps read P back with
// tcgen05.ld and subtract it from C_ij (C -= P once, as the mma.sync
// products do).  Each worker CTA allocates its 128 TMEM columns once.
struct TcWorker {
  uint64_t* mbar;       // MMA completion (one phase per task)
  uint32_t tmem;        // TMEM base: one accumulator of 64 columns per row pair
  uint32_t phase;
  int max_pairs;        // row pairs per task: 2 (single matrix) or 1 (batch)
  unsigned char* base;  // 1024-byte aligned operand area
};
constexpr uint32_t TC_A_BYTES = tc::operand_bytes(128);  // one M = 128 operand half (hi or lo)
constexpr uint32_t TC_B_BYTES = tc::operand_bytes(64);
// A hi, A lo (max_pairs row pairs each), B hi, B lo, and the alignment slack
constexpr size_t tc_worker_smem_bytes(int max_pairs) { return 2 * max_pairs * TC_A_BYTES + 2 * TC_B_BYTES + 1024; }
// TMEM columns: a power of two >= 32
__host__ __device__ constexpr uint32_t tc_cols(int max_pairs) { return max_pairs > 1 ? 128u : 64u; }

__device__ __forceinline__ void tc_worker_begin(uint64_t* mbar, uint32_t* s_tmem, unsigned char* smem, int max_pairs,
                                                TcWorker& w) {
  if (threadIdx.x == 0) tc::mbar_init(mbar, 1);
  if (threadIdx.x < 32) tc::tmem_alloc(s_tmem, tc_cols(max_pairs));
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  w.mbar = mbar;
  w.tmem = *s_tmem;
  w.phase = 0;
  w.max_pairs = max_pairs;
  w.base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem) + 1023) & ~uintptr_t(1023));
}

__device__ __forceinline__ void tc_worker_end(const TcWorker& w) {
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(w.tmem, tc_cols(w.max_pairs));
}

// U(i + r, j, k) for r < rows (rows <= 2 max_pairs) on the tensor cores (the
// dependencies are met).  Returns false if the MMAs did not complete within
// the spin limit (the run is then aborted like an expired flag wait).
__device__ bool update_rows_tc(const DFArgs& a, int i, int rows, int j, int k, TcWorker& w) {
  unsigned char* Ahi = w.base;
  unsigned char* Alo = Ahi + w.max_pairs * TC_A_BYTES;
  unsigned char* Bhi = Alo + w.max_pairs * TC_A_BYTES;
  unsigned char* Blo = Bhi + TC_B_BYTES;
  const int pairs = (rows + 1) >> 1;
  {
    // L_jk and the rows' L_ik, all loads in flight together
    tc::SplitTile t[5];
    t[0] = tc::SplitTile{tile<float>(a, j, k), 64, 0, Bhi, Blo};
#pragma unroll
    for (int r = 0; r < 4; ++r)
      t[1 + r] = tc::SplitTile{tile<float>(a, i + (r < rows ? r : 0), k), 128, 64 * (r & 1),
                               Ahi + (r >> 1) * TC_A_BYTES, Alo + (r >> 1) * TC_A_BYTES};
    tc::split_tiles_all<THREADS, 5>(t, 1 + rows, a.ld);
  }
  tc::fence_proxy_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    for (int p = 0; p < pairs; ++p)
      tc::issue_product(w.tmem + 64 * p, tc::smem_u32(Ahi + p * TC_A_BYTES), tc::smem_u32(Alo + p * TC_A_BYTES),
                        tc::smem_u32(Bhi), tc::smem_u32(Blo));
    tc::mma_commit(w.mbar);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = warp & 3, g = warp >> 2;
  const int m = 32 * q + lane;  // accumulator row = TMEM lane
  const int p = pairs == 2 ? g : 0;
  const int c0 = pairs == 2 ? 0 : 32 * g;
  const int nh = pairs == 2 ? 2 : 1;  // 32-column halves this warp reads
  const int rr = 2 * p + (m >> 6);    // row tile in the group (warp-uniform)
  bool ok = tc::mbar_wait(w.mbar, w.phase, a.spin_limit);
  if (!ok) tc::mbar_wait(w.mbar, w.phase, a.spin_limit);  // the MMAs must not outlive the TMEM
  ok = __syncthreads_and(ok) != 0;                          // one verdict for the whole CTA
  if (!ok && threadIdx.x == 0) {
    atomicExch(a.ctl + 1, 1);
    atomicOr(a.err, PBG_DEV_ERR_BARRIER);
    atomicCAS(a.info, 0, -1);
  }
  w.phase ^= 1;
  tc::fence_after_sync();
  // P from TMEM into shared memory, row-major [rows * 64][LDA] over the A
  // operands (the MMAs that read them are complete) ...
  float* Ps = reinterpret_cast<float*>(w.base);
  if (ok && rr < rows) {
    for (int h = 0; h < nh; ++h) {
      float v[32];
      tc::tmem_ld32(w.tmem + ((uint32_t)(32 * q) << 16) + 64 * p + c0 + 32 * h, v);
      float* dst = Ps + (size_t)(64 * rr + (m & 63)) * LDA + c0 + 32 * h;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        *reinterpret_cast<float4*>(dst + 4 * u) = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
    }
  }
  __syncthreads();
  // ... then C -= P with coalesced 16-byte accesses (a row of 64 per 16 threads)
  if (ok)
    for (int e = threadIdx.x; e < rows * NB * 16; e += THREADS) {
      const int row = e >> 4, c4 = e & 15;
      float4* gp = reinterpret_cast<float4*>(tile<float>(a, i + (row >> 6), j) + (size_t)(row & 63) * a.ld) + c4;
      float4 cv = __ldcg(gp);
      const float4 pv = *reinterpret_cast<const float4*>(Ps + (size_t)row * LDA + 4 * c4);
      cv.x -= pv.x;
      cv.y -= pv.y;
      cv.z -= pv.z;
      cv.w -= pv.w;
      *gp = cv;
    }
  tc::fence_before_sync();
  __syncthreads();
  return ok;
}

// ---------------------------------------------------------------- inv(L) in the task list
// With DFArgs::X set, the factorisation's task list also forms X = inv(L)
// (its off-diagonal tiles; the diagonal ones are the inv(L_kk) in invdiag),
// right-looking over the columns of L:
//   X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj    (i > j),
// accumulated as V_ij = -sum_k L_ik X_kj in X's own tile (i, j), in k order:
//   XG(i, j, k), j <= k <= i-2: V_ij -= L_ik X_kj for rows i and i+1 (they
//     share X_kj); needs L_ik final, X_kj final and the k - j earlier terms;
//   XZ(i, j): V_ij -= L_{i,i-1} X_{i-1,j}, then X_ij = X_ii V_ij; needs
//     L_{i,i-1}, X_{i-1,j}, inv(L_ii) (fin(i,i) = 2) and the earlier terms.
// xupd(i, j) counts the applied terms, xfin(i, j) = 1 marks X_ij final.  The
// list places XZ(k+1, .) and XG(., ., k) right after panel k's block, after
// every task (or chain step) they depend on.  Tiles written in this kernel
// are read through L2 (.cg loads, cp.async.cg).

template <typename T>
__device__ __forceinline__ const T* xtile(const DFArgs& a, int k, int j) {
  return k == j ? reinterpret_cast<const T*>(a.invdiag) + (size_t)j * NB * NB
                : reinterpret_cast<const T*>(a.X) + (size_t)k * NB * a.ld + (size_t)j * NB;
}
template <typename T>
__device__ __forceinline__ T* xtile_out(const DFArgs& a, int i, int j) {
  return reinterpret_cast<T*>(a.X) + (size_t)i * NB * a.ld + (size_t)j * NB;
}

// s[c][r] = g[r][c] through L2, all of a thread's loads in flight first.
template <typename T>
__device__ __forceinline__ void stage_transposed_cg(const T* g, int ld, T* s) {
  T v[TILE_PER_THREAD];
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) {
    const int e = threadIdx.x + q * THREADS;
    v[q] = ldcg(g + (size_t)(e >> 6) * ld + (e & 63));
  }
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) {
    const int e = threadIdx.x + q * THREADS;
    s[(e & 63) * LDA + (e >> 6)] = v[q];
  }
}

template <typename T>
__device__ __forceinline__ void acc_to_smem_transposed(const T acc[16], T* s) {
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) s[acc_col(cs) * LDA + acc_row(rs)] = acc[TileMMA<T>::idx(rs, cs)];
}

// XG(i, j, k) for rows i .. i+rows-1 (rows <= 2).  Shared memory: three tiles.
template <typename T>
__device__ void inverse_update(const DFArgs& a, int i, int rows, int j, int k, T* s) {
  T* sB = s;
  T* sA0 = s + NB * LDA;
  T* sA1 = s + 2 * NB * LDA;
  stage_async(tile<T>(a, i, k), a.ld, sA0, LDA);
  if (rows > 1) stage_async(tile<T>(a, i + 1, k), a.ld, sA1, LDA);
  T acc0[16], acc1[16];
  if (k > j) {
    load_acc(xtile_out<T>(a, i, j), a.ld, acc0);
    if (rows > 1) load_acc(xtile_out<T>(a, i + 1, j), a.ld, acc1);
  } else {
#pragma unroll
    for (int e = 0; e < 16; ++e) acc0[e] = acc1[e] = T(0);
  }
  stage_transposed_cg<T>(xtile<T>(a, k, j), k == j ? NB : a.ld, sB);  // X_kj^T
  cp_async_wait_all();
  __syncthreads();
  TileMMA<T>::sub(sA0, sB, acc0);
  if (rows > 1) TileMMA<T>::sub(sA1, sB, acc1);
  store_acc(xtile_out<T>(a, i, j), a.ld, acc0);
  if (rows > 1) store_acc(xtile_out<T>(a, i + 1, j), a.ld, acc1);
}

// XZ(i, j).  Shared memory: three tiles.
template <typename T>
__device__ void inverse_finish(const DFArgs& a, int i, int j, T* s) {
  T* sB = s;
  T* sA = s + NB * LDA;
  T* sX = s + 2 * NB * LDA;
  stage_async(tile<T>(a, i, i - 1), a.ld, sA, LDA);
  stage_async(reinterpret_cast<const T*>(a.invdiag) + (size_t)i * NB * NB, NB, sX, LDA);  // X_ii
  T acc[16];
  if (i - 1 > j) {
    load_acc(xtile_out<T>(a, i, j), a.ld, acc);
  } else {
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = T(0);
  }
  stage_transposed_cg<T>(xtile<T>(a, i - 1, j), i - 1 == j ? NB : a.ld, sB);  // X_{i-1,j}^T
  cp_async_wait_all();
  __syncthreads();
  TileMMA<T>::sub(sA, sB, acc);  // V_ij complete
  __syncthreads();
  acc_to_smem_transposed(acc, sB);  // V^T
  __syncthreads();
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = T(0);
  TileMMA<T>::sub(sX, sB, acc);  // -X_ii V
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = -acc[e];
  store_acc(xtile_out<T>(a, i, j), a.ld, acc);
}

// The worker CTAs' task loop.  FP32 lists (T = float): every update task
// (one to four rows) runs on the tcgen05 tensor cores (update_rows_tc, w
// holds the CTA's TMEM); FP64 lists: DMMA tile products.
template <typename T>
__device__ void df_worker_loop(const DFArgs& a, unsigned char* smem, int* s_task_p, int* s_ok_p, TcWorker* w) {
  int& s_task = *s_task_p;
  int& s_ok = *s_ok_p;
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + NB * LDA;
  const int nt = a.nt;
  while (true) {
    if (threadIdx.x == 0) s_task = ld_acquire(a.ctl + 1) ? a.ntasks : atomicAdd(a.ctl, 1);
    __syncthreads();
    const int t = s_task;
    __syncthreads();
    if (t >= a.ntasks) return;
    const int4 tk = a.tasks[t];
    const int type = tk.x, i = tk.y, j = tk.z, k = tk.w;
    TRACE(0, t);
    TRACE(3, t);
    T acc[16];
    if (sizeof(T) == 4 && (type == TASK_U || type == TASK_U2 || type == TASK_U3 || type == TASK_U4)) {
      // U(i + r, j, k), r < rows: L_(i+r)k, L_jk final and the k previous updates of each (i + r, j)
      const int rows = type == TASK_U ? 1 : type == TASK_U2 ? 2 : type == TASK_U3 ? 3 : 4;
      const int* fl[9];
      int tg[9];
      fl[0] = a.fin + j * nt + k;
      tg[0] = 1;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int rr = r < rows ? r : 0;
        fl[1 + 2 * r] = a.fin + (i + rr) * nt + k;
        tg[1 + 2 * r] = 1;
        fl[2 + 2 * r] = a.upd + (i + rr) * nt + j;
        tg[2 + 2 * r] = k;
      }
      if (!wait_all(a, fl, tg, 1 + 2 * rows, &s_ok)) return;
      TRACE(1, t);
      if (!update_rows_tc(a, i, rows, j, k, *w)) return;
      if (threadIdx.x < rows) st_release(a.upd + (i + threadIdx.x) * nt + j, k + 1);
      TRACE(2, t);
    } else if (type == TASK_XG) {
      const int rows = i + 1 < nt ? 2 : 1;
      const int* fl[5] = {k == j ? a.fin + j * nt + j : a.xfin + k * nt + j, a.fin + i * nt + k,
                          a.xupd + i * nt + j, a.fin + (i + rows - 1) * nt + k, a.xupd + (i + rows - 1) * nt + j};
      const int tg[5] = {k == j ? 2 : 1, 1, k - j, 1, k - j};
      if (!wait_all(a, fl, tg, 5, &s_ok)) return;
      TRACE(1, t);
      inverse_update<T>(a, i, rows, j, k, sA);
      __syncthreads();
      if (threadIdx.x < rows) st_release(a.xupd + (i + threadIdx.x) * nt + j, k - j + 1);
      TRACE(2, t);
    } else if (type == TASK_XZ) {
      const int* fl[4] = {a.fin + i * nt + i - 1, i - 1 == j ? a.fin + j * nt + j : a.xfin + (i - 1) * nt + j,
                          a.fin + i * nt + i, a.xupd + i * nt + j};
      const int tg[4] = {1, i - 1 == j ? 2 : 1, 2, i - 1 - j};
      if (!wait_all(a, fl, tg, 4, &s_ok)) return;
      TRACE(1, t);
      inverse_finish<T>(a, i, j, sA);
      publish(a.xfin + i * nt + j, 1);
      TRACE(2, t);
    } else if (type == TASK_I) {
      // I(k): inv(L_kk) for the solves of column k, from the stored L_kk
      if (!wait_geq(a, a.fin + k * nt + k, 1, &s_ok)) return;
      TRACE(1, t);
      double* Lk = reinterpret_cast<double*>(smem);
      double* Xw = Lk + NB * LDA;
      double* Tm = Xw + NB * LDA;
      double* Rv = Tm + 32 * 36;
      const T* g = tile<T>(a, k, k);
      T v[TILE_PER_THREAD];  // all loads in flight before the first store
#pragma unroll
      for (int q = 0; q < TILE_PER_THREAD; ++q) {
        const int e = threadIdx.x + q * THREADS;
        v[q] = ldcg(g + (size_t)(e >> 6) * a.ld + (e & 63));
      }
#pragma unroll
      for (int q = 0; q < TILE_PER_THREAD; ++q) {
        const int e = threadIdx.x + q * THREADS, r = e >> 6, c = e & 63;
        Lk[r * LDA + c] = c <= r ? (double)v[q] : 0.0;
      }
      __syncthreads();
      if (threadIdx.x < NB) Rv[threadIdx.x] = 1.0 / Lk[threadIdx.x * LDA + threadIdx.x];
      __syncthreads();
      store_inverse<double, T>(a, k, Lk, Rv, Xw, Tm);
      publish(a.fin + k * nt + k, 2);
      TRACE(2, t);
    } else if (type == TASK_U) {
      // U(i, j, k): needs L_ik, L_jk final and the k previous updates of (i, j)
      const int* fl[3] = {a.fin + i * nt + k, a.fin + j * nt + k, a.upd + i * nt + j};
      const int tg[3] = {1, 1, k};
      if (!wait_all(a, fl, tg, 3, &s_ok)) return;
      TRACE(1, t);
      update_tile(a, i, j, k, acc, sA, sB, sB + NB * LDA);
      publish(a.upd + i * nt + j, k + 1);
      TRACE(2, t);
    } else if (type == TASK_U2) {
      // U(i, j, k) and U(i+1, j, k): L_ik, L_{i+1,k}, L_jk final, k previous updates of both
      const int* fl[5] = {a.fin + i * nt + k, a.fin + (i + 1) * nt + k, a.fin + j * nt + k, a.upd + i * nt + j,
                          a.upd + (i + 1) * nt + j};
      const int tg[5] = {1, 1, 1, k, k};
      if (!wait_all(a, fl, tg, 5, &s_ok)) return;
      TRACE(1, t);
      update_tile_pair(a, i, j, k, acc, sA);
      __syncthreads();
      if (threadIdx.x == 0) {
        st_release(a.upd + i * nt + j, k + 1);
        st_release(a.upd + (i + 1) * nt + j, k + 1);
      }
      TRACE(2, t);
    } else {
      // S(i, j), i >= j + 2: the tile after its last update, times inv(L_jj)^T
      const int col = j;
      if (col > 0) {
        const int* fl[3] = {a.fin + i * nt + col - 1, a.fin + col * nt + col - 1, a.upd + i * nt + col};
        const int tg[3] = {1, 1, col - 1};
        if (!wait_all(a, fl, tg, 3, &s_ok)) return;
        load_and_update(a, i, col, col - 1, acc, sA, sB);  // ends with a barrier: smem is free
      } else {
        load_acc(tile<T>(a, i, col), a.ld, acc);
      }
      if (!wait_geq(a, a.fin + col * nt + col, 2, &s_ok)) return;  // inv(L_col,col) stored
      TRACE(1, t);
      stage_async(reinterpret_cast<const T*>(a.invdiag) + (size_t)col * NB * NB, NB, sB, LDA);
      acc_to_smem(acc, sA);
      cp_async_wait_all();
      __syncthreads();
      solve_by_inverse(sA, sB, acc);
      store_acc(tile<T>(a, i, col), a.ld, acc);
      publish(a.fin + i * nt + col, 1);
      TRACE(2, t);
    }
    __syncthreads();
  }
}

// F32CHAIN (FP32 matrices only): the chain CTA runs the FP32 chain
// (run_chain_f32) and the task list has no I(k) tasks; otherwise run_chain,
// whose diagonal tiles are factored in FP64.  The FP32 workers hold TMEM for
// their tensor-core updates from start to end.
template <typename T, bool F32CHAIN>
__global__ void __launch_bounds__(THREADS, 1) chol_df_kernel(DFArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_task, s_ok;
  if (blockIdx.x == 0) {
    if constexpr (F32CHAIN) run_chain_f32(a, smem, &s_ok);
    else run_chain<T>(a, smem, &s_ok);
    return;
  }
  if constexpr (sizeof(T) == 4) {
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_tmem;
    TcWorker w;
    tc_worker_begin(&s_mbar, &s_tmem, smem, 2, w);
    df_worker_loop<T>(a, smem, &s_task, &s_ok, &w);
    tc_worker_end(w);
  } else {
    df_worker_loop<T>(a, smem, &s_task, &s_ok, nullptr);
  }
}

// Batched FP64 factorisation (right-looking; the mixed batch runs the
// left-looking chol_batch_ll_kernel below): every task comes from the shared
// list (there is no chain CTA); F(k) applies its last update itself.  Shared
// memory: two tiles (sA, sB) for the updates and solves; F uses two tiles
// (L_kk, inverse) over the same bytes and the factor scratch after them.
constexpr size_t batch_smem_bytes() {
  // an F task's factor scratch, or a paired update's five tiles
  return std::max(sizeof(double) * (2 * NB * LDA + factor_smem_elems<double>()), 5 * NB * LDA * sizeof(double));
}

// The FP64 batched kernel's task loop: DMMA updates in pairs (five tiles
// staged in one round, the loads overlapped with the math inside the CTA).
template <typename T>
__device__ void batch_worker_loop(const CholRep* __restrict__ reps, const int4* __restrict__ tasks, int ntasks,
                                  int* ctl, unsigned char* smem) {
  __shared__ int s_task, s_ok;
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + NB * LDA;
  double* Lk64 = reinterpret_cast<double*>(smem);
  double* X64 = Lk64 + NB * LDA;
  double* fs64 = X64 + NB * LDA;
  while (true) {
    if (threadIdx.x == 0) s_task = ld_acquire(ctl + 1) ? ntasks : atomicAdd(ctl, 1);
    __syncthreads();
    const int t = s_task;
    __syncthreads();
    if (t >= ntasks) return;
    const int4 tk = tasks[t];
    const int type = tk.x & 7, i = tk.y, j = tk.z, k = tk.w;
    const CholRep& R = reps[tk.x >> 3];
    DFArgs a;
    a.A = R.A;
    a.ld = R.ld;
    a.n = R.n;
    a.nt = R.nt;
    a.ntasks = ntasks;
    a.tasks = tasks;
    a.ctl = ctl;
    a.upd = R.upd;
    a.fin = R.fin;
    a.info = R.info;
    a.invdiag = R.invdiag;
    a.err = reinterpret_cast<unsigned*>(ctl + 3);
    a.spin_limit = SPIN_LIMIT;
    const int nt = a.nt;
    T acc[16];
    if (type == TASK_U) {
      const int* fl[3] = {a.fin + i * nt + k, a.fin + j * nt + k, a.upd + i * nt + j};
      const int tg[3] = {1, 1, k};
      if (!wait_all(a, fl, tg, 3, &s_ok)) return;
      load_and_update(a, i, j, k, acc, sA, sB);
      store_acc(tile<T>(a, i, j), a.ld, acc);
      publish(a.upd + i * nt + j, k + 1);
    } else if (type == TASK_U2) {
      const int* fl[5] = {a.fin + i * nt + k, a.fin + (i + 1) * nt + k, a.fin + j * nt + k, a.upd + i * nt + j,
                          a.upd + (i + 1) * nt + j};
      const int tg[5] = {1, 1, 1, k, k};
      if (!wait_all(a, fl, tg, 5, &s_ok)) return;
      update_tile_pair(a, i, j, k, acc, sA);
      __syncthreads();
      if (threadIdx.x == 0) {
        st_release(a.upd + i * nt + j, k + 1);
        st_release(a.upd + (i + 1) * nt + j, k + 1);
      }
    } else {
      const int col = j;
      if (col > 0) {
        const int* fl[3] = {a.fin + i * nt + col - 1, a.fin + col * nt + col - 1, a.upd + i * nt + col};
        const int tg[3] = {1, 1, col - 1};
        if (!wait_all(a, fl, tg, 3, &s_ok)) return;
        load_and_update(a, i, col, col - 1, acc, sA, sB);  // ends with a barrier: smem is free
      } else {
        load_acc(tile<T>(a, i, col), a.ld, acc);
      }
      if (type == TASK_F) {
        factor_tile<double>(a, col, acc, fs64, Lk64, X64);
      } else {
        if (!wait_geq(a, a.fin + col * nt + col, 1, &s_ok)) return;
        stage_async(reinterpret_cast<const T*>(a.invdiag) + (size_t)col * NB * NB, NB, sB, LDA);
        acc_to_smem(acc, sA);
        cp_async_wait_all();
        __syncthreads();
        solve_by_inverse(sA, sB, acc);
        store_acc(tile<T>(a, i, col), a.ld, acc);
      }
      publish(a.fin + i * nt + col, 1);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(THREADS, 1) chol_batch_kernel(const CholRep* __restrict__ reps,
                                                                 const int4* __restrict__ tasks, int ntasks,
                                                                 int* ctl) {
  static_assert(sizeof(T) == 8, "the mixed batch runs chol_batch_ll_kernel");
  extern __shared__ __align__(16) unsigned char smem[];
  batch_worker_loop<T>(reps, tasks, ntasks, ctl, smem);
}

// ---------------------------------------------------------------- left-looking batched factorisation
// The mixed batch factors every replica left-looking on the tcgen05 tensor
// cores.  A task owns the row tiles i and i + 1 of column j of L (only i
// when i + 1 = nt) and forms
//   U_rj = A_rj - sum_{k < j} L_rk L_jk^T        (r = i, i + 1)
// as one M = 128, N = 64, K = 64 j product accumulated in TMEM: for each k
// the tiles L_ik, L_{i+1,k}, L_jk are split into TF32 hi / lo halves in
// shared memory and three MMAs per K-step add A_hi B_hi + A_hi B_lo + A_lo
// B_hi to the accumulator, while the tiles of k + 1 and k + 2 are on their
// way (cp.async into two raw FP32 stages).  Then, by the task's kind:
//   LL_DIAG (i = j): F(j) -- L_jj and inv(L_jj) in FP32, as the FP32 chain
//     forms them -- published at once, then S(j + 1, j) = U inv(L_jj)^T with
//     the inverse still in shared memory;
//   LL_UPDATE (i > j): U written over A's tiles, upd[r] = j + 1;
//   LL_SOLVE (i > j, a later segment): S(i, j), S(i + 1, j) from the stored
//     U once F(j) is published.
// Every tile is read as A once and written twice (U, then L), where a
// right-looking update reads and writes its tile once per panel.  Flags:
// fin[r] = the number of final tiles of row r, upd[r] = the columns of row r
// whose U is stored.  A row's tiles become final in column order (tile
// (r, j) needs (r, j - 1)), so one counter per row says which L_rk are
// ready.  Every task depends only on earlier tasks of the list.
constexpr uint32_t LL_A_BYTES = tc::operand_bytes(128);
constexpr uint32_t LL_B_BYTES = tc::operand_bytes(64);
constexpr uint32_t LL_OPERAND_BYTES = 2 * LL_A_BYTES + 2 * LL_B_BYTES;
// The operands (from the 1024-byte aligned start of dynamic shared memory),
// two raw FP32 stages of a K-step's tiles, then the worker's words
// (LLShared).  After the last product the operand bytes hold P ([128][LDA]
// floats from 0), the U tiles ([64][LDA] at LL_U0 and LL_U1) and the factor
// scratch (from 0).
struct LLShared {
  uint64_t mbar, conv;
  uint32_t tmem;
  int task, ok, seen[3];
};
constexpr uint32_t LL_RAW_BYTES = 3 * NB * NB * sizeof(float);  // one raw stage: L_ik, L_{i+1,k}, L_jk
constexpr uint32_t LL_SHARED_OFFSET = LL_OPERAND_BYTES + 2 * LL_RAW_BYTES;
constexpr size_t ll_smem_bytes() { return LL_SHARED_OFFSET + sizeof(LLShared); }
static_assert(ll_smem_bytes() <= 227 * 1024, "the worker does not fit an SM");
// task kinds of the left-looking list
enum : int { LL_DIAG = 0, LL_UPDATE = 1, LL_SOLVE = 2 };
// K-steps (of 64) accumulated in TMEM before the sum is added in FP32
constexpr int LL_CHUNK = 4;
constexpr uint32_t LL_U0 = 40960, LL_U1 = 61440;
static_assert(factor_task_f32_smem_bytes() <= LL_U0, "the factor scratch overlaps U0");
static_assert(sizeof(float) * 128 * LDA <= LL_U0, "P overlaps U0");
static_assert(LL_U1 + sizeof(float) * NB * LDA <= LL_OPERAND_BYTES, "U1 lies outside the operand bytes");

struct LLWorker {
  uint64_t* mbar;       // completion of the products of one K-step
  uint64_t* conv;       // every thread's operands of a K-step written (THREADS arrivals)
  uint32_t tmem;        // TMEM base: the 128 x 64 FP32 accumulator
  uint32_t phase;
  uint32_t conv_phase;  // thread 0's
  unsigned char* base;  // 1024-byte aligned operand area
};

__device__ __forceinline__ DFArgs batch_args(const CholRep& R, const int4* tasks, int ntasks, int* ctl) {
  DFArgs a;
  a.A = R.A;
  a.ld = R.ld;
  a.n = R.n;
  a.nt = R.nt;
  a.ntasks = ntasks;
  a.tasks = tasks;
  a.ctl = ctl;
  a.upd = R.upd;
  a.fin = R.fin;
  a.info = R.info;
  a.invdiag = R.invdiag;
  a.err = reinterpret_cast<unsigned*>(ctl + 3);
  a.spin_limit = SPIN_LIMIT;
  a.X = nullptr;
  a.xupd = nullptr;
  a.xfin = nullptr;
  return a;
}

// Warp 0 waits until base[rows[q]] >= target for every slot q in mask
// (bounded, with the abort polling of wait_all).  seen[q] (touched by warp 0
// only) keeps the largest count observed for slot q in this task, so a wait
// that an earlier observation already satisfies costs no memory round trip.
// *s_ok only ever goes from 1 to 0.  Ends with a CTA barrier.
__device__ bool ll_wait_rows(const DFArgs& a, const int* base, const int (&rows)[3], unsigned mask, int target,
                             int* seen, int* s_ok) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const bool mine = lane < 3 && ((mask >> lane) & 1u);
    const int* flag = mine ? base + rows[lane < 3 ? lane : 0] : nullptr;
    bool done = !mine || seen[lane] >= target;
    bool ok = true;
    for (long long it = 0;; ++it) {
      if (!done) {
        const int v = ld_acquire(flag);
        if (v >= target) {
          seen[lane] = v;
          done = true;
        }
      }
      if (__all_sync(0xffffffffu, done)) break;
      if ((it & 15) == 15) {
        const int ab = __shfl_sync(0xffffffffu, lane == 0 ? ld_acquire(a.ctl + 1) : 0, 0);
        if (ab) {
          ok = false;
          break;
        }
      }
      if (it + 1 > a.spin_limit) {
        if (lane == 0) {
          atomicExch(a.ctl + 1, 1);
          atomicAdd(a.ctl + 2, 1);
          atomicOr(a.err, PBG_DEV_ERR_BARRIER);
          atomicCAS(a.info, 0, -1);
        }
        ok = false;
        break;
      }
      if (it > 256) __nanosleep(200);
    }
    if (lane == 0 && !ok) *s_ok = 0;
  }
  __syncthreads();
  return *s_ok != 0;
}


// cp.async (16 bytes, through L2) of this thread's share of a 64 x 64 FP32
// tile into a row-major [64][64] stage; the same thread converts the same
// chunks later, so its own wait_group makes them visible to it.
__device__ __forceinline__ void ll_fetch_tile(const float* src, int ld, float* raw) {
#pragma unroll
  for (int e = 0; e < tc::TileShare<THREADS>::PER; ++e) {
    const int q = threadIdx.x + e * THREADS, r = q >> 4, c = q & 15;
    cp_async16(raw + r * NB + 4 * c, src + (size_t)r * ld + 4 * c);
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The tiles of K-step k (L_ik, L_{i+1,k}, L_jk) into a raw stage, one group.
__device__ __forceinline__ void ll_fetch_step(const DFArgs& a, int i, bool two, int j, int k, float* raw) {
  ll_fetch_tile(tile<float>(a, i, k), a.ld, raw);
  if (two) ll_fetch_tile(tile<float>(a, i + 1, k), a.ld, raw + NB * NB);
  ll_fetch_tile(tile<float>(a, j, k), a.ld, raw + 2 * NB * NB);
  cp_async_commit();
}

// This thread's share of a raw stage tile, back into registers.
__device__ __forceinline__ void ll_share_from_raw(const float* raw, tc::TileShare<THREADS>& s) {
#pragma unroll
  for (int e = 0; e < tc::TileShare<THREADS>::PER; ++e) {
    const int q = threadIdx.x + e * THREADS, r = q >> 4, c = q & 15;
    s.v[e] = *reinterpret_cast<const float4*>(raw + r * NB + 4 * c);
  }
}

// Per-thread bounded wait until base[rows[q]] >= target for q = 0, 1, 2,
// with the counts observed so far kept in the thread's registers (seen): a
// wait that an earlier observation satisfies costs nothing, and the thread's
// own acquire orders its later reads (no barrier).  false: the wait gave up
// (recorded like an expired wait_all) or the run was aborted.
__device__ bool ll_thread_wait_rows(const DFArgs& a, const int* base, const int (&rows)[3], int target,
                                    int (&seen)[3]) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    for (long long it = 0; seen[q] < target; ++it) {
      const int v = ld_acquire(base + rows[q]);
      if (v >= target) {
        seen[q] = v;
        break;
      }
      if ((it & 63) == 63) {
        if (ld_acquire(a.ctl + 1)) return false;
        if (it > a.spin_limit) {
          atomicExch(a.ctl + 1, 1);
          atomicAdd(a.ctl + 2, 1);
          atomicOr(a.err, PBG_DEV_ERR_BARRIER);
          atomicCAS(a.info, 0, -1);
          return false;
        }
        __nanosleep(64);
      }
    }
  }
  return true;
}

__device__ __forceinline__ void ll_arrive(uint64_t* m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(m)) : "memory");
}

// P = sum_{k < j} [L_ik; L_{i+1,k}] L_jk^T into shared memory ([128][LDA]
// floats at the operand area's start), for j > 0.  The tiles of K-step k + 2
// are fetched (cp.async, two raw stages) while the products of k run.  No
// CTA barrier inside the K loop: every thread fetches and converts only its
// own chunks (so the raw stages need no hand-over), waits for the previous
// products on their mbarrier before overwriting the operands, and arrives on
// the conversion mbarrier; thread 0 waits for all arrivals and issues the
// MMAs.  Returns false (after a CTA barrier) if the run was aborted, with no
// products of this CTA left in flight.
__device__ bool ll_products(const DFArgs& a, int i, int j, LLWorker& w) {
  const int tid = threadIdx.x;
  const bool two = i + 1 < a.nt;
  unsigned char* Ahi = w.base;
  unsigned char* Alo = Ahi + LL_A_BYTES;
  unsigned char* Bhi = Alo + LL_A_BYTES;
  unsigned char* Blo = Bhi + LL_B_BYTES;
  float* raw[2] = {reinterpret_cast<float*>(w.base + LL_OPERAND_BYTES),
                   reinterpret_cast<float*>(w.base + LL_OPERAND_BYTES + LL_RAW_BYTES)};
  const int rows[3] = {i, two ? i + 1 : i, j};
  int seen[3] = {0, 0, 0};
  if (!two) {
    // rows 64 .. 127 of both A halves stay zero for the whole task: bytes
    // 8192 .. 16383 of each of the two K blocks (16384 bytes each)
    for (int e = tid; e < 4 * 512; e += THREADS) {
      const int part = e >> 9, off = (e & 511) * 16;
      unsigned char* p = (part & 1 ? Alo : Ahi) + (part >> 1) * 16384 + 8192 + off;
      *reinterpret_cast<uint4*>(p) = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  long long c0 = LLCLK();
  bool ok = ll_thread_wait_rows(a, a.fin, rows, 1, seen);
  if (ok) ll_fetch_step(a, i, two, j, 0, raw[0]);
  else cp_async_commit();
  if (j > 1) {
    ok = ok && ll_thread_wait_rows(a, a.fin, rows, 2, seen);
    if (ok) ll_fetch_step(a, i, two, j, 1, raw[1]);
    else cp_async_commit();
  }
  LLPROF(2, LLCLK() - c0);
  // the products accumulate in TMEM for LL_CHUNK K-steps at a time; each
  // chunk's sum is then added in FP32 to racc (this thread's row m, columns
  // 32 g .. 32 g + 31), so no accumulation runs longer than K = 64 LL_CHUNK
  // in the tensor cores
  const int warp = tid >> 5, lane = tid & 31, q = warp & 3, g = warp >> 2;
  const int m = 32 * q + lane;
  const uint32_t tacc = w.tmem + ((uint32_t)(32 * q) << 16) + 32 * g;
  float racc[32];
#pragma unroll
  for (int u = 0; u < 32; ++u) racc[u] = 0.0f;
  for (int k = 0; k < j; ++k) {
    float* st = raw[k & 1];
    c0 = LLCLK();
    if (k + 1 < j) cp_async_wait_group<1>();
    else cp_async_wait_group<0>();
    if (k > 0) {  // the products of k - 1 have read the operands
      if (!tc::mbar_wait(w.mbar, w.phase, a.spin_limit)) ok = false;
      w.phase ^= 1;
      tc::fence_after_sync();
      if (k % LL_CHUNK == 0) {
        // a chunk is complete: fold it into racc before the next product
        // starts the accumulator from zero (ordered by the conversion mbarrier)
        float v[32];
        tc::tmem_ld32(tacc, v);
#pragma unroll
        for (int u = 0; u < 32; ++u) racc[u] += v[u];
        tc::fence_before_sync();
      }
    }
    const long long c1 = LLCLK();
    LLPROF(3, c1 - c0);
    {
      tc::TileShare<THREADS> s;
      ll_share_from_raw(st, s);
      tc::store_share_split<THREADS>(s, 128, 0, Ahi, Alo);
      if (two) {
        ll_share_from_raw(st + NB * NB, s);
        tc::store_share_split<THREADS>(s, 128, 64, Ahi, Alo);
      }
      ll_share_from_raw(st + 2 * NB * NB, s);
      tc::store_share_split<THREADS>(s, 64, 0, Bhi, Blo);
    }
    tc::fence_proxy_smem();
    ll_arrive(w.conv);
    if (tid == 0) {
      if (!tc::mbar_wait(w.conv, w.conv_phase, a.spin_limit)) ok = false;  // every thread's operands written
      w.conv_phase ^= 1;
      tc::fence_after_sync();
      tc::issue_product(w.tmem, tc::smem_u32(Ahi), tc::smem_u32(Alo), tc::smem_u32(Bhi), tc::smem_u32(Blo),
                        k % LL_CHUNK != 0 ? 1u : 0u);
      tc::mma_commit(w.mbar);
    }
    c0 = LLCLK();
    LLPROF(4, c0 - c1);
    if (k + 1 == j) {
      // both raw stages are consumed: A's tiles (i, j), (i + 1, j) for the
      // difference U = A - P come in while the last products run, each
      // thread's chunks where ll_difference reads them
      float* As = raw[0];
      for (int e = tid; e < (two ? 128 : 64) * 16; e += THREADS) {
        const int row = e >> 4, c4 = e & 15;
        cp_async16(As + row * NB + 4 * c4, tile<float>(a, i + (row >> 6), j) + (size_t)(row & 63) * a.ld + 4 * c4);
      }
      cp_async_commit();
    }
    if (k + 2 < j) {
      ok = ok && ll_thread_wait_rows(a, a.fin, rows, k + 3, seen);
      if (ok) ll_fetch_step(a, i, two, j, k + 2, st);
      else cp_async_commit();
      LLPROF(2, LLCLK() - c0);
    }
  }
  c0 = LLCLK();
  if (!tc::mbar_wait(w.mbar, w.phase, a.spin_limit)) ok = false;
  w.phase ^= 1;
  ok = __syncthreads_and(ok) != 0;
  LLPROF(3, LLCLK() - c0);
  if (!ok) {
    if (tid == 0) {
      atomicExch(a.ctl + 1, 1);
      atomicOr(a.err, PBG_DEV_ERR_BARRIER);
      atomicCAS(a.info, 0, -1);
    }
    return false;
  }
  tc::fence_after_sync();
  // P = racc + the last chunk from TMEM, into shared memory, row m = TMEM lane
  {
    float v[32];
    tc::tmem_ld32(tacc, v);
#pragma unroll
    for (int u = 0; u < 32; ++u) racc[u] += v[u];
  }
  if (two || q < 2) {  // warp-uniform
    float* dst = reinterpret_cast<float*>(w.base) + (size_t)m * LDA + 32 * g;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      *reinterpret_cast<float4*>(dst + 4 * u) =
          make_float4(racc[4 * u], racc[4 * u + 1], racc[4 * u + 2], racc[4 * u + 3]);
  }
  tc::fence_before_sync();
  __syncthreads();
  return true;
}

// U = A - P for rows i (and i + 1) of column j, a row of 64 per 16 threads;
// A from its prefetched copy As (row-major [128][64], j > 0) or from global
// memory (j = 0, no P); into the [64][LDA] tiles U0 / U1 in shared memory,
// or in place into A when to_global.
__device__ __forceinline__ void ll_difference(const DFArgs& a, int i, int j, bool two, const float* Ps,
                                              const float* As, float* U0, float* U1, bool to_global) {
  if (j > 0) cp_async_wait_group<0>();  // this thread's chunks of A, fetched during the last products
  for (int e = threadIdx.x; e < (two ? 128 : 64) * 16; e += THREADS) {
    const int row = e >> 4, c4 = e & 15;
    float4* gp = reinterpret_cast<float4*>(tile<float>(a, i + (row >> 6), j) + (size_t)(row & 63) * a.ld) + c4;
    float4 cv = j > 0 ? *reinterpret_cast<const float4*>(As + row * NB + 4 * c4) : __ldcg(gp);
    if (j > 0) {
      const float4 pv = *reinterpret_cast<const float4*>(Ps + (size_t)row * LDA + 4 * c4);
      cv.x -= pv.x;
      cv.y -= pv.y;
      cv.z -= pv.z;
      cv.w -= pv.w;
    }
    if (to_global) *gp = cv;
    else *reinterpret_cast<float4*>((row < 64 ? U0 : U1) + (row & 63) * LDA + 4 * c4) = cv;
  }
}

// One task of the left-looking list (kinds in cholesky_replica_tasks).
// Returns false if the run was aborted (nothing of this CTA in flight then).
__device__ bool ll_task(const DFArgs& a, int kind, int i, int j, LLWorker& w, int* seen, int* s_ok) {
  const int tid = threadIdx.x;
  const bool two = i + 1 < a.nt;
  const int rows[3] = {i, two ? i + 1 : i, j};
  if (tid < 3) seen[tid] = 0;
  float* Ps = reinterpret_cast<float*>(w.base);
  float* U0 = reinterpret_cast<float*>(w.base + LL_U0);
  float* U1 = reinterpret_cast<float*>(w.base + LL_U1);
  long long c0 = LLCLK();
  LLPROF(0, 1);
  LLPROF(1, j);
  if (kind != LL_SOLVE) {
    if (j > 0 && !ll_products(a, i, j, w)) return false;
    c0 = LLCLK();
    ll_difference(a, i, j, two, Ps, reinterpret_cast<const float*>(w.base + LL_OPERAND_BYTES), U0, U1,
                  kind == LL_UPDATE);
    __syncthreads();
    LLPROF(5, LLCLK() - c0);
    c0 = LLCLK();
  }
  float acc[16];
  if (kind == LL_DIAG) {
    // F(j) over P's bytes (no longer read), then S(j + 1, j) with inv(L_jj)
    // where factor_task_f32 left it
    LLPROF(11, 1);
    smem_to_acc(U0, acc);
    factor_task_f32(a, j, acc, w.base);
    publish(a.fin + j, j + 1);
    if (two) {
      solve_by_inverse(U1, reinterpret_cast<const float*>(w.base) + NB * LDA, acc);
      store_acc(tile<float>(a, j + 1, j), a.ld, acc);
      publish(a.fin + j + 1, j + 1);
    }
    LLPROF(6, LLCLK() - c0);
  } else if (kind == LL_UPDATE) {
    // U_ij (and U_{i+1,j}) stay in A's tiles for the solve task
    if (tid == 0) {
      st_release(a.upd + i, j + 1);
      if (two) st_release(a.upd + i + 1, j + 1);
    }
  } else {
    if (!ll_wait_rows(a, a.upd, rows, two ? 3u : 1u, j + 1, seen, s_ok)) return false;  // U_ij in A
    if (!ll_wait_rows(a, a.fin, rows, 4u, j + 1, seen, s_ok)) return false;             // F(j)
    LLPROF(7, LLCLK() - c0);
    c0 = LLCLK();
    float* Xs = reinterpret_cast<float*>(w.base);
    stage_async(reinterpret_cast<const float*>(a.invdiag) + (size_t)j * NB * NB, NB, Xs, LDA);
    stage_async(tile<float>(a, i, j), a.ld, U0, LDA);
    if (two) stage_async(tile<float>(a, i + 1, j), a.ld, U1, LDA);
    cp_async_wait_all();
    __syncthreads();
    solve_by_inverse(U0, Xs, acc);
    store_acc(tile<float>(a, i, j), a.ld, acc);
    if (two) {
      solve_by_inverse(U1, Xs, acc);
      store_acc(tile<float>(a, i + 1, j), a.ld, acc);
    }
    __syncthreads();
    if (tid == 0) {
      st_release(a.fin + i, j + 1);
      if (two) st_release(a.fin + i + 1, j + 1);
    }
    LLPROF(8, LLCLK() - c0);
  }
  __syncthreads();  // the next task overwrites the shared memory
  return true;
}

// One CTA per SM (192 KB of shared memory, 64 TMEM columns), all co-resident
// (cooperative launch).
__global__ void __launch_bounds__(THREADS, 1) chol_batch_ll_kernel(const CholRep* __restrict__ reps,
                                                                   const int4* __restrict__ tasks, int ntasks,
                                                                   int* ctl) {
  extern __shared__ __align__(1024) unsigned char ll_smem[];
  unsigned char* smem = ll_smem;
  if (tc::smem_u32(smem) & 1023u) {
    // the operands need a 1024-byte aligned start: give up on the whole run,
    // every replica reported as not factored (info -1)
    if (threadIdx.x == 0) {
      atomicExch(ctl + 1, 1);
      atomicOr(reinterpret_cast<unsigned*>(ctl + 3), PBG_DEV_ERR_BARRIER);
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x)
      atomicCAS(reps[tasks[t].x >> 3].info, 0, -1);
    return;
  }
  LLShared* sh = reinterpret_cast<LLShared*>(smem + LL_SHARED_OFFSET);
  if (threadIdx.x == 0) {
    tc::mbar_init(&sh->mbar, 1);
    tc::mbar_init(&sh->conv, THREADS);
    sh->ok = 1;
  }
  if (threadIdx.x < 32) tc::tmem_alloc(&sh->tmem, 64);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  LLWorker w;
  w.mbar = &sh->mbar;
  w.conv = &sh->conv;
  w.tmem = sh->tmem;
  w.phase = 0;
  w.conv_phase = 0;
  w.base = smem;
  const long long k0 = LLCLK();
  while (true) {
    const long long f0 = LLCLK();
    if (threadIdx.x == 0) sh->task = ld_acquire(ctl + 1) ? ntasks : atomicAdd(ctl, 1);
    __syncthreads();
    const int t = sh->task;
    __syncthreads();
    LLPROF(9, LLCLK() - f0);
    if (t >= ntasks) break;
    const int4 tk = tasks[t];
    const DFArgs a = batch_args(reps[tk.x >> 3], tasks, ntasks, ctl);
    if (!ll_task(a, tk.x & 7, tk.y, tk.z, w, sh->seen, &sh->ok)) break;
  }
  LLPROF(10, LLCLK() - k0);
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(w.tmem, 64);
}

std::mutex g_task_mu;
std::map<int, std::pair<int4*, int>> g_task_tables;

// Task list of the worker CTAs for an nt x nt tile grid (see the file comment).
// group: updates per task down a column (2; 4 for the FP32 kernel, whose
// updates run on the tcgen05 tensor cores); inverse: the tasks that form
// X = inv(L) as well;
// inv_tasks: the I(k) tasks that invert the diagonal tiles (left out when the
// chain CTA stores the inverses itself).
int get_task_table(int nt, int group, bool inv_tasks, bool inverse, const int4** out, int* count) {
  std::lock_guard<std::mutex> lk(g_task_mu);
  const int key = ((nt * 8 + group) * 2 + (inv_tasks ? 1 : 0)) * 2 + (inverse ? 1 : 0);
  auto it = g_task_tables.find(key);
  if (it != g_task_tables.end()) {
    *out = it->second.first;
    *count = it->second.second;
    return PBG_OK;
  }
  // The chain tasks F(k) and S(k+1, k) run on the chain CTA and are left out;
  // so is I(nt-1), which the chain forms after its last factorisation.
  std::vector<int4> t;
  if (nt > 1 && inv_tasks) t.push_back(make_int4(TASK_I, 0, 0, 0));
  for (int i = 2; i < nt; ++i) t.push_back(make_int4(TASK_S, i, 0, 0));
  for (int k = 0; k + 1 < nt; ++k) {
    // the last update of the chain's S(k+2, k+1), first: it runs during F(k+1)
    if (k + 2 < nt) t.push_back(make_int4(TASK_U, k + 2, k + 1, k));
    if (k + 2 < nt && inv_tasks) t.push_back(make_int4(TASK_I, 0, 0, k + 1));
    for (int i = k + 3; i < nt; ++i) t.push_back(make_int4(TASK_S, i, k + 1, k + 1));
    // the rest of column k+1 of the update with panel k is fused into F(k+1)
    // and the workers' S(., k+1); the plain updates cover columns >= k+2, the
    // one gating the next panel first
    // (rows grouped: U(i, jj, k), U(i+1, jj, k) [, U(i+2, jj, k)] share L_jj,k)
    for (int jj = k + 2; jj < nt; ++jj) {
      int i = jj;
      if (group >= 4)
        for (; i + 3 < nt; i += 4) t.push_back(make_int4(TASK_U4, i, jj, k));
      if (group >= 3)
        for (; i + 2 < nt; i += 3) t.push_back(make_int4(TASK_U3, i, jj, k));
      for (; i + 1 < nt; i += 2) t.push_back(make_int4(TASK_U2, i, jj, k));
      if (i < nt) t.push_back(make_int4(TASK_U, i, jj, k));
    }
    if (inverse) {
      // X = inv(L): row k+1 finished, then column k's contributions to the
      // rows below (pairs of rows)
      for (int j = 0; j <= k; ++j) t.push_back(make_int4(TASK_XZ, k + 1, j, 0));
      for (int j = 0; j <= k; ++j)
        for (int i = k + 2; i < nt; i += 2) t.push_back(make_int4(TASK_XG, i, j, k));
    }
  }
  int4* d = nullptr;
  if (!t.empty()) {
    if (cudaMalloc(&d, t.size() * sizeof(int4)) != cudaSuccess) {
      cudaGetLastError();
      return PBG_ERR_NOMEM;
    }
    PBG_CUDA_TRY(cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice));
  }
  g_task_tables[key] = std::make_pair(d, (int)t.size());
  *out = d;
  *count = (int)t.size();
  return PBG_OK;
}

template <typename T, bool F32CHAIN>
size_t df_smem_bytes() {
  // the chain, or a grouped update (the tensor-core operands in FP32, five
  // tiles in FP64)
  return std::max(F32CHAIN ? chain_f32_smem_bytes() : chain_smem_bytes<T>(),
                  sizeof(T) == 4 ? tc_worker_smem_bytes(2) : 5 * NB * LDA * sizeof(T));
}

// tasks_override / spin_limit: only for the wait-expiry self-test.
// X (or null): also form X = inv(L) (off-diagonal tiles); ints then holds
// the X flags after the factorisation's.
template <typename T, bool F32CHAIN = false>
int launch_df(T* A, int n, int ld, int* info, void* invdiag, int* ints, unsigned* err, cudaStream_t st,
              const int4* tasks_override = nullptr, int ntasks_override = 0, long long spin_limit = SPIN_LIMIT,
              T* X = nullptr) {
  static_assert(!F32CHAIN || sizeof(T) == 4, "the FP32 chain factors FP32 matrices");
  const int nt = ld / NB;
  const int4* tasks = nullptr;
  int ntasks = 0;
  if (tasks_override) {
    tasks = tasks_override;
    ntasks = ntasks_override;
  } else {
    int rc = get_task_table(nt, sizeof(T) == 4 ? 4 : 2, !F32CHAIN, X != nullptr, &tasks, &ntasks);
    if (rc) return rc;
  }
  const size_t smem = df_smem_bytes<T, F32CHAIN>();
  static int max_blocks_per_sm = -1;
  static int num_sms = 0;
  if (max_blocks_per_sm < 0) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(chol_df_kernel<T, F32CHAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    int dev;
    PBG_CUDA_TRY(cudaGetDevice(&dev));
    PBG_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    PBG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_blocks_per_sm, chol_df_kernel<T, F32CHAIN>,
                                                               THREADS, smem));
    if (max_blocks_per_sm < 1) {
      pbg_set_error_message("cholesky kernel does not fit on an SM");
      return PBG_ERR_CUDA;
    }
  }
  // one CTA per SM: the chain CTA has its SM to itself
  int grid = num_sms;
  if (grid > ntasks + 1) grid = ntasks + 1;  // the chain CTA plus the shared tasks
  PBG_CUDA_TRY(cudaMemsetAsync(ints, 0, (3 + (X ? 4 : 2) * (size_t)nt * nt) * sizeof(int), st));
  PBG_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
  DFArgs args;
  args.A = A;
  args.ld = ld;
  args.n = n;
  args.nt = nt;
  args.ntasks = ntasks;
  args.tasks = tasks;
  args.ctl = ints;
  args.upd = ints + 3;
  args.fin = ints + 3 + nt * nt;
  args.X = X;
  args.xupd = ints + 3 + 2 * nt * nt;
  args.xfin = ints + 3 + 3 * nt * nt;
  args.info = info;
  args.invdiag = invdiag;
  args.err = err;
  args.spin_limit = spin_limit;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PBG_CUDA_TRY(cudaLaunchKernelEx(&cfg, chol_df_kernel<T, F32CHAIN>, args));
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace

// Self-test of the bounded waits (no counterpart in the reference): factors a
// 192 x 192 SPD matrix with a task list from which the host drops the update
// U(2,2,0), so the wait of F(2) for it can never be satisfied.  The wait
// gives up after spin_limit polls; the launch must end with info = -1 and the
// barrier error bit, the device must stay usable, and a normal
// factorisation right after must succeed.  Returns PBG_OK when all of that
// holds; *info_out and *err_out receive what the aborted launch reported.
extern "C" __attribute__((visibility("default"))) int pbg_selftest_wait_expiry(long long spin_limit, int* info_out,
                                                                                unsigned* err_out) {
  using namespace pbg;
  const int n = 192, ld = 192, nt = 3;
  if (spin_limit < 1 || spin_limit > (1LL << 24)) return PBG_ERR_ARG;
  const int4* full = nullptr;
  int nfull = 0;
  int rc = get_task_table(nt, 2, true, false, &full, &nfull);
  if (rc) return rc;
  std::vector<int4> tasks(nfull);
  PBG_CUDA_TRY(cudaMemcpy(tasks.data(), full, nfull * sizeof(int4), cudaMemcpyDeviceToHost));
  const auto dropped = std::remove_if(tasks.begin(), tasks.end(), [](const int4& t) {
    return (t.x == TASK_U || t.x == TASK_U2) && t.y == 2 && t.z == 2 && t.w == 0;
  });
  if (dropped == tasks.end()) return PBG_ERR_STATE;
  tasks.erase(dropped, tasks.end());
  std::vector<double> h((size_t)ld * ld, 0.0);
  for (int i = 0; i < n; ++i) {
    h[(size_t)i * ld + i] = 4.0;
    if (i > 0) h[(size_t)i * ld + i - 1] = h[(size_t)(i - 1) * ld + i] = 1.0;
  }
  double *A = nullptr, *inv = nullptr;
  int4* dt = nullptr;
  int* ints = nullptr;
  const size_t nints = 3 + 2 * (size_t)nt * nt + 2;
  bool ok = cudaMalloc(&A, h.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&inv, (size_t)nt * NB * NB * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&dt, tasks.size() * sizeof(int4)) == cudaSuccess &&
            cudaMalloc(&ints, nints * sizeof(int)) == cudaSuccess;
  int result = PBG_OK;
  if (!ok) {
    cudaGetLastError();
    result = PBG_ERR_NOMEM;
  } else {
    int* info = ints + nints - 2;
    unsigned* err = reinterpret_cast<unsigned*>(ints + nints - 1);
    int hinfo = 0;
    unsigned herr = 0;
    cudaMemcpy(A, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dt, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice);
    cudaMemset(err, 0, sizeof(unsigned));
    result = launch_df<double>(A, n, ld, info, inv, ints, err, 0, dt, (int)tasks.size(), spin_limit);
    if (result == PBG_OK && cudaDeviceSynchronize() != cudaSuccess) result = PBG_ERR_CUDA;
    if (result == PBG_OK) {
      cudaMemcpy(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost);
      if (info_out) *info_out = hinfo;
      if (err_out) *err_out = herr;
      if (hinfo != -1 || !(herr & PBG_DEV_ERR_BARRIER)) result = PBG_ERR_STATE;
    }
    if (result == PBG_OK) {
      // the context is still usable: the full task list factors the matrix
      cudaMemcpy(A, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemset(err, 0, sizeof(unsigned));
      result = launch_df<double>(A, n, ld, info, inv, ints, err, 0);
      if (result == PBG_OK && cudaDeviceSynchronize() != cudaSuccess) result = PBG_ERR_CUDA;
      if (result == PBG_OK) {
        cudaMemcpy(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost);
        if (hinfo != 0) result = PBG_ERR_STATE;
      }
    }
  }
  if (A) cudaFree(A);
  if (inv) cudaFree(inv);
  if (dt) cudaFree(dt);
  if (ints) cudaFree(ints);
  if (result != PBG_OK && result != PBG_ERR_CUDA)
    pbg_set_error_message("wait-expiry self-test: the aborted launch or the follow-up factorisation misbehaved");
  return result;
}

#ifdef PBG_TASK_TRACE
extern "C" __attribute__((visibility("default"))) int pbg_task_trace(long long* host, int ntasks) {
  PBG_CUDA_TRY(cudaMemcpyFromSymbol(host, g_task_trace, sizeof(long long) * 4 * ntasks));
  return PBG_OK;
}
extern "C" __attribute__((visibility("default"))) int pbg_ll_profile(long long* host, int ctas) {
  PBG_CUDA_TRY(cudaMemcpyFromSymbol(host, g_ll_prof, sizeof(long long) * 16 * ctas));
  return PBG_OK;
}
extern "C" __attribute__((visibility("default"))) int pbg_chain_trace(long long* host, int nt) {
  PBG_CUDA_TRY(cudaMemcpyFromSymbol(host, g_chain_trace, sizeof(long long) * 8 * nt));
  return PBG_OK;
}
#endif

// Scratch of one factorisation: task counter, abort flag, per-tile flags,
// error word.
size_t df_work_bytes(int ld) {
  const int nt = ld / NB;
  return (3 + 4 * (size_t)nt * nt + 1) * sizeof(int) + 64;
}

// Factors A in place and writes the inverse of every diagonal factor tile to
// invdiag (nt x 64 x 64 row-major tiles, precision of A; the solves of the
// factorisation use them, and so do the SPD inverse and the triangular solve
// of the midpoint scheme).  Both A and invdiag start on 16-byte boundaries.
int launch_cholesky_df(void* A, int n, int ld, int precision, int* info, void* invdiag, void* work,
                       cudaStream_t st, void* X) {
  const int nt = ld / NB;
  if (reinterpret_cast<uintptr_t>(A) % 16 != 0 || reinterpret_cast<uintptr_t>(invdiag) % 16 != 0) {
    pbg_set_error_message("cholesky: the matrix and its workspace must start on 16-byte boundaries");
    return PBG_ERR_ARG;
  }
  int* ints = static_cast<int*>(work);
  unsigned* err = reinterpret_cast<unsigned*>(ints + 3 + 4 * (size_t)nt * nt);
  if (precision == PBG_PREC_FP64)
    return launch_df<double>((double*)A, n, ld, info, invdiag, ints, err, st, nullptr, 0, SPIN_LIMIT, (double*)X);
  if (precision == PBG_PREC_MIXED_FP64_DIAG)
    return launch_df<float, false>((float*)A, n, ld, info, invdiag, ints, err, st, nullptr, 0, SPIN_LIMIT,
                                   (float*)X);
  return launch_df<float, true>((float*)A, n, ld, info, invdiag, ints, err, st, nullptr, 0, SPIN_LIMIT, (float*)X);
}


// One replica's tasks in its own order, cut into segments: segment 0 =
// F(0), S(i, 0); then for each k three segments F(k+1) | U(i, j, k) (j >= k+2)
// | S(i, k+1) (i >= k+2).  F(k+1) and S(., k+1) apply their update with panel
// k themselves.  seg_start holds 1 + 3(nt-1) segment starts and the end.
// A batch merges the replicas' lists segment number by segment number (all
// replicas' segment s, larger matrices first, then segment s+1): every
// replica's F(k+1), then every replica's U(., ., k), then every replica's
// S(., k+1), so the solves are fetched after their factorisations had the
// whole update phase to finish.  F(k+1) and U(., ., k) depend only on block
// k-1; S(., k+1) on F(k+1) and block k-1: every task depends only on earlier
// tasks.  The tasks carry replica tag 0; the merge writes the replica index.
//
// The mixed-precision lists are left-looking (chol_batch_ll_kernel), two
// segments per column j: LL_DIAG for rows (j, j + 1) and LL_UPDATE for the
// row pairs (j + 2, j + 3), (j + 4, j + 5), ...; then LL_SOLVE for the same
// pairs.  Merged by segment number, every replica's solves of column j come
// after every replica's updates of column j, so F(j) has had that phase to
// finish; column j + 1's tasks need column j's solves and come after them.
void cholesky_replica_tasks(int nt, int precision, std::vector<int4>& tasks, std::vector<int>& seg_start) {
  tasks.clear();
  seg_start.clear();
  if (nt < 1) return;
  if (precision != PBG_PREC_FP64) {
    for (int j = 0; j < nt; ++j) {
      seg_start.push_back((int)tasks.size());
      tasks.push_back(make_int4(LL_DIAG, j, j, 0));
      for (int i = j + 2; i < nt; i += 2) tasks.push_back(make_int4(LL_UPDATE, i, j, 0));
      seg_start.push_back((int)tasks.size());
      for (int i = j + 2; i < nt; i += 2) tasks.push_back(make_int4(LL_SOLVE, i, j, 0));
    }
    seg_start.push_back((int)tasks.size());
    return;
  }
  seg_start.push_back(0);
  tasks.push_back(make_int4(TASK_F, 0, 0, 0));
  for (int i = 1; i < nt; ++i) tasks.push_back(make_int4(TASK_S, i, 0, 0));
  for (int k = 0; k + 1 < nt; ++k) {
    seg_start.push_back((int)tasks.size());
    tasks.push_back(make_int4(TASK_F, k + 1, k + 1, k + 1));
    seg_start.push_back((int)tasks.size());
    for (int jj = k + 2; jj < nt; ++jj) {  // rows paired, as in the single-matrix list
      int i = jj;
      for (; i + 1 < nt; i += 2) tasks.push_back(make_int4(TASK_U2, i, jj, k));
      if (i < nt) tasks.push_back(make_int4(TASK_U, i, jj, k));
    }
    seg_start.push_back((int)tasks.size());
    for (int i = k + 2; i < nt; ++i) tasks.push_back(make_int4(TASK_S, i, k + 1, k + 1));
  }
  seg_start.push_back((int)tasks.size());
}

// Resident CTAs per SM of the batched factorisation kernel of this
// precision (the occupancy query, once per precision) and the SM count.
int cholesky_batch_residency(int precision, int* ctas_per_sm, int* sms) {
  const bool f64 = precision == PBG_PREC_FP64;
  const size_t smem = f64 ? batch_smem_bytes() : ll_smem_bytes();
  static int blocks_per_sm[2] = {-1, -1};
  static int num_sms = 0;
  int& bps = blocks_per_sm[f64 ? 0 : 1];
  if (bps < 0) {
    int dev;
    PBG_CUDA_TRY(cudaGetDevice(&dev));
    PBG_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    int b = 0;
    if (f64) {
      PBG_CUDA_TRY(cudaFuncSetAttribute(chol_batch_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PBG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, chol_batch_kernel<double>, THREADS, smem));
    } else {
      PBG_CUDA_TRY(cudaFuncSetAttribute(chol_batch_ll_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PBG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, chol_batch_ll_kernel, THREADS, smem));
    }
    if (b < 1) {
      pbg_set_error_message("batched cholesky kernel does not fit on an SM");
      return PBG_ERR_CUDA;
    }
    bps = b;
  }
  *ctas_per_sm = bps;
  *sms = num_sms;
  return PBG_OK;
}

int launch_cholesky_batch(int precision, const CholRep* reps, const int4* tasks, int ntasks, int* ctl,
                          int ctas_per_sm, cudaStream_t st) {
  if (ntasks <= 0) return PBG_OK;
  const bool f64 = precision == PBG_PREC_FP64;
  const size_t smem = f64 ? batch_smem_bytes() : ll_smem_bytes();
  int bps = 0, num_sms = 0;
  int rc = cholesky_batch_residency(precision, &bps, &num_sms);
  if (rc) return rc;
  int grid = num_sms * (ctas_per_sm > 0 ? std::min(ctas_per_sm, bps) : bps);
  if (grid > ntasks) grid = ntasks;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (f64) PBG_CUDA_TRY(cudaLaunchKernelEx(&cfg, chol_batch_kernel<double>, reps, tasks, ntasks, ctl));
  else {
    const cudaError_t e = cudaLaunchKernelEx(&cfg, chol_batch_ll_kernel, reps, tasks, ntasks, ctl);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
      // say what the asked-for residency would need
      cudaGetLastError();
      size_t avail = 0;
      cudaFuncAttributes fa = {};
      cudaOccupancyAvailableDynamicSMemPerBlock(&avail, chol_batch_ll_kernel, grid / num_sms, THREADS);
      cudaFuncGetAttributes(&fa, chol_batch_ll_kernel);
      cudaGetLastError();
      pbg_set_error_message(
          "batched factorisation: %d CTAs per SM do not fit (%zu bytes of dynamic shared memory per CTA, %zu "
          "available at that residency; %d registers per thread, %zu bytes static shared memory)",
          grid / num_sms, smem, avail, fa.numRegs, fa.sharedSizeBytes);
      return PBG_ERR_CUDA;
    }
    PBG_CUDA_TRY(e);
  }
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}


// ---------------------------------------------------------------- SPD inverse on the tensor cores
// inv(A) = X^T X with A = L L^T and X = inv(L): the data-flow factorisation
// forms X's off-diagonal tiles in the same launch (XG / XZ tasks), then X's
// diagonal tiles are copied from invdiag and X^T X runs with one CTA per lower
// tile.  Every tile product is
// TileMMA: FP64 DMMA for FP64 matrices, 3xTF32 split products with FP32
// accumulation for FP32 ones.  Used by the SPD inverse of the FP64
// lubrication path (cholesky.cu) and by the mixed lubricated path, which also
// reads the factor of kBT inv(R) off X (tc_reversed_factor).
//
// Mixed workspace (tc_inverse_work_bytes): [inv(L_kk) tiles][data-flow
// scratch][X: ld x ld][F: ld x ld], F the matrix to factor (in place).

namespace {

template <typename T>
constexpr size_t tc_smem_bytes() {
  return 2 * NB * LDA * sizeof(T);
}

// Transposed staging of a 64 x 64 tile, s[c][r] = g[r][c] (rows of LDA in
// smem), in two halves so that a thread's 16 global loads are all in flight
// before the first shared store: load_tile_regs, then store_tile_transposed.
template <typename T>
__device__ __forceinline__ void load_tile_regs(const T* __restrict__ g, int ld, T (&v)[TILE_PER_THREAD]) {
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) {
    const int e = threadIdx.x + q * THREADS;
    v[q] = g[(size_t)(e >> 6) * ld + (e & 63)];
  }
}
template <typename T>
__device__ __forceinline__ void store_tile_transposed(const T (&v)[TILE_PER_THREAD], T* s) {
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) {
    const int e = threadIdx.x + q * THREADS;
    s[(e & 63) * LDA + (e >> 6)] = v[q];
  }
}
template <typename T>
__device__ __forceinline__ void stage_transposed(const T* __restrict__ g, int ld, T* s) {
  T v[TILE_PER_THREAD];
  load_tile_regs(g, ld, v);
  store_tile_transposed(v, s);
}

// X_kk = inv(L_kk), upper triangle zero (one CTA per diagonal tile).
template <typename T>
__global__ void __launch_bounds__(THREADS) trtri_diag_kernel(const T* __restrict__ invdiag, T* X, int ld) {
  const int k = blockIdx.x;
  T* g = X + (size_t)k * NB * ld + (size_t)k * NB;
  const T* inv = invdiag + (size_t)k * NB * NB;
  T v[TILE_PER_THREAD];
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) v[q] = inv[threadIdx.x + q * THREADS];
#pragma unroll
  for (int q = 0; q < TILE_PER_THREAD; ++q) {
    const int e = threadIdx.x + q * THREADS, r = e >> 6, c = e & 63;
    g[(size_t)r * ld + c] = c <= r ? v[q] : T(0);
  }
}

// out_IJ = scale (X^T X)_IJ = scale sum_{k >= I} X_kI^T X_kJ for the lower
// tile (I, J), written to (I, J) and (J, I); with `reversed` every element
// (r, c) goes to (ld-1-r, ld-1-c) instead.
template <typename T>
__global__ void __launch_bounds__(THREADS) lauum_tc_kernel(const T* __restrict__ X, int ld, int nt, T scale,
                                                           int reversed, T* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + NB * LDA;
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) ++I;
  while (I * (I + 1) / 2 > b) --I;
  const int J = b - I * (I + 1) / 2;
  T acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = T(0);
  // the tiles of step k+1 are loaded into registers while step k multiplies
  T va[TILE_PER_THREAD], vb[TILE_PER_THREAD];
  load_tile_regs(X + (size_t)I * NB * ld + (size_t)I * NB, ld, va);
  load_tile_regs(X + (size_t)I * NB * ld + (size_t)J * NB, ld, vb);
  for (int k = I; k < nt; ++k) {
    store_tile_transposed(va, sA);
    store_tile_transposed(vb, sB);
    __syncthreads();
    if (k + 1 < nt) {
      load_tile_regs(X + (size_t)(k + 1) * NB * ld + (size_t)I * NB, ld, va);
      load_tile_regs(X + (size_t)(k + 1) * NB * ld + (size_t)J * NB, ld, vb);
    }
    TileMMA<T>::sub(sA, sB, acc);
    __syncthreads();
  }
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 8; ++cs) {
      const T v = -acc[TileMMA<T>::idx(rs, cs)] * scale;
      int r = I * NB + acc_row(rs), c = J * NB + acc_col(cs);
      if (reversed) {
        r = ld - 1 - r;
        c = ld - 1 - c;
      }
      out[(size_t)r * ld + c] = v;
      if (I != J) out[(size_t)c * ld + r] = v;  // a diagonal tile writes each element once
    }
}

// B[i][j] = scale X[ld-1-j][ld-1-i] for the lower triangle of B (32 x 32
// tiles through smem; tiles above the diagonal are not written).
template <typename T>
__global__ void reversed_transpose_kernel(const T* __restrict__ X, int ld, T scale, T* __restrict__ B) {
  __shared__ T t[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int x0r = ld - 32 * (bj + 1), x0c = ld - 32 * (bi + 1);
  for (int r = threadIdx.y; r < 32; r += blockDim.y) t[r][threadIdx.x] = X[(size_t)(x0r + r) * ld + x0c + threadIdx.x];
  __syncthreads();
  for (int rr = threadIdx.y; rr < 32; rr += blockDim.y)
    B[(size_t)(bi * 32 + rr) * ld + bj * 32 + threadIdx.x] = scale * t[31 - threadIdx.x][31 - rr];
}

// inv(B_II) for B = s J G^{-T} J (G lower, order ld, J the reversal of all ld
// indices): (1/s) J G_I'I'^T J with I' = nt-1-I, from the lower triangle of
// G's diagonal tile.
template <typename T>
__global__ void b_invdiag_kernel(const T* __restrict__ G, int ld, int nt, T inv_scale, T* __restrict__ invdiag) {
  const int I = blockIdx.x, Ip = nt - 1 - I;
  const T* g = G + (size_t)Ip * NB * ld + (size_t)Ip * NB;
  T* o = invdiag + (size_t)I * NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    o[e] = r >= c ? inv_scale * g[(size_t)(NB - 1 - c) * ld + (NB - 1 - r)] : T(0);
  }
}

// ---------------------------------------------------------------- X^T X on tcgen05 (FP32)
// out = scale X^T X for the lower-triangular FP32 X (the SPD inverse's
// symmetric product in the mixed lubricated path): a CTA forms the output
// tiles (I, J) and (I + 1, J) (only (I, J) when I + 1 = nt) as one M = 128,
// N = 64 product over the K range k = I .. nt-1,
//   [X_kI^T; X_{k,I+1}^T] X_kJ    (X_{I,I+1} above the diagonal taken as 0),
// in 3xTF32 on the tensor cores.  Per K-step the three tiles arrive row-major
// by cp.async two K-steps ahead (raw stages); the transposition is done by
// the split into the K-major hi / lo operands (column m of X_kI becomes row
// m of A).  The accumulator restarts in TMEM every SYM_CHUNK K-steps and the
// chunk sums are added in FP32 (as in the left-looking batch kernel).
// Each element is written once: (r, c) and, off the diagonal tiles, (c, r);
// with `reversed`, (ld-1-r, ld-1-c) instead.
constexpr int SYM_CHUNK = 4;
constexpr uint32_t SYM_SHARED_OFFSET = LL_OPERAND_BYTES + 2 * LL_RAW_BYTES;
constexpr size_t sym_smem_bytes() { return SYM_SHARED_OFFSET + 16; }  // mbarrier, TMEM address
static_assert(sym_smem_bytes() <= 227 * 1024, "the symmetric product does not fit an SM");

// Output tile pairs: for each J, I = J, J + 2, J + 4, ...
__host__ __device__ inline int sym_pairs(int nt) {
  int n = 0;
  for (int J = 0; J < nt; ++J) n += (nt - J + 1) / 2;
  return n;
}

// The K-step k tiles: X_kI, X_{k,I+1} (when it is a lower tile), X_kJ.
__device__ __forceinline__ void sym_fetch_step(const float* X, int ld, int I, int J, int k, bool two, float* raw) {
  const float* row = X + (size_t)k * NB * ld;
  ll_fetch_tile(row + (size_t)I * NB, ld, raw);
  if (two && k >= I + 1) ll_fetch_tile(row + (size_t)(I + 1) * NB, ld, raw + NB * NB);
  ll_fetch_tile(row + (size_t)J * NB, ld, raw + 2 * NB * NB);
  cp_async_commit();
}

__global__ void __launch_bounds__(THREADS, 1) sym_tc_kernel(const float* __restrict__ X, int ld, int nt, float scale,
                                                           int reversed, float* __restrict__ out, int* info) {
  extern __shared__ __align__(1024) unsigned char sym_smem[];
  unsigned char* base = sym_smem;
  const int tid = threadIdx.x;
  if (tc::smem_u32(base) & 1023u) {  // the operands need a 1024-byte aligned start
    if (tid == 0) atomicCAS(info, 0, -1);
    return;
  }
  uint64_t* mbar = reinterpret_cast<uint64_t*>(base + SYM_SHARED_OFFSET);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(base + SYM_SHARED_OFFSET + 8);
  int b = blockIdx.x, J = 0;
  for (; J < nt; ++J) {
    const int cnt = (nt - J + 1) / 2;
    if (b < cnt) break;
    b -= cnt;
  }
  const int I = J + 2 * b;
  const bool two = I + 1 < nt;
  if (tid == 0) tc::mbar_init(mbar, 1);
  if (tid < 32) tc::tmem_alloc(s_tmem, 64);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;
  uint32_t phase = 0;
  unsigned char* Ahi = base;
  unsigned char* Alo = Ahi + LL_A_BYTES;
  unsigned char* Bhi = Alo + LL_A_BYTES;
  unsigned char* Blo = Bhi + LL_B_BYTES;
  float* raw[2] = {reinterpret_cast<float*>(base + LL_OPERAND_BYTES),
                   reinterpret_cast<float*>(base + LL_OPERAND_BYTES + LL_RAW_BYTES)};
  const int warp = tid >> 5, lane = tid & 31, q = warp & 3, g = warp >> 2;
  const uint32_t tacc = tmem + ((uint32_t)(32 * q) << 16) + 32 * g;
  // this thread's operand rows: A row ma (chunks 2e + tid / 128), B row nb
  // (chunks 4e + tid / 64)
  const int ma = tid & 127, nb = tid & 63;
  sym_fetch_step(X, ld, I, J, I, two, raw[0]);
  if (I + 1 < nt) sym_fetch_step(X, ld, I, J, I + 1, two, raw[1]);
  float racc[32];
#pragma unroll
  for (int u = 0; u < 32; ++u) racc[u] = 0.0f;
  bool ok = true;
  for (int k = I; k < nt; ++k) {
    const int s = k - I;
    float* st = raw[s & 1];
    if (k + 1 < nt) cp_async_wait_group<1>();
    else cp_async_wait_group<0>();
    __syncthreads();  // every thread's copies of this K-step are in
    if (s > 0) {      // the products of the previous K-step have read the operands
      if (!tc::mbar_wait(mbar, phase, SPIN_LIMIT)) ok = false;
      phase ^= 1;
      tc::fence_after_sync();
      if (s % SYM_CHUNK == 0) {
        float v[32];
        tc::tmem_ld32(tacc, v);
#pragma unroll
        for (int u = 0; u < 32; ++u) racc[u] += v[u];
        tc::fence_before_sync();
      }
    }
    // A row ma: column ma of X_kI (ma < 64) or of X_{k,I+1} (zero for k = I
    // or beyond the last tile); chunk c holds K = 4c .. 4c+3 (rows of X)
    {
      const bool zero = ma >= 64 && !(two && k >= I + 1);
      const float* src = st + (ma < 64 ? 0 : NB * NB) + (ma & 63);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int c = 2 * e + (tid >> 7);
        float4 x = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (!zero) x = make_float4(src[(4 * c) * NB], src[(4 * c + 1) * NB], src[(4 * c + 2) * NB], src[(4 * c + 3) * NB]);
        tc::store_split_chunk(x, tc::sw128_offset(128, ma, c), Ahi, Alo);
      }
      const float* srcb = st + 2 * NB * NB + nb;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int c = 4 * e + (tid >> 6);
        const float4 x =
            make_float4(srcb[(4 * c) * NB], srcb[(4 * c + 1) * NB], srcb[(4 * c + 2) * NB], srcb[(4 * c + 3) * NB]);
        tc::store_split_chunk(x, tc::sw128_offset(64, nb, c), Bhi, Blo);
      }
    }
    tc::fence_proxy_smem();
    __syncthreads();  // operands written; every thread is past its reads of this stage
    if (tid == 0) {
      tc::fence_after_sync();
      tc::issue_product(tmem, tc::smem_u32(Ahi), tc::smem_u32(Alo), tc::smem_u32(Bhi), tc::smem_u32(Blo),
                        s % SYM_CHUNK != 0 ? 1u : 0u);
      tc::mma_commit(mbar);
    }
    if (k + 2 < nt) sym_fetch_step(X, ld, I, J, k + 2, two, st);
  }
  if (!tc::mbar_wait(mbar, phase, SPIN_LIMIT)) ok = false;
  ok = __syncthreads_and(ok) != 0;
  tc::fence_after_sync();
  {
    float v[32];
    tc::tmem_ld32(tacc, v);
#pragma unroll
    for (int u = 0; u < 32; ++u) racc[u] += v[u];
  }
  const int m = 32 * q + lane, t = m >> 6;
  if (ok && (t == 0 || two)) {
    const int It = I + t;
    const int r0 = It * NB + (m & 63), c0 = J * NB + 32 * g;
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      const float v = racc[u] * scale;
      int r = r0, c = c0 + u;
      if (reversed) {
        r = ld - 1 - r;
        c = ld - 1 - c;
      }
      out[(size_t)r * ld + c] = v;
      if (It != J) out[(size_t)c * ld + r] = v;
    }
  }
  if (!ok && tid == 0) atomicCAS(info, 0, -1);
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) tc::tmem_dealloc(tmem, 64);
}

// Dynamic shared memory above the 48 KB default (the FP64 tiles), set on the
// current device before each use.
template <typename T>
int set_tc_smem() {
  constexpr int smem = (int)tc_smem_bytes<T>();
  PBG_CUDA_TRY(cudaFuncSetAttribute(lauum_tc_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  return PBG_OK;
}

template <typename T>
int lauum_tc(const T* X, int ld, T scale, bool reversed, T* out, cudaStream_t st) {
  const int nt = ld / NB;
  if (int rc = set_tc_smem<T>()) return rc;
  lauum_tc_kernel<T><<<nt * (nt + 1) / 2, THREADS, tc_smem_bytes<T>(), st>>>(X, ld, nt, scale, reversed ? 1 : 0,
                                                                             out);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace

int launch_trtri_diag(const void* invdiag, void* X, int ld, int precision, cudaStream_t st) {
  if (ld % NB != 0 || ld <= 0) return PBG_ERR_ARG;
  const int nt = ld / NB;
  if (precision == PBG_PREC_FP64) trtri_diag_kernel<double><<<nt, THREADS, 0, st>>>((const double*)invdiag, (double*)X, ld);
  else trtri_diag_kernel<float><<<nt, THREADS, 0, st>>>((const float*)invdiag, (float*)X, ld);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_lauum_tc(const void* X, int ld, double scale, bool reversed, void* out, int precision, cudaStream_t st) {
  if (ld % NB != 0 || ld <= 0) return PBG_ERR_ARG;
  if (precision == PBG_PREC_FP64) return lauum_tc<double>((const double*)X, ld, scale, reversed, (double*)out, st);
  return lauum_tc<float>((const float*)X, ld, (float)scale, reversed, (float*)out, st);
}

// The data-flow scratch rounded up to 256 bytes, so X and F start aligned
// whatever the tile count (the scratch itself is 80 + 8 nt^2 bytes).
static size_t tc_scratch_bytes(int ld) { return (df_work_bytes(ld) + 255) / 256 * 256; }

size_t tc_inverse_work_bytes(int ld) {
  const size_t nt = ld / NB;
  return nt * NB * NB * sizeof(float) + tc_scratch_bytes(ld) + 2 * (size_t)ld * ld * sizeof(float);
}

TcInverseWork tc_inverse_work(void* work, int ld) {
  const size_t nt = ld / NB;
  unsigned char* p = static_cast<unsigned char*>(work);
  TcInverseWork w;
  w.invdiag = reinterpret_cast<float*>(p);
  w.scratch = p + nt * NB * NB * sizeof(float);
  w.X = reinterpret_cast<float*>(static_cast<unsigned char*>(w.scratch) + tc_scratch_bytes(ld));
  w.F = w.X + (size_t)ld * ld;
  return w;
}

int tc_factor_invert(int ld, int* info, void* work, cudaStream_t st) {
  if (ld % NB != 0 || ld <= 0) return PBG_ERR_ARG;
  const TcInverseWork w = tc_inverse_work(work, ld);
  if (reinterpret_cast<uintptr_t>(w.X) % 16 != 0) {
    pbg_set_error_message("tensor-core inverse: misaligned workspace");
    return PBG_ERR_ARG;
  }
  // the factorisation forms X's off-diagonal tiles in the same launch
  int rc = launch_cholesky_df(w.F, ld, ld, PBG_PREC_MIXED, info, w.invdiag, w.scratch, st, w.X);
  if (rc != PBG_OK) return rc;
  return launch_trtri_diag(w.invdiag, w.X, ld, PBG_PREC_MIXED, st);
}

int tc_lauum(const float* X, int ld, float scale, bool reversed, float* out, int* info, cudaStream_t st) {
  if (ld % NB != 0 || ld <= 0) return PBG_ERR_ARG;
  const int nt = ld / NB;
  PBG_CUDA_TRY(cudaFuncSetAttribute(sym_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sym_smem_bytes()));
  sym_tc_kernel<<<sym_pairs(nt), THREADS, sym_smem_bytes(), st>>>(X, ld, nt, scale, reversed ? 1 : 0, out, info);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int tc_reversed_factor(const float* X, const float* G, int ld, double s, float* B, float* invdiag,
                       cudaStream_t st) {
  const int nt = ld / NB;
  reversed_transpose_kernel<float><<<dim3(ld / 32, ld / 32), dim3(32, 8), 0, st>>>(X, ld, (float)s, B);
  PBG_CHECK_LAUNCH();
  b_invdiag_kernel<float><<<nt, THREADS, 0, st>>>(G, ld, nt, (float)(1.0 / s), invdiag);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
