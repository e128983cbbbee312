// Data-flow tiled Cholesky factorisation on sm_100a (the factor of
// numpy.linalg.cholesky at src/bdsim/pyBrown/box.py:554).
//
// One persistent kernel, all CTAs co-resident (cooperative launch).  The
// 64 x 64 tiles of the lower triangle are processed as tasks taken in a fixed
// order from an atomic counter:
//   F(k)     diagonal tile k: its last update (column k-1), then the
//            factorisation -- 8-column panels chained by one warp in registers
//            with rsqrt pivots, rank-8 trailing updates by the whole CTA -- and
//            the full inverse of the factor tile (8 x 8 diagonal blocks, then
//            the off-diagonal blocks by block distance);
//   S(i, k)  tile (i, k) below the diagonal: its last update, then
//            L_ik = A_ik inv(L_kk)^T as one tensor-core tile product;
//   U(i,j,k) trailing update A_ij -= L_ik L_jk^T (j >= k+2) on the tensor
//            cores: FP64 DMMA (mma.sync m8n8k4 f64) in the FP64 path,
//            3xTF32 split products (mma.sync m16n8k8 tf32, hi*hi + hi*lo +
//            lo*hi, FP32 accumulation) in the mixed path.
// The diagonal tiles are factored in the precision of the matrix: FP64 in
// the FP64 path, FP32 in the mixed path.
// Task order: F(0), S(.,0), then for each k: F(k+1), S(.,k+1), U(.,.,k) -- the
// next panel comes before the bulk of the current trailing update (look-ahead
// of one panel), and every task depends only on tasks earlier in the list, so
// with all CTAs resident the lowest unfinished task can always run.
//
// Dependencies are tracked per tile: upd[i][j] counts applied updates,
// fin[i][j] marks a final L tile.  Waits spin on these flags with a bounded
// iteration count; on expiry the kernel raises an abort flag, marks info = -1
// and every CTA returns.  Tile data written by other CTAs is read with
// L2-coherent loads (ld.global.cg).
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

namespace {

constexpr int NB = 64;
constexpr int THREADS = 256;
constexpr int LDA = NB + 4;   // staged tile row (bank-conflict-free fragment loads)
constexpr int LDT = NB + 1;   // FP64 factor tile row
constexpr long long SPIN_LIMIT = 1LL << 24;

enum : int { TASK_F = 0, TASK_S = 1, TASK_U = 2 };

struct DFArgs {
  void* A;
  int ld, n, nt, ntasks;
  const int4* tasks;
  int* ctl;      // [0] next task, [1] abort, [2] spin failures
  int* upd;      // nt * nt
  int* fin;      // nt * nt
  int* info;
  void* leafinv; // nt * 8 * 64 (T): inverses of the 8 x 8 diagonal blocks of each L_kk
  unsigned* err;
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
// [fetch, waits done, end] in globaltimer ns and the SM id.
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
#else
#define TRACE(slot, t)
#endif

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }

// Thread 0 waits until every flags[q] >= targets[q] (bounded); returns false
// if the run was aborted.  The acquire loads by thread 0 followed by the CTA
// barrier order every thread's later reads after the producers' release.
__device__ bool wait_all(const DFArgs& a, const int* const* flags, const int* targets, int count, int* s_ok) {
  if (threadIdx.x == 0) {
    int ok = 1;
    for (int q = 0; q < count && ok; ++q) {
      long long it = 0;
      while (ld_acquire(flags[q]) < targets[q]) {
        if (ld_acquire(a.ctl + 1)) { ok = 0; break; }
        if (++it > SPIN_LIMIT) {
          atomicExch(a.ctl + 1, 1);
          atomicAdd(a.ctl + 2, 1);
          atomicOr(a.err, PBG_DEV_ERR_BARRIER);
          atomicCAS(a.info, 0, -1);  // -1: the factorisation gave up waiting
          ok = 0;
          break;
        }
        __nanosleep(it < 64 ? 20 : 200);
      }
    }
    *s_ok = ok;
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

// ---------------------------------------------------------------- tile GEMM
// Accumulator layout: 16 elements per thread; warp w owns rows 16*(w/2).. and
// columns 32*(w%2).. of the 64 x 64 tile.  acc_coord gives element e's place.
template <typename T> struct TileMMA;

template <> struct TileMMA<double> {
  // mma.m8n8k4 f64: 2 m-tiles x 4 n-tiles of 8 x 8, 2 accumulators each.
  static __device__ __forceinline__ void coord(int e, int& r, int& c) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int mt = e >> 3, nt = (e >> 1) & 3, h = e & 1;
    r = 16 * (w >> 1) + 8 * mt + (lane >> 2);
    c = 32 * (w & 1) + 8 * nt + 2 * (lane & 3) + h;
  }
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
  static __device__ __forceinline__ void coord(int e, int& r, int& c) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nt = e >> 2, q = e & 3;
    r = 16 * (w >> 1) + (lane >> 2) + 8 * (q >> 1);
    c = 32 * (w & 1) + 8 * nt + 2 * (lane & 3) + (q & 1);
  }
  static __device__ __forceinline__ void sub(const float* sA, const float* sB, float acc[16]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1), g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int k0 = 0; k0 < NB; k0 += 8) {
      // split the (negated) A fragment and the B fragments into tf32 hi + lo
      unsigned ah[4], al[4];
      {
        const float v[4] = {-sA[(m0 + g) * LDA + k0 + t], -sA[(m0 + g + 8) * LDA + k0 + t],
                            -sA[(m0 + g) * LDA + k0 + t + 4], -sA[(m0 + g + 8) * LDA + k0 + t + 4]};
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
        float* c = acc + 4 * nt;
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
  }
};

template <typename T>
__device__ __forceinline__ void load_acc(const T* g, int ld, T acc[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    int r, c;
    TileMMA<T>::coord(e, r, c);
    acc[e] = ldcg(g + (size_t)r * ld + c);
  }
}

template <typename T>
__device__ __forceinline__ void store_acc(T* g, int ld, const T acc[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    int r, c;
    TileMMA<T>::coord(e, r, c);
    g[(size_t)r * ld + c] = acc[e];
  }
}

// Apply update U(i, j, k) to acc (tile (i, j) already in acc).
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
// Factor the 64 x 64 tile held in acc (already fully updated) in T arithmetic.
// The tile stays in the accumulator registers for all eight 8-column panels:
// the owners of panel p copy its column strip to shared memory, warp 0 factors
// it (register chain, rsqrt pivots) and inverts its 8 x 8 diagonal block,
// then every thread takes the final panel values back and applies the rank-8
// update to its own trailing elements.  Two CTA barriers per panel.
template <typename T>
__device__ __forceinline__ T rsqrt_t(T x);
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

constexpr int PB = 8;  // panel strip row length

template <typename T>
__device__ __forceinline__ void factor_tile(const DFArgs& a, int k, T acc[16], unsigned char* smem) {
  T* P = reinterpret_cast<T*>(smem);  // [64][PB] current panel strip
  T* X = P + NB * PB;                 // [8][8][8] inverted diagonal 8 x 8 blocks
  T* Rinv = X + 8 * 64;               // [8] 1 / L_jj of the current panel
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // element coordinates are recomputed where needed (keeping 32 of them live
  // in registers made the FP64 build spill)
#pragma unroll 1
  for (int p = 0; p < 8; ++p) {
    const int c0 = 8 * p;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      int r, c;
      TileMMA<T>::coord(e, r, c);
      if (c >= c0 && c < c0 + 8 && r >= c0) P[r * PB + c - c0] = acc[e];
    }
    __syncthreads();
    if (warp == 0) {
      const int r0 = c0 + lane, r1 = c0 + 32 + lane;
      const bool v0 = r0 < NB, v1 = r1 < NB;
      T p0[8], p1[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        p0[c] = v0 ? P[r0 * PB + c] : T(0);
        p1[c] = v1 ? P[r1 * PB + c] : T(0);
      }
      // Branch-free chain: every lane takes the pivot by shuffle and computes
      // its rsqrt; a non-positive pivot is only recorded here and reported
      // after the panel (a branch holding an atomic inside the unrolled chain
      // slows it several-fold).
      int bad = -1;
      // 1 / L_jj goes to Rinv for the 8 x 8 block inverse
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const T d = __shfl_sync(0xffffffffu, p0[j], j);
        if (!(d > T(0)) && bad < 0) bad = j;
        const T rs = rsqrt_t<T>(d);
        if (lane == 0) Rinv[j] = rs;
        p0[j] = lane == j ? d * rs : (lane > j ? p0[j] * rs : p0[j]);  // L_jj = sqrt(d)
        p1[j] *= rs;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (c > j) {
            const T lc = __shfl_sync(0xffffffffu, p0[j], c);
            if (lane >= c) p0[c] -= p0[j] * lc;
            p1[c] -= p1[j] * lc;
          }
        }
      }
      if (lane == 0 && bad >= 0 && k * NB + c0 + bad < a.n) atomicCAS(a.info, 0, k * NB + c0 + bad + 1);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (v0) P[r0 * PB + c] = c <= lane ? p0[c] : T(0);
        if (v1) P[r1 * PB + c] = p1[c];
      }
      __syncwarp();
      // inverse of the 8 x 8 diagonal block: lane c < 8 owns column c
      if (lane < 8) {
        T x[8];
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
          T sacc = 0;
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (q < ii && q >= lane) sacc += P[(c0 + ii) * PB + q] * x[q];
          x[ii] = ii < lane ? T(0) : (ii == lane ? Rinv[ii] : -sacc * Rinv[ii]);
        }
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) X[p * 64 + ii * 8 + lane] = x[ii];
      }
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      int r, c;
      TileMMA<T>::coord(e, r, c);
      if (c >= c0 && c < c0 + 8) {
        if (r >= c0) acc[e] = P[r * PB + c - c0];
      } else if (c >= c0 + 8 && r >= c) {
        T s0 = 0, s1 = 0;
#pragma unroll
        for (int q = 0; q < 8; q += 2) {
          s0 += P[r * PB + q] * P[c * PB + q];
          s1 += P[r * PB + q + 1] * P[c * PB + q + 1];
        }
        acc[e] -= s0 + s1;
      }
    }
    // the next panel's strip is written only after everyone has read this one
    __syncthreads();
  }
  T* g = tile<T>(a, k, k);
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    int r, c;
    TileMMA<T>::coord(e, r, c);
    g[(size_t)r * a.ld + c] = c <= r ? acc[e] : T(0);
  }
  T* li = reinterpret_cast<T*>(a.leafinv) + (size_t)k * 8 * 64;
  for (int t = tid; t < 8 * 64; t += THREADS) li[t] = X[t];
}

// ---------------------------------------------------------------- S(i, k)
// acc holds the updated A_ik; computes L_ik = A_ik L_kk^-T in T arithmetic by
// 8-column blocks: X_b = (A_b - sum_{b'<b} X_b' L_bb'^T) inv(L_bb)^T.
// Row r belongs to the four threads 4r .. 4r+3 (two columns of each block),
// so rows proceed independently with warp-level syncs only.
constexpr int LDW = NB + 4;

template <typename T>
__device__ __forceinline__ void solve_tile(const DFArgs& a, int i, int k, const T acc[16], unsigned char* smem) {
  T* C = reinterpret_cast<T*>(smem);  // [64][LDW] rhs, becomes X
  T* Lk = C + NB * LDW;               // [64][LDW] L_kk
  T* Inv = Lk + NB * LDW;             // [8][8][8]
  T* W = Inv + 8 * 64;                // [64][9]
  const int tid = threadIdx.x;
  stage_async(tile<T>(a, k, k), a.ld, Lk, LDW);
  {
    const T* li = reinterpret_cast<const T*>(a.leafinv) + (size_t)k * 8 * 64;
    constexpr int chunks = 8 * 64 * (int)sizeof(T) / 16;
    constexpr int elems = 16 / (int)sizeof(T);
    for (int t = tid; t < chunks; t += THREADS) cp_async16(Inv + t * elems, li + t * elems);
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    int r, c;
    TileMMA<T>::coord(e, r, c);
    C[r * LDW + c] = acc[e];
  }
  cp_async_wait_all();
  __syncthreads();
  const int r = tid >> 2, q2 = 2 * (tid & 3);
  // block loop kept rolled: the kernel's code footprint matters more than
  // the loop overhead (the persistent kernel runs every task type)
#pragma unroll 1
  for (int b = 0; b < 8; ++b) {
    const int o = 8 * b;
    T u0 = 0, u1 = 0, v0 = 0, v1 = 0;
#pragma unroll 4
    for (int j = 0; j < o; j += 2) {
      const T x0 = C[r * LDW + j], x1 = C[r * LDW + j + 1];
      u0 += x0 * Lk[(o + q2) * LDW + j];
      v0 += x1 * Lk[(o + q2) * LDW + j + 1];
      u1 += x0 * Lk[(o + q2 + 1) * LDW + j];
      v1 += x1 * Lk[(o + q2 + 1) * LDW + j + 1];
    }
    W[r * 9 + q2] = C[r * LDW + o + q2] - (u0 + v0);
    W[r * 9 + q2 + 1] = C[r * LDW + o + q2 + 1] - (u1 + v1);
    __syncwarp();
    T s0 = 0, s1 = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const T wq = W[r * 9 + q];
      s0 += wq * Inv[b * 64 + q2 * 8 + q];  // inv is lower: zero above the diagonal
      s1 += wq * Inv[b * 64 + (q2 + 1) * 8 + q];
    }
    C[r * LDW + o + q2] = s0;
    C[r * LDW + o + q2 + 1] = s1;
    __syncwarp();
  }
  __syncthreads();
  T* g = tile<T>(a, i, k);
  for (int t = tid; t < NB * NB; t += THREADS) {
    const int rr = t >> 6, c = t & 63;
    g[(size_t)rr * a.ld + c] = C[rr * LDW + c];
  }
}

// Inverse of every diagonal factor tile (one CTA per tile), from L_kk and the
// inverted 8 x 8 blocks: X_ab = -inv(L_aa) sum_{c=b}^{a-1} L_ac X_cb by block
// distance.  Needed only by the SPD inverse and the midpoint triangular solve.
template <typename T>
__global__ void __launch_bounds__(THREADS) diag_inverse_kernel(const T* __restrict__ A, int ld,
                                                               const T* __restrict__ leafinv,
                                                               T* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* L = reinterpret_cast<T*>(smem_raw);  // [64][LDT]
  T* X = L + NB * LDT;                    // [64][LDT]
  T* Tm = X + NB * LDT;                   // [7][8][9]
  const int k = blockIdx.x, tid = threadIdx.x;
  const T* g = A + (size_t)k * NB * ld + (size_t)k * NB;
  for (int t = tid; t < NB * NB; t += THREADS) {
    const int r = t >> 6, c = t & 63;
    L[r * LDT + c] = g[(size_t)r * ld + c];
    X[r * LDT + c] = T(0);
  }
  __syncthreads();
  const T* li = leafinv + (size_t)k * 8 * 64;
  for (int t = tid; t < 8 * 64; t += THREADS) {
    const int b = t >> 6, r = (t >> 3) & 7, c = t & 7;
    X[(8 * b + r) * LDT + 8 * b + c] = li[t];
  }
  __syncthreads();
  for (int d = 1; d < 8; ++d) {
    const int nblk = 8 - d;
    for (int t = tid; t < nblk * 64; t += THREADS) {
      const int b = t >> 6, r = (t >> 3) & 7, c = t & 7, aa = b + d;
      T s0 = 0;
      for (int q = 8 * b; q < 8 * aa; ++q) s0 += L[(8 * aa + r) * LDT + q] * X[q * LDT + 8 * b + c];
      Tm[b * 72 + r * 9 + c] = s0;
    }
    __syncthreads();
    for (int t = tid; t < nblk * 64; t += THREADS) {
      const int b = t >> 6, r = (t >> 3) & 7, c = t & 7, aa = b + d;
      T v = 0;
      for (int q = 0; q <= r; ++q) v -= X[(8 * aa + r) * LDT + 8 * aa + q] * Tm[b * 72 + q * 9 + c];
      X[(8 * aa + r) * LDT + 8 * b + c] = v;
    }
    __syncthreads();
  }
  T* o = out + (size_t)k * NB * NB;
  for (int t = tid; t < NB * NB; t += THREADS) o[t] = X[(t >> 6) * LDT + (t & 63)];
}

template <typename T>
__global__ void __launch_bounds__(THREADS, 2) chol_df_kernel(DFArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_task, s_ok;
  T* sA = reinterpret_cast<T*>(smem);
  T* sB = sA + NB * LDA;
  const int nt = a.nt;
  // Block 0 is the chain CTA: it runs, in order, every diagonal factorisation
  // F(k) and the solve S(k+1, k) that gates F(k+1), so that code stays warm in
  // one SM and the chain has no inter-CTA hand-off.  The other CTAs take the
  // remaining tasks from the shared counter, in list order.
  const bool chain = blockIdx.x == 0;
  int chain_step = 0;
  while (true) {
    int t, type, i, j, k;
    if (chain) {
      if (chain_step >= 2 * nt - 1) return;
      const int kk = chain_step >> 1;
      if (chain_step & 1) { type = TASK_S; i = kk + 1; j = k = kk; }
      else { type = TASK_F; i = j = k = kk; }
      t = a.ntasks + chain_step;  // trace slot after the shared tasks
      ++chain_step;
      if (threadIdx.x == 0 && ld_acquire(a.ctl + 1)) s_task = -1;
      else if (threadIdx.x == 0) s_task = 0;
      __syncthreads();
      if (s_task < 0) return;
      __syncthreads();
    } else {
      if (threadIdx.x == 0) s_task = ld_acquire(a.ctl + 1) ? a.ntasks : atomicAdd(a.ctl, 1);
      __syncthreads();
      t = s_task;
      __syncthreads();
      if (t >= a.ntasks) return;
      const int4 tk = a.tasks[t];
      type = tk.x; i = tk.y; j = tk.z; k = tk.w;
    }
    TRACE(0, t);
    TRACE(3, t);
    T acc[16];
    if (type == TASK_U) {
      // U(i, j, k): needs L_ik, L_jk final and the k previous updates of (i, j)
      const int* fl[3] = {a.fin + i * nt + k, a.fin + j * nt + k, a.upd + i * nt + j};
      const int tg[3] = {1, 1, k};
      if (!wait_all(a, fl, tg, 3, &s_ok)) return;
      TRACE(1, t);
      load_and_update(a, i, j, k, acc, sA, sB);
      store_acc(tile<T>(a, i, j), a.ld, acc);
      publish(a.upd + i * nt + j, k + 1);
      TRACE(2, t);
    } else {
      // F(j) (i == j) or S(i, j): the tile in column j, after its last update
      const int col = j;
      if (col > 0) {
        const int* fl[3] = {a.fin + i * nt + col - 1, a.fin + col * nt + col - 1, a.upd + i * nt + col};
        const int tg[3] = {1, 1, col - 1};
        if (!wait_all(a, fl, tg, 3, &s_ok)) return;
        load_and_update(a, i, col, col - 1, acc, sA, sB);
      } else {
        load_acc(tile<T>(a, i, col), a.ld, acc);
      }
      if (type == TASK_F) {
        TRACE(1, t);
        factor_tile<T>(a, col, acc, smem);
      } else {
        if (!wait_geq(a, a.fin + col * nt + col, 1, &s_ok)) return;
        TRACE(1, t);
        solve_tile<T>(a, i, col, acc, smem);
      }
      publish(a.fin + i * nt + col, 1);
      TRACE(2, t);
    }
    __syncthreads();
  }
}

std::mutex g_task_mu;
std::map<int, std::pair<int4*, int>> g_task_tables;

// Task list of an nt x nt tile grid (see the file comment).
int get_task_table(int nt, const int4** out, int* count) {
  std::lock_guard<std::mutex> lk(g_task_mu);
  auto it = g_task_tables.find(nt);
  if (it != g_task_tables.end()) {
    *out = it->second.first;
    *count = it->second.second;
    return PBG_OK;
  }
  // The chain tasks F(k) and S(k+1, k) run on the chain CTA and are left out.
  std::vector<int4> t;
  for (int i = 2; i < nt; ++i) t.push_back(make_int4(TASK_S, i, 0, 0));
  for (int k = 0; k + 1 < nt; ++k) {
    for (int i = k + 3; i < nt; ++i) t.push_back(make_int4(TASK_S, i, k + 1, k + 1));
    // column k+1 of the update with panel k is fused into F(k+1) / S(., k+1);
    // the plain updates cover columns >= k+2, the one gating the next panel first
    for (int jj = k + 2; jj < nt; ++jj)
      for (int i = jj; i < nt; ++i) t.push_back(make_int4(TASK_U, i, jj, k));
  }
  int4* d = nullptr;
  if (cudaMalloc(&d, t.size() * sizeof(int4)) != cudaSuccess) {
    cudaGetLastError();
    return PBG_ERR_NOMEM;
  }
  PBG_CUDA_TRY(cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice));
  g_task_tables[nt] = std::make_pair(d, (int)t.size());
  *out = d;
  *count = (int)t.size();
  return PBG_OK;
}

template <typename T>
size_t df_smem_bytes() {
  const size_t gemm = 2 * sizeof(T) * NB * LDA;
  const size_t fac = sizeof(T) * (NB * PB + 8 * 64 + 8);
  const size_t sol = sizeof(T) * (2 * NB * LDW + 8 * 64 + NB * 9);
  size_t m = gemm > fac ? gemm : fac;
  return m > sol ? m : sol;
}

template <typename T>
int launch_df(T* A, int n, int ld, int* info, void* leafinv, int* ints, unsigned* err, cudaStream_t st) {
  const int nt = ld / NB;
  const int4* tasks = nullptr;
  int ntasks = 0;
  int rc = get_task_table(nt, &tasks, &ntasks);
  if (rc) return rc;
  const size_t smem = df_smem_bytes<T>();
  static int max_blocks_per_sm = -1;
  static int num_sms = 0;
  if (max_blocks_per_sm < 0) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(chol_df_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev;
    PBG_CUDA_TRY(cudaGetDevice(&dev));
    PBG_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    PBG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_blocks_per_sm, chol_df_kernel<T>, THREADS, smem));
    if (max_blocks_per_sm < 1) {
      pbg_set_error_message("cholesky kernel does not fit on an SM");
      return PBG_ERR_CUDA;
    }
  }
  int grid = num_sms * max_blocks_per_sm;
  if (grid > ntasks + 1) grid = ntasks + 1;  // the chain CTA plus the shared tasks
  PBG_CUDA_TRY(cudaMemsetAsync(ints, 0, (3 + 2 * (size_t)nt * nt) * sizeof(int), st));
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
  args.info = info;
  args.leafinv = leafinv;
  args.err = err;
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
  PBG_CUDA_TRY(cudaLaunchKernelEx(&cfg, chol_df_kernel<T>, args));
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace

#ifdef PBG_TASK_TRACE
extern "C" __attribute__((visibility("default"))) int pbg_task_trace(long long* host, int ntasks) {
  PBG_CUDA_TRY(cudaMemcpyFromSymbol(host, g_task_trace, sizeof(long long) * 4 * ntasks));
  return PBG_OK;
}
#endif

// Scratch of one factorisation: leaf inverses, task counter, abort flag,
// per-tile flags, error word.
size_t df_work_bytes(int ld) {
  const int nt = ld / NB;
  return (size_t)nt * 8 * 64 * sizeof(double) + (3 + 2 * (size_t)nt * nt + 1) * sizeof(int) + 64;
}

// Factors A in place.  With invdiag non-null, the inverse of every diagonal
// factor tile is then written there (nt x 64 x 64, precision of A).
int launch_cholesky_df(void* A, int n, int ld, int precision, int* info, void* invdiag, void* work,
                       cudaStream_t st) {
  const int nt = ld / NB;
  unsigned char* w = static_cast<unsigned char*>(work);
  void* leafinv = w;
  int* ints = reinterpret_cast<int*>(w + (size_t)nt * 8 * 64 * sizeof(double));
  unsigned* err = reinterpret_cast<unsigned*>(ints + 3 + 2 * (size_t)nt * nt);
  int rc = precision == PBG_PREC_FP64 ? launch_df<double>((double*)A, n, ld, info, leafinv, ints, err, st)
                                      : launch_df<float>((float*)A, n, ld, info, leafinv, ints, err, st);
  if (rc != PBG_OK || !invdiag) return rc;
  const size_t smem = (precision == PBG_PREC_FP64 ? 8 : 4) * (2 * NB * LDT + 7 * 72);
  if (precision == PBG_PREC_FP64) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(diag_inverse_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    diag_inverse_kernel<double><<<nt, THREADS, smem, st>>>((const double*)A, ld, (const double*)leafinv, (double*)invdiag);
  } else {
    PBG_CUDA_TRY(cudaFuncSetAttribute(diag_inverse_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    diag_inverse_kernel<float><<<nt, THREADS, smem, st>>>((const float*)A, ld, (const float*)leafinv, (float*)invdiag);
  }
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
