// 3xTF32 tile products on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// P = A B^T for 64 x 64 FP32 tiles: A is one or two stacked row tiles (an
// M = 128 operand), B one tile (N = 64), K = 64.  Each FP32 operand is split
// as x = hi + lo with hi = rna_tf32(x) and lo = rna_tf32(x - hi), and
//   P = A_hi B_hi + A_hi B_lo + A_lo B_hi
// accumulates in FP32 in tensor memory (TMEM), from zero.  The operands are
// written by the CTA's threads into shared memory in the canonical K-major
// 128-byte-swizzle layout; one thread issues the MMAs and commits them to an
// mbarrier; the accumulator is read back with tcgen05.ld by the four warps
// whose TMEM lane quarters hold its rows.
//
// Shared-memory layout of one K-major operand of R rows (R = 64 or 128) and
// K = 64 FP32: two K blocks (k 0..31, 32..63) of R rows x 128 bytes; row r of
// a block starts at (r / 8) * 1024 + (r % 8) * 128 and its 16-byte chunk c
// (k = 4c .. 4c+3 within the block) sits at chunk c ^ (r % 8).  Each block
// starts 1024-byte aligned.  The MMA for k-step s (8 elements, 32 bytes)
// reads block s / 4 from byte 32 (s % 4) of each row: its descriptor's start
// address advances by 32 bytes inside the swizzle atom.
#pragma once
#include <cstdint>

namespace pbg {
namespace tc {

constexpr int TILE = 64;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t rna_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity to complete: false after
// `limit` polls (each try_wait itself blocks for a bounded, hardware-chosen time).
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

// ---------------------------------------------------------------- TMEM
// Warp-wide (all 32 lanes of one warp): allocate `cols` columns (a power of
// two >= 32) and write the TMEM address to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor cores' reads.
__device__ __forceinline__ void fence_proxy_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 32 columns of FP32 from TMEM (lane quarter of the calling warp).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// ---------------------------------------------------------------- descriptors
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address, bits 0-13
  d |= (uint64_t)1 << 16;                              // leading byte offset (unused for this layout): 16 B
  d |= (uint64_t)(1024 >> 4) << 32;                    // stride byte offset: 1024 B
  d |= (uint64_t)1 << 46;                              // descriptor version 1
  d |= (uint64_t)2 << 61;                              // layout: 128-byte swizzle
  return d;
}
// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

// ---------------------------------------------------------------- operands
// Byte offset of (row r, 16-byte chunk c of K, c = 0..15) in a K-major
// swizzled operand of R rows.
__device__ __forceinline__ uint32_t sw128_offset(int R, int r, int c) {
  const int kb = c >> 3, cc = c & 7;
  return (uint32_t)(kb * R * 128 + (r >> 3) * 1024 + (r & 7) * 128 + ((cc ^ (r & 7)) << 4));
}

// Bytes of the hi and lo halves of an R-row operand.
__host__ __device__ constexpr uint32_t operand_bytes(int R) { return (uint32_t)R * TILE * 4; }

// One 64 x 64 FP32 source tile and where its TF32 halves go: rows
// row0 .. row0 + 63 of the R-row operands at hi and lo.
struct SplitTile {
  const float* src;
  int R, row0;
  unsigned char* hi;
  unsigned char* lo;
};

// One thread's share of a 64 x 64 FP32 tile: PER 16-byte chunks, chunk e at
// row (tid + e NTHREADS) / 16, columns 4 ((tid + e NTHREADS) % 16) .. +3.
template <int NTHREADS>
struct TileShare {
  static constexpr int PER = TILE * 16 / NTHREADS;
  float4 v[PER];
};

// Issues the loads of this thread's share (through L2; no wait).
template <int NTHREADS>
__device__ __forceinline__ void load_share(const float* src, int ld, TileShare<NTHREADS>& s) {
#pragma unroll
  for (int e = 0; e < TileShare<NTHREADS>::PER; ++e) {
    const int i = threadIdx.x + e * NTHREADS, r = i >> 4, c = i & 15;
    s.v[e] = __ldcg(reinterpret_cast<const float4*>(src + (size_t)r * ld + 4 * c));
  }
}

// Writes the hi / lo TF32 halves of this thread's share into rows
// row0 .. row0 + 63 of the R-row K-major operands at hi and lo.
template <int NTHREADS>
__device__ __forceinline__ void store_share_split(const TileShare<NTHREADS>& s, int R, int row0, unsigned char* hi,
                                                  unsigned char* lo) {
#pragma unroll
  for (int e = 0; e < TileShare<NTHREADS>::PER; ++e) {
    const int i = threadIdx.x + e * NTHREADS, r = row0 + (i >> 4), c = i & 15;
    const uint32_t off = sw128_offset(R, r, c);
    const float x[4] = {s.v[e].x, s.v[e].y, s.v[e].z, s.v[e].w};
    uint32_t h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      h[u] = rna_tf32(x[u]);
      l[u] = rna_tf32(x[u] - __uint_as_float(h[u]));
    }
    *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// Writes the hi / lo TF32 halves of four FP32 values (one 16-byte chunk) at
// byte offset off of the hi and lo operands.
__device__ __forceinline__ void store_split_chunk(float4 x4, uint32_t off, unsigned char* hi, unsigned char* lo) {
  const float x[4] = {x4.x, x4.y, x4.z, x4.w};
  uint32_t h[4], l[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    h[u] = rna_tf32(x[u]);
    l[u] = rna_tf32(x[u] - __uint_as_float(h[u]));
  }
  *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// Loads up to MAXT 64 x 64 FP32 tiles (row stride ld) and writes their hi /
// lo TF32 halves into the operands: every thread issues all of its loads
// (16 bytes each, through L2) before the first conversion, so the tiles cost
// one memory round trip together.  All NTHREADS threads of the CTA call it.
template <int NTHREADS, int MAXT>
__device__ __forceinline__ void split_tiles_all(const SplitTile (&t)[MAXT], int count, int ld) {
  TileShare<NTHREADS> v[MAXT];
#pragma unroll
  for (int q = 0; q < MAXT; ++q)
    if (q < count) load_share<NTHREADS>(t[q].src, ld, v[q]);
#pragma unroll
  for (int q = 0; q < MAXT; ++q)
    if (q < count) store_share_split<NTHREADS>(v[q], t[q].R, t[q].row0, t[q].hi, t[q].lo);
}

// Issues P = A_hi B_hi + A_hi B_lo + A_lo B_hi (M = 128, N = 64, K = 64) into
// the TMEM accumulator d_tmem: from zero, or added to it with accumulate = 1.
// One thread.
__device__ __forceinline__ void issue_product(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                              uint32_t b_lo, uint32_t accumulate = 0) {
  constexpr uint32_t idesc = idesc_tf32(128, 64);
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint32_t ka = (uint32_t)((s >> 2) * 128 * 128 + (s & 3) * 32);  // A: 128 rows per K block
    const uint32_t kb = (uint32_t)((s >> 2) * 64 * 128 + (s & 3) * 32);   // B: 64 rows per K block
    mma_tf32(d_tmem, sw128_desc(a_hi + ka), sw128_desc(b_hi + kb), idesc, s > 0 ? 1u : accumulate);
    mma_tf32(d_tmem, sw128_desc(a_hi + ka), sw128_desc(b_lo + kb), idesc, 1u);
    mma_tf32(d_tmem, sw128_desc(a_lo + ka), sw128_desc(b_hi + kb), idesc, 1u);
  }
}

}  // namespace tc
}  // namespace pbg
