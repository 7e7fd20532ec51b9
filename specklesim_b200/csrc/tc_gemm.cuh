// Complex GEMM update on the 5th-generation tensor cores (tcgen05, sm_100a):
//
//     C -= A B        A: m x K, B: K x n, C: m x n, complex
//
// C is complex64 stored as two real planes (Cr, Ci), column-major.  The operands are
// split into pairs x = hi + lo and every complex product is formed from the three products
// hi*hi + hi*lo + lo*hi of each real product: Cr -= Ar Br - Ai Bi, Ci -= Ar Bi + Ai Br,
// accumulated in FP32 in tensor memory.  Two splits:
//   3xTF32 (kind::tf32): hi rounded to tf32, lo the exact remainder; ~2^-21 relative,
//     FP32-level; 8 K per MMA.
//   split-FP16 (kind::f16, both operands f16): each operand scaled by a power of two s
//     that puts its largest magnitude below 2^14, hi = f16(s x), lo = f16(s x - hi), the
//     accumulator multiplied back by 1 / (s_A s_B), exact; hi and lo keep 11 bits each, so
//     the products are as accurate as 3xTF32 relative to the operands' largest entries, and
//     an MMA takes 16 K at the same issue rate: twice the tf32 throughput.
//
// Operands are pre-tiled in global memory in the shape the MMA reads from shared memory,
// so each pipeline stage is one contiguous bulk (TMA) copy:
//   block (tile t of 128 rows, K chunk c of 8): 4 planes (re hi, re lo, im hi, im lo),
//   each 128 rows x 8 tf32 in the K-major no-swizzle canonical layout: core matrices of
//   8 rows x 16 bytes (4 tf32), core (k/4, r/8) at byte ((k/4) * 16 + r/8) * 128, row r%8
//   at +16 (r%8), element k%4 at +4 (k%4).  LBO (next 4 k) = 2048 B, SBO (next 8 rows) =
//   128 B.  One block = 16 KB; blocks ordered [tile][chunk].
// A's rows are C's rows (M); B is tiled by C's columns (the MMA's N rows), K-major too.
//
// Kernel: one CTA (8 warps) per 128 x 128 tile of C, two CTAs per SM so that one's
// epilogue overlaps the other's MMAs.  Warp 0 lane 0 issues the bulk copies into a
// 3-stage ring (32 KB per stage: one A block, one B block); warp 1 lane 0 issues the MMAs
// (M = 128, N = 128, K = 8, 12 per stage) and commits each stage back to the
// producer; then all four warps read the accumulators (warp w owns TMEM lanes 32w..32w+31
// = rows of C) and subtract them from C.  Every wait on an mbarrier is bounded: a wait
// that runs out sets *err and the CTA skips the rest of its work, waiting (also bounded)
// for its own MMAs before it frees tensor memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sie {
namespace tc {

constexpr int TILE = 128;                 // rows of an operand tile; C tile is TILE x TILE
constexpr int KC = 8;                     // K per pipeline stage (one MMA of K = 8)
constexpr int PLANE_BYTES = TILE * KC * 4;  // 4 KB
constexpr int BLOCK_BYTES = 4 * PLANE_BYTES;  // 16 KB: re hi, re lo, im hi, im lo
constexpr int STAGES = 3;
constexpr int STAGE_BYTES = 2 * BLOCK_BYTES;  // A block + B block
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + barriers, alignment slack: 97 KB,
                                                         // two CTAs per SM (TMEM 2 x 256 columns)
constexpr unsigned WAIT_LIMIT = 1u << 26;   // polls of one mbarrier before giving up
constexpr int GROUP_M = 16;               // row tiles swept together across the column tiles

// byte offset of element (r, k) inside one plane of a block
__host__ __device__ __forceinline__ int plane_offset(int r, int k) {
  return (((k >> 2) * 16 + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 3) << 2);
}
// the same for the f16 planes: a block covers KC_F16 = 16 K; core matrices of 8 rows x
// 16 bytes (8 f16), so the byte layout, LBO and SBO are those of the tf32 planes
constexpr int KC_F16 = 16;
constexpr int F16_TOP = 14;  // scaled operands stay below 2^14 (f16 overflows at 65504)
__host__ __device__ __forceinline__ int plane_offset_f16(int r, int k) {
  return (((k >> 3) * 16 + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1);
}

// hi = x rounded to tf32 (low 13 mantissa bits zero), lo = x - hi exactly
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  const unsigned u = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
  hi = __uint_as_float(u);
  lo = x - hi;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// true once the phase with the given parity has completed; false after WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned i = 0; i < WAIT_LIMIT; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle, LBO 2048 B, SBO 128 B
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(2048 >> 4) << 16) | ((uint64_t)(128 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = 128, A negated
__host__ __device__ constexpr uint32_t idesc_tf32(bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(TILE >> 3) << 17) |
         ((uint32_t)(TILE >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate ? 1u : 0u));
}
// instruction descriptor for kind::f16: D f32, A and B f16, both K-major, M = N = 128
__host__ __device__ constexpr uint32_t idesc_f16(bool neg_a) {
  return (1u << 4) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(TILE >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate ? 1u : 0u));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

}  // namespace tc
}  // namespace sie
