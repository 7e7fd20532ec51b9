// Tensor-core complex GEMM update C -= A B (tcgen05, 3xTF32 or split-FP16); layout and
// scheme in tc_gemm.cuh.  Used by the mixed-precision dense LU (dense_lu_tc.cu) for its trailing
// updates, the only O(N^3) work of the direct solve.
#include <cuda_fp16.h>

#include "sie_internal.h"
#include "tc_gemm.cuh"

namespace sie {
namespace tc {

// Largest |re| and |im| of an operand region: cols columns of len contiguous elements at
// stride ld, folded into *out (the bits of a non-negative float order like the float).
__global__ void __launch_bounds__(256) k_absmax(const float* __restrict__ sr, const float* __restrict__ si,
                                                size_t ld, int len, int cols, unsigned* out) {
  __shared__ float red[8];
  float m = 0.f;
  for (int c = blockIdx.y; c < cols; c += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
      const size_t o = (size_t)c * ld + i;
      m = fmaxf(m, fmaxf(fabsf(sr[o]), fabsf(si[o])));
    }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
    atomicMax(out, __float_as_uint(m));
  }
}

// the power-of-two exponent e with amax = f 2^e, f in [0.5, 1): the operand is scaled by
// 2^(F16_TOP - e)
__device__ __forceinline__ int f16_exponent(const unsigned* amax) {
  int e = 0;
  frexpf(__uint_as_float(*amax), &e);
  return e;
}

// Pre-tiles rows [0, rows) x K [0, K) of an operand into blocks [tile][chunk] (layout in
// tc_gemm.cuh), splitting each value into its tf32 pair (H = false, chunks of KC = 8) or,
// scaled by 2^(F16_TOP - e) with e from *amax, its f16 pair (H = true, chunks of KC_F16 =
// 16); rows and K past the operand are zero.  Element (r, k) is src[k * ld + r]
// (column-major, the A operand: r a row of C) or, with trans, src[r * ld + k] (the B
// operand read from a column-major K x n matrix: r a column of C).  Grid: (TILE * kc / 256,
// chunks, tiles), 256 threads.
template <bool H>
__global__ void __launch_bounds__(256) k_tile(const float* __restrict__ sr, const float* __restrict__ si,
                                              size_t ld, int rows, int K, int trans, int nchunks,
                                              const unsigned* amax, char* __restrict__ out) {
  constexpr int kc = H ? KC_F16 : KC;
  const int c = blockIdx.y, t = blockIdx.z;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // element of the block
  int r, k;
  if (trans) {  // consecutive threads read consecutive k (contiguous in src)
    k = e % kc;
    r = e / kc;
  } else {
    r = e % TILE;
    k = e / TILE;
  }
  const int gr = t * TILE + r, gk = c * kc + k;
  float vr = 0.f, vi = 0.f;
  if (gr < rows && gk < K) {
    const size_t o = trans ? (size_t)gr * ld + gk : (size_t)gk * ld + gr;
    vr = sr[o];
    vi = si[o];
  }
  char* blkbase = out + ((size_t)t * nchunks + c) * BLOCK_BYTES;
  if (H) {
    const float sc = ldexpf(1.f, F16_TOP - f16_exponent(amax));
    vr *= sc;
    vi *= sc;
    const __half rh = __float2half_rn(vr), ih = __float2half_rn(vi);
    const __half rl = __float2half_rn(vr - __half2float(rh));
    const __half il = __float2half_rn(vi - __half2float(ih));
    char* blk = blkbase + plane_offset_f16(r, k);
    *(__half*)(blk) = rh;
    *(__half*)(blk + PLANE_BYTES) = rl;
    *(__half*)(blk + 2 * PLANE_BYTES) = ih;
    *(__half*)(blk + 3 * PLANE_BYTES) = il;
  } else {
    float rh, rl, ih, il;
    tf32_split(vr, rh, rl);
    tf32_split(vi, ih, il);
    char* blk = blkbase + plane_offset(r, k);
    *(float*)(blk) = rh;
    *(float*)(blk + PLANE_BYTES) = rl;
    *(float*)(blk + 2 * PLANE_BYTES) = ih;
    *(float*)(blk + 3 * PLANE_BYTES) = il;
  }
}

// C tile (mt, nt) -= A tile row mt times B tile row nt.  Persistent: CTA b takes tiles b,
// b + gridDim.x, ...; the stage ring's phases run on across tiles (chunk counter g), the
// done barrier flips once per tile, and a CTA barrier after each epilogue frees the
// accumulators before the next tile's first MMA.
__device__ __forceinline__ void tile_coords(int tile, int m, int n, int& mt, int& nt) {
  // groups of GROUP_M row tiles, each swept across the column tiles, so the CTAs in flight
  // share a few A and B tiles in L2 (a row-tile-fastest order would cycle every A tile of
  // the operand through L2 for each column tile)
  const int tm = (m + TILE - 1) / TILE, tn = (n + TILE - 1) / TILE;
  const int per = GROUP_M * tn;
  const int g = tile / per, r = tile - g * per;
  const int gm = min(GROUP_M, tm - g * GROUP_M);
  nt = r / gm;
  mt = g * GROUP_M + (r - nt * gm);
}

template <bool H>
__global__ void __launch_bounds__(256, 2) k_gemm(const char* __restrict__ At, const char* __restrict__ Bt,
                                                 int nchunks, float* __restrict__ Cr, float* __restrict__ Ci,
                                                 size_t ldc, int m, int n, const unsigned* amax, int* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
  uint64_t* full = (uint64_t*)(sm + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tslot = (uint32_t*)(done + 1);
  __shared__ int fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = ((m + TILE - 1) / TILE) * ((n + TILE - 1) / TILE);
  if (threadIdx.x == 0) {
    fail = 0;
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    // 256 columns: the real accumulator in 0..127, the imaginary one in 128..255
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  int it = 0;
  unsigned g0 = 0;  // chunks of the earlier tiles of this CTA
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++, g0 += nchunks) {
    int mt, nt;
    tile_coords(tile, m, n, mt, nt);
    if (!fail && warp == 0 && lane == 0) {
      // producer: one A block and one B block per stage
      const char* a0 = At + (size_t)mt * nchunks * BLOCK_BYTES;
      const char* b0 = Bt + (size_t)nt * nchunks * BLOCK_BYTES;
      for (int c = 0; c < nchunks; c++) {
        const unsigned g = g0 + c;
        const int s = g % STAGES;
        if (g >= STAGES && !mbar_wait(&empty[s], ((g / STAGES) - 1) & 1)) {
          atomicOr(err, 1);
          fail = 1;
          break;
        }
        unsigned char* st = sm + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        bulk_g2s(st, a0 + (size_t)c * BLOCK_BYTES, BLOCK_BYTES, &full[s]);
        bulk_g2s(st + BLOCK_BYTES, b0 + (size_t)c * BLOCK_BYTES, BLOCK_BYTES, &full[s]);
      }
    } else if (!fail && warp == 1 && lane == 0) {
      // MMA issuer
      const uint32_t idp = H ? idesc_f16(false) : idesc_tf32(false);
      const uint32_t idn = H ? idesc_f16(true) : idesc_tf32(true);
      // one MMA (K = 8 tf32 or 16 f16) per pair of planes of a stage
      auto mma = [&](uint32_t d, uint64_t a, uint64_t b, uint32_t id, bool acc) {
        if (H)
          mma_f16(d, a, b, id, acc);
        else
          mma_tf32(d, a, b, id, acc);
      };
      const uint32_t dr = tmem, di = tmem + TILE;
      bool first = true;
      for (int c = 0; c < nchunks; c++) {
        const unsigned g = g0 + c;
        const int s = g % STAGES;
        if (!mbar_wait(&full[s], (g / STAGES) & 1)) {
          atomicOr(err, 2);
          fail = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t sa = smem_u32(sm + s * STAGE_BYTES), sb = sa + BLOCK_BYTES;
        {
          const uint64_t arh = smem_desc(sa), arl = smem_desc(sa + PLANE_BYTES);
          const uint64_t aih = smem_desc(sa + 2 * PLANE_BYTES), ail = smem_desc(sa + 3 * PLANE_BYTES);
          const uint64_t brh = smem_desc(sb), brl = smem_desc(sb + PLANE_BYTES);
          const uint64_t bih = smem_desc(sb + 2 * PLANE_BYTES), bil = smem_desc(sb + 3 * PLANE_BYTES);
          // Re += Ar Br - Ai Bi
          mma(dr, arh, brh, idp, !first);
          mma(dr, arh, brl, idp, true);
          mma(dr, arl, brh, idp, true);
          mma(dr, aih, bih, idn, true);
          mma(dr, aih, bil, idn, true);
          mma(dr, ail, bih, idn, true);
          // Im += Ar Bi + Ai Br
          mma(di, arh, bih, idp, !first);
          mma(di, arh, bil, idp, true);
          mma(di, arl, bih, idp, true);
          mma(di, aih, brh, idp, true);
          mma(di, aih, brl, idp, true);
          mma(di, ail, brh, idp, true);
          first = false;
        }
        mma_commit(&empty[s]);
      }
      // arrives once every MMA issued above has completed
      mma_commit(done);
    }
    __syncwarp();
    const bool ok = mbar_wait(done, it & 1);
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok) atomicOr(err, 4);
    __syncthreads();
    if (ok && !fail) {
      // the f16 operands were scaled by powers of two: undo it exactly
      const float inv = H ? ldexpf(1.f, f16_exponent(amax) + f16_exponent(amax + 1) - 2 * F16_TOP) : 1.f;
      // eight warps: warp w reads TMEM lanes 32 (w % 4) .. (its rows of C) for the column
      // half w / 4, so twice the loads are in flight
      const int wl = warp & 3, half = warp >> 2;
      const int row = mt * TILE + wl * 32 + lane;
      const uint32_t lane_base = tmem + ((uint32_t)(wl * 32) << 16);
#pragma unroll 1
      for (int j0 = half * (TILE / 2); j0 < (half + 1) * (TILE / 2); j0 += 16) {
        uint32_t vr[16], vi[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]),
              "=r"(vr[7]), "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]),
              "=r"(vr[14]), "=r"(vr[15])
            : "r"(lane_base + j0));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]),
              "=r"(vi[7]), "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]),
              "=r"(vi[14]), "=r"(vi[15])
            : "r"(lane_base + TILE + j0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < m) {
          // 16 loads of C first, then their stores: independent requests in flight
          const int ncol = min(16, n - (nt * TILE + j0));
          float* pr = Cr + (size_t)(nt * TILE + j0) * ldc + row;
          float* pi = Ci + (size_t)(nt * TILE + j0) * ldc + row;
#pragma unroll
          for (int h = 0; h < 16; h += 8) {
            float cr[8], ci[8];
#pragma unroll
            for (int j = 0; j < 8; j++)
              if (h + j < ncol) {
                cr[j] = pr[(size_t)(h + j) * ldc];
                ci[j] = pi[(size_t)(h + j) * ldc];
              }
#pragma unroll
            for (int j = 0; j < 8; j++)
              if (h + j < ncol) {
                pr[(size_t)(h + j) * ldc] = cr[j] - __uint_as_float(vr[h + j]) * inv;
                pi[(size_t)(h + j) * ldc] = ci[j] - __uint_as_float(vi[h + j]) * inv;
              }
          }
        }
      }
    }
    // every warp has read its accumulators before the next tile's MMAs overwrite them
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (fail || !ok) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem));
}

// Host side: number of 128-row tiles and K chunks of an operand (8 K per tf32 chunk, 16
// per f16 chunk).
inline int tiles(int rows) { return (rows + TILE - 1) / TILE; }
inline int chunks(int K, bool f16) {
  const int kc = f16 ? KC_F16 : KC;
  return (K + kc - 1) / kc;
}
inline size_t tiled_bytes(int rows, int K, bool f16) { return (size_t)tiles(rows) * chunks(K, f16) * BLOCK_BYTES; }

// the larger of the two layouts (the tf32 one)
size_t tiled_bytes_host(int rows, int K) { return tiled_bytes(rows, K, false); }

// Tiles an operand.  With f16, *amax (zeroed here) first receives the operand's largest
// magnitude, from which the tiling and the GEMM take its scale; amax[0] belongs to A and
// amax[1] to B of the update that follows.
int tile_operand(const float* sr, const float* si, size_t ld, int rows, int K, bool trans, char* out,
                 cudaStream_t st, bool f16, unsigned* amax) {
  if (f16) {
    SIE_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned), st));
    const int len = trans ? K : rows, cols = trans ? rows : K;
    dim3 ga((len + 255) / 256 < 8 ? (len + 255) / 256 : 8, cols < 1024 ? cols : 1024);
    k_absmax<<<ga, 256, 0, st>>>(sr, si, ld, len, cols, amax);
    count_launch();
    dim3 g(TILE * KC_F16 / 256, chunks(K, true), tiles(rows));
    k_tile<true><<<g, 256, 0, st>>>(sr, si, ld, rows, K, trans ? 1 : 0, chunks(K, true), amax, out);
  } else {
    dim3 g(TILE * KC / 256, chunks(K, false), tiles(rows));
    k_tile<false><<<g, 256, 0, st>>>(sr, si, ld, rows, K, trans ? 1 : 0, chunks(K, false), amax, out);
  }
  count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// C (m x n, planes Cr / Ci, leading dimension ldc) -= A B from pre-tiled operands, on at
// most max_ctas persistent CTAs (0: one per tile); amax: the operands' maxima (f16).
int gemm_update(const char* At, const char* Bt, int K, float* Cr, float* Ci, size_t ldc, int m, int n,
                int* d_err, cudaStream_t st, int max_ctas, bool f16, const unsigned* amax) {
  long long nt = (long long)tiles(m) * tiles(n);
  if (nt > 2147483647LL) return fail(SIE_ERR_ARG, "tensor-core update: too many tiles");
  if (max_ctas > 0 && nt > max_ctas) nt = max_ctas;
  if (f16) {
    SIE_CUDA(raise_smem(k_gemm<true>, SMEM_BYTES));
    k_gemm<true><<<(unsigned)nt, 256, SMEM_BYTES, st>>>(At, Bt, chunks(K, true), Cr, Ci, ldc, m, n, amax, d_err);
  } else {
    SIE_CUDA(raise_smem(k_gemm<false>, SMEM_BYTES));
    k_gemm<false><<<(unsigned)nt, 256, SMEM_BYTES, st>>>(At, Bt, chunks(K, false), Cr, Ci, ldc, m, n, amax, d_err);
  }
  count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

}  // namespace tc
}  // namespace sie
