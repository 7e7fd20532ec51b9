// Mixed-precision direct solve of the dense system: LU with partial pivoting of the
// complex64 matrix, its O(N^3) trailing updates on the tensor cores (tc_gemm.cu: split-FP16
// products with power-of-two operand scaling, or 3xTF32), then iterative refinement in
// FP64 against the FP64 dense product.
//
// The reference's direct path (lib_sie_tri_solver_normal_I,
// src/lib_sie_tri_solver_normal.f90:64-217, with ZGESV in solver_LU,
// src/lib_sie_math.f90:649-676) factorises the FP64 matrix; sie_solve_direct does the
// same with cuSOLVER.  Here the factorisation runs in FP32 arithmetic and the solution is
// refined in FP64 (x += U^-1 L^-1 P (b - Z x)) until the true backward error meets the
// tolerance, which it does while cond(Z) times the factorisation's rounding stays below
// one.
//
// Blocked right-looking LU, panel width 512 (256 with SIE_LU_NB=256), on the matrix
// stored as two FP32 planes (real, imaginary), column-major, internal unknown order:
//   1. panel, in 64-column blocks of 8-column sub-panels: each sub-panel is one
//      cooperative launch that, column by column, agrees on the pivot (one bounded grid
//      barrier per column), moves the pivot row, scales the column and updates the
//      sub-panel; then its row swaps for the panel's other columns, its U
//      rows and a rank-8 update of its block's later columns; after each block, its U
//      rows of the panel's later columns and one tensor-core update of those columns;
//   2. the panel's row swaps applied to every column left and right of it;
//   3. U12 = L11^-1 A12 in 256-row halves, each an in-place tensor-core update with
//      M = I - L11^-1 of the half's diagonal block;
//   4. A22 -= L21 U12 on the tensor cores: first the next panel's columns, then, on a
//      second (low-priority) stream, the rest, which runs beside the next panel (look-ahead).
#include <chrono>
#include <cmath>
#include <vector>

#include "sie_internal.h"
#include "tc_gemm.cuh"

namespace sie {
namespace tc {
int tile_operand(const float* sr, const float* si, size_t ld, int rows, int K, bool trans, char* out,
                 cudaStream_t st, bool f16, unsigned* amax);
int gemm_update(const char* At, const char* Bt, int K, float* Cr, float* Ci, size_t ldc, int m, int n,
                int* d_err, cudaStream_t st, int max_ctas, bool f16, const unsigned* amax);
size_t tiled_bytes_host(int rows, int K);
}  // namespace tc

static const int LU_NB = 256;  // the narrower panel width (SIE_LU_NB=256); L11 blocks of U12
static const int LU_NBX = 512;  // the default panel width (the trailing updates' K)
// sub-panel width inside a panel: each column step of the panel kernel streams the
// sub-panel's remaining columns through L2, so narrower sub-panels move fewer bytes per
// column (slab10 factorisation 2.23 s with 8 against 2.35 s with 16)
static const int LU_SB = 8;
static const int LU_TB = 128;  // diagonal blocks of the triangular solves
// multiprocessors the look-ahead update leaves to the panels: the panel chain is the
// factorisation's critical path, and its sub-panel kernel, which streams the sub-panel
// through L2 once per column, speeds up with more of them (slab10: 2.37-2.40 s with 24
// against 2.43-2.45 s with 12, 2.41-2.42 s with 36)
static const int LU_FREE_SMS = 24;
static const int PANEL_MAX_BLOCKS = 256;  // largest grid of the cooperative panel kernel

// Dense panels (cfg.dense = 1) -> FP32 planes of Z in the internal interleaved order
// (unknown 2m + a of edge m), column-major.
__global__ void k_expand_dense32(const long long* base, const int* box_first, const int* box_cnt,
                                 const int* ncols, int nbox, const zc* va, const zc* vb, const zc* vd, zc cfac,
                                 int M, float* Zr, float* Zi) {
  const long long ld = 2LL * M;
  for (int A = blockIdx.y; A < nbox; A += gridDim.y) {
    const int nr = box_cnt[A], nc = ncols[A], f = box_first[A];
    const long long tot = (long long)nr * nc;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tot;
         k += (long long)gridDim.x * blockDim.x) {
      const int r = (int)(k / nc), j = (int)(k % nc);
      const long long o = base[A] + k;
      const long long m = f + r, n = j;
      const zc a = va[o], b = vb[o], d = vd[o], c = cfac * b;
      const long long p00 = (2 * n) * ld + 2 * m, p01 = (2 * n + 1) * ld + 2 * m;
      Zr[p00] = (float)a.re;
      Zi[p00] = (float)a.im;
      Zr[p01] = (float)b.re;
      Zi[p01] = (float)b.im;
      Zr[p00 + 1] = (float)c.re;
      Zi[p00 + 1] = (float)c.im;
      Zr[p01 + 1] = (float)d.re;
      Zi[p01 + 1] = (float)d.im;
    }
  }
}

// Pivot comparison: larger |a|^2 first, the smaller row index on ties (the first maximum,
// as izamax).
__device__ __forceinline__ void argmax_pair(float& best, int& bi, float ov, int oi) {
  if (ov > best || (ov == best && oi < bi)) {
    best = ov;
    bi = oi;
  }
}

// Per-block slot of the panel kernel's pivot search: the block's largest |a|^2 in the
// column being searched, its row, and that row's values in the sub-panel's columns from
// the searched column on (the pivot row, if it wins).
struct PanelSlot {
  float mx;
  int ix;
  float2 row[LU_SB];
};
// the panel scratch: error word, two generations of slots, then one barrier counter per
// sub-panel launch and the barrier's give-up flag
static const size_t PANEL_SLOTS_OFF = 256;
static const size_t PANEL_CNT_OFF = PANEL_SLOTS_OFF + 2 * PANEL_MAX_BLOCKS * sizeof(PanelSlot);
static size_t panel_cnt_bytes(int n) { return ((size_t)n / LU_SB + 2) * sizeof(unsigned); }
// then the swap plan of the latest panel: {count, src[2 LU_NBX], dst[2 LU_NBX]}
static size_t panel_plan_off(int n) { return (PANEL_CNT_OFF + panel_cnt_bytes(n) + 255) / 256 * 256; }
// and the operand maxima of the split-FP16 updates (the trailing ones, then the panel's own)
static size_t panel_amax_off(int n) { return (panel_plan_off(n) + (1 + 4 * LU_NBX) * sizeof(int) + 15) / 16 * 16; }
static size_t panel_scratch_bytes(int n) { return panel_amax_off(n) + 4 * sizeof(unsigned); }

// Grid barrier of the cooperative sub-panel kernel (all its blocks are resident) on a
// counter that only grows within one launch: the m-th barrier waits for m * gridDim.x
// arrivals.  The wait is bounded: a block that sees no progress for about a second sets
// *bad and stops waiting; later barriers then pass straight through, and the host reports
// the error.
__device__ __forceinline__ void panel_bar(unsigned* cnt, unsigned* bad, unsigned target) {
  __syncthreads();
  if (threadIdx.x == 0) {
    // release: the block's writes (ordered before by the CTA barrier) are visible to any
    // block that acquires the count
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
    volatile unsigned* vb = bad;
    long long it = 0;
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
      if (v >= target || *vb != 0) break;
      if (++it > (1LL << 21)) {
        atomicExch(bad, 1u);
        break;
      }
    }
  }
  __syncthreads();
}

// Block-wide argmax of (value, row) pairs (ties to the smaller row); returns the winner to
// every thread, and whether the calling thread holds it (the lowest such thread).
__device__ __forceinline__ void block_argmax(float v, int i, float* sv, int* si, int* st, float& bv, int& bi,
                                             bool& mine, int* winner = nullptr) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  float best = v;
  int idx = i, who = threadIdx.x;
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o), ow = __shfl_xor_sync(0xffffffffu, who, o);
    if (ov > best || (ov == best && (oi < idx || (oi == idx && ow < who)))) {
      best = ov;
      idx = oi;
      who = ow;
    }
  }
  if (l == 0) {
    sv[w] = best;
    si[w] = idx;
    st[w] = who;
  }
  __syncthreads();
  best = sv[0];
  idx = si[0];
  who = st[0];
  for (int k = 1; k < (int)(blockDim.x >> 5); k++)
    if (sv[k] > best || (sv[k] == best && (si[k] < idx || (si[k] == idx && st[k] < who)))) {
      best = sv[k];
      idx = si[k];
      who = st[k];
    }
  __syncthreads();  // sv/si/st are reused by the next call
  bv = best;
  bi = idx;
  mine = who == (int)threadIdx.x;
  if (winner) *winner = who;
}

// One sub-panel [s0, s1) of the panel [k0, k1) factorised by one cooperative launch, one
// grid barrier per column.  Before the barrier that ends column j - 1, every block has
// published its candidate for column j in slots[gen]: the largest |a|^2 among its rows and
// that row's values in columns [j, s1).  After it, every block reduces the slots to the
// same pivot p (the first maximum, as izamax) and takes the pivot row from the winning
// slot, so nobody reads row p from the matrix.  Row j and row p trade places logically in
// the sub-panel's columns: the thread that owns row p reads the old row j, writes the
// pivot row into row j and the updated old row j into row p, and swaps the two rows' L
// values in the columns [s0, j).  Their values in the panel's other columns are swapped
// after the launch (k_sub_finish), as nothing here reads them.  Each row r > j is then scaled and updated, and the block's best candidate
// for column j + 1 goes to the other generation of slots: every thread keeps the values of
// its best row in shared memory, so the winner's row is published without a reload.
// Matrix and slot reads bypass L1 (__ldcg): other blocks' writes are seen through L2.
__global__ void __launch_bounds__(256, 4) k_subpanel(float* Ar, float* Ai, size_t ld, int n, int s0, int s1, int k0,
                                                     int k1, int* ipiv, int* err, PanelSlot* slots, unsigned* cnt,
                                                     unsigned* bad) {
  __shared__ float sv[8];
  __shared__ int si[8], st[8];
  __shared__ float2 urow[LU_SB];
  __shared__ float2 cand[LU_SB - 1][256];  // each thread's best row, columns j + 1 .. s1 - 1
  __shared__ int piv_s, win_s;
  const unsigned G = gridDim.x;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = G * blockDim.x;
  unsigned nbar = 0;
  // publish the block's candidate (row bi, of the column c) into slot generation gen
  auto publish = [&](float best, int bi, int c, int gen) {
    float bv;
    int brow;
    bool mine;
    block_argmax(best, bi, sv, si, st, bv, brow, mine);
    PanelSlot* sl = slots + (size_t)gen * PANEL_MAX_BLOCKS + blockIdx.x;
    if (mine) {
      sl->mx = bv;
      sl->ix = brow;
      if (brow < n)  // the winner wrote this row itself: its own writes are visible to it
        for (int k = 0; k < s1 - c; k++)
          sl->row[k] = make_float2(__ldcg(Ar + (size_t)(c + k) * ld + brow), __ldcg(Ai + (size_t)(c + k) * ld + brow));
    }
  };
  {  // candidates of the first column
    float best = -1.f;
    int bi = n;
    for (int r = s0 + gtid; r < n; r += gstride) {
      const float a = __ldcg(Ar + (size_t)s0 * ld + r), b = __ldcg(Ai + (size_t)s0 * ld + r);
      argmax_pair(best, bi, a * a + b * b, r);
    }
    publish(best, bi, s0, 0);
  }
  panel_bar(cnt, bad, ++nbar * G);
  for (int j = s0; j < s1; j++) {
    const int gen = (j - s0) & 1, wj = s1 - j;
    // the pivot: every block reduces the same slots in the same way
    {
      const PanelSlot* sl = slots + (size_t)gen * PANEL_MAX_BLOCKS;
      float v = -1.f;
      int i = n;
      if (threadIdx.x < G) {
        v = __ldcg(&sl[threadIdx.x].mx);
        i = __ldcg(&sl[threadIdx.x].ix);
      }
      float bv;
      int bi;
      bool mine;
      block_argmax(v, i, sv, si, st, bv, bi, mine);
      if (mine) win_s = threadIdx.x;  // the winning block
      __syncthreads();
      const int wb = win_s;
      if (threadIdx.x < wj) {
        const float2* rw = &sl[wb].row[threadIdx.x];
        urow[threadIdx.x] = make_float2(__ldcg(&rw->x), __ldcg(&rw->y));
      }
      if (threadIdx.x == 0) {
        piv_s = bi;
        if (blockIdx.x == 0) {
          ipiv[j] = bi;
          if (!(bv > 0.f) || !isfinite(bv) || bi >= n) atomicOr(err, 8);  // singular or non-finite
        }
      }
      __syncthreads();
    }
    const int p = piv_s < n ? piv_s : j;
    const float2 pv = urow[0];
    const float den = pv.x * pv.x + pv.y * pv.y;
    float best = -1.f;
    int bi = n;
    for (int r = j + 1 + gtid; r < n; r += gstride) {
      const int src = r == p ? j : r;  // logical row r lives in physical row j until now
      float xr[LU_SB], xi[LU_SB];
#pragma unroll
      for (int k = 0; k < LU_SB; k++)
        if (k < wj) {
          const size_t o = (size_t)(j + k) * ld + src;
          xr[k] = __ldcg(Ar + o);
          xi[k] = __ldcg(Ai + o);
        }
      if (r == p) {  // row j becomes the pivot row
#pragma unroll
        for (int k = 0; k < LU_SB; k++)
          if (k < wj) {
            const size_t o = (size_t)(j + k) * ld + j;
            Ar[o] = urow[k].x;
            Ai[o] = urow[k].y;
          }
      }
      const float lr = (xr[0] * pv.x + xi[0] * pv.y) / den, li = (xi[0] * pv.x - xr[0] * pv.y) / den;
      Ar[(size_t)j * ld + r] = lr;
      Ai[(size_t)j * ld + r] = li;
#pragma unroll
      for (int k = 1; k < LU_SB; k++)
        if (k < wj) {
          const float ur = urow[k].x, ui = urow[k].y;
          xr[k] -= lr * ur - li * ui;
          xi[k] -= lr * ui + li * ur;
          const size_t o = (size_t)(j + k) * ld + r;
          Ar[o] = xr[k];
          Ai[o] = xi[k];
        }
      if (wj > 1) {
        const float v = xr[1] * xr[1] + xi[1] * xi[1];
        if (v > best || (v == best && r < bi)) {
          best = v;
          bi = r;
#pragma unroll
          for (int k = 1; k < LU_SB; k++)
            if (k < wj) cand[k - 1][threadIdx.x] = make_float2(xr[k], xi[k]);
        }
      }
      if (r == p) {  // rows j and p also trade their L values in the columns [s0, j), in
                     // two halves whose loads are issued together
#pragma unroll
        for (int h = 0; h < LU_SB; h += LU_SB / 2) {
          float er[LU_SB / 2], ei[LU_SB / 2], fr[LU_SB / 2], fi[LU_SB / 2];
#pragma unroll
          for (int k = 0; k < LU_SB / 2; k++)
            if (s0 + h + k < j) {
              er[k] = __ldcg(Ar + (size_t)(s0 + h + k) * ld + j);
              ei[k] = __ldcg(Ai + (size_t)(s0 + h + k) * ld + j);
              fr[k] = __ldcg(Ar + (size_t)(s0 + h + k) * ld + p);
              fi[k] = __ldcg(Ai + (size_t)(s0 + h + k) * ld + p);
            }
#pragma unroll
          for (int k = 0; k < LU_SB / 2; k++)
            if (s0 + h + k < j) {
              Ar[(size_t)(s0 + h + k) * ld + j] = fr[k];
              Ai[(size_t)(s0 + h + k) * ld + j] = fi[k];
              Ar[(size_t)(s0 + h + k) * ld + p] = er[k];
              Ai[(size_t)(s0 + h + k) * ld + p] = ei[k];
            }
        }
      }
    }
    if (j + 1 < s1) {
      float bv;
      int brow, who;
      bool mine;
      block_argmax(best, bi, sv, si, st, bv, brow, mine, &who);
      PanelSlot* sl = slots + (size_t)(gen ^ 1) * PANEL_MAX_BLOCKS + blockIdx.x;
      if (threadIdx.x == 0) {
        sl->mx = bv;
        sl->ix = brow;
      }
      if (brow < n && (int)threadIdx.x < wj - 1) sl->row[threadIdx.x] = cand[threadIdx.x][who];
      panel_bar(cnt, bad, ++nbar * G);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && __ldcg(bad) != 0) atomicOr(err, 16);  // a barrier gave up
}


__device__ __forceinline__ void ll_put(unsigned long long* p, unsigned tag, unsigned bits) {
  const unsigned long long w = ((unsigned long long)tag << 32) | bits;
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long ll_ld(const unsigned long long* p) {
  unsigned long long w;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}
// The payload of *p once it carries tag (w: a first load of it).  Bounded: after about
// two million reloads without the tag, or once another thread gave up, it sets *bad and
// returns whatever it holds; the host reports the error.
__device__ __forceinline__ unsigned ll_wait(const unsigned long long* p, unsigned long long w, unsigned tag,
                                            unsigned* bad) {
  long long it = 0;
  while ((unsigned)(w >> 32) != tag) {
    if ((++it & 63) == 0) {
      if (*(volatile unsigned*)bad != 0) break;
      if (it > (1LL << 21)) {
        atomicExch(bad, 1u);
        break;
      }
    }
    w = ll_ld(p);
  }
  return (unsigned)w;
}

// After the sub-panel [s0, s1) of the panel [k0, k1): its row interchanges applied, in
// order, to the panel's columns outside the sub-panel (the sub-panel's own columns were
// swapped by k_subpanel), then its rows of the later columns of its 64-column block
// [s1, uend), U = L11^-1 A (L11 the unit lower triangle of the sub-panel's diagonal
// block).  A thread per panel column, LU_FIN_T columns per block: the rows the swaps reach
// (the sub-panel's rows and the pivot rows below it, at most 2 LU_SB) are loaded together
// into shared memory, swapped there and written back.  No block writes the sub-panel's
// columns, so every block reads L11 from memory without waiting on the others.
static const int LU_FIN_T = 64;
__global__ void __launch_bounds__(LU_FIN_T) k_sub_finish(float* Ar, float* Ai, size_t ld, int k0, int s0, int s1,
                                                         int k1, int uend, const int* ipiv) {
  __shared__ int pv[LU_SB], slot[LU_SB], first[LU_SB], srow[2 * LU_SB];
  __shared__ int nslot;
  __shared__ float2 vals[2 * LU_SB][LU_FIN_T];
  __shared__ float2 L11[LU_SB][LU_SB];  // [column t][row i]
  const int w = s1 - s0, tid = threadIdx.x;
  if (tid < w) pv[tid] = ipiv[s0 + tid];
  __syncthreads();
  // slots 0 .. w - 1: rows s0 .. s1 - 1; then each distinct pivot row below s1, in order of
  // its first appearance (thread j finds pivot j's slot)
  if (tid < w) {
    const int p = pv[tid];
    int f = tid;
    if (p >= s1)
      for (int j = 0; j < tid; j++)
        if (pv[j] == p) {
          f = j;
          break;
        }
    first[tid] = f;
  }
  __syncthreads();
  if (tid < w) {
    const int p = pv[tid];
    if (p < s1) {
      slot[tid] = p - s0;
    } else {
      int rank = 0;  // first appearances below s1 before this pivot's
      for (int j = 0; j < first[tid]; j++) rank += (pv[j] >= s1 && first[j] == j) ? 1 : 0;
      slot[tid] = w + rank;
      if (first[tid] == tid) srow[w + rank] = p;
    }
    srow[tid] = s0 + tid;
  }
  if (tid == 0) {
    int cnt = 0;
    for (int j = 0; j < w; j++) cnt += (pv[j] >= s1 && first[j] == j) ? 1 : 0;
    nslot = w + cnt;
  }
  __syncthreads();
  const int ns = nslot;
  const int c = k0 + blockIdx.x * LU_FIN_T + tid;
  if (c < k1 && (c < s0 || c >= s1)) {
#pragma unroll
    for (int q = 0; q < 2 * LU_SB; q++)
      if (q < ns) vals[q][tid] = make_float2(Ar[(size_t)c * ld + srow[q]], Ai[(size_t)c * ld + srow[q]]);
    for (int j = 0; j < w; j++) {
      const int q = slot[j];
      if (q != j) {
        const float2 t = vals[j][tid];
        vals[j][tid] = vals[q][tid];
        vals[q][tid] = t;
      }
    }
#pragma unroll
    for (int q = 0; q < 2 * LU_SB; q++)
      if (q < ns) {
        Ar[(size_t)c * ld + srow[q]] = vals[q][tid].x;
        Ai[(size_t)c * ld + srow[q]] = vals[q][tid].y;
      }
  }
  // U rows of the block's columns in [s1, uend)
  const int cb0 = k0 + blockIdx.x * LU_FIN_T;
  if (s1 >= uend || cb0 + LU_FIN_T <= s1 || cb0 >= uend) return;  // uniform over the block
  for (int e = tid; e < w * w; e += blockDim.x) {
    const int t = e / w, i = e - t * w;
    L11[t][i] = make_float2(Ar[(size_t)(s0 + t) * ld + s0 + i], Ai[(size_t)(s0 + t) * ld + s0 + i]);
  }
  __syncthreads();
  if (c < s1 || c >= uend) return;
  float xr[LU_SB], xi[LU_SB];
#pragma unroll
  for (int i = 0; i < LU_SB; i++) {  // rows s0 .. s1 - 1 of column c, after the swaps above
    xr[i] = i < w ? vals[i][tid].x : 0.f;
    xi[i] = i < w ? vals[i][tid].y : 0.f;
  }
#pragma unroll
  for (int i = 1; i < LU_SB; i++)
#pragma unroll
    for (int t = 0; t < i; t++) {
      const float lr = t < w && i < w ? L11[t][i].x : 0.f, li = t < w && i < w ? L11[t][i].y : 0.f;
      xr[i] -= lr * xr[t] - li * xi[t];
      xi[i] -= lr * xi[t] + li * xr[t];
    }
#pragma unroll
  for (int i = 1; i < LU_SB; i++)
    if (i < w) {
      Ar[(size_t)c * ld + s0 + i] = xr[i];
      Ai[(size_t)c * ld + s0 + i] = xi[i];
    }
}

// U rows [b0, b1) of the panel's columns [c0, c1): x = L^-1 x with L the unit lower
// triangle of the 64-column block's diagonal (b1 - b0 <= LU_BB).  A block per LU_BB
// columns, a thread per column; L and the columns in shared memory (dynamic, 64 KB).
static const int LU_BB = 64;
__global__ void __launch_bounds__(LU_BB) k_blk_trsm(float* Ar, float* Ai, size_t ld, int b0, int b1, int c0,
                                                    int c1) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float2(*L)[LU_BB] = reinterpret_cast<float2(*)[LU_BB]>(smraw);                      // [col t][row i]
  float2(*X)[LU_BB] = reinterpret_cast<float2(*)[LU_BB]>(smraw + LU_BB * LU_BB * 8);  // [row i][thread]
  const int w = b1 - b0, t = threadIdx.x;
  for (int e0 = t; e0 < w * w; e0 += 8 * LU_BB) {
    float2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int e = e0 + q * LU_BB, col = e / w, row = e - col * w;
      v[q] = e < w * w ? make_float2(Ar[(size_t)(b0 + col) * ld + b0 + row], Ai[(size_t)(b0 + col) * ld + b0 + row])
                       : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int e = e0 + q * LU_BB, col = e / w, row = e - col * w;
      if (e < w * w) L[col][row] = v[q];
    }
  }
  const int c = c0 + blockIdx.x * LU_BB + t;
  const bool live = c < c1;
  for (int i0 = 0; i0 < w; i0 += 16) {
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++)
      v[q] = live && i0 + q < w ? make_float2(Ar[(size_t)c * ld + b0 + i0 + q], Ai[(size_t)c * ld + b0 + i0 + q])
                                : make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 16; q++)
      if (i0 + q < w) X[i0 + q][t] = v[q];
  }
  __syncthreads();
  if (!live) return;
  for (int i = 1; i < w; i++) {
    float2 x = X[i][t];
    for (int k = 0; k < i; k++) {
      const float2 l = L[k][i], y = X[k][t];
      x.x -= l.x * y.x - l.y * y.y;
      x.y -= l.x * y.y + l.y * y.x;
    }
    X[i][t] = x;
    Ar[(size_t)c * ld + b0 + i] = x.x;
    Ai[(size_t)c * ld + b0 + i] = x.y;
  }
}

// Rank-w update of the later columns of the sub-panel's 64-column block by a factored
// sub-panel [s0, s1): a_rc -= sum_t l_rt u_tc for rows r >= s1 and columns c in [s1, uend).  The sub-panel's U
// rows in shared memory; thread per row, its w L values in registers, the columns in
// groups of 8 whose loads are issued together.
static const int LU_UPD_CG = 8;
static const int LU_UPD_SLICE = 64;  // columns per block of the grid's second dimension
__global__ void __launch_bounds__(256, 2) k_sub_update(float* Ar, float* Ai, size_t ld, int n, int s0, int s1,
                                                    int uend) {
  __shared__ float ur[LU_SB][LU_NB], ui[LU_SB][LU_NB];
  const int w = s1 - s0, nc = uend - s1;
  for (int e0 = threadIdx.x; e0 < LU_SB * LU_NB; e0 += 4 * blockDim.x) {
    float vr[4], vi[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = e0 + q * blockDim.x, t = e / LU_NB, c = e - t * LU_NB;
      const bool in = e < LU_SB * LU_NB && t < w && c < nc;
      vr[q] = in ? Ar[(size_t)(s1 + c) * ld + s0 + t] : 0.f;
      vi[q] = in ? Ai[(size_t)(s1 + c) * ld + s0 + t] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = e0 + q * blockDim.x, t = e / LU_NB, c = e - t * LU_NB;
      if (e < LU_SB * LU_NB) {
        ur[t][c] = vr[q];
        ui[t][c] = vi[q];
      }
    }
  }
  __syncthreads();
  const int r = s1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float lr[LU_SB], li[LU_SB];
#pragma unroll
  for (int t = 0; t < LU_SB; t++) {
    lr[t] = t < w ? Ar[(size_t)(s0 + t) * ld + r] : 0.f;
    li[t] = t < w ? Ai[(size_t)(s0 + t) * ld + r] : 0.f;
  }
  // this block's slice of LU_UPD_SLICE columns
  const int cend = min(nc, (int)(blockIdx.y + 1) * LU_UPD_SLICE);
#pragma unroll 1
  for (int c0 = blockIdx.y * LU_UPD_SLICE; c0 < cend; c0 += LU_UPD_CG) {
    float cr[LU_UPD_CG], ci[LU_UPD_CG];
#pragma unroll
    for (int g = 0; g < LU_UPD_CG; g++) {
      const size_t o = (size_t)(s1 + c0 + g) * ld + r;
      cr[g] = c0 + g < cend ? Ar[o] : 0.f;
      ci[g] = c0 + g < cend ? Ai[o] : 0.f;
    }
#pragma unroll
    for (int t = 0; t < LU_SB; t++) {  // rows t >= w of ur/ui are zero
      const float l_r = lr[t], l_i = li[t];
#pragma unroll
      for (int g = 0; g < LU_UPD_CG; g++) {
        const float a = ur[t][c0 + g], b = ui[t][c0 + g];
        cr[g] -= l_r * a - l_i * b;
        ci[g] -= l_r * b + l_i * a;
      }
    }
#pragma unroll
    for (int g = 0; g < LU_UPD_CG; g++)
      if (c0 + g < cend) {
        const size_t o = (size_t)(s1 + c0 + g) * ld + r;
        Ar[o] = cr[g];
        Ai[o] = ci[g];
      }
  }
}

// The row swaps ipiv[k0 .. k1) of one panel (applied in order, as LAPACK's laswp) as one
// gather: after them, row dst[i] holds the old row src[i], for the nb positions of the
// panel and the rows outside it that the swaps reach (at most nb more).  One block; the
// swaps are followed in order, the lookup of a row outside the panel searched by all
// threads.  plan = {count, src[2 LU_NBX], dst[2 LU_NBX]}.
__global__ void __launch_bounds__(256) k_swap_plan(const int* ipiv, int k0, int k1, int* plan) {
  __shared__ int pos[2 * LU_NBX], cont[2 * LU_NBX], ip[LU_NBX];
  __shared__ int nx, found;
  const int nb = k1 - k0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    pos[i] = cont[i] = k0 + i;
    ip[i] = ipiv[k0 + i];
  }
  if (threadIdx.x == 0) nx = 0;
  __syncthreads();
  for (int j = 0; j < nb; j++) {
    const int p = ip[j];
    if (p == k0 + j) continue;  // uniform: every thread reads the same ip[j]
    int idx = p - k0;
    if (p >= k1) {
      if (threadIdx.x == 0) found = -1;
      __syncthreads();
      for (int t = threadIdx.x; t < nx; t += blockDim.x)
        if (pos[nb + t] == p) found = nb + t;
      __syncthreads();
      if (threadIdx.x == 0 && found < 0) {
        pos[nb + nx] = cont[nb + nx] = p;
        found = nb + nx;
        nx++;
      }
      __syncthreads();
      idx = found;
    }
    if (threadIdx.x == 0) {
      const int t = cont[j];
      cont[j] = cont[idx];
      cont[idx] = t;
    }
    __syncthreads();
  }
  const int cnt = nb + nx;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    plan[1 + i] = cont[i];
    plan[1 + 2 * LU_NBX + i] = pos[i];
  }
  if (threadIdx.x == 0) plan[0] = cnt;
}

// The plan applied to every column outside the panel [k0, k1): a block per tile of
// LU_SWAP_TC columns, a thread per plan entry; all of a tile's reads happen before any
// of its writes.
static const int LU_SWAP_TC = 8;
__global__ void __launch_bounds__(2 * LU_NBX) k_swap_apply(float* Ar, float* Ai, size_t ld, int n, int k0, int k1,
                                                    const int* plan) {
  const int cnt = plan[0];
  const int i = threadIdx.x;
  const int outside = n - (k1 - k0);
  int src = 0, dst = 0;
  if (i < cnt) {
    src = plan[1 + i];
    dst = plan[1 + 2 * LU_NBX + i];
  }
  float vr[LU_SWAP_TC], vi[LU_SWAP_TC];
  const int c0 = blockIdx.x * LU_SWAP_TC;
#pragma unroll
  for (int t = 0; t < LU_SWAP_TC; t++) {
    int c = c0 + t;
    vr[t] = vi[t] = 0.f;
    if (i < cnt && c < outside) {
      if (c >= k0) c += k1 - k0;
      vr[t] = Ar[(size_t)c * ld + src];
      vi[t] = Ai[(size_t)c * ld + src];
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < LU_SWAP_TC; t++) {
    int c = c0 + t;
    if (i < cnt && c < outside) {
      if (c >= k0) c += k1 - k0;
      Ar[(size_t)c * ld + dst] = vr[t];
      Ai[(size_t)c * ld + dst] = vi[t];
    }
  }
}

// Copies the nb x nb diagonal block at (k0, k0) of the two planes into shared memory
// ([col][row], leading dimension LU_TB), eight loads in flight per thread.
__device__ __forceinline__ void stage_block(const float* Ar, const float* Ai, size_t ld, int k0, int nb, float* Dr,
                                            float* Di) {
  const int tot = nb * nb;
  for (int e0 = threadIdx.x; e0 < tot; e0 += 8 * blockDim.x) {
    float vr[8], vi[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int e = e0 + q * blockDim.x;
      const int col = e / nb, row = e - col * nb;
      vr[q] = e < tot ? Ar[(size_t)(k0 + col) * ld + k0 + row] : 0.f;
      vi[q] = e < tot ? Ai[(size_t)(k0 + col) * ld + k0 + row] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int e = e0 + q * blockDim.x;
      const int col = e / nb, row = e - col * nb;
      if (e < tot) {
        Dr[col * LU_TB + row] = vr[q];
        Di[col * LU_TB + row] = vi[q];
      }
    }
  }
}

// The inverses of diagonal blocks of the factors: grid block b covers rows
// [128 (blk0 + b), min(128 (blk0 + b + 1), n)) and gives its unit lower triangle's inverse
// in slab 2 b and (with a second grid row) its upper triangle's in slab 2 b + 1, each
// 128 KB ([plane][col][row], LU_TB x LU_TB, zero past a ragged block).  Formed for all
// blocks once after the factorisation, so that a triangular solve applies a diagonal
// block as one matrix-vector product instead of a 128-step substitution, and for the two
// blocks of each panel's L11.  16 warps: the block in shared memory, a warp per column of
// the inverse (column c solves against e_c).
__global__ void __launch_bounds__(512) k_diag_inverse(const float* Ar, const float* Ai, size_t ld, int n, int blk0,
                                                      float* out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float* Dr = reinterpret_cast<float*>(smraw);  // [col][row]
  float* Di = Dr + LU_TB * LU_TB;
  const int k0 = (blk0 + blockIdx.x) * LU_TB, nb = min(LU_TB, n - k0);  // rows [k0, min(k0 + 128, n))
  const bool lower = blockIdx.y == 0;
  stage_block(Ar, Ai, ld, k0, nb, Dr, Di);
  __syncthreads();
  float* o = out + ((size_t)blockIdx.x * 2 + (lower ? 0 : 1)) * 2 * LU_TB * LU_TB;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = warp; c < LU_TB; c += nw) {
    float xr[4], xi[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      xr[q] = (lane + 32 * q == c && c < nb) ? 1.f : 0.f;
      xi[q] = 0.f;
    }
    if (c < nb) {
      if (lower) {
        for (int i = c; i < nb; i++) {
          const int q0 = i >> 5;
          float vr = 0.f, vi = 0.f;
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (q == q0) {
              vr = __shfl_sync(0xffffffffu, xr[q], i & 31);
              vi = __shfl_sync(0xffffffffu, xi[q], i & 31);
            }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int r = lane + 32 * q;
            if (r > i && r < nb) {
              const float lr = Dr[i * LU_TB + r], li = Di[i * LU_TB + r];
              xr[q] -= lr * vr - li * vi;
              xi[q] -= lr * vi + li * vr;
            }
          }
        }
      } else {
        for (int i = c; i >= 0; i--) {
          const int q0 = i >> 5;
          float br = 0.f, bi = 0.f;
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (q == q0) {
              br = __shfl_sync(0xffffffffu, xr[q], i & 31);
              bi = __shfl_sync(0xffffffffu, xi[q], i & 31);
            }
          const float ur = Dr[i * LU_TB + i], ui = Di[i * LU_TB + i];
          const float den = ur * ur + ui * ui;
          const float vr = (br * ur + bi * ui) / den, vi = (bi * ur - br * ui) / den;
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int r = lane + 32 * q;
            if (r == i) {
              xr[q] = vr;
              xi[q] = vi;
            } else if (r < i) {
              const float lr = Dr[i * LU_TB + r], li = Di[i * LU_TB + r];
              xr[q] -= lr * vr - li * vi;
              xi[q] -= lr * vi + li * vr;
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      o[c * LU_TB + lane + 32 * q] = xr[q];
      o[LU_TB * LU_TB + c * LU_TB + lane + 32 * q] = xi[q];
    }
  }
}

// M = I - L11^-1 for a panel's unit lower diagonal block of nb <= 256 rows, made of the
// 128-row blocks A (top) and B (bottom) and the block C below A: from the inverses of A
// and B (slabs 0 and 2 of inv), M11 = I - A^-1, M22 = I - B^-1, M21 = B^-1 C A^-1 and
// M12 = 0, column-major with leading dimension LU_NB.  Then U12 = L11^-1 A12 is the
// in-place update A12 -= M A12, a tensor-core GEMM.  Grid: a block per column j of M,
// 128 threads.
__global__ void __launch_bounds__(LU_TB) k_l11_m(const float* Ar, const float* Ai, size_t ld, int k0, int nb,
                                                 const float* inv, float* Mr, float* Mi) {
  __shared__ float tr[LU_TB], ti[LU_TB];
  const int j = blockIdx.x, r = threadIdx.x;
  const int n1 = min(LU_TB, nb), n2 = nb - n1;
  const size_t sl = (size_t)LU_TB * LU_TB;
  const float *Ar_inv = inv, *Ai_inv = inv + sl;              // A^-1: [col][row]
  const float *Br_inv = inv + 4 * sl, *Bi_inv = inv + 5 * sl;  // B^-1 (slab 2)
  float* mr = Mr + (size_t)j * LU_NB;
  float* mi = Mi + (size_t)j * LU_NB;
  if (j < n1) {
    if (r < n1) {
      mr[r] = (r == j ? 1.f : 0.f) - Ar_inv[(size_t)j * LU_TB + r];
      mi[r] = -Ai_inv[(size_t)j * LU_TB + r];
    }
    if (n2 > 0) {
      // t = C A^-1[:, j], C(r, k) = L11(n1 + r, k)
      float sr = 0.f, si = 0.f;
      if (r < n2) {
#pragma unroll 16
        for (int k = 0; k < n1; k++) {
          const float cr = Ar[(size_t)(k0 + k) * ld + k0 + n1 + r], ci = Ai[(size_t)(k0 + k) * ld + k0 + n1 + r];
          const float ar = Ar_inv[(size_t)j * LU_TB + k], ai = Ai_inv[(size_t)j * LU_TB + k];
          sr += cr * ar - ci * ai;
          si += cr * ai + ci * ar;
        }
      }
      tr[r] = sr;
      ti[r] = si;
      __syncthreads();
      if (r < n2) {  // M21[:, j] = B^-1 t
        float ur = 0.f, ui = 0.f;
#pragma unroll 16
        for (int k = 0; k < n2; k++) {
          const float br = Br_inv[(size_t)k * LU_TB + r], bi = Bi_inv[(size_t)k * LU_TB + r];
          ur += br * tr[k] - bi * ti[k];
          ui += br * ti[k] + bi * tr[k];
        }
        mr[n1 + r] = ur;
        mi[n1 + r] = ui;
      }
    }
  } else {
    const int jj = j - n1;
    if (r < n1) {
      mr[r] = 0.f;
      mi[r] = 0.f;
    }
    if (r < n2) {
      mr[n1 + r] = (r == jj ? 1.f : 0.f) - Br_inv[(size_t)jj * LU_TB + r];
      mi[n1 + r] = -Bi_inv[(size_t)jj * LU_TB + r];
    }
  }
}

// Solves with the factors, one vector (complex64, internal order) in place.  Diagonal
// block: x[k0 .. k0 + nb) = D^-1 x with D^-1 the block's precomputed inverse (L11^-1 or
// U11^-1).  The inverse arrives by one bulk copy on an mbarrier (bounded wait: on give-up
// the kernel records bit 32 in *err, waits once more, bounded, for the copy, and leaves x
// alone); two threads per row then form the product from shared memory.
__global__ void __launch_bounds__(256) k_trsv_diag(const float* dinv, int k0, int nb, cc* x, int* err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ float br[LU_TB], bi[LU_TB];
  float* Dr = reinterpret_cast<float*>(smraw);  // [col][row]
  float* Di = Dr + LU_TB * LU_TB;
  const unsigned bytes = 2u * LU_TB * LU_TB * sizeof(float);
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::mbar_expect_tx(&bar, bytes);
    tc::bulk_g2s(Dr, dinv, bytes, &bar);
  }
  if (threadIdx.x < LU_TB) {
    const int r = threadIdx.x;
    br[r] = r < nb ? x[k0 + r].re : 0.f;
    bi[r] = r < nb ? x[k0 + r].im : 0.f;
  }
  __syncthreads();
  if (!tc::mbar_wait(&bar, 0)) {
    if (threadIdx.x == 0) atomicOr(err, 32);
    tc::mbar_wait(&bar, 0);
    return;
  }
  const int r = threadIdx.x >> 1, h = threadIdx.x & 1;
  float sr = 0.f, si = 0.f;
#pragma unroll 8
  for (int c = h * (LU_TB / 2); c < (h + 1) * (LU_TB / 2); c++) {
    const float ar = Dr[c * LU_TB + r], ai = Di[c * LU_TB + r];
    sr += ar * br[c] - ai * bi[c];
    si += ar * bi[c] + ai * br[c];
  }
  sr += __shfl_xor_sync(0xffffffffu, sr, 1);
  si += __shfl_xor_sync(0xffffffffu, si, 1);
  if (h == 0 && r < nb) x[k0 + r] = mk<float>(sr, si);
}

// x[rows r0 .. r1) -= A[r0 .. r1, k0 .. k0 + nb) x[k0 .. k0 + nb): eight threads per row,
// each 16 columns with their loads in flight together, summed by shuffles.
__global__ void __launch_bounds__(256) k_trsv_gemv(const float* Ar, const float* Ai, size_t ld, int k0, int nb,
                                                   int r0, int r1, cc* x) {
  __shared__ float br[LU_TB], bi[LU_TB];
  for (int r = threadIdx.x; r < LU_TB; r += blockDim.x) {
    br[r] = r < nb ? x[k0 + r].re : 0.f;
    bi[r] = r < nb ? x[k0 + r].im : 0.f;
  }
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = r0 + (t >> 3), part = t & 7;
  const bool live = i < r1;
  float sr = 0.f, si = 0.f;
  if (live) {
    float ar[16], ai[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int j = part * 16 + q;
      ar[q] = j < nb ? Ar[(size_t)(k0 + j) * ld + i] : 0.f;
      ai[q] = j < nb ? Ai[(size_t)(k0 + j) * ld + i] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int j = part * 16 + q;
      sr += ar[q] * br[j] - ai[q] * bi[j];
      si += ar[q] * bi[j] + ai[q] * br[j];
    }
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if (live && part == 0) {
    x[i].re -= sr;
    x[i].im -= si;
  }
}

// y[i] = x[perm[i]]: the factorisation's row interchanges as one gather
__global__ void k_permute(const int* perm, int n, const cc* x, cc* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[perm[i]];
}

__global__ void k_scale_to32(const zc* a, cc* b, int n, double s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = mk<float>((float)(a[i].re * s), (float)(a[i].im * s));
}
__global__ void k_add_from32(zc* x, const cc* d, int n, double s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i].re += (double)d[i].re * s;
    x[i].im += (double)d[i].im * s;
  }
}
__global__ void k_resid(const zc* b, const zc* ax, zc* r, int n, double* nrm2) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const zc v = b[i] - ax[i];
    r[i] = v;
    acc += cabs2(v);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(nrm2, acc);
}

}  // namespace sie

using namespace sie;

// State of the complex64 factorisation, kept in the context between solves.
struct LuTc {
  float* Ar = nullptr;
  float* Ai = nullptr;
  int* ipiv = nullptr;
  int n = 0;
  double factor_s = 0;
};

static int lu_tc_factor(sie_ctx* c) {
  if (c->d_lu32 && c->lu32_valid) return SIE_OK;
  c->lu32_valid = false;
  const int n = 2 * c->M;
  const size_t ld = (size_t)n;
  cudaStream_t s = c->stream;
  // the factors and the workspace stay allocated until sie_release_factors (a later
  // factorisation of the same context reuses them)
  const size_t scr_bytes = panel_scratch_bytes(n);
  if (!c->d_lu32 && cudaMalloc(&c->d_lu32, ld * n * sizeof(float)) != cudaSuccess) c->d_lu32 = nullptr;
  if (!c->d_lu32i && cudaMalloc(&c->d_lu32i, ld * n * sizeof(float)) != cudaSuccess) c->d_lu32i = nullptr;
  if (!c->d_piv32 && cudaMalloc(&c->d_piv32, (size_t)n * sizeof(int)) != cudaSuccess) c->d_piv32 = nullptr;
  if (!c->d_lu_at && cudaMalloc(&c->d_lu_at, tc::tiled_bytes_host(n, LU_NBX)) != cudaSuccess) c->d_lu_at = nullptr;
  if (!c->d_lu_bt && cudaMalloc(&c->d_lu_bt, tc::tiled_bytes_host(n, LU_NBX)) != cudaSuccess) c->d_lu_bt = nullptr;
  // the panel's own updates (beside the previous trailing update, which still reads At, Bt)
  if (!c->d_lu_at2 && cudaMalloc(&c->d_lu_at2, tc::tiled_bytes_host(n, LU_BB) + tc::tiled_bytes_host(LU_NBX, LU_BB)) !=
                          cudaSuccess)
    c->d_lu_at2 = nullptr;
  // a panel's L11 work: two blocks' inverse slabs (4 x 128 KB with the unused upper ones),
  // then M = I - L11^-1 in two LU_NB x LU_NB planes
  if (!c->d_lu_minv &&
      cudaMalloc(&c->d_lu_minv, (8 * (size_t)LU_TB * LU_TB + 2 * (size_t)LU_NB * LU_NB) * sizeof(float)) != cudaSuccess)
    c->d_lu_minv = nullptr;
  const int ndiag = (n + LU_TB - 1) / LU_TB;
  if (!c->d_lu_diag && cudaMalloc(&c->d_lu_diag, (size_t)ndiag * 4 * LU_TB * LU_TB * sizeof(float)) != cudaSuccess)
    c->d_lu_diag = nullptr;
  if (!c->d_lu_scr || c->lu_scr_bytes < scr_bytes) {
    if (c->d_lu_scr) cudaFree(c->d_lu_scr);
    if (cudaMalloc(&c->d_lu_scr, scr_bytes) != cudaSuccess) c->d_lu_scr = nullptr;
    c->lu_scr_bytes = c->d_lu_scr ? scr_bytes : 0;
  }
  if (!c->d_lu32 || !c->d_lu32i || !c->d_piv32 || !c->d_lu_at || !c->d_lu_bt || !c->d_lu_scr || !c->d_lu_diag ||
      !c->d_lu_minv || !c->d_lu_at2) {
    cudaGetLastError();
    return fail(SIE_ERR_NOMEM, "mixed LU: device memory");
  }
  float* Ar = c->d_lu32;
  float* Ai = c->d_lu32i;
  int* ipiv = c->d_piv32;
  char* At = c->d_lu_at;
  char* Bt = c->d_lu_bt;
  char* At2 = c->d_lu_at2;
  char* Bt2 = At2 + tc::tiled_bytes_host(n, LU_BB);
  int* err = (int*)c->d_lu_scr;
  PanelSlot* slots = (PanelSlot*)((char*)c->d_lu_scr + PANEL_SLOTS_OFF);
  unsigned* pcnt = (unsigned*)((char*)c->d_lu_scr + PANEL_CNT_OFF);  // one counter per sub-panel launch
  unsigned* pbad = pcnt + (n / LU_SB + 1);
  int* plan = (int*)((char*)c->d_lu_scr + panel_plan_off(n));
  unsigned* amax = (unsigned*)((char*)c->d_lu_scr + panel_amax_off(n));
  int rc = SIE_OK;
  auto t0 = std::chrono::steady_clock::now();
  cudaMemsetAsync(c->d_lu_scr, 0, scr_bytes, s);
  {
    dim3 g(64, std::min(c->near.nbox, 1024));
    k_expand_dense32<<<g, 256, 0, s>>>(c->d_base, c->d_box_first, c->d_box_cnt, c->d_ncols, c->near.nbox, c->d_na,
                                       c->d_nb, c->d_nd, c->cfac, c->M, Ar, Ai);
    count_launch();
  }
  // CUDA events around every trailing update, read once the factorisation has finished
  std::vector<cudaEvent_t> evs;
  auto new_event = [&]() {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) == cudaSuccess) evs.push_back(e);
    return e;
  };
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> gemm_ev;
  double gemm_flops = 0;
  const size_t trsm_smem = (size_t)2 * LU_TB * LU_TB * sizeof(float);
  const size_t blk_smem = (size_t)2 * LU_BB * LU_BB * sizeof(float2);
  if (raise_smem(k_diag_inverse, trsm_smem) != cudaSuccess || raise_smem(k_blk_trsm, blk_smem) != cudaSuccess)
    rc = fail(SIE_ERR_CUDA, "mixed LU: shared memory");
  // optional per-phase device times (SIE_LU_PHASES=1): panel, swaps, L11 solve, tiling
  const char* pe = getenv("SIE_LU_PHASES");
  const bool phases = pe && atoi(pe) != 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ph_ev[4];
  auto mark = [&](int which, bool start, cudaEvent_t& keep) {
    if (!phases) return;
    cudaEvent_t e = new_event();
    if (!e) return;
    cudaEventRecord(e, s);
    if (start) keep = e;
    else ph_ev[which].push_back({keep, e});
  };
  cudaEvent_t pk = nullptr;
  // Look-ahead: the panel chain runs on a high-priority stream sp.  After a panel's
  // update, the columns of the next panel are updated first (on sp), and the rest of the
  // trailing update goes to a low-priority stream sg, where it runs beside the next
  // panel's factorisation (disjoint columns).  The next row swaps and operand tiling wait
  // for it.
  cudaStream_t sp = nullptr, sg = nullptr;
  cudaEvent_t ev_start = nullptr, ev_tiled = nullptr, ev_rest = nullptr, ev_sp = nullptr, ev_sg = nullptr;
  {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&sp, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&sg, cudaStreamNonBlocking, lo) != cudaSuccess)
      rc = fail(SIE_ERR_CUDA, "mixed LU: streams");
    for (cudaEvent_t* e : {&ev_start, &ev_tiled, &ev_rest, &ev_sp, &ev_sg})
      if (rc == SIE_OK && cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(SIE_ERR_CUDA, "mixed LU: events");
    if (rc == SIE_OK) {
      cudaEventRecord(ev_start, s);
      cudaStreamWaitEvent(sp, ev_start, 0);
      cudaStreamWaitEvent(sg, ev_start, 0);
    }
  }
  const cudaStream_t s_main = s;
  // the look-ahead update leaves LU_FREE_SMS multiprocessors to the panel chain (two
  // persistent CTAs per multiprocessor)
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  int free_sms = LU_FREE_SMS;
  if (const char* e = getenv("SIE_LU_FREE_SMS")) free_sms = std::max(0, std::min(nsm - 1, atoi(e)));
  const int rest_ctas = 2 * std::max(1, nsm - free_sms);
  // SIE_LU_LOOKAHEAD=0 runs the whole trailing update on the panel stream (same work)
  const char* la = getenv("SIE_LU_LOOKAHEAD");
  const bool lookahead = !(la && atoi(la) == 0);
  // trailing updates in split-FP16 unless this context's refinement needed 3xTF32 before
  // (or SIE_LU_GEMM=tf32 asks for it)
  // panel width: LU_NBX (trailing updates of K = 512, which read and write the trailing
  // matrix half as often per flop as K = 256: 2.60 s against 2.90 s for the slab10 solve),
  // or LU_NB with SIE_LU_NB=256
  int pnb = LU_NBX;
  if (const char* e = getenv("SIE_LU_NB")) pnb = atoi(e) >= LU_NBX ? LU_NBX : LU_NB;
  // the panel's block width: LU_BB, or with 256-column panels the whole panel
  // (SIE_LU_BLOCK=256: every sub-panel updates all of the panel's later columns on the CUDA
  // cores; k_sub_update holds at most LU_NB columns of U, so 512-column panels keep LU_BB)
  int pbb = LU_BB;
  if (const char* e = getenv("SIE_LU_BLOCK")) pbb = atoi(e) >= LU_NB && pnb <= LU_NB ? pnb : LU_BB;
  const char* gp = getenv("SIE_LU_GEMM");
  const bool gh = c->lu_f16_ok && !(gp && std::string(gp) == "tf32");
  c->tm.lu_f16 = gh ? 1 : 0;
  c->tm.lu_factorizations += 1;
  // the cooperative panel kernel: blocks that fit on the multiprocessors the look-ahead
  // update leaves free, or on all of them without look-ahead (all resident at once)
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subpanel, 256, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int panel_sms = lookahead ? std::max(free_sms, 1) : nsm;
  int panel_blocks = std::max(1, std::min(PANEL_MAX_BLOCKS, std::min(per_sm, 4) * panel_sms));
  if (const char* e = getenv("SIE_LU_PANEL_BLOCKS"))
    panel_blocks = std::max(1, std::min(panel_blocks, atoi(e)));
  s = sp;  // the phase marks and the panel chain
  bool rest_pending = false;
  for (int k0 = 0; k0 < n && rc == SIE_OK; k0 += pnb) {
    const int nb = std::min(pnb, n - k0), k1 = k0 + nb;
    mark(0, true, pk);
    // the panel in 64-column blocks of LU_SB-column sub-panels: inside a block, each
    // sub-panel updates the block's later columns (CUDA cores); after a block, its U rows
    // of the panel's remaining columns and one tensor-core update of those columns
    for (int s0 = k0; s0 < k1; s0 += LU_SB) {
      const int s1 = std::min(s0 + LU_SB, k1);
      const int b0 = k0 + (s0 - k0) / pbb * pbb, b1 = std::min(b0 + pbb, k1);
      {
        int ns0 = s0, ns1 = s1, nn0 = n, kk0 = k0, kk1 = k1;
        size_t ldd = ld;
        unsigned* cnt = pcnt + s0 / LU_SB;  // a fresh (zeroed) counter for every launch
        void* args[] = {&Ar, &Ai, &ldd, &nn0, &ns0, &ns1, &kk0, &kk1, &ipiv, &err, &slots, &cnt, &pbad};
        if (cudaLaunchCooperativeKernel((const void*)k_subpanel, dim3(panel_blocks), dim3(256), args, 0, sp) !=
            cudaSuccess) {
          rc = fail(SIE_ERR_CUDA, "mixed LU: cooperative panel launch");
          break;
        }
        count_launch();
      }
      k_sub_finish<<<(k1 - k0 + LU_FIN_T - 1) / LU_FIN_T, LU_FIN_T, 0, sp>>>(Ar, Ai, ld, k0, s0, s1, k1, b1, ipiv);
      count_launch();
      if (s1 < b1 && s1 < n) {
        if (b1 - s1 > LU_NB) {  // k_sub_update holds LU_NB columns of U in shared memory
          rc = fail(SIE_ERR_ARG, "mixed LU: block wider than the sub-panel update's tile");
          break;
        }
        k_sub_update<<<dim3((n - s1 + 255) / 256, (b1 - s1 + LU_UPD_SLICE - 1) / LU_UPD_SLICE), 256, 0, sp>>>(
            Ar, Ai, ld, n, s0, s1, b1);
        count_launch();
      }
      if (s1 == b1 && b1 < k1 && rc == SIE_OK) {
        const int w = b1 - b0;
        if (w > LU_BB) {  // k_blk_trsm holds LU_BB columns of L in shared memory
          rc = fail(SIE_ERR_ARG, "mixed LU: block wider than the triangular solve's tile");
          break;
        }
        k_blk_trsm<<<(k1 - b1 + LU_BB - 1) / LU_BB, LU_BB, blk_smem, sp>>>(Ar, Ai, ld, b0, b1, b1, k1);
        count_launch();
        rc = tc::tile_operand(Ar + (size_t)b0 * ld + b1, Ai + (size_t)b0 * ld + b1, ld, n - b1, w, false, At2, sp, gh,
                              amax + 2);
        if (rc == SIE_OK)
          rc = tc::tile_operand(Ar + (size_t)b1 * ld + b0, Ai + (size_t)b1 * ld + b0, ld, k1 - b1, w, true, Bt2, sp,
                                gh, amax + 3);
        if (rc == SIE_OK)
          rc = tc::gemm_update(At2, Bt2, w, Ar + (size_t)b1 * ld + b1, Ai + (size_t)b1 * ld + b1, ld, n - b1, k1 - b1,
                               err, sp, 0, gh, amax + 2);
      }
    }
    mark(0, false, pk);
    if (rest_pending) cudaStreamWaitEvent(sp, ev_rest, 0);  // the previous trailing update
    mark(1, true, pk);
    if (n - nb > 0) {
      k_swap_plan<<<1, 256, 0, sp>>>(ipiv, k0, k1, plan);
      count_launch();
      k_swap_apply<<<(n - nb + LU_SWAP_TC - 1) / LU_SWAP_TC, 2 * nb, 0, sp>>>(Ar, Ai, ld, n, k0, k1, plan);
      count_launch();
    }
    mark(1, false, pk);
    if (k1 < n) {
      mark(2, true, pk);
      // U12 = L11^-1 A12, in halves of at most LU_NB rows: each half as the in-place
      // tensor-core update A12 -= (I - L11^-1) A12 (the inverses of L11's two 128-row
      // blocks, then M = I - L11^-1 by k_l11_m, then the GEMM); a second half first loses
      // L(h, first half) times the first half's U rows
      float* inv = c->d_lu_minv;
      float* Mr = inv + 8 * (size_t)LU_TB * LU_TB;
      float* Mi = Mr + (size_t)LU_NB * LU_NB;
      for (int h0 = k0; h0 < k1 && rc == SIE_OK; h0 += LU_NB) {
        const int hb = std::min(LU_NB, k1 - h0), h1 = h0 + hb;
        if (h0 > k0) {
          rc = tc::tile_operand(Ar + (size_t)k0 * ld + h0, Ai + (size_t)k0 * ld + h0, ld, hb, h0 - k0, false, At, sp,
                                gh, amax);
          if (rc == SIE_OK)
            rc = tc::tile_operand(Ar + (size_t)k1 * ld + k0, Ai + (size_t)k1 * ld + k0, ld, n - k1, h0 - k0, true, Bt,
                                  sp, gh, amax + 1);
          if (rc == SIE_OK)
            rc = tc::gemm_update(At, Bt, h0 - k0, Ar + (size_t)k1 * ld + h0, Ai + (size_t)k1 * ld + h0, ld, hb, n - k1,
                                 err, sp, 0, gh, amax);
          if (rc != SIE_OK) break;
        }
        k_diag_inverse<<<dim3((hb + LU_TB - 1) / LU_TB, 1), 512, trsm_smem, sp>>>(Ar, Ai, ld, h1, h0 / LU_TB, inv);
        count_launch();
        k_l11_m<<<hb, LU_TB, 0, sp>>>(Ar, Ai, ld, h0, hb, inv, Mr, Mi);
        count_launch();
        rc = tc::tile_operand(Mr, Mi, LU_NB, hb, hb, false, At, sp, gh, amax);
        if (rc == SIE_OK)
          rc = tc::tile_operand(Ar + (size_t)k1 * ld + h0, Ai + (size_t)k1 * ld + h0, ld, n - k1, hb, true, Bt, sp, gh,
                                amax + 1);
        if (rc == SIE_OK)
          rc = tc::gemm_update(At, Bt, hb, Ar + (size_t)k1 * ld + h0, Ai + (size_t)k1 * ld + h0, ld, hb, n - k1, err,
                               sp, 0, gh, amax);
      }
      mark(2, false, pk);
      const int m = n - k1, nn = std::min(pnb, m);
      // A22 -= L21 U12 on the tensor cores
      mark(3, true, pk);
      rc = tc::tile_operand(Ar + (size_t)k0 * ld + k1, Ai + (size_t)k0 * ld + k1, ld, m, nb, false, At, sp, gh, amax);
      if (rc == SIE_OK)
        rc = tc::tile_operand(Ar + (size_t)k1 * ld + k0, Ai + (size_t)k1 * ld + k0, ld, m, nb, true, Bt, sp, gh,
                              amax + 1);
      mark(3, false, pk);
      cudaEventRecord(ev_tiled, sp);
      const cudaStream_t srest = lookahead ? sg : sp;
      if (rc == SIE_OK && m > nn) {
        // the columns past the next panel, on sg
        cudaStreamWaitEvent(sg, ev_tiled, 0);
        cudaEvent_t e0 = new_event(), e1 = new_event();
        if (e0) cudaEventRecord(e0, srest);
        // the B tiles past the next panel's nn columns
        const int kc = gh ? tc::KC_F16 : tc::KC;
        const size_t boff = (size_t)(nn / tc::TILE) * ((nb + kc - 1) / kc) * tc::BLOCK_BYTES;
        rc = tc::gemm_update(At, Bt + boff, nb, Ar + (size_t)(k1 + nn) * ld + k1, Ai + (size_t)(k1 + nn) * ld + k1,
                             ld, m, m - nn, err, srest, lookahead ? rest_ctas : 0, gh, amax);
        if (e1) cudaEventRecord(e1, srest);
        if (e0 && e1) gemm_ev.push_back({e0, e1});
        cudaEventRecord(ev_rest, srest);
        rest_pending = true;
        gemm_flops += 8.0 * m * (double)(m - nn) * nb;
      }
      // the next panel's columns, on sp
      cudaEvent_t e0 = new_event(), e1 = new_event();
      if (e0) cudaEventRecord(e0, sp);
      if (rc == SIE_OK)
        rc = tc::gemm_update(At, Bt, nb, Ar + (size_t)k1 * ld + k1, Ai + (size_t)k1 * ld + k1, ld, m, nn, err, sp, 0,
                             gh, amax);
      if (e1) cudaEventRecord(e1, sp);
      if (e0 && e1) gemm_ev.push_back({e0, e1});
      gemm_flops += 8.0 * m * (double)nn * nb;
    }
    if (cudaGetLastError() != cudaSuccess && rc == SIE_OK) rc = fail(SIE_ERR_CUDA, "mixed LU: launch");
  }
  s = s_main;
  if (ev_sp && ev_sg) {
    cudaEventRecord(ev_sp, sp);
    cudaEventRecord(ev_sg, sg);
    cudaStreamWaitEvent(s, ev_sp, 0);
    cudaStreamWaitEvent(s, ev_sg, 0);
  }
  if (rc == SIE_OK) {
    const size_t ism = (size_t)2 * LU_TB * LU_TB * sizeof(float);
    if (raise_smem(k_diag_inverse, ism) != cudaSuccess) {
      rc = fail(SIE_ERR_CUDA, "mixed LU: shared memory");
    } else {
      k_diag_inverse<<<dim3(ndiag, 2), 512, ism, s>>>(Ar, Ai, ld, n, 0, c->d_lu_diag);
      count_launch();
    }
  }
  int herr = 0;
  if (rc == SIE_OK && (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                       cudaStreamSynchronize(s) != cudaSuccess))
    rc = fail(SIE_ERR_CUDA, "mixed LU: factorisation");
  if (rc == SIE_OK) {
    // the interchanges as one permutation, for the solves
    std::vector<int> piv(n), perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    if (cudaMemcpy(piv.data(), ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(SIE_ERR_CUDA, "mixed LU: pivots");
    for (int j = 0; j < n && rc == SIE_OK; j++) std::swap(perm[j], perm[piv[j]]);
    if (rc == SIE_OK && ((!c->d_perm32 && cudaMalloc(&c->d_perm32, (size_t)n * sizeof(int)) != cudaSuccess) ||
                         (!c->d_tmp32 && cudaMalloc(&c->d_tmp32, (size_t)n * sizeof(cc)) != cudaSuccess) ||
                         cudaMemcpy(c->d_perm32, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice) !=
                             cudaSuccess))
      rc = fail(SIE_ERR_NOMEM, "mixed LU: permutation");
  }
  if (rc == SIE_OK && (herr & 8)) rc = fail(SIE_ERR_NONFINITE, "mixed LU: singular or non-finite pivot");
  if (rc == SIE_OK && (herr & 16)) rc = fail(SIE_ERR_CUDA, "mixed LU: a grid barrier of the panel kernel timed out");
  if (rc == SIE_OK && herr) rc = fail(SIE_ERR_CUDA, "mixed LU: a tensor-core pipeline wait timed out");
  c->tm.lu_factor_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  double gms = 0;
  for (auto& pe : gemm_ev) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, pe.first, pe.second) == cudaSuccess) gms += ms;
  }
  c->tm.lu_gemm_ms = gms;
  for (int q = 0; q < 4; q++) {
    double t = 0;
    for (auto& pe2 : ph_ev[q]) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, pe2.first, pe2.second) == cudaSuccess) t += ms;
    }
    c->tm.lu_phase_ms[q] = t;
  }
  c->tm.lu_gemm_flops = gemm_flops;
  c->tm.lu_gemm_launches = (int)gemm_ev.size();
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  for (cudaEvent_t e : {ev_start, ev_tiled, ev_rest, ev_sp, ev_sg})
    if (e) cudaEventDestroy(e);
  if (sp) cudaStreamDestroy(sp);
  if (sg) cudaStreamDestroy(sg);
  c->lu32_valid = rc == SIE_OK;
  return rc;
}

// x = U^-1 L^-1 P x with the complex64 factors (internal order, in place).
static int lu_tc_solve32(sie_ctx* c, cc* x, cudaStream_t s) {
  const int n = 2 * c->M;
  const size_t ld = (size_t)n;
  const float *Ar = c->d_lu32, *Ai = c->d_lu32i;
  int* err = (int*)c->d_lu_scr;
  k_permute<<<148, 256, 0, s>>>(c->d_perm32, n, x, c->d_tmp32);
  count_launch();
  SIE_CUDA(cudaMemcpyAsync(x, c->d_tmp32, (size_t)n * sizeof(cc), cudaMemcpyDeviceToDevice, s));
  const size_t dsm = (size_t)2 * LU_TB * LU_TB * sizeof(float);
  SIE_CUDA(raise_smem(k_trsv_diag, dsm));
  const size_t slab = (size_t)2 * LU_TB * LU_TB;
  for (int k0 = 0; k0 < n; k0 += LU_TB) {
    const int nb = std::min(LU_TB, n - k0), k1 = k0 + nb;
    k_trsv_diag<<<1, 256, dsm, s>>>(c->d_lu_diag + (size_t)(2 * (k0 / LU_TB)) * slab, k0, nb, x, err);
    count_launch();
    if (k1 < n) {
      k_trsv_gemv<<<(8 * (n - k1) + 255) / 256, 256, 0, s>>>(Ar, Ai, ld, k0, nb, k1, n, x);
      count_launch();
    }
  }
  for (int k0 = ((n - 1) / LU_TB) * LU_TB; k0 >= 0; k0 -= LU_TB) {
    const int nb = std::min(LU_TB, n - k0);
    k_trsv_diag<<<1, 256, dsm, s>>>(c->d_lu_diag + (size_t)(2 * (k0 / LU_TB) + 1) * slab, k0, nb, x, err);
    count_launch();
    if (k0 > 0) {
      k_trsv_gemv<<<(8 * k0 + 255) / 256, 256, 0, s>>>(Ar, Ai, ld, k0, nb, 0, k0, x);
      count_launch();
    }
  }
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// One or more right-hand sides on device buffers (external order, stride 2M).
static int solve_direct_mixed_dev(sie_ctx* c, const zc* d_b, zc* d_x, int nrhs, double tolerance,
                                  int max_refinements, sie_stats* stats, cudaStream_t s) {
  auto t0 = std::chrono::steady_clock::now();
  c->tm.lu_factorizations = 0;
  SIE_TRY(lu_tc_factor(c));
  const int n = 2 * c->M;
  const size_t bytes = (size_t)n * sizeof(zc);
  // the refinement's vectors: allocated with the first solve and kept with the factors
  // (a cudaMalloc / cudaFree pair per solve cost up to 0.7 s now and then on a device with
  // tens of GB allocated)
  int rc = SIE_OK;
  if (!c->d_lu_ref &&
      cudaMalloc(&c->d_lu_ref, 4 * bytes + (size_t)n * sizeof(cc) + 2 * sizeof(double)) != cudaSuccess) {
    c->d_lu_ref = nullptr;
    cudaGetLastError();
    rc = fail(SIE_ERR_NOMEM, "mixed direct solve: device buffers");
  }
  zc* bi = (zc*)c->d_lu_ref;
  zc *xi = bi + n, *ax = bi + 2 * (size_t)n, *r = bi + 3 * (size_t)n;
  cc* d32 = (cc*)(bi + 4 * (size_t)n);
  double* nrm = (double*)(d32 + n);
  for (int k = 0; k < nrhs && rc == SIE_OK; k++) {
    auto tk = std::chrono::steady_clock::now();
    const size_t off = (size_t)k * n;
    double bn2 = 0, rn2 = 0, prev2 = 0;
    int steps = 0;
    bool stalled = false;  // split-FP16 factors that do not contract the residual
    const bool h_factors = c->tm.lu_f16 != 0;
    rc = gather_ext_to_int(c, d_b + off, bi, 1, s);
    cudaMemsetAsync(xi, 0, bytes, s);
    // r = b - Z x in FP64 (x = 0 at the start), then d = LU^-1 r in complex64 (r scaled to
    // unit norm) and x += d, until ||r|| <= tolerance ||b||
    for (; rc == SIE_OK; steps++) {
      if (steps == 0) {
        cudaMemsetAsync(ax, 0, bytes, s);
      } else {
        rc = near_matvec64(c, xi, ax, 1, false, s);
        if (rc != SIE_OK) break;
      }
      cudaMemsetAsync(nrm, 0, sizeof(double), s);
      k_resid<<<296, 256, 0, s>>>(bi, ax, r, n, nrm);
      count_launch();
      int herr = 0;
      if (cudaMemcpyAsync(&rn2, nrm, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaMemcpyAsync(&herr, c->d_lu_scr, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = fail(SIE_ERR_CUDA, "mixed direct solve: residual");
        break;
      }
      if (herr & 32) {
        rc = fail(SIE_ERR_CUDA, "mixed direct solve: a triangular solve's block copy timed out");
        break;
      }
      if (steps == 0) bn2 = rn2;
      const bool done = std::isfinite(rn2) && (bn2 == 0.0 || rn2 <= tolerance * tolerance * bn2);
      // each correction must at least halve the residual (the factors' error times cond(Z)
      // well below one); split-FP16 factors that do not are replaced by 3xTF32 ones
      if (h_factors && !done && steps >= 2 && (!std::isfinite(rn2) || rn2 > 0.25 * prev2)) {
        stalled = true;
        break;
      }
      prev2 = rn2;
      if (!std::isfinite(rn2)) {
        rc = fail(SIE_ERR_NONFINITE, "mixed direct solve: non-finite residual");
        break;
      }
      if (done || steps > max_refinements) break;
      const double rn = std::sqrt(rn2);
      k_scale_to32<<<296, 256, 0, s>>>(r, d32, n, 1.0 / rn);
      count_launch();
      rc = lu_tc_solve32(c, d32, s);
      if (rc != SIE_OK) break;
      k_add_from32<<<296, 256, 0, s>>>(xi, d32, n, rn);
      count_launch();
    }
    if (rc != SIE_OK) break;
    if (stalled) {  // factorise again with 3xTF32 updates and redo this right-hand side
      c->lu_f16_ok = false;
      c->lu32_valid = false;
      rc = lu_tc_factor(c);
      if (rc != SIE_OK) break;
      k--;
      continue;
    }
    rc = scatter_int_to_ext(c, xi, d_x + off, 1, s);
    if (rc == SIE_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(SIE_ERR_CUDA, "mixed direct solve");
    const double be = bn2 > 0 ? std::sqrt(rn2 / bn2) : 0.0;
    const bool conv = be <= tolerance;
    if (stats) {
      stats[k].iterations = steps;
      stats[k].inner_iterations = 0;
      stats[k].matvecs = steps;
      stats[k].converged = conv;
      stats[k].backward_error_arnoldi = be;
      stats[k].backward_error_true = be;
      stats[k].seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - (k == 0 ? t0 : tk)).count();
    }
    if (rc == SIE_OK && !conv) rc = fail(SIE_ERR_NOCONV, "mixed direct solve: refinement did not reach the tolerance");
  }
  return rc;
}

static int check_direct_mixed(sie_ctx* c, int nrhs, double tolerance, int max_refinements, const char* who) {
  if (!c || nrhs < 1 || !(tolerance > 0) || max_refinements < 0)
    return fail(SIE_ERR_ARG, std::string(who) + ": bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, std::string(who) + ": sie_setup not called");
  if (!c->cfg.dense) return fail(SIE_ERR_STATE, std::string(who) + ": needs a context set up with dense = 1");
  return SIE_OK;
}

extern "C" int sie_solve_direct_mixed_device(sie_ctx* c, const double* d_b, double* d_x, int nrhs,
                                             double tolerance, int max_refinements, sie_stats* stats,
                                             void* stream) {
  SIE_TRY(check_direct_mixed(c, nrhs, tolerance, max_refinements, "sie_solve_direct_mixed_device"));
  if (!d_b || !d_x) return fail(SIE_ERR_ARG, "sie_solve_direct_mixed_device: null buffer");
  SIE_CUDA(cudaSetDevice(c->device));
  return solve_direct_mixed_dev(c, (const zc*)d_b, (zc*)d_x, nrhs, tolerance, max_refinements, stats,
                                stream ? (cudaStream_t)stream : c->stream);
}

extern "C" int sie_solve_direct_mixed(sie_ctx* c, const double* b, double* x, int nrhs, double tolerance,
                                      int max_refinements, sie_stats* stats) {
  SIE_TRY(check_direct_mixed(c, nrhs, tolerance, max_refinements, "sie_solve_direct_mixed"));
  if (!b || !x) return fail(SIE_ERR_ARG, "sie_solve_direct_mixed: null buffer");
  SIE_CUDA(cudaSetDevice(c->device));
  for (size_t i = 0; i < (size_t)4 * c->M * nrhs; i++)
    if (!std::isfinite(b[i])) return fail(SIE_ERR_NONFINITE, "sie_solve_direct_mixed: non-finite right-hand side");
  const size_t bytes = (size_t)2 * c->M * nrhs * sizeof(zc);
  // device copies of b and x, kept with the factors and grown when nrhs grows
  if (c->lu_io_bytes < 2 * bytes) {
    if (c->d_lu_io) cudaFree(c->d_lu_io);
    c->d_lu_io = nullptr;
    c->lu_io_bytes = 0;
    if (cudaMalloc(&c->d_lu_io, 2 * bytes) != cudaSuccess) {
      c->d_lu_io = nullptr;
      cudaGetLastError();
      return fail(SIE_ERR_NOMEM, "sie_solve_direct_mixed: device buffers");
    }
    c->lu_io_bytes = 2 * bytes;
  }
  zc* db = (zc*)c->d_lu_io;
  zc* dx = (zc*)((char*)c->d_lu_io + bytes);
  int rc = SIE_OK;
  if (cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct_mixed: copy");
  if (rc == SIE_OK) rc = solve_direct_mixed_dev(c, db, dx, nrhs, tolerance, max_refinements, stats, c->stream);
  if ((rc == SIE_OK || rc == SIE_ERR_NOCONV) &&
      (cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
       cudaStreamSynchronize(c->stream) != cudaSuccess))
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct_mixed: copy back");
  return rc;
}

extern "C" int sie_release_factors(sie_ctx* c) {
  if (!c) return fail(SIE_ERR_ARG, "sie_release_factors: null context");
  SIE_CUDA(cudaSetDevice(c->device));
  if (c->stream) SIE_CUDA(cudaStreamSynchronize(c->stream));
  for (void* p : {(void*)c->d_lu, (void*)c->d_piv, (void*)c->d_lu32, (void*)c->d_lu32i, (void*)c->d_piv32,
                  (void*)c->d_perm32, (void*)c->d_tmp32, (void*)c->d_lu_at, (void*)c->d_lu_bt, c->d_lu_scr,
                  (void*)c->d_lu_diag, (void*)c->d_lu_minv, (void*)c->d_lu_at2, (void*)c->d_lu_ref, c->d_lu_io})
    if (p) cudaFree(p);
  c->d_lu = nullptr;
  c->d_piv = nullptr;
  c->d_lu32 = c->d_lu32i = nullptr;
  c->d_piv32 = c->d_perm32 = nullptr;
  c->d_tmp32 = nullptr;
  c->d_lu_at = c->d_lu_bt = nullptr;
  c->d_lu_scr = nullptr;
  c->d_lu_diag = nullptr;
  c->d_lu_minv = nullptr;
  c->d_lu_at2 = nullptr;
  c->d_lu_ref = nullptr;
  c->d_lu_io = nullptr;
  c->lu_io_bytes = 0;
  c->lu_scr_bytes = 0;
  c->lu64_valid = c->lu32_valid = false;
  return SIE_OK;
}

extern "C" int sie_invalidate_factors(sie_ctx* c) {
  if (!c) return fail(SIE_ERR_ARG, "sie_invalidate_factors: null context");
  SIE_CUDA(cudaSetDevice(c->device));
  if (c->stream) SIE_CUDA(cudaStreamSynchronize(c->stream));
  c->lu64_valid = c->lu32_valid = false;
  return SIE_OK;
}
