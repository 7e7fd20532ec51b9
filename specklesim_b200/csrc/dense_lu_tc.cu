// Mixed-precision direct solve of the dense system: LU with partial pivoting of the
// complex64 matrix, its O(N^3) trailing updates on the tensor cores (tc_gemm.cu, 3xTF32,
// FP32-accurate), then iterative refinement in FP64 against the FP64 dense product.
//
// The reference's direct path (lib_sie_tri_solver_normal_I,
// src/lib_sie_tri_solver_normal.f90:64-217, with ZGESV in solver_LU,
// src/lib_sie_math.f90:649-676) factorises the FP64 matrix; sie_solve_direct does the
// same with cuSOLVER.  Here the factorisation runs in FP32 arithmetic and the solution is
// refined in FP64 (x += U^-1 L^-1 P (b - Z x)) until the true backward error meets the
// tolerance, which it does while cond(Z) times the factorisation's rounding stays below
// one.
//
// Blocked right-looking LU, panel width NB = 256, on the matrix stored as two FP32
// planes (real, imaginary), column-major, internal unknown order:
//   1. panel, in sub-panels of 16 columns: each sub-panel is one cooperative launch that,
//      column by column, agrees on the pivot, swaps rows across the panel, scales the
//      column and updates the sub-panel (two bounded grid barriers per column); then the
//      sub-panel's U rows (L11^-1) and one rank-16 update of the panel's later columns;
//   2. the panel's row swaps applied to every column left and right of it;
//   3. U12 = L11^-1 A12 by 128-row diagonal blocks: a warp per column with the block in
//      shared memory, the rows below it updated on the tensor cores;
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
                 cudaStream_t st);
int gemm_update(const char* At, const char* Bt, int K, float* Cr, float* Ci, size_t ldc, int m, int n,
                int* d_err, cudaStream_t st, int max_ctas = 0);
size_t tiled_bytes_host(int rows, int K);
}  // namespace tc

static const int LU_NB = 256;  // panel width (the tensor-core update's K)
static const int LU_SB = 16;   // sub-panel width inside a panel
static const int LU_TB = 128;  // diagonal blocks of the triangular solves
static const int LU_FREE_SMS = 12;  // multiprocessors the look-ahead update leaves to the panels
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

// Grid barrier of the cooperative sub-panel kernel (all its blocks are resident).  The
// wait is bounded: a block that sees no progress for about a second records the failure
// in st[2] and stops waiting; later barriers then pass straight through, and the host
// reports the error.  st = {arrival count, generation, error}.
__device__ void lu_grid_bar(unsigned* st, unsigned nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &st[1];
    volatile unsigned* bad = &st[2];
    if (*bad == 0) {
      const unsigned g = *gen;
      __threadfence();
      const unsigned arrived = atomicAdd(&st[0], 1u) + 1u;
      if (arrived == nblocks) {
        atomicExch(&st[0], 0u);
        __threadfence();
        atomicAdd(&st[1], 1u);
      } else {
        long long it = 0;
        while (*gen == g && *bad == 0) {
          if (++it > (1LL << 24)) {
            atomicExch(&st[2], 1u);
            break;
          }
          __nanosleep(64);
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// One sub-panel [s0, s1) of the panel [k0, k1) factorised by one cooperative launch: for
// each column j, every block reduces the published maxima of column j to the same pivot
// p, block 0 swaps rows j and p across the panel and records p; after a grid barrier every
// thread scales its rows of column j by the pivot and updates them in the sub-panel's
// later columns with row j, and publishes its maximum of the updated column j + 1; a
// second barrier ends the step.  Matrix reads bypass L1 (__ldcg): rows written by other
// blocks are seen through L2.  pmax / pidx: one slot per block.
__global__ void __launch_bounds__(256) k_subpanel(float* Ar, float* Ai, size_t ld, int n, int s0, int s1, int k0,
                                                  int k1, int* ipiv, int* err, float* pmax, int* pidx,
                                                  unsigned* bar) {
  __shared__ float sv[8];
  __shared__ int si[8];
  __shared__ int piv_s;
  const unsigned G = gridDim.x;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = G * blockDim.x;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  auto publish = [&](float best, int bi) {
    for (int o = 16; o > 0; o >>= 1)
      argmax_pair(best, bi, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o));
    if (l == 0) {
      sv[w] = best;
      si[w] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 1; k < (int)(blockDim.x >> 5); k++) argmax_pair(best, bi, sv[k], si[k]);
      pmax[blockIdx.x] = best;
      pidx[blockIdx.x] = bi;
    }
  };
  {  // maxima of the first column
    float best = -1.f;
    int bi = n;
    for (int r = s0 + gtid; r < n; r += gstride) {
      const float a = __ldcg(Ar + (size_t)s0 * ld + r), b = __ldcg(Ai + (size_t)s0 * ld + r);
      argmax_pair(best, bi, a * a + b * b, r);
    }
    publish(best, bi);
  }
  lu_grid_bar(bar, G);
  for (int j = s0; j < s1; j++) {
    if (threadIdx.x < 32) {
      float best = -1.f;
      int bi = n;
      for (int k = threadIdx.x; k < (int)G; k += 32) argmax_pair(best, bi, __ldcg(pmax + k), __ldcg(pidx + k));
      for (int o = 16; o > 0; o >>= 1)
        argmax_pair(best, bi, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o));
      if (threadIdx.x == 0) {
        piv_s = bi;
        if (blockIdx.x == 0) {
          ipiv[j] = bi;
          if (!(best > 0.f) || !isfinite(best) || bi >= n) atomicOr(err, 8);  // singular or non-finite
        }
      }
    }
    __syncthreads();
    const int p = piv_s;
    if (blockIdx.x == 0 && p != j && p < n)
      for (int c = k0 + (int)threadIdx.x; c < k1; c += blockDim.x) {
        const size_t a = (size_t)c * ld + j, b = (size_t)c * ld + p;
        const float tr = __ldcg(Ar + a), ti = __ldcg(Ai + a);
        Ar[a] = __ldcg(Ar + b);
        Ai[a] = __ldcg(Ai + b);
        Ar[b] = tr;
        Ai[b] = ti;
      }
    lu_grid_bar(bar, G);
    // row j is final: its pivot and its values in the sub-panel's later columns
    const float pr = __ldcg(Ar + (size_t)j * ld + j), pi = __ldcg(Ai + (size_t)j * ld + j);
    const float den = pr * pr + pi * pi;
    const int wj = s1 - j - 1;
    float ur[LU_SB], ui[LU_SB];
#pragma unroll
    for (int k = 0; k < LU_SB; k++)
      if (k < wj) {
        ur[k] = __ldcg(Ar + (size_t)(j + 1 + k) * ld + j);
        ui[k] = __ldcg(Ai + (size_t)(j + 1 + k) * ld + j);
      }
    float best = -1.f;
    int bi = n;
    for (int r = j + 1 + gtid; r < n; r += gstride) {
      // every load of the row first (one round trip to L2), then the arithmetic and stores
      float ar = __ldcg(Ar + (size_t)j * ld + r), ai = __ldcg(Ai + (size_t)j * ld + r);
      float xr[LU_SB], xi[LU_SB];
#pragma unroll
      for (int k = 0; k < LU_SB; k++)
        if (k < wj) {
          const size_t o = (size_t)(j + 1 + k) * ld + r;
          xr[k] = __ldcg(Ar + o);
          xi[k] = __ldcg(Ai + o);
        }
      const float lr = (ar * pr + ai * pi) / den, li = (ai * pr - ar * pi) / den;
      Ar[(size_t)j * ld + r] = lr;
      Ai[(size_t)j * ld + r] = li;
#pragma unroll
      for (int k = 0; k < LU_SB; k++)
        if (k < wj) {
          const size_t o = (size_t)(j + 1 + k) * ld + r;
          xr[k] -= lr * ur[k] - li * ui[k];
          xi[k] -= lr * ui[k] + li * ur[k];
          Ar[o] = xr[k];
          Ai[o] = xi[k];
        }
      if (wj > 0) argmax_pair(best, bi, xr[0] * xr[0] + xi[0] * xi[0], r);
    }
    if (j + 1 < s1) publish(best, bi);
    lu_grid_bar(bar, G);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && __ldcg(bar + 2) != 0) atomicOr(err, 16);  // a barrier gave up
}

// Sub-panel [s0, s1) of a panel ending at k1: its rows of the panel's later columns,
// U = L11^-1 A (L11 the unit lower triangle of the sub-panel's diagonal block).  Thread
// per column c in [s1, k1).
__global__ void k_sub_trsm(float* Ar, float* Ai, size_t ld, int s0, int s1, int k1) {
  const int c = s1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= k1) return;
  const int w = s1 - s0;
  float xr[LU_SB], xi[LU_SB];
  for (int i = 0; i < w; i++) {
    xr[i] = Ar[(size_t)c * ld + s0 + i];
    xi[i] = Ai[(size_t)c * ld + s0 + i];
  }
  for (int i = 1; i < w; i++)
    for (int t = 0; t < i; t++) {
      const float lr = Ar[(size_t)(s0 + t) * ld + s0 + i], li = Ai[(size_t)(s0 + t) * ld + s0 + i];
      xr[i] -= lr * xr[t] - li * xi[t];
      xi[i] -= lr * xi[t] + li * xr[t];
    }
  for (int i = 1; i < w; i++) {
    Ar[(size_t)c * ld + s0 + i] = xr[i];
    Ai[(size_t)c * ld + s0 + i] = xi[i];
  }
}

// Rank-w update of the panel's later columns by a factored sub-panel [s0, s1):
// a_rc -= sum_t l_rt u_tc for rows r >= s1 and columns c in [s1, k1).  The sub-panel's U
// rows in shared memory; thread per row.
__global__ void __launch_bounds__(256) k_sub_update(float* Ar, float* Ai, size_t ld, int n, int s0, int s1,
                                                    int k1) {
  __shared__ float ur[LU_SB][LU_NB], ui[LU_SB][LU_NB];
  const int w = s1 - s0, nc = k1 - s1;
  for (int e = threadIdx.x; e < w * nc; e += blockDim.x) {
    const int t = e / nc, c = e - t * nc;
    ur[t][c] = Ar[(size_t)(s1 + c) * ld + s0 + t];
    ui[t][c] = Ai[(size_t)(s1 + c) * ld + s0 + t];
  }
  __syncthreads();
  const int r = s1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float lr[LU_SB], li[LU_SB];
  for (int t = 0; t < w; t++) {
    lr[t] = Ar[(size_t)(s0 + t) * ld + r];
    li[t] = Ai[(size_t)(s0 + t) * ld + r];
  }
  for (int c = 0; c < nc; c++) {
    float sr = 0.f, si = 0.f;
#pragma unroll
    for (int t = 0; t < LU_SB; t++)
      if (t < w) {
        sr += lr[t] * ur[t][c] - li[t] * ui[t][c];
        si += lr[t] * ui[t][c] + li[t] * ur[t][c];
      }
    const size_t o = (size_t)(s1 + c) * ld + r;
    Ar[o] -= sr;
    Ai[o] -= si;
  }
}

// Row swaps ipiv[k0 .. k1) applied in order to the columns [c, c + 1) of every thread
// outside the panel [k0, k1).
__global__ void k_laswp(float* Ar, float* Ai, size_t ld, int n, int k0, int k1, const int* ipiv) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int outside = n - (k1 - k0);
  if (c >= outside) return;
  if (c >= k0) c += k1 - k0;
  float* cr = Ar + (size_t)c * ld;
  float* ci = Ai + (size_t)c * ld;
  for (int j = k0; j < k1; j++) {
    const int p = ipiv[j];
    if (p != j) {
      float t = cr[j];
      cr[j] = cr[p];
      cr[p] = t;
      t = ci[j];
      ci[j] = ci[p];
      ci[p] = t;
    }
  }
}

// X = L^-1 X in place for a diagonal block of the factors: L the unit lower triangle of
// the nb x nb block at (k0, k0) (nb <= LU_TB), X its rows [k0, k0 + nb) in columns [c0, n).
// L in shared memory; one warp per column, lane l holding rows l, l + 32, l + 64, l + 96.
__global__ void __launch_bounds__(256) k_trsm_l(float* Ar, float* Ai, size_t ld, int n, int k0, int nb, int c0) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float* Lr = reinterpret_cast<float*>(smraw);  // [col][row], nb x nb
  float* Li = Lr + LU_TB * LU_TB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int col = e / nb, row = e - col * nb;
    Lr[col * LU_TB + row] = Ar[(size_t)(k0 + col) * ld + k0 + row];
    Li[col * LU_TB + row] = Ai[(size_t)(k0 + col) * ld + k0 + row];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = c0 + blockIdx.x * 8 + warp; c < n; c += gridDim.x * 8) {
    float* cr = Ar + (size_t)c * ld + k0;
    float* ci = Ai + (size_t)c * ld + k0;
    float xr[4], xi[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = lane + 32 * q;
      xr[q] = r < nb ? cr[r] : 0.f;
      xi[q] = r < nb ? ci[r] : 0.f;
    }
    for (int i = 0; i < nb; i++) {
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
          const float lr = Lr[i * LU_TB + r], li = Li[i * LU_TB + r];
          xr[q] -= lr * vr - li * vi;
          xi[q] -= lr * vi + li * vr;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = lane + 32 * q;
      if (r < nb) {
        cr[r] = xr[q];
        ci[r] = xi[q];
      }
    }
  }
}

// Solves with the factors, one vector (complex64, internal order) in place.  Diagonal
// block: x[k0 .. k0 + nb) = L11^-1 x (lower, unit diagonal) or U11^-1 x (upper), with the
// block staged in shared memory first (coalesced), then one warp runs the substitution.
__global__ void __launch_bounds__(256) k_trsv_block(const float* Ar, const float* Ai, size_t ld, int k0, int nb,
                                                    int lower, cc* x) {
  extern __shared__ __align__(16) unsigned char smraw[];
  float* Dr = reinterpret_cast<float*>(smraw);  // [col][row]
  float* Di = Dr + LU_TB * LU_TB;
  __shared__ float br[LU_TB], bi[LU_TB];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int col = e / nb, row = e - col * nb;
    Dr[col * LU_TB + row] = Ar[(size_t)(k0 + col) * ld + k0 + row];
    Di[col * LU_TB + row] = Ai[(size_t)(k0 + col) * ld + k0 + row];
  }
  for (int r = threadIdx.x; r < nb; r += blockDim.x) {
    br[r] = x[k0 + r].re;
    bi[r] = x[k0 + r].im;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lower) {
      for (int i = 0; i < nb; i++) {
        const float vr = br[i], vi = bi[i];
        __syncwarp();
        for (int r = i + 1 + lane; r < nb; r += 32) {
          const float lr = Dr[i * LU_TB + r], li = Di[i * LU_TB + r];
          br[r] -= lr * vr - li * vi;
          bi[r] -= lr * vi + li * vr;
        }
        __syncwarp();
      }
    } else {
      for (int i = nb - 1; i >= 0; i--) {
        if (lane == 0) {
          const float ur = Dr[i * LU_TB + i], ui = Di[i * LU_TB + i];
          const float den = ur * ur + ui * ui;
          const float xr = (br[i] * ur + bi[i] * ui) / den, xi = (bi[i] * ur - br[i] * ui) / den;
          br[i] = xr;
          bi[i] = xi;
        }
        __syncwarp();
        const float vr = br[i], vi = bi[i];
        for (int r = lane; r < i; r += 32) {
          const float ur = Dr[i * LU_TB + r], ui = Di[i * LU_TB + r];
          br[r] -= ur * vr - ui * vi;
          bi[r] -= ur * vi + ui * vr;
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  for (int r = threadIdx.x; r < nb; r += blockDim.x) x[k0 + r] = mk<float>(br[r], bi[r]);
}

// x[rows r0 .. r1) -= A[r0 .. r1, k0 .. k0 + nb) x[k0 .. k0 + nb); thread per row.
__global__ void __launch_bounds__(256) k_trsv_gemv(const float* Ar, const float* Ai, size_t ld, int k0, int nb,
                                                   int r0, int r1, cc* x) {
  __shared__ float br[LU_TB], bi[LU_TB];
  for (int r = threadIdx.x; r < nb; r += blockDim.x) {
    br[r] = x[k0 + r].re;
    bi[r] = x[k0 + r].im;
  }
  __syncthreads();
  const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r1) return;
  float sr = 0.f, si = 0.f;
  for (int j = 0; j < nb; j++) {
    const float ar = Ar[(size_t)(k0 + j) * ld + i], ai = Ai[(size_t)(k0 + j) * ld + i];
    sr += ar * br[j] - ai * bi[j];
    si += ar * bi[j] + ai * br[j];
  }
  x[i].re -= sr;
  x[i].im -= si;
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
  if (c->d_lu32) return SIE_OK;
  const int n = 2 * c->M;
  const size_t ld = (size_t)n;
  cudaStream_t s = c->stream;
  float *Ar = nullptr, *Ai = nullptr;
  int *ipiv = nullptr, *err = nullptr;
  char *At = nullptr, *Bt = nullptr;
  void* pscr = nullptr;  // pivot search: per-block maxima and indices, and the block counter
  int rc = SIE_OK;
  auto cleanup = [&]() {
    if (At) cudaFree(At);
    if (Bt) cudaFree(Bt);
    if (err) cudaFree(err);
    if (pscr) cudaFree(pscr);
  };
  SIE_CUDA(cudaMalloc(&Ar, ld * n * sizeof(float)));
  if (cudaMalloc(&Ai, ld * n * sizeof(float)) != cudaSuccess || cudaMalloc(&ipiv, (size_t)n * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&At, tc::tiled_bytes_host(n, LU_NB)) != cudaSuccess ||
      cudaMalloc(&Bt, tc::tiled_bytes_host(n, LU_NB)) != cudaSuccess ||
      cudaMalloc(&pscr, (size_t)PANEL_MAX_BLOCKS * 8 + 64) != cudaSuccess) {
    cudaFree(Ar);
    if (Ai) cudaFree(Ai);
    if (ipiv) cudaFree(ipiv);
    cleanup();
    return fail(SIE_ERR_NOMEM, "mixed LU: device memory");
  }
  c->d_lu32 = Ar;
  c->d_lu32i = Ai;
  c->d_piv32 = ipiv;
  auto t0 = std::chrono::steady_clock::now();
  cudaMemsetAsync(err, 0, sizeof(int), s);
  float* pmax = (float*)pscr;
  int* pidx = (int*)((char*)pscr + (size_t)PANEL_MAX_BLOCKS * 4);
  unsigned* pbar = (unsigned*)((char*)pscr + (size_t)PANEL_MAX_BLOCKS * 8);  // count, generation, error
  cudaMemsetAsync(pbar, 0, 4 * sizeof(unsigned), s);
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
  if (raise_smem(k_trsm_l, trsm_smem) != cudaSuccess) rc = fail(SIE_ERR_CUDA, "mixed LU: shared memory");
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
  // the cooperative panel kernel: blocks that fit on the multiprocessors the look-ahead
  // update leaves free (all of them resident at once)
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subpanel, 256, 0) != cudaSuccess) per_sm = 1;
  const int panel_blocks = std::max(1, std::min(PANEL_MAX_BLOCKS, std::min(per_sm, 4) * std::max(free_sms, 1)));
  s = sp;  // the phase marks and the panel chain
  bool rest_pending = false;
  for (int k0 = 0; k0 < n && rc == SIE_OK; k0 += LU_NB) {
    const int nb = std::min(LU_NB, n - k0), k1 = k0 + nb;
    mark(0, true, pk);
    // the panel in sub-panels of LU_SB columns: column steps inside the sub-panel, then
    // one rank-LU_SB update of the panel's later columns
    for (int s0 = k0; s0 < k1; s0 += LU_SB) {
      const int s1 = std::min(s0 + LU_SB, k1);
      {
        int ns0 = s0, ns1 = s1, nn0 = n, kk0 = k0, kk1 = k1;
        size_t ldd = ld;
        void* args[] = {&Ar, &Ai, &ldd, &nn0, &ns0, &ns1, &kk0, &kk1, &ipiv, &err, &pmax, &pidx, &pbar};
        if (cudaLaunchCooperativeKernel((const void*)k_subpanel, dim3(panel_blocks), dim3(256), args, 0, sp) !=
            cudaSuccess) {
          rc = fail(SIE_ERR_CUDA, "mixed LU: cooperative panel launch");
          break;
        }
        count_launch();
      }
      if (s1 < k1) {
        k_sub_trsm<<<1, LU_NB, 0, sp>>>(Ar, Ai, ld, s0, s1, k1);
        count_launch();
        if (s1 < n) {
          k_sub_update<<<(n - s1 + 255) / 256, 256, 0, sp>>>(Ar, Ai, ld, n, s0, s1, k1);
          count_launch();
        }
      }
    }
    mark(0, false, pk);
    if (rest_pending) cudaStreamWaitEvent(sp, ev_rest, 0);  // the previous trailing update
    mark(1, true, pk);
    if (n - nb > 0) {
      k_laswp<<<(n - nb + 255) / 256, 256, 0, sp>>>(Ar, Ai, ld, n, k0, k1, ipiv);
      count_launch();
    }
    mark(1, false, pk);
    if (k1 < n) {
      mark(2, true, pk);
      // U12 = L11^-1 A12 by diagonal blocks of LU_TB: each block's rows are solved, then the
      // rows below it in the panel lose L21-block times them (a tensor-core update)
      for (int d0 = k0; d0 < k1 && rc == SIE_OK; d0 += LU_TB) {
        const int db = std::min(LU_TB, k1 - d0), d1 = d0 + db;
        k_trsm_l<<<std::min(1184, (n - k1 + 7) / 8), 256, trsm_smem, sp>>>(Ar, Ai, ld, n, d0, db, k1);
        count_launch();
        if (d1 < k1) {
          const int mb = k1 - d1;
          rc = tc::tile_operand(Ar + (size_t)d0 * ld + d1, Ai + (size_t)d0 * ld + d1, ld, mb, db, false, At, sp);
          if (rc == SIE_OK)
            rc = tc::tile_operand(Ar + (size_t)k1 * ld + d0, Ai + (size_t)k1 * ld + d0, ld, n - k1, db, true, Bt, sp);
          if (rc == SIE_OK)
            rc = tc::gemm_update(At, Bt, db, Ar + (size_t)k1 * ld + d1, Ai + (size_t)k1 * ld + d1, ld, mb, n - k1,
                                 err, sp);
        }
      }
      mark(2, false, pk);
      const int m = n - k1, nn = std::min(LU_NB, m);
      // A22 -= L21 U12 on the tensor cores
      mark(3, true, pk);
      rc = tc::tile_operand(Ar + (size_t)k0 * ld + k1, Ai + (size_t)k0 * ld + k1, ld, m, nb, false, At, sp);
      if (rc == SIE_OK) rc = tc::tile_operand(Ar + (size_t)k1 * ld + k0, Ai + (size_t)k1 * ld + k0, ld, m, nb, true, Bt, sp);
      mark(3, false, pk);
      cudaEventRecord(ev_tiled, sp);
      const cudaStream_t srest = lookahead ? sg : sp;
      if (rc == SIE_OK && m > nn) {
        // the columns past the next panel, on sg
        cudaStreamWaitEvent(sg, ev_tiled, 0);
        cudaEvent_t e0 = new_event(), e1 = new_event();
        if (e0) cudaEventRecord(e0, srest);
        // the B tiles past the next panel's nn columns
        const size_t boff = (size_t)(nn / tc::TILE) * ((nb + tc::KC - 1) / tc::KC) * tc::BLOCK_BYTES;
        rc = tc::gemm_update(At, Bt + boff, nb, Ar + (size_t)(k1 + nn) * ld + k1, Ai + (size_t)(k1 + nn) * ld + k1,
                             ld, m, m - nn, err, srest, lookahead ? rest_ctas : 0);
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
        rc = tc::gemm_update(At, Bt, nb, Ar + (size_t)k1 * ld + k1, Ai + (size_t)k1 * ld + k1, ld, m, nn, err, sp);
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
    if (rc == SIE_OK && (cudaMalloc(&c->d_perm32, (size_t)n * sizeof(int)) != cudaSuccess ||
                         cudaMalloc(&c->d_tmp32, (size_t)n * sizeof(cc)) != cudaSuccess ||
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
  cleanup();
  if (rc != SIE_OK) {
    for (void* p : {(void*)c->d_lu32, (void*)c->d_lu32i, (void*)c->d_piv32, (void*)c->d_perm32, (void*)c->d_tmp32})
      if (p) cudaFree(p);
    c->d_lu32 = c->d_lu32i = nullptr;
    c->d_piv32 = c->d_perm32 = nullptr;
    c->d_tmp32 = nullptr;
  }
  return rc;
}

// x = U^-1 L^-1 P x with the complex64 factors (internal order, in place).
static int lu_tc_solve32(sie_ctx* c, cc* x, cudaStream_t s) {
  const int n = 2 * c->M;
  const size_t ld = (size_t)n;
  const float *Ar = c->d_lu32, *Ai = c->d_lu32i;
  k_permute<<<148, 256, 0, s>>>(c->d_perm32, n, x, c->d_tmp32);
  count_launch();
  SIE_CUDA(cudaMemcpyAsync(x, c->d_tmp32, (size_t)n * sizeof(cc), cudaMemcpyDeviceToDevice, s));
  const size_t dsm = (size_t)2 * LU_TB * LU_TB * sizeof(float);
  SIE_CUDA(raise_smem(k_trsv_block, dsm));
  for (int k0 = 0; k0 < n; k0 += LU_TB) {
    const int nb = std::min(LU_TB, n - k0), k1 = k0 + nb;
    k_trsv_block<<<1, 256, dsm, s>>>(Ar, Ai, ld, k0, nb, 1, x);
    count_launch();
    if (k1 < n) {
      k_trsv_gemv<<<(n - k1 + 255) / 256, 256, 0, s>>>(Ar, Ai, ld, k0, nb, k1, n, x);
      count_launch();
    }
  }
  for (int k0 = ((n - 1) / LU_TB) * LU_TB; k0 >= 0; k0 -= LU_TB) {
    const int nb = std::min(LU_TB, n - k0);
    k_trsv_block<<<1, 256, dsm, s>>>(Ar, Ai, ld, k0, nb, 0, x);
    count_launch();
    if (k0 > 0) {
      k_trsv_gemv<<<(k0 + 255) / 256, 256, 0, s>>>(Ar, Ai, ld, k0, nb, 0, k0, x);
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
  SIE_TRY(lu_tc_factor(c));
  const int n = 2 * c->M;
  const size_t bytes = (size_t)n * sizeof(zc);
  zc *bi = nullptr, *xi = nullptr, *ax = nullptr, *r = nullptr;
  cc* d32 = nullptr;
  double* nrm = nullptr;
  int rc = SIE_OK;
  if (cudaMalloc(&bi, bytes) != cudaSuccess || cudaMalloc(&xi, bytes) != cudaSuccess ||
      cudaMalloc(&ax, bytes) != cudaSuccess || cudaMalloc(&r, bytes) != cudaSuccess ||
      cudaMalloc(&d32, (size_t)n * sizeof(cc)) != cudaSuccess || cudaMalloc(&nrm, sizeof(double)) != cudaSuccess)
    rc = fail(SIE_ERR_NOMEM, "mixed direct solve: device buffers");
  for (int k = 0; k < nrhs && rc == SIE_OK; k++) {
    auto tk = std::chrono::steady_clock::now();
    const size_t off = (size_t)k * n;
    double bn2 = 0, rn2 = 0;
    int steps = 0;
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
      if (cudaMemcpyAsync(&rn2, nrm, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = fail(SIE_ERR_CUDA, "mixed direct solve: residual");
        break;
      }
      if (steps == 0) bn2 = rn2;
      if (!std::isfinite(rn2)) {
        rc = fail(SIE_ERR_NONFINITE, "mixed direct solve: non-finite residual");
        break;
      }
      if (bn2 == 0.0 || rn2 <= tolerance * tolerance * bn2 || steps > max_refinements) break;
      const double rn = std::sqrt(rn2);
      k_scale_to32<<<296, 256, 0, s>>>(r, d32, n, 1.0 / rn);
      count_launch();
      rc = lu_tc_solve32(c, d32, s);
      if (rc != SIE_OK) break;
      k_add_from32<<<296, 256, 0, s>>>(xi, d32, n, rn);
      count_launch();
    }
    if (rc != SIE_OK) break;
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
  for (void* p : {(void*)bi, (void*)xi, (void*)ax, (void*)r, (void*)d32, (void*)nrm})
    if (p) cudaFree(p);
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
  zc *db = nullptr, *dx = nullptr;
  SIE_CUDA(cudaMalloc(&db, bytes));
  if (cudaMalloc(&dx, bytes) != cudaSuccess) {
    cudaFree(db);
    return fail(SIE_ERR_NOMEM, "sie_solve_direct_mixed: device buffers");
  }
  int rc = SIE_OK;
  if (cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct_mixed: copy");
  if (rc == SIE_OK) rc = solve_direct_mixed_dev(c, db, dx, nrhs, tolerance, max_refinements, stats, c->stream);
  if ((rc == SIE_OK || rc == SIE_ERR_NOCONV) &&
      (cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
       cudaStreamSynchronize(c->stream) != cudaSuccess))
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct_mixed: copy back");
  cudaFree(db);
  cudaFree(dx);
  return rc;
}

extern "C" int sie_release_factors(sie_ctx* c) {
  if (!c) return fail(SIE_ERR_ARG, "sie_release_factors: null context");
  SIE_CUDA(cudaSetDevice(c->device));
  if (c->stream) SIE_CUDA(cudaStreamSynchronize(c->stream));
  for (void* p : {(void*)c->d_lu, (void*)c->d_piv, (void*)c->d_lu32, (void*)c->d_lu32i, (void*)c->d_piv32,
                  (void*)c->d_perm32, (void*)c->d_tmp32})
    if (p) cudaFree(p);
  c->d_lu = nullptr;
  c->d_piv = nullptr;
  c->d_lu32 = c->d_lu32i = nullptr;
  c->d_piv32 = c->d_perm32 = nullptr;
  c->d_tmp32 = nullptr;
  return SIE_OK;
}
