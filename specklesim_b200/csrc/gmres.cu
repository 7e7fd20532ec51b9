// Restarted GMRES on the GPU with the semantics of the CERFACS zgmres driver
// used by the reference (src/lib/libmath_external/src/algorithm_842/zPackgmres.f90
// :537-1565, called through lib_math_solver_gmres_run,
// src/lib/libmath/src/math/lib_math_solver_GMRES.f90:159-379): iterative modified
// Gram-Schmidt (icntl(5) = 1), BLAS Givens rotations (zrotg/zrot), convergence
// on the Arnoldi backward error ||r||/||b|| confirmed by the true residual, and
// the recurrence for the restart residual (icntl(8) = 0).
//
// All vectors and the Hessenberg matrix stay on the device; the host only reads
// a few scalars per Arnoldi step to steer the iteration.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <vector>

#include <cooperative_groups.h>

#include "sie_internal.h"

namespace sie {

static const int RB = 296;   // reduction blocks (2 x 148 SMs)
static const int RT_ = 256;  // threads per reduction block

struct GmState {
  // scalars shared between the small kernels
  double dloo2;     // sum |h|^2 of the current pass
  double dnormw;
  double dloo;
  double bea;
  double nrm;       // generic norm result
  int reorth;
  int passes;       // MGS passes of the last Arnoldi step
  unsigned bar_count, bar_gen;  // grid barrier of the fused Arnoldi kernel
  int bar_err;      // set if a grid barrier wait gave up
  int spin_limit;   // polls before a barrier or exchange wait gives up (<= 0: the default)
};

// Polls of one grid-barrier or exchange wait before it gives up: about a second by
// default; SIE_GRID_SPIN_LIMIT in the environment sets it (a test makes the waits run out).
static int grid_spin_limit_host() {
  const char* e = getenv("SIE_GRID_SPIN_LIMIT");
  return e ? std::max(1, atoi(e)) : 0;
}
__device__ __forceinline__ long long spin_limit(const GmState* gs, long long dflt) {
  const int v = *(volatile const int*)&gs->spin_limit;
  return v > 0 ? (long long)v : dflt;
}

__device__ __forceinline__ zc warp_sum(zc v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.re += __shfl_xor_sync(0xffffffff, v.re, o);
    v.im += __shfl_xor_sync(0xffffffff, v.im, o);
  }
  return v;
}

// block-wide sum, result valid in thread 0
__device__ zc block_sum(zc v) {
  __shared__ zc sh[32];
  v = warp_sum(v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  zc r = mk<double>(0, 0);
  if (threadIdx.x < 32) {
    r = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : mk<double>(0, 0);
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

// Sum of the per-block partials in a fixed order (every block computes the same value).
__device__ zc reduce_partials(const zc* part, int np) {
  __shared__ zc res;
  zc v = mk<double>(0, 0);
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
  v = block_sum(v);
  if (threadIdx.x == 0) res = v;
  __syncthreads();
  zc r = res;
  __syncthreads();
  return r;
}

// Same, reading the partials from L2 (they were written by other SMs inside the same
// kernel, so an L1 line from an earlier use of the buffer may be stale).
__device__ zc reduce_partials_l2(const zc* part, int np) {
  __shared__ zc res2;
  zc v = mk<double>(0, 0);
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    double2 t = __ldcg(reinterpret_cast<const double2*>(part) + i);
    v += mk<double>(t.x, t.y);
  }
  v = block_sum(v);
  if (threadIdx.x == 0) res2 = v;
  __syncthreads();
  zc r = res2;
  __syncthreads();
  return r;
}

// One fused MGS step: finish h_j = <V_j, w> from the partials of the previous
// launch, w -= h_j V_j, and start <V_next, w> (next >= 0) or ||w||^2 (next < 0).
__global__ void __launch_bounds__(RT_) k_mgs(zc* __restrict__ w, const zc* __restrict__ Vj,
                                             const zc* __restrict__ Vn, const zc* part_in,
                                             zc* part_out, int n, zc* Hcol, int j, GmState* gs) {
  zc h = mk<double>(0, 0);
  if (Vj) {
    h = reduce_partials(part_in, gridDim.x);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      Hcol[j] += h;
      gs->dloo2 += cabs2(h);
    }
  }
  zc acc = mk<double>(0, 0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    zc wi = w[i];
    if (Vj) {
      wi = wi - h * Vj[i];
      w[i] = wi;
    }
    if (Vn)
      acc = cfma_conj(Vn[i], wi, acc);
    else
      acc.re += cabs2(wi);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part_out[blockIdx.x] = acc;
}

// partial dot <a, b> (or ||a||^2 when b == nullptr)
__global__ void __launch_bounds__(RT_) k_dot(const zc* a, const zc* b, int n, zc* part_out) {
  zc acc = mk<double>(0, 0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (b)
      acc = cfma_conj(a[i], b[i], acc);
    else
      acc.re += cabs2(a[i]);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part_out[blockIdx.x] = acc;
}

__global__ void k_norm_final(const zc* part, int np, GmState* gs) {
  zc s = reduce_partials(part, np);
  if (threadIdx.x == 0) gs->nrm = sqrt(s.re);
}

// end of an MGS pass: dnormw, dloo and the IMGS re-orthogonalisation test
__global__ void k_pass_final(const zc* part, int np, GmState* gs, int northo) {
  zc s = reduce_partials(part, np);
  if (threadIdx.x == 0) {
    double dnormw = sqrt(s.re);
    double dloo = sqrt(gs->dloo2);
    gs->dnormw = dnormw;
    gs->dloo = dloo;
    gs->reorth = (dnormw <= dloo && northo < 3) ? 1 : 0;
  }
}

__global__ void k_scale_copy(const zc* w, zc* v, int n, const GmState* gs) {
  double inv = 1.0 / gs->dnormw;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = w[i] * inv;
}
__global__ void k_scale_copy_s(const zc* w, zc* v, int n, double beta) {
  double inv = 1.0 / beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = w[i] * inv;
}
__global__ void k_copy(const zc* a, zc* b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ void k_zero(zc* a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    a[i] = mk<double>(0, 0);
}
// c = a - b
__global__ void k_sub(const zc* a, const zc* b, zc* c, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    c[i] = a[i] - b[i];
}
// c = a + b
__global__ void k_add(const zc* a, const zc* b, zc* c, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    c[i] = a[i] + b[i];
}
// y = a + V(:, 0:k) coef (coef on the device)
__global__ void k_combine(const zc* a, const zc* V, const zc* coef, int k, int n, size_t ld, zc* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    zc s = a ? a[i] : mk<double>(0, 0);
    for (int j = 0; j < k; j++) s = cfma(V[(size_t)j * ld + i], coef[j], s);
    y[i] = s;
  }
}

// BLAS zrotg (reference BLAS): c real, s complex
__device__ void zrotg(zc ca, zc cb, double& c, zc& s) {
  double aca = sqrt(cabs2(ca));
  if (aca == 0.0) {
    c = 0.0;
    s = mk<double>(1.0, 0.0);
    return;
  }
  double acb = sqrt(cabs2(cb));
  double scale = aca + acb;
  double na = aca / scale, nb = acb / scale;
  double norm = scale * sqrt(na * na + nb * nb);
  zc alpha = ca / aca;
  c = aca / norm;
  s = alpha * conj(cb) / norm;
}
// BLAS zrot on one pair: x' = c x + s y ; y' = c y - conj(s) x
__device__ __forceinline__ void zrot(zc& x, zc& y, double c, zc s) {
  zc t = x * c + s * y;
  y = y * c - conj(s) * x;
  x = t;
}

// H is (m+1) x (m+1), column-major with leading dimension m+1; column m holds the rhs.
#define HIDX(i, j) ((size_t)(j) * (m + 1) + (i))

// New column jh (0-based) of H: H(jh+1, jh) = dnormw, previous rotations, new
// rotation, rhs update, bea = |H(jh+1, m)| / bn.
__global__ void k_givens(zc* H, int m, int jh, double* rc, zc* rs, GmState* gs, double bn) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  H[HIDX(jh + 1, jh)] = mk<double>(gs->dnormw, 0.0);
  for (int j = 0; j < jh; j++) zrot(H[HIDX(j, jh)], H[HIDX(j + 1, jh)], rc[j], rs[j]);
  double c;
  zc s;
  zrotg(H[HIDX(jh, jh)], H[HIDX(jh + 1, jh)], c, s);
  rc[jh] = c;
  rs[jh] = s;
  zrot(H[HIDX(jh, m)], H[HIDX(jh + 1, m)], c, s);
  zrot(H[HIDX(jh, jh)], H[HIDX(jh + 1, jh)], c, s);
  H[HIDX(jh + 1, jh)] = mk<double>(0, 0);
  gs->bea = sqrt(cabs2(H[HIDX(jh + 1, m)])) / bn;
}

// Grid-wide barrier of the fused Arnoldi kernel.  The kernel is launched cooperatively,
// so all its blocks are resident; the wait is still bounded: a block that sees no
// progress for about a second records the failure in bar_err and stops waiting, later
// barriers then pass straight through, and the host reports the error.
__device__ void grid_bar(GmState* gs, unsigned nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &gs->bar_gen;
    volatile int* err = &gs->bar_err;
    if (*err == 0) {
      unsigned g = *gen;
      __threadfence();
      unsigned arrived = atomicAdd(&gs->bar_count, 1u) + 1u;
      if (arrived == nblocks) {
        atomicExch(&gs->bar_count, 0u);
        __threadfence();
        atomicAdd(&gs->bar_gen, 1u);
      } else {
        long long it = 0;
        const long long lim = spin_limit(gs, 1LL << 24);
        while (*gen == g && *err == 0) {
          if (++it > lim) {
            atomicExch(&gs->bar_err, 1);
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

// One Arnoldi step after the matvec, fused: iterative modified Gram-Schmidt of w
// against V(:, 0:jH) (passes repeated while dnormw <= dloo, at most 3), H(:, jH),
// V(:, jH+1) = w / dnormw, and the Givens update of column jH with the Arnoldi
// backward error.  Every block reduces the per-block partials in the same order, so
// all blocks see the same h_j and take the same re-orthogonalisation decision.
// store a complex128 value in the storage precision of a Krylov basis
template <typename VT> __device__ __forceinline__ cx<VT> narrow(zc a);
template <> __device__ __forceinline__ zc narrow<double>(zc a) { return a; }
template <> __device__ __forceinline__ cc narrow<float>(zc a) { return mk<float>((float)a.re, (float)a.im); }

template <typename VT>
__global__ void __launch_bounds__(512) k_arnoldi(cx<VT>* __restrict__ w, cx<VT>* __restrict__ V, size_t ld,
                                                 int n, int jH, zc* H, int m, double* rc, zc* rs,
                                                 zc* part, GmState* gs, double bn) {
  const unsigned nb = gridDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  zc* Hc = H + (size_t)jH * (m + 1);
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i <= jH; i += blockDim.x) Hc[i] = mk<double>(0, 0);
  int buf = 0, pass = 1;
  double dnormw = 0, dloo = 0;
  for (;; pass++) {
    double dloo2 = 0;
    zc acc = mk<double>(0, 0);
    for (int i = t0; i < n; i += stride) acc = cfma_conj(cvt_z(V[i]), cvt_z(w[i]), acc);
    acc = block_sum(acc);
    if (threadIdx.x == 0) __stcg(reinterpret_cast<double2*>(part) + buf * nb + blockIdx.x, make_double2(acc.re, acc.im));
    grid_bar(gs, nb);
    for (int j = 0; j <= jH; j++) {
      const zc h = reduce_partials_l2(part + buf * nb, nb);
      buf ^= 1;
      if (blockIdx.x == 0 && threadIdx.x == 0) Hc[j] += h;
      dloo2 += cabs2(h);
      const cx<VT>* Vj = V + (size_t)j * ld;
      acc = mk<double>(0, 0);
      if (j < jH) {
        const cx<VT>* Vn = Vj + ld;
        for (int i = t0; i < n; i += stride) {
          zc wi = cvt_z(w[i]) - h * cvt_z(Vj[i]);
          w[i] = narrow<VT>(wi);
          acc = cfma_conj(cvt_z(Vn[i]), wi, acc);
        }
      } else {
        for (int i = t0; i < n; i += stride) {
          zc wi = cvt_z(w[i]) - h * cvt_z(Vj[i]);
          w[i] = narrow<VT>(wi);
          acc.re += cabs2(wi);
        }
      }
      acc = block_sum(acc);
      if (threadIdx.x == 0) __stcg(reinterpret_cast<double2*>(part) + buf * nb + blockIdx.x, make_double2(acc.re, acc.im));
      grid_bar(gs, nb);
    }
    const zc s2 = reduce_partials_l2(part + buf * nb, nb);
    buf ^= 1;
    dnormw = sqrt(s2.re);
    dloo = sqrt(dloo2);
    if (!(dnormw <= dloo && pass < 3)) break;
  }
  cx<VT>* Vnew = V + (size_t)(jH + 1) * ld;
  const double inv = 1.0 / dnormw;
  for (int i = t0; i < n; i += stride) Vnew[i] = narrow<VT>(cvt_z(w[i]) * inv);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    gs->dnormw = dnormw;
    gs->dloo = dloo;
    gs->passes = pass;
    H[HIDX(jH + 1, jH)] = mk<double>(dnormw, 0.0);
    for (int j = 0; j < jH; j++) zrot(H[HIDX(j, jH)], H[HIDX(j + 1, jH)], rc[j], rs[j]);
    double c;
    zc sn;
    zrotg(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    rc[jH] = c;
    rs[jH] = sn;
    zrot(H[HIDX(jH, m)], H[HIDX(jH + 1, m)], c, sn);
    zrot(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    H[HIDX(jH + 1, jH)] = mk<double>(0, 0);
    gs->bea = sqrt(cabs2(H[HIDX(jH + 1, m)])) / bn;
  }
}

// ---------------------------------------------------------------------------
// Register-resident variant of the fused Arnoldi step for n <= 148 x 512 x 8.  Each
// thread keeps EPT elements of w in registers for the whole step.  A global reduction is
// one all-to-all exchange: every block publishes its partial in its own slot of the
// round's buffer with a round tag, and every block reads all slots in the same order,
// so all blocks get bit-identical sums with no separate barrier.  The next basis
// column is loaded while the exchange is in flight.
struct __align__(32) ArSlot {
  double re, im;
  unsigned tag;
  unsigned pad[3];
};
static const int AR_THREADS = 512;

__device__ zc ar_allreduce(zc v, ArSlot* slots, unsigned round, unsigned tag, int nb, GmState* gs) {
  __shared__ zc bc;
  v = block_sum(v);
  ArSlot* buf = slots + (size_t)(round & 1u) * nb;
  if (threadIdx.x == 0) {
    __stcg(&buf[blockIdx.x].re, v.re);
    __stcg(&buf[blockIdx.x].im, v.im);
    __threadfence();
    atomicExch(&buf[blockIdx.x].tag, tag);
  }
  if (threadIdx.x < 32) {
    zc acc = mk<double>(0, 0);
    for (int i = threadIdx.x; i < nb; i += 32) {
      volatile unsigned* pt = &buf[i].tag;
      long long it = 0;
      const long long lim = spin_limit(gs, 1LL << 22);
      while (*pt != tag) {
        if (*(volatile int*)&gs->bar_err) break;
        if (++it > lim) {
          atomicExch(&gs->bar_err, 1);
          break;
        }
      }
      __threadfence();
      acc += mk<double>(__ldcg(&buf[i].re), __ldcg(&buf[i].im));
    }
    acc = warp_sum(acc);
    if (threadIdx.x == 0) bc = acc;
  }
  __syncthreads();
  zc r = bc;
  __syncthreads();
  return r;
}

template <int EPT>
__global__ void __launch_bounds__(AR_THREADS, 1) k_arnoldi_reg(
    zc* __restrict__ w, zc* __restrict__ V, size_t ld, int n, int jH, zc* H, int m, double* rc,
    zc* rs, ArSlot* slots, unsigned epoch, GmState* gs, double bn) {
  const int nb = gridDim.x;
  const int i0 = blockIdx.x * AR_THREADS + threadIdx.x, stride = nb * AR_THREADS;
  zc wr[EPT], vr[EPT], vn[EPT];
#pragma unroll
  for (int e = 0; e < EPT; e++) {
    int i = i0 + e * stride;
    wr[e] = i < n ? w[i] : mk<double>(0, 0);
  }
  zc* Hc = H + (size_t)jH * (m + 1);
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i <= jH; i += blockDim.x) Hc[i] = mk<double>(0, 0);
  unsigned round = 0;
  auto tag = [&]() { return (epoch << 12) | (round & 4095u); };
  int pass = 1;
  double dnormw = 0, dloo = 0;
  for (;; pass++) {
    double dloo2 = 0;
    zc acc = mk<double>(0, 0);
#pragma unroll
    for (int e = 0; e < EPT; e++) {
      int i = i0 + e * stride;
      double2 t = i < n ? __ldcg(reinterpret_cast<const double2*>(V) + i) : make_double2(0.0, 0.0);
      vr[e] = mk<double>(t.x, t.y);
      acc = cfma_conj(vr[e], wr[e], acc);
    }
    for (int j = 0; j <= jH; j++) {
      if (j < jH) {
        const double2* Vn = reinterpret_cast<const double2*>(V + (size_t)(j + 1) * ld);
#pragma unroll
        for (int e = 0; e < EPT; e++) {
          int i = i0 + e * stride;
          double2 t = i < n ? __ldcg(Vn + i) : make_double2(0.0, 0.0);
          vn[e] = mk<double>(t.x, t.y);
        }
      }
      const zc h = ar_allreduce(acc, slots, round, tag(), nb, gs);
      round++;
      if (blockIdx.x == 0 && threadIdx.x == 0) Hc[j] += h;
      dloo2 += cabs2(h);
      acc = mk<double>(0, 0);
#pragma unroll
      for (int e = 0; e < EPT; e++) {
        wr[e] = wr[e] - h * vr[e];
        if (j < jH) {
          acc = cfma_conj(vn[e], wr[e], acc);
          vr[e] = vn[e];
        } else {
          acc.re += cabs2(wr[e]);
        }
      }
    }
    const zc s2 = ar_allreduce(acc, slots, round, tag(), nb, gs);
    round++;
    dnormw = sqrt(s2.re);
    dloo = sqrt(dloo2);
    if (!(dnormw <= dloo && pass < 3)) break;
  }
  const double inv = 1.0 / dnormw;
  zc* Vnew = V + (size_t)(jH + 1) * ld;
#pragma unroll
  for (int e = 0; e < EPT; e++) {
    int i = i0 + e * stride;
    if (i < n) {
      w[i] = wr[e];
      Vnew[i] = wr[e] * inv;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    gs->dnormw = dnormw;
    gs->dloo = dloo;
    gs->passes = pass;
    H[HIDX(jH + 1, jH)] = mk<double>(dnormw, 0.0);
    for (int j = 0; j < jH; j++) zrot(H[HIDX(j, jH)], H[HIDX(j + 1, jH)], rc[j], rs[j]);
    double c;
    zc sn;
    zrotg(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    rc[jH] = c;
    rs[jH] = sn;
    zrot(H[HIDX(jH, m)], H[HIDX(jH + 1, m)], c, sn);
    zrot(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    H[HIDX(jH + 1, jH)] = mk<double>(0, 0);
    gs->bea = sqrt(cabs2(H[HIDX(jH + 1, m)])) / bn;
  }
}

// ---------------------------------------------------------------------------
// Single-cluster variant for n <= 16 x 512 x 8: one thread-block cluster of up to 16
// CTAs (co-scheduled by the hardware) runs the whole Arnoldi step with w in registers.
// A global reduction is: block sum -> own shared-memory slot -> cluster barrier ->
// warp 0 reads the slots of all CTAs through distributed shared memory in rank order,
// so every CTA forms the same sum.  The next basis column is loaded before the barrier.
static const int CL_THREADS = 512;

// First half of a cluster reduction: block sum, publish it in this CTA's slot, arrive.
__device__ __forceinline__ void cl_publish(zc v, zc* slot, int buf) {
  v = block_sum(v);
  if (threadIdx.x == 0) slot[buf] = v;
  cooperative_groups::this_cluster().barrier_arrive();
}
// Second half: wait, sum the slots of all CTAs in rank order (warp 0), broadcast.
__device__ __forceinline__ zc cl_collect(zc* slot, zc* bc, int buf) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  cl.barrier_wait();
  if (threadIdx.x < 32) {
    const unsigned nr = cl.num_blocks();
    zc a = mk<double>(0, 0);
    if (threadIdx.x < nr) a = *cl.map_shared_rank(slot + buf, threadIdx.x);
    a = warp_sum(a);
    if (threadIdx.x == 0) bc[buf] = a;
  }
  __syncthreads();
  return bc[buf];
}

template <typename VT, int EPT>
__global__ void __launch_bounds__(CL_THREADS, 1) k_arnoldi_cl(
    cx<VT>* __restrict__ w, cx<VT>* __restrict__ V, size_t ld, int n, int jH, zc* H, int m, double* rc,
    zc* rs, GmState* gs, double bn) {
  __shared__ zc slot[2], bc[2];
  const int nb = gridDim.x;
  const int i0 = blockIdx.x * CL_THREADS + threadIdx.x, stride = nb * CL_THREADS;
  zc wr[EPT], vr[EPT], vn[EPT];
#pragma unroll
  for (int e = 0; e < EPT; e++) {
    int i = i0 + e * stride;
    wr[e] = i < n ? cvt_z(w[i]) : mk<double>(0, 0);
  }
  zc* Hc = H + (size_t)jH * (m + 1);
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i <= jH; i += blockDim.x) Hc[i] = mk<double>(0, 0);
  int buf = 0, pass = 1;
  double dnormw = 0, dloo = 0;
  for (;; pass++) {
    double dloo2 = 0;
    zc acc = mk<double>(0, 0);
#pragma unroll
    for (int e = 0; e < EPT; e++) {
      int i = i0 + e * stride;
      vr[e] = i < n ? cvt_z(V[i]) : mk<double>(0, 0);
      acc = cfma_conj(vr[e], wr[e], acc);
    }
    for (int j = 0; j <= jH; j++) {
      cl_publish(acc, slot, buf);
      if (j < jH) {  // the next column streams in while the cluster barrier completes
        const cx<VT>* Vn = V + (size_t)(j + 1) * ld;
#pragma unroll
        for (int e = 0; e < EPT; e++) {
          int i = i0 + e * stride;
          vn[e] = i < n ? cvt_z(Vn[i]) : mk<double>(0, 0);
        }
      }
      const zc h = cl_collect(slot, bc, buf);
      buf ^= 1;
      if (blockIdx.x == 0 && threadIdx.x == 0) Hc[j] += h;
      dloo2 += cabs2(h);
      acc = mk<double>(0, 0);
#pragma unroll
      for (int e = 0; e < EPT; e++) {
        wr[e] = wr[e] - h * vr[e];
        if (j < jH) {
          acc = cfma_conj(vn[e], wr[e], acc);
          vr[e] = vn[e];
        } else {
          acc.re += cabs2(wr[e]);
        }
      }
    }
    cl_publish(acc, slot, buf);
    const zc s2 = cl_collect(slot, bc, buf);
    buf ^= 1;
    dnormw = sqrt(s2.re);
    dloo = sqrt(dloo2);
    if (!(dnormw <= dloo && pass < 3)) break;
  }
  const double inv = 1.0 / dnormw;
  cx<VT>* Vnew = V + (size_t)(jH + 1) * ld;
#pragma unroll
  for (int e = 0; e < EPT; e++) {
    int i = i0 + e * stride;
    if (i < n) {
      w[i] = narrow<VT>(wr[e]);
      Vnew[i] = narrow<VT>(wr[e] * inv);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    gs->dnormw = dnormw;
    gs->dloo = dloo;
    gs->passes = pass;
    H[HIDX(jH + 1, jH)] = mk<double>(dnormw, 0.0);
    for (int j = 0; j < jH; j++) zrot(H[HIDX(j, jH)], H[HIDX(j + 1, jH)], rc[j], rs[j]);
    double c;
    zc sn;
    zrotg(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    rc[jH] = c;
    rs[jH] = sn;
    zrot(H[HIDX(jH, m)], H[HIDX(jH + 1, m)], c, sn);
    zrot(H[HIDX(jH, jH)], H[HIDX(jH + 1, jH)], c, sn);
    H[HIDX(jH + 1, jH)] = mk<double>(0, 0);
    gs->bea = sqrt(cabs2(H[HIDX(jH + 1, m)])) / bn;
  }
  // no CTA may leave while another still reads its slots
  cooperative_groups::this_cluster().sync();
}

// y = H(0:k, 0:k)^{-1} H(0:k, m)   (ztrsv 'U','N','N')
__global__ void k_trsv(const zc* H, int m, int k, zc* y) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < k; i++) y[i] = H[HIDX(i, m)];
  for (int i = k - 1; i >= 0; i--) {
    y[i] = y[i] / H[HIDX(i, i)];
    for (int j = 0; j < i; j++) y[j] = y[j] - y[i] * H[HIDX(j, i)];
  }
}

// restart recurrence: beta = |H(m, m)|; rotations in reverse on column m
__global__ void k_restart_rhs(zc* H, int m, const double* rc, const zc* rs, GmState* gs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  gs->nrm = sqrt(cabs2(H[HIDX(m, m)]));
  for (int j = m - 1; j >= 0; j--) {
    H[HIDX(j, m)] = mk<double>(0, 0);
    zc ms = mk<double>(-rs[j].re, -rs[j].im);
    zrot(H[HIDX(j, m)], H[HIDX(j + 1, m)], rc[j], ms);
  }
}

__global__ void k_hinit(zc* H, int m, double beta) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > m) return;
  H[HIDX(i, m)] = (i == 0) ? mk<double>(beta, 0) : mk<double>(0, 0);
}
__global__ void k_hcol_zero(zc* H, int m, int jh) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= jh) H[HIDX(i, jh)] = mk<double>(0, 0);
}
__global__ void k_gs_reset(GmState* gs) {
  gs->dloo2 = 0;
}

static const int AR_MAXB = 1024;  // largest grid of the fused Arnoldi kernel

struct Gm {
  int n, m;
  zc *V, *w, *r0, *xc, *y, *H, *part_a, *part_b, *part2, *rs;
  double* rc;
  GmState* gs;
  GmState* hgs;  // pinned host copies of gs, one slot per Arnoldi step parity
  int ar_blocks; // grid of the fused Arnoldi kernel
  ArSlot* slots; // exchange slots of the register-resident Arnoldi kernel (2 x AR_MAXB)
  int reg_ept, reg_blocks;  // its elements per thread and grid (0: not usable)
  int cl_ept, cl_size;      // single-cluster Arnoldi kernel (0: not usable)
};

template <typename VT, int EPT>
static int cl_setup(int cs, cudaStream_t s, bool& ok) {
  ok = false;
  if (cs > 8)
    SIE_CUDA(cudaFuncSetAttribute(k_arnoldi_cl<VT, EPT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(cs);
  lc.blockDim = dim3(CL_THREADS);
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  int nclus = 0;
  if (cudaOccupancyMaxActiveClusters(&nclus, k_arnoldi_cl<VT, EPT>, &lc) != cudaSuccess) {
    cudaGetLastError();
    return SIE_OK;
  }
  ok = nclus >= 1;
  return SIE_OK;
}

template <typename VT, int EPT>
static int cl_launch(int cs, cudaStream_t s, cx<VT>* w, cx<VT>* V, size_t ld, int n, int jH, zc* H, int m,
                     double* rc, zc* rs, GmState* gs, double bn) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(cs);
  lc.blockDim = dim3(CL_THREADS);
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  SIE_CUDA(cudaLaunchKernelEx(&lc, k_arnoldi_cl<VT, EPT>, w, V, ld, n, jH, H, m, rc, rs, gs, bn));
  return SIE_OK;
}

static int gm_alloc(sie_ctx* c, int m, Gm& g) {
  int n = 2 * c->M;
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t o = need;
    need += (bytes + 255) & ~(size_t)255;
    return o;
  };
  size_t oV = add((size_t)(m + 1) * n * sizeof(zc));
  size_t ow = add((size_t)n * sizeof(zc));
  size_t or0 = add((size_t)n * sizeof(zc));
  size_t oxc = add((size_t)n * sizeof(zc));
  size_t oy = add((size_t)(m + 1) * sizeof(zc));
  size_t oH = add((size_t)(m + 1) * (m + 1) * sizeof(zc));
  size_t opa = add(RB * sizeof(zc));
  size_t opb = add(RB * sizeof(zc));
  size_t ors = add((size_t)(m + 1) * sizeof(zc));
  size_t orc = add((size_t)(m + 1) * sizeof(double));
  size_t ogs = add(sizeof(GmState));
  size_t op2 = add((size_t)2 * AR_MAXB * sizeof(zc));
  size_t osl = add((size_t)2 * AR_MAXB * sizeof(ArSlot));
  if (c->gm_bytes < need) {
    if (c->d_gm) cudaFree(c->d_gm);
    c->d_gm = nullptr;
    c->gm_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_gm, need));
    SIE_CUDA(cudaMemset(c->d_gm, 0, need));
    c->gm_bytes = need;
  }
  if (!c->h_gm) SIE_CUDA(cudaHostAlloc(&c->h_gm, 2 * sizeof(GmState), cudaHostAllocDefault));
  if (c->ar_blocks == 0) {
    int per_sm = 0, nsm = 0;
    SIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arnoldi<double>, 512, 0));
    SIE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    c->ar_blocks = std::max(1, std::min(AR_MAXB, std::min(per_sm, 2) * nsm));
  }
  char* b = (char*)c->d_gm;
  g.n = n;
  g.m = m;
  g.V = (zc*)(b + oV);
  g.w = (zc*)(b + ow);
  g.r0 = (zc*)(b + or0);
  g.xc = (zc*)(b + oxc);
  g.y = (zc*)(b + oy);
  g.H = (zc*)(b + oH);
  g.part_a = (zc*)(b + opa);
  g.part_b = (zc*)(b + opb);
  g.rs = (zc*)(b + ors);
  g.rc = (double*)(b + orc);
  g.gs = (GmState*)(b + ogs);
  g.part2 = (zc*)(b + op2);
  g.slots = (ArSlot*)(b + osl);
  // register-resident Arnoldi kernel: the fewest elements per thread that keep the grid
  // at <= 32 blocks, else 8 per thread on up to one block per SM
  g.cl_ept = g.cl_size = 0;
  {
    const int epts[4] = {1, 2, 4, 8};
    for (int k = 0; k < 4 && !g.cl_ept; k++) {
      int cs = (n + CL_THREADS * epts[k] - 1) / (CL_THREADS * epts[k]);
      if (cs > 16) continue;
      bool ok = false;
      int r = epts[k] == 1 ? cl_setup<double, 1>(cs, c->stream, ok)
              : epts[k] == 2 ? cl_setup<double, 2>(cs, c->stream, ok)
              : epts[k] == 4 ? cl_setup<double, 4>(cs, c->stream, ok)
                             : cl_setup<double, 8>(cs, c->stream, ok);
      if (r != SIE_OK) return r;
      if (ok) {
        g.cl_ept = epts[k];
        g.cl_size = cs;
      }
    }
  }
  g.reg_ept = g.reg_blocks = 0;
  if (m <= 1300) {
    int nsm = 0;
    SIE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int epts[4] = {1, 2, 4, 8};
    for (int k = 0; k < 4 && !g.reg_ept; k++) {
      int nbk = (n + AR_THREADS * epts[k] - 1) / (AR_THREADS * epts[k]);
      if (nbk <= 32 || (epts[k] == 8 && nbk <= nsm)) {
        g.reg_ept = epts[k];
        g.reg_blocks = nbk;
      }
    }
  }
  g.hgs = (GmState*)c->h_gm;
  g.ar_blocks = std::max(1, std::min(c->ar_blocks, (n + 511) / 512));
  return SIE_OK;
}

static int read_gs(sie_ctx* c, Gm& g, GmState& h) {
  SIE_CUDA(cudaMemcpyAsync(&h, g.gs, sizeof(GmState), cudaMemcpyDeviceToHost, c->stream));
  SIE_CUDA(cudaStreamSynchronize(c->stream));
  return SIE_OK;
}

static int norm2(sie_ctx* c, Gm& g, const zc* a, double& out) {
  k_dot<<<RB, RT_, 0, c->stream>>>(a, nullptr, g.n, g.part_a); sie::count_launch();
  k_norm_final<<<1, RT_, 0, c->stream>>>(g.part_a, RB, g.gs); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  GmState h;
  SIE_TRY(read_gs(c, g, h));
  out = h.nrm;
  return SIE_OK;
}

// Launch the fused Arnoldi step jH on the FP64 basis of g (kernel chosen by
// c->arnoldi_mode and the vector length).
static int arnoldi_launch64(sie_ctx* c, Gm& g, int jH, double bn, cudaStream_t s) {
  size_t ldv = (size_t)g.n;
  int nn = g.n, jj = jH, mm = g.m;
  double bnv = bn;
  if (g.cl_ept && c->arnoldi_mode == 2) {
    int rr = g.cl_ept == 1 ? cl_launch<double, 1>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
             : g.cl_ept == 2 ? cl_launch<double, 2>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
             : g.cl_ept == 4 ? cl_launch<double, 4>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
                             : cl_launch<double, 8>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv);
    if (rr != SIE_OK) return rr;
  } else if (g.reg_ept && c->arnoldi_mode >= 1) {
    unsigned epoch = c->ar_epoch;
    c->ar_epoch = (c->ar_epoch + 1) & 0xFFFFFu;
    if (c->ar_epoch == 0) c->ar_epoch = 1;
    void* args[] = {&g.w, &g.V, &ldv, &nn, &jj, &g.H, &mm, &g.rc, &g.rs, &g.slots, &epoch, &g.gs, &bnv};
    const void* fn = g.reg_ept == 1 ? (const void*)k_arnoldi_reg<1>
                     : g.reg_ept == 2 ? (const void*)k_arnoldi_reg<2>
                     : g.reg_ept == 4 ? (const void*)k_arnoldi_reg<4>
                                      : (const void*)k_arnoldi_reg<8>;
    SIE_CUDA(cudaLaunchCooperativeKernel(fn, dim3(g.reg_blocks), dim3(AR_THREADS), args, 0, s));
  } else {
    void* args[] = {&g.w, &g.V, &ldv, &nn, &jj, &g.H, &mm, &g.rc, &g.rs, &g.part2, &g.gs, &bnv};
    SIE_CUDA(cudaLaunchCooperativeKernel((const void*)k_arnoldi<double>, dim3(g.ar_blocks), dim3(512), args, 0, s));
  }
  sie::count_launch();
  return SIE_OK;
}

}  // namespace sie

using namespace sie;


int sie::gmres_solve(sie_ctx* c, const zc* d_b_ext, zc* d_x_ext, const sie_solver_cfg* cfg,
                     sie_stats* st) {
  if (cfg->precision == SIE_MIXED) return fgmres_mixed(c, d_b_ext, d_x_ext, cfg, st);
  cudaStream_t s = c->stream;
  int m = cfg->restart;
  Gm g;
  {
    int r = gm_alloc(c, m, g);
    if (r != SIE_OK) return r;
  }
  int n = g.n;
  size_t ld = (size_t)n;
  auto t0 = std::chrono::steady_clock::now();
  c->tm.gm_passes = c->tm.gm_steps = 0;
  // grid barrier state (bar_count, bar_gen, bar_err) starts clean for every solve
  SIE_CUDA(cudaMemsetAsync(&g.gs->bar_count, 0, 2 * sizeof(unsigned) + sizeof(int), s));
  {
    const int lim = grid_spin_limit_host();
    SIE_CUDA(cudaMemcpyAsync(&g.gs->spin_limit, &lim, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  cudaEventRecord(c->ev[12], s);
  // internal layout: b -> d_yi (kept), x -> d_xi
  zc* b = c->d_yi;
  zc* x = c->d_xi;
  int r = gather_ext_to_int(c, d_b_ext, b, 1, s);
  if (r != SIE_OK) return r;
  if (cfg->use_initial_guess) {
    r = gather_ext_to_int(c, d_x_ext, x, 1, s);
  } else {
    k_zero<<<RB, RT_, 0, s>>>(x, n); sie::count_launch();
  }
  if (r != SIE_OK) return r;
  int matvecs = 0;
  auto matvec = [&](const zc* in, zc* out) -> int {
    matvecs++;
    return sie_internal_matvec(c, in, out, 1, s, false);
  };
  // With the near-field preconditioner the Arnoldi process runs on Z P (right
  // preconditioning): its residual is the true one, and the iterate is x + P V y.
  const bool pre = c->precond == SIE_PRECOND_NEAR;
  auto op = [&](const zc* in, zc* out) -> int {
    if (!pre) return matvec(in, out);
    SIE_TRY(ras_apply64(c, in, g.r0, s));
    return matvec(g.r0, out);
  };
  // out = x + (P) V(:, 0:k) y; uses g.r0 and g.w as scratch when preconditioned
  auto update = [&](int k, zc* out) -> int {
    if (!pre) {
      k_combine<<<RB, RT_, 0, s>>>(x, g.V, g.y, k, n, ld, out); sie::count_launch();
      return SIE_OK;
    }
    k_combine<<<RB, RT_, 0, s>>>(nullptr, g.V, g.y, k, n, ld, g.r0); sie::count_launch();
    SIE_TRY(ras_apply64(c, g.r0, g.w, s));
    k_add<<<RB, RT_, 0, s>>>(x, g.w, out, n); sie::count_launch();
    return SIE_OK;
  };
  auto finish = [&](int code, int iters, double bea, double be, int conv) {
    scatter_int_to_ext(c, x, d_x_ext, 1, s);
    cudaEventRecord(c->ev[13], s);
    cudaEventSynchronize(c->ev[13]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[12], c->ev[13]);
    if (st) {
      st->iterations = iters;
      st->matvecs = matvecs;
      st->converged = conv;
      st->backward_error_arnoldi = bea;
      st->backward_error_true = be;
      st->seconds = ms * 1e-3;
    }
    return code;
  };
  double bn = 0;
  r = norm2(c, g, b, bn);
  if (r != SIE_OK) return r;
  if (!std::isfinite(bn)) return fail(SIE_ERR_NONFINITE, "GMRES: non-finite right-hand side");
  if (bn == 0.0) {
    k_zero<<<RB, RT_, 0, s>>>(x, n); sie::count_launch();
    return finish(SIE_OK, 0, 0, 0, 1);
  }
  // r0 = b - A x  (or b)
  if (cfg->use_initial_guess) {
    SIE_TRY(matvec(x, g.r0));
    k_sub<<<RB, RT_, 0, s>>>(b, g.r0, g.w, n); sie::count_launch();
  } else {
    k_copy<<<RB, RT_, 0, s>>>(b, g.w, n); sie::count_launch();
  }
  double beta = 0;
  r = norm2(c, g, g.w, beta);
  if (r != SIE_OK) return r;
  if (beta == 0.0) return finish(SIE_OK, 0, 0, 0, 1);
  k_scale_copy_s<<<RB, RT_, 0, s>>>(g.w, g.V, n, beta); sie::count_launch();
  int iterOut = 0, compRsd = 0;
  double bea = 1e300, be = 1e300, trueNormRes = 0;
  int itermax = cfg->max_iterations;
  // The scalars of Arnoldi step jH are copied to pinned slot jH & 1 and marked by
  // event ev[14 + (jH & 1)].  The host enqueues step jH + 1 before it reads step jH,
  // so the GPU never waits for the host.  A step enqueued after the one that ends the
  // solve only touches w, V(:, jH+2), H(:, jH+1) and rows jH+1.. of the right-hand
  // column, none of which the final update reads.
  auto post = [&](int jH) -> int {
    SIE_CUDA(cudaMemcpyAsync(&g.hgs[jH & 1], g.gs, sizeof(GmState), cudaMemcpyDeviceToHost, s));
    SIE_CUDA(cudaEventRecord(c->ev[14 + (jH & 1)], s));
    return SIE_OK;
  };
  auto arnoldi = [&](int jH) -> int { return arnoldi_launch64(c, g, jH, bn, s); };
  // Decide step p once its scalars are on the host: 1 = the solve ends (x final),
  // 0 = go on; negative = error code.
  int end_code = SIE_OK;
  auto decide = [&](int p) -> int {
    SIE_CUDA(cudaEventSynchronize(c->ev[14 + (p & 1)]));
    GmState h = g.hgs[p & 1];
    c->tm.gm_passes += h.passes;
    c->tm.gm_steps += 1;
    if (h.bar_err) return -fail(SIE_ERR_CUDA, "GMRES: a grid barrier of the Arnoldi step timed out");
    if (!std::isfinite(h.dnormw)) return -fail(SIE_ERR_NONFINITE, "GMRES: non-finite Arnoldi vector");
    bea = h.bea;
    if (!std::isfinite(bea)) return -fail(SIE_ERR_NONFINITE, "GMRES: non-finite residual estimate");
    int it = iterOut * m + p + 1;
    if (bea <= cfg->tolerance || it >= itermax) {
      compRsd = 1;
      // xCurrent = x + V y
      k_trsv<<<1, 1, 0, s>>>(g.H, m, p + 1, g.y); sie::count_launch();
      {
        int ru = update(p + 1, g.xc);
        if (ru != SIE_OK) return -ru;
      }
      // true residual
      int rr = matvec(g.xc, g.w);
      if (rr != SIE_OK) return -rr;
      k_sub<<<RB, RT_, 0, s>>>(b, g.w, g.w, n); sie::count_launch();
      rr = norm2(c, g, g.w, trueNormRes);
      if (rr != SIE_OK) return -rr;
      be = trueNormRes / bn;
      if (be <= cfg->tolerance || it >= itermax) {
        k_copy<<<RB, RT_, 0, s>>>(g.xc, x, n); sie::count_launch();
        int conv = be <= cfg->tolerance;
        end_code = finish(conv ? SIE_OK : fail(SIE_ERR_NOCONV, "GMRES: no convergence"), it, bea,
                          trueNormRes / bn, conv);
        return 1;
      }
    }
    return 0;
  };
  while (true) {
    k_hinit<<<(m + 1 + 127) / 128, 128, 0, s>>>(g.H, m, beta); sie::count_launch();
    int pending = -1;
    for (int jH = 0; jH < m; jH++) {
      // w = A V_jH, then the fused orthogonalisation / Givens step
      SIE_TRY(op(g.V + (size_t)jH * ld, g.w));
      SIE_TRY(arnoldi(jH));
      SIE_TRY(post(jH));
      SIE_CUDA(cudaGetLastError());
      if (pending >= 0) {
        int d = decide(pending);
        if (d < 0) return -d;
        if (d == 1) return end_code;
      }
      pending = jH;
      if (iterOut * m + jH + 1 >= itermax) break;  // the budget ends with this step
      if (cfg->time_limit_s > 0) {
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > cfg->time_limit_s) {
          int d = decide(pending);
          if (d < 0) return -d;
          if (d == 1) return end_code;
          finish(SIE_ERR_TIMEOUT, iterOut * m + jH + 1, bea, be, 0);
          return fail(SIE_ERR_TIMEOUT, "GMRES: time limit reached");
        }
      }
    }
    {
      int d = decide(pending);
      if (d < 0) return -d;
      if (d == 1) return end_code;
    }
    iterOut++;
    if (bea > cfg->tolerance) {
      k_trsv<<<1, 1, 0, s>>>(g.H, m, m, g.y); sie::count_launch();
      SIE_TRY(update(m, g.xc));
    }
    k_copy<<<RB, RT_, 0, s>>>(g.xc, x, n); sie::count_launch();
    if (compRsd == 1) {
      SIE_TRY(matvec(x, g.r0));
      k_sub<<<RB, RT_, 0, s>>>(b, g.r0, g.w, n); sie::count_launch();
      r = norm2(c, g, g.w, beta);
      if (r != SIE_OK) return r;
    } else {
      k_restart_rhs<<<1, 1, 0, s>>>(g.H, m, g.rc, g.rs, g.gs); sie::count_launch();
      // w = V(:, 0:m+1) H(:, m)
      k_combine<<<RB, RT_, 0, s>>>(nullptr, g.V, g.H + (size_t)m * (m + 1), m + 1, n, ld, g.w); sie::count_launch();
      GmState h;
      SIE_TRY(read_gs(c, g, h));
      beta = h.nrm;
    }
    k_scale_copy_s<<<RB, RT_, 0, s>>>(g.w, g.V, n, beta); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
}

// ---------------------------------------------------------------------------
// Mixed precision (SIE_MIXED): flexible GMRES in FP64 whose preconditioner is one cycle
// of GMRES in FP32 on the complex64 operator.  The outer Arnoldi basis, the Hessenberg
// matrix, the true residual and the solution stay FP64; the inner Krylov vectors are
// complex64 (dot products accumulated in FP64).  The inner operator is within ~1e-3 of
// the FP64 one on 0.6-lambda leaf boxes (the K = 19 translations cancel heavily), which
// is what a preconditioner needs; the outer FP64 products remove that error.

namespace sie {

template <typename VT>
__global__ void __launch_bounds__(RT_) k_norm2_t(const cx<VT>* a, int n, zc* part_out) {
  zc acc = mk<double>(0, 0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc.re += cabs2(cvt_z(a[i]));
  acc = block_sum(acc);
  if (threadIdx.x == 0) part_out[blockIdx.x] = acc;
}
template <typename VT>
__global__ void k_scale_t(const cx<VT>* a, cx<VT>* b, int n, double s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = narrow<VT>(cvt_z(a[i]) * s);
}
// y = V(:, 0:k) coef
template <typename VT>
__global__ void k_combine_t(const cx<VT>* V, size_t ld, const zc* coef, int k, int n, cx<VT>* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    zc s = mk<double>(0, 0);
    for (int j = 0; j < k; j++) s = cfma(cvt_z(V[(size_t)j * ld + i]), coef[j], s);
    y[i] = narrow<VT>(s);
  }
}

struct Gm32 {
  int n, m;
  cc *V, *w;
  zc *H, *y, *rs, *part, *part2;
  double* rc;
  GmState* gs;
  int cl_ept, cl_size, ar_blocks;
};

static int gm32_alloc(sie_ctx* c, int m, Gm32& g) {
  int n = 2 * c->M;
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t o = need;
    need += (bytes + 255) & ~(size_t)255;
    return o;
  };
  size_t oV = add((size_t)(m + 1) * n * sizeof(cc)), ow = add((size_t)n * sizeof(cc));
  size_t oH = add((size_t)(m + 1) * (m + 1) * sizeof(zc)), oy = add((size_t)(m + 1) * sizeof(zc));
  size_t ors = add((size_t)(m + 1) * sizeof(zc)), orc = add((size_t)(m + 1) * sizeof(double));
  size_t op = add(RB * sizeof(zc)), op2 = add((size_t)2 * AR_MAXB * sizeof(zc));
  size_t ogs = add(sizeof(GmState));
  if (c->gm32_bytes < need) {
    if (c->d_gm32) cudaFree(c->d_gm32);
    c->d_gm32 = nullptr;
    c->gm32_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_gm32, need));
    SIE_CUDA(cudaMemset(c->d_gm32, 0, need));
    c->gm32_bytes = need;
  }
  char* b = (char*)c->d_gm32;
  g.n = n;
  g.m = m;
  g.V = (cc*)(b + oV);
  g.w = (cc*)(b + ow);
  g.H = (zc*)(b + oH);
  g.y = (zc*)(b + oy);
  g.rs = (zc*)(b + ors);
  g.rc = (double*)(b + orc);
  g.part = (zc*)(b + op);
  g.part2 = (zc*)(b + op2);
  g.gs = (GmState*)(b + ogs);
  g.cl_ept = g.cl_size = 0;
  const int epts[4] = {1, 2, 4, 8};
  for (int k = 0; k < 4 && !g.cl_ept; k++) {
    int cs = (n + CL_THREADS * epts[k] - 1) / (CL_THREADS * epts[k]);
    if (cs > 16) continue;
    bool ok = false;
    int r = epts[k] == 1 ? cl_setup<float, 1>(cs, c->stream, ok)
            : epts[k] == 2 ? cl_setup<float, 2>(cs, c->stream, ok)
            : epts[k] == 4 ? cl_setup<float, 4>(cs, c->stream, ok)
                           : cl_setup<float, 8>(cs, c->stream, ok);
    if (r != SIE_OK) return r;
    if (ok) {
      g.cl_ept = epts[k];
      g.cl_size = cs;
    }
  }
  int per_sm = 0, nsm = 0;
  SIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arnoldi<float>, 512, 0));
  SIE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  g.ar_blocks = std::max(1, std::min(std::min(AR_MAXB, std::min(per_sm, 2) * nsm), (n + 511) / 512));
  return SIE_OK;
}

static int arnoldi_launch32(Gm32& g, int jH, double bn, cudaStream_t s) {
  size_t ldv = (size_t)g.n;
  int nn = g.n, jj = jH, mm = g.m;
  double bnv = bn;
  if (g.cl_ept) {
    int rr = g.cl_ept == 1 ? cl_launch<float, 1>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
             : g.cl_ept == 2 ? cl_launch<float, 2>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
             : g.cl_ept == 4 ? cl_launch<float, 4>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv)
                             : cl_launch<float, 8>(g.cl_size, s, g.w, g.V, ldv, nn, jj, g.H, mm, g.rc, g.rs, g.gs, bnv);
    if (rr != SIE_OK) return rr;
  } else {
    void* args[] = {&g.w, &g.V, &ldv, &nn, &jj, &g.H, &mm, &g.rc, &g.rs, &g.part2, &g.gs, &bnv};
    SIE_CUDA(cudaLaunchCooperativeKernel((const void*)k_arnoldi<float>, dim3(g.ar_blocks), dim3(512), args, 0, s));
  }
  sie::count_launch();
  return SIE_OK;
}

// One cycle of FP32 GMRES from z = 0 on A32 z = r (complex64, internal layout): at most
// g.m steps, stopping once the Arnoldi residual estimate |H(j+1, m)| / ||r|| <= tol.
static int inner_gmres32(sie_ctx* c, Gm32& g, const cc* r, cc* z, double tol, int& its, int& mvs) {
  cudaStream_t s = c->stream;
  int n = g.n, m = g.m;
  size_t ld = (size_t)n;
  its = 0;
  k_norm2_t<float><<<RB, RT_, 0, s>>>(r, n, g.part); sie::count_launch();
  k_norm_final<<<1, RT_, 0, s>>>(g.part, RB, g.gs); sie::count_launch();
  SIE_CUDA(cudaMemsetAsync(&g.gs->bar_count, 0, 2 * sizeof(unsigned) + sizeof(int), s));
  {
    const int lim = grid_spin_limit_host();
    SIE_CUDA(cudaMemcpyAsync(&g.gs->spin_limit, &lim, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  GmState h;
  SIE_CUDA(cudaMemcpyAsync(&h, g.gs, sizeof(GmState), cudaMemcpyDeviceToHost, s));
  SIE_CUDA(cudaStreamSynchronize(s));
  double beta = h.nrm;
  if (!(beta > 0) || !std::isfinite(beta)) {
    SIE_CUDA(cudaMemsetAsync(z, 0, (size_t)n * sizeof(cc), s));
    return std::isfinite(beta) ? SIE_OK : fail(SIE_ERR_NONFINITE, "inner GMRES: non-finite vector");
  }
  k_scale_t<float><<<RB, RT_, 0, s>>>(r, g.V, n, 1.0 / beta); sie::count_launch();
  k_hinit<<<(m + 1 + 127) / 128, 128, 0, s>>>(g.H, m, beta); sie::count_launch();
  // As in the FP64 solver, the scalars of step j go to pinned slot j & 1 and are read
  // one step late, so the GPU never waits for the host; a step queued after the one
  // that meets the tolerance is not used by the update below.
  GmState* slots = (GmState*)c->h_gm;
  int k = 0;
  auto check = [&](int p, bool& stop) -> int {
    SIE_CUDA(cudaEventSynchronize(c->ev[14 + (p & 1)]));
    const GmState hp = slots[p & 1];
    if (hp.bar_err) return fail(SIE_ERR_CUDA, "inner GMRES: a grid barrier timed out");
    if (!std::isfinite(hp.dnormw) || !std::isfinite(hp.bea))
      return fail(SIE_ERR_NONFINITE, "inner GMRES: non-finite Arnoldi vector");
    k = p + 1;
    stop = hp.bea <= tol || hp.dnormw == 0.0;
    return SIE_OK;
  };
  bool stop = false;
  // with the near-field preconditioner the inner cycle runs on Z P and returns P (V y);
  // r is no longer read once V(:, 0) holds it, so c->d_xi32 is the scratch vector
  const bool pre = c->precond == SIE_PRECOND_NEAR;
  cc* tmp = c->d_xi32;
  for (int j = 0; j < m && !stop; j++) {
    const cc* vj = g.V + (size_t)j * ld;
    if (pre) {
      SIE_TRY(ras_apply32(c, vj, tmp, s));
      vj = tmp;
    }
    SIE_TRY(sie_internal_matvec32(c->inner ? c->inner : c, vj, g.w, s, false));
    mvs++;
    SIE_TRY(arnoldi_launch32(g, j, beta, s));
    SIE_CUDA(cudaMemcpyAsync(&slots[j & 1], g.gs, sizeof(GmState), cudaMemcpyDeviceToHost, s));
    SIE_CUDA(cudaEventRecord(c->ev[14 + (j & 1)], s));
    if (j > 0) SIE_TRY(check(j - 1, stop));
    if (!stop && j == m - 1) SIE_TRY(check(j, stop));
  }
  k_trsv<<<1, 1, 0, s>>>(g.H, m, k, g.y); sie::count_launch();
  if (pre) {
    k_combine_t<float><<<RB, RT_, 0, s>>>(g.V, ld, g.y, k, n, tmp); sie::count_launch();
    SIE_TRY(ras_apply32(c, tmp, z, s));
  } else {
    k_combine_t<float><<<RB, RT_, 0, s>>>(g.V, ld, g.y, k, n, z); sie::count_launch();
  }
  SIE_CUDA(cudaGetLastError());
  its = k;
  return SIE_OK;
}

int fgmres_mixed(sie_ctx* c, const zc* d_b_ext, zc* d_x_ext, const sie_solver_cfg* cfg, sie_stats* st) {
  cudaStream_t s = c->stream;
  if (cfg->inner_restart < 1 || !(cfg->inner_tolerance > 0))
    return fail(SIE_ERR_ARG, "mixed solve: bad inner solver settings");
  SIE_TRY(make_f32_tables(c));
  if (c->inner) SIE_TRY(make_f32_tables(c->inner));
  SIE_TRY(ras_to_f32(c));
  int m = cfg->restart;
  Gm g;
  SIE_TRY(gm_alloc(c, m, g));
  Gm32 gi;
  SIE_TRY(gm32_alloc(c, cfg->inner_restart, gi));
  int n = g.n;
  size_t ld = (size_t)n;
  size_t zbytes = (size_t)m * n * sizeof(zc);
  if (c->gmz_bytes < zbytes) {
    if (c->d_gmz) cudaFree(c->d_gmz);
    c->d_gmz = nullptr;
    c->gmz_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_gmz, zbytes));
    c->gmz_bytes = zbytes;
  }
  zc* Z = (zc*)c->d_gmz;
  c->tm.gm_passes = c->tm.gm_steps = 0;
  SIE_CUDA(cudaMemsetAsync(&g.gs->bar_count, 0, 2 * sizeof(unsigned) + sizeof(int), s));
  {
    const int lim = grid_spin_limit_host();
    SIE_CUDA(cudaMemcpyAsync(&g.gs->spin_limit, &lim, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  cudaEventRecord(c->ev[12], s);
  zc* b = c->d_yi;
  zc* x = c->d_xi;
  SIE_TRY(gather_ext_to_int(c, d_b_ext, b, 1, s));
  if (cfg->use_initial_guess) {
    SIE_TRY(gather_ext_to_int(c, d_x_ext, x, 1, s));
  } else {
    k_zero<<<RB, RT_, 0, s>>>(x, n); sie::count_launch();
  }
  int mv64 = 0, mv32 = 0, inner_total = 0, it = 0;
  auto finish = [&](int code, double bea, double be, int conv) {
    scatter_int_to_ext(c, x, d_x_ext, 1, s);
    cudaEventRecord(c->ev[13], s);
    cudaEventSynchronize(c->ev[13]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[12], c->ev[13]);
    if (st) {
      st->iterations = it;
      st->inner_iterations = inner_total;
      st->matvecs = mv64 + mv32;
      st->converged = conv;
      st->backward_error_arnoldi = bea;
      st->backward_error_true = be;
      st->seconds = ms * 1e-3;
    }
    return code;
  };
  double bn = 0;
  SIE_TRY(norm2(c, g, b, bn));
  if (!std::isfinite(bn)) return fail(SIE_ERR_NONFINITE, "mixed solve: non-finite right-hand side");
  if (bn == 0.0) {
    k_zero<<<RB, RT_, 0, s>>>(x, n); sie::count_launch();
    return finish(SIE_OK, 0, 0, 1);
  }
  double bea = 1e300, be = 1e300;
  while (true) {
    // r0 = b - A x (FP64), beta = ||r0||
    if (it == 0 && !cfg->use_initial_guess) {
      k_copy<<<RB, RT_, 0, s>>>(b, g.w, n); sie::count_launch();
    } else {
      SIE_TRY(sie_internal_matvec(c, x, g.r0, 1, s, false));
      mv64++;
      k_sub<<<RB, RT_, 0, s>>>(b, g.r0, g.w, n); sie::count_launch();
    }
    double beta = 0;
    SIE_TRY(norm2(c, g, g.w, beta));
    be = beta / bn;
    if (be <= cfg->tolerance) return finish(SIE_OK, bea, be, 1);
    if (it >= cfg->max_iterations)
      return finish(fail(SIE_ERR_NOCONV, "mixed solve: no convergence"), bea, be, 0);
    k_scale_copy_s<<<RB, RT_, 0, s>>>(g.w, g.V, n, beta); sie::count_launch();
    k_hinit<<<(m + 1 + 127) / 128, 128, 0, s>>>(g.H, m, beta); sie::count_launch();
    int k = 0;
    for (int j = 0; j < m; j++) {
      // z_j = inner solve of A z = V_j (complex64), kept in FP64 in Z
      SIE_TRY(to_c64(g.V + (size_t)j * ld, c->d_xi32, n, s));
      int its = 0;
      SIE_TRY(inner_gmres32(c, gi, c->d_xi32, c->d_yi32, cfg->inner_tolerance, its, mv32));
      inner_total += its;
      SIE_TRY(to_c128(c->d_yi32, Z + (size_t)j * ld, n, s));
      // w = A z_j (FP64) and the FP64 Arnoldi step
      SIE_TRY(sie_internal_matvec(c, Z + (size_t)j * ld, g.w, 1, s, false));
      mv64++;
      SIE_TRY(arnoldi_launch64(c, g, j, bn, s));
      GmState h;
      SIE_TRY(read_gs(c, g, h));
      c->tm.gm_passes += h.passes;
      c->tm.gm_steps += 1;
      if (h.bar_err) return fail(SIE_ERR_CUDA, "mixed solve: a grid barrier timed out");
      if (!std::isfinite(h.dnormw) || !std::isfinite(h.bea))
        return fail(SIE_ERR_NONFINITE, "mixed solve: non-finite Arnoldi vector");
      bea = h.bea;
      it++;
      k = j + 1;
      if (bea <= cfg->tolerance || it >= cfg->max_iterations || h.dnormw == 0.0) break;
      if (cfg->time_limit_s > 0) {
        float el = 0;
        cudaEventRecord(c->ev[13], s);
        cudaEventSynchronize(c->ev[13]);
        cudaEventElapsedTime(&el, c->ev[12], c->ev[13]);
        if (el * 1e-3 > cfg->time_limit_s) {
          finish(SIE_ERR_TIMEOUT, bea, be, 0);
          return fail(SIE_ERR_TIMEOUT, "mixed solve: time limit reached");
        }
      }
    }
    // x += Z(:, 0:k) y
    k_trsv<<<1, 1, 0, s>>>(g.H, m, k, g.y); sie::count_launch();
    k_combine<<<RB, RT_, 0, s>>>(x, Z, g.y, k, n, ld, g.xc); sie::count_launch();
    k_copy<<<RB, RT_, 0, s>>>(g.xc, x, n); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
    // the loop head recomputes the true residual in FP64 and decides
  }
}


// ---------------------------------------------------------------------------
// Batched mixed-precision solve: R systems Z x_r = b_r of one matrix advance in lockstep,
// so each product is one batched matvec that reads the near panels, radiation patterns
// and translation tables once for all R vectors.  Outer FP64 flexible GMRES and inner
// complex64 GMRES as in fgmres_mixed.  Each new Krylov vector of the batch is
// orthogonalised by classical Gram-Schmidt applied twice (CGS2): one reduction per pass
// for all basis columns at once, where modified Gram-Schmidt needs one per column.  The
// inner cycle runs its fixed number of steps with no host synchronisation; a system that
// meets the inner tolerance earlier keeps the solution of that step.  Per-system
// scalars live on the device; the host reads them once per outer step.

static const int BNB = 64;     // blocks per system in the batched vector kernels
static const int BJG = 8;      // basis columns per reduction sweep
static const int BJMAX = 64;   // largest basis (restart + 1) of the batched solver

struct BState {
  double beta;    // norm of the cycle's starting vector
  double bn;      // norm the Arnoldi residual estimate is relative to
  double bea;     // that estimate at the last step the system took
  double dnormw;
  int k;          // steps of the cycle that the update uses
  int done;       // met its tolerance, broke down, or was frozen at the cycle start
  int pad[2];
};

// Block sums of BJG complex values (256 threads); the results land in out[0 .. BJG-1].
__device__ void block_sum_g(zc* v, zc* sh, zc* out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < BJG; j++) v[j] = warp_sum(v[j]);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < BJG; j++) sh[w * BJG + j] = v[j];
  __syncthreads();
  if (threadIdx.x < BJG) {
    zc s = mk<double>(0, 0);
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sh[k * BJG + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Partial dots <V_j, w> (j < ncol) over this block's elements of one system.
template <typename VT>
__device__ void bdots_chunk(const cx<VT>* Vr, size_t ldj, const cx<VT>* wr, int n, int ncol, zc* pr) {
  __shared__ zc sh[8 * BJG], res[BJG];
  for (int j0 = 0; j0 < ncol; j0 += BJG) {
    zc acc[BJG];
#pragma unroll
    for (int jj = 0; jj < BJG; jj++) acc[jj] = mk<double>(0, 0);
    for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) {
      const zc wi = cvt_z(wr[i]);
#pragma unroll
      for (int jj = 0; jj < BJG; jj++)
        if (j0 + jj < ncol) acc[jj] = cfma_conj(cvt_z(Vr[(size_t)(j0 + jj) * ldj + i]), wi, acc[jj]);
    }
    block_sum_g(acc, sh, res);
    if (threadIdx.x < BJG && j0 + (int)threadIdx.x < ncol) pr[j0 + threadIdx.x] = res[threadIdx.x];
  }
}

template <typename VT>
__global__ void __launch_bounds__(RT_) k_bdots(const cx<VT>* __restrict__ V, size_t ldj,
                                               const cx<VT>* __restrict__ w, int n, int ncol, zc* part,
                                               int ldp) {
  const int r = blockIdx.y;
  bdots_chunk<VT>(V + (size_t)r * n, ldj, w + (size_t)r * n, n, ncol,
                  part + ((size_t)r * BNB + blockIdx.x) * ldp);
}

// One CGS pass: h = the sum of the partial dots in a fixed order (every block of the
// system forms the same h), H(:, hcol) = h (add = 0) or += h, w -= V h; then the partial
// dots of the new w (next = 0) or its partial squared norm (next = 1).
template <typename VT>
__global__ void __launch_bounds__(RT_) k_bupdate(const cx<VT>* __restrict__ V, size_t ldj, cx<VT>* w, int n,
                                                 int ncol, const zc* part_in, zc* part_out, int ldp, zc* H,
                                                 int m, int hcol, int add, int next) {
  __shared__ zc h[BJMAX];
  const int r = blockIdx.y;
  for (int j = threadIdx.x; j < ncol; j += blockDim.x) {
    zc s = mk<double>(0, 0);
    const zc* p = part_in + (size_t)r * BNB * ldp + j;
    for (int b = 0; b < BNB; b++) s += p[(size_t)b * ldp];
    h[j] = s;
  }
  __syncthreads();
  if (blockIdx.x == 0) {
    zc* Hc = H + (size_t)r * (m + 1) * (m + 1) + (size_t)hcol * (m + 1);
    for (int j = threadIdx.x; j < ncol; j += blockDim.x) Hc[j] = add ? Hc[j] + h[j] : h[j];
  }
  cx<VT>* wr = w + (size_t)r * n;
  const cx<VT>* Vr = V + (size_t)r * n;
  double nrm = 0;
  for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) {
    zc wi = cvt_z(wr[i]);
    for (int j = 0; j < ncol; j++) wi = wi - h[j] * cvt_z(Vr[(size_t)j * ldj + i]);
    const cx<VT> wn = narrow<VT>(wi);
    wr[i] = wn;
    nrm += cabs2(cvt_z(wn));
  }
  zc* pr = part_out + ((size_t)r * BNB + blockIdx.x) * ldp;
  if (next) {
    const zc v = block_sum(mk<double>(nrm, 0));
    if (threadIdx.x == 0) pr[0] = v;
    return;
  }
  // each thread reads back only the elements it wrote above
  bdots_chunk<VT>(Vr, ldj, wr, n, ncol, pr);
}

// Partial squared norms of the R vectors a_r.
template <typename VT>
__global__ void __launch_bounds__(RT_) k_bnorm(const cx<VT>* a, int n, zc* part, int ldp) {
  const int r = blockIdx.y;
  const cx<VT>* ar = a + (size_t)r * n;
  double s = 0;
  for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) s += cabs2(cvt_z(ar[i]));
  const zc v = block_sum(mk<double>(s, 0));
  if (threadIdx.x == 0) part[((size_t)r * BNB + blockIdx.x) * ldp] = v;
}

// Start of a cycle: beta_r = ||src_r||, V_0 = src_r / beta_r, H(:, m) = beta_r e_1.
// set_bn: the Arnoldi estimate is relative to beta (inner solve); otherwise to the bn the
// state already holds.  frozen[r] != 0 marks a system that takes no step in this cycle.
template <typename VS, typename VT>
__global__ void __launch_bounds__(RT_) k_binit(const cx<VS>* src, int n, const zc* part, int ldp,
                                               cx<VT>* V0, zc* H, int m, BState* st, int set_bn,
                                               const int* frozen) {
  __shared__ double sb;
  const int r = blockIdx.y;
  if (threadIdx.x == 0) {
    double s = 0;
    for (int b = 0; b < BNB; b++) s += part[((size_t)r * BNB + b) * ldp].re;
    sb = sqrt(s);
  }
  __syncthreads();
  const double beta = sb;
  const double inv = beta > 0 ? 1.0 / beta : 0.0;
  const cx<VS>* sr = src + (size_t)r * n;
  cx<VT>* vr = V0 + (size_t)r * n;
  for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) vr[i] = narrow<VT>(cvt_z(sr[i]) * inv);
  if (blockIdx.x == 0) {
    zc* Hr = H + (size_t)r * (m + 1) * (m + 1);
    for (int i = threadIdx.x; i <= m; i += blockDim.x) Hr[HIDX(i, m)] = mk<double>(i == 0 ? beta : 0.0, 0.0);
    if (threadIdx.x == 0) {
      BState& S = st[r];
      S.beta = beta;
      if (set_bn) S.bn = beta;
      S.k = 0;
      S.dnormw = 0;
      S.bea = S.bn > 0 ? beta / S.bn : 0.0;
      S.done = (beta == 0.0) || (frozen && frozen[r]);
    }
  }
}

// End of a step: dnormw = ||w||, V_{jcol+1} = w / dnormw, the Givens update of column jcol
// and the residual estimate; a system stops counting steps once it meets tol.
template <typename VT>
__global__ void __launch_bounds__(RT_) k_bfinish(cx<VT>* V, size_t ldj, const cx<VT>* w, int n, int jcol,
                                                 const zc* part, int ldp, zc* H, int m, double* rc, zc* rs,
                                                 BState* st, double tol) {
  __shared__ double sdn;
  const int r = blockIdx.y;
  if (threadIdx.x == 0) {
    double s = 0;
    for (int b = 0; b < BNB; b++) s += part[((size_t)r * BNB + b) * ldp].re;
    sdn = sqrt(s);
  }
  __syncthreads();
  const double dn = sdn;
  const double inv = dn > 0 ? 1.0 / dn : 0.0;
  cx<VT>* vn = V + (size_t)(jcol + 1) * ldj + (size_t)r * n;
  const cx<VT>* wr = w + (size_t)r * n;
  for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) vn[i] = narrow<VT>(cvt_z(wr[i]) * inv);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    zc* Hr = H + (size_t)r * (m + 1) * (m + 1);
    double* rcr = rc + (size_t)r * (m + 1);
    zc* rsr = rs + (size_t)r * (m + 1);
    Hr[HIDX(jcol + 1, jcol)] = mk<double>(dn, 0.0);
    for (int j = 0; j < jcol; j++) zrot(Hr[HIDX(j, jcol)], Hr[HIDX(j + 1, jcol)], rcr[j], rsr[j]);
    double cr;
    zc sn;
    zrotg(Hr[HIDX(jcol, jcol)], Hr[HIDX(jcol + 1, jcol)], cr, sn);
    rcr[jcol] = cr;
    rsr[jcol] = sn;
    zrot(Hr[HIDX(jcol, m)], Hr[HIDX(jcol + 1, m)], cr, sn);
    zrot(Hr[HIDX(jcol, jcol)], Hr[HIDX(jcol + 1, jcol)], cr, sn);
    Hr[HIDX(jcol + 1, jcol)] = mk<double>(0, 0);
    BState& S = st[r];
    S.dnormw = dn;
    if (!S.done) {
      const double bea = S.bn > 0 ? sqrt(cabs2(Hr[HIDX(jcol + 1, m)])) / S.bn : 0.0;
      S.bea = bea;
      S.k = jcol + 1;
      if (bea <= tol || dn == 0.0 || !isfinite(bea)) S.done = 1;
    }
  }
}

// y_r = H_r(0:k, 0:k)^{-1} H_r(0:k, m) with k = the system's step count.
__global__ void k_btrsv(const zc* H, int m, const BState* st, zc* y) {
  if (threadIdx.x != 0) return;
  const int r = blockIdx.x;
  const zc* Hr = H + (size_t)r * (m + 1) * (m + 1);
  zc* yr = y + (size_t)r * (m + 1);
  const int k = st[r].k;
  for (int i = 0; i < k; i++) yr[i] = Hr[HIDX(i, m)];
  for (int i = k - 1; i >= 0; i--) {
    yr[i] = yr[i] / Hr[HIDX(i, i)];
    for (int j = 0; j < i; j++) yr[j] = yr[j] - yr[i] * Hr[HIDX(j, i)];
  }
}

// out_r (+)= sum_{j < k_r} y_r[j] V_j
template <typename VT, typename VO>
__global__ void __launch_bounds__(RT_) k_bcombine(const cx<VT>* __restrict__ V, size_t ldj, const zc* y, int ly,
                                                  const BState* st, int n, cx<VO>* out, int add) {
  const int r = blockIdx.y;
  const int k = st[r].k;
  const zc* yr = y + (size_t)r * ly;
  cx<VO>* orr = out + (size_t)r * n;
  for (int i = blockIdx.x * RT_ + threadIdx.x; i < n; i += BNB * RT_) {
    zc s = add ? cvt_z(orr[i]) : mk<double>(0, 0);
    for (int j = 0; j < k; j++) s = cfma(cvt_z(V[(size_t)j * ldj + (size_t)r * n + i]), yr[j], s);
    orr[i] = narrow<VO>(s);
  }
}

struct GmB {
  int n, R, mi, mo, ldp;
  size_t ldj;         // R * n: one basis column of the batch
  cc *V32, *w32, *r32, *z32;
  zc *Hi, *rsi, *yi, *W, *Zb, *w64, *x, *b, *r0, *Ho, *rso, *yo, *pA, *pB;
  double *rci, *rco;
  BState *sti, *sto;
  int* fin;
};

static int gmb_alloc(sie_ctx* c, int R, int mi, int mo, GmB& g) {
  const int n = 2 * c->M;
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t o = need;
    need += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t vr = (size_t)R * n;
  const int ldp = BJMAX;
  size_t oV32 = add((mi + 1) * vr * sizeof(cc)), ow32 = add(vr * sizeof(cc)), or32 = add(vr * sizeof(cc)),
         oz32 = add(vr * sizeof(cc));
  size_t oHi = add((size_t)R * (mi + 1) * (mi + 1) * sizeof(zc)), orsi = add((size_t)R * (mi + 1) * sizeof(zc)),
         oyi = add((size_t)R * (mi + 1) * sizeof(zc)), orci = add((size_t)R * (mi + 1) * sizeof(double));
  size_t oW = add((mo + 1) * vr * sizeof(zc)), oZ = add(mo * vr * sizeof(zc)), ow64 = add(vr * sizeof(zc)),
         ox = add(vr * sizeof(zc)), ob = add(vr * sizeof(zc)), or0 = add(vr * sizeof(zc));
  size_t oHo = add((size_t)R * (mo + 1) * (mo + 1) * sizeof(zc)), orso = add((size_t)R * (mo + 1) * sizeof(zc)),
         oyo = add((size_t)R * (mo + 1) * sizeof(zc)), orco = add((size_t)R * (mo + 1) * sizeof(double));
  size_t opA = add((size_t)R * BNB * ldp * sizeof(zc)), opB = add((size_t)R * BNB * ldp * sizeof(zc));
  size_t osti = add(R * sizeof(BState)), osto = add(R * sizeof(BState)), ofin = add(R * sizeof(int));
  if (c->gmb_bytes < need) {
    if (c->d_gmb) cudaFree(c->d_gmb);
    c->d_gmb = nullptr;
    c->gmb_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_gmb, need));
    c->gmb_bytes = need;
  }
  SIE_CUDA(cudaMemsetAsync(c->d_gmb, 0, need, c->stream));
  if (!c->h_gmb)
    SIE_CUDA(cudaHostAlloc(&c->h_gmb, SIE_BATCH_MAX * (sizeof(BState) + sizeof(int)), cudaHostAllocDefault));
  char* p = (char*)c->d_gmb;
  g.n = n;
  g.R = R;
  g.mi = mi;
  g.mo = mo;
  g.ldp = ldp;
  g.ldj = vr;
  g.V32 = (cc*)(p + oV32);
  g.w32 = (cc*)(p + ow32);
  g.r32 = (cc*)(p + or32);
  g.z32 = (cc*)(p + oz32);
  g.Hi = (zc*)(p + oHi);
  g.rsi = (zc*)(p + orsi);
  g.yi = (zc*)(p + oyi);
  g.rci = (double*)(p + orci);
  g.W = (zc*)(p + oW);
  g.Zb = (zc*)(p + oZ);
  g.w64 = (zc*)(p + ow64);
  g.x = (zc*)(p + ox);
  g.b = (zc*)(p + ob);
  g.r0 = (zc*)(p + or0);
  g.Ho = (zc*)(p + oHo);
  g.rso = (zc*)(p + orso);
  g.yo = (zc*)(p + oyo);
  g.rco = (double*)(p + orco);
  g.pA = (zc*)(p + opA);
  g.pB = (zc*)(p + opB);
  g.sti = (BState*)(p + osti);
  g.sto = (BState*)(p + osto);
  g.fin = (int*)(p + ofin);
  return SIE_OK;
}

// One Arnoldi step of the batch after the product w = A V_j: CGS2 against V_0..V_j, then
// the new basis column and the Givens update.
template <typename VT>
static int barnoldi(cx<VT>* V, size_t ldj, cx<VT>* w, int n, int R, int j, zc* pA, zc* pB, int ldp, zc* H,
                    int m, double* rc, zc* rs, BState* st, double tol, cudaStream_t s) {
  dim3 g(BNB, R);
  k_bdots<VT><<<g, RT_, 0, s>>>(V, ldj, w, n, j + 1, pA, ldp); sie::count_launch();
  k_bupdate<VT><<<g, RT_, 0, s>>>(V, ldj, w, n, j + 1, pA, pB, ldp, H, m, j, 0, 0); sie::count_launch();
  k_bupdate<VT><<<g, RT_, 0, s>>>(V, ldj, w, n, j + 1, pB, pA, ldp, H, m, j, 1, 1); sie::count_launch();
  k_bfinish<VT><<<g, RT_, 0, s>>>(V, ldj, w, n, j, pA, ldp, H, m, rc, rs, st, tol); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// One inner cycle for all R systems: z_r ~ A32^{-1} rhs_r (complex64, internal layout).
static int inner_batch32(sie_ctx* c, GmB& g, double tol) {
  cudaStream_t s = c->stream;
  const int n = g.n, R = g.R, mi = g.mi;
  dim3 grid(BNB, R);
  k_bnorm<float><<<grid, RT_, 0, s>>>(g.r32, n, g.pA, g.ldp); sie::count_launch();
  k_binit<float, float><<<grid, RT_, 0, s>>>(g.r32, n, g.pA, g.ldp, g.V32, g.Hi, mi, g.sti, 1, nullptr);
  sie::count_launch();
  // with the near-field preconditioner the cycle runs on Z P and returns P (V y); r32 is
  // no longer read once V(:, 0) holds it, so it is the scratch batch
  const bool pre = c->precond == SIE_PRECOND_NEAR;
  for (int j = 0; j < mi; j++) {
    const cc* vj = g.V32 + (size_t)j * g.ldj;
    if (pre) {
      SIE_TRY(ras_apply32(c, vj, g.r32, s, R));
      vj = g.r32;
    }
    SIE_TRY(sie_internal_matvec_b32(c->inner ? c->inner : c, vj, g.w32, R, s));
    SIE_TRY(barnoldi<float>(g.V32, g.ldj, g.w32, n, R, j, g.pA, g.pB, g.ldp, g.Hi, mi, g.rci, g.rsi, g.sti, tol, s));
  }
  k_btrsv<<<R, 32, 0, s>>>(g.Hi, mi, g.sti, g.yi); sie::count_launch();
  k_bcombine<float, float><<<grid, RT_, 0, s>>>(g.V32, g.ldj, g.yi, mi + 1, g.sti, n, pre ? g.r32 : g.z32, 0);
  sie::count_launch();
  if (pre) SIE_TRY(ras_apply32(c, g.r32, g.z32, s, R));
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// The inner cycle of the batch as a CUDA graph: every launch of one cycle (about 17 per
// inner step) is captured once per solve and replayed for the later outer steps.  Its
// pointers and scalars are fixed for the solve (input r32, output z32, the basis, the
// tables).  The first cycle runs uncaptured, so the lazily made buffers of the batched
// products exist before the capture; a capture that fails falls back to plain launches.
struct InnerGraph {
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels = 0;
  bool tried = false;
  ~InnerGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

static int inner_cycle(sie_ctx* c, GmB& g, double tol, InnerGraph& ig, bool first) {
  cudaStream_t s = c->stream;
  if (ig.exec) {
    SIE_CUDA(cudaGraphLaunch(ig.exec, s));
    count_launches(ig.kernels);
    c->tm.graph_replays += 1;
    return SIE_OK;
  }
  const char* ge = getenv("SIE_GRAPH");
  const bool enabled = !(ge && atoi(ge) == 0);
  if (first || ig.tried || !enabled) return inner_batch32(c, g, tol);
  ig.tried = true;
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    const int r = inner_batch32(c, g, tol);
    const cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (r == SIE_OK && e == cudaSuccess && graph &&
        cudaGraphInstantiate(&ig.exec, graph, 0) == cudaSuccess) {
      size_t nn = 0;
      cudaGraphGetNodes(graph, nullptr, &nn);
      std::vector<cudaGraphNode_t> nodes(nn);
      if (nn) cudaGraphGetNodes(graph, nodes.data(), &nn);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ig.kernels++;
      }
    } else {
      ig.exec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
  }
  cudaGetLastError();  // a failed capture leaves no sticky error; fall back to launches
  if (ig.exec) {
    SIE_CUDA(cudaGraphLaunch(ig.exec, s));
    count_launches(ig.kernels);
    c->tm.graph_replays += 1;
    return SIE_OK;
  }
  return inner_batch32(c, g, tol);
}

int fgmres_mixed_batch(sie_ctx* c, const zc* d_b_ext, zc* d_x_ext, int R, const sie_solver_cfg* cfg,
                       sie_stats* stats) {
  InnerGraph ig;
  bool first_cycle = true;
  c->tm.graph_replays = 0;
  cudaStream_t s = c->stream;
  const int mo = cfg->restart, mi = cfg->inner_restart;
  if (R < 1 || R > SIE_BATCH_MAX) return fail(SIE_ERR_ARG, "batched solve: bad batch size");
  if (mi < 1 || mi + 1 > BJMAX || mo + 1 > BJMAX || !(cfg->inner_tolerance > 0))
    return fail(SIE_ERR_ARG, "batched solve: restarts must be 1..63");
  SIE_TRY(make_f32_tables(c));
  if (c->inner) SIE_TRY(make_f32_tables(c->inner));
  SIE_TRY(ras_to_f32(c));
  GmB g;
  SIE_TRY(gmb_alloc(c, R, mi, mo, g));
  const int n = g.n;
  const size_t vr = (size_t)R * n;
  dim3 grid(BNB, R);
  BState* hst = (BState*)c->h_gmb;
  int* hfin = (int*)(hst + SIE_BATCH_MAX);
  cudaEventRecord(c->ev[12], s);
  SIE_TRY(gather_ext_to_int(c, d_b_ext, g.b, R, s));
  if (cfg->use_initial_guess) SIE_TRY(gather_ext_to_int(c, d_x_ext, g.x, R, s));
  // ||b_r|| into sto[r].bn (the outer estimate is relative to it)
  k_bnorm<double><<<grid, RT_, 0, s>>>(g.b, n, g.pA, g.ldp); sie::count_launch();
  k_binit<double, double><<<grid, RT_, 0, s>>>(g.b, n, g.pA, g.ldp, g.W, g.Ho, mo, g.sto, 1, nullptr);
  sie::count_launch();
  SIE_CUDA(cudaMemcpyAsync(hst, g.sto, R * sizeof(BState), cudaMemcpyDeviceToHost, s));
  SIE_CUDA(cudaStreamSynchronize(s));
  std::vector<double> bn(R), be(R, 1e300), bea(R, 1e300);
  std::vector<int> its(R, 0), conv(R, 0), mv(R, 0);
  for (int r = 0; r < R; r++) {
    bn[r] = hst[r].beta;
    if (!std::isfinite(bn[r])) return fail(SIE_ERR_NONFINITE, "batched solve: non-finite right-hand side");
    hfin[r] = bn[r] == 0.0;  // x = 0 solves it
    if (hfin[r]) conv[r] = 1, be[r] = bea[r] = 0;
  }
  int it = 0;
  auto finish = [&](int code) {
    scatter_int_to_ext(c, g.x, d_x_ext, R, s);
    cudaEventRecord(c->ev[13], s);
    cudaEventSynchronize(c->ev[13]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[12], c->ev[13]);
    if (stats)
      for (int r = 0; r < R; r++) {
        stats[r].iterations = its[r];
        stats[r].inner_iterations = its[r] * mi;
        stats[r].matvecs = mv[r];
        stats[r].converged = conv[r];
        stats[r].backward_error_arnoldi = bea[r];
        stats[r].backward_error_true = be[r];
        stats[r].seconds = ms * 1e-3;
      }
    return code;
  };
  bool first = true;
  while (true) {
    // r0 = b - A x in FP64 for the whole batch, then the cycle's start vectors
    if (first && !cfg->use_initial_guess) {
      k_copy<<<RB, RT_, 0, s>>>(g.b, g.w64, (int)vr); sie::count_launch();
    } else {
      SIE_TRY(sie_internal_matvec_b(c, g.x, g.r0, R, s));
      for (int r = 0; r < R; r++)
        if (!hfin[r]) mv[r]++;
      k_sub<<<RB, RT_, 0, s>>>(g.b, g.r0, g.w64, (int)vr); sie::count_launch();
    }
    first = false;
    SIE_CUDA(cudaMemcpyAsync(g.fin, hfin, R * sizeof(int), cudaMemcpyHostToDevice, s));
    k_bnorm<double><<<grid, RT_, 0, s>>>(g.w64, n, g.pA, g.ldp); sie::count_launch();
    k_binit<double, double><<<grid, RT_, 0, s>>>(g.w64, n, g.pA, g.ldp, g.W, g.Ho, mo, g.sto, 0, g.fin);
    sie::count_launch();
    SIE_CUDA(cudaMemcpyAsync(hst, g.sto, R * sizeof(BState), cudaMemcpyDeviceToHost, s));
    SIE_CUDA(cudaStreamSynchronize(s));
    bool all = true, frozen_changed = false;
    for (int r = 0; r < R; r++) {
      if (hfin[r]) continue;
      if (!std::isfinite(hst[r].beta)) return finish(fail(SIE_ERR_NONFINITE, "batched solve: non-finite residual"));
      be[r] = hst[r].beta / bn[r];
      if (be[r] <= cfg->tolerance) {
        hfin[r] = 1;
        conv[r] = 1;
        frozen_changed = true;
      } else {
        all = false;
      }
    }
    if (all) return finish(SIE_OK);
    if (it >= cfg->max_iterations) return finish(fail(SIE_ERR_NOCONV, "batched solve: no convergence"));
    if (frozen_changed) {  // systems that just converged take no further steps
      SIE_CUDA(cudaMemcpyAsync(g.fin, hfin, R * sizeof(int), cudaMemcpyHostToDevice, s));
      k_binit<double, double><<<grid, RT_, 0, s>>>(g.w64, n, g.pA, g.ldp, g.W, g.Ho, mo, g.sto, 0, g.fin);
      sie::count_launch();
    }
    for (int j = 0; j < mo; j++) {
      SIE_TRY(to_c64(g.W + (size_t)j * g.ldj, g.r32, vr, s));
      SIE_TRY(inner_cycle(c, g, cfg->inner_tolerance, ig, first_cycle));
      first_cycle = false;
      SIE_TRY(to_c128(g.z32, g.Zb + (size_t)j * g.ldj, vr, s));
      SIE_TRY(sie_internal_matvec_b(c, g.Zb + (size_t)j * g.ldj, g.w64, R, s));
      SIE_TRY(barnoldi<double>(g.W, g.ldj, g.w64, n, R, j, g.pA, g.pB, g.ldp, g.Ho, mo, g.rco, g.rso, g.sto,
                               cfg->tolerance, s));
      it++;
      SIE_CUDA(cudaMemcpyAsync(hst, g.sto, R * sizeof(BState), cudaMemcpyDeviceToHost, s));
      SIE_CUDA(cudaStreamSynchronize(s));
      bool alldone = true;
      for (int r = 0; r < R; r++) {
        if (hfin[r]) continue;
        its[r]++;
        mv[r] += mi + 1;
        if (!std::isfinite(hst[r].bea)) return finish(fail(SIE_ERR_NONFINITE, "batched solve: non-finite Arnoldi vector"));
        bea[r] = hst[r].bea;
        if (!hst[r].done) alldone = false;
      }
      if (alldone || it >= cfg->max_iterations) break;
      if (cfg->time_limit_s > 0) {
        float el = 0;
        cudaEventRecord(c->ev[13], s);
        cudaEventSynchronize(c->ev[13]);
        cudaEventElapsedTime(&el, c->ev[12], c->ev[13]);
        if (el * 1e-3 > cfg->time_limit_s) {
          finish(SIE_ERR_TIMEOUT);
          return fail(SIE_ERR_TIMEOUT, "batched solve: time limit reached");
        }
      }
    }
    // x_r += Z_r y_r over the steps each system took
    k_btrsv<<<R, 32, 0, s>>>(g.Ho, mo, g.sto, g.yo); sie::count_launch();
    k_bcombine<double, double><<<grid, RT_, 0, s>>>(g.Zb, g.ldj, g.yo, mo + 1, g.sto, n, g.x, 1);
    sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
}

}  // namespace sie
