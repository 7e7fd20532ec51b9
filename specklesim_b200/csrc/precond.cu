// Near-field restricted additive Schwarz (RAS) preconditioner.
//
// The reference offers only a left Jacobi scaling by the self blocks
// (lib_sie_ml_fmm_preconditioner_left, src/lib_sie_tri_mlfmm_interface.f90:323-339),
// off by default.  ICTF and PMCHWT are first-kind formulations: on a rough plasmonic
// slab (Re eps = -11.7) the system has cond(Z) ~ 1e7 already at 5k unknowns, and
// unpreconditioned GMRES stalls.  This preconditioner is built from the near matrix
// alone (no extra integrals):
//
//   for each leaf box A, S_A = E2(A) (A and its neighbour boxes, the columns of A's near
//   panel).  L_A = Z_near restricted to S_A x S_A, where an entry (i, j) is the near
//   block of (i, j) if box(j) is in E2(box(i)) and zero otherwise.  The preconditioner's
//   rows of A's unknowns are the rows of L_A^{-1} that belong to A:
//       P[A, S_A] = E_A^T L_A^{-1}.
//
// P has the sparsity of the near panels (rows of A, columns E2(A)), stored as a full 2x2
// block per panel element (4 complex values: no symmetry between the off-diagonal
// blocks), and is applied with the same chunked panel kernel shape as the near product.
// The solvers use it on the right (x = P u), so their residuals stay the true ones.
//
// Set-up: per leaf box, the local matrix is expanded on the device from the near panels
// (k_ras_local), factorised by LU with partial pivoting, and the rows are obtained by one
// transposed solve with the 2|A| unit vectors of A (L_A^T Y = E_A, Y = P[A, S_A]^T).  The
// LU and the solve are cuSOLVER calls (getrf/getrs), set-up only; the product kernel is
// this file's own.
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "sie_internal.h"

namespace sie {

// One (B, C) box pair of a local system: rows of box B, columns of box C.
struct RasPair {
  int B, C;        // leaf boxes
  int row0, col0;  // first local edge of B and of C in S_A
  int off;         // first column of C inside B's near panel, -1 if C is not in E2(B)
  int pad;
};

// L (column-major, leading dimension ld = 2 n_A), one block per box pair.
__global__ void k_ras_local(const long long* __restrict__ base, const int* __restrict__ box_first,
                            const int* __restrict__ box_cnt, const int* __restrict__ ncols,
                            const zc* __restrict__ va, const zc* __restrict__ vb,
                            const zc* __restrict__ vd, zc cfac, const RasPair* __restrict__ pairs,
                            int ld, zc* __restrict__ L) {
  const RasPair p = pairs[blockIdx.x];
  const int nr = box_cnt[p.B], nc = box_cnt[p.C];
  const int pnc = ncols[p.B];
  const int tot = nr * nc;
  for (int k = threadIdx.x; k < tot; k += blockDim.x) {
    const int r = k / nc, cl = k - r * nc;
    zc a = mk<double>(0, 0), b = a, c = a, d = a;
    if (p.off >= 0) {
      const long long o = base[p.B] + (long long)r * pnc + p.off + cl;
      a = va[o];
      b = vb[o];
      c = cfac * b;
      d = vd[o];
    }
    const size_t i = 2 * (size_t)(p.row0 + r), j = 2 * (size_t)(p.col0 + cl);
    L[j * ld + i] = a;
    L[(j + 1) * ld + i] = b;
    L[j * ld + i + 1] = c;
    L[(j + 1) * ld + i + 1] = d;
  }
}

// Y (ld x 2 nA, column-major) = the unit vectors of A's unknowns inside S_A.
__global__ void k_ras_units(zc* Y, int ld, int self0, int nA) {
  const size_t tot = (size_t)ld * 2 * nA;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (size_t)gridDim.x * blockDim.x) {
    const size_t col = k / ld, row = k - col * ld;
    Y[k] = mk<double>(row == 2 * (size_t)self0 + col ? 1.0 : 0.0, 0.0);
  }
}

// P panel of A from Y: P[2r + a][2j + b] = Y[2j + b][2r + a].  A failed factorisation
// (info != 0) is recorded in *err.
__global__ void k_ras_store(const zc* __restrict__ Y, int ld, int nA, int nS, long long pbase,
                            const int* __restrict__ info, int* err, zc* pa, zc* pb, zc* pc, zc* pd) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && *info != 0) atomicOr(err, 1);
  const long long tot = (long long)nA * nS;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(k / nS), j = (int)(k - (long long)r * nS);
    const size_t c0 = (size_t)(2 * r) * ld, c1 = (size_t)(2 * r + 1) * ld;
    const long long o = pbase + k;
    pa[o] = Y[c0 + 2 * j];
    pb[o] = Y[c0 + 2 * j + 1];
    pc[o] = Y[c1 + 2 * j];
    pd[o] = Y[c1 + 2 * j + 1];
  }
}

// y = P x over work chunks of at most 32 rows of one leaf box (the near product's
// chunks): x of the panel's columns is gathered into shared memory, then each warp
// streams whole rows of the four block arrays against it.  gridDim.y vectors at the
// given stride (a batch): the blocks of one chunk read the same panel rows, mostly
// from L2.
template <typename T, int NW>
__global__ void __launch_bounds__(32 * NW) k_ras_apply(const long long* __restrict__ base,
                                                   const int* __restrict__ box_first,
                                                   const int* __restrict__ box_cnt,
                                                   const int* __restrict__ nbr_ptr,
                                                   const int* __restrict__ nbr_box,
                                                   const int* __restrict__ ncols,
                                                   const cx<T>* __restrict__ pa,
                                                   const cx<T>* __restrict__ pb,
                                                   const cx<T>* __restrict__ pc,
                                                   const cx<T>* __restrict__ pd,
                                                   const int4* __restrict__ chunks,
                                                   const cx<T>* __restrict__ x, cx<T>* __restrict__ y,
                                                   size_t stride) {
  extern __shared__ __align__(16) unsigned char smraw[];
  x += blockIdx.y * stride;  // vector blockIdx.y of a batch
  y += blockIdx.y * stride;
  cx<T>* xs = reinterpret_cast<cx<T>*>(smraw);  // [ncols][J, M]
  const int4 ch = chunks[blockIdx.x];
  const int A = ch.x, f = ch.y, cnt = ch.z;
  const int nc = ncols[A];
  const long long b0 = base[A] + (long long)(f - box_first[A]) * nc;
  const unsigned long long pol = l2_evict_first_policy();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int col0 = 0;
  for (int k = nbr_ptr[A]; k < nbr_ptr[A + 1]; k++) {
    const int B = nbr_box[k];
    const int c = box_cnt[B], fb = box_first[B];
    for (int j = threadIdx.x; j < 2 * c; j += blockDim.x) xs[2 * col0 + j] = x[2 * fb + j];
    col0 += c;
  }
  __syncthreads();
  for (int row = warp; row < cnt; row += NW) {
    const long long o = b0 + (long long)row * nc;
    cx<T> sJ = mk<T>(0, 0), sM = mk<T>(0, 0);
#pragma unroll 4
    for (int j = lane; j < nc; j += 32) {
      const cx<T> a = ld_stream(pa + o + j, pol), b = ld_stream(pb + o + j, pol);
      const cx<T> c = ld_stream(pc + o + j, pol), d = ld_stream(pd + o + j, pol);
      const cx<T> xj = xs[2 * j], xm = xs[2 * j + 1];
      sJ = cfma(a, xj, sJ);
      sJ = cfma(b, xm, sJ);
      sM = cfma(c, xj, sM);
      sM = cfma(d, xm, sM);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      sJ.re += __shfl_xor_sync(0xffffffffu, sJ.re, s);
      sJ.im += __shfl_xor_sync(0xffffffffu, sJ.im, s);
      sM.re += __shfl_xor_sync(0xffffffffu, sM.re, s);
      sM.im += __shfl_xor_sync(0xffffffffu, sM.im, s);
    }
    if (lane == 0) {
      cx<T>* yr = y + 2 * (size_t)(f + row);
      yr[0] = sJ;
      yr[1] = sM;
    }
  }
}

__global__ void k_c128_to_c64(const zc* a, cc* b, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = mk<float>((float)a[i].re, (float)a[i].im);
}

static size_t ras_smem(const sie_ctx* c, size_t elem) { return std::max<size_t>((size_t)c->ncols_max * 2 * elem, 16); }

void ras_release(sie_ctx* c) {
  void* p[] = {c->d_pa, c->d_pb, c->d_pc, c->d_pd, c->d_pa32, c->d_pb32, c->d_pc32, c->d_pd32};
  for (void* q : p)
    if (q) cudaFree(q);
  c->d_pa = c->d_pb = c->d_pc = c->d_pd = nullptr;
  c->d_pa32 = c->d_pb32 = c->d_pc32 = c->d_pd32 = nullptr;
  c->precond = SIE_PRECOND_NONE;
}

// Device workspace of the set-up, freed on every exit path.
struct RasWork {
  std::vector<void*> ptrs;
  std::vector<cusolverDnHandle_t> handles;
  std::vector<cudaStream_t> streams;
  ~RasWork() {
    for (auto s : streams) cudaStreamSynchronize(s);
    for (auto h : handles) cusolverDnDestroy(h);
    for (auto s : streams) cudaStreamDestroy(s);
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

int ras_build(sie_ctx* c) {
  if (c->cfg.dense) return fail(SIE_ERR_STATE, "near-field preconditioner: not for dense contexts (use sie_solve_direct)");
  const NearLayout& N = c->near;
  const int nbox = N.nbox;
  const long long nnz = N.nnz;
  // host tables: the E2 list of every box with each member's first column in the panel
  std::vector<std::vector<std::pair<int, int>>> colof(nbox);
  for (int B = 0; B < nbox; B++) {
    int off = 0;
    for (int k = N.nbr_ptr[B]; k < N.nbr_ptr[B + 1]; k++) {
      colof[B].push_back({N.nbr_box[k], off});
      off += N.box_cnt[N.nbr_box[k]];
    }
  }
  auto find_col = [&](int B, int C) {
    const auto& v = colof[B];
    auto it = std::lower_bound(v.begin(), v.end(), std::make_pair(C, -1));
    return (it != v.end() && it->first == C) ? it->second : -1;
  };
  std::vector<long long> pair_ptr(nbox + 1, 0);
  std::vector<RasPair> pairs;
  std::vector<int> self0(nbox, -1);
  for (int A = 0; A < nbox; A++) {
    const auto& SA = colof[A];
    for (const auto& bi : SA) {
      if (bi.first == A) self0[A] = bi.second;
      for (const auto& ci : SA) {
        RasPair p;
        p.B = bi.first;
        p.C = ci.first;
        p.row0 = bi.second;
        p.col0 = ci.second;
        p.off = find_col(bi.first, ci.first);
        p.pad = 0;
        pairs.push_back(p);
      }
    }
    pair_ptr[A + 1] = (long long)pairs.size();
    if (self0[A] < 0) return fail(SIE_ERR_STATE, "near-field preconditioner: a box is missing from its own E2 list");
  }
  const int nmax = 2 * c->ncols_max;
  int amax = 0;
  for (int A = 0; A < nbox; A++) amax = std::max(amax, N.box_cnt[A]);
  const size_t lbytes = (size_t)nmax * nmax * sizeof(zc);
  const size_t ybytes = (size_t)nmax * 2 * amax * sizeof(zc);
  // concurrent factorisations: up to 4, within 8 GB of workspace
  int ns = 4;
  while (ns > 1 && (size_t)ns * (lbytes + ybytes) > ((size_t)8 << 30)) ns--;
  ras_release(c);
  RasWork W;
  RasPair* d_pairs = nullptr;
  SIE_CUDA(W.alloc(&d_pairs, pairs.size() * sizeof(RasPair)));
  SIE_CUDA(cudaMemcpy(d_pairs, pairs.data(), pairs.size() * sizeof(RasPair), cudaMemcpyHostToDevice));
  const size_t pbytes = (size_t)std::max<long long>(nnz, 1) * sizeof(zc);
  SIE_CUDA(cudaMalloc(&c->d_pa, pbytes));
  SIE_CUDA(cudaMalloc(&c->d_pb, pbytes));
  SIE_CUDA(cudaMalloc(&c->d_pc, pbytes));
  SIE_CUDA(cudaMalloc(&c->d_pd, pbytes));
  int* d_err = nullptr;
  SIE_CUDA(W.alloc(&d_err, sizeof(int)));
  SIE_CUDA(cudaMemset(d_err, 0, sizeof(int)));
  std::vector<zc*> L(ns), Y(ns), work(ns);
  std::vector<int*> piv(ns);
  int lwork = 0;
  for (int s = 0; s < ns; s++) {
    cudaStream_t st;
    SIE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    W.streams.push_back(st);
    cusolverDnHandle_t h;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return fail(SIE_ERR_CUDA, "cusolverDnCreate");
    W.handles.push_back(h);
    if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return fail(SIE_ERR_CUDA, "cusolverDnSetStream");
    SIE_CUDA(W.alloc(&L[s], lbytes));
    SIE_CUDA(W.alloc(&Y[s], ybytes));
    SIE_CUDA(W.alloc(&piv[s], (size_t)(nmax + 2) * sizeof(int)));  // pivots, getrf info, getrs info
  }
  if (cusolverDnZgetrf_bufferSize(W.handles[0], nmax, nmax, (cuDoubleComplex*)L[0], nmax, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(SIE_ERR_CUDA, "cusolverDnZgetrf_bufferSize");
  for (int s = 0; s < ns; s++) SIE_CUDA(W.alloc(&work[s], (size_t)std::max(lwork, 1) * sizeof(zc)));
  // the near panels are complete once the context's stream has drained
  SIE_CUDA(cudaStreamSynchronize(c->stream));
  // largest local systems first, so the concurrent streams finish together
  std::vector<int> order(nbox);
  for (int A = 0; A < nbox; A++) order[A] = A;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return N.ncols[a] > N.ncols[b]; });
  for (int t = 0; t < nbox; t++) {
    const int A = order[t], s = t % ns;
    cudaStream_t st = W.streams[s];
    const int n = 2 * N.ncols[A], nA = N.box_cnt[A];
    const int np = (int)(pair_ptr[A + 1] - pair_ptr[A]);
    k_ras_local<<<np, 256, 0, st>>>(c->d_base, c->d_box_first, c->d_box_cnt, c->d_ncols, c->d_na, c->d_nb,
                                    c->d_nd, c->cfac, d_pairs + pair_ptr[A], n, L[s]);
    count_launch();
    k_ras_units<<<148, 256, 0, st>>>(Y[s], n, self0[A], nA);
    count_launch();
    SIE_CUDA(cudaGetLastError());
    if (cusolverDnZgetrf(W.handles[s], n, n, (cuDoubleComplex*)L[s], n, (cuDoubleComplex*)work[s], piv[s],
                         piv[s] + nmax) != CUSOLVER_STATUS_SUCCESS)
      return fail(SIE_ERR_CUDA, "near-field preconditioner: cusolverDnZgetrf");
    if (cusolverDnZgetrs(W.handles[s], CUBLAS_OP_T, n, 2 * nA, (const cuDoubleComplex*)L[s], n, piv[s],
                         (cuDoubleComplex*)Y[s], n, piv[s] + nmax + 1) != CUSOLVER_STATUS_SUCCESS)
      return fail(SIE_ERR_CUDA, "near-field preconditioner: cusolverDnZgetrs");
    k_ras_store<<<148, 256, 0, st>>>(Y[s], n, nA, N.ncols[A], N.base[A], piv[s] + nmax, d_err, c->d_pa,
                                     c->d_pb, c->d_pc, c->d_pd);
    count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  for (auto st : W.streams) SIE_CUDA(cudaStreamSynchronize(st));
  int err = 0;
  SIE_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    ras_release(c);
    return fail(SIE_ERR_NONFINITE, "near-field preconditioner: a local system is singular");
  }
  if (ras_smem(c, sizeof(zc)) > (size_t)200 * 1024) {
    ras_release(c);
    return fail(SIE_ERR_ARG, "near-field preconditioner: a near panel is too wide for the product kernel");
  }
  SIE_CUDA(raise_smem(k_ras_apply<double, 8>, ras_smem(c, sizeof(zc))));
  SIE_CUDA(raise_smem(k_ras_apply<float, 8>, ras_smem(c, sizeof(cc))));
  c->precond = SIE_PRECOND_NEAR;
  return SIE_OK;
}

int ras_to_f32(sie_ctx* c) {
  if (c->d_pa32 || c->precond != SIE_PRECOND_NEAR) return SIE_OK;
  const long long n = std::max<long long>(c->near.nnz, 1);
  SIE_CUDA(cudaMalloc(&c->d_pa32, n * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_pb32, n * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_pc32, n * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_pd32, n * sizeof(cc)));
  k_c128_to_c64<<<4 * 148, 256, 0, c->stream>>>(c->d_pa, c->d_pa32, n); count_launch();
  k_c128_to_c64<<<4 * 148, 256, 0, c->stream>>>(c->d_pb, c->d_pb32, n); count_launch();
  k_c128_to_c64<<<4 * 148, 256, 0, c->stream>>>(c->d_pc, c->d_pc32, n); count_launch();
  k_c128_to_c64<<<4 * 148, 256, 0, c->stream>>>(c->d_pd, c->d_pd32, n); count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int ras_apply64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st, int R) {
  k_ras_apply<double, 8><<<dim3(c->n_rchunk, R), 256, ras_smem(c, sizeof(zc)), st>>>(
      c->d_base, c->d_box_first, c->d_box_cnt, c->d_nbr_ptr, c->d_nbr_box, c->d_ncols, c->d_pa, c->d_pb, c->d_pc,
      c->d_pd, (const int4*)c->d_rchunk, x, y, (size_t)2 * c->M);
  count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int ras_apply32(sie_ctx* c, const cc* x, cc* y, cudaStream_t st, int R) {
  k_ras_apply<float, 8><<<dim3(c->n_rchunk, R), 256, ras_smem(c, sizeof(cc)), st>>>(
      c->d_base, c->d_box_first, c->d_box_cnt, c->d_nbr_ptr, c->d_nbr_box, c->d_ncols, c->d_pa32, c->d_pb32,
      c->d_pc32, c->d_pd32, (const int4*)c->d_rchunk, x, y, (size_t)2 * c->M);
  count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

}  // namespace sie

using namespace sie;

extern "C" int sie_set_preconditioner(sie_ctx* c, int kind) {
  if (!c) return fail(SIE_ERR_ARG, "sie_set_preconditioner: null context");
  if (kind != SIE_PRECOND_NONE && kind != SIE_PRECOND_NEAR)
    return fail(SIE_ERR_ARG, "sie_set_preconditioner: unknown kind");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_set_preconditioner: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  if (kind == SIE_PRECOND_NONE) {
    SIE_CUDA(cudaStreamSynchronize(c->stream));
    ras_release(c);
    return SIE_OK;
  }
  if (c->precond == SIE_PRECOND_NEAR) return SIE_OK;
  auto t0 = std::chrono::steady_clock::now();
  const int r = ras_build(c);
  c->tm.precond_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

extern "C" int sie_precondition_right(sie_ctx* c, const double* v1, double* v2) {
  if (!c || !v1 || !v2) return fail(SIE_ERR_ARG, "sie_precondition_right: bad argument");
  if (c->precond != SIE_PRECOND_NEAR) return fail(SIE_ERR_STATE, "sie_precondition_right: no preconditioner set");
  SIE_CUDA(cudaSetDevice(c->device));
  const size_t bytes = (size_t)2 * c->M * sizeof(zc);
  zc *dext = nullptr, *dint = nullptr, *dout = nullptr;
  SIE_CUDA(cudaMalloc(&dext, bytes));
  int rc = SIE_OK;
  if (cudaMalloc(&dint, bytes) != cudaSuccess || cudaMalloc(&dout, bytes) != cudaSuccess)
    rc = fail(SIE_ERR_NOMEM, "sie_precondition_right: device buffers");
  if (rc == SIE_OK && cudaMemcpyAsync(dext, v1, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = fail(SIE_ERR_CUDA, "sie_precondition_right: copy");
  if (rc == SIE_OK) rc = gather_ext_to_int(c, dext, dint, 1, c->stream);
  if (rc == SIE_OK) rc = ras_apply64(c, dint, dout, c->stream);
  if (rc == SIE_OK) rc = scatter_int_to_ext(c, dout, dext, 1, c->stream);
  if (rc == SIE_OK && (cudaMemcpyAsync(v2, dext, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                       cudaStreamSynchronize(c->stream) != cudaSuccess))
    rc = fail(SIE_ERR_CUDA, "sie_precondition_right: copy back");
  cudaFree(dext);
  if (dint) cudaFree(dint);
  if (dout) cudaFree(dout);
  return rc;
}
