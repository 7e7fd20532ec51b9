// Direct solve of the dense system for small bodies: the reference's "normal" solver
// (lib_sie_tri_solver_normal_I, src/lib_sie_tri_solver_normal.f90:64-217) fills the full
// FP64 matrix and calls ZGESV (solver_LU, src/lib_sie_math.f90:649-676).  Here the dense
// near panels (cfg.dense = 1: every pair in the near matrix) are expanded on the GPU into
// one column-major N x N matrix in the internal interleaved (J, M) order, factorised once
// with cuSOLVER's LU with partial pivoting and reused for every right-hand side.
#include <cusolverDn.h>

#include "sie_internal.h"

namespace sie {

// Panel element (A, r, j) -> Z[2m + a, 2n + b] with m = first(A) + r and n = j (in dense
// mode the panel columns are all edges in internal order).
__global__ void k_expand_dense(const long long* base, const int* box_first, const int* box_cnt,
                               const int* ncols, int nbox, const zc* va, const zc* vb,
                               const zc* vd, zc cfac, int M, zc* Z) {
  long long ld = 2LL * M;
  for (int A = blockIdx.y; A < nbox; A += gridDim.y) {
    int nr = box_cnt[A], nc = ncols[A], f = box_first[A];
    long long tot = (long long)nr * nc;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tot;
         k += (long long)gridDim.x * blockDim.x) {
      int r = (int)(k / nc), j = (int)(k % nc);
      long long o = base[A] + k;
      long long m = f + r, n = j;
      zc a = va[o], b = vb[o], d = vd[o];
      Z[(2 * n) * ld + 2 * m] = a;
      Z[(2 * n + 1) * ld + 2 * m] = b;
      Z[(2 * n) * ld + 2 * m + 1] = cfac * b;
      Z[(2 * n + 1) * ld + 2 * m + 1] = d;
    }
  }
}

}  // namespace sie

using namespace sie;

static int lu_factor(sie_ctx* c) {
  if (c->d_lu && c->lu64_valid) return SIE_OK;
  int n = 2 * c->M;
  size_t bytes = (size_t)n * n * sizeof(zc);
  if (!c->d_lu) SIE_CUDA(cudaMalloc(&c->d_lu, bytes));
  if (!c->d_piv) SIE_CUDA(cudaMalloc(&c->d_piv, (size_t)(n + 1) * sizeof(int)));
  dim3 g(64, std::min(c->near.nbox, 1024));
  k_expand_dense<<<g, 256, 0, c->stream>>>(c->d_base, c->d_box_first, c->d_box_cnt, c->d_ncols,
                                            c->near.nbox, c->d_na, c->d_nb, c->d_nd, c->cfac,
                                            c->M, (zc*)c->d_lu);
  count_launch();
  SIE_CUDA(cudaGetLastError());
  cusolverDnHandle_t h = nullptr;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return fail(SIE_ERR_CUDA, "cusolverDnCreate");
  int rc = SIE_OK;
  int lwork = 0;
  cuDoubleComplex* work = nullptr;
  if (cusolverDnSetStream(h, c->stream) != CUSOLVER_STATUS_SUCCESS ||
      cusolverDnZgetrf_bufferSize(h, n, n, (cuDoubleComplex*)c->d_lu, n, &lwork) != CUSOLVER_STATUS_SUCCESS)
    rc = fail(SIE_ERR_CUDA, "cusolverDnZgetrf_bufferSize");
  if (rc == SIE_OK && cudaMalloc(&work, (size_t)std::max(lwork, 1) * sizeof(cuDoubleComplex)) != cudaSuccess)
    rc = fail(SIE_ERR_NOMEM, "LU workspace");
  if (rc == SIE_OK && cusolverDnZgetrf(h, n, n, (cuDoubleComplex*)c->d_lu, n, work, c->d_piv,
                                       c->d_piv + n) != CUSOLVER_STATUS_SUCCESS)
    rc = fail(SIE_ERR_CUDA, "cusolverDnZgetrf");
  int info = 0;
  if (rc == SIE_OK) {
    if (cudaMemcpyAsync(&info, c->d_piv + n, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
      rc = fail(SIE_ERR_CUDA, "LU info");
    else if (info != 0)
      rc = fail(SIE_ERR_NONFINITE, "LU: singular matrix (zero pivot)");
  }
  if (work) cudaFree(work);
  cusolverDnDestroy(h);
  if (rc != SIE_OK) {
    cudaFree(c->d_lu);
    cudaFree(c->d_piv);
    c->d_lu = nullptr;
    c->d_piv = nullptr;
  }
  c->lu64_valid = rc == SIE_OK;
  return rc;
}

extern "C" int sie_solve_direct(sie_ctx* c, const double* b, double* x, int nrhs) {
  if (!c || !b || !x || nrhs < 1) return fail(SIE_ERR_ARG, "sie_solve_direct: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_solve_direct: sie_setup not called");
  if (!c->cfg.dense) return fail(SIE_ERR_STATE, "sie_solve_direct: needs a context set up with dense = 1");
  SIE_CUDA(cudaSetDevice(c->device));
  for (size_t i = 0; i < (size_t)4 * c->M * nrhs; i++)
    if (!std::isfinite(b[i])) return fail(SIE_ERR_NONFINITE, "sie_solve_direct: non-finite right-hand side");
  SIE_TRY(lu_factor(c));
  int n = 2 * c->M;
  size_t bytes = (size_t)n * nrhs * sizeof(zc);
  zc *dext = nullptr, *dint = nullptr;
  SIE_CUDA(cudaMalloc(&dext, bytes));
  SIE_CUDA(cudaMalloc(&dint, bytes));
  int rc = SIE_OK;
  if (cudaMemcpyAsync(dext, b, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct: copy");
  if (rc == SIE_OK) rc = gather_ext_to_int(c, dext, dint, nrhs, c->stream);
  cusolverDnHandle_t h = nullptr;
  if (rc == SIE_OK && cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) rc = fail(SIE_ERR_CUDA, "cusolverDnCreate");
  if (rc == SIE_OK && (cusolverDnSetStream(h, c->stream) != CUSOLVER_STATUS_SUCCESS ||
                       cusolverDnZgetrs(h, CUBLAS_OP_N, n, nrhs, (const cuDoubleComplex*)c->d_lu, n,
                                        c->d_piv, (cuDoubleComplex*)dint, n,
                                        c->d_piv + n) != CUSOLVER_STATUS_SUCCESS))
    rc = fail(SIE_ERR_CUDA, "cusolverDnZgetrs");
  if (h) cusolverDnDestroy(h);
  if (rc == SIE_OK) rc = scatter_int_to_ext(c, dint, dext, nrhs, c->stream);
  if (rc == SIE_OK && (cudaMemcpyAsync(x, dext, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                       cudaStreamSynchronize(c->stream) != cudaSuccess))
    rc = fail(SIE_ERR_CUDA, "sie_solve_direct: copy back");
  cudaFree(dext);
  cudaFree(dint);
  return rc;
}

// Z^H y = g in place on one internal-layout vector with the LU factors (adjoint solve of
// the shape gradient on a dense context).
int sie::lu_solve_adjoint(sie_ctx* c, zc* d_int) {
  SIE_TRY(lu_factor(c));
  int n = 2 * c->M;
  cusolverDnHandle_t h = nullptr;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return fail(SIE_ERR_CUDA, "cusolverDnCreate");
  int rc = SIE_OK;
  if (cusolverDnSetStream(h, c->stream) != CUSOLVER_STATUS_SUCCESS ||
      cusolverDnZgetrs(h, CUBLAS_OP_C, n, 1, (const cuDoubleComplex*)c->d_lu, n, c->d_piv,
                       (cuDoubleComplex*)d_int, n, c->d_piv + n) != CUSOLVER_STATUS_SUCCESS)
    rc = fail(SIE_ERR_CUDA, "cusolverDnZgetrs (adjoint)");
  cusolverDnDestroy(h);
  if (rc == SIE_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(SIE_ERR_CUDA, "adjoint LU solve");
  return rc;
}
