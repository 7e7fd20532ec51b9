// Internal state of the B200 SIE library (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "../../include/sie_gpu.h"

namespace sie {

// Unsuffixed Fortran literals of the reference are binary32
// (src/lib_sie_constants.f90:9-11, no real-kind promotion in the build).
static const double C0 = (double)2.99792458e+8f;
static const double EPS0 = (double)8.854187817e-12f;
static const double MU0 = (double)1.2566370614e-6f;
static const double PI = 3.141592653589793238462643383279502884;

void set_error(const std::string& msg);
// number of kernels launched by this library since load (for the bench's launch count)
void count_launch();
void count_launches(unsigned long long n);  // kernels of a replayed CUDA graph
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// Host-to-device copy that has landed when it returns.  A plain cudaMemcpy from pageable
// memory may return while its DMA is still in flight, and the library's kernels run on
// a stream that does not wait for the legacy default stream.
inline cudaError_t h2d(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(cudaStreamLegacy);
}

// Allow kernel fn up to `bytes` of dynamic shared memory.  The limit is a property of the
// function for the whole process, shared by every context, so it is only ever raised:
// lowering it for one mesh would make another context's launches fail.
template <typename F>
inline cudaError_t raise_smem(F* fn, size_t bytes) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, (const void*)fn);
  if (e != cudaSuccess) return e;
  if ((int)bytes <= a.maxDynamicSharedSizeBytes) return cudaSuccess;
  return cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define SIE_TRY(x)               \
  do {                           \
    int _r = (x);                \
    if (_r != SIE_OK) return _r; \
  } while (0)

#define SIE_CUDA(call)                                      \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return sie::cuda_fail(_e, #call); \
  } while (0)

// Triangle quadrature rule (src/lib_sie_integration_points.f90:7-141).
struct Rule {
  int n;
  double a[12], b[12], w[12];
};
Rule make_rule(int ngp);

// Half RWG basis of one edge side (fn_rwg, src/lib_sie_type_function.f90:12-20).
struct FnD {
  double c[9];  // p1, p2, pc
  double area, length, df, sgn;
  double mid[3], nq[3];
  int tri;
  int pad;
};

struct Material {
  double k0, omega, my1, my2;
  zc k1, k2, eps1, eps2, eta1, eta2, eta_a;
};

// Device copy of everything the fill kernels need.
struct FillArgs {
  const FnD* fn;        // 2 per internal edge
  const double* rref;   // per internal edge
  const double* cent;   // 3 per triangle
  Material mt;
  Rule R;
  int formulation;
  int fix_itbn;
  int smooth;  // 1: x_nt kept in FP64 (shape gradient), 0: rounded to binary32 as the reference
};

// Near-field matrix laid out per leaf box A: rows = edges of A (internal order),
// columns = edges of the present boxes of E2(A) (self + neighbours, ascending
// box index) -- a dense (|A| x |E2(A)|) panel of 2x2 complex blocks.
struct NearLayout {
  int nbox;
  std::vector<int> box_first, box_cnt;   // leaf boxes in internal edge numbering
  std::vector<int> nbr_ptr, nbr_box;     // E2 box lists per leaf box
  std::vector<int> ncols;                // columns per leaf box
  std::vector<long long> base;           // value offset of the panel of box A
  long long nnz;
};

// Interpolation between the k-space samplings of two levels as a sparse real matrix
// acting on each (theta, phi) item pair of a box's coefficients.
struct InterpDev {
  int rows = 0;               // 2 Q_out
  int* ptr = nullptr;         // rows + 1
  int* col = nullptr;         // into the 2 Q_in input values (theta values, then phi)
  double* val = nullptr;
  float* val32 = nullptr;     // complex64 passes (made with the other complex64 tables)
  long long nnz = 0;
  // the same stencil tap-major (ELL): tap t of row r at [t * rows + r], rows padded to
  // ew taps with weight 0, so a warp's 32 rows read each tap coalesced; the taps of the
  // few longer rows (the poles of the anterpolation) past ew in a CSR overflow
  int ew = 0;
  int* ecol = nullptr;
  double* eval = nullptr;
  float* eval32 = nullptr;
  int* optr = nullptr;
  int* ocol = nullptr;
  double* oval = nullptr;
  float* oval32 = nullptr;
  long long onnz = 0;
};

struct Level {
  int l = 0;
  int nb = 0;
  // k-space sampling of this level (truncation number K, Q = 2 K^2 + 2 directions)
  int K = 0, Q = 0;
  double* khat = nullptr;     // 3 x Q
  double* trf = nullptr;      // Q quadrature weights
  float* trf32 = nullptr;
  // between this level and its children (l + 1) when their samplings differ: up = child
  // -> this level (SS), dn = this level -> child (RR, the transpose of up)
  InterpDev up, dn;
  std::vector<uint64_t> box;  // Morton indices, ascending
  // device
  zc* C = nullptr;            // nb x 8 x Q
  zc* D = nullptr;            // nb x 8 x Q
  zc* tl = nullptr;           // 343 x 2 x Q
  // on the PARENT level's sampling (Q_{l-1}): the SS shift follows the interpolation to
  // the parent's sampling, and the RR shift precedes the anterpolation to this level's
  zc* ph_up = nullptr;        // 8 octants x 2 media x Q_{l-1}  exp(+i k khat.(x_child - x_parent))
  zc* ph_dn = nullptr;        // 8 octants x 2 media x Q_{l-1}  exp(-i k khat.(x_child - x_parent))
  int* i4_ptr = nullptr;      // nb + 1
  int* i4_src = nullptr;      // source box index (same level)
  int* i4_off = nullptr;      // TL offset index 0..342
  int* ch_ptr = nullptr;      // children (level l+1) per box: nb + 1
  int* ch_idx = nullptr;
  int* ch_oct = nullptr;
  int* parent = nullptr;      // parent index (level l-1) per box, -1 if none
  int* oct = nullptr;         // octant of the box in its parent
  bool only_k1 = false;       // TL for k2 is zero at this level
  long long n_i4 = 0;
  // sibling groups (children of one parent at level l-1) for the SR translation
  int ngrp = 0;
  int* grp_sib = nullptr;     // ngrp x 8 box indices (-1: absent)
  int* grp_src = nullptr;     // ngrp x 27 x 8 candidate source box indices (-1: absent)
  // present siblings x present sources outside the parent, per group; the groups are
  // stored in descending order of it, so that the warps of one block get equal work
  std::vector<int> grp_cost;
  // complex64 copies for the FP32 matvec (made on first use)
  cc* tl32 = nullptr;
  cc* ph_up32 = nullptr;
  cc* ph_dn32 = nullptr;
  // coefficients of a batch of R right-hand sides: nb x R x 8 x Q (made on first use)
  void* Cb = nullptr;
  void* Db = nullptr;
  size_t cdb_bytes = 0;
};

struct Timings {
  double fill_ms = 0, rt_ms = 0, tl_ms = 0, setup_ms = 0;
  double mv_total_ms = 0, mv_near_ms = 0, mv_agg_ms = 0, mv_ss_ms = 0, mv_sr_ms = 0,
         mv_rr_ms = 0, mv_recv_ms = 0;
  double gm_passes = 0, gm_steps = 0;  // MGS passes and Arnoldi steps of the last solve
  double graph_replays = 0;            // inner cycles replayed from a CUDA graph, last batched solve
  double precond_ms = 0;               // set-up of the near-field preconditioner (host wall time)
  double lu_factor_ms = 0;             // complex64 tensor-core LU of the mixed direct solve
  double lu_gemm_ms = 0;               // of which its tensor-core trailing updates (CUDA events)
  double lu_gemm_flops = 0;            // complex flops of those updates (8 per multiply-add)
  int lu_gemm_launches = 0;
  double lu_phase_ms[4] = {0, 0, 0, 0};  // panel, row swaps, L11 solve, operand tiling (SIE_LU_PHASES=1)
  int lu_f16 = 0;                      // the last factorisation's trailing updates: 1 split-FP16, 0 3xTF32
  int lu_factorizations = 0;           // factorisations of the last mixed direct solve
};

}  // namespace sie

struct sie_ctx {
  sie_config cfg;
  sie::Material mt;
  sie::Rule R;
  int device = 0;
  cudaStream_t stream = nullptr, stream2 = nullptr;
  cudaStream_t own_stream = nullptr;  // the library's stream when the caller set its own
  cudaEvent_t ev[16];
  // the near-field product runs on stream2 next to the far-field passes
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // near product on stream2: 0 no (sequential), 1 forked at the start of the product,
  // 2 forked once the leaf aggregate is queued, beside the translations only, 3 forked
  // once the SS passes are queued, beside the SR and RR passes
  int overlap_near = 2;

  // mesh (reference order)
  int nv = 0, nt = 0, M = 0;
  std::vector<double> verts;
  std::vector<int> tris;
  std::vector<int> elem, corner;  // 2 per edge (reference order)
  std::vector<double> cent;       // 3 per triangle
  std::vector<sie::FnD> fn_ext;   // 2 per edge, reference order
  std::vector<int> side_v;        // 8 per edge side (p1, p2, pc, tri, triangle's vertices, 0)
  // tree
  double D = 0, xmin[3] = {0, 0, 0};
  int l_min = 0, l_max = 0;
  std::vector<uint64_t> leaf;     // per edge (reference order)
  std::vector<int> perm;          // internal -> reference edge index
  std::vector<int> iperm;         // reference -> internal
  sie::NearLayout near;
  std::vector<sie::Level> lv;     // index = level
  // K and Q of the leaf level (radiation patterns, aggregate, receive); the other levels
  // keep theirs in lv[l].K, lv[l].Q
  int K = 0, Q = 0;
  std::vector<int> level_K;       // requested truncation number per level (0: cfg K)
  bool level_k = false;           // some level's sampling differs from the leaf's
  void* d_lvtmp = nullptr;        // coefficients of one level on its parent's sampling
  size_t lvtmp_bytes = 0;
  bool setup_done = false;
  // SR kernel: 0 one thread per (target box, direction); 1 sibling groups;
  // 2 sibling groups with the translation table staged in shared memory;
  // 3 one warp per sibling group (compacted source lists, prefetched coefficients);
  // 4 the same without branches in the sibling loop (zero TL row for near pairs);
  // 5 present siblings only, TL index linear in the two octants
  int sr_mode = 5;
  // receive: 0 one block per leaf box; 1 chunks of <= 32 edges with pre-combined D
  int recv_mode = 1;
  // aggregate: 0 one thread per (box, direction); 1 eight edge groups per block
  int agg_mode = 1;

  // device arrays
  sie::FnD* d_fn = nullptr;       // internal order
  double* d_rref = nullptr;
  double* d_cent = nullptr;
  int* d_perm = nullptr;
  int* d_box_first = nullptr;     // leaf boxes
  int* d_box_cnt = nullptr;
  int* d_nbr_ptr = nullptr;
  int* d_nbr_box = nullptr;
  int* d_ncols = nullptr;
  long long* d_base = nullptr;
  int* d_edge_box = nullptr;      // leaf box of each internal edge
  int* d_rchunk = nullptr;        // receive chunks: (box, first edge, count, 0) per chunk
  int n_rchunk = 0;
  int ncols_max = 0;              // widest near panel (columns)
  // near product: 0 one warp per row; 1 chunks of rows with the panel's x in shared memory;
  // 2 the same with 4-warp blocks, of which one fits on an SM beside two SR blocks
  int near_mode = 1;
  // near values: ICTF / PMCHWT store (a, b, d), c = cfac * b
  zc* d_na = nullptr;
  zc* d_nb = nullptr;
  zc* d_nd = nullptr;
  zc* d_naT = nullptr;            // transposed panels (adjoint product, made on first use)
  zc* d_nbT = nullptr;
  zc* d_ndT = nullptr;
  cc* d_na32 = nullptr;
  cc* d_nb32 = nullptr;
  cc* d_nd32 = nullptr;
  zc cfac;
  // near-field RAS preconditioner (SIE_PRECOND_NEAR): full 2x2 blocks on the near panels'
  // layout; complex64 copies for the mixed solver's inner products (made on first use)
  int precond = SIE_PRECOND_NONE;
  zc* d_pa = nullptr;
  zc* d_pb = nullptr;
  zc* d_pc = nullptr;
  zc* d_pd = nullptr;
  cc* d_pa32 = nullptr;
  cc* d_pb32 = nullptr;
  cc* d_pc32 = nullptr;
  cc* d_pd32 = nullptr;
  zc* d_diag = nullptr;           // Jacobi diagonal, internal interleaved (J, M)
  // far field
  double* d_khat = nullptr;       // 3 x Q
  double* d_tth = nullptr;
  double* d_tph = nullptr;
  double* d_trf = nullptr;
  int* d_qperm = nullptr;         // direction q' with khat_q' = -khat_q, per direction q
  double* d_boxc = nullptr;       // leaf box centres (3 per leaf box)
  // gradient (made on the first sie_grad call): side vertex ids in internal order, the
  // vertex coordinates, and the workspace
  int* d_side = nullptr;
  double* d_vert = nullptr;
  int* d_tri_verts = nullptr;
  void* d_grad_ws = nullptr;
  size_t grad_ws_bytes = 0;
  int op_adjoint = 0;             // the solver's products apply Z^H (adjoint solve)
  sie_ctx* inner = nullptr;       // operator of the mixed solver's inner products (null: this one)
  zc* d_rt = nullptr;             // internal edge x 4 x Q
  cc* d_rt32 = nullptr;
  float* d_trf32 = nullptr;
  bool f32_ready = false;         // complex64 tables made
  cc* d_xi32 = nullptr;           // FP32 work vectors (internal layout)
  cc* d_yi32 = nullptr;
  cc* d_xb32 = nullptr;           // FP32 vectors of a batched product (b32_rhs of each)
  cc* d_yb32 = nullptr;
  size_t b32_rhs = 0;
  // work vectors (internal layout, interleaved J/M per edge)
  zc* d_xi = nullptr;
  zc* d_yi = nullptr;
  size_t work_rhs = 0;
  // solver workspace
  void* d_gm = nullptr;
  size_t gm_bytes = 0;
  void* d_gm32 = nullptr;         // inner FP32 GMRES workspace (mixed precision)
  size_t gm32_bytes = 0;
  void* d_gmz = nullptr;          // flexible GMRES directions Z (mixed precision)
  size_t gmz_bytes = 0;
  void* d_gmb = nullptr;          // batched mixed-precision solver workspace
  size_t gmb_bytes = 0;
  void* d_io = nullptr;           // staging of the host-buffer entry points (two halves)
  size_t io_bytes = 0;
  void* d_lu = nullptr;           // dense LU factors (column-major N x N, internal order)
  int* d_piv = nullptr;           // pivots (N) + info
  float* d_lu32 = nullptr;        // complex64 LU factors of the mixed direct solve: real plane,
  float* d_lu32i = nullptr;       // imaginary plane (column-major N x N, internal order)
  int* d_piv32 = nullptr;         // and their row interchanges,
  int* d_perm32 = nullptr;        // the same as one permutation (row i of P A is row perm[i] of A)
  cc* d_tmp32 = nullptr;          // work vector of the triangular solves
  char* d_lu_at = nullptr;        // mixed LU workspace: the pre-tiled A and B operands of the
  char* d_lu_bt = nullptr;        // trailing updates,
  void* d_lu_scr = nullptr;       // the panel kernel's slots, barrier counters and error word
  float* d_lu_diag = nullptr;     // the inverses of the factors' diagonal blocks, for the solves
  float* d_lu_minv = nullptr;     // a panel's I - L11^-1 and its blocks' inverses
  char* d_lu_at2 = nullptr;       // the panel's own tensor-core updates: tiled L and U blocks
  void* d_lu_ref = nullptr;       // the refinement's vectors (b, x, Zx, r, the complex64 step, norms)
  void* d_lu_io = nullptr;        // device copies of b and x for the host-buffer direct solve
  size_t lu_io_bytes = 0;
  size_t lu_scr_bytes = 0;
  // the factors above are current (sie_invalidate_factors clears these and keeps the memory,
  // sie_release_factors frees it)
  bool lu64_valid = false;
  bool lu32_valid = false;
  // the mixed LU's trailing updates may run in split-FP16: cleared when the refinement on
  // such factors stalls, after which this context factorises with 3xTF32
  bool lu_f16_ok = true;
  void* h_gm = nullptr;           // pinned host slots for the solver's scalars
  void* h_gmb = nullptr;          // pinned host copy of the batched solver's per-system state
  int ar_blocks = 0;              // co-resident grid of the fused Arnoldi kernel
  unsigned ar_epoch = 1;          // launch counter tagging the Arnoldi exchange rounds
  // Arnoldi step: 0 grid-barrier kernel; 1 register-resident kernel with tagged exchanges;
  // 2 one thread-block cluster (falls back to 1, then 0, when the vector is too long)
  int arnoldi_mode = 2;

  sie::Timings tm;
};

// Functions shared between the translation units of the library.
namespace sie {
int near_fill(sie_ctx* c, int* d_tri_verts);
int near_blocks_list(sie_ctx* c, int* d_tri_verts, const int* d_m, const int* d_n, int cnt,
                     zc* d_out);
int near_matvec64(sie_ctx* c, const zc* x, zc* y, int nrhs, bool accum, cudaStream_t st);
int near_matvec32(sie_ctx* c, const cc* x, cc* y, int nrhs, bool accum, cudaStream_t st);
int near_to_f32(sie_ctx* c);
int near_prepare_kernels(sie_ctx* c);
int far_build_tables(sie_ctx* c, const double* d_boxc);
// far-field passes; wait_recv (may be null) is waited for before the receive adds into y
// after_agg (may be null) is called once the leaf aggregate is queued
int far_matvec64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st, cudaEvent_t* ev,
                 cudaEvent_t wait_recv = nullptr, const std::function<int()>* after_agg = nullptr);
int far_matvec32(sie_ctx* c, const cc* x, cc* y, cudaStream_t st, cudaEvent_t* ev,
                 cudaEvent_t wait_recv = nullptr, const std::function<int()>* after_agg = nullptr);
int far_prepare_kernels(sie_ctx* c);
// Gauss-Legendre nodes and weights on [-1, 1], nodes ascending.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);
// Sparse real matrix in CSR form.
struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
};
// Local Lagrange interpolation (2p x 2p stencil) of a (theta, phi) pattern pair from the
// Kc sampling to the Kp sampling: rows 2 Qp (theta values, then phi), columns 2 Qc.
// With transpose, the anterpolation (its transpose).
int interp_csr(int p, int Kc, int Kp, bool transpose, Csr& out);
// Products of a batch of R right-hand sides (internal layout, vector r at offset r * 2M).
// The near product writes y; the far product adds into it.
int near_matvec_b64(sie_ctx* c, const zc* x, zc* y, int R, cudaStream_t st);
int near_matvec_b32(sie_ctx* c, const cc* x, cc* y, int R, cudaStream_t st);
int far_matvec_b64(sie_ctx* c, const zc* x, zc* y, int R, cudaStream_t st, cudaEvent_t wait_recv = nullptr,
                   const std::function<int()>* after_agg = nullptr);
int far_matvec_b32(sie_ctx* c, const cc* x, cc* y, int R, cudaStream_t st, cudaEvent_t wait_recv = nullptr,
                   const std::function<int()>* after_agg = nullptr);
// transposed products (y = Z^T x, FP64, internal layout): the near one writes y, the far
// one adds into it
int near_matvec_adj64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st);
int far_matvec_adj64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st);
// shape gradient pieces (grad: one double per mesh vertex, accumulated with atomics)
int grad_near(sie_ctx* c, const zc* lam, const zc* I, double h, double* grad, cudaStream_t st);
int grad_far(sie_ctx* c, const zc* lam, const zc* I, double h, double* grad, void* ws, cudaStream_t st);
int grad_rhs(sie_ctx* c, const zc* lam, const double* kin, const double* Ein, double h, double* grad,
             cudaStream_t st);
int field_adjoint_rhs(sie_ctx* c, const zc* E, const double* pts, int npts, zc* g, cudaStream_t st);
int grad_field(sie_ctx* c, const zc* E, const double* pts, int npts, const zc* I, double h, double* grad,
               cudaStream_t st);
// largest batch one launch sequence carries (larger batches go in slices)
static const int SIE_BATCH_MAX = 16;
int ensure_batch32(sie_ctx* c, int nrhs);
// complex64 copies of the near panels, radiation patterns, TL and phase tables
int make_f32_tables(sie_ctx* c);
int to_c64(const zc* in, cc* out, size_t n, cudaStream_t st);
int to_c128(const cc* in, zc* out, size_t n, cudaStream_t st);
int gather_ext_to_int(sie_ctx* c, const zc* ext, zc* in, int nrhs, cudaStream_t st);
int scatter_int_to_ext(sie_ctx* c, const zc* in, zc* ext, int nrhs, cudaStream_t st);
int phase_tables(sie_ctx* c, Level& L, int l, const double* khat_parent, int Qp);
int diag_extract(sie_ctx* c);
// near-field restricted additive Schwarz preconditioner: build, release, y = P x
int ras_build(sie_ctx* c);
void ras_release(sie_ctx* c);
int ras_to_f32(sie_ctx* c);
// R vectors at stride 2M
int ras_apply64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st, int R = 1);
int ras_apply32(sie_ctx* c, const cc* x, cc* y, cudaStream_t st, int R = 1);
int jacobi_apply(sie_ctx* c, const zc* v1, zc* v2, cudaStream_t st);
int rhs_planewave_dev(sie_ctx* c, const double* d_k, const double* d_E, int nrhs, zc* d_b_int);
int farfield_dev(sie_ctx* c, const zc* d_x_int, const double* d_pts, int npts, zc* d_E, zc* d_H,
                 double* d_I);
// the same in the medium mt (wavenumber k1, permeability my1, permittivity eps1)
int farfield_dev(sie_ctx* c, const Material& mt, const zc* d_x_int, const double* d_pts, int npts, zc* d_E,
                 zc* d_H, double* d_I);
int gmres_solve(sie_ctx* c, const zc* d_b, zc* d_x, const sie_solver_cfg* cfg, sie_stats* st);
int fgmres_mixed(sie_ctx* c, const zc* d_b, zc* d_x, const sie_solver_cfg* cfg, sie_stats* st);
// Z^H y = g in place (dense contexts, LU factors made on first use)
int lu_solve_adjoint(sie_ctx* c, zc* d_int);
// R systems with the same matrix solved together (R <= SIE_BATCH_MAX)
int fgmres_mixed_batch(sie_ctx* c, const zc* d_b, zc* d_x, int R, const sie_solver_cfg* cfg,
                       sie_stats* st);
}  // namespace sie

int sie_internal_matvec(sie_ctx* c, const zc* xi, zc* yi, int nrhs, cudaStream_t st, bool timed);
// the same product with complex64 tables and vectors
int sie_internal_matvec32(sie_ctx* c, const cc* xi, cc* yi, cudaStream_t st, bool timed);
// batched products of R vectors (internal layout, stride 2M; sliced by SIE_BATCH_MAX)
int sie_internal_matvec_b(sie_ctx* c, const zc* xi, zc* yi, int R, cudaStream_t st);
// y = Z^H x for one vector (internal layout)
int sie_internal_matvec_adj(sie_ctx* c, const zc* xi, zc* yi, cudaStream_t st);
int sie_internal_matvec_b32(sie_ctx* c, const cc* xi, cc* yi, int R, cudaStream_t st);
