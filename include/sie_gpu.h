/*
 * sie_gpu.h -- C-ABI of the B200 SIE hot path (libsiegpu.so).
 *
 * Drop-in boundary for SpeckleSim's surface-integral-equation matvec path:
 * the RWG near-field impedance fill with Hänninen singularity subtraction and
 * the MLFMM matrix-vector product that GMRES calls.  Every function returns an
 * int status (SIE_OK = 0); sie_last_error() gives the message of the last
 * failure on the calling thread.  Plain pointers and sizes only.
 *
 * Vector layout (all complex vectors): interleaved (re, im) doubles, length 2*N
 * doubles per right-hand side with N = 2*M unknowns; element i < M is the
 * electric coefficient J of RWG edge i and element M + i its magnetic
 * coefficient, edges in the reference's neighbour-scan order
 * (src/lib_sie_tri_calculation_mod.f90:865-905).  Several right-hand sides are
 * stored one after another (column-major N x nrhs).
 *
 * Sign convention: exp(+i w t), Green function exp(-i k R)/(4 pi R)
 * (src/lib_sie_tri_calculation_mod.f90:1421-1432); a lossy body therefore has a
 * NEGATIVE imaginary relative permittivity.
 */
#ifndef SIE_GPU_H
#define SIE_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SIE_OK 0
#define SIE_ERR_ARG 1       /* bad argument (null pointer, size, option) */
#define SIE_ERR_CUDA 2      /* a CUDA call failed or no device */
#define SIE_ERR_STATE 3     /* call order violated (e.g. matvec before setup) */
#define SIE_ERR_NOMEM 4     /* device or host allocation failed */
#define SIE_ERR_MESH 5      /* mesh is not a valid triangle surface */
#define SIE_ERR_NOCONV 6    /* GMRES, or a mixed direct solve's refinement, did not reach the tolerance */
#define SIE_ERR_TIMEOUT 7   /* host-side time limit reached */
#define SIE_ERR_NONFINITE 8 /* NaN/Inf met in an input or a result */

#define SIE_PMCHWT 1
#define SIE_ICTF 3

#define SIE_FP64 0  /* every step in double precision */
#define SIE_MIXED 1 /* FP32 bulk matvec (used by the mixed-precision solver) */

typedef struct sie_ctx sie_ctx;

/* Module globals of the reference set before lib_sie_ml_fmm_precalculation_tri
 * (src/lib_sie_data_container.f90:22-96, main.f90:221-241). */
typedef struct {
  double lambda;                   /* illumination_p%lambda [m] */
  double eps_r1_re, eps_r1_im;     /* background relative permittivity (1, 0) */
  double eps_r2_re, eps_r2_im;     /* body relative permittivity.  As in the reference,
                                      eps_r2_im != 0 keeps the body-medium translations
                                      at the leaf level only: right for metals, far off
                                      for weakly lossy dielectrics (use dense = 1) */
  int formulation;                 /* SIE_ICTF (calc_p(3)=3, default) or SIE_PMCHWT */
  int ngp;                         /* triangle rule points, ng = 3 (1,3,4,6,7,12) */
  int tree_s_opt;                  /* tree_s_opt = 250 */
  int truncation_number;           /* truncation_number_default = 19 */
  int normal_convention;           /* calc_p(7): 1 or 2 */
  int fix_itbn;                    /* 0 reproduces the IT_bn bracket of :2142 */
  int device;                      /* CUDA device ordinal */
  int dense;                       /* 1: no MLFMM, every pair in the near matrix */
} sie_config;

typedef struct {
  int restart;           /* GMRES restart m (reference: restart = max_iterations) */
  int max_iterations;    /* icntl(7) */
  double tolerance;      /* cntl(1): backward-error tolerance */
  int use_initial_guess; /* icntl(6); x holds the guess on entry */
  int precision;         /* SIE_FP64: zgmres semantics on the GPU;
                            SIE_MIXED: FP64 outer FGMRES around an FP32 inner GMRES */
  int inner_restart;     /* SIE_MIXED: inner FP32 GMRES restart */
  double inner_tolerance;/* SIE_MIXED: inner relative residual reduction */
  double time_limit_s;   /* host-side wall limit, 0 = none */
} sie_solver_cfg;

typedef struct {
  int iterations;              /* info(2) (outer iterations for SIE_MIXED) */
  int inner_iterations;        /* SIE_MIXED: total inner iterations */
  int matvecs;                 /* matvec applications (all precisions) */
  int converged;               /* 1 if the backward error reached the tolerance */
  double backward_error_arnoldi; /* last Arnoldi estimate (bea) */
  double backward_error_true;    /* rinfo(2): ||b - Ax|| / ||b|| */
  double seconds;              /* device time of the solve */
} sie_stats;

/* Fill *cfg with the reference defaults (ICTF, ng = 3, s_opt = 250, K = 19). */
void sie_config_default(sie_config* cfg);
void sie_solver_default(sie_solver_cfg* cfg);

const char* sie_last_error(void);
const char* sie_version(void);

/* Replaces data_import_tri + precalculation_fn + the tree constructor
 * (src/lib_sie_tri_mlfmm_interface.f90:59-92 up to lib_sie_constructor_tri).
 * verts: nv x 3 doubles; tris: nt x 3 vertex indices, 0-based. */
int sie_init(const sie_config* cfg, const double* verts, int nv, const int* tris, int nt,
             sie_ctx** out);

/* Truncation number of every MLFMM level, truncation_number(l)%n of the reference
 * (Truncation_number_calculation, src/lib_sie_mlfmm.f90:631-701, which sets
 * truncation_number_default on every level and leaves its per-level rule commented
 * out).  K[l] for levels l = 0 .. n-1 (0: cfg->truncation_number); call between sie_init
 * and sie_setup.  K must not grow from a level to its children.  Where a child level's K
 * is smaller than its parent's, SS interpolates the child's coefficients to the parent's
 * sampling (Lagrange_Interpolation_New, src/lib_sie_mlfmm.f90:268-390, 6 x 6 stencil, the
 * reference's dormant branch at src/lib_sie_tri_mlfmm_interface.f90:486-507) and RR
 * returns by its transpose.  Three departures from that dormant branch, each needed for
 * a correct product: SR weights every level by its own quadrature; RR anterpolates (the
 * reference interpolates, :638-640); the receive takes khat x f at the -z pole in the
 * pole's Cartesian components.  sie_num_directions then gives the leaf level's Q.  The
 * transposed product and sie_grad refuse such contexts (SIE_ERR_STATE). */
int sie_set_level_truncation(sie_ctx* ctx, const int* K, int n);

/* Number of RWG edges M (m_pairs) and the MLFMM levels of the tree. */
int sie_info(const sie_ctx* ctx, int* n_edges, int* l_min, int* l_max, long long* near_nnz);

/* Replaces the rest of lib_sie_ml_fmm_precalculation_tri: near-field CSR fill
 * (precalculation_near_field_csr_tri :779-863), radiation patterns
 * (PreCalculate_RT, lib_sie_tri_mlfmm.f90:503-539), translation tables
 * (precalculation_LT3_TL, lib_sie_mlfmm.f90:27-82) and the Jacobi diagonal
 * (precalculation_diagonal_element :94-109). */
int sie_setup(sie_ctx* ctx);

/* y = Z x for nrhs right-hand sides (host arrays, stride 2M); nrhs > 1 goes through the
 * product in batches of up to 16 vectors that share every read of the tables.  Replaces the matvec
 * callback lib_sie_ml_fmm_calculate_vector_b_tri
 * (src/lib_sie_tri_mlfmm_interface.f90:285-319). */
int sie_matvec(sie_ctx* ctx, const double* x, double* y, int nrhs, int precision);

/* Same on device arrays (no host copies); stream may be NULL. */
int sie_matvec_device(sie_ctx* ctx, const double* d_x, double* d_y, int nrhs, int precision,
                      void* stream);

/* Autotuner: times the product of the given precision on this context's mesh with each
 * kernel variant (near panels, aggregate, SR translation, receive, and where the near
 * product forks beside the far passes), one knob at a time, and keeps the fastest.  All
 * variants compute the same product (to the last bits of summation order).  ms[0], ms[1]
 * (may be NULL): device time of one product before and after; modes[5] (may be NULL): the
 * chosen near, aggregate, SR, receive and fork variants.  No counterpart in the reference. */
int sie_autotune(sie_ctx* ctx, int precision, double* ms, int* modes);

/* Operator of the SIE_MIXED solver's inner complex64 products: another context set up on
 * the same mesh with the same tree (e.g. a lower truncation number, a cheaper
 * preconditioner operator); NULL restores ctx itself.  The outer FP64 products, and so the
 * solution's accuracy, stay those of ctx.  No counterpart in the reference.  The caller
 * keeps `inner` alive while it is linked. */
int sie_set_inner_operator(sie_ctx* ctx, sie_ctx* inner);

/* Conjugate-transpose product y = Z^H x in FP64 for nrhs vectors (stride 2M), the operator
 * of the adjoint solve Z^H lambda = dJ/dI* that a far-field gradient needs.  The reference
 * has no adjoint; this is the exact transpose of the product sie_matvec applies (near
 * panels transposed; far field A^T (pi T pi) R^T with pi the khat -> -khat permutation of
 * the k-space sampling), so <Z^H u, v> = <u, Z v> to rounding. */
int sie_matvec_adjoint(sie_ctx* ctx, const double* x, double* y, int nrhs);
/* Same on device arrays; stream may be NULL. */
int sie_matvec_adjoint_device(sie_ctx* ctx, const double* d_x, double* d_y, int nrhs, void* stream);

/* Shape gradient of the far-field objective J = sum_o |E(r_o)|^2 4 pi |r_o|^2 (the intensity
 * of sie_farfield summed over the npts points pts) with respect to the z coordinate of
 * every mesh vertex, at the solution x of Z x = b for the plane wave (k_in, E_in) of
 * sie_rhs_planewave.  No counterpart in the reference.  It solves the adjoint system
 * Z^H lambda = dJ/dx* with FP64 GMRES (cfg: restart, iterations, tolerance; its stats in
 * *stats) and returns dJ/dz = 2 Re sum_o E_o^H dE_o/dz + 2 Re lambda^H (db/dz - dZ/dz x):
 * the near blocks, radiation patterns and right-hand side are recomputed on the device
 * with each vertex moved by +-1e-6 lambda, the field factors (whose observation points are
 * far away) by +-1e-4 lambda (central differences), the tree and the near/far split held
 * fixed.  dJdz: nv doubles; J (may be NULL): the objective.
 * Returns SIE_ERR_NOCONV (with the gradient filled in) if the adjoint solve stops short. */
int sie_grad(sie_ctx* ctx, const double* x, const double* k_in, const double* E_in, const double* pts,
             int npts, const sie_solver_cfg* cfg, double* dJdz, double* J, sie_stats* stats);

/* Plane-wave right-hand sides, get_vector_b_tri + incident_field_tri_general
 * (src/lib_sie_tri_calculation_mod.f90:391-460, 939-1002).  k_in, E_in: 3 x nrhs. */
int sie_rhs_planewave(sie_ctx* ctx, const double* k_in, const double* E_in, int nrhs, double* b);

/* Incident direction and polarisation as in kin_and_Ein_calculation
 * (src/lib_sie_math.f90:259-293): theta, phi [rad], pol 1 = TM, 2 = TE,
 * k_dir = calc_p(7).  Writes k_in[3], E_in[3]. */
int sie_incidence(double theta, double phi, int pol, int k_dir, double* k_in, double* E_in);

/* The ngp-point triangle rule the fill kernels use, Quadrature_tri
 * (src/lib_sie_integration_points.f90:7-143): barycentric points (alpha, beta) and
 * weights summing to 1, each the binary32 value of the reference's literal.  alpha,
 * beta, w: room for 12 values; *n = ngp.  Host only; no device is needed.  ngp other
 * than 1, 3, 4, 6, 7, 12 gives SIE_ERR_ARG. */
int sie_quadrature_rule(int ngp, double* alpha, double* beta, double* w, int* n);

/* Solve Z x = b for nrhs right-hand sides (stride 2M).  With precision SIE_FP64 each is
 * solved in turn with zgmres semantics; with SIE_MIXED and nrhs > 1 they are solved in
 * batches of up to 16 that advance in lockstep, one batched product per step (restart
 * and inner_restart at most 63 there).  Replaces lib_sie_solver_gmres_run
 * (src/lib_sie_solver_gmres_interface.f90:123-211) and the CERFACS zgmres
 * driver (src/lib/libmath_external/src/algorithm_842/zPackgmres.f90:537-1565). */
int sie_solve(sie_ctx* ctx, const double* b, double* x, int nrhs, const sie_solver_cfg* cfg,
              sie_stats* stats);
int sie_solve_device(sie_ctx* ctx, const double* d_b, double* d_x, int nrhs,
                     const sie_solver_cfg* cfg, sie_stats* stats);

/* Direct solve of the dense system, the reference's normal solver
 * (lib_sie_tri_solver_normal_I, src/lib_sie_tri_solver_normal.f90:64-217, with ZGESV in
 * solver_LU, src/lib_sie_math.f90:649-676).  Needs a context set up with dense = 1; the
 * LU factors are made on the first call and kept for later right-hand sides. */
int sie_solve_direct(sie_ctx* ctx, const double* b, double* x, int nrhs);

/* Mixed-precision direct solve of the dense system (context set up with dense = 1): LU
 * with partial pivoting of the complex64 matrix whose trailing updates run on the tensor
 * cores as split-FP16 products (each operand block scaled by a power of two and split
 * into two FP16 parts, three products accumulated in FP32), then iterative refinement in
 * FP64, x += U^-1 L^-1 P (b - Z x) with the FP64 dense product, until ||b - Z x|| <=
 * tolerance ||b|| or max_refinements corrections.  If a refinement step fails to halve
 * the residual, the matrix is factorised again with 3xTF32 updates (FP32-accurate) and the
 * refinement restarts.  The factors are made on the first call and kept.
 * Same role as sie_solve_direct (ZGESV of the reference's normal solver,
 * src/lib_sie_tri_solver_normal.f90:64-217); the refinement converges while cond(Z)
 * times the FP32 rounding stays below one.  stats (may be NULL): per right-hand side,
 * iterations = refinement steps, backward_error_true = ||b - Z x|| / ||b|| in FP64,
 * seconds = wall time (the first includes the factorisation).  SIE_ERR_NOCONV if the
 * tolerance is not met. */
int sie_solve_direct_mixed(sie_ctx* ctx, const double* b, double* x, int nrhs, double tolerance,
                           int max_refinements, sie_stats* stats);
/* Same on device buffers; the work runs on stream (NULL: the context's stream) and the
 * call returns when the solutions are in d_x. */
int sie_solve_direct_mixed_device(sie_ctx* ctx, const double* d_b, double* d_x, int nrhs, double tolerance,
                                  int max_refinements, sie_stats* stats, void* stream);
/* Frees the LU factors that sie_solve_direct and sie_solve_direct_mixed keep, with their
 * workspace (tiled operands, the solves' vectors and staging buffers), so that the next
 * direct solve factorises again (e.g. after the caller changed nothing but wants the
 * memory back).  No counterpart in the reference, which factorises in every run. */
int sie_release_factors(sie_ctx* ctx);
/* Marks the kept LU factors out of date and keeps their device memory: the next direct
 * solve factorises again into the same buffers, without allocating.  For a caller that
 * refactorises the same context repeatedly; sie_release_factors frees the memory. */
int sie_invalidate_factors(sie_ctx* ctx);

/* Left Jacobi preconditioner, lib_sie_ml_fmm_preconditioner_left
 * (src/lib_sie_tri_mlfmm_interface.f90:323-339): v2 = v1 / diag. */
int sie_precondition_left(sie_ctx* ctx, const double* v1, double* v2);

#define SIE_PRECOND_NONE 0 /* no preconditioner (the reference default, main.f90:232) */
#define SIE_PRECOND_NEAR 1 /* near-field restricted additive Schwarz, applied on the right */

/* Preconditioner of every later sie_solve on ctx.  No counterpart in the reference,
 * whose only option is the left Jacobi scaling of sie_precondition_left (off by
 * default).  SIE_PRECOND_NEAR builds, from the near matrix alone, one local system per
 * leaf box A over A and its neighbour boxes (the near panel's columns), factorises it
 * and keeps the rows of its inverse that belong to A's unknowns: an operator with the
 * near matrix's sparsity, 64 bytes per 2x2 block (complex64 copy for the mixed solver
 * made on first use).  The solvers apply it on the right (Z P u = b, x = P u), so the
 * reported residuals are those of Z x = b.  Set-up costs one LU per leaf box of twice
 * the box's E2 edge count.  Not for dense contexts.  SIE_PRECOND_NONE frees it. */
int sie_set_preconditioner(sie_ctx* ctx, int kind);
/* v2 = P v1 with the preconditioner of sie_set_preconditioner (host vectors). */
int sie_precondition_right(sie_ctx* ctx, const double* v1, double* v2);

/* Scattered E and H at observation points (Integration_scattered_field_tri,
 * src/lib_sie_tri_calculation_mod.f90:2782-2825) and the 'rcs' intensity
 * |E|^2 4 pi |r|^2 (src/lib_sie_tri_solver_normal.f90:325-342).
 * pts: npts x 3; E, H: npts x 3 complex (may be NULL); intensity: npts.
 * As in the reference, E leaves out the electric scalar-potential term (:2815
 * multiplies it by 0), so E is right only in its transverse far-zone part; H keeps
 * every term and is right at any point in the background medium. */
int sie_farfield(sie_ctx* ctx, const double* x, const double* pts, int npts, double* E,
                 double* H, double* intensity);

/* E and H at npts points inside the body, Integration_scattered_field_tri_within_medium
 * (src/lib_sie_tri_calculation_mod.f90:2829-2877): the field that the negated currents
 * radiate into the medium of relative permittivity eps_r (the reference passes the
 * evaluation point's medium, eps_r2 inside the body) with the wavenumber k0 sqrt(eps_r),
 * mu_0 and eps_0 eps_r, the scalar-potential term of E included, on the 3-point rule of
 * sie_farfield.  x: the 2M currents in sie_farfield's layout; E, H: npts x 3 complex
 * (either may be NULL).  It is the total field there; the caller (the reference's
 * lib_sie_tri_observation_field_calculation, src/lib_sie_tri_solver_normal.f90:385-407)
 * adds no incident field to it. */
int sie_field_interior(sie_ctx* ctx, const double* x, const double* pts, int npts, double eps_r_re,
                       double eps_r_im, double* E, double* H);

/* Introspection for parity tests. */
int sie_get_edges(const sie_ctx* ctx, int* elem, int* corner);
int sie_get_tree(const sie_ctx* ctx, double* D_xmin, long long* leaf_box);
/* 2x2 blocks (D11, D12, D21, D22 complex) of arbitrary edge pairs through the
 * fill kernels. */
int sie_get_blocks(sie_ctx* ctx, const int* m, const int* n, int cnt, double* out);
/* Near-field matrix entry (m, n) as stored after sie_setup (0 if not near). */
int sie_get_near_entries(sie_ctx* ctx, const int* m, const int* n, int cnt, double* out);
/* Radiation patterns of edges (4 x Q complex each: med1 theta, med1 phi, med2 theta, med2 phi). */
int sie_get_rt(sie_ctx* ctx, const int* edges, int cnt, double* out);
int sie_num_directions(const sie_ctx* ctx, int* Q);
/* Device-side timings of the last sie_setup / sie_matvec phases [ms]:
 * fill, RT+TL, set-up, matvec total, near, aggregate, SS, SR, RR, receive; then
 * out[10] = mean Gram-Schmidt passes per Arnoldi step of the last solve; out[11] = inner
 * cycles of the last batched mixed solve replayed from their captured CUDA graph;
 * out[12] = set-up of the near-field preconditioner (host wall time); out[13] = the
 * complex64 tensor-core LU of sie_solve_direct_mixed (host wall time), out[14] its
 * tensor-core trailing updates (CUDA events on the launching stream, summed), out[15]
 * their complex flops (8 per complex multiply-add), out[16] their launches; out[17..20]
 * with SIE_LU_PHASES=1 in the environment, the device time of the LU's panels, row swaps,
 * L11 solves and operand tiling; out[21] = 1 if the last factorisation's trailing updates
 * ran in split-FP16, 0 for 3xTF32; out[22] = factorisations in the last mixed direct solve
 * (2 when the split-FP16 factors stalled the refinement and it factorised again). */
int sie_get_timings(const sie_ctx* ctx, double* out, int n);

/* Launch all further work of ctx on the caller's CUDA stream (NULL: back to the
 * library's own stream). */
int sie_set_stream(sie_ctx* ctx, void* stream);

/* Number of kernels this library has launched since it was loaded. */
unsigned long long sie_launch_count(void);

/* Largest mesh (RWG edges) sie_farfield_device_noalloc accepts. */
#define SIE_NOALLOC_MAX_EDGES 131072

/* sie_farfield on device buffers, allocating no device memory.  No counterpart
 * in the reference (its field evaluation, Integration_scattered_field_tri in
 * src/lib_sie_tri_calculation_mod.f90:2782-2825, runs on the host).
 * d_x: 2M complex currents in the sie_farfield layout; d_pts: npts x 3;
 * d_E, d_H: npts x 3 complex; d_I: npts (none may be NULL).  The work is queued
 * on `stream` (NULL: the context's stream) and the call returns without waiting;
 * the outputs are valid once that stream has reached it.
 * Scratch: one library-wide device array of 2 x SIE_NOALLOC_MAX_EDGES complex
 * values per GPU; meshes with more edges get SIE_ERR_ARG.  Calls that may run at
 * the same time on one GPU (other streams, other threads, other contexts) share
 * that array and race: order them on one stream.  The first call on each GPU
 * looks the array up (cudaGetSymbolAddress); make it before any stream capture.
 * The address is kept for the life of the process: after a cudaDeviceReset it is
 * stale, so do not call this entry point again once the device has been reset.
 * The caller's current device is the same after the call as before it. */
int sie_farfield_device_noalloc(sie_ctx* ctx, const double* d_x, const double* d_pts, int npts,
                                double* d_E, double* d_H, double* d_I, void* stream);

int sie_free(sie_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* SIE_GPU_H */
