// Layout conversion, right-hand sides, Jacobi diagonal, translation phases and
// the scattered-field evaluation.
#include <vector>
#include <algorithm>

#include "sie_internal.h"
#include "geom.cuh"

namespace sie {

// reference layout [J_0..J_{M-1}, M_0..M_{M-1}] <-> internal interleaved (J, M)
// per edge in box order
__global__ void k_gather(const zc* ext, zc* in, const int* perm, int M, int nrhs) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)M * nrhs) return;
  int r = (int)(i / M), e = (int)(i % M);
  int s = perm[e];
  const zc* x = ext + (size_t)r * 2 * M;
  zc* o = in + (size_t)r * 2 * M;
  o[2 * e] = x[s];
  o[2 * e + 1] = x[s + M];
}
__global__ void k_scatter(const zc* in, zc* ext, const int* perm, int M, int nrhs) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)M * nrhs) return;
  int r = (int)(i / M), e = (int)(i % M);
  int s = perm[e];
  const zc* x = in + (size_t)r * 2 * M;
  zc* o = ext + (size_t)r * 2 * M;
  o[s] = x[2 * e];
  o[s + M] = x[2 * e + 1];
}

int gather_ext_to_int(sie_ctx* c, const zc* ext, zc* in, int nrhs, cudaStream_t st) {
  long long n = (long long)c->M * nrhs;
  k_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ext, in, c->d_perm, c->M, nrhs); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}
int scatter_int_to_ext(sie_ctx* c, const zc* in, zc* ext, int nrhs, cudaStream_t st) {
  long long n = (long long)c->M * nrhs;
  k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, ext, c->d_perm, c->M, nrhs); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// exp(+/- i k khat.r) for the 8 child octants of a level (r = x_child - x_parent)
__global__ void k_phase(double h, zc k1, zc k2, const double* khat, int Q, zc* up, zc* dn) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int o = blockIdx.y;
  if (q >= Q) return;
  double rx = ((o >> 2) & 1) ? h : -h, ry = ((o >> 1) & 1) ? h : -h, rz = (o & 1) ? h : -h;
  double t = khat[3 * q] * rx + khat[3 * q + 1] * ry + khat[3 * q + 2] * rz;
  for (int md = 0; md < 2; md++) {
    zc k = md == 0 ? k1 : k2;
    // exp(+i k t) = exp(-i (-k) t)
    up[((size_t)o * 2 + md) * Q + q] = cexp_mik(mk<double>(-k.re, -k.im), t);
    dn[((size_t)o * 2 + md) * Q + q] = cexp_mik(k, t);
  }
}

// Shift tables of level l's boxes from and to their parents, on the parent's sampling
// (khat_parent, Qp directions).
int phase_tables(sie_ctx* c, Level& L, int l, const double* khat_parent, int Qp) {
  double h = ldexp(1.0, -(l + 1)) * c->D;
  dim3 g((Qp + 127) / 128, 8);
  k_phase<<<g, 128, 0, c->stream>>>(h, c->mt.k1, c->mt.k2, khat_parent, Qp, L.ph_up, L.ph_dn); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// Jacobi diagonal (precalculation_diagonal_element :94-109): D11, D22 of (m, m)
__global__ void k_diag(const zc* na, const zc* nd, const long long* idx, int M, zc* diag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  diag[2 * i] = na[idx[i]];
  diag[2 * i + 1] = nd[idx[i]];
}

int diag_extract(sie_ctx* c) {
  const NearLayout& N = c->near;
  std::vector<long long> idx(c->M);
  for (int A = 0; A < N.nbox; A++) {
    int col = 0;
    for (int k = N.nbr_ptr[A]; k < N.nbr_ptr[A + 1]; k++) {
      if (N.nbr_box[k] == A) break;
      col += N.box_cnt[N.nbr_box[k]];
    }
    for (int r = 0; r < N.box_cnt[A]; r++)
      idx[N.box_first[A] + r] = N.base[A] + (long long)r * N.ncols[A] + col + r;
  }
  long long* d_idx = nullptr;
  SIE_CUDA(cudaMalloc(&d_idx, idx.size() * sizeof(long long)));
  SIE_CUDA(h2d(d_idx, idx.data(), idx.size() * sizeof(long long)));
  SIE_CUDA(cudaMalloc(&c->d_diag, 2 * (size_t)c->M * sizeof(zc)));
  k_diag<<<(c->M + 255) / 256, 256, 0, c->stream>>>(c->d_na, c->d_nd, d_idx, c->M, c->d_diag); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  SIE_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(d_idx);
  return SIE_OK;
}

// get_vector_b_tri (:391-460) + incident_field_tri_general (:939-1002), plane wave
// Right-hand side of one edge for one plane wave (get_vector_b_tri :391-460): the J and M
// rows, ICTF-scaled.
__device__ __forceinline__ void rhs_edge(const FnD& f0, const FnD& f1, const Rule& R, const Material& mt,
                                         int formulation, vd k, const double E0[3], zc& bJ, zc& bM) {
  zc S1 = mk<double>(0, 0), S2 = S1;
  double hc = mt.my1 * C0;
  for (int ot = 0; ot < 2; ot++) {
    const FnD& f = ot ? f1 : f0;
    for (int j = 0; j < R.n; j++) {
      double w0 = 1 - R.a[j] - R.b[j];
      vd Ra = mkv<double>(w0 * f.c[0] + R.a[j] * f.c[3] + R.b[j] * f.c[6],
                          w0 * f.c[1] + R.a[j] * f.c[4] + R.b[j] * f.c[7],
                          w0 * f.c[2] + R.a[j] * f.c[5] + R.b[j] * f.c[8]);
      vd rfm = (Ra - mkv<double>(f.c[6], f.c[7], f.c[8])) * f.df * 0.5;
      // exp(-i conj(k1) k_in.R)
      zc ph = cexp_mik(conj(mt.k1), dot(k, Ra));
      zc E[3] = {ph * E0[0], ph * E0[1], ph * E0[2]};
      zc H[3] = {(E[2] * k.y - E[1] * k.z) / hc, (E[0] * k.z - E[2] * k.x) / hc,
                 (E[1] * k.x - E[0] * k.y) / hc};
      double wa = R.w[j] * f.area;
      S1 += (E[0] * rfm.x + E[1] * rfm.y + E[2] * rfm.z) * wa;
      S2 += (H[0] * rfm.x + H[1] * rfm.y + H[2] * rfm.z) * wa;
    }
  }
  if (formulation == SIE_ICTF) {
    bJ = S1 / mt.eta_a;
    bM = S2 * mt.eta_a;
  } else {
    bJ = S1;
    bM = S2;
  }
}

__global__ void k_rhs(const FnD* fn, int M, Rule R, Material mt, int formulation, const double* kin,
                      const double* Ein, int nrhs, zc* b) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)M * nrhs) return;
  int r = (int)(i / M), e = (int)(i % M);
  vd k = mkv<double>(kin[3 * r], kin[3 * r + 1], kin[3 * r + 2]);
  double E0[3] = {Ein[3 * r], Ein[3 * r + 1], Ein[3 * r + 2]};
  zc* o = b + (size_t)r * 2 * M;
  rhs_edge(fn[2 * e], fn[2 * e + 1], R, mt, formulation, k, E0, o[2 * e], o[2 * e + 1]);
}

int rhs_planewave_dev(sie_ctx* c, const double* d_k, const double* d_E, int nrhs, zc* d_b_int) {
  long long n = (long long)c->M * nrhs;
  k_rhs<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(c->d_fn, c->M, c->R, c->mt,
                                                            c->cfg.formulation, d_k, d_E, nrhs,
                                                            d_b_int); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// Integration_scattered_field_tri (:2782-2825): E, H at r from all edges with a
// 3-point rule; the E scalar-potential term is multiplied by zero in the
// reference and is left out.  Intensity = |E|^2 4 pi |r|^2 (:325-342).
// One block per observation point.
__global__ void k_field(const FnD* fn, const zc* x, int M, Material mt, const double* pts,
                        int npts, zc* Eo, zc* Ho, double* Io) {
  int p = blockIdx.x;
  if (p >= npts) return;
  const float ra3[3] = {0.16666666666667f, 0.16666666666667f, 0.66666666666667f};
  const float rb3[3] = {0.16666666666667f, 0.66666666666667f, 0.16666666666667f};
  const double w3 = (double)0.33333333333333f;
  vd ra = mkv<double>(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]);
  zc E[3], H[3];
  for (int d = 0; d < 3; d++) E[d] = H[d] = mk<double>(0, 0);
  zc iwm = mk<double>(0, mt.omega * mt.my1);
  zc iwe = mt.eps1 * mk<double>(0, mt.omega);
  zc inv_iwm = mk<double>(1, 0) / iwm;
  for (int e = threadIdx.x; e < M; e += blockDim.x) {
    zc J = x[2 * e], Mm = x[2 * e + 1];
    for (int t = 0; t < 2; t++) {
      const FnD& f = fn[2 * e + t];
      double dfm = f.sgn * f.length;
      for (int i = 0; i < 3; i++) {
        double a = ra3[i], b = rb3[i], w0 = 1 - a - b;
        vd rq = mkv<double>(w0 * f.c[0] + a * f.c[3] + b * f.c[6],
                            w0 * f.c[1] + a * f.c[4] + b * f.c[7],
                            w0 * f.c[2] + a * f.c[5] + b * f.c[8]);
        vd fm = (rq - mkv<double>(f.c[6], f.c[7], f.c[8])) * 0.5 * dfm;
        vd dv = ra - rq;
        double R = vlen(dv);
        zc ex = cexp_mik(mt.k1, R);
        zc ikR = mk<double>(-mt.k1.im * R, mt.k1.re * R);
        zc G = ex * (1.0 / (4 * PI * R));
        zc DG = -((mk<double>(1, 0) + ikR) * ex) * (1.0 / (4 * PI * R * R));
        zc gg[3] = {DG * (dv.x / R), DG * (dv.y / R), DG * (dv.z / R)};
        double fv[3] = {fm.x, fm.y, fm.z};
        zc Mf[3] = {Mm * fv[0], Mm * fv[1], Mm * fv[2]};
        zc cMg[3] = {Mf[1] * gg[2] - Mf[2] * gg[1], Mf[2] * gg[0] - Mf[0] * gg[2],
                     Mf[0] * gg[1] - Mf[1] * gg[0]};
        zc fg[3] = {gg[2] * fv[1] - gg[1] * fv[2], gg[0] * fv[2] - gg[2] * fv[0],
                    gg[1] * fv[0] - gg[0] * fv[1]};
        zc a1 = iwm * J * G;
        zc a2 = iwe * Mm * G;
        zc a3 = inv_iwm * Mm * dfm;
        for (int d = 0; d < 3; d++) {
          E[d] -= (a1 * fv[d] - cMg[d]) * w3;
          H[d] -= (a2 * fv[d] - a3 * gg[d] + J * fg[d]) * w3;
        }
      }
    }
  }
  // block reduction of 12 doubles
  __shared__ double red[32][12];
  double v[12];
  for (int d = 0; d < 3; d++) {
    v[2 * d] = E[d].re;
    v[2 * d + 1] = E[d].im;
    v[6 + 2 * d] = H[d].re;
    v[6 + 2 * d + 1] = H[d].im;
  }
  for (int k = 0; k < 12; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffff, v[k], o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 12; k++) red[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[12] = {0};
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      for (int k = 0; k < 12; k++) s[k] += red[w][k];
    double e2 = 0;
    for (int d = 0; d < 3; d++) {
      Eo[3 * p + d] = mk<double>(s[2 * d], s[2 * d + 1]);
      Ho[3 * p + d] = mk<double>(s[6 + 2 * d], s[6 + 2 * d + 1]);
      e2 += s[2 * d] * s[2 * d] + s[2 * d + 1] * s[2 * d + 1];
    }
    double r2 = ra.x * ra.x + ra.y * ra.y + ra.z * ra.z;
    Io[p] = e2 * 4 * PI * r2;
  }
}

int farfield_dev(sie_ctx* c, const Material& mt, const zc* d_x_int, const double* d_pts, int npts, zc* d_E,
                 zc* d_H, double* d_I) {
  k_field<<<npts, 256, 0, c->stream>>>(c->d_fn, d_x_int, c->M, mt, d_pts, npts, d_E, d_H, d_I); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}
int farfield_dev(sie_ctx* c, const zc* d_x_int, const double* d_pts, int npts, zc* d_E, zc* d_H,
                 double* d_I) {
  return farfield_dev(c, c->mt, d_x_int, d_pts, npts, d_E, d_H, d_I);
}

__global__ void k_z2c(const zc* a, cc* b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = mk<float>((float)a[i].re, (float)a[i].im);
}
__global__ void k_c2z(const cc* a, zc* b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = mk<double>((double)a[i].re, (double)a[i].im);
}

int to_c64(const zc* in, cc* out, size_t n, cudaStream_t st) {
  unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_z2c<<<std::max(g, 1u), 256, 0, st>>>(in, out, n); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}
int to_c128(const cc* in, zc* out, size_t n, cudaStream_t st) {
  unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_c2z<<<std::max(g, 1u), 256, 0, st>>>(in, out, n); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

__global__ void k_jacobi(const zc* v1, const zc* diag, int n, zc* v2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v2[i] = v1[i] / diag[i];
}

int jacobi_apply(sie_ctx* c, const zc* v1, zc* v2, cudaStream_t st) {
  int n = 2 * c->M;
  k_jacobi<<<(n + 255) / 256, 256, 0, st>>>(v1, c->d_diag, n, v2); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}


// ---------------------------------------------------------------------------
// Far-field objective J = sum_o w_o |E(r_o)|^2, w_o = 4 pi |r_o|^2 (the intensity of
// k_field), and the pieces of its shape gradient that live on single edges.

// E(r_o) = sum_e FJ_e J_e + FM_e M_e: the per-edge field factors of k_field
// (Integration_scattered_field_tri :2782-2825, the scalar-potential term multiplied by 0).
__device__ __forceinline__ void field_factors(const FnD& f0, const FnD& f1, vd ra, const Material& mt, zc FJ[3],
                                              zc FM[3]) {
  const float ra3[3] = {0.16666666666667f, 0.16666666666667f, 0.66666666666667f};
  const float rb3[3] = {0.16666666666667f, 0.66666666666667f, 0.16666666666667f};
  const double w3 = (double)0.33333333333333f;
  const zc iwm = mk<double>(0, mt.omega * mt.my1);
  for (int d = 0; d < 3; d++) FJ[d] = FM[d] = mk<double>(0, 0);
  for (int t = 0; t < 2; t++) {
    const FnD& f = t ? f1 : f0;
    double dfm = f.sgn * f.length;
    for (int i = 0; i < 3; i++) {
      double a = ra3[i], b = rb3[i], w0 = 1 - a - b;
      vd rq = mkv<double>(w0 * f.c[0] + a * f.c[3] + b * f.c[6], w0 * f.c[1] + a * f.c[4] + b * f.c[7],
                          w0 * f.c[2] + a * f.c[5] + b * f.c[8]);
      vd fm = (rq - mkv<double>(f.c[6], f.c[7], f.c[8])) * 0.5 * dfm;
      vd dv = ra - rq;
      double R = vlen(dv);
      zc ex = cexp_mik(mt.k1, R);
      zc ikR = mk<double>(-mt.k1.im * R, mt.k1.re * R);
      zc G = ex * (1.0 / (4 * PI * R));
      zc DG = -((mk<double>(1, 0) + ikR) * ex) * (1.0 / (4 * PI * R * R));
      zc gg[3] = {DG * (dv.x / R), DG * (dv.y / R), DG * (dv.z / R)};
      double fv[3] = {fm.x, fm.y, fm.z};
      zc fxg[3] = {fv[1] * gg[2] - fv[2] * gg[1], fv[2] * gg[0] - fv[0] * gg[2], fv[0] * gg[1] - fv[1] * gg[0]};
      zc a1 = iwm * G;
      for (int d = 0; d < 3; d++) {
        FJ[d] -= a1 * fv[d] * w3;
        FM[d] += fxg[d] * w3;
      }
    }
  }
}

// g = dJ/dI* = sum_o w_o F_o^H E_o, the right-hand side of the adjoint solve (internal layout).
__global__ void k_field_adjoint_rhs(const FnD* fn, int M, Material mt, const zc* E, const double* pts, int npts,
                                    zc* g) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M) return;
  zc gJ = mk<double>(0, 0), gM = gJ;
  for (int o = 0; o < npts; o++) {
    const vd ra = mkv<double>(pts[3 * o], pts[3 * o + 1], pts[3 * o + 2]);
    const double w = 4 * PI * dot(ra, ra);
    zc FJ[3], FM[3];
    field_factors(fn[2 * e], fn[2 * e + 1], ra, mt, FJ, FM);
    for (int d = 0; d < 3; d++) {
      gJ += conj(FJ[d]) * E[3 * o + d] * w;
      gM += conj(FM[d]) * E[3 * o + d] * w;
    }
  }
  g[2 * e] = gJ;
  g[2 * e + 1] = gM;
}

// Explicit term 2 Re sum_o w_o E_o^H dF_o I per (edge, vertex slot), central differences.
__global__ void k_grad_field(const SideV* sv, const FnD* fn, const double* V, int normal_convention, double h,
                             int M, Material mt, const zc* E, const double* pts, int npts, const zc* I,
                             double* grad) {
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= 4LL * M) return;
  const int e = (int)(it >> 2), slot = (int)(it & 3);
  const int v = edge_vertex(sv, e, slot);
  FnD fp[2], fmn[2];
  for (int ll = 0; ll < 2; ll++) {
    fp[ll] = side_fn(sv[2 * e + ll], fn[2 * e + ll].sgn, V, normal_convention, v, h);
    fmn[ll] = side_fn(sv[2 * e + ll], fn[2 * e + ll].sgn, V, normal_convention, v, -h);
  }
  const zc iJ = I[2 * e], iM = I[2 * e + 1];
  const double inv = 0.5 / h;
  zc acc = mk<double>(0, 0);
  for (int o = 0; o < npts; o++) {
    const vd ra = mkv<double>(pts[3 * o], pts[3 * o + 1], pts[3 * o + 2]);
    const double w = 4 * PI * dot(ra, ra);
    zc FJp[3], FMp[3], FJm[3], FMm[3];
    field_factors(fp[0], fp[1], ra, mt, FJp, FMp);
    field_factors(fmn[0], fmn[1], ra, mt, FJm, FMm);
    for (int d = 0; d < 3; d++)
      acc += conj(E[3 * o + d]) * (((FJp[d] - FJm[d]) * iJ + (FMp[d] - FMm[d]) * iM) * (inv * w));
  }
  atomicAdd(grad + v, 2.0 * acc.re);
}

// 2 Re(lambda^H db) per (edge, vertex slot), central differences of the plane-wave rows.
__global__ void k_grad_rhs(const SideV* sv, const FnD* fn, const double* V, int normal_convention, double h,
                           int M, Rule R, Material mt, int formulation, const double* kin, const double* Ein,
                           const zc* lam, double* grad) {
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= 4LL * M) return;
  const int e = (int)(it >> 2), slot = (int)(it & 3);
  const int v = edge_vertex(sv, e, slot);
  const vd k = mkv<double>(kin[0], kin[1], kin[2]);
  const double E0[3] = {Ein[0], Ein[1], Ein[2]};
  zc bp[2], bm[2];
  FnD f0 = side_fn(sv[2 * e], fn[2 * e].sgn, V, normal_convention, v, h);
  FnD f1 = side_fn(sv[2 * e + 1], fn[2 * e + 1].sgn, V, normal_convention, v, h);
  rhs_edge(f0, f1, R, mt, formulation, k, E0, bp[0], bp[1]);
  f0 = side_fn(sv[2 * e], fn[2 * e].sgn, V, normal_convention, v, -h);
  f1 = side_fn(sv[2 * e + 1], fn[2 * e + 1].sgn, V, normal_convention, v, -h);
  rhs_edge(f0, f1, R, mt, formulation, k, E0, bm[0], bm[1]);
  const double inv = 0.5 / h;
  const zc val = conj(lam[2 * e]) * ((bp[0] - bm[0]) * inv) + conj(lam[2 * e + 1]) * ((bp[1] - bm[1]) * inv);
  atomicAdd(grad + v, 2.0 * val.re);
}

int field_adjoint_rhs(sie_ctx* c, const zc* E, const double* pts, int npts, zc* g, cudaStream_t st) {
  k_field_adjoint_rhs<<<(c->M + 127) / 128, 128, 0, st>>>(c->d_fn, c->M, c->mt, E, pts, npts, g);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int grad_field(sie_ctx* c, const zc* E, const double* pts, int npts, const zc* I, double h, double* grad,
               cudaStream_t st) {
  const long long n = 4LL * c->M;
  k_grad_field<<<(unsigned)((n + 127) / 128), 128, 0, st>>>((const SideV*)c->d_side, c->d_fn, c->d_vert,
                                                            c->cfg.normal_convention, h, c->M, c->mt, E, pts,
                                                            npts, I, grad);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int grad_rhs(sie_ctx* c, const zc* lam, const double* kin, const double* Ein, double h, double* grad,
             cudaStream_t st) {
  const long long n = 4LL * c->M;
  k_grad_rhs<<<(unsigned)((n + 127) / 128), 128, 0, st>>>((const SideV*)c->d_side, c->d_fn, c->d_vert,
                                                          c->cfg.normal_convention, h, c->M, c->R, c->mt,
                                                          c->cfg.formulation, kin, Ein, lam, grad);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

}  // namespace sie

using namespace sie;

extern "C" int sie_precondition_left(sie_ctx* c, const double* v1, double* v2) {
  if (!c || !v1 || !v2) return fail(SIE_ERR_ARG, "sie_precondition_left: null argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_precondition_left: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  size_t bytes = (size_t)2 * c->M * sizeof(zc);
  zc *d1 = nullptr, *d2 = nullptr, *e1 = nullptr;
  SIE_CUDA(cudaMalloc(&d1, bytes));
  SIE_CUDA(cudaMalloc(&d2, bytes));
  SIE_CUDA(cudaMalloc(&e1, bytes));
  SIE_CUDA(h2d(e1, v1, bytes));
  int r = gather_ext_to_int(c, e1, d1, 1, c->stream);
  if (r == SIE_OK) r = jacobi_apply(c, d1, d2, c->stream);
  if (r == SIE_OK) r = scatter_int_to_ext(c, d2, e1, 1, c->stream);
  if (r == SIE_OK) {
    cudaStreamSynchronize(c->stream);
    if (cudaMemcpy(v2, e1, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
      r = fail(SIE_ERR_CUDA, "sie_precondition_left: copy");
  }
  cudaFree(d1);
  cudaFree(d2);
  cudaFree(e1);
  return r;
}
