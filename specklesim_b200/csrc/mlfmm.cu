// MLFMM far field on the GPU: radiation patterns, translation tables and the
// level-synchronous upward / downward / receive passes.
//
// Reference: the plug-ins of src/lib_sie_tri_mlfmm_interface.f90 (get_C
// :395-448, translation_SS :466-528, translation_SR :547-586, translation_RR
// :600-655, get_v_y_j :690-751), MLFMM_tri_summation_New and PreCalculate_RT in
// src/lib_sie_tri_mlfmm.f90 (:416-583), TL_km_ml_fmm in src/lib_sie_mlfmm.f90
// (:129-188) and the pass order of src/lib/libmlfmm/lib/lib_ml_fmm.f90 (:269-1110).
//
// Coefficient layout per box: 8 items x Q directions, item order
//   0,1 = theta J (k1,k2)   2,3 = theta M (k1,k2)
//   4,5 = phi   J (k1,k2)   6,7 = phi   M (k1,k2)
// (a_nm(1..4), b_nm(1..4) of lib_ml_fmm_coefficient).  Medium = item & 1.
#include <algorithm>
#include <type_traits>

#include "sie_internal.h"
#include "geom.cuh"

namespace sie {

// ---------------------------------------------------------------------------
// Radiation pattern per edge about the centre of its leaf box
// (RT_function_SCSArr_New :543-583): for every direction q and medium,
//   sum_sides sum_j 0.5*sign*len*(r_j - v) exp(-i k khat.(r_j - Rc)) w_j
// projected on theta-hat (a_nm) and phi-hat (b_nm).
// Radiation pattern of one edge in one direction: medium 1 theta, phi, medium 2 theta, phi.
__device__ __forceinline__ void rt_edge_q(const FnD& f0, const FnD& f1, vd Rc, vd kh, vd th, vd ph,
                                          const Rule& R, zc k1, zc k2, zc out[4]) {
  zc a1 = mk<double>(0, 0), b1 = a1, a2 = a1, b2 = a1;
  for (int ll = 0; ll < 2; ll++) {
    const FnD& f = ll ? f1 : f0;
    double dfm = f.sgn * f.length;
    zc sa[3] = {mk<double>(0, 0), mk<double>(0, 0), mk<double>(0, 0)};
    zc sb[3] = {sa[0], sa[0], sa[0]};
    for (int j = 0; j < R.n; j++) {
      double w0 = 1 - R.a[j] - R.b[j];
      vd Ro = mkv<double>(w0 * f.c[0] + R.a[j] * f.c[3] + R.b[j] * f.c[6],
                          w0 * f.c[1] + R.a[j] * f.c[4] + R.b[j] * f.c[7],
                          w0 * f.c[2] + R.a[j] * f.c[5] + R.b[j] * f.c[8]);
      vd fm = (Ro - mkv<double>(f.c[6], f.c[7], f.c[8])) * 0.5 * dfm;
      double tmp = dot(kh, Ro - Rc);
      zc e1 = cexp_mik(k1, tmp) * R.w[j];
      zc e2 = cexp_mik(k2, tmp) * R.w[j];
      sa[0] += e1 * fm.x;
      sa[1] += e1 * fm.y;
      sa[2] += e1 * fm.z;
      sb[0] += e2 * fm.x;
      sb[1] += e2 * fm.y;
      sb[2] += e2 * fm.z;
    }
    a1 += sa[0] * th.x + sa[1] * th.y + sa[2] * th.z;
    b1 += sa[0] * ph.x + sa[1] * ph.y + sa[2] * ph.z;
    a2 += sb[0] * th.x + sb[1] * th.y + sb[2] * th.z;
    b2 += sb[0] * ph.x + sb[1] * ph.y + sb[2] * ph.z;
  }
  out[0] = a1;
  out[1] = b1;
  out[2] = a2;
  out[3] = b2;
}

__global__ void k_rt(const FnD* fn, const double* boxc, const int* edge_box, int M, Rule R,
                     zc k1, zc k2, const double* khat, const double* tth, const double* tph, int Q,
                     zc* rt, int e0) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int e = e0 + blockIdx.y;
  if (q >= Q || e >= M) return;
  int b = edge_box[e];
  vd Rc = mkv<double>(boxc[3 * b], boxc[3 * b + 1], boxc[3 * b + 2]);
  vd kh = mkv<double>(khat[3 * q], khat[3 * q + 1], khat[3 * q + 2]);
  vd th = mkv<double>(tth[3 * q], tth[3 * q + 1], tth[3 * q + 2]);
  vd ph = mkv<double>(tph[3 * q], tph[3 * q + 1], tph[3 * q + 2]);
  zc o4[4];
  rt_edge_q(fn[2 * e], fn[2 * e + 1], Rc, kh, th, ph, R, k1, k2, o4);
  zc* o = rt + (size_t)e * 4 * Q;
  o[0 * Q + q] = o4[0];
  o[1 * Q + q] = o4[1];
  o[2 * Q + q] = o4[2];
  o[3 * Q + q] = o4[3];
}

// ---------------------------------------------------------------------------
// Spherical Hankel functions of the second kind for every TL offset and medium
// (lib_math_hankel_spherical_2 = j - i y, lib_math_bessel.f90:935-990).
// Real argument: j_n by Miller's downward recurrence, y_n upward.  Complex
// argument: h2 by upward recurrence from h2_{-1} = e^{-iz}/z, h2_0 = i e^{-iz}/z.
__device__ void hankel2_dev(zc z, int K, zc* h) {
  if (z.im == 0.0) {
    double x = z.re;
    double sx, cxv;
    sincos(x, &sx, &cxv);
    double ym1 = -cxv / x, y0 = ym1;
    double y1 = -cxv / (x * x) - sx / x;
    // y_n upward
    double yp = y0, yc = y1;
    h[0].im = -y0;
    if (K > 1) h[1].im = -y1;
    for (int n = 1; n + 1 < K; n++) {
      double yn = (2 * n + 1) / x * yc - yp;
      yp = yc;
      yc = yn;
      h[n + 1].im = -yn;
    }
    // j_n downward (Miller), normalised on j0 or j1
    int start = K + 20;
    int s2 = (int)fabs(x) + 40;
    if (s2 > start) start = s2;
    double jn1 = 0.0, jn = 1e-300;
    double j0v = sx / x, j1v = sx / (x * x) - cxv / x;
    // first pass: find scale, storing the values of orders < K as we go
    double store[64];
    for (int n = start; n >= 1; n--) {
      double jm = (2 * n + 1) / x * jn - jn1;
      jn1 = jn;
      jn = jm;
      if (fabs(jn) > 1e250) {
        jn *= 1e-250;
        jn1 *= 1e-250;
        for (int k = 0; k < K && k < 64; k++) store[k] *= 1e-250;
      }
      if (n - 1 < K) store[n - 1] = jn;
      if (n < K) store[n] = jn1;
    }
    double sc = (fabs(j0v) >= fabs(j1v)) ? j0v / store[0] : j1v / store[1];
    for (int n = 0; n < K; n++) h[n].re = store[n] * sc;
    return;
  }
  zc mi = mk<double>(0.0, -1.0);
  zc e = cexp(mi * z);
  zc hm1 = e / z;
  zc h0 = mk<double>(0.0, 1.0) * e / z;
  h[0] = h0;
  zc prev = hm1, cur = h0;
  for (int n = 0; n + 1 < K; n++) {
    zc nx = (mk<double>((double)(2 * n + 1), 0.0) / z) * cur - prev;
    prev = cur;
    cur = nx;
    h[n + 1] = cur;
  }
}

__global__ void k_hankel(double xmin, double dx, zc k1, zc k2, int K, bool only_k1, zc* hk) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 343) return;
  int i = t / 49, j = (t / 7) % 7, k = t % 7;
  vd r = mkv<double>(xmin + i * dx, xmin + j * dx, xmin + k * dx);
  double rl = vlen(r);
  zc hb[64];
  for (int md = 0; md < 2; md++) {
    zc* o = hk + ((size_t)t * 2 + md) * K;
    bool excluded = (i >= 2 && i <= 4 && j >= 2 && j <= 4 && k >= 2 && k <= 4);
    if (excluded || (md == 1 && only_k1)) {
      for (int n = 0; n < K; n++) o[n] = mk<double>(0, 0);
      continue;
    }
    zc kk = md == 0 ? k1 : k2;
    hankel2_dev(kk * rl, K, hb);
    for (int n = 0; n < K; n++) o[n] = hb[n];
  }
}

// TL_km_ml_fmm (lib_sie_mlfmm.f90:129-188):
//   TL(q) = sum_{n=1..K} h2_{n-1}(kR) (-i)^n (2n-1) P_{n-1}(rhat.khat_q) k / (4 pi)^2
__global__ void k_tl(double xmin, double dx, const zc* hk, zc k1, zc k2, int K, int Q,
                     const double* khat, zc* tl) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int t = blockIdx.y;
  if (q >= Q) return;
  int i = t / 49, j = (t / 7) % 7, k = t % 7;
  vd r = mkv<double>(xmin + i * dx, xmin + j * dx, xmin + k * dx);
  double rl = vlen(r);
  vd rh = r / rl;
  double x = rh.x * khat[3 * q] + rh.y * khat[3 * q + 1] + rh.z * khat[3 * q + 2];
  const double c16 = (4 * PI) * (4 * PI);
  for (int md = 0; md < 2; md++) {
    const zc* h = hk + ((size_t)t * 2 + md) * K;
    zc kd = md == 0 ? k1 : k2;
    zc acc = mk<double>(0, 0);
    double p0 = 1.0, p1 = x;
    zc mi = mk<double>(1.0, 0.0);
    for (int n = 1; n <= K; n++) {
      double P = (n == 1) ? p0 : (n == 2 ? p1 : 0.0);
      if (n >= 3) {
        int nn = n - 2;  // P_{nn+1} from P_nn, P_{nn-1}
        double p2 = ((2 * nn + 1) * x * p1 - nn * p0) / (nn + 1);
        p0 = p1;
        p1 = p2;
        P = p1;
      }
      mi = mi * mk<double>(0.0, -1.0);
      acc += ((h[n - 1] * mi) * (double)(2 * (n - 1) + 1)) * P * kd / c16;
    }
    tl[((size_t)t * 2 + md) * Q + q] = acc;
  }
}

// ---------------------------------------------------------------------------
// Upward pass step 1 (lib_sie_ml_fmm_get_C :395-448): C = sum conj(RT) x over
// the edges of each leaf box.  Block per leaf box, threads over directions.
template <typename T>
__global__ void __launch_bounds__(128) k_aggregate(const cx<T>* __restrict__ rt,
                                                   const int* box_first, const int* box_cnt,
                                                   int Q, const cx<T>* __restrict__ x,
                                                   cx<T>* __restrict__ C) {
  int b = blockIdx.y;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  int f = box_first[b], cnt = box_cnt[b];
  cx<T> acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = mk<T>(0, 0);
#pragma unroll 2
  for (int e = f; e < f + cnt; e++) {
    const cx<T>* r = rt + (size_t)e * 4 * Q;
    cx<T> xe = x[2 * e], xh = x[2 * e + 1];
    cx<T> ra1 = r[q], rb1 = r[Q + q], ra2 = r[2 * Q + q], rb2 = r[3 * Q + q];
    acc[0] = cfma_conj(ra1, xe, acc[0]);
    acc[1] = cfma_conj(ra2, xe, acc[1]);
    acc[2] = cfma_conj(ra1, xh, acc[2]);
    acc[3] = cfma_conj(ra2, xh, acc[3]);
    acc[4] = cfma_conj(rb1, xe, acc[4]);
    acc[5] = cfma_conj(rb2, xe, acc[5]);
    acc[6] = cfma_conj(rb1, xh, acc[6]);
    acc[7] = cfma_conj(rb2, xh, acc[7]);
  }
  cx<T>* o = C + (size_t)b * 8 * Q;
#pragma unroll
  for (int i = 0; i < 8; i++) o[i * Q + q] = acc[i];
}

// Same sum with a block per (leaf box, 32 directions): the 8 warps take every 8th edge
// of the box, so each box's radiation patterns stream through 8 independent load
// chains; the partial sums meet in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) k_aggregate_eg(const cx<T>* __restrict__ rt,
                                                      const int* box_first, const int* box_cnt,
                                                      int Q, const cx<T>* __restrict__ x,
                                                      cx<T>* __restrict__ C) {
  __shared__ cx<T> red[8][8][33];
  const int b = blockIdx.y;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x * 32 + lane;
  const bool qok = q < Q;
  const unsigned long long pol = l2_evict_first_policy();
  const int f = box_first[b], cnt = box_cnt[b];
  cx<T> acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = mk<T>(0, 0);
  if (qok) {
#pragma unroll 2
    for (int e = f + w; e < f + cnt; e += 8) {
      const cx<T>* r = rt + (size_t)e * 4 * Q + q;
      cx<T> xe = x[2 * e], xh = x[2 * e + 1];
      cx<T> ra1 = ld_stream(r, pol), rb1 = ld_stream(r + Q, pol), ra2 = ld_stream(r + 2 * Q, pol),
            rb2 = ld_stream(r + 3 * Q, pol);
      acc[0] = cfma_conj(ra1, xe, acc[0]);
      acc[1] = cfma_conj(ra2, xe, acc[1]);
      acc[2] = cfma_conj(ra1, xh, acc[2]);
      acc[3] = cfma_conj(ra2, xh, acc[3]);
      acc[4] = cfma_conj(rb1, xe, acc[4]);
      acc[5] = cfma_conj(rb2, xe, acc[5]);
      acc[6] = cfma_conj(rb1, xh, acc[6]);
      acc[7] = cfma_conj(rb2, xh, acc[7]);
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) red[w][i][lane] = acc[i];
  __syncthreads();
  // warp w now owns item w
  cx<T> s = red[0][w][lane];
#pragma unroll
  for (int k = 1; k < 8; k++) s += red[k][w][lane];
  if (qok) C[((size_t)b * 8 + w) * Q + q] = s;
}

// Upward pass step 2 (translation_SS :466-528): parent C = sum over children
// of C_child * exp(+i k khat.(x_child - x_parent)).  nmed = 1 skips medium 2.
template <typename T>
__global__ void k_ss(const cx<T>* __restrict__ Cc, const int* ch_ptr, const int* ch_idx,
                     const int* ch_oct, const cx<T>* __restrict__ ph, int Q, int nmed,
                     cx<T>* __restrict__ Cp) {
  int b = blockIdx.y;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  cx<T> acc[8];
  for (int i = 0; i < 8; i++) acc[i] = mk<T>(0, 0);
  for (int k = ch_ptr[b]; k < ch_ptr[b + 1]; k++) {
    int c = ch_idx[k], o = ch_oct[k];
    const cx<T>* src = Cc + (size_t)c * 8 * Q;
    for (int md = 0; md < nmed; md++) {
      cx<T> p = ph[((size_t)o * 2 + md) * Q + q];
      for (int it = md; it < 8; it += 2) acc[it] = cfma(src[it * Q + q], p, acc[it]);
    }
  }
  cx<T>* out = Cp + (size_t)b * 8 * Q;
  for (int i = 0; i < 8; i++) out[i * Q + q] = acc[i];
}

// Downward pass step 1 (translation_SR :547-586 over lib_tree_get_domain_i4):
// D~ = sum_{I4} C_src * TRF * TL(x_box - x_src).
template <typename T>
__global__ void k_sr(const cx<T>* __restrict__ C, const int* i4_ptr, const int* i4_src,
                     const int* i4_off, const cx<T>* __restrict__ tl, const T* __restrict__ trf,
                     int Q, int nmed, cx<T>* __restrict__ D) {
  int b = blockIdx.y;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  cx<T> acc[8];
  for (int i = 0; i < 8; i++) acc[i] = mk<T>(0, 0);
  T w = trf[q];
  for (int k = i4_ptr[b]; k < i4_ptr[b + 1]; k++) {
    int s = i4_src[k], t = i4_off[k];
    const cx<T>* src = C + (size_t)s * 8 * Q;
    for (int md = 0; md < nmed; md++) {
      cx<T> f = tl[((size_t)t * 2 + md) * Q + q] * w;
      for (int it = md; it < 8; it += 2) acc[it] = cfma(src[it * Q + q], f, acc[it]);
    }
  }
  cx<T>* out = D + (size_t)b * 8 * Q;
  for (int i = 0; i < 8; i++) out[i * Q + q] = acc[i];
}

// The same translation organised by sibling groups: the 8 children of one parent
// P share the candidate sources, the (up to) 216 children of the 27 boxes around
// P; a source is in I4 of sibling o exactly when their offset has a component of
// magnitude >= 2.  Every source coefficient is read once per group instead of once
// per target.  One thread per (group, direction); NI items of medium md per pass.
template <typename T, int NI>
__global__ void __launch_bounds__(128) k_sr_group(const cx<T>* __restrict__ C,
                                                  const int* __restrict__ grp_sib,
                                                  const int* __restrict__ grp_src,
                                                  const cx<T>* __restrict__ tl,
                                                  const T* __restrict__ trf, int Q, int md,
                                                  int item0, int zero_other,
                                                  cx<T>* __restrict__ D) {
  __shared__ int s_sib[8];
  __shared__ int s_src[216];
  int g = blockIdx.y;
  for (int i = threadIdx.x; i < 216; i += blockDim.x) s_src[i] = grp_src[(size_t)g * 216 + i];
  if (threadIdx.x < 8) s_sib[threadIdx.x] = grp_sib[(size_t)g * 8 + threadIdx.x];
  __syncthreads();
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  cx<T> acc[8][NI];
#pragma unroll
  for (int o = 0; o < 8; o++)
#pragma unroll
    for (int i = 0; i < NI; i++) acc[o][i] = mk<T>(0, 0);
  const cx<T>* tlq = tl + (size_t)md * Q + q;  // + t * 2 * Q
  for (int d = 0; d < 27; d++) {
    int dx = d / 9 - 1, dy = (d / 3) % 3 - 1, dz = d % 3 - 1;
    for (int c = 0; c < 8; c++) {
      int s = s_src[d * 8 + c];
      if (s < 0) continue;
      const cx<T>* src = C + (size_t)s * 8 * Q + q;
      cx<T> cs[NI];
#pragma unroll
      for (int i = 0; i < NI; i++) cs[i] = src[(size_t)(md + 2 * (item0 + i)) * Q];
      int bx = (c >> 2) & 1, by = (c >> 1) & 1, bz = c & 1;
#pragma unroll
      for (int o = 0; o < 8; o++) {
        if (s_sib[o] < 0) continue;
        int ox = ((o >> 2) & 1) - bx - 2 * dx;
        int oy = ((o >> 1) & 1) - by - 2 * dy;
        int oz = (o & 1) - bz - 2 * dz;
        if (ox > -2 && ox < 2 && oy > -2 && oy < 2 && oz > -2 && oz < 2) continue;
        int t = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
        cx<T> f = tlq[(size_t)t * 2 * Q];
#pragma unroll
        for (int i = 0; i < NI; i++) acc[o][i] = cfma(cs[i], f, acc[o][i]);
      }
    }
  }
  T w = trf[q];
#pragma unroll
  for (int o = 0; o < 8; o++) {
    int b = s_sib[o];
    if (b < 0) continue;
    cx<T>* out = D + (size_t)b * 8 * Q + q;
#pragma unroll
    for (int i = 0; i < NI; i++) out[(size_t)(md + 2 * (item0 + i)) * Q] = acc[o][i] * w;
    if (zero_other) {
#pragma unroll
      for (int i = 0; i < NI; i++) out[(size_t)((1 - md) + 2 * (item0 + i)) * Q] = mk<T>(0, 0);
    }
  }
}

// Sibling-group SR with the translation table of a tile of SR_TQ directions staged in
// shared memory (343 offsets x SR_TQ), so each (source, sibling) pair costs one
// shared-memory read of TL instead of an L2 read.  Block = SR_GB groups x SR_TQ
// directions; all four items of medium md in one pass.
#define SR_TQ 16
#define SR_GB 8
template <typename T>
__global__ void __launch_bounds__(SR_TQ* SR_GB) k_sr_group_tl(
    const cx<T>* __restrict__ C, const int* __restrict__ grp_sib, const int* __restrict__ grp_src,
    int ngrp, const cx<T>* __restrict__ tl, const T* __restrict__ trf, int Q, int md,
    int zero_other, cx<T>* __restrict__ D) {
  extern __shared__ unsigned char smraw[];
  cx<T>* sTL = reinterpret_cast<cx<T>*>(smraw);                  // [343][SR_TQ]
  int* s_src = reinterpret_cast<int*>(sTL + 343 * SR_TQ);         // [SR_GB][216]
  int* s_sib = s_src + SR_GB * 216;                               // [SR_GB][8]
  int q0 = blockIdx.x * SR_TQ;
  int g0 = blockIdx.y * SR_GB;
  int tid = threadIdx.x;
  for (int i = tid; i < 343 * SR_TQ; i += blockDim.x) {
    int t = i / SR_TQ, j = i - t * SR_TQ;
    int q = q0 + j;
    sTL[i] = (q < Q) ? tl[((size_t)t * 2 + md) * Q + q] : mk<T>(0, 0);
  }
  for (int i = tid; i < SR_GB * 216; i += blockDim.x) {
    int g = g0 + i / 216;
    s_src[i] = (g < ngrp) ? grp_src[(size_t)g * 216 + (i % 216)] : -1;
  }
  for (int i = tid; i < SR_GB * 8; i += blockDim.x) {
    int g = g0 + i / 8;
    s_sib[i] = (g < ngrp) ? grp_sib[(size_t)g * 8 + (i % 8)] : -1;
  }
  __syncthreads();
  int gi = tid / SR_TQ, qi = tid - gi * SR_TQ;
  int q = q0 + qi;
  if (q >= Q || g0 + gi >= ngrp) return;
  const int* src_l = s_src + gi * 216;
  const int* sib_l = s_sib + gi * 8;
  cx<T> acc[8][4];
#pragma unroll
  for (int o = 0; o < 8; o++)
#pragma unroll
    for (int i = 0; i < 4; i++) acc[o][i] = mk<T>(0, 0);
  for (int d = 0; d < 27; d++) {
    int dx = d / 9 - 1, dy = (d / 3) % 3 - 1, dz = d % 3 - 1;
    for (int c = 0; c < 8; c++) {
      int s = src_l[d * 8 + c];
      if (s < 0) continue;
      const cx<T>* src = C + (size_t)s * 8 * Q + q;
      cx<T> cs[4];
#pragma unroll
      for (int i = 0; i < 4; i++) cs[i] = src[(size_t)(md + 2 * i) * Q];
      int bx = (c >> 2) & 1, by = (c >> 1) & 1, bz = c & 1;
#pragma unroll
      for (int o = 0; o < 8; o++) {
        if (sib_l[o] < 0) continue;
        int ox = ((o >> 2) & 1) - bx - 2 * dx;
        int oy = ((o >> 1) & 1) - by - 2 * dy;
        int oz = (o & 1) - bz - 2 * dz;
        if (ox > -2 && ox < 2 && oy > -2 && oy < 2 && oz > -2 && oz < 2) continue;
        int t = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
        cx<T> f = sTL[t * SR_TQ + qi];
#pragma unroll
        for (int i = 0; i < 4; i++) acc[o][i] = cfma(cs[i], f, acc[o][i]);
      }
    }
  }
  T w = trf[q];
#pragma unroll
  for (int o = 0; o < 8; o++) {
    int b = sib_l[o];
    if (b < 0) continue;
    cx<T>* out = D + (size_t)b * 8 * Q + q;
#pragma unroll
    for (int i = 0; i < 4; i++) out[(size_t)(md + 2 * i) * Q] = acc[o][i] * w;
    if (zero_other) {
#pragma unroll
      for (int i = 0; i < 4; i++) out[(size_t)((1 - md) + 2 * i) * Q] = mk<T>(0, 0);
    }
  }
}

// Sibling-group SR, one warp per group.  A warp covers SRW_QT directions x 2 item
// halves of one sibling group, so every branch on the group's data is warp-uniform.
// Per block: the TL tile of SRW_QT directions (343 offsets) and the offset table
// (216 source slots x 8 siblings -> TL index, -1 inside the near zone) sit in shared
// memory; each warp compacts its group's present sources into a list and streams the
// two coefficients of its item half for the next source while it applies the current
// one to the 8 siblings.
#define SRW_QT 16
#define SRW_GB 8
template <typename T>
__global__ void __launch_bounds__(32 * SRW_GB, 2) k_sr_warp(
    const cx<T>* __restrict__ C, const int* __restrict__ grp_sib, const int* __restrict__ grp_src,
    int ngrp, const cx<T>* __restrict__ tl, const T* __restrict__ trf, int Q, int md,
    int zero_other, cx<T>* __restrict__ D) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sTL = reinterpret_cast<cx<T>*>(smraw);                         // [343][SRW_QT]
  short* s_tix = reinterpret_cast<short*>(sTL + 343 * SRW_QT);          // [216][8]
  int* s_list = reinterpret_cast<int*>(s_tix + 216 * 8);                // [SRW_GB][216]
  const int q0 = blockIdx.x * SRW_QT;
  const int tid = threadIdx.x;
  for (int i = tid; i < 343 * SRW_QT; i += blockDim.x) {
    int t = i / SRW_QT, j = i - t * SRW_QT;
    int q = q0 + j;
    sTL[i] = (q < Q) ? tl[((size_t)t * 2 + md) * Q + q] : mk<T>(0, 0);
  }
  for (int i = tid; i < 216 * 8; i += blockDim.x) {
    int dc = i >> 3, o = i & 7;
    int d = dc >> 3, c = dc & 7;
    int ox = ((o >> 2) & 1) - ((c >> 2) & 1) - 2 * (d / 9 - 1);
    int oy = ((o >> 1) & 1) - ((c >> 1) & 1) - 2 * ((d / 3) % 3 - 1);
    int oz = (o & 1) - (c & 1) - 2 * (d % 3 - 1);
    bool nearz = ox > -2 && ox < 2 && oy > -2 && oy < 2 && oz > -2 && oz < 2;
    s_tix[i] = nearz ? (short)-1 : (short)((ox + 3) * 49 + (oy + 3) * 7 + (oz + 3));
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  const int g = blockIdx.y * SRW_GB + w;
  if (g >= ngrp) return;
  // sibling boxes (lanes 0..7) and their presence mask
  int sib = (lane < 8) ? grp_sib[(size_t)g * 8 + lane] : -1;
  const unsigned smask = __ballot_sync(0xffffffffu, sib >= 0) & 0xffu;
  // compact list of present sources: (box << 8) | slot
  int* lst = s_list + w * 216;
  int cnt = 0;
  for (int base = 0; base < 216; base += 32) {
    int dc = base + lane;
    int s = (dc < 216) ? grp_src[(size_t)g * 216 + dc] : -1;
    unsigned bal = __ballot_sync(0xffffffffu, s >= 0);
    if (s >= 0) lst[cnt + __popc(bal & ((1u << lane) - 1u))] = (s << 8) | dc;
    cnt += __popc(bal);
  }
  __syncwarp();
  const int ih = lane >> 4, qi = lane & 15;
  const int q = q0 + qi;
  const bool qok = q < Q;
  const cx<T>* Cq = C + (qok ? q : 0);
  const int it0 = md + 4 * ih, it1 = it0 + 2;
  cx<T> acc[8][2];
#pragma unroll
  for (int o = 0; o < 8; o++) acc[o][0] = acc[o][1] = mk<T>(0, 0);
  if (cnt > 0) {
    int e = lst[0];
    size_t sb = (size_t)(e >> 8) * 8;
    cx<T> n0 = Cq[(sb + it0) * Q], n1 = Cq[(sb + it1) * Q];
    for (int i = 0; i < cnt; i++) {
      const cx<T> c0 = n0, c1 = n1;
      const int dc = e & 255;
      if (i + 1 < cnt) {
        e = lst[i + 1];
        sb = (size_t)(e >> 8) * 8;
        n0 = Cq[(sb + it0) * Q];
        n1 = Cq[(sb + it1) * Q];
      }
      const int4 tv = *reinterpret_cast<const int4*>(s_tix + dc * 8);
      const int tw[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
      for (int o = 0; o < 8; o++) {
        int t = (o & 1) ? (tw[o >> 1] >> 16) : (int)(short)(tw[o >> 1] & 0xffff);
        if (t >= 0 && ((smask >> o) & 1u)) {
          cx<T> f = sTL[t * SRW_QT + qi];
          acc[o][0] = cfma(c0, f, acc[o][0]);
          acc[o][1] = cfma(c1, f, acc[o][1]);
        }
      }
    }
  }
  const T wq = trf[qok ? q : 0];
#pragma unroll
  for (int o = 0; o < 8; o++) {
    int b = __shfl_sync(0xffffffffu, sib, o);
    if (b < 0 || !qok) continue;
    cx<T>* out = D + (size_t)b * 8 * Q + q;
    out[(size_t)it0 * Q] = acc[o][0] * wq;
    out[(size_t)it1 * Q] = acc[o][1] * wq;
    if (zero_other) {
      out[(size_t)(it0 ^ 1) * Q] = mk<T>(0, 0);
      out[(size_t)(it1 ^ 1) * Q] = mk<T>(0, 0);
    }
  }
}

template <typename T>
static size_t sr_warp_smem() {
  return (size_t)343 * SRW_QT * sizeof(cx<T>) + (size_t)216 * 8 * sizeof(short) +
         (size_t)SRW_GB * 216 * sizeof(int);
}

// Branch-free form of k_sr_warp.  The TL tile gets a zero row (index 343) that every
// pair inside the near zone points to, and absent siblings accumulate into registers
// that are never stored, so the loop over the 8 siblings has no branches: its 8 TL
// reads and 16 complex FMAs can all be in flight together.  Source slots inside the
// parent itself (all siblings, all near) are dropped when the list is compacted.
template <typename T>
__global__ void __launch_bounds__(32 * SRW_GB, 2) k_sr_warp_bf(
    const cx<T>* __restrict__ C, const int* __restrict__ grp_sib, const int* __restrict__ grp_src,
    int ngrp, const cx<T>* __restrict__ tl, const T* __restrict__ trf, int Q, int md,
    int zero_other, cx<T>* __restrict__ D) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sTL = reinterpret_cast<cx<T>*>(smraw);                         // [344][SRW_QT]
  short* s_tix = reinterpret_cast<short*>(sTL + 344 * SRW_QT);          // [216][8]
  int* s_list = reinterpret_cast<int*>(s_tix + 216 * 8);                // [SRW_GB][216]
  const int q0 = blockIdx.x * SRW_QT;
  const int tid = threadIdx.x;
  for (int i = tid; i < 344 * SRW_QT; i += blockDim.x) {
    int t = i / SRW_QT, j = i - t * SRW_QT;
    int q = q0 + j;
    sTL[i] = (t < 343 && q < Q) ? tl[((size_t)t * 2 + md) * Q + q] : mk<T>(0, 0);
  }
  for (int i = tid; i < 216 * 8; i += blockDim.x) {
    int dc = i >> 3, o = i & 7;
    int d = dc >> 3, c = dc & 7;
    int ox = ((o >> 2) & 1) - ((c >> 2) & 1) - 2 * (d / 9 - 1);
    int oy = ((o >> 1) & 1) - ((c >> 1) & 1) - 2 * ((d / 3) % 3 - 1);
    int oz = (o & 1) - (c & 1) - 2 * (d % 3 - 1);
    bool nearz = ox > -2 && ox < 2 && oy > -2 && oy < 2 && oz > -2 && oz < 2;
    s_tix[i] = nearz ? (short)343 : (short)((ox + 3) * 49 + (oy + 3) * 7 + (oz + 3));
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  const int g = blockIdx.y * SRW_GB + w;
  if (g >= ngrp) return;
  int sib = (lane < 8) ? grp_sib[(size_t)g * 8 + lane] : -1;
  int* lst = s_list + w * 216;
  int cnt = 0;
  for (int base = 0; base < 216; base += 32) {
    int dc = base + lane;
    int s = (dc < 216 && (dc >> 3) != 13) ? grp_src[(size_t)g * 216 + dc] : -1;
    unsigned bal = __ballot_sync(0xffffffffu, s >= 0);
    if (s >= 0) lst[cnt + __popc(bal & ((1u << lane) - 1u))] = (s << 8) | dc;
    cnt += __popc(bal);
  }
  __syncwarp();
  const int ih = lane >> 4, qi = lane & 15;
  const int q = q0 + qi;
  const bool qok = q < Q;
  const cx<T>* Cq = C + (qok ? q : 0);
  const int it0 = md + 4 * ih, it1 = it0 + 2;
  cx<T> acc[8][2];
#pragma unroll
  for (int o = 0; o < 8; o++) acc[o][0] = acc[o][1] = mk<T>(0, 0);
  if (cnt > 0) {
    int e = lst[0];
    size_t sb = (size_t)(e >> 8) * 8;
    cx<T> n0 = Cq[(sb + it0) * Q], n1 = Cq[(sb + it1) * Q];
    for (int i = 0; i < cnt; i++) {
      const cx<T> c0 = n0, c1 = n1;
      const int dc = e & 255;
      if (i + 1 < cnt) {
        e = lst[i + 1];
        sb = (size_t)(e >> 8) * 8;
        n0 = Cq[(sb + it0) * Q];
        n1 = Cq[(sb + it1) * Q];
      }
      const int4 tv = *reinterpret_cast<const int4*>(s_tix + dc * 8);
      const int tw[4] = {tv.x, tv.y, tv.z, tv.w};
      cx<T> f[8];
#pragma unroll
      for (int o = 0; o < 8; o++) {
        int t = (o & 1) ? (tw[o >> 1] >> 16) : (tw[o >> 1] & 0xffff);
        f[o] = sTL[t * SRW_QT + qi];
      }
#pragma unroll
      for (int o = 0; o < 8; o++) {
        acc[o][0] = cfma(c0, f[o], acc[o][0]);
        acc[o][1] = cfma(c1, f[o], acc[o][1]);
      }
    }
  }
  const T wq = trf[qok ? q : 0];
#pragma unroll
  for (int o = 0; o < 8; o++) {
    int b = __shfl_sync(0xffffffffu, sib, o);
    if (b < 0 || !qok) continue;
    cx<T>* out = D + (size_t)b * 8 * Q + q;
    out[(size_t)it0 * Q] = acc[o][0] * wq;
    out[(size_t)it1 * Q] = acc[o][1] * wq;
    if (zero_other) {
      out[(size_t)(it0 ^ 1) * Q] = mk<T>(0, 0);
      out[(size_t)(it1 ^ 1) * Q] = mk<T>(0, 0);
    }
  }
}

// Sibling-group SR over the present siblings only.  The TL offset index is linear in the
// two octants: t = T0(source slot) + off(target octant), with
//   T0 = (3 - c_x - 2 d_x) 49 + (3 - c_y - 2 d_y) 7 + (3 - c_z - 2 d_z),
//   off = o_x 49 + o_y 7 + o_z,
// and TL is exactly zero on the 27 near offsets (they are excluded when TL is built), so
// the loop over the NS present siblings needs neither a table nor a branch.  NS is a
// template parameter; each warp dispatches on its group's sibling count.
// HINT (FP64 only): bit 1 streams the D stores (evict-first), bit 2 loads the source
// coefficients with an evict-last L2 policy.  D is read once later, while each level's C
// is re-read by up to 27 groups; without the hints, the D writes push C out of L2.
template <typename T, int NS, int PD, int HINT = 0>
__device__ __forceinline__ void sr_ns_body(const int* lst, int cnt, const cx<T>* Cq, int it0, int it1,
                                           const cx<T>* sTL, int qi, const int* sibc, const int* offc,
                                           bool qok, T wq, int Q, int q, int zero_other,
                                           cx<T>* __restrict__ D) {
  unsigned long long pol = 0;
  if constexpr ((HINT & 2) != 0) pol = l2_evict_last_policy();
  (void)pol;
  int off[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) off[k] = offc[k] * SRW_QT + qi;
  cx<T> acc[NS][2];
#pragma unroll
  for (int k = 0; k < NS; k++) acc[k][0] = acc[k][1] = mk<T>(0, 0);
  // coefficients of the next PD sources stay in flight in registers
  cx<T> p0[PD], p1[PD];
#pragma unroll
  for (int d = 0; d < PD; d++) {
    if (d < cnt) {
      size_t sb = (size_t)(lst[d] >> 9) * 8;
      if constexpr (HINT & 2) {
        p0[d] = ld_keep(Cq + (sb + it0) * Q, pol);
        p1[d] = ld_keep(Cq + (sb + it1) * Q, pol);
      } else {
        p0[d] = Cq[(sb + it0) * Q];
        p1[d] = Cq[(sb + it1) * Q];
      }
    }
  }
  for (int i = 0; i < cnt; i++) {
    const cx<T> c0 = p0[0], c1 = p1[0];
    const int t0 = (lst[i] & 511) * SRW_QT;
#pragma unroll
    for (int d = 0; d + 1 < PD; d++) {
      p0[d] = p0[d + 1];
      p1[d] = p1[d + 1];
    }
    if (i + PD < cnt) {
      size_t sb = (size_t)(lst[i + PD] >> 9) * 8;
      if constexpr (HINT & 2) {
        p0[PD - 1] = ld_keep(Cq + (sb + it0) * Q, pol);
        p1[PD - 1] = ld_keep(Cq + (sb + it1) * Q, pol);
      } else {
        p0[PD - 1] = Cq[(sb + it0) * Q];
        p1[PD - 1] = Cq[(sb + it1) * Q];
      }
    }
    cx<T> f[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) f[k] = sTL[t0 + off[k]];
#pragma unroll
    for (int k = 0; k < NS; k++) {
      acc[k][0] = cfma(c0, f[k], acc[k][0]);
      acc[k][1] = cfma(c1, f[k], acc[k][1]);
    }
  }
  if (!qok) return;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    cx<T>* out = D + (size_t)sibc[k] * 8 * Q + q;
    if constexpr (HINT & 1) {
      st_stream(out + (size_t)it0 * Q, acc[k][0] * wq);
      st_stream(out + (size_t)it1 * Q, acc[k][1] * wq);
      if (zero_other) {
        st_stream(out + (size_t)(it0 ^ 1) * Q, mk<T>(0, 0));
        st_stream(out + (size_t)(it1 ^ 1) * Q, mk<T>(0, 0));
      }
    } else {
      out[(size_t)it0 * Q] = acc[k][0] * wq;
      out[(size_t)it1 * Q] = acc[k][1] * wq;
      if (zero_other) {
        out[(size_t)(it0 ^ 1) * Q] = mk<T>(0, 0);
        out[(size_t)(it1 ^ 1) * Q] = mk<T>(0, 0);
      }
    }
  }
}

template <typename T, int PD, int HINT = 0>
__global__ void __launch_bounds__(32 * SRW_GB, 2) k_sr_warp_ns(
    const cx<T>* __restrict__ C, const int* __restrict__ grp_sib, const int* __restrict__ grp_src,
    int ngrp, const cx<T>* __restrict__ tl, const T* __restrict__ trf, int Q, int md,
    int zero_other, cx<T>* __restrict__ D) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sTL = reinterpret_cast<cx<T>*>(smraw);                  // [343][SRW_QT]
  int* s_list = reinterpret_cast<int*>(sTL + 343 * SRW_QT);      // [SRW_GB][216]
  int* s_sib = s_list + SRW_GB * 216;                            // [SRW_GB][8] present boxes
  int* s_off = s_sib + SRW_GB * 8;                               // [SRW_GB][8] their octant offsets
  const int q0 = blockIdx.x * SRW_QT;
  const int tid = threadIdx.x;
  for (int i = tid; i < 343 * SRW_QT; i += blockDim.x) {
    int t = i / SRW_QT, j = i - t * SRW_QT;
    int q = q0 + j;
    sTL[i] = (q < Q) ? tl[((size_t)t * 2 + md) * Q + q] : mk<T>(0, 0);
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  const int g = blockIdx.y * SRW_GB + w;
  if (g >= ngrp) return;
  // present siblings, compacted in octant order
  int sib = (lane < 8) ? grp_sib[(size_t)g * 8 + lane] : -1;
  const unsigned smask = __ballot_sync(0xffffffffu, sib >= 0) & 0xffu;
  const int ns = __popc(smask);
  if (sib >= 0) {
    int k = __popc(smask & ((1u << lane) - 1u));
    s_sib[w * 8 + k] = sib;
    s_off[w * 8 + k] = ((lane >> 2) & 1) * 49 + ((lane >> 1) & 1) * 7 + (lane & 1);
  }
  // present sources outside the parent itself: (box << 9) | T0
  int* lst = s_list + w * 216;
  int cnt = 0;
  for (int base = 0; base < 216; base += 32) {
    int dc = base + lane;
    int d = dc >> 3, c = dc & 7;
    int s = (dc < 216 && d != 13) ? grp_src[(size_t)g * 216 + dc] : -1;
    unsigned bal = __ballot_sync(0xffffffffu, s >= 0);
    if (s >= 0) {
      int t0 = (3 - ((c >> 2) & 1) - 2 * (d / 9 - 1)) * 49 + (3 - ((c >> 1) & 1) - 2 * ((d / 3) % 3 - 1)) * 7 +
               (3 - (c & 1) - 2 * (d % 3 - 1));
      lst[cnt + __popc(bal & ((1u << lane) - 1u))] = (s << 9) | t0;
    }
    cnt += __popc(bal);
  }
  __syncwarp();
  const int ih = lane >> 4, qi = lane & 15;
  const int q = q0 + qi;
  const bool qok = q < Q;
  const cx<T>* Cq = C + (qok ? q : 0);
  const int it0 = md + 4 * ih, it1 = it0 + 2;
  const T wq = trf[qok ? q : 0];
  const int* sibc = s_sib + w * 8;
  const int* offc = s_off + w * 8;
  switch (ns) {
    case 1: sr_ns_body<T, 1, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 2: sr_ns_body<T, 2, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 3: sr_ns_body<T, 3, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 4: sr_ns_body<T, 4, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 5: sr_ns_body<T, 5, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 6: sr_ns_body<T, 6, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 7: sr_ns_body<T, 7, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    case 8: sr_ns_body<T, 8, PD, HINT>(lst, cnt, Cq, it0, it1, sTL, qi, sibc, offc, qok, wq, Q, q, zero_other, D); break;
    default: break;
  }
}

template <typename T>
static size_t sr_warp_ns_smem() {
  return (size_t)343 * SRW_QT * sizeof(cx<T>) + (size_t)SRW_GB * (216 + 16) * sizeof(int);
}


template <typename T>
static size_t sr_warp_bf_smem() {
  return (size_t)344 * SRW_QT * sizeof(cx<T>) + (size_t)216 * 8 * sizeof(short) +
         (size_t)SRW_GB * 216 * sizeof(int);
}

// Downward pass step 2 (translation_RR :600-655): D += D_parent * exp(-i k khat.(x_child - x_parent)).
template <typename T>
__global__ void k_rr(const cx<T>* __restrict__ Dp, const int* parent, const int* oct,
                     const cx<T>* __restrict__ ph, int Q, int nmed, cx<T>* __restrict__ D) {
  int b = blockIdx.y;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  int p = parent[b];
  if (p < 0) return;
  int o = oct[b];
  const cx<T>* src = Dp + (size_t)p * 8 * Q;
  cx<T>* dst = D + (size_t)b * 8 * Q;
  for (int md = 0; md < nmed; md++) {
    cx<T> f = ph[((size_t)o * 2 + md) * Q + q];
    for (int it = md; it < 8; it += 2) dst[it * Q + q] = cfma(src[it * Q + q], f, dst[it * Q + q]);
  }
}

// Final summation far part (get_v_y_j :690-751 + MLFMM_tri_summation_New
// :416-497).  Block per leaf box; D of the box in shared memory; one warp per
// edge reduces over the directions.
struct RecvConst {
  zc kd[2], my_d[2], eps_d[2];
  zc s1f, s2f;  // ICTF scaling of the two outputs
  // The receive rotates the pattern, f_rk = (-f_phi, f_theta) = khat x f.  At the -z pole
  // (the last direction) the stored components are Cartesian (theta-hat = x, phi-hat =
  // y), for which khat x f = (f_y, -f_x): the k terms change sign.  With one K on every
  // level D is zero there (TRF is 0 at the poles) and the reference's formula is kept
  // (pole_fix = 0); anterpolated D is not zero, and per-level truncation sets it.
  int pole_fix;
};
// the k factor of direction q in the receive
__device__ __forceinline__ zc recv_kd(const RecvConst& rc, int md, int q, int Q) {
  return (rc.pole_fix && q == Q - 1) ? -rc.kd[md] : rc.kd[md];
}

template <typename T>
__global__ void k_receive(const cx<T>* __restrict__ rt, const int* box_first, const int* box_cnt,
                          const cx<T>* __restrict__ D, int Q, RecvConst rc,
                          cx<T>* __restrict__ y) {
  extern __shared__ unsigned char smraw[];
  cx<T>* sD = reinterpret_cast<cx<T>*>(smraw);
  int b = blockIdx.x;
  const cx<T>* Db = D + (size_t)b * 8 * Q;
  for (int i = threadIdx.x; i < 8 * Q; i += blockDim.x) sD[i] = Db[i];
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int f = box_first[b], cnt = box_cnt[b];
  for (int e = f + warp; e < f + cnt; e += nw) {
    const cx<T>* r = rt + (size_t)e * 4 * Q;
    // per medium: Sa = sum(fa D_i + fb D_{4+i}), Sb = sum(fb D_i - fa D_{4+i}),
    //             Sc = sum(fa D_{2+i} + fb D_{6+i}), Sd = sum(fa D_{6+i} - fb D_{2+i})
    cx<T> S[2][4];
    for (int md = 0; md < 2; md++)
      for (int k = 0; k < 4; k++) S[md][k] = mk<T>(0, 0);
#pragma unroll 3
    for (int q = lane; q < Q; q += 32) {
      const T sg = (rc.pole_fix && q == Q - 1) ? (T)-1 : (T)1;  // k terms at the -z pole
#pragma unroll
      for (int md = 0; md < 2; md++) {
        cx<T> fa = r[(2 * md) * Q + q], fb = r[(2 * md + 1) * Q + q];
        cx<T> dJt = sD[(0 + md) * Q + q], dMt = sD[(2 + md) * Q + q];
        cx<T> dJp = sD[(4 + md) * Q + q], dMp = sD[(6 + md) * Q + q];
        S[md][0] = cfma(fa, dJt, S[md][0]);
        S[md][0] = cfma(fb, dJp, S[md][0]);
        S[md][1] = cfma(fb * sg, dJt, S[md][1]);
        S[md][1] = cfma(-fa * sg, dJp, S[md][1]);
        S[md][2] = cfma(fa, dMt, S[md][2]);
        S[md][2] = cfma(fb, dMp, S[md][2]);
        S[md][3] = cfma(fa * sg, dMp, S[md][3]);
        S[md][3] = cfma(-fb * sg, dMt, S[md][3]);
      }
    }
    for (int md = 0; md < 2; md++)
      for (int k = 0; k < 4; k++)
        for (int o = 16; o > 0; o >>= 1) {
          S[md][k].re += __shfl_xor_sync(0xffffffff, S[md][k].re, o);
          S[md][k].im += __shfl_xor_sync(0xffffffff, S[md][k].im, o);
        }
    if (lane == 0) {
      zc s1 = mk<double>(0, 0), s2 = s1;
      for (int md = 0; md < 2; md++) {
        zc Sa = mk<double>(S[md][0].re, S[md][0].im), Sb = mk<double>(S[md][1].re, S[md][1].im);
        zc Sc = mk<double>(S[md][2].re, S[md][2].im), Sd = mk<double>(S[md][3].re, S[md][3].im);
        s1 += rc.kd[md] * Sd + rc.my_d[md] * Sa;
        s2 += rc.kd[md] * Sb + rc.eps_d[md] * Sc;
      }
      s1 = s1 * rc.s1f;
      s2 = s2 * rc.s2f;
      y[2 * e] += mk<T>((T)s1.re, (T)s1.im);
      y[2 * e + 1] += mk<T>((T)s2.re, (T)s2.im);
    }
  }
}

// Receive over work chunks of at most 32 edges of one leaf box.  The eight D items of
// the box are first folded, per medium, into the four vectors the two outputs need:
//   s1 = sum_q fa (my D_Jt + kd D_Mp) + fb (my D_Jp - kd D_Mt)
//   s2 = sum_q fa (eps D_Mt - kd D_Jp) + fb (kd D_Jt + eps D_Mp)
// (the same sums as k_receive, regrouped), scaled by the formulation factors.  Each warp
// then streams the radiation patterns of two edges at a time against them.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_receive_chunk(const cx<T>* __restrict__ rt,
                                                          const int4* __restrict__ chunks,
                                                          const cx<T>* __restrict__ D, int Q,
                                                          RecvConst rc, cx<T>* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sU = reinterpret_cast<cx<T>*>(smraw);  // [md][A1, B1, A2, B2][Q]
  const int4 ch = chunks[blockIdx.x];
  const int b = ch.x, f = ch.y, cnt = ch.z;
  const cx<T>* Db = D + (size_t)b * 8 * Q;
  for (int q = threadIdx.x; q < Q; q += blockDim.x) {
#pragma unroll
    for (int md = 0; md < 2; md++) {
      zc dJt = cvt_z(Db[(0 + md) * Q + q]), dMt = cvt_z(Db[(2 + md) * Q + q]);
      zc dJp = cvt_z(Db[(4 + md) * Q + q]), dMp = cvt_z(Db[(6 + md) * Q + q]);
      const zc kd = recv_kd(rc, md, q, Q);
      zc A1 = (rc.my_d[md] * dJt + kd * dMp) * rc.s1f;
      zc B1 = (rc.my_d[md] * dJp - kd * dMt) * rc.s1f;
      zc A2 = (rc.eps_d[md] * dMt - kd * dJp) * rc.s2f;
      zc B2 = (kd * dJt + rc.eps_d[md] * dMp) * rc.s2f;
      cx<T>* u = sU + (size_t)md * 4 * Q + q;
      u[0] = mk<T>((T)A1.re, (T)A1.im);
      u[Q] = mk<T>((T)B1.re, (T)B1.im);
      u[2 * Q] = mk<T>((T)A2.re, (T)A2.im);
      u[3 * Q] = mk<T>((T)B2.re, (T)B2.im);
    }
  }
  __syncthreads();
  const unsigned long long pol = l2_evict_first_policy();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e0 = f + 2 * warp; e0 < f + cnt; e0 += 16) {
    const bool two = e0 + 1 < f + cnt;
    const cx<T>* r0 = rt + (size_t)e0 * 4 * Q;
    const cx<T>* r1 = two ? r0 + 4 * Q : r0;
    cx<T> s[2][2];
    s[0][0] = s[0][1] = s[1][0] = s[1][1] = mk<T>(0, 0);
#pragma unroll 2
    for (int q = lane; q < Q; q += 32) {
      cx<T> u[8];
#pragma unroll
      for (int k = 0; k < 8; k++) u[k] = sU[k * Q + q];
      cx<T> a0[4], a1[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        a0[k] = ld_stream(r0 + k * Q + q, pol);
        a1[k] = ld_stream(r1 + k * Q + q, pol);
      }
#pragma unroll
      for (int md = 0; md < 2; md++) {
        // rows of RT: 2 md = theta (fa), 2 md + 1 = phi (fb)
        s[0][0] = cfma(a0[2 * md], u[4 * md + 0], s[0][0]);
        s[0][0] = cfma(a0[2 * md + 1], u[4 * md + 1], s[0][0]);
        s[0][1] = cfma(a0[2 * md], u[4 * md + 2], s[0][1]);
        s[0][1] = cfma(a0[2 * md + 1], u[4 * md + 3], s[0][1]);
        s[1][0] = cfma(a1[2 * md], u[4 * md + 0], s[1][0]);
        s[1][0] = cfma(a1[2 * md + 1], u[4 * md + 1], s[1][0]);
        s[1][1] = cfma(a1[2 * md], u[4 * md + 2], s[1][1]);
        s[1][1] = cfma(a1[2 * md + 1], u[4 * md + 3], s[1][1]);
      }
    }
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int k = 0; k < 2; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          s[j][k].re += __shfl_xor_sync(0xffffffffu, s[j][k].re, o);
          s[j][k].im += __shfl_xor_sync(0xffffffffu, s[j][k].im, o);
        }
    if (lane < 4) {
      int j = lane >> 1, k = lane & 1;
      if (j == 0 || two) {
        cx<T> v = (j == 0) ? (k == 0 ? s[0][0] : s[0][1]) : (k == 0 ? s[1][0] : s[1][1]);
        y[2 * (e0 + j) + k] += v;
      }
    }
  }
}

template <typename T>
__global__ void k_zero(cx<T>* p, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = mk<T>(0, 0);
}

// ---------------------------------------------------------------------------
// Batches of R right-hand sides.  Vector r sits at x + r * 2M (internal layout) and the
// level coefficients of box b hold R x 8 items, [b][r][item][Q], so item r * 8 + i has
// medium i & 1 as in the single product.  Every radiation pattern, translation table
// and phase factor read from memory is applied to all R vectors.

#define AGB_E 16  // edges per shared-memory tile of the batched aggregate

// C_box[r] = sum_e conj(RT_e) x_e[r]: block per (leaf box, 32 directions); the radiation
// patterns of AGB_E edges and their R x (J, M) coefficients are staged in shared memory,
// and warp w accumulates vectors w, w + 8, ... (RPW of them).
template <typename T, int RPW>
__global__ void __launch_bounds__(256) k_agg_b(const cx<T>* __restrict__ rt, const int* box_first,
                                               const int* box_cnt, int Q, const cx<T>* __restrict__ x,
                                               int M, int R, cx<T>* __restrict__ C) {
  __shared__ cx<T> srt[AGB_E][4][32];
  __shared__ cx<T> sx[AGB_E][2][8 * RPW];
  const int b = blockIdx.y, q0 = blockIdx.x * 32;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = q0 + lane;
  const int f = box_first[b], cnt = box_cnt[b];
  const size_t ldx = (size_t)2 * M;
  cx<T> acc[RPW][8];
#pragma unroll
  for (int rr = 0; rr < RPW; rr++)
#pragma unroll
    for (int i = 0; i < 8; i++) acc[rr][i] = mk<T>(0, 0);
  for (int e0 = 0; e0 < cnt; e0 += AGB_E) {
    const int ne = min(AGB_E, cnt - e0);
    for (int i = threadIdx.x; i < ne * 128; i += 256) {
      const int e = i >> 7, k = (i >> 5) & 3, j = i & 31;
      srt[e][k][j] = (q0 + j < Q) ? rt[(size_t)(f + e0 + e) * 4 * Q + (size_t)k * Q + q0 + j] : mk<T>(0, 0);
    }
    for (int i = threadIdx.x; i < ne * 2 * R; i += 256) {
      const int e = i / (2 * R), rem = i - e * 2 * R;
      sx[e][rem & 1][rem >> 1] = x[(size_t)(rem >> 1) * ldx + 2 * (f + e0 + e) + (rem & 1)];
    }
    __syncthreads();
    for (int e = 0; e < ne; e++) {
      const cx<T> ra1 = srt[e][0][lane], rb1 = srt[e][1][lane], ra2 = srt[e][2][lane], rb2 = srt[e][3][lane];
#pragma unroll
      for (int rr = 0; rr < RPW; rr++) {
        const int r = w + 8 * rr;
        if (r < R) {
          const cx<T> xe = sx[e][0][r], xh = sx[e][1][r];
          acc[rr][0] = cfma_conj(ra1, xe, acc[rr][0]);
          acc[rr][1] = cfma_conj(ra2, xe, acc[rr][1]);
          acc[rr][2] = cfma_conj(ra1, xh, acc[rr][2]);
          acc[rr][3] = cfma_conj(ra2, xh, acc[rr][3]);
          acc[rr][4] = cfma_conj(rb1, xe, acc[rr][4]);
          acc[rr][5] = cfma_conj(rb2, xe, acc[rr][5]);
          acc[rr][6] = cfma_conj(rb1, xh, acc[rr][6]);
          acc[rr][7] = cfma_conj(rb2, xh, acc[rr][7]);
        }
      }
    }
    __syncthreads();
  }
  if (q >= Q) return;
#pragma unroll
  for (int rr = 0; rr < RPW; rr++) {
    const int r = w + 8 * rr;
    if (r < R) {
      cx<T>* o = C + ((size_t)b * R + r) * 8 * Q + q;
#pragma unroll
      for (int i = 0; i < 8; i++) o[(size_t)i * Q] = acc[rr][i];
    }
  }
}

// SS of a batch: thread per (direction, parent box, vector r).
template <typename T>
__global__ void k_ss_b(const cx<T>* __restrict__ Cc, const int* ch_ptr, const int* ch_idx,
                       const int* ch_oct, const cx<T>* __restrict__ ph, int Q, int nmed, int R,
                       cx<T>* __restrict__ Cp) {
  const int b = blockIdx.y, r = blockIdx.z;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  cx<T> acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = mk<T>(0, 0);
  for (int k = ch_ptr[b]; k < ch_ptr[b + 1]; k++) {
    const int c = ch_idx[k], o = ch_oct[k];
    const cx<T>* src = Cc + ((size_t)c * R + r) * 8 * Q + q;
#pragma unroll
    for (int md = 0; md < 2; md++) {
      if (md < nmed) {
        const cx<T> p = ph[((size_t)o * 2 + md) * Q + q];
#pragma unroll
        for (int it = 0; it < 8; it += 2) acc[it + md] = cfma(src[(size_t)(it + md) * Q], p, acc[it + md]);
      }
    }
  }
  cx<T>* out = Cp + ((size_t)b * R + r) * 8 * Q + q;
#pragma unroll
  for (int i = 0; i < 8; i++) out[(size_t)i * Q] = acc[i];
}

// Fold of the eight D items of one (box, vector, direction) into the eight values the
// receive multiplies the radiation patterns by: per medium A1, B1 (first output) and
// A2, B2 (second output), as in k_receive_chunk, in FP64.  out[md * 4 + {A1, B1, A2, B2}].
__device__ __forceinline__ void recv_fold(const zc d[8], const RecvConst& rc, zc u[8], int q, int Q) {
#pragma unroll
  for (int md = 0; md < 2; md++) {
    const zc dJt = d[0 + md], dMt = d[2 + md], dJp = d[4 + md], dMp = d[6 + md];
    const zc kd = recv_kd(rc, md, q, Q);
    u[md * 4 + 0] = (rc.my_d[md] * dJt + kd * dMp) * rc.s1f;
    u[md * 4 + 1] = (rc.my_d[md] * dJp - kd * dMt) * rc.s1f;
    u[md * 4 + 2] = (rc.eps_d[md] * dMt - kd * dJp) * rc.s2f;
    u[md * 4 + 3] = (kd * dJt + rc.eps_d[md] * dMp) * rc.s2f;
  }
}

// RR of a batch: D_child[r] += D_parent[r] * exp(-i k khat.(x_child - x_parent)).  On the
// leaf level (fold = 1) the result is folded in place for the receive (recv_fold).
template <typename T>
__global__ void k_rr_b(const cx<T>* __restrict__ Dp, const int* parent, const int* oct,
                       const cx<T>* __restrict__ ph, int Q, int nmed, int R, int fold, RecvConst rc,
                       cx<T>* __restrict__ D) {
  const int b = blockIdx.y, r = blockIdx.z;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  const int p = parent[b];
  cx<T>* dst = D + ((size_t)b * R + r) * 8 * Q + q;
  cx<T> d[8];
#pragma unroll
  for (int i = 0; i < 8; i++) d[i] = dst[(size_t)i * Q];
  if (p >= 0) {
    const int o = oct[b];
    const cx<T>* src = Dp + ((size_t)p * R + r) * 8 * Q + q;
#pragma unroll
    for (int md = 0; md < 2; md++) {
      if (md < nmed) {
        const cx<T> f = ph[((size_t)o * 2 + md) * Q + q];
#pragma unroll
        for (int it = 0; it < 8; it += 2) d[it + md] = cfma(src[(size_t)(it + md) * Q], f, d[it + md]);
      }
    }
  }
  if (fold) {
    zc dz[8], u[8];
#pragma unroll
    for (int i = 0; i < 8; i++) dz[i] = cvt_z(d[i]);
    recv_fold(dz, rc, u, q, Q);
#pragma unroll
    for (int i = 0; i < 8; i++) dst[(size_t)i * Q] = mk<T>((T)u[i].re, (T)u[i].im);
  } else if (p >= 0) {
#pragma unroll
    for (int i = 0; i < 8; i++) dst[(size_t)i * Q] = d[i];
  }
}

// SR of a batch over the present siblings of one group (the k_sr_warp_ns scheme).  For
// each source the NS translation factors are read from shared memory once and applied to
// RC vectors, items it0 and it0 + 2 of each; ni = 8 R items per box.
template <typename T, int NS, int RC>
__device__ __forceinline__ void sr_nsb_body(const int* lst, int cnt, const cx<T>* Cq, int ni, int it0,
                                            const cx<T>* sTL, int qi, const int* sibc, const int* offc,
                                            bool qok, T wq, int Q, int zero_other,
                                            cx<T>* __restrict__ Dq) {
  int off[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) off[k] = offc[k] * SRW_QT + qi;
  cx<T> acc[RC][NS][2];
#pragma unroll
  for (int rc = 0; rc < RC; rc++)
#pragma unroll
    for (int k = 0; k < NS; k++) acc[rc][k][0] = acc[rc][k][1] = mk<T>(0, 0);
  for (int i = 0; i < cnt; i++) {
    const int s = lst[i];
    const size_t sb = (size_t)(s >> 9) * ni + it0;
    const int t0 = (s & 511) * SRW_QT;
    cx<T> c0[RC], c1[RC];
#pragma unroll
    for (int rc = 0; rc < RC; rc++) {
      c0[rc] = Cq[(sb + 8 * rc) * Q];
      c1[rc] = Cq[(sb + 8 * rc + 2) * Q];
    }
    cx<T> f[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) f[k] = sTL[t0 + off[k]];
#pragma unroll
    for (int rc = 0; rc < RC; rc++)
#pragma unroll
      for (int k = 0; k < NS; k++) {
        acc[rc][k][0] = cfma(c0[rc], f[k], acc[rc][k][0]);
        acc[rc][k][1] = cfma(c1[rc], f[k], acc[rc][k][1]);
      }
  }
  if (!qok) return;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    cx<T>* out = Dq + (size_t)sibc[k] * ni * Q;
#pragma unroll
    for (int rc = 0; rc < RC; rc++) {
      const int i0 = it0 + 8 * rc;
      out[(size_t)i0 * Q] = acc[rc][k][0] * wq;
      out[(size_t)(i0 + 2) * Q] = acc[rc][k][1] * wq;
      if (zero_other) {
        out[(size_t)(i0 ^ 1) * Q] = mk<T>(0, 0);
        out[(size_t)((i0 + 2) ^ 1) * Q] = mk<T>(0, 0);
      }
    }
  }
}

template <typename T, int RC>
__global__ void __launch_bounds__(32 * SRW_GB, 2) k_sr_ns_b(
    const cx<T>* __restrict__ C, const int* __restrict__ grp_sib, const int* __restrict__ grp_src,
    int ngrp, const cx<T>* __restrict__ tl, const T* __restrict__ trf, int Q, int md,
    int zero_other, int R, cx<T>* __restrict__ D) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sTL = reinterpret_cast<cx<T>*>(smraw);                  // [343][SRW_QT]
  int* s_list = reinterpret_cast<int*>(sTL + 343 * SRW_QT);      // [SRW_GB][216]
  int* s_sib = s_list + SRW_GB * 216;                            // [SRW_GB][8]
  int* s_off = s_sib + SRW_GB * 8;                               // [SRW_GB][8]
  const int q0 = blockIdx.x * SRW_QT;
  const int tid = threadIdx.x;
  for (int i = tid; i < 343 * SRW_QT; i += blockDim.x) {
    const int t = i / SRW_QT, j = i - t * SRW_QT;
    const int q = q0 + j;
    sTL[i] = (q < Q) ? tl[((size_t)t * 2 + md) * Q + q] : mk<T>(0, 0);
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  const int g = blockIdx.y * SRW_GB + w;
  if (g >= ngrp) return;
  const int sib = (lane < 8) ? grp_sib[(size_t)g * 8 + lane] : -1;
  const unsigned smask = __ballot_sync(0xffffffffu, sib >= 0) & 0xffu;
  const int ns = __popc(smask);
  if (sib >= 0) {
    const int k = __popc(smask & ((1u << lane) - 1u));
    s_sib[w * 8 + k] = sib;
    s_off[w * 8 + k] = ((lane >> 2) & 1) * 49 + ((lane >> 1) & 1) * 7 + (lane & 1);
  }
  int* lst = s_list + w * 216;
  int cnt = 0;
  for (int base = 0; base < 216; base += 32) {
    const int dc = base + lane;
    const int d = dc >> 3, c = dc & 7;
    const int s = (dc < 216 && d != 13) ? grp_src[(size_t)g * 216 + dc] : -1;
    const unsigned bal = __ballot_sync(0xffffffffu, s >= 0);
    if (s >= 0) {
      const int t0 = (3 - ((c >> 2) & 1) - 2 * (d / 9 - 1)) * 49 + (3 - ((c >> 1) & 1) - 2 * ((d / 3) % 3 - 1)) * 7 +
                     (3 - (c & 1) - 2 * (d % 3 - 1));
      lst[cnt + __popc(bal & ((1u << lane) - 1u))] = (s << 9) | t0;
    }
    cnt += __popc(bal);
  }
  __syncwarp();
  const int ih = lane >> 4, qi = lane & 15;
  const int q = q0 + qi;
  const bool qok = q < Q;
  const cx<T>* Cq = C + (qok ? q : 0);
  cx<T>* Dq = D + (qok ? q : 0);
  const T wq = trf[qok ? q : 0];
  const int* sibc = s_sib + w * 8;
  const int* offc = s_off + w * 8;
  const int ni = 8 * R;
  // blockIdx.z picks the RC vectors: the slowest grid dimension, so the blocks resident at
  // any time read the coefficients of only RC vectors, a slice that stays in L2 while the
  // ~27 sibling groups around each source box read it
  const int it0 = md + 4 * ih + 8 * (blockIdx.z * RC);
  switch (ns) {
    case 1: sr_nsb_body<T, 1, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 2: sr_nsb_body<T, 2, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 3: sr_nsb_body<T, 3, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 4: sr_nsb_body<T, 4, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 5: sr_nsb_body<T, 5, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 6: sr_nsb_body<T, 6, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 7: sr_nsb_body<T, 7, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    case 8: sr_nsb_body<T, 8, RC>(lst, cnt, Cq, ni, it0, sTL, qi, sibc, offc, qok, wq, Q, zero_other, Dq); break;
    default: break;
  }
}

// Receive of a batch as a small complex GEMM per chunk of <= 32 edges of one leaf box:
//   y[r][e][o] += sum over (medium md, row ab, direction q) of RT[e][2 md + ab][q] U[r][md][o][ab][q]
// with U the folded leaf coefficients (recv_fold, written by the leaf RR).  The block is 4
// direction groups x 64 threads; thread (eq, rp) of a group owns edges eq, eq + 8, eq + 16,
// eq + 24 and vectors 2 rp, 2 rp + 1 (both outputs): 16 accumulators, 16 shared-memory
// reads per 32 complex FMAs.  Tiles of QT directions of RT ([row][edge][q]) and U
// ([k][r][q]) stream in by asynchronous copies into two buffers, the next tile loading
// while the current one is used; the padded rows keep a warp's reads on distinct banks.
// The four groups take every fourth direction of a tile and their sums meet in shared
// memory at the end.
template <typename T> struct RecvTile { static const int QT = 16; };

template <typename T>
static size_t recv_g_smem() {
  const int QT = RecvTile<T>::QT, QP = QT + 2;
  size_t tiles = (size_t)2 * (4 * 32 + 8 * 16) * QP * sizeof(cx<T>);
  size_t red = (size_t)4 * 32 * 16 * 2 * sizeof(cx<T>);
  return std::max(tiles, red);
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(256) k_recv_g(const cx<T>* __restrict__ rt, const int4* __restrict__ chunks,
                                                const cx<T>* __restrict__ U, int Q, int M, int R,
                                                cx<T>* __restrict__ y) {
  constexpr int QT = RecvTile<T>::QT, QP = QT + 2;
  constexpr int EPC = 16 / (int)sizeof(cx<T>);   // directions per 16-byte piece
  constexpr int PPR = QT / EPC;                   // pieces per tile row
  constexpr int BUF = (4 * 32 + 8 * 16) * QP;     // complex values per buffer
  constexpr bool split = sizeof(T) == 4;          // FP32: a fresh partial per tile
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);    // [2][sRT 4 x 32 x QP, sU 8 x 16 x QP]
  const int4 ch = chunks[blockIdx.x];
  const int b = ch.x, f = ch.y, cnt = ch.z;
  const int tid = threadIdx.x, kg = tid >> 6, t = tid & 63;
  const int eq = t & 7, rp = t >> 3;
  const cx<T>* Ub = U + (size_t)b * R * 8 * Q;
  auto stage = [&](int q0, int buf) {
    cx<T>* sRT = sm + buf * BUF;
    cx<T>* sU = sRT + 4 * 32 * QP;
    for (int i = tid; i < 4 * 32 * PPR; i += 256) {  // RT rows (row, edge)
      const int row = i / (32 * PPR), rem = i - row * 32 * PPR, e = rem / PPR, part = rem - e * PPR;
      const int qs = q0 + part * EPC;
      const int bytes = e < cnt ? max(0, min(16, (Q - qs) * (int)sizeof(cx<T>))) : 0;
      const cx<T>* src = bytes > 0 ? rt + (size_t)(f + e) * 4 * Q + (size_t)row * Q + qs : rt;
      cp_async16(sRT + (row * 32 + e) * QP + part * EPC, src, bytes);
    }
    for (int i = tid; i < 8 * 16 * PPR; i += 256) {  // U rows (k, vector)
      const int k = i / (16 * PPR), rem = i - k * 16 * PPR, r = rem / PPR, part = rem - r * PPR;
      const int qs = q0 + part * EPC;
      const int bytes = r < R ? max(0, min(16, (Q - qs) * (int)sizeof(cx<T>))) : 0;
      const cx<T>* src = bytes > 0 ? Ub + ((size_t)r * 8 + k) * Q + qs : Ub;
      cp_async16(sU + (k * 16 + r) * QP + part * EPC, src, bytes);
    }
    cp_async_commit();
  };
  cx<T> acc[4][2][2];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int jr = 0; jr < 2; jr++) acc[j][jr][0] = acc[j][jr][1] = mk<T>(0, 0);
  const int ntile = (Q + QT - 1) / QT;
  stage(0, 0);
  for (int tt = 0; tt < ntile; tt++) {
    if (tt + 1 < ntile) {
      stage((tt + 1) * QT, (tt + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const cx<T>* sRT = sm + (tt & 1) * BUF;
    const cx<T>* sU = sRT + 4 * 32 * QP;
    cx<T> pt[4][2][2];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int jr = 0; jr < 2; jr++)
#pragma unroll
        for (int o = 0; o < 2; o++) pt[j][jr][o] = split ? mk<T>(0, 0) : acc[j][jr][o];
#pragma unroll 2
    for (int qq = kg; qq < QT; qq += 4) {
#pragma unroll
      for (int md = 0; md < 2; md++) {
        cx<T> a[4][2], u[2][2][2];
#pragma unroll
        for (int ab = 0; ab < 2; ab++)
#pragma unroll
          for (int j = 0; j < 4; j++) a[j][ab] = sRT[((2 * md + ab) * 32 + eq + 8 * j) * QP + qq];
#pragma unroll
        for (int o = 0; o < 2; o++)
#pragma unroll
          for (int ab = 0; ab < 2; ab++)
#pragma unroll
            for (int jr = 0; jr < 2; jr++) u[jr][o][ab] = sU[((md * 4 + o * 2 + ab) * 16 + 2 * rp + jr) * QP + qq];
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int jr = 0; jr < 2; jr++)
#pragma unroll
            for (int o = 0; o < 2; o++) {
              pt[j][jr][o] = cfma(a[j][0], u[jr][o][0], pt[j][jr][o]);
              pt[j][jr][o] = cfma(a[j][1], u[jr][o][1], pt[j][jr][o]);
            }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int jr = 0; jr < 2; jr++)
#pragma unroll
        for (int o = 0; o < 2; o++) acc[j][jr][o] = split ? acc[j][jr][o] + pt[j][jr][o] : pt[j][jr][o];
    __syncthreads();  // the buffer is refilled by the next iteration's copies
  }
  // the four direction groups' partial sums: red[kg][e][r][o]
  cx<T>* red = sm;
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int jr = 0; jr < 2; jr++)
#pragma unroll
      for (int o = 0; o < 2; o++)
        red[(((size_t)kg * 32 + eq + 8 * j) * 16 + 2 * rp + jr) * 2 + o] = acc[j][jr][o];
  __syncthreads();
  const size_t ldy = (size_t)2 * M;
  for (int i = tid; i < 32 * 16 * 2; i += 256) {
    const int e = i >> 5, r = (i >> 1) & 15, o = i & 1;
    if (e < cnt && r < R) {
      cx<T> s = red[i];
      s += red[1024 + i];
      s += red[2048 + i];
      s += red[3072 + i];
      y[(size_t)r * ldy + 2 * (f + e) + o] += s;
    }
  }
}

// ---------------------------------------------------------------------------
// host side

int far_build_tables(sie_ctx* c, const double* d_boxc) {
  cudaStream_t st = c->stream;
  int Q = c->Q, K = c->K, M = c->M;
  // radiation patterns
  {
    // one launch per 65,535 edges (the grid's y limit)
    for (int e0 = 0; e0 < M; e0 += 65535) {
      dim3 g((Q + 127) / 128, std::min(65535, M - e0));
      k_rt<<<g, 128, 0, st>>>(c->d_fn, d_boxc, c->d_edge_box, M, c->R, c->mt.k1, c->mt.k2, c->d_khat,
                              c->d_tth, c->d_tph, Q, c->d_rt, e0); sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
  }
  // TL tables per level, each on its level's sampling
  int Kmax = K;
  for (int l = c->l_min; l <= c->l_max; l++) Kmax = std::max(Kmax, c->lv[l].K);
  zc* hk = nullptr;
  SIE_CUDA(cudaMalloc(&hk, (size_t)343 * 2 * Kmax * sizeof(zc)));
  for (int l = c->l_min; l <= c->l_max; l++) {
    Level& L = c->lv[l];
    double dc = ldexp(1.0, -l) * c->D;
    double xmn = -3 * dc, xmx = -xmn;
    double dx = (xmx - xmn) / 6;
    k_hankel<<<(343 + 63) / 64, 64, 0, st>>>(xmn, dx, c->mt.k1, c->mt.k2, L.K, L.only_k1, hk); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
    dim3 g((L.Q + 127) / 128, 343);
    k_tl<<<g, 128, 0, st>>>(xmn, dx, hk, c->mt.k1, c->mt.k2, L.K, L.Q, L.khat, L.tl); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  SIE_CUDA(cudaStreamSynchronize(st));
  cudaFree(hk);
  return SIE_OK;
}

// Tables of the precision the pass runs in.
template <typename T> static const cx<T>* tlp(const Level& L);
template <> const zc* tlp<double>(const Level& L) { return L.tl; }
template <> const cc* tlp<float>(const Level& L) { return L.tl32; }
template <typename T> static const cx<T>* php_up(const Level& L);
template <> const zc* php_up<double>(const Level& L) { return L.ph_up; }
template <> const cc* php_up<float>(const Level& L) { return L.ph_up32; }
template <typename T> static const cx<T>* php_dn(const Level& L);
template <> const zc* php_dn<double>(const Level& L) { return L.ph_dn; }
template <> const cc* php_dn<float>(const Level& L) { return L.ph_dn32; }
template <typename T> static const T* trfp(const Level& L);
template <> const double* trfp<double>(const Level& L) { return L.trf; }
template <> const float* trfp<float>(const Level& L) { return L.trf32; }
template <typename T> static const T* ivalp(const InterpDev& I);
template <> const double* ivalp<double>(const InterpDev& I) { return I.val; }
template <> const float* ivalp<float>(const InterpDev& I) { return I.val32; }
template <typename T> static const T* ievalp(const InterpDev& I);
template <> const double* ievalp<double>(const InterpDev& I) { return I.eval; }
template <> const float* ievalp<float>(const InterpDev& I) { return I.eval32; }
template <typename T> static const T* iovalp(const InterpDev& I);
template <> const double* iovalp<double>(const InterpDev& I) { return I.oval; }
template <> const float* iovalp<float>(const InterpDev& I) { return I.oval32; }

// Interpolation between two levels' samplings on every (theta, phi) item pair of nbox
// coefficient blocks [8][Q]: out[b][item][q] (+)= sum_k val[k] in[b][...][col[k]], with
// inputs and outputs ordered (theta values, then phi values) as the CSR rows and
// columns are.  Thread per (output row, block, item pair).
template <typename T>
__global__ void __launch_bounds__(128) k_interp(const int* __restrict__ ptr, const int* __restrict__ col,
                                                const T* __restrict__ val, int rows,
                                                const cx<T>* __restrict__ in, int Qi,
                                                cx<T>* __restrict__ out, int Qo, int accum) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const size_t b = blockIdx.y;
  const int p = blockIdx.z;
  const cx<T>* a = in + (b * 8 + p) * (size_t)Qi;       // theta item p
  const cx<T>* bb = in + (b * 8 + p + 4) * (size_t)Qi;  // its phi item
  cx<T> acc = mk<T>(0, 0);
  for (int k = ptr[r]; k < ptr[r + 1]; k++) {
    const int j = col[k];
    const cx<T> v = j < Qi ? a[j] : bb[j - Qi];
    const T w = val[k];
    acc.re = fma(w, v.re, acc.re);
    acc.im = fma(w, v.im, acc.im);
  }
  const int item = r < Qo ? p : p + 4, q = r < Qo ? r : r - Qo;
  cx<T>* o = out + (b * 8 + item) * (size_t)Qo + q;
  if (accum) *o += acc;
  else *o = acc;
}

// The same on the tap-major stencil: the block's inputs staged in shared memory, a thread
// per output row, four taps' (column, weight) pairs loaded together (coalesced across the
// warp's rows) before their shared-memory reads and multiply-adds; the long rows' remaining
// taps from the CSR overflow.  A block takes np of the four item pairs (pairs
// blockIdx.y * np ..), so that a sampling too large for all eight items in shared memory
// runs as two blocks of two pairs.
template <typename T>
__global__ void __launch_bounds__(256) k_interp_e(const int* __restrict__ ecol, const T* __restrict__ eval, int ew,
                                                  const int* __restrict__ optr, const int* __restrict__ ocol,
                                                  const T* __restrict__ oval, int rows,
                                                  const cx<T>* __restrict__ in, int Qi,
                                                  cx<T>* __restrict__ out, int Qo, int accum, int np) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* xs = reinterpret_cast<cx<T>*>(smraw);  // [theta items p0 .. p0 + np, then phi items][Qi]
  const size_t b = blockIdx.x;
  const int p0 = blockIdx.y * np;
  const cx<T>* src = in + b * 8 * (size_t)Qi;
  for (int i = threadIdx.x; i < 2 * np * Qi; i += blockDim.x) {
    const int h = i / (np * Qi), rem = i - h * np * Qi;  // h: 0 theta, 1 phi
    xs[i] = src[(size_t)(4 * h + p0) * Qi + rem];
  }
  __syncthreads();
  cx<T>* dst = out + b * 8 * (size_t)Qo;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    cx<T> acc[4];
#pragma unroll
    for (int p = 0; p < 4; p++) acc[p] = mk<T>(0, 0);
    for (int t0 = 0; t0 < ew; t0 += 4) {
      int j[4];
      T w[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const bool in_ = t0 + u < ew;
        j[u] = in_ ? ecol[(size_t)(t0 + u) * rows + r] : 0;
        w[u] = in_ ? eval[(size_t)(t0 + u) * rows + r] : (T)0;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const cx<T>* sp = j[u] < Qi ? xs + j[u] : xs + (size_t)np * Qi + (j[u] - Qi);
#pragma unroll
        for (int p = 0; p < 4; p++)
          if (p < np) {
            const cx<T> v = sp[(size_t)p * Qi];
            acc[p].re = fma(w[u], v.re, acc[p].re);
            acc[p].im = fma(w[u], v.im, acc[p].im);
          }
      }
    }
    for (int k = optr[r]; k < optr[r + 1]; k++) {
      const int j = ocol[k];
      const T w = oval[k];
      const cx<T>* sp = j < Qi ? xs + j : xs + (size_t)np * Qi + (j - Qi);
#pragma unroll
      for (int p = 0; p < 4; p++)
        if (p < np) {
          const cx<T> v = sp[(size_t)p * Qi];
          acc[p].re = fma(w, v.re, acc[p].re);
          acc[p].im = fma(w, v.im, acc[p].im);
        }
    }
    const int q = r < Qo ? r : r - Qo, i0 = r < Qo ? 0 : 4;
#pragma unroll
    for (int p = 0; p < 4; p++)
      if (p < np) {
        cx<T>* o = dst + (size_t)(i0 + p0 + p) * Qo + q;
        if (accum) *o += acc[p];
        else *o = acc[p];
      }
  }
}

// nbox blocks of [8][Qi] through I into blocks of [8][Qo] (Qo = I.rows / 2).
template <typename T>
static int interp_run(const InterpDev& I, const cx<T>* in, int Qi, cx<T>* out, size_t nbox, bool accum,
                      cudaStream_t st) {
  const size_t smem = (size_t)8 * Qi * sizeof(cx<T>);
  // all four item pairs per block; a sampling too large for eight items in shared memory
  // takes the CSR kernel on global memory below (many more blocks in flight, which measured
  // faster than two staged blocks of two pairs)
  const int np = smem <= (size_t)200 * 1024 ? 4 : 0;
  if (np > 0 && ievalp<T>(I)) {
    const size_t sm = smem * np / 4;
    SIE_CUDA(raise_smem(k_interp_e<T>, sm));
    for (size_t b0 = 0; b0 < nbox; b0 += 65535u) {
      const unsigned nb = (unsigned)std::min<size_t>(65535u, nbox - b0);
      k_interp_e<T><<<dim3(nb, 4 / np), 256, sm, st>>>(I.ecol, ievalp<T>(I), I.ew, I.optr, I.ocol, iovalp<T>(I),
                                                       I.rows, in + b0 * 8 * Qi, Qi, out + b0 * 8 * (I.rows / 2),
                                                       I.rows / 2, accum ? 1 : 0, np);
      sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
    return SIE_OK;
  }
  for (size_t b0 = 0; b0 < nbox; b0 += 65535) {
    const unsigned nb = (unsigned)std::min<size_t>(65535, nbox - b0);
    dim3 g((I.rows + 127) / 128, nb, 4);
    k_interp<T><<<g, 128, 0, st>>>(I.ptr, I.col, ivalp<T>(I), I.rows, in + b0 * 8 * Qi, Qi,
                                   out + b0 * 8 * (I.rows / 2), I.rows / 2, accum ? 1 : 0);
    sie::count_launch();
  }
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// Work buffer for coefficients on another level's sampling, grown on demand.
static int lvtmp(sie_ctx* c, size_t bytes, void** p) {
  if (c->lvtmp_bytes < bytes) {
    if (c->d_lvtmp) cudaFree(c->d_lvtmp);
    c->d_lvtmp = nullptr;
    c->lvtmp_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_lvtmp, bytes));
    c->lvtmp_bytes = bytes;
  }
  *p = c->d_lvtmp;
  return SIE_OK;
}

// Factors of the final far summation (MLFMM_tri_summation_New,
// lib_sie_tri_mlfmm.f90:416-497) and the ICTF output scaling (:486-488).
static RecvConst recv_const(const sie_ctx* c) {
  RecvConst rc;
  zc I = mk<double>(0, 1);
  rc.kd[0] = c->mt.k1 * I;
  rc.kd[1] = c->mt.k2 * I;
  rc.my_d[0] = mk<double>(0, c->mt.my1 * c->mt.omega);
  rc.my_d[1] = mk<double>(0, c->mt.my2 * c->mt.omega);
  rc.eps_d[0] = c->mt.eps1 * I * c->mt.omega;
  rc.eps_d[1] = c->mt.eps2 * I * c->mt.omega;
  if (c->cfg.formulation == SIE_ICTF) {
    rc.s1f = mk<double>(1, 0) / c->mt.eta_a;
    rc.s2f = c->mt.eta_a;
  } else {
    rc.s1f = mk<double>(1, 0);
    rc.s2f = mk<double>(1, 0);
  }
  rc.pole_fix = c->level_k ? 1 : 0;
  return rc;
}

// The translation passes between the leaf aggregate and the receive: SS up the tree, SR on
// every level, RR down, from the level coefficients C to the leaf D (events 2, 3, 4).
template <typename T>
static int far_translate_t(sie_ctx* c, cudaStream_t st, cudaEvent_t* ev,
                           const std::function<int()>* after_ss = nullptr) {
  const int L0 = c->l_min, L1 = c->l_max;
  const bool k2c = c->mt.k2.im != 0.0;
  const int thr = 128;
  // up 2: a child level with a smaller sampling is interpolated to the parent's first
  // (translation_SS, lib_sie_tri_mlfmm_interface.f90:486-507), then shifted on it
  for (int l = L1 - 1; l >= L0; l--) {
    Level& P = c->lv[l];
    Level& Ch = c->lv[l + 1];
    const int Q = P.Q;
    const cx<T>* src = (const cx<T>*)Ch.C;
    if (Ch.Q != Q) {
      void* tmp = nullptr;
      SIE_TRY(lvtmp(c, (size_t)Ch.nb * 8 * Q * sizeof(cx<T>), &tmp));
      SIE_TRY(interp_run<T>(P.up, src, Ch.Q, (cx<T>*)tmp, Ch.nb, false, st));
      src = (const cx<T>*)tmp;
    }
    dim3 g((Q + thr - 1) / thr, P.nb);
    k_ss<T><<<g, thr, 0, st>>>(src, P.ch_ptr, P.ch_idx, P.ch_oct,
                               php_up<T>(Ch), Q, k2c ? 1 : 2, (cx<T>*)P.C); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  if (ev) cudaEventRecord(ev[2], st);
  if (after_ss) SIE_TRY((*after_ss)());
  // down 1
  for (int l = L0; l <= L1; l++) {
    Level& L = c->lv[l];
    const int Q = L.Q;
    if (c->sr_mode == 0) {
      dim3 g((Q + thr - 1) / thr, L.nb);
      k_sr<T><<<g, thr, 0, st>>>((const cx<T>*)L.C, L.i4_ptr, L.i4_src, L.i4_off,
                                 tlp<T>(L), trfp<T>(L), Q, L.only_k1 ? 1 : 2,
                                 (cx<T>*)L.D); sie::count_launch();
    } else if (c->sr_mode == 5 && L.nb < (1 << 22)) {  // source box and T0 share one int
      dim3 g((Q + SRW_QT - 1) / SRW_QT, (L.ngrp + SRW_GB - 1) / SRW_GB);
      int nmed = L.only_k1 ? 1 : 2;
      for (int md = 0; md < nmed; md++) {
        // FP64: coefficient loads evict-last, D stores streaming (measured on slab10:
        // SR 0.380 -> 0.360 ms, the same bits); complex64 keeps plain accesses
        constexpr int hint = std::is_same<T, double>::value ? 3 : 0;
        k_sr_warp_ns<T, 1, hint><<<g, 32 * SRW_GB, sr_warp_ns_smem<T>(), st>>>(
            (const cx<T>*)L.C, L.grp_sib, L.grp_src, L.ngrp, tlp<T>(L), trfp<T>(L), Q, md, nmed == 1, (cx<T>*)L.D);
        sie::count_launch();
      }
    } else if (c->sr_mode >= 4 && L.nb < (1 << 23)) {
      dim3 g((Q + SRW_QT - 1) / SRW_QT, (L.ngrp + SRW_GB - 1) / SRW_GB);
      int nmed = L.only_k1 ? 1 : 2;
      for (int md = 0; md < nmed; md++) {
        k_sr_warp_bf<T><<<g, 32 * SRW_GB, sr_warp_bf_smem<T>(), st>>>(
            (const cx<T>*)L.C, L.grp_sib, L.grp_src, L.ngrp, tlp<T>(L),
            trfp<T>(L), Q, md, nmed == 1, (cx<T>*)L.D); sie::count_launch();
      }
    } else if (c->sr_mode >= 3 && L.nb < (1 << 23)) {  // source box and slot share one int
      dim3 g((Q + SRW_QT - 1) / SRW_QT, (L.ngrp + SRW_GB - 1) / SRW_GB);
      int nmed = L.only_k1 ? 1 : 2;
      for (int md = 0; md < nmed; md++) {
        k_sr_warp<T><<<g, 32 * SRW_GB, sr_warp_smem<T>(), st>>>(
            (const cx<T>*)L.C, L.grp_sib, L.grp_src, L.ngrp, tlp<T>(L),
            trfp<T>(L), Q, md, nmed == 1, (cx<T>*)L.D); sie::count_launch();
      }
    } else if (c->sr_mode == 2) {
      dim3 g((Q + SR_TQ - 1) / SR_TQ, (L.ngrp + SR_GB - 1) / SR_GB);
      size_t smem = (size_t)343 * SR_TQ * sizeof(cx<T>) + (size_t)SR_GB * (216 + 8) * sizeof(int);
      int nmed = L.only_k1 ? 1 : 2;
      for (int md = 0; md < nmed; md++) {
        k_sr_group_tl<T><<<g, SR_TQ * SR_GB, smem, st>>>((const cx<T>*)L.C, L.grp_sib, L.grp_src,
                                                          L.ngrp, tlp<T>(L),
                                                          trfp<T>(L), Q, md, nmed == 1,
                                                          (cx<T>*)L.D); sie::count_launch();
      }
    } else {
      dim3 g((Q + thr - 1) / thr, L.ngrp);
      int nmed = L.only_k1 ? 1 : 2;
      for (int md = 0; md < nmed; md++)
        for (int i0 = 0; i0 < 4; i0 += 2) {
          k_sr_group<T, 2><<<g, thr, 0, st>>>((const cx<T>*)L.C, L.grp_sib, L.grp_src,
                                              tlp<T>(L), trfp<T>(L), Q, md, i0,
                                              nmed == 1, (cx<T>*)L.D); sie::count_launch();
        }
    }
    SIE_CUDA(cudaGetLastError());
  }
  if (ev) cudaEventRecord(ev[3], st);
  // down 2: a child level with a smaller sampling takes the parent's D shifted on the
  // parent's sampling, then anterpolated (the transpose of the SS interpolation)
  for (int l = L0 + 1; l <= L1; l++) {
    Level& L = c->lv[l];
    Level& P = c->lv[l - 1];
    int nmed = (k2c && l < L1) ? 1 : 2;
    // D_k2 of the parent is zero when its level only carries k1
    if (k2c) nmed = 1;
    if (L.Q != P.Q) {
      const int Qp = P.Q;
      void* tmp = nullptr;
      const size_t n = (size_t)L.nb * 8 * Qp;
      SIE_TRY(lvtmp(c, n * sizeof(cx<T>), &tmp));
      SIE_CUDA(cudaMemsetAsync(tmp, 0, n * sizeof(cx<T>), st));
      dim3 g((Qp + thr - 1) / thr, L.nb);
      k_rr<T><<<g, thr, 0, st>>>((const cx<T>*)P.D, L.parent, L.oct, php_dn<T>(L), Qp, nmed,
                                 (cx<T>*)tmp); sie::count_launch();
      SIE_CUDA(cudaGetLastError());
      SIE_TRY(interp_run<T>(P.dn, (const cx<T>*)tmp, Qp, (cx<T>*)L.D, L.nb, true, st));
      continue;
    }
    const int Q = L.Q;
    dim3 g((Q + thr - 1) / thr, L.nb);
    k_rr<T><<<g, thr, 0, st>>>((const cx<T>*)P.D, L.parent, L.oct, php_dn<T>(L), Q, nmed,
                               (cx<T>*)L.D); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  if (ev) cudaEventRecord(ev[4], st);
  return SIE_OK;
}

template <typename T>
int far_matvec_t(sie_ctx* c, const cx<T>* rt, const cx<T>* x, cx<T>* y, cudaStream_t st,
                 cudaEvent_t* ev, cudaEvent_t wait_recv, const std::function<int()>* after_agg) {
  int Q = c->Q;
  int L1 = c->l_max;
  // up 1
  {
    Level& L = c->lv[L1];
    if (c->agg_mode == 1) {
      dim3 g((Q + 31) / 32, L.nb);
      k_aggregate_eg<T><<<g, 256, 0, st>>>(rt, c->d_box_first, c->d_box_cnt, Q, x, (cx<T>*)L.C); sie::count_launch();
    } else {
      dim3 g((Q + 127) / 128, L.nb);
      k_aggregate<T><<<g, 128, 0, st>>>(rt, c->d_box_first, c->d_box_cnt, Q, x, (cx<T>*)L.C); sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
  }
  if (ev) cudaEventRecord(ev[1], st);
  const bool at_sr = c->overlap_near == 3;  // the hook runs once the SS passes are queued
  if (after_agg && !at_sr) SIE_TRY((*after_agg)());
  SIE_TRY(far_translate_t<T>(c, st, ev, at_sr ? after_agg : nullptr));
  // the receive adds into y, which the near product (possibly on another stream) writes
  if (wait_recv) SIE_CUDA(cudaStreamWaitEvent(st, wait_recv, 0));
  // final far summation
  {
    Level& L = c->lv[L1];
    const RecvConst rc = recv_const(c);
    size_t smem = (size_t)8 * Q * sizeof(cx<T>);
    if (c->recv_mode == 1) {
      k_receive_chunk<T><<<c->n_rchunk, 256, smem, st>>>(rt, (const int4*)c->d_rchunk,
                                                         (const cx<T>*)L.D, Q, rc, y); sie::count_launch();
    } else {
      k_receive<T><<<L.nb, 256, smem, st>>>(rt, c->d_box_first, c->d_box_cnt, (const cx<T>*)L.D, Q,
                                            rc, y); sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
  }
  if (ev) cudaEventRecord(ev[5], st);
  return SIE_OK;
}

// ---------------------------------------------------------------------------
// Transpose of the far product, Z_far^T = A^T (pi T pi) R^T.  A is the leaf aggregate, R the
// receive (fold of D, then the sum against the radiation patterns), T the translation
// passes, and pi the direction permutation q -> q' with khat_q' = -khat_q.  The transpose
// of a step that multiplies by a function of khat (SS, SR, RR phases and TL) is the same
// step at -khat: SS^T = pi RR pi, RR^T = pi SS pi, SR^T = pi SR pi, so T^T = pi T pi and
// the translation passes run unchanged between the two permutations.

// R^T then pi: per (leaf box, direction) C[b][i][pi(q)] = Fold^T(sum_e RT_e(q) y_e); thread per
// (direction, leaf box).  (An 8-edge-group block as in k_aggregate_eg measured slower here.)
__global__ void k_adj_in(const zc* __restrict__ rt, const int* box_first, const int* box_cnt, int Q,
                         const zc* __restrict__ y, const int* __restrict__ qperm, RecvConst rc,
                         zc* __restrict__ C) {
  const int b = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q) return;
  zc U[2][2][2];  // [md][o][ab]: o = output of the receive, ab = theta / phi row
#pragma unroll
  for (int md = 0; md < 2; md++) U[md][0][0] = U[md][0][1] = U[md][1][0] = U[md][1][1] = mk<double>(0, 0);
  const int f = box_first[b], cnt = box_cnt[b];
  for (int e = f; e < f + cnt; e++) {
    const zc* r = rt + (size_t)e * 4 * Q + q;
    const zc y0 = y[2 * e], y1 = y[2 * e + 1];
#pragma unroll
    for (int md = 0; md < 2; md++)
#pragma unroll
      for (int ab = 0; ab < 2; ab++) {
        const zc v = r[(size_t)(2 * md + ab) * Q];
        U[md][0][ab] = cfma(v, y0, U[md][0][ab]);
        U[md][1][ab] = cfma(v, y1, U[md][1][ab]);
      }
  }
  // transpose of the fold (A1, B1, A2, B2) = F (dJt, dMt, dJp, dMp) of the receive
  zc d[8];
#pragma unroll
  for (int md = 0; md < 2; md++) {
    const zc A1 = U[md][0][0], B1 = U[md][0][1], A2 = U[md][1][0], B2 = U[md][1][1];
    d[0 + md] = rc.s1f * rc.my_d[md] * A1 + rc.s2f * rc.kd[md] * B2;
    d[2 + md] = rc.s2f * rc.eps_d[md] * A2 - rc.s1f * rc.kd[md] * B1;
    d[4 + md] = rc.s1f * rc.my_d[md] * B1 - rc.s2f * rc.kd[md] * A2;
    d[6 + md] = rc.s1f * rc.kd[md] * A1 + rc.s2f * rc.eps_d[md] * B2;
  }
  zc* o = C + (size_t)b * 8 * Q + qperm[q];
#pragma unroll
  for (int i = 0; i < 8; i++) o[(size_t)i * Q] = d[i];
}

// pi then A^T over chunks of <= 32 edges (as k_receive_chunk): the box's D, permuted, in
// shared memory; each warp streams the radiation patterns of two edges at a time.
//   x_e[J] = sum_q conj(RT) of the J items of D[b][.][pi(q)], the same for M.
__global__ void __launch_bounds__(256, 2) k_adj_out(const zc* __restrict__ rt, const int4* __restrict__ chunks,
                                                    int Q, const zc* __restrict__ D, const int* __restrict__ qperm,
                                                    zc* __restrict__ x) {
  extern __shared__ __align__(16) unsigned char smraw[];
  zc* sD = reinterpret_cast<zc*>(smraw);  // [8][Q], direction q holds D at pi(q)
  const int4 ch = chunks[blockIdx.x];
  const int b = ch.x, f = ch.y, cnt = ch.z;
  const zc* Db = D + (size_t)b * 8 * Q;
  for (int i = threadIdx.x; i < 8 * Q; i += blockDim.x) {
    const int it = i / Q, q = i - it * Q;
    sD[i] = Db[(size_t)it * Q + qperm[q]];
  }
  __syncthreads();
  const unsigned long long pol = l2_evict_first_policy();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e0 = f + 2 * warp; e0 < f + cnt; e0 += 16) {
    const bool two = e0 + 1 < f + cnt;
    const zc* r0 = rt + (size_t)e0 * 4 * Q;
    const zc* r1 = two ? r0 + 4 * Q : r0;
    zc s[2][2];
    s[0][0] = s[0][1] = s[1][0] = s[1][1] = mk<double>(0, 0);
    for (int q = lane; q < Q; q += 32) {
      zc g[8];
#pragma unroll
      for (int k = 0; k < 8; k++) g[k] = sD[k * Q + q];
      zc a0[4], a1[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        a0[k] = ld_stream(r0 + k * Q + q, pol);
        a1[k] = ld_stream(r1 + k * Q + q, pol);
      }
      // rows: 0 a1 (medium 1 theta), 1 b1, 2 a2, 3 b2; items J: 0 a1, 1 a2, 4 b1, 5 b2; M: 2, 3, 6, 7
      s[0][0] = cfma_conj(a0[0], g[0], cfma_conj(a0[2], g[1], cfma_conj(a0[1], g[4], cfma_conj(a0[3], g[5], s[0][0]))));
      s[0][1] = cfma_conj(a0[0], g[2], cfma_conj(a0[2], g[3], cfma_conj(a0[1], g[6], cfma_conj(a0[3], g[7], s[0][1]))));
      s[1][0] = cfma_conj(a1[0], g[0], cfma_conj(a1[2], g[1], cfma_conj(a1[1], g[4], cfma_conj(a1[3], g[5], s[1][0]))));
      s[1][1] = cfma_conj(a1[0], g[2], cfma_conj(a1[2], g[3], cfma_conj(a1[1], g[6], cfma_conj(a1[3], g[7], s[1][1]))));
    }
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int k = 0; k < 2; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          s[j][k].re += __shfl_xor_sync(0xffffffffu, s[j][k].re, o);
          s[j][k].im += __shfl_xor_sync(0xffffffffu, s[j][k].im, o);
        }
    if (lane < 4) {
      const int j = lane >> 1, k = lane & 1;
      if (j == 0 || two) x[2 * (e0 + j) + k] += (j == 0) ? (k == 0 ? s[0][0] : s[0][1]) : (k == 0 ? s[1][0] : s[1][1]);
    }
  }
}

// y += Z_far^T x (FP64, internal layout); uses the one-vector level buffers C and D.
int far_matvec_adj64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st) {
  if (c->level_k)
    return fail(SIE_ERR_STATE, "transposed product: not available with per-level truncation numbers");
  const int Q = c->Q, L1 = c->l_max;
  Level& L = c->lv[L1];
  {
    dim3 g((Q + 127) / 128, L.nb);
    k_adj_in<<<g, 128, 0, st>>>(c->d_rt, c->d_box_first, c->d_box_cnt, Q, x, c->d_qperm, recv_const(c), L.C);
    sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  SIE_TRY(far_translate_t<double>(c, st, nullptr));
  k_adj_out<<<c->n_rchunk, 256, (size_t)8 * Q * sizeof(zc), st>>>(c->d_rt, (const int4*)c->d_rchunk, Q, L.D,
                                                                  c->d_qperm, y);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// Far part of the shape gradient.  With the leaf fields U (the folded D of the forward
// product on I, what the receive multiplies the patterns by) and C~ (the leaf
// coefficients of the transposed chain on conj(lambda), read at pi(q)):
//   lambda^H dZ_far I = sum_e [ sum_q dRT_e . (conj(lambda_e) U) + sum_q C~ . conj(dRT_e) I_e ].
// Block per (edge, vertex slot): the edge's 4 x Q patterns are differentiated by central
// differences with that vertex moved by +-h, and -2 Re(...) goes to grad[vertex].
__global__ void __launch_bounds__(256) k_grad_far(const SideV* __restrict__ sv, const FnD* __restrict__ fn,
                                                  const double* __restrict__ V, int normal_convention, double h,
                                                  Rule R, zc k1, zc k2, const double* khat, const double* tth,
                                                  const double* tph, const double* boxc, const int* edge_box,
                                                  int Q, const zc* __restrict__ U, const zc* __restrict__ Da,
                                                  const int* __restrict__ qperm, const zc* __restrict__ lam,
                                                  const zc* __restrict__ I, double* grad) {
  const int e = blockIdx.x, slot = blockIdx.y;
  const int v = edge_vertex(sv, e, slot);
  const int b = edge_box[e];
  const vd Rc = mkv<double>(boxc[3 * b], boxc[3 * b + 1], boxc[3 * b + 2]);
  FnD fp[2], fmn[2];
  for (int ll = 0; ll < 2; ll++) {
    fp[ll] = side_fn(sv[2 * e + ll], fn[2 * e + ll].sgn, V, normal_convention, v, h);
    fmn[ll] = side_fn(sv[2 * e + ll], fn[2 * e + ll].sgn, V, normal_convention, v, -h);
  }
  const zc lJ = conj(lam[2 * e]), lM = conj(lam[2 * e + 1]), iJ = I[2 * e], iM = I[2 * e + 1];
  const zc* Ub = U + (size_t)b * 8 * Q;
  const zc* Db = Da + (size_t)b * 8 * Q;
  const double inv = 0.5 / h;
  zc acc = mk<double>(0, 0);
  for (int q = threadIdx.x; q < Q; q += blockDim.x) {
    const vd kh = mkv<double>(khat[3 * q], khat[3 * q + 1], khat[3 * q + 2]);
    const vd th = mkv<double>(tth[3 * q], tth[3 * q + 1], tth[3 * q + 2]);
    const vd ph = mkv<double>(tph[3 * q], tph[3 * q + 1], tph[3 * q + 2]);
    zc rp[4], rm[4], d[4];
    rt_edge_q(fp[0], fp[1], Rc, kh, th, ph, R, k1, k2, rp);
    rt_edge_q(fmn[0], fmn[1], Rc, kh, th, ph, R, k1, k2, rm);
    for (int k = 0; k < 4; k++) d[k] = (rp[k] - rm[k]) * inv;
    // receive side: rows 2 md + ab against the folded U (index md * 4 + o * 2 + ab)
    for (int md = 0; md < 2; md++)
      for (int ab = 0; ab < 2; ab++)
        acc += d[2 * md + ab] * (lJ * Ub[(size_t)(md * 4 + ab) * Q + q] + lM * Ub[(size_t)(md * 4 + 2 + ab) * Q + q]);
    // aggregate side: items of C = sum conj(RT) x (0: a1 J, 1: a2 J, 2: a1 M, 3: a2 M,
    // 4: b1 J, 5: b2 J, 6: b1 M, 7: b2 M)
    const int qq = qperm[q];
    const zc c0 = Db[0 * (size_t)Q + qq], c1 = Db[1 * (size_t)Q + qq], c2 = Db[2 * (size_t)Q + qq],
             c3 = Db[3 * (size_t)Q + qq], c4 = Db[4 * (size_t)Q + qq], c5 = Db[5 * (size_t)Q + qq],
             c6 = Db[6 * (size_t)Q + qq], c7 = Db[7 * (size_t)Q + qq];
    acc += conj(d[0]) * (c0 * iJ + c2 * iM) + conj(d[2]) * (c1 * iJ + c3 * iM) +
           conj(d[1]) * (c4 * iJ + c6 * iM) + conj(d[3]) * (c5 * iJ + c7 * iM);
  }
  __shared__ double red[2][8];
  double re = acc.re;
  for (int o = 16; o > 0; o >>= 1) re += __shfl_xor_sync(0xffffffffu, re, o);
  if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = re;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[0][w];
    atomicAdd(grad + v, -2.0 * s);
  }
}

// D of the leaf level folded in place (recv_fold), one-vector layout [box][8][Q].
__global__ void k_fold_leaf(zc* D, int nb, int Q, RecvConst rc) {
  const int b = blockIdx.y, q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Q || b >= nb) return;
  zc* d = D + (size_t)b * 8 * Q + q;
  zc in[8], u[8];
  for (int i = 0; i < 8; i++) in[i] = d[(size_t)i * Q];
  recv_fold(in, rc, u, q, Q);
  for (int i = 0; i < 8; i++) d[(size_t)i * Q] = u[i];
}

__global__ void k_conj_copy(const zc* a, zc* b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = conj(a[i]);
}

// ws: 2 x (leaf boxes x 8 x Q) + 2M complex128.
int grad_far(sie_ctx* c, const zc* lam, const zc* I, double h, double* grad, void* ws, cudaStream_t st) {
  if (c->level_k) return fail(SIE_ERR_STATE, "shape gradient: not available with per-level truncation numbers");
  const int Q = c->Q, L1 = c->l_max;
  Level& L = c->lv[L1];
  const size_t nl = (size_t)L.nb * 8 * Q;
  zc* U = (zc*)ws;
  zc* Da = U + nl;
  zc* lc = Da + nl;
  const RecvConst rc = recv_const(c);
  // forward: leaf D of the product on I, folded
  {
    dim3 g((Q + 31) / 32, L.nb);
    k_aggregate_eg<double><<<g, 256, 0, st>>>(c->d_rt, c->d_box_first, c->d_box_cnt, Q, I, L.C);
    sie::count_launch();
    SIE_TRY(far_translate_t<double>(c, st, nullptr));
    SIE_CUDA(cudaMemcpyAsync(U, L.D, nl * sizeof(zc), cudaMemcpyDeviceToDevice, st));
    k_fold_leaf<<<dim3((Q + 127) / 128, L.nb), 128, 0, st>>>(U, L.nb, Q, rc);
    sie::count_launch();
  }
  // transposed chain on conj(lambda)
  {
    k_conj_copy<<<296, 256, 0, st>>>(lam, lc, (size_t)2 * c->M);
    sie::count_launch();
    dim3 g((Q + 127) / 128, L.nb);
    k_adj_in<<<g, 128, 0, st>>>(c->d_rt, c->d_box_first, c->d_box_cnt, Q, lc, c->d_qperm, rc, L.C);
    sie::count_launch();
    SIE_TRY(far_translate_t<double>(c, st, nullptr));
    SIE_CUDA(cudaMemcpyAsync(Da, L.D, nl * sizeof(zc), cudaMemcpyDeviceToDevice, st));
  }
  k_grad_far<<<dim3(c->M, 4), 256, 0, st>>>((const SideV*)c->d_side, c->d_fn, c->d_vert, c->cfg.normal_convention,
                                            h, c->R, c->mt.k1, c->mt.k2, c->d_khat, c->d_tth, c->d_tph, c->d_boxc,
                                            c->d_edge_box, Q, U, Da, c->d_qperm, lam, I, grad);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int far_matvec64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st, cudaEvent_t* ev,
                 cudaEvent_t wait_recv, const std::function<int()>* after_agg) {
  return far_matvec_t<double>(c, c->d_rt, x, y, st, ev, wait_recv, after_agg);
}

int far_matvec32(sie_ctx* c, const cc* x, cc* y, cudaStream_t st, cudaEvent_t* ev,
                 cudaEvent_t wait_recv, const std::function<int()>* after_agg) {
  return far_matvec_t<float>(c, c->d_rt32, x, y, st, ev, wait_recv, after_agg);
}

// Batched coefficient buffers of every level, grown to R vectors of type T.
template <typename T>
static int ensure_batch_coeffs(sie_ctx* c, int R) {
  for (int l = c->l_min; l <= c->l_max; l++) {
    Level& L = c->lv[l];
    size_t need = (size_t)L.nb * 8 * R * L.Q * sizeof(cx<T>);
    if (L.cdb_bytes >= need) continue;
    if (L.Cb) cudaFree(L.Cb);
    if (L.Db) cudaFree(L.Db);
    L.Cb = L.Db = nullptr;
    L.cdb_bytes = 0;
    SIE_CUDA(cudaMalloc(&L.Cb, need));
    SIE_CUDA(cudaMalloc(&L.Db, need));
    L.cdb_bytes = need;
  }
  return SIE_OK;
}

template <typename T>
static int far_matvec_b_t(sie_ctx* c, const cx<T>* rt, const cx<T>* x, cx<T>* y, int R,
                          cudaStream_t st, cudaEvent_t wait_recv, const std::function<int()>* after_agg) {
  if (R < 1 || R > SIE_BATCH_MAX) return fail(SIE_ERR_ARG, "batched far product: bad batch size");
  SIE_TRY(ensure_batch_coeffs<T>(c, R));
  const int Q = c->Q, L0 = c->l_min, L1 = c->l_max, M = c->M;
  const bool k2c = c->mt.k2.im != 0.0;
  const int thr = 128;
  {
    Level& L = c->lv[L1];
    dim3 g((Q + 31) / 32, L.nb);
    if (R <= 8)
      k_agg_b<T, 1><<<g, 256, 0, st>>>(rt, c->d_box_first, c->d_box_cnt, Q, x, M, R, (cx<T>*)L.Cb);
    else
      k_agg_b<T, 2><<<g, 256, 0, st>>>(rt, c->d_box_first, c->d_box_cnt, Q, x, M, R, (cx<T>*)L.Cb);
    sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  if (after_agg) SIE_TRY((*after_agg)());
  // the batch layout [box][r][8][Q] is nb * R blocks of [8][Q] for the interpolation
  for (int l = L1 - 1; l >= L0; l--) {
    Level& P = c->lv[l];
    Level& Ch = c->lv[l + 1];
    const int Qp = P.Q;
    const cx<T>* src = (const cx<T>*)Ch.Cb;
    if (Ch.Q != Qp) {
      void* tmp = nullptr;
      SIE_TRY(lvtmp(c, (size_t)Ch.nb * R * 8 * Qp * sizeof(cx<T>), &tmp));
      SIE_TRY(interp_run<T>(P.up, src, Ch.Q, (cx<T>*)tmp, (size_t)Ch.nb * R, false, st));
      src = (const cx<T>*)tmp;
    }
    dim3 g((Qp + thr - 1) / thr, P.nb, R);
    k_ss_b<T><<<g, thr, 0, st>>>(src, P.ch_ptr, P.ch_idx, P.ch_oct, php_up<T>(Ch), Qp,
                                 k2c ? 1 : 2, R, (cx<T>*)P.Cb); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  for (int l = L0; l <= L1; l++) {
    Level& L = c->lv[l];
    const int Ql = L.Q;
    if (L.nb >= (1 << 22)) return fail(SIE_ERR_ARG, "batched far product: too many boxes on a level");
    const unsigned gx = (Ql + SRW_QT - 1) / SRW_QT, gy = (L.ngrp + SRW_GB - 1) / SRW_GB;
    const int nmed = L.only_k1 ? 1 : 2;
    for (int md = 0; md < nmed; md++) {
      // two vectors per source read in FP32; one in FP64, whose accumulators are twice as wide
      bool done = false;
      if constexpr (sizeof(T) == 4) {
        if (R % 2 == 0) {
          k_sr_ns_b<T, 2><<<dim3(gx, gy, R / 2), 32 * SRW_GB, sr_warp_ns_smem<T>(), st>>>(
              (const cx<T>*)L.Cb, L.grp_sib, L.grp_src, L.ngrp, tlp<T>(L), trfp<T>(L), Ql, md, nmed == 1, R,
              (cx<T>*)L.Db);
          done = true;
        }
      }
      if (!done)
        k_sr_ns_b<T, 1><<<dim3(gx, gy, R), 32 * SRW_GB, sr_warp_ns_smem<T>(), st>>>(
            (const cx<T>*)L.Cb, L.grp_sib, L.grp_src, L.ngrp, tlp<T>(L), trfp<T>(L), Ql, md, nmed == 1, R,
            (cx<T>*)L.Db);
      sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
  }
  // RR down to the leaves; the leaf level's kernel also folds D for the receive (with a
  // single level there is no RR, and the same kernel only folds: every parent is absent).
  // A child level with a smaller sampling takes the parent's D shifted on the parent's
  // sampling and anterpolated; the leaf level's fold then runs as a pass of its own.
  const RecvConst rcn = recv_const(c);
  for (int l = (L1 > L0 ? L0 + 1 : L1); l <= L1; l++) {
    Level& L = c->lv[l];
    Level& P = c->lv[l > L0 ? l - 1 : l];
    if (l > L0 && L.Q != P.Q) {
      const int Qp = P.Q;
      void* tmp = nullptr;
      const size_t n = (size_t)L.nb * R * 8 * Qp;
      SIE_TRY(lvtmp(c, n * sizeof(cx<T>), &tmp));
      SIE_CUDA(cudaMemsetAsync(tmp, 0, n * sizeof(cx<T>), st));
      dim3 g((Qp + thr - 1) / thr, L.nb, R);
      k_rr_b<T><<<g, thr, 0, st>>>((const cx<T>*)P.Db, L.parent, L.oct, php_dn<T>(L), Qp, k2c ? 1 : 2, R, 0,
                                   rcn, (cx<T>*)tmp); sie::count_launch();
      SIE_CUDA(cudaGetLastError());
      SIE_TRY(interp_run<T>(P.dn, (const cx<T>*)tmp, Qp, (cx<T>*)L.Db, (size_t)L.nb * R, true, st));
      if (l == L1) {  // fold only: no medium is shifted
        dim3 gf((L.Q + thr - 1) / thr, L.nb, R);
        k_rr_b<T><<<gf, thr, 0, st>>>((const cx<T>*)P.Db, L.parent, L.oct, php_dn<T>(L), L.Q, 0, R, 1, rcn,
                                      (cx<T>*)L.Db); sie::count_launch();
        SIE_CUDA(cudaGetLastError());
      }
      continue;
    }
    dim3 g((L.Q + thr - 1) / thr, L.nb, R);
    k_rr_b<T><<<g, thr, 0, st>>>((const cx<T>*)P.Db, L.parent, L.oct, php_dn<T>(L), L.Q, k2c ? 1 : 2, R,
                                 l == L1, rcn, (cx<T>*)L.Db); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  // the receive adds into y, which the near product (possibly on another stream) writes
  if (wait_recv) SIE_CUDA(cudaStreamWaitEvent(st, wait_recv, 0));
  {
    Level& L = c->lv[L1];
    k_recv_g<T><<<c->n_rchunk, 256, recv_g_smem<T>(), st>>>(rt, (const int4*)c->d_rchunk, (const cx<T>*)L.Db,
                                                             Q, M, R, y);
    sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  return SIE_OK;
}

int far_matvec_b64(sie_ctx* c, const zc* x, zc* y, int R, cudaStream_t st, cudaEvent_t wait_recv,
                   const std::function<int()>* after_agg) {
  return far_matvec_b_t<double>(c, c->d_rt, x, y, R, st, wait_recv, after_agg);
}

int far_matvec_b32(sie_ctx* c, const cc* x, cc* y, int R, cudaStream_t st, cudaEvent_t wait_recv,
                   const std::function<int()>* after_agg) {
  return far_matvec_b_t<float>(c, c->d_rt32, x, y, R, st, wait_recv, after_agg);
}

__global__ void k_trf_f32(const double* a, float* b, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// complex64 copies of everything the FP32 product reads (once per context).  The
// coefficient buffers C and D of every level are shared with the FP64 product: a
// complex64 pass uses the first half of each.
int make_f32_tables(sie_ctx* c) {
  if (c->f32_ready) return SIE_OK;
  cudaStream_t st = c->stream;
  size_t nnz = (size_t)std::max<long long>(c->near.nnz, 1);
  SIE_CUDA(cudaMalloc(&c->d_na32, nnz * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_nb32, nnz * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_nd32, nnz * sizeof(cc)));
  SIE_TRY(near_to_f32(c));
  if (!c->cfg.dense) {
    int Q = c->Q;
    size_t nrt = (size_t)c->M * 4 * Q;
    SIE_CUDA(cudaMalloc(&c->d_rt32, nrt * sizeof(cc)));
    SIE_TRY(to_c64(c->d_rt, c->d_rt32, nrt, st));
    SIE_CUDA(cudaMalloc(&c->d_trf32, (size_t)Q * sizeof(float)));
    k_trf_f32<<<(Q + 255) / 256, 256, 0, st>>>(c->d_trf, c->d_trf32, Q); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
    for (int l = c->l_min; l <= c->l_max; l++) {
      Level& L = c->lv[l];
      const int Qs = c->lv[l > c->l_min ? l - 1 : l].Q;  // the shift tables' (parent) sampling
      size_t ntl = (size_t)343 * 2 * L.Q, nph = (size_t)8 * 2 * Qs;
      SIE_CUDA(cudaMalloc(&L.tl32, ntl * sizeof(cc)));
      SIE_CUDA(cudaMalloc(&L.ph_up32, nph * sizeof(cc)));
      SIE_CUDA(cudaMalloc(&L.ph_dn32, nph * sizeof(cc)));
      SIE_TRY(to_c64(L.tl, L.tl32, ntl, st));
      SIE_TRY(to_c64(L.ph_up, L.ph_up32, nph, st));
      SIE_TRY(to_c64(L.ph_dn, L.ph_dn32, nph, st));
      SIE_CUDA(cudaMalloc(&L.trf32, (size_t)L.Q * sizeof(float)));
      k_trf_f32<<<(L.Q + 255) / 256, 256, 0, st>>>(L.trf, L.trf32, L.Q); sie::count_launch();
      for (InterpDev* I : {&L.up, &L.dn})
        if (I->nnz > 0) {
          SIE_CUDA(cudaMalloc(&I->val32, (size_t)I->nnz * sizeof(float)));
          k_trf_f32<<<(unsigned)((I->nnz + 255) / 256), 256, 0, st>>>(I->val, I->val32, (int)I->nnz);
          sie::count_launch();
          const int ne = I->ew * I->rows;
          SIE_CUDA(cudaMalloc(&I->eval32, (size_t)std::max(ne, 1) * sizeof(float)));
          if (ne > 0) {
            k_trf_f32<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(I->eval, I->eval32, ne);
            sie::count_launch();
          }
          SIE_CUDA(cudaMalloc(&I->oval32, (size_t)I->onnz * sizeof(float)));
          k_trf_f32<<<(unsigned)((I->onnz + 255) / 256), 256, 0, st>>>(I->oval, I->oval32, (int)I->onnz);
          sie::count_launch();
        }
      SIE_CUDA(cudaGetLastError());
    }
  }
  size_t n = (size_t)2 * c->M;
  SIE_CUDA(cudaMalloc(&c->d_xi32, n * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_yi32, n * sizeof(cc)));
  SIE_CUDA(cudaStreamSynchronize(st));
  c->f32_ready = true;
  return SIE_OK;
}

int far_prepare_kernels(sie_ctx* c) {
  size_t smem64 = (size_t)8 * c->Q * sizeof(zc);
  size_t smem32 = (size_t)8 * c->Q * sizeof(cc);
  SIE_CUDA(raise_smem(k_receive<double>,
                                (int)smem64));
  SIE_CUDA(raise_smem(k_receive<float>,
                                (int)smem32));
  SIE_CUDA(raise_smem(k_receive_chunk<double>,
                                (int)smem64));
  SIE_CUDA(raise_smem(k_receive_chunk<float>,
                                (int)smem32));
  size_t sr64 = (size_t)343 * SR_TQ * sizeof(zc) + (size_t)SR_GB * (216 + 8) * sizeof(int);
  size_t sr32 = (size_t)343 * SR_TQ * sizeof(cc) + (size_t)SR_GB * (216 + 8) * sizeof(int);
  SIE_CUDA(raise_smem(k_sr_group_tl<double>,
                                (int)sr64));
  SIE_CUDA(raise_smem(k_sr_group_tl<float>,
                                (int)sr32));
  SIE_CUDA(raise_smem(k_sr_warp<double>,
                                (int)sr_warp_smem<double>()));
  SIE_CUDA(raise_smem(k_sr_warp<float>,
                                (int)sr_warp_smem<float>()));
  SIE_CUDA(raise_smem(k_sr_warp_bf<double>,
                                (int)sr_warp_bf_smem<double>()));
  SIE_CUDA(raise_smem(k_sr_warp_ns<double, 1, 3>, sr_warp_ns_smem<double>()));
  SIE_CUDA(raise_smem(k_sr_warp_ns<float, 1>,
                                (int)sr_warp_ns_smem<float>()));
  SIE_CUDA(raise_smem(k_sr_warp_bf<float>,
                                (int)sr_warp_bf_smem<float>()));
  SIE_CUDA(raise_smem(k_sr_ns_b<double, 1>, sr_warp_ns_smem<double>()));
  SIE_CUDA(raise_smem(k_sr_ns_b<float, 1>, sr_warp_ns_smem<float>()));
  SIE_CUDA(raise_smem(k_sr_ns_b<float, 2>, sr_warp_ns_smem<float>()));
  SIE_CUDA(raise_smem(k_recv_g<double>, recv_g_smem<double>()));
  SIE_CUDA(raise_smem(k_adj_out, (size_t)8 * c->Q * sizeof(zc)));
  SIE_CUDA(raise_smem(k_recv_g<float>, recv_g_smem<float>()));
  return SIE_OK;
}

}  // namespace sie
