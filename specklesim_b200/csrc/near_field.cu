// Near-field impedance fill (FP64) and the near-field block-panel matvec.
//
// Math follows lib_sie_get_impedance_edges and the integration routines of
// src/lib_sie_tri_calculation_mod.f90 (cited per function).  Only the Kt and Tt
// operators enter ICTF (:1876-1919) and PMCHWT (:1713-1769), so Kn/Tn (and
// with them IT_bn and the :2142 bracket) are not evaluated here.
#include <cub/cub.cuh>

#include "sie_internal.h"
#include "geom.cuh"

namespace sie {

__device__ __forceinline__ vd ldv(const double* p) { return mkv<double>(p[0], p[1], p[2]); }
__device__ __forceinline__ double f32(double x) { return (double)(float)x; }

__device__ __forceinline__ vd simplex(double a, double b, const FnD& f) {
  double w0 = 1 - a - b;
  return mkv<double>(w0 * f.c[0] + a * f.c[3] + b * f.c[6], w0 * f.c[1] + a * f.c[4] + b * f.c[7],
                     w0 * f.c[2] + a * f.c[5] + b * f.c[8]);
}

// Diver_Green (:1421-1432): G = e^{-ikR}/(4 pi R), DG = -(1+ikR) e^{-ikR}/(4 pi R^2)
__device__ __forceinline__ void green(zc k, double R, zc& G, zc& DG) {
  zc e = cexp_mik(k, R);
  zc ikR = mk<double>(-k.im * R, k.re * R);
  double inv = 1.0 / (4 * PI * R);
  G = e * inv;
  DG = -((mk<double>(1.0, 0.0) + ikR) * e) * (inv / R);
}
// Diver_Green_s (:1435-1451), smoothed kernel
__device__ __forceinline__ void green_s(zc k, double R, zc& Gs, zc& DGs) {
  zc k2 = k * k;
  if (R == 0.0) {
    Gs = mk<double>(k.im / (4 * PI), -k.re / (4 * PI));  // -i k / (4 pi)
    DGs = k2 * (1.0 / (8 * PI));
    return;
  }
  zc e = cexp_mik(k, R);
  zc ikR = mk<double>(-k.im * R, k.re * R);
  Gs = (e - mk<double>(1.0, 0.0)) * (1.0 / (4 * PI * R)) + k2 * (R / (8 * PI));
  DGs = (mk<double>(1.0, 0.0) - (mk<double>(1.0, 0.0) + ikR) * e) * (1.0 / (4 * PI * R * R)) +
        k2 * (1.0 / (8 * PI));
}

// Iq_L (:1074-1119) for q = -1, 1, 3 at once.
__device__ void iq_line(vd Ra, vd p1, vd p2, double& n1, double& p1o, double& p3o) {
  vd d = p2 - p1;
  vd s = d / vlen(d);
  double Sp = dot(p2 - Ra, s);
  double Sn = dot(p1 - Ra, s);
  double Rn = vlen(Ra - p1);
  double Rp = vlen(Ra - p2);
  double Sum_p = Rp + Sp, Sum_n = Rn + Sn, Dif_p = Rp - Sp, Dif_n = Rn - Sn;
  double R0 = sqrt(Rp * Rp - Sp * Sp);
  double il;
  if (R0 == 0.0)
    il = log(Sp / Sn);
  else if (fabs(Dif_p) > fabs(Sum_n))
    il = log(Dif_n / Dif_p);
  else
    il = log(Sum_p / Sum_n);
  double ilp1 = 0.5 * R0 * R0 * il + 0.5 * (Sp * Rp - Sn * Rn);
  n1 = il;
  p1o = ilp1;
  p3o = 0.75 * R0 * R0 * ilp1 + 0.25 * (Sp * Rp * Rp * Rp - Sn * Rn * Rn * Rn);
}

// Analytic parts of the singular inner integral for one observation point:
// Iq_s (:1256-1331), K2q (:1333-1364), K3q (:1397-1419), K4q (:1366-1395).
struct HannOut {
  double Is_n1, Is_p1;  // Iq_s(-1), Iq_s(1) (self: Iq_s(1) = 0)
  vd K2n1, K2p1, K4n1, K4p1;
};

__device__ void hanninen(vd Ra, const FnD& f, bool self, HannOut& o) {
  vd c0 = ldv(f.c), c1 = ldv(f.c + 3), c2 = ldv(f.c + 6);
  vd nq = ldv(f.nq), mid = ldv(f.mid);
  vd a0 = (c0 - Ra) / vlen(c0 - Ra);
  vd a1 = (c1 - Ra) / vlen(c1 - Ra);
  vd a2 = (c2 - Ra) / vlen(c2 - Ra);
  double x = 1 + dot(a0, a1) + dot(a0, a2) + dot(a1, a2);
  double y = fabs(dot(a0, cross(a1, a2)));
  double Om = 2 * atan2(y, x);
  double h = dot(nq, Ra - mid);
  double Is_n3 = 0.0;
  if (h != 0.0 && !self && Om <= PI && Om > -PI) Is_n3 = -1 / h * Om;
  vd m[3];
  {
    vd t0 = cross(nq, c2 - c1);
    m[0] = t0 / vlen(t0);
    vd t1 = cross(nq, c0 - c2);
    m[1] = t1 / vlen(t1);
    vd t2 = cross(nq, c1 - c0);
    m[2] = t2 / vlen(t2);
  }
  // edge_vectors_assigned (:2706-2717): (ps, pt) = (c2,c1), (c0,c2), (c1,c0)
  vd ps[3] = {c2, c0, c1};
  vd pt[3] = {c1, c2, c0};
  double sumA_n1 = 0, sumA_p1 = 0;
  vd sB_n1 = mkv<double>(0, 0, 0), sB_p1 = sB_n1, sB_p3 = sB_n1;
  for (int i = 0; i < 3; i++) {
    double tv = dot(m[i], Ra - (pt[i] + ps[i]) / 2.0);
    double n1, p1, p3;
    iq_line(Ra, pt[i], ps[i], n1, p1, p3);  // Iq_s uses (p_t, p_s)
    sumA_n1 += tv * n1;
    sumA_p1 += tv * p1;
    iq_line(Ra, ps[i], pt[i], n1, p1, p3);  // K2q/K3q/K4q use (p_s, p_t)
    sB_n1 = sB_n1 + m[i] * n1;
    sB_p1 = sB_p1 + m[i] * p1;
    sB_p3 = sB_p3 + m[i] * p3;
  }
  double Is_n1 = 1.0 * (-1 * h * h * Is_n3 - sumA_n1);
  double Is_p1 = (double)(1.0f / 3.0f) * (1 * h * h * Is_n1 - sumA_p1);
  double Iqs_m3 = Is_n3;                   // Iq_s(-3)
  double Iqs_m1 = Is_n1;                   // Iq_s(-1)
  double Iqs_p1 = self ? 0.0 : Is_p1;      // Iq_s(1)
  o.Is_n1 = Iqs_m1;
  o.Is_p1 = Iqs_p1;
  vd rho = Ra - nq * h;
  o.K2n1 = (sB_p1 * 1.0 + (rho - c2) * Iqs_m1) * (f.df * 0.5);
  o.K2p1 = (sB_p3 * (double)(1.0f / 3.0f) + (rho - c2) * Iqs_p1) * (f.df * 0.5);
  if (self) {
    o.K4n1 = mkv<double>(0, 0, 0);
    o.K4p1 = o.K4n1;
  } else {
    vd K3n1 = sB_n1 - nq * (h * (-1.0)) * Iqs_m3;
    vd K3p1 = sB_p1 - nq * (h * 1.0) * Iqs_m1;
    o.K4n1 = cross(Ra - c2, K3n1) * (-f.df * 0.5);
    o.K4p1 = cross(Ra - c2, K3p1) * (-f.df * 0.5);
  }
}

struct KT {
  zc Kt[2], Tt[2];
};

// tri_outer_integration (:2255-2302), Kt and Tt for both media.
__device__ KT outer_regular(const FnD& fm, const FnD& fn, const FillArgs& A) {
  KT r;
  zc kk[2] = {A.mt.k1, A.mt.k2};
  for (int md = 0; md < 2; md++) r.Kt[md] = r.Tt[md] = mk<double>(0, 0);
  double xnt = 0;
  vd vm = ldv(fm.c + 6), vn = ldv(fn.c + 6), nqm = ldv(fm.nq);
  for (int j = 0; j < A.R.n; j++) {
    vd ra = simplex(A.R.a[j], A.R.b[j], fm);
    vd rfm = (ra - vm) * 0.5 * fm.df;
    vd rfa = (ra - vn) * 0.5 * fn.df;
    double trf = A.R.w[j] * fm.area;
    zc IK[2][3], ITa[2][3], ITbt[2];
    for (int md = 0; md < 2; md++) {
      for (int d = 0; d < 3; d++) IK[md][d] = ITa[md][d] = mk<double>(0, 0);
      ITbt[md] = mk<double>(0, 0);
    }
    for (int i = 0; i < A.R.n; i++) {
      vd rq = simplex(A.R.a[i], A.R.b[i], fn);
      vd rfn = (rq - vn) * 0.5 * fn.df;
      vd Rv = ra - rq;
      double Rl = vlen(Rv);
      vd Rn = Rv / Rl;
      vd cr = cross(rfn, Rn);
      double tr = A.R.w[i] * fn.area;
      for (int md = 0; md < 2; md++) {
        zc G, DG;
        green(kk[md], Rl, G, DG);
        zc dgt = DG * tr, gt = G * tr;
        IK[md][0] += dgt * cr.x;
        IK[md][1] += dgt * cr.y;
        IK[md][2] += dgt * cr.z;
        ITa[md][0] += gt * rfn.x;
        ITa[md][1] += gt * rfn.y;
        ITa[md][2] += gt * rfn.z;
        ITbt[md] += gt * fn.df;
      }
    }
    for (int md = 0; md < 2; md++) {
      zc k = kk[md];
      zc kdotIK = IK[md][0] * rfm.x + IK[md][1] * rfm.y + IK[md][2] * rfm.z;
      zc rITa = ITa[md][0] * rfm.x + ITa[md][1] * rfm.y + ITa[md][2] * rfm.z;
      r.Kt[md] += kdotIK * trf;
      zc ts = (mk<double>(1.0, 0.0) / k) * ITbt[md] * fm.df;
      zc in = k * rITa - ts;
      r.Tt[md] += mk<double>(-in.im * trf, in.re * trf);  // i*trf*(...)
    }
    xnt -= dot(cross(nqm, rfm), rfa) * trf;
  }
  double xf = A.smooth ? xnt : f32(xnt);  // cmplx(x_nt, 0.0) is binary32
  r.Kt[0] += mk<double>(-0.5 * xf, 0.0);
  r.Kt[1] += mk<double>(0.5 * xf, 0.0);
  return r;
}

// tri_outer_integration_singular (:2199-2253) with the smooth part
// (:2071-2107) and the analytic part (:2109-2145), Kt and Tt for both media.
__device__ KT outer_singular(const FnD& fm, const FnD& fn, bool self, const FillArgs& A) {
  KT r;
  zc kk[2] = {A.mt.k1, A.mt.k2};
  for (int md = 0; md < 2; md++) r.Kt[md] = r.Tt[md] = mk<double>(0, 0);
  double xnt = 0;
  vd vm = ldv(fm.c + 6), vn = ldv(fn.c + 6), nqm = ldv(fm.nq);
  const double c4 = 1 / (4 * PI), c8 = 1 / (8 * PI);
  for (int j = 0; j < A.R.n; j++) {
    vd ra = simplex(A.R.a[j], A.R.b[j], fm);
    vd rfm = (ra - vm) * 0.5 * fm.df;
    vd rfa = (ra - vn) * 0.5 * fn.df;
    double trf = A.R.w[j] * fm.area;
    HannOut H;
    hanninen(ra, fn, self, H);
    zc IK[2][3], ITa[2][3], ITbt[2];
    for (int md = 0; md < 2; md++) {
      zc k2 = kk[md] * kk[md];
      zc m8 = k2 * (-c8);
      // singular part
      if (self) {
        IK[md][0] = IK[md][1] = IK[md][2] = mk<double>(0, 0);
      } else {
        IK[md][0] = mk<double>(c4 * H.K4n1.x, 0) + m8 * H.K4p1.x;
        IK[md][1] = mk<double>(c4 * H.K4n1.y, 0) + m8 * H.K4p1.y;
        IK[md][2] = mk<double>(c4 * H.K4n1.z, 0) + m8 * H.K4p1.z;
      }
      ITa[md][0] = mk<double>(c4 * H.K2n1.x, 0) + m8 * H.K2p1.x;
      ITa[md][1] = mk<double>(c4 * H.K2n1.y, 0) + m8 * H.K2p1.y;
      ITa[md][2] = mk<double>(c4 * H.K2n1.z, 0) + m8 * H.K2p1.z;
      ITbt[md] = mk<double>(fn.df * c4 * H.Is_n1, 0) - k2 * (fn.df * c8 * H.Is_p1);
    }
    // smooth part
    for (int i = 0; i < A.R.n; i++) {
      vd rq = simplex(A.R.a[i], A.R.b[i], fn);
      vd rfn = (rq - vn) * 0.5 * fn.df;
      vd Rv = ra - rq;
      double Rl = vlen(Rv);
      double tr = A.R.w[i] * fn.area;
      vd cr = mkv<double>(0, 0, 0);
      if (!self) cr = cross(rfn, Rv / Rl);
      for (int md = 0; md < 2; md++) {
        zc Gs, DGs;
        green_s(kk[md], Rl, Gs, DGs);
        zc gt = Gs * tr;
        if (!self) {
          zc dgt = DGs * tr;
          IK[md][0] += dgt * cr.x;
          IK[md][1] += dgt * cr.y;
          IK[md][2] += dgt * cr.z;
        }
        ITa[md][0] += gt * rfn.x;
        ITa[md][1] += gt * rfn.y;
        ITa[md][2] += gt * rfn.z;
        ITbt[md] += gt * fn.df;
      }
    }
    for (int md = 0; md < 2; md++) {
      zc k = kk[md];
      zc kdotIK = IK[md][0] * rfm.x + IK[md][1] * rfm.y + IK[md][2] * rfm.z;
      zc rITa = ITa[md][0] * rfm.x + ITa[md][1] * rfm.y + ITa[md][2] * rfm.z;
      r.Kt[md] += kdotIK * trf;
      zc ts = (mk<double>(1.0, 0.0) / k) * ITbt[md] * fm.df;
      zc in = k * rITa - ts;
      r.Tt[md] += mk<double>(-in.im * trf, in.re * trf);
    }
    xnt -= dot(cross(nqm, rfm), rfa) * trf;
  }
  double xf = A.smooth ? xnt : f32(xnt);
  r.Kt[0] += mk<double>(-0.5 * xf, 0.0);
  r.Kt[1] += mk<double>(0.5 * xf, 0.0);
  return r;
}

// tri_outer_integration_edge_adjacent (:2165-2197), PMCHWT only: Kt with a
// 12-point rule on both triangles.
__device__ zc outer_edge_adjacent(const FnD& fm, const FnD& fn, int md, zc k, bool smooth) {
  const float ra12[12] = {0.249286745170910f, 0.249286745170910f, 0.501426509658180f,
                          0.063089014491500f, 0.063089014491500f, 0.873821971017000f,
                          0.310352451033780f, 0.636502499121400f, 0.053145049844820f,
                          0.636502499121400f, 0.310352451033780f, 0.053145049844820f};
  const float rb12[12] = {0.249286745170910f, 0.501426509658180f, 0.249286745170910f,
                          0.063089014491500f, 0.873821971017000f, 0.063089014491500f,
                          0.636502499121400f, 0.053145049844820f, 0.310352451033780f,
                          0.310352451033780f, 0.053145049844820f, 0.636502499121400f};
  const float rw12[12] = {0.116786275726380f, 0.116786275726380f, 0.116786275726380f,
                          0.0508449063702100f, 0.0508449063702100f, 0.0508449063702100f,
                          0.0828510756183700f, 0.0828510756183700f, 0.0828510756183700f,
                          0.0828510756183700f, 0.0828510756183700f, 0.0828510756183700f};
  zc Kt = mk<double>(0, 0);
  double xnt = 0;
  vd vm = ldv(fm.c + 6), vn = ldv(fn.c + 6), nqm = ldv(fm.nq);
  for (int j = 0; j < 12; j++) {
    vd ra = simplex(ra12[j], rb12[j], fm);
    vd rfm = (ra - vm) * 0.5 * fm.df;
    vd rfa = (ra - vn) * 0.5 * fn.df;
    double trf = (double)rw12[j] * fm.area;
    zc Ik[3] = {mk<double>(0, 0), mk<double>(0, 0), mk<double>(0, 0)};
    for (int i = 0; i < 12; i++) {
      vd rq = simplex(ra12[i], rb12[i], fn);
      vd rfq = (rq - vn) * 0.5 * fn.df;
      vd Rv = ra - rq;
      double Rl = vlen(Rv);
      zc G, DG;
      green(k, Rl, G, DG);
      vd cr = cross(rfq, Rv / Rl);
      zc t = DG * ((double)rw12[i] * fn.area);
      Ik[0] += t * cr.x;
      Ik[1] += t * cr.y;
      Ik[2] += t * cr.z;
    }
    Kt += (Ik[0] * rfm.x + Ik[1] * rfm.y + Ik[2] * rfm.z) * trf;
    xnt -= dot(rfa, cross(nqm, rfm)) * trf;
  }
  double xf = smooth ? xnt : f32(xnt);
  return Kt + mk<double>((md == 1 ? -0.5 : 0.5) * xf, 0.0);
}

// zz of one (t, s) triangle pair (ICTF :1876-1919 / PMCHWT :1713-1769)
__device__ __forceinline__ void combine(const KT& r, const FillArgs& A, zc& a, zc& b, zc& d) {
  const Material& m = A.mt;
  zc Kt = r.Kt[0] + r.Kt[1];
  if (A.formulation == SIE_PMCHWT) {
    a += m.eta1 * r.Tt[0] + m.eta2 * r.Tt[1];
    b += -Kt;
    d += r.Tt[0] / m.eta1 + r.Tt[1] / m.eta2;
  } else {
    a += (m.eta1 * r.Tt[0] + m.eta2 * r.Tt[1]) / m.eta_a;
    b += -(Kt / m.eta_a);
    d += (r.Tt[0] / m.eta1 + r.Tt[1] / m.eta2) * m.eta_a;
  }
}

__device__ __forceinline__ bool pair_singular(int m, int n, int t, int s, const FillArgs& A,
                                              int& p, int& q) {
  p = A.fn[2 * m + t].tri;
  q = A.fn[2 * n + s].tri;
  const double* cp = A.cent + 3 * p;
  const double* cq = A.cent + 3 * q;
  double dx = cp[0] - cq[0], dy = cp[1] - cq[1], dz = cp[2] - cq[2];
  double r_ob = sqrt(dx * dx + dy * dy + dz * dz);
  return !(r_ob > 1.5 * A.rref[m]);
}

// Singular (t, s) term of triangles p, q with the sides given explicitly.
__device__ KT singular_pair_f(const FnD& fm, const FnD& fn, int p, int q, const FillArgs& A,
                              const int* tri_verts) {
  bool self = (p == q);
  KT r = outer_singular(fm, fn, self, A);
  if (A.formulation == SIE_PMCHWT && !self) {
    int cnt = 0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) cnt += (tri_verts[3 * p + a] == tri_verts[3 * q + b]);
    if (cnt == 2) {
      r.Kt[0] = outer_edge_adjacent(fm, fn, 1, A.mt.k1, A.smooth);
      r.Kt[1] = outer_edge_adjacent(fm, fn, 2, A.mt.k2, A.smooth);
    }
  }
  return r;
}

__device__ KT singular_pair(int m, int n, int t, int s, int p, int q, const FillArgs& A,
                            const int* tri_verts) {
  return singular_pair_f(A.fn[2 * m + t], A.fn[2 * n + s], p, q, A, tri_verts);
}

// -------------------------------------------------------------------------
// Panel indexing: flat block index -> (box A, row, column) -> (m, n) internal.
struct PanelArgs {
  int nbox;
  const long long* base;   // nbox + 1
  const int* box_first;
  const int* box_cnt;
  const int* nbr_ptr;
  const int* nbr_box;
  const int* ncols;
};

__device__ __forceinline__ void panel_mn(long long idx, const PanelArgs& P, int& m, int& n, int& A) {
  int lo = 0, hi = P.nbox - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (P.base[mid] <= idx) lo = mid;
    else hi = mid - 1;
  }
  A = lo;
  long long off = idx - P.base[A];
  int nc = P.ncols[A];
  int row = (int)(off / nc);
  int col = (int)(off - (long long)row * nc);
  m = P.box_first[A] + row;
  for (int k = P.nbr_ptr[A]; k < P.nbr_ptr[A + 1]; k++) {
    int B = P.nbr_box[k];
    int c = P.box_cnt[B];
    if (col < c) {
      n = P.box_first[B] + col;
      return;
    }
    col -= c;
  }
  n = -1;
}

__global__ void k_count_singular(PanelArgs P, FillArgs A, long long nnz, unsigned int* cnt) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nnz) return;
  int m, n, B;
  panel_mn(idx, P, m, n, B);
  int c = 0, p, q;
  for (int t = 0; t < 2; t++)
    for (int s = 0; s < 2; s++) c += pair_singular(m, n, t, s, A, p, q) ? 1 : 0;
  cnt[idx] = (unsigned int)c;
}

struct SingItem {
  long long blk;
  int m, n;
  int ts;  // t*2 + s
  int pad;
};

__global__ void k_emit_singular(PanelArgs P, FillArgs A, long long nnz, const unsigned int* cnt,
                                const unsigned int* off, SingItem* items) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nnz) return;
  if (cnt[idx] == 0) return;
  int m, n, B;
  panel_mn(idx, P, m, n, B);
  unsigned int o = off[idx];
  int p, q;
  for (int t = 0; t < 2; t++)
    for (int s = 0; s < 2; s++)
      if (pair_singular(m, n, t, s, A, p, q)) {
        SingItem it;
        it.blk = idx;
        it.m = m;
        it.n = n;
        it.ts = t * 2 + s;
        it.pad = 0;
        items[o++] = it;
      }
}

// zz contributions (a, b, d) of each singular item
__global__ void k_singular(FillArgs A, const int* tri_verts, const SingItem* items, long long nitem,
                           zc* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitem) return;
  SingItem it = items[i];
  int t = it.ts >> 1, s = it.ts & 1;
  int p, q;
  pair_singular(it.m, it.n, t, s, A, p, q);
  KT r = singular_pair(it.m, it.n, t, s, p, q, A, tri_verts);
  zc a = mk<double>(0, 0), b = a, d = a;
  combine(r, A, a, b, d);
  out[3 * i] = a;
  out[3 * i + 1] = b;
  out[3 * i + 2] = d;
}

// Regular pairs of every block + the precomputed singular items of the block.
__global__ void __launch_bounds__(128) k_fill_regular(PanelArgs P, FillArgs A, long long nnz,
                                                      const unsigned int* cnt,
                                                      const unsigned int* off, const zc* sing,
                                                      zc* na, zc* nb, zc* nd) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nnz) return;
  int m, n, B;
  panel_mn(idx, P, m, n, B);
  zc a = mk<double>(0, 0), b = a, d = a;
  int p, q;
  for (int t = 0; t < 2; t++)
    for (int s = 0; s < 2; s++) {
      if (pair_singular(m, n, t, s, A, p, q)) continue;
      KT r = outer_regular(A.fn[2 * m + t], A.fn[2 * n + s], A);
      combine(r, A, a, b, d);
    }
  int c = cnt[idx];
  if (c) {
    unsigned int o = off[idx];
    for (int k = 0; k < c; k++) {
      a += sing[3 * (o + k)];
      b += sing[3 * (o + k) + 1];
      d += sing[3 * (o + k) + 2];
    }
  }
  na[idx] = a;
  nb[idx] = b;
  nd[idx] = d;
}

// Arbitrary (m, n) list (tests and the dense path): everything inline.
__global__ void k_blocks_list(FillArgs A, const int* tri_verts, const int* ms, const int* ns,
                              int cnt, zc* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  int m = ms[i], n = ns[i];
  zc a = mk<double>(0, 0), b = a, d = a;
  int p, q;
  for (int t = 0; t < 2; t++)
    for (int s = 0; s < 2; s++) {
      KT r;
      if (pair_singular(m, n, t, s, A, p, q))
        r = singular_pair(m, n, t, s, p, q, A, tri_verts);
      else
        r = outer_regular(A.fn[2 * m + t], A.fn[2 * n + s], A);
      combine(r, A, a, b, d);
    }
  out[3 * i] = a;
  out[3 * i + 1] = b;
  out[3 * i + 2] = d;
}

__global__ void k_to_f32(const zc* a, cc* b, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = mk<float>((float)a[i].re, (float)a[i].im);
}

// -------------------------------------------------------------------------
// Near-field panel matvec.  One warp per row; the row's columns are the
// concatenated edge ranges of E2(A); x is interleaved (J, M) per internal edge.
// y_J += a xJ + b xM ; y_M += (cfac b) xJ + d xM.
template <typename T, bool ACCUM>
__global__ void __launch_bounds__(256) k_near_spmv(PanelArgs P, const cx<T>* __restrict__ va,
                                                   const cx<T>* __restrict__ vb,
                                                   const cx<T>* __restrict__ vd_,
                                                   const int* __restrict__ edge_box, int M,
                                                   cx<T> cfac, const cx<T>* __restrict__ x,
                                                   cx<T>* __restrict__ y, int nrhs) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= M) return;
  int m = warp;
  int A = edge_box[m];
  int row = m - P.box_first[A];
  int nc = P.ncols[A];
  long long base = P.base[A] + (long long)row * nc;
  for (int r = 0; r < nrhs; r++) {
    const cx<T>* xr = x + (size_t)r * 2 * M;
    cx<T> sJ = mk<T>(0, 0), sM = mk<T>(0, 0);
    int col0 = 0;
    for (int k = P.nbr_ptr[A]; k < P.nbr_ptr[A + 1]; k++) {
      int B = P.nbr_box[k];
      int c = P.box_cnt[B], f = P.box_first[B];
      for (int j = lane; j < c; j += 32) {
        long long o = base + col0 + j;
        cx<T> a = va[o], b = vb[o], d = vd_[o];
        cx<T> xj = xr[2 * (f + j)], xm = xr[2 * (f + j) + 1];
        sJ = cfma(a, xj, sJ);
        sJ = cfma(b, xm, sJ);
        sM = cfma(cfac * b, xj, sM);
        sM = cfma(d, xm, sM);
      }
      col0 += c;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sJ.re += __shfl_xor_sync(0xffffffff, sJ.re, o);
      sJ.im += __shfl_xor_sync(0xffffffff, sJ.im, o);
      sM.re += __shfl_xor_sync(0xffffffff, sM.re, o);
      sM.im += __shfl_xor_sync(0xffffffff, sM.im, o);
    }
    if (lane == 0) {
      cx<T>* yr = y + (size_t)r * 2 * M;
      if (ACCUM) {
        yr[2 * m] += sJ;
        yr[2 * m + 1] += sM;
      } else {
        yr[2 * m] = sJ;
        yr[2 * m + 1] = sM;
      }
    }
  }
}

// Near product over work chunks of at most 32 rows of one leaf box A.  All rows of A
// share the panel's columns, so the chunk first gathers x of those columns into shared
// memory (J, M per column) and then streams the a, b, d rows against it: every lane
// walks the whole concatenated column range, with no partial warps at box seams.
template <typename T, bool ACCUM, int NW = 8>
__global__ void __launch_bounds__(32 * NW) k_near_panel(PanelArgs P, const cx<T>* __restrict__ va,
                                                    const cx<T>* __restrict__ vb,
                                                    const cx<T>* __restrict__ vd_,
                                                    const int4* __restrict__ chunks, int M,
                                                    cx<T> cfac, const cx<T>* __restrict__ x,
                                                    cx<T>* __restrict__ y, int nrhs) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* xs = reinterpret_cast<cx<T>*>(smraw);  // [ncols][J, M]
  const int4 ch = chunks[blockIdx.x];
  const int A = ch.x, f = ch.y, cnt = ch.z;
  const int nc = P.ncols[A];
  const long long base = P.base[A] + (long long)(f - P.box_first[A]) * nc;
  const unsigned long long pol = l2_evict_first_policy();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k0 = P.nbr_ptr[A], k1 = P.nbr_ptr[A + 1];
  for (int r = 0; r < nrhs; r++) {
    const cx<T>* xr = x + (size_t)r * 2 * M;
    if (r > 0) __syncthreads();
    int col0 = 0;
    for (int k = k0; k < k1; k++) {
      const int B = P.nbr_box[k];
      const int c = P.box_cnt[B], fb = P.box_first[B];
      for (int j = threadIdx.x; j < 2 * c; j += blockDim.x) xs[2 * col0 + j] = xr[2 * fb + j];
      col0 += c;
    }
    __syncthreads();
    for (int row = warp; row < cnt; row += NW) {
      const long long o = base + (long long)row * nc;
      cx<T> sJ = mk<T>(0, 0), sM = mk<T>(0, 0), tM = mk<T>(0, 0);
#pragma unroll 4
      for (int j = lane; j < nc; j += 32) {
        cx<T> a = ld_stream(va + o + j, pol), b = ld_stream(vb + o + j, pol), d = ld_stream(vd_ + o + j, pol);
        cx<T> xj = xs[2 * j], xm = xs[2 * j + 1];
        sJ = cfma(a, xj, sJ);
        sJ = cfma(b, xm, sJ);
        tM = cfma(b, xj, tM);
        sM = cfma(d, xm, sM);
      }
      sM = cfma(cfac, tM, sM);
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        sJ.re += __shfl_xor_sync(0xffffffffu, sJ.re, s);
        sJ.im += __shfl_xor_sync(0xffffffffu, sJ.im, s);
        sM.re += __shfl_xor_sync(0xffffffffu, sM.re, s);
        sM.im += __shfl_xor_sync(0xffffffffu, sM.im, s);
      }
      if (lane == 0) {
        cx<T>* yr = y + (size_t)r * 2 * M + 2 * (f + row);
        if (ACCUM) {
          yr[0] += sJ;
          yr[1] += sM;
        } else {
          yr[0] = sJ;
          yr[1] = sM;
        }
      }
    }
  }
}

// Near product of a batch of R vectors: block per (chunk of <= 32 rows of box A, group of
// RG vectors).  The chunk gathers x of the panel's columns for its RG vectors into shared
// memory ([vector][J, M][column], so consecutive lanes read consecutive words), then each
// warp streams rows of the panel once and applies every value to all RG vectors.  The
// groups of one chunk are adjacent blocks and mostly read the panel rows from L2.
template <typename T, int RG>
__global__ void __launch_bounds__(256) k_near_b(PanelArgs P, const cx<T>* __restrict__ va,
                                                const cx<T>* __restrict__ vb,
                                                const cx<T>* __restrict__ vd_,
                                                const int4* __restrict__ chunks, int ngr, int M,
                                                cx<T> cfac, const cx<T>* __restrict__ x, int R,
                                                cx<T>* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* xs = reinterpret_cast<cx<T>*>(smraw);  // [RG][J, M][ncols]
  const int ci = blockIdx.x / ngr, g = blockIdx.x - ci * ngr;
  const int4 ch = chunks[ci];
  const int A = ch.x, f = ch.y, cnt = ch.z;
  const int nc = P.ncols[A];
  const long long base = P.base[A] + (long long)(f - P.box_first[A]) * nc;
  const int r0 = g * RG, nr = min(RG, R - r0);
  const size_t ldx = (size_t)2 * M;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int col0 = 0;
  for (int k = P.nbr_ptr[A]; k < P.nbr_ptr[A + 1]; k++) {
    const int B = P.nbr_box[k];
    const int c = P.box_cnt[B], fb = P.box_first[B];
    for (int j = threadIdx.x; j < 2 * RG * c; j += blockDim.x) {
      const int rr = j / (2 * c), rem = j - rr * 2 * c;
      const int col = rem >> 1, h = rem & 1;
      xs[((size_t)rr * 2 + h) * nc + col0 + col] =
          rr < nr ? x[(size_t)(r0 + rr) * ldx + 2 * (fb + col) + h] : mk<T>(0, 0);
    }
    col0 += c;
  }
  __syncthreads();
  for (int row = warp; row < cnt; row += 8) {
    const long long o = base + (long long)row * nc;
    cx<T> sJ[RG], sM[RG], tM[RG];
#pragma unroll
    for (int rr = 0; rr < RG; rr++) sJ[rr] = sM[rr] = tM[rr] = mk<T>(0, 0);
#pragma unroll 2
    for (int j = lane; j < nc; j += 32) {
      const cx<T> a = va[o + j], b = vb[o + j], d = vd_[o + j];
#pragma unroll
      for (int rr = 0; rr < RG; rr++) {
        const cx<T> xj = xs[(size_t)(2 * rr) * nc + j], xm = xs[(size_t)(2 * rr + 1) * nc + j];
        sJ[rr] = cfma(a, xj, sJ[rr]);
        sJ[rr] = cfma(b, xm, sJ[rr]);
        tM[rr] = cfma(b, xj, tM[rr]);
        sM[rr] = cfma(d, xm, sM[rr]);
      }
    }
#pragma unroll
    for (int rr = 0; rr < RG; rr++) {
      sM[rr] = cfma(cfac, tM[rr], sM[rr]);
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        sJ[rr].re += __shfl_xor_sync(0xffffffffu, sJ[rr].re, s);
        sJ[rr].im += __shfl_xor_sync(0xffffffffu, sJ[rr].im, s);
        sM[rr].re += __shfl_xor_sync(0xffffffffu, sM[rr].re, s);
        sM[rr].im += __shfl_xor_sync(0xffffffffu, sM[rr].im, s);
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int rr = 0; rr < RG; rr++) {
        if (rr < nr) {
          cx<T>* yr = y + (size_t)(r0 + rr) * ldx + 2 * (f + row);
          yr[0] = sJ[rr];
          yr[1] = sM[rr];
        }
      }
    }
  }
}

// Transposed near panels, made once for the adjoint product.  E2 is symmetric, so the
// transposed matrix has the forward panels' layout: element (row n, column m) of box B's
// panel is Z[m, n], found in the panel of box(m) at row m and at the column of n, which
// lies in the column range of B there.  The 2 x 2 block [[a, b], [cfac b, d]] transposes
// to [[a, cfac b], [b, d]]; stored as (a, cfac b, d), the forward product kernels apply it
// with cfac replaced by 1 / cfac.
__global__ void k_transpose_panels(PanelArgs P, const int* __restrict__ edge_box, long long nnz,
                                   const zc* __restrict__ va, const zc* __restrict__ vb,
                                   const zc* __restrict__ vd_, zc cfac, zc* __restrict__ ta,
                                   zc* __restrict__ tb, zc* __restrict__ td) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nnz) return;
  int n, m, B;
  panel_mn(idx, P, n, m, B);  // transposed panel of box B: row edge n, column edge m
  const int Bm = edge_box[m];
  int col0 = 0;
  for (int k = P.nbr_ptr[Bm]; k < P.nbr_ptr[Bm + 1]; k++) {
    const int Bp = P.nbr_box[k];
    if (Bp == B) break;
    col0 += P.box_cnt[Bp];
  }
  const long long src = P.base[Bm] + (long long)(m - P.box_first[Bm]) * P.ncols[Bm] + col0 + (n - P.box_first[B]);
  ta[idx] = va[src];
  tb[idx] = cfac * vb[src];
  td[idx] = vd_[src];
}

// Near part of the shape gradient: for every near block (m, n) and triangle pair (t, s),
// the z derivative of the (t, s) term with respect to each vertex of the two triangles, by
// central differences of the term rebuilt with that vertex moved by +-h (same quadrature
// and the same singular / regular choice as the fill), contracted as -2 Re(conj(lambda_m)
// dZ_mn I_n) into grad[vertex].
__global__ void __launch_bounds__(128) k_grad_near(PanelArgs P, FillArgs A, const int* tri_verts,
                                                   const SideV* __restrict__ sv, const double* __restrict__ V,
                                                   int normal_convention, double h, long long nnz,
                                                   const zc* __restrict__ lam, const zc* __restrict__ I,
                                                   zc cfac, double* grad) {
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= 4 * nnz) return;
  const long long idx = it >> 2;
  const int t = (int)(it >> 1) & 1, s = (int)it & 1;
  int m, n, B;
  panel_mn(idx, P, m, n, B);
  int p, q;
  const bool sing = pair_singular(m, n, t, s, A, p, q);
  const SideV sm = sv[2 * m + t], sn = sv[2 * n + s];
  const double sgm = A.fn[2 * m + t].sgn, sgn = A.fn[2 * n + s].sgn;
  const zc lJ = conj(lam[2 * m]), lM = conj(lam[2 * m + 1]), iJ = I[2 * n], iM = I[2 * n + 1];
  const int vs[6] = {sm.t0, sm.t1, sm.t2, sn.t0, sn.t1, sn.t2};
  for (int k = 0; k < 6; k++) {
    const int v = vs[k];
    bool dup = false;
    for (int j = 0; j < k; j++) dup |= (vs[j] == v);
    if (dup) continue;
    zc ab[2][3];
    for (int pm = 0; pm < 2; pm++) {
      const double dz = pm ? -h : h;
      const FnD fm = side_fn(sm, sgm, V, normal_convention, v, dz);
      const FnD fn = side_fn(sn, sgn, V, normal_convention, v, dz);
      const KT r = sing ? singular_pair_f(fm, fn, p, q, A, tri_verts) : outer_regular(fm, fn, A);
      zc a = mk<double>(0, 0), b = a, d = a;
      combine(r, A, a, b, d);
      ab[pm][0] = a;
      ab[pm][1] = b;
      ab[pm][2] = d;
    }
    const double inv = 0.5 / h;
    const zc da = (ab[0][0] - ab[1][0]) * inv, db = (ab[0][1] - ab[1][1]) * inv, dd = (ab[0][2] - ab[1][2]) * inv;
    const zc val = lJ * (da * iJ + db * iM) + lM * (cfac * db * iJ + dd * iM);
    atomicAdd(grad + v, -2.0 * val.re);
  }
}

PanelArgs panel_args(sie_ctx* c);
FillArgs fill_args(sie_ctx* c);

int grad_near(sie_ctx* c, const zc* lam, const zc* I, double h, double* grad, cudaStream_t st) {
  const long long nnz = c->near.nnz;
  const long long work = 4 * nnz;
  FillArgs A = fill_args(c);
  A.smooth = 1;  // differentiate the x_nt term without its binary32 rounding (a staircase)
  k_grad_near<<<(unsigned)((work + 127) / 128), 128, 0, st>>>(panel_args(c), A, c->d_tri_verts,
                                                              (const SideV*)c->d_side, c->d_vert,
                                                              c->cfg.normal_convention, h, nnz, lam, I, c->cfac,
                                                              grad);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

// -------------------------------------------------------------------------
// host wrappers

// vectors per block of the batched near product
template <typename T> struct NearGroup { static const int RG = sizeof(T) == 4 ? 4 : 2; };

// Shared memory of the batched near product; 0 if the widest panel does not fit.
template <typename T>
static size_t near_b_smem(const sie_ctx* c) {
  size_t s = (size_t)c->ncols_max * 2 * NearGroup<T>::RG * sizeof(cx<T>);
  return s <= (size_t)200 * 1024 ? std::max<size_t>(s, 16) : 0;
}

// Shared memory the chunked near product needs; 0 if the widest panel does not fit.
template <typename T>
static size_t near_panel_smem(const sie_ctx* c) {
  size_t s = (size_t)c->ncols_max * 2 * sizeof(cx<T>);
  return s <= (size_t)200 * 1024 ? std::max<size_t>(s, 16) : 0;
}

int near_prepare_kernels(sie_ctx* c) {
  if (size_t s = near_panel_smem<double>(c)) {
    SIE_CUDA(raise_smem(k_near_panel<double, true>, s));
    SIE_CUDA(raise_smem(k_near_panel<double, false>, s));
    SIE_CUDA(raise_smem(k_near_panel<double, true, 4>, s));
    SIE_CUDA(raise_smem(k_near_panel<double, false, 4>, s));
  }
  if (size_t s = near_panel_smem<float>(c)) {
    SIE_CUDA(raise_smem(k_near_panel<float, true>, s));
    SIE_CUDA(raise_smem(k_near_panel<float, false>, s));
    SIE_CUDA(raise_smem(k_near_panel<float, true, 4>, s));
    SIE_CUDA(raise_smem(k_near_panel<float, false, 4>, s));
  }
  if (size_t s = near_b_smem<double>(c)) SIE_CUDA(raise_smem(k_near_b<double, NearGroup<double>::RG>, s));
  if (size_t s = near_b_smem<float>(c)) SIE_CUDA(raise_smem(k_near_b<float, NearGroup<float>::RG>, s));
  return SIE_OK;
}

PanelArgs panel_args(sie_ctx* c) {
  PanelArgs P;
  P.nbox = c->near.nbox;
  P.base = c->d_base;
  P.box_first = c->d_box_first;
  P.box_cnt = c->d_box_cnt;
  P.nbr_ptr = c->d_nbr_ptr;
  P.nbr_box = c->d_nbr_box;
  P.ncols = c->d_ncols;
  return P;
}

FillArgs fill_args(sie_ctx* c) {
  FillArgs A;
  A.fn = c->d_fn;
  A.rref = c->d_rref;
  A.cent = c->d_cent;
  A.mt = c->mt;
  A.R = c->R;
  A.formulation = c->cfg.formulation;
  A.fix_itbn = c->cfg.fix_itbn;
  A.smooth = 0;
  return A;
}

int near_fill(sie_ctx* c, int* d_tri_verts) {
  long long nnz = c->near.nnz;
  PanelArgs P = panel_args(c);
  FillArgs A = fill_args(c);
  cudaStream_t st = c->stream;
  unsigned int* cnt = nullptr;
  unsigned int* off = nullptr;
  SIE_CUDA(cudaMalloc(&cnt, (nnz + 16) * sizeof(unsigned int)));
  SIE_CUDA(cudaMalloc(&off, (nnz + 16) * sizeof(unsigned int)));
  int thr = 256;
  long long blocks = (nnz + thr - 1) / thr;
  k_count_singular<<<(unsigned)blocks, thr, 0, st>>>(P, A, nnz, cnt); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  // exclusive scan of the counts (values <= 4 per block)
  size_t tmp_bytes = 0;
  SIE_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, off, (int)nnz, st));
  void* tmp = nullptr;
  SIE_CUDA(cudaMalloc(&tmp, tmp_bytes + 16));
  SIE_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, off, (int)nnz, st));
  unsigned int last_off = 0;
  unsigned int last_cnt = 0;
  SIE_CUDA(cudaMemcpyAsync(&last_off, off + nnz - 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  SIE_CUDA(cudaMemcpyAsync(&last_cnt, cnt + nnz - 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  SIE_CUDA(cudaStreamSynchronize(st));
  long long nitem = (long long)last_off + last_cnt;
  SingItem* items = nullptr;
  zc* sing = nullptr;
  SIE_CUDA(cudaMalloc(&items, (nitem + 1) * sizeof(SingItem)));
  SIE_CUDA(cudaMalloc(&sing, (nitem + 1) * 3 * sizeof(zc)));
  k_emit_singular<<<(unsigned)blocks, thr, 0, st>>>(P, A, nnz, cnt, off, items); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  if (nitem > 0) {
    k_singular<<<(unsigned)((nitem + 63) / 64), 64, 0, st>>>(A, d_tri_verts, items, nitem, sing); sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  k_fill_regular<<<(unsigned)((nnz + 127) / 128), 128, 0, st>>>(P, A, nnz, cnt, off, sing, c->d_na,
                                                               c->d_nb, c->d_nd); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  SIE_CUDA(cudaStreamSynchronize(st));
  cudaFree(cnt);
  cudaFree(off);
  cudaFree(tmp);
  cudaFree(items);
  cudaFree(sing);
  return SIE_OK;
}

int near_blocks_list(sie_ctx* c, int* d_tri_verts, const int* d_m, const int* d_n, int cnt,
                     zc* d_out) {
  FillArgs A = fill_args(c);
  k_blocks_list<<<(cnt + 63) / 64, 64, 0, c->stream>>>(A, d_tri_verts, d_m, d_n, cnt, d_out); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int near_to_f32(sie_ctx* c) {
  long long n = c->near.nnz;
  unsigned g = (unsigned)((n + 255) / 256);
  k_to_f32<<<g, 256, 0, c->stream>>>(c->d_na, c->d_na32, n); sie::count_launch();
  k_to_f32<<<g, 256, 0, c->stream>>>(c->d_nb, c->d_nb32, n); sie::count_launch();
  k_to_f32<<<g, 256, 0, c->stream>>>(c->d_nd, c->d_nd32, n); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

template <typename T>
int near_matvec_t(sie_ctx* c, const cx<T>* va, const cx<T>* vb, const cx<T>* vdd, cx<T> cfac,
                  const cx<T>* x, cx<T>* y, int nrhs, bool accum, cudaStream_t st) {
  PanelArgs P = panel_args(c);
  size_t smem = near_panel_smem<T>(c);
  if (c->near_mode == 2 && smem && c->n_rchunk > 0) {
    const int4* ch = (const int4*)c->d_rchunk;
    if (accum) {
      k_near_panel<T, true, 4><<<c->n_rchunk, 128, smem, st>>>(P, va, vb, vdd, ch, c->M, cfac, x, y, nrhs); sie::count_launch();
    } else {
      k_near_panel<T, false, 4><<<c->n_rchunk, 128, smem, st>>>(P, va, vb, vdd, ch, c->M, cfac, x, y, nrhs); sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
    return SIE_OK;
  }
  if (c->near_mode == 1 && smem && c->n_rchunk > 0) {
    const int4* ch = (const int4*)c->d_rchunk;
    if (accum) {
      k_near_panel<T, true><<<c->n_rchunk, 256, smem, st>>>(P, va, vb, vdd, ch, c->M, cfac, x, y, nrhs); sie::count_launch();
    } else {
      k_near_panel<T, false><<<c->n_rchunk, 256, smem, st>>>(P, va, vb, vdd, ch, c->M, cfac, x, y, nrhs); sie::count_launch();
    }
    SIE_CUDA(cudaGetLastError());
    return SIE_OK;
  }
  long long threads = (long long)c->M * 32;
  unsigned g = (unsigned)((threads + 255) / 256);
  if (accum) {
    k_near_spmv<T, true><<<g, 256, 0, st>>>(P, va, vb, vdd, c->d_edge_box, c->M, cfac, x, y, nrhs); sie::count_launch();
  } else {
    k_near_spmv<T, false><<<g, 256, 0, st>>>(P, va, vb, vdd, c->d_edge_box, c->M, cfac, x, y, nrhs); sie::count_launch();
  }
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int near_matvec64(sie_ctx* c, const zc* x, zc* y, int nrhs, bool accum, cudaStream_t st) {
  return near_matvec_t<double>(c, c->d_na, c->d_nb, c->d_nd, c->cfac, x, y, nrhs, accum, st);
}
int near_matvec32(sie_ctx* c, const cc* x, cc* y, int nrhs, bool accum, cudaStream_t st) {
  cc cf = mk<float>((float)c->cfac.re, (float)c->cfac.im);
  return near_matvec_t<float>(c, c->d_na32, c->d_nb32, c->d_nd32, cf, x, y, nrhs, accum, st);
}

// Batched near product (writes y); panels too wide for the batched kernel's shared memory
// take the one-vector-at-a-time product.
template <typename T>
static int near_matvec_b_t(sie_ctx* c, const cx<T>* va, const cx<T>* vb, const cx<T>* vdd, cx<T> cfac,
                           const cx<T>* x, cx<T>* y, int R, cudaStream_t st) {
  const size_t smem = near_b_smem<T>(c);
  if (!smem || c->n_rchunk < 1) return near_matvec_t<T>(c, va, vb, vdd, cfac, x, y, R, false, st);
  const int RG = NearGroup<T>::RG;
  const int ngr = (R + RG - 1) / RG;
  k_near_b<T, NearGroup<T>::RG><<<(unsigned)c->n_rchunk * ngr, 256, smem, st>>>(
      panel_args(c), va, vb, vdd, (const int4*)c->d_rchunk, ngr, c->M, cfac, x, R, y);
  sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int near_matvec_adj64(sie_ctx* c, const zc* x, zc* y, cudaStream_t st) {
  const long long nnz = c->near.nnz;
  if (!c->d_naT) {
    const size_t bytes = (size_t)std::max<long long>(nnz, 1) * sizeof(zc);
    SIE_CUDA(cudaMalloc(&c->d_naT, bytes));
    SIE_CUDA(cudaMalloc(&c->d_nbT, bytes));
    SIE_CUDA(cudaMalloc(&c->d_ndT, bytes));
    k_transpose_panels<<<(unsigned)((nnz + 255) / 256), 256, 0, st>>>(panel_args(c), c->d_edge_box, nnz, c->d_na,
                                                                      c->d_nb, c->d_nd, c->cfac, c->d_naT,
                                                                      c->d_nbT, c->d_ndT);
    sie::count_launch();
    SIE_CUDA(cudaGetLastError());
  }
  const zc inv = mk<double>(1.0, 0.0) / c->cfac;
  return near_matvec_t<double>(c, c->d_naT, c->d_nbT, c->d_ndT, inv, x, y, 1, false, st);
}

int near_matvec_b64(sie_ctx* c, const zc* x, zc* y, int R, cudaStream_t st) {
  return near_matvec_b_t<double>(c, c->d_na, c->d_nb, c->d_nd, c->cfac, x, y, R, st);
}
int near_matvec_b32(sie_ctx* c, const cc* x, cc* y, int R, cudaStream_t st) {
  cc cf = mk<float>((float)c->cfac.re, (float)c->cfac.im);
  return near_matvec_b_t<float>(c, c->d_na32, c->d_nb32, c->d_nd32, cf, x, y, R, st);
}

}  // namespace sie
