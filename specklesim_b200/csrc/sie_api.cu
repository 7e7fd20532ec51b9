// C-ABI entry points, mesh/tree set-up and matvec orchestration of libsiegpu.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "sie_internal.h"

namespace sie {

static thread_local std::string g_err = "";
static unsigned long long g_launches = 0;
void count_launch() { __atomic_add_fetch(&g_launches, 1ULL, __ATOMIC_RELAXED); }
void count_launches(unsigned long long n) { __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED); }

void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) {
    // a failed allocation is not sticky: clear it, so that the next check of the runtime's
    // last error (after a later launch) does not report it again
    cudaGetLastError();
    return SIE_ERR_NOMEM;
  }
  return SIE_ERR_CUDA;
}

// src/lib_sie_integration_points.f90:7-141; the literals are binary32.
Rule make_rule(int ngp) {
  Rule r;
  memset(&r, 0, sizeof(r));
  r.n = ngp;
  if (ngp == 1) {
    r.a[0] = 0.33333333333333f;
    r.b[0] = 0.33333333333333f;
    r.w[0] = 1.0f;
  } else if (ngp == 3) {
    const float a[3] = {0.16666666666667f, 0.16666666666667f, 0.66666666666667f};
    const float b[3] = {0.16666666666667f, 0.66666666666667f, 0.16666666666667f};
    for (int i = 0; i < 3; i++) {
      r.a[i] = a[i];
      r.b[i] = b[i];
      r.w[i] = 0.33333333333333f;
    }
  } else if (ngp == 4) {
    const float a[4] = {0.33333333333333f, 0.20000000000000f, 0.20000000000000f, 0.60000000000000f};
    const float b[4] = {0.33333333333333f, 0.20000000000000f, 0.60000000000000f, 0.20000000000000f};
    const float w[4] = {-0.56250000000000f, 0.52083333333333f, 0.52083333333333f,
                        0.52083333333333f};
    for (int i = 0; i < 4; i++) {
      r.a[i] = a[i];
      r.b[i] = b[i];
      r.w[i] = w[i];
    }
  } else if (ngp == 6) {
    const float a[6] = {0.44594849091597f, 0.44594849091597f, 0.10810301816807f,
                        0.09157621350977f, 0.09157621350977f, 0.81684757298046f};
    const float b[6] = {0.44594849091597f, 0.10810301816807f, 0.44594849091597f,
                        0.09157621350977f, 0.81684757298046f, 0.09157621350977f};
    const float w[6] = {0.22338158967801f, 0.22338158967801f, 0.22338158967801f,
                        0.10995174365532f, 0.10995174365532f, 0.10995174365532f};
    for (int i = 0; i < 6; i++) {
      r.a[i] = a[i];
      r.b[i] = b[i];
      r.w[i] = w[i];
    }
  } else if (ngp == 7) {
    const float a[7] = {0.33333333333333f, 0.47014206410511f, 0.47014206410511f,
                        0.05971587178977f, 0.10128650732346f, 0.10128650732346f,
                        0.79742698535309f};
    const float b[7] = {0.33333333333333f, 0.47014206410511f, 0.05971587178977f,
                        0.47014206410511f, 0.10128650732346f, 0.79742698535309f,
                        0.10128650732346f};
    const float w[7] = {0.22500000000000f, 0.13239415278851f, 0.13239415278851f,
                        0.13239415278851f, 0.12593918054483f, 0.12593918054483f,
                        0.12593918054483f};
    for (int i = 0; i < 7; i++) {
      r.a[i] = a[i];
      r.b[i] = b[i];
      r.w[i] = w[i];
    }
  } else if (ngp == 12) {
    const float a[12] = {0.249286745170910f, 0.249286745170910f, 0.501426509658180f,
                         0.063089014491500f, 0.063089014491500f, 0.873821971017000f,
                         0.310352451033780f, 0.636502499121400f, 0.053145049844820f,
                         0.636502499121400f, 0.310352451033780f, 0.053145049844820f};
    const float b[12] = {0.249286745170910f, 0.501426509658180f, 0.249286745170910f,
                         0.063089014491500f, 0.873821971017000f, 0.063089014491500f,
                         0.636502499121400f, 0.053145049844820f, 0.310352451033780f,
                         0.310352451033780f, 0.053145049844820f, 0.636502499121400f};
    const float w[12] = {0.116786275726380f, 0.116786275726380f, 0.116786275726380f,
                         0.0508449063702100f, 0.0508449063702100f, 0.0508449063702100f,
                         0.0828510756183700f, 0.0828510756183700f, 0.0828510756183700f,
                         0.0828510756183700f, 0.0828510756183700f, 0.0828510756183700f};
    for (int i = 0; i < 12; i++) {
      r.a[i] = a[i];
      r.b[i] = b[i];
      r.w[i] = w[i];
    }
  } else {
    r.n = 0;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Morton universal index (src/lib/libtree/lib/lib_tree_helper_functions.f90:217-379,
// 1652-1875): x is the most significant bit of every triple.
static const int L_TH = 21;
static inline uint64_t morton3(uint64_t ix, uint64_t iy, uint64_t iz, int l) {
  uint64_t n = 0;
  for (int b = l - 1; b >= 0; b--)
    n = (n << 3) | (((ix >> b) & 1) << 2) | (((iy >> b) & 1) << 1) | ((iz >> b) & 1);
  return n;
}
static inline void demorton3(uint64_t n, int l, int64_t& ix, int64_t& iy, int64_t& iz) {
  ix = iy = iz = 0;
  for (int b = 0; b < l; b++) {
    iz |= (int64_t)((n >> (3 * b)) & 1) << b;
    iy |= (int64_t)((n >> (3 * b + 1)) & 1) << b;
    ix |= (int64_t)((n >> (3 * b + 2)) & 1) << b;
  }
}
static inline uint64_t coord_bits(double f, int l) {
  if (!(f > 0.0)) return 0;
  return (uint64_t)std::floor(std::ldexp(f, l));
}

static void box_centre(const sie_ctx* c, uint64_t n, int l, double* out) {
  int64_t i[3];
  demorton3(n, l, i[0], i[1], i[2]);
  double s = std::ldexp(1.0, -l);
  for (int d = 0; d < 3; d++) out[d] = s * (i[d] + 0.5) * c->D + c->xmin[d];
}

static int index_of(const std::vector<uint64_t>& v, uint64_t n) {
  auto it = std::lower_bound(v.begin(), v.end(), n);
  if (it == v.end() || *it != n) return -1;
  return (int)(it - v.begin());
}

// k = 1 neighbours at level l, self excluded (lib_tree_hf_get_neighbour_all_xD)
static void neighbours(uint64_t n, int l, std::vector<uint64_t>& out) {
  out.clear();
  int64_t ix, iy, iz;
  demorton3(n, l, ix, iy, iz);
  int64_t ub = ((int64_t)1 << l) - 1;
  for (int dx = -1; dx <= 1; dx++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dz = -1; dz <= 1; dz++) {
        int64_t a = ix + dx, b = iy + dy, cc = iz + dz;
        if (a < 0 || b < 0 || cc < 0 || a > ub || b > ub || cc > ub) continue;
        uint64_t m = morton3(a, b, cc, l);
        if (m != n) out.push_back(m);
      }
}

// ---------------------------------------------------------------------------
// Mesh topology: find_neighbours (:865-905) in the order of its (i<j) scan,
// fn_parameter_type (:1539-1586).
static int build_mesh(sie_ctx* c) {
  int nt = c->nt;
  c->cent.resize(3 * (size_t)nt);
  for (int t = 0; t < nt; t++) {
    for (int d = 0; d < 3; d++) {
      double a = c->verts[3 * c->tris[3 * t] + d], b = c->verts[3 * c->tris[3 * t + 1] + d],
             e = c->verts[3 * c->tris[3 * t + 2] + d];
      c->cent[3 * t + d] = (a + b + e) / 3.0;
    }
  }
  std::unordered_map<uint64_t, std::vector<int>> emap;
  emap.reserve((size_t)nt * 2);
  for (int t = 0; t < nt; t++)
    for (int e = 0; e < 3; e++) {
      uint64_t a = (uint32_t)c->tris[3 * t + e], b = (uint32_t)c->tris[3 * t + (e + 1) % 3];
      if (a > b) std::swap(a, b);
      emap[(a << 32) | b].push_back(t);
    }
  std::vector<std::pair<int, int>> prs;
  prs.reserve((size_t)nt * 2);
  for (auto& kv : emap) {
    auto& L = kv.second;
    std::sort(L.begin(), L.end());
    for (size_t i = 0; i < L.size(); i++)
      for (size_t j = i + 1; j < L.size(); j++) prs.push_back({L[i], L[j]});
  }
  std::sort(prs.begin(), prs.end());
  prs.erase(std::unique(prs.begin(), prs.end()), prs.end());
  c->elem.clear();
  c->corner.clear();
  for (auto& pr : prs) {
    int i = pr.first, j = pr.second;
    int com[3], nc = 0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        if (c->tris[3 * i + a] == c->tris[3 * j + b] && nc < 3) com[nc++] = c->tris[3 * i + a];
    if (nc != 2) continue;
    c->elem.push_back(i);
    c->elem.push_back(j);
    c->corner.push_back(com[0]);
    c->corner.push_back(com[1]);
  }
  c->M = (int)c->elem.size() / 2;
  if (c->M == 0) return fail(SIE_ERR_MESH, "mesh has no interior edge (no RWG basis)");
  c->fn_ext.resize(2 * (size_t)c->M);
  c->side_v.resize(16 * (size_t)c->M);
  const double* P = c->verts.data();
  for (int e = 0; e < c->M; e++) {
    for (int ot = 0; ot < 2; ot++) {
      int t = c->elem[2 * e + ot];
      int c1 = c->corner[2 * e], c2 = c->corner[2 * e + 1];
      int nv = 0, ipc = 0;
      for (int j = 0; j < 3; j++) {
        int v = c->tris[3 * t + j];
        if (v != c1 && v != c2) {
          ipc = v;
          nv = j + 1;
        }
      }
      const int* T = &c->tris[3 * t];
      int i1, i2;
      if (nv == 1) {
        i1 = T[1];
        i2 = T[2];
      } else if (nv == 2) {
        i1 = T[2];
        i2 = T[0];
      } else {
        i1 = T[0];
        i2 = T[1];
      }
      FnD f;
      memset(&f, 0, sizeof(f));
      vd p1 = mkv<double>(P[3 * i1], P[3 * i1 + 1], P[3 * i1 + 2]);
      vd p2 = mkv<double>(P[3 * i2], P[3 * i2 + 1], P[3 * i2 + 2]);
      vd pc = mkv<double>(P[3 * ipc], P[3 * ipc + 1], P[3 * ipc + 2]);
      f.c[0] = p1.x; f.c[1] = p1.y; f.c[2] = p1.z;
      f.c[3] = p2.x; f.c[4] = p2.y; f.c[5] = p2.z;
      f.c[6] = pc.x; f.c[7] = pc.y; f.c[8] = pc.z;
      f.length = vlen(p1 - p2);
      f.area = 0.5 * vlen(cross(p1 - pc, p2 - pc));
      if (!(f.area > 0.0)) return fail(SIE_ERR_MESH, "degenerate triangle " + std::to_string(t));
      f.sgn = (ot == 0) ? 1.0 : -1.0;
      f.df = f.sgn * f.length / f.area;
      for (int d = 0; d < 3; d++) f.mid[d] = c->cent[3 * t + d];
      vd a, b;
      if (c->cfg.normal_convention == 1) {
        a = p1 - p2;
        b = pc - p2;
      } else {
        a = pc - p1;
        b = p2 - p1;
      }
      vd n = cross(a, b);
      double ln = vlen(n);
      f.nq[0] = n.x / ln;
      f.nq[1] = n.y / ln;
      f.nq[2] = n.z / ln;
      f.tri = t;
      c->fn_ext[2 * e + ot] = f;
      const int* tv = &c->tris[3 * t];
      const int sv[8] = {i1, i2, ipc, t, tv[0], tv[1], tv[2], 0};
      for (int k = 0; k < 8; k++) c->side_v[8 * (2 * (size_t)e + ot) + k] = sv[k];
    }
  }
  return SIE_OK;
}

// Octree of the edge midpoints (lib_tree_constructor, lib_tree.f90:176-321;
// scaling :370-434; lib_tree_get_level_max :1290-1345).
static int build_tree(sie_ctx* c) {
  int M = c->M;
  std::vector<double> pos(3 * (size_t)M);
  for (int e = 0; e < M; e++) {
    const FnD& f = c->fn_ext[2 * e];
    for (int d = 0; d < 3; d++) pos[3 * e + d] = (f.c[d] + f.c[3 + d]) / 2.0;  // fn_edge_center
  }
  double xmax[3], Dd[3];
  for (int d = 0; d < 3; d++) {
    c->xmin[d] = 1e300;
    xmax[d] = -1e300;
  }
  for (int e = 0; e < M; e++)
    for (int d = 0; d < 3; d++) {
      c->xmin[d] = std::min(c->xmin[d], pos[3 * e + d]);
      xmax[d] = std::max(xmax[d], pos[3 * e + d]);
    }
  for (int d = 0; d < 3; d++) Dd[d] = (xmax[d] - c->xmin[d]) * (1 + std::ldexp(1.0, -52));
  c->D = std::max(Dd[0], std::max(Dd[1], Dd[2]));
  if (!(c->D > 0.0)) return fail(SIE_ERR_MESH, "all edge midpoints coincide");
  std::vector<uint64_t> nth(M);
  for (int e = 0; e < M; e++) {
    uint64_t ic[3];
    for (int d = 0; d < 3; d++) ic[d] = coord_bits((pos[3 * e + d] - c->xmin[d]) / c->D, L_TH);
    nth[e] = morton3(ic[0], ic[1], ic[2], L_TH);
  }
  std::vector<uint64_t> srt = nth;
  std::sort(srt.begin(), srt.end());
  int s = c->cfg.tree_s_opt;
  int l_max = 1;
  for (long i = 0; i + s < (long)M; i++) {
    uint64_t a = srt[i], b = srt[i + s];
    for (int lev = L_TH - 1; lev >= 0; lev--) {
      int sh = 3 * (L_TH - lev);
      if ((a >> sh) == (b >> sh)) {
        l_max = std::max(l_max, lev + 1);
        break;
      }
    }
  }
  if (c->cfg.dense) l_max = 1;
  c->l_max = l_max;
  c->l_min = std::min(2, l_max);
  c->leaf.resize(M);
  for (int e = 0; e < M; e++) c->leaf[e] = nth[e] >> (3 * (L_TH - l_max));
  // internal order: edges sorted by leaf box (stable)
  c->perm.resize(M);
  for (int e = 0; e < M; e++) c->perm[e] = e;
  std::stable_sort(c->perm.begin(), c->perm.end(),
                   [&](int a, int b) { return c->leaf[a] < c->leaf[b]; });
  c->iperm.resize(M);
  for (int i = 0; i < M; i++) c->iperm[c->perm[i]] = i;
  c->lv.assign(l_max + 1, Level());
  for (int l = c->l_min; l <= l_max; l++) {
    std::vector<uint64_t> v(M);
    for (int e = 0; e < M; e++) v[e] = c->leaf[e] >> (3 * (l_max - l));
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    c->lv[l].l = l;
    c->lv[l].box = v;
    c->lv[l].nb = (int)v.size();
    c->lv[l].only_k1 = (c->mt.k2.im != 0.0) && (l < l_max);
  }
  // leaf boxes in internal numbering
  NearLayout& N = c->near;
  const std::vector<uint64_t>& lb = c->lv[l_max].box;
  N.nbox = (int)lb.size();
  N.box_first.assign(N.nbox, 0);
  N.box_cnt.assign(N.nbox, 0);
  for (int i = 0; i < M; i++) {
    int b = index_of(lb, c->leaf[c->perm[i]]);
    if (N.box_cnt[b] == 0) N.box_first[b] = i;
    N.box_cnt[b]++;
  }
  N.nbr_ptr.assign(N.nbox + 1, 0);
  N.nbr_box.clear();
  N.ncols.assign(N.nbox, 0);
  N.base.assign(N.nbox + 1, 0);
  std::vector<uint64_t> nb;
  for (int a = 0; a < N.nbox; a++) {
    std::vector<int> lst;
    if (c->cfg.dense) {
      for (int b = 0; b < N.nbox; b++) lst.push_back(b);
    } else {
      neighbours(lb[a], l_max, nb);
      lst.push_back(a);
      for (uint64_t n : nb) {
        int b = index_of(lb, n);
        if (b >= 0) lst.push_back(b);
      }
      std::sort(lst.begin(), lst.end());
    }
    int nc = 0;
    for (int b : lst) {
      N.nbr_box.push_back(b);
      nc += N.box_cnt[b];
    }
    N.nbr_ptr[a + 1] = (int)N.nbr_box.size();
    N.ncols[a] = nc;
    N.base[a + 1] = N.base[a] + (long long)N.box_cnt[a] * nc;
  }
  N.nnz = N.base[N.nbox];
  return SIE_OK;
}

template <typename T>
static int upload(T** d, const std::vector<T>& h) {
  size_t n = std::max<size_t>(h.size(), 1);
  SIE_CUDA(cudaMalloc(d, n * sizeof(T)));
  if (!h.empty()) SIE_CUDA(h2d(*d, h.data(), h.size() * sizeof(T)));
  return SIE_OK;
}


// I4 interaction lists, children and parents of every level (lib_tree_get_domain_i4,
// lib_tree.f90:1096-1245).
static int build_levels(sie_ctx* c) {
  std::vector<uint64_t> par, own;
  for (int l = c->l_min; l <= c->l_max; l++) {
    Level& L = c->lv[l];
    std::vector<int> i4p(L.nb + 1, 0), i4s, i4o;
    for (int b = 0; b < L.nb; b++) {
      uint64_t n = L.box[b];
      if (!c->cfg.dense && l >= 1) {
        neighbours(n >> 3, l - 1, par);
        par.push_back(n >> 3);
        neighbours(n, l, own);
        own.push_back(n);
        std::sort(own.begin(), own.end());
        std::vector<uint64_t> cand;
        for (uint64_t p : par)
          for (uint64_t ch = 0; ch < 8; ch++) {
            uint64_t m = (p << 3) | ch;
            if (!std::binary_search(own.begin(), own.end(), m)) cand.push_back(m);
          }
        std::sort(cand.begin(), cand.end());
        int64_t ax, ay, az;
        demorton3(n, l, ax, ay, az);
        for (uint64_t m : cand) {
          int s = index_of(L.box, m);
          if (s < 0) continue;
          int64_t bx, by, bz;
          demorton3(m, l, bx, by, bz);
          int t = (int)((ax - bx + 3) * 49 + (ay - by + 3) * 7 + (az - bz + 3));
          i4s.push_back(s);
          i4o.push_back(t);
        }
      }
      i4p[b + 1] = (int)i4s.size();
    }
    L.n_i4 = (long long)i4s.size();
    SIE_TRY(upload(&L.i4_ptr, i4p));
    SIE_TRY(upload(&L.i4_src, i4s));
    SIE_TRY(upload(&L.i4_off, i4o));
    // sibling groups: parents at level l-1 and the children of their 27 neighbours
    {
      std::vector<uint64_t> parents;
      for (uint64_t n : L.box) parents.push_back(n >> 3);
      parents.erase(std::unique(parents.begin(), parents.end()), parents.end());
      std::vector<int> gs(parents.size() * 8, -1), gsrc(parents.size() * 216, -1);
      int64_t ub = (l >= 1) ? (((int64_t)1 << (l - 1)) - 1) : 0;
      for (size_t g = 0; g < parents.size(); g++) {
        uint64_t P = parents[g];
        for (int o = 0; o < 8; o++) gs[g * 8 + o] = index_of(L.box, (P << 3) | (uint64_t)o);
        int64_t px, py, pz;
        demorton3(P, l - 1, px, py, pz);
        for (int d = 0; d < 27; d++) {
          int64_t a = px + d / 9 - 1, b = py + (d / 3) % 3 - 1, cc = pz + d % 3 - 1;
          if (l < 1 || a < 0 || b < 0 || cc < 0 || a > ub || b > ub || cc > ub) continue;
          uint64_t Pn = morton3(a, b, cc, l - 1);
          for (int ch = 0; ch < 8; ch++) gsrc[g * 216 + d * 8 + ch] = index_of(L.box, (Pn << 3) | (uint64_t)ch);
        }
      }
      L.ngrp = (int)parents.size();
      // descending work, stable: the SR kernels give each warp one group, and a block
      // lasts as long as its heaviest warp.  Every box has one group, and a group writes
      // only its own boxes, so the order changes no result.
      std::vector<int> cost(L.ngrp), ord(L.ngrp);
      for (int g = 0; g < L.ngrp; g++) {
        int ns = 0, cnt = 0;
        for (int o = 0; o < 8; o++) ns += gs[(size_t)g * 8 + o] >= 0;
        for (int dc = 0; dc < 216; dc++) cnt += (dc >> 3) != 13 && gsrc[(size_t)g * 216 + dc] >= 0;
        cost[g] = ns * cnt;
        ord[g] = g;
      }
      std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
      std::vector<int> gs2(gs.size()), gsrc2(gsrc.size());
      L.grp_cost.resize(L.ngrp);
      for (int g = 0; g < L.ngrp; g++) {
        std::copy(gs.begin() + (size_t)ord[g] * 8, gs.begin() + (size_t)ord[g] * 8 + 8, gs2.begin() + (size_t)g * 8);
        std::copy(gsrc.begin() + (size_t)ord[g] * 216, gsrc.begin() + (size_t)ord[g] * 216 + 216,
                  gsrc2.begin() + (size_t)g * 216);
        L.grp_cost[g] = cost[ord[g]];
      }
      SIE_TRY(upload(&L.grp_sib, gs2));
      SIE_TRY(upload(&L.grp_src, gsrc2));
    }
    // children at l+1
    std::vector<int> chp(L.nb + 1, 0), chi, cho;
    if (l < c->l_max) {
      Level& C = c->lv[l + 1];
      for (int b = 0; b < L.nb; b++) {
        for (uint64_t o = 0; o < 8; o++) {
          int ci = index_of(C.box, (L.box[b] << 3) | o);
          if (ci >= 0) {
            chi.push_back(ci);
            cho.push_back((int)o);
          }
        }
        chp[b + 1] = (int)chi.size();
      }
    }
    SIE_TRY(upload(&L.ch_ptr, chp));
    SIE_TRY(upload(&L.ch_idx, chi));
    SIE_TRY(upload(&L.ch_oct, cho));
    std::vector<int> pa(L.nb, -1), oc(L.nb, 0);
    if (l > c->l_min) {
      Level& P = c->lv[l - 1];
      for (int b = 0; b < L.nb; b++) {
        pa[b] = index_of(P.box, L.box[b] >> 3);
        oc[b] = (int)(L.box[b] & 7);
      }
    }
    SIE_TRY(upload(&L.parent, pa));
    SIE_TRY(upload(&L.oct, oc));
  }
  return SIE_OK;
}

// Gauss-Legendre nodes, ascending (the reference uses the Glaser-Liu-Rokhlin
// rule, src/Gauss_Quadrature_Fast.f90:424-498; both are exact to rounding).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  auto leg = [n](double z, double& pn, double& dpn) {
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    pn = p1;
    dpn = n * (z * p1 - p0) / (z * z - 1.0);
  };
  for (int i = 0; i < n; i++) {
    double z = std::cos(PI * (i + 0.75) / (n + 0.5));
    double pn, dp;
    int extra = 0;
    for (int it = 0; it < 100 && extra < 2; it++) {
      leg(z, pn, dp);
      double dz = pn / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-15) extra++;
    }
    leg(z, pn, dp);
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1 - z * z) * dp * dp);
  }
}

// Khat_and_TRF_ExtendedK (src/lib_sie_mlfmm.f90:190-240): directions, transfer vectors
// and quadrature weights of the K sampling, poles last.
static void sampling_tables(int K, std::vector<double>& kh, std::vector<double>& th, std::vector<double>& ph,
                            std::vector<double>& trf) {
  const int Ns = 2 * K * K, Q = Ns + 2;
  std::vector<double> xx, ww;
  gauss_legendre(K, xx, ww);
  kh.assign(3 * (size_t)Q, 0.0);
  th.assign(3 * (size_t)Q, 0.0);
  ph.assign(3 * (size_t)Q, 0.0);
  trf.assign(Q, 0.0);
  double dphi = 2 * PI / (2 * K);
  for (int j = 0; j < K; j++)
    for (int k = 0; k < 2 * K; k++) {
      double phi = k * dphi;
      int i = k + j * 2 * K;
      double st = std::sin(std::acos(xx[j]));
      kh[3 * i] = st * std::cos(phi);
      kh[3 * i + 1] = st * std::sin(phi);
      kh[3 * i + 2] = xx[j];
      th[3 * i] = xx[j] * std::cos(phi);
      th[3 * i + 1] = xx[j] * std::sin(phi);
      th[3 * i + 2] = -st;
      ph[3 * i] = -std::sin(phi);
      ph[3 * i + 1] = std::cos(phi);
      ph[3 * i + 2] = 0.0;
      trf[i] = ww[j] * dphi;
    }
  double pk[2][3] = {{0, 0, 1}, {0, 0, -1}};
  for (int p = 0; p < 2; p++) {
    int i = Ns + p;
    for (int d = 0; d < 3; d++) kh[3 * i + d] = pk[p][d];
    th[3 * i] = 1; th[3 * i + 1] = 0; th[3 * i + 2] = 0;
    ph[3 * i] = 0; ph[3 * i + 1] = 1; ph[3 * i + 2] = 0;
    trf[i] = 0.0;
  }
}

// Truncation number of level l: the one requested for it, else the configuration's.
static int level_truncation(const sie_ctx* c, int l) {
  return (l < (int)c->level_K.size() && c->level_K[l] > 0) ? c->level_K[l] : c->cfg.truncation_number;
}

// Samplings of every level.  The leaf level's is also the context's own (c->K, c->Q and
// the d_khat/d_tth/d_tph/d_trf arrays: radiation patterns, aggregate and receive).
static int build_sampling(sie_ctx* c) {
  for (int l = c->l_min; l < c->l_max; l++)
    if (level_truncation(c, l + 1) > level_truncation(c, l))
      return fail(SIE_ERR_ARG, "per-level truncation numbers must not grow from a level to its children");
  c->level_k = false;
  for (int l = c->l_min; l <= c->l_max; l++) {
    Level& L = c->lv[l];
    L.K = level_truncation(c, l);
    L.Q = 2 * L.K * L.K + 2;
    c->level_k |= L.K != level_truncation(c, c->l_max);
    std::vector<double> kh, th, ph, trf;
    sampling_tables(L.K, kh, th, ph, trf);
    SIE_TRY(upload(&L.khat, kh));
    SIE_TRY(upload(&L.trf, trf));
  }
  int K = level_truncation(c, c->l_max), Ns = 2 * K * K, Q = Ns + 2;
  c->K = K;
  c->Q = Q;
  std::vector<double> kh, th, ph, trf;
  sampling_tables(K, kh, th, ph, trf);
  // direction of -khat for every direction (used by the transposed product): theta ->
  // pi - theta is Gauss node K-1-j, phi -> phi + pi is k + K, and the two poles swap
  std::vector<int> qp(Q);
  for (int j = 0; j < K; j++)
    for (int k = 0; k < 2 * K; k++) qp[k + j * 2 * K] = (k + K) % (2 * K) + (K - 1 - j) * 2 * K;
  qp[Ns] = Ns + 1;
  qp[Ns + 1] = Ns;
  for (int i = 0; i < Q; i++)
    for (int d = 0; d < 3; d++)
      if (std::fabs(kh[3 * qp[i] + d] + kh[3 * i + d]) > 1e-12)
        return fail(SIE_ERR_STATE, "k-space sampling is not symmetric under khat -> -khat");
  SIE_TRY(upload(&c->d_qperm, qp));
  SIE_TRY(upload(&c->d_khat, kh));
  SIE_TRY(upload(&c->d_tth, th));
  SIE_TRY(upload(&c->d_tph, ph));
  SIE_TRY(upload(&c->d_trf, trf));
  return SIE_OK;
}

// Interpolation (child -> parent) and anterpolation (parent -> child) matrices between
// level l and level l + 1 when their samplings differ (stencil of 2p x 2p, p = 3, as the
// reference's Lagrange_Interpolation_New calls use).
static int upload_interp(const Csr& A, InterpDev& d) {
  d.rows = A.rows;
  d.nnz = (long long)A.val.size();
  SIE_TRY(upload(&d.ptr, A.ptr));
  SIE_TRY(upload(&d.col, A.col));
  SIE_TRY(upload(&d.val, A.val));
  // ELL width: the row length that covers 99.5 % of the rows, a multiple of 4
  std::vector<int> len(A.rows);
  for (int r = 0; r < A.rows; r++) len[r] = A.ptr[r + 1] - A.ptr[r];
  std::vector<int> sorted_len = len;
  std::sort(sorted_len.begin(), sorted_len.end());
  int ew = A.rows ? sorted_len[std::min(A.rows - 1, (int)(0.995 * A.rows))] : 0;
  ew = (ew + 3) / 4 * 4;
  std::vector<int> ec((size_t)ew * A.rows, 0), op(A.rows + 1, 0), oc;
  std::vector<double> ev((size_t)ew * A.rows, 0.0), ov;
  for (int r = 0; r < A.rows; r++) {
    for (int k = A.ptr[r]; k < A.ptr[r + 1]; k++) {
      const int t = k - A.ptr[r];
      if (t < ew) {
        const size_t o = (size_t)t * A.rows + r;
        ec[o] = A.col[k];
        ev[o] = A.val[k];
      } else {
        oc.push_back(A.col[k]);
        ov.push_back(A.val[k]);
      }
    }
    op[r + 1] = (int)oc.size();
  }
  if (oc.empty()) {  // keep the overflow arrays non-empty
    oc.push_back(0);
    ov.push_back(0.0);
  }
  d.ew = ew;
  d.onnz = (long long)ov.size();
  SIE_TRY(upload(&d.ecol, ec));
  SIE_TRY(upload(&d.eval, ev));
  SIE_TRY(upload(&d.optr, op));
  SIE_TRY(upload(&d.ocol, oc));
  SIE_TRY(upload(&d.oval, ov));
  return SIE_OK;
}

static int build_interp(sie_ctx* c) {
  size_t tmp = 0;
  for (int l = c->l_min; l < c->l_max; l++) {
    Level& P = c->lv[l];
    Level& Ch = c->lv[l + 1];
    if (P.K == Ch.K) continue;
    Csr up, dn;
    SIE_TRY(interp_csr(3, Ch.K, P.K, false, up));
    SIE_TRY(interp_csr(3, Ch.K, P.K, true, dn));
    SIE_TRY(upload_interp(up, P.up));
    SIE_TRY(upload_interp(dn, P.dn));
    tmp = std::max(tmp, (size_t)Ch.nb * 8 * P.Q * sizeof(zc));
  }
  if (tmp) {
    SIE_CUDA(cudaMalloc(&c->d_lvtmp, tmp));
    c->lvtmp_bytes = tmp;
  }
  return SIE_OK;
}

static Material make_material(const sie_config& cfg) {
  Material m;
  auto csqrt = [](zc z) {
    double r = std::hypot(z.re, z.im);
    double a = std::sqrt((r + std::fabs(z.re)) / 2);
    if (a == 0.0) return mk<double>(0, 0);
    if (z.re >= 0) return mk<double>(a, z.im / (2 * a));
    return mk<double>(std::fabs(z.im) / (2 * a), z.im >= 0 ? a : -a);
  };
  m.k0 = 2 * PI / cfg.lambda;
  m.omega = 2 * PI * C0 / cfg.lambda;
  m.my1 = MU0;
  m.my2 = MU0;
  zc er1 = mk<double>(cfg.eps_r1_re, cfg.eps_r1_im), er2 = mk<double>(cfg.eps_r2_re, cfg.eps_r2_im);
  m.k1 = csqrt(er1) * m.k0;
  m.k2 = csqrt(er2) * m.k0;
  m.eps1 = er1 * EPS0;
  m.eps2 = er2 * EPS0;
  m.eta1 = csqrt(mk<double>(m.my1, 0) / m.eps1);
  m.eta2 = csqrt(mk<double>(m.my2, 0) / m.eps2);
  m.eta_a = (m.eta1 + m.eta2) * 0.5;
  return m;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Device staging for the host-buffer entry points (input and output halves), kept per
// context and only grown: a cudaMalloc/cudaFree pair per call costs a device-wide
// synchronisation and, measured on the slab workload, up to ~0.1 s per solve.
static int io_buffers(sie_ctx* c, size_t bytes, zc** in, zc** out) {
  size_t half = (bytes + 255) & ~(size_t)255;
  if (c->io_bytes < 2 * half) {
    if (c->d_io) cudaFree(c->d_io);
    c->d_io = nullptr;
    c->io_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_io, 2 * half));
    c->io_bytes = 2 * half;
  }
  *in = (zc*)c->d_io;
  *out = (zc*)((char*)c->d_io + c->io_bytes / 2);
  return SIE_OK;
}

static int ensure_work(sie_ctx* c, int nrhs) {
  if ((size_t)nrhs <= c->work_rhs) return SIE_OK;
  if (c->d_xi) cudaFree(c->d_xi);
  if (c->d_yi) cudaFree(c->d_yi);
  c->d_xi = c->d_yi = nullptr;
  size_t n = (size_t)2 * c->M * nrhs;
  SIE_CUDA(cudaMalloc(&c->d_xi, n * sizeof(zc)));
  SIE_CUDA(cudaMalloc(&c->d_yi, n * sizeof(zc)));
  c->work_rhs = nrhs;
  return SIE_OK;
}

// complex64 vectors of a batched mixed-precision product
int ensure_batch32(sie_ctx* c, int nrhs) {
  if ((size_t)nrhs <= c->b32_rhs) return SIE_OK;
  if (c->d_xb32) cudaFree(c->d_xb32);
  if (c->d_yb32) cudaFree(c->d_yb32);
  c->d_xb32 = c->d_yb32 = nullptr;
  c->b32_rhs = 0;
  size_t n = (size_t)2 * c->M * nrhs;
  SIE_CUDA(cudaMalloc(&c->d_xb32, n * sizeof(cc)));
  SIE_CUDA(cudaMalloc(&c->d_yb32, n * sizeof(cc)));
  c->b32_rhs = nrhs;
  return SIE_OK;
}

}  // namespace sie

using namespace sie;

// Device matvec on internal-layout vectors: y = Z x (one right-hand side per call).
// Phase times of the product just queued (events 0, 6, 1..5 recorded by the passes).
static void record_phase_times(sie_ctx* c, cudaStream_t st) {
  cudaEventRecord(c->ev[7], st);
  cudaEventSynchronize(c->ev[7]);
  float a = 0;
  cudaEventElapsedTime(&a, c->ev[0], c->ev[7]);
  c->tm.mv_total_ms = a;
  cudaEventElapsedTime(&a, c->ev[0], c->ev[6]);
  c->tm.mv_near_ms = a;
  if (!c->cfg.dense) {
    cudaEventElapsedTime(&a, c->overlap_near ? c->ev[0] : c->ev[6], c->ev[1]);
    c->tm.mv_agg_ms = a;
    cudaEventElapsedTime(&a, c->ev[1], c->ev[2]);
    c->tm.mv_ss_ms = a;
    cudaEventElapsedTime(&a, c->ev[2], c->ev[3]);
    c->tm.mv_sr_ms = a;
    cudaEventElapsedTime(&a, c->ev[3], c->ev[4]);
    c->tm.mv_rr_ms = a;
    cudaEventElapsedTime(&a, c->ev[4], c->ev[5]);
    c->tm.mv_recv_ms = a;
  }
}

int sie_internal_matvec(sie_ctx* c, const zc* xi, zc* yi, int nrhs, cudaStream_t st, bool timed) {
  if (c->op_adjoint) {  // the solver is running the adjoint system Z^H lambda = g
    for (int r = 0; r < nrhs; r++)
      SIE_TRY(sie_internal_matvec_adj(c, xi + (size_t)r * 2 * c->M, yi + (size_t)r * 2 * c->M, st));
    return SIE_OK;
  }
  for (int r = 0; r < nrhs; r++) {
    const zc* x = xi + (size_t)r * 2 * c->M;
    zc* y = yi + (size_t)r * 2 * c->M;
    if (timed) cudaEventRecord(c->ev[0], st);
    if (!c->cfg.dense && c->overlap_near) {
      // the HBM-bound near product on stream2 overlaps the latency-bound translations
      // (mode 2: forked after the HBM-bound aggregate, so the two do not share bandwidth);
      // the receive waits for it because both write y
      const std::function<int()> fork = [&]() -> int {
        SIE_CUDA(cudaEventRecord(c->ev_fork, st));
        SIE_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
        SIE_TRY(near_matvec64(c, x, y, 1, false, c->stream2));
        if (timed) cudaEventRecord(c->ev[6], c->stream2);
        SIE_CUDA(cudaEventRecord(c->ev_join, c->stream2));
        return SIE_OK;
      };
      if (c->overlap_near == 1) SIE_TRY(fork());
      SIE_TRY(far_matvec64(c, x, y, st, timed ? c->ev : nullptr, c->ev_join,
                           c->overlap_near >= 2 ? &fork : nullptr));
    } else {
      SIE_TRY(near_matvec64(c, x, y, 1, false, st));
      if (timed) cudaEventRecord(c->ev[6], st);
      if (!c->cfg.dense) SIE_TRY(far_matvec64(c, x, y, st, timed ? c->ev : nullptr));
    }
    if (timed) record_phase_times(c, st);
  }
  return SIE_OK;
}

int sie_internal_matvec32(sie_ctx* c, const cc* x, cc* y, cudaStream_t st, bool timed) {
  if (timed) cudaEventRecord(c->ev[0], st);
  if (!c->cfg.dense && c->overlap_near) {
    const std::function<int()> fork = [&]() -> int {
      SIE_CUDA(cudaEventRecord(c->ev_fork, st));
      SIE_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
      SIE_TRY(near_matvec32(c, x, y, 1, false, c->stream2));
      if (timed) cudaEventRecord(c->ev[6], c->stream2);
      SIE_CUDA(cudaEventRecord(c->ev_join, c->stream2));
      return SIE_OK;
    };
    if (c->overlap_near == 1) SIE_TRY(fork());
    SIE_TRY(far_matvec32(c, x, y, st, timed ? c->ev : nullptr, c->ev_join,
                         c->overlap_near >= 2 ? &fork : nullptr));
  } else {
    SIE_TRY(near_matvec32(c, x, y, 1, false, st));
    if (timed) cudaEventRecord(c->ev[6], st);
    if (!c->cfg.dense) SIE_TRY(far_matvec32(c, x, y, st, timed ? c->ev : nullptr));
  }
  if (timed) record_phase_times(c, st);
  return SIE_OK;
}

// Batched products: the near panels write y, the far passes add into it.  As in the
// one-vector product, the near panels run on stream2 beside the translations and the
// receive waits for them.  Batches larger than SIE_BATCH_MAX go in slices.
template <typename T, typename NF, typename FF>
static int matvec_b_t(sie_ctx* c, const cx<T>* x, cx<T>* y, int R, cudaStream_t st, NF near, FF far) {
  const size_t n = (size_t)2 * c->M;
  for (int r0 = 0; r0 < R; r0 += SIE_BATCH_MAX) {
    const int nr = std::min(SIE_BATCH_MAX, R - r0);
    if (!c->cfg.dense && c->overlap_near) {
      const std::function<int()> fork = [&]() -> int {
        SIE_CUDA(cudaEventRecord(c->ev_fork, st));
        SIE_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
        SIE_TRY(near(c, x + r0 * n, y + r0 * n, nr, c->stream2));
        SIE_CUDA(cudaEventRecord(c->ev_join, c->stream2));
        return SIE_OK;
      };
      if (c->overlap_near == 1) SIE_TRY(fork());
      SIE_TRY(far(c, x + r0 * n, y + r0 * n, nr, st, c->ev_join, c->overlap_near >= 2 ? &fork : nullptr));
    } else {
      SIE_TRY(near(c, x + r0 * n, y + r0 * n, nr, st));
      if (!c->cfg.dense) SIE_TRY(far(c, x + r0 * n, y + r0 * n, nr, st, nullptr, nullptr));
    }
  }
  return SIE_OK;
}

__global__ void k_conj_inplace(zc* a, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i].im = -a[i].im;
}

// y = Z^H x = conj(Z^T conj(x)); x is conjugated in place and back.  The transposed near
// panels write y, the transposed far passes add into it.
int sie_internal_matvec_adj(sie_ctx* c, const zc* x, zc* y, cudaStream_t st) {
  const size_t n = (size_t)2 * c->M;
  zc* xw = const_cast<zc*>(x);
  k_conj_inplace<<<296, 256, 0, st>>>(xw, n); sie::count_launch();
  SIE_TRY(near_matvec_adj64(c, x, y, st));
  if (!c->cfg.dense) SIE_TRY(far_matvec_adj64(c, x, y, st));
  k_conj_inplace<<<296, 256, 0, st>>>(xw, n); sie::count_launch();
  k_conj_inplace<<<296, 256, 0, st>>>(y, n); sie::count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}

int sie_internal_matvec_b(sie_ctx* c, const zc* x, zc* y, int R, cudaStream_t st) {
  return matvec_b_t<double>(c, x, y, R, st, near_matvec_b64, far_matvec_b64);
}

int sie_internal_matvec_b32(sie_ctx* c, const cc* x, cc* y, int R, cudaStream_t st) {
  return matvec_b_t<float>(c, x, y, R, st, near_matvec_b32, far_matvec_b32);
}

extern "C" {

void sie_config_default(sie_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->lambda = 500e-9;
  cfg->eps_r1_re = 1.0;
  cfg->eps_r1_im = 0.0;
  cfg->eps_r2_re = 18.392;
  cfg->eps_r2_im = -0.4164;
  cfg->formulation = SIE_ICTF;
  cfg->ngp = 3;
  cfg->tree_s_opt = 250;
  cfg->truncation_number = 19;
  cfg->normal_convention = 2;
  cfg->fix_itbn = 0;
  cfg->device = 0;
  cfg->dense = 0;
}

void sie_solver_default(sie_solver_cfg* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->restart = 50;
  cfg->max_iterations = 650;
  cfg->tolerance = 1e-6;
  cfg->use_initial_guess = 0;
  cfg->precision = SIE_FP64;
  cfg->inner_restart = 30;
  cfg->inner_tolerance = 1e-4;
  cfg->time_limit_s = 0;
}

const char* sie_last_error(void) { return g_err.c_str(); }

unsigned long long sie_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int sie_set_stream(sie_ctx* c, void* stream) {
  if (!c) return fail(SIE_ERR_ARG, "sie_set_stream: null context");
  SIE_CUDA(cudaSetDevice(c->device));
  SIE_CUDA(cudaStreamSynchronize(c->stream));
  if (!c->own_stream) c->own_stream = c->stream;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return SIE_OK;
}
const char* sie_version(void) { return "specklesim_b200 0.1 (sm_100a)"; }

int sie_init(const sie_config* cfg, const double* verts, int nv, const int* tris, int nt,
             sie_ctx** out) {
  if (!cfg || !verts || !tris || !out) return fail(SIE_ERR_ARG, "sie_init: null argument");
  *out = nullptr;
  if (nv < 3 || nt < 2) return fail(SIE_ERR_ARG, "sie_init: mesh too small");
  if (!(cfg->lambda > 0)) return fail(SIE_ERR_ARG, "sie_init: lambda must be > 0");
  if (cfg->formulation != SIE_ICTF && cfg->formulation != SIE_PMCHWT)
    return fail(SIE_ERR_ARG, "sie_init: formulation must be SIE_ICTF or SIE_PMCHWT");
  Rule R = make_rule(cfg->ngp);
  if (R.n == 0) return fail(SIE_ERR_ARG, "sie_init: ngp must be one of 1,3,4,6,7,12");
  if (cfg->truncation_number < 1 || cfg->truncation_number > 60)
    return fail(SIE_ERR_ARG, "sie_init: truncation_number must be in 1..60");
  if (cfg->tree_s_opt < 1) return fail(SIE_ERR_ARG, "sie_init: tree_s_opt must be >= 1");
  for (int i = 0; i < 3 * nt; i++)
    if (tris[i] < 0 || tris[i] >= nv) return fail(SIE_ERR_MESH, "sie_init: vertex index out of range");
  for (int i = 0; i < 3 * nv; i++)
    if (!std::isfinite(verts[i])) return fail(SIE_ERR_NONFINITE, "sie_init: non-finite vertex");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(SIE_ERR_CUDA, "sie_init: no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(SIE_ERR_ARG, "sie_init: bad device");
  sie_ctx* c = new sie_ctx();
  c->cfg = *cfg;
  c->device = cfg->device;
  c->R = R;
  c->mt = make_material(*cfg);
  c->K = cfg->truncation_number;
  c->nv = nv;
  c->nt = nt;
  c->verts.assign(verts, verts + 3 * (size_t)nv);
  c->tris.assign(tris, tris + 3 * (size_t)nt);
  auto cleanup = [&](int r) {
    sie_free(c);
    return r;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return cleanup(fail(SIE_ERR_CUDA, "cudaSetDevice"));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(SIE_ERR_CUDA, "stream"));
  if (cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(SIE_ERR_CUDA, "stream"));
  for (int i = 0; i < 16; i++) cudaEventCreate(&c->ev[i]);
  cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
  int r = build_mesh(c);
  if (r != SIE_OK) return cleanup(r);
  r = build_tree(c);
  if (r != SIE_OK) return cleanup(r);
  // ICTF: D21 = -eta_a^2 D12 ; PMCHWT: D21 = -D12
  c->cfac = (cfg->formulation == SIE_ICTF) ? -(c->mt.eta_a * c->mt.eta_a) : mk<double>(-1.0, 0.0);
  // kernel variant of the SR translation (tuning knob; both give the same sums)
  if (const char* e = getenv("SIE_SR_MODE")) c->sr_mode = std::max(0, std::min(5, atoi(e)));
  if (const char* e = getenv("SIE_RECV_MODE")) c->recv_mode = std::max(0, std::min(1, atoi(e)));
  if (const char* e = getenv("SIE_AGG_MODE")) c->agg_mode = std::max(0, std::min(1, atoi(e)));
  if (const char* e = getenv("SIE_NEAR_MODE")) c->near_mode = std::max(0, std::min(2, atoi(e)));
  if (const char* e = getenv("SIE_ARNOLDI_MODE")) c->arnoldi_mode = std::max(0, std::min(2, atoi(e)));
  if (const char* e = getenv("SIE_OVERLAP")) c->overlap_near = std::max(0, std::min(3, atoi(e)));
  *out = c;
  return SIE_OK;
}

int sie_info(const sie_ctx* c, int* n_edges, int* l_min, int* l_max, long long* nnz) {
  if (!c) return fail(SIE_ERR_ARG, "sie_info: null context");
  if (n_edges) *n_edges = c->M;
  if (l_min) *l_min = c->l_min;
  if (l_max) *l_max = c->l_max;
  if (nnz) *nnz = c->near.nnz;
  return SIE_OK;
}

int sie_set_level_truncation(sie_ctx* c, const int* K, int n) {
  if (!c || n < 0 || (n > 0 && !K)) return fail(SIE_ERR_ARG, "sie_set_level_truncation: bad argument");
  if (c->setup_done) return fail(SIE_ERR_STATE, "sie_set_level_truncation: call it before sie_setup");
  for (int i = 0; i < n; i++)
    if (K[i] < 0 || K[i] > 200) return fail(SIE_ERR_ARG, "sie_set_level_truncation: truncation number out of range");
  c->level_K.assign(K, K + n);
  const int KL = level_truncation(c, c->l_max);
  for (int l = c->l_min; l < c->l_max; l++)
    if (level_truncation(c, l + 1) > level_truncation(c, l)) {
      c->level_K.clear();
      return fail(SIE_ERR_ARG, "sie_set_level_truncation: truncation numbers must not grow toward the leaf level");
    }
  c->K = KL;
  return SIE_OK;
}

int sie_num_directions(const sie_ctx* c, int* Q) {
  if (!c || !Q) return fail(SIE_ERR_ARG, "null argument");
  *Q = 2 * c->K * c->K + 2;
  return SIE_OK;
}

int sie_setup(sie_ctx* c) {
  if (!c) return fail(SIE_ERR_ARG, "sie_setup: null context");
  if (c->setup_done) return SIE_OK;
  SIE_CUDA(cudaSetDevice(c->device));
  auto t0 = std::chrono::steady_clock::now();
  int M = c->M;
  // internal-order fn table and per-edge data
  std::vector<FnD> fn(2 * (size_t)M);
  std::vector<double> rref(M);
  std::vector<int> ebox(M);
  for (int i = 0; i < M; i++) {
    int e = c->perm[i];
    fn[2 * i] = c->fn_ext[2 * e];
    fn[2 * i + 1] = c->fn_ext[2 * e + 1];
    const double* a = &c->cent[3 * c->elem[2 * e]];
    const double* b = &c->cent[3 * c->elem[2 * e + 1]];
    rref[i] = std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
                        (a[2] - b[2]) * (a[2] - b[2]));
  }
  for (int b = 0; b < c->near.nbox; b++)
    for (int k = 0; k < c->near.box_cnt[b]; k++) ebox[c->near.box_first[b] + k] = b;
  SIE_TRY(upload(&c->d_fn, fn));
  SIE_TRY(upload(&c->d_rref, rref));
  SIE_TRY(upload(&c->d_cent, c->cent));
  SIE_TRY(upload(&c->d_perm, c->perm));
  SIE_TRY(upload(&c->d_edge_box, ebox));
  SIE_TRY(upload(&c->d_box_first, c->near.box_first));
  SIE_TRY(upload(&c->d_box_cnt, c->near.box_cnt));
  {
    // work units of the near-panel product and of the far-field receive: at most 32
    // edges (rows) of one leaf box
    std::vector<int> ch;
    for (int b = 0; b < c->near.nbox; b++)
      for (int k = 0; k < c->near.box_cnt[b]; k += 32) {
        ch.push_back(b);
        ch.push_back(c->near.box_first[b] + k);
        ch.push_back(std::min(32, c->near.box_cnt[b] - k));
        ch.push_back(0);
      }
    c->n_rchunk = (int)(ch.size() / 4);
    SIE_TRY(upload(&c->d_rchunk, ch));
    c->ncols_max = 0;
    for (int b = 0; b < c->near.nbox; b++) c->ncols_max = std::max(c->ncols_max, c->near.ncols[b]);
  }
  SIE_TRY(upload(&c->d_nbr_ptr, c->near.nbr_ptr));
  SIE_TRY(upload(&c->d_nbr_box, c->near.nbr_box));
  SIE_TRY(upload(&c->d_ncols, c->near.ncols));
  SIE_TRY(upload(&c->d_base, c->near.base));
  int* d_tv = nullptr;
  SIE_TRY(upload(&d_tv, c->tris));
  // near-field values
  size_t nnz = (size_t)c->near.nnz;
  SIE_CUDA(cudaMalloc(&c->d_na, std::max<size_t>(nnz, 1) * sizeof(zc)));
  SIE_CUDA(cudaMalloc(&c->d_nb, std::max<size_t>(nnz, 1) * sizeof(zc)));
  SIE_CUDA(cudaMalloc(&c->d_nd, std::max<size_t>(nnz, 1) * sizeof(zc)));
  cudaEventRecord(c->ev[8], c->stream);
  int r = near_fill(c, d_tv);
  cudaEventRecord(c->ev[9], c->stream);
  cudaFree(d_tv);
  if (r != SIE_OK) return r;
  SIE_TRY(near_prepare_kernels(c));
  SIE_TRY(diag_extract(c));
  // far field
  if (!c->cfg.dense) {
    SIE_TRY(build_sampling(c));
    SIE_TRY(build_levels(c));
    int Q = c->Q;
    std::vector<double> boxc(3 * (size_t)c->near.nbox);
    for (int b = 0; b < c->near.nbox; b++)
      box_centre(c, c->lv[c->l_max].box[b], c->l_max, &boxc[3 * b]);
    SIE_TRY(upload(&c->d_boxc, boxc));
    const double* d_boxc = c->d_boxc;
    SIE_CUDA(cudaMalloc(&c->d_rt, (size_t)M * 4 * Q * sizeof(zc)));
    for (int l = c->l_min; l <= c->l_max; l++) {
      Level& L = c->lv[l];
      // the shift tables of level l live on its parent's sampling
      const Level& S = c->lv[l > c->l_min ? l - 1 : l];
      SIE_CUDA(cudaMalloc(&L.C, (size_t)L.nb * 8 * L.Q * sizeof(zc)));
      SIE_CUDA(cudaMalloc(&L.D, (size_t)L.nb * 8 * L.Q * sizeof(zc)));
      SIE_CUDA(cudaMalloc(&L.tl, (size_t)343 * 2 * L.Q * sizeof(zc)));
      SIE_CUDA(cudaMalloc(&L.ph_up, (size_t)8 * 2 * S.Q * sizeof(zc)));
      SIE_CUDA(cudaMalloc(&L.ph_dn, (size_t)8 * 2 * S.Q * sizeof(zc)));
      SIE_TRY(phase_tables(c, L, l, S.khat, S.Q));
    }
    SIE_TRY(build_interp(c));
    cudaEventRecord(c->ev[10], c->stream);
    r = far_build_tables(c, d_boxc);
    cudaEventRecord(c->ev[11], c->stream);
    if (r != SIE_OK) return r;
    SIE_TRY(far_prepare_kernels(c));
  }
  SIE_CUDA(cudaStreamSynchronize(c->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[8], c->ev[9]);
  c->tm.fill_ms = ms;
  if (!c->cfg.dense) {
    cudaEventElapsedTime(&ms, c->ev[10], c->ev[11]);
    c->tm.rt_ms = ms;
  }
  c->tm.setup_ms = ms_since(t0);
  c->setup_done = true;
  return SIE_OK;
}

int sie_matvec_device(sie_ctx* c, const double* d_x, double* d_y, int nrhs, int precision,
                      void* stream) {
  if (!c || !d_x || !d_y || nrhs < 1) return fail(SIE_ERR_ARG, "sie_matvec_device: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_matvec_device: sie_setup not called");
  if (precision != SIE_FP64 && precision != SIE_MIXED)
    return fail(SIE_ERR_ARG, "sie_matvec_device: bad precision");
  SIE_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  SIE_TRY(ensure_work(c, nrhs));
  SIE_TRY(gather_ext_to_int(c, (const zc*)d_x, c->d_xi, nrhs, st));
  if (nrhs > 1) {
    // the vectors go through the product together: one read of the tables per batch
    cudaEventRecord(c->ev[0], st);
    if (precision == SIE_MIXED) {
      SIE_TRY(make_f32_tables(c));
      SIE_TRY(ensure_batch32(c, nrhs));
      size_t n = (size_t)2 * c->M * nrhs;
      SIE_TRY(to_c64(c->d_xi, c->d_xb32, n, st));
      SIE_TRY(sie_internal_matvec_b32(c, c->d_xb32, c->d_yb32, nrhs, st));
      SIE_TRY(to_c128(c->d_yb32, c->d_yi, n, st));
    } else {
      SIE_TRY(sie_internal_matvec_b(c, c->d_xi, c->d_yi, nrhs, st));
    }
    cudaEventRecord(c->ev[7], st);
    SIE_TRY(scatter_int_to_ext(c, c->d_yi, (zc*)d_y, nrhs, st));
    SIE_CUDA(cudaStreamSynchronize(st));
    float a = 0;
    cudaEventElapsedTime(&a, c->ev[0], c->ev[7]);
    c->tm.mv_total_ms = a;
    return SIE_OK;
  }
  if (precision == SIE_MIXED) {
    // complex64 product: tables and vectors in FP32, result widened back to FP64
    SIE_TRY(make_f32_tables(c));
    size_t n = (size_t)2 * c->M;
    for (int r = 0; r < nrhs; r++) {
      SIE_TRY(to_c64(c->d_xi + r * n, c->d_xi32, n, st));
      SIE_TRY(sie_internal_matvec32(c, c->d_xi32, c->d_yi32, st, r == nrhs - 1));
      SIE_TRY(to_c128(c->d_yi32, c->d_yi + r * n, n, st));
    }
  } else {
    SIE_TRY(sie_internal_matvec(c, c->d_xi, c->d_yi, nrhs, st, true));
  }
  SIE_TRY(scatter_int_to_ext(c, c->d_yi, (zc*)d_y, nrhs, st));
  SIE_CUDA(cudaStreamSynchronize(st));
  return SIE_OK;
}

int sie_matvec(sie_ctx* c, const double* x, double* y, int nrhs, int precision) {
  if (!c || !x || !y || nrhs < 1) return fail(SIE_ERR_ARG, "sie_matvec: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_matvec: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  size_t bytes = (size_t)2 * c->M * nrhs * sizeof(zc);
  for (size_t i = 0; i < (size_t)4 * c->M * nrhs; i++)
    if (!std::isfinite(x[i])) return fail(SIE_ERR_NONFINITE, "sie_matvec: non-finite input");
  zc *dx = nullptr, *dy = nullptr;
  SIE_TRY(io_buffers(c, bytes, &dx, &dy));
  int r = SIE_OK;
  if (cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    r = fail(SIE_ERR_CUDA, "sie_matvec: H2D copy");
  if (r == SIE_OK) r = sie_matvec_device(c, (const double*)dx, (double*)dy, nrhs, precision, c->stream);
  if (r == SIE_OK && (cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                      cudaStreamSynchronize(c->stream) != cudaSuccess))
    r = fail(SIE_ERR_CUDA, "sie_matvec: D2H copy");
  return r;
}

// Minimum over `reps` products (after two warm-up ones) of the device time of one product
// of the given precision on fixed vectors.
static int time_product(sie_ctx* c, int precision, int reps, double& ms) {
  cudaStream_t st = c->stream;
  ms = 1e300;
  for (int i = 0; i < reps + 2; i++) {
    cudaEventRecord(c->ev[8], st);
    if (precision == SIE_MIXED)
      SIE_TRY(sie_internal_matvec32(c, c->d_xi32, c->d_yi32, st, false));
    else
      SIE_TRY(sie_internal_matvec(c, c->d_xi, c->d_yi, 1, st, false));
    cudaEventRecord(c->ev[9], st);
    SIE_CUDA(cudaEventSynchronize(c->ev[9]));
    float a = 0;
    cudaEventElapsedTime(&a, c->ev[8], c->ev[9]);
    if (i >= 2) ms = std::min(ms, (double)a);
  }
  return SIE_OK;
}

int sie_autotune(sie_ctx* c, int precision, double* ms, int* modes) {
  if (!c) return fail(SIE_ERR_ARG, "sie_autotune: null context");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_autotune: sie_setup not called");
  if (precision != SIE_FP64 && precision != SIE_MIXED) return fail(SIE_ERR_ARG, "sie_autotune: bad precision");
  SIE_CUDA(cudaSetDevice(c->device));
  SIE_TRY(ensure_work(c, 1));
  if (precision == SIE_MIXED) SIE_TRY(make_f32_tables(c));
  const size_t n = (size_t)2 * c->M;
  // fixed finite inputs (the values do not change the work)
  SIE_CUDA(cudaMemsetAsync(c->d_xi, 0x3f, n * sizeof(zc), c->stream));
  if (precision == SIE_MIXED) SIE_CUDA(cudaMemsetAsync(c->d_xi32, 0x3f, n * sizeof(cc), c->stream));
  // coordinate descent over the variant knobs, each at its best value so far
  int* knob[5] = {&c->near_mode, &c->agg_mode, &c->sr_mode, &c->recv_mode, &c->overlap_near};
  const int lo[5] = {0, 0, 1, 0, 0}, hi[5] = {2, 1, 5, 1, 3};
  double best = 0;
  SIE_TRY(time_product(c, precision, 5, best));
  if (ms) ms[0] = best;
  for (int k = 0; k < 5; k++) {
    if (c->cfg.dense && k > 0) break;  // a dense context has no far passes
    const int keep = *knob[k];
    int arg = keep;
    for (int v = lo[k]; v <= hi[k]; v++) {
      if (v == keep) continue;
      *knob[k] = v;
      double t = 0;
      SIE_TRY(time_product(c, precision, 5, t));
      if (t < best) {
        best = t;
        arg = v;
      }
    }
    *knob[k] = arg;
  }
  if (ms) ms[1] = best;
  if (modes)
    for (int k = 0; k < 5; k++) modes[k] = *knob[k];
  return SIE_OK;
}

int sie_set_inner_operator(sie_ctx* c, sie_ctx* inner) {
  if (!c) return fail(SIE_ERR_ARG, "sie_set_inner_operator: null context");
  if (inner) {
    if (!c->setup_done || !inner->setup_done) return fail(SIE_ERR_STATE, "sie_set_inner_operator: sie_setup not called");
    if (inner == c || inner->M != c->M || inner->perm != c->perm || inner->device != c->device)
      return fail(SIE_ERR_ARG, "sie_set_inner_operator: needs a different context on the same mesh, tree and device");
    if (inner->inner) return fail(SIE_ERR_ARG, "sie_set_inner_operator: the inner context has an inner operator itself");
  }
  c->inner = inner;
  return SIE_OK;
}

int sie_matvec_adjoint_device(sie_ctx* c, const double* d_x, double* d_y, int nrhs, void* stream) {
  if (!c || !d_x || !d_y || nrhs < 1) return fail(SIE_ERR_ARG, "sie_matvec_adjoint_device: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_matvec_adjoint_device: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  SIE_TRY(ensure_work(c, nrhs));
  SIE_TRY(gather_ext_to_int(c, (const zc*)d_x, c->d_xi, nrhs, st));
  const size_t n = (size_t)2 * c->M;
  for (int r = 0; r < nrhs; r++) SIE_TRY(sie_internal_matvec_adj(c, c->d_xi + r * n, c->d_yi + r * n, st));
  SIE_TRY(scatter_int_to_ext(c, c->d_yi, (zc*)d_y, nrhs, st));
  SIE_CUDA(cudaStreamSynchronize(st));
  return SIE_OK;
}

int sie_matvec_adjoint(sie_ctx* c, const double* x, double* y, int nrhs) {
  if (!c || !x || !y || nrhs < 1) return fail(SIE_ERR_ARG, "sie_matvec_adjoint: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_matvec_adjoint: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  size_t bytes = (size_t)2 * c->M * nrhs * sizeof(zc);
  for (size_t i = 0; i < (size_t)4 * c->M * nrhs; i++)
    if (!std::isfinite(x[i])) return fail(SIE_ERR_NONFINITE, "sie_matvec_adjoint: non-finite input");
  zc *dx = nullptr, *dy = nullptr;
  SIE_TRY(io_buffers(c, bytes, &dx, &dy));
  int r = SIE_OK;
  if (cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    r = fail(SIE_ERR_CUDA, "sie_matvec_adjoint: H2D copy");
  if (r == SIE_OK) r = sie_matvec_adjoint_device(c, (const double*)dx, (double*)dy, nrhs, c->stream);
  if (r == SIE_OK && (cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                      cudaStreamSynchronize(c->stream) != cudaSuccess))
    r = fail(SIE_ERR_CUDA, "sie_matvec_adjoint: D2H copy");
  return r;
}

int sie_quadrature_rule(int ngp, double* alpha, double* beta, double* w, int* n) {
  if (!alpha || !beta || !w || !n) return fail(SIE_ERR_ARG, "sie_quadrature_rule: null argument");
  const Rule r = make_rule(ngp);
  if (r.n == 0) return fail(SIE_ERR_ARG, "sie_quadrature_rule: ngp must be 1, 3, 4, 6, 7 or 12");
  for (int i = 0; i < r.n; i++) {
    alpha[i] = r.a[i];
    beta[i] = r.b[i];
    w[i] = r.w[i];
  }
  *n = r.n;
  return SIE_OK;
}

int sie_incidence(double theta, double phi, int pol, int k_dir, double* k_in, double* E_in) {
  if (!k_in || !E_in) return fail(SIE_ERR_ARG, "sie_incidence: null argument");
  if (k_dir != 1 && k_dir != 2) return fail(SIE_ERR_ARG, "sie_incidence: k_dir must be 1 or 2");
  double sgn = (k_dir == 1) ? 1.0 : -1.0;
  double ep[2] = {pol == 1 ? 1.0 : 0.0, pol == 1 ? 0.0 : 1.0};
  k_in[0] = std::sin(theta) * std::cos(phi);
  k_in[1] = std::sin(theta) * std::sin(phi);
  k_in[2] = sgn * std::cos(theta);
  // field_rotation_matrix (main.f90:297-323)
  double a = std::sin(theta), b = std::cos(theta), cc = std::sin(phi), d = std::cos(phi);
  double Rm[3][2] = {{d * d * b + cc * cc, cc * d * (b - 1)},
                     {cc * d * (b - 1), cc * cc * b + d * d},
                     {a * d, a * cc}};
  for (int i = 0; i < 3; i++) E_in[i] = Rm[i][0] * ep[0] + Rm[i][1] * ep[1];
  return SIE_OK;
}

int sie_rhs_planewave(sie_ctx* c, const double* k_in, const double* E_in, int nrhs, double* b) {
  if (!c || !k_in || !E_in || !b || nrhs < 1) return fail(SIE_ERR_ARG, "sie_rhs_planewave: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_rhs_planewave: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  SIE_TRY(ensure_work(c, nrhs));
  double *dk = nullptr, *dE = nullptr;
  zc* db = nullptr;
  size_t bytes = (size_t)2 * c->M * nrhs * sizeof(zc);
  SIE_CUDA(cudaMalloc(&dk, 3 * nrhs * sizeof(double)));
  SIE_CUDA(cudaMalloc(&dE, 3 * nrhs * sizeof(double)));
  SIE_CUDA(cudaMalloc(&db, bytes));
  SIE_CUDA(h2d(dk, k_in, 3 * nrhs * sizeof(double)));
  SIE_CUDA(h2d(dE, E_in, 3 * nrhs * sizeof(double)));
  int r = rhs_planewave_dev(c, dk, dE, nrhs, c->d_yi);
  if (r == SIE_OK) r = scatter_int_to_ext(c, c->d_yi, db, nrhs, c->stream);
  if (r == SIE_OK && (cudaStreamSynchronize(c->stream) != cudaSuccess ||
                      cudaMemcpy(b, db, bytes, cudaMemcpyDeviceToHost) != cudaSuccess))
    r = fail(SIE_ERR_CUDA, "sie_rhs_planewave: D2H copy");
  cudaFree(dk);
  cudaFree(dE);
  cudaFree(db);
  return r;
}

int sie_solve_device(sie_ctx* c, const double* d_b, double* d_x, int nrhs, const sie_solver_cfg* cfg,
                     sie_stats* stats) {
  if (!c || !d_b || !d_x || nrhs < 1 || !cfg) return fail(SIE_ERR_ARG, "sie_solve_device: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_solve_device: sie_setup not called");
  if (cfg->restart < 1 || cfg->max_iterations < 1 || !(cfg->tolerance > 0))
    return fail(SIE_ERR_ARG, "sie_solve_device: bad solver configuration");
  SIE_CUDA(cudaSetDevice(c->device));
  SIE_TRY(ensure_work(c, 1));
  int rc_all = SIE_OK;
  if (cfg->precision == SIE_MIXED && nrhs > 1) {
    // right-hand sides in batches: one batched product per step for the whole batch
    for (int r0 = 0; r0 < nrhs; r0 += SIE_BATCH_MAX) {
      const int nr = std::min(SIE_BATCH_MAX, nrhs - r0);
      const size_t off = (size_t)r0 * 2 * c->M;
      int rc = fgmres_mixed_batch(c, (const zc*)d_b + off, (zc*)d_x + off, nr, cfg, stats ? stats + r0 : nullptr);
      if (rc != SIE_OK && rc != SIE_ERR_NOCONV) return rc;
      if (rc == SIE_ERR_NOCONV) rc_all = rc;
    }
    return rc_all;
  }
  for (int r = 0; r < nrhs; r++) {
    const zc* b = (const zc*)d_b + (size_t)r * 2 * c->M;
    zc* x = (zc*)d_x + (size_t)r * 2 * c->M;
    sie_stats st;
    memset(&st, 0, sizeof(st));
    int rc = gmres_solve(c, b, x, cfg, &st);
    if (stats) stats[r] = st;
    if (rc != SIE_OK && rc != SIE_ERR_NOCONV) return rc;
    if (rc == SIE_ERR_NOCONV) rc_all = rc;
  }
  return rc_all;
}

int sie_solve(sie_ctx* c, const double* b, double* x, int nrhs, const sie_solver_cfg* cfg,
              sie_stats* stats) {
  if (!c || !b || !x || nrhs < 1 || !cfg) return fail(SIE_ERR_ARG, "sie_solve: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_solve: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  for (size_t i = 0; i < (size_t)4 * c->M * nrhs; i++)
    if (!std::isfinite(b[i])) return fail(SIE_ERR_NONFINITE, "sie_solve: non-finite right-hand side");
  size_t bytes = (size_t)2 * c->M * nrhs * sizeof(zc);
  zc *db = nullptr, *dx = nullptr;
  SIE_TRY(io_buffers(c, bytes, &db, &dx));
  SIE_CUDA(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, c->stream));
  if (cfg->use_initial_guess) SIE_CUDA(cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, c->stream));
  int r = sie_solve_device(c, (const double*)db, (double*)dx, nrhs, cfg, stats);
  if ((r == SIE_OK || r == SIE_ERR_NOCONV) &&
      (cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
       cudaStreamSynchronize(c->stream) != cudaSuccess))
    r = fail(SIE_ERR_CUDA, "sie_solve: D2H copy");
  return r;
}

// Gradient tables (once per context): side vertex ids in internal order, vertex
// coordinates and triangle vertices.
static int grad_tables(sie_ctx* c) {
  if (c->d_side) return SIE_OK;
  std::vector<int> sv(16 * (size_t)c->M);
  for (int i = 0; i < c->M; i++) {
    const int e = c->perm[i];
    for (int k = 0; k < 16; k++) sv[16 * (size_t)i + k] = c->side_v[16 * (size_t)e + k];
  }
  SIE_TRY(upload(&c->d_vert, c->verts));
  SIE_TRY(upload(&c->d_tri_verts, c->tris));
  SIE_TRY(upload(&c->d_side, sv));
  return SIE_OK;
}

int sie_grad(sie_ctx* c, const double* x, const double* k_in, const double* E_in, const double* pts, int npts,
             const sie_solver_cfg* cfg, double* dJdz, double* J, sie_stats* stats) {
  if (c && c->level_k)
    return fail(SIE_ERR_STATE, "sie_grad: not available with per-level truncation numbers");
  if (!c || !x || !k_in || !E_in || !pts || npts < 1 || !cfg || !dJdz)
    return fail(SIE_ERR_ARG, "sie_grad: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_grad: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  SIE_TRY(grad_tables(c));
  cudaStream_t st = c->stream;
  const size_t n = (size_t)2 * c->M;
  const size_t nl = c->cfg.dense ? 0 : (size_t)c->lv[c->l_max].nb * 8 * c->Q;
  // workspace: x, g, lambda (internal and external), E, H, I, pts, plane wave, grad, far part
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t o = need;
    need += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t ox = add(n * sizeof(zc)), oxe = add(n * sizeof(zc)), og = add(n * sizeof(zc)),
               oge = add(n * sizeof(zc)), ol = add(n * sizeof(zc)), ole = add(n * sizeof(zc)),
               oE = add(3 * (size_t)npts * sizeof(zc)), oH = add(3 * (size_t)npts * sizeof(zc)),
               oI = add((size_t)npts * sizeof(double)), op = add(3 * (size_t)npts * sizeof(double)),
               ok = add(6 * sizeof(double)), ogr = add((size_t)c->nv * sizeof(double)),
               ofar = add((2 * nl + n) * sizeof(zc));
  if (c->grad_ws_bytes < need) {
    if (c->d_grad_ws) cudaFree(c->d_grad_ws);
    c->d_grad_ws = nullptr;
    c->grad_ws_bytes = 0;
    SIE_CUDA(cudaMalloc(&c->d_grad_ws, need));
    c->grad_ws_bytes = need;
  }
  char* w = (char*)c->d_grad_ws;
  zc *xi = (zc*)(w + ox), *xe = (zc*)(w + oxe), *gi = (zc*)(w + og), *ge = (zc*)(w + oge);
  zc *li = (zc*)(w + ol), *le = (zc*)(w + ole), *dE = (zc*)(w + oE), *dH = (zc*)(w + oH);
  double *dI = (double*)(w + oI), *dp = (double*)(w + op), *dk = (double*)(w + ok), *dg = (double*)(w + ogr);
  SIE_CUDA(h2d(xe, x, n * sizeof(zc)));
  SIE_CUDA(h2d(dp, pts, 3 * (size_t)npts * sizeof(double)));
  SIE_CUDA(h2d(dk, k_in, 3 * sizeof(double)));
  SIE_CUDA(h2d(dk + 3, E_in, 3 * sizeof(double)));
  SIE_TRY(gather_ext_to_int(c, xe, xi, 1, st));
  // objective and the adjoint right-hand side dJ/dI*
  SIE_TRY(farfield_dev(c, xi, dp, npts, dE, dH, dI));
  SIE_TRY(field_adjoint_rhs(c, dE, dp, npts, gi, st));
  SIE_TRY(scatter_int_to_ext(c, gi, ge, 1, st));
  SIE_CUDA(cudaStreamSynchronize(st));
  if (J) {
    std::vector<double> I(npts);
    SIE_CUDA(cudaMemcpy(I.data(), dI, (size_t)npts * sizeof(double), cudaMemcpyDeviceToHost));
    double s = 0;
    for (double v : I) s += v;
    *J = s;
  }
  // adjoint solve Z^H lambda = g (FP64 GMRES on the conjugate-transpose product)
  sie_solver_cfg acfg = *cfg;
  acfg.precision = SIE_FP64;
  acfg.use_initial_guess = 0;
  sie_stats ast;
  memset(&ast, 0, sizeof(ast));
  SIE_TRY(ensure_work(c, 1));
  int rc = SIE_OK;
  if (c->cfg.dense) {  // the LU factors give the adjoint solution directly
    SIE_CUDA(cudaMemcpyAsync(li, gi, n * sizeof(zc), cudaMemcpyDeviceToDevice, st));
    SIE_TRY(lu_solve_adjoint(c, li));
    ast.converged = 1;
  } else {
    c->op_adjoint = 1;
    rc = gmres_solve(c, ge, le, &acfg, &ast);
    c->op_adjoint = 0;
    if (rc != SIE_OK && rc != SIE_ERR_NOCONV) {
      if (stats) *stats = ast;
      return rc;
    }
    SIE_TRY(gather_ext_to_int(c, le, li, 1, st));
  }
  if (stats) *stats = ast;
  // dJ/dz = explicit far-field term + 2 Re lambda^H (db - dZ I)
  const double h = 1e-6 * c->cfg.lambda;
  // SIE_GRAD_PARTS (bit mask, default all): 1 field factors, 2 right-hand side, 4 near
  // blocks, 8 far field -- for checking the terms one at a time
  int parts = 15;
  if (const char* e = getenv("SIE_GRAD_PARTS")) parts = atoi(e);
  SIE_CUDA(cudaMemsetAsync(dg, 0, (size_t)c->nv * sizeof(double), st));
  // the observation points are metres away (~1e7 lambda), so their distances carry an
  // absolute rounding of ~1e-16 m: the field factors take a step of 1e-4 lambda, where
  // the phase difference is well above that noise (truncation error ~(k h)^2 = 4e-7)
  if (parts & 1) SIE_TRY(grad_field(c, dE, dp, npts, xi, 1e-4 * c->cfg.lambda, dg, st));
  if (parts & 2) SIE_TRY(grad_rhs(c, li, dk, dk + 3, h, dg, st));
  if (parts & 4) SIE_TRY(grad_near(c, li, xi, h, dg, st));
  if ((parts & 8) && !c->cfg.dense) SIE_TRY(grad_far(c, li, xi, h, dg, w + ofar, st));
  SIE_CUDA(cudaStreamSynchronize(st));
  SIE_CUDA(cudaMemcpy(dJdz, dg, (size_t)c->nv * sizeof(double), cudaMemcpyDeviceToHost));
  return rc;
}

int sie_farfield(sie_ctx* c, const double* x, const double* pts, int npts, double* E, double* H,
                 double* intensity) {
  if (!c || !x || !pts || npts < 1) return fail(SIE_ERR_ARG, "sie_farfield: bad argument");
  SIE_CUDA(cudaSetDevice(c->device));
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_farfield: sie_setup not called");
  SIE_TRY(ensure_work(c, 1));
  size_t bytes = (size_t)2 * c->M * sizeof(zc);
  zc *dx = nullptr, *dE = nullptr, *dH = nullptr;
  double *dp = nullptr, *dI = nullptr;
  SIE_CUDA(cudaMalloc(&dx, bytes));
  SIE_CUDA(cudaMalloc(&dp, 3 * (size_t)npts * sizeof(double)));
  SIE_CUDA(cudaMalloc(&dE, 3 * (size_t)npts * sizeof(zc)));
  SIE_CUDA(cudaMalloc(&dH, 3 * (size_t)npts * sizeof(zc)));
  SIE_CUDA(cudaMalloc(&dI, (size_t)npts * sizeof(double)));
  SIE_CUDA(h2d(dx, x, bytes));
  SIE_CUDA(h2d(dp, pts, 3 * (size_t)npts * sizeof(double)));
  int r = gather_ext_to_int(c, dx, c->d_xi, 1, c->stream);
  if (r == SIE_OK) r = farfield_dev(c, c->d_xi, dp, npts, dE, dH, dI);
  if (r == SIE_OK) {
    cudaStreamSynchronize(c->stream);
    if (E) cudaMemcpy(E, dE, 3 * (size_t)npts * sizeof(zc), cudaMemcpyDeviceToHost);
    if (H) cudaMemcpy(H, dH, 3 * (size_t)npts * sizeof(zc), cudaMemcpyDeviceToHost);
    if (intensity) cudaMemcpy(intensity, dI, (size_t)npts * sizeof(double), cudaMemcpyDeviceToHost);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_fail(e, "sie_farfield copies");
  }
  cudaFree(dx);
  cudaFree(dp);
  cudaFree(dE);
  cudaFree(dH);
  cudaFree(dI);
  return r;
}

// Integration_scattered_field_tri_within_medium (:2829-2877) as two passes of the
// exterior field kernel in the interior medium (km = k0 sqrt(eps_r), mu_0,
// eps_2 = eps_0 eps_r): the negated currents give H and E without its scalar-potential
// term; the currents (J, M) = (0, -J / eps_2) with permeability 1 and permittivity 0 give,
// as their H, that term, -(1/(i w eps_2)) SE dfm grad G summed and negated like the rest.
int sie_field_interior(sie_ctx* c, const double* x, const double* pts, int npts, double eps_r_re, double eps_r_im,
                       double* E, double* H) {
  if (!c || !x || !pts || npts < 1) return fail(SIE_ERR_ARG, "sie_field_interior: bad argument");
  if (!std::isfinite(eps_r_re) || !std::isfinite(eps_r_im) || (eps_r_re == 0.0 && eps_r_im == 0.0))
    return fail(SIE_ERR_ARG, "sie_field_interior: eps_r must be finite and non-zero");
  SIE_CUDA(cudaSetDevice(c->device));
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_field_interior: sie_setup not called");
  SIE_TRY(ensure_work(c, 1));
  const int M = c->M;
  const std::complex<double> km = c->mt.k0 * std::sqrt(std::complex<double>(eps_r_re, eps_r_im));
  const zc eps2 = mk<double>(eps_r_re, eps_r_im) * EPS0;
  Material m1 = c->mt;
  m1.k1 = mk<double>(km.real(), km.imag());
  m1.my1 = MU0;
  m1.eps1 = eps2;
  Material m2 = m1;
  m2.my1 = 1.0;
  m2.eps1 = mk<double>(0, 0);
  const zc* xz = reinterpret_cast<const zc*>(x);
  std::vector<zc> xab((size_t)4 * M);  // the two passes' currents, external order
  for (int m = 0; m < M; m++) {
    xab[m] = -xz[m];
    xab[(size_t)M + m] = -xz[(size_t)M + m];
    xab[(size_t)2 * M + m] = mk<double>(0, 0);
    xab[(size_t)3 * M + m] = -(xz[m] / eps2);
  }
  const size_t vb = (size_t)2 * M * sizeof(zc), fb = 3 * (size_t)npts * sizeof(zc);
  zc *dx = nullptr, *dE = nullptr, *dH = nullptr;
  double *dp = nullptr, *dI = nullptr;
  int r = SIE_OK;
  if (cudaMalloc(&dx, 2 * vb) != cudaSuccess || cudaMalloc(&dp, 3 * (size_t)npts * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dE, 2 * fb) != cudaSuccess || cudaMalloc(&dH, 2 * fb) != cudaSuccess ||
      cudaMalloc(&dI, (size_t)npts * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    r = fail(SIE_ERR_NOMEM, "sie_field_interior: device memory");
  }
  if (r == SIE_OK && (h2d(dx, xab.data(), 2 * vb) != cudaSuccess ||
                      h2d(dp, pts, 3 * (size_t)npts * sizeof(double)) != cudaSuccess))
    r = fail(SIE_ERR_CUDA, "sie_field_interior: copies");
  // pass 1 into (dE, dH), pass 2 into the second halves; the gathers and kernels share
  // the context's stream, so pass 2's gather waits for pass 1's kernel
  if (r == SIE_OK) r = gather_ext_to_int(c, dx, c->d_xi, 1, c->stream);
  if (r == SIE_OK) r = farfield_dev(c, m1, c->d_xi, dp, npts, dE, dH, dI);
  if (r == SIE_OK) r = gather_ext_to_int(c, dx + 2 * (size_t)M, c->d_xi, 1, c->stream);
  if (r == SIE_OK) r = farfield_dev(c, m2, c->d_xi, dp, npts, dE + 3 * (size_t)npts, dH + 3 * (size_t)npts, dI);
  if (r == SIE_OK) {
    std::vector<zc> hE(6 * (size_t)npts), hH(6 * (size_t)npts);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
        cudaMemcpy(hE.data(), dE, 2 * fb, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hH.data(), dH, 2 * fb, cudaMemcpyDeviceToHost) != cudaSuccess) {
      r = cuda_fail(cudaGetLastError(), "sie_field_interior");
    } else {
      for (size_t i = 0; i < 3 * (size_t)npts; i++) {
        const zc e = hE[i] + hH[3 * (size_t)npts + i];
        if (E) {
          E[2 * i] = e.re;
          E[2 * i + 1] = e.im;
        }
        if (H) {
          H[2 * i] = hH[i].re;
          H[2 * i + 1] = hH[i].im;
        }
      }
    }
  }
  cudaFree(dx);
  cudaFree(dp);
  cudaFree(dE);
  cudaFree(dH);
  cudaFree(dI);
  return r;
}

int sie_get_edges(const sie_ctx* c, int* elem, int* corner) {
  if (!c || !elem || !corner) return fail(SIE_ERR_ARG, "sie_get_edges: null argument");
  std::copy(c->elem.begin(), c->elem.end(), elem);
  std::copy(c->corner.begin(), c->corner.end(), corner);
  return SIE_OK;
}

int sie_get_tree(const sie_ctx* c, double* D_xmin, long long* leaf) {
  if (!c) return fail(SIE_ERR_ARG, "sie_get_tree: null context");
  if (D_xmin) {
    D_xmin[0] = c->D;
    for (int d = 0; d < 3; d++) D_xmin[1 + d] = c->xmin[d];
  }
  if (leaf)
    for (int e = 0; e < c->M; e++) leaf[e] = (long long)c->leaf[e];
  return SIE_OK;
}

int sie_get_blocks(sie_ctx* c, const int* m, const int* n, int cnt, double* out) {
  if (!c || !m || !n || !out || cnt < 1) return fail(SIE_ERR_ARG, "sie_get_blocks: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_get_blocks: sie_setup not called");
  SIE_CUDA(cudaSetDevice(c->device));
  std::vector<int> mi(cnt), ni(cnt);
  for (int i = 0; i < cnt; i++) {
    if (m[i] < 0 || m[i] >= c->M || n[i] < 0 || n[i] >= c->M)
      return fail(SIE_ERR_ARG, "sie_get_blocks: edge index out of range");
    mi[i] = c->iperm[m[i]];
    ni[i] = c->iperm[n[i]];
  }
  int *dm = nullptr, *dn = nullptr, *dtv = nullptr;
  zc* dout = nullptr;
  SIE_TRY(upload(&dm, mi));
  SIE_TRY(upload(&dn, ni));
  SIE_TRY(upload(&dtv, c->tris));
  SIE_CUDA(cudaMalloc(&dout, (size_t)cnt * 3 * sizeof(zc)));
  int r = near_blocks_list(c, dtv, dm, dn, cnt, dout);
  std::vector<zc> h((size_t)cnt * 3);
  if (r == SIE_OK) {
    cudaStreamSynchronize(c->stream);
    if (cudaMemcpy(h.data(), dout, h.size() * sizeof(zc), cudaMemcpyDeviceToHost) != cudaSuccess)
      r = fail(SIE_ERR_CUDA, "sie_get_blocks: copy");
  }
  cudaFree(dm);
  cudaFree(dn);
  cudaFree(dtv);
  cudaFree(dout);
  if (r != SIE_OK) return r;
  for (int i = 0; i < cnt; i++) {
    zc a = h[3 * i], b = h[3 * i + 1], d = h[3 * i + 2];
    zc cc = c->cfac * b;
    zc v[4] = {a, b, cc, d};
    for (int k = 0; k < 4; k++) {
      out[8 * i + 2 * k] = v[k].re;
      out[8 * i + 2 * k + 1] = v[k].im;
    }
  }
  return SIE_OK;
}

int sie_get_near_entries(sie_ctx* c, const int* m, const int* n, int cnt, double* out) {
  if (!c || !m || !n || !out || cnt < 1) return fail(SIE_ERR_ARG, "sie_get_near_entries: bad argument");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_get_near_entries: sie_setup not called");
  const NearLayout& N = c->near;
  std::vector<long long> idx(cnt, -1);
  std::vector<int> ebox(c->M);
  for (int b = 0; b < N.nbox; b++)
    for (int k = 0; k < N.box_cnt[b]; k++) ebox[N.box_first[b] + k] = b;
  for (int i = 0; i < cnt; i++) {
    if (m[i] < 0 || m[i] >= c->M || n[i] < 0 || n[i] >= c->M)
      return fail(SIE_ERR_ARG, "sie_get_near_entries: edge index out of range");
    int mi = c->iperm[m[i]], ni = c->iperm[n[i]];
    int A = ebox[mi], B = ebox[ni];
    int col = 0;
    bool found = false;
    for (int k = N.nbr_ptr[A]; k < N.nbr_ptr[A + 1]; k++) {
      int bb = N.nbr_box[k];
      if (bb == B) {
        col += ni - N.box_first[B];
        found = true;
        break;
      }
      col += N.box_cnt[bb];
    }
    if (found) idx[i] = N.base[A] + (long long)(mi - N.box_first[A]) * N.ncols[A] + col;
  }
  for (int i = 0; i < cnt; i++) {
    zc v[3] = {mk<double>(0, 0), mk<double>(0, 0), mk<double>(0, 0)};
    if (idx[i] >= 0) {
      SIE_CUDA(cudaMemcpy(&v[0], c->d_na + idx[i], sizeof(zc), cudaMemcpyDeviceToHost));
      SIE_CUDA(cudaMemcpy(&v[1], c->d_nb + idx[i], sizeof(zc), cudaMemcpyDeviceToHost));
      SIE_CUDA(cudaMemcpy(&v[2], c->d_nd + idx[i], sizeof(zc), cudaMemcpyDeviceToHost));
    }
    zc cc = c->cfac * v[1];
    if (idx[i] < 0) cc = mk<double>(0, 0);
    zc w[4] = {v[0], v[1], cc, v[2]};
    for (int k = 0; k < 4; k++) {
      out[8 * i + 2 * k] = w[k].re;
      out[8 * i + 2 * k + 1] = w[k].im;
    }
  }
  return SIE_OK;
}

int sie_get_rt(sie_ctx* c, const int* edges, int cnt, double* out) {
  if (!c || !edges || !out || cnt < 1) return fail(SIE_ERR_ARG, "sie_get_rt: bad argument");
  if (!c->setup_done || !c->d_rt) return fail(SIE_ERR_STATE, "sie_get_rt: no radiation patterns");
  size_t per = (size_t)4 * c->Q;
  for (int i = 0; i < cnt; i++) {
    if (edges[i] < 0 || edges[i] >= c->M) return fail(SIE_ERR_ARG, "sie_get_rt: edge out of range");
    int ei = c->iperm[edges[i]];
    SIE_CUDA(cudaMemcpy(out + 2 * per * i, c->d_rt + per * ei, per * sizeof(zc), cudaMemcpyDeviceToHost));
  }
  return SIE_OK;
}

int sie_get_timings(const sie_ctx* c, double* out, int n) {
  if (!c || !out) return fail(SIE_ERR_ARG, "sie_get_timings: null argument");
  double v[23] = {c->tm.fill_ms, c->tm.rt_ms, c->tm.setup_ms, c->tm.mv_total_ms,
                  c->tm.mv_near_ms, c->tm.mv_agg_ms, c->tm.mv_ss_ms, c->tm.mv_sr_ms,
                  c->tm.mv_rr_ms, c->tm.mv_recv_ms,
                  c->tm.gm_steps > 0 ? c->tm.gm_passes / c->tm.gm_steps : 0.0, c->tm.graph_replays,
                  c->tm.precond_ms, c->tm.lu_factor_ms, c->tm.lu_gemm_ms, c->tm.lu_gemm_flops,
                  (double)c->tm.lu_gemm_launches, c->tm.lu_phase_ms[0], c->tm.lu_phase_ms[1],
                  c->tm.lu_phase_ms[2], c->tm.lu_phase_ms[3], (double)c->tm.lu_f16,
                  (double)c->tm.lu_factorizations};
  for (int i = 0; i < n && i < 23; i++) out[i] = v[i];
  return SIE_OK;
}

int sie_free(sie_ctx* c) {
  if (!c) return SIE_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  ras_release(c);
  void* ptrs[] = {c->d_fn, c->d_rref, c->d_cent, c->d_perm, c->d_box_first, c->d_box_cnt,
                  c->d_nbr_ptr, c->d_nbr_box, c->d_ncols, c->d_base, c->d_edge_box, c->d_rchunk, c->d_na,
                  c->d_nb, c->d_nd, c->d_na32, c->d_nb32, c->d_nd32, c->d_diag, c->d_khat,
                  c->d_tth, c->d_tph, c->d_trf, c->d_rt, c->d_rt32, c->d_trf32, c->d_xi32, c->d_yi32, c->d_xi, c->d_yi, c->d_gm, c->d_gm32, c->d_gmz, c->d_lu, c->d_piv, c->d_io,
                  c->d_xb32, c->d_yb32, c->d_gmb, c->d_qperm, c->d_boxc, c->d_side, c->d_vert,
                  c->d_grad_ws, c->d_tri_verts, c->d_naT, c->d_nbT, c->d_ndT, c->d_lu32, c->d_lu32i, c->d_piv32,
                  c->d_perm32, c->d_tmp32, c->d_lu_at, c->d_lu_bt, c->d_lu_scr,
                  c->d_lu_diag, c->d_lu_minv, c->d_lu_at2, c->d_lu_ref, c->d_lu_io};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->d_lvtmp) cudaFree(c->d_lvtmp);
  for (auto& L : c->lv) {
    void* lp[] = {L.C, L.D, L.tl, L.ph_up, L.ph_dn, L.tl32, L.ph_up32, L.ph_dn32, L.i4_ptr, L.i4_src, L.i4_off,
                  L.ch_ptr, L.ch_idx, L.ch_oct, L.parent, L.oct, L.grp_sib, L.grp_src, L.Cb, L.Db,
                  L.khat, L.trf, L.trf32, L.up.ptr, L.up.col, L.up.val, L.up.val32, L.dn.ptr, L.dn.col,
                  L.dn.val, L.dn.val32, L.up.ecol, L.up.eval, L.up.eval32, L.dn.ecol, L.dn.eval,
                  L.dn.eval32, L.up.optr, L.up.ocol, L.up.oval, L.up.oval32, L.dn.optr, L.dn.ocol,
                  L.dn.oval, L.dn.oval32};
    for (void* p : lp)
      if (p) cudaFree(p);
  }
  if (c->h_gm) cudaFreeHost(c->h_gm);
  if (c->h_gmb) cudaFreeHost(c->h_gmb);
  for (int i = 0; i < 16; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  else if (c->stream) cudaStreamDestroy(c->stream);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  delete c;
  return SIE_OK;
}

}  // extern "C"
