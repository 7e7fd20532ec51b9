// RWG half-basis geometry rebuilt on the device from the vertex coordinates, with one
// vertex moved along z.  The gradient kernels differentiate the near blocks, radiation
// patterns, right-hand side and far field of an edge by central differences of these
// rebuilt sides; the formulas are those of the host tables (fn_parameter_type,
// src/lib_sie_tri_calculation_mod.f90:1539-1586).
#pragma once
#include "sie_internal.h"

namespace sie {

// Vertex indices of one half basis: p1, p2 (the edge, in the triangle's cyclic order), pc
// (the free vertex), and the triangle's own vertex order for its centroid.
struct SideV {
  int p1, p2, pc, tri;
  int t0, t1, t2, pad;
};

__device__ __forceinline__ vd vert_z(const double* V, int i, int pv, double dz) {
  return mkv<double>(V[3 * i], V[3 * i + 1], V[3 * i + 2] + (i == pv ? dz : 0.0));
}

// FnD of side s with vertex pv shifted by dz along z (pv < 0: unshifted).
__device__ __forceinline__ FnD side_fn(const SideV& s, double sgn, const double* V, int normal_convention,
                                       int pv, double dz) {
  FnD f;
  const vd p1 = vert_z(V, s.p1, pv, dz), p2 = vert_z(V, s.p2, pv, dz), pc = vert_z(V, s.pc, pv, dz);
  f.c[0] = p1.x; f.c[1] = p1.y; f.c[2] = p1.z;
  f.c[3] = p2.x; f.c[4] = p2.y; f.c[5] = p2.z;
  f.c[6] = pc.x; f.c[7] = pc.y; f.c[8] = pc.z;
  f.length = vlen(p1 - p2);
  f.area = 0.5 * vlen(cross(p1 - pc, p2 - pc));
  f.sgn = sgn;
  f.df = sgn * f.length / f.area;
  const vd a = vert_z(V, s.t0, pv, dz), b = vert_z(V, s.t1, pv, dz), e = vert_z(V, s.t2, pv, dz);
  f.mid[0] = (a.x + b.x + e.x) / 3.0;
  f.mid[1] = (a.y + b.y + e.y) / 3.0;
  f.mid[2] = (a.z + b.z + e.z) / 3.0;
  vd u, w;
  if (normal_convention == 1) {
    u = p1 - p2;
    w = pc - p2;
  } else {
    u = pc - p1;
    w = p2 - p1;
  }
  const vd n = cross(u, w);
  const double ln = vlen(n);
  f.nq[0] = n.x / ln;
  f.nq[1] = n.y / ln;
  f.nq[2] = n.z / ln;
  f.tri = s.tri;
  f.pad = 0;
  return f;
}

// The four vertices an edge's basis depends on: the two edge corners and the two free
// vertices, slot 0..3.
__device__ __forceinline__ int edge_vertex(const SideV* sv, int e, int slot) {
  const SideV& s0 = sv[2 * e];
  return slot == 0 ? s0.p1 : slot == 1 ? s0.p2 : slot == 2 ? s0.pc : sv[2 * e + 1].pc;
}

}  // namespace sie
