"""Host logic of the differentiation check at size (tests/c5_check.py), on CPU: the edge-to-
triangle table of a closed mesh and the count of (edge, side, triangle) triples whose
singular/regular quadrature choice (centroid distance against 1.5 times the edge's centroid
distance) changes between two vertex sets."""
import numpy as np

from tests import problems as P
from tests.c5_check import _edge_triangles, singular_flips


def _brute_flips(Vm, Vp, T, et):
    cm, cp = Vm[T].mean(axis=1), Vp[T].mean(axis=1)
    n = 0
    for e in range(len(et)):
        rm = np.linalg.norm(cm[et[e, 0]] - cm[et[e, 1]])
        rp = np.linalg.norm(cp[et[e, 0]] - cp[et[e, 1]])
        for p in et[e]:
            a = np.linalg.norm(cm - cm[p], axis=1) <= 1.5 * rm
            b = np.linalg.norm(cp - cp[p], axis=1) <= 1.5 * rp
            n += int(np.count_nonzero(a != b))
    return n


def test_edge_triangles_of_a_closed_mesh():
    V, T = P.sphere(1)
    et = _edge_triangles(np.asarray(T))
    assert et.shape == (3 * len(T) // 2, 2)
    # each edge's two triangles share exactly its two vertices
    for a, b in et:
        assert len(set(T[a]) & set(T[b])) == 2


def test_singular_flips_match_a_brute_force_count():
    V, T = P.slab(cells=6, length_wl=1.5, seed=2, rms_wl=0.2, corr_wl=0.5, thickness_wl=0.5)
    T = np.asarray(T)
    et = _edge_triangles(T)
    assert singular_flips(V, V.copy(), T, et) == 0
    rng = np.random.default_rng(0)
    for step in (1e-3, 2e-2, 1e-1):
        Vp = V.copy()
        v = rng.integers(0, 49)  # a vertex of the rough top face
        Vp[v, 2] += step * P.WL
        assert singular_flips(V, Vp, T, et) == _brute_flips(V, Vp, T, et)


def _brute_crossings(Vm, Vp, T, et):
    from tests.c5_check import _RULE3
    n = 0
    singular = []
    for V in (Vm, Vp):
        c = V[T].mean(axis=1)
        rm = np.zeros(len(T))
        for a, b in et:
            r = np.linalg.norm(c[a] - c[b])
            rm[a], rm[b] = max(rm[a], r), max(rm[b], r)
        singular.append(np.linalg.norm(c[:, None, :] - c[None, :, :], axis=2) <= 1.5 * rm[:, None])
    S = singular[0] | singular[1]
    for p, q in zip(*np.nonzero(S)):
        if p == q:
            continue
        for V_a, V_b in ((Vm, Vp),):
            hs = []
            for V in (V_a, V_b):
                P, Q = V[T[p]], V[T[q]]
                nq = np.cross(Q[1] - Q[0], Q[2] - Q[0])
                hs.append((_RULE3 @ P - Q[0]) @ nq)
            n += int(np.count_nonzero(np.sign(hs[0]) != np.sign(hs[1])))
    return n


def test_plane_crossings_match_a_brute_force_count():
    """Outer quadrature points of singular pairs that cross the source triangle's plane
    between two vertex sets (the kink of the unsigned solid angle), against a count over
    every pair of the mesh."""
    from tests.c5_check import plane_crossings
    V, T = P.slab(cells=6, length_wl=1.5, seed=2, rms_wl=0.2, corr_wl=0.5, thickness_wl=0.5)
    T = np.asarray(T)
    et = _edge_triangles(T)
    assert plane_crossings(V, V.copy(), T, et) == 0
    rng = np.random.default_rng(1)
    seen = 0
    for step in (1e-3, 3e-2, 1e-1, 3e-1):
        Vp = V.copy()
        v = rng.integers(0, 49)  # a vertex of the rough top face
        Vp[v, 2] += step * P.WL
        n = plane_crossings(V, Vp, T, et)
        assert n == _brute_crossings(V, Vp, T, et)
        seen += n
    assert seen > 0  # the larger steps carry points across planes
