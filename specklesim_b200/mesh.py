"""Synthetic triangle meshes and the reference's pp_/tt_ mesh files.

Orientation convention: the vertex order of every triangle gives a right-hand
normal pointing INTO the body, as the reference's own sphere generator does
(recursive_triangulation, src/lib_sie_tri_calculation_mod.f90:646-701: element
(1,5,3) of the octahedron has the inward normal (-1,-1,-1)).  The RWG normal
fn%nq (norm_vec_r_new, :1017-1033) is then the outward normal.
"""
import numpy as np


def _orient_inward(verts, tris, outward):
    """Flip triangles whose right-hand normal points along `outward` (per-triangle vectors)."""
    a, b, c = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    n = np.cross(b - a, c - a)
    flip = np.einsum("ij,ij->i", n, outward) > 0
    t = tris.copy()
    t[flip, 1], t[flip, 2] = tris[flip, 2], tris[flip, 1]
    return t


def icosphere(subdivisions=3, radius=1.0):
    """Icosphere with 20 * 4**subdivisions triangles (subdivision 3: 1280 triangles, 1920 edges)."""
    p = (1 + 5 ** 0.5) / 2
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p),
         (0, 1, -p), (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(x, float) / np.linalg.norm(x) for x in v]
    faces = list(f)
    for _ in range(subdivisions):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius
    T = np.array(faces, dtype=np.int32)
    cen = V[T].mean(axis=1)
    return V, _orient_inward(V, T, cen)


def gaussian_rough_surface(n, length, rms, corr_len, seed):
    """Heights on an (n+1) x (n+1) vertex grid over a `length` x `length` patch.

    White noise N(0,1) from numpy.random.default_rng(seed), filtered (periodic FFT
    convolution) by exp(-2 r^2 / corr_len^2) so the surface has the Gaussian
    correlation exp(-r^2 / corr_len^2), then scaled to zero mean and RMS `rms`.
    """
    rng = np.random.default_rng(seed)
    m = n + 1
    w = rng.standard_normal((m, m))
    d = length / n
    k = np.fft.fftfreq(m, d=1.0) * m
    k = np.minimum(np.abs(k), m - np.abs(k)) * d
    r2 = k[:, None] ** 2 + k[None, :] ** 2
    g = np.exp(-2.0 * r2 / corr_len ** 2)
    h = np.real(np.fft.ifft2(np.fft.fft2(w) * np.fft.fft2(g)))
    h -= h.mean()
    s = h.std()
    if s > 0:
        h *= rms / s
    return h


def rough_slab(n, length, thickness, rms, corr_len, seed, nz=None, heights=None):
    """Closed slab: rough top z = h(x, y) on an n x n grid over [-L/2, L/2]^2,
    flat bottom and vertical side walls (nz layers).

    The bottom lies at z = -thickness, or lower if the rough top dips within a
    quarter of the thickness of it (so the body never self-intersects).
    Returns (verts (nv,3), tris (nt,3) int32, 0-based, inward right-hand normals).
    """
    h = gaussian_rough_surface(n, length, rms, corr_len, seed) if heights is None else heights
    m = n + 1
    xs = np.linspace(-length / 2, length / 2, m)
    zb = min(-thickness, h.min() - 0.25 * thickness)
    if nz is None:
        nz = max(1, int(round(thickness / (length / n))))
    verts = []
    top = np.zeros((m, m), dtype=np.int64)
    bot = np.zeros((m, m), dtype=np.int64)
    for i in range(m):
        for j in range(m):
            top[i, j] = len(verts)
            verts.append((xs[i], xs[j], h[i, j]))
    for i in range(m):
        for j in range(m):
            bot[i, j] = len(verts)
            verts.append((xs[i], xs[j], zb))
    # boundary loop of the grid (counter-clockwise seen from above)
    loop = [(i, 0) for i in range(m - 1)] + [(m - 1, j) for j in range(m - 1)] + \
           [(i, m - 1) for i in range(m - 1, 0, -1)] + [(0, j) for j in range(m - 1, 0, -1)]
    nl = len(loop)
    side = np.zeros((nl, nz + 1), dtype=np.int64)
    for a, (i, j) in enumerate(loop):
        side[a, 0] = top[i, j]
        side[a, nz] = bot[i, j]
        for k in range(1, nz):
            side[a, k] = len(verts)
            z = h[i, j] + (zb - h[i, j]) * k / nz
            verts.append((xs[i], xs[j], z))
    V = np.array(verts, dtype=float)
    tris, outw = [], []
    for i in range(n):
        for j in range(n):
            a, b, c, d = top[i, j], top[i + 1, j], top[i + 1, j + 1], top[i, j + 1]
            tris += [(a, b, c), (a, c, d)]
            outw += [(0, 0, 1)] * 2
            a, b, c, d = bot[i, j], bot[i + 1, j], bot[i + 1, j + 1], bot[i, j + 1]
            tris += [(a, b, c), (a, c, d)]
            outw += [(0, 0, -1)] * 2
    for a in range(nl):
        b = (a + 1) % nl
        (i0, j0), (i1, j1) = loop[a], loop[b]
        # outward direction of this wall segment
        if j0 == 0 and j1 == 0:
            o = (0, -1, 0)
        elif i0 == m - 1 and i1 == m - 1:
            o = (1, 0, 0)
        elif j0 == m - 1 and j1 == m - 1:
            o = (0, 1, 0)
        else:
            o = (-1, 0, 0)
        for k in range(nz):
            p, q, r, s = side[a, k], side[b, k], side[b, k + 1], side[a, k + 1]
            tris += [(p, q, r), (p, r, s)]
            outw += [o] * 2
    T = np.array(tris, dtype=np.int32)
    return V, _orient_inward(V, T, np.array(outw, float))


def slab_config(length_wl, wavelength, rms_wl, corr_wl, seed, cells=None, thickness_wl=1.0):
    """Rough slab of the benchmark recipes in metres (grid of ~wavelength/6.4 cells by default)."""
    if cells is None:
        cells = int(round(length_wl * 6.4))
    return rough_slab(cells, length_wl * wavelength, thickness_wl * wavelength,
                      rms_wl * wavelength, corr_wl * wavelength, seed,
                      nz=max(1, int(round(thickness_wl * cells / length_wl))))


def read_pp_tt(pp_file, tt_file):
    """read_pp_tt_file_tri (src/lib_sie_tri_data_container.f90:226-261): whitespace
    separated coordinates (3 per node) and 1-based node indices (3 per element)."""
    pp = np.loadtxt(pp_file, dtype=float).reshape(-1, 3)
    tt = np.loadtxt(tt_file, dtype=np.int64).reshape(-1, 3) - 1
    return pp, tt.astype(np.int32)


def write_pp_tt(pp_file, tt_file, verts, tris):
    np.savetxt(pp_file, np.asarray(verts, float), fmt="%.17e")
    np.savetxt(tt_file, np.asarray(tris, np.int64) + 1, fmt="%d")


def edge_count(tris):
    """Interior edges (RWG unknowns per current) of a closed triangle surface."""
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    return int((cnt >= 2).sum())


def winding_number(verts, tris, pts, chunk=2048):
    """Generalised winding number of the closed triangle surface at each point: the sum of
    the signed solid angles of its triangles (Van Oosterom and Strackee, IEEE Trans.
    Biomed. Eng. 30 (1983) 125) over 4 pi.  +-1 inside (the sign follows the triangles'
    orientation), 0 outside."""
    V = np.asarray(verts, dtype=np.float64)
    T = np.asarray(tris)
    P = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    A, B, C = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    out = np.empty(len(P))
    for s in range(0, len(P), chunk):
        p = P[s:s + chunk, None, :]
        a, b, c = A[None] - p, B[None] - p, C[None] - p
        la, lb, lc = (np.linalg.norm(v, axis=2) for v in (a, b, c))
        num = np.einsum("ijk,ijk->ij", a, np.cross(b, c))
        den = (la * lb * lc + np.einsum("ijk,ijk->ij", a, b) * lc + np.einsum("ijk,ijk->ij", a, c) * lb
               + np.einsum("ijk,ijk->ij", b, c) * la)
        out[s:s + chunk] = 2 * np.arctan2(num, den).sum(axis=1) / (4 * np.pi)
    return out


def inside(verts, tris, pts):
    """True for points inside the closed triangle surface (|winding number| > 1/2): the
    medium-2 points of a near-field map.  The reference classifies map points by its
    analytic shapes (sphere radius, grating profile, rough-surface boundary file;
    get_evaluation_points_domain_new, src/lib_sie_math.f90:360-530); this uses the
    meshed surface itself."""
    return np.abs(winding_number(verts, tris, pts)) > 0.5
