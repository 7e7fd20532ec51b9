"""CPU oracle of the SpeckleSim SIE hot path -- TEST INFRASTRUCTURE ONLY.

Python side of oracle/sie_oracle.cpp (a plain FP64 C++ restatement of the
reference Fortran) plus a numpy restatement of the CERFACS zgmres driver.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module, and only as the checker / the timed CPU baseline.  The product library
(specklesim_b200) never imports it.

Parity pins: Hankel h2 and GMRES against the reference's own known-answer tests
(tests/golden); the SIE blocks/matvec have no golden vectors in the reference
(its SIE fixtures are missing), see tests/test_oracle_*.py for the probes used
instead.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sie_oracle.cpp")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libsieoracle.so")


def build(force=False):
    """g++ -O2 -fopenmp -shared (the oracle is plain C++, no CUDA)."""
    os.makedirs(BUILD, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + ".tmp"
    cmd = ["g++", "-O2", "-fopenmp", "-shared", "-fPIC", "-std=c++17", "-o", tmp, SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        dp, ip, lp, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.c_void_p
        sig = {
            "orc_create": (vp, [dp, C.c_int, ip, C.c_int, C.c_double, C.c_double, C.c_double,
                                C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_free": (None, [vp]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_num_edges": (C.c_int, [vp]),
            "orc_edges": (None, [vp, ip, ip]),
            "orc_material": (None, [vp, dp]),
            "orc_blocks": (None, [vp, ip, ip, C.c_int, dp]),
            "orc_dense": (None, [vp, dp]),
            "orc_tree": (C.c_int, [vp]),
            "orc_tree_info": (None, [vp, ip, dp, lp]),
            "orc_num_boxes": (C.c_int, [vp, C.c_int]),
            "orc_boxes": (None, [vp, C.c_int, lp]),
            "orc_i4": (C.c_int, [vp, C.c_longlong, C.c_int, lp]),
            "orc_neighbours": (C.c_int, [C.c_longlong, C.c_int, lp]),
            "orc_universal_index": (C.c_longlong, [dp, C.c_int]),
            "orc_quad_rule": (C.c_int, [C.c_int, dp, dp, dp]),
            "orc_setup_fmm": (C.c_longlong, [vp]),
            "orc_set_level_k": (None, [vp, ip, C.c_int]),
            "orc_level_Q": (C.c_int, [vp, C.c_int]),
            "orc_near_csr": (None, [vp, ip, ip, dp]),
            "orc_Q": (C.c_int, [vp]),
            "orc_sampling": (None, [vp, dp, dp, dp, dp]),
            "orc_rt": (None, [vp, dp]),
            "orc_tl": (None, [vp, C.c_int, dp]),
            "orc_matvec": (None, [vp, dp, dp, C.c_int]),
            "orc_rhs": (None, [vp, dp, dp, dp]),
            "orc_field": (None, [vp, dp, dp, C.c_int, dp, dp]),
            "orc_set_xnt_binary32": (None, [C.c_int]),
            "orc_field_interior": (None, [vp, dp, dp, C.c_int, C.c_double, C.c_double, dp, dp]),
            "orc_field_medium": (None, [vp, dp, dp, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, dp, dp]),
            "orc_hankel2": (None, [C.c_double, C.c_double, C.c_int, dp]),
            "orc_gauss_legendre": (None, [C.c_int, dp, dp]),
            "orc_lagrange_interp": (None, [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp]),
            "orc_hanninen": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp]),
            "orc_fn": (None, [vp, C.c_int, C.c_int, dp]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _l(a):
    return a.ctypes.data_as(C.POINTER(C.c_longlong))


FORM = {"PMCHWT": 1, "ICTF": 3}


class Oracle:
    def __init__(self, verts, tris, wavelength, eps_r2, formulation="ICTF", ngp=3, tree_s_opt=250,
                 truncation_number=19, normal_convention=2, fix_itbn=False, threads=0):
        L = lib()
        if threads:
            L.orc_set_threads(int(threads))
        self.v = np.ascontiguousarray(verts, np.float64)
        self.t = np.ascontiguousarray(tris, np.int32)
        e = complex(eps_r2)
        self.h = L.orc_create(_d(self.v), self.v.shape[0], _i(self.t), self.t.shape[0], float(wavelength),
                              e.real, e.imag, FORM[formulation], int(ngp), int(tree_s_opt),
                              int(truncation_number), int(normal_convention), int(bool(fix_itbn)))
        self.M = L.orc_num_edges(self.h)
        self.N = 2 * self.M
        self.nnz = None

    def close(self):
        if self.h:
            lib().orc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def edges(self):
        e = np.zeros(2 * self.M, np.int32)
        c = np.zeros(2 * self.M, np.int32)
        lib().orc_edges(self.h, _i(e), _i(c))
        return e.reshape(-1, 2), c.reshape(-1, 2)

    def material(self):
        o = np.zeros(18)
        lib().orc_material(self.h, _d(o))
        v = o[0::2] + 1j * o[1::2]
        return dict(zip(["k0", "omega", "k1", "k2", "eps1", "eps2", "eta1", "eta2", "eta_a"], v))

    def blocks(self, m, n):
        m = np.ascontiguousarray(m, np.int32)
        n = np.ascontiguousarray(n, np.int32)
        out = np.zeros((len(m), 4), np.complex128)
        lib().orc_blocks(self.h, _i(m), _i(n), len(m), _d(out.view(np.float64)))
        return out

    def dense(self):
        Z = np.zeros((self.N, self.N), np.complex128)
        lib().orc_dense(self.h, _d(Z.view(np.float64)))
        return Z

    def tree(self):
        lmax = lib().orc_tree(self.h)
        ll = np.zeros(2, np.int32)
        d = np.zeros(4)
        leaf = np.zeros(self.M, np.int64)
        lib().orc_tree_info(self.h, _i(ll), _d(d), _l(leaf))
        return dict(l_min=int(ll[0]), l_max=int(ll[1]), D=d[0], xmin=d[1:], leaf=leaf)

    def boxes(self, level):
        n = lib().orc_num_boxes(self.h, level)
        out = np.zeros(n, np.int64)
        if n:
            lib().orc_boxes(self.h, level, _l(out))
        return out

    def i4(self, n, level):
        out = np.zeros(1000, np.int64)
        k = lib().orc_i4(self.h, int(n), int(level), _l(out))
        return out[:k]

    def set_level_truncation(self, k_by_level):
        """Truncation number per tree level ({level: K}; levels left out keep the
        context's K), the reference's truncation_number(l)%n.  Call before setup_fmm.
        A level whose K differs from its parent's takes the interpolation branches of SS
        and RR (lib_sie_tri_mlfmm_interface.f90:486-507, :622-640)."""
        n = max(k_by_level) + 1
        arr = np.zeros(n, np.int32)
        for l, k in k_by_level.items():
            arr[l] = int(k)
        lib().orc_set_level_k(self.h, _i(arr), n)

    def setup_fmm(self):
        self.nnz = lib().orc_setup_fmm(self.h)
        if self.nnz < 0:
            raise ValueError("truncation numbers must not grow from a level to its children")
        self.Q = lib().orc_Q(self.h)
        return self.nnz

    def near_csr(self):
        ia = np.zeros(self.M + 1, np.int32)
        ja = np.zeros(self.nnz, np.int32)
        v = np.zeros((self.nnz, 4), np.complex128)
        lib().orc_near_csr(self.h, _i(ia), _i(ja), _d(v.view(np.float64)))
        return ia, ja, v

    def sampling(self):
        Q = self.Q
        kh, th, ph, w = np.zeros((Q, 3)), np.zeros((Q, 3)), np.zeros((Q, 3)), np.zeros(Q)
        lib().orc_sampling(self.h, _d(kh), _d(th), _d(ph), _d(w))
        return kh, th, ph, w

    def rt(self):
        out = np.zeros((self.M, 4, self.Q), np.complex128)
        lib().orc_rt(self.h, _d(out.view(np.float64)))
        return out

    def tl(self, level):
        out = np.zeros((343, 2, lib().orc_level_Q(self.h, int(level))), np.complex128)
        lib().orc_tl(self.h, int(level), _d(out.view(np.float64)))
        return out

    def matvec(self, x, faithful_lookup=False):
        x = np.ascontiguousarray(x, np.complex128)
        y = np.zeros_like(x)
        lib().orc_matvec(self.h, _d(x.view(np.float64)), _d(y.view(np.float64)), int(faithful_lookup))
        return y

    def rhs(self, k_in, E_in):
        k = np.ascontiguousarray(k_in, np.float64)
        e = np.ascontiguousarray(E_in, np.float64)
        b = np.zeros(self.N, np.complex128)
        lib().orc_rhs(self.h, _d(k), _d(e), _d(b.view(np.float64)))
        return b

    def field(self, x, pts):
        x = np.ascontiguousarray(x, np.complex128)
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        E = np.zeros((p.shape[0], 3), np.complex128)
        H = np.zeros((p.shape[0], 3), np.complex128)
        lib().orc_field(self.h, _d(x.view(np.float64)), _d(p), p.shape[0], _d(E.view(np.float64)),
                        _d(H.view(np.float64)))
        I = np.sum(np.abs(E) ** 2, axis=1) * 4 * np.pi * np.sum(p * p, axis=1)
        return E, H, I

    def field_interior(self, x, pts, eps_r):
        """E, H at points inside the body (Integration_scattered_field_tri_within_medium,
        src/lib_sie_tri_calculation_mod.f90:2829-2877) in the medium of relative
        permittivity eps_r."""
        x = np.ascontiguousarray(x, np.complex128)
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        E = np.zeros((p.shape[0], 3), np.complex128)
        H = np.zeros((p.shape[0], 3), np.complex128)
        er = complex(eps_r)
        lib().orc_field_interior(self.h, _d(x.view(np.float64)), _d(p), p.shape[0], er.real, er.imag,
                                 _d(E.view(np.float64)), _d(H.view(np.float64)))
        return E, H

    def field_medium(self, x, pts, k, my, eps):
        """The exterior routine (Integration_scattered_field_tri) with the medium's
        wavenumber k, permeability my and permittivity eps replaced."""
        x = np.ascontiguousarray(x, np.complex128)
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        E = np.zeros((p.shape[0], 3), np.complex128)
        H = np.zeros((p.shape[0], 3), np.complex128)
        k, eps = complex(k), complex(eps)
        lib().orc_field_medium(self.h, _d(x.view(np.float64)), _d(p), p.shape[0], k.real, k.imag, float(my),
                               eps.real, eps.imag, _d(E.view(np.float64)), _d(H.view(np.float64)))
        return E, H

    def hanninen(self, m, tt, n, ll, ia, q):
        out = np.zeros(13)
        lib().orc_hanninen(self.h, m, tt, n, ll, ia, q, _d(out))
        return dict(K2=out[0:3], K3=out[3:6], K4=out[6:9], Is=out[9], Ra=out[10:13])

    def fn(self, e, ot):
        out = np.zeros(18)
        lib().orc_fn(self.h, e, ot, _d(out))
        return dict(c=out[0:9].reshape(3, 3), area=out[9], length=out[10], df=out[11],
                    mid=out[12:15], nq=out[15:18])


def set_xnt_binary32(on):
    """Round the x_nt term of the singular outer integrals to binary32 as the reference
    does (True, the default) or keep it in FP64 (False), for every later fill."""
    lib().orc_set_xnt_binary32(1 if on else 0)


def quad_rule(ngp):
    """Barycentric points (alpha, beta) and weights of the ngp-point triangle rule, as the
    oracle uses them: Quadrature_tri."""
    a, b, w = np.zeros(12), np.zeros(12), np.zeros(12)
    n = lib().orc_quad_rule(int(ngp), _d(a), _d(b), _d(w))
    return a[:n], b[:n], w[:n]


def universal_index(point, level):
    """Box index (Morton, x the most significant bit) at `level` of a point in the unit
    cube: lib_tree_hf_get_universal_index."""
    p = np.ascontiguousarray(point, np.float64)
    return int(lib().orc_universal_index(_d(p), int(level)))


def neighbours(n, level):
    """The up-to-26 level-`level` boxes around box n, x outer, y middle, z inner, n
    itself left out: lib_tree_hf_get_neighbour_all_xD with k = 1."""
    out = np.zeros(26, np.int64)
    k = lib().orc_neighbours(int(n), int(level), _l(out))
    return out[:k]


def hankel2(z, n):
    out = np.zeros(2 * n)
    lib().orc_hankel2(float(np.real(z)), float(np.imag(z)), int(n), _d(out))
    return out[0::2] + 1j * out[1::2]


def gauss_legendre(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss_legendre(int(n), _d(x), _d(w))
    return x, w


def lagrange_interp(p, k_from, k_to, fa, fb):
    """Local Lagrange interpolation of one (theta, phi) far-field pattern pair from the
    K = k_from sampling to K = k_to (Lagrange_Interpolation_New, lib_sie_mlfmm.f90:268-390;
    stencil of 2p x 2p points, p = 3 in the reference).  fa, fb: 2 k_from^2 + 2 complex
    values in the sampling order of `Oracle.sampling`, the last two being the +z and -z
    poles, which hold the Cartesian x and y components.  Returns (ga, gb)."""
    qf, qt = 2 * k_from * k_from + 2, 2 * k_to * k_to + 2
    a = np.ascontiguousarray(np.asarray(fa, dtype=np.complex128).reshape(qf)).view(np.float64)
    b = np.ascontiguousarray(np.asarray(fb, dtype=np.complex128).reshape(qf)).view(np.float64)
    ga, gb = np.zeros(2 * qt), np.zeros(2 * qt)
    lib().orc_lagrange_interp(int(p), int(k_from), int(k_to), _d(a), _d(b), _d(ga), _d(gb))
    return ga.view(np.complex128), gb.view(np.complex128)


# ---------------------------------------------------------------------------
# zgmres restated (src/lib/libmath_external/src/algorithm_842/zPackgmres.f90:537-1565):
# no preconditioning, IMGS (icntl(5)=1), recurrence at restart (icntl(8)=0),
# Arnoldi backward error |H(jH+1,m+1)|/||b|| confirmed by the true residual.

def _zrotg(ca, cb):
    aca = abs(ca)
    if aca == 0.0:
        return 0.0, 1.0 + 0j
    acb = abs(cb)
    scale = aca + acb
    norm = scale * np.sqrt((aca / scale) ** 2 + (acb / scale) ** 2)
    alpha = ca / aca
    return aca / norm, alpha * np.conj(cb) / norm


def _zrot(x, y, c, s):
    return c * x + s * y, c * y - np.conj(s) * x


def zgmres(matvec, b, m, tol, itermax, x0=None, history=None):
    """Returns x, info dict(iterations, bea, be, converged, matvecs)."""
    n = b.shape[0]
    nmv = 0
    x = np.zeros(n, np.complex128) if x0 is None else np.array(x0, np.complex128)
    bn = np.sqrt(np.real(np.vdot(b, b)))
    if bn == 0:
        return np.zeros(n, np.complex128), dict(iterations=0, bea=0.0, be=0.0, converged=True, matvecs=0)
    if x0 is not None:
        r0 = b - matvec(x)
        nmv += 1
    else:
        r0 = b.copy()
    w = r0
    beta = np.sqrt(np.real(np.vdot(w, w)))
    if beta == 0:
        return x, dict(iterations=0, bea=0.0, be=0.0, converged=True, matvecs=nmv)
    V = np.zeros((n, m + 1), np.complex128)
    H = np.zeros((m + 1, m + 1), np.complex128)
    rc = np.zeros(m + 1)
    rs = np.zeros(m + 1, np.complex128)
    V[:, 0] = w / beta
    iterOut = 0
    compRsd = 0
    bea = be = np.inf
    xc = None
    while True:
        H[:, m] = 0
        H[0, m] = beta
        jH = 0
        while jH < m:
            w = matvec(V[:, jH])
            nmv += 1
            H[: jH + 1, jH] = 0
            northo = 0
            while True:
                northo += 1
                dloo = 0.0
                for j in range(jH + 1):
                    dvi = np.vdot(V[:, j], w)
                    H[j, jH] += dvi
                    dloo += abs(dvi) ** 2
                    w = w - dvi * V[:, j]
                dnormw = np.sqrt(np.real(np.vdot(w, w)))
                dloo = np.sqrt(dloo)
                if not (dnormw <= dloo and northo < 3):
                    break
            H[jH + 1, jH] = dnormw
            V[:, jH + 1] = w / dnormw
            for j in range(jH):
                H[j, jH], H[j + 1, jH] = _zrot(H[j, jH], H[j + 1, jH], rc[j], rs[j])
            c, s = _zrotg(H[jH, jH], H[jH + 1, jH])
            rc[jH], rs[jH] = c, s
            H[jH, m], H[jH + 1, m] = _zrot(H[jH, m], H[jH + 1, m], c, s)
            H[jH, jH], H[jH + 1, jH] = _zrot(H[jH, jH], H[jH + 1, jH], c, s)
            H[jH + 1, jH] = 0
            bea = abs(H[jH + 1, m]) / bn
            it = iterOut * m + jH + 1
            if history is not None:
                history.append(bea)
            if bea <= tol or it >= itermax:
                compRsd = 1
                y = np.linalg.solve(np.triu(H[: jH + 1, : jH + 1]), H[: jH + 1, m])
                xc = x + V[:, : jH + 1] @ y
                wt = b - matvec(xc)
                nmv += 1
                be = np.sqrt(np.real(np.vdot(wt, wt))) / bn
                if be <= tol or it >= itermax:
                    return xc, dict(iterations=it, bea=bea, be=be, converged=bool(be <= tol), matvecs=nmv)
            jH += 1
        iterOut += 1
        if bea > tol:
            y = np.linalg.solve(np.triu(H[:m, :m]), H[:m, m])
            xc = x + V[:, :m] @ y
        x = xc
        if compRsd:
            w = b - matvec(x)
            nmv += 1
            beta = np.sqrt(np.real(np.vdot(w, w)))
        else:
            beta = abs(H[m, m])
            for j in range(m - 1, -1, -1):
                H[j, m] = 0
                H[j, m], H[j + 1, m] = _zrot(H[j, m], H[j + 1, m], rc[j], -rs[j])
            w = V @ H[:, m]
        V[:, 0] = w / beta
