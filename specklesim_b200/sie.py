"""Python host side of the B200 SIE path: a thin object over the C-ABI.

`Sie` owns one GPU context (one mesh, one material, one MLFMM set-up).  All
compute goes through libsiegpu.so; nothing here evaluates the operator on the
CPU.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import SieConfig, SieError, SieSolverCfg, SieStats, check, dptr, iptr, lptr

FORMULATIONS = {"PMCHWT": _lib.SIE_PMCHWT, "ICTF": _lib.SIE_ICTF}
PRECISIONS = {"fp64": _lib.SIE_FP64, "mixed": _lib.SIE_MIXED}


def incidence(theta, phi, pol="TM", k_dir=2):
    """k_in and E_in of kin_and_Ein_calculation (src/lib_sie_math.f90:259-293)."""
    lib = _lib.load()
    k = np.zeros(3)
    e = np.zeros(3)
    check(lib.sie_incidence(float(theta), float(phi), 1 if pol == "TM" else 2, int(k_dir), dptr(k), dptr(e)))
    return k, e


def quadrature_rule(ngp):
    """(alpha, beta, w) of the ngp-point triangle rule that the fill kernels use
    (Quadrature_tri, src/lib_sie_integration_points.f90:7-143).  Needs no GPU."""
    lib = _lib.load()
    a, b, w = np.zeros(12), np.zeros(12), np.zeros(12)
    n = C.c_int()
    check(lib.sie_quadrature_rule(int(ngp), dptr(a), dptr(b), dptr(w), C.byref(n)))
    return a[:n.value], b[:n.value], w[:n.value]


class Sie:
    def __init__(self, verts, tris, wavelength, eps_r2, eps_r1=1.0, formulation="ICTF", ngp=3,
                 tree_s_opt=250, truncation_number=19, normal_convention=2, fix_itbn=False,
                 device=0, dense=False, level_truncation=None):
        lib = _lib.load()
        cfg = SieConfig()
        lib.sie_config_default(C.byref(cfg))
        cfg.lambda_ = float(wavelength)
        e1, e2 = complex(eps_r1), complex(eps_r2)
        cfg.eps_r1_re, cfg.eps_r1_im = e1.real, e1.imag
        cfg.eps_r2_re, cfg.eps_r2_im = e2.real, e2.imag
        cfg.formulation = FORMULATIONS[formulation] if isinstance(formulation, str) else int(formulation)
        cfg.ngp = int(ngp)
        cfg.tree_s_opt = int(tree_s_opt)
        cfg.truncation_number = int(truncation_number)
        cfg.normal_convention = int(normal_convention)
        cfg.fix_itbn = int(bool(fix_itbn))
        cfg.device = int(device)
        cfg.dense = int(bool(dense))
        self.cfg = cfg
        v = np.ascontiguousarray(verts, dtype=np.float64)
        t = np.ascontiguousarray(tris, dtype=np.int32)
        self.verts, self.tris = v, t
        self._h = C.c_void_p()
        check(lib.sie_init(C.byref(cfg), dptr(v), v.shape[0], iptr(t), t.shape[0], C.byref(self._h)))
        self._lib = lib
        m, l0, l1, nnz = C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
        check(lib.sie_info(self._h, C.byref(m), C.byref(l0), C.byref(l1), C.byref(nnz)))
        self.n_edges = m.value
        self.nv = v.shape[0]
        self.l_min, self.l_max = l0.value, l1.value
        self.near_nnz = nnz.value
        self._setup = False
        if level_truncation:
            # {level: K}: truncation number per MLFMM level (others keep truncation_number)
            kl = np.zeros(max(level_truncation) + 1, np.int32)
            for l, k in level_truncation.items():
                kl[l] = int(k)
            check(lib.sie_set_level_truncation(self._h, iptr(kl), len(kl)))

    # --- set-up -----------------------------------------------------------
    def setup(self):
        if not self._setup:
            check(self._lib.sie_setup(self._h))
            self._setup = True
        return self

    @property
    def n(self):
        return 2 * self.n_edges

    # --- operator -----------------------------------------------------------
    def matvec(self, x, precision="fp64"):
        x = _lib.as_c128(x)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        xx = np.ascontiguousarray(x.reshape(self.n, nrhs).T)
        y = np.zeros_like(xx)
        check(self._lib.sie_matvec(self._h, dptr(xx.view(np.float64)), dptr(y.view(np.float64)), nrhs,
                                   PRECISIONS[precision]))
        y = y.T
        return y[:, 0] if x.ndim == 1 else y

    def autotune(self, precision="fp64"):
        """Pick the fastest kernel variants for this mesh; returns the product's device time
        before and after [ms] and the chosen variants."""
        ms = np.zeros(2)
        modes = np.zeros(5, dtype=np.int32)
        check(self._lib.sie_autotune(self._h, PRECISIONS[precision], dptr(ms), iptr(modes)))
        names = ["near", "aggregate", "sr", "receive", "overlap"]
        return ms[0], ms[1], dict(zip(names, modes.tolist()))

    def set_inner_operator(self, other):
        """Inner complex64 products of the mixed solver through `other` (a context on the
        same mesh and tree, e.g. with a lower truncation number); None restores this one."""
        check(self._lib.sie_set_inner_operator(self._h, other._h if other is not None else None))
        self._inner = other  # keep it alive while linked

    def matvec_adjoint(self, x):
        """y = Z^H x (FP64), the operator of the adjoint solve."""
        x = _lib.as_c128(x)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        xx = np.ascontiguousarray(x.reshape(self.n, nrhs).T)
        y = np.zeros_like(xx)
        check(self._lib.sie_matvec_adjoint(self._h, dptr(xx.view(np.float64)), dptr(y.view(np.float64)), nrhs))
        y = y.T
        return y[:, 0] if x.ndim == 1 else y

    def grad(self, x, k_in, E_in, pts, restart=50, max_iterations=2000, tolerance=1e-10,
             raise_on_noconv=True):
        """Objective J = sum of far-field intensities at pts for the solution x of the plane
        wave (k_in, E_in), and dJ/dz of every mesh vertex (adjoint solve in FP64)."""
        lib = self._lib
        x = np.ascontiguousarray(_lib.as_c128(x))
        k = np.ascontiguousarray(k_in, dtype=np.float64)
        e = np.ascontiguousarray(E_in, dtype=np.float64)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        cfg = SieSolverCfg()
        lib.sie_solver_default(C.byref(cfg))
        cfg.restart, cfg.max_iterations, cfg.tolerance = int(restart), int(max_iterations), float(tolerance)
        g = np.zeros(self.nv)
        J = C.c_double()
        st = SieStats()
        code = lib.sie_grad(self._h, dptr(x.view(np.float64)), dptr(k), dptr(e), dptr(p), p.shape[0],
                            C.byref(cfg), dptr(g), C.byref(J), C.byref(st))
        if code != _lib.SIE_OK and not (code == _lib.SIE_ERR_NOCONV and not raise_on_noconv):
            check(code)
        return J.value, g, {f: getattr(st, f) for f, _ in SieStats._fields_}

    def matvec_device(self, d_x, d_y, nrhs=1, precision="fp64", stream=0):
        """Device-pointer matvec (torch tensors' data_ptr() or raw addresses)."""
        check(self._lib.sie_matvec_device(self._h, C.c_void_p(d_x), C.c_void_p(d_y), nrhs,
                                          PRECISIONS[precision], C.c_void_p(stream)))

    def rhs_planewave(self, k_in, E_in):
        k = np.ascontiguousarray(np.atleast_2d(k_in), dtype=np.float64)
        e = np.ascontiguousarray(np.atleast_2d(E_in), dtype=np.float64)
        nrhs = k.shape[0]
        b = np.zeros((nrhs, self.n), dtype=np.complex128)
        check(self._lib.sie_rhs_planewave(self._h, dptr(k), dptr(e), nrhs, dptr(b.view(np.float64))))
        return b[0] if np.ndim(k_in) == 1 else b.T

    def solve(self, b, restart=50, max_iterations=650, tolerance=1e-6, x0=None, precision="fp64",
              inner_restart=30, inner_tolerance=1e-4, time_limit_s=0.0, raise_on_noconv=True):
        lib = self._lib
        b = _lib.as_c128(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bb = np.ascontiguousarray(b.reshape(self.n, nrhs).T)
        x = np.zeros_like(bb) if x0 is None else np.ascontiguousarray(_lib.as_c128(x0).reshape(self.n, nrhs).T)
        cfg = SieSolverCfg()
        lib.sie_solver_default(C.byref(cfg))
        cfg.restart, cfg.max_iterations, cfg.tolerance = int(restart), int(max_iterations), float(tolerance)
        cfg.use_initial_guess = int(x0 is not None)
        cfg.precision = PRECISIONS[precision]
        cfg.inner_restart, cfg.inner_tolerance = int(inner_restart), float(inner_tolerance)
        cfg.time_limit_s = float(time_limit_s)
        stats = (SieStats * nrhs)()
        code = lib.sie_solve(self._h, dptr(bb.view(np.float64)), dptr(x.view(np.float64)), nrhs,
                             C.byref(cfg), stats)
        if code != _lib.SIE_OK and not (code == _lib.SIE_ERR_NOCONV and not raise_on_noconv):
            check(code)
        st = [{f: getattr(s, f) for f, _ in SieStats._fields_} for s in stats]
        x = x.T
        return (x[:, 0], st[0]) if b.ndim == 1 else (x, st)

    def solve_direct(self, b):
        """LU solve of the dense system (context made with dense=True)."""
        b = _lib.as_c128(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bb = np.ascontiguousarray(b.reshape(self.n, nrhs).T)
        x = np.zeros_like(bb)
        check(self._lib.sie_solve_direct(self._h, dptr(bb.view(np.float64)), dptr(x.view(np.float64)), nrhs))
        x = x.T
        return x[:, 0] if b.ndim == 1 else x

    def set_preconditioner(self, kind="near"):
        """Preconditioner of later solves: "near" (near-field restricted additive Schwarz,
        applied on the right) or None."""
        kinds = {None: _lib.SIE_PRECOND_NONE, "none": _lib.SIE_PRECOND_NONE, "near": _lib.SIE_PRECOND_NEAR}
        check(self._lib.sie_set_preconditioner(self._h, kinds[kind]))
        return self

    def precondition_right(self, v1):
        """P v1 with the preconditioner of set_preconditioner."""
        v1 = _lib.as_c128(v1)
        v2 = np.zeros_like(v1)
        check(self._lib.sie_precondition_right(self._h, dptr(v1.view(np.float64)), dptr(v2.view(np.float64))))
        return v2

    def solve_direct_mixed(self, b, tolerance=1e-10, max_refinements=30, raise_on_noconv=True):
        """Direct solve with a complex64 tensor-core LU and FP64 iterative refinement
        (context made with dense=True); returns the currents and the per-vector stats."""
        b = _lib.as_c128(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bb = np.ascontiguousarray(b.reshape(self.n, nrhs).T)
        x = np.zeros_like(bb)
        stats = (SieStats * nrhs)()
        code = self._lib.sie_solve_direct_mixed(self._h, dptr(bb.view(np.float64)), dptr(x.view(np.float64)), nrhs,
                                                float(tolerance), int(max_refinements), stats)
        if code != _lib.SIE_OK and not (code == _lib.SIE_ERR_NOCONV and not raise_on_noconv):
            check(code)
        st = [{f: getattr(s, f) for f, _ in SieStats._fields_} for s in stats]
        x = x.T
        return (x[:, 0], st[0]) if b.ndim == 1 else (x, st)

    def release_factors(self):
        """Drop the kept LU factors (the next direct solve factorises again)."""
        check(self._lib.sie_release_factors(self._h))

    def invalidate_factors(self):
        """Mark the kept LU factors out of date but keep their memory (the next direct solve
        factorises again into the same buffers)."""
        check(self._lib.sie_invalidate_factors(self._h))

    def precondition_left(self, v1):
        v1 = _lib.as_c128(v1)
        v2 = np.zeros_like(v1)
        check(self._lib.sie_precondition_left(self._h, dptr(v1.view(np.float64)), dptr(v2.view(np.float64))))
        return v2

    def farfield(self, x, pts):
        x = _lib.as_c128(x)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        npts = p.shape[0]
        E = np.zeros((npts, 3), np.complex128)
        H = np.zeros((npts, 3), np.complex128)
        I = np.zeros(npts)
        check(self._lib.sie_farfield(self._h, dptr(x.view(np.float64)), dptr(p), npts,
                                     dptr(E.view(np.float64)), dptr(H.view(np.float64)), dptr(I)))
        return E, H, I

    def field_interior(self, x, pts, eps_r=None):
        """E, H at points inside the body (Integration_scattered_field_tri_within_medium,
        src/lib_sie_tri_calculation_mod.f90:2829-2877): the total field there, in the
        medium of relative permittivity eps_r (the body's, eps_r2, by default)."""
        x = _lib.as_c128(x)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        npts = p.shape[0]
        er = complex(self.cfg.eps_r2_re, self.cfg.eps_r2_im) if eps_r is None else complex(eps_r)
        E = np.zeros((npts, 3), np.complex128)
        H = np.zeros((npts, 3), np.complex128)
        check(self._lib.sie_field_interior(self._h, dptr(x.view(np.float64)), dptr(p), npts, er.real, er.imag,
                                           dptr(E.view(np.float64)), dptr(H.view(np.float64))))
        return E, H

    def near_field(self, x, pts, inside=None, k_in=None, E_in=None):
        """E, H of a near-field map, as the plane-wave branch of
        lib_sie_tri_observation_field_calculation (src/lib_sie_tri_solver_normal.f90:
        385-420): points with inside[i] true (by default: inside the context's closed
        mesh, mesh.inside) get the interior field (eps_r2), with a
        component of E below 1e-20 in modulus set to zero together with the same
        component of H, as the reference does; the others get the scattered field plus,
        when k_in and E_in are given (the reference's total_field), the incident plane
        wave of lib_sie_tri_input_field_calculation (src/lib_sie_tri_calculation_mod.f90:
        2604-2609): E_in exp(-i k1 k_in . r), H = k1 k_in x E / (mu_1 omega).  Every point
        uses the 3-point rule, as the reference does for rough surfaces; for spheres it
        raises it near the surface (ngp_near_field_distance_tri, :2627-2670)."""
        x = _lib.as_c128(x)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        if inside is None:
            from .mesh import inside as inside_mesh
            inside = inside_mesh(self.verts, self.tris, p)
        inside = np.asarray(inside, dtype=bool).reshape(-1)
        if inside.size != p.shape[0]:
            raise ValueError("near_field: inside must have one entry per point")
        E = np.zeros((p.shape[0], 3), np.complex128)
        H = np.zeros((p.shape[0], 3), np.complex128)
        if inside.any():
            Ei, Hi = self.field_interior(x, p[inside])
            small = np.abs(Ei) < 1e-20
            Ei[small] = 0
            Hi[small] = 0
            E[inside], H[inside] = Ei, Hi
        out = ~inside
        if out.any():
            Es, Hs, _ = self.farfield(x, p[out])
            if k_in is not None:
                mu0 = float(np.float32(1.2566370614e-6))
                c0 = float(np.float32(2.99792458e8))
                lam = float(self.cfg.lambda_)
                k1 = 2 * np.pi / lam * np.sqrt(complex(self.cfg.eps_r1_re, self.cfg.eps_r1_im))
                omega = 2 * np.pi * c0 / lam
                kv = np.asarray(k_in, dtype=np.float64).reshape(3)
                Einc = np.asarray(E_in, dtype=np.complex128).reshape(1, 3) * np.exp(-1j * k1 * (p[out] @ kv))[:, None]
                Hinc = np.cross(k1 * kv[None, :], Einc) / (mu0 * omega)
                Es = Es + Einc
                Hs = Hs + Hinc
            E[out], H[out] = Es, Hs
        return E, H

    def farfield_device_noalloc(self, d_x, d_pts, npts, d_E, d_H, d_I, stream=0):
        """Far field on device buffers (raw addresses) with no device allocation; the
        work is queued on `stream` and not waited for."""
        check(self._lib.sie_farfield_device_noalloc(
            self._h, C.c_void_p(d_x), C.c_void_p(d_pts), int(npts), C.c_void_p(d_E),
            C.c_void_p(d_H), C.c_void_p(d_I), C.c_void_p(stream)))

    # --- introspection ------------------------------------------------------
    def edges(self):
        e = np.zeros(2 * self.n_edges, np.int32)
        c = np.zeros(2 * self.n_edges, np.int32)
        check(self._lib.sie_get_edges(self._h, iptr(e), iptr(c)))
        return e.reshape(-1, 2), c.reshape(-1, 2)

    def tree(self):
        d = np.zeros(4)
        leaf = np.zeros(self.n_edges, np.int64)
        check(self._lib.sie_get_tree(self._h, dptr(d), lptr(leaf)))
        return d[0], d[1:], leaf

    def blocks(self, m, n):
        m = np.ascontiguousarray(m, np.int32)
        n = np.ascontiguousarray(n, np.int32)
        out = np.zeros((len(m), 4), np.complex128)
        check(self._lib.sie_get_blocks(self._h, iptr(m), iptr(n), len(m), dptr(out.view(np.float64))))
        return out

    def near_entries(self, m, n):
        m = np.ascontiguousarray(m, np.int32)
        n = np.ascontiguousarray(n, np.int32)
        out = np.zeros((len(m), 4), np.complex128)
        check(self._lib.sie_get_near_entries(self._h, iptr(m), iptr(n), len(m), dptr(out.view(np.float64))))
        return out

    def rt(self, edges):
        e = np.ascontiguousarray(edges, np.int32)
        q = C.c_int()
        check(self._lib.sie_num_directions(self._h, C.byref(q)))
        out = np.zeros((len(e), 4, q.value), np.complex128)
        check(self._lib.sie_get_rt(self._h, iptr(e), len(e), dptr(out.view(np.float64))))
        return out

    def timings(self):
        v = np.zeros(23)
        check(self._lib.sie_get_timings(self._h, dptr(v), 23))
        keys = ["fill_ms", "rt_tl_ms", "setup_ms", "mv_total_ms", "mv_near_ms", "mv_agg_ms",
                "mv_ss_ms", "mv_sr_ms", "mv_rr_ms", "mv_recv_ms", "gm_passes_per_step", "graph_replays",
                "precond_ms", "lu_factor_ms", "lu_gemm_ms", "lu_gemm_flops", "lu_gemm_launches",
                "lu_panel_ms", "lu_swap_ms", "lu_trsm_ms", "lu_tile_ms", "lu_f16", "lu_factorizations"]
        return dict(zip(keys, v))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sie_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
