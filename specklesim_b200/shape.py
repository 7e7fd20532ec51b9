"""Height-map shape parameterisation of a rough slab and the far-field speckle objective
as a torch autograd function.

The rough top face of a slab moves as z = z0 + B c: c are the controls of a uniform
bicubic B-spline grid over the patch, B their basis evaluated at the top-face vertices.
The objective J is the far-field intensity summed over observation points; its gradient
dJ/dc = B^T dJ/dz comes from one adjoint solve in `Sie.grad`.
"""
import numpy as np


def bspline_basis_1d(x, x0, x1, n):
    """Uniform cubic B-spline basis (n functions, n >= 4) covering [x0, x1]: values at x,
    shape (len(x), n).  Knot spacing (x1 - x0) / (n - 3); function i is centred at
    x0 + (i - 1) * spacing, so every point of the interval sees four functions."""
    x = np.asarray(x, dtype=float)
    h = (x1 - x0) / (n - 3)
    c = x0 + (np.arange(n) - 1) * h
    u = np.abs(x[:, None] - c[None, :]) / h
    return np.where(u < 1, (4 - 6 * u ** 2 + 3 * u ** 3) / 6, np.where(u < 2, (2 - u) ** 3 / 6, 0.0))


class BSplineHeight:
    """n x n bicubic B-spline grid over [x0, x1] x [y0, y1]."""

    def __init__(self, n, x0, x1, y0, y1):
        self.n, self.x0, self.x1, self.y0, self.y1 = n, x0, x1, y0, y1

    def matrix(self, xy):
        """Basis at points xy (k, 2): (k, n * n), column i * n + j = B_i(x) B_j(y)."""
        Bx = bspline_basis_1d(xy[:, 0], self.x0, self.x1, self.n)
        By = bspline_basis_1d(xy[:, 1], self.y0, self.y1, self.n)
        return (Bx[:, :, None] * By[:, None, :]).reshape(len(xy), -1)


def cone_points(n, axis, half_angle_deg, seed, r=5.0):
    """n observation points at distance r, directions uniform over the cone of the given
    half angle around `axis`."""
    rng = np.random.default_rng(seed)
    a = np.asarray(axis, dtype=float)
    a = a / np.linalg.norm(a)
    cmin = np.cos(np.deg2rad(half_angle_deg))
    ct = rng.uniform(cmin, 1.0, n)
    ph = rng.uniform(0.0, 2 * np.pi, n)
    st = np.sqrt(1 - ct ** 2)
    t = np.cross(a, [1.0, 0, 0] if abs(a[0]) < 0.9 else [0, 1.0, 0])
    t /= np.linalg.norm(t)
    u = np.cross(a, t)
    d = ct[:, None] * a + st[:, None] * (np.cos(ph)[:, None] * t + np.sin(ph)[:, None] * u)
    return r * d


class SpeckleProblem:
    """A rough slab whose top-face vertices (indices `top`) follow z0 + B c, lit by one
    plane wave; J = sum of far-field intensities at `pts`.  dense=True solves the dense
    system by LU (exact); otherwise FP64 MLFMM GMRES to `tolerance`."""

    def __init__(self, V0, T, top, spline, wavelength, eps_r2, k_in, E_in, pts, dense=False,
                 tree_s_opt=250, tolerance=1e-10, restart=50, max_iterations=4000, mixed_direct=False):
        self.V0 = np.asarray(V0, dtype=float)
        self.T = np.asarray(T)
        self.top = np.asarray(top)
        self.B = spline.matrix(self.V0[self.top, :2])
        self.wl, self.eps = wavelength, eps_r2
        self.k_in, self.E_in, self.pts = np.asarray(k_in, float), np.asarray(E_in, float), np.asarray(pts, float)
        self.dense, self.s_opt = dense, tree_s_opt
        # dense=True with mixed_direct: objective() solves with the complex64 tensor-core LU
        # and FP64 refinement to `tolerance`; value_and_grad() keeps the FP64 LU, whose
        # factors also give the adjoint solve
        self.mixed_direct = mixed_direct
        self.solver = dict(restart=restart, max_iterations=max_iterations, tolerance=tolerance)

    def vertices(self, c):
        V = self.V0.copy()
        V[self.top, 2] += self.B @ np.asarray(c, dtype=float)
        return V

    def _context(self, V):
        from .sie import Sie
        if self.dense:
            return Sie(V, self.T, self.wl, self.eps, dense=True).setup()
        return Sie(V, self.T, self.wl, self.eps, tree_s_opt=self.s_opt).setup()

    def _solve(self, g, mixed=True):
        b = g.rhs_planewave(self.k_in, self.E_in)
        if self.dense and self.mixed_direct and mixed:
            x, _ = g.solve_direct_mixed(b, tolerance=self.solver["tolerance"])
            return x
        if self.dense:
            return g.solve_direct(b)
        x, _ = g.solve(b, **self.solver)
        return x

    def objective(self, c):
        """J at controls c."""
        g = self._context(self.vertices(c))
        try:
            x = self._solve(g)
            return float(np.sum(g.farfield(x, self.pts)[2]))
        finally:
            g.close()

    def value_and_grad(self, c):
        """J and dJ/dc (one forward solve, one adjoint solve)."""
        g = self._context(self.vertices(c))
        try:
            x = self._solve(g, mixed=False)
            J, dz, _ = g.grad(x, self.k_in, self.E_in, self.pts, **self.solver)
            return J, self.B.T @ dz[self.top]
        finally:
            g.close()


def speckle_objective(problem):
    """torch.autograd.Function computing J(c) for `problem` (a SpeckleProblem), with the
    adjoint gradient as its backward."""
    import torch

    class _Speckle(torch.autograd.Function):
        @staticmethod
        def forward(ctx, c):
            J, dc = problem.value_and_grad(c.detach().cpu().numpy())
            ctx.save_for_backward(torch.as_tensor(dc, dtype=c.dtype))
            return torch.tensor(J, dtype=c.dtype)

        @staticmethod
        def backward(ctx, gout):
            (dc,) = ctx.saved_tensors
            return gout * dc

    return _Speckle.apply
