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

Run: python -m tests.c5_check  (prints one JSON line; exit status 1 if a control is off
by more than 1e-4 relative)."""
import json
import sys
import time

import numpy as np


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
    rows = []
    t0 = time.perf_counter()
    for i in picks:
        cp, cm = c0.copy(), c0.copy()
        cp[i] += h
        cm[i] -= h
        fd = (pb.objective(cp) - pb.objective(cm)) / (2 * h)
        rows.append((int(i), float(grad[i]), float(fd), float(abs(grad[i] - fd) / max(abs(fd), 1e-300))))
    t_fd = time.perf_counter() - t0
    worst = max(r[3] for r in rows)
    out = {"workload": "slab10 seed 2, 64 x 64 B-spline controls N(0, 0.05 lambda), 256 directions in a "
                       "20-degree cone around specular, 32 random controls, step 1e-4 lambda",
           "J": J, "gradient_seconds": t_grad, "finite_difference_seconds": t_fd,
           "max_rel_err": worst, "within_1e-4": int(sum(r[3] <= 1e-4 for r in rows)),
           "controls": [{"index": r[0], "adjoint": r[1], "fd": r[2], "rel_err": r[3]} for r in rows]}
    print(json.dumps(out))
    return 0 if worst <= 1e-4 else 1


if __name__ == "__main__":
    sys.exit(main())
