"""Benchmark of the SIE hot path: plane-wave solves per second on the rough-slab
workload (10 lambda x 10 lambda, ~19.5k triangles, ~29k RWG edges, plain FP64
MLFMM + GMRES to 1e-6).

One step = one GMRES solve of one right-hand side on a set-up problem (near
field, radiation patterns and translation tables are built once, as the
reference does for its incidence-angle loop, main.f90:450-463).  `value` times
the device solve (inputs resident in HBM); `e2e` times the public host API with
the right-hand side copied in from pinned memory and the currents copied out.

Multi-GPU (torchrun): every rank solves its own realisation (seed = rank),
weak scaling, no collective on the data path; timings are max-reduced.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s @1e-5 far-field err vs FP64: mixed vs plain FP64 GPU; matvec % HBM peak"
WL = 632.8e-9
EPS = -11.7 - 1.26j  # exp(+iwt) convention of the reference (lossy => Im < 0)

WORKLOADS = {
    # the headline case: 10 lambda x 10 lambda rough slab, seed 0, corr 1 lambda, RMS 0.5 lambda,
    # 1 lambda thick
    "slab10": dict(length_wl=10.0, rms_wl=0.5, corr_wl=1.0, thickness_wl=1.0, cells=64, seed=0),
    # a small case for quick checks
    "slab4": dict(length_wl=4.0, rms_wl=0.3, corr_wl=1.0, thickness_wl=1.0, cells=24, seed=0),
}


# matvecs of one budgeted FP64 solve on the GPU (650 Arnoldi steps + the final true
# residual); the CPU arm times matvecs and multiplies by this count
MATVECS_PER_SOLVE = {"slab10": 651, "slab4": 651}


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                pw.append(float(r[2]))
                for n, v in zip(names, r[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w": statistics.median(pw) if pw else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_mesh(wl_name, seed):
    from specklesim_b200 import mesh
    w = dict(WORKLOADS[wl_name])
    w["seed"] = seed
    return mesh.slab_config(w["length_wl"], WL, w["rms_wl"], w["corr_wl"], w["seed"], cells=w["cells"],
                            thickness_wl=w["thickness_wl"])


def level_stats(g):
    """Boxes per MLFMM level and I4 (far-interaction) pairs per level, from the leaf Morton
    indices the library reports (the I4 rule: children of the parent's neighbours that are
    not neighbours themselves)."""
    _, _, leaf = g.tree()
    out = []
    for l in range(g.l_min, g.l_max + 1):
        boxes = np.unique(leaf >> (3 * (g.l_max - l)))
        coords = np.stack([demorton(boxes, l, k) for k in range(3)], axis=1)
        have = {tuple(c) for c in coords}
        n_i4 = 0
        for c in coords:
            p = c // 2
            for d in np.ndindex(3, 3, 3):
                pn = p + np.array(d) - 1
                for ch in np.ndindex(2, 2, 2):
                    s = 2 * pn + np.array(ch)
                    if np.max(np.abs(s - c)) > 1 and tuple(s) in have:
                        n_i4 += 1
        out.append((l, len(boxes), n_i4))
    return out


def demorton(b, l, axis):
    """Coordinate `axis` (0 = x, most significant) of Morton indices b at level l."""
    v = np.zeros_like(b)
    for bit in range(l):
        v |= ((b >> (3 * bit + 2 - axis)) & 1) << bit
    return v


def matvec_algorithmic(g, Q):
    """Algorithmic DRAM bytes of one FP64 matvec, and the FP64 flops of its SR step.
    Bytes: near panels (a, b, d: 48 B per 2x2 block), radiation patterns read by the
    aggregate and the receive, x in and y out, C and D of every level written and read.
    The SR source coefficients are read from L2 (each level's C fits), so they are not
    DRAM bytes.  SR flops: 4 complex multiply-adds = 32 real flops per (I4 pair,
    direction, medium); medium 2 only on the leaf level (k2 complex)."""
    M, N, s = g.n_edges, g.n, 16
    st = level_stats(g)
    near = g.near_nnz * 3 * s
    rt = 2 * M * 4 * Q * s
    xy = 2 * N * s
    coeff = sum(nb * 8 * Q * s * 4 for _, nb, _ in st)
    sr_flops = sum(ni4 * Q * 32 * (2 if l == g.l_max else 1) for l, _, ni4 in st)
    return dict(near=near, rt=rt, xy=xy, coeff=coeff, total=near + rt + xy + coeff, sr_flops=sr_flops,
                levels=st)


def fp64_dgemm_tflops(dev):
    """FP64 denominator measured on this GPU: best of 5 torch float64 matmuls (cuBLAS DGEMM)."""
    import torch
    a = torch.randn(4096, 4096, dtype=torch.float64, device=dev)
    b = torch.randn(4096, 4096, dtype=torch.float64, device=dev)
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * 4096 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


EPS_CONVERGING = 2.25 - 0.01j


def hemisphere_grid(n=128, r=5.0):
    """The 128 x 128 (theta, phi) grid over the upper hemisphere at r = 5 m."""
    th = (np.arange(n) + 0.5) * (0.5 * np.pi / n)
    ph = (np.arange(n) + 0.5) * (2 * np.pi / n)
    T, P = np.meshgrid(th, ph, indexing="ij")
    return r * np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=-1).reshape(-1, 3)


def mixed_vs_fp64(V, T, tol):
    """Solves/s of the mixed-precision solver (FP64 flexible GMRES around FP32 GMRES)
    against the plain FP64 GMRES, both to the same backward error, and the relative error
    of the mixed far-field intensity on the 128 x 128 hemisphere grid.  The slab mesh of
    the workload with a dielectric body: the metallic ICTF system stalls in both
    precisions, so it gives no equal-accuracy comparison."""
    from specklesim_b200 import Sie, incidence
    g = Sie(V, T, WL, EPS_CONVERGING, tree_s_opt=250, truncation_number=19).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    pts = hemisphere_grid()
    x64, s64 = g.solve(b, restart=50, max_iterations=4000, tolerance=tol, raise_on_noconv=False)
    xm, sm = g.solve(b, restart=10, max_iterations=100, tolerance=tol, precision="mixed",
                     inner_restart=30, inner_tolerance=1e-2, raise_on_noconv=False)
    xm, sm = g.solve(b, restart=10, max_iterations=100, tolerance=tol, precision="mixed",
                     inner_restart=30, inner_tolerance=1e-2, raise_on_noconv=False)
    I64 = g.farfield(x64, pts)[2]
    Im = g.farfield(xm, pts)[2]
    # the inner products through a K = 12 operator on the same mesh (a cheaper preconditioner
    # operator; the outer FP64 products stay K = 19)
    gi = Sie(V, T, WL, EPS_CONVERGING, tree_s_opt=250, truncation_number=12).setup()
    g.set_inner_operator(gi)
    xk, sk = g.solve(b, restart=10, max_iterations=100, tolerance=tol, precision="mixed",
                     inner_restart=60, inner_tolerance=1e-2, raise_on_noconv=False)
    g.set_inner_operator(None)
    Ik = g.farfield(xk, pts)[2]
    batched = batched_mixed(g, pts, tol, inner=gi)
    g.close()
    gi.close()
    return {
        "workload": f"same slab mesh, eps = {EPS_CONVERGING} (converging), tolerance {tol}",
        "fp64": {"solves_per_s": 1.0 / s64["seconds"], "iterations": s64["iterations"],
                 "backward_error": s64["backward_error_true"], "converged": bool(s64["converged"])},
        "mixed": {"solves_per_s": 1.0 / sm["seconds"], "outer_iterations": sm["iterations"],
                  "inner_iterations": sm["inner_iterations"], "backward_error": sm["backward_error_true"],
                  "converged": bool(sm["converged"]), "inner": "GMRES(30) FP32 to 1e-2, outer FGMRES(10) FP64"},
        "speedup": s64["seconds"] / sm["seconds"],
        "mixed_inner_k12": {"speedup": s64["seconds"] / sk["seconds"], "outer_iterations": sk["iterations"],
                            "converged": bool(sk["converged"]),
                            "farfield_rel_err_vs_fp64": float(np.linalg.norm(Ik - I64) / np.linalg.norm(I64)),
                            "inner": "GMRES(60) complex64 through a K = 12 context to 1e-2, outer FGMRES(10) FP64"},
        "farfield_rel_err_vs_fp64": float(np.linalg.norm(Im - I64) / np.linalg.norm(I64)),
        "currents_rel_err_vs_fp64": float(np.linalg.norm(xm - x64) / np.linalg.norm(x64)),
        "farfield_points": int(pts.shape[0]),
        "batched": batched,
    }


def batched_mixed(g, pts, tol, inner=None, fp64_sample=4):
    """The 16 plane waves of the batching form (theta 0/10/20/30 deg x phi 0/90 deg x TE/TM)
    solved together by the batched mixed-precision solver, against plain FP64 GMRES solves
    of the first `fp64_sample` of them one at a time (FP64 time per solve = mean over the
    sample).  Errors: currents and 128 x 128 far-field intensity of the sampled columns.
    With `inner` the inner complex64 products go through that context (a lower truncation
    number); the same batch is also timed with the inner products on g itself."""
    from specklesim_b200 import incidence
    incs = [incidence(np.deg2rad(t), np.deg2rad(p), pol, 2)
            for t in (0, 10, 20, 30) for p in (0, 90) for pol in ("TM", "TE")]
    B = np.stack([g.rhs_planewave(k, E) for k, E in incs], axis=1)
    kw = dict(restart=10, max_iterations=100, tolerance=tol, precision="mixed", inner_restart=60,
              inner_tolerance=1e-2, raise_on_noconv=False)
    Xb, sb = g.solve(B[:, :2], **kw)  # warm-up (allocation of the batch workspace)
    Xb, sb = g.solve(B, **kw)
    t_same = sb[0]["seconds"]
    its_same = max(s["iterations"] for s in sb)
    if inner is not None:
        g.set_inner_operator(inner)
        Xb, sb = g.solve(B[:, :2], **kw)
        Xb, sb = g.solve(B, **kw)
        g.set_inner_operator(None)
    t_batch = sb[0]["seconds"]
    t64, ferr, cerr = [], [], []
    for j in range(fp64_sample):
        x64, s64 = g.solve(B[:, j], restart=50, max_iterations=4000, tolerance=tol, raise_on_noconv=False)
        t64.append(s64["seconds"])
        I64 = g.farfield(x64, pts)[2]
        Ib = g.farfield(Xb[:, j], pts)[2]
        ferr.append(float(np.linalg.norm(Ib - I64) / np.linalg.norm(I64)))
        cerr.append(float(np.linalg.norm(Xb[:, j] - x64) / np.linalg.norm(x64)))
    per64 = float(np.mean(t64))
    return {
        "rhs": B.shape[1], "seconds": t_batch, "solves_per_s": B.shape[1] / t_batch,
        "fp64_seconds_per_solve": per64, "fp64_sample": fp64_sample,
        "speedup_vs_fp64": per64 / (t_batch / B.shape[1]),
        "outer_iterations_max": max(s["iterations"] for s in sb),
        "backward_error_max": max(s["backward_error_true"] for s in sb),
        "converged": all(bool(s["converged"]) for s in sb),
        "farfield_rel_err_vs_fp64_max": max(ferr), "currents_rel_err_vs_fp64_max": max(cerr),
        "inner": "lockstep GMRES(60) complex64 to 1e-2 on one batched product per step, outer FGMRES(10) FP64",
        "inner_operator": ("K = 12 (Q = 290) complex64 MLFMM on the same mesh; outer products K = 19"
                           if inner is not None else "the outer operator (K = 19) in complex64"),
        "same_operator": {"seconds": t_same, "speedup_vs_fp64": per64 / (t_same / B.shape[1]),
                          "outer_iterations_max": its_same},
    }


def gradient_timing(tol):
    """One shape gradient in the differentiation form's setting: slab10 with seed 2 and the
    metal, 256 observation directions in a 20-degree cone around specular.  ICTF on this
    slab stalls in GMRES, so the forward and the adjoint solves both run the reference's
    budget (restart 50, 650 iterations); the time is sie_grad's wall time (adjoint solve
    plus the derivative kernels over all vertices)."""
    from specklesim_b200 import Sie, incidence
    from specklesim_b200.shape import cone_points
    V, T = build_mesh("slab10", 2)
    g = Sie(V, T, WL, EPS, tree_s_opt=250, truncation_number=19).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    x, _ = g.solve(g.rhs_planewave(k, E), restart=50, max_iterations=650, tolerance=tol, raise_on_noconv=False)
    pts = cone_points(256, [0, 0, 1], 20.0, seed=2)
    kw = dict(restart=50, max_iterations=650, tolerance=tol, raise_on_noconv=False)
    g.grad(x, k, E, pts[:8], **kw)  # warm-up: gradient tables and workspace
    t0 = time.perf_counter()
    J, dz, st = g.grad(x, k, E, pts, **kw)
    t = time.perf_counter() - t0
    g.close()
    return {"workload": "slab10 seed 2, eps -11.7-1.26i, 256 directions in a 20-degree cone around specular",
            "vertices": int(len(V)), "seconds": t, "adjoint_solve_seconds": st["seconds"],
            "adjoint_iterations": st["iterations"], "derivative_kernels_seconds": t - st["seconds"],
            "objective": J}


def committed_traffic():
    """DRAM bytes (read + write) of one matvec's kernels from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "matvec_dram_traffic_slab10.md")
    try:
        for line in open(p):
            if line.startswith("total_dram_bytes_per_matvec:"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


def cpu_reference(V, T, matvecs_per_solve, threads, s_opt=250, budget_matvecs=2):
    """The oracle (C++ restatement of the reference) timed on the host cores."""
    from oracle.oracle import Oracle
    o = Oracle(V, T, WL, EPS, tree_s_opt=s_opt, threads=threads)
    t0 = time.perf_counter()
    o.tree()
    o.setup_fmm()
    t_setup = time.perf_counter() - t0
    x = np.random.default_rng(0).standard_normal(o.N) + 0j
    ts = []
    for _ in range(budget_matvecs):
        t1 = time.perf_counter()
        o.matvec(x)
        ts.append(time.perf_counter() - t1)
    t_mv = min(ts)
    o.close()
    per_solve = t_mv * matvecs_per_solve
    return dict(value=1.0 / per_solve, unit="solves/s", cores=threads, kind="port",
                sample=(f"oracle C++ restatement (OpenMP, {threads} threads): set-up {t_setup:.1f} s untimed, "
                        f"{budget_matvecs} MLFMM matvecs timed ({t_mv:.3f} s each); solves/s = "
                        f"1 / (matvec time x {matvecs_per_solve} matvecs per solve of the GPU run)"),
                setup_s=t_setup, matvec_s=t_mv)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="slab10", choices=list(WORKLOADS))
    ap.add_argument("--restart", type=int, default=50)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--max-iterations", type=int, default=650)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--reference-matvecs-per-solve", type=int, default=0)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's CPU implementation of the path (the oracle port) on the host cores
        if rank != 0:
            return
        V, T = build_mesh(args.workload, 0)
        threads = os.cpu_count() or 1
        mps = args.reference_matvecs_per_solve or MATVECS_PER_SOLVE[args.workload]
        cb = cpu_reference(V, T, mps, threads)
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / cb["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload} rough slab (seed 0), ICTF, ng=3, s_opt=250, K=19",
                       "matvecs_per_solve": mps},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    from specklesim_b200 import Sie, incidence, _lib

    V, T = build_mesh(args.workload, rank)
    t0 = time.perf_counter()
    g = Sie(V, T, WL, EPS, tree_s_opt=250, truncation_number=19, device=local)
    g.setup()
    setup_s = time.perf_counter() - t0
    # kernel variants picked for this mesh by the library's autotuner (same product)
    tune_before, tune_after, tune_modes = g.autotune("fp64")
    lib = _lib.load()
    stream = torch.cuda.Stream()
    _lib.check(lib.sie_set_stream(g._h, __import__("ctypes").c_void_p(stream.cuda_stream)))

    k, E = incidence(0.0, 0.0, "TM", 2)  # x-polarised normal incidence along -z
    b_host = g.rhs_planewave(k, E)
    N = g.n
    dev = torch.device("cuda", local)
    with torch.cuda.stream(stream):
        b = torch.from_numpy(b_host.view(np.float64)).to(dev)
        x = torch.zeros_like(b)
    stream.synchronize()

    import ctypes as C
    cfg = _lib.SieSolverCfg()
    lib.sie_solver_default(C.byref(cfg))
    cfg.restart, cfg.max_iterations, cfg.tolerance = args.restart, args.max_iterations, args.tol
    st = _lib.SieStats()

    def solve_dev():
        rc = lib.sie_solve_device(g._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1, C.byref(cfg),
                                  C.byref(st))
        if rc != _lib.SIE_ERR_NOCONV:  # the budgeted solve ends like the reference's info(1) = -4
            _lib.check(rc)

    for _ in range(args.warmup):
        solve_dev()
    iters, mvs, conv, be = st.iterations, st.matvecs, st.converged, st.backward_error_true

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = lib.sie_launch_count()
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            solve_dev()
        e1.record(stream)
        barrier()
    launches = lib.sie_launch_count() - l0
    t_dev = e0.elapsed_time(e1) / 1000.0
    if world > 1:
        tt = torch.tensor([t_dev], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev = float(tt.item())
    value = world * args.steps / t_dev

    # ---- end to end through the public host API (pinned host buffers)
    bp = torch.from_numpy(b_host.view(np.float64).copy()).pin_memory()
    xp = torch.zeros_like(bp).pin_memory()
    stats = (_lib.SieStats * 1)()
    dp = C.POINTER(C.c_double)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk_e2e:
        e2.record(stream)
        for _ in range(args.steps):
            rc = lib.sie_solve(g._h, C.cast(bp.data_ptr(), dp), C.cast(xp.data_ptr(), dp), 1, C.byref(cfg), stats)
            if rc != _lib.SIE_ERR_NOCONV:
                _lib.check(rc)
        e3.record(stream)
        barrier()
    t_e2e = e2.elapsed_time(e3) / 1000.0
    if world > 1:
        tt = torch.tensor([t_e2e], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = world * args.steps / t_e2e
    x_e2e = xp.numpy().view(np.complex128)

    # ---- matvec phases and roofline (one timed matvec)
    y = torch.empty_like(b)
    _lib.check(lib.sie_matvec_device(g._h, C.c_void_p(b.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0,
                                     C.c_void_p(stream.cuda_stream)))
    for _ in range(3):
        _lib.check(lib.sie_matvec_device(g._h, C.c_void_p(b.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    tm = g.timings()
    Q = 2 * 19 * 19 + 2
    peak, peak_kind = peaks()
    # The product above runs the near panels on a second stream beside the translations,
    # so its per-phase events overlap. Each phase's own duration comes from a second
    # context on the same mesh whose product runs the phases one after another.
    os.environ["SIE_OVERLAP"] = "0"
    try:
        gs = Sie(V, T, WL, EPS, tree_s_opt=250, truncation_number=19, device=local).setup()
    finally:
        del os.environ["SIE_OVERLAP"]
    for _ in range(4):
        _lib.check(lib.sie_matvec_device(gs._h, C.c_void_p(b.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    tms = gs.timings()
    gs.close()
    phases = {k: tms[k] for k in ("mv_near_ms", "mv_agg_ms", "mv_ss_ms", "mv_sr_ms", "mv_rr_ms", "mv_recv_ms")}
    phases["serial_total_ms"] = tms["mv_total_ms"]
    mvb = matvec_algorithmic(g, Q)
    mv_ms = tm["mv_total_ms"]
    ach = mvb["total"] / (mv_ms * 1e-3) / 1e9
    # The hot-path unit is one MLFMM matvec (near panels + aggregate + SS + SR + RR +
    # receive), HBM-bound as a whole; the per-phase entries give each kernel's own bound.
    fp64_peak = fp64_dgemm_tflops(dev)
    ph_rows = {
        "near": ("hbm", mvb["near"], phases["mv_near_ms"]),
        "aggregate": ("hbm", mvb["rt"] / 2 + N * 16, phases["mv_agg_ms"]),
        "receive": ("hbm", mvb["rt"] / 2 + 2 * N * 16, phases["mv_recv_ms"]),
        "sr": ("fp64", mvb["sr_flops"], phases["mv_sr_ms"]),
    }
    per_phase = {}
    for k, (bound, units, ms) in ph_rows.items():
        if bound == "hbm":
            a = units / (ms * 1e-3) / 1e9
            per_phase[k] = {"bound": "hbm", "achieved": a, "unit": "GB/s", "frac": a / peak, "ms": ms}
        else:
            a = units / (ms * 1e-3) / 1e12
            per_phase[k] = {"bound": "fp64", "achieved": a, "unit": "TFLOP/s", "peak": fp64_peak,
                            "peak_source": "measured here: torch float64 matmul (cuBLAS DGEMM) 4096^3",
                            "frac": a / fp64_peak if fp64_peak else None, "ms": ms}
    roof = {"kernel": "one MLFMM matvec (all phases)", "bound": "hbm", "achieved": ach, "peak": peak,
            "unit": "GB/s", "frac": ach / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "bytes_per_launch": mvb["total"], "launch_ms": mv_ms, "traffic": committed_traffic(),
            "per_phase": per_phase}
    mv_frac = ach / peak

    # ---- mixed precision against plain FP64 at equal tolerance (rank 0, N = 1)
    mixed = None
    grad = None
    if rank == 0 and world == 1 and not args.no_mixed:
        mixed = mixed_vs_fp64(V, T, args.tol)
        grad = gradient_timing(args.tol)

    # ---- CPU baseline: the oracle on the host cores (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cb = cpu_reference(V, T, mvs, threads)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        res = b_host - g.matvec(x_e2e)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {
                "workload": (f"{args.workload}: rough slab {WORKLOADS[args.workload]['length_wl']} lambda, "
                             f"lambda=632.8nm, eps=-11.7-1.26i (exp(+iwt)), seed=rank, {T.shape[0]} triangles, "
                             f"{g.n_edges} RWG edges, ICTF, ng=3, s_opt=250, K=19, l={g.l_min}..{g.l_max}"),
                "precision": "fp64", "solver": f"GMRES(IMGS) restart {args.restart}, tol {args.tol}",
                "iterations": iters, "matvecs_per_solve": mvs, "converged": bool(conv),
                "backward_error": be, "max_iterations": args.max_iterations, "setup_s": setup_s,
                "near_nnz_blocks": g.near_nnz, "matvec_ms": tm["mv_total_ms"],
                "autotune": {"matvec_ms_before": tune_before, "matvec_ms_after": tune_after, "variants": tune_modes},
                "matvec_phases_ms": phases, "matvec_phases_note": "phases timed one after another; "
                "matvec_ms runs the near panels concurrently with the translations",
                "levels_boxes_i4_pairs": mvb["levels"], "gs_passes_per_arnoldi_step": tm["gm_passes_per_step"],
                "matvec_hbm_frac": mv_frac, "fill_ms": tm["fill_ms"],
                "residual_e2e": float(np.linalg.norm(res) / np.linalg.norm(b_host)),
                "mixed_vs_fp64": mixed, "shape_gradient": grad,
                "l2": "inputs > L2 (near panels and radiation patterns are GBs)",
            },
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": N * 16, "d2h_bytes_per_step": N * 16,
                    "clocks": clk_e2e.summary()},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
