"""Benchmark of the SIE hot path on the rough-slab workload of the reference's configuration
(10 lambda x 10 lambda, 19,456 triangles, 29,184 RWG edges, metal eps = -11.7 - 1.26i,
ICTF): converged solves per second.

On this plasmonic slab no iterative solve converges: the MLFMM product is 6.7 % off the
dense one with the reference's K = 19 on every level (1e-5 with per-level truncation
numbers), the system amplifies operator error by >= 7,000, and GMRES, also with the
near-field RAS preconditioner, stalls above 0.4 after 1,000-2,000 steps.  So a converged
solve is a direct one, and one step is one direct solve of one plane wave: the LU
factorisation of the FP64 dense matrix (filled once, as the reference's normal solver
does) and the solution.

`value` is the mixed-precision direct solve (complex64 LU whose trailing updates run on
the tensor cores as 3xTF32 products, FP64 iterative refinement to a backward error of
1e-10) on device-resident buffers; the plain FP64 direct solve (cuSOLVER ZGETRF/ZGETRS,
the reference's ZGESV) is timed beside it, with the far-field error between the two.
`e2e` is the mixed solve through the host-buffer API.  `roofline` is the tensor-core
trailing update, the dominant kernel; `roofline_matvec` keeps the MLFMM product against
HBM.

Multi-GPU (torchrun): every rank solves its own realisation (seed = rank), weak scaling, no
collective on the data path; timings are max-reduced.

`--impl reference` times the reference's own algorithm for this workload (the oracle, a
C++ restatement of it: MLFMM with K = 19 on every level, no preconditioner, zgmres with
restart = max_iterations = 650 as main.f90:226-230 sets) on the host cores; its solve is
650 iterations, which do not reach the tolerance on this slab.
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
    # 1 lambda thick; truncation numbers per MLFMM level (2.5 / 1.25 / 0.625 lambda boxes)
    "slab10": dict(length_wl=10.0, rms_wl=0.5, corr_wl=1.0, thickness_wl=1.0, cells=64, seed=0,
                   level_k={2: 34, 3: 23, 4: 19}, inner_k={2: 26, 3: 17, 4: 12}),
    # a small case for quick checks
    "slab4": dict(length_wl=4.0, rms_wl=0.3, corr_wl=1.0, thickness_wl=1.0, cells=24, seed=0,
                  level_k=None, inner_k={3: 12, 2: 12}),
}
DIRECT = dict(tolerance=1e-10, max_refinements=40)
REFERENCE_ITERATIONS = 650  # main.f90:226-230: max_iterations = restart = 650


def config_of(name, T=None, M=None):
    w = WORKLOADS[name]
    return {
        "workload": (f"{name}: rough slab {w['length_wl']} lambda (seed=rank), lambda=632.8nm, "
                     f"eps=-11.7-1.26i (exp(+iwt)), ICTF, ng=3"
                     + (f", {T} triangles, {M} RWG edges" if T else "")),
        "l2": "inputs > L2 (the dense matrix is tens of GB; the MLFMM tables are GBs)",
    }


SOLVER_OURS = ("direct: dense FP64 fill, complex64 LU with partial pivoting (trailing updates on the tensor "
               "cores, split-FP16 with a 3xTF32 fallback) and FP64 iterative refinement to "
               f"{DIRECT['tolerance']}")


def mesh_edges(T):
    from specklesim_b200 import mesh
    return mesh.edge_count(T)


def host_cpu():
    """nproc and the CPU model of this host."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


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


def matvec_algorithmic(g, level_k, K=19):
    """Algorithmic DRAM bytes of one FP64 matvec, and the FP64 flops of its SR step.
    Bytes: near panels (a, b, d: 48 B per 2x2 block), radiation patterns read by the
    aggregate and the receive (leaf sampling), x in and y out, C and D of every level
    written and read (each level's own sampling), and the coefficients of a level carried
    on its parent's sampling between the interpolation and the shift (SS) or the shift and
    the anterpolation (RR).  The SR source coefficients are read from L2 (each level's C
    fits), so they are not DRAM bytes.  SR flops: 4 complex multiply-adds = 32 real flops
    per (I4 pair, direction, medium); medium 2 only on the leaf level (k2 complex)."""
    M, N, s = g.n_edges, g.n, 16
    st = level_stats(g)
    Kl = {l: (level_k or {}).get(l, K) for l, _, _ in st}
    Ql = {l: 2 * k * k + 2 for l, k in Kl.items()}
    Qleaf = Ql[g.l_max]
    near = g.near_nnz * 3 * s
    rt = 2 * M * 4 * Qleaf * s
    xy = 2 * N * s
    coeff = sum(nb * 8 * Ql[l] * s * 4 for l, nb, _ in st)
    interp = sum(nb * 8 * Ql[l - 1] * s * 4 for l, nb, _ in st if l > g.l_min and Ql[l] != Ql[l - 1])
    sr_flops = sum(ni4 * Ql[l] * 32 * (2 if l == g.l_max else 1) for l, _, ni4 in st)
    return dict(near=near, rt=rt, xy=xy, coeff=coeff + interp, total=near + rt + xy + coeff + interp,
                sr_flops=sr_flops, levels=st, Q=Ql)


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


def hemisphere_grid(n=128, r=5.0):
    """The 128 x 128 (theta, phi) grid over the upper hemisphere at r = 5 m."""
    th = (np.arange(n) + 0.5) * (0.5 * np.pi / n)
    ph = (np.arange(n) + 0.5) * (2 * np.pi / n)
    T, P = np.meshgrid(th, ph, indexing="ij")
    return r * np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=-1).reshape(-1, 3)


def _stats(ts):
    return {"median_s": float(statistics.median(ts)), "min_s": float(min(ts)), "max_s": float(max(ts)),
            "repeats": len(ts)}


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


def cpu_reference(V, T, threads, iters_per_step, steps, warmup, s_opt=250):
    """The reference's algorithm on the host cores: the oracle (C++ restatement, OpenMP)
    set up with K = 19 on every level, and the numpy restatement of zgmres (IMGS, Givens,
    restart = max_iterations) driving the oracle's MLFMM product.  A step runs
    `iters_per_step` Arnoldi steps of that GMRES from x0 = 0 on the plane-wave right-hand
    side (one matvec each); a reference solve is REFERENCE_ITERATIONS of them."""
    from oracle.oracle import Oracle, zgmres
    from specklesim_b200 import incidence
    o = Oracle(V, T, WL, EPS, tree_s_opt=s_opt, threads=threads)
    t0 = time.perf_counter()
    o.tree()
    o.setup_fmm()
    t_setup = time.perf_counter() - t0
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = o.rhs(k, E)
    ts = []
    for i in range(warmup + steps):
        t1 = time.perf_counter()
        zgmres(o.matvec, b, iters_per_step, 1e-30, iters_per_step)
        if i >= warmup:
            ts.append(time.perf_counter() - t1)
    o.close()
    t_step = statistics.median(ts)
    # zgmres ends a budget with the true residual: iters_per_step + 1 products per step
    per_mv = t_step / (iters_per_step + 1)
    per_solve = per_mv * (REFERENCE_ITERATIONS + 1)
    return dict(value=1.0 / per_solve, unit="solves/s", cores=threads, kind="port",
                sample=(f"oracle C++ restatement of the reference (OpenMP, {threads} threads), K = 19 on every "
                        f"level, no preconditioner: set-up {t_setup:.1f} s untimed; each step = {iters_per_step} "
                        f"GMRES steps + the final true residual (numpy zgmres restatement driving the oracle "
                        f"product, {per_mv:.3f} s per product with its Arnoldi step); solves/s = 1 / "
                        f"({REFERENCE_ITERATIONS + 1} products: the reference's max_iterations of {REFERENCE_ITERATIONS} "
                        "and the final residual; its solve does not reach the tolerance on this slab).  The "
                        "orthogonalisation against up to 650 basis vectors of the later steps is not in the "
                        "sample, which favours the CPU"),
                setup_s=t_setup, step_s=t_step, ts=ts)


def mlfmm_matvec(V, T, local, stream, b, peak, peak_kind):
    """The MLFMM product on the same mesh (the reference's operator: s_opt = 250, K = 19
    on every level) against HBM: one product timed with CUDA events after the autotuner
    picked its kernel variants, each phase's own duration from a second context whose
    product runs the phases one after another, and the product with per-level truncation
    numbers for comparison."""
    import ctypes as C
    from specklesim_b200 import Sie, _lib
    lib = _lib.load()
    g = Sie(V, T, WL, EPS, tree_s_opt=250, truncation_number=19, device=local).setup()
    tune_before, tune_after, tune_modes = g.autotune("fp64")
    _lib.check(lib.sie_set_stream(g._h, C.c_void_p(stream.cuda_stream)))
    import torch
    y = torch.empty_like(b)
    for _ in range(4):
        _lib.check(lib.sie_matvec_device(g._h, C.c_void_p(b.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    tm = g.timings()
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
    mvb = matvec_algorithmic(g, None)
    mv_ms = tm["mv_total_ms"]
    ach = mvb["total"] / (mv_ms * 1e-3) / 1e9
    N = g.n
    per_phase = {}
    for k_, (units, ms) in {"near": (mvb["near"], phases["mv_near_ms"]),
                            "aggregate": (mvb["rt"] / 2 + N * 16, phases["mv_agg_ms"]),
                            "receive": (mvb["rt"] / 2 + 2 * N * 16, phases["mv_recv_ms"])}.items():
        a = units / (ms * 1e-3) / 1e9
        per_phase[k_] = {"bound": "hbm", "achieved": a, "unit": "GB/s", "frac": a / peak, "ms": ms}
    a = mvb["sr_flops"] / (phases["mv_sr_ms"] * 1e-3) / 1e12
    per_phase["sr"] = {"bound": "fp64", "achieved": a, "unit": "TFLOP/s", "ms": phases["mv_sr_ms"]}
    g.close()
    # per-level truncation numbers (accurate on the 2.5 lambda boxes)
    kk = WORKLOADS["slab10"]["level_k"]
    gl = Sie(V, T, WL, EPS, tree_s_opt=250, truncation_number=19, device=local, level_truncation=kk).setup()
    _lib.check(lib.sie_set_stream(gl._h, C.c_void_p(stream.cuda_stream)))
    for _ in range(4):
        _lib.check(lib.sie_matvec_device(gl._h, C.c_void_p(b.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    tml = gl.timings()
    mvl = matvec_algorithmic(gl, kk)
    gl.close()
    return {"kernel": "one MLFMM matvec (all phases), K = 19 on every level", "bound": "hbm", "achieved": ach,
            "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)", "bytes_per_launch": mvb["total"],
            "launch_ms": mv_ms, "traffic": committed_traffic(), "per_phase": per_phase, "phases_ms": phases,
            "autotune": {"matvec_ms_before": tune_before, "matvec_ms_after": tune_after, "variants": tune_modes},
            "levels_boxes_i4_pairs": mvb["levels"],
            "level_truncation": {"K": {str(k): v for k, v in kk.items()}, "matvec_ms": tml["mv_total_ms"],
                                 "bytes_per_launch": mvl["total"],
                                 "achieved_gbs": mvl["total"] / (tml["mv_total_ms"] * 1e-3) / 1e9}}


def c3_record(local, stream, peak, s_opt=250):
    """The 30 lambda x 30 lambda slab of the C2 recipe with seed 1 at its stated size (the
    precision configuration's mesh).  On this metal no iterative solve converges (as on
    slab10) and the dense matrix would take N^2 x 16 B, terabytes, so the record is what
    the library does at this size: the set-up, the K = 19 product against HBM, and budgeted
    FP64 GMRES steps (n > 65,536: the Arnoldi step leaves the single-cluster kernel)."""
    import ctypes as C
    import torch
    from specklesim_b200 import Sie, _lib, incidence, mesh
    lib = _lib.load()
    t0 = time.perf_counter()
    V, T = mesh.slab_config(30.0, WL, 0.5, 1.0, 1, thickness_wl=1.0)
    mesh_s = time.perf_counter() - t0
    free0 = torch.cuda.mem_get_info(local)[0]
    t0 = time.perf_counter()
    g = Sie(V, T, WL, EPS, tree_s_opt=s_opt, truncation_number=19, device=local).setup()
    setup_s = time.perf_counter() - t0
    used_gb = (free0 - torch.cuda.mem_get_info(local)[0]) / 1e9
    _lib.check(lib.sie_set_stream(g._h, C.c_void_p(stream.cuda_stream)))
    k, E = incidence(0.0, 0.0, "TM", 2)
    b_host = g.rhs_planewave(k, E)
    with torch.cuda.stream(stream):
        bd = torch.from_numpy(b_host.view(np.float64)).to(f"cuda:{local}")
        yd = torch.empty_like(bd)
    for _ in range(3):
        _lib.check(lib.sie_matvec_device(g._h, C.c_void_p(bd.data_ptr()), C.c_void_p(yd.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        _lib.check(lib.sie_matvec_device(g._h, C.c_void_p(bd.data_ptr()), C.c_void_p(yd.data_ptr()), 1, 0,
                                         C.c_void_p(stream.cuda_stream)))
    e1.record(stream)
    e1.synchronize()
    mv_ms = e0.elapsed_time(e1) / reps
    mvb = matvec_algorithmic(g, None)
    ach = mvb["total"] / (mv_ms * 1e-3) / 1e9
    t0 = time.perf_counter()
    x, st = g.solve(b_host, restart=30, max_iterations=30, tolerance=1e-12, raise_on_noconv=False)
    gm_s = time.perf_counter() - t0
    out = {"workload": "slab30: rough slab 30 lambda, seed 1, RMS 0.5 lambda, corr 1 lambda, 1 lambda thick, "
                       "metal, ICTF, s_opt 250, K = 19",
           "triangles": int(T.shape[0]), "edges": g.n_edges, "unknowns": g.n,
           "levels_boxes_i4_pairs": mvb["levels"], "mesh_s": mesh_s, "setup_s": setup_s,
           "device_gb": used_gb, "near_blocks": g.near_nnz,
           "matvec_ms": mv_ms, "matvec_bytes": mvb["total"], "matvec_gbs": ach, "matvec_frac_hbm": ach / peak,
           "gmres30": {"iterations": st["iterations"], "backward_error": st["backward_error_true"], "seconds": gm_s,
                       "ms_per_iteration": 1e3 * gm_s / max(st["iterations"], 1)}}
    g.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="slab10", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-matvec", action="store_true")
    ap.add_argument("--no-c3", action="store_true", help="skip the 30 lambda record")
    ap.add_argument("--fp64-repeats", type=int, default=3)
    ap.add_argument("--reference-iterations-per-step", type=int, default=2)
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
        cb = cpu_reference(V, T, threads, args.reference_iterations_per_step, args.steps, args.warmup)
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * cb["step_s"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(args.workload, T.shape[0], mesh_edges(T)),
            "solver": "the reference's: MLFMM (K = 19 on every level) + zgmres, restart = max_iterations = 650",
            "step": (f"{args.reference_iterations_per_step} GMRES steps of the reference's MLFMM solver (+ the final "
                     f"residual); value = 1 / ({REFERENCE_ITERATIONS + 1} products)"),
            "cpu_baseline": {**{k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}, "host": host_cpu()},
            "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import ctypes as C
    import torch
    import torch.distributed as dist

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    from specklesim_b200 import Sie, incidence, _lib

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(t):
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    V, T = build_mesh(args.workload, rank)
    dev = torch.device("cuda", local)
    lib = _lib.load()
    stream = torch.cuda.Stream(dev)
    peak_hbm, peak_kind = peaks()

    # ---- dense set-up: the FP64 matrix (every pair through the near-field fill kernels)
    t0 = time.perf_counter()
    d = Sie(V, T, WL, EPS, device=local, dense=True).setup()
    fill_s = time.perf_counter() - t0
    _lib.check(lib.sie_set_stream(d._h, C.c_void_p(stream.cuda_stream)))
    k, E = incidence(0.0, 0.0, "TM", 2)  # x-polarised normal incidence along -z
    b_host = d.rhs_planewave(k, E)
    N = d.n
    with torch.cuda.stream(stream):
        b = torch.from_numpy(b_host.view(np.float64)).to(dev)
        x = torch.zeros_like(b)
    stream.synchronize()
    st = _lib.SieStats()
    steps_info = []

    def mixed_dev():
        _lib.check(lib.sie_invalidate_factors(d._h))  # refactorise every step, into the kept memory
        _lib.check(lib.sie_solve_direct_mixed_device(d._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1,
                                                     DIRECT["tolerance"], DIRECT["max_refinements"], C.byref(st),
                                                     C.c_void_p(stream.cuda_stream)))
        steps_info.append((st.seconds, st.iterations, st.backward_error_true))

    for _ in range(args.warmup):
        mixed_dev()
    steps_info.clear()

    # ---- device-resident timed region: one direct solve (LU + refinement) per step
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = lib.sie_launch_count()
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            mixed_dev()
        e1.record(stream)
        barrier()
    launches = lib.sie_launch_count() - l0
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    value = world * args.steps / t_dev
    tmd = d.timings()
    xm = x.cpu().numpy().view(np.complex128).copy()

    # ---- end to end through the public host API (pinned host buffers), min(K, 3) steps
    ke = min(args.steps, 3)
    bp = torch.from_numpy(b_host.view(np.float64).copy()).pin_memory()
    xp = torch.zeros_like(bp).pin_memory()
    stats = (_lib.SieStats * 1)()
    dp = C.POINTER(C.c_double)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk_e2e:
        e2.record(stream)
        for _ in range(ke):
            _lib.check(lib.sie_invalidate_factors(d._h))
            _lib.check(lib.sie_solve_direct_mixed(d._h, C.cast(bp.data_ptr(), dp), C.cast(xp.data_ptr(), dp), 1,
                                                  DIRECT["tolerance"], DIRECT["max_refinements"], stats))
        e3.record(stream)
        barrier()
    t_e2e = max_over_ranks(e2.elapsed_time(e3) / 1000.0)
    e2e = world * ke / t_e2e

    # ---- the plain FP64 direct solve (cuSOLVER ZGETRF + ZGETRS) beside it, and the
    # far-field error between the two on the 128 x 128 hemisphere grid (rank 0)
    fp64 = None
    if rank == 0:
        t64 = []
        x64 = None
        _lib.check(lib.sie_release_factors(d._h))  # the complex64 factors' memory back
        for _ in range(args.fp64_repeats):
            _lib.check(lib.sie_invalidate_factors(d._h))
            t1 = time.perf_counter()
            x64 = d.solve_direct(b_host)
            t64.append(time.perf_counter() - t1)
        _lib.check(lib.sie_release_factors(d._h))
        pts = hemisphere_grid()
        I64 = d.farfield(x64, pts)[2]
        Im = d.farfield(xm, pts)[2]
        r64 = float(np.linalg.norm(d.matvec(x64) - b_host) / np.linalg.norm(b_host))
        tmed = [s_ for s_, _, _ in steps_info]
        fp64 = {
            "fp64": {"solves_per_s": 1.0 / statistics.median(t64), **_stats(t64), "backward_error": r64,
                     "solver": "cuSOLVER ZGETRF + ZGETRS (host buffers), refactorised every solve into kept memory "
                               "(the first repeat allocates it)"},
            "mixed": {"solves_per_s": 1.0 / statistics.median(tmed), **_stats(tmed),
                      "refinement_steps": [i for _, i, _ in steps_info][-1],
                      "backward_error": max(be for _, _, be in steps_info)},
            "speedup_vs_fp64": statistics.median(t64) / statistics.median(tmed),
            "mixed_breakdown_s": {"lu_factor": tmd["lu_factor_ms"] / 1e3, "lu_trailing_updates": tmd["lu_gemm_ms"] / 1e3,
                                  "expand_refine_and_rest": statistics.median(tmed) - tmd["lu_factor_ms"] / 1e3},
            "farfield_rel_err_vs_fp64": float(np.linalg.norm(Im - I64) / np.linalg.norm(I64)),
            "currents_rel_err_vs_fp64": float(np.linalg.norm(xm - x64) / np.linalg.norm(x64)),
            "farfield_points": int(pts.shape[0]),
        }
    d.close()
    torch.cuda.empty_cache()

    # ---- roofline of the dominant kernel: the tensor-core trailing update of the LU.  Both
    # splits run 3 tensor products per real product, 4 real products per complex one: 3 x 8 =
    # 24 tensor flops per complex multiply-add.  Split-FP16 (kind::f16) runs at the dense
    # f16/bf16 rate, 3xTF32 (kind::tf32) at half of it.  The updates run inside a step of
    # seconds under the power cap, so the denominator is the sustained dense rate
    f16 = bool(tmd["lu_f16"])
    try:
        pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        bf = float(pk["bf16_tflops_sustained"])
        peak_t, peak_src = (bf, "measured (MEASURED_PEAKS.json bf16_tflops_sustained, the dense f16 rate over "
                                "seconds under the power cap)") if f16 else \
            (bf / 2, "measured (MEASURED_PEAKS.json bf16_tflops_sustained / 2, the dense tf32 rate)")
    except Exception:
        peak_t, peak_src = (1400.0, "fallback (1.4 PFLOP/s sustained)") if f16 else \
            (700.0, "fallback (1.4 PFLOP/s sustained / 2)")
    g_ms = tmd["lu_gemm_ms"]
    useful = tmd["lu_gemm_flops"]
    tensor_tf = 3 * useful / (g_ms * 1e-3) / 1e12 if g_ms > 0 else None
    roof = {"kernel": ("tc::k_gemm, the LU's trailing update A22 -= L21 U12 " +
                       ("(tcgen05.mma kind::f16, split-FP16 with power-of-two operand scaling)" if f16 else
                        "(tcgen05.mma kind::tf32, 3xTF32)")),
            "bound": "tensor", "achieved": tensor_tf, "peak": peak_t, "unit": "TFLOP/s",
            "frac": tensor_tf / peak_t if tensor_tf else None, "peak_source": peak_src, "traffic": None,
            "launches_per_step": tmd["lu_gemm_launches"], "ms_per_step": g_ms,
            "useful_complex_tflops": useful / (g_ms * 1e-3) / 1e12 if g_ms > 0 else None,
            "lu_factor_ms": tmd["lu_factor_ms"], "factorizations_last_step": tmd["lu_factorizations"]}

    # ---- the MLFMM product against HBM (rank 0, N = 1)
    rmv = None
    if rank == 0 and world == 1 and not args.no_matvec:
        rmv = mlfmm_matvec(V, T, local, stream, b, peak_hbm, peak_kind)
    c3 = None
    if rank == 0 and world == 1 and not args.no_c3:
        c3 = c3_record(local, stream, peak_hbm)

    # ---- CPU baseline: the reference's algorithm on the host cores (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cb = cpu_reference(V, T, threads, 2, 2, 1)
        cpu = {**{k_: cb[k_] for k_ in ("value", "unit", "cores", "kind", "sample")}, "host": host_cpu()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64+f64", "data": "synthetic",
            "config": config_of(args.workload, T.shape[0], N // 2),
            "solver": SOLVER_OURS,
            "details": {"unknowns": N, "fill_s": fill_s, "mixed_vs_fp64": fp64,
                        "step": "one direct solve of one plane wave: LU of the dense matrix (refactorised every "
                                "step into memory kept from the first) and FP64 refinement"},
            "roofline": roof,
            "roofline_matvec": rmv,
            "slab30": c3,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": N * 16, "d2h_bytes_per_step": N * 16,
                    "steps": ke, "clocks": clk_e2e.summary()},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
