#!/usr/bin/env python
"""Benchmark of the reconstruction hot path on B200.

Workload (default): 2,000,000 oriented points on a torus (R = 1.0, r = 0.35, area-uniform,
position noise 0.002, normals tipped by a 0.05 rad Gaussian, FP32 storage), depth 10 (1.07e9
FEM nodes), quadratic B-splines (degree 2), screening weight 4.0, scale 1.1; FP32
multigrid-preconditioned CG with FP64 residual refinement to a relative residual <= 1e-6.
One step = one full reconstruction (transform, splat, right-hand side, solve, iso value,
marching cubes) of that cloud.

  value      points/s with the points already in HBM (pr_ctx_reconstruct_device)
  e2e        points/s through pr_ctx_reconstruct with pinned host input and the mesh copied
             back to host memory
  solve_gbs  algorithmic bytes of the solve / solve time; the FP64 solve of the same system
             is timed beside it (fp64_* keys)
  roofline   the kernel with the largest share of the step in the ncu launch list: the FP32
             Chebyshev smoothing step of the degree-2 finest level (k_op3r, mode kOpCheb),
             timed alone with CUDA events on the library's stream; every other finest-level
             pass (CG direction pass, fused first Chebyshev steps, residual, transfers, the
             FP64 refinement step, the plain A x) is under "kernels"
  accuracy   coefficient relative L2 of the mixed and FP64 solutions against each other and
             against an FP64 solve to 1e-10, the largest mixed target meeting 1e-6, and the
             vertex distance between the two meshes over the bbox diagonal (untimed)
  degree1    the same cloud with the crate's basis (linear B-splines): device-resident step,
             mixed and FP64 solves, and its finest-level solver kernels timed alone
  cpu_baseline  measured on the host: iterations of the crate's CG loop (oracle restatement,
             FP64, all host threads) on the same depth-10 degree-2 system, one iteration timed
             per sample and reported as points / (one iteration's time), an upper bound on the
             CPU path's points/s; the crate's own CSR path needs ~1 TB of host RAM at depth 10

--impl reference times the same CPU leg, one CG iteration per step.  --config 1 runs the plain
method instead (100,000 sphere points, depth 8, the crate's cascade with cg_iters 8) end to end
in both arms.

Multi-GPU: one process per GPU (torchrun); each rank reconstructs its own cloud (replicas,
weak scaling, no collective on the data path); value = all ranks' points / max rank time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 1|2]
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "points/s & solve GB/s at depth 10: FP32+refine vs FP64 GPU at ≤1e-6 residual"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--points", type=int, default=2_000_000)
    ap.add_argument("--depth", type=int, default=10)
    ap.add_argument("--degree", type=int, default=2, choices=[1, 2],
                    help="B-spline degree of the headline workload (2: the quadratic basis of the depth-10 "
                         "mixed-precision config; 1: the crate's own basis)")
    ap.add_argument("--no-degree1", action="store_true", help="skip the secondary degree-1 measurement")
    ap.add_argument("--fp64-steps", type=int, default=None, help="steps of the FP64 comparison (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--roofline-reps", type=int, default=20)
    ap.add_argument("--kernel", default=None,
                    help="micro-benchmark one solver kernel at --depth (spmv, spmv_xpby, smooth_first, smooth, "
                         "smooth_prolong_dot, resid_restrict, stencil_per_node, or 'all')")
    ap.add_argument("--fp64", action="store_true", help="--kernel in FP64")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--batch", type=int, default=0,
                    help="instead of the default workload: the batched workload with this many clouds "
                         "(256 = the full batch), timed through pr_reconstruct_batch")
    ap.add_argument("--concurrency", type=int, default=4, help="--batch: contexts (streams) used")
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 5],
                    help="2: the depth-10 mixed-precision workload (default); 1: the plain method (100k sphere "
                         "points, depth 8, the crate's cascade with cg_iters 8), end to end in both arms; 5: the "
                         "large workload (20M points, union of 32 spheres + 1%% outliers, adaptive depth 12)")
    ap.add_argument("--large-points", type=int, default=20_000_000, help="--config 5: cloud size")
    ap.add_argument("--large-depth", type=int, default=12, help="--config 5: band depth")
    ap.add_argument("--large-coarse", type=int, default=9, help="--config 5: coarse (dense) depth")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the coefficient / vertex error block")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint workload's timing")
    ap.add_argument("--only-device", action="store_true",
                    help="warm-up + timed device-resident steps only (for profiler launch lists)")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, backend):
    import datetime

    import torch.distributed as dist
    if ws > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return dist if ws > 1 else None


def reduce_max(dist, value, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Each rank reconstructs its own cloud of the same workload (replicas, weak scaling)."""
    from poissonreconstruction_b200 import synthetic
    return synthetic.SEED_BASE + 2 + 1000 * rank


def reduce_sum(dist, value, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline (oracle)
def _host_gb():
    try:
        import psutil
        return psutil.virtual_memory().available / 1e9
    except ImportError:
        return float("inf")


class CpuCG:
    """The CPU leg: the crate's CG loop (solve_cg, src/solvers.rs:20-69), FP64, all host threads,
    on the oracle's matrix-free operator of this cloud's system (degree 2: stiffness of the quadratic
    basis + screening of every point; degree 1: the crate's own assemble_system entries), from
    x = 0 with a seeded random right-hand side (an iteration costs the same for any b).  One
    step() = one CG iteration over the full grid, timed with the host clock.  The depth is the
    benchmark's unless the host lacks the memory (about 6.5 vectors of 8^depth doubles)."""

    def __init__(self, pts, depth, degree, pw=4.0):
        import oracle
        self.depth = depth
        need = 7.0 * 8.0 ** depth * 8 / 1e9
        while depth > 6 and _host_gb() < need + 4.0:
            depth -= 1
            need /= 8.0
        self.run_depth = depth
        self.degree = degree
        unit, _ = oracle.to_unit(pts)
        t0 = time.perf_counter()
        if degree == 2:
            self.tree = oracle.Tree2(depth, unit, pw)
            self.tree.release_field()
            b = np.random.default_rng(20260102).standard_normal(8 ** depth)
            self.cg = oracle.CG2(self.tree, b)
        else:
            self.tree = oracle.Tree(depth, unit)
            self.tree.release_field()
            b = np.random.default_rng(20260102).standard_normal(8 ** depth)
            self.cg = oracle.CG1(self.tree, b, pw)
        del b
        self.setup_s = time.perf_counter() - t0
        self.points = len(pts)
        self.cores = oracle.num_threads()

    def step(self):
        t0 = time.perf_counter()
        self.cg.step()
        return time.perf_counter() - t0

    def describe(self, seconds):
        n = 8 ** self.run_depth
        # bytes one iteration of the crate's loop moves: A d (read d, write q), d.q, x += a d,
        # r -= a q, r.r, d = r + b d, in FP64
        gb = 14.0 * n * 8 / 1e9
        sample = ("one iteration of the crate's CG loop (solve_cg, src/solvers.rs:20-69) per step, FP64, %d host "
                  "threads, on the oracle's matrix-free degree-%d operator of this %d-point cloud at depth %d "
                  "(%d unknowns, screening of every point), from x = 0 with a seeded random right-hand side; "
                  "value = points / time of ONE iteration, an upper bound on the CPU path's points/s (a "
                  "reconstruction adds setup, many iterations and extraction); %.1f s untimed setup"
                  % (self.cores, self.degree, self.points, self.run_depth, n, self.setup_s))
        if self.run_depth != self.depth:
            sample += "; depth %d instead of %d: not enough free host memory" % (self.run_depth, self.depth)
        return {"value": self.points / seconds, "unit": "points/s", "cores": self.cores, "kind": "port",
                "sample": sample, "seconds_per_iteration": seconds, "cg_iteration_gbs": gb / seconds}


def run_reference(a):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from poissonreconstruction_b200 import synthetic
    if a.config == 1:
        return run_reference_plain(a)
    if a.config == 5:
        print(json.dumps({"impl": "reference", "unavailable": "depth 12 has no CPU path: the crate's dense grid would "
                          "hold 6.9e10 nodes (its CSR several TB of host memory); compared against the FP64 GPU "
                          "solve of the same band system instead"}), flush=True)
        return 0
    pts = synthetic.torus(a.points)
    cpu = CpuCG(pts, a.depth, a.degree)
    for _ in range(a.warmup):
        cpu.step()
    times = [cpu.step() for _ in range(a.steps)]
    sec = statistics.mean(times)
    d = cpu.describe(sec)
    value = d["value"]
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 * sec, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(a, len(pts)),
           "solve_gbs": d["cg_iteration_gbs"],
           "cpu_baseline": {k: d[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------ plain-method workload (both arms)
PLAIN = {"points": 100_000, "depth": 8, "point_weight": 4.0, "cg_iters": 8, "cg_accuracy": 1e-3}


def plain_config():
    return {"workload": "sphere_100k_depth8_reference_schedule", "points": PLAIN["points"], "depth": PLAIN["depth"],
            "degree": 1, "point_weight": PLAIN["point_weight"], "scale": 1.1,
            "solve": "the crate's cascade: GS(20) + CG(cg_iters=8) at depth 6, prolongation, GS(20) + CG(2)",
            "parallelism": "single"}


def run_reference_plain(a):
    """The crate's reconstruct (the oracle's restatement: CSR assembly, cascade with sequential
    Gauss-Seidel, serial marching cubes) on the plain-method cloud, end to end per step."""
    import oracle
    from poissonreconstruction_b200 import synthetic
    pts = synthetic.sphere(PLAIN["points"])
    kw = dict(depth=PLAIN["depth"], point_weight=PLAIN["point_weight"], solve_mode=0, cg_iters=PLAIN["cg_iters"],
              cg_accuracy=PLAIN["cg_accuracy"])
    for _ in range(a.warmup):
        oracle.reconstruct(pts, **kw)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        oracle.reconstruct(pts, **kw)
        times.append(time.perf_counter() - t0)
    sec = statistics.mean(times)
    value = len(pts) / sec
    cpu = {"value": value, "unit": "points/s", "cores": oracle.num_threads(), "kind": "port",
           "sample": "the whole reconstruction per step (the oracle's restatement of the crate's path, FP64, %d "
                     "host threads where the crate uses rayon)" % oracle.num_threads()}
    print(json.dumps({"impl": "reference", "metric": "plain-method reconstruction throughput", "value": value,
                      "unit": "points/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                      "ms_per_step": 1000.0 * sec, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic", "config": plain_config(), "cpu_baseline": cpu,
                      "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)
    return 0


def run_ours_plain(a):
    """The plain-method workload on the GPU through the public call (pinned host points in, mesh
    back in host memory), with the crate's own cascade (PR_SOLVE_REFERENCE_SCHEDULE)."""
    import torch

    import poissonreconstruction_b200 as prb
    from poissonreconstruction_b200 import synthetic
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = prb.Context(local, stream=stream.cuda_stream)
    pts = synthetic.sphere(PLAIN["points"])
    h_pts = torch.from_numpy(pts).pin_memory()
    d_pts = torch.from_numpy(pts).to(dev)
    params = prb.ReconstructParams(depth=PLAIN["depth"], point_weight=PLAIN["point_weight"],
                                   solve_mode=prb.PR_SOLVE_REFERENCE_SCHEDULE, cg_iters=PLAIN["cg_iters"],
                                   cg_accuracy=PLAIN["cg_accuracy"])
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(a.warmup):
        ctx.reconstruct(h_pts.numpy(), params)
    ev = []
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            ctx.reconstruct_device(d_pts.data_ptr(), len(pts), params)
            e.record(stream)
            ev.append((s, e))
        torch.cuda.synchronize(dev)
    ms = statistics.mean(s.elapsed_time(e) for s, e in ev)
    e2e = []
    mesh = None
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        mesh = None
        t0 = time.perf_counter()
        mesh, st = ctx.reconstruct(h_pts.numpy(), params)
        e2e.append(1000.0 * (time.perf_counter() - t0))
    e2e_ms = statistics.mean(e2e)
    d2h = int(mesh.vertices.nbytes + mesh.triangles.nbytes)
    ctx.close()
    print(json.dumps({"metric": "plain-method reconstruction throughput", "value": len(pts) / (ms / 1000.0),
                      "unit": "points/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": dict(plain_config(), l2="flushed between steps (256 MiB)"),
                      "e2e": {"value": len(pts) / (e2e_ms / 1000.0), "unit": "points/s",
                              "h2d_bytes_per_step": len(pts) * 48, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
                      "mesh": {"vertices": int(st.mesh_vertices), "triangles": int(st.mesh_triangles)},
                      "clocks": clocks.summary()}), flush=True)
    return 0


def run_ours_large(a):
    """The large workload: 20,000,000 points on the union of 32 spheres plus 1% outliers, adaptive
    (narrow-band) reconstruction at depth 12 over a dense depth-9 level, degree 2, FP32 + FP64
    refinement to 1e-6, against the FP64 solve of the same band system."""
    import torch

    import poissonreconstruction_b200 as prb
    from poissonreconstruction_b200 import synthetic
    from scipy.spatial import cKDTree
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = prb.Context(local, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    pts = synthetic.union_of_spheres(a.large_points)
    gen_s = time.perf_counter() - t0
    P = len(pts)
    d_pts = torch.from_numpy(pts).to(dev)
    h_pts = torch.from_numpy(pts).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    params = prb.ReconstructParams(depth=a.large_depth, coarse_depth=a.large_coarse, degree=2, point_weight=4.0,
                                   scale=1.1, precision=prb.PR_PRECISION_MIXED, target_rel_residual=1e-6)
    params64 = dataclasses_replace(params, precision=prb.PR_PRECISION_FP64)

    def steps(par, k):
        ms, sts = [], []
        for _ in range(k):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            st = ctx.reconstruct_device(d_pts.data_ptr(), P, par)
            e.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(s.elapsed_time(e))
            sts.append(st)
        return ms, sts

    steps(params, max(1, a.warmup))
    with ClockSampler(local) as clocks:
        ms, sts = steps(params, a.steps)
    st = sts[-1]
    if a.only_device:
        print(json.dumps({"ms_per_step": statistics.mean(ms), "stage_ms": {
            "transform": 1000 * st.time_transform, "setup": 1000 * st.time_tree, "solve": 1000 * st.time_solve,
            "extract": 1000 * st.time_extract}, "pcg_iterations": st.pcg_iterations,
            "refinement_steps": st.refinement_steps, "rel_residual": st.rel_residual}), flush=True)
        ctx.close()
        return 0
    f32 = ctx.band_vector(1)
    v32 = ctx.mesh().vertices
    e2e = []
    for _ in range(a.steps):
        mesh = None
        t1 = time.perf_counter()
        mesh, _ = ctx.reconstruct(h_pts.numpy(), params)
        e2e.append(1000.0 * (time.perf_counter() - t1))
    d2h = int(mesh.vertices.nbytes + mesh.triangles.nbytes)
    mesh = None
    ms64, sts64 = steps(params64, 1)
    f64 = ctx.band_vector(1)
    v64 = ctx.mesh().vertices
    _, _, codes = ctx.band_info()
    # the adjoint pass: mean chi^2 at 1,000,000 other samples of the same surface, gradients w.r.t.
    # every point; FP64 on the FP64 state (untimed reference), then timed on the mixed state
    adjoint = None
    if not a.no_adjoint:
        q = synthetic.union_of_spheres(1_000_000, outlier_frac=0.0, sample_seed=synthetic.SEED_BASE + 55)[:, :3]
        _, dp64, dn64, ast64 = ctx.loss_backward(q, n_points=P)
        ctx.solve(pts, params)
        ctx.loss_backward(q, n_points=P)  # warm-up
        t1 = time.perf_counter()
        _, dp, dn, ast = ctx.loss_backward(q, n_points=P)
        bw_ms = 1000.0 * (time.perf_counter() - t1)

        def rel(u, v):
            return float(np.linalg.norm(u - v) / np.linalg.norm(v))
        adjoint = {"queries": len(q), "loss": ast.loss, "backward_ms": bw_ms,
                   "adjoint_solve_ms": 1000.0 * ast.time_solve, "pcg_iterations": ast.pcg_iterations,
                   "refinement_steps": ast.refinement_steps, "rel_residual": ast.rel_residual,
                   "converged": ast.converged, "queries_off_band": ast.queries_off_band,
                   "grad_rel_l2_mixed_vs_fp64": {"positions": rel(dp, dp64), "normals": rel(dn, dn64)},
                   "fp64_backward_converged": ast64.converged}
        dp = dn = dp64 = dn64 = None
    coef_err = float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64))
    diag = float(np.linalg.norm(pts[:, :3].max(0) - pts[:, :3].min(0)))
    if len(v32) == len(v64):  # same cut edges: vertex i is the same grid edge in both meshes
        dv = np.linalg.norm(v32 - v64, axis=1)
        verr = {"max_over_bbox_diag": float(dv.max() / diag), "matched": "by grid edge"}
    else:
        sample = np.random.default_rng(0).choice(len(v32), min(len(v32), 2_000_000), replace=False)
        dv, _ = cKDTree(v64).query(v32[sample])
        verr = {"max_over_bbox_diag": float(dv.max() / diag),
                "p999_over_bbox_diag": float(np.quantile(dv, 0.999) / diag),
                "matched": "nearest FP64 vertex, 2M-vertex sample"}
    ms_mean = statistics.mean(ms)
    print(json.dumps({
        "metric": "large-workload reconstruction throughput (adaptive depth 12)", "value": P / (ms_mean / 1000.0),
        "unit": "points/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_mean,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 refinement",
        "data": "synthetic",
        "config": {"workload": "union32_spheres_%dm_depth%d_adaptive" % (round(P / 1e6), a.large_depth), "points": P,
                   "depth": a.large_depth, "coarse_depth": a.large_coarse,
                   "degree": 2, "point_weight": 4.0, "scale": 1.1, "target_rel_residual": 1e-6,
                   "l2": "flushed between steps (256 MiB)"},
        "bricks": int(len(codes)), "band_nodes": int(512 * len(codes)),
        "stage_ms": {"transform": 1000 * st.time_transform, "coarse_setup_and_band_setup": 1000 * st.time_tree,
                     "solve_coarse_and_band": 1000 * st.time_solve, "extract": 1000 * st.time_extract},
        "solve_gbs": st.solve_bytes / st.time_solve / 1e9 if st.time_solve > 0 else None,
        "pcg_iterations": st.pcg_iterations, "refinement_steps": st.refinement_steps, "rel_residual": st.rel_residual,
        "fp64_ms_per_step": ms64[0], "fp64_solve_ms": 1000 * sts64[0].time_solve,
        "fp64_rel_residual": sts64[0].rel_residual,
        "accuracy": {"coef_rel_l2_mixed_vs_fp64": coef_err, "vertex_err_mixed_vs_fp64": verr,
                     "vertices": [int(len(v32)), int(len(v64))]},
        "mesh": {"vertices": int(st.mesh_vertices), "triangles": int(st.mesh_triangles), "iso": st.iso_value},
        "peak_device_gb": st.peak_device_bytes / 1e9,
        "e2e": {"value": P / (statistics.mean(e2e) / 1000.0), "unit": "points/s", "h2d_bytes_per_step": P * 48,
                "d2h_bytes_per_step": d2h, "ms_per_step": statistics.mean(e2e)},
        "adjoint": adjoint, "clocks": clocks.summary(), "generator_s": gen_s}), flush=True)
    ctx.close()
    return 0


def dataclasses_replace(obj, **kw):
    import dataclasses
    return dataclasses.replace(obj, **kw)


def workload_config(a, points):
    return {"workload": "torus_2m_depth%d_degree%d" % (a.depth, a.degree), "points": points,
            "depth": a.depth, "degree": a.degree, "point_weight": 4.0,
            "scale": 1.1, "precision": "fp32 pcg + fp64 refinement", "target_rel_residual": 1e-6,
            "parallelism": "replicas" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else "single",
            "l2": "flushed between steps (256 MiB)"}


# ------------------------------------------------------------------ our arm
def run_ours(a):
    import torch

    import poissonreconstruction_b200 as prb
    from poissonreconstruction_b200 import synthetic

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = dist_init(ws, "nccl")
    # the library runs on this (non-default) stream, so CUDA events recorded on it time its kernels
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = prb.Context(local, stream=stream.cuda_stream)

    pts = synthetic.torus(a.points, seed=replica_seed(rank))
    P = len(pts)
    d_pts = torch.from_numpy(pts).to(dev)
    h_pts = torch.from_numpy(pts).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    params = prb.ReconstructParams(depth=a.depth, point_weight=4.0, scale=1.1, degree=a.degree,
                                   precision=prb.PR_PRECISION_MIXED, target_rel_residual=1e-6)
    params64 = prb.ReconstructParams(depth=a.depth, point_weight=4.0, scale=1.1, degree=a.degree,
                                     precision=prb.PR_PRECISION_FP64, target_rel_residual=1e-6)

    def device_steps(par, k, record):
        ev = []
        stats = []
        for _ in range(k):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            st = ctx.reconstruct_device(d_pts.data_ptr(), P, par)
            e.record(stream)
            ev.append((s, e))
            stats.append(st)
        torch.cuda.synchronize(dev)
        return [s.elapsed_time(e) for s, e in ev], stats

    # warm-up
    device_steps(params, a.warmup, False)

    # timed region: device-resident input
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    l0, p0 = prb.kernel_launches()
    with ClockSampler(local) as clocks:
        ms_list, stats = device_steps(params, a.steps, True)
    l1, p1 = prb.kernel_launches()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    if a.only_device:
        if rank == 0:
            st = stats[-1]
            print(json.dumps({"ms_per_step": statistics.mean(ms_list), "solve_ms": 1000 * st.time_solve,
                              "pcg_iterations": st.pcg_iterations, "refinement_steps": st.refinement_steps,
                              "rel_residual": st.rel_residual, "launches_per_step": (l1 - l0) / max(1, a.steps)}))
        ctx.close()
        return 0
    ms_mean = statistics.mean(ms_list)
    ms_max = reduce_max(dist, ms_mean, dev)
    total_points = reduce_sum(dist, float(P), dev)
    value = total_points / (ms_max / 1000.0)
    st = stats[-1]
    solve_s = statistics.mean(s.time_solve for s in stats)
    solve_gbs = st.solve_bytes / solve_s / 1e9 if solve_s > 0 else None


    # e2e: host (pinned) input, mesh copied back, through the public call
    e2e_ms, e2e_lib, e2e_copy, e2e_stages = [], [], [], []
    mesh = None
    for _ in range(a.warmup):  # untimed: the first calls pin the host blocks the mesh lands in
        mesh, _ = ctx.reconstruct(h_pts.numpy(), params)
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        mesh = None  # free the previous mesh outside the timed region
        t0 = time.perf_counter()
        mesh, st_e = ctx.reconstruct(h_pts.numpy(), params)
        e2e_ms.append(1000.0 * (time.perf_counter() - t0))
        e2e_lib.append(1000.0 * st_e.time_total)
        e2e_stage = {"transform_incl_h2d": st_e.time_transform, "tree_splat_rhs": st_e.time_tree,
                     "solve": st_e.time_solve, "extract": st_e.time_extract, "mesh_copy": st_e.time_mesh_copy}
        e2e_copy.append(1000.0 * st_e.time_mesh_copy)
        e2e_stages.append({k: round(1000.0 * v, 2) for k, v in e2e_stage.items()})
    e2e_ms_max = reduce_max(dist, statistics.mean(e2e_ms), dev)
    e2e_value = total_points / (e2e_ms_max / 1000.0)
    h2d = P * 48
    d2h = int(mesh.vertices.nbytes + mesh.triangles.nbytes)
    mesh = None

    # FP64 comparison arm (same system, same target), warmed up like the mixed arm, in a context of
    # its own: at depth 10 the two arms' buffers do not fit one device together
    # accuracy (untimed): the mixed solution and mesh of the timed configuration
    acc = None
    if not a.no_accuracy and rank == 0:
        ctx.reconstruct_device(d_pts.data_ptr(), P, params)
        acc = {"x_mixed": ctx.coefficients(), "v_mixed": ctx.mesh().vertices}
    ctx.close()
    ctx = prb.Context(local, stream=stream.cuda_stream)
    k64 = a.fp64_steps if a.fp64_steps is not None else a.steps
    device_steps(params64, 1, False)
    ms64, stats64 = device_steps(params64, max(1, k64), True)
    solve64_s = statistics.mean(s.time_solve for s in stats64)
    accuracy = None
    if acc is not None:
        acc["x_fp64"] = ctx.coefficients()
        acc["v_fp64"] = ctx.mesh().vertices
        ctx, accuracy = accuracy_block(ctx, lambda: prb.Context(local, stream=stream.cuda_stream), d_pts, P, pts, a,
                                       acc)
    acc = None
    ctx.close()
    ctx = prb.Context(local, stream=stream.cuda_stream)

    # roofline: every fine-level solver kernel timed alone with CUDA events on the library's
    # stream; the roofline entry is the kernel with the largest share of the step's kernel time in
    # the ncu launch list of this workload (degree 2: the Chebyshev smoothing step, three launches
    # per V-cycle; degree 1: the post-smoothing sweep fused with the prolongation and the r.z
    # product)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    kernels = {}
    if a.degree == 2:
        # every finest-level pass of the degree-2 solve (FP32 unless marked), the FP64 refinement
        # step, and the plain A x (the SpMV alone)
        names = ("d2_cheb", "d2_cg_dir", "d2_cheb_f", "d2_cheb_pf", "d2_resid", "d2_restrict", "d2_prolong",
                 "d2_refine:f64", "d2_apply")
        dom = "d2_cheb"
    else:
        names = ("smooth_prolong_dot", "cg_update_presmooth", "resid_restrict", "spmv_xpby", "spmv")
        dom = "smooth_prolong_dot"
    for nm in names:
        kn, _, prec = nm.partition(":")
        ms, by = ctx.kernel_bench(kn, a.depth, prb.PR_PRECISION_FP64 if prec == "f64" else prb.PR_PRECISION_MIXED,
                                  a.roofline_reps)
        kernels[nm] = {"ms_per_launch": ms, "algorithmic_bytes": by, "achieved_gbs": by / (ms / 1000.0) / 1e9,
                       "frac": by / (ms / 1000.0) / 1e9 / peak}
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = tr.get("%s_f32_depth%d_bytes_per_launch" % (dom, a.depth))
    except (OSError, ValueError):
        pass
    achieved = kernels[dom]["achieved_gbs"]

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        leg = CpuCG(pts, a.depth, a.degree)
        leg.step()  # warm-up iteration
        d = leg.describe(statistics.mean(leg.step() for _ in range(3)))
        cpu = {k: d[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu["cg_iteration_gbs"] = d["cg_iteration_gbs"]
        leg = None

    # the other basis on the same cloud (device-resident steps, mixed and FP64), in a fresh context
    # once the headline context has released its buffers
    other = None
    if not a.no_degree1 and a.degree == 2:
        ctx.close()
        ctx = prb.Context(local, stream=stream.cuda_stream)
        q1 = prb.ReconstructParams(depth=a.depth, point_weight=4.0, scale=1.1, degree=1,
                                   precision=prb.PR_PRECISION_MIXED, target_rel_residual=1e-6)
        q1_64 = prb.ReconstructParams(depth=a.depth, point_weight=4.0, scale=1.1, degree=1,
                                      precision=prb.PR_PRECISION_FP64, target_rel_residual=1e-6)
        device_steps(q1, 1, False)
        m1, s1 = device_steps(q1, a.steps, True)
        m1_64, s1_64 = device_steps(q1_64, max(1, k64), True)
        t1 = statistics.mean(x.time_solve for x in s1)
        t1_64 = statistics.mean(x.time_solve for x in s1_64)
        # the degree-1 finest-level solver kernels, each timed alone as above (FP32)
        k1 = {}
        for nm in ("smooth_prolong_dot", "cg_update_presmooth", "resid_restrict", "spmv_xpby", "spmv"):
            ms, by = ctx.kernel_bench(nm, a.depth, prb.PR_PRECISION_MIXED, a.roofline_reps)
            k1[nm] = {"ms_per_launch": ms, "algorithmic_bytes": by, "achieved_gbs": by / (ms / 1000.0) / 1e9,
                      "frac": by / (ms / 1000.0) / 1e9 / peak}
        other = {"degree": 1, "value": total_points / (reduce_max(dist, statistics.mean(m1), dev) / 1000.0),
                 "unit": "points/s", "ms_per_step": statistics.mean(m1), "solve_ms": 1000.0 * t1,
                 "solve_gbs": s1[-1].solve_bytes / t1 / 1e9 if t1 > 0 else None,
                 "pcg_iterations": s1[-1].pcg_iterations, "rel_residual": s1[-1].rel_residual,
                 "fp64_solve_ms": 1000.0 * t1_64, "mixed_vs_fp64_solve_speedup": t1_64 / t1 if t1 > 0 else None,
                 "kernels": k1}

    # the adjoint workload (1,000,000 superquadric points, depth 9, loss = mean chi^2 at 200,000
    # surface points): forward solve and backward pass timed on the host clock (mixed precision,
    # 1e-6), untimed warm-up first
    adjoint = None
    if rank == 0 and not a.no_adjoint:
        ctx.close()
        ctx = prb.Context(local, stream=stream.cuda_stream)
        apts = synthetic.superquadric(1_000_000)
        aq = synthetic.superquadric_queries(200_000)
        ap = prb.ReconstructParams(depth=9, point_weight=4.0, scale=1.1, precision=prb.PR_PRECISION_MIXED,
                                   target_rel_residual=1e-6)
        fw, bw, ast = [], [], None
        for k in range(4):
            t0 = time.perf_counter()
            ctx.solve(apts, ap)
            t1 = time.perf_counter()
            _, _, _, ast = ctx.loss_backward(aq)
            t2 = time.perf_counter()
            if k > 0:
                fw.append(1000.0 * (t1 - t0))
                bw.append(1000.0 * (t2 - t1))
        adjoint = {"workload": "superquadric_1m_depth9_200k_queries", "forward_ms": statistics.mean(fw),
                   "backward_ms": statistics.mean(bw), "adjoint_solve_ms": 1000.0 * ast.time_solve,
                   "adjoint_rel_residual": ast.rel_residual, "adjoint_pcg_iterations": ast.pcg_iterations,
                   "points_per_s_forward_plus_backward": len(apts) / ((statistics.mean(fw) + statistics.mean(bw))
                                                                      / 1000.0),
                   "note": "host clock, points and queries from host memory, gradients copied back"}
        apts = aq = None

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 refinement", "data": "synthetic",
            "config": workload_config(a, P),
            "solve_gbs": solve_gbs, "solve_ms": 1000.0 * solve_s, "rel_residual": st.rel_residual,
            "pcg_iterations": st.pcg_iterations, "refinement_steps": st.refinement_steps,
            "fp64_solve_ms": 1000.0 * solve64_s, "fp64_ms_per_step": statistics.mean(ms64),
            "fp64_rel_residual": stats64[-1].rel_residual, "fp64_pcg_iterations": stats64[-1].pcg_iterations,
            "mixed_vs_fp64_solve_speedup": solve64_s / solve_s if solve_s > 0 else None,
            "stage_ms": {"transform": 1000 * st.time_transform, "tree_splat_rhs": 1000 * st.time_tree,
                         "solve": 1000 * st.time_solve, "extract": 1000 * st.time_extract},
            "mesh": {"vertices": int(st.mesh_vertices), "triangles": int(st.mesh_triangles),
                     "iso": st.iso_value},
            "peak_device_gb": st.peak_device_bytes / 1e9,
            "roofline": {"kernel": "%s (fp32, depth %d)" % (dom, a.depth), "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                         "traffic": traffic, "algorithmic_bytes": kernels[dom]["algorithmic_bytes"],
                         "ms_per_launch": kernels[dom]["ms_per_launch"]},
            "kernels": kernels,
            "accuracy": accuracy,
            "adjoint": adjoint,
            "degree1": other,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms_max, "steps_ms": e2e_ms, "steps_stage_ms": e2e_stages,
                    "library_ms": statistics.mean(e2e_lib),
                    "mesh_copy_ms": statistics.mean(e2e_copy),
                    "last_step_stage_ms": {k: 1000.0 * v for k, v in e2e_stage.items()}},
            "clocks": clocks.summary(),
            "gpu_launches": int(l1 - l0),
            "gpu_launches_per_step": int((l1 - l0) / max(1, a.steps)),
            "library_primitive_calls": int((p1 - p0) / max(1, a.steps)),
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_kernel_bench(a):
    import poissonreconstruction_b200 as prb
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    names = list(prb.Context.KERNELS) if a.kernel == "all" else [a.kernel]
    prec = prb.PR_PRECISION_FP64 if a.fp64 else prb.PR_PRECISION_MIXED
    with prb.Context(0) as ctx:
        for nm in names:
            ms, by = ctx.kernel_bench(nm, a.depth, prec, a.reps)
            gbs = by / (ms / 1000.0) / 1e9
            print(json.dumps({"kernel": nm, "depth": a.depth, "dtype": "f64" if a.fp64 else "f32",
                              "ms_per_launch": ms, "algorithmic_bytes": by, "achieved_gbs": gbs,
                              "frac_of_measured_peak": gbs / peak if peak else None}), flush=True)
    return 0


def run_batch(a):
    """Batched workload: clouds of 1e4..5e5 points (ellipsoids and tori, depth 7/8/9 by size),
    end to end through pr_reconstruct_batch (host input, meshes back in host memory)."""
    import poissonreconstruction_b200 as prb
    from poissonreconstruction_b200 import synthetic
    clouds = synthetic.batch_clouds(a.batch)
    pts = [c for c, _ in clouds]
    params = [prb.ReconstructParams(depth=d, point_weight=4.0) for _, d in clouds]
    total = sum(len(c) for c in pts)
    for _ in range(a.warmup):
        out = prb.reconstruct_batch(pts, params, concurrency=a.concurrency)
        del out
    ms = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        out = prb.reconstruct_batch(pts, params, concurrency=a.concurrency)
        ms.append(1000.0 * (time.perf_counter() - t0))
        tris = sum(m.triangles.shape[0] for m, _ in out)
        conv = all(st.converged for _, st in out)
        del out
    t = statistics.mean(ms)
    # per-cloud coefficient error of the mixed-precision solve against the FP64 solve (untimed)
    errs = []
    with prb.Context(0) as ctx:
        for c_pts, c_par in zip(pts, params):
            ctx.solve(c_pts, c_par)
            xm = ctx.coefficients()
            ctx.solve(c_pts, prb.ReconstructParams(depth=c_par.depth, point_weight=c_par.point_weight,
                                                   precision=prb.PR_PRECISION_FP64))
            x64 = ctx.coefficients()
            errs.append(float(np.linalg.norm(xm - x64) / np.linalg.norm(x64)))
    print(json.dumps({"metric": "batched reconstruction throughput", "value": a.batch / (t / 1000.0),
                      "unit": "clouds/s", "points_per_s": total / (t / 1000.0), "ms_per_batch": t,
                      "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "data": "synthetic",
                      "config": {"workload": "batch_%d" % a.batch, "clouds": a.batch, "points": total,
                                 "depths": {str(d): sum(1 for _, dd in clouds if dd == d) for d in (7, 8, 9)},
                                 "point_weight": 4.0, "concurrency": a.concurrency},
                      "triangles": tris, "all_converged": conv,
                      "coef_rel_l2_mixed_vs_fp64": {"max": max(errs), "median": statistics.median(errs)},
                      "packing": "clouds of one depth solved together, one launch per solver step for every "
                                 "cloud of a pack (packs sized by free device memory); setup and extraction "
                                 "per cloud on host threads",
                      "autotune": prb.autotune_log().strip().splitlines()}),
          flush=True)
    return 0


def accuracy_block(ctx, new_ctx, d_pts, P, pts, a, acc):
    """Coefficient and vertex error of the timed solves (mixed and FP64 at the 1e-6 target) against
    each other and against an FP64 solve to 1e-10 (untimed), and the largest mixed target residual
    whose coefficients are within 1e-6 of that reference.  ctx is the FP64 arm's context; the mixed
    solves run in a fresh one (at depth 10 the two precisions' buffers do not fit one device
    together).  Returns (the context in use, the block)."""
    import poissonreconstruction_b200 as prb
    from scipy.spatial import cKDTree

    def rel(u, v):
        return float(np.linalg.norm(u - v) / np.linalg.norm(v))

    def solve(prec, tol):
        ctx.reconstruct_device(d_pts.data_ptr(), P, prb.ReconstructParams(
            depth=a.depth, point_weight=4.0, scale=1.1, degree=a.degree, precision=prec, target_rel_residual=tol,
            max_iters=400))
        return ctx.coefficients()

    x_ref = solve(prb.PR_PRECISION_FP64, 1e-10)
    ctx.close()
    ctx = new_ctx()
    out = {"coef_rel_l2_mixed_vs_fp64": rel(acc["x_mixed"], acc["x_fp64"]),
           "coef_rel_l2_mixed_vs_fp64_1e-10": rel(acc["x_mixed"], x_ref),
           "coef_rel_l2_fp64_vs_fp64_1e-10": rel(acc["x_fp64"], x_ref)}
    meets = None
    for tol in (1e-6, 1e-7, 1e-8, 1e-9):
        e = out["coef_rel_l2_mixed_vs_fp64_1e-10"] if tol == 1e-6 else rel(solve(prb.PR_PRECISION_MIXED, tol), x_ref)
        out["coef_rel_l2_mixed_%.0e_vs_fp64_1e-10" % tol] = e
        if e <= 1e-6:
            meets = tol
            break
    out["mixed_target_meeting_1e-6_coefficients"] = meets
    diag = float(np.linalg.norm(pts[:, :3].max(0) - pts[:, :3].min(0)))
    d, _ = cKDTree(acc["v_fp64"]).query(acc["v_mixed"])
    out["vertex_err_mixed_vs_fp64_max_over_bbox_diag"] = float(d.max() / diag)
    out["vertex_err_mixed_vs_fp64_p999_over_bbox_diag"] = float(np.quantile(d, 0.999) / diag)
    out["vertices"] = [int(len(acc["v_mixed"])), int(len(acc["v_fp64"]))]
    return ctx, out


def main():
    a = parse()
    if a.batch:
        return run_batch(a)
    if a.kernel:
        return run_kernel_bench(a)
    if a.impl == "reference":
        return run_reference(a)
    if a.config == 1:
        return run_ours_plain(a)
    if a.config == 5:
        return run_ours_large(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
