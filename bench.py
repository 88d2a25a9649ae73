#!/usr/bin/env python
"""Benchmark of the reconstruction hot path on B200.

Workload: 2,000,000 oriented points on a torus (R = 1.0, r = 0.35, area-uniform, position
noise 0.002, normals tipped by a 0.05 rad Gaussian, FP32 storage), depth 10 (1.07e9 FEM
nodes), screening weight 4.0, scale 1.1; FP32 multigrid-preconditioned CG with FP64
residual refinement to a relative residual <= 1e-6.  One step = one full reconstruction
(transform, splat, right-hand side, solve, iso value, marching cubes) of that cloud.

  value      points/s with the points already in HBM (pr_ctx_reconstruct_device)
  e2e        points/s through pr_ctx_reconstruct with pinned host input and the mesh copied
             back to host memory
  solve_gbs  algorithmic bytes of the solve / solve time; the FP64 solve of the same system
             is timed beside it (fp64_* keys)
  roofline   the solver kernel with the largest share of the step (the FP32 post-smoothing
             sweep fused with the prolongation and r.z) timed alone with CUDA events on the
             library's stream; the other fine-level solver kernels are reported under "kernels"
  cpu_baseline  the CPU oracle (the crate's schedule restated in C++) at depth 7 on the same
             cloud, extrapolated to depth 10 (x512 nodes): the crate itself needs ~1 TB of
             host RAM at depth 10

Multi-GPU: one process per GPU (torchrun); each rank reconstructs its own cloud (replicas,
weak scaling, no collective on the data path); value = all ranks' points / max rank time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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
CPU_DEPTH = 7


def cpu_sample(pts, depth_target):
    """The crate's schedule (oracle restatement, all host threads) on the full cloud at
    depth 7; per-node work scales with the node count, so the depth-10 time is
    extrapolated by 8^(depth_target - 7)."""
    import oracle
    t0 = time.perf_counter()
    v, t, st, _ = oracle.reconstruct(pts, depth=CPU_DEPTH, point_weight=4.0, solve_mode=0, cg_iters=500,
                                     cg_accuracy=1e-3)
    dt = time.perf_counter() - t0
    scale = 8.0 ** (depth_target - CPU_DEPTH)
    return {"value": len(pts) / (dt * scale), "unit": "points/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": "oracle (C++ FP64 restatement of the crate's cascade schedule) on the full %d-point cloud "
                      "at depth %d: %.2f s measured, extrapolated x%d to depth %d; the crate's own CSR path "
                      "needs ~1 TB host RAM at depth 10" % (len(pts), CPU_DEPTH, dt, int(scale), depth_target),
            "seconds_measured": dt}


def run_reference(a):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from poissonreconstruction_b200 import synthetic
    pts = synthetic.torus(a.points)
    for _ in range(a.warmup):
        cpu_sample(pts[: min(len(pts), 200_000)], a.depth)
    times = []
    last = None
    for _ in range(a.steps):
        last = cpu_sample(pts, a.depth)
        times.append(last["seconds_measured"] * 8.0 ** (a.depth - CPU_DEPTH))
    ms = 1000.0 * statistics.mean(times)
    value = len(pts) / (ms / 1000.0)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "torus_2m_depth%d_degree%d" % (a.depth, a.degree), "points": len(pts),
                      "depth": a.depth, "point_weight": 4.0, "cpu_sample_depth": CPU_DEPTH,
                      "reference_basis": "degree 1: the crate's reconstruct has no degree-2 path"},
           "cpu_baseline": {k: last[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


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
    e2e_ms, e2e_lib, e2e_copy = [], [], []
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
    e2e_ms_max = reduce_max(dist, statistics.mean(e2e_ms), dev)
    e2e_value = total_points / (e2e_ms_max / 1000.0)
    h2d = P * 48
    d2h = int(mesh.vertices.nbytes + mesh.triangles.nbytes)
    mesh = None

    # FP64 comparison arm (same system, same target), warmed up like the mixed arm, in a context of
    # its own: at depth 10 the two arms' buffers do not fit one device together
    ctx.close()
    ctx = prb.Context(local, stream=stream.cuda_stream)
    k64 = a.fp64_steps if a.fp64_steps is not None else a.steps
    device_steps(params64, 1, False)
    ms64, stats64 = device_steps(params64, max(1, k64), True)
    solve64_s = statistics.mean(s.time_solve for s in stats64)
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
        names = ("d2_cheb", "d2_cheb_f", "d2_cheb_pf", "d2_resid", "d2_apply", "d2_restrict", "d2_prolong")
        dom = "d2_cheb"
    else:
        names = ("smooth_prolong_dot", "cg_update_presmooth", "resid_restrict", "spmv_xpby", "spmv")
        dom = "smooth_prolong_dot"
    for nm in names:
        ms, by = ctx.kernel_bench(nm, a.depth, prb.PR_PRECISION_MIXED, a.roofline_reps)
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
        cpu = cpu_sample(pts, a.depth)
        cpu.pop("seconds_measured", None)

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
        other = {"degree": 1, "value": total_points / (reduce_max(dist, statistics.mean(m1), dev) / 1000.0),
                 "unit": "points/s", "ms_per_step": statistics.mean(m1), "solve_ms": 1000.0 * t1,
                 "solve_gbs": s1[-1].solve_bytes / t1 / 1e9 if t1 > 0 else None,
                 "pcg_iterations": s1[-1].pcg_iterations, "rel_residual": s1[-1].rel_residual,
                 "fp64_solve_ms": 1000.0 * t1_64, "mixed_vs_fp64_solve_speedup": t1_64 / t1 if t1 > 0 else None}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 refinement", "data": "synthetic",
            "config": {"workload": "torus_2m_depth%d_degree%d" % (a.depth, a.degree), "points": P,
                       "depth": a.depth, "degree": a.degree, "point_weight": 4.0,
                       "scale": 1.1, "precision": "fp32 pcg + fp64 refinement", "target_rel_residual": 1e-6,
                       "parallelism": "replicas" if ws > 1 else "single", "l2": "flushed between steps (256 MiB)"},
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
            "degree1": other,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms_max, "library_ms": statistics.mean(e2e_lib),
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
    print(json.dumps({"metric": "batched reconstruction throughput", "value": a.batch / (t / 1000.0),
                      "unit": "clouds/s", "points_per_s": total / (t / 1000.0), "ms_per_batch": t,
                      "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "data": "synthetic",
                      "config": {"workload": "batch_%d" % a.batch, "clouds": a.batch, "points": total,
                                 "depths": {str(d): sum(1 for _, dd in clouds if dd == d) for d in (7, 8, 9)},
                                 "point_weight": 4.0, "concurrency": a.concurrency},
                      "triangles": tris, "all_converged": conv}), flush=True)
    return 0


def main():
    a = parse()
    if a.batch:
        return run_batch(a)
    if a.kernel:
        return run_kernel_bench(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
