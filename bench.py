#!/usr/bin/env python
"""Benchmark of the PFEM remesh-and-solve path on B200.

One step = one remesh of the 4M-point meshing-stress cloud (Karras LBVH with
63-bit Morton codes + 3D alpha shape with exact predicates, free-surface
flags and CSR output), inputs resident in HBM.  The line also carries:
  e2e           the same metric through the public host API (AlphaShape3D_set_nodes
                from pinned host memory ... AlphaShape3D_get_elem into pinned host memory)
  roofline      of the dominant kernel (the star pass): FP32 arithmetic from its
                counted insphere work (AlphaShape3D_get_work) against the FP32
                peak at the sampled SM clock, with its DRAM traffic per launch
                from an ncu capture; "hbm" lists the HBM-bound kernels
                (radix sort at 4M and 64M keys, LBVH and TRBVH stages)
  cpu_baseline  the reference's own sources (oracle/_ref) on the host cores:
                all threads on the 223,766-point corner of the cloud, one thread
                and all threads on the 25k-point meshing-stress cloud
  same_sample   this library on the same 223,766-point corner (a same-input pair)
  remesh3d_uniform  the reference's uniform3D harness clouds (published example
                and the paper's sweep)
  trbvh         TRBVH (treelet 7) over the 4M cloud
  solve         the dam-break pressure solve (FP64 Jacobi-PCG vs mixed precision)
  pfem          the 4M-particle PFEM step loop
  pfem_dynamics the fractional-step dam break (gravity, viscosity, walls), 1M particles
  remesh2d      the 2D alpha shape on the reference's uniform2D 1M cloud
  delaunay2d    the 2D Delaunay mesher (Mesh2D) on a 1M uniform cloud, Qhull beside it
Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one independent replica per GPU (the remesh does not shard here).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "remesh Mpts/s (LBVH + 3D alpha shape), meshing-stress 4M cloud"
UNIT = "Mpts/s"
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes per launch of the star pass on the 4M meshing-stress cloud:
# dram__bytes_read.sum + dram__bytes_write.sum of one k_star launch on the 1M
# cloud of the same composition (1.978 GB, profiles/k_star_1m_stress.md),
# scaled by the number of stars.
K_STAR_DRAM_BYTES_4M = 4 * 1_978_000_000
CPU_ONE_THREAD_POINTS = 25_000   # meshing-stress cloud timed with one host thread


def _workloads():
    """stream_b200/workloads.py loaded by path: pure NumPy, so the reference arm
    never maps this library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_sb_workloads", os.path.join(ROOT, "stream_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(n: int, alpha: float, ws: int) -> dict:
    """The config dict both arms print (the driver compares them)."""
    return {"workload": "meshing-stress cloud: 60% uniform in [0,1]^3, 30% in 32 Gaussian blobs "
                        "(sigma 0.01), 10% distinct 100^3 lattice sites; alpha = 1.5 N^-1/3; "
                        "63-bit Morton LBVH + 3D alpha shape (exact predicates)",
            "points": n, "alpha": alpha, "seed": 0,
            "l2": "256 MiB write between timed steps", "parallelism": f"replicas x{ws}"}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = f"/tmp/sb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, busy_floor_mhz: float = 500.0) -> dict:
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5], p[6], p[7], p[8]))
            except ValueError:
                continue
        os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        busy = [r for r in rows if r[0] >= busy_floor_mhz] or rows
        reasons = set()
        for r in busy:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[2:]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """The largest x over all ranks (the timing rule: the slowest replica
    sets the step time); x itself without a process group."""
    if not dist:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(ws: int, n: int, ms: float) -> float:
    """Whole-job Mpts/s of ws replicas of n points each, at the slowest step time ms."""
    return ws * n / (ms / 1e3) / 1e6


class _QuietStdout:
    """Silence the C-level stdout (the reference prints one line per truncated
    star, DirectAlphaShape3D.cpp:362) while the CPU baseline runs."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def run_cpu_reference(pts, alpha, steps: int, warmup: int, threads: int | None = None):
    """The reference's own sources built for the host (oracle/_ref); falls back
    to the plain-C restatement if absent.  threads: OpenMP threads (default:
    all host threads).  Returns (kind, per-run seconds)."""
    from oracle.oracle import Reference, Restatement
    kind = "reference"
    try:
        ref = Reference()
        fn0 = lambda: ref.ashape3d(pts, alpha)  # noqa: E731
    except FileNotFoundError:
        kind = "port"
        r = Restatement()
        fn0 = lambda: r.ashape3d(pts, alpha)  # noqa: E731
    import ctypes as _ct
    gomp = _ct.CDLL("libgomp.so.1")
    saved = gomp.omp_get_max_threads()
    gomp.omp_set_num_threads(int(threads or os.cpu_count() or 1))

    def fn():
        with _QuietStdout():
            fn0()
    try:
        for _ in range(warmup):
            fn()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
    finally:
        gomp.omp_set_num_threads(saved)
    return kind, ts


def cpu_baselines(wl, pts4, al4, target: int, runs: int = 5):
    """Host-core baselines of the reference path: all threads on the
    corner sample of the cloud (its outputs are pinned bit for bit against
    this library's), and one thread vs all threads on a 25k-point
    meshing-stress cloud.  Median of `runs` after one warm-up each."""
    cores = os.cpu_count() or 1
    sp, sa, frac = wl.sub_cube(pts4, al4, target)
    kind, ts = run_cpu_reference(sp, sa, runs, 1, threads=cores)
    ms = 1e3 * statistics.median(ts)
    p1, a1 = wl.meshing_stress(CPU_ONE_THREAD_POINTS, seed=0)
    _, t1 = run_cpu_reference(p1, a1, runs, 1, threads=1)
    _, tn = run_cpu_reference(p1, a1, runs, 1, threads=cores)
    ms1, msn = 1e3 * statistics.median(t1), 1e3 * statistics.median(tn)
    return {"value": round(len(sp) / (ms / 1e3) / 1e6, 4), "unit": UNIT, "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": f"{len(sp)} points of the 4M cloud (corner box {frac:.3f} of its extent, same alpha), "
                      f"all {cores} host threads, median of {runs} after 1 warm-up: {ms:.0f} ms per run",
            "ms_per_run": round(ms, 1), "points": len(sp),
            "small_cloud": {"workload": f"meshing_stress({CPU_ONE_THREAD_POINTS}, seed=0), alpha = 1.5 N^-1/3",
                            "one_thread_ms": round(ms1, 1), "all_threads_ms": round(msn, 1),
                            "one_thread_mpts_s": round(CPU_ONE_THREAD_POINTS / ms1 / 1e3, 5),
                            "all_threads_mpts_s": round(CPU_ONE_THREAD_POINTS / msn / 1e3, 5),
                            "speedup": round(ms1 / msn, 2), "runs": runs}}


def bench_reference_arm(a):
    """The reference's own CPU path (oracle/_ref) on this arm's config.  The
    reference cannot mesh the whole 4M cloud (it sizes its neighbour table by
    the uncapped neighbour counts, src/mesh/DirectAlphaShape3D.cpp:235-297,
    which for the blob cores overflows its 32-bit offsets), so each step is
    the corner of the cloud that cpu_baseline and same_sample use."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    wl = _workloads()
    pts, alpha = wl.meshing_stress(a.points, seed=a.seed)
    sp, sa, frac = wl.sub_cube(pts, alpha, a.cpu_sample)
    cores = os.cpu_count() or 1
    kind, ts = run_cpu_reference(sp, sa, a.steps, a.warmup, threads=cores)
    ms = 1e3 * statistics.median(ts)
    val = len(sp) / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": UNIT, "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(len(pts), float(alpha[0]), ws),
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
                         "sample": f"each step: the {len(sp)}-point corner of the {a.points}-point cloud (box "
                                   f"{frac:.3f} of its extent, same alpha; the whole cloud overflows the "
                                   f"reference's 32-bit neighbour offsets), all {cores} host threads, median of "
                                   f"{a.steps}"},
        "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line, default=_json_default), flush=True)
    return 0


def bench_ours(a):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import stream_b200
    from stream_b200 import lib, workloads
    from stream_b200.mesh import AlphaShape3D

    P = ctypes.c_void_p
    lib.AlphaShape3D_set_stream.argtypes = [P, P]
    lib.AlphaShape3D_set_profiling.argtypes = [P, ctypes.c_int]
    lib.AlphaShape3D_get_profile.argtypes = [P, P]
    lib.AlphaShape3D_get_profile_stages.argtypes = [P, P, ctypes.c_uint32, P]
    lib.AlphaShape3D_set_work_counters.argtypes = [P, ctypes.c_int]
    lib.AlphaShape3D_get_work.argtypes = [P, P]
    lib.AlphaShape3D_init.argtypes = [P]
    lib.AlphaShape3D_compute.argtypes = [P]
    lib.stream_b200_launch_count.restype = ctypes.c_ulonglong
    from stream_b200.mesh.ashape3d import (AlphaShape3D_get_elem, AlphaShape3D_get_nelem,
                                           AlphaShape3D_set_nodes)
    if not stream_b200.device_ok():
        raise RuntimeError("bench.py: no B200 visible")

    pts, alpha = workloads.meshing_stress(a.points, seed=a.seed)
    n = len(pts)
    stream = torch.cuda.current_stream()
    d_in = torch.from_numpy(np.concatenate([pts, alpha[:, None]], axis=1)).cuda()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    mesh = AlphaShape3D()
    h = mesh.mesh
    lib.AlphaShape3D_set_stream(h, P(stream.cuda_stream))
    mesh.nnodes = n
    stream_b200.check(lib.AlphaShape3D_set_nodes_device(h, n, P(d_in.data_ptr())), "set_nodes_device")

    def step():
        lib.AlphaShape3D_init(h)
        lib.AlphaShape3D_compute(h)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    st = mesh.status
    if st & 0x1B1:
        raise RuntimeError(f"remesh status 0x{st:x}: {stream_b200.last_error()}")
    counters = mesh.counters()
    n_elems = lib.AlphaShape3D_get_nelem(h)

    # ---- device-resident timing -------------------------------------------------
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.stream_b200_launch_count()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1.0)  # write > L2 between timed steps
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    launches = int(lib.stream_b200_launch_count() - l0)
    ms = max_over_ranks(sum(times) / len(times), dist)
    if dist:
        dist.barrier()
    clocks = clk.summary()
    value = replica_rate(ws, n, ms)

    # ---- per-stage profile (live CUDA events inside the library) -----------------
    lib.AlphaShape3D_set_profiling(h, 1)
    prof_runs = []
    for _ in range(3):
        flush.fill_(1.0)
        step()
        ms8 = np.zeros(8, np.float32)
        stream_b200.check(lib.AlphaShape3D_get_profile_stages(h, ms8.ctypes.data_as(P), 8, None), "get_profile")
        prof_runs.append(ms8)
    # one more step with the counting build of the star pass (same outputs):
    # stage-1 FP32 insphere tests and stage-2 FP64 evaluations, 117 flops each
    work = np.zeros(2, np.uint64)
    lib.AlphaShape3D_set_work_counters(h, 1)
    flush.fill_(1.0)
    step()
    stream_b200.check(lib.AlphaShape3D_get_work(h, work.ctypes.data_as(P)), "get_work")
    lib.AlphaShape3D_set_work_counters(h, 0)
    lib.AlphaShape3D_set_profiling(h, 0)
    prof = np.median(np.stack(prof_runs), axis=0)
    names = ["bbox_morton_hist", "radix_sort", "gather_karras_fit", "candidates", "star", "star_exact",
             "scan_readback", "compress"]
    stages = {k: round(float(v), 4) for k, v in zip(names, prof)}
    hbm, peak_kind = _peaks()
    # Radix sort: 8 onesweep passes over (u64 key, u32 value): 24 B per key per
    # pass (+8 B/key up-front histogram fused into the Morton kernel).
    sort_bytes = 8 * 24 * n
    sort_gbs = sort_bytes / (prof[1] / 1e3) / 1e9
    # The dominant kernel is the star pass (k_star): per point it reads its
    # candidate list once (4 B x candidates), its coordinates (16 B) and writes
    # its outputs (masks 32 B, counts 10 B); its conflict tests run from L1/L2
    # and registers.  It is bound by FP32 arithmetic issue (and divergence), not
    # by HBM: achieved = counted work (FP32 insphere filters and FP64
    # semi-static evaluations, 117 flops each) over its CUDA-event time,
    # against the nominal FP32 peak (148 SMs x 128 lanes x 2 flops) at the SM
    # clock sampled during the timed steps.
    star_bytes = n * (4 * 70 + 16 + 42)
    sm_mhz = float((clocks or {}).get("sm_mhz") or 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    star_flops = 117.0 * (float(work[0]) + float(work[1]))
    alu_ach = star_flops / (prof[4] / 1e3) / 1e12
    roofline = {"bound": "alu", "kernel": "k_star (star pass)", "achieved": round(alu_ach, 2),
                "peak": round(fp32_peak, 1), "unit": "TFLOP/s", "frac": round(alu_ach / fp32_peak, 4),
                "peak_kind": f"nominal FP32 at the sampled SM clock ({sm_mhz:.0f} MHz); no measured FP32 peak",
                "traffic": K_STAR_DRAM_BYTES_4M,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_star launch on the 1M "
                                  "meshing-stress cloud, scaled to 4M by the star count",
                "algorithmic_bytes_per_launch": star_bytes,
                "flops_per_launch": star_flops, "insphere_tests": int(work[0]), "fp64_filter_evals": int(work[1]),
                "flops_per_test": 117, "ms_per_launch": round(float(prof[4]), 4),
                "hbm": {"peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                        "radix_sort_4m": {"achieved": round(sort_gbs, 1), "frac": round(sort_gbs / hbm, 4),
                                          "ms": round(float(prof[1]), 4), "algorithmic_bytes": sort_bytes,
                                          "note": "8 onesweep passes x 24 B per key; 192 MB, L2-resident"}}}

    # Stage throughputs: points sorted, BVH nodes built (gather + Karras + fit of
    # the 2N - 1 nodes), tets produced by the two star passes.
    rates = {"sorted_mpts_s": round(n / (prof[1] / 1e3) / 1e6, 1),
             "bvh_mnodes_s": round((2 * n - 1) / (prof[2] / 1e3) / 1e6, 1),
             "tets_m_s": round(n_elems / ((prof[4] + prof[5]) / 1e3) / 1e6, 1)}

    # ---- end to end through the public host API -----------------------------------
    # Pinned host buffers, passed to the reference-named entry points as numpy views.
    pin_xyz = torch.from_numpy(pts).pin_memory()
    pin_al = torch.from_numpy(alpha).pin_memory()
    pin_out = torch.empty((int(n_elems * 1.2) + 1024, 4), dtype=torch.int32).pin_memory()
    np_xyz, np_al = pin_xyz.numpy(), pin_al.numpy()
    e2e_times = []
    d2h = 0
    for i in range(a.warmup + a.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        AlphaShape3D_set_nodes(h, n, np_xyz, np_al)
        lib.AlphaShape3D_init(h)
        lib.AlphaShape3D_compute(h)
        ne = AlphaShape3D_get_nelem(h)
        if ne > pin_out.shape[0]:
            pin_out = torch.empty((ne, 4), dtype=torch.int32).pin_memory()
        AlphaShape3D_get_elem(h, pin_out[:ne].numpy().view(np.uint32))
        e1.record(stream)
        e1.synchronize()
        if i >= a.warmup:
            e2e_times.append(e0.elapsed_time(e1))
            d2h = 16 * ne
    e2e_ms = max_over_ranks(sum(e2e_times) / len(e2e_times), dist)
    e2e = {"value": round(replica_rate(ws, n, e2e_ms), 4), "unit": UNIT, "h2d_bytes_per_step": 16 * n,
           "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms, 3)}

    # ---- pressure solve (dam-break column) -----------------------------------------
    solve = solve_4m = pfem = None
    if not a.no_solve:
        solve = bench_solve(a, torch, stream)
        if a.heldout_points:
            solve_4m = bench_solve(a, torch, stream, h=(0.4 * 0.8 * 0.4 / a.heldout_points) ** (1.0 / 3.0),
                                   methods=(("fp64_jacobi_pcg", 0), ("fsai_mixed_ir", 2), ("ky_fsai_mixed_ir", 3)),
                                   reps=2)
    if a.pfem_steps:
        pfem = bench_pfem(a)
    pfem_dyn = bench_pfem_dynamics(a) if a.pfem_dyn_steps else None
    remesh2d = bench_remesh2d(a, torch) if a.points2d else None
    delaunay2d = bench_delaunay2d(a, torch) if a.points_delaunay2d else None

    # ---- the same corner sample on the GPU, TRBVH, 64M sort, uniform3D -----------------
    wl = _workloads()
    same = bench_same_sample(a, torch, wl, pts, alpha)
    trbvh = bench_trbvh(a, torch, pts, alpha) if a.trbvh else None
    lbvh64 = bench_lbvh_device(a, torch, hbm) if a.lbvh_points else None
    if lbvh64:
        roofline["hbm"]["radix_sort_64m"] = lbvh64.pop("sort_roofline")
    uni3d = bench_uniform3d(a, torch, wl) if a.uniform3d else None
    plain = bench_plain(a, torch, wl) if a.plain_points else None

    # ---- CPU baseline ----------------------------------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        cpu = cpu_baselines(wl, pts, alpha, a.cpu_sample, runs=5)
        same["cpu_reference_ms"] = cpu["ms_per_run"]
        same["gpu_over_cpu_e2e"] = round(cpu["ms_per_run"] / same["e2e_ms"], 1)

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, float(alpha[0]), ws), "tets": int(n_elems),
        "roofline": roofline, "stages_ms": stages, "rates": rates, "counters": counters, "cpu_baseline": cpu,
        "same_sample": same, "e2e": e2e, "trbvh": trbvh, "lbvh_64m": lbvh64, "remesh3d_uniform": uni3d,
        "plain_200k": plain,
        "gpu_launches": launches, "gpu_launches_per_step": launches // max(1, a.steps), "clocks": clocks,
        "solve": solve,
        "solve_heldout": solve_4m,
        "pfem": pfem,
        "pfem_dynamics": pfem_dyn,
        "remesh2d": remesh2d,
        "delaunay2d": delaunay2d,
    }
    print(json.dumps(line, default=_json_default), flush=True)
    return 0


def _json_default(o):
    if isinstance(o, (np.floating,)):
        return float(o)
    if isinstance(o, (np.integer,)):
        return int(o)
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError(type(o))


def _mesher_on_stream(torch, pts, alpha, morton_bits=63):
    """An AlphaShape3D handle on torch's current stream with its points on the
    device (float4 x, y, z, alpha)."""
    import stream_b200
    from stream_b200 import lib
    from stream_b200.mesh import AlphaShape3D
    P = ctypes.c_void_p
    stream = torch.cuda.current_stream()
    d_in = torch.from_numpy(np.concatenate([pts, alpha[:, None]], axis=1).astype(np.float32)).cuda()
    m = AlphaShape3D(morton_bits=morton_bits)
    lib.AlphaShape3D_set_stream(m.mesh, P(stream.cuda_stream))
    m.nnodes = len(pts)
    stream_b200.check(lib.AlphaShape3D_set_nodes_device(m.mesh, len(pts), P(d_in.data_ptr())), "set_nodes_device")
    return m, d_in, stream


def _time_remesh(torch, pts, alpha, warmup, steps, flush, morton_bits=63, keep=False):
    """Median device ms of init + compute (CUDA events on the handle's stream,
    L2 flushed before each step), median e2e ms through the host API (points
    from pinned host memory, tets back to pinned host memory), and the tets
    (and the meshed handle when keep is set)."""
    from stream_b200 import lib
    from stream_b200.mesh.ashape3d import AlphaShape3D_get_elem, AlphaShape3D_get_nelem, AlphaShape3D_set_nodes
    m, d_in, stream = _mesher_on_stream(torch, pts, alpha, morton_bits)
    h = m.mesh
    dev = []
    for i in range(warmup + steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.AlphaShape3D_init(h)
        lib.AlphaShape3D_compute(h)
        e1.record(stream)
        e1.synchronize()
        if i >= warmup:
            dev.append(e0.elapsed_time(e1))
    if m.status & 0x1B1:
        raise RuntimeError(f"remesh status 0x{m.status:x}")
    ne = AlphaShape3D_get_nelem(h)
    pin_xyz = torch.from_numpy(np.ascontiguousarray(pts)).pin_memory()
    pin_al = torch.from_numpy(np.ascontiguousarray(alpha)).pin_memory()
    pin_out = torch.empty((ne + 1024, 4), dtype=torch.int32).pin_memory()
    e2e = []
    for i in range(warmup + steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        AlphaShape3D_set_nodes(h, len(pts), pin_xyz.numpy(), pin_al.numpy())
        lib.AlphaShape3D_init(h)
        lib.AlphaShape3D_compute(h)
        k = AlphaShape3D_get_nelem(h)
        AlphaShape3D_get_elem(h, pin_out[:k].numpy().view(np.uint32))
        e1.record(stream)
        e1.synchronize()
        if i >= warmup:
            e2e.append(e0.elapsed_time(e1))
    if keep:
        return float(np.median(dev)), float(np.median(e2e)), int(ne), m
    return float(np.median(dev)), float(np.median(e2e)), int(ne)


def cpu_solve_baselines(ps):
    """The same system solved on the host: the reference's own FP32 Jacobi-PCG
    (oracle/_ref, all host threads; its stopping rule, sqrt(r.z) <= 1e-6
    absolute, src/numerics/conjugate_gradient.cpp:61-136) and an FP64
    Jacobi-PCG in NumPy/SciPy to ||b - Ax|| <= 1e-10 ||b||."""
    import scipy.sparse as sp
    row, col, val, b = ps.get_csr()
    n = len(b)
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    out = {}
    try:
        from oracle.oracle import Reference
        ref = Reference()
        with _QuietStdout():  # the reference prints its residuals
            t0 = time.perf_counter()
            x, it = ref.cg_f32(row, col, val.astype(np.float32), b.astype(np.float32), np.zeros(n, np.float32))
            ms = 1e3 * (time.perf_counter() - t0)
        out["reference_fp32_jacobi_pcg"] = {
            "kind": "reference", "cores": os.cpu_count() or 1, "ms": round(ms, 2), "iterations": it,
            "relres": float(np.linalg.norm(b - A @ x.astype(np.float64)) / np.linalg.norm(b)),
            "stop": "sqrt(r.z) <= 1e-6 (absolute, FP32), the reference's rule"}
    except FileNotFoundError:
        out["reference_fp32_jacobi_pcg"] = None
    d = A.diagonal()
    t0 = time.perf_counter()
    x = np.zeros(n)
    r = b.copy()
    z = r / d
    p = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    it = 0
    while np.linalg.norm(r) > 1e-10 * bn and it < 20 * n:
        q = A @ p
        al = rz / (p @ q)
        x += al * p
        r -= al * q
        z = r / d
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
        it += 1
    ms = 1e3 * (time.perf_counter() - t0)
    out["numpy_fp64_jacobi_pcg"] = {"kind": "port", "cores": 1, "ms": round(ms, 2), "iterations": it,
                                    "relres": float(np.linalg.norm(b - A @ x) / bn), "stop": "1e-10 relative"}
    return out


def bench_plain(a, torch, wl):
    """The plain-method chain on 200,000 uniform points (FP64 coordinates from a
    seeded generator, meshed in FP32 as the reference's Sphere3D holds them):
    30-bit Morton codes, sort, LBVH, Delaunay + alpha shape with alpha =
    1.3 N^-1/3, P1 Laplacian on the kept tets (f = 1, u = 0 on the
    alpha-shape boundary nodes), FP64 Jacobi-PCG to ||b - Ax|| <= 1e-10 ||b||.
    Remesh: CUDA events on the mesher's stream; assembly: host clock between
    device-wide synchronisations (it runs on the system's own stream); solve:
    the solver's own events."""
    from stream_b200.numerics import PoissonSystem
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    pts, alpha = wl.uniform_cube(a.plain_points, seed=a.seed)
    dev, e2e, ne, m = _time_remesh(torch, pts, alpha, max(3, a.warmup), a.steps, flush, morton_bits=30, keep=True)
    ps = PoissonSystem()
    asm = []
    for i in range(max(3, a.warmup) + a.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ps.assemble(m, rhs="one")  # runs on the system's own stream
        torch.cuda.synchronize()
        asm.append(1e3 * (time.perf_counter() - t0))
    n, nnz = ps.size()
    solves = [ps.solve(method=0, rtol=1e-10)[1] for _ in range(3)]
    rep = min(solves, key=lambda r: r["ms"])
    solve_ms = rep["ms"]
    asm_ms = float(np.median(asm[max(3, a.warmup):]))
    cpu = None
    if not a.no_cpu:
        cpu = cpu_solve_baselines(ps)
    return {"workload": f"{len(pts)} points uniform in [0,1)^3 (seed {a.seed}), 30-bit Morton codes, alpha = "
                        f"1.3 N^-1/3 = {float(alpha[0]):.6g}; P1 Laplacian, f = 1, u = 0 on boundary nodes; "
                        f"FP64 Jacobi-PCG to 1e-10",
            "cpu_solve": cpu,
            "points": len(pts), "tets": ne, "rows": n, "nnz": nnz, "nnz_per_row": round(nnz / max(1, n), 2),
            "remesh_ms": round(dev, 4), "remesh_e2e_ms": round(e2e, 3), "assembly_ms": round(asm_ms, 4),
            "solve_ms": round(solve_ms, 3), "iterations": rep["iterations"], "relres": rep["relres"],
            "converged": rep["converged"], "chain_ms": round(dev + asm_ms + solve_ms, 3)}


def bench_same_sample(a, torch, wl, pts, alpha):
    """This library on the corner of the cloud that the CPU baseline and the
    reference arm time (same points, same alpha): a same-input pair."""
    sp, sa, frac = wl.sub_cube(pts, alpha, a.cpu_sample)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    dev, e2e, ne = _time_remesh(torch, sp, sa, max(3, a.warmup), a.steps, flush)
    return {"workload": f"the {len(sp)}-point corner (box {frac:.3f} of the extent) of the same cloud, same alpha",
            "points": len(sp), "tets": ne, "device_ms": round(dev, 3), "e2e_ms": round(e2e, 3),
            "mpts_s": round(len(sp) / dev / 1e3, 3), "e2e_mpts_s": round(len(sp) / e2e / 1e3, 3)}


def bench_uniform3d(a, torch, wl):
    """The reference's uniform3D harness clouds (testcases/IMR26/uniform3D.cpp:
    glibc srand(42), x, y, z = (float) rand() / RAND_MAX): the published example
    (100,000 points, alpha 0.022: 526,040 tets, ttot 28.0 ms on the author's RTX
    4060, testcases/IMR26/README.md:93-99) and the paper's sweep (README.md:80-86).
    ttot here = init + compute (the reference's ttot = tlbvh + tashape leaves out
    tcompress; compute() here includes the compress step)."""
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    out = []
    for n, al in ((100_000, 0.022),) + tuple(wl.UNIFORM3D_SWEEP):
        pts, alpha = wl.glibc_uniform_cube(n, al)
        dev, e2e, ne = _time_remesh(torch, pts, alpha, max(3, a.warmup), a.steps, flush)
        rec = {"points": n, "alpha": al, "tets": ne, "ttot_ms": round(dev, 4), "e2e_ms": round(e2e, 3),
               "mpts_s": round(n / dev / 1e3, 2)}
        if (n, al) == (100_000, 0.022):
            rec["published_reference"] = {"ttot_ms": 28.0, "tets": 526040,
                                          "source": "testcases/IMR26/README.md:93-99 (RTX 4060, implied)"}
            if not a.no_cpu:
                kind, ts = run_cpu_reference(pts, alpha, 3, 1, threads=os.cpu_count() or 1)
                rec["cpu_reference"] = {"ms": round(1e3 * statistics.median(ts), 2), "kind": kind,
                                        "cores": os.cpu_count() or 1, "sample": "the whole cloud, median of 3"}
        out.append(rec)
    return out


def bench_trbvh(a, torch, pts, alpha):
    """TRBVH over the meshing-stress cloud (spheres of radius alpha): Apetrei
    build + 3 rounds of treelet-7 restructuring with the 3D surface-area SAH.
    Device time = the CUDA events the handle records between its stages."""
    from stream_b200.geometry import Sphere3DTRBVH
    n = len(pts)
    xyzr = np.concatenate([pts, alpha[:, None]], 1).astype(np.float32)
    t = Sphere3DTRBVH()
    t.set_objects(xyzr, treelet_size=7, area3d=True, rounds=3)
    t.set_profiling(True)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    runs = []
    for i in range(max(3, a.warmup) + a.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        if t.build() != 0:
            raise RuntimeError("TRBVH build status")
        if i >= max(3, a.warmup):
            runs.append(t.profile())
    st = {k: float(np.median([r[k] for r in runs])) for k in runs[0]}
    total = sum(st.values())
    return {"workload": f"{n} spheres (the meshing-stress cloud, radius = alpha), treelet 7, 3 rounds, 3D SAH",
            "build_ms": round(total, 3), "stages_ms": {k: round(v, 4) for k, v in st.items()},
            "mpts_s": round(n / total / 1e3, 1), "bvh_mnodes_s": round((2 * n - 1) / total / 1e3, 1),
            "hierarchy_mnodes_s": round((2 * n - 1) / (st["apetrei"] + st["treelets"]) / 1e3, 1)}


def bench_lbvh_device(a, torch, hbm):
    """Sphere3DLBVH over lbvh_points uniform spheres already on the device (the
    64M-key case of the sort): stage times and the onesweep sort's algorithmic
    bandwidth, 8 passes x (8 B key + 4 B value) read and written per key."""
    from stream_b200.geometry import Sphere3DLBVH
    n = a.lbvh_points
    g = torch.Generator(device="cuda").manual_seed(a.seed)
    x = torch.rand((n, 4), device="cuda", generator=g)
    x[:, 3] = 0.25 * n ** (-1.0 / 3.0)
    b = Sphere3DLBVH()
    b.set_objects_device(x.data_ptr(), n, 63, False)
    b.set_profiling(True)
    runs = []
    for i in range(max(3, a.warmup) + a.steps):
        torch.cuda.synchronize()
        if b.build() != 0:
            raise RuntimeError("LBVH build status")
        if i >= max(3, a.warmup):
            runs.append(b.profile())
    st = {k: float(np.median([r[k] for r in runs])) for k in runs[0]}
    sort_bytes = 8 * 24 * n
    sort_gbs = sort_bytes / (st["radix_sort"] / 1e3) / 1e9
    gather_gbs = 36 * n / (st["gather"] / 1e3) / 1e9
    del x
    return {"workload": f"{n} uniform spheres resident on the device, 63-bit codes",
            "build_ms": round(sum(st.values()), 3), "stages_ms": {k: round(v, 4) for k, v in st.items()},
            "sorted_mpts_s": round(n / st["radix_sort"] / 1e3, 1),
            "bvh_mnodes_s": round((2 * n - 1) / (st["gather"] + st["karras_fit"]) / 1e3, 1),
            "gather_gbs": round(gather_gbs, 1),
            "sort_roofline": {"achieved": round(sort_gbs, 1), "frac": round(sort_gbs / hbm, 4),
                              "ms": round(st["radix_sort"], 4), "algorithmic_bytes": sort_bytes,
                              "note": f"{n} keys, 8 passes x 24 B per key"}}


def bench_solve(a, torch, stream, h=None, methods=(("fp64_jacobi_pcg", 0), ("mixed_ir", 1), ("fsai_mixed_ir", 2),
                                                  ("ky_fsai_mixed_ir", 3)), reps=2):
    """Dam-break pressure system: remesh, assemble, then FP64 Jacobi-PCG,
    Jacobi mixed-precision refinement, learned-FSAI mixed-precision
    refinement (the network shipped with the package) and the same refinement
    with the Kolotilina-Yeremin FSAI (exact local solves, the G the network's
    functional is minimised by) to ||b - Ax|| <= 1e-8 ||b||.  Each solve
    starts from x = 0; the FSAI times include the preconditioner's set-up and
    network inference (or local solves) on this system."""
    from stream_b200.numerics import FsaiModel
    h = a.solve_h if h is None else h
    ps = _dambreak_system(h, a.seed)
    n, nnz = ps.size()
    out = {"workload": f"dam-break column 0.4x0.8x0.4, h={h:.6g}, jitter 0.1h, alpha=1.2h, "
                       f"RHS = div u (8 Fourier modes), free surface p=0", "n": n, "nnz": nnz}
    model = FsaiModel.trained()
    x64 = None
    xs = {}
    for name, method in methods:
        rs = []
        for _ in range(reps):
            if method in (2, 3):
                ps.set_fsai(model)  # rebuilds the preconditioner (set-up + inference) inside the timed solve
            x, rep = ps.solve(method=method, rtol=1e-8)
            if method in (2, 3):
                rep.update({k: v for k, v in ps.fsai_stats().items() if k != "fallback"})
            rs.append(rep)
        rep = min(rs, key=lambda r: r["ms"])
        xs[name] = x
        if method == 0:
            x64 = x
            rep["x_err_vs_fp64"] = 0.0
        else:
            rep["x_err_vs_fp64"] = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
        rep["s"] = rep.pop("ms") / 1e3
        # algorithmic HBM bytes of one CG iteration (matrix streamed once, each
        # vector read or written once per kernel) over the whole solve's time
        if method == 0:
            per_it = 12 * nnz + 108 * n
        elif method == 1:
            per_it = 8 * nnz + 56 * n
        else:
            ne = rep.get("lower_edges", (nnz + n) // 2)
            per_it = 8 * nnz + 12 * ne + 76 * n
        rep["cg_algorithmic_gbs"] = round(per_it * rep["iterations"] / rep["s"] / 1e9, 1)
        out[name] = rep
    # Error of each solution against an FP64 Jacobi-PCG solve to 1e-13 (untimed).
    xr, rr = ps.solve(method=0, rtol=1e-13, maxit=4 * out["fp64_jacobi_pcg"]["iterations"] + 1000)
    out["fp64_1e13"] = {"iterations": rr["iterations"], "relres": rr["relres"], "converged": rr["converged"]}
    for name, _ in methods:
        out[name]["x_err_vs_fp64_1e13"] = float(np.linalg.norm(xs[name] - xr) / np.linalg.norm(xr))
    base = out["fp64_jacobi_pcg"]["s"]
    if "mixed_ir" in out:
        out["mixed_over_fp64_time"] = round(out["mixed_ir"]["s"] / base, 4)
    out["fsai_mixed_over_fp64_time"] = round(out["fsai_mixed_ir"]["s"] / base, 4)
    if "ky_fsai_mixed_ir" in out:
        out["ky_fsai_mixed_over_fp64_time"] = round(out["ky_fsai_mixed_ir"]["s"] / base, 4)
    return out


def bench_remesh2d(a, torch):
    """2D alpha shape on the reference's uniform2D benchmark cloud
    (testcases/IMR26/uniform2D.cpp; README.md:48-54 publishes 1,877,465
    triangles and ttot = 22.35 ms for -n 1000000 -a 0.0012): glibc srand(42)
    points, one AlphaShape2D handle, init() + compute() per step as the
    reference's harness times them (tlbvh + tashape; compress is inside
    compute() here, as in the reference's C entry point).  Device time = CUDA
    events around each step; a 256 MiB write between steps flushes L2; e2e =
    set_nodes from host arrays + init + compute + get_elem to host, wall clock.
    CPU arm: the reference's own 2D sources built for the host (oracle/_ref),
    all host threads, on the full cloud."""
    from stream_b200 import workloads
    from stream_b200.mesh import AlphaShape2D
    n = a.points2d
    pts, al = workloads.glibc_uniform_square(n, 0.0012)
    m = AlphaShape2D()
    m.set_profiling(True)
    m.set_nodes(pts, al)
    m.compute()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    ts, stages = [], []
    for i in range(a.warmup + a.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        m.init()
        m.compute()
        p = m.profile()
        if i >= a.warmup:
            ts.append(sum(p.values()))
            stages.append(p)
    ms = float(np.median(ts))
    ntri = int(len(m.get_elem()))
    e2e = []
    for i in range(a.warmup + a.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.set_nodes(pts, al)
        m.compute()
        el = m.get_elem()
        t1 = time.perf_counter()
        if i >= a.warmup:
            e2e.append(1e3 * (t1 - t0))
    e2e_ms = float(np.median(e2e))
    cpu = None
    if not a.no_cpu:
        from oracle.oracle import Reference, Restatement
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        try:
            ref, kind = Reference(), "reference"
        except FileNotFoundError:
            ref, kind = Restatement(), "port"
        with _QuietStdout():
            ref.ashape2d(pts, al)
        cts = []
        for _ in range(3):
            t0 = time.perf_counter()
            with _QuietStdout():
                r = ref.ashape2d(pts, al)
            cts.append(1e3 * (time.perf_counter() - t0))
        cms = float(np.median(cts))
        cpu = {"ms": round(cms, 2), "mpts_s": round(n / cms / 1e3, 3), "kind": kind,
               "cores": int(os.environ["OMP_NUM_THREADS"]), "triangles": int(len(r.elems)),
               "sample": f"the full {n}-point cloud, median of 3 after 1 warm-up (includes the ctypes copies)"}
    return {"workload": f"uniform2D: {n} points, glibc srand(42) rand()/RAND_MAX in [0,1]^2, alpha = 0.0012; "
                        "64-bit 2D Morton LBVH + 2D alpha shape (exact predicates)",
            "points": n, "triangles": ntri, "ms_per_step": round(ms, 4), "mpts_s": round(n / ms / 1e3, 3),
            "stages_ms": {k: round(float(np.median([p[k] for p in stages])), 4) for k in stages[0]},
            "e2e": {"ms_per_step": round(e2e_ms, 3), "mpts_s": round(n / e2e_ms / 1e3, 3),
                    "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 12 * ntri},
            "counters": m.counters(), "cpu_reference": cpu,
            "published_reference": {"ttot_ms": 22.35, "triangles": 1877465,
                                    "source": "testcases/IMR26/README.md:48-54 (RTX 4060, implied)"}}


def bench_delaunay2d(a, torch):
    """2D Delaunay mesher (Mesh2D, src/mesh/mesh.cpp:806-862) on a uniform
    cloud: set_nodes + init, insert_morton_neighbors, insert_BVH_neighbors,
    insert_iterative, remove_super_nodes and the compress of get_nelem per
    step, timed per phase by wall clock around the calls (each call waits for
    its device work; L2 flushed between steps); e2e adds the host copies in
    and out (get_elem).  The reference's own Mesh2D overruns its traversal
    heap on such clouds (mesh.cpp:471, 509, 548), so the CPU comparison is
    Qhull (scipy.spatial.Delaunay, one thread) on the same points."""
    from stream_b200.mesh import Mesh2D
    n = a.points_delaunay2d
    xy = np.random.default_rng(0).random((n, 2)).astype(np.float32)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    m = Mesh2D()
    names = ("set_nodes_init", "morton", "bvh", "iterative", "compress")
    phases, e2e = [], []
    for i in range(a.warmup + a.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t = [time.perf_counter()]
        m.set_nodes(xy)
        t.append(time.perf_counter())
        m.insert_morton_neighbors()
        t.append(time.perf_counter())
        m.insert_BVH_neighbors()
        t.append(time.perf_counter())
        m.insert_iterative()
        t.append(time.perf_counter())
        m.remove_super_nodes()
        e = m.get_elem()
        t.append(time.perf_counter())
        if i >= a.warmup:
            phases.append(np.diff(t) * 1e3)
            e2e.append((t[-1] - t[0]) * 1e3)
    med = np.median(np.stack(phases), 0)
    mesh_ms = float(med[1:4].sum())
    cpu = None
    if not a.no_cpu:
        from scipy.spatial import Delaunay
        sample = xy[:min(n, 1_000_000)]
        t0 = time.perf_counter()
        d = Delaunay(sample.astype(np.float64))
        cms = 1e3 * (time.perf_counter() - t0)
        cpu = {"ms": round(cms, 2), "mpts_s": round(len(sample) / cms / 1e3, 3), "kind": "qhull", "cores": 1,
               "triangles": int(len(d.simplices)), "sample": f"{len(sample)} points of the same cloud, one run"}
    return {"workload": f"{n} uniform points in [0,1]^2 (numpy seed 0), float32; Delaunay triangulation with 3 super "
                        "nodes, super triangles removed",
            "points": n, "triangles": int(len(e)), "status": m.status, "incomplete": m.counters()["incomplete"],
            "phases_ms": {k: round(float(v), 3) for k, v in zip(names, med)},
            "insert_ms": round(mesh_ms, 3), "insert_mpts_s": round(n / mesh_ms / 1e3, 3),
            "e2e": {"ms_per_step": round(float(np.median(e2e)), 3), "mpts_s": round(n / float(np.median(e2e)) / 1e3, 3),
                    "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 12 * int(len(e))},
            "cpu_qhull": cpu}


def bench_pfem(a):
    """PFEM step loop: a dam-break column of pfem_points particles advected by
    a Taylor-Green field (amplitude 0.5, dt = 0.002), remeshed, assembled and
    solved with the learned-FSAI mixed solver (Jacobi-PCG fallback) every
    step.  One untimed step, then pfem_steps steps; per-phase device times
    are CUDA events recorded by the library between the phases."""
    import math
    from stream_b200 import workloads
    from stream_b200.numerics import FsaiModel
    from stream_b200.pfem import PfemLoop, TaylorGreen
    h = (0.4 * 0.8 * 0.4 / a.pfem_points) ** (1.0 / 3.0)
    pts, al = workloads.dambreak_column(h=h, seed=a.seed)
    rng = np.random.default_rng(a.seed + 1)
    k = rng.normal(size=(8, 3)) * 6.0
    amp = rng.normal(size=(8, 3)) * 0.1
    modes = np.concatenate([k, np.sum(amp * k, 1, keepdims=True), rng.uniform(0, 2 * math.pi, (8, 1))], 1)
    flow = TaylorGreen(center=(0.2, 0.4, 0.2), k=2 * math.pi / 0.4, amp=0.5)
    loop = PfemLoop(pts.astype(np.float64), float(al[0]), flow, modes.astype(np.float32), FsaiModel.trained())
    loop.step(0.002)
    reps = [loop.step(0.002) for _ in range(a.pfem_steps)]
    keys = ("advect_ms", "remesh_ms", "assembly_ms", "precond_ms", "solve_ms", "step_ms")
    mean = {k: round(float(np.mean([r[k] for r in reps])), 3) for k in keys}
    return {"workload": f"dam-break column {len(pts)} particles (h={h:.5f}, alpha=1.2h), Taylor-Green "
                        f"amplitude 0.5, k = 2 pi / 0.4, dt = 0.002; learned-FSAI mixed solve to 1e-8",
            "particles": len(pts), "steps": a.pfem_steps, "ms_per_step": mean["step_ms"], "breakdown_ms": mean,
            "iterations_mean": round(float(np.mean([r["iterations"] for r in reps])), 1),
            "fallback_fraction": float(np.mean([r["fallback"] for r in reps])),
            "relres_max": float(max(r["relres"] for r in reps)),
            "tets_last": reps[-1]["tets"], "all_converged": all(r["converged"] for r in reps)}


def bench_pfem_dynamics(a):
    """The step loop with the fractional-step dynamics (gravity, viscosity,
    walls): a dam-break column of pfem_dyn_points particles collapsing in a
    tank 3 x its width, dt = 0.002, learned-FSAI mixed pressure solve to 1e-8.
    One untimed step, then pfem_dyn_steps steps (library CUDA events)."""
    from stream_b200 import workloads
    from stream_b200.numerics import FsaiModel
    from stream_b200.pfem import PfemLoop, Physics
    h = (0.4 * 0.8 * 0.4 / a.pfem_dyn_points) ** (1.0 / 3.0)
    pts, al = workloads.dambreak_column(h=h, seed=a.seed)
    loop = PfemLoop(pts.astype(np.float64), float(al[0]), model=FsaiModel.trained())
    loop.set_physics(Physics(g=(0.0, -9.81, 0.0), nu=1e-6, rho=1000.0, lo=(0.0, 0.0, 0.0), hi=(1.2, 1.0, 0.4)))
    loop.step(0.002)
    reps = [loop.step(0.002) for _ in range(a.pfem_dyn_steps)]
    keys = ("advect_ms", "remesh_ms", "assembly_ms", "precond_ms", "solve_ms", "step_ms")
    mean = {("velocity_update_ms" if k == "advect_ms" else k): round(float(np.mean([r[k] for r in reps])), 3)
            for k in keys}
    x = loop.particles()
    return {"workload": f"dam break: column 0.4 x 0.8 x 0.4 of {len(pts)} particles (h={h:.5f}, alpha=1.2h) in a "
                        "1.2 x 1.0 x 0.4 tank, g = 9.81, nu = 1e-6, rho = 1000, dt = 0.002; fractional step, "
                        "learned-FSAI mixed pressure solve to 1e-8",
            "particles": len(pts), "steps": a.pfem_dyn_steps, "ms_per_step": mean["step_ms"], "breakdown_ms": mean,
            "iterations_mean": round(float(np.mean([r["iterations"] for r in reps])), 1),
            "fallback_fraction": float(np.mean([r["fallback"] for r in reps])),
            "all_converged": all(r["converged"] for r in reps),
            "front_x_end": round(float(x[:, 0].max()), 4), "front_x_start": round(float(pts[:, 0].max()), 4)}


def _dambreak_system(h, seed):
    """Remeshed dam-break column with the divergence right-hand side of the solve benchmark."""
    from stream_b200 import workloads
    from stream_b200.mesh import AlphaShape3D
    from stream_b200.numerics import PoissonSystem
    pts, al = workloads.dambreak_column(h=h, seed=seed)
    m = AlphaShape3D()
    m.set_nodes(pts, al)
    m.compute()
    rng = np.random.default_rng(seed)
    modes = []
    for _ in range(8):
        k = rng.integers(-3, 4, size=3) * np.pi / 0.4
        amp = rng.standard_normal(3)
        modes.append([k[0], k[1], k[2], float(amp @ k), rng.uniform(0, 2 * np.pi)])
    ps = PoissonSystem()
    ps.assemble(m, rhs="div", modes=np.array(modes, np.float32))
    return ps


def run_once(a):
    """A single remesh or a single pair of solves, nothing timed: the process ncu attaches to."""
    from stream_b200 import workloads
    from stream_b200.mesh import AlphaShape3D
    if a.workload == "pfem":
        a.pfem_steps = 2
        print(json.dumps({"once": "pfem", **bench_pfem(a)}))
        return 0
    if a.workload == "pfemdyn":
        a.pfem_dyn_steps = 2
        print(json.dumps({"once": "pfemdyn", **bench_pfem_dynamics(a)}))
        return 0
    if a.workload == "solve":
        from stream_b200.numerics import FsaiModel, PoissonSystem
        ps = _dambreak_system(a.solve_h, a.seed)
        ps.set_fsai(FsaiModel.trained())
        _, r2 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=1e-8)
        _, r3 = ps.solve(method=PoissonSystem.KY_FSAI_MIXED, rtol=1e-8)
        _, r0 = ps.solve(method=PoissonSystem.FP64_JACOBI, rtol=1e-8)
        print(json.dumps({"once": "solve", "n": ps.size()[0], "fsai_mixed": r2, "ky_fsai_mixed": r3,
                          "fp64_jacobi": r0}))
        return 0
    if a.workload == "lbvh":  # Sphere3DLBVH build over --points uniform points already on the device
        import torch
        from stream_b200.geometry import Sphere3DLBVH
        g = torch.Generator(device="cuda").manual_seed(a.seed)
        x = torch.rand((a.points, 4), device="cuda", generator=g)
        x[:, 3] = 0.01
        bvh = Sphere3DLBVH()
        bvh.set_objects_device(x.data_ptr(), a.points, 63, True)
        ts = []
        for _ in range(a.warmup + a.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = bvh.build()
            ts.append(time.perf_counter() - t0)
        best = min(ts[a.warmup:]) if a.steps else min(ts)
        print(json.dumps({"once": "lbvh", "points": a.points, "build_ms_best": round(1e3 * best, 3), "status": st}))
        return 0
    if a.workload == "trbvh":  # TRBVH (treelet 7, 3 rounds) over the meshing-stress cloud of --points
        from stream_b200.geometry import Sphere3DTRBVH
        pts, al = workloads.meshing_stress(a.points, seed=a.seed)
        t = Sphere3DTRBVH()
        t.set_objects(np.concatenate([pts, al[:, None]], 1).astype(np.float32), treelet_size=7, area3d=True,
                      rounds=3)
        t.set_profiling(True)
        st = t.build()
        print(json.dumps({"once": "trbvh", "points": len(pts), "status": st, "stages_ms": t.profile()}))
        return 0
    if a.workload == "uniform2d":  # the reference's uniform2D cloud (glibc srand(42)), alpha 0.0012
        from stream_b200.mesh import AlphaShape2D
        pts, al = workloads.glibc_uniform_square(a.points2d, 0.0012)
        m2 = AlphaShape2D()
        m2.set_nodes(pts, al)
        m2.compute()
        print(json.dumps({"once": "uniform2d", "points": len(pts), "triangles": int(len(m2.get_elem()))}))
        return 0
    if a.workload == "delaunay2d":  # Mesh2D over --points2d uniform points, all phases
        from stream_b200.mesh import Mesh2D
        xy = np.random.default_rng(a.seed).random((a.points2d, 2)).astype(np.float32)
        m2 = Mesh2D()
        m2.set_nodes(xy)
        m2.insert_morton_neighbors()
        m2.insert_BVH_neighbors()
        m2.insert_iterative()
        m2.remove_super_nodes()
        print(json.dumps({"once": "delaunay2d", "points": len(xy), "triangles": int(len(m2.get_elem())),
                          **m2.counters()}))
        return 0
    if a.workload == "uniform":
        pts, al = workloads.uniform_cube(a.points, seed=a.seed)
    else:
        pts, al = workloads.meshing_stress(a.points, seed=a.seed)
    m = AlphaShape3D()
    m.set_nodes(pts, al)
    m.compute()
    print(json.dumps({"once": a.workload, "points": len(pts), "tets": int(len(m.get_elem()))}))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--points", type=int, default=4_000_000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=200_000,
                    help="points (at least) of the corner of the cloud timed on the host and on the GPU")
    ap.add_argument("--solve-h", type=float, default=0.005)
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--heldout-points", type=int, default=4_000_000,
                    help="held-out dam-break system for the FSAI vs Jacobi comparison (0: skip)")
    ap.add_argument("--pfem-points", type=int, default=4_000_000)
    ap.add_argument("--pfem-steps", type=int, default=100, help="PFEM loop steps timed (0: skip)")
    ap.add_argument("--pfem-dyn-points", type=int, default=1_000_000, help="particles of the fractional-step dam break")
    ap.add_argument("--pfem-dyn-steps", type=int, default=20, help="fractional-step dam-break steps (0: skip)")
    ap.add_argument("--plain-points", type=int, default=200_000,
                    help="plain-method chain: uniform cloud, 30-bit codes, P1 assembly, FP64 PCG to 1e-10 (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--points2d", type=int, default=1_000_000, help="2D alpha-shape cloud size (0: skip)")
    ap.add_argument("--points-delaunay2d", type=int, default=1_000_000, help="2D Delaunay (Mesh2D) cloud size (0: skip)")
    ap.add_argument("--trbvh", type=int, default=1, help="time the TRBVH over the cloud (0: skip)")
    ap.add_argument("--lbvh-points", type=int, default=64 * 1024 * 1024,
                    help="device-resident LBVH build of this many spheres (0: skip)")
    ap.add_argument("--uniform3d", type=int, default=1, help="time the uniform3D harness clouds (0: skip)")
    ap.add_argument("--workload", choices=["stress", "uniform", "solve", "pfem", "pfemdyn", "lbvh", "trbvh",
                                           "uniform2d", "delaunay2d"],
                    default="stress",
                    help="--once workload: a remesh of the stress or uniform cloud, dam-break solves (learned FSAI, KY-FSAI, FP64 Jacobi), "
                         "three PFEM steps, Sphere3DLBVH builds over --points device points (--warmup, --steps), "
                         "three fractional-step dam-break steps (--pfem-dyn-points), "
                         "one TRBVH build over the stress cloud, the uniform2D cloud, or a 2D Delaunay "
                         "triangulation (Mesh2D) of --points2d uniform points")
    ap.add_argument("--once", action="store_true",
                    help="one remesh of the workload and exit (a driver for profiler captures)")
    a = ap.parse_args(argv)
    if a.once:
        return run_once(a)
    if a.warmup < 3 and a.impl == "ours":
        print("bench.py: warm-up below 3 is not a valid measurement", file=sys.stderr)
    if a.impl == "reference":
        return bench_reference_arm(a)
    return bench_ours(a)


if __name__ == "__main__":
    sys.exit(main())
