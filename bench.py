#!/usr/bin/env python
"""Benchmark of the PFEM remesh-and-solve path on B200.

One step = one remesh of the 4M-point meshing-stress cloud (Karras LBVH with
63-bit Morton codes + 3D alpha shape with exact predicates, free-surface
flags and CSR output), inputs resident in HBM.  The line also carries:
  e2e           the same metric through the public host API (AlphaShape3D_set_nodes
                from pinned host memory ... AlphaShape3D_get_elem into pinned host memory)
  roofline      of the dominant kernel, from live per-stage CUDA-event timings;
                "alu" holds the star pass against the FP32 peak from its counted
                insphere work (AlphaShape3D_get_work)
  cpu_baseline  the reference's own sources (oracle/_ref) on the host cores,
                on a bounded spatial sample of the same cloud
  solve         the dam-break pressure solve (FP64 Jacobi-PCG vs mixed precision)
  pfem          the 4M-particle PFEM step loop
  remesh2d      the 2D alpha shape on the reference's uniform2D 1M cloud
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


def cpu_sample(pts: np.ndarray, alpha: np.ndarray, target: int):
    """Spatial sub-cube of the cloud holding ~target points (same alpha, so the
    same local density and neighbour counts as the full workload)."""
    lo = pts.min(axis=0)
    hi = pts.max(axis=0)
    for s in np.linspace(0.2, 1.0, 33):
        box_hi = lo + s * (hi - lo)
        m = np.all(pts <= box_hi, axis=1)
        if m.sum() >= target:
            return np.ascontiguousarray(pts[m]), np.ascontiguousarray(alpha[m]), float(s)
    return pts, alpha, 1.0


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


def run_cpu_reference(pts, alpha, steps: int, warmup: int):
    """The reference's own sources built for the host (oracle/_ref) with all
    host threads; falls back to the plain-C restatement if absent."""
    from oracle.oracle import Reference, Restatement
    kind = "reference"
    try:
        ref = Reference()
        fn0 = lambda: ref.ashape3d(pts, alpha)  # noqa: E731
    except FileNotFoundError:
        kind = "port"
        r = Restatement()
        fn0 = lambda: r.ashape3d(pts, alpha)  # noqa: E731

    def fn():
        with _QuietStdout():
            fn0()
    for _ in range(warmup):
        fn()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return kind, ts


def bench_reference_arm(a):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from stream_b200 import workloads
    pts, alpha = workloads.meshing_stress(a.points, seed=a.seed)
    sp, sa, frac = cpu_sample(pts, alpha, a.cpu_sample)
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    kind, ts = run_cpu_reference(sp, sa, a.steps, a.warmup)
    ms = 1e3 * statistics.median(ts)
    val = len(sp) / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": UNIT, "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"meshing-stress cloud, spatial sample of {len(sp)} of {a.points} points "
                               f"(sub-cube fraction {frac:.3f}, same alpha), reference CPU path",
                   "points": len(sp), "alpha": float(sa[0])},
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                         "kind": kind,
                         "sample": f"{len(sp)} points of the 4M meshing-stress cloud (sub-cube), median of {a.steps}"},
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
    # Star kernel (dominant): per point it reads its candidate list once (4 B x
    # candidates), its coordinates (16 B) and writes its outputs (masks 32 B,
    # counts 10 B); everything else stays on chip or in L1.  Algorithmic bytes
    # per point are tiny, so its HBM fraction is low: it is FP32-ALU bound.
    star_bytes = n * (4 * 70 + 16 + 42)
    dom = max(range(len(names)), key=lambda i: prof[i])
    dom_name = names[dom]
    if dom_name == "radix_sort":
        ach, traffic_note = sort_gbs, sort_bytes
    else:
        ach = star_bytes / (prof[dom] / 1e3) / 1e9
    # The star pass is bound by FP32 arithmetic, not HBM: its counted work
    # against the FP32 peak (148 SMs x 128 lanes x 2 flops x the SM clock
    # sampled during the timed steps).
    sm_mhz = float((clocks or {}).get("sm_mhz") or 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    star_flops32 = 117.0 * float(work[0])
    star_flops64 = 117.0 * float(work[1])
    alu_ach = (star_flops32 + star_flops64) / (prof[4] / 1e3) / 1e12
    alu = {"kernel": "star", "achieved": round(alu_ach, 2), "peak": round(fp32_peak, 1), "unit": "TFLOP/s",
           "frac": round(alu_ach / fp32_peak, 4),
           "peak_kind": f"nominal FP32 at the sampled SM clock ({sm_mhz:.0f} MHz)",
           "insphere_tests": int(work[0]), "fp64_filter_evals": int(work[1]), "flops_per_test": 117,
           "ms_per_launch": round(float(prof[4]), 4)}
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(ach / hbm, 4), "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": star_bytes if dom_name != "radix_sort" else sort_bytes,
                "ms_per_launch": round(float(prof[dom]), 4),
                "sort": {"achieved": round(sort_gbs, 1), "frac": round(sort_gbs / hbm, 4), "ms": round(float(prof[1]), 4),
                         "algorithmic_bytes": sort_bytes},
                "alu": alu}

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
                                   methods=(("fp64_jacobi_pcg", 0), ("fsai_mixed_ir", 2)), reps=2)
    if a.pfem_steps:
        pfem = bench_pfem(a)
    remesh2d = bench_remesh2d(a, torch) if a.points2d else None

    # ---- CPU baseline ----------------------------------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        sp, sa, frac = cpu_sample(pts, alpha, a.cpu_sample)
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        kind, ts = run_cpu_reference(sp, sa, steps=3, warmup=1)
        cms = 1e3 * statistics.median(ts)
        cpu = {"value": round(len(sp) / (cms / 1e3) / 1e6, 4), "unit": UNIT,
               "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
               "sample": f"{len(sp)} points of the same cloud (sub-cube {frac:.3f} of the box, same alpha), "
                         f"median of 3 after 1 warm-up, {cms:.0f} ms each"}

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "meshing-stress cloud: 60% uniform in [0,1]^3, 30% in 32 Gaussian blobs "
                               "(sigma 0.01), 10% distinct 100^3 lattice sites; alpha = 1.5 N^-1/3; "
                               "63-bit Morton LBVH + 3D alpha shape (exact predicates)",
                   "points": n, "alpha": float(alpha[0]), "tets": int(n_elems),
                   "l2": "256 MiB write between timed steps", "parallelism": f"replicas x{ws}"},
        "roofline": roofline, "stages_ms": stages, "rates": rates, "counters": counters, "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches, "gpu_launches_per_step": launches // max(1, a.steps), "clocks": clocks,
        "solve": solve,
        "solve_heldout": solve_4m,
        "pfem": pfem,
        "remesh2d": remesh2d,
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


def bench_solve(a, torch, stream, h=None, methods=(("fp64_jacobi_pcg", 0), ("mixed_ir", 1), ("fsai_mixed_ir", 2)),
                reps=2):
    """Dam-break pressure system: remesh, assemble, then FP64 Jacobi-PCG,
    Jacobi mixed-precision refinement and learned-FSAI mixed-precision
    refinement (the network shipped with the package) to ||b - Ax|| <= 1e-8
    ||b||.  Each solve starts from x = 0; the FSAI time includes the
    preconditioner's set-up and network inference on this system."""
    from stream_b200.numerics import FsaiModel
    h = a.solve_h if h is None else h
    ps = _dambreak_system(h, a.seed)
    n, nnz = ps.size()
    out = {"workload": f"dam-break column 0.4x0.8x0.4, h={h:.6g}, jitter 0.1h, alpha=1.2h, "
                       f"RHS = div u (8 Fourier modes), free surface p=0", "n": n, "nnz": nnz}
    model = FsaiModel.trained()
    x64 = None
    for name, method in methods:
        rs = []
        for _ in range(reps):
            if method == 2:
                ps.set_fsai(model)  # rebuilds the preconditioner (set-up + inference) inside the timed solve
            x, rep = ps.solve(method=method, rtol=1e-8)
            if method == 2:
                rep.update({k: v for k, v in ps.fsai_stats().items() if k != "fallback"})
            rs.append(rep)
        rep = min(rs, key=lambda r: r["ms"])
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
    base = out["fp64_jacobi_pcg"]["s"]
    if "mixed_ir" in out:
        out["mixed_over_fp64_time"] = round(out["mixed_ir"]["s"] / base, 4)
    out["fsai_mixed_over_fp64_time"] = round(out["fsai_mixed_ir"]["s"] / base, 4)
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
    if a.workload == "solve":
        from stream_b200.numerics import FsaiModel, PoissonSystem
        ps = _dambreak_system(a.solve_h, a.seed)
        ps.set_fsai(FsaiModel.trained())
        _, r2 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=1e-8)
        _, r0 = ps.solve(method=PoissonSystem.FP64_JACOBI, rtol=1e-8)
        print(json.dumps({"once": "solve", "n": ps.size()[0], "fsai_mixed": r2, "fp64_jacobi": r0}))
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
    if a.workload == "uniform2d":  # the reference's uniform2D cloud (glibc srand(42)), alpha 0.0012
        from stream_b200.mesh import AlphaShape2D
        pts, al = workloads.glibc_uniform_square(a.points2d, 0.0012)
        m2 = AlphaShape2D()
        m2.set_nodes(pts, al)
        m2.compute()
        print(json.dumps({"once": "uniform2d", "points": len(pts), "triangles": int(len(m2.get_elem()))}))
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
    ap.add_argument("--cpu-sample", type=int, default=200_000)
    ap.add_argument("--solve-h", type=float, default=0.005)
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--heldout-points", type=int, default=4_000_000,
                    help="held-out dam-break system for the FSAI vs Jacobi comparison (0: skip)")
    ap.add_argument("--pfem-points", type=int, default=4_000_000)
    ap.add_argument("--pfem-steps", type=int, default=5, help="PFEM loop steps timed (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--points2d", type=int, default=1_000_000, help="2D alpha-shape cloud size (0: skip)")
    ap.add_argument("--workload", choices=["stress", "uniform", "solve", "pfem", "lbvh", "uniform2d"], default="stress",
                    help="--once workload: a remesh of the stress or uniform cloud, one pair of dam-break solves, "
                         "three PFEM steps, or Sphere3DLBVH builds over --points device points (--warmup, --steps)")
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
