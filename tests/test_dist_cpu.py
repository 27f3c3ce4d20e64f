"""CPU, world size 2 over gloo (127.0.0.1): the multi-GPU path of bench.py is
independent replicas (the remesh and the solve do not shard), so what crosses
ranks is the timing rule -- the slowest replica's step time, as a max over
ranks -- and the whole-job rate computed from it; and the reference arm, which
only rank 0 runs."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(100.0 + 25.0 * rank, dist, device="cpu")  # rank 1 is the slow replica
        rate = bench.replica_rate(world, 4_000_000, ms)
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in out:
        assert ms == 125.0                       # every rank sees the slowest replica
        assert rate == pytest.approx(2 * 4_000_000 / 0.125 / 1e6)


def test_single_process_timing_is_identity():
    import bench
    assert bench.max_over_ranks(7.5, None) == 7.5
    assert bench.replica_rate(1, 1_000_000, 10.0) == pytest.approx(100.0)


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    """Under torchrun only rank 0 runs the CPU reference; the others exit 0."""
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class A:
        points, seed, cpu_sample, steps, warmup = 4_000_000, 0, 1000, 1, 0
    assert bench.bench_reference_arm(A()) == 0


def test_reference_arm_does_not_map_the_library():
    """bench.py --impl reference times the reference's own sources only: the
    process never maps stream_b200's CUDA library, and its config equals the
    GPU arm's."""
    import json
    import os
    import subprocess
    import sys
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, json; sys.argv = ['bench.py']; import bench;"
            "bench.main(['--impl', 'reference', '--points', '40000', '--cpu-sample', '3000', '--steps', '1', "
            "'--warmup', '0']);"
            "maps = open('/proc/self/maps').read();"
            "print('MAPPED' if 'libstream_b200' in maps else 'CLEAN'); print('MOD' if 'stream_b200' in sys.modules else 'NOMOD')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=root, check=True,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    import bench
    line = json.loads(next(ln for ln in lines if ln.startswith("{")))
    assert lines[-2:] == ["CLEAN", "NOMOD"], lines[-2:]
    assert line["impl"] == "reference"
    assert line["config"] == bench.workload_config(40000, line["config"]["alpha"], 1)
