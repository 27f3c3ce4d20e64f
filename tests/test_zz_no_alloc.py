"""stream_b200_conflict_batch_noalloc: the conflict predicate for callers that
cannot allocate device memory.

A host program that hands the library only device buffers it already owns (a
fixed memory budget or its own pool), or a plugin loaded into one, cannot
call cudaMalloc.  This entry point takes the caller's device arrays and keeps
the exact stage's scratch in a fixed device array, so it allocates nothing.
The test checks it on two calls in a row against the allocating entry point,
stream_b200_conflict_batch (bit for bit), and against the oracle's conflict
decision (the sign of the reference's det), and that a batch above the
256-quintuple limit is refused.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = ctypes.c_void_p


def _quintuples(rng, m):
    """Hard cases: exactly co-spherical cube corners (exact stage + SoS), one-ulp
    perturbations of them, coordinates near the origin, and random points."""
    cube = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]], float)
    out = []
    while len(out) < m:
        kind = len(out) % 4
        sel = rng.choice(8, 5, replace=False)
        if kind == 0:
            p = cube[sel] * rng.choice([1 / 99.0, 0.37, 1.0]) + rng.choice([0.0, 0.5])
        elif kind == 1:
            p = (cube[sel] * 0.1 + rng.random(3) * 0.1).astype(np.float32)
            p[rng.integers(0, 5)] = np.nextafter(p[rng.integers(0, 5)], np.float32(1.0))
        elif kind == 2:
            p = cube[sel] * (3 / 99.0)
        else:
            p = rng.random((5, 3))
        out.append(np.asarray(p, np.float32))
    pts = np.stack(out).astype(np.float32)
    ids = np.stack([rng.permutation(10_000)[:5] for _ in range(m)]).astype(np.uint32)
    return pts, ids


def _allocating(lib, pts, ids):
    out = np.zeros(len(pts), np.float32)
    lib.stream_b200_conflict_batch.argtypes = [ctypes.c_uint32, P, P, P]
    rc = lib.stream_b200_conflict_batch(len(pts), pts.ctypes.data_as(P), ids.ctypes.data_as(P),
                                        out.ctypes.data_as(P))
    assert rc == 0
    return out


def test_noalloc_matches_allocating_entry_point(sb, restate):
    import torch
    from stream_b200 import lib
    lib.stream_b200_conflict_batch_noalloc.argtypes = [ctypes.c_uint32, P, P, P, P]
    lib.stream_b200_conflict_batch_noalloc.restype = ctypes.c_int
    rng = np.random.default_rng(2024)
    for call in range(2):  # two calls in a row share (and reuse) the fixed scratch
        pts, ids = _quintuples(rng, 256)
        want = _allocating(lib, pts, ids)
        d_pts = torch.from_numpy(pts).cuda()
        d_ids = torch.from_numpy(ids.view(np.int32)).cuda()
        d_out = torch.full((len(pts),), float("nan"), dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream()
        rc = lib.stream_b200_conflict_batch_noalloc(len(pts), P(d_pts.data_ptr()), P(d_ids.data_ptr()),
                                                    P(d_out.data_ptr()), P(stream.cuda_stream))
        assert rc == 0, (call, rc)
        got = d_out.cpu().numpy()
        # Bit-exact: the same decision procedure (the predicate tests compare
        # decisions; here even the returned values agree exactly).
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), call
        # The oracle's decision (DirectAlphaShape3D.cpp:423-480): conflict iff det > 0.
        ref_det, _ = restate.conflict_batch(pts, ids)
        assert np.array_equal(got > 0, ref_det > 0), call


def test_noalloc_rejects_oversized_batch(sb):
    import torch
    from stream_b200 import STREAM_ST_BAD_INPUT, last_error, lib
    lib.stream_b200_conflict_batch_noalloc.argtypes = [ctypes.c_uint32, P, P, P, P]
    lib.stream_b200_conflict_batch_noalloc.restype = ctypes.c_int
    d = torch.zeros(257 * 15, dtype=torch.float32, device="cuda")
    di = torch.zeros(257 * 5, dtype=torch.int32, device="cuda")
    do = torch.zeros(257, dtype=torch.float32, device="cuda")
    rc = lib.stream_b200_conflict_batch_noalloc(257, P(d.data_ptr()), P(di.data_ptr()), P(do.data_ptr()), None)
    assert rc == STREAM_ST_BAD_INPUT
    assert "256" in last_error()
