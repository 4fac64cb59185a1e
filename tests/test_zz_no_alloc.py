"""Allocation-free occupancy entry point (ovx_fdg_occupancy_noalloc).

Some hosts cannot let a library allocate device memory (an application that
gives all device memory to its own pool at start-up, a plugin host whose
allocator owns the device, a latency-critical thread that must not hit the
synchronisation cudaMalloc/cudaFree can imply).  This entry point uses only a
fixed scratch array inside the library.  Its results must equal those of the
allocating occupancy entry point, on consecutive calls that share the scratch.
This file is collected last on purpose.
"""
import numpy as np
import pytest

import fdg_workloads as W
from oracle import oracle as O


def _soup(w):
    v, f, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
    return np.ascontiguousarray(v[f.astype(np.int64)]), vs, gr


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point(cuda):
    import torch
    import ovx_fdg_abi as abi

    cases = [W.ico_cap(0), W.ico_cap(3)] + [c for c in W.small_cases() if c.name != "empty"]
    ctx = abi.Context(cuda.index or 0)
    try:
        for w in cases:
            tri, vs, gr = _soup(w)
            t = torch.from_numpy(tri).to(cuda)
            want = ctx.occupancy(t, vs, gr).cpu().numpy()
            for call in range(2):  # consecutive calls share (and must clear) the scratch
                rc, n, got = abi.occupancy_noalloc(t, vs, gr)
                torch.cuda.synchronize()
                assert rc == abi.OK, (w.name, call, rc)
                assert n == want.shape[0], (w.name, call, n, want.shape[0])
                assert np.array_equal(got.cpu().numpy(), want), (w.name, call)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_noalloc_grid_256_and_limits(cuda):
    import torch
    import ovx_fdg_abi as abi

    w = W.primitives(5, faces_total=20_000)
    w = W.Workload(w.name, w.vertices, w.faces, 256, w.aabb)
    tri, vs, gr = _soup(w)
    t = torch.from_numpy(tri).to(cuda)
    ctx = abi.Context(cuda.index or 0)
    try:
        want = ctx.occupancy(t, vs, gr).cpu().numpy()
    finally:
        ctx.close()
    for _ in range(2):
        rc, n, got = abi.occupancy_noalloc(t, vs, gr)
        torch.cuda.synchronize()
        assert rc == abi.OK and n == want.shape[0]
        assert np.array_equal(got.cpu().numpy(), want)
    # output buffer too small: CAPACITY, N reported, nothing written
    rc, n, _ = abi.occupancy_noalloc(t, vs, gr, capacity=want.shape[0] - 1)
    assert rc == 5 and n == want.shape[0]
    # grid beyond the fixed scratch (64^3 bricks > 32768): CAPACITY
    big = np.array([1.0 / 512] * 3, np.float32)
    rc, n, _ = abi.occupancy_noalloc(t, big, [0, 0, 0, 512, 512, 512])
    assert rc == 5 and n == 0


@pytest.mark.gpu
def test_noalloc_brick_limit_exact_and_one_over(cuda):
    """A non-cubic grid of exactly 32768 bricks (64 x 32 x 16, so the row-base
    slot right after the bitmap is in use) matches the allocating entry point;
    one brick more (3 x 11 x 993 = 32769) is refused with CAPACITY."""
    import torch
    import ovx_fdg_abi as abi

    w = W.primitives(6, faces_total=20_000)
    w = W.Workload(w.name, w.vertices, w.faces, [512, 256, 128], w.aabb)
    tri, vs, gr = _soup(w)
    assert (gr[3] // 8) * (gr[4] // 8) * (gr[5] // 8) == 32768
    t = torch.from_numpy(tri).to(cuda)
    ctx = abi.Context(cuda.index or 0)
    try:
        want = ctx.occupancy(t, vs, gr).cpu().numpy()
    finally:
        ctx.close()
    assert want.shape[0] > 0
    for _ in range(2):
        rc, n, got = abi.occupancy_noalloc(t, vs, gr)
        torch.cuda.synchronize()
        assert rc == abi.OK and n == want.shape[0]
        assert np.array_equal(got.cpu().numpy(), want)
    rc, n, _ = abi.occupancy_noalloc(t, vs, [0, 0, 0, 24, 88, 7944])
    assert rc == 5 and n == 0


@pytest.mark.gpu
def test_noalloc_lowpoly_grid_256(cuda):
    """Large triangles (a low-poly soup on a 256^3 grid): each (triangle, axis)
    pair is scanned by one thread here, so this is the slow case of this entry
    point; results still equal the allocating entry point's."""
    import torch
    import ovx_fdg_abi as abi

    w = W.lowpoly(5, faces_total=600, grid_size=256)
    tri, vs, gr = _soup(w)
    t = torch.from_numpy(tri).to(cuda)
    ctx = abi.Context(cuda.index or 0)
    try:
        want = ctx.occupancy(t, vs, gr).cpu().numpy()
    finally:
        ctx.close()
    for _ in range(2):
        rc, n, got = abi.occupancy_noalloc(t, vs, gr)
        torch.cuda.synchronize()
        assert rc == abi.OK and n == want.shape[0]
        assert np.array_equal(got.cpu().numpy(), want)
