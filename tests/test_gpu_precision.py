"""Compensated precision mode (precision='compensated'): occupancy and flags
equal the exact mode's, and the dual vertices come closer to the FP64
restatement of the same algorithm.  Prints, per config, the error of both
modes against FP64 and against the reference CPU path (in voxel edges) and
the share of voxels solved in FP64."""
import json

import numpy as np
import pytest

import fdg_workloads as W
from fdg_check import canon
from oracle import oracle as O


def _run(w, cuda, precision):
    import torch
    import ovx_fdg_abi as abi

    ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
    g = np.broadcast_to(np.asarray(w.grid_size, np.int32), (3,))
    vs = ((ab[1] - ab[0]) / g.astype(np.float32)).astype(np.float32)
    ctx = abi.Context(cuda.index or 0)
    try:
        ctx.set_precision(precision)
        out = ctx.mesh_to_fdg(torch.from_numpy(w.vertices).to(cuda), torch.from_numpy(w.faces).to(cuda), ab[0], vs,
                              [0, 0, 0, int(g[0]), int(g[1]), int(g[2])], w.face_weight, w.boundary_weight,
                              w.regularization_weight)
        routed = ctx.last_counts()["routed_fp64"]
        return tuple(t.cpu().numpy() for t in out), routed
    finally:
        ctx.close()


def _err(a, b, w):
    ab = np.asarray(w.aabb, np.float64).reshape(2, 3)
    edge = (ab[1] - ab[0]) / np.asarray(w.grid_size, np.float64)
    e = np.sqrt((((a.astype(np.float64) - b.astype(np.float64)) / edge) ** 2).sum(1))
    return {"rms": float(np.sqrt((e ** 2).mean())), "max": float(e.max()), "share_above_1e-2": float((e > 1e-2).mean()),
            "share_above_1e-4": float((e > 1e-4).mean())}


def _check(w, cuda):
    (ev, ed, ei), _ = _run(w, cuda, 0)
    (cv, cd, ci), routed = _run(w, cuda, 1)
    ev, ed, ei = canon(ev, ed, ei)
    cv, cd, ci = canon(cv, cd, ci)
    assert np.array_equal(ev, cv) and np.array_equal(ei, ci), "occupancy or flags changed"
    r64 = O.run_workload(w, "f64")
    dv, dd, _ = canon(r64.voxels, r64.dual, r64.intersected)
    assert np.array_equal(dv, ev)
    stats = {"workload": w.name, "grid": w.grid_size, "faces": w.num_faces, "voxels": int(ev.shape[0]),
             "exact_vs_fp64": _err(ed, dd, w), "compensated_vs_fp64": _err(cd, dd, w),
             "compensated_vs_cpu": _err(cd, ed, w), "routed_fp64_share": routed / max(1, ev.shape[0])}
    print("precision:", json.dumps(stats))
    assert stats["compensated_vs_fp64"]["rms"] < stats["exact_vs_fp64"]["rms"]
    assert stats["compensated_vs_fp64"]["max"] <= np.sqrt(3.0) + 1e-6
    return stats


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ico_cap", "primitives"])
def test_compensated_closer_to_fp64(cuda, name):
    _check(W.ico_cap(0) if name == "ico_cap" else W.primitives(1), cuda)


@pytest.mark.gpu
@pytest.mark.slow
def test_compensated_precision_stress_sheets(cuda):
    """The precision-stress config: 200k faces of near-coplanar sheets, creases
    and slivers at grid 1024."""
    _check(W.sheets(3), cuda)


@pytest.mark.gpu
def test_compensated_batch_equals_single(cuda):
    import torch
    import o_voxel

    ws = W.batch(seed=9, n_meshes=4, f_lo=2_000, f_hi=30_000, grids=(64, 128))
    meshes = [(torch.from_numpy(w.vertices).to(cuda), torch.from_numpy(w.faces).to(cuda)) for w in ws]
    kw = dict(face_weight=1.0, boundary_weight=0.2, regularization_weight=1e-2, precision="compensated")
    outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch(meshes, grid_size=[w.grid_size for w in ws],
                                                            aabb=[w.aabb for w in ws], **kw)
    for w, (v, f), out in zip(ws, meshes, outs):
        single = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=w.grid_size, aabb=w.aabb, **kw)
        for a, b in zip(out, single):
            assert torch.equal(a, b), w.name
