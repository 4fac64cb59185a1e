"""GPU parity at full size: the 10.3M-face subdivided mesh at grid 512 and 1024,
a low-poly mesh of large triangles at grid 512 and 1024, and the grid-1024
precision-stress sheets, bit for bit against the CPU oracle.

The sheets case also states the dual-vertex error of the FP32 path (GPU and
CPU alike) against the FP64 restatement of the same algorithm, in voxel edges.
"""
import json

import numpy as np
import pytest

import fdg_workloads as W
from fdg_check import assert_fdg_equal, canon
from oracle import oracle as O


def _gpu_abi(w, device):
    import torch
    import ovx_fdg_abi as abi

    _, _, vs, gr = O.grid_args(w.vertices[:1], w.faces[:1], w.grid_size, w.aabb)
    ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
    ctx = abi.Context(device.index or 0)
    try:
        vt = torch.from_numpy(np.ascontiguousarray(w.vertices)).to(device)
        ft = torch.from_numpy(np.ascontiguousarray(w.faces)).to(device)
        out = ctx.mesh_to_fdg(vt, ft, ab[0], vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        torch.cuda.synchronize()
        return tuple(t.cpu().numpy() for t in out)
    finally:
        ctx.close()


def _oracle(w, precision="f32"):
    r = O.run_workload(w, precision)
    return r.voxels, r.dual, r.intersected


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.parametrize("grid", [512, 1024])
def test_subdivided_10m_faces(cuda, grid):
    w = W.subdivided(1, grid_size=grid)
    assert w.num_faces == 10_299_999
    assert_fdg_equal(_gpu_abi(w, cuda), _oracle(w), f"subdivided grid {grid}")


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [512, 1024])
def test_lowpoly_large_triangles(cuda, grid):
    """About 1200 triangles on a fine grid: nearly every (triangle, axis) pair
    and face box goes through the large-triangle paths, cut into units."""
    w = W.lowpoly(5, grid_size=grid)
    assert_fdg_equal(_gpu_abi(w, cuda), _oracle(w), f"lowpoly grid {grid}")


def fp64_error(w, got):
    """Error of a conversion's dual vertices against the FP64 restatement of
    the same algorithm, per voxel in voxel edges (the FP32 reference CPU path
    has the same error: the GPU result equals it bit for bit)."""
    gv, gd, _ = canon(*got)
    dv, dd, _ = canon(*_oracle(w, "f64"))
    assert np.array_equal(gv, dv), "FP64 restatement has a different occupancy"
    ab = np.asarray(w.aabb, np.float64).reshape(2, 3)
    edge = (ab[1] - ab[0]) / np.asarray(w.grid_size, np.float64)
    per_voxel = np.sqrt((((gd.astype(np.float64) - dd.astype(np.float64)) / edge) ** 2).sum(1))
    return {"workload": w.name, "grid": w.grid_size, "faces": w.num_faces, "voxels": int(gv.shape[0]),
            "rms_voxel": float(np.sqrt((per_voxel ** 2).mean())), "max_voxel": float(per_voxel.max()),
            "p99_voxel": float(np.quantile(per_voxel, 0.99)),
            "frac_above_1e-3": float((per_voxel > 1e-3).mean()),
            "frac_above_1e-2": float((per_voxel > 1e-2).mean())}


@pytest.mark.gpu
@pytest.mark.slow
def test_sheets_grid1024_precision(cuda):
    """The precision-stress case: 200k faces (2000 near-coplanar sheets, 1000
    creases, 20% slivers) at grid 1024, exact against the oracle; its error
    against FP64 is stated."""
    w = W.sheets(3)
    assert w.num_faces == 200_000
    got = _gpu_abi(w, cuda)
    assert_fdg_equal(got, _oracle(w), "sheets grid 1024")
    stats = fp64_error(w, got)
    print("FP32 path vs FP64 restatement:", json.dumps(stats))
    # the dual vertex lies in (or on the faces of) its voxel in both precisions
    assert stats["max_voxel"] <= np.sqrt(3.0) + 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ico_cap", "primitives"])
def test_fp64_error_stated(cuda, name):
    """The dual-vertex error against the FP64 restatement, stated for the
    small CPU-runnable mesh (grid 64) and the 282k-face mesh (grid 512)."""
    w = W.ico_cap(0) if name == "ico_cap" else W.primitives(1)
    got = _gpu_abi(w, cuda)
    assert_fdg_equal(got, _oracle(w), name)
    stats = fp64_error(w, got)
    print("FP32 path vs FP64 restatement:", json.dumps(stats))
    assert stats["max_voxel"] <= np.sqrt(3.0) + 1e-6
