"""Batched conversion (mesh_to_flexible_dual_grid_batch): every mesh's result
must equal the single-mesh API's (same rows, same order) and the oracle's."""
import numpy as np
import pytest

import fdg_workloads as W
from fdg_check import assert_fdg_equal
from oracle import oracle as O


_ORACLE = {}


def _oracle(w, key):
    if key not in _ORACLE:
        r = O.run_workload(w)
        _ORACLE[key] = (r.voxels, r.dual, r.intersected)
    return _ORACLE[key]


def _upload(ws, device):
    import torch

    return [(torch.from_numpy(w.vertices).to(device), torch.from_numpy(w.faces).to(device)) for w in ws]


@pytest.mark.gpu
@pytest.mark.parametrize("group", [0, 400_000])
def test_batch_matches_oracle_and_single(cuda, group):
    """12 meshes in one batched pipeline (group 0), or cut into groups of about
    400k expected records each: every mesh equals the single-mesh API's rows
    and the oracle."""
    import torch
    import o_voxel

    ws = W.batch(seed=7, n_meshes=12, f_lo=500, f_hi=20_000, grids=(64, 128, 256))
    meshes = _upload(ws, cuda)
    kw = dict(face_weight=1.0, boundary_weight=0.2, regularization_weight=1e-2)
    outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch(
        meshes, grid_size=[w.grid_size for w in ws], aabb=[w.aabb for w in ws], max_group_records=group, **kw)
    torch.cuda.synchronize()
    assert len(outs) == len(ws)
    for w, (v, f), out in zip(ws, meshes, outs):
        got = tuple(t.cpu().numpy() for t in out)
        single = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=w.grid_size, aabb=w.aabb, **kw)
        for a, b in zip(got, single):
            assert np.array_equal(a, b.cpu().numpy()), w.name
        assert_fdg_equal(got, _oracle(w, ("batch7", w.name)), w.name)


@pytest.mark.gpu
def test_batch_shared_grid_and_empty(cuda):
    import torch
    import o_voxel

    ws = [W.ico_cap(0), W.ico_cap(1), W.ico_cap(2)]
    meshes = _upload(ws, cuda)
    meshes.append((torch.zeros((0, 3), device=cuda), torch.zeros((0, 3), dtype=torch.int64, device=cuda)))
    outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch(meshes, grid_size=64, aabb=W.UNIT_AABB,
                                                            boundary_weight=0.2, regularization_weight=1e-2)
    torch.cuda.synchronize()
    for w, out in zip(ws, outs[:3]):
        r = O.run_workload(w)
        assert_fdg_equal(tuple(t.cpu().numpy() for t in out), (r.voxels, r.dual, r.intersected), w.name)
    assert all(t.shape[0] == 0 for t in outs[3])
    assert o_voxel.convert.mesh_to_flexible_dual_grid_batch([], grid_size=64, aabb=W.UNIT_AABB) == []


@pytest.mark.gpu
def test_batch_error_is_raised(cuda):
    import torch
    import o_voxel

    good = _upload([W.ico_cap(0)], cuda)[0]
    bad = (torch.rand(4, 3, device=cuda) - 0.5, torch.tensor([[0, 1, 2], [1, 2, 9]], device=cuda))
    with pytest.raises(RuntimeError, match="face index"):
        o_voxel.convert.mesh_to_flexible_dual_grid_batch([good, bad, good], grid_size=32, aabb=W.UNIT_AABB)
    # the pool stays usable
    outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch([good], grid_size=64, aabb=W.UNIT_AABB,
                                                            boundary_weight=0.2, regularization_weight=1e-2)
    w = W.ico_cap(0)
    r = O.run_workload(w)
    assert_fdg_equal(tuple(t.cpu().numpy() for t in outs[0]), (r.voxels, r.dual, r.intersected), "after error")


@pytest.mark.gpu
@pytest.mark.slow
def test_full_256_mesh_batch(cuda):
    """The 256-mesh mixed batch that bench.py times (faces log-uniform 1k-500k,
    grids 64-512, per-mesh aabb): every mesh equals the single-mesh API row for
    row, and a seeded subset -- including every grid-512 mesh of 300k faces or
    more, up to four -- equals the oracle."""
    import torch
    import o_voxel

    ws = W.batch(4)
    meshes = _upload(ws, cuda)
    kw = dict(face_weight=1.0, boundary_weight=0.2, regularization_weight=1e-2)
    outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch(
        meshes, grid_size=[w.grid_size for w in ws], aabb=[w.aabb for w in ws], **kw)
    torch.cuda.synchronize()
    assert len(outs) == len(ws)
    big = [i for i, w in enumerate(ws) if w.grid_size == 512 and w.num_faces >= 300_000][:4]
    assert big, "the batch has grid-512 meshes of 300k faces or more"
    rng = np.random.default_rng(11)
    subset = sorted(set(big) | set(rng.choice(len(ws), size=8, replace=False).tolist()))
    for i, (w, (v, f), out) in enumerate(zip(ws, meshes, outs)):
        single = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=w.grid_size, aabb=w.aabb, **kw)
        for a, b in zip(out, single):
            assert torch.equal(a, b), (i, w.name)
        if i in subset:
            assert_fdg_equal(tuple(t.cpu().numpy() for t in out), _oracle(w, ("batch4", w.name)), w.name)


@pytest.mark.gpu
def test_batch_mixed_index_types_and_z_order(cuda):
    """int32 and int64 faces in one batch, and z-order rows: each mesh equals
    the single-mesh API with the same order."""
    import torch
    import o_voxel

    ws = W.batch(seed=9, n_meshes=6, f_lo=2_000, f_hi=30_000, grids=(64, 128))
    meshes = _upload(ws, cuda)
    meshes = [(v, f.int() if i % 2 else f) for i, (v, f) in enumerate(meshes)]
    kw = dict(face_weight=1.0, boundary_weight=0.2, regularization_weight=1e-2)
    for order in (None, "z_order"):
        outs = o_voxel.convert.mesh_to_flexible_dual_grid_batch(
            meshes, grid_size=[w.grid_size for w in ws], aabb=[w.aabb for w in ws], order=order, **kw)
        for w, (v, f), out in zip(ws, meshes, outs):
            single = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=w.grid_size, aabb=w.aabb, order=order, **kw)
            for a, b in zip(out, single):
                assert torch.equal(a, b), (w.name, order)
