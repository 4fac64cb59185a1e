"""Host-side mirror of the reference wrapper (o_voxel/convert/flexible_dual_grid.py):
argument checks, grid derivation, and the CUDA-only rule."""
import numpy as np
import pytest
import torch

import o_voxel
from o_voxel.convert import flexible_dual_grid as fdg


def test_shape_assertions_match_reference_messages():
    v = torch.zeros(4, 2)
    f = torch.zeros(2, 3, dtype=torch.int64)
    with pytest.raises(AssertionError, match="vertices must have 3 columns"):
        fdg._grid_setup(v, f, None, 8, [[0, 0, 0], [1, 1, 1]])
    with pytest.raises(AssertionError, match="Either voxel_size or grid_size must be provided"):
        fdg._grid_setup(torch.zeros(4, 3), f, None, None, None)
    with pytest.raises(AssertionError, match="faces must be a 2D tensor"):
        fdg._grid_setup(torch.zeros(4, 3), torch.zeros(6, dtype=torch.int64), None, 8, None)


def test_grid_derivation_float32():
    v = torch.rand(10, 3)
    f = torch.zeros(3, 3, dtype=torch.int64)
    aabb = [[-0.5, -0.25, 0.0], [0.5, 0.75, 0.3]]
    _, _, _, aabb_cpu, vs, gr = fdg._grid_setup(v, f, None, [64, 32, 17], aabb)
    a = np.asarray(aabb, np.float32)
    want = ((a[1] - a[0]) / np.array([64, 32, 17], np.float32)).astype(np.float32)
    assert np.array_equal(np.asarray(vs, np.float32), want)
    assert gr == [0, 0, 0, 64, 32, 17]
    # voxel_size form derives grid_size by rounding, as the reference does
    _, _, _, _, vs2, gr2 = fdg._grid_setup(v, f, 0.125, None, [[0, 0, 0], [1, 1, 1]])
    assert gr2 == [0, 0, 0, 8, 8, 8] and vs2 == [0.125] * 3


@pytest.mark.gpu
def test_cuda_metadata_rule(cuda):
    # grid_size without aabb on CUDA inputs needs a device->host read; the reference refuses it
    v = torch.zeros(3, 3, device=cuda)
    f = torch.zeros(1, 3, dtype=torch.int64, device=cuda)
    with pytest.raises(AssertionError, match="CUDA inputs require CPU aabb"):
        fdg._grid_setup(v, f, None, 8, None)


def test_cpu_tensors_rejected():
    v = torch.zeros(3, 3)
    f = torch.tensor([[0, 1, 2]])
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=8, aabb=[[0, 0, 0], [1, 1, 1]])
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        o_voxel.convert.intersect_occ(v, f, grid_size=8, aabb=[[0, 0, 0], [1, 1, 1]])


def test_signature_matches_reference():
    import inspect

    sig = inspect.signature(o_voxel.convert.mesh_to_flexible_dual_grid)
    # the reference's parameters, in order, then this implementation's optional ones
    assert list(sig.parameters) == ["vertices", "faces", "voxel_size", "grid_size", "aabb", "face_weight",
                                    "boundary_weight", "regularization_weight", "timing", "order", "precision",
                                    "route_tolerance"]
    d = {k: p.default for k, p in sig.parameters.items()}
    assert d["face_weight"] == 1.0 and d["boundary_weight"] == 1.0 and d["regularization_weight"] == 0.1
    assert d["order"] is None and d["precision"] is None


def test_precision_argument_checks():
    import torch

    v = torch.zeros((3, 3))
    f = torch.tensor([[0, 1, 2]])
    with pytest.raises(ValueError, match="precision"):
        o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=8, aabb=[[0, 0, 0], [1, 1, 1]], precision="fp16")


def test_order_and_serialize_argument_checks():
    import torch

    v = torch.zeros(3, 3)
    f = torch.tensor([[0, 1, 2]])
    with pytest.raises(ValueError, match="order"):
        o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=8, aabb=[[0, 0, 0], [1, 1, 1]], order="hilbert")
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        o_voxel.serialize.encode_seq(torch.zeros(4, 3, dtype=torch.int32))
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        o_voxel.serialize.encode_seq(torch.zeros(4, 3, dtype=torch.int32), mode="hilbert")
    with pytest.raises(ValueError):
        o_voxel.serialize.decode_seq(torch.zeros(4, dtype=torch.int32), mode="peano")
