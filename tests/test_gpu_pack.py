"""pack_flexible_dual_grid against the reference example's own torch
expressions (examples/mesh2ovox.py:51-54), evaluated on the same outputs."""
import numpy as np
import pytest

import fdg_workloads as W


@pytest.mark.gpu
def test_pack_matches_reference_expressions(cuda):
    import torch
    import o_voxel

    w = W.primitives(2, faces_total=60_000)
    v = torch.from_numpy(w.vertices).to(cuda)
    f = torch.from_numpy(w.faces).to(cuda)
    vox, dual, inter = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())
    RES = w.grid_size
    du, iu = o_voxel.convert.pack_flexible_dual_grid(vox, dual, inter, RES)
    want_d = (torch.clamp(dual * RES - vox, 0, 1) * 255).type(torch.uint8)
    want_i = (inter[:, 0:1] + 2 * inter[:, 1:2] + 4 * inter[:, 2:3]).type(torch.uint8)
    assert du.dtype == torch.uint8 and iu.dtype == torch.uint8 and iu.shape == (vox.shape[0], 1)
    assert torch.equal(du, want_d)
    assert torch.equal(iu, want_i)
    e = torch.zeros((0, 3), dtype=torch.int32, device=cuda)
    a, b = o_voxel.convert.pack_flexible_dual_grid(e, e.float(), e.bool(), 64)
    assert a.shape == (0, 3) and b.shape == (0, 1)
