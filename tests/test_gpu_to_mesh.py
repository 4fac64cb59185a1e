"""flexible_dual_grid_to_mesh on the GPU against the numpy restatement of the
reference (oracle/fdg_mesh_oracle.py): vertices bit for bit, the same quads
in the same order and the same split of each."""
import numpy as np
import pytest

import fdg_workloads as W
from oracle import fdg_mesh_oracle as M


def _fdg(w, cuda):
    import torch
    import o_voxel

    v = torch.from_numpy(w.vertices).to(cuda)
    f = torch.from_numpy(w.faces).to(cuda)
    return o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["alignment", "split_weight", "train"])
@pytest.mark.parametrize("name", ["ico_cap", "primitives60k"])
def test_to_mesh_matches_oracle(cuda, name, mode):
    import torch
    import o_voxel

    w = W.ico_cap(0) if name == "ico_cap" else W.primitives(2, faces_total=60_000)
    vox, dual, inter = _fdg(w, cuda)
    g = w.grid_size
    vs = (np.float32(1.0) / np.float32(g))
    # dual vertices as in-voxel offsets (the convention this function takes)
    rel = (dual / torch.tensor(vs, device=cuda) - vox.float()).clamp(0, 1)
    sw = None
    if mode != "alignment":
        sw = torch.rand(vox.shape[0], 1, device=cuda, generator=torch.Generator(cuda).manual_seed(3)) + 0.05
    verts, tris = o_voxel.convert.flexible_dual_grid_to_mesh(vox, rel, inter, sw, W.UNIT_AABB, grid_size=g,
                                                             train=mode == "train")
    want_v, want_t = M.to_mesh(vox.cpu().numpy(), rel.cpu().numpy(), inter.cpu().numpy(),
                               None if sw is None else sw.cpu().numpy(), [g, g, g], [vs, vs, vs], [-0.5, -0.5, -0.5],
                               train=mode == "train")
    assert verts.dtype == torch.float32 and tris.dtype == torch.int32
    assert np.array_equal(verts.cpu().numpy().view(np.uint32), want_v.view(np.uint32))
    assert tris.shape[0] > 0
    assert np.array_equal(tris.cpu().numpy(), want_t)


@pytest.mark.gpu
def test_to_mesh_key_aliasing_and_empty(cuda):
    """A neighbour one past the last z aliases voxel (x, y+1, 0) through the flat
    key, as in the reference's hashmap; an empty grid gives an empty mesh."""
    import torch
    import o_voxel

    g = 4
    coords = np.array([[1, 1, 3], [1, 2, 0], [1, 2, 3], [1, 3, 0], [2, 2, 2]], dtype=np.int32)
    flags = np.zeros((5, 3), dtype=bool)
    flags[0, 0] = True  # x-edge of (1,1,3): neighbours (1,1,4)->(1,2,0), (1,2,4)->(1,3,0), (1,2,3)
    dual = np.full((5, 3), 0.5, dtype=np.float32)
    c = torch.from_numpy(coords).to(cuda)
    verts, tris = o_voxel.convert.flexible_dual_grid_to_mesh(c, torch.from_numpy(dual).to(cuda),
                                                             torch.from_numpy(flags).to(cuda), None,
                                                             [[0, 0, 0], [1, 1, 1]], grid_size=g)
    want_v, want_t = M.to_mesh(coords, dual, flags, None, [g, g, g], [0.25] * 3, [0, 0, 0])
    assert want_t.shape[0] == 2  # the aliased quad exists in the reference semantics
    assert np.array_equal(tris.cpu().numpy(), want_t)
    assert np.array_equal(verts.cpu().numpy(), want_v)
    e = torch.zeros((0, 3), dtype=torch.int32, device=cuda)
    v0, t0 = o_voxel.convert.flexible_dual_grid_to_mesh(e, e.float(), e.bool(), None, [[0, 0, 0], [1, 1, 1]], grid_size=8)
    assert v0.shape == (0, 3) and t0.shape == (0, 3)
