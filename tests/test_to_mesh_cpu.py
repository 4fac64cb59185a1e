"""flexible_dual_grid_to_mesh, CPU side: the numpy restatement
(oracle/fdg_mesh_oracle.py) against the golden outputs of the reference's own
Python function (tests/golden/to_mesh.npz, tests/golden/make_to_mesh_golden.py),
and the CPU restatement of the reference hashmap on hand cases."""
import os

import numpy as np
import pytest
import torch

from oracle import fdg_mesh_oracle as M
from oracle import ref_hashmap_cpu as H

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "to_mesh.npz")
MODES = ("alignment", "split_weight", "train")


def golden_case(z, name, mode):
    """(coords, dual, flags, split_weight or None, grid, voxel_size, aabb_min) and the expected (vertices, triangles)."""
    g = z[f"{name}/grid"]
    aabb = z[f"{name}/aabb"]
    vs = ((aabb[1] - aabb[0]) / g.astype(np.float32)).astype(np.float32)  # float32, as the reference divides
    sw = None if mode == "alignment" else z[f"{name}/split_weight"]
    verts = z[f"{name}/vertices"]
    if mode == "train":
        verts = np.concatenate([verts, z[f"{name}/train/mid_vertices"]])
    args = (z[f"{name}/coords"], z[f"{name}/dual"], z[f"{name}/flags"], sw, g, vs, aabb[0])
    return args, (verts, z[f"{name}/{mode}/triangles"])


def _cases():
    z = np.load(GOLDEN)
    return [(str(n), m) for n in z["cases"] for m in MODES]


@pytest.mark.parametrize("name,mode", _cases())
def test_restatement_matches_reference_function(name, mode):
    z = np.load(GOLDEN)
    args, (want_v, want_t) = golden_case(z, name, mode)
    v, t = M.to_mesh(*args, train=mode == "train")
    assert np.array_equal(v.view(np.uint32), want_v.view(np.uint32))
    assert np.array_equal(t, want_t)


def test_golden_covers_out_of_grid_neighbours():
    """The hand case has intersected edges whose neighbours lie past the last
    grid layer: the reference finds no quad there."""
    z = np.load(GOLDEN)
    c = z["edge_layers/coords"]
    g = int(z["edge_layers/grid"][0])
    flags = z["edge_layers/flags"]
    nbr = M.EDGE_NBR[None] + c[:, None, None, :]
    outside = ((nbr < 0) | (nbr >= g)).any(-1).any(-1)  # [N,3]
    assert (outside & flags).any()
    # keys of those neighbours alias in-grid voxels that are active: a flat-key
    # lookup without the bounds check would have produced extra quads
    assert z["edge_layers/alignment/triangles"].shape[0] == 4


def test_hashmap_restatement_semantics():
    keys = torch.full((16,), 0xFFFFFFFF, dtype=torch.uint32)
    vals = torch.empty((16,), dtype=torch.uint32)
    coords = torch.tensor([[0, 1, 1, 3], [0, 1, 2, 0], [0, 3, 3, 3]], dtype=torch.int32)
    H.clear()
    H.hashmap_insert_3d_idx_as_val_cuda(keys, vals, coords, 4, 4, 4)
    q = torch.tensor([[0, 1, 1, 3], [0, 1, 1, 4], [0, 1, 2, 0], [0, 3, 3, 3], [0, -1, 0, 0], [0, 2, 2, 2]], dtype=torch.int32)
    got = H.hashmap_lookup_3d_cuda(keys, vals, q, 4, 4, 4).numpy().astype(np.int64)
    # (1,1,4) is outside the grid although its flat key equals (1,2,0)'s
    assert got.tolist() == [0, 0xFFFFFFFF, 1, 2, 0xFFFFFFFF, 0xFFFFFFFF]
