"""flexible_dual_grid_to_mesh on the GPU against the reference: the golden
outputs of the reference's own Python function (tests/golden/to_mesh.npz),
the numpy restatement pinned to them (oracle/fdg_mesh_oracle.py) on larger
grids, and the reference's own hashmap kernels (src/hash/hash.cu, built into
oracle/_ref) against the CPU restatement the golden script runs them with."""
import os

import numpy as np
import pytest

import fdg_workloads as W
from oracle import fdg_mesh_oracle as M
from oracle import ref_hashmap_cpu as H
from test_to_mesh_cpu import GOLDEN, MODES, golden_case


def _fdg(w, cuda):
    import torch
    import o_voxel

    v = torch.from_numpy(w.vertices).to(cuda)
    f = torch.from_numpy(w.faces).to(cuda)
    return o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())


def _cases():
    z = np.load(GOLDEN)
    return [(str(n), m) for n in z["cases"] for m in MODES]


@pytest.mark.gpu
@pytest.mark.parametrize("name,mode", _cases())
def test_to_mesh_matches_reference_function(cuda, name, mode):
    import torch
    import o_voxel

    z = np.load(GOLDEN)
    (coords, dual, flags, sw, g, vs, amin), (want_v, want_t) = golden_case(z, name, mode)
    verts, tris = o_voxel.convert.flexible_dual_grid_to_mesh(
        torch.from_numpy(coords).to(cuda), torch.from_numpy(dual).to(cuda), torch.from_numpy(flags).to(cuda),
        None if sw is None else torch.from_numpy(sw).to(cuda), z[f"{name}/aabb"].tolist(), grid_size=g.tolist(),
        train=mode == "train")
    assert verts.dtype == torch.float32 and tris.dtype == torch.int32
    assert np.array_equal(verts.cpu().numpy().view(np.uint32), want_v.view(np.uint32))
    assert np.array_equal(tris.cpu().numpy(), want_t)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["ico_cap", "primitives60k"])
def test_to_mesh_matches_restatement(cuda, name, mode):
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
    assert np.array_equal(verts.cpu().numpy().view(np.uint32), want_v.view(np.uint32))
    assert tris.shape[0] > 0
    assert np.array_equal(tris.cpu().numpy(), want_t)


@pytest.mark.gpu
def test_to_mesh_out_of_grid_neighbours_and_empty(cuda):
    """Neighbours past the last grid layer are absent (the reference's lookup
    bounds-checks them), though their flat keys equal in-grid voxels' keys; an
    empty grid gives an empty mesh."""
    import torch
    import o_voxel

    g = 4
    coords = np.array([[1, 1, 3], [1, 2, 0], [1, 2, 3], [1, 3, 0], [2, 2, 2]], dtype=np.int32)
    flags = np.zeros((5, 3), dtype=bool)
    flags[0, 0] = True  # x-edge of (1,1,3): neighbours (1,1,4), (1,2,4) are outside; their keys equal (1,2,0), (1,3,0)
    dual = np.full((5, 3), 0.5, dtype=np.float32)
    verts, tris = o_voxel.convert.flexible_dual_grid_to_mesh(torch.from_numpy(coords).to(cuda), torch.from_numpy(dual).to(cuda),
                                                             torch.from_numpy(flags).to(cuda), None,
                                                             [[0, 0, 0], [1, 1, 1]], grid_size=g)
    assert tris.shape[0] == 0
    want_v, want_t = M.to_mesh(coords, dual, flags, None, [g, g, g], [0.25] * 3, [0, 0, 0])
    assert want_t.shape[0] == 0
    assert np.array_equal(verts.cpu().numpy(), want_v)
    e = torch.zeros((0, 3), dtype=torch.int32, device=cuda)
    v0, t0 = o_voxel.convert.flexible_dual_grid_to_mesh(e, e.float(), e.bool(), None, [[0, 0, 0], [1, 1, 1]], grid_size=8)
    assert v0.shape == (0, 3) and t0.shape == (0, 3)


def _ref_hash_module():
    import importlib.util

    from oracle import build as B

    if not os.path.exists(B.REF_HASH_SO):
        pytest.skip("reference hashmap not built (needs the reference source tree at build time)")
    spec = importlib.util.spec_from_file_location("hash_ref", B.REF_HASH_SO)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(4, 4, 4), (64, 48, 40), (512, 512, 512)])
def test_reference_hashmap_matches_restatement(cuda, dims):
    """The reference's hashmap kernels (insert 3d idx-as-value, lookup 3d) give the
    same lookups as the CPU restatement the golden script uses, for in-grid
    keys, absent keys and coordinates outside the grid on every side."""
    import torch

    ref = _ref_hash_module()
    W_, H_, D_ = dims
    rng = np.random.default_rng(sum(dims))
    n = min(W_ * H_ * D_ // 2, 20000)
    flat = rng.choice(W_ * H_ * D_, size=n, replace=False)
    xyz = np.stack([flat // (H_ * D_), (flat // D_) % H_, flat % D_], 1).astype(np.int32)
    coords = np.concatenate([np.zeros((n, 1), np.int32), xyz], 1)
    q = np.concatenate([xyz + rng.integers(-1, 2, size=xyz.shape).astype(np.int32),
                        rng.integers(-2, max(dims) + 2, size=(4000, 3)).astype(np.int32)])
    q = np.concatenate([np.zeros((q.shape[0], 1), np.int32), q], 1)
    cap = 2 * n
    keys = torch.full((cap,), 0xFFFFFFFF, dtype=torch.uint32, device=cuda)
    vals = torch.empty((cap,), dtype=torch.uint32, device=cuda)
    ref.hashmap_insert_3d_idx_as_val_cuda(keys, vals, torch.from_numpy(coords).to(cuda), W_, H_, D_)
    got = ref.hashmap_lookup_3d_cuda(keys, vals, torch.from_numpy(q).to(cuda), W_, H_, D_)
    torch.cuda.synchronize()
    kc = torch.full((cap,), 0xFFFFFFFF, dtype=torch.uint32)
    vc = torch.empty((cap,), dtype=torch.uint32)
    H.clear()
    H.hashmap_insert_3d_idx_as_val_cuda(kc, vc, torch.from_numpy(coords), W_, H_, D_)
    want = H.hashmap_lookup_3d_cuda(kc, vc, torch.from_numpy(q), W_, H_, D_)
    assert np.array_equal(got.cpu().numpy().astype(np.int64), want.numpy().astype(np.int64))
