"""Generate to_mesh.npz: golden outputs of the reference's own
o_voxel.convert.flexible_dual_grid_to_mesh (o_voxel/convert/flexible_dual_grid.py:332-477).

The reference function is imported from the reference source tree and run on
CPU tensors.  Its two CUDA hashmap calls (flexible_dual_grid.py:430,437) are
served by the CPU restatement in oracle/ref_hashmap_cpu.py, which a GPU test
pins against the reference's hashmap kernels compiled from src/hash/hash.cu.
Its one device-specific call, ``torch.arange(..., device="cuda")`` in training
mode (flexible_dual_grid.py:474), is served on the CPU.  Everything else is
the reference's own torch code, unmodified.

Inputs: flexible dual grids made by the C oracle from three seeded meshes
(dual vertices given as in-voxel offsets, the convention the function takes),
plus a hand-made grid whose quads touch the last grid layer.  Each case is
run in the three modes (normal-alignment split, split weights, training mode).

Run from the repository root, with the reference source tree at
$OVX_REFERENCE_ROOT:
    OVX_REFERENCE_ROOT=<reference tree> python tests/golden/make_to_mesh_golden.py
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "o-voxel-gpu_b200"))
sys.path.insert(0, REPO)

import torch  # noqa: E402

import fdg_workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref_hashmap_cpu as H  # noqa: E402


class _TorchOnCpu(types.ModuleType):
    """torch, with device="cuda" arguments of arange served on the CPU."""

    def __init__(self):
        super().__init__("torch")

    def __getattr__(self, name):
        return getattr(torch, name)

    @staticmethod
    def arange(*args, **kw):
        if kw.get("device") == "cuda":
            kw["device"] = "cpu"
        return torch.arange(*args, **kw)


def load_reference_function():
    root = os.environ.get("OVX_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set OVX_REFERENCE_ROOT to the reference source tree")
    pkg = types.ModuleType("ovx_reference")
    pkg.__path__ = []
    pkg._C = types.SimpleNamespace(hashmap_insert_3d_idx_as_val_cuda=H.hashmap_insert_3d_idx_as_val_cuda,
                                   hashmap_lookup_3d_cuda=H.hashmap_lookup_3d_cuda)
    conv = types.ModuleType("ovx_reference.convert")
    conv.__path__ = []
    sys.modules["ovx_reference"] = pkg
    sys.modules["ovx_reference.convert"] = conv
    name = "ovx_reference.convert.flexible_dual_grid"
    spec = importlib.util.spec_from_file_location(name, os.path.join(root, "o_voxel", "convert", "flexible_dual_grid.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    mod.torch = _TorchOnCpu()
    return mod.flexible_dual_grid_to_mesh


def fdg_of(w):
    """Oracle conversion of a workload -> (coords, in-voxel offsets, flags, grid, aabb)."""
    r = O.run_workload(w)
    g = w.grid_size
    v, f, vs, gr = O.grid_args(w.vertices, w.faces, g, w.aabb)
    vs = np.asarray(vs, np.float32)
    rel = np.clip((r.dual.astype(np.float32) / vs).astype(np.float32) - r.voxels.astype(np.float32), 0, 1).astype(np.float32)
    return r.voxels.astype(np.int32), rel, r.intersected.astype(bool), g, np.asarray(w.aabb, np.float32)


def tight(w, grid):
    """The workload on its own bounding box, so that voxels reach the last grid layer."""
    lo, hi = w.vertices.min(0), w.vertices.max(0)
    w.aabb = [lo.tolist(), hi.tolist()]
    w.grid_size = grid
    return w


def cases():
    out = []
    ico = W.ico_cap(0)
    ico.grid_size = 40
    out.append(("ico_cap_g40",) + fdg_of(ico))
    out.append(("primitives_tight24",) + fdg_of(tight(W.primitives(2, faces_total=20_000), 24)))
    out.append(("lowpoly_tight28",) + fdg_of(tight(W.lowpoly(5, faces_total=600, grid_size=28), 28)))
    # hand-made: quads around the last z layer and the last y layer of a 4^3 grid
    coords = np.array([[1, 1, 3], [1, 2, 0], [1, 2, 3], [1, 3, 0], [2, 2, 2], [1, 1, 2], [1, 2, 2], [3, 3, 3],
                       [3, 3, 2], [3, 2, 3], [3, 2, 2]], dtype=np.int32)
    flags = np.zeros((coords.shape[0], 3), dtype=bool)
    flags[0, 0] = True
    flags[5, 0] = True
    flags[7, :] = True
    flags[10, 0] = True
    dual = np.random.default_rng(9).random((coords.shape[0], 3)).astype(np.float32)
    out.append(("edge_layers", coords, dual, flags, 4, np.array([[0, 0, 0], [1, 1, 1]], np.float32)))
    return out


def main():
    fn = load_reference_function()
    arrays = {}
    names = []
    for name, coords, dual, flags, g, aabb in cases():
        names.append(name)
        n = coords.shape[0]
        sw = (np.random.default_rng(3).random((n, 1)).astype(np.float32) + np.float32(0.05)).astype(np.float32)
        arrays[f"{name}/coords"] = coords
        arrays[f"{name}/dual"] = dual
        arrays[f"{name}/flags"] = flags
        arrays[f"{name}/split_weight"] = sw
        arrays[f"{name}/grid"] = np.array([g, g, g], np.int32)
        arrays[f"{name}/aabb"] = aabb
        for mode in ("alignment", "split_weight", "train"):
            H.clear()
            verts, tris = fn(torch.from_numpy(coords), torch.from_numpy(dual), torch.from_numpy(flags),
                             None if mode == "alignment" else torch.from_numpy(sw), aabb.tolist(), grid_size=g,
                             train=mode == "train")
            verts = verts.numpy().astype(np.float32)
            if mode == "alignment":
                arrays[f"{name}/vertices"] = verts
            else:
                # the first N vertices are the same in every mode; training mode appends one per quad
                assert np.array_equal(verts[:n].view(np.uint32), arrays[f"{name}/vertices"].view(np.uint32))
                if mode == "train":
                    arrays[f"{name}/train/mid_vertices"] = verts[n:]
            arrays[f"{name}/{mode}/triangles"] = tris.numpy().astype(np.int32)
            print(f"{name:20s} {mode:12s} voxels {n:6d} vertices {verts.shape[0]:6d} triangles {tris.shape[0]:6d}")
    arrays["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "to_mesh.npz"), **arrays)


if __name__ == "__main__":
    main()
