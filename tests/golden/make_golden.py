"""Generate the golden fixtures in this directory from the reference's own CPU
implementation (src/convert/flexible_dual_grid.cpp, built into oracle/_ref by
oracle/build.py against the project's Eigen-API shim).

Each fixture stores the grid-local inputs exactly as the reference operator
receives them (float32 shifted vertices, int32 faces, float32 voxel size,
grid range, weights) and the reference outputs in the reference's own row
order (first-touch insertion order): voxel coordinates, dual vertices and
intersected flags, plus the occupancy-only result of intersect_occ_cpu.

Run from the repository root where the reference source tree is available:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "o-voxel-gpu_b200"))
sys.path.insert(0, REPO)

import fdg_workloads as W  # noqa: E402
from oracle import build as B  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    B.build_ref()
    mod = O.ref_module()
    if mod is None:
        raise SystemExit("reference CPU implementation not built (needs the reference source tree)")
    import torch

    cases = W.small_cases() + [W.ico_cap(0), W.ico_cap(1)]
    for w in cases:
        v, f, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        vox, dual, inter = O.ref_mesh_to_fdg(v, f, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        tri = torch.from_numpy(np.ascontiguousarray(v[f.astype(np.int64)]).reshape(-1, 3, 3))
        occ = mod.intersect_occ_cpu(tri, [float(x) for x in vs], [int(x) for x in gr]).numpy()
        name = f"{w.name}_{len(f)}" if w.name.startswith("ico_cap") else w.name
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), vertices=v, faces=f, voxel_size=vs, grid_range=gr,
                            weights=np.array([w.face_weight, w.boundary_weight, w.regularization_weight], np.float32),
                            voxels=vox, dual=dual, intersected=inter, occupancy=occ)
        print(f"{name}: {len(f)} faces -> {len(vox)} voxels")


if __name__ == "__main__":
    main()
