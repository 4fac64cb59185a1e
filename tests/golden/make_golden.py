"""Generate the golden fixtures in this directory from the reference's own CPU
implementation (src/convert/flexible_dual_grid.cpp, built into oracle/_ref by
oracle/build.py against the project's Eigen-API shim).

Each fixture stores the grid-local inputs exactly as the reference operator
receives them (float32 shifted vertices, int32 faces, float32 voxel size,
grid range, weights) and the reference outputs in the reference's own row
order (first-touch insertion order): voxel coordinates, dual vertices and
intersected flags, plus the occupancy-only result of intersect_occ_cpu.

Also z_order.npz and hilbert.npz: serialisation codes from the reference's
own CPU implementations (src/serialize/z_order.cu and hilbert.cu, built into
oracle/_ref).

Run from the repository root where the reference source tree is available:
    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py z_order    # only the z-order fixture
    python tests/golden/make_golden.py hilbert    # only the Hilbert fixture
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


def make_z_order():
    """z_order.npz: seeded coordinates in [0, 1024) (plus the extremes) and the
    reference's CPU z-order codes of them (src/serialize/z_order.cu, built into
    oracle/_ref/zorder_ref.so), and the reference's decode of those codes."""
    B.build_ref_zorder()
    L = O.ref_z_order_lib()
    if L is None:
        raise SystemExit("reference z-order source not built (needs the reference source tree)")
    rng = np.random.default_rng(1234)
    xyz = rng.integers(0, 1024, size=(4096, 3), dtype=np.uint32)
    edge = np.array([[0, 0, 0], [1023, 1023, 1023], [1023, 0, 0], [0, 1023, 0], [0, 0, 1023], [512, 256, 128],
                     [1, 2, 4], [7, 7, 7], [8, 8, 8], [511, 512, 513]], dtype=np.uint32)
    xyz = np.ascontiguousarray(np.concatenate([edge, xyz]))
    x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
    n = xyz.shape[0]
    codes = np.empty(n, dtype=np.uint32)
    L.ref_z_order_encode(n, x.ctypes.data, y.ctypes.data, z.ctypes.data, codes.ctypes.data)
    dx, dy, dz = (np.empty(n, dtype=np.uint32) for _ in range(3))
    L.ref_z_order_decode(n, codes.ctypes.data, dx.ctypes.data, dy.ctypes.data, dz.ctypes.data)
    np.savez_compressed(os.path.join(HERE, "z_order.npz"), xyz=xyz.astype(np.int32), codes=codes.astype(np.int32),
                        decoded=np.stack([dx, dy, dz], 1).astype(np.int32))
    print(f"z_order: {n} coordinates")


def make_hilbert():
    """hilbert.npz: the same kind of coordinates, the reference's CPU Hilbert
    codes of them (src/serialize/hilbert.cu, built into oracle/_ref/hilbert_ref.so),
    and the reference's decode of those codes."""
    B.build_ref_hilbert()
    L = O.ref_hilbert_lib()
    if L is None:
        raise SystemExit("reference Hilbert source not built (needs the reference source tree)")
    rng = np.random.default_rng(4321)
    xyz = rng.integers(0, 1024, size=(4096, 3), dtype=np.uint32)
    edge = np.array([[0, 0, 0], [1023, 1023, 1023], [1023, 0, 0], [0, 1023, 0], [0, 0, 1023], [512, 256, 128],
                     [1, 2, 4], [7, 7, 7], [8, 8, 8], [511, 512, 513], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.uint32)
    xyz = np.ascontiguousarray(np.concatenate([edge, xyz]))
    x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
    n = xyz.shape[0]
    codes = np.empty(n, dtype=np.uint32)
    L.ref_hilbert_encode(n, x.ctypes.data, y.ctypes.data, z.ctypes.data, codes.ctypes.data)
    dx, dy, dz = (np.empty(n, dtype=np.uint32) for _ in range(3))
    L.ref_hilbert_decode(n, codes.ctypes.data, dx.ctypes.data, dy.ctypes.data, dz.ctypes.data)
    np.savez_compressed(os.path.join(HERE, "hilbert.npz"), xyz=xyz.astype(np.int32), codes=codes.astype(np.int32),
                        decoded=np.stack([dx, dy, dz], 1).astype(np.int32))
    print(f"hilbert: {n} coordinates")


def main():
    if len(sys.argv) > 1 and sys.argv[1] in ("z_order", "hilbert"):
        (make_z_order if sys.argv[1] == "z_order" else make_hilbert)()
        return
    make_z_order()
    make_hilbert()
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
