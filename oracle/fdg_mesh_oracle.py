"""CPU restatement of o_voxel.convert.flexible_dual_grid_to_mesh
(o_voxel/convert/flexible_dual_grid.py:332-477; its voxel lookup follows
src/hash/hash.cu:269-300 and :366-420) in numpy float32 -- test
infrastructure only.

The restatement follows the reference's tensor operations one by one (each op
rounded to float32).  A neighbour voxel outside [0, grid) on any axis is not
looked up and counts as absent, as the reference's hashmap_lookup_3d kernel
does (hash.cu:283-286).

Pinned: it equals the golden outputs of the reference's own Python function
(tests/golden/to_mesh.npz, made by tests/golden/make_to_mesh_golden.py) bit for
bit on every case and mode there.
"""
import numpy as np

# voxels around the edge of a voxel along x, y, z, in quad order (flexible_dual_grid.py:369-376)
EDGE_NBR = np.array([
    [[0, 0, 0], [0, 0, 1], [0, 1, 1], [0, 1, 0]],
    [[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]],
    [[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0]],
], dtype=np.int64)
SPLIT_1 = np.array([0, 1, 2, 0, 2, 3])
SPLIT_2 = np.array([0, 1, 3, 3, 1, 2])
SPLIT_TRAIN = np.array([0, 1, 4, 1, 2, 4, 2, 3, 4, 3, 0, 4])


def _cross(a, b):
    f = np.float32
    return np.stack([(a[:, 1] * b[:, 2]).astype(f) - (a[:, 2] * b[:, 1]).astype(f),
                     (a[:, 2] * b[:, 0]).astype(f) - (a[:, 0] * b[:, 2]).astype(f),
                     (a[:, 0] * b[:, 1]).astype(f) - (a[:, 1] * b[:, 0]).astype(f)], 1).astype(f)


def _align(v, t):
    n0 = _cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    n1 = _cross(v[t[:, 2]] - v[t[:, 1]], v[t[:, 3]] - v[t[:, 1]])
    p = (n0 * n1).astype(np.float32)
    return np.abs((p[:, 0] + p[:, 1]).astype(np.float32) + p[:, 2]).astype(np.float32)


def to_mesh(coords, dual, flags, split_weight, grid_size, voxel_size, aabb_min, train=False):
    coords = np.asarray(coords, dtype=np.int64)
    dual = np.asarray(dual, dtype=np.float32)
    flags = np.asarray(flags, dtype=bool).reshape(-1, 3)
    gx, gy, gz = (int(x) for x in grid_size)
    vs = np.asarray(voxel_size, dtype=np.float32)
    amin = np.asarray(aabb_min, dtype=np.float32)
    n = coords.shape[0]
    keys = coords[:, 0] * gy * gz + coords[:, 1] * gz + coords[:, 2]
    table = {}
    for i, k in enumerate(keys.tolist()):
        table.setdefault(k, i)
    nbr = coords[:, None, None, :] + EDGE_NBR[None]  # [N,3,4,3]
    cand = nbr[flags]  # [M,4,3], (voxel, axis) order
    ck = cand[..., 0] * gy * gz + cand[..., 1] * gz + cand[..., 2]
    inside = ((cand >= 0) & (cand < np.array([gx, gy, gz]))).all(-1)
    ck = np.where(inside, ck, -1)
    idx = np.array([[table.get(k, -1) for k in row] for row in ck.tolist()], dtype=np.int64).reshape(-1, 4)
    quads = idx[(idx >= 0).all(1)]
    verts = (((coords.astype(np.float32) + dual).astype(np.float32) * vs).astype(np.float32) + amin).astype(np.float32)
    if not train:
        if split_weight is None:
            t0 = quads[:, SPLIT_1]
            t1 = quads[:, SPLIT_2]
            tris = np.where((_align(verts, t0) > _align(verts, t1))[:, None], t0, t1).reshape(-1, 3)
        else:
            w = np.asarray(split_weight, dtype=np.float32).reshape(-1)[quads]
            w02 = (w[:, 0] * w[:, 2]).astype(np.float32)
            w13 = (w[:, 1] * w[:, 3]).astype(np.float32)
            tris = np.where((w02 > w13)[:, None], quads[:, SPLIT_1], quads[:, SPLIT_2]).reshape(-1, 3)
        return verts, tris.astype(np.int32)
    w = np.asarray(split_weight, dtype=np.float32).reshape(-1)[quads]
    q = verts[quads]
    m02 = ((q[:, 0] + q[:, 2]).astype(np.float32) / np.float32(2)).astype(np.float32)
    m13 = ((q[:, 1] + q[:, 3]).astype(np.float32) / np.float32(2)).astype(np.float32)
    w02 = (w[:, 0] * w[:, 2]).astype(np.float32)[:, None]
    w13 = (w[:, 1] * w[:, 3]).astype(np.float32)[:, None]
    mid = ((w02 * m02).astype(np.float32) + (w13 * m13).astype(np.float32)).astype(np.float32) / (w02 + w13).astype(np.float32)
    verts = np.concatenate([verts, mid.astype(np.float32)])
    qi = np.concatenate([quads, np.arange(n, n + quads.shape[0])[:, None]], 1)
    return verts, qi[:, SPLIT_TRAIN].reshape(-1, 3).astype(np.int32)
