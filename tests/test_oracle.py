"""The CPU oracle (C restatement of the reference CPU path) against the
reference's own outputs: golden fixtures made from the reference source
(tests/golden/make_golden.py), and the reference source itself where built."""
import glob
import os

import numpy as np
import pytest

import fdg_workloads as W
from oracle import oracle as O

# conversion fixtures (z_order.npz and hilbert.npz hold serialisation codes, covered by
# test_serialize_cpu.py; to_mesh.npz the inverse path, covered by test_to_mesh_cpu.py)
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if os.path.basename(p) not in ("z_order.npz", "hilbert.npz", "to_mesh.npz"))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path):
    g = np.load(path)
    fw, bw, rw = (float(x) for x in g["weights"])
    r = O.mesh_to_fdg(g["vertices"], g["faces"], g["voxel_size"], g["grid_range"], fw, bw, rw)
    # same row order: both follow the reference's first-touch insertion order
    assert np.array_equal(r.voxels, g["voxels"])
    assert np.array_equal(r.intersected, g["intersected"])
    assert np.array_equal(r.dual.astype(np.float32).view(np.uint32), g["dual"].view(np.uint32))
    tri = g["vertices"][g["faces"].astype(np.int64)]
    occ = O.intersect_occ(tri, g["voxel_size"], g["grid_range"])
    assert np.array_equal(occ, g["occupancy"])


def test_golden_set_present():
    assert len(GOLDEN) >= 10


@pytest.mark.skipif(O.ref_module() is None, reason="reference CPU source not built here")
@pytest.mark.parametrize("seed", [2, 5, 11])
def test_oracle_matches_reference_source(seed):
    cases = [W.ico_cap(seed), W.primitives(seed, faces_total=12_000)]
    for w in cases:
        w = W.Workload(w.name, w.vertices, w.faces, 96 if w.name == "primitives" else w.grid_size, w.aabb,
                       w.face_weight, w.boundary_weight, w.regularization_weight)
        v, f, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        r = O.mesh_to_fdg(v, f, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        vox, dual, inter = O.ref_mesh_to_fdg(v, f, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        assert np.array_equal(r.voxels, vox), w.name
        assert np.array_equal(r.intersected, inter), w.name
        assert np.array_equal(r.dual.view(np.uint32), dual.view(np.uint32)), w.name


def test_fp64_variant_same_geometry():
    """The FP64 build keeps every geometric decision (occupancy, flags) and only
    changes the quadric arithmetic; its dual vertices stay close to the FP32 ones."""
    w = W.ico_cap(0)
    a = O.run_workload(w, "f32")
    b = O.run_workload(w, "f64")
    assert np.array_equal(a.voxels, b.voxels)
    assert np.array_equal(a.intersected, b.intersected)
    vs = 1.0 / 64
    err = np.abs(a.dual.astype(np.float64) - b.dual) / vs
    assert np.sqrt(np.mean(err ** 2)) < 1e-2


def test_bad_index_rejected():
    v = np.zeros((3, 3), np.float32)
    with pytest.raises(RuntimeError):
        O.mesh_to_fdg(v, np.array([[0, 1, 5]], np.int32), np.full(3, 0.1, np.float32), np.array([0, 0, 0, 8, 8, 8], np.int32),
                      1.0, 1.0, 0.1)
