"""Comparison helpers shared by the tests (canonical row order, exact checks)."""
import numpy as np


def canonical_order(vox: np.ndarray) -> np.ndarray:
    """Row permutation sorting voxels by (z, y, x)."""
    vox = np.asarray(vox).reshape(-1, 3)
    return np.lexsort((vox[:, 0], vox[:, 1], vox[:, 2]))


def canon(vox, *cols):
    o = canonical_order(vox)
    return (np.asarray(vox)[o],) + tuple(np.asarray(c)[o] for c in cols)


def assert_fdg_equal(got, want, label=""):
    """got/want: (voxels [N,3] int32, dual [N,3] float32, intersected [N,3] bool), any row order.
    Occupancy and flags must match exactly; dual vertices bit for bit."""
    gv, gd, gi = (np.asarray(x) for x in got)
    wv, wd, wi = (np.asarray(x) for x in want)
    assert gv.shape == wv.shape, f"{label}: voxel count {gv.shape[0]} != {wv.shape[0]}"
    gv, gd, gi = canon(gv, gd, gi)
    wv, wd, wi = canon(wv, wd, wi)
    assert np.array_equal(gv, wv), f"{label}: occupancy differs"
    bad_flags = np.sum(np.any(gi.astype(bool) != wi.astype(bool), axis=1))
    assert bad_flags == 0, f"{label}: {bad_flags} voxels with different intersected flags"
    gd = np.ascontiguousarray(gd, dtype=np.float32)
    wd = np.ascontiguousarray(wd, dtype=np.float32)
    diff = np.any(gd.view(np.uint32) != wd.view(np.uint32), axis=1)
    if diff.any():
        idx = np.nonzero(diff)[0][:5]
        err = np.abs(gd - wd).max()
        raise AssertionError(f"{label}: {diff.sum()} dual vertices differ in bits (max abs {err:.3g}); "
                             f"first rows {gv[idx].tolist()} got {gd[idx].tolist()} want {wd[idx].tolist()}")
