"""Serialisation codes (o_voxel.serialize, modes 'z_order' and 'hilbert'): the
oracle's restatements against the golden codes made by the reference's own CPU
implementations."""
import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "z_order.npz")
GOLDEN_HILBERT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hilbert.npz")


def test_oracle_z_order_matches_golden():
    d = np.load(GOLDEN)
    xyz = d["xyz"]
    codes = O.z_order_encode(xyz[:, 0], xyz[:, 1], xyz[:, 2])
    assert np.array_equal(codes, d["codes"])
    x, y, z = O.z_order_decode(d["codes"])
    assert np.array_equal(np.stack([x, y, z], 1), d["decoded"])


def test_oracle_z_order_matches_reference_build():
    L = O.ref_z_order_lib()
    if L is None:
        import pytest

        pytest.skip("reference z-order source not built here")
    rng = np.random.default_rng(5)
    xyz = np.ascontiguousarray(rng.integers(0, 1024, size=(20000, 3), dtype=np.uint32))
    x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
    ref = np.empty(xyz.shape[0], dtype=np.uint32)
    L.ref_z_order_encode(xyz.shape[0], x.ctypes.data, y.ctypes.data, z.ctypes.data, ref.ctypes.data)
    assert np.array_equal(O.z_order_encode(x, y, z), ref.astype(np.int32))


def test_z_order_sorts_like_the_brick_decomposition():
    """The library emits z-order rows brick by brick: a voxel's code is its
    8^3 brick's code followed by the 9-bit code of its position in the brick."""
    rng = np.random.default_rng(9)
    xyz = rng.integers(0, 1024, size=(5000, 3)).astype(np.int32)
    full = O.z_order_encode(xyz[:, 0], xyz[:, 1], xyz[:, 2]).astype(np.int64)
    brick = O.z_order_encode(xyz[:, 0] >> 3, xyz[:, 1] >> 3, xyz[:, 2] >> 3).astype(np.int64)
    local = O.z_order_encode(xyz[:, 0] & 7, xyz[:, 1] & 7, xyz[:, 2] & 7).astype(np.int64)
    assert np.array_equal(full, (brick << 9) | local)


def test_oracle_hilbert_matches_golden():
    d = np.load(GOLDEN_HILBERT)
    xyz = d["xyz"]
    codes = O.hilbert_encode(xyz[:, 0], xyz[:, 1], xyz[:, 2])
    assert np.array_equal(codes, d["codes"])
    x, y, z = O.hilbert_decode(d["codes"])
    assert np.array_equal(np.stack([x, y, z], 1), d["decoded"])
    assert np.array_equal(d["decoded"], xyz)  # the reference's decode inverts its encode


def test_oracle_hilbert_matches_reference_build():
    L = O.ref_hilbert_lib()
    if L is None:
        import pytest

        pytest.skip("reference Hilbert source not built here")
    rng = np.random.default_rng(6)
    xyz = np.ascontiguousarray(rng.integers(0, 1024, size=(20000, 3), dtype=np.uint32))
    x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
    ref = np.empty(xyz.shape[0], dtype=np.uint32)
    L.ref_hilbert_encode(xyz.shape[0], x.ctypes.data, y.ctypes.data, z.ctypes.data, ref.ctypes.data)
    assert np.array_equal(O.hilbert_encode(x, y, z), ref.astype(np.int32))


def test_hilbert_curve_is_continuous():
    """Consecutive Hilbert codes are face neighbours: decoding codes 0..4095
    (a 16^3 block of the curve) steps by exactly one voxel each time."""
    codes = np.arange(4096, dtype=np.int32)
    x, y, z = O.hilbert_decode(codes)
    step = np.abs(np.diff(np.stack([x, y, z], 1).astype(np.int64), axis=0)).sum(1)
    assert np.all(step == 1)
    assert np.array_equal(O.hilbert_encode(x, y, z), codes)
