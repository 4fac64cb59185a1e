"""Output row order: order='z_order' gives the native rows sorted by their
o_voxel.serialize.encode_seq code, identically; encode_seq / decode_seq on
the GPU, in both modes (z_order, hilbert), against the golden codes of the
reference implementation."""
import os

import numpy as np
import pytest

import fdg_workloads as W
from fdg_check import assert_fdg_equal
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "z_order.npz")
GOLDEN_HILBERT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hilbert.npz")


@pytest.mark.gpu
def test_encode_decode_seq_golden(cuda):
    import torch
    import o_voxel

    d = np.load(GOLDEN)
    xyz = torch.from_numpy(d["xyz"]).to(cuda)
    codes = o_voxel.serialize.encode_seq(xyz)
    assert np.array_equal(codes.cpu().numpy(), d["codes"])
    back = o_voxel.serialize.decode_seq(codes)
    assert np.array_equal(back.cpu().numpy(), d["decoded"])
    # a permutation of the columns, against the oracle
    perm = [2, 0, 1]
    codes_p = o_voxel.serialize.encode_seq(xyz, permute=perm).cpu().numpy()
    x = d["xyz"]
    assert np.array_equal(codes_p, O.z_order_encode(x[:, 2], x[:, 0], x[:, 1]))
    assert np.array_equal(o_voxel.serialize.decode_seq(torch.from_numpy(codes_p).to(cuda), permute=perm).cpu().numpy(), x)


@pytest.mark.gpu
def test_encode_decode_seq_hilbert_golden(cuda):
    import torch
    import o_voxel

    d = np.load(GOLDEN_HILBERT)
    xyz = torch.from_numpy(d["xyz"]).to(cuda)
    codes = o_voxel.serialize.encode_seq(xyz, mode="hilbert")
    assert np.array_equal(codes.cpu().numpy(), d["codes"])
    back = o_voxel.serialize.decode_seq(codes, mode="hilbert")
    assert np.array_equal(back.cpu().numpy(), d["decoded"])
    perm = [1, 2, 0]
    codes_p = o_voxel.serialize.encode_seq(xyz, permute=perm, mode="hilbert").cpu().numpy()
    x = d["xyz"]
    assert np.array_equal(codes_p, O.hilbert_encode(x[:, 1], x[:, 2], x[:, 0]))
    back_p = o_voxel.serialize.decode_seq(torch.from_numpy(codes_p).to(cuda), permute=perm, mode="hilbert")
    assert np.array_equal(back_p.cpu().numpy(), x)
    # every code of a 64^3 block of the curve, through the C ABI, against the oracle
    all_codes = torch.arange(1 << 18, dtype=torch.int32, device=cuda)
    dec = o_voxel.serialize.decode_seq(all_codes, mode="hilbert").cpu().numpy()
    ox, oy, oz = O.hilbert_decode(np.arange(1 << 18, dtype=np.int32))
    assert np.array_equal(dec, np.stack([ox, oy, oz], 1))
    assert np.array_equal(o_voxel.serialize.encode_seq(torch.from_numpy(dec).to(cuda), mode="hilbert").cpu().numpy(),
                          np.arange(1 << 18, dtype=np.int32))


def _by_code(vox, *cols):
    code = O.z_order_encode(vox[:, 0], vox[:, 1], vox[:, 2])
    o = np.argsort(code, kind="stable")
    return (vox[o],) + tuple(c[o] for c in cols)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ico_cap", "primitives60k", "anisotropic"])
def test_z_order_output(cuda, name):
    import torch
    import o_voxel

    w = {"ico_cap": lambda: W.ico_cap(0), "primitives60k": lambda: W.primitives(2, faces_total=60_000),
         "anisotropic": lambda: {c.name: c for c in W.small_cases()}["ico_anisotropic"]}[name]()
    v = torch.from_numpy(w.vertices).to(cuda)
    f = torch.from_numpy(w.faces).to(cuda)
    nat = [t.cpu().numpy() for t in o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())]
    zo = [t.cpu().numpy() for t in o_voxel.convert.mesh_to_flexible_dual_grid(v, f, order="z_order", **w.kwargs())]
    code = O.z_order_encode(zo[0][:, 0], zo[0][:, 1], zo[0][:, 2])
    assert np.all(np.diff(code.astype(np.int64)) > 0), "rows not in ascending z-order"
    want = _by_code(*nat)
    for a, b in zip(zo, want):
        assert np.array_equal(a, b)
    r = O.run_workload(w)
    assert_fdg_equal(tuple(zo), (r.voxels, r.dual, r.intersected), name)
    # occupancy only, and the batched form
    occ = o_voxel.convert.intersect_occ(v, f, grid_size=w.grid_size, aabb=w.aabb, order="z_order").cpu().numpy()
    assert np.array_equal(occ, zo[0])
    (bz,) = o_voxel.convert.mesh_to_flexible_dual_grid_batch([(v, f)], grid_size=w.grid_size, aabb=w.aabb,
                                                             order="z_order", **{k: x for k, x in w.kwargs().items()
                                                                                 if k not in ("grid_size", "aabb")})
    for a, b in zip(bz, zo):
        assert np.array_equal(a.cpu().numpy(), b)
