"""GPU parity: the CUDA path against the CPU oracle, bit for bit.

Occupancy, intersected flags and dual vertices must be identical to the oracle
(the reference CPU algorithm restated in C, pinned against the reference's own
source), after putting both results in the same row order.
"""
import numpy as np
import pytest

import fdg_workloads as W
from fdg_check import assert_fdg_equal, canon
from oracle import oracle as O

SMALL = {w.name: w for w in W.small_cases()}


def _gpu_api(w, device):
    import torch
    import o_voxel

    v = torch.from_numpy(w.vertices).to(device)
    f = torch.from_numpy(w.faces).to(device)
    out = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())
    torch.cuda.synchronize()
    return tuple(t.cpu().numpy() for t in out)


def _gpu_abi(w, device, faces_dtype="int64"):
    import torch
    import ovx_fdg_abi as abi

    v, f, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
    ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
    ctx = abi.Context(device.index or 0)
    try:
        vt = torch.from_numpy(np.ascontiguousarray(w.vertices)).to(device)
        ft = torch.from_numpy(np.ascontiguousarray(w.faces.astype(faces_dtype))).to(device)
        out = ctx.mesh_to_fdg(vt, ft, ab[0], vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        torch.cuda.synchronize()
        return tuple(t.cpu().numpy() for t in out)
    finally:
        ctx.close()


def _oracle(w):
    r = O.run_workload(w)
    return r.voxels, r.dual, r.intersected


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SMALL))
def test_small_cases_api(cuda, name):
    w = SMALL[name]
    assert_fdg_equal(_gpu_api(w, cuda), _oracle(w), name)


@pytest.mark.gpu
@pytest.mark.parametrize("faces_dtype", ["int32", "int64"])
def test_ico_cap_abi(cuda, faces_dtype):
    w = W.ico_cap(0)
    assert_fdg_equal(_gpu_abi(w, cuda, faces_dtype), _oracle(w), f"ico_cap/{faces_dtype}")


@pytest.mark.gpu
def test_ico_cap_api_seeds(cuda):
    for seed in range(4):
        w = W.ico_cap(seed)
        assert_fdg_equal(_gpu_api(w, cuda), _oracle(w), f"ico_cap seed {seed}")


@pytest.mark.gpu
def test_weight_gates(cuda):
    """face_weight / boundary_weight / regularization_weight <= 0 switch their stages off."""
    base = W.ico_cap(1)
    for fw, bw, rw in [(0.0, 0.2, 1e-2), (1.0, 0.0, 1e-2), (1.0, 0.2, 0.0), (0.0, 0.0, 0.0), (2.5, 3.0, 0.5)]:
        w = W.Workload(base.name, base.vertices, base.faces, base.grid_size, base.aabb, fw, bw, rw)
        assert_fdg_equal(_gpu_api(w, cuda), _oracle(w), f"weights {fw},{bw},{rw}")


@pytest.mark.gpu
def test_primitives_280k(cuda):
    """The 280k-face, grid-512 workload: exact occupancy, flags and dual vertices."""
    w = W.primitives(1)
    assert_fdg_equal(_gpu_api(w, cuda), _oracle(w), "primitives")


@pytest.mark.gpu
def test_deterministic_repeat(cuda):
    """Two runs give identical bytes in identical row order."""
    w = W.primitives(2, faces_total=60_000)
    a = _gpu_api(w, cuda)
    b = _gpu_api(w, cuda)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_intersect_occ(cuda):
    import torch
    import o_voxel

    for w in [W.ico_cap(0), SMALL["outside_aabb"], SMALL["ico_anisotropic"]]:
        v = torch.from_numpy(w.vertices).to(cuda)
        f = torch.from_numpy(w.faces).to(cuda)
        got = o_voxel.convert.intersect_occ(v, f, grid_size=w.grid_size, aabb=w.aabb).cpu().numpy()
        vv, ff, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        want = O.intersect_occ(vv[ff.astype(np.int64)], vs, gr)
        assert np.array_equal(canon(got)[0], canon(want)[0]), w.name


@pytest.mark.gpu
def test_bad_face_index_raises(cuda):
    import torch
    import o_voxel

    v = torch.rand(4, 3, device=cuda) - 0.5
    f = torch.tensor([[0, 1, 2], [1, 2, 7]], device=cuda)
    with pytest.raises(RuntimeError, match="face index"):
        o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=16, aabb=W.UNIT_AABB)
    # the context stays usable afterwards
    w = SMALL["dyadic_tilted"]
    assert_fdg_equal(_gpu_api(w, cuda), _oracle(w), "after error")


def _face_heavy_workload():
    """Eight medium, slightly tilted triangles at grid 128: each hits hundreds of
    voxels in the face and scanline stages, far more than the library's first
    guess of records per triangle, and spans about 16 bricks (the large-triangle
    units of large_rows and large_faces)."""
    rng = np.random.default_rng(11)
    verts, faces = [], []
    for k in range(8):
        c = rng.uniform(-0.25, 0.25, size=3)
        a = np.array([0.0, 0.0, 0.0])
        b = np.array([0.22, 0.01, 0.004])
        d = np.array([0.02, 0.21, 0.008])
        tri = np.stack([a, b, d]) - (a + b + d) / 3.0 + c
        verts.append(tri)
        faces.append(np.arange(3) + 3 * k)
    return W.Workload("face_heavy", np.concatenate(verts).astype(np.float32), np.stack(faces).astype(np.int64),
                      128, W.UNIT_AABB)


@pytest.mark.gpu
def test_face_record_staging_and_fallback(cuda):
    """The first conversion on a fresh context overflows the staging arrays for
    face and scanline records and re-runs those stages in the fill pass; the
    second one fits and buckets the staged records.  Both are bit-exact."""
    import torch
    import ovx_fdg_abi as abi

    w = _face_heavy_workload()
    want = _oracle(w)
    _, _, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
    ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
    ctx = abi.Context(cuda.index or 0)
    try:
        vt = torch.from_numpy(w.vertices).to(cuda)
        ft = torch.from_numpy(w.faces).to(cuda)
        for step in ("fill pass", "staged"):
            out = ctx.mesh_to_fdg(vt, ft, ab[0], vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
            torch.cuda.synchronize()
            assert_fdg_equal(tuple(t.cpu().numpy() for t in out), want, f"face_heavy ({step})")
    finally:
        ctx.close()


@pytest.mark.gpu
def test_two_streams_share_the_context(cuda):
    """Back-to-back conversions on two streams through the shared context: the
    second waits for the first's queued work, so both stay exact."""
    import torch
    import o_voxel

    wa = W.primitives(2, faces_total=60_000)
    wb = W.ico_cap(3)
    sa, sb = torch.cuda.Stream(cuda), torch.cuda.Stream(cuda)
    va, fa = torch.from_numpy(wa.vertices).to(cuda), torch.from_numpy(wa.faces).to(cuda)
    vb, fb = torch.from_numpy(wb.vertices).to(cuda), torch.from_numpy(wb.faces).to(cuda)
    torch.cuda.synchronize()
    outs = []
    for _ in range(3):
        with torch.cuda.stream(sa):
            oa = o_voxel.convert.mesh_to_flexible_dual_grid(va, fa, **wa.kwargs())
        with torch.cuda.stream(sb):
            ob = o_voxel.convert.mesh_to_flexible_dual_grid(vb, fb, **wb.kwargs())
        outs.append((oa, ob))
    torch.cuda.synchronize()
    ra, rb = _oracle(wa), _oracle(wb)
    for oa, ob in outs:
        assert_fdg_equal(tuple(t.cpu().numpy() for t in oa), ra, "stream a")
        assert_fdg_equal(tuple(t.cpu().numpy() for t in ob), rb, "stream b")


@pytest.mark.gpu
def test_host_tensors(cuda):
    """CPU inputs (the reference's CPU call) convert on the GPU and come back as
    CPU tensors equal to the device results and to the oracle."""
    import torch
    import o_voxel

    w = W.ico_cap(0)
    v, f = torch.from_numpy(w.vertices), torch.from_numpy(w.faces)
    host = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **w.kwargs())
    assert all(t.device.type == "cpu" for t in host)
    dev = o_voxel.convert.mesh_to_flexible_dual_grid(v.to(cuda), f.to(cuda), **w.kwargs())
    for h, d in zip(host, dev):
        assert torch.equal(h, d.cpu())
    r = O.run_workload(w, "f32")
    assert_fdg_equal(tuple(t.numpy() for t in host), (r.voxels, r.dual, r.intersected), "host tensors")
    # aabb derived from the CPU vertices, as the reference CPU path does
    kw = dict(w.kwargs())
    kw.pop("aabb")
    host2 = o_voxel.convert.mesh_to_flexible_dual_grid(v, f, **kw)
    lo, hi = v.min(0).values, v.max(0).values
    pad = (hi - lo) / (kw["grid_size"] - 1)
    box = torch.stack([lo - pad * 0.5, hi + pad * 0.5]).tolist()
    dev2 = o_voxel.convert.mesh_to_flexible_dual_grid(v.to(cuda), f.to(cuda), aabb=box, **kw)
    for h, d in zip(host2, dev2):
        assert torch.equal(h, d.cpu())
    occ = o_voxel.convert.intersect_occ(v, f, grid_size=w.grid_size, aabb=w.aabb)
    assert occ.device.type == "cpu"
    assert torch.equal(occ, o_voxel.convert.intersect_occ(v.to(cuda), f.to(cuda), grid_size=w.grid_size, aabb=w.aabb).cpu())
    batch = o_voxel.convert.mesh_to_flexible_dual_grid_batch([(v, f), (v.to(cuda), f.to(cuda))], grid_size=w.grid_size,
                                                            aabb=w.aabb, face_weight=w.face_weight,
                                                            boundary_weight=w.boundary_weight,
                                                            regularization_weight=w.regularization_weight)
    assert batch[0][0].device.type == "cpu" and batch[1][0].is_cuda
    for a, b, c in zip(batch[0], batch[1], host):
        assert torch.equal(a, b.cpu()) and torch.equal(a, c)


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [0, 7])
def test_constrained_list_full(cuda, limit, monkeypatch):
    """Voxels that the deferred constrained-search list cannot take (its room
    capped by OVX_FDG_CLIST_LIMIT at context creation) are searched inline by
    the accumulate kernels: the results stay bit-exact, for the short-list
    kernel and (a 40k-face mesh on a 24^3 grid, whose lists run long) the
    long-list kernels."""
    import torch
    import ovx_fdg_abi as abi

    monkeypatch.setenv("OVX_FDG_CLIST_LIMIT", str(limit))
    coarse = W.primitives(3, faces_total=40_000)
    coarse.grid_size = 24
    for w in (W.ico_cap(1), W.primitives(3, faces_total=40_000), coarse):
        _, _, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
        ctx = abi.Context(cuda.index or 0)
        try:
            vt = torch.from_numpy(w.vertices).to(cuda)
            ft = torch.from_numpy(w.faces).to(cuda)
            out = ctx.mesh_to_fdg(vt, ft, ab[0], vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
            torch.cuda.synchronize()
            assert_fdg_equal(tuple(t.cpu().numpy() for t in out), _oracle(w), f"{w.name} clist limit {limit}")
        finally:
            ctx.close()


@pytest.mark.gpu
def test_work_list_replay(cuda, monkeypatch):
    """Work lists sized from a tiny guess (OVX_FDG_LIST_GUESS=1) overflow on
    the first conversion -- the large pairs and large triangles of a low-poly
    mesh, the long and the plain boundary edges of an open mesh -- and begin
    runs once more with exact sizes; results stay bit-exact, and the next
    conversion on the context fits the first time."""
    import torch
    import ovx_fdg_abi as abi

    monkeypatch.setenv("OVX_FDG_LIST_GUESS", "1")
    lp = W.lowpoly(5, faces_total=600, grid_size=256)
    # the same triangles with no vertex shared: every edge is a boundary edge, most of them long
    soup = W.Workload("lowpoly_soup", lp.vertices[lp.faces].reshape(-1, 3).copy(),
                      np.arange(3 * lp.faces.shape[0], dtype=np.int64).reshape(-1, 3), lp.grid_size, lp.aabb)
    for w in (lp, soup, W.ico_cap(2)):
        _, _, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
        want = _oracle(w)
        ctx = abi.Context(cuda.index or 0)
        try:
            vt = torch.from_numpy(w.vertices).to(cuda)
            ft = torch.from_numpy(w.faces).to(cuda)
            for step in ("replayed", "sized"):
                out = ctx.mesh_to_fdg(vt, ft, ab[0], vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
                torch.cuda.synchronize()
                assert_fdg_equal(tuple(t.cpu().numpy() for t in out), want, f"{w.name} ({step})")
        finally:
            ctx.close()
