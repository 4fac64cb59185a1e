"""Mesh -> flexible dual grid, B200 implementation behind the reference API.

Signature, defaults, argument checks and the derivation of ``aabb`` /
``voxel_size`` / ``grid_size`` follow the reference wrapper
(``o_voxel/convert/flexible_dual_grid.py:38-205`` and ``:208-329``): the same
assertions with the same messages, float32 ``voxel_size = (aabb1 - aabb0) /
grid_size`` computed on the host, ``grid_range = [0, 0, 0, gx, gy, gz]``, and
vertices shifted by ``aabb[0]`` in float32 before the conversion (fused into the
kernels here when ``aabb[0]`` is known on the host).

Differences, all deliberate:
  * Host (CPU) inputs are converted on the current CUDA device: they go up
    through pinned memory and the results come back as CPU tensors (the
    reference would run its single-threaded CPU code).  There is no CPU
    implementation in this product: without a CUDA device, CPU inputs raise
    ``RuntimeError``.
  * int64 faces are consumed directly instead of being cast to int32; indices
    outside ``[0, V)`` raise ``RuntimeError`` (the reference reads out of bounds).
  * Output rows are in a deterministic brick order (8x8x8 bricks, x fastest),
    not in an arbitrary order.  Values are bit-identical to the reference CPU path.
"""
from typing import Any, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _tuning

FloatArrayLike = Union[float, List[Any], Tuple[Any, ...], np.ndarray, torch.Tensor]
IntArrayLike = Union[int, List[Any], Tuple[Any, ...], np.ndarray, torch.Tensor]
ArrayLike = Union[List[Any], Tuple[Any, ...], np.ndarray, torch.Tensor]

__all__ = [
    "mesh_to_flexible_dual_grid",
    "mesh_to_flexible_dual_grid_batch",
    "intersect_occ",
    "flexible_dual_grid_to_mesh",
    "pack_flexible_dual_grid",
]

_C = None


def _ext():
    """The compiled extension; importing it fails loudly if it was not built."""
    global _C
    if _C is None:
        from .. import _C as ext  # noqa: WPS433

        _C = ext
    return _C


def _grid_setup(vertices, faces, voxel_size, grid_size, aabb):
    """Argument normalisation shared by both entry points (reference wrapper :79-178)."""
    assert isinstance(vertices, torch.Tensor), f"vertices must be a torch.Tensor, but got {type(vertices)}"
    assert isinstance(faces, torch.Tensor), f"faces must be a torch.Tensor, but got {type(faces)}"
    assert vertices.dim() == 2, f"vertices must be a 2D tensor, but got {vertices.shape}"
    assert vertices.size(1) == 3, f"vertices must have 3 columns, but got {vertices.size(1)}"
    assert faces.dim() == 2, f"faces must be a 2D tensor, but got {faces.shape}"
    assert faces.size(1) == 3, f"faces must have 3 columns, but got {faces.size(1)}"
    assert vertices.device == faces.device, "vertices and faces must be on the same device"
    assert voxel_size is not None or grid_size is not None, "Either voxel_size or grid_size must be provided"

    device = vertices.device
    vertices = vertices.to(device=device, dtype=torch.float32).contiguous()
    if faces.dtype not in (torch.int32, torch.int64):
        faces = faces.to(device=device, dtype=torch.int32)
    faces = faces.contiguous()
    voxel_size_cpu = None
    grid_size_cpu = None
    aabb_cpu = None

    if voxel_size is not None:
        if isinstance(voxel_size, float):
            voxel_size = [voxel_size, voxel_size, voxel_size]
        if isinstance(voxel_size, (list, tuple)):
            voxel_size = np.array(voxel_size)
        if isinstance(voxel_size, np.ndarray):
            voxel_size_cpu = torch.tensor(voxel_size, dtype=torch.float32)
            voxel_size = voxel_size_cpu
        else:
            assert isinstance(voxel_size, torch.Tensor), f"voxel_size must be a float, list, tuple, np.ndarray, or torch.Tensor, but got {type(voxel_size)}"
            assert not voxel_size.is_cuda, "voxel_size Tensor metadata must be on CPU; pass Python values to avoid implicit CUDA sync"
            voxel_size_cpu = voxel_size.to(dtype=torch.float32).contiguous()
        assert isinstance(voxel_size, torch.Tensor), f"voxel_size must be a float, list, tuple, np.ndarray, or torch.Tensor, but got {type(voxel_size)}"
        voxel_size = voxel_size_cpu  # host metadata; moved to the device only for an aabb derived there
        assert voxel_size.dim() == 1, f"voxel_size must be a 1D tensor, but got {voxel_size.shape}"
        assert voxel_size.size(0) == 3, f"voxel_size must have 3 elements, but got {voxel_size.size(0)}"

    if grid_size is not None:
        if isinstance(grid_size, int):
            grid_size = [grid_size, grid_size, grid_size]
        if isinstance(grid_size, (list, tuple)):
            grid_size = np.array(grid_size)
        if isinstance(grid_size, np.ndarray):
            grid_size_cpu = torch.tensor(grid_size, dtype=torch.int32)
            grid_size = grid_size_cpu
        else:
            assert isinstance(grid_size, torch.Tensor), f"grid_size must be an int, list, tuple, np.ndarray, or torch.Tensor, but got {type(grid_size)}"
            assert not grid_size.is_cuda, "grid_size Tensor metadata must be on CPU; pass Python values to avoid implicit CUDA sync"
            grid_size_cpu = grid_size.to(dtype=torch.int32).contiguous()
        assert isinstance(grid_size, torch.Tensor), f"grid_size must be an int, list, tuple, np.ndarray, or torch.Tensor, but got {type(grid_size)}"
        grid_size = grid_size_cpu  # host metadata; moved to the device only for an aabb derived there
        assert grid_size.dim() == 1, f"grid_size must be a 1D tensor, but got {grid_size.shape}"
        assert grid_size.size(0) == 3, f"grid_size must have 3 elements, but got {grid_size.size(0)}"

    if aabb is not None:
        if isinstance(aabb, (list, tuple)):
            aabb = np.array(aabb)
        if isinstance(aabb, np.ndarray):
            aabb_cpu = torch.tensor(aabb, dtype=torch.float32)
            aabb = aabb_cpu
        else:
            assert isinstance(aabb, torch.Tensor), f"aabb must be a list, tuple, np.ndarray, or torch.Tensor, but got {type(aabb)}"
            assert not aabb.is_cuda, "aabb Tensor metadata must be on CPU; pass Python values to avoid implicit CUDA sync"
            aabb_cpu = aabb.to(dtype=torch.float32).contiguous()
        assert isinstance(aabb, torch.Tensor), f"aabb must be a list, tuple, np.ndarray, or torch.Tensor, but got {type(aabb)}"
        aabb = aabb_cpu  # host metadata: the conversion takes aabb[0] and the voxel size as host values
        assert aabb.dim() == 2, f"aabb must be a 2D tensor, but got {aabb.shape}"
        assert aabb.size(0) == 2, f"aabb must have 2 rows, but got {aabb.size(0)}"
        assert aabb.size(1) == 3, f"aabb must have 3 columns, but got {aabb.size(1)}"

    if aabb is None:
        min_xyz = vertices.min(dim=0).values
        max_xyz = vertices.max(dim=0).values
        if voxel_size is not None:
            voxel_size = voxel_size.to(device=device)
            padding = torch.ceil((max_xyz - min_xyz) / voxel_size) * voxel_size - (max_xyz - min_xyz)
            min_xyz -= padding * 0.5
            max_xyz += padding * 0.5
        if grid_size is not None:
            grid_size = grid_size.to(device=device)
            padding = (max_xyz - min_xyz) / (grid_size - 1)
            min_xyz -= padding * 0.5
            max_xyz += padding * 0.5
        aabb = torch.stack([min_xyz, max_xyz], dim=0).float().contiguous()

    if voxel_size_cpu is None:
        assert grid_size_cpu is not None
        if aabb_cpu is None:
            assert not aabb.is_cuda, "CUDA inputs require CPU aabb or explicit voxel_size to avoid implicit CUDA sync"
            aabb_cpu = aabb.detach()
        voxel_size_cpu = ((aabb_cpu[1] - aabb_cpu[0]) / grid_size_cpu).to(dtype=torch.float32).contiguous()
    if grid_size_cpu is None:
        assert voxel_size_cpu is not None
        if aabb_cpu is None:
            assert not aabb.is_cuda, "CUDA inputs require CPU aabb or explicit grid_size to avoid implicit CUDA sync"
            aabb_cpu = aabb.detach()
        grid_size_cpu = ((aabb_cpu[1] - aabb_cpu[0]) / voxel_size_cpu).round().to(dtype=torch.int32).contiguous()
    voxel_size_arg = [float(x) for x in voxel_size_cpu.tolist()]
    grid_range_arg = [0, 0, 0] + [int(x) for x in grid_size_cpu.tolist()]
    return vertices, faces, aabb, aabb_cpu, voxel_size_arg, grid_range_arg


def _order_code(order: Optional[str]) -> int:
    if order is None or order == "brick":
        return 0
    if order == "z_order":
        return 1
    raise ValueError(f"order must be None, 'brick' or 'z_order', got {order!r}")


def _precision_code(precision: Optional[str]) -> int:
    if precision is None or precision == "exact":
        return 0
    if precision == "compensated":
        return 1
    raise ValueError(f"precision must be None, 'exact' or 'compensated', got {precision!r}")


def _require_cuda(t: torch.Tensor, name: str):
    if not t.is_cuda:
        raise RuntimeError(f"{name}: this implementation runs on CUDA tensors only (got a {t.device} tensor)")


def _host_device(t: torch.Tensor, name: str) -> torch.device:
    """The CUDA device that converts host (CPU) inputs: the current one."""
    if not torch.cuda.is_available():
        raise RuntimeError(f"{name}: this implementation runs on CUDA tensors only (got a {t.device} tensor "
                           "and no CUDA device is available)")
    return torch.device("cuda", torch.cuda.current_device())


def _upload(t: torch.Tensor, dev: torch.device) -> torch.Tensor:
    return t.contiguous().pin_memory().to(dev, non_blocking=True)


def _download(ts):
    """Device results -> CPU tensors (pinned), after the copies have landed."""
    hs = tuple(torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in ts)
    for h, t in zip(hs, ts):
        h.copy_(t, non_blocking=True)
    if ts:
        torch.cuda.current_stream(ts[0].device).synchronize()
    return hs


@torch.no_grad()
def mesh_to_flexible_dual_grid(
    vertices: torch.Tensor,
    faces: torch.Tensor,
    voxel_size: Optional[FloatArrayLike] = None,
    grid_size: Optional[IntArrayLike] = None,
    aabb: Optional[ArrayLike] = None,
    face_weight: float = 1.0,
    boundary_weight: float = 1.0,
    regularization_weight: float = 0.1,
    timing: bool = False,
    order: Optional[str] = None,
    precision: Optional[str] = None,
    route_tolerance: float = 1e-3,
) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """
    Convert a triangle mesh into a sparse flexible dual grid.

    Args:
        vertices (torch.Tensor): [V, 3] mesh vertices (CUDA; CPU tensors are converted on the
            current CUDA device and give CPU results).
        faces (torch.Tensor): [F, 3] triangle vertex indices (int32 or int64, on the vertices' device).
        voxel_size: size of each voxel (float or 3 values); one of voxel_size/grid_size is required.
        grid_size: voxels per axis (int or 3 values).
        aabb: [[x0, y0, z0], [x1, y1, z1]] bounding box; computed from the vertices if omitted.
        face_weight (float): gates the face term of the QEF (> 0 adds it).
        boundary_weight (float): weight of the boundary-edge term of the QEF (> 0 adds it).
        regularization_weight (float): weight pulling each dual vertex toward the mean intersection point.
        timing (bool): accepted for compatibility; ignored (as on the reference CUDA path).
        order (str): row order of the outputs (not in the reference, whose GPU order is
            arbitrary): None or 'brick' -- 8x8x8 bricks then voxels, x-fastest;
            'z_order' -- ascending o_voxel.serialize.encode_seq code, the order the
            reference's examples obtain by sorting on it.
        precision (str): arithmetic of the quadric sums and solves (not in the
            reference): None or 'exact' -- bit-identical to the reference CPU path;
            'compensated' -- FP32 sums with two-sum error terms merged in FP64,
            FP64 regularisation, and an FP64 solve for the voxels whose FP32 solve
            error estimate exceeds route_tolerance voxel edges.  Occupancy and flags
            do not change; dual vertices move toward an FP64 evaluation.
        route_tolerance (float): see precision.

    Returns:
        voxel_indices (torch.Tensor): [N, 3] int32 occupied voxel coordinates.
        dual_vertices (torch.Tensor): [N, 3] float32 dual vertices in grid-local coordinates
            (``aabb[0]`` subtracted, not added back, as in the reference).
        intersected (torch.Tensor): [N, 3] bool; axis a is set when the voxel's edge along a
            starting at its min corner crosses the surface.
    """
    oc = _order_code(order)
    pc = _precision_code(precision)
    vertices, faces, aabb, aabb_cpu, voxel_size_arg, grid_range_arg = _grid_setup(vertices, faces, voxel_size, grid_size, aabb)
    host = not vertices.is_cuda
    if host:
        dev = _host_device(vertices, "mesh_to_flexible_dual_grid")
        if aabb_cpu is None:
            aabb_cpu = aabb.detach()
        vertices, faces = _upload(vertices, dev), _upload(faces, dev)
    _tuning.apply(_ext(), vertices.device.index, max(grid_range_arg[3:]))
    if aabb_cpu is not None:
        origin = [float(x) for x in aabb_cpu[0].tolist()]
        out = _ext().mesh_to_flexible_dual_grid_cuda_ex(vertices, faces, origin, voxel_size_arg, grid_range_arg,
                                                        float(face_weight), float(boundary_weight),
                                                        float(regularization_weight), oc, pc, float(route_tolerance))
    else:
        # aabb derived on the device: shift with torch, exactly like the reference wrapper
        vertices = vertices - aabb[0].reshape(1, 3)
        out = _ext().mesh_to_flexible_dual_grid_cuda(vertices, faces, voxel_size_arg, grid_range_arg, float(face_weight),
                                                     float(boundary_weight), float(regularization_weight), oc, pc,
                                                     float(route_tolerance))
    return _download(out) if host else out


@torch.no_grad()
def intersect_occ(
    vertices: torch.Tensor,
    faces: torch.Tensor,
    voxel_size: Optional[FloatArrayLike] = None,
    grid_size: Optional[IntArrayLike] = None,
    aabb: Optional[ArrayLike] = None,
    order: Optional[str] = None,
) -> torch.Tensor:
    """
    Return only the voxel coordinates intersected by a triangle mesh ([N, 3] int32).

    Same grid setup, occupancy rules and `order` option as
    mesh_to_flexible_dual_grid, without quadrics or dual vertices.
    """
    vertices, faces, aabb, aabb_cpu, voxel_size_arg, grid_range_arg = _grid_setup(vertices, faces, voxel_size, grid_size, aabb)
    host = not vertices.is_cuda
    if host:
        dev = _host_device(vertices, "intersect_occ")
        vertices, faces, aabb = _upload(vertices, dev), _upload(faces, dev), aabb.to(dev)
    vertices = vertices - aabb.to(vertices.device)[0].reshape(1, 3)
    triangles = vertices[faces.to(dtype=torch.long)].contiguous()
    _tuning.apply(_ext(), vertices.device.index, max(grid_range_arg[3:]))
    out = _ext().intersect_occ_cuda(triangles, voxel_size_arg, grid_range_arg, _order_code(order))
    return _download((out,))[0] if host else out


@torch.no_grad()
def mesh_to_flexible_dual_grid_batch(
    meshes: Sequence[Tuple[torch.Tensor, torch.Tensor]],
    voxel_size=None,
    grid_size=None,
    aabb=None,
    face_weight: float = 1.0,
    boundary_weight: float = 1.0,
    regularization_weight: float = 0.1,
    max_group_records: int = 128_000_000,
    order: Optional[str] = None,
    precision: Optional[str] = None,
    route_tolerance: float = 1e-3,
) -> List[Tuple[torch.Tensor, torch.Tensor, torch.Tensor]]:
    """
    Convert many meshes at once; returns one (voxel_indices, dual_vertices,
    intersected) tuple per mesh, each exactly what mesh_to_flexible_dual_grid
    returns for that mesh.

    Args:
        meshes: sequence of (vertices [V,3], faces [F,3]) CUDA tensors, all on one device
            (CPU meshes are uploaded to the current CUDA device and give CPU results).
        voxel_size, grid_size, aabb: as in mesh_to_flexible_dual_grid, either one value
            for every mesh or a list with one value per mesh (with exactly three
            meshes a list of three numbers is one per-axis value: give per-mesh
            sizes as three 3-element lists).
        face_weight, boundary_weight, regularization_weight: shared by all meshes.
        max_group_records: the meshes are converted in groups of consecutive
            meshes whose expected quadric records (about 8 per unit of grid face
            area plus 3 per triangle) stay within this budget, which bounds the
            device workspace (about 100 bytes a record); 0 puts every mesh in one
            group.
        order, precision, route_tolerance: as in mesh_to_flexible_dual_grid.

    The reference has no batched form.  Here every kernel of the conversion
    runs once over all meshes of a group (their triangles, bricks and vertices
    laid out one mesh after another), with one host synchronisation per group,
    so many small and mid-sized meshes cost one pipeline instead of one each.
    Work runs on the current stream; each mesh's tensors are views of the
    group's output tensors.
    """
    n = len(meshes)

    def per_mesh_list(x, shape_one):
        # one value per mesh: a list/tuple of n values, unless it already has the
        # shape of a single value (one 3-vector, one [[x0,y0,z0],[x1,y1,z1]] box)
        if x is None or isinstance(x, (torch.Tensor, np.ndarray)) or not isinstance(x, (list, tuple)) or len(x) != n:
            return False
        return np.asarray(x, dtype=np.float64).shape != shape_one

    def per_mesh(x, i, is_list):
        return x[i] if is_list else x

    vs_list = per_mesh_list(voxel_size, (3,)) if not isinstance(voxel_size, float) else False
    gs_list = per_mesh_list(grid_size, (3,)) if not isinstance(grid_size, int) else False
    ab_list = per_mesh_list(aabb, (2, 3))
    fast = _batch_fast_args(meshes, grid_size, aabb, voxel_size, gs_list, ab_list)
    if fast is not None:
        verts, fcs, origins, vsizes, granges = fast
        host = [False] * n
        meshes = ()
    else:
        verts, fcs, origins, vsizes, granges, host = [], [], [], [], [], []
    for i, (v, f) in enumerate(meshes):
        v, f, ab, ab_cpu, vs_arg, gr_arg = _grid_setup(v, f, per_mesh(voxel_size, i, vs_list),
                                                      per_mesh(grid_size, i, gs_list), per_mesh(aabb, i, ab_list))
        host.append(not v.is_cuda)
        if host[-1]:
            dev = _host_device(v, "mesh_to_flexible_dual_grid_batch")
            v, f = _upload(v, dev), _upload(f, dev)
        if ab_cpu is None:
            ab_cpu = ab.detach().cpu()
        verts.append(v)
        fcs.append(f)
        origins.append([float(x) for x in ab_cpu[0].tolist()])
        vsizes.append(vs_arg)
        granges.append(gr_arg)
    if verts:
        # one set of shapes for the whole batch: the bucket of its largest grid, whose meshes dominate the work
        _tuning.apply(_ext(), verts[0].device.index, max(max(g[3:]) for g in granges))
    out = _ext().mesh_to_flexible_dual_grid_cuda_batch(verts, fcs, origins, vsizes, granges, float(face_weight),
                                                       float(boundary_weight), float(regularization_weight),
                                                       int(max_group_records), _order_code(order),
                                                       _precision_code(precision), float(route_tolerance))
    return [_download(o) if h else o for o, h in zip(out, host)]


def _batch_fast_args(meshes, grid_size, aabb, voxel_size, gs_list, ab_list):
    """The batch's per-mesh arguments in one pass, for the common form: CUDA
    float32 vertices [V,3] and int32/int64 faces [F,3] on one device, grid_size
    and aabb given (one each, or one per mesh), no voxel_size.  The values are
    those of the per-mesh derivation (float32 voxel size (aabb1 - aabb0) /
    grid, grid_range [0, 0, 0, g...], origin aabb0).  None when the arguments
    are of another form; the per-mesh derivation, with its checks, then runs."""
    if voxel_size is not None or grid_size is None or aabb is None or not meshes:
        return None
    dev = None
    for v, f in meshes:
        if not (isinstance(v, torch.Tensor) and isinstance(f, torch.Tensor) and v.is_cuda and f.is_cuda
                and v.dtype == torch.float32 and f.dtype in (torch.int32, torch.int64) and v.dim() == 2
                and v.size(1) == 3 and f.dim() == 2 and f.size(1) == 3 and v.is_contiguous() and f.is_contiguous()):
            return None
        if dev is None:
            dev = v.device
        if v.device != dev or f.device != dev:
            return None
    n = len(meshes)
    try:
        if isinstance(grid_size, torch.Tensor) or isinstance(aabb, torch.Tensor):
            return None
        g = np.asarray(grid_size if gs_list else [grid_size] * n, dtype=np.int64)
        if g.ndim == 1:
            g = np.repeat(g[:, None], 3, axis=1)
        ab = np.asarray(aabb if ab_list else [aabb] * n, dtype=np.float32)
    except (TypeError, ValueError):
        return None
    if g.shape != (n, 3) or ab.shape != (n, 2, 3) or (g <= 0).any():
        return None
    vs = ((ab[:, 1] - ab[:, 0]) / g.astype(np.int32).astype(np.float32)).astype(np.float32)
    verts = [v for v, _ in meshes]
    fcs = [f for _, f in meshes]
    origins = ab[:, 0].astype(np.float64).tolist()
    vsizes = vs.astype(np.float64).tolist()
    granges = [[0, 0, 0] + [int(x) for x in row] for row in g.tolist()]
    return verts, fcs, origins, vsizes, granges


@torch.no_grad()
def flexible_dual_grid_to_mesh(
    coords: torch.Tensor,
    dual_vertices: torch.Tensor,
    intersected_flag: torch.Tensor,
    split_weight: Optional[torch.Tensor],
    aabb: ArrayLike,
    voxel_size: Optional[FloatArrayLike] = None,
    grid_size: Optional[IntArrayLike] = None,
    train: bool = False,
):
    """
    Extract a triangle mesh from a sparse flexible dual grid (the inverse path of
    mesh_to_flexible_dual_grid; reference o_voxel/convert/flexible_dual_grid.py:332-477).

    Every intersected voxel edge whose four surrounding voxels are active gives
    one quad of their dual vertices, split into two triangles (by the larger
    normal alignment, or by split_weight), or into four around a weighted middle
    vertex in training mode.

    Args:
        coords: [N, 3] voxel coordinates (CUDA).
        dual_vertices: [N, 3] dual vertices as offsets inside their voxels (voxel units).
        intersected_flag: [N, 3] bool edge flags.
        split_weight: [N] or [N, 1] split weights, or None.
        aabb: [[x0, y0, z0], [x1, y1, z1]].
        voxel_size / grid_size: one of them is required.
        train: training-mode split (needs split_weight).

    Returns:
        vertices ([N (+ quads in training mode), 3] float32, world coordinates),
        faces ([2 * quads (4 * quads in training mode), 3] int32).
    """
    _require_cuda(coords, "flexible_dual_grid_to_mesh")
    if isinstance(aabb, (list, tuple)):
        aabb = np.array(aabb)
    if isinstance(aabb, np.ndarray):
        aabb = torch.tensor(aabb, dtype=torch.float32)
    assert isinstance(aabb, torch.Tensor), f"aabb must be a list, tuple, np.ndarray, or torch.Tensor, but got {type(aabb)}"
    aabb = aabb.detach().to("cpu", torch.float32)
    assert aabb.dim() == 2 and aabb.size(0) == 2 and aabb.size(1) == 3, f"aabb must be [2, 3], got {tuple(aabb.shape)}"
    if voxel_size is not None:
        if isinstance(voxel_size, float):
            voxel_size = [voxel_size, voxel_size, voxel_size]
        vs_t = torch.as_tensor(np.asarray(voxel_size) if not isinstance(voxel_size, torch.Tensor) else voxel_size,
                               dtype=torch.float32).cpu()
        gs_t = ((aabb[1] - aabb[0]) / vs_t).round().int()
    else:
        assert grid_size is not None, "Either voxel_size or grid_size must be provided"
        if isinstance(grid_size, int):
            grid_size = [grid_size, grid_size, grid_size]
        gs_t = torch.as_tensor(np.asarray(grid_size) if not isinstance(grid_size, torch.Tensor) else grid_size,
                               dtype=torch.int32).cpu()
        vs_t = (aabb[1] - aabb[0]) / gs_t
    assert vs_t.numel() == 3 and gs_t.numel() == 3, "voxel_size and grid_size must have 3 elements"
    sw = None
    if split_weight is not None:
        sw = split_weight.reshape(-1)
    return _ext().flexible_dual_grid_to_mesh_cuda(coords, dual_vertices, intersected_flag, sw,
                                                  [int(x) for x in gs_t.tolist()], [float(x) for x in vs_t.tolist()],
                                                  [float(x) for x in aabb[0].tolist()], bool(train))


@torch.no_grad()
def pack_flexible_dual_grid(voxel_indices: torch.Tensor, dual_vertices: torch.Tensor, intersected: torch.Tensor,
                            grid_size: IntArrayLike) -> Tuple[torch.Tensor, torch.Tensor]:
    """
    Pack a conversion's outputs into the .vxz attributes the reference's example
    writes (examples/mesh2ovox.py:51-54), in one kernel:

        dual_vertices_u8 = uint8(clamp(dual_vertices * grid_size - voxel_indices, 0, 1) * 255)   [N, 3]
        intersected_u8   = x + 2 y + 4 z of the edge flags                                 [N, 1]

    dual_vertices are the grid-local outputs of mesh_to_flexible_dual_grid over a
    unit-extent aabb (as in that example); grid_size is an int or three ints.
    """
    _require_cuda(voxel_indices, "pack_flexible_dual_grid")
    if isinstance(grid_size, int):
        grid_size = [grid_size] * 3
    res = [float(np.float32(x)) for x in (grid_size.tolist() if isinstance(grid_size, torch.Tensor) else grid_size)]
    assert len(res) == 3, "grid_size must be an int or 3 values"
    return _ext().pack_flexible_dual_grid_cuda(voxel_indices, dual_vertices, intersected, res)
