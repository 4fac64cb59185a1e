"""ctypes binding of the C ABI in include/ovx_fdg.h (libovx_fdg.so).

This is the binding a non-torch host (or a test) uses to reach the library
without the torch extension.  Device memory for inputs and outputs is supplied
by the caller as raw CUDA pointers; the helpers below take torch CUDA tensors
for convenience.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libovx_fdg.so")

OK = 0
STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "BAD_FACE_INDEX", 3: "CUDA_ERROR", 4: "OUT_OF_MEMORY", 5: "CAPACITY",
          6: "INTERNAL"}

# (name, restype, argtypes) for every function declared in include/ovx_fdg.h
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_F = ctypes.c_float
PROTOTYPES = [
    ("ovx_fdg_context_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    ("ovx_fdg_context_destroy", None, [_P]),
    ("ovx_fdg_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("ovx_fdg_last_error", ctypes.c_char_p, [_P]),
    ("ovx_fdg_workspace_bytes", _I64, [_P]),
    ("ovx_fdg_set_profiling", ctypes.c_int, [_P, ctypes.c_int]),
    ("ovx_fdg_stage_times", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    ("ovx_fdg_stage_name", ctypes.c_char_p, [ctypes.c_int]),
    ("ovx_fdg_kernel_launches", _I64, [_P]),
    ("ovx_fdg_last_counts", ctypes.c_int, [_P, ctypes.POINTER(_I64), ctypes.c_int]),
    ("ovx_fdg_set_output_order", ctypes.c_int, [_P, ctypes.c_int]),
    ("ovx_fdg_set_tuning", ctypes.c_int, [_P, _P]),
    ("ovx_fdg_set_precision", ctypes.c_int, [_P, ctypes.c_int, _F]),
    ("ovx_fdg_get_tuning", ctypes.c_int, [_P, _P]),
    ("ovx_z_order_encode", ctypes.c_int, [_P, _P, _P, _P, _I64, _P]),
    ("ovx_z_order_decode", ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    ("ovx_hilbert_encode", ctypes.c_int, [_P, _P, _P, _P, _I64, _P]),
    ("ovx_hilbert_decode", ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    ("ovx_fdg_pack", ctypes.c_int, [_P, _P, _P, _P, _I64, _P, _P, _P]),
    ("ovx_fdg_mesh_context_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    ("ovx_fdg_mesh_context_destroy", None, [_P]),
    ("ovx_fdg_mesh_last_error", ctypes.c_char_p, [_P]),
    ("ovx_fdg_to_mesh_begin", ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I64, _P, _P, _P, ctypes.c_int32,
                                             ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    ("ovx_fdg_to_mesh_finish", ctypes.c_int, [_P, _P, _P, _P]),
    ("ovx_fdg_begin", ctypes.c_int, [_P, _P, _P, _I64, _P, ctypes.c_int32, _I64, _P, _P, _F, _F, _F, ctypes.POINTER(_I64)]),
    ("ovx_fdg_finish", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("ovx_fdg_sync_status", ctypes.c_int, [_P, _P]),
    ("ovx_fdg_begin_batch", ctypes.c_int, [_P, _P, _P, ctypes.c_int32, _F, _F, _F, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    ("ovx_fdg_finish_batch", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("ovx_fdg_occupancy_begin", ctypes.c_int, [_P, _P, _P, _I64, _P, ctypes.POINTER(_I64)]),
    ("ovx_fdg_occupancy_finish", ctypes.c_int, [_P, _P, _P]),
    ("ovx_fdg_occupancy_noalloc", ctypes.c_int, [_P, _P, _I64, _P, _P, _I64, ctypes.POINTER(_I64)]),
]


class Grid(ctypes.Structure):
    _fields_ = [("voxel_size", ctypes.c_float * 3), ("grid_min", ctypes.c_int32 * 3), ("grid_max", ctypes.c_int32 * 3)]


TUNING_FIELDS = ("unit_cells", "warp_scan_cells", "inline_face_bricks", "dense_candidates", "long_walk")


class Tuning(ctypes.Structure):
    """ovx_fdg_tuning: work shapes of a context's conversions."""
    _fields_ = [(name, ctypes.c_int32) for name in TUNING_FIELDS]


class MeshDesc(ctypes.Structure):
    """ovx_fdg_mesh: one mesh of a batched conversion."""
    _fields_ = [("vertices", ctypes.c_void_p), ("num_vertices", ctypes.c_int64), ("faces", ctypes.c_void_p),
                ("face_index_bytes", ctypes.c_int32), ("num_faces", ctypes.c_int64), ("origin", ctypes.c_float * 3),
                ("grid", Grid)]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libovx_fdg.so is not built ({LIB_PATH}); run o-voxel-gpu_b200/ovx_build.py")
        _LIB = ctypes.CDLL(LIB_PATH)
        for name, res, args in PROTOTYPES:
            fn = getattr(_LIB, name)
            fn.restype = res
            fn.argtypes = args
    return _LIB


class FdgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def make_grid(voxel_size, grid_range) -> Grid:
    g = Grid()
    for a in range(3):
        g.voxel_size[a] = float(voxel_size[a])
        g.grid_min[a] = int(grid_range[a])
        g.grid_max[a] = int(grid_range[3 + a])
    return g


class Context:
    """One ovx_fdg_context on one device."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        rc = self._lib.ovx_fdg_context_create(int(device), ctypes.byref(h))
        if rc != OK:
            raise FdgError(rc, "ovx_fdg_context_create")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            self._lib.ovx_fdg_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != OK:
            msg = self._lib.ovx_fdg_last_error(self.handle)
            raise FdgError(rc, f"{what}: {msg.decode() if msg else ''}")

    def workspace_bytes(self) -> int:
        return int(self._lib.ovx_fdg_workspace_bytes(self.handle))

    def set_profiling(self, enable: bool = True):
        self._check(self._lib.ovx_fdg_set_profiling(self.handle, 1 if enable else 0), "ovx_fdg_set_profiling")

    def stage_times(self) -> dict:
        """Stage durations (ms) of the last conversion; waits for it."""
        buf = (ctypes.c_float * 16)()
        n = self._lib.ovx_fdg_stage_times(self.handle, buf, 16)
        if n < 0:
            raise FdgError(-n, "ovx_fdg_stage_times")
        return {self._lib.ovx_fdg_stage_name(i).decode(): float(buf[i]) for i in range(n)}

    def kernel_launches(self) -> int:
        return int(self._lib.ovx_fdg_kernel_launches(self.handle))

    def set_tuning(self, tuning=None):
        """tuning: dict of ovx_fdg_tuning fields (missing ones keep their
        defaults), or None for the defaults."""
        if tuning is None:
            self._check(self._lib.ovx_fdg_set_tuning(self.handle, None), "ovx_fdg_set_tuning")
            return
        t = Tuning()
        self._check(self._lib.ovx_fdg_set_tuning(self.handle, None), "ovx_fdg_set_tuning")
        self._check(self._lib.ovx_fdg_get_tuning(self.handle, ctypes.byref(t)), "ovx_fdg_get_tuning")
        for k, v in tuning.items():
            setattr(t, k, int(v))
        self._check(self._lib.ovx_fdg_set_tuning(self.handle, ctypes.byref(t)), "ovx_fdg_set_tuning")

    def get_tuning(self) -> dict:
        t = Tuning()
        self._check(self._lib.ovx_fdg_get_tuning(self.handle, ctypes.byref(t)), "ovx_fdg_get_tuning")
        return {k: int(getattr(t, k)) for k in TUNING_FIELDS}

    def set_output_order(self, order: int):
        """0: brick order (default), 1: ascending z-order code."""
        self._check(self._lib.ovx_fdg_set_output_order(self.handle, int(order)), "ovx_fdg_set_output_order")

    def set_precision(self, precision: int = 0, route_tolerance: float = 1e-3):
        """0: exact (default), 1: compensated sums with FP64 routing of voxels
        whose FP32 solve error estimate exceeds route_tolerance voxel edges."""
        self._check(self._lib.ovx_fdg_set_precision(self.handle, int(precision), float(route_tolerance)),
                    "ovx_fdg_set_precision")

    def last_counts(self) -> dict:
        """Sizes of the last conversion (voxels, occupied bricks, records, boundary edges, grid bricks, and the
        voxels the compensated mode solved in FP64)."""
        buf = (_I64 * 6)()
        n = self._lib.ovx_fdg_last_counts(self.handle, buf, 6)
        if n < 0:
            raise FdgError(-n, "ovx_fdg_last_counts")
        names = ("voxels", "bricks_occupied", "records", "boundary_edges", "bricks_grid", "routed_fp64")
        return {names[i]: int(buf[i]) for i in range(n)}

    def mesh_to_fdg(self, vertices, faces, origin, voxel_size, grid_range, fw, bw, rw, stream=None, check=True):
        """vertices: CUDA float32 [V,3]; faces: CUDA int32/int64 [F,3]; returns torch tensors."""
        import torch

        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(vertices.device).cuda_stream)
        grid = make_grid(voxel_size, grid_range)
        org = (ctypes.c_float * 3)(*[float(x) for x in origin]) if origin is not None else None
        n = ctypes.c_int64(0)
        rc = self._lib.ovx_fdg_begin(self.handle, st, ctypes.c_void_p(vertices.data_ptr()), vertices.shape[0],
                                     ctypes.c_void_p(faces.data_ptr() if faces.numel() else 0), faces.element_size(),
                                     faces.shape[0], ctypes.cast(org, ctypes.c_void_p) if org is not None else None,
                                     ctypes.byref(grid), float(fw), float(bw), float(rw), ctypes.byref(n))
        self._check(rc, "ovx_fdg_begin")
        N = n.value
        vox = torch.empty((N, 3), dtype=torch.int32, device=vertices.device)
        dual = torch.empty((N, 3), dtype=torch.float32, device=vertices.device)
        inter = torch.empty((N, 3), dtype=torch.bool, device=vertices.device)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t.numel() else 0)  # noqa: E731
        rc = self._lib.ovx_fdg_finish(self.handle, st, ptr(vox), ptr(dual), ptr(inter))
        self._check(rc, "ovx_fdg_finish")
        if check:
            self._check(self._lib.ovx_fdg_sync_status(self.handle, st), "ovx_fdg_sync_status")
        return vox, dual, inter

    def mesh_to_fdg_batch(self, meshes, fw, bw, rw, stream=None, check=True):
        """meshes: list of (vertices, faces, origin, voxel_size, grid_range) with
        CUDA tensors; one batched conversion; returns per-mesh torch tensors
        (views of one output buffer)."""
        import torch

        dev = meshes[0][0].device
        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)
        descs = (MeshDesc * len(meshes))()
        for d, (v, f, origin, vs, gr) in zip(descs, meshes):
            d.vertices = v.data_ptr() if v.numel() else None
            d.num_vertices = v.shape[0]
            d.faces = f.data_ptr() if f.numel() else None
            d.face_index_bytes = f.element_size()
            d.num_faces = f.shape[0]
            for a in range(3):
                d.origin[a] = float(origin[a])
            d.grid = make_grid(vs, gr)
        nv = (_I64 * len(meshes))()
        total = _I64(0)
        self._check(self._lib.ovx_fdg_begin_batch(self.handle, st, ctypes.cast(descs, ctypes.c_void_p), len(meshes), float(fw),
                                                  float(bw), float(rw), nv, ctypes.byref(total)), "ovx_fdg_begin_batch")
        N = total.value
        vox = torch.empty((N, 3), dtype=torch.int32, device=dev)
        dual = torch.empty((N, 3), dtype=torch.float32, device=dev)
        inter = torch.empty((N, 3), dtype=torch.bool, device=dev)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t.numel() else 0)  # noqa: E731
        self._check(self._lib.ovx_fdg_finish_batch(self.handle, st, ptr(vox), ptr(dual), ptr(inter)), "ovx_fdg_finish_batch")
        if check:
            self._check(self._lib.ovx_fdg_sync_status(self.handle, st), "ovx_fdg_sync_status")
        out, row = [], 0
        for i in range(len(meshes)):
            out.append((vox[row:row + nv[i]], dual[row:row + nv[i]], inter[row:row + nv[i]]))
            row += nv[i]
        return out

    def occupancy(self, triangles, voxel_size, grid_range, stream=None):
        import torch

        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(triangles.device).cuda_stream)
        grid = make_grid(voxel_size, grid_range)
        n = ctypes.c_int64(0)
        rc = self._lib.ovx_fdg_occupancy_begin(self.handle, st, ctypes.c_void_p(triangles.data_ptr() if triangles.numel() else 0),
                                               triangles.shape[0], ctypes.byref(grid), ctypes.byref(n))
        self._check(rc, "ovx_fdg_occupancy_begin")
        vox = torch.empty((n.value, 3), dtype=torch.int32, device=triangles.device)
        rc = self._lib.ovx_fdg_occupancy_finish(self.handle, st, ctypes.c_void_p(vox.data_ptr() if vox.numel() else 0))
        self._check(rc, "ovx_fdg_occupancy_finish")
        return vox


def occupancy_noalloc(triangles, voxel_size, grid_range, capacity=None, stream=None):
    """Allocation-free occupancy (ovx_fdg_occupancy_noalloc): the library uses
    only its fixed internal scratch; the output buffer is allocated here by
    torch on behalf of the caller.  Returns (status, N, voxels[:N])."""
    import torch

    dev = triangles.device
    st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)
    grid = make_grid(voxel_size, grid_range)
    if capacity is None:
        capacity = 4 * 1024 * 1024
    out = torch.empty((max(capacity, 1), 3), dtype=torch.int32, device=dev)
    n = ctypes.c_int64(0)
    rc = lib().ovx_fdg_occupancy_noalloc(st, ctypes.c_void_p(triangles.data_ptr() if triangles.numel() else 0),
                                         triangles.shape[0], ctypes.byref(grid), ctypes.c_void_p(out.data_ptr()),
                                         capacity, ctypes.byref(n))
    return rc, n.value, out[: min(n.value, capacity)]
