"""ctypes front end of the CPU oracle (test infrastructure only).

Only the tests, the smoke check and the CPU-baseline leg of ``bench.py`` use
this module; the product never imports it.

* ``mesh_to_fdg``      -- the plain-C restatement (``fdg_oracle.c``) of the
                          reference CPU path, ``precision="f32"`` (exact) or
                          ``"f64"`` (FP64 quadrics, accumulation and solve).
* ``intersect_occ``    -- occupancy only.
* ``ref_module``       -- the reference's own CPU source compiled against the
                          Eigen-API shim (``oracle/_ref``), when it was built.
* ``grid_args``        -- the reference Python wrapper's argument derivation
                          (``o_voxel/convert/flexible_dual_grid.py:88-181``) for the
                          ``grid_size`` + ``aabb`` form, in numpy float32.
"""
from __future__ import annotations

import ctypes
import importlib.machinery
import importlib.util
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Out(ctypes.Structure):
    _fields_ = [
        ("num_voxels", ctypes.c_int64),
        ("voxels", ctypes.c_void_p),
        ("dual", ctypes.c_void_p),
        ("intersected", ctypes.c_void_p),
        ("qef", ctypes.c_void_p),
        ("mean_sum", ctypes.c_void_p),
        ("cnt", ctypes.c_void_p),
        ("num_boundary_edges", ctypes.c_int64),
        ("elem_size", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(HERE, "libfdg_oracle.so")
        if not os.path.exists(so):
            from . import build as _b  # type: ignore

            _b.build_oracle()
        _LIB = ctypes.CDLL(so)
        for name in ("fdg_oracle_mesh_to_fdg_f32", "fdg_oracle_mesh_to_fdg_f64"):
            fn = getattr(_LIB, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.POINTER(_Out)]
        _LIB.fdg_oracle_intersect_occ.restype = ctypes.c_int
        _LIB.fdg_oracle_intersect_occ.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_void_p)]
        _LIB.fdg_oracle_free.argtypes = [ctypes.POINTER(_Out)]
        _LIB.fdg_oracle_free_ptr.argtypes = [ctypes.c_void_p]
        _LIB.fdg_oracle_z_order_encode.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4
        _LIB.fdg_oracle_z_order_decode.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4
        _LIB.fdg_oracle_hilbert_encode.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4
        _LIB.fdg_oracle_hilbert_decode.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4
    return _LIB


def z_order_encode(x, y, z) -> np.ndarray:
    """Oracle z-order codes (int32) of int coordinates in [0, 1024)."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.int32) for a in (x, y, z))
    out = np.empty(x.shape[0], dtype=np.int32)
    lib().fdg_oracle_z_order_encode(x.shape[0], x.ctypes.data, y.ctypes.data, z.ctypes.data, out.ctypes.data)
    return out


def z_order_decode(codes):
    codes = np.ascontiguousarray(codes, dtype=np.int32)
    x, y, z = (np.empty(codes.shape[0], dtype=np.int32) for _ in range(3))
    lib().fdg_oracle_z_order_decode(codes.shape[0], codes.ctypes.data, x.ctypes.data, y.ctypes.data, z.ctypes.data)
    return x, y, z


def hilbert_encode(x, y, z) -> np.ndarray:
    """Oracle Hilbert codes (int32) of int coordinates in [0, 1024)."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.int32) for a in (x, y, z))
    out = np.empty(x.shape[0], dtype=np.int32)
    lib().fdg_oracle_hilbert_encode(x.shape[0], x.ctypes.data, y.ctypes.data, z.ctypes.data, out.ctypes.data)
    return out


def hilbert_decode(codes):
    codes = np.ascontiguousarray(codes, dtype=np.int32)
    x, y, z = (np.empty(codes.shape[0], dtype=np.int32) for _ in range(3))
    lib().fdg_oracle_hilbert_decode(codes.shape[0], codes.ctypes.data, x.ctypes.data, y.ctypes.data, z.ctypes.data)
    return x, y, z


def ref_hilbert_lib():
    """The reference's own CPU Hilbert functions (oracle/_ref/hilbert_ref.so), or None if not built."""
    so = os.path.join(HERE, "_ref", "hilbert_ref.so")
    if not os.path.exists(so):
        return None
    L = ctypes.CDLL(so)
    L.ref_hilbert_encode.argtypes = [ctypes.c_size_t] + [ctypes.c_void_p] * 4
    L.ref_hilbert_decode.argtypes = [ctypes.c_size_t] + [ctypes.c_void_p] * 4
    return L


def ref_z_order_lib():
    """The reference's own CPU z-order functions (oracle/_ref/zorder_ref.so), or None if not built."""
    so = os.path.join(HERE, "_ref", "zorder_ref.so")
    if not os.path.exists(so):
        return None
    L = ctypes.CDLL(so)
    L.ref_z_order_encode.argtypes = [ctypes.c_size_t] + [ctypes.c_void_p] * 4
    L.ref_z_order_decode.argtypes = [ctypes.c_size_t] + [ctypes.c_void_p] * 4
    return L


@dataclass
class OracleResult:
    voxels: np.ndarray  # [N,3] int32, insertion order
    dual: np.ndarray  # [N,3]
    intersected: np.ndarray  # [N,3] bool
    qef: np.ndarray  # [N,10] accumulated quadric before regularisation
    mean_sum: np.ndarray  # [N,3]
    cnt: np.ndarray  # [N]
    num_boundary_edges: int


def _copy(ptr, dtype, shape):
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype)
    buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype).reshape(shape).copy()


def mesh_to_fdg(vertices, faces, voxel_size, grid_range, face_weight, boundary_weight, regularization_weight,
                precision="f32") -> OracleResult:
    """Run the oracle on grid-local (already shifted) float32 vertices and int faces."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    vs = np.ascontiguousarray(voxel_size, dtype=np.float32)
    gr = np.ascontiguousarray(grid_range, dtype=np.int32)
    out = _Out()
    fn = lib().fdg_oracle_mesh_to_fdg_f32 if precision == "f32" else lib().fdg_oracle_mesh_to_fdg_f64
    rc = fn(v.ctypes.data, v.shape[0], f.ctypes.data, f.shape[0], vs.ctypes.data, gr.ctypes.data,
            float(face_weight), float(boundary_weight), float(regularization_weight), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    try:
        n = out.num_voxels
        rdt = np.float32 if out.elem_size == 4 else np.float64
        return OracleResult(
            voxels=_copy(out.voxels, np.int32, (n, 3)),
            dual=_copy(out.dual, rdt, (n, 3)),
            intersected=_copy(out.intersected, np.uint8, (n, 3)).astype(bool),
            qef=_copy(out.qef, rdt, (n, 10)),
            mean_sum=_copy(out.mean_sum, rdt, (n, 3)),
            cnt=_copy(out.cnt, rdt, (n,)),
            num_boundary_edges=int(out.num_boundary_edges),
        )
    finally:
        lib().fdg_oracle_free(ctypes.byref(out))


def intersect_occ(triangles, voxel_size, grid_range) -> np.ndarray:
    t = np.ascontiguousarray(triangles, dtype=np.float32).reshape(-1, 9)
    vs = np.ascontiguousarray(voxel_size, dtype=np.float32)
    gr = np.ascontiguousarray(grid_range, dtype=np.int32)
    n = ctypes.c_int64(0)
    p = ctypes.c_void_p(0)
    rc = lib().fdg_oracle_intersect_occ(t.ctypes.data, t.shape[0], vs.ctypes.data, gr.ctypes.data, ctypes.byref(n),
                                        ctypes.byref(p))
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    try:
        return _copy(p.value, np.int32, (n.value, 3)) if n.value else np.zeros((0, 3), np.int32)
    finally:
        lib().fdg_oracle_free_ptr(p)


def grid_args(vertices, faces, grid_size, aabb):
    """Reference wrapper derivation for the grid_size+aabb form: float32
    voxel_size = (aabb1 - aabb0) / grid, grid_range = [0,0,0,gx,gy,gz], vertices
    shifted by aabb0 in float32, faces cast to int32."""
    g = np.array([grid_size] * 3 if np.isscalar(grid_size) else grid_size, dtype=np.int32)
    ab = np.asarray(aabb, dtype=np.float32).reshape(2, 3)
    vs = ((ab[1] - ab[0]) / g.astype(np.float32)).astype(np.float32)
    gr = np.array([0, 0, 0, g[0], g[1], g[2]], dtype=np.int32)
    v = (np.asarray(vertices, dtype=np.float32) - ab[0].reshape(1, 3)).astype(np.float32)
    f = np.asarray(faces).astype(np.int32)
    return v, f, vs, gr


def run_workload(w, precision="f32") -> OracleResult:
    v, f, vs, gr = grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
    return mesh_to_fdg(v, f, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight, precision)


_REF = "unset"


def ref_module():
    """The reference CPU source compiled against the Eigen shim, or None if it was not built."""
    global _REF
    if _REF == "unset":
        import sysconfig

        path = os.path.join(HERE, "_ref", "fdg_ref" + sysconfig.get_config_var("EXT_SUFFIX"))
        if not os.path.exists(path):
            _REF = None
        else:
            import torch  # noqa: F401  (provides libtorch symbols)

            loader = importlib.machinery.ExtensionFileLoader("fdg_ref", path)
            spec = importlib.util.spec_from_file_location("fdg_ref", path, loader=loader)
            mod = importlib.util.module_from_spec(spec)
            loader.exec_module(mod)
            _REF = mod
    return _REF


def ref_mesh_to_fdg(vertices, faces, voxel_size, grid_range, fw, bw, rw):
    import torch

    m = ref_module()
    if m is None:
        raise RuntimeError("reference CPU path not built (oracle/_ref)")
    vt = torch.from_numpy(np.ascontiguousarray(vertices, dtype=np.float32))
    ft = torch.from_numpy(np.ascontiguousarray(faces, dtype=np.int32))
    vox, dual, inter = m.mesh_to_flexible_dual_grid_cpu(vt, ft, [float(x) for x in voxel_size],
                                                        [int(x) for x in grid_range], float(fw), float(bw), float(rw),
                                                        False)
    return vox.numpy(), dual.numpy(), inter.numpy()
