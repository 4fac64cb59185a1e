"""B200-native drop-in for the mesh -> flexible dual grid path of ``o_voxel``.

Only the conversion path is provided (``o_voxel.convert.mesh_to_flexible_dual_grid``
and ``o_voxel.convert.intersect_occ``); it runs on CUDA tensors through the
``o_voxel._C`` extension and the ``libovx_fdg`` C ABI.
"""
from . import convert  # noqa: F401

__all__ = ["convert"]
