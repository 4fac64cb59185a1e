"""B200-native drop-in for the mesh -> flexible dual grid path of ``o_voxel``.

Only the conversion path is provided (``o_voxel.convert.mesh_to_flexible_dual_grid``,
its batched form and ``o_voxel.convert.intersect_occ``) plus the z-order codes of
``o_voxel.serialize`` that order its output; it runs on CUDA tensors through the
``o_voxel._C`` extension and the ``libovx_fdg`` C ABI.
"""
from . import convert  # noqa: F401
from . import serialize  # noqa: F401

__all__ = ["convert", "serialize"]
