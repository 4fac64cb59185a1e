"""Work shapes of the conversions (ovx_fdg_tuning) by grid size.

The table o_voxel/tuning.json is written by the project's tuner
(o-voxel-gpu_b200/fdg_tune.py), which times conversions of seeded meshes of
each grid-size bucket on the GPU over a set of candidate shapes.  Each bucket
holds the largest grid extent it covers and the five shape values in
ovx_fdg_tuning field order.  The values change speed only, never results.
Without the table (or with OVX_FDG_TUNING=off) the library defaults are used.
"""
import json
import os

FIELDS = ("unit_cells", "warp_scan_cells", "inline_face_bricks", "dense_candidates", "long_walk")
PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tuning.json")

_TABLE = None
_APPLIED = {}


def table():
    """[(max_grid, values), ...] sorted by max_grid; empty without a table."""
    global _TABLE
    if _TABLE is None:
        rows = []
        if os.environ.get("OVX_FDG_TUNING", "").lower() != "off" and os.path.exists(PATH):
            with open(PATH) as f:
                data = json.load(f)
            for b in data.get("buckets", []):
                rows.append((int(b["max_grid"]), tuple(int(b["tuning"][k]) for k in FIELDS)))
        _TABLE = sorted(rows)
    return _TABLE


def values_for(grid_extent: int):
    """Shape values for a grid whose largest extent is grid_extent (() = defaults)."""
    rows = table()
    for max_grid, values in rows:
        if grid_extent <= max_grid:
            return values
    return rows[-1][1] if rows else ()


def apply(ext, device: int, grid_extent: int):
    """Sets the shapes of the device's conversion contexts for a grid of this
    extent, when they differ from the ones set last."""
    values = values_for(int(grid_extent))
    if _APPLIED.get(device) != values:
        ext.set_tuning_cuda(int(device), list(values))
        _APPLIED[device] = values
