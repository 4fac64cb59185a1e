"""Work shapes (ovx_fdg_tuning) change speed only: conversions under extreme
shapes -- every pair cut into units, every face box on the large-triangle
pass, every item tested by the whole warp, every boundary edge walked by a
warp, and the opposite extremes -- and the tuned table's shapes equal the
defaults' results bit for bit."""
import numpy as np
import pytest

import fdg_workloads as W

EXTREMES = [
    {"unit_cells": 8, "warp_scan_cells": 1, "inline_face_bricks": 1, "dense_candidates": 0, "long_walk": 1},
    {"unit_cells": 4096, "warp_scan_cells": 1 << 20, "inline_face_bricks": 4096, "dense_candidates": 512, "long_walk": 1 << 20},
    {"unit_cells": 128, "warp_scan_cells": 512, "inline_face_bricks": 16, "dense_candidates": 64, "long_walk": 32},
]


def _args(w):
    import torch

    ab = np.asarray(w.aabb, np.float32).reshape(2, 3)
    g = np.broadcast_to(np.asarray(w.grid_size, np.int32), (3,))
    vs = ((ab[1] - ab[0]) / g.astype(np.float32)).astype(np.float32)
    dev = torch.device("cuda:0")
    return (torch.from_numpy(w.vertices).to(dev), torch.from_numpy(w.faces).to(dev), ab[0], vs,
            [0, 0, 0, int(g[0]), int(g[1]), int(g[2])], w.face_weight, w.boundary_weight, w.regularization_weight)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ico_cap", "lowpoly256", "primitives40k"])
def test_shapes_do_not_change_results(cuda, name):
    import torch
    import ovx_fdg_abi as abi

    w = {"ico_cap": lambda: W.ico_cap(0), "lowpoly256": lambda: W.lowpoly(5, faces_total=600, grid_size=256),
         "primitives40k": lambda: W.primitives(3, faces_total=40_000)}[name]()
    a = _args(w)
    ctx = abi.Context(cuda.index or 0)
    try:
        want = [t.clone() for t in ctx.mesh_to_fdg(*a)]
        from o_voxel.convert import _tuning

        table = [dict(zip(_tuning.FIELDS, values)) for _, values in _tuning.table()]
        for shapes in EXTREMES + table:
            ctx.set_tuning(shapes)
            assert ctx.get_tuning() == shapes
            got = ctx.mesh_to_fdg(*a)
            for x, y in zip(got, want):
                assert torch.equal(x, y), (name, shapes)
        ctx.set_tuning(None)
        assert ctx.get_tuning() == {"unit_cells": 64, "warp_scan_cells": 256, "inline_face_bricks": 8,
                                    "dense_candidates": 32, "long_walk": 64}
        with pytest.raises(abi.FdgError):
            ctx.set_tuning({"unit_cells": 4})
    finally:
        ctx.close()
