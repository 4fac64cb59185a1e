"""Work-shape tuner for the flexible-dual-grid conversion (ovx_fdg_tuning).

For each grid-size bucket (64, 128, 256, 512, 1024) it builds seeded meshes
like the mixed-batch workload (primitive soups, face counts log-uniform in
1k-500k, per-mesh aabb) at that grid, plus the 282k-face primitives mesh on
the unit box (counted twice), and times their conversions through the
C ABI (CUDA events, device-resident inputs) while it searches the five shape
values by coordinate descent from the library defaults: each value in turn is
set to each of its candidates, and the fastest setting is kept when it beats
the current one by more than 1%; two passes.  The defaults and the chosen
shapes are then timed again side by side, and a bucket keeps the defaults
unless its tuned shapes measured faster.  Shapes change speed, not results.

Writes o_voxel/tuning.json, which o_voxel reads to set the shapes per call by
the grid's largest extent.  Run on the GPU that will convert:

    python o-voxel-gpu_b200/fdg_tune.py [--buckets 64,128,256,512,1024] [--meshes 6]
"""
import argparse
import json
import os
import statistics
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

FIELDS = ("unit_cells", "warp_scan_cells", "inline_face_bricks", "dense_candidates", "long_walk")
DEFAULTS = {"unit_cells": 64, "warp_scan_cells": 256, "inline_face_bricks": 8, "dense_candidates": 32, "long_walk": 64}
CANDIDATES = {
    "unit_cells": (32, 64, 128, 256),
    "warp_scan_cells": (128, 256, 512, 1024),
    "inline_face_bricks": (4, 8, 16, 32),
    "dense_candidates": (16, 32, 64),
    "long_walk": (32, 64, 128),
}
OUT = os.path.join(HERE, "o_voxel", "tuning.json")


def grid_args(w):
    """float32 voxel size (aabb1 - aabb0) / grid, grid_range [0, 0, 0, g...], origin aabb0."""
    import numpy as np

    ab = np.asarray(w.aabb, dtype=np.float32).reshape(2, 3)
    g = np.broadcast_to(np.asarray(w.grid_size, dtype=np.int32), (3,))
    vs = ((ab[1] - ab[0]) / g.astype(np.float32)).astype(np.float32)
    return ab[0], vs, [0, 0, 0, int(g[0]), int(g[1]), int(g[2])]


class Bucket:
    """The seeded meshes of one grid bucket, on the device, and a timer for them."""

    def __init__(self, grid, n_meshes, dev):
        import torch

        import fdg_workloads as W

        self.grid = grid
        self.ws = W.batch(seed=100 + grid, n_meshes=n_meshes, f_lo=1_000, f_hi=500_000, grids=(grid,))
        # and the 282k-face primitives mesh on the unit box at this grid, twice (it is the single-mesh headline case)
        p = W.primitives(1)
        p.grid_size = grid
        self.ws += [p, p]
        self.args = []
        for w in self.ws:
            origin, vs, gr = grid_args(w)
            self.args.append((torch.from_numpy(w.vertices).to(dev), torch.from_numpy(w.faces).to(dev), origin, vs, gr,
                              w.face_weight, w.boundary_weight, w.regularization_weight))
        self.faces = sum(w.num_faces for w in self.ws)

    def time_ms(self, ctx, reps=2):
        """Sum over the meshes of the median device time of `reps` conversions (after one warm-up each)."""
        import torch

        total = 0.0
        for v, f, origin, vs, gr, fw, bw, rw in self.args:
            ctx.mesh_to_fdg(v, f, origin, vs, gr, fw, bw, rw, check=False)
            ms = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                ctx.mesh_to_fdg(v, f, origin, vs, gr, fw, bw, rw, check=False)
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            total += statistics.median(ms)
        return total


def tune_bucket(b, ctx, passes=2, log=print):
    best = dict(DEFAULTS)
    ctx.set_tuning(best)
    best_ms = b.time_ms(ctx)
    log(f"grid {b.grid}: defaults {best_ms:.2f} ms")
    for p in range(passes):
        changed = False
        for name in FIELDS:
            for cand in CANDIDATES[name]:
                if cand == best[name]:
                    continue
                trial = dict(best, **{name: cand})
                ctx.set_tuning(trial)
                ms = b.time_ms(ctx)
                if ms < best_ms * 0.99:
                    best, best_ms, changed = trial, ms, True
                    log(f"grid {b.grid}: pass {p} {name}={cand} {ms:.2f} ms")
        if not changed:
            break
    # defaults and the choice side by side, three times each
    ctx.set_tuning(DEFAULTS)
    d = [b.time_ms(ctx, reps=3) for _ in range(3)]
    ctx.set_tuning(best)
    t = [b.time_ms(ctx, reps=3) for _ in range(3)]
    d_ms, t_ms = statistics.median(d), statistics.median(t)
    if t_ms >= d_ms:
        best, t_ms = dict(DEFAULTS), d_ms
    return best, d_ms, t_ms


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--buckets", default="64,128,256,512,1024")
    ap.add_argument("--meshes", type=int, default=6, help="seeded meshes per bucket")
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args(argv)

    import torch

    import ovx_fdg_abi as abi

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    ctx = abi.Context(0)
    t0 = time.time()
    buckets = []
    for g in (int(x) for x in args.buckets.split(",")):
        b = Bucket(g, args.meshes, dev)
        best, d_ms, t_ms = tune_bucket(b, ctx, log=lambda m: print(m, file=sys.stderr, flush=True))
        buckets.append({"max_grid": g, "tuning": best, "default_ms": d_ms, "tuned_ms": t_ms, "meshes": len(b.ws),
                        "faces": int(b.faces)})
        del b
        torch.cuda.empty_cache()
    ctx.close()
    out = {"device": torch.cuda.get_device_name(dev), "seconds": time.time() - t0,
           "method": "coordinate descent from the defaults, 2 passes, 1% acceptance; per bucket the sum over seeded "
                     "meshes of the median conversion time", "command": "python o-voxel-gpu_b200/fdg_tune.py",
           "buckets": buckets}
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
