"""Run one synthetic workload through the C ABI a few times and report timings.

    python o-voxel-gpu_b200/fdg_run.py --workload primitives --conversions 3
    python o-voxel-gpu_b200/fdg_run.py --workload subdivided --grid 1024 --stages

Workloads: ico_cap (5120 faces, grid 64), primitives (282k faces, grid 512),
subdivided (10.3M faces, grid 512 or 1024), sheets (precision stress, grid 1024),
lowpoly (about 1200 large faces, grid 512 or 1024).
Every conversion goes through ovx_fdg_begin/ovx_fdg_finish on the current
stream; with --stages the last conversion is repeated with the library's stage
timers on.  Prints one JSON line.  This is the command the kernel launch lists
and DRAM-traffic captures under profiles/ were taken with.
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def make_workload(name: str, grid: int = 0):
    import fdg_workloads as W

    if name == "ico_cap":
        return W.ico_cap(0)
    if name == "primitives":
        return W.primitives(1)
    if name == "subdivided":
        return W.subdivided(1, grid_size=grid or 512)
    if name == "sheets":
        return W.sheets(3)
    if name == "lowpoly":
        return W.lowpoly(5, grid_size=grid or 512)
    raise SystemExit(f"unknown workload {name}")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", default="primitives")
    ap.add_argument("--grid", type=int, default=0, help="grid size for the subdivided workload (512 or 1024)")
    ap.add_argument("--conversions", type=int, default=3)
    ap.add_argument("--stages", action="store_true")
    args = ap.parse_args(argv)

    import torch

    import ovx_fdg_abi as abi

    w = make_workload(args.workload, args.grid)
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    import numpy as np

    kw = w.kwargs()
    # wrapper derivation for the grid_size + aabb form: float32 voxel size, origin aabb[0]
    ab = np.asarray(kw["aabb"], dtype=np.float32).reshape(2, 3)
    g = np.full(3, kw["grid_size"], dtype=np.int32)
    vs = (ab[1] - ab[0]) / g.astype(np.float32)
    grid_range = [0, 0, 0, int(g[0]), int(g[1]), int(g[2])]
    aabb0 = ab[0]
    v = torch.from_numpy(w.vertices).to(dev)
    f = torch.from_numpy(w.faces).to(dev)
    ctx = abi.Context(0)
    times = []
    n = 0
    for _ in range(max(1, args.conversions)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        vox, _, _ = ctx.mesh_to_fdg(v, f, aabb0, vs, grid_range, kw["face_weight"], kw["boundary_weight"],
                                    kw["regularization_weight"])
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        n = vox.shape[0]
    out = {"workload": w.name, "faces": int(w.num_faces), "vertices": int(w.vertices.shape[0]),
           "grid": int(w.grid_size), "voxels": int(n), "ms": times,
           "launches_per_conversion": ctx.kernel_launches() // max(1, args.conversions),
           "workspace_bytes": ctx.workspace_bytes(), "counts": ctx.last_counts()}
    if args.stages:
        ctx.set_profiling(True)
        ctx.mesh_to_fdg(v, f, aabb0, vs, grid_range, kw["face_weight"], kw["boundary_weight"],
                        kw["regularization_weight"])
        out["stage_ms"] = ctx.stage_times()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
