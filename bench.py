"""Benchmark: mesh -> flexible dual grid on B200.

One step = one full conversion (occupancy, quadrics, solve) of the seeded
282k-face / grid-512 primitives mesh (the reference's headline single-mesh
case; its asset is not distributed, so a synthetic stand-in with the same
size is used).  Prints one JSON line on rank 0.

  value      Mfaces/s with inputs resident in HBM, through the C ABI
             (libovx_fdg), CUDA events per step, L2 flushed between steps
  e2e        the same metric through o_voxel.convert.mesh_to_flexible_dual_grid
             with pinned host inputs: H2D copy, conversion, D2H of all outputs
  roofline   compulsory bytes of a conversion (12V + 8*3F + 27N) over the
             conversion time against the measured HBM copy bandwidth
  workloads  the 10.3M-face subdivided mesh at grid 512, timed the same way,
             with its own roofline and memory
  reference_gpu  the reference's own CUDA implementation of the path: not
             run (it stalled on the 282k-face mesh; see REFERENCE_GPU_UNAVAILABLE)
  cpu_baseline  the reference's CPU implementation on the host cores: every
             core converts the full 282k-face mesh once
  batched    256 mixed meshes (grids 64-512): the batched API against one
             call per mesh, meshes/s of each (single GPU only)

--impl reference times the reference CPU implementation alone, on the same
mesh: one step = every host core converts the full mesh once.

--workload NAME [--grid G] [--stages] runs one synthetic workload a few times
through the C ABI and prints its own JSON line (per-workload timings; the
command the ncu captures under profiles/ name).

Multi-GPU: replicas only (each rank converts its own copy; no collective).
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "o-voxel-gpu_b200"))
sys.path.insert(0, REPO)

METRIC = "Mfaces/s & meshes/s mesh→FDG @grid512, batched vs plain GPU, exact occ"
# reference CUDA path as published: 280k faces at grid 512 in 27.1 ms on an RTX 4090 (README.md:39)
PUBLISHED_MFACES = 10.3
HEADLINE = "primitives-282k-faces-grid512"
LARGE = "subdivided-10.3M-faces-grid512"
CPU_BUDGET_S = 150.0  # timed CPU reference steps stop once this much time has gone


_T0 = time.perf_counter()


def progress(msg):
    """One timestamped progress line on stderr (the JSON result goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def load_workload(name=HEADLINE):
    import fdg_workloads as W

    if name == HEADLINE:
        return W.primitives(1)
    if name == LARGE:
        return W.subdivided(1, grid_size=512)
    raise ValueError(name)


def grid_args(w):
    """The reference wrapper's derivation for the grid_size + aabb form
    (o_voxel/convert/flexible_dual_grid.py:161-178): float32 voxel size
    (aabb1 - aabb0) / grid, grid_range [0, 0, 0, g...], origin aabb0."""
    import numpy as np

    ab = np.asarray(w.aabb, dtype=np.float32).reshape(2, 3)
    g = np.broadcast_to(np.asarray(w.grid_size, dtype=np.int32), (3,))
    vs = ((ab[1] - ab[0]) / g.astype(np.float32)).astype(np.float32)
    return ab[0], vs, [0, 0, 0, int(g[0]), int(g[1]), int(g[2])]


def apply_tuned_shapes(ctx, w):
    """The library's tuned work shapes (o_voxel/tuning.json) for this workload's
    grid, as the o_voxel wrapper applies them, on a C-ABI context."""
    from o_voxel.convert import _tuning

    values = _tuning.values_for(max(grid_args(w)[2][3:]))
    ctx.set_tuning(dict(zip(_tuning.FIELDS, values)) if values else None)


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(V, F, N, face_bytes=8):
    """Compulsory I/O of one conversion: vertices in, faces in, voxels, dual
    vertices and flags out (12V + 3F x face index bytes + 27N)."""
    return 12 * V + face_bytes * 3 * F + 27 * N


def headline_config(w, voxels: int, world: int) -> dict:
    """The workload description both arms report, key for key."""
    return {"workload": HEADLINE, "faces": int(w.num_faces), "vertices": int(w.vertices.shape[0]), "voxels": int(voxels),
            "grid": 512, "weights": [w.face_weight, w.boundary_weight, w.regularization_weight], "faces_dtype": "int64",
            "l2": "GPU arm: flushed between steps by a 256 MB write outside the timed events; CPU arm: host code, "
                  "no GPU cache involved",
            "parallelism": f"replicas x{world}"}


# ----------------------------------------------------------------------------- CPU baseline
def _ref_worker(args):
    """Runs in a spawned process: one conversion of the mesh by the reference CPU code."""
    kind, v, f, vs, gr, fw, bw, rw = args
    sys.path.insert(0, REPO)
    from oracle import oracle as O

    t0 = time.perf_counter()
    if kind == "reference":
        vox = O.ref_mesh_to_fdg(v, f, vs, gr, fw, bw, rw)[0]
    else:
        vox = O.mesh_to_fdg(v, f, vs, gr, fw, bw, rw).voxels
    return time.perf_counter() - t0, int(vox.shape[0])


REF_PROCESS_BYTES = 2 << 30  # one full-mesh reference conversion peaks at about 1.6 GB of host memory


def cpu_processes():
    """Host cores to run reference conversions on: every core, at most 32, and
    no more than the available host memory holds at REF_PROCESS_BYTES each."""
    n = os.cpu_count() or 1
    try:
        import psutil

        n = min(n, max(1, int(psutil.virtual_memory().available // REF_PROCESS_BYTES)))
    except Exception:
        pass
    return max(1, min(n, 32))


class CpuBaseline:
    """The reference CPU implementation on all host cores.  The reference CPU
    path is single-threaded (flexible_dual_grid.cpp:660-992), so a step runs
    one full conversion of the mesh on every core at once: the step's wall
    time gives the throughput of the whole host, each process's own time the
    latency of one conversion."""

    def __init__(self, w, cores=None):
        from oracle import oracle as O

        self.kind = "reference" if O.ref_module() is not None else "port"
        v, f, vs, gr = O.grid_args(w.vertices, w.faces, w.grid_size, w.aabb)
        self.faces = int(f.shape[0])
        self.cores = cores or cpu_processes()
        self.job = (self.kind, v, f, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        self.pool = mp.get_context("spawn").Pool(self.cores)
        self.latencies = []
        self.voxels = 0

    def step(self):
        t0 = time.perf_counter()
        res = self.pool.map(_ref_worker, [self.job] * self.cores)
        wall = time.perf_counter() - t0
        self.latencies.extend(r[0] for r in res)
        self.voxels = res[0][1]
        return wall

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self, value):
        src = ("reference src/convert/flexible_dual_grid.cpp built against the Eigen-API shim" if self.kind == "reference"
               else "C restatement of it")
        return {"value": value, "unit": "Mfaces/s", "cores": self.cores, "kind": self.kind,
                "latency_ms": 1e3 * statistics.median(self.latencies) if self.latencies else None,
                "latency_note": "one single-threaded conversion of the full mesh, median over the processes of the timed steps",
                "sample": f"the full {self.faces}-face grid-512 mesh, one conversion per core per step, {self.cores} cores ({src})"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                  "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        while not self._stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            self.samples.append([x.strip() for x in line.split(",")])
        p.terminate()
        try:
            p.wait(timeout=5)
        except Exception:
            p.kill()

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, name in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    """The reference CPU implementation alone, on the headline mesh.  A step
    converts the full mesh once on every host core; the first step warms the
    processes.  A CPU step takes tens of seconds, so the timed steps stop after
    CPU_BUDGET_S (at least two), and the line reports the steps that ran."""
    if rank != 0:
        return
    w = load_workload()
    progress("reference arm: starting the CPU process pool")
    cb = CpuBaseline(w)
    warm = min(args.warmup, 1)
    for _ in range(warm):
        cb.step()
    cb.latencies.clear()
    times = []
    t_start = time.perf_counter()
    while len(times) < args.steps and (len(times) < 2 or time.perf_counter() - t_start < CPU_BUDGET_S):
        times.append(cb.step())
        progress(f"reference arm: step {len(times)} took {times[-1]:.1f} s")
    cb.close()
    t = sum(times) / len(times)
    value = cb.cores * cb.faces / t / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mfaces/s", "n_gpus": args.gpus,
            "steps": len(times), "warmup": warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "steps_note": f"a step converts the full mesh on every core ({t:.1f} s); timed steps stop after {CPU_BUDGET_S:.0f} s "
                          f"(at least two) and one warm-up step is run, so that the run ends within minutes",
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64,f32",
            "data": "synthetic: seeded 48-primitive mesh (no dataset on the box)",
            "config": headline_config(w, cb.voxels, args.gpus),
            "cpu_baseline": cb.describe(value),
            "e2e": {"value": value, "unit": "Mfaces/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- batched workload
def run_batched(dev, steps=10, warmup=2):
    """256 seeded meshes built like the 282k-face one, face counts log-uniform in
    [1k, 500k] (about 21M faces in all), grid 64/128/256/512 per mesh, per-mesh
    aabb: the batched API against the same meshes converted one call at a time."""
    import torch

    import fdg_workloads as W
    import o_voxel

    ws = W.batch(4)
    meshes = [(torch.from_numpy(w.vertices).to(dev), torch.from_numpy(w.faces).to(dev)) for w in ws]
    F = sum(w.num_faces for w in ws)
    kw = dict(face_weight=1.0, boundary_weight=0.2, regularization_weight=1e-2)
    grids = [w.grid_size for w in ws]
    aabbs = [w.aabb for w in ws]

    def plain():
        for (v, f), w in zip(meshes, ws):
            o_voxel.convert.mesh_to_flexible_dual_grid(v, f, grid_size=w.grid_size, aabb=w.aabb, **kw)

    def batched():
        o_voxel.convert.mesh_to_flexible_dual_grid_batch(meshes, grid_size=grids, aabb=aabbs, **kw)

    def timed(fn):
        # the contexts reach their largest workspaces during the warm-up
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms), ms

    t_plain, plain_ms = timed(plain)
    t_batch, batch_ms = timed(batched)
    return {"workload": "256 meshes, faces log-uniform 1k-500k, grids 64-512, per-mesh aabb",
            "meshes": len(ws), "faces": int(F), "steps": steps, "warmup": warmup,
            "timing": "median of the steps (CUDA events on the caller's stream, host included)",
            "plain_step_ms": plain_ms, "batched_step_ms": batch_ms,
            "plain_ms": t_plain, "plain_spread_ms": [min(plain_ms), max(plain_ms)],
            "plain_meshes_per_s": len(ws) / (t_plain / 1e3),
            "batched_ms": t_batch, "batched_spread_ms": [min(batch_ms), max(batch_ms)],
            "batched_meshes_per_s": len(ws) / (t_batch / 1e3),
            "batched_mfaces_per_s": F / (t_batch / 1e3) / 1e6, "speedup": t_plain / t_batch,
            "api": "o_voxel.convert.mesh_to_flexible_dual_grid_batch (one pipeline per group of meshes, default "
                   "max_group_records) vs one mesh_to_flexible_dual_grid call per mesh"}


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(ms: float, world: int, device) -> float:
    """The largest of the ranks' times (every rank calls this, in the same
    order); the tensor lives on `device` (CUDA under NCCL, CPU under gloo)."""
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(faces: int, world: int, ms_per_step: float) -> float:
    """Whole-job Mfaces/s of `world` replicas, each converting `faces` faces per
    step, timed by the slowest rank."""
    return world * faces / (ms_per_step / 1e3) / 1e6


# ----------------------------------------------------------------------------- timing helpers
def time_steps(fn, steps, stream, flush):
    """Per-step device times (ms) of fn() with CUDA events on `stream`, the L2
    flushed (a 256 MB write) before every step, outside the events."""
    import torch

    ms = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


REFERENCE_GPU_UNAVAILABLE = (
    "not run: the reference's CUDA path (built from its sources by baseline/build_ref_gpu.py, sm_100) gave no result "
    "for over 25 minutes on the 282k-face mesh and was killed; the same benchmark without it finished in 30 s. "
    "Its brick-publication wait (src/convert/mesh_to_flexible_dual_grid_gpu/intersect_qef.cu:364-373) has no bound, "
    "so it is not run again on the shared GPUs")


# ----------------------------------------------------------------------------- our arm
def measure_workload(name, w, dev, stream, flush, steps, ours_out=None):
    """Device-resident timing of one workload through a fresh C-ABI context
    (cold first call, then warm steps), its roofline and memory."""
    import torch

    import ovx_fdg_abi as abi

    F, V = w.num_faces, w.vertices.shape[0]
    origin, vs, gr = grid_args(w)
    vd = torch.from_numpy(w.vertices).to(dev)
    fd = torch.from_numpy(w.faces).to(dev)
    ctx = abi.Context(dev.index)
    apply_tuned_shapes(ctx, w)
    kw = (origin, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
    one = lambda: ctx.mesh_to_fdg(vd, fd, *kw, check=False)  # noqa: E731
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    out = one()
    c1.record(stream)
    c1.synchronize()
    cold = c0.elapsed_time(c1)
    for _ in range(3):
        out = one()
    ms = time_steps(one, steps, stream, flush)
    progress(f"{name}: this library {statistics.median(ms):.2f} ms")
    ctx._check(abi.lib().ovx_fdg_sync_status(ctx.handle, abi.ctypes.c_void_p(stream.cuda_stream)), "status")
    N = int(out[0].shape[0])
    t = statistics.median(ms)
    peak, peak_kind = peaks()
    b_alg = algorithmic_bytes(V, F, N)
    res = {"faces": F, "vertices": V, "voxels": N, "grid": int(gr[3]), "steps": steps, "ms": t,
           "ms_spread": [min(ms), max(ms)], "mfaces_per_s": F / (t / 1e3) / 1e6, "cold_ms": cold,
           "roofline": {"bound": "hbm", "algorithmic_bytes": b_alg, "achieved": b_alg / (t / 1e3) / 1e9, "peak": peak,
                        "unit": "GB/s", "frac": b_alg / (t / 1e3) / 1e9 / peak, "peak_source": peak_kind},
           "memory": {"workspace_bytes": int(ctx.workspace_bytes()), "output_bytes": 27 * N,
                      "note": "the library's workspace after this workload on a fresh context, plus the outputs"}}
    if ours_out is not None:
        ours_out.append(out)
    ctx.close()
    return res


def run_ours(args, rank, world):
    import numpy as np
    import torch

    import ovx_fdg_abi as abi
    import o_voxel

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    w = load_workload()
    F, V = w.num_faces, w.vertices.shape[0]
    origin, vs, gr = grid_args(w)
    vd = torch.from_numpy(w.vertices).to(dev)
    fd = torch.from_numpy(w.faces).to(dev)  # int64, consumed as supplied
    ctx = abi.Context(dev.index)
    apply_tuned_shapes(ctx, w)
    kw = (origin, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def one():
        return ctx.mesh_to_fdg(vd, fd, *kw, check=False)

    # cold: the first conversion on a fresh context, workspace growth included
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    out = one()
    c1.record(stream)
    c1.synchronize()
    cold_ms = c0.elapsed_time(c1)
    for _ in range(max(args.warmup, 3)):
        out = one()
    torch.cuda.synchronize()
    N = int(out[0].shape[0])

    # device-resident timed region
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    clocks.start()
    launches0 = ctx.kernel_launches()
    progress("headline: timed region")
    ms = time_steps(one, args.steps, stream, flush)
    torch.cuda.synchronize()
    launches = ctx.kernel_launches() - launches0
    clk = clocks.stop()
    t_total = max_over_ranks(sum(ms), world, dev)
    if world > 1:
        torch.distributed.barrier()
    ms_per_step = t_total / args.steps
    value = replica_value(F, world, ms_per_step)
    ctx._check(abi.lib().ovx_fdg_sync_status(ctx.handle, abi.ctypes.c_void_p(stream.cuda_stream)), "status")

    # stage breakdown (separate, profiled conversion)
    ctx.set_profiling(True)
    flush.zero_()
    one()
    stages = ctx.stage_times()
    ctx.set_profiling(False)

    # end to end through the public API, host buffers: every step copies its
    # inputs in from pinned host memory, converts, and copies all outputs back.
    # Steps alternate between two streams so that one step's output copy
    # overlaps the next step's conversion (the library orders the conversions
    # themselves); the time is the whole run's, start to finish.
    vh = torch.from_numpy(w.vertices).pin_memory()
    fh = torch.from_numpy(w.faces).pin_memory()
    slots = [tuple(torch.empty((N, 3), dtype=dt).pin_memory() for dt in (torch.int32, torch.float32, torch.bool))
             for _ in range(2)]
    streams = [torch.cuda.Stream(dev) for _ in range(2)]

    def e2e_step(k):
        with torch.cuda.stream(streams[k % 2]):
            vdev = vh.to(dev, non_blocking=True)
            fdev = fh.to(dev, non_blocking=True)
            outs = o_voxel.convert.mesh_to_flexible_dual_grid(vdev, fdev, **w.kwargs())
            for h, d in zip(slots[k % 2], outs):
                h.copy_(d, non_blocking=True)

    def e2e_run(steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st_ in streams:
            st_.wait_event(e0)
        for k in range(steps):
            e2e_step(k)
        for st_ in streams:
            stream.wait_stream(st_)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    progress("end to end")
    e2e_run(2)
    e2e_ms = max_over_ranks(e2e_run(args.steps), world, dev) / args.steps
    e2e_value = replica_value(F, world, e2e_ms)

    if rank != 0:
        ctx.close()
        return
    peak, peak_kind = peaks()
    b_alg = algorithmic_bytes(V, F, N)
    achieved = b_alg / (ms_per_step / 1e3) / 1e9
    traffic = None
    tf = os.path.join(REPO, "profiles", "fdg_traffic.json")
    if os.path.exists(tf):
        with open(tf) as fh_:
            traffic = json.load(fh_).get("dram_bytes_per_conversion")
    total_stage = sum(x for x in stages.values() if x > 0) or 1.0
    dom = max(stages.items(), key=lambda kv: kv[1]) if stages else ("", 0.0)
    workspace = int(ctx.workspace_bytes())
    ctx.close()
    del out

    # the other workload, single GPU only
    workloads = {}
    reference_gpu = {"available": False, "why": REFERENCE_GPU_UNAVAILABLE}
    head = measure_workload(HEADLINE, w, dev, stream, flush, args.steps)
    if world == 1 and not args.no_large:
        wl = load_workload(LARGE)
        workloads[LARGE] = measure_workload(LARGE, wl, dev, stream, flush, max(3, min(args.steps, 10)))
        del wl
        torch.cuda.empty_cache()

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        progress("CPU baseline")
        cb = CpuBaseline(w)
        cpu_t = cb.step()
        cb.close()
        cpu = cb.describe(cb.cores * cb.faces / cpu_t / 1e6)
    batched = None
    if not args.no_batch and world == 1:
        progress("batched")
        batched = run_batched(dev)
    line = {
        "metric": METRIC, "value": value, "unit": "Mfaces/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_MFACES, "dtype": "f64,f32",
        "data": "synthetic: seeded 48-primitive mesh (no dataset on the box)",
        "config": headline_config(w, N, world),
        "meshes_per_s": world / (ms_per_step / 1e3),
        "batched": batched,
        "e2e": {"value": e2e_value, "unit": "Mfaces/s", "ms_per_step": e2e_ms, "h2d_bytes_per_step": 12 * V + 8 * 3 * F,
                "d2h_bytes_per_step": 27 * N, "api": "o_voxel.convert.mesh_to_flexible_dual_grid",
                "pipelining": "two streams; a step's output copy overlaps the next step's conversion; whole-run time"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "scope": "whole conversion: compulsory bytes 12V+24F+27N over the conversion time",
                     "dominant_stage": {"name": dom[0], "ms": dom[1], "share": dom[1] / total_stage}},
        "stage_ms": stages,
        "cold_ms": cold_ms,
        "memory": {"workspace_bytes": workspace, "torch_max_allocated_bytes": int(torch.cuda.max_memory_allocated(dev)),
                   "note": "workspace: the conversion context's buffers (grown to the largest conversion); torch: outputs, inputs, "
                           "the 256 MB L2 flush buffer and the batched leg"},
        "workloads": {HEADLINE: head, **workloads},
        "reference_gpu": reference_gpu,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- one workload
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


def run_one_workload(args):
    """Runs one synthetic workload through the C ABI `--conversions` times and
    prints its timings (ms per conversion, CUDA events), sizes and, with
    --stages, the stage times of one more conversion."""
    import torch

    import ovx_fdg_abi as abi

    w = make_workload(args.workload, args.grid)
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    origin, vs, gr = grid_args(w)
    v = torch.from_numpy(w.vertices).to(dev)
    f = torch.from_numpy(w.faces).to(dev)
    ctx = abi.Context(0)
    apply_tuned_shapes(ctx, w)
    times, n = [], 0
    for _ in range(max(1, args.conversions)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        vox, _, _ = ctx.mesh_to_fdg(v, f, origin, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        n = vox.shape[0]
    out = {"workload": w.name, "faces": int(w.num_faces), "vertices": int(w.vertices.shape[0]),
           "grid": int(gr[3]), "voxels": int(n), "ms": times,
           "launches_per_conversion": ctx.kernel_launches() // max(1, args.conversions),
           "workspace_bytes": ctx.workspace_bytes(), "counts": ctx.last_counts()}
    if args.stages:
        ctx.set_profiling(True)
        ctx.mesh_to_fdg(v, f, origin, vs, gr, w.face_weight, w.boundary_weight, w.regularization_weight)
        out["stage_ms"] = ctx.stage_times()
    ctx.close()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-mesh batched measurement")
    ap.add_argument("--no-large", action="store_true", help="skip the 10.3M-face workload")
    ap.add_argument("--workload", default=None, help="run one workload and print its timings instead (ico_cap, primitives, "
                                                     "subdivided, sheets, lowpoly)")
    ap.add_argument("--grid", type=int, default=0, help="grid size for --workload subdivided / lowpoly")
    ap.add_argument("--conversions", type=int, default=3, help="conversions for --workload")
    ap.add_argument("--stages", action="store_true", help="stage times for --workload")
    args = ap.parse_args()
    if args.workload:
        run_one_workload(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
