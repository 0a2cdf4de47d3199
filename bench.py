"""Throughput benchmark of the cubvh query path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rays_displaced|rays_incoherent|udf_icosphere|dense_tori|raystab_displaced|
                                grad_displaced|batch_256|sparse_mc_band]

Default workload (``rays_displaced``): displaced icosphere level 6 (81,920
faces); one step = ray_trace of 33,554,432 camera rays (8 poses x 2048^2,
fov 50 deg, radius 2.5) + signed_distance(mode='watertight') of 8,388,608
points (half uniform in [-1,1]^3, half within +-0.02 of the surface).
Metric: queries/s (rays + points) over the whole job.  Inputs are larger
than L2 (805 MB of rays), so no L2 flush is inserted between steps.

``value`` times the kernels with inputs and outputs resident in HBM; ``e2e``
times the public API with host tensors (cuBVH.ray_trace / signed_distance /
unsigned_distance with ``out=`` pinned host tensors, ``non_blocking`` on one
stream per op): every input is copied to the GPU and every output back
inside the timed region, the copies of one chunk (and of one op) overlapping
the kernels of another.  ``--impl reference`` times the reference's algorithm restated on the
CPU (the oracle's FP32 mirror of its BVH4 build and traversals) on all host
cores, on a bounded sample of the same workload per step.

Multi-GPU: one process per GPU (torchrun); each rank runs its own replica of
the workload (weak scaling; the path has no cross-GPU exchange).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mesh queries/s (ray_trace + signed_distance watertight), 1 B200"
# ops over a voxel grid (no query count, no traversal)
GRID_OPS = ("floodfill", "udf_to_sdf")
# queries per step of the CPU legs (the reference's host traversals): both
# arms time the same strided sample of the workload, about 4 s of CPU work
CPU_SAMPLE = 4 << 20


def _launches() -> int:
    """Kernels launched so far by libcubvh_b200 in this process (the library
    counts its own launches; torch's kernels are not included)."""
    from cubvh_b200._lib import kernel_launches
    return kernel_launches()


# ----------------------------------------------------------------- helpers
def _rank_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of x over all ranks of the default process group (x itself
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(op: str, workload: str, n_queries: int = 0):
    """DRAM bytes (read + write) of one call of `op` over n_queries, from the
    committed ncu summary profiles/traffic_<workload>.json: its captured bytes
    per query times n_queries (the BVH stays in L2, so traffic grows with the
    queries), or its full-size figure when no query count is given."""
    path = os.path.join(ROOT, "profiles", f"traffic_{workload}.json")
    try:
        with open(path) as fh:
            e = json.load(fh)[op]
        if n_queries and "captured_queries" in e:
            return float(e["captured_dram_bytes"]) * n_queries / float(e["captured_queries"])
        return float(e["dram_bytes_per_full_launch"])
    except Exception:
        return None


def _profile_l2(op: str, workload: str):
    """L2 figures of `op` from the committed ncu summary
    profiles/l2_<workload>.json (a capture of a smaller case of the same
    workload): L2 GB/s, L2 throughput as a fraction of its peak, and the
    issue-active fraction of its kernels, time-weighted."""
    path = os.path.join(ROOT, "profiles", f"l2_{workload}.json")
    try:
        with open(path) as fh:
            e = json.load(fh)[op]
        return {"gbs": e["l2_gbs"], "frac_of_l2_peak": e["lts_pct"] / 100.0,
                "issue_active_frac": e["issue_active_pct"] / 100.0,
                "kernels": sorted(e["kernels"]), "source": os.path.relpath(path, ROOT),
                "case_queries": e["captured_queries"]}
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi sampling (every 100 ms) of SM clock and throttle reasons
    during a region.  The sampler is running before the region starts; a
    region shorter than the sampling period that catches no sample reports the
    first sample taken after it (``window`` says which)."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def _reader(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line))

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._reader, daemon=True)
        self.thread.start()
        deadline = time.perf_counter() + 10.0
        while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
            time.sleep(0.01)
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *exc):
        if self.proc is None:
            return False
        self.t1 = time.perf_counter()
        deadline = self.t1 + 1.0
        while not any(t > self.t1 for t, _ in self.lines) and time.perf_counter() < deadline:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        return False

    def summary(self):
        if self.proc is None:
            return None
        inside = [ln for t, ln in self.lines if self.t0 <= t <= self.t1]
        window = "timed region"
        if not inside:
            after = [ln for t, ln in self.lines if t > self.t1][:1]
            inside, window = after, "first sample after a region shorter than the 100 ms sampling period"
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in inside:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0])); mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "window": window}


# --------------------------------------------------------------- workloads
def build_workload(name: str, res: int = 2048, sdf_points: int = 8 << 20, grid: int = 512):
    from cubvh_b200 import workloads as W
    if name == "rays_displaced":
        w = W.rays_displaced(res=res, n_sdf=sdf_points)
        return dict(name=name, vertices=w["vertices"], faces=w["faces"],
                    ops=[("ray", (w["rays_o"], w["rays_d"])), ("sdf_watertight", (w["points"],))],
                    desc=f"displaced icosphere L6 (81,920 faces); {8 * res * res:,} rays (8 x {res}^2 pinhole, "
                         f"fov 50, r 2.5) + {sdf_points:,} watertight SDF points")
    if name == "rays_incoherent":
        v, f = W.displaced_icosphere(6, 1)
        n = 16 << 20
        ro, rd = W.incoherent_rays(n)
        return dict(name=name, vertices=v, faces=f, ops=[("ray", (ro, rd))], cpu_sample=1 << 20,
                    desc=f"displaced icosphere L6 (81,920 faces); {n:,} incoherent rays: half from U[-1,1]^3 in "
                         "random directions, half from the radius-3 sphere at random points of [-0.8,0.8]^3")
    if name == "udf_icosphere":
        w = W.udf_icosphere()
        return dict(name=name, vertices=w["vertices"], faces=w["faces"],
                    ops=[("udf_uvw", (w["points"],))],
                    desc="icosphere L4 r 0.8 (5,120 faces); 1,048,576 points U[-1,1]^3, uvw on")
    if name == "dense_tori":
        w = W.dense_tori(grid)
        g = W.dense_grid(w["grid_res"])
        return dict(name=name, vertices=w["vertices"], faces=w["faces"],
                    ops=[("udf", (g,)), ("floodfill", (grid,)), ("udf_to_sdf", (grid,))],
                    desc=f"12 tori (174,778 faces, 10% removed); UDF on the {grid}^3 grid + floodfill of udf < 2/{grid} "
                         "+ the fused udf -> sdf step (occupancy, floodfill, signs)")
    if name == "grad_displaced":
        w = W.grad_displaced()
        return dict(name=name, vertices=w["vertices"], faces=w["faces"], ops=[("udf", (w["points"],))],
                    desc="displaced icosphere L6 (81,920 faces); 4,194,304 points (half U[-1,1]^3, half "
                         "+-0.05 of the surface); fwd + bwd w.r.t. points and vertices")
    if name == "raystab_displaced":
        v, f = W.displaced_icosphere(6, 1)
        lo, hi = v.min(0), v.max(0)
        c, h = (lo + hi) / 2, (hi - lo) / 2 * 1.1
        p = (c + np.random.default_rng(5).uniform(-1, 1, (2 << 20, 3)) * h).astype(np.float32)
        # ~3,000 box and ~1,300 triangle tests per query in the reference
        # traversal: a 512k-query CPU sample keeps that leg near 10-20 s
        return dict(name=name, vertices=v, faces=f, ops=[("sdf_raystab", (p,))], cpu_sample=1 << 19,
                    desc="displaced icosphere L6 (81,920 faces); 2,097,152 raystab SDF points uniform in the "
                         "bounding box dilated by 10% (the batched workload's query distribution)")
    if name == "batch_256":
        raise SystemExit("batch_256 has no single-mesh CPU view")
    raise SystemExit(f"unknown workload {name}")


def build_time_device(cubvh, wl, dev, reps=3):
    """Seconds to build the workload's BVH on the GPU (best of reps, after
    one warm-up build; outside every timed region)."""
    import torch
    cubvh.cuBVH(wl["vertices"], wl["faces"], device_build=True)
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cubvh.cuBVH(wl["vertices"], wl["faces"], device_build=True)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def build_time_reference(wl):
    """Seconds for the reference's own host build (its BVH4 median-split
    build: src/bvh.cu compiled into oracle/_ref, else the oracle's FP32
    restatement of it)."""
    from oracle import oracle as O
    cls = O.ReferenceBVH if O.ref_bvh_available() else O.RefBVH
    t0 = time.perf_counter()
    cls(wl["vertices"], wl["faces"])
    return time.perf_counter() - t0


def n_queries(op, args):
    if op in GRID_OPS:
        return 0
    return len(args[0])


def io_bytes_per_query(op):
    return {"ray": 48, "sdf_watertight": 24, "sdf_raystab": 24, "udf": 24, "udf_uvw": 36}.get(op, 0)


def traversal_counts(wl, sample_stride=64):
    """Box / triangle tests per query of the reference traversal (FP32 mirror
    of the reference, oracle/), measured on a strided sample."""
    from oracle import oracle as O
    ref = O.RefBVH(wl["vertices"], wl["faces"])
    out = {}
    for op, args in wl["ops"]:
        if op in GRID_OPS:
            continue
        if op == "ray":
            ro, rd = args[0][::sample_stride], args[1][::sample_stride]
            *_, c = ref.ray_trace(ro, rd, count=True)
            n = len(ro)
        elif op in ("sdf_watertight", "sdf_raystab"):
            p = args[0][::sample_stride]
            *_, c = ref.signed_distance(p, mode=0 if op == "sdf_watertight" else 1, count=True)
            n = len(p)
        else:
            p = args[0][::sample_stride]
            *_, c = ref.unsigned_distance(p, return_uvw=False, count=True)
            n = len(p)
        out[op] = (c[0] / n, c[1] / n)
    return out


# -------------------------------------------------------------- CPU arms
def cpu_time_sample(wl, max_queries, threads=None):
    """Time the reference's CPU path on a strided sample of at most
    ~max_queries queries spread over every op: its own __host__ traversals
    (src/bvh.cu compiled into oracle/_ref, kind "reference") on all OpenMP
    threads, or, where that library is not built, the oracle's FP32
    restatement of them (kind "port", the same bits: tests/test_ref_bvh.py).
    Returns (queries, seconds, threads, description, kind)."""
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    kind = "reference" if O.ref_bvh_available() else "port"
    ref = O.ReferenceBVH(wl["vertices"], wl["faces"]) if kind == "reference" else O.RefBVH(wl["vertices"], wl["faces"])
    nthr = threads or O.threads()
    total = sum(len(a[0]) for op, a in wl["ops"] if op not in GRID_OPS)
    stride = max(1, -(-total // int(max_queries)))
    q, t, parts = 0, 0.0, []
    for op, args in wl["ops"]:
        if op in GRID_OPS:
            continue
        if op == "ray":
            ro, rd = np.ascontiguousarray(args[0][::stride]), np.ascontiguousarray(args[1][::stride])
            t0 = time.perf_counter()
            ref.ray_trace(ro, rd, threads=nthr) if kind == "reference" else ref.ray_trace(ro, rd)
            dt = time.perf_counter() - t0
            n = len(ro)
        else:
            p = np.ascontiguousarray(args[0][::stride])
            kw = {"threads": nthr} if kind == "reference" else {}
            t0 = time.perf_counter()
            if op in ("sdf_watertight", "sdf_raystab"):
                if kind == "reference":  # raystab seeds each query's stab rays with its index in the call
                    ref.signed_distance(args[0], mode=0 if op == "sdf_watertight" else 1, stride=stride, **kw)
                else:
                    ref.signed_distance(p, mode=0 if op == "sdf_watertight" else 1)
            else:
                ref.unsigned_distance(p, return_uvw=(op == "udf_uvw"), **kw)
            dt = time.perf_counter() - t0
            n = len(p)
        q += n; t += dt
        parts.append(f"{op}: {n} of {len(args[0])}")
    src = ("the reference's own host traversals (src/bvh.cu, oracle/_ref)" if kind == "reference"
           else "the oracle's FP32 restatement of the reference's traversals")
    return q, t, nthr, "every %d-th query (%s); %s" % (stride, "; ".join(parts), src), kind


def reference_cuda_floodfill(wl, steps, warmup):
    """The reference's own CUDA floodfill (oracle/_ref, compiled from its
    include/gpu/floodfill.cuh) on the workload's occupancy grid: wall time of
    its host entry point `_floodfill_batch` (cudaMalloc, host->device copy of
    the grid, its hook/compress passes, device->host copy of the labels,
    cudaFree) with pageable host buffers.  The grid is udf < 2/res, the udf
    taken from the oracle's FP32 mirror of the reference traversal on the host
    cores, so no kernel of this package runs in the reference arm."""
    from oracle import oracle as O
    import torch
    if not O.ref_floodfill_available():
        return {"unavailable": "oracle/_ref/libref_floodfill.so not built (needs the reference tree)"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    res = next(a[0] for op, a in wl["ops"] if op == "floodfill")
    pts = next(a[0] for op, a in wl["ops"] if op == "udf")
    t0 = time.perf_counter()
    if O.ref_bvh_available():   # the reference's own CUDA unsigned distance
        R = O.ReferenceBVH(wl["vertices"], wl["faces"])
        P = torch.from_numpy(pts).cuda()
        d = torch.empty(len(pts), device=P.device)
        fid = torch.empty(len(pts), dtype=torch.int64, device=P.device)
        R.unsigned_distance_gpu(P.data_ptr(), len(pts), d.data_ptr(), fid.data_ptr(), 0,
                                torch.cuda.current_stream().cuda_stream)
        udf = d.cpu().numpy()
        del P, d, fid
        udf_src = "the reference's CUDA unsigned distance (oracle/_ref)"
    else:
        udf = O.RefBVH(wl["vertices"], wl["faces"]).unsigned_distance(pts)[0]
        udf_src = "the oracle's FP32 restatement of the reference traversal on the host cores"
    t_udf = time.perf_counter() - t0
    grid = np.ascontiguousarray(udf.reshape(res, res, res) < np.float32(2.0 / res))
    for _ in range(max(1, warmup)):
        O.ref_floodfill(grid)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.ref_floodfill(grid)
        times.append(time.perf_counter() - t0)
    return {"e2e_ms": 1e3 * statistics.median(times), "steps": steps,
            "grid": f"{res}^3 occupancy udf < 2/{res}, blocked fraction {grid.mean():.4f}",
            "host_buffers": "pageable numpy arrays",
            "occupancy_udf": f"{udf_src}, {t_udf:.1f} s"}


def reference_cuda_queries(wl, steps, warmup, dev=None):
    """The reference's own CUDA query kernels (src/bvh.cu's launchers,
    compiled unchanged into oracle/_ref/libref_bvh.so) on the workload's
    query ops: one thread per query, 128-thread blocks, on the current
    stream.  value: device-resident inputs and outputs, CUDA events around
    each op; e2e: the reference API's own flow from pinned host tensors
    (whole-array upload, kernel, whole-array download), CUDA events.  Its
    BVH build and its lazy first-query upload are outside both."""
    import torch
    from oracle import oracle as O
    if not O.ref_bvh_available():
        return {"unavailable": "oracle/_ref/libref_bvh.so not built (needs the reference checkout)"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    dev = dev or torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    t0 = time.perf_counter()
    R = O.ReferenceBVH(wl["vertices"], wl["faces"])
    build_s = time.perf_counter() - t0
    ops = []
    for op, a in wl["ops"]:
        if op in GRID_OPS:
            continue
        if op == "ray":
            hin = [torch.from_numpy(a[0]).pin_memory(), torch.from_numpy(a[1]).pin_memory()]
            n = hin[0].shape[0]
            outs = [torch.empty(n, 3, device=dev), torch.empty(n, dtype=torch.int64, device=dev),
                    torch.empty(n, device=dev)]

            def call(di, o=outs, n=n):
                R.ray_trace_gpu(di[0].data_ptr(), di[1].data_ptr(), n, o[0].data_ptr(), o[1].data_ptr(),
                                o[2].data_ptr(), sp)
        else:
            hin = [torch.from_numpy(a[0]).pin_memory()]
            n = hin[0].shape[0]
            outs = [torch.empty(n, device=dev), torch.empty(n, dtype=torch.int64, device=dev)]
            if op == "udf_uvw":
                outs.append(torch.empty(n, 3, device=dev))
            mode = {"sdf_watertight": 0, "sdf_raystab": 1}.get(op)

            def call(di, o=outs, n=n, mode=mode):
                u = o[2].data_ptr() if len(o) > 2 else 0
                if mode is None:
                    R.unsigned_distance_gpu(di[0].data_ptr(), n, o[0].data_ptr(), o[1].data_ptr(), u, sp)
                else:
                    R.signed_distance_gpu(di[0].data_ptr(), n, mode, o[0].data_ptr(), o[1].data_ptr(), u, sp)
        din = [t.to(dev) for t in hin]
        hout = [torch.empty(o.shape, dtype=o.dtype, pin_memory=True) for o in outs]
        ops.append((op, n, call, din, hin, outs, hout))
    if not ops:
        return {}
    for _ in range(max(1, warmup)):
        for _, _, call, din, *_ in ops:
            call(din)
    torch.cuda.synchronize()
    res, q, tot, tot_e2e = {}, 0, 0.0, 0.0
    for op, n, call, din, hin, outs, hout in ops:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        for _ in range(steps):
            call(din)
        ev[1].record(stream)
        # the reference API's flow with host tensors: .cuda() of the inputs,
        # the kernel, .cpu() of the outputs
        ev[2].record(stream)
        for _ in range(steps):
            dd = [h.to(dev, non_blocking=True) for h in hin]
            call(dd)
            for o, h in zip(outs, hout):
                h.copy_(o, non_blocking=True)
        ev[3].record(stream)
        torch.cuda.synchronize()
        ms, ms_e2e = ev[0].elapsed_time(ev[1]) / steps, ev[2].elapsed_time(ev[3]) / steps
        res[op] = {"queries": n, "ms_per_launch": ms, "queries_per_s": n / (ms / 1e3), "e2e_ms": ms_e2e}
        q += n; tot += ms; tot_e2e += ms_e2e
    return {"value": q / (tot / 1e3), "unit": "queries/s", "ms_per_step": tot,
            "e2e": {"value": q / (tot_e2e / 1e3), "ms_per_step": tot_e2e,
                    "host_buffers": "pinned, whole-array copies around each call"},
            "steps": steps, "ops": res, "reference_build_s": build_s,
            "kernels": "src/bvh.cu unsigned_distance_kernel / signed_distance_*_kernel / raytrace_kernel "
                       "(1 thread per query, 128-thread blocks)"}


def workload_config(wl, world):
    """The `config` object both arms print (the same for the same workload)."""
    q = sum(len(a[0]) for op, a in wl["ops"] if op not in GRID_OPS)
    return {"workload": wl["name"], "description": wl["desc"], "queries_per_step": q,
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank, world, _ = _rank_info()
    if rank != 0:
        return
    wl = build_workload(args.workload, args.res, args.sdf_points, args.grid)
    ref_cuda = {}
    try:
        import torch
        if torch.cuda.is_available():
            ref_cuda = reference_cuda_queries(wl, max(3, min(args.steps, 5)), args.warmup)
    except Exception as e:  # the CPU arm stands on its own
        ref_cuda = {"unavailable": f"{type(e).__name__}: {e}"}
    if any(op == "floodfill" for op, _ in wl["ops"]):
        ref_cuda["floodfill"] = reference_cuda_floodfill(wl, args.steps, args.warmup)
    per_step = wl.get("cpu_sample", CPU_SAMPLE)   # the same bounded sample as the GPU arm's cpu_baseline
    for _ in range(min(args.warmup, 1)):
        cpu_time_sample(wl, per_step)
    qs, ts = 0, 0.0
    for _ in range(args.steps):
        q, t, thr, desc, kind = cpu_time_sample(wl, per_step)
        qs += q; ts += t
    val = qs / ts
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * ts / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded meshes and queries)",
        "config": workload_config(wl, world),
        "cpu_baseline": {"value": val, "unit": "queries/s", "cores": thr, "kind": kind, "sample": desc},
        "e2e": {"value": val, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if ref_cuda:
        line["reference_cuda"] = ref_cuda
    print(json.dumps(line), flush=True)


def parity_sample(wl, op_outs, per_op=4096):
    """Outside the timed region: the last step's outputs of each query op on
    a strided sample of per_op queries against the FP64 brute-force oracle
    (distances / depths within 1e-6 relative + 1e-7 absolute, face ids equal,
    signs equal)."""
    from oracle import oracle as O
    rec = {}
    v, f = wl["vertices"], wl["faces"]
    for op, a in wl["ops"]:
        if op not in op_outs:
            continue
        n = len(a[0])
        stride = max(1, n // per_op)
        if stride % 2 == 0:
            stride += 1      # odd strides cross image rows and grid lines
        idx = np.arange(0, n, stride)
        outs = [t[idx.tolist()].cpu().numpy() if t is not None else None for t in op_outs[op]]
        if op == "ray":
            t64, f64, _ = O.ray64(v, f, a[0][idx], a[1][idx])
            got_d, got_f = outs[2].astype(np.float64), outs[1]
            want_d, hit = t64, f64 >= 0
            sign_ok = True
        else:
            if op == "sdf_watertight":
                want, f64, _ = O.sdf_watertight64(v, f, a[0][idx])
            elif op == "sdf_raystab":
                want, f64, _ = O.sdf_raystab64(v, f, a[0][idx], i0=0, dirs=_stab_dirs_sample(idx))
            else:
                want, f64, _, _, _ = O.udf64(v, f, a[0][idx])
            got_d, got_f = outs[0].astype(np.float64), outs[1]
            sign_ok = bool(np.array_equal(np.signbit(outs[0]), np.signbit(want.astype(np.float32))))
            want_d, hit = np.abs(want), np.ones(len(idx), bool)
            got_d = np.abs(got_d)
        err = np.abs(got_d - want_d)[hit]
        rel = err / np.maximum(want_d[hit], 1e-300)
        within = bool((err <= 1e-7 + 1e-6 * want_d[hit]).all())
        rec[op] = {"sample": int(len(idx)), "stride": int(stride), "max_abs_err": float(err.max()) if err.size else 0.0,
                   "max_rel_err": float(rel.max()) if rel.size else 0.0, "within_tolerance": within,
                   "face_id_equal": bool(np.array_equal(got_f, f64)), "signs_equal": sign_ok}
    return rec


def _stab_dirs_sample(idx):
    """Stab directions of queries idx (the reference's device directions
    where oracle/_ref is built, else this library's, equal to them)."""
    import torch
    from oracle import oracle as O
    from cubvh_b200._lib import lib
    out = np.empty((len(idx), 32, 3), np.float32)
    buf = torch.empty(1, 32, 3, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for k, i in enumerate(idx):
        if O.ref_bvh_available():
            O.ref_stab_dirs_gpu_ptr(int(i), 1, buf.data_ptr(), s)
        else:
            lib().cubvh_stab_directions(int(i), 1, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(s))
        out[k] = buf[0].cpu().numpy()
    return out


# the other configurations, each in a process of its own after the headline
CONFIG_RUNS = [("C0", ["--workload", "udf_icosphere"]), ("C2", ["--workload", "dense_tori"]),
               ("C3", ["--workload", "grad_displaced", "--adam-steps", "50"]), ("C4", ["--workload", "batch_256"])]


def run_config_records(args):
    """Runs bench.py once per other configuration (C0, C2, C3, C4) with this
    run's --steps / --warmup and returns their JSON lines, keyed by config."""
    out = {}
    for key, extra in CONFIG_RUNS:
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--steps", str(args.steps), "--warmup",
               str(args.warmup), "--no-configs"] + extra
        t0 = time.perf_counter()
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            rec = json.loads(lines[-1]) if r.returncode == 0 and lines else {
                "failed": f"exit {r.returncode}", "stderr_tail": r.stderr[-2000:]}
        except subprocess.TimeoutExpired:
            rec = {"failed": "timeout after 900 s"}
        rec["wall_s"] = time.perf_counter() - t0
        out[key] = rec
    return out


# -------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import cubvh_b200 as cubvh
    from cubvh_b200._lib import lib, check

    wl = build_workload(args.workload, args.res, args.sdf_points, args.grid)
    t0 = time.perf_counter()
    bvh = cubvh.cuBVH(wl["vertices"], wl["faces"])
    build_host_s = time.perf_counter() - t0
    build_dev_s = build_time_device(cubvh, wl, dev)
    L = lib()
    h = bvh.impl.raw
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())

    # device-resident inputs / outputs
    dev_ops = []
    op_outs = {}
    for op, a in wl["ops"]:
        if op == "ray":
            ro = torch.from_numpy(a[0]).to(dev); rd = torch.from_numpy(a[1]).to(dev)
            n = ro.shape[0]
            outs = (torch.empty(n, 3, device=dev), torch.empty(n, dtype=torch.int64, device=dev),
                    torch.empty(n, device=dev))
            fn = (lambda ro=ro, rd=rd, n=n, o=outs: check(
                L.cubvh_ray_trace(h, P(ro), P(rd), n, P(o[0]), P(o[1]), P(o[2]), sp), "ray_trace"))
            dev_ops.append((op, n, fn, "ray: k_ray"))
            op_outs[op] = outs
        elif op in ("sdf_watertight", "sdf_raystab", "udf", "udf_uvw"):
            p = torch.from_numpy(a[0]).to(dev)
            n = p.shape[0]
            d = torch.empty(n, device=dev); fid = torch.empty(n, dtype=torch.int64, device=dev)
            uvw = torch.empty(n, 3, device=dev) if op == "udf_uvw" else None
            uptr = P(uvw) if uvw is not None else ctypes.c_void_p(0)
            if op == "sdf_watertight":
                fn = (lambda p=p, n=n, d=d, fid=fid: check(
                    L.cubvh_signed_distance(h, P(p), n, 0, P(d), P(fid), ctypes.c_void_p(0), sp), "sdf"))
                kname = "sdf_watertight: Morton bucketing + k_udf<0,1> + k_sign_watertight"
            elif op == "sdf_raystab":
                fn = (lambda p=p, n=n, d=d, fid=fid: check(
                    L.cubvh_signed_distance(h, P(p), n, 1, P(d), P(fid), ctypes.c_void_p(0), sp), "sdf"))
                kname = "sdf_raystab: Morton bucketing + k_udf<0,1> + k_sign_raystab"
            else:
                fn = (lambda p=p, n=n, d=d, fid=fid, u=uptr: check(
                    L.cubvh_unsigned_distance(h, P(p), n, P(d), P(fid), u, sp), "udf"))
                kname = "%s: Morton bucketing + k_udf<%d,0>" % (op, 1 if uvw is not None else 0)
            dev_ops.append((op, n, fn, kname))
            op_outs[op] = (d, fid, uvw)
            if args.workload == "dense_tori":
                occ_src = d
        elif op == "udf_to_sdf":
            res = a[0]
            sdf_out = torch.empty(res, res, res, device=dev)
            nb = ctypes.c_size_t()
            check(L.cubvh_floodfill_workspace_size(1, res, res, res, ctypes.byref(nb)), "ws")
            ws2 = torch.empty(nb.value, dtype=torch.uint8, device=dev)

            def fn(res=res, out=sdf_out, ws=ws2, nb=nb.value):
                check(L.cubvh_udf_to_sdf(P(occ_src), 1, res, res, res, ctypes.c_float(2.0 / res), P(out), P(ws), nb,
                                         sp), "udf_to_sdf")
            dev_ops.append((op, 0, fn, "udf_to_sdf: pack of udf < eps, floodfill passes, signed write"))
        elif op == "floodfill":
            res = a[0]
            grid = torch.empty(res, res, res, dtype=torch.bool, device=dev)
            lab = torch.empty(res, res, res, dtype=torch.int32, device=dev)
            nb = ctypes.c_size_t()
            check(L.cubvh_floodfill_workspace_size(1, res, res, res, ctypes.byref(nb)), "ws")
            ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)

            # the occupancy grid (the floodfill's input) is made from this
            # step's UDF by its own timed op, so floodfill times its kernels only
            def occ(res=res, grid=grid):
                torch.lt(occ_src.view(res, res, res), 2.0 / res, out=grid)

            def fn(res=res, grid=grid, lab=lab, ws=ws, nb=nb.value):
                check(L.cubvh_floodfill(P(grid), 1, res, res, res, P(lab), P(ws), nb, sp), "floodfill")
            dev_ops.append(("occupancy", 0, occ, "occupancy: udf < 2/res (torch.lt)"))
            dev_ops.append((op, 0, fn, "floodfill: tile, merge, resolve and label kernels"))

    q_per_step = sum(n for _, n, _, _ in dev_ops)

    def step(evs=None):
        for i, (_, _, fn, _) in enumerate(dev_ops):
            if evs is not None:
                evs[i][0].record(stream)
            fn()
            if evs is not None:
                evs[i][1].record(stream)

    # warm-up (also uploads the BVH)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    kev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in dev_ops]
           for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    n_launch0 = _launches()
    with ClockSampler(local) as clk:
        t0.record(stream)
        for s in range(args.steps):
            step(kev[s])
        t1.record(stream)
        barrier()
    gpu_launches = _launches() - n_launch0
    ms = t0.elapsed_time(t1)
    per_op_ms = [sum(kev[s][i][0].elapsed_time(kev[s][i][1]) for s in range(args.steps)) / args.steps
                 for i in range(len(dev_ops))]
    ms = max_over_ranks(ms, dev)
    value = world * q_per_step * args.steps / (ms / 1e3)

    # ---- e2e through the public API from pinned host buffers
    host_in = []
    for op, a in wl["ops"]:
        if op in GRID_OPS:
            continue
        host_in.append((op, [torch.from_numpy(x).pin_memory() for x in a]))
    e2e_steps = max(2, min(args.steps, 5))
    pinned_out = {}

    # ops are issued in increasing order of copy bytes per query: the copy
    # engines take queued copies roughly in order, so a compute-bound op's small
    # uploads go first and its kernels run while a transfer-bound op (rays, 48 B
    # per query) streams; the transfer-bound op's stream has high priority, so
    # its chunks' kernels are not held behind the others'
    def _bytes_per_query(item):
        op, tensors = item
        n = tensors[0].shape[0]
        out_b = {"ray": 24, "udf_uvw": 24}.get(op, 12)
        return sum(t.numel() * t.element_size() for t in tensors) / n + out_b
    host_in = sorted(host_in, key=_bytes_per_query)
    op_streams = [torch.cuda.Stream(dev, priority=-1 if op == "ray" else 0) for op, _ in host_in]

    def e2e_step():
        # host tensors in and out: each call streams its queries through the GPU
        # in chunks (upload, kernels and download overlapped); the ops are issued
        # non-blocking on one stream each, so one op's copies overlap another's
        # kernels, and the step ends when every result is in its pinned tensor
        h2d = d2h = 0
        for (op, tensors), ost in zip(host_in, op_streams):
            h2d += sum(t.numel() * t.element_size() for t in tensors)
            n = tensors[0].shape[0]
            if op not in pinned_out:
                if op == "ray":
                    shapes = [((n, 3), torch.float32), ((n,), torch.int64), ((n,), torch.float32)]
                else:
                    shapes = [((n,), torch.float32), ((n,), torch.int64)]
                    if op == "udf_uvw":
                        shapes.append(((n, 3), torch.float32))
                pinned_out[op] = [torch.empty(sh, dtype=dt, pin_memory=True) for sh, dt in shapes]
            outs = pinned_out[op]
            with torch.cuda.stream(ost):
                if op == "ray":
                    bvh.ray_trace(tensors[0], tensors[1], out=outs, non_blocking=True)
                elif op == "sdf_watertight":
                    bvh.signed_distance(tensors[0], mode="watertight", out=outs, non_blocking=True)
                elif op == "sdf_raystab":
                    bvh.signed_distance(tensors[0], mode="raystab", out=outs, non_blocking=True)
                else:
                    bvh.unsigned_distance(tensors[0], return_uvw=(op == "udf_uvw"), out=outs, non_blocking=True)
            d2h += sum(t.numel() * t.element_size() for t in outs)
        for ost in op_streams:
            ost.synchronize()
        return h2d, d2h

    for _ in range(3):  # warm-up: first calls grow the allocators' pools
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    # wall clock: host dispatch, both copies and the kernels, synchronised
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        h2d, d2h = e2e_step()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - w0) * 1e3
    barrier()
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_val = world * q_per_step * e2e_steps / (e2e_ms / 1e3)

    # floodfill from a pageable host grid to host labels through the public
    # API, the same footing as the reference arm's CUDA floodfill timing
    ff_host_ms = ff_cpu = None
    if any(op == "floodfill" for op, _ in wl["ops"]):
        res = next(a[0] for op, a in wl["ops"] if op == "floodfill")
        g_host = (occ_src.view(res, res, res) < 2.0 / res).cpu()
        for _ in range(2):
            cubvh.floodfill(g_host).cpu()
        torch.cuda.synchronize()
        tt = []
        for _ in range(max(3, min(args.steps, 5))):
            w0 = time.perf_counter()
            cubvh.floodfill(g_host).cpu()
            tt.append(time.perf_counter() - w0)
        ff_host_ms = 1e3 * statistics.median(tt)
        # CPU-baseline leg: the oracle's single-thread floodfill (union-find
        # giving min-index labels) on the same grid, timed beside ours, and
        # the full-grid labels compared with it (outside every timed region)
        from oracle import oracle as O
        g_np = g_host.numpy()
        w0 = time.perf_counter()
        cpu_lab = O.floodfill(g_np)
        ff_cpu = {"ms": 1e3 * (time.perf_counter() - w0), "threads": 1,
                  "labels_equal_ours": bool(np.array_equal(cpu_lab, cubvh.floodfill(g_host).cpu().numpy()))}

    line = None
    if rank == 0:
        # roofline of the dominant kernel: algorithmic bytes per launch (query
        # I/O + box and triangle bytes of the reference traversal) / its time
        counts = traversal_counts(wl)
        peak, peak_kind = _peaks()
        dom = max(range(len(dev_ops)), key=lambda i: per_op_ms[i])
        op, n, _, kname = dev_ops[dom]
        if op in GRID_OPS:  # floodfill: 1 B in + 4 B out per voxel; udf_to_sdf: 4 B in + 4 B out
            alg = (5.0 if op == "floodfill" else 8.0) * args.grid ** 3
        else:
            nb_, nt_ = counts[op]
            alg = n * (io_bytes_per_query(op) + 24.0 * nb_ + 36.0 * nt_)
        achieved = alg / (per_op_ms[dom] / 1e3) / 1e9
        # CPU-baseline leg: the reference's algorithm restated in oracle/ is
        # timed here (queries and its host BVH build) as a baseline beside
        # ours; nothing measured above runs through it
        cpu_q, cpu_t, cpu_thr, cpu_desc, cpu_kind = cpu_time_sample(wl, wl.get("cpu_sample", CPU_SAMPLE))
        ops_detail = {"bvh_build": {"faces": int(len(wl["faces"])), "host_sah_s": build_host_s,
                                    "device_lbvh_s": build_dev_s, "reference_cpu_s": build_time_reference(wl)}}
        for i, (o, nq, _, kn) in enumerate(dev_ops):
            d = {"kernel": kn, "ms_per_launch": per_op_ms[i]}
            if nq:
                d["queries"] = nq
                d["queries_per_s"] = nq / (per_op_ms[i] / 1e3)
                if o in counts:
                    d["ref_traversal_boxes_per_query"] = counts[o][0]
                    d["ref_traversal_tris_per_query"] = counts[o][1]
            if o == "floodfill" and ff_host_ms is not None:
                d["e2e_host_pageable_ms"] = ff_host_ms
                d["cpu_oracle_single_thread"] = ff_cpu
            if o in GRID_OPS:  # 1 B in + 4 B out (floodfill), 4 B in + 4 B out (udf_to_sdf) per voxel
                gbs = (5.0 if o == "floodfill" else 8.0) * args.grid ** 3 / (per_op_ms[i] / 1e3) / 1e9
                d["hbm_gbs"] = gbs
                d["hbm_frac"] = gbs / peak
            ops_detail[o] = d
        parity = parity_sample(wl, op_outs)
        ref_cuda = None
        if world == 1:
            ref_cuda = reference_cuda_queries(wl, max(3, min(args.steps, 5)), 1, dev)
            for o, r in (ref_cuda.get("ops") or {}).items():
                if o in ops_detail:
                    ops_detail[o]["reference_cuda_ms_per_launch"] = r["ms_per_launch"]
                    ops_detail[o]["speedup_vs_reference_cuda"] = r["ms_per_launch"] / ops_detail[o]["ms_per_launch"]
            if any(op == "floodfill" for op, _ in wl["ops"]):
                ref_cuda["floodfill"] = reference_cuda_floodfill(wl, 3, 1)
        l2 = _profile_l2(op, wl["name"])
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes and queries)",
            "config": workload_config(wl, world),
            "e2e": {"value": e2e_val, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": _profile_traffic(op, wl["name"], n),
                         "algorithmic_bytes_per_launch": alg,
                         "l2": l2, "l2_frac": l2["frac_of_l2_peak"] if l2 else None,
                         "note": "achieved counts the reference traversal's bytes (query I/O + 24 B per box + "
                                 "36 B per triangle test) against the HBM copy bandwidth; the BVH is L1/L2-"
                                 "resident, so l2 (ncu) shows the kernels' own L2 load and issue figures"},
            "cpu_baseline": {"value": cpu_q / cpu_t, "unit": "queries/s", "cores": cpu_thr, "kind": cpu_kind,
                             "sample": cpu_desc},
            "gpu_launches": gpu_launches,
            "clocks": clk.summary(),
            "ops": ops_detail,
            "parity": parity,
        }
        if ref_cuda is not None:
            line["reference_cuda"] = ref_cuda
        if world == 1 and args.configs and args.workload == "rays_displaced":
            line["configs"] = run_config_records(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ------------------------------------------------- forward + backward arms
def _timed(fn, steps, stream):
    import torch
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(steps):
        fn()
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps


def run_ours_fwd_bwd(args):
    """grad_displaced: distance + backward w.r.t. points and vertices (and the
    200-step Adam sphere fit); batch_256: 256 meshes in one arena launch vs
    one cuBVH call per mesh, forward + backward w.r.t. the points."""
    import torch
    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import cubvh_b200 as cubvh
    from cubvh_b200 import workloads as W
    stream = torch.cuda.current_stream(dev)
    extra = {}
    if args.workload == "grad_displaced":
        w = W.grad_displaced()
        bvh = cubvh.cuBVH(w["vertices"], w["faces"])
        pts = torch.from_numpy(w["points"]).to(dev)
        wts = torch.from_numpy(w["weights"]).to(dev)
        V = torch.from_numpy(w["vertices"]).to(dev)
        nq = pts.shape[0]

        def step():
            p = pts.detach().requires_grad_()
            v = V.detach().requires_grad_()
            d, _, _ = bvh.unsigned_distance(p, vertices=v)
            (wts * d).sum().backward()

        desc = ("displaced icosphere L6 (81,920 faces); 4,194,304 points; loss sum(w*udf); "
                "grads w.r.t. points and vertices")
        kname = "fwd_bwd: Morton bucketing + k_udf + face counting sort + k_backward"
        # Adam: fit a level-5 sphere's vertices to samples of this mesh's surface
        rng = np.random.default_rng(3)
        samples = torch.from_numpy(W.surface_points(w["vertices"], w["faces"], nq, 0.0, rng)).to(dev)
        v5, f5 = W.icosphere(5, 0.5)
        fit = cubvh.cuBVH(v5, f5)
        vv = torch.from_numpy(v5).to(dev).requires_grad_()
        opt = torch.optim.Adam([vv], lr=2e-3)

        def adam_step():
            opt.zero_grad(set_to_none=True)
            d, _, _ = fit.unsigned_distance(samples, vertices=vv)
            loss = d.mean()
            loss.backward()
            opt.step()
            return loss

        l0 = float(adam_step().item())
        ams = _timed(adam_step, max(1, args.adam_steps - 1), stream)
        l1 = float(adam_step().item())
        extra["adam_fit"] = {"steps": args.adam_steps, "ms_per_step": ams, "loss_first": l0, "loss_last": l1,
                             "fwd_bwd_queries_per_s": nq / (ams / 1e3),
                             "sphere": "icosphere L5 (20,480 faces)", "samples": nq}
    else:
        from cubvh_b200.autotune import autotune_leaf_sizes
        ms = W.batch_256(n_meshes=args.meshes)
        meshes = [(m["vertices"], m["faces"]) for m in ms]
        qs = [m["points"] for m in ms]
        modes = ["unsigned" if i % 2 == 0 else "raystab" for i in range(len(ms))]
        leaves, report = autotune_leaf_sizes(meshes, qs, modes, sample=32768, repeats=2, device=dev)
        t0 = time.perf_counter()
        arena = cubvh.BVHArena(meshes, leaf_sizes=leaves)
        arena_host_s = time.perf_counter() - t0
        cubvh.BVHArena(meshes[:2], leaf_sizes=leaves[:2], device_build=True)  # warm-up
        arena_dev, arena_dev_s = None, float("inf")
        for _ in range(3):  # best of 3 whole-arena builds (host concatenation, upload, GPU build)
            del arena_dev
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            arena_dev = cubvh.BVHArena(meshes, leaf_sizes=leaves, device_build=True)
            torch.cuda.synchronize()
            arena_dev_s = min(arena_dev_s, time.perf_counter() - t0)
        counts = [len(q) for q in qs]
        arena.set_queries(counts, modes, device=dev)
        pts = torch.from_numpy(np.concatenate(qs)).to(dev)
        nq = pts.shape[0]

        def step():
            p = pts.detach().requires_grad_()
            d, _, _ = arena.distance(p)
            d.sum().backward()

        # the same work as one cuBVH per mesh, one call (and backward) each
        bvhs = [cubvh.cuBVH(v, f) for v, f in meshes]
        off = np.concatenate([[0], np.cumsum(counts)])
        views = [pts[off[i]:off[i + 1]] for i in range(len(ms))]

        def per_call():
            for b_, q_, mode in zip(bvhs, views, modes):
                p = q_.detach().requires_grad_()
                d = b_.unsigned_distance(p)[0] if mode == "unsigned" else b_.signed_distance(p, mode=mode)[0]
                d.sum().backward()

        per_call()
        pc_ms = _timed(per_call, 3, stream)
        # the reference's own CUDA kernels, one call per mesh (forward only:
        # the reference has no backward), inputs already on the device
        ref_pc = None
        from oracle import oracle as O
        if O.ref_bvh_available() and world == 1:
            rbvhs = [O.ReferenceBVH(v, f) for v, f in meshes]
            rout = [(torch.empty(len(q_), device=dev), torch.empty(len(q_), dtype=torch.int64, device=dev))
                    for q_ in views]
            sp_ = stream.cuda_stream

            def ref_per_call():
                for rb, q_, mode, (rd_, rf_) in zip(rbvhs, views, modes, rout):
                    if mode == "unsigned":
                        rb.unsigned_distance_gpu(q_.data_ptr(), q_.shape[0], rd_.data_ptr(), rf_.data_ptr(), 0, sp_)
                    else:
                        rb.signed_distance_gpu(q_.data_ptr(), q_.shape[0], 1, rd_.data_ptr(), rf_.data_ptr(), 0, sp_)

            ref_per_call()
            ref_pc = _timed(ref_per_call, 3, stream)
            del rbvhs, rout
        desc = (f"{len(ms)} meshes (displaced icospheres L2-7 / tori, {sum(len(f) for _, f in meshes):,} faces), "
                f"{nq:,} queries (10k-2M per mesh, log-uniform), even meshes unsigned, odd raystab; fwd + bwd")
        kname = "batched fwd_bwd: arena bucketing + k_udf + k_sign_raystab + k_arena_backward_points"
        extra["per_call"] = {"ms_per_step": pc_ms, "queries_per_s": nq / (pc_ms / 1e3), "steps": 3,
                             "what": "one cuBVH per mesh, one forward call and its backward each"}
        if ref_pc is not None:
            extra["per_call_reference_cuda"] = {
                "ms_per_step": ref_pc, "queries_per_s": nq / (ref_pc / 1e3), "steps": 3,
                "what": "the reference's own CUDA kernels (src/bvh.cu), one call per mesh, forward only "
                        "(it has no backward)"}
        extra["autotune"] = {str(k): v for k, v in report.items()}
        # the same step on the arena built on the GPU (linear BVHs)
        arena_dev.set_queries(counts, modes, device=dev)

        def step_dev():
            p = pts.detach().requires_grad_()
            d, _, _ = arena_dev.distance(p)
            d.sum().backward()

        step_dev()
        extra["arena_build"] = {"faces": int(sum(len(f) for _, f in meshes)), "host_s": arena_host_s,
                                "device_one_pass_s": arena_dev_s,
                                "step_ms_on_device_built_arena": _timed(step_dev, 2, stream)}
        del arena_dev
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    n_launch0 = _launches()
    with ClockSampler(local) as clk:
        ms_step = _timed(step, args.steps, stream)
    gpu_launches = _launches() - n_launch0
    ms_step = max_over_ranks(ms_step, dev)
    value = world * nq / (ms_step / 1e3)
    if args.workload == "batch_256":
        extra["speedup_vs_per_call"] = extra["per_call"]["ms_per_step"] / ms_step
        if "per_call_reference_cuda" in extra:
            extra["speedup_vs_reference_per_call"] = extra["per_call_reference_cuda"]["ms_per_step"] / ms_step
    # e2e: host points in, gradients and distances back
    hp = pts.detach().cpu().pin_memory()
    hd = torch.empty(nq, pin_memory=True)
    hg = torch.empty(nq, 3, pin_memory=True)

    def e2e():
        p = hp.to(dev, non_blocking=True).requires_grad_()
        if args.workload == "batch_256":
            d, _, _ = arena.distance(p)
        else:
            d, _, _ = bvh.unsigned_distance(p, vertices=V.detach().requires_grad_())
        d.sum().backward()
        hd.copy_(d.detach(), non_blocking=True)
        hg.copy_(p.grad, non_blocking=True)

    for _ in range(2):
        e2e()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for _ in range(max(2, min(args.steps, 3))):
        e2e()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - w0) * 1e3 / max(2, min(args.steps, 3)), dev)
    if rank == 0:
        peak, peak_kind = _peaks()
        # algorithmic bytes per fwd+bwd query: forward query I/O (12 in, 12
        # out) + backward (12 p, 8 face, 4 grad, 4 dist read, 12 grad written)
        io = 24 + 40
        achieved = nq * io / (ms_step / 1e3) / 1e9
        line = {
            "metric": "mesh queries/s, forward + backward", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded meshes and queries)",
            "config": {"workload": args.workload, "description": desc, "queries_per_step": nq,
                       "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
            "e2e": {"value": world * nq / (e2e_ms / 1e3), "unit": "queries/s",
                    "h2d_bytes_per_step": nq * 12, "d2h_bytes_per_step": nq * 16},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": nq * io,
                         "note": "query I/O bytes only (no traversal bytes) for the fwd+bwd workloads"},
            "cpu_baseline": None, "gpu_launches": gpu_launches, "clocks": clk.summary(), "ops": extra,
        }
        if args.workload == "grad_displaced":
            wl = build_workload("grad_displaced")
            cq, ct, cthr, cdesc, ckind = cpu_time_sample(wl, 4 << 20)
            line["cpu_baseline"] = {"value": cq / ct, "unit": "queries/s", "cores": cthr, "kind": ckind,
                                    "sample": cdesc + " (forward only: the reference has no backward)"}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ------------------------------------------------ sparse marching cubes arm
def smc_band(n=192, r=80.2):
    """The voxels of a band around a sphere (radius r in voxel units, centre
    near n/2) with the sphere's signed distance at their corners: int32
    coords [N, 3], float32 corners [N, 8] in the corner order of the API."""
    off = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
    c = np.array([n / 2 + 0.3, n / 2 - 0.2, n / 2 + 0.1])
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    keep = np.abs(np.linalg.norm(g + 0.5 - c, axis=1) - r) < 2.5
    g = g[keep]
    f = (np.linalg.norm(g[:, None, :] + off[None] - c, axis=-1) - r).astype(np.float32)
    return g.astype(np.int32), f


SMC_METRIC = "voxels/s (sparse marching cubes), 1 B200"
SMC_DESC = "voxels of a band around a sphere of radius 80.2 on a 192^3 grid, its signed distance at the corners, iso 0"


def run_smc(args):
    """Sparse marching cubes on the sphere band: `value` times the public call
    on device tensors (its host round trips for the output sizes included);
    `e2e` adds the upload of the voxels and the download of the mesh."""
    import torch
    import cubvh_b200 as cubvh
    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    coords, corners = smc_band()
    n = len(coords)
    ct, ft = torch.from_numpy(coords).to(dev), torch.from_numpy(corners).to(dev)
    for _ in range(args.warmup):
        v, t = cubvh.sparse_marching_cubes(ct, ft, 0.0)
    torch.cuda.synchronize()
    n_launch0 = _launches()
    with ClockSampler(local) as clk:
        w0 = time.perf_counter()
        for _ in range(args.steps):
            v, t = cubvh.sparse_marching_cubes(ct, ft, 0.0)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - w0) * 1e3 / args.steps
    gpu_launches = _launches() - n_launch0
    ch, fh = torch.from_numpy(coords).pin_memory(), torch.from_numpy(corners).pin_memory()
    w0 = time.perf_counter()
    for _ in range(args.steps):
        v, t = cubvh.sparse_marching_cubes(ch, fh, 0.0)
        vh, th = v.cpu(), t.cpu()
    e2e_ms = (time.perf_counter() - w0) * 1e3 / args.steps
    line = {"metric": SMC_METRIC, "value": n / (ms / 1e3), "unit": "voxels/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (analytic sphere distance)",
            "config": {"workload": "sparse_mc_band", "description": SMC_DESC, "voxels": n,
                       "vertices": int(vh.shape[0]), "triangles": int(th.shape[0])},
            "e2e": {"value": n / (e2e_ms / 1e3), "unit": "voxels/s", "h2d_bytes_per_step": n * (12 + 32),
                    "d2h_bytes_per_step": int(vh.numel() * 4 + th.numel() * 4)},
            "gpu_launches": gpu_launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference_smc(args):
    """The reference's own CUDA sparse marching cubes (oracle/_ref, compiled
    from its include/gpu/spcumc.cuh) on the same voxels, host arrays in and
    out (its device allocations and copies included)."""
    rank, _, _ = _rank_info()
    if rank != 0:
        return
    from oracle import oracle as O
    coords, corners = smc_band()
    if not O.ref_sparse_mc_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_sparse_mc.so not built"}))
        return
    for _ in range(args.warmup):
        O.ref_sparse_mc(coords, corners, 0.0)
    w0 = time.perf_counter()
    for _ in range(args.steps):
        O.ref_sparse_mc(coords, corners, 0.0)
    ms = (time.perf_counter() - w0) * 1e3 / args.steps
    val = len(coords) / (ms / 1e3)
    print(json.dumps({"impl": "reference", "metric": SMC_METRIC, "value": val, "unit": "voxels/s", "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic (analytic sphere distance)",
                      "config": {"workload": "sparse_mc_band", "description": SMC_DESC, "voxels": len(coords)},
                      "reference_cuda": {"sparse_mc": {"e2e_ms": ms, "host_buffers": "numpy arrays"}},
                      "cpu_baseline": None,
                      "e2e": {"value": val, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rays_displaced",
                    choices=["rays_displaced", "rays_incoherent", "udf_icosphere", "dense_tori", "raystab_displaced",
                             "grad_displaced", "batch_256", "sparse_mc_band"])
    ap.add_argument("--adam-steps", type=int, default=200, help="grad_displaced: sphere-fitting steps")
    ap.add_argument("--meshes", type=int, default=256, help="batch_256: number of meshes")
    ap.add_argument("--res", type=int, default=2048, help="camera resolution (rays_displaced)")
    ap.add_argument("--sdf-points", type=int, default=8 << 20, help="SDF queries (rays_displaced)")
    ap.add_argument("--grid", type=int, default=512, help="grid resolution (dense_tori)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="headline workload only (by default a 1-GPU run of the default workload also runs "
                         "C0, C2, C3 and C4 and adds their lines under 'configs')")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "sparse_mc_band":
        run_reference_smc(args) if args.impl == "reference" else run_smc(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload in ("grad_displaced", "batch_256"):
        run_ours_fwd_bwd(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
