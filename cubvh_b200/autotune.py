"""Leaf-size autotuner for ``BVHArena``.

Meshes are bucketed by face count; for each bucket the tuner builds its
median mesh with every candidate leaf size, times the bucket's dominant query
mode on a sample of that mesh's queries with CUDA events, and keeps the
fastest.  The block size (128 threads) and the packet width (32 queries per
warp, one packet in flight per warp) are fixed by the kernels.
"""

from __future__ import annotations

import numpy as np
import torch

from .arena import BVHArena

BUCKETS = (0, 2_000, 20_000, 200_000)
LEAF_SIZES = (2, 3, 4)


def bucket_of(n_faces: int) -> int:
    b = 0
    for i, lo in enumerate(BUCKETS):
        if n_faces >= lo:
            b = i
    return b


def autotune_leaf_sizes(meshes, queries, modes, sample=65536, repeats=3, device="cuda"):
    """meshes: list of (V, F); queries: list of [n_m, 3] arrays; modes: list of
    mode names.  Returns (per-mesh leaf sizes, {bucket: (leaf, ms per query set)})."""
    by_bucket = {}
    for m, (v, f) in enumerate(meshes):
        by_bucket.setdefault(bucket_of(len(f)), []).append(m)
    choice, report = {}, {}
    dev = torch.device(device)
    for b, members in by_bucket.items():
        members = sorted(members, key=lambda m: len(meshes[m][1]))
        m = members[len(members) // 2]
        mode = max(set(modes[i] for i in members), key=lambda x: sum(modes[i] == x for i in members))
        q = np.asarray(queries[m], np.float32)
        if len(q) > sample:
            q = q[np.random.default_rng(0).choice(len(q), sample, replace=False)]
        pts = torch.from_numpy(np.ascontiguousarray(q)).to(dev)
        times = {}
        for leaf in LEAF_SIZES:
            ar = BVHArena([meshes[m]], leaf_sizes=[leaf])
            ar.set_queries([len(q)], [mode], device=dev)
            ar.distance(pts)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(repeats):
                ar.distance(pts)
            e1.record()
            torch.cuda.synchronize(dev)
            times[leaf] = e0.elapsed_time(e1) / repeats
        best = min(times, key=times.get)
        choice[b] = best
        report[b] = {"mesh": m, "faces": len(meshes[m][1]), "mode": mode, "ms": times, "leaf": best}
    return [choice[bucket_of(len(f))] for _, f in meshes], report
