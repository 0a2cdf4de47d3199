"""Many meshes, one launch: ``BVHArena``.

No counterpart in the reference (one mesh per ``cuBVH``, one kernel launch
per call).  The meshes are built into one node / triangle arena; a query
layout (how many queries each mesh has, in consecutive rows of one points
tensor, and each mesh's mode) is fixed once with ``set_queries``; after that
``distance`` serves every query of every mesh with one bucketing pass, one
packet-traversal launch and one launch per sign mode present, and is
differentiable w.r.t. the points.  ``capture`` records those launches in a
CUDA graph for repeated use with fixed input / output buffers.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import check, lib

__all__ = ["BVHArena"]

_MODES = {"unsigned": 0, "watertight": 1, "raystab": 2}


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class _ArenaFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, arena, return_uvw):
        d, fid, uvw = arena._run(points, return_uvw)
        ctx.arena = arena
        ctx.save_for_backward(points, fid, d)
        ctx.mark_non_differentiable(fid)
        if uvw is not None:
            ctx.mark_non_differentiable(uvw)
        return d, fid, uvw

    @staticmethod
    def backward(ctx, gd, _gf, _gu):
        points, fid, d = ctx.saved_tensors
        gp = torch.empty_like(points)
        with torch.cuda.device(points.device):
            check(lib().cubvh_arena_backward(ctx.arena._h, _p(points), _p(fid), _p(gd.contiguous().float()),
                                             _p(d), _p(gp), _stream(points.device)), "arena_backward")
        return gp, None, None


class BVHArena:
    """meshes: list of (vertices [V, 3], faces [F, 3]) (numpy or torch);
    leaf_sizes: optional per-mesh leaf size in [1, 4] (see autotune)."""

    def __init__(self, meshes, leaf_sizes=None, device_build=False):
        # device_build: build all meshes on the current GPU in one pass
        # (linear BVHs; the same query results as the default host build)
        self._keep = []
        vs, fs, nv, nf = [], [], [], []
        for v, f in meshes:
            if torch.is_tensor(v): v = v.detach().cpu().numpy()
            if torch.is_tensor(f): f = f.detach().cpu().numpy()
            v = np.ascontiguousarray(v, dtype=np.float32)
            f = np.ascontiguousarray(f, dtype=np.int64)
            self._keep += [v, f]
            vs.append(v.ctypes.data); fs.append(f.ctypes.data); nv.append(len(v)); nf.append(len(f))
        M = len(vs)
        VP = (ctypes.c_void_p * M)(*vs)
        FP = (ctypes.c_void_p * M)(*fs)
        NV = (ctypes.c_int64 * M)(*nv)
        NF = (ctypes.c_int64 * M)(*nf)
        LS = (ctypes.c_int32 * M)(*leaf_sizes) if leaf_sizes is not None else None
        h = ctypes.c_void_p()
        args = (M, ctypes.cast(VP, ctypes.c_void_p), ctypes.cast(NV, ctypes.c_void_p),
                ctypes.cast(FP, ctypes.c_void_p), ctypes.cast(NF, ctypes.c_void_p),
                ctypes.cast(LS, ctypes.c_void_p) if LS is not None else None)
        if device_build:
            dev = torch.device("cuda", torch.cuda.current_device())
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            check(lib().cubvh_arena_create_device(*args, stream, ctypes.byref(h)), "arena")
        else:
            check(lib().cubvh_arena_create(*args, ctypes.byref(h)), "arena")
        self._h = h
        self._keep = None
        self.n_meshes = M
        self.n_queries = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().cubvh_arena_destroy(h)
            except Exception:
                pass
            self._h = None

    def info(self):
        m, f, n = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().cubvh_arena_info(self._h, ctypes.byref(m), ctypes.byref(f), ctypes.byref(n)), "arena_info")
        return {"meshes": m.value, "faces": f.value, "nodes": n.value}

    def set_queries(self, counts, modes, device=None):
        """counts[m] queries for mesh m (consecutive rows); modes[m] in
        'unsigned' | 'watertight' | 'raystab'.  Uploads the layout to the
        current (or given) CUDA device."""
        counts = [int(c) for c in counts]
        if len(counts) != self.n_meshes or len(modes) != self.n_meshes:
            raise RuntimeError("set_queries needs one count and one mode per mesh")
        off = np.zeros(self.n_meshes + 1, np.int64)
        off[1:] = np.cumsum(counts)
        md = np.array([_MODES[m] for m in modes], np.uint32)
        with torch.cuda.device(device if device is not None else torch.cuda.current_device()):
            check(lib().cubvh_arena_set_queries(self._h, off.ctypes.data, md.ctypes.data), "set_queries")
        self.n_queries = int(off[-1])
        self.offsets = off

    def _run(self, points, return_uvw, out=None):
        n = points.shape[0]
        if out is None:
            d = torch.empty(n, dtype=torch.float32, device=points.device)
            fid = torch.empty(n, dtype=torch.int64, device=points.device)
            uvw = torch.empty(n, 3, dtype=torch.float32, device=points.device) if return_uvw else None
        else:
            d, fid, uvw = out
        with torch.cuda.device(points.device):
            check(lib().cubvh_arena_distance(self._h, _p(points), _p(d), _p(fid), _p(uvw), _stream(points.device)),
                  "arena_distance")
        return d, fid, uvw

    def distance(self, points, return_uvw=False):
        """points: CUDA float [n_queries, 3] laid out as in set_queries.
        Returns (distance, face_id within the mesh, uvw or None); signed
        where the mesh's mode is signed; differentiable w.r.t. points."""
        if self.n_queries is None:
            raise RuntimeError("call set_queries first")
        points = points.float()
        if not points.is_cuda: points = points.cuda()
        points = points.contiguous()
        if points.shape != (self.n_queries, 3):
            raise RuntimeError(f"points must be [{self.n_queries}, 3] for this layout")
        if torch.is_grad_enabled() and points.requires_grad:
            return _ArenaFn.apply(points, self, return_uvw)
        return self._run(points.detach(), return_uvw)

    def capture(self, points, return_uvw=False):
        """Record one distance call on the fixed tensor `points` in a CUDA
        graph.  Returns (replay, (distance, face_id, uvw)): replay() reruns the
        queries on the current contents of `points` into the same outputs."""
        n = points.shape[0]
        out = (torch.empty(n, device=points.device), torch.empty(n, dtype=torch.int64, device=points.device),
               torch.empty(n, 3, device=points.device) if return_uvw else None)
        s = torch.cuda.Stream(points.device)
        s.wait_stream(torch.cuda.current_stream(points.device))
        with torch.cuda.stream(s):
            self._run(points, return_uvw, out)      # warm-up outside the graph
        torch.cuda.current_stream(points.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._run(points, return_uvw, out)
        return g.replay, out
