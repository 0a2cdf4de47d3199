"""cubvh_floodfill_noalloc: the floodfill entry point for callers that may not
allocate GPU memory while they run (for example code living inside another
framework's memory pool, where a cudaMalloc or cudaFree would stall the
device or bypass the pool).  Its scratch is a fixed 32 MiB array inside the
library, so the call needs no workspace and allocates nothing.

Checked through the C ABI against the regular cubvh_floodfill (which takes a
caller workspace) on two calls in a row, so that anything the first call left
in the shared scratch would show up in the second; labels must match bit for
bit, and the bound status of each call (read with cubvh_floodfill_check and
a NULL workspace) must be clear.  This file runs last so that a failure here
does not hide the rest.
"""

import ctypes

import numpy as np
import pytest
import torch

from cubvh_b200 import _lib

pytestmark = pytest.mark.gpu


def _noalloc():
    L = _lib.lib()
    fn = L.cubvh_floodfill_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return L, fn


def _regular(L, grid, stream):
    B, H, W, D = grid.shape
    nb = ctypes.c_size_t()
    assert L.cubvh_floodfill_workspace_size(B, H, W, D, ctypes.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device=grid.device)
    out = torch.empty(grid.shape, dtype=torch.int32, device=grid.device)
    rc = L.cubvh_floodfill(grid.data_ptr(), B, H, W, D, out.data_ptr(), ws.data_ptr(), nb.value, stream)
    assert rc == 0, L.cubvh_last_error()
    return out


def test_floodfill_noalloc_matches_regular_twice():
    dev = torch.device("cuda:0")
    L, fn = _noalloc()
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(123)
    grids = [rng.random((1, 96, 96, 96)) < 0.45,          # first call
             rng.random((2, 40, 72, 56)) < 0.3]           # second call, other shape
    for g in grids:
        grid = torch.from_numpy(g).to(dev)
        B, H, W, D = grid.shape
        got = torch.full(grid.shape, -7, dtype=torch.int32, device=dev)
        rc = fn(grid.data_ptr(), B, H, W, D, got.data_ptr(), stream)
        assert rc == 0, L.cubvh_last_error()
        # the bound status of this call, read from the built-in array
        assert L.cubvh_floodfill_check(None, B, H, W, D, stream) == 0, L.cubvh_last_error()
        want = _regular(L, grid, stream)
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_floodfill_noalloc_rejects_large_grid():
    dev = torch.device("cuda:0")
    L, fn = _noalloc()
    grid = torch.zeros(1, 256, 256, 256, dtype=torch.bool, device=dev)
    out = torch.empty(grid.shape, dtype=torch.int32, device=dev)
    rc = fn(grid.data_ptr(), 1, 256, 256, 256, out.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    assert rc == 1
    assert b"scratch" in L.cubvh_last_error()
