"""GPU floodfill parity: labels must equal the oracle's bit for bit."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,p", [
    ((32, 32, 32), 0.45), ((1, 17, 9, 40), 0.3), ((3, 33, 31, 29), 0.35), ((2, 64, 64, 64), 0.55),
    ((1, 5, 7, 3), 0.2), ((1, 1, 1, 1), 0.0), ((1, 2, 3, 100), 0.4), ((1, 40, 1, 1), 0.1),
    # tiles with more runs than the shared-memory union-find holds (global parents)
    ((1, 64, 512, 4), 0.5),
    # rows of more than 2048 bitmask words (tiles of one row in several chunks), with and
    # without whole words per row
    ((1, 3, 70016, 2), 0.3), ((1, 2, 70000, 1), 0.3),
])
def test_floodfill_random(oracle, dev, shape, p):
    rng = np.random.default_rng(abs(hash(shape)) % 1000)
    g = rng.random(shape) < p
    got = cubvh.floodfill(torch.from_numpy(g).to(dev), check_bounds=True).cpu().numpy()
    assert got.shape == g.shape and got.dtype == np.int32
    assert np.array_equal(got, oracle.floodfill(g))


def test_floodfill_all_free_all_blocked(oracle, dev):
    g = torch.zeros(2, 16, 16, 16, dtype=torch.bool, device=dev)
    lab = cubvh.floodfill(g)
    assert (lab[0] == 0).all() and (lab[1] == 16 ** 3).all()
    lab = cubvh.floodfill(torch.ones(16, 16, 16, dtype=torch.bool, device=dev))
    assert (lab == -1).all()


def test_floodfill_spiral_maze(oracle, dev):
    # long, thin free path: many merges along one component
    n = 96
    g = np.ones((n, n, n), bool)
    g[:, 1::2, :] = False                      # free slabs
    g[:, 2::4, 0] = False                      # connectors alternate ends
    g[:, 4::4, -1] = False
    got = cubvh.floodfill(torch.from_numpy(g).to(dev)).cpu().numpy()
    assert np.array_equal(got, oracle.floodfill(g))


def test_floodfill_occupancy_pipeline(oracle, dev):
    # udf -> occupancy -> floodfill, as in the reference's readme recipe
    v, f = W.random_tori(2, n_tori=4, n_major=64, n_minor=16)
    bvh = cubvh.cuBVH(v, f)
    res = 96
    pts = torch.from_numpy(W.dense_grid(res)).to(dev)
    udf, _, _ = bvh.unsigned_distance(pts)
    occ = (udf < 2 / res).view(res, res, res)
    got = cubvh.floodfill(occ, check_bounds=True).cpu().numpy()
    assert np.array_equal(got, oracle.floodfill(occ.cpu().numpy()))
    assert got[0, 0, 0] == 0


def test_floodfill_rejects_non_bool(dev):
    with pytest.raises(RuntimeError):
        cubvh.floodfill(torch.zeros(4, 4, 4, dtype=torch.int32, device=dev))


@pytest.mark.parametrize("shape", [(32, 32, 32), (2, 24, 17, 40), (1, 9, 64, 7), (3, 16, 16, 16), (1, 64, 512, 4),
                                   (1, 3, 70016, 2)])
def test_udf_to_sdf_random(oracle, dev, shape):
    """Fused occupancy -> floodfill -> signed grid against the reference recipe
    (oracle floodfill + the same float32 arithmetic), bit for bit; includes
    volumes whose first voxel is occupied and NaN distances."""
    rng = np.random.default_rng(sum(shape))
    u = rng.random(shape).astype(np.float32)
    u[rng.random(shape) < 0.35] = 0.0           # occupied walls
    if len(shape) == 4:
        u[-1, 0, 0, 0] = 0.0                    # last volume: first voxel occupied
    u.reshape(-1)[rng.choice(u.size, 5, replace=False)] = np.nan
    eps = 0.05
    got = cubvh.udf_to_sdf(torch.from_numpy(u).to(dev), eps=eps, check_bounds=True).cpu().numpy()
    want = oracle.udf_to_sdf(u, eps)
    assert got.dtype == np.float32 and got.shape == u.shape
    assert np.array_equal(got, want, equal_nan=True)


def test_udf_to_sdf_sphere_grid(oracle, dev):
    """The reference pipeline on a mesh: dense UDF of a sphere on a 64^3
    grid, then the signed grid; the same as torch ops around floodfill, and
    negative inside the sphere."""
    v, f = W.icosphere(3, 0.6)
    res = 64
    g = torch.linspace(-1, 1, res, device=dev)
    pts = torch.stack(torch.meshgrid(g, g, g, indexing="ij"), -1).view(-1, 3)
    udf = cubvh.cuBVH(v, f).unsigned_distance(pts)[0].view(res, res, res)
    eps = 2.0 / res
    sdf = cubvh.udf_to_sdf(udf)
    lab = cubvh.floodfill(udf < eps)
    ref = udf - eps
    inner = (lab != lab[0, 0, 0]) & (ref > 0)
    ref[inner] *= -1
    assert torch.equal(sdf, ref)
    r = pts.norm(dim=1).view(res, res, res)
    assert (sdf[r < 0.4] < 0).all() and (sdf[r > 0.8] > 0).all()


@pytest.mark.parametrize("shape", [(1, 40, 64, 24), (2, 12, 96, 20)])
def test_c_abi_unaligned_buffers(oracle, dev, shape):
    """W % 32 == 0 grids (W = shape[2], the reference's row length) through the C ABI with the grid, labels, udf and sdf
    pointers moved off 16-byte alignment (the byte-wise pack and the
    word-per-store label/sdf writers) and aligned (the 16-byte paths): the
    same labels and signed grids either way."""
    import ctypes
    from cubvh_b200._lib import lib, check
    L = lib()
    B, H, Wd, D = shape
    n = B * H * Wd * D
    rng = np.random.default_rng(n)
    g = rng.random(shape) < 0.45
    u = rng.random(shape).astype(np.float32)
    u[rng.random(shape) < 0.35] = 0.0
    want_lab, want_sdf = oracle.floodfill(g), oracle.udf_to_sdf(u, 0.05)
    nb = ctypes.c_size_t()
    check(L.cubvh_floodfill_workspace_size(B, H, Wd, D, ctypes.byref(nb)), "ws")
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    sp = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for off in (0, 1):
        gbuf = torch.zeros(n + 16, dtype=torch.uint8, device=dev)
        gbuf[off:off + n] = torch.from_numpy(g.reshape(-1).astype(np.uint8)).to(dev)
        lbuf = torch.full((n + 4,), -7, dtype=torch.int32, device=dev)
        check(L.cubvh_floodfill(ctypes.c_void_p(gbuf.data_ptr() + off), B, H, Wd, D,
                                ctypes.c_void_p(lbuf.data_ptr() + 4 * off), ctypes.c_void_p(ws.data_ptr()),
                                nb.value, sp), "floodfill")
        got = lbuf[off:off + n].cpu().numpy().reshape(shape)
        assert np.array_equal(got, want_lab)
        assert (lbuf[:off] == -7).all() and (lbuf[off + n:] == -7).all()
        ubuf = torch.zeros(n + 4, dtype=torch.float32, device=dev)
        ubuf[off:off + n] = torch.from_numpy(u.reshape(-1)).to(dev)
        sbuf = torch.full((n + 4,), 7.0, dtype=torch.float32, device=dev)
        check(L.cubvh_udf_to_sdf(ctypes.c_void_p(ubuf.data_ptr() + 4 * off), B, H, Wd, D, ctypes.c_float(0.05),
                                 ctypes.c_void_p(sbuf.data_ptr() + 4 * off), ctypes.c_void_p(ws.data_ptr()),
                                 nb.value, sp), "udf_to_sdf")
        assert np.array_equal(sbuf[off:off + n].cpu().numpy().reshape(shape), want_sdf)
        assert (sbuf[:off] == 7.0).all() and (sbuf[off + n:] == 7.0).all()


@pytest.mark.parametrize("shape,p", [((1, 96, 96, 96), 0.3), ((2, 64, 64, 64), 0.6), ((1, 8, 32, 8), 0.5)])
def test_floodfill_aligned_rows(oracle, dev, shape, p):
    """Rows of whole 32-voxel words (the 16-byte label store path)."""
    g = np.random.default_rng(int(p * 10) + shape[-1]).random(shape) < p
    got = cubvh.floodfill(torch.from_numpy(g).to(dev), check_bounds=True).cpu().numpy()
    assert np.array_equal(got, oracle.floodfill(g))
