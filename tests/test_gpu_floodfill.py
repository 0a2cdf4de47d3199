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
