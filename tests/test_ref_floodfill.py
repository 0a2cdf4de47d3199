"""Floodfill parity against the REFERENCE'S OWN outputs.

tests/golden/ref_floodfill.npz holds the labels that the reference's CUDA
floodfill (include/gpu/floodfill.cuh, built from the reference tree into
oracle/_ref by `make -C oracle ref`) returned for 13 grids; make_ref_floodfill.py
beside it regenerates them on a GPU.  The CPU test pins the floodfill oracle to
those labels; the GPU tests check the CUDA floodfill against them and, where
oracle/_ref was built, against the reference running live on larger grids."""

import os

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

R = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_floodfill.npz"))
CASES = sorted({k.rsplit("_", 1)[0] for k in R.files})


def _grid(name):
    shape = tuple(int(s) for s in R[name + "_shape"])
    return np.unpackbits(R[name + "_grid"])[:int(np.prod(shape))].astype(bool).reshape(shape)


def test_fixture_cases_cover_the_edges():
    assert len(CASES) == 13
    shapes = {n: tuple(R[n + "_shape"]) for n in CASES}
    assert shapes["batch3"][0] == 3 and shapes["tiny"][1:] == (3, 3, 3)
    assert (R["blocked_ref"] == -1).all() and (R["free_ref"] == 0).all()
    # W != D: the reference's x = l % W decode differs from the memory layout
    assert shapes["rand25"][2] != shapes["rand25"][3]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_labels(oracle, name):
    assert np.array_equal(oracle.floodfill(_grid(name)), R[name + "_ref"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_matches_reference_labels(dev, name):
    got = cubvh.floodfill(torch.from_numpy(_grid(name)).to(dev), check_bounds=True).cpu().numpy()
    assert np.array_equal(got, R[name + "_ref"])


def _snake(n):
    g = np.ones((1, n, n, n), bool)
    for w in range(n):
        if w % 2 == 0:
            g[0, 0, w, :] = False
        else:
            g[0, 0, w, n - 1 if (w // 2) % 2 == 0 else 0] = False
    return g


def _live_cases():
    out = [("rand96_%g" % p, (1, 96, 96, 96), p) for p in (0.2, 0.3, 0.45, 0.6, 0.7)]
    out += [("rand_80x96x112", (1, 80, 96, 112), 0.6), ("batch2_64", (2, 64, 64, 64), 0.45),
            ("tori128", None, None), ("snake48", None, None)]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name,shape,p", _live_cases(), ids=[c[0] for c in _live_cases()])
def test_cuda_matches_live_reference(oracle, dev, name, shape, p):
    if not oracle.ref_floodfill_available():
        pytest.skip("oracle/_ref/libref_floodfill.so not built (needs the reference tree)")
    if name == "tori128":
        v, f = W.random_tori(2)
        udf, _, _ = cubvh.cuBVH(v, f).unsigned_distance(torch.from_numpy(W.dense_grid(128)).to(dev))
        g = (udf.view(1, 128, 128, 128) < 2.0 / 128).cpu().numpy()
    elif name == "snake48":
        g = _snake(48)
    else:
        g = np.random.default_rng(int(p * 100)).random(shape) < p
    ours = cubvh.floodfill(torch.from_numpy(g).to(dev)).cpu().numpy()
    assert np.array_equal(ours, oracle.ref_floodfill(g))
