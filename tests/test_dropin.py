"""The `cubvh` drop-in package: the reference's Python surface
(cubvh/api.py) over the `_cubvh` torch extension, itself a thin layer over
the C ABI.  CPU tests cover construction, state_dict and the error surface;
the GPU tests (marked) check that every query through the extension gives
the bits of the same query through cubvh_b200."""

import numpy as np
import pytest
import torch

import cubvh
import cubvh_b200
from cubvh_b200 import workloads as W


def test_surface_names():
    for name in ("cuBVH", "floodfill", "sparse_marching_cubes"):
        assert callable(getattr(cubvh, name))
    with pytest.raises(AttributeError, match="scope"):
        cubvh.fill_holes
    with pytest.raises(AttributeError):
        cubvh.no_such_thing


def test_state_dict_round_trip_and_versions():
    v, f = W.displaced_icosphere(3, 1)
    b = cubvh.cuBVH(torch.from_numpy(v), torch.from_numpy(f).int())    # torch inputs, int32 faces
    sd = b.state_dict()
    assert sd["nodes"].dtype == torch.int32 and sd["nodes"].shape[1] == 9
    assert sd["triangles"].shape == (len(f), 12) and sd["version"].tolist() == [1]
    # same records as cubvh_b200 (both are the reference build's records)
    sd2 = cubvh_b200.cuBVH(v, f).state_dict()
    assert torch.equal(sd["nodes"], sd2["nodes"]) and torch.equal(sd["triangles"], sd2["triangles"])
    back = cubvh.cuBVH.from_state_dict(sd).state_dict()
    assert all(torch.equal(back[k], sd[k]) for k in sd)
    # unversioned (reference) dicts load; unknown versions do not
    cubvh.cuBVH.from_state_dict({"nodes": sd["nodes"], "triangles": sd["triangles"]})
    cubvh.cuBVH.from_state_dict(dict(sd, version=1))
    for bad in (torch.tensor([3], dtype=torch.int32), 2, "1"):
        with pytest.raises(RuntimeError, match="version"):
            cubvh.cuBVH.from_state_dict(dict(sd, version=bad))


def test_errors_like_reference():
    v, f = W.icosphere(0)
    with pytest.raises(AssertionError):
        cubvh.cuBVH(v, f[:8])
    bad = f.copy()
    bad[0, 0] = 99
    with pytest.raises(RuntimeError, match="vertex index"):
        cubvh.cuBVH(v, bad)
    with pytest.raises(RuntimeError, match="triangles"):
        cubvh.cuBVH.from_state_dict({"nodes": torch.zeros(1, 9, dtype=torch.int32)})
    with pytest.raises(RuntimeError, match="nodes"):
        cubvh.cuBVH.from_state_dict({"triangles": torch.zeros(9, 12, dtype=torch.int32)})
    b = cubvh.cuBVH(v, f)
    with pytest.raises(KeyError):
        b.signed_distance(torch.zeros(4, 3), mode="pathescape")


@pytest.mark.gpu
def test_queries_equal_cubvh_b200(dev):
    v, f = W.displaced_icosphere(4, 1)
    a, b = cubvh.cuBVH(v, f), cubvh_b200.cuBVH(v, f)
    rng = np.random.default_rng(5)
    p = torch.from_numpy(rng.uniform(-1, 1, (7, 300, 3)).astype(np.float32)).to(dev)   # prefix shape kept
    for ra, rb in [(a.unsigned_distance(p, return_uvw=True), b.unsigned_distance(p, return_uvw=True)),
                   (a.signed_distance(p), b.signed_distance(p)),
                   (a.signed_distance(p, return_uvw=True, mode="raystab"),
                    b.signed_distance(p, return_uvw=True, mode="raystab"))]:
        for x, y in zip(ra, rb):
            if x is None:
                assert y is None
            else:
                assert x.shape[:2] == (7, 300) and torch.equal(x, y)
    ro = torch.zeros(2, 500, 3, device=dev)
    ro[..., 2] = 2.5
    rd = torch.from_numpy(rng.normal(size=(2, 500, 3)).astype(np.float32)).to(dev)
    rd[..., 2] = -4
    rd = rd / rd.norm(dim=-1, keepdim=True)
    for x, y in zip(a.ray_trace(ro, rd.double()), b.ray_trace(ro, rd)):     # dtype coerced like the reference
        assert x.shape[:2] == (2, 500) and torch.equal(x, y)
    # CPU queries are moved to the GPU, as in the reference
    d, _, _ = a.unsigned_distance(p.cpu())
    assert d.is_cuda and torch.equal(d, b.unsigned_distance(p)[0])


@pytest.mark.gpu
def test_floodfill_and_marching_cubes_equal_cubvh_b200(dev):
    rng = np.random.default_rng(6)
    g = torch.from_numpy(rng.random((2, 20, 24, 28)) < 0.4).to(dev)
    assert torch.equal(cubvh.floodfill(g), cubvh_b200.floodfill(g))
    assert torch.equal(cubvh.floodfill(g[0]), cubvh_b200.floodfill(g[0]))
    coords = torch.from_numpy(np.stack(np.meshgrid(*[np.arange(6)] * 3, indexing="ij"), -1).reshape(-1, 3)).int()
    corners = torch.from_numpy(rng.standard_normal((len(coords), 8)).astype(np.float32))
    va, ta = cubvh.sparse_marching_cubes(coords.to(dev), corners.to(dev), 0.0)
    vb, tb = cubvh_b200.sparse_marching_cubes(coords.to(dev), corners.to(dev), 0.0)
    assert torch.equal(va, vb) and torch.equal(ta, tb)
