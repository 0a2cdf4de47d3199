"""Sparse marching cubes against the reference's own outputs.

tests/golden/ref_sparse_mc.npz holds the vertex and triangle arrays that the
reference's CUDA sparse marching cubes (include/gpu/spcumc.cuh, built from the
reference tree into oracle/_ref) returned for three voxel sets
(make_ref_sparse_mc.py beside it); tests/golden/ref_mc_cases.npz its triangle
list for each of the 256 corner configurations of one voxel (its case table,
make_ref_mc_cases.py).  By default the vertex and triangle arrays must equal
the reference's index for index (the oracle's restatement on the CPU, the
CUDA kernels on the GPU).  The optional closed triangulation
(triangulation="closed") is this library's own: the tests check what holds
for any correct triangulation there: closed and consistently oriented where
the corner values agree, no edge in more than two triangles, the same
enclosed volume."""

import os
import sys

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_sparse_mc as M  # noqa: E402

R = np.load(os.path.join(HERE, "golden", "ref_sparse_mc.npz"))
TABLE = np.load(os.path.join(HERE, "golden", "ref_mc_cases.npz"))["tri_edges"]
CASES = M.cases()
EDGE_CORNERS = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6], [6, 7], [7, 4], [0, 4], [1, 5], [2, 6],
                         [3, 7]])


def _edges(t):
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    _, cnt = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    _, dcnt = np.unique(e, axis=0, return_counts=True)
    return e, cnt, dcnt


def _volume(v, t):
    a, b, c = (v[t[:, k]].astype(np.float64) for k in range(3))
    return np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6


def _rot(t):
    k = np.argmin(t, 1)
    r = np.arange(len(t))
    return np.stack([t[r, k], t[r, (k + 1) % 3], t[r, (k + 2) % 3]], 1)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_vertices_match_reference(oracle, name):
    coords, corners, iso = CASES[name]
    assert np.array_equal(oracle.sparse_mc_vertices(coords, corners, iso), R[name + "_verts"])


def test_case_table_cuts_only_cut_edges():
    """Every triangle of the reference's case table joins three different
    edges that the configuration cuts (one corner inside); empty and full
    cubes have no triangle."""
    for c in range(256):
        inside = [(c >> k) & 1 for k in range(8)]
        cut = {e for e, (a, b) in enumerate(EDGE_CORNERS) if inside[a] != inside[b]}
        row = TABLE[c][TABLE[c] >= 0]
        assert len(row) % 3 == 0 and set(row.tolist()) <= cut
        assert all(len(set(row[i:i + 3].tolist())) == 3 for i in range(0, len(row), 3))
        if not cut:
            assert len(row) == 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_triangles_match_reference(oracle, name):
    coords, corners, iso = CASES[name]
    assert np.array_equal(oracle.sparse_mc_triangles(coords, corners, iso, TABLE), R[name + "_tris"])


def _run(name, dev, ensure=False, triangulation="reference"):
    coords, corners, iso = CASES[name]
    v, t = cubvh.sparse_marching_cubes(torch.from_numpy(coords).to(dev), torch.from_numpy(corners).to(dev), iso,
                                       ensure_consistency=ensure, triangulation=triangulation)
    assert v.dtype == torch.float32 and t.dtype == torch.int32 and v.is_cuda and t.is_cuda
    return v.cpu().numpy(), t.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_vertices_and_triangles_match_reference(dev, name):
    v, t = _run(name, dev)
    assert np.array_equal(v, R[name + "_verts"])
    assert np.array_equal(t, R[name + "_tris"])          # index for index
    _, tc = _run(name, dev, triangulation="closed")
    assert tc.min() >= 0 and tc.max() < len(v)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_single_triangle_cubes_match_reference(oracle, dev, name):
    """A cube with exactly three cut edges (one corner on its own side) has a
    single triangle: the reference's, with the same orientation."""
    coords, corners, iso = CASES[name]
    _, vi, ei, ids = oracle.sparse_mc_vertices(coords, corners, iso, return_ids=True)
    ncut = np.bincount(vi, minlength=len(coords))
    single = np.nonzero(ncut == 3)[0]
    assert len(single) > 50
    want = {tuple(sorted(ids[vi == s])) for s in single}
    _, t = _run(name, dev, triangulation="closed")
    ours = {tuple(sorted(x)): tuple(r) for x, r in zip(t, _rot(t))}
    ref = {tuple(sorted(x)): tuple(r) for x, r in zip(R[name + "_tris"], _rot(R[name + "_tris"]))}
    for key in want:
        assert key in ours and key in ref and ours[key] == ref[key]


@pytest.mark.gpu
def test_sphere_closed_oriented_same_volume(dev):
    v, t = _run("sphere", dev, triangulation="closed")
    _, cnt, dcnt = _edges(t)
    assert (cnt == 2).all() and (dcnt == 1).all()        # closed, each edge once each way
    assert len(t) == len(R["sphere_tris"])
    vol, ref_vol = _volume(v, t), _volume(R["sphere_verts"], R["sphere_tris"])
    assert vol > 0 and abs(vol - ref_vol) < 1e-3 * ref_vol   # normals from inside to outside


@pytest.mark.gpu
def test_lattice_manifold(dev):
    """Random values on a full 12^3 block (many ambiguous faces): every edge
    inside the block is in exactly two triangles, once in each direction;
    open edges lie on the block's outer faces only."""
    v, t = _run("lattice", dev, triangulation="closed")
    e, cnt, dcnt = _edges(t)
    assert (cnt <= 2).all() and (dcnt == 1).all()
    und, c2 = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    open_v = v[und[c2 == 1].reshape(-1)]
    assert np.all(np.any((open_v == 0) | (open_v == 12), axis=1))


@pytest.mark.gpu
def test_ensure_consistency(oracle, dev):
    """Averaged shared corners: the vertices the reference gives, up to the
    order of the sums (1 ulp of the corner values)."""
    if not oracle.ref_sparse_mc_available():
        pytest.skip("oracle/_ref/libref_sparse_mc.so not built")
    coords, corners, iso = CASES["random"]
    rv, _ = oracle.ref_sparse_mc(coords, corners, iso, True)
    v, t = _run("random", dev, ensure=True)
    assert v.shape == rv.shape and np.abs(v - rv).max() < 4e-6


@pytest.mark.gpu
def test_live_reference_larger(oracle, dev):
    if not oracle.ref_sparse_mc_available():
        pytest.skip("oracle/_ref/libref_sparse_mc.so not built")
    for coords, corners, iso in (M.sphere_band(n=64, c=(31.7, 32.2, 30.9), r=25.3) + (0.0,),
                                 M.random_subset(seed=9, n=40, frac=0.3) + (-0.2,)):
        rv, rt = oracle.ref_sparse_mc(coords, corners, iso)
        v, t = cubvh.sparse_marching_cubes(torch.from_numpy(coords).to(dev), torch.from_numpy(corners).to(dev), iso)
        assert np.array_equal(v.cpu().numpy(), rv)
        assert np.array_equal(t.cpu().numpy(), rt)


@pytest.mark.gpu
def test_empty_and_errors(dev):
    v, t = cubvh.sparse_marching_cubes(torch.zeros(0, 3, dtype=torch.int32, device=dev),
                                       torch.zeros(0, 8, device=dev), 0.0)
    assert v.shape == (0, 3) and t.shape == (0, 3)
    v, t = cubvh.sparse_marching_cubes(torch.zeros(5, 3, dtype=torch.int32, device=dev),
                                       torch.ones(5, 8, device=dev), 0.0)
    assert v.shape == (0, 3) and t.shape == (0, 3)
    with pytest.raises(RuntimeError):
        cubvh.sparse_marching_cubes(torch.zeros(5, 3, dtype=torch.int32, device=dev), torch.ones(5, 7, device=dev), 0.0)


def _model_tris(oracle, coords, corners, iso):
    import smc_model
    _, vi, ei, ids = oracle.sparse_mc_vertices(coords, corners, iso, return_ids=True)
    return smc_model.mesh_triangles(coords, corners, iso, vi, ei, ids)


@pytest.mark.parametrize("seed", range(25))
def test_model_closed_on_random_lattices(oracle, seed):
    """The triangulation rules (tests/smc_model.py, the kernels' rules) on a
    random field over a 6^3 block: every edge inside the block in exactly two
    triangles, once in each direction."""
    coords, corners = M.lattice_field(seed=100 + seed, n=6)
    v = oracle.sparse_mc_vertices(coords, corners, 0.0)
    t = _model_tris(oracle, coords, corners, 0.0)
    e, cnt, dcnt = _edges(t)
    assert (cnt <= 2).all() and (dcnt == 1).all()
    und, c2 = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    open_v = v[und[c2 == 1].reshape(-1)]
    assert np.all(np.any((open_v == 0) | (open_v == 6), axis=1))


def test_model_single_triangles_match_reference(oracle):
    for name in sorted(CASES):
        coords, corners, iso = CASES[name]
        t = _model_tris(oracle, coords, corners, iso)
        ref = set(map(tuple, _rot(R[name + "_tris"])))
        _, vi, ei, ids = oracle.sparse_mc_vertices(coords, corners, iso, return_ids=True)
        ncut = np.bincount(vi, minlength=len(coords))
        single = set(np.nonzero(ncut == 3)[0])
        own = {tuple(sorted(ids[vi == s])) for s in single}
        mine = [tuple(r) for x, r in zip(t, _rot(t)) if tuple(sorted(x)) in own]
        assert len(mine) == len(own) and all(m in ref for m in mine)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_kernels_match_model(oracle, dev, name):
    coords, corners, iso = CASES[name]
    _, t = _run(name, dev, triangulation="closed")
    assert np.array_equal(t, _model_tris(oracle, coords, corners, iso))


@pytest.mark.gpu
def test_fetch_on_another_stream(dev):
    """C ABI: a result built on one stream and fetched on another equals the
    one-stream result (the fetch waits for the building stream's kernels)."""
    import ctypes
    from cubvh_b200 import api
    from cubvh_b200._lib import check, lib
    coords, corners, iso = M.sphere_band(n=64, c=(31.7, 32.2, 30.9), r=25.3) + (0.0,)
    c = torch.from_numpy(coords).to(dev)
    v = torch.from_numpy(corners).to(dev)
    want_v, want_t = cubvh.sparse_marching_cubes(c, v, iso)
    build, fetch = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    res, nv, nt = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int64()
    check(lib().cubvh_sparse_marching_cubes(api._ptr(c), api._ptr(v), len(coords), float(iso), 0,
                                            ctypes.c_void_p(build.cuda_stream), ctypes.byref(res),
                                            ctypes.byref(nv), ctypes.byref(nt)), "sparse_marching_cubes")
    try:
        with torch.cuda.stream(fetch):
            got_v = torch.empty(nv.value, 3, dtype=torch.float32, device=dev)
            got_t = torch.empty(nt.value, 3, dtype=torch.int32, device=dev)
        check(lib().cubvh_sparse_mc_fetch(res, api._ptr(got_v), api._ptr(got_t), ctypes.c_void_p(fetch.cuda_stream)),
              "sparse_mc_fetch")
        fetch.synchronize()
    finally:
        check(lib().cubvh_sparse_mc_free(res), "sparse_mc_free")
    assert torch.equal(got_v, want_v) and torch.equal(got_t, want_t)


def _quantised_field(seed, n, levels):
    rng = np.random.default_rng(seed)
    field = rng.choice(levels, size=(n + 1, n + 1, n + 1)).astype(np.float32)
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    cp = g[:, None, :] + M.OFF[None]
    return g.astype(np.int32), field[cp[..., 0], cp[..., 1], cp[..., 2]]


@pytest.mark.parametrize("levels,iso", [((-1.0, 0.0, 1.0), 0.0), ((-1.0, 0.0, 1.0), 0.5), ((-1.0, 1.0), 0.0),
                                        ((0.0, 1.0, 2.0, 3.0), 1.5)])
def test_model_closed_on_quantised_lattices(oracle, levels, iso):
    """Fields with exact ties (corners equal to iso, flat saddles): still
    closed and consistently oriented inside the block, no triangle repeats a
    vertex."""
    for seed in range(8):
        coords, corners = _quantised_field(seed, 6, list(levels))
        v = oracle.sparse_mc_vertices(coords, corners, iso)
        t = _model_tris(oracle, coords, corners, iso)
        if len(t) == 0:
            continue
        e, cnt, dcnt = _edges(t)
        assert (cnt <= 2).all() and (dcnt == 1).all()
        und, c2 = np.unique(np.sort(e, 1), axis=0, return_counts=True)
        open_v = v[und[c2 == 1].reshape(-1)]
        assert np.all(np.any((open_v == 0) | (open_v == 6), axis=1))
        assert not np.any((t[:, 0] == t[:, 1]) | (t[:, 1] == t[:, 2]) | (t[:, 0] == t[:, 2]))
