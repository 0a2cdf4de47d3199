"""The reference's own BVH code (src/bvh.cu, compiled unchanged into
oracle/_ref/libref_bvh.so against the project-written Eigen stand-in) pins the
oracle and the state_dict format (CPU tests here; the GPU comparisons with the
reference's CUDA kernels are in test_gpu_ref_bvh.py).

- The oracle's FP32 restatement of the reference (oracle.cpp, used as the
  reference mirror and the CPU baseline) gives the same bits as the
  reference's own host build for the BVH records, distances, face ids, uvw,
  both signed modes and rays.
- cuBVH.state_dict() writes the same node and triangle records as the
  reference's own build.
- The host stab-ray directions of the oracle (libm sin/cos) are the reference
  host build's.
"""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_bvh_available(),
                                reason="oracle/_ref/libref_bvh.so not built (needs the reference checkout)")


def _signed_zero_sheet():
    """A flat sheet in z = 0 with -0.0 mixed into the coordinates (ties and
    signed zeros in the median splits and the boxes)."""
    g = np.stack(np.meshgrid(np.arange(40), np.arange(40), indexing="ij"), -1).reshape(-1, 2)
    v = np.concatenate([g * 0.01, np.zeros((len(g), 1))], 1).astype(np.float32)
    v[::3, 2] = -0.0
    v[::7, 0] = -0.0 * v[::7, 0]
    i = np.nonzero((g[:, 0] < 39) & (g[:, 1] < 39))[0]
    return v, np.concatenate([np.stack([i, i + 40, i + 1], 1), np.stack([i + 1, i + 40, i + 41], 1)])


def _meshes():
    yield "icosphere4", W.icosphere(4, 0.8)
    yield "sheet", _signed_zero_sheet()
    yield "displaced5", W.displaced_icosphere(5, 1)
    yield "dodecahedron", W.dodecahedron()
    v, f = W.random_tori(2, n_tori=3, n_major=48, n_minor=12)
    yield "tori3", (v, f)


MESHES = dict(_meshes())


@pytest.mark.parametrize("name", list(MESHES))
def test_state_dict_records_equal_reference_build(name):
    v, f = MESHES[name]
    ref_nodes, ref_tris = O.ReferenceBVH(v, f).state_dict_arrays()
    sd = cubvh.cuBVH(v, f).state_dict()
    assert np.array_equal(sd["nodes"].numpy(), ref_nodes)
    assert np.array_equal(sd["triangles"].numpy(), ref_tris)


def _queries(v, f, n, seed):
    """Half uniform in the dilated bounding box, half within 0.01 of the surface."""
    rng = np.random.default_rng(seed)
    lo, hi = v.min(0) - 0.2, v.max(0) + 0.2
    far = rng.uniform(lo, hi, (n - n // 2, 3)).astype(np.float32)
    return np.concatenate([far, W.surface_points(v, f, n // 2, 0.01, rng)], 0)


@pytest.mark.parametrize("name", list(MESHES))
def test_fp32_restatement_equals_reference_host(name):
    v, f = MESHES[name]
    R, M = O.ReferenceBVH(v, f), O.RefBVH(v, f)
    pts = _queries(v, f, 6000, 7)
    a, b = R.unsigned_distance(pts, return_uvw=True), M.unsigned_distance(pts, return_uvw=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    a, b = R.signed_distance(pts, 0, return_uvw=True), M.signed_distance(pts, 0, return_uvw=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    # raystab with host (libm) stab directions on both sides; queries start at
    # index 1000 within the call
    a = R.signed_distance(pts[:800], 1, first_index=1000)
    b = M.signed_distance(np.concatenate([np.zeros((1000, 3), np.float32), pts[:800]]), 1)
    assert np.array_equal(a[0], b[0][1000:]) and np.array_equal(a[1], b[1][1000:])
    rng = np.random.default_rng(3)
    ro = (rng.standard_normal((4000, 3)) * 2).astype(np.float32)
    rd = (pts[:4000] - ro).astype(np.float32)
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    a, b = R.ray_trace(ro, rd), M.ray_trace(ro, rd)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_stride_sampling_matches_dense():
    v, f = MESHES["icosphere4"]
    R = O.ReferenceBVH(v, f)
    pts = W.uniform_points(3000, 1)
    d, fid, _ = R.unsigned_distance(pts)
    d3, fid3, _ = R.unsigned_distance(pts, stride=3)
    assert np.array_equal(d[::3], d3) and np.array_equal(fid[::3], fid3)
    s, g, _ = R.signed_distance(pts, 1)
    s3, g3, _ = R.signed_distance(pts, 1, stride=3)
    assert np.array_equal(s[::3], s3)


def test_host_stab_directions_equal_oracle_libm():
    ref = O.ref_stab_dirs_host(2000, 12345)
    assert np.array_equal(ref, O.stab_dirs(2000, 12345))


def test_reference_build_accepts_torch_style_inputs():
    v, f = MESHES["dodecahedron"]
    R = O.ReferenceBVH(torch.from_numpy(v).numpy(), f.astype(np.int32))
    assert R.n_nodes > 0
    with pytest.raises(ValueError):
        O.ReferenceBVH(v, f + len(v))
