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

import os

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


# ------------------------------------------------ recorded reference outputs
# tests/golden/ref_bvh.npz: the reference's CUDA kernels and host build on four
# cases (make_ref_bvh.py beside it), including its test's own dodecahedron.
FIX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_bvh.npz"))
FIX_CASES = ["dodeca", "ico3", "disp4", "tori3"]


@pytest.mark.parametrize("name", FIX_CASES)
def test_reference_host_build_reproduces_fixture(name):
    """The live host build of the reference (this checkout's oracle/_ref) gives
    the recorded host outputs bit for bit."""
    g = lambda k: FIX[f"{name}_{k}"]
    R = O.ReferenceBVH(g("v"), g("f"))
    for tag, mode in (("udf", None), ("sdfw", 0), ("sdfr", 1)):
        d, fid, uvw = (R.unsigned_distance(g("pts"), return_uvw=True) if mode is None
                       else R.signed_distance(g("pts"), mode, return_uvw=True))
        assert np.array_equal(d, g(f"host_{tag}_d")) and np.array_equal(fid, g(f"host_{tag}_fid"))
        assert np.array_equal(uvw, g(f"host_{tag}_uvw"))
    pos, fid, dep = R.ray_trace(g("ro"), g("rd"))
    assert np.array_equal(fid, g("host_ray_fid")) and np.array_equal(dep, g("host_ray_depth"))


@pytest.mark.parametrize("name", FIX_CASES)
def test_oracle_agrees_with_recorded_reference(oracle, name):
    """The FP64 oracle against the reference's recorded CUDA outputs: face ids
    differ only at ties (FP64 distances within 1e-7), distances and depths
    within the reference's FP32 error, signs equal except on points within
    1e-6 of the surface (where FP32 cannot decide)."""
    g = lambda k: FIX[f"{name}_{k}"]
    v, f, pts = g("v"), g("f"), g("pts")
    od, ofid, _, _, _ = oracle.udf64(v, f, pts)
    rfid = g("gpu_udf_fid")
    mm = ofid != rfid
    if mm.any():
        a, _ = oracle.face_dist64(v, f, pts[mm], rfid[mm])
        assert np.abs(a - od[mm]).max() <= 1e-7
    assert np.abs(g("gpu_udf_d").astype(np.float64) - od).max() < 1e-6
    sw, _, _ = oracle.sdf_watertight64(v, f, pts)
    far = np.abs(sw) > 1e-6
    assert np.array_equal(np.signbit(g("gpu_sdfw_d"))[far], (sw < 0)[far])
    t, rf, _ = oracle.ray64(v, f, g("ro"), g("rd"))
    hit = rf >= 0
    assert np.array_equal(hit, g("gpu_ray_fid") >= 0)
    assert np.abs(g("gpu_ray_depth")[hit].astype(np.float64) - t[hit]).max() < 1e-5
    if f"{name}_gpu_stab_dirs" in FIX.files:
        sr, _, _ = oracle.sdf_raystab64(v, f, pts, dirs=g("gpu_stab_dirs"))
        far = np.abs(sr) > 1e-6
        assert np.array_equal(np.signbit(g("gpu_sdfr_d"))[far], (sr < 0)[far])


def test_fixture_dodecahedron_is_the_reference_tests():
    """The dodecahedron case is the reference test's own solid: 20 vertices on
    the unit sphere, 36 faces, every vertex used."""
    v, f = FIX["dodeca_v"], FIX["dodeca_f"]
    assert v.shape == (20, 3) and f.shape == (36, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-6)
    assert np.array_equal(np.unique(f), np.arange(20))
