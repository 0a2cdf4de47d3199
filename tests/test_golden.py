"""Frozen fixtures (tests/golden/golden.npz, written by make_golden.py): the
oracle must still reproduce them (CPU) and the kernels must match them (GPU)."""

import os

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz"))


def test_oracle_reproduces_fixtures(oracle):
    d, fid, uvw, _, nn = oracle.udf64(G["dodeca_v"], G["dodeca_f"], G["dodeca_pts"])
    assert np.array_equal(d, G["dodeca_dist"]) and np.array_equal(fid, G["dodeca_fid"])
    assert np.array_equal(uvw, G["dodeca_uvw"])
    sw, _, _ = oracle.sdf_watertight64(G["dodeca_v"], G["dodeca_f"], G["dodeca_pts"])
    sr, _, _ = oracle.sdf_raystab64(G["dodeca_v"], G["dodeca_f"], G["dodeca_pts"])
    assert np.array_equal(sw, G["dodeca_sdf_w"]) and np.array_equal(sr, G["dodeca_sdf_r"])
    t, rfid, _ = oracle.ray64(G["ico_v"], G["ico_f"], G["rays_o"], G["rays_d"])
    assert np.array_equal(t, G["ray_t"]) and np.array_equal(rfid, G["ray_fid"])
    assert np.array_equal(oracle.floodfill(G["ff_grid"]), G["ff_labels"])
    assert np.array_equal(oracle.stab_offsets(64), G["stab_offsets"])
    # a closed solid: the watertight and raystab signs agree, and the
    # dodecahedron's circumradius-1 points inside are negative
    assert np.array_equal(np.sign(sw), np.sign(sr))
    assert (sw[np.linalg.norm(G["dodeca_pts"], axis=1) < 0.7] < 0).all()


@pytest.mark.gpu
def test_kernels_match_fixtures(dev):
    bvh = cubvh.cuBVH(G["dodeca_v"], G["dodeca_f"])
    p = torch.from_numpy(G["dodeca_pts"]).to(dev)
    d, fid, uvw = bvh.unsigned_distance(p, return_uvw=True)
    assert np.array_equal(d.cpu().numpy(), G["dodeca_dist"].astype(np.float32))
    assert np.array_equal(fid.cpu().numpy(), G["dodeca_fid"])
    assert np.array_equal(uvw.cpu().numpy(), G["dodeca_uvw"].astype(np.float32))
    sw, _, _ = bvh.signed_distance(p, mode="watertight")
    sr, _, _ = bvh.signed_distance(p, mode="raystab")
    assert np.array_equal(sw.cpu().numpy(), G["dodeca_sdf_w"].astype(np.float32))
    assert np.array_equal(sr.cpu().numpy(), G["dodeca_sdf_r"].astype(np.float32))
    b2 = cubvh.cuBVH(G["ico_v"], G["ico_f"])
    _, rfid, t = b2.ray_trace(torch.from_numpy(G["rays_o"]).to(dev), torch.from_numpy(G["rays_d"]).to(dev))
    assert np.array_equal(t.cpu().numpy(), G["ray_t"].astype(np.float32))
    assert np.array_equal(rfid.cpu().numpy(), G["ray_fid"])
    lab = cubvh.floodfill(torch.from_numpy(G["ff_grid"]).to(dev))
    assert np.array_equal(lab.cpu().numpy(), G["ff_labels"])
