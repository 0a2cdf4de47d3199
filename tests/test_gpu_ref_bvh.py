"""GPU parity against the REFERENCE'S OWN CUDA kernels, on the full-size
inputs of the benchmark configurations.

The reference's src/bvh.cu, compiled unchanged into oracle/_ref/libref_bvh.so
(against the project-written Eigen stand-in), runs its four kernels on the
same device tensors as ours.  The rules (FP64 brute force = the oracle):

- stab directions: ours equal the reference's device directions bit for bit;
- distances, depths and uvw: ours within 1e-6 relative / 1e-7 absolute of
  FP64 on a strided sample (the reference's own largest error is reported
  beside ours: its FP32 arithmetic does not always meet that bound);
- face_id: where ours and the reference's differ, the two faces must be a
  tie (FP64 distances / depths within 1e-7) or the reference's face must be
  the FP64-farther one; never ours;
- signs: every disagreement with the reference is listed with the FP64
  verdict, which must side with ours;
- floodfill: the 512^3 tori occupancy labels equal the reference's.

Each test records its counts in a JSON report (environment variable
CUBVH_PARITY_REPORT names the file; one JSON object per line)."""

import json
import os

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_bvh_available(),
                                 reason="oracle/_ref/libref_bvh.so not built (needs the reference checkout)")]

RTOL, ATOL, TIE = 1e-6, 1e-7, 1e-7


def _report(name, rec):
    rec = dict(test=name, **rec)
    print(json.dumps(rec))
    path = os.environ.get("CUBVH_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(rec) + "\n")


def _np(t):
    return t.detach().cpu().numpy()


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _rel_err(got, want):
    err = np.abs(got.astype(np.float64) - want)
    return err, err / np.maximum(np.abs(want), 1e-300)


def _within(got, want):
    err = np.abs(got.astype(np.float64) - want)
    return err <= ATOL + RTOL * np.abs(want)


def _ref_distance(R, P, mode=None, uvw=False):
    n = P.shape[0]
    d = torch.empty(n, device=P.device)
    fid = torch.empty(n, dtype=torch.int64, device=P.device)
    u = torch.empty(n, 3, device=P.device) if uvw else None
    if mode is None:
        R.unsigned_distance_gpu(P.data_ptr(), n, d.data_ptr(), fid.data_ptr(), u.data_ptr() if uvw else 0,
                                _stream(P.device))
    else:
        R.signed_distance_gpu(P.data_ptr(), n, mode, d.data_ptr(), fid.data_ptr(), u.data_ptr() if uvw else 0,
                              _stream(P.device))
    torch.cuda.synchronize()
    return d, fid, u


def _face_mismatches(v, f, pts, ours, ref, limit=20000):
    """FP64 distances of both faces where the face ids differ: (checked, ties,
    reference farther, ours farther, largest gap)."""
    mm = np.nonzero(ours != ref)[0]
    sel = mm[:: max(1, len(mm) // limit)] if len(mm) else mm
    if len(sel) == 0:
        return dict(face_mismatch=0)
    a, _ = O.face_dist64(v, f, pts[sel], ours[sel])
    b, _ = O.face_dist64(v, f, pts[sel], ref[sel])
    gap = b - a
    return dict(face_mismatch=int(len(mm)), checked=int(len(sel)), ties=int((np.abs(gap) <= TIE).sum()),
                ref_farther=int((gap > TIE).sum()), ours_farther=int((gap < -TIE).sum()),
                max_gap=float(np.abs(gap).max()))


def test_stab_directions_equal_reference(dev):
    from cubvh_b200._lib import lib
    import ctypes
    for first in (0, 7, (1 << 31) - (1 << 18)):
        n = 1 << 18
        ours = torch.empty(n, 32, 3, device=dev)
        ref = torch.empty(n, 32, 3, device=dev)
        assert lib().cubvh_stab_directions(first, n, ctypes.c_void_p(ours.data_ptr()),
                                           ctypes.c_void_p(_stream(dev))) == 0
        O.ref_stab_dirs_gpu_ptr(first, n, ref.data_ptr(), _stream(dev))
        torch.cuda.synchronize()
        assert torch.equal(ours.view(torch.int32), ref.view(torch.int32)), f"first {first}"
    # the host build of the same code (host sincosf, no FMA) differs in the last bits
    host = O.ref_stab_dirs_host(4096, first)
    _report("stab_directions", dict(queries=3 << 18, equal=True, host_build_components_compared=host.size,
                                    host_build_components_differing=int((host != _np(ref[:4096])).sum())))


def test_c0_udf_uvw_vs_reference(dev):
    w = W.udf_icosphere()
    v, f, pts = w["vertices"], w["faces"], w["points"]
    P = torch.from_numpy(pts).to(dev)
    d, fid, uvw = cubvh.cuBVH(v, f).unsigned_distance(P, return_uvw=True)
    rd, rfid, ruvw = _ref_distance(O.ReferenceBVH(v, f), P, uvw=True)
    d, fid, uvw, rd, rfid, ruvw = map(_np, (d, fid, uvw, rd, rfid, ruvw))
    rec = _face_mismatches(v, f, pts, fid, rfid)
    assert rec.get("ours_farther", 0) == 0
    sub = np.arange(0, len(pts), 16)
    od, ofid, ouvw, _, _ = O.udf64(v, f, pts[sub])
    assert _within(d[sub], od).all() and np.array_equal(fid[sub], ofid)
    assert _within(uvw[sub], ouvw).all()
    e_o, r_o = _rel_err(d[sub], od)
    e_r, r_r = _rel_err(rd[sub], od)
    same = rfid[sub] == ofid
    eu_r = np.abs(ruvw[sub][same].astype(np.float64) - ouvw[same])
    rec.update(queries=len(pts), sample=len(sub), ours_max_abs=float(e_o.max()), ours_max_rel=float(r_o.max()),
               ref_max_abs=float(e_r.max()), ref_max_rel=float(r_r.max()),
               ref_outside_tolerance=int((~_within(rd[sub], od)).sum()),
               ours_uvw_max_abs=float(np.abs(uvw[sub].astype(np.float64) - ouvw).max()),
               ref_uvw_max_abs=float(eu_r.max()) if eu_r.size else 0.0)
    _report("C0 udf+uvw icosphere L4, 1,048,576 points", rec)


def test_c1_rays_vs_reference(dev):
    v, f = W.displaced_icosphere(6, 1)
    ro_np, rd_np = W.camera_rays(8, 2048, 50.0, 2.5, 1)
    ro, rdir = torch.from_numpy(ro_np).to(dev), torch.from_numpy(rd_np).to(dev)
    _, fid, depth = cubvh.cuBVH(v, f).ray_trace(ro, rdir)
    n = ro.shape[0]
    rpos = torch.empty(n, 3, device=dev)
    rfid = torch.empty(n, dtype=torch.int64, device=dev)
    rdep = torch.empty(n, device=dev)
    O.ReferenceBVH(v, f).ray_trace_gpu(ro.data_ptr(), rdir.data_ptr(), n, rpos.data_ptr(), rfid.data_ptr(),
                                       rdep.data_ptr(), _stream(dev))
    torch.cuda.synchronize()
    fid, depth, rfid, rdep = map(_np, (fid, depth, rfid, rdep))
    hit_mm = np.nonzero((fid >= 0) != (rfid >= 0))[0]
    face_mm = np.nonzero((fid != rfid) & (fid >= 0) & (rfid >= 0))[0]
    rec = dict(rays=n, hits=int((fid >= 0).sum()), hit_mismatch=int(len(hit_mm)), face_mismatch=int(len(face_mm)))
    # every disagreement, judged by FP64 (ray64: exact closest hit, lowest face on ties)
    check = np.concatenate([hit_mm, face_mm[:: max(1, len(face_mm) // 4000)]])
    if len(check):
        t64, f64, fl64 = O.ray64(v, f, ro_np[check], rd_np[check])
        ours_ok = fid[check] == f64
        ref_ok = rfid[check] == f64
        # a face pair hit within 1e-7 of each other is a tie
        tie = np.zeros(len(check), bool)
        both = (fid[check] >= 0) & (rfid[check] >= 0)
        if both.any():
            tie[both] = np.abs(rdep[check][both].astype(np.float64) - t64[both]) <= TIE + RTOL * t64[both]
        rec.update(checked=int(len(check)), ours_equal_fp64=int(ours_ok.sum()), ref_equal_fp64=int(ref_ok.sum()),
                   ref_ties=int((~ref_ok & tie).sum()), fp64_ambiguous=int(((fl64 & 1) != 0).sum()))
        assert (ours_ok | ((fl64 & 1) != 0)).all(), "our ray face differs from FP64"
    sub = np.arange(0, n, 4099)
    t64, f64, _ = O.ray64(v, f, ro_np[sub], rd_np[sub])
    h = f64 >= 0
    assert np.array_equal(fid[sub], f64) and _within(depth[sub][h], t64[h]).all()
    e_o, r_o = _rel_err(depth[sub][h], t64[h])
    e_r, r_r = _rel_err(rdep[sub][h], t64[h])
    rec.update(sample=len(sub), sample_hits=int(h.sum()), ours_depth_max_abs=float(e_o.max()),
               ours_depth_max_rel=float(r_o.max()), ref_depth_max_abs=float(e_r.max()),
               ref_depth_max_rel=float(r_r.max()), ref_outside_tolerance=int((~_within(rdep[sub][h], t64[h])).sum()))
    _report("C1 ray_trace displaced icosphere L6, 8 x 2048^2 rays", rec)


def _sign_disagreements(v, f, pts, d, rd, mode, dirs=None, limit=4000):
    neg, rneg = d < 0, rd < 0
    mm = np.nonzero(neg != rneg)[0]
    rec = dict(sign_mismatch=int(len(mm)))
    if len(mm):
        sel = mm[:limit]
        if mode == "watertight":
            sd, _, fl = O.sdf_watertight64(v, f, pts[sel])
        else:
            sd, _, fl = O.sdf_raystab64(v, f, pts[sel], dirs=dirs[sel])
        ours_ok = neg[sel] == (sd < 0)
        rec.update(checked=int(len(sel)), ours_equal_fp64=int(ours_ok.sum()),
                   ref_equal_fp64=int((rneg[sel] == (sd < 0)).sum()), fp64_flagged=int((fl != 0).sum()),
                   examples=[dict(index=int(i), ours=float(d[i]), reference=float(rd[i]), fp64=float(s))
                             for i, s in zip(sel[:8], sd[:8])])
        assert ours_ok.all(), "a sign of ours differs from the FP64 verdict"
    return rec


def test_c1_sdf_watertight_vs_reference(dev):
    w = W.rays_displaced(res=8)   # the C1 mesh and its 8,388,608 SDF points (rays unused)
    v, f, pts = w["vertices"], w["faces"], w["points"]
    P = torch.from_numpy(pts).to(dev)
    d, fid, _ = cubvh.cuBVH(v, f).signed_distance(P, mode="watertight")
    rd, rfid, _ = _ref_distance(O.ReferenceBVH(v, f), P, mode=0)
    d, fid, rd, rfid = map(_np, (d, fid, rd, rfid))
    rec = _sign_disagreements(v, f, pts, d, rd, "watertight")
    rec.update(_face_mismatches(v, f, pts, fid, rfid, limit=4000))
    assert rec.get("ours_farther", 0) == 0
    sub = np.arange(0, len(pts), 1031)
    sd, sfid, _ = O.sdf_watertight64(v, f, pts[sub])
    assert np.array_equal(np.signbit(d[sub]), np.signbit(sd.astype(np.float32)))
    assert _within(np.abs(d[sub]), np.abs(sd)).all()
    e_r, r_r = _rel_err(np.abs(rd[sub]), np.abs(sd))
    rec.update(queries=len(pts), sample=len(sub), ref_max_abs=float(e_r.max()), ref_max_rel=float(r_r.max()))
    _report("C1 signed_distance watertight, 8,388,608 points", rec)


def test_c1_sdf_raystab_vs_reference(dev, stab_dirs):
    v, f = W.displaced_icosphere(6, 1)
    lo, hi = v.min(0), v.max(0)
    c, h = (lo + hi) / 2, (hi - lo) / 2 * 1.1
    pts = (c + np.random.default_rng(5).uniform(-1, 1, (1 << 20, 3)) * h).astype(np.float32)
    P = torch.from_numpy(pts).to(dev)
    d, fid, _ = cubvh.cuBVH(v, f).signed_distance(P, mode="raystab")
    rd, rfid, _ = _ref_distance(O.ReferenceBVH(v, f), P, mode=1)
    d, fid, rd, rfid = map(_np, (d, fid, rd, rfid))
    dirs = stab_dirs(len(pts))   # the reference's device directions of every query
    rec = _sign_disagreements(v, f, pts, d, rd, "raystab", dirs=dirs)
    rec.update(queries=len(pts), inside=int((d < 0).sum()))
    sub = np.arange(0, len(pts), 257)
    sd, _, _ = O.sdf_raystab64(v, f, pts[sub], dirs=dirs[sub])
    assert np.array_equal(np.signbit(d[sub]), np.signbit(sd.astype(np.float32)))
    rec.update(sample=len(sub))
    _report("raystab on the C1 mesh, 1,048,576 points in its box dilated by 10%", rec)


def test_c2_udf_and_floodfill_vs_reference(dev):
    w = W.dense_tori(512)
    v, f = w["vertices"], w["faces"]
    grid = W.dense_grid(512)
    P = torch.from_numpy(grid).to(dev)
    d, fid, _ = cubvh.cuBVH(v, f).unsigned_distance(P)
    rd, rfid, _ = _ref_distance(O.ReferenceBVH(v, f), P)
    occ = (d < 2.0 / 512).view(512, 512, 512)
    rocc = (rd < 2.0 / 512).view(512, 512, 512)
    labels = cubvh.floodfill(occ)
    d, fid, rd, rfid = map(_np, (d, fid, rd, rfid))
    rec = _face_mismatches(v, f, grid, fid, rfid, limit=4000)
    assert rec.get("ours_farther", 0) == 0
    sub = np.arange(0, len(grid), 16411)
    od, ofid, _, _, _ = O.udf64(v, f, grid[sub])
    assert _within(d[sub], od).all() and np.array_equal(fid[sub], ofid)
    e_r, r_r = _rel_err(rd[sub], od)
    rec.update(queries=len(grid), sample=len(sub), ref_max_abs=float(e_r.max()), ref_max_rel=float(r_r.max()),
               occupancy_voxels_differing=int((occ != rocc).sum().item()))
    # floodfill of our occupancy by the reference's own CUDA floodfill
    if O.ref_floodfill_available():
        g = _np(occ)
        assert np.array_equal(_np(labels), O.ref_floodfill(g))
        rec.update(floodfill_512_equal=True, blocked=int(g.sum()))
    _report("C2 udf 512^3 grid of 12 tori + floodfill", rec)


# ------------------------------------------------ recorded reference outputs
FIX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_bvh.npz"))


@pytest.mark.parametrize("name", ["dodeca", "ico3", "disp4", "tori3"])
def test_ours_vs_recorded_reference(dev, stab_dirs, name):
    """Our kernels on the fixture inputs against the reference's recorded CUDA
    outputs (tests/golden/ref_bvh.npz): face ids equal except at FP64 ties,
    signs equal except where FP64 sides with ours, hits equal except where
    FP64 sides with ours."""
    g = lambda k: FIX[f"{name}_{k}"]
    v, f, pts = g("v"), g("f"), g("pts")
    bvh = cubvh.cuBVH(v, f)
    P = torch.from_numpy(pts).to(dev)
    d, fid, uvw = map(_np, bvh.unsigned_distance(P, return_uvw=True))
    rec = dict(udf=_face_mismatches(v, f, pts, fid, g("gpu_udf_fid")))
    assert rec["udf"].get("ours_farther", 0) == 0
    dirs = g("gpu_stab_dirs") if f"{name}_gpu_stab_dirs" in FIX.files else stab_dirs(len(pts))
    for tag, mode in (("sdfw", "watertight"), ("sdfr", "raystab")):
        sd, sfid, _ = map(lambda t: _np(t) if t is not None else None, bvh.signed_distance(P, mode=mode))
        rec[tag] = _sign_disagreements(v, f, pts, sd, g(f"gpu_{tag}_d"), mode, dirs=dirs)
        rec[tag].update(_face_mismatches(v, f, pts, sfid, g(f"gpu_{tag}_fid")))
        assert rec[tag].get("ours_farther", 0) == 0
    _, rfid, rdep = map(_np, bvh.ray_trace(torch.from_numpy(g("ro")).to(dev), torch.from_numpy(g("rd")).to(dev)))
    mm = np.nonzero(rfid != g("gpu_ray_fid"))[0]
    rec["ray"] = dict(face_mismatch=int(len(mm)))
    if len(mm):
        t64, f64, fl = O.ray64(v, f, g("ro")[mm], g("rd")[mm])
        assert ((rfid[mm] == f64) | ((fl & 1) != 0)).all()
        rec["ray"].update(ours_equal_fp64=int((rfid[mm] == f64).sum()),
                          ref_equal_fp64=int((g("gpu_ray_fid")[mm] == f64).sum()))
    _report(f"recorded reference outputs: {name}", rec)
