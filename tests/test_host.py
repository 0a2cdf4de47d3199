"""Host-side checks that need no GPU: the C ABI exports, the BVH layout
invariants (every quantised box contains what it bounds), the reference-format
state_dict, the Python surface's error behaviour, and the multi-rank timing
reduction (gloo, two processes)."""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import _lib
from cubvh_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

NODE = np.dtype([('o', '<f4', 3), ('e', 'i1', 3), ('nint', 'u1'), ('cb', '<i4'), ('tb', '<i4'), ('meta', 'u1', 8),
                 ('qlx', 'u1', 8), ('qly', 'u1', 8), ('qlz', 'u1', 8), ('qhx', 'u1', 8), ('qhy', 'u1', 8),
                 ('qhz', 'u1', 8)])
TRI = np.dtype([('a', '<f4', 3), ('id', '<i4'), ('b', '<f4', 3), ('ke2', '<f4'), ('c', '<f4', 3), ('k', '<f4')])
REFNODE = np.dtype([('lo', '<f4', 3), ('hi', '<f4', 3), ('left', '<i4'), ('right', '<i4'), ('escape', '<i4')])


def header_functions():
    src = open(os.path.join(ROOT, "include", "cubvh_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(cubvh_\w+)\(", src, re.M)))


def test_library_exports_every_header_function():
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/cubvh_b200.h but not exported"
    assert _lib.version().startswith("cubvh_b200")


def layout(bvh):
    nf, nn, depth = bvh._info()
    nodes = np.zeros(nn, NODE)
    tris = np.zeros(nf, TRI)
    assert _lib.lib().cubvh_bvh_layout(bvh.impl.raw, nodes.ctypes.data, tris.ctypes.data) == 0
    return nodes, tris, depth


def decode(n):
    s = np.ldexp(np.float32(1), n['e'].astype(np.int32)).astype(np.float32)
    lo = np.stack([n['o'][k] + n[f'ql{a}'].astype(np.float32) * s[k] for k, a in enumerate('xyz')], 1)
    hi = np.stack([n['o'][k] + n[f'qh{a}'].astype(np.float32) * s[k] for k, a in enumerate('xyz')], 1)
    return lo.astype(np.float32), hi.astype(np.float32)


@pytest.mark.parametrize("mesh", ["ico3", "tori", "dodeca"])
def test_bvh_layout_invariants(mesh):
    if mesh == "ico3":
        v, f = W.displaced_icosphere(3, 1)
    elif mesh == "tori":
        v, f = W.random_tori(2, n_tori=3, n_major=40, n_minor=10)
    else:
        v, f = W.dodecahedron()
    nodes, tris, depth = layout(cubvh.cuBVH(v, f))
    assert depth <= 13
    # the soup holds every face exactly once, with its own vertices
    assert np.array_equal(np.sort(tris['id']), np.arange(len(f)))
    tv = v[f[tris['id']]]
    assert np.array_equal(tris['a'], tv[:, 0]) and np.array_equal(tris['b'], tv[:, 1])
    assert np.array_equal(tris['c'], tv[:, 2])
    tlo = np.minimum(np.minimum(tris['a'], tris['b']), tris['c'])
    thi = np.maximum(np.maximum(tris['a'], tris['b']), tris['c'])

    def subtree_box(i):
        n = nodes[i]
        lo, hi = decode(n)
        blo, bhi = np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)
        for j in range(8):
            m = n['meta'][j]
            if m == 0xFF:
                continue
            if m & 0x80:
                clo, chi = subtree_box(n['cb'] + (m & 7))
            else:
                s0 = n['tb'] + (m & 31)
                s1 = s0 + ((m >> 5) & 3) + 1
                clo, chi = tlo[s0:s1].min(0), thi[s0:s1].max(0)
            assert (lo[j] <= clo).all() and (hi[j] >= chi).all(), "quantised child box does not contain its content"
            blo, bhi = np.minimum(blo, clo), np.maximum(bhi, chi)
        return blo, bhi

    lo, hi = subtree_box(0)
    assert np.array_equal(lo, tlo.min(0)) and np.array_equal(hi, thi.max(0))


def test_state_dict_reference_format():
    v, f = W.displaced_icosphere(3, 1)
    bvh = cubvh.cuBVH(v, f)
    sd = bvh.state_dict()
    nodes, tris = sd["nodes"], sd["triangles"]
    assert nodes.dtype == torch.int32 and nodes.shape[1] == 9
    assert tris.dtype == torch.int32 and tris.shape == (len(f), 12)
    N = nodes.numpy().view(REFNODE).reshape(-1)
    T = tris.numpy()
    xyz = T[:, :9].copy().view(np.float32).reshape(-1, 3, 3)
    ids = T[:, 10:12].copy().view(np.int64).reshape(-1)
    assert np.array_equal(np.sort(ids), np.arange(len(f)))
    assert np.array_equal(xyz, v[f[ids]])
    covered = np.zeros(len(f), int)
    order = []

    def walk(i, esc):
        order.append(i)
        n = N[i]
        assert n['escape'] == esc
        if n['left'] < 0:
            s0, s1 = -n['left'] - 1, -n['right'] - 1
            assert 0 < s1 - s0 <= 8 or len(f) <= 8
            covered[s0:s1] += 1
            box = xyz[s0:s1].reshape(-1, 3)
            assert (n['lo'] <= box.min(0)).all() and (n['hi'] >= box.max(0)).all()
            return
        assert n['right'] == n['left'] + 4          # exactly four children
        for c in range(n['left'], n['right']):
            walk(c, c + 1 if c + 1 < n['right'] else esc)

    walk(0, -1)
    assert (covered == 1).all() and len(order) == len(N)
    # deterministic: the reloaded BVH exports the same records
    sd2 = cubvh.cuBVH.from_state_dict(sd).state_dict()
    assert torch.equal(sd2["nodes"], nodes) and torch.equal(sd2["triangles"], tris)


def test_state_dict_version():
    v, f = W.icosphere(2)
    sd = cubvh.cuBVH(v, f).state_dict()
    assert sd["version"].dtype == torch.int32 and sd["version"].tolist() == [1]
    # the reloaded BVH returns the loaded records unchanged (as the reference's)
    back = cubvh.cuBVH.from_state_dict(sd).state_dict()
    assert all(torch.equal(back[k], sd[k]) for k in ("nodes", "triangles", "version"))
    # reference dicts carry no version and load the same
    ref = cubvh.cuBVH.from_state_dict({"nodes": sd["nodes"], "triangles": sd["triangles"]})
    assert torch.equal(ref.state_dict()["triangles"], sd["triangles"])
    assert cubvh.cuBVH.from_state_dict(dict(sd, version=1)).num_faces == len(f)
    for bad in (torch.tensor([2], dtype=torch.int32), 0, "1"):
        with pytest.raises(RuntimeError, match="version"):
            cubvh.cuBVH.from_state_dict(dict(sd, version=bad))
    with pytest.raises(RuntimeError, match="nodes"):
        cubvh.cuBVH.from_state_dict(dict(sd, nodes=sd["nodes"].float()))


def test_from_state_dict_ids_survive():
    v, f = W.icosphere(1)
    sd = cubvh.cuBVH(v, f).state_dict()
    _, tris, _ = layout(cubvh.cuBVH.from_state_dict(sd))
    assert np.array_equal(np.sort(tris['id']), np.arange(len(f)))


def test_errors_match_reference_surface():
    v, f = W.icosphere(0)
    with pytest.raises(AssertionError):
        cubvh.cuBVH(v, f[:8])                      # at least 9 faces
    bad = f.copy()
    bad[3, 1] = len(v)
    with pytest.raises(RuntimeError, match="vertex index"):
        cubvh.cuBVH(v, bad)
    vn = v.copy()
    vn[2, 0] = np.nan
    with pytest.raises(RuntimeError, match="finite"):
        cubvh.cuBVH(vn, f)
    with pytest.raises(RuntimeError):
        cubvh.cuBVH(v[:, :2], f)
    with pytest.raises(RuntimeError, match="triangles"):
        cubvh.cuBVH.from_state_dict({"nodes": torch.zeros(1, 9, dtype=torch.int32)})
    with pytest.raises(RuntimeError, match="nodes"):
        cubvh.cuBVH.from_state_dict({"triangles": torch.zeros(9, 12, dtype=torch.int32)})
    # torch inputs are detached and moved to the host, like the reference
    b = cubvh.cuBVH(torch.from_numpy(v).requires_grad_(), torch.from_numpy(f))
    assert b.num_faces == len(f)


def test_c_abi_argument_checks():
    L = _lib.lib()
    out = ctypes.c_void_p()
    assert L.cubvh_bvh_create(None, 3, None, 1, ctypes.byref(out)) == 1
    assert b"null" in L.cubvh_last_error()
    nb = ctypes.c_size_t()
    assert L.cubvh_floodfill_workspace_size(1, 2048, 2048, 1024, ctypes.byref(nb)) == 1
    assert L.cubvh_floodfill_workspace_size(1, 64, 64, 64, ctypes.byref(nb)) == 0
    small = nb.value
    assert L.cubvh_floodfill_workspace_size(2, 64, 64, 64, ctypes.byref(nb)) == 0 and nb.value > small
    v, f = W.icosphere(1)
    bvh = cubvh.cuBVH(v, f)
    assert L.cubvh_signed_distance(bvh.impl.raw, None, 5, 7, None, None, None, None) == 1
    assert b"mode" in L.cubvh_last_error()
    assert L.cubvh_unsigned_distance(bvh.impl.raw, None, 0, None, None, None, None) == 0   # empty: no-op


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(10.0 + rank * 5.0)
    q.put((rank, got))
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: 15.0, 1: 15.0}


def test_sparse_mc_abi_without_device_work():
    """Argument checks and the empty result of the sparse marching cubes
    entry points need no GPU: errors come back as status 1, an empty voxel
    set gives an empty result that fetches and frees without device work."""
    L = _lib.lib()
    res, nv, nt = ctypes.c_void_p(), ctypes.c_int64(7), ctypes.c_int64(7)
    assert L.cubvh_sparse_marching_cubes(None, None, 5, 0.0, 0, None, ctypes.byref(res), ctypes.byref(nv),
                                         ctypes.byref(nt)) == 1
    assert b"null" in L.cubvh_last_error() and not res.value and nv.value == 0 and nt.value == 0
    assert L.cubvh_sparse_marching_cubes(None, None, -1, 0.0, 0, None, ctypes.byref(res), ctypes.byref(nv),
                                         ctypes.byref(nt)) == 1
    assert b"negative" in L.cubvh_last_error()
    assert L.cubvh_sparse_marching_cubes(None, None, 0, 0.0, 0, None, None, ctypes.byref(nv), ctypes.byref(nt)) == 1
    assert L.cubvh_sparse_mc_fetch(None, None, None, None) == 1
    assert L.cubvh_sparse_mc_free(None) == 0
    assert L.cubvh_sparse_marching_cubes(None, None, 0, 0.0, 0, None, ctypes.byref(res), ctypes.byref(nv),
                                         ctypes.byref(nt)) == 0
    assert res.value and nv.value == 0 and nt.value == 0
    assert L.cubvh_sparse_mc_fetch(res, None, None, None) == 0
    assert L.cubvh_sparse_mc_free(res) == 0


LAYOUT_SHA256 = {
    # sha256 of the node and triangle arrays (cubvh_bvh_layout) of the host
    # build; the build splits large ranges across threads, and the tree must
    # not depend on how they are scheduled
    "ico6": "cbd9bfb9d61c2d311a3d0a082e9ebfd14603362bb27c64da15979a0af5d52596",
    "tori": "087878f061f19febd794558cfa5f6f961b4c98d0d7097a9c46862118821e646e",
    "ico3": "7f0e5649b0dcbb5ef1dc884eb1f0686ad9db985fb5076507bf35891cb406ead5",
}


@pytest.mark.parametrize("mesh", sorted(LAYOUT_SHA256))
def test_host_build_is_deterministic(mesh):
    import hashlib
    v, f = {"ico6": lambda: W.displaced_icosphere(6, 1), "tori": lambda: W.random_tori(2),
            "ico3": lambda: W.displaced_icosphere(3, 1)}[mesh]()
    for _ in range(2):
        nodes, tris, _ = layout(cubvh.cuBVH(v, f))
        assert hashlib.sha256(nodes.tobytes() + tris.tobytes()).hexdigest() == LAYOUT_SHA256[mesh]


def test_triangle_error_factors():
    """Each triangle record carries the FP32 distance filter's error factor
    K = max(1, 0.3 (1 + g) + 1e-7 g^2), g = |b-a| |c-a| / |(b-a) x (c-a)|,
    and K times its squared longest edge; zero-area triangles (a point, a
    segment, repeated vertices) carry K = 1e30."""
    v, f = W.random_tori(2, n_tori=2, n_major=40, n_minor=6)
    nv = len(v)
    extra = np.array([[0.2, 0.1, 0.85], [0.3, 0.1, 0.85], [0.4, 0.1, 0.85], [-0.3, -0.2, 0.9]], np.float32)
    v = np.concatenate([v, extra]).astype(np.float32)
    f = np.concatenate([f, [[nv, nv + 1, nv + 2], [nv + 3, nv + 3, nv + 3], [0, 0, 1]]]).astype(np.int64)
    _, tris, _ = layout(cubvh.cuBVH(v, f))
    a, b, c = (tris[k].astype(np.float64) for k in "abc")
    u, w = b - a, a - c
    nn = (np.cross(u, w) ** 2).sum(1)
    degenerate = nn < 1e-30
    assert degenerate.sum() == 3
    assert (tris["k"][degenerate] == np.float32(1e30)).all()
    g = np.sqrt((u * u).sum(1)[~degenerate] * (w * w).sum(1)[~degenerate] / nn[~degenerate])
    want = np.maximum(1.0, 0.3 * (1 + g) + 1e-7 * g * g)
    np.testing.assert_allclose(tris["k"][~degenerate], want, rtol=1e-6)
    assert 0.05 < (tris["k"] > 1).mean() < 0.95
    l2 = np.stack([(u * u).sum(1), ((c - b) ** 2).sum(1), (w * w).sum(1)]).max(0)
    np.testing.assert_allclose(tris["ke2"], tris["k"] * l2, rtol=1e-6)


def test_c_abi_rejects_bad_arguments_before_any_device_work():
    """Every entry point checks its arguments before it touches CUDA: on a
    host without a GPU, bad arguments come back as status 1 with a message,
    and empty work as status 0."""
    L = _lib.lib()
    P = ctypes.c_void_p
    out = P()
    v, f = W.icosphere(1)
    bvh = cubvh.cuBVH(v, f)
    h = bvh.impl.raw
    V = np.ascontiguousarray(v, np.float32)

    def bad(rc, needle=None):
        assert rc == 1
        msg = L.cubvh_last_error()
        assert msg
        if needle:
            assert needle.encode() in msg, msg

    bad(L.cubvh_bvh_create_device(None, 3, None, 1, 4, None, ctypes.byref(out)), "null")
    bad(L.cubvh_bvh_create_device(V.ctypes.data, 0, V.ctypes.data, 1, 4, None, ctypes.byref(out)), "empty")
    bad(L.cubvh_bvh_create_from_records(None, 5, ctypes.byref(out)), "null")
    bad(L.cubvh_bvh_create_from_records(V.ctypes.data, 0, ctypes.byref(out)), "no triangle records")
    bad(L.cubvh_bvh_info(None, None, None, None), "null")
    bad(L.cubvh_bvh_state_dict(h, None, None), "null")
    bad(L.cubvh_bvh_layout(h, None, None), "null")
    bad(L.cubvh_bvh_upload(None), "null")
    bad(L.cubvh_unsigned_distance(None, None, 5, None, None, None, None), "null")
    bad(L.cubvh_ray_trace(h, None, None, -1, None, None, None, None), "negative")
    assert L.cubvh_ray_trace(h, None, None, 0, None, None, None, None) == 0
    bad(L.cubvh_ray_trace(h, None, None, 4, None, None, None, None), "null")
    bad(L.cubvh_ray_trace_host(h, None, None, 4, None, None, None, None), "null")
    bad(L.cubvh_signed_distance_host(h, None, 4, 5, None, None, None, None), "mode")
    bad(L.cubvh_bvh_refit(h, None, len(V), None), "null")
    bad(L.cubvh_bvh_refit(h, V.ctypes.data, len(V) + 1, None), "vertex count")
    bad(L.cubvh_distance_backward(h, None, -2, None, None, None, None, None, None, None), "negative")
    assert L.cubvh_distance_backward(h, None, 0, None, None, None, None, None, None, None) == 0
    bad(L.cubvh_distance_backward(h, None, 3, None, None, None, None, None, None, None), "null")
    # NULL workspace = the no-allocation floodfill's array, which a 256^3 grid exceeds
    bad(L.cubvh_floodfill_check(None, 1, 256, 256, 256, None), "scratch")
    bad(L.cubvh_floodfill_check(None, -1, 4, 4, 4, None), "negative")
    bad(L.cubvh_udf_to_sdf(None, 1, 4, 4, 4, 0.01, None, None, 0, None), "null")
    assert L.cubvh_udf_to_sdf(None, 0, 4, 4, 4, 0.01, None, None, 0, None) == 0
    bad(L.cubvh_floodfill_noalloc(None, 1, 4, 4, 4, None, None), "null")
    bad(L.cubvh_floodfill(None, -1, 4, 4, 4, None, None, 0, None), "negative")

    # arena: built on the host; its query calls refuse to run before a layout
    F = np.ascontiguousarray(f, np.int64)
    vp = (ctypes.c_void_p * 1)(V.ctypes.data)
    fp = (ctypes.c_void_p * 1)(F.ctypes.data)
    nv = (ctypes.c_int64 * 1)(len(V))
    nf = (ctypes.c_int64 * 1)(len(F))
    bad(L.cubvh_arena_create_device(0, vp, nv, fp, nf, None, None, ctypes.byref(out)), "at least one mesh")
    a = P()
    assert L.cubvh_arena_create(1, vp, nv, fp, nf, None, ctypes.byref(a)) == 0
    try:
        bad(L.cubvh_arena_distance(a, None, None, None, None, None), "set_queries")
        bad(L.cubvh_arena_backward(a, None, None, None, None, None, None), "set_queries")
        bad(L.cubvh_arena_set_queries(a, None, None), "null")
        off = np.array([1, 5], np.int64)
        md = np.array([0], np.uint32)
        bad(L.cubvh_arena_set_queries(a, off.ctypes.data, md.ctypes.data), "query_offsets[0]")
        off = np.array([0, 5], np.int64)
        md = np.array([3], np.uint32)
        bad(L.cubvh_arena_set_queries(a, off.ctypes.data, md.ctypes.data), "mode")
    finally:
        assert L.cubvh_arena_destroy(a) == 0


def test_build_threads_env_same_tree():
    """CUBVH_B200_BUILD_THREADS caps the host build's threads (read once per
    process); the tree is the same for any count."""
    import subprocess
    import sys
    code = ("import sys, hashlib; sys.path.insert(0, 'tests')\n"
            "import cubvh_b200 as cubvh\n"
            "from cubvh_b200 import workloads as W\n"
            "from test_host import layout\n"
            "n, t, _ = layout(cubvh.cuBVH(*W.displaced_icosphere(6, 1)))\n"
            "print(hashlib.sha256(n.tobytes() + t.tobytes()).hexdigest())\n")
    for threads in ("1", "2"):
        env = dict(os.environ, CUBVH_B200_BUILD_THREADS=threads)
        r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        assert r.stdout.strip().splitlines()[-1] == LAYOUT_SHA256["ico6"]


def _signed_zero_sheet():
    """A flat 60 x 60 sheet in z = 0 with -0.0 mixed into the coordinates
    (ties and signed zeros in the reference-format sort and boxes)."""
    g = np.stack(np.meshgrid(np.arange(60), np.arange(60), indexing="ij"), -1).reshape(-1, 2)
    v = np.concatenate([g * 0.01, np.zeros((len(g), 1))], 1).astype(np.float32)
    v[::3, 2] = -0.0
    v[::7, 0] = -0.0 * v[::7, 0]
    i = np.nonzero((g[:, 0] < 59) & (g[:, 1] < 59))[0]
    return v, np.concatenate([np.stack([i, i + 60, i + 1], 1), np.stack([i + 1, i + 60, i + 61], 1)])


STATE_DICT_SHA256 = {
    # sha256 of the nodes and triangles records state_dict returns: the
    # records of the reference's own build of the mesh (tests/test_ref_bvh.py
    # compares them with that build when it is compiled)
    "ico6": "c5b808b0440a125cba10bf420ef95edcb34b5ccfe1e361174777a008a3f07370",
    "tori": "5398185421d1f1c871f012593428baa9b6517f7c4a139f5b3aea837bbe4ef8d3",
    "sheet": "8661958b7122c397f8412af019b4dd713296a0da201c97afcabcced720c3fa61",
}


@pytest.mark.parametrize("mesh", sorted(STATE_DICT_SHA256))
def test_state_dict_records_pinned(mesh):
    import hashlib
    v, f = {"ico6": lambda: W.displaced_icosphere(6, 1), "tori": lambda: W.random_tori(2),
            "sheet": _signed_zero_sheet}[mesh]()
    sd = cubvh.cuBVH(v, f).state_dict()
    digest = hashlib.sha256(sd["nodes"].numpy().tobytes() + sd["triangles"].numpy().tobytes()).hexdigest()
    assert digest == STATE_DICT_SHA256[mesh]


def test_state_dict_sizes_for_many_face_counts():
    """The node-record count state_dict reports (computed from the face count
    alone) is the one its records have, for small and uneven counts."""
    rng = np.random.default_rng(7)
    for nf in list(range(9, 80)) + [255, 256, 257, 1023, 4097, 30011]:
        v = rng.random((nf * 3, 3)).astype(np.float32)
        f = np.arange(nf * 3, dtype=np.int64).reshape(-1, 3)
        sd = cubvh.cuBVH(v, f).state_dict()
        nodes, tris = sd["nodes"], sd["triangles"]
        assert tris.shape == (nf, 12) and nodes.shape[1] == 9
        # every node's child links point inside the array; leaves cover all faces once
        recs = nodes.numpy().view(REFNODE).reshape(-1)
        inner = recs["left"] >= 0
        assert np.all(recs["right"][inner] <= len(recs))
        leaf_ranges = sorted((-l - 1, -r - 1) for l, r in zip(recs["left"][~inner], recs["right"][~inner]))
        assert leaf_ranges[0][0] == 0 and leaf_ranges[-1][1] == nf
        assert all(a[1] == b[0] for a, b in zip(leaf_ranges, leaf_ranges[1:]))


def test_bench_reference_arm_contract():
    """`bench.py --impl reference` (the reference's host traversals timed on
    the CPU) prints one JSON line with the contract's keys, on a tiny
    rays_displaced workload."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--res", "32",
                          "--sdf-points", "2048", "--steps", "1", "--warmup", "3"],
                         cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "queries/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "rays_displaced"


def test_incoherent_rays_workload():
    """The incoherent-ray generator behind bench.py's rays_incoherent
    workload: float32 unit directions; the first half start in [-1, 1]^3, the
    second half on the radius-3 sphere, pointing into [-0.8, 0.8]^3."""
    o, d = W.incoherent_rays(1001, seed=3)
    assert o.shape == d.shape == (1001, 3) and o.dtype == d.dtype == np.float32
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, rtol=1e-6)
    h = 1001 // 2
    assert (np.abs(o[:h]) <= 1).all()
    np.testing.assert_allclose(np.linalg.norm(o[h:], axis=1), 3.0, rtol=1e-6)
    # the second half's rays pass through a point of the inner box, so they
    # come within its half-diagonal 0.8 sqrt(3) of the centre
    oo, dd = o[h:].astype(np.float64), d[h:].astype(np.float64)
    closest = oo - dd * (oo * dd).sum(1, keepdims=True)
    assert (np.linalg.norm(closest, axis=1) <= 0.8 * np.sqrt(3) + 1e-5).all()
    o2, d2 = W.incoherent_rays(1001, seed=3)
    assert np.array_equal(o, o2) and np.array_equal(d, d2)
