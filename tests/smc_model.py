"""A plain-Python statement of the sparse-marching-cubes triangulation in
cubvh_b200/csrc/sparse_mc.cu (face walks, saddle-decided four-cut faces,
fans from an apex whose diagonals stay off faces crossed twice by a loop, ear
clipping otherwise), used by the tests to check the rules on the CPU and the
kernels against them.  Vertex ids come from oracle.sparse_mc_vertices."""

import numpy as np

EDGE_CORNERS = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
FACE_CORNERS = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
FACE_EDGES = [(3, 2, 1, 0), (4, 5, 6, 7), (0, 9, 4, 8), (11, 6, 10, 2), (8, 7, 11, 3), (1, 10, 5, 9)]


def _f32(x):
    return np.float32(x)


def saddle_inside(a, b, c, d, iso):
    num = _f32(_f32(a * c) - _f32(b * d))
    den = _f32(_f32(a + c) - _f32(b + d))
    lim = _f32(iso * den)
    if den > 0:
        return num < lim
    if den < 0:
        return num > lim
    return False


def links(v, iso):
    inside = [v[k] < iso for k in range(8)]
    cut = [inside[a] != inside[b] for a, b in EDGE_CORNERS]
    nxt = {}
    for f in range(6):
        fin = [inside[c] for c in FACE_CORNERS[f]]
        cr = sum(fin[i] != fin[(i + 1) % 4] for i in range(4))
        if cr == 0:
            continue
        join = cr == 4 and saddle_inside(*[v[c] for c in FACE_CORNERS[f]], iso)
        for i in range(4):
            ip = (i + 3) % 4
            eb, ea = FACE_EDGES[f][ip], FACE_EDGES[f][i]
            if cr == 2:
                if fin[i] and not fin[ip]:
                    j = i
                    while fin[(j + 1) % 4]:
                        j = (j + 1) % 4
                    nxt[eb] = FACE_EDGES[f][j]
            elif join:
                if not fin[i]:
                    nxt[ea] = eb
            elif fin[i]:
                nxt[eb] = ea
    return cut, nxt


def triangles(v, iso):
    """Triangles of one voxel as triples of edge numbers, in kernel order."""
    v = [np.float32(x) for x in v]
    iso = np.float32(iso)
    cut, nxt = links(v, iso)
    loops, loop_of, left = [], {}, [e for e in range(12) if cut[e]]
    while left:
        s = left[0]
        loop, e = [], s
        while True:
            loop.append(e)
            loop_of[e] = len(loops)
            left.remove(e)
            e = nxt[e]
            if e == s:
                break
        loops.append(loop)
    mark = {e: 0 for e in range(12)}
    for f in range(6):
        es = FACE_EDGES[f]
        if all(cut[e] for e in es) and len({loop_of[e] for e in es}) == 1:
            for e in es:
                mark[e] |= 1 << f
    out = []
    for q in loops:
        L = len(q)
        apex = None
        for k in range(L):
            if all(not (mark[q[k]] & mark[q[j]]) for j in range(L) if (j - k) % L not in (0, 1, L - 1)):
                apex = k
                break
        if apex is not None:
            for m in range(1, L - 1):
                out.append((q[apex], q[(apex + m) % L], q[(apex + m + 1) % L]))
        else:
            ring = list(q)
            while len(ring) >= 3:
                r = len(ring)
                ear = 1
                for m in range(r):
                    if r == 3 or not (mark[ring[(m - 1) % r]] & mark[ring[(m + 1) % r]]):
                        ear = m
                        break
                out.append((ring[(ear - 1) % r], ring[ear], ring[(ear + 1) % r]))
                ring.pop(ear)
    return out


def mesh_triangles(coords, corners, iso, vi, ei, ids):
    """Triangle array (merged vertex ids) of a voxel set, voxel by voxel."""
    idmap = {(int(a), int(b)): int(c) for a, b, c in zip(vi, ei, ids)}
    out = []
    for i in range(len(coords)):
        for t in triangles(corners[i], iso):
            out.append([idmap[(i, e)] for e in t])
    return np.array(out, np.int32).reshape(-1, 3)
