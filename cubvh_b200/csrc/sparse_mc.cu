// Sparse marching cubes: a triangle mesh of the iso-surface of per-voxel
// corner values over a sparse set of voxels.
//
// Reference: include/gpu/spcumc.cuh (`_sparse_marching_cubes`), entry
// cubvh/api.py:173-187.  Kept alike because they are the interface or decide
// the vertex array: the corner order of the [N, 8] input (offsets (0,0,0),
// (1,0,0), (1,1,0), (0,1,0), then the same at z + 1), the edge numbering
// (bottom square, top square, verticals), a corner is inside when its value
// is below iso, a vertex on every edge with one corner inside at
// t = clamp((iso - va) / (vb - va), 0, 1) (0.5 when |vb - va| < 1e-30) from
// the edge's first corner, vertices shared by voxels merged by their edge key
// (lower corner, axis) with the copy of the lowest voxel kept and the array
// sorted by key, and triangles listed voxel by voxel.  The optional corner
// averaging replaces every corner value by the mean over the voxels sharing
// that corner.
//
// Triangulation.  By default the reference's: each voxel's triangles come
// from the marching-cubes case table of its corner configuration (mc_cases.h,
// recovered from the reference's own outputs for the 256 configurations:
// tests/golden/make_ref_mc_cases.py), table triangle (e0, e1, e2) written as
// vertices (e0, e2, e1), voxel by voxel, so the triangle array equals the
// reference's index for index.  The table is the public marching-cubes case
// table; its configurations with faces cut four times (the ambiguous cases)
// are triangulated without looking at the face's saddle, so neighbouring
// cubes can disagree and leave holes there.
//
// Optionally (flag kSmcClosed) this file's own triangulation, no lookup
// table: on each cube face, walk its corners counter-clockwise as seen from
// outside the cube; a segment of the surface joins an edge where the walk
// enters the inside region to the next edge where it leaves it.  A face with
// four cut edges (inside corners on a diagonal) is resolved by the sign of
// its bilinear saddle (Nielson and Hamann's asymptotic decider): the two
// inside corners are joined through the face when the saddle value is below
// iso.  Both cubes sharing a face take the same decision, so the surface is
// closed wherever the corner values agree.  Every cut edge is entered on one
// of its faces and left on the other, so the segments form closed loops.
// Each loop, started at its lowest edge, is cut into a triangle fan from the
// first vertex none of whose diagonals joins two edges of one face that the
// loop crosses twice (such a diagonal would lie in that face and be shared
// with the neighbouring cube's triangles); when no vertex qualifies, ears
// whose closing diagonal avoids such faces are clipped one by one.
// Triangles face from the inside (values below iso) to the outside.  A cube
// with one corner inside gives the same triangle as the table.
#include <cstddef>
#include <cstdint>
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include <vector>

#include "launches.h"
#include "kernels.h"
#include "mc_cases.h"
#include "scan.cuh"

namespace cubvh {
namespace {

__constant__ int8_t c_corner_off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                          {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int8_t c_edge_corners[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                             {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
// Faces: corners counter-clockwise seen from outside the cube, and the edge
// from corner i to corner i + 1 of that cycle.
__constant__ int8_t c_face_corners[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                            {3, 7, 6, 2}, {0, 4, 7, 3}, {1, 2, 6, 5}};
__constant__ int8_t c_face_edges[6][4] = {{3, 2, 1, 0}, {4, 5, 6, 7}, {0, 9, 4, 8},
                                          {11, 6, 10, 2}, {8, 7, 11, 3}, {1, 10, 5, 9}};

struct Cube {
    float v[8];
    uint32_t inside;  // bit c: corner c below iso
    uint32_t cut;     // bit e: edge e has one corner inside
};

__device__ __forceinline__ Cube load_cube(const float* __restrict__ corners, int64_t i, float iso) {
    Cube c;
    c.inside = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        c.v[k] = corners[8 * i + k];
        if (c.v[k] < iso) c.inside |= 1u << k;
    }
    c.cut = 0;
#pragma unroll
    for (int e = 0; e < 12; ++e)
        if (((c.inside >> c_edge_corners[e][0]) ^ (c.inside >> c_edge_corners[e][1])) & 1u) c.cut |= 1u << e;
    return c;
}

// True when the bilinear interpolant of a face with inside corners on one
// diagonal has its saddle below iso (the inside corners are joined across
// the face).  a, c and b, d are the two diagonals in cycle order.  Rounded
// operations only (no contraction): swapping the diagonals negates numerator
// and denominator exactly, so the two cubes sharing the face agree.
__device__ __forceinline__ bool saddle_inside(float a, float b, float c, float d, float iso) {
    const float num = __fsub_rn(__fmul_rn(a, c), __fmul_rn(b, d));
    const float den = __fsub_rn(__fadd_rn(a, c), __fadd_rn(b, d));
    const float lim = __fmul_rn(iso, den);
    if (den > 0.f) return num < lim;
    if (den < 0.f) return num > lim;
    return false;  // flat saddle: keep the inside corners apart
}

// nxt[e] for every cut edge e: the edge the surface loop goes to after e.
__device__ __forceinline__ void surface_links(const Cube& c, float iso, int8_t nxt[12]) {
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        bool in[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) in[i] = (c.inside >> c_face_corners[f][i]) & 1u;
        int crossings = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) crossings += in[i] != in[(i + 1) & 3];
        if (crossings == 0) continue;
        bool join_inside = false;  // four crossings: are the inside corners joined?
        if (crossings == 4)
            join_inside = saddle_inside(c.v[c_face_corners[f][0]], c.v[c_face_corners[f][1]],
                                        c.v[c_face_corners[f][2]], c.v[c_face_corners[f][3]], iso);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int ip = (i + 3) & 3;  // previous corner in the cycle
            const int e_before = c_face_edges[f][ip], e_after = c_face_edges[f][i];
            if (crossings == 2) {
                // the inside run starts at the corner after the in-edge
                if (in[i] && !in[ip]) {
                    int j = i;
                    while (in[(j + 1) & 3]) j = (j + 1) & 3;
                    nxt[e_before] = c_face_edges[f][j];
                }
            } else if (join_inside) {
                // segments around the outside corners: in-edge after it -> out-edge before it
                if (!in[i]) nxt[e_after] = e_before;
            } else {
                // segments around the inside corners: in-edge before it -> out-edge after it
                if (in[i]) nxt[e_before] = e_after;
            }
        }
    }
}

__device__ __forceinline__ int n_triangles(const Cube& c, float iso) {
    if (!c.cut) return 0;
    int8_t nxt[12];
    surface_links(c, iso, nxt);
    uint32_t left = c.cut;
    int loops = 0;
    // nxt is a permutation of the cut edges (each is entered on one of its
    // faces and left on the other): the walks close; 12 steps bound them all
    int steps = 0;
    while (left && steps < 12) {
        const int s = __ffs(left) - 1;
        int e = s;
        do { left &= ~(1u << e); e = nxt[e]; ++steps; } while (e != s && steps < 12);
        ++loops;
    }
    return __popc(c.cut) - 2 * loops;
}

// triangles of a corner configuration in the case table
__device__ __forceinline__ int n_table_triangles(uint32_t inside) {
    int t = 0;
    while (t < 5 && c_mc_tri[inside][3 * t] >= 0) ++t;
    return t;
}

__global__ void k_smc_count(int64_t n, const float* __restrict__ corners, float iso, bool table,
                            uint32_t* __restrict__ nv, uint32_t* __restrict__ nt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Cube c = load_cube(corners, i, iso);
        nv[i] = __popc(c.cut);
        nt[i] = (uint32_t)(table ? n_table_triangles(c.inside) : n_triangles(c, iso));
    }
}

struct KeyPack {
    int32_t minx, miny, minz;
    uint64_t ry, rz;  // extents (in corners) along y and z
};
__device__ __forceinline__ uint64_t pack_point(int x, int y, int z, const KeyPack& k) {
    return ((uint64_t)(uint32_t)(x - k.minx) * k.ry + (uint64_t)(uint32_t)(y - k.miny)) * k.rz +
           (uint64_t)(uint32_t)(z - k.minz);
}

// Vertices (position, edge key) in edge order and triangles (indices into
// this launch's vertex list, before merging) of every voxel.
__global__ void k_smc_emit(int64_t n, const int32_t* __restrict__ coords, const float* __restrict__ corners,
                           float iso, bool table, const uint32_t* __restrict__ vpre, const uint32_t* __restrict__ tpre,
                           KeyPack kp, float* __restrict__ pos, uint64_t* __restrict__ key,
                           int32_t* __restrict__ tri) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Cube c = load_cube(corners, i, iso);
        if (!c.cut) continue;
        const int x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
        const uint32_t vb = vpre[i];
        uint32_t k = vb;
        for (int e = 0; e < 12; ++e) {
            if (!((c.cut >> e) & 1u)) continue;
            const int a = c_edge_corners[e][0], b = c_edge_corners[e][1];
            const float va = c.v[a], vv = c.v[b];
            const float den = __fsub_rn(vv, va);
            float t;
            if (fabsf(den) < 1e-30f) {
                t = 0.5f;
            } else {
                t = __fdiv_rn(__fsub_rn(iso, va), den);
                t = fminf(fmaxf(t, 0.f), 1.f);
            }
            const int ax = x + c_corner_off[a][0], ay = y + c_corner_off[a][1], az = z + c_corner_off[a][2];
            const int bx = x + c_corner_off[b][0], by = y + c_corner_off[b][1], bz = z + c_corner_off[b][2];
            pos[3 * k] = __fmaf_rn(t, __fsub_rn((float)bx, (float)ax), (float)ax);
            pos[3 * k + 1] = __fmaf_rn(t, __fsub_rn((float)by, (float)ay), (float)ay);
            pos[3 * k + 2] = __fmaf_rn(t, __fsub_rn((float)bz, (float)az), (float)az);
            const int axis = ax != bx ? 0 : (ay != by ? 1 : 2);
            key[k] = pack_point(min(ax, bx), min(ay, by), min(az, bz), kp) * 3u + (uint64_t)axis;
            ++k;
        }
        uint32_t t_out = tpre[i];
        const uint32_t t_end = tpre[i + 1];  // the count pass's triangles: never write past them
        auto vid = [&](int e) { return (int32_t)(vb + __popc(c.cut & ((1u << e) - 1u))); };
        if (table) {
            // the case table's triangles, written (e0, e2, e1) as the reference does
            for (int t = 0; t < 5 && t_out < t_end; ++t) {
                const int e0 = c_mc_tri[c.inside][3 * t];
                if (e0 < 0) break;
                tri[3 * t_out] = vid(e0);
                tri[3 * t_out + 1] = vid(c_mc_tri[c.inside][3 * t + 2]);
                tri[3 * t_out + 2] = vid(c_mc_tri[c.inside][3 * t + 1]);
                ++t_out;
            }
            continue;
        }
        int8_t nxt[12];
        surface_links(c, iso, nxt);
        // loops, in order of their lowest edge
        int8_t loop_of[12];
        int8_t seq[12];
        int8_t start[7];
        int nl = 0, len = 0;
        {
            uint32_t left = c.cut;
            while (left && nl < 6 && len < 12) {
                const int s0 = __ffs(left) - 1;
                start[nl] = (int8_t)len;
                int e = s0;
                do { left &= ~(1u << e); loop_of[e] = (int8_t)nl; seq[len++] = (int8_t)e; e = nxt[e]; }
                while (e != s0 && len < 12);
                ++nl;
            }
            start[nl] = (int8_t)len;
        }
        // mark[e]: faces with four cut edges whose two segments both lie in e's
        // loop; two such vertices not joined by a segment must not be joined by
        // a diagonal either (it would lie in the face, and the neighbouring cube
        // could use it too)
        uint8_t mark[12];
#pragma unroll
        for (int e = 0; e < 12; ++e) mark[e] = 0;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const int e0 = c_face_edges[f][0], e1 = c_face_edges[f][1], e2 = c_face_edges[f][2],
                      e3 = c_face_edges[f][3];
            if (((c.cut >> e0) & (c.cut >> e1) & (c.cut >> e2) & (c.cut >> e3) & 1u) &&
                loop_of[e0] == loop_of[e1] && loop_of[e1] == loop_of[e2] && loop_of[e2] == loop_of[e3]) {
                mark[e0] |= 1u << f; mark[e1] |= 1u << f; mark[e2] |= 1u << f; mark[e3] |= 1u << f;
            }
        }
        for (int l = 0; l < nl && t_out < t_end; ++l) {
            const int b0 = start[l], L = start[l + 1] - start[l];
            int8_t* q = seq + b0;
            // fan apex: the first vertex none of whose diagonals joins two
            // vertices of one marked face
            int apex = -1;
            for (int k = 0; k < L && apex < 0; ++k) {
                bool ok = true;
                for (int j = 0; j < L && ok; ++j) {
                    const int dj = (j - k + L) % L;
                    if (dj <= 1 || dj == L - 1) continue;
                    if (mark[q[k]] & mark[q[j]]) ok = false;
                }
                if (ok) apex = k;
            }
            if (apex >= 0) {
                for (int m = 1; m + 1 < L && t_out < t_end; ++m) {
                    tri[3 * t_out] = vid(q[apex]);
                    tri[3 * t_out + 1] = vid(q[(apex + m) % L]);
                    tri[3 * t_out + 2] = vid(q[(apex + m + 1) % L]);
                    ++t_out;
                }
            } else {
                // ear clipping: cut the first ear whose new edge is allowed (any
                // ear if none is), keeping the loop's orientation
                int8_t ring[12];
                for (int m = 0; m < L; ++m) ring[m] = q[m];
                int r = L;
                while (r >= 3 && t_out < t_end) {
                    int ear = 1;
                    for (int m = 0; m < r; ++m) {
                        const int a0 = ring[(m + r - 1) % r], a2 = ring[(m + 1) % r];
                        if (r == 3 || !(mark[a0] & mark[a2])) { ear = m; break; }
                    }
                    tri[3 * t_out] = vid(ring[(ear + r - 1) % r]);
                    tri[3 * t_out + 1] = vid(ring[ear]);
                    tri[3 * t_out + 2] = vid(ring[(ear + 1) % r]);
                    ++t_out;
                    for (int m = ear; m + 1 < r; ++m) ring[m] = ring[m + 1];
                    --r;
                }
            }
        }
    }
}

__global__ void k_smc_iota(int64_t m, int32_t* __restrict__ a) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = (int32_t)i;
}

// sorted keys: head[i] = first of its run; unique id = inclusive scan - 1
__global__ void k_smc_heads(int64_t m, const uint64_t* __restrict__ key, uint32_t* __restrict__ head) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}
// ids: exclusive scan of heads; the run's first (lowest emission index, the
// sort being stable) supplies the merged vertex's position
__global__ void k_smc_merge(int64_t m, const uint32_t* __restrict__ head, const uint32_t* __restrict__ ids,
                            const int32_t* __restrict__ order, const float* __restrict__ pos,
                            int32_t* __restrict__ map, float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t id = (int32_t)(ids[i] + head[i]) - 1;
        const int32_t src = order[i];
        map[src] = id;
        if (head[i]) {
            out[3 * id] = pos[3 * src];
            out[3 * id + 1] = pos[3 * src + 1];
            out[3 * id + 2] = pos[3 * src + 2];
        }
    }
}
__global__ void k_smc_remap(int64_t n3, const int32_t* __restrict__ map, int32_t* __restrict__ tri) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x)
        tri[i] = map[tri[i]];
}

// corner averaging: keys of the 8 corners of every voxel
__global__ void k_smc_corner_keys(int64_t n, const int32_t* __restrict__ coords, KeyPack kp,
                                  uint64_t* __restrict__ key, int32_t* __restrict__ idx) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < 8 * n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = j >> 3;
        const int c = (int)(j & 7);
        key[j] = pack_point(coords[3 * i] + c_corner_off[c][0], coords[3 * i + 1] + c_corner_off[c][1],
                            coords[3 * i + 2] + c_corner_off[c][2], kp);
        idx[j] = (int32_t)j;
    }
}
// one thread per run of equal corner keys: the mean of the run's values, in
// run order (voxel order), written back to every member
__global__ void k_smc_corner_mean(int64_t m, const uint64_t* __restrict__ key, const int32_t* __restrict__ idx,
                                  const float* __restrict__ in, float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && key[i] == key[i - 1]) continue;
        float sum = 0.f;
        int cnt = 0;
        int64_t j = i;
        do { sum = __fadd_rn(sum, in[idx[j]]); ++cnt; ++j; } while (j < m && key[j] == key[i]);
        const float mean = __fdiv_rn(sum, (float)cnt);
        for (int64_t q = i; q < j; ++q) out[idx[q]] = mean;
    }
}

__global__ void k_smc_bounds(int64_t n, const int32_t* __restrict__ coords, int32_t* __restrict__ b) {
    int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { lo[k] = min(lo[k], coords[3 * i + k]); hi[k] = max(hi[k], coords[3 * i + k]); }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = __reduce_min_sync(0xFFFFFFFFu, lo[k]);
        hi[k] = __reduce_max_sync(0xFFFFFFFFu, hi[k]);
    }
    // warps meet in shared memory, then one atomic per block and bound (the
    // six global words are the only addresses every block updates)
    __shared__ int32_t sb[6];
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? INT32_MAX : INT32_MIN;
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) { atomicMin(&sb[k], lo[k]); atomicMax(&sb[3 + k], hi[k]); }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&b[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&b[threadIdx.x], sb[threadIdx.x]);
}
__global__ void k_smc_bounds_init(int32_t* b) {
    if (threadIdx.x < 3) b[threadIdx.x] = INT32_MAX;
    else if (threadIdx.x < 6) b[threadIdx.x] = INT32_MIN;
}

unsigned grid_for(int64_t n) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (n + 255) / 256;
    const int64_t cap = (int64_t)nsm * 16;
    return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

int bits_for(uint64_t v) {  // bits to hold values below v
    int b = 0;
    while (b < 64 && (uint64_t(1) << b) < v) ++b;
    return b;
}

template <class T>
cudaError_t pool_get(cudaMemPool_t pool, cudaStream_t s, T** out, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16, pool, s);
    if (e == cudaSuccess) *out = static_cast<T*>(q);
    return e;
}

// Stream-ordered temporaries of one call: every buffer taken from `get` is
// returned with cudaFreeAsync on the same stream, early through `put` or at
// scope exit, so an error return in the middle of the pipeline leaks nothing.
struct AsyncTemps {
    cudaMemPool_t pool;
    cudaStream_t s;
    std::vector<void*> p;
    AsyncTemps(cudaMemPool_t pl, cudaStream_t st) : pool(pl), s(st) {}
    AsyncTemps(const AsyncTemps&) = delete;
    AsyncTemps& operator=(const AsyncTemps&) = delete;
    ~AsyncTemps() { for (void* q : p) cudaFreeAsync(q, s); }
    template <class T>
    cudaError_t get(T** out, size_t count) {
        const cudaError_t e = pool_get(pool, s, out, count);
        if (e == cudaSuccess) p.push_back(*out);
        return e;
    }
    void put(void* q) {
        for (size_t i = 0; i < p.size(); ++i)
            if (p[i] == q) { cudaFreeAsync(q, s); p.erase(p.begin() + (std::ptrdiff_t)i); return; }
    }
};

}  // namespace

// Temporaries and results come from the library's pool on `stream`; the
// results stay in `out` (owned by the caller through cubvh_sparse_mc_*,
// which releases them on an error return as well).
int sparse_mc_run(const int32_t* coords, const float* corners, int64_t n, float iso, bool ensure_consistency,
                  bool closed, cudaStream_t s, SparseMCResult& out, std::string& err) {
    out = SparseMCResult{};
    if (n <= 0) return 0;
    if (n > (int64_t)INT32_MAX / 12) { err = "too many voxels (the vertex count must fit in int32)"; return 1; }
    cudaError_t e;
    auto fail = [&](cudaError_t x, const char* what) { err = std::string(what) + ": " + cudaGetErrorString(x); return 2; };
    cudaMemPool_t pool = nullptr;
    if ((e = library_pool(&pool)) != cudaSuccess) return fail(e, "memory pool");
    AsyncTemps tmp(pool, s);
    // coordinate bounds -> key packing (host round trip)
    int32_t* d_b = nullptr;
    if ((e = tmp.get(&d_b, 6)) != cudaSuccess) return fail(e, "pool allocation");
    k_smc_bounds_init<<<1, 32, 0, s>>>(d_b); count_launch();
    k_smc_bounds<<<grid_for(n), 256, 0, s>>>(n, coords, d_b); count_launch();
    int32_t b[6];
    if ((e = cudaMemcpyAsync(b, d_b, sizeof(b), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(e, "sparse marching cubes bounds");
    tmp.put(d_b);
    const uint64_t rx = (uint64_t)((int64_t)b[3] - b[0] + 2), ry = (uint64_t)((int64_t)b[4] - b[1] + 2),
                   rz = (uint64_t)((int64_t)b[5] - b[2] + 2);
    const int key_bits = bits_for(rx) + bits_for(ry) + bits_for(rz) + 2;
    if (key_bits > 64) { err = "voxel coordinate range too large for 64-bit edge keys"; return 1; }
    const KeyPack kp{b[0], b[1], b[2], ry, rz};
    const unsigned g = grid_for(n);

    const float* use = corners;
    if (ensure_consistency) {
        const int64_t m8 = 8 * n;
        float* avg = nullptr;
        uint64_t *ck = nullptr, *ck2 = nullptr;
        int32_t *ci = nullptr, *ci2 = nullptr;
        const int cbits = bits_for(rx) + bits_for(ry) + bits_for(rz);
        if ((e = tmp.get(&avg, m8)) != cudaSuccess || (e = tmp.get(&ck, m8)) != cudaSuccess ||
            (e = tmp.get(&ck2, m8)) != cudaSuccess || (e = tmp.get(&ci, m8)) != cudaSuccess ||
            (e = tmp.get(&ci2, m8)) != cudaSuccess)
            return fail(e, "pool allocation");
        k_smc_corner_keys<<<grid_for(m8), 256, 0, s>>>(n, coords, kp, ck, ci); count_launch();
        size_t tb = 0;
        char* cub_tmp = nullptr;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, ck, ck2, ci, ci2, (int)m8, 0, cbits, s);
        if ((e = tmp.get(&cub_tmp, tb)) != cudaSuccess) return fail(e, "pool allocation");
        if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, tb, ck, ck2, ci, ci2, (int)m8, 0, cbits, s)) != cudaSuccess)
            return fail(e, "corner sort");
        count_launch();
        tmp.put(cub_tmp);
        k_smc_corner_mean<<<grid_for(m8), 256, 0, s>>>(m8, ck2, ci2, corners, avg); count_launch();
        tmp.put(ck); tmp.put(ck2); tmp.put(ci); tmp.put(ci2);
        use = avg;  // freed at scope exit, after the kernels that read it
    }

    uint32_t *nv = nullptr, *nt = nullptr, *bs = nullptr;
    const int64_t nb = scan::num_chunks(n) + 1;
    if ((e = tmp.get(&nv, n + 1)) != cudaSuccess || (e = tmp.get(&nt, n + 1)) != cudaSuccess ||
        (e = tmp.get(&bs, nb)) != cudaSuccess)
        return fail(e, "pool allocation");
    k_smc_count<<<g, 256, 0, s>>>(n, use, iso, !closed, nv, nt); count_launch();
    scan::exclusive(nv, bs, n, s);   // nv[n] = total
    scan::exclusive(nt, bs, n, s);
    uint32_t tot[2];
    if ((e = cudaMemcpyAsync(&tot[0], nv + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[1], nt + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(e, "sparse marching cubes counts");
    const int64_t m = tot[0], t = tot[1];
    float* pos = nullptr;
    uint64_t *key = nullptr, *key2 = nullptr;
    int32_t *ord = nullptr, *ord2 = nullptr, *map = nullptr;
    uint32_t *head = nullptr, *ids = nullptr, *bs2 = nullptr;
    if (m > 0) {
        const int64_t nb2 = scan::num_chunks(m) + 1;
        if ((e = tmp.get(&pos, 3 * m)) != cudaSuccess || (e = tmp.get(&key, m)) != cudaSuccess ||
            (e = tmp.get(&key2, m)) != cudaSuccess || (e = tmp.get(&ord, m)) != cudaSuccess ||
            (e = tmp.get(&ord2, m)) != cudaSuccess || (e = tmp.get(&map, m)) != cudaSuccess ||
            (e = tmp.get(&head, m + 1)) != cudaSuccess || (e = tmp.get(&ids, m + 1)) != cudaSuccess ||
            (e = tmp.get(&bs2, nb2)) != cudaSuccess ||
            (e = pool_get(pool, s, &out.tris, (size_t)(3 * t))) != cudaSuccess)
            return fail(e, "sparse marching cubes buffers");
        k_smc_emit<<<g, 256, 0, s>>>(n, coords, use, iso, !closed, nv, nt, kp, pos, key, out.tris); count_launch();
        // emission index as the value: the stable sort keeps each key's lowest first
        k_smc_iota<<<grid_for(m), 256, 0, s>>>(m, ord); count_launch();
        size_t tb = 0;
        char* cub_tmp = nullptr;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, ord, ord2, (int)m, 0, key_bits, s);
        if ((e = tmp.get(&cub_tmp, tb)) != cudaSuccess) return fail(e, "pool allocation");
        if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, tb, key, key2, ord, ord2, (int)m, 0, key_bits, s)) !=
            cudaSuccess)
            return fail(e, "edge key sort");
        count_launch();
        k_smc_heads<<<grid_for(m), 256, 0, s>>>(m, key2, head); count_launch();
        if ((e = cudaMemcpyAsync(ids, head, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
            return fail(e, "cudaMemcpyAsync");
        scan::exclusive(ids, bs2, m, s);  // ids[m] = merged vertex count
        uint32_t u = 0;
        if ((e = cudaMemcpyAsync(&u, ids + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return fail(e, "sparse marching cubes merge");
        if ((e = pool_get(pool, s, &out.verts, (size_t)3 * u)) != cudaSuccess)
            return fail(e, "vertex buffer");
        k_smc_merge<<<grid_for(m), 256, 0, s>>>(m, head, ids, ord2, pos, map, out.verts); count_launch();
        if (t > 0) { k_smc_remap<<<grid_for(3 * t), 256, 0, s>>>(3 * t, map, out.tris); count_launch(); }
        out.n_verts = u;
        out.n_tris = t;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "sparse marching cubes launch");
    return 0;
}

// The caller has waited for every stream that used the buffers (host-side),
// so the frees need no ordering: the per-thread stream takes them.
void sparse_mc_release(SparseMCResult& r) {
    if (r.verts) cudaFreeAsync(r.verts, cudaStreamPerThread);
    if (r.tris) cudaFreeAsync(r.tris, cudaStreamPerThread);
    r = SparseMCResult{};
}

}  // namespace cubvh
