// Query kernels over one compressed 8-wide BVH (layout.h): unsigned distance,
// the two sign passes of signed distance (watertight / raystab), and
// closest-hit ray tracing.
//
// Reference kernels replaced: src/bvh.cu:631-740 and the traversals they
// call (src/bvh.cu:250-427): one thread per query, 128-thread blocks, a
// 32-entry local stack, children re-sorted per visit.
//
// Execution model here:
//  * one thread owns one query, but warps are persistent: each warp walks a
//    block-cyclic sequence of 32-query blocks (warp w takes blocks w, w + W,
//    w + 2W, ...) and hands the next query of its current block to any lane
//    whose query finished (ballot + popc), so lanes never idle while the warp
//    still has work; there are no global atomics and the assignment is
//    deterministic;
//  * traversal is "while-while": lanes keep descending inner nodes until
//    every lane of the warp holds a leaf (or is done), then all test their
//    leaves together, which keeps node and leaf work converged;
//  * point queries are visited in Morton-cell order (a counting sort of the
//    points into 2^(3b) cells of the BVH box) so that the 32 lanes of a warp
//    traverse nearly the same nodes; the permutation only reorders work,
//    every result is written to the query's own index;
//  * children are visited nearest-first (8 keys sorted as packed 32-bit
//    integers); the nearest child is descended directly, the rest pushed on
//    a local-memory stack with their lower-bound key, re-checked on pop.
#include <climits>
#include <cstdint>
#include <cooperative_groups.h>
#include <cub/block/block_radix_sort.cuh>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "launches.h"
#include "geom.cuh"
#include "kernels.h"
#include "scan.cuh"

namespace cubvh {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kQBlock = 128;  // threads per block of the query kernels

// ------------------------------------------------------------------ nodes
struct NodeView {
    float ox, oy, oz, sx, sy, sz;
    int child_base, tri_base;
    uint32_t meta0, meta1;
    uint32_t lx0, lx1, ly0, ly1, lz0, lz1, hx0, hx1, hy0, hy1, hz0, hz1;
};

__device__ __forceinline__ NodeView load_node(const CNode* __restrict__ nodes, int i) {
    const uint4* p = reinterpret_cast<const uint4*>(nodes + i);
    const uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3), w4 = __ldg(p + 4);
    NodeView n;
    n.ox = __uint_as_float(w0.x); n.oy = __uint_as_float(w0.y); n.oz = __uint_as_float(w0.z);
    n.sx = exp2i((int)(int8_t)(w0.w & 0xFF));
    n.sy = exp2i((int)(int8_t)((w0.w >> 8) & 0xFF));
    n.sz = exp2i((int)(int8_t)((w0.w >> 16) & 0xFF));
    n.child_base = (int)w1.x; n.tri_base = (int)w1.y; n.meta0 = w1.z; n.meta1 = w1.w;
    n.lx0 = w2.x; n.lx1 = w2.y; n.ly0 = w2.z; n.ly1 = w2.w;
    n.lz0 = w3.x; n.lz1 = w3.y; n.hx0 = w3.z; n.hx1 = w3.w;
    n.hy0 = w4.x; n.hy1 = w4.y; n.hz0 = w4.z; n.hz1 = w4.w;
    return n;
}
// A node's links (what a warp-uniform traversal needs besides the boxes).
struct NodeLinks {
    int child_base, tri_base;
    uint32_t meta0, meta1;
};
template <class N>
__device__ __forceinline__ uint32_t meta_of(const N& n, int j) {
    return ((j < 4 ? n.meta0 : n.meta1) >> (8 * (j & 3))) & 0xFFu;
}
// byte k of w as a float: 0x4B0000qq is 2^23 + q, minus 2^23 is q exactly
__device__ __forceinline__ float qbyte(uint32_t w, int k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + (unsigned)k)) - 8388608.0f;
}
// origin + q * 2^e: exact product, one rounding (same as the host check)
__device__ __forceinline__ void child_box(const NodeView& n, int j, float3& lo, float3& hi) {
    const int b = j & 3;
    const bool h = j >= 4;
    lo.x = fmaf(qbyte(h ? n.lx1 : n.lx0, b), n.sx, n.ox);
    lo.y = fmaf(qbyte(h ? n.ly1 : n.ly0, b), n.sy, n.oy);
    lo.z = fmaf(qbyte(h ? n.lz1 : n.lz0, b), n.sz, n.oz);
    hi.x = fmaf(qbyte(h ? n.hx1 : n.hx0, b), n.sx, n.ox);
    hi.y = fmaf(qbyte(h ? n.hy1 : n.hy0, b), n.sy, n.oy);
    hi.z = fmaf(qbyte(h ? n.hz1 : n.hz0, b), n.sz, n.oz);
}
// >= 0: internal node index; < 0: leaf, -(slot * 4 + count - 1) - 1
template <class N>
__device__ __forceinline__ int child_ref(const N& n, uint32_t m) {
    if (m & 0x80u) return n.child_base + (int)(m & 7u);
    return -((((n.tri_base + (int)(m & 31u)) << 2) | (int)((m >> 5) & 3u)) + 1);
}

// Cooperative decode for warp-uniform traversals (every lane visits the same
// node): lane l < 12 loads word l of the quantised bytes (coordinate l / 2 =
// lo x, y, z, hi x, y, z of children 4 * (l % 2) .. + 3), decodes it as
// child_box does and stores the floats in the warp's box table s (64 floats,
// 16-byte aligned): child j at s[8j .. 8j + 7] = lo.xyz, -, hi.xyz, -.  The
// whole warp then reads the boxes with broadcast loads instead of decoding
// all 48 bounds in every lane.  Called by all lanes.
__device__ __forceinline__ NodeLinks decode_node_warp(const CNode* __restrict__ nodes, int i, float* s) {
    const int lane = threadIdx.x & 31;
    const uint4* p = reinterpret_cast<const uint4*>(nodes + i);
    const uint4 l = __ldg(p + 1);
    uint4 h = make_uint4(0u, 0u, 0u, 0u);
    uint32_t q = 0u;
    if (lane < 12) {  // loads first: they do not wait for the table to be free
        h = __ldg(p);
        q = __ldg(reinterpret_cast<const uint32_t*>(p + 2) + lane);
    }
    __syncwarp();  // the previous node's boxes have been read
    if (lane < 12) {
        const int c = lane >> 1;
        const int ax = c < 3 ? c : c - 3;
        const float o = __uint_as_float(ax == 0 ? h.x : (ax == 1 ? h.y : h.z));
        const float sc = exp2i((int)(int8_t)((h.w >> (8 * ax)) & 0xFFu));
        float* d = s + 32 * (lane & 1) + (c < 3 ? c : c + 1);
#pragma unroll
        for (int b = 0; b < 4; ++b) d[8 * b] = fmaf(qbyte(q, b), sc, o);
    }
    __syncwarp();
    return NodeLinks{(int)l.x, (int)l.y, l.z, l.w};
}
// Cooperative load of a leaf's triangles (slots s0 .. s1 - 1, at most four,
// contiguous) into the warp's table: lane l < 3 * count loads 16-byte word l,
// so the leaf costs one memory latency instead of one per triangle.  Called
// by all lanes; the table is the box table (the two are used in turn).
__device__ __forceinline__ void load_leaf_warp(const CTri* __restrict__ tris, int s0, int s1, float* s) {
    const int lane = threadIdx.x & 31;
    const bool ld = lane < 3 * (s1 - s0);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ld) v = __ldg(reinterpret_cast<const float4*>(tris + s0) + lane);
    __syncwarp();  // the previous contents have been read
    if (ld) reinterpret_cast<float4*>(s)[lane] = v;
    __syncwarp();
}
// triangle i of the leaf in the warp's table
__device__ __forceinline__ TriV warp_tri(const float* s, int i) {
    const float4* p = reinterpret_cast<const float4*>(s) + 3 * i;
    const float4 w0 = p[0], w1 = p[1], w2 = p[2];
    TriV t;
    t.a = make_float3(w0.x, w0.y, w0.z); t.id = __float_as_int(w0.w);
    t.b = make_float3(w1.x, w1.y, w1.z); t.ke2 = w1.w;
    t.c = make_float3(w2.x, w2.y, w2.z); t.k = w2.w;
    return t;
}
__device__ __forceinline__ void warp_box(const float* s, int j, float3& lo, float3& hi) {
    const float4 a = *reinterpret_cast<const float4*>(s + 8 * j);
    const float4 b = *reinterpret_cast<const float4*>(s + 8 * j + 4);
    lo = make_float3(a.x, a.y, a.z);
    hi = make_float3(b.x, b.y, b.z);
}

// Batcher odd-even merge sort network for 8 keys (19 comparators), ascending.
#define CUBVH_CS(i, j) { const uint32_t a_ = k[i], b_ = k[j]; k[i] = min(a_, b_); k[j] = max(a_, b_); }
__device__ __forceinline__ void sort8(uint32_t k[8]) {
    CUBVH_CS(0, 1) CUBVH_CS(2, 3) CUBVH_CS(4, 5) CUBVH_CS(6, 7)
    CUBVH_CS(0, 2) CUBVH_CS(1, 3) CUBVH_CS(4, 6) CUBVH_CS(5, 7)
    CUBVH_CS(1, 2) CUBVH_CS(5, 6)
    CUBVH_CS(0, 4) CUBVH_CS(1, 5) CUBVH_CS(2, 6) CUBVH_CS(3, 7)
    CUBVH_CS(2, 4) CUBVH_CS(3, 5)
    CUBVH_CS(1, 2) CUBVH_CS(3, 4) CUBVH_CS(5, 6)
}
#undef CUBVH_CS

__device__ __forceinline__ float box_d2(float3 p, float3 lo, float3 hi) {
    const float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.f);
    const float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.f);
    const float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.f);
    return dx * dx + dy * dy + dz * dz;
}
// Conservative slab interval: computed bounds widened by 1e-6 relative
// (each bound carries at most three roundings).
// SAFE: for rays with a zero direction component (inv = +-inf).  A ray with
// d.x == 0 stays in the x slab of a box for every t if lo.x <= o.x <= hi.x
// and never otherwise; (lo.x - o.x) * inv.x is +-inf except when the origin
// lies on the plane (0 * inf = NaN), which then counts as inside the slab.
template <bool SAFE = false>
__device__ __forceinline__ void box_ray(float3 o, float3 inv, float3 lo, float3 hi, float& tn, float& tf) {
    float t0x = (lo.x - o.x) * inv.x, t1x = (hi.x - o.x) * inv.x;
    float t0y = (lo.y - o.y) * inv.y, t1y = (hi.y - o.y) * inv.y;
    float t0z = (lo.z - o.z) * inv.z, t1z = (hi.z - o.z) * inv.z;
    if (SAFE) {
        if (t0x != t0x) t0x = -inv.x;
        if (t1x != t1x) t1x = inv.x;
        if (t0y != t0y) t0y = -inv.y;
        if (t1y != t1y) t1y = inv.y;
        if (t0z != t0z) t0z = -inv.z;
        if (t1z != t1z) t1z = inv.z;
    }
    tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    tn -= 1e-6f * fabsf(tn);
    tf += 1e-6f * fabsf(tf);
}
// 1/d per axis for box_ray; a ray with an infinite reciprocal (a zero or
// subnormal direction component) must use box_ray<true>.
__device__ __forceinline__ float3 ray_inv(float3 d) { return make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z); }
__device__ __forceinline__ bool ray_degenerate(float3 inv) { return isinf(inv.x) || isinf(inv.y) || isinf(inv.z); }
// 1/d with the hardware approximation (at most 1 ulp off: box_ray's 1e-6
// widening covers it) for unit directions; zero and subnormal components
// give +-inf, as ray_inv.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float3 ray_inv_approx(float3 d) {
    return make_float3(rcp_approx(d.x), rcp_approx(d.y), rcp_approx(d.z));
}

// Any-hit traversal step: push the children of node nd that the ray (o, inv)
// enters within [0, cull].
template <bool SAFE>
__device__ __forceinline__ void push_ray_children(const NodeView& nd, float3 o, float3 inv, float cull, int* st,
                                                  int& sp) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t m = meta_of(nd, j);
        float3 lo, hi;
        child_box(nd, j, lo, hi);
        float tn, tf;
        box_ray<SAFE>(o, inv, lo, hi, tn, tf);
        if (m != kEmpty && tn <= tf && tf >= 0.f && tn <= cull) st[sp++] = child_ref(nd, m);
    }
}

// Entry distance (as ordered bits) of the ray into each child of nd, kFull
// where the ray does not need the child.
// The same step for a ray without zero direction components, with the
// node's affine decode folded into the ray: along axis a the plane of byte q
// is met at t = (origin_a + q * s_a - o_a) * inv_a, computed as
// fma(q, A_a, B_a) with A_a = s_a * inv_a and B_a = (origin_a - o_a) * inv_a.
// Against the decoded plane (itself origin + q * s rounded once) this is off
// by less than 6 * 2^-24 * S_a, S_a = |origin_a * inv_a| + 255 |A_a| + |B_a|
// (inv from the hardware reciprocal, within 1 ulp), so entries are computed
// with B_a - E_a and exits with B_a + E_a, E_a = 1e-6 * S_a (about 16 * 2^-24
// * S_a).  The ray's direction signs fix which of a child's two planes is
// the near one on each axis, so no per-child min / max is needed.
__device__ __forceinline__ void push_ray_children_affine(const NodeView& nd, float3 o, float3 inv, float cull,
                                                         int* st, int& sp) {
    const float ax = nd.sx * inv.x, ay = nd.sy * inv.y, az = nd.sz * inv.z;
    const float bx = (nd.ox - o.x) * inv.x, by = (nd.oy - o.y) * inv.y, bz = (nd.oz - o.z) * inv.z;
    const float ex = 1e-6f * (fabsf(nd.ox * inv.x) + 255.f * fabsf(ax) + fabsf(bx));
    const float ey = 1e-6f * (fabsf(nd.oy * inv.y) + 255.f * fabsf(ay) + fabsf(by));
    const float ez = 1e-6f * (fabsf(nd.oz * inv.z) + 255.f * fabsf(az) + fabsf(bz));
    const float nbx = bx - ex, fbx = bx + ex, nby = by - ey, fby = by + ey, nbz = bz - ez, fbz = bz + ez;
    const bool px = inv.x >= 0.f, py = inv.y >= 0.f, pz = inv.z >= 0.f;
    // near / far quantised words per axis (children 0-3, 4-7)
    const uint32_t nx0 = px ? nd.lx0 : nd.hx0, nx1 = px ? nd.lx1 : nd.hx1;
    const uint32_t fx0 = px ? nd.hx0 : nd.lx0, fx1 = px ? nd.hx1 : nd.lx1;
    const uint32_t ny0 = py ? nd.ly0 : nd.hy0, ny1 = py ? nd.ly1 : nd.hy1;
    const uint32_t fy0 = py ? nd.hy0 : nd.ly0, fy1 = py ? nd.hy1 : nd.ly1;
    const uint32_t nz0 = pz ? nd.lz0 : nd.hz0, nz1 = pz ? nd.lz1 : nd.hz1;
    const uint32_t fz0 = pz ? nd.hz0 : nd.lz0, fz1 = pz ? nd.hz1 : nd.lz1;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t m = meta_of(nd, j);
        const int b = j & 3;
        const bool h = j >= 4;
        const float tn = fmaxf(fmaxf(fmaf(qbyte(h ? nx1 : nx0, b), ax, nbx), fmaf(qbyte(h ? ny1 : ny0, b), ay, nby)),
                               fmaf(qbyte(h ? nz1 : nz0, b), az, nbz));
        const float tf = fminf(fminf(fmaf(qbyte(h ? fx1 : fx0, b), ax, fbx), fmaf(qbyte(h ? fy1 : fy0, b), ay, fby)),
                               fmaf(qbyte(h ? fz1 : fz0, b), az, fbz));
        if (m != kEmpty && tn <= tf && tf >= 0.f && tn <= cull) st[sp++] = child_ref(nd, m);
    }
}

template <bool SAFE>
__device__ __forceinline__ void ray_child_keys(const NodeLinks& nd, const float* sb, float3 o, float3 inv, float cull,
                                               uint32_t k[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float3 lo, hi;
        warp_box(sb, j, lo, hi);
        float tn, tf;
        box_ray<SAFE>(o, inv, lo, hi, tn, tf);
        const float key = fmaxf(tn, 0.f);
        const bool need = meta_of(nd, j) != kEmpty && tn <= tf && tf >= 0.f && key <= cull;
        k[j] = need ? __float_as_uint(key) : kFull;
    }
}
// Closest-hit step of one lane's own walk: entry distance (ordered bits of
// max(tn, 0), child index in the low 3 bits) of the ray into each child of
// nd that it enters within [0, cull], kFull for the others.  degen (a zero
// or subnormal direction component): box_ray<true> on the decoded boxes;
// else the affine fold of push_ray_children_affine (same error margins).
__device__ __forceinline__ void lane_child_keys(const NodeView& nd, float3 o, float3 inv, bool degen, float cull,
                                                uint32_t k[8]) {
    if (degen) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float3 lo, hi;
            child_box(nd, j, lo, hi);
            float tn, tf;
            box_ray<true>(o, inv, lo, hi, tn, tf);
            const float key = fmaxf(tn, 0.f);
            const bool need = meta_of(nd, j) != kEmpty && tn <= tf && tf >= 0.f && key <= cull;
            k[j] = need ? ((__float_as_uint(key) & ~7u) | (uint32_t)j) : kFull;
        }
        return;
    }
    const float ax = nd.sx * inv.x, ay = nd.sy * inv.y, az = nd.sz * inv.z;
    const float bx = (nd.ox - o.x) * inv.x, by = (nd.oy - o.y) * inv.y, bz = (nd.oz - o.z) * inv.z;
    const float ex = 1e-6f * (fabsf(nd.ox * inv.x) + 255.f * fabsf(ax) + fabsf(bx));
    const float ey = 1e-6f * (fabsf(nd.oy * inv.y) + 255.f * fabsf(ay) + fabsf(by));
    const float ez = 1e-6f * (fabsf(nd.oz * inv.z) + 255.f * fabsf(az) + fabsf(bz));
    const float nbx = bx - ex, fbx = bx + ex, nby = by - ey, fby = by + ey, nbz = bz - ez, fbz = bz + ez;
    const bool px = inv.x >= 0.f, py = inv.y >= 0.f, pz = inv.z >= 0.f;
    const uint32_t nx0 = px ? nd.lx0 : nd.hx0, nx1 = px ? nd.lx1 : nd.hx1;
    const uint32_t fx0 = px ? nd.hx0 : nd.lx0, fx1 = px ? nd.hx1 : nd.lx1;
    const uint32_t ny0 = py ? nd.ly0 : nd.hy0, ny1 = py ? nd.ly1 : nd.hy1;
    const uint32_t fy0 = py ? nd.hy0 : nd.ly0, fy1 = py ? nd.hy1 : nd.ly1;
    const uint32_t nz0 = pz ? nd.lz0 : nd.hz0, nz1 = pz ? nd.lz1 : nd.hz1;
    const uint32_t fz0 = pz ? nd.hz0 : nd.lz0, fz1 = pz ? nd.hz1 : nd.lz1;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int b = j & 3;
        const bool h = j >= 4;
        const float tn = fmaxf(fmaxf(fmaf(qbyte(h ? nx1 : nx0, b), ax, nbx), fmaf(qbyte(h ? ny1 : ny0, b), ay, nby)),
                               fmaf(qbyte(h ? nz1 : nz0, b), az, nbz));
        const float tf = fminf(fminf(fmaf(qbyte(h ? fx1 : fx0, b), ax, fbx), fmaf(qbyte(h ? fy1 : fy0, b), ay, fby)),
                               fmaf(qbyte(h ? fz1 : fz0, b), az, fbz));
        const float key = fmaxf(tn, 0.f);
        const bool need = meta_of(nd, j) != kEmpty && tn <= tf && tf >= 0.f && key <= cull;
        k[j] = need ? ((__float_as_uint(key) & ~7u) | (uint32_t)j) : kFull;
    }
}
__device__ __forceinline__ float cull_of(double best) { return __double2float_ru(dM(best, 1.000001)); }
__device__ __forceinline__ void leaf_range(int ref, int& s0, int& s1) {
    const int code = -ref - 1;
    s0 = code >> 2; s1 = s0 + (code & 3) + 1;
}


// Dynamic packet queue: a warp takes `grab` consecutive 32-query packets per
// atomicAdd on a per-launch counter (zeroed before the launch), so warps that
// drew cheap packets keep taking more and no SM idles while work remains.
//
// Block budget (left != nullptr): the block's warps take at most *left grabs
// between them (a shared-memory count), then stop, and the block exits.  A
// launch of many such blocks (yield_shape) drains the same queue in short
// block lifetimes, so blocks of kernels on higher-priority streams get SMs
// between them instead of waiting for the whole launch.
struct PacketQueue {
    unsigned long long* ctr;
    int64_t npk, grab, next, end;
    int* left;
    __device__ __forceinline__ PacketQueue(unsigned long long* c, int64_t npk_, int64_t g, int* left_ = nullptr)
        : ctr(c), npk(npk_), grab(g), next(0), end(0), left(left_) {}
    __device__ __forceinline__ unsigned long long grab_start() {
        if (left && atomicSub(left, 1) <= 0) return (unsigned long long)npk;  // budget spent: done
        return atomicAdd(ctr, (unsigned long long)grab);
    }
    // index of the warp's next packet, or -1 when done
    __device__ __forceinline__ int64_t take() {
        if (next == end) {
            unsigned long long b = 0;
            if ((threadIdx.x & 31) == 0) b = grab_start();
            next = (int64_t)__shfl_sync(kFull, b, 0);
            end = next + grab;
        }
        const int64_t p = next++;
        return p < npk ? p : -1;
    }
    // the warp's next range of packets [b, e), false when done (warp-collective)
    __device__ __forceinline__ bool take_range(int64_t& b, int64_t& e) {
        unsigned long long v = 0;
        if ((threadIdx.x & 31) == 0) v = grab_start();
        b = (int64_t)__shfl_sync(kFull, v, 0);
        e = b + grab < npk ? b + grab : npk;
        return b < npk;
    }
};

// What a launch works on: implicit 32-query packets over one BVH (root node
// 0), or a table of packets, each up to 32 consecutive positions of the
// query order on one mesh of an arena (root node, face-0 slot and first
// query index of that mesh).
struct Work {
    const PacketDesc* table;  // nullptr: implicit packets
    const MeshDesc* meshes;
    int64_t n;                // implicit: queries; table: packets
    int slot0;                // implicit: face-0 slot of the single BVH
    int64_t qbase = 0;        // implicit: index of query 0 within its call (raystab streams)
    __device__ __forceinline__ int64_t packets() const { return table ? n : (n + 31) >> 5; }
    __device__ __forceinline__ void get(int64_t p, int64_t& start, int& count, int& root, int& s0,
                                        int64_t& qoff) const {
        if (table) {
            const PacketDesc d = table[p];
            const MeshDesc m = meshes[d.mesh];
            start = d.start; count = d.count; root = m.root; s0 = m.slot0; qoff = m.qoff;
        } else {
            start = p * 32; count = (int)min((int64_t)32, n - start); root = 0; s0 = slot0; qoff = -qbase;
        }
    }
};

__device__ __forceinline__ float3 load3(const float* __restrict__ a, int64_t i) {
    return make_float3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
}

// ------------------------------------------------------- unsigned distance
// Warp-uniform stack of a packet traversal, distributed over the lanes'
// registers: entry e lives in lane e % 32, register slot e / 32 (kStack = 96
// entries).  push / pop are called by all lanes with the same arguments.
struct WarpStack {
    int r0 = 0, r1 = 0, r2 = 0;
    uint32_t k0 = 0, k1 = 0, k2 = 0;
    int sp = 0;
    __device__ __forceinline__ void push(int ref, uint32_t key) {
        if ((int)(threadIdx.x & 31) == (sp & 31)) {
            const int s = sp >> 5;
            if (s == 0) { r0 = ref; k0 = key; } else if (s == 1) { r1 = ref; k1 = key; } else { r2 = ref; k2 = key; }
        }
        ++sp;
    }
    __device__ __forceinline__ void pop(int& ref, uint32_t& key) {
        --sp;
        const int s = sp >> 5;
        ref = __shfl_sync(kFull, s == 0 ? r0 : (s == 1 ? r1 : r2), sp & 31);
        key = __shfl_sync(kFull, s == 0 ? k0 : (s == 1 ? k1 : k2), sp & 31);
    }
    // next entry whose key some lane still needs (key <= cullmax)
    __device__ __forceinline__ bool next(uint32_t cullmax, int& cur) {
        while (sp > 0) {
            int ref; uint32_t key;
            pop(ref, key);
            if (key <= cullmax) { cur = ref; return true; }
        }
        return false;
    }
};

// The same stack in the warp's shared memory (ref and key tables of
// kSmemStack entries each); push / pop are called by all lanes with the same
// arguments, lane 0 writes.  k_ray uses it (C1 rays 6.49 -> 6.40 ms against
// the register stack); for the distance kernels it was not faster.
constexpr int kSmemStack = kStack;
struct WarpStackSmem {
    int* ref; uint32_t* key;
    int sp = 0;
    __device__ __forceinline__ WarpStackSmem(int* r, uint32_t* k) : ref(r), key(k) {}
    __device__ __forceinline__ void push(int r, uint32_t k) {
        __syncwarp();   // earlier reads of the slot are done
        if ((threadIdx.x & 31) == 0) { ref[sp] = r; key[sp] = k; }
        ++sp;
        __syncwarp();
    }
    __device__ __forceinline__ bool next(uint32_t cullmax, int& cur) {
        while (sp > 0) {
            --sp;
            const int r = ref[sp];
            const uint32_t k = key[sp];
            if (k <= cullmax) { cur = r; return true; }
        }
        return false;
    }
};

constexpr int kCand = 8;         // per-lane candidate list of the distance search
constexpr int kHeavyMinWork = 256;  // a packet is never handed off below this many visits


// Exact nearest triangle of 32 Morton-adjacent points per warp (a packet):
// the warp walks the union of the lanes' search paths with warp-uniform
// control flow.  A child is visited if any lane's FP32 box distance is within
// that lane's bound (ballot), in the order of the smallest such distance
// (warp min).  Leaves run the FP32 triangle test in every lane; each lane
// keeps U, an upper bound of its squared distance (FP32 estimate + its error
// bound), and a short list of triangles whose lower bound is within U.  At
// the end every lane evaluates its surviving candidates in double: the
// minimum (ties -> lowest face index) is the exact nearest triangle.
//
// Tail control: a packet whose walk grows past a warp's fair share of the
// launch (the mean node + leaf visits of the packets finished so far, in
// stats[0] / stats[1], times the packets per warp `ppw`; at least
// kHeavyMinWork) would hold the launch's tail alone: points deep inside a
// closed mesh or near its medial axis are about equally far from very many
// triangles.  Such a packet stops and appends its queries to the heavy list,
// which k_udf_heavy serves with a warp per query.  When the list is full the
// packet finishes here instead.
//
// The check costs registers in the traversal loop, so it is compiled in
// (TAIL) only for launches with few packets per warp (below 24): with ppw packets per
// warp at most one packet in ppw can pass the fair share, and only such
// launches end on a few long packets.
template <bool UVW, bool SLOT, bool TAIL>
__global__ void __launch_bounds__(kQBlock) k_udf(Work w, const uint32_t* __restrict__ order,
                                                 const float* __restrict__ pts, float* __restrict__ dist,
                                                 int64_t* __restrict__ face_id, float* __restrict__ uvw,
                                                 int32_t* __restrict__ slot_out, const CNode* __restrict__ nodes,
                                                 const CTri* __restrict__ tris,
                                                 unsigned long long* __restrict__ ctr, int64_t grab,
                                                 uint2* __restrict__ heavy, unsigned long long* __restrict__ n_heavy,
                                                 int64_t heavy_cap, unsigned long long* __restrict__ stats,
                                                 float ppw, int block_grabs) {
    const int lane = threadIdx.x & 31;
    __shared__ __align__(16) float s_box[kQBlock / 32][64];
    __shared__ int s_left;
    float* sb = s_box[threadIdx.x >> 5];
    if (block_grabs > 0) {  // uniform: the launch's block budget
        if (threadIdx.x == 0) s_left = block_grabs;
        __syncthreads();
    }
    PacketQueue pq(ctr, w.packets(), grab, block_grabs > 0 ? &s_left : nullptr);
    for (int64_t pk = pq.take(); pk >= 0; pk = pq.take()) {
        int64_t start, qoff;
        int cnt, root, slot_face0;
        w.get(pk, start, cnt, root, slot_face0, qoff);
        const int64_t qi = start + lane;
        const bool act = lane < cnt;
        const int64_t idx = act ? (order ? (int64_t)order[qi] : qi) : 0;
        const float3 p = act ? load3(pts, idx) : make_float3(0.f, 0.f, 0.f);
        // U: upper bound of the lane's nearest squared distance (MAX_DIST^2)
        float U = act ? 1e6f : -1.f;
        float cull = act ? U * 1.000002f : -1.f;
        int cs[kCand];
        float cl[kCand];
        int nc = 0;
        double bx = 1e6;     // exact best of flushed candidates
        int sx = -1, ix = 0;
        auto flush = [&](bool final_pass) {
            for (int i = 0; i < nc; ++i) {
                if (final_pass && cl[i] > U) continue;
                const TriV t = load_tri(tris, cs[i]);
                double bary[3]; d3 cp;
                const double e = closest_on_tri_d(to_d3(p), to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
                if (e < bx || (e == bx && (sx < 0 || t.id < ix))) { bx = e; sx = cs[i]; ix = t.id; }
            }
            nc = 0;
        };
        uint32_t cullmax = __reduce_max_sync(kFull, __float_as_uint(fmaxf(cull, 0.f)));
        WarpStack st;
        int cur = root;
        bool live = __any_sync(kFull, act);
        int work = 0;
        bool handed_off = false;
        while (live) {
            // warp-uniform; checked every 64 visits from kHeavyMinWork on
            if (TAIL && (++work & 63) == 0 && work >= kHeavyMinWork) {
                unsigned long long su = 0, np = 0;
                if (lane == 0) {
                    su = *reinterpret_cast<volatile unsigned long long*>(stats);
                    np = *reinterpret_cast<volatile unsigned long long*>(stats + 1);
                }
                su = __shfl_sync(kFull, su, 0);
                np = __shfl_sync(kFull, np, 0);
                if (np >= 32 && (float)work > (float)su / (float)np * ppw) {
                    unsigned long long b = 0;
                    if (lane == 0) b = atomicAdd(n_heavy, (unsigned long long)cnt);
                    b = __shfl_sync(kFull, b, 0);
                    const uint32_t mesh = w.table ? (uint32_t)w.table[pk].mesh : 0u;
                    if (act && (int64_t)b + lane < heavy_cap) heavy[b + lane] = make_uint2((uint32_t)idx, mesh);
                    if ((int64_t)b + cnt <= heavy_cap) { handed_off = true; break; }
                    // list full: finish the packet here (later checks append again; the list
                    // length used is min(count, capacity))
                }
            }
            if (cur >= 0) {
                const NodeLinks nd = decode_node_warp(nodes, cur, sb);
                uint32_t k[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float3 lo, hi;
                    warp_box(sb, j, lo, hi);
                    const float d2 = box_d2(p, lo, hi);
                    const bool need = meta_of(nd, j) != kEmpty && d2 <= cull;
                    const uint32_t kmin = __reduce_min_sync(kFull, need ? __float_as_uint(d2) : kFull);
                    k[j] = kmin != kFull ? ((kmin & ~7u) | (uint32_t)j) : kFull;
                }
                sort8(k);
#pragma unroll
                for (int i = 7; i >= 1; --i)
                    if (k[i] != kFull) st.push(child_ref(nd, meta_of(nd, (int)(k[i] & 7u))), k[i] & ~7u);
                if (k[0] != kFull) cur = child_ref(nd, meta_of(nd, (int)(k[0] & 7u)));
                else live = st.next(cullmax, cur);
            } else {
                int s0, s1;
                leaf_range(cur, s0, s1);
                load_leaf_warp(tris, s0, s1, sb);
                for (int s = s0; s < s1; ++s) {
                    const TriV t = warp_tri(sb, s - s0);
                    float err;
                    const float e32 = tri_d2_f(p, t, &err);
                    const float lb = e32 - err;
                    if (act && lb <= U) {
                        U = fminf(U, e32 + err);
                        if (nc == kCand) {  // keep only live candidates, else settle them exactly
                            int m = 0;
                            for (int i = 0; i < nc; ++i)
                                if (cl[i] <= U) { cs[m] = cs[i]; cl[m] = cl[i]; ++m; }
                            nc = m;
                            if (nc == kCand) {
                                flush(false);
                                U = fminf(U, __double2float_ru(bx));
                            }
                        }
                        cs[nc] = s; cl[nc] = lb; ++nc;
                    }
                }
                cull = act ? U * 1.000002f : -1.f;
                cullmax = __reduce_max_sync(kFull, __float_as_uint(fmaxf(cull, 0.f)));
                live = st.next(cullmax, cur);
            }
        }
        if (TAIL && !handed_off && lane == 0) {
            atomicAdd(stats, (unsigned long long)work);
            atomicAdd(stats + 1, 1ull);
        }
        if (handed_off || !act) continue;
        flush(true);
        double d64;
        if (sx < 0) {  // nothing within MAX_DIST: distance 0 on face 0
            sx = slot_face0; d64 = 0.0;
            ix = load_tri(tris, sx).id;
        } else {
            d64 = __dsqrt_rn(bx);
        }
        dist[idx] = __double2float_rn(d64);
        face_id[idx] = (int64_t)ix;
        if (SLOT) slot_out[idx] = sx;
        if (UVW) {
            const TriV t = load_tri(tris, sx);
            double bary[3]; d3 cp;
            closest_on_tri_d(to_d3(p), to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
            uvw[3 * idx] = __double2float_rn(bary[0]);
            uvw[3 * idx + 1] = __double2float_rn(bary[1]);
            uvw[3 * idx + 2] = __double2float_rn(bary[2]);
        }
    }
}


// ---------------------------------------------------------- heavy queries
// One warp per query handed off by k_udf.  Each step pops up to four live
// nodes from a stack in shared memory (lane = child j of popped node i,
// 8 * i + j), pushes the internal children within the bound and tests the
// triangles of the leaf children 32 at a time, one per lane.  U (an upper
// bound of the squared distance) and the candidate list are the warp's, and
// candidates are settled in double exactly as in k_udf, so the result is the
// same exact nearest triangle (lowest face index on ties).
constexpr int kHStack = 512;
constexpr int kHCand = 64;
// Each step pushes at most 32 children one level below the deepest node it
// popped, so the stack holds at most one such batch per tree level.
static_assert(kHStack >= 32 * (kMaxDepth + 1), "heavy-query stack too small for the tree depth");
struct HeavyWarp {
    int ref[kHStack];
    uint32_t key[kHStack];
    int pop[4];
    int tslot[4 * 32];
    int cs[kHCand];
    float cl[kHCand];
};

// Exact minimum (ties -> lowest face index) over the candidates i < nc whose
// lower bound is <= lim, merged into (bx, sx, ix); warp-parallel, the result
// is the same in every lane.
__device__ void heavy_settle(const HeavyWarp& S, int nc, float lim, const CTri* __restrict__ tris, float3 p,
                             double& bx, int& sx, int& ix) {
    const int lane = threadIdx.x & 31;
    double e = CUDART_INF;
    int s = -1, id = INT_MAX;
    for (int i = lane; i < nc; i += 32) {
        if (S.cl[i] > lim) continue;
        const int sl = S.cs[i];
        const TriV t = load_tri(tris, sl);
        double bary[3]; d3 cp;
        const double d = closest_on_tri_d(to_d3(p), to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
        if (d < e || (d == e && t.id < id)) { e = d; s = sl; id = t.id; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double e2 = __shfl_xor_sync(kFull, e, o);
        const int s2 = __shfl_xor_sync(kFull, s, o), id2 = __shfl_xor_sync(kFull, id, o);
        if (e2 < e || (e2 == e && id2 < id)) { e = e2; s = s2; id = id2; }
    }
    if (s >= 0 && (e < bx || (e == bx && (sx < 0 || id < ix)))) { bx = e; sx = s; ix = id; }
}

template <bool UVW, bool SLOT>
__global__ void __launch_bounds__(kQBlock) k_udf_heavy(const uint2* __restrict__ heavy,
                                                       const unsigned long long* __restrict__ n_heavy,
                                                       int64_t heavy_cap, const MeshDesc* __restrict__ meshes,
                                                       int slot_face0, const float* __restrict__ pts,
                                                       float* __restrict__ dist, int64_t* __restrict__ face_id,
                                                       float* __restrict__ uvw, int32_t* __restrict__ slot_out,
                                                       const CNode* __restrict__ nodes, const CTri* __restrict__ tris,
                                                       unsigned long long* __restrict__ ctr) {
    __shared__ HeavyWarp shw[kQBlock / 32];
    HeavyWarp& S = shw[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t nh_all = (int64_t)*n_heavy;
    const int64_t nh = nh_all < heavy_cap ? nh_all : heavy_cap;
    while (true) {
        unsigned long long qi = 0;
        if (lane == 0) qi = atomicAdd(ctr, 1ull);
        qi = __shfl_sync(kFull, qi, 0);
        if ((int64_t)qi >= nh) break;
        const uint2 hq = heavy[qi];
        const int64_t idx = hq.x;
        int root = 0, s0 = slot_face0;
        if (meshes) {
            const MeshDesc md = meshes[hq.y];
            root = md.root;
            s0 = md.slot0;
        }
        const float3 p = load3(pts, idx);
        float U = 1e6f;  // MAX_DIST^2
        double bx = 1e6;
        int sx = -1, ix = 0;
        int nc = 0, sp = 1;
        __syncwarp();  // the previous query is done with S
        if (lane == 0) { S.ref[0] = root; S.key[0] = 0u; }
        __syncwarp();
        while (sp > 0) {
            const float cull = U * 1.000002f;
            // pop: of the top 32 entries, the first four (from the top) whose
            // key is within the bound; the culled ones above them go too
            const int pos = sp - 1 - lane;
            const bool alive = pos >= 0 && S.key[pos] <= __float_as_uint(cull);
            const unsigned m = __ballot_sync(kFull, alive);
            int nn = __popc(m), used = sp < 32 ? sp : 32;
            if (nn >= 4) {  // up to and including the fourth live entry
                unsigned m4 = m;
                m4 &= m4 - 1u;
                m4 &= m4 - 1u;
                m4 &= m4 - 1u;
                used = __ffs(m4);
                nn = 4;
            }
            if (alive && __popc(m & lt) < 4) S.pop[__popc(m & lt)] = S.ref[pos];
            sp -= used;
            __syncwarp();
            // children of the popped nodes
            const int ni = lane >> 3, j = lane & 7;
            bool take = false, leaf = false;
            int cref = 0;
            uint32_t key = 0u;
            if (ni < nn) {
                const NodeView nd = load_node(nodes, S.pop[ni]);
                const uint32_t mm = meta_of(nd, j);
                if (mm != kEmpty) {
                    float3 lo, hi;
                    child_box(nd, j, lo, hi);
                    const float d2 = box_d2(p, lo, hi);
                    if (d2 <= cull) {
                        take = true;
                        key = __float_as_uint(d2);
                        cref = child_ref(nd, mm);
                        leaf = cref < 0;
                    }
                }
            }
            const unsigned mi = __ballot_sync(kFull, take && !leaf);
            if (take && !leaf) {
                const int q = sp + __popc(mi & lt);
                S.ref[q] = cref;
                S.key[q] = key;
            }
            sp += __popc(mi);
            // the leaf children's triangles, 32 per round
            int c = 0, a = 0;
            if (take && leaf) {
                int b;
                leaf_range(cref, a, b);
                c = b - a;
            }
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const int T = __shfl_sync(kFull, incl, 31);
            for (int i = 0; i < c; ++i) S.tslot[incl - c + i] = a + i;
            __syncwarp();
            for (int base = 0; base < T; base += 32) {
                const int t = base + lane;
                float e32 = 0.f, err = 0.f;
                int slot = -1;
                if (t < T) {
                    slot = S.tslot[t];
                    e32 = tri_d2_f(p, load_tri(tris, slot), &err);
                }
                const float ub = t < T ? e32 + err : CUDART_INF_F;
                U = fminf(U, __uint_as_float(__reduce_min_sync(kFull, __float_as_uint(ub))));
                const float lb = e32 - err;
                const bool cand = t < T && lb <= U;
                const unsigned mc = __ballot_sync(kFull, cand);
                if (nc + __popc(mc) > kHCand) {  // warp-uniform: drop dead candidates, else settle them
                    int keep = 0;
                    for (int i0 = 0; i0 < nc; i0 += 32) {
                        const int i = i0 + lane;
                        const bool kp = i < nc && S.cl[i] <= U;
                        const int cs_i = kp ? S.cs[i] : 0;
                        const float cl_i = kp ? S.cl[i] : 0.f;
                        const unsigned mk = __ballot_sync(kFull, kp);
                        __syncwarp();  // every lane has read its entry
                        if (kp) {
                            S.cs[keep + __popc(mk & lt)] = cs_i;
                            S.cl[keep + __popc(mk & lt)] = cl_i;
                        }
                        keep += __popc(mk);
                        __syncwarp();
                    }
                    nc = keep;
                    if (nc + __popc(mc) > kHCand) {
                        heavy_settle(S, nc, CUDART_INF_F, tris, p, bx, sx, ix);
                        U = fminf(U, __double2float_ru(bx));
                        nc = 0;
                        __syncwarp();
                    }
                }
                if (cand) {
                    S.cs[nc + __popc(mc & lt)] = slot;
                    S.cl[nc + __popc(mc & lt)] = lb;
                }
                nc += __popc(mc);
                __syncwarp();
            }
        }
        heavy_settle(S, nc, U, tris, p, bx, sx, ix);
        if (lane == 0) {
            double d64;
            if (sx < 0) {  // nothing within MAX_DIST: distance 0 on face 0
                sx = s0;
                d64 = 0.0;
                ix = load_tri(tris, sx).id;
            } else {
                d64 = __dsqrt_rn(bx);
            }
            dist[idx] = __double2float_rn(d64);
            face_id[idx] = (int64_t)ix;
            if (SLOT) slot_out[idx] = sx;
            if (UVW) {
                const TriV t = load_tri(tris, sx);
                double bary[3]; d3 cp;
                closest_on_tri_d(to_d3(p), to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
                uvw[3 * idx] = __double2float_rn(bary[0]);
                uvw[3 * idx + 1] = __double2float_rn(bary[1]);
                uvw[3 * idx + 2] = __double2float_rn(bary[2]);
            }
        }
    }
}

// ------------------------------------------------------------ watertight
// Sum of unit normals of every triangle whose squared distance to cp is
// below 1e-6 (src/bvh.cu:356-396; the division by the count does not change
// the sign and is omitted).  cp lies on the triangle in soup slot `own` (the
// query's nearest), so that one needs no distance test.
__device__ d3 normal_sum(const CNode* __restrict__ nodes, const CTri* __restrict__ tris, d3 cp, int root, int own) {
    const float3 cf = make_float3(__double2float_rn(cp.x), __double2float_rn(cp.y), __double2float_rn(cp.z));
    const float cinf = f3inf(cf);
    const float r = 1e-3f + 4e-7f * (1.f + cinf);
    const float r2 = r * r * 1.00001f;
    const float slack = 1e-9f * (1.f + cinf);
    d3 sum{0.0, 0.0, 0.0};
    int st[kStack];
    int sp = 0;
    st[sp++] = root;
    while (sp > 0) {
        const int ref = st[--sp];
        if (ref >= 0) {
            const NodeView nd = load_node(nodes, ref);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t m = meta_of(nd, j);
                float3 lo, hi;
                child_box(nd, j, lo, hi);
                if (m != kEmpty && box_d2(cf, lo, hi) <= r2) st[sp++] = child_ref(nd, m);
            }
        } else {
            int s0, s1;
            leaf_range(ref, s0, s1);
            for (int s = s0; s < s1; ++s) {
                const TriV t = load_tri(tris, s);
                float err;
                const float d2 = tri_d2_f(cf, t, &err);
                if (d2 - err - slack > 1.000001e-6f) continue;
                double bary[3]; d3 q;
                const d3 a = to_d3(t.a), b = to_d3(t.b), c = to_d3(t.c);
                if (s == own || closest_on_tri_d(cp, a, b, c, bary, &q) < 1e-6) {
                    const d3 nr = dcross(dsub(b, a), dsub(c, a));
                    const double len = __dsqrt_rn(ddot(nr, nr));
                    if (len > 0.0) sum = dadd(sum, d3{dD(nr.x, len), dD(nr.y, len), dD(nr.z, len)});
                }
            }
        }
    }
    return sum;
}

// normal_sum over a precomputed candidate list of cp's triangle (k_near_lists):
// the same tests in the same order, without the walk from the root, and the
// unit normals read from the table k_near_lists computed them into (the same
// operations as normal_sum's).
__device__ d3 normal_sum_list(const CTri* __restrict__ tris, d3 cp, int own, const int32_t* __restrict__ lst,
                              int count, const double* __restrict__ nrm) {
    const float3 cf = make_float3(__double2float_rn(cp.x), __double2float_rn(cp.y), __double2float_rn(cp.z));
    const float slack = 1e-9f * (1.f + f3inf(cf));
    d3 sum{0.0, 0.0, 0.0};
    for (int k = 0; k < count; ++k) {
        const int s = __ldg(lst + k);
        const TriV t = load_tri(tris, s);
        float err;
        const float d2 = tri_d2_f(cf, t, &err);
        if (d2 - err - slack > 1.000001e-6f) continue;
        double bary[3]; d3 q;
        if (s == own || closest_on_tri_d(cp, to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &q) < 1e-6)
            // a zero normal (degenerate triangle) leaves the sum unchanged: its
            // components are never -0, so adding +0 is exact
            sum = dadd(sum, d3{__ldg(nrm + 3 * s), __ldg(nrm + 3 * s + 1), __ldg(nrm + 3 * s + 2)});
    }
    return sum;
}

// True when an axis among the two triangles' normals and the nine cross
// products of their edges separates a and b by more than r: then no point of
// b lies within r of a point of a.  Any axis u is a valid separating axis, so
// rounding in u itself is harmless; each projection onto u is off by at most
// a few ulps of |u| max|v|, covered by the margin 2e-6 (1 + scale) |u| added to
// r (scale: the larger max |coordinate| of the two triangles).  Degenerate
// axes (|u| = 0) separate nothing.
__device__ bool tri_gap_exceeds(const TriV& a, const TriV& b, float r, float scale) {
    const float3 ea[3] = {f3sub(a.b, a.a), f3sub(a.c, a.b), f3sub(a.a, a.c)};
    const float3 eb[3] = {f3sub(b.b, b.a), f3sub(b.c, b.b), f3sub(b.a, b.c)};
    const float rr = r + 2e-6f * (1.f + scale);
    auto sep = [&](float3 u) {
        const float l2 = f3dot(u, u);
        if (!(l2 > 0.f)) return false;
        const float a0 = f3dot(u, a.a), a1 = f3dot(u, a.b), a2 = f3dot(u, a.c);
        const float b0 = f3dot(u, b.a), b1 = f3dot(u, b.b), b2 = f3dot(u, b.c);
        const float amin = fminf(a0, fminf(a1, a2)), amax = fmaxf(a0, fmaxf(a1, a2));
        const float bmin = fminf(b0, fminf(b1, b2)), bmax = fmaxf(b0, fmaxf(b1, b2));
        return fmaxf(bmin - amax, amin - bmax) > rr * 1.0001f * sqrtf(l2);
    };
    if (sep(f3cross(ea[0], ea[1])) || sep(f3cross(eb[0], eb[1]))) return true;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (sep(f3cross(ea[i], eb[j]))) return true;
    return false;
}

// Candidate lists of the watertight normal sum.  For soup slot t: every slot
// whose triangle's bounding box meets t's box grown by r = 1.001e-3 + 1e-6 (1 +
// max |coordinate|) and that no separating axis (tri_gap_exceeds) puts more
// than r from t, in the order normal_sum's walk reaches them (depth-first,
// children in the same push order, slots ascending in a leaf).  A point cp on
// triangle t has every triangle within normal_sum's radius of it on t's list
// (the radius is at most 1e-3 + 4e-7 (1 + |cp|_inf) and |cp| <= max |vertex|),
// so the list replaces the walk and keeps the summation order.  cnt[t] = -1
// when more than kNear slots qualify: that query walks the tree.
__global__ void __launch_bounds__(kQBlock) k_near_lists(int64_t nt, const CNode* __restrict__ nodes,
                                                        const CTri* __restrict__ tris, int root,
                                                        int32_t* __restrict__ cnt, int32_t* __restrict__ lst,
                                                        double* __restrict__ nrm, int* __restrict__ any_ovf) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
        const TriV a = load_tri(tris, (int)t);
        {
            const d3 da = to_d3(a.a), db = to_d3(a.b), dc = to_d3(a.c);
            const d3 nr = dcross(dsub(db, da), dsub(dc, da));
            const double len = __dsqrt_rn(ddot(nr, nr));
            const bool ok = len > 0.0;
            nrm[3 * t] = ok ? dD(nr.x, len) : 0.0;
            nrm[3 * t + 1] = ok ? dD(nr.y, len) : 0.0;
            nrm[3 * t + 2] = ok ? dD(nr.z, len) : 0.0;
        }
        float3 lo = make_float3(fminf(a.a.x, fminf(a.b.x, a.c.x)), fminf(a.a.y, fminf(a.b.y, a.c.y)),
                                fminf(a.a.z, fminf(a.b.z, a.c.z)));
        float3 hi = make_float3(fmaxf(a.a.x, fmaxf(a.b.x, a.c.x)), fmaxf(a.a.y, fmaxf(a.b.y, a.c.y)),
                                fmaxf(a.a.z, fmaxf(a.b.z, a.c.z)));
        const float vinf = fmaxf(f3inf(lo), f3inf(hi));
        const float r = 1.001e-3f + 1e-6f * (1.f + vinf);
        lo = make_float3(lo.x - r, lo.y - r, lo.z - r);
        hi = make_float3(hi.x + r, hi.y + r, hi.z + r);
        int32_t* out = lst + t * kNear;
        int c = 0;
        int st[kStack];
        int sp = 0;
        st[sp++] = root;
        while (sp > 0) {
            const int ref = st[--sp];
            if (ref >= 0) {
                const NodeView nd = load_node(nodes, ref);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t m = meta_of(nd, j);
                    float3 clo, chi;
                    child_box(nd, j, clo, chi);
                    if (m != kEmpty && clo.x <= hi.x && clo.y <= hi.y && clo.z <= hi.z && chi.x >= lo.x &&
                        chi.y >= lo.y && chi.z >= lo.z)
                        st[sp++] = child_ref(nd, m);
                }
            } else {
                int s0, s1;
                leaf_range(ref, s0, s1);
                for (int s = s0; s < s1; ++s) {
                    const TriV b = load_tri(tris, s);
                    if (fminf(b.a.x, fminf(b.b.x, b.c.x)) <= hi.x && fminf(b.a.y, fminf(b.b.y, b.c.y)) <= hi.y &&
                        fminf(b.a.z, fminf(b.b.z, b.c.z)) <= hi.z && fmaxf(b.a.x, fmaxf(b.b.x, b.c.x)) >= lo.x &&
                        fmaxf(b.a.y, fmaxf(b.b.y, b.c.y)) >= lo.y && fmaxf(b.a.z, fmaxf(b.b.z, b.c.z)) >= lo.z &&
                        (s == (int)t ||
                         !tri_gap_exceeds(a, b, r, fmaxf(vinf, fmaxf(f3inf(b.a), fmaxf(f3inf(b.b), f3inf(b.c))))))) {
                        if (c < kNear) out[c] = s;
                        ++c;
                    }
                }
            }
        }
        cnt[t] = c <= kNear ? c : -1;
        if (c > kNear) atomicOr(any_ovf, 1);
    }
}

// Watertight sign: copysign(distance, normal_sum . (p - cp)), cp the closest
// point of the query's nearest triangle (soup slot `own`).  LIST: the normal
// sum over own's candidate list; a query whose list overflowed is queued in
// ovf for k_sign_watertight_ovf (single BVH).  !LIST: the walk (arenas).
template <bool LIST>
__global__ void __launch_bounds__(kQBlock)
k_sign_watertight(Work w, const uint32_t* __restrict__ order, const float* __restrict__ pts, float* __restrict__ dist,
                  const int32_t* __restrict__ slots, const CNode* __restrict__ nodes, const CTri* __restrict__ tris,
                  const NearLists near, uint32_t* __restrict__ ovf, unsigned long long* __restrict__ ovf_n,
                  unsigned long long* __restrict__ ctr, int64_t grab, int block_grabs) {
    __shared__ int s_left;
    if (block_grabs > 0) {
        if (threadIdx.x == 0) s_left = block_grabs;
        __syncthreads();
    }
    PacketQueue pq(ctr, w.packets(), grab, block_grabs > 0 ? &s_left : nullptr);
    for (int64_t pk = pq.take(); pk >= 0; pk = pq.take()) {
        int64_t start, qoff;
        int cnt, root, s0;
        w.get(pk, start, cnt, root, s0, qoff);
        if ((int)(threadIdx.x & 31) >= cnt) continue;
        const int64_t q = start + (threadIdx.x & 31);
        const int64_t idx = order ? (int64_t)order[q] : q;
        const int own = slots[idx];
        const int nc = LIST ? __ldg(near.cnt + own) : -1;  // in flight during the closest point
        const d3 pd = to_d3(load3(pts, idx));
        const TriV t = load_tri(tris, own);
        double bary[3]; d3 cp;
        closest_on_tri_d(pd, to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
        if (LIST && nc < 0) {
            ovf[atomicAdd(ovf_n, 1ull)] = (uint32_t)idx;
            continue;
        }
        const d3 ns = LIST ? normal_sum_list(tris, cp, own, near.lst + (int64_t)own * kNear, nc, near.nrm)
                           : normal_sum(nodes, tris, cp, root, own);
        // copysign(distance, avg_normal . (p - cp))
        const double s = ddot(ns, dsub(pd, cp));
        const float d = dist[idx];
        dist[idx] = signbit(s) ? -d : d;
    }
}
// The queries k_sign_watertight<true> queued (their lists overflowed): the
// walk from root 0.
__global__ void __launch_bounds__(kQBlock) k_sign_watertight_ovf(const uint32_t* __restrict__ ovf,
                                                                 const unsigned long long* __restrict__ ovf_n,
                                                                 const float* __restrict__ pts,
                                                                 float* __restrict__ dist,
                                                                 const int32_t* __restrict__ slots,
                                                                 const CNode* __restrict__ nodes,
                                                                 const CTri* __restrict__ tris) {
    const int64_t n = (int64_t)*ovf_n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t idx = ovf[i];
        const int own = slots[idx];
        const d3 pd = to_d3(load3(pts, idx));
        const TriV t = load_tri(tris, own);
        double bary[3]; d3 cp;
        closest_on_tri_d(pd, to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
        const d3 ns = normal_sum(nodes, tris, cp, 0, own);
        const double s = ddot(ns, dsub(pd, cp));
        const float d = dist[idx];
        dist[idx] = signbit(s) ? -d : d;
    }
}

// --------------------------------------------------------------- raystab
// Negative iff all 64 stab rays (for k = 0..31: -d_k, then +d_k) hit the mesh
// within [0, 1000) (src/bvh.cu:408-427); the first miss ends the query.
// Whether all rays hit does not depend on the order they are traced in.
//
// Work is per lane, not per warp: a warp takes a chunk of packets (queries in
// Morton-cell order) and each lane takes the chunk's next query from a
// shared-memory counter whenever its own query ends, and starts its next
// stab ray as soon as the current one hits.  Stab directions differ from
// lane to lane and inside queries need 64 rays where outside ones end after a
// few, so lanes never wait for one another except at the end of a chunk.
// The per-query setup (query index, stab stream offset, root) is computed by
// the whole warp in lockstep when the chunk is taken.
//
// With max_rays < 64 this is the first of two passes: a query whose first
// max_rays rays all hit is not finished here but appended to `cand` (query
// index, stab offset, root: warp-aggregated atomic on cand_n), for
// k_sign_raystab_lines.  Outside points mostly see their first rays miss
// and end in this pass; the candidates are mostly inside points, which need
// every ray.
constexpr int kChunkMax = 2;  // packets per raystab chunk
__global__ void __launch_bounds__(kQBlock) k_sign_raystab(Work w, const uint32_t* __restrict__ order,
                                                          const float* __restrict__ pts, float* __restrict__ dist,
                                                          const CNode* __restrict__ nodes,
                                                          const CTri* __restrict__ tris,
                                                          unsigned long long* __restrict__ ctr, int64_t grab,
                                                          int max_rays, uint4* __restrict__ cand,
                                                          unsigned long long* __restrict__ cand_n) {
    __shared__ int s_next[kQBlock / 32];
    __shared__ uint4 s_q[kQBlock / 32][kChunkMax * 32];  // query index, offset x/y bits, root (-1: none)
    const int wib = threadIdx.x >> 5;
    const float tmaxf = 1000.0f;
    const float cull = cull_of(1000.0);
    PacketQueue pq(ctr, w.packets(), grab);
    int64_t pk0, pk1;
    while (pq.take_range(pk0, pk1)) {
        const int total = (int)(pk1 - pk0) * 32;
        for (int i = threadIdx.x & 31; i < total; i += 32) {
            int64_t start, qoff;
            int cnt, rt, s0;
            w.get(pk0 + (i >> 5), start, cnt, rt, s0, qoff);
            uint4 e = make_uint4(0u, 0u, 0u, 0xFFFFFFFFu);
            if ((i & 31) < cnt) {
                const int64_t qi = start + (i & 31);
                const int64_t id = order ? (int64_t)order[qi] : qi;
                // the stab stream of a query is its index within its own call / mesh
                const float2 o2 = stab_offset((uint32_t)(id - qoff));
                e = make_uint4((uint32_t)id, __float_as_uint(o2.x), __float_as_uint(o2.y), (uint32_t)rt);
            }
            s_q[wib][i] = e;
        }
        if ((threadIdx.x & 31) == 0) s_next[wib] = 0;
        __syncwarp();
        int64_t idx = -1;  // current query, -1: none
        int root = 0;
        float3 p = make_float3(0.f, 0.f, 0.f), sd = p, d = p, inv = p;
        float2 off = make_float2(0.f, 0.f);
        float dinf = 0.f;
        bool degen = false;
        uint32_t r = 0;    // ray r: -d_{r/2} for even r, +d_{r/2} for odd r
        int st[kStack];
        int sp = 0;
        while (true) {
            if (idx < 0) {
                int i;
                while ((i = atomicAdd(&s_next[wib], 1)) < total) {
                    const uint4 e = s_q[wib][i];
                    if (e.w != 0xFFFFFFFFu) {
                        idx = e.x;
                        off = make_float2(__uint_as_float(e.y), __uint_as_float(e.z));
                        root = (int)e.w;
                        break;
                    }
                }
                if (idx < 0) break;
                p = load3(pts, idx);
                r = 0;
                sd = stab_dir(0, off);
                d = make_float3(-sd.x, -sd.y, -sd.z);
                inv = ray_inv_approx(d);
                degen = ray_degenerate(inv);
                dinf = f3inf(d);
                sp = 0;
                st[sp++] = root;
            }
            if (sp == 0) { idx = -1; continue; }  // ray r missed: outside
            const int ref = st[--sp];
            bool hit = false;
            if (ref >= 0) {
                const NodeView nd = load_node(nodes, ref);
                if (degen) push_ray_children<true>(nd, p, inv, cull, st, sp);
                else push_ray_children_affine(nd, p, inv, cull, st, sp);
            } else {
                int a, b;
                leaf_range(ref, a, b);
                for (int s = a; s < b && !hit; ++s) {
                    const TriV t = load_tri(tris, s);
                    float tt, terr;
                    const int c = ray_tri_f(p, d, dinf, t, tmaxf, &tt, &terr);
                    if (c == 1) hit = true;
                    else if (c < 0) {
                        double t64;
                        hit = ray_tri_d(to_d3(p), to_d3(d), to_d3(t.a), to_d3(t.b), to_d3(t.c), 1000.0, &t64);
                    }
                }
            }
            if (hit) {
                if (++r == 64) {  // every ray hit: inside
                    dist[idx] = -dist[idx];
                    idx = -1;
                    continue;
                }
                if ((int)r == max_rays) {  // first pass: the rest goes to k_sign_raystab_lines
                    const cooperative_groups::coalesced_group g = cooperative_groups::coalesced_threads();
                    unsigned long long b = 0;
                    if (g.thread_rank() == 0) b = atomicAdd(cand_n, (unsigned long long)g.size());
                    b = g.shfl(b, 0) + g.thread_rank();
                    cand[b] = make_uint4((uint32_t)idx, __float_as_uint(off.x), __float_as_uint(off.y),
                                         (uint32_t)root);
                    idx = -1;
                    continue;
                }
                if (r & 1) d = sd;
                else { sd = stab_dir(r >> 1, off); d = make_float3(-sd.x, -sd.y, -sd.z); }
                inv = ray_inv_approx(d);
                degen = ray_degenerate(inv);
                dinf = f3inf(d);
                sp = 0;
                st[sp++] = root;
            }
        }
        __syncwarp();
    }
}

// Second raystab pass: a warp per candidate query.  The query's rays
// first_ray .. 63 (ray 2k = -d_k, ray 2k + 1 = +d_k, all from the query
// point; the first pass traced the others) form a pool: lane l starts with
// ray first_ray + l and, whenever its ray hits, takes the next ray of the
// pool, so lanes stay busy until the pool is empty.  A ray that finds no hit
// ends the query for the whole warp (__any_sync): the point is outside; when
// the pool is empty and every lane's ray has hit, it is inside.  Each step
// of a lane is one inner node or one triangle, so lanes at inner nodes and
// lanes at leaves run steps of similar length side by side.  The rays of a
// warp start at the same point, so the first levels of their walks read the
// same nodes.  Warps take candidates from a counter in the order the first
// pass appended them (near one another in space).
__global__ void __launch_bounds__(kQBlock, 10) k_sign_raystab_lines(const float* __restrict__ pts,
                                                                float* __restrict__ dist,
                                                                const CNode* __restrict__ nodes,
                                                                const CTri* __restrict__ tris,
                                                                const uint4* __restrict__ cand,
                                                                const unsigned long long* __restrict__ cand_n,
                                                                unsigned long long* __restrict__ next, int first_ray) {
    __shared__ int s_pool[kQBlock / 32];
    __shared__ float3 s_dir[kQBlock / 32][32];   // the query's stab directions d_0 .. d_31
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned long long n = *cand_n;
    const float tmaxf = 1000.0f;
    const float cull = cull_of(1000.0);
    int st[kStack];
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(next, 1ull);
        c = __shfl_sync(kFull, c, 0);
        if (c >= n) break;
        const uint4 e = cand[c];
        const int64_t idx = e.x;
        const float2 off = make_float2(__uint_as_float(e.y), __uint_as_float(e.z));
        const int root = (int)e.w;
        const float3 p = load3(pts, idx);
        if (lane == 0) s_pool[wib] = first_ray + 32;
        s_dir[wib][lane] = stab_dir((uint32_t)lane, off);   // lane k: direction k
        __syncwarp();
        int ray = first_ray + lane;            // >= 64: this lane has no ray left
        float3 d = make_float3(0.f, 0.f, 0.f), inv = d;
        bool degen = false;
        float dinf = 0.f;
        int sp = 0, ls = 0, le = 0;            // stack; triangles [ls, le) of the current leaf
        auto start_ray = [&]() {
            const float3 sd = s_dir[wib][ray >> 1];
            d = (ray & 1) ? sd : make_float3(-sd.x, -sd.y, -sd.z);
            inv = ray_inv_approx(d);
            degen = ray_degenerate(inv);
            dinf = f3inf(d);
            sp = 0;
            st[sp++] = root;
            ls = le = 0;
        };
        if (ray < 64) start_ray();
        bool inside = false;
        while (true) {
            bool miss = false;
            if (ray < 64) {
                bool hit = false;
                if (ls >= le) {
                    if (sp == 0) {
                        miss = true;
                    } else {
                        const int ref = st[--sp];
                        if (ref >= 0) {
                            const NodeView nd = load_node(nodes, ref);
                            if (degen) push_ray_children<true>(nd, p, inv, cull, st, sp);
                            else push_ray_children_affine(nd, p, inv, cull, st, sp);
                        } else {
                            leaf_range(ref, ls, le);
                        }
                    }
                }
                if (ls < le) {                 // one triangle of the current leaf
                    const TriV t = load_tri(tris, ls++);
                    float tt, terr;
                    const int cl = ray_tri_f(p, d, dinf, t, tmaxf, &tt, &terr);
                    if (cl == 1) hit = true;
                    else if (cl < 0) {
                        double t64;
                        hit = ray_tri_d(to_d3(p), to_d3(d), to_d3(t.a), to_d3(t.b), to_d3(t.c), 1000.0, &t64);
                    }
                }
                if (hit) {
                    ray = atomicAdd(&s_pool[wib], 1);
                    if (ray < 64) start_ray();
                }
            }
            if (__any_sync(kFull, miss)) break;            // a stab ray left the mesh: outside
            if (__all_sync(kFull, ray >= 64)) { inside = true; break; }
        }
        if (inside && lane == 0) dist[idx] = -dist[idx];
        __syncwarp();
    }
}

// ---------------------------------------------------------------- rays
constexpr int kUnit = 8;   // rays per unit of the ray packet order (k_ray_order), 4 units per packet
// Ray of `lane` in packet pk: the unit lane / 8 of the packet's four entries
// of order[] (units of 8 consecutive rays); n when there is none.
__device__ __forceinline__ int64_t packet_ray(int64_t pk, int lane, int64_t n, const uint32_t* __restrict__ order) {
    const int64_t units = (n + kUnit - 1) / kUnit;
    const int64_t slot = pk * (32 / kUnit) + lane / kUnit;
    return slot < units ? (int64_t)__ldg(order + slot) * kUnit + lane % kUnit : n;
}
// A packet is traced as a packet only when its rays are nearly parallel
// (unit directions within kCohDir, max-norm, of one another's: about 6
// degrees) and start close together (origins within kCohOrigin of the root
// box's extent), as k_ray_order judges it; the others go to k_ray_lanes,
// where each ray walks alone: the union of 32 unrelated walks costs far more
// than their longest one.
constexpr float kCohDir = 0.1f;
constexpr float kCohOrigin = 0.01f;
// Closest hit of 32 rays per warp (a packet: the rays of 4 consecutive
// entries of `order`, units of 8 consecutive rays sorted so that nearby ones
// are side by side (k_ray_order); packets k_ray_order marked incoherent are
// skipped, k_ray_lanes traces them):
// warp-uniform walk of
// the union of the rays' paths, children in the order of the smallest entry
// distance of any ray that needs them.  Each lane keeps U, an upper bound of
// its closest hit (certain FP32 hits: t + error bound), and a short list of
// triangles that may still be closer (certain or undecided hits whose lower
// bound is within U); the list is settled in double at the end: exact t of
// the closest hit, ties -> lowest face index.
__global__ void __launch_bounds__(kQBlock) k_ray(int64_t n, const uint32_t* __restrict__ order,
                                                 const float* __restrict__ ro,
                                                 const float* __restrict__ rd, float* __restrict__ pos,
                                                 int64_t* __restrict__ face_id, float* __restrict__ depth,
                                                 const CNode* __restrict__ nodes, const CTri* __restrict__ tris,
                                                 unsigned long long* __restrict__ ctr, int64_t grab,
                                                 const uint8_t* __restrict__ skip) {
    const int lane = threadIdx.x & 31;
    __shared__ __align__(16) float s_box[kQBlock / 32][64];
    float* sb = s_box[threadIdx.x >> 5];
    __shared__ int s_sref[kQBlock / 32][kSmemStack];
    __shared__ uint32_t s_skey[kQBlock / 32][kSmemStack];
    PacketQueue pq(ctr, (n + 31) >> 5, grab);
    for (int64_t pk = pq.take(); pk >= 0; pk = pq.take()) {
        if (__ldg(skip + pk)) continue;   // incoherent: k_ray_lanes traces it
        const int64_t q = packet_ray(pk, lane, n, order);
        const bool act = q < n;
        const float3 o = act ? load3(ro, q) : make_float3(0.f, 0.f, 0.f);
        const float3 d = act ? load3(rd, q) : make_float3(1.f, 1.f, 1.f);
        const float3 inv = ray_inv(d);
        const bool degen = __any_sync(kFull, act && ray_degenerate(inv));  // warp-uniform
        const float dinf = f3inf(d);
        const d3 od = to_d3(o), dd = to_d3(d);
        float U = act ? 1000.0f : -1.f;             // MAX_DIST
        float cull = act ? U * 1.000002f : -1.f;
        int cs[kCand];
        float cl[kCand];
        int nc = 0;
        double bt = 1000.0;
        int sx = -1, ix = -1;
        auto flush = [&](bool final_pass) {
            for (int i = 0; i < nc; ++i) {
                if (final_pass && cl[i] > U) continue;
                const TriV t = load_tri(tris, cs[i]);
                double t64;
                if (!ray_tri_d(od, dd, to_d3(t.a), to_d3(t.b), to_d3(t.c), 1000.0, &t64)) continue;
                if (t64 < bt || (t64 == bt && (sx < 0 || t.id < ix))) { bt = t64; sx = cs[i]; ix = t.id; }
            }
            nc = 0;
        };
        uint32_t cullmax = __reduce_max_sync(kFull, __float_as_uint(fmaxf(cull, 0.f)));
        WarpStackSmem st(s_sref[threadIdx.x >> 5], s_skey[threadIdx.x >> 5]);
        int cur = 0;
        bool live = __any_sync(kFull, act);
        while (live) {
            if (cur >= 0) {
                const NodeLinks nd = decode_node_warp(nodes, cur, sb);
                uint32_t k[8];
                if (degen) ray_child_keys<true>(nd, sb, o, inv, cull, k);
                else ray_child_keys<false>(nd, sb, o, inv, cull, k);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t kmin = __reduce_min_sync(kFull, k[j]);
                    k[j] = kmin != kFull ? ((kmin & ~7u) | (uint32_t)j) : kFull;
                }
                sort8(k);
#pragma unroll
                for (int i = 7; i >= 1; --i)
                    if (k[i] != kFull) st.push(child_ref(nd, meta_of(nd, (int)(k[i] & 7u))), k[i] & ~7u);
                if (k[0] != kFull) cur = child_ref(nd, meta_of(nd, (int)(k[0] & 7u)));
                else live = st.next(cullmax, cur);
            } else {
                int s0, s1;
                leaf_range(cur, s0, s1);
                load_leaf_warp(tris, s0, s1, sb);
                for (int s = s0; s < s1; ++s) {
                    const TriV t = warp_tri(sb, s - s0);
                    float tt, terr;
                    const int r = ray_tri_f(o, d, dinf, t, 1000.0f, &tt, &terr);
                    const float lb = tt - terr;
                    if (act && r != 0 && lb <= U) {
                        if (r == 1) U = fminf(U, tt + terr);
                        if (nc == kCand) {
                            int m = 0;
                            for (int i = 0; i < nc; ++i)
                                if (cl[i] <= U) { cs[m] = cs[i]; cl[m] = cl[i]; ++m; }
                            nc = m;
                            if (nc == kCand) {
                                flush(false);
                                if (sx >= 0) U = fminf(U, __double2float_ru(bt));
                            }
                        }
                        cs[nc] = s; cl[nc] = lb; ++nc;
                    }
                }
                cull = act ? U * 1.000002f : -1.f;
                cullmax = __reduce_max_sync(kFull, __float_as_uint(fmaxf(cull, 0.f)));
                live = st.next(cullmax, cur);
            }
        }
        if (!act) continue;
        flush(true);
        depth[q] = __double2float_rn(bt);
        pos[3 * q] = __double2float_rn(dA((double)o.x, dM(bt, (double)d.x)));
        pos[3 * q + 1] = __double2float_rn(dA((double)o.y, dM(bt, (double)d.y)));
        pos[3 * q + 2] = __double2float_rn(dA((double)o.z, dM(bt, (double)d.z)));
        face_id[q] = sx >= 0 ? (int64_t)ix : (int64_t)-1;
    }
}

// ------------------------------------------------------ Morton bucketing
// Points are counted into 2^(3b) cells of their own bounding box (computed
// on the device) and scattered in Morton order of the cells.  Within a cell
// the order is that of the atomics (irrelevant: results are per query).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// order-preserving float <-> uint32 map (for atomicMin / atomicMax)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}
__global__ void k_box_init(uint32_t* box) {
    if (threadIdx.x < 3) box[threadIdx.x] = 0xFFFFFFFFu;
    else if (threadIdx.x < 6) box[threadIdx.x] = 0u;
}
__global__ void k_box(int64_t n, const float* __restrict__ pts, uint32_t* __restrict__ box) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float3 p = load3(pts, i);
        const float c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (isfinite(c[k])) { lo[k] = min(lo[k], f2o(c[k])); hi[k] = max(hi[k], f2o(c[k])); }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = __reduce_min_sync(kFull, lo[k]);
        hi[k] = __reduce_max_sync(kFull, hi[k]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { atomicMin(&box[k], lo[k]); atomicMax(&box[3 + k], hi[k]); }
    }
}
__device__ __forceinline__ uint32_t cell_of(float3 p, const uint32_t* __restrict__ box, int bits) {
    const float side = (float)(1 << bits), m = side - 1.f;
    const float c[3] = {p.x, p.y, p.z};
    uint32_t g[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float lo = o2f(box[k]), hi = o2f(box[3 + k]);
        const float s = hi > lo ? side / (hi - lo) : 0.f;
        const float v = (c[k] - lo) * s;
        g[k] = (uint32_t)fminf(fmaxf(v == v ? v : 0.f, 0.f), m);
    }
    return spread3(g[0]) | (spread3(g[1]) << 1) | (spread3(g[2]) << 2);
}
__global__ void k_cell_hist(int64_t n, const float* __restrict__ pts, const uint32_t* __restrict__ box, int bits,
                            uint32_t* __restrict__ hist) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        atomicAdd(&hist[cell_of(load3(pts, i), box, bits)], 1u);
}
__global__ void k_cell_scatter(int64_t n, const float* __restrict__ pts, const uint32_t* __restrict__ box, int bits,
                               uint32_t* __restrict__ offs, uint32_t* __restrict__ order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        order[atomicAdd(&offs[cell_of(load3(pts, i), box, bits)], 1u)] = (uint32_t)i;
}

// Closest hit of the rays of the incoherent packets k_ray listed: a warp
// takes a packet, and each lane walks its own ray alone (own stack in local
// memory, children nearest first, a child popped only while its entry
// distance is within the lane's bound U).  A step is one node or one leaf.
// Filters, candidate list and the FP64 settlement are k_ray's, so every
// result is the one k_ray would give.
__global__ void __launch_bounds__(kQBlock) k_ray_lanes(int64_t n, const uint32_t* __restrict__ order,
                                                       const float* __restrict__ ro, const float* __restrict__ rd,
                                                       float* __restrict__ pos, int64_t* __restrict__ face_id,
                                                       float* __restrict__ depth, const CNode* __restrict__ nodes,
                                                       const CTri* __restrict__ tris,
                                                       const uint32_t* __restrict__ lanes,
                                                       const unsigned long long* __restrict__ lanes_n,
                                                       unsigned long long* __restrict__ next) {
    const int lane = threadIdx.x & 31;
    const unsigned long long count = *lanes_n;
    int st_ref[kStack];
    uint32_t st_key[kStack];
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(next, 1ull);
        c = __shfl_sync(kFull, c, 0);
        if (c >= count) break;
        const int64_t q = packet_ray((int64_t)lanes[c], lane, n, order);
        const bool act = q < n;
        const float3 o = act ? load3(ro, q) : make_float3(0.f, 0.f, 0.f);
        const float3 d = act ? load3(rd, q) : make_float3(1.f, 1.f, 1.f);
        const float3 inv = ray_inv(d);
        const bool degen = ray_degenerate(inv);
        const float dinf = f3inf(d);
        const d3 od = to_d3(o), dd = to_d3(d);
        float U = 1000.0f;                          // MAX_DIST
        float cull = U * 1.000002f;
        int cs[kCand];
        float cl[kCand];
        int nc = 0;
        double bt = 1000.0;
        int sx = -1, ix = -1;
        auto flush = [&](bool final_pass) {
            for (int i = 0; i < nc; ++i) {
                if (final_pass && cl[i] > U) continue;
                const TriV t = load_tri(tris, cs[i]);
                double t64;
                if (!ray_tri_d(od, dd, to_d3(t.a), to_d3(t.b), to_d3(t.c), 1000.0, &t64)) continue;
                if (t64 < bt || (t64 == bt && (sx < 0 || t.id < ix))) { bt = t64; sx = cs[i]; ix = t.id; }
            }
            nc = 0;
        };
        int sp = 0, cur = 0;
        bool live = act;
        while (live) {
            if (cur >= 0) {
                const NodeView nd = load_node(nodes, cur);
                uint32_t k[8];
                lane_child_keys(nd, o, inv, degen, cull, k);
                sort8(k);
#pragma unroll
                for (int i = 7; i >= 1; --i)
                    if (k[i] != kFull) { st_ref[sp] = child_ref(nd, meta_of(nd, (int)(k[i] & 7u))); st_key[sp] = k[i] & ~7u; ++sp; }
                if (k[0] != kFull) { cur = child_ref(nd, meta_of(nd, (int)(k[0] & 7u))); continue; }
            } else {
                int s0, s1;
                leaf_range(cur, s0, s1);
                for (int s = s0; s < s1; ++s) {
                    const TriV t = load_tri(tris, s);
                    float tt, terr;
                    const int r = ray_tri_f(o, d, dinf, t, 1000.0f, &tt, &terr);
                    const float lb = tt - terr;
                    if (r != 0 && lb <= U) {
                        if (r == 1) U = fminf(U, tt + terr);
                        if (nc == kCand) {
                            int m = 0;
                            for (int i = 0; i < nc; ++i)
                                if (cl[i] <= U) { cs[m] = cs[i]; cl[m] = cl[i]; ++m; }
                            nc = m;
                            if (nc == kCand) {
                                flush(false);
                                if (sx >= 0) U = fminf(U, __double2float_ru(bt));
                            }
                        }
                        cs[nc] = s; cl[nc] = lb; ++nc;
                    }
                }
                cull = U * 1.000002f;
            }
            live = false;             // the next entry whose box is still within the bound
            while (sp > 0) {
                --sp;
                if (__uint_as_float(st_key[sp]) <= cull) { cur = st_ref[sp]; live = true; break; }
            }
        }
        if (!act) continue;
        flush(true);
        depth[q] = __double2float_rn(bt);
        pos[3 * q] = __double2float_rn(dA((double)o.x, dM(bt, (double)d.x)));
        pos[3 * q + 1] = __double2float_rn(dA((double)o.y, dM(bt, (double)d.y)));
        pos[3 * q + 2] = __double2float_rn(dA((double)o.z, dM(bt, (double)d.z)));
        face_id[q] = sx >= 0 ? (int64_t)ix : (int64_t)-1;
    }
}

// ---------------------------------------------------------- ray windows
// Packet order of rays.  Rays are taken in units of kUnit consecutive rays,
// and each window of kOrdUnits consecutive units is sorted by the Morton
// code of the point where one ray of the unit (its fourth) enters the root
// node's box (its origin when it starts inside), on cells of one size on all
// three axes (the window's largest extent / 1024); units whose ray misses
// the box go after the others, in the Morton order of where that ray passes
// closest to the box centre (clamped into the cells), then the window's tail
// past the last unit.  A packet is four consecutive units of the sorted
// order.  Camera rays stored row by row then make packets of 8 pixels from
// each of 4 neighbouring rows instead of 32 x 1 strips, and the union of the
// 32 rays' walks visits far fewer nodes (C1 camera rays: k_ray 6.4 -> 5.1
// ms, for a sort of 1,024 keys per 8,192 rays).  The order changes no
// result: each ray's hit is its own.
constexpr int kOrdThreads = 256, kOrdItems = 4;
constexpr int kOrdUnits = kOrdThreads * kOrdItems;    // 1024 units = 8192 rays per window
// Entry point of ray (o, d) into the box [lo, lo + 255 * 2^ex] (the origin when
// the ray starts inside; non-finite coordinates become 0): 0, or 1 when the
// ray misses the box (e = the point where it passes closest to the box
// centre, for t >= 0).
__device__ __forceinline__ int ray_entry(float3 o, float3 d, const float lo[3], const int ex[3], float e[3]) {
    const float oc[3] = {o.x, o.y, o.z}, dc[3] = {d.x, d.y, d.z};
    float tn = 0.f, tf = CUDART_INF_F;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float hi = fmaf(255.f, exp2i(ex[k]), lo[k]);
        const float inv = 1.f / dc[k];
        const float ta = (lo[k] - oc[k]) * inv, tb = (hi - oc[k]) * inv;
        tn = fmaxf(tn, fminf(ta, tb));   // NaN (0 * inf) leaves the bound as it was
        tf = fminf(tf, fmaxf(ta, tb));
    }
    const int miss = tn <= tf ? 0 : 1;
    if (miss) {                       // where the ray passes closest to the box centre
        float cd = 0.f, dd = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (lo[k] + fmaf(255.f, exp2i(ex[k]), lo[k]));
            cd = fmaf(c - oc[k], dc[k], cd);
            dd = fmaf(dc[k], dc[k], dd);
        }
        tn = fmaxf(cd / dd, 0.f);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = fmaf(dc[k], tn, oc[k]);
        e[k] = isfinite(v) ? v : 0.f;
    }
    return miss;
}
// One block per window: entry points of the units' rays, the box of those
// that enter, Morton keys, a block radix sort of (key, unit in the window),
// and the sorted unit indices written to order[].  Then each packet of the
// window (4 consecutive sorted units) is judged: coherent when each unit's
// first and last rays lie within kCohDir (unit directions, max-norm) and
// kCohOrigin (origins) of the unit's fourth ray, and each unit's fourth ray
// within the same of the first unit's.  skip[p] = 1 marks the others for
// k_ray, and they are listed for k_ray_lanes.
__global__ void __launch_bounds__(kOrdThreads) k_ray_order(int64_t n, const float* __restrict__ ro,
                                                           const float* __restrict__ rd,
                                                           const CNode* __restrict__ nodes,
                                                           uint32_t* __restrict__ order, uint8_t* __restrict__ skip,
                                                           uint32_t* __restrict__ lanes,
                                                           unsigned long long* __restrict__ lanes_n) {
    using Sort = cub::BlockRadixSort<uint32_t, kOrdThreads, kOrdItems, uint16_t>;
    __shared__ typename Sort::TempStorage s_sort;
    __shared__ uint32_t s_box[6];
    __shared__ float s_ray[kOrdUnits][6];     // each unit's fourth ray: unit direction, origin
    __shared__ uint8_t s_bad[kOrdUnits];       // the unit's first or last ray strays from its fourth
    __shared__ uint16_t s_sorted[kOrdUnits];
    const int64_t units = (n + kUnit - 1) / kUnit;
    const int64_t u0 = (int64_t)blockIdx.x * kOrdUnits;
    const int t = threadIdx.x;
    if (t < 3) s_box[t] = 0xFFFFFFFFu;
    else if (t < 6) s_box[t] = 0u;
    const NodeView root = load_node(nodes, 0);
    const float blo[3] = {root.ox, root.oy, root.oz};
    const int bex[3] = {nodes[0].ex, nodes[0].ey, nodes[0].ez};
    const float spread_max = kCohOrigin * 255.f * fmaxf(fmaxf(root.sx, root.sy), root.sz);
    float ep[kOrdItems][3];
    int kind[kOrdItems];              // 0 enters the box, 1 misses it, 2 past the last unit
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
#pragma unroll
    for (int i = 0; i < kOrdItems; ++i) {
        const int li = i * kOrdThreads + t;
        const int64_t u = u0 + li;
        kind[i] = 2;
        ep[i][0] = ep[i][1] = ep[i][2] = 0.f;
        if (u >= units) continue;
        const int64_t q = min(u * kUnit + kUnit / 2 - 1, n - 1);
        const float3 o = load3(ro, q), d = load3(rd, q);
        kind[i] = ray_entry(o, d, blo, bex, ep[i]);
        if (kind[i] == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) { lo[k] = min(lo[k], f2o(ep[i][k])); hi[k] = max(hi[k], f2o(ep[i][k])); }
        }
        const float il = rsqrtf(f3dot(d, d));
        const float3 v = make_float3(d.x * il, d.y * il, d.z * il);
        bool bad = false;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t qe = e == 0 ? u * kUnit : min(u * kUnit + kUnit - 1, n - 1);
            const float3 oe = load3(ro, qe), de = load3(rd, qe);
            const float ie = rsqrtf(f3dot(de, de));
            const float3 ve = make_float3(de.x * ie, de.y * ie, de.z * ie);
            bad |= !(f3inf(f3sub(ve, v)) <= kCohDir && f3inf(f3sub(oe, o)) <= spread_max);   // NaN: bad
        }
        s_ray[li][0] = v.x; s_ray[li][1] = v.y; s_ray[li][2] = v.z;
        s_ray[li][3] = o.x; s_ray[li][4] = o.y; s_ray[li][5] = o.z;
        s_bad[li] = bad || !(f3inf(v) <= 2.f);   // a non-finite (or zero) fourth direction: bad
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = __reduce_min_sync(kFull, lo[k]);
        hi[k] = __reduce_max_sync(kFull, hi[k]);
    }
    __syncthreads();                  // s_box initialised
    if ((t & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { atomicMin(&s_box[k], lo[k]); atomicMax(&s_box[3 + k], hi[k]); }
    }
    __syncthreads();
    float wlo[3], ext = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        wlo[k] = o2f(s_box[k]);
        ext = fmaxf(ext, o2f(s_box[3 + k]) - wlo[k]);   // no entry point: the box is empty, ext stays 0
    }
    const float sc = ext > 0.f ? 1024.f / ext : 0.f;
    uint32_t key[kOrdItems];
    uint16_t val[kOrdItems];
#pragma unroll
    for (int i = 0; i < kOrdItems; ++i) {
        val[i] = (uint16_t)(i * kOrdThreads + t);
        if (kind[i] == 2) { key[i] = 0x80000000u; continue; }
        uint32_t g[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) g[k] = (uint32_t)fminf(fmaxf((ep[i][k] - wlo[k]) * sc, 0.f), 1023.f);
        key[i] = spread3(g[0]) | (spread3(g[1]) << 1) | (spread3(g[2]) << 2) | (kind[i] == 1 ? 0x40000000u : 0u);
    }
    Sort(s_sort).SortBlockedToStriped(key, val, 0, 32);
#pragma unroll
    for (int i = 0; i < kOrdItems; ++i) {
        const int rank = i * kOrdThreads + t;            // rank of the window
        s_sorted[rank] = val[i];
        if (u0 + rank < units) order[u0 + rank] = (uint32_t)(u0 + val[i]);
    }
    __syncthreads();
    // packet t of the window: sorted units 4t .. 4t + 3
    const int64_t pk = (int64_t)blockIdx.x * (kOrdUnits / 4) + t;
    const bool valid = u0 + 4 * t < units;
    bool inc = false;
    if (valid) {
        const int f = s_sorted[4 * t];
        inc = s_bad[f];
        for (int j = 1; j < 4 && u0 + 4 * t + j < units; ++j) {
            const int v = s_sorted[4 * t + j];
            float dv = 0.f, dov = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                dv = fmaxf(dv, fabsf(s_ray[v][k] - s_ray[f][k]));
                dov = fmaxf(dov, fabsf(s_ray[v][3 + k] - s_ray[f][3 + k]));
            }
            inc |= s_bad[v] || !(dv <= kCohDir && dov <= spread_max);
        }
        skip[pk] = inc ? 1 : 0;
    }
    const unsigned m = __ballot_sync(kFull, valid && inc);
    if (m) {                          // one atomic per warp
        unsigned long long base = 0;
        if ((t & 31) == __ffs(m) - 1) base = atomicAdd(lanes_n, (unsigned long long)__popc(m));
        base = __shfl_sync(kFull, base, __ffs(m) - 1);
        if (valid && inc) lanes[base + __popc(m & ((1u << (t & 31)) - 1u))] = (uint32_t)pk;
    }
}

// --------------------------------------------------------------- launchers
namespace {

int sm_count() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}
template <class K>
unsigned persistent_grid(K kernel, int64_t n) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kQBlock, 0);
    if (per_sm < 1) per_sm = 1;
    const int64_t want = (n + kQBlock - 1) / kQBlock;
    const int64_t cap = (int64_t)sm_count() * per_sm;
    return (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
}

int cell_bits(int64_t n) {
    int b = 4;
    while (b < 8 && ((int64_t)1 << (3 * (b + 1))) <= 2 * n) ++b;
    return b;
}

}  // namespace

// Heavy-query list length for n queries: a 32nd of them (at least 32768, at
// most n); a full list only means packets finish in place.
int64_t heavy_cap_for(int64_t n) {
    const int64_t c = n / 32 > 32768 ? n / 32 : 32768;
    return c < n ? c : n;
}

namespace {
// launches with fewer packets per warp run k_udf with tail control
constexpr float kTailPpw = 24.f;
// packets per warp of a launch
float packets_per_warp(int64_t packets, unsigned grid) {
    return (float)packets / (float)((int64_t)grid * (kQBlock / 32));
}
}  // namespace

namespace {
// Ray launch workspace: counters (256 bytes), the unit order, a skip flag
// per packet, the list of incoherent packets; byte offsets and total.
struct RayWs { size_t order, skip, lanes, end; };
RayWs ray_ws(int64_t n) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t units = (size_t)((n + kUnit - 1) / kUnit), packets = (size_t)((n + 31) / 32);
    RayWs r;
    r.order = 256;
    r.skip = r.order + al(sizeof(uint32_t) * units);
    r.lanes = r.skip + al(packets);
    r.end = r.lanes + al(sizeof(uint32_t) * packets);
    return r;
}
}  // namespace

size_t query_workspace_bytes(int mode, int64_t n) {
    size_t b = 256;                                               // packet counters
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    if (mode >= 0 && n >= kSortMinQueries) {
        const int64_t cells = (int64_t)1 << (3 * cell_bits(n));
        b += al(sizeof(uint32_t) * n);                            // order
        b += al(sizeof(uint32_t) * (cells + 1));                  // cell counts / offsets
        b += al(sizeof(uint32_t) * (scan::num_chunks(cells) + 1));
        b += al(sizeof(uint32_t) * 8);                            // query box
    }
    if (mode > 0) b += al(sizeof(int32_t) * n);                   // winning slots
    if (mode == 1) b += al(sizeof(uint32_t) * n);                 // watertight overflow queue
    if (mode >= 0) b += al(sizeof(uint2) * heavy_cap_for(n));     // heavy-query list
    if (mode == 2) b += al(sizeof(uint4) * n);                    // raystab candidates (second pass)
    if (mode == -1) b = ray_ws(n).end;                           // unit order, skip flags, incoherent packets
    return b;
}

namespace {
// Slots of the 256-byte counter block at the head of a launch's workspace
// (32 uint64, zeroed at the start of every launch); each has one user.
enum : int {
    kCtUdf = 0,         // k_udf packet queue
    kCtSign = 1,        // sign-pass packet queue (watertight, or the first raystab pass of a single BVH)
    kCtArenaRs = 2,     // first raystab pass of an arena (its watertight pass takes kCtSign)
    kCtHeavyN = 6,      // heavy-query list length
    kCtHeavyNext = 7,   // k_udf_heavy queue
    kCtStats = 8,       // k_udf tail statistics: node + leaf visits (8), packets finished (9)
    kCtOvfN = 10,       // watertight overflow queue length
    kCtCandN = 12,      // raystab second-pass candidates
    kCtLinesNext = 13,  // raystab second-pass queue
    kCtRayLanesN = 14,  // incoherent ray packets listed by k_ray
    kCtRayLanesNext = 15,  // k_ray_lanes queue
};
// packets per atomic grab: about 64 grabs per warp of the launch
int64_t grab_for(int64_t n, unsigned grid) {
    const int64_t packets = (n + 31) / 32;
    const int64_t warps = (int64_t)grid * (kQBlock / 32);
    const int64_t g = packets / (warps * 64);
    return g < 1 ? 1 : g;
}
// Launch shape of a yielding launch (PacketQueue block budget): kYieldWaves
// times the persistent grid g, each block taking at most block_grabs grabs,
// twice the queue's grabs in all, so the queue is always drained (a warp
// stops only when its block's budget is spent or the queue is empty) and a
// block lives for about 1 / (kYieldWaves / 2) of the launch.  off: the
// persistent launch (g blocks, no budget).
constexpr unsigned kYieldWaves = 4;  // measured against 8 and 16
struct LaunchShape { unsigned grid; int block_grabs; };
LaunchShape yield_shape(unsigned g, int64_t n, int64_t grab, bool on) {
    if (!on) return {g, 0};
    const int64_t grabs = ((n + 31) / 32 + grab - 1) / grab;
    int64_t G = (int64_t)g * kYieldWaves;
    if (G > 2 * grabs) G = 2 * grabs > 0 ? 2 * grabs : 1;
    const int64_t bg = (2 * grabs + G - 1) / G;
    return {(unsigned)G, (int)(bg > 0 ? bg : 1)};
}
// raystab chunk: kChunkMax packets (64 queries for 32 lanes: a lane whose
// query ends early takes another one; larger chunks cost more in lane-by-lane
// query setup than they save), one packet when the launch has fewer than two
// packets per warp
int64_t chunk_for(int64_t n, unsigned grid) {
    const int64_t packets = (n + 31) / 32;
    const int64_t warps = (int64_t)grid * (kQBlock / 32);
    return packets >= (int64_t)kChunkMax * warps ? kChunkMax : 1;
}
}  // namespace

namespace {
// Rays the first raystab pass traces per query before handing the query to
// the second pass (a line of two rays per stab direction).
constexpr int kRaystabFirstRays = 2;
// The two raystab passes over the packets of `w` (n queries): counters ctr
// (first pass), cand_n (candidates appended), lines_next (second-pass
// queue); cand holds up to n candidates.
void launch_raystab(const Work& w, int64_t n, const uint32_t* order, const float* pts, float* dist,
                    const CNode* nodes, const CTri* tris, unsigned long long* ctr, uint4* cand,
                    unsigned long long* cand_n, unsigned long long* lines_next, cudaStream_t stream) {
    const unsigned g = persistent_grid(k_sign_raystab, n);
    k_sign_raystab<<<g, kQBlock, 0, stream>>>(w, order, pts, dist, nodes, tris, ctr, chunk_for(n, g),
                                              kRaystabFirstRays, cand, cand_n); count_launch();
    const unsigned g2 = persistent_grid(k_sign_raystab_lines, n);
    k_sign_raystab_lines<<<g2, kQBlock, 0, stream>>>(pts, dist, nodes, tris, cand, cand_n, lines_next,
                                                     kRaystabFirstRays); count_launch();
}
}  // namespace

cudaError_t launch_distance(int mode, bool want_uvw, int64_t n, const float* pts, float* dist, int64_t* fid,
                            float* uvw, const CNode* nodes, const CTri* tris, int slot_face0, NearLists near,
                            void* ws, cudaStream_t stream, int64_t qbase, bool yield) {
    if (n <= 0) return cudaSuccess;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    char* w = static_cast<char*>(ws);
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(w); w += 256;
    cudaError_t e = cudaMemsetAsync(ctr, 0, 256, stream);
    if (e != cudaSuccess) return e;
    uint32_t* order = nullptr;
    if (n >= kSortMinQueries) {
        const int bits = cell_bits(n);
        const int64_t cells = (int64_t)1 << (3 * bits);
        order = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * n);
        uint32_t* hist = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * (cells + 1));
        uint32_t* bsum = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * (scan::num_chunks(cells) + 1));
        uint32_t* box = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * 8);
        if ((e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (cells + 1), stream)) != cudaSuccess) return e;
        const unsigned g = (unsigned)sm_count() * 8;
        k_box_init<<<1, 32, 0, stream>>>(box); count_launch();
        k_box<<<g, 256, 0, stream>>>(n, pts, box); count_launch();
        k_cell_hist<<<g, 256, 0, stream>>>(n, pts, box, bits, hist); count_launch();
        scan::exclusive(hist, bsum, cells, stream);
        k_cell_scatter<<<g, 256, 0, stream>>>(n, pts, box, bits, hist, order); count_launch();
    }
    int32_t* slots = mode != 0 ? reinterpret_cast<int32_t*>(w) : nullptr;
    if (mode != 0) w += al(sizeof(int32_t) * n);
    uint32_t* ovf = mode == 1 ? reinterpret_cast<uint32_t*>(w) : nullptr;
    if (mode == 1) w += al(sizeof(uint32_t) * n);
    uint2* heavy = reinterpret_cast<uint2*>(w);
    const int64_t hcap = heavy_cap_for(n);
    w += al(sizeof(uint2) * hcap);
    const Work work{nullptr, nullptr, n, slot_face0, qbase};
#define CUBVH_L(U, S) do { const unsigned g_ = persistent_grid(k_udf<U, S, false>, n); \
        const float ppw_ = packets_per_warp((n + 31) / 32, g_); \
        if (ppw_ >= kTailPpw) { \
            const LaunchShape y_ = yield_shape(g_, n, grab_for(n, g_), yield); \
            k_udf<U, S, false><<<y_.grid, kQBlock, 0, stream>>>(work, order, pts, dist, fid, uvw, slots, nodes, tris, \
                                                           ctr + kCtUdf, grab_for(n, g_), heavy, ctr + kCtHeavyN, hcap, ctr + kCtStats, ppw_, \
                                                           y_.block_grabs); count_launch(); \
        } else { \
            const unsigned gt_ = persistent_grid(k_udf<U, S, true>, n); \
            const LaunchShape y_ = yield_shape(gt_, n, grab_for(n, gt_), yield); \
            k_udf<U, S, true><<<y_.grid, kQBlock, 0, stream>>>(work, order, pts, dist, fid, uvw, slots, nodes, tris, \
                                                           ctr + kCtUdf, grab_for(n, gt_), heavy, ctr + kCtHeavyN, hcap, ctr + kCtStats, \
                                                           packets_per_warp((n + 31) / 32, gt_), y_.block_grabs); count_launch(); \
            const unsigned gh_ = persistent_grid(k_udf_heavy<U, S>, 32 * hcap); \
            k_udf_heavy<U, S><<<gh_, kQBlock, 0, stream>>>(heavy, ctr + kCtHeavyN, hcap, nullptr, slot_face0, pts, dist, \
                                                           fid, uvw, slots, nodes, tris, ctr + kCtHeavyNext); count_launch(); \
        } } while (0)
    if (mode == 0) { if (want_uvw) CUBVH_L(true, false); else CUBVH_L(false, false); }
    else { if (want_uvw) CUBVH_L(true, true); else CUBVH_L(false, true); }
#undef CUBVH_L
    if (mode == 1) {
        if (near.cnt) {
            const unsigned g = persistent_grid(k_sign_watertight<true>, n);
            const LaunchShape y = yield_shape(g, n, grab_for(n, g), yield);
            k_sign_watertight<true><<<y.grid, kQBlock, 0, stream>>>(work, order, pts, dist, slots, nodes, tris, near, ovf,
                                                                    ctr + kCtOvfN, ctr + kCtSign, grab_for(n, g),
                                                                    y.block_grabs); count_launch();
            if (near.ovf) {
                const unsigned go = persistent_grid(k_sign_watertight_ovf, n);
                k_sign_watertight_ovf<<<go, kQBlock, 0, stream>>>(ovf, ctr + kCtOvfN, pts, dist, slots, nodes, tris); count_launch();
            }
        } else {
            const unsigned g = persistent_grid(k_sign_watertight<false>, n);
            const LaunchShape y = yield_shape(g, n, grab_for(n, g), yield);
            k_sign_watertight<false><<<y.grid, kQBlock, 0, stream>>>(work, order, pts, dist, slots, nodes, tris, near,
                                                                     nullptr, nullptr, ctr + kCtSign, grab_for(n, g),
                                                                     y.block_grabs); count_launch();
        }
    } else if (mode == 2) {
        uint4* cand = reinterpret_cast<uint4*>(w);
        launch_raystab(work, n, order, pts, dist, nodes, tris, ctr + kCtSign, cand, ctr + kCtCandN, ctr + kCtLinesNext,
                       stream);
    }
    return cudaGetLastError();
}

cudaError_t launch_near_lists(int64_t n_tris, const CNode* nodes, const CTri* tris, int32_t* cnt, int32_t* lst,
                              double* nrm, int* any_ovf, cudaStream_t stream) {
    if (n_tris <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(any_ovf, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    const unsigned g = persistent_grid(k_near_lists, n_tris);
    k_near_lists<<<g, kQBlock, 0, stream>>>(n_tris, nodes, tris, 0, cnt, lst, nrm, any_ovf); count_launch();
    return cudaGetLastError();
}

cudaError_t launch_ray(int64_t n, const float* ro, const float* rd, float* pos, int64_t* fid, float* depth,
                       const CNode* nodes, const CTri* tris, void* ws, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(ws);
    cudaError_t e = cudaMemsetAsync(ctr, 0, 256, stream);
    if (e != cudaSuccess) return e;
    const RayWs r = ray_ws(n);
    char* w = static_cast<char*>(ws);
    uint32_t* order = reinterpret_cast<uint32_t*>(w + r.order);
    uint8_t* skip = reinterpret_cast<uint8_t*>(w + r.skip);
    uint32_t* lanes = reinterpret_cast<uint32_t*>(w + r.lanes);
    const int64_t units = (n + kUnit - 1) / kUnit;
    k_ray_order<<<(unsigned)((units + kOrdUnits - 1) / kOrdUnits), kOrdThreads, 0, stream>>>(
        n, ro, rd, nodes, order, skip, lanes, ctr + kCtRayLanesN); count_launch();
    const unsigned g = persistent_grid(k_ray, n);
    k_ray<<<g, kQBlock, 0, stream>>>(n, order, ro, rd, pos, fid, depth, nodes, tris, ctr + kCtUdf, grab_for(n, g),
                                     skip); count_launch();
    const unsigned gl = persistent_grid(k_ray_lanes, n);
    k_ray_lanes<<<gl, kQBlock, 0, stream>>>(n, order, ro, rd, pos, fid, depth, nodes, tris, lanes,
                                            ctr + kCtRayLanesN, ctr + kCtRayLanesNext); count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------ arena
// Query -> mesh: binary search over the meshes' first query indices.
__device__ __forceinline__ int mesh_of(const int64_t* __restrict__ qoff, int M, int64_t i) {
    int lo = 0, hi = M - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (qoff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ uint32_t arena_cell(float3 p, const ArenaSortDesc& s) {
    const float side = (float)(1 << s.bits), m = side - 1.f;
    const float c[3] = {p.x, p.y, p.z};
    uint32_t g[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sc = s.hi[k] > s.lo[k] ? side / (s.hi[k] - s.lo[k]) : 0.f;
        const float v = (c[k] - s.lo[k]) * sc;
        g[k] = (uint32_t)fminf(fmaxf(v == v ? v : 0.f, 0.f), m);
    }
    return (uint32_t)s.cell_off + (spread3(g[0]) | (spread3(g[1]) << 1) | (spread3(g[2]) << 2));
}
__global__ void k_arena_hist(int64_t n, const float* __restrict__ pts, const int64_t* __restrict__ qoff, int M,
                             const ArenaSortDesc* __restrict__ sd, uint32_t* __restrict__ hist) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        atomicAdd(&hist[arena_cell(load3(pts, i), sd[mesh_of(qoff, M, i)])], 1u);
}
__global__ void k_arena_scatter(int64_t n, const float* __restrict__ pts, const int64_t* __restrict__ qoff, int M,
                                const ArenaSortDesc* __restrict__ sd, uint32_t* __restrict__ offs,
                                uint32_t* __restrict__ order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        order[atomicAdd(&offs[arena_cell(load3(pts, i), sd[mesh_of(qoff, M, i)])], 1u)] = (uint32_t)i;
}

cudaError_t launch_arena_distance(const ArenaLaunch& a, const float* pts, float* dist, int64_t* fid, float* uvw,
                                  cudaStream_t stream) {
    if (a.n_queries <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(a.counters, 0, 256, stream);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.hist, 0, sizeof(uint32_t) * (a.n_cells + 1), stream)) != cudaSuccess) return e;
    const unsigned g = (unsigned)sm_count() * 8;
    k_arena_hist<<<g, 256, 0, stream>>>(a.n_queries, pts, a.qoff, a.n_meshes, a.sort, a.hist); count_launch();
    scan::exclusive(a.hist, a.bsum, a.n_cells, stream);
    k_arena_scatter<<<g, 256, 0, stream>>>(a.n_queries, pts, a.qoff, a.n_meshes, a.sort, a.hist, a.order); count_launch();
    const bool signed_any = a.n_wt_packets > 0 || a.n_rs_packets > 0;
    const Work all{a.packets, a.meshes, a.n_packets, 0};
#define CUBVH_L(U, S) do { const unsigned g_ = persistent_grid(k_udf<U, S, false>, a.n_queries); \
        const float ppw_ = packets_per_warp(a.n_packets, g_); \
        if (ppw_ >= kTailPpw) { \
            k_udf<U, S, false><<<g_, kQBlock, 0, stream>>>(all, a.order, pts, dist, fid, uvw, a.slots, a.nodes, \
                                                           a.tris, a.counters + kCtUdf, grab_for(a.n_queries, g_), a.heavy, \
                                                           a.counters + kCtHeavyN, a.heavy_cap, a.counters + kCtStats, ppw_, 0); count_launch(); \
        } else { \
            const unsigned gt_ = persistent_grid(k_udf<U, S, true>, a.n_queries); \
            k_udf<U, S, true><<<gt_, kQBlock, 0, stream>>>(all, a.order, pts, dist, fid, uvw, a.slots, a.nodes, \
                                                           a.tris, a.counters + kCtUdf, grab_for(a.n_queries, gt_), a.heavy, \
                                                           a.counters + kCtHeavyN, a.heavy_cap, a.counters + kCtStats, \
                                                           packets_per_warp(a.n_packets, gt_), 0); count_launch(); \
            const unsigned gh_ = persistent_grid(k_udf_heavy<U, S>, 32 * a.heavy_cap); \
            k_udf_heavy<U, S><<<gh_, kQBlock, 0, stream>>>(a.heavy, a.counters + kCtHeavyN, a.heavy_cap, a.meshes, 0, pts, \
                                                           dist, fid, uvw, a.slots, a.nodes, a.tris, \
                                                           a.counters + kCtHeavyNext); count_launch(); \
        } } while (0)
    if (uvw) { if (signed_any) CUBVH_L(true, true); else CUBVH_L(true, false); }
    else { if (signed_any) CUBVH_L(false, true); else CUBVH_L(false, false); }
#undef CUBVH_L
    if (a.n_wt_packets > 0) {
        const Work w{a.wt_packets, a.meshes, a.n_wt_packets, 0};
        const unsigned gw = persistent_grid(k_sign_watertight<false>, 32 * a.n_wt_packets);
        k_sign_watertight<false><<<gw, kQBlock, 0, stream>>>(w, a.order, pts, dist, a.slots, a.nodes, a.tris,
                                                             NearLists{}, nullptr, nullptr, a.counters + kCtSign,
                                                             grab_for(32 * a.n_wt_packets, gw), 0); count_launch();
    }
    if (a.n_rs_packets > 0) {
        const Work w{a.rs_packets, a.meshes, a.n_rs_packets, 0};
        launch_raystab(w, 32 * a.n_rs_packets, a.order, pts, dist, a.nodes, a.tris, a.counters + kCtArenaRs,
                       a.rs_cand, a.counters + kCtCandN, a.counters + kCtLinesNext, stream);
    }
    return cudaGetLastError();
}

int cell_bits_for(int64_t n) { return cell_bits(n); }

// The raystab stab directions of queries first .. first+n-1 (inspection):
// dirs[(i * 32 + k) * 3 + c], the same stab_dir values the sign pass uses.
__global__ void k_stab_dirs(int64_t n, uint32_t first, float* __restrict__ dirs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 off = stab_offset(first + (uint32_t)i);
    float* o = dirs + i * 96;
    for (uint32_t k = 0; k < 32; ++k) {
        const float3 d = stab_dir(k, off);
        o[3 * k] = d.x;
        o[3 * k + 1] = d.y;
        o[3 * k + 2] = d.z;
    }
}

cudaError_t launch_stab_dirs(int64_t first, int64_t n, float* dirs, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_stab_dirs<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(n, (uint32_t)first, dirs); count_launch();
    return cudaGetLastError();
}

cudaError_t upload_constants() {
    float lat[64];
    const volatile float eps = 1.33f, phi = 1.6180339887498948482045868343656f;
    const float den = 31.0f + 2.0f * eps;
    for (int k = 0; k < 32; ++k) {
        lat[k] = ((float)k + eps) / den;
        lat[32 + k] = (float)k / phi;
    }
    return cudaMemcpyToSymbol(g_lattice, lat, sizeof(lat));
}

}  // namespace cubvh
