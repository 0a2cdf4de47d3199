// Query kernels: unsigned distance, signed distance (watertight / raystab) and
// closest-hit ray tracing over one compressed 8-wide BVH (layout.h).
//
// Reference kernels replaced: src/bvh.cu:631-740 (unsigned_distance_kernel,
// signed_distance_{watertight,raystab}_kernel, raytrace_kernel) and the
// traversals they call (src/bvh.cu:250-427).  One thread owns one query; the
// traversal stack (node or leaf reference + lower-bound key) lives in local
// memory; children are visited nearest-first (sorted 32-bit keys).
#include <cstdint>
#include <cuda_runtime.h>

#include "geom.cuh"
#include "kernels.h"

namespace cubvh {

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
__device__ __forceinline__ uint32_t meta_of(const NodeView& n, int j) {
    return ((j < 4 ? n.meta0 : n.meta1) >> (8 * (j & 3))) & 0xFFu;
}
__device__ __forceinline__ void child_box(const NodeView& n, int j, float3& lo, float3& hi) {
    const int b = j & 3;
    const bool h = j >= 4;
    lo.x = fmaf(qf(h ? n.lx1 : n.lx0, b), n.sx, n.ox);
    lo.y = fmaf(qf(h ? n.ly1 : n.ly0, b), n.sy, n.oy);
    lo.z = fmaf(qf(h ? n.lz1 : n.lz0, b), n.sz, n.oz);
    hi.x = fmaf(qf(h ? n.hx1 : n.hx0, b), n.sx, n.ox);
    hi.y = fmaf(qf(h ? n.hy1 : n.hy0, b), n.sy, n.oy);
    hi.z = fmaf(qf(h ? n.hz1 : n.hz0, b), n.sz, n.oz);
}
// >= 0: internal node index; < 0: leaf, -(slot * 4 + count - 1) - 1
__device__ __forceinline__ int child_ref(const NodeView& n, uint32_t m) {
    if (m & 0x80u) return n.child_base + (int)(m & 7u);
    return -((((n.tri_base + (int)(m & 31u)) << 2) | (int)((m >> 5) & 3u)) + 1);
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
__device__ __forceinline__ void box_ray(float3 o, float3 inv, float3 lo, float3 hi, float& tn, float& tf) {
    const float t0x = (lo.x - o.x) * inv.x, t1x = (hi.x - o.x) * inv.x;
    const float t0y = (lo.y - o.y) * inv.y, t1y = (hi.y - o.y) * inv.y;
    const float t0z = (lo.z - o.z) * inv.z, t1z = (hi.z - o.z) * inv.z;
    tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    tn -= 1e-6f * fabsf(tn);
    tf += 1e-6f * fabsf(tf);
}
__device__ __forceinline__ float cull_of(double best) { return __double2float_ru(dM(best, 1.000001)); }
__device__ __forceinline__ void leaf_range(int ref, int& s0, int& s1) {
    const int code = -ref - 1;
    s0 = code >> 2; s1 = s0 + (code & 3) + 1;
}

// ---------------------------------------------------------- nearest triangle
// Exact (double) nearest triangle within squared distance best (in/out);
// ties -> lowest original face index.  slot = -1 if none.
__device__ void nearest_tri(const CNode* __restrict__ nodes, const CTri* __restrict__ tris, float3 p,
                            double& best, int& slot, int& id) {
    int2 st[kStack];
    int sp = 0;
    st[sp++] = make_int2(0, 0);
    float cull = cull_of(best);
    const d3 pd = to_d3(p);
    while (sp > 0) {
        const int2 e = st[--sp];
        if (__int_as_float(e.y) > cull) continue;
        if (e.x >= 0) {
            const NodeView n = load_node(nodes, e.x);
            uint32_t k[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float3 lo, hi;
                child_box(n, j, lo, hi);
                const float d2 = box_d2(p, lo, hi);
                k[j] = (meta_of(n, j) != kEmpty && d2 <= cull) ? ((__float_as_uint(d2) & ~7u) | (uint32_t)j)
                                                                 : 0xFFFFFFFFu;
            }
            sort8(k);
#pragma unroll
            for (int i = 7; i >= 0; --i)
                if (k[i] != 0xFFFFFFFFu)
                    st[sp++] = make_int2(child_ref(n, meta_of(n, (int)(k[i] & 7u))), (int)(k[i] & ~7u));
        } else {
            int s0, s1;
            leaf_range(e.x, s0, s1);
            for (int s = s0; s < s1; ++s) {
                const TriV t = load_tri(tris, s);
                float err;
                const float d2 = tri_d2_f(p, t, &err);
                if (d2 - err > cull) continue;
                double bary[3]; d3 cp;
                const double e64 = closest_on_tri_d(pd, to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
                if (e64 < best || (e64 == best && (slot < 0 || t.id < id))) {
                    best = e64; slot = s; id = t.id;
                    cull = cull_of(best);
                }
            }
        }
    }
}

// --------------------------------------------------------------- ray search
// Closest hit with 0 <= t < tmax (exact double t; ties -> lowest face index).
__device__ void closest_hit(const CNode* __restrict__ nodes, const CTri* __restrict__ tris, float3 o, float3 d,
                            double& best_t, int& slot, int& id) {
    const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const float dinf = f3inf(d);
    const float tmaxf = (float)best_t;
    const double tmax = best_t;
    const d3 od = to_d3(o), dd = to_d3(d);
    int2 st[kStack];
    int sp = 0;
    st[sp++] = make_int2(0, 0);
    float cull = cull_of(best_t);
    while (sp > 0) {
        const int2 e = st[--sp];
        if (__int_as_float(e.y) > cull) continue;
        if (e.x >= 0) {
            const NodeView n = load_node(nodes, e.x);
            uint32_t k[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float3 lo, hi;
                child_box(n, j, lo, hi);
                float tn, tf;
                box_ray(o, inv, lo, hi, tn, tf);
                const float key = fmaxf(tn, 0.f);
                k[j] = (meta_of(n, j) != kEmpty && tn <= tf && tf >= 0.f && key <= cull)
                           ? ((__float_as_uint(key) & ~7u) | (uint32_t)j) : 0xFFFFFFFFu;
            }
            sort8(k);
#pragma unroll
            for (int i = 7; i >= 0; --i)
                if (k[i] != 0xFFFFFFFFu)
                    st[sp++] = make_int2(child_ref(n, meta_of(n, (int)(k[i] & 7u))), (int)(k[i] & ~7u));
        } else {
            int s0, s1;
            leaf_range(e.x, s0, s1);
            for (int s = s0; s < s1; ++s) {
                const TriV t = load_tri(tris, s);
                float tt, terr;
                const int r = ray_tri_f(o, d, dinf, t, tmaxf, &tt, &terr);
                if (r == 0 || tt - terr > cull) continue;
                double t64;
                if (!ray_tri_d(od, dd, to_d3(t.a), to_d3(t.b), to_d3(t.c), tmax, &t64)) continue;
                if (t64 < best_t || (t64 == best_t && (slot < 0 || t.id < id))) {
                    best_t = t64; slot = s; id = t.id;
                    cull = cull_of(best_t);
                }
            }
        }
    }
}

// Any hit with 0 <= t < tmax.
__device__ bool any_hit(const CNode* __restrict__ nodes, const CTri* __restrict__ tris, float3 o, float3 d,
                        double tmax) {
    const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const float dinf = f3inf(d);
    const float tmaxf = (float)tmax;
    const float cull = cull_of(tmax);
    const d3 od = to_d3(o), dd = to_d3(d);
    int st[kStack];
    int sp = 0;
    st[sp++] = 0;
    while (sp > 0) {
        const int ref = st[--sp];
        if (ref >= 0) {
            const NodeView n = load_node(nodes, ref);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t m = meta_of(n, j);
                float3 lo, hi;
                child_box(n, j, lo, hi);
                float tn, tf;
                box_ray(o, inv, lo, hi, tn, tf);
                if (m != kEmpty && tn <= tf && tf >= 0.f && tn <= cull) st[sp++] = child_ref(n, m);
            }
        } else {
            int s0, s1;
            leaf_range(ref, s0, s1);
            for (int s = s0; s < s1; ++s) {
                const TriV t = load_tri(tris, s);
                float tt, terr;
                const int r = ray_tri_f(o, d, dinf, t, tmaxf, &tt, &terr);
                if (r == 1) return true;
                if (r < 0) {
                    double t64;
                    if (ray_tri_d(od, dd, to_d3(t.a), to_d3(t.b), to_d3(t.c), tmax, &t64)) return true;
                }
            }
        }
    }
    return false;
}

// Sum of unit normals of every triangle whose squared distance to cp is
// below 1e-6 (src/bvh.cu:356-396, without the division by the count, which
// does not change the sign).
__device__ d3 normal_sum(const CNode* __restrict__ nodes, const CTri* __restrict__ tris, d3 cp) {
    const float3 cf = make_float3(__double2float_rn(cp.x), __double2float_rn(cp.y), __double2float_rn(cp.z));
    const float cinf = f3inf(cf);
    const float r = 1e-3f + 4e-7f * (1.f + cinf);
    const float r2 = r * r * 1.00001f;
    const float slack = 1e-9f * (1.f + cinf);
    d3 sum{0.0, 0.0, 0.0};
    int st[kStack];
    int sp = 0;
    st[sp++] = 0;
    while (sp > 0) {
        const int ref = st[--sp];
        if (ref >= 0) {
            const NodeView n = load_node(nodes, ref);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t m = meta_of(n, j);
                float3 lo, hi;
                child_box(n, j, lo, hi);
                if (m != kEmpty && box_d2(cf, lo, hi) <= r2) st[sp++] = child_ref(n, m);
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
                if (closest_on_tri_d(cp, a, b, c, bary, &q) < 1e-6) {
                    const d3 nr = dcross(dsub(b, a), dsub(c, a));
                    const double len = __dsqrt_rn(ddot(nr, nr));
                    if (len > 0.0) sum = dadd(sum, d3{dD(nr.x, len), dD(nr.y, len), dD(nr.z, len)});
                }
            }
        }
    }
    return sum;
}

// ------------------------------------------------------------------ kernels
template <int MODE, bool UVW>
__global__ void __launch_bounds__(128) k_distance(int64_t n, const float* __restrict__ pts,
                                                  float* __restrict__ dist, int64_t* __restrict__ face_id,
                                                  float* __restrict__ uvw, const CNode* __restrict__ nodes,
                                                  const CTri* __restrict__ tris, int slot_face0) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 p = make_float3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    double best = 1e6;  // MAX_DIST^2 (src/bvh.cu:17-18)
    int slot = -1, id = 0;
    nearest_tri(nodes, tris, p, best, slot, id);
    double dist64;
    if (slot < 0) {  // nothing within MAX_DIST: distance 0 on face 0
        slot = slot_face0; dist64 = 0.0;
        id = load_tri(tris, slot).id;
    } else {
        dist64 = __dsqrt_rn(best);
    }
    const d3 pd = to_d3(p);
    double out = dist64;
    if (MODE != 0 || UVW) {
        const TriV t = load_tri(tris, slot);
        double bary[3]; d3 cp;
        closest_on_tri_d(pd, to_d3(t.a), to_d3(t.b), to_d3(t.c), bary, &cp);
        if (UVW) {
            uvw[3 * i] = __double2float_rn(bary[0]);
            uvw[3 * i + 1] = __double2float_rn(bary[1]);
            uvw[3 * i + 2] = __double2float_rn(bary[2]);
        }
        if (MODE == 1) {
            const d3 ns = normal_sum(nodes, tris, cp);
            out = copysign(dist64, ddot(ns, dsub(pd, cp)));
        }
    }
    if (MODE == 2) {
        const float2 off = stab_offset((uint32_t)i);
        bool inside = true;
        for (uint32_t k = 0; k < 32 && inside; ++k) {
            const float3 dir = stab_dir(k, off);
            const float3 ndir = make_float3(-dir.x, -dir.y, -dir.z);
            if (!any_hit(nodes, tris, p, ndir, 1000.0) || !any_hit(nodes, tris, p, dir, 1000.0)) inside = false;
        }
        if (inside) out = -dist64;
    }
    dist[i] = __double2float_rn(out);
    face_id[i] = (int64_t)id;
}

__global__ void __launch_bounds__(128) k_ray(int64_t n, const float* __restrict__ ro, const float* __restrict__ rd,
                                             float* __restrict__ pos, int64_t* __restrict__ face_id,
                                             float* __restrict__ depth, const CNode* __restrict__ nodes,
                                             const CTri* __restrict__ tris) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 o = make_float3(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]);
    const float3 d = make_float3(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]);
    double t = 1000.0;  // MAX_DIST
    int slot = -1, id = -1;
    closest_hit(nodes, tris, o, d, t, slot, id);
    depth[i] = __double2float_rn(t);
    pos[3 * i] = __double2float_rn(dA((double)o.x, dM(t, (double)d.x)));
    pos[3 * i + 1] = __double2float_rn(dA((double)o.y, dM(t, (double)d.y)));
    pos[3 * i + 2] = __double2float_rn(dA((double)o.z, dM(t, (double)d.z)));
    face_id[i] = slot >= 0 ? (int64_t)id : (int64_t)-1;
}

// --------------------------------------------------------------- launchers
static inline unsigned grid_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

cudaError_t launch_distance(int mode, bool want_uvw, int64_t n, const float* pts, float* dist, int64_t* fid,
                            float* uvw, const CNode* nodes, const CTri* tris, int slot_face0,
                            cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const dim3 grid(grid_for(n, 128)), block(128);
#define CUBVH_L(M, U) k_distance<M, U><<<grid, block, 0, stream>>>(n, pts, dist, fid, uvw, nodes, tris, slot_face0)
    if (mode == 0) { if (want_uvw) CUBVH_L(0, true); else CUBVH_L(0, false); }
    else if (mode == 1) { if (want_uvw) CUBVH_L(1, true); else CUBVH_L(1, false); }
    else { if (want_uvw) CUBVH_L(2, true); else CUBVH_L(2, false); }
#undef CUBVH_L
    return cudaGetLastError();
}

cudaError_t launch_ray(int64_t n, const float* ro, const float* rd, float* pos, int64_t* fid, float* depth,
                       const CNode* nodes, const CTri* tris, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_ray<<<grid_for(n, 128), 128, 0, stream>>>(n, ro, rd, pos, fid, depth, nodes, tris);
    return cudaGetLastError();
}

cudaError_t upload_constants() {
    double s[14], c[14];
    s[0] = 1.0; c[0] = 1.0;
    for (int k = 1; k < 14; ++k) {
        s[k] = -s[k - 1] / (double)((2 * k) * (2 * k + 1));
        c[k] = -c[k - 1] / (double)((2 * k - 1) * (2 * k));
    }
    cudaError_t e = cudaMemcpyToSymbol(c_sin_coef, s, sizeof(s));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_cos_coef, c, sizeof(c));
}

}  // namespace cubvh
