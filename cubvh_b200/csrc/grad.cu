// Differentiable distance queries: refit of the BVH to moved vertices and the
// backward of unsigned / signed distance.
//
// No counterpart in the reference (its cuBVH detaches the vertices and has no
// backward; cubvh/api.py:16-17).  For a query point p whose nearest point on
// its face f is c = sum_k lambda_k v_k (barycentric lambda), d = |p - c| and,
// by the envelope theorem,
//     d d / d p   =  (p - c) / d
//     d d / d v_k = -lambda_k (p - c) / d      (k = the three vertices of f)
// A signed distance carries its sign s as a constant factor.  The closest
// point is recomputed in double from the saved face id (nothing else is kept
// from the forward).  Vertex gradients are accumulated per face with a warp
// segmented reduction over queries sorted by face, so a face hit by many
// queries costs one set of atomics per warp segment instead of one per query.
#include <cstdint>
#include <cuda_runtime.h>

#include "launches.h"
#include "geom.cuh"
#include "kernels.h"
#include "scan.cuh"

namespace cubvh {
namespace {

constexpr unsigned kFullMask = 0xFFFFFFFFu;

// ------------------------------------------------------------------- refit
__device__ __forceinline__ float3 load3g(const float* __restrict__ a, int64_t i) {
    return make_float3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
}
__device__ __forceinline__ float3 vtx(const float* __restrict__ V, int i) {
    return make_float3(V[3 * i], V[3 * i + 1], V[3 * i + 2]);
}

__global__ void k_refit_soup(int64_t nt, CTri* __restrict__ tris, const int32_t* __restrict__ fv,
                             const float* __restrict__ V) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nt) return;
    CTri t = tris[s];
    const int f = t.id;
    const float3 a = vtx(V, fv[3 * f]), b = vtx(V, fv[3 * f + 1]), c = vtx(V, fv[3 * f + 2]);
    t.ax = a.x; t.ay = a.y; t.az = a.z;
    t.bx = b.x; t.by = b.y; t.bz = b.z;
    t.cx = c.x; t.cy = c.y; t.cz = c.z;
    // error scales as on the host: K, K * squared longest edge
    const float3 e[3] = {f3sub(b, a), f3sub(c, b), f3sub(a, c)};
    float e2 = 0.f;
#pragma unroll
    for (int u = 0; u < 3; ++u) e2 = fmaxf(e2, __fadd_rn(__fadd_rn(__fmul_rn(e[u].x, e[u].x), __fmul_rn(e[u].y, e[u].y)),
                                                         __fmul_rn(e[u].z, e[u].z)));
    const float va[3] = {a.x, a.y, a.z}, vb[3] = {b.x, b.y, b.z}, vc[3] = {c.x, c.y, c.z};
    t.k = tri_error_factor(va, vb, vc);
    t.ke2 = __fmul_rn(t.k, e2);
    tris[s] = t;
}

__device__ __forceinline__ int pick_exp(float o, float hi) {
    if (!(hi > o)) return -100;
    int e = (int)ceil(log2((double)(hi - o) / 255.0)) - 1;
    e = max(e, -100);
    while (fmaf(255.0f, exp2i(e), o) < hi) ++e;  // exact product, one rounding
    return e;
}

// One BFS level of nodes: exact box of each node from its children (leaf
// triangles, or the exact boxes of child nodes written by the deeper level),
// then the node's frame and the conservative quantisation of its children.
__global__ void k_refit_level(int l0, int l1, CNode* __restrict__ nodes, const CTri* __restrict__ tris,
                              float* __restrict__ nbox) {
    const int i = l0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= l1) return;
    CNode nd = nodes[i];
    float clo[8][3], chi[8][3];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int j = 0; j < 8; ++j) {
        const uint8_t m = nd.meta[j];
        for (int k = 0; k < 3; ++k) { clo[j][k] = INFINITY; chi[j][k] = -INFINITY; }
        if (m == kEmpty) continue;
        if (m & 0x80) {
            const float* b = nbox + 6 * (int64_t)(nd.child_base + (m & 7));
            for (int k = 0; k < 3; ++k) { clo[j][k] = b[k]; chi[j][k] = b[3 + k]; }
        } else {
            const int s0 = nd.tri_base + (m & 31), s1 = s0 + ((m >> 5) & 3) + 1;
            for (int s = s0; s < s1; ++s) {
                const CTri& t = tris[s];
                const float v[9] = {t.ax, t.ay, t.az, t.bx, t.by, t.bz, t.cx, t.cy, t.cz};
                for (int u = 0; u < 3; ++u)
                    for (int k = 0; k < 3; ++k) {
                        clo[j][k] = fminf(clo[j][k], v[3 * u + k]);
                        chi[j][k] = fmaxf(chi[j][k], v[3 * u + k]);
                    }
            }
        }
        for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], clo[j][k]); hi[k] = fmaxf(hi[k], chi[j][k]); }
    }
    float* nb = nbox + 6 * (int64_t)i;
    for (int k = 0; k < 3; ++k) { nb[k] = lo[k]; nb[3 + k] = hi[k]; }
    nd.ox = lo[0]; nd.oy = lo[1]; nd.oz = lo[2];
    const int ex[3] = {pick_exp(lo[0], hi[0]), pick_exp(lo[1], hi[1]), pick_exp(lo[2], hi[2])};
    nd.ex = (int8_t)ex[0]; nd.ey = (int8_t)ex[1]; nd.ez = (int8_t)ex[2];
    uint8_t* qlo[3] = {nd.qlo_x, nd.qlo_y, nd.qlo_z};
    uint8_t* qhi[3] = {nd.qhi_x, nd.qhi_y, nd.qhi_z};
    for (int j = 0; j < 8; ++j) {
        if (nd.meta[j] == kEmpty) continue;
        for (int k = 0; k < 3; ++k) {
            const float s = exp2i(ex[k]), o = lo[k];
            int ql = (int)floor((double)(clo[j][k] - o) / (double)s);
            int qh = (int)ceil((double)(chi[j][k] - o) / (double)s);
            ql = min(max(ql, 0), 255); qh = min(max(qh, 0), 255);
            while (ql > 0 && fmaf((float)ql, s, o) > clo[j][k]) --ql;
            while (qh < 255 && fmaf((float)qh, s, o) < chi[j][k]) ++qh;
            qlo[k][j] = (uint8_t)ql; qhi[k][j] = (uint8_t)qh;
        }
    }
    nodes[i] = nd;
}

// ---------------------------------------------------------------- backward
__global__ void k_face_hist(int64_t n, const int64_t* __restrict__ fid, int64_t nf, uint32_t* __restrict__ hist) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t f = fid[i];
        atomicAdd(&hist[(f >= 0 && f < nf) ? f : nf], 1u);
    }
}
__global__ void k_face_scatter(int64_t n, const int64_t* __restrict__ fid, int64_t nf, uint32_t* __restrict__ offs,
                               uint32_t* __restrict__ order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t f = fid[i];
        order[atomicAdd(&offs[(f >= 0 && f < nf) ? f : nf], 1u)] = (uint32_t)i;
    }
}

// Queries in face order; lane values of one face within a warp are summed by
// an inclusive segmented scan (shuffles), the segment's last lane adds them.
__global__ void __launch_bounds__(256) k_backward(
    int64_t n, const uint32_t* __restrict__ order, const float* __restrict__ pts, const int64_t* __restrict__ fid,
    const float* __restrict__ gout, const float* __restrict__ dist, const float* __restrict__ V,
    const int32_t* __restrict__ fv, const int32_t* __restrict__ fslot, const CTri* __restrict__ tris, int64_t nf,
    float* __restrict__ gpts, float* __restrict__ gV) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarp_total = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += nwarp_total * 32) {
        const int64_t q = base + lane;
        const bool act = q < n;
        int64_t f = -1;
        float c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (act) {
            const int64_t i = order[q];
            f = fid[i];
            const float g = gout[i], d = dist[i];
            float gp[3] = {0.f, 0.f, 0.f};
            if (f >= 0 && f < nf && g != 0.f && d != 0.f) {
                d3 a, b, cc;
                if (V && fv) {
                    a = to_d3(vtx(V, fv[3 * f])); b = to_d3(vtx(V, fv[3 * f + 1])); cc = to_d3(vtx(V, fv[3 * f + 2]));
                } else if (fslot[f] >= 0) {
                    const TriV t = load_tri(tris, fslot[f]);
                    a = to_d3(t.a); b = to_d3(t.b); cc = to_d3(t.c);
                } else {
                    a = b = cc = d3{0.0, 0.0, 0.0};
                }
                const d3 p = to_d3(load3g(pts, i));
                double lam[3]; d3 cp;
                const double d2 = closest_on_tri_d(p, a, b, cc, lam, &cp);
                if (d2 > 0.0) {
                    const double sc = (signbit(d) ? -(double)g : (double)g) / __dsqrt_rn(d2);
                    const d3 r = dsub(p, cp);
                    gp[0] = (float)(r.x * sc); gp[1] = (float)(r.y * sc); gp[2] = (float)(r.z * sc);
                    for (int k = 0; k < 3; ++k) {
                        c[3 * k] = (float)(-lam[k] * r.x * sc);
                        c[3 * k + 1] = (float)(-lam[k] * r.y * sc);
                        c[3 * k + 2] = (float)(-lam[k] * r.z * sc);
                    }
                }
            }
            if (gpts) { gpts[3 * i] = gp[0]; gpts[3 * i + 1] = gp[1]; gpts[3 * i + 2] = gp[2]; }
        }
        if (!gV || !fv) continue;
        // segmented inclusive scan over lanes with equal face id
        const int64_t fprev = __shfl_up_sync(kFullMask, f, 1);
        const bool head = lane == 0 || fprev != f;
        const unsigned heads = __ballot_sync(kFullMask, head);
        // first lane of my segment
        const int seg0 = 31 - __clz(heads & ((2u << lane) - 1u));
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const float v = __shfl_up_sync(kFullMask, c[k], o);
                if (lane - o >= seg0) c[k] += v;
            }
        }
        const int64_t fnext = __shfl_down_sync(kFullMask, f, 1);
        const bool tail = lane == 31 || fnext != f || base + lane + 1 >= n;
        if (act && tail && f >= 0 && f < nf) {
            for (int k = 0; k < 3; ++k) {
                const int v = fv[3 * f + k];
                atomicAdd(&gV[3 * v], c[3 * k]);
                atomicAdd(&gV[3 * v + 1], c[3 * k + 1]);
                atomicAdd(&gV[3 * v + 2], c[3 * k + 2]);
            }
        }
    }
}

__device__ __forceinline__ int mesh_of_q(const int64_t* __restrict__ qoff, int M, int64_t i) {
    int lo = 0, hi = M - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (qoff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Arena: gradients w.r.t. the query points only, one thread per query.
__global__ void k_arena_backward_points(int64_t n, const float* __restrict__ pts, const int64_t* __restrict__ fid,
                                        const float* __restrict__ gout, const float* __restrict__ dist,
                                        const int64_t* __restrict__ qoff, int M, const int64_t* __restrict__ face_off,
                                        const int32_t* __restrict__ gslot, const CTri* __restrict__ tris,
                                        float* __restrict__ gpts) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int m = mesh_of_q(qoff, M, i);
        const int64_t f = fid[i];
        const int64_t nfm = face_off[m + 1] - face_off[m];
        const float g = gout[i], d = dist[i];
        float gp[3] = {0.f, 0.f, 0.f};
        if (f >= 0 && f < nfm && g != 0.f && d != 0.f) {
            const int32_t s = gslot[face_off[m] + f];
            if (s >= 0) {
                const TriV t = load_tri(tris, s);
                const d3 p = to_d3(load3g(pts, i));
                double lam[3]; d3 cp;
                const double d2 = closest_on_tri_d(p, to_d3(t.a), to_d3(t.b), to_d3(t.c), lam, &cp);
                if (d2 > 0.0) {
                    const double sc = (signbit(d) ? -(double)g : (double)g) / __dsqrt_rn(d2);
                    const d3 r = dsub(p, cp);
                    gp[0] = (float)(r.x * sc); gp[1] = (float)(r.y * sc); gp[2] = (float)(r.z * sc);
                }
            }
        }
        gpts[3 * i] = gp[0]; gpts[3 * i + 1] = gp[1]; gpts[3 * i + 2] = gp[2];
    }
}

}  // namespace

cudaError_t launch_refit(int64_t n_tris, CTri* tris, const int32_t* face_vidx, const float* V, CNode* nodes,
                         float* node_box, const int32_t* level_start, int n_levels, cudaStream_t stream) {
    if (n_tris <= 0) return cudaSuccess;
    k_refit_soup<<<(unsigned)((n_tris + 255) / 256), 256, 0, stream>>>(n_tris, tris, face_vidx, V); count_launch();
    for (int l = n_levels - 1; l >= 0; --l) {
        const int l0 = level_start[l], l1 = level_start[l + 1];
        if (l1 <= l0) continue;
        k_refit_level<<<(unsigned)((l1 - l0 + 63) / 64), 64, 0, stream>>>(l0, l1, nodes, tris, node_box); count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_arena_backward(int64_t n, const float* pts, const int64_t* fid, const float* gout,
                                  const float* dist, const int64_t* qoff, int M, const int64_t* face_off,
                                  const int32_t* gslot, const CTri* tris, float* gpts, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_arena_backward_points<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, pts, fid, gout, dist, qoff, M, face_off,
                                                                             gslot, tris, gpts); count_launch();
    return cudaGetLastError();
}

size_t backward_workspace_bytes(int64_t n, int64_t nf) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    return al(sizeof(uint32_t) * n) + al(sizeof(uint32_t) * (nf + 2)) + al(sizeof(uint32_t) * (scan::num_chunks(nf + 1) + 1));
}

cudaError_t launch_backward(int64_t n, const float* pts, const int64_t* fid, const float* gout, const float* dist,
                            const float* V, const int32_t* fv, const int32_t* fslot, const CTri* tris, int64_t nf,
                            float* gpts, float* gV, void* ws, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    char* w = static_cast<char*>(ws);
    uint32_t* order = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * n);
    uint32_t* hist = reinterpret_cast<uint32_t*>(w); w += al(sizeof(uint32_t) * (nf + 2));
    uint32_t* bsum = reinterpret_cast<uint32_t*>(w);
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (nf + 2), stream);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned g = (unsigned)nsm * 8;
    k_face_hist<<<g, 256, 0, stream>>>(n, fid, nf, hist); count_launch();
    scan::exclusive(hist, bsum, nf + 1, stream);
    k_face_scatter<<<g, 256, 0, stream>>>(n, fid, nf, hist, order); count_launch();
    k_backward<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, order, pts, fid, gout, dist, V, fv, fslot, tris, nf,
                                                                gpts, gV); count_launch();
    return cudaGetLastError();
}

}  // namespace cubvh
