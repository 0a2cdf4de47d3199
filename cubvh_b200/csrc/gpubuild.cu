// BVH construction on the GPU (the reference builds on the host only:
// TriangleBvh4::build, src/bvh.cu:515-620).  The result has exactly the
// layout of the host builder (layout.h; build.cpp): 8-wide nodes stored
// breadth first with each node's internal children consecutive, leaves of at
// most `max_leaf` triangles whose triangles are consecutive in the soup and
// numbered in the order of their node, child boxes quantised with the same
// conservative rounding.  Only the tree differs: a linear BVH instead of the
// host's binned SAH.
//
// Many meshes are built in one pass (the batched arena): keys carry the mesh
// index above the Morton code, so each mesh's faces are one sorted range and
// one subtree of the radix tree, whose root starts the mesh's wide tree.
//
//   1. per face: its mesh, bounds, centroid, the 48-byte triangle record
//      (face index within its mesh), checks of the vertex indices and
//      coordinates (reported through a flag word)
//   2. key = mesh index << 30 | 30-bit Morton code of the centroid in its
//      mesh's centroid box; pairs (key, face) radix sorted; equal keys are
//      told apart by sorted position in the prefix function
//   3. binary radix tree over the sorted keys (Karras, "Maximizing
//      parallelism in the construction of BVHs, octrees, and k-d trees",
//      HPG 2012), boxes bottom up (the second child to arrive at a node
//      computes it; the first returns, so no thread waits)
//   4. breadth-first collapse to 8-wide, one level per pass: a node takes the
//      two children of its binary node and keeps replacing its widest (by
//      surface area, or by triangle count) internal child by that child's two
//      children until it has 8; a binary node covering at most `max_leaf`
//      triangles is a leaf.  Level 0 holds every mesh's root.  Per level:
//      expand, scan of internal-child and triangle counts, emit (quantised
//      node, soup records, next level).
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "build.h"
#include "gpubuild.h"
#include "kernels.h"
#include "launches.h"
#include "scan.cuh"

namespace cubvh {
namespace {

constexpr int kBlk = 256;

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kBlk - 1) / kBlk); }

// order-preserving float <-> uint32 (for atomicMin / atomicMax of floats)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void k_bounds_init(uint32_t* cb, int32_t M) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 6 * (int64_t)M) return;
    cb[i] = (i % 6) < 3 ? 0xFFFFFFFFu : 0u;
}

// mesh of global face / sorted position i: the last m with off[m] <= i
__device__ __forceinline__ int32_t mesh_of_face(const int64_t* __restrict__ off, int32_t M, int64_t i) {
    int32_t lo = 0, hi = M - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// 1. face bounds [lo, hi] (6 floats), centroid, triangle record in face
// order; flag bit 1: vertex index out of range, bit 2: non-finite coordinate
__global__ void k_prep(const float* __restrict__ v, const int64_t* __restrict__ voff,
                       const int64_t* __restrict__ f, const int64_t* __restrict__ foff, int32_t M, int64_t nf,
                       float* __restrict__ fbox, float* __restrict__ cen, CTri* __restrict__ rec,
                       uint32_t* __restrict__ cbounds, int* __restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int32_t m = mesh_of_face(foff, M, i);
    const int64_t v0 = voff[m], nv = voff[m + 1] - v0;
    float p[3][3];
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
        int64_t vi = f[3 * i + k];
        if (vi < 0 || vi >= nv) { atomicOr(flag, 1); ok = false; vi = 0; }
        for (int c = 0; c < 3; ++c) {
            p[k][c] = v[3 * (v0 + vi) + c];
            if (!isfinite(p[k][c])) { atomicOr(flag, 2); ok = false; }
        }
    }
    if (!ok)
        for (int k = 0; k < 3; ++k) p[k][0] = p[k][1] = p[k][2] = 0.f;
    float lo[3], hi[3];
    for (int c = 0; c < 3; ++c) {
        lo[c] = fminf(fminf(p[0][c], p[1][c]), p[2][c]);
        hi[c] = fmaxf(fmaxf(p[0][c], p[1][c]), p[2][c]);
        fbox[6 * i + c] = lo[c];
        fbox[6 * i + 3 + c] = hi[c];
        const float mc = __fmul_rn(0.5f, __fadd_rn(lo[c], hi[c]));
        cen[3 * i + c] = mc;
        atomicMin(&cbounds[6 * m + c], f2o(mc));
        atomicMax(&cbounds[6 * m + 3 + c], f2o(mc));
    }
    // error scales of the FP32 distance filter, with the host builder's operations
    float e2 = 0.f;
    for (int u = 0; u < 3; ++u) {
        const float* q0 = p[u];
        const float* q1 = p[(u + 1) % 3];
        const float dx = __fsub_rn(q1[0], q0[0]), dy = __fsub_rn(q1[1], q0[1]), dz = __fsub_rn(q1[2], q0[2]);
        e2 = fmaxf(e2, __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    }
    CTri t;
    t.ax = p[0][0]; t.ay = p[0][1]; t.az = p[0][2]; t.id = (int32_t)(i - foff[m]);
    t.k = tri_error_factor(p[0], p[1], p[2]);
    t.bx = p[1][0]; t.by = p[1][1]; t.bz = p[1][2]; t.ke2 = __fmul_rn(t.k, e2);
    t.cx = p[2][0]; t.cy = p[2][1]; t.cz = p[2][2];
    rec[i] = t;
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 2. keys: mesh << 30 | Morton code, value: global face index
__global__ void k_keys(const float* __restrict__ cen, const int64_t* __restrict__ foff, int32_t M, int64_t nf,
                       const uint32_t* __restrict__ cbounds, uint64_t* __restrict__ keys,
                       uint32_t* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int32_t m = mesh_of_face(foff, M, i);
    uint32_t q[3];
    for (int c = 0; c < 3; ++c) {
        const float lo = o2f(cbounds[6 * m + c]), hi = o2f(cbounds[6 * m + 3 + c]);
        const float ext = hi - lo;
        const float t = ext > 0.f ? (cen[3 * i + c] - lo) / ext : 0.f;
        q[c] = (uint32_t)fminf(fmaxf(t * 1024.f, 0.f), 1023.f);
    }
    const uint32_t code = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    keys[i] = ((uint64_t)(uint32_t)m << 30) | (uint64_t)code;
    vals[i] = (uint32_t)i;
}

// common prefix length of sorted keys i and j (-1 outside [0, n)); equal keys
// continue with the bits of the sorted positions (Karras 2012, section 4)
__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t x = k[i] ^ k[j];
    if (x) return __clzll((long long)x);
    return 64 + __clz((int)((uint32_t)i ^ (uint32_t)j));
}

// 3a. binary radix tree.  References: internal node i -> i (0..n-2), leaf
// (sorted position) j -> n - 1 + j.  first/last: covered sorted range.
__global__ void k_radix_tree(const uint64_t* __restrict__ k, int64_t n, int32_t* __restrict__ left,
                             int32_t* __restrict__ right, int32_t* __restrict__ parent, int32_t* __restrict__ first,
                             int32_t* __restrict__ last) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int64_t lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;  // at most ~log2(n) doublings
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int64_t s = 0;
    for (int64_t t = (l + 1) / 2;; t = (t + 1) / 2) {
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    const int32_t lref = (int32_t)(lo == gamma ? (n - 1 + gamma) : gamma);
    const int32_t rref = (int32_t)(hi == gamma + 1 ? (n - 1 + gamma + 1) : gamma + 1);
    left[i] = lref;
    right[i] = rref;
    parent[lref] = (int32_t)i;
    parent[rref] = (int32_t)i;
    first[i] = (int32_t)lo;
    last[i] = (int32_t)hi;
}

// 3b. boxes bottom up: leaf boxes come from the sorted faces; at each node
// the second arriving child computes the union, the first one returns
__global__ void k_tree_boxes(const uint32_t* __restrict__ sval, int64_t n, const float* __restrict__ fbox,
                             const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                             const int32_t* __restrict__ parent, float* __restrict__ box,
                             uint32_t* __restrict__ arrived) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t face = sval[j];
    float* lb = box + 6 * (n - 1 + j);
    for (int c = 0; c < 6; ++c) lb[c] = fbox[6 * face + c];
    int32_t p = n > 1 ? parent[n - 1 + j] : -1;
    while (p >= 0) {
        __threadfence();
        if (atomicAdd(&arrived[p], 1u) == 0u) return;  // the sibling finishes this node
        __threadfence();
        const float* a = box + 6 * left[p];
        const float* b = box + 6 * right[p];
        float* o = box + 6 * p;
        for (int c = 0; c < 3; ++c) {
            o[c] = fminf(__ldcg(a + c), __ldcg(b + c));
            o[3 + c] = fmaxf(__ldcg(a + 3 + c), __ldcg(b + 3 + c));
        }
        p = parent[p];
    }
}

// 3c. each mesh's root: the node covering exactly its sorted range
// [foff[m], foff[m + 1]) (a leaf for a one-face mesh)
__global__ void k_roots(const int32_t* __restrict__ first, const int32_t* __restrict__ last, int64_t n,
                        const int64_t* __restrict__ foff, int32_t M, int32_t* __restrict__ roots) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M && foff[i + 1] - foff[i] == 1) roots[i] = (int32_t)(n - 1 + foff[i]);
    if (i >= n - 1) return;
    const int32_t m = mesh_of_face(foff, M, first[i]);
    if (first[i] == foff[m] && last[i] == foff[m + 1] - 1) roots[m] = (int32_t)i;
}

struct TreeView {
    int64_t n;
    const int32_t *left, *right, *first, *last;
    const float* box;
    const int64_t* foff;       // mesh face offsets [M + 1]
    const int32_t* leaf_size;  // per mesh
    int32_t M;
    __device__ __forceinline__ int32_t mesh(int32_t r) const { return mesh_of_face(foff, M, lo_of(r)); }
    __device__ __forceinline__ int64_t lo_of(int32_t r) const { return r < n - 1 ? first[r] : r - (n - 1); }
    __device__ __forceinline__ int64_t hi_of(int32_t r) const { return r < n - 1 ? last[r] : r - (n - 1); }
    __device__ __forceinline__ int count(int32_t r) const { return (int)(hi_of(r) - lo_of(r) + 1); }
    __device__ __forceinline__ float area(int32_t r) const {
        const float* b = box + 6 * r;
        const float x = b[3] - b[0], y = b[4] - b[1], z = b[5] - b[2];
        return x * y + y * z + z * x;
    }
};

// 4a. children of each wide node of the level: wch[8 w ..], and per node the
// number of internal children and of triangles in its leaf children
__global__ void k_wide_expand(TreeView t, const int32_t* __restrict__ refs, int64_t m, int by_count,
                              int32_t* __restrict__ wch, uint32_t* __restrict__ nint, uint32_t* __restrict__ ntri) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= m) return;
    const int32_t b = refs[w];
    const int max_leaf = t.leaf_size[t.mesh(b)];
    int32_t ch[kWidth];
    int nc;
    if (t.count(b) <= max_leaf) {
        ch[0] = b;
        nc = 1;
    } else {
        ch[0] = t.left[b];
        ch[1] = t.right[b];
        nc = 2;
        while (nc < kWidth) {
            int bi = -1;
            float bw = -1.f;
            for (int i = 0; i < nc; ++i) {
                if (t.count(ch[i]) <= max_leaf) continue;
                const float wgt = by_count ? (float)t.count(ch[i]) : t.area(ch[i]);
                if (wgt > bw) { bw = wgt; bi = i; }
            }
            if (bi < 0) break;
            const int32_t c = ch[bi];
            for (int i = nc; i > bi + 1; --i) ch[i] = ch[i - 1];
            ch[bi] = t.left[c];
            ch[bi + 1] = t.right[c];
            ++nc;
        }
    }
    uint32_t ni = 0, nt = 0;
    for (int i = 0; i < kWidth; ++i) {
        wch[kWidth * w + i] = i < nc ? ch[i] : -1;
        if (i < nc) {
            const int cnt = t.count(ch[i]);
            if (cnt <= max_leaf) nt += (uint32_t)cnt;
            else ++ni;
        }
    }
    nint[w] = ni;
    ntri[w] = nt;
}

// Host builder's rounding rules (build.cpp: pick_exponent, quantise_child),
// with the products computed exactly as the query kernels decode them.
__device__ int pick_exponent_d(float o, float hi) {
    if (!(hi > o)) return -100;
    int e = (int)ceil(log2((double)(hi - o) / 255.0)) - 1;
    e = e < -100 ? -100 : e;
    while (__fadd_rn(o, __fmul_rn(255.0f, ldexpf(1.0f, e))) < hi) ++e;
    return e;
}
__device__ void quantise_d(float o, int e, float lo, float hi, uint8_t& qlo, uint8_t& qhi) {
    const float s = ldexpf(1.0f, e);
    int ql = (int)floor((double)__fsub_rn(lo, o) / (double)s);
    int qh = (int)ceil((double)__fsub_rn(hi, o) / (double)s);
    ql = ql < 0 ? 0 : (ql > 255 ? 255 : ql);
    qh = qh < 0 ? 0 : (qh > 255 ? 255 : qh);
    while (ql > 0 && fmaf((float)ql, s, o) > lo) --ql;
    while (qh < 255 && fmaf((float)qh, s, o) < hi) ++qh;
    qlo = (uint8_t)ql;
    qhi = (uint8_t)qh;
}

// 4b. emit the level's nodes (global index base + w), their leaf triangles
// (soup from tri_base0 + tri prefix) and the next level's binary nodes
__global__ void k_wide_emit(TreeView t, const int32_t* __restrict__ refs, int64_t m,
                            const int32_t* __restrict__ wch, const uint32_t* __restrict__ int_pre,
                            const uint32_t* __restrict__ tri_pre, int64_t base, int64_t next_base,
                            int64_t tri_base0, const uint32_t* __restrict__ sval, const CTri* __restrict__ rec,
                            CNode* __restrict__ nodes, CTri* __restrict__ soup, int32_t* __restrict__ next_refs,
                            int32_t* __restrict__ slot_face0, int32_t* __restrict__ gslot) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= m) return;
    const int max_leaf = t.leaf_size[t.mesh(refs[w])];
    const float* nb = t.box + 6 * refs[w];
    CNode nd;
    memset(&nd, 0, sizeof(nd));
    for (int j = 0; j < kWidth; ++j) nd.meta[j] = kEmpty;
    nd.ox = nb[0]; nd.oy = nb[1]; nd.oz = nb[2];
    const int ex = pick_exponent_d(nb[0], nb[3]), ey = pick_exponent_d(nb[1], nb[4]), ez = pick_exponent_d(nb[2], nb[5]);
    nd.ex = (int8_t)ex; nd.ey = (int8_t)ey; nd.ez = (int8_t)ez;
    nd.child_base = (int32_t)(next_base + int_pre[w]);
    const int64_t tb = tri_base0 + tri_pre[w];
    nd.tri_base = (int32_t)tb;
    int slot = 0, off = 0;
    for (int j = 0; j < kWidth; ++j) {
        const int32_t c = wch[kWidth * w + j];
        if (c < 0) break;
        const float* cb = t.box + 6 * c;
        quantise_d(nd.ox, ex, cb[0], cb[3], nd.qlo_x[j], nd.qhi_x[j]);
        quantise_d(nd.oy, ey, cb[1], cb[4], nd.qlo_y[j], nd.qhi_y[j]);
        quantise_d(nd.oz, ez, cb[2], cb[5], nd.qlo_z[j], nd.qhi_z[j]);
        const int cnt = t.count(c);
        if (cnt <= max_leaf) {
            const int64_t s0 = t.lo_of(c);
            for (int q = 0; q < cnt; ++q) {
                const int64_t face = sval[s0 + q];
                const CTri r = rec[face];
                const int64_t slot = tb + off + q;
                soup[slot] = r;
                if (r.id == 0) slot_face0[t.mesh(c)] = (int32_t)slot;
                if (gslot) gslot[face] = (int32_t)slot;
            }
            nd.meta[j] = (uint8_t)(((cnt - 1) << 5) | off);
            off += cnt;
        } else {
            nd.meta[j] = (uint8_t)(0x80 | slot);
            next_refs[int_pre[w] + slot] = c;
            ++slot;
        }
    }
    nd.n_internal = (uint8_t)slot;
    nodes[base + w] = nd;
}

__global__ void k_mesh_boxes(const float* __restrict__ box, const int32_t* __restrict__ roots, int32_t M,
                             float* __restrict__ mbox) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 6 * (int64_t)M) return;
    mbox[i] = box[6 * roots[i / 6] + i % 6];
}

struct DevBufs {
    std::vector<void*> ptrs;
    ~DevBufs() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    cudaError_t get(T** p, size_t count) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
        if (e == cudaSuccess) { ptrs.push_back(q); *p = static_cast<T*>(q); }
        return e;
    }
};

}  // namespace

int build_meshes_device(const float* v, const int64_t* f, const std::vector<int64_t>& voff,
                        const std::vector<int64_t>& foff, const std::vector<int32_t>& leaf, cudaStream_t s,
                        DeviceBuild& out, std::string& err, bool want_gslot) {
#define CUBVH_CK(expr) do { const cudaError_t e_ = (expr); if (e_ != cudaSuccess) { \
        err = std::string(#expr) + ": " + cudaGetErrorString(e_); return 2; } } while (0)
    const int32_t M = (int32_t)leaf.size();
    if (M <= 0 || (int64_t)voff.size() != M + 1 || (int64_t)foff.size() != M + 1) { err = "bad mesh table"; return 1; }
    const int64_t n = foff[M];
    for (int32_t m = 0; m < M; ++m) {
        if (foff[m + 1] - foff[m] <= 0 || voff[m + 1] - voff[m] <= 0) { err = "mesh " + std::to_string(m) + " is empty"; return 1; }
        if (leaf[m] < 1 || leaf[m] > kMaxLeafTris) { err = "leaf size must be in [1, 4]"; return 1; }
    }
    if (n > (int64_t)(1 << 28)) { err = "too many faces (limit 2^28)"; return 1; }
    DevBufs B;
    const int64_t ni = n > 1 ? n - 1 : 1;
    float *fbox, *cen, *box, *mbox;
    CTri* rec;
    uint32_t *cb, *arrived, *vals, *vals2;
    int* flag;
    uint64_t *keys, *keys2;
    int64_t *d_voff, *d_foff;
    int32_t *d_leaf, *roots, *left, *right, *parent, *first, *last;
    CUBVH_CK(B.get(&d_voff, M + 1));
    CUBVH_CK(B.get(&d_foff, M + 1));
    CUBVH_CK(B.get(&d_leaf, M));
    CUBVH_CK(B.get(&roots, M));
    CUBVH_CK(B.get(&mbox, 6 * (int64_t)M));
    CUBVH_CK(B.get(&fbox, 6 * n));
    CUBVH_CK(B.get(&cen, 3 * n));
    CUBVH_CK(B.get(&rec, n));
    CUBVH_CK(B.get(&cb, 6 * (int64_t)M));
    CUBVH_CK(B.get(&flag, 1));
    CUBVH_CK(B.get(&keys, n));
    CUBVH_CK(B.get(&keys2, n));
    CUBVH_CK(B.get(&vals, n));
    CUBVH_CK(B.get(&vals2, n));
    CUBVH_CK(B.get(&left, ni));
    CUBVH_CK(B.get(&right, ni));
    CUBVH_CK(B.get(&parent, ni + n));
    CUBVH_CK(B.get(&first, ni));
    CUBVH_CK(B.get(&last, ni));
    CUBVH_CK(B.get(&box, 6 * (ni + n)));
    CUBVH_CK(B.get(&arrived, ni));
    CUBVH_CK(cudaMemcpyAsync(d_voff, voff.data(), sizeof(int64_t) * (M + 1), cudaMemcpyHostToDevice, s));
    CUBVH_CK(cudaMemcpyAsync(d_foff, foff.data(), sizeof(int64_t) * (M + 1), cudaMemcpyHostToDevice, s));
    CUBVH_CK(cudaMemcpyAsync(d_leaf, leaf.data(), sizeof(int32_t) * M, cudaMemcpyHostToDevice, s));
    CUBVH_CK(cudaMemsetAsync(flag, 0, sizeof(int), s));
    CUBVH_CK(cudaMemsetAsync(arrived, 0, sizeof(uint32_t) * ni, s));
    CUBVH_CK(cudaMemsetAsync(parent, 0xFF, sizeof(int32_t) * (ni + n), s));  // -1: a root
    k_bounds_init<<<blocks_for(6 * (int64_t)M), kBlk, 0, s>>>(cb, M); count_launch();
    k_prep<<<blocks_for(n), kBlk, 0, s>>>(v, d_voff, f, d_foff, M, n, fbox, cen, rec, cb, flag); count_launch();
    int hflag = 0;
    CUBVH_CK(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUBVH_CK(cudaStreamSynchronize(s));
    if (hflag & 1) { err = "a face has a vertex index outside [0, n_vertices)"; return 1; }
    if (hflag & 2) { err = "vertex coordinates must be finite"; return 1; }
    k_keys<<<blocks_for(n), kBlk, 0, s>>>(cen, d_foff, M, n, cb, keys, vals); count_launch();
    int kbits = 30;
    while (kbits < 64 && ((uint64_t)(M - 1) >> (kbits - 30)) != 0) ++kbits;
    size_t tmp_bytes = 0;
    CUBVH_CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, (int)n, 0, kbits, s));
    uint8_t* tmp;
    CUBVH_CK(B.get(&tmp, tmp_bytes));
    CUBVH_CK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, (int)n, 0, kbits, s));
    count_launch();
    if (n > 1) { k_radix_tree<<<blocks_for(n - 1), kBlk, 0, s>>>(keys2, n, left, right, parent, first, last); count_launch(); }
    k_tree_boxes<<<blocks_for(n), kBlk, 0, s>>>(vals2, n, fbox, left, right, parent, box, arrived); count_launch();
    k_roots<<<blocks_for(std::max<int64_t>(n - 1, M)), kBlk, 0, s>>>(first, last, n, d_foff, M, roots); count_launch();
    k_mesh_boxes<<<blocks_for(6 * (int64_t)M), kBlk, 0, s>>>(box, roots, M, mbox); count_launch();
    const TreeView t{n, left, right, first, last, box, d_foff, d_leaf, M};

    // 4. levels (breadth first), level 0 = the M roots.  Every node below
    // level 0 consumes a distinct binary internal node.
    const int64_t wmax = ni + M;
    CNode* nodes;
    CTri* soup;
    int32_t *refs_a, *refs_b, *wch, *slot0, *gslot = nullptr;
    uint32_t *nint, *ntri, *bsum;
    CUBVH_CK(B.get(&nodes, wmax));
    CUBVH_CK(B.get(&soup, n));
    CUBVH_CK(B.get(&refs_a, wmax));
    CUBVH_CK(B.get(&refs_b, wmax));
    CUBVH_CK(B.get(&wch, kWidth * wmax));
    CUBVH_CK(B.get(&nint, wmax + 1));
    CUBVH_CK(B.get(&ntri, wmax + 1));
    CUBVH_CK(B.get(&bsum, scan::num_chunks(wmax) + 2));
    CUBVH_CK(B.get(&slot0, M));
    if (want_gslot) CUBVH_CK(B.get(&gslot, n));
    for (int by_count = 0; by_count < 2; ++by_count) {
        std::vector<int32_t> level_start{0};
        int64_t m = M, base = 0, tri0 = 0;
        CUBVH_CK(cudaMemcpyAsync(refs_a, roots, sizeof(int32_t) * M, cudaMemcpyDeviceToDevice, s));
        int32_t* cur = refs_a;
        int32_t* nxt = refs_b;
        bool deep = false;
        while (m > 0) {
            if ((int)level_start.size() > kMaxDepth) { deep = true; break; }
            k_wide_expand<<<blocks_for(m), kBlk, 0, s>>>(t, cur, m, by_count, wch, nint, ntri); count_launch();
            scan::exclusive(nint, bsum, m, s);
            scan::exclusive(ntri, bsum, m, s);
            uint32_t tot[2];
            CUBVH_CK(cudaMemcpyAsync(&tot[0], nint + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CUBVH_CK(cudaMemcpyAsync(&tot[1], ntri + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            k_wide_emit<<<blocks_for(m), kBlk, 0, s>>>(t, cur, m, wch, nint, ntri, base, base + m, tri0, vals2, rec,
                                                       nodes, soup, nxt, slot0, gslot); count_launch();
            CUBVH_CK(cudaStreamSynchronize(s));
            base += m;
            tri0 += tot[1];
            level_start.push_back((int32_t)base);
            m = tot[0];
            std::swap(cur, nxt);
            if (base + m > wmax) { err = "GPU build: node count overflow"; return 2; }
        }
        if (deep) continue;
        if (tri0 != n) { err = "GPU build: triangle count mismatch"; return 2; }
        out.n_nodes = base;
        out.depth = (int)level_start.size() - 1;
        out.level_start = level_start;
        out.nodes = nullptr;
        out.tris = nullptr;
        out.gslot = nullptr;
        out.slot0.resize(M);
        out.mesh_box.resize(6 * (size_t)M);
        CUBVH_CK(cudaMemcpyAsync(out.slot0.data(), slot0, sizeof(int32_t) * M, cudaMemcpyDeviceToHost, s));
        CUBVH_CK(cudaMemcpyAsync(out.mesh_box.data(), mbox, sizeof(float) * 6 * M, cudaMemcpyDeviceToHost, s));
        if (cudaMalloc(&out.nodes, sizeof(CNode) * base) != cudaSuccess ||
            cudaMalloc(&out.tris, sizeof(CTri) * n) != cudaSuccess ||
            (want_gslot && cudaMalloc(&out.gslot, sizeof(int32_t) * n) != cudaSuccess)) {
            cudaFree(out.nodes); cudaFree(out.tris); cudaFree(out.gslot);
            out.nodes = nullptr; out.tris = nullptr; out.gslot = nullptr;
            err = "cudaMalloc of the built BVH failed"; return 2;
        }
        CUBVH_CK(cudaMemcpyAsync(out.nodes, nodes, sizeof(CNode) * base, cudaMemcpyDeviceToDevice, s));
        CUBVH_CK(cudaMemcpyAsync(out.tris, soup, sizeof(CTri) * n, cudaMemcpyDeviceToDevice, s));
        if (want_gslot) CUBVH_CK(cudaMemcpyAsync(out.gslot, gslot, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
        CUBVH_CK(cudaStreamSynchronize(s));
        out.slot_of_face0 = out.slot0[0];
        for (int c = 0; c < 3; ++c) { out.lo[c] = out.mesh_box[c]; out.hi[c] = out.mesh_box[3 + c]; }
        return 0;
    }
    err = "GPU build: tree deeper than the traversal stack supports";
    return 1;
#undef CUBVH_CK
}

int build_bvh_device(const float* v, int64_t nv, const int64_t* f, int64_t nf, int max_leaf, cudaStream_t s,
                     DeviceBuild& out, std::string& err) {
    if (nf <= 0 || nv <= 0) { err = "empty mesh"; return 1; }
    return build_meshes_device(v, f, {0, nv}, {0, nf}, {max_leaf}, s, out, err, false);
}

}  // namespace cubvh
