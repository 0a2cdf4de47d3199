// Voxel floodfill: 6-connected components of free voxels (grid == 0), every
// free voxel labelled with the smallest global linear index of its
// component, occupied voxels -1.
//
// Reference: include/gpu/floodfill.cuh:14-272 iterates hook / pointer-jump
// passes over int32 labels with a host-side convergence flag and a device
// synchronisation per pass; when it converges its labels are exactly the
// component minima.  Its neighbour decode (x = l % W, y = (l / W) % H,
// z = l / (W*H), strides 1, W, W*H) treats each [H, W, D] volume's memory as
// a C-order [D][H][W] array; this implementation uses the same neighbourhood
// (identical to [H][W][D] when H = W = D).
//
// Algorithm (five passes, no host round trip):
//   1. pack      free-voxel bitmask, one 32-bit word per 32 voxels of a row
//                (a row = W consecutive voxels of memory)
//   2. count     run starts per row and per word (exclusive prefix in row)
//   3. scan      exclusive prefix of the per-row counts -> global run ids in
//                linear order (so run id order == start index order)
//   4. union     runs of adjacent rows (y-1 and z-1) that overlap are merged
//                in a lock-free union-find that always links the larger root
//                under the smaller one: every root is its component's
//                smallest run id, i.e. its smallest voxel index
//   5. label     each run gets its root's start index; the label write is a
//                coalesced streaming store of the int32 output
#include <cstdint>
#include <cuda_runtime.h>

#include "launches.h"
#include "kernels.h"
#include "scan.cuh"

namespace cubvh {
namespace {

constexpr int kStepLimit = 1 << 24;   // bound on any union-find walk

struct FFPlan {
    int64_t rows, wpr, words, max_runs, ntot;
    size_t off_bits, off_wpref, off_rowoff, off_blocksum, off_start, off_parent, off_status, total;
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

FFPlan make_plan(int B, int H, int W, int D) {
    FFPlan p{};
    p.rows = (int64_t)B * D * H;
    p.wpr = (W + 31) / 32;
    p.words = p.rows * p.wpr;
    p.max_runs = p.rows * (int64_t)((W + 1) / 2);
    p.ntot = p.rows * W;
    const int64_t nblk = scan::num_chunks(p.rows);
    size_t o = 0;
    p.off_bits = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_wpref = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_rowoff = o; o = align256(o + sizeof(uint32_t) * (p.rows + 1));
    p.off_blocksum = o; o = align256(o + sizeof(uint32_t) * (nblk + 1));
    p.off_start = o; o = align256(o + sizeof(int32_t) * p.max_runs);
    p.off_parent = o; o = align256(o + sizeof(int32_t) * p.max_runs);
    p.off_status = o; o = align256(o + 16);
    p.total = o;
    return p;
}

// 1. free mask: bit x of word w of row r is set iff voxel r*W + 32w + x is free
__global__ void k_pack(const uint8_t* __restrict__ grid, uint32_t* __restrict__ bits, int64_t rows, int W,
                       int64_t wpr) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t words = rows * wpr;
    for (int64_t w = warp; w < words; w += nwarps) {
        const int64_t r = w / wpr;
        const int x = (int)(w - r * wpr) * 32 + lane;
        bool fr = false;
        if (x < W) fr = grid[r * W + x] == 0;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, fr);
        if (lane == 0) bits[w] = m;
    }
}
// fast path for W % 32 == 0 with a 16-byte aligned grid: one uint4 (16
// voxels) per thread, two threads per 32-bit word
__global__ void k_pack16(const uint4* __restrict__ grid, uint32_t* __restrict__ bits, int64_t n16) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i - (threadIdx.x & 31) < n16; i += stride) {
        uint32_t m = 0;
        if (i < n16) {
            const uint4 v = __ldcs(grid + i);
            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    m |= (((w4[q] >> (8 * b)) & 0xFFu) == 0u ? 1u : 0u) << (4 * q + b);
        }
        const uint32_t other = __shfl_down_sync(0xFFFFFFFFu, m, 1);
        if (i < n16 && (i & 1) == 0) bits[i >> 1] = m | (other << 16);
    }
}

// 1'. free mask of an unsigned-distance grid thresholded at eps: a voxel is
// occupied iff udf < eps (a NaN distance is free, as !(NaN < eps))
__global__ void k_pack_udf(const float* __restrict__ udf, uint32_t* __restrict__ bits, int64_t rows, int W,
                           int64_t wpr, float eps) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t words = rows * wpr;
    for (int64_t w = warp; w < words; w += nwarps) {
        const int64_t r = w / wpr;
        const int x = (int)(w - r * wpr) * 32 + lane;
        bool fr = false;
        if (x < W) fr = !(__ldg(udf + r * W + x) < eps);
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, fr);
        if (lane == 0) bits[w] = m;
    }
}

__device__ __forceinline__ uint32_t starts_of(uint32_t f, uint32_t prev_word) {
    return f & ~((f << 1) | (prev_word >> 31));
}

// 2. run counts: per word, the exclusive prefix of run starts within its row;
// per row, the total.
__global__ void k_count(const uint32_t* __restrict__ bits, uint32_t* __restrict__ wpref,
                        uint32_t* __restrict__ rowcnt, int64_t rows, int64_t wpr) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const uint32_t* b = bits + r * wpr;
    uint32_t prev = 0, acc = 0;
    for (int64_t w = 0; w < wpr; ++w) {
        const uint32_t f = b[w];
        wpref[r * wpr + w] = acc;
        acc += __popc(starts_of(f, prev));
        prev = f;
    }
    rowcnt[r] = acc;
}

// 3. exclusive scan of the per-row counts: scan.cuh

// 4a. run records: start index and self parent
__global__ void k_runs(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                       int32_t* __restrict__ start, int32_t* __restrict__ parent, int64_t rows, int64_t wpr,
                       int W) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    uint32_t id = rowoff[r], prev = 0;
    for (int64_t w = 0; w < wpr; ++w) {
        const uint32_t f = bits[r * wpr + w];
        uint32_t s = starts_of(f, prev);
        prev = f;
        while (s) {
            const int x = __ffs(s) - 1;
            s &= s - 1;
            start[id] = (int32_t)(r * W + w * 32 + x);
            parent[id] = (int32_t)id;
            ++id;
        }
    }
}

__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x, int* status) {
    int32_t p = parent[x];
    int steps = 0;
    while (p != x) {
        const int32_t gp = parent[p];
        if (gp < p) parent[x] = gp;  // path halving; parents only decrease
        x = p; p = gp;
        if (++steps > kStepLimit) { atomicExch(status, 1); break; }
    }
    return x;
}
__device__ __forceinline__ void uf_union(int32_t* parent, int32_t a, int32_t b, int* status) {
    a = uf_find(parent, a, status);
    b = uf_find(parent, b, status);
    int steps = 0;
    while (a != b) {
        if (a > b) { const int32_t t = a; a = b; b = t; }
        // link root b under a; fails if b is no longer a root
        const int32_t old = atomicCAS(&parent[b], b, a);
        if (old == b) break;
        b = uf_find(parent, old, status);
        if (++steps > kStepLimit) { atomicExch(status, 1); break; }
    }
}

// 4b. merge overlapping runs of row r and row r - dr (dr = 1 for y-1 when
// y > 0, dr = H for z-1 when z > 0).  For each maximal common free segment,
// and at every run start inside it, the two runs covering that voxel are
// united.
__global__ void k_union(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                        const uint32_t* __restrict__ wpref, int32_t* __restrict__ parent, int* __restrict__ status,
                        int64_t rows, int64_t wpr, int H, int D) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * rows) return;
    const int64_t r = t >> 1;
    const int dir = (int)(t & 1);
    const int64_t rl = r % ((int64_t)D * H);
    const int y = (int)(rl % H), z = (int)(rl / H);
    if (dir == 0 && y == 0) return;
    if (dir == 1 && z == 0) return;
    const int64_t q = r - (dir == 0 ? 1 : H);
    const uint32_t* br = bits + r * wpr;
    const uint32_t* bq = bits + q * wpr;
    uint32_t pr = 0, pq = 0, pm = 0;
    for (int64_t w = 0; w < wpr; ++w) {
        const uint32_t fr = br[w], fq = bq[w];
        const uint32_t sr = starts_of(fr, pr), sq = starts_of(fq, pq);
        const uint32_t m = fr & fq;
        uint32_t ev = m & (starts_of(m, pm) | sr | sq);
        pr = fr; pq = fq; pm = m;
        if (!ev) continue;
        const uint32_t cr = rowoff[r] + wpref[r * wpr + w], cq = rowoff[q] + wpref[q * wpr + w];
        while (ev) {
            const int x = __ffs(ev) - 1;
            ev &= ev - 1;
            const uint32_t upto = (x == 31) ? 0xFFFFFFFFu : ((2u << x) - 1u);
            const int32_t a = (int32_t)(cr + __popc(sr & upto) - 1);
            const int32_t b = (int32_t)(cq + __popc(sq & upto) - 1);
            uf_union(parent, a, b, status);
        }
    }
}

// 5a. parent[i] <- root of i.  The walk only reads: the single write per
// entry stores its final root, so a finished entry is never overwritten by
// a stale ancestor (every value read is a valid ancestor either way).
__global__ void k_root(int32_t* __restrict__ parent, const uint32_t* __restrict__ rowoff, int64_t rows,
                       int* __restrict__ status) {
    const uint32_t n = rowoff[rows];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t x = (int32_t)i, p = parent[x];
        int steps = 0;
        while (p != x) {
            x = p; p = parent[x];
            if (++steps > kStepLimit) { atomicExch(status, 1); break; }
        }
        parent[i] = x;
    }
}
__global__ void k_root_label(int32_t* __restrict__ parent, const int32_t* __restrict__ start,
                             const uint32_t* __restrict__ rowoff, int64_t rows) {
    const uint32_t n = rowoff[rows];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        parent[i] = start[parent[i]];
}

// 5b. labels: one warp writes 32 consecutive voxels per store (128 B).  Lane
// k of the warp decodes word w0 + k once (its row, its first voxel and how
// many of its 32 bits lie inside the row); the loop over the 32 words then
// only shuffles those values.
__global__ void k_write(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                        const uint32_t* __restrict__ wpref, const int32_t* __restrict__ runlab,
                        int32_t* __restrict__ labels, int64_t rows, int64_t wpr, int W) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t words = rows * wpr;
    const uint32_t below = (lane == 31) ? 0xFFFFFFFFu : ((2u << lane) - 1u);
    for (int64_t w0 = warp * 32; w0 < words; w0 += nwarps * 32) {
        const int64_t wk = w0 + lane;
        uint32_t f = 0, s = 0, base = 0, vb = 0;
        int nval = 0;
        if (wk < words) {
            const int64_t r = wk / wpr, wi = wk - r * wpr;
            f = bits[wk];
            const uint32_t prev = wi > 0 ? bits[wk - 1] : 0u;
            s = starts_of(f, prev);
            base = rowoff[r] + wpref[wk];
            vb = (uint32_t)(r * W + wi * 32);   // < 2^31 voxels (checked on the host)
            nval = min(32, W - (int)wi * 32);
        }
        const int nw = (int)min((int64_t)32, words - w0);
        for (int k = 0; k < nw; ++k) {
            const uint32_t fk = __shfl_sync(0xFFFFFFFFu, f, k);
            const uint32_t sk = __shfl_sync(0xFFFFFFFFu, s, k);
            const uint32_t bk = __shfl_sync(0xFFFFFFFFu, base, k);
            const uint32_t vk = __shfl_sync(0xFFFFFFFFu, vb, k);
            const int nk = __shfl_sync(0xFFFFFFFFu, nval, k);
            if (lane < nk) {
                int32_t lab = -1;
                if ((fk >> lane) & 1u) lab = __ldg(runlab + (bk + __popc(sk & below) - 1));
                __stcs(labels + vk + lane, lab);
            }
        }
    }
}

// 5b (W % 32 == 0, 16-byte aligned output).  Rows hold whole words, so voxel
// 32 w + b is bit b of word w.  A warp covers 4 words (128 voxels) per step:
// lane l takes word l / 8 and its 4 bits from 4 (l % 8), and writes their
// labels with one 16-byte streaming store (512 contiguous bytes per warp).
__device__ __forceinline__ void run_labels4(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                                            const uint32_t* __restrict__ wpref,
                                            const int32_t* __restrict__ runlab, uint32_t w, uint32_t wpr,
                                            uint32_t q, int32_t o[4]) {
    const uint32_t r = w / wpr, wi = w - r * wpr;
    const uint32_t f = bits[w];
    const uint32_t s = starts_of(f, wi ? bits[w - 1] : 0u);
    const uint32_t base = rowoff[r] + wpref[w];
    uint32_t cnt = __popc(s & ((1u << q) - 1u));   // run starts below bit q
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cnt += (s >> (q + j)) & 1u;
        o[j] = ((f >> (q + j)) & 1u) ? __ldg(runlab + (base + cnt - 1)) : -1;
    }
}
__global__ void k_write4(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                         const uint32_t* __restrict__ wpref, const int32_t* __restrict__ runlab,
                         int4* __restrict__ labels, uint32_t words, uint32_t wpr) {
    const int lane = threadIdx.x & 31;
    const uint32_t sub = (uint32_t)lane >> 3, q = (uint32_t)(lane & 7) * 4;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c * 4 < (int64_t)words; c += nwarps) {
        const uint32_t w = (uint32_t)(c * 4) + sub;
        if (w >= words) continue;
        int32_t o[4];
        run_labels4(bits, rowoff, wpref, runlab, w, wpr, q, o);
        __stcs(labels + (size_t)w * 8 + (lane & 7), make_int4(o[0], o[1], o[2], o[3]));
    }
}

// 5'. signed distances instead of labels: s = udf - eps, negated where the
// voxel's label (-1 when occupied) differs from the label of its volume's
// first voxel (b, 0, 0, 0) and s > 0.  Same traversal of the run tables as
// k_write; the first voxel's label is its row's first run when it is free.
__global__ void k_write_sdf(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                            const uint32_t* __restrict__ wpref, const int32_t* __restrict__ runlab,
                            const float* __restrict__ udf, float* __restrict__ sdf, int64_t rows, int64_t wpr,
                            int W, int64_t rows_per_volume, float eps) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t words = rows * wpr;
    const uint32_t below = (lane == 31) ? 0xFFFFFFFFu : ((2u << lane) - 1u);
    for (int64_t w0 = warp * 32; w0 < words; w0 += nwarps * 32) {
        const int64_t wk = w0 + lane;
        uint32_t f = 0, s = 0, base = 0, vb = 0;
        int nval = 0;
        int32_t empty = -1;
        if (wk < words) {
            const int64_t r = wk / wpr, wi = wk - r * wpr;
            f = bits[wk];
            const uint32_t prev = wi > 0 ? bits[wk - 1] : 0u;
            s = starts_of(f, prev);
            base = rowoff[r] + wpref[wk];
            vb = (uint32_t)(r * W + wi * 32);
            nval = min(32, W - (int)wi * 32);
            const int64_t r0 = (r / rows_per_volume) * rows_per_volume;
            if (bits[r0 * wpr] & 1u) empty = __ldg(runlab + rowoff[r0]);
        }
        const int nw = (int)min((int64_t)32, words - w0);
        for (int k = 0; k < nw; ++k) {
            const uint32_t fk = __shfl_sync(0xFFFFFFFFu, f, k);
            const uint32_t sk = __shfl_sync(0xFFFFFFFFu, s, k);
            const uint32_t bk = __shfl_sync(0xFFFFFFFFu, base, k);
            const uint32_t vk = __shfl_sync(0xFFFFFFFFu, vb, k);
            const int nk = __shfl_sync(0xFFFFFFFFu, nval, k);
            const int32_t ek = __shfl_sync(0xFFFFFFFFu, empty, k);
            if (lane < nk) {
                int32_t lab = -1;
                if ((fk >> lane) & 1u) lab = __ldg(runlab + (bk + __popc(sk & below) - 1));
                const float d = __fsub_rn(__ldcs(udf + vk + lane), eps);
                __stcs(sdf + vk + lane, (lab != ek && d > 0.f) ? -d : d);
            }
        }
    }
}
// 5' (W % 32 == 0, 16-byte aligned udf and sdf): the k_write4 layout, one
// 16-byte load of udf and one 16-byte store of sdf per lane.
__global__ void k_write_sdf4(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                             const uint32_t* __restrict__ wpref, const int32_t* __restrict__ runlab,
                             const float4* __restrict__ udf, float4* __restrict__ sdf, uint32_t words,
                             uint32_t wpr, uint32_t rows_per_volume, float eps) {
    const int lane = threadIdx.x & 31;
    const uint32_t sub = (uint32_t)lane >> 3, q = (uint32_t)(lane & 7) * 4;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c * 4 < (int64_t)words; c += nwarps) {
        const uint32_t w = (uint32_t)(c * 4) + sub;
        if (w >= words) continue;
        int32_t o[4];
        run_labels4(bits, rowoff, wpref, runlab, w, wpr, q, o);
        const uint32_t r0 = (w / wpr / rows_per_volume) * rows_per_volume;
        const int32_t empty = (bits[(size_t)r0 * wpr] & 1u) ? __ldg(runlab + rowoff[r0]) : -1;
        const size_t i4 = (size_t)w * 8 + (lane & 7);
        const float4 u = __ldcs(udf + i4);
        float d[4] = {__fsub_rn(u.x, eps), __fsub_rn(u.y, eps), __fsub_rn(u.z, eps), __fsub_rn(u.w, eps)};
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (o[j] != empty && d[j] > 0.f) d[j] = -d[j];
        __stcs(sdf + i4, make_float4(d[0], d[1], d[2], d[3]));
    }
}

__global__ void k_zero(int* p) { *p = 0; }

// 2-5a. runs, union-find over adjacent rows, run labels (parent[] := label)
void label_runs(const FFPlan& p, int H, int D, uint32_t* bits, uint32_t* wpref, uint32_t* rowoff, uint32_t* bsum,
                int32_t* start, int32_t* parent, int* status, unsigned sgrid, cudaStream_t stream) {
    const unsigned rgrid = (unsigned)((p.rows + 255) / 256);
    k_count<<<rgrid, 256, 0, stream>>>(bits, wpref, rowoff, p.rows, p.wpr); count_launch();
    scan::exclusive(rowoff, bsum, p.rows, stream);
    k_runs<<<rgrid, 256, 0, stream>>>(bits, rowoff, start, parent, p.rows, p.wpr, (int)(p.ntot / p.rows)); count_launch();
    const unsigned ugrid = (unsigned)((2 * p.rows + 255) / 256);
    k_union<<<ugrid, 256, 0, stream>>>(bits, rowoff, wpref, parent, status, p.rows, p.wpr, H, D); count_launch();
    k_root<<<sgrid, 256, 0, stream>>>(parent, rowoff, p.rows, status); count_launch();
    k_root_label<<<sgrid, 256, 0, stream>>>(parent, start, rowoff, p.rows); count_launch();
}

}  // namespace

size_t floodfill_workspace_bytes(int B, int H, int W, int D) { return make_plan(B, H, W, D).total; }
size_t floodfill_status_offset(int B, int H, int W, int D) { return make_plan(B, H, W, D).off_status; }

cudaError_t launch_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* ws,
                             cudaStream_t stream) {
    const FFPlan p = make_plan(B, H, W, D);
    if (p.ntot <= 0) return cudaSuccess;
    char* base = static_cast<char*>(ws);
    uint32_t* bits = reinterpret_cast<uint32_t*>(base + p.off_bits);
    uint32_t* wpref = reinterpret_cast<uint32_t*>(base + p.off_wpref);
    uint32_t* rowoff = reinterpret_cast<uint32_t*>(base + p.off_rowoff);
    uint32_t* bsum = reinterpret_cast<uint32_t*>(base + p.off_blocksum);
    int32_t* start = reinterpret_cast<int32_t*>(base + p.off_start);
    int32_t* parent = reinterpret_cast<int32_t*>(base + p.off_parent);
    int* status = reinterpret_cast<int*>(base + p.off_status);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned sgrid = (unsigned)nsm * 8;

    k_zero<<<1, 1, 0, stream>>>(status); count_launch();
    if (W % 32 == 0 && (reinterpret_cast<uintptr_t>(grid) & 15) == 0) {
        const int64_t n16 = p.ntot / 16;
        k_pack16<<<sgrid, 256, 0, stream>>>(reinterpret_cast<const uint4*>(grid), bits, n16); count_launch();
    } else {
        k_pack<<<sgrid, 256, 0, stream>>>(grid, bits, p.rows, W, p.wpr); count_launch();
    }
    label_runs(p, H, D, bits, wpref, rowoff, bsum, start, parent, status, sgrid, stream);
    if (W % 32 == 0 && (reinterpret_cast<uintptr_t>(labels) & 15) == 0) {
        k_write4<<<sgrid, 256, 0, stream>>>(bits, rowoff, wpref, parent, reinterpret_cast<int4*>(labels),
                                            (uint32_t)p.words, (uint32_t)p.wpr); count_launch();
    } else {
        k_write<<<sgrid, 256, 0, stream>>>(bits, rowoff, wpref, parent, labels, p.rows, p.wpr, W); count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_udf_to_sdf(const float* udf, int B, int H, int W, int D, float eps, float* sdf, void* ws,
                              cudaStream_t stream) {
    const FFPlan p = make_plan(B, H, W, D);
    if (p.ntot <= 0) return cudaSuccess;
    char* base = static_cast<char*>(ws);
    uint32_t* bits = reinterpret_cast<uint32_t*>(base + p.off_bits);
    uint32_t* wpref = reinterpret_cast<uint32_t*>(base + p.off_wpref);
    uint32_t* rowoff = reinterpret_cast<uint32_t*>(base + p.off_rowoff);
    uint32_t* bsum = reinterpret_cast<uint32_t*>(base + p.off_blocksum);
    int32_t* start = reinterpret_cast<int32_t*>(base + p.off_start);
    int32_t* parent = reinterpret_cast<int32_t*>(base + p.off_parent);
    int* status = reinterpret_cast<int*>(base + p.off_status);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned sgrid = (unsigned)nsm * 8;

    k_zero<<<1, 1, 0, stream>>>(status); count_launch();
    k_pack_udf<<<sgrid, 256, 0, stream>>>(udf, bits, p.rows, W, p.wpr, eps); count_launch();
    label_runs(p, H, D, bits, wpref, rowoff, bsum, start, parent, status, sgrid, stream);
    if (W % 32 == 0 && ((reinterpret_cast<uintptr_t>(udf) | reinterpret_cast<uintptr_t>(sdf)) & 15) == 0) {
        k_write_sdf4<<<sgrid, 256, 0, stream>>>(bits, rowoff, wpref, parent, reinterpret_cast<const float4*>(udf),
                                                reinterpret_cast<float4*>(sdf), (uint32_t)p.words, (uint32_t)p.wpr,
                                                (uint32_t)((int64_t)D * H), eps); count_launch();
    } else {
        k_write_sdf<<<sgrid, 256, 0, stream>>>(bits, rowoff, wpref, parent, udf, sdf, p.rows, p.wpr, W,
                                               (int64_t)D * H, eps); count_launch();
    }
    return cudaGetLastError();
}

}  // namespace cubvh
