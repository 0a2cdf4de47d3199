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
// Algorithm (four kernels, no host round trip).  A row is W consecutive
// voxels of memory; a run is a maximal stretch of free voxels in a row.
//   1. tile     one block per tile of T consecutive rows of one z-slice:
//               packs the tile's free-voxel bitmask (one 32-bit word per 32
//               voxels) into shared memory and global memory, counts run
//               starts per row and per word, numbers the tile's runs in
//               linear order (run id = tile * capacity + index in tile, so
//               run ids are ordered like the runs' first voxels), unites the
//               runs of adjacent rows of the tile (y - 1) in a union-find in
//               shared memory (global memory for tiles with more runs than
//               fit), and stores every run's root within the tile
//   2. merge    unites runs across tiles: every row with its z - 1 row, and
//               the first row of each tile with the last row of the tile
//               above; lock-free union-find on the global roots that always
//               links the larger root under the smaller, so every root is
//               its component's smallest run id, i.e. smallest voxel index
//   3. resolve  every run's label = its root's first voxel
//   4. label    the int32 labels, 16-byte streaming stores (or the signed
//               distances of udf_to_sdf)
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "launches.h"
#include "kernels.h"

namespace cubvh {
namespace {

constexpr int kStepLimit = 1 << 24;   // bound on any union-find walk
constexpr int kTileThreads = 512;
constexpr int kTileWords = 2048;       // bitmask words of a tile (8 KB of shared memory)
constexpr int kSmemRuns = 6144;        // a tile's runs unite in shared memory up to this count

struct FFPlan {
    int64_t rows, wpr, words, ntot;
    int H, W;
    int tile_rows;                     // T: rows per tile; a tile never spans two z-slices
    int64_t tiles_per_slice, ntiles;
    int64_t cap;                       // run ids per tile: T * ceil(W / 2)
    bool bits_in_smem;
    size_t smem_bytes;
    size_t off_bits, off_wpref, off_rowoff, off_tcount, off_start, off_parent, off_status, total;
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

FFPlan make_plan(int B, int H, int W, int D) {
    FFPlan p{};
    p.H = H; p.W = W;
    p.rows = (int64_t)B * D * H;
    p.wpr = (W + 31) / 32;
    p.words = p.rows * p.wpr;
    p.ntot = p.rows * W;
    // rows per tile: about kTileWords words, the slice split evenly
    const int64_t tmax = std::max<int64_t>(1, std::min<int64_t>(H, kTileWords / std::max<int64_t>(p.wpr, 1)));
    p.tiles_per_slice = (H + tmax - 1) / tmax;
    p.tile_rows = (int)((H + p.tiles_per_slice - 1) / p.tiles_per_slice);
    p.cap = (int64_t)p.tile_rows * ((W + 1) / 2);
    // run ids must stay below 2^31; one row per tile always does (ceil(W/2) <= W)
    if ((int64_t)B * D * p.tiles_per_slice * p.cap > (int64_t)INT32_MAX) {
        p.tile_rows = 1;
        p.tiles_per_slice = H;
        p.cap = (W + 1) / 2;
    }
    p.ntiles = (int64_t)B * D * p.tiles_per_slice;
    p.bits_in_smem = (int64_t)p.tile_rows * p.wpr <= kTileWords;
    p.smem_bytes = sizeof(uint32_t) * ((p.bits_in_smem ? (size_t)p.tile_rows * p.wpr : 0) + (p.tile_rows + 1) + 32 +
                                       kSmemRuns);
    size_t o = 0;
    p.off_bits = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_wpref = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_rowoff = o; o = align256(o + sizeof(uint32_t) * p.rows);
    p.off_tcount = o; o = align256(o + sizeof(uint32_t) * p.ntiles);
    p.off_start = o; o = align256(o + sizeof(int32_t) * p.ntiles * p.cap);
    p.off_parent = o; o = align256(o + sizeof(int32_t) * p.ntiles * p.cap);
    p.off_status = o; o = align256(o + 16);
    p.total = o;
    return p;
}

__device__ __forceinline__ uint32_t starts_of(uint32_t f, uint32_t prev_word) {
    return f & ~((f << 1) | (prev_word >> 31));
}

// Union-find on int32 parents (shared or global memory through a generic
// pointer).  Parents only decrease; every walk is bounded (status := 1).
__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x, int* status) {
    int32_t p = parent[x];
    int steps = 0;
    while (p != x) {
        const int32_t gp = parent[p];
        if (gp < p) parent[x] = gp;  // path halving
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
// Root of x by reading only (the parents may be shortened concurrently by
// writers that store final roots, which are valid ancestors).
__device__ __forceinline__ int32_t uf_root(const int32_t* parent, int32_t x, int* status) {
    int32_t p = parent[x];
    int steps = 0;
    while (p != x) {
        x = p; p = parent[x];
        if (++steps > kStepLimit) { atomicExch(status, 1); break; }
    }
    return x;
}

// Unites the runs of row r (run ids from cr0) with the overlapping runs of
// row q (run ids from cq0): at every maximal common free segment and every
// run start inside one, the two runs covering that voxel are united.
__device__ __forceinline__ void unite_rows(const uint32_t* br, const uint32_t* bq, int64_t wpr, int32_t cr0,
                                           int32_t cq0, int32_t* parent, int* status) {
    uint32_t pr = 0, pq = 0, pm = 0;
    int32_t cr = cr0, cq = cq0;
    for (int64_t w = 0; w < wpr; ++w) {
        const uint32_t fr = br[w], fq = bq[w];
        const uint32_t sr = starts_of(fr, pr), sq = starts_of(fq, pq);
        const uint32_t m = fr & fq;
        uint32_t ev = m & (starts_of(m, pm) | sr | sq);
        pr = fr; pq = fq; pm = m;
        while (ev) {
            const int x = __ffs(ev) - 1;
            ev &= ev - 1;
            const uint32_t upto = (x == 31) ? 0xFFFFFFFFu : ((2u << x) - 1u);
            uf_union(parent, cr + __popc(sr & upto) - 1, cq + __popc(sq & upto) - 1, status);
        }
        cr += __popc(sr);
        cq += __popc(sq);
    }
}

// Free-voxel sources of the tile kernel: a bool grid (free = 0) or an
// unsigned-distance grid thresholded at eps (free = !(udf < eps), so a NaN
// distance is free).  vec: W % 32 == 0 and a 16-byte aligned array, so a
// tile's voxels are whole words and are read 16 bytes per load.
struct GridSrc {
    const uint8_t* g;
    bool vec;
    __device__ __forceinline__ bool free_at(int64_t i) const { return g[i] == 0; }
};
struct UdfSrc {
    const float* u;
    float eps;
    bool vec;
    __device__ __forceinline__ bool free_at(int64_t i) const { return !(__ldg(u + i) < eps); }
};

// Packs voxels [v0, v0 + 32 * nwords) (whole rows, W % 32 == 0) into nwords
// words, stored to gout[k] and, when sout is not null, sout[k].  Called by
// all threads of the block.
__device__ __forceinline__ void put_word(uint32_t* sout, uint32_t* gout, int k, uint32_t m) {
    if (sout) sout[k] = m;
    gout[k] = m;
}
// bit k set iff byte k of x is zero (the per-byte compare yields 0xFF / 0;
// the multiply gathers the four byte-low bits into bits 24-27, one each)
__device__ __forceinline__ uint32_t zero_bytes4(uint32_t x) {
    return ((__vcmpeq4(x, 0u) & 0x01010101u) * 0x01020408u) >> 24;
}
__device__ __forceinline__ void pack_vec(const GridSrc& s, int64_t v0, int nwords, uint32_t* sout, uint32_t* gout) {
    const uint4* g = reinterpret_cast<const uint4*>(s.g + v0);
    const int nch = 2 * nwords;  // 16 voxels per chunk
    for (int c0 = 0; c0 < nch; c0 += 4 * kTileThreads) {
        uint4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            v[j] = c < nch ? __ldcs(g + c) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            const uint32_t m = zero_bytes4(v[j].x) | (zero_bytes4(v[j].y) << 4) | (zero_bytes4(v[j].z) << 8) |
                               (zero_bytes4(v[j].w) << 12);
            const uint32_t other = __shfl_down_sync(0xFFFFFFFFu, m, 1);
            if (c < nch && (c & 1) == 0) put_word(sout, gout, c >> 1, m | (other << 16));
        }
    }
}
__device__ __forceinline__ void pack_vec(const UdfSrc& s, int64_t v0, int nwords, uint32_t* sout, uint32_t* gout) {
    const float4* u = reinterpret_cast<const float4*>(s.u + v0);
    const int nch = 8 * nwords;  // 4 voxels per chunk
    for (int c0 = 0; c0 < nch; c0 += 4 * kTileThreads) {
        float4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            v[j] = c < nch ? __ldg(u + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            uint32_t m = (!(v[j].x < s.eps) ? 1u : 0u) | (!(v[j].y < s.eps) ? 2u : 0u) |
                         (!(v[j].z < s.eps) ? 4u : 0u) | (!(v[j].w < s.eps) ? 8u : 0u);
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 1) << 4;
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 2) << 8;
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 4) << 16;
            if (c < nch && (c & 7) == 0) put_word(sout, gout, c >> 3, m);
        }
    }
}

// 1. One block per tile (rows r0 .. r0 + T - 1 of one z-slice).
template <class Src>
__global__ void __launch_bounds__(kTileThreads, 2)
k_ff_tile(Src src, int W, int64_t wpr, int T, int64_t tiles_per_slice, int H, int64_t cap, bool bits_in_smem,
          uint32_t* __restrict__ bits, uint32_t* __restrict__ wpref, uint32_t* __restrict__ rowoff,
          uint32_t* __restrict__ tcount, int32_t* __restrict__ start, int32_t* __restrict__ parent,
          int* __restrict__ status) {
    extern __shared__ uint32_t smem[];
    const int64_t tile = blockIdx.x;
    const int64_t slice = tile / tiles_per_slice;
    const int y0 = (int)(tile - slice * tiles_per_slice) * T;
    const int nrow = min(T, H - y0);                  // rows of this tile
    const int64_t r0 = slice * H + y0;                // first row
    const int64_t tbase = tile * cap;                 // first run id of the tile
    const int nwords = (int)(nrow * wpr);
    uint32_t* sbits = smem;
    uint32_t* rowbase = smem + (bits_in_smem ? (int64_t)T * wpr : 0);   // [T + 1]
    uint32_t* wsum = rowbase + T + 1;                                  // [32]
    int32_t* spar = reinterpret_cast<int32_t*>(wsum + 32);             // [kSmemRuns]
    uint32_t* gbits = bits + r0 * wpr;

    // bitmask of the tile
    uint32_t* sout = bits_in_smem ? sbits : nullptr;
    if (src.vec) {
        pack_vec(src, r0 * W, nwords, sout, gbits);
    } else {
        const int lane = threadIdx.x & 31;
        for (int k = threadIdx.x >> 5; k < nwords; k += kTileThreads / 32) {
            const int row = (int)(k / wpr);
            const int x = (int)(k - (int64_t)row * wpr) * 32 + lane;
            const bool fr = x < W && src.free_at((r0 + row) * W + x);
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, fr);
            if (lane == 0) put_word(sout, gbits, k, m);
        }
    }
    __syncthreads();
    const uint32_t* tb = bits_in_smem ? sbits : gbits;
    // run starts per row and per word
    for (int k = threadIdx.x; k < nrow; k += kTileThreads) {
        uint32_t prev = 0, acc = 0;
        for (int64_t w = 0; w < wpr; ++w) {
            const uint32_t f = tb[k * wpr + w];
            wpref[(r0 + k) * wpr + w] = acc;
            acc += __popc(starts_of(f, prev));
            prev = f;
        }
        rowbase[k] = acc;
    }
    __syncthreads();
    // exclusive scan of the row counts (rowbase[nrow] = the tile's runs)
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        constexpr int kWarps = kTileThreads / 32;
        const int per = (nrow + kTileThreads - 1) / kTileThreads;
        const int b0 = threadIdx.x * per, b1 = min(b0 + per, nrow);
        uint32_t sum = 0;
        for (int i = b0; i < b1; ++i) sum += rowbase[i];
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint32_t v = lane < kWarps ? wsum[lane] : 0u, vi = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, vi, o);
                if (lane >= o) vi += t;
            }
            if (lane < kWarps) wsum[lane] = vi - v;   // exclusive warp offsets
        }
        __syncthreads();
        uint32_t run = wsum[warp] + inc - sum;
        for (int i = b0; i < b1; ++i) {
            const uint32_t c = rowbase[i];
            rowbase[i] = run;
            run += c;
        }
        if (b0 < nrow && b1 == nrow) rowbase[nrow] = run;
    }
    __syncthreads();
    const int32_t nruns = (int32_t)rowbase[nrow];
    int32_t* par = nruns <= kSmemRuns ? spar : parent + tbase;
    if (threadIdx.x == 0) tcount[tile] = (uint32_t)nruns;
    // run records: rowoff, the runs' first voxels, self parents
    for (int k = threadIdx.x; k < nrow; k += kTileThreads) {
        const int64_t r = r0 + k;
        rowoff[r] = (uint32_t)(tbase + rowbase[k]);
        int32_t id = (int32_t)rowbase[k];
        uint32_t prev = 0;
        for (int64_t w = 0; w < wpr; ++w) {
            const uint32_t f = tb[k * wpr + w];
            uint32_t sw = starts_of(f, prev);
            prev = f;
            while (sw) {
                const int x = __ffs(sw) - 1;
                sw &= sw - 1;
                start[tbase + id] = (int32_t)(r * W + w * 32 + x);   // < 2^31 voxels (host check)
                par[id] = id;
                ++id;
            }
        }
    }
    __syncthreads();
    // y - 1 neighbours inside the tile
    for (int k = threadIdx.x + 1; k < nrow; k += kTileThreads)
        unite_rows(tb + k * wpr, tb + (k - 1) * wpr, wpr, (int32_t)rowbase[k], (int32_t)rowbase[k - 1], par, status);
    __syncthreads();
    // roots within the tile (in place, local ids), then as global run ids
    for (int32_t i = threadIdx.x; i < nruns; i += kTileThreads) par[i] = uf_root(par, i, status);
    __syncthreads();
    for (int32_t i = threadIdx.x; i < nruns; i += kTileThreads) parent[tbase + i] = (int32_t)tbase + par[i];
}

// 2. Unions across tiles: row r with its z - 1 row (r - H), and the first row
// of a tile with the row above it (y - 1) when that row is in another tile.
__global__ void k_ff_merge(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                           int32_t* __restrict__ parent, int* __restrict__ status, int64_t rows, int64_t wpr, int H,
                           int D, int T) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * rows) return;
    const int64_t r = t >> 1;
    const int dir = (int)(t & 1);
    const int64_t rl = r % ((int64_t)D * H);
    const int y = (int)(rl % H), z = (int)(rl / H);
    if (dir == 0 && (y == 0 || y % T != 0)) return;
    if (dir == 1 && z == 0) return;
    const int64_t q = r - (dir == 0 ? 1 : H);
    unite_rows(bits + r * wpr, bits + q * wpr, wpr, (int32_t)rowoff[r], (int32_t)rowoff[q], parent, status);
}

// 3. start[run] := start[root] for every run (a root's own entry is already
// its label, and only non-root entries are written, so concurrent readers of
// roots' entries see final values).
__global__ void k_ff_resolve(const uint32_t* __restrict__ tcount, int64_t ntiles, int64_t cap,
                             const int32_t* __restrict__ parent, int32_t* __restrict__ start,
                             int* __restrict__ status) {
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int32_t n = (int32_t)tcount[tile];
        const int32_t base = (int32_t)(tile * cap);
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const int32_t g = base + i;
            const int32_t root = uf_root(parent, g, status);
            if (root != g) start[g] = start[root];
        }
    }
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
struct WordRuns {
    uint32_t f, s, base;   // free bits, run starts, run id of the run before the word's first start
};
__device__ __forceinline__ WordRuns word_runs(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowoff,
                                              const uint32_t* __restrict__ wpref, uint32_t w, uint32_t wpr) {
    const uint32_t r = w / wpr, wi = w - r * wpr;
    const uint32_t f = bits[w];
    return WordRuns{f, starts_of(f, wi ? bits[w - 1] : 0u), rowoff[r] + wpref[w]};
}
// labels of bits q .. q + 3 of the word (-1 where occupied)
__device__ __forceinline__ void labels4(const WordRuns& wr, const int32_t* __restrict__ runlab, uint32_t q,
                                        int32_t o[4]) {
    uint32_t cnt = __popc(wr.s & ((1u << q) - 1u));   // run starts below bit q
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cnt += (wr.s >> (q + j)) & 1u;
        o[j] = ((wr.f >> (q + j)) & 1u) ? __ldg(runlab + (wr.base + cnt - 1)) : -1;
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
        labels4(word_runs(bits, rowoff, wpref, w, wpr), runlab, q, o);
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
        labels4(word_runs(bits, rowoff, wpref, w, wpr), runlab, q, o);
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

struct FFBufs {
    uint32_t *bits, *wpref, *rowoff, *tcount;
    int32_t *start, *parent;
    int* status;
};
FFBufs carve(const FFPlan& p, void* ws) {
    char* base = static_cast<char*>(ws);
    return FFBufs{reinterpret_cast<uint32_t*>(base + p.off_bits), reinterpret_cast<uint32_t*>(base + p.off_wpref),
                  reinterpret_cast<uint32_t*>(base + p.off_rowoff), reinterpret_cast<uint32_t*>(base + p.off_tcount),
                  reinterpret_cast<int32_t*>(base + p.off_start), reinterpret_cast<int32_t*>(base + p.off_parent),
                  reinterpret_cast<int*>(base + p.off_status)};
}

// 1-3: tiles, cross-tile unions, run labels (start[] := label of each run)
template <class Src>
void label_runs(const FFPlan& p, int D, const Src& src, const FFBufs& b, unsigned sgrid, cudaStream_t stream) {
    k_zero<<<1, 1, 0, stream>>>(b.status); count_launch();
    k_ff_tile<Src><<<(unsigned)p.ntiles, kTileThreads, p.smem_bytes, stream>>>(
        src, p.W, p.wpr, p.tile_rows, p.tiles_per_slice, p.H, p.cap, p.bits_in_smem, b.bits, b.wpref, b.rowoff,
        b.tcount, b.start, b.parent, b.status); count_launch();
    const unsigned mgrid = (unsigned)((2 * p.rows + 255) / 256);
    k_ff_merge<<<mgrid, 256, 0, stream>>>(b.bits, b.rowoff, b.parent, b.status, p.rows, p.wpr, p.H, D,
                                          p.tile_rows); count_launch();
    k_ff_resolve<<<sgrid, 256, 0, stream>>>(b.tcount, p.ntiles, p.cap, b.parent, b.start, b.status); count_launch();
}

unsigned stream_grid() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)nsm * 8;
}

}  // namespace

size_t floodfill_workspace_bytes(int B, int H, int W, int D) { return make_plan(B, H, W, D).total; }
size_t floodfill_status_offset(int B, int H, int W, int D) { return make_plan(B, H, W, D).off_status; }

cudaError_t launch_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* ws,
                             cudaStream_t stream) {
    const FFPlan p = make_plan(B, H, W, D);
    if (p.ntot <= 0) return cudaSuccess;
    const FFBufs b = carve(p, ws);
    const unsigned sgrid = stream_grid();
    const GridSrc src{grid, W % 32 == 0 && (reinterpret_cast<uintptr_t>(grid) & 15) == 0};
    label_runs(p, D, src, b, sgrid, stream);
    if (W % 32 == 0 && (reinterpret_cast<uintptr_t>(labels) & 15) == 0) {
        k_write4<<<sgrid, 256, 0, stream>>>(b.bits, b.rowoff, b.wpref, b.start, reinterpret_cast<int4*>(labels),
                                            (uint32_t)p.words, (uint32_t)p.wpr); count_launch();
    } else {
        k_write<<<sgrid, 256, 0, stream>>>(b.bits, b.rowoff, b.wpref, b.start, labels, p.rows, p.wpr, W); count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_udf_to_sdf(const float* udf, int B, int H, int W, int D, float eps, float* sdf, void* ws,
                              cudaStream_t stream) {
    const FFPlan p = make_plan(B, H, W, D);
    if (p.ntot <= 0) return cudaSuccess;
    const FFBufs b = carve(p, ws);
    const unsigned sgrid = stream_grid();
    const bool vec = W % 32 == 0 && ((reinterpret_cast<uintptr_t>(udf) | reinterpret_cast<uintptr_t>(sdf)) & 15) == 0;
    const UdfSrc src{udf, eps, vec};
    label_runs(p, D, src, b, sgrid, stream);
    if (vec) {
        k_write_sdf4<<<sgrid, 256, 0, stream>>>(b.bits, b.rowoff, b.wpref, b.start,
                                                reinterpret_cast<const float4*>(udf), reinterpret_cast<float4*>(sdf),
                                                (uint32_t)p.words, (uint32_t)p.wpr, (uint32_t)((int64_t)D * H), eps);
        count_launch();
    } else {
        k_write_sdf<<<sgrid, 256, 0, stream>>>(b.bits, b.rowoff, b.wpref, b.start, udf, sdf, p.rows, p.wpr, W,
                                               (int64_t)D * H, eps); count_launch();
    }
    return cudaGetLastError();
}

}  // namespace cubvh
