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
//   1. tile     one block per tile of T consecutive rows of one z-slice,
//               four bitmask words per thread: packs the tile's free-voxel
//               bitmask (one 32-bit word per 32 voxels) into shared and
//               global memory, marks run starts per word, numbers the tile's
//               runs in linear order with one block-wide scan of the words'
//               start counts (run id = tile * capacity + index in tile, so
//               run ids are ordered like the runs' first voxels), unites the
//               runs of adjacent rows of the tile (y - 1) word by word in a
//               union-find in shared memory (global memory for tiles with
//               more runs than fit), and stores every run's root within the
//               tile
//   2. merge    unites runs across tiles: every row with its z - 1 row, and
//               the first row of each tile with the last row of the tile
//               above; lock-free union-find on the global roots that always
//               links the larger root under the smaller, so every root is
//               its component's smallest run id, i.e. smallest voxel index
//   3. resolve  every run's label = its root's first voxel (for the tiles
//               the label writer does not stage)
//   4. label    one block per tile: the tile's run labels (each run's
//               root's first voxel), start marks and run bases staged in
//               shared memory, then the int32 labels (or the signed
//               distances of udf_to_sdf) written with 16-byte streaming
//               stores; rows of W % 32 != 0 voxels: a warp per 32 words
//               over the resolved labels
// The tile kernel keeps the bitmask and every row's first run id (rowid);
// for the row-wise label writer (rows of W % 32 != 0 voxels) also per word
// its run starts (starts) and the id of the last run that starts before it
// (wbase: the run covering bit x of word w is wbase[w] + popc(starts[w] &
// bits 0..x) - 1).  The tile label writer recomputes both from the bitmask.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "launches.h"
#include "kernels.h"

namespace cubvh {
namespace {

constexpr int kStepLimit = 1 << 24;   // bound on any union-find walk
// 256 threads and 1,024 words per tile: four tiles in flight per SM (512
// threads: tile kernel 93 -> 73 us at 512^3; 128 threads: the tile kernel is
// faster still but the merge, with twice the tile boundaries, slower)
constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;
// the tile kernel at 40 registers: six tiles in flight per SM (512^3 tile
// kernel 74 -> 65 us against four; eight spill and are slower)
constexpr int kTileBlocksPerSM = 6;
constexpr int kTileWords = 4 * kTileThreads;   // bitmask words per tile chunk: four per thread
constexpr int kSmemRuns = 12 * kTileThreads;   // a tile's runs unite (and are labelled) in shared memory up to this count

struct FFPlan {
    int64_t rows, wpr, words, ntot;
    int H, W;
    int wpr_shift;                     // log2(wpr) when wpr is a power of two, else -1
    int tile_rows;                     // T: rows per tile; a tile never spans two z-slices
    int64_t tiles_per_slice, ntiles;
    int64_t cap;                       // run ids per tile: T * ceil(W / 2)
    size_t off_bits, off_starts, off_wbase, off_rowid, off_tcount, off_start, off_parent, off_status, total;
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

FFPlan make_plan(int B, int H, int W, int D) {
    FFPlan p{};
    p.H = H; p.W = W;
    p.rows = (int64_t)B * D * H;
    p.wpr = (W + 31) / 32;
    p.words = p.rows * p.wpr;
    p.ntot = p.rows * W;
    p.wpr_shift = -1;
    for (int k = 0; k < 31; ++k)
        if (((int64_t)1 << k) == p.wpr) p.wpr_shift = k;
    // rows per tile: about kTileWords words (one chunk), the slice split evenly;
    // rows of more than kTileWords words: one row per tile, in several chunks
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
    size_t o = 0;
    p.off_bits = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_starts = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_wbase = o; o = align256(o + sizeof(uint32_t) * p.words);
    p.off_rowid = o; o = align256(o + sizeof(uint32_t) * p.rows);
    p.off_tcount = o; o = align256(o + sizeof(uint32_t) * p.ntiles);
    p.off_start = o; o = align256(o + sizeof(int32_t) * p.ntiles * p.cap);
    p.off_parent = o; o = align256(o + sizeof(int32_t) * p.ntiles * p.cap);
    p.off_status = o; o = align256(o + 16);
    p.total = o;
    return p;
}

// Row and position in the row of bitmask word w.
__device__ __forceinline__ void word_pos(int64_t w, int64_t wpr, int shift, int64_t& row, int64_t& wi) {
    if (shift >= 0) { row = w >> shift; wi = w & (wpr - 1); }
    else { row = w / wpr; wi = w - row * wpr; }
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
    float* d;   // vec: receives udf - eps (the unsigned part of the signed grid) as the udf is read
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
    float4* d = reinterpret_cast<float4*>(s.d + v0);
    const int nch = 8 * nwords;  // 4 voxels per chunk
    for (int c0 = 0; c0 < nch; c0 += 4 * kTileThreads) {
        float4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            v[j] = c < nch ? __ldcs(u + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * kTileThreads + (int)threadIdx.x;
            if (c < nch)
                __stcs(d + c, make_float4(__fsub_rn(v[j].x, s.eps), __fsub_rn(v[j].y, s.eps), __fsub_rn(v[j].z, s.eps),
                                          __fsub_rn(v[j].w, s.eps)));
            uint32_t m = (!(v[j].x < s.eps) ? 1u : 0u) | (!(v[j].y < s.eps) ? 2u : 0u) |
                         (!(v[j].z < s.eps) ? 4u : 0u) | (!(v[j].w < s.eps) ? 8u : 0u);
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 1) << 4;
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 2) << 8;
            m |= __shfl_down_sync(0xFFFFFFFFu, m, 4) << 16;
            if (c < nch && (c & 7) == 0) put_word(sout, gout, c >> 3, m);
        }
    }
}

// Exclusive scan of one value per thread over the block (kTileThreads
// threads); *total receives the block's sum.  Called by all threads; wsum:
// kTileWarps + 1 words of shared memory, free again after the next barrier.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* wsum, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t x = lane < kTileWarps ? wsum[lane] : 0u;
        uint32_t xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, xi, o);
            if (lane >= o) xi += t;
        }
        if (lane < kTileWarps) wsum[lane] = xi - x;     // exclusive warp offsets
        if (lane == kTileWarps - 1) wsum[kTileWarps] = xi;
    }
    __syncthreads();
    *total = wsum[kTileWarps];
    return wsum[warp] + inc - v;
}

// 1. One block per tile (rows r0 .. r0 + T - 1 of one z-slice), in chunks
// of kTileWords bitmask words (one chunk unless a row has more words; such
// tiles hold one row, whose runs have no y - 1 neighbour inside the tile).
// Thread t owns words 4t .. 4t + 3 of the chunk.
template <class Src>
__global__ void __launch_bounds__(kTileThreads, kTileBlocksPerSM)
k_ff_tile(Src src, int W, int64_t wpr, int shift, int T, int64_t tiles_per_slice, int H, int64_t cap,
          bool store_words, uint32_t* __restrict__ bits, uint32_t* __restrict__ starts, uint32_t* __restrict__ wbase,
          uint32_t* __restrict__ rowid,
          uint32_t* __restrict__ tcount, int32_t* __restrict__ start, int32_t* __restrict__ parent,
          int* __restrict__ status) {
    __shared__ __align__(16) uint32_t sbits[kTileWords];
    __shared__ __align__(16) uint32_t sw[kTileWords];   // runs of the tile before each word
    __shared__ uint32_t wsum[32];
    __shared__ int32_t spar[kSmemRuns];
    const int64_t tile = blockIdx.x;
    const int64_t slice = tile / tiles_per_slice;
    const int y0 = (int)(tile - slice * tiles_per_slice) * T;
    const int nrow = min(T, H - y0);                  // rows of this tile
    const int64_t r0 = slice * H + y0;                // first row
    const int64_t tbase = tile * cap;                 // first run id of the tile
    const int64_t w0 = r0 * wpr;                      // first word
    const int64_t nwords = (int64_t)nrow * wpr;
    const bool one = nwords <= kTileWords;
    const int t4 = 4 * (int)threadIdx.x;
    int32_t* par = parent + tbase;                    // shared memory when the tile's runs fit
    uint32_t carry = 0;                               // runs in earlier chunks
    for (int64_t c0 = 0; c0 < nwords; c0 += kTileWords) {
        const int nw = (int)min((int64_t)kTileWords, nwords - c0);
        const int64_t g0 = w0 + c0;                   // first word of the chunk
        // free-voxel bitmask of the chunk
        if (src.vec) {
            pack_vec(src, g0 * 32, nw, sbits, bits + g0);
        } else {
            const int lane = threadIdx.x & 31;
            for (int k = threadIdx.x >> 5; k < nw; k += kTileWarps) {
                int64_t row, wi;
                word_pos(g0 + k, wpr, shift, row, wi);
                const int x = (int)wi * 32 + lane;
                const bool fr = x < W && src.free_at(row * W + x);
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, fr);
                if (lane == 0) put_word(sbits, bits + g0, k, m);
            }
        }
        __syncthreads();
        // run starts of the thread's words, their counts scanned over the block
        uint32_t st[4], tot = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int w = t4 + j;
            st[j] = 0u;
            if (w < nw) {
                int64_t row, wi;
                word_pos(g0 + w, wpr, shift, row, wi);
                const uint32_t prev = wi == 0 ? 0u : (w > 0 ? sbits[w - 1] : bits[g0 - 1]);
                st[j] = starts_of(sbits[w], prev);
            }
            tot += __popc(st[j]);
        }
        uint32_t total;
        const uint32_t ex = carry + block_exclusive(tot, wsum, &total);
        if (one) par = carry + total <= (uint32_t)kSmemRuns ? spar : parent + tbase;
        // per word: its starts, its run base, and each run's first voxel and self parent
        uint32_t run = ex;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int w = t4 + j;
            if (w < nw) {
                sw[w] = run;
                if (store_words) {
                    starts[g0 + w] = st[j];
                    wbase[g0 + w] = (uint32_t)(tbase + run);
                }
                int64_t row, wi;
                word_pos(g0 + w, wpr, shift, row, wi);
                if (wi == 0) rowid[row] = (uint32_t)(tbase + run);   // the row's first run
                if (st[j]) {
                    const int64_t v0 = row * W + wi * 32;   // < 2^31 voxels (host check)
                    uint32_t sj = st[j];
                    int32_t id = (int32_t)run;
                    while (sj) {
                        const int x = __ffs(sj) - 1;
                        sj &= sj - 1;
                        start[tbase + id] = (int32_t)(v0 + x);
                        par[id] = id;
                        ++id;
                    }
                }
            }
            run += __popc(st[j]);
        }
        carry += total;
        __syncthreads();
    }
    const int32_t nruns = (int32_t)carry;
    if (threadIdx.x == 0) tcount[tile] = carry;
    // y - 1 neighbours inside the tile, word by word: at every maximal common
    // free segment and every run start inside one, unite the two runs
    // covering that voxel (uniting rows in binary-tree rounds instead, which
    // bounds the forest's depth, measured 40 % slower: the rounds' barriers
    // cost more than the longer paths)
    if (one && nrow > 1) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int w = t4 + j;
            if (w < wpr || w >= nwords) continue;
            const int q = w - (int)wpr;
            int64_t row, wi;
            word_pos(w0 + w, wpr, shift, row, wi);
            const uint32_t pw = wi ? sbits[w - 1] : 0u, pq = wi ? sbits[q - 1] : 0u;
            const uint32_t f = sbits[w], fq = sbits[q];
            const uint32_t sr = starts_of(f, pw), sq = starts_of(fq, pq);
            const uint32_t m = f & fq;
            uint32_t ev = m & (starts_of(m, pw & pq) | sr | sq);
            while (ev) {
                const int x = __ffs(ev) - 1;
                ev &= ev - 1;
                const uint32_t upto = (x == 31) ? 0xFFFFFFFFu : ((2u << x) - 1u);
                uf_union(par, (int32_t)(sw[w] + __popc(sr & upto)) - 1, (int32_t)(sw[q] + __popc(sq & upto)) - 1,
                         status);
            }
        }
        __syncthreads();
    }
    // roots within the tile (in place, local ids), then as global run ids
    for (int32_t i = threadIdx.x; i < nruns; i += kTileThreads) par[i] = uf_root(par, i, status);
    __syncthreads();
    for (int32_t i = threadIdx.x; i < nruns; i += kTileThreads) parent[tbase + i] = (int32_t)tbase + par[i];
}

// 2. Unions across tiles: row r with its z - 1 row (r - H), and the first row
// of a tile with the row above it (y - 1) when that row is in another tile.
// A row's first run id is rowid[row].  At every maximal
// common free segment of the two rows and every run start inside one, the
// two runs covering that voxel are united, through their current parents
// (the tile kernel left every run pointing at its tile root): consecutive
// rows of a tile mostly give the same pair of roots, so each thread keeps
// its first kMergePairs distinct pairs, lanes holding equal pairs are
// matched across the warp, and one lane per pair unites it (further pairs
// are united directly).
constexpr int kMergePairs = 4;
__global__ void k_ff_merge(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowid,
                           int32_t* __restrict__ parent, int* __restrict__ status, int64_t rows, int64_t wpr, int H,
                           int D, int T) {
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t r = t >> 1;
    const int dir = (int)(t & 1);
    bool valid = t < 2 * rows;
    if (valid) {
        const int64_t rl = r % ((int64_t)D * H);
        const int y = (int)(rl % H), z = (int)(rl / H);
        valid = dir == 0 ? (y != 0 && y % T == 0) : z != 0;
    }
    uint64_t pairs[kMergePairs];
    int np = 0;
    if (valid) {
        const int64_t q = r - (dir == 0 ? 1 : H);
        const uint32_t* br = bits + r * wpr;
        const uint32_t* bq = bits + q * wpr;
        int32_t cr = (int32_t)rowid[r], cq = (int32_t)rowid[q];
        uint32_t pr = 0, pq = 0, pm = 0;
        // words four at a time (16-byte loads when the rows are 16-byte aligned)
        const bool v4 = (wpr & 3) == 0;
        for (int64_t w0 = 0; w0 < wpr; w0 += 4) {
            uint32_t fr4[4], fq4[4];
            if (v4) {
                const uint4 a = *reinterpret_cast<const uint4*>(br + w0), c = *reinterpret_cast<const uint4*>(bq + w0);
                fr4[0] = a.x; fr4[1] = a.y; fr4[2] = a.z; fr4[3] = a.w;
                fq4[0] = c.x; fq4[1] = c.y; fq4[2] = c.z; fq4[3] = c.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    fr4[j] = w0 + j < wpr ? br[w0 + j] : 0u;
                    fq4[j] = w0 + j < wpr ? bq[w0 + j] : 0u;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t fr = fr4[j], fq = fq4[j];
                const uint32_t sr = starts_of(fr, pr), sq = starts_of(fq, pq);
                const uint32_t m = fr & fq;
                uint32_t ev = m & (starts_of(m, pm) | sr | sq);
                pr = fr; pq = fq; pm = m;
                while (ev) {
                    const int x = __ffs(ev) - 1;
                    ev &= ev - 1;
                    const uint32_t upto = (x == 31) ? 0xFFFFFFFFu : ((2u << x) - 1u);
                    const int32_t ra = parent[cr + __popc(sr & upto) - 1], rb = parent[cq + __popc(sq & upto) - 1];
                    if (ra == rb) continue;
                    const uint64_t key = ra < rb ? ((uint64_t)(uint32_t)ra << 32) | (uint32_t)rb
                                                 : ((uint64_t)(uint32_t)rb << 32) | (uint32_t)ra;
                    if (np > 0 && pairs[np - 1] == key) continue;
                    if (np < kMergePairs) pairs[np++] = key;
                    else uf_union(parent, ra, rb, status);
                }
                cr += __popc(sr);
                cq += __popc(sq);
            }
        }
    }
#pragma unroll
    for (int e = 0; e < kMergePairs; ++e) {
        const bool has = e < np;
        const unsigned act = __ballot_sync(0xFFFFFFFFu, has);
        if (!act) break;
        if (has) {
            const unsigned same = __match_any_sync(act, pairs[e]);
            if (__ffs(same) - 1 == lane)
                uf_union(parent, (int32_t)(pairs[e] >> 32), (int32_t)(uint32_t)pairs[e], status);
        }
    }
}

// 3. start[run] := start[root] for every run of the tiles with more than
// `skip_upto` runs (a root's own entry is already its label, and only
// non-root entries are written, so concurrent readers of roots' entries see
// final values).  The tile label writer resolves the runs of the tiles it
// stages in shared memory itself (skip_upto = kSmemRuns).
__global__ void k_ff_resolve(const uint32_t* __restrict__ tcount, int64_t ntiles, int64_t cap,
                             const int32_t* __restrict__ parent, int32_t* __restrict__ start,
                             int* __restrict__ status, uint32_t skip_upto) {
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int32_t n = (int32_t)tcount[tile];
        if ((uint32_t)n <= skip_upto) continue;
        const int32_t base = (int32_t)(tile * cap);
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const int32_t g = base + i;
            const int32_t root = uf_root(parent, g, status);
            if (root != g) start[g] = start[root];
        }
    }
}

// 4 (W % 32 == 0, 16-byte aligned output).  One block per tile: the tile's
// run labels (up to kSmemRuns) and its words' free bits are staged in shared
// memory with coalesced loads, the words' run starts and run bases
// (tile-relative) recomputed from the bits with one block-wide scan, then
// each thread writes groups of 4 voxels (bits 4k .. 4k + 3 of a word) with
// 16-byte streaming stores, consecutive threads consecutive groups.
// SDF: the signed distance s = udf - eps instead of the label, negated where
// the voxel's label (-1 when occupied) differs from the label of its
// volume's first voxel (b, 0, 0, 0) and s > 0; the tile kernel has already
// stored s (reading the udf once), so only groups holding a voxel to negate
// are read and rewritten.
template <bool SDF>
__global__ void __launch_bounds__(kTileThreads)
k_write_tile(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ rowid,
             const uint32_t* __restrict__ tcount, const int32_t* __restrict__ runlab,
             const int32_t* __restrict__ parent, int* __restrict__ status, int64_t wpr, int shift, int T,
             int64_t tiles_per_slice, int H, int64_t cap, int4* __restrict__ labels, float4* __restrict__ sdf,
             int64_t rows_per_volume) {
    __shared__ int32_t slab[kSmemRuns];
    __shared__ __align__(16) uint32_t sf[kTileWords], ss[kTileWords], sb[kTileWords];
    __shared__ uint32_t wsum[32];
    const int64_t tile = blockIdx.x;
    const int64_t slice = tile / tiles_per_slice;
    const int y0 = (int)(tile - slice * tiles_per_slice) * T;
    const int nrow = min(T, H - y0);
    const int64_t r0 = slice * H + y0;
    const int64_t tbase = tile * cap;
    const int64_t w0 = r0 * wpr;
    const int64_t nwords = (int64_t)nrow * wpr;
    const uint32_t n = tcount[tile];
    const bool inl = n <= (uint32_t)kSmemRuns;
    int32_t empty = -1;
    if (SDF) {
        const int64_t rv = (r0 / rows_per_volume) * rows_per_volume;
        if (bits[rv * wpr] & 1u) empty = runlab[uf_root(parent, (int32_t)rowid[rv], status)];
    }
    // staged tiles: each run's label is its root's first voxel (k_ff_resolve
    // skipped these tiles); other tiles' labels were resolved in place
    bool other = !inl;   // SDF: the tile may hold a run whose label differs from empty
    if (inl)
        for (uint32_t i = threadIdx.x; i < n; i += kTileThreads) {
            const int32_t l = runlab[uf_root(parent, (int32_t)(tbase + i), status)];
            slab[i] = l;
            other |= l != empty;
        }
    // SDF: sdf already holds udf - eps, and only free voxels of runs labelled
    // differently from the volume's first voxel can flip; a tile with none
    // is done
    if (SDF && !__syncthreads_or(other)) return;
    const int32_t* lab = inl ? slab : runlab + tbase;
    const int t4 = 4 * (int)threadIdx.x;
    uint32_t carry = 0;   // runs of the tile in earlier chunks
    for (int64_t c0 = 0; c0 < nwords; c0 += kTileWords) {
        const int nw = (int)min((int64_t)kTileWords, nwords - c0);
        const int64_t g0 = w0 + c0;
        __syncthreads();   // the previous chunk's words have been read
        for (int k = threadIdx.x; k < nw; k += kTileThreads) sf[k] = bits[g0 + k];
        __syncthreads();
        // run starts of the thread's words and the tile-relative index of the
        // last run before each word (block-wide scan of the start counts)
        uint32_t stw[4], tot = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int w = t4 + j;
            stw[j] = 0u;
            if (w < nw) {
                int64_t k, wi;
                word_pos(c0 + w, wpr, shift, k, wi);
                const uint32_t prev = wi == 0 ? 0u : (w > 0 ? sf[w - 1] : bits[g0 - 1]);
                stw[j] = starts_of(sf[w], prev);
            }
            tot += __popc(stw[j]);
        }
        uint32_t total;
        uint32_t run = carry + block_exclusive(tot, wsum, &total);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (t4 + j < nw) { ss[t4 + j] = stw[j]; sb[t4 + j] = run; }
            run += __popc(stw[j]);
        }
        carry += total;
        __syncthreads();
        for (int g = threadIdx.x; g < 8 * nw; g += kTileThreads) {
            const size_t i4 = (size_t)g0 * 8 + g;     // 16-byte group of the whole grid
            const int k = g >> 3;
            const uint32_t q = (uint32_t)(g & 7) * 4;
            const uint32_t f = sf[k], st = ss[k], base = sb[k];
            uint32_t cnt = base + __popc(st & ((1u << q) - 1u));   // runs starting before bit q, plus the base
            int32_t o[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                cnt += (st >> (q + j)) & 1u;
                o[j] = ((f >> (q + j)) & 1u) ? lab[cnt - 1] : -1;
            }
            if (SDF) {
                // sdf already holds udf - eps (written by the tile kernel); a
                // voxel flips when its label differs from the volume's first
                // voxel's and the value is positive, which needs a free voxel
                // (occupied ones have udf < eps), so groups without a free
                // voxel of another component stay as they are
                bool any = false;
#pragma unroll
                for (int j = 0; j < 4; ++j) any |= o[j] >= 0 && o[j] != empty;
                if (any) {
                    const float4 v = sdf[i4];
                    float d[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (o[j] != empty && d[j] > 0.f) d[j] = -d[j];
                    __stcs(sdf + i4, make_float4(d[0], d[1], d[2], d[3]));
                }
            } else {
                __stcs(labels + i4, make_int4(o[0], o[1], o[2], o[3]));
            }
        }
        __syncthreads();
    }
}

// 4 (rows of W % 32 != 0 voxels): one warp writes 32 consecutive voxels per
// store (128 B).  Lane k of the warp decodes word w0 + k once (its row, its
// first voxel and how many of its 32 bits lie inside the row); the loop over
// the 32 words then only shuffles those values.  SDF as k_write_tile.
template <bool SDF>
__global__ void k_write_rows(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ starts,
                             const uint32_t* __restrict__ wbase, const int32_t* __restrict__ runlab,
                             int32_t* __restrict__ labels, const float* __restrict__ udf, float* __restrict__ sdf,
                             int64_t rows, int64_t wpr, int W, int64_t rows_per_volume, float eps) {
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
            s = starts[wk];
            base = wbase[wk];
            vb = (uint32_t)(r * W + wi * 32);   // < 2^31 voxels (checked on the host)
            nval = min(32, W - (int)wi * 32);
            if (SDF) {
                const int64_t rv = (r / rows_per_volume) * rows_per_volume;
                if (bits[rv * wpr] & 1u) empty = __ldg(runlab + wbase[rv * wpr]);
            }
        }
        const int nw = (int)min((int64_t)32, words - w0);
        for (int k = 0; k < nw; ++k) {
            const uint32_t fk = __shfl_sync(0xFFFFFFFFu, f, k);
            const uint32_t sk = __shfl_sync(0xFFFFFFFFu, s, k);
            const uint32_t bk = __shfl_sync(0xFFFFFFFFu, base, k);
            const uint32_t vk = __shfl_sync(0xFFFFFFFFu, vb, k);
            const int nk = __shfl_sync(0xFFFFFFFFu, nval, k);
            const int32_t ek = SDF ? __shfl_sync(0xFFFFFFFFu, empty, k) : -1;
            if (lane < nk) {
                int32_t lab = -1;
                if ((fk >> lane) & 1u) lab = __ldg(runlab + (bk + __popc(sk & below) - 1));
                if (SDF) {
                    const float d = __fsub_rn(__ldcs(udf + vk + lane), eps);
                    __stcs(sdf + vk + lane, (lab != ek && d > 0.f) ? -d : d);
                } else {
                    __stcs(labels + vk + lane, lab);
                }
            }
        }
    }
}

__global__ void k_zero(int* p) { *p = 0; }

struct FFBufs {
    uint32_t *bits, *starts, *wbase, *rowid, *tcount;
    int32_t *start, *parent;
    int* status;
};
FFBufs carve(const FFPlan& p, void* ws) {
    char* base = static_cast<char*>(ws);
    return FFBufs{reinterpret_cast<uint32_t*>(base + p.off_bits), reinterpret_cast<uint32_t*>(base + p.off_starts),
                  reinterpret_cast<uint32_t*>(base + p.off_wbase), reinterpret_cast<uint32_t*>(base + p.off_rowid),
                  reinterpret_cast<uint32_t*>(base + p.off_tcount),
                  reinterpret_cast<int32_t*>(base + p.off_start), reinterpret_cast<int32_t*>(base + p.off_parent),
                  reinterpret_cast<int*>(base + p.off_status)};
}

// 1-3: tiles, cross-tile unions, run labels (start[] := label of each run)
// tile_writer: the labels are written by k_write_tile, which resolves the
// runs of the tiles it stages itself.
template <class Src>
void label_runs(const FFPlan& p, int D, const Src& src, const FFBufs& b, unsigned sgrid, bool tile_writer,
                cudaStream_t stream) {
    k_zero<<<1, 1, 0, stream>>>(b.status); count_launch();
    k_ff_tile<Src><<<(unsigned)p.ntiles, kTileThreads, 0, stream>>>(
        src, p.W, p.wpr, p.wpr_shift, p.tile_rows, p.tiles_per_slice, p.H, p.cap, !tile_writer, b.bits, b.starts,
        b.wbase, b.rowid, b.tcount, b.start, b.parent, b.status); count_launch();
    const unsigned mgrid = (unsigned)((2 * p.rows + 255) / 256);
    k_ff_merge<<<mgrid, 256, 0, stream>>>(b.bits, b.rowid, b.parent, b.status, p.rows, p.wpr, p.H, D,
                                          p.tile_rows); count_launch();
    k_ff_resolve<<<sgrid, 256, 0, stream>>>(b.tcount, p.ntiles, p.cap, b.parent, b.start, b.status,
                                            tile_writer ? (uint32_t)kSmemRuns : 0u); count_launch();
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
    const bool tile_writer = W % 32 == 0 && (reinterpret_cast<uintptr_t>(labels) & 15) == 0;
    label_runs(p, D, src, b, sgrid, tile_writer, stream);
    if (tile_writer) {
        k_write_tile<false><<<(unsigned)p.ntiles, kTileThreads, 0, stream>>>(
            b.bits, b.rowid, b.tcount, b.start, b.parent, b.status, p.wpr, p.wpr_shift, p.tile_rows,
            p.tiles_per_slice, p.H, p.cap, reinterpret_cast<int4*>(labels), nullptr, 1); count_launch();
    } else {
        k_write_rows<false><<<sgrid, 256, 0, stream>>>(b.bits, b.starts, b.wbase, b.start, labels, nullptr, nullptr,
                                                       p.rows, p.wpr, W, 1, 0.f); count_launch();
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
    const UdfSrc src{udf, eps, vec, sdf};
    label_runs(p, D, src, b, sgrid, vec, stream);
    if (vec) {
        k_write_tile<true><<<(unsigned)p.ntiles, kTileThreads, 0, stream>>>(
            b.bits, b.rowid, b.tcount, b.start, b.parent, b.status, p.wpr, p.wpr_shift, p.tile_rows,
            p.tiles_per_slice, p.H, p.cap, nullptr, reinterpret_cast<float4*>(sdf), (int64_t)D * H);
        count_launch();
    } else {
        k_write_rows<true><<<sgrid, 256, 0, stream>>>(b.bits, b.starts, b.wbase, b.start, nullptr, udf, sdf, p.rows,
                                                      p.wpr, W, (int64_t)D * H, eps); count_launch();
    }
    return cudaGetLastError();
}

}  // namespace cubvh
