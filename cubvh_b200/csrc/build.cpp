// Host BVH construction: binned-SAH binary tree, collapsed to 8-wide nodes,
// emitted in breadth-first order with quantised child boxes (layout.h).
//
// The reference builds a BVH4 by centroid median splits on the host
// (src/bvh.cu:515-620) and stores 36-byte nodes; this builder targets the
// 80-byte compressed node instead.  export_reference_format() writes, for
// state_dict, the records of the reference's own build of the same mesh.
//
// The binary tree is built by recursion over triangle ranges; large ranges
// hand their left half to another thread, and the breadth-first collapse
// fills node boxes and triangle records in parallel.  The output does not
// depend on the thread count.  Box arithmetic uses SSE (part of the x86-64
// base instruction set) in the operand order that reproduces std::min /
// std::max bit for bit.
#include "build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <immintrin.h>
#include <functional>
#include <limits>
#include <numeric>
#include <exception>
#include <system_error>
#include <thread>

namespace cubvh {
namespace {

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const float* p) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    void grow(const Box& b) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
    }
    float area() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0.f)) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

// The same box in SSE registers (lane 3 unused).  Every operation gives the
// bits Box's gives: std::min(a, b) is (b < a ? b : a), which is
// _mm_min_ps(b, a), and std::max(a, b) is (a < b ? b : a), _mm_max_ps(b, a);
// the area is computed from the lanes with Box::area's expression.
struct Box4 {
    __m128 lo, hi;  // no initialiser, so arrays of records stay trivial: see empty()
    static Box4 empty() { return Box4{_mm_set1_ps(INFINITY), _mm_set1_ps(-INFINITY)}; }
    void grow(const Box4& b) { lo = _mm_min_ps(b.lo, lo); hi = _mm_max_ps(b.hi, hi); }
    void grow_point(__m128 p) { lo = _mm_min_ps(p, lo); hi = _mm_max_ps(p, hi); }
    Box box() const {
        alignas(16) float l[4], h[4];
        _mm_store_ps(l, lo); _mm_store_ps(h, hi);
        Box r;
        for (int k = 0; k < 3; ++k) { r.lo[k] = l[k]; r.hi[k] = h[k]; }
        return r;
    }
    float area() const {  // Box::area on the lanes: the same rounded hi - lo
        alignas(16) float d[4];
        _mm_store_ps(d, _mm_sub_ps(hi, lo));
        const float dx = d[0], dy = d[1], dz = d[2];
        if (!(dx >= 0.f)) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node2 {
    Box box;
    int left = -1, right = -1;     // internal children
    int begin = 0, count = 0;      // leaf range (count > 0 for leaves)
};

// One triangle's box, centroid and face index: the builder keeps these
// records in the order it partitions them, so every pass over a range reads
// memory sequentially.
struct alignas(16) Prim {
    Box4 box;
    float c[3];
    int id;
};

struct Builder {
    RawVec<Prim> prim;

    static constexpr int kBins = 32;
    static constexpr float kTrav = 1.0f, kIsect = 1.0f;
    // ranges at least this large may build their left half on another thread
    static constexpr int kParMin = 4096;
    int max_leaf = kMaxLeafTris;
    std::atomic<int> spare{0};     // threads that may still be started

    bool take_thread() {
        int s = spare.load();
        while (s > 0 && !spare.compare_exchange_weak(s, s - 1)) {}
        return s > 0;
    }

    static int make_leaf(std::vector<Node2>& nodes, int b, int e, const Box& box) {
        Node2 n; n.box = box; n.begin = b; n.count = e - b;
        nodes.push_back(n);
        return (int)nodes.size() - 1;
    }

    static int bin_of(float c, float lo, float k) {
        const int bi = (int)((c - lo) * k);
        return std::min(std::max(bi, 0), kBins - 1);
    }

    // Binary node for prim[b, e) and its subtree, appended to `nodes`; the
    // returned index is the subtree's root.  The tree depends only on the
    // range's contents, not on which thread or vector builds it.
    int build(int b, int e, std::vector<Node2>& nodes) {
        Box4 box4 = Box4::empty(), cb4 = Box4::empty();
        for (int i = b; i < e; ++i) {
            box4.grow(prim[i].box);
            cb4.grow_point(_mm_loadu_ps(prim[i].c));  // lane 3 reads id: unused
        }
        const Box box = box4.box(), cb = cb4.box();
        const int n = e - b;
        if (n == 1) return make_leaf(nodes, b, e, box);

        // binned SAH over the three axes, all binned in one pass.  Only
        // non-empty bins are visited: every split between two consecutive
        // non-empty bins puts the same triangles on each side at the same
        // cost, and the lowest such split (the one just after the lower
        // bin) is the one a sweep over all bins keeps.
        bool act[3];
        float kk[3];
        for (int ax = 0; ax < 3; ++ax) {
            const float ext = cb.hi[ax] - cb.lo[ax];
            act[ax] = ext > 0.f;
            kk[ax] = act[ax] ? (float)kBins * (1.f - 1e-6f) / ext : 0.f;
        }
        Box4 bb[3][kBins];
        for (auto& row : bb)
            for (Box4& x : row) x = Box4::empty();
        int bc[3][kBins] = {};
        uint32_t used[3] = {0u, 0u, 0u};  // bit i: bin i of the axis is non-empty
        // bin indices of the three axes at once: per lane the same rounded
        // subtract and multiply and the same truncation as bin_of
        const __m128 lo4 = _mm_setr_ps(cb.lo[0], cb.lo[1], cb.lo[2], 0.f);
        const __m128 k4 = _mm_setr_ps(kk[0], kk[1], kk[2], 0.f);
        for (int i = b; i < e; ++i) {
            const Prim& p = prim[i];
            alignas(16) int32_t q[4];
            _mm_store_si128(reinterpret_cast<__m128i*>(q),
                            _mm_cvttps_epi32(_mm_mul_ps(_mm_sub_ps(_mm_loadu_ps(p.c), lo4), k4)));
            for (int ax = 0; ax < 3; ++ax) {
                if (!act[ax]) continue;
                const int bi = std::min(std::max(q[ax], 0), kBins - 1);
                bc[ax][bi]++;
                used[ax] |= 1u << bi;
                bb[ax][bi].grow(p.box);
            }
        }
        float best_cost = INFINITY; int best_axis = -1, best_split = -1;
        for (int ax = 0; ax < 3; ++ax) {
            if (!act[ax]) continue;
            int ne[kBins], nb = 0;
            for (uint32_t m = used[ax]; m; m &= m - 1) ne[nb++] = __builtin_ctz(m);
            if (nb < 2) continue;
            float ra[kBins]; int rc[kBins];  // suffix area / count from non-empty bin j up
            Box4 acc = bb[ax][ne[nb - 1]]; int cnt = bc[ax][ne[nb - 1]];
            for (int j = nb - 2; j >= 1; --j) {
                acc.grow(bb[ax][ne[j]]); cnt += bc[ax][ne[j]];
                ra[j] = acc.area(); rc[j] = cnt;
            }
            ra[nb - 1] = bb[ax][ne[nb - 1]].area(); rc[nb - 1] = bc[ax][ne[nb - 1]];
            acc = Box4::empty(); cnt = 0;
            for (int j = 0; j < nb - 1; ++j) {
                acc.grow(bb[ax][ne[j]]); cnt += bc[ax][ne[j]];
                const float c = acc.area() * cnt + ra[j + 1] * rc[j + 1];
                if (c < best_cost) { best_cost = c; best_axis = ax; best_split = ne[j]; }
            }
        }
        const float parea = std::max(box.area(), 1e-30f);
        const float split_cost = kTrav + kIsect * best_cost / parea;
        if (n <= max_leaf && (best_axis < 0 || kIsect * n <= split_cost))
            return make_leaf(nodes, b, e, box);

        int mid;
        if (best_axis < 0) {
            mid = b + n / 2;  // all centroids coincide: split the range
        } else {
            const float lo = cb.lo[best_axis], k = kk[best_axis];
            auto it = std::partition(prim.begin() + b, prim.begin() + e,
                                     [&](const Prim& p) { return bin_of(p.c[best_axis], lo, k) <= best_split; });
            mid = (int)(it - prim.begin());
            if (mid == b || mid == e) mid = b + n / 2;
        }
        const int me = (int)nodes.size();
        nodes.emplace_back();
        nodes[me].box = box;
        int l, r;
        std::vector<Node2> ln;
        int lroot = -1;
        std::exception_ptr fail;
        std::thread t;
        if (n >= kParMin && take_thread()) {
            // left half on a thread of its own, into its own vector, spliced
            // after the right half (child indices shifted by the splice point)
            ln.reserve(2 * (size_t)(mid - b));
            try {
                t = std::thread([&] {
                    try { lroot = build(b, mid, ln); } catch (...) { fail = std::current_exception(); }
                });
            } catch (const std::system_error&) {  // no thread to be had: build it here
                spare.fetch_add(1);
            }
        }
        if (t.joinable()) {
            try {
                r = build(mid, e, nodes);
            } catch (...) {
                t.join();
                throw;
            }
            t.join();
            spare.fetch_add(1);
            if (fail) std::rethrow_exception(fail);
            const int off = (int)nodes.size();
            for (Node2 nd : ln) {
                if (nd.count == 0) { nd.left += off; nd.right += off; }
                nodes.push_back(nd);
            }
            l = lroot + off;
        } else {
            l = build(b, mid, nodes);
            r = build(mid, e, nodes);
        }
        nodes[me].left = l; nodes[me].right = r;
        return me;
    }
};

// 2^e as a float: built from its exponent bits where 2^e is a normal float
// (the same value std::ldexp(1.0f, e) returns), std::ldexp elsewhere.
float pow2f(int e) {
    if (e >= -126 && e <= 127) {
        const uint32_t bits = (uint32_t)(e + 127) << 23;
        float f;
        std::memcpy(&f, &bits, sizeof(f));
        return f;
    }
    return std::ldexp(1.0f, e);
}

// Smallest e such that o + 255 * 2^e >= hi in float arithmetic.
int pick_exponent(float o, float hi) {
    if (!(hi > o)) return -100;
    int e = (int)std::ceil(std::log2((double)(hi - o) / 255.0)) - 1;
    e = std::max(e, -100);
    while (o + 255.0f * pow2f(e) < hi) ++e;
    return e;
}

void quantise_child(const CNode& nd, int j, const Box& cb, CNode& out) {
    const float o[3] = {nd.ox, nd.oy, nd.oz};
    const int ex[3] = {nd.ex, nd.ey, nd.ez};
    uint8_t* qlo[3] = {out.qlo_x, out.qlo_y, out.qlo_z};
    uint8_t* qhi[3] = {out.qhi_x, out.qhi_y, out.qhi_z};
    for (int k = 0; k < 3; ++k) {
        const float s = pow2f(ex[k]);
        int ql = (int)std::floor((double)(cb.lo[k] - o[k]) / (double)s);
        int qh = (int)std::ceil((double)(cb.hi[k] - o[k]) / (double)s);
        ql = std::min(std::max(ql, 0), 255); qh = std::min(std::max(qh, 0), 255);
        while (ql > 0 && o[k] + (float)ql * s > cb.lo[k]) --ql;
        while (qh < 255 && o[k] + (float)qh * s < cb.hi[k]) ++qh;
        qlo[k][j] = (uint8_t)ql; qhi[k][j] = (uint8_t)qh;
    }
}

void set_frame(CNode& nd, const Box& b) {
    nd.ox = b.lo[0]; nd.oy = b.lo[1]; nd.oz = b.lo[2];
    nd.ex = (int8_t)pick_exponent(b.lo[0], b.hi[0]);
    nd.ey = (int8_t)pick_exponent(b.lo[1], b.hi[1]);
    nd.ez = (int8_t)pick_exponent(b.lo[2], b.hi[2]);
}

// Error scales used by the single-precision distance filter of the query
// kernels: K and K * squared longest edge.
void set_error_scales(CTri& t) {
    const float v[3][3] = {{t.ax, t.ay, t.az}, {t.bx, t.by, t.bz}, {t.cx, t.cy, t.cz}};
    float e2 = 0.f;
    for (int u = 0; u < 3; ++u) {
        const float* q0 = v[u]; const float* q1 = v[(u + 1) % 3];
        const float dx = q1[0] - q0[0], dy = q1[1] - q0[1], dz = q1[2] - q0[2];
        e2 = std::max(e2, dx * dx + dy * dy + dz * dz);
    }
    t.k = tri_error_factor(v[0], v[1], v[2]);
    t.ke2 = t.k * e2;
}

Box tri_box(const CTri& t) {
    Box b;
    const float a[3] = {t.ax, t.ay, t.az}, bb[3] = {t.bx, t.by, t.bz}, c[3] = {t.cx, t.cy, t.cz};
    b.grow(a); b.grow(bb); b.grow(c);
    return b;
}

}  // namespace

int host_build_threads() {
    static const int n = [] {
        const char* v = std::getenv("CUBVH_B200_BUILD_THREADS");
        if (v) {
            char* end = nullptr;
            const long x = std::strtol(v, &end, 10);
            if (end != v && *end == '\0' && x > 0) return (int)std::min<long>(x, 1 << 16);
        }
        return (int)std::max(1u, std::thread::hardware_concurrency());
    }();
    return n;
}

bool build_bvh(const float* xyz, int64_t nf, HostBvh& out, std::string& err, int max_leaf, int threads) {
    if (nf <= 0) { err = "mesh has no faces"; return false; }
    if (nf > (int64_t)(1 << 28)) { err = "too many faces (limit 2^28)"; return false; }
    if (threads <= 0) threads = host_build_threads();
    std::atomic<bool> finite{true};
    parallel_for(nf, threads, 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t i = 9 * lo; i < 9 * hi; ++i)
            if (!std::isfinite(xyz[i])) { finite = false; return; }
    });
    if (!finite) { err = "vertex coordinates must be finite"; return false; }

    if (max_leaf < 1 || max_leaf > kMaxLeafTris) { err = "leaf size must be in [1, 4]"; return false; }
    Builder B;
    B.max_leaf = max_leaf;
    B.spare = threads - 1;
    B.prim.resize(nf);  // uninitialised: filled (first touched) in parallel
    parallel_for(nf, threads, 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t f = lo; f < hi; ++f) {
            Prim& p = B.prim[f];
            Box b; b.grow(xyz + 9 * f); b.grow(xyz + 9 * f + 3); b.grow(xyz + 9 * f + 6);
            p.box.lo = _mm_setr_ps(b.lo[0], b.lo[1], b.lo[2], 0.f);
            p.box.hi = _mm_setr_ps(b.hi[0], b.hi[1], b.hi[2], 0.f);
            for (int k = 0; k < 3; ++k) p.c[k] = 0.5f * (b.lo[k] + b.hi[k]);
            p.id = (int)f;
        }
    });
    std::vector<Node2> nodes;
    nodes.reserve(2 * nf);
    const int root = B.build(0, (int)nf, nodes);

    // collapse to 8-wide: each wide node lists binary-tree nodes as children
    // children of wide node r: open the largest-area internal child in place
    // (its two children take its position) until kWidth children or leaves only
    auto expand = [&](int r, int* ch) {
        if (nodes[r].count > 0) { ch[0] = r; return 1; }
        int m = 2;
        ch[0] = nodes[r].left; ch[1] = nodes[r].right;
        while (m < kWidth) {
            int bi = -1; float ba = -1.f;
            for (int i = 0; i < m; ++i) {
                const Node2& n = nodes[ch[i]];
                if (n.count > 0) continue;
                const float a = n.box.area();
                if (a > ba) { ba = a; bi = i; }
            }
            if (bi < 0) break;
            const int c = ch[bi];
            for (int i = m; i > bi + 1; --i) ch[i] = ch[i - 1];
            ch[bi] = nodes[c].left;
            ch[bi + 1] = nodes[c].right;
            ++m;
        }
        return m;
    };

    out.nodes.clear(); out.tris.clear();
    std::vector<int32_t> soup((size_t)nf);  // soup slot -> face id, filled in leaf order
    int64_t n_soup = 0;
    struct Item { int bin; int level; };
    struct Kids { int ch[kWidth]; int n; };
    std::vector<Item> queue{{root, 1}};
    std::vector<Kids> kids;
    queue.reserve(nodes.size());       // wide nodes <= binary nodes
    kids.reserve(nodes.size());
    out.nodes.reserve(nodes.size());
    out.nodes.emplace_back();
    int max_depth = 1;
    // breadth-first pass: children, slots, child and triangle bases, soup
    // order (the indices depend on the order, so this pass is serial)
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        const Item it = queue[qi];
        Kids k;
        k.n = expand(it.bin, k.ch);
        CNode nd;
        std::memset(&nd, 0, sizeof(nd));
        std::memset(nd.meta, kEmpty, sizeof(nd.meta));
        nd.child_base = (int32_t)out.nodes.size();
        nd.tri_base = (int32_t)n_soup;
        int slot = 0;
        for (int j = 0; j < k.n; ++j) {
            const Node2& c = nodes[k.ch[j]];
            if (c.count > 0) {
                const int off = (int)(n_soup - nd.tri_base);
                for (int t = c.begin; t < c.begin + c.count; ++t) soup[(size_t)n_soup++] = B.prim[t].id;
                nd.meta[j] = (uint8_t)(((c.count - 1) << 5) | off);
            } else {
                nd.meta[j] = (uint8_t)(0x80 | slot);
                ++slot;
                queue.push_back({k.ch[j], it.level + 1});
                out.nodes.emplace_back();
                max_depth = std::max(max_depth, it.level + 1);
            }
        }
        nd.n_internal = (uint8_t)slot;
        out.nodes[qi] = nd;
        kids.push_back(k);
    }
    // every node's frame and quantised child boxes depend on its own boxes
    // only: nodes in parallel
    parallel_for((int64_t)queue.size(), threads, 2048, [&](int64_t lo, int64_t hi) {
        for (int64_t qi = lo; qi < hi; ++qi) {
            CNode& nd = out.nodes[(size_t)qi];
            set_frame(nd, nodes[queue[(size_t)qi].bin].box);
            const Kids& k = kids[(size_t)qi];
            for (int j = 0; j < k.n; ++j) quantise_child(nd, j, nodes[k.ch[j]].box, nd);
        }
    });
    // triangle records in soup order, slots in parallel; the vertex reads
    // follow the leaves, not the input order, so they are prefetched ahead
    out.tris.resize((size_t)n_soup);
    parallel_for(n_soup, threads, 16384, [&](int64_t lo, int64_t hi) {
        constexpr int64_t kAhead = 16;
        for (int64_t t = lo; t < hi; ++t) {
            if (t + kAhead < hi) {
                const float* q = xyz + 9 * (int64_t)soup[(size_t)(t + kAhead)];
                __builtin_prefetch(q);
                __builtin_prefetch(q + 8);
            }
            const int f = soup[(size_t)t];
            const float* p = xyz + 9 * (int64_t)f;
            CTri tr;
            tr.ax = p[0]; tr.ay = p[1]; tr.az = p[2]; tr.id = f;
            tr.bx = p[3]; tr.by = p[4]; tr.bz = p[5];
            tr.cx = p[6]; tr.cy = p[7]; tr.cz = p[8];
            set_error_scales(tr);
            if (f == 0) out.slot_of_face0 = t;  // one slot holds face 0: one writer
            out.tris[(size_t)t] = tr;
        }
    });
    out.depth = max_depth;
    out.level_start.assign(1, 0);
    for (size_t qi = 1; qi < queue.size(); ++qi)
        if (queue[qi].level != queue[qi - 1].level) out.level_start.push_back((int32_t)qi);
    out.level_start.push_back((int32_t)queue.size());
    const Box& rb = nodes[root].box;
    for (int k = 0; k < 3; ++k) { out.lo[k] = rb.lo[k]; out.hi[k] = rb.hi[k]; }
    if (out.depth > kMaxDepth) {
        err = "BVH deeper than the traversal stack supports (" + std::to_string(out.depth) + " levels)";
        return false;
    }
    return true;
}

void refit_host(HostBvh& bvh) {
    // children always follow their parent in breadth-first order: sweep back
    const int64_t nn = (int64_t)bvh.nodes.size();
    std::vector<Box> nb(nn);
    for (int64_t i = nn - 1; i >= 0; --i) {
        CNode& nd = bvh.nodes[i];
        Box cbox[kWidth];
        Box all;
        for (int j = 0; j < kWidth; ++j) {
            const uint8_t m = nd.meta[j];
            if (m == kEmpty) continue;
            if (m & 0x80) cbox[j] = nb[nd.child_base + (m & 7)];
            else {
                const int off = m & 31, cnt = (m >> 5) + 1;
                for (int t = 0; t < cnt; ++t) cbox[j].grow(tri_box(bvh.tris[nd.tri_base + off + t]));
            }
            all.grow(cbox[j]);
        }
        set_frame(nd, all);
        for (int j = 0; j < kWidth; ++j)
            if (nd.meta[j] != kEmpty) quantise_child(nd, j, cbox[j], nd);
        nb[i] = all;
    }
}

// ---------------------------------------------------------------------------
// reference record format (state_dict)
// ---------------------------------------------------------------------------
int64_t reference_format_nodes(int64_t nf) {
    if (nf < 4) return 1;
    int64_t count = 1;
    std::vector<int64_t> ranges{nf};
    while (!ranges.empty()) {
        const int64_t n = ranges.back();
        ranges.pop_back();
        // halves of halves: n/2 / 2, n/2 - n/2 / 2, (n - n/2) / 2, ...
        const int64_t h0 = n / 2, h1 = n - h0;
        const int64_t parts[4] = {h0 / 2, h0 - h0 / 2, h1 / 2, h1 - h1 / 2};
        for (int64_t m : parts) {
            ++count;
            if (m > 8) ranges.push_back(m);
        }
    }
    return count;
}

// The reference's BVH4 build (src/bvh.cu:515-620), restated so that the
// records are the ones the reference's own build writes for the same mesh:
//  - a range is cut in two at its middle (std::nth_element, count / 2) along
//    the axis of largest centroid variance, the mean and variance summed in
//    float in the range's current order (first largest axis on ties); the
//    two halves are cut the same way, the second half first, giving four
//    children per inner node;
//  - children of at most 8 triangles become leaves; larger ones are pushed on
//    a stack and split when popped (last pushed first), which numbers nodes
//    in the reference's order;
//  - node boxes scan the range's vertices (a, b, c per triangle) from the
//    first vertex with std::min / std::max;
//  - escape links in pre-order: the next sibling, else the parent's escape.
// std::nth_element's permutation depends only on the comparison results, so
// sorting 16-byte (centroid, face) records gives the reference's order of
// its 48-byte triangles.  Meshes of fewer than 4 triangles (which the
// reference cannot build) give one leaf.
void export_reference_format(const float* xyz, const int64_t* ids, int64_t nf, RefFormat& out) {
    struct RNode { float lo[3], hi[3]; int32_t left, right, escape; };
    static_assert(sizeof(RNode) == 36, "reference node record is 36 bytes");
    struct Rec { float c[3]; int32_t f; };
    std::vector<Rec> rec((size_t)nf);
    for (int64_t f = 0; f < nf; ++f) {
        const float* p = xyz + 9 * f;
        // Triangle::centroid(): (a + b + c) / 3 per component, left to right
        for (int k = 0; k < 3; ++k) rec[(size_t)f].c[k] = (p[k] + p[3 + k] + p[6 + k]) / 3.0f;
        rec[(size_t)f].f = (int32_t)f;
    }
    auto box_of = [&](int64_t b, int64_t e, RNode& n) {
        const float* p0 = xyz + 9 * (int64_t)rec[(size_t)b].f;
        for (int k = 0; k < 3; ++k) n.lo[k] = n.hi[k] = p0[k];
        for (int64_t i = b; i < e; ++i) {
            const float* p = xyz + 9 * (int64_t)rec[(size_t)i].f;
            for (int v = 0; v < 3; ++v)
                for (int k = 0; k < 3; ++k) {
                    n.lo[k] = std::min(n.lo[k], p[3 * v + k]);
                    n.hi[k] = std::max(n.hi[k], p[3 * v + k]);
                }
        }
    };
    std::vector<RNode> nodes(1);
    box_of(0, nf, nodes[0]);
    nodes[0].escape = -1;
    if (nf < 4) {
        nodes[0].left = -1;
        nodes[0].right = -(int32_t)nf - 1;
    } else {
        struct Range { int32_t node; int64_t b, e; };
        std::vector<Range> stack{{0, 0, nf}};
        while (!stack.empty()) {
            const Range r = stack.back();
            stack.pop_back();
            int64_t cb[4] = {r.b}, ce[4] = {r.e};
            for (int nc = 1; nc < 4; nc *= 2) {
                for (int i = nc - 1; i >= 0; --i) {
                    const int64_t b = cb[i], e = ce[i];
                    const float cnt = (float)(e - b);
                    float mean[3] = {0.f, 0.f, 0.f}, var[3] = {0.f, 0.f, 0.f};
                    for (int64_t j = b; j < e; ++j)
                        for (int k = 0; k < 3; ++k) mean[k] = mean[k] + rec[(size_t)j].c[k];
                    for (int k = 0; k < 3; ++k) mean[k] = mean[k] / cnt;
                    for (int64_t j = b; j < e; ++j)
                        for (int k = 0; k < 3; ++k) {
                            const float d = rec[(size_t)j].c[k] - mean[k];
                            var[k] = var[k] + d * d;
                        }
                    for (int k = 0; k < 3; ++k) var[k] = var[k] / cnt;
                    int ax = 0;
                    for (int k = 1; k < 3; ++k)
                        if (var[k] > var[ax]) ax = k;
                    const int64_t m = b + (e - b) / 2;
                    std::nth_element(rec.begin() + b, rec.begin() + m, rec.begin() + e,
                                     [ax](const Rec& x, const Rec& y) { return x.c[ax] < y.c[ax]; });
                    cb[2 * i] = b;
                    ce[2 * i + 1] = e;
                    ce[2 * i] = cb[2 * i + 1] = m;
                }
            }
            const int32_t first = (int32_t)nodes.size();
            nodes[(size_t)r.node].left = first;
            for (int c = 0; c < 4; ++c) {
                RNode n;
                box_of(cb[c], ce[c], n);
                n.escape = -1;
                if (ce[c] - cb[c] <= 8) {
                    n.left = -(int32_t)cb[c] - 1;
                    n.right = -(int32_t)ce[c] - 1;
                } else {
                    n.left = n.right = 0;
                    stack.push_back({first + c, cb[c], ce[c]});
                }
                nodes.push_back(n);
            }
            nodes[(size_t)r.node].right = first + 4;
        }
    }
    std::vector<std::pair<int32_t, int32_t>> work{{0, -1}};
    while (!work.empty()) {
        const auto [ni, esc] = work.back();
        work.pop_back();
        nodes[(size_t)ni].escape = esc;
        if (nodes[(size_t)ni].left < 0) continue;  // leaf
        const int32_t f0 = nodes[(size_t)ni].left, f1 = nodes[(size_t)ni].right;
        for (int32_t c = f1 - 1; c >= f0; --c) work.push_back({c, c + 1 < f1 ? c + 1 : esc});
    }
    out.nodes.resize(nodes.size() * 9);
    std::memcpy(out.nodes.data(), nodes.data(), nodes.size() * sizeof(RNode));
    out.tris.assign((size_t)nf * 12, 0);
    for (int64_t i = 0; i < nf; ++i) {
        const int64_t f = rec[(size_t)i].f;
        std::memcpy(&out.tris[12 * (size_t)i], xyz + 9 * f, 9 * sizeof(float));
        const int64_t id = ids ? ids[f] : f;
        std::memcpy(&out.tris[12 * (size_t)i + 10], &id, sizeof(int64_t));
    }
}

}  // namespace cubvh
