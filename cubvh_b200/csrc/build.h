// Host-side BVH construction and the reference's state_dict format.
#pragma once
#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <system_error>
#include <thread>
#include <utility>
#include <vector>

#include "layout.h"

namespace cubvh {

// std::allocator whose resize leaves trivially constructible elements
// uninitialised, so the threads that fill a large array are the first to
// touch its pages (first touch of fresh memory costs more than the writes)
template <class T>
struct NoInitAlloc : std::allocator<T> {
    NoInitAlloc() = default;
    template <class U> NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U> struct rebind { using other = NoInitAlloc<U>; };
    template <class U> void construct(U* p) noexcept { ::new ((void*)p) U; }
    template <class U, class... A> void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
};
template <class T> using RawVec = std::vector<T, NoInitAlloc<T>>;

// fn(lo, hi) over [0, n) split into contiguous ranges of at least `grain`
// items on up to `threads` threads (the caller's thread takes the first
// range; a range whose thread cannot be started runs on the caller's thread).
// fn must not throw.
template <class F>
void parallel_for(int64_t n, int threads, int64_t grain, F fn) {
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(threads, (n + grain - 1) / grain));
    if (parts <= 1) { fn(0, n); return; }
    std::vector<std::thread> pool;
    std::vector<int64_t> inline_parts;
    // both vectors sized up front: growing them inside the loop could throw
    // with threads already running, which would terminate the process
    pool.reserve((size_t)parts - 1);
    inline_parts.reserve((size_t)parts - 1);
    for (int64_t i = 1; i < parts; ++i) {
        const int64_t lo = n * i / parts, hi = n * (i + 1) / parts;
        try {
            pool.emplace_back([=, &fn] { fn(lo, hi); });
        } catch (const std::system_error&) {
            inline_parts.push_back(i);
        }
    }
    fn(0, n / parts);
    for (int64_t i : inline_parts) fn(n * i / parts, n * (i + 1) / parts);
    for (auto& t : pool) t.join();
}

struct HostBvh {
    RawVec<CNode> nodes;           // node 0 is the root
    RawVec<CTri> tris;             // leaf-ordered soup
    int depth = 0;                 // internal levels (root = 1)
    // nodes are stored breadth first: level l (root = 0) is the index range
    // [level_start[l], level_start[l + 1])
    std::vector<int32_t> level_start;
    int64_t slot_of_face0 = 0;     // soup slot of original face 0
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // scene bounds
    // face -> vertex indices, for refit / vertex gradients (empty when the
    // BVH was created from triangle records)
    RawVec<int32_t> faces;         // [F, 3], original face order
    int64_t n_vertices = 0;
};

// Host threads a build may use: CUBVH_B200_BUILD_THREADS when set to a
// positive integer (read once), otherwise every hardware thread.
int host_build_threads();

// Builds the wide BVH over triangles (a, b, c per face, original face index
// = position).  tri_xyz: [F, 9] floats.  Returns false and sets err on bad input.
// threads: host threads the build may use (0 = host_build_threads()); the
// tree is the same for any count.
bool build_bvh(const float* tri_xyz, int64_t n_faces, HostBvh& out, std::string& err,
               int max_leaf = kMaxLeafTris, int threads = 0);

// Recomputes the quantised boxes of every node from the current triangle
// soup, keeping the topology (used after the soup's vertices moved).
void refit_host(HostBvh& bvh);

// The reference's on-disk format (include/gpu/bvh.cuh:84-109,
// src/api_gpu.cu:110-121): the BVH4 the reference's own median-split build
// (src/bvh.cu:515-620) makes, record for record,
// as int32 [n_nodes, 9] records (box min, box max, left, right, escape) and
// the triangle soup in that BVH's order as int32 [F, 12] records (a, b, c,
// 4 pad bytes, int64 original index).
struct RefFormat {
    std::vector<int32_t> nodes;    // n_nodes * 9
    std::vector<int32_t> tris;     // n_faces * 12
};
// ids: face id of each triangle of tri_xyz (NULL = its position).
void export_reference_format(const float* tri_xyz, const int64_t* ids, int64_t n_faces, RefFormat& out);
// Node records export_reference_format writes for n_faces triangles: the
// tree's shape depends on the count only (each range halved, then each half
// halved, down to leaves of at most 8).
int64_t reference_format_nodes(int64_t n_faces);

}  // namespace cubvh
