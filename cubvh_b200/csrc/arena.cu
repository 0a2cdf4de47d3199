// BVH arena: many meshes concatenated into one node / triangle array so that
// all their queries run in one launch (no counterpart in the reference,
// which serves one mesh per cuBVH object and one kernel launch per call).
//
// Layout: each mesh is built on the host (in parallel), its node indices and
// triangle slots rebased by the mesh's offsets; a mesh is addressed by its
// root node.  A query layout (cubvh_arena_set_queries) fixes how many
// queries each mesh has (contiguous ranges of one points array) and its
// mode; it precomputes, once, the packet tables (up to 32 consecutive
// Morton-ordered queries of one mesh per packet), the per-mesh bucketing
// boxes, and a workspace sized for that layout.  After that,
// cubvh_arena_distance issues only stream-ordered work (no allocation, no
// host synchronisation), so a sequence of calls can be captured in a CUDA
// graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <numeric>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/cubvh_b200.h"
#include "build.h"
#include "gpubuild.h"
#include "kernels.h"
#include "scan.cuh"

namespace cubvh {
int set_error(int code, const std::string& msg);
}
using namespace cubvh;

// host arrays are RawVec (build.h): filled in parallel after sizing
struct cubvh_arena {
    int32_t M = 0;
    RawVec<CNode> nodes;
    RawVec<CTri> tris;
    std::vector<int32_t> root, slot0;
    std::vector<int64_t> face_off;   // [M + 1]
    RawVec<int32_t> gslot;           // [total faces] soup slot of (mesh, face)
    std::vector<float> box;          // [M][6]
    int64_t n_nodes = 0, n_tris = 0;
    std::mutex mu;
    int device = -1;
    CNode* d_nodes = nullptr;
    CTri* d_tris = nullptr;
    int64_t* d_face_off = nullptr;
    int32_t* d_gslot = nullptr;
    // query layout
    bool has_layout = false;
    int64_t n_queries = 0;
    void* d_layout = nullptr;
    ArenaLaunch L{};
};

namespace {

int cuda_err(cudaError_t e, const char* what) {
    return set_error(CUBVH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// fn() on up to n threads, the caller's included; fn takes its own work from
// a shared counter and must not throw.  Threads that cannot be started are
// not used, and every started thread is joined before returning.
template <class F>
void run_workers(int n, F fn) {
    std::vector<std::thread> pool;
    pool.reserve((size_t)std::max(0, n - 1));
    for (int t = 1; t < n; ++t) {
        try {
            pool.emplace_back(fn);
        } catch (const std::system_error&) {
            break;
        }
    }
    fn();
    for (auto& th : pool) th.join();
}

int arena_device(cubvh_arena* a) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(a->mu);
    if (a->device >= 0) {
        if (a->device != dev) return set_error(CUBVH_ERR_INVALID, "arena lives on another device");
        return CUBVH_OK;
    }
    const size_t nb = a->nodes.size() * sizeof(CNode), tb = a->tris.size() * sizeof(CTri);
    const size_t fb = a->face_off.size() * sizeof(int64_t), sb = a->gslot.size() * sizeof(int32_t);
    // a failed upload leaves the arena host-only (device stays -1, pointers
    // null), so a later call retries from scratch instead of leaking
    auto drop = [&](cudaError_t err, const char* what) {
        for (void** q : {(void**)&a->d_nodes, (void**)&a->d_tris, (void**)&a->d_face_off, (void**)&a->d_gslot})
            if (*q) { cudaFree(*q); *q = nullptr; }
        return cuda_err(err, what);
    };
    if ((e = cudaMalloc(&a->d_nodes, nb)) != cudaSuccess ||
        (e = cudaMalloc(&a->d_tris, tb)) != cudaSuccess ||
        (e = cudaMalloc(&a->d_face_off, fb)) != cudaSuccess ||
        (e = cudaMalloc(&a->d_gslot, sb)) != cudaSuccess)
        return drop(e, "cudaMalloc(arena)");
    if ((e = cudaMemcpy(a->d_nodes, a->nodes.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(a->d_tris, a->tris.data(), tb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(a->d_face_off, a->face_off.data(), fb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(a->d_gslot, a->gslot.data(), sb, cudaMemcpyHostToDevice)) != cudaSuccess)
        return drop(e, "arena upload");
    a->device = dev;
    // the raystab sign pass reads the stab-direction tables: set them on this
    // device even when no single-BVH query has run on it yet
    if ((e = ensure_constants(dev)) != cudaSuccess) return cuda_err(e, "constant upload");
    return CUBVH_OK;
}

}  // namespace

#define ARENA_GUARD_BEGIN try {
#define ARENA_GUARD_END                                                             \
    } catch (const std::bad_alloc&) {                                               \
        return set_error(CUBVH_ERR_NOMEM, "host allocation failed");                \
    } catch (const std::exception& ex) {                                            \
        return set_error(CUBVH_ERR_INVALID, ex.what());                             \
    }

extern "C" {

int cubvh_arena_create(int32_t n_meshes, const float* const* vertices, const int64_t* n_vertices,
                       const int64_t* const* faces, const int64_t* n_faces, const int32_t* max_leaf,
                       cubvh_arena** out) {
    ARENA_GUARD_BEGIN
    if (!out) return set_error(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (n_meshes <= 0 || !vertices || !n_vertices || !faces || !n_faces)
        return set_error(CUBVH_ERR_INVALID, "arena needs at least one mesh and non-null arrays");
    const int M = n_meshes;
    for (int m = 0; m < M; ++m) {
        if (!vertices[m] || !faces[m] || n_vertices[m] <= 0 || n_faces[m] <= 0)
            return set_error(CUBVH_ERR_INVALID, "mesh " + std::to_string(m) + " is empty or null");
        const int leaf = max_leaf ? max_leaf[m] : kMaxLeafTris;
        if (leaf < 1 || leaf > kMaxLeafTris)
            return set_error(CUBVH_ERR_INVALID, "mesh " + std::to_string(m) + ": leaf size must be in [1, 4]");
    }
    // gather and build every mesh, in parallel: one thread per mesh at a
    // time (each build single-threaded), largest meshes first from a shared
    // queue so the last builds to finish are small ones.  Errors are reported
    // as a serial pass would: a bad vertex index (lowest mesh, first face)
    // before any build error (lowest mesh); once an index error is known,
    // the remaining meshes are still checked but not built.
    std::vector<HostBvh> hb(M);
    std::vector<std::string> index_err(M), build_err(M);
    std::atomic<bool> any_index_err{false};
    const int nthr = std::max(1, std::min<int>(M, host_build_threads()));
    std::vector<int> order(M);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n_faces[a] > n_faces[b]; });
    std::atomic<int> next{0};
    run_workers(nthr, [&] {
        for (int i; (i = next.fetch_add(1)) < M;) {
            const int m = order[i];
            try {  // an exception must not leave the worker thread
                std::vector<float> xyz((size_t)n_faces[m] * 9);
                int64_t bad = -1;
                for (int64_t f = 0; f < n_faces[m] && bad < 0; ++f)
                    for (int k = 0; k < 3; ++k) {
                        const int64_t v = faces[m][3 * f + k];
                        if (v < 0 || v >= n_vertices[m]) { bad = f; break; }
                        std::memcpy(&xyz[(size_t)f * 9 + 3 * k], vertices[m] + 3 * v, 3 * sizeof(float));
                    }
                if (bad >= 0) {
                    index_err[m] = "mesh " + std::to_string(m) + " face " + std::to_string(bad) +
                                   " has a vertex index out of range";
                    any_index_err = true;
                    continue;
                }
                if (any_index_err) continue;
                const int leaf = max_leaf ? max_leaf[m] : kMaxLeafTris;
                std::string err;
                if (!build_bvh(xyz.data(), n_faces[m], hb[m], err, leaf, 1))
                    build_err[m] = "mesh " + std::to_string(m) + ": " + (err.empty() ? "build failed" : err);
            } catch (const std::bad_alloc&) {
                build_err[m] = "mesh " + std::to_string(m) + ": host allocation failed";
            } catch (const std::exception& ex) {
                build_err[m] = "mesh " + std::to_string(m) + ": " + ex.what();
            }
        }
    });
    for (int m = 0; m < M; ++m)
        if (!index_err[m].empty()) return set_error(CUBVH_ERR_INVALID, index_err[m]);
    for (int m = 0; m < M; ++m)
        if (!build_err[m].empty()) return set_error(CUBVH_ERR_INVALID, build_err[m]);
    std::unique_ptr<cubvh_arena> a(new cubvh_arena());  // released to the caller on success
    a->M = M;
    a->root.resize(M); a->slot0.resize(M); a->face_off.assign(M + 1, 0); a->box.resize((size_t)M * 6);
    size_t nn = 0, nt = 0;
    for (int m = 0; m < M; ++m) { nn += hb[m].nodes.size(); nt += hb[m].tris.size(); }
    if (nn >= (size_t)INT32_MAX || nt >= (size_t)(1u << 28))
        return set_error(CUBVH_ERR_INVALID, "arena too large (2^31 nodes / 2^28 triangles)");
    // offsets of every mesh in the concatenated arrays, then each mesh's
    // rebased nodes, triangles and face -> slot map written in parallel into
    // its own ranges (every face of a mesh is in its soup, so every gslot
    // entry is written)
    std::vector<size_t> node_off(M + 1, 0), tri_off(M + 1, 0);
    for (int m = 0; m < M; ++m) {
        node_off[m + 1] = node_off[m] + hb[m].nodes.size();
        tri_off[m + 1] = tri_off[m] + hb[m].tris.size();
        a->face_off[m + 1] = a->face_off[m] + n_faces[m];
        a->root[m] = (int32_t)node_off[m];
        a->slot0[m] = (int32_t)tri_off[m] + (int32_t)hb[m].slot_of_face0;
        for (int k = 0; k < 3; ++k) { a->box[6 * m + k] = hb[m].lo[k]; a->box[6 * m + 3 + k] = hb[m].hi[k]; }
    }
    a->nodes.resize(nn); a->tris.resize(nt); a->gslot.resize(nt);
    next = 0;
    run_workers(nthr, [&] {
        for (int i; (i = next.fetch_add(1)) < M;) {
            const int m = order[i];
            const int32_t no = (int32_t)node_off[m], to = (int32_t)tri_off[m];
            CNode* dn = a->nodes.data() + node_off[m];
            for (const CNode& src : hb[m].nodes) {
                CNode nd = src;
                nd.child_base += no; nd.tri_base += to;
                *dn++ = nd;
            }
            std::memcpy(a->tris.data() + tri_off[m], hb[m].tris.data(), hb[m].tris.size() * sizeof(CTri));
            int32_t* gs = a->gslot.data() + a->face_off[m];
            for (size_t s = 0; s < hb[m].tris.size(); ++s) gs[hb[m].tris[s].id] = to + (int32_t)s;
            HostBvh().nodes.swap(hb[m].nodes);  // release the per-mesh copy early
            HostBvh().tris.swap(hb[m].tris);
        }
    });
    a->n_nodes = (int64_t)a->nodes.size();
    a->n_tris = (int64_t)a->tris.size();
    *out = a.release();
    return CUBVH_OK;
    ARENA_GUARD_END
}

int cubvh_arena_create_device(int32_t n_meshes, const float* const* vertices, const int64_t* n_vertices,
                              const int64_t* const* faces, const int64_t* n_faces, const int32_t* max_leaf,
                              void* stream, cubvh_arena** out) {
    ARENA_GUARD_BEGIN
    if (!out) return set_error(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (n_meshes <= 0 || !vertices || !n_vertices || !faces || !n_faces)
        return set_error(CUBVH_ERR_INVALID, "arena needs at least one mesh and non-null arrays");
    const int M = n_meshes;
    std::vector<int64_t> voff(M + 1, 0), foff(M + 1, 0);
    std::vector<int32_t> leaf(M);
    for (int m = 0; m < M; ++m) {
        if (!vertices[m] || !faces[m] || n_vertices[m] <= 0 || n_faces[m] <= 0)
            return set_error(CUBVH_ERR_INVALID, "mesh " + std::to_string(m) + " is empty or null");
        leaf[m] = max_leaf ? max_leaf[m] : kMaxLeafTris;
        voff[m + 1] = voff[m] + n_vertices[m];
        foff[m + 1] = foff[m] + n_faces[m];
    }
    if (foff[M] >= (int64_t)(1 << 28)) return set_error(CUBVH_ERR_INVALID, "arena too large (2^28 triangles)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    // one upload of all vertices and faces
    float* dv = nullptr;
    int64_t* df = nullptr;
    if ((e = cudaMalloc(&dv, sizeof(float) * 3 * voff[M])) != cudaSuccess) return cuda_err(e, "cudaMalloc(vertices)");
    if ((e = cudaMalloc(&df, sizeof(int64_t) * 3 * foff[M])) != cudaSuccess) { cudaFree(dv); return cuda_err(e, "cudaMalloc(faces)"); }
    for (int m = 0; m < M && e == cudaSuccess; ++m) {
        e = cudaMemcpyAsync(dv + 3 * voff[m], vertices[m], sizeof(float) * 3 * n_vertices[m], cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(df + 3 * foff[m], faces[m], sizeof(int64_t) * 3 * n_faces[m], cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) { cudaFree(dv); cudaFree(df); return cuda_err(e, "arena mesh upload"); }
    DeviceBuild db;
    std::string err;
    const int rc = build_meshes_device(dv, df, voff, foff, leaf, s, db, err, true);
    cudaFree(dv);
    cudaFree(df);
    if (rc != 0) return set_error(rc == 1 ? CUBVH_ERR_INVALID : CUBVH_ERR_CUDA, err);
    auto* a = new cubvh_arena();
    a->M = M;
    a->root.resize(M);
    for (int m = 0; m < M; ++m) a->root[m] = m;  // level 0 of the build holds the roots
    a->slot0 = db.slot0;
    a->face_off = foff;
    a->box = db.mesh_box;
    a->n_nodes = db.n_nodes;
    a->n_tris = foff[M];
    a->d_nodes = db.nodes;
    a->d_tris = db.tris;
    a->d_gslot = db.gslot;
    if ((e = cudaMalloc(&a->d_face_off, sizeof(int64_t) * (M + 1))) != cudaSuccess ||
        (e = cudaMemcpy(a->d_face_off, foff.data(), sizeof(int64_t) * (M + 1), cudaMemcpyHostToDevice)) != cudaSuccess) {
        a->device = dev;
        cubvh_arena_destroy(a);
        return cuda_err(e, "arena face offsets");
    }
    a->device = dev;
    if ((e = ensure_constants(dev)) != cudaSuccess) {
        cubvh_arena_destroy(a);
        return cuda_err(e, "constant upload");
    }
    *out = a;
    return CUBVH_OK;
    ARENA_GUARD_END
}

int cubvh_arena_destroy(cubvh_arena* a) {
    if (!a) return CUBVH_OK;
    if (a->device >= 0) {
        int cur = 0;
        const bool have = cudaGetDevice(&cur) == cudaSuccess;
        if (cudaSetDevice(a->device) == cudaSuccess) {
            cudaFree(a->d_nodes); cudaFree(a->d_tris); cudaFree(a->d_face_off); cudaFree(a->d_gslot);
            if (a->d_layout) cudaFree(a->d_layout);
        }
        if (have) cudaSetDevice(cur);
    }
    delete a;
    return CUBVH_OK;
}

int cubvh_arena_info(const cubvh_arena* a, int32_t* n_meshes, int64_t* n_faces, int64_t* n_nodes) {
    if (!a) return set_error(CUBVH_ERR_INVALID, "arena is null");
    if (n_meshes) *n_meshes = a->M;
    if (n_faces) *n_faces = a->n_tris;
    if (n_nodes) *n_nodes = a->n_nodes;
    return CUBVH_OK;
}

int cubvh_arena_set_queries(cubvh_arena* a, const int64_t* query_offsets, const uint32_t* modes) {
    ARENA_GUARD_BEGIN
    if (!a || !query_offsets || !modes) return set_error(CUBVH_ERR_INVALID, "null argument");
    const int M = a->M;
    if (query_offsets[0] != 0) return set_error(CUBVH_ERR_INVALID, "query_offsets[0] must be 0");
    for (int m = 0; m < M; ++m) {
        if (query_offsets[m + 1] < query_offsets[m]) return set_error(CUBVH_ERR_INVALID, "query_offsets must not decrease");
        if (modes[m] > 2) return set_error(CUBVH_ERR_INVALID, "mode must be 0 (unsigned), 1 (watertight) or 2 (raystab)");
    }
    const int64_t Q = query_offsets[M];
    if (Q >= (int64_t)UINT32_MAX) return set_error(CUBVH_ERR_INVALID, "2^32 or more queries in one arena layout");
    int rc = arena_device(a);
    if (rc != CUBVH_OK) return rc;
    // host tables
    std::vector<MeshDesc> meshes(M);
    std::vector<ArenaSortDesc> sort(M);
    std::vector<PacketDesc> all, wt, rs;
    int64_t cells = 0;
    for (int m = 0; m < M; ++m) {
        const int64_t q0 = query_offsets[m], nq = query_offsets[m + 1] - q0;
        meshes[m] = MeshDesc{a->root[m], a->slot0[m], q0};
        ArenaSortDesc& s = sort[m];
        for (int k = 0; k < 3; ++k) {  // the mesh box widened by a quarter of its extent
            const float lo = a->box[6 * m + k], hi = a->box[6 * m + 3 + k], pad = 0.25f * (hi - lo) + 1e-6f;
            s.lo[k] = lo - pad; s.hi[k] = hi + pad;
        }
        s.bits = nq > 0 ? std::min(cell_bits_for(nq), 6) : 0;
        s.cell_off = cells;
        cells += (int64_t)1 << (3 * s.bits);
        for (int64_t p = 0; p < nq; p += 32) {
            const PacketDesc d{q0 + p, (int32_t)std::min<int64_t>(32, nq - p), m};
            all.push_back(d);
            if (modes[m] == 1) wt.push_back(d);
            if (modes[m] == 2) rs.push_back(d);
        }
    }
    // one device allocation for the layout and its workspace
    size_t off = 0;
    const size_t o_qoff = off; off += al(sizeof(int64_t) * (M + 1));
    const size_t o_mesh = off; off += al(sizeof(MeshDesc) * M);
    const size_t o_sort = off; off += al(sizeof(ArenaSortDesc) * M);
    const size_t o_all = off; off += al(sizeof(PacketDesc) * std::max<size_t>(all.size(), 1));
    const size_t o_wt = off; off += al(sizeof(PacketDesc) * std::max<size_t>(wt.size(), 1));
    const size_t o_rs = off; off += al(sizeof(PacketDesc) * std::max<size_t>(rs.size(), 1));
    const size_t o_ctr = off; off += 256;
    const size_t o_order = off; off += al(sizeof(uint32_t) * std::max<int64_t>(Q, 1));
    const size_t o_hist = off; off += al(sizeof(uint32_t) * (cells + 1));
    const size_t o_bsum = off; off += al(sizeof(uint32_t) * (scan::num_chunks(cells) + 1));
    const size_t o_slots = off; off += al(sizeof(int32_t) * std::max<int64_t>(Q, 1));
    const int64_t hcap = heavy_cap_for(std::max<int64_t>(Q, 1));
    const size_t o_heavy = off; off += al(sizeof(uint2) * hcap);
    const int64_t n_rs_q = (int64_t)rs.size() * 32;                // raystab candidates (second pass)
    const size_t o_cand = off; off += al(sizeof(uint4) * std::max<int64_t>(n_rs_q, 1));
    std::lock_guard<std::mutex> lk(a->mu);
    if (a->d_layout) { cudaFree(a->d_layout); a->d_layout = nullptr; a->has_layout = false; }
    cudaError_t e = cudaMalloc(&a->d_layout, off);
    if (e != cudaSuccess) return cuda_err(e, "cudaMalloc(arena layout)");
    char* base = static_cast<char*>(a->d_layout);
    auto up = [&](size_t o, const void* src, size_t bytes) {
        return bytes ? cudaMemcpy(base + o, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    if ((e = up(o_qoff, query_offsets, sizeof(int64_t) * (M + 1))) != cudaSuccess ||
        (e = up(o_mesh, meshes.data(), sizeof(MeshDesc) * M)) != cudaSuccess ||
        (e = up(o_sort, sort.data(), sizeof(ArenaSortDesc) * M)) != cudaSuccess ||
        (e = up(o_all, all.data(), sizeof(PacketDesc) * all.size())) != cudaSuccess ||
        (e = up(o_wt, wt.data(), sizeof(PacketDesc) * wt.size())) != cudaSuccess ||
        (e = up(o_rs, rs.data(), sizeof(PacketDesc) * rs.size())) != cudaSuccess)
        return cuda_err(e, "arena layout upload");
    ArenaLaunch& L = a->L;
    L.nodes = a->d_nodes; L.tris = a->d_tris;
    L.n_meshes = M; L.n_queries = Q;
    L.qoff = reinterpret_cast<const int64_t*>(base + o_qoff);
    L.meshes = reinterpret_cast<const MeshDesc*>(base + o_mesh);
    L.sort = reinterpret_cast<const ArenaSortDesc*>(base + o_sort);
    L.n_cells = cells;
    L.packets = reinterpret_cast<const PacketDesc*>(base + o_all); L.n_packets = (int64_t)all.size();
    L.wt_packets = reinterpret_cast<const PacketDesc*>(base + o_wt); L.n_wt_packets = (int64_t)wt.size();
    L.rs_packets = reinterpret_cast<const PacketDesc*>(base + o_rs); L.n_rs_packets = (int64_t)rs.size();
    L.counters = reinterpret_cast<unsigned long long*>(base + o_ctr);
    L.order = reinterpret_cast<uint32_t*>(base + o_order);
    L.hist = reinterpret_cast<uint32_t*>(base + o_hist);
    L.bsum = reinterpret_cast<uint32_t*>(base + o_bsum);
    L.slots = reinterpret_cast<int32_t*>(base + o_slots);
    L.heavy = reinterpret_cast<uint2*>(base + o_heavy);
    L.heavy_cap = hcap;
    L.rs_cand = reinterpret_cast<uint4*>(base + o_cand);
    a->n_queries = Q;
    a->has_layout = true;
    return CUBVH_OK;
    ARENA_GUARD_END
}

int cubvh_arena_distance(cubvh_arena* a, const float* points, float* distances, int64_t* face_id, float* uvw,
                         void* stream) {
    ARENA_GUARD_BEGIN
    if (!a) return set_error(CUBVH_ERR_INVALID, "arena is null");
    if (!a->has_layout) return set_error(CUBVH_ERR_INVALID, "call cubvh_arena_set_queries first");
    if (a->n_queries == 0) return CUBVH_OK;
    if (!points || !distances || !face_id) return set_error(CUBVH_ERR_INVALID, "points/distances/face_id is null");
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != a->device) return set_error(CUBVH_ERR_INVALID, "arena lives on another device");
    const cudaError_t e = launch_arena_distance(a->L, points, distances, face_id, uvw, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_err(e, "arena launch");
    return CUBVH_OK;
    ARENA_GUARD_END
}

int cubvh_arena_backward(cubvh_arena* a, const float* points, const int64_t* face_id, const float* grad_distances,
                         const float* distances, float* grad_points, void* stream) {
    ARENA_GUARD_BEGIN
    if (!a) return set_error(CUBVH_ERR_INVALID, "arena is null");
    if (!a->has_layout) return set_error(CUBVH_ERR_INVALID, "call cubvh_arena_set_queries first");
    if (a->n_queries == 0) return CUBVH_OK;
    if (!points || !face_id || !grad_distances || !distances || !grad_points)
        return set_error(CUBVH_ERR_INVALID, "null argument");
    const cudaError_t e = launch_arena_backward(a->n_queries, points, face_id, grad_distances, distances, a->L.qoff,
                                                a->M, a->d_face_off, a->d_gslot, a->d_tris, grad_points,
                                                (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_err(e, "arena backward launch");
    return CUBVH_OK;
    ARENA_GUARD_END
}

}  // extern "C"
