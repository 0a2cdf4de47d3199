// C ABI (include/cubvh_b200.h): BVH handles, lazy per-device upload, query
// and floodfill entry points.  Every entry point catches C++ exceptions and
// turns them into a status code plus a per-thread message.
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <exception>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cubvh_b200.h"
#include "build.h"
#include "gpubuild.h"
#include "launches.h"
#include "kernels.h"

using namespace cubvh;

// Streams and events of the host-buffer queries: one set per caller stream
// (up to kMaxPipes per device copy, created on first use), so that calls
// issued on different streams overlap (one call's copies run beside another
// call's kernels) while calls on one stream stay in order.
// Device staging sets (chunks in flight) of a host-buffer query pipe.
constexpr int kStageSets = 4;
struct HostPipe {
    cudaStream_t caller = nullptr;
    cudaStream_t cin = nullptr, cout = nullptr, comp_s[kStageSets] = {};
    cudaEvent_t start = nullptr, in[kStageSets] = {}, comp[kStageSets] = {}, out[kStageSets] = {};
    char* stage = nullptr;         // staging sets and workspaces, kept between calls
    size_t stage_bytes = 0;
    bool ready = false;
};

struct DevCopy {
    int device = -1;
    std::deque<HostPipe> pipes;
    CNode* nodes = nullptr;
    CTri* tris = nullptr;
    int32_t* face_vidx = nullptr;  // [F, 3] (meshes only), uploaded on first use
    int32_t* face_slot = nullptr;  // [F] soup slot of each face id, -1 if none
    float* node_box = nullptr;     // [n_nodes, 6] refit scratch
    int32_t* near_cnt = nullptr;   // watertight candidate lists (launch_near_lists)
    int32_t* near_lst = nullptr;
    double* near_nrm = nullptr;
    int* near_flag = nullptr;      // device int: some list overflowed
    bool near_ovf = false;
    bool near_valid = false;       // false until built, and again after a refit
    bool near_off = false;         // lists not kept (too large or allocation failed)
};

struct cubvh_bvh {
    HostBvh host;
    RawVec<float> xyz;            // [F, 9] a, b, c of each face, face order
    RawVec<int64_t> ids;          // face id of each face (position for meshes)
    // state_dict records this BVH was loaded from (cubvh_bvh_create_from_state_dict),
    // returned unchanged by cubvh_bvh_state_dict as the reference does
    std::vector<int32_t> sd_nodes, sd_tris;
    std::mutex mu;
    std::deque<DevCopy> dev;      // stable addresses across push_back
};

namespace {
std::mutex g_const_mu;
std::vector<int> g_const_ready;  // devices whose __constant__ tables are set
}  // namespace

cudaError_t cubvh::ensure_constants(int device) {
    std::lock_guard<std::mutex> lk(g_const_mu);
    for (int d : g_const_ready) if (d == device) return cudaSuccess;
    const cudaError_t e = upload_constants();
    if (e == cudaSuccess) g_const_ready.push_back(device);
    return e;
}

// The library's stream-ordered pool on the current device.  Calls take their
// scratch (query, ray, backward and floodfill workspaces, sparse marching
// cubes temporaries) from it with cudaMallocFromPoolAsync and return it with
// cudaFreeAsync.  The default pool's release threshold is 0: every stream or
// device wait hands freed memory back to the driver and the next call maps
// it again (1.5-2 ms per call, more than a small query's kernels).  This pool
// keeps up to kPoolKeepBytes between calls and returns what is above that at
// each wait.
cudaError_t cubvh::library_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;  // by device ordinal, created on first use
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= dev) pools.resize((size_t)dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return e;
        uint64_t keep = kPoolKeepBytes;
        if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        pools[dev] = p;
    }
    *out = pools[dev];
    return cudaSuccess;
}

namespace {

thread_local std::string g_err;

// Scratch of `bytes` on stream s: from the library pool, or, while s is
// being captured into a CUDA graph, with cudaMallocAsync (the graph then owns
// the allocation as a memory node).
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
    if (bytes == 0) bytes = 16;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return e;
    if (cap != cudaStreamCaptureStatusNone) return cudaMallocAsync(p, bytes, s);
    cudaMemPool_t pool = nullptr;
    if ((e = library_pool(&pool)) != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* what) {
    return fail(CUBVH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
int host_threads() { return host_build_threads(); }


// Device copy of the BVH on the current device (uploaded on first use).
int device_copy(cubvh_bvh* h, DevCopy** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(h->mu);
    for (auto& d : h->dev)
        if (d.device == device) { *out = &d; return CUBVH_OK; }
    if ((e = ensure_constants(device)) != cudaSuccess) return cuda_fail(e, "constant upload");
    DevCopy d;
    d.device = device;
    const size_t nb = h->host.nodes.size() * sizeof(CNode), tb = h->host.tris.size() * sizeof(CTri);
    if ((e = cudaMalloc(&d.nodes, nb)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(nodes)");
    if ((e = cudaMalloc(&d.tris, tb)) != cudaSuccess) { cudaFree(d.nodes); return cuda_fail(e, "cudaMalloc(triangles)"); }
    if ((e = cudaMemcpy(d.nodes, h->host.nodes.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.tris, h->host.tris.data(), tb, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(d.nodes); cudaFree(d.tris);
        return cuda_fail(e, "BVH upload");
    }
    h->dev.push_back(d);
    *out = &h->dev.back();
    return CUBVH_OK;
}

// face -> vertex indices and face -> soup slot on the device (once).
int grad_buffers(cubvh_bvh* h, DevCopy* d, bool need_vidx) {
    std::lock_guard<std::mutex> lk(h->mu);
    cudaError_t e;
    const size_t nf = h->ids.size();
    if (!d->face_slot) {
        std::vector<int32_t> slot(nf, -1);
        for (size_t s = 0; s < h->host.tris.size(); ++s) {
            const int32_t id = h->host.tris[s].id;
            if (id >= 0 && (size_t)id < nf) slot[(size_t)id] = (int32_t)s;
        }
        if ((e = cudaMalloc(&d->face_slot, nf * sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(face_slot)");
        if ((e = cudaMemcpy(d->face_slot, slot.data(), nf * sizeof(int32_t), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "upload(face_slot)");
    }
    if (need_vidx && !d->face_vidx) {
        if (h->host.faces.empty()) return fail(CUBVH_ERR_INVALID, "this BVH was created from triangle records: it has no vertex indices");
        if ((e = cudaMalloc(&d->face_vidx, nf * 3 * sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(face_vidx)");
        if ((e = cudaMemcpy(d->face_vidx, h->host.faces.data(), nf * 3 * sizeof(int32_t), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "upload(face_vidx)");
    }
    return CUBVH_OK;
}

// Watertight candidate lists of this device copy: built on first use on the
// caller's stream and waited for, so that calls on any stream see finished
// lists; rebuilt after a refit.  Not built while the stream is being captured
// into a graph, nor for BVHs whose lists would exceed 1 GiB: the sign pass
// then walks the tree, with the same results.
int near_lists(cubvh_bvh* h, DevCopy* d, cudaStream_t s, NearLists* out) {
    *out = NearLists{};
    std::lock_guard<std::mutex> lk(h->mu);
    if (d->near_off) return CUBVH_OK;
    const int64_t nt = (int64_t)h->host.tris.size();
    if (!d->near_valid) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t e = cudaStreamIsCapturing(s, &cs);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone) return CUBVH_OK;
        if (!d->near_cnt) {
            const size_t lb = (size_t)nt * kNear * sizeof(int32_t);
            if (lb > ((size_t)1 << 30) || cudaMalloc(&d->near_cnt, (size_t)nt * sizeof(int32_t)) != cudaSuccess) {
                cudaGetLastError();
                d->near_cnt = nullptr;
                d->near_off = true;
                return CUBVH_OK;
            }
            if (cudaMalloc(&d->near_lst, lb) != cudaSuccess ||
                cudaMalloc(&d->near_nrm, (size_t)nt * 3 * sizeof(double)) != cudaSuccess ||
                cudaMalloc(&d->near_flag, sizeof(int)) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(d->near_cnt);
                if (d->near_lst) cudaFree(d->near_lst);
                if (d->near_nrm) cudaFree(d->near_nrm);
                d->near_cnt = nullptr;
                d->near_lst = nullptr;
                d->near_nrm = nullptr;
                d->near_off = true;
                return CUBVH_OK;
            }
        }
        int flag = 0;
        if ((e = launch_near_lists(nt, d->nodes, d->tris, d->near_cnt, d->near_lst, d->near_nrm, d->near_flag, s)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(&flag, d->near_flag, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "watertight candidate lists");
        d->near_ovf = flag != 0;
        d->near_valid = true;
    }
    out->cnt = d->near_cnt; out->lst = d->near_lst; out->nrm = d->near_nrm; out->ovf = d->near_ovf;
    return CUBVH_OK;
}

int finish_build(cubvh_bvh* h) {
    std::string err;
    if (!build_bvh(h->xyz.data(), (int64_t)h->ids.size(), h->host, err, kMaxLeafTris, host_threads()))
        return fail(CUBVH_ERR_INVALID, err);
    // triangle ids: stored face ids (int32 in the node layout)
    std::atomic<bool> fits{true};
    parallel_for((int64_t)h->host.tris.size(), host_threads(), 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t s = lo; s < hi; ++s) {
            CTri& t = h->host.tris[(size_t)s];
            const int64_t id = h->ids[(size_t)t.id];
            if (id < INT32_MIN || id > INT32_MAX) { fits = false; return; }
            t.id = (int32_t)id;
        }
    });
    if (!fits) return fail(CUBVH_ERR_INVALID, "face id does not fit in int32");
    return CUBVH_OK;
}

}  // namespace

namespace cubvh {
// Status + message of a failed call for cubvh_last_error() (other files).
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace cubvh

#define CUBVH_GUARD_BEGIN try {
#define CUBVH_GUARD_END                                                          \
    } catch (const std::bad_alloc&) {                                            \
        return fail(CUBVH_ERR_NOMEM, "host allocation failed");                  \
    } catch (const std::exception& ex) {                                         \
        return fail(CUBVH_ERR_INVALID, ex.what());                               \
    } catch (...) {                                                              \
        return fail(CUBVH_ERR_INVALID, "unknown error");                         \
    }

namespace cubvh {
std::atomic<uint64_t> g_kernel_launches{0};
}  // namespace cubvh

extern "C" {

const char* cubvh_version(void) { return "cubvh_b200 0.1.0 (sm_100a)"; }

uint64_t cubvh_kernel_launches(void) { return cubvh::g_kernel_launches.load(std::memory_order_relaxed); }

const char* cubvh_last_error(void) { return g_err.c_str(); }

int cubvh_bvh_create(const float* vertices, int64_t n_vertices, const int64_t* faces, int64_t n_faces,
                     cubvh_bvh** out) {
    CUBVH_GUARD_BEGIN
    if (!out) return fail(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!vertices || !faces) return fail(CUBVH_ERR_INVALID, "vertices/faces is null");
    if (n_vertices <= 0 || n_faces <= 0) return fail(CUBVH_ERR_INVALID, "empty mesh");
    std::unique_ptr<cubvh_bvh> h(new cubvh_bvh());
    h->xyz.resize((size_t)n_faces * 9);  // uninitialised: filled in parallel
    h->ids.resize((size_t)n_faces);
    h->host.faces.resize((size_t)n_faces * 3);
    h->host.n_vertices = n_vertices;
    // faces in parallel; a range stops at its first bad face, so the lowest
    // of those is the first bad face of the mesh, the one reported
    std::atomic<int64_t> first_bad{INT64_MAX};
    parallel_for(n_faces, host_threads(), 65536, [&](int64_t lo, int64_t hi) {
        for (int64_t f = lo; f < hi; ++f) {
            for (int k = 0; k < 3; ++k) {
                const int64_t v = faces[3 * f + k];
                if (v < 0 || v >= n_vertices) {
                    int64_t cur = first_bad.load();
                    while (f < cur && !first_bad.compare_exchange_weak(cur, f)) {}
                    return;
                }
                std::memcpy(&h->xyz[(size_t)f * 9 + 3 * k], vertices + 3 * v, 3 * sizeof(float));
                h->host.faces[(size_t)f * 3 + k] = (int32_t)v;
            }
            h->ids[(size_t)f] = f;
        }
    });
    if (first_bad.load() != INT64_MAX) {
        const int64_t f = first_bad.load();
        int64_t v = 0;
        for (int k = 0; k < 3; ++k) {
            v = faces[3 * f + k];
            if (v < 0 || v >= n_vertices) break;
        }
        return fail(CUBVH_ERR_INVALID, "face " + std::to_string(f) + " has vertex index " + std::to_string(v) +
                                           " outside [0, " + std::to_string(n_vertices) + ")");
    }
    const int rc = finish_build(h.get());
    if (rc != CUBVH_OK) return rc;
    *out = h.release();
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_create_device(const float* vertices, int64_t n_vertices, const int64_t* faces, int64_t n_faces,
                            int32_t max_leaf, void* stream, cubvh_bvh** out) {
    CUBVH_GUARD_BEGIN
    if (!out) return fail(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!vertices || !faces) return fail(CUBVH_ERR_INVALID, "vertices/faces is null");
    if (n_vertices <= 0 || n_faces <= 0) return fail(CUBVH_ERR_INVALID, "empty mesh");
    if (n_vertices > INT32_MAX) return fail(CUBVH_ERR_INVALID, "more than 2^31-1 vertices");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = ensure_constants(device)) != cudaSuccess) return cuda_fail(e, "constant upload");
    cudaStream_t s = (cudaStream_t)stream;
    DeviceBuild db;
    std::string err;
    const int rc = build_bvh_device(vertices, n_vertices, faces, n_faces, max_leaf ? max_leaf : kMaxLeafTris, s, db, err);
    if (rc != 0) return fail(rc == 1 ? CUBVH_ERR_INVALID : CUBVH_ERR_CUDA, err);
    auto* h = new cubvh_bvh();
    HostBvh& hb = h->host;
    hb.nodes.resize((size_t)db.n_nodes);
    hb.tris.resize((size_t)n_faces);
    std::vector<int64_t> f64((size_t)n_faces * 3);
    if ((e = cudaMemcpyAsync(hb.nodes.data(), db.nodes, sizeof(CNode) * db.n_nodes, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hb.tris.data(), db.tris, sizeof(CTri) * n_faces, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(f64.data(), faces, sizeof(int64_t) * 3 * n_faces, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        cudaFree(db.nodes); cudaFree(db.tris); delete h;
        return cuda_fail(e, "GPU build download");
    }
    hb.depth = db.depth;
    hb.level_start = db.level_start;
    hb.slot_of_face0 = db.slot_of_face0;
    for (int k = 0; k < 3; ++k) { hb.lo[k] = db.lo[k]; hb.hi[k] = db.hi[k]; }
    hb.n_vertices = n_vertices;
    hb.faces.resize((size_t)n_faces * 3);
    for (size_t i = 0; i < f64.size(); ++i) hb.faces[i] = (int32_t)f64[i];
    // face-order coordinates and ids (state_dict export, other devices)
    h->xyz.resize((size_t)n_faces * 9);
    h->ids.resize((size_t)n_faces);
    for (const CTri& t : hb.tris) {
        float* p = &h->xyz[(size_t)t.id * 9];
        p[0] = t.ax; p[1] = t.ay; p[2] = t.az; p[3] = t.bx; p[4] = t.by; p[5] = t.bz;
        p[6] = t.cx; p[7] = t.cy; p[8] = t.cz;
        h->ids[(size_t)t.id] = t.id;
    }
    DevCopy d;
    d.device = device;
    d.nodes = db.nodes;
    d.tris = db.tris;
    h->dev.push_back(d);
    *out = h;
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_create_from_records(const int32_t* rec, int64_t n_faces, cubvh_bvh** out) {
    CUBVH_GUARD_BEGIN
    if (!out) return fail(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!rec) return fail(CUBVH_ERR_INVALID, "triangle records are null");
    if (n_faces <= 0) return fail(CUBVH_ERR_INVALID, "no triangle records");
    auto* h = new cubvh_bvh();
    h->xyz.resize((size_t)n_faces * 9);
    h->ids.resize((size_t)n_faces);
    for (int64_t f = 0; f < n_faces; ++f) {
        std::memcpy(&h->xyz[(size_t)f * 9], rec + 12 * f, 9 * sizeof(float));
        std::memcpy(&h->ids[(size_t)f], rec + 12 * f + 10, sizeof(int64_t));
    }
    const int rc = finish_build(h);
    if (rc != CUBVH_OK) { delete h; return rc; }
    *out = h;
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_create_from_state_dict(const int32_t* node_records, int64_t n_node_records, const int32_t* rec,
                                     int64_t n_faces, cubvh_bvh** out) {
    CUBVH_GUARD_BEGIN
    if (!out) return fail(CUBVH_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!node_records || n_node_records <= 0) return fail(CUBVH_ERR_INVALID, "no node records");
    cubvh_bvh* h = nullptr;
    const int rc = cubvh_bvh_create_from_records(rec, n_faces, &h);
    if (rc != CUBVH_OK) return rc;
    h->sd_nodes.assign(node_records, node_records + 9 * n_node_records);
    h->sd_tris.assign(rec, rec + 12 * n_faces);
    *out = h;
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_destroy(cubvh_bvh* h) {
    CUBVH_GUARD_BEGIN
    if (!h) return CUBVH_OK;
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    for (auto& d : h->dev) {
        if (cudaSetDevice(d.device) == cudaSuccess) {
            cudaFree(d.nodes); cudaFree(d.tris);
            if (d.face_vidx) cudaFree(d.face_vidx);
            if (d.face_slot) cudaFree(d.face_slot);
            if (d.node_box) cudaFree(d.node_box);
            if (d.near_cnt) cudaFree(d.near_cnt);
            if (d.near_lst) cudaFree(d.near_lst);
            if (d.near_nrm) cudaFree(d.near_nrm);
            if (d.near_flag) cudaFree(d.near_flag);
            for (auto& p : d.pipes) {
                if (p.stage) cudaFree(p.stage);
                if (!p.ready) continue;
                cudaStreamDestroy(p.cin); cudaStreamDestroy(p.cout);
                cudaEventDestroy(p.start);
                for (int k = 0; k < kStageSets; ++k) {
                    cudaStreamDestroy(p.comp_s[k]);
                    cudaEventDestroy(p.in[k]); cudaEventDestroy(p.comp[k]); cudaEventDestroy(p.out[k]);
                }
            }
        }
    }
    if (have && !h->dev.empty()) cudaSetDevice(cur);
    delete h;
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_info(const cubvh_bvh* h, int64_t* n_faces, int64_t* n_nodes, int32_t* depth) {
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n_faces) *n_faces = (int64_t)h->ids.size();
    if (n_nodes) *n_nodes = (int64_t)h->host.nodes.size();
    if (depth) *depth = h->host.depth;
    return CUBVH_OK;
}

int cubvh_bvh_state_dict_sizes(const cubvh_bvh* h, int64_t* n_node_records, int64_t* n_tri_records) {
    CUBVH_GUARD_BEGIN
    if (!h || !n_node_records || !n_tri_records) return fail(CUBVH_ERR_INVALID, "null argument");
    // no build needed for the sizes
    *n_node_records = h->sd_nodes.empty() ? reference_format_nodes((int64_t)h->ids.size())
                                          : (int64_t)h->sd_nodes.size() / 9;
    *n_tri_records = (int64_t)h->ids.size();
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_state_dict(const cubvh_bvh* h, int32_t* node_records, int32_t* tri_records) {
    CUBVH_GUARD_BEGIN
    if (!h || !node_records || !tri_records) return fail(CUBVH_ERR_INVALID, "null argument");
    if (!h->sd_nodes.empty()) {
        std::memcpy(node_records, h->sd_nodes.data(), h->sd_nodes.size() * sizeof(int32_t));
        std::memcpy(tri_records, h->sd_tris.data(), h->sd_tris.size() * sizeof(int32_t));
        return CUBVH_OK;
    }
    RefFormat rf;
    export_reference_format(h->xyz.data(), h->ids.data(), (int64_t)h->ids.size(), rf);
    if ((int64_t)rf.nodes.size() != 9 * reference_format_nodes((int64_t)h->ids.size()))
        return fail(CUBVH_ERR_INVALID, "internal: reference-format node count mismatch");
    std::memcpy(node_records, rf.nodes.data(), rf.nodes.size() * sizeof(int32_t));
    std::memcpy(tri_records, rf.tris.data(), rf.tris.size() * sizeof(int32_t));
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_layout(const cubvh_bvh* h, void* nodes_out, void* tris_out) {
    if (!h || !nodes_out || !tris_out) return fail(CUBVH_ERR_INVALID, "null argument");
    std::memcpy(nodes_out, h->host.nodes.data(), h->host.nodes.size() * sizeof(CNode));
    std::memcpy(tris_out, h->host.tris.data(), h->host.tris.size() * sizeof(CTri));
    return CUBVH_OK;
}

int cubvh_bvh_upload(cubvh_bvh* h) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    DevCopy* d;
    return device_copy(h, &d);
    CUBVH_GUARD_END
}

int cubvh_unsigned_distance(cubvh_bvh* h, const float* points, int64_t n, float* distances, int64_t* face_id,
                            float* uvw, void* stream) {
    return cubvh_signed_distance(h, points, n, 0xFFFFFFFFu, distances, face_id, uvw, stream);
}

int cubvh_signed_distance(cubvh_bvh* h, const float* points, int64_t n, uint32_t mode, float* distances,
                          int64_t* face_id, float* uvw, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative query count");
    if (mode != 0 && mode != 1 && mode != 0xFFFFFFFFu)
        return fail(CUBVH_ERR_INVALID, "mode must be 0 (watertight) or 1 (raystab)");
    if (n == 0) return CUBVH_OK;
    if (!points || !distances || !face_id) return fail(CUBVH_ERR_INVALID, "points/distances/face_id is null");
    if (n > (int64_t)UINT32_MAX) return fail(CUBVH_ERR_INVALID, "more than 2^32-1 queries in one call");
    DevCopy* d;
    const int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    const int kmode = mode == 0xFFFFFFFFu ? 0 : (int)mode + 1;
    cudaStream_t s = (cudaStream_t)stream;
    NearLists near;
    if (kmode == 1) {
        const int rc2 = near_lists(h, d, s, &near);
        if (rc2 != CUBVH_OK) return rc2;
    }
    const size_t wsb = query_workspace_bytes(kmode, n);
    void* ws = nullptr;
    cudaError_t e;
    if ((e = pool_alloc(&ws, wsb, s)) != cudaSuccess) return cuda_fail(e, "query workspace allocation");
    e = launch_distance(kmode, uvw != nullptr, n, points, distances, face_id, uvw, d->nodes, d->tris,
                        (int)h->host.slot_of_face0, near, ws, s);
    if (ws) {
        const cudaError_t e2 = cudaFreeAsync(ws, s);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return cuda_fail(e, "distance kernel launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_ray_trace(cubvh_bvh* h, const float* rays_o, const float* rays_d, int64_t n, float* positions,
                    int64_t* face_id, float* depth, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative ray count");
    if (n == 0) return CUBVH_OK;
    if (!rays_o || !rays_d || !positions || !face_id || !depth)
        return fail(CUBVH_ERR_INVALID, "null ray or output pointer");
    DevCopy* d;
    const int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    void* ws = nullptr;
    cudaError_t e = pool_alloc(&ws, query_workspace_bytes(-1, n), s);
    if (e != cudaSuccess) return cuda_fail(e, "ray workspace allocation");
    e = launch_ray(n, rays_o, rays_d, positions, face_id, depth, d->nodes, d->tris, ws, s);
    const cudaError_t e2 = cudaFreeAsync(ws, s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(e, "ray kernel launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

// ------------------------------------------------------- host-buffer queries
// Queries whose inputs and outputs are in host memory run in chunks of
// kHostChunk queries through kStageSets device staging sets (inputs, outputs
// and a query workspace each).  For chunk c (set k = c % kStageSets) the
// copy-in stream uploads its inputs once the kernels of the set's previous
// chunk are done, compute stream k runs the kernels once the inputs are in
// and the set's previous outputs are downloaded, and the copy-out stream
// downloads the outputs once the kernels are done: uploads, kernels of
// several chunks and downloads overlap, and a chunk's kernels fill the SMs
// that the previous chunk's last packets leave idle.  Four sets rather than
// two let a copy-bound call keep uploading while another call's kernels hold
// the SMs (C1 rays + watertight points from host buffers: 24.4 -> 23.2 ms).
// The distance and sign passes run as yielding launches (short-lived blocks
// over the same packet queue), so a call on a higher-priority stream gets SMs
// for its chunk kernels within a block lifetime (23.6 -> 22.8 ms; 1 % slower
// alone).  Every internal stream first waits for the caller's stream; the
// caller's stream then waits for the last downloads.  The staging memory
// belongs to the pipe (one per caller stream) and is kept for the next call:
// allocated on first use, regrown when a call needs more, freed with the BVH
// handle.  Host memory should be page-locked: copies from or to pageable
// memory are staged by the driver and a download to pageable memory blocks
// the enqueueing thread until it is done.
}  // extern "C"

namespace {
// Queries per chunk (2M: measured against 1M and 4M, and against chunks of
// a fixed byte size).
constexpr int64_t kHostChunk = (int64_t)1 << 21;
int64_t host_chunk(int64_t n) { return n < kHostChunk ? n : kHostChunk; }
struct HostArray {
    void* host;
    size_t bytes_per_query;
};

constexpr size_t kMaxPipes = 8;
// The caller stream's pipe (the last one is shared once kMaxPipes exist).
int host_pipe(DevCopy* d, cudaStream_t caller, HostPipe** out) {
    for (auto& q : d->pipes)
        if (q.ready && q.caller == caller) { *out = &q; return CUBVH_OK; }
    if (d->pipes.size() >= kMaxPipes) { *out = &d->pipes.back(); return CUBVH_OK; }
    d->pipes.emplace_back();
    HostPipe& p = d->pipes.back();
    p.caller = caller;
    if (!p.ready) {
        // the internal streams take the caller stream's priority: a caller can
        // give a transfer-bound batch's kernels precedence over others
        int prio = 0;
        cudaError_t e = cudaStreamGetPriority(caller, &prio);
        auto ev = [&](cudaEvent_t* x) { if (e == cudaSuccess) e = cudaEventCreateWithFlags(x, cudaEventDisableTiming); };
        auto mk = [&](cudaStream_t* x) {
            if (e == cudaSuccess) e = cudaStreamCreateWithPriority(x, cudaStreamNonBlocking, prio);
        };
        mk(&p.cin); mk(&p.cout);
        ev(&p.start);
        for (int k = 0; k < kStageSets; ++k) { mk(&p.comp_s[k]); ev(&p.in[k]); ev(&p.comp[k]); ev(&p.out[k]); }
        if (e != cudaSuccess) {
            for (cudaStream_t x : {p.cin, p.cout})
                if (x) cudaStreamDestroy(x);
            if (p.start) cudaEventDestroy(p.start);
            for (int k = 0; k < kStageSets; ++k) {
                if (p.comp_s[k]) cudaStreamDestroy(p.comp_s[k]);
                for (cudaEvent_t x : {p.in[k], p.comp[k], p.out[k]})
                    if (x) cudaEventDestroy(x);
            }
            d->pipes.pop_back();
            return cuda_fail(e, "host-buffer query streams");
        }
        p.ready = true;
    }
    *out = &p;
    return CUBVH_OK;
}

// launch(in, out, ws, first, count, stream): the kernels of one chunk, in[i] /
// out[i] the device copies of the i-th input / output array.
// chunk: queries per chunk (host_chunk), which ws_bytes is sized for.
template <class Launch>
int run_host_pipeline(cubvh_bvh* h, DevCopy* d, cudaStream_t s, int64_t n, int64_t chunk,
                      const std::vector<HostArray>& ins, const std::vector<HostArray>& outs, size_t ws_bytes,
                      Launch launch) {
    constexpr int sets = kStageSets;
    std::lock_guard<std::mutex> lk(h->mu);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        return fail(CUBVH_ERR_INVALID, "host-buffer queries cannot run while the stream is being captured");
    HostPipe* p;
    int rc = host_pipe(d, s, &p);
    if (rc != CUBVH_OK) return rc;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t per_set = 0;
    for (const auto& a : ins) per_set += al(a.bytes_per_query * (size_t)chunk);
    for (const auto& a : outs) per_set += al(a.bytes_per_query * (size_t)chunk);
    const size_t need = (size_t)sets * (per_set + al(ws_bytes));
    if (need > p->stage_bytes) {  // grow: wait until the previous calls on this pipe are done with it
        e = cudaStreamSynchronize(p->cout);
        for (int k = 0; k < kStageSets && e == cudaSuccess; ++k) e = cudaStreamSynchronize(p->comp_s[k]);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->cin);
        if (e != cudaSuccess) return cuda_fail(e, "host-query staging");
        if (p->stage) cudaFree(p->stage);
        p->stage = nullptr;
        p->stage_bytes = 0;
        if ((e = cudaMalloc(reinterpret_cast<void**>(&p->stage), need)) != cudaSuccess)
            return cuda_fail(e, "cudaMalloc(host-query staging)");
        p->stage_bytes = need;
    }
    char* base = p->stage;
    std::vector<char*> dev_in[kStageSets], dev_out[kStageSets];
    void* ws[kStageSets];
    for (int k = 0; k < sets; ++k) {
        char* q = base + k * per_set;
        for (const auto& a : ins) { dev_in[k].push_back(q); q += al(a.bytes_per_query * (size_t)chunk); }
        for (const auto& a : outs) { dev_out[k].push_back(q); q += al(a.bytes_per_query * (size_t)chunk); }
        ws[k] = base + (size_t)sets * per_set + k * al(ws_bytes);
    }
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; return e == cudaSuccess; };
    ok(cudaEventRecord(p->start, s));
    // every internal stream starts after the caller's earlier work and after
    // the previous call on this pipe has downloaded its last chunks (its
    // uploads and kernels come before those); an event never recorded is a no-op
    auto after_previous = [&](cudaStream_t q) {
        ok(cudaStreamWaitEvent(q, p->start, 0));
        for (int k = 0; k < kStageSets; ++k) ok(cudaStreamWaitEvent(q, p->out[k], 0));
    };
    after_previous(p->cin);
    after_previous(p->cout);
    for (int k = 0; k < kStageSets; ++k) after_previous(p->comp_s[k]);
    const int64_t nchunks = (n + chunk - 1) / chunk;
    for (int64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
        const int k = (int)(c % sets);
        const int64_t first = c * chunk, cnt = n - first < chunk ? n - first : chunk;
        if (c >= sets) ok(cudaStreamWaitEvent(p->cin, p->comp[k], 0));
        for (size_t i = 0; i < ins.size(); ++i)
            ok(cudaMemcpyAsync(dev_in[k][i], static_cast<const char*>(ins[i].host) + first * ins[i].bytes_per_query,
                               cnt * ins[i].bytes_per_query, cudaMemcpyHostToDevice, p->cin));
        ok(cudaEventRecord(p->in[k], p->cin));
        cudaStream_t cs = p->comp_s[k];
        ok(cudaStreamWaitEvent(cs, p->in[k], 0));
        if (c >= sets) ok(cudaStreamWaitEvent(cs, p->out[k], 0));
        if (e == cudaSuccess) ok(launch(dev_in[k], dev_out[k], ws[k], first, cnt, cs));
        ok(cudaEventRecord(p->comp[k], cs));
        ok(cudaStreamWaitEvent(p->cout, p->comp[k], 0));
        for (size_t i = 0; i < outs.size(); ++i)
            ok(cudaMemcpyAsync(static_cast<char*>(outs[i].host) + first * outs[i].bytes_per_query, dev_out[k][i],
                               cnt * outs[i].bytes_per_query, cudaMemcpyDeviceToHost, p->cout));
        ok(cudaEventRecord(p->out[k], p->cout));
    }
    for (int64_t k = 0; k < sets && k < nchunks; ++k) ok(cudaStreamWaitEvent(s, p->out[k], 0));
    if (e != cudaSuccess) {
        // copies already queued may still read or write the caller's host
        // buffers: let them finish before reporting the error
        cudaStreamSynchronize(p->cin);
        for (int k = 0; k < kStageSets; ++k) cudaStreamSynchronize(p->comp_s[k]);
        cudaStreamSynchronize(p->cout);
        return cuda_fail(e, "host-buffer query");
    }
    return CUBVH_OK;
}
}  // namespace

extern "C" {

int cubvh_ray_trace_host(cubvh_bvh* h, const float* rays_o, const float* rays_d, int64_t n, float* positions,
                         int64_t* face_id, float* depth, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative ray count");
    if (n == 0) return CUBVH_OK;
    if (!rays_o || !rays_d || !positions || !face_id || !depth)
        return fail(CUBVH_ERR_INVALID, "null ray or output pointer");
    DevCopy* d;
    const int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t chunk = host_chunk(n);
    return run_host_pipeline(
        h, d, s, n, chunk, {{const_cast<float*>(rays_o), 12}, {const_cast<float*>(rays_d), 12}},
        {{positions, 12}, {face_id, 8}, {depth, 4}}, query_workspace_bytes(-1, chunk),
        [&](const std::vector<char*>& in, const std::vector<char*>& out, void* ws, int64_t, int64_t cnt,
            cudaStream_t cs) {
            return launch_ray(cnt, reinterpret_cast<const float*>(in[0]), reinterpret_cast<const float*>(in[1]),
                              reinterpret_cast<float*>(out[0]), reinterpret_cast<int64_t*>(out[1]),
                              reinterpret_cast<float*>(out[2]), d->nodes, d->tris, ws, cs);
        });
    CUBVH_GUARD_END
}

int cubvh_signed_distance_host(cubvh_bvh* h, const float* points, int64_t n, uint32_t mode, float* distances,
                               int64_t* face_id, float* uvw, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative query count");
    if (mode != 0 && mode != 1 && mode != 0xFFFFFFFFu)
        return fail(CUBVH_ERR_INVALID, "mode must be 0 (watertight), 1 (raystab) or 0xFFFFFFFF (unsigned)");
    if (n == 0) return CUBVH_OK;
    if (!points || !distances || !face_id) return fail(CUBVH_ERR_INVALID, "points/distances/face_id is null");
    if (n > (int64_t)UINT32_MAX) return fail(CUBVH_ERR_INVALID, "more than 2^32-1 queries in one call");
    DevCopy* d;
    int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    const int kmode = mode == 0xFFFFFFFFu ? 0 : (int)mode + 1;
    cudaStream_t s = (cudaStream_t)stream;
    NearLists near;
    if (kmode == 1 && (rc = near_lists(h, d, s, &near)) != CUBVH_OK) return rc;
    std::vector<HostArray> outs{{distances, 4}, {face_id, 8}};
    if (uvw) outs.push_back({uvw, 12});
    const int64_t chunk = host_chunk(n);
    const int slot0 = (int)h->host.slot_of_face0;
    return run_host_pipeline(
        h, d, s, n, chunk, {{const_cast<float*>(points), 12}}, outs, query_workspace_bytes(kmode, chunk),
        [&](const std::vector<char*>& in, const std::vector<char*>& out, void* ws, int64_t first, int64_t cnt,
            cudaStream_t cs) {
            return launch_distance(kmode, uvw != nullptr, cnt, reinterpret_cast<const float*>(in[0]),
                                   reinterpret_cast<float*>(out[0]), reinterpret_cast<int64_t*>(out[1]),
                                   uvw ? reinterpret_cast<float*>(out[2]) : nullptr, d->nodes, d->tris, slot0, near,
                                   ws, cs, first, /*yield=*/true);
        });
    CUBVH_GUARD_END
}

// ---------------------------------------------------- sparse marching cubes
struct cubvh_smc {
    SparseMCResult r;
    int device = -1;
    cudaEvent_t done = nullptr;          // recorded on the building stream after its last kernel
    std::vector<cudaEvent_t> fetched;    // recorded on each fetch's stream after its copies
};

int cubvh_sparse_marching_cubes(const int32_t* coords, const float* corners, int64_t n, float iso,
                                int ensure_consistency, void* stream, cubvh_smc** out, int64_t* n_verts,
                                int64_t* n_tris) {
    CUBVH_GUARD_BEGIN
    if (!out || !n_verts || !n_tris) return fail(CUBVH_ERR_INVALID, "out/n_verts/n_tris is null");
    *out = nullptr; *n_verts = 0; *n_tris = 0;
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative voxel count");
    if (n > 0 && (!coords || !corners)) return fail(CUBVH_ERR_INVALID, "coords/corners is null");
    auto* m = new cubvh_smc();
    if (n == 0) {  // empty result: no device work, no buffers, no event
        *out = m;
        return CUBVH_OK;
    }
    cudaGetDevice(&m->device);
    std::string err;
    const int rc = sparse_mc_run(coords, corners, n, iso, (ensure_consistency & CUBVH_SMC_ENSURE_CONSISTENCY) != 0,
                                 (ensure_consistency & CUBVH_SMC_CLOSED) != 0, (cudaStream_t)stream, m->r, err);
    if (rc != 0) {
        cudaStreamSynchronize((cudaStream_t)stream);  // kernels may still write the result buffers
        cubvh_sparse_mc_free(m);
        return fail(rc == 1 ? CUBVH_ERR_INVALID : CUBVH_ERR_CUDA, err);
    }
    // the merge and remap kernels may still run: a fetch on another stream waits for them
    cudaError_t e = cudaEventCreateWithFlags(&m->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(m->done, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        cudaStreamSynchronize((cudaStream_t)stream);
        cubvh_sparse_mc_free(m);
        return cuda_fail(e, "sparse marching cubes event");
    }
    *out = m;
    *n_verts = m->r.n_verts;
    *n_tris = m->r.n_tris;
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_sparse_mc_fetch(cubvh_smc* m, float* verts, int32_t* tris, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!m) return fail(CUBVH_ERR_INVALID, "result is null");
    if ((m->r.n_verts && !verts) || (m->r.n_tris && !tris)) return fail(CUBVH_ERR_INVALID, "verts/tris is null");
    if (!m->r.n_verts && !m->r.n_tris) return CUBVH_OK;  // nothing to copy
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = m->done ? cudaStreamWaitEvent(s, m->done, 0) : cudaSuccess;
    if (e == cudaSuccess && m->r.n_verts)
        e = cudaMemcpyAsync(verts, m->r.verts, sizeof(float) * 3 * m->r.n_verts, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && m->r.n_tris)
        e = cudaMemcpyAsync(tris, m->r.tris, sizeof(int32_t) * 3 * m->r.n_tris, cudaMemcpyDeviceToDevice, s);
    cudaEvent_t ev = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        m->fetched.push_back(ev);  // owned by the result from here on
        e = cudaEventRecord(ev, s);
    }
    if (e != cudaSuccess) {
        cudaStreamSynchronize(s);  // the free must not overtake copies already queued
        return cuda_fail(e, "sparse marching cubes fetch");
    }
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_sparse_mc_free(cubvh_smc* m) {
    if (!m) return CUBVH_OK;
    if (m->device < 0) {  // empty result: nothing on a device
        delete m;
        return CUBVH_OK;
    }
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    if (cudaSetDevice(m->device) == cudaSuccess) {
        // wait for this result's own work only: the build and every fetch
        if (m->done) cudaEventSynchronize(m->done);
        for (cudaEvent_t ev : m->fetched) cudaEventSynchronize(ev);
        sparse_mc_release(m->r);
        if (m->done) cudaEventDestroy(m->done);
        for (cudaEvent_t ev : m->fetched) cudaEventDestroy(ev);
    }
    if (have) cudaSetDevice(cur);
    delete m;
    return CUBVH_OK;
}

static int check_grid_dims(int B, int H, int W, int D) {
    if (B < 0 || H < 0 || W < 0 || D < 0) return fail(CUBVH_ERR_INVALID, "negative grid dimension");
    const int64_t ntot = (int64_t)B * H * W * D;
    if (ntot >= (int64_t)INT32_MAX) return fail(CUBVH_ERR_INVALID, "grid has 2^31 or more voxels (int32 labels)");
    return CUBVH_OK;
}

int cubvh_floodfill_workspace_size(int B, int H, int W, int D, size_t* bytes) {
    if (!bytes) return fail(CUBVH_ERR_INVALID, "bytes is null");
    const int rc = check_grid_dims(B, H, W, D);
    if (rc != CUBVH_OK) return rc;
    *bytes = floodfill_workspace_bytes(B, H, W, D);
    return CUBVH_OK;
}

int cubvh_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* workspace,
                    size_t workspace_bytes, void* stream) {
    CUBVH_GUARD_BEGIN
    int rc = check_grid_dims(B, H, W, D);
    if (rc != CUBVH_OK) return rc;
    if ((int64_t)B * H * W * D == 0) return CUBVH_OK;
    if (!grid || !labels) return fail(CUBVH_ERR_INVALID, "grid/labels is null");
    const size_t need = floodfill_workspace_bytes(B, H, W, D);
    cudaStream_t s = (cudaStream_t)stream;
    void* ws = workspace;
    cudaError_t e;
    if (ws) {
        if (workspace_bytes < need) return fail(CUBVH_ERR_INVALID, "workspace smaller than cubvh_floodfill_workspace_size()");
        if (reinterpret_cast<uintptr_t>(ws) & 255) return fail(CUBVH_ERR_INVALID, "workspace must be 256-byte aligned");
    } else if ((e = pool_alloc(&ws, need, s)) != cudaSuccess) {
        return cuda_fail(e, "floodfill workspace allocation");
    }
    e = launch_floodfill(grid, B, H, W, D, labels, ws, s);
    if (!workspace) {
        const cudaError_t e2 = cudaFreeAsync(ws, s);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return cuda_fail(e, "floodfill launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_udf_to_sdf(const float* udf, int B, int H, int W, int D, float eps, float* sdf, void* workspace,
                     size_t workspace_bytes, void* stream) {
    CUBVH_GUARD_BEGIN
    int rc = check_grid_dims(B, H, W, D);
    if (rc != CUBVH_OK) return rc;
    if ((int64_t)B * H * W * D == 0) return CUBVH_OK;
    if (!udf || !sdf) return fail(CUBVH_ERR_INVALID, "udf/sdf is null");
    if (!(eps == eps)) return fail(CUBVH_ERR_INVALID, "eps is NaN");
    const size_t need = floodfill_workspace_bytes(B, H, W, D);
    cudaStream_t s = (cudaStream_t)stream;
    void* ws = workspace;
    cudaError_t e;
    if (ws) {
        if (workspace_bytes < need) return fail(CUBVH_ERR_INVALID, "workspace smaller than cubvh_floodfill_workspace_size()");
        if (reinterpret_cast<uintptr_t>(ws) & 255) return fail(CUBVH_ERR_INVALID, "workspace must be 256-byte aligned");
    } else if ((e = pool_alloc(&ws, need, s)) != cudaSuccess) {
        return cuda_fail(e, "udf_to_sdf workspace allocation");
    }
    e = launch_udf_to_sdf(udf, B, H, W, D, eps, sdf, ws, s);
    if (!workspace) {
        const cudaError_t e2 = cudaFreeAsync(ws, s);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return cuda_fail(e, "udf_to_sdf launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_floodfill_check(const void* workspace, int B, int H, int W, int D, void* stream) {
    CUBVH_GUARD_BEGIN
    int rc = check_grid_dims(B, H, W, D);
    if (rc != CUBVH_OK) return rc;
    if (!workspace) {
        // the fixed array of cubvh_floodfill_noalloc
        std::string err;
        void* ws = nullptr;
        if ((rc = floodfill_noalloc_fits(B, H, W, D, err)) != CUBVH_OK ||
            (rc = floodfill_noalloc_scratch(&ws, err)) != CUBVH_OK)
            return fail(rc, err);
        workspace = ws;
    }
    int status = 0;
    const char* p = static_cast<const char*>(workspace) + floodfill_status_offset(B, H, W, D);
    cudaError_t e = cudaMemcpyAsync(&status, p, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "floodfill status read");
    if (status != 0) return fail(CUBVH_ERR_DEVICE_BOUND, "floodfill: a union-find walk exceeded its step bound");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_bvh_refit(cubvh_bvh* h, const float* vertices, int64_t n_vertices, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h || !vertices) return fail(CUBVH_ERR_INVALID, "bvh/vertices is null");
    if (h->host.faces.empty()) return fail(CUBVH_ERR_INVALID, "refit needs a BVH created from vertices and faces");
    if (n_vertices != h->host.n_vertices)
        return fail(CUBVH_ERR_INVALID, "refit: vertex count differs from the mesh the BVH was built on");
    DevCopy* d;
    int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    if ((rc = grad_buffers(h, d, true)) != CUBVH_OK) return rc;
    cudaError_t e;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        if (!d->node_box && (e = cudaMalloc(&d->node_box, h->host.nodes.size() * 6 * sizeof(float))) != cudaSuccess)
            return cuda_fail(e, "cudaMalloc(refit scratch)");
        d->near_valid = false;  // the triangles move: rebuild the watertight lists on next use
    }
    e = launch_refit((int64_t)h->host.tris.size(), d->tris, d->face_vidx, vertices, d->nodes, d->node_box,
                     h->host.level_start.data(), (int)h->host.level_start.size() - 1, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "refit launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_distance_backward(cubvh_bvh* h, const float* points, int64_t n, const int64_t* face_id,
                            const float* grad_distances, const float* distances, const float* vertices,
                            float* grad_points, float* grad_vertices, void* stream) {
    CUBVH_GUARD_BEGIN
    if (!h) return fail(CUBVH_ERR_INVALID, "bvh is null");
    if (n < 0) return fail(CUBVH_ERR_INVALID, "negative query count");
    if (n == 0) return CUBVH_OK;
    if (!points || !face_id || !grad_distances || !distances)
        return fail(CUBVH_ERR_INVALID, "points/face_id/grad_distances/distances is null");
    if (grad_vertices && !vertices) return fail(CUBVH_ERR_INVALID, "grad_vertices needs the current vertices");
    DevCopy* d;
    int rc = device_copy(h, &d);
    if (rc != CUBVH_OK) return rc;
    if ((rc = grad_buffers(h, d, vertices != nullptr)) != CUBVH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nf = (int64_t)h->ids.size();
    void* ws = nullptr;
    cudaError_t e = pool_alloc(&ws, backward_workspace_bytes(n, nf), s);
    if (e != cudaSuccess) return cuda_fail(e, "backward workspace allocation");
    e = launch_backward(n, points, face_id, grad_distances, distances, vertices, vertices ? d->face_vidx : nullptr,
                        d->face_slot, d->tris, nf, grad_points, grad_vertices, ws, s);
    const cudaError_t e2 = cudaFreeAsync(ws, s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(e, "backward launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

int cubvh_stab_directions(int64_t first, int64_t n, float* dirs, void* stream) {
    CUBVH_GUARD_BEGIN
    if (n < 0 || first < 0) return fail(CUBVH_ERR_INVALID, "negative query index or count");
    if (n == 0) return CUBVH_OK;
    if (!dirs) return fail(CUBVH_ERR_INVALID, "dirs is null");
    if (first + n > ((int64_t)1 << 32)) return fail(CUBVH_ERR_INVALID, "query indices beyond 2^32");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = ensure_constants(device)) != cudaSuccess) return cuda_fail(e, "constant upload");
    if ((e = launch_stab_dirs(first, n, dirs, (cudaStream_t)stream)) != cudaSuccess)
        return cuda_fail(e, "stab directions launch");
    return CUBVH_OK;
    CUBVH_GUARD_END
}

// Floodfill that allocates nothing: see include/cubvh_b200.h.
int cubvh_floodfill_noalloc(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* stream) {
    CUBVH_GUARD_BEGIN
    const int rc = check_grid_dims(B, H, W, D);
    if (rc != CUBVH_OK) return rc;
    if ((int64_t)B * H * W * D == 0) return CUBVH_OK;
    if (!grid || !labels) return fail(CUBVH_ERR_INVALID, "grid/labels is null");
    std::string err;
    const int st = floodfill_noalloc(grid, B, H, W, D, labels, (cudaStream_t)stream, err);
    if (st != CUBVH_OK) return fail(st, err);
    return CUBVH_OK;
    CUBVH_GUARD_END
}

}  // extern "C"
