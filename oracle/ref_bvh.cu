// TEST INFRASTRUCTURE ONLY.  Compiles the reference's own BVH query code
// (ashawkey/cubvh src/bvh.cu with include/gpu/{common.h, triangle.cuh,
// bounding_box.cuh, bvh.cuh, pcg32.h, gpu_memory.h}) unchanged, from the
// reference tree where it lies (oracle/Makefile, target `ref`), into
// oracle/_ref/libref_bvh.so.  The Eigen it includes is the project-written
// stand-in under oracle/eigen_standin (the reference's Eigen submodule is
// empty).  The tests compare the cubvh_b200 kernels with the reference's
// outputs through it, and bench.py's reference arm times it; the cubvh_b200
// package never loads it.
//
// What it exposes, all from the reference's own code:
//  - the BVH4 build (src/bvh.cu:515-620) over the triangle soup built the way
//    cuBVHImpl builds it (src/api_gpu.cu:21-40: face i -> Triangle{a, b, c, i},
//    leaf size 8), and its nodes / triangles in state_dict byte order;
//  - the four GPU launchers (src/bvh.cu:430-513), on the caller's stream, with
//    the node upload done lazily by the reference itself;
//  - the same four queries on the host cores: the reference's __host__
//    traversals (src/bvh.cu:145-427) called per query exactly as the kernels
//    call them (src/bvh.cu:631-740), split over OpenMP threads;
//  - the raystab stab-ray directions as the reference's device code computes
//    them (pcg32 advanced by 2*i, two next_float draws, fibonacci_dir<32>:
//    src/bvh.cu:658-685, 408-427, include/gpu/common.h:63-96).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <string>
#include <vector>

#include <omp.h>

#include "src/bvh.cu"  // found through -I<reference>; includes gpu/*.h via -I<reference>/include

namespace {

using cubvh::Triangle;
using cubvh::TriangleBvhNode;

// The reference's BVH4 with access to its node array (protected in
// TriangleBvh) and the triangle soup that cuBVHImpl keeps beside it.
struct RefMesh : public cubvh::TriangleBvh4 {
    std::vector<Triangle> tris;
    cubvh::GPUMemory<Triangle> tris_gpu;
    const std::vector<TriangleBvhNode>& nodes() const { return m_nodes; }
    const Triangle* gpu_tris() {
        if (tris_gpu.data() == nullptr) tris_gpu.resize_and_copy_from_host(tris);  // api_gpu.cu:77-79
        return tris_gpu.data();
    }
};

thread_local std::string g_err;

// Runs fn, turning a C++ exception (or, with cuda = true, a CUDA error left
// by the launch) into status 2 and a message.  Host-only work passes
// cuda = false, so that it also runs on machines without a GPU.
template <class F>
int guarded(F fn, bool cuda = true) {
    try {
        fn();
    } catch (const std::exception& e) {
        g_err = e.what();
        return 2;
    }
    if (!cuda) return 0;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_err = cudaGetErrorString(e);
        return 2;
    }
    return 0;
}

inline Eigen::Vector3f load3(const float* p, int64_t i) { return Eigen::Vector3f(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline void store3(float* p, int64_t i, const Eigen::Vector3f& v) {
    p[3 * i] = v.x();
    p[3 * i + 1] = v.y();
    p[3 * i + 2] = v.z();
}

// Kernel: the stab directions of queries first .. first+n-1, [n, 32, 3],
// computed exactly as signed_distance_raystab_kernel does for its thread i.
__global__ void stab_directions_kernel(uint32_t n, uint32_t first, float* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = first + k;
    cubvh::pcg32 rng;
    rng.advance(i * 2);
    Eigen::Vector2f offset = {rng.next_float(), rng.next_float()};
    for (uint32_t j = 0; j < 32; ++j) {
        const Eigen::Vector3f d = cubvh::fibonacci_dir<32>(j, offset);
        float* o = out + ((size_t)k * 32 + j) * 3;
        o[0] = d.x();
        o[1] = d.y();
        o[2] = d.z();
    }
}

}  // namespace

extern "C" {

const char* ref_bvh_last_error() { return g_err.c_str(); }

// verts: float32 [nv, 3]; faces: int64 [nf, 3] (validated by the caller).
void* ref_bvh_create(const float* verts, int64_t nv, const int64_t* faces, int64_t nf) {
    (void)nv;
    RefMesh* m = nullptr;
    const int rc = guarded([&] {
        m = new RefMesh();
        m->tris.resize((size_t)nf);
        for (int64_t i = 0; i < nf; ++i) {
            Triangle& t = m->tris[(size_t)i];
            t.a = load3(verts, faces[3 * i]);
            t.b = load3(verts, faces[3 * i + 1]);
            t.c = load3(verts, faces[3 * i + 2]);
            t.id = i;
        }
        m->build(m->tris, 8);
    }, false);
    if (rc != 0) {
        delete m;
        return nullptr;
    }
    return m;
}

void ref_bvh_destroy(void* h) { delete static_cast<RefMesh*>(h); }

int64_t ref_bvh_num_nodes(void* h) { return (int64_t)static_cast<RefMesh*>(h)->nodes().size(); }

// nodes: int32 [n_nodes, 9]; tris: int32 [nf, 12] (the state_dict records).
void ref_bvh_export(void* h, int32_t* nodes, int32_t* tris) {
    RefMesh* m = static_cast<RefMesh*>(h);
    static_assert(sizeof(TriangleBvhNode) == 36 && sizeof(Triangle) == 48, "reference record sizes");
    std::memcpy(nodes, m->nodes().data(), m->nodes().size() * sizeof(TriangleBvhNode));
    std::memcpy(tris, m->tris.data(), m->tris.size() * sizeof(Triangle));
}

// ---- the reference's GPU launchers (device pointers, caller stream)

int ref_bvh_unsigned_distance_gpu(void* h, const float* pts, int64_t n, float* dist, int64_t* fid, float* uvw,
                                  void* stream) {
    RefMesh* m = static_cast<RefMesh*>(h);
    return guarded([&] { m->unsigned_distance_gpu((uint32_t)n, pts, dist, fid, uvw, m->gpu_tris(), (cudaStream_t)stream); });
}

int ref_bvh_signed_distance_gpu(void* h, const float* pts, int64_t n, int mode, float* dist, int64_t* fid,
                                float* uvw, void* stream) {
    RefMesh* m = static_cast<RefMesh*>(h);
    return guarded([&] {
        m->signed_distance_gpu((uint32_t)n, (uint32_t)mode, pts, dist, fid, uvw, m->gpu_tris(), (cudaStream_t)stream);
    });
}

int ref_bvh_ray_trace_gpu(void* h, const float* ro, const float* rd, int64_t n, float* pos, int64_t* fid,
                          float* depth, void* stream) {
    RefMesh* m = static_cast<RefMesh*>(h);
    return guarded([&] { m->ray_trace_gpu((uint32_t)n, ro, rd, pos, fid, depth, m->gpu_tris(), (cudaStream_t)stream); });
}

// The same directions from the reference's host build of the same code
// (host sincosf and host float rounding).
void ref_stab_directions_host(int64_t first, int64_t n, float* out) {
    for (int64_t k = 0; k < n; ++k) {
        const uint32_t i = (uint32_t)(first + k);
        cubvh::pcg32 rng;
        rng.advance(i * 2);
        Eigen::Vector2f offset = {rng.next_float(), rng.next_float()};
        for (uint32_t j = 0; j < 32; ++j) store3(out, k * 32 + j, cubvh::fibonacci_dir<32>(j, offset));
    }
}

int ref_stab_directions_gpu(int64_t first, int64_t n, float* out, void* stream) {
    return guarded([&] {
        if (n <= 0) return;
        stab_directions_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>((uint32_t)n,
                                                                                              (uint32_t)first, out);
    });
}

// ---- the reference's host traversals, per query as its kernels do

// stride: take every stride-th query (sample for timing); outputs are dense
// [ceil(n / stride)].  threads <= 0: all OpenMP threads.
int ref_bvh_unsigned_distance_host(void* h, const float* pts, int64_t n, int64_t stride, float* dist, int64_t* fid,
                                   float* uvw, int threads) {
    RefMesh* m = static_cast<RefMesh*>(h);
    const TriangleBvhNode* nodes = m->nodes().data();
    const Triangle* tris = m->tris.data();
    const int64_t cnt = (n + stride - 1) / stride;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int64_t k = 0; k < cnt; ++k) {
        const Eigen::Vector3f point = load3(pts, k * stride);
        auto res = cubvh::TriangleBvh4::closest_triangle(point, nodes, tris, cubvh::MAX_DIST * cubvh::MAX_DIST);
        dist[k] = res.second;
        fid[k] = tris[res.first].id;
        if (uvw) store3(uvw, k, tris[res.first].barycentric(tris[res.first].closest_point(point)));
    }
    return 0;
}

// first_index: the call-wide index of query 0 (raystab seeds pcg32 with it).
int ref_bvh_signed_distance_host(void* h, const float* pts, int64_t n, int64_t stride, int mode, int64_t first_index,
                                 float* dist, int64_t* fid, float* uvw, int threads) {
    RefMesh* m = static_cast<RefMesh*>(h);
    const TriangleBvhNode* nodes = m->nodes().data();
    const Triangle* tris = m->tris.data();
    const int64_t cnt = (n + stride - 1) / stride;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t k = 0; k < cnt; ++k) {
        const Eigen::Vector3f point = load3(pts, k * stride);
        std::pair<int, float> res;
        if (mode == 0) {
            res = cubvh::TriangleBvh4::signed_distance_watertight(point, nodes, tris, cubvh::MAX_DIST * cubvh::MAX_DIST);
        } else {
            const uint32_t i = (uint32_t)(first_index + k * stride);
            cubvh::pcg32 rng;
            rng.advance(i * 2);
            res = cubvh::TriangleBvh4::signed_distance_raystab(point, nodes, tris, cubvh::MAX_DIST * cubvh::MAX_DIST,
                                                               rng);
        }
        dist[k] = res.second;
        fid[k] = tris[res.first].id;
        if (uvw) store3(uvw, k, tris[res.first].barycentric(tris[res.first].closest_point(point)));
    }
    return 0;
}

int ref_bvh_ray_trace_host(void* h, const float* ro, const float* rd, int64_t n, int64_t stride, float* pos,
                           int64_t* fid, float* depth, int threads) {
    RefMesh* m = static_cast<RefMesh*>(h);
    const TriangleBvhNode* nodes = m->nodes().data();
    const Triangle* tris = m->tris.data();
    const int64_t cnt = (n + stride - 1) / stride;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int64_t k = 0; k < cnt; ++k) {
        const Eigen::Vector3f o = load3(ro, k * stride), d = load3(rd, k * stride);
        auto res = cubvh::TriangleBvh4::ray_intersect(o, d, nodes, tris);
        depth[k] = res.second;
        store3(pos, k, o + res.second * d);
        fid[k] = res.first >= 0 ? tris[res.first].id : -1;
    }
    return 0;
}

}  // extern "C"
