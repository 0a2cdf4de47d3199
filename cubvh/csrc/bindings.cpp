// The `_cubvh` torch extension: the reference's pybind module surface
// (src/bindings.cpp:14-32: class cuBVH with ray_trace / unsigned_distance /
// signed_distance / state_dict, create_cuBVH, from_state_dict, floodfill,
// sparse_marching_cubes) as a thin layer over the C ABI of
// libcubvh_b200.so (include/cubvh_b200.h).  Every call forwards to one C
// entry point; a non-zero status becomes a C++ exception, which pybind11
// turns into RuntimeError, as the reference's TORCH_CHECK / runtime_error do.
//
// Differences from the reference's binding, all on the safe side: query
// tensors are checked (device, dtype, shape, contiguity) before the launch,
// each call runs on the device of its tensors (device guard), and floodfill
// runs on the current stream and reports the union-find bound.
#include <torch/extension.h>
#include <pybind11/numpy.h>

#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>

#include "../../include/cubvh_b200.h"

namespace py = pybind11;

namespace {

// Record format written by state_dict(): the reference's records (version 1).
constexpr int32_t kStateDictVersion = 1;

void check(int rc, const char* what) {
    if (rc != CUBVH_OK) throw std::runtime_error(std::string(what) + ": " + cubvh_last_error());
}

void* stream_of(const at::Tensor& t) { return at::cuda::getCurrentCUDAStream(t.device().index()).stream(); }

// CUDA, contiguous, dtype, [n, cols] (cols == 0: [n]).
void expect(const at::Tensor& t, at::ScalarType dt, int64_t n, int64_t cols, const char* name) {
    TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
    TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
    TORCH_CHECK(t.scalar_type() == dt, name, " has dtype ", t.scalar_type(), ", expected ", dt);
    if (cols == 0) {
        TORCH_CHECK(t.dim() == 1 && t.size(0) == n, name, " must have shape [", n, "]");
    } else {
        TORCH_CHECK(t.dim() == 2 && t.size(0) == n && t.size(1) == cols, name, " must have shape [", n, ", ", cols,
                    "]");
    }
}

void same_device(const at::Tensor& a, const at::Tensor& b, const char* name) {
    TORCH_CHECK(a.device() == b.device(), name, " is on ", b.device(), ", the queries on ", a.device());
}

class cuBVH {
public:
    explicit cuBVH(cubvh_bvh* h) : h_(h) {}
    ~cuBVH() { cubvh_bvh_destroy(h_); }
    cuBVH(const cuBVH&) = delete;
    cuBVH& operator=(const cuBVH&) = delete;

    // src/api_gpu.cu:70-82; outputs preallocated by the caller, asynchronous
    void ray_trace(at::Tensor rays_o, at::Tensor rays_d, at::Tensor positions, at::Tensor face_id,
                   at::Tensor depth) {
        const int64_t n = rays_o.size(0);
        expect(rays_o, at::kFloat, n, 3, "rays_o");
        expect(rays_d, at::kFloat, n, 3, "rays_d");
        expect(positions, at::kFloat, n, 3, "positions");
        expect(face_id, at::kLong, n, 0, "face_id");
        expect(depth, at::kFloat, n, 0, "depth");
        for (const at::Tensor* t : {&rays_d, &positions, &face_id, &depth}) same_device(rays_o, *t, "an output");
        const c10::cuda::CUDAGuard guard(rays_o.device());
        check(cubvh_ray_trace(h_, rays_o.data_ptr<float>(), rays_d.data_ptr<float>(), n, positions.data_ptr<float>(),
                              face_id.data_ptr<int64_t>(), depth.data_ptr<float>(), stream_of(rays_o)),
              "ray_trace");
    }

    // src/api_gpu.cu:84-97
    void unsigned_distance(at::Tensor positions, at::Tensor distances, at::Tensor face_id,
                           c10::optional<at::Tensor> uvw) {
        query(positions, distances, face_id, uvw, 0xFFFFFFFFu, "unsigned_distance");
    }

    // src/api_gpu.cu:99-108; mode 0 watertight, 1 raystab
    void signed_distance(at::Tensor positions, at::Tensor distances, at::Tensor face_id,
                         c10::optional<at::Tensor> uvw, uint32_t mode) {
        TORCH_CHECK(mode <= 1, "signed_distance: mode must be 0 (watertight) or 1 (raystab)");
        query(positions, distances, face_id, uvw, mode, "signed_distance");
    }

    // src/api_gpu.cu:110-121, include/gpu/bvh.cuh:84-94: CPU int32 records
    std::unordered_map<std::string, at::Tensor> state_dict() const {
        int64_t nn = 0, nt = 0;
        check(cubvh_bvh_state_dict_sizes(h_, &nn, &nt), "state_dict");
        at::Tensor nodes = at::empty({nn, 9}, at::TensorOptions().dtype(at::kInt));
        at::Tensor tris = at::empty({nt, 12}, at::TensorOptions().dtype(at::kInt));
        check(cubvh_bvh_state_dict(h_, nodes.data_ptr<int32_t>(), tris.data_ptr<int32_t>()), "state_dict");
        at::Tensor version = at::full({1}, kStateDictVersion, at::TensorOptions().dtype(at::kInt));
        return {{"nodes", nodes}, {"triangles", tris}, {"version", version}};
    }

private:
    void query(at::Tensor& positions, at::Tensor& distances, at::Tensor& face_id, c10::optional<at::Tensor>& uvw,
               uint32_t mode, const char* what) {
        const int64_t n = positions.size(0);
        expect(positions, at::kFloat, n, 3, "positions");
        expect(distances, at::kFloat, n, 0, "distances");
        expect(face_id, at::kLong, n, 0, "face_id");
        same_device(positions, distances, "distances");
        same_device(positions, face_id, "face_id");
        float* uvw_ptr = nullptr;
        if (uvw.has_value()) {
            expect(*uvw, at::kFloat, n, 3, "uvw");
            same_device(positions, *uvw, "uvw");
            uvw_ptr = uvw->data_ptr<float>();
        }
        const c10::cuda::CUDAGuard guard(positions.device());
        check(cubvh_signed_distance(h_, positions.data_ptr<float>(), n, mode, distances.data_ptr<float>(),
                                    face_id.data_ptr<int64_t>(), uvw_ptr, stream_of(positions)),
              what);
    }

    cubvh_bvh* h_;
};

// src/api_gpu.cu:21-40, 127-129: vertices float [V, 3], triangles integer
// [F, 3] (host arrays; any numeric dtype is cast, as pybind's Eigen
// conversion does for the reference)
cuBVH* create_cuBVH(py::array_t<float, py::array::c_style | py::array::forcecast> vertices,
                    py::array_t<int64_t, py::array::c_style | py::array::forcecast> triangles) {
    TORCH_CHECK(vertices.ndim() == 2 && vertices.shape(1) == 3, "vertices must be [V, 3]");
    TORCH_CHECK(triangles.ndim() == 2 && triangles.shape(1) == 3, "triangles must be [F, 3]");
    cubvh_bvh* h = nullptr;
    check(cubvh_bvh_create(vertices.data(), vertices.shape(0), triangles.data(), triangles.shape(0), &h),
          "create_cuBVH");
    return new cuBVH(h);
}

// src/api_gpu.cu:47-68, 131-133
cuBVH* from_state_dict(const std::unordered_map<std::string, at::Tensor>& sd) {
    auto ver = sd.find("version");
    if (ver != sd.end()) {
        const at::Tensor& v = ver->second;
        TORCH_CHECK(v.numel() == 1 && !v.is_floating_point() && v.item<int64_t>() == kStateDictVersion,
                    "state_dict format version is not supported (this library reads version ", kStateDictVersion,
                    " and unversioned reference dicts)");
    }
    auto tri = sd.find("triangles");
    if (tri == sd.end()) throw std::runtime_error("state_dict missing 'triangles' tensor");
    auto nod = sd.find("nodes");
    if (nod == sd.end()) throw std::runtime_error("State dict does not contain 'nodes'");
    TORCH_CHECK(tri->second.is_cpu(), "triangles must be on CPU");
    TORCH_CHECK(nod->second.is_cpu(), "nodes must be on CPU");
    const at::Tensor tris = tri->second.contiguous(), nodes = nod->second.contiguous();
    TORCH_CHECK(tris.scalar_type() == at::kInt && tris.dim() == 2 && tris.size(1) == 12,
                "triangles must be an int32 [F, 12] tensor of triangle records");
    TORCH_CHECK(nodes.scalar_type() == at::kInt && nodes.dim() == 2 && nodes.size(1) == 9 && nodes.size(0) > 0,
                "nodes must be an int32 [n, 9] tensor of node records");
    cubvh_bvh* h = nullptr;
    check(cubvh_bvh_create_from_state_dict(nodes.data_ptr<int32_t>(), nodes.size(0), tris.data_ptr<int32_t>(),
                                           tris.size(0), &h),
          "from_state_dict");
    return new cuBVH(h);
}

// src/api_gpu.cu:136-152: bool [B, H, W, D] -> int32 labels, returned when done
at::Tensor floodfill(at::Tensor grid) {
    TORCH_CHECK(grid.is_cuda(), "floodfill expects a CUDA grid");
    TORCH_CHECK(grid.scalar_type() == at::kBool, "floodfill expects a bool grid, got ", grid.scalar_type());
    TORCH_CHECK(grid.dim() == 4, "floodfill expects [B, H, W, D]");
    grid = grid.contiguous();
    const c10::cuda::CUDAGuard guard(grid.device());
    const int B = (int)grid.size(0), H = (int)grid.size(1), W = (int)grid.size(2), D = (int)grid.size(3);
    at::Tensor labels = at::empty(grid.sizes(), grid.options().dtype(at::kInt));
    size_t nbytes = 0;
    check(cubvh_floodfill_workspace_size(B, H, W, D, &nbytes), "floodfill");
    at::Tensor ws = at::empty({(int64_t)std::max<size_t>(nbytes, 1)}, grid.options().dtype(at::kByte));
    void* s = stream_of(grid);
    check(cubvh_floodfill(reinterpret_cast<const uint8_t*>(grid.data_ptr<bool>()), B, H, W, D,
                          labels.data_ptr<int32_t>(), ws.data_ptr(), nbytes, s),
          "floodfill");
    check(cubvh_floodfill_check(ws.data_ptr(), B, H, W, D, s), "floodfill");
    return labels;
}

// src/api_gpu.cu:154-215: coords int32 [N, 3], corners float [N, 8] (CUDA)
std::tuple<at::Tensor, at::Tensor> sparse_marching_cubes(at::Tensor coords, at::Tensor corners, double iso,
                                                         bool ensure_consistency) {
    TORCH_CHECK(coords.is_cuda() && corners.is_cuda(), "sparse_marching_cubes expects CUDA tensors");
    coords = coords.to(at::kInt).contiguous();
    corners = corners.to(at::kFloat).contiguous();
    TORCH_CHECK(coords.dim() == 2 && coords.size(1) == 3 && corners.dim() == 2 && corners.size(1) == 8 &&
                    coords.size(0) == corners.size(0),
                "sparse_marching_cubes expects coords [N, 3] and corners [N, 8]");
    same_device(coords, corners, "corners");
    const c10::cuda::CUDAGuard guard(coords.device());
    void* s = stream_of(coords);
    cubvh_smc* res = nullptr;
    int64_t nv = 0, nt = 0;
    check(cubvh_sparse_marching_cubes(coords.data_ptr<int32_t>(), corners.data_ptr<float>(), coords.size(0),
                                      (float)iso, ensure_consistency ? 1 : 0, s, &res, &nv, &nt),
          "sparse_marching_cubes");
    at::Tensor verts = at::empty({nv, 3}, corners.options());
    at::Tensor tris = at::empty({nt, 3}, coords.options());
    const int rc = cubvh_sparse_mc_fetch(res, verts.data_ptr<float>(), tris.data_ptr<int32_t>(), s);
    cubvh_sparse_mc_free(res);
    check(rc, "sparse_marching_cubes");
    return {verts, tris};
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.doc() = "cubvh drop-in extension over the cubvh_b200 C ABI";
    py::class_<cuBVH>(m, "cuBVH")
        .def("ray_trace", &cuBVH::ray_trace)
        .def("unsigned_distance", &cuBVH::unsigned_distance)
        .def("signed_distance", &cuBVH::signed_distance)
        .def("state_dict", &cuBVH::state_dict);
    m.def("create_cuBVH", &create_cuBVH);
    m.def("from_state_dict", &from_state_dict);
    m.def("floodfill", &floodfill);
    m.def("sparse_marching_cubes", &sparse_marching_cubes, py::arg("coords"), py::arg("corners"), py::arg("iso"),
          py::arg("ensure_consistency") = false);
}
