// TEST INFRASTRUCTURE ONLY.  Compiles the reference's own CUDA sparse
// marching cubes (ashawkey/cubvh include/gpu/spcumc.cuh,
// `_sparse_marching_cubes`; its Python entry is cubvh/api.py:173-187 through
// src/api_gpu.cu:154-215) from the reference tree where it lies
// (oracle/Makefile, target `ref`) into oracle/_ref/libref_sparse_mc.so.  The
// tests compare the sparse marching cubes of cubvh_b200 with it.  The
// cubvh_b200 package never loads it.
//
// The wrapper takes host arrays, copies them to the device, runs the
// reference's function on the default stream and returns its vertex and
// triangle arrays in malloc'd host buffers (ref_sparse_mc_free releases them).
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "gpu/spcumc.cuh"  // found through -I<reference>/include

extern "C" int ref_sparse_mc(const int32_t* coords, const float* corners, int n, float iso, int ensure_consistency,
                             float** verts, int* n_verts, int32_t** tris, int* n_tris) {
    *verts = nullptr; *tris = nullptr; *n_verts = 0; *n_tris = 0;
    if (n <= 0) return 0;
    int* d_coords = nullptr;
    float* d_corners = nullptr;
    if (cudaMalloc(&d_coords, sizeof(int) * 3 * (size_t)n) != cudaSuccess ||
        cudaMalloc(&d_corners, sizeof(float) * 8 * (size_t)n) != cudaSuccess) return 2;
    cudaMemcpy(d_coords, coords, sizeof(int) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_corners, corners, sizeof(float) * 8 * (size_t)n, cudaMemcpyHostToDevice);
    int rc = 0;
    {
        auto mesh = _sparse_marching_cubes(d_coords, d_corners, n, iso, ensure_consistency != 0, 0);
        const size_t m = mesh.first.size(), t = mesh.second.size();
        *verts = static_cast<float*>(malloc(sizeof(float) * 3 * (m ? m : 1)));
        *tris = static_cast<int32_t*>(malloc(sizeof(int32_t) * 3 * (t ? t : 1)));
        if (m) cudaMemcpy(*verts, thrust::raw_pointer_cast(mesh.first.data()), sizeof(float) * 3 * m,
                          cudaMemcpyDeviceToHost);
        if (t) cudaMemcpy(*tris, thrust::raw_pointer_cast(mesh.second.data()), sizeof(int32_t) * 3 * t,
                          cudaMemcpyDeviceToHost);
        *n_verts = (int)m;
        *n_tris = (int)t;
        if (cudaDeviceSynchronize() != cudaSuccess) rc = 2;
    }
    cudaFree(d_coords);
    cudaFree(d_corners);
    return rc;
}

extern "C" void ref_sparse_mc_free(void* p) { free(p); }
