// BVH construction on the GPU (gpubuild.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "layout.h"

namespace cubvh {

// A BVH built on the current device, in the host builder's layout.
struct DeviceBuild {
    CNode* nodes = nullptr;        // device, n_nodes; the caller frees (cudaFree)
    CTri* tris = nullptr;          // device, one per face
    int64_t n_nodes = 0;
    int depth = 0;                 // internal levels (root = 1)
    std::vector<int32_t> level_start;  // breadth-first level ranges, as HostBvh
    int64_t slot_of_face0 = 0;     // of mesh 0
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // box of mesh 0
    // many meshes: mesh m's root is node m (level 0 holds the roots)
    std::vector<int32_t> slot0;    // soup slot of each mesh's face 0
    std::vector<float> mesh_box;   // [M][6] lo, hi
    int32_t* gslot = nullptr;      // device [total faces]: soup slot of each (mesh, face) (on request)
};

// v: device float [nv, 3]; f: device int64 [nf, 3].  Synchronous on stream s.
// Returns 0, 1 (invalid mesh: bad index, non-finite coordinate, too deep)
// or 2 (CUDA failure); err describes a failure.
int build_bvh_device(const float* v, int64_t nv, const int64_t* f, int64_t nf, int max_leaf, cudaStream_t s,
                     DeviceBuild& out, std::string& err);

// Many meshes in one pass.  v: device float [sum nv, 3]; f: device int64
// [sum nf, 3], vertex indices local to their mesh; voff / foff: host [M + 1]
// vertex / face offsets of the meshes; leaf: host [M] leaf sizes.  Triangle
// ids are face indices within their mesh.  want_gslot: also return the face
// -> soup slot map (out.gslot, device, the caller frees).
int build_meshes_device(const float* v, const int64_t* f, const std::vector<int64_t>& voff,
                        const std::vector<int64_t>& foff, const std::vector<int32_t>& leaf, cudaStream_t s,
                        DeviceBuild& out, std::string& err, bool want_gslot);

}  // namespace cubvh
