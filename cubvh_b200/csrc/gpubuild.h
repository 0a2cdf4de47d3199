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
    int64_t slot_of_face0 = 0;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// v: device float [nv, 3]; f: device int64 [nf, 3].  Synchronous on stream s.
// Returns 0, 1 (invalid mesh: bad index, non-finite coordinate, too deep)
// or 2 (CUDA failure); err describes a failure.
int build_bvh_device(const float* v, int64_t nv, const int64_t* f, int64_t nf, int max_leaf, cudaStream_t s,
                     DeviceBuild& out, std::string& err);

}  // namespace cubvh
