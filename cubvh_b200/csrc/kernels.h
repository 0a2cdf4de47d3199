// Kernel launchers shared by the C-ABI layer (abi.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "layout.h"

namespace cubvh {

cudaError_t upload_constants();

// Point queries at least this many are visited in Morton-cell order.
constexpr int64_t kSortMinQueries = 2048;

// Device scratch bytes of a query launch: launch_distance (mode 0..2) or
// launch_ray (mode -1) for n queries.
size_t query_workspace_bytes(int mode, int64_t n);
// mode 0 unsigned, 1 watertight sign, 2 raystab sign.  ws:
// query_workspace_bytes(mode, n) bytes, 256-byte aligned.
cudaError_t launch_distance(int mode, bool want_uvw, int64_t n, const float* pts, float* dist, int64_t* fid,
                            float* uvw, const CNode* nodes, const CTri* tris, int slot_face0, void* ws,
                            cudaStream_t stream);
cudaError_t launch_ray(int64_t n, const float* ro, const float* rd, float* pos, int64_t* fid, float* depth,
                       const CNode* nodes, const CTri* tris, void* ws, cudaStream_t stream);

// refit / backward (grad.cu)
cudaError_t launch_refit(int64_t n_tris, CTri* tris, const int32_t* face_vidx, const float* V, CNode* nodes,
                         float* node_box, const int32_t* level_start, int n_levels, cudaStream_t stream);
size_t backward_workspace_bytes(int64_t n, int64_t nf);
cudaError_t launch_backward(int64_t n, const float* pts, const int64_t* fid, const float* gout, const float* dist,
                            const float* V, const int32_t* fv, const int32_t* fslot, const CTri* tris, int64_t nf,
                            float* gpts, float* gV, void* ws, cudaStream_t stream);

// floodfill (floodfill.cu)
size_t floodfill_workspace_bytes(int B, int H, int W, int D);
cudaError_t launch_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels,
                             void* workspace, cudaStream_t stream);
// Offset of the int32 status word inside the floodfill workspace.
size_t floodfill_status_offset(int B, int H, int W, int D);
// Floodfill with the library's fixed scratch array (floodfill_noalloc.cu).
int floodfill_noalloc(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, cudaStream_t stream,
                      std::string& err);

}  // namespace cubvh
