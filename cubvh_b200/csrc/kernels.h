// Kernel launchers shared by the C-ABI layer (abi.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "layout.h"

namespace cubvh {

cudaError_t upload_constants();
// upload_constants() once per device (the current one must be `device`):
// every entry point that launches query kernels on a device calls it first.
cudaError_t ensure_constants(int device);
// The library's stream-ordered memory pool on the current device (created on
// first use; abi.cu), which keeps up to kPoolKeepBytes between calls.
constexpr uint64_t kPoolKeepBytes = 512ull << 20;
cudaError_t library_pool(cudaMemPool_t* out);
// Raystab stab directions of queries first .. first+n-1 into float [n, 32, 3].
cudaError_t launch_stab_dirs(int64_t first, int64_t n, float* dirs, cudaStream_t stream);

// Arena work descriptors (query.cu): a packet is up to 32 consecutive
// positions of the (sorted) query order, all on one mesh.
struct PacketDesc { int64_t start; int32_t count; int32_t mesh; };
struct MeshDesc { int32_t root; int32_t slot0; int64_t qoff; };

// Per-mesh Morton bucketing of an arena's queries: box of the mesh's
// queries, bits per axis, first cell of the mesh in the global histogram.
struct ArenaSortDesc { float lo[3], hi[3]; int32_t bits; int64_t cell_off; };

// Everything one arena launch needs (device pointers unless noted).
struct ArenaLaunch {
    const CNode* nodes; const CTri* tris;
    int32_t n_meshes;
    int64_t n_queries;
    const int64_t* qoff;               // [M + 1] first query of each mesh
    const MeshDesc* meshes;            // [M]
    const ArenaSortDesc* sort;         // [M]
    int64_t n_cells;
    const PacketDesc* packets; int64_t n_packets;        // every query
    const PacketDesc* wt_packets; int64_t n_wt_packets;  // watertight meshes
    const PacketDesc* rs_packets; int64_t n_rs_packets;  // raystab meshes
    unsigned long long* counters;      // 256 bytes
    uint32_t* order; uint32_t* hist; uint32_t* bsum; int32_t* slots;
    uint2* heavy; int64_t heavy_cap;   // heavy-query list (heavy_cap_for(n_queries) entries)
    uint4* rs_cand;                    // raystab second-pass candidates (32 * n_rs_packets entries)
};
cudaError_t launch_arena_distance(const ArenaLaunch& a, const float* pts, float* dist, int64_t* fid, float* uvw,
                                  cudaStream_t stream);
int cell_bits_for(int64_t n);
int64_t heavy_cap_for(int64_t n);

// Point queries at least this many are visited in Morton-cell order.
constexpr int64_t kSortMinQueries = 2048;

// Device scratch bytes of a query launch: launch_distance (mode 0..2) or
// launch_ray (mode -1) for n queries.
size_t query_workspace_bytes(int mode, int64_t n);
// mode 0 unsigned, 1 watertight sign, 2 raystab sign.  ws:
// query_workspace_bytes(mode, n) bytes, 256-byte aligned.
// Watertight candidate lists of a single BVH (root node 0, launch_near_lists):
// for each soup slot t, cnt[t] slots at lst[t * kNear ...] (cnt[t] = -1: more
// than kNear), and nrm[3t .. 3t + 2] the FP64 unit normal of slot t (zero for
// a degenerate triangle); ovf: some slot's list overflowed (those queries take
// a second pass that walks the tree).  cnt nullptr: every query walks.
constexpr int kNear = 32;
struct NearLists {
    const int32_t* cnt = nullptr; const int32_t* lst = nullptr; const double* nrm = nullptr;
    bool ovf = false;
};
// qbase: index of query 0 within the caller's whole call (the raystab stab
// directions follow the query index; a call split into chunks passes each
// chunk's first index).  yield: the distance and watertight sign passes run
// as many short-lived blocks instead of one persistent wave, so kernels of
// higher-priority streams get SMs during them (host-buffer pipelines).
cudaError_t launch_distance(int mode, bool want_uvw, int64_t n, const float* pts, float* dist, int64_t* fid,
                            float* uvw, const CNode* nodes, const CTri* tris, int slot_face0, NearLists near,
                            void* ws, cudaStream_t stream, int64_t qbase = 0, bool yield = false);
// any_ovf: one device int, set to 1 when some list overflowed.
cudaError_t launch_near_lists(int64_t n_tris, const CNode* nodes, const CTri* tris, int32_t* cnt, int32_t* lst,
                              double* nrm, int* any_ovf, cudaStream_t stream);
cudaError_t launch_ray(int64_t n, const float* ro, const float* rd, float* pos, int64_t* fid, float* depth,
                       const CNode* nodes, const CTri* tris, void* ws, cudaStream_t stream);

// refit / backward (grad.cu)
cudaError_t launch_refit(int64_t n_tris, CTri* tris, const int32_t* face_vidx, const float* V, CNode* nodes,
                         float* node_box, const int32_t* level_start, int n_levels, cudaStream_t stream);
size_t backward_workspace_bytes(int64_t n, int64_t nf);
cudaError_t launch_arena_backward(int64_t n, const float* pts, const int64_t* fid, const float* gout,
                                  const float* dist, const int64_t* qoff, int M, const int64_t* face_off,
                                  const int32_t* gslot, const CTri* tris, float* gpts, cudaStream_t stream);
cudaError_t launch_backward(int64_t n, const float* pts, const int64_t* fid, const float* gout, const float* dist,
                            const float* V, const int32_t* fv, const int32_t* fslot, const CTri* tris, int64_t nf,
                            float* gpts, float* gV, void* ws, cudaStream_t stream);

// floodfill (floodfill.cu)
size_t floodfill_workspace_bytes(int B, int H, int W, int D);
cudaError_t launch_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels,
                             void* workspace, cudaStream_t stream);
// Floodfill of the occupancy udf < eps with a signed-distance epilogue
// (same workspace as launch_floodfill).
cudaError_t launch_udf_to_sdf(const float* udf, int B, int H, int W, int D, float eps, float* sdf,
                              void* workspace, cudaStream_t stream);
// Offset of the int32 status word inside the floodfill workspace.
size_t floodfill_status_offset(int B, int H, int W, int D);
// Floodfill with the library's fixed scratch array (floodfill_noalloc.cu).
int floodfill_noalloc(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, cudaStream_t stream,
                      std::string& err);
// CUBVH_OK when a [B, H, W, D] floodfill fits that array, else
// CUBVH_ERR_INVALID with a message.
int floodfill_noalloc_fits(int B, int H, int W, int D, std::string& err);
// Device address of that array on the current device.
int floodfill_noalloc_scratch(void** ws, std::string& err);

// Sparse marching cubes (sparse_mc.cu): device coords int32 [n, 3] and
// corners float32 [n, 8]; the merged vertices float32 [n_verts, 3] and
// triangles int32 [n_tris, 3] are allocated into `out` from the library's
// stream-ordered pool of the current device (released with
// sparse_mc_release once no stream reads them any more).  Returns 0, 1 (bad
// input, err set) or 2 (CUDA error, err set).
struct SparseMCResult {
    float* verts = nullptr;
    int32_t* tris = nullptr;
    int64_t n_verts = 0, n_tris = 0;
};
// closed: this library's own closed triangulation instead of the reference's
// case table (sparse_mc.cu).
int sparse_mc_run(const int32_t* coords, const float* corners, int64_t n, float iso, bool ensure_consistency,
                  bool closed, cudaStream_t stream, SparseMCResult& out, std::string& err);
void sparse_mc_release(SparseMCResult& r);

}  // namespace cubvh
