/*
 * cubvh_b200 C ABI: mesh queries (unsigned / signed distance, closest-hit
 * ray tracing) over a BVH, and voxel floodfill, on NVIDIA B200 (sm_100a).
 *
 * Plain C: pointers, sizes, int status codes.  Device pointers are CUDA
 * device (or managed) memory on the current device; `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Query
 * calls are asynchronous with respect to the host, like the reference's
 * (they launch on the given stream and return).  No C++ exception crosses
 * this boundary; on failure a call returns a non-zero status and
 * cubvh_last_error() describes it (per calling thread).
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the ashawkey/cubvh project).
 */
#ifndef CUBVH_B200_H
#define CUBVH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cubvh_status {
    CUBVH_OK = 0,
    CUBVH_ERR_INVALID = 1,      /* bad argument (null pointer, size, mode) */
    CUBVH_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed */
    CUBVH_ERR_DEVICE_BOUND = 3, /* a device-side loop bound was hit */
    CUBVH_ERR_NOMEM = 4         /* host or device allocation failed */
};

typedef struct cubvh_bvh cubvh_bvh;

/* Library version string. */
const char* cubvh_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* cubvh_last_error(void);

/* Number of CUDA kernels this library has launched in the process so far
 * (counted on the host at each launch; replays of a CUDA graph that captured
 * them are not counted).  For measurement; no counterpart in the reference. */
uint64_t cubvh_kernel_launches(void);

/* Build a BVH on the host from an indexed mesh; touches no GPU (the device
 * copy is made by the first query on each device).
 * vertices: float32 [n_vertices, 3] (host); faces: int64 [n_faces, 3] (host),
 * each index in [0, n_vertices).  face_id outputs are face row indices.
 * Replaces cuBVHImpl(vertices, triangles) + TriangleBvh4::build
 * (src/api_gpu.cu:21-44, src/bvh.cu:515-620) behind create_cuBVH
 * (src/bindings.cpp:23). */
int cubvh_bvh_create(const float* vertices, int64_t n_vertices, const int64_t* faces, int64_t n_faces,
                     cubvh_bvh** out);

/* Build the BVH on the current GPU (no counterpart in the reference, which
 * builds on the host only: TriangleBvh4::build, src/bvh.cu:515-620).
 * vertices: device float32 [n_vertices, 3]; faces: device int64
 * [n_faces, 3]; max_leaf in [1, 4] (0 = 4).  A linear BVH (sorted Morton
 * codes, binary radix tree, collapsed to the 8-wide layout of
 * cubvh_bvh_create); query results are identical to those of a host-built
 * BVH.  Synchronous on `stream`; the device copy for the current device is
 * the built one, and a host copy is kept as for cubvh_bvh_create.  Fails
 * with CUBVH_ERR_INVALID on a bad vertex index, a non-finite coordinate or a
 * tree deeper than 13 levels. */
int cubvh_bvh_create_device(const float* vertices, int64_t n_vertices, const int64_t* faces, int64_t n_faces,
                            int32_t max_leaf, void* stream, cubvh_bvh** out);

/* Build a BVH from triangle records in the reference's state_dict format:
 * int32 [n_faces, 12] per record = float a[3], b[3], c[3], 4 pad bytes,
 * int64 face id (host).  The reference's node records are not needed (the
 * BVH is rebuilt).  Replaces cuBVHImpl(state_dict) (src/api_gpu.cu:47-68)
 * behind from_state_dict (src/bindings.cpp:24). */
int cubvh_bvh_create_from_records(const int32_t* tri_records, int64_t n_faces, cubvh_bvh** out);
/* As cubvh_bvh_create_from_records, and the BVH keeps the node records
 * (int32 [n_node_records, 9], host) and triangle records it was loaded from:
 * cubvh_bvh_state_dict then returns exactly those records, as the reference's
 * state_dict does after load_state_dict (include/gpu/bvh.cuh:84-109,
 * src/api_gpu.cu:47-68, 110-121).  The node records are stored, not checked;
 * queries use the BVH rebuilt from the triangles. */
int cubvh_bvh_create_from_state_dict(const int32_t* node_records, int64_t n_node_records,
                                     const int32_t* tri_records, int64_t n_faces, cubvh_bvh** out);

/* Release the BVH and its device copies.  Replaces the pybind-owned
 * delete of cuBVH (src/bindings.cpp:17-21). */
int cubvh_bvh_destroy(cubvh_bvh* bvh);

/* Sizes / shape of the built BVH (host memory only). */
int cubvh_bvh_info(const cubvh_bvh* bvh, int64_t* n_faces, int64_t* n_nodes, int32_t* depth);

/* Reference-format state_dict: number of node records (int32 x 9 each) and
 * triangle records (int32 x 12 each), then the records themselves written to
 * host buffers of those sizes: the records of the reference's own BVH4
 * build (src/bvh.cu:515-620) of this mesh, record for record, or the loaded
 * records for a BVH from cubvh_bvh_create_from_state_dict.  Replaces
 * cuBVH::state_dict (src/api_gpu.cu:110-121, include/gpu/bvh.cuh:84-94). */
int cubvh_bvh_state_dict_sizes(const cubvh_bvh* bvh, int64_t* n_node_records, int64_t* n_tri_records);
int cubvh_bvh_state_dict(const cubvh_bvh* bvh, int32_t* node_records, int32_t* tri_records);

/* Inspection (no counterpart in the reference): host copies of the
 * in-memory layout, nodes as n_nodes * 80 bytes and triangles as
 * n_faces * 48 bytes (see cubvh_b200/csrc/layout.h). */
int cubvh_bvh_layout(const cubvh_bvh* bvh, void* nodes_out, void* tris_out);

/* Copy the BVH to the current device now (otherwise the first query does;
 * the first query on a device is therefore synchronous). */
int cubvh_bvh_upload(cubvh_bvh* bvh);

/* Unsigned distance from each point to the mesh.
 * points float32 [n, 3]; distances float32 [n]; face_id int64 [n];
 * uvw float32 [n, 3] barycentric weights of the closest point on face_id,
 * or NULL.  Points farther than 1000 from every triangle get distance 0 and
 * face 0.  Replaces cuBVH::unsigned_distance (src/api_gpu.cu:83-95,
 * src/bvh.cu:468-488, 687-712). */
int cubvh_unsigned_distance(cubvh_bvh* bvh, const float* points, int64_t n, float* distances, int64_t* face_id,
                            float* uvw, void* stream);

/* Signed distance, inside negative.  mode 0 = 'watertight' (sign of the
 * averaged normal around the closest point), 1 = 'raystab' (negative iff all
 * 64 stab rays of the query hit the mesh).  The raystab rays of point i use
 * the query index i within this call.  Replaces cuBVH::signed_distance
 * (src/api_gpu.cu:97-108, src/bvh.cu:430-466, 631-685). */
int cubvh_signed_distance(cubvh_bvh* bvh, const float* points, int64_t n, uint32_t mode, float* distances,
                          int64_t* face_id, float* uvw, void* stream);

/* Closest hit along each ray with 0 <= t < 1000.
 * rays_o, rays_d float32 [n, 3]; positions float32 [n, 3] = o + t d;
 * face_id int64 [n] (-1 on a miss); depth float32 [n] (1000 on a miss).
 * Rays are traced in groups of nearby rays (groups of rays that are not
 * near one another ray by ray); each ray's result is its own, whatever the
 * order of the rays or how they are split across calls.
 * Replaces cuBVH::ray_trace (src/api_gpu.cu:70-81, src/bvh.cu:490-513,
 * 714-740). */
int cubvh_ray_trace(cubvh_bvh* bvh, const float* rays_o, const float* rays_d, int64_t n, float* positions,
                    int64_t* face_id, float* depth, void* stream);

/* Host-buffer variants of the three queries: every pointer except the
 * handle is host memory (page-locked for asynchronous copies), the results
 * are those of cubvh_ray_trace / cubvh_signed_distance on the same inputs,
 * bit for bit.  The queries run in chunks of 2,097,152 whose upload, kernels
 * and download overlap on six internal streams (copy-in, copy-out, one
 * compute stream per staging set), with the priority of `stream`; on
 * return the work is queued behind `stream` and `stream` waits for it:
 * synchronize `stream` before reading the outputs.  Calls on different
 * streams overlap, and the distance kernels of these calls yield SMs to
 * higher-priority streams between short-lived blocks.  The device staging
 * memory (four chunks of inputs, outputs and workspace: ~400 MB for rays)
 * is kept per caller stream until the BVH is destroyed;
 * a call that needs more than its stream's staging synchronizes that
 * staging's earlier work and reallocates it.  A stream being captured into
 * a graph is rejected (status 1).
 * mode as cubvh_signed_distance, or 0xFFFFFFFF for unsigned distance.
 * Replaces the reference's queries called with CPU tensors, which it copies
 * to the GPU whole before tracing (cubvh/api.py:38-65, 67-126); the results
 * stay on the GPU there. */
int cubvh_ray_trace_host(cubvh_bvh* bvh, const float* rays_o, const float* rays_d, int64_t n, float* positions,
                         int64_t* face_id, float* depth, void* stream);
int cubvh_signed_distance_host(cubvh_bvh* bvh, const float* points, int64_t n, uint32_t mode, float* distances,
                               int64_t* face_id, float* uvw, void* stream);

/* Sparse marching cubes.  coords int32 [n, 3] voxel coordinates and
 * corners float32 [n, 8] corner values (corner order (0,0,0), (1,0,0),
 * (1,1,0), (0,1,0), (0,0,1), (1,0,1), (1,1,1), (0,1,1) from the voxel's
 * coordinate), both device memory; iso the level; ensure_consistency holds
 * flags: CUBVH_SMC_ENSURE_CONSISTENCY (1, the reference's boolean) first
 * replaces every corner value by its mean over the voxels sharing the
 * corner; CUBVH_SMC_CLOSED (2) triangulates with this library's own closed
 * triangulation instead of the reference's case table.  Runs on `stream`
 * and waits for it (the output sizes depend on the data); *out receives a result holding *n_verts vertices (float32
 * [n_verts, 3], voxel units) and *n_tris triangles (int32 [n_tris, 3]);
 * cubvh_sparse_mc_fetch copies them into device arrays of those sizes on
 * its own `stream` (any stream: the copies wait for the building stream's
 * last kernels), cubvh_sparse_mc_free releases the result (it waits for this
 * result's build and fetches first, not for other work on the device).  The
 * result's memory, and the call's temporaries, come from the library's
 * stream-ordered pool (it keeps up to 512 MiB per device between calls).  The
 * vertex array equals the reference's (one vertex per cut voxel edge, merged
 * across voxels, sorted by edge), and so does the triangle array, index for
 * index (the reference's marching-cubes case table, voxel by voxel); with
 * CUBVH_SMC_CLOSED the triangles are this library's own (see sparse_mc.cu):
 * a closed, consistently oriented surface where the corner values agree.
 * Replaces sparse_marching_cubes (src/api_gpu.cu:154-215,
 * include/gpu/spcumc.cuh `_sparse_marching_cubes`). */
typedef struct cubvh_smc cubvh_smc;
#define CUBVH_SMC_ENSURE_CONSISTENCY 1
#define CUBVH_SMC_CLOSED 2
int cubvh_sparse_marching_cubes(const int32_t* coords, const float* corners, int64_t n, float iso,
                                int ensure_consistency, void* stream, cubvh_smc** out, int64_t* n_verts,
                                int64_t* n_tris);
int cubvh_sparse_mc_fetch(cubvh_smc* result, float* verts, int32_t* tris, void* stream);
int cubvh_sparse_mc_free(cubvh_smc* result);

/* Differentiable queries (no counterpart in the reference, whose cuBVH
 * detaches the vertices: cubvh/api.py:16-17).
 *
 * cubvh_bvh_refit: move the BVH's vertices to `vertices` (device float32
 * [n_vertices, 3], same count and faces as at creation) and refit the device
 * copy on the current device: same tree, boxes recomputed bottom-up.  Needs a
 * BVH created with cubvh_bvh_create.  The host copy (state_dict) keeps the
 * creation-time geometry.
 *
 * cubvh_distance_backward: gradients of unsigned or signed distances.  For
 * query i with face face_id[i], closest point c (recomputed in double on the
 * current geometry: `vertices` if given, else the BVH's own triangles) and
 * sign s of distances[i]:
 *   grad_points[i]     = grad_distances[i] * s * (p - c) / |p - c|
 *   grad_vertices[v_k] += -lambda_k * grad_distances[i] * s * (p - c) / |p - c|
 * (lambda = barycentric weights of c).  grad_points (float32 [n, 3]) is
 * overwritten; grad_vertices (float32 [n_vertices, 3], needs `vertices` and
 * a BVH created from a mesh) is accumulated into.  Either may be NULL.
 * Queries with distance 0 contribute nothing. */
int cubvh_bvh_refit(cubvh_bvh* bvh, const float* vertices, int64_t n_vertices, void* stream);
int cubvh_distance_backward(cubvh_bvh* bvh, const float* points, int64_t n, const int64_t* face_id,
                            const float* grad_distances, const float* distances, const float* vertices,
                            float* grad_points, float* grad_vertices, void* stream);

/* Batched queries over many meshes in one launch (no counterpart in the
 * reference, which serves one mesh per cuBVH object and one launch per call).
 *
 * cubvh_arena_create: build every mesh (host, in parallel) into one arena;
 * vertices[m] float32 [n_vertices[m], 3], faces[m] int64 [n_faces[m], 3]
 * (host); max_leaf[m] in [1, 4] (NULL = 4) is the leaf size of mesh m.
 * cubvh_arena_set_queries: fix the query layout: the queries of mesh m are
 * rows [query_offsets[m], query_offsets[m + 1]) of one points array (host
 * int64 [M + 1]); modes[m] (host uint32 [M]) is 0 unsigned, 1 watertight,
 * 2 raystab (stab streams use the query's index within its mesh).  Uploads
 * the layout and sizes its workspace (synchronous; call before capture).
 * cubvh_arena_distance: all queries of all meshes; face_id is the face index
 * within the query's mesh; uvw may be NULL.  Only stream-ordered work: can be
 * captured in a CUDA graph; calls on one arena must not overlap on the GPU.
 * cubvh_arena_backward: gradients w.r.t. the query points (as
 * cubvh_distance_backward; grad_points overwritten). */
typedef struct cubvh_arena cubvh_arena;
int cubvh_arena_create(int32_t n_meshes, const float* const* vertices, const int64_t* n_vertices,
                       const int64_t* const* faces, const int64_t* n_faces, const int32_t* max_leaf,
                       cubvh_arena** out);
/* cubvh_arena_create_device: the same arena built on the current GPU in one
 * pass for all meshes (linear BVHs in the same layout; query results are
 * identical).  Same host arguments as cubvh_arena_create; synchronous on
 * `stream`; the arena lives on the current device. */
int cubvh_arena_create_device(int32_t n_meshes, const float* const* vertices, const int64_t* n_vertices,
                              const int64_t* const* faces, const int64_t* n_faces, const int32_t* max_leaf,
                              void* stream, cubvh_arena** out);
int cubvh_arena_destroy(cubvh_arena* arena);
int cubvh_arena_info(const cubvh_arena* arena, int32_t* n_meshes, int64_t* n_faces, int64_t* n_nodes);
int cubvh_arena_set_queries(cubvh_arena* arena, const int64_t* query_offsets, const uint32_t* modes);
int cubvh_arena_distance(cubvh_arena* arena, const float* points, float* distances, int64_t* face_id, float* uvw,
                         void* stream);
int cubvh_arena_backward(cubvh_arena* arena, const float* points, const int64_t* face_id,
                         const float* grad_distances, const float* distances, float* grad_points, void* stream);

/* Stab directions of the raystab sign (inspection; no entry point of the
 * reference exposes them): for queries first .. first+n-1 of a call, float32
 * [n, 32, 3] unit vectors d_k written to device memory `dirs` on `stream`;
 * query i casts -d_k and +d_k for k = 0..31.  They are the reference's
 * device directions bit for bit: pcg32 advanced by 2i, two next_float draws
 * as the lattice offset, fibonacci_dir<32> with CUDA's sincosf
 * (src/bvh.cu:408-427, 658-685; include/gpu/common.h:63-96). */
int cubvh_stab_directions(int64_t first, int64_t n, float* dirs, void* stream);

/* Floodfill of a batch of boolean grids: grid uint8/bool [B, H, W, D]
 * (nonzero = occupied), labels int32 [B, H, W, D]: -1 for occupied voxels,
 * else the smallest global linear index of the voxel's 6-connected free
 * component (neighbourhood as the reference: the memory of each volume read
 * as C-order [D][H][W]).  B*H*W*D must be below 2^31.
 * Scratch: pass `workspace` of at least cubvh_floodfill_workspace_size()
 * bytes (device memory, 256-byte aligned), or NULL to let the call take it
 * from the library's stream-ordered pool.  Asynchronous; when a
 * workspace is passed, cubvh_floodfill_check() reports device-side bound
 * hits of the last call that used it.
 * Replaces floodfill (src/api_gpu.cu:136-152, include/gpu/floodfill.cuh:157-272). */
int cubvh_floodfill_workspace_size(int B, int H, int W, int D, size_t* bytes);
int cubvh_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* workspace,
                    size_t workspace_bytes, void* stream);
/* Synchronises `stream` and returns CUBVH_ERR_DEVICE_BOUND if the floodfill
 * that last used `workspace` (same B, H, W, D) hit a device-side bound.
 * workspace NULL: the fixed array of cubvh_floodfill_noalloc, i.e. the last
 * no-allocation floodfill (same B, H, W, D). */
int cubvh_floodfill_check(const void* workspace, int B, int H, int W, int D, void* stream);

/* Signed distance grid from an unsigned one, fused into the floodfill (the
 * occupancy -> SDF step of the reference's watertight recipe,
 * test/benchmark_watertight.py:89-143 and readme.md:95-102, which the
 * reference does in torch around floodfill).  udf float32 [B, H, W, D]
 * (device); sdf float32 of the same shape (may not alias udf).  For each
 * volume b: occupied = udf < eps; labels = floodfill(occupied);
 * s = udf - eps (float32); sdf = -s where the voxel's label (-1 when
 * occupied) differs from the label of voxel (b, 0, 0, 0) and s > 0, else s.
 * Workspace, asynchrony and cubvh_floodfill_check as cubvh_floodfill (same
 * size: cubvh_floodfill_workspace_size). */
int cubvh_udf_to_sdf(const float* udf, int B, int H, int W, int D, float eps, float* sdf, void* workspace,
                     size_t workspace_bytes, void* stream);

/* Floodfill for callers that must not allocate GPU memory during the call
 * (code running inside another framework's memory pool or arena that forbids
 * cudaMalloc / cudaFree, or loops that must never touch the allocator).  No
 * counterpart in the reference.  Same arguments and results as
 * cubvh_floodfill, but the scratch is a 32 MiB array compiled into the
 * library, so no workspace is passed and nothing is allocated: grids whose
 * scratch (cubvh_floodfill_workspace_size) exceeds 32 MiB, about 192^3
 * voxels, are rejected with CUBVH_ERR_INVALID.  Every GPU that loads this
 * part of the library keeps the 32 MiB until the process exits.  The first
 * call on each device looks up the array's device address (with that device
 * current); make that first call before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (different streams, or
 * different host threads without ordering) race and corrupt each other's
 * results, so order them.  The call clears everything it reads, so no state
 * carries over between calls.  cubvh_floodfill_check(NULL, B, H, W, D,
 * stream) reports a device-side bound hit of the last call.  The array's
 * address is looked up once per device, so calls must not span a
 * cudaDeviceReset of that device. */
int cubvh_floodfill_noalloc(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUBVH_B200_H */
