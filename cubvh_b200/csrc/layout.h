// In-HBM layout of one BVH (host and device view).
//
// Nodes are 8-wide with child boxes quantised to 8 bits per axis relative to
// the node's origin and a per-axis power-of-two scale (the compressed wide
// node of Ylitie, Karras & Laine, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", HPG 2017).  One node is 80 bytes = five
// 16-byte words, read with five 128-bit loads.  Decoding a child bound is
// origin + q * 2^e: the product is exact, so the decoded box is the same float
// box on host and device, and the builder makes it contain the child exactly.
//
// Triangles are a soup in leaf order, 48 bytes = three 16-byte words each:
// (a.xyz, original face index), (b.xyz, squared longest edge),
// (c.xyz, largest edge-vector component).
// The reference stores 36-byte nodes and 48-byte unaligned triangles
// (include/gpu/bvh.cuh:14-21, include/gpu/triangle.cuh:174-175).
#pragma once
#include <cstdint>

namespace cubvh {

constexpr int kWidth = 8;          // children per node
constexpr int kMaxLeafTris = 4;    // triangles per leaf child
constexpr uint8_t kEmpty = 0xFF;   // meta value of an unused child slot

// meta byte of a child slot:
//   0xFF              empty
//   0x80 | slot       internal child; node index = child_base + slot
//   (cnt-1)<<5 | off  leaf child; triangles [tri_base+off, tri_base+off+cnt)
struct alignas(16) CNode {
    float ox, oy, oz;              // origin (lower corner of the node box)
    int8_t ex, ey, ez;             // per-axis scale exponents
    uint8_t n_internal;            // number of internal children
    int32_t child_base;            // index of the first internal child node
    int32_t tri_base;              // first triangle slot of the leaf children
    uint8_t meta[8];
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(CNode) == 80, "node must be 80 bytes");

struct alignas(16) CTri {
    float ax, ay, az; int32_t id;  // original face index
    float bx, by, bz; float e2;    // squared longest edge (error scale)
    float cx, cy, cz; float einf;  // max(|b-a|_inf, |c-a|_inf) (error scale)
};
static_assert(sizeof(CTri) == 48, "triangle must be 48 bytes");

// Maximum number of internal levels of a tree that the traversal stack of the
// query kernels supports: stack size kStack >= 7 * depth + 1.
constexpr int kStack = 96;
constexpr int kMaxDepth = (kStack - 1) / 7;

}  // namespace cubvh
