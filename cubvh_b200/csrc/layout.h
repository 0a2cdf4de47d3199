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
// (a.xyz, original face index), (b.xyz, K * squared longest edge),
// (c.xyz, K), K >= 1 the error factor of the FP32 distance filter
// (tri_error_factor).
// The reference stores 36-byte nodes and 48-byte unaligned triangles
// (include/gpu/bvh.cuh:14-21, include/gpu/triangle.cuh:174-175).
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CUBVH_HD __host__ __device__
#else
#define CUBVH_HD
#endif

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
    float bx, by, bz; float ke2;   // K * squared longest edge (error scale)
    float cx, cy, cz; float k;     // K = tri_error_factor(a, b, c)
};
static_assert(sizeof(CTri) == 48, "triangle must be 48 bytes");

// Double operations rounded once each, on host and device alike (the device
// compiler would otherwise fuse a multiply and an add).
CUBVH_HD inline double mul_rn(double x, double y) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(x, y);
#else
    return x * y;
#endif
}
CUBVH_HD inline double add_rn(double x, double y) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(x, y);
#else
    return x + y;
#endif
}
CUBVH_HD inline double sub_rn(double x, double y) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(x, y);
#else
    return x - y;
#endif
}

// Error factor K of a triangle's FP32 point-triangle filter, whose error
// bound is 8e-6 K (|p-a|^2 + e2), e2 the squared longest edge.  The filter
// takes the distance to the plane from the float normal n = (b-a) x (a-c),
// whose rounding error is below 3 sqrt(2) eps |b-a| |c-a| + eps |n|: relative
// to |n| that is r <= 4.25 eps g + eps, with g = |b-a| |c-a| / |n| one over
// the sine of the angle at a.  The distance to the plane, and the choice of
// face or edges by the edge planes, then carry an error in the squared
// distance below (4 r + 13 eps + (2 r + 4 eps)^2) |p-a|^2 ~ (17 eps (g + 1) +
// (8.5 eps g)^2) |p-a|^2.  K = max(1, 0.3 (1 + g) + 1e-7 g^2): 8e-6 * 0.3 =
// 2.4e-6 covers 17 eps 2.4 times over, 8e-13 covers (8.5 eps)^2 3 times over,
// and past g ~ 2e6, where the float normal may point anywhere, the bound
// exceeds 3 |p-a|^2, more than the error of any value the filter computes
// (each is at most |p-a|^2 (1 + 10 eps)).  K = 1 for g <= 2.33, where the
// plain bound (~134 eps) holds.  A zero or tiny area (|n|^2 < 1e-30: points,
// segments, repeated vertices, edges below ~1e-15) gives K = 1e30, a bound
// that no value of the filter passes, so the triangle is settled in double.
// g is evaluated in double from the float vertices (their differences are
// exact there).
CUBVH_HD inline float tri_error_factor(const float a[3], const float b[3], const float c[3]) {
    double u[3], w[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = sub_rn((double)b[k], (double)a[k]);
        w[k] = sub_rn((double)a[k], (double)c[k]);
    }
    const double n0 = sub_rn(mul_rn(u[1], w[2]), mul_rn(u[2], w[1]));
    const double n1 = sub_rn(mul_rn(u[2], w[0]), mul_rn(u[0], w[2]));
    const double n2 = sub_rn(mul_rn(u[0], w[1]), mul_rn(u[1], w[0]));
    const double nn = add_rn(add_rn(mul_rn(n0, n0), mul_rn(n1, n1)), mul_rn(n2, n2));
    const double uu = add_rn(add_rn(mul_rn(u[0], u[0]), mul_rn(u[1], u[1])), mul_rn(u[2], u[2]));
    const double ww = add_rn(add_rn(mul_rn(w[0], w[0]), mul_rn(w[1], w[1])), mul_rn(w[2], w[2]));
    if (!(nn >= 1e-30)) return 1e30f;
    const double g = std::sqrt(mul_rn(uu, ww) / nn);
    const double K = add_rn(mul_rn(0.3, add_rn(1.0, g)), mul_rn(1e-7, mul_rn(g, g)));
    if (!(K > 1.0)) return 1.0f;
    return K < 1e30 ? (float)K : 1e30f;
}

// Maximum number of internal levels of a tree that the traversal stack of the
// query kernels supports: stack size kStack >= 7 * depth + 1.
constexpr int kStack = 96;
constexpr int kMaxDepth = (kStack - 1) / 7;

}  // namespace cubvh
