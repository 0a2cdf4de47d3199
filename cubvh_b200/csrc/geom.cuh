// Device geometry for the query kernels.
//
// Every reported number (distance, closest point, uvw, ray depth) and every
// hit / miss / sign decision is computed in double with a fixed evaluation
// order through the non-contracting intrinsics (__dadd_rn, __dmul_rn, ...),
// so it is a pure function of the float inputs.  Single-precision versions of
// the same tests run first with an explicit rounding-error bound: they decide
// only the cases whose answer the bound makes certain, everything else falls
// through to the double evaluation ("filtered predicates").
//
// Semantics follow the reference:
//   point-triangle distance   include/gpu/triangle.cuh:46-68 (+ closest point
//                             and barycentric uvw :114-158)
//   ray-triangle hit          include/gpu/triangle.cuh:27-39: hit iff the
//                             barycentrics are inside and 0 <= t < 1000
//                             (src/bvh.cu:17, 254), both faces count
//   watertight sign           src/bvh.cu:356-406
//   raystab sign              src/bvh.cu:408-427 with the per-query pcg32
//                             stream (include/gpu/pcg32.h) and the Fibonacci
//                             stab directions (include/gpu/common.h:63-96)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "layout.h"

namespace cubvh {

// ------------------------------------------------------------------ double
struct d3 { double x, y, z; };
__device__ __forceinline__ double dA(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dS(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dM(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dD(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ d3 dsub(d3 a, d3 b) { return d3{dS(a.x, b.x), dS(a.y, b.y), dS(a.z, b.z)}; }
__device__ __forceinline__ d3 dadd(d3 a, d3 b) { return d3{dA(a.x, b.x), dA(a.y, b.y), dA(a.z, b.z)}; }
__device__ __forceinline__ d3 dscale(d3 a, double s) { return d3{dM(a.x, s), dM(a.y, s), dM(a.z, s)}; }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return dA(dA(dM(a.x, b.x), dM(a.y, b.y)), dM(a.z, b.z)); }
__device__ __forceinline__ d3 dcross(d3 a, d3 b) {
    return d3{dS(dM(a.y, b.z), dM(a.z, b.y)), dS(dM(a.z, b.x), dM(a.x, b.z)), dS(dM(a.x, b.y), dM(a.y, b.x))};
}
__device__ __forceinline__ d3 to_d3(float3 v) { return d3{(double)v.x, (double)v.y, (double)v.z}; }

struct TriV { float3 a, b, c; float ke2, k; int id; };

__device__ __forceinline__ TriV load_tri(const CTri* __restrict__ tris, int slot) {
    const float4* p = reinterpret_cast<const float4*>(tris + slot);
    const float4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2);
    TriV t;
    t.a = make_float3(w0.x, w0.y, w0.z); t.id = __float_as_int(w0.w);
    t.b = make_float3(w1.x, w1.y, w1.z); t.ke2 = w1.w;
    t.c = make_float3(w2.x, w2.y, w2.z); t.k = w2.w;
    return t;
}

__device__ __forceinline__ double seg_closest_d(d3 p, d3 p0, d3 p1, double* s_out) {
    const d3 e = dsub(p1, p0);
    const double ee = ddot(e, e);
    double s = 0.0;
    if (ee > 0.0) {
        s = dD(ddot(dsub(p, p0), e), ee);
        if (s < 0.0) s = 0.0;
        if (s > 1.0) s = 1.0;
    }
    const d3 q = dadd(p0, dscale(e, s));
    const d3 r = dsub(p, q);
    *s_out = s;
    return ddot(r, r);
}

// Closest point on a triangle by Voronoi regions (Ericson, "Real-Time
// Collision Detection", 2005, sec. 5.1.5) with a segment fallback for
// degenerate triangles.  Returns the squared distance.
static __device__ __noinline__ double closest_on_tri_d(d3 p, d3 a, d3 b, d3 c, double bary[3], d3* cp_out) {
    const d3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    double u, v, w;
    d3 cp;
    const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { u = 1.0; v = 0.0; w = 0.0; cp = a; goto done; }
    {
        const d3 bp = dsub(p, b);
        const double d3v = ddot(ab, bp), d4 = ddot(ac, bp);
        if (d3v >= 0.0 && d4 <= d3v) { u = 0.0; v = 1.0; w = 0.0; cp = b; goto done; }
        const double vc = dS(dM(d1, d4), dM(d3v, d2));
        if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) {
            const double t = dD(d1, dS(d1, d3v));
            u = dS(1.0, t); v = t; w = 0.0; cp = dadd(a, dscale(ab, t)); goto done;
        }
        const d3 cpv = dsub(p, c);
        const double d5 = ddot(ab, cpv), d6 = ddot(ac, cpv);
        if (d6 >= 0.0 && d5 <= d6) { u = 0.0; v = 0.0; w = 1.0; cp = c; goto done; }
        const double vb = dS(dM(d5, d2), dM(d1, d6));
        if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
            const double t = dD(d2, dS(d2, d6));
            u = dS(1.0, t); v = 0.0; w = t; cp = dadd(a, dscale(ac, t)); goto done;
        }
        const double va = dS(dM(d3v, d6), dM(d5, d4));
        const double e43 = dS(d4, d3v), e56 = dS(d5, d6);
        if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) {
            const double t = dD(e43, dA(e43, e56));
            u = 0.0; v = dS(1.0, t); w = t; cp = dadd(b, dscale(dsub(c, b), t)); goto done;
        }
        const double denom = dA(dA(va, vb), vc);
        if (denom > 0.0) {
            v = dD(vb, denom); w = dD(vc, denom); u = dS(dS(1.0, v), w);
            cp = dadd(dadd(a, dscale(ab, v)), dscale(ac, w));
            goto done;
        }
        double s0, s1, s2;
        const double q0 = seg_closest_d(p, a, b, &s0);
        const double q1 = seg_closest_d(p, b, c, &s1);
        const double q2 = seg_closest_d(p, c, a, &s2);
        if (q0 <= q1 && q0 <= q2) { u = dS(1.0, s0); v = s0; w = 0.0; cp = dadd(a, dscale(ab, s0)); }
        else if (q1 <= q2) { u = 0.0; v = dS(1.0, s1); w = s1; cp = dadd(b, dscale(dsub(c, b), s1)); }
        else { u = s2; v = 0.0; w = dS(1.0, s2); cp = dadd(c, dscale(dsub(a, c), s2)); }
    }
done:
    bary[0] = u; bary[1] = v; bary[2] = w;
    *cp_out = cp;
    const d3 r = dsub(p, cp);
    return ddot(r, r);
}

// Ray-triangle in double (numerator form): hit iff det != 0, u >= 0, v >= 0,
// u + v <= 1, 0 <= t < tmax.  Writes t = tn / det.
static __device__ __noinline__ bool ray_tri_d(d3 o, d3 d, d3 a, d3 b, d3 c, double tmax, double* t_out) {
    const d3 e1 = dsub(b, a), e2 = dsub(c, a);
    const d3 pv = dcross(d, e2);
    const double det = ddot(e1, pv);
    const d3 s = dsub(o, a);
    const double un = ddot(s, pv);
    const d3 qv = dcross(s, e1);
    const double vn = ddot(d, qv);
    const double tn = ddot(e2, qv);
    double A, U, V, T;
    if (det > 0.0) { A = det; U = un; V = vn; T = tn; }
    else if (det < 0.0) { A = -det; U = -un; V = -vn; T = -tn; }
    else { *t_out = 0.0; return false; }
    *t_out = dD(tn, det);
    return (U >= 0.0) && (V >= 0.0) && (dA(U, V) <= A) && (T >= 0.0) && (T < dM(tmax, A));
}

// -------------------------------------------------------------- float filters
__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 f3cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float f3inf(float3 a) { return fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fabsf(a.z)); }
__device__ __forceinline__ float sgn1(float x) { return copysignf(1.0f, x); }
__device__ __forceinline__ float sat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// Single-precision squared point-triangle distance (edge / face selection of
// Quilez's udTriangle) and an absolute bound on its rounding error:
// 8e-6 * K * (|p-a|^2 + longest edge^2).  With K = 1 it covers ~130 single
// roundings of the local scale, several times what the expression performs
// when the triangle's normal at a is well conditioned; K > 1 widens it for
// the others, degenerate triangles included (layout.h, tri_error_factor).
// The face value's denominator |n|^2 is floored at 1e-36, so a zero normal
// gives a number (at most |p-a|^2) rather than 0 / 0.
__device__ __forceinline__ float tri_d2_f(float3 p, const TriV& t, float* err) {
    const float3 v21 = f3sub(t.b, t.a), p1 = f3sub(p, t.a);
    const float3 v32 = f3sub(t.c, t.b), p2 = f3sub(p, t.b);
    const float3 v13 = f3sub(t.a, t.c), p3 = f3sub(p, t.c);
    const float3 nor = f3cross(v21, v13);
    const float s = sgn1(f3dot(f3cross(v21, nor), p1)) + sgn1(f3dot(f3cross(v32, nor), p2)) +
                    sgn1(f3dot(f3cross(v13, nor), p3));
    float d2;
    if (s < 2.0f) {
        const float k1 = sat(__fdividef(f3dot(v21, p1), f3dot(v21, v21)));
        const float k2 = sat(__fdividef(f3dot(v32, p2), f3dot(v32, v32)));
        const float k3 = sat(__fdividef(f3dot(v13, p3), f3dot(v13, v13)));
        const float3 q1 = make_float3(v21.x * k1 - p1.x, v21.y * k1 - p1.y, v21.z * k1 - p1.z);
        const float3 q2 = make_float3(v32.x * k2 - p2.x, v32.y * k2 - p2.y, v32.z * k2 - p2.z);
        const float3 q3 = make_float3(v13.x * k3 - p3.x, v13.y * k3 - p3.y, v13.z * k3 - p3.z);
        d2 = fminf(fminf(f3dot(q1, q1), f3dot(q2, q2)), f3dot(q3, q3));
    } else {
        const float nd = f3dot(nor, p1);
        d2 = __fdividef(nd * nd, fmaxf(f3dot(nor, nor), 1e-36f));
    }
    *err = 8e-6f * fmaf(t.k, f3dot(p1, p1), t.ke2);
    return d2;
}

// Single-precision ray-triangle classification: 1 = certainly a hit with
// 0 <= t < tmax, 0 = certainly not, -1 = undecided (use ray_tri_d).
// On 1 / -1 writes t (float) and an absolute bound of its error.
// Bounds: each numerator is a triple product of three vectors whose inputs
// carry one rounding each; its computed error is below 42 eps times the
// product of the operands' max-norms, and 8e-6 > 130 eps.
__device__ __forceinline__ int ray_tri_f(float3 o, float3 d, float dinf, const TriV& t, float tmax,
                                         float* t_out, float* terr) {
    const float3 e1 = f3sub(t.b, t.a), e2 = f3sub(t.c, t.a), s = f3sub(o, t.a);
    const float3 pv = f3cross(d, e2);
    const float det = f3dot(e1, pv);
    const float un = f3dot(s, pv);
    const float3 qv = f3cross(s, e1);
    const float vn = f3dot(d, qv);
    const float tn = f3dot(e2, qv);
    const float E = fmaxf(f3inf(e1), f3inf(e2)), S = f3inf(s);
    const float c = 8e-6f;
    const float Bdet = c * dinf * E * E;
    const float Bsd = c * S * dinf * E;
    const float Bt = c * S * E * E;
    const float A = fabsf(det);
    if (!(A > Bdet)) { *t_out = 0.f; *terr = INFINITY; return -1; }
    const float sg = det > 0.f ? 1.f : -1.f;
    const float U = sg * un, V = sg * vn, T = sg * tn;
    const float W = A - U - V;
    const float Bw = Bdet + 2.f * Bsd + 1e-6f * (A + fabsf(U) + fabsf(V));
    const float lim = tmax * A;
    const float Blim = tmax * Bdet + Bt + 1e-6f * lim;
    if (U < -Bsd || V < -Bsd || W < -Bw || T < -Bt || T > lim + Blim) return 0;
    const float tt = __fdividef(T, A);
    *t_out = tt;
    *terr = (Bt + fabsf(tt) * Bdet) / (A - Bdet) + 1e-6f * fabsf(tt);
    if (U > Bsd && V > Bsd && W > Bw && T > Bt && T < lim - Blim) return 1;
    return -1;
}

// Quantised child box decode: origin + q * 2^e (exact product, one rounding).
__device__ __forceinline__ float qf(uint32_t word, int byte) {
    return (float)((word >> (8 * byte)) & 0xFFu);
}
__device__ __forceinline__ float exp2i(int e) { return __int_as_float((e + 127) << 23); }

// ------------------------------------------------------------ stab directions
// Lattice terms of direction k: (k + 1.33) / (31 + 2 * 1.33) at [k] and
// k / golden ratio at [32 + k], float IEEE divisions done by the host (the
// same values as computing them here); read per lane through L1.
static __device__ float g_lattice[64];

// pcg32 with the default state and stream, advanced by 2*i; two next_float
// draws give the query's lattice offset.
__device__ __forceinline__ uint32_t pcg_next(uint64_t& state, uint64_t inc) {
    const uint64_t old = state;
    state = old * 0x5851f42d4c957f2dULL + inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
}
__device__ __forceinline__ float2 stab_offset(uint32_t i) {
    const uint64_t inc = 0xda3e39cb94b95bdbULL;
    uint64_t state = 0x853c49e6748fea9bULL;
    uint64_t cur_mult = 0x5851f42d4c957f2dULL, cur_plus = inc, acc_mult = 1u, acc_plus = 0u;
    uint64_t delta = (uint64_t)(uint32_t)(i * 2u);
    while (delta > 0) {
        if (delta & 1) { acc_mult *= cur_mult; acc_plus = acc_plus * cur_mult + cur_plus; }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1;
    }
    state = acc_mult * state + acc_plus;
    const uint32_t u0 = pcg_next(state, inc), u1 = pcg_next(state, inc);
    return make_float2(__uint_as_float((u0 >> 9) | 0x3f800000u) - 1.0f,
                       __uint_as_float((u1 >> 9) | 0x3f800000u) - 1.0f);
}
// Direction k of the 32-ray Fibonacci lattice (epsilon 1.33) with offset:
// the reference's device arithmetic (include/gpu/common.h:63-96 compiled by
// nvcc with its default contraction): cos(theta) = 1 - 2a, phi = 2 pi (b -
// 0.5), sin(theta) = sqrt(max(fma(-cos, cos, 1), 0)), CUDA's sincosf for
// phi, each product rounded on its own.  The directions equal the
// reference's CUDA build bit for bit (tested against it).
__device__ __forceinline__ float3 stab_dir(uint32_t k, float2 off) {
    float a = __fadd_rn(__ldg(&g_lattice[k]), off.x);
    a = __fsub_rn(a, floorf(a));
    float b = __fadd_rn(__ldg(&g_lattice[32 + k]), off.y);
    b = __fsub_rn(b, floorf(b));
    const float cos_t = __fmaf_rn(-2.0f, a, 1.0f);  // -2a is exact: the same as a product and a sum
    const float phi = __fmul_rn(__fmul_rn(2.0f, 3.14159265358979323846f), __fsub_rn(b, 0.5f));
    const float sin_t = __fsqrt_rn(fmaxf(__fmaf_rn(-cos_t, cos_t, 1.0f), 0.0f));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return make_float3(__fmul_rn(sin_t, cp), __fmul_rn(sin_t, sp), cos_t);
}

}  // namespace cubvh
