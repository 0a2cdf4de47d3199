// CPU oracle for the cubvh query path.  TEST INFRASTRUCTURE ONLY: the product
// (cubvh_b200) never links, loads or calls anything in this file.  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
// checker / the timed CPU reference.
//
// Two independent restatements live here:
//
//  (1) An FP64 brute-force oracle (orc_*64): exact-as-double point-triangle
//      distance / closest point / barycentric uvw, ray-triangle hit and depth,
//      and the reference's two sign rules (watertight normal averaging and
//      raystab ray stabbing), evaluated over ALL faces without any BVH.  Every
//      double expression is written with an explicit evaluation order and the
//      file is compiled with -ffp-contract=off, so the numbers are a pure
//      function of the inputs.
//
//  (2) An FP32 mirror of the reference's own CPU-compilable path (orc_ref_*):
//      the BVH4 median-split build and the stack traversals with the same
//      single-precision formulas (Quilez triangle tests, safe_divide slab test,
//      pcg32 + Fibonacci stab rays).  It supplies the reference's face choice /
//      sign behaviour, the traversal work counters used for the roofline's
//      algorithmic bytes, and it is the CPU baseline timed by bench.py.
//
// Parity pinning: the reference's BVH code cannot be compiled in this image
// (every BVH header includes Eigen; its Eigen submodule is empty and Eigen is
// not installed), and the reference's tests hold no golden vectors for this
// path (they compare with trimesh at runtime).  The FP64 distance / ray / sign
// oracle is pinned by analytic known answers (tests/test_oracle.py) and the
// pcg32 restatement by the published PCG32 known-answer sequence; its parity
// with the reference's own outputs is UNPINNED.  The floodfill IS pinned to
// the reference's own outputs: its CUDA floodfill (include/gpu/floodfill.cuh,
// CUDA runtime only) is compiled from the reference tree into oracle/_ref, and
// orc_floodfill reproduces its labels bit for bit on the 13 grids of
// tests/golden/ref_floodfill.npz (tests/test_ref_floodfill.py).
//
// Reference files followed (paths relative to the cubvh project root):
//   include/gpu/triangle.cuh:27-68, 114-158     triangle tests, closest point, uvw
//   include/gpu/bounding_box.cuh:151-218        slab test, point-box distance
//   include/gpu/common.h:49-106                 sign, clamp, fibonacci_dir, safe_divide
//   include/gpu/pcg32.h:44-170                  pcg32
//   src/bvh.cu:17-18, 42-139, 145-427, 515-620  constants, traversals, BVH4 build
//   include/gpu/floodfill.cuh:14-272            floodfill semantics

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stack>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(__FMA__) || defined(__FP_FAST_FMA)
#error "oracle.cpp must be compiled without FMA contraction (-ffp-contract=off, no -mfma)"
#endif

extern "C" {

// ---------------------------------------------------------------------------
// threads
// ---------------------------------------------------------------------------
static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads() {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// (1) FP64 brute force
// ---------------------------------------------------------------------------
struct D3 { double x, y, z; };
static inline D3 d3(const float* p) { return D3{(double)p[0], (double)p[1], (double)p[2]}; }
static inline D3 sub(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline D3 add(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline D3 scale(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
// dot order: (x*x' + y*y') + z*z'
static inline double dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline D3 cross(D3 a, D3 b) {
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct Tri64 { D3 a, b, c; };
static inline Tri64 tri64(const float* V, const int64_t* F, int64_t f) {
    const int64_t* t = F + 3 * f;
    return Tri64{d3(V + 3 * t[0]), d3(V + 3 * t[1]), d3(V + 3 * t[2])};
}

// Closest point on segment [p0,p1] to p: writes parameter s in [0,1].
static inline double seg_closest(D3 p, D3 p0, D3 p1, double* s_out) {
    D3 e = sub(p1, p0);
    double ee = dot(e, e);
    double s = 0.0;
    if (ee > 0.0) {
        s = dot(sub(p, p0), e) / ee;
        if (s < 0.0) s = 0.0;
        if (s > 1.0) s = 1.0;
    }
    D3 q = add(p0, scale(e, s));
    D3 r = sub(p, q);
    *s_out = s;
    return dot(r, r);
}

// Closest point on triangle (a,b,c) to p: the Voronoi-region method of
// Ericson, "Real-Time Collision Detection" (2005) sec. 5.1.5, with a
// segment fallback for degenerate triangles.  Returns squared distance;
// writes barycentric weights (of a, b, c) and the closest point.
static double closest_on_tri(D3 p, const Tri64& T, double bary[3], D3* cp_out) {
    const D3 a = T.a, b = T.b, c = T.c;
    const D3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    double u, v, w;
    D3 cp;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { u = 1.0; v = 0.0; w = 0.0; cp = a; goto done; }
    {
        const D3 bp = sub(p, b);
        const double d3v = dot(ab, bp), d4 = dot(ac, bp);
        if (d3v >= 0.0 && d4 <= d3v) { u = 0.0; v = 1.0; w = 0.0; cp = b; goto done; }
        const double vc = d1 * d4 - d3v * d2;
        if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) {
            const double t = d1 / (d1 - d3v);
            u = 1.0 - t; v = t; w = 0.0; cp = add(a, scale(ab, t)); goto done;
        }
        const D3 cpv = sub(p, c);
        const double d5 = dot(ab, cpv), d6 = dot(ac, cpv);
        if (d6 >= 0.0 && d5 <= d6) { u = 0.0; v = 0.0; w = 1.0; cp = c; goto done; }
        const double vb = d5 * d2 - d1 * d6;
        if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
            const double t = d2 / (d2 - d6);
            u = 1.0 - t; v = 0.0; w = t; cp = add(a, scale(ac, t)); goto done;
        }
        const double va = d3v * d6 - d5 * d4;
        const double e43 = d4 - d3v, e56 = d5 - d6;
        if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) {
            const double t = e43 / (e43 + e56);
            u = 0.0; v = 1.0 - t; w = t; cp = add(b, scale(sub(c, b), t)); goto done;
        }
        const double denom = (va + vb) + vc;
        if (denom > 0.0) {
            v = vb / denom; w = vc / denom; u = (1.0 - v) - w;
            cp = add(add(a, scale(ab, v)), scale(ac, w));
            goto done;
        }
        // degenerate (collinear / zero-area) triangle: best of the three edges
        double s0, s1, s2;
        const double q0 = seg_closest(p, a, b, &s0);
        const double q1 = seg_closest(p, b, c, &s1);
        const double q2 = seg_closest(p, c, a, &s2);
        if (q0 <= q1 && q0 <= q2) { u = 1.0 - s0; v = s0; w = 0.0; cp = add(a, scale(ab, s0)); }
        else if (q1 <= q2) { u = 0.0; v = 1.0 - s1; w = s1; cp = add(b, scale(sub(c, b), s1)); }
        else { u = s2; v = 0.0; w = 1.0 - s2; cp = add(c, scale(sub(a, c), s2)); }
    }
done:
    bary[0] = u; bary[1] = v; bary[2] = w;
    *cp_out = cp;
    const D3 r = sub(p, cp);
    return dot(r, r);
}

// Brute-force unsigned distance.  dist = sqrt of the minimum squared distance;
// fid = lowest face index among exact (double) minima; n_near = number of faces
// whose distance is within tie_eps of the minimum (>= 1); uvw/cp for fid.
void orc_udf64(const float* V, int64_t nv, const int64_t* F, int64_t nf,
               const float* pts, int64_t n, double tie_eps,
               double* dist, int64_t* fid, double* uvw, double* cp, int32_t* n_near) {
    (void)nv;
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int64_t i = 0; i < n; ++i) {
        const D3 p = d3(pts + 3 * i);
        double best = std::numeric_limits<double>::infinity();
        int64_t bf = -1;
        double bb[3] = {0, 0, 0};
        D3 bcp{0, 0, 0};
        std::vector<double> dd((size_t)nf);
        for (int64_t f = 0; f < nf; ++f) {
            double bary[3]; D3 c;
            const double d2 = closest_on_tri(p, tri64(V, F, f), bary, &c);
            dd[(size_t)f] = d2;
            if (d2 < best) { best = d2; bf = f; bb[0] = bary[0]; bb[1] = bary[1]; bb[2] = bary[2]; bcp = c; }
        }
        double dmin = std::sqrt(best);
        int32_t cnt = 0;
        for (int64_t f = 0; f < nf; ++f)
            if (std::sqrt(dd[(size_t)f]) - dmin <= tie_eps) ++cnt;
        if (!(best <= 1e6)) {
            // nothing within MAX_DIST = 1000 (src/bvh.cu:17-18, 346-350):
            // distance 0 on the first triangle (here: face 0)
            bf = 0; dmin = 0.0; cnt = 1;
            closest_on_tri(p, tri64(V, F, 0), bb, &bcp);
        }
        dist[i] = dmin; fid[i] = bf;
        if (uvw) { uvw[3 * i] = bb[0]; uvw[3 * i + 1] = bb[1]; uvw[3 * i + 2] = bb[2]; }
        if (cp) { cp[3 * i] = bcp.x; cp[3 * i + 1] = bcp.y; cp[3 * i + 2] = bcp.z; }
        if (n_near) n_near[i] = cnt;
    }
}

// Exact distance / uvw from each point to one given face.
void orc_face_dist64(const float* V, const int64_t* F, const float* pts, const int64_t* fids,
                     int64_t n, double* dist, double* uvw) {
#pragma omp parallel for schedule(static) num_threads(orc_get_threads())
    for (int64_t i = 0; i < n; ++i) {
        double bary[3]; D3 c;
        const double d2 = closest_on_tri(d3(pts + 3 * i), tri64(V, F, fids[i]), bary, &c);
        dist[i] = std::sqrt(d2);
        if (uvw) { uvw[3 * i] = bary[0]; uvw[3 * i + 1] = bary[1]; uvw[3 * i + 2] = bary[2]; }
    }
}

// Distance from double points to double triangles (one triangle per point),
// tri: [n, 9]; also the closest point's barycentric weights.  Used for the
// finite-difference pins of the distance gradients.
void orc_tri_dist64d(const double* tri, const double* pts, int64_t n, double* dist, double* bary_out) {
    for (int64_t i = 0; i < n; ++i) {
        const double* t = tri + 9 * i;
        const Tri64 T{D3{t[0], t[1], t[2]}, D3{t[3], t[4], t[5]}, D3{t[6], t[7], t[8]}};
        double bary[3]; D3 c;
        dist[i] = std::sqrt(closest_on_tri(D3{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, T, bary, &c));
        if (bary_out) { bary_out[3 * i] = bary[0]; bary_out[3 * i + 1] = bary[1]; bary_out[3 * i + 2] = bary[2]; }
    }
}

// Ray/triangle in double (Moller-Trumbore arrangement; same predicate as the
// reference's Quilez test without its safe_divide clamp): hit iff det != 0,
// u >= 0, v >= 0, u + v <= 1, 0 <= t < tmax.  Evaluated in numerator space.
// margin_out = min(u, v, 1-u-v) (normalised), graze_out = |cos| of incidence.
struct RayHit { bool hit; double t; double margin; double graze; };
static inline RayHit ray_tri64(D3 o, D3 d, const Tri64& T, double tmax) {
    RayHit r{false, 0.0, -1.0, 0.0};
    const D3 e1 = sub(T.b, T.a), e2 = sub(T.c, T.a);
    const D3 pv = cross(d, e2);
    const double det = dot(e1, pv);
    const D3 s = sub(o, T.a);
    const double un = dot(s, pv);
    const D3 qv = cross(s, e1);
    const double vn = dot(d, qv);
    const double tn = dot(e2, qv);
    double A, U, Vv, Tn;
    if (det > 0.0) { A = det; U = un; Vv = vn; Tn = tn; }
    else if (det < 0.0) { A = -det; U = -un; Vv = -vn; Tn = -tn; }
    else { return r; }
    r.hit = (U >= 0.0) && (Vv >= 0.0) && ((U + Vv) <= A) && (Tn >= 0.0) && (Tn < tmax * A);
    r.t = tn / det;
    const double u = U / A, v = Vv / A;
    r.margin = std::min(std::min(u, v), (1.0 - u) - v);
    const D3 nrm = cross(e1, e2);
    const double nn = std::sqrt(dot(nrm, nrm)) * std::sqrt(dot(d, d));
    r.graze = nn > 0.0 ? A / nn : 0.0;
    return r;
}

// Closest hit.  t/fid = smallest double t among hits (ties -> lowest face);
// depth = tmax and fid = -1 on a miss.  flags bit0: some face has |margin| <
// eps_b or graze < eps_g while being a hit candidate (t in range); bit1: a second
// hit lies within tie_eps of the closest.
void orc_ray64(const float* V, const int64_t* F, int64_t nf, const float* ro, const float* rd,
               int64_t n, double tmax, double eps_b, double eps_g, double tie_eps,
               double* t_out, int64_t* fid_out, int32_t* flags) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int64_t i = 0; i < n; ++i) {
        const D3 o = d3(ro + 3 * i), d = d3(rd + 3 * i);
        double bt = tmax; int64_t bf = -1; int32_t fl = 0;
        std::vector<double> hits;
        for (int64_t f = 0; f < nf; ++f) {
            const RayHit h = ray_tri64(o, d, tri64(V, F, f), tmax);
            const bool in_range = h.t > -eps_b && h.t < tmax * (1.0 + eps_b);
            if (in_range && (std::fabs(h.margin) < eps_b || (h.graze < eps_g && h.margin > -eps_b)))
                fl |= 1;
            if (h.hit) {
                hits.push_back(h.t);
                if (h.t < bt) { bt = h.t; bf = f; }
            }
        }
        int cnt = 0;
        for (double t : hits) if (t - bt <= tie_eps) ++cnt;
        if (cnt > 1) fl |= 2;
        t_out[i] = bt; fid_out[i] = bf; flags[i] = fl;
    }
}

// Any-hit in [0, tmax) over all faces; sets *amb when a face is near the
// classification boundary.
static bool any_hit64(const float* V, const int64_t* F, int64_t nf, D3 o, D3 d, double tmax,
                      double eps_b, double eps_g, bool* amb) {
    bool hit = false;
    for (int64_t f = 0; f < nf; ++f) {
        const RayHit h = ray_tri64(o, d, tri64(V, F, f), tmax);
        const bool in_range = h.t > -eps_b && h.t < tmax * (1.0 + eps_b);
        if (in_range && (std::fabs(h.margin) < eps_b || (h.graze < eps_g && h.margin > -eps_b)))
            *amb = true;
        if (h.hit) hit = true;
    }
    return hit;
}

// Watertight sign rule of the reference (src/bvh.cu:356-406) in double: the
// closest point cp of the nearest face, the sum of unit normals of every face
// with squared distance to cp below 1e-6, and the sign of that sum dotted with
// (p - cp).  flags bit0: |dot| tiny relative to its magnitude or a face sits on
// the 1e-6 membership threshold; bit1: dist == 0.
void orc_sdf_watertight64(const float* V, const int64_t* F, int64_t nf, const float* pts, int64_t n,
                          double* sdist, int64_t* fid_out, int32_t* flags) {
    std::vector<double> dist(n), cp(3 * n);
    std::vector<int64_t> fid(n);
    orc_udf64(V, 0, F, nf, pts, n, 0.0, dist.data(), fid.data(), nullptr, cp.data(), nullptr);
#pragma omp parallel for schedule(dynamic, 16) num_threads(orc_get_threads())
    for (int64_t i = 0; i < n; ++i) {
        const D3 p = d3(pts + 3 * i);
        const D3 c{cp[3 * i], cp[3 * i + 1], cp[3 * i + 2]};
        D3 nsum{0, 0, 0};
        int32_t fl = 0;
        for (int64_t f = 0; f < nf; ++f) {
            double bary[3]; D3 q;
            const Tri64 T = tri64(V, F, f);
            const double d2 = closest_on_tri(c, T, bary, &q);
            if (std::fabs(d2 - 1e-6) <= 1e-12) fl |= 1;
            if (d2 < 1e-6) {
                const D3 nr = cross(sub(T.b, T.a), sub(T.c, T.a));
                const double len = std::sqrt(dot(nr, nr));
                if (len > 0.0) nsum = add(nsum, D3{nr.x / len, nr.y / len, nr.z / len});
            }
        }
        const D3 r = sub(p, c);
        const double dd = dot(nsum, r);
        const double mag = std::sqrt(dot(nsum, nsum)) * std::sqrt(dot(r, r));
        if (std::fabs(dd) <= 1e-12 * mag) fl |= 1;
        if (dist[i] == 0.0) fl |= 2;
        sdist[i] = std::copysign(dist[i], dd);
        if (fid_out) fid_out[i] = fid[i];
        flags[i] = fl;
    }
}

// --- pcg32 (include/gpu/pcg32.h:44-170): default state/stream, advance, next_float
static const uint64_t PCG_STATE = 0x853c49e6748fea9bULL;
static const uint64_t PCG_INC = 0xda3e39cb94b95bdbULL;
static const uint64_t PCG_MULT = 0x5851f42d4c957f2dULL;
struct Pcg { uint64_t state, inc; };
static inline uint32_t pcg_next(Pcg& g) {
    const uint64_t old = g.state;
    g.state = old * PCG_MULT + g.inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
}
static inline void pcg_seed(Pcg& g, uint64_t initstate, uint64_t initseq) {
    g.state = 0u; g.inc = (initseq << 1u) | 1u;
    pcg_next(g); g.state += initstate; pcg_next(g);
}
static inline void pcg_advance(Pcg& g, int64_t delta_) {
    uint64_t cur_mult = PCG_MULT, cur_plus = g.inc, acc_mult = 1u, acc_plus = 0u;
    uint64_t delta = (uint64_t)delta_;
    while (delta > 0) {
        if (delta & 1) { acc_mult *= cur_mult; acc_plus = acc_plus * cur_mult + cur_plus; }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        delta /= 2;
    }
    g.state = acc_mult * g.state + acc_plus;
}
static inline float pcg_next_float(Pcg& g) {
    union { uint32_t u; float f; } x;
    x.u = (pcg_next(g) >> 9) | 0x3f800000u;
    return x.f - 1.0f;
}
// Known-answer hook: seed(initstate, initseq) then n next_uint values.
void orc_pcg32_seq(uint64_t initstate, uint64_t initseq, int n, uint32_t* out) {
    Pcg g; pcg_seed(g, initstate, initseq);
    for (int i = 0; i < n; ++i) out[i] = pcg_next(g);
}
// The reference's per-query stab offset: default generator advanced by 2*i
// (src/bvh.cu:667-668; i is the uint32 query index, 2*i wraps in uint32).
void orc_stab_offsets(int64_t n, int64_t i0, float* out2) {
    for (int64_t k = 0; k < n; ++k) {
        Pcg g{PCG_STATE, PCG_INC};
        const uint32_t i = (uint32_t)(i0 + k);
        pcg_advance(g, (int64_t)(uint32_t)(i * 2u));
        out2[2 * k] = pcg_next_float(g);
        out2[2 * k + 1] = pcg_next_float(g);
    }
}

// fibonacci_dir<32> (include/gpu/common.h:63-96) in the reference's float
// operation order with the host's sin / cos (what the reference's own host
// build computes; its CUDA build calls the device sincosf and contracts
// 1 - cos^2 into a fused multiply-add, so its directions can differ in the
// last bit: the GPU tests pass those directions in as a table).
static inline void stab_dir(uint32_t i, float ox, float oy, float out[3]) {
    const float eps = 1.33f;
    const float den = (float)31u + 2.0f * eps;
    float a = ((float)i + eps) / den + ox;
    a = a - std::floor(a);
    const float GOLDEN = 1.6180339887498948482045868343656f;
    float b = (float)i / GOLDEN + oy;
    b = b - std::floor(b);
    const float PI = 3.14159265358979323846f;
    const float cos_theta = -2.0f * a + 1.0f;
    const float phi = (2.0f * PI) * (b - 0.5f);
    const float sin_theta = std::sqrt(std::max(1.0f - cos_theta * cos_theta, 0.0f));
    const float sp = std::sin(phi), cp = std::cos(phi);
    out[0] = sin_theta * cp; out[1] = sin_theta * sp; out[2] = cos_theta;
}
void orc_stab_dirs(int64_t n, int64_t i0, float* out) {
    for (int64_t k = 0; k < n; ++k) {
        float off[2];
        orc_stab_offsets(1, i0 + k, off);
        for (uint32_t r = 0; r < 32; ++r)
            stab_dir(r, off[0], off[1], out + 3 * (32 * k + r));
    }
}

// Raystab sign rule (src/bvh.cu:408-427) in double: negative iff all 64 rays
// (-d_k then +d_k, k = 0..31) hit within [0, 1000).  i0 = index of the
// first point within its call.  dirs: float [n, 32, 3] stab directions of
// the n points, or NULL for the host rule above (stab_dir).
void orc_sdf_raystab64(const float* V, const int64_t* F, int64_t nf, const float* pts, int64_t n,
                       int64_t i0, double eps_b, double eps_g, const float* dirs,
                       double* sdist, int64_t* fid_out, int32_t* flags) {
    std::vector<double> dist(n);
    std::vector<int64_t> fid(n);
    orc_udf64(V, 0, F, nf, pts, n, 0.0, dist.data(), fid.data(), nullptr, nullptr, nullptr);
#pragma omp parallel for schedule(dynamic, 4) num_threads(orc_get_threads())
    for (int64_t i = 0; i < n; ++i) {
        float off[2];
        orc_stab_offsets(1, i0 + i, off);
        const D3 p = d3(pts + 3 * i);
        bool inside = true, amb = false;
        for (uint32_t k = 0; k < 32 && inside; ++k) {
            float dir[3];
            if (dirs) for (int c = 0; c < 3; ++c) dir[c] = dirs[(32 * i + k) * 3 + c];
            else stab_dir(k, off[0], off[1], dir);
            const float ndir[3] = {-dir[0], -dir[1], -dir[2]};
            if (!any_hit64(V, F, nf, p, d3(ndir), 1000.0, eps_b, eps_g, &amb)) { inside = false; break; }
            if (!any_hit64(V, F, nf, p, d3(dir), 1000.0, eps_b, eps_g, &amb)) { inside = false; break; }
        }
        sdist[i] = inside ? -dist[i] : dist[i];
        if (fid_out) fid_out[i] = fid[i];
        flags[i] = (amb ? 1 : 0) | (dist[i] == 0.0 ? 2 : 0);
    }
}

// ---------------------------------------------------------------------------
// floodfill (include/gpu/floodfill.cuh:14-272): 6-connected components of free
// voxels (grid == 0); label = smallest global linear index in the component,
// -1 for occupied voxels.  The reference decodes a voxel's local index as
// x = l % W, y = (l / W) % H, z = l / (W*H) with neighbour strides 1, W, W*H,
// i.e. it treats each [H, W, D] volume's memory as a C-order [D][H][W] array;
// this oracle follows that exactly (identical to [H][W][D] when H = W = D).
// Union-find with min-index roots; labels doubles as the parent array.
// ---------------------------------------------------------------------------
static inline int32_t uf_find(int32_t* par, int32_t x) {
    while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
    return x;
}
int orc_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels) {
    const int64_t nvol = (int64_t)H * W * D, ntot = nvol * B;
    if (ntot > (int64_t)INT32_MAX) return 1;
    const int64_t sy = W, sz = (int64_t)W * H;
    for (int64_t i = 0; i < ntot; ++i) labels[i] = grid[i] ? -1 : (int32_t)i;
    for (int b = 0; b < B; ++b) {
        const int64_t base = (int64_t)b * nvol;
        for (int64_t l = 0; l < nvol; ++l) {
            const int64_t i = base + l;
            if (grid[i]) continue;
            const int64_t x = l % W, y = (l / W) % H, z = l / sz;
            const int64_t nb[3] = {x > 0 ? i - 1 : -1, y > 0 ? i - sy : -1, z > 0 ? i - sz : -1};
            for (int k = 0; k < 3; ++k) {
                if (nb[k] < 0 || grid[nb[k]]) continue;
                int32_t ra = uf_find(labels, (int32_t)i), rb = uf_find(labels, (int32_t)nb[k]);
                if (ra == rb) continue;
                if (ra < rb) labels[rb] = ra; else labels[ra] = rb;
            }
        }
    }
    for (int64_t i = 0; i < ntot; ++i)
        if (labels[i] >= 0) labels[i] = uf_find(labels, (int32_t)i);
    return 0;
}

// ---------------------------------------------------------------------------
// (2) FP32 mirror of the reference's CPU-compilable path
// ---------------------------------------------------------------------------
struct F3 { float x, y, z; };
static inline F3 f3sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline F3 f3add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline F3 f3mul(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
// Eigen's unrolled 3-term reduction: p0 + (p1 + p2)
static inline float f3dot(F3 a, F3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
static inline float f3sq(F3 a) { return f3dot(a, a); }
static inline F3 f3cross(F3 a, F3 b) {
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float fsign(float x) { return std::copysign(1.0f, x); }
static inline float fclamp(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }
static inline float fminr(float a, float b) { return (b < a) ? b : a; }  // std::min
static inline float safe_divide(float num, float den, float eps = 1e-6f) {
    if (std::fabs(den) < eps) { if (den <= 0) return -(num / eps); else return num / eps; }
    return num / den;
}

struct RTri { F3 a, b, c; int32_t pad; int64_t id; };  // 48 B, the reference's Triangle
static_assert(sizeof(RTri) == 48, "Triangle record must be 48 bytes");
struct RBox { F3 mn, mx; };
struct RNode { RBox bb; int32_t left, right, escape; };  // 36 B, TriangleBvhNode
static_assert(sizeof(RNode) == 36, "node record must be 36 bytes");

static inline F3 rnormal(const RTri& t) {  // (b-a).cross(c-a).normalized()
    F3 n = f3cross(f3sub(t.b, t.a), f3sub(t.c, t.a));
    const float z = f3sq(n);
    if (z > 0.f) { const float s = std::sqrt(z); n = F3{n.x / s, n.y / s, n.z / s}; }
    return n;
}
// triangle.cuh:46-68 (Quilez udTriangle)
static inline float rdist_sq(const RTri& t, F3 pos) {
    const F3 v21 = f3sub(t.b, t.a), p1 = f3sub(pos, t.a);
    const F3 v32 = f3sub(t.c, t.b), p2 = f3sub(pos, t.b);
    const F3 v13 = f3sub(t.a, t.c), p3 = f3sub(pos, t.c);
    const F3 nor = f3cross(v21, v13);
    const float s = fsign(f3dot(f3cross(v21, nor), p1)) + fsign(f3dot(f3cross(v32, nor), p2)) +
                    fsign(f3dot(f3cross(v13, nor), p3));
    if (s < 2.0f) {
        const float e1 = f3sq(f3sub(f3mul(v21, fclamp(f3dot(v21, p1) / f3sq(v21), 0.f, 1.f)), p1));
        const float e2 = f3sq(f3sub(f3mul(v32, fclamp(f3dot(v32, p2) / f3sq(v32), 0.f, 1.f)), p2));
        const float e3 = f3sq(f3sub(f3mul(v13, fclamp(f3dot(v13, p3) / f3sq(v13), 0.f, 1.f)), p3));
        return fminr(fminr(e1, e2), e3);
    }
    const float nd = f3dot(nor, p1);
    return nd * nd / f3sq(nor);
}
// triangle.cuh:27-39 (Quilez intersector, t = 1e6 on a miss)
static inline float rray_tri(const RTri& t, F3 ro, F3 rd) {
    const F3 v1v0 = f3sub(t.b, t.a), v2v0 = f3sub(t.c, t.a), rov0 = f3sub(ro, t.a);
    const F3 n = f3cross(v1v0, v2v0);
    const F3 q = f3cross(rov0, rd);
    const float d = safe_divide(1.0f, f3dot(rd, n));
    const float u = d * -f3dot(q, v2v0);
    const float v = d * f3dot(q, v1v0);
    float tt = d * -f3dot(n, rov0);
    if (u < 0.0f || u > 1.0f || v < 0.0f || (u + v) > 1.0f || tt < 0.0f) tt = 1e6f;
    return tt;
}
// triangle.cuh:74-139 closest_point, :141-158 barycentric
static inline bool rpoint_in_tri(const RTri& t, F3 p) {
    const F3 la = f3sub(t.a, p), lb = f3sub(t.b, p), lc = f3sub(t.c, p);
    const F3 u = f3cross(lb, lc), v = f3cross(lc, la), w = f3cross(la, lb);
    if (f3dot(u, v) < 0.0f) return false;
    if (f3dot(u, w) < 0.0f) return false;
    return true;
}
static inline F3 rclosest_to_line(F3 a, F3 b, F3 c) {
    float tt = f3dot(f3sub(c, a), f3sub(b, a)) / f3dot(f3sub(b, a), f3sub(b, a));
    tt = std::max(std::min(tt, 1.0f), 0.0f);
    return f3add(a, f3mul(f3sub(b, a), tt));
}
static inline F3 rclosest_point(const RTri& t, F3 point) {
    const F3 n = rnormal(t);
    const float k = f3dot(n, f3sub(point, t.a));
    point = f3sub(point, f3mul(n, k));
    if (rpoint_in_tri(t, point)) return point;
    const F3 c1 = rclosest_to_line(t.a, t.b, point);
    const F3 c2 = rclosest_to_line(t.b, t.c, point);
    const F3 c3 = rclosest_to_line(t.c, t.a, point);
    const float m1 = f3sq(f3sub(point, c1)), m2 = f3sq(f3sub(point, c2)), m3 = f3sq(f3sub(point, c3));
    float mn = std::min(m1, m2); mn = std::min(mn, m3);
    if (mn == m1) return c1;
    if (mn == m2) return c2;
    return c3;
}
static inline F3 rbarycentric(const RTri& t, F3 p) {
    const F3 v0 = f3sub(t.b, t.a), v1 = f3sub(t.c, t.a), v2 = f3sub(p, t.a);
    const float d00 = f3dot(v0, v0), d01 = f3dot(v0, v1), d11 = f3dot(v1, v1);
    const float d20 = f3dot(v2, v0), d21 = f3dot(v2, v1);
    const float denom = d00 * d11 - d01 * d01;
    const float v = (d11 * d20 - d01 * d21) / denom;
    const float w = (d00 * d21 - d01 * d20) / denom;
    const float u = (float)(1.0 - (double)v - (double)w);
    return F3{u, v, w};
}
// bounding_box.cuh:151-198, 216-218
static inline float rbox_ray_tmin(const RBox& b, F3 pos, F3 dir) {
    float tmin = safe_divide(b.mn.x - pos.x, dir.x);
    float tmax = safe_divide(b.mx.x - pos.x, dir.x);
    if (tmin > tmax) std::swap(tmin, tmax);
    float tymin = safe_divide(b.mn.y - pos.y, dir.y);
    float tymax = safe_divide(b.mx.y - pos.y, dir.y);
    if (tymin > tymax) std::swap(tymin, tymax);
    if (tmin > tymax || tymin > tmax) return std::numeric_limits<float>::max();
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float tzmin = safe_divide(b.mn.z - pos.z, dir.z);
    float tzmax = safe_divide(b.mx.z - pos.z, dir.z);
    if (tzmin > tzmax) std::swap(tzmin, tzmax);
    if (tmin > tzmax || tzmin > tmax) return std::numeric_limits<float>::max();
    if (tzmin > tmin) tmin = tzmin;
    return tmin;
}
static inline float rbox_dist_sq(const RBox& b, F3 p) {
    const F3 q{std::max(std::max(b.mn.x - p.x, p.x - b.mx.x), 0.0f),
               std::max(std::max(b.mn.y - p.y, p.y - b.mx.y), 0.0f),
               std::max(std::max(b.mn.z - p.z, p.z - b.mx.z), 0.0f)};
    return f3sq(q);
}
static inline float rcentroid(const RTri& t, int axis) {
    const float* a = &t.a.x; const float* b = &t.b.x; const float* c = &t.c.x;
    return (a[axis] + b[axis] + c[axis]) / 3;
}

struct RefBvh {
    std::vector<RTri> tris;
    std::vector<RNode> nodes;
};
static RBox rbox_of(std::vector<RTri>::iterator b, std::vector<RTri>::iterator e) {
    RBox bb{b->a, b->a};
    for (auto it = b; it != e; ++it) {
        for (const F3& v : {it->a, it->b, it->c}) {
            bb.mn = F3{std::min(bb.mn.x, v.x), std::min(bb.mn.y, v.y), std::min(bb.mn.z, v.z)};
            bb.mx = F3{std::max(bb.mx.x, v.x), std::max(bb.mx.y, v.y), std::max(bb.mx.z, v.z)};
        }
    }
    return bb;
}
// src/bvh.cu:515-620: BVH4, two rounds of median split on the axis of largest
// centroid variance, leaf <= n_per_leaf, pre-order escape links.
static void ref_build(RefBvh& B, uint32_t n_per_leaf) {
    auto& T = B.tris; auto& N = B.nodes;
    N.clear(); N.emplace_back();
    N.front().bb = rbox_of(T.begin(), T.end());
    struct BuildNode { int node_idx; std::vector<RTri>::iterator begin, end; };
    std::stack<BuildNode> st;
    st.push({0, T.begin(), T.end()});
    while (!st.empty()) {
        const BuildNode curr = st.top(); st.pop();
        BuildNode ch[4];
        ch[0].begin = curr.begin; ch[0].end = curr.end;
        int nc = 1;
        while (nc < 4) {
            for (int i = nc - 1; i >= 0; --i) {
                BuildNode& c = ch[i];
                const float cnt = (float)std::distance(c.begin, c.end);
                F3 mean{0, 0, 0};
                for (auto it = c.begin; it != c.end; ++it) {
                    const F3 cen{((it->a.x + it->b.x) + it->c.x) / 3.0f,
                                 ((it->a.y + it->b.y) + it->c.y) / 3.0f,
                                 ((it->a.z + it->b.z) + it->c.z) / 3.0f};
                    mean = f3add(mean, cen);
                }
                mean = F3{mean.x / cnt, mean.y / cnt, mean.z / cnt};
                F3 var{0, 0, 0};
                for (auto it = c.begin; it != c.end; ++it) {
                    const F3 cen{((it->a.x + it->b.x) + it->c.x) / 3.0f,
                                 ((it->a.y + it->b.y) + it->c.y) / 3.0f,
                                 ((it->a.z + it->b.z) + it->c.z) / 3.0f};
                    const F3 df = f3sub(cen, mean);
                    var = f3add(var, F3{df.x * df.x, df.y * df.y, df.z * df.z});
                }
                var = F3{var.x / cnt, var.y / cnt, var.z / cnt};
                int axis = 0;
                if (var.y > var.x) axis = 1;
                if (var.z > (axis == 0 ? var.x : var.y)) axis = 2;
                auto m = c.begin + std::distance(c.begin, c.end) / 2;
                std::nth_element(c.begin, m, c.end, [&](const RTri& t1, const RTri& t2) {
                    return rcentroid(t1, axis) < rcentroid(t2, axis);
                });
                ch[i * 2].begin = ch[i].begin;
                ch[i * 2 + 1].end = ch[i].end;
                ch[i * 2].end = ch[i * 2 + 1].begin = m;
            }
            nc *= 2;
        }
        N[curr.node_idx].left = (int)N.size();
        for (int i = 0; i < 4; ++i) {
            BuildNode& c = ch[i];
            c.node_idx = (int)N.size();
            N.emplace_back();
            N.back().bb = rbox_of(c.begin, c.end);
            if ((uint32_t)std::distance(c.begin, c.end) <= n_per_leaf) {
                N.back().left = -(int)std::distance(T.begin(), c.begin) - 1;
                N.back().right = -(int)std::distance(T.begin(), c.end) - 1;
            } else {
                st.push(c);
            }
        }
        N[curr.node_idx].right = (int)N.size();
    }
    for (auto& nd : N) nd.escape = -1;
    // pre-order escape threading (iterative form of the reference's recursion)
    std::vector<std::pair<int, int>> work{{0, -1}};
    while (!work.empty()) {
        auto [ni, esc] = work.back(); work.pop_back();
        N[ni].escape = esc;
        if (N[ni].left < 0) continue;
        const int first = N[ni].left, end = N[ni].right;
        for (int c = end - 1; c >= first; --c) work.push_back({c, (c + 1 < end) ? c + 1 : esc});
    }
}

struct Counters { int64_t box, tri; };

// src/bvh.cu:300-353 closest_triangle (+ stackless fallback :178-213)
static std::pair<int, float> ref_closest_stackless(const RefBvh& B, F3 p, float maxd2, Counters* c) {
    float best = maxd2; int bi = -1; int idx = 0;
    while (idx != -1) {
        const RNode& nd = B.nodes[idx];
        if (c) c->box++;
        if (rbox_dist_sq(nd.bb, p) > best) { idx = nd.escape; continue; }
        if (nd.left < 0) {
            const int end = -nd.right - 1;
            for (int i = -nd.left - 1; i < end; ++i) {
                if (c) c->tri++;
                const float d2 = rdist_sq(B.tris[i], p);
                if (d2 <= best) { best = d2; bi = i; }
            }
            idx = nd.escape;
        } else idx = nd.left;
    }
    if (bi == -1) { bi = 0; best = 0.0f; }
    return {bi, std::sqrt(best)};
}
struct DI { float d; int i; };
static inline void cas(DI& a, DI& b) { if (a.d < b.d) std::swap(a, b); }
static inline void sort4(DI v[4]) { cas(v[0], v[2]); cas(v[1], v[3]); cas(v[0], v[1]); cas(v[2], v[3]); cas(v[1], v[2]); }
static std::pair<int, float> ref_closest(const RefBvh& B, F3 p, float maxd2, Counters* c) {
    int st[32]; int cnt = 0; bool over = false;
    st[cnt++] = 0;
    float best = maxd2; int bi = -1;
    while (cnt > 0) {
        const int idx = st[--cnt];
        const RNode& nd = B.nodes[idx];
        if (nd.left < 0) {
            const int end = -nd.right - 1;
            for (int i = -nd.left - 1; i < end; ++i) {
                if (c) c->tri++;
                const float d2 = rdist_sq(B.tris[i], p);
                if (d2 <= best) { best = d2; bi = i; }
            }
        } else {
            DI ch[4];
            for (int i = 0; i < 4; ++i) {
                if (c) c->box++;
                ch[i] = DI{rbox_dist_sq(B.nodes[nd.left + i].bb, p), nd.left + i};
            }
            sort4(ch);
            for (int i = 0; i < 4; ++i)
                if (ch[i].d <= best) { if (cnt >= 32) over = true; else st[cnt++] = ch[i].i; }
        }
        if (over) return ref_closest_stackless(B, p, best, c);
    }
    if (bi == -1) { bi = 0; best = 0.0f; }
    return {bi, std::sqrt(best)};
}
// src/bvh.cu:145-176, 250-298 ray_intersect
static std::pair<int, float> ref_ray_stackless(const RefBvh& B, F3 ro, F3 rd, Counters* c) {
    float mint = 1000.0f; int bi = -1; int idx = 0;
    while (idx != -1) {
        const RNode& nd = B.nodes[idx];
        if (c) c->box++;
        if (rbox_ray_tmin(nd.bb, ro, rd) >= mint) { idx = nd.escape; continue; }
        if (nd.left < 0) {
            const int end = -nd.right - 1;
            for (int i = -nd.left - 1; i < end; ++i) {
                if (c) c->tri++;
                const float t = rray_tri(B.tris[i], ro, rd);
                if (t < mint) { mint = t; bi = i; }
            }
            idx = nd.escape;
        } else idx = nd.left;
    }
    return {bi, mint};
}
static std::pair<int, float> ref_ray(const RefBvh& B, F3 ro, F3 rd, Counters* c) {
    int st[32]; int cnt = 0; bool over = false;
    st[cnt++] = 0;
    float mint = 1000.0f; int bi = -1;
    while (cnt > 0) {
        const int idx = st[--cnt];
        const RNode& nd = B.nodes[idx];
        if (nd.left < 0) {
            const int end = -nd.right - 1;
            for (int i = -nd.left - 1; i < end; ++i) {
                if (c) c->tri++;
                const float t = rray_tri(B.tris[i], ro, rd);
                if (t < mint) { mint = t; bi = i; }
            }
        } else {
            DI ch[4];
            for (int i = 0; i < 4; ++i) {
                if (c) c->box++;
                ch[i] = DI{rbox_ray_tmin(B.nodes[nd.left + i].bb, ro, rd), nd.left + i};
            }
            sort4(ch);
            for (int i = 0; i < 4; ++i)
                if (ch[i].d < mint) { if (cnt >= 32) over = true; else st[cnt++] = ch[i].i; }
        }
        if (over) return ref_ray_stackless(B, ro, rd, c);
    }
    return {bi, mint};
}
// src/bvh.cu:216-248, 356-396 avg_normal_around_point
static F3 ref_avg_normal(const RefBvh& B, F3 p, Counters* c) {
    const float EPS = 1e-6f;
    int st[32]; int cnt = 0; bool over = false;
    st[cnt++] = 0;
    float tw = 0; F3 res{0, 0, 0};
    while (cnt > 0) {
        const int idx = st[--cnt];
        const RNode& nd = B.nodes[idx];
        if (nd.left < 0) {
            const int end = -nd.right - 1;
            for (int i = -nd.left - 1; i < end; ++i) {
                if (c) c->tri++;
                if (rdist_sq(B.tris[i], p) < EPS) { res = f3add(res, rnormal(B.tris[i])); tw += 1; }
            }
        } else {
            for (int i = 0; i < 4; ++i) {
                if (c) c->box++;
                if (rbox_dist_sq(B.nodes[nd.left + i].bb, p) < EPS) {
                    if (cnt >= 32) over = true; else st[cnt++] = nd.left + i;
                }
            }
        }
    }
    if (over) {  // stackless fallback
        tw = 0; res = F3{0, 0, 0};
        int idx = 0;
        while (idx != -1) {
            const RNode& nd = B.nodes[idx];
            if (rbox_dist_sq(nd.bb, p) >= EPS) { idx = nd.escape; continue; }
            if (nd.left < 0) {
                const int end = -nd.right - 1;
                for (int i = -nd.left - 1; i < end; ++i)
                    if (rdist_sq(B.tris[i], p) < EPS) { res = f3add(res, rnormal(B.tris[i])); tw += 1; }
                idx = nd.escape;
            } else idx = nd.left;
        }
    }
    return F3{res.x / tw, res.y / tw, res.z / tw};
}

void* orc_ref_build(const float* V, int64_t nv, const int64_t* F, int64_t nf, int n_per_leaf) {
    (void)nv;
    RefBvh* B = new RefBvh();
    B->tris.resize((size_t)nf);
    for (int64_t i = 0; i < nf; ++i) {
        const int64_t* t = F + 3 * i;
        RTri& r = B->tris[(size_t)i];
        r.a = F3{V[3 * t[0]], V[3 * t[0] + 1], V[3 * t[0] + 2]};
        r.b = F3{V[3 * t[1]], V[3 * t[1] + 1], V[3 * t[1] + 2]};
        r.c = F3{V[3 * t[2]], V[3 * t[2] + 1], V[3 * t[2] + 2]};
        r.pad = 0; r.id = i;
    }
    ref_build(*B, (uint32_t)n_per_leaf);
    return B;
}
void orc_ref_free(void* h) { delete (RefBvh*)h; }
int64_t orc_ref_num_nodes(void* h) { return (int64_t)((RefBvh*)h)->nodes.size(); }
// state_dict byte images: nodes [n, 9] int32, triangles [F, 12] int32
void orc_ref_state(void* h, int32_t* nodes, int32_t* tris) {
    RefBvh* B = (RefBvh*)h;
    std::memcpy(nodes, B->nodes.data(), B->nodes.size() * sizeof(RNode));
    std::memcpy(tris, B->tris.data(), B->tris.size() * sizeof(RTri));
}

// src/bvh.cu:687-712 unsigned_distance_kernel; counters (optional) sum work.
void orc_ref_udf(void* h, const float* pts, int64_t n, float* dist, int64_t* fid, float* uvw,
                 int64_t* counters) {
    const RefBvh& B = *(RefBvh*)h;
    int64_t cb = 0, ct = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(orc_get_threads()) reduction(+ : cb, ct)
    for (int64_t i = 0; i < n; ++i) {
        Counters c{0, 0};
        const F3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        const auto r = ref_closest(B, p, 1000.0f * 1000.0f, counters ? &c : nullptr);
        dist[i] = r.second;
        fid[i] = B.tris[r.first].id;
        if (uvw) {
            const F3 cp = rclosest_point(B.tris[r.first], p);
            const F3 b = rbarycentric(B.tris[r.first], cp);
            uvw[3 * i] = b.x; uvw[3 * i + 1] = b.y; uvw[3 * i + 2] = b.z;
        }
        cb += c.box; ct += c.tri;
    }
    if (counters) { counters[0] = cb; counters[1] = ct; }
}
// src/bvh.cu:714-740 raytrace_kernel
void orc_ref_ray(void* h, const float* ro, const float* rd, int64_t n, float* pos, int64_t* fid,
                 float* depth, int64_t* counters) {
    const RefBvh& B = *(RefBvh*)h;
    int64_t cb = 0, ct = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(orc_get_threads()) reduction(+ : cb, ct)
    for (int64_t i = 0; i < n; ++i) {
        Counters c{0, 0};
        const F3 o{ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]}, d{rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]};
        const auto r = ref_ray(B, o, d, counters ? &c : nullptr);
        depth[i] = r.second;
        const F3 q = f3add(o, f3mul(d, r.second));
        pos[3 * i] = q.x; pos[3 * i + 1] = q.y; pos[3 * i + 2] = q.z;
        fid[i] = r.first >= 0 ? B.tris[r.first].id : -1;
        cb += c.box; ct += c.tri;
    }
    if (counters) { counters[0] = cb; counters[1] = ct; }
}
// src/bvh.cu:398-427, 631-685 signed distance kernels (mode 0 watertight, 1 raystab)
void orc_ref_sdf(void* h, const float* pts, int64_t n, int mode, float* dist, int64_t* fid,
                 float* uvw, int64_t* counters) {
    const RefBvh& B = *(RefBvh*)h;
    int64_t cb = 0, ct = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(orc_get_threads()) reduction(+ : cb, ct)
    for (int64_t i = 0; i < n; ++i) {
        Counters c{0, 0};
        Counters* cp_ = counters ? &c : nullptr;
        const F3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        const auto r = ref_closest(B, p, 1000.0f * 1000.0f, cp_);
        float sd = r.second;
        if (mode == 0) {
            const F3 cp = rclosest_point(B.tris[r.first], p);
            const F3 an = ref_avg_normal(B, cp, cp_);
            sd = std::copysign(r.second, f3dot(an, f3sub(p, cp)));
        } else {
            float off[2];
            orc_stab_offsets(1, i, off);
            bool inside = true;
            for (uint32_t k = 0; k < 32 && inside; ++k) {
                float dir[3];
                stab_dir(k, off[0], off[1], dir);
                const F3 d{dir[0], dir[1], dir[2]}, nd{-dir[0], -dir[1], -dir[2]};
                if (ref_ray(B, p, nd, cp_).first < 0 || ref_ray(B, p, d, cp_).first < 0) inside = false;
            }
            sd = inside ? -r.second : r.second;
        }
        dist[i] = sd;
        fid[i] = B.tris[r.first].id;
        if (uvw) {
            const F3 cp = rclosest_point(B.tris[r.first], p);
            const F3 b = rbarycentric(B.tris[r.first], cp);
            uvw[3 * i] = b.x; uvw[3 * i + 1] = b.y; uvw[3 * i + 2] = b.z;
        }
        cb += c.box; ct += c.tri;
    }
    if (counters) { counters[0] = cb; counters[1] = ct; }
}

}  // extern "C"
