// pt_oracle.cpp — CPU restatement of PathTracerGLSL's generated transport loop.
//
// TEST INFRASTRUCTURE ONLY (the oracle): linked by tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / reference arm as the checker; the product never links it.
//
// This is a scalar, data-driven restatement of the program the reference's Generate
// stage emits for a scene x strategy (the unrolled arms of
// src/compiler/generate/features/*.ts become loops over the packed scene of
// include/ptx_rt.h).  Every function names the reference file:line it follows.  The
// arithmetic is binary32 in the GLSL operation order; it is pinned against the
// reference's own programs compiled on the host (oracle/_ref) and the witness values.
//
// Parallelism: OpenMP over pixels (the reference's only parallel axis, one fragment
// per pixel).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <type_traits>
#include <limits>
#include <omp.h>

#include "../include/ptx_rt.h"

// The float transcendentals of the walk.  By default the host libm's float functions;
// built with ORACLE_WIDE_MATH they are evaluated in double and rounded once, which gives
// a second, independent binary32 libm.  Renders with the two differ only where one
// function result differs by an ulp and a later comparison flips: the rate at which that
// happens is the rate expected between any two correct libms (the device's included).
// Double arguments (the forward mode's duals) always take the double functions.
namespace fm {
#ifdef ORACLE_WIDE_MATH
#define FM_F1(name) inline float name(float x) { return (float)std::name((double)x); }
#define FM_F2(name) inline float name(float x, float y) { return (float)std::name((double)x, (double)y); }
#else
#define FM_F1(name) inline float name(float x) { return std::name(x); }
#define FM_F2(name) inline float name(float x, float y) { return std::name(x, y); }
#endif
#define FM_D1(name) inline double name(double x) { return std::name(x); }
#define FM_D2(name) inline double name(double x, double y) { return std::name(x, y); }
FM_F1(exp) FM_F1(log) FM_F1(sin) FM_F1(cos) FM_F1(tan) FM_F1(tanh) FM_F1(atanh) FM_F1(cosh) FM_F2(atan2) FM_F2(pow)
FM_D1(exp) FM_D1(log) FM_D1(sin) FM_D1(cos) FM_D1(tan) FM_D1(tanh) FM_D1(atanh) FM_D1(cosh) FM_D2(atan2) FM_D2(pow)
#undef FM_F1
#undef FM_F2
#undef FM_D1
#undef FM_D2
}  // namespace fm

namespace {

// ---------------------------------------------------------------- vector helpers
struct v3 {
    float x, y, z;
    v3() : x(0), y(0), z(0) {}
    v3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit v3(float s) : x(s), y(s), z(s) {}
    float& operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};
inline v3 operator+(v3 a, v3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline v3 operator-(v3 a, v3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline v3 operator*(v3 a, v3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline v3 operator/(v3 a, v3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline v3 operator*(v3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline v3 operator*(float s, v3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline v3 operator/(v3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline v3 operator-(v3 a) { return v3(-a.x, -a.y, -a.z); }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
inline float length(v3 a) { return std::sqrt(dot(a, a)); }
inline v3 normalize(v3 a) { return a * (1.0f / length(a)); }
inline float fminf_(float a, float b) { return b < a ? b : a; }
inline float fmaxf_(float a, float b) { return a < b ? b : a; }
inline v3 vmin(v3 a, v3 b) { return v3(fminf_(a.x, b.x), fminf_(a.y, b.y), fminf_(a.z, b.z)); }
inline v3 vmax(v3 a, v3 b) { return v3(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z)); }
inline v3 vexp(v3 a) { return v3(fm::exp(a.x), fm::exp(a.y), fm::exp(a.z)); }
inline v3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }
inline float clampf(float x, float lo, float hi) { return fminf_(fmaxf_(x, lo), hi); }
inline float signf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

constexpr float PI = 3.14159265359f;       // math.glsl PI
constexpr float TWO_PI = 6.28318530718f;   // math.glsl TWO_PI
constexpr float MAX_DIST = 1000.0f;        // math.glsl MAX_DIST
constexpr float EPS_INTERFACE = 0.001f;    // math.glsl EPS_INTERFACE
constexpr float MARCH_CLEARANCE = 0.001f;  // math.glsl MARCH_CLEARANCE
constexpr float SHADOW_BACKOFF = 0.002f;   // math.glsl:39 SHADOW_BACKOFF
constexpr float FP_UNCERTAINTY_REL = 3.0517578125e-5f;
constexpr float FP_UNCERTAINTY_ABS = 1.52587890625e-5f;

constexpr uint32_t LOBE_REFLECTION = 1u, LOBE_TRANSMISSION = 2u, LOBE_DELTA = 4u, LOBE_MEDIUM = 8u;
constexpr uint32_t LIGHT_DELTA = 1u;

// spectrum helpers (components/color/spectrum.glsl:1-24), N = 3
inline float spectrum_average(v3 s) { float sum = s[0]; sum += s[1]; sum += s[2]; return sum * (1.0f / 3.0f); }
inline float spectrum_max(v3 s) { float m = s[2]; m = fmaxf_(s[1], m); m = fmaxf_(s[0], m); return m; }
inline bool spectrum_is_black(v3 s) { return s.x <= 0.f && s.y <= 0.f && s.z <= 0.f; }
inline int spectrum_sample_channel(float u) { int c = (int)(u * 3.0f); return c < 2 ? c : 2; }

// The spectral carrier: four wavelength lanes (color/spectral/types.glsl, SPECTRUM_N = 4),
// with the spectrum helpers of spectrum.glsl:1-24 at N = 4.
struct s4 {
    float x, y, z, w;
    s4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    explicit s4(float s) : x(s), y(s), z(s), w(s) {}
    s4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float operator[](int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    float& operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};
inline s4 operator+(s4 a, s4 b) { return s4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline s4 operator-(s4 a, s4 b) { return s4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline s4 operator*(s4 a, s4 b) { return s4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline s4 operator/(s4 a, s4 b) { return s4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
inline s4 operator*(s4 a, float t) { return s4(a.x * t, a.y * t, a.z * t, a.w * t); }
inline s4 operator*(float t, s4 a) { return s4(t * a.x, t * a.y, t * a.z, t * a.w); }
inline s4 operator/(s4 a, float t) { return s4(a.x / t, a.y / t, a.z / t, a.w / t); }
inline s4 operator-(s4 a) { return s4(-a.x, -a.y, -a.z, -a.w); }
inline s4 vexp(s4 a) { return s4(fm::exp(a.x), fm::exp(a.y), fm::exp(a.z), fm::exp(a.w)); }
inline s4 vmax(s4 a, s4 b) { return s4(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z), fmaxf_(a.w, b.w)); }
inline float spectrum_average(s4 s) { float sum = s.x; sum += s.y; sum += s.z; sum += s.w; return sum * (1.0f / 4.0f); }
inline float spectrum_max(s4 s) { float m = s.w; m = fmaxf_(s.z, m); m = fmaxf_(s.y, m); m = fmaxf_(s.x, m); return m; }
inline bool spectrum_is_zero(v3 s) { return s.x == 0.0f && s.y == 0.0f && s.z == 0.0f; }
inline bool spectrum_is_zero(s4 s) { return s.x == 0.0f && s.y == 0.0f && s.z == 0.0f && s.w == 0.0f; }
inline bool spectrum_is_black(s4 s) { return s.x <= 0.f && s.y <= 0.f && s.z <= 0.f && s.w <= 0.f; }
// the channel of the chromatic free-flight draw: one of the carrier's N lanes
template <class Col> inline int sample_channel(float u);
template <> inline int sample_channel<v3>(float u) { return spectrum_sample_channel(u); }
template <> inline int sample_channel<s4>(float u) { int c = (int)(u * 4.0f); return c < 3 ? c : 3; }

// ---------------------------------------------------------------- RNG (pcg4d.glsl:12-40)
struct Rng {
    uint32_t base, dim;
    static void pcg4d(uint32_t v[4]) {
        for (int i = 0; i < 4; ++i) v[i] = v[i] * 1664525u + 1013904223u;
        v[0] += v[1] * v[3]; v[1] += v[2] * v[0]; v[2] += v[0] * v[1]; v[3] += v[1] * v[2];
        for (int i = 0; i < 4; ++i) v[i] ^= v[i] >> 16u;
        v[0] += v[1] * v[3]; v[1] += v[2] * v[0]; v[2] += v[0] * v[1]; v[3] += v[1] * v[2];
    }
    void init(uint32_t px, uint32_t py, uint32_t sample_count, uint32_t salt) {
        uint32_t v[4] = {px, py, sample_count, salt};
        pcg4d(v);
        base = v[0];
        dim = 0;
    }
    float next() {
        uint32_t v[4] = {base, dim++, 0u, 0u};
        pcg4d(v);
        return (float)(v[0] >> 8) * (1.0f / 16777216.0f);
    }
};

// The shadow query's own stream (heterogeneous media): hashed from the path's base and its
// sampler dimension at the NEE site (the device queues shadow queries, so they cannot draw
// from the path's own stream in the reference's order).
inline Rng shadow_rng(uint32_t base, uint32_t seed) {
    uint32_t v[4] = {base, seed, 0x53484457u, 0u};
    Rng::pcg4d(v);
    Rng r;
    r.base = v[0];
    r.dim = 0;
    return r;
}

// ---------------------------------------------------------------- core structs (structs.glsl)
struct Frame { v3 t, b, n; };
struct Ray { v3 o, d; };
struct Hit {
    float t; v3 p; Frame frame; v3 ng;
    int region_from, region_to, region_owner, element;
    float eps;
    float alpha = -1.0f;   // per-triangle GGX alpha of a mesh hit, < 0 = the material's
    int prim = -1;         // original triangle index of a mesh hit
};
template <class Col> struct LightSampleT { v3 wi; float distance; Col radiance; float pdf; uint32_t flags; int light_id; };
template <class Col> struct ISampleT { v3 wi; Col weight; float pdf; uint32_t flags; };
using LightSample = LightSampleT<v3>;
using ISample = ISampleT<v3>;

// fp_uncertainty (math.glsl:54-56)
inline float fp_uncertainty(v3 p) {
    return fmaxf_(FP_UNCERTAINTY_ABS, FP_UNCERTAINTY_REL * fmaxf_(std::fabs(p.x), fmaxf_(std::fabs(p.y), std::fabs(p.z))));
}
// ambient_frame (components/ambient/euclidean/euclidean.glsl:6-33)
inline Frame ambient_frame(v3 n) {
    v3 nn = normalize(n);
    v3 t = std::fabs(nn.x) < 0.9f ? v3(1, 0, 0) : v3(0, 1, 0);
    t = normalize(t - dot(t, nn) * nn);
    return Frame{t, cross(nn, t), nn};
}
// build_basis (math.glsl)
inline void build_basis(v3 n, v3& t, v3& b) {
    v3 up = std::fabs(n.y) < 0.999f ? v3(0, 1, 0) : v3(1, 0, 0);
    t = normalize(cross(up, n));
    b = cross(n, t);
}
// dielectric_fresnel (math.glsl:95-102)
inline float dielectric_fresnel(float cos_i, float eta) {
    float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = std::sqrt(1.0f - sin2_t);
    float r_par = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    float r_perp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (r_par * r_par + r_perp * r_perp);
}
// schlick_fresnel (math.glsl:83-85)
template <class Col> inline Col schlick_fresnel(Col f0, float c) { return f0 + (Col(1.0f) - f0) * fm::pow(1.0f - c, 5.0f); }
// ray_spawn (glsl/core/ray.glsl:29-32)
inline Ray ray_spawn(const Hit& h, v3 wi) {
    float side = dot(wi, h.ng) >= 0.0f ? 1.0f : -1.0f;
    return Ray{h.p + (h.ng * side) * h.eps, wi};
}

// ---------------------------------------------------------------- shapes (components/geometry)
// sphere_intersect (geometry/sphere/sphere.glsl:28-46) — robust Haines form
inline bool sphere_intersect(const Ray& r, v3 c, float rad, float& t) {
    v3 oc = r.o - c;
    float b = dot(oc, r.d);
    v3 perp = oc - b * r.d;
    float disc = rad * rad - dot(perp, perp);
    if (disc < 0.0f) return false;
    float cc = dot(oc, oc) - rad * rad;
    float q = (b >= 0.0f) ? -b - std::sqrt(disc) : -b + std::sqrt(disc);
    if (q == 0.0f) return false;
    float ta = q, tb = cc / q;
    t = (cc < 0.0f) ? fmaxf_(ta, tb) : fminf_(ta, tb);
    return t > 0.0f;
}
inline float sphere_sdf(v3 p, v3 c, float rad) { return length(p - c) - rad; }
// plane_intersect (geometry/plane/plane.glsl)
inline bool plane_intersect(const Ray& r, v3 n, float off, float& t) {
    float denom = dot(r.d, n);
    if (std::fabs(denom) < 1e-8f) return false;
    t = -(dot(r.o, n) + off) / denom;
    return t > 0.0f;
}
inline float plane_sdf(v3 p, v3 n, float off) { return dot(p, n) + off; }
// quad_intersect (geometry/quad/quad.glsl:9-22)
inline bool quad_intersect(const Ray& r, v3 corner, v3 e1, v3 e2, v3 n, float& t) {
    float denom = dot(r.d, n);
    if (std::fabs(denom) < 1e-8f) return false;
    t = dot(corner - r.o, n) / denom;
    if (t <= 0.0f) return false;
    v3 local = r.o + r.d * t - corner;
    float e11 = dot(e1, e1), e22 = dot(e2, e2), e12 = dot(e1, e2);
    float d1 = dot(local, e1), d2 = dot(local, e2);
    float det = e11 * e22 - e12 * e12;
    float u = (d1 * e22 - d2 * e12) / det;
    float v = (d2 * e11 - d1 * e12) / det;
    return u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f;
}
// box_intersect / box_sdf / box_normal (geometry/box/box.glsl)
inline bool box_intersect(const Ray& r, v3 c, v3 h, float& t) {
    v3 inv = v3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    v3 t0 = (c - h - r.o) * inv;
    v3 t1 = (c + h - r.o) * inv;
    v3 tsm = vmin(t0, t1), tbg = vmax(t0, t1);
    float tn = fmaxf_(fmaxf_(tsm.x, tsm.y), tsm.z);
    float tf = fminf_(fminf_(tbg.x, tbg.y), tbg.z);
    if (tf < tn) return false;
    t = (tn < 0.0f) ? tf : tn;
    return t > 0.0f;
}
inline float box_sdf(v3 p, v3 c, v3 h) {
    v3 d = v3(std::fabs(p.x - c.x), std::fabs(p.y - c.y), std::fabs(p.z - c.z)) - h;
    return length(vmax(d, v3(0.0f))) + fminf_(fmaxf_(d.x, fmaxf_(d.y, d.z)), 0.0f);
}
inline v3 box_normal(v3 p, v3 c, v3 h) {
    v3 q = (p - c) / h;
    v3 a(std::fabs(q.x), std::fabs(q.y), std::fabs(q.z));
    if (a.x >= a.y && a.x >= a.z) return v3(signf(q.x), 0, 0);
    if (a.y >= a.z) return v3(0, signf(q.y), 0);
    return v3(0, 0, signf(q.z));
}

// ---------------------------------------------------------------- meshes
// Triangle leaf: Moller-Trumbore of the reference's mesh_tri_test
// (src/components/intersection/mesh/mesh.glsl:41-59); e1, e2 from the float32 positions.
inline bool tri_test(v3 ro, v3 rd, v3 a, v3 e1, v3 e2, float& t) {
    v3 gnorm = cross(e1, e2);
    float det = -dot(rd, gnorm);
    if (std::fabs(det) < 1e-12f) return false;
    float invdet = 1.0f / det;
    v3 ao = ro - a;
    v3 dao = cross(ao, rd);
    float u = dot(e2, dao) * invdet;
    float v = -dot(e1, dao) * invdet;
    t = dot(ao, gnorm) * invdet;
    float w = 1.0f - u - v;
    const float E = 1e-6f;
    return u >= -E && v >= -E && w >= -E;
}

// The oracle's own mesh acceleration: a median-split BVH over triangle boxes (4 triangles
// per leaf).  Its shape is irrelevant to the result: the nearest hit over a triangle set is
// the minimum of the same per-triangle t values whatever the tree.
struct OMesh {
    std::vector<v3> a, e1, e2;
    std::vector<v3> pb, pc;            // the second and third vertices (mesh lights)
    std::vector<float> light_cdf;      // normalised cumulative world area (mesh lights)
    std::vector<float> alpha;
    struct Node { float mn[3], mx[3]; int left, right, start, count; };
    std::vector<Node> nodes;
    std::vector<int> idx;
    float root_mn[3], root_mx[3];

    void build(const ptr_mesh_desc& md) {
        const int T = md.n_triangles;
        a.resize(T); e1.resize(T); e2.resize(T); alpha.assign(T, -1.0f);
        std::vector<float> bmn(3 * (size_t)T), bmx(3 * (size_t)T), cen(3 * (size_t)T);
        for (int t = 0; t < T; ++t) {
            const float* p0 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t];
            const float* p1 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 1];
            const float* p2 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 2];
            a[t] = v3(p0[0], p0[1], p0[2]);
            pb.push_back(v3(p1[0], p1[1], p1[2]));
            pc.push_back(v3(p2[0], p2[1], p2[2]));
            e1[t] = v3(p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]);
            e2[t] = v3(p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]);
            if (md.tri_alpha) alpha[t] = md.tri_alpha[t];
            for (int k = 0; k < 3; ++k) {
                bmn[3 * (size_t)t + k] = std::min(p0[k], std::min(p1[k], p2[k]));
                bmx[3 * (size_t)t + k] = std::max(p0[k], std::max(p1[k], p2[k]));
                cen[3 * (size_t)t + k] = 0.5f * (bmn[3 * (size_t)t + k] + bmx[3 * (size_t)t + k]);
            }
        }
        // lights/mesh/mesh.ts:69-95 packMeshLight: float64 triangle areas from the float32
        // world vertices, the normalised running sum rounded to float32, the last entry 1
        std::vector<double> area(T);
        double acc = 0.0;
        for (int t = 0; t < T; ++t) {
            const float* p0 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t];
            const float* p1 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 1];
            const float* p2 = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 2];
            double u[3], w[3];
            for (int k = 0; k < 3; ++k) { u[k] = (double)p1[k] - p0[k]; w[k] = (double)p2[k] - p0[k]; }
            const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
            area[t] = std::sqrt(cx * cx + cy * cy + cz * cz) / 2.0;
            acc += area[t];
        }
        light_cdf.resize(T);
        double run = 0.0;
        for (int t = 0; t < T; ++t) {
            run += area[t];
            light_cdf[t] = acc > 0.0 ? (float)(run / acc) : (float)((double)(t + 1) / T);
        }
        if (T > 0) light_cdf[T - 1] = 1.0f;
        idx.resize(T);
        for (int i = 0; i < T; ++i) idx[i] = i;
        nodes.clear();
        nodes.reserve(2 * (size_t)T);
        build_rec(0, T, bmn, bmx, cen);
        for (int k = 0; k < 3; ++k) { root_mn[k] = nodes[0].mn[k]; root_mx[k] = nodes[0].mx[k]; }
    }
    int build_rec(int s0, int s1, const std::vector<float>& bmn, const std::vector<float>& bmx, const std::vector<float>& cen) {
        Node nd;
        for (int k = 0; k < 3; ++k) { nd.mn[k] = 1e30f; nd.mx[k] = -1e30f; }
        for (int i = s0; i < s1; ++i)
            for (int k = 0; k < 3; ++k) {
                nd.mn[k] = std::min(nd.mn[k], bmn[3 * (size_t)idx[i] + k]);
                nd.mx[k] = std::max(nd.mx[k], bmx[3 * (size_t)idx[i] + k]);
            }
        int me = (int)nodes.size();
        nodes.push_back(nd);
        if (s1 - s0 <= 4) {
            nodes[me].left = nodes[me].right = -1;
            nodes[me].start = s0;
            nodes[me].count = s1 - s0;
            return me;
        }
        int axis = 0;
        float ext = -1.0f;
        for (int k = 0; k < 3; ++k) if (nd.mx[k] - nd.mn[k] > ext) { ext = nd.mx[k] - nd.mn[k]; axis = k; }
        int mid = (s0 + s1) / 2;
        std::nth_element(idx.begin() + s0, idx.begin() + mid, idx.begin() + s1,
                         [&](int x, int y) { return cen[3 * (size_t)x + axis] < cen[3 * (size_t)y + axis]; });
        int l = build_rec(s0, mid, bmn, bmx, cen);
        int r = build_rec(mid, s1, bmn, bmx, cen);
        nodes[me].left = l;
        nodes[me].right = r;
        nodes[me].start = nodes[me].count = 0;
        return me;
    }
    // entry distance of the ray into the node box, or +inf when it misses within tmax
    // (conservative: only prunes and orders, never decides a hit)
    static float box_entry(const Node& n, v3 ro, v3 inv, float tmax) {
        float tn = 0.0f, tf = tmax;
        for (int k = 0; k < 3; ++k) {
            float t0 = (n.mn[k] - ro[k]) * inv[k], t1 = (n.mx[k] - ro[k]) * inv[k];
            if (t0 != t0 || t1 != t1) continue;   // ray on the slab plane with a zero direction: no constraint
            tn = std::max(tn, std::min(t0, t1));
            tf = std::min(tf, std::max(t0, t1));
        }
        return tn <= tf * 1.0001f + 1e-6f ? tn : std::numeric_limits<float>::infinity();
    }
    static bool box_hit(const Node& n, v3 ro, v3 inv, float tmax) {
        return box_entry(n, ro, inv, tmax) != std::numeric_limits<float>::infinity();
    }
    // nearest triangle with t in (0, tmax); returns the triangle index or -1
    int nearest(v3 ro, v3 rd, float& tmax) const {
        v3 inv(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
        int best = -1;
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const Node& n = nodes[stack[--sp]];
            if (!box_hit(n, ro, inv, tmax)) continue;
            if (n.left < 0) {
                for (int i = n.start; i < n.start + n.count; ++i) {
                    int t_i = idx[i];
                    float t;
                    if (tri_test(ro, rd, a[t_i], e1[t_i], e2[t_i], t) && t > 0.0f && (t < tmax || (t == tmax && best >= 0 && t_i < best))) {
                        tmax = t;
                        best = t_i;
                    }
                }
            } else {
                // front to back: push the farther child first
                float tl = box_entry(nodes[n.left], ro, inv, tmax), tr = box_entry(nodes[n.right], ro, inv, tmax);
                bool hl = tl != std::numeric_limits<float>::infinity(), hr = tr != std::numeric_limits<float>::infinity();
                if (hl && hr) {
                    if (tl <= tr) { stack[sp++] = n.right; stack[sp++] = n.left; }
                    else { stack[sp++] = n.left; stack[sp++] = n.right; }
                } else if (hl) stack[sp++] = n.left;
                else if (hr) stack[sp++] = n.right;
            }
        }
        return best;
    }
    bool any(v3 ro, v3 rd, float max_dist) const {
        float tm = max_dist;
        v3 inv(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const Node& n = nodes[stack[--sp]];
            if (!box_hit(n, ro, inv, tm)) continue;
            if (n.left < 0) {
                for (int i = n.start; i < n.start + n.count; ++i) {
                    int t_i = idx[i];
                    float t;
                    if (tri_test(ro, rd, a[t_i], e1[t_i], e2[t_i], t) && t > 0.0f && t < max_dist) return true;
                }
            } else {
                stack[sp++] = n.left;
                stack[sp++] = n.right;
            }
        }
        return false;
    }
};

// Placement algebra (intersection/instancing/placement.glsl:19-41).
inline v3 qrot(const float* q, v3 v) {
    v3 qv(q[0], q[1], q[2]);
    return v + 2.0f * cross(qv, cross(qv, v) + q[3] * v);
}
inline v3 placement_normal(const float* q, v3 n) {
    float c[4] = {-q[0], -q[1], -q[2], q[3]};
    return qrot(c, n);
}

struct OBatch {
    int shape, mesh;
    std::vector<float> place;    // 8 per instance (q, ts)
    std::vector<float> sphere;   // 4 per instance: world centre, world radius (sphere batches)
    std::vector<float> wbox;     // 6 per instance: world box of a mesh instance (culling only)
};

// Ray vs world box (culling only: conservative, never decides a hit).
inline bool ray_box_cull(const float* b, v3 ro, v3 rd, float tmax) {
    float tn = 0.0f, tf = tmax;
    for (int k = 0; k < 3; ++k) {
        float inv = 1.0f / rd[k];
        float t0 = (b[k] - ro[k]) * inv, t1 = (b[3 + k] - ro[k]) * inv;
        if (t0 != t0 || t1 != t1) continue;
        tn = std::max(tn, std::min(t0, t1));
        tf = std::min(tf, std::max(t0, t1));
    }
    return tn <= tf * 1.0001f + 1e-5f;
}

// ---------------------------------------------------------------- scene
struct Scene {
    const ptr_scene_desc* d;
    const ptr_program_desc* prog;
    std::vector<int> light_of_region;  // region -> light index (light_of), -1 none
    std::vector<int> batch_light_base; // batch -> light id of its instance 0, -1 none
    bool tree = false;                 // light-tree selection
    bool env_samplable, env_select_live;
    bool has_media;

    std::vector<OMesh> meshes;
    std::vector<OBatch> batches;

    explicit Scene(const ptr_scene_desc* sd, const ptr_program_desc* pd) : d(sd), prog(pd) {
        meshes.resize(sd->n_meshes > 0 ? sd->n_meshes : 0);
        for (int i = 0; i < sd->n_meshes; ++i) meshes[i].build(sd->meshes[i]);
        batches.resize(sd->n_batches > 0 ? sd->n_batches : 0);
        for (int i = 0; i < sd->n_batches; ++i) {
            const ptr_batch_desc& bd = sd->batches[i];
            OBatch& b = batches[i];
            b.shape = bd.prototype_shape;
            b.mesh = bd.prototype_ref;
            b.place.assign(bd.placements, bd.placements + 8 * (size_t)bd.n_instances);
            if (b.shape == PTR_SHAPE_MESH) {
                const OMesh& m = meshes[b.mesh];
                for (int k = 0; k < bd.n_instances; ++k) {
                    const float* pl = bd.placements + 8 * (size_t)k;
                    float bx[6] = {1e30f, 1e30f, 1e30f, -1e30f, -1e30f, -1e30f};
                    for (int c = 0; c < 8; ++c) {
                        double lx = (c & 1) ? m.root_mx[0] : m.root_mn[0];
                        double ly = (c & 2) ? m.root_mx[1] : m.root_mn[1];
                        double lz = (c & 4) ? m.root_mx[2] : m.root_mn[2];
                        double sc = pl[7];
                        double vx = sc * lx - pl[4], vy = sc * ly - pl[5], vz = sc * lz - pl[6];
                        double cx = -pl[0], cy = -pl[1], cz = -pl[2], w = pl[3];
                        double c1x = cy * vz - cz * vy + w * vx, c1y = cz * vx - cx * vz + w * vy, c1z = cx * vy - cy * vx + w * vz;
                        double c2x = cy * c1z - cz * c1y, c2y = cz * c1x - cx * c1z, c2z = cx * c1y - cy * c1x;
                        double wp[3] = {vx + 2.0 * c2x, vy + 2.0 * c2y, vz + 2.0 * c2z};
                        for (int a = 0; a < 3; ++a) {
                            bx[a] = std::min(bx[a], (float)wp[a] - 1e-4f * (1.0f + std::fabs((float)wp[a])));
                            bx[3 + a] = std::max(bx[3 + a], (float)wp[a] + 1e-4f * (1.0f + std::fabs((float)wp[a])));
                        }
                    }
                    b.wbox.insert(b.wbox.end(), bx, bx + 6);
                }
            }
            if (b.shape == PTR_SHAPE_SPHERE) {
                for (int k = 0; k < bd.n_instances; ++k) {
                    const float* pl = bd.placements + 8 * (size_t)k;
                    // world centre = rotate(conj(q), s*c - t_rigid) in double, then float
                    double sc = pl[7];
                    double vx = sc * bd.proto[0] - pl[4], vy = sc * bd.proto[1] - pl[5], vz = sc * bd.proto[2] - pl[6];
                    double cx = -pl[0], cy = -pl[1], cz = -pl[2], w = pl[3];
                    double c1x = cy * vz - cz * vy + w * vx, c1y = cz * vx - cx * vz + w * vy, c1z = cx * vy - cy * vx + w * vz;
                    double c2x = cy * c1z - cz * c1y, c2y = cz * c1x - cx * c1z, c2z = cx * c1y - cy * c1x;
                    b.sphere.push_back((float)(vx + 2.0 * c2x));
                    b.sphere.push_back((float)(vy + 2.0 * c2y));
                    b.sphere.push_back((float)(vz + 2.0 * c2z));
                    b.sphere.push_back((float)(sc * bd.proto[3]));
                }
            }
        }
        light_of_region.assign(sd->n_regions, -1);
        for (int i = 0; i < sd->n_lights; ++i)
            if (sd->lights[i].region >= 0) light_of_region[sd->lights[i].region] = i;
        for (int i = 0; i < sd->n_batches; ++i) batch_light_base.push_back(sd->batches[i].light_base);
        tree = pd->light_tree != 0 && sd->n_tree_nodes > 0;
        env_samplable = sd->env.kind != PTR_ENV_NONE && sd->env.sample_as_light;
        env_select_live = env_samplable && sd->n_lights > 0;
        has_media = sd->ambient_material >= 0 && (sd->materials[sd->ambient_material].flags & PTR_MATF_MEDIUM);
        for (int i = 0; i < sd->n_materials; ++i)
            if (sd->materials[i].flags & PTR_MATF_MEDIUM) has_media = true;
    }
    const ptr_material* mat(int m) const { return (m >= 0 && m < d->n_materials) ? &d->materials[m] : nullptr; }
    // material_of (generated, features/intersection.ts): region -> material; -1 = ambient
    int material_of(int region) const {
        if (region < 0) return d->ambient_material;
        return d->regions[region].material;
    }
    float ior_of(int region) const { return region < 0 ? 1.0f : d->regions[region].ior; }
    bool material_is_emissive(int m) const { auto* p = mat(m); return p && (p->flags & PTR_MATF_EMISSIVE); }
    bool is_null_interface(int m) const { auto* p = mat(m); return p && p->model == PTR_MAT_NONE; }
    bool material_has_medium(int m) const { auto* p = mat(m); return p && (p->flags & PTR_MATF_MEDIUM); }
    bool material_has_nondelta_lobes(int m) const {
        auto* p = mat(m);
        return p && (p->model == PTR_MAT_LAMBERT || p->model == PTR_MAT_GGX || p->model == PTR_MAT_ROUGH_DIELECTRIC);
    }

    // primitive_intersect (features/intersection.ts:801-824, primitiveHitFill :695-715),
    // mesh arms (generateMeshDispatch :890-915) and instance leaves (instanceLeafItem :981-1066)
    bool primitive_intersect(const Ray& r, Hit& hit) const {
        bool found = false;
        for (int i = 0; i < d->n_regions; ++i) {
            const ptr_region& g = d->regions[i];
            if (g.shape == PTR_SHAPE_MESH) {
                const OMesh& m = meshes[g.ref];
                float t = hit.t;
                int tri = m.nearest(r.o, r.d, t);
                if (tri >= 0) {
                    hit.t = t;
                    found = true;
                    hit.p = r.o + r.d * t;
                    hit.eps = fp_uncertainty(hit.p);
                    v3 gl = cross(m.e1[tri], m.e2[tri]);
                    hit.frame = ambient_frame(normalize(gl));
                    hit.ng = normalize(gl);
                    hit.region_owner = i;
                    hit.element = 0;
                    hit.alpha = m.alpha[tri];
                    hit.prim = tri;
                }
                continue;
            }
            if (g.shape == PTR_SHAPE_INSTANCES) {
                const OBatch& b = batches[g.ref];
                const int N = (int)b.place.size() / 8;
                for (int k = 0; k < N; ++k) {
                    if (b.shape == PTR_SHAPE_SPHERE) {
                        const float* sp = &b.sphere[4 * (size_t)k];
                        float t;
                        if (sphere_intersect(r, v3(sp[0], sp[1], sp[2]), sp[3], t) && t < hit.t) {
                            hit.t = t;
                            found = true;
                            hit.p = r.o + r.d * t;
                            hit.eps = fp_uncertainty(hit.p);
                            hit.frame = ambient_frame(normalize(hit.p - v3(sp[0], sp[1], sp[2])));
                            hit.ng = hit.frame.n;
                            hit.region_owner = i;
                            hit.element = k;
                            hit.alpha = -1.0f;
                            hit.prim = -1;
                        }
                        continue;
                    }
                    if (!ray_box_cull(&b.wbox[6 * (size_t)k], r.o, r.d, hit.t)) continue;
                    const float* q = &b.place[8 * (size_t)k];
                    const float s = q[7];
                    v3 ro = (qrot(q, r.o) + v3(q[4], q[5], q[6])) / s;
                    v3 rd = qrot(q, r.d) / s;
                    const OMesh& m = meshes[b.mesh];
                    float t = hit.t;
                    int tri = m.nearest(ro, rd, t);
                    if (tri >= 0) {
                        hit.t = t;
                        found = true;
                        hit.p = r.o + r.d * t;
                        hit.eps = fp_uncertainty(hit.p);
                        v3 gl = cross(m.e1[tri], m.e2[tri]);
                        hit.frame = ambient_frame(normalize(placement_normal(q, gl)));
                        hit.ng = normalize(placement_normal(q, gl));
                        hit.region_owner = i;
                        hit.element = k;
                        hit.alpha = m.alpha[tri];
                        hit.prim = tri;
                    }
                }
                continue;
            }
            float t;
            v3 n;
            bool ok = false;
            switch (g.shape) {
                case PTR_SHAPE_PLANE: ok = plane_intersect(r, ld3(g.p), g.p[3], t); break;
                case PTR_SHAPE_SPHERE: ok = sphere_intersect(r, ld3(g.p), g.p[3], t); break;
                case PTR_SHAPE_QUAD: ok = quad_intersect(r, ld3(g.p), ld3(g.p + 3), ld3(g.p + 6), ld3(g.p + 9), t); break;
                case PTR_SHAPE_BOX: ok = box_intersect(r, ld3(g.p), ld3(g.p + 3), t); break;
                default: break;
            }
            if (!(ok && t < hit.t)) continue;
            hit.t = t;
            found = true;
            hit.p = r.o + r.d * t;
            hit.eps = fp_uncertainty(hit.p);
            switch (g.shape) {
                case PTR_SHAPE_PLANE: n = ld3(g.p); break;
                case PTR_SHAPE_SPHERE: n = normalize(hit.p - ld3(g.p)); break;
                case PTR_SHAPE_QUAD: n = ld3(g.p + 9); break;
                default: n = box_normal(hit.p, ld3(g.p), ld3(g.p + 3)); break;
            }
            hit.frame = ambient_frame(n);
            hit.ng = hit.frame.n;
            hit.region_owner = i;
            hit.element = 0;
            hit.alpha = -1.0f;
            hit.prim = -1;
        }
        return found;
    }
    bool scene_intersect_any(const Ray& r, float maxDist) const {
        for (int i = 0; i < d->n_regions; ++i) {
            const ptr_region& g = d->regions[i];
            if (g.shape == PTR_SHAPE_MESH) {
                if (meshes[g.ref].any(r.o, r.d, maxDist)) return true;
                continue;
            }
            if (g.shape == PTR_SHAPE_INSTANCES) {
                const OBatch& b = batches[g.ref];
                const int N = (int)b.place.size() / 8;
                for (int k = 0; k < N; ++k) {
                    if (b.shape == PTR_SHAPE_SPHERE) {
                        const float* sp = &b.sphere[4 * (size_t)k];
                        float t;
                        if (sphere_intersect(r, v3(sp[0], sp[1], sp[2]), sp[3], t) && t < maxDist) return true;
                        continue;
                    }
                    if (!ray_box_cull(&b.wbox[6 * (size_t)k], r.o, r.d, maxDist)) continue;
                    const float* q = &b.place[8 * (size_t)k];
                    v3 ro = (qrot(q, r.o) + v3(q[4], q[5], q[6])) / q[7];
                    v3 rd = qrot(q, r.d) / q[7];
                    if (meshes[b.mesh].any(ro, rd, maxDist)) return true;
                }
                continue;
            }
            float t;
            bool ok = false;
            switch (g.shape) {
                case PTR_SHAPE_PLANE: ok = plane_intersect(r, ld3(g.p), g.p[3], t); break;
                case PTR_SHAPE_SPHERE: ok = sphere_intersect(r, ld3(g.p), g.p[3], t); break;
                case PTR_SHAPE_QUAD: ok = quad_intersect(r, ld3(g.p), ld3(g.p + 3), ld3(g.p + 6), ld3(g.p + 9), t); break;
                case PTR_SHAPE_BOX: ok = box_intersect(r, ld3(g.p), ld3(g.p + 3), t); break;
                default: break;
            }
            if (ok && t < maxDist) return true;
        }
        return false;
    }
    // scene_region_at (features/intersection.ts:1121-1225): innermost-wins point classification
    int scene_region_at(v3 p) const {
        int region = -1;
        float best = -1.0e20f;
        for (int i = 0; i < d->n_regions; ++i) {
            const ptr_region& g = d->regions[i];
            float dd;
            if (g.shape == PTR_SHAPE_INSTANCES) {
                // instanced sphere batch: every containing instance competes (innermost wins)
                const OBatch& b = batches[g.ref];
                if (b.shape != PTR_SHAPE_SPHERE) continue;
                for (size_t k = 0; k + 3 < b.sphere.size(); k += 4) {
                    float ds = sphere_sdf(p, v3(b.sphere[k], b.sphere[k + 1], b.sphere[k + 2]), b.sphere[k + 3]);
                    if (ds < 0.0f && ds > best) { best = ds; region = i; }
                }
                continue;
            }
            switch (g.shape) {
                case PTR_SHAPE_PLANE: dd = plane_sdf(p, ld3(g.p), g.p[3]); break;
                case PTR_SHAPE_SPHERE: dd = sphere_sdf(p, ld3(g.p), g.p[3]); break;
                case PTR_SHAPE_BOX: dd = box_sdf(p, ld3(g.p), ld3(g.p + 3)); break;
                default: dd = 1.0e20f; break;   // thin owners never claim containment
            }
            if (dd < 0.0f && dd > best) { best = dd; region = i; }
        }
        return region;
    }
    // scene_intersect (features/intersection.ts:1665-1713 generateSceneIntersect)
    bool scene_intersect(const Ray& r, Hit& hit) const {
        hit.t = MAX_DIST;
        hit.eps = MARCH_CLEARANCE;
        bool found = primitive_intersect(r, hit);
        if (found) {
            int outside = scene_region_at(hit.p + hit.ng * EPS_INTERFACE);
            if (dot(r.d, hit.ng) < 0.0f) {
                hit.region_from = outside;
                hit.region_to = hit.region_owner;
            } else {
                hit.region_from = d->regions[hit.region_owner].thin
                    ? scene_region_at(hit.p + hit.ng * (-EPS_INTERFACE))
                    : hit.region_owner;
                hit.region_to = outside;
                hit.frame = ambient_frame(-hit.frame.n);
                hit.ng = -hit.ng;
            }
        }
        return found;
    }
};

// ---------------------------------------------------------------- materials
// lambert (materials/lambert/lambert.glsl:7-37)
template <class Col> inline Col lambert_eval(v3 wi, v3 wo, const Hit& h, Col albedo) {
    if (dot(wi, h.frame.n) * dot(wo, h.frame.n) <= 0.0f) return Col(0.0f);
    return albedo * (1.0f / PI);
}
template <class Col> inline ISampleT<Col> lambert_sample(v3 wo, const Hit& h, Col albedo, float, float u0, float u1) {
    const Frame& f = h.frame;
    v3 n = dot(wo, f.n) < 0.0f ? -f.n : f.n;
    float cos_theta = std::sqrt(u1);
    float sin_theta = std::sqrt(fmaxf_(0.0f, 1.0f - u1));
    float phi = TWO_PI * u0;
    ISampleT<Col> s;
    s.wi = normalize(f.t * (sin_theta * fm::cos(phi)) + f.b * (sin_theta * fm::sin(phi)) + n * cos_theta);
    s.weight = albedo;
    s.pdf = cos_theta * (1.0f / PI);
    s.flags = LOBE_REFLECTION;
    return s;
}
inline float lambert_pdf(v3 wi, v3 wo, const Hit& h) {
    float c = dot(wi, h.frame.n) * signf(dot(wo, h.frame.n));
    return fmaxf_(0.0f, c) * (1.0f / PI);
}
// microfacet (glsl/core/microfacet.glsl:22-54)
inline v3 mf_to_local(const Frame& f, v3 v) { return v3(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }
inline v3 mf_from_local(const Frame& f, v3 v) { return normalize(f.t * v.x + f.b * v.y + f.n * v.z); }
inline float mf_D(v3 h, float a) { float t = h.z * h.z * (a * a - 1.0f) + 1.0f; return a * a / (PI * t * t); }
inline float mf_G1(v3 v, float a) { float c = std::fabs(v.z); return 2.0f * c / (c + std::sqrt(a * a + (1.0f - a * a) * c * c)); }
inline v3 mf_sample_vndf(v3 wol, float a, float u0, float u1) {
    v3 vh = normalize(v3(a * wol.x, a * wol.y, wol.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    v3 T1 = lensq > 0.0f ? v3(-vh.y, vh.x, 0.0f) * (1.0f / std::sqrt(lensq)) : v3(1, 0, 0);
    v3 T2 = cross(vh, T1);
    float rr = std::sqrt(u0);
    float phi = TWO_PI * u1;
    float t1 = rr * fm::cos(phi);
    float t2 = rr * fm::sin(phi);
    float s_ = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - s_) * std::sqrt(fmaxf_(0.0f, 1.0f - t1 * t1)) + s_ * t2;
    v3 nh = t1 * T1 + t2 * T2 + std::sqrt(fmaxf_(0.0f, 1.0f - t1 * t1 - t2 * t2)) * vh;
    return normalize(v3(a * nh.x, a * nh.y, fmaxf_(1e-6f, nh.z)));
}
// ggx conductor (materials/ggx/ggx.glsl:16-64)
template <class Col> inline Col ggx_eval(v3 wi, v3 wo, const Hit& h, Col f0, float a) {
    v3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return Col(0.0f);
    v3 hh = normalize(wil + wol);
    Col F = schlick_fresnel(f0, std::fabs(dot(wol, hh)));
    return F * (mf_D(hh, a) * mf_G1(wil, a) * mf_G1(wol, a) / (4.0f * std::fabs(wil.z) * std::fabs(wol.z)));
}
template <class Col> inline ISampleT<Col> ggx_sample(v3 wo, const Hit& h, Col f0, float a, float u0, float u1) {
    v3 wol = mf_to_local(h.frame, wo);
    float side = wol.z < 0.0f ? -1.0f : 1.0f;
    wol = wol * side;
    v3 hh = mf_sample_vndf(wol, a, u0, u1);
    v3 i = -wol;
    v3 wil = i - 2.0f * dot(hh, i) * hh;   // reflect(-wol, h)
    ISampleT<Col> s;
    if (wil.z <= 0.0f) { s.wi = wo; s.weight = Col(0.0f); s.pdf = 0.0f; s.flags = LOBE_REFLECTION; return s; }
    Col F = schlick_fresnel(f0, std::fabs(dot(wol, hh)));
    s.weight = F * mf_G1(wil, a);
    s.pdf = mf_G1(wol, a) * mf_D(hh, a) / (4.0f * std::fabs(wol.z));
    s.flags = LOBE_REFLECTION;
    s.wi = mf_from_local(h.frame, wil * side);
    return s;
}
inline float ggx_pdf(v3 wi, v3 wo, const Hit& h, float a) {
    v3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return 0.0f;
    v3 hh = normalize(wil + wol);
    return mf_G1(wol, a) * mf_D(hh, a) / (4.0f * std::fabs(wol.z));
}

// mirror (materials/mirror/mirror.glsl): one delta lobe weighted by Schlick Fresnel
template <class Col> inline ISampleT<Col> mirror_sample(v3 wo, const Hit& h, Col f0) {
    v3 n = h.frame.n;
    float cos_i = clampf(dot(wo, n), 1e-6f, 1.0f);
    ISampleT<Col> s;
    s.wi = normalize(2.0f * cos_i * n - wo);
    s.weight = schlick_fresnel(f0, cos_i);
    s.pdf = 0.0f;
    s.flags = LOBE_REFLECTION | LOBE_DELTA;
    return s;
}
// rough dielectric (materials/rough_dielectric/rough_dielectric.glsl): Walter 2007 two-lobe
// microfacet BSDF, VNDF sampling, exact Fresnel, eta^2 on the transmission lobe; wo in the
// frame's upper hemisphere, eta = n_i / n_t, equal indices = delta pass-through
inline bool rough_half(v3 wil, v3 wol, float eta, v3& m) {
    float etap = wil.z > 0.0f ? 1.0f : 1.0f / eta;
    m = wil * etap + wol;
    if (dot(m, m) <= 0.0f) return false;
    m = normalize(m);
    if (m.z < 0.0f) m = -m;
    return dot(m, wil) * wil.z >= 0.0f && dot(m, wol) * wol.z >= 0.0f;
}
template <class Col> inline Col rough_dielectric_eval_local(v3 wil, v3 wol, Col tint, float a, float n_i, float n_t) {
    if (wol.z <= 0.0f || wil.z == 0.0f) return Col(0.0f);
    if (n_i == n_t) return Col(0.0f);
    float eta = n_i / n_t;
    v3 m;
    if (!rough_half(wil, wol, eta, m)) return Col(0.0f);
    float cos_om = clampf(std::fabs(dot(wol, m)), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    float DG = mf_D(m, a) * mf_G1(wol, a) * mf_G1(wil, a);
    if (wil.z > 0.0f) return Col(1.0f) * (DG * F / (4.0f * wil.z * wol.z));
    float denom = dot(wil, m) + dot(wol, m) * eta;
    denom *= denom;
    float ft = DG * (1.0f - F) * std::fabs(dot(wil, m) * dot(wol, m) / (wil.z * wol.z * denom));
    return tint * (ft * eta * eta);
}
inline float rough_dielectric_pdf_local(v3 wil, v3 wol, float a, float n_i, float n_t) {
    if (wol.z <= 0.0f || wil.z == 0.0f) return 0.0f;
    if (n_i == n_t) return 0.0f;
    float eta = n_i / n_t;
    v3 m;
    if (!rough_half(wil, wol, eta, m)) return 0.0f;
    float cos_om = clampf(std::fabs(dot(wol, m)), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    if (wil.z > 0.0f) return F * mf_G1(wol, a) * mf_D(m, a) / (4.0f * wol.z);
    float denom = dot(wil, m) + dot(wol, m) * eta;
    denom *= denom;
    return (1.0f - F) * mf_G1(wol, a) * mf_D(m, a) * cos_om / wol.z * std::fabs(dot(wil, m)) / denom;
}
// the sampled lobe in the local frame (wil); the caller maps it out of the frame
template <class Col>
inline ISampleT<Col> rough_dielectric_sample_local(v3 wol, Col tint, float a, float n_i, float n_t, float uc, float u0,
                                                   float u1) {
    ISampleT<Col> s;
    s.wi = wol;
    s.weight = Col(0.0f);
    s.pdf = 0.0f;
    s.flags = LOBE_REFLECTION;
    if (wol.z <= 0.0f) return s;
    float eta = n_i / n_t;
    if (n_i == n_t) {
        s.wi = -wol;
        s.weight = tint;
        s.flags = LOBE_TRANSMISSION | LOBE_DELTA;
        return s;
    }
    v3 m = mf_sample_vndf(wol, a, u0, u1);
    float cos_om = clampf(dot(wol, m), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    v3 wil;
    if (uc < F) {
        v3 i = -wol;
        wil = i - 2.0f * dot(m, i) * m;
        if (wil.z <= 0.0f) return s;
        s.weight = Col(1.0f) * mf_G1(wil, a);
        s.pdf = F * mf_G1(wol, a) * mf_D(m, a) / (4.0f * wol.z);
        s.flags = LOBE_REFLECTION;
    } else {
        float sin2_t = eta * eta * (1.0f - cos_om * cos_om);
        float cos_t = std::sqrt(fmaxf_(0.0f, 1.0f - sin2_t));
        wil = normalize(-eta * wol + (eta * cos_om - cos_t) * m);
        if (wil.z >= 0.0f) return s;
        float denom = dot(wil, m) + dot(wol, m) * eta;
        denom *= denom;
        s.weight = tint * (mf_G1(wil, a) * eta * eta);
        s.pdf = (1.0f - F) * mf_G1(wol, a) * mf_D(m, a) * cos_om / wol.z * std::fabs(dot(wil, m)) / denom;
        s.flags = LOBE_TRANSMISSION;
    }
    s.wi = wil;
    return s;
}

// ---------------------------------------------------------------- media (transport/volume/analytic)
template <class Col> struct MediumSampleT { bool scattered; float t; Col weight; v3 exit_p, exit_dir; };
using MediumSample = MediumSampleT<v3>;

// ---- heterogeneous media (transport/volume/delta_tracking/delta_tracking.glsl)
// The coefficient field: the stack program of a GLSL expression of p, interpreted with
// the same operations in the same order as the device.
inline float fract_(float x) { return x - std::floor(x); }
inline v3 field_eval(const uint32_t* code, v3 p) {
    v3 st[PTR_FIELD_MAX_STACK];
    int sp = 0;
    auto fl = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };
    for (int pc = 0;;) {
        const uint32_t op = code[pc++];
        if (op == PTR_FOP_END) break;
        if (op == PTR_FOP_CONST) { st[sp++] = v3(fl(code[pc]), fl(code[pc + 1]), fl(code[pc + 2])); pc += 3; continue; }
        if (op == PTR_FOP_P) { st[sp++] = p; continue; }
        if (op == PTR_FOP_SWZ) { float x = st[sp - 1][(int)code[pc++]]; st[sp - 1] = v3(x, x, x); continue; }
        if (op >= PTR_FOP_ADD && op <= PTR_FOP_DIV) {
            v3 b = st[--sp], a = st[sp - 1];
            st[sp - 1] = op == PTR_FOP_ADD ? a + b : op == PTR_FOP_SUB ? a - b : op == PTR_FOP_MUL ? a * b
                       : v3(a.x / b.x, a.y / b.y, a.z / b.z);
            continue;
        }
        if (op >= PTR_FOP_NEG && op <= PTR_FOP_FRACT) {
            v3 a = st[sp - 1];
            for (int k = 0; k < 3; ++k) {
                float x = a[k];
                switch (op) {
                    case PTR_FOP_NEG: x = -x; break;
                    case PTR_FOP_EXP: x = fm::exp(x); break;
                    case PTR_FOP_LOG: x = fm::log(x); break;
                    case PTR_FOP_SIN: x = fm::sin(x); break;
                    case PTR_FOP_COS: x = fm::cos(x); break;
                    case PTR_FOP_SQRT: x = std::sqrt(x); break;
                    case PTR_FOP_ABS: x = std::fabs(x); break;
                    case PTR_FOP_FLOOR: x = std::floor(x); break;
                    default: x = fract_(x); break;
                }
                a[k] = x;
            }
            st[sp - 1] = a;
            continue;
        }
        if (op >= PTR_FOP_POW && op <= PTR_FOP_STEP) {
            v3 b = st[--sp], a = st[sp - 1];
            for (int k = 0; k < 3; ++k) {
                float x = a[k], y = b[k];
                switch (op) {
                    case PTR_FOP_POW: x = fm::pow(x, y); break;
                    case PTR_FOP_MIN: x = y < x ? y : x; break;
                    case PTR_FOP_MAX: x = x < y ? y : x; break;
                    case PTR_FOP_MOD: x = x - y * std::floor(x / y); break;
                    default: x = y < x ? 0.0f : 1.0f; break;   // step(edge = a, x = b)
                }
                a[k] = x;
            }
            st[sp - 1] = a;
            continue;
        }
        if (op >= PTR_FOP_CLAMP && op <= PTR_FOP_SMOOTHSTEP) {
            v3 c = st[--sp], b = st[--sp], a = st[sp - 1];
            for (int k = 0; k < 3; ++k) {
                float x;
                if (op == PTR_FOP_CLAMP) {
                    x = a[k] < b[k] ? b[k] : a[k];
                    x = c[k] < x ? c[k] : x;
                } else if (op == PTR_FOP_MIX) {
                    x = a[k] * (1.0f - c[k]) + b[k] * c[k];
                } else {
                    float t = (c[k] - a[k]) / (b[k] - a[k]);
                    t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
                    x = t * t * (3.0f - 2.0f * t);
                }
                a[k] = x;
            }
            st[sp - 1] = a;
            continue;
        }
        if (op == PTR_FOP_DOT) { v3 b = st[--sp]; float dd = dot(st[sp - 1], b); st[sp - 1] = v3(dd, dd, dd); continue; }
        if (op == PTR_FOP_LENGTH) { float l = std::sqrt(dot(st[sp - 1], st[sp - 1])); st[sp - 1] = v3(l, l, l); continue; }
        v3 z = st[--sp], y = st[--sp], x = st[sp - 1];   // VEC3
        st[sp - 1] = v3(x.x, y.x, z.x);
    }
    return st[0];
}
// medium_sample_analytic (transport/volume/analytic/analytic.glsl:9-43)
template <class Col>
inline MediumSampleT<Col> medium_sample_analytic(Col sigma_a, Col sigma_s, const Ray& r, float t_max, float x0, float x1) {
    Col sigma_t = sigma_a + sigma_s;
    int c = sample_channel<Col>(x0);
    float sc = sigma_t[c];
    float t = sc == 0.0f ? t_max : -fm::log(1.0f - x1) / sc;
    MediumSampleT<Col> ms;
    if (t < t_max) {
        Col tr = vexp(-sigma_t * t);
        float pdf = spectrum_average(sigma_t * tr);
        ms.scattered = true;
        ms.t = t;
        ms.exit_p = r.o + r.d * t;
        ms.exit_dir = r.d;
        ms.weight = sigma_s * tr / fmaxf_(pdf, 1e-20f);
    } else {
        Col tr = vexp(-sigma_t * t_max);
        float pdf = spectrum_average(tr);
        ms.scattered = false;
        ms.t = t_max;
        ms.weight = tr / fmaxf_(pdf, 1e-20f);
    }
    return ms;
}
// hg (volume_scattering/hg/hg.glsl:11-42) — forward convention
inline float hg_eval(v3 wi, v3 wo, float g) {
    float c = dot(wi, -wo);
    float d = 1.0f + g * g - 2.0f * g * c;
    return (1.0f - g * g) / (4.0f * PI * d * std::sqrt(fmaxf_(d, 1e-8f)));
}
template <class Col> inline ISampleT<Col> hg_sample(v3 wo, float g, float x0, float x1) {
    float cos_theta;
    if (std::fabs(g) < 1e-3f) cos_theta = 1.0f - 2.0f * x0;
    else {
        float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * x0);
        cos_theta = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sin_theta = std::sqrt(fmaxf_(0.0f, 1.0f - cos_theta * cos_theta));
    float phi = TWO_PI * x1;
    v3 t, b;
    build_basis(-wo, t, b);
    ISampleT<Col> s;
    s.wi = normalize(t * (sin_theta * fm::cos(phi)) + b * (sin_theta * fm::sin(phi)) + (-wo) * cos_theta);
    s.weight = Col(1.0f);
    s.pdf = spectrum_average(Col(hg_eval(s.wi, wo, g)));
    s.flags = LOBE_MEDIUM;
    return s;
}

// ---------------------------------------------------------------- forward-mode duals
// FP64 dual numbers (value, derivative along one parameter) for the forward-mode reference
// of the path-replay adjoint (oracle_forward_tile).  The functions below are the BSDF,
// phase and Fresnel formulas of this file (same expressions, in float64), differentiated
// by the dual arithmetic itself: they check the adjoint's hand-derived log-derivatives.
struct Dual { double v, d; };
inline Dual dc(double v) { return {v, 0.0}; }
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
inline Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
inline Dual dsqrt(Dual a) { double r = std::sqrt(a.v); return {r, r > 0.0 ? a.d / (2.0 * r) : 0.0}; }
inline Dual dexp(Dual a) { double e = fm::exp(a.v); return {e, e * a.d}; }
constexpr double PI_D = 3.14159265359;   // the same constant as PI, in float64

// Trowbridge-Reitz D, separable Smith G1 (microfacet.glsl:22-54) with a dual alpha.
inline Dual mf_D_dual(double hz, Dual a) {
    Dual a2 = a * a;
    Dual t = hz * hz * (a2 - 1.0) + 1.0;
    return a2 / (PI_D * t * t);
}
inline Dual mf_G1_dual(double c, Dual a) {
    c = std::fabs(c);
    Dual a2 = a * a;
    return 2.0 * c / (c + dsqrt(a2 + (1.0 - a2) * c * c));
}
// The GGX conductor's f without its Fresnel factor (ggx.glsl:16-64), dual alpha.
inline Dual ggx_fs_dual(v3 wi, v3 wo, const Frame& f, Dual a) {
    const double wil[3] = {(double)dot(wi, f.t), (double)dot(wi, f.b), (double)dot(wi, f.n)};
    const double wol[3] = {(double)dot(wo, f.t), (double)dot(wo, f.b), (double)dot(wo, f.n)};
    if (wil[2] * wol[2] <= 0.0) return dc(0.0);
    double h[3] = {wil[0] + wol[0], wil[1] + wol[1], wil[2] + wol[2]};
    const double hl = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    const double hz = h[2] / hl;
    return mf_D_dual(hz, a) * mf_G1_dual(wil[2], a) * mf_G1_dual(wol[2], a) /
           (4.0 * std::fabs(wil[2]) * std::fabs(wol[2]));
}
// Henyey-Greenstein (hg.glsl:11-42, forward convention), dual g.
inline Dual hg_dual(v3 wi, v3 wo, Dual g) {
    const double c = (double)dot(wi, -wo);
    Dual d = 1.0 + g * g - 2.0 * g * c;
    Dual dd = d.v > 1e-8 ? d : dc(1e-8);
    return (1.0 - g * g) / (4.0 * PI_D * d * dsqrt(dd));
}
// Unpolarised dielectric Fresnel (math.glsl:95-102), dual relative IOR.
inline Dual fresnel_dual(double cos_i, Dual eta) {
    Dual sin2_t = eta * eta * (1.0 - cos_i * cos_i);
    if (sin2_t.v >= 1.0) return dc(1.0);
    Dual cos_t = dsqrt(1.0 - sin2_t);
    Dual r_par = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    Dual r_perp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5 * (r_par * r_par + r_perp * r_perp);
}

// ---------------------------------------------------------------- the renderer
struct Counters { uint64_t closest = 0, shadow = 0; };

// ---------------------------------------------------------------- spectral colour model
// spectral_curves (color/spectral/lookup.glsl:1-7): row 0 of the curve table, CIE x, y, z
// and luminance-normalised D65 per 5 nm from 360 nm, linearly interpolated.
inline void spectral_curves(const ptr_scene_desc& d, float lambda, float out[4]) {
    float x = (lambda - 360.0f) / 5.0f;
    int i = (int)x;
    i = i < 93 ? i : 93;
    const float* a = d.spectral->curves + 4 * i;
    const float* b = a + 4;
    float f = x - (float)i;
    for (int k = 0; k < 4; ++k) out[k] = a[k] * (1.0f - f) + b[k] * f;
}
// One lane of a lifted colour record: the bounded sigmoid of spectral_bounded
// (lookup.glsl:38-48) over the record's host-fitted coefficients, times its scale
// (color_lift_coefficient, :52-56); Planck relative to 550 nm (blackbody.glsl:4-10);
// or a grey constant; then D65 for emission (color_lift_emission, :57-61).
inline float spectrum_lane(const ptr_scene_desc& d, const ptr_spectrum& sp, float lambda) {
    float v;
    if (sp.kind == PTR_SPEC_LIFTED) {
        float t = (lambda - 360.0f) / 470.0f;
        float p = (sp.c[0] * t + sp.c[1]) * t + sp.c[2];
        v = clampf(0.5f + 0.5f * p / std::sqrt(1.0f + p * p), 0.0f, 1.0f);
        v = sp.scale * v;
    } else if (sp.kind == PTR_SPEC_BLACKBODY) {
        float q = 14387768.775039338f / sp.c[0];
        float ratio = 550.0f / lambda;
        float ratio2 = ratio * ratio;
        v = sp.c[1] * (fm::exp(q / 550.0f) - 1.0f) * ratio2 * ratio2 * ratio / (fm::exp(q / lambda) - 1.0f);
        v = sp.scale * v;
    } else {
        v = sp.scale;
    }
    if (sp.d65) {
        float c[4];
        spectral_curves(d, lambda, c);
        v = v * c[3];
    }
    return v;
}
// wavelengths_sample (color/spectral/spectral.glsl:1-10): one number, four cyclic quarter
// offsets in CDF space, each lane with its own density: the truncated sech^2 of
// visible.glsl:3-13 or uniform.glsl:1-2, over the program's range.
inline void wavelengths_sample(const ptr_program_desc& P, float u, float lam[4], float pdf[4]) {
    for (int k = 0; k < 4; ++k) {
        float v = u + 0.25f * (float)k;
        v = v - std::floor(v);
        if (P.wavelengths == PTR_WAVELENGTHS_UNIFORM) {
            lam[k] = P.lambda_min + (P.lambda_max - P.lambda_min) * v;
            pdf[k] = 1.0f / (P.lambda_max - P.lambda_min);
        } else {
            float a = fm::tanh(0.0072f * (P.lambda_min - 538.0f));
            float b = fm::tanh(0.0072f * (P.lambda_max - 538.0f));
            lam[k] = 538.0f + fm::atanh(a * (1.0f - v) + b * v) / 0.0072f;
            float c = fm::cosh(0.0072f * (lam[k] - 538.0f));
            pdf[k] = 0.0072f / ((b - a) * c * c);
        }
    }
}
// color_to_pixel (spectral.glsl:27-33) with the CIE 1931 sensor (sensor/cie1931/cie1931.glsl:3-5):
// 0.25 * sum_i (M xyz(lambda_i) / int ybar) (L_i / pdf_i).
inline v3 color_to_pixel(const ptr_scene_desc& d, s4 L, const float lam[4], const float pdf[4]) {
    const float* M = d.spectral->xyz_to_rgb;
    v3 pixel(0.0f);
    for (int k = 0; k < 4; ++k) {
        float c[4];
        spectral_curves(d, lam[k], c);
        v3 rgb(M[0] * c[0] + M[1] * c[1] + M[2] * c[2], M[3] * c[0] + M[4] * c[1] + M[5] * c[2],
               M[6] * c[0] + M[7] * c[1] + M[8] * c[2]);
        pixel = pixel + rgb / d.spectral->cie_y_integral * (L[k] / pdf[k]);
    }
    return 0.25f * pixel;
}

// The walk, generic over the colour carrier: v3 (RGB) or s4 (four wavelength lanes of
// measurement.color 'spectral').  Colours of materials, lights and the environment come
// from the colour accessors below: the RGB records, or the spectral records evaluated at
// the path's wavelengths.
template <class Col>
struct TracerT {
    static constexpr bool SPECTRAL = std::is_same<Col, s4>::value;
    using LS = LightSampleT<Col>;
    using IS = ISampleT<Col>;
    using MS = MediumSampleT<Col>;
    const Scene& S;
    const ptr_scene_desc& d;
    const ptr_program_desc& P;
    Rng rng;
    Counters cnt;
    float wl[4] = {0.f, 0.f, 0.f, 0.f};   // the path's wavelengths (spectral only)
    TracerT(const Scene& s) : S(s), d(*s.d), P(*s.prog) {}

    // ---- colour accessors (RGB records; or color/spectral/lookup.glsl:38-59 and
    // spectra/blackbody/blackbody.glsl:4-10 over the lifted records, per lane)
    Col spec(const ptr_spectrum& sp) const {
        if constexpr (SPECTRAL) {
            return s4(spectrum_lane(d, sp, wl[0]), spectrum_lane(d, sp, wl[1]), spectrum_lane(d, sp, wl[2]),
                      spectrum_lane(d, sp, wl[3]));
        } else {
            return Col(0.0f);
        }
    }
    Col c_albedo(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].albedo); else return ld3(d.materials[mi].albedo); }
    Col c_emission(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].emission); else return ld3(d.materials[mi].emission); }
    Col c_tint(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].transmittance); else return ld3(d.materials[mi].transmittance); }
    Col c_f0(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].f0); else return ld3(d.materials[mi].f0); }
    Col c_sigma_a(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].sigma_a); else return ld3(d.materials[mi].sigma_a); }
    Col c_sigma_s(int mi) const { if constexpr (SPECTRAL) return spec(d.spectral->materials[mi].sigma_s); else return ld3(d.materials[mi].sigma_s); }
    Col c_light(int li) const { if constexpr (SPECTRAL) return spec(d.spectral->lights[li]); else return ld3(d.lights[li].radiance); }
    Col c_env() const { if constexpr (SPECTRAL) return spec(d.spectral->env); else return ld3(d.env.color); }
    int mat_index(const ptr_material& m) const { return (int)(&m - d.materials); }

    // ---- forward-mode tangents (oracle_forward_tile only; null in the plain renders, whose
    // float32 walk they never touch).  d throughput / d theta_k and d radiance / d theta_k
    // per channel in float64, k = PTR_GRAD_SLOTS * material + slot, stored at [3 k + c].
    // The estimator differentiated is the adjoint's: sampled directions and distances,
    // sampling densities, MIS weights and roulette probabilities are held fixed (detached),
    // and each weight site contributes the derivative of its own formula.
    struct Tan { int K = 0; std::vector<double> thr, rad; };
    Tan* tan = nullptr;
    struct DW { int k; double d[3]; };   // one parameter's derivative of a weight, per channel
    static constexpr int kMaxDW = 16;
    int slot_k(int mat, int slot) const { return PTR_GRAD_SLOTS * mat + slot; }
    void tan_reset() {
        std::fill(tan->thr.begin(), tan->thr.end(), 0.0);
        std::fill(tan->rad.begin(), tan->rad.end(), 0.0);
    }
    // throughput <- throughput * W:  d thr = d thr * W + thr * dW
    void tan_mul(Col thr, Col W, const DW* dw, int n) {
        if (!tan) return;
        for (int k = 0; k < tan->K; ++k)
            for (int c = 0; c < 3; ++c) tan->thr[3 * k + c] *= (double)W[c];
        for (int j = 0; j < n; ++j)
            for (int c = 0; c < 3; ++c) tan->thr[3 * dw[j].k + c] += (double)thr[c] * dw[j].d[c];
    }
    // radiance += throughput * X:  d rad += d thr * X + thr * dX
    void tan_add(Col thr, Col X, const DW* dw, int n) {
        if (!tan) return;
        for (int k = 0; k < tan->K; ++k)
            for (int c = 0; c < 3; ++c) tan->rad[3 * k + c] += tan->thr[3 * k + c] * (double)X[c];
        for (int j = 0; j < n; ++j)
            for (int c = 0; c < 3; ++c) tan->rad[3 * dw[j].k + c] += (double)thr[c] * dw[j].d[c];
    }
    // grey homogeneous medium parameters (channel 0): sigma_t and the albedo a
    void grey_params(int med, double& st, double& a) const {
        const ptr_material& m = d.materials[med];
        st = (double)m.sigma_a[0] + (double)m.sigma_s[0];
        a = st > 0.0 ? (double)m.sigma_s[0] / st : 0.0;
    }
    // the dielectric IOR parameter a region's IOR follows, or -1
    int ior_param(int region) const {
        if (region < 0) return -1;
        const int m = d.regions[region].material;
        return (m >= 0 && d.materials[m].model == PTR_MAT_DIELECTRIC) ? slot_k(m, PTR_GRAD_IOR) : -1;
    }
    // the per-parameter derivatives X dlog_k of X from its log-derivatives, appended at n
    static int dw_from_dlog(Col X, const std::vector<std::pair<int, double>>& dlog, std::vector<DW>& out, int n) {
        if (out.size() < (size_t)n + dlog.size()) out.resize((size_t)n + dlog.size());
        for (const auto& e : dlog) {
            out[n].k = e.first;
            for (int c = 0; c < 3; ++c) out[n].d[c] = (double)X[c] * e.second;
            ++n;
        }
        return n;
    }

    bool intersect(const Ray& r, Hit& h) { cnt.closest++; return S.scene_intersect(r, h); }

    // ---- environment (features/environment.ts:109-252): constant env (T3 uniform sphere)
    // or an equirect table read through equirect_uv (env/equirect/equirect_map.glsl:15-21,
    // bilinear, wrap u, clamp v) and sampled by env/sampler_cdf.glsl:13-84.
    void equirect_uv(v3 dir, float& u, float& v) const {
        v3 n = normalize(dir);
        float phi = (n.x == 0.0f && n.z == 0.0f ? 0.0f : fm::atan2(n.z, n.x)) + d.env.rotation;
        float theta = fm::atan2(std::sqrt(n.x * n.x + n.z * n.z), n.y);
        u = phi * (1.0f / TWO_PI) + 0.5f;
        u = u - std::floor(u);
        v = theta * (1.0f / PI);
    }
    v3 env_texel(int i, int j) const {
        const float* p = d.env.radiance + 4 * ((size_t)j * d.env.width + i);
        return v3(p[0], p[1], p[2]);
    }
    Col environment_radiance(v3 dir) const {
        if (d.env.kind == PTR_ENV_CONSTANT) return c_env() * d.env.intensity;
        if constexpr (SPECTRAL) return Col(0.0f);   // spectral programs take constant environments only
        else return image_radiance(dir);
    }
    v3 image_radiance(v3 dir) const {
        if (d.env.kind != PTR_ENV_IMAGE) return v3(0.0f);
        const int W = d.env.width, H = d.env.height;
        float u, v;
        equirect_uv(dir, u, v);
        float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
        float fx0 = std::floor(x), fy0 = std::floor(y);
        float ax = x - fx0, ay = y - fy0;
        int i0 = (int)fx0, j0 = (int)fy0, i1 = i0 + 1, j1 = j0 + 1;
        i0 = ((i0 % W) + W) % W;
        i1 = ((i1 % W) + W) % W;
        j0 = std::min(std::max(j0, 0), H - 1);
        j1 = std::min(std::max(j1, 0), H - 1);
        v3 top = env_texel(i0, j0) * (1.0f - ax) + env_texel(i1, j0) * ax;
        v3 bot = env_texel(i0, j1) * (1.0f - ax) + env_texel(i1, j1) * ax;
        return (top * (1.0f - ay) + bot * ay) * d.env.intensity;
    }
    float marg(int j) const { return d.env.marginal[j]; }
    float cond(int j, int i) const { return d.env.conditional[(size_t)j * d.env.width + i]; }
    float uniform_fraction() const { return marg(d.env.height - 1) > 0.0f ? 0.0625f : 1.0f; }
    float table_pdf(v3 dir) const {
        const int W = d.env.width, H = d.env.height;
        float u, v;
        equirect_uv(dir, u, v);
        int i = std::min(std::max((int)(u * (float)W), 0), W - 1);
        int j = std::min(std::max((int)(v * (float)H), 0), H - 1);
        float dm = marg(j) - (j > 0 ? marg(j - 1) : 0.0f);
        float dc = cond(j, i) - (i > 0 ? cond(j, i - 1) : 0.0f);
        float theta = PI * ((float)j + 0.5f) / (float)H;
        float domega = (TWO_PI / (float)W) * 2.0f * fm::sin(theta) * fm::sin(0.5f * PI / (float)H);
        return (dc * dm) / domega;
    }
    v3 sample_table(float x0, float x1) const {
        const int W = d.env.width, H = d.env.height;
        int lo = 0, hi = H - 1;
        while (lo < hi) { int mid = (lo + hi) >> 1; if (x0 >= marg(mid)) lo = mid + 1; else hi = mid; }
        int j = lo;
        float mlo = j > 0 ? marg(j - 1) : 0.0f;
        float dm = marg(j) - mlo;
        float vf = dm > 0.0f ? clampf((x0 - mlo) / dm, 0.0f, 0.9999999f) : 0.5f;
        lo = 0; hi = W - 1;
        while (lo < hi) { int mid = (lo + hi) >> 1; if (x1 >= cond(j, mid)) lo = mid + 1; else hi = mid; }
        int i = lo;
        float clo = i > 0 ? cond(j, i - 1) : 0.0f;
        float dc = cond(j, i) - clo;
        float uf = dc > 0.0f ? clampf((x1 - clo) / dc, 0.0f, 0.9999999f) : 0.5f;
        float phi = (((float)i + uf) / (float)W - 0.5f) * TWO_PI - d.env.rotation;
        bool north = 2 * j < H;
        float row = north ? (float)j : (float)(H - j - 1);
        float a = fm::sin(0.5f * PI * row / (float)H);
        float b = fm::sin(0.5f * PI * (row + 1.0f) / (float)H);
        float tt = north ? vf : 1.0f - vf;
        float h = (a * a) * (1.0f - tt) + (b * b) * tt;
        float y = (north ? 1.0f : -1.0f) * (1.0f - 2.0f * h);
        float rr = 2.0f * std::sqrt(h * (1.0f - h));
        return v3(rr * fm::cos(phi), y, rr * fm::sin(phi));
    }
    LS environment_sample(float x0, float x1) const {
        LS ls;
        if (d.env.kind == PTR_ENV_IMAGE) {
            float a = uniform_fraction();
            if (x0 < a) {
                float y = 1.0f - 2.0f * (x0 / a);
                float r = std::sqrt(fmaxf_(0.0f, 1.0f - y * y));
                float phi = TWO_PI * x1;
                ls.wi = v3(r * fm::cos(phi), y, r * fm::sin(phi));
            } else {
                ls.wi = sample_table((x0 - a) / (1.0f - a), x1);
            }
            ls.distance = MAX_DIST;
            ls.radiance = environment_radiance(ls.wi);
            ls.pdf = environment_pdf(ls.wi);
            ls.flags = 0u;
            ls.light_id = -1;
            return ls;
        }
        float z = 1.0f - 2.0f * x0;
        float r = std::sqrt(fmaxf_(0.0f, 1.0f - z * z));
        float phi = TWO_PI * x1;
        ls.wi = v3(r * fm::cos(phi), z, r * fm::sin(phi));
        ls.distance = MAX_DIST;
        ls.radiance = c_env() * d.env.intensity;
        ls.pdf = 1.0f / (4.0f * PI);
        ls.flags = 0u;
        ls.light_id = -1;
        return ls;
    }
    float environment_pdf(v3 dir) const {
        if (d.env.kind != PTR_ENV_IMAGE) return 1.0f / (4.0f * PI);
        float a = uniform_fraction();
        return (1.0f - a) * table_pdf(dir) + a / (4.0f * PI);
    }

    // ---- lights (lights/quad/quad.glsl:14-41, sphere/sphere.glsl:21-71, point/point.glsl:11-23,
    // mesh/mesh.glsl:18-75)
    // mesh light point: binary search for the smallest triangle whose cumulative area
    // exceeds x0, x0 rescaled within its span, the square-root map; n = unit winding normal
    v3 mesh_light_point(const ptr_light& l, float x0, float x1, v3& n) const {
        const OMesh& m = S.meshes[(int)l.p[0]];
        int lo = 0, hi = (int)m.light_cdf.size() - 1;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (m.light_cdf[mid] <= x0) lo = mid + 1;
            else hi = mid;
        }
        float c0 = lo > 0 ? m.light_cdf[lo - 1] : 0.0f;
        float c1 = m.light_cdf[lo];
        float xr = clampf((x0 - c0) / fmaxf_(c1 - c0, 1.0e-12f), 0.0f, 0.9999999f);
        v3 a = m.a[lo], b = m.pb[lo], c = m.pc[lo];
        float su = std::sqrt(xr);
        n = normalize(cross(b - a, c - a));
        return a * (1.0f - su) + b * (su * (1.0f - x1)) + c * (su * x1);
    }
    LS light_sample_one(const ptr_light& l, v3 p, float x0, float x1) const {
        LS ls;
        const int li = (int)(&l - d.lights);
        ls.radiance = c_light(li);
        ls.flags = 0u;
        ls.light_id = -1;
        if (l.kind == PTR_LIGHT_MESH) {   // radiance without falloff; one-sided
            v3 n;
            v3 q = mesh_light_point(l, x0, x1, n);
            v3 dd = q - p;
            float d2 = dot(dd, dd);
            ls.wi = dd * (1.0f / std::sqrt(d2));
            ls.distance = std::sqrt(d2);
            float cos_l = dot(n, -ls.wi);
            if (!(cos_l > 0.0f)) { ls.pdf = 0.0f; return ls; }
            ls.pdf = d2 / (l.p[12] * cos_l);
            return ls;
        }
        if (l.kind == PTR_LIGHT_QUAD) {
            v3 corner = ld3(l.p), e1 = ld3(l.p + 3), e2 = ld3(l.p + 6), nrm = ld3(l.p + 9);
            float area = l.p[12];
            v3 q = corner + x0 * e1 + x1 * e2;
            v3 dd = q - p;
            float d2 = dot(dd, dd);
            ls.wi = dd * (1.0f / std::sqrt(d2));
            ls.distance = std::sqrt(d2);
            float cos_l = dot(nrm, -ls.wi);
            if (cos_l <= 0.0f) { ls.pdf = 0.0f; return ls; }
            ls.pdf = d2 / (area * cos_l);
            return ls;
        }
        if (l.kind == PTR_LIGHT_SPHERE) {
            v3 c = ld3(l.p);
            float r = l.p[3];
            v3 to_c = c - p;
            float dc2 = dot(to_c, to_c);
            if (dc2 <= r * r) { ls.wi = v3(0, 1, 0); ls.distance = 1.0f; ls.pdf = 0.0f; return ls; }
            float sin2_max = r * r / dc2;
            float omc_max = sin2_max / (1.0f + std::sqrt(fmaxf_(0.0f, 1.0f - sin2_max)));
            float w_t = x0 * omc_max;
            float cos_t = 1.0f - w_t;
            float sin_t = std::sqrt(fmaxf_(0.0f, w_t * (2.0f - w_t)));
            float phi = TWO_PI * x1;
            v3 w = to_c * (1.0f / std::sqrt(dc2));
            v3 t, b;
            build_basis(w, t, b);
            ls.wi = normalize(t * (sin_t * fm::cos(phi)) + b * (sin_t * fm::sin(phi)) + w * cos_t);
            ls.pdf = 1.0f / (TWO_PI * omc_max);
            float proj = dot(to_c, ls.wi);
            v3 perp = to_c - proj * ls.wi;
            float disc = fmaxf_(0.0f, r * r - dot(perp, perp));
            ls.distance = (dc2 - r * r) / (proj + std::sqrt(disc));
            return ls;
        }
        // point (delta): radiance = I / d^2 folded in, pdf 1 (point.glsl:11-23)
        v3 pos = ld3(l.p);
        v3 dd = pos - p;
        float d2 = dot(dd, dd);
        ls.wi = dd * (1.0f / std::sqrt(d2));
        ls.distance = std::sqrt(d2);
        ls.radiance = c_light(li) / d2;
        ls.pdf = 1.0f;
        ls.flags = LIGHT_DELTA;
        return ls;
    }
    float light_pdf_one(const ptr_light& l, v3 p, v3 light_p, v3 light_n, v3 wi) const {
        if (l.kind == PTR_LIGHT_MESH) {   // d^2 / (A cos_l) whichever triangle was hit
            float cos_l = dot(light_n, -wi);
            if (cos_l <= 0.0f) return 0.0f;
            v3 dd = light_p - p;
            return dot(dd, dd) / (l.p[12] * cos_l);
        }
        if (l.kind == PTR_LIGHT_QUAD) {
            float cos_l = dot(ld3(l.p + 9), -wi);
            if (cos_l <= 0.0f) return 0.0f;
            v3 dd = light_p - p;
            return dot(dd, dd) / (l.p[12] * cos_l);
        }
        if (l.kind == PTR_LIGHT_SPHERE) {
            v3 to_c = ld3(l.p) - p;
            float dc2 = dot(to_c, to_c);
            float r = l.p[3];
            if (dc2 <= r * r) return 0.0f;
            float sin2_max = r * r / dc2;
            float omc = sin2_max / (1.0f + std::sqrt(fmaxf_(0.0f, 1.0f - sin2_max)));
            return 1.0f / (TWO_PI * omc);
        }
        return 0.0f;
    }
    // lighting_sample_finite: power CDF + cdf_rescale (features/lighting.ts:546-637)
    LS lighting_sample_finite(v3 p, float x0, float x1) const {
        LS ls;
        if (d.n_lights == 1) {
            ls = light_sample_one(d.lights[0], p, x0, x1);
            ls.light_id = 0;
            return ls;
        }
        int id = d.n_lights - 1;
        for (int i = 0; i < d.n_lights - 1; ++i)
            if (x0 < d.lights[i].select_cdf) { id = i; break; }
        float lo = id == 0 ? 0.0f : d.lights[id - 1].select_cdf;
        float sel = d.lights[id].select_pdf;
        float xr = (x0 - lo) / sel;
        ls = light_sample_one(d.lights[id], p, clampf(xr, 0.0f, 0.9999999f), x1);
        ls.light_id = id;
        ls.pdf *= sel;
        return ls;
    }
    // ---- light-tree selection (accel/light_tree/light_tree.glsl:28-77; the walk pair of
    // features/lighting.ts:767-824).  Query: receiving point, shading normal (0 at a medium
    // event), two-sided receiver (rough dielectric: no below-horizon cull).
    struct Query { v3 p, n; bool two_sided; };
    static float tree_importance(v3 bmin, v3 bmax, float phi, const Query& q) {
        v3 c = 0.5f * (bmin + bmax);
        v3 e = bmax - bmin;
        v3 dd = c - q.p;
        float d2raw = dot(dd, dd);
        float diag2 = 0.25f * dot(e, e);
        float base = phi / fmaxf_(d2raw, fmaxf_(diag2, 1e-8f));
        if (dot(q.n, q.n) < 0.5f) return base;
        v3 far_c(q.n.x >= 0.0f ? bmax.x : bmin.x, q.n.y >= 0.0f ? bmax.y : bmin.y, q.n.z >= 0.0f ? bmax.z : bmin.z);
        float h = dot(q.n, far_c - q.p);
        if (q.two_sided) {
            v3 near_c = bmin + bmax - far_c;
            h = fmaxf_(h, -dot(q.n, near_c - q.p));
        } else if (h <= 0.0f) {
            return 0.0f;
        }
        float cos_c = dot(q.n, dd) * (1.0f / std::sqrt(fmaxf_(d2raw, 1e-12f)));
        if (q.two_sided) cos_c = std::fabs(cos_c);
        v3 a = q.p - bmin, b = bmax - q.p;
        v3 dmx(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z));
        float lo = h * (1.0f / std::sqrt(fmaxf_(dot(dmx, dmx), 1e-12f)));
        return base * fminf_(1.0f, fmaxf_(cos_c, lo));
    }
    // node i: (min.xyz, phi) at 8i, (max.xyz, link) at 8i + 4; p_l of the left child, or
    // -1 on a dead descent
    float tree_left(int ni, const Query& q, int& L, int& R) const {
        const float* T = d.light_tree;
        L = ni + 1;
        R = (int)T[8 * (size_t)ni + 7];
        float iw_l = tree_importance(ld3(T + 8 * (size_t)L), ld3(T + 8 * (size_t)L + 4), T[8 * (size_t)L + 3], q);
        float iw_r = tree_importance(ld3(T + 8 * (size_t)R), ld3(T + 8 * (size_t)R + 4), T[8 * (size_t)R + 3], q);
        float isum = iw_l + iw_r;
        if (!(isum > 0.0f)) return -1.0f;
        return iw_l / isum;
    }
    int tree_pick(const Query& q, float xi, float& pmf) {
        const float* T = d.light_tree;
        pmf = 1.0f;
        int ni = 0;
        for (int lvl = 0; lvl < 48 && T[8 * (size_t)ni + 7] >= 0.0f; ++lvl) {
            int L, R;
            float p_l = tree_left(ni, q, L, R);
            if (p_l < 0.0f) { pmf = 0.0f; return -1; }
            if (xi < p_l) { pmf *= p_l; ni = L; }
            else { pmf *= (1.0f - p_l); ni = R; }
            xi = rng.next();
        }
        if (T[8 * (size_t)ni + 7] >= 0.0f) { pmf = 0.0f; return -1; }
        return (int)(-T[8 * (size_t)ni + 7] - 1.0f);
    }
    float tree_pmf(const Query& q, int light) const {
        const float* T = d.light_tree;
        uint32_t tw = d.light_trails[2 * (size_t)light];
        float pmf = 1.0f;
        int ni = 0;
        for (int lvl = 0; lvl < 48 && T[8 * (size_t)ni + 7] >= 0.0f; ++lvl) {
            if (lvl == 24) tw = d.light_trails[2 * (size_t)light + 1];
            int L, R;
            float p_l = tree_left(ni, q, L, R);
            if (p_l < 0.0f) return 0.0f;
            if ((tw & 1u) == 0u) { pmf *= p_l; ni = L; }
            else { pmf *= (1.0f - p_l); ni = R; }
            tw >>= 1u;
        }
        return pmf;
    }
    LS lighting_sample_tree(const Query& q, float x0, float x1) {
        LS ls;
        float sel;
        int id = tree_pick(q, x0, sel);
        if (id < 0) { ls.pdf = 0.0f; return ls; }
        float lx = rng.next();
        ls = light_sample_one(d.lights[id], q.p, lx, x1);
        ls.light_id = id;
        ls.pdf *= sel;
        return ls;
    }

    // lighting_sample: two-stage env-vs-finite (features/lighting.ts generateLightSampling)
    LS lighting_sample(const Query& q, float x0, float x1) {
        if (d.n_lights == 0) {
            if (S.env_samplable) return environment_sample(x0, x1);
            LS ls; ls.pdf = 0.0f; return ls;
        }
        if (!S.env_select_live) return S.tree ? lighting_sample_tree(q, x0, x1) : lighting_sample_finite(q.p, x0, x1);
        float pe = d.env.select_prob;
        if (x0 < pe) {
            LS ls = environment_sample(clampf(x0 / pe, 0.0f, 0.9999999f), x1);
            ls.pdf *= pe;
            return ls;
        }
        float fx = clampf((x0 - pe) / (1.0f - pe), 0.0f, 0.9999999f);
        LS ls = S.tree ? lighting_sample_tree(q, fx, x1) : lighting_sample_finite(q.p, fx, x1);
        ls.pdf *= (1.0f - pe);
        return ls;
    }
    // lighting_pdf (features/lighting.ts:639-693, 903-940): q = the stored selection context
    float lighting_pdf(const Query& q, v3 wi, int lid, const Hit& lh) const {
        const ptr_light& l = d.lights[lid];
        float sel = S.tree ? tree_pmf(q, lid) : d.n_lights == 1 ? 1.0f : l.select_pdf;
        float pe = S.env_select_live ? (1.0f - d.env.select_prob) : 1.0f;
        return sel * pe * light_pdf_one(l, q.p, lh.p, lh.ng, wi);
    }
    // the light of an emitter hit: its region's, or an instance light of its batch
    int emitter_light(const Hit& hit) const {
        int lid = S.light_of_region[hit.region_to];
        if (lid < 0 && hit.region_to == hit.region_owner) {
            const ptr_region& g = d.regions[hit.region_owner];
            if (g.shape == PTR_SHAPE_INSTANCES && S.batch_light_base[g.ref] >= 0) lid = S.batch_light_base[g.ref] + hit.element;
        }
        return lid;
    }

    // ---- material dispatch (features/materials.ts:902-954)
    float hit_alpha = -1.0f;   // the current vertex's per-triangle alpha (mesh hits)
    float alpha_of(const ptr_material& m) const { return hit_alpha >= 0.0f ? hit_alpha : m.alpha; }
    IS surface_sample(const ptr_material& m, v3 wo, const Hit& h, float uc, float u0, float u1) const {
        const int mi = mat_index(m);
        if (m.model == PTR_MAT_LAMBERT) return lambert_sample(wo, h, c_albedo(mi), uc, u0, u1);
        if (m.model == PTR_MAT_GGX) return ggx_sample(wo, h, c_f0(mi), alpha_of(m), u0, u1);
        if (m.model == PTR_MAT_MIRROR) return mirror_sample(wo, h, c_f0(mi));
        if (m.model == PTR_MAT_ROUGH_DIELECTRIC) {
            IS s = rough_dielectric_sample_local(mf_to_local(h.frame, wo), c_tint(mi), alpha_of(m), S.ior_of(h.region_from),
                                                 S.ior_of(h.region_to), uc, u0, u1);
            if (spectrum_is_zero(s.weight) && !(s.flags & LOBE_DELTA)) s.wi = wo;
            else if (s.flags & LOBE_DELTA) s.wi = -wo;
            else s.wi = mf_from_local(h.frame, s.wi);
            return s;
        }
        // dielectric (materials/dielectric/dielectric.glsl:14-52)
        float n_i = S.ior_of(h.region_from), n_t = S.ior_of(h.region_to);
        float eta = n_i / n_t;
        v3 n = h.frame.n;
        float cos_i = clampf(dot(wo, n), 1e-6f, 1.0f);
        float F = dielectric_fresnel(cos_i, eta);
        IS s;
        if (uc < F) {
            s.wi = normalize(2.0f * cos_i * n - wo);
            s.weight = Col(1.0f);
            s.pdf = 0.0f;
            s.flags = LOBE_REFLECTION | LOBE_DELTA;
        } else {
            float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
            float cos_t = std::sqrt(fmaxf_(0.0f, 1.0f - sin2_t));
            s.wi = normalize(-eta * wo + (eta * cos_i - cos_t) * n);
            float radiance_scale = (n_i * n_i) / (n_t * n_t);
            s.weight = c_tint(mi) * radiance_scale;
            s.pdf = 0.0f;
            s.flags = LOBE_TRANSMISSION | LOBE_DELTA;
        }
        return s;
    }
    Col surface_eval(const ptr_material& m, v3 wi, v3 wo, const Hit& h) const {
        const int mi = mat_index(m);
        if (m.model == PTR_MAT_LAMBERT) return lambert_eval(wi, wo, h, c_albedo(mi));
        if (m.model == PTR_MAT_GGX) return ggx_eval(wi, wo, h, c_f0(mi), alpha_of(m));
        if (m.model == PTR_MAT_ROUGH_DIELECTRIC)
            return rough_dielectric_eval_local(mf_to_local(h.frame, wi), mf_to_local(h.frame, wo), c_tint(mi), alpha_of(m),
                                               S.ior_of(h.region_from), S.ior_of(h.region_to));
        return Col(0.0f);
    }
    float surface_pdf(const ptr_material& m, v3 wi, v3 wo, const Hit& h) const {
        if (m.model == PTR_MAT_LAMBERT) return lambert_pdf(wi, wo, h);
        if (m.model == PTR_MAT_GGX) return ggx_pdf(wi, wo, h, alpha_of(m));
        if (m.model == PTR_MAT_ROUGH_DIELECTRIC)
            return rough_dielectric_pdf_local(mf_to_local(h.frame, wi), mf_to_local(h.frame, wo), alpha_of(m),
                                              S.ior_of(h.region_from), S.ior_of(h.region_to));
        return 0.0f;
    }

    // ---- media dispatch (features/materials.ts:675-866)
    // a medium scatters when it has sigma_s and measurement.scattering is 'full'
    bool scatter_live(int med) const { return P.scattering && (d.materials[med].flags & PTR_MATF_SCATTERING); }
    // medium_transmittance (analytic.glsl:49-51): Beer-Lambert over sigma_t; under
    // scattering 'ignored' the medium is absorbing-only (sigma_t = sigma_a)
    Col medium_transmittance(int med, float len) const {
        Col st = scatter_live(med) ? c_sigma_a(med) + c_sigma_s(med) : c_sigma_a(med);
        return vexp(-st * len);
    }
    // ---- heterogeneous media: the D1-clamped fields and the tracking arms
    bool is_het(int med) const { return d.materials[med].field_a != 0 || d.materials[med].field_s != 0; }
    void het_props(const ptr_material& m, v3 p, v3& sa, v3& ss) const {
        sa = m.field_a ? field_eval(d.field_code + (m.field_a - 1), p) : ld3(m.sigma_a);
        ss = m.field_s ? field_eval(d.field_code + (m.field_s - 1), p) : ld3(m.sigma_s);
        v3 st = sa + ss;
        float smax = fmaxf_(st.x, fmaxf_(st.y, st.z));
        float scale = smax > m.majorant ? m.majorant / smax : 1.0f;
        sa = sa * scale;
        ss = ss * scale;
    }
    static int tracking_cap(float lambda) { return (int)std::ceil(lambda + 6.5f * std::sqrt(lambda) + 12.0f); }
    // delta tracking (Kutz et al. 2017, Algorithm 4; average-based probabilities)
    MediumSample medium_sample_delta(const ptr_material& m, const Ray& r, float t_max, float x0, float x1) {
        MediumSample ms;
        ms.scattered = false;
        ms.t = t_max;
        const float sbar = m.majorant;
        v3 w(1.0f);
        float t = 0.0f, xd = x0, xe = x1;
        const int cap = tracking_cap(sbar * t_max);
        for (int i = 0; i < cap; ++i) {
            t += -fm::log(1.0f - xd) / sbar;
            if (t >= t_max) { ms.weight = w; return ms; }
            v3 p = r.o + r.d * t;
            v3 sa, ss;
            het_props(m, p, sa, ss);
            v3 sn = vmax(v3(sbar) - (sa + ss), v3(0.0f));
            float pa = spectrum_average(sa * w);
            float ps = spectrum_average(ss * w);
            float pn = spectrum_average(sn * w);
            float c = pa + ps + pn;
            if (c <= 0.0f) { ms.weight = v3(0.0f); return ms; }
            pa /= c; ps /= c; pn /= c;
            if (xe < pa) { ms.weight = v3(0.0f); return ms; }
            if (xe < pa + ps) {
                ms.scattered = true;
                ms.t = t;
                ms.exit_p = p;
                ms.exit_dir = r.d;
                ms.weight = w * ss / (sbar * fmaxf_(ps, 1e-20f));
                return ms;
            }
            w = w * sn / (sbar * fmaxf_(pn, 1e-20f));
            xd = rng.next();
            xe = rng.next();
        }
        ms.weight = w;
        return ms;
    }
    // ratio tracking (Novak et al. 2014): sigma_a for the pass-through arm, sigma_t with
    // pbrt's roulette for shadow segments
    v3 medium_ratio_track(const ptr_material& m, const Ray& r, float len, Rng& g, bool extinction) const {
        const float sbar = m.majorant;
        v3 T(1.0f);
        float t = 0.0f;
        const int cap = tracking_cap(sbar * len);
        for (int i = 0; i < cap; ++i) {
            t += -fm::log(1.0f - g.next()) / sbar;
            if (t >= len) return T;
            v3 sa, ss;
            het_props(m, r.o + r.d * t, sa, ss);
            T = T * (vmax(v3(sbar) - (extinction ? sa + ss : sa), v3(0.0f)) / sbar);
            if (extinction && spectrum_max(T) < 0.05f) {
                if (g.next() < 0.75f) return v3(0.0f);
                T = T / 0.25f;
            }
        }
        return T;
    }
    uint32_t shadow_seed = 0;   // the path's sampler dimension at the current NEE site

    Col medium_survival(int med) const {
        Col sa = c_sigma_a(med), ss = c_sigma_s(med);
        return ss / vmax(ss + sa, Col(1e-9f));
    }

    // shadow_transmittance: opaque (transport/shadow/opaque/opaque.glsl:16-19) or the
    // media segment walker (transport/shadow/media/media.glsl:29-62)
    // dlog (forward mode): d log T / d theta_k of every medium segment crossed, appended
    Col shadow_transmittance(Ray sr, v3 light_p, int crossings_left, std::vector<std::pair<int, double>>* dlog = nullptr) {
        cnt.shadow++;
        if (!S.has_media) {
            float maxDist = length(light_p - sr.o) - SHADOW_BACKOFF;
            return S.scene_intersect_any(sr, maxDist) ? Col(0.0f) : Col(1.0f);
        }
        Col T(1.0f);
        int medium = S.scene_region_at(sr.o);
        Ray seg = sr;
        Rng srng;
        bool srng_live = false;
        for (int crossed = 0; crossed <= crossings_left; crossed++) {
            float remaining = length(light_p - seg.o) - SHADOW_BACKOFF;
            if (remaining <= 0.0f) return T;
            Hit h;
            bool hit_boundary = S.scene_intersect(seg, h) && h.t < remaining;
            float seg_len = hit_boundary ? h.t : remaining;
            int med_mat = S.material_of(medium);
            if (S.material_has_medium(med_mat) && !SPECTRAL && is_het(med_mat)) {
                if (!srng_live) { srng = shadow_rng(rng.base, shadow_seed); srng_live = true; }
                if constexpr (!SPECTRAL) T = T * medium_ratio_track(d.materials[med_mat], seg, seg_len, srng, scatter_live(med_mat));
            } else if (S.material_has_medium(med_mat)) {
                T = T * medium_transmittance(med_mat, seg_len);
                if (dlog) {   // T_seg = exp(-sigma len), sigma = st (scattering) or (1 - a) st
                    double st, a;
                    grey_params(med_mat, st, a);
                    if (scatter_live(med_mat)) {
                        dlog->push_back({slot_k(med_mat, PTR_GRAD_SIGMA_T), -(double)seg_len});
                    } else {
                        dlog->push_back({slot_k(med_mat, PTR_GRAD_SIGMA_T), -(1.0 - a) * (double)seg_len});
                        dlog->push_back({slot_k(med_mat, PTR_GRAD_MEDIUM_ALBEDO), st * (double)seg_len});
                    }
                }
            }
            if (!hit_boundary) return T;
            if (!S.is_null_interface(S.material_of(h.region_owner))) return Col(0.0f);
            medium = h.region_to;
            seg = ray_spawn(h, seg.d);
            seg.d = normalize(light_p - seg.o);
        }
        return Col(0.0f);
    }

    static float power_heuristic(float pf, float pg) {
        float f2 = pf * pf;
        if (f2 >= 1.0e38f) return 1.0f;
        return f2 / fmaxf_(1e-20f, f2 + pg * pg);
    }

    // ---- equiangular medium NEE, one estimate per medium segment with segment-start
    // throughput (transport/techniques/equiangular/equiangular.glsl:18-57; Kulla & Fajardo
    // 2012).  The light is picked by the lighting CDF (lighting_query_delta,
    // features/lighting.ts:303-341): a delta light gives its position and intensity as in
    // the reference.  Area lights (quad, sphere) are an extension the reference's
    // Validator rejects: a uniform point on the light's area is drawn first (two more
    // numbers), the estimate then carries Le * cos_l / (d^2 * pdf_area).
    void equiangular_sample_direct(const Ray& r, int med_mat, float t_max, Col thr, Col& radiance, int crossings_left) {
        const ptr_material& mm = d.materials[med_mat];
        float uc = rng.next();
        int id = d.n_lights - 1;
        if (d.n_lights > 1)
            for (int i = 0; i < d.n_lights - 1; ++i)
                if (uc < d.lights[i].select_cdf) { id = i; break; }
        const ptr_light& l = d.lights[id];
        const float sel = d.n_lights == 1 ? 1.0f : l.select_pdf;
        v3 pos, nl(0.0f);
        float pdf_area = 1.0f;
        const bool area = l.kind != PTR_LIGHT_POINT;
        if (area) {
            float y0 = rng.next(), y1 = rng.next();
            if (l.kind == PTR_LIGHT_QUAD) {
                pos = ld3(l.p) + y0 * ld3(l.p + 3) + y1 * ld3(l.p + 6);
                nl = ld3(l.p + 9);
                pdf_area = 1.0f / l.p[12];
            } else if (l.kind == PTR_LIGHT_MESH) {
                pos = mesh_light_point(l, y0, y1, nl);
                pdf_area = 1.0f / l.p[12];
            } else {
                float z = 1.0f - 2.0f * y0;
                float rr = std::sqrt(fmaxf_(0.0f, 1.0f - z * z));
                float phi = TWO_PI * y1;
                nl = v3(rr * fm::cos(phi), z, rr * fm::sin(phi));
                pos = ld3(l.p) + nl * l.p[3];
                pdf_area = 1.0f / (4.0f * PI * l.p[3] * l.p[3]);
            }
        } else {
            pos = ld3(l.p);
        }
        // the light's frame over the segment: closest approach t_c, perpendicular h
        v3 D = pos - r.o;
        float t_c = dot(D, r.d);
        float h2 = fmaxf_(dot(D, D) - t_c * t_c, 1e-8f);
        float h = std::sqrt(h2);
        float theta_a = fm::atan2(0.0f - t_c, h);
        float theta_b = fm::atan2(t_max - t_c, h);
        float u = rng.next();
        float theta = theta_a * (1.0f - u) + theta_b * u;
        float t = t_c + h * fm::tan(theta);
        float pdf_t = h / ((theta_b - theta_a) * (h2 + (t - t_c) * (t - t_c)));
        v3 p_evt = r.o + r.d * t;
        Col sigma_s = c_sigma_s(med_mat);
        if (spectrum_is_black(sigma_s)) return;
        Col T_seg = vexp(-(c_sigma_a(med_mat) + sigma_s) * t);
        v3 to_light = pos - p_evt;
        float d2 = fmaxf_(dot(to_light, to_light), 1e-8f);
        float dist = std::sqrt(d2);
        v3 wi = to_light / dist;
        Col Le;
        float denom;
        if (area) {
            float cos_l = dot(nl, -wi);
            if (!(cos_l > 0.0f)) return;
            Le = c_light(id) * (cos_l / d2);
            denom = pdf_t * (pdf_area * sel);
        } else {
            Le = c_light(id) / d2;
            denom = pdf_t * sel;
        }
        Col vis = shadow_transmittance(Ray{p_evt, wi}, pos, crossings_left);
        if (spectrum_is_black(vis)) return;
        Col ph(hg_eval(wi, -r.d, mm.phase_g));
        radiance = radiance + thr * T_seg * sigma_s * ph * Le * vis / denom;
    }

    // d w_c / d F0_c of a weight w_c = F_c(F0_c) x (terms free of F0), Schlick's F at cosine c:
    // w_c (1 - (1 - c)^5) / F_c, one entry per channel, appended at n.
    int dw_schlick_f0(int mat, const ptr_material& m, double c, Col w, DW* dw, int n) const {
        const double s5 = fm::pow(1.0 - c, 5.0);
        for (int ch = 0; ch < 3; ++ch) {
            const double F = (double)m.f0[ch] + (1.0 - (double)m.f0[ch]) * s5;
            dw[n].k = slot_k(mat, PTR_GRAD_COLOR_R + ch);
            dw[n].d[0] = dw[n].d[1] = dw[n].d[2] = 0.0;
            dw[n].d[ch] = F > 0.0 ? (double)w[ch] * (1.0 - s5) / F : 0.0;
            ++n;
        }
        return n;
    }
    // the cosine Schlick's F of the GGX conductor sees for the pair (wi, wo)
    static double ggx_fresnel_cos(v3 wi, v3 wo, const Hit& h) {
        v3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
        v3 hh = normalize(wil + wol);
        return (double)std::fabs(dot(wol, hh));
    }

    // The continuation lobe's weight derivative (forward mode).  Lambert: w = albedo.
    // GGX: w = F(F0) fs(alpha) cos / pdf with the pdf detached, so dw = w d log F(F0)
    // per channel and w d log fs(alpha).  Mirror: w = F(F0).  Dielectric:
    // w = F / F_detached (reflection) or T (n_i / n_t)^2 (1 - F) / (1 - F)_detached
    // (refraction), differentiated along the IORs of the two regions the interface joins,
    // and along the transmittance T on refraction.
    void tan_continuation(const ptr_material& m, int mat, v3 wo, const Hit& hit, const IS& bs, Col thr, DW* dw) {
        int n = 0;
        if (m.model == PTR_MAT_LAMBERT) {
            for (int c = 0; c < 3; ++c) {
                dw[n].k = slot_k(mat, PTR_GRAD_COLOR_R + c);
                dw[n].d[0] = dw[n].d[1] = dw[n].d[2] = 0.0;
                dw[n].d[c] = 1.0;
                ++n;
            }
        } else if (m.model == PTR_MAT_MIRROR) {
            n = dw_schlick_f0(mat, m, (double)clampf(dot(wo, hit.frame.n), 1e-6f, 1.0f), bs.weight, dw, n);
        } else if (m.model == PTR_MAT_GGX) {
            n = dw_schlick_f0(mat, m, ggx_fresnel_cos(bs.wi, wo, hit), bs.weight, dw, n);
            if (hit_alpha < 0.0f) {
                const Dual fs = ggx_fs_dual(bs.wi, wo, hit.frame, Dual{(double)m.alpha, 1.0});
                dw[n].k = slot_k(mat, PTR_GRAD_ALPHA);
                for (int c = 0; c < 3; ++c) dw[n].d[c] = fs.v > 0.0 ? (double)bs.weight[c] * fs.d / fs.v : 0.0;
                ++n;
            }
        } else if (m.model == PTR_MAT_DIELECTRIC) {
            const float n_i = S.ior_of(hit.region_from), n_t = S.ior_of(hit.region_to);
            const float cos_i = clampf(dot(wo, hit.frame.n), 1e-6f, 1.0f);
            const float F_det = dielectric_fresnel(cos_i, n_i / n_t);
            const int kf = ior_param(hit.region_from), kt = ior_param(hit.region_to);
            const int ks[2] = {kf, kt != kf ? kt : -1};
            for (int j = 0; j < 2; ++j) {
                if (ks[j] < 0) continue;
                const Dual ni{(double)n_i, ks[j] == kf ? 1.0 : 0.0}, nt{(double)n_t, ks[j] == kt ? 1.0 : 0.0};
                const Dual F = fresnel_dual((double)cos_i, ni / nt);
                dw[n].k = ks[j];
                if (bs.flags & LOBE_REFLECTION) {
                    for (int c = 0; c < 3; ++c) dw[n].d[c] = F.d / (double)F_det;
                } else {
                    const Dual scale = (ni * ni) / (nt * nt);
                    const double dd = (scale.d * (1.0 - F.v) - scale.v * F.d) / (1.0 - (double)F_det);
                    for (int c = 0; c < 3; ++c) dw[n].d[c] = (double)m.transmittance[c] * dd;
                }
                ++n;
            }
            if (bs.flags & LOBE_TRANSMISSION) {   // d w_c / d T_c = (n_i / n_t)^2
                const double scale = (double)((n_i * n_i) / (n_t * n_t));
                for (int c = 0; c < 3; ++c) {
                    dw[n].k = slot_k(mat, PTR_GRAD_COLOR_R + c);
                    dw[n].d[0] = dw[n].d[1] = dw[n].d[2] = 0.0;
                    dw[n].d[c] = scale;
                    ++n;
                }
            }
        }
        tan_mul(thr, bs.weight, dw, n);
    }

    // ---- the walk (transport/integrators/pt/pt.ts:299-464, as emitted for media scenes)
    Col transport_trace(Ray ray) {
        const bool nee = P.direct != PTR_DIRECT_NONE;
        const bool mis = P.direct == PTR_DIRECT_MIS;
        const bool media = S.has_media;
        const int N = P.max_bounces;
        // path_state_init (pt.ts:147-176)
        Col throughput(1.0f), radiance(0.0f);
        bool prev_was_delta = true;
        float prev_bsdf_pdf = 0.0f;
        v3 prev_qp = ray.o;
        v3 prev_qn(0.0f);
        bool prev_q2 = false;
        float eta_scale = 1.0f;
        int current_medium = media ? S.scene_region_at(ray.o) : -1;
        int null_crossings = 0;
        Ray r = ray;

        auto roulette = [&](int bounce) -> bool {   // pt.ts:204-222
            if (P.rr_start < 0) return true;
            if (bounce < P.rr_start) return true;
            float p_survive = fminf_(P.rr_max_survival, spectrum_max(throughput) * eta_scale);
            if (p_survive <= 0.0f) return false;
            if (rng.next() > p_survive) return false;
            if (tan) for (double& x : tan->thr) x /= (double)p_survive;
            throughput = throughput / p_survive;
            return true;
        };
        auto roulette_interior = [&](int bounce, Col survival) -> bool {   // pt.ts:230-283
            if (P.rr_start < 0) return true;
            if (bounce < P.rr_start) return true;
            float p_survive = spectrum_max(survival);
            if (p_survive <= 0.0f) return false;
            if (rng.next() > p_survive) return false;
            if (tan) for (double& x : tan->thr) x /= (double)p_survive;
            throughput = throughput / p_survive;
            return true;
        };
        auto w_emitter = [&](const Hit& hit) -> float {   // combiner.ts:27-46
            if (!nee) return 1.0f;
            int lid = hit.region_to >= 0 ? emitter_light(hit) : -1;
            if (lid < 0 || prev_was_delta) return 1.0f;
            if (!mis) return 0.0f;
            return power_heuristic(prev_bsdf_pdf, lighting_pdf(Query{prev_qp, prev_qn, prev_q2}, r.d, lid, hit));
        };
        auto w_env = [&]() -> float {   // combiner.ts:49-65
            if (!(S.env_samplable && nee)) return 1.0f;
            if (prev_was_delta) return 1.0f;
            if (!mis) return 0.0f;
            float pe = S.env_select_live ? d.env.select_prob : 1.0f;
            return power_heuristic(prev_bsdf_pdf, pe * environment_pdf(r.d));
        };
        int shadow_left_base = P.max_null_crossings;
        if (tan) tan_reset();
        std::vector<DW> dw(tan ? kMaxDW : 0);
        std::vector<std::pair<int, double>> dlog_vis;

        for (int bounce = 0; bounce <= N; bounce++) {
            Hit hit;
            bool boundary = intersect(r, hit);
            if (media) {
                // the volumetric call site (pt.ts walk): one segment, random2() drawn for
                // every medium arm, scattering or absorbing-only (features/materials.ts:675-746)
                int med_mat = S.material_of(current_medium);
                if (S.material_has_medium(med_mat)) {
                    // the per-segment equiangular site precedes the transmittance sample
                    // (pt.ts:322-328); it places an event, so it is part of the budget
                    if (P.equiangular && bounce < N)
                        equiangular_sample_direct(r, med_mat, boundary ? hit.t : MAX_DIST, throughput, radiance,
                                                  shadow_left_base - null_crossings);
                    float x0 = rng.next(), x1 = rng.next();
                    float t_max = boundary ? hit.t : MAX_DIST;
                    const ptr_material& mm = d.materials[med_mat];
                    const bool het = !SPECTRAL && is_het(med_mat);
                    if (het && !scatter_live(med_mat)) {   // ratio-tracked pass-through
                        if constexpr (!SPECTRAL) throughput = throughput * medium_ratio_track(mm, r, t_max, rng, false);
                    } else if (!scatter_live(med_mat)) {
                        // absorbing-only arm (deterministic): weight = exp(-sigma_a t_max)
                        if (tan) {   // exp(-(1 - a) st t_max)
                            double st, a;
                            grey_params(med_mat, st, a);
                            const Dual w_st = dexp(-(1.0 - a) * Dual{st, 1.0} * (double)t_max);
                            const Dual w_a = dexp(-(1.0 - Dual{a, 1.0}) * st * (double)t_max);
                            dw[0] = {slot_k(med_mat, PTR_GRAD_SIGMA_T), {w_st.d, w_st.d, w_st.d}};
                            dw[1] = {slot_k(med_mat, PTR_GRAD_MEDIUM_ALBEDO), {w_a.d, w_a.d, w_a.d}};
                            tan_mul(throughput, vexp(-c_sigma_a(med_mat) * t_max), dw.data(), 2);
                        }
                        throughput = throughput * vexp(-c_sigma_a(med_mat) * t_max);
                    } else {
                        MS ms;
                        if constexpr (!SPECTRAL) {
                            ms = het ? medium_sample_delta(mm, r, t_max, x0, x1)
                                     : medium_sample_analytic(c_sigma_a(med_mat), c_sigma_s(med_mat), r, t_max, x0, x1);
                        } else {
                            ms = medium_sample_analytic(c_sigma_a(med_mat), c_sigma_s(med_mat), r, t_max, x0, x1);
                        }
                        if (tan) {   // free flight with the detached channel-MIS density
                            double st, a;
                            grey_params(med_mat, st, a);
                            const Col sigma_t = c_sigma_a(med_mat) + c_sigma_s(med_mat);
                            if (ms.scattered) {   // a st exp(-st t) / pdf
                                const float pdf = fmaxf_(spectrum_average(sigma_t * vexp(-sigma_t * ms.t)), 1e-20f);
                                const Dual w_st = a * Dual{st, 1.0} * dexp(-Dual{st, 1.0} * (double)ms.t) / (double)pdf;
                                const Dual w_a = Dual{a, 1.0} * st * fm::exp(-st * (double)ms.t) / (double)pdf;
                                dw[0] = {slot_k(med_mat, PTR_GRAD_SIGMA_T), {w_st.d, w_st.d, w_st.d}};
                                dw[1] = {slot_k(med_mat, PTR_GRAD_MEDIUM_ALBEDO), {w_a.d, w_a.d, w_a.d}};
                                tan_mul(throughput, ms.weight, dw.data(), 2);
                            } else {              // exp(-st t_max) / P
                                const float pdf = fmaxf_(spectrum_average(vexp(-sigma_t * t_max)), 1e-20f);
                                const Dual w_st = dexp(-Dual{st, 1.0} * (double)t_max) / (double)pdf;
                                dw[0] = {slot_k(med_mat, PTR_GRAD_SIGMA_T), {w_st.d, w_st.d, w_st.d}};
                                tan_mul(throughput, ms.weight, dw.data(), 1);
                            }
                        }
                        throughput = throughput * ms.weight;
                        if (ms.scattered) {
                            if (bounce == N) break;
                            v3 p_evt = ms.exit_p;
                            v3 wo_med = -ms.exit_dir;
                            // light_sample_direct_medium (techniques/light/light_medium.glsl:7-18);
                            // the equiangular site replaces it (pt.ts:379)
                            if (nee && !P.equiangular) {
                                float y0 = rng.next(), y1 = rng.next();
                                LS ls = lighting_sample(Query{p_evt, v3(0.0f), false}, y0, y1);
                                shadow_seed = rng.dim;
                                if (ls.pdf > 0.0f) {
                                    v3 light_p = p_evt + ls.wi * ls.distance;
                                    dlog_vis.clear();
                                    Col vis = shadow_transmittance(Ray{p_evt, ls.wi}, light_p, shadow_left_base - null_crossings,
                                                                   tan ? &dlog_vis : nullptr);
                                    if (!spectrum_is_black(vis)) {
                                        float w = 1.0f;
                                        if (mis && !(ls.flags & LIGHT_DELTA))   // hg_pdf = spectrum_average(hg_eval)
                                            w = power_heuristic(ls.pdf, spectrum_average(Col(hg_eval(ls.wi, wo_med, mm.phase_g))));
                                        if (tan) {   // X = Le p_HG(g) T w / pdf
                                            const Col X = ls.radiance * Col(hg_eval(ls.wi, wo_med, mm.phase_g)) * vis * w / ls.pdf;
                                            const Dual ph = hg_dual(ls.wi, wo_med, Dual{(double)mm.phase_g, 1.0});
                                            int n = 0;
                                            dw[n].k = slot_k(med_mat, PTR_GRAD_HG_G);
                                            for (int c = 0; c < 3; ++c)
                                                dw[n].d[c] = (double)ls.radiance[c] * ph.d * (double)vis[c] * (double)w / (double)ls.pdf;
                                            n = dw_from_dlog(X, dlog_vis, dw, n + 1);
                                            tan_add(throughput, X, dw.data(), n);
                                        }
                                        radiance = radiance + throughput * ls.radiance * Col(hg_eval(ls.wi, wo_med, mm.phase_g)) * vis * w / ls.pdf;
                                    }
                                }
                            }
                            // kernel_sample_phase (techniques/kernel/kernel_phase.glsl:7-15)
                            float z0 = rng.next(), z1 = rng.next();
                            IS ps = hg_sample<Col>(wo_med, mm.phase_g, z0, z1);
                            if (tan) {   // p_HG(g) / pdf
                                const Dual ph = hg_dual(ps.wi, wo_med, Dual{(double)mm.phase_g, 1.0});
                                const double dg = ph.d / (double)ps.pdf;
                                dw[0] = {slot_k(med_mat, PTR_GRAD_HG_G), {dg, dg, dg}};
                                tan_mul(throughput, ps.weight, dw.data(), 1);
                            }
                            throughput = throughput * ps.weight;
                            prev_was_delta = false;
                            prev_bsdf_pdf = ps.pdf;
                            prev_qp = p_evt;
                            prev_qn = v3(0.0f);
                            prev_q2 = false;
                            r = Ray{p_evt, ps.wi};
                            // tracking arms settled absorption in their lottery: nothing is owed
                            if (!het && !roulette_interior(bounce, medium_survival(med_mat))) break;
                            continue;
                        }
                    }
                }
            }
            if (!boundary) {   // kernel_score_miss (kernel.glsl:11-14)
                if (tan) tan_add(throughput, w_env() * environment_radiance(r.d), nullptr, 0);
                radiance = radiance + throughput * w_env() * environment_radiance(r.d);
                break;
            }
            if (media && hit.region_from != current_medium) current_medium = hit.region_from;
            int mat = S.material_of(hit.region_owner);
            if (media && S.is_null_interface(mat)) {   // pt.ts:404-417 null pass-through
                current_medium = hit.region_to;
                r = ray_spawn(hit, r.d);
                null_crossings++;
                if (null_crossings > P.max_null_crossings) break;
                bounce--;
                continue;
            }
            v3 wo = -r.d;
            hit_alpha = hit.alpha;
            // kernel_score_emitter_hit (kernel.glsl:16-25)
            int mat_emit = S.material_of(hit.region_to);
            if (S.material_is_emissive(mat_emit)) {
                if (tan) tan_add(throughput, w_emitter(hit) * c_emission(mat_emit), nullptr, 0);
                radiance = radiance + throughput * w_emitter(hit) * c_emission(mat_emit);
            }
            if (bounce == N) break;
            const ptr_material& m = d.materials[mat];
            // light_sample_direct (techniques/light/light.glsl:8-28)
            if (nee && S.material_has_nondelta_lobes(mat)) {
                float y0 = rng.next(), y1 = rng.next();
                LS ls = lighting_sample(Query{hit.p, hit.frame.n, m.model == PTR_MAT_ROUGH_DIELECTRIC}, y0, y1);
                shadow_seed = rng.dim;
                if (ls.pdf > 0.0f) {
                    v3 light_p = hit.p + ls.wi * ls.distance;
                    Ray sr = ray_spawn(hit, ls.wi);
                    sr.d = normalize(light_p - sr.o);
                    dlog_vis.clear();
                    Col vis = shadow_transmittance(sr, light_p, shadow_left_base - null_crossings, tan ? &dlog_vis : nullptr);
                    if (!spectrum_is_black(vis)) {
                        Col f = surface_eval(m, ls.wi, wo, hit);
                        float cos_i = std::fabs(dot(ls.wi, hit.frame.n));
                        float w = 1.0f;
                        if (mis && !(ls.flags & LIGHT_DELTA)) w = power_heuristic(ls.pdf, surface_pdf(m, ls.wi, wo, hit));
                        if (tan) {   // X = Le f cos T w / pdf
                            const Col X = ls.radiance * f * cos_i * vis * w / ls.pdf;
                            int n = 0;
                            if (m.model == PTR_MAT_LAMBERT) {   // f = albedo / pi
                                for (int c = 0; c < 3; ++c) {
                                    dw[n].k = slot_k(mat, PTR_GRAD_ALBEDO_R + c);
                                    dw[n].d[0] = dw[n].d[1] = dw[n].d[2] = 0.0;
                                    if (f[c] != 0.0f)
                                        dw[n].d[c] = (double)ls.radiance[c] * (1.0 / PI_D) * (double)cos_i * (double)vis[c] *
                                                     (double)w / (double)ls.pdf;
                                    ++n;
                                }
                            } else if (m.model == PTR_MAT_GGX) {   // f = F(F0) fs(alpha)
                                n = dw_schlick_f0(mat, m, ggx_fresnel_cos(ls.wi, wo, hit), X, dw.data(), n);
                                if (hit_alpha < 0.0f) {
                                    const Dual fs = ggx_fs_dual(ls.wi, wo, hit.frame, Dual{(double)m.alpha, 1.0});
                                    dw[n].k = slot_k(mat, PTR_GRAD_ALPHA);
                                    for (int c = 0; c < 3; ++c) dw[n].d[c] = fs.v > 0.0 ? (double)X[c] * fs.d / fs.v : 0.0;
                                    ++n;
                                }
                            }
                            n = dw_from_dlog(X, dlog_vis, dw, n);
                            tan_add(throughput, X, dw.data(), n);
                        }
                        radiance = radiance + throughput * ls.radiance * f * cos_i * vis * w / ls.pdf;
                    }
                }
            }
            // kernel_sample_continuation (kernel.glsl:27-34)
            float uc = rng.next();
            float u0 = rng.next(), u1 = rng.next();
            IS bs = surface_sample(m, wo, hit, uc, u0, u1);
            if (spectrum_is_black(bs.weight)) break;
            if (tan) tan_continuation(m, mat, wo, hit, bs, throughput, dw.data());
            throughput = throughput * bs.weight;
            prev_was_delta = (bs.flags & LOBE_DELTA) != 0u;
            prev_bsdf_pdf = bs.pdf;
            prev_qp = hit.p;
            prev_qn = hit.frame.n;
            prev_q2 = m.model == PTR_MAT_ROUGH_DIELECTRIC;
            if (bs.flags & LOBE_TRANSMISSION) {
                if (media) current_medium = hit.region_to;
                float rr = S.ior_of(hit.region_to) / S.ior_of(hit.region_from);   // pt.ts:447-455
                eta_scale *= rr * rr;
            }
            if (!roulette(bounce)) break;
            r = ray_spawn(hit, bs.wi);
        }
        return radiance;
    }
};
using Tracer = TracerT<v3>;

// camera_generateRay (camera/pinhole/pinhole.glsl:4-18) + pixel_sample (pixel/box/box.glsl:5)
inline Ray camera_ray(const ptr_camera& c, int W, int H, float fx, float fy) {
    float ndcx = (2.0f * fx / (float)W) - 1.0f;
    float ndcy = (2.0f * fy / (float)H) - 1.0f;
    ndcx *= c.aspect;
    v3 dir = normalize(ld3(c.forward) + ndcx * c.tan_fov * ld3(c.right) + ndcy * c.tan_fov * ld3(c.up));
    return Ray{ld3(c.position), dir};
}

}  // namespace

extern "C" {

// The coefficient field program starting at code[start], evaluated at n points (3 floats
// each) into out (3 floats each).
void oracle_field_eval(const uint32_t* code, int start, const float* p, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        v3 v = field_eval(code + start, v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]));
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
}

// Render frame->spp samples for every pixel; accumulate per-pixel sum / sum of squares
// (float64, 3 per pixel, row 0 = bottom).  Returns counters through out_counts[2]
// (closest-hit queries, shadow queries) when non-null.
int oracle_render_tile(const ptr_scene_desc* sd, const ptr_program_desc* pd, const ptr_frame* fr,
                       int x0, int y0, int tw, int th,
                       double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads);

int oracle_render(const ptr_scene_desc* sd, const ptr_program_desc* pd, const ptr_frame* fr,
                  double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads) {
    if (!fr) return -1;
    return oracle_render_tile(sd, pd, fr, 0, 0, fr->width, fr->height, sum, sumsq, samples_out, out_counts, threads);
}

// Render the tile [x0, x0+tw) x [y0, y0+th) of the frame's image (the camera sees the
// whole frame->width x frame->height image); outputs are indexed within the tile.
static int render_tile_scene(const Scene& S, const ptr_frame* fr, int x0, int y0, int tw, int th,
                             double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads);

int oracle_render_tile(const ptr_scene_desc* sd, const ptr_program_desc* pd, const ptr_frame* fr,
                       int x0, int y0, int tw, int th,
                       double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads) {
    if (!sd || !pd || !fr) return -1;
    Scene S(sd, pd);
    return render_tile_scene(S, fr, x0, y0, tw, th, sum, sumsq, samples_out, out_counts, threads);
}

// A prepared scene (its mesh acceleration built once): the descriptor and program are
// copied; the arrays they point to must stay alive while the session is used.
struct OracleSession {
    ptr_scene_desc desc;
    ptr_program_desc prog;
    Scene* scene;
};

void* oracle_session_create(const ptr_scene_desc* sd, const ptr_program_desc* pd) {
    OracleSession* s = new OracleSession();
    s->desc = *sd;
    s->prog = *pd;
    s->scene = new Scene(&s->desc, &s->prog);
    return s;
}

void oracle_session_free(void* h) {
    OracleSession* s = (OracleSession*)h;
    delete s->scene;
    delete s;
}

int oracle_session_render_tile(void* h, const ptr_frame* fr, int x0, int y0, int tw, int th,
                               double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads) {
    OracleSession* s = (OracleSession*)h;
    return render_tile_scene(*s->scene, fr, x0, y0, tw, th, sum, sumsq, samples_out, out_counts, threads);
}

// Forward-mode reference of the path-replay adjoint (ptr_backward), in float64.  The walk
// and its random numbers are the plain render's (float32, so every sampling decision is
// the GPU's); alongside it each path carries d throughput / d theta and d radiance /
// d theta for every material slot, with the adjoint's detached conventions (Tracer::Tan).
// Output per pixel of the tile and channel: the sum over the frame's samples of
// d L / d theta_k, jac[(3 * pixel + c) * K + k], K = PTR_GRAD_SLOTS * n_materials; and
// the sample sum of L (sum[3 * pixel + c]).  Returns -2 for programs outside the
// adjoint's model (equiangular medium NEE, spectral colour, chromatic media).
int oracle_forward_tile(const ptr_scene_desc* sd, const ptr_program_desc* pd, const ptr_frame* fr,
                        int x0, int y0, int tw, int th, double* jac, double* sum, int threads) {
    if (!sd || !pd || !fr || !jac) return -1;
    if (pd->equiangular != PTR_EQUIANGULAR_OFF || pd->color != PTR_COLOR_RGB) return -2;
    for (int i = 0; i < sd->n_materials; ++i) {
        const ptr_material& m = sd->materials[i];
        if ((m.flags & PTR_MATF_MEDIUM) && !(m.sigma_a[0] == m.sigma_a[1] && m.sigma_a[0] == m.sigma_a[2] &&
                                             m.sigma_s[0] == m.sigma_s[1] && m.sigma_s[0] == m.sigma_s[2]))
            return -2;
    }
    Scene S(sd, pd);
    // engine.imageSize: the full image when this frame is a tile of it (pinhole.glsl:6)
    const int W = fr->image_size[0] > 0 ? fr->image_size[0] : fr->width;
    const int H = fr->image_size[1] > 0 ? fr->image_size[1] : fr->height;
    const int K = PTR_GRAD_SLOTS * sd->n_materials;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        Tracer T(S);
        Tracer::Tan tan;
        tan.K = K;
        tan.thr.assign(3 * (size_t)K, 0.0);
        tan.rad.assign(3 * (size_t)K, 0.0);
        T.tan = &tan;
#pragma omp for schedule(dynamic, 1)
        for (int ty = 0; ty < th; ++ty) {
            const int y = y0 + ty;
            for (int tx = 0; tx < tw; ++tx) {
                const int x = x0 + tx;
                const size_t pix = (size_t)ty * tw + tx;
                for (int k = 0; k < fr->spp; ++k) {
                    T.rng.init((uint32_t)(x + fr->pixel_offset[0]), (uint32_t)(y + fr->pixel_offset[1]),
                               (uint32_t)(fr->first_sample + k), fr->reset_salt);
                    float pxf = (float)x + 0.5f + (float)fr->pixel_offset[0];
                    float pyf = (float)y + 0.5f + (float)fr->pixel_offset[1];
                    float a0 = T.rng.next(), a1 = T.rng.next();
                    float fx = pxf + (a0 - 0.5f), fy = pyf + (a1 - 0.5f);
                    T.rng.next(); T.rng.next();
                    v3 L = T.transport_trace(camera_ray(fr->camera, W, H, fx, fy));
                    for (int c = 0; c < 3; ++c) {
                        if (sum) sum[3 * pix + c] += (double)L[c];
                        double* jrow = jac + (3 * pix + c) * (size_t)K;
                        for (int q = 0; q < K; ++q) jrow[q] += tan.rad[3 * (size_t)q + c];
                    }
                }
            }
        }
    }
    return 0;
}

// The RGB walk, or the spectral one: four wavelengths drawn between the film point and
// the lens draws (accumulation.ts main(): cameraSample, then wavelengths_sample), each
// sample's lanes projected to linear sRGB by color_to_pixel before the fold.
}  // extern "C"

template <class Col>
static int render_tile_scene_t(const Scene& S, const ptr_frame* fr, int x0, int y0, int tw, int th,
                               double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads) {
    // engine.imageSize: the full image when this frame is a tile of it (pinhole.glsl:6)
    const int W = fr->image_size[0] > 0 ? fr->image_size[0] : fr->width;
    const int H = fr->image_size[1] > 0 ? fr->image_size[1] : fr->height;
    uint64_t closest = 0, shadow = 0;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : closest, shadow)
    {
        TracerT<Col> T(S);
#pragma omp for schedule(dynamic, 1)
        for (int ty = 0; ty < th; ++ty) {
            const int y = y0 + ty;
            for (int tx = 0; tx < tw; ++tx) {
                const int x = x0 + tx;
                size_t pix = (size_t)ty * tw + tx;
                for (int k = 0; k < fr->spp; ++k) {
                    uint32_t px = (uint32_t)(x + fr->pixel_offset[0]);
                    uint32_t py = (uint32_t)(y + fr->pixel_offset[1]);
                    T.rng.init(px, py, (uint32_t)(fr->first_sample + k), fr->reset_salt);
                    // main(): pixel = gl_FragCoord + offset; film = pixel + (xi - 0.5)
                    float pxf = (float)x + 0.5f + (float)fr->pixel_offset[0];
                    float pyf = (float)y + 0.5f + (float)fr->pixel_offset[1];
                    float a0 = T.rng.next(), a1 = T.rng.next();
                    float fx = pxf + (a0 - 0.5f), fy = pyf + (a1 - 0.5f);
                    float lam[4], lpdf[4];
                    if constexpr (std::is_same<Col, s4>::value) {
                        wavelengths_sample(*S.prog, T.rng.next(), lam, lpdf);
                        for (int q = 0; q < 4; ++q) T.wl[q] = lam[q];
                    }
                    T.rng.next(); T.rng.next();   // xiLens (pinhole ignores it)
                    Ray r = camera_ray(fr->camera, W, H, fx, fy);
                    v3 L;
                    if constexpr (std::is_same<Col, s4>::value) L = color_to_pixel(*S.d, T.transport_trace(r), lam, lpdf);
                    else L = T.transport_trace(r);
                    if (samples_out) {
                        float* o = samples_out + 3 * ((size_t)k * tw * th + pix);
                        o[0] = L.x; o[1] = L.y; o[2] = L.z;
                    }
                    if (sum) {
                        for (int c = 0; c < 3; ++c) {
                            sum[3 * pix + c] += (double)L[c];
                            sumsq[3 * pix + c] += (double)L[c] * (double)L[c];
                        }
                    }
                }
            }
        }
        closest += T.cnt.closest;
        shadow += T.cnt.shadow;
    }
    if (out_counts) { out_counts[0] = closest; out_counts[1] = shadow; }
    return 0;
}

static int render_tile_scene(const Scene& S, const ptr_frame* fr, int x0, int y0, int tw, int th,
                             double* sum, double* sumsq, float* samples_out, uint64_t* out_counts, int threads) {
    if (S.prog->color == PTR_COLOR_SPECTRAL) {
        if (!S.d->spectral) return -1;
        return render_tile_scene_t<s4>(S, fr, x0, y0, tw, th, sum, sumsq, samples_out, out_counts, threads);
    }
    return render_tile_scene_t<v3>(S, fr, x0, y0, tw, th, sum, sumsq, samples_out, out_counts, threads);
}

extern "C" {


// The rough dielectric in its local frame (n = +z, wo in the upper hemisphere), for the
// BSDF property tests: eval (rgb) and pdf of n (wi, wo) pairs; n samples for n (uc, u0, u1).
int oracle_rough_dielectric_eval_n(int n, float alpha, float n_i, float n_t, const float* tint, const float* wi,
                                   const float* wo, float* f_out, float* pdf_out) {
    ptr_material m{};
    for (int c = 0; c < 3; ++c) m.transmittance[c] = tint[c];
    for (int k = 0; k < n; ++k) {
        v3 wil(wi[3 * k], wi[3 * k + 1], wi[3 * k + 2]), wol(wo[3 * k], wo[3 * k + 1], wo[3 * k + 2]);
        v3 f = rough_dielectric_eval_local(wil, wol, ld3(m.transmittance), alpha, n_i, n_t);
        f_out[3 * k] = f.x; f_out[3 * k + 1] = f.y; f_out[3 * k + 2] = f.z;
        pdf_out[k] = rough_dielectric_pdf_local(wil, wol, alpha, n_i, n_t);
    }
    return 0;
}
int oracle_rough_dielectric_sample_n(int n, float alpha, float n_i, float n_t, const float* tint, const float* wo,
                                     const float* u, float* wi_out, float* weight_out, float* pdf_out, int* flags_out) {
    ptr_material m{};
    for (int c = 0; c < 3; ++c) m.transmittance[c] = tint[c];
    for (int k = 0; k < n; ++k) {
        ISample smp = rough_dielectric_sample_local(v3(wo[3 * k], wo[3 * k + 1], wo[3 * k + 2]), ld3(m.transmittance),
                                                    alpha, n_i, n_t, u[3 * k], u[3 * k + 1], u[3 * k + 2]);
        wi_out[3 * k] = smp.wi.x; wi_out[3 * k + 1] = smp.wi.y; wi_out[3 * k + 2] = smp.wi.z;
        weight_out[3 * k] = smp.weight.x; weight_out[3 * k + 1] = smp.weight.y; weight_out[3 * k + 2] = smp.weight.z;
        pdf_out[k] = smp.pdf;
        flags_out[k] = (int)smp.flags;
    }
    return 0;
}

// Nearest-hit queries with the oracle's own acceleration: per ray (o.xyz, d.xyz) the
// region (-1 = miss), the instance index (element; 0 outside instanced batches), the
// original triangle index (-1 if not a mesh hit) and t.  Ties at equal t resolve in scan
// order: the lower region, instance and triangle index.
int oracle_trace_closest(const ptr_scene_desc* sd, const ptr_program_desc* pd, const float* rays, int n,
                         int* region, int* element, int* prim, float* t_out) {
    Scene S(sd, pd);
#pragma omp parallel for schedule(dynamic, 64)
    for (int k = 0; k < n; ++k) {
        Ray r{v3(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]), v3(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5])};
        Hit h;
        h.t = MAX_DIST;
        h.eps = MARCH_CLEARANCE;
        bool f = S.primitive_intersect(r, h);
        region[k] = f ? h.region_owner : -1;
        if (element) element[k] = f ? h.element : 0;
        prim[k] = f ? h.prim : -1;
        t_out[k] = h.t;
    }
    return 0;
}

// Brute-force nearest triangle of one mesh (every triangle, the same leaf test).
int oracle_mesh_brute(const ptr_mesh_desc* md, const float* rays, int n, int* prim, float* t_out) {
    OMesh m;
    m.build(*md);
#pragma omp parallel for schedule(dynamic, 64)
    for (int k = 0; k < n; ++k) {
        v3 ro(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]), rd(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]);
        float tmax = MAX_DIST;
        int best = -1;
        for (int i = 0; i < md->n_triangles; ++i) {
            float t;
            if (tri_test(ro, rd, m.a[i], m.e1[i], m.e2[i], t) && t > 0.0f && t < tmax) { tmax = t; best = i; }
        }
        prim[k] = best;
        t_out[k] = tmax;
    }
    return 0;
}

}  // extern "C"
