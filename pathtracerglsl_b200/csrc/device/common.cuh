// common.cuh — device math shared by every occupant of the transport loop.
//
// binary32 throughout; the library is compiled with -fmad=false so products and sums
// round exactly as written (the reference's GLSL operation order), which keeps the device
// results comparable sample-for-sample with the CPU restatement.
#pragma once
#ifndef __CUDACC_RTC__   // NVRTC builds (ptr_specialize) get the fixed-width types from their prelude
#include <cstdint>
#include <cuda_runtime.h>
#endif
#include "ptx_rt.h"

namespace ptx {

// The walk's float transcendentals.  By default CUDA's single-precision functions; a
// build with PTR_WIDE_MATH (ptr_specialize with that define) evaluates them in double and
// rounds once, the same functions as the oracle's wide twin, so that samples can be
// compared without the two libms' last-ulp differences.
#ifdef PTR_WIDE_MATH
#define PTR_M1(name, fn) __device__ __forceinline__ float name(float x) { return (float)fn((double)x); }
#define PTR_M2(name, fn) __device__ __forceinline__ float name(float x, float y) { return (float)fn((double)x, (double)y); }
#else
#define PTR_M1(name, fn) __device__ __forceinline__ float name(float x) { return fn##f(x); }
#define PTR_M2(name, fn) __device__ __forceinline__ float name(float x, float y) { return fn##f(x, y); }
#endif
PTR_M1(m_exp, exp) PTR_M1(m_log, log) PTR_M1(m_sin, sin) PTR_M1(m_cos, cos) PTR_M1(m_tan, tan)
PTR_M1(m_tanh, tanh) PTR_M1(m_atanh, atanh) PTR_M1(m_cosh, cosh) PTR_M2(m_atan2, atan2) PTR_M2(m_pow, pow)
#undef PTR_M1
#undef PTR_M2

// ---- scene specialisation.  The generic library keeps every occupant (all masks on, the
// region list read from the scene).  A build for one scene x strategy defines the masks of
// the occupants it holds and, optionally, its region count and region shapes as
// compile-time lists: absent occupants fold away (smaller kernels, fewer instruction-cache
// misses in divergent warps) and the region loops unroll into one arm per region with its
// intersection routine resolved at compile time, like the reference's generated arms.
#ifndef PTR_SPEC_MATS
#define PTR_SPEC_MATS 0xFFu     // bit per PTR_MAT_*
#endif
#ifndef PTR_SPEC_LIGHTS
#define PTR_SPEC_LIGHTS 0xFFu   // bit per PTR_LIGHT_*
#endif
#ifndef PTR_SPEC_ENVS
#define PTR_SPEC_ENVS 0xFFu     // bit per PTR_ENV_*
#endif
#ifndef PTR_SPEC_SHAPES
#define PTR_SPEC_SHAPES 0xFFu   // bit per PTR_SHAPE_*
#endif
#ifndef PTR_SPEC_TREE
#define PTR_SPEC_TREE 1         // 0: the build never selects lights with the light tree
#endif
#ifndef PTR_SPEC_NREGIONS
#define PTR_SPEC_NREGIONS 0     // 1..16: the region count and PTR_SPEC_SHAPE_CODE (the region BVH unused)
#endif
__host__ __device__ constexpr bool has_mat(int m) { return ((PTR_SPEC_MATS) >> m) & 1u; }
__host__ __device__ constexpr bool has_light(int k) { return ((PTR_SPEC_LIGHTS) >> k) & 1u; }
__host__ __device__ constexpr bool has_env(int k) { return ((PTR_SPEC_ENVS) >> k) & 1u; }
__host__ __device__ constexpr bool has_shape(int k) { return ((PTR_SPEC_SHAPES) >> k) & 1u; }
// (material models and light kinds are dispatched through their registries, occupant.cuh)
#if PTR_SPEC_NREGIONS > 0
static_assert(PTR_SPEC_NREGIONS <= 16, "the shape code holds 16 regions");
// region k's PTR_SHAPE_* in bits [4k, 4k + 4) of PTR_SPEC_SHAPE_CODE
__host__ __device__ constexpr int spec_shape(int k) { return (int)(((unsigned long long)(PTR_SPEC_SHAPE_CODE) >> (4 * k)) & 0xFull); }
#endif

struct f3 {
    float x, y, z;
    __host__ __device__ f3() : x(0.f), y(0.f), z(0.f) {}
    __host__ __device__ f3(float a, float b, float c) : x(a), y(b), z(c) {}
    __host__ __device__ explicit f3(float s) : x(s), y(s), z(s) {}
    __device__ float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 operator/(f3 a, f3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ f3 operator-(f3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return f3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 normalize(f3 a) { return a * (1.0f / length(a)); }
// GLSL min/max: min(x, y) = y < x ? y : x
__device__ __forceinline__ float gmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float gmax(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return f3(gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)); }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return f3(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)); }
__device__ __forceinline__ f3 vexp(f3 a) { return f3(m_exp(a.x), m_exp(a.y), m_exp(a.z)); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
__device__ __forceinline__ float signf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
__device__ __forceinline__ f3 ld3(const float* p) { return f3(p[0], p[1], p[2]); }
__device__ __forceinline__ f3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// The spectral colour model's carrier: four wavelength lanes (color/spectral/types.glsl,
// Spectrum = vec4), with the same component-wise operations as the RGB f3.
struct s4 {
    float x, y, z, w;
    __host__ __device__ s4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    __host__ __device__ s4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    __host__ __device__ explicit s4(float s) : x(s), y(s), z(s), w(s) {}
    __device__ float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};
__device__ __forceinline__ s4 operator+(s4 a, s4 b) { return s4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ s4 operator-(s4 a, s4 b) { return s4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ s4 operator*(s4 a, s4 b) { return s4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ s4 operator/(s4 a, s4 b) { return s4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
__device__ __forceinline__ s4 operator*(s4 a, float s) { return s4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ s4 operator*(float s, s4 a) { return s4(s * a.x, s * a.y, s * a.z, s * a.w); }
__device__ __forceinline__ s4 operator/(s4 a, float s) { return s4(a.x / s, a.y / s, a.z / s, a.w / s); }
__device__ __forceinline__ s4 operator-(s4 a) { return s4(-a.x, -a.y, -a.z, -a.w); }

// Scalar constants of the reference's core math (glsl/core/math.glsl).
constexpr float kPi = 3.14159265359f;
constexpr float kTwoPi = 6.28318530718f;
constexpr float kMaxDist = 1000.0f;           // MAX_DIST: the far clip
constexpr float kEpsInterface = 0.001f;       // EPS_INTERFACE: classification probe depth
constexpr float kMarchClearance = 0.001f;     // MARCH_CLEARANCE: conservative Hit.eps seed
constexpr float kShadowBackoff = 0.002f;      // SHADOW_BACKOFF (math.glsl:39)
constexpr float kFpRel = 3.0517578125e-5f;    // 256 ulps relative
constexpr float kFpAbs = 1.52587890625e-5f;   // 2^-16 absolute floor

constexpr uint32_t kLobeReflection = 1u, kLobeTransmission = 2u, kLobeDelta = 4u, kLobeMedium = 8u;
constexpr uint32_t kLightDelta = 1u;

// Spectrum helpers over the three RGB transport channels (components/color/spectrum.glsl).
__device__ __forceinline__ float spectrum_average(f3 s) { float a = s.x; a += s.y; a += s.z; return a * (1.0f / 3.0f); }
__device__ __forceinline__ float spectrum_max(f3 s) { float m = s.z; m = gmax(s.y, m); m = gmax(s.x, m); return m; }
__device__ __forceinline__ bool spectrum_is_black(f3 s) { return s.x <= 0.f && s.y <= 0.f && s.z <= 0.f; }
__device__ __forceinline__ int spectrum_sample_channel(float u) { int c = (int)(u * 3.0f); return c < 2 ? c : 2; }
__device__ __forceinline__ float spectrum_average(s4 s) { float a = s.x; a += s.y; a += s.z; a += s.w; return a * (1.0f / 4.0f); }
__device__ __forceinline__ float spectrum_max(s4 s) { float m = s.w; m = gmax(s.z, m); m = gmax(s.y, m); m = gmax(s.x, m); return m; }
__device__ __forceinline__ bool spectrum_is_black(s4 s) { return s.x <= 0.f && s.y <= 0.f && s.z <= 0.f && s.w <= 0.f; }
__device__ __forceinline__ s4 vexp(s4 a) { return s4(m_exp(a.x), m_exp(a.y), m_exp(a.z), m_exp(a.w)); }
__device__ __forceinline__ s4 vmax(s4 a, s4 b) { return s4(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z), gmax(a.w, b.w)); }
// Uniform lane choice for channel-MIS: min(int(u * N), N - 1).
template <class Col> __device__ __forceinline__ int sample_channel(float u);
template <> __device__ __forceinline__ int sample_channel<f3>(float u) { return spectrum_sample_channel(u); }
template <> __device__ __forceinline__ int sample_channel<s4>(float u) { int c = (int)(u * 4.0f); return c < 3 ? c : 3; }
// Pool records: colours live in float4 slots (RGB uses xyz).
template <class Col> __device__ __forceinline__ Col col_ld(float4 v);
template <> __device__ __forceinline__ f3 col_ld<f3>(float4 v) { return f3(v.x, v.y, v.z); }
template <> __device__ __forceinline__ s4 col_ld<s4>(float4 v) { return s4(v.x, v.y, v.z, v.w); }
__device__ __forceinline__ float4 col_st(f3 c, float w) { return make_float4(c.x, c.y, c.z, w); }
__device__ __forceinline__ float4 col_st(s4 c, float) { return make_float4(c.x, c.y, c.z, c.w); }

// ---- counter-based sampler: the pcg4d hash of Jarzynski & Olano ("Hash Functions for
// GPU Rendering", JCGT 2020), keyed per (pixel, sample, reset salt) with a dimension
// counter; the 24 high bits give an exactly representable float in [0, 1).
// (components/sampler/pcg4d/pcg4d.glsl:12-40)
__device__ __forceinline__ uint4 pcg4d(uint4 v) {
    v.x = v.x * 1664525u + 1013904223u;
    v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u;
    v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16u; v.y ^= v.y >> 16u; v.z ^= v.z >> 16u; v.w ^= v.w >> 16u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
struct Rng {
    uint32_t base, dim;
    __device__ __forceinline__ void init(uint32_t px, uint32_t py, uint32_t sample, uint32_t salt) {
        base = pcg4d(make_uint4(px, py, sample, salt)).x;
        dim = 0u;
    }
    __device__ __forceinline__ float next() {
        uint32_t u = pcg4d(make_uint4(base, dim, 0u, 0u)).x;
        dim += 1u;
        return (float)(u >> 8) * (1.0f / 16777216.0f);
    }
};

// ---- frames, Fresnel, spawn ---------------------------------------------------------
struct Frame { f3 t, b, n; };

// Positional error bound of a floating-point-accurate hit point (math.glsl:54-56).
__device__ __forceinline__ float fp_uncertainty(f3 p) {
    return gmax(kFpAbs, kFpRel * gmax(fabsf(p.x), gmax(fabsf(p.y), fabsf(p.z))));
}
// Shading frame from a normal (the Euclidean ambient_frame, euclidean.glsl:6-33).
__device__ __forceinline__ Frame ambient_frame(f3 n) {
    f3 nn = normalize(n);
    f3 t = fabsf(nn.x) < 0.9f ? f3(1.f, 0.f, 0.f) : f3(0.f, 1.f, 0.f);
    t = normalize(t - dot(t, nn) * nn);
    Frame f;
    f.t = t; f.b = cross(nn, t); f.n = nn;
    return f;
}
// Orthonormal completion used by samplers (math.glsl build_basis).
__device__ __forceinline__ void build_basis(f3 n, f3& t, f3& b) {
    f3 up = fabsf(n.y) < 0.999f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
    t = normalize(cross(up, n));
    b = cross(n, t);
}
// Exact unpolarised dielectric Fresnel, eta = n_i / n_t (math.glsl:95-102).
__device__ __forceinline__ float dielectric_fresnel(float cos_i, float eta) {
    float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin2_t);
    float r_par = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    float r_perp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (r_par * r_par + r_perp * r_perp);
}
template <class Col>
__device__ __forceinline__ Col schlick_fresnel(Col f0, float c) {
    return f0 + (Col(1.0f) - f0) * m_pow(1.0f - c, 5.0f);
}
__device__ __forceinline__ float power_heuristic(float pf, float pg) {
    float f2 = pf * pf;
    if (f2 >= 1.0e38f) return 1.0f;
    return f2 / gmax(1e-20f, f2 + pg * pg);
}

struct Ray { f3 o, d; };

// The hit record every arm fills (structs.glsl Hit), minus the wavelengths.
struct Hit {
    float t;
    f3 p;
    Frame frame;
    f3 ng;
    int region_from, region_to, region_owner, element;
    float eps;
    float alpha;   // per-triangle GGX alpha when the mesh carries one, else < 0
};

// Escape to wi's side of the true surface by the hit's own uncertainty (ray.glsl:29-32).
__device__ __forceinline__ Ray ray_spawn(const Hit& h, f3 wi) {
    float side = dot(wi, h.ng) >= 0.0f ? 1.0f : -1.0f;
    Ray r;
    r.o = h.p + (h.ng * side) * h.eps;
    r.d = wi;
    return r;
}

}  // namespace ptx
