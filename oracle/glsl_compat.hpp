// glsl_compat.hpp — a small GLSL ES 3.00 compatibility layer for C++20.
//
// TEST INFRASTRUCTURE ONLY.  This header lets the reference's own generated fragment
// programs (the assembled GLSL stored in the reference's snapshot file
// tests/compiler/__snapshots__/generated-glsl.snapshot.test.ts.snap) compile as plain
// C++ on the CPU, so the oracle can run the reference's shader math without any
// graphics stack.  Nothing in the product links it.
//
// Scope: exactly the GLSL subset those programs use — float/int/uint/bool vectors of
// size 2..4, component access (.x .y .z .w and .r .g .b .a as members; multi-letter
// swizzles are rewritten by the translator into method calls such as .xyz()),
// component-wise arithmetic, the built-in functions, and sampler2D/texelFetch over
// host arrays.  Arithmetic is IEEE binary32 through libm (sqrtf, expf, ...); the
// translator appends an 'f' to every floating literal so no expression is silently
// evaluated in double precision.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace glsl {

typedef unsigned int uint;

template <typename T, int N> struct V;

#define GLSL_VEC_COMMON(N)                                                        \
    T& operator[](int i) { return (&x)[i]; }                                      \
    const T& operator[](int i) const { return (&x)[i]; }

template <typename T> struct V<T, 2> {
    union { T x; T r; };
    union { T y; T g; };
    V() : x(T(0)), y(T(0)) {}
    explicit V(T s) : x(s), y(s) {}
    V(T a, T b) : x(a), y(b) {}
    template <typename U> explicit V(const V<U, 2>& o) : x(T(o.x)), y(T(o.y)) {}
    template <typename U> explicit V(const V<U, 3>& o) : x(T(o.x)), y(T(o.y)) {}
    template <typename U> explicit V(const V<U, 4>& o) : x(T(o.x)), y(T(o.y)) {}
    GLSL_VEC_COMMON(2)
    V<T, 2> xy() const { return V<T, 2>(x, y); }
    V<T, 2> yx() const { return V<T, 2>(y, x); }
    V<T, 3> xxx() const;
    V<T, 3> xyy() const;
    V<T, 3> yxy() const;
    V<T, 3> yyx() const;
};

template <typename T> struct V<T, 3> {
    union { T x; T r; };
    union { T y; T g; };
    union { T z; T b; };
    V() : x(T(0)), y(T(0)), z(T(0)) {}
    explicit V(T s) : x(s), y(s), z(s) {}
    V(T a, T b_, T c) : x(a), y(b_), z(c) {}
    V(const V<T, 2>& v, T c) : x(v.x), y(v.y), z(c) {}
    V(T a, const V<T, 2>& v) : x(a), y(v.x), z(v.y) {}
    template <typename U> explicit V(const V<U, 3>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    template <typename U> explicit V(const V<U, 4>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    GLSL_VEC_COMMON(3)
    V<T, 2> xy() const { return V<T, 2>(x, y); }
    V<T, 2> xz() const { return V<T, 2>(x, z); }
    V<T, 2> yz() const { return V<T, 2>(y, z); }
    V<T, 2> zx() const { return V<T, 2>(z, x); }
    V<T, 3> xyz() const { return *this; }
    V<T, 3> rgb() const { return *this; }
    V<T, 3> xxx() const { return V<T, 3>(x, x, x); }
    V<T, 3> xyy() const { return V<T, 3>(x, y, y); }
    V<T, 3> yxy() const { return V<T, 3>(y, x, y); }
    V<T, 3> yyx() const { return V<T, 3>(y, y, x); }
};

template <typename T> struct V<T, 4> {
    union { T x; T r; };
    union { T y; T g; };
    union { T z; T b; };
    union { T w; T a; };
    V() : x(T(0)), y(T(0)), z(T(0)), w(T(0)) {}
    explicit V(T s) : x(s), y(s), z(s), w(s) {}
    V(T a_, T b_, T c, T d) : x(a_), y(b_), z(c), w(d) {}
    V(const V<T, 3>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    V(const V<T, 2>& v, T c, T d) : x(v.x), y(v.y), z(c), w(d) {}
    V(const V<T, 2>& v, const V<T, 2>& u) : x(v.x), y(v.y), z(u.x), w(u.y) {}
    template <typename U> explicit V(const V<U, 4>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
    GLSL_VEC_COMMON(4)
    V<T, 2> xy() const { return V<T, 2>(x, y); }
    V<T, 2> zw() const { return V<T, 2>(z, w); }
    V<T, 2> xz() const { return V<T, 2>(x, z); }
    V<T, 3> xyz() const { return V<T, 3>(x, y, z); }
    V<T, 3> rgb() const { return V<T, 3>(x, y, z); }
    V<T, 3> yzw() const { return V<T, 3>(y, z, w); }
};

template <typename T> V<T, 3> V<T, 2>::xxx() const { return V<T, 3>(x, x, x); }
template <typename T> V<T, 3> V<T, 2>::xyy() const { return V<T, 3>(x, y, y); }
template <typename T> V<T, 3> V<T, 2>::yxy() const { return V<T, 3>(y, x, y); }
template <typename T> V<T, 3> V<T, 2>::yyx() const { return V<T, 3>(y, y, x); }

typedef V<float, 2> vec2;
typedef V<float, 3> vec3;
typedef V<float, 4> vec4;
typedef V<int, 2> ivec2;
typedef V<int, 3> ivec3;
typedef V<int, 4> ivec4;
typedef V<uint, 2> uvec2;
typedef V<uint, 3> uvec3;
typedef V<uint, 4> uvec4;
typedef V<bool, 2> bvec2;
typedef V<bool, 3> bvec3;
typedef V<bool, 4> bvec4;

// ---- component-wise operators --------------------------------------------------
#define GLSL_BINOP(OP, OPA)                                                                   \
    template <typename T, int N> V<T, N> operator OP(const V<T, N>& a, const V<T, N>& b) {    \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] OP b[i]; return r; }               \
    template <typename T, int N> V<T, N> operator OP(const V<T, N>& a, T s) {                 \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] OP s; return r; }                  \
    template <typename T, int N> V<T, N> operator OP(T s, const V<T, N>& a) {                 \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = s OP a[i]; return r; }                  \
    template <typename T, int N> V<T, N>& operator OPA(V<T, N>& a, const V<T, N>& b) {        \
        for (int i = 0; i < N; ++i) a[i] = a[i] OP b[i]; return a; }                          \
    template <typename T, int N> V<T, N>& operator OPA(V<T, N>& a, T s) {                     \
        for (int i = 0; i < N; ++i) a[i] = a[i] OP s; return a; }

GLSL_BINOP(+, +=)
GLSL_BINOP(-, -=)
GLSL_BINOP(*, *=)
GLSL_BINOP(/, /=)
GLSL_BINOP(^, ^=)
GLSL_BINOP(&, &=)
GLSL_BINOP(|, |=)
GLSL_BINOP(%, %=)
GLSL_BINOP(>>, >>=)
GLSL_BINOP(<<, <<=)
#undef GLSL_BINOP

template <typename T, int N> V<T, N> operator-(const V<T, N>& a) {
    V<T, N> r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r;
}
template <typename T, int N> bool operator==(const V<T, N>& a, const V<T, N>& b) {
    for (int i = 0; i < N; ++i) if (!(a[i] == b[i])) return false; return true;
}
template <typename T, int N> bool operator!=(const V<T, N>& a, const V<T, N>& b) { return !(a == b); }

// ---- scalar built-ins (binary32 through libm) -------------------------------------
inline float radians(float d) { return d * 0.017453292519943295f; }
inline float sin(float x) { return ::sinf(x); }
inline float cos(float x) { return ::cosf(x); }
inline float tan(float x) { return ::tanf(x); }
inline float asin(float x) { return ::asinf(x); }
inline float acos(float x) { return ::acosf(x); }
inline float atan(float y, float x) { return ::atan2f(y, x); }
inline float atan(float x) { return ::atanf(x); }
inline float sinh(float x) { return ::sinhf(x); }
inline float cosh(float x) { return ::coshf(x); }
inline float tanh(float x) { return ::tanhf(x); }
inline float pow(float a, float b) { return ::powf(a, b); }
inline float exp(float x) { return ::expf(x); }
inline float log(float x) { return ::logf(x); }
inline float exp2(float x) { return ::exp2f(x); }
inline float log2(float x) { return ::log2f(x); }
inline float sqrt(float x) { return ::sqrtf(x); }
inline float inversesqrt(float x) { return 1.0f / ::sqrtf(x); }
inline float abs(float x) { return ::fabsf(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline int sign(int x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
inline float floor(float x) { return ::floorf(x); }
inline float ceil(float x) { return ::ceilf(x); }
inline float round(float x) { return ::roundf(x); }
inline float trunc(float x) { return ::truncf(x); }
inline float fract(float x) { return x - ::floorf(x); }
inline float mod(float x, float y) { return x - y * ::floorf(x / y); }
// GLSL min/max/clamp: the spec's min(x,y) = y < x ? y : x.
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline uint min(uint a, uint b) { return b < a ? b : a; }
inline uint max(uint a, uint b) { return a < b ? b : a; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float step(float e, float x) { return x < e ? 0.0f : 1.0f; }
inline float smoothstep(float e0, float e1, float x) {
    float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline bool isnan(float x) { return std::isnan(x); }
inline bool isinf(float x) { return std::isinf(x); }
inline uint floatBitsToUint(float f) { uint u; std::memcpy(&u, &f, 4); return u; }
inline int floatBitsToInt(float f) { int u; std::memcpy(&u, &f, 4); return u; }
inline float uintBitsToFloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float intBitsToFloat(int u) { float f; std::memcpy(&f, &u, 4); return f; }

// ---- component-wise lifts ----------------------------------------------------------
#define GLSL_LIFT1(F)                                                                    \
    template <typename T, int N> V<T, N> F(const V<T, N>& a) {                           \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = F(a[i]); return r; }
#define GLSL_LIFT2(F)                                                                    \
    template <typename T, int N> V<T, N> F(const V<T, N>& a, const V<T, N>& b) {         \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = F(a[i], b[i]); return r; }         \
    template <typename T, int N> V<T, N> F(const V<T, N>& a, T b) {                      \
        V<T, N> r; for (int i = 0; i < N; ++i) r[i] = F(a[i], b); return r; }
GLSL_LIFT1(sin) GLSL_LIFT1(cos) GLSL_LIFT1(tan) GLSL_LIFT1(asin) GLSL_LIFT1(acos)
GLSL_LIFT1(atan) GLSL_LIFT1(exp) GLSL_LIFT1(log) GLSL_LIFT1(exp2) GLSL_LIFT1(log2)
GLSL_LIFT1(sqrt) GLSL_LIFT1(inversesqrt) GLSL_LIFT1(abs) GLSL_LIFT1(sign)
GLSL_LIFT1(floor) GLSL_LIFT1(ceil) GLSL_LIFT1(fract) GLSL_LIFT1(round) GLSL_LIFT1(trunc)
GLSL_LIFT1(tanh) GLSL_LIFT1(sinh) GLSL_LIFT1(cosh)
GLSL_LIFT2(pow) GLSL_LIFT2(min) GLSL_LIFT2(max) GLSL_LIFT2(mod) GLSL_LIFT2(atan)
#undef GLSL_LIFT1
#undef GLSL_LIFT2

template <typename T, int N> V<T, N> clamp(const V<T, N>& x, const V<T, N>& lo, const V<T, N>& hi) {
    V<T, N> r; for (int i = 0; i < N; ++i) r[i] = clamp(x[i], lo[i], hi[i]); return r;
}
template <typename T, int N> V<T, N> clamp(const V<T, N>& x, T lo, T hi) {
    V<T, N> r; for (int i = 0; i < N; ++i) r[i] = clamp(x[i], lo, hi); return r;
}
template <int N> V<float, N> mix(const V<float, N>& a, const V<float, N>& b, float t) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = mix(a[i], b[i], t); return r;
}
template <int N> V<float, N> mix(const V<float, N>& a, const V<float, N>& b, const V<float, N>& t) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = mix(a[i], b[i], t[i]); return r;
}
template <int N> V<float, N> mix(const V<float, N>& a, const V<float, N>& b, const V<bool, N>& t) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = t[i] ? b[i] : a[i]; return r;
}
template <int N> V<float, N> step(const V<float, N>& e, const V<float, N>& x) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = step(e[i], x[i]); return r;
}
template <int N> V<float, N> step(float e, const V<float, N>& x) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = step(e, x[i]); return r;
}
template <int N> V<float, N> smoothstep(float e0, float e1, const V<float, N>& x) {
    V<float, N> r; for (int i = 0; i < N; ++i) r[i] = smoothstep(e0, e1, x[i]); return r;
}

// Geometric functions evaluate in the GLSL spec's order (x0*y0 + x1*y1 + ...).
template <int N> float dot(const V<float, N>& a, const V<float, N>& b) {
    float s = a[0] * b[0];
    for (int i = 1; i < N; ++i) s = s + a[i] * b[i];
    return s;
}
inline float dot(float a, float b) { return a * b; }
template <int N> float length(const V<float, N>& a) { return ::sqrtf(dot(a, a)); }
inline float length(float a) { return ::fabsf(a); }
template <int N> float distance(const V<float, N>& a, const V<float, N>& b) { return length(a - b); }
template <int N> V<float, N> normalize(const V<float, N>& a) { return a * (1.0f / length(a)); }
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <int N> V<float, N> reflect(const V<float, N>& i, const V<float, N>& n) {
    return i - 2.0f * dot(n, i) * n;
}
template <int N> V<float, N> refract(const V<float, N>& i, const V<float, N>& n, float eta) {
    float k = 1.0f - eta * eta * (1.0f - dot(n, i) * dot(n, i));
    if (k < 0.0f) return V<float, N>(0.0f);
    return eta * i - (eta * dot(n, i) + ::sqrtf(k)) * n;
}

#define GLSL_CMP(NAME, OP)                                                               \
    template <typename T, int N> V<bool, N> NAME(const V<T, N>& a, const V<T, N>& b) {   \
        V<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] OP b[i]; return r; }
GLSL_CMP(lessThan, <) GLSL_CMP(lessThanEqual, <=) GLSL_CMP(greaterThan, >)
GLSL_CMP(greaterThanEqual, >=) GLSL_CMP(equal, ==) GLSL_CMP(notEqual, !=)
#undef GLSL_CMP
template <int N> bool all(const V<bool, N>& b) { for (int i = 0; i < N; ++i) if (!b[i]) return false; return true; }
template <int N> bool any(const V<bool, N>& b) { for (int i = 0; i < N; ++i) if (b[i]) return true; return false; }
template <int N> V<bool, N> not_(const V<bool, N>& b) { V<bool, N> r; for (int i = 0; i < N; ++i) r[i] = !b[i]; return r; }
template <int N> V<bool, N> isnan(const V<float, N>& a) { V<bool, N> r; for (int i = 0; i < N; ++i) r[i] = std::isnan(a[i]); return r; }
template <int N> V<bool, N> isinf(const V<float, N>& a) { V<bool, N> r; for (int i = 0; i < N; ++i) r[i] = std::isinf(a[i]); return r; }

// ---- samplers: host arrays addressed like WebGL2 textures -------------------------
// An RGBA32F / RGBA32UI texture is a row-major host array of width*height texels.
struct sampler2D {
    const float* data = nullptr;
    int width = 0, height = 0;
};
struct usampler2D {
    const uint* data = nullptr;
    int width = 0, height = 0;
};
inline vec4 texelFetch(const sampler2D& s, ivec2 c, int /*lod*/) {
    if (!s.data || c.x < 0 || c.y < 0 || c.x >= s.width || c.y >= s.height) return vec4(0.0f);
    const float* p = s.data + 4 * ((size_t)c.y * s.width + c.x);
    return vec4(p[0], p[1], p[2], p[3]);
}
inline uvec4 texelFetch(const usampler2D& s, ivec2 c, int /*lod*/) {
    if (!s.data || c.x < 0 || c.y < 0 || c.x >= s.width || c.y >= s.height) return uvec4(0u);
    const uint* p = s.data + 4 * ((size_t)c.y * s.width + c.x);
    return uvec4(p[0], p[1], p[2], p[3]);
}
inline ivec2 textureSize(const sampler2D& s, int) { return ivec2(s.width, s.height); }
inline ivec2 textureSize(const usampler2D& s, int) { return ivec2(s.width, s.height); }

}  // namespace glsl
