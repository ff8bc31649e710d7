// microfacet.cuh — the microfacet machinery the GGX conductor and the rough dielectric share
// (glsl/core/microfacet.glsl:22-54): Trowbridge-Reitz D, separable Smith G1, Heitz 2018
// visible-normal sampling, and their alpha derivatives; Schlick's F0 derivative (the GGX
// conductor and the mirror).
#pragma once
#include "materials/material.cuh"

namespace ptx {

__device__ __forceinline__ f3 mf_to_local(const Frame& f, f3 v) { return f3(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }
__device__ __forceinline__ f3 mf_from_local(const Frame& f, f3 v) { return normalize(f.t * v.x + f.b * v.y + f.n * v.z); }
__device__ __forceinline__ float mf_D(f3 h, float a) {
    float t = h.z * h.z * (a * a - 1.0f) + 1.0f;
    return a * a / (kPi * t * t);
}
__device__ __forceinline__ float mf_G1(f3 v, float a) {
    float c = fabsf(v.z);
    return 2.0f * c / (c + sqrtf(a * a + (1.0f - a * a) * c * c));
}
__device__ __forceinline__ f3 mf_sample_vndf(f3 wol, float a, float u0, float u1) {
    f3 vh = normalize(f3(a * wol.x, a * wol.y, wol.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    f3 T1 = lensq > 0.0f ? f3(-vh.y, vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : f3(1.f, 0.f, 0.f);
    f3 T2 = cross(vh, T1);
    float rr = sqrtf(u0);
    float phi = kTwoPi * u1;
    float t1 = rr * m_cos(phi);
    float t2 = rr * m_sin(phi);
    float s_ = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - s_) * sqrtf(gmax(0.0f, 1.0f - t1 * t1)) + s_ * t2;
    f3 nh = t1 * T1 + t2 * T2 + sqrtf(gmax(0.0f, 1.0f - t1 * t1 - t2 * t2)) * vh;
    return normalize(f3(a * nh.x, a * nh.y, gmax(1e-6f, nh.z)));
}

// d log D / d alpha of the Trowbridge-Reitz distribution at half-vector cosine hz.
__device__ __forceinline__ float mf_dlogD(float hz, float a) {
    float t = hz * hz * (a * a - 1.0f) + 1.0f;
    return 2.0f / a - 4.0f * a * hz * hz / t;
}
// d log G1 / d alpha of the separable Smith term at cosine c.
__device__ __forceinline__ float mf_dlogG1(float c, float a) {
    c = fabsf(c);
    float s = sqrtf(a * a + (1.0f - a * a) * c * c);
    return -(a * (1.0f - c * c) / s) / (c + s);
}
// d log F_c / d F0_c of Schlick's Fresnel F = F0 + (1 - F0) (1 - c)^5, per channel.
__device__ __forceinline__ f3 schlick_dlog_f0(f3 f0, float c) {
    const float s5 = m_pow(1.0f - c, 5.0f);
    const f3 F = f0 + (f3(1.0f) - f0) * s5;
    return f3(1.0f - s5) / vmax(F, f3(1e-20f));
}

}  // namespace ptx
