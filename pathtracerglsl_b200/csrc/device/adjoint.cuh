// adjoint.cuh — derivative terms of the path-replay adjoint (no counterpart in the reference).
//
// Path replay backpropagation (Vicini, Speierer & Jakob, "Path Replay Backpropagation",
// SIGGRAPH 2021) with detached sampling: a path's contribution is a product of per-vertex
// weights w_j = f_j / p_j whose sampling densities p_j are held fixed, so the derivative of
// everything the path gathers after vertex j is (radiance still to come) * d log f_j / d theta.
// The replay knows the radiance still to come because the forward pass of the same
// counter-based path stored its total.  MIS weights and roulette probabilities are
// detached too (they sum to one / keep the estimator unbiased for every theta, so their
// derivatives vanish in expectation).
//
// Per material, PTR_GRAD_SLOTS parameters (include/ptx_rt.h): the model's colour (rgb:
// Lambert albedo, GGX / mirror F0, dielectric transmittance), GGX alpha, dielectric IOR, grey
// homogeneous medium sigma_t, single-scattering albedo and HG g.
// For the IOR only the interface terms (Fresnel lobe choice, the eta^2 radiance factor) are
// differentiated: the refracted direction's own dependence on the IOR would need an
// attached derivative of every later vertex.
#pragma once
#include "occupants.cuh"

namespace ptx {

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
// d log f / d alpha of the GGX conductor for the pair (wi, wo) (Fresnel does not depend on alpha).
__device__ __forceinline__ float ggx_dlog_alpha(f3 wi, f3 wo, const Hit& h, float a) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return 0.0f;
    f3 hh = normalize(wil + wol);
    return mf_dlogD(hh.z, a) + mf_dlogG1(wil.z, a) + mf_dlogG1(wol.z, a);
}
// d log F_c / d F0_c of Schlick's Fresnel F = F0 + (1 - F0) (1 - c)^5, per channel.
__device__ __forceinline__ f3 schlick_dlog_f0(f3 f0, float c) {
    const float s5 = m_pow(1.0f - c, 5.0f);
    const f3 F = f0 + (f3(1.0f) - f0) * s5;
    return f3(1.0f - s5) / vmax(F, f3(1e-20f));
}
// d log f_c / d F0_c of the GGX conductor for the pair (wi, wo): only Fresnel depends on F0.
__device__ __forceinline__ f3 ggx_dlog_f0(f3 wi, f3 wo, const Hit& h, f3 f0) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return f3(0.0f);
    f3 hh = normalize(wil + wol);
    return schlick_dlog_f0(f0, fabsf(dot(wol, hh)));
}
// d log p_HG / d g (forward convention, hg.glsl:11-42).
__device__ __forceinline__ float hg_dlog_g(f3 wi, f3 wo, float g) {
    float c = dot(wi, -wo);
    float d = gmax(1.0f + g * g - 2.0f * g * c, 1e-8f);
    return -2.0f * g / (1.0f - g * g) - 1.5f * (2.0f * g - 2.0f * c) / d;
}
// Exact unpolarised Fresnel in float64 (the derivative below differences it).
__device__ __forceinline__ double fresnel_d(double cos_i, double eta) {
    double sin2_t = eta * eta * (1.0 - cos_i * cos_i);
    if (sin2_t >= 1.0) return 1.0;
    double cos_t = sqrt(1.0 - sin2_t);
    double rp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    double rs = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5 * (rp * rp + rs * rs);
}
// d log w / d ior of the smooth dielectric's sampled lobe, where ior is the IOR of the
// region the interface belongs to (n_t on entry, n_i on exit).  Reflection: w = F / F_detached;
// refraction: w = T (n_i/n_t)^2 (1-F) / (1-F)_detached.
__device__ __forceinline__ float dielectric_dlog_ior(float cos_i, float n_i, float n_t, bool entering, bool refracted) {
    const double eta = (double)n_i / (double)n_t;
    const double deta = entering ? -(double)n_i / ((double)n_t * (double)n_t) : 1.0 / (double)n_t;
    const double c = (double)fminf(fmaxf(cos_i, 1e-6f), 1.0f);
    const double h = 1e-6 * eta;
    const double F = fresnel_d(c, eta);
    const double dF = (fresnel_d(c, eta + h) - fresnel_d(c, eta - h)) / (2.0 * h) * deta;
    if (!refracted) return F > 0.0 ? (float)(dF / F) : 0.0f;
    const double own = entering ? (double)n_t : (double)n_i;
    const double dscale = (entering ? -2.0 : 2.0) / own;
    return (float)(dscale - (F < 1.0 ? dF / (1.0 - F) : 0.0));
}

// Grey homogeneous medium: sigma_t and the single-scattering albedo a
// (sigma_s = a sigma_t, sigma_a = (1 - a) sigma_t), read from channel 0.
struct GreyMedium { float st, a; };
__device__ __forceinline__ GreyMedium grey_medium(const ptr_material& m) {
    GreyMedium g;
    g.st = m.sigma_a[0] + m.sigma_s[0];
    g.a = g.st > 0.0f ? m.sigma_s[0] / g.st : 0.0f;
    return g;
}

// Per-block gradient accumulators in shared memory (float64), flushed to the global
// float64 gradient buffer at the end of the kernel.
struct GradAcc {
    double* s;     // shared: PTR_GRAD_SLOTS per material
    f3 dl;         // the path's adjoint radiance (dLoss/dI of its pixel / spp)
    // per-channel slots [slot0, slot0+2]: grad_c += dl_c X_c dlog_c
    __device__ __forceinline__ void vec(int mat, int slot0, f3 X, f3 dlog) const {
        double* b = s + PTR_GRAD_SLOTS * mat + slot0;
        float v0 = dl.x * X.x * dlog.x, v1 = dl.y * X.y * dlog.y, v2 = dl.z * X.z * dlog.z;
        if (v0 != 0.0f) atomicAdd(b + 0, (double)v0);
        if (v1 != 0.0f) atomicAdd(b + 1, (double)v1);
        if (v2 != 0.0f) atomicAdd(b + 2, (double)v2);
    }
    // scalar slot: grad += (dl . X) dlog
    __device__ __forceinline__ void scl(int mat, int slot, f3 X, float dlog) const {
        float v = (dl.x * X.x + dl.y * X.y + dl.z * X.z) * dlog;
        if (v != 0.0f) atomicAdd(s + PTR_GRAD_SLOTS * mat + slot, (double)v);
    }
};

__device__ __forceinline__ void grad_block_init(double* s, int n) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) s[k] = 0.0;
    __syncthreads();
}
__device__ __forceinline__ void grad_block_flush(const double* s, int n, double* g) {
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        if (s[k] != 0.0) atomicAdd(g + k, s[k]);
}

// Shadow-record kinds of the per-vertex lobe derivative D = dlog f(wi_light) - dlog w_cont.
// GGX: the per-channel F0 part in xyz, the alpha part in w.
constexpr int kGradKindNone = 0, kGradKindAlbedo = 1, kGradKindGGX = 2, kGradKindPhase = 3;

}  // namespace ptx
