// dielectric.cuh — the smooth dielectric with the eta^2 radiance factor
// (materials/dielectric/dielectric.glsl:14-52): one delta lobe chosen by exact Fresnel.
// Adjoint: the transmittance (colour slots, refraction only) and the IOR's interface terms.
#pragma once
#include "materials/material.cuh"

namespace ptx {

template <class Col>
__device__ __forceinline__ ISample<Col> dielectric_sample(f3 wo, const Hit& h, Col tint, float n_i, float n_t, float uc) {
    float eta = n_i / n_t;
    f3 n = h.frame.n;
    float cos_i = clampf(dot(wo, n), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_i, eta);
    ISample<Col> s;
    if (uc < F) {
        s.wi = normalize(2.0f * cos_i * n - wo);
        s.weight = Col(1.0f);
        s.pdf = 0.0f;
        s.flags = kLobeReflection | kLobeDelta;
    } else {
        float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
        float cos_t = sqrtf(gmax(0.0f, 1.0f - sin2_t));
        s.wi = normalize(-eta * wo + (eta * cos_i - cos_t) * n);
        float radiance_scale = (n_i * n_i) / (n_t * n_t);
        s.weight = tint * radiance_scale;
        s.pdf = 0.0f;
        s.flags = kLobeTransmission | kLobeDelta;
    }
    return s;
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
// d log w / d ior of the sampled lobe, where ior is the IOR of the region the interface
// belongs to (n_t on entry, n_i on exit).  Reflection: w = F / F_detached; refraction:
// w = T (n_i/n_t)^2 (1-F) / (1-F)_detached.
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

struct Dielectric : MaterialModel {
    static constexpr int kId = PTR_MAT_DIELECTRIC;
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float uc, float, float) {
        return dielectric_sample(wo, s.hit, Colors<Col>::tint(s.S, s.mat, s.wl), s.n_from, s.n_to, uc);
    }
    __device__ static void cont_grad(const MatSite<f3>& s, const ISample<f3>& bs, f3 wo, const GradAcc& ga, f3 lrem, bool,
                                     NeeGrad&) {
        const Hit& hit = s.hit;
        if (bs.flags & kLobeTransmission)   // w = T (n_i / n_t)^2: d log w / d T = 1 / T
            ga.vec(s.mat, PTR_GRAD_COLOR_R, lrem, f3(1.0f) / vmax(ld3(s.m.transmittance), f3(1e-20f)));
        const bool entering = hit.region_to == hit.region_owner;
        if (entering || hit.region_from == hit.region_owner) {
            float ci = dot(wo, hit.frame.n);
            float d = dielectric_dlog_ior(ci, s.n_from, s.n_to, entering, (bs.flags & kLobeTransmission) != 0u);
            ga.scl(s.mat, PTR_GRAD_IOR, lrem, d);
        }
    }
};

}  // namespace ptx
