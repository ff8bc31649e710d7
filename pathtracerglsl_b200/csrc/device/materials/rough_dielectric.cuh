// rough_dielectric.cuh — the rough dielectric (materials/rough_dielectric/rough_dielectric.glsl):
// the two-lobe microfacet BSDF of Walter et al. 2007 with visible-normal sampling, exact
// Fresnel and the eta^2 radiance factor on the transmission lobe.  wo lies in the frame's
// upper hemisphere (the frame faces region_from); eta = n_i / n_t; equal indices make the
// interface a delta pass-through.  Non-delta on both sides, so light selection queries a
// sphere of directions.  Not differentiated by the adjoint.
#pragma once
#include "materials/microfacet.cuh"

namespace ptx {

// generalised half vector of a (wi, wo) pair, faced upward; false for a degenerate pair or
// a back-facing microfacet (shared by eval and pdf)
__device__ __forceinline__ bool rough_half(f3 wil, f3 wol, float eta, f3& m) {
    float etap = wil.z > 0.0f ? 1.0f : 1.0f / eta;
    m = wil * etap + wol;
    if (dot(m, m) <= 0.0f) return false;
    m = normalize(m);
    if (m.z < 0.0f) m = -m;
    return dot(m, wil) * wil.z >= 0.0f && dot(m, wol) * wol.z >= 0.0f;
}
template <class Col>
__device__ __forceinline__ Col rough_dielectric_eval(f3 wi, f3 wo, const Hit& h, Col tint, float a, float n_i, float n_t) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wol.z <= 0.0f || wil.z == 0.0f) return Col(0.0f);
    if (n_i == n_t) return Col(0.0f);
    float eta = n_i / n_t;
    f3 m;
    if (!rough_half(wil, wol, eta, m)) return Col(0.0f);
    float cos_om = clampf(fabsf(dot(wol, m)), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    float DG = mf_D(m, a) * mf_G1(wol, a) * mf_G1(wil, a);
    if (wil.z > 0.0f) return Col(1.0f) * (DG * F / (4.0f * wil.z * wol.z));
    float denom = dot(wil, m) + dot(wol, m) * eta;
    denom *= denom;
    float ft = DG * (1.0f - F) * fabsf(dot(wil, m) * dot(wol, m) / (wil.z * wol.z * denom));
    return tint * (ft * eta * eta);
}
__device__ __forceinline__ float rough_dielectric_pdf(f3 wi, f3 wo, const Hit& h, float a, float n_i, float n_t) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wol.z <= 0.0f || wil.z == 0.0f) return 0.0f;
    if (n_i == n_t) return 0.0f;
    float eta = n_i / n_t;
    f3 m;
    if (!rough_half(wil, wol, eta, m)) return 0.0f;
    float cos_om = clampf(fabsf(dot(wol, m)), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    if (wil.z > 0.0f) return F * mf_G1(wol, a) * mf_D(m, a) / (4.0f * wol.z);
    float denom = dot(wil, m) + dot(wol, m) * eta;
    denom *= denom;
    return (1.0f - F) * mf_G1(wol, a) * mf_D(m, a) * cos_om / wol.z * fabsf(dot(wil, m)) / denom;
}
template <class Col>
__device__ __forceinline__ ISample<Col> rough_dielectric_sample(f3 wo, const Hit& h, Col tint, float a, float n_i, float n_t,
                                                                float uc, float u0, float u1) {
    f3 wol = mf_to_local(h.frame, wo);
    ISample<Col> s;
    s.wi = wo;
    s.weight = Col(0.0f);
    s.pdf = 0.0f;
    s.flags = kLobeReflection;
    if (wol.z <= 0.0f) return s;
    float eta = n_i / n_t;
    if (n_i == n_t) {   // index-matched: the delta pass-through
        s.wi = -wo;
        s.weight = tint;
        s.flags = kLobeTransmission | kLobeDelta;
        return s;
    }
    f3 m = mf_sample_vndf(wol, a, u0, u1);
    float cos_om = clampf(dot(wol, m), 1e-6f, 1.0f);
    float F = dielectric_fresnel(cos_om, eta);
    f3 wil;
    if (uc < F) {
        f3 i = -wol;
        wil = i - 2.0f * dot(m, i) * m;
        if (wil.z <= 0.0f) return s;
        s.weight = Col(1.0f) * mf_G1(wil, a);
        s.pdf = F * mf_G1(wol, a) * mf_D(m, a) / (4.0f * wol.z);
        s.flags = kLobeReflection;
    } else {
        float sin2_t = eta * eta * (1.0f - cos_om * cos_om);
        float cos_t = sqrtf(gmax(0.0f, 1.0f - sin2_t));
        wil = normalize(-eta * wol + (eta * cos_om - cos_t) * m);
        if (wil.z >= 0.0f) return s;
        float denom = dot(wil, m) + dot(wol, m) * eta;
        denom *= denom;
        s.weight = tint * (mf_G1(wil, a) * eta * eta);
        s.pdf = (1.0f - F) * mf_G1(wol, a) * mf_D(m, a) * cos_om / wol.z * fabsf(dot(wil, m)) / denom;
        s.flags = kLobeTransmission;
    }
    s.wi = mf_from_local(h.frame, wil);
    return s;
}

struct RoughDielectric : MaterialModel {
    static constexpr int kId = PTR_MAT_ROUGH_DIELECTRIC;
    static constexpr bool kNonDelta = true;
    static constexpr bool kSphereQuery = true;
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float uc, float u0, float u1) {
        return rough_dielectric_sample(wo, s.hit, Colors<Col>::tint(s.S, s.mat, s.wl), s.alpha, s.n_from, s.n_to, uc, u0, u1);
    }
    template <class Col>
    __device__ static Col eval(const MatSite<Col>& s, f3 wi, f3 wo) {
        return rough_dielectric_eval(wi, wo, s.hit, Colors<Col>::tint(s.S, s.mat, s.wl), s.alpha, s.n_from, s.n_to);
    }
    template <class Col>
    __device__ static float pdf(const MatSite<Col>& s, f3 wi, f3 wo) {
        return rough_dielectric_pdf(wi, wo, s.hit, s.alpha, s.n_from, s.n_to);
    }
};

}  // namespace ptx
