// ggx.cuh — the GGX conductor (materials/ggx/ggx.glsl:16-64): Trowbridge-Reitz microfacets
// with visible-normal sampling and Schlick Fresnel of F0; alpha per triangle where the mesh
// carries one.  Adjoint: F0 (colour slots) and, for the material's own alpha, alpha.
#pragma once
#include "materials/microfacet.cuh"

namespace ptx {

template <class Col>
__device__ __forceinline__ Col ggx_eval(f3 wi, f3 wo, const Hit& h, Col f0, float a) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return Col(0.0f);
    f3 hh = normalize(wil + wol);
    Col F = schlick_fresnel(f0, fabsf(dot(wol, hh)));
    return F * (mf_D(hh, a) * mf_G1(wil, a) * mf_G1(wol, a) / (4.0f * fabsf(wil.z) * fabsf(wol.z)));
}
template <class Col>
__device__ __forceinline__ ISample<Col> ggx_sample(f3 wo, const Hit& h, Col f0, float a, float u0, float u1) {
    f3 wol = mf_to_local(h.frame, wo);
    float side = wol.z < 0.0f ? -1.0f : 1.0f;
    wol = wol * side;
    f3 hh = mf_sample_vndf(wol, a, u0, u1);
    f3 i = -wol;
    f3 wil = i - 2.0f * dot(hh, i) * hh;
    ISample<Col> s;
    if (wil.z <= 0.0f) { s.wi = wo; s.weight = Col(0.0f); s.pdf = 0.0f; s.flags = kLobeReflection; return s; }
    Col F = schlick_fresnel(f0, fabsf(dot(wol, hh)));
    s.weight = F * mf_G1(wil, a);
    s.pdf = mf_G1(wol, a) * mf_D(hh, a) / (4.0f * fabsf(wol.z));
    s.flags = kLobeReflection;
    s.wi = mf_from_local(h.frame, wil * side);
    return s;
}
__device__ __forceinline__ float ggx_pdf(f3 wi, f3 wo, const Hit& h, float a) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return 0.0f;
    f3 hh = normalize(wil + wol);
    return mf_G1(wol, a) * mf_D(hh, a) / (4.0f * fabsf(wol.z));
}
// d log f / d alpha for the pair (wi, wo) (Fresnel does not depend on alpha).
__device__ __forceinline__ float ggx_dlog_alpha(f3 wi, f3 wo, const Hit& h, float a) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return 0.0f;
    f3 hh = normalize(wil + wol);
    return mf_dlogD(hh.z, a) + mf_dlogG1(wil.z, a) + mf_dlogG1(wol.z, a);
}
// d log f_c / d F0_c for the pair (wi, wo): only Fresnel depends on F0.
__device__ __forceinline__ f3 ggx_dlog_f0(f3 wi, f3 wo, const Hit& h, f3 f0) {
    f3 wil = mf_to_local(h.frame, wi), wol = mf_to_local(h.frame, wo);
    if (wil.z * wol.z <= 0.0f) return f3(0.0f);
    f3 hh = normalize(wil + wol);
    return schlick_dlog_f0(f0, fabsf(dot(wol, hh)));
}

struct GGX : MaterialModel {
    static constexpr int kId = PTR_MAT_GGX;
    static constexpr bool kNonDelta = true;
    __device__ static f3 aov(const ptr_material& m) { return ld3(m.f0); }
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float, float u0, float u1) {
        return ggx_sample(wo, s.hit, Colors<Col>::f0(s.S, s.mat, s.wl), s.alpha, u0, u1);
    }
    template <class Col>
    __device__ static Col eval(const MatSite<Col>& s, f3 wi, f3 wo) {
        return ggx_eval(wi, wo, s.hit, Colors<Col>::f0(s.S, s.mat, s.wl), s.alpha);
    }
    template <class Col>
    __device__ static float pdf(const MatSite<Col>& s, f3 wi, f3 wo) { return ggx_pdf(wi, wo, s.hit, s.alpha); }
    __device__ static void nee_grad(const MatSite<f3>& s, f3 wi, f3 wo, NeeGrad& g) {
        g.kind = kGradKindGGX;
        g.dnee = ggx_dlog_f0(wi, wo, s.hit, ld3(s.m.f0));
        g.dw = s.hit.alpha < 0.0f ? ggx_dlog_alpha(wi, wo, s.hit, s.alpha) : 0.0f;
    }
    __device__ static void cont_grad(const MatSite<f3>& s, const ISample<f3>& bs, f3 wo, const GradAcc& ga, f3 lrem,
                                     bool shadow, NeeGrad& g) {
        f3 dF = ggx_dlog_f0(bs.wi, wo, s.hit, ld3(s.m.f0));
        ga.vec(s.mat, PTR_GRAD_COLOR_R, lrem, dF);
        if (shadow) g.dnee = g.dnee - dF;
        if (s.hit.alpha < 0.0f) {   // a per-triangle alpha is not a material parameter
            float da = ggx_dlog_alpha(bs.wi, wo, s.hit, s.alpha);
            ga.scl(s.mat, PTR_GRAD_ALPHA, lrem, da);
            if (shadow) g.dw -= da;
        }
    }
};

}  // namespace ptx
