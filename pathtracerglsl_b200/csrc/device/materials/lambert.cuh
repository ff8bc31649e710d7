// lambert.cuh — the Lambert diffuse reflector (materials/lambert/lambert.glsl:7-37):
// cosine-weighted sampling about the side wo lies on; the only model whose emission makes a
// surface an emitter.  Adjoint: the albedo (colour slots).
#pragma once
#include "materials/material.cuh"

namespace ptx {

template <class Col>
__device__ __forceinline__ Col lambert_eval(f3 wi, f3 wo, const Hit& h, Col albedo) {
    if (dot(wi, h.frame.n) * dot(wo, h.frame.n) <= 0.0f) return Col(0.0f);
    return albedo * (1.0f / kPi);
}
template <class Col>
__device__ __forceinline__ ISample<Col> lambert_sample(f3 wo, const Hit& h, Col albedo, float u0, float u1) {
    f3 n = dot(wo, h.frame.n) < 0.0f ? -h.frame.n : h.frame.n;
    float cos_theta = sqrtf(u1);
    float sin_theta = sqrtf(gmax(0.0f, 1.0f - u1));
    float phi = kTwoPi * u0;
    float sp, cp;
    sp = m_sin(phi);
    cp = m_cos(phi);
    ISample<Col> s;
    s.wi = normalize(h.frame.t * (sin_theta * cp) + h.frame.b * (sin_theta * sp) + n * cos_theta);
    s.weight = albedo;
    s.pdf = cos_theta * (1.0f / kPi);
    s.flags = kLobeReflection;
    return s;
}
__device__ __forceinline__ float lambert_pdf(f3 wi, f3 wo, const Hit& h) {
    float c = dot(wi, h.frame.n) * signf(dot(wo, h.frame.n));
    return gmax(0.0f, c) * (1.0f / kPi);
}

struct Lambert : MaterialModel {
    static constexpr int kId = PTR_MAT_LAMBERT;
    static constexpr bool kNonDelta = true;
    __device__ static f3 aov(const ptr_material& m) { return ld3(m.albedo); }
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float, float u0, float u1) {
        return lambert_sample(wo, s.hit, Colors<Col>::albedo(s.S, s.mat, s.wl), u0, u1);
    }
    template <class Col>
    __device__ static Col eval(const MatSite<Col>& s, f3 wi, f3 wo) {
        return lambert_eval(wi, wo, s.hit, Colors<Col>::albedo(s.S, s.mat, s.wl));
    }
    template <class Col>
    __device__ static float pdf(const MatSite<Col>& s, f3 wi, f3 wo) { return lambert_pdf(wi, wo, s.hit); }
    // f = albedo / pi and w_cont = albedo: d log / d albedo_c = 1 / albedo_c for both
    __device__ static void nee_grad(const MatSite<f3>& s, f3, f3, NeeGrad& g) {
        g.kind = kGradKindAlbedo;
        g.dnee = f3(1.0f) / vmax(ld3(s.m.albedo), f3(1e-20f));
    }
    __device__ static void cont_grad(const MatSite<f3>& s, const ISample<f3>&, f3, const GradAcc& ga, f3 lrem, bool shadow,
                                     NeeGrad& g) {
        f3 dlog = f3(1.0f) / vmax(ld3(s.m.albedo), f3(1e-20f));
        ga.vec(s.mat, PTR_GRAD_ALBEDO_R, lrem, dlog);
        if (shadow) g.dnee = g.dnee - dlog;
    }
};

}  // namespace ptx
