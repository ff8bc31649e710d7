// mirror.cuh — the mirror (materials/mirror/mirror.glsl): one delta reflection lobe
// weighted by Schlick Fresnel of F0.  Adjoint: F0 (colour slots).
#pragma once
#include "materials/microfacet.cuh"

namespace ptx {

template <class Col>
__device__ __forceinline__ ISample<Col> mirror_sample(f3 wo, const Hit& h, Col f0) {
    f3 n = h.frame.n;
    float cos_i = clampf(dot(wo, n), 1e-6f, 1.0f);
    ISample<Col> s;
    s.wi = normalize(2.0f * cos_i * n - wo);
    s.weight = schlick_fresnel(f0, cos_i);
    s.pdf = 0.0f;
    s.flags = kLobeReflection | kLobeDelta;
    return s;
}

struct Mirror : MaterialModel {
    static constexpr int kId = PTR_MAT_MIRROR;
    __device__ static f3 aov(const ptr_material& m) { return ld3(m.f0); }
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float, float, float) {
        return mirror_sample(wo, s.hit, Colors<Col>::f0(s.S, s.mat, s.wl));
    }
    // w = Schlick F(F0, cos_i)
    __device__ static void cont_grad(const MatSite<f3>& s, const ISample<f3>&, f3 wo, const GradAcc& ga, f3 lrem, bool,
                                     NeeGrad&) {
        float ci = clampf(dot(wo, s.hit.frame.n), 1e-6f, 1.0f);
        ga.vec(s.mat, PTR_GRAD_COLOR_R, lrem, schlick_dlog_f0(ld3(s.m.f0), ci));
    }
};

}  // namespace ptx
