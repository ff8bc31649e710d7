// null.cuh — the null interface ('none'): a medium boundary with no optical surface.  In
// kernels built with media the transport passes straight through it (pt.ts:404-417) before
// any surface work; without media it samples as a smooth dielectric between the IORs of
// its two sides (its own region's IOR is 1), weighted by the transmittance.
#pragma once
#include "materials/dielectric.cuh"

namespace ptx {

struct Null : MaterialModel {
    static constexpr int kId = PTR_MAT_NONE;
    template <class Col>
    __device__ static ISample<Col> sample(const MatSite<Col>& s, f3 wo, float uc, float, float) {
        return dielectric_sample(wo, s.hit, Colors<Col>::tint(s.S, s.mat, s.wl), s.n_from, s.n_to, uc);
    }
};

}  // namespace ptx
