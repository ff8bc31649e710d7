// material.cuh — the surface occupant interface: what k_shade asks of a material model.
//
// A material model is one header in this folder defining a struct derived from
// MaterialModel, plus one line in registry.cuh (the device counterpart of the reference's
// MATERIAL_MODELS registry, src/components/materials/index.ts, and of its generated dispatch
// over it, src/compiler/generate/features/materials.ts:902-954).  The per-scene kernels
// pick models up through the census mask (has_mat(kId)): absent models fold away.
//
//   kId           its ptr_material.model value (PTR_MAT_*, a C ABI constant)
//   kNonDelta     it has a non-delta lobe: NEE and MIS evaluate eval() / pdf() toward lights
//   kSphereQuery  light selection queries a sphere of directions around the point (a
//                 transmissive non-delta lobe sees lights on both sides)
//   aov(m)        the first-hit albedo picture's colour
//   sample(...)   the continuation lobe: direction, weight f cos / pdf, pdf, lobe flags
//   eval / pdf    the non-delta lobe toward a light direction (kNonDelta models only)
//   nee_grad      the adjoint's shadow-record terms: d log f toward the light
//   cont_grad     the adjoint's continuation terms: d log (weight) of the sampled lobe
#pragma once
#include "occupants.cuh"
#include "adjoint.cuh"
#include "occupant.cuh"

namespace ptx {

// Everything a model reads at a surface hit.
template <class Col>
struct MatSite {
    const DevScene& S;
    int mat;                  // material index
    const ptr_material& m;
    const Hit& hit;
    const Wl& wl;
    float alpha;              // the triangle's GGX alpha where the mesh carries one, else the material's
    float n_from, n_to;       // IORs of the regions on the incident and the far side
};

// The adjoint's record of a vertex's NEE query: which slots its lobe derivative feeds
// (kGradKind*), the per-channel part and the scalar part.
struct NeeGrad {
    int kind;
    f3 dnee;
    float dw;
};

struct MaterialModel {
    static constexpr bool kNonDelta = false;
    static constexpr bool kSphereQuery = false;
    __device__ static f3 aov(const ptr_material& m) { return ld3(m.transmittance); }
    __device__ static void nee_grad(const MatSite<f3>&, f3, f3, NeeGrad&) {}
    __device__ static void cont_grad(const MatSite<f3>&, const ISample<f3>&, f3, const GradAcc&, f3, bool, NeeGrad&) {}
};

// Family predicates of material dispatches (occupant.cuh): the build holds the model, and
// it has a non-delta lobe / queries lights over the sphere.
template <class M> struct MatPresent { static constexpr bool value = has_mat(M::kId); };
template <class M> struct MatNonDelta { static constexpr bool value = has_mat(M::kId) && M::kNonDelta; };
template <class M> struct MatSphereQuery { static constexpr bool value = has_mat(M::kId) && M::kSphereQuery; };

}  // namespace ptx
