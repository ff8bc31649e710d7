// material.cuh — the surface occupant interface: what k_shade asks of a material model.
//
// A material model is one header in this folder defining a struct derived from
// MaterialModel, plus one line in registry.cuh (the device counterpart of the reference's
// MATERIAL_MODELS registry, src/components/materials/index.ts, and of its generated dispatch
// over it, src/compiler/generate/features/materials.ts:902-954).  The per-scene kernels
// pick models up through the census mask (has_mat(kModel)): absent models fold away.
//
//   kModel        its ptr_material.model value (PTR_MAT_*, a C ABI constant)
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

template <class... M> struct ModelList {};

// A model takes part in a dispatch when the build holds it and, for a non-delta dispatch,
// when it has a non-delta lobe.
template <bool NONDELTA, class M>
__host__ __device__ constexpr bool model_present() { return has_mat(M::kModel) && (!NONDELTA || M::kNonDelta); }
template <bool NONDELTA, class... M>
__host__ __device__ constexpr bool any_present(ModelList<M...>) { return (false || ... || model_present<NONDELTA, M>()); }

// Calls f(M{}) for the registered model M of `model`.  Models the build lacks are not
// instantiated; the last present model in registry order takes whatever was not matched
// before it without a comparison (the final else of a generated if-chain), so a build
// holding one model calls it directly.  False when the build holds no candidate.
template <bool NONDELTA, class F>
__device__ __forceinline__ bool dispatch_model(int, F&, ModelList<>) { return false; }
template <bool NONDELTA, class F, class M0, class... Ms>
__device__ __forceinline__ bool dispatch_model(int model, F& f, ModelList<M0, Ms...>) {
    if constexpr (model_present<NONDELTA, M0>()) {
        if constexpr (!any_present<NONDELTA>(ModelList<Ms...>{})) {
            f(M0{});
            return true;
        } else {
            if (model == M0::kModel) {
                f(M0{});
                return true;
            }
        }
    }
    return dispatch_model<NONDELTA>(model, f, ModelList<Ms...>{});
}

// True when `model` is a present model whose trait P holds (compared only where needed).
template <template <class> class P>
__device__ __forceinline__ bool model_has(int, ModelList<>) { return false; }
template <template <class> class P, class M0, class... Ms>
__device__ __forceinline__ bool model_has(int model, ModelList<M0, Ms...>) {
    if constexpr (has_mat(M0::kModel) && P<M0>::value) {
        if (model == M0::kModel) return true;
    }
    return model_has<P>(model, ModelList<Ms...>{});
}
template <class M> struct IsNonDelta { static constexpr bool value = M::kNonDelta; };
template <class M> struct IsSphereQuery { static constexpr bool value = M::kSphereQuery; };

}  // namespace ptx
