// registry.cuh — the material models of this build, one line each (the reference's
// MATERIAL_MODELS, src/components/materials/index.ts).  A new model is a header in this
// folder and a line here; its PTR_MAT_* value is a C ABI constant (include/ptx_rt.h) and its
// host-side packing a row of pathtracerglsl_b200/occupants.py.  k_shade reaches every model
// through dispatch_material / material_in over this list, and the per-scene kernels keep only the
// models of the scene's census (has_mat).
#pragma once
#include "materials/lambert.cuh"
#include "materials/dielectric.cuh"
#include "materials/ggx.cuh"
#include "materials/mirror.cuh"
#include "materials/null.cuh"
#include "materials/rough_dielectric.cuh"

namespace ptx {

using MaterialModels = OccupantList<
    Lambert,
    Dielectric,
    GGX,
    Mirror,
    Null,
    RoughDielectric>;
static_assert(ids_distinct(MaterialModels{}), "material model ids must be distinct and below 32");

// f(M{}) for the model of `model` among those P admits (GUARDED: the caller knows `model`
// is one of them); false when none matches.
template <template <class> class P, bool GUARDED = false, class F>
__device__ __forceinline__ bool dispatch_material(int model, F& f) {
    return dispatch_occupant<P, MatPresent, GUARDED>(model, f, MaterialModels{});
}
template <template <class> class P>
__device__ __forceinline__ bool material_in(int model) { return occupant_in<P>(model, MaterialModels{}); }

}  // namespace ptx
