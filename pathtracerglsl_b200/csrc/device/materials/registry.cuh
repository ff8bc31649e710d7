// registry.cuh — the material models of this build, one line each (the reference's
// MATERIAL_MODELS, src/components/materials/index.ts).  A new model is a header in this
// folder and a line here; its PTR_MAT_* value is a C ABI constant (include/ptx_rt.h) and its
// host-side packing a row of pathtracerglsl_b200/occupants.py.  k_shade reaches every model
// through dispatch_model / model_has over this list, and the per-scene kernels keep only the
// models of the scene's census (has_mat).
#pragma once
#include "materials/lambert.cuh"
#include "materials/dielectric.cuh"
#include "materials/ggx.cuh"
#include "materials/mirror.cuh"
#include "materials/null.cuh"
#include "materials/rough_dielectric.cuh"

namespace ptx {

using MaterialModels = ModelList<
    Lambert,
    Dielectric,
    GGX,
    Mirror,
    Null,
    RoughDielectric>;

// every model id fits the census mask and appears once
template <class... M>
__host__ __device__ constexpr bool models_distinct(ModelList<M...>) {
    unsigned bits = 0u;
    bool ok = true;
    ((ok = ok && M::kModel >= 0 && M::kModel < 32 && !(bits & (1u << M::kModel)), bits |= 1u << M::kModel), ...);
    return ok;
}
static_assert(models_distinct(MaterialModels{}), "material model ids must be distinct and below 32");

}  // namespace ptx
