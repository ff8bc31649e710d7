// registry.cuh — the light kinds of this build, one line each (the reference's LIGHT_KINDS,
// src/components/lights/index.ts).  A new kind is a header in this folder and a line here;
// its PTR_LIGHT_* value is a C ABI constant (include/ptx_rt.h) and its host-side record a
// row of pathtracerglsl_b200/occupants.py.  Light sampling and MIS reach every kind through
// dispatch_light / light_in over this list; the per-scene kernels keep the scene's kinds
// (has_light).
#pragma once
#include "lights/quad.cuh"
#include "lights/sphere.cuh"
#include "lights/point.cuh"
#include "lights/mesh.cuh"

namespace ptx {

using LightKinds = OccupantList<
    QuadLight,
    SphereLight,
    PointLight,
    MeshLight>;
static_assert(ids_distinct(LightKinds{}), "light kind ids must be distinct and below 32");

// f(K{}) for the kind `kind` among those P admits (GUARDED: the caller knows `kind` is one
// of them); false when none matches.
template <template <class> class P, bool GUARDED = false, class F>
__device__ __forceinline__ bool dispatch_light(int kind, F& f) {
    return dispatch_occupant<P, LightPresent, GUARDED>(kind, f, LightKinds{});
}
template <template <class> class P>
__device__ __forceinline__ bool light_in(int kind) { return occupant_in<P>(kind, LightKinds{}); }

}  // namespace ptx
