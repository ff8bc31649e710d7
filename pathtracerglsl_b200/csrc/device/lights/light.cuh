// light.cuh — the light occupant interface: what NEE, MIS and the equiangular medium
// estimator ask of a light kind.
//
// A light kind is one header in this folder defining a struct derived from LightKind, plus
// one line in registry.cuh (the device counterpart of the reference's LIGHT_KINDS registry,
// src/components/lights/index.ts, and of its generated dispatch, features/lighting.ts:
// 546-693).  The per-scene kernels keep only the scene's kinds (has_light(kId)).
//
//   kId          its ptr_light.kind value (PTR_LIGHT_*, a C ABI constant)
//   kDelta       a delta light (no area: never hit, not in MIS)
//   sample(...)  a direction toward the light from p, its distance, radiance and
//                solid-angle density (area kinds) or delta flag
//   pdf(...)     the solid-angle density of the light point light_p (normal light_n) seen
//                along wi from p (area kinds; the emitter-hit side of MIS)
//   area_point   a uniform point on the light, its normal and area density (area kinds;
//                the equiangular extension's target)
#pragma once
#include "scene.cuh"
#include "sample.cuh"
#include "occupant.cuh"

namespace ptx {

struct LightKind {
    static constexpr bool kDelta = false;
    __device__ static float pdf(const ptr_light&, f3, f3, f3, f3) { return 0.0f; }
};

// Family predicates of light dispatches: the build holds the kind, and it has an area.
template <class K> struct LightPresent { static constexpr bool value = has_light(K::kId); };
template <class K> struct LightArea { static constexpr bool value = has_light(K::kId) && !K::kDelta; };

}  // namespace ptx
