// sample.cuh — the records occupants return: a sampled lobe (direction, weight = f cos / pdf,
// pdf, lobe flags) and a light sample (direction, distance, radiance, solid-angle density,
// flags, the light's id).
#pragma once
#include "common.cuh"

namespace ptx {

template <class Col = f3> struct ISample { f3 wi; Col weight; float pdf; uint32_t flags; };
template <class Col = f3> struct LightSample { f3 wi; float distance; Col radiance; float pdf; uint32_t flags; int light_id; };

}  // namespace ptx
