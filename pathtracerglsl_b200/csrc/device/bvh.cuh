// bvh.cuh — acceleration-structure arms of the scene queries (meshes, instanced batches).
#pragma once
#include "scene.cuh"

namespace ptx {

struct HitRec;

__device__ __forceinline__ void accel_closest(const DevScene&, const ptr_region&, int, const Ray&, HitRec&) {}
__device__ __forceinline__ bool accel_any(const DevScene&, const ptr_region&, const Ray&, float) { return false; }
__device__ __forceinline__ float accel_region_sdf(const DevScene&, const ptr_region&, f3) { return 1.0e20f; }
__device__ __forceinline__ f3 accel_hit_normal(const DevScene&, const ptr_region&, const HitRec&, const Ray&, Hit& h) {
    h.eps = kMarchClearance;
    return f3(0.f, 1.f, 0.f);
}

}  // namespace ptx
