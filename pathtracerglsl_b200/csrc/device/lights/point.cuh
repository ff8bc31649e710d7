// point.cuh — the point light (lights/point/point.glsl): a delta light of intensity
// `radiance` (W/sr) with inverse-square falloff.  p: position(3).
#pragma once
#include "lights/light.cuh"

namespace ptx {

struct PointLight : LightKind {
    static constexpr int kId = PTR_LIGHT_POINT;
    static constexpr bool kDelta = true;
    template <class Col>
    __device__ static LightSample<Col> sample(const DevScene&, const ptr_light& l, Col le, f3 p, float, float) {
        LightSample<Col> ls;
        ls.light_id = -1;
        f3 dd = ld3(l.p) - p;
        float d2 = dot(dd, dd);
        ls.wi = dd * (1.0f / sqrtf(d2));
        ls.distance = sqrtf(d2);
        ls.radiance = le / d2;
        ls.pdf = 1.0f;
        ls.flags = kLightDelta;
        return ls;
    }
};

}  // namespace ptx
