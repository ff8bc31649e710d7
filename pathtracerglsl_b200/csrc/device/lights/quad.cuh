// quad.cuh — the quad area light (lights/quad/quad.glsl:14-41): a uniform point on the
// parallelogram, area density converted to solid angle; one-sided along its normal.
// p: corner(3) edge1(3) edge2(3) normal(3) area(1).
#pragma once
#include "lights/light.cuh"

namespace ptx {

struct QuadLight : LightKind {
    static constexpr int kId = PTR_LIGHT_QUAD;
    template <class Col>
    __device__ static LightSample<Col> sample(const DevScene&, const ptr_light& l, Col le, f3 p, float x0, float x1) {
        LightSample<Col> ls;
        ls.radiance = le;
        ls.flags = 0u;
        ls.light_id = -1;
        f3 q = ld3(l.p) + x0 * ld3(l.p + 3) + x1 * ld3(l.p + 6);
        f3 dd = q - p;
        float d2 = dot(dd, dd);
        ls.wi = dd * (1.0f / sqrtf(d2));
        ls.distance = sqrtf(d2);
        float cos_l = dot(ld3(l.p + 9), -ls.wi);
        if (cos_l <= 0.0f) { ls.pdf = 0.0f; return ls; }
        ls.pdf = d2 / (l.p[12] * cos_l);
        return ls;
    }
    __device__ static float pdf(const ptr_light& l, f3 p, f3 light_p, f3, f3 wi) {
        float cos_l = dot(ld3(l.p + 9), -wi);
        if (cos_l <= 0.0f) return 0.0f;
        f3 dd = light_p - p;
        return dot(dd, dd) / (l.p[12] * cos_l);
    }
    __device__ static void area_point(const DevScene&, const ptr_light& l, float y0, float y1, f3& pos, f3& nl, float& pdf_area) {
        pos = ld3(l.p) + y0 * ld3(l.p + 3) + y1 * ld3(l.p + 6);
        nl = ld3(l.p + 9);
        pdf_area = 1.0f / l.p[12];
    }
};

}  // namespace ptx
