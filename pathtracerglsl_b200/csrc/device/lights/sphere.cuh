// sphere.cuh — the sphere area light (lights/sphere/sphere.glsl:21-71): directions uniform
// in the visible cone, distance to the near intersection.  p: center(3) radius(1).
#pragma once
#include "lights/light.cuh"

namespace ptx {

// 1 - cos(theta_max) of the cone a sphere of radius r subtends at squared distance dc2
__device__ __forceinline__ float sphere_omc_max(float r, float dc2) {
    float sin2_max = r * r / dc2;
    return sin2_max / (1.0f + sqrtf(gmax(0.0f, 1.0f - sin2_max)));
}

struct SphereLight : LightKind {
    static constexpr int kId = PTR_LIGHT_SPHERE;
    template <class Col>
    __device__ static LightSample<Col> sample(const DevScene&, const ptr_light& l, Col le, f3 p, float x0, float x1) {
        LightSample<Col> ls;
        ls.radiance = le;
        ls.flags = 0u;
        ls.light_id = -1;
        f3 to_c = ld3(l.p) - p;
        float r = l.p[3];
        float dc2 = dot(to_c, to_c);
        if (dc2 <= r * r) { ls.wi = f3(0.f, 1.f, 0.f); ls.distance = 1.0f; ls.pdf = 0.0f; return ls; }
        float omc = sphere_omc_max(r, dc2);
        float w_t = x0 * omc;
        float cos_t = 1.0f - w_t;
        float sin_t = sqrtf(gmax(0.0f, w_t * (2.0f - w_t)));
        float phi = kTwoPi * x1;
        f3 w = to_c * (1.0f / sqrtf(dc2));
        f3 t, b;
        build_basis(w, t, b);
        ls.wi = normalize(t * (sin_t * m_cos(phi)) + b * (sin_t * m_sin(phi)) + w * cos_t);
        ls.pdf = 1.0f / (kTwoPi * omc);
        float proj = dot(to_c, ls.wi);
        f3 perp = to_c - proj * ls.wi;
        float disc = gmax(0.0f, r * r - dot(perp, perp));
        ls.distance = (dc2 - r * r) / (proj + sqrtf(disc));
        return ls;
    }
    __device__ static float pdf(const ptr_light& l, f3 p, f3, f3, f3) {
        f3 to_c = ld3(l.p) - p;
        float dc2 = dot(to_c, to_c);
        float r = l.p[3];
        if (dc2 <= r * r) return 0.0f;
        return 1.0f / (kTwoPi * sphere_omc_max(r, dc2));
    }
    __device__ static void area_point(const DevScene&, const ptr_light& l, float y0, float y1, f3& pos, f3& nl, float& pdf_area) {
        float z = 1.0f - 2.0f * y0;
        float rr = sqrtf(gmax(0.0f, 1.0f - z * z));
        float phi = kTwoPi * y1;
        nl = f3(rr * m_cos(phi), z, rr * m_sin(phi));
        pos = ld3(l.p) + nl * l.p[3];
        pdf_area = 1.0f / (4.0f * kPi * l.p[3] * l.p[3]);
    }
};

}  // namespace ptx
