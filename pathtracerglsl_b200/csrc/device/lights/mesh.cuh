// mesh.cuh — the mesh area light (lights/mesh/mesh.glsl:18-75): an emissive mesh object,
// a triangle picked by the world-area CDF and a uniform point on it; no distance falloff
// beyond the solid-angle conversion, one-sided along the winding normal.  Uniform area over
// the whole mesh makes the density d^2 / (A cos_l) whichever triangle was hit.
// p: mesh index(1, as float) .. world area(p[12]).
#pragma once
#include "lights/light.cuh"

namespace ptx {

// The smallest triangle whose cumulative area exceeds x0 (a zero-area triangle is never
// picked), x0 rescaled within its span, a uniform point by the square-root map; n is the
// unit winding normal cross(b-a, c-a), NaN for a triangle degenerate in float32.
__device__ __noinline__ f3 mesh_light_point(const DevScene& S, const ptr_light& l, float x0, float x1, f3& n) {
    const DevMesh& m = S.meshes[(int)l.p[0]];
    const float* cdf = m.light_cdf;
    int lo = 0, hi = m.n_tris - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= x0) lo = mid + 1;
        else hi = mid;
    }
    float c0 = lo > 0 ? __ldg(cdf + lo - 1) : 0.0f;
    float c1 = __ldg(cdf + lo);
    float xr = clampf((x0 - c0) / gmax(c1 - c0, 1.0e-12f), 0.0f, 0.9999999f);
    f3 a = xyz(__ldg(m.light_tri + 3 * lo)), b = xyz(__ldg(m.light_tri + 3 * lo + 1)), c = xyz(__ldg(m.light_tri + 3 * lo + 2));
    float su = sqrtf(xr);
    n = normalize(cross(b - a, c - a));
    return a * (1.0f - su) + b * (su * (1.0f - x1)) + c * (su * x1);
}

struct MeshLight : LightKind {
    static constexpr int kId = PTR_LIGHT_MESH;
    template <class Col>
    __device__ static LightSample<Col> sample(const DevScene& S, const ptr_light& l, Col le, f3 p, float x0, float x1) {
        LightSample<Col> ls;
        ls.radiance = le;
        ls.flags = 0u;
        ls.light_id = -1;
        f3 n;
        f3 q = mesh_light_point(S, l, x0, x1, n);
        f3 dd = q - p;
        float d2 = dot(dd, dd);
        ls.wi = dd * (1.0f / sqrtf(d2));
        ls.distance = sqrtf(d2);
        float cos_l = dot(n, -ls.wi);
        if (!(cos_l > 0.0f)) { ls.pdf = 0.0f; return ls; }
        ls.pdf = d2 / (l.p[12] * cos_l);
        return ls;
    }
    // light_n: the hit's geometric normal
    __device__ static float pdf(const ptr_light& l, f3 p, f3 light_p, f3 light_n, f3 wi) {
        float cos_l = dot(light_n, -wi);
        if (cos_l <= 0.0f) return 0.0f;
        f3 dd = light_p - p;
        return dot(dd, dd) / (l.p[12] * cos_l);
    }
    __device__ static void area_point(const DevScene& S, const ptr_light& l, float y0, float y1, f3& pos, f3& nl, float& pdf_area) {
        pos = mesh_light_point(S, l, y0, y1, nl);
        pdf_area = 1.0f / l.p[12];
    }
};

}  // namespace ptx
