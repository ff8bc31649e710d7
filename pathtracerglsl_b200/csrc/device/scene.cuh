// scene.cuh — the device-resident scene and its geometry queries.
//
// Analytic regions (plane, sphere, quad, box) are closed-form arms evaluated in region
// order, exactly the reference's unrolled primitive dispatch
// (src/compiler/generate/features/intersection.ts:801-824); meshes and instanced batches
// are walked through their acceleration structures (bvh.cuh).  Region classification
// (scene_region_at, intersection.ts:1121-1225) is the innermost-wins point query.
#pragma once
#include "common.cuh"

namespace ptx {

// Mesh BLAS on the device: triangles (3 float4 each: v0 | e1, alpha | e2, in leaf order),
// binary BVH nodes (2 float4: (min.xyz, A) (max.xyz, B), bvh.ts:344-383 layout) and the
// compressed wide BVH (5 uint4 = 80 B per node, cwbvh.ts:18-31 layout) with its own
// triangle order.
struct DevMesh {
    const float4* tri;        // binary-BVH leaf order
    const float4* tri_w;      // wide-BVH leaf order
    const float4* bvh;
    const uint4* cwbvh;
    int n_tris, n_nodes, n_cw_nodes, pad;
    // mesh lights only (NULL otherwise), in the caller's triangle order: the normalised
    // cumulative world-area CDF (T floats) and the vertices a, b, c (3 float4 per triangle)
    const float* light_cdf;
    const float4* light_tri;
};

// Instanced batch: placements in TLAS leaf order, 2 float4 each — mesh prototypes
// (q, ts) with ts = (t_rigid.xyz, s); sphere prototypes (world centre, world radius)
// folded into the first float4 (the params tier).
struct DevBatch {
    const float4* place;
    const float4* tlas;       // binary BVH over the instances' world boxes
    int n_inst, proto_shape, proto_mesh, n_tlas;
    const uint4* tlas_w;      // compressed wide BVH over the same boxes (NULL: binary only)
    const float4* place_w;    // the placements in the wide BVH's leaf order
    // light-tree selection with this batch's instances as lights: the light id of each
    // placement in the binary / wide TLAS leaf order (NULL: the instances are no lights)
    const int* light_of;
    const int* light_of_w;
    // the caller's index of each placement in the binary / wide TLAS leaf order (the tie
    // rule between instances, and the element a hit query reports)
    const int* inst_id;
    const int* inst_id_w;
};

struct DevScene {
    const ptr_region* regions;
    const ptr_material* materials;
    const ptr_light* lights;
    const int* light_of_region;
    const DevMesh* meshes;
    const DevBatch* batches;
    unsigned* err_flags;      // device guard flags (stack overflow, iteration guard)
    unsigned long long* work; // instrumented pass only: [0] BLAS nodes, [1] triangles,
                              // [2] TLAS nodes, [3] instances entered (NULL = not counted)
    // Region BVH over the bounded analytic regions (sphere, box, quad): the scene table
    // walk of the reference's 'table' object dispatch.  NULL = scan every region in order.
    const float4* region_bvh;     // 2 float4 per node, leaf items index region_items
    const int* region_items;      // leaf order -> region index
    const int* linear_regions;    // regions outside the BVH (planes, meshes, batches), in order
    // Without a region BVH: the region list as runs of one shape, (shape, first, count, 0)
    // in region order, so the scan dispatches once per run (NULL: per region)
    const int4* region_runs;
    int n_linear, n_region_nodes, n_runs, pad_r1;
    int n_regions, n_materials, n_lights, ambient_material;
    int has_media, accel, n_meshes, n_batches;
    int inst_accel;           // PTR_ACCEL_* of the instanced batches' TLAS
    int flat_region = -1;     // the one acceleration region when every other region is analytic
                              // and there is no region BVH (refilling closest-hit loop), else -1
    int has_het;              // some medium has a coefficient field (heterogeneous media)
    int pad_i2;
    float sort_c[4];          // centre of the bounded geometry (ray-coherence keys)
    // environment
    int env_kind, env_samplable, env_select_live, env_w;
    int env_h, pad0, pad1, pad2;
    float env_color[4];
    float env_intensity, env_select_prob, env_rotation, pad3;
    const float4* env_map;    // W*H RGBA, row 0 = v = 0 (+Y pole)
    const float* env_marg;    // H cumulative (marginal over rows)
    const float* env_cond;    // H*W cumulative (conditional within each row)
    // spectral colour model (NULL / unused for RGB scenes): the lifted colours of every
    // material and light, the constant environment, and the sensor tables
    const ptr_spectral_material* spec_mats;
    const ptr_spectrum* spec_lights;
    const float4* spec_curves;   // 95 x (xbar, ybar, zbar, D65) at 5 nm from 360 nm
    ptr_spectrum spec_env;
    float spec_m[9];             // XYZ -> linear sRGB, row-major
    float spec_y;                // int ybar d lambda
    // light tree (light-tree selection; NULL otherwise): 2 float4 per node (min.xyz, phi |
    // max.xyz, link), and the two trail words of every light
    const float4* light_tree;
    const uint2* light_trails;
    // heterogeneous media: the coefficient fields' stack programs (NULL: none)
    const uint32_t* field_code;
};

// ---- closed-form arms (components/geometry/*/*.glsl) ------------------------------------
// Sphere: the robust Haines–Günther–Akenine-Möller roots, inside-test root selection
// (sphere.glsl:28-46).
__device__ __forceinline__ bool sphere_intersect(const Ray& r, f3 c, float rad, float& t) {
    f3 oc = r.o - c;
    float b = dot(oc, r.d);
    f3 perp = oc - b * r.d;
    float disc = rad * rad - dot(perp, perp);
    if (disc < 0.0f) return false;
    float cc = dot(oc, oc) - rad * rad;
    float q = (b >= 0.0f) ? -b - sqrtf(disc) : -b + sqrtf(disc);
    if (q == 0.0f) return false;
    float ta = q, tb = cc / q;
    t = (cc < 0.0f) ? gmax(ta, tb) : gmin(ta, tb);
    return t > 0.0f;
}
__device__ __forceinline__ bool plane_intersect(const Ray& r, f3 n, float off, float& t) {
    float denom = dot(r.d, n);
    if (fabsf(denom) < 1e-8f) return false;
    t = -(dot(r.o, n) + off) / denom;
    return t > 0.0f;
}
// Quad: plane root + inside test through the 2x2 Gram system (quad.glsl:9-22).
__device__ __forceinline__ bool quad_intersect(const Ray& r, f3 corner, f3 e1, f3 e2, f3 n, float& t) {
    float denom = dot(r.d, n);
    if (fabsf(denom) < 1e-8f) return false;
    t = dot(corner - r.o, n) / denom;
    if (t <= 0.0f) return false;
    f3 local = r.o + r.d * t - corner;
    float e11 = dot(e1, e1), e22 = dot(e2, e2), e12 = dot(e1, e2);
    float d1 = dot(local, e1), d2 = dot(local, e2);
    float det = e11 * e22 - e12 * e12;
    float u = (d1 * e22 - d2 * e12) / det;
    float v = (d2 * e11 - d1 * e12) / det;
    return u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f;
}
// Box: slab method with inside-test root selection (box.glsl).
__device__ __forceinline__ bool box_intersect(const Ray& r, f3 c, f3 h, float& t) {
    f3 inv = f3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    f3 t0 = (c - h - r.o) * inv;
    f3 t1 = (c + h - r.o) * inv;
    f3 tsm = vmin(t0, t1), tbg = vmax(t0, t1);
    float tn = gmax(gmax(tsm.x, tsm.y), tsm.z);
    float tf = gmin(gmin(tbg.x, tbg.y), tbg.z);
    if (tf < tn) return false;
    t = (tn < 0.0f) ? tf : tn;
    return t > 0.0f;
}
__device__ __forceinline__ float box_sdf(f3 p, f3 c, f3 h) {
    f3 d = f3(fabsf(p.x - c.x), fabsf(p.y - c.y), fabsf(p.z - c.z)) - h;
    return length(vmax(d, f3(0.0f))) + gmin(gmax(d.x, gmax(d.y, d.z)), 0.0f);
}
__device__ __forceinline__ f3 box_normal(f3 p, f3 c, f3 h) {
    f3 q = (p - c) / h;
    f3 a(fabsf(q.x), fabsf(q.y), fabsf(q.z));
    if (a.x >= a.y && a.x >= a.z) return f3(signf(q.x), 0.f, 0.f);
    if (a.y >= a.z) return f3(0.f, signf(q.y), 0.f);
    return f3(0.f, 0.f, signf(q.z));
}

// One analytic arm: root of region g (of the given shape) along r (false when the shape
// is not analytic).
__device__ __forceinline__ bool analytic_root_shape(int shape, const ptr_region& g, const Ray& r, float& t) {
    switch (shape) {
        case PTR_SHAPE_PLANE: return has_shape(PTR_SHAPE_PLANE) && plane_intersect(r, ld3(g.p), g.p[3], t);
        case PTR_SHAPE_SPHERE: return has_shape(PTR_SHAPE_SPHERE) && sphere_intersect(r, ld3(g.p), g.p[3], t);
        case PTR_SHAPE_QUAD:
            return has_shape(PTR_SHAPE_QUAD) && quad_intersect(r, ld3(g.p), ld3(g.p + 3), ld3(g.p + 6), ld3(g.p + 9), t);
        case PTR_SHAPE_BOX: return has_shape(PTR_SHAPE_BOX) && box_intersect(r, ld3(g.p), ld3(g.p + 3), t);
        default: return false;
    }
}
__device__ __forceinline__ bool analytic_root(const ptr_region& g, const Ray& r, float& t) {
    return analytic_root_shape(g.shape, g, r, t);
}
// Signed distance of an analytic solid (thin owners and meshes never claim containment).
__device__ __forceinline__ float analytic_sdf_shape(int shape, const ptr_region& g, f3 p) {
    switch (shape) {
        case PTR_SHAPE_PLANE: return has_shape(PTR_SHAPE_PLANE) ? dot(p, ld3(g.p)) + g.p[3] : 1.0e20f;
        case PTR_SHAPE_SPHERE: return has_shape(PTR_SHAPE_SPHERE) ? length(p - ld3(g.p)) - g.p[3] : 1.0e20f;
        case PTR_SHAPE_BOX: return has_shape(PTR_SHAPE_BOX) ? box_sdf(p, ld3(g.p), ld3(g.p + 3)) : 1.0e20f;
        default: return 1.0e20f;
    }
}
__device__ __forceinline__ float analytic_sdf(const ptr_region& g, f3 p) { return analytic_sdf_shape(g.shape, g, p); }
// Outward normal of an analytic arm at its hit point.
__device__ __forceinline__ f3 analytic_normal(const ptr_region& g, f3 p) {
    switch (g.shape) {
        case PTR_SHAPE_PLANE: return ld3(g.p);
        case PTR_SHAPE_SPHERE: return normalize(p - ld3(g.p));
        case PTR_SHAPE_QUAD: return ld3(g.p + 9);
        default: return box_normal(p, ld3(g.p), ld3(g.p + 3));
    }
}

}  // namespace ptx
