// rails.cuh — gathers from the reference's packed scene-data channels (rail v2:
// src/components/data/pack.ts writers, src/components/data/ledger.ts bases) into this
// library's device layouts.  The channels arrive as flat float4 texel arrays; ids are exact
// floats (< 2^24), checked on the host before any of these run.  The binary BVH nodes and
// placement records are used in place; only triangles, mesh-light tables and params-tier
// placements are gathered.
#pragma once
#include "common.cuh"

namespace ptx {
namespace rails {

// Positions (3 floats per vertex) from the vertices channel's vec3 texels.
__global__ void k_positions(const float4* v, long long base, int n, float* pos) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 t = v[base + i];
        pos[3 * (size_t)i] = t.x;
        pos[3 * (size_t)i + 1] = t.y;
        pos[3 * (size_t)i + 2] = t.z;
    }
}

// The caller-order index triples of a mesh from its leaf-order index texels (order: the
// caller index of each leaf triangle, or NULL for leaf order).
__global__ void k_caller_indices(const float4* idx, long long tbase, int n, const uint32_t* order, unsigned* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 t = idx[tbase + i];
        const size_t c = order ? order[i] : (uint32_t)i;
        out[3 * c] = (unsigned)t.x;
        out[3 * c + 1] = (unsigned)t.y;
        out[3 * c + 2] = (unsigned)t.z;
    }
}

// Leaf-order triangle records for the binary walk: (v0 | caller index, e1 | alpha, e2), the
// edges rounded in float32 as the host builder's records are.
__global__ void k_leaf_tris(const float* pos, const float4* idx, long long tbase, int n, const uint32_t* order,
                            const float* alpha, float4* tri) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 t = idx[tbase + i];
        const unsigned ia = (unsigned)t.x, ib = (unsigned)t.y, ic = (unsigned)t.z;
        const int c = order ? (int)order[i] : i;
        const float* a = pos + 3 * (size_t)ia;
        const float* b = pos + 3 * (size_t)ib;
        const float* cc = pos + 3 * (size_t)ic;
        tri[3 * (size_t)i] = make_float4(a[0], a[1], a[2], __int_as_float(c));
        tri[3 * (size_t)i + 1] = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], alpha ? alpha[c] : -1.0f);
        tri[3 * (size_t)i + 2] = make_float4(cc[0] - a[0], cc[1] - a[1], cc[2] - a[2], 0.0f);
    }
}

// A mesh light's triangles (world a, b, c, leaf order) from its world-position bake.
__global__ void k_light_tris(const float4* v, long long wbase, const float4* idx, long long tbase, int n, float4* lt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 t = idx[tbase + i];
        const unsigned k[3] = {(unsigned)t.x, (unsigned)t.y, (unsigned)t.z};
        for (int j = 0; j < 3; ++j) {
            const float4 p = v[wbase + k[j]];
            lt[3 * (size_t)i + j] = make_float4(p.x, p.y, p.z, 0.0f);
        }
    }
}

// One scalar per texel (.x): the mesh-light CDF.
__global__ void k_scalars(const float4* rec, long long base, int n, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = rec[base + i].x;
}

// Params-tier placements (one texel each) at this library's two texels per instance.
__global__ void k_restride(const float4* rec, long long base, int n, float4* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[2 * (size_t)i] = rec[base + i];
        out[2 * (size_t)i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

}  // namespace rails
}  // namespace ptx
