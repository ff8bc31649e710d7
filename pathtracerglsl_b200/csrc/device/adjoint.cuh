// adjoint.cuh — derivative terms of the path-replay adjoint (no counterpart in the reference).
//
// Path replay backpropagation (Vicini, Speierer & Jakob, "Path Replay Backpropagation",
// SIGGRAPH 2021) with detached sampling: a path's contribution is a product of per-vertex
// weights w_j = f_j / p_j whose sampling densities p_j are held fixed, so the derivative of
// everything the path gathers after vertex j is (radiance still to come) * d log f_j / d theta.
// The replay knows the radiance still to come because the forward pass of the same
// counter-based path stored its total.  MIS weights and roulette probabilities are
// detached too (they sum to one / keep the estimator unbiased for every theta, so their
// derivatives vanish in expectation).
//
// Per material, PTR_GRAD_SLOTS parameters (include/ptx_rt.h): the model's colour (rgb:
// Lambert albedo, GGX / mirror F0, dielectric transmittance), GGX alpha, dielectric IOR, grey
// homogeneous medium sigma_t, single-scattering albedo and HG g.
// For the IOR only the interface terms (Fresnel lobe choice, the eta^2 radiance factor) are
// differentiated: the refracted direction's own dependence on the IOR would need an
// attached derivative of every later vertex.
#pragma once
#include "occupants.cuh"

namespace ptx {

// The surface models' own derivative terms live beside them (materials/*.cuh: nee_grad,
// cont_grad); here are the medium's and the accumulators.

// d log p_HG / d g (forward convention, hg.glsl:11-42).
__device__ __forceinline__ float hg_dlog_g(f3 wi, f3 wo, float g) {
    float c = dot(wi, -wo);
    float d = gmax(1.0f + g * g - 2.0f * g * c, 1e-8f);
    return -2.0f * g / (1.0f - g * g) - 1.5f * (2.0f * g - 2.0f * c) / d;
}
// Grey homogeneous medium: sigma_t and the single-scattering albedo a
// (sigma_s = a sigma_t, sigma_a = (1 - a) sigma_t), read from channel 0.
struct GreyMedium { float st, a; };
__device__ __forceinline__ GreyMedium grey_medium(const ptr_material& m) {
    GreyMedium g;
    g.st = m.sigma_a[0] + m.sigma_s[0];
    g.a = g.st > 0.0f ? m.sigma_s[0] / g.st : 0.0f;
    return g;
}

// Per-block gradient accumulators in shared memory (float64), flushed to the global
// float64 gradient buffer at the end of the kernel.
struct GradAcc {
    double* s;     // shared: PTR_GRAD_SLOTS per material
    f3 dl;         // the path's adjoint radiance (dLoss/dI of its pixel / spp)
    // per-channel slots [slot0, slot0+2]: grad_c += dl_c X_c dlog_c
    __device__ __forceinline__ void vec(int mat, int slot0, f3 X, f3 dlog) const {
        double* b = s + PTR_GRAD_SLOTS * mat + slot0;
        float v0 = dl.x * X.x * dlog.x, v1 = dl.y * X.y * dlog.y, v2 = dl.z * X.z * dlog.z;
        if (v0 != 0.0f) atomicAdd(b + 0, (double)v0);
        if (v1 != 0.0f) atomicAdd(b + 1, (double)v1);
        if (v2 != 0.0f) atomicAdd(b + 2, (double)v2);
    }
    // scalar slot: grad += (dl . X) dlog
    __device__ __forceinline__ void scl(int mat, int slot, f3 X, float dlog) const {
        float v = (dl.x * X.x + dl.y * X.y + dl.z * X.z) * dlog;
        if (v != 0.0f) atomicAdd(s + PTR_GRAD_SLOTS * mat + slot, (double)v);
    }
};

__device__ __forceinline__ void grad_block_init(double* s, int n) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) s[k] = 0.0;
    __syncthreads();
}
__device__ __forceinline__ void grad_block_flush(const double* s, int n, double* g) {
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        if (s[k] != 0.0) atomicAdd(g + k, s[k]);
}

// Shadow-record kinds of the per-vertex lobe derivative D = dlog f(wi_light) - dlog w_cont.
// GGX: the per-channel F0 part in xyz, the alpha part in w.
constexpr int kGradKindNone = 0, kGradKindAlbedo = 1, kGradKindGGX = 2, kGradKindPhase = 3;

}  // namespace ptx
