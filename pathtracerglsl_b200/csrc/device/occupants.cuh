// occupants.cuh — lights, environment and media of the transport loop, and the colour
// models every occupant reads through.
//
// One function family per occupant, selected by the light record's kind (the device
// counterpart of the reference's generated dispatch over its registries,
// src/compiler/generate/features/lighting.ts:546-693).  Surface material models live in
// materials/, one header each, listed in materials/registry.cuh.
#pragma once
#include "scene.cuh"
#include "sample.cuh"
#include "lights/registry.cuh"

namespace ptx {

// ---- colour models ---------------------------------------------------------------------
// RGB reads the material/light records' rgb directly; the spectral model evaluates the
// host-lifted ptr_spectrum of each colour at the path's four wavelengths
// (color/spectral/lookup.glsl:38-59, spectra/blackbody/blackbody.glsl:4-10).
struct Wl { float4 lambda; };

__device__ __forceinline__ float4 spectral_curves(const DevScene& S, float lambda) {
    float x = (lambda - 360.0f) / 5.0f;
    int i = (int)x;
    i = i < 93 ? i : 93;
    float4 a = __ldg(S.spec_curves + i), b = __ldg(S.spec_curves + i + 1);
    float f = x - (float)i;
    return make_float4(a.x * (1.0f - f) + b.x * f, a.y * (1.0f - f) + b.y * f, a.z * (1.0f - f) + b.z * f,
                       a.w * (1.0f - f) + b.w * f);
}
__device__ __forceinline__ float spec_lane(const DevScene& S, const ptr_spectrum& sp, float lambda) {
    float v;
    if (sp.kind == PTR_SPEC_LIFTED) {
        float t = (lambda - 360.0f) / 470.0f;
        float p = (sp.c[0] * t + sp.c[1]) * t + sp.c[2];
        v = clampf(0.5f + 0.5f * p / sqrtf(1.0f + p * p), 0.0f, 1.0f);
        v = sp.scale * v;
    } else if (sp.kind == PTR_SPEC_BLACKBODY) {
        float q = 14387768.775039338f / sp.c[0];
        float ratio = 550.0f / lambda;
        float ratio2 = ratio * ratio;
        v = sp.c[1] * (m_exp(q / 550.0f) - 1.0f) * ratio2 * ratio2 * ratio / (m_exp(q / lambda) - 1.0f);
        v = sp.scale * v;
    } else {
        v = sp.scale;
    }
    if (sp.d65) v = v * spectral_curves(S, lambda).w;
    return v;
}
__device__ __forceinline__ s4 spec_eval(const DevScene& S, const ptr_spectrum& sp, const Wl& wl) {
    return s4(spec_lane(S, sp, wl.lambda.x), spec_lane(S, sp, wl.lambda.y), spec_lane(S, sp, wl.lambda.z),
              spec_lane(S, sp, wl.lambda.w));
}

template <class Col> struct Colors;
template <> struct Colors<f3> {
    __device__ static f3 albedo(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].albedo); }
    __device__ static f3 emission(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].emission); }
    __device__ static f3 tint(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].transmittance); }
    __device__ static f3 f0(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].f0); }
    __device__ static f3 sigma_a(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].sigma_a); }
    __device__ static f3 sigma_s(const DevScene& S, int mi, const Wl&) { return ld3(S.materials[mi].sigma_s); }
    __device__ static f3 light(const DevScene& S, int li, const Wl&) { return ld3(S.lights[li].radiance); }
    __device__ static f3 env_color(const DevScene& S, const Wl&) { return ld3(S.env_color); }
};
template <> struct Colors<s4> {
    __device__ static s4 albedo(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].albedo, w); }
    __device__ static s4 emission(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].emission, w); }
    __device__ static s4 tint(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].transmittance, w); }
    __device__ static s4 f0(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].f0, w); }
    __device__ static s4 sigma_a(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].sigma_a, w); }
    __device__ static s4 sigma_s(const DevScene& S, int mi, const Wl& w) { return spec_eval(S, S.spec_mats[mi].sigma_s, w); }
    __device__ static s4 light(const DevScene& S, int li, const Wl& w) { return spec_eval(S, S.spec_lights[li], w); }
    __device__ static s4 env_color(const DevScene& S, const Wl& w) { return spec_eval(S, S.spec_env, w); }
};

// ---- surface material models: one header each under materials/ (registry.cuh) ---------

// ---- HG phase, forward convention (volume_scattering/hg/hg.glsl:11-42) -----------------
__device__ __forceinline__ float hg_eval(f3 wi, f3 wo, float g) {
    float c = dot(wi, -wo);
    float d = 1.0f + g * g - 2.0f * g * c;
    return (1.0f - g * g) / (4.0f * kPi * d * sqrtf(gmax(d, 1e-8f)));
}
template <class Col>
__device__ __forceinline__ ISample<Col> hg_sample(f3 wo, float g, float x0, float x1) {
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = 1.0f - 2.0f * x0;
    } else {
        float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * x0);
        cos_theta = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sin_theta = sqrtf(gmax(0.0f, 1.0f - cos_theta * cos_theta));
    float phi = kTwoPi * x1;
    f3 t, b;
    build_basis(-wo, t, b);
    ISample<Col> s;
    s.wi = normalize(t * (sin_theta * m_cos(phi)) + b * (sin_theta * m_sin(phi)) + (-wo) * cos_theta);
    s.weight = Col(1.0f);
    float e = hg_eval(s.wi, wo, g);
    s.pdf = spectrum_average(Col(e));
    s.flags = kLobeMedium;
    return s;
}

// ---- environment (features/environment.ts) ----------------------------------------------
// constant: closed-form radiance, uniform-sphere NEE (T3).  image: an equirect RGB table
// read through equirect_uv (env/equirect/equirect_map.glsl:15-21) with bilinear
// filtering (wrap in u, clamp in v), importance-sampled by the 2-level CDF of
// env/sampler_cdf.glsl:13-84 mixed with 1/16 uniform-sphere probability.
__device__ __forceinline__ float2 equirect_uv(const DevScene& S, f3 dir) {
    f3 n = normalize(dir);
    float phi = (n.x == 0.0f && n.z == 0.0f ? 0.0f : m_atan2(n.z, n.x)) + S.env_rotation;
    float theta = m_atan2(sqrtf(n.x * n.x + n.z * n.z), n.y);
    float u = phi * (1.0f / kTwoPi) + 0.5f;
    u = u - floorf(u);
    return make_float2(u, theta * (1.0f / kPi));
}
__device__ __forceinline__ f3 env_map_bilinear(const DevScene& S, float2 uv) {
    const int W = S.env_w, H = S.env_h;
    float x = uv.x * (float)W - 0.5f, y = uv.y * (float)H - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    float ax = x - fx0, ay = y - fy0;
    int i0 = (int)fx0, j0 = (int)fy0;
    int i1 = i0 + 1, j1 = j0 + 1;
    i0 = ((i0 % W) + W) % W;
    i1 = ((i1 % W) + W) % W;
    j0 = j0 < 0 ? 0 : (j0 >= H ? H - 1 : j0);
    j1 = j1 < 0 ? 0 : (j1 >= H ? H - 1 : j1);
    float4 c00 = __ldg(S.env_map + (size_t)j0 * W + i0), c10 = __ldg(S.env_map + (size_t)j0 * W + i1);
    float4 c01 = __ldg(S.env_map + (size_t)j1 * W + i0), c11 = __ldg(S.env_map + (size_t)j1 * W + i1);
    f3 top = xyz(c00) * (1.0f - ax) + xyz(c10) * ax;
    f3 bot = xyz(c01) * (1.0f - ax) + xyz(c11) * ax;
    return top * (1.0f - ay) + bot * ay;
}
// The spectral model supports the constant environment only (image environments are
// rejected on the host).
template <class Col>
__device__ __forceinline__ Col env_radiance(const DevScene& S, f3 dir, const Wl& wl) {
    if (has_env(PTR_ENV_CONSTANT) && S.env_kind == PTR_ENV_CONSTANT) return Colors<Col>::env_color(S, wl) * S.env_intensity;
    if constexpr (sizeof(Col) == sizeof(f3)) {
        if (has_env(PTR_ENV_IMAGE) && S.env_kind == PTR_ENV_IMAGE)
            return env_map_bilinear(S, equirect_uv(S, dir)) * S.env_intensity;
    }
    return Col(0.0f);
}
__device__ __forceinline__ float env_marg(const DevScene& S, int j) { return __ldg(S.env_marg + j); }
__device__ __forceinline__ float env_cond(const DevScene& S, int j, int i) { return __ldg(S.env_cond + (size_t)j * S.env_w + i); }
__device__ __forceinline__ float env_texel_domega(int j, int W, int H) {
    float theta = kPi * ((float)j + 0.5f) / (float)H;
    return (kTwoPi / (float)W) * 2.0f * m_sin(theta) * m_sin(0.5f * kPi / (float)H);
}
__device__ __forceinline__ float env_uniform_fraction(const DevScene& S) {
    return env_marg(S, S.env_h - 1) > 0.0f ? 0.0625f : 1.0f;
}
__device__ __forceinline__ float env_table_pdf(const DevScene& S, f3 dir) {
    const int W = S.env_w, H = S.env_h;
    float2 uv = equirect_uv(S, dir);
    int i = (int)(uv.x * (float)W);
    int j = (int)(uv.y * (float)H);
    i = i < 0 ? 0 : (i > W - 1 ? W - 1 : i);
    j = j < 0 ? 0 : (j > H - 1 ? H - 1 : j);
    float d_marg = env_marg(S, j) - (j > 0 ? env_marg(S, j - 1) : 0.0f);
    float d_cond = env_cond(S, j, i) - (i > 0 ? env_cond(S, j, i - 1) : 0.0f);
    return (d_cond * d_marg) / env_texel_domega(j, W, H);
}
__device__ __forceinline__ f3 env_chart_sample(const DevScene& S, int ci, int cj, float ux, float uy) {
    const int W = S.env_w, H = S.env_h;
    float phi = (((float)ci + ux) / (float)W - 0.5f) * kTwoPi - S.env_rotation;
    bool north = 2 * cj < H;
    float row = north ? (float)cj : (float)(H - cj - 1);
    float a = m_sin(0.5f * kPi * row / (float)H);
    float b = m_sin(0.5f * kPi * (row + 1.0f) / (float)H);
    float t = north ? uy : 1.0f - uy;
    float h = (a * a) * (1.0f - t) + (b * b) * t;
    float y = (north ? 1.0f : -1.0f) * (1.0f - 2.0f * h);
    float r = 2.0f * sqrtf(h * (1.0f - h));
    return f3(r * m_cos(phi), y, r * m_sin(phi));
}
__device__ __forceinline__ f3 env_sample_table(const DevScene& S, float x0, float x1) {
    const int W = S.env_w, H = S.env_h;
    const float kFracMax = 0.9999999f;
    int lo = 0, hi = H - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (x0 >= env_marg(S, mid)) lo = mid + 1; else hi = mid;
    }
    int j = lo;
    float m_lo = j > 0 ? env_marg(S, j - 1) : 0.0f;
    float d_marg = env_marg(S, j) - m_lo;
    float v_frac = d_marg > 0.0f ? clampf((x0 - m_lo) / d_marg, 0.0f, kFracMax) : 0.5f;
    lo = 0;
    hi = W - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (x1 >= env_cond(S, j, mid)) lo = mid + 1; else hi = mid;
    }
    int i = lo;
    float c_lo = i > 0 ? env_cond(S, j, i - 1) : 0.0f;
    float d_cond = env_cond(S, j, i) - c_lo;
    float u_frac = d_cond > 0.0f ? clampf((x1 - c_lo) / d_cond, 0.0f, kFracMax) : 0.5f;
    return env_chart_sample(S, i, j, u_frac, v_frac);
}
__device__ __forceinline__ float env_pdf(const DevScene& S, f3 dir) {
    if (!has_env(PTR_ENV_IMAGE) || S.env_kind != PTR_ENV_IMAGE) return 1.0f / (4.0f * kPi);
    float a = env_uniform_fraction(S);
    return (1.0f - a) * env_table_pdf(S, dir) + a / (4.0f * kPi);
}
template <class Col>
__device__ __forceinline__ LightSample<Col> env_sample(const DevScene& S, float x0, float x1, const Wl& wl) {
    LightSample<Col> ls;
    if (has_env(PTR_ENV_IMAGE) && S.env_kind == PTR_ENV_IMAGE) {
        float a = env_uniform_fraction(S);
        if (x0 < a) {
            float y = 1.0f - 2.0f * (x0 / a);
            float r = sqrtf(gmax(0.0f, 1.0f - y * y));
            float phi = kTwoPi * x1;
            ls.wi = f3(r * m_cos(phi), y, r * m_sin(phi));
        } else {
            ls.wi = env_sample_table(S, (x0 - a) / (1.0f - a), x1);
        }
        ls.distance = kMaxDist;
        ls.radiance = env_radiance<Col>(S, ls.wi, wl);
        ls.pdf = env_pdf(S, ls.wi);
        ls.flags = 0u;
        ls.light_id = -1;
        return ls;
    }
    float z = 1.0f - 2.0f * x0;
    float r = sqrtf(gmax(0.0f, 1.0f - z * z));
    float phi = kTwoPi * x1;
    ls.wi = f3(r * m_cos(phi), z, r * m_sin(phi));
    ls.distance = kMaxDist;
    ls.radiance = Colors<Col>::env_color(S, wl) * S.env_intensity;
    ls.pdf = 1.0f / (4.0f * kPi);
    ls.flags = 0u;
    ls.light_id = -1;
    return ls;
}

// ---- lights: one header per kind under lights/ (registry.cuh) ----------------------------
// One light of the roster: a direction toward it, its distance, radiance and density.
template <class Col>
__device__ LightSample<Col> light_sample_one(const DevScene& S, const ptr_light& l, Col le, f3 p, float x0, float x1) {
    LightSample<Col> ls;   // a kind the build lacks samples nothing
    ls.wi = f3(0.f, 1.f, 0.f);
    ls.distance = 1.0f;
    ls.radiance = le;
    ls.pdf = 0.0f;
    ls.flags = 0u;
    ls.light_id = -1;
    auto one = [&](auto K) { ls = decltype(K)::template sample<Col>(S, l, le, p, x0, x1); };
    dispatch_light<LightPresent>(l.kind, one);
    return ls;
}
// The solid-angle density of an area light's point light_p (normal light_n: the hit's
// geometric normal) along wi from p; 0 for a delta light.
__device__ __forceinline__ float light_pdf_one(const ptr_light& l, f3 p, f3 light_p, f3 light_n, f3 wi) {
    float pdf = 0.0f;
    auto one = [&](auto K) { pdf = decltype(K)::pdf(l, p, light_p, light_n, wi); };
    dispatch_light<LightArea>(l.kind, one);
    return pdf;
}
// ---- light-tree selection (accel/light_tree/light_tree.glsl:28-77; the walk pair of
// features/lighting.ts:767-824) ----------------------------------------------------------
// The selection context: the receiving point, its shading normal (zero at a medium event:
// no orientation) and whether the receiver's BSDF covers the whole sphere (rough
// dielectric), which disarms the below-horizon cull (pt.ts:125-139).
struct LightQuery { f3 p, n; bool two_sided; };

// Importance of a subtree for the query: phi over the clamped squared distance to the box
// centre (Conty-Kulla's near-field rule), times a best-case cosine built from the box's
// corner that lies farthest along n (an exact below-horizon cull for one-sided receivers)
// and the centre cosine.
__device__ __forceinline__ float light_tree_importance(f3 bmin, f3 bmax, float phi, const LightQuery& q) {
    f3 c = 0.5f * (bmin + bmax);
    f3 e = bmax - bmin;
    f3 d = c - q.p;
    float d2raw = dot(d, d);
    float diag2 = 0.25f * dot(e, e);
    float base = phi / gmax(d2raw, gmax(diag2, 1e-8f));
    if (dot(q.n, q.n) < 0.5f) return base;
    f3 far_c(q.n.x >= 0.0f ? bmax.x : bmin.x, q.n.y >= 0.0f ? bmax.y : bmin.y, q.n.z >= 0.0f ? bmax.z : bmin.z);
    float h = dot(q.n, far_c - q.p);
    if (q.two_sided) {
        f3 near_c = bmin + bmax - far_c;
        h = gmax(h, -dot(q.n, near_c - q.p));
    } else if (h <= 0.0f) {
        return 0.0f;
    }
    float cos_c = dot(q.n, d) * (1.0f / sqrtf(gmax(d2raw, 1e-12f)));
    if (q.two_sided) cos_c = fabsf(cos_c);
    f3 dmx = vmax(q.p - bmin, bmax - q.p);
    float lo = h * (1.0f / sqrtf(gmax(dot(dmx, dmx), 1e-12f)));
    return base * gmin(1.0f, gmax(cos_c, lo));
}
// One descent step shared by the pick and the pmf walks: both children's importances and
// the left probability (isum <= 0: a dead descent).
struct TreeStep { int L, R; float4 l1, r1; float p_l; bool dead; };
__device__ __forceinline__ TreeStep light_tree_step(const float4* T, int ni, float4 n1, const LightQuery& q) {
    TreeStep s;
    s.L = ni + 1;
    s.R = (int)n1.w;
    float4 l0 = __ldg(T + 2 * s.L), r0 = __ldg(T + 2 * s.R);
    s.l1 = __ldg(T + 2 * s.L + 1);
    s.r1 = __ldg(T + 2 * s.R + 1);
    float iw_l = light_tree_importance(xyz(l0), xyz(s.l1), l0.w, q);
    float iw_r = light_tree_importance(xyz(r0), xyz(s.r1), r0.w, q);
    float isum = iw_l + iw_r;
    s.dead = !(isum > 0.0f);
    s.p_l = s.dead ? 0.0f : iw_l / isum;
    return s;
}
// Stochastic descent: importance-weighted child choice with a fresh number per level below
// the first; returns the light (or -1 on a dead descent, pmf 0) and the product pmf.
__device__ __forceinline__ int light_tree_pick(const DevScene& S, const LightQuery& q, float xi, Rng& rng, float& pmf) {
    const float4* T = S.light_tree;
    pmf = 1.0f;
    int ni = 0;
    float4 n1 = __ldg(T + 1);
    for (int lvl = 0; lvl < 48 && n1.w >= 0.0f; ++lvl) {
        TreeStep st = light_tree_step(T, ni, n1, q);
        if (st.dead) { pmf = 0.0f; return -1; }
        if (xi < st.p_l) { pmf *= st.p_l; ni = st.L; n1 = st.l1; }
        else { pmf *= (1.0f - st.p_l); ni = st.R; n1 = st.r1; }
        xi = rng.next();
    }
    if (n1.w >= 0.0f) { pmf = 0.0f; return -1; }
    return (int)(-n1.w - 1.0f);
}
// The MIS pmf of a light: its stored trail replayed with the stored query, through the
// same step arithmetic as the pick (p_l and 1 - p_l).
__device__ __forceinline__ float light_tree_pmf(const DevScene& S, const LightQuery& q, int light) {
    const float4* T = S.light_tree;
    uint2 tr = __ldg(S.light_trails + light);
    unsigned tw = tr.x;
    float pmf = 1.0f;
    int ni = 0;
    float4 n1 = __ldg(T + 1);
    for (int lvl = 0; lvl < 48 && n1.w >= 0.0f; ++lvl) {
        if (lvl == 24) tw = tr.y;
        TreeStep st = light_tree_step(T, ni, n1, q);
        if (st.dead) return 0.0f;
        if ((tw & 1u) == 0u) { pmf *= st.p_l; ni = st.L; n1 = st.l1; }
        else { pmf *= (1.0f - st.p_l); ni = st.R; n1 = st.r1; }
        tw >>= 1u;
    }
    return pmf;
}
template <class Col>
__device__ LightSample<Col> lighting_sample_tree(const DevScene& S, const LightQuery& q, float x0, float x1, Rng& rng,
                                                 const Wl& wl) {
    LightSample<Col> ls;
    float sel;
    int id = light_tree_pick(S, q, x0, rng, sel);
    if (id < 0) { ls.pdf = 0.0f; return ls; }   // dead descent: a zero-contribution event
    float lx = rng.next();
    ls = light_sample_one(S, S.lights[id], Colors<Col>::light(S, id, wl), q.p, lx, x1);
    ls.light_id = id;
    ls.pdf *= sel;
    return ls;
}

// Finite-light selection by the power CDF with the rescaled coordinate (lighting.ts:546-637).
template <class Col>
__device__ LightSample<Col> lighting_sample_finite(const DevScene& S, f3 p, float x0, float x1, const Wl& wl) {
    if (S.n_lights == 1) {
        LightSample<Col> ls = light_sample_one(S, S.lights[0], Colors<Col>::light(S, 0, wl), p, x0, x1);
        ls.light_id = 0;
        return ls;
    }
    int id = S.n_lights - 1;
    for (int i = 0; i < S.n_lights - 1; ++i)
        if (x0 < S.lights[i].select_cdf) { id = i; break; }
    float lo = id == 0 ? 0.0f : S.lights[id - 1].select_cdf;
    float sel = S.lights[id].select_pdf;
    float xr = (x0 - lo) / sel;
    LightSample<Col> ls = light_sample_one(S, S.lights[id], Colors<Col>::light(S, id, wl), p, clampf(xr, 0.0f, 0.9999999f), x1);
    ls.light_id = id;
    ls.pdf *= sel;
    return ls;
}
// Two-stage env-vs-finite draw (lighting.ts generateLightSampling).
// (tree: the light-tree walk replaces the finite stage, lighting.ts:830-900)
template <class Col>
__device__ LightSample<Col> lighting_sample(const DevScene& S, const LightQuery& q, float x0, float x1, Rng& rng,
                                            bool tree, const Wl& wl) {
    if (S.n_lights == 0) {
        if (S.env_samplable) return env_sample<Col>(S, x0, x1, wl);
        LightSample<Col> ls;
        ls.pdf = 0.0f;
        return ls;
    }
    tree = PTR_SPEC_TREE && tree;
    if (!S.env_select_live)
        return tree ? lighting_sample_tree<Col>(S, q, x0, x1, rng, wl) : lighting_sample_finite<Col>(S, q.p, x0, x1, wl);
    float pe = S.env_select_prob;
    if (x0 < pe) {
        LightSample<Col> ls = env_sample<Col>(S, clampf(x0 / pe, 0.0f, 0.9999999f), x1, wl);
        ls.pdf *= pe;
        return ls;
    }
    float fx = clampf((x0 - pe) / (1.0f - pe), 0.0f, 0.9999999f);
    LightSample<Col> ls = tree ? lighting_sample_tree<Col>(S, q, fx, x1, rng, wl) : lighting_sample_finite<Col>(S, q.p, fx, x1, wl);
    ls.pdf *= (1.0f - pe);
    return ls;
}
// q: the selection context stored when the path left the previous vertex
__device__ __forceinline__ float lighting_pdf(const DevScene& S, const LightQuery& q, f3 wi, int lid, f3 light_p,
                                              f3 light_n, bool tree) {
    const ptr_light& l = S.lights[lid];
    float sel = (PTR_SPEC_TREE && tree) ? light_tree_pmf(S, q, lid) : S.n_lights == 1 ? 1.0f : l.select_pdf;
    float pe = S.env_select_live ? (1.0f - S.env_select_prob) : 1.0f;
    return sel * pe * light_pdf_one(l, q.p, light_p, light_n, wi);
}
// The light id of an emitter hit: the region's light, or an instance light of the batch
// (the TLAS leaf order the hit was found in)
__device__ __forceinline__ int emitter_light(const DevScene& S, const Hit& hit) {
    int lid = S.light_of_region[hit.region_to];
    if (PTR_SPEC_TREE && has_shape(PTR_SHAPE_INSTANCES) && lid < 0 && hit.region_to == hit.region_owner) {
        const ptr_region& g = S.regions[hit.region_owner];
        if (g.shape == PTR_SHAPE_INSTANCES) {
            const DevBatch& b = S.batches[g.ref];
            const int* lo = (S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w) ? b.light_of_w : b.light_of;
            if (lo) lid = __ldg(lo + hit.element);
        }
    }
    return lid;
}

// ---- homogeneous media: chromatic channel-MIS free flight (analytic.glsl:9-51) ---------
template <class Col> struct MediumSample { bool scattered; Col weight; f3 exit_p, exit_dir; };

// ---- heterogeneous media (transport/volume/delta_tracking/delta_tracking.glsl) ----------
// A coefficient field: the stack program of a GLSL expression of p (validated at upload:
// known opcodes, stack depth within PTR_FIELD_MAX_STACK, END inside the table).
__device__ __forceinline__ float fract_(float x) { return x - floorf(x); }
__device__ f3 field_eval(const uint32_t* code, f3 p) {
    f3 st[PTR_FIELD_MAX_STACK];
    int sp = 0;
    for (int pc = 0;;) {
        const uint32_t op = __ldg(code + pc++);
        if (op == PTR_FOP_END) break;
        if (op == PTR_FOP_CONST) {
            st[sp++] = f3(__uint_as_float(__ldg(code + pc)), __uint_as_float(__ldg(code + pc + 1)),
                          __uint_as_float(__ldg(code + pc + 2)));
            pc += 3;
            continue;
        }
        if (op == PTR_FOP_P) { st[sp++] = p; continue; }
        if (op == PTR_FOP_SWZ) {
            const uint32_t c = __ldg(code + pc++);
            f3 v = st[sp - 1];
            float x = c == 0 ? v.x : c == 1 ? v.y : v.z;
            st[sp - 1] = f3(x, x, x);
            continue;
        }
        if (op >= PTR_FOP_ADD && op <= PTR_FOP_DIV) {
            f3 b = st[--sp], a = st[sp - 1];
            st[sp - 1] = op == PTR_FOP_ADD ? a + b : op == PTR_FOP_SUB ? a - b
                       : op == PTR_FOP_MUL ? a * b : f3(a.x / b.x, a.y / b.y, a.z / b.z);
            continue;
        }
        if (op >= PTR_FOP_NEG && op <= PTR_FOP_FRACT) {
            f3 a = st[sp - 1];
            float r[3] = {a.x, a.y, a.z};
            for (int k = 0; k < 3; ++k) {
                float x = r[k];
                switch (op) {
                    case PTR_FOP_NEG: x = -x; break;
                    case PTR_FOP_EXP: x = m_exp(x); break;
                    case PTR_FOP_LOG: x = m_log(x); break;
                    case PTR_FOP_SIN: x = m_sin(x); break;
                    case PTR_FOP_COS: x = m_cos(x); break;
                    case PTR_FOP_SQRT: x = sqrtf(x); break;
                    case PTR_FOP_ABS: x = fabsf(x); break;
                    case PTR_FOP_FLOOR: x = floorf(x); break;
                    default: x = fract_(x); break;
                }
                r[k] = x;
            }
            st[sp - 1] = f3(r[0], r[1], r[2]);
            continue;
        }
        if (op >= PTR_FOP_POW && op <= PTR_FOP_STEP) {
            f3 b = st[--sp], a = st[sp - 1];
            float ra[3] = {a.x, a.y, a.z}, rb[3] = {b.x, b.y, b.z};
            for (int k = 0; k < 3; ++k) {
                float x = ra[k], y = rb[k];
                switch (op) {
                    case PTR_FOP_POW: x = m_pow(x, y); break;
                    case PTR_FOP_MIN: x = y < x ? y : x; break;
                    case PTR_FOP_MAX: x = x < y ? y : x; break;
                    case PTR_FOP_MOD: x = x - y * floorf(x / y); break;
                    default: x = y < x ? 0.0f : 1.0f; break;   // step(edge = a, x = b)
                }
                ra[k] = x;
            }
            st[sp - 1] = f3(ra[0], ra[1], ra[2]);
            continue;
        }
        if (op >= PTR_FOP_CLAMP && op <= PTR_FOP_SMOOTHSTEP) {
            f3 c = st[--sp], b = st[--sp], a = st[sp - 1];
            float ra[3] = {a.x, a.y, a.z}, rb[3] = {b.x, b.y, b.z}, rc[3] = {c.x, c.y, c.z};
            for (int k = 0; k < 3; ++k) {
                float x;
                if (op == PTR_FOP_CLAMP) {
                    x = ra[k] < rb[k] ? rb[k] : ra[k];
                    x = rc[k] < x ? rc[k] : x;
                } else if (op == PTR_FOP_MIX) {
                    x = ra[k] * (1.0f - rc[k]) + rb[k] * rc[k];
                } else {   // smoothstep(e0 = a, e1 = b, x = c)
                    float t = (rc[k] - ra[k]) / (rb[k] - ra[k]);
                    t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
                    x = t * t * (3.0f - 2.0f * t);
                }
                ra[k] = x;
            }
            st[sp - 1] = f3(ra[0], ra[1], ra[2]);
            continue;
        }
        if (op == PTR_FOP_DOT) {
            f3 b = st[--sp], a = st[sp - 1];
            float d = dot(a, b);
            st[sp - 1] = f3(d, d, d);
            continue;
        }
        if (op == PTR_FOP_LENGTH) {
            float l = sqrtf(dot(st[sp - 1], st[sp - 1]));
            st[sp - 1] = f3(l, l, l);
            continue;
        }
        // PTR_FOP_VEC3: three broadcast scalars into one vector
        f3 z = st[--sp], y = st[--sp], x = st[sp - 1];
        st[sp - 1] = f3(x.x, y.x, z.x);
    }
    return st[0];
}
__device__ __forceinline__ bool mat_is_het(const ptr_material& m) { return (m.field_a | m.field_s) != 0; }
// The rendered medium at p: the fields (or constants), scaled down proportionally where the
// maximum extinction exceeds the majorant (the D1 ceiling of the generated lookup).
struct HetProps { f3 sa, ss; };
__device__ __forceinline__ HetProps het_props(const DevScene& S, const ptr_material& m, f3 p) {
    HetProps h;
    h.sa = m.field_a ? field_eval(S.field_code + (m.field_a - 1), p) : ld3(m.sigma_a);
    h.ss = m.field_s ? field_eval(S.field_code + (m.field_s - 1), p) : ld3(m.sigma_s);
    f3 st = h.sa + h.ss;
    float smax = gmax(st.x, gmax(st.y, st.z));
    float scale = smax > m.majorant ? m.majorant / smax : 1.0f;
    h.sa = h.sa * scale;
    h.ss = h.ss * scale;
    return h;
}
// The loop bound of a tracking walk of mean lambda tentative collisions (overrun chance
// below 1e-10 for every lambda)
__device__ __forceinline__ int tracking_cap(float lambda) {
    return (int)ceilf(lambda + 6.5f * sqrtf(lambda) + 12.0f);
}
// Delta tracking of a scattering segment (Kutz et al. 2017, Algorithm 4, with the
// history-aware average-based probabilities): xi are the site's two numbers, later
// collisions draw from the path's stream.  Absorption terminates (weight 0).
__device__ MediumSample<f3> medium_sample_delta(const DevScene& S, const ptr_material& m, const Ray& r, float t_max,
                                                float x0, float x1, Rng& rng) {
    MediumSample<f3> ms;
    ms.scattered = false;
    ms.weight = f3(1.0f);
    const float sbar = m.majorant;
    f3 w(1.0f);
    float t = 0.0f, xd = x0, xe = x1;
    const int cap = tracking_cap(sbar * t_max);
    for (int i = 0; i < cap; ++i) {
        t += -m_log(1.0f - xd) / sbar;
        if (t >= t_max) { ms.weight = w; return ms; }
        f3 p = r.o + r.d * t;
        HetProps h = het_props(S, m, p);
        f3 sn = vmax(f3(sbar) - (h.sa + h.ss), f3(0.0f));
        float pa = spectrum_average(h.sa * w);
        float ps = spectrum_average(h.ss * w);
        float pn = spectrum_average(sn * w);
        float c = pa + ps + pn;
        if (c <= 0.0f) { ms.weight = f3(0.0f); return ms; }
        pa /= c; ps /= c; pn /= c;
        if (xe < pa) { ms.weight = f3(0.0f); return ms; }
        if (xe < pa + ps) {
            ms.scattered = true;
            ms.exit_p = p;
            ms.exit_dir = r.d;
            ms.weight = w * h.ss / (sbar * gmax(ps, 1e-20f));
            return ms;
        }
        w = w * sn / (sbar * gmax(pn, 1e-20f));
        xd = rng.next();
        xe = rng.next();
    }
    ms.weight = w;
    return ms;
}
// Ratio tracking of exp(-int sigma) along a segment (Novak et al. 2014): sigma_a alone
// for the absorbing-only pass-through of the walk, sigma_t with pbrt's roulette (below
// 0.05, survive 1/4 with weight 4) for shadow segments.
__device__ f3 medium_ratio_track(const DevScene& S, const ptr_material& m, const Ray& r, float len, Rng& rng,
                                 bool extinction) {
    const float sbar = m.majorant;
    f3 T(1.0f);
    float t = 0.0f;
    const int cap = tracking_cap(sbar * len);
    for (int i = 0; i < cap; ++i) {
        t += -m_log(1.0f - rng.next()) / sbar;
        if (t >= len) return T;
        HetProps h = het_props(S, m, r.o + r.d * t);
        T = T * (vmax(f3(sbar) - (extinction ? h.sa + h.ss : h.sa), f3(0.0f)) / sbar);
        if (extinction && spectrum_max(T) < 0.05f) {
            if (rng.next() < 0.75f) return f3(0.0f);
            T = T / 0.25f;
        }
    }
    return T;
}
// The shadow query's own stream: hashed from the path's sampler base and its dimension
// at the NEE site, so a queued shadow query draws independently of the path's order.
__device__ __forceinline__ Rng shadow_rng(uint32_t base, uint32_t seed) {
    Rng r;
    r.base = pcg4d(make_uint4(base, seed, 0x53484457u, 0u)).x;
    r.dim = 0u;
    return r;
}
template <class Col>
__device__ __forceinline__ MediumSample<Col> medium_sample_analytic(Col sigma_a, Col sigma_s, const Ray& r, float t_max,
                                                                    float x0, float x1) {
    Col sigma_t = sigma_a + sigma_s;
    int c = sample_channel<Col>(x0);
    float sc = sigma_t[c];
    float t = sc == 0.0f ? t_max : -m_log(1.0f - x1) / sc;
    MediumSample<Col> ms;
    if (t < t_max) {
        Col tr = vexp(-sigma_t * t);
        float pdf = spectrum_average(sigma_t * tr);
        ms.scattered = true;
        ms.exit_p = r.o + r.d * t;
        ms.exit_dir = r.d;
        ms.weight = sigma_s * tr / gmax(pdf, 1e-20f);
    } else {
        Col tr = vexp(-sigma_t * t_max);
        float pdf = spectrum_average(tr);
        ms.scattered = false;
        ms.weight = tr / gmax(pdf, 1e-20f);
    }
    return ms;
}

// ---- equiangular medium NEE (transport/techniques/equiangular/equiangular.glsl:18-57;
// Kulla & Fajardo 2012): one estimate per medium segment with segment-start throughput.
// A light is picked by the lighting CDF (lighting_query_delta, features/lighting.ts:303-341);
// for a delta light its position and intensity are used as in the reference; area lights
// (quad, sphere, mesh: an extension the reference's Validator rejects) first draw a uniform point
// on their area and carry Le * cos_l / (d^2 * pdf_area).  The distance t along the segment
// is uniform in the angle subtended at the light point.  Returns true when a shadow query
// is due: from p_evt towards light_pos, adding contrib * visibility / denom.
template <class Col> struct EquiangularQuery { f3 p_evt, wi, light_pos; Col contrib; float denom; };
template <class Col>
__device__ __forceinline__ bool equiangular_site(const DevScene& S, int med_mat, const Ray& r, float t_max,
                                                 Rng& rng, Col thr, const Wl& wl, EquiangularQuery<Col>& q) {
    const ptr_material& mm = S.materials[med_mat];
    float uc = rng.next();
    int id = S.n_lights - 1;
    if (S.n_lights > 1)
        for (int i = 0; i < S.n_lights - 1; ++i)
            if (uc < S.lights[i].select_cdf) { id = i; break; }
    const ptr_light& l = S.lights[id];
    const float sel = S.n_lights == 1 ? 1.0f : l.select_pdf;
    f3 pos, nl(0.0f);
    float pdf_area = 1.0f;
    const bool area = light_in<LightArea>(l.kind);
    if (area) {
        float y0 = rng.next();
        float y1 = rng.next();
        auto ap = [&](auto K) { decltype(K)::area_point(S, l, y0, y1, pos, nl, pdf_area); };
        dispatch_light<LightArea, true>(l.kind, ap);
    } else {
        pos = ld3(l.p);
    }
    f3 D = pos - r.o;
    float t_c = dot(D, r.d);
    float h2 = gmax(dot(D, D) - t_c * t_c, 1e-8f);
    float h = sqrtf(h2);
    float theta_a = m_atan2(0.0f - t_c, h);
    float theta_b = m_atan2(t_max - t_c, h);
    float u = rng.next();
    float theta = theta_a * (1.0f - u) + theta_b * u;
    float t = t_c + h * m_tan(theta);
    float pdf_t = h / ((theta_b - theta_a) * (h2 + (t - t_c) * (t - t_c)));
    q.p_evt = r.o + r.d * t;
    Col sigma_s = Colors<Col>::sigma_s(S, med_mat, wl);
    if (spectrum_is_black(sigma_s)) return false;
    Col T_seg = vexp(-(Colors<Col>::sigma_a(S, med_mat, wl) + sigma_s) * t);
    f3 to_light = pos - q.p_evt;
    float d2 = gmax(dot(to_light, to_light), 1e-8f);
    float dist = sqrtf(d2);
    q.wi = to_light / dist;
    Col Le;
    if (area) {
        float cos_l = dot(nl, -q.wi);
        if (!(cos_l > 0.0f)) return false;
        Le = Colors<Col>::light(S, id, wl) * (cos_l / d2);
        q.denom = pdf_t * (pdf_area * sel);
    } else {
        Le = Colors<Col>::light(S, id, wl) / d2;
        q.denom = pdf_t * sel;
    }
    q.light_pos = pos;
    Col ph(hg_eval(q.wi, -r.d, mm.phase_g));
    q.contrib = thr * T_seg * sigma_s * ph * Le;
    return true;
}

}  // namespace ptx
