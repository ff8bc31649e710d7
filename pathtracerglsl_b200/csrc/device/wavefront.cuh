// wavefront.cuh — the transport loop as a wavefront of kernels over a path pool.
//
// The reference runs the whole walk (transport/integrators/pt/pt.ts:299-464) as one
// fragment per pixel.  Here each path lives in struct-of-arrays state in HBM and the walk
// is split at its two traversals:
//
//   k_generate  camera rays + path_state_init for one wave of (pixel, sample) paths
//   k_closest   nearest hit of every live path (the scene_intersect traversal)
//   k_shade     one walk iteration: medium segment, null pass-through, emitter scoring,
//               NEE sampling (emits a shadow query), BSDF continuation, roulette, spawn;
//               live paths are compacted into the next queue with warp ballots
//   k_shadow    visibility / transmittance of the queued shadow queries, folded into
//               the owning path's radiance
//   k_film      per-pixel FP64 sum and sum of squares over the wave's samples
//
// Every path draws its random numbers in exactly the order of the reference's walk
// (the sampler is counter-based, so a path's stream does not depend on scheduling), and
// its radiance is accumulated in the same order: emission, then the vertex's NEE term,
// then the next vertex's emission.
#pragma once
#include "occupants.cuh"
#include "bvh.cuh"
#include "adjoint.cuh"
#include "materials/registry.cuh"

namespace ptx {

// Path pool (indexed by path slot).
// One field of a two-field path record: path i's value at p[2 i] and the partner field's
// at p[2 i + 1], so the two 16-byte fields a kernel reads and writes together fill one
// 32-byte sector (a surviving path's store never half-fills a sector that the L2 would
// first have to read back from DRAM).
template <class T> struct Pair {
    T* p;
    __host__ __device__ __forceinline__ T& operator[](long long i) const { return p[2 * i]; }
    __host__ __device__ __forceinline__ explicit operator bool() const { return p != nullptr; }
};

struct PathPool {
    Pair<float4> ray_o;  // origin.xyz, prev_bsdf_pdf          } one record
    Pair<float4> ray_d;  // direction.xyz, eta_scale           }
    Pair<float4> thr;    // throughput.xyz, -                  } one record
    Pair<float4> rad;    // radiance.xyz, -                    }
    Pair<float4> prev_q; // stored light-query point (prev_query.p)  } one record, with st
    float4* prev_n;    // stored light-query normal and two-sidedness (light-tree selection)
    unsigned* sh_seed; // the shadow query's sampler dimension at its NEE site (heterogeneous media)
    // first-hit pictures (programs with measurement.aovs; NULL otherwise): per path its
    // albedo and normal samples (2 float4), per pixel their FP64 sums (albedo block of 3
    // doubles per pixel, then the normal block)
    float4* aov;
    double* aov_sum;
    Pair<int4> st;       // bounce, current_medium, null_crossings, prev_was_delta
    uint2* rng;        // sampler base, dimension
    Pair<float4> hit;    // t, u, v, - ; (region, element, prim) in hit_i    } one record
    Pair<int4> hit_i;    // region_owner, element, prim, -                   }
    // shadow queries (one per path and iteration at most)
    Pair<float4> sh_o;   // origin.xyz, max distance (opaque form)     } one record
    Pair<float4> sh_d;   // direction.xyz, crossings left (as int)     }
    Pair<float4> sh_lp;  // light point.xyz, MIS weight                } one record
    Pair<float4> sh_c;   // contribution prefix throughput*Le*f*cos (xyz), pdf  }
    // second shadow slot: the per-segment equiangular query of the same iteration (a path
    // may issue it and a surface NEE query in one walk iteration); NULL when unused
    Pair<float4> sh2_o;
    Pair<float4> sh2_d;
    Pair<float4> sh2_lp;
    Pair<float4> sh2_c;
    int* q[2];         // live-path queues (ping-pong)
    int* shq;          // shadow queue
    int* shq2;         // second-slot shadow queue (count in cnt[4])
    unsigned int* cnt; // [0],[1] queue counts, [2] shadow count, [3] error flags, [4] slot-2 shadow count
    unsigned long long* stats; // [0] closest queries, [1] shadow queries, [2] paths
    long long* wave;   // [0] first global path index of the wave, [1] wave size
    int* job;          // batched renders: the job (scene x program x frame) of each path
    // adjoint replay only (NULL otherwise)
    float4* l_rem;     // radiance the path has still to gather (forward total minus what it gathered)
    float4* dl;        // adjoint radiance of the path: dLoss/dI of its pixel / spp
    float4* sh_g;      // shadow query: lobe derivative D = dlog f(wi_light) - dlog w_cont (xyz)
    int* sh_gm;        // shadow query: vertex material | kind << 16
    // spectral colour model only (NULL otherwise): the path's four wavelengths and their
    // sampling densities; the shadow queries' pdfs (the colour fills all four lanes)
    float4* wl;
    float4* wl_pdf;
    float* sh_pdf;
    float* sh2_pdf;
    // occupant-sorted shading queue: k_closest keys every live path by the occupant it will
    // shade (material model of the hit, inside a medium or not) and counts the keys; a scan
    // and a scatter rebuild the live queue grouped by key before k_shade (sort_buckets <= 1:
    // off, k_shade reads the compacted queue as it is)
    int sort_buckets;
    int* q_sorted;
    unsigned char* sort_key;  // shading class per path (indexed by path)
    unsigned* sort_hist;      // counting-sort scratch: [key][chunk] counts, then offsets
    // work tickets of the queue kernels ([0] k_closest, [1] / [2] k_shadow slots 0 / 1,
    // [3] k_shade), each cleared by the kernel that runs before its consumer; NULL: the
    // kernels fall back to a static grid-stride loop
    unsigned* fetch;
    // ray-coherence order (tuning ray_sort): k_shade keys every spawned ray and every shadow
    // query by (direction octant, origin octant about the scene centre); counting sorts
    // rebuild the closest-hit and shadow queues grouped by key for the traversal kernels
    // (k_shade itself keeps reading the compacted queue q[in])
    int ray_sort;             // keys and sorted queues are written
    int ray_in;               // this k_closest reads q_ray (set per launch; 0 for camera rays)
    unsigned char* rkey;      // key per position of the next live queue
    unsigned char* skey;      // key per position of the shadow queue
    int* q_ray;
    int* shq_s;
    // the adjoint's walk log (ptr_backward; NULL otherwise): for walk iterations below
    // hit_log_iters the forward walk records, per path, four float4 at
    // [4 * (iter * hit_log_stride + path)]: its closest hit (hit, hit_i), then its slot-0
    // shadow query's visibility and media (ShadowLog).  The replay of the same paths reads
    // them back instead of walking the scene again.  iter and hit_log_mode (1 record,
    // 2 replay) are set per launch.
    float4* hit_log;
    long long hit_log_stride;
    int hit_log_iters, hit_log_mode, iter, pad_log;
};

constexpr int kRayBuckets = 64;   // ray_key values
__device__ __forceinline__ unsigned ray_key(const DevScene& S, f3 o, f3 d) {
    unsigned k = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    k = (k << 3) | (o.x > S.sort_c[0] ? 1u : 0u) | (o.y > S.sort_c[1] ? 2u : 0u) | (o.z > S.sort_c[2] ? 4u : 0u);
    return k;
}
// The queue a k_closest of iteration `in` reads.
__device__ __forceinline__ const int* closest_queue(const PathPool& pool, int in);

// Warp-uniform cursor over a device-counted queue.  With a ticket counter every warp takes
// the next 32 entries when it is done with its last ones, so warps whose rays are long do
// not hold the others' work back (dynamic balance on a one-wave resident grid); without
// one, a grid-stride loop whose trip count is rounded to whole warps.
struct QueueCursor {
    unsigned n, stride, k;
    unsigned* ticket;
    __device__ __forceinline__ QueueCursor(unsigned n_, unsigned* t) : n(n_), ticket(t) {
        stride = gridDim.x * blockDim.x;
        k = blockIdx.x * blockDim.x + threadIdx.x - stride;
    }
    __device__ __forceinline__ bool next(unsigned& out) {
        if (ticket) {
            unsigned base = 0u;
            if ((threadIdx.x & 31u) == 0u) base = atomicAdd(ticket, 32u);
            base = __shfl_sync(0xffffffffu, base, 0);
            out = base + (threadIdx.x & 31u);
            return base < n;
        }
        k += stride;
        out = k;
        return k < ((n + 31u) & ~31u);
    }
};

// Adjoint replay tables: the adjoint image (3 floats per pixel, row 0 at the bottom), the
// per-sample scale and the float64 gradient buffer (PTR_GRAD_SLOTS per material).
struct AdjParams {
    const float* dl_image;
    float inv_spp;
    double* grads;
};

struct FrameParams {
    int width, height, spp, first_sample;
    uint32_t salt;
    int px_off, py_off;
    int img_w, img_h;  // the full image the camera maps film points through
    long long total;   // width*height*spp
    int capacity;
    ptr_camera cam;
    int wavelengths;   // PTR_WAVELENGTHS_* (spectral programs)
    float lambda_min, lambda_max;
};

struct ProgParams {
    int max_bounces, direct, rr_start, max_null;
    float rr_max_survival;
    int scattering;
    int equiangular;   // PTR_EQUIANGULAR_*: per-segment medium NEE replaces the at-vertex site
    int light_tree;    // light-tree selection (the scene carries the tree)
};

// Batched renders: per job its scene, program knobs, frame and film; offsets[j] is the
// first global path index of job j (offsets[n_jobs] = total paths).
struct BatchJob {
    FrameParams frame;
    double* sum;
    double* sumsq;
};
struct BatchTables {
    const DevScene* scenes;
    const ProgParams* progs;
    const BatchJob* jobs;
    const long long* offsets;
    int n_jobs;
    long long total;
    int capacity;
};

// The job of global path index g: the last j with offsets[j] <= g.  A batched wave's pool
// slot i holds path base + i for the whole wave (base = pool.wave[0]), so the kernels find a
// path's job from its slot by this search over the small, cached offsets table instead of
// a per-path load from HBM that every scene-table read would wait for.
__device__ __forceinline__ int job_of(const BatchTables& bt, long long g) {
    int lo = 0, hi = bt.n_jobs - 1;   // last j with offsets[j] <= g
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (bt.offsets[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The jobs of a batched wave's slots.  A wave that lies inside one job (every wave of a
// large job but its last) needs no search at all: its job is found once per thread.
struct WaveJobs {
    long long base = 0;
    int single = 0;   // >= 0: every slot of the wave belongs to this job
    WaveJobs() = default;
    __device__ __forceinline__ WaveJobs(const PathPool& pool, const BatchTables& bt) {
        base = pool.wave[0];
        const int j = job_of(bt, base);
        single = bt.offsets[j + 1] >= base + pool.wave[1] ? j : -1;
    }
    __device__ __forceinline__ int of(const BatchTables& bt, int slot) const {
        return single >= 0 ? single : job_of(bt, base + slot);
    }
};

constexpr unsigned kErrStack = 1u;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated append: one atomic per warp, slots in lane order.
__device__ __forceinline__ int warp_append(unsigned* counter, bool pred) {
    unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0u) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return pred ? (int)(base + __popc(mask & lanemask_lt())) : -1;
}

// ---- scene queries -------------------------------------------------------------------
// Nearest hit over every arm; returns region (or -1), element, primitive and t.

__device__ __forceinline__ float4 int4_as_float4(int4 v) {
    return make_float4(__int_as_float(v.x), __int_as_float(v.y), __int_as_float(v.z), __int_as_float(v.w));
}
__device__ __forceinline__ int4 float4_as_int4(float4 v) {
    return make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z), __float_as_int(v.w));
}
template <int V> struct ShapeC { static constexpr int value = V; };
// Calls f(ShapeC<shape>{}, first, end) for each same-shape run of the region list, the
// shape a compile-time constant for the analytic shapes the build holds (one dispatch per
// run instead of one per region); other runs get f(ShapeC<-1>{}, ...).
template <class F>
__device__ __forceinline__ void for_region_runs(const DevScene& S, F&& f) {
    for (int q = 0; q < S.n_runs; ++q) {
        const int4 run = __ldg(S.region_runs + q);
        const int a = run.y, b = run.y + run.z;
        if (has_shape(PTR_SHAPE_SPHERE) && run.x == PTR_SHAPE_SPHERE) f(ShapeC<PTR_SHAPE_SPHERE>{}, a, b);
        else if (has_shape(PTR_SHAPE_QUAD) && run.x == PTR_SHAPE_QUAD) f(ShapeC<PTR_SHAPE_QUAD>{}, a, b);
        else f(ShapeC<-1>{}, a, b);
    }
}

// The root of region i inside a run of one analytic shape, its parameters fetched as
// aligned float4s: an uploaded region table is 256-byte aligned and its records 80 bytes,
// so a record's bytes 16..79 are four float4s (ior, p[0..2]), (p[3..6]), (p[7..10]),
// (p[11..14]).  Same operands as analytic_root_shape, fewer load instructions.
template <int SH>
__device__ __forceinline__ bool run_root(const DevScene& S, int i, const Ray& r, float& t) {
    const float4* g4 = reinterpret_cast<const float4*>(S.regions + i);
    if constexpr (SH == PTR_SHAPE_SPHERE) {
        const float4 a = __ldg(g4 + 1), b = __ldg(g4 + 2);
        return sphere_intersect(r, f3(a.y, a.z, a.w), b.x, t);
    } else if constexpr (SH == PTR_SHAPE_QUAD) {
        const float4 a = __ldg(g4 + 1), b = __ldg(g4 + 2), c = __ldg(g4 + 3), d = __ldg(g4 + 4);
        return quad_intersect(r, f3(a.y, a.z, a.w), f3(b.x, b.y, b.z), f3(b.w, c.x, c.y), f3(c.z, c.w, d.x), t);
    } else {
        return analytic_root(S.regions[i], r, t);
    }
}
#ifndef __CUDACC_RTC__   // (NVRTC has no offsetof; the library build checks the layout)
static_assert(sizeof(ptr_region) == 80 && __builtin_offsetof(ptr_region, p) == 20, "run_root's float4 view of a region record");
#endif

__device__ __forceinline__ HitRec scene_closest(const DevScene& S, const Ray& r, Work* w = nullptr) {
    HitRec h;
    h.t = kMaxDist;
    h.u = h.v = 0.f;
    h.region = -1;
    h.element = 0;
    h.prim = -1;
    auto arm = [&](int i, const ptr_region& g, int shape) {
        if (shape >= PTR_SHAPE_MESH) {
            accel_closest(S, g, i, r, h, w);
            return;
        }
        float t;
        if (analytic_root_shape(shape, g, r, t) && t < h.t) {
            h.t = t;
            h.region = i;
            h.element = 0;
            h.prim = -1;
        }
    };
#if PTR_SPEC_NREGIONS > 0
    constexpr bool tabled = false;
#pragma unroll
    for (int k = 0; k < PTR_SPEC_NREGIONS; ++k) {
        const int sh = spec_shape(k);   // folds to a constant in each unrolled arm
        float t;
        bool hit = false;
        if (sh == PTR_SHAPE_SPHERE) hit = run_root<PTR_SHAPE_SPHERE>(S, k, r, t);
        else if (sh == PTR_SHAPE_QUAD) hit = run_root<PTR_SHAPE_QUAD>(S, k, r, t);
        else arm(k, S.regions[k], sh);
        if (hit && t < h.t) {
            h.t = t;
            h.region = k;
            h.element = 0;
            h.prim = -1;
        }
    }
#else
    const bool tabled = S.region_bvh != nullptr;
    if (!tabled && S.region_runs) {
        for_region_runs(S, [&](auto sc, int a, int b) {
            constexpr int SH = decltype(sc)::value;
            for (int i = a; i < b; ++i) {
                if constexpr (SH >= 0) {
                    float t;
                    if (run_root<SH>(S, i, r, t) && t < h.t) {
                        h.t = t;
                        h.region = i;
                        h.element = 0;
                        h.prim = -1;
                    }
                } else {
                    arm(i, S.regions[i], S.regions[i].shape);
                }
            }
        });
    } else {
        const int n = tabled ? S.n_linear : S.n_regions;
        for (int k = 0; k < n; ++k) {
            const int i = tabled ? S.linear_regions[k] : k;
            arm(i, S.regions[i], S.regions[i].shape);
        }
    }
#endif
    if (tabled) {
        float tb = h.t;
        walk_binary(S, S.region_bvh, r.o, r.d, tb, [&](int off, int cnt) {
            for (int j = off; j < off + cnt; ++j) {
                const int i = S.region_items[j];
                float t;
                // strict '<', and on an exact tie the lower region index (the order of the
                // unrolled arms) keeps the hit
                if (analytic_root(S.regions[i], r, t) && (t < tb || (t == tb && h.region > i))) {
                    tb = t;
                    h.t = t;
                    h.region = i;
                    h.element = 0;
                    h.prim = -1;
                }
            }
            return false;
        });
    }
    return h;
}

__device__ __forceinline__ bool scene_any(const DevScene& S, const Ray& r, float max_dist, Work* w = nullptr) {
    auto arm = [&](const ptr_region& g, int shape) -> bool {
        if (shape >= PTR_SHAPE_MESH) return accel_any(S, g, r, max_dist, w);
        float t;
        return analytic_root_shape(shape, g, r, t) && t < max_dist;
    };
#if PTR_SPEC_NREGIONS > 0
    constexpr bool tabled = false;
#pragma unroll
    for (int k = 0; k < PTR_SPEC_NREGIONS; ++k) {
        const int sh = spec_shape(k);   // folds to a constant in each unrolled arm
        float t;
        if (sh == PTR_SHAPE_SPHERE) {
            if (run_root<PTR_SHAPE_SPHERE>(S, k, r, t) && t < max_dist) return true;
        } else if (sh == PTR_SHAPE_QUAD) {
            if (run_root<PTR_SHAPE_QUAD>(S, k, r, t) && t < max_dist) return true;
        } else if (arm(S.regions[k], sh)) {
            return true;
        }
    }
#else
    const bool tabled = S.region_bvh != nullptr;
    if (!tabled && S.region_runs) {
        bool hit = false;
        for (int q = 0; q < S.n_runs && !hit; ++q) {
            const int4 run = __ldg(S.region_runs + q);
            const int a = run.y, b = run.y + run.z;
            float t;
            if (has_shape(PTR_SHAPE_SPHERE) && run.x == PTR_SHAPE_SPHERE) {
                for (int i = a; i < b && !hit; ++i) hit = run_root<PTR_SHAPE_SPHERE>(S, i, r, t) && t < max_dist;
            } else if (has_shape(PTR_SHAPE_QUAD) && run.x == PTR_SHAPE_QUAD) {
                for (int i = a; i < b && !hit; ++i) hit = run_root<PTR_SHAPE_QUAD>(S, i, r, t) && t < max_dist;
            } else {
                for (int i = a; i < b && !hit; ++i) hit = arm(S.regions[i], S.regions[i].shape);
            }
        }
        if (hit) return true;
    } else {
        const int n = tabled ? S.n_linear : S.n_regions;
        for (int k = 0; k < n; ++k) {
            const int i = tabled ? S.linear_regions[k] : k;
            if (arm(S.regions[i], S.regions[i].shape)) return true;
        }
    }
#endif
    if (tabled) {
        return walk_binary(S, S.region_bvh, r.o, r.d, max_dist, [&](int off, int cnt) {
            for (int j = off; j < off + cnt; ++j) {
                float t;
                if (analytic_root(S.regions[S.region_items[j]], r, t) && t < max_dist) return true;
            }
            return false;
        });
    }
    return false;
}

// Innermost-wins point classification (features/intersection.ts:1121-1225); with a region
// BVH the bounded solids are found by the containment descent (bvh.ts bvhPointWalkLines).
__device__ __forceinline__ int scene_region_at(const DevScene& S, f3 p) {
    int region = -1;
    float best = -1.0e20f;
    auto arm = [&](int i, const ptr_region& g, int shape) {
        float d = shape == PTR_SHAPE_INSTANCES ? accel_region_sdf(S, g, p) : analytic_sdf_shape(shape, g, p);
        if (d < 0.0f && (d > best || (d == best && i < region))) { best = d; region = i; }
    };
#if PTR_SPEC_NREGIONS > 0
    constexpr bool tabled = false;
#pragma unroll
    for (int k = 0; k < PTR_SPEC_NREGIONS; ++k) arm(k, S.regions[k], spec_shape(k));
#else
    const bool tabled = S.region_bvh != nullptr;
    if (!tabled && S.region_runs) {
        for_region_runs(S, [&](auto sc, int a, int b) {
            constexpr int SH = decltype(sc)::value;
            for (int i = a; i < b; ++i) {
                if constexpr (SH == PTR_SHAPE_SPHERE) {   // the sphere's centre and radius as two float4 loads
                    const float4* g4 = reinterpret_cast<const float4*>(S.regions + i);
                    const float4 c = __ldg(g4 + 1), rr = __ldg(g4 + 2);
                    const float d = length(p - f3(c.y, c.z, c.w)) - rr.x;
                    if (d < 0.0f && (d > best || (d == best && i < region))) { best = d; region = i; }
                } else {
                    arm(i, S.regions[i], SH >= 0 ? SH : S.regions[i].shape);
                }
            }
        });
    } else {
        const int n = tabled ? S.n_linear : S.n_regions;
        for (int k = 0; k < n; ++k) {
            const int i = tabled ? S.linear_regions[k] : k;
            arm(i, S.regions[i], S.regions[i].shape);
        }
    }
#endif
    if (tabled) {
        int stack[kBvhStack];
        int ptr = 0;
        stack[0] = 0;
        while (ptr >= 0) {
            int ni = stack[ptr];
            ptr--;
            float4 n0 = __ldg(S.region_bvh + 2 * ni), n1 = __ldg(S.region_bvh + 2 * ni + 1);
            if (!(p.x >= n0.x && p.y >= n0.y && p.z >= n0.z && p.x <= n1.x && p.y <= n1.y && p.z <= n1.z)) continue;
            if (n0.w >= 0.0f) {
                for (int j = (int)n1.w; j < (int)n1.w + (int)n0.w; ++j) {
                    const int i = S.region_items[j];
                    float d = analytic_sdf(S.regions[i], p);
                    if (d < 0.0f && (d > best || (d == best && i < region))) { best = d; region = i; }
                }
            } else {
                int L = ni + 1, R = (int)n1.w;
                if (ptr + 2 < kBvhStack) { stack[++ptr] = L; stack[++ptr] = R; }
                else flag_error(S, kErrBvhStack);
            }
        }
    }
    return region;
}

// Complete the hit record: point, uncertainty, frame, and the region classification of
// scene_intersect (intersection.ts:1665-1713).
__device__ __forceinline__ void fill_hit(const DevScene& S, const Ray& r, const HitRec& hr, Hit& h) {
    h.t = hr.t;
    h.p = r.o + r.d * hr.t;
    h.region_owner = hr.region;
    h.element = hr.element;
    h.alpha = -1.0f;
    const ptr_region& g = S.regions[hr.region];
    if (g.shape == PTR_SHAPE_MESH || (g.shape == PTR_SHAPE_INSTANCES && S.batches[g.ref].proto_shape == PTR_SHAPE_MESH)) {
        // mesh hits: frame from the (normalised) shading normal, ng the triangle's plane normal
        f3 ngv;
        f3 n = accel_hit_normal(S, g, hr, r, h, ngv);
        h.frame = ambient_frame(n);
        h.ng = ngv;
    } else {
        f3 n;
        if (g.shape == PTR_SHAPE_INSTANCES) {
            f3 unused;
            n = accel_hit_normal(S, g, hr, r, h, unused);
        } else {
            n = analytic_normal(g, h.p);
            h.eps = fp_uncertainty(h.p);
        }
        h.frame = ambient_frame(n);
        h.ng = h.frame.n;   // a primitive's normal is its true surface normal
    }
    int outside = scene_region_at(S, h.p + h.ng * kEpsInterface);
    if (dot(r.d, h.ng) < 0.0f) {
        h.region_from = outside;
        h.region_to = hr.region;
    } else {
        h.region_from = g.thin ? scene_region_at(S, h.p + h.ng * (-kEpsInterface)) : hr.region;
        h.region_to = outside;
        h.frame = ambient_frame(-h.frame.n);
        h.ng = -h.ng;
    }
}

__device__ __forceinline__ int material_of(const DevScene& S, int region) {
    return region < 0 ? S.ambient_material : S.regions[region].material;
}
__device__ __forceinline__ float ior_of(const DevScene& S, int region) {
    return region < 0 ? 1.0f : S.regions[region].ior;
}
__device__ __forceinline__ bool mat_has_medium(const DevScene& S, int m) {
    return m >= 0 && (S.materials[m].flags & PTR_MATF_MEDIUM);
}
__device__ __forceinline__ bool scatter_live(const DevScene& S, const ProgParams& P, int m) {
    return P.scattering && (S.materials[m].flags & PTR_MATF_SCATTERING);
}
template <class Col>
__device__ __forceinline__ Col medium_transmittance(const DevScene& S, const ProgParams& P, int m, float len, const Wl& wl) {
    Col st = scatter_live(S, P, m) ? Colors<Col>::sigma_a(S, m, wl) + Colors<Col>::sigma_s(S, m, wl)
                                   : Colors<Col>::sigma_a(S, m, wl);
    return vexp(-st * len);
}

// wavelengths_sample (color/spectral/spectral.glsl:1-10): one number, four cyclic
// quarter-interval offsets in CDF space, each lane with its own marginal density; the
// visible density is the normalised sech^2 (visible.glsl:3-13), or uniform (uniform.glsl).
__device__ __forceinline__ void wavelengths_sample(const FrameParams& F, float u, float4& lam, float4& pdf) {
    float l[4], p[4];
    for (int k = 0; k < 4; ++k) {
        float v = u + 0.25f * (float)k;
        v = v - floorf(v);
        if (F.wavelengths == PTR_WAVELENGTHS_UNIFORM) {
            l[k] = F.lambda_min + (F.lambda_max - F.lambda_min) * v;
            p[k] = 1.0f / (F.lambda_max - F.lambda_min);
        } else {
            float a = m_tanh(0.0072f * (F.lambda_min - 538.0f));
            float b = m_tanh(0.0072f * (F.lambda_max - 538.0f));
            l[k] = 538.0f + m_atanh(a * (1.0f - v) + b * v) / 0.0072f;
            float c = m_cosh(0.0072f * (l[k] - 538.0f));
            p[k] = 0.0072f / ((b - a) * c * c);
        }
    }
    lam = make_float4(l[0], l[1], l[2], l[3]);
    pdf = make_float4(p[0], p[1], p[2], p[3]);
}

// color_to_pixel (spectral.glsl:27-33) with the CIE 1931 sensor (sensor/cie1931/cie1931.glsl:3-5):
// 0.25 * sum_i M xyz(lambda_i) / int(ybar) * (L_i / pdf_i).
__device__ __forceinline__ f3 color_to_pixel(const DevScene& S, float4 L, float4 lam, float4 pdf) {
    const float Ls[4] = {L.x, L.y, L.z, L.w}, ls[4] = {lam.x, lam.y, lam.z, lam.w}, ps[4] = {pdf.x, pdf.y, pdf.z, pdf.w};
    f3 pixel(0.0f);
    for (int k = 0; k < 4; ++k) {
        float4 c = spectral_curves(S, ls[k]);
        f3 rgb(S.spec_m[0] * c.x + S.spec_m[1] * c.y + S.spec_m[2] * c.z,
               S.spec_m[3] * c.x + S.spec_m[4] * c.y + S.spec_m[5] * c.z,
               S.spec_m[6] * c.x + S.spec_m[7] * c.y + S.spec_m[8] * c.z);
        pixel = pixel + rgb / S.spec_y * (Ls[k] / ps[k]);
    }
    return 0.25f * pixel;
}

// ---- kernels ---------------------------------------------------------------------------

// Camera rays for one wave (accumulation.ts:14-26 cameraSample; pinhole.glsl:4-18).
template <bool ADJ = false, bool SPECTRAL = false>
__global__ void k_generate(DevScene S, PathPool pool, const FrameParams* fp, AdjParams adj = AdjParams{}) {
    const FrameParams F = *fp;
    long long base = pool.wave[0];
    long long n = F.total - base;
    if (n > F.capacity) n = F.capacity;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        pool.cnt[0] = (unsigned)n;
        pool.wave[1] = n;
        pool.stats[2] += (unsigned long long)n;
        if (pool.fetch) pool.fetch[0] = 0u;
    }
    const long long npix = (long long)F.width * F.height;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long g = base + i;
        int pix = (int)(g % npix);
        int sample = (int)(g / npix);
        int x = pix % F.width, y = pix / F.width;
        Rng rng;
        rng.init((uint32_t)(x + F.px_off), (uint32_t)(y + F.py_off), (uint32_t)(F.first_sample + sample), F.salt);
        float pxf = (float)x + 0.5f + (float)F.px_off;
        float pyf = (float)y + 0.5f + (float)F.py_off;
        float a0 = rng.next();
        float a1 = rng.next();
        float fx = pxf + (a0 - 0.5f), fy = pyf + (a1 - 0.5f);
        if (SPECTRAL) {   // wavelengths_sample, between the film point and the camera ray
            float4 lam, pdf;
            wavelengths_sample(F, rng.next(), lam, pdf);
            pool.wl[i] = lam;
            pool.wl_pdf[i] = pdf;
        }
        rng.next();   // the lens draw (a pinhole has no aperture)
        rng.next();
        float ndcx = (2.0f * fx / (float)F.img_w) - 1.0f;
        float ndcy = (2.0f * fy / (float)F.img_h) - 1.0f;
        ndcx *= F.cam.aspect;
        f3 dir = normalize(ld3(F.cam.forward) + ndcx * F.cam.tan_fov * ld3(F.cam.right) +
                           ndcy * F.cam.tan_fov * ld3(F.cam.up));
        f3 o = ld3(F.cam.position);
        int medium = S.has_media ? scene_region_at(S, o) : -1;
        if (ADJ) {   // replay: the forward pass left this path's total radiance in rad
            pool.l_rem[i] = pool.rad[i];
            const float* g = adj.dl_image + 3 * (size_t)pix;
            pool.dl[i] = make_float4(g[0] * adj.inv_spp, g[1] * adj.inv_spp, g[2] * adj.inv_spp, 0.f);
        }
        pool.ray_o[i] = f4(o, 0.0f);
        pool.ray_d[i] = f4(dir, 1.0f);
        pool.thr[i] = make_float4(1.f, 1.f, 1.f, 1.f);   // the spectral model's fourth lane included
        pool.rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        pool.prev_q[i] = f4(o, 0.0f);
        pool.st[i] = make_int4(0, medium, 0, 1);
        pool.rng[i] = make_uint2(rng.base, rng.dim);
        if (pool.aov) { pool.aov[2 * i] = make_float4(0.f, 0.f, 0.f, 0.f); pool.aov[2 * i + 1] = make_float4(0.f, 0.f, 0.f, 0.f); }
        pool.q[0][i] = (int)i;
    }
}

#ifndef PTR_TRACE_MIN_BLOCKS
#define PTR_TRACE_MIN_BLOCKS 4
#endif

// Fold a thread's tally into S.work (one atomic per warp and counter).
__device__ __forceinline__ void flush_work(const DevScene& S, const Work& w) {
    unsigned v[4] = {w.nodes, w.tris, w.tlas, w.inst};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        unsigned x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(&S.work[k], (unsigned long long)x);
    }
}

constexpr int kMaxSortBuckets = 32;
// Shading class of a live path: 0 miss, 1 + the material model of the surface it hit; with
// more than 8 buckets, + 8 when its segment starts inside a medium (the medium arm runs first).
__device__ __forceinline__ unsigned shade_key(const DevScene& S, int region, int cur_med, int buckets) {
    unsigned k = 0u;
    if (region >= 0) {
        const int m = S.regions[region].material;
        k = 1u + (unsigned)(m >= 0 ? S.materials[m].model : 0);
    }
    if (buckets > 8) {
        const int mm = cur_med < 0 ? S.ambient_material : S.regions[cur_med].material;
        if (mm >= 0 && (S.materials[mm].flags & PTR_MATF_MEDIUM)) k += 8u;
    }
    return k < (unsigned)buckets ? k : (unsigned)buckets - 1u;
}

// Nearest hit of every live path (and, for the sorted queue, its shading key).
// Closest hits of a queue whose scene is analytic regions plus one instanced mesh batch
// walked by the flat two-level loop: a lane whose query ends takes the next ray at once
// (warp-aggregated tickets whenever at least kRefillMin lanes are idle) instead of idling
// until the warp's slowest ray is done.  The regions before and after the instanced one
// are tested in region order around the walk, as in scene_closest, so hits are identical.
// (PTR_REFILL=0 builds keep the per-warp queue cursor everywhere.)
#ifndef PTR_REFILL
#define PTR_REFILL 1
#endif
constexpr int kRefillMin = 8;
template <bool COUNT>
__device__ __forceinline__ void closest_refill(const DevScene& S, const PathPool& pool, const int* q, unsigned n, int buckets,
                                               unsigned* ticket, Work* w) {
    const int fr = S.flat_region;
    const DevBatch& b = S.batches[S.regions[fr].ref];
    const DevMesh& m = S.meshes[b.proto_mesh];
    const unsigned lane = threadIdx.x & 31u;
    InstFlat f;
    Ray r;
    HitRec h;
    int i = -1, steps = 0;
    bool active = false, exhausted = false;
    for (;;) {
        if (!exhausted) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (__popc(need) >= kRefillMin) {
                const int leader = __ffs(need) - 1;
                unsigned base = 0u;
                if ((int)lane == leader) base = atomicAdd(ticket, (unsigned)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (unsigned)__popc(need) >= n) exhausted = true;
                if (!active) {
                    const unsigned k = base + __popc(need & lanemask_lt());
                    if (k < n) {
                        i = q[k];
                        r.o = xyz(pool.ray_o[i]);
                        r.d = xyz(pool.ray_d[i]);
                        h.t = kMaxDist;
                        h.u = h.v = 0.f;
                        h.region = -1;
                        h.element = 0;
                        h.prim = -1;
                        for (int g = 0; g < fr; ++g) {
                            float t;
                            if (analytic_root(S.regions[g], r, t) && t < h.t) { h.t = t; h.region = g; h.element = 0; h.prim = -1; }
                        }
                        f.init(r, h.t);
                        steps = 0;
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (!active) continue;
        bool more = f.step<false>(S, b, m, fr, r, h, 0.0f, COUNT ? w : nullptr);
        if (more && ++steps >= kFlatGuard) {
            flag_error(S, kErrCwGuard);
            more = false;
        }
        if (!more) {
            for (int g = fr + 1; g < S.n_regions; ++g) {
                float t;
                if (analytic_root(S.regions[g], r, t) && t < h.t) { h.t = t; h.region = g; h.element = 0; h.prim = -1; }
            }
            pool.hit[i] = make_float4(h.t, h.u, h.v, 0.f);
            pool.hit_i[i] = make_int4(h.region, h.element, h.prim, 0);
            if (buckets > 1) pool.sort_key[i] = (unsigned char)shade_key(S, h.region, pool.st[i].y, buckets);
            active = false;
        }
    }
}

template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256, PTR_TRACE_MIN_BLOCKS) k_closest(DevScene S0, PathPool pool, int in, BatchTables bt) {
    const int buckets = pool.sort_buckets;
    unsigned n = pool.cnt[in];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        pool.cnt[in ^ 1] = 0u;
        pool.cnt[2] = 0u;
        pool.cnt[4] = 0u;
        pool.stats[0] += n;
        if (pool.fetch) { pool.fetch[1] = 0u; pool.fetch[2] = 0u; pool.fetch[3] = 0u; }
    }
    const int* q = closest_queue(pool, in);
    Work w{0u, 0u, 0u, 0u};
    if (PTR_REFILL && !BATCH && pool.fetch && S0.flat_region >= 0 && inst_mesh_flat_ok(S0, S0.batches[S0.regions[S0.flat_region].ref])) {
        closest_refill<COUNT>(S0, pool, q, n, buckets, pool.fetch + 0, &w);
        if (COUNT) flush_work(S0, w);
        return;
    }
    const WaveJobs wj = BATCH ? WaveJobs(pool, bt) : WaveJobs{};
    // the adjoint's hit log: this launch's slice, when its iteration is logged
    float4* log = (!BATCH && pool.hit_log && pool.iter < pool.hit_log_iters)
                      ? pool.hit_log + 4 * (size_t)pool.iter * (size_t)pool.hit_log_stride : nullptr;
    QueueCursor cur(n, pool.fetch ? pool.fetch + 0 : nullptr);
    unsigned k;
    while (cur.next(k)) {
        if (k >= n) continue;
        int i = q[k];
        const DevScene& S = BATCH ? bt.scenes[wj.of(bt, i)] : S0;
        float4 hf;
        int4 hi;
        if (log && pool.hit_log_mode == 2) {   // the replay: the forward walk's hit of this path
            hf = log[4 * (size_t)i];
            hi = float4_as_int4(log[4 * (size_t)i + 1]);
        } else {
            Ray r;
            r.o = xyz(pool.ray_o[i]);
            r.d = xyz(pool.ray_d[i]);
            HitRec h = scene_closest(S, r, COUNT ? &w : nullptr);
            hf = make_float4(h.t, h.u, h.v, 0.f);
            hi = make_int4(h.region, h.element, h.prim, 0);
            if (log && pool.hit_log_mode == 1) {
                log[4 * (size_t)i] = hf;
                log[4 * (size_t)i + 1] = int4_as_float4(hi);
            }
        }
        pool.hit[i] = hf;
        pool.hit_i[i] = hi;
        if (buckets > 1) pool.sort_key[i] = (unsigned char)shade_key(S, hi.x, pool.st[i].y, buckets);
    }
    if (COUNT) flush_work(S0, w);
}

// Counting sort of a device-counted queue by 1-byte keys (< kMaxKeys), in three launches
// on fixed grids: per-chunk key counts, one scan into per-(key, chunk) offsets, and a
// scatter that reserves slots from shared-memory offsets.  Each of kSortChunks blocks owns
// one contiguous chunk of the queue (a multiple of kSortVec entries), so global traffic is
// the keys twice, the source once and the destination once, and no global atomics are
// taken.  Each thread reads kSortVec consecutive keys with one 16-byte load (and their
// sources with four), and lanes with equal keys find each other with seven ballots (a
// warp multi-split).  The consumers are order-independent; the order within a key only
// matters for their memory coalescing.
// GATHER: the keys are indexed by path (keys[src[k]]) rather than by queue position.
// Queues shorter than kSortMin are not sorted: every consumer reads the unsorted queue
// then (sorted_queue), deciding from the same device count as the sort kernels.
constexpr int kSortChunks = 512;
constexpr int kMaxKeys = 64;
constexpr int kSortThreads = 256;
constexpr int kSortVec = 16;
constexpr int kSortScanThreads = 1024;
constexpr int kSortEntries = kMaxKeys * kSortChunks;
constexpr int kSortScanPer = kSortEntries / kSortScanThreads;   // 32: one padded smem row per thread
static_assert(kSortScanPer == 32, "the scan's padded layout assumes 32 entries per thread");
constexpr size_t kSortScanSmem = (size_t)(kSortEntries + kSortEntries / 32) * sizeof(unsigned);
constexpr unsigned kSortMin = 65536u;
constexpr unsigned kNoKey = (unsigned)kMaxKeys;   // 7-bit key of an idle lane
__device__ __forceinline__ const int* sorted_queue(const int* sorted, const int* plain, unsigned n) {
    return n >= kSortMin ? sorted : plain;
}
__device__ __forceinline__ void sort_chunk(unsigned n, unsigned& lo, unsigned& hi) {
    unsigned chunk = (n + kSortChunks - 1) / kSortChunks;
    chunk = (chunk + kSortVec - 1) & ~(unsigned)(kSortVec - 1);
    lo = min(n, blockIdx.x * chunk);
    hi = min(n, lo + chunk);
}
// Lanes of the warp whose 7-bit key equals this lane's (all lanes take part).
__device__ __forceinline__ unsigned warp_peers(unsigned key) {
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const unsigned m = __ballot_sync(0xffffffffu, (key >> b) & 1u);
        peers &= ((key >> b) & 1u) ? m : ~m;
    }
    return peers;
}
// Keys (and, if asked or gathering, sources) of entries [base, base + kSortVec) below hi;
// base is a multiple of kSortVec, so the full-width loads are 16-byte aligned.
template <bool GATHER>
__device__ __forceinline__ void sort_load(const int* src, const unsigned char* keys, unsigned base, unsigned hi,
                                          unsigned (&key)[kSortVec], int (&val)[kSortVec], bool want_val) {
    if (base + kSortVec <= hi) {
        if (GATHER || want_val) {
#pragma unroll
            for (int v = 0; v < kSortVec / 4; ++v) {
                const int4 x = *reinterpret_cast<const int4*>(src + base + 4 * v);
                val[4 * v] = x.x; val[4 * v + 1] = x.y; val[4 * v + 2] = x.z; val[4 * v + 3] = x.w;
            }
        }
        if (GATHER) {
#pragma unroll
            for (int j = 0; j < kSortVec; ++j) key[j] = keys[(unsigned)val[j]];
        } else {
            const uint4 x = *reinterpret_cast<const uint4*>(keys + base);
            const unsigned w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int j = 0; j < kSortVec; ++j) key[j] = (w[j >> 2] >> (8 * (j & 3))) & 0xffu;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kSortVec; ++j) {
            const unsigned k = base + j;
            const bool v = k < hi;
            val[j] = (v && (GATHER || want_val)) ? src[k] : 0;
            key[j] = v ? (unsigned)keys[GATHER ? (unsigned)val[j] : k] : kNoKey;
        }
    }
}
// Counts of every key (all kMaxKeys rows are written, unused ones zero).
template <bool GATHER>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const int* src, const unsigned char* keys, const unsigned* count, unsigned* hist) {
    const unsigned n = *count;
    if (n < kSortMin) return;
    __shared__ unsigned h[kMaxKeys];
    if (threadIdx.x < kMaxKeys) h[threadIdx.x] = 0u;
    __syncthreads();
    unsigned lo, hi;
    sort_chunk(n, lo, hi);
    for (unsigned k0 = lo; k0 < hi; k0 += kSortThreads * kSortVec) {   // block-uniform trip count
        unsigned key[kSortVec];
        int val[kSortVec];
        sort_load<GATHER>(src, keys, k0 + threadIdx.x * kSortVec, hi, key, val, false);
#pragma unroll
        for (int j = 0; j < kSortVec; ++j) {
            const unsigned peers = warp_peers(key[j]);
            if (key[j] != kNoKey && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[key[j]], (unsigned)__popc(peers));
        }
    }
    __syncthreads();
    if (threadIdx.x < kMaxKeys) hist[threadIdx.x * kSortChunks + blockIdx.x] = h[threadIdx.x];
}
// Exclusive scan, in place, of the key-major [kMaxKeys][kSortChunks] counts: one block
// stages them in shared memory with coalesced loads (one padding word per 32 entries, so
// the per-thread rows below are bank-conflict free), scans, and writes them back.
__global__ void __launch_bounds__(kSortScanThreads) k_sort_scan(const unsigned* count, unsigned* hist) {
    if (*count < kSortMin) return;
    extern __shared__ unsigned sm[];
    __shared__ unsigned warp_sum[kSortScanThreads / 32];
    for (int e = threadIdx.x; e < kSortEntries; e += kSortScanThreads) sm[e + (e >> 5)] = hist[e];
    __syncthreads();
    const int row = threadIdx.x * (kSortScanPer + 1);   // entries [32 t, 32 t + 32) of the padded layout
    unsigned s = 0u;
#pragma unroll
    for (int j = 0; j < kSortScanPer; ++j) s += sm[row + j];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned w = warp_sum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sum[lane] = w;
    }
    __syncthreads();
    unsigned run = incl - s + (warp ? warp_sum[warp - 1] : 0u);
#pragma unroll
    for (int j = 0; j < kSortScanPer; ++j) {
        const unsigned c = sm[row + j];
        sm[row + j] = run;
        run += c;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kSortEntries; e += kSortScanThreads) hist[e] = sm[e + (e >> 5)];
}
// The scatter stages each warp's 32 * kSortVec entries in shared memory (16-byte loads),
// then places them in rounds of 32 consecutive entries: peers of one round land in one
// contiguous run, so a sorted queue keeps the compaction's ascending path order within
// its runs (the pool's SoA reads of its consumers stay coalesced).
template <bool GATHER>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const int* src, const unsigned char* keys, const unsigned* count,
                                                               const unsigned* offsets, int* dst) {
    const unsigned n = *count;
    if (n < kSortMin) return;
    constexpr int kSpan = 32 * kSortVec;   // entries one warp stages per round
    __shared__ unsigned base[kMaxKeys];
    __shared__ __align__(16) int s_val[kSortThreads / 32][kSpan];
    __shared__ __align__(16) unsigned char s_key[kSortThreads / 32][kSpan];
    if (threadIdx.x < kMaxKeys) base[threadIdx.x] = offsets[threadIdx.x * kSortChunks + blockIdx.x];
    __syncthreads();
    unsigned lo, hi;
    sort_chunk(n, lo, hi);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* sv = s_val[warp];
    unsigned char* sk = s_key[warp];
    for (unsigned k0 = lo; k0 < hi; k0 += kSortThreads * kSortVec) {   // block-uniform trip count
        const unsigned ws = k0 + warp * kSpan;
        const unsigned b = ws + lane * kSortVec;
        if (b + kSortVec <= hi) {
#pragma unroll
            for (int v = 0; v < kSortVec / 4; ++v)
                *reinterpret_cast<int4*>(sv + lane * kSortVec + 4 * v) = *reinterpret_cast<const int4*>(src + b + 4 * v);
            if (!GATHER) *reinterpret_cast<uint4*>(sk + lane * kSortVec) = *reinterpret_cast<const uint4*>(keys + b);
        } else {
            for (int j = 0; j < kSortVec; ++j) {
                if (b + j < hi) {
                    sv[lane * kSortVec + j] = src[b + j];
                    if (!GATHER) sk[lane * kSortVec + j] = keys[b + j];
                }
            }
        }
        __syncwarp();
#pragma unroll 4
        for (int j = 0; j < kSortVec; ++j) {
            const int e = j * 32 + lane;
            const bool valid = ws + e < hi;
            const int val = valid ? sv[e] : 0;
            const unsigned key = valid ? (unsigned)(GATHER ? keys[(unsigned)val] : sk[e]) : kNoKey;
            const unsigned peers = warp_peers(key);
            const int leader = __ffs(peers) - 1;
            unsigned o = 0u;
            if (valid && lane == leader) o = atomicAdd(&base[key], (unsigned)__popc(peers));
            o = __shfl_sync(0xffffffffu, o, leader);
            if (valid) dst[o + __popc(peers & lanemask_lt())] = val;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ const int* closest_queue(const PathPool& pool, int in) {
    return pool.ray_in ? sorted_queue(pool.q_ray, pool.q[in], pool.cnt[in]) : pool.q[in];
}

// One walk iteration for every live path.
#ifndef PTR_SHADE_MIN_BLOCKS
#define PTR_SHADE_MIN_BLOCKS 3
#endif
// ADJ: the replay pass of the adjoint — the same walk on the same random numbers, which
// also scatters d Loss / d theta into per-block float64 accumulators (dynamic shared
// memory: PTR_GRAD_SLOTS doubles per material).
// Col: f3 (RGB) or s4 (spectral, four wavelength lanes; the adjoint is RGB only).
template <class Col, int DIRECT, bool MEDIA, bool BATCH, bool ADJ = false>
__global__ void __launch_bounds__(256, PTR_SHADE_MIN_BLOCKS) k_shade(DevScene S0, PathPool pool, ProgParams P0, int in, BatchTables bt,
                                                                     AdjParams adj = AdjParams{}) {
    constexpr bool SPECTRAL = sizeof(Col) == sizeof(s4);
    static_assert(!(ADJ && SPECTRAL), "the adjoint replay is RGB only");
    using CM = Colors<Col>;
    extern __shared__ double s_grad[];
    if constexpr (ADJ) grad_block_init(s_grad, PTR_GRAD_SLOTS * S0.n_materials);
    const unsigned n = pool.cnt[in];
    // the compacted queue, not the ray-coherence one: compaction keeps path indices nearly
    // ascending, so the pool's SoA reads and writes stay coalesced
    const int* q = pool.sort_buckets > 1 ? sorted_queue(pool.q_sorted, pool.q[in], n) : pool.q[in];
    int* qout = pool.q[in ^ 1];
    const bool nee = DIRECT != PTR_DIRECT_NONE;
    const bool mis = DIRECT == PTR_DIRECT_MIS;
    if (blockIdx.x == 0 && threadIdx.x == 0 && pool.fetch) pool.fetch[0] = 0u;   // the next k_closest's ticket
    const WaveJobs wj = BATCH ? WaveJobs(pool, bt) : WaveJobs{};
    QueueCursor cur(n, pool.fetch ? pool.fetch + 3 : nullptr);
    unsigned k;
    while (cur.next(k)) {
        bool alive = false, shadow = false, shadow2 = false;
        int i = -1;
        unsigned rk = 0u, sk = 0u;   // ray-coherence keys of the spawned ray / shadow query
        if (k < n) {
            i = q[k];
            const int job = BATCH ? wj.of(bt, i) : 0;
            const DevScene& S = BATCH ? bt.scenes[job] : S0;
            const ProgParams& P = BATCH ? bt.progs[job] : P0;
            float4 ro = pool.ray_o[i], rd = pool.ray_d[i];
            Ray r;
            r.o = xyz(ro);
            r.d = xyz(rd);
            float prev_bsdf_pdf = ro.w;
            float eta_scale = rd.w;
            Col thr = col_ld<Col>(pool.thr[i]);
            Col rad = col_ld<Col>(pool.rad[i]);
            f3 prev_qp = xyz(pool.prev_q[i]);
            Wl wl;
            const bool tree = PTR_SPEC_TREE && P.light_tree;
            if constexpr (SPECTRAL) wl.lambda = pool.wl[i];
            int4 st = pool.st[i];
            int bounce = st.x, cur_med = st.y, nulls = st.z;
            bool prev_delta = st.w != 0;
            uint2 rs = pool.rng[i];
            Rng rng;
            rng.base = rs.x;
            rng.dim = rs.y;
            Col lrem(0.0f);
            GradAcc ga;
            int sh_mat = 0;
            // the NEE query's lobe derivative: dlog f toward the light (per channel) and its
            // scalar part (GGX alpha beside the per-channel F0 part)
            NeeGrad sg{kGradKindNone, f3(0.0f), 0.0f};
            if constexpr (ADJ) {
                lrem = xyz(pool.l_rem[i]);
                ga.s = s_grad;
                ga.dl = xyz(pool.dl[i]);
            }
            float4 hf = pool.hit[i];
            int4 hi = pool.hit_i[i];
            HitRec hr;
            hr.t = hf.x; hr.u = hf.y; hr.v = hf.z;
            hr.region = hi.x; hr.element = hi.y; hr.prim = hi.z;
            const bool boundary = hr.region >= 0;
            const int N = P.max_bounces;
            Hit hit;
            if (boundary) fill_hit(S, r, hr, hit);
            bool done = false, handled = false;

            // -- the volumetric call site: one segment (features/materials.ts:675-746)
            if (MEDIA) {
                int med_mat = material_of(S, cur_med);
                if (mat_has_medium(S, med_mat)) {
                    const ptr_material& mm = S.materials[med_mat];
                    // the per-segment equiangular site precedes the transmittance sample
                    // (pt.ts:322-328) and rides the second shadow slot
                    if (P.equiangular && bounce < N) {
                        EquiangularQuery<Col> eq;
                        if (equiangular_site<Col>(S, med_mat, r, boundary ? hr.t : kMaxDist, rng, thr, wl, eq)) {
                            pool.sh2_o[i] = f4(eq.p_evt, 0.0f);
                            pool.sh2_d[i] = f4(eq.wi, __int_as_float(P.max_null - nulls));
                            pool.sh2_lp[i] = f4(eq.light_pos, 1.0f);
                            pool.sh2_c[i] = col_st(eq.contrib, eq.denom);
                            if constexpr (SPECTRAL) pool.sh2_pdf[i] = eq.denom;
                            shadow2 = true;
                        }
                    }
                    float x0 = rng.next();
                    float x1 = rng.next();
                    float t_max = boundary ? hr.t : kMaxDist;
                    // heterogeneous media take the tracking arms (delta_tracking.glsl)
                    const bool het = !SPECTRAL && S.has_het && mat_is_het(mm);
                    if (!scatter_live(S, P, med_mat) && !het) {
                        thr = thr * vexp(-CM::sigma_a(S, med_mat, wl) * t_max);
                        if constexpr (ADJ) {   // w = exp(-(1-a) st t)
                            GreyMedium gm = grey_medium(mm);
                            ga.scl(med_mat, PTR_GRAD_SIGMA_T, lrem, -(1.0f - gm.a) * t_max);
                            ga.scl(med_mat, PTR_GRAD_MEDIUM_ALBEDO, lrem, gm.st * t_max);
                        }
                    } else {
                        MediumSample<Col> ms;
                        if constexpr (!SPECTRAL) {
                            if (het && scatter_live(S, P, med_mat)) {
                                ms = medium_sample_delta(S, mm, r, t_max, x0, x1, rng);
                            } else if (het) {   // absorbing only: the ratio-tracked pass-through
                                ms.scattered = false;
                                ms.weight = medium_ratio_track(S, mm, r, t_max, rng, false);
                            } else {
                                ms = medium_sample_analytic<Col>(CM::sigma_a(S, med_mat, wl), CM::sigma_s(S, med_mat, wl),
                                                                 r, t_max, x0, x1);
                            }
                        } else {
                            ms = medium_sample_analytic<Col>(CM::sigma_a(S, med_mat, wl), CM::sigma_s(S, med_mat, wl),
                                                             r, t_max, x0, x1);
                        }
                        thr = thr * ms.weight;
                        if constexpr (ADJ) {   // scattered at t: w = a st exp(-st t)/pdf; passed: exp(-st t_max)/P
                            GreyMedium gm = grey_medium(mm);
                            if (ms.scattered) {
                                float t_evt = dot(ms.exit_p - r.o, r.d);
                                ga.scl(med_mat, PTR_GRAD_SIGMA_T, lrem, 1.0f / gm.st - t_evt);
                                ga.scl(med_mat, PTR_GRAD_MEDIUM_ALBEDO, lrem, 1.0f / gm.a);
                            } else {
                                ga.scl(med_mat, PTR_GRAD_SIGMA_T, lrem, -t_max);
                            }
                        }
                        if (ms.scattered) {
                            handled = true;
                            if (bounce == N) {
                                done = true;
                            } else {
                                f3 p_evt = ms.exit_p;
                                f3 wo_med = -ms.exit_dir;
                                if (nee && !P.equiangular) {   // light_sample_direct_medium (light_medium.glsl:7-18)
                                    float y0 = rng.next();
                                    float y1 = rng.next();
                                    LightQuery lq{p_evt, f3(0.0f), false};   // no orientation at a medium event
                                    LightSample<Col> ls = lighting_sample<Col>(S, lq, y0, y1, rng, tree, wl);
                                    if (S.has_het) pool.sh_seed[i] = rng.dim;
                                    if (ls.pdf > 0.0f) {
                                        f3 light_p = p_evt + ls.wi * ls.distance;
                                        float ph = hg_eval(ls.wi, wo_med, mm.phase_g);
                                        float w = 1.0f;
                                        if (mis && !(ls.flags & kLightDelta)) w = power_heuristic(ls.pdf, spectrum_average(Col(ph)));
                                        pool.sh_o[i] = f4(p_evt, 0.0f);
                                        pool.sh_d[i] = f4(ls.wi, __int_as_float(P.max_null - nulls));
                                        pool.sh_lp[i] = f4(light_p, w);
                                        pool.sh_c[i] = col_st(thr * ls.radiance * Col(ph), ls.pdf);
                                        if constexpr (SPECTRAL) pool.sh_pdf[i] = ls.pdf;
                                        shadow = true;
                                        if constexpr (ADJ) {
                                            sg.kind = kGradKindPhase;
                                            sh_mat = med_mat;
                                            sg.dnee = f3(hg_dlog_g(ls.wi, wo_med, mm.phase_g), 0.0f, 0.0f);
                                        }
                                    }
                                }
                                float z0 = rng.next();
                                float z1 = rng.next();
                                ISample<Col> ps = hg_sample<Col>(wo_med, mm.phase_g, z0, z1);
                                thr = thr * ps.weight;
                                if constexpr (ADJ) {   // phase continuation: w = p_HG / pdf_detached
                                    float dg = hg_dlog_g(ps.wi, wo_med, mm.phase_g);
                                    ga.scl(med_mat, PTR_GRAD_HG_G, lrem, dg);
                                    if (shadow) sg.dnee.x -= dg;
                                }
                                prev_delta = false;
                                prev_bsdf_pdf = ps.pdf;
                                prev_qp = p_evt;
                                if (tree) pool.prev_n[i] = make_float4(0.f, 0.f, 0.f, 0.f);   // no orientation
                                r.o = p_evt;
                                r.d = ps.wi;
                                // roulette_interior (pt.ts:230-283); nothing is owed after a
                                // tracking arm, whose lottery settled absorption already
                                bool survive = true;
                                if (P.rr_start >= 0 && bounce >= P.rr_start && !het) {
                                    Col ss = CM::sigma_s(S, med_mat, wl), sa = CM::sigma_a(S, med_mat, wl);
                                    Col surv = ss / vmax(ss + sa, Col(1e-9f));
                                    float p_survive = spectrum_max(surv);
                                    if (p_survive <= 0.0f) survive = false;
                                    else if (rng.next() > p_survive) survive = false;
                                    else thr = thr / p_survive;
                                }
                                if (survive) { bounce += 1; alive = true; }
                                else done = true;
                            }
                        }
                    }
                }
            }
            if (!handled) {
                if (!boundary) {   // kernel_score_miss (kernel.glsl:11-14)
                    float w = 1.0f;
                    if (nee && S.env_samplable && !prev_delta) {
                        if (!mis) w = 0.0f;
                        else {
                            float pe = S.env_select_live ? S.env_select_prob : 1.0f;
                            w = power_heuristic(prev_bsdf_pdf, pe * env_pdf(S, r.d));
                        }
                    }
                    Col e = thr * w * env_radiance<Col>(S, r.d, wl);
                    rad = rad + e;
                    if constexpr (ADJ) lrem = lrem - e;
                    done = true;
                } else {
                    if (MEDIA && hit.region_from != cur_med) cur_med = hit.region_from;
                    int mat = material_of(S, hit.region_owner);
                    const ptr_material& m = S.materials[mat];
                    if (MEDIA && m.model == PTR_MAT_NONE) {   // null pass-through (pt.ts:404-417)
                        cur_med = hit.region_to;
                        Ray nr = ray_spawn(hit, r.d);
                        r = nr;
                        nulls += 1;
                        if (nulls > P.max_null) done = true;
                        else alive = true;
                    } else {
                        f3 wo = -r.d;
                        // the AOV capture (pt.ts:422-433): the first non-null surface before
                        // any event, weighted by the arrival throughput
                        if constexpr (!SPECTRAL) {
                            if (bounce == 0 && pool.aov) {
                                f3 fact = ld3(m.transmittance);
                                auto aov = [&](auto M) { fact = decltype(M)::aov(m); };
                                dispatch_material<MatPresent>(m.model, aov);
                                fact = vmin(vmax(fact, f3(0.0f)), f3(1.0f));
                                f3 nf = dot(hit.frame.n, wo) < 0.0f ? -hit.frame.n : hit.frame.n;
                                pool.aov[2 * i] = f4(fact * thr, 0.0f);
                                pool.aov[2 * i + 1] = f4(nf * spectrum_average(thr), 0.0f);
                            }
                        }
                        // kernel_score_emitter_hit (kernel.glsl:16-25; combiner.ts:27-46)
                        int mat_emit = material_of(S, hit.region_to);
                        if (mat_emit >= 0 && (S.materials[mat_emit].flags & PTR_MATF_EMISSIVE)) {
                            float w = 1.0f;
                            if (nee) {
                                int lid = hit.region_to >= 0 ? emitter_light(S, hit) : -1;
                                if (lid >= 0 && !prev_delta) {
                                    if (!mis) w = 0.0f;
                                    else {
                                        // the stored selection context (its normal and sidedness
                                        // only under light-tree selection)
                                        LightQuery pq{prev_qp, f3(0.0f), false};
                                        if (tree) {
                                            float4 pqn = pool.prev_n[i];
                                            pq.n = xyz(pqn);
                                            pq.two_sided = pqn.w != 0.0f;
                                        }
                                        w = power_heuristic(prev_bsdf_pdf, lighting_pdf(S, pq, r.d, lid, hit.p, hit.ng, tree));
                                    }
                                }
                            }
                            Col e = thr * w * CM::emission(S, mat_emit, wl);
                            rad = rad + e;
                            if constexpr (ADJ) lrem = lrem - e;
                        }
                        if (bounce == N) {
                            done = true;
                        } else {
                            const float alpha = hit.alpha >= 0.0f ? hit.alpha : m.alpha;
                            // light queries with sphere support (a transmissive non-delta lobe)
                            const bool rough = material_in<MatSphereQuery>(m.model);
                            const bool nondelta = material_in<MatNonDelta>(m.model);
                            const float n_from = ior_of(S, hit.region_from), n_to = ior_of(S, hit.region_to);
                            const MatSite<Col> site{S, mat, m, hit, wl, alpha, n_from, n_to};
                            // light_sample_direct (light.glsl:8-28)
                            if (nee && nondelta) {
                                float y0 = rng.next();
                                float y1 = rng.next();
                                LightQuery lq{hit.p, hit.frame.n, rough};   // rough glass: sphere support
                                LightSample<Col> ls = lighting_sample<Col>(S, lq, y0, y1, rng, tree, wl);
                                if (MEDIA && S.has_het) pool.sh_seed[i] = rng.dim;
                                if (ls.pdf > 0.0f) {
                                    f3 light_p = hit.p + ls.wi * ls.distance;
                                    Ray sr = ray_spawn(hit, ls.wi);
                                    sr.d = normalize(light_p - sr.o);
                                    Col f(0.0f);
                                    float bp = 0.0f;
                                    const bool want_pdf = mis && !(ls.flags & kLightDelta);
                                    auto lobe = [&](auto M) {
                                        f = decltype(M)::eval(site, ls.wi, wo);
                                        if (want_pdf) bp = decltype(M)::pdf(site, ls.wi, wo);
                                    };
                                    dispatch_material<MatNonDelta, true>(m.model, lobe);   // nondelta holds here
                                    float cos_i = fabsf(dot(ls.wi, hit.frame.n));
                                    float w = 1.0f;
                                    if (want_pdf) w = power_heuristic(ls.pdf, bp);
                                    float maxd = length(light_p - sr.o) - kShadowBackoff;
                                    pool.sh_o[i] = f4(sr.o, maxd);
                                    pool.sh_d[i] = f4(sr.d, __int_as_float(P.max_null - nulls));
                                    pool.sh_lp[i] = f4(light_p, w);
                                    pool.sh_c[i] = col_st(thr * ls.radiance * f * cos_i, ls.pdf);
                                    if constexpr (SPECTRAL) pool.sh_pdf[i] = ls.pdf;
                                    shadow = true;
                                    if constexpr (ADJ) {
                                        sh_mat = mat;
                                        auto ng = [&](auto M) { decltype(M)::nee_grad(site, ls.wi, wo, sg); };
                                        dispatch_material<MatNonDelta, true>(m.model, ng);
                                    }
                                }
                            }
                            // kernel_sample_continuation (kernel.glsl:27-34)
                            float uc = rng.next();
                            float u0 = rng.next();
                            float u1 = rng.next();
                            ISample<Col> bs;
                            bs.weight = Col(0.0f);   // stays black only in a build without the scene's models
                            auto cont = [&](auto M) { bs = decltype(M)::sample(site, wo, uc, u0, u1); };
                            dispatch_material<MatPresent>(m.model, cont);
                            if (spectrum_is_black(bs.weight)) {
                                done = true;
                            } else {
                                thr = thr * bs.weight;
                                if constexpr (ADJ) {   // the continuation lobe: d log w_cont
                                    auto cg = [&](auto M) { decltype(M)::cont_grad(site, bs, wo, ga, lrem, shadow, sg); };
                                    dispatch_material<MatPresent>(m.model, cg);
                                }
                                prev_delta = (bs.flags & kLobeDelta) != 0u;
                                prev_bsdf_pdf = bs.pdf;
                                prev_qp = hit.p;
                                if (tree) pool.prev_n[i] = f4(hit.frame.n, rough ? 1.0f : 0.0f);
                                if (bs.flags & kLobeTransmission) {
                                    if (MEDIA) cur_med = hit.region_to;
                                    float rr = ior_of(S, hit.region_to) / ior_of(S, hit.region_from);
                                    eta_scale *= rr * rr;
                                }
                                // roulette (pt.ts:204-222)
                                bool survive = true;
                                if (P.rr_start >= 0 && bounce >= P.rr_start) {
                                    float p_survive = gmin(P.rr_max_survival, spectrum_max(thr) * eta_scale);
                                    if (p_survive <= 0.0f) survive = false;
                                    else if (rng.next() > p_survive) survive = false;
                                    else thr = thr / p_survive;
                                }
                                if (survive) {
                                    r = ray_spawn(hit, bs.wi);
                                    bounce += 1;
                                    alive = true;
                                } else {
                                    done = true;
                                }
                            }
                        }
                    }
                }
            }
            (void)done;
            if (pool.ray_sort) {
                if (alive) rk = ray_key(S, r.o, r.d);
                if (shadow) {
                    float4 so = pool.sh_o[i], sd = pool.sh_d[i];
                    sk = ray_key(S, xyz(so), xyz(sd));
                }
            }
            pool.rad[i] = col_st(rad, 0.0f);
            pool.thr[i] = col_st(thr, 0.0f);   // with rad: the whole record, for a dying path too
            if constexpr (ADJ) {
                pool.l_rem[i] = f4(lrem, 0.0f);
                if (shadow) {
                    pool.sh_g[i] = f4(sg.dnee, sg.dw);
                    pool.sh_gm[i] = sh_mat | (sg.kind << 16);
                }
            }
            if (alive) {
                pool.ray_o[i] = f4(r.o, prev_bsdf_pdf);
                pool.ray_d[i] = f4(r.d, eta_scale);
                pool.prev_q[i] = f4(prev_qp, 0.0f);
                pool.st[i] = make_int4(bounce, cur_med, nulls, prev_delta ? 1 : 0);
                pool.rng[i] = make_uint2(rng.base, rng.dim);
            }
        }
        int slot = warp_append(&pool.cnt[in ^ 1], alive);
        if (alive) qout[slot] = i;
        int sslot = warp_append(&pool.cnt[2], shadow);
        if (shadow) pool.shq[sslot] = i;
        if (pool.ray_sort) {
            if (alive) pool.rkey[slot] = (unsigned char)rk;
            if (shadow) pool.skey[sslot] = (unsigned char)sk;
        }
        if (MEDIA) {
            int s2 = warp_append(&pool.cnt[4], shadow2);
            if (shadow2) pool.shq2[s2] = i;
        }
    }
    if constexpr (ADJ) grad_block_flush(s_grad, PTR_GRAD_SLOTS * S0.n_materials, adj.grads);
}

// Shadow queries: opaque visibility (shadow/opaque/opaque.glsl:16-19) or the media
// segment walker (shadow/media/media.glsl:29-62); the surviving fraction scales the
// stored contribution prefix into the path's radiance.
// slot 1 reads the second shadow slot (the equiangular segment queries); its launch
// precedes the slot-0 launch of the same iteration, so the two never add to one path's
// radiance concurrently.
// ADJ: the replay pass also folds the query's gradient terms — the lobe derivative D of
// its vertex and d log T / d theta of every medium segment the shadow ray crossed.
constexpr int kAdjMaxMedia = 4;            // distinct media one adjoint shadow query may cross
constexpr unsigned kErrAdjMedia = 8u;      // ... more were crossed (their terms were dropped)
// Opaque shadow queries over the same scene form, with the same per-lane refill: the
// regions before the instanced one, the flat any-hit walk, then the regions after it (the
// order of scene_any); an unoccluded query adds its stored contribution as k_shadow does.
template <class Col, bool COUNT>
__device__ __forceinline__ void shadow_refill(const DevScene& S, const PathPool& pool, const int* shq, unsigned n, int slot,
                                              const Pair<float4> a_o, const Pair<float4> a_d, const Pair<float4> a_lp,
                                              const Pair<float4> a_c, unsigned* ticket, Work* w) {
    constexpr bool SPECTRAL = sizeof(Col) == sizeof(s4);
    const int fr = S.flat_region;
    const DevBatch& b = S.batches[S.regions[fr].ref];
    const DevMesh& m = S.meshes[b.proto_mesh];
    const unsigned lane = threadIdx.x & 31u;
    InstFlat f;
    Ray r;
    HitRec unused;
    float max_dist = 0.0f;
    int i = -1, steps = 0;
    bool active = false, exhausted = false;
    for (;;) {
        if (!exhausted) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (__popc(need) >= kRefillMin) {
                const int leader = __ffs(need) - 1;
                unsigned base = 0u;
                if ((int)lane == leader) base = atomicAdd(ticket, (unsigned)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (unsigned)__popc(need) >= n) exhausted = true;
                if (!active) {
                    const unsigned k = base + __popc(need & lanemask_lt());
                    if (k < n) {
                        i = shq[k];
                        const float4 so = a_o[i], sd = a_d[i];
                        r.o = xyz(so);
                        r.d = xyz(sd);
                        max_dist = so.w;
                        bool blocked = false;
                        for (int g = 0; g < fr && !blocked; ++g) {
                            float t;
                            blocked = analytic_root(S.regions[g], r, t) && t < max_dist;
                        }
                        if (!blocked) {            // an occluded query is finished: nothing to add
                            f.init(r, max_dist);
                            steps = 0;
                            active = true;
                        }
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (!active) continue;
        bool more = f.step<true>(S, b, m, fr, r, unused, max_dist, COUNT ? w : nullptr);
        if (more && ++steps >= kFlatGuard) {
            flag_error(S, kErrCwGuard);
            more = false;
        }
        if (!more) {
            bool blocked = f.found;
            for (int g = fr + 1; g < S.n_regions && !blocked; ++g) {
                float t;
                blocked = analytic_root(S.regions[g], r, t) && t < max_dist;
            }
            if (!blocked) {
                const float4 c = a_c[i];
                const Col cc = col_ld<Col>(c);
                float cpdf = c.w;
                if constexpr (SPECTRAL) cpdf = slot ? pool.sh2_pdf[i] : pool.sh_pdf[i];
                const Col vis(1.0f);
                const Col add = cc * vis * a_lp[i].w / cpdf;
                pool.rad[i] = col_st(col_ld<Col>(pool.rad[i]) + add, 0.0f);
            }
            active = false;
        }
    }
}

template <class Col, bool MEDIA, bool COUNT, bool BATCH, bool ADJ = false>
__global__ void __launch_bounds__(256, PTR_TRACE_MIN_BLOCKS) k_shadow(DevScene S0, PathPool pool, ProgParams P0, BatchTables bt,
                                                                      int slot, AdjParams adj = AdjParams{}) {
    constexpr bool SPECTRAL = sizeof(Col) == sizeof(s4);
    static_assert(!(ADJ && SPECTRAL), "the adjoint replay is RGB only");
    extern __shared__ double s_grad[];
    if constexpr (ADJ) grad_block_init(s_grad, PTR_GRAD_SLOTS * S0.n_materials);
    const unsigned n = pool.cnt[slot ? 4 : 2];
    if (blockIdx.x == 0 && threadIdx.x == 0) pool.stats[1] += n;
    const int* shq = slot ? pool.shq2 : (pool.ray_sort ? sorted_queue(pool.shq_s, pool.shq, n) : pool.shq);
    const Pair<float4> a_o = slot ? pool.sh2_o : pool.sh_o;
    const Pair<float4> a_d = slot ? pool.sh2_d : pool.sh_d;
    const Pair<float4> a_lp = slot ? pool.sh2_lp : pool.sh_lp;
    const Pair<float4> a_c = slot ? pool.sh2_c : pool.sh_c;
    Work wk{0u, 0u, 0u, 0u};
    // the adjoint's walk log: this launch's slot-0 shadow records (two float4 per path after
    // its closest hit: visibility rgb and the media count, then up to two (medium, length)
    // pairs; a count of -1 marks a query the replay walks again)
    float4* slog = nullptr;
    if constexpr (!BATCH && !SPECTRAL)
        if (slot == 0 && pool.hit_log && pool.iter < pool.hit_log_iters)
            slog = pool.hit_log + 4 * (size_t)pool.iter * (size_t)pool.hit_log_stride + 2;
    const bool rec = !ADJ && slog && pool.hit_log_mode == 1;
    const bool rep = ADJ && slog && pool.hit_log_mode == 2;
    if (PTR_REFILL && !MEDIA && !BATCH && !ADJ && !rec && pool.fetch && S0.flat_region >= 0 &&
        inst_mesh_flat_ok(S0, S0.batches[S0.regions[S0.flat_region].ref])) {
        shadow_refill<Col, COUNT>(S0, pool, shq, n, slot, a_o, a_d, a_lp, a_c, pool.fetch + 1 + slot, &wk);
        if (COUNT) flush_work(S0, wk);
        return;
    }
    const WaveJobs wj = BATCH ? WaveJobs(pool, bt) : WaveJobs{};
    QueueCursor cur(n, pool.fetch ? pool.fetch + 1 + slot : nullptr);
    unsigned k;
    while (cur.next(k)) {
        if (k >= n) continue;
        int i = shq[k];
        const int job = BATCH ? wj.of(bt, i) : 0;
        const DevScene& S = BATCH ? bt.scenes[job] : S0;
        const ProgParams& P = BATCH ? bt.progs[job] : P0;
        float4 so = a_o[i], sd = a_d[i], lp = a_lp[i], c = a_c[i];
        Col cc = col_ld<Col>(c);
        float cpdf = c.w;
        Wl wl;
        if constexpr (SPECTRAL) {
            cpdf = slot ? pool.sh2_pdf[i] : pool.sh_pdf[i];
            wl.lambda = pool.wl[i];
        }
        Ray sr;
        sr.o = xyz(so);
        sr.d = xyz(sd);
        Col vis;
        int mm_id[kAdjMaxMedia];
        float mm_len[kAdjMaxMedia];
        int n_mm = 0;
        bool logged = false;
        if constexpr (ADJ) {
            if (rep) {   // the forward walk's visibility and media of this same query
                const float4 a = slog[4 * (size_t)i], b = slog[4 * (size_t)i + 1];
                n_mm = __float_as_int(a.w);
                logged = n_mm >= 0;
                if (logged) {
                    vis = Col(a.x, a.y, a.z);
                    mm_id[0] = __float_as_int(b.x);
                    mm_len[0] = b.y;
                    mm_id[1] = __float_as_int(b.z);
                    mm_len[1] = b.w;
                } else {
                    n_mm = 0;
                }
            }
        }
        if (logged) {
        } else if (!MEDIA) {
            vis = scene_any(S, sr, so.w, COUNT ? &wk : nullptr) ? Col(0.0f) : Col(1.0f);
        } else {
            f3 light_p = xyz(lp);
            int crossings_left = __float_as_int(sd.w);
            Col T(1.0f);
            Rng srng;
            bool srng_live = false;
            int medium = scene_region_at(S, sr.o);
            Ray seg = sr;
            bool finished = false;
            for (int crossed = 0; crossed <= crossings_left; crossed++) {
                float remaining = length(light_p - seg.o) - kShadowBackoff;
                if (remaining <= 0.0f) { finished = true; break; }
                HitRec hr = scene_closest(S, seg, COUNT ? &wk : nullptr);
                bool hit_boundary = hr.region >= 0 && hr.t < remaining;
                float seg_len = hit_boundary ? hr.t : remaining;
                int med_mat = material_of(S, medium);
                if (mat_has_medium(S, med_mat)) {
                    bool het = false;
                    if constexpr (!SPECTRAL) {
                        const ptr_material& smm = S.materials[med_mat];
                        if (S.has_het && mat_is_het(smm)) {   // ratio tracking on the query's own stream
                            het = true;
                            if (!srng_live) { srng = shadow_rng(pool.rng[i].x, pool.sh_seed[i]); srng_live = true; }
                            T = T * medium_ratio_track(S, smm, seg, seg_len, srng, scatter_live(S, P, med_mat));
                        }
                    }
                    if (!het) T = T * medium_transmittance<Col>(S, P, med_mat, seg_len, wl);
                    if (ADJ || rec) {
                        int e = 0;
                        while (e < n_mm && mm_id[e] != med_mat) e++;
                        if (e < n_mm) mm_len[e] += seg_len;
                        else if (n_mm < kAdjMaxMedia) { mm_id[n_mm] = med_mat; mm_len[n_mm] = seg_len; n_mm++; }
                        else if (ADJ) flag_error(S, kErrAdjMedia);   // (a recording walk logs -1 here)
                    }
                }
                if (!hit_boundary) { finished = true; break; }
                // an optical surface blocks the query: decided from the hit region alone,
                // before the hit's frame and its region classification
                const int om = material_of(S, hr.region);
                if (!(om >= 0 && S.materials[om].model == PTR_MAT_NONE)) { T = Col(0.0f); finished = true; break; }
                Hit h;
                fill_hit(S, seg, hr, h);
                medium = h.region_to;
                seg = ray_spawn(h, seg.d);
                seg.d = normalize(light_p - seg.o);
            }
            vis = finished ? T : Col(0.0f);
        }
        if constexpr (!ADJ && !SPECTRAL) {
            if (rec) {
                const bool fits = n_mm <= 2;
                slog[4 * (size_t)i] = make_float4(vis.x, vis.y, vis.z, __int_as_float(fits ? n_mm : -1));
                slog[4 * (size_t)i + 1] = make_float4(__int_as_float(n_mm > 0 ? mm_id[0] : -1), n_mm > 0 ? mm_len[0] : 0.0f,
                                                      __int_as_float(n_mm > 1 ? mm_id[1] : -1), n_mm > 1 ? mm_len[1] : 0.0f);
            }
        }
        if (!spectrum_is_black(vis)) {
            float w = lp.w;
            Col add = cc * vis * w / cpdf;
            pool.rad[i] = col_st(col_ld<Col>(pool.rad[i]) + add, 0.0f);
            if constexpr (ADJ) {
                GradAcc ga;
                ga.s = s_grad;
                ga.dl = xyz(pool.dl[i]);
                float4 lr = pool.l_rem[i];
                pool.l_rem[i] = make_float4(lr.x - add.x, lr.y - add.y, lr.z - add.z, 0.f);
                const int gm = pool.sh_gm[i];
                const int kind = gm >> 16, vmat = gm & 0xFFFF;
                const float4 Dg = pool.sh_g[i];
                const f3 D = xyz(Dg);
                if (kind == kGradKindAlbedo) ga.vec(vmat, PTR_GRAD_COLOR_R, add, D);
                else if (kind == kGradKindGGX) {
                    ga.vec(vmat, PTR_GRAD_COLOR_R, add, D);
                    ga.scl(vmat, PTR_GRAD_ALPHA, add, Dg.w);
                }
                else if (kind == kGradKindPhase) ga.scl(vmat, PTR_GRAD_HG_G, add, D.x);
                for (int e = 0; e < n_mm; ++e) {   // T = exp(-st len) (scattering) or exp(-(1-a) st len)
                    GreyMedium g = grey_medium(S.materials[mm_id[e]]);
                    if (scatter_live(S, P, mm_id[e])) {
                        ga.scl(mm_id[e], PTR_GRAD_SIGMA_T, add, -mm_len[e]);
                    } else {
                        ga.scl(mm_id[e], PTR_GRAD_SIGMA_T, add, -(1.0f - g.a) * mm_len[e]);
                        ga.scl(mm_id[e], PTR_GRAD_MEDIUM_ALBEDO, add, g.st * mm_len[e]);
                    }
                }
            }
        }
    }
    if (COUNT) flush_work(S0, wk);
    if constexpr (ADJ) grad_block_flush(s_grad, PTR_GRAD_SLOTS * S0.n_materials, adj.grads);
}

// Fold the wave's per-path radiance into the film, per pixel in sample order; then
// advance the wave cursor.
// SPECTRAL: each sample's four lanes are projected to linear sRGB first (color_to_pixel).
template <bool SPECTRAL = false>
__global__ void k_film(PathPool pool, const FrameParams* fp, double* sum, double* sumsq, float* samples_out,
                       DevScene S = DevScene{}) {
    const FrameParams F = *fp;
    const long long base = pool.wave[0];
    const long long n = pool.wave[1];
    const long long npix = (long long)F.width * F.height;
    const long long nslot = n < npix ? n : npix;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nslot; j += (long long)gridDim.x * blockDim.x) {
        int pix = (int)((base + j) % npix);
        double s0 = sum[3 * pix + 0], s1 = sum[3 * pix + 1], s2 = sum[3 * pix + 2];
        double q0 = sumsq[3 * pix + 0], q1 = sumsq[3 * pix + 1], q2 = sumsq[3 * pix + 2];
        for (long long i = j; i < n; i += npix) {
            float4 L = pool.rad[i];
            if (SPECTRAL) {
                f3 px = color_to_pixel(S, L, pool.wl[i], pool.wl_pdf[i]);
                L = make_float4(px.x, px.y, px.z, 0.0f);
            }
            s0 += (double)L.x; s1 += (double)L.y; s2 += (double)L.z;
            q0 += (double)L.x * (double)L.x; q1 += (double)L.y * (double)L.y; q2 += (double)L.z * (double)L.z;
            if (samples_out) {
                long long g = base + i;
                samples_out[3 * g + 0] = L.x; samples_out[3 * g + 1] = L.y; samples_out[3 * g + 2] = L.z;
            }
        }
        sum[3 * pix + 0] = s0; sum[3 * pix + 1] = s1; sum[3 * pix + 2] = s2;
        sumsq[3 * pix + 0] = q0; sumsq[3 * pix + 1] = q1; sumsq[3 * pix + 2] = q2;
        if (pool.aov_sum) {   // the first-hit pictures, in the same sample order
            double* as = pool.aov_sum + 3 * (size_t)pix;
            double* ns = pool.aov_sum + 3 * ((size_t)npix + pix);
            double a0 = as[0], a1 = as[1], a2 = as[2], n0 = ns[0], n1 = ns[1], n2 = ns[2];
            for (long long i = j; i < n; i += npix) {
                float4 a = pool.aov[2 * i], b = pool.aov[2 * i + 1];
                a0 += (double)a.x; a1 += (double)a.y; a2 += (double)a.z;
                n0 += (double)b.x; n1 += (double)b.y; n2 += (double)b.z;
            }
            as[0] = a0; as[1] = a1; as[2] = a2;
            ns[0] = n0; ns[1] = n1; ns[2] = n2;
        }
    }
}

// ---- batched renders ------------------------------------------------------------------

// Camera rays for one wave of the concatenated job space.
__global__ void k_generate_batch(PathPool pool, BatchTables bt) {
    long long base = pool.wave[0];
    long long n = bt.total - base;
    if (n > bt.capacity) n = bt.capacity;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        pool.cnt[0] = (unsigned)n;
        pool.wave[1] = n;
        pool.stats[2] += (unsigned long long)n;
        if (pool.fetch) pool.fetch[0] = 0u;
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long g = base + i;
        int j = job_of(bt, g);
        const FrameParams& F = bt.jobs[j].frame;
        const DevScene& S = bt.scenes[j];
        long long local = g - bt.offsets[j];
        const long long npix = (long long)F.width * F.height;
        int pix = (int)(local % npix);
        int sample = (int)(local / npix);
        int x = pix % F.width, y = pix / F.width;
        Rng rng;
        rng.init((uint32_t)(x + F.px_off), (uint32_t)(y + F.py_off), (uint32_t)(F.first_sample + sample), F.salt);
        float pxf = (float)x + 0.5f + (float)F.px_off;
        float pyf = (float)y + 0.5f + (float)F.py_off;
        float a0 = rng.next();
        float a1 = rng.next();
        float fx = pxf + (a0 - 0.5f), fy = pyf + (a1 - 0.5f);
        rng.next();
        rng.next();
        float ndcx = (2.0f * fx / (float)F.img_w) - 1.0f;
        float ndcy = (2.0f * fy / (float)F.img_h) - 1.0f;
        ndcx *= F.cam.aspect;
        f3 dir = normalize(ld3(F.cam.forward) + ndcx * F.cam.tan_fov * ld3(F.cam.right) +
                           ndcy * F.cam.tan_fov * ld3(F.cam.up));
        f3 o = ld3(F.cam.position);
        int medium = S.has_media ? scene_region_at(S, o) : -1;
        pool.ray_o[i] = f4(o, 0.0f);
        pool.ray_d[i] = f4(dir, 1.0f);
        pool.thr[i] = make_float4(1.f, 1.f, 1.f, 0.f);
        pool.rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        pool.prev_q[i] = f4(o, 0.0f);
        pool.st[i] = make_int4(0, medium, 0, 1);
        pool.rng[i] = make_uint2(rng.base, rng.dim);
        pool.job[i] = j;
        pool.q[0][i] = (int)i;
    }
}

// Fold the wave's radiance into each job's film.  Within a wave the paths of job j are the
// contiguous range [s, e) of the concatenated index space, and one pixel's samples lie npix
// apart in it.  The first npix paths of the range (one per pixel the wave touches) each add
// their pixel's samples to the film in sample order, like k_film: the film is the sequential
// FP64 sum of every pixel's samples in sample order, so a batched film equals the job's plain
// film bit for bit, however the waves split the jobs.
__global__ void k_film_batch(PathPool pool, BatchTables bt) {
    const long long base = pool.wave[0];
    const long long n = pool.wave[1];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int j = pool.job[i];
        const BatchJob& J = bt.jobs[j];
        const long long npix = (long long)J.frame.width * J.frame.height;
        const long long off = bt.offsets[j];
        const long long g = base + i;
        if (g - (off > base ? off : base) >= npix) continue;   // not the first visit of its pixel in this wave
        const long long job_end = j + 1 < bt.n_jobs ? bt.offsets[j + 1] : bt.total;
        const long long end = job_end < base + n ? job_end : base + n;
        const long long pix = (g - off) % npix;
        double* su = J.sum + 3 * pix;
        double* sq = J.sumsq + 3 * pix;
        double s0 = su[0], s1 = su[1], s2 = su[2], q0 = sq[0], q1 = sq[1], q2 = sq[2];
        for (long long k = g; k < end; k += npix) {
            const float4 L = pool.rad[k - base];
            s0 += (double)L.x; s1 += (double)L.y; s2 += (double)L.z;
            q0 += (double)L.x * (double)L.x; q1 += (double)L.y * (double)L.y; q2 += (double)L.z * (double)L.z;
        }
        su[0] = s0; su[1] = s1; su[2] = s2;
        sq[0] = q0; sq[1] = q1; sq[2] = q2;
    }
}

// Raw nearest-hit queries (tests and tools): per ray (o.xyz, d.xyz) the region, the
// element (instance), the ORIGINAL triangle index (or -1) and t (kMaxDist on a miss).
__global__ void k_trace_rays(DevScene S, const float* rays, int n, int* region, int* element, int* prim, float* t_out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        Ray r;
        r.o = f3(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]);
        r.d = f3(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]);
        HitRec h = scene_closest(S, r);
        int orig = -1;
        if (h.region >= 0 && h.prim >= 0) {
            const ptr_region& g = S.regions[h.region];
            const DevMesh& m = S.meshes[g.shape == PTR_SHAPE_MESH ? g.ref : S.batches[g.ref].proto_mesh];
            const float4* tri = (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) ? m.tri_w : m.tri;
            orig = __float_as_int(tri[3 * h.prim].w);
        }
        int el = h.element;
        if (h.region >= 0 && S.regions[h.region].shape == PTR_SHAPE_INSTANCES) {   // the caller's instance index
            const DevBatch& b = S.batches[S.regions[h.region].ref];
            el = ((S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w) ? b.inst_id_w : b.inst_id)[h.element];
        }
        region[k] = h.region;
        element[k] = el;
        prim[k] = orig;
        t_out[k] = h.t;
    }
}

__global__ void k_set_frame(FrameParams* dst, FrameParams F) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst = F;
}

__global__ void k_advance(PathPool pool) {
    if (blockIdx.x == 0 && threadIdx.x == 0) pool.wave[0] += pool.wave[1];
}

// Mean / variance exports from the FP64 film.
__global__ void k_export(const double* sum, const double* sumsq, double nsamples, int npix, int what, float* out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npix * 3; j += gridDim.x * blockDim.x) {
        double m = sum[j] / nsamples;
        if (what == 0) out[j] = (float)m;
        else {
            double v = sumsq[j] / nsamples - m * m;
            if (v < 0.0) v = 0.0;
            out[j] = (float)(nsamples > 1.0 ? v * nsamples / (nsamples - 1.0) : 0.0);
        }
    }
}

}  // namespace ptx
