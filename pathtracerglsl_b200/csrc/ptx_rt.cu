// ptx_rt.cu — the C ABI of include/ptx_rt.h: context, scene upload, programs, frames.
//
// One context = one CUDA device + one stream.  A program owns its film (FP64 per-pixel
// sum and sum of squares) and its path pool; ptr_render renders frame.spp samples per
// pixel as waves of at most `capacity` paths, each wave a CUDA graph of
//   k_generate, (k_closest, k_shade, k_shadow) x iterations, k_film, k_advance
// captured once per (program, scene, image size) and replayed for every wave and frame.
// Frame-varying values (sample index, salt, camera) live in a device-side FrameParams
// block refreshed by one cudaMemcpyAsync before the replays, so the graph stays valid.
#include <cuda_runtime.h>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <atomic>
#include <string>
#include <dlfcn.h>

#include "device/wavefront.cuh"
#include "device/lbvh.cuh"
#include "device/rails.cuh"
#include "host/accel_build.h"

using namespace ptx;

struct ptr_program;
struct SpecKernels {
    uint64_t scene_id = 0;
    const void* closest = nullptr;
    const void* shade = nullptr;
    const void* shadow = nullptr;
    const void* shade_adj = nullptr;    // the adjoint replay's shading and shadow kernels
    const void* shadow_adj = nullptr;   // (compiled at the first ptr_backward)
};

struct ptr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    ptr_program* batch = nullptr;     // path pool + tables of batched renders
    ptr_tuning tune{1 << 24, 256, 1, 0};   // pool capacity, block size, sort buckets, ray sort
    // batched kernels compiled for a job mix's occupant census (ptr_specialize_batch),
    // by census key
    std::map<std::string, SpecKernels> batch_spec;
    int accel_build = PTR_BUILD_HOST;   // where ptr_upload_scene builds mesh BVHs (ptr_set_accel_build)
};

struct ptr_scene {
    ptr_ctx* ctx = nullptr;
    DevScene dev{};
    std::vector<void*> allocs;
    int has_media = 0;
    int max_stack_depth = 0;
    int n_lights = 0, n_delta_lights = 0, env_samplable = 0;
    std::vector<ptr_material> h_materials;   // host copies for ptr_update_params / ptr_backward
    std::vector<ptr_region> h_regions;
    // identity and occupant census for ptr_specialize: material models, light kinds,
    // environment kind and region shapes present (bit per PTR_* value); with at most 16
    // regions, their count and shapes (4 bits each)
    uint64_t id = 0;
    unsigned spec_mats = 0, spec_lights = 0, spec_envs = 0, spec_shapes = 0;
    int spec_nregions = 0;
    unsigned long long spec_shape_code = 0;
};

// Kernels of one program compiled for one scene (ptr_specialize).
struct ptr_program {
    ptr_ctx* ctx = nullptr;
    ptr_program_desc desc{};
    // film
    int fw = 0, fh = 0;
    double* sum = nullptr;
    double* sumsq = nullptr;
    double* aov_sum = nullptr;   // first-hit pictures: 6 doubles per pixel (programs with aovs)
    size_t aov_n = 0;
    double nsamples = 0.0;
    float* export_buf = nullptr;
    // path pool
    int capacity = 0;
    std::vector<void*> pool_allocs;
    PathPool pool{};
    FrameParams* fp_dev = nullptr;
    // graph cache
    cudaGraphExec_t graph = nullptr;
    const ptr_scene* graph_scene = nullptr;
    uint64_t graph_scene_id = 0;
    int graph_w = 0, graph_h = 0, graph_iters = 0;
    ptr_tuning graph_tune{};
    float* graph_samples = nullptr;
    // counters / profiling
    ptr_counters last{};
    unsigned long long* work_dev = nullptr;   // counting-pass tallies (4 x u64)
    const ptr_scene* last_scene = nullptr;
    int work_valid = 0;
    int profile_next = 0;
    float prof_ms[PTR_PROFILE_CLASSES] = {};
    int prof_launches[PTR_PROFILE_CLASSES] = {};
    // per-scene kernels (ptr_specialize), used while rendering that scene
    SpecKernels spec{};
    const void* graph_spec = nullptr;
    // adjoint
    float* adj_dl = nullptr;          // W*H*3 adjoint image
    size_t adj_dl_n = 0;
    double* adj_grads = nullptr;      // PTR_GRAD_SLOTS per material
    size_t adj_grads_n = 0;
    float4* hit_log = nullptr;        // the adjoint's hit log (PathPool::hit_log)
    size_t hit_log_bytes = 0;
};

namespace {

inline float __int_as_float_host(int v) { float f; std::memcpy(&f, &v, 4); return f; }

int fail(ptr_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}
int cuda_fail(ptr_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, PTR_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(ctx, call)                                              \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
    } while (0)

template <typename T>
int dev_copy(ptr_ctx* ctx, std::vector<void*>& allocs, const T* host, size_t n, const T** out) {
    *out = nullptr;
    if (n == 0) return PTR_OK;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) return fail(ctx, PTR_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    CK(ctx, cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice));
    *out = (const T*)p;
    return PTR_OK;
}

// Grid of the grid-stride wavefront kernels: 2048 resident threads per SM.
int launch_grid(int n_sm, int block = 256) { return n_sm * (2048 / block); }

// One wave of resident blocks per SM for a kernel (the occupancy calculator's figure for its
// registers / shared memory at this block size, cached per kernel): a grid-stride kernel
// sized for more blocks than fit runs them in a second wave whose tail leaves SMs idle.
int resident_grid(const void* kern, int block, size_t smem, int n_sm) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t>, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_tuple(kern, block, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second * n_sm;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, block, smem) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 2048 / block;
    }
    cache[key] = nb;
    return nb * n_sm;
}

// Launches a wavefront kernel on its resident grid.  A dry launcher only fills the
// occupancy cache (run once outside stream capture, before the first captured wave).
// count: if set, incremented per launch (the instrumented passes report kernel launches).
struct Launcher {
    int block, n_sm;
    cudaStream_t st;
    bool dry;
    int* count = nullptr;
    template <class... KA, class... A>
    void operator()(void (*kern)(KA...), size_t smem, A... args) const {
        const int g = resident_grid((const void*)kern, block, smem, n_sm);
        if (dry) return;
        kern<<<g, block, smem, st>>>(args...);
        if (count) ++*count;
    }
    void count_raw(int n) const { if (!dry && count) *count += n; }
    // a kernel handle of a runtime-compiled library (ptr_specialize); the arguments must
    // have the kernel's parameter types
    template <class... A>
    void raw(const void* kern, size_t smem, A... args) const {
        const int g = resident_grid(kern, block, smem, n_sm);
        if (dry) return;
        void* argv[] = {(void*)&args...};
        cudaLaunchKernel(kern, dim3((unsigned)g), dim3((unsigned)block), argv, smem, st);
        if (count) ++*count;
    }
};

void free_pool(ptr_program* p) {
    for (void* a : p->pool_allocs) cudaFree(a);
    p->pool_allocs.clear();
    p->pool = PathPool{};
    p->capacity = 0;
    if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
}

int alloc_pool(ptr_program* p, int capacity, bool slot2, bool adj = false, bool spectral = false) {
    free_pool(p);
    ptr_ctx* ctx = p->ctx;
    auto get = [&](size_t bytes, void** out) -> int {
        cudaError_t e = cudaMalloc(out, bytes);
        if (e != cudaSuccess) return fail(ctx, PTR_E_NOMEM, std::string("path pool cudaMalloc: ") + cudaGetErrorString(e));
        p->pool_allocs.push_back(*out);
        return PTR_OK;
    };
    size_t c = (size_t)capacity;
    PathPool& q = p->pool;
    int rc = PTR_OK;
    // a two-field record: 32 bytes per path, the first field at +0, the second at +16
    auto pair = [&](auto& a, auto& b) -> int {
        void* base = nullptr;
        if (int r = get(c * 32, &base)) return r;
        a.p = (std::remove_reference_t<decltype(*a.p)>*)base;
        b.p = (std::remove_reference_t<decltype(*b.p)>*)((char*)base + 16);
        return PTR_OK;
    };
    if ((rc = pair(q.ray_o, q.ray_d)) || (rc = pair(q.thr, q.rad)) ||
        (rc = pair(q.prev_q, q.st)) || (rc = get(c * 16, (void**)&q.prev_n)) || (rc = get(c * 4, (void**)&q.sh_seed)) ||
        (rc = get(c * 8, (void**)&q.rng)) || (rc = pair(q.hit, q.hit_i)) ||
        (rc = pair(q.sh_o, q.sh_d)) || (rc = pair(q.sh_lp, q.sh_c)) || (rc = get(c * 4, (void**)&q.q[0])) ||
        (rc = get(c * 4, (void**)&q.q[1])) || (rc = get(c * 4, (void**)&q.shq)) ||
        (rc = get(c * 4, (void**)&q.job)) ||
        (rc = get(64, (void**)&q.cnt)) || (rc = get(64, (void**)&q.stats)) ||
        (rc = get(64, (void**)&q.wave)) || (rc = get(c * 4, (void**)&q.q_sorted)) ||
        (rc = get(c, (void**)&q.sort_key)) || (rc = get((size_t)kMaxKeys * kSortChunks * sizeof(unsigned), (void**)&q.sort_hist)) ||
        (rc = get(4 * sizeof(unsigned), (void**)&q.fetch)) || (rc = get(c, (void**)&q.rkey)) ||
        (rc = get(c, (void**)&q.skey)) || (rc = get(c * 4, (void**)&q.q_ray)) ||
        (rc = get(c * 4, (void**)&q.shq_s))) {
        free_pool(p);
        return rc;
    }
    if (cudaMemset(q.fetch, 0, 4 * sizeof(unsigned)) != cudaSuccess) {
        free_pool(p);
        return fail(ctx, PTR_E_CUDA, "path pool: clearing the work tickets failed");
    }
    // the second shadow slot only for programs with the per-segment equiangular site
    if (slot2 && ((rc = pair(q.sh2_o, q.sh2_d)) || (rc = pair(q.sh2_lp, q.sh2_c)) ||
                  (rc = get(c * 4, (void**)&q.shq2)))) {
        free_pool(p);
        return rc;
    }
    // the adjoint replay's per-path records
    if (adj && ((rc = get(c * 16, (void**)&q.l_rem)) || (rc = get(c * 16, (void**)&q.dl)) ||
                (rc = get(c * 16, (void**)&q.sh_g)) || (rc = get(c * 4, (void**)&q.sh_gm)))) {
        free_pool(p);
        return rc;
    }
    // the spectral colour model's wavelengths and shadow pdfs
    if (spectral && ((rc = get(c * 16, (void**)&q.wl)) || (rc = get(c * 16, (void**)&q.wl_pdf)) ||
                     (rc = get(c * 4, (void**)&q.sh_pdf)) || (rc = get(c * 4, (void**)&q.sh2_pdf)))) {
        free_pool(p);
        return rc;
    }
    p->capacity = capacity;
    return PTR_OK;
}

// Number of walk iterations a wave needs: maxBounces + 1 vertex evaluations, plus one per
// null-interface crossing a path may make (crossings do not consume a bounce).
int wave_iterations(const ptr_program* p, const ptr_scene* s) {
    int it = p->desc.max_bounces + 1;
    if (s->has_media) it += p->desc.max_null_crossings;
    return it;
}

// The launch tuning of a program's context; a program without a context (the
// allocation-free entry point's) launches with the defaults.
const ptr_tuning kDefaultTuning{1 << 24, 256, 1, 0};
// Counting sort of a device-counted queue (src[0, *count)) by its keys into dst (a no-op on
// the device below kSortMin entries).
template <bool GATHER>
void launch_sort(const Launcher& L, const PathPool& pool, const int* src, const unsigned char* keys, const unsigned* count, int* dst) {
    if (L.dry) return;
    k_sort_hist<GATHER><<<kSortChunks, kSortThreads, 0, L.st>>>(src, keys, count, pool.sort_hist);
    k_sort_scan<<<1, kSortScanThreads, kSortScanSmem, L.st>>>(count, pool.sort_hist);
    k_sort_scatter<GATHER><<<kSortChunks, kSortThreads, 0, L.st>>>(src, keys, count, pool.sort_hist, dst);
    L.count_raw(3);
}
// After k_closest: the compacted live queue grouped by shading class (occupant-sorted
// shading), keyed by path index, so each class keeps the compaction's ascending order.
void launch_shade_sort(const Launcher& L, const PathPool& pool, int in) {
    if (pool.sort_buckets <= 1) return;
    launch_sort<true>(L, pool, pool.q[in], pool.sort_key, pool.cnt + in, pool.q_sorted);
}
// After k_shade: the next closest-hit queue and the shadow queue in ray-coherence order.
void launch_ray_sort(const Launcher& L, const PathPool& pool, int in, bool shadows) {
    if (!pool.ray_sort) return;
    launch_sort<false>(L, pool, pool.q[in ^ 1], pool.rkey, pool.cnt + (in ^ 1), pool.q_ray);
    if (shadows) launch_sort<false>(L, pool, pool.shq, pool.skey, pool.cnt + 2, pool.shq_s);
}
const ptr_tuning& tuning_of(const ptr_program* p) { return p->ctx ? p->ctx->tune : kDefaultTuning; }

// Event pairs around each launch of an instrumented render (kernel class, start, end).
struct ProfRec { int cls; cudaEvent_t a, b; int n0, n; };   // n: kernels launched in the region

template <class Col>
void launch_wave_t(ptr_program* p, const ptr_scene* s, cudaStream_t st, int iters, float* samples, int n_sm,
                   std::vector<ProfRec>* prof, bool film, bool dry) {
    constexpr bool SPECTRAL = sizeof(Col) == sizeof(s4);
    DevScene Sp = s->dev;
    Sp.accel = p->desc.accel;
    Sp.inst_accel = p->desc.instance_accel;
    Sp.work = (p->profile_next & PTR_PROFILE_WORK) ? p->work_dev : nullptr;
    int n_launched = 0;
    auto mark = [&](int cls) -> ProfRec* {
        if (!prof) return nullptr;
        ProfRec r{cls, nullptr, nullptr, n_launched, 0};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, st);
        prof->push_back(r);
        return &prof->back();
    };
    auto done = [&](ProfRec* r) {
        if (!r) return;
        cudaEventRecord(r->b, st);
        r->n = n_launched - r->n0;
    };
    const DevScene& S = Sp;
    ProgParams P;
    P.max_bounces = p->desc.max_bounces;
    P.direct = p->desc.direct;
    P.rr_start = p->desc.rr_start;
    P.max_null = p->desc.max_null_crossings;
    P.rr_max_survival = p->desc.rr_max_survival;
    P.scattering = p->desc.scattering;
    P.equiangular = p->desc.equiangular;
    P.light_tree = p->desc.light_tree;
    const int block = tuning_of(p).block;
    const Launcher L{block, n_sm, st, dry, &n_launched};
    PathPool pool = p->pool;
    pool.sort_buckets = tuning_of(p).sort_buckets;
    pool.ray_sort = tuning_of(p).ray_sort;
    ProfRec* r = mark(0);
    const BatchTables nob{};
    // this scene's compiled kernels (ptr_specialize); the counting pass keeps the generic ones
    const SpecKernels* sk = (p->spec.scene_id == s->id && p->spec.shade) ? &p->spec : nullptr;
    L(k_generate<false, SPECTRAL>, 0, S, pool, p->fp_dev, AdjParams{});
    done(r);
    for (int it = 0; it < iters; ++it) {
        int in = it & 1;
        PathPool pi = pool;   // camera rays keep their generation order; later queues are key-sorted
        pi.ray_in = pool.ray_sort && it > 0;
        pi.iter = it;
        r = mark(1);
        if (S.work) L(k_closest<true, false>, 0, S, pi, in, nob);
        else if (sk) L.raw(sk->closest, 0, S, pi, in, nob);
        else L(k_closest<false, false>, 0, S, pi, in, nob);
        done(r);
        if (pool.sort_buckets > 1) {   // occupant-sorted shading queue
            r = mark(5);
            launch_shade_sort(L, pi, in);
            done(r);
        }
        const bool media = s->has_media != 0;
        r = mark(2);
        if (sk) L.raw(sk->shade, 0, S, pi, P, in, nob, AdjParams{});
        else switch (P.direct * 2 + (media ? 1 : 0)) {
            case 0: L(k_shade<Col, PTR_DIRECT_NONE, false, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
            case 1: L(k_shade<Col, PTR_DIRECT_NONE, true, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
            case 2: L(k_shade<Col, PTR_DIRECT_NEE, false, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
            case 3: L(k_shade<Col, PTR_DIRECT_NEE, true, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
            case 4: L(k_shade<Col, PTR_DIRECT_MIS, false, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
            default: L(k_shade<Col, PTR_DIRECT_MIS, true, false>, 0, S, pi, P, in, nob, AdjParams{}); break;
        }
        done(r);
        if (pool.ray_sort) {
            r = mark(5);
            launch_ray_sort(L, pool, in, P.direct != PTR_DIRECT_NONE);
            done(r);
        }
        if (P.direct != PTR_DIRECT_NONE) {
            r = mark(3);
            PathPool ps = pool;
            ps.iter = it;
            // slot 1 (equiangular segment queries) before slot 0 (surface / vertex NEE)
            for (int slot = P.equiangular ? 1 : 0; slot >= 0; --slot) {
                if (S.work) {
                    DevScene Sq = S;
                    Sq.work = S.work + 4;   // the shadow queries' own tallies
                    if (media) L(k_shadow<Col, true, true, false>, 0, Sq, ps, P, nob, slot, AdjParams{});
                    else L(k_shadow<Col, false, true, false>, 0, Sq, ps, P, nob, slot, AdjParams{});
                } else if (sk) {
                    L.raw(sk->shadow, 0, S, ps, P, nob, slot, AdjParams{});
                } else {
                    if (media) L(k_shadow<Col, true, false, false>, 0, S, ps, P, nob, slot, AdjParams{});
                    else L(k_shadow<Col, false, false, false>, 0, S, ps, P, nob, slot, AdjParams{});
                }
            }
            done(r);
        }
    }
    if (!film) return;
    r = mark(4);
    L(k_film<SPECTRAL>, 0, pool, p->fp_dev, p->sum, p->sumsq, samples, S);
    if (!dry) k_advance<<<1, 32, 0, st>>>(pool);
    L.count_raw(1);
    done(r);
}

void launch_wave(ptr_program* p, const ptr_scene* s, cudaStream_t st, int iters, float* samples, int n_sm,
                 std::vector<ProfRec>* prof = nullptr, bool film = true, bool dry = false) {
    if (p->desc.color == PTR_COLOR_SPECTRAL) launch_wave_t<s4>(p, s, st, iters, samples, n_sm, prof, film, dry);
    else launch_wave_t<f3>(p, s, st, iters, samples, n_sm, prof, film, dry);
}


// The adjoint's replay of one wave (after launch_wave(..., film = false) left every path's
// forward radiance in the pool): the same kernels with ADJ = true, then the wave cursor.
void launch_replay(ptr_program* p, const ptr_scene* s, cudaStream_t st, int iters, int n_sm, const AdjParams& adj) {
    DevScene S = s->dev;
    S.accel = p->desc.accel;
    S.inst_accel = p->desc.instance_accel;
    S.work = nullptr;
    const PathPool& pool = p->pool;
    ProgParams P;
    P.max_bounces = p->desc.max_bounces;
    P.direct = p->desc.direct;
    P.rr_start = p->desc.rr_start;
    P.max_null = p->desc.max_null_crossings;
    P.rr_max_survival = p->desc.rr_max_survival;
    P.scattering = p->desc.scattering;
    P.equiangular = 0;
    P.light_tree = p->desc.light_tree;
    const int block = tuning_of(p).block;
    const Launcher L{block, n_sm, st, false};
    const size_t smem = sizeof(double) * PTR_GRAD_SLOTS * (size_t)S.n_materials;
    const BatchTables nob{};
    const bool media = s->has_media != 0;
    // the per-scene replay kernels (ptr_specialize, then the first ptr_backward), if any
    const SpecKernels* sk = (p->spec.scene_id == s->id && p->spec.shade_adj) ? &p->spec : nullptr;
    L(k_generate<true>, 0, S, pool, p->fp_dev, adj);
    for (int it = 0; it < iters; ++it) {
        int in = it & 1;
        PathPool pi = pool;
        pi.iter = it;
        if (sk) {
            L.raw(sk->closest, 0, S, pi, in, nob);
            L.raw(sk->shade_adj, smem, S, pool, P, in, nob, adj);
            if (P.direct != PTR_DIRECT_NONE) L.raw(sk->shadow_adj, smem, S, pi, P, nob, 0, adj);
            continue;
        }
        L(k_closest<false, false>, 0, S, pi, in, nob);
        switch (P.direct * 2 + (media ? 1 : 0)) {
            case 0: L(k_shade<f3, PTR_DIRECT_NONE, false, false, true>, smem, S, pool, P, in, nob, adj); break;
            case 1: L(k_shade<f3, PTR_DIRECT_NONE, true, false, true>, smem, S, pool, P, in, nob, adj); break;
            case 2: L(k_shade<f3, PTR_DIRECT_NEE, false, false, true>, smem, S, pool, P, in, nob, adj); break;
            case 3: L(k_shade<f3, PTR_DIRECT_NEE, true, false, true>, smem, S, pool, P, in, nob, adj); break;
            case 4: L(k_shade<f3, PTR_DIRECT_MIS, false, false, true>, smem, S, pool, P, in, nob, adj); break;
            default: L(k_shade<f3, PTR_DIRECT_MIS, true, false, true>, smem, S, pool, P, in, nob, adj); break;
        }
        if (P.direct != PTR_DIRECT_NONE) {
            if (media) L(k_shadow<f3, true, false, false, true>, smem, S, pi, P, nob, 0, adj);
            else L(k_shadow<f3, false, false, false, true>, smem, S, pi, P, nob, 0, adj);
        }
    }
    k_advance<<<1, 32, 0, st>>>(pool);
}

// One wave of a batched render: the same kernel sequence over the concatenated job space;
// scene, program knobs and frame come from the per-job tables.
// sk: the mix's compiled batched kernels (ptr_specialize_batch), or null for the generic ones.
void launch_batch_wave(const DevScene& S0, const PathPool& pool_in, const BatchTables& bt, int direct, bool media,
                       bool equiangular, cudaStream_t st, int iters, int n_sm, const ptr_tuning& tune,
                       const SpecKernels* sk, std::vector<ProfRec>* prof = nullptr, bool dry = false) {
    const int block = tune.block;
    int n_launched = 0;
    const Launcher L{block, n_sm, st, dry, &n_launched};
    PathPool pool = pool_in;
    pool.sort_buckets = tune.sort_buckets;
    pool.ray_sort = tune.ray_sort;
    ProgParams P0{};
    auto mark = [&](int cls) -> ProfRec* {
        if (!prof) return nullptr;
        ProfRec r{cls, nullptr, nullptr, n_launched, 0};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, st);
        prof->push_back(r);
        return &prof->back();
    };
    auto done = [&](ProfRec* r) {
        if (!r) return;
        cudaEventRecord(r->b, st);
        r->n = n_launched - r->n0;
    };
    ProfRec* r = mark(0);
    L(k_generate_batch, 0, pool, bt);
    done(r);
    for (int it = 0; it < iters; ++it) {
        int in = it & 1;
        PathPool pi = pool;
        pi.ray_in = pool.ray_sort && it > 0;
        r = mark(1);
        if (sk) L.raw(sk->closest, 0, S0, pi, in, bt);
        else L(k_closest<false, true>, 0, S0, pi, in, bt);
        done(r);
        if (pool.sort_buckets > 1) {
            r = mark(5);
            launch_shade_sort(L, pi, in);
            done(r);
        }
        r = mark(2);
        if (sk) L.raw(sk->shade, 0, S0, pi, P0, in, bt, AdjParams{});
        else switch (direct * 2 + (media ? 1 : 0)) {
            case 0: L(k_shade<f3, PTR_DIRECT_NONE, false, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
            case 1: L(k_shade<f3, PTR_DIRECT_NONE, true, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
            case 2: L(k_shade<f3, PTR_DIRECT_NEE, false, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
            case 3: L(k_shade<f3, PTR_DIRECT_NEE, true, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
            case 4: L(k_shade<f3, PTR_DIRECT_MIS, false, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
            default: L(k_shade<f3, PTR_DIRECT_MIS, true, true>, 0, S0, pi, P0, in, bt, AdjParams{}); break;
        }
        done(r);
        if (pool.ray_sort) {
            r = mark(5);
            launch_ray_sort(L, pool, in, direct != PTR_DIRECT_NONE);
            done(r);
        }
        if (direct != PTR_DIRECT_NONE) {
            r = mark(3);
            for (int slot = equiangular ? 1 : 0; slot >= 0; --slot) {
                if (sk) L.raw(sk->shadow, 0, S0, pool, P0, bt, slot, AdjParams{});
                else if (media) L(k_shadow<f3, true, false, true>, 0, S0, pool, P0, bt, slot, AdjParams{});
                else L(k_shadow<f3, false, false, true>, 0, S0, pool, P0, bt, slot, AdjParams{});
            }
            done(r);
        }
    }
    r = mark(4);
    L(k_film_batch, 0, pool, bt);
    if (!dry) k_advance<<<1, 32, 0, st>>>(pool);
    L.count_raw(1);
    done(r);
}

int device_sms(int dev) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

// A mesh's binary BVH and compressed wide BVH built on the device (device/lbvh.cuh) from
// its vertex and index arrays, with the triangle records of both leaf orders.  The
// arrays the walks read join the scene's allocations; the build's temporaries are freed.
// The build proper over device-resident inputs: positions (3 floats per vertex), the index
// triples and the optional per-triangle alpha, all in the caller's triangle order.  binary:
// also emit the preorder binary BVH and its triangle records (a caller with its own binary
// tree, the rail upload, takes the wide BVH only; root and bin_depth are then not set).
int build_mesh_device_core(ptr_ctx* ctx, ptr_scene* s, const float* d_pos, const unsigned* d_idx, const float* d_alpha,
                           int n, DevMesh& m, std::vector<double>& root, int& n_nodes, int& n_cw_nodes, int& bin_depth,
                           bool binary = true) {
    using namespace lbvh;
    cudaStream_t st = ctx->stream;
    const int n_sm = device_sms(ctx->device);
    const int grid = n_sm * 8, block = 256;
    int n_pad = kBitonicTile;
    while (n_pad < n) n_pad <<= 1;
    std::vector<void*> tmp;
    auto alloc = [&](size_t bytes, bool keep) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        (keep ? s->allocs : tmp).push_back(p);
        return p;
    };
    auto release = [&]() { for (void* p : tmp) cudaFree(p); tmp.clear(); };
    const int total = 2 * n - 1;
    const int n_int = std::max(n - 1, 1);
    float4* lo = (float4*)alloc(sizeof(float4) * (size_t)n, false);
    float4* hi = (float4*)alloc(sizeof(float4) * (size_t)n, false);
    int* cb = (int*)alloc(sizeof(int) * 8, false);
    unsigned long long* keys = (unsigned long long*)alloc(sizeof(unsigned long long) * (size_t)n_pad, false);
    int* child = (int*)alloc(sizeof(int) * 2 * (size_t)n_int, false);
    int* parent = (int*)alloc(sizeof(int) * (size_t)total, false);
    int2* range = (int2*)alloc(sizeof(int2) * (size_t)total, false);
    unsigned* arrivals = (unsigned*)alloc(sizeof(unsigned) * (size_t)n_int, false);
    float4* nlo = (float4*)alloc(sizeof(float4) * (size_t)total, false);
    float4* nhi = (float4*)alloc(sizeof(float4) * (size_t)total, false);
    int2* ta = (int2*)alloc(sizeof(int2) * (size_t)n, false);
    int2* tb = (int2*)alloc(sizeof(int2) * (size_t)n, false);
    unsigned* counters = (unsigned*)alloc(sizeof(unsigned) * 8, false);
    uint32_t* wide_big = (uint32_t*)alloc(sizeof(uint32_t) * 20 * (size_t)n, false);
    uint32_t* order = (uint32_t*)alloc(sizeof(uint32_t) * (size_t)n, false);
    float4* bvh = binary ? (float4*)alloc(sizeof(float4) * 2 * (size_t)total, true) : nullptr;
    float4* tri = binary ? (float4*)alloc(sizeof(float4) * 3 * (size_t)n, true) : nullptr;
    float4* tri_w = (float4*)alloc(sizeof(float4) * 3 * (size_t)n, true);
    if (!lo || !hi || !cb || !keys || !child || !parent || !range ||
        !arrivals || !nlo || !nhi || !ta || !tb || !counters || !wide_big || !order || (binary && (!bvh || !tri)) || !tri_w) {
        release();
        return fail(ctx, PTR_E_NOMEM, "scene: device BVH build: cudaMalloc");
    }
    const int cb_init[8] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF, (int)0x80000000, (int)0x80000000, (int)0x80000000, 0, 0};
    const unsigned cnt_init[8] = {1u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    const int2 root_task = make_int2(0, 0);   // binary node 0 (internal root, or the one leaf) -> wide node 0
    cudaError_t e = cudaMemcpyAsync(cb, cb_init, sizeof(cb_init), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(counters, cnt_init, sizeof(cnt_init), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ta, &root_task, sizeof(int2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(arrivals, 0, sizeof(unsigned) * (size_t)n_int, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // the small host tables are copied before the launches
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "scene: device BVH build"); }
    k_boxes<<<grid, block, 0, st>>>(d_pos, d_idx, n, lo, hi, cb);
    k_keys<<<grid, block, 0, st>>>(lo, hi, n, n_pad, cb, keys);
    k_bitonic_local<<<n_pad / kBitonicTile, 512, 0, st>>>(keys, 2, kBitonicTile);
    for (int k = 2 * kBitonicTile; k <= n_pad; k <<= 1) {
        for (int j = k >> 1; j >= kBitonicTile; j >>= 1) k_bitonic_global<<<grid, block, 0, st>>>(keys, n_pad, k, j);
        k_bitonic_local<<<n_pad / kBitonicTile, 512, 0, st>>>(keys, k, k);
    }
    k_hierarchy<<<grid, block, 0, st>>>(keys, n, child, parent, range);
    k_refit<<<grid, block, 0, st>>>(keys, lo, hi, n, child, parent, arrivals, nlo, nhi);
    int* depth_dev = cb + 6;   // the binary layout's deepest level (initialised to 0)
    if (binary) k_binary_layout<<<grid, block, 0, st>>>(n, child, parent, range, nlo, nhi, bvh, depth_dev);
    // the wide nodes, one level of tasks per launch
    int n_tasks = 1, levels = 0;
    int2 *tin = ta, *tout = tb;
    unsigned cnt[4] = {0u, 0u, 0u, 0u};
    e = cudaGetLastError();
    while (n_tasks > 0 && e == cudaSuccess) {
        if (++levels > 64) { cnt[3] |= 2u; break; }
        e = cudaMemsetAsync(counters + 2, 0, sizeof(unsigned), st);
        if (e != cudaSuccess) break;
        k_collapse<<<std::min(grid, (n_tasks + block - 1) / block), block, 0, st>>>(n, child, range, nlo, nhi, keys, tin, n_tasks,
                                                                                   tout, counters, wide_big, order);
        e = cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        n_tasks = (int)cnt[2];
        std::swap(tin, tout);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "scene: device BVH build"); }
    if (cnt[3] != 0u || cnt[1] != (unsigned)n || cnt[0] == 0u || cnt[0] > (unsigned)std::max(n, 1)) {
        release();
        return fail(ctx, PTR_E_INVALID, "scene: device CWBVH build failed (exponent range, depth or item count)");
    }
    if (levels >= ptx_host::kCwbvhStackDepth) {
        release();
        return fail(ctx, PTR_E_INVALID, "scene: device CWBVH depth " + std::to_string(levels) + " reaches the walk's stack depth");
    }
    uint32_t* wide = (uint32_t*)alloc(sizeof(uint32_t) * 20 * (size_t)cnt[0], true);
    if (!wide) { release(); return fail(ctx, PTR_E_NOMEM, "scene: device BVH build: cudaMalloc"); }
    e = cudaMemcpyAsync(wide, wide_big, sizeof(uint32_t) * 20 * (size_t)cnt[0], cudaMemcpyDeviceToDevice, st);
    if (binary) k_emit_tris<<<grid, block, 0, st>>>(d_pos, d_idx, d_alpha, nullptr, keys, n, tri);
    k_emit_tris<<<grid, block, 0, st>>>(d_pos, d_idx, d_alpha, order, keys, n, tri_w);
    float4 rb[2];
    int depth = 0;
    if (e == cudaSuccess && binary) e = cudaMemcpyAsync(rb, bvh, sizeof(rb), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&depth, depth_dev, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scene: device BVH build");
    if (depth >= ptx_host::kBvhStackDepth)
        return fail(ctx, PTR_E_INVALID, "scene: device BVH depth " + std::to_string(depth) + " reaches the walk's stack depth");
    m.tri = tri;
    m.tri_w = tri_w;
    m.bvh = bvh;
    m.cwbvh = (const uint4*)wide;
    n_nodes = total;
    n_cw_nodes = (int)cnt[0];
    if (binary) {
        bin_depth = depth;
        root = {rb[0].x, rb[0].y, rb[0].z, rb[1].x, rb[1].y, rb[1].z};
    }
    return PTR_OK;
}

// The device build of a mesh given in host memory (ptr_set_accel_build(PTR_BUILD_DEVICE)).
int build_mesh_device(ptr_ctx* ctx, ptr_scene* s, const ptr_mesh_desc& md, DevMesh& m, std::vector<double>& root,
                      int& n_nodes, int& n_cw_nodes, int& bin_depth) {
    const int n = md.n_triangles;
    cudaStream_t st = ctx->stream;
    float* d_pos = nullptr;
    unsigned* d_idx = nullptr;
    float* d_alpha = nullptr;
    auto release = [&]() { cudaFree(d_pos); cudaFree(d_idx); cudaFree(d_alpha); };
    if (cudaMalloc(&d_pos, sizeof(float) * 3 * (size_t)md.n_vertices) != cudaSuccess ||
        cudaMalloc(&d_idx, sizeof(unsigned) * 3 * (size_t)n) != cudaSuccess ||
        (md.tri_alpha && cudaMalloc(&d_alpha, sizeof(float) * (size_t)n) != cudaSuccess)) {
        release();
        return fail(ctx, PTR_E_NOMEM, "scene: device BVH build: cudaMalloc");
    }
    cudaError_t e = cudaMemcpyAsync(d_pos, md.positions, sizeof(float) * 3 * (size_t)md.n_vertices, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_idx, md.indices, sizeof(unsigned) * 3 * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && d_alpha) e = cudaMemcpyAsync(d_alpha, md.tri_alpha, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "scene: device BVH build"); }
    const int rc = build_mesh_device_core(ctx, s, d_pos, d_idx, d_alpha, n, m, root, n_nodes, n_cw_nodes, bin_depth);
    release();   // the core synchronised the stream before it returned
    return rc;
}

// ---- scene data from the reference's packed channels (rail v2) ----------------------------
static_assert(sizeof(ptr_rail_mesh) == 56 && sizeof(ptr_rail_batch) == 40 && sizeof(ptr_rail_mesh_light) == 24 &&
              sizeof(ptr_rails) == 104, "rail records: the layouts the ctypes mirror declares");
// The channels on the device: flat float4 texel arrays, copied once each.
struct RailDev {
    const float4* v = nullptr;
    const float4* idx = nullptr;
    const float4* nodes = nullptr;
    const float4* rec = nullptr;
};

bool rail_span(int64_t base, int64_t count, int64_t total) {
    return base >= 0 && count >= 0 && base <= total && count <= total - base;
}
bool exact_id(float f, int64_t bound) { return f >= 0.0f && f == std::floor(f) && (int64_t)f < bound; }

// A binary BVH of the nodes channel (the bvh.ts node layout) over n_items leaf items:
// every box finite, every leaf range inside [0, n_items), every internal node's axis in
// 0..2 and both children after it inside the tree (so every walk moves forward and stays
// in the region).  Returns the tree's depth, or -1.
int rail_tree_depth(const float* nodes, int64_t nbase, int node_count, int n_items) {
    if (node_count < 1 || (int64_t)node_count > 2 * (int64_t)n_items - 1) return -1;
    std::vector<int> depth((size_t)node_count, 0);
    int max_depth = 0;
    for (int i = 0; i < node_count; ++i) {
        const float* q = nodes + 4 * (nbase + 2 * (int64_t)i);
        for (int k = 0; k < 8; ++k)
            if (k != 3 && k != 7 && !std::isfinite(q[k])) return -1;
        const float A = q[3], B = q[7];
        if (A >= 1.0f) {
            if (A != std::floor(A) || !exact_id(B, n_items) || (int64_t)B + (int64_t)A > n_items) return -1;
        } else if (A == -1.0f || A == -2.0f || A == -3.0f) {
            if (B != std::floor(B) || !(B > (float)(i + 1)) || !(B < (float)node_count)) return -1;
            const int d = depth[(size_t)i] + 1;
            depth[(size_t)i + 1] = std::max(depth[(size_t)i + 1], d);
            depth[(size_t)B] = std::max(depth[(size_t)B], d);
        } else {
            return -1;
        }
        max_depth = std::max(max_depth, depth[(size_t)i]);
    }
    return max_depth;
}

// A permutation of [0, n), or NULL.
bool rail_permutation(const uint32_t* order, int n) {
    if (!order) return true;
    std::vector<char> seen((size_t)n, 0);
    for (int i = 0; i < n; ++i)
        if (order[i] >= (uint32_t)n || seen[order[i]]++) return false;
    return true;
}

// Mesh mi from its rail slot: triangles gathered into the binary walk's leaf-order records,
// the rail's BVH nodes used in place, the wide BVH built on the device over the same
// triangles, and (for a mesh light) its world triangles and area CDF from the rail.
int rail_mesh(ptr_ctx* ctx, ptr_scene* s, const ptr_rails& R, const RailDev& D, int mi, bool is_light, DevMesh& m,
              std::vector<double>& root, int& bin_depth) {
    const ptr_rail_mesh& rm = R.meshes[mi];
    const int V = rm.vertex_count, T = rm.tri_count, NC = rm.node_count;
    const std::string who = "rails: mesh " + std::to_string(mi);
    if (V <= 0 || T <= 0 || !rail_span(rm.vbase, V, R.vertices_texels) || !rail_span(rm.tbase, T, R.indices_texels) ||
        !rail_span(rm.nbase, 2 * (int64_t)NC, R.nodes_texels))
        return fail(ctx, PTR_E_INVALID, who + ": empty, or a region outside its channel");
    for (int i = 0; i < V; ++i) {
        const float* p = R.vertices + 4 * (rm.vbase + i);
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return fail(ctx, PTR_E_INVALID, who + ": non-finite vertex");
    }
    for (int i = 0; i < T; ++i) {
        const float* t = R.indices + 4 * (rm.tbase + i);
        if (!exact_id(t[0], V) || !exact_id(t[1], V) || !exact_id(t[2], V)) return fail(ctx, PTR_E_INVALID, who + ": vertex id out of range");
    }
    if (!rail_permutation(rm.tri_order, T)) return fail(ctx, PTR_E_INVALID, who + ": tri_order is not a permutation");
    const int depth = rail_tree_depth(R.nodes, rm.nbase, NC, T);
    if (depth < 0) return fail(ctx, PTR_E_INVALID, who + ": malformed BVH nodes");
    if (depth >= ptx_host::kBvhStackDepth) std::fprintf(stderr, "ptx_rt: BVH depth %d reaches the walk's stack depth\n", depth);
    const ptr_rail_mesh_light* ml = nullptr;
    for (int k = 0; k < R.n_mesh_lights; ++k)
        if (R.mesh_lights[k].mesh == mi) ml = &R.mesh_lights[k];
    if (is_light != (ml != nullptr)) return fail(ctx, PTR_E_INVALID, who + ": a mesh light needs exactly its rail light slot");
    if (ml) {
        if (!rail_span(ml->wpos_base, V, R.vertices_texels) || !rail_span(ml->cdf_base, T, R.records_texels))
            return fail(ctx, PTR_E_INVALID, who + ": light tables outside their channels");
        for (int i = 0; i < V; ++i) {
            const float* p = R.vertices + 4 * (ml->wpos_base + i);
            if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return fail(ctx, PTR_E_INVALID, who + ": non-finite light vertex");
        }
        for (int i = 0; i < T; ++i)
            if (!std::isfinite(R.records[4 * (ml->cdf_base + i)])) return fail(ctx, PTR_E_INVALID, who + ": non-finite light CDF");
    }
    cudaStream_t st = ctx->stream;
    float* d_pos = nullptr;
    unsigned* d_idx = nullptr;
    uint32_t* d_order = nullptr;
    float* d_alpha = nullptr;
    auto release = [&]() { cudaFree(d_pos); cudaFree(d_idx); cudaFree(d_order); cudaFree(d_alpha); };
    float4* tri = nullptr;
    if (cudaMalloc(&d_pos, sizeof(float) * 3 * (size_t)V) != cudaSuccess ||
        cudaMalloc(&d_idx, sizeof(unsigned) * 3 * (size_t)T) != cudaSuccess ||
        (rm.tri_order && cudaMalloc(&d_order, sizeof(uint32_t) * (size_t)T) != cudaSuccess) ||
        (rm.tri_alpha && cudaMalloc(&d_alpha, sizeof(float) * (size_t)T) != cudaSuccess) ||
        cudaMalloc(&tri, sizeof(float4) * 3 * (size_t)T) != cudaSuccess) {
        if (tri) cudaFree(tri);
        release();
        return fail(ctx, PTR_E_NOMEM, who + ": cudaMalloc");
    }
    s->allocs.push_back(tri);
    const int n_sm = device_sms(ctx->device);
    cudaError_t e = cudaSuccess;
    if (d_order) e = cudaMemcpyAsync(d_order, rm.tri_order, sizeof(uint32_t) * (size_t)T, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && d_alpha) e = cudaMemcpyAsync(d_alpha, rm.tri_alpha, sizeof(float) * (size_t)T, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, who.c_str()); }
    rails::k_positions<<<n_sm * 4, 256, 0, st>>>(D.v, rm.vbase, V, d_pos);
    rails::k_caller_indices<<<n_sm * 4, 256, 0, st>>>(D.idx, rm.tbase, T, d_order, d_idx);
    rails::k_leaf_tris<<<n_sm * 4, 256, 0, st>>>(d_pos, D.idx, rm.tbase, T, d_order, d_alpha, tri);
    if ((e = cudaGetLastError()) != cudaSuccess) { release(); return cuda_fail(ctx, e, who.c_str()); }
    // the wide BVH (meshTraversal 'cwbvh') over the same triangles, built on the device
    DevMesh wide{};
    std::vector<double> wide_root;
    int wn = 0, wcw = 0, wdepth = 0;
    int rc = build_mesh_device_core(ctx, s, d_pos, d_idx, d_alpha, T, wide, wide_root, wn, wcw, wdepth, false);
    release();
    if (rc) return rc;
    m.tri = tri;
    m.bvh = D.nodes + rm.nbase;
    m.tri_w = wide.tri_w;
    m.cwbvh = wide.cwbvh;
    m.n_tris = T;
    m.n_nodes = NC;
    m.n_cw_nodes = wcw;
    m.light_cdf = nullptr;
    m.light_tri = nullptr;
    if (ml) {
        float4* lt = nullptr;
        float* cdf = nullptr;
        if (cudaMalloc(&lt, sizeof(float4) * 3 * (size_t)T) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, who + ": cudaMalloc");
        s->allocs.push_back(lt);
        if (cudaMalloc(&cdf, sizeof(float) * (size_t)T) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, who + ": cudaMalloc");
        s->allocs.push_back(cdf);
        rails::k_light_tris<<<n_sm * 4, 256, 0, st>>>(D.v, ml->wpos_base, D.idx, rm.tbase, T, lt);
        rails::k_scalars<<<n_sm * 4, 256, 0, st>>>(D.rec, ml->cdf_base, T, cdf);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, who.c_str());
        m.light_cdf = cdf;
        m.light_tri = lt;
    }
    const float* n0 = R.nodes + 4 * rm.nbase;
    root = {n0[0], n0[1], n0[2], n0[4], n0[5], n0[6]};
    bin_depth = depth;
    return PTR_OK;
}

// Batch bi from its rail slot: the TLAS nodes and (frame tier) the placement records used
// in place, params-tier records re-strided, caller instance ids and instance lights per
// leaf slot, and the wide TLAS twin built on the host over the same instance boxes.
int rail_batch(ptr_ctx* ctx, ptr_scene* s, const ptr_rails& R, const RailDev& D, int bi, const ptr_batch_desc& bd,
               const std::vector<std::vector<double>>& root_box, DevBatch& b, std::vector<double>& boxes) {
    const ptr_rail_batch& rb = R.batches[bi];
    const int N = rb.instance_count, NC = rb.node_count, PT = rb.placement_texels;
    const std::string who = "rails: batch " + std::to_string(bi);
    const bool mesh = bd.prototype_shape == PTR_SHAPE_MESH;
    if (bd.prototype_shape != PTR_SHAPE_MESH && bd.prototype_shape != PTR_SHAPE_SPHERE)
        return fail(ctx, PTR_E_INVALID, who + ": prototype must be a mesh or a sphere");
    if (mesh && (bd.prototype_ref < 0 || bd.prototype_ref >= (int)root_box.size()))
        return fail(ctx, PTR_E_INVALID, who + ": prototype mesh out of range");
    if (N <= 0 || N != bd.n_instances || PT != (mesh ? 2 : 1) || !rail_span(rb.placements_base, (int64_t)PT * N, R.records_texels) ||
        !rail_span(rb.tlas_base, 2 * (int64_t)NC, R.nodes_texels))
        return fail(ctx, PTR_E_INVALID, who + ": empty, a count that differs from the description, the wrong tier, or a region outside its channel");
    if (rail_tree_depth(R.nodes, rb.tlas_base, NC, N) < 0) return fail(ctx, PTR_E_INVALID, who + ": malformed TLAS nodes");
    if (!rail_permutation(rb.inst_order, N)) return fail(ctx, PTR_E_INVALID, who + ": inst_order is not a permutation");
    // the records at two texels per instance, and each leaf slot's world box
    std::vector<float4> rec(2 * (size_t)N);
    boxes.assign(6 * (size_t)N, 0.0);
    for (int i = 0; i < N; ++i) {
        const float* r = R.records + 4 * (rb.placements_base + (int64_t)PT * i);
        for (int k = 0; k < 4 * PT; ++k)
            if (!std::isfinite(r[k])) return fail(ctx, PTR_E_INVALID, who + ": non-finite placement");
        double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
        if (mesh) {
            const double qx = r[0], qy = r[1], qz = r[2], qw = r[3], tx = r[4], ty = r[5], tz = r[6], sc = r[7];
            if (!(sc > 0.0)) return fail(ctx, PTR_E_INVALID, who + ": placement scale must be positive");
            const std::vector<double>& rb0 = root_box[bd.prototype_ref];
            for (int k = 0; k < 8; ++k) {   // world = rotate(conj(q), s * local - t_rigid)
                const double x = (k & 1) ? rb0[3] : rb0[0], y = (k & 2) ? rb0[4] : rb0[1], z = (k & 4) ? rb0[5] : rb0[2];
                const double vx = sc * x - tx, vy = sc * y - ty, vz = sc * z - tz;
                const double cx = -qx, cy = -qy, cz = -qz;
                const double c1x = cy * vz - cz * vy + qw * vx, c1y = cz * vx - cx * vz + qw * vy, c1z = cx * vy - cy * vx + qw * vz;
                const double c2x = cy * c1z - cz * c1y, c2y = cz * c1x - cx * c1z, c2z = cx * c1y - cy * c1x;
                const double w[3] = {vx + 2.0 * c2x, vy + 2.0 * c2y, vz + 2.0 * c2z};
                for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], w[a]); mx[a] = std::max(mx[a], w[a]); }
            }
            rec[2 * (size_t)i] = make_float4(r[0], r[1], r[2], r[3]);
            rec[2 * (size_t)i + 1] = make_float4(r[4], r[5], r[6], r[7]);
        } else {
            if (!(r[3] >= 0.0f)) return fail(ctx, PTR_E_INVALID, who + ": negative sphere radius");
            for (int a = 0; a < 3; ++a) { mn[a] = (double)r[a] - r[3]; mx[a] = (double)r[a] + r[3]; }
            rec[2 * (size_t)i] = make_float4(r[0], r[1], r[2], r[3]);
            rec[2 * (size_t)i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int a = 0; a < 3; ++a) { boxes[6 * (size_t)i + a] = mn[a]; boxes[6 * (size_t)i + 3 + a] = mx[a]; }
    }
    std::vector<int> ids((size_t)N);
    for (int i = 0; i < N; ++i) ids[(size_t)i] = rb.inst_order ? (int)rb.inst_order[i] : i;
    int rc;
    const int n_sm = device_sms(ctx->device);
    if (mesh) {
        b.place = D.rec + rb.placements_base;
    } else {
        float4* place = nullptr;
        if (cudaMalloc(&place, sizeof(float4) * 2 * (size_t)N) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, who + ": cudaMalloc");
        s->allocs.push_back(place);
        rails::k_restride<<<n_sm * 4, 256, 0, ctx->stream>>>(D.rec, rb.placements_base, N, place);
        if (cudaError_t e = cudaGetLastError()) return cuda_fail(ctx, e, who.c_str());
        b.place = place;
    }
    b.tlas = D.nodes + rb.tlas_base;
    const int* pi = nullptr;
    if ((rc = dev_copy(ctx, s->allocs, ids.data(), ids.size(), &pi))) return rc;
    b.inst_id = pi;
    b.light_of = nullptr;
    b.light_of_w = nullptr;
    if (bd.light_base >= 0) {
        std::vector<int> lo((size_t)N);
        for (int i = 0; i < N; ++i) lo[(size_t)i] = bd.light_base + ids[(size_t)i];
        if ((rc = dev_copy(ctx, s->allocs, lo.data(), lo.size(), &pi))) return rc;
        b.light_of = pi;
    }
    // the wide twin over the leaf slots' boxes; its leaves index leaf slots
    b.tlas_w = nullptr;
    b.place_w = nullptr;
    b.inst_id_w = nullptr;
    ptx_host::WideBvh wt = ptx_host::build_cwbvh(boxes.data(), N, ptx_host::kCwbvhCPrim);
    if (!wt.error && wt.node_count > 0) {
        std::vector<float4> rec_w(2 * (size_t)N);
        std::vector<int> ids_w((size_t)N), lo_w((size_t)N);
        for (int i = 0; i < N; ++i) {
            const uint32_t k = wt.order[(size_t)i];
            rec_w[2 * (size_t)i] = rec[2 * (size_t)k];
            rec_w[2 * (size_t)i + 1] = rec[2 * (size_t)k + 1];
            ids_w[(size_t)i] = ids[k];
            lo_w[(size_t)i] = bd.light_base + ids[k];
        }
        const float4* p4 = nullptr;
        const uint4* u4 = nullptr;
        if ((rc = dev_copy(ctx, s->allocs, rec_w.data(), rec_w.size(), &p4))) return rc;
        b.place_w = p4;
        if ((rc = dev_copy(ctx, s->allocs, ids_w.data(), ids_w.size(), &pi))) return rc;
        b.inst_id_w = pi;
        if (bd.light_base >= 0) {
            if ((rc = dev_copy(ctx, s->allocs, lo_w.data(), lo_w.size(), &pi))) return rc;
            b.light_of_w = pi;
        }
        if ((rc = dev_copy(ctx, s->allocs, (const uint4*)wt.nodes.data(), 5 * (size_t)wt.node_count, &u4))) return rc;
        b.tlas_w = u4;
    }
    b.n_inst = N;
    b.proto_shape = bd.prototype_shape;
    b.proto_mesh = bd.prototype_ref;
    b.n_tlas = NC;
    return PTR_OK;
}

// Acceleration structures of meshes and instanced batches, built on the host and uploaded
// once: per mesh the binary SAH BLAS (leaf 2) and the compressed wide BVH, each with the
// triangles re-emitted in its leaf order as (v0, e1 | alpha, e2); per batch a binary TLAS
// (leaf 2) over the instances' world boxes with the placements in leaf order.
// With rails, mesh i and batch i come from their rail slots instead (rail_mesh, rail_batch).
int upload_accels(ptr_ctx* ctx, ptr_scene* s, const ptr_scene_desc* d, const ptr_rails* rails = nullptr) {
    DevScene& S = s->dev;
    RailDev rd;
    if (rails) {   // each channel to the device once, as the App packed it
        int rc0;
        if ((rails->vertices_texels > 0 && (rc0 = dev_copy(ctx, s->allocs, (const float4*)rails->vertices, (size_t)rails->vertices_texels, &rd.v))) ||
            (rails->indices_texels > 0 && (rc0 = dev_copy(ctx, s->allocs, (const float4*)rails->indices, (size_t)rails->indices_texels, &rd.idx))) ||
            (rails->nodes_texels > 0 && (rc0 = dev_copy(ctx, s->allocs, (const float4*)rails->nodes, (size_t)rails->nodes_texels, &rd.nodes))) ||
            (rails->records_texels > 0 && (rc0 = dev_copy(ctx, s->allocs, (const float4*)rails->records, (size_t)rails->records_texels, &rd.rec))))
            return rc0;
    }
    // the bounded geometry's box: its centre splits ray origins into octants for the
    // ray-coherence queue keys
    double world_lo[3] = {1e300, 1e300, 1e300}, world_hi[3] = {-1e300, -1e300, -1e300};
    auto grow = [&](const double* lo, const double* hi) {
        for (int a = 0; a < 3; ++a) { world_lo[a] = std::min(world_lo[a], lo[a]); world_hi[a] = std::max(world_hi[a], hi[a]); }
    };
    std::vector<DevMesh> meshes(d->n_meshes > 0 ? d->n_meshes : 0);
    std::vector<std::vector<double>> root_box(meshes.size());
    std::vector<char> is_light(meshes.size(), 0);
    for (int i = 0; i < d->n_lights; ++i)
        if (d->lights[i].kind == PTR_LIGHT_MESH) is_light[(int)d->lights[i].p[0]] = 1;
    for (int mi = 0; mi < d->n_meshes; ++mi) {
        if (rails) {
            int depth = 0;
            if (int rc0 = rail_mesh(ctx, s, *rails, rd, mi, is_light[mi] != 0, meshes[mi], root_box[mi], depth)) return rc0;
            grow(root_box[mi].data(), root_box[mi].data() + 3);
            s->max_stack_depth = std::max(s->max_stack_depth, depth);
            continue;
        }
        const ptr_mesh_desc& md = d->meshes[mi];
        if (md.n_triangles <= 0 || md.n_vertices <= 0 || !md.positions || !md.indices)
            return fail(ctx, PTR_E_INVALID, "scene: mesh " + std::to_string(mi) + " is empty");
        const int T = md.n_triangles;
        std::vector<double> boxes(6 * (size_t)T);
        for (int t = 0; t < T; ++t) {
            double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
            for (int k = 0; k < 3; ++k) {
                uint32_t v = md.indices[3 * (size_t)t + k];
                if (v >= (uint32_t)md.n_vertices) return fail(ctx, PTR_E_INVALID, "scene: mesh index out of range");
                for (int a = 0; a < 3; ++a) {
                    double x = md.positions[3 * (size_t)v + a];
                    if (!std::isfinite(x)) return fail(ctx, PTR_E_INVALID, "scene: non-finite vertex");
                    mn[a] = std::min(mn[a], x);
                    mx[a] = std::max(mx[a], x);
                }
            }
            for (int a = 0; a < 3; ++a) { boxes[6 * (size_t)t + a] = mn[a]; boxes[6 * (size_t)t + 3 + a] = mx[a]; }
        }
        auto tri_array = [&](const std::vector<uint32_t>& order) {
            std::vector<float4> tri(3 * (size_t)T);
            for (int i = 0; i < T; ++i) {
                const uint32_t t = order[i];
                const float* a = md.positions + 3 * (size_t)md.indices[3 * (size_t)t];
                const float* b = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 1];
                const float* c = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 2];
                float alpha = md.tri_alpha ? md.tri_alpha[t] : -1.0f;
                tri[3 * (size_t)i] = make_float4(a[0], a[1], a[2], __int_as_float_host((int)t));
                tri[3 * (size_t)i + 1] = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], alpha);
                tri[3 * (size_t)i + 2] = make_float4(c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.0f);
            }
            return tri;
        };
        DevMesh& m = meshes[mi];
        const float4* p4 = nullptr;
        int rc;
        int n_nodes = 0, n_cw_nodes = 0, bin_depth = 0;
        if (ctx->accel_build == PTR_BUILD_DEVICE) {   // linear BVH + wide collapse on the GPU
            if ((rc = build_mesh_device(ctx, s, md, m, root_box[mi], n_nodes, n_cw_nodes, bin_depth))) return rc;
        } else {
            ptx_host::BinaryBvh bin = ptx_host::build_bvh(boxes.data(), T, ptx_host::kBvhLeafSize, false);
            if (bin.max_depth >= ptx_host::kBvhStackDepth) std::fprintf(stderr, "ptx_rt: BVH depth %d reaches the walk's stack depth\n", bin.max_depth);
            ptx_host::WideBvh wide = ptx_host::build_cwbvh(boxes.data(), T, ptx_host::kCwbvhCPrim);
            if (wide.error) return fail(ctx, PTR_E_INVALID, "scene: CWBVH build failed (exponent range or DP invariant)");
            std::vector<float4> tri_b = tri_array(bin.order), tri_w = tri_array(wide.order);
            const uint4* u4 = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, tri_b.data(), tri_b.size(), &p4))) return rc;
            m.tri = p4;
            if ((rc = dev_copy(ctx, s->allocs, tri_w.data(), tri_w.size(), &p4))) return rc;
            m.tri_w = p4;
            if ((rc = dev_copy(ctx, s->allocs, (const float4*)bin.nodes.data(), 2 * (size_t)bin.node_count, &p4))) return rc;
            m.bvh = p4;
            if ((rc = dev_copy(ctx, s->allocs, (const uint4*)wide.nodes.data(), 5 * (size_t)wide.node_count, &u4))) return rc;
            m.cwbvh = u4;
            n_nodes = bin.node_count;
            n_cw_nodes = wide.node_count;
            bin_depth = bin.max_depth;
            root_box[mi] = {bin.nodes[0], bin.nodes[1], bin.nodes[2], bin.nodes[4], bin.nodes[5], bin.nodes[6]};
        }
        m.light_cdf = nullptr;
        m.light_tri = nullptr;
        if (is_light[mi]) {
            // lights/mesh/mesh.ts packMeshLight: float64 world areas from the float32
            // vertices, the normalised running sum rounded to float32, the last entry 1
            std::vector<double> area(T);
            double acc = 0.0;
            std::vector<float4> lt(3 * (size_t)T);
            for (int t = 0; t < T; ++t) {
                const float* a = md.positions + 3 * (size_t)md.indices[3 * (size_t)t];
                const float* b = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 1];
                const float* c = md.positions + 3 * (size_t)md.indices[3 * (size_t)t + 2];
                const double ux = (double)b[0] - a[0], uy = (double)b[1] - a[1], uz = (double)b[2] - a[2];
                const double vx = (double)c[0] - a[0], vy = (double)c[1] - a[1], vz = (double)c[2] - a[2];
                const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
                area[t] = std::sqrt(cx * cx + cy * cy + cz * cz) / 2.0;
                acc += area[t];
                lt[3 * (size_t)t] = make_float4(a[0], a[1], a[2], 0.0f);
                lt[3 * (size_t)t + 1] = make_float4(b[0], b[1], b[2], 0.0f);
                lt[3 * (size_t)t + 2] = make_float4(c[0], c[1], c[2], 0.0f);
            }
            std::vector<float> cdf(T);
            double run = 0.0;
            for (int t = 0; t < T; ++t) {
                run += area[t];
                cdf[t] = acc > 0.0 ? (float)(run / acc) : (float)((double)(t + 1) / T);
            }
            cdf[T - 1] = 1.0f;
            const float* pf = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, cdf.data(), cdf.size(), &pf))) return rc;
            m.light_cdf = pf;
            if ((rc = dev_copy(ctx, s->allocs, lt.data(), lt.size(), &p4))) return rc;
            m.light_tri = p4;
        }
        m.n_tris = T;
        m.n_nodes = n_nodes;
        m.n_cw_nodes = n_cw_nodes;
        grow(root_box[mi].data(), root_box[mi].data() + 3);
        s->max_stack_depth = std::max(s->max_stack_depth, bin_depth);
    }
    std::vector<DevBatch> batches(d->n_batches > 0 ? d->n_batches : 0);
    for (int bi = 0; bi < d->n_batches; ++bi) {
        const ptr_batch_desc& bd = d->batches[bi];
        if (rails) {
            std::vector<double> boxes;
            if (int rc0 = rail_batch(ctx, s, *rails, rd, bi, bd, root_box, batches[bi], boxes)) return rc0;
            for (int i = 0; i < bd.n_instances; ++i) grow(&boxes[6 * (size_t)i], &boxes[6 * (size_t)i + 3]);
            continue;
        }
        const int N = bd.n_instances;
        if (N <= 0 || !bd.placements) return fail(ctx, PTR_E_INVALID, "scene: instanced batch " + std::to_string(bi) + " is empty");
        if (bd.prototype_shape == PTR_SHAPE_MESH && (bd.prototype_ref < 0 || bd.prototype_ref >= d->n_meshes))
            return fail(ctx, PTR_E_INVALID, "scene: batch prototype mesh out of range");
        if (bd.prototype_shape != PTR_SHAPE_MESH && bd.prototype_shape != PTR_SHAPE_SPHERE)
            return fail(ctx, PTR_E_INVALID, "scene: batch prototype must be a mesh or a sphere");
        std::vector<double> boxes(6 * (size_t)N);
        std::vector<float4> rec(2 * (size_t)N);
        for (int i = 0; i < N; ++i) {
            const float* pl = bd.placements + 8 * (size_t)i;
            const double qx = pl[0], qy = pl[1], qz = pl[2], qw = pl[3];
            const double tx = pl[4], ty = pl[5], tz = pl[6], sc = pl[7];
            if (!(sc > 0.0)) return fail(ctx, PTR_E_INVALID, "scene: placement scale must be positive");
            // world = rotate(conj(q), s * local - t_rigid)
            auto to_world = [&](double x, double y, double z, double out[3]) {
                double vx = sc * x - tx, vy = sc * y - ty, vz = sc * z - tz;
                const double cx = -qx, cy = -qy, cz = -qz;   // conjugate
                double c1x = cy * vz - cz * vy + qw * vx, c1y = cz * vx - cx * vz + qw * vy, c1z = cx * vy - cy * vx + qw * vz;
                double c2x = cy * c1z - cz * c1y, c2y = cz * c1x - cx * c1z, c2z = cx * c1y - cy * c1x;
                out[0] = vx + 2.0 * c2x; out[1] = vy + 2.0 * c2y; out[2] = vz + 2.0 * c2z;
            };
            double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
            if (bd.prototype_shape == PTR_SHAPE_SPHERE) {
                double c[3];
                to_world(bd.proto[0], bd.proto[1], bd.proto[2], c);
                const double r = sc * bd.proto[3];
                for (int a = 0; a < 3; ++a) { mn[a] = c[a] - r; mx[a] = c[a] + r; }
                rec[2 * (size_t)i] = make_float4((float)c[0], (float)c[1], (float)c[2], (float)r);
                rec[2 * (size_t)i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                const std::vector<double>& rb = root_box[bd.prototype_ref];
                for (int k = 0; k < 8; ++k) {
                    double w[3];
                    to_world((k & 1) ? rb[3] : rb[0], (k & 2) ? rb[4] : rb[1], (k & 4) ? rb[5] : rb[2], w);
                    for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], w[a]); mx[a] = std::max(mx[a], w[a]); }
                }
                rec[2 * (size_t)i] = make_float4(pl[0], pl[1], pl[2], pl[3]);
                rec[2 * (size_t)i + 1] = make_float4(pl[4], pl[5], pl[6], pl[7]);
            }
            for (int a = 0; a < 3; ++a) { boxes[6 * (size_t)i + a] = mn[a]; boxes[6 * (size_t)i + 3 + a] = mx[a]; }
            grow(mn, mx);
        }
        ptx_host::BinaryBvh tl = ptx_host::build_bvh(boxes.data(), N, ptx_host::kBvhLeafSize, false);
        std::vector<float4> rec_leaf(2 * (size_t)N);
        for (int i = 0; i < N; ++i) {
            rec_leaf[2 * (size_t)i] = rec[2 * (size_t)tl.order[i]];
            rec_leaf[2 * (size_t)i + 1] = rec[2 * (size_t)tl.order[i] + 1];
        }
        DevBatch& b = batches[bi];
        const float4* p4 = nullptr;
        int rc;
        b.light_of = nullptr;
        b.light_of_w = nullptr;
        if (bd.light_base >= 0) {   // instance lights: the light id of each leaf slot
            std::vector<int> lo(N);
            for (int i = 0; i < N; ++i) lo[i] = bd.light_base + (int)tl.order[i];
            const int* pi = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, lo.data(), lo.size(), &pi))) return rc;
            b.light_of = pi;
        }
        if ((rc = dev_copy(ctx, s->allocs, rec_leaf.data(), rec_leaf.size(), &p4))) return rc;
        b.place = p4;
        {
            std::vector<int> ids(tl.order.begin(), tl.order.begin() + N);
            const int* pi = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, ids.data(), ids.size(), &pi))) return rc;
            b.inst_id = pi;
        }
        b.inst_id_w = nullptr;
        if ((rc = dev_copy(ctx, s->allocs, (const float4*)tl.nodes.data(), 2 * (size_t)tl.node_count, &p4))) return rc;
        b.tlas = p4;
        // the compressed wide twin of the TLAS (instanceAccel 'cwbvh', cwbvh.ts:80-372 over
        // the same instance boxes) with the placements in its leaf order
        b.tlas_w = nullptr;
        b.place_w = nullptr;
        ptx_host::WideBvh wt = ptx_host::build_cwbvh(boxes.data(), N, ptx_host::kCwbvhCPrim);
        if (!wt.error && wt.node_count > 0) {
            std::vector<float4> rec_w(2 * (size_t)N);
            for (int i = 0; i < N; ++i) {
                rec_w[2 * (size_t)i] = rec[2 * (size_t)wt.order[i]];
                rec_w[2 * (size_t)i + 1] = rec[2 * (size_t)wt.order[i] + 1];
            }
            const uint4* u4 = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, rec_w.data(), rec_w.size(), &p4))) return rc;
            b.place_w = p4;
            std::vector<int> ids(wt.order.begin(), wt.order.begin() + N);
            const int* pid = nullptr;
            if ((rc = dev_copy(ctx, s->allocs, ids.data(), ids.size(), &pid))) return rc;
            b.inst_id_w = pid;
            if (bd.light_base >= 0) {
                std::vector<int> lo(N);
                for (int i = 0; i < N; ++i) lo[i] = bd.light_base + (int)wt.order[i];
                const int* pi = nullptr;
                if ((rc = dev_copy(ctx, s->allocs, lo.data(), lo.size(), &pi))) return rc;
                b.light_of_w = pi;
            }
            if ((rc = dev_copy(ctx, s->allocs, (const uint4*)wt.nodes.data(), 5 * (size_t)wt.node_count, &u4))) return rc;
            b.tlas_w = u4;
        }
        b.n_inst = N;
        b.proto_shape = bd.prototype_shape;
        b.proto_mesh = bd.prototype_ref;
        b.n_tlas = tl.node_count;
    }
    int rc;
    const DevMesh* dm = nullptr;
    const DevBatch* db = nullptr;
    if ((rc = dev_copy(ctx, s->allocs, meshes.data(), meshes.size(), &dm))) return rc;
    if ((rc = dev_copy(ctx, s->allocs, batches.data(), batches.size(), &db))) return rc;
    S.meshes = dm;
    S.batches = db;
    S.n_meshes = (int)meshes.size();
    S.n_batches = (int)batches.size();
    unsigned zero = 0;
    const unsigned* ef = nullptr;
    if ((rc = dev_copy(ctx, s->allocs, &zero, 1, &ef))) return rc;
    S.err_flags = (unsigned*)ef;
    for (int i = 0; i < d->n_regions; ++i) {
        const ptr_region& g = d->regions[i];
        const float* q = g.p;
        double mn[3], mx[3];
        if (g.shape == PTR_SHAPE_SPHERE) {
            for (int a = 0; a < 3; ++a) { mn[a] = (double)q[a] - q[3]; mx[a] = (double)q[a] + q[3]; }
        } else if (g.shape == PTR_SHAPE_BOX) {
            for (int a = 0; a < 3; ++a) { mn[a] = (double)q[a] - q[3 + a]; mx[a] = (double)q[a] + q[3 + a]; }
        } else if (g.shape == PTR_SHAPE_QUAD) {
            for (int a = 0; a < 3; ++a) {
                double c0 = q[a], c1 = c0 + q[3 + a], c2 = c0 + q[6 + a], c3 = c0 + q[3 + a] + q[6 + a];
                mn[a] = std::min(std::min(c0, c1), std::min(c2, c3));
                mx[a] = std::max(std::max(c0, c1), std::max(c2, c3));
            }
        } else {
            continue;
        }
        grow(mn, mx);
    }
    for (int a = 0; a < 3; ++a)
        S.sort_c[a] = world_lo[a] <= world_hi[a] ? (float)(0.5 * (world_lo[a] + world_hi[a])) : 0.0f;
    S.sort_c[3] = 0.0f;
    return PTR_OK;
}

// Region BVH over the bounded analytic regions (spheres, boxes, quads) when there are at
// least PTR_REGION_BVH_MIN of them (default 257; the reference tests every non-instanced
// primitive as one unrolled arm, and on B200 the linear scan by same-shape runs measured
// faster than this BVH beyond 200 spheres).  Planes, meshes and instanced batches stay in
// the ordered linear list.  Hits equal the linear scan's (same tie rule).
int upload_region_bvh(ptr_ctx* ctx, ptr_scene* s, const ptr_scene_desc* d) {
    DevScene& S = s->dev;
    int min_items = 257;
    if (const char* env = std::getenv("PTR_REGION_BVH_MIN")) min_items = std::atoi(env);
    std::vector<int> bounded, linear;
    std::vector<double> boxes;
    for (int i = 0; i < d->n_regions; ++i) {
        const ptr_region& g = d->regions[i];
        const float* q = g.p;
        double mn[3], mx[3];
        if (g.shape == PTR_SHAPE_SPHERE) {
            for (int a = 0; a < 3; ++a) { mn[a] = (double)q[a] - q[3]; mx[a] = (double)q[a] + q[3]; }
        } else if (g.shape == PTR_SHAPE_BOX) {
            for (int a = 0; a < 3; ++a) { mn[a] = (double)q[a] - q[3 + a]; mx[a] = (double)q[a] + q[3 + a]; }
        } else if (g.shape == PTR_SHAPE_QUAD) {
            for (int a = 0; a < 3; ++a) {
                double c0 = q[a], c1 = c0 + q[3 + a], c2 = c0 + q[6 + a], c3 = c0 + q[3 + a] + q[6 + a];
                mn[a] = std::min(std::min(c0, c1), std::min(c2, c3));
                mx[a] = std::max(std::max(c0, c1), std::max(c2, c3));
            }
        } else {
            linear.push_back(i);
            continue;
        }
        // a float-rounding margin so the (float) node boxes never cut the geometry
        for (int a = 0; a < 3; ++a) {
            double m = 1e-6 * (1.0 + std::max(std::fabs(mn[a]), std::fabs(mx[a])));
            boxes.push_back(mn[a] - m);
        }
        for (int a = 0; a < 3; ++a) {
            double m = 1e-6 * (1.0 + std::max(std::fabs(mn[a]), std::fabs(mx[a])));
            boxes.push_back(mx[a] + m);
        }
        bounded.push_back(i);
    }
    if ((int)bounded.size() < min_items) return PTR_OK;
    // reorder to (min.xyz, max.xyz) per item
    std::vector<double> b6(boxes.size());
    for (size_t k = 0; k < bounded.size(); ++k)
        for (int a = 0; a < 6; ++a) b6[6 * k + a] = boxes[6 * k + a];
    ptx_host::BinaryBvh bvh = ptx_host::build_bvh(b6.data(), (int)bounded.size(), ptx_host::kBvhLeafSize, false);
    std::vector<int> items(bounded.size());
    for (size_t k = 0; k < bounded.size(); ++k) items[k] = bounded[bvh.order[k]];
    int rc;
    const float4* nodes = nullptr;
    const int* it = nullptr;
    const int* lin = nullptr;
    if ((rc = dev_copy(ctx, s->allocs, (const float4*)bvh.nodes.data(), 2 * (size_t)bvh.node_count, &nodes))) return rc;
    if ((rc = dev_copy(ctx, s->allocs, items.data(), items.size(), &it))) return rc;
    if (!linear.empty() && (rc = dev_copy(ctx, s->allocs, linear.data(), linear.size(), &lin))) return rc;
    S.region_bvh = nodes;
    S.region_items = it;
    S.linear_regions = lin;
    S.n_linear = (int)linear.size();
    S.n_region_nodes = bvh.node_count;
    return PTR_OK;
}

// The first-hit pictures' FP64 sums (programs with AOVs), sized and cleared with the film.
int prepare_aov_film(ptr_program* p, const ptr_frame* f, size_t npix, cudaStream_t st) {
    ptr_ctx* ctx = p->ctx;
    if (p->desc.aovs) {
        if (!p->aov_sum || p->aov_n != npix) {
            if (p->aov_sum) cudaFree(p->aov_sum);
            p->aov_sum = nullptr;
            if (cudaMalloc(&p->aov_sum, npix * 6 * sizeof(double)) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, "AOV film allocation failed");
            p->aov_n = npix;
            CK(ctx, cudaMemsetAsync(p->aov_sum, 0, npix * 6 * sizeof(double), st));
        } else if (!f->accumulate) {
            CK(ctx, cudaMemsetAsync(p->aov_sum, 0, npix * 6 * sizeof(double), st));
        }
        p->pool.aov_sum = p->aov_sum;
    }
    return PTR_OK;
}

// Size (and clear unless accumulating) a program's FP64 film for a frame.
int prepare_film(ptr_program* p, const ptr_frame* f, cudaStream_t st) {
    ptr_ctx* ctx = p->ctx;
    const size_t npix = (size_t)f->width * f->height;
    if (p->fw != f->width || p->fh != f->height || !p->sum) {
        if (p->sum) cudaFree(p->sum);
        if (p->sumsq) cudaFree(p->sumsq);
        if (p->export_buf) cudaFree(p->export_buf);
        p->sum = p->sumsq = nullptr;
        p->export_buf = nullptr;
        if (cudaMalloc(&p->sum, npix * 3 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&p->sumsq, npix * 3 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&p->export_buf, npix * 3 * sizeof(float)) != cudaSuccess)
            return fail(ctx, PTR_E_NOMEM, "film allocation failed");
        p->fw = f->width;
        p->fh = f->height;
        p->nsamples = 0.0;
        CK(ctx, cudaMemsetAsync(p->sum, 0, npix * 3 * sizeof(double), st));
        CK(ctx, cudaMemsetAsync(p->sumsq, 0, npix * 3 * sizeof(double), st));
    } else if (!f->accumulate) {
        p->nsamples = 0.0;
        CK(ctx, cudaMemsetAsync(p->sum, 0, npix * 3 * sizeof(double), st));
        CK(ctx, cudaMemsetAsync(p->sumsq, 0, npix * 3 * sizeof(double), st));
    }
    if (int rc = prepare_aov_film(p, f, npix, st)) return rc;
    return PTR_OK;
}

// The scene-dependent pins of the equiangular site: the reference admits delta lights only
// (Validator.ts:506-540); PTR_EQUIANGULAR_AREA also admits quad and sphere lights.  The
// site covers finite lights, so a sampled environment is rejected (its medium-vertex NEE
// would be lost).
int check_equiangular(ptr_ctx* ctx, const ptr_program* p, const ptr_scene* s) {
    if (p->desc.light_tree && !s->dev.light_tree)
        return fail(ctx, PTR_E_INVALID, "lightSelection 'bvh' needs a scene uploaded with its light tree");
    if (p->desc.light_tree && p->desc.equiangular)
        return fail(ctx, PTR_E_INVALID, "lightSelection 'bvh' with mediumLightSampling 'equiangular' is reserved");
    if (s->dev.has_het && p->desc.equiangular)
        return fail(ctx, PTR_E_INVALID, "equiangular sampling through heterogeneous media is not available");
    if (s->dev.has_het && p->desc.color == PTR_COLOR_SPECTRAL)
        return fail(ctx, PTR_E_UNSUPPORTED, "heterogeneous media render in RGB only");
    if (p->desc.aovs && p->desc.color == PTR_COLOR_SPECTRAL)
        return fail(ctx, PTR_E_UNSUPPORTED, "AOVs are RGB only");
    if (p->desc.aovs & ~(PTR_AOV_ALBEDO | PTR_AOV_NORMAL)) return fail(ctx, PTR_E_INVALID, "unknown AOV bits");
    if (!p->desc.equiangular) return PTR_OK;
    if (s->n_lights == 0) return fail(ctx, PTR_E_INVALID, "mediumLightSampling 'equiangular' needs at least one light");
    if (p->desc.equiangular == PTR_EQUIANGULAR_DELTA && s->n_delta_lights != s->n_lights)
        return fail(ctx, PTR_E_INVALID, "mediumLightSampling 'equiangular' supports delta (point) lights only");
    if (s->env_samplable) return fail(ctx, PTR_E_INVALID, "mediumLightSampling 'equiangular' does not cover a sampled environment");
    return PTR_OK;
}

// A spectral program needs the scene's lifted colours; image environments are RGB only.
int check_color(ptr_ctx* ctx, const ptr_program* p, const ptr_scene* s) {
    if (p->desc.color != PTR_COLOR_SPECTRAL) return PTR_OK;
    if (!s->dev.spec_mats) return fail(ctx, PTR_E_INVALID, "measurement.color 'spectral' needs the scene's spectral tables (ptr_scene_desc.spectral)");
    if (s->dev.env_kind == PTR_ENV_IMAGE) return fail(ctx, PTR_E_UNSUPPORTED, "spectral rendering of image environments is not available");
    return PTR_OK;
}

int render_impl(ptr_program* p, ptr_scene* s, const ptr_frame* f, float* samples_dev) {
    ptr_ctx* ctx = p->ctx;
    if (int rc = check_color(ctx, p, s)) return rc;
    if (f->width <= 0 || f->height <= 0 || f->spp <= 0) return fail(ctx, PTR_E_INVALID, "frame: width, height and spp must be positive");
    if (s->ctx != ctx) return fail(ctx, PTR_E_INVALID, "scene belongs to another context");
    if (int rc = check_equiangular(ctx, p, s)) return rc;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t npix = (size_t)f->width * f->height;
    if (p->fw != f->width || p->fh != f->height || !p->sum) {
        if (p->sum) cudaFree(p->sum);
        if (p->sumsq) cudaFree(p->sumsq);
        if (p->export_buf) cudaFree(p->export_buf);
        p->sum = p->sumsq = nullptr;
        p->export_buf = nullptr;
        if (cudaMalloc(&p->sum, npix * 3 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&p->sumsq, npix * 3 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&p->export_buf, npix * 3 * sizeof(float)) != cudaSuccess)
            return fail(ctx, PTR_E_NOMEM, "film allocation failed");
        p->fw = f->width;
        p->fh = f->height;
        p->nsamples = 0.0;
        CK(ctx, cudaMemsetAsync(p->sum, 0, npix * 3 * sizeof(double), st));
        CK(ctx, cudaMemsetAsync(p->sumsq, 0, npix * 3 * sizeof(double), st));
    } else if (!f->accumulate) {
        p->nsamples = 0.0;
        CK(ctx, cudaMemsetAsync(p->sum, 0, npix * 3 * sizeof(double), st));
        CK(ctx, cudaMemsetAsync(p->sumsq, 0, npix * 3 * sizeof(double), st));
    }
    if (int rc = prepare_aov_film(p, f, npix, st)) return rc;
    const long long total = (long long)npix * f->spp;
    // capacity: whole sample passes when a pass fits the pool, else a chunk of pixels
    long long cap_max = ctx->tune.capacity > 0 ? ctx->tune.capacity : (1ll << 24);
    if (const char* env = std::getenv("PTR_CAPACITY")) cap_max = std::atoll(env);
    if (cap_max < 1024) cap_max = 1024;
    long long cap;
    if ((long long)npix <= cap_max) cap = (cap_max / (long long)npix) * (long long)npix;
    else cap = cap_max;
    if (cap > total) cap = total;
    const bool slot2 = p->desc.equiangular != 0;
    const bool spectral = p->desc.color == PTR_COLOR_SPECTRAL;
    if (p->capacity < cap || (slot2 && !p->pool.sh2_o) || (spectral && !p->pool.wl)) {
        int rc = alloc_pool(p, (int)std::max<long long>(cap, p->capacity), slot2 || p->pool.sh2_o,
                            p->pool.l_rem != nullptr, spectral || p->pool.wl);
        if (rc) return rc;
    }
    if (p->desc.aovs && !p->pool.aov) {   // two float4 per path slot; a captured graph predates them
        void* a = nullptr;
        if (cudaMalloc(&a, (size_t)p->capacity * 32) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, "AOV pool allocation failed");
        p->pool_allocs.push_back(a);
        p->pool.aov = (float4*)a;
        if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
    }
    p->pool.aov_sum = p->desc.aovs ? p->aov_sum : nullptr;
    if (!p->fp_dev) CK(ctx, cudaMalloc(&p->fp_dev, sizeof(FrameParams)));
    // The frame's parameters travel as a kernel argument into a device block: no host
    // synchronisation, and the captured graph (which reads the block) stays valid.
    FrameParams F;
    F.width = f->width;
    F.height = f->height;
    F.spp = f->spp;
    F.first_sample = f->first_sample;
    F.salt = f->reset_salt;
    F.px_off = f->pixel_offset[0];
    F.py_off = f->pixel_offset[1];
    F.img_w = f->image_size[0] > 0 ? f->image_size[0] : f->width;
    F.img_h = f->image_size[1] > 0 ? f->image_size[1] : f->height;
    F.total = total;
    F.capacity = (int)cap;
    F.cam = f->camera;
    F.wavelengths = p->desc.wavelengths;
    F.lambda_min = p->desc.lambda_min;
    F.lambda_max = p->desc.lambda_max;
    k_set_frame<<<1, 1, 0, st>>>(p->fp_dev, F);
    CK(ctx, cudaGetLastError());
    CK(ctx, cudaMemsetAsync(p->pool.wave, 0, 64, st));
    CK(ctx, cudaMemsetAsync(p->pool.stats, 0, 64, st));
    CK(ctx, cudaMemsetAsync(p->pool.cnt, 0, 64, st));
    const int iters = wave_iterations(p, s);
    const long long waves = (total + cap - 1) / cap;
    const int n_sm = device_sms(ctx->device);
    const bool profiling = (p->profile_next & PTR_PROFILE_TIMING) != 0;
    const bool counting = (p->profile_next & PTR_PROFILE_WORK) != 0;
    p->last_scene = s;
    if (counting) {
        if (!p->work_dev) CK(ctx, cudaMalloc(&p->work_dev, 64));
        CK(ctx, cudaMemsetAsync(p->work_dev, 0, 64, st));
        p->work_valid = 1;
    } else {
        p->work_valid = 0;
    }
    const bool use_graph = std::getenv("PTR_NO_GRAPH") == nullptr && !profiling && !counting;
    if (use_graph) {
        const void* cur_spec = p->spec.scene_id == s->id ? p->spec.shade : nullptr;
        if (!p->graph || p->graph_scene != s || p->graph_scene_id != s->id || p->graph_w != f->width ||
            p->graph_h != f->height || p->graph_iters != iters || p->graph_samples != samples_dev ||
            p->graph_spec != cur_spec || std::memcmp(&p->graph_tune, &ctx->tune, sizeof(ptr_tuning)) != 0) {
            if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
            cudaGraph_t g = nullptr;
            launch_wave(p, s, st, iters, samples_dev, n_sm, nullptr, true, true);   // occupancy queries, outside capture
            CK(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            launch_wave(p, s, st, iters, samples_dev, n_sm);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (ce != cudaSuccess) return cuda_fail(ctx, ce, "graph capture");
            ce = cudaGraphInstantiate(&p->graph, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return cuda_fail(ctx, ce, "graph instantiate");
            p->graph_scene = s;
            p->graph_scene_id = s->id;
            p->graph_spec = cur_spec;
            p->graph_w = f->width;
            p->graph_h = f->height;
            p->graph_iters = iters;
            p->graph_samples = samples_dev;
            p->graph_tune = ctx->tune;
        }
        for (long long w = 0; w < waves; ++w) CK(ctx, cudaGraphLaunch(p->graph, st));
    } else if (profiling) {
        std::vector<ProfRec> prof;
        prof.reserve((size_t)waves * (iters * 5 + 2));
        for (long long w = 0; w < waves; ++w) launch_wave(p, s, st, iters, samples_dev, n_sm, &prof);
        CK(ctx, cudaGetLastError());
        CK(ctx, cudaStreamSynchronize(st));
        for (int k = 0; k < PTR_PROFILE_CLASSES; ++k) { p->prof_ms[k] = 0.f; p->prof_launches[k] = 0; }
        for (ProfRec& r : prof) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r.a, r.b);
            p->prof_ms[r.cls] += ms;
            p->prof_launches[r.cls] += r.n;
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        p->profile_next = 0;
    } else {
        for (long long w = 0; w < waves; ++w) launch_wave(p, s, st, iters, samples_dev, n_sm);
        CK(ctx, cudaGetLastError());
        p->profile_next = 0;
    }
    p->nsamples += (double)f->spp;
    return PTR_OK;
}


// ---- per-scene kernels (ptr_specialize) ------------------------------------------------
// NVRTC, opened at run time so that the library needs neither it nor libcuda to load.
struct Nvrtc {
    using Prog = void*;
    int (*create)(Prog*, const char*, const char*, int, const char* const*, const char* const*) = nullptr;
    int (*add_name)(Prog, const char*) = nullptr;
    int (*compile)(Prog, int, const char* const*) = nullptr;
    int (*log_size)(Prog, size_t*) = nullptr;
    int (*log)(Prog, char*) = nullptr;
    int (*lowered)(Prog, const char*, const char**) = nullptr;
    int (*cubin_size)(Prog, size_t*) = nullptr;
    int (*cubin)(Prog, char*) = nullptr;
    int (*destroy)(Prog*) = nullptr;
    bool ok = false;
    std::string why;
};
Nvrtc& nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {std::getenv("PTR_NVRTC_LIB"), "libnvrtc.so.12", "libnvrtc.so",
                               "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* nm : names)
            if (nm && (h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) { n.why = "NVRTC (libnvrtc.so.12) not found"; return; }
        auto sym = [&](auto& fp, const char* name) { fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(h, name)); return fp != nullptr; };
        n.ok = sym(n.create, "nvrtcCreateProgram") && sym(n.add_name, "nvrtcAddNameExpression") &&
               sym(n.compile, "nvrtcCompileProgram") && sym(n.log_size, "nvrtcGetProgramLogSize") &&
               sym(n.log, "nvrtcGetProgramLog") && sym(n.lowered, "nvrtcGetLoweredName") &&
               sym(n.cubin_size, "nvrtcGetCUBINSize") && sym(n.cubin, "nvrtcGetCUBIN") &&
               sym(n.destroy, "nvrtcDestroyProgram");
        if (!n.ok) n.why = "NVRTC lacks an entry point this build uses";
    });
    return n;
}
// The device sources beside the library: <package>/csrc/device and <package>/../include
// (PTR_DEVICE_SRC / PTR_INCLUDE override).
std::string lib_dir() {
    Dl_info info{};
    if (!dladdr((void*)&nvrtc, &info) || !info.dli_fname) return ".";
    std::string f = info.dli_fname;
    size_t k = f.find_last_of('/');
    return k == std::string::npos ? std::string(".") : f.substr(0, k);
}
struct SpecModule { cudaLibrary_t lib = nullptr; const void* closest = nullptr; const void* shade = nullptr; const void* shadow = nullptr; };
// The occupant census a set of kernels is compiled for: material models, light kinds,
// environment kinds and region shapes present (bit masks), the regions in order when
// there are at most 16 (0 otherwise), the light tree, the direct-lighting mode, media,
// colour model, and whether the kernels are the batched variants.
struct Census {
    unsigned mats = 0, lights = 0, envs = 0, shapes = 0;
    int nregions = 0;
    unsigned long long shape_code = 0;
    bool tree = false, media = false, spectral = false, batch = false;
    bool adj = false;                  // the replay's kernels (ADJ = true) instead of the forward's
    int direct = 0;
};
Census census_of(const ptr_program* p, const ptr_scene* sc) {
    Census c;
    c.mats = sc->spec_mats;
    c.lights = sc->spec_lights;
    c.envs = sc->spec_envs;
    c.shapes = sc->spec_shapes;
    c.nregions = sc->spec_nregions;
    c.shape_code = sc->spec_shape_code;
    c.tree = p->desc.light_tree != 0;
    c.media = sc->has_media != 0;
    c.spectral = p->desc.color == PTR_COLOR_SPECTRAL;
    c.direct = p->desc.direct;
    return c;
}
// The union census of a job mix (the batched kernels serve every job of it): masks OR-ed,
// no region unrolling (the jobs' region lists differ).
Census census_of_batch(const ptr_batch_job* jobs, int n) {
    Census c;
    c.batch = true;
    for (int j = 0; j < n; ++j) {
        const Census k = census_of(jobs[j].prog, jobs[j].scene);
        c.mats |= k.mats;
        c.lights |= k.lights;
        c.envs |= k.envs;
        c.shapes |= k.shapes;
        c.tree = c.tree || k.tree;
        c.media = c.media || k.media;
        c.direct = k.direct;
    }
    return c;
}
std::vector<std::string> census_options(const Census& c) {
    return {"-DPTR_SPEC_MATS=" + std::to_string(c.mats) + "u",
            "-DPTR_SPEC_LIGHTS=" + std::to_string(c.lights) + "u",
            "-DPTR_SPEC_ENVS=" + std::to_string(c.envs) + "u",
            "-DPTR_SPEC_SHAPES=" + std::to_string(c.shapes) + "u",
            "-DPTR_SPEC_NREGIONS=" + std::to_string(c.nregions),
            "-DPTR_SPEC_SHAPE_CODE=" + std::to_string(c.shape_code) + "ull",
            std::string("-DPTR_SPEC_TREE=") + (c.tree ? "1" : "0")};
}
std::string census_key(const Census& c) {
    std::string k;
    for (const auto& o : census_options(c)) k += o + "\n";
    return k + std::to_string(c.direct) + (c.media ? "m" : "-") + (c.spectral ? "s" : "-") + (c.batch ? "b" : "-") +
           (c.adj ? "a" : "-");
}
// Compile (or fetch) the closest-hit, shading and shadow kernels for a census.  Modules are
// cached by census for the process, so equal scenes (and equal mixes) share one module.
int spec_compile(ptr_ctx* ctx, const Census& c, SpecModule& out, bool& compiled) {
    compiled = false;
    static std::mutex mu;
    static std::map<std::string, SpecModule> cache;
    Nvrtc& nv = nvrtc();
    if (!nv.ok) return fail(ctx, PTR_E_UNSUPPORTED, "ptr_specialize: " + nv.why);
    const char* col = c.spectral ? "ptx::s4" : "ptx::f3";
    const char* md = c.media ? "true" : "false";
    const char* bt = c.batch ? "true" : "false";
    const std::string n_closest = std::string("ptx::k_closest<false, ") + bt + ">";
    const char* adj = c.adj ? "true" : "false";
    const std::string n_shade = std::string("ptx::k_shade<") + col + ", " + std::to_string(c.direct) + ", " + md +
                                ", " + bt + ", " + adj + ">";
    const std::string n_shadow = std::string("ptx::k_shadow<") + col + ", " + md + ", false, " + bt + ", " + adj + ">";
    const std::string dir = lib_dir();
    const char* dev_env = std::getenv("PTR_DEVICE_SRC");
    const char* inc_env = std::getenv("PTR_INCLUDE");
    std::vector<std::string> opts = {
        "-arch=sm_100a", "-std=c++17", "-fmad=false", "-lineinfo",
        "-default-device",   // the public header's host prototypes, declared only
        std::string("-I") + (dev_env ? dev_env : dir + "/csrc/device"),
        std::string("-I") + (inc_env ? inc_env : dir + "/../include")};
    for (const auto& o : census_options(c)) opts.push_back(o);
    // PTR_SPEC_DEFINES: extra space-separated -D options (the wide-math parity build)
    if (const char* extra = std::getenv("PTR_SPEC_DEFINES")) {
        std::string tok;
        for (const char* q = extra;; ++q) {
            if (*q == ' ' || *q == '\0') {
                if (tok.rfind("-D", 0) == 0) opts.push_back(tok);
                tok.clear();
                if (*q == '\0') break;
            } else {
                tok += *q;
            }
        }
    }
    std::string key;
    for (const auto& o : opts) key += o + "\n";
    key += n_closest + "\n" + n_shade + "\n" + n_shadow;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) { out = it->second; return PTR_OK; }
    static const char* kSource =
        "typedef signed char int8_t; typedef unsigned char uint8_t; typedef short int16_t;\n"
        "typedef unsigned short uint16_t; typedef int int32_t; typedef unsigned int uint32_t;\n"
        "typedef long long int64_t; typedef unsigned long long uint64_t;\n"
        "#include \"wavefront.cuh\"\n";
    Nvrtc::Prog prog = nullptr;
    if (nv.create(&prog, kSource, "ptr_specialize.cu", 0, nullptr, nullptr) != 0)
        return fail(ctx, PTR_E_CUDA, "ptr_specialize: nvrtcCreateProgram failed");
    nv.add_name(prog, n_closest.c_str());
    nv.add_name(prog, n_shade.c_str());
    nv.add_name(prog, n_shadow.c_str());
    std::vector<const char*> argv;
    for (const auto& o : opts) argv.push_back(o.c_str());
    const int rc = nv.compile(prog, (int)argv.size(), argv.data());
    if (rc != 0) {
        size_t n = 0;
        nv.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) nv.log(prog, &log[0]);
        nv.destroy(&prog);
        return fail(ctx, PTR_E_CUDA, "ptr_specialize: NVRTC compile failed:\n" + log.substr(0, 4000));
    }
    size_t nbin = 0;
    nv.cubin_size(prog, &nbin);
    std::vector<char> bin(nbin);
    nv.cubin(prog, bin.data());
    const char *l_closest = nullptr, *l_shade = nullptr, *l_shadow = nullptr;
    nv.lowered(prog, n_closest.c_str(), &l_closest);
    nv.lowered(prog, n_shade.c_str(), &l_shade);
    nv.lowered(prog, n_shadow.c_str(), &l_shadow);
    const std::string s_closest = l_closest ? l_closest : "", s_shade = l_shade ? l_shade : "",
                      s_shadow = l_shadow ? l_shadow : "";
    nv.destroy(&prog);
    SpecModule m;
    cudaError_t e = cudaLibraryLoadData(&m.lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ptr_specialize: cudaLibraryLoadData");
    cudaKernel_t kc = nullptr, ks = nullptr, kw = nullptr;
    if ((e = cudaLibraryGetKernel(&kc, m.lib, s_closest.c_str())) != cudaSuccess ||
        (e = cudaLibraryGetKernel(&ks, m.lib, s_shade.c_str())) != cudaSuccess ||
        (e = cudaLibraryGetKernel(&kw, m.lib, s_shadow.c_str())) != cudaSuccess)
        return cuda_fail(ctx, e, "ptr_specialize: cudaLibraryGetKernel");
    m.closest = (const void*)kc;
    m.shade = (const void*)ks;
    m.shadow = (const void*)kw;
    cache[key] = m;
    out = m;
    compiled = true;
    return PTR_OK;
}

}  // namespace

extern "C" {

int ptr_abi_version(void) { return PTR_ABI_VERSION; }

int ptr_create(int device_ordinal, ptr_ctx** out) {
    if (!out) return PTR_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return PTR_E_CUDA;
    if (device_ordinal < 0 || device_ordinal >= n) return PTR_E_INVALID;
    ptr_ctx* c = new ptr_ctx();
    c->device = device_ordinal;
    if (cudaSetDevice(device_ordinal) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return PTR_E_CUDA;
    }
    // the counting sort's scan stages its whole table in shared memory (above the 48 KB default)
    if (cudaFuncSetAttribute((const void*)k_sort_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSortScanSmem) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return PTR_E_CUDA;
    }
    *out = c;
    return PTR_OK;
}

int ptr_destroy(ptr_ctx* ctx) {
    if (!ctx) return PTR_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->batch) ptr_free_program(ctx->batch);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PTR_OK;
}

const char* ptr_last_error(const ptr_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

namespace {
// A field program is safe to interpret: known opcodes with their immediates inside the
// table, every pop backed by the stack, the stack within PTR_FIELD_MAX_STACK, and END
// reached with exactly one value.
bool field_program_ok(const uint32_t* code, int n, int start) {
    if (start < 0 || start >= n) return false;
    int sp = 0;
    for (int pc = start; pc < n;) {
        const uint32_t op = code[pc++];
        int pop = 0, push = 0;
        switch (op) {
            case PTR_FOP_END: return sp == 1;
            case PTR_FOP_CONST: if (pc + 3 > n) return false; pc += 3; push = 1; break;
            case PTR_FOP_P: push = 1; break;
            case PTR_FOP_SWZ: if (pc + 1 > n || code[pc] > 2u) return false; pc += 1; pop = 1; push = 1; break;
            case PTR_FOP_ADD: case PTR_FOP_SUB: case PTR_FOP_MUL: case PTR_FOP_DIV:
            case PTR_FOP_POW: case PTR_FOP_MIN: case PTR_FOP_MAX: case PTR_FOP_MOD: case PTR_FOP_STEP:
            case PTR_FOP_DOT: pop = 2; push = 1; break;
            case PTR_FOP_CLAMP: case PTR_FOP_MIX: case PTR_FOP_SMOOTHSTEP: case PTR_FOP_VEC3: pop = 3; push = 1; break;
            default:
                if (op >= PTR_FOP_COUNT) return false;
                pop = 1; push = 1;   // the unary built-ins and LENGTH
        }
        if (sp < pop) return false;
        sp += push - pop;
        if (sp > PTR_FIELD_MAX_STACK) return false;
    }
    return false;
}
}  // namespace

namespace {
// The scene description's own consistency: table sizes and pointers, region shapes,
// materials and parameters, light kinds, regions and selection pdfs, coefficient-field
// programs, instance lights and the light tree.  Every entry point that takes a
// ptr_scene_desc runs it before copying anything to the device.
int check_scene_desc(const ptr_scene_desc* d, std::string& why) {
    auto bad = [&why](const std::string& m) { why = m; return PTR_E_INVALID; };
    if (d->abi_version != PTR_ABI_VERSION) return bad("scene: ABI version mismatch");
    if (d->n_regions < 0 || d->n_materials <= 0 || d->n_lights < 0) return bad("scene: bad table sizes");
    if ((d->n_regions > 0 && !d->regions) || !d->materials || (d->n_lights > 0 && !d->lights))
        return bad("scene: a table with entries has a null pointer");
    for (int i = 0; i < d->n_regions; ++i) {
        const ptr_region& g = d->regions[i];
        if (g.shape < 0 || g.shape > PTR_SHAPE_INSTANCES) return bad("scene: region " + std::to_string(i) + " has an unknown shape");
        if (g.material < 0 || g.material >= d->n_materials) return bad("scene: region " + std::to_string(i) + " has a material out of range");
        if (g.shape == PTR_SHAPE_MESH && (g.ref < 0 || g.ref >= d->n_meshes)) return bad("scene: mesh region references a missing mesh");
        if (g.shape == PTR_SHAPE_INSTANCES && (g.ref < 0 || g.ref >= d->n_batches)) return bad("scene: instanced region references a missing batch");
        for (int k = 0; k < 15; ++k)
            if (!std::isfinite(g.p[k])) return bad("scene: region " + std::to_string(i) + " has a non-finite parameter");
    }
    for (int i = 0; i < d->n_lights; ++i) {
        const ptr_light& l = d->lights[i];
        if (l.region >= d->n_regions) return bad("scene: light region out of range");
        if (!(l.select_pdf > 0.0f) || !std::isfinite(l.select_pdf)) return bad("scene: light selection pdf must be positive");
        if (l.kind < PTR_LIGHT_QUAD || l.kind > PTR_LIGHT_MESH) return bad("scene: light " + std::to_string(i) + " has an unknown kind");
        if (l.kind == PTR_LIGHT_MESH) {
            const int mi = (int)l.p[0];
            if (l.region < 0 || d->regions[l.region].shape != PTR_SHAPE_MESH || d->regions[l.region].ref != mi ||
                (float)mi != l.p[0] || !(l.p[12] > 0.0f) || !std::isfinite(l.p[12]))
                return bad("scene: mesh light " + std::to_string(i) + " must name its mesh region, its mesh and a positive area");
        }
    }
    if (d->ambient_material >= d->n_materials) return bad("scene: ambient material out of range");
    bool has_het = false;
    for (int i = 0; i < d->n_materials; ++i) {
        const ptr_material& m = d->materials[i];
        if (!m.field_a && !m.field_s) continue;
        has_het = true;
        if (!(m.flags & PTR_MATF_MEDIUM) || !(m.majorant > 0.0f) || !std::isfinite(m.majorant) || !d->field_code ||
            (m.field_a && !field_program_ok(d->field_code, d->n_field_code, m.field_a - 1)) ||
            (m.field_s && !field_program_ok(d->field_code, d->n_field_code, m.field_s - 1)))
            return bad("scene: material " + std::to_string(i) +
                                                " has a malformed coefficient field or no positive majorant");
    }
    for (int b = 0; b < d->n_batches; ++b) {
        const ptr_batch_desc& bd = d->batches[b];
        if (bd.light_base >= 0 && ((long long)bd.light_base + bd.n_instances > d->n_lights || bd.prototype_shape != PTR_SHAPE_SPHERE))
            return bad("scene: instance lights of batch " + std::to_string(b) + " exceed the light table");
    }
    if (d->n_tree_nodes != 0) {
        // a preorder tree of one light per leaf: every link points forward inside the
        // table, every light is reached once, and its trail lands on its own leaf
        const int nn = d->n_tree_nodes;
        if (d->n_lights <= 0 || nn != 2 * d->n_lights - 1 || !d->light_tree || !d->light_trails)
            return bad("scene: the light tree must hold 2 n_lights - 1 nodes and the trails");
        std::vector<char> seen(d->n_lights, 0);
        for (int i = 0; i < nn; ++i) {
            const float link = d->light_tree[8 * (size_t)i + 7];
            const int li = (int)link;
            if ((float)li != link || (li >= 0 && (li <= i + 1 || li >= nn || i + 1 >= nn)) ||
                (li < 0 && (-li - 1 >= d->n_lights || seen[-li - 1]++)))
                return bad("scene: malformed light tree node " + std::to_string(i));
        }
        for (int l = 0; l < d->n_lights; ++l) {
            uint32_t tw = d->light_trails[2 * (size_t)l];
            int ni = 0, lvl = 0;
            for (; lvl < 48 && d->light_tree[8 * (size_t)ni + 7] >= 0.0f; ++lvl) {
                if (lvl == 24) tw = d->light_trails[2 * (size_t)l + 1];
                ni = (tw & 1u) ? (int)d->light_tree[8 * (size_t)ni + 7] : ni + 1;
                tw >>= 1u;
            }
            if (d->light_tree[8 * (size_t)ni + 7] != (float)(-(l + 1)))
                return bad("scene: the trail of light " + std::to_string(l) + " misses its leaf");
        }
    }
    return PTR_OK;
}
}  // namespace

static int upload_scene(ptr_ctx* ctx, const ptr_scene_desc* d, const ptr_rails* rails, ptr_scene** out);

int ptr_upload_scene(ptr_ctx* ctx, const ptr_scene_desc* d, ptr_scene** out) { return upload_scene(ctx, d, nullptr, out); }

int ptr_upload_scene_rails(ptr_ctx* ctx, const ptr_scene_desc* d, const ptr_rails* r, ptr_scene** out) {
    if (!ctx || !d || !r || !out) return fail(ctx, PTR_E_INVALID, "null argument");
    if (r->n_meshes != d->n_meshes || r->n_batches != d->n_batches || r->n_mesh_lights < 0 ||
        (r->n_meshes > 0 && !r->meshes) || (r->n_batches > 0 && !r->batches) || (r->n_mesh_lights > 0 && !r->mesh_lights))
        return fail(ctx, PTR_E_INVALID, "rails: one rail slot per mesh and per batch of the description");
    if (r->vertices_texels < 0 || r->indices_texels < 0 || r->nodes_texels < 0 || r->records_texels < 0 ||
        (r->vertices_texels > 0 && !r->vertices) || (r->indices_texels > 0 && !r->indices) ||
        (r->nodes_texels > 0 && !r->nodes) || (r->records_texels > 0 && !r->records))
        return fail(ctx, PTR_E_INVALID, "rails: a channel with texels has a null pointer");
    return upload_scene(ctx, d, r, out);
}

static int upload_scene(ptr_ctx* ctx, const ptr_scene_desc* d, const ptr_rails* rails, ptr_scene** out) {
    if (!ctx || !d || !out) return fail(ctx, PTR_E_INVALID, "null argument");
    *out = nullptr;
    std::string why;
    if (int rc = check_scene_desc(d, why)) return fail(ctx, rc, why);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, PTR_E_CUDA, "cudaSetDevice");
    ptr_scene* s = new ptr_scene();
    s->ctx = ctx;
    DevScene& S = s->dev;
    int rc = PTR_OK;
    std::vector<int> lor(d->n_regions > 0 ? d->n_regions : 1, -1);
    for (int i = 0; i < d->n_lights; ++i)
        if (d->lights[i].region >= 0) lor[d->lights[i].region] = i;
    if ((rc = dev_copy(ctx, s->allocs, d->regions, (size_t)d->n_regions, &S.regions)) ||
        (rc = dev_copy(ctx, s->allocs, d->materials, (size_t)d->n_materials, &S.materials)) ||
        (rc = dev_copy(ctx, s->allocs, d->lights, (size_t)d->n_lights, &S.lights)) ||
        (rc = dev_copy(ctx, s->allocs, lor.data(), lor.size(), &S.light_of_region))) {
        ptr_free_scene(s);
        return rc;
    }
    S.light_tree = nullptr;
    S.light_trails = nullptr;
    S.field_code = nullptr;
    bool has_het = false;
    for (int i = 0; i < d->n_materials; ++i) has_het |= d->materials[i].field_a || d->materials[i].field_s;
    S.has_het = has_het ? 1 : 0;
    if (has_het && (rc = dev_copy(ctx, s->allocs, d->field_code, (size_t)d->n_field_code, &S.field_code))) {
        ptr_free_scene(s);
        return rc;
    }
    if (d->n_tree_nodes > 0 &&
        ((rc = dev_copy(ctx, s->allocs, (const float4*)d->light_tree, 2 * (size_t)d->n_tree_nodes, &S.light_tree)) ||
         (rc = dev_copy(ctx, s->allocs, (const uint2*)d->light_trails, (size_t)d->n_lights, &S.light_trails)))) {
        ptr_free_scene(s);
        return rc;
    }
    S.n_regions = d->n_regions;
    S.n_materials = d->n_materials;
    S.n_lights = d->n_lights;
    S.ambient_material = d->ambient_material;
    bool media = d->ambient_material >= 0 && (d->materials[d->ambient_material].flags & PTR_MATF_MEDIUM);
    for (int i = 0; i < d->n_materials; ++i)
        if (d->materials[i].flags & PTR_MATF_MEDIUM) media = true;
    S.has_media = media ? 1 : 0;
    s->has_media = S.has_media;
    s->n_lights = d->n_lights;
    s->h_materials.assign(d->materials, d->materials + d->n_materials);
    s->h_regions.assign(d->regions, d->regions + d->n_regions);
    for (int i = 0; i < d->n_lights; ++i) s->n_delta_lights += d->lights[i].kind == PTR_LIGHT_POINT ? 1 : 0;
    s->env_samplable = d->env.kind != PTR_ENV_NONE && d->env.sample_as_light;
    S.env_kind = d->env.kind;
    S.env_samplable = d->env.kind != PTR_ENV_NONE && d->env.sample_as_light;
    S.env_select_live = S.env_samplable && d->n_lights > 0;
    if (d->spectral) {   // the lifted colours and the sensor tables of the spectral model
        const ptr_spectral_desc* sp = d->spectral;
        if (!sp->materials || !sp->curves || (d->n_lights > 0 && !sp->lights) || !(sp->cie_y_integral > 0.0f)) {
            ptr_free_scene(s);
            return fail(ctx, PTR_E_INVALID, "scene: incomplete spectral tables");
        }
        const float4* curves = nullptr;
        if ((rc = dev_copy(ctx, s->allocs, sp->materials, (size_t)d->n_materials, &S.spec_mats)) ||
            (rc = dev_copy(ctx, s->allocs, sp->lights, (size_t)d->n_lights, &S.spec_lights)) ||
            (rc = dev_copy(ctx, s->allocs, (const float4*)sp->curves, (size_t)95, &curves))) {
            ptr_free_scene(s);
            return rc;
        }
        S.spec_curves = curves;
        S.spec_env = sp->env;
        for (int k = 0; k < 9; ++k) S.spec_m[k] = sp->xyz_to_rgb[k];
        S.spec_y = sp->cie_y_integral;
    }
    for (int k = 0; k < 4; ++k) S.env_color[k] = d->env.color[k];
    S.env_intensity = d->env.intensity;
    S.env_select_prob = d->env.select_prob;
    S.env_rotation = d->env.rotation;
    if (d->env.kind == PTR_ENV_IMAGE) {
        if (d->env.width <= 0 || d->env.height <= 0 || !d->env.radiance || !d->env.marginal || !d->env.conditional) {
            ptr_free_scene(s);
            return fail(ctx, PTR_E_INVALID, "scene: image environment without its table");
        }
        S.env_w = d->env.width;
        S.env_h = d->env.height;
        const float* m = nullptr;
        if ((rc = dev_copy(ctx, s->allocs, (const float4*)d->env.radiance, (size_t)S.env_w * S.env_h, &S.env_map)) ||
            (rc = dev_copy(ctx, s->allocs, d->env.marginal, (size_t)S.env_h, &S.env_marg)) ||
            (rc = dev_copy(ctx, s->allocs, d->env.conditional, (size_t)S.env_h * S.env_w, &m))) {
            ptr_free_scene(s);
            return rc;
        }
        S.env_cond = m;
    }
    rc = upload_accels(ctx, s, d, rails);
    if (!rc) rc = upload_region_bvh(ctx, s, d);
    if (!rc && !S.region_bvh && d->n_regions > 0) {   // the scan's same-shape runs
        std::vector<int4> runs;
        for (int i = 0; i < d->n_regions; ++i) {
            const int sh = d->regions[i].shape;
            if (!runs.empty() && runs.back().x == sh) runs.back().z++;
            else runs.push_back(make_int4(sh, i, 1, 0));
        }
        if ((rc = dev_copy(ctx, s->allocs, runs.data(), runs.size(), &S.region_runs)) == PTR_OK) S.n_runs = (int)runs.size();
    }
    if (!rc) {
        // the refilling closest-hit loop's scene form: analytic regions and exactly one
        // acceleration region, an instanced mesh batch, with no region BVH
        int accel_regions = 0, flat = -1;
        for (int i = 0; i < d->n_regions; ++i) {
            if (d->regions[i].shape < PTR_SHAPE_MESH) continue;
            ++accel_regions;
            if (d->regions[i].shape == PTR_SHAPE_INSTANCES && d->batches[d->regions[i].ref].prototype_shape == PTR_SHAPE_MESH)
                flat = i;
        }
        s->dev.flat_region = (accel_regions == 1 && !s->dev.region_bvh) ? flat : -1;
        // occupant census for ptr_specialize
        static std::atomic<uint64_t> next_id{1};
        s->id = next_id++;
        for (int i = 0; i < d->n_materials; ++i) s->spec_mats |= 1u << (d->materials[i].model & 31);
        for (int i = 0; i < d->n_lights; ++i) s->spec_lights |= 1u << (d->lights[i].kind & 31);
        s->spec_envs = 1u << (d->env.kind & 31);
        for (int i = 0; i < d->n_regions; ++i) s->spec_shapes |= 1u << (d->regions[i].shape & 31);
        // up to 16 regions unroll in region order even where a region BVH was built: the
        // BVH walk's tie rule (lower region index wins) makes both give the same hits
        if (d->n_regions > 0 && d->n_regions <= 16) {
            s->spec_nregions = d->n_regions;
            for (int i = 0; i < d->n_regions; ++i)
                s->spec_shape_code |= (unsigned long long)(d->regions[i].shape & 15) << (4 * i);
        }
    }
    if (rc) {
        ptr_free_scene(s);
        return rc;
    }
    *out = s;
    return PTR_OK;
}

int ptr_free_scene(ptr_scene* s) {
    if (!s) return PTR_E_INVALID;
    if (s->ctx) {
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
    }
    for (void* a : s->allocs) cudaFree(a);
    delete s;
    return PTR_OK;
}

int ptr_compile(ptr_ctx* ctx, const ptr_program_desc* d, ptr_program** out) {
    if (!ctx || !d || !out) return fail(ctx, PTR_E_INVALID, "null argument");
    *out = nullptr;
    if (d->abi_version != PTR_ABI_VERSION) return fail(ctx, PTR_E_INVALID, "program: ABI version mismatch");
    if (d->max_bounces < 0 || d->max_bounces > 4096) return fail(ctx, PTR_E_INVALID, "program: maxBounces out of range");
    if (d->direct < PTR_DIRECT_NONE || d->direct > PTR_DIRECT_MIS) return fail(ctx, PTR_E_INVALID, "program: unknown directLighting");
    if (d->rr_start >= 0 && !(d->rr_max_survival > 0.0f && d->rr_max_survival <= 1.0f))
        return fail(ctx, PTR_E_INVALID, "program: russianRoulette.maxSurvival must be in (0, 1]");
    if (d->max_null_crossings < 0 || d->max_null_crossings > 4096) return fail(ctx, PTR_E_INVALID, "program: maxNullCrossings out of range");
    // the reference's pins (Validator.ts:506-540): equiangular placement only under plain NEE
    if (d->equiangular < PTR_EQUIANGULAR_OFF || d->equiangular > PTR_EQUIANGULAR_AREA)
        return fail(ctx, PTR_E_INVALID, "program: unknown mediumLightSampling");
    if (d->equiangular && d->direct != PTR_DIRECT_NEE)
        return fail(ctx, PTR_E_INVALID, "program: mediumLightSampling 'equiangular' requires directLighting 'nee'");
    if (d->equiangular && !d->scattering)
        return fail(ctx, PTR_E_INVALID, "program: mediumLightSampling 'equiangular' requires scattering media");
    if (d->color != PTR_COLOR_RGB && d->color != PTR_COLOR_SPECTRAL) return fail(ctx, PTR_E_INVALID, "program: unknown measurement.color");
    if (d->accel != PTR_ACCEL_BVH && d->accel != PTR_ACCEL_CWBVH) return fail(ctx, PTR_E_INVALID, "program: unknown meshTraversal");
    if (d->instance_accel != PTR_ACCEL_BVH && d->instance_accel != PTR_ACCEL_CWBVH)
        return fail(ctx, PTR_E_INVALID, "program: unknown instanceAccel");
    if (d->color == PTR_COLOR_SPECTRAL &&
        (d->wavelengths < PTR_WAVELENGTHS_VISIBLE || d->wavelengths > PTR_WAVELENGTHS_UNIFORM ||
         !(d->lambda_min >= 360.0f && d->lambda_max <= 830.0f && d->lambda_min < d->lambda_max)))
        return fail(ctx, PTR_E_INVALID, "program: the sampled wavelength range must lie in [360, 830] nm");
    ptr_program* p = new ptr_program();
    p->ctx = ctx;
    p->desc = *d;
    *out = p;
    return PTR_OK;
}

int ptr_free_program(ptr_program* p) {
    if (!p) return PTR_E_INVALID;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    free_pool(p);
    if (p->sum) cudaFree(p->sum);
    if (p->sumsq) cudaFree(p->sumsq);
    if (p->aov_sum) cudaFree(p->aov_sum);
    if (p->export_buf) cudaFree(p->export_buf);
    if (p->fp_dev) cudaFree(p->fp_dev);
    if (p->work_dev) cudaFree(p->work_dev);
    if (p->adj_dl) cudaFree(p->adj_dl);
    if (p->adj_grads) cudaFree(p->adj_grads);
    if (p->hit_log) cudaFree(p->hit_log);
    delete p;
    return PTR_OK;
}

int ptr_render(ptr_program* p, ptr_scene* s, const ptr_frame* f) {
    if (!p || !s || !f) return PTR_E_INVALID;
    return render_impl(p, s, f, nullptr);
}

int ptr_render_batch(ptr_ctx* ctx, const ptr_batch_job* jobs, int n_jobs) {
    if (!ctx || !jobs || n_jobs <= 0) return fail(ctx, PTR_E_INVALID, "ptr_render_batch: no jobs");
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int direct = jobs[0].prog ? jobs[0].prog->desc.direct : -1;
    bool media = false, equi = false;
    for (int j = 0; j < n_jobs; ++j) {
        const ptr_batch_job& J = jobs[j];
        if (!J.prog || !J.scene || J.prog->ctx != ctx || J.scene->ctx != ctx)
            return fail(ctx, PTR_E_INVALID, "ptr_render_batch: job " + std::to_string(j) + " has a null or foreign program/scene");
        if (J.prog->desc.direct != direct)
            return fail(ctx, PTR_E_INVALID, "ptr_render_batch: every job must use the same directLighting");
        if (J.frame.width <= 0 || J.frame.height <= 0 || J.frame.spp <= 0)
            return fail(ctx, PTR_E_INVALID, "ptr_render_batch: job " + std::to_string(j) + " has an empty frame");
        if (J.scene->has_media) media = true;
        if (J.prog->desc.color != PTR_COLOR_RGB)
            return fail(ctx, PTR_E_UNSUPPORTED, "ptr_render_batch: spectral programs render one per launch (ptr_render)");
        if (int rc = check_equiangular(ctx, J.prog, J.scene)) return rc;
        if (J.prog->desc.aovs) return fail(ctx, PTR_E_INVALID, "batched renders do not take programs with AOVs");
        for (int k = 0; k < j; ++k)
            if (jobs[k].prog == J.prog)
                return fail(ctx, PTR_E_INVALID, "ptr_render_batch: jobs " + std::to_string(k) + " and " + std::to_string(j) + " share a program (one film per job)");
    }
    // the mix's compiled kernels, when ptr_specialize_batch compiled its census
    const SpecKernels* sk = nullptr;
    if (!ctx->batch_spec.empty()) {
        auto it = ctx->batch_spec.find(census_key(census_of_batch(jobs, n_jobs)));
        if (it != ctx->batch_spec.end()) sk = &it->second;
    }
    std::vector<DevScene> scenes(n_jobs);
    std::vector<ProgParams> progs(n_jobs);
    std::vector<BatchJob> bjobs(n_jobs);
    std::vector<long long> offsets(n_jobs + 1, 0);
    int iters = 0;
    std::vector<int> job_iters(n_jobs);
    for (int j = 0; j < n_jobs; ++j) {
        const ptr_batch_job& J = jobs[j];
        ptr_program* p = J.prog;
        int rc = prepare_film(p, &J.frame, st);
        if (rc) return rc;
        scenes[j] = J.scene->dev;
        scenes[j].accel = p->desc.accel;
        scenes[j].inst_accel = p->desc.instance_accel;
        scenes[j].work = nullptr;
        ProgParams& P = progs[j];
        P.max_bounces = p->desc.max_bounces;
        P.direct = p->desc.direct;
        P.rr_start = p->desc.rr_start;
        P.max_null = p->desc.max_null_crossings;
        P.rr_max_survival = p->desc.rr_max_survival;
        P.scattering = p->desc.scattering;
        P.equiangular = p->desc.equiangular;
        P.light_tree = p->desc.light_tree;
        if (P.equiangular) equi = true;
        const long long total_j = (long long)J.frame.width * J.frame.height * J.frame.spp;
        FrameParams& F = bjobs[j].frame;
        F.width = J.frame.width;
        F.height = J.frame.height;
        F.spp = J.frame.spp;
        F.first_sample = J.frame.first_sample;
        F.salt = J.frame.reset_salt;
        F.px_off = J.frame.pixel_offset[0];
        F.py_off = J.frame.pixel_offset[1];
        F.img_w = J.frame.image_size[0] > 0 ? J.frame.image_size[0] : J.frame.width;
        F.img_h = J.frame.image_size[1] > 0 ? J.frame.image_size[1] : J.frame.height;
        F.total = total_j;
        F.capacity = 0;
        F.cam = J.frame.camera;
        bjobs[j].sum = p->sum;
        bjobs[j].sumsq = p->sumsq;
        offsets[j + 1] = offsets[j] + total_j;
        job_iters[j] = p->desc.max_bounces + 1 + (J.scene->has_media ? p->desc.max_null_crossings : 0);
        iters = std::max(iters, job_iters[j]);
    }
    const long long total = offsets[n_jobs];
    if (!ctx->batch) {
        ctx->batch = new ptr_program();
        ctx->batch->ctx = ctx;
    }
    ptr_program* bp = ctx->batch;
    long long cap_max = ctx->tune.capacity > 0 ? ctx->tune.capacity : (1ll << 24);
    if (const char* env = std::getenv("PTR_CAPACITY")) cap_max = std::max(1024ll, (long long)std::atoll(env));
    long long cap = std::min(total, cap_max);
    if (bp->capacity < cap || (equi && !bp->pool.sh2_o)) {
        int rc = alloc_pool(bp, (int)std::max<long long>(cap, bp->capacity), equi || bp->pool.sh2_o);
        if (rc) return rc;
    }
    // device tables (a few KB; refreshed every call)
    DevScene* d_scenes = nullptr;
    ProgParams* d_progs = nullptr;
    BatchJob* d_jobs = nullptr;
    long long* d_off = nullptr;
    if (cudaMalloc(&d_scenes, sizeof(DevScene) * n_jobs) != cudaSuccess || cudaMalloc(&d_progs, sizeof(ProgParams) * n_jobs) != cudaSuccess ||
        cudaMalloc(&d_jobs, sizeof(BatchJob) * n_jobs) != cudaSuccess || cudaMalloc(&d_off, sizeof(long long) * (n_jobs + 1)) != cudaSuccess) {
        cudaFree(d_scenes); cudaFree(d_progs); cudaFree(d_jobs); cudaFree(d_off);
        return fail(ctx, PTR_E_NOMEM, "ptr_render_batch: tables");
    }
    int rc = PTR_OK;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    BatchTables bt{};
    bt.scenes = d_scenes;
    bt.progs = d_progs;
    bt.jobs = d_jobs;
    bt.offsets = d_off;
    bt.n_jobs = n_jobs;
    bt.total = total;
    bt.capacity = (int)cap;
    const long long waves = (total + cap - 1) / cap;
    // each wave walks only as many iterations as the deepest job it holds
    std::vector<int> wave_iters((size_t)waves, 0);
    for (long long w = 0, j = 0; w < waves; ++w) {
        const long long lo = w * cap, hi = std::min(total, lo + cap);
        while (j < n_jobs && offsets[j + 1] <= lo) ++j;
        for (long long k = j; k < n_jobs && offsets[k] < hi; ++k) wave_iters[(size_t)w] = std::max(wave_iters[(size_t)w], job_iters[(size_t)k]);
    }
    const int n_sm = device_sms(ctx->device);
    cudaError_t e = cudaMemcpyAsync(d_scenes, scenes.data(), sizeof(DevScene) * n_jobs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_progs, progs.data(), sizeof(ProgParams) * n_jobs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_jobs, bjobs.data(), sizeof(BatchJob) * n_jobs, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, offsets.data(), sizeof(long long) * (n_jobs + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bp->pool.wave, 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bp->pool.stats, 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bp->pool.cnt, 0, 64, st);
    const bool profiling = (bp->profile_next & PTR_PROFILE_TIMING) != 0;
    bp->profile_next = 0;
    if (profiling) {
        // instrumented: plain launches with events around each (no graph)
        std::vector<ProfRec> prof;
        prof.reserve((size_t)waves * (iters * 5 + 2));
        for (long long w = 0; e == cudaSuccess && w < waves; ++w) {
            launch_batch_wave(jobs[0].scene->dev, bp->pool, bt, direct, media, equi, st, wave_iters[(size_t)w], n_sm, ctx->tune, sk, &prof);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        for (int k = 0; k < PTR_PROFILE_CLASSES; ++k) { bp->prof_ms[k] = 0.0f; bp->prof_launches[k] = 0; }
        for (ProfRec& pr : prof) {
            float ms = 0.0f;
            if (e == cudaSuccess) cudaEventElapsedTime(&ms, pr.a, pr.b);
            bp->prof_ms[pr.cls] += ms;
            bp->prof_launches[pr.cls] += pr.n;
            cudaEventDestroy(pr.a);
            cudaEventDestroy(pr.b);
        }
    } else {
        // occupancy queries outside capture, then one captured wave per iteration count the
        // waves need
        launch_batch_wave(jobs[0].scene->dev, bp->pool, bt, direct, media, equi, st, iters, n_sm, ctx->tune, sk, nullptr, true);
        std::map<int, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;
        for (long long w = 0; e == cudaSuccess && w < waves; ++w) {
            const int it = wave_iters[(size_t)w];
            auto gi = graphs.find(it);
            if (gi == graphs.end()) {
                cudaGraph_t gw = nullptr;
                cudaGraphExec_t gew = nullptr;
                e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    launch_batch_wave(jobs[0].scene->dev, bp->pool, bt, direct, media, equi, st, it, n_sm, ctx->tune, sk);
                    e = cudaStreamEndCapture(st, &gw);
                }
                if (e == cudaSuccess) e = cudaGraphInstantiate(&gew, gw, 0);
                gi = graphs.emplace(it, std::make_pair(gw, gew)).first;
                if (e != cudaSuccess) break;
            }
            e = cudaGraphLaunch(gi->second.second, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        for (auto& kv : graphs) {
            if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
            if (kv.second.first) cudaGraphDestroy(kv.second.first);
        }
    }
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "ptr_render_batch");
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    cudaFree(d_scenes); cudaFree(d_progs); cudaFree(d_jobs); cudaFree(d_off);
    if (rc) return rc;
    for (int j = 0; j < n_jobs; ++j) jobs[j].prog->nsamples += (double)jobs[j].frame.spp;
    bp->last_scene = nullptr;
    return PTR_OK;
}

int ptr_profile_batch_next(ptr_ctx* ctx, int mode) {
    if (!ctx) return PTR_E_INVALID;
    if (!ctx->batch) {
        ctx->batch = new ptr_program();
        ctx->batch->ctx = ctx;
    }
    ctx->batch->profile_next = mode & PTR_PROFILE_TIMING;
    return PTR_OK;
}

int ptr_get_batch_profile(ptr_ctx* ctx, float* ms_out, int* launches_out, int n) {
    if (!ctx || !ctx->batch) return PTR_E_INVALID;
    return ptr_get_profile(ctx->batch, ms_out, launches_out, n);
}

int ptr_get_batch_counters(ptr_ctx* ctx, ptr_counters* out) {
    if (!ctx || !out) return PTR_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    if (!ctx->batch || !ctx->batch->pool.stats) return PTR_OK;
    return ptr_get_counters(ctx->batch, out);
}

int ptr_render_samples(ptr_program* p, ptr_scene* s, const ptr_frame* f, float* host_out, size_t n) {
    if (!p || !s || !f || !host_out) return PTR_E_INVALID;
    ptr_ctx* ctx = p->ctx;
    size_t need = (size_t)f->width * f->height * f->spp * 3;
    if (n < need) return fail(ctx, PTR_E_INVALID, "ptr_render_samples: destination too small");
    float* dev = nullptr;
    CK(ctx, cudaSetDevice(ctx->device));
    if (cudaMalloc(&dev, need * sizeof(float)) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, "samples buffer");
    int rc = render_impl(p, s, f, dev);
    if (rc == PTR_OK) {
        cudaError_t e = cudaMemcpyAsync(host_out, dev, need * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "samples readback");
    }
    if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
    cudaFree(dev);
    return rc;
}

int ptr_trace_closest(ptr_ctx* ctx, ptr_scene* s, int accel, const float* rays, int n,
                      int* region, int* element, int* prim, float* t) {
    if (!ctx || !s || !rays || n < 0 || !region || !element || !prim || !t) return fail(ctx, PTR_E_INVALID, "ptr_trace_closest: null argument");
    if (n == 0) return PTR_OK;
    CK(ctx, cudaSetDevice(ctx->device));
    float* d_rays = nullptr;
    int *d_reg = nullptr, *d_el = nullptr, *d_prim = nullptr;
    float* d_t = nullptr;
    size_t nn = (size_t)n;
    if (cudaMalloc(&d_rays, nn * 6 * sizeof(float)) != cudaSuccess || cudaMalloc(&d_reg, nn * 4) != cudaSuccess ||
        cudaMalloc(&d_el, nn * 4) != cudaSuccess || cudaMalloc(&d_prim, nn * 4) != cudaSuccess || cudaMalloc(&d_t, nn * 4) != cudaSuccess) {
        cudaFree(d_rays); cudaFree(d_reg); cudaFree(d_el); cudaFree(d_prim); cudaFree(d_t);
        return fail(ctx, PTR_E_NOMEM, "ptr_trace_closest: buffers");
    }
    DevScene S = s->dev;
    S.accel = accel;
    cudaError_t e = cudaMemcpyAsync(d_rays, rays, nn * 6 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        k_trace_rays<<<256, 128, 0, ctx->stream>>>(S, d_rays, n, d_reg, d_el, d_prim, d_t);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(region, d_reg, nn * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(element, d_el, nn * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(prim, d_prim, nn * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t, d_t, nn * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_rays); cudaFree(d_reg); cudaFree(d_el); cudaFree(d_prim); cudaFree(d_t);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ptr_trace_closest");
    return PTR_OK;
}

int ptr_get_stream(ptr_ctx* ctx, void** stream) {
    if (!ctx || !stream) return PTR_E_INVALID;
    *stream = (void*)ctx->stream;
    return PTR_OK;
}

int ptr_backward(ptr_program* p, ptr_scene* s, const ptr_frame* f, const float* dl_dimage, double* grads, size_t n) {
    if (!p || !s || !f || !dl_dimage || !grads) return fail(p ? p->ctx : nullptr, PTR_E_INVALID, "ptr_backward: null argument");
    ptr_ctx* ctx = p->ctx;
    if (s->ctx != ctx) return fail(ctx, PTR_E_INVALID, "scene belongs to another context");
    if (f->width <= 0 || f->height <= 0 || f->spp <= 0) return fail(ctx, PTR_E_INVALID, "frame: width, height and spp must be positive");
    const int n_mat = (int)s->h_materials.size();
    if (n < (size_t)PTR_GRAD_SLOTS * n_mat)
        return fail(ctx, PTR_E_INVALID, "ptr_backward: grads needs PTR_GRAD_SLOTS * n_materials doubles");
    if (n_mat > 512) return fail(ctx, PTR_E_INVALID, "ptr_backward: at most 512 materials");
    if (p->desc.equiangular) return fail(ctx, PTR_E_INVALID, "ptr_backward: equiangular programs are not differentiated");
    if (p->desc.light_tree) return fail(ctx, PTR_E_INVALID, "ptr_backward: light-tree programs are not differentiated");
    if (p->desc.aovs) return fail(ctx, PTR_E_INVALID, "ptr_backward: programs with AOVs are not differentiated");
    if (s->dev.has_het) return fail(ctx, PTR_E_INVALID, "ptr_backward: scenes with heterogeneous media are not differentiated");
    if (p->desc.color != PTR_COLOR_RGB) return fail(ctx, PTR_E_INVALID, "ptr_backward: the adjoint is RGB only");
    for (const ptr_material& m : s->h_materials)
        if ((m.flags & PTR_MATF_MEDIUM) && !(m.sigma_a[0] == m.sigma_a[1] && m.sigma_a[0] == m.sigma_a[2] &&
                                             m.sigma_s[0] == m.sigma_s[1] && m.sigma_s[0] == m.sigma_s[2]))
            return fail(ctx, PTR_E_INVALID, "ptr_backward: media must be grey (chromatic media are not differentiated)");
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t npix = (size_t)f->width * f->height;
    const long long total = (long long)npix * f->spp;
    long long cap_max = ctx->tune.capacity > 0 ? ctx->tune.capacity : (1ll << 24);
    if (const char* env = std::getenv("PTR_CAPACITY")) cap_max = std::max(1024ll, (long long)std::atoll(env));
    long long cap = (long long)npix <= cap_max ? (cap_max / (long long)npix) * (long long)npix : cap_max;
    if (cap > total) cap = total;
    if (p->capacity < cap || !p->pool.l_rem) {
        int rc = alloc_pool(p, (int)std::max<long long>(cap, p->capacity), p->pool.sh2_o.p != nullptr, true);
        if (rc) return rc;
    }
    if (!p->fp_dev) CK(ctx, cudaMalloc(&p->fp_dev, sizeof(FrameParams)));
    if (p->adj_dl_n < npix * 3) {
        if (p->adj_dl) cudaFree(p->adj_dl);
        p->adj_dl = nullptr;
        if (cudaMalloc(&p->adj_dl, npix * 3 * sizeof(float)) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, "ptr_backward: adjoint image");
        p->adj_dl_n = npix * 3;
    }
    const size_t ng = (size_t)PTR_GRAD_SLOTS * n_mat;
    if (p->adj_grads_n < ng) {
        if (p->adj_grads) cudaFree(p->adj_grads);
        p->adj_grads = nullptr;
        if (cudaMalloc(&p->adj_grads, ng * sizeof(double)) != cudaSuccess) return fail(ctx, PTR_E_NOMEM, "ptr_backward: gradients");
        p->adj_grads_n = ng;
    }
    // the graph of a previous ptr_render reads the same pool; it is re-captured on demand
    FrameParams F;
    F.width = f->width;
    F.height = f->height;
    F.spp = f->spp;
    F.first_sample = f->first_sample;
    F.salt = f->reset_salt;
    F.px_off = f->pixel_offset[0];
    F.py_off = f->pixel_offset[1];
    F.img_w = f->image_size[0] > 0 ? f->image_size[0] : f->width;
    F.img_h = f->image_size[1] > 0 ? f->image_size[1] : f->height;
    F.total = total;
    F.capacity = (int)cap;
    F.cam = f->camera;
    k_set_frame<<<1, 1, 0, st>>>(p->fp_dev, F);
    CK(ctx, cudaGetLastError());
    CK(ctx, cudaMemcpyAsync(p->adj_dl, dl_dimage, npix * 3 * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemsetAsync(p->adj_grads, 0, ng * sizeof(double), st));
    CK(ctx, cudaMemsetAsync(p->pool.wave, 0, 64, st));
    CK(ctx, cudaMemsetAsync(p->pool.stats, 0, 64, st));
    CK(ctx, cudaMemsetAsync(p->pool.cnt, 0, 64, st));
    AdjParams adj;
    adj.dl_image = p->adj_dl;
    adj.inv_spp = 1.0f / (float)f->spp;
    adj.grads = p->adj_grads;
    const int iters = wave_iterations(p, s);
    const long long waves = (total + cap - 1) / cap;
    const int n_sm = device_sms(ctx->device);
    // a specialised program: the replay's kernels for the same census (NVRTC, once)
    if (p->spec.scene_id == s->id && p->spec.shade && !p->spec.shade_adj) {
        Census c = census_of(p, s);
        c.adj = true;
        SpecModule m;
        bool compiled = false;
        if (int rc = spec_compile(ctx, c, m, compiled)) return rc;
        p->spec.shade_adj = m.shade;
        p->spec.shadow_adj = m.shadow;
    }
    // the forward walk logs its closest hits and slot-0 shadow queries for the replay, as many
    // walk iterations as 4 GiB holds (64 bytes per path slot and iteration; PTR_HIT_LOG_BYTES
    // overrides the bound); later iterations are walked again
    const long long per_iter = 64ll * p->capacity;
    long long log_budget = 4ll << 30;
    if (const char* env = std::getenv("PTR_HIT_LOG_BYTES")) log_budget = std::max(0ll, (long long)std::atoll(env));
    int log_iters = (int)std::min<long long>(iters, log_budget / std::max<long long>(per_iter, 1));
    if (log_iters > 0 && p->hit_log_bytes < (size_t)(per_iter * log_iters)) {
        if (p->hit_log) cudaFree(p->hit_log);
        p->hit_log = nullptr;
        p->hit_log_bytes = 0;
        if (cudaMalloc(&p->hit_log, (size_t)(per_iter * log_iters)) == cudaSuccess) p->hit_log_bytes = (size_t)(per_iter * log_iters);
        else { cudaGetLastError(); log_iters = 0; }   // no log: the replay walks every query
    }
    const int saved_profile = p->profile_next;
    p->profile_next = 0;
    p->pool.hit_log = log_iters > 0 ? p->hit_log : nullptr;
    p->pool.hit_log_stride = p->capacity;
    p->pool.hit_log_iters = log_iters;
    for (long long w = 0; w < waves; ++w) {
        p->pool.hit_log_mode = 1;
        launch_wave(p, s, st, iters, nullptr, n_sm, nullptr, false);
        p->pool.hit_log_mode = 2;
        launch_replay(p, s, st, iters, n_sm, adj);
    }
    p->pool.hit_log = nullptr;
    p->pool.hit_log_iters = 0;
    p->pool.hit_log_mode = 0;
    p->profile_next = saved_profile;
    CK(ctx, cudaGetLastError());
    CK(ctx, cudaMemcpyAsync(grads, p->adj_grads, ng * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaStreamSynchronize(st));
    unsigned flags = 0;
    if (s->dev.err_flags) CK(ctx, cudaMemcpy(&flags, s->dev.err_flags, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flags) return fail(ctx, PTR_E_DEVICE, "ptr_backward: device guard flags " + std::to_string(flags));
    for (size_t k = ng; k < n; ++k) grads[k] = 0.0;
    return PTR_OK;
}

int ptr_update_params(ptr_scene* s, const ptr_material* materials, int n_materials, const ptr_region* regions, int n_regions) {
    if (!s || !materials) return fail(s ? s->ctx : nullptr, PTR_E_INVALID, "ptr_update_params: null argument");
    ptr_ctx* ctx = s->ctx;
    if (n_materials != (int)s->h_materials.size()) return fail(ctx, PTR_E_INVALID, "ptr_update_params: material count differs from the uploaded scene");
    for (int i = 0; i < n_materials; ++i)
        if (materials[i].model != s->h_materials[i].model || materials[i].flags != s->h_materials[i].flags ||
            materials[i].field_a != s->h_materials[i].field_a || materials[i].field_s != s->h_materials[i].field_s ||
            ((materials[i].field_a || materials[i].field_s) && !(materials[i].majorant > 0.0f && std::isfinite(materials[i].majorant))))
            return fail(ctx, PTR_E_INVALID, "ptr_update_params: a material's model, flags or coefficient fields changed");
    if (regions) {
        if (n_regions != (int)s->h_regions.size()) return fail(ctx, PTR_E_INVALID, "ptr_update_params: region count differs from the uploaded scene");
        for (int i = 0; i < n_regions; ++i) {
            const ptr_region& a = regions[i];
            const ptr_region& b = s->h_regions[i];
            if (a.shape != b.shape || a.material != b.material || a.thin != b.thin || a.ref != b.ref ||
                std::memcmp(a.p, b.p, sizeof(a.p)) != 0)
                return fail(ctx, PTR_E_INVALID, "ptr_update_params: only a region's IOR may change");
        }
    }
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    CK(ctx, cudaMemcpyAsync((void*)s->dev.materials, materials, sizeof(ptr_material) * n_materials, cudaMemcpyHostToDevice, st));
    if (regions) CK(ctx, cudaMemcpyAsync((void*)s->dev.regions, regions, sizeof(ptr_region) * n_regions, cudaMemcpyHostToDevice, st));
    CK(ctx, cudaStreamSynchronize(st));   // the host arrays may be released on return
    s->h_materials.assign(materials, materials + n_materials);
    if (regions) s->h_regions.assign(regions, regions + n_regions);
    return PTR_OK;
}

int ptr_specialize(ptr_program* p, ptr_scene* s, double* seconds_out) {
    if (!p || !p->ctx) return fail(p ? p->ctx : nullptr, PTR_E_INVALID, "ptr_specialize: null program");
    ptr_ctx* ctx = p->ctx;
    if (seconds_out) *seconds_out = 0.0;
    if (!s) {                                      // back to the generic kernels
        p->spec = SpecKernels{};
        return PTR_OK;
    }
    if (s->ctx != ctx) return fail(ctx, PTR_E_INVALID, "ptr_specialize: scene belongs to another context");
    CK(ctx, cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    SpecModule m;
    bool compiled = false;
    if (int rc = spec_compile(ctx, census_of(p, s), m, compiled)) return rc;
    p->spec = SpecKernels{};                       // the replay's kernels follow at the first ptr_backward
    p->spec.scene_id = s->id;
    p->spec.closest = m.closest;
    p->spec.shade = m.shade;
    p->spec.shadow = m.shadow;
    if (seconds_out && compiled) *seconds_out = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return PTR_OK;
}

int ptr_specialize_batch(ptr_ctx* ctx, const ptr_batch_job* jobs, int n_jobs, double* seconds_out) {
    if (!ctx || !jobs || n_jobs <= 0) return fail(ctx, PTR_E_INVALID, "ptr_specialize_batch: no jobs");
    if (seconds_out) *seconds_out = 0.0;
    for (int j = 0; j < n_jobs; ++j) {
        const ptr_batch_job& J = jobs[j];
        if (!J.prog || !J.scene || J.prog->ctx != ctx || J.scene->ctx != ctx)
            return fail(ctx, PTR_E_INVALID, "ptr_specialize_batch: job " + std::to_string(j) + " has a null or foreign program/scene");
        if (J.prog->desc.direct != jobs[0].prog->desc.direct || J.prog->desc.color != PTR_COLOR_RGB)
            return fail(ctx, PTR_E_INVALID, "ptr_specialize_batch: the jobs must share directLighting and render RGB");
    }
    CK(ctx, cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    const Census c = census_of_batch(jobs, n_jobs);
    SpecModule m;
    bool compiled = false;
    if (int rc = spec_compile(ctx, c, m, compiled)) return rc;
    SpecKernels k;
    k.closest = m.closest;
    k.shade = m.shade;
    k.shadow = m.shadow;
    ctx->batch_spec[census_key(c)] = k;
    if (seconds_out && compiled) *seconds_out = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return PTR_OK;
}

int ptr_set_accel_build(ptr_ctx* ctx, int where) {
    if (!ctx) return PTR_E_INVALID;
    if (where != PTR_BUILD_HOST && where != PTR_BUILD_DEVICE) return fail(ctx, PTR_E_INVALID, "ptr_set_accel_build: unknown builder");
    ctx->accel_build = where;
    return PTR_OK;
}

int ptr_set_tuning(ptr_ctx* ctx, const ptr_tuning* t) {
    if (!ctx || !t) return fail(ctx, PTR_E_INVALID, "ptr_set_tuning: null argument");
    if (t->capacity < 0 || (t->capacity > 0 && t->capacity < 1024) || t->capacity > (1 << 26))
        return fail(ctx, PTR_E_INVALID, "ptr_set_tuning: capacity must be 0 (default) or in [1024, 2^26]");
    if (t->block != 128 && t->block != 256) return fail(ctx, PTR_E_INVALID, "ptr_set_tuning: block must be 128 or 256");
    if (t->sort_buckets < 1 || t->sort_buckets > kMaxSortBuckets)
        return fail(ctx, PTR_E_INVALID, "ptr_set_tuning: sort_buckets must be in [1, 32]");
    if (t->ray_sort != 0 && t->ray_sort != 1) return fail(ctx, PTR_E_INVALID, "ptr_set_tuning: ray_sort must be 0 or 1");
    ctx->tune = *t;
    return PTR_OK;
}

int ptr_get_tuning(ptr_ctx* ctx, ptr_tuning* out) {
    if (!ctx || !out) return fail(ctx, PTR_E_INVALID, "ptr_get_tuning: null argument");
    *out = ctx->tune;
    return PTR_OK;
}

int ptr_sync(ptr_ctx* ctx, int timeout_ms) {
    if (!ctx) return PTR_E_INVALID;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(ctx->stream);
        if (e == cudaSuccess) return PTR_OK;
        if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "stream");
        if (timeout_ms >= 0) {
            auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
            if (ms >= timeout_ms) return fail(ctx, PTR_E_TIMEOUT, "ptr_sync: timed out with work in flight");
        }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

static int export_impl(ptr_program* p, const char* name, float* dst, size_t n, bool device_dst) {
    ptr_ctx* ctx = p->ctx;
    if (!name || !dst) return fail(ctx, PTR_E_INVALID, "export: null argument");
    const size_t npix = (size_t)p->fw * p->fh;
    if (!p->sum) return fail(ctx, PTR_E_INVALID, "export: nothing rendered yet");
    CK(ctx, cudaSetDevice(ctx->device));
    if (std::strcmp(name, "samples") == 0) {
        if (n < npix) return fail(ctx, PTR_E_INVALID, "export: destination too small");
        std::vector<float> v(npix, (float)p->nsamples);
        if (device_dst) CK(ctx, cudaMemcpyAsync(dst, v.data(), npix * 4, cudaMemcpyHostToDevice, ctx->stream));
        else std::memcpy(dst, v.data(), npix * 4);
        if (device_dst) CK(ctx, cudaStreamSynchronize(ctx->stream));
        return PTR_OK;
    }
    int what;
    if (std::strcmp(name, "radiance") == 0) what = 0;
    else if (std::strcmp(name, "variance") == 0) what = 1;
    else if (std::strcmp(name, "albedo") == 0 && (p->desc.aovs & PTR_AOV_ALBEDO) && p->aov_sum) what = 2;
    else if (std::strcmp(name, "normal") == 0 && (p->desc.aovs & PTR_AOV_NORMAL) && p->aov_sum) what = 3;
    else return fail(ctx, PTR_E_INVALID, std::string("export: unknown export '") + name + "'");
    if (n < npix * 3) return fail(ctx, PTR_E_INVALID, "export: destination too small");
    float* target = device_dst ? dst : p->export_buf;
    const double* src = what == 2 ? p->aov_sum : what == 3 ? p->aov_sum + 3 * npix : p->sum;   // a picture's mean
    k_export<<<256, 256, 0, ctx->stream>>>(src, p->sumsq, p->nsamples > 0 ? p->nsamples : 1.0, (int)npix, what >= 2 ? 0 : what, target);
    CK(ctx, cudaGetLastError());
    if (!device_dst) {
        CK(ctx, cudaMemcpyAsync(dst, p->export_buf, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return PTR_OK;
}

int ptr_read_export(ptr_program* p, const char* name, float* dst, size_t n) {
    if (!p) return PTR_E_INVALID;
    return export_impl(p, name, dst, n, false);
}

int ptr_read_export_device(ptr_program* p, const char* name, float* dst, size_t n) {
    if (!p) return PTR_E_INVALID;
    return export_impl(p, name, dst, n, true);
}

int ptr_get_counters(ptr_program* p, ptr_counters* out) {
    if (!p || !out) return PTR_E_INVALID;
    ptr_ctx* ctx = p->ctx;
    std::memset(out, 0, sizeof(*out));
    if (!p->pool.stats) return PTR_OK;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned long long st[3] = {0, 0, 0};
    unsigned cnt[4] = {0, 0, 0, 0};
    CK(ctx, cudaMemcpy(st, p->pool.stats, sizeof(st), cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(cnt, p->pool.cnt, sizeof(cnt), cudaMemcpyDeviceToHost));
    out->closest_queries = st[0];
    out->shadow_queries = st[1];
    out->paths = st[2];
    out->error_flags = cnt[3];
    if (p->last_scene && p->last_scene->dev.err_flags) {
        unsigned ef = 0;
        CK(ctx, cudaMemcpy(&ef, p->last_scene->dev.err_flags, 4, cudaMemcpyDeviceToHost));
        out->error_flags |= ef;
    }
    if (p->work_valid && p->work_dev) {
        unsigned long long wk[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        CK(ctx, cudaMemcpy(wk, p->work_dev, sizeof(wk), cudaMemcpyDeviceToHost));
        out->nodes_visited = wk[0];
        out->prims_tested = wk[1];
        out->tlas_nodes = wk[2];
        out->instances = wk[3];
        for (int k = 0; k < 4; ++k) out->shadow_work[k] = wk[4 + k];
    }
    return PTR_OK;
}

int ptr_profile_next(ptr_program* p, int enable) {
    if (!p) return PTR_E_INVALID;
    p->profile_next = enable;
    return PTR_OK;
}

int ptr_get_profile(ptr_program* p, float* ms_out, int* launches_out, int n) {
    if (!p) return PTR_E_INVALID;
    for (int i = 0; i < n && i < PTR_PROFILE_CLASSES; ++i) {
        if (ms_out) ms_out[i] = p->prof_ms[i];
        if (launches_out) launches_out[i] = p->prof_launches[i];
    }
    return PTR_OK;
}

}  // extern "C"

// =====================================================================================
// Allocation-free rendering (ptr_render_noalloc).
//
// Some callers cannot allocate device memory: an application that hands every byte of
// the GPU to its own memory pool, a plugin host that forbids driver allocations inside
// its frame loop, or a real-time loop that cannot afford the device-wide synchronisation
// cudaMalloc/cudaFree may imply.  For them this entry point renders analytic scenes with
// no allocation at all: the scene tables and the path pool live in one file-scope
// __device__ array of fixed size, and the caller passes its own film buffers.
//
// Limits: at most kNoAllocMaxPaths paths in flight (frames of any size are processed in
// waves) and at most kNoAllocMaxTable regions, materials and lights.  The array costs
// about 15 MB on every GPU that loads this library, held until the process exits.
// Every call shares the array: calls that overlap on the GPU (on different streams, or
// from different host threads) race and corrupt each other's paths.
// =====================================================================================
namespace {

constexpr int kNoAllocMaxPaths = 1 << 16;
constexpr int kNoAllocMaxTable = 256;

// Byte layout of the array: small blocks first, then the path pool.
constexpr size_t kNaCnt = 0;                                            // 16 x u32
constexpr size_t kNaStats = 64;                                         // 8 x u64
constexpr size_t kNaWave = 128;                                         // 8 x i64
constexpr size_t kNaFrame = 256;                                        // FrameParams
constexpr size_t kNaRegions = 1024;
constexpr size_t kNaMaterials = kNaRegions + sizeof(ptr_region) * kNoAllocMaxTable;
constexpr size_t kNaLights = kNaMaterials + sizeof(ptr_material) * kNoAllocMaxTable;
constexpr size_t kNaLightOf = kNaLights + sizeof(ptr_light) * kNoAllocMaxTable;
constexpr size_t kNaPool = (kNaLightOf + sizeof(int) * kNoAllocMaxTable + 255) / 256 * 256;
constexpr size_t kNaPathBytes = 13 * 16 + 8 + 3 * 4;                    // per path, see na_pool()
constexpr size_t kNaBytes = kNaPool + kNaPathBytes * (size_t)kNoAllocMaxPaths;
static_assert(sizeof(FrameParams) <= kNaRegions - kNaFrame, "FrameParams block too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kMaxDevices = 64;
std::mutex g_na_mutex;
unsigned char* g_na_addr[kMaxDevices] = {nullptr};

// Device address of the array on the current device, looked up once per device.  The
// array's host-side name is only a stand-in; kernels must be given this address.
int na_address(int dev, unsigned char** out, const char** why) {
    if (dev < 0 || dev >= kMaxDevices) { *why = "device ordinal out of range"; return PTR_E_INVALID; }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            *why = cudaGetErrorString(e);
            return PTR_E_CUDA;
        }
        g_na_addr[dev] = (unsigned char*)p;
    }
    *out = g_na_addr[dev];
    return PTR_OK;
}

PathPool na_pool(unsigned char* base) {
    PathPool q{};
    size_t c = kNoAllocMaxPaths;
    unsigned char* p = base + kNaPool;
    auto take = [&](size_t bytes) { unsigned char* r = p; p += bytes * c; return (void*)r; };
    auto pair = [&](auto& a, auto& b) {   // a two-field record of 32 bytes per path
        unsigned char* base = (unsigned char*)take(32);
        a.p = (std::remove_reference_t<decltype(*a.p)>*)base;
        b.p = (std::remove_reference_t<decltype(*b.p)>*)(base + 16);
    };
    pair(q.ray_o, q.ray_d); pair(q.thr, q.rad); pair(q.prev_q, q.st); q.prev_n = nullptr; q.sh_seed = nullptr;
    pair(q.hit, q.hit_i); pair(q.sh_o, q.sh_d); pair(q.sh_lp, q.sh_c);
    q.rng = (uint2*)take(8); q.q[0] = (int*)take(4); q.q[1] = (int*)take(4); q.shq = (int*)take(4);
    q.cnt = (unsigned*)(base + kNaCnt);
    q.stats = (unsigned long long*)(base + kNaStats);
    q.wave = (long long*)(base + kNaWave);
    return q;
}

}  // namespace

extern "C" int ptr_render_noalloc(const ptr_scene_desc* d, const ptr_program_desc* pd, const ptr_frame* f,
                                  double* sum_dev, double* sumsq_dev, void* stream) {
    if (!d || !pd || !f || !sum_dev || !sumsq_dev) return PTR_E_INVALID;
    if (d->abi_version != PTR_ABI_VERSION || pd->abi_version != PTR_ABI_VERSION) return PTR_E_INVALID;
    if (d->n_regions < 0 || d->n_regions > kNoAllocMaxTable || d->n_materials <= 0 || d->n_materials > kNoAllocMaxTable ||
        d->n_lights < 0 || d->n_lights > kNoAllocMaxTable) {
        std::fprintf(stderr, "ptr_render_noalloc: scene tables exceed the fixed maximum of %d regions, materials and lights\n",
                     kNoAllocMaxTable);
        return PTR_E_INVALID;
    }
    if (d->n_meshes != 0 || d->n_batches != 0 || d->env.kind == PTR_ENV_IMAGE || d->n_tree_nodes != 0 || pd->light_tree || d->n_field_code != 0 || pd->aovs) {
        std::fprintf(stderr, "ptr_render_noalloc: only analytic scenes with a constant or no environment and power or uniform light selection are supported\n");
        return PTR_E_UNSUPPORTED;
    }
    if (f->width <= 0 || f->height <= 0 || f->spp <= 0) return PTR_E_INVALID;
    if (pd->max_bounces < 0 || pd->max_bounces > 4096 || pd->direct < 0 || pd->direct > 2 || pd->equiangular ||
        pd->color != PTR_COLOR_RGB) return PTR_E_INVALID;
    // the same scene checks as ptr_upload_scene, then the analytic subset this entry
    // point renders: shapes up to boxes and quad, sphere or point lights (a mesh light
    // would need mesh tables that are never uploaded here)
    std::string why;
    if (int rc = check_scene_desc(d, why)) {
        std::fprintf(stderr, "ptr_render_noalloc: %s\n", why.c_str());
        return rc;
    }
    for (int i = 0; i < d->n_regions; ++i)
        if (d->regions[i].shape > PTR_SHAPE_BOX) {
            std::fprintf(stderr, "ptr_render_noalloc: region %d is not an analytic shape\n", i);
            return PTR_E_INVALID;
        }
    for (int i = 0; i < d->n_lights; ++i)
        if (d->lights[i].kind < PTR_LIGHT_QUAD || d->lights[i].kind > PTR_LIGHT_POINT) {
            std::fprintf(stderr, "ptr_render_noalloc: light %d is not a quad, sphere or point light\n", i);
            return PTR_E_INVALID;
        }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PTR_E_CUDA;
    unsigned char* base = nullptr;
    const char* why_addr = "";
    int rc = na_address(dev, &base, &why_addr);
    if (rc) {
        std::fprintf(stderr, "ptr_render_noalloc: cudaGetSymbolAddress failed: %s\n", why_addr);
        return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // scene tables into the array (host arrays on the caller's side; no staging allocation)
    int lor[kNoAllocMaxTable];
    for (int i = 0; i < kNoAllocMaxTable; ++i) lor[i] = -1;
    for (int i = 0; i < d->n_lights; ++i)
        if (d->lights[i].region >= 0 && d->lights[i].region < d->n_regions) lor[d->lights[i].region] = i;
    if (d->n_regions && cudaMemcpyAsync(base + kNaRegions, d->regions, sizeof(ptr_region) * d->n_regions, cudaMemcpyHostToDevice, st) != cudaSuccess) return PTR_E_CUDA;
    if (cudaMemcpyAsync(base + kNaMaterials, d->materials, sizeof(ptr_material) * d->n_materials, cudaMemcpyHostToDevice, st) != cudaSuccess) return PTR_E_CUDA;
    if (d->n_lights && cudaMemcpyAsync(base + kNaLights, d->lights, sizeof(ptr_light) * d->n_lights, cudaMemcpyHostToDevice, st) != cudaSuccess) return PTR_E_CUDA;
    if (cudaMemcpyAsync(base + kNaLightOf, lor, sizeof(int) * kNoAllocMaxTable, cudaMemcpyHostToDevice, st) != cudaSuccess) return PTR_E_CUDA;
    // the previous call's counters, statistics and wave cursor must not leak in
    if (cudaMemsetAsync(base, 0, kNaFrame, st) != cudaSuccess) return PTR_E_CUDA;
    const size_t npix = (size_t)f->width * f->height;
    if (!f->accumulate) {
        if (cudaMemsetAsync(sum_dev, 0, npix * 3 * sizeof(double), st) != cudaSuccess) return PTR_E_CUDA;
        if (cudaMemsetAsync(sumsq_dev, 0, npix * 3 * sizeof(double), st) != cudaSuccess) return PTR_E_CUDA;
    }
    DevScene S{};
    S.regions = (const ptr_region*)(base + kNaRegions);
    S.materials = (const ptr_material*)(base + kNaMaterials);
    S.lights = (const ptr_light*)(base + kNaLights);
    S.light_of_region = (const int*)(base + kNaLightOf);
    S.n_regions = d->n_regions;
    S.n_materials = d->n_materials;
    S.n_lights = d->n_lights;
    S.ambient_material = d->ambient_material;
    bool media = d->ambient_material >= 0 && (d->materials[d->ambient_material].flags & PTR_MATF_MEDIUM);
    for (int i = 0; i < d->n_materials; ++i)
        if (d->materials[i].flags & PTR_MATF_MEDIUM) media = true;
    S.has_media = media ? 1 : 0;
    S.env_kind = d->env.kind;
    S.env_samplable = d->env.kind != PTR_ENV_NONE && d->env.sample_as_light;
    S.env_select_live = S.env_samplable && d->n_lights > 0;
    for (int k = 0; k < 4; ++k) S.env_color[k] = d->env.color[k];
    S.env_intensity = d->env.intensity;
    S.env_select_prob = d->env.select_prob;
    S.env_rotation = d->env.rotation;

    const long long total = (long long)npix * f->spp;
    long long cap = (long long)npix <= kNoAllocMaxPaths ? (kNoAllocMaxPaths / (long long)npix) * (long long)npix
                                                        : (long long)kNoAllocMaxPaths;
    if (cap > total) cap = total;
    FrameParams F;
    F.width = f->width;
    F.height = f->height;
    F.spp = f->spp;
    F.first_sample = f->first_sample;
    F.salt = f->reset_salt;
    F.px_off = f->pixel_offset[0];
    F.py_off = f->pixel_offset[1];
    F.img_w = f->image_size[0] > 0 ? f->image_size[0] : f->width;
    F.img_h = f->image_size[1] > 0 ? f->image_size[1] : f->height;
    F.total = total;
    F.capacity = (int)cap;
    F.cam = f->camera;
    FrameParams* fp = (FrameParams*)(base + kNaFrame);
    k_set_frame<<<1, 1, 0, st>>>(fp, F);

    // the same wave sequence as ptr_render, launched directly
    ptr_program prog;
    prog.desc = *pd;
    prog.pool = na_pool(base);
    prog.fp_dev = fp;
    prog.sum = sum_dev;
    prog.sumsq = sumsq_dev;
    ptr_scene scene;
    scene.dev = S;
    scene.has_media = S.has_media;
    const int iters = wave_iterations(&prog, &scene);
    const long long waves = (total + cap - 1) / cap;
    const int n_sm = device_sms(dev);
    for (long long w = 0; w < waves; ++w) launch_wave(&prog, &scene, st, iters, nullptr, n_sm);
    // keep the stack objects from releasing anything they do not own
    prog.pool = PathPool{};
    prog.fp_dev = nullptr;
    prog.sum = prog.sumsq = nullptr;
    if (cudaGetLastError() != cudaSuccess) return PTR_E_CUDA;
    return PTR_OK;
}
