// lbvh.cuh — mesh acceleration structures built on the device (no counterpart in the
// reference, which builds on the host: buildBVHCore / buildCWBVH, bvh.ts:132-343 and
// cwbvh.ts:80-372, in a Web Worker).
//
// A linear BVH (Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees, and
// k-d Trees", HPG 2012) over 30-bit Morton codes of the triangle box centres:
//   1. per triangle its float box and centre; the centres' bounds by block reduction and
//      order-preserving integer atomics;
//   2. 64-bit keys (Morton code << 32 | triangle), all distinct, sorted by a bitonic
//      network (shared-memory stages for strides below 1024, global passes above);
//   3. the binary hierarchy: one thread per internal node finds its key range and split
//      from common-prefix lengths; leaves are the sorted triangles;
//   4. node boxes bottom-up, the second thread to reach a node joining its children's
//      boxes (a fence before each arrival counter);
//   5. the binary walk's layout: nodes renumbered in preorder (left child = node + 1),
//      from each node's leaf range, depth and right turns;
//   6. the compressed wide BVH (the 80-byte node format of cwbvh.ts:18-31 the walk reads):
//      top-down, level by level, each wide node gathers up to eight children by opening
//      its largest child until eight are reached (children of at most three triangles
//      become leaf children: an LBVH subtree covers a contiguous run of sorted
//      triangles), takes octant slots, allocates its internal children and leaf items
//      with atomics, and quantizes the children's boxes conservatively against its
//      power-of-two grid exactly as the host encoder does.
// Every box a walk tests contains the triangles below it, so nearest hits (and, with the
// walks' tie rule, hit IDs) are those of any other valid tree; only the node visit counts
// differ from the host's SAH trees.
#pragma once
#include "common.cuh"

namespace ptx {
namespace lbvh {

constexpr unsigned long long kPadKey = 0xFFFFFFFFFFFFFFFFull;

// float <-> order-preserving signed int (monotonic for every finite float)
__device__ __forceinline__ int f2o(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

// 10 bits spread to every third bit
__device__ __forceinline__ unsigned spread3(unsigned v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// 1. Per-triangle boxes (lo, hi as float4; .w unused) and the centres' bounds
// (cbound[0..2] min, [3..5] max, as order-preserving ints; initialised by the host).
__global__ void k_boxes(const float* pos, const unsigned* idx, int n, float4* lo, float4* hi, int* cbound) {
    __shared__ int s_b[6];
    if (threadIdx.x < 6) s_b[threadIdx.x] = threadIdx.x < 3 ? 0x7FFFFFFF : (int)0x80000000;
    __syncthreads();
    int b[6] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF, (int)0x80000000, (int)0x80000000, (int)0x80000000};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        float mn[3], mx[3];
        for (int a = 0; a < 3; ++a) { mn[a] = 3.0e38f; mx[a] = -3.0e38f; }
        for (int k = 0; k < 3; ++k) {
            const float* p = pos + 3 * (size_t)idx[3 * (size_t)t + k];
            for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], p[a]); mx[a] = fmaxf(mx[a], p[a]); }
        }
        lo[t] = make_float4(mn[0], mn[1], mn[2], 0.0f);
        hi[t] = make_float4(mx[0], mx[1], mx[2], 0.0f);
        for (int a = 0; a < 3; ++a) {
            const int c = f2o(0.5f * (mn[a] + mx[a]));
            b[a] = min(b[a], c);
            b[3 + a] = max(b[3 + a], c);
        }
    }
    for (int a = 0; a < 6; ++a) {
        int v = b[a];
        for (int o = 16; o > 0; o >>= 1) {
            const int u = __shfl_xor_sync(0xffffffffu, v, o);
            v = a < 3 ? min(v, u) : max(v, u);
        }
        if ((threadIdx.x & 31) == 0) {
            if (a < 3) atomicMin(&s_b[a], v);
            else atomicMax(&s_b[a], v);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&cbound[threadIdx.x], s_b[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&cbound[threadIdx.x], s_b[threadIdx.x]);
}

// 2a. Keys: 30-bit Morton code of the normalised centre above the triangle index; the
// padding up to a power of two takes the largest key.
__global__ void k_keys(const float4* lo, const float4* hi, int n, int n_pad, const int* cbound,
                       unsigned long long* keys) {
    const float b0[3] = {o2f(cbound[0]), o2f(cbound[1]), o2f(cbound[2])};
    const float b1[3] = {o2f(cbound[3]), o2f(cbound[4]), o2f(cbound[5])};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_pad; t += gridDim.x * blockDim.x) {
        if (t >= n) { keys[t] = kPadKey; continue; }
        const float4 a = lo[t], c = hi[t];
        const float ctr[3] = {0.5f * (a.x + c.x), 0.5f * (a.y + c.y), 0.5f * (a.z + c.z)};
        unsigned q[3];
        for (int k = 0; k < 3; ++k) {
            const float ext = b1[k] - b0[k];
            float u = ext > 0.0f ? (ctr[k] - b0[k]) / ext : 0.5f;
            u = fminf(fmaxf(u, 0.0f), 1.0f);
            q[k] = min(1023u, (unsigned)(u * 1024.0f));
        }
        const unsigned code = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
        keys[t] = ((unsigned long long)code << 32) | (unsigned)t;
    }
}

// 2b. Bitonic sort of n_pad (a power of two, at least kBitonicTile) keys.  k_bitonic_local:
// every stage with a stride below the block's 1024 keys in shared memory (all stages of
// k <= 1024 when k_from == 2, else the strides j < 1024 of stage k_from); k_bitonic_global:
// one stride j >= 1024.  The direction of a pair comes from its global index, so the
// blocks' local sorts alternate as the global network requires.
constexpr int kBitonicTile = 1024;
__global__ void __launch_bounds__(512) k_bitonic_local(unsigned long long* keys, int k_from, int k_to) {
    __shared__ unsigned long long s[kBitonicTile];
    const size_t base = (size_t)blockIdx.x * kBitonicTile;
    for (int e = threadIdx.x; e < kBitonicTile; e += blockDim.x) s[e] = keys[base + e];
    __syncthreads();
    for (int k = k_from; k <= k_to; k <<= 1) {
        for (int j = min(k >> 1, kBitonicTile >> 1); j > 0; j >>= 1) {
            for (int e = threadIdx.x; e < kBitonicTile / 2; e += blockDim.x) {
                const int i = 2 * e - (e & (j - 1));   // the lower index of the pair
                const int p = i + j;
                const size_t gi = base + i;
                const bool up = (gi & (size_t)k) == 0;
                const unsigned long long a = s[i], b = s[p];
                if ((a > b) == up) { s[i] = b; s[p] = a; }
            }
            __syncthreads();
        }
    }
    for (int e = threadIdx.x; e < kBitonicTile; e += blockDim.x) keys[base + e] = s[e];
}
__global__ void k_bitonic_global(unsigned long long* keys, int n_pad, int k, int j) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_pad / 2; e += gridDim.x * blockDim.x) {
        const size_t i = 2 * (size_t)e - ((size_t)e & (size_t)(j - 1));
        const size_t p = i + (size_t)j;
        const bool up = (i & (size_t)k) == 0;
        const unsigned long long a = keys[i], b = keys[p];
        if ((a > b) == up) { keys[i] = b; keys[p] = a; }
    }
}

// 3. Karras hierarchy.  Internal nodes 0 .. n-2, leaves n-1 .. 2n-2 (leaf n-1+p holds the
// sorted triangle p).  child[2i], child[2i+1]; parent of every node (root: -1); the leaf
// range [first, last] of every node.
__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(keys[i] ^ keys[j]);
}
__global__ void k_hierarchy(const unsigned long long* keys, int n, int* child, int* parent, int2* range) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int s = 0;
        for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        const int g = i + s * d + min(d, 0);
        const int first = min(i, j), last = max(i, j);
        const int left = first == g ? (n - 1) + g : g;
        const int right = last == g + 1 ? (n - 1) + g + 1 : g + 1;
        child[2 * i] = left;
        child[2 * i + 1] = right;
        parent[left] = i;
        parent[right] = i;
        range[i] = make_int2(first, last);
        if (i == 0) parent[0] = -1;
    }
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        range[(n - 1) + p] = make_int2(p, p);
    if (n == 1 && blockIdx.x == 0 && threadIdx.x == 0) parent[0] = -1;
}

// 4. Boxes bottom-up (nlo / nhi per node; leaves from the sorted triangles).
__global__ void k_refit(const unsigned long long* keys, const float4* lo, const float4* hi, int n, const int* child,
                        const int* parent, unsigned* arrivals, float4* nlo, float4* nhi) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int t = (int)(keys[p] & 0xFFFFFFFFull);
        int node = (n - 1) + p;
        nlo[node] = lo[t];
        nhi[node] = hi[t];
        __threadfence();
        node = parent[node];
        while (node >= 0) {
            if (atomicAdd(&arrivals[node], 1u) == 0u) break;   // the sibling's thread comes back here
            __threadfence();
            const int a = child[2 * node], b = child[2 * node + 1];
            // the sibling's box was written by another thread: read it past the L1
            const float4 la = __ldcg(nlo + a), lb = __ldcg(nlo + b), ha = __ldcg(nhi + a), hb = __ldcg(nhi + b);
            nlo[node] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.0f);
            nhi[node] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.0f);
            __threadfence();
            node = parent[node];
        }
    }
}

// 5. The binary walk's layout: preorder index of node v = depth(v) + 2 first(v) - right
// turns on its root path (the nodes before v are its ancestors and the subtrees to the
// left of its path, 2k - 1 nodes per subtree of k leaves).  Internal: (lo, -(axis + 1))
// (hi, right child); leaf: (lo, 1) (hi, sorted position).  Also the deepest level.
__global__ void k_binary_layout(int n, const int* child, const int* parent, const int2* range, const float4* nlo,
                                const float4* nhi, float4* out, int* max_depth) {
    const int total = 2 * n - 1;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int depth = 0, right = 0;
        for (int c = v, p = parent[v]; p >= 0; c = p, p = parent[p]) {
            ++depth;
            if (child[2 * p + 1] == c) ++right;
        }
        const int pre = depth + 2 * range[v].x - right;
        const float4 a = nlo[v], b = nhi[v];
        if (v >= n - 1) {
            out[2 * pre] = make_float4(a.x, a.y, a.z, 1.0f);
            out[2 * pre + 1] = make_float4(b.x, b.y, b.z, (float)(v - (n - 1)));
        } else {
            const int r = child[2 * v + 1];
            const int rpre = (depth + 1) + 2 * range[r].x - (right + 1);
            const float ex = b.x - a.x, ey = b.y - a.y, ez = b.z - a.z;
            const int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
            out[2 * pre] = make_float4(a.x, a.y, a.z, -(float)(axis + 1));
            out[2 * pre + 1] = make_float4(b.x, b.y, b.z, (float)rpre);
        }
        atomicMax(max_depth, depth);
    }
}

// 6. Compressed wide nodes, one level of tasks (binary node, wide node index) per launch.
__device__ __forceinline__ float next_down(float f) {
    if (f == 0.0f) return -__int_as_float(1);
    const unsigned u = __float_as_uint(f);
    return __uint_as_float(f > 0.0f ? u - 1u : u + 1u);
}
__device__ __forceinline__ float f32_floor(double v) {
    const float f = (float)v;
    return (double)f > v ? next_down(f) : f;
}
__device__ __forceinline__ float pow2_of(int b) { return __uint_as_float((unsigned)b << 23); }
__device__ __forceinline__ int exp_byte(float p, double hi) {
    const double extent = hi - (double)p;
    int b = extent > 0.0 ? max(1, (int)ceil(log2(extent / 255.0)) + 127) : 1;
    while (b < 255 && (double)(float)((double)p + 255.0 * (double)pow2_of(b)) < hi) ++b;
    return b;
}
__device__ __forceinline__ int quant(double v, float p, float s, bool up) {
    int q = up ? (int)ceil((v - (double)p) / (double)s) : (int)floor((v - (double)p) / (double)s);
    q = max(0, min(255, q));
    if (up) {
        while ((double)(float)((double)p + (double)q * (double)s) < v && q < 255) ++q;
    } else {
        while ((double)(float)((double)p + (double)q * (double)s) > v && q > 0) --q;
    }
    return q;
}
__device__ __forceinline__ float half_area(float4 a, float4 b) {
    const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    return dx * dy + dy * dz + dz * dx;
}
// counters: [0] wide nodes allocated, [1] leaf items placed, [2] next level's tasks,
// [3] error flag (quantization range)
__global__ void k_collapse(int n, const int* child, const int2* range, const float4* nlo, const float4* nhi,
                           const unsigned long long* keys, const int2* tasks, int n_tasks, int2* next,
                           unsigned* counters, uint32_t* nodes, uint32_t* order) {
    for (int ti = blockIdx.x * blockDim.x + threadIdx.x; ti < n_tasks; ti += gridDim.x * blockDim.x) {
        const int b = tasks[ti].x, w = tasks[ti].y;
        int mem[8];
        int cnt = 0;
        if (b >= n - 1) {
            mem[cnt++] = b;   // a one-triangle mesh: the root is a leaf
        } else {
            mem[cnt++] = child[2 * b];
            mem[cnt++] = child[2 * b + 1];
            while (cnt < 8) {   // open the largest child that cannot be a leaf child
                int best = -1;
                float ba = -1.0f;
                for (int m = 0; m < cnt; ++m) {
                    const int v = mem[m];
                    const int2 r = range[v];
                    if (v >= n - 1 || r.y - r.x + 1 <= 3) continue;
                    const float a = half_area(nlo[v], nhi[v]);
                    if (a > ba) { ba = a; best = m; }
                }
                if (best < 0) break;
                const int v = mem[best];
                mem[best] = child[2 * v];
                mem[cnt++] = child[2 * v + 1];
            }
        }
        float4 plo = nlo[mem[0]], phi = nhi[mem[0]];
        for (int m = 1; m < cnt; ++m) {
            const float4 a = nlo[mem[m]], c = nhi[mem[m]];
            plo = make_float4(fminf(plo.x, a.x), fminf(plo.y, a.y), fminf(plo.z, a.z), 0.0f);
            phi = make_float4(fmaxf(phi.x, c.x), fmaxf(phi.y, c.y), fmaxf(phi.z, c.z), 0.0f);
        }
        // octant slots (the host encoder's rule: child centre against the node centre,
        // collisions to the next free slot)
        const double pcx = ((double)plo.x + phi.x) * 0.5, pcy = ((double)plo.y + phi.y) * 0.5,
                     pcz = ((double)plo.z + phi.z) * 0.5;
        int slot_of[8];
        for (int s = 0; s < 8; ++s) slot_of[s] = -1;
        int n_int = 0, n_items = 0;
        for (int m = 0; m < cnt; ++m) {
            const float4 a = nlo[mem[m]], c = nhi[mem[m]];
            const double cx = ((double)a.x + c.x) * 0.5, cy = ((double)a.y + c.y) * 0.5, cz = ((double)a.z + c.z) * 0.5;
            int s = (cx - pcx > 0 ? 1 : 0) | (cy - pcy > 0 ? 2 : 0) | (cz - pcz > 0 ? 4 : 0);
            while (slot_of[s] >= 0) s = (s + 1) & 7;
            slot_of[s] = m;
            const int2 r = range[mem[m]];
            const int k = r.y - r.x + 1;
            if (k <= 3) n_items += k;
            else ++n_int;
        }
        // the grid first: a node outside the exponent range allocates nothing (its items
        // stay unplaced, which the host reports)
        const float p0 = f32_floor(plo.x), p1 = f32_floor(plo.y), p2 = f32_floor(plo.z);
        const int ebx = exp_byte(p0, phi.x), eby = exp_byte(p1, phi.y), ebz = exp_byte(p2, phi.z);
        if (ebx > 254 || eby > 254 || ebz > 254) { atomicOr(&counters[3], 1u); continue; }
        const int child_base = n_int ? (int)atomicAdd(&counters[0], (unsigned)n_int) : 0;
        const int prim_base = n_items ? (int)atomicAdd(&counters[1], (unsigned)n_items) : 0;
        const int task_base = n_int ? (int)atomicAdd(&counters[2], (unsigned)n_int) : 0;
        const float sx = pow2_of(ebx), sy = pow2_of(eby), sz = pow2_of(ebz);
        uint32_t qlo[24], qhi[24], meta[8];
        for (int s = 0; s < 8; ++s) {
            qlo[s] = qlo[8 + s] = qlo[16 + s] = 255u;
            qhi[s] = qhi[8 + s] = qhi[16 + s] = 0u;
            meta[s] = 0u;
        }
        unsigned imask = 0u;
        int ci = 0, off = 0;
        for (int s = 0; s < 8; ++s) {
            const int m = slot_of[s];
            if (m < 0) continue;
            const int v = mem[m];
            const float4 a = nlo[v], c = nhi[v];
            qlo[s] = (uint32_t)quant(a.x, p0, sx, false);
            qlo[8 + s] = (uint32_t)quant(a.y, p1, sy, false);
            qlo[16 + s] = (uint32_t)quant(a.z, p2, sz, false);
            qhi[s] = (uint32_t)quant(c.x, p0, sx, true);
            qhi[8 + s] = (uint32_t)quant(c.y, p1, sy, true);
            qhi[16 + s] = (uint32_t)quant(c.z, p2, sz, true);
            const int2 r = range[v];
            const int k = r.y - r.x + 1;
            if (k <= 3) {
                meta[s] = ((((1u << k) - 1u) << 5) | (unsigned)off);
                for (int q = 0; q < k; ++q) order[prim_base + off + q] = (uint32_t)(keys[r.x + q] & 0xFFFFFFFFull);
                off += k;
            } else {
                imask |= 1u << s;
                meta[s] = 0x20u | (24u + (unsigned)s);
                next[task_base + ci] = make_int2(v, child_base + ci);
                ++ci;
            }
        }
        uint32_t* o = nodes + 20 * (size_t)w;
        o[0] = __float_as_uint(p0);
        o[1] = __float_as_uint(p1);
        o[2] = __float_as_uint(p2);
        o[3] = (uint32_t)ebx | ((uint32_t)eby << 8) | ((uint32_t)ebz << 16) | (imask << 24);
        o[4] = (uint32_t)child_base;
        o[5] = (uint32_t)prim_base;
        o[6] = meta[0] | (meta[1] << 8) | (meta[2] << 16) | (meta[3] << 24);
        o[7] = meta[4] | (meta[5] << 8) | (meta[6] << 16) | (meta[7] << 24);
        for (int ww = 0; ww < 6; ++ww) {
            const uint32_t* src = ww < 3 ? qlo : qhi;
            const int so = (ww % 3) * 8;
            o[8 + 2 * ww] = src[so] | (src[so + 1] << 8) | (src[so + 2] << 16) | (src[so + 3] << 24);
            o[9 + 2 * ww] = src[so + 4] | (src[so + 5] << 8) | (src[so + 6] << 16) | (src[so + 7] << 24);
        }
    }
}

// 7. Triangle records in a leaf order: (v0, caller index | e1, alpha | e2).
__global__ void k_emit_tris(const float* pos, const unsigned* idx, const float* alpha, const uint32_t* order,
                            const unsigned long long* keys, int n, float4* tri) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned t = order ? order[i] : (unsigned)(keys[i] & 0xFFFFFFFFull);
        const float* a = pos + 3 * (size_t)idx[3 * (size_t)t];
        const float* b = pos + 3 * (size_t)idx[3 * (size_t)t + 1];
        const float* c = pos + 3 * (size_t)idx[3 * (size_t)t + 2];
        tri[3 * (size_t)i] = make_float4(a[0], a[1], a[2], __int_as_float((int)t));
        tri[3 * (size_t)i + 1] = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], alpha ? alpha[t] : -1.0f);
        tri[3 * (size_t)i + 2] = make_float4(c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.0f);
    }
}

}  // namespace lbvh
}  // namespace ptx
