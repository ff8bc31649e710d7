// bvh.cuh — acceleration-structure arms of the scene queries: triangle meshes (binary BVH
// or compressed wide BVH BLAS) and instanced batches (binary TLAS over placements).
//
// Triangle leaf: Moller-Trumbore as the reference's mesh_tri_test
//   (src/components/intersection/mesh/mesh.glsl:41-59), flat geometric normal.
// Binary walk: the stack-DFS of mesh_nearest_bvh (mesh.glsl:162-191) with the padded slab
//   test bvh_aabb_hit (accel/bvh/bvh.glsl:28-36), near child first by the split axis.
// Wide walk: the octant-ordered CWBVH walk (intersection/index.ts:99-158): per-node ray
//   transform, one-FMA quantized slabs, find-MSB child order, node groups on a small stack.
//   Nodes are fetched as five 128-bit loads.
// Placements (intersection/instancing/placement.glsl:19-41): world -> rigid frame by the
//   stored quaternion q and ts = (t_rigid, s); mesh prototypes are intersected in their
//   local frame with the t-preserving (un-normalised) direction.
#pragma once
#include "scene.cuh"

namespace ptx {

#ifndef PTR_CW_NEARFAR
#define PTR_CW_NEARFAR 0
#endif
constexpr float kBvhTfarPad = 1.00000024f;   // BVH_TFAR_PAD (Ize 2013 far-plane pad)
constexpr int kBvhStack = 64;                // BVH_STACK_DEPTH
constexpr int kCwStack = 24;                 // CWBVH_STACK_DEPTH
constexpr unsigned kErrBvhStack = 1u;        // a binary walk dropped a subtree (stack full)
constexpr unsigned kErrCwStack = 2u;         // a wide walk dropped a node group
constexpr unsigned kErrCwGuard = 4u;         // a wide walk hit its iteration guard

struct HitRec { float t, u, v; int region, element, prim; };

// Per-thread work tally (instrumented pass only): the timed kernels pass a null tally,
// which the inlined walks fold away.
struct Work { unsigned nodes, tris, tlas, inst; };

__device__ __forceinline__ void flag_error(const DevScene& S, unsigned bit) {
    if (S.err_flags) atomicOr(S.err_flags, bit);
}

// ---- placement algebra ------------------------------------------------------------------
__device__ __forceinline__ f3 qrot(float4 q, f3 v) {
    f3 qv(q.x, q.y, q.z);
    return v + 2.0f * cross(qv, cross(qv, v) + q.w * v);
}
__device__ __forceinline__ f3 placement_rigid(float4 q, float4 ts, f3 p) { return qrot(q, p) + f3(ts.x, ts.y, ts.z); }
__device__ __forceinline__ f3 placement_normal(float4 q, f3 n) { return qrot(make_float4(-q.x, -q.y, -q.z, q.w), n); }

// ---- triangle leaf --------------------------------------------------------------------
__device__ __forceinline__ bool tri_test(f3 ro, f3 rd, f3 a, f3 e1, f3 e2, float& t) {
    f3 gnorm = cross(e1, e2);
    float det = -dot(rd, gnorm);
    if (fabsf(det) < 1e-12f) return false;
    float invdet = 1.0f / det;
    f3 ao = ro - a;
    f3 dao = cross(ao, rd);
    float u = dot(e2, dao) * invdet;
    float v = -dot(e1, dao) * invdet;
    t = dot(ao, gnorm) * invdet;
    float w = 1.0f - u - v;
    const float E = 1e-6f;
    return u >= -E && v >= -E && w >= -E;
}
__device__ __forceinline__ void load_tri(const float4* tri, int i, f3& a, f3& e1, f3& e2) {
    float4 t0 = __ldg(tri + 3 * i), t1 = __ldg(tri + 3 * i + 1), t2 = __ldg(tri + 3 * i + 2);
    a = xyz(t0); e1 = xyz(t1); e2 = xyz(t2);
}
// The caller's index of the triangle in leaf slot i (stored in the record's first w).
__device__ __forceinline__ int tri_orig(const float4* tri, int i) { return __float_as_int(__ldg(&tri[3 * (size_t)i].w)); }

// Hits at equal t resolve in one order whatever the traversal visits first: the lower
// region index, then the lower instance index (the caller's placement order), then the
// lower triangle index of the caller's mesh.  The oracle's ordered scans give that order,
// so hit IDs agree at ties too.  Node tests keep boxes entered exactly at the current t
// (a tied triangle may sit on the box's near face); leaf tests take t == tmax only when
// it wins the tie.  NoTie: no tie with the incoming tmax is won (a plain mesh region;
// its incoming tmax belongs to an earlier region).
struct NoTie { __device__ __forceinline__ bool operator()() const { return false; } };

// ---- binary BVH walk --------------------------------------------------------------------
__device__ __forceinline__ bool aabb_hit(float4 n0, float4 n1, f3 ro, f3 inv, float tmax) {
    float tx0 = (n0.x - ro.x) * inv.x, tx1 = (n1.x - ro.x) * inv.x;
    float ty0 = (n0.y - ro.y) * inv.y, ty1 = (n1.y - ro.y) * inv.y;
    float tz0 = (n0.z - ro.z) * inv.z, tz1 = (n1.z - ro.z) * inv.z;
    float tn = gmax(gmax(gmin(tx0, tx1), gmin(ty0, ty1)), gmin(tz0, tz1));
    float tf = gmin(gmin(gmax(tx0, tx1), gmax(ty0, ty1)), gmax(tz0, tz1)) * kBvhTfarPad;
    float tenter = gmax(tn, 0.0f);
    return tf >= tenter && tenter <= tmax;
}

// Leaf(off, cnt) -> for nearest walks updates the caller's tmax itself; returns true to
// stop the walk (any-hit found).
template <class Leaf>
__device__ __forceinline__ bool walk_binary(const DevScene& S, const float4* nodes, f3 ro, f3 rd, const float& tmax, Leaf leaf,
                                            unsigned* visits = nullptr) {
    f3 inv(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    int stack[kBvhStack];
    int ptr = 0;
    stack[0] = 0;
    while (ptr >= 0) {
        int ni = stack[ptr];
        ptr--;
        if (visits) (*visits)++;
        float4 n0 = __ldg(nodes + 2 * ni), n1 = __ldg(nodes + 2 * ni + 1);
        if (!aabb_hit(n0, n1, ro, inv, tmax)) continue;
        if (n0.w >= 0.0f) {
            if (leaf((int)n1.w, (int)n0.w)) return true;
        } else {
            int axis = (int)(-n0.w - 1.0f);
            int L = ni + 1, R = (int)n1.w;
            bool nf = (axis == 0 ? rd.x : (axis == 1 ? rd.y : rd.z)) >= 0.0f;
            if (ptr + 2 < kBvhStack) {
                stack[++ptr] = nf ? R : L;
                stack[++ptr] = nf ? L : R;
            } else {
                flag_error(S, kErrBvhStack);
            }
        }
    }
    return false;
}

// ---- compressed wide BVH walk ---------------------------------------------------------------
__device__ __forceinline__ int find_msb24(unsigned v) { return 31 - __clz(v); }
// Byte k of word as a float, exactly: the byte is permuted into the mantissa of 2^23
// (bits 0x4B0000bb) and 2^23 is subtracted.  One PRMT + one FADD on the integer / FMA pipes
// instead of an I2F conversion (the conversion unit was the walk's busiest pipe).
__device__ __forceinline__ float byte_as_float(unsigned word, unsigned k) {
    return __fadd_rn(__uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u | k)), -8388608.0f);
}
__device__ __forceinline__ float clamp_dir(float d) { return fabsf(d) < 1e-20f ? (d < 0.0f ? -1e-20f : 1e-20f) : d; }

// Per-ray set-up of a wide walk: the direction with zero components clamped (slab
// reciprocals stay finite), its reciprocal and the inverted octant that orders children.
struct CwRay { f3 inv; unsigned octinv; };
__device__ __forceinline__ CwRay cw_ray(f3 rd) {
    f3 rdc(clamp_dir(rd.x), clamp_dir(rd.y), clamp_dir(rd.z));
    CwRay c;
    c.octinv = 7u - ((rdc.x < 0.0f ? 1u : 0u) | (rdc.y < 0.0f ? 2u : 0u) | (rdc.z < 0.0f ? 4u : 0u));
    c.inv = f3(1.0f / rdc.x, 1.0f / rdc.y, 1.0f / rdc.z);
    return c;
}
// One CWBVH node against the ray: the hit internal children as an octant-ordered bit mask
// (hits, with the node's child base and internal-child mask for the group) and the hit
// leaf triangles as bits above the node's triangle base (leaf_bits, leaf_base).
struct CwNodeHits { unsigned hits, leaf_bits, child_base, imask, leaf_base; };
__device__ __forceinline__ CwNodeHits cw_node(const uint4* nd, f3 ro, const CwRay& cr, float tmax) {
    uint4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3), n4 = __ldg(nd + 4);
    f3 p(__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z));
    f3 dq = f3(__uint_as_float((n0.w & 0xFFu) << 23), __uint_as_float(((n0.w >> 8) & 0xFFu) << 23),
               __uint_as_float(((n0.w >> 16) & 0xFFu) << 23)) * cr.inv;
    f3 oq = (p - ro) * cr.inv;
#if PTR_CW_NEARFAR
    // the ray's octant picks which quantized bound of each axis is the near plane (the slab
    // values are the same as min / max of the two, without computing both orders)
    const bool nx = (cr.octinv & 1u) == 0u, ny = (cr.octinv & 2u) == 0u, nz = (cr.octinv & 4u) == 0u;
#endif
    CwNodeHits o;
    o.hits = 0u;
    o.leaf_bits = 0u;
    o.child_base = n1.x;
    o.leaf_base = n1.y;
    o.imask = (n0.w >> 24) & 0xFFu;
#pragma unroll
    for (unsigned sl = 0u; sl < 8u; sl++) {
        const unsigned sh = 8u * (sl & 3u);
        unsigned m = ((sl < 4u ? n1.z : n1.w) >> sh) & 0xFFu;
        if (m == 0u) continue;
        const unsigned kb = sl & 3u;
        const unsigned wlx = sl < 4u ? n2.x : n2.y, wly = sl < 4u ? n2.z : n2.w, wlz = sl < 4u ? n3.x : n3.y;
        const unsigned whx = sl < 4u ? n3.z : n3.w, why = sl < 4u ? n4.x : n4.y, whz = sl < 4u ? n4.z : n4.w;
#if PTR_CW_NEARFAR
        float nearx = __fmaf_rn(byte_as_float(nx ? whx : wlx, kb), dq.x, oq.x);
        float fary = __fmaf_rn(byte_as_float(ny ? wly : why, kb), dq.y, oq.y);
        float neary = __fmaf_rn(byte_as_float(ny ? why : wly, kb), dq.y, oq.y);
        float farx = __fmaf_rn(byte_as_float(nx ? wlx : whx, kb), dq.x, oq.x);
        float nearz = __fmaf_rn(byte_as_float(nz ? whz : wlz, kb), dq.z, oq.z);
        float farz = __fmaf_rn(byte_as_float(nz ? wlz : whz, kb), dq.z, oq.z);
        float tn = gmax(gmax(nearx, neary), gmax(nearz, 0.0f));
        float tf = gmin(gmin(farx, fary), gmin(farz, tmax)) * kBvhTfarPad;
#else
        float qlx = byte_as_float(wlx, kb), qly = byte_as_float(wly, kb), qlz = byte_as_float(wlz, kb);
        float qhx = byte_as_float(whx, kb), qhy = byte_as_float(why, kb), qhz = byte_as_float(whz, kb);
        float lox = __fmaf_rn(qlx, dq.x, oq.x), hix = __fmaf_rn(qhx, dq.x, oq.x);
        float loy = __fmaf_rn(qly, dq.y, oq.y), hiy = __fmaf_rn(qhy, dq.y, oq.y);
        float loz = __fmaf_rn(qlz, dq.z, oq.z), hiz = __fmaf_rn(qhz, dq.z, oq.z);
        float tn = gmax(gmax(gmin(lox, hix), gmin(loy, hiy)), gmax(gmin(loz, hiz), 0.0f));
        float tf = gmin(gmin(gmax(lox, hix), gmax(loy, hiy)), gmin(gmax(loz, hiz), tmax)) * kBvhTfarPad;
#endif
        if (tf < tn) continue;
        if ((m & 0xE0u) == 0x20u && (m & 0x1Fu) >= 24u) o.hits |= 1u << ((((m & 0x1Fu) - 24u) ^ cr.octinv) & 7u);
        else o.leaf_bits |= (m >> 5) << (m & 0x1Fu);
    }
    return o;
}
// The next child of a node group: pops the highest hit bit and maps it to the child index.
__device__ __forceinline__ unsigned cw_next_child(unsigned& g_hits, unsigned g_base, unsigned g_imask, unsigned octinv) {
    int bit = find_msb24(g_hits);
    g_hits &= ~(1u << (unsigned)bit);
    unsigned slot = ((unsigned)bit ^ octinv) & 7u;
    return g_base + __popc(g_imask & ((1u << slot) - 1u));
}

// Leaf(item) for one leaf item index (wide-order); returns true to stop.
template <class Leaf>
__device__ __forceinline__ bool walk_wide(const DevScene& S, const uint4* nodes, f3 ro, f3 rd, const float& tmax, Leaf leaf,
                                          unsigned* visits = nullptr) {
    const CwRay cr = cw_ray(rd);
    // node-group stack in thread-local memory (a wide TLAS walk nests a BLAS walk inside
    // its leaves, each with its own stack)
    uint2 stack[kCwStack];
    int ptr = -1;
    unsigned g_base = 0u, g_hits = 1u << (cr.octinv & 7u), g_imask = 1u;
    for (int guard = 0; guard < 65536; guard++) {
        if (g_hits == 0u) {   // pop a group and go on to its next node in the same iteration
            if (ptr < 0) return false;
            const uint2 top = stack[ptr];
            g_base = top.x;
            g_hits = top.y & 0xFFu;
            g_imask = top.y >> 8;
            ptr--;
        }
        const unsigned child = cw_next_child(g_hits, g_base, g_imask, cr.octinv);
        if (g_hits != 0u) {
            if (ptr + 1 < kCwStack) { ptr++; stack[ptr] = make_uint2(g_base, g_hits | (g_imask << 8)); }
            else flag_error(S, kErrCwStack);
        }
        if (visits) (*visits)++;
        const CwNodeHits nh = cw_node(nodes + 5 * (size_t)child, ro, cr, tmax);
        unsigned leaf_bits = nh.leaf_bits;
        while (leaf_bits != 0u) {
            int lb = find_msb24(leaf_bits);
            leaf_bits &= ~(1u << (unsigned)lb);
            if (leaf((int)nh.leaf_base + lb)) return true;
        }
        if (nh.hits != 0u) { g_base = nh.child_base; g_hits = nh.hits; g_imask = nh.imask; }
        else g_hits = 0u;
    }
    flag_error(S, kErrCwGuard);
    return false;
}

// ---- one mesh BLAS in a given frame (ro/rd already in the mesh's local frame) --------------
// tie_in(): whether this walk wins a tie with the incoming tmax (a lower instance index
// than the hit that set it); ties inside the walk go to the lower triangle index.
template <class Tie = NoTie>
__device__ __forceinline__ bool mesh_nearest(const DevScene& S, const DevMesh& m, f3 ro, f3 rd, float& tmax, int& prim,
                                             Work* w = nullptr, Tie tie_in = Tie{}) {
    bool found = false;
    const float4* tri = (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) ? m.tri_w : m.tri;
    auto take = [&](int i, float t) {
        return t > 0.0f && (t < tmax || (t == tmax && (found ? tri_orig(tri, i) < tri_orig(tri, prim) : tie_in())));
    };
    if (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) {
        walk_wide(S, m.cwbvh, ro, rd, tmax, [&](int i) {
            f3 a, e1, e2;
            if (w) w->tris++;
            load_tri(tri, i, a, e1, e2);
            float t;
            if (tri_test(ro, rd, a, e1, e2, t) && take(i, t)) { tmax = t; prim = i; found = true; }
            return false;
        }, w ? &w->nodes : nullptr);
    } else {
        walk_binary(S, m.bvh, ro, rd, tmax, [&](int off, int cnt) {
            for (int i = off; i < off + cnt; ++i) {
                f3 a, e1, e2;
                if (w) w->tris++;
                load_tri(tri, i, a, e1, e2);
                float t;
                if (tri_test(ro, rd, a, e1, e2, t) && take(i, t)) { tmax = t; prim = i; found = true; }
            }
            return false;
        }, w ? &w->nodes : nullptr);
    }
    return found;
}
__device__ __forceinline__ bool mesh_any(const DevScene& S, const DevMesh& m, f3 ro, f3 rd, float max_dist, Work* w = nullptr) {
    if (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) {
        const float4* tri = m.tri_w;
        return walk_wide(S, m.cwbvh, ro, rd, max_dist, [&](int i) {
            f3 a, e1, e2;
            if (w) w->tris++;
            load_tri(tri, i, a, e1, e2);
            float t;
            return tri_test(ro, rd, a, e1, e2, t) && t > 0.0f && t < max_dist;
        }, w ? &w->nodes : nullptr);
    }
    const float4* tri = m.tri;
    return walk_binary(S, m.bvh, ro, rd, max_dist, [&](int off, int cnt) {
        for (int i = off; i < off + cnt; ++i) {
            f3 a, e1, e2;
            if (w) w->tris++;
            load_tri(tri, i, a, e1, e2);
            float t;
            if (tri_test(ro, rd, a, e1, e2, t) && t > 0.0f && t < max_dist) return true;
        }
        return false;
    }, w ? &w->nodes : nullptr);
}

// ---- instanced meshes: binary TLAS over CWBVH BLAS as one flat loop -------------------------
// The nested form (accel_closest / accel_any) runs each instance's BLAS walk to the end
// inside the TLAS leaf that reached it, so in a warp every lane whose TLAS step did not
// enter an instance waits for the other lanes' whole BLAS walks.  Here one loop advances
// each lane by one step — a TLAS node, the next instance of the current TLAS leaf, or a
// BLAS node with its leaf triangles — so lanes at different levels proceed together.  Per
// lane the sequence of node visits, leaf tests and tmax updates is that of the nested
// walks, so hits (and the work tallies) are identical.  ANY: stop at the first triangle hit.
// The walk as a resumable state: init() for one ray, then step() until it reports the end.
// A step runs the bookkeeping transitions in line instead of spending a loop iteration on
// each: a TLAS leaf enters its first instance and that instance's BLAS root in the same
// step, a group pop goes straight on to the popped node, and a finished BLAS walk hands
// over to the next instance or TLAS node at the start of the next step.
struct InstFlat {
    f3 winv;                               // TLAS: world-ray reciprocal, node stack, leaf range
    int tstack[kBvhStack];
    int tptr, li, lend;
    f3 ro, rd;                             // BLAS: the entered instance's frame and group stack
    CwRay cr;
    uint2 stack[kCwStack];
    int ptr;
    unsigned g_base, g_hits, g_imask;
    float t, t_near;                       // t: BLAS tmax; t_near: TLAS culling distance
    int prim, inst, phase;                 // phase: 0 TLAS node, 1 next instance, 2 BLAS step
    bool found;
    __device__ __forceinline__ void init(const Ray& r, float t0) {
        winv = f3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
        tptr = 0;
        tstack[0] = 0;
        li = lend = 0;
        ptr = -1;
        g_hits = 0u;
        t_near = t0;
        phase = 0;
        found = false;
    }
    // One step; false once the query is over.  Closest (ANY = false): h takes every nearer
    // instance hit.  Any-hit: returns false with `found` set at the first hit.
    template <bool ANY>
    __device__ __forceinline__ bool step(const DevScene& S, const DevBatch& b, const DevMesh& m, int region, const Ray& r,
                                         HitRec& h, float max_dist, Work* w) {
        if (phase == 2 && g_hits == 0u && ptr < 0) {   // the BLAS walk is done
            if (!ANY && found) {
                t_near = t;
                h.t = t;
                h.region = region;
                h.element = inst;
                h.prim = prim;
            }
            phase = li < lend ? 1 : 0;
        }
        if (phase == 0) {
            if (tptr < 0) return false;
            const int ni = tstack[tptr--];
            if (w) w->tlas++;
            const float4 n0 = __ldg(b.tlas + 2 * ni), n1 = __ldg(b.tlas + 2 * ni + 1);
            if (!aabb_hit(n0, n1, r.o, winv, t_near)) return true;
            if (n0.w >= 0.0f) {
                li = (int)n1.w;
                lend = li + (int)n0.w;
                phase = 1;                 // enter its first instance in this step
            } else {
                const int axis = (int)(-n0.w - 1.0f);
                const int L = ni + 1, R = (int)n1.w;
                const bool nf = (axis == 0 ? r.d.x : (axis == 1 ? r.d.y : r.d.z)) >= 0.0f;
                if (tptr + 2 < kBvhStack) {
                    tstack[++tptr] = nf ? R : L;
                    tstack[++tptr] = nf ? L : R;
                } else {
                    flag_error(S, kErrBvhStack);
                }
                return true;
            }
        }
        if (phase == 1) {
            if (li >= lend) { phase = 0; return true; }
            inst = li++;
            const float4 q = __ldg(b.place + 2 * inst), ts = __ldg(b.place + 2 * inst + 1);
            const float s = ts.w;
            if (w) w->inst++;
            ro = placement_rigid(q, ts, r.o) / s;
            rd = qrot(q, r.d) / s;
            cr = cw_ray(rd);
            ptr = -1;
            g_base = 0u;
            g_hits = 1u << (cr.octinv & 7u);
            g_imask = 1u;
            t = t_near;
            prim = -1;
            found = false;
            phase = 2;                     // and walk its BLAS root in this step
        }
        if (g_hits == 0u) {                // pop a group (the stack is not empty here)
            const uint2 top = stack[ptr];
            g_base = top.x;
            g_hits = top.y & 0xFFu;
            g_imask = top.y >> 8;
            ptr--;
        }
        const unsigned child = cw_next_child(g_hits, g_base, g_imask, cr.octinv);
        if (g_hits != 0u) {
            if (ptr + 1 < kCwStack) { ptr++; stack[ptr] = make_uint2(g_base, g_hits | (g_imask << 8)); }
            else flag_error(S, kErrCwStack);
        }
        if (w) w->nodes++;
        const CwNodeHits nh = cw_node(m.cwbvh + 5 * (size_t)child, ro, cr, ANY ? max_dist : t);
        unsigned leaf_bits = nh.leaf_bits;
        while (leaf_bits != 0u) {
            const int lb = find_msb24(leaf_bits);
            leaf_bits &= ~(1u << (unsigned)lb);
            const int i = (int)nh.leaf_base + lb;
            f3 a, e1, e2;
            if (w) w->tris++;
            load_tri(m.tri_w, i, a, e1, e2);
            float tt;
            if (ANY) {
                if (tri_test(ro, rd, a, e1, e2, tt) && tt > 0.0f && tt < max_dist) {
                    found = true;
                    return false;
                }
            } else if (tri_test(ro, rd, a, e1, e2, tt) && tt > 0.0f &&
                       (tt < t || (tt == t && (found ? tri_orig(m.tri_w, i) < tri_orig(m.tri_w, prim)
                                                     : (h.region == region && __ldg(b.inst_id + inst) < __ldg(b.inst_id + h.element)))))) {
                t = tt;
                prim = i;
                found = true;
            }
        }
        if (nh.hits != 0u) { g_base = nh.child_base; g_hits = nh.hits; g_imask = nh.imask; }
        else g_hits = 0u;
        return true;
    }
};
constexpr int kFlatGuard = 1 << 22;        // steps of one query before the walk gives up
template <bool ANY>
__device__ __forceinline__ bool inst_mesh_flat(const DevScene& S, const DevBatch& b, int region, const Ray& r, HitRec& h,
                                               float max_dist, Work* w) {
    const DevMesh& m = S.meshes[b.proto_mesh];
    InstFlat f;
    f.init(r, ANY ? max_dist : h.t);
    for (int guard = 0; guard < kFlatGuard; ++guard)
        if (!f.step<ANY>(S, b, m, region, r, h, max_dist, w)) return ANY && f.found;
    flag_error(S, kErrCwGuard);
    return false;
}
// The flat loop applies to mesh prototypes walked as CWBVH under the binary TLAS
// (PTR_FLAT_INST=0 builds keep the nested walks everywhere).
#ifndef PTR_FLAT_INST
#define PTR_FLAT_INST 1
#endif
__device__ __forceinline__ bool inst_mesh_flat_ok(const DevScene& S, const DevBatch& b) {
    return PTR_FLAT_INST && b.proto_shape == PTR_SHAPE_MESH && S.accel == PTR_ACCEL_CWBVH &&
           !(S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w) && S.meshes[b.proto_mesh].cwbvh != nullptr;
}

// ---- region arms ------------------------------------------------------------------------
__device__ __forceinline__ void accel_closest(const DevScene& S, const ptr_region& g, int region, const Ray& r, HitRec& h,
                                              Work* w = nullptr) {
    if (g.shape == PTR_SHAPE_MESH) {
        const DevMesh& m = S.meshes[g.ref];
        int prim = -1;
        float t = h.t;
        if (mesh_nearest(S, m, r.o, r.d, t, prim, w)) {
            h.t = t;
            h.region = region;
            h.element = 0;
            h.prim = prim;
        }
        return;
    }
    const DevBatch& b = S.batches[g.ref];
    if (inst_mesh_flat_ok(S, b)) {
        inst_mesh_flat<false>(S, b, region, r, h, 0.0f, w);
        return;
    }
    float t_near = h.t;
    const bool wide = S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w;
    const float4* place = wide ? b.place_w : b.place;
    const int* inst_id = wide ? b.inst_id_w : b.inst_id;
    // an instance wins a tie with the current hit when that hit is an instance of this
    // batch with a higher placement index
    auto wins_tie = [&](int i) { return h.region == region && __ldg(inst_id + i) < __ldg(inst_id + h.element); };
    // one instance: the params-tier sphere, or the mesh prototype in the placement's frame
    auto instance = [&](int i) {
        if (b.proto_shape == PTR_SHAPE_SPHERE) {
            float4 rec = __ldg(place + 2 * i);
            float t;
            if (sphere_intersect(r, xyz(rec), rec.w, t) && (t < t_near || (t == t_near && wins_tie(i)))) {
                t_near = t; h.t = t; h.region = region; h.element = i; h.prim = -1;
            }
        } else {
            float4 q = __ldg(place + 2 * i), ts = __ldg(place + 2 * i + 1);
            float s = ts.w;
            if (w) w->inst++;
            f3 ro = placement_rigid(q, ts, r.o) / s;
            f3 rd = qrot(q, r.d) / s;
            int prim = -1;
            float t = t_near;
            if (mesh_nearest(S, S.meshes[b.proto_mesh], ro, rd, t, prim, w, [&] { return wins_tie(i); })) {
                t_near = t; h.t = t; h.region = region; h.element = i; h.prim = prim;
            }
        }
    };
    if (wide) {   // the reference's CWBVH instance accel (intersection/index.ts:99-158)
        walk_wide(S, b.tlas_w, r.o, r.d, t_near, [&](int i) { instance(i); return false; }, w ? &w->tlas : nullptr);
        return;
    }
    walk_binary(S, b.tlas, r.o, r.d, t_near, [&](int off, int cnt) {
        for (int i = off; i < off + cnt; ++i) instance(i);
        return false;
    }, w ? &w->tlas : nullptr);
}

__device__ __forceinline__ bool accel_any(const DevScene& S, const ptr_region& g, const Ray& r, float max_dist,
                                          Work* w = nullptr) {
    if (g.shape == PTR_SHAPE_MESH) return mesh_any(S, S.meshes[g.ref], r.o, r.d, max_dist, w);
    const DevBatch& b = S.batches[g.ref];
    if (inst_mesh_flat_ok(S, b)) {
        HitRec unused;
        return inst_mesh_flat<true>(S, b, 0, r, unused, max_dist, w);
    }
    const bool wide = S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w;
    const float4* place = wide ? b.place_w : b.place;
    auto instance = [&](int i) -> bool {
        if (b.proto_shape == PTR_SHAPE_SPHERE) {
            float4 rec = __ldg(place + 2 * i);
            float t;
            return sphere_intersect(r, xyz(rec), rec.w, t) && t < max_dist;
        }
        float4 q = __ldg(place + 2 * i), ts = __ldg(place + 2 * i + 1);
        float s = ts.w;
        if (w) w->inst++;
        f3 ro = placement_rigid(q, ts, r.o) / s;
        f3 rd = qrot(q, r.d) / s;
        return mesh_any(S, S.meshes[b.proto_mesh], ro, rd, max_dist, w);
    };
    if (wide) return walk_wide(S, b.tlas_w, r.o, r.d, max_dist, instance, w ? &w->tlas : nullptr);
    return walk_binary(S, b.tlas, r.o, r.d, max_dist, [&](int off, int cnt) {
        for (int i = off; i < off + cnt; ++i)
            if (instance(i)) return true;
        return false;
    }, w ? &w->tlas : nullptr);
}

// Containment of an instanced SPHERE batch (the TLAS point descent of scene_region_at):
// the least-negative signed distance among the instances that contain p, else 1e20.
// Mesh batches are thin (no containment).
__device__ __forceinline__ float accel_region_sdf(const DevScene& S, const ptr_region& g, f3 p) {
    const DevBatch& b = S.batches[g.ref];
    if (b.proto_shape != PTR_SHAPE_SPHERE) return 1.0e20f;
    float best = -1.0e20f;
    bool any = false;
    int stack[kBvhStack];
    int ptr = 0;
    stack[0] = 0;
    while (ptr >= 0) {
        int ni = stack[ptr];
        ptr--;
        float4 n0 = __ldg(b.tlas + 2 * ni), n1 = __ldg(b.tlas + 2 * ni + 1);
        if (!(p.x >= n0.x && p.y >= n0.y && p.z >= n0.z && p.x <= n1.x && p.y <= n1.y && p.z <= n1.z)) continue;
        if (n0.w >= 0.0f) {
            int off = (int)n1.w, cnt = (int)n0.w;
            for (int i = off; i < off + cnt; ++i) {
                float4 rec = __ldg(b.place + 2 * i);
                float ds = length(p - xyz(rec)) - rec.w;
                if (ds < 0.0f && ds > best) { best = ds; any = true; }
            }
        } else {
            int L = ni + 1, R = (int)n1.w;
            if (ptr + 2 < kBvhStack) { stack[++ptr] = L; stack[++ptr] = R; }
            else flag_error(S, kErrBvhStack);
        }
    }
    return any ? best : 1.0e20f;
}

// Hit normals of an acceleration-structure hit (world space): shading normal (returned)
// and the geometric normal (h.ng), plus eps and the per-triangle alpha.
__device__ __forceinline__ f3 accel_hit_normal(const DevScene& S, const ptr_region& g, const HitRec& hr, const Ray&, Hit& h, f3& ng) {
    h.eps = fp_uncertainty(h.p);
    if (g.shape == PTR_SHAPE_INSTANCES) {
        const DevBatch& b = S.batches[g.ref];
        // hr.element indexes the placements of the TLAS the hit was found with
        const float4* place = (S.inst_accel == PTR_ACCEL_CWBVH && b.tlas_w) ? b.place_w : b.place;
        if (b.proto_shape == PTR_SHAPE_SPHERE) {
            float4 rec = __ldg(place + 2 * hr.element);
            f3 n = normalize(h.p - xyz(rec));
            ng = n;   // a primitive's normal is its true surface normal (set from frame.n)
            return n;
        }
        const DevMesh& m = S.meshes[b.proto_mesh];
        float4 q = __ldg(place + 2 * hr.element);
        const float4* tri = (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) ? m.tri_w : m.tri;
        f3 a, e1, e2;
        load_tri(tri, hr.prim, a, e1, e2);
        f3 gl = cross(e1, e2);
        float al = __ldg(&tri[3 * hr.prim + 1].w);
        if (al >= 0.0f) h.alpha = al;
        ng = normalize(placement_normal(q, gl));
        return normalize(placement_normal(q, gl));
    }
    const DevMesh& m = S.meshes[g.ref];
    const float4* tri = (S.accel == PTR_ACCEL_CWBVH && m.cwbvh) ? m.tri_w : m.tri;
    f3 a, e1, e2;
    load_tri(tri, hr.prim, a, e1, e2);
    f3 gl = cross(e1, e2);
    float al = __ldg(&tri[3 * hr.prim + 1].w);
    if (al >= 0.0f) h.alpha = al;
    ng = normalize(gl);
    return normalize(gl);
}

}  // namespace ptx
