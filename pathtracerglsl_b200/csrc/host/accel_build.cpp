// accel_build.cpp — host builders of the acceleration structures the device walks.
//
// binary BVH: the binned-SAH build over a flat AABB list of the reference
//   (src/components/accel/bvh/bvh.ts:132-343 buildBVHCore, :344-383 buildBVHNodesFlat):
//   12 bins per axis binned in one pass, prefix/suffix sweeps, cost A_L*N_L + A_R*N_R
//   against the leaf cost A*N, in-place partition, median fallback.  The float
//   semantics are the reference's (boxes in double, centroids and sweep areas stored as
//   float, node boxes stored as float) so the trees are the same trees.
//   Node: 8 floats (min.xyz, A) (max.xyz, B); A >= 0 leaf (count = A, offset = B),
//   A < 0 internal (axis = -A-1, right child = B, left child = index + 1).
// CWBVH: the compressed wide BVH of Ylitie, Karras & Laine (HPG 2017) as the reference
//   builds it (src/components/accel/cwbvh/cwbvh.ts:80-372): binary SAH tree with one
//   item per leaf, bottom-up collapse dynamic program (paper Eq. 5-8), octant slot
//   assignment, conservative 8-bit quantization against per-node power-of-two grids,
//   80-byte nodes (20 u32).
#include "accel_build.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace ptx_host {

namespace {

constexpr int kBins = 12;
constexpr double kInf = std::numeric_limits<double>::infinity();

struct Box6 { double v[6]; };

inline void reset_box(double* b) {
    b[0] = b[1] = b[2] = kInf;
    b[3] = b[4] = b[5] = -kInf;
}
inline void grow_box(double* b, const double* s) {
    for (int a = 0; a < 3; ++a) {
        if (s[a] < b[a]) b[a] = s[a];
        if (s[3 + a] > b[3 + a]) b[3 + a] = s[3 + a];
    }
}
inline double box_area(const double* b) {
    double dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
    const double* boxes;
    int n;
    int leaf_size;
    bool always_split;
    std::vector<float> cen[3];
    std::vector<uint32_t> order;
    std::vector<float>* nodes;   // 8 floats per node
    int node_count = 0;
    int max_depth = 0;

    int emit(int start, int end, int depth) {
        if (depth > max_depth) max_depth = depth;
        const int node = node_count++;
        double bounds[6], cb[6];
        reset_box(bounds);
        reset_box(cb);
        for (int i = start; i < end; ++i) {
            const uint32_t t = order[i];
            const double* bx = boxes + 6 * (size_t)t;
            for (int a = 0; a < 3; ++a) {
                if (bx[a] < bounds[a]) bounds[a] = bx[a];
                if (bx[3 + a] > bounds[3 + a]) bounds[3 + a] = bx[3 + a];
                const double c = cen[a][t];
                if (c < cb[a]) cb[a] = c;
                if (c > cb[3 + a]) cb[3 + a] = c;
            }
        }
        const int count = end - start;
        auto leaf = [&]() {
            float* o = nodes->data() + 8 * (size_t)node;
            o[0] = (float)bounds[0]; o[1] = (float)bounds[1]; o[2] = (float)bounds[2];
            o[3] = (float)count;
            o[4] = (float)bounds[3]; o[5] = (float)bounds[4]; o[6] = (float)bounds[5];
            o[7] = (float)start;
            return node;
        };
        if (count <= leaf_size) return leaf();

        int best_axis = -1, best_split = -1;
        double best_cost = kInf;
        bool valid[3];
        double scale[3];
        for (int a = 0; a < 3; ++a) {
            valid[a] = cb[3 + a] - cb[a] >= 1e-12;
            scale[a] = valid[a] ? kBins / (cb[3 + a] - cb[a]) : 0.0;
        }
        if (valid[0] || valid[1] || valid[2]) {
            double bin_box[3][kBins][6];
            int bin_cnt[3][kBins];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < kBins; ++b) { reset_box(bin_box[a][b]); bin_cnt[a][b] = 0; }
            for (int i = start; i < end; ++i) {
                const uint32_t t = order[i];
                const double* bx = boxes + 6 * (size_t)t;
                for (int a = 0; a < 3; ++a) {
                    if (!valid[a]) continue;
                    int b = (int)std::floor(((double)cen[a][t] - cb[a]) * scale[a]);
                    if (b < 0) b = 0;
                    if (b >= kBins) b = kBins - 1;
                    bin_cnt[a][b]++;
                    grow_box(bin_box[a][b], bx);
                }
            }
            for (int a = 0; a < 3; ++a) {
                if (!valid[a]) continue;
                float left_area[kBins - 1], right_area[kBins - 1];
                int left_cnt[kBins - 1], right_cnt[kBins - 1];
                double acc[6];
                reset_box(acc);
                int c = 0;
                for (int b = 0; b < kBins - 1; ++b) {
                    grow_box(acc, bin_box[a][b]);
                    c += bin_cnt[a][b];
                    left_area[b] = (float)box_area(acc);
                    left_cnt[b] = c;
                }
                reset_box(acc);
                c = 0;
                for (int b = kBins - 1; b > 0; --b) {
                    grow_box(acc, bin_box[a][b]);
                    c += bin_cnt[a][b];
                    right_area[b - 1] = (float)box_area(acc);
                    right_cnt[b - 1] = c;
                }
                for (int b = 0; b < kBins - 1; ++b) {
                    if (left_cnt[b] == 0 || right_cnt[b] == 0) continue;
                    const double cost = (double)left_area[b] * (double)left_cnt[b] + (double)right_area[b] * (double)right_cnt[b];
                    if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = b; }
                }
            }
        }
        if (!always_split) {
            const double leaf_cost = box_area(bounds) * (double)count;
            if (best_axis == -1 || best_cost >= leaf_cost) return leaf();
        }
        int mid = -1;
        if (best_axis != -1) {
            const double plo = cb[best_axis];
            const double s = kBins / (cb[3 + best_axis] - cb[best_axis]);
            const std::vector<float>& c = cen[best_axis];
            int m = start;
            for (int i = start; i < end; ++i) {
                const uint32_t t = order[i];
                int b = (int)std::floor(((double)c[t] - plo) * s);
                if (b < 0) b = 0;
                if (b >= kBins) b = kBins - 1;
                if (b <= best_split) { std::swap(order[i], order[m]); ++m; }
            }
            if (m > start && m < end) mid = m;
        }
        if (mid == -1) mid = (start + end) >> 1;
        const double mn[3] = {bounds[0], bounds[1], bounds[2]};
        const double mx[3] = {bounds[3], bounds[4], bounds[5]};
        emit(start, mid, depth + 1);
        const int right = emit(mid, end, depth + 1);
        float* o = nodes->data() + 8 * (size_t)node;
        o[0] = (float)mn[0]; o[1] = (float)mn[1]; o[2] = (float)mn[2];
        o[3] = (float)(-1 - std::max(best_axis, 0));
        o[4] = (float)mx[0]; o[5] = (float)mx[1]; o[6] = (float)mx[2];
        o[7] = (float)right;
        return node;
    }
};

inline uint32_t float_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bits_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

}  // namespace

BinaryBvh build_bvh(const double* boxes, int n, int leaf_size, bool always_split) {
    BinaryBvh out;
    if (n <= 0) return out;
    Builder b;
    b.boxes = boxes;
    b.n = n;
    b.leaf_size = leaf_size;
    b.always_split = always_split;
    for (int a = 0; a < 3; ++a) {
        b.cen[a].resize(n);
        for (int t = 0; t < n; ++t) b.cen[a][t] = (float)((boxes[6 * (size_t)t + a] + boxes[6 * (size_t)t + 3 + a]) * 0.5);
    }
    b.order.resize(n);
    for (int i = 0; i < n; ++i) b.order[i] = (uint32_t)i;
    out.nodes.assign(8 * (size_t)(2 * n - 1), 0.0f);
    b.nodes = &out.nodes;
    b.emit(0, n, 0);
    out.nodes.resize(8 * (size_t)b.node_count);
    out.node_count = b.node_count;
    out.order = std::move(b.order);
    out.max_depth = b.max_depth;
    return out;
}

WideBvh build_cwbvh(const double* boxes, int n, double c_prim) {
    WideBvh out;
    if (n <= 0) return out;
    BinaryBvh bin = build_bvh(boxes, n, 1, true);
    const float* bn = bin.nodes.data();
    const int BN = bin.node_count;
    auto is_leaf = [&](int i) { return bn[8 * (size_t)i + 3] >= 0.0f; };
    auto right_of = [&](int i) { return (int)bn[8 * (size_t)i + 7]; };

    std::vector<uint32_t> start(BN), end(BN);
    std::vector<float> area_of(BN);
    std::vector<double> fb(6 * (size_t)BN);
    for (int i = BN - 1; i >= 0; --i) {
        const float* q = bn + 8 * (size_t)i;
        const double dx = (double)q[4] - q[0], dy = (double)q[5] - q[1], dz = (double)q[6] - q[2];
        area_of[i] = (float)std::max(0.0, 2.0 * (dx * dy + dy * dz + dz * dx));
        double* f = &fb[6 * (size_t)i];
        if (is_leaf(i)) {
            start[i] = (uint32_t)q[7];
            end[i] = start[i] + (uint32_t)q[3];
            for (int a = 0; a < 3; ++a) { f[a] = kInf; f[3 + a] = -kInf; }
            for (uint32_t k = start[i]; k < end[i]; ++k) {
                const uint32_t item = bin.order[k];
                for (int a = 0; a < 3; ++a) {
                    f[a] = std::min(f[a], boxes[6 * (size_t)item + a]);
                    f[3 + a] = std::max(f[3 + a], boxes[6 * (size_t)item + 3 + a]);
                }
            }
        } else {
            const int l = i + 1, r = right_of(i);
            start[i] = start[l];
            end[i] = end[r];
            for (int a = 0; a < 3; ++a) {
                f[a] = std::min(fb[6 * (size_t)l + a], fb[6 * (size_t)r + a]);
                f[3 + a] = std::max(fb[6 * (size_t)l + 3 + a], fb[6 * (size_t)r + 3 + a]);
            }
        }
    }
    auto prims_of = [&](int i) { return (int)(end[i] - start[i]); };

    // Collapse DP: cost[n][i-1] = C(n, i), i in 1..7 (paper Eq. 5-8), float stores.
    std::vector<float> cost(7 * (size_t)BN);
    std::vector<uint8_t> choice(7 * (size_t)BN);
    const float kInfF = std::numeric_limits<float>::infinity();
    auto distribute = [&](int l, int r, int j) -> double {
        double best = kInf;
        for (int k = std::max(1, j - 7); k < j && k <= 7; ++k) {
            const double c = (double)cost[7 * (size_t)l + k - 1] + (double)cost[7 * (size_t)r + (j - k) - 1];
            if (c < best) best = c;
        }
        return best;
    };
    for (int i2 = BN - 1; i2 >= 0; --i2) {
        const double A = area_of[i2];
        if (is_leaf(i2)) {
            for (int i = 0; i < 7; ++i) { cost[7 * (size_t)i2 + i] = (float)(A * c_prim); choice[7 * (size_t)i2 + i] = 0; }
            continue;
        }
        const int l = i2 + 1, r = right_of(i2);
        const int P = prims_of(i2);
        const double c_leaf = P <= 3 ? A * P * c_prim : kInf;
        const double c_internal = distribute(l, r, 8) + A * 1.0;
        if (c_leaf <= c_internal) { cost[7 * (size_t)i2] = (float)c_leaf; choice[7 * (size_t)i2] = 0; }
        else { cost[7 * (size_t)i2] = (float)c_internal; choice[7 * (size_t)i2] = 1; }
        for (int i = 2; i <= 7; ++i) {
            const double carry = cost[7 * (size_t)i2 + i - 2];
            const double dist = distribute(l, r, i);
            if (dist < carry) { cost[7 * (size_t)i2 + i - 1] = (float)dist; choice[7 * (size_t)i2 + i - 1] = 3; }
            else { cost[7 * (size_t)i2 + i - 1] = (float)carry; choice[7 * (size_t)i2 + i - 1] = 2; }
        }
    }
    (void)kInfF;
    // Forest backtracking (the distribute split re-derived by the same argmin).
    std::vector<int> stack_buf;
    auto forest_of = [&](auto&& self, int node, int i, std::vector<int>& outv) -> void {
        if (i == 1 || is_leaf(node)) { outv.push_back(node); return; }
        const uint8_t ch = choice[7 * (size_t)node + i - 1];
        if (ch == 2) { self(self, node, i - 1, outv); return; }
        const int l = node + 1, r = right_of(node);
        int best_k = -1;
        double best = kInf;
        for (int k = std::max(1, i - 7); k < i && k <= 7; ++k) {
            const double c = (double)cost[7 * (size_t)l + k - 1] + (double)cost[7 * (size_t)r + (i - k) - 1];
            if (c < best) { best = c; best_k = k; }
        }
        self(self, l, best_k, outv);
        self(self, r, i - best_k, outv);
    };
    auto children_of = [&](int node) {
        std::vector<int> outv;
        if (is_leaf(node)) { outv.push_back(node); return outv; }
        const int l = node + 1, r = right_of(node);
        int best_k = -1;
        double best = kInf;
        for (int k = 1; k <= 7; ++k) {
            const double c = (double)cost[7 * (size_t)l + k - 1] + (double)cost[7 * (size_t)r + (8 - k) - 1];
            if (c < best) { best = c; best_k = k; }
        }
        forest_of(forest_of, l, best_k, outv);
        forest_of(forest_of, r, 8 - best_k, outv);
        return outv;
    };
    auto is_leaf_child = [&](int m) { return choice[7 * (size_t)m] == 0; };

    // Pass 1: count wide nodes.
    int wide = 0;
    {
        std::vector<int> todo{0};
        while (!todo.empty()) {
            int nd = todo.back();
            todo.pop_back();
            ++wide;
            for (int m : children_of(nd)) if (!is_leaf_child(m)) todo.push_back(m);
        }
    }
    out.nodes.assign(20 * (size_t)wide, 0u);
    out.order.assign(n, 0u);
    int node_cursor = 1, item_cursor = 0, max_depth = 0;

    auto next_down = [](float f) -> float {
        if (f == 0.0f) return -bits_float(1u);
        uint32_t u = float_bits(f);
        return bits_float(f > 0.0f ? u - 1 : u + 1);
    };
    auto f32_floor = [&](double v) -> float {
        float f = (float)v;
        return (double)f > v ? next_down(f) : f;
    };
    auto exp_byte = [](float p, double hi) -> int {
        const double extent = hi - (double)p;
        int b;
        if (!(extent > 0.0)) b = 1;
        else b = std::max(1, (int)std::ceil(std::log2(extent / 255.0)) + 127);
        while (b < 255 && (double)(float)((double)p + 255.0 * (double)bits_float((uint32_t)b << 23)) < hi) ++b;
        return b;
    };
    auto quant = [](double v, float p, float s, bool up) -> int {
        int q = up ? (int)std::ceil((v - (double)p) / (double)s) : (int)std::floor((v - (double)p) / (double)s);
        q = std::max(0, std::min(255, q));
        if (up) {
            while ((double)(float)((double)p + (double)q * (double)s) < v && q < 255) ++q;
        } else {
            while ((double)(float)((double)p + (double)q * (double)s) > v && q > 0) --q;
        }
        return q;
    };
    auto slot_for = [&](int node, double px, double py, double pz) -> int {
        const float* q = bn + 8 * (size_t)node;
        const double cx = ((double)q[0] + q[4]) * 0.5;
        const double cy = ((double)q[1] + q[5]) * 0.5;
        const double cz = ((double)q[2] + q[6]) * 0.5;
        return (cx - px > 0 ? 1 : 0) | (cy - py > 0 ? 2 : 0) | (cz - pz > 0 ? 4 : 0);
    };
    bool ok = true;
    auto emit = [&](auto&& self, int node, int wide_idx, int depth) -> void {
        if (depth > max_depth) max_depth = depth;
        std::vector<int> members = children_of(node);
        double bx0 = kInf, by0 = kInf, bz0 = kInf, bx1 = -kInf, by1 = -kInf, bz1 = -kInf;
        for (int m : members) {
            const double* f = &fb[6 * (size_t)m];
            bx0 = std::min(bx0, f[0]); by0 = std::min(by0, f[1]); bz0 = std::min(bz0, f[2]);
            bx1 = std::max(bx1, f[3]); by1 = std::max(by1, f[4]); bz1 = std::max(bz1, f[5]);
        }
        const double pcx = (bx0 + bx1) * 0.5, pcy = (by0 + by1) * 0.5, pcz = (bz0 + bz1) * 0.5;
        int slot_of[8];
        for (int s = 0; s < 8; ++s) slot_of[s] = -1;
        for (int mi = 0; mi < (int)members.size(); ++mi) {
            int s = slot_for(members[mi], pcx, pcy, pcz);
            while (slot_of[s] >= 0) s = (s + 1) & 7;
            slot_of[s] = mi;
        }
        const float p0 = f32_floor(bx0), p1 = f32_floor(by0), p2 = f32_floor(bz0);
        const int ebx = exp_byte(p0, bx1), eby = exp_byte(p1, by1), ebz = exp_byte(p2, bz1);
        if (ebx > 254 || eby > 254 || ebz > 254) { ok = false; return; }
        const float sx = bits_float((uint32_t)ebx << 23), sy = bits_float((uint32_t)eby << 23), sz = bits_float((uint32_t)ebz << 23);
        uint32_t* o = out.nodes.data() + 20 * (size_t)wide_idx;
        o[0] = float_bits(p0);
        o[1] = float_bits(p1);
        o[2] = float_bits(p2);
        int imask = 0, internal_count = 0;
        for (int s = 0; s < 8; ++s)
            if (slot_of[s] >= 0 && !is_leaf_child(members[slot_of[s]])) ++internal_count;
        const int child_base = node_cursor;
        node_cursor += internal_count;
        const int prim_base = item_cursor;
        uint8_t qlo[24], qhi[24], meta[8];
        for (int s = 0; s < 8; ++s) {
            qlo[s] = qlo[8 + s] = qlo[16 + s] = 255;
            qhi[s] = qhi[8 + s] = qhi[16 + s] = 0;
            meta[s] = 0;
        }
        for (int s = 0; s < 8; ++s) {
            const int mi = slot_of[s];
            if (mi < 0) continue;
            const int m = members[mi];
            const double* f = &fb[6 * (size_t)m];
            qlo[s] = (uint8_t)quant(f[0], p0, sx, false);
            qlo[8 + s] = (uint8_t)quant(f[1], p1, sy, false);
            qlo[16 + s] = (uint8_t)quant(f[2], p2, sz, false);
            qhi[s] = (uint8_t)quant(f[3], p0, sx, true);
            qhi[8 + s] = (uint8_t)quant(f[4], p1, sy, true);
            qhi[16 + s] = (uint8_t)quant(f[5], p2, sz, true);
            if (is_leaf_child(m)) {
                const int count = prims_of(m);
                const int offset = item_cursor - prim_base;
                if (count > 3 || offset + count > 24) { ok = false; return; }
                meta[s] = (uint8_t)((((1 << count) - 1) << 5) | offset);
                for (uint32_t i = start[m]; i < end[m]; ++i) out.order[item_cursor++] = bin.order[i];
            } else {
                imask |= 1 << s;
                meta[s] = (uint8_t)(0x20 | (24 + s));
            }
        }
        o[3] = (uint32_t)ebx | ((uint32_t)eby << 8) | ((uint32_t)ebz << 16) | ((uint32_t)imask << 24);
        o[4] = (uint32_t)child_base;
        o[5] = (uint32_t)prim_base;
        o[6] = meta[0] | (meta[1] << 8) | (meta[2] << 16) | ((uint32_t)meta[3] << 24);
        o[7] = meta[4] | (meta[5] << 8) | (meta[6] << 16) | ((uint32_t)meta[7] << 24);
        for (int w = 0; w < 6; ++w) {
            const uint8_t* src = w < 3 ? qlo : qhi;
            const int off = (w % 3) * 8;
            o[8 + 2 * w] = src[off] | (src[off + 1] << 8) | (src[off + 2] << 16) | ((uint32_t)src[off + 3] << 24);
            o[9 + 2 * w] = src[off + 4] | (src[off + 5] << 8) | (src[off + 6] << 16) | ((uint32_t)src[off + 7] << 24);
        }
        int ci = 0;
        for (int s = 0; s < 8; ++s) {
            const int mi = slot_of[s];
            if (mi >= 0 && !is_leaf_child(members[mi])) self(self, members[mi], child_base + ci++, depth + 1);
        }
    };
    emit(emit, 0, 0, 1);
    if (!ok || node_cursor != wide || item_cursor != n) {
        out.nodes.clear();
        out.order.clear();
        out.node_count = 0;
        out.error = 1;
        return out;
    }
    out.node_count = wide;
    out.max_depth = max_depth;
    return out;
}

}  // namespace ptx_host

// ---- C entry points: the builders on their own (tests, tools) ------------------------
extern "C" int ptr_build_bvh(const double* boxes, int n, int leaf_size, int always_split,
                             float* nodes_out, int nodes_cap, uint32_t* order_out, int* node_count, int* max_depth) {
    if (!boxes || n < 0 || !node_count) return -1;
    ptx_host::BinaryBvh b = ptx_host::build_bvh(boxes, n, leaf_size, always_split != 0);
    *node_count = b.node_count;
    if (max_depth) *max_depth = b.max_depth;
    if (nodes_out) {
        if (nodes_cap < b.node_count) return -1;
        std::memcpy(nodes_out, b.nodes.data(), sizeof(float) * 8 * (size_t)b.node_count);
    }
    if (order_out && n > 0) std::memcpy(order_out, b.order.data(), sizeof(uint32_t) * (size_t)n);
    return 0;
}

extern "C" int ptr_build_cwbvh(const double* boxes, int n, double c_prim,
                               uint32_t* nodes_out, int nodes_cap, uint32_t* order_out, int* node_count, int* max_depth) {
    if (!boxes || n < 0 || !node_count) return -1;
    ptx_host::WideBvh w = ptx_host::build_cwbvh(boxes, n, c_prim);
    if (w.error) return -1;
    *node_count = w.node_count;
    if (max_depth) *max_depth = w.max_depth;
    if (nodes_out) {
        if (nodes_cap < w.node_count) return -1;
        std::memcpy(nodes_out, w.nodes.data(), sizeof(uint32_t) * 20 * (size_t)w.node_count);
    }
    if (order_out && n > 0) std::memcpy(order_out, w.order.data(), sizeof(uint32_t) * (size_t)n);
    return 0;
}
