// Light tree for light-tree selection (estimator.lightSelection 'bvh';
// accel/light_tree/light_tree.ts:44-72).  A binary tree over the scene's finite lights
// with exactly one light per leaf, so 2n - 1 nodes, laid out in preorder: the left child
// of node i is i + 1, the right child is stored.  Each node records its box and the
// emitted power of its subtree.  Splits minimise the power-weighted surface-area cost
// phi_L * SA(box_L) + phi_R * SA(box_R) over 16 centroid bins along the widest centroid
// axis.  A node whose centroids coincide, or one that could otherwise pass the 48-level
// trail cap, is halved in its current order (the sorted-median fallback); that keeps the
// stochastic descent proportional to power among coincident lights.
//
// Per light, the trail records the root-to-leaf decisions (0 = left, 1 = right) least
// significant bit first: word 0 holds levels 0-23, word 1 holds levels 24-47.  The
// pdf walk replays it, so the pdf it returns is the one the sampler drew with.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ptx_rt.h"

namespace {

constexpr int kBins = 16;
constexpr int kMaxDepth = 48;

struct Builder {
    const double* box;
    const double* power;
    float* nodes;
    uint32_t* trails;
    std::vector<int> order;
    int next = 0;
    int max_depth = 0;
    bool overflow = false;

    static double area(const double* b) {
        double dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
    static void grow(double* b, const double* o) {
        for (int a = 0; a < 3; ++a) {
            b[a] = std::min(b[a], o[a]);
            b[3 + a] = std::max(b[3 + a], o[3 + a]);
        }
    }
    static void empty(double* b) {
        for (int a = 0; a < 3; ++a) { b[a] = 1e300; b[3 + a] = -1e300; }
    }

    // emits the node for order[s0, s1) at index `ni`; returns nothing (the right child's
    // index is written into the node when it is known)
    void build(int s0, int s1, int depth, uint32_t lo, uint32_t hi) {
        const int ni = next++;
        max_depth = std::max(max_depth, depth);
        double b[6];
        empty(b);
        double phi = 0.0;
        for (int k = s0; k < s1; ++k) {
            grow(b, box + 6 * (size_t)order[k]);
            phi += power[order[k]];
        }
        float* nd = nodes + 8 * (size_t)ni;
        nd[0] = (float)b[0]; nd[1] = (float)b[1]; nd[2] = (float)b[2];
        nd[3] = (float)phi;
        nd[4] = (float)b[3]; nd[5] = (float)b[4]; nd[6] = (float)b[5];
        const int count = s1 - s0;
        if (count == 1) {
            const int light = order[s0];
            nd[7] = (float)(-(light + 1));
            trails[2 * (size_t)light] = lo;
            trails[2 * (size_t)light + 1] = hi;
            return;
        }
        if (depth >= kMaxDepth) { overflow = true; nd[7] = -1.0f; return; }
        int mid = s0 + count / 2;
        // levels left for this subtree: a halving split always fits them
        const int need = (int)std::ceil(std::log2((double)count));
        const bool forced = depth + need >= kMaxDepth - 1;
        double cmin[3] = {1e300, 1e300, 1e300}, cmax[3] = {-1e300, -1e300, -1e300};
        for (int k = s0; k < s1; ++k) {
            const double* o = box + 6 * (size_t)order[k];
            for (int a = 0; a < 3; ++a) {
                double c = 0.5 * (o[a] + o[3 + a]);
                cmin[a] = std::min(cmin[a], c);
                cmax[a] = std::max(cmax[a], c);
            }
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (cmax[a] - cmin[a] > cmax[axis] - cmin[axis]) axis = a;
        const double ext = cmax[axis] - cmin[axis];
        if (!forced && ext > 0.0) {
            double bb[kBins][6], bp[kBins];
            int bc[kBins];
            for (int i = 0; i < kBins; ++i) { empty(bb[i]); bp[i] = 0.0; bc[i] = 0; }
            auto bin_of = [&](int light) {
                const double* o = box + 6 * (size_t)light;
                double c = 0.5 * (o[axis] + o[3 + axis]);
                int i = (int)((c - cmin[axis]) / ext * kBins);
                return std::min(std::max(i, 0), kBins - 1);
            };
            for (int k = s0; k < s1; ++k) {
                int i = bin_of(order[k]);
                grow(bb[i], box + 6 * (size_t)order[k]);
                bp[i] += power[order[k]];
                bc[i] += 1;
            }
            // sweep: cost of splitting after bin i; ties go to the more even count
            double lb[6], rb_[kBins][6], rp[kBins];
            int rc[kBins];
            empty(lb);
            double acc_b[6];
            empty(acc_b);
            double acc_p = 0.0;
            int acc_c = 0;
            for (int i = kBins - 1; i > 0; --i) {
                grow(acc_b, bb[i]);
                acc_p += bp[i];
                acc_c += bc[i];
                std::memcpy(rb_[i], acc_b, sizeof(acc_b));
                rp[i] = acc_p;
                rc[i] = acc_c;
            }
            double best = 1e300;
            int best_i = -1, best_bal = 1 << 30;
            double lp = 0.0;
            int lc = 0;
            for (int i = 0; i < kBins - 1; ++i) {
                grow(lb, bb[i]);
                lp += bp[i];
                lc += bc[i];
                if (lc == 0 || rc[i + 1] == 0) continue;
                double cost = lp * area(lb) + rp[i + 1] * area(rb_[i + 1]);
                int bal = std::abs(lc - rc[i + 1]);
                if (cost < best * (1.0 - 1e-12) || (cost <= best * (1.0 + 1e-12) && bal < best_bal)) {
                    best = cost;
                    best_i = i;
                    best_bal = bal;
                }
            }
            if (best_i >= 0) {
                auto it = std::stable_partition(order.begin() + s0, order.begin() + s1,
                                                [&](int light) { return bin_of(light) <= best_i; });
                mid = (int)(it - order.begin());
            }
        }
        if (mid <= s0 || mid >= s1) mid = s0 + count / 2;
        const uint32_t bit_lo = depth < 24 ? (1u << depth) : 0u;
        const uint32_t bit_hi = depth >= 24 ? (1u << (depth - 24)) : 0u;
        build(s0, mid, depth + 1, lo, hi);
        const int right = next;
        nd = nodes + 8 * (size_t)ni;
        nd[7] = (float)right;
        build(mid, s1, depth + 1, lo | bit_lo, hi | bit_hi);
    }
};

}  // namespace

extern "C" int ptr_build_light_tree(const double* boxes, const double* powers, int32_t n, float* nodes_out,
                                    uint32_t* trails_out) {
    if (n <= 0 || !boxes || !powers || !nodes_out || !trails_out) return PTR_E_INVALID;
    if (n > (1 << 24)) return PTR_E_INVALID;   // links and light ids travel as exact floats
    for (int i = 0; i < n; ++i) {
        if (!(powers[i] > 0.0) || !std::isfinite(powers[i])) return PTR_E_INVALID;
        for (int k = 0; k < 6; ++k)
            if (!std::isfinite(boxes[6 * (size_t)i + k])) return PTR_E_INVALID;
    }
    Builder b;
    b.box = boxes;
    b.power = powers;
    b.nodes = nodes_out;
    b.trails = trails_out;
    b.order.resize(n);
    for (int i = 0; i < n; ++i) b.order[i] = i;
    std::memset(trails_out, 0, sizeof(uint32_t) * 2 * (size_t)n);
    b.build(0, n, 0, 0u, 0u);
    if (b.overflow || b.next != 2 * n - 1) return PTR_E_INVALID;
    return b.max_depth;
}
