// accel_build.h — host builders of the binary BVH and the compressed wide BVH.
#pragma once
#include <cstdint>
#include <vector>

namespace ptx_host {

struct BinaryBvh {
    std::vector<float> nodes;      // 8 floats per node
    std::vector<uint32_t> order;   // leaf order -> item index
    int node_count = 0;
    int max_depth = 0;
};

struct WideBvh {
    std::vector<uint32_t> nodes;   // 20 u32 per node
    std::vector<uint32_t> order;   // wide-leaf order -> item index
    int node_count = 0;
    int max_depth = 0;
    int error = 0;
};

// boxes: 6 doubles per item (min.xyz, max.xyz)
BinaryBvh build_bvh(const double* boxes, int n, int leaf_size, bool always_split);
WideBvh build_cwbvh(const double* boxes, int n, double c_prim);

constexpr int kBvhLeafSize = 2;       // BVH_LEAF_SIZE / TLAS_LEAF_SIZE (bvh.ts)
constexpr int kBvhStackDepth = 64;    // BVH_STACK_DEPTH
constexpr int kCwbvhStackDepth = 24;  // CWBVH_STACK_DEPTH
constexpr double kCwbvhCPrim = 0.3;   // CWBVH_C_PRIM_DEFAULT

}  // namespace ptx_host
