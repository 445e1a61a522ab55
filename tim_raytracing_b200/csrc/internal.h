// internal.h -- host-side structures shared by the C-ABI implementation files.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/tim_rt.h"

namespace timrt {

void set_error(const std::string& msg);

// Host image of the 8-wide quantised BVH built from the reference binary tree.
struct WideHost {
    std::vector<uint32_t> nodes;     // 20 words per node
    std::vector<float> tris;         // 12 floats per leaf triangle
    // per leaf triangle, 8 words about its binary leaf: lo.xyz of the intersection
    // of the leaf's box and all its ancestors' boxes, the leaf's nid, hi.xyz of
    // that intersection, and a flag: 1 when the reference tests the leaf without a
    // box (single-leaf tree), 2 when the intersection is empty
    std::vector<uint32_t> tri_leaf;
    uint32_t num_nodes = 0;
    uint32_t root_is_leaf = 0;
    uint32_t max_depth = 0;
};

// Validates a fillGpuBuffer image (ranges, node links, leaf offsets, vertex
// indices) so kernels never index out of bounds; also returns the tree depth.
bool validate_bvh(const uint8_t* blob, uint64_t n_bytes, const uint32_t ranges[7][2], uint32_t num_nodes,
                  uint32_t num_vertex, uint32_t num_lights, uint32_t num_blas, uint32_t* depth_out, std::string& err);

// Collapses the binary tree into 8-wide nodes with 8-bit quantised child boxes.
bool build_wide(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                WideHost& out, std::string& err);

}  // namespace timrt
