// internal.h -- host-side structures shared by the C-ABI implementation files.
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include "../../include/tim_rt.h"

namespace timrt {

void set_error(const std::string& msg);

// Allocator whose value-initialisation leaves trivial elements uninitialised, so
// that resize() of an array about to be overwritten in full does not zero it first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) { ::new (static_cast<void*>(p)) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
template <class T>
using RawVec = std::vector<T, NoInitAlloc<T>>;

// Host image of the 8-wide quantised BVH built from the reference binary tree.
struct WideHost {
    RawVec<uint32_t> nodes;          // 20 words per node
    RawVec<float> tris;              // 12 floats per leaf triangle
    // per leaf triangle, 8 words about its binary leaf: lo.xyz of the intersection
    // of the leaf's box and all its ancestors' boxes, the leaf's nid, hi.xyz of
    // that intersection, and a flag: 1 when the reference tests the leaf without a
    // box (single-leaf tree), 2 when the intersection is empty
    RawVec<uint32_t> tri_leaf;
    uint32_t num_nodes = 0;
    uint32_t root_is_leaf = 0;
    uint32_t max_depth = 0;
};

// Validates a fillGpuBuffer image (ranges, node links, leaf offsets, vertex
// indices) so kernels never index out of bounds; also returns the tree depth.
bool validate_bvh(const uint8_t* blob, uint64_t n_bytes, const uint32_t ranges[7][2], uint32_t num_nodes,
                  uint32_t num_vertex, uint32_t num_lights, uint32_t num_blas, uint32_t* depth_out, std::string& err);

// The plain form's copy of the leaf triangles: per node a 16-byte record (first
// triangle, leaf header, leaf-data offset, 0) and per triangle 48 bytes
// (p0, vertexOffset) (p1 - p0, index01) (p2 - p0, index2_matId), so that a leaf
// visit reads one record and each triangle test three 16-byte vectors.
void build_leaf_tris(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                     RawVec<float>& tris, RawVec<uint32_t>& info);

// Collapses the binary tree into 8-wide nodes with 8-bit quantised child boxes.
bool build_wide(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                WideHost& out, std::string& err);

}  // namespace timrt
