// bvh_build_gpu.cu -- GPU BVH builder writing the reference's fillGpuBuffer
// layout (BVHBuilder.cpp:1319-1534), with the node numbering and leaf-data order
// of the host builder (bvh_build.cpp), for fast scene turnaround:
//   1. triangle boxes and centroids, centroid bounds;
//   2. 63-bit Morton codes of the centroids (one scale for all three axes: the
//      largest centroid extent), radix sort (CUB, stable);
//   3. radix tree over the sorted codes (Karras 2012, "Maximizing parallelism in
//      the construction of BVHs, octrees, and k-d trees"): internal node i covers
//      a key range split at its highest differing bit, equal keys split by index;
//      its leaves are single triangles;
//   4. bottom-up boxes, triangle counts and surface-area costs (the second child
//      to arrive at a node merges), each node choosing between staying internal
//      and becoming one leaf of its (at most max_leaf_size) triangles;
//   5. treelet restructuring (Karras & Aila 2013, "Fast Parallel Construction of
//      High-Quality Bounding Volume Hierarchies"): bottom-up again, each internal
//      node, once both its subtrees are final, takes the treelet of up to 7 nodes
//      below it (opening the largest-area inner node each time) and rebuilds the
//      treelet's topology and leaf choices from the surface-area cost of every
//      subset of its leaves (exact dynamic programme over the 127 subsets, a warp
//      per treelet); four passes. The topmost nodes that chose to be leaves are
//      the final tree's leaves, their triangles the radix leaves below them;
//   5c. per node of the final tree its depth and pre-order rank among internal
//      nodes by walking to the root, which gives the host builder's numbering:
//      root 0, the children of the internal node of rank r at 2r+1 and 2r+2;
//   6. leaf sizes, exclusive scan in node order, leaf data (header, triangle
//      records left to right below the leaf, light ids: sphere vs widened leaf
//      box, at most 15) and node records (parent, sibling, children, leaf offset,
//      widened child boxes), copied back into the host image.
// Trees deeper than max_depth (the reference's traversal keeps a 32-bit
// bitstack) are refused with TIM_RT_EUNSUPPORTED.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include "context.h"

struct tim_rt_bvh_blob {   // same definition as bvh_build.cpp
    std::vector<uint8_t> bytes;
    uint32_t ranges[7][2];
    tim_rt_push_constants pc;
    float aabb[6];
};

namespace timrt {
namespace {

constexpr uint32_t kNone = 0x3FFFFFFFu;

struct Aabb {
    float lo[3], hi[3];
};

__device__ __forceinline__ uint32_t f2ord(float f) {   // order-preserving float -> uint
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Triangle boxes and centroids (the host builder's: box of the three vertices,
// centroid = its midpoint); bounds of the centroids; bad indices or non-finite
// positions set err.
__global__ void k_tri_boxes(const float* pos, uint32_t nv, const uint32_t* tri, uint32_t n, Aabb* boxes,
                            float4* cen, uint32_t* cbounds, uint32_t* err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {0.f, 0.f, 0.f};
    bool ok = false;
    if (t < n) {
        const uint32_t r0 = tri[3 * t], r1 = tri[3 * t + 1], r2 = tri[3 * t + 2];
        const uint64_t i0 = (uint64_t)r0 + (r1 & 0xFFFFu), i1 = (uint64_t)r0 + (r1 >> 16), i2 = (uint64_t)r0 + (r2 & 0xFFFFu);
        if (i0 >= nv || i1 >= nv || i2 >= nv) {
            atomicOr(err, 1u);
        } else {
            Aabb b;
            bool fin = true;
            for (int a = 0; a < 3; ++a) {
                const float p0 = pos[3 * i0 + a], p1 = pos[3 * i1 + a], p2 = pos[3 * i2 + a];
                b.lo[a] = fminf(fminf(p0, p1), p2);
                b.hi[a] = fmaxf(fmaxf(p0, p1), p2);
                fin = fin && isfinite(p0) && isfinite(p1) && isfinite(p2);
                c[a] = 0.5f * (b.lo[a] + b.hi[a]);
            }
            if (!fin) atomicOr(err, 2u);
            boxes[t] = b;
            cen[t] = make_float4(c[0], c[1], c[2], 0.f);
            ok = fin;
        }
    }
    // block-wide min / max of the centroids, then one atomic per block and axis
    __shared__ uint32_t smin[3], smax[3];
    if (threadIdx.x < 3) { smin[threadIdx.x] = 0xFFFFFFFFu; smax[threadIdx.x] = 0u; }
    __syncthreads();
    if (ok)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&smin[a], f2ord(c[a]));
            atomicMax(&smax[a], f2ord(c[a]));
        }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(cbounds + threadIdx.x, smin[threadIdx.x]);
        atomicMax(cbounds + 3 + threadIdx.x, smax[threadIdx.x]);
    }
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const float4* cen, uint32_t n, const uint32_t* cbounds, uint64_t* keys, uint32_t* vals) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float4 c = cen[t];
    const float cv[3] = {c.x, c.y, c.z};
    uint64_t q[3];
    // one scale for all three axes (the largest centroid extent): a flat scene's
    // thin axis then enters the key only at the depth where its cells are as wide
    // as the other axes', instead of being split as often as the wide axes
    float ext = 0.f;
    for (int a = 0; a < 3; ++a) ext = fmaxf(ext, ord2f(cbounds[3 + a]) - ord2f(cbounds[a]));
    for (int a = 0; a < 3; ++a) {
        const float lo = ord2f(cbounds[a]);
        float u = ext > 0.f ? (cv[a] - lo) / ext : 0.f;
        u = fminf(fmaxf(u, 0.f), 1.f);
        q[a] = (uint64_t)(u * 2097151.0f);
    }
    keys[t] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    vals[t] = t;
}

// Common-prefix length of keys i and j (equal keys: 64 + that of the indices).
__device__ __forceinline__ int delta(const uint64_t* k, uint32_t n, int i, int j) {
    if (j < 0 || j >= (int)n) return -1;
    const uint64_t a = k[i], b = k[j];
    return a == b ? 64 + __clz((uint32_t)(i ^ j)) : __clzll(a ^ b);
}

// Radix tree: internal node i in [0, n-2], handle i; leaf j at handle n-1+j.
__global__ void k_radix_tree(const uint64_t* k, uint32_t n, uint32_t* left, uint32_t* right, uint32_t* first,
                             uint32_t* last, uint32_t* parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)n - 1) return;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int s = 0;
    for (int div = 2;; div <<= 1) {
        const int t = (l + div - 1) / div;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const uint32_t L = lo == gamma ? (n - 1u) + (uint32_t)gamma : (uint32_t)gamma;
    const uint32_t R = hi == gamma + 1 ? (n - 1u) + (uint32_t)(gamma + 1) : (uint32_t)(gamma + 1);
    left[i] = L;
    right[i] = R;
    first[i] = (uint32_t)lo;
    last[i] = (uint32_t)hi;
    parent[L] = (uint32_t)i;
    parent[R] = (uint32_t)i;
    if (i == 0) parent[0] = kNone;
}

// A box written by another thread, read past L1 (after its writer's fence).
__device__ __forceinline__ Aabb load_box_cg(const Aabb* p) {
    const float* f = reinterpret_cast<const float*>(p);
    Aabb b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = __ldcg(f + a);
        b.hi[a] = __ldcg(f + 3 + a);
    }
    return b;
}

__device__ __forceinline__ uint32_t hsize(uint32_t h, uint32_t n, const uint32_t* first, const uint32_t* last) {
    return h < n - 1u ? last[h] - first[h] + 1u : 1u;
}
__device__ __forceinline__ uint32_t hfirst(uint32_t h, uint32_t n, const uint32_t* first) {
    return h < n - 1u ? first[h] : h - (n - 1u);
}

// From every leaf of the final tree (a handle of at most max_leaf triangles whose
// parent has more) up to the root: the second child to arrive at a node merges the
// boxes and internal counts of both children and goes on.
__global__ void k_bottom_up(uint32_t n, uint32_t max_leaf, const uint32_t* left, const uint32_t* right,
                            const uint32_t* first, const uint32_t* last, const uint32_t* parent, const uint32_t* order,
                            const Aabb* tri_box, Aabb* box, uint32_t* icount, uint32_t* arrive) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u || h == 0u) return;
    const uint32_t sz = hsize(h, n, first, last);
    if (sz > max_leaf || hsize(parent[h], n, first, last) <= max_leaf) return;
    Aabb b;
    for (int a = 0; a < 3; ++a) { b.lo[a] = INFINITY; b.hi[a] = -INFINITY; }
    const uint32_t f = hfirst(h, n, first);
    for (uint32_t q = 0; q < sz; ++q) {
        const Aabb t = tri_box[order[f + q]];
        for (int a = 0; a < 3; ++a) { b.lo[a] = fminf(b.lo[a], t.lo[a]); b.hi[a] = fmaxf(b.hi[a], t.hi[a]); }
    }
    box[h] = b;
    icount[h] = 0;
    uint32_t cur = h;
    while (cur != 0u) {
        const uint32_t p = parent[cur];
        __threadfence();
        if (atomicAdd(arrive + p, 1u) == 0u) return;   // the sibling finishes this node
        __threadfence();
        const uint32_t L = left[p], R = right[p];
        const Aabb bl = load_box_cg(box + L);
        const Aabb br = load_box_cg(box + R);
        Aabb m;
        for (int a = 0; a < 3; ++a) { m.lo[a] = fminf(bl.lo[a], br.lo[a]); m.hi[a] = fmaxf(bl.hi[a], br.hi[a]); }
        box[p] = m;
        icount[p] = 1u + __ldcg(icount + L) + __ldcg(icount + R);
        cur = p;
    }
}

// Per handle: bit 0 = in the final tree, bit 1 = a leaf of the final tree.
constexpr uint32_t kInTree = 1u, kIsLeaf = 2u;

// The Morton-code tree's own leaves (the fallback when the restructured tree is
// too deep): every subtree of at most max_leaf triangles whose parent has more is
// a leaf; size = triangles under the handle.
__global__ void k_mark(uint32_t n, uint32_t max_leaf, const uint32_t* first, const uint32_t* last,
                       const uint32_t* parent, uint32_t* flags, uint32_t* size) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u) return;
    const uint32_t sz = hsize(h, n, first, last);
    const bool in_tree = h == 0u || hsize(parent[h], n, first, last) > max_leaf;
    flags[h] = in_tree ? (kInTree | (sz <= max_leaf ? kIsLeaf : 0u)) : 0u;
    size[h] = sz;
}

__device__ __forceinline__ float half_area(const Aabb& b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}
__device__ __forceinline__ Aabb merge_box(const Aabb& a, const Aabb& b) {
    Aabb m;
    for (int k = 0; k < 3; ++k) { m.lo[k] = fminf(a.lo[k], b.lo[k]); m.hi[k] = fmaxf(a.hi[k], b.hi[k]); }
    return m;
}

// Surface-area costs (Karras & Aila 2013, section 4): an internal node costs ci
// per unit area, a leaf ct per triangle per unit area (the build parameters
// traversal_cost and intersection_cost); a subtree of at most max_leaf triangles
// may become one leaf, whichever costs less:
//   C(x) = min(ci * A(x) + C(left) + C(right), ct * A(x) * N(x) if N(x) <= max_leaf).
constexpr int kTreeletLeaves = 7, kSubsets = 1 << kTreeletLeaves;
constexpr uint32_t kTreeletWarps = 4;    // warps per block of the treelet pass
constexpr int kTreeletPasses = 4;        // restructuring passes over the whole tree
constexpr uint8_t kCollapse = 0x80u;     // s_part: the subset becomes one leaf (low 7 bits: its split)

// Triangle counts, costs and leaf choices of every handle of the single-triangle
// radix tree, bottom-up with arrival counters from its n leaves.
__global__ void k_sah_cost(uint32_t n, uint32_t max_leaf, float ci_, float ct, const uint32_t* left, const uint32_t* right,
                           const uint32_t* parent, const Aabb* box, float* cost, uint32_t* size, uint8_t* coll,
                           uint32_t* arrive) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u || h < n - 1u) return;
    cost[h] = ct * half_area(box[h]);
    size[h] = 1u;
    coll[h] = 0u;
    uint32_t cur = h;
    while (cur != 0u) {
        const uint32_t p = parent[cur];
        __threadfence();
        if (atomicAdd(arrive + p, 1u) == 0u) return;
        __threadfence();
        const uint32_t L = left[p], R = right[p];
        const float a = half_area(load_box_cg(box + p));
        const uint32_t sz = __ldcg(size + L) + __ldcg(size + R);
        const float ci = ci_ * a + __ldcg(cost + L) + __ldcg(cost + R);
        const float cl = sz <= max_leaf ? ct * a * (float)sz : INFINITY;
        size[p] = sz;
        coll[p] = cl <= ci ? 1u : 0u;
        cost[p] = fminf(cl, ci);
        cur = p;
    }
}

// One treelet pass, a warp per treelet: every lane walks from one radix leaf up
// to the root; the lane that arrives second at a node has the treelet rooted
// there to restructure, and the warp takes its lanes' treelets one after another,
// the 127 subsets of a treelet spread over its 32 lanes. Every node below a
// treelet root is final by then (its subtree's walks have all passed), so the
// warp owns the treelet; writes are fenced before the next arrival, reads of
// other warps' writes bypass L1.
__global__ void __launch_bounds__(kTreeletWarps * 32) k_treelet(uint32_t n, uint32_t max_leaf, float ci_, float ct,
                                                                uint32_t* left, uint32_t* right, uint32_t* parent,
                                                                Aabb* box, float* cost, uint32_t* size, uint8_t* coll,
                                                                uint32_t* arrive) {
    __shared__ float s_area_all[kTreeletWarps][kSubsets];
    __shared__ float s_cost_all[kTreeletWarps][kSubsets];
    __shared__ uint8_t s_part_all[kTreeletWarps][kSubsets];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    float* s_area = s_area_all[w];
    float* s_cost = s_cost_all[w];
    uint8_t* s_part = s_part_all[w];
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;   // radix leaf j: handle n - 1 + j
    bool active = j < n;
    uint32_t cur = n - 1u + j;
    for (;;) {
        // one step up for every walking lane
        bool pending = false;
        uint32_t p = 0;
        if (active) {
            if (cur == 0u) {
                active = false;
            } else {
                p = parent[cur];
                __threadfence();
                if (atomicAdd(arrive + p, 1u) == 0u) {
                    active = false;   // the sibling's walk finishes this node
                } else {
                    __threadfence();
                    pending = true;
                }
            }
        }
        uint32_t todo = __ballot_sync(0xFFFFFFFFu, pending);
        if (todo == 0u) break;   // walking lanes are exactly the pending ones
        // A node whose parent holds at most 7 triangles is left alone: the parent's
        // treelet opens every node below it, so its programme covers every
        // topology and leaf choice of this subtree too.
        const bool redundant = pending && p != 0u && __ldcg(size + parent[p]) <= (uint32_t)kTreeletLeaves;
        todo &= ~__ballot_sync(0xFFFFFFFFu, redundant);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1u;
            const uint32_t root = __shfl_sync(0xFFFFFFFFu, p, src);
            // the treelet below root (every lane forms it, from the same loads):
            // open the largest-area internal node until 7 leaves
            uint32_t leaf[kTreeletLeaves], inner[kTreeletLeaves - 2];
            Aabb lb[kTreeletLeaves];
            float la[kTreeletLeaves];   // area of an internal leaf of the treelet, -1 for a triangle
            int nl = 2, ni = 0;
            leaf[0] = __ldcg(left + root);
            leaf[1] = __ldcg(right + root);
            lb[0] = load_box_cg(box + leaf[0]);
            lb[1] = load_box_cg(box + leaf[1]);
            la[0] = leaf[0] >= n - 1u ? -1.0f : half_area(lb[0]);
            la[1] = leaf[1] >= n - 1u ? -1.0f : half_area(lb[1]);
            while (nl < kTreeletLeaves) {
                int best = -1;
                float ba = -1.0f;
                for (int i = 0; i < nl; ++i)
                    if (la[i] > ba) { ba = la[i]; best = i; }
                if (best < 0) break;
                const uint32_t x = leaf[best];
                inner[ni++] = x;
                leaf[best] = __ldcg(left + x);
                leaf[nl] = __ldcg(right + x);
                lb[best] = load_box_cg(box + leaf[best]);
                lb[nl] = load_box_cg(box + leaf[nl]);
                la[best] = leaf[best] >= n - 1u ? -1.0f : half_area(lb[best]);
                la[nl] = leaf[nl] >= n - 1u ? -1.0f : half_area(lb[nl]);
                ++nl;
            }
            if (nl < 3) continue;   // two triangles: nothing to rearrange
            uint32_t lsz[kTreeletLeaves];
            float lcost[kTreeletLeaves];
#pragma unroll
            for (int i = 0; i < kTreeletLeaves; ++i) {
                lsz[i] = i < nl ? __ldcg(size + leaf[i]) : 0u;
                lcost[i] = i < nl ? __ldcg(cost + leaf[i]) : 0.f;
            }
            // area of every subset of the treelet's leaves; a single leaf keeps its
            // cost, a larger subset starts at its cost as one leaf (if small enough)
            const uint32_t full = (1u << nl) - 1u;
            for (uint32_t sub = lane + 1u; sub <= full; sub += 32u) {
                Aabb u;
                for (int k = 0; k < 3; ++k) { u.lo[k] = INFINITY; u.hi[k] = -INFINITY; }
                uint32_t cnt = 0;
                float single = 0.f;
#pragma unroll
                for (int i = 0; i < kTreeletLeaves; ++i)
                    if (sub & (1u << i)) {
                        u = merge_box(u, lb[i]);
                        cnt += lsz[i];
                        single = lcost[i];
                    }
                const float a = half_area(u);
                s_area[sub] = a;
                s_cost[sub] = (sub & (sub - 1u)) == 0u ? single : (cnt <= max_leaf ? ct * a * (float)cnt : INFINITY);
            }
            __syncwarp();
            // best split of every subset, by size: all proper subsets are done first.
            // A split (P, sub \ P) is taken once, with P holding sub's lowest leaf.
            // The two largest sizes have few subsets with many splits each (7 leaves:
            // one set of 63 splits, seven of 31): there the lanes of a group share one
            // subset's splits and reduce; smaller sizes take a subset per lane.
            for (int k = 2; k <= nl; ++k) {
                if (nl >= 5 && k >= nl - 1) {
                    const uint32_t G = k == nl ? 32u : 4u;   // lanes per subset
                    const uint32_t gi = lane / G, gl = lane % G;
                    // subset gi of this size: the whole set, or the set without leaf gi
                    const bool real = k == nl ? gi == 0u : gi < (uint32_t)nl;
                    const uint32_t sub = k == nl ? full : (real ? full ^ (1u << gi) : full);
                    const uint32_t low = sub & (0u - sub), rest = sub ^ low;
                    const uint32_t nsplit = (1u << (k - 1)) - 1u;   // subsets q of rest but rest itself
                    float best = INFINITY;
                    uint32_t bp = 0xFFu;
                    for (uint32_t j = gl; real && j < nsplit; j += G) {
                        uint32_t q = 0, jj = j;   // the j-th subset of rest: j's bits on rest's bits
                        for (uint32_t b = rest; b; b &= b - 1u, jj >>= 1)
                            if (jj & 1u) q |= b & (0u - b);
                        const uint32_t P = q | low;
                        const float c = s_cost[P] + s_cost[sub ^ P];
                        if (c < best || (c == best && P < bp)) { best = c; bp = P; }
                    }
                    for (uint32_t o = G >> 1; o; o >>= 1) {   // least cost in the group, ties to the lower split
                        const float ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
                        const uint32_t op = __shfl_xor_sync(0xFFFFFFFFu, bp, o);
                        if (ob < best || (ob == best && op < bp)) { best = ob; bp = op; }
                    }
                    if (real && gl == 0u) {
                        const float ci = ci_ * s_area[sub] + best;
                        const float cl = s_cost[sub];
                        s_cost[sub] = fminf(cl, ci);
                        s_part[sub] = (uint8_t)(bp == 0xFFu ? low : bp) | (cl <= ci ? kCollapse : 0u);
                    }
                    __syncwarp();
                    continue;
                }
                for (uint32_t sub = lane + 1u; sub <= full; sub += 32u) {
                    if (__popc(sub) != k) continue;
                    const uint32_t low = sub & (0u - sub), rest = sub ^ low;
                    float best = INFINITY;
                    uint32_t bp = low;
                    for (uint32_t q = rest;; q = (q - 1u) & rest) {
                        const uint32_t P = q | low;
                        if (P != sub) {
                            const float c = s_cost[P] + s_cost[sub ^ P];
                            if (c < best) { best = c; bp = P; }
                        }
                        if (q == 0u) break;
                    }
                    const float ci = ci_ * s_area[sub] + best;
                    const float cl = s_cost[sub];
                    s_cost[sub] = fminf(cl, ci);
                    s_part[sub] = (uint8_t)bp | (cl <= ci ? kCollapse : 0u);
                }
                __syncwarp();
            }
            // rebuild (lane 0): root keeps its place; the other internal nodes are
            // reused in order. A subset that becomes one leaf still gets its best
            // split below it, so its triangles stay reachable from it.
            if (lane == 0u) {
                uint32_t stk_node[kTreeletLeaves], stk_set[kTreeletLeaves];
                int sp = 0, next = 0;
                stk_node[sp] = root;
                stk_set[sp++] = full;
                while (sp > 0) {
                    --sp;
                    const uint32_t node = stk_node[sp], set = stk_set[sp];
                    const uint8_t part = s_part[set];
                    const uint32_t P = part & (kCollapse - 1u), Q = set ^ P;
                    uint32_t kid[2];
                    const uint32_t sides[2] = {P, Q};
                    for (int k = 0; k < 2; ++k) {
                        if ((sides[k] & (sides[k] - 1u)) == 0u) {
                            kid[k] = leaf[__ffs(sides[k]) - 1];
                        } else {
                            kid[k] = inner[next++];
                            stk_node[sp] = kid[k];
                            stk_set[sp++] = sides[k];
                        }
                        parent[kid[k]] = node;
                    }
                    left[node] = kid[0];
                    right[node] = kid[1];
                    Aabb u;
                    for (int k = 0; k < 3; ++k) { u.lo[k] = INFINITY; u.hi[k] = -INFINITY; }
                    uint32_t cnt = 0;
#pragma unroll
                    for (int i = 0; i < kTreeletLeaves; ++i)
                        if (set & (1u << i)) {
                            u = merge_box(u, lb[i]);
                            cnt += lsz[i];
                        }
                    box[node] = u;
                    size[node] = cnt;
                    coll[node] = (part & kCollapse) ? 1u : 0u;
                    cost[node] = s_cost[set];
                }
                __threadfence();
            }
            __syncwarp();
        }
        if (pending) cur = p;
    }
}

// Final tree: a handle is in it unless an ancestor became a leaf; it is a leaf if
// it is a triangle or became a leaf itself.
__global__ void k_final_flags(uint32_t n, const uint32_t* parent, const uint8_t* coll, uint32_t* flags) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u) return;
    bool in_tree = true;
    for (uint32_t a = h; a != 0u;) {
        a = parent[a];
        if (coll[a]) { in_tree = false; break; }
    }
    flags[h] = in_tree ? (kInTree | ((h >= n - 1u || coll[h]) ? kIsLeaf : 0u)) : 0u;
}

// Internal-node counts again after the treelet passes (leaves 0).
__global__ void k_recount(uint32_t n, const uint32_t* left, const uint32_t* right, const uint32_t* parent,
                          const uint32_t* flags, uint32_t* icount, uint32_t* arrive) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u || h == 0u || (flags[h] & (kInTree | kIsLeaf)) != (kInTree | kIsLeaf)) return;
    icount[h] = 0u;
    uint32_t cur = h;
    while (cur != 0u) {
        const uint32_t p = parent[cur];
        __threadfence();
        if (atomicAdd(arrive + p, 1u) == 0u) return;
        __threadfence();
        icount[p] = 1u + __ldcg(icount + left[p]) + __ldcg(icount + right[p]);
        cur = p;
    }
}

// Per node of the final tree: depth, and output id from the pre-order rank of
// internal nodes (rank(child) = rank(parent) + 1, plus the left sibling's internal
// count for a right child); the root is 0, the children of rank r are 2r+1, 2r+2.
__global__ void k_number(uint32_t n, const uint32_t* left, const uint32_t* parent, const uint32_t* flags,
                         const uint32_t* icount, uint32_t* out_id, uint32_t* rank_of, uint32_t* max_depth) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u) return;
    if (!(flags[h] & kInTree)) return;
    // rank of h (meaningful for internal nodes) and depth
    uint32_t rank = 0, depth = 0, cur = h;
    while (cur != 0u) {
        const uint32_t p = parent[cur];
        rank += 1u;
        if (left[p] != cur) rank += icount[left[p]];
        ++depth;
        cur = p;
    }
    if (!(flags[h] & kIsLeaf)) rank_of[h] = rank;
    atomicMax(max_depth, depth);
    if (h == 0u) {
        out_id[0] = 0u;
        return;
    }
    const uint32_t p = parent[h];
    uint32_t prank = 0, c2 = p;
    while (c2 != 0u) {
        const uint32_t pp = parent[c2];
        prank += 1u;
        if (left[pp] != c2) prank += icount[left[pp]];
        c2 = pp;
    }
    out_id[h] = 1u + 2u * prank + (left[p] == h ? 0u : 1u);
}

__device__ __forceinline__ float widen_lo(float x) { return x - (1e-6f + fabsf(x) * 9.5367431640625e-07f); }   // 2^-20
__device__ __forceinline__ float widen_hi(float x) { return x + (1e-6f + fabsf(x) * 9.5367431640625e-07f); }

// Leaf sizes (header + 3 words per triangle + light ids), indexed by output id;
// internal nodes 0. Light ids: sphere (centre, radius) vs the widened leaf box,
// at most 15 (BVHBuilder.cpp:36-42,749-756 with the 4-bit count kept below 16).
__global__ void k_leaf_sizes(uint32_t n, const uint32_t* size, const uint32_t* flags, const uint32_t* out_id,
                             const Aabb* box, const float* lights, uint32_t num_lights, uint32_t* leaf_size,
                             uint32_t* leaf_nl) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u || h == 0u) return;
    if ((flags[h] & (kInTree | kIsLeaf)) != (kInTree | kIsLeaf)) return;
    const uint32_t sz = size[h];
    const Aabb b = box[h];
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = widen_lo(b.lo[a]); hi[a] = widen_hi(b.hi[a]); }
    uint32_t nl = 0;
    for (uint32_t l = 0; l < num_lights && nl < 15u; ++l) {
        const float* f = lights + 14u * l + 1u;
        const float r = f[3];
        float d2 = 0.f;
        for (int a = 0; a < 3; ++a) {
            const float c = fminf(fmaxf(f[a], lo[a]), hi[a]);
            d2 += (c - f[a]) * (c - f[a]);
        }
        if (d2 < r * r) ++nl;
    }
    const uint32_t id = out_id[h];
    leaf_size[id] = 1u + 3u * sz + nl;
    leaf_nl[id] = nl;
}

// Node records (packNodeData, BVHBuilder.cpp:1283-1317) and leaf data. A leaf's
// triangles are the radix leaves below it, left to right (a walk over the links
// without a stack: down the left edge, up past right children, over to the
// sibling).
__global__ void k_emit(uint32_t n, const uint32_t* left, const uint32_t* right, const uint32_t* size,
                       const uint32_t* parent, const uint32_t* flags, const uint32_t* out_id, const Aabb* box,
                       const uint32_t* order, const uint32_t* tri, const float* lights, uint32_t num_lights,
                       const uint32_t* leaf_off, const uint32_t* leaf_nl, uint32_t* nodes, uint32_t* leaf) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 2u * n - 1u) return;
    if (!(flags[h] & kInTree)) return;
    const uint32_t sz = size[h];
    const bool inner = !(flags[h] & kIsLeaf);
    const uint32_t id = out_id[h];
    uint32_t* w = nodes + 16ull * id;
    if (h == 0u) {
        w[0] = kNone;
        w[1] = kNone;
    } else {
        const uint32_t p = parent[h];
        const uint32_t sib = left[p] == h ? right[p] : left[p];
        w[0] = out_id[p];
        w[1] = out_id[sib] | ((flags[sib] & kIsLeaf) ? 0x80000000u : 0u);
    }
    float f[12] = {};
    if (inner) {
        const uint32_t L = left[h], R = right[h];
        w[2] = out_id[L] | ((flags[L] & kIsLeaf) ? 0x80000000u : 0u) | ((flags[R] & kIsLeaf) ? 0x40000000u : 0u);
        w[3] = 0xFFFFFFFFu;
        const Aabb b0 = box[L], b1 = box[R];
        f[0] = widen_lo(b0.lo[0]); f[1] = widen_lo(b0.lo[1]); f[2] = widen_hi(b0.hi[0]); f[3] = widen_hi(b0.hi[1]);
        f[4] = widen_lo(b1.lo[0]); f[5] = widen_lo(b1.lo[1]); f[6] = widen_hi(b1.hi[0]); f[7] = widen_hi(b1.hi[1]);
        f[8] = widen_lo(b0.lo[2]); f[9] = widen_hi(b0.hi[2]); f[10] = widen_lo(b1.lo[2]); f[11] = widen_hi(b1.hi[2]);
    } else {
        w[2] = kNone;
        const uint32_t off = leaf_off[id], nl = leaf_nl[id];
        w[3] = off;
        uint32_t* o = leaf + off;
        o[0] = sz | (nl << 28);
        uint32_t cur = h, q = 0;
        for (;;) {
            while (cur < n - 1u) cur = left[cur];
            const uint32_t t = order[cur - (n - 1u)];
            o[1 + 3 * q] = tri[3 * t];
            o[2 + 3 * q] = tri[3 * t + 1];
            o[3 + 3 * q] = tri[3 * t + 2];
            ++q;
            while (cur != h && left[parent[cur]] != cur) cur = parent[cur];
            if (cur == h || q >= sz) break;
            cur = right[parent[cur]];
        }
        // light ids, the same test as k_leaf_sizes
        const Aabb b = box[h];
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) { lo[a] = widen_lo(b.lo[a]); hi[a] = widen_hi(b.hi[a]); }
        uint32_t k = 0;
        for (uint32_t l = 0; l < num_lights && k < nl; ++l) {
            const float* fl = lights + 14u * l + 1u;
            const float r = fl[3];
            float d2 = 0.f;
            for (int a = 0; a < 3; ++a) {
                const float c = fminf(fmaxf(fl[a], lo[a]), hi[a]);
                d2 += (c - fl[a]) * (c - fl[a]);
            }
            if (d2 < r * r) o[1 + 3 * sz + k++] = l;
        }
    }
    for (int q = 0; q < 12; ++q) w[4 + q] = __float_as_uint(f[q]);
}

uint32_t align32(uint32_t x) { return (x + 31u) & ~31u; }

// Carves the buffers of one build out of the context's build scratch, which
// grows to the largest build seen and is kept for the next one (no allocation or
// free per build once warm).
struct Carve {
    uint8_t* base = nullptr;
    uint64_t used = 0;
    template <class T>
    T* take(uint64_t count) {
        T* p = reinterpret_cast<T*>(base + used);
        used += (std::max<uint64_t>(16, sizeof(T) * count) + 255ull) & ~255ull;
        return p;
    }
};

#define GB_CUDA(x)                                                                        \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string("tim_rt_build_bvh_gpu: ") + cudaGetErrorString(e_));    \
            return TIM_RT_EDEVICE;                                                        \
        }                                                                                 \
    } while (0)

}  // namespace
}  // namespace timrt

using namespace timrt;

extern "C" {

int tim_rt_build_bvh_gpu(tim_rt_ctx* c, const float* pos, uint32_t num_vertex, const uint32_t* tri, uint32_t num_tris,
                         const void* materials, uint32_t num_materials, const void* lights, uint32_t num_lights,
                         const tim_rt_build_params* params, tim_rt_bvh_blob** out) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!out || !pos || !tri || num_tris == 0 || num_vertex == 0) {
        set_error("tim_rt_build_bvh_gpu: null argument, no triangles or no vertices");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    tim_rt_build_params p;
    tim_rt_build_params_default(&p);
    if (params) p = *params;
    if (p.max_leaf_size == 0 || p.max_leaf_size > 4095u || p.max_depth == 0 || p.max_depth > 32u) {
        set_error("tim_rt_build_bvh_gpu: max_leaf_size must be 1..4095 and max_depth 1..32");
        return TIM_RT_EINVAL;
    }
    if (!(p.traversal_cost > 0.f && p.traversal_cost < 1e30f && p.intersection_cost > 0.f &&
          p.intersection_cost < 1e30f)) {
        set_error("tim_rt_build_bvh_gpu: traversal_cost and intersection_cost must be positive and finite");
        return TIM_RT_EINVAL;
    }
    if (num_lights && !lights) {
        set_error("tim_rt_build_bvh_gpu: lights pointer is null");
        return TIM_RT_EINVAL;
    }
    if (num_tris <= p.max_leaf_size || num_tris >= (1u << 29)) {
        // a single leaf (or a size the 32-bit handles cannot hold): the host builder
        return tim_rt_build_bvh(pos, num_vertex, tri, num_tris, materials, num_materials, lights, num_lights, &p, out);
    }
    const uint32_t n = num_tris, nh = 2u * n - 1u;
    cudaStream_t st = c->stream;
    // CUB temporary sizes (the scan's for the largest possible node count)
    size_t sort_bytes = 0, scan_bytes = 0;
    GB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                            (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0, 63, st));
    GB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)nh + 1, st));
    // every buffer of the build, with upper bounds for the node and leaf arrays:
    // at most nh nodes; leaf words at most 16 per leaf (header + 15 lights) + 3 per triangle
    Carve K;
    auto plan = [&](Carve& k) {
        k.take<float>(3ull * num_vertex); k.take<uint32_t>(3ull * n); k.take<uint32_t>(8); k.take<uint32_t>(8);
        k.take<Aabb>(n); k.take<float4>(n); k.take<uint64_t>(n); k.take<uint64_t>(n); k.take<uint32_t>(n);
        k.take<uint32_t>(n); k.take<uint32_t>(n); k.take<uint32_t>(n); k.take<uint32_t>(n); k.take<uint32_t>(n);
        k.take<uint32_t>(nh); k.take<Aabb>(nh); k.take<uint32_t>(nh); k.take<uint32_t>(n); k.take<uint32_t>(nh);
        k.take<uint32_t>(nh); k.take<uint32_t>(1); k.take<float>(14ull * std::max(num_lights, 1u));
        k.take<uint8_t>(sort_bytes); k.take<uint32_t>(nh + 1ull); k.take<uint32_t>(nh); k.take<uint32_t>(nh + 1ull);
        k.take<uint8_t>(scan_bytes); k.take<uint32_t>(16ull * nh); k.take<uint32_t>(19ull * n);
        k.take<uint32_t>(nh); k.take<float>(nh); k.take<uint32_t>(n); k.take<uint32_t>(n); k.take<uint32_t>(nh);
        k.take<uint32_t>(nh); k.take<uint8_t>(nh);
    };
    plan(K);
    if (c->bld.bytes < K.used) {
        cudaStreamSynchronize(st);
        dev_free(c, c->bld);
        if ((rc = dev_alloc(c, c->bld, K.used))) return rc;
    }
    K.base = static_cast<uint8_t*>(c->bld.ptr);
    K.used = 0;
    float* d_pos = K.take<float>(3ull * num_vertex);
    uint32_t* d_tri = K.take<uint32_t>(3ull * n);
    uint32_t* d_err = K.take<uint32_t>(8);
    uint32_t* d_cb = K.take<uint32_t>(8);
    Aabb* d_tbox = K.take<Aabb>(n);
    float4* d_cen = K.take<float4>(n);
    uint64_t* d_keys = K.take<uint64_t>(n);
    uint64_t* d_keys2 = K.take<uint64_t>(n);
    uint32_t* d_vals = K.take<uint32_t>(n);
    uint32_t* d_order = K.take<uint32_t>(n);
    uint32_t* d_left = K.take<uint32_t>(n);
    uint32_t* d_right = K.take<uint32_t>(n);
    uint32_t* d_first = K.take<uint32_t>(n);
    uint32_t* d_last = K.take<uint32_t>(n);
    uint32_t* d_parent = K.take<uint32_t>(nh);
    Aabb* d_box = K.take<Aabb>(nh);
    uint32_t* d_icount = K.take<uint32_t>(nh);
    uint32_t* d_arrive = K.take<uint32_t>(n);
    uint32_t* d_outid = K.take<uint32_t>(nh);
    uint32_t* d_rank = K.take<uint32_t>(nh);
    uint32_t* d_maxd = K.take<uint32_t>(1);
    float* d_lights = K.take<float>(14ull * std::max(num_lights, 1u));
    uint8_t* d_tmp = K.take<uint8_t>(sort_bytes);
    uint32_t* d_lsize = K.take<uint32_t>(nh + 1ull);
    uint32_t* d_lnl = K.take<uint32_t>(nh);
    uint32_t* d_loff = K.take<uint32_t>(nh + 1ull);
    uint8_t* d_scan = K.take<uint8_t>(scan_bytes);
    uint32_t* d_nodes = K.take<uint32_t>(16ull * nh);
    uint32_t* d_leaf = K.take<uint32_t>(19ull * n);
    uint32_t* d_flags = K.take<uint32_t>(nh);
    float* d_cost = K.take<float>(nh);
    uint32_t* d_left0 = K.take<uint32_t>(n);
    uint32_t* d_right0 = K.take<uint32_t>(n);
    uint32_t* d_parent0 = K.take<uint32_t>(nh);
    uint32_t* d_size = K.take<uint32_t>(nh);
    uint8_t* d_coll = K.take<uint8_t>(nh);
    if (K.used > c->bld.bytes) {   // the plan above and these takes list the same buffers
        set_error("tim_rt_build_bvh_gpu: scratch plan mismatch");
        return TIM_RT_EDEVICE;
    }
    GB_CUDA(cudaMemcpyAsync(d_pos, pos, 12ull * num_vertex, cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_tri, tri, 12ull * n, cudaMemcpyHostToDevice, st));
    if (num_lights) GB_CUDA(cudaMemcpyAsync(d_lights, lights, 56ull * num_lights, cudaMemcpyHostToDevice, st));
    const uint32_t cb_init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
    GB_CUDA(cudaMemcpyAsync(d_cb, cb_init, sizeof(cb_init), cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    const uint32_t B = 256, g1 = (n + B - 1) / B, gh = (nh + B - 1) / B;
    k_tri_boxes<<<g1, B, 0, st>>>(d_pos, num_vertex, d_tri, n, d_tbox, d_cen, d_cb, d_err);
    GB_CUDA(cudaGetLastError());
    k_morton<<<g1, B, 0, st>>>(d_cen, n, d_cb, d_keys, d_vals);
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, sort_bytes, d_keys, d_keys2, d_vals, d_order, (int)n, 0, 63, st));
    k_radix_tree<<<(n - 1 + B - 1) / B, B, 0, st>>>(d_keys2, n, d_left, d_right, d_first, d_last, d_parent);
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaMemsetAsync(d_arrive, 0, 4ull * n, st));
    GB_CUDA(cudaMemsetAsync(d_maxd, 0, 4, st));
    // boxes of every handle of the single-triangle radix tree (its Morton-code
    // links are kept: a restructured tree deeper than max_depth -- surface-area-
    // optimal treelets can lean -- falls back to it)
    k_bottom_up<<<gh, B, 0, st>>>(n, 1u, d_left, d_right, d_first, d_last, d_parent, d_order, d_tbox, d_box, d_icount,
                                  d_arrive);
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaMemcpyAsync(d_left0, d_left, 4ull * n, cudaMemcpyDeviceToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_right0, d_right, 4ull * n, cudaMemcpyDeviceToDevice, st));
    GB_CUDA(cudaMemcpyAsync(d_parent0, d_parent, 4ull * nh, cudaMemcpyDeviceToDevice, st));
    // costs and leaf choices, two treelet passes, the final tree's leaves, then
    // internal-node counts and numbering
    GB_CUDA(cudaMemsetAsync(d_arrive, 0, 4ull * n, st));
    k_sah_cost<<<gh, B, 0, st>>>(n, p.max_leaf_size, p.traversal_cost, p.intersection_cost, d_left, d_right, d_parent, d_box, d_cost, d_size, d_coll,
                                 d_arrive);
    GB_CUDA(cudaGetLastError());
    for (int pass = 0; pass < kTreeletPasses; ++pass) {
        GB_CUDA(cudaMemsetAsync(d_arrive, 0, 4ull * n, st));
        k_treelet<<<(n + kTreeletWarps * 32 - 1) / (kTreeletWarps * 32), kTreeletWarps * 32, 0, st>>>(
            n, p.max_leaf_size, p.traversal_cost, p.intersection_cost, d_left, d_right, d_parent, d_box, d_cost, d_size,
            d_coll, d_arrive);
        GB_CUDA(cudaGetLastError());
    }
    k_final_flags<<<gh, B, 0, st>>>(n, d_parent, d_coll, d_flags);
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cudaMemsetAsync(d_arrive, 0, 4ull * n, st));
    k_recount<<<gh, B, 0, st>>>(n, d_left, d_right, d_parent, d_flags, d_icount, d_arrive);
    GB_CUDA(cudaGetLastError());
    k_number<<<gh, B, 0, st>>>(n, d_left, d_parent, d_flags, d_icount, d_outid, d_rank, d_maxd);
    GB_CUDA(cudaGetLastError());
    uint32_t h_err = 0, h_maxd = 0, h_root_icount = 0;
    GB_CUDA(cudaMemcpyAsync(&h_err, d_err, 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaMemcpyAsync(&h_maxd, d_maxd, 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaMemcpyAsync(&h_root_icount, d_icount, 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    if (h_err & 1u) {
        set_error("tim_rt_build_bvh_gpu: a triangle indexes past num_vertex");
        return TIM_RT_EINVAL;
    }
    if (h_err & 2u) {
        set_error("tim_rt_build_bvh_gpu: non-finite vertex position");
        return TIM_RT_EINVAL;
    }
    if (h_maxd > p.max_depth) {
        // back to the Morton-code tree: its links, then boxes, counts and numbering again
        GB_CUDA(cudaMemcpyAsync(d_left, d_left0, 4ull * n, cudaMemcpyDeviceToDevice, st));
        GB_CUDA(cudaMemcpyAsync(d_right, d_right0, 4ull * n, cudaMemcpyDeviceToDevice, st));
        GB_CUDA(cudaMemcpyAsync(d_parent, d_parent0, 4ull * nh, cudaMemcpyDeviceToDevice, st));
        GB_CUDA(cudaMemsetAsync(d_arrive, 0, 4ull * n, st));
        GB_CUDA(cudaMemsetAsync(d_maxd, 0, 4, st));
        k_bottom_up<<<gh, B, 0, st>>>(n, p.max_leaf_size, d_left, d_right, d_first, d_last, d_parent, d_order, d_tbox,
                                      d_box, d_icount, d_arrive);
        GB_CUDA(cudaGetLastError());
        k_mark<<<gh, B, 0, st>>>(n, p.max_leaf_size, d_first, d_last, d_parent, d_flags, d_size);
        GB_CUDA(cudaGetLastError());
        k_number<<<gh, B, 0, st>>>(n, d_left, d_parent, d_flags, d_icount, d_outid, d_rank, d_maxd);
        GB_CUDA(cudaGetLastError());
        GB_CUDA(cudaMemcpyAsync(&h_maxd, d_maxd, 4, cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaMemcpyAsync(&h_root_icount, d_icount, 4, cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaStreamSynchronize(st));
    }
    if (h_maxd > p.max_depth) {
        set_error("tim_rt_build_bvh_gpu: the Morton-code tree is " + std::to_string(h_maxd) +
                  " levels deep, above max_depth " + std::to_string(p.max_depth) +
                  " (the reference traversal's bitstack); use tim_rt_build_bvh");
        return TIM_RT_EUNSUPPORTED;
    }
    const uint32_t num_nodes = 1u + 2u * h_root_icount;
    GB_CUDA(cudaMemsetAsync(d_lsize, 0, 4ull * (num_nodes + 1), st));
    GB_CUDA(cudaMemsetAsync(d_lnl, 0, 4ull * num_nodes, st));
    k_leaf_sizes<<<gh, B, 0, st>>>(n, d_size, d_flags, d_outid, d_box, d_lights, num_lights, d_lsize, d_lnl);
    GB_CUDA(cudaGetLastError());
    GB_CUDA(cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_lsize, d_loff, (int)num_nodes + 1, st));
    uint32_t leaf_words = 0;
    GB_CUDA(cudaMemcpyAsync(&leaf_words, d_loff + num_nodes, 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    if (leaf_words > 19ull * n) {   // cannot happen: at most 16 words per leaf plus 3 per triangle
        set_error("tim_rt_build_bvh_gpu: leaf data larger than its bound");
        return TIM_RT_EDEVICE;
    }
    k_emit<<<gh, B, 0, st>>>(n, d_left, d_right, d_size, d_parent, d_flags, d_outid, d_box, d_order, d_tri, d_lights,
                             num_lights, d_loff, d_lnl, d_nodes, d_leaf);
    GB_CUDA(cudaGetLastError());

    // host image: fillGpuBuffer section order and 32-byte alignment
    auto blob = std::make_unique<tim_rt_bvh_blob>();
    uint32_t off = 0;
    auto place = [&](int r, uint32_t bytes) {
        blob->ranges[r][0] = off;
        blob->ranges[r][1] = std::max(32u, bytes);
        off += align32(bytes);
    };
    place(TIM_RT_RANGE_BLAS, 0);
    place(TIM_RT_RANGE_TRI, 12u * n);
    place(TIM_RT_RANGE_PRIM, 0);
    place(TIM_RT_RANGE_MAT, 48u * num_materials);
    place(TIM_RT_RANGE_LIGHT, 56u * num_lights);
    place(TIM_RT_RANGE_NODE, 64u * num_nodes);
    blob->ranges[TIM_RT_RANGE_LEAF][0] = off;
    blob->ranges[TIM_RT_RANGE_LEAF][1] = 4u * leaf_words;
    blob->bytes.assign((uint64_t)off + 4ull * leaf_words, 0);
    uint8_t* b = blob->bytes.data();
    GB_CUDA(cudaMemcpyAsync(b + blob->ranges[TIM_RT_RANGE_NODE][0], d_nodes, 64ull * num_nodes, cudaMemcpyDeviceToHost,
                            st));
    GB_CUDA(cudaMemcpyAsync(b + blob->ranges[TIM_RT_RANGE_LEAF][0], d_leaf, 4ull * leaf_words, cudaMemcpyDeviceToHost,
                            st));
    Aabb root;
    GB_CUDA(cudaMemcpyAsync(&root, d_box, sizeof(Aabb), cudaMemcpyDeviceToHost, st));
    std::memcpy(b + blob->ranges[TIM_RT_RANGE_TRI][0], tri, 12ull * n);
    if (num_materials && materials) std::memcpy(b + blob->ranges[TIM_RT_RANGE_MAT][0], materials, 48ull * num_materials);
    if (num_lights) std::memcpy(b + blob->ranges[TIM_RT_RANGE_LIGHT][0], lights, 56ull * num_lights);
    GB_CUDA(cudaStreamSynchronize(st));
    blob->pc.numTriangles = n;
    blob->pc.numBlas = 0;
    blob->pc.numPrimitives = 0;
    blob->pc.numLights = num_lights;
    blob->pc.numNodes = num_nodes;
    for (int a = 0; a < 3; ++a) {   // the widened root box, as the host builder reports it
        blob->aabb[a] = root.lo[a] - (1e-6f + std::fabs(root.lo[a]) * 9.5367431640625e-07f);
        blob->aabb[3 + a] = root.hi[a] + (1e-6f + std::fabs(root.hi[a]) * 9.5367431640625e-07f);
    }
    *out = blob.release();
    return TIM_RT_OK;
}

}  // extern "C"
