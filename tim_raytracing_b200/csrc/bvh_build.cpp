// bvh_build.cpp -- product-side BVH builder that writes the reference's
// fillGpuBuffer layout (BVHBuilder.cpp:1319-1534): binned SAH over triangle
// centroids (32 bins x 3 axes), object splits only, leaves of at most
// max_leaf_size triangles, deterministic node numbering (children allocated in
// adjacent pairs in depth-first order, child ids above parent ids, as the
// reference's builder also produces), subtrees above 32K triangles built on
// parallel threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <memory>
#include <thread>
#include <vector>
#include "internal.h"

using namespace timrt;

struct tim_rt_bvh_blob {
    std::vector<uint8_t> bytes;
    uint32_t ranges[7][2];
    tim_rt_push_constants pc;
    float aabb[6];
};

namespace {

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    double area() const {
        if (lo[0] > hi[0]) return 0.0;
        const double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1], dz = (double)hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct TNode {
    Box box;
    std::unique_ptr<TNode> kid[2];
    uint32_t first = 0, count = 0;
};

struct Ctx {
    const std::vector<Box>* tb;
    const std::vector<float>* cen;   // 3 per triangle
    std::vector<uint32_t>* idx;
    tim_rt_build_params p;
    std::atomic<int> threads_left;
};

constexpr int kBins = 32;

std::unique_ptr<TNode> build_rec(Ctx& c, uint32_t first, uint32_t count, uint32_t depth) {
    auto node = std::make_unique<TNode>();
    node->first = first;
    node->count = count;
    uint32_t* ids = c.idx->data() + first;
    Box cb;
    for (uint32_t i = 0; i < count; ++i) {
        node->box.grow((*c.tb)[ids[i]]);
        cb.grow(&(*c.cen)[3ull * ids[i]]);
    }
    if (count <= c.p.max_leaf_size || depth >= c.p.max_depth) return node;

    // binned SAH
    int best_axis = -1, best_split = -1;
    double best_cost = INFINITY;
    for (int a = 0; a < 3; ++a) {
        const double ext = (double)cb.hi[a] - cb.lo[a];
        if (!(ext > 0.0)) continue;
        Box bb[kBins];
        uint32_t bc[kBins] = {};
        const double k = kBins / ext;
        for (uint32_t i = 0; i < count; ++i) {
            int b = (int)(((double)(*c.cen)[3ull * ids[i] + a] - cb.lo[a]) * k);
            b = std::min(std::max(b, 0), kBins - 1);
            bc[b]++;
            bb[b].grow((*c.tb)[ids[i]]);
        }
        double ra[kBins];
        uint32_t rc[kBins];
        Box acc;
        uint32_t n = 0;
        for (int b = kBins - 1; b > 0; --b) {
            acc.grow(bb[b]);
            n += bc[b];
            ra[b] = acc.area();
            rc[b] = n;
        }
        Box lacc;
        uint32_t ln = 0;
        for (int s = 1; s < kBins; ++s) {
            lacc.grow(bb[s - 1]);
            ln += bc[s - 1];
            if (ln == 0 || rc[s] == 0) continue;
            const double cost = lacc.area() * ln + ra[s] * rc[s];
            if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = s; }
        }
    }
    uint32_t mid;
    if (best_axis >= 0) {
        const int a = best_axis;
        const double k = kBins / ((double)cb.hi[a] - cb.lo[a]);
        const float lo = cb.lo[a];
        uint32_t* m = std::partition(ids, ids + count, [&](uint32_t t) {
            int b = (int)(((double)(*c.cen)[3ull * t + a] - lo) * k);
            b = std::min(std::max(b, 0), kBins - 1);
            return b < best_split;
        });
        mid = (uint32_t)(m - ids);
    } else {
        // all centroids coincide: split the list in half
        mid = count / 2;
    }
    if (mid == 0 || mid == count) mid = count / 2;
    node->count = 0;
    const bool par = count > 32768u && c.threads_left.fetch_sub(1) > 0;
    if (par) {
        auto fut = std::async(std::launch::async, [&]() { return build_rec(c, first, mid, depth + 1); });
        node->kid[1] = build_rec(c, first + mid, count - mid, depth + 1);
        node->kid[0] = fut.get();
    } else {
        if (count > 32768u) c.threads_left.fetch_add(1);
        node->kid[0] = build_rec(c, first, mid, depth + 1);
        node->kid[1] = build_rec(c, first + mid, count - mid, depth + 1);
    }
    return node;
}

float widen_lo(float x) { return x - (1e-6f + std::fabs(x) * 9.5367431640625e-07f); }   // 2^-20
float widen_hi(float x) { return x + (1e-6f + std::fabs(x) * 9.5367431640625e-07f); }

uint32_t align32(uint32_t x) { return (x + 31u) & ~31u; }

// Node records of one finished image, read back for the two-level composition.
struct ImageView {
    const uint32_t* nodes;   // 16 words per node
    const uint32_t* leaf;
    uint32_t num_nodes, leaf_words;
};

ImageView view_of(const tim_rt_bvh_blob& b) {
    ImageView v;
    v.nodes = reinterpret_cast<const uint32_t*>(b.bytes.data() + b.ranges[TIM_RT_RANGE_NODE][0]);
    v.leaf = reinterpret_cast<const uint32_t*>(b.bytes.data() + b.ranges[TIM_RT_RANGE_LEAF][0]);
    v.num_nodes = b.pc.numNodes;
    v.leaf_words = b.ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    return v;
}

}  // namespace

extern "C" {

void tim_rt_build_params_default(tim_rt_build_params* p) {
    if (!p) return;
    p->max_leaf_size = 4;
    p->max_depth = 30;
    p->traversal_cost = 1.0f;
    p->intersection_cost = 0.4f;
    p->num_threads = 0;
}

int tim_rt_build_bvh(const float* pos, uint32_t num_vertex, const uint32_t* tri, uint32_t num_tris,
                     const void* materials, uint32_t num_materials, const void* lights, uint32_t num_lights,
                     const tim_rt_build_params* params, tim_rt_bvh_blob** out) {
    if (!out || !pos || !tri || num_tris == 0) {
        set_error("tim_rt_build_bvh: null argument or no triangles");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    tim_rt_build_params p;
    tim_rt_build_params_default(&p);
    if (params) p = *params;
    if (p.max_leaf_size == 0 || p.max_leaf_size > 4095u || p.max_depth == 0 || p.max_depth > 32u) {
        set_error("tim_rt_build_bvh: max_leaf_size must be 1..4095 and max_depth 1..32");
        return TIM_RT_EINVAL;
    }
    if (num_lights && !lights) {
        set_error("tim_rt_build_bvh: lights pointer is null");
        return TIM_RT_EINVAL;
    }
    std::vector<Box> tb(num_tris);
    std::vector<float> cen(3ull * num_tris);
    for (uint32_t t = 0; t < num_tris; ++t) {
        const uint32_t* r = tri + 3ull * t;
        const uint64_t i0 = (uint64_t)r[0] + (r[1] & 0xFFFFu), i1 = (uint64_t)r[0] + (r[1] >> 16),
                       i2 = (uint64_t)r[0] + (r[2] & 0xFFFFu);
        if (i0 >= num_vertex || i1 >= num_vertex || i2 >= num_vertex) {
            set_error("tim_rt_build_bvh: triangle " + std::to_string(t) + " indexes past num_vertex");
            return TIM_RT_EINVAL;
        }
        // checked per coordinate: the box's min / max would step over a NaN
        for (const uint64_t i : {i0, i1, i2})
            for (int a = 0; a < 3; ++a)
                if (!std::isfinite(pos[3 * i + a])) {
                    set_error("tim_rt_build_bvh: non-finite vertex position");
                    return TIM_RT_EINVAL;
                }
        tb[t].grow(pos + 3 * i0);
        tb[t].grow(pos + 3 * i1);
        tb[t].grow(pos + 3 * i2);
        for (int a = 0; a < 3; ++a) cen[3ull * t + a] = 0.5f * (tb[t].lo[a] + tb[t].hi[a]);
    }
    std::vector<uint32_t> idx(num_tris);
    for (uint32_t t = 0; t < num_tris; ++t) idx[t] = t;
    Ctx c{&tb, &cen, &idx, p, {0}};
    const int hw = p.num_threads ? (int)p.num_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    c.threads_left = hw - 1;
    std::unique_ptr<TNode> root = build_rec(c, 0, num_tris, 0);

    // Flatten: node 0 = root; an inner node's children get ids (k, k+1) in depth-first order.
    struct Item { const TNode* n; uint32_t id; uint32_t parent; uint32_t sibling; bool sib_leaf; };
    std::vector<const TNode*> order;      // by id
    std::vector<uint32_t> parent_of, sibling_of;
    std::vector<uint8_t> sib_leaf;
    order.push_back(root.get());
    parent_of.push_back(0x3FFFFFFFu);
    sibling_of.push_back(0x3FFFFFFFu);
    sib_leaf.push_back(0);
    std::vector<uint32_t> left_of(1, 0x3FFFFFFFu);
    {
        std::vector<uint32_t> stack = {0};
        while (!stack.empty()) {
            const uint32_t id = stack.back();
            stack.pop_back();
            const TNode* n = order[id];
            if (!n->kid[0]) continue;
            const uint32_t l = (uint32_t)order.size();
            order.push_back(n->kid[0].get());
            order.push_back(n->kid[1].get());
            left_of[id] = l;
            left_of.push_back(0x3FFFFFFFu);
            left_of.push_back(0x3FFFFFFFu);
            parent_of.push_back(id);
            parent_of.push_back(id);
            sibling_of.push_back(l + 1);
            sibling_of.push_back(l);
            sib_leaf.push_back(!n->kid[1]->kid[0]);
            sib_leaf.push_back(!n->kid[0]->kid[0]);
            stack.push_back(l + 1);
            stack.push_back(l);
        }
    }
    const uint32_t num_nodes = (uint32_t)order.size();
    if (num_nodes >= 0x3FFFFFFFu) {
        set_error("tim_rt_build_bvh: too many nodes");
        return TIM_RT_EINVAL;
    }
    // widened boxes of every node (the box its parent stores for it)
    std::vector<Box> wbox(num_nodes);
    for (uint32_t i = 0; i < num_nodes; ++i)
        for (int a = 0; a < 3; ++a) {
            wbox[i].lo[a] = widen_lo(order[i]->box.lo[a]);
            wbox[i].hi[a] = widen_hi(order[i]->box.hi[a]);
        }
    // leaf data: header, triangle records, light ids (sphere vs leaf box, BVHBuilder.cpp:36-42,749-756)
    const uint8_t* L = static_cast<const uint8_t*>(lights);
    std::vector<uint32_t> leaf;
    std::vector<uint32_t> leaf_off(num_nodes, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < num_nodes; ++i) {
        const TNode* n = order[i];
        if (n->kid[0]) continue;
        std::vector<uint32_t> lids;
        for (uint32_t l = 0; l < num_lights && lids.size() < 15u; ++l) {
            float f[13];
            std::memcpy(f, L + 56ull * l + 4, 52);
            const float r = f[3];
            float d2 = 0.f;
            for (int a = 0; a < 3; ++a) {
                const float cpt = std::min(std::max(f[a], wbox[i].lo[a]), wbox[i].hi[a]);
                d2 += (cpt - f[a]) * (cpt - f[a]);
            }
            if (d2 < r * r) lids.push_back(l);
        }
        if (n->count > 4095u) {
            set_error("tim_rt_build_bvh: a leaf would hold more than 4095 triangles; raise max_depth");
            return TIM_RT_EINVAL;
        }
        leaf_off[i] = (uint32_t)leaf.size();
        leaf.push_back(n->count | ((uint32_t)lids.size() << 28));
        for (uint32_t k = 0; k < n->count; ++k) {
            const uint32_t* r = tri + 3ull * idx[n->first + k];
            leaf.insert(leaf.end(), r, r + 3);
        }
        leaf.insert(leaf.end(), lids.begin(), lids.end());
    }
    // byte image, section order and 32-byte alignment of fillGpuBuffer
    auto blob = std::make_unique<tim_rt_bvh_blob>();
    uint32_t off = 0;
    auto place = [&](int r, uint32_t bytes) {
        blob->ranges[r][0] = off;
        blob->ranges[r][1] = std::max(32u, bytes);
        off += align32(bytes);
    };
    place(TIM_RT_RANGE_BLAS, 0);
    place(TIM_RT_RANGE_TRI, 12u * num_tris);
    place(TIM_RT_RANGE_PRIM, 0);
    place(TIM_RT_RANGE_MAT, 48u * num_materials);
    place(TIM_RT_RANGE_LIGHT, 56u * num_lights);
    place(TIM_RT_RANGE_NODE, 64u * num_nodes);
    blob->ranges[TIM_RT_RANGE_LEAF][0] = off;
    blob->ranges[TIM_RT_RANGE_LEAF][1] = 4u * (uint32_t)leaf.size();
    blob->bytes.assign((uint64_t)off + 4ull * leaf.size(), 0);
    uint8_t* b = blob->bytes.data();
    std::memcpy(b + blob->ranges[TIM_RT_RANGE_TRI][0], tri, 12ull * num_tris);
    if (num_materials && materials) std::memcpy(b + blob->ranges[TIM_RT_RANGE_MAT][0], materials, 48ull * num_materials);
    if (num_lights) std::memcpy(b + blob->ranges[TIM_RT_RANGE_LIGHT][0], lights, 56ull * num_lights);
    std::memcpy(b + blob->ranges[TIM_RT_RANGE_LEAF][0], leaf.data(), 4ull * leaf.size());
    uint32_t* nodes = reinterpret_cast<uint32_t*>(b + blob->ranges[TIM_RT_RANGE_NODE][0]);
    for (uint32_t i = 0; i < num_nodes; ++i) {
        uint32_t* w = nodes + 16ull * i;
        const uint32_t l = left_of[i];
        const bool inner = l != 0x3FFFFFFFu;
        // BVHBuilder.cpp:1283-1317 packNodeData
        w[0] = parent_of[i];
        w[1] = sibling_of[i] | ((i != 0 && sib_leaf[i]) ? 0x80000000u : 0u);
        w[2] = inner ? (l | (!order[l]->kid[0] ? 0x80000000u : 0u) | (!order[l + 1]->kid[0] ? 0x40000000u : 0u))
                     : 0x3FFFFFFFu;
        w[3] = leaf_off[i];
        float f[12] = {};
        if (inner) {
            const Box& b0 = wbox[l];
            const Box& b1 = wbox[l + 1];
            f[0] = b0.lo[0]; f[1] = b0.lo[1]; f[2] = b0.hi[0]; f[3] = b0.hi[1];
            f[4] = b1.lo[0]; f[5] = b1.lo[1]; f[6] = b1.hi[0]; f[7] = b1.hi[1];
            f[8] = b0.lo[2]; f[9] = b0.hi[2]; f[10] = b1.lo[2]; f[11] = b1.hi[2];
        }
        std::memcpy(w + 4, f, 48);
    }
    blob->pc.numTriangles = num_tris;
    blob->pc.numBlas = 0;
    blob->pc.numPrimitives = 0;
    blob->pc.numLights = num_lights;
    blob->pc.numNodes = num_nodes;
    for (int a = 0; a < 3; ++a) {
        blob->aabb[a] = wbox[0].lo[a];
        blob->aabb[3 + a] = wbox[0].hi[a];
    }
    *out = blob.release();
    return TIM_RT_OK;
}

// Two-level image (the layout BVHBuilder::fillGpuBuffer gives a top-level
// builder with BLAS instances, BVHBuilder.cpp:1319-1534): one BLAS per instance,
// built by tim_rt_build_bvh over the instance's triangles (no lights: the
// reference asserts BLAS nodes carry none, BVHBuilder.cpp:1450), then a top level
// over the instances' boxes built by the same binned SAH with leaves of at most
// tlas_max_leaf instances. Node array: the top-level nodes first, then every
// BLAS's nodes in instance order, ids shifted by the BLAS's first node
// (BVHBuilder.cpp:1441-1457); the leaf data of top-level leaves holds a header with
// no triangles, the instance ids and the light ids; BlasHeader i holds instance i's
// (widened) box and rootIndex, its root's node id (BVHBuilder.cpp:1521-1533).
int tim_rt_build_bvh_tlas(const float* pos, uint32_t num_vertex, const uint32_t* tri, uint32_t num_tris,
                          const uint32_t* inst_first, const uint32_t* inst_count, uint32_t num_instances,
                          const void* materials, uint32_t num_materials, const void* lights, uint32_t num_lights,
                          const tim_rt_build_params* params, uint32_t tlas_max_leaf, tim_rt_bvh_blob** out) {
    if (!out || !pos || !tri || !inst_first || !inst_count || num_instances == 0 || num_instances > 255u * 4095u ||
        tlas_max_leaf == 0 || tlas_max_leaf > 255u) {
        set_error("tim_rt_build_bvh_tlas: null argument, no instances, or tlas_max_leaf not in 1..255");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    tim_rt_build_params p;
    tim_rt_build_params_default(&p);
    if (params) p = *params;
    if (num_lights && !lights) {
        set_error("tim_rt_build_bvh_tlas: lights pointer is null");
        return TIM_RT_EINVAL;
    }
    // the BLASes: each an inner-node root (the reference's walk enters rootIndex as an
    // inner node, bvhCollision.glsl:336-343), so an instance needs two triangles and
    // a leaf size below its triangle count
    std::vector<std::unique_ptr<tim_rt_bvh_blob>> blas(num_instances);
    for (uint32_t i = 0; i < num_instances; ++i) {
        if ((uint64_t)inst_first[i] + inst_count[i] > num_tris || inst_count[i] < 2u) {
            set_error("tim_rt_build_bvh_tlas: instance " + std::to_string(i) +
                      " needs at least 2 triangles inside the triangle array");
            return TIM_RT_EINVAL;
        }
        tim_rt_build_params bp = p;
        bp.max_leaf_size = std::min(p.max_leaf_size, inst_count[i] - 1u);
        tim_rt_bvh_blob* b = nullptr;
        const int rc = tim_rt_build_bvh(pos, num_vertex, tri + 3ull * inst_first[i], inst_count[i], nullptr, 0, nullptr,
                                        0, &bp, &b);
        if (rc != TIM_RT_OK) return rc;
        blas[i].reset(b);
        if (b->pc.numNodes < 3u) {
            set_error("tim_rt_build_bvh_tlas: instance " + std::to_string(i) + " did not split into two leaves");
            return TIM_RT_EINVAL;
        }
    }
    // the top level over the instance boxes (the BLAS root boxes, widened as stored)
    std::vector<Box> ib(num_instances);
    std::vector<float> icen(3ull * num_instances);
    for (uint32_t i = 0; i < num_instances; ++i) {
        for (int a = 0; a < 3; ++a) {
            ib[i].lo[a] = blas[i]->aabb[a];
            ib[i].hi[a] = blas[i]->aabb[3 + a];
            icen[3ull * i + a] = 0.5f * (ib[i].lo[a] + ib[i].hi[a]);
        }
    }
    std::vector<uint32_t> iidx(num_instances);
    for (uint32_t i = 0; i < num_instances; ++i) iidx[i] = i;
    tim_rt_build_params tp = p;
    tp.max_leaf_size = tlas_max_leaf;
    Ctx c{&ib, &icen, &iidx, tp, {0}};
    c.threads_left = 0;
    std::unique_ptr<TNode> root = build_rec(c, 0, num_instances, 0);
    std::vector<const TNode*> order(1, root.get());
    std::vector<uint32_t> parent_of(1, 0x3FFFFFFFu), sibling_of(1, 0x3FFFFFFFu), left_of(1, 0x3FFFFFFFu);
    std::vector<uint8_t> sib_leaf(1, 0);
    for (std::vector<uint32_t> stack = {0}; !stack.empty();) {
        const uint32_t id = stack.back();
        stack.pop_back();
        const TNode* n = order[id];
        if (!n->kid[0]) continue;
        const uint32_t l = (uint32_t)order.size();
        order.push_back(n->kid[0].get());
        order.push_back(n->kid[1].get());
        left_of[id] = l;
        left_of.insert(left_of.end(), {0x3FFFFFFFu, 0x3FFFFFFFu});
        parent_of.insert(parent_of.end(), {id, id});
        sibling_of.insert(sibling_of.end(), {l + 1, l});
        sib_leaf.push_back(!n->kid[1]->kid[0]);
        sib_leaf.push_back(!n->kid[0]->kid[0]);
        stack.push_back(l + 1);
        stack.push_back(l);
    }
    const uint32_t top_nodes = (uint32_t)order.size();
    std::vector<uint32_t> base(num_instances);
    uint64_t total_nodes = top_nodes;
    for (uint32_t i = 0; i < num_instances; ++i) {
        base[i] = (uint32_t)total_nodes;
        total_nodes += blas[i]->pc.numNodes;
    }
    if (total_nodes >= 0x3FFFFFFFull) {
        set_error("tim_rt_build_bvh_tlas: too many nodes");
        return TIM_RT_EINVAL;
    }
    std::vector<Box> wbox(top_nodes);
    for (uint32_t i = 0; i < top_nodes; ++i)
        for (int a = 0; a < 3; ++a) {
            wbox[i].lo[a] = widen_lo(order[i]->box.lo[a]);
            wbox[i].hi[a] = widen_hi(order[i]->box.hi[a]);
        }
    // leaf data: the top-level leaves (instance ids, light ids), then every BLAS's
    const uint8_t* L = static_cast<const uint8_t*>(lights);
    std::vector<uint32_t> leaf;
    std::vector<uint32_t> leaf_off(top_nodes, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < top_nodes; ++i) {
        const TNode* n = order[i];
        if (n->kid[0]) continue;
        std::vector<uint32_t> lids;
        for (uint32_t l = 0; l < num_lights && lids.size() < 15u; ++l) {
            float f[13];
            std::memcpy(f, L + 56ull * l + 4, 52);
            float d2 = 0.f;
            for (int a = 0; a < 3; ++a) {
                const float cpt = std::min(std::max(f[a], wbox[i].lo[a]), wbox[i].hi[a]);
                d2 += (cpt - f[a]) * (cpt - f[a]);
            }
            if (d2 < f[3] * f[3]) lids.push_back(l);
        }
        leaf_off[i] = (uint32_t)leaf.size();
        leaf.push_back((n->count << 12) | ((uint32_t)lids.size() << 28));
        for (uint32_t k = 0; k < n->count; ++k) leaf.push_back(iidx[n->first + k]);
        leaf.insert(leaf.end(), lids.begin(), lids.end());
    }
    std::vector<uint32_t> leaf_base(num_instances);
    for (uint32_t i = 0; i < num_instances; ++i) {
        const ImageView v = view_of(*blas[i]);
        leaf_base[i] = (uint32_t)leaf.size();
        leaf.insert(leaf.end(), v.leaf, v.leaf + v.leaf_words);
    }
    auto blob = std::make_unique<tim_rt_bvh_blob>();
    uint32_t off = 0;
    auto place = [&](int r, uint64_t bytes) {
        blob->ranges[r][0] = off;
        blob->ranges[r][1] = std::max<uint32_t>(32u, (uint32_t)bytes);
        off += align32((uint32_t)bytes);
    };
    place(TIM_RT_RANGE_BLAS, 32ull * num_instances);
    place(TIM_RT_RANGE_TRI, 12ull * num_tris);
    place(TIM_RT_RANGE_PRIM, 0);
    place(TIM_RT_RANGE_MAT, 48ull * num_materials);
    place(TIM_RT_RANGE_LIGHT, 56ull * num_lights);
    place(TIM_RT_RANGE_NODE, 64ull * total_nodes);
    blob->ranges[TIM_RT_RANGE_LEAF][0] = off;
    blob->ranges[TIM_RT_RANGE_LEAF][1] = 4u * (uint32_t)leaf.size();
    blob->bytes.assign((uint64_t)off + 4ull * leaf.size(), 0);
    uint8_t* b = blob->bytes.data();
    std::memcpy(b + blob->ranges[TIM_RT_RANGE_TRI][0], tri, 12ull * num_tris);
    if (num_materials && materials) std::memcpy(b + blob->ranges[TIM_RT_RANGE_MAT][0], materials, 48ull * num_materials);
    if (num_lights) std::memcpy(b + blob->ranges[TIM_RT_RANGE_LIGHT][0], lights, 56ull * num_lights);
    std::memcpy(b + blob->ranges[TIM_RT_RANGE_LEAF][0], leaf.data(), 4ull * leaf.size());
    // BlasHeader: minExtent, matId, maxExtent, rootIndex (primitive_cpp.glsl:88-94)
    for (uint32_t i = 0; i < num_instances; ++i) {
        uint32_t* h = reinterpret_cast<uint32_t*>(b + blob->ranges[TIM_RT_RANGE_BLAS][0]) + 8ull * i;
        std::memcpy(h, &blas[i]->aabb[0], 12);
        h[3] = 0u;
        std::memcpy(h + 4, &blas[i]->aabb[3], 12);
        h[7] = base[i];
    }
    uint32_t* nodes = reinterpret_cast<uint32_t*>(b + blob->ranges[TIM_RT_RANGE_NODE][0]);
    for (uint32_t i = 0; i < top_nodes; ++i) {
        uint32_t* w = nodes + 16ull * i;
        const uint32_t l = left_of[i];
        const bool inner = l != 0x3FFFFFFFu;
        w[0] = parent_of[i];
        w[1] = sibling_of[i] | ((i != 0 && sib_leaf[i]) ? 0x80000000u : 0u);
        w[2] = inner ? (l | (!order[l]->kid[0] ? 0x80000000u : 0u) | (!order[l + 1]->kid[0] ? 0x40000000u : 0u))
                     : 0x3FFFFFFFu;
        w[3] = leaf_off[i];
        float f[12] = {};
        if (inner) {
            const Box& b0 = wbox[l];
            const Box& b1 = wbox[l + 1];
            f[0] = b0.lo[0]; f[1] = b0.lo[1]; f[2] = b0.hi[0]; f[3] = b0.hi[1];
            f[4] = b1.lo[0]; f[5] = b1.lo[1]; f[6] = b1.hi[0]; f[7] = b1.hi[1];
            f[8] = b0.lo[2]; f[9] = b0.hi[2]; f[10] = b1.lo[2]; f[11] = b1.hi[2];
        }
        std::memcpy(w + 4, f, 48);
    }
    // the BLAS nodes, ids shifted (an invalid id stays invalid), leaf offsets moved
    auto shift = [](uint32_t id, uint32_t by) {
        return (id & 0x3FFFFFFFu) == 0x3FFFFFFFu ? id : ((id & 0x3FFFFFFFu) + by) | (id & 0xC0000000u);
    };
    for (uint32_t i = 0; i < num_instances; ++i) {
        const ImageView v = view_of(*blas[i]);
        for (uint32_t k = 0; k < v.num_nodes; ++k) {
            const uint32_t* src = v.nodes + 16ull * k;
            uint32_t* w = nodes + 16ull * (base[i] + k);
            std::memcpy(w, src, 64);
            w[0] = shift(src[0], base[i]);
            w[1] = shift(src[1], base[i]);
            w[2] = shift(src[2], base[i]);
            w[3] = src[3] == 0xFFFFFFFFu ? src[3] : src[3] + leaf_base[i];
        }
    }
    blob->pc.numTriangles = num_tris;
    blob->pc.numBlas = num_instances;
    blob->pc.numPrimitives = 0;
    blob->pc.numLights = num_lights;
    blob->pc.numNodes = (uint32_t)total_nodes;
    for (int a = 0; a < 3; ++a) {
        blob->aabb[a] = wbox[0].lo[a];
        blob->aabb[3 + a] = wbox[0].hi[a];
    }
    *out = blob.release();
    return TIM_RT_OK;
}

int tim_rt_bvh_blob_info(const tim_rt_bvh_blob* blob, const uint8_t** bytes, uint64_t* size, uint32_t ranges[7][2],
                         tim_rt_push_constants* pc, float aabb[6]) {
    if (!blob) {
        set_error("null blob");
        return TIM_RT_EINVAL;
    }
    if (bytes) *bytes = blob->bytes.data();
    if (size) *size = blob->bytes.size();
    if (ranges) std::memcpy(ranges, blob->ranges, sizeof(blob->ranges));
    if (pc) *pc = blob->pc;
    if (aabb) std::memcpy(aabb, blob->aabb, sizeof(blob->aabb));
    return TIM_RT_OK;
}

void tim_rt_bvh_blob_free(tim_rt_bvh_blob* blob) { delete blob; }

}  // extern "C"
