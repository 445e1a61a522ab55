// bvh_layout.cpp -- host-side checks of the reference BVH image and the
// collapse of its binary tree into the 8-wide quantised form.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <deque>
#include <thread>
#include "internal.h"

namespace timrt {

namespace {
constexpr uint32_t kInvalid = 0x3FFFFFFFu;   // BVHBuilder.cpp:1287 InvalidNodeId = NID_MASK
constexpr uint32_t kLeafBit = 0x80000000u, kMask = 0x3FFFFFFFu, kLeftLeaf = 0x80000000u, kRightLeaf = 0x40000000u;

struct PNode { uint32_t nid[4]; float n0xy[4]; float n1xy[4]; float nz[4]; };   // primitive_cpp.glsl:80-86

bool range_ok(const uint32_t r[2], uint64_t need, uint64_t n_bytes) {
    return (uint64_t)r[0] + need <= n_bytes && need <= (uint64_t)r[1] + 0u;
}
}  // namespace

bool validate_bvh(const uint8_t* blob, uint64_t n_bytes, const uint32_t ranges[7][2], uint32_t num_nodes,
                  uint32_t num_vertex, uint32_t num_lights, uint32_t num_blas, uint32_t* depth_out, std::string& err) {
    if (!blob || num_nodes == 0) { err = "empty BVH"; return false; }
    if (ranges[TIM_RT_RANGE_NODE][0] % 16u) { err = "node range not 16-byte aligned"; return false; }
    for (int i = 0; i < 7; ++i)
        if (ranges[i][0] % 4u) { err = "range offset not 4-byte aligned"; return false; }
    if (!range_ok(ranges[TIM_RT_RANGE_NODE], 64ull * num_nodes, n_bytes)) { err = "node range outside the buffer"; return false; }
    if (!range_ok(ranges[TIM_RT_RANGE_LIGHT], 56ull * num_lights, n_bytes)) { err = "light range outside the buffer"; return false; }
    if (!range_ok(ranges[TIM_RT_RANGE_BLAS], 32ull * num_blas, n_bytes)) { err = "blas range outside the buffer"; return false; }
    if ((uint64_t)ranges[TIM_RT_RANGE_LEAF][0] + ranges[TIM_RT_RANGE_LEAF][1] > n_bytes) { err = "leaf range outside the buffer"; return false; }
    const PNode* nodes = reinterpret_cast<const PNode*>(blob + ranges[TIM_RT_RANGE_NODE][0]);
    const uint32_t* leaf = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_LEAF][0]);
    const uint64_t leaf_words = ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    std::vector<uint8_t> depth(num_nodes, 0);
    uint32_t max_depth = 0;
    auto inner_ok = [&](uint32_t i) { return (nodes[i].nid[2] & kMask) != kInvalid; };
    if (num_nodes > 1 && !inner_ok(0)) { err = "root has no children"; return false; }
    for (uint32_t i = 0; i < num_nodes; ++i) {
        const PNode& n = nodes[i];
        const uint32_t left = n.nid[2] & kMask;
        if (left != kInvalid) {
            if (left <= i || (uint64_t)left + 1u >= num_nodes) { err = "node " + std::to_string(i) + ": child id out of order or out of range"; return false; }
            const uint32_t d = depth[i] + 1u;
            if (d > 32u) { err = "tree deeper than 32 levels (the reference traversal's bitstack width)"; return false; }
            depth[left] = depth[left + 1u] = (uint8_t)d;
            max_depth = std::max(max_depth, d);
            if (!(n.nid[2] & kLeftLeaf) && !inner_ok(left)) { err = "node " + std::to_string(left) + " used as inner node without children"; return false; }
            if (!(n.nid[2] & kRightLeaf) && !inner_ok(left + 1u)) { err = "node " + std::to_string(left + 1) + " used as inner node without children"; return false; }
        }
        const uint32_t off = n.nid[3];
        if (off != 0xFFFFFFFFu) {
            if (off >= leaf_words) { err = "node " + std::to_string(i) + ": leaf offset out of range"; return false; }
            const uint32_t hdr = leaf[off];
            const uint32_t nt = hdr & 0xFFFu, nb = (hdr >> 12) & 0xFFu, np = (hdr >> 20) & 0xFFu, nl = (hdr >> 28) & 0xFu;
            const uint64_t end = 1ull + off + 3ull * nt + nb + np + nl;
            if (end > leaf_words) { err = "node " + std::to_string(i) + ": leaf data past the leaf range"; return false; }
            for (uint32_t t = 0; t < nt; ++t) {
                const uint32_t* r = leaf + 1u + off + 3u * t;
                const uint64_t i0 = (uint64_t)r[0] + (r[1] & 0xFFFFu), i1 = (uint64_t)r[0] + (r[1] >> 16),
                               i2 = (uint64_t)r[0] + (r[2] & 0xFFFFu);
                if (i0 >= num_vertex || i1 >= num_vertex || i2 >= num_vertex) {
                    err = "node " + std::to_string(i) + ": triangle vertex index >= num_vertex";
                    return false;
                }
            }
            for (uint32_t b = 0; b < nb; ++b)
                if (leaf[1u + off + 3u * nt + b] >= num_blas) { err = "blas id out of range"; return false; }
            for (uint32_t l = 0; l < nl; ++l)
                if (leaf[1u + off + 3u * nt + nb + np + l] >= num_lights) { err = "light id out of range"; return false; }
        }
    }
    if (depth_out) *depth_out = max_depth;
    return true;
}

// ---------------------------------------------------------------------------------- leaf-triangle copy

// Per node: (first triangle in `tris`, leaf header word, leaf-data offset, 0); a
// node without leaf data (offset 0xFFFFFFFF) gets header 0, as the kernels read
// it. Per leaf-data triangle record, in node order and, within a node, in the
// leaf's stored order: (p0, vertexOffset) (p1 - p0, index01) (p2 - p0,
// index2_matId) as 12 floats, the edges being the same rounded differences
// CollideTriangle forms (collision.glsl:60-61). Runs after validate_bvh, so every
// offset and vertex index is in range.
void build_leaf_tris(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                     RawVec<float>& tris, RawVec<uint32_t>& info) {
    const PNode* nodes = reinterpret_cast<const PNode*>(blob + ranges[TIM_RT_RANGE_NODE][0]);
    const uint32_t* leaf = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_LEAF][0]);
    info.resize(4ull * num_nodes);
    uint64_t total = 0;
    for (uint32_t i = 0; i < num_nodes; ++i) {
        const uint32_t off = nodes[i].nid[3];
        const uint32_t hdr = off == 0xFFFFFFFFu ? 0u : leaf[off];
        info[4ull * i + 0] = (uint32_t)total;
        info[4ull * i + 1] = hdr;
        info[4ull * i + 2] = off;
        info[4ull * i + 3] = 0u;
        total += hdr & 0xFFFu;
    }
    tris.resize(12ull * total);
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint32_t chunk = (num_nodes + hw - 1u) / hw;
    auto fill = [&](uint32_t n0, uint32_t n1) {
        for (uint32_t i = n0; i < n1; ++i) {
            const uint32_t nt = info[4ull * i + 1] & 0xFFFu;
            float* out = tris.data() + 12ull * info[4ull * i];
            for (uint32_t t = 0; t < nt; ++t, out += 12) {
                const uint32_t* r = leaf + 1u + info[4ull * i + 2] + 3u * t;
                const float* P0 = pos + 3ull * (r[0] + (r[1] & 0xFFFFu));
                const float* P1 = pos + 3ull * (r[0] + (r[1] >> 16));
                const float* P2 = pos + 3ull * (r[0] + (r[2] & 0xFFFFu));
                for (int a = 0; a < 3; ++a) {
                    out[a] = P0[a];
                    out[4 + a] = P1[a] - P0[a];
                    out[8 + a] = P2[a] - P0[a];
                }
                std::memcpy(out + 3, &r[0], 4);
                std::memcpy(out + 7, &r[1], 4);
                std::memcpy(out + 11, &r[2], 4);
            }
        }
    };
    if (total < 65536u || hw == 1u) {
        fill(0, num_nodes);
        return;
    }
    std::vector<std::thread> pool;
    for (uint32_t n0 = 0; n0 < num_nodes; n0 += chunk) pool.emplace_back(fill, n0, std::min(num_nodes, n0 + chunk));
    for (std::thread& t : pool) t.join();
}

// ---------------------------------------------------------------------------------- 8-wide collapse

namespace {

struct Slot {
    uint32_t id;        // binary node id | kLeafBit for leaves
    float lo[3], hi[3]; // box the reference stores for this subtree (in its parent record)
    // per axis, the intersection of this box and the boxes of all its binary
    // ancestors (each box's two planes taken as min / max)
    float elo[3], ehi[3];
};

void child_slots(const PNode& n, Slot& a, Slot& b, const Slot* parent) {
    const uint32_t left = n.nid[2] & kMask;
    a.id = left | ((n.nid[2] & kLeftLeaf) ? kLeafBit : 0u);
    b.id = (left + 1u) | ((n.nid[2] & kRightLeaf) ? kLeafBit : 0u);
    a.lo[0] = n.n0xy[0]; a.lo[1] = n.n0xy[1]; a.lo[2] = n.nz[0];
    a.hi[0] = n.n0xy[2]; a.hi[1] = n.n0xy[3]; a.hi[2] = n.nz[1];
    b.lo[0] = n.n1xy[0]; b.lo[1] = n.n1xy[1]; b.lo[2] = n.nz[2];
    b.hi[0] = n.n1xy[2]; b.hi[1] = n.n1xy[3]; b.hi[2] = n.nz[3];
    for (Slot* c : {&a, &b})
        for (int ax = 0; ax < 3; ++ax) {
            const float lo = std::min(c->lo[ax], c->hi[ax]), hi = std::max(c->lo[ax], c->hi[ax]);
            c->elo[ax] = parent ? std::max(parent->elo[ax], lo) : lo;
            c->ehi[ax] = parent ? std::min(parent->ehi[ax], hi) : hi;
        }
}

double area(const Slot& s) {
    const double dx = std::fabs((double)s.hi[0] - s.lo[0]), dy = std::fabs((double)s.hi[1] - s.lo[1]),
                 dz = std::fabs((double)s.hi[2] - s.lo[2]);
    return dx * dy + dy * dz + dz * dx;
}

// Plane o + sc * q compared with a float bound in real arithmetic: the kernel
// evaluates planes in t-space, so the quantised box must contain the
// reference box exactly, not only after rounding. Extended precision plus a
// relative margin of 2^-60 keeps the comparison one-sided; q = 0 (the plane
// is o itself) is compared exactly.
bool plane_le(float o, float sc, uint32_t q, float x) {   // o + sc*q <= x
    if (q == 0) return o <= x;
    const long double v = (long double)o + (long double)sc * (long double)q;
    const long double m = fabsl((long double)x) * 8.67e-19L + 1e-300L;
    return v <= (long double)x - m;
}
bool plane_ge(float o, float sc, uint32_t q, float x) {   // o + sc*q >= x
    if (q == 0) return o >= x;
    const long double v = (long double)o + (long double)sc * (long double)q;
    const long double m = fabsl((long double)x) * 8.67e-19L + 1e-300L;
    return v >= (long double)x + m;
}

// Places up to 8 children in the 8 slots by their direction from the node
// centre: slot bit a set means "on the + side of axis a". The (child, slot)
// pair that best matches is taken first (greedy; Ylitie et al. 2017 use an
// auction for the same assignment). A ray then visits its hit slots in the
// order slot XOR octant(ray), which is roughly front to back, with no sort.
// A single-leaf root keeps its leaf in slot 0.
void assign_octant_slots(const std::vector<Slot>& fr, bool single_leaf_root, int slot_child[8]) {
    for (int k = 0; k < 8; ++k) slot_child[k] = -1;
    const int n = (int)fr.size();
    if (single_leaf_root || n == 0) {
        for (int i = 0; i < n && i < 8; ++i) slot_child[i] = i;
        return;
    }
    double c[3];
    double cen[8][3];
    for (int a = 0; a < 3; ++a) {
        double mn = INFINITY, mx = -INFINITY;
        for (int i = 0; i < n; ++i) {
            mn = std::min(mn, (double)std::min(fr[i].lo[a], fr[i].hi[a]));
            mx = std::max(mx, (double)std::max(fr[i].lo[a], fr[i].hi[a]));
            cen[i][a] = 0.5 * ((double)fr[i].lo[a] + (double)fr[i].hi[a]);
        }
        c[a] = 0.5 * (mn + mx);
    }
    bool child_done[8] = {};
    for (int step = 0; step < n; ++step) {
        double best = INFINITY;
        int bi = -1, bs = -1;
        for (int i = 0; i < n; ++i) {
            if (child_done[i]) continue;
            for (int s = 0; s < 8; ++s) {
                if (slot_child[s] >= 0) continue;
                double cost = 0.0;
                for (int a = 0; a < 3; ++a) cost -= (cen[i][a] - c[a]) * (((s >> a) & 1) ? 1.0 : -1.0);
                // the first candidate is taken whatever its cost, so that a NaN cost
                // (a corrupt, non-finite box) cannot leave the child without a slot
                if (bi < 0 || cost < best) { best = cost; bi = i; bs = s; }
            }
        }
        slot_child[bs] = bi;
        child_done[bi] = true;
    }
}

// Quantises one axis of the slot boxes: chooses the scale exponent and the
// outward-rounded 8-bit bounds; returns false if no exponent fits.
bool quantise_axis(const float* lo, const float* hi, int n, float& origin, uint8_t& ebiased, uint8_t* qlo, uint8_t* qhi) {
    float mn = INFINITY, mx = -INFINITY;
    for (int k = 0; k < n; ++k) { mn = std::min(mn, lo[k]); mx = std::max(mx, hi[k]); }
    if (!std::isfinite(mn) || !std::isfinite(mx)) return false;
    origin = mn;
    const double extent = (double)mx - (double)mn;
    int e = 1;
    if (extent > 0.0) {
        const double want = extent / 255.0;
        e = (int)std::ceil(std::log2(want)) + 127;
        if (e < 1) e = 1;
    }
    for (; e <= 167; ++e) {   // scale <= 2^40 keeps scale / d finite in the kernel
        float sc;
        const uint32_t bits = (uint32_t)e << 23;
        std::memcpy(&sc, &bits, 4);
        bool ok = true;
        for (int k = 0; k < n && ok; ++k) {
            double fl = std::floor(((double)lo[k] - (double)origin) / sc);
            long q = (long)std::max(0.0, std::min(255.0, fl));
            while (q > 0 && !plane_le(origin, sc, (uint32_t)q, lo[k])) --q;
            if (!plane_le(origin, sc, (uint32_t)q, lo[k])) { ok = false; break; }
            double ch = std::ceil(((double)hi[k] - (double)origin) / sc);
            long r = (long)std::max(0.0, std::min(255.0, ch));
            while (r < 255 && !plane_ge(origin, sc, (uint32_t)r, hi[k])) ++r;
            if (!plane_ge(origin, sc, (uint32_t)r, hi[k])) { ok = false; break; }
            if (r < q) r = q;
            qlo[k] = (uint8_t)q;
            qhi[k] = (uint8_t)r;
        }
        if (ok) { ebiased = (uint8_t)e; return true; }
    }
    return false;
}

}  // namespace

namespace {

// One wide node to fill: its index in the node array being written, the binary
// subtrees that become its slots, and its depth.
struct Job {
    uint32_t w;
    std::vector<Slot> slots;
    uint32_t depth;
};

// Wide nodes, leaf-triangle records and their binary-leaf records of one part of
// the collapse (the whole tree, or one subtree built on a worker thread).
struct Part {
    RawVec<uint32_t> nodes;          // 20 words per node (each written in full by its fill)
    RawVec<float> tris;              // 12 floats per leaf triangle
    RawVec<uint32_t> tri_leaf;       // 8 words per leaf triangle
    uint32_t num_nodes = 0;
    uint32_t max_depth = 0;
    std::string err;
};

struct Collapse {
    const PNode* nodes;
    const uint32_t* leaf;
    uint64_t leaf_words;
    const float* pos;
    bool root_is_leaf;

    uint32_t leaf_tris(uint32_t nid) const {
        const uint32_t off = nodes[nid & kMask].nid[3];
        if (off == 0xFFFFFFFFu || off >= leaf_words) return 0u;
        return leaf[off] & 0xFFFu;
    }

    void emit_tris(Part& out, uint32_t nid, const Slot& box, bool no_box_test) const {
        const uint32_t nm = nid & kMask;
        uint32_t e[8];
        std::memcpy(&e[0], box.elo, 12);
        e[3] = nm;
        std::memcpy(&e[4], box.ehi, 12);
        // 1: tested without a box; 2: the boxes on its path do not overlap, so
        // reachability cannot be shown from E (the kernel uses the binary walk)
        const bool empty = box.elo[0] > box.ehi[0] || box.elo[1] > box.ehi[1] || box.elo[2] > box.ehi[2];
        e[7] = no_box_test ? 1u : (empty ? 2u : 0u);
        const uint32_t off = nodes[nm].nid[3];
        const uint32_t nt = leaf_tris(nid);
        for (uint32_t t = 0; t < nt; ++t) {
            const uint32_t* r = leaf + 1u + off + 3u * t;
            const uint32_t i0 = r[0] + (r[1] & 0xFFFFu), i1 = r[0] + (r[1] >> 16), i2 = r[0] + (r[2] & 0xFFFFu);
            const float* P0 = pos + 3ull * i0;
            const float* P1 = pos + 3ull * i1;
            const float* P2 = pos + 3ull * i2;
            float w[12];
            w[0] = P0[0]; w[1] = P0[1]; w[2] = P0[2];
            w[4] = P1[0] - P0[0]; w[5] = P1[1] - P0[1]; w[6] = P1[2] - P0[2];
            w[8] = P2[0] - P0[0]; w[9] = P2[1] - P0[1]; w[10] = P2[2] - P0[2];
            std::memcpy(&w[3], &r[0], 4);
            std::memcpy(&w[7], &r[1], 4);
            std::memcpy(&w[11], &r[2], 4);
            out.tris.insert(out.tris.end(), w, w + 12);
            out.tri_leaf.insert(out.tri_leaf.end(), e, e + 8);
        }
    }

    // Choice of the slots of every wide node: a dynamic programme over the binary
    // tree for the cut of at most 8 subtrees of least surface-area cost (the
    // collapse of Ylitie, Karras & Laine 2017, section 3.1, restricted to cuts of
    // the reference tree so that every slot stays one binary subtree and every
    // binary leaf keeps its triangles and order). cost[x][k] is the least cost of
    // covering the subtree of x with at most k slots: a leaf slot costs
    // A * (c_leaf + c_tri * triangles), an internal slot A * c_node plus the best
    // cover of its two children by at most 8 slots, A the surface area of the box
    // the parent record stores; leaves without triangles take no slot. Filled
    // bottom-up over node ids (children have larger ids than their parent).
    static constexpr float kNodeCost = 1.0f, kLeafCost = 0.15f, kTriCost = 0.25f;
    std::vector<float> cost;            // 9 per node (as a child of its parent)
    std::vector<int8_t> choice;         // 9 per node: -1 = one slot, j = j slots on the left child's side
    std::vector<int8_t> split;          // per left child id: slots on its side in its parent's wide node
    bool boxes_finite = true;           // every child box of the tree is finite (else the collapse refuses it)

    static float slot_area(const float lo[3], const float hi[3]) {
        const float dx = std::fabs(hi[0] - lo[0]), dy = std::fabs(hi[1] - lo[1]), dz = std::fabs(hi[2] - lo[2]);
        const float a = dx * dy + dy * dz + dz * dx;
        return std::isfinite(a) ? a : 3.0e38f;
    }

    void plan(uint32_t num_nodes) {
        const float inf = INFINITY;
        cost.assign(9ull * num_nodes, inf);
        choice.assign(9ull * num_nodes, (int8_t)-1);
        split.assign(num_nodes, (int8_t)1);
        // best cover of an internal node's two children by at most k slots
        auto pair_best = [&](uint32_t l, int k, int& jbest) {
            float best = inf;
            jbest = -1;
            for (int j = 0; j <= k; ++j) {
                const float v = cost[9ull * l + j] + cost[9ull * (l + 1u) + (k - j)];
                if (v < best) { best = v; jbest = j; }
            }
            return best;
        };
        for (uint32_t pi = num_nodes; pi-- > 0;) {
            const PNode& p = nodes[pi];
            const uint32_t left = p.nid[2] & kMask;
            if (left == kInvalid) continue;
            Slot a, b;
            child_slots(p, a, b, nullptr);
            for (int ax = 0; ax < 3; ++ax)
                boxes_finite = boxes_finite && std::isfinite(a.lo[ax]) && std::isfinite(a.hi[ax]) &&
                               std::isfinite(b.lo[ax]) && std::isfinite(b.hi[ax]);
            for (const Slot* c : {&a, &b}) {
                const uint32_t ci = c->id & kMask;
                float* f = cost.data() + 9ull * ci;
                int8_t* ch = choice.data() + 9ull * ci;
                const float area_c = slot_area(c->lo, c->hi);
                if (c->id & kLeafBit) {
                    const uint32_t nt = leaf_tris(c->id);
                    for (int k = 0; k <= 8; ++k) f[k] = nt == 0u ? 0.0f : (k == 0 ? inf : area_c * (kLeafCost + kTriCost * (float)nt));
                    continue;
                }
                const uint32_t cl = nodes[ci].nid[2] & kMask;   // validated: an inner node has children
                int j8;
                const float single = area_c * kNodeCost + pair_best(cl, 8, j8);
                split[cl] = (int8_t)j8;
                for (int k = 0; k <= 8; ++k) {
                    int j;
                    float best = pair_best(cl, k, j);   // several slots below this node
                    int8_t c8 = (int8_t)j;
                    if (k >= 1 && single <= best) { best = single; c8 = -1; }
                    f[k] = best;
                    ch[k] = c8;
                }
            }
        }
        const uint32_t root_left = nodes[0].nid[2] & kMask;
        if (root_left != kInvalid) {   // a single-leaf tree has no wide node to plan
            int j0;
            pair_best(root_left, 8, j0);
            split[root_left] = (int8_t)j0;
        }
    }

    // The slots of the cut of x's subtree by at most k slots (the plan's choice).
    void cut(const Slot& x, int k, std::vector<Slot>& out) const {
        if (x.id & kLeafBit) {
            if (leaf_tris(x.id) > 0u) out.push_back(x);   // leaves of no triangle never produce hits
            return;
        }
        const int8_t c = choice[9ull * (x.id & kMask) + k];
        if (c < 0) {
            out.push_back(x);
            return;
        }
        Slot a, b;
        child_slots(nodes[x.id & kMask], a, b, &x);
        cut(a, c, out);
        cut(b, k - c, out);
    }

    // The slots of the wide node of the binary node whose children are a and b.
    std::vector<Slot> expand(const std::vector<Slot>& ab) const {
        std::vector<Slot> kept;
        const int j = split[ab[0].id & kMask];
        cut(ab[0], j < 0 ? 1 : j, kept);
        cut(ab[1], j < 0 ? 1 : 8 - j, kept);
        return kept;
    }

    // Writes wide node job.w of `out` and queues its internal children (numbered
    // consecutively after the nodes `out` holds).
    bool fill(const Job& job, Part& out, std::deque<Job>& q) const {
        out.max_depth = std::max(out.max_depth, job.depth);
        const std::vector<Slot>& fr = job.slots;
        int slot_child[8];
        assign_octant_slots(fr, root_is_leaf, slot_child);
        const int nf = (int)fr.size();
        float lo[3][8], hi[3][8];
        for (int i = 0; i < nf; ++i)
            for (int a = 0; a < 3; ++a) {
                lo[a][i] = std::min(fr[i].lo[a], fr[i].hi[a]);   // the slab test orders each axis itself
                hi[a][i] = std::max(fr[i].lo[a], fr[i].hi[a]);
            }
        uint8_t e[3] = {1, 1, 1}, cq_lo[3][8] = {}, cq_hi[3][8] = {}, qlo[3][8] = {}, qhi[3][8] = {};
        float origin[3] = {0.f, 0.f, 0.f};
        if (nf > 0) {
            for (int a = 0; a < 3; ++a)
                if (!quantise_axis(lo[a], hi[a], nf, origin[a], e[a], cq_lo[a], cq_hi[a])) {
                    out.err = "box bounds cannot be quantised (non-finite coordinates, or a node wider than 255 * 2^40)";
                    return false;
                }
        }
        Slot sl[8];
        bool used[8] = {};
        for (int k = 0; k < 8; ++k) {
            const int i = slot_child[k];
            if (i < 0) {   // empty slot: an inverted box, which the kernel's slab test rejects
                for (int a = 0; a < 3; ++a) { qlo[a][k] = 255; qhi[a][k] = 0; }
                continue;
            }
            used[k] = true;
            sl[k] = fr[i];
            for (int a = 0; a < 3; ++a) { qlo[a][k] = cq_lo[a][i]; qhi[a][k] = cq_hi[a][i]; }
        }
        uint32_t imask = 0, n_internal = 0;
        for (int k = 0; k < 8; ++k)
            if (used[k] && !(sl[k].id & kLeafBit)) { imask |= 1u << k; ++n_internal; }
        const uint32_t child_base = out.num_nodes;
        out.num_nodes += n_internal;
        out.nodes.resize(20ull * out.num_nodes);
        uint32_t* w = out.nodes.data() + 20ull * job.w;
        std::memset(w, 0, 80);
        std::memcpy(&w[0], &origin[0], 4);
        std::memcpy(&w[1], &origin[1], 4);
        std::memcpy(&w[2], &origin[2], 4);
        w[3] = (uint32_t)e[0] | ((uint32_t)e[1] << 8) | ((uint32_t)e[2] << 16) | (imask << 24);
        w[4] = child_base;
        w[5] = (uint32_t)(out.tris.size() / 12);
        uint8_t meta[8] = {};
        for (int k = 0; k < 8; ++k) {
            if (used[k] && (sl[k].id & kLeafBit)) {
                const uint32_t nt = leaf_tris(sl[k].id);
                if (nt > 255u) { out.err = "a leaf holds more than 255 triangles (8-wide slot limit)"; return false; }
                meta[k] = (uint8_t)nt;
                emit_tris(out, sl[k].id, sl[k], root_is_leaf);
            }
        }
        std::memcpy(&w[6], meta, 8);
        uint8_t* qb = reinterpret_cast<uint8_t*>(&w[8]);
        for (int k = 0; k < 8; ++k) {
            qb[0 + k] = qlo[0][k]; qb[8 + k] = qlo[1][k]; qb[16 + k] = qlo[2][k];
            qb[24 + k] = qhi[0][k]; qb[32 + k] = qhi[1][k]; qb[40 + k] = qhi[2][k];
        }
        uint32_t ci = child_base;
        for (int k = 0; k < 8; ++k) {
            if (used[k] && !(sl[k].id & kLeafBit)) {
                Slot a, b;
                child_slots(nodes[sl[k].id], a, b, &sl[k]);
                q.push_back({ci++, expand({a, b}), job.depth + 1u});
            }
        }
        return true;
    }

    // Every wide node below (and including) `job`, into a fresh part whose node 0
    // is the job's own node.
    void subtree(const Job& job, Part& out) const {
        out.num_nodes = 1;
        out.nodes.resize(20);
        std::deque<Job> q;
        q.push_back({0u, job.slots, job.depth});
        while (!q.empty()) {
            Job j = std::move(q.front());
            q.pop_front();
            if (!fill(j, out, q)) return;
        }
    }
};

}  // namespace

bool build_wide(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                WideHost& out, std::string& err) {
    Collapse C;
    C.nodes = reinterpret_cast<const PNode*>(blob + ranges[TIM_RT_RANGE_NODE][0]);
    C.leaf = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_LEAF][0]);
    C.leaf_words = ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    C.pos = pos;
    C.root_is_leaf = num_nodes == 1u;
    C.plan(num_nodes);
    if (!C.boxes_finite) {
        // a non-finite box can make the reference skip a subtree the 8-wide form would open
        err = "box bounds cannot be quantised (non-finite coordinates)";
        return false;
    }
    out = WideHost();
    Part top;
    top.nodes.reserve(20ull * (num_nodes / 4 + 4));
    top.nodes.resize(20);
    top.num_nodes = 1;
    std::deque<Job> q;
    if (C.root_is_leaf) {
        Slot s;
        s.id = kLeafBit;
        for (int a = 0; a < 3; ++a) { s.lo[a] = s.hi[a] = s.elo[a] = s.ehi[a] = 0.f; }
        q.push_back({0u, {s}, 1u});
        out.root_is_leaf = 1u;
    } else {
        Slot a, b;
        child_slots(C.nodes[0], a, b, nullptr);
        q.push_back({0u, C.expand({a, b}), 1u});
    }
    // breadth first on this thread until there are enough independent subtrees ...
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t enough = num_nodes > 16384u && hw > 1u ? 256u : (size_t)-1;
    while (!q.empty() && q.size() < enough) {
        Job j = std::move(q.front());
        q.pop_front();
        if (!C.fill(j, top, q)) { err = top.err; return false; }
    }
    // ... then each pending subtree on a worker thread, merged in queue order
    // (the numbering does not depend on the number of threads)
    std::vector<Job> pending(std::make_move_iterator(q.begin()), std::make_move_iterator(q.end()));
    std::vector<Part> parts(pending.size());
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < pending.size();) C.subtree(pending[k], parts[k]);
    };
    std::vector<std::thread> pool;
    const size_t nthreads = pending.empty() ? 0 : std::min<size_t>(hw, pending.size());
    for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(work);
    if (nthreads) work();
    for (std::thread& t : pool) t.join();
    uint32_t max_depth = top.max_depth;
    // merge: the parts' nodes follow the top nodes in queue order, each part's node 0
    // replaces its pending slot; sizes first, then copies and index fix-ups in parallel
    std::vector<uint64_t> node_off(parts.size()), tri_off(parts.size());
    uint64_t nn = top.num_nodes, nt = top.tris.size() / 12;
    for (size_t k = 0; k < parts.size(); ++k) {
        if (!parts[k].err.empty()) { err = parts[k].err; return false; }
        max_depth = std::max(max_depth, parts[k].max_depth);
        node_off[k] = nn;
        tri_off[k] = nt;
        nn += parts[k].num_nodes - 1u;
        nt += parts[k].tris.size() / 12;
    }
    if (nn >= (1u << 24)) { err = "more than 2^24 8-wide nodes"; return false; }
    top.nodes.resize(20ull * nn);
    top.tris.resize(12ull * nt);
    top.tri_leaf.resize(8ull * nt);
    next = 0;
    auto merge = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < parts.size();) {
            Part& p = parts[k];
            for (uint32_t i = 0; i < p.num_nodes; ++i) {
                uint32_t* w = p.nodes.data() + 20ull * i;
                w[4] = (uint32_t)node_off[k] + w[4] - 1u;   // children: local ids >= 1
                w[5] += (uint32_t)tri_off[k];
            }
            std::memcpy(top.nodes.data() + 20ull * pending[k].w, p.nodes.data(), 80);
            if (p.num_nodes > 1u)
                std::memcpy(top.nodes.data() + 20ull * node_off[k], p.nodes.data() + 20, 80ull * (p.num_nodes - 1u));
            if (!p.tris.empty()) {
                std::memcpy(top.tris.data() + 12ull * tri_off[k], p.tris.data(), 4ull * p.tris.size());
                std::memcpy(top.tri_leaf.data() + 8ull * tri_off[k], p.tri_leaf.data(), 4ull * p.tri_leaf.size());
            }
            RawVec<uint32_t>().swap(p.nodes);   // release the part's memory early
            RawVec<float>().swap(p.tris);
            RawVec<uint32_t>().swap(p.tri_leaf);
        }
    };
    pool.clear();
    for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(merge);
    if (nthreads) merge();
    for (std::thread& t : pool) t.join();
    top.num_nodes = (uint32_t)nn;
    out.nodes = std::move(top.nodes);
    out.tris = std::move(top.tris);
    out.tri_leaf = std::move(top.tri_leaf);
    out.num_nodes = top.num_nodes;
    out.max_depth = max_depth;
    if (out.max_depth > 32u) { err = "8-wide tree deeper than 32 levels"; return false; }
    if (out.num_nodes >= (1u << 24)) { err = "more than 2^24 8-wide nodes"; return false; }
    return true;
}

// ---------------------------------------------------------------------------------- 8-wide check

namespace {

bool same_bits(const float* a, const float* b, int n) { return std::memcmp(a, b, 4 * (size_t)n) == 0; }

// One wide node of the check: its index and the binary subtrees that must be its slots.
struct CheckJob {
    uint32_t w;
    std::vector<Slot> slots;
    uint32_t depth;
};

}  // namespace

// Checks an 8-wide form against the binary tree it was built from. It replays the
// collapse's choice of slots (the same expand and octant placement) from the
// root and verifies, node by node: each used slot's 8-bit box contains the box
// the reference stores for that subtree (per plane, in extended precision);
// empty slots hold the inverted box and no triangles; internal slots point at
// distinct, in-range nodes; each leaf slot holds exactly its binary leaf's
// triangles in the leaf's order, with the reference's records, p0 and the
// rounded edges p1 - p0 and p2 - p0 bit for bit, and per triangle the leaf's id,
// its ancestor-intersection box and its flag. Finally every wide node and every
// wide triangle must have been reached exactly once.
bool check_wide(const uint8_t* blob, const uint32_t ranges[7][2], uint32_t num_nodes, const float* pos,
                const WideHost& w, tim_rt_wide_report& rep, std::string& err) {
    Collapse C;
    C.nodes = reinterpret_cast<const PNode*>(blob + ranges[TIM_RT_RANGE_NODE][0]);
    C.leaf = reinterpret_cast<const uint32_t*>(blob + ranges[TIM_RT_RANGE_LEAF][0]);
    C.leaf_words = ranges[TIM_RT_RANGE_LEAF][1] / 4u;
    C.pos = pos;
    C.root_is_leaf = num_nodes == 1u;
    C.plan(num_nodes);
    std::memset(&rep, 0, sizeof(rep));
    if (!C.boxes_finite) { err = "box bounds cannot be quantised (non-finite coordinates)"; return false; }
    const uint64_t nw = w.num_nodes, nt = w.tris.size() / 12;
    if (nw == 0 || w.nodes.size() != 20ull * nw || w.tri_leaf.size() != 8ull * nt) { err = "8-wide arrays have inconsistent sizes"; return false; }
    std::vector<uint8_t> node_seen(nw, 0), tri_seen(nt, 0);
    std::vector<CheckJob> stack;
    if (C.root_is_leaf) {
        Slot s;
        s.id = kLeafBit;
        for (int a = 0; a < 3; ++a) { s.lo[a] = s.hi[a] = s.elo[a] = s.ehi[a] = 0.f; }
        stack.push_back({0u, {s}, 1u});
    } else {
        Slot a, b;
        child_slots(C.nodes[0], a, b, nullptr);
        stack.push_back({0u, C.expand({a, b}), 1u});
    }
    auto fail = [&](uint32_t wi, const std::string& what) {
        err = "8-wide node " + std::to_string(wi) + ": " + what;
        return false;
    };
    while (!stack.empty()) {
        CheckJob job = std::move(stack.back());
        stack.pop_back();
        const uint32_t wi = job.w;
        if (wi >= nw) return fail(wi, "index out of range");
        if (node_seen[wi]) return fail(wi, "reached twice");
        node_seen[wi] = 1;
        rep.depth = std::max(rep.depth, job.depth);
        const uint32_t* W = w.nodes.data() + 20ull * wi;
        float origin[3];
        std::memcpy(origin, W, 12);
        const uint32_t e[3] = {W[3] & 0xFFu, (W[3] >> 8) & 0xFFu, (W[3] >> 16) & 0xFFu};
        const uint32_t imask = W[3] >> 24, child_base = W[4], tri_base = W[5];
        uint8_t meta[8], qb[48];
        std::memcpy(meta, &W[6], 8);
        std::memcpy(qb, &W[8], 48);
        int slot_child[8];
        assign_octant_slots(job.slots, C.root_is_leaf, slot_child);
        uint32_t used = 0, tri_cursor = tri_base;
        for (int k = 0; k < 8; ++k) {
            const int i = slot_child[k];
            if (i < 0) {
                for (int a = 0; a < 3; ++a)
                    if (qb[8 * a + k] != 255u || qb[24 + 8 * a + k] != 0u) return fail(wi, "empty slot without the inverted box");
                if (meta[k] || ((imask >> k) & 1u)) return fail(wi, "empty slot with content");
                continue;
            }
            ++used;
            const Slot& sl = job.slots[i];
            for (int a = 0; a < 3; ++a) {
                float sc;
                const uint32_t bits = e[a] << 23;
                std::memcpy(&sc, &bits, 4);
                const float lo = std::min(sl.lo[a], sl.hi[a]), hi = std::max(sl.lo[a], sl.hi[a]);
                if (!plane_le(origin[a], sc, qb[8 * a + k], lo) || !plane_ge(origin[a], sc, qb[24 + 8 * a + k], hi))
                    return fail(wi, "slot " + std::to_string(k) + " box does not contain the reference box");
            }
            if (sl.id & kLeafBit) {
                if ((imask >> k) & 1u) return fail(wi, "leaf slot marked internal");
                const uint32_t n = C.leaf_tris(sl.id);
                if (meta[k] != n) return fail(wi, "leaf slot triangle count differs from the binary leaf");
                ++rep.leaf_slots;
                const uint32_t nm = sl.id & kMask, off = C.nodes[nm].nid[3];
                for (uint32_t t = 0; t < n; ++t, ++tri_cursor) {
                    if (tri_cursor >= nt) return fail(wi, "leaf triangles out of range");
                    if (tri_seen[tri_cursor]) return fail(wi, "wide triangle used twice");
                    tri_seen[tri_cursor] = 1;
                    const uint32_t* r = C.leaf + 1u + off + 3u * t;
                    const float* T = w.tris.data() + 12ull * tri_cursor;
                    uint32_t rec[3];
                    std::memcpy(&rec[0], &T[3], 4);
                    std::memcpy(&rec[1], &T[7], 4);
                    std::memcpy(&rec[2], &T[11], 4);
                    if (rec[0] != r[0] || rec[1] != r[1] || rec[2] != r[2]) return fail(wi, "triangle record differs");
                    const float* P0 = pos + 3ull * (r[0] + (r[1] & 0xFFFFu));
                    const float* P1 = pos + 3ull * (r[0] + (r[1] >> 16));
                    const float* P2 = pos + 3ull * (r[0] + (r[2] & 0xFFFFu));
                    const float e1[3] = {P1[0] - P0[0], P1[1] - P0[1], P1[2] - P0[2]};
                    const float e2[3] = {P2[0] - P0[0], P2[1] - P0[1], P2[2] - P0[2]};
                    if (!same_bits(T, P0, 3) || !same_bits(T + 4, e1, 3) || !same_bits(T + 8, e2, 3))
                        return fail(wi, "triangle vertices or edges differ");
                    const uint32_t* L = w.tri_leaf.data() + 8ull * tri_cursor;
                    float elo[3], ehi[3];
                    std::memcpy(elo, &L[0], 12);
                    std::memcpy(ehi, &L[4], 12);
                    const bool empty = sl.elo[0] > sl.ehi[0] || sl.elo[1] > sl.ehi[1] || sl.elo[2] > sl.ehi[2];
                    const uint32_t flag = C.root_is_leaf ? 1u : (empty ? 2u : 0u);
                    if (L[3] != nm || L[7] != flag || !same_bits(elo, sl.elo, 3) || !same_bits(ehi, sl.ehi, 3))
                        return fail(wi, "binary-leaf record of a triangle differs");
                }
            } else {
                if (!((imask >> k) & 1u)) return fail(wi, "internal slot not marked internal");
                if (meta[k]) return fail(wi, "internal slot with triangles");
                ++rep.internal_slots;
                const uint32_t child = child_base + (uint32_t)__builtin_popcount(imask & ((1u << k) - 1u));
                Slot a, b;
                child_slots(C.nodes[sl.id], a, b, &sl);
                stack.push_back({child, C.expand({a, b}), job.depth + 1u});
            }
        }
        ++rep.slot_histogram[used];
    }
    for (uint64_t i = 0; i < nw; ++i)
        if (!node_seen[i]) { err = "8-wide node " + std::to_string(i) + " is not reachable"; return false; }
    for (uint64_t i = 0; i < nt; ++i)
        if (!tri_seen[i]) { err = "8-wide triangle " + std::to_string(i) + " belongs to no leaf slot"; return false; }
    rep.nodes = (uint32_t)nw;
    rep.triangles = (uint32_t)nt;
    rep.device_bytes = 80ull * nw + 48ull * nt + 32ull * nt;
    if (rep.depth != w.max_depth) { err = "8-wide depth differs from the recorded depth"; return false; }
    return true;
}

}  // namespace timrt

extern "C" int tim_rt_wide_check(const void* bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                                 const tim_rt_push_constants* pc, const float* pos, uint32_t num_vertex,
                                 tim_rt_wide_report* report) {
    if (!bvh_bytes || !ranges || !pc || !pos || !report) {
        timrt::set_error("tim_rt_wide_check: null argument");
        return TIM_RT_EINVAL;
    }
    std::memset(report, 0, sizeof(*report));
    std::string err;
    const uint8_t* blob = static_cast<const uint8_t*>(bvh_bytes);
    uint32_t depth = 0;
    if (!timrt::validate_bvh(blob, n_bytes, ranges, pc->numNodes, num_vertex, pc->numLights, pc->numBlas, &depth, err)) {
        timrt::set_error("tim_rt_wide_check: " + err);
        return TIM_RT_EINVAL;
    }
    timrt::WideHost w;
    if (!timrt::build_wide(blob, ranges, pc->numNodes, pos, w, err) ||
        !timrt::check_wide(blob, ranges, pc->numNodes, pos, w, *report, err)) {
        timrt::set_error("tim_rt_wide_check: " + err);
        return TIM_RT_EINVAL;
    }
    return TIM_RT_OK;
}
