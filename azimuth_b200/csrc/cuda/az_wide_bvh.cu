// Collapse of a binary BVH into 8-wide compressed nodes (host side).
//
// The binary LBVH built on the GPU (az_bvh_build.cu) is read back and turned
// into WideNode records: every wide node takes a binary node and repeatedly
// opens the child with the largest surface area until it has `width` (2, 4
// or 8) children;
// subtrees of at most `max_leaf` primitives become leaf children.  Children
// are placed in the slot matching the octant of their centre relative to the
// node centre, so a ray visits slots near-first by XOR-ing with its direction
// octant.  Child boxes are quantised conservatively to an 8-bit grid per node.
// Leaf primitives are re-ordered so that every node's leaf primitives are
// consecutive (prim_base + offset).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "az_internal.h"

namespace az {
namespace {

struct Item {
    uint32_t ref;        // binary node index (global) or sorted primitive position
    bool prim;           // single primitive
    uint32_t first, count;
    float lo[3], hi[3];
};

struct Range {
    uint32_t first, count;
};

double Area(const float lo[3], const float hi[3]) {
    double dx = std::max(0.0, (double)hi[0] - lo[0]), dy = std::max(0.0, (double)hi[1] - lo[1]),
           dz = std::max(0.0, (double)hi[2] - lo[2]);
    return dx * dy + dy * dz + dz * dx;
}

struct Collapser {
    const std::vector<azd::BVHNode> &bin;
    uint32_t node_base;                  // global index of bin[0]
    std::vector<Range> range;            // per binary node (local index)
    uint32_t max_leaf;
    uint32_t width = 8;                  // children per wide node: 2, 4 or 8
    std::vector<azd::WideNode> &out;
    uint32_t wide_base;                  // global index of out[0]
    std::vector<uint32_t> &prim_order;   // output slot -> sorted primitive position
    uint32_t prim_out_base;              // global index of prim_order[0]
    uint32_t max_depth = 0;
    bool bad_box = false;                // a quantised box failed to contain its child

    Collapser(const std::vector<azd::BVHNode> &b, uint32_t nb, uint32_t ml, std::vector<azd::WideNode> &o, uint32_t wb,
              std::vector<uint32_t> &po, uint32_t pob)
        : bin(b), node_base(nb), max_leaf(ml), out(o), wide_base(wb), prim_order(po), prim_out_base(pob) {}

    Item ChildItem(const azd::BVHNode &n, int c) {
        Item it;
        uint32_t ref = c == 0 ? n.ch.x : n.ch.y, cnt = c == 0 ? n.ch.z : n.ch.w;
        const float *bx = &n.bx.x, *by = &n.by.x, *bz = &n.bz.x;
        it.lo[0] = bx[2 * c]; it.hi[0] = bx[2 * c + 1];
        it.lo[1] = by[2 * c]; it.hi[1] = by[2 * c + 1];
        it.lo[2] = bz[2 * c]; it.hi[2] = bz[2 * c + 1];
        it.ref = ref;
        if (cnt) {
            it.prim = true;
            it.first = ref;
            it.count = 1;
        } else {
            it.prim = false;
            const Range &r = range[ref - node_base];
            it.first = r.first;
            it.count = r.count;
        }
        return it;
    }

    // primitive ranges of every binary node, bottom-up without recursion
    void Ranges(uint32_t root) {
        range.assign(bin.size(), Range{0, 0});
        std::vector<std::pair<uint32_t, int>> st{{root, 0}};
        while (!st.empty()) {
            auto &top = st.back();
            const azd::BVHNode &n = bin[top.first - node_base];
            if (top.second == 0) {
                top.second = 1;
                for (int c = 0; c < 2; c++) {
                    uint32_t cnt = c == 0 ? n.ch.z : n.ch.w, ref = c == 0 ? n.ch.x : n.ch.y;
                    if (!cnt) st.push_back({ref, 0});
                }
                continue;
            }
            uint32_t lo = UINT32_MAX, hi = 0;
            for (int c = 0; c < 2; c++) {
                uint32_t cnt = c == 0 ? n.ch.z : n.ch.w, ref = c == 0 ? n.ch.x : n.ch.y;
                uint32_t f, k;
                if (cnt) { f = ref; k = 1; } else { f = range[ref - node_base].first; k = range[ref - node_base].count; }
                lo = std::min(lo, f);
                hi = std::max(hi, f + k);
            }
            range[top.first - node_base] = Range{lo, hi - lo};
            st.pop_back();
        }
    }

    void Quantize(azd::WideNode &w, const Item *kids, const int *slot_of, int nk) {
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = 0; i < nk; i++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], kids[i].lo[a]);
                hi[a] = std::max(hi[a], kids[i].hi[a]);
            }
        // Per axis a grid origin p and a power-of-two step with at least one
        // full step of slack on both sides of every child box, including the
        // ones on the node's own bounds: the device folds the byte-to-float
        // bias into its slab-test FMA at a cost of up to half a step.
        float p[3];
        int e[3];
        for (int a = 0; a < 3; a++) {
            double mag = std::max(std::fabs((double)lo[a]), std::fabs((double)hi[a]));
            double ext = std::max((double)hi[a] - lo[a], std::max(mag * 1e-6, 1e-30));
            int ex = (int)std::ceil(std::log2(ext / 251.0));
            ex = std::max(-126, std::min(127, ex));
            while (true) {
                const double step = std::ldexp(1.0, ex);
                // origin: a float at least one step below lo
                float pa = (float)((double)lo[a] - step);
                while ((double)pa > (double)lo[a] - step) pa = nextafterf(pa, -FLT_MAX);
                const double top = std::ceil(((double)hi[a] - pa) / step) + 1.0;   // hi's byte, with slack
                if (top <= 255.0 || ex >= 127) {
                    p[a] = pa;
                    e[a] = ex;
                    break;
                }
                ex++;
            }
        }
        w.px = p[0]; w.py = p[1]; w.pz = p[2];
        w.ex = (uint8_t)(e[0] + 127); w.ey = (uint8_t)(e[1] + 127); w.ez = (uint8_t)(e[2] + 127);
        uint8_t *qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z}, *qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
        for (int s = 0; s < 8; s++)
            for (int a = 0; a < 3; a++) { qlo[a][s] = 255; qhi[a][s] = 0; }
        for (int i = 0; i < nk; i++) {
            int s = slot_of[i];
            for (int a = 0; a < 3; a++) {
                double step = std::ldexp(1.0, e[a]);
                double l = std::floor(((double)kids[i].lo[a] - p[a]) / step) - 1.0;   // one step of slack
                double h = std::ceil(((double)kids[i].hi[a] - p[a]) / step) + 1.0;
                qlo[a][s] = (uint8_t)std::max(0.0, std::min(255.0, l));
                qhi[a][s] = (uint8_t)std::max(0.0, std::min(255.0, h));
                // the decoded box must hold the child with a full step to spare on both sides
                if ((double)p[a] + qlo[a][s] * step > (double)kids[i].lo[a] - step ||
                    (double)p[a] + qhi[a][s] * step < (double)kids[i].hi[a] + step)
                    bad_box = true;
            }
        }
    }

    // Builds the wide node for `item` at global index `self`.
    void Build(const Item &item, uint32_t self, uint32_t depth) {
        max_depth = std::max(max_depth, depth);
        Item kids[8];
        int nk = 0;
        if (item.prim || item.count <= max_leaf) {
            kids[nk++] = item;   // a hierarchy of at most max_leaf primitives: one leaf child
        } else {
            const azd::BVHNode &n = bin[item.ref - node_base];
            kids[nk++] = ChildItem(n, 0);
            kids[nk++] = ChildItem(n, 1);
        }
        while (nk < (int)width) {
            int best = -1;
            double best_area = -1.0;
            for (int i = 0; i < nk; i++) {
                if (kids[i].prim || kids[i].count < 2) continue;
                // open big subtrees first; small ones only while slots are free
                double a = Area(kids[i].lo, kids[i].hi) * (kids[i].count > max_leaf ? 2.0 : 1.0);
                if (a > best_area) { best_area = a; best = i; }
            }
            if (best < 0) break;
            const azd::BVHNode &n = bin[kids[best].ref - node_base];
            Item a = ChildItem(n, 0), b = ChildItem(n, 1);
            kids[best] = a;
            kids[nk++] = b;
        }
        // slot assignment: child centre octant relative to the node centre
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = 0; i < nk; i++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], kids[i].lo[a]);
                hi[a] = std::max(hi[a], kids[i].hi[a]);
            }
        struct Cand { double score; int kid, slot; };
        std::vector<Cand> cand;
        for (int i = 0; i < nk; i++)
            for (int s = 0; s < 8; s++) {
                double sc = 0.0;
                for (int a = 0; a < 3; a++) {
                    double ext = std::max(1e-30, (double)hi[a] - lo[a]);
                    double c = (0.5 * ((double)kids[i].lo[a] + kids[i].hi[a]) - 0.5 * ((double)lo[a] + hi[a])) / ext;
                    sc += ((s >> a) & 1) ? c : -c;
                }
                cand.push_back(Cand{sc, i, s});
            }
        std::sort(cand.begin(), cand.end(), [](const Cand &x, const Cand &y) { return x.score > y.score; });
        int slot_of[8], kid_of[8];
        for (int i = 0; i < 8; i++) { slot_of[i] = -1; kid_of[i] = -1; }
        for (const Cand &c : cand)
            if (slot_of[c.kid] < 0 && kid_of[c.slot] < 0) {
                slot_of[c.kid] = c.slot;
                kid_of[c.slot] = c.kid;
            }
        azd::WideNode w;
        memset(&w, 0, sizeof(w));
        Quantize(w, kids, slot_of, nk);
        // inner children: consecutive node indices in slot order
        uint32_t n_inner = 0;
        for (int s = 0; s < 8; s++)
            if (kid_of[s] >= 0 && kids[kid_of[s]].count > max_leaf) n_inner++;
        uint32_t child_base = wide_base + (uint32_t)out.size();
        out.resize(out.size() + n_inner);
        w.child_base = child_base;
        w.prim_base = prim_out_base + (uint32_t)prim_order.size();
        uint32_t off = 0;
        uint8_t imask = 0;
        for (int s = 0; s < 8; s++) {
            int k = kid_of[s];
            if (k < 0) continue;
            if (kids[k].count > max_leaf) {
                imask |= (uint8_t)(1u << s);
            } else {
                for (uint32_t j = 0; j < kids[k].count; j++) prim_order.push_back(kids[k].first + j);
                w.meta[s] = (uint8_t)((kids[k].count << 5) | off);
                off += kids[k].count;
            }
        }
        w.imask = imask;
        out[self - wide_base] = w;
        uint32_t rank = 0;
        for (int s = 0; s < 8; s++) {
            int k = kid_of[s];
            if (k < 0 || kids[k].count <= max_leaf) continue;
            Build(kids[k], child_base + rank, depth + 1);
            rank++;
        }
    }
};

}  // namespace

int CollapseToWide(const std::vector<azd::BVHNode> &bin, uint32_t bin_base, uint32_t bin_root, uint32_t max_leaf,
                   uint32_t width, std::vector<azd::WideNode> &out, std::vector<uint32_t> &prim_order,
                   uint32_t prim_out_base, uint32_t *root_out, uint32_t *depth_out) {
    if (max_leaf < 1 || max_leaf > 3) return SetError(AZ_ERR_INVALID_ARGUMENT, "leaf size must be 1..3");
    if (width != 2 && width != 4 && width != 8) return SetError(AZ_ERR_INVALID_ARGUMENT, "BVH width must be 2, 4 or 8");
    // `out` may already hold the nodes of earlier hierarchies: indices are global
    Collapser C(bin, bin_base, max_leaf, out, 0, prim_order, prim_out_base);
    C.width = width;
    uint32_t self = (uint32_t)out.size();
    C.Ranges(bin_root);
    Item root;
    const azd::BVHNode &rn = bin[bin_root - bin_base];
    root.ref = bin_root;
    root.prim = false;
    root.first = C.range[bin_root - bin_base].first;
    root.count = C.range[bin_root - bin_base].count;
    for (int a = 0; a < 3; a++) { root.lo[a] = FLT_MAX; root.hi[a] = -FLT_MAX; }
    const float *bx = &rn.bx.x, *by = &rn.by.x, *bz = &rn.bz.x;
    for (int c = 0; c < 2; c++) {
        root.lo[0] = std::min(root.lo[0], bx[2 * c]); root.hi[0] = std::max(root.hi[0], bx[2 * c + 1]);
        root.lo[1] = std::min(root.lo[1], by[2 * c]); root.hi[1] = std::max(root.hi[1], by[2 * c + 1]);
        root.lo[2] = std::min(root.lo[2], bz[2 * c]); root.hi[2] = std::max(root.hi[2], bz[2 * c + 1]);
    }
    out.resize(out.size() + 1);
    C.Build(root, self, 0);
    *root_out = self;
    if (depth_out) *depth_out = C.max_depth;
    if (C.bad_box) return SetError(AZ_ERR_CUDA, "BVH collapse: a quantised box does not contain its child");
    // structural check of the new nodes before they reach the device
    const uint32_t n_prims = (uint32_t)prim_order.size();
    for (uint32_t i = self; i < out.size(); i++) {
        const azd::WideNode &w = out[i];
        uint32_t inner = (uint32_t)__builtin_popcount(w.imask);
        if (inner && (w.child_base <= i || w.child_base + inner > out.size()))
            return SetError(AZ_ERR_CUDA, "BVH collapse: child index out of range");
        for (int s = 0; s < 8; s++) {
            if ((w.imask >> s) & 1) {
                if (w.meta[s]) return SetError(AZ_ERR_CUDA, "BVH collapse: inner slot with leaf data");
                continue;
            }
            uint32_t cnt = w.meta[s] >> 5, off = w.meta[s] & 31u;
            if (cnt > max_leaf || w.prim_base < prim_out_base ||
                w.prim_base - prim_out_base + off + cnt > n_prims)
                return SetError(AZ_ERR_CUDA, "BVH collapse: leaf range out of range");
        }
    }
    return AZ_OK;
}

}  // namespace az
