// bvh_build.cu -- host-side construction of the 8-wide bounding-volume
// hierarchy the tracers use to find candidate leaves in the world tree.
//
// merlict finds candidates by walking its own frame tree, whose octant
// clustering (merlict/Frame.cpp:190-255) gives heavily overlapping bounding
// spheres: ~400 sphere tests per photon in the light-field telescope.  The
// tracers instead walk a BVH built here by binned surface-area-heuristic
// splits over the leaves' bounding spheres, collapsed to eight children per
// node.  The BVH only proposes candidates; every candidate is then put
// through merlict's own bounding-sphere test of that leaf and merlict's
// intersection, and ties are broken in merlict's visiting order, so the
// closest hit is merlict's.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

struct Box {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
    double hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    void grow(const Box& b) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    void grow(const double* p) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    double area() const {
        if (hi[0] < lo[0]) return 0.0;
        const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0*(dx*dy + dy*dz + dz*dx);
    }
};

struct BNode {            // binary build node
    Box box;
    int32_t left = -1, right = -1;
    int32_t begin = 0, end = 0;   // leaf range when left < 0
};

constexpr int kLeafMax = 4;
constexpr int kBins = 16;

class Builder {
 public:
    std::vector<Box> prim_box;
    std::vector<double> centroid;   // 3 per primitive
    std::vector<int32_t> order;     // permutation of primitive ids
    std::vector<BNode> nodes;

    int32_t build(int32_t begin, int32_t end, int depth) {
        const int32_t id = (int32_t)nodes.size();
        nodes.emplace_back();
        Box box, cbox;
        for (int32_t i = begin; i < end; i++) {
            box.grow(prim_box[order[i]]);
            cbox.grow(&centroid[3*(size_t)order[i]]);
        }
        nodes[id].box = box;
        const int32_t n = end - begin;
        if (n <= kLeafMax) {
            nodes[id].begin = begin;
            nodes[id].end = end;
            return id;
        }
        int axis = 0;
        double ext = -1.0;
        for (int k = 0; k < 3; k++)
            if (cbox.hi[k] - cbox.lo[k] > ext) { ext = cbox.hi[k] - cbox.lo[k]; axis = k; }
        int32_t mid = begin + n/2;
        if (ext > 0.0 && depth <= 40) {
            Box bin_box[kBins];
            int32_t bin_count[kBins] = {0};
            const double scale = kBins/ext;
            auto bin_of = [&](int32_t p) {
                int b = (int)((centroid[3*(size_t)p + axis] - cbox.lo[axis])*scale);
                return std::min(std::max(b, 0), kBins - 1);
            };
            for (int32_t i = begin; i < end; i++) {
                const int b = bin_of(order[i]);
                bin_count[b]++;
                bin_box[b].grow(prim_box[order[i]]);
            }
            double best = DBL_MAX;
            int best_split = -1;
            for (int s = 1; s < kBins; s++) {
                Box l, r;
                int32_t nl = 0, nr = 0;
                for (int b = 0; b < s; b++) { if (bin_count[b]) { l.grow(bin_box[b]); nl += bin_count[b]; } }
                for (int b = s; b < kBins; b++) { if (bin_count[b]) { r.grow(bin_box[b]); nr += bin_count[b]; } }
                if (!nl || !nr) continue;
                const double cost = l.area()*nl + r.area()*nr;
                if (cost < best) { best = cost; best_split = s; }
            }
            if (best_split > 0) {
                int32_t* first = order.data() + begin;
                int32_t* last = order.data() + end;
                int32_t* m = std::partition(first, last, [&](int32_t p) { return bin_of(p) < best_split; });
                mid = (int32_t)(m - order.data());
                if (mid == begin || mid == end) mid = begin + n/2;
            } else {
                std::sort(order.begin() + begin, order.begin() + end, [&](int32_t a, int32_t b) {
                    return centroid[3*(size_t)a + axis] < centroid[3*(size_t)b + axis];
                });
            }
        }
        const int32_t l = build(begin, mid, depth + 1);
        const int32_t r = build(mid, end, depth + 1);
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }
};

float round_down(double x) {
    float f = (float)x;
    if ((double)f > x) f = std::nextafter(f, -FLT_MAX);
    return f;
}
float round_up(double x) {
    float f = (float)x;
    if ((double)f < x) f = std::nextafter(f, FLT_MAX);
    return f;
}

}  // namespace

// Builds the BVH of all leaves with geometry.  `inflate` widens every leaf
// box (absolute, metres) so that single-precision slab tests stay
// conservative.
void build_bvh(const mlgpu_flat_scene* f, double inflate, BvhHost* out) {
    out->nodes.clear();
    out->leaf_ids.clear();
    out->levels = 0;
    Builder b;
    for (int32_t l = 0; l < f->num_leaves; l++) {
        if (f->leaf_primitive[l] == MLGPU_PRIM_NONE) continue;
        const double* c = f->node_sphere + 4*(size_t)f->leaf_node[l];
        Box box;
        const double r = c[3] + inflate;
        for (int k = 0; k < 3; k++) { box.lo[k] = c[k] - r; box.hi[k] = c[k] + r; }
        b.prim_box.push_back(box);
        b.centroid.push_back(c[0]);
        b.centroid.push_back(c[1]);
        b.centroid.push_back(c[2]);
        out->leaf_ids.push_back(l);
    }
    const int32_t n = (int32_t)out->leaf_ids.size();
    if (n == 0) return;
    b.order.resize(n);
    for (int32_t i = 0; i < n; i++) b.order[i] = i;
    b.nodes.reserve(2*(size_t)n);
    b.build(0, n, 0);
    // primitive order of the leaf ranges
    std::vector<int32_t> ids(n);
    for (int32_t i = 0; i < n; i++) ids[i] = out->leaf_ids[b.order[i]];
    out->leaf_ids.swap(ids);

    // collapse to kBvhWidth-wide nodes, breadth first from the root
    std::vector<int32_t> queue = {0};
    std::vector<int32_t> wide_of(b.nodes.size(), -1);
    std::vector<int32_t> level = {0};   // per wide node
    wide_of[0] = 0;
    out->nodes.emplace_back();
    out->levels = 1;
    for (size_t qi = 0; qi < queue.size(); qi++) {
        const int32_t bn = queue[qi];
        const int32_t w = wide_of[bn];
        std::vector<int32_t> kids;
        if (b.nodes[bn].left < 0) {
            kids.push_back(bn);   // a root that is a leaf
        } else {
            kids.push_back(b.nodes[bn].left);
            kids.push_back(b.nodes[bn].right);
            while (kids.size() < (size_t)kBvhWidth) {
                int best = -1;
                double area = -1.0;
                for (size_t k = 0; k < kids.size(); k++) {
                    const BNode& c = b.nodes[kids[k]];
                    if (c.left >= 0 && c.box.area() > area) { area = c.box.area(); best = (int)k; }
                }
                if (best < 0) break;
                const BNode c = b.nodes[kids[best]];
                kids[best] = c.left;
                kids.push_back(c.right);
            }
        }
        BvhNode node;
        std::memset(&node, 0, sizeof(node));
        for (int k = 0; k < kBvhWidth; k++) {
            node.lo[0][k] = 1.0f; node.hi[0][k] = -1.0f;   // empty slot never hits
            node.lo[1][k] = 1.0f; node.hi[1][k] = -1.0f;
            node.lo[2][k] = 1.0f; node.hi[2][k] = -1.0f;
            node.child[k] = kBvhEmpty;
        }
        for (size_t k = 0; k < kids.size(); k++) {
            const BNode& c = b.nodes[kids[k]];
            for (int a = 0; a < 3; a++) {
                node.lo[a][k] = round_down(c.box.lo[a]);
                node.hi[a][k] = round_up(c.box.hi[a]);
            }
            if (c.left < 0) {
                const int32_t count = c.end - c.begin;
                node.child[k] = kBvhLeafFlag | (c.begin << 3) | (count - 1);
            } else {
                const int32_t idx = (int32_t)out->nodes.size();
                out->nodes.emplace_back();
                level.push_back(level[w] + 1);
                out->levels = std::max(out->levels, level[w] + 2);
                wide_of[kids[k]] = idx;
                queue.push_back(kids[k]);
                node.child[k] = idx;
            }
        }
        out->nodes[w] = node;
    }
    // nodes were numbered in breadth-first order, so each level is a range
    out->level_start.assign((size_t)out->levels + 1, (int32_t)out->nodes.size());
    for (int32_t i = (int32_t)level.size() - 1; i >= 0; i--) out->level_start[level[i]] = i;
    out->level_start[0] = 0;
}

// Quantises a node's float boxes (already rounded outwards) to QNode: per
// axis the origin is the smallest low bound and the step the smallest power
// of two with 255 steps reaching the largest high bound; each bound is
// rounded outwards to whole steps.  origin + q * 2^e is evaluated in double,
// where it is exact for the magnitudes a scenery has, and each bound is
// checked against the float box it stands for.
void quantise_bvh_node(const BvhNode& n, QNode* q) {
    std::memset(q, 0, sizeof(*q));
    uint32_t exps = 0;
    for (int a = 0; a < 3; a++) {
        float lo = FLT_MAX, hi = -FLT_MAX;
        for (int k = 0; k < kBvhWidth; k++) {
            if (n.child[k] == kBvhEmpty) continue;
            lo = std::min(lo, n.lo[a][k]);
            hi = std::max(hi, n.hi[a][k]);
        }
        if (lo > hi) { lo = 0.0f; hi = 0.0f; }   // no children (not built)
        const double ext = (double)hi - (double)lo;
        int e = -126;                            // the smallest normal step
        while (e < 127 && std::ldexp(255.0, e) < ext) e++;
        const double step = std::ldexp(1.0, e);
        q->origin[a] = lo;
        exps |= (uint32_t)(e + 127) << (8*a);
        for (int k = 0; k < kBvhWidth; k++) {
            uint32_t ql = 0, qh = 0;
            if (n.child[k] != kBvhEmpty) {
                double l = std::floor(((double)n.lo[a][k] - (double)lo)/step);
                double h = std::ceil(((double)n.hi[a][k] - (double)lo)/step);
                l = std::min(std::max(l, 0.0), 255.0);
                h = std::min(std::max(h, 0.0), 255.0);
                while (l > 0.0 && (double)lo + l*step > (double)n.lo[a][k]) l -= 1.0;
                while (h < 255.0 && (double)lo + h*step < (double)n.hi[a][k]) h += 1.0;
                ql = (uint32_t)l;
                qh = (uint32_t)h;
            }
            q->qlo[a][k >> 2] |= ql << (8*(k & 3));
            q->qhi[a][k >> 2] |= qh << (8*(k & 3));
        }
    }
    q->exps = exps;
    for (int k = 0; k < kBvhWidth; k++) q->child[k] = n.child[k];
}

}  // namespace mlgpu
