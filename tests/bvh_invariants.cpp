// Host-side checks of the BVH the tracers walk (csrc/bvh_build.cu), built
// by tests/test_bvh_invariants.py with the host compiler.  The BVH only
// proposes candidate leaves, so the tracers stay exact as long as
//   * every child box of every node contains the bounding sphere of every
//     leaf beneath that child (a box that missed one could lose a hit),
//   * every leaf with geometry sits in exactly one leaf range,
//   * the children of a node of level L are nodes of level L + 1 (each
//     level is the index range the level kernels walk) and empty child
//     slots hold kBvhEmpty.
#include <cstdint>
#include <vector>

#include "mlgpu_internal.h"

using mlgpu::BvhHost;
using mlgpu::BvhNode;
using mlgpu::kBvhEmpty;
using mlgpu::kBvhLeafFlag;
using mlgpu::kBvhWidth;

namespace {

void leaves_under(const BvhHost& b, int32_t ref, std::vector<int32_t>* out) {
    if (ref == kBvhEmpty) return;
    if (ref & kBvhLeafFlag) {
        const int32_t start = (ref & 0x7fffffff) >> 3, count = (ref & 7) + 1;
        for (int32_t j = start; j < start + count; j++) out->push_back(b.leaf_ids[j]);
        return;
    }
    for (int k = 0; k < kBvhWidth; k++) leaves_under(b, b.nodes[ref].child[k], out);
}

int level_of(const BvhHost& b, int32_t node) {
    for (int l = 0; l < b.levels; l++)
        if (node >= b.level_start[l] && node < b.level_start[l + 1]) return l;
    return -1;
}

}  // namespace

// Returns the number of violations; info = {nodes, levels, width, leaves in ranges}.
extern "C" int64_t bvh_invariants(const mlgpu_flat_scene* f, int64_t* info) {
    BvhHost b;
    mlgpu::build_bvh(f, 0.0, &b);
    info[0] = (int64_t)b.nodes.size();
    info[1] = b.levels;
    info[2] = kBvhWidth;
    info[3] = (int64_t)b.leaf_ids.size();
    int64_t bad = 0;
    // each leaf with geometry in exactly one reachable leaf range
    std::vector<int32_t> seen(f->num_leaves > 0 ? f->num_leaves : 1, 0);
    std::vector<int32_t> all;
    if (!b.nodes.empty()) leaves_under(b, 0, &all);
    for (int32_t l : all) {
        if (l < 0 || l >= f->num_leaves) { bad++; continue; }
        seen[l]++;
    }
    for (int32_t l = 0; l < f->num_leaves; l++) {
        const bool geometry = f->leaf_primitive[l] != MLGPU_PRIM_NONE;
        if (seen[l] != (geometry ? 1 : 0)) bad++;
    }
    if ((int64_t)b.level_start.size() != (int64_t)b.levels + 1) bad++;
    for (size_t n = 0; n < b.nodes.size(); n++) {
        const BvhNode& node = b.nodes[n];
        const int level = level_of(b, (int32_t)n);
        if (level < 0) bad++;
        for (int k = 0; k < kBvhWidth; k++) {
            const int32_t ref = node.child[k];
            if (ref == kBvhEmpty) continue;
            if (!(ref & kBvhLeafFlag) && level_of(b, ref) != level + 1) bad++;
            std::vector<int32_t> under;
            leaves_under(b, ref, &under);
            if (under.empty()) bad++;
            for (int32_t l : under) {
                const double* c = f->node_sphere + 4*(size_t)f->leaf_node[l];
                for (int a = 0; a < 3; a++)
                    if (!((double)node.lo[a][k] <= c[a] - c[3] && (double)node.hi[a][k] >= c[a] + c[3]))
                        bad++;
            }
        }
    }
    return bad;
}
