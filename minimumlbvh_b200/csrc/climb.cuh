// The agglomerative bottom-up build of one tree (build_lbvh,
// minimum_lbvh.h:284-361), shared by the single-mesh and the batched builds.
#pragma once

#include <cstdint>

#include "../../include/mlbvh.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {

__device__ __forceinline__ uint32_t exch_acq_rel(uint32_t* p, uint32_t v)
{
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ uint32_t delta_at(const uint32_t* __restrict__ keys, uint32_t i)
{
    return split_delta(keys[i], keys[i + 1]);
}

// build_lbvh (minimum_lbvh.h:284-361) for sorted leaf i of a tree of n
// leaves: climbs from the leaf to the root. The hand-off word per internal
// node lives in its own array (reset before the build) and is exchanged with
// acquire-release semantics, so the first walker's child slot is visible to
// the second; the sibling bounds are then read from L2. The merged box is
// formed as max/min(box of child 1, box of child 0) whichever walker arrives
// second, which is the order the reference's serial CPU build produces (its
// second arrival always comes from the right).
__device__ __forceinline__ void climb(const float* __restrict__ tris, uint32_t n, uint32_t i,
                                      const uint32_t* __restrict__ sortedKeys, const uint32_t* __restrict__ sortedIdx,
                                      mlbvh_internal_node* __restrict__ nodes, uint32_t* __restrict__ handoff,
                                      mlbvh_node_index* __restrict__ root, uint8_t* __restrict__ deltas)
{
    const uint32_t nInternals = n - 1;
    const uint32_t tri = sortedIdx[i];
    if (tri >= n) return;  // only after a sort whose bounded wait gave up (error word set)
    if (deltas && i < nInternals) deltas[i] = (uint8_t)delta_at(sortedKeys, i);

    f3 v0, v1, v2;
    load_triangle(tris, tri, v0, v1, v2);
    f3 lo = mk(kFltMax, kFltMax, kFltMax), hi = mk(-kFltMax, -kFltMax, -kFltMax);
    lo = smin3(lo, v0);
    hi = smax3(hi, v0);
    lo = smin3(lo, v1);
    hi = smax3(hi, v1);
    lo = smin3(lo, v2);
    hi = smax3(hi, v2);

    uint32_t leafLower = i, leafUpper = i;
    uint32_t node = tri | kLeafBit;
    while (leafUpper - leafLower < nInternals) {
        const uint32_t deltaL = 0 < leafLower ? delta_at(sortedKeys, leafLower - 1) : 0xFFFFFFFFu;
        const uint32_t deltaR = leafUpper < nInternals ? delta_at(sortedKeys, leafUpper) : 0xFFFFFFFFu;
        const int goLeft = deltaL < deltaR ? 1 : 0;
        const uint32_t parent = goLeft ? leafLower - 1 : leafUpper;

        mlbvh_internal_node* p = nodes + parent;
        p->children[goLeft] = node;
        float* box = p->aabbs[goLeft].lower;
        box[0] = lo.x;
        box[1] = lo.y;
        box[2] = lo.z;
        box[3] = hi.x;
        box[4] = hi.y;
        box[5] = hi.z;
        if (!(node & kLeafBit)) nodes[node].parent = parent;

        uint32_t other = exch_acq_rel(handoff + parent, goLeft ? leafUpper : leafLower);
        if (other == 0xFFFFFFFFu) return;  // first arrival: the sibling finishes this node

        leafLower = min(leafLower, other);
        leafUpper = max(leafUpper, other);
        p->context = leafUpper < nInternals ? leafUpper : 0xFFFFFFFFu;
        const float* ob = p->aabbs[goLeft ^ 1].lower;
        const f3 olo = mk(__ldcg(ob + 0), __ldcg(ob + 1), __ldcg(ob + 2));
        const f3 ohi = mk(__ldcg(ob + 3), __ldcg(ob + 4), __ldcg(ob + 5));
        if (goLeft) {  // this walker is child 1
            lo = smin3(lo, olo);
            hi = smax3(hi, ohi);
        } else {
            lo = smin3(olo, lo);
            hi = smax3(ohi, hi);
        }
        node = parent;
    }
    *root = node;
    if (!(node & kLeafBit)) nodes[node].parent = kInvalid;
}

}  // namespace mlbvh
