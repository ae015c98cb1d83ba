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

// A triangle's three corners with three 16-byte loads: the 48-byte window
// from the triangle's address rounded down to 16 bytes holds its 36 bytes;
// the corners are picked out by the triangle's offset in that window. A
// window that would reach past `end` (the last triangles) takes nine scalar
// loads instead, so nothing is read outside the array.
__device__ __forceinline__ void load_triangle_v(const float* __restrict__ t, const float* end, f3& v0, f3& v1,
                                                f3& v2)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(t);
    const uintptr_t a0 = a & ~uintptr_t(15);
    if (a0 + 48 > reinterpret_cast<uintptr_t>(end)) {
        v0 = mk(__ldg(t + 0), __ldg(t + 1), __ldg(t + 2));
        v1 = mk(__ldg(t + 3), __ldg(t + 4), __ldg(t + 5));
        v2 = mk(__ldg(t + 6), __ldg(t + 7), __ldg(t + 8));
        return;
    }
    const float4* q = reinterpret_cast<const float4*>(a0);
    const float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
    const float f[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
    const int off = (int)((a - a0) >> 2);  // 0..3
    float c[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) c[j] = off == 0 ? f[j] : off == 1 ? f[j + 1] : off == 2 ? f[j + 2] : f[j + 3];
    v0 = mk(c[0], c[1], c[2]);
    v1 = mk(c[3], c[4], c[5]);
    v2 = mk(c[6], c[7], c[8]);
}

// The box of a leaf's triangle as build_lbvh forms it (minimum_lbvh.h:300-307):
// the empty box extended by the three corners in order.
__device__ __forceinline__ void leaf_box(const float* __restrict__ tris, uint32_t n, uint32_t tri, f3& lo, f3& hi)
{
    f3 v0, v1, v2;
    load_triangle_v(tris + 9ull * tri, tris + 9ull * n, v0, v1, v2);
    lo = mk(kFltMax, kFltMax, kFltMax);
    hi = mk(-kFltMax, -kFltMax, -kFltMax);
    lo = smin3(lo, v0);
    hi = smax3(hi, v0);
    lo = smin3(lo, v1);
    hi = smax3(hi, v1);
    lo = smin3(lo, v2);
    hi = smax3(hi, v2);
}

// Stages a CTA's leaf boxes for climb's leaf pairs: every thread of the CTA
// calls it (before any of them returns), with valid = false where it has no
// leaf. sBox holds 6 floats per thread.
__device__ __forceinline__ void stage_leaf_box(float* sBox, int t, bool valid, f3 lo, f3 hi)
{
    if (valid) {
        sBox[6 * t + 0] = lo.x;
        sBox[6 * t + 1] = lo.y;
        sBox[6 * t + 2] = lo.z;
        sBox[6 * t + 3] = hi.x;
        sBox[6 * t + 4] = hi.y;
        sBox[6 * t + 5] = hi.z;
    }
    __syncthreads();
}

// build_lbvh (minimum_lbvh.h:284-361) for sorted leaf i of a tree of n
// leaves (triangle `tri`, box lo/hi): climbs from the leaf to the root. The
// hand-off word per internal node lives in its own array (reset before the
// build) and is exchanged with acquire-release semantics, so the first
// walker's child slot is visible to the second; the sibling bounds are then
// read from L2. The merged box is formed as max/min(box of child 1, box of
// child 0) whichever walker arrives second, which is the order the
// reference's serial CPU build produces (its second arrival always comes from
// the right). A child slot is written with two vector stores (children word
// apart), the sibling's box read with two vector loads; of the two key deltas
// at the range's ends only the one at the end that moved is recomputed. The
// node array must be 16-byte aligned.
//
// Leaf pairs: where leaves i and i + 1 both climb to node i (leaf i goes
// right, leaf i + 1 goes left) and their threads t, t + 1 are in one CTA,
// the pair meets without the hand-off word: leaf i writes its slot and stops,
// leaf i + 1 takes leaf i's box from the CTA's staged boxes (sBox, written
// before a barrier) and goes on from node i. Both threads decide this from the
// same key deltas; a pair split across two CTAs uses the hand-off word.
// Nothing else changes: the node words written are the same. A caller that
// passes t = 0 and tLast = -1 (and no sBox) turns leaf pairs off.
__device__ __forceinline__ void climb(uint32_t n, uint32_t i, uint32_t tri, f3 lo, f3 hi,
                                      const uint32_t* __restrict__ sortedKeys,
                                      mlbvh_internal_node* __restrict__ nodes, uint32_t* __restrict__ handoff,
                                      mlbvh_node_index* __restrict__ root, uint8_t* __restrict__ deltas,
                                      const float* sBox, int t, int tLast)
{
    const uint32_t nInternals = n - 1;
    if (deltas && i < nInternals) deltas[i] = (uint8_t)delta_at(sortedKeys, i);

    uint32_t leafLower = i, leafUpper = i;
    uint32_t deltaL = 0 < leafLower ? delta_at(sortedKeys, leafLower - 1) : 0xFFFFFFFFu;
    uint32_t deltaR = leafUpper < nInternals ? delta_at(sortedKeys, leafUpper) : 0xFFFFFFFFu;
    uint32_t node = tri | kLeafBit;
    if (nInternals > 0) {
        if (!(deltaL < deltaR)) {  // parent i, this leaf is child 0
            const uint32_t dR2 = i + 1 < nInternals ? delta_at(sortedKeys, i + 1) : 0xFFFFFFFFu;
            if (deltaR < dR2 && t < tLast) {  // leaf i + 1 goes left to node i too, in this CTA
                mlbvh_internal_node* p = nodes + i;
                float* pw = reinterpret_cast<float*>(p);
                p->children[0] = node;
                *reinterpret_cast<float2*>(pw + 2) = make_float2(lo.x, lo.y);
                *reinterpret_cast<float4*>(pw + 4) = make_float4(lo.z, hi.x, hi.y, hi.z);
                return;
            }
        } else {  // parent i - 1, this leaf is child 1
            const uint32_t dL2 = 1 < i ? delta_at(sortedKeys, i - 2) : 0xFFFFFFFFu;
            if (!(dL2 < deltaL) && t > 0) {  // leaf i - 1 goes right to node i - 1, in this CTA
                const uint32_t parent = i - 1;
                mlbvh_internal_node* p = nodes + parent;
                float* pw = reinterpret_cast<float*>(p);
                p->children[1] = node;
                *reinterpret_cast<float4*>(pw + 8) = make_float4(lo.x, lo.y, lo.z, hi.x);
                *reinterpret_cast<float2*>(pw + 12) = make_float2(hi.y, hi.z);
                const float* ob = sBox + 6 * (t - 1);
                lo = smin3(lo, mk(ob[0], ob[1], ob[2]));
                hi = smax3(hi, mk(ob[3], ob[4], ob[5]));
                leafLower = parent;
                deltaL = dL2;
                p->context = leafUpper < nInternals ? leafUpper : 0xFFFFFFFFu;
                node = parent;
            }
        }
    }
    while (leafUpper - leafLower < nInternals) {
        const int goLeft = deltaL < deltaR ? 1 : 0;
        const uint32_t parent = goLeft ? leafLower - 1 : leafUpper;

        mlbvh_internal_node* p = nodes + parent;
        float* pw = reinterpret_cast<float*>(p);
        p->children[goLeft] = node;
        if (goLeft) {  // aabbs[1]: bytes 32-55
            *reinterpret_cast<float4*>(pw + 8) = make_float4(lo.x, lo.y, lo.z, hi.x);
            *reinterpret_cast<float2*>(pw + 12) = make_float2(hi.y, hi.z);
        } else {  // aabbs[0]: bytes 8-31
            *reinterpret_cast<float2*>(pw + 2) = make_float2(lo.x, lo.y);
            *reinterpret_cast<float4*>(pw + 4) = make_float4(lo.z, hi.x, hi.y, hi.z);
        }
        if (!(node & kLeafBit)) nodes[node].parent = parent;

        const uint32_t other = exch_acq_rel(handoff + parent, goLeft ? leafUpper : leafLower);
        if (other == 0xFFFFFFFFu) return;  // first arrival: the sibling finishes this node

        if (other < leafLower) {
            leafLower = other;
            deltaL = 0 < leafLower ? delta_at(sortedKeys, leafLower - 1) : 0xFFFFFFFFu;
        } else {
            leafUpper = other;
            deltaR = leafUpper < nInternals ? delta_at(sortedKeys, leafUpper) : 0xFFFFFFFFu;
        }
        p->context = leafUpper < nInternals ? leafUpper : 0xFFFFFFFFu;
        f3 olo, ohi;
        if (goLeft) {  // the sibling is child 0
            const float2 a = __ldcg(reinterpret_cast<const float2*>(pw + 2));
            const float4 b = __ldcg(reinterpret_cast<const float4*>(pw + 4));
            olo = mk(a.x, a.y, b.x);
            ohi = mk(b.y, b.z, b.w);
        } else {
            const float4 a = __ldcg(reinterpret_cast<const float4*>(pw + 8));
            const float2 b = __ldcg(reinterpret_cast<const float2*>(pw + 12));
            olo = mk(a.x, a.y, a.z);
            ohi = mk(a.w, b.x, b.y);
        }
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
