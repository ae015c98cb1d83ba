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

// ------------------------------------------------------------ tile climb
// build_lbvh (minimum_lbvh.h:284-361) with the hand-offs of a CTA's own nodes
// in shared memory. A CTA holds the leaves [t0, t1] of one tile. The range
// [L, U] of internal node p (split between leaves p and p + 1) follows from
// the split deltas alone: L = 1 + the nearest j < p with delta(j) >= delta(p),
// U = the nearest k > p with delta(k) > delta(p) (deltas outside [0, n - 2]
// count as infinite), which is the range the climb gives p (its parent rule
// goes left exactly when delta(lo - 1) < delta(hi)). A node whose range lies
// in the tile is "interior": both walkers that reach it climb from leaves of
// this CTA, so they meet through a shared-memory hand-off word and a
// shared-memory copy of each child's box, ordered at block scope. Every other
// node (its range crosses a tile boundary; a few per cent of them) takes the
// GPU-scope acquire-release hand-off of climb(). Both walkers of a node
// decide alike, since each decides from the same deltas. The node words
// written are climb()'s.
// leaves per tile = threads per CTA of the tile climb (build-time override for sweeps: -DMLBVH_BUILD_TILE=...)
#ifndef MLBVH_BUILD_TILE
#define MLBVH_BUILD_TILE 64
#endif
constexpr uint32_t kTileLeaves = MLBVH_BUILD_TILE;
struct TileClimbShared {
    uint32_t delta[kTileLeaves + 1];  // delta(t0 - 1 + j), j = 0 .. kTileLeaves
    uint32_t hand[kTileLeaves];       // hand-off word of node t0 + j
    uint32_t interior[kTileLeaves / 32];
    float box[kTileLeaves][2][6];     // child boxes of node t0 + j (index: the child's side)
};

// Stages the tile's deltas, resets its hand-off words and marks its interior
// nodes; every thread of the CTA calls it (it ends with a barrier). keys: the
// sorted Morton keys of all n leaves. Leaves may belong to several trees laid
// end to end (the batched build): [segStart, segEnd) is the range of the tree
// of this thread's leaf t0 + threadIdx.x ([0, n) for a single tree; a thread
// past the last leaf passes segEnd <= its leaf + 1). The delta between the
// last leaf of one tree and the first of the next is staged as infinite, the
// value the climb of each tree gives the deltas outside its own range, so no
// node range crosses a tree boundary. Node p is interior exactly when some
// delta(j), t0 - 1 <= j < p, is >= delta(p) (then L(p) >= t0) and some
// delta(k), p < k <= t1, is > delta(p) (then U(p) <= t1): delta(p) against the
// exclusive prefix and suffix maxima of the tile's deltas, two max-scans of
// the CTA (warp shuffles, then the warps' totals). Needs blockDim.x ==
// kTileLeaves.
__device__ __forceinline__ void tile_climb_prepare(TileClimbShared& sh, const uint32_t* __restrict__ keys, uint32_t n,
                                                   uint32_t t0, uint32_t segStart, uint32_t segEnd)
{
    __shared__ uint32_t s_warpMax[2][kTileLeaves / 32];
    const uint32_t t1 = min(t0 + kTileLeaves - 1, n - 1);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // slot j holds delta(t0 - 1 + j): slot tid + 1 the delta right of this
    // thread's leaf, slot 0 the one left of the tile
    const uint32_t g = t0 + tid;
    sh.delta[tid + 1] = g + 1 < segEnd ? delta_at(keys, g) : 0xFFFFFFFFu;
    if (tid == 0) sh.delta[0] = t0 > segStart ? delta_at(keys, t0 - 1) : 0xFFFFFFFFu;
    sh.hand[tid] = 0xFFFFFFFFu;
    __syncthreads();
    // prefix: max of delta(t0 - 1 .. t0 - 1 + tid), i.e. of the deltas left of node t0 + tid
    uint32_t pre = sh.delta[tid];
    // suffix: max of delta(t0 + tid .. t1)
    uint32_t suf = t0 + tid <= t1 ? sh.delta[tid + 1] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, pre, o);
        const uint32_t b = __shfl_down_sync(0xffffffffu, suf, o);
        if (lane >= (uint32_t)o) pre = max(pre, a);
        if (lane + o < 32) suf = max(suf, b);
    }
    if (lane == 31) s_warpMax[0][warp] = pre;
    if (lane == 0) s_warpMax[1][warp] = suf;
    __syncthreads();
    uint32_t carry = 0u;  // max of the later warps' deltas
    for (uint32_t w = 0; w < warp; ++w) pre = max(pre, s_warpMax[0][w]);
    for (uint32_t w = warp + 1; w < kTileLeaves / 32; ++w) carry = max(carry, s_warpMax[1][w]);
    suf = max(suf, carry);
    // node p = t0 + tid needs the suffix from delta(p + 1): the next thread's (the later warps' for lane 31)
    uint32_t sufNext = __shfl_down_sync(0xffffffffu, suf, 1);
    if (lane == 31) sufNext = carry;
    const uint32_t p = t0 + tid, dp = sh.delta[tid + 1];
    const bool interior = p < t1 && dp <= pre && dp < sufNext;
    const uint32_t mask = __ballot_sync(0xffffffffu, interior);
    if (lane == 0) sh.interior[warp] = mask;
    __syncthreads();
}

// The climb of sorted leaf i (triangle `tri`, box lo/hi) of a tree of n
// leaves, in a tile prepared by tile_climb_prepare. tileBase: the tree's own
// index of the tile's first leaf, modulo 2^32 (t0 for a single tree; below 0,
// wrapped, for a tree that starts inside the tile). sortedKeys, nodes,
// handoff, root: the tree's own arrays. Node words, parent links, root: as
// climb().
__device__ __forceinline__ void climb_tile(TileClimbShared& sh, uint32_t tileBase, uint32_t n, uint32_t i,
                                           uint32_t tri, f3 lo, f3 hi, const uint32_t* __restrict__ sortedKeys,
                                           mlbvh_internal_node* __restrict__ nodes, uint32_t* __restrict__ handoff,
                                           mlbvh_node_index* __restrict__ root, uint8_t* __restrict__ deltas)
{
    const uint32_t nInternals = n - 1;
    // delta(g), 0 <= g < n - 1, from the tile's copy where it holds it (slot
    // g + 1 - tileBase, wrapping large left of the tile), else from the keys
    auto delta_of = [&](uint32_t g) -> uint32_t {
        const uint32_t s = g + 1 - tileBase;
        return s <= kTileLeaves ? sh.delta[s] : delta_at(sortedKeys, g);
    };
    if (deltas && i < nInternals) deltas[i] = (uint8_t)sh.delta[i + 1 - tileBase];

    uint32_t leafLower = i, leafUpper = i;
    uint32_t deltaL = 0 < leafLower ? delta_of(leafLower - 1) : 0xFFFFFFFFu;
    uint32_t deltaR = leafUpper < nInternals ? delta_of(leafUpper) : 0xFFFFFFFFu;
    uint32_t node = tri | kLeafBit;
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

        const uint32_t j = parent - tileBase;  // wraps (large) below the tile
        const bool interior = j < kTileLeaves && ((sh.interior[j >> 5] >> (j & 31)) & 1u);
        const uint32_t mine = goLeft ? leafUpper : leafLower;
        uint32_t other;
        f3 olo, ohi;
        if (interior) {
            float* b = sh.box[j][goLeft];
            b[0] = lo.x; b[1] = lo.y; b[2] = lo.z; b[3] = hi.x; b[4] = hi.y; b[5] = hi.z;
            __threadfence_block();
            other = atomicExch(sh.hand + j, mine);
            if (other == 0xFFFFFFFFu) return;  // first arrival: the sibling finishes this node
            __threadfence_block();
            const float* ob = sh.box[j][1 - goLeft];
            olo = mk(ob[0], ob[1], ob[2]);
            ohi = mk(ob[3], ob[4], ob[5]);
        } else {
            other = exch_acq_rel(handoff + parent, mine);
            if (other == 0xFFFFFFFFu) return;
            if (goLeft) {  // the sibling is child 0
                const float2 a = __ldcg(reinterpret_cast<const float2*>(pw + 2));
                const float4 c = __ldcg(reinterpret_cast<const float4*>(pw + 4));
                olo = mk(a.x, a.y, c.x);
                ohi = mk(c.y, c.z, c.w);
            } else {
                const float4 a = __ldcg(reinterpret_cast<const float4*>(pw + 8));
                const float2 c = __ldcg(reinterpret_cast<const float2*>(pw + 12));
                olo = mk(a.x, a.y, a.z);
                ohi = mk(a.w, c.x, c.y);
            }
        }
        if (other < leafLower) {
            leafLower = other;
            deltaL = 0 < leafLower ? delta_of(leafLower - 1) : 0xFFFFFFFFu;
        } else {
            leafUpper = other;
            deltaR = leafUpper < nInternals ? delta_of(leafUpper) : 0xFFFFFFFFu;
        }
        p->context = leafUpper < nInternals ? leafUpper : 0xFFFFFFFFu;
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
