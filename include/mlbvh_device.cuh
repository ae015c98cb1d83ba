// Shared device code of minimumlbvh_b200: vector arithmetic with the exact
// rounding of the reference's host build, Morton coding, the stack-free
// traversal and the sample streams.
//
// Bit-exactness with the reference's CPU path (minimum_lbvh.h compiled for
// the host) rests on three rules, applied to every kernel in this library:
//   * the library is compiled with -fmad=false, so each written * and + rounds
//     on its own, in source order, as the host does under -ffp-contract=off;
//   * division and sqrtf are IEEE round-to-nearest (no fast-math), and
//     normalize is v * (1 / sqrtf(dot(v, v))), the host rsqrtf
//     (helper_math.h:154-157);
//   * fminf/fmaxf on the host are selects, `a < b ? a : b` (helper_math.h:
//     134-142); where the operand order can show (AABB merges that may see
//     +0 and -0) the same selects are used here.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mlbvh.h"


namespace mlbvh {

constexpr float kFltMax = 3.402823466e+38F;  // minimum_lbvh.h:37
constexpr uint32_t kMortonMax = 0x1FFFFF;   // minimum_lbvh.h:38
constexpr uint32_t kInvalid = 0x7FFFFFFFu;  // NodeIndex::invalid()
constexpr uint32_t kLeafBit = 0x80000000u;
// Upper bound on traversal steps per ray. A valid tree of n leaves needs at
// most 4n steps (each internal node entered from above and from both
// children, each leaf once); the bound only matters for a corrupt tree, where
// it turns an endless walk into a wrong answer.
constexpr uint32_t kMaxTraversalSteps = 1u << 26;

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ f3 operator/(f3 a, f3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }

// Host-build fminf/fmaxf (helper_math.h:134-142).
__device__ __forceinline__ float smin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float smax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ f3 smin3(f3 a, f3 b) { return mk(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
__device__ __forceinline__ f3 smax3(f3 a, f3 b) { return mk(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }

__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ f3 normalize(f3 v)
{
    float invLen = 1.0f / sqrtf(dot(v, v));
    return v * invLen;
}
__device__ __forceinline__ f3 lerp(f3 a, f3 b, float t) { return a + t * (b - a); }
__device__ __forceinline__ float clampf(float f, float a, float b) { return smax(a, smin(f, b)); }
__device__ __forceinline__ int clampi(int f, int a, int b)
{
    int m = f < b ? f : b;
    return a > m ? a : m;
}
// float -> int as the reference's x86 host build converts (cvttss2si):
// truncation; NaN and out-of-range values give 0x80000000.
__device__ __forceinline__ int f2i_host(float x)
{
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return (int)0x80000000u;
    return __float2int_rz(x);
}

// ---------------------------------------------------------------- Morton
// splat3 (minimum_lbvh.h:173-182): low 21 bits of a, three apart.
__device__ __forceinline__ uint64_t splat3(uint32_t a)
{
    uint64_t x = a & 0x1fffffu;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
// AABB::encodeMortonCode (minimum_lbvh.h:246-251) then the top 32 of the 63
// bits (minimum_lbvh.cu:89).
__device__ __forceinline__ uint32_t morton32(f3 lower, f3 upper, f3 p)
{
    f3 q = (p - lower) / (upper - lower) * (float)(kMortonMax + 1);
    uint32_t cx = (uint32_t)clampi(f2i_host(q.x), 0, kMortonMax);
    uint32_t cy = (uint32_t)clampi(f2i_host(q.y), 0, kMortonMax);
    uint32_t cz = (uint32_t)clampi(f2i_host(q.z), 0, kMortonMax);
    uint64_t m = splat3(cx) | splat3(cy) << 1 | splat3(cz) << 2;
    return (uint32_t)(m >> 31);
}
// delta (minimum_lbvh.h:140-143)
__device__ __forceinline__ uint32_t split_delta(uint32_t a, uint32_t b) { return 32u - __clz(a ^ b); }

// ------------------------------------------------------------- geometry
__device__ __forceinline__ float4 ldg4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// A triangle (36 B, 4-byte aligned) as three points, read-only path.
__device__ __forceinline__ void load_triangle(const float* __restrict__ tris, uint32_t i, f3& v0, f3& v1, f3& v2)
{
    const float* t = tris + 9ull * i;
    v0 = mk(__ldg(t + 0), __ldg(t + 1), __ldg(t + 2));
    v1 = mk(__ldg(t + 3), __ldg(t + 4), __ldg(t + 5));
    v2 = mk(__ldg(t + 6), __ldg(t + 7), __ldg(t + 8));
}

// intersectRayTriangle (minimum_lbvh.h:363-413): plane distance, inclusive
// [t_min, t_max] test, then the three edge volumes (a-b)x(a+b) whose signs
// must agree (edge-watertight), barycentrics from the volumes.
__device__ __forceinline__ bool intersect_triangle(float& tOut, float& uOut, float& vOut, f3& ngOut, float t_min,
                                                   float t_max, f3 ro, f3 rd, f3 v0, f3 v1, f3 v2)
{
    f3 e0 = v1 - v0;
    f3 e1 = v2 - v1;
    f3 ng = cross(e0, e1);
    float t = dot(v0 - ro, ng) / dot(ng, rd);
    if (t_min <= t && t <= t_max) {
        f3 e2 = v0 - v2;
        f3 ro2 = ro * 2.0f;
        float u_vol = dot(cross(e2, (v0 + v2) - ro2), rd);
        float v_vol = dot(cross(e0, (v1 + v0) - ro2), rd);
        float w_vol = dot(cross(e1, (v2 + v1) - ro2), rd);
        if (fminf(fminf(u_vol, v_vol), w_vol) < 0.0f && 0.0f < fmaxf(fmaxf(u_vol, v_vol), w_vol)) return false;
        float vol = u_vol + v_vol + w_vol;
        tOut = t;
        uOut = u_vol / vol;
        vOut = v_vol / vol;
        ngOut = ng;
        return true;
    }
    return false;
}

// invRd (minimum_lbvh.h:898-901)
__device__ __forceinline__ f3 inv_rd(f3 rd)
{
    return mk(clampf(1.0f / rd.x, -kFltMax, kFltMax), clampf(1.0f / rd.y, -kFltMax, kFltMax),
              clampf(1.0f / rd.z, -kFltMax, kFltMax));
}

// slabs (minimum_lbvh.h:82-96) for one box given as (lower, upper); the
// entry is clipped to tmin (0 in the reference) and the exit, inflated by
// 1.00000024, to knownHitT. Only the sign of a zero can differ between
// fminf/fmaxf and the host selects here, and no comparison below sees it.
// slab_offsets takes the planes already relative to the ray origin (lo - ro,
// hi - ro); slab is slab_offsets(lo - ro, hi - ro, ...), the same operations.
__device__ __forceinline__ float2 slab_offsets(f3 dlo, f3 dhi, f3 inv, float tmin, float knownHitT)
{
    f3 t0 = dlo * inv;
    f3 t1 = dhi * inv;
    float rmin = fmaxf(fmaxf(fminf(t0.x, t1.x), fminf(t0.y, t1.y)), fminf(t0.z, t1.z));
    float rmax = fminf(fminf(fmaxf(t0.x, t1.x), fmaxf(t0.y, t1.y)), fmaxf(t0.z, t1.z)) * 1.00000024f;
    rmin = fmaxf(rmin, 0.0f);
    rmin = fmaxf(rmin, tmin);
    rmax = fminf(rmax, knownHitT);
    return make_float2(rmin, rmax);
}
__device__ __forceinline__ float2 slab(f3 ro, f3 inv, f3 lo, f3 hi, float tmin, float knownHitT)
{
    return slab_offsets(lo - ro, hi - ro, inv, tmin, knownHitT);
}

struct HitRecord {
    float t;
    float u, v;
    f3 ng;
    uint32_t tri;
};

// One internal node as the traversal needs it: 4 x 16-byte read-only loads of
// the 64-byte InternalNode.
struct NodeView {
    uint32_t c0, c1, parent, context;
    f3 lo0, hi0, lo1, hi1;
};
// 32 bytes through the read-only path in one instruction (ld.global.nc.v8,
// sm_100 and later); p must be 32-byte aligned.
__device__ __forceinline__ void ldg32(const void* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// kWide: two 32-byte loads (the node array must be 32-byte aligned, as the
// library's entry points check); otherwise four 16-byte loads.
template <bool kWide = false>
__device__ __forceinline__ NodeView load_node(const mlbvh_internal_node* __restrict__ nodes, uint32_t i)
{
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    float4 a, b, c, d;
    if (kWide) {
        ldg32(p, a, b);
        ldg32(p + 2, c, d);
    } else {
        a = __ldg(p + 0);
        b = __ldg(p + 1);
        c = __ldg(p + 2);
        d = __ldg(p + 3);
    }
    NodeView n;
    n.c0 = __float_as_uint(a.x);
    n.c1 = __float_as_uint(a.y);
    n.lo0 = mk(a.z, a.w, b.x);
    n.hi0 = mk(b.y, b.z, b.w);
    n.lo1 = mk(c.x, c.y, c.z);
    n.hi1 = mk(c.w, d.x, d.y);
    n.parent = __float_as_uint(d.z);
    n.context = __float_as_uint(d.w);
    return n;
}

// intersect_stackfree (minimum_lbvh.h:981-1061). Parent-pointer traversal:
// from the parent go to the nearer hit child (entry distance, ties to the
// left child) or back up; from the near child go to the far child when both
// boxes are still hit, else up; from the far child go up. Both child boxes
// are re-tested on every visit against the current closest t.
//
// stackfree_step advances the walk (curr, prev) by one leaf test or one
// internal-node visit and returns true when the walk is over. With kCount,
// nv and nt count internal-node visits and triangle tests (the traffic
// model of the roofline). kWide selects 32-byte node loads (see load_node).
template <bool kAny, bool kCount, bool kWide = false>
__device__ __forceinline__ bool stackfree_step(uint32_t& curr, uint32_t& prev, HitRecord& hit,
                                               const mlbvh_internal_node* __restrict__ nodes,
                                               const float* __restrict__ tris, f3 ro, f3 rd, f3 inv, float tmin,
                                               uint32_t& nv, uint32_t& nt)
{
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const uint32_t ti = curr & ~kLeafBit;
        f3 v0, v1, v2;
        load_triangle(tris, ti, v0, v1, v2);
        float t, u, v;
        f3 ng;
        if (intersect_triangle(t, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2)) {
            hit.t = t;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = ti;
            if (kAny) return true;
        }
        const uint32_t s = curr;
        curr = prev;
        prev = s;
        return curr == kInvalid;
    }
    if (kCount) ++nv;
    const NodeView nd = load_node<kWide>(nodes, curr);
    const float2 rl = slab(ro, inv, nd.lo0, nd.hi0, tmin, hit.t);
    const float2 rr = slab(ro, inv, nd.lo1, nd.hi1, tmin, hit.t);
    const bool hitL = rl.x <= rl.y;
    const bool hitR = rr.x <= rr.y;
    uint32_t nearN = nd.c0, farN = nd.c1;
    int nHits = 0;
    if (hitL && hitR) {
        if (rr.x < rl.x) {
            nearN = nd.c1;
            farN = nd.c0;
        }
        nHits = 2;
    } else if (hitL || hitR) {
        nHits = 1;
        nearN = hitR ? farN : nearN;
    }
    uint32_t next;
    if (prev == nd.parent)
        next = 0 < nHits ? nearN : nd.parent;
    else if (prev == nearN)
        next = nHits == 2 ? farN : nd.parent;
    else
        next = nd.parent;
    prev = curr;
    curr = next;
    return curr == kInvalid;
}

// Stack entries of the replay walks. A closest-hit walk keeps the pending far
// child and its entry distance; an any-hit walk keeps the child alone: its
// hit.t does not change before the first hit, which ends the walk, so every
// pending child still passes the entry test when it is popped.
template <bool kAny>
struct ReplayStack {
    using Entry = uint2;
};
template <>
struct ReplayStack<true> {
    using Entry = uint32_t;
};

// intersect_stackfree's leaf order and hit.t updates without its revisits
// (the replay walk). Where both child boxes are hit, the far child and its
// entry distance are pushed and the near child is entered; when a subtree is
// done, entries are popped and an entry is entered iff its entry distance is
// still <= hit.t. That is exactly when the stack-free walk, back at the parent
// from the near child, finds both boxes still hit: a box's entry distance does
// not depend on hit.t, and the near entry never exceeds the far one. So the
// same leaves are tested in the same order against the same hit.t, and the
// Hit record is the stack-free walk's bit for bit, ties included, while every
// internal node is loaded once instead of up to three times.
//
// The stack holds kDepth entries of this thread at stack[d * stride]
// (shared memory, one column per thread). A push onto a full stack hands the
// walk to stackfree_step at (near child, this node), marked by depth = -1;
// climbing through the parent links, it re-derives every entry still on the
// stack. Start a walk with curr = root, depth = 0.
template <bool kAny, bool kCount, int kDepth>
__device__ __forceinline__ bool stackfree_replay_step(uint32_t& curr, uint32_t& prev, int& depth,
                                                      typename ReplayStack<kAny>::Entry* stack,
                                                      int stride, HitRecord& hit,
                                                      const mlbvh_internal_node* __restrict__ nodes,
                                                      const float* __restrict__ tris, f3 ro, f3 rd, f3 inv, float tmin,
                                                      uint32_t& nv, uint32_t& nt)
{
    if (depth < 0) return stackfree_step<kAny, kCount, true>(curr, prev, hit, nodes, tris, ro, rd, inv, tmin, nv, nt);
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const uint32_t ti = curr & ~kLeafBit;
        f3 v0, v1, v2;
        load_triangle(tris, ti, v0, v1, v2);
        float t, u, v;
        f3 ng;
        if (intersect_triangle(t, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2)) {
            hit.t = t;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = ti;
            if (kAny) return true;
        }
    } else {
        if (kCount) ++nv;
        const NodeView nd = load_node<true>(nodes, curr);
        const float2 rl = slab(ro, inv, nd.lo0, nd.hi0, tmin, hit.t);
        const float2 rr = slab(ro, inv, nd.lo1, nd.hi1, tmin, hit.t);
        const bool hitL = rl.x <= rl.y, hitR = rr.x <= rr.y;
        if (hitL && hitR) {
            const bool swap = rr.x < rl.x;
            const uint32_t nearN = swap ? nd.c1 : nd.c0, farN = swap ? nd.c0 : nd.c1;
            if (depth == kDepth) {  // full: continue as the stack-free walk
                depth = -1;
                prev = curr;
                curr = nearN;
                return false;
            }
            if constexpr (kAny)
                stack[depth * stride] = farN;
            else
                stack[depth * stride] = make_uint2(farN, __float_as_uint(swap ? rl.x : rr.x));
            ++depth;
            curr = nearN;
            return false;
        }
        if (hitL || hitR) {
            curr = hitL ? nd.c0 : nd.c1;
            return false;
        }
    }
    if constexpr (kAny) {
        if (depth == 0) return true;
        curr = stack[--depth * stride];
        return false;
    } else {
        while (depth > 0) {
            const uint2 e = stack[--depth * stride];
            if (__uint_as_float(e.y) <= hit.t) {
                curr = e.x;
                return false;
            }
        }
        return true;
    }
}

// The replay walk over leaf-ordered triangles: mlbvh_qtri records (48 bytes,
// 16-byte aligned, corners + original index) in sorted leaf order. A leaf
// child of internal node j is leaf j (left child) or leaf j + 1 (right child),
// so the walk names a leaf by its position (kLeafBit | position) and reads its
// triangle with three 16-byte loads; the Hit record reports the original
// index stored in the record. Same leaves, same order, same Hit records as
// stackfree_replay_step. After a stack overflow the stack-free walk continues
// over the original leaf names and the reference triangle array `tris`.
template <bool kAny, bool kCount, int kDepth>
__device__ __forceinline__ bool stackfree_replay_step_lo(uint32_t& curr, uint32_t& prev, int& depth,
                                                         typename ReplayStack<kAny>::Entry* stack, int stride,
                                                         HitRecord& hit, const mlbvh_internal_node* __restrict__ nodes,
                                                         const float* __restrict__ tris,
                                                         const mlbvh_qtri* __restrict__ leafTris, f3 ro, f3 rd,
                                                         f3 inv, float tmin, uint32_t& nv, uint32_t& nt)
{
    if (depth < 0) return stackfree_step<kAny, kCount, true>(curr, prev, hit, nodes, tris, ro, rd, inv, tmin, nv, nt);
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const float4* t = reinterpret_cast<const float4*>(leafTris + (curr & ~kLeafBit));
        const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        float tt, u, v;
        f3 ng;
        if (intersect_triangle(tt, u, v, ng, tmin, hit.t, ro, rd, mk(a.x, a.y, a.z), mk(a.w, b.x, b.y),
                               mk(b.z, b.w, c.x))) {
            hit.t = tt;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = __float_as_uint(c.y);
            if (kAny) return true;
        }
    } else {
        if (kCount) ++nv;
        const NodeView nd = load_node<true>(nodes, curr);
        const float2 rl = slab(ro, inv, nd.lo0, nd.hi0, tmin, hit.t);
        const float2 rr = slab(ro, inv, nd.lo1, nd.hi1, tmin, hit.t);
        const bool hitL = rl.x <= rl.y, hitR = rr.x <= rr.y;
        const uint32_t e0 = (nd.c0 & kLeafBit) ? (kLeafBit | curr) : nd.c0;
        const uint32_t e1 = (nd.c1 & kLeafBit) ? (kLeafBit | (curr + 1)) : nd.c1;
        if (hitL && hitR) {
            const bool swap = rr.x < rl.x;
            if (depth == kDepth) {  // full: continue as the stack-free walk, over the original leaf names
                depth = -1;
                prev = curr;
                curr = swap ? nd.c1 : nd.c0;
                return false;
            }
            if constexpr (kAny)
                stack[depth * stride] = swap ? e0 : e1;
            else
                stack[depth * stride] = make_uint2(swap ? e0 : e1, __float_as_uint(swap ? rl.x : rr.x));
            ++depth;
            curr = swap ? e1 : e0;
            return false;
        }
        if (hitL || hitR) {
            curr = hitL ? e0 : e1;
            return false;
        }
    }
    if constexpr (kAny) {
        if (depth == 0) return true;
        curr = stack[--depth * stride];
        return false;
    } else {
        while (depth > 0) {
            const uint2 e = stack[--depth * stride];
            if (__uint_as_float(e.y) <= hit.t) {
                curr = e.x;
                return false;
            }
        }
        return true;
    }
}

template <bool kAny, bool kCount = false, bool kWide = false>
__device__ __forceinline__ void trace_stackfree(HitRecord& hit, const mlbvh_internal_node* __restrict__ nodes,
                                                const float* __restrict__ tris, uint32_t root, f3 ro, f3 rd,
                                                f3 inv, float tmin, uint32_t* visits = nullptr,
                                                uint32_t* tests = nullptr)
{
    uint32_t curr = root, prev = kInvalid, nv = 0, nt = 0;
    for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
        if (stackfree_step<kAny, kCount, kWide>(curr, prev, hit, nodes, tris, ro, rd, inv, tmin, nv, nt)) break;
    if (kCount) {
        *visits += nv;
        *tests += nt;
    }
}

// intersect_escape_link (minimum_lbvh.h:1063-1137): after a left child the
// walk moves to the right child through the parent; after a right child it
// follows the rope in `context` (the node whose left subtree starts the next
// leaf range). A one-leaf tree is tested directly (the reference would read
// nodes[invalid] there).
template <bool kAny>
__device__ __forceinline__ void trace_escape(HitRecord& hit, const mlbvh_internal_node* __restrict__ nodes,
                                             const float* __restrict__ tris, uint32_t root, f3 ro, f3 rd, f3 inv,
                                             float tmin)
{
    auto leaf = [&](uint32_t n) -> bool {
        uint32_t ti = n & ~kLeafBit;
        f3 v0, v1, v2;
        load_triangle(tris, ti, v0, v1, v2);
        float t, u, v;
        f3 ng;
        if (intersect_triangle(t, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2)) {
            hit.t = t;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = ti;
            return true;
        }
        return false;
    };
    if (root & kLeafBit) {
        leaf(root);
        return;
    }
    uint32_t curr = root, prev = kInvalid, steps = 0;
    while (curr != kInvalid && ++steps < kMaxTraversalSteps) {
        if (curr & kLeafBit) {
            if (leaf(curr) && kAny) break;
            const NodeView pn = load_node(nodes, prev & ~kLeafBit);
            if (pn.c0 == curr) {
                uint32_t s = curr;
                curr = prev;
                prev = s;
                continue;
            }
            uint32_t next = pn.context != 0xFFFFFFFFu ? pn.context : kInvalid;
            prev = curr;
            curr = next;
            continue;
        }
        const NodeView nd = load_node(nodes, curr);
        f3 lo, hi;
        uint32_t hitChild, miss;
        if (prev == nd.parent) {
            lo = nd.lo0;
            hi = nd.hi0;
            hitChild = nd.c0;
            miss = curr;
        } else {
            lo = nd.lo1;
            hi = nd.hi1;
            hitChild = nd.c1;
            miss = nd.context != 0xFFFFFFFFu ? nd.context : kInvalid;
        }
        float2 r = slab(ro, inv, lo, hi, tmin, hit.t);
        uint32_t next = r.x <= r.y ? hitChild : miss;
        prev = curr;
        curr = next;
    }
}

// intersect_stackfull (minimum_lbvh.h:912-973): explicit stack of far
// children (capacity entries; a push beyond it is dropped); closest hit only,
// as in the reference.
__device__ __forceinline__ void trace_stackfull(HitRecord& hit, const mlbvh_internal_node* __restrict__ nodes,
                                                const float* __restrict__ tris, uint32_t root, f3 ro, f3 rd, f3 inv,
                                                float tmin, uint32_t* stack, int capacity)
{
    int sp = 0;
    uint32_t node = root, steps = 0;
    while (node != kInvalid && ++steps < kMaxTraversalSteps) {
        if (node & kLeafBit) {
            uint32_t ti = node & ~kLeafBit;
            f3 v0, v1, v2;
            load_triangle(tris, ti, v0, v1, v2);
            float t, u, v;
            f3 ng;
            if (intersect_triangle(t, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2)) {
                hit.t = t;
                hit.u = u;
                hit.v = v;
                hit.ng = ng;
                hit.tri = ti;
            }
            node = sp == 0 ? kInvalid : stack[--sp];
            continue;
        }
        const NodeView nd = load_node(nodes, node);
        float2 rl = slab(ro, inv, nd.lo0, nd.hi0, tmin, hit.t);
        float2 rr = slab(ro, inv, nd.lo1, nd.hi1, tmin, hit.t);
        bool hitL = rl.x <= rl.y, hitR = rr.x <= rr.y;
        if (hitL && hitR) {
            uint32_t nearN = nd.c0, farN = nd.c1;
            if (rr.x < rl.x) {
                nearN = nd.c1;
                farN = nd.c0;
            }
            node = nearN;
            if (sp < capacity) stack[sp++] = farN;
        } else if (hitL || hitR) {
            node = hitL ? nd.c0 : nd.c1;
        } else {
            node = sp == 0 ? kInvalid : stack[--sp];
        }
    }
}

// ------------------------------------------------------------ samples
// sobol.h:31-39 (Laine-Karras style hash permutation, Burley 2020)
__device__ __forceinline__ uint32_t lk_permutation(uint32_t x, uint32_t seed)
{
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
__device__ __forceinline__ uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed)
{
    return __brev(lk_permutation(__brev(x), seed));
}
// Sobol's second dimension as a Pascal-matrix product (sobol.h:51-59)
__device__ __forceinline__ uint32_t pascal(uint32_t v)
{
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    return v;
}
__device__ __forceinline__ float random_float(uint32_t u)
{
    return (float)(u >> 8) / (float)((0xFFFFFFFFu >> 8) + 1);
}
__device__ __forceinline__ uint32_t hash_pcg(uint32_t v)  // sobol.h:76-81
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
__device__ __forceinline__ void pcg3d(uint32_t& x, uint32_t& y, uint32_t& z)  // sobol.h:83-107
{
    uint32_t vx = x * 1664525u + 1013904223u;
    uint32_t vy = y * 1664525u + 1013904223u;
    uint32_t vz = z * 1664525u + 1013904223u;
    vx += vy * vz;
    vy += vz * vx;
    vz += vx * vy;
    vx ^= vx >> 16;
    vy ^= vy >> 16;
    vz ^= vz >> 16;
    vx += vy * vz;
    vy += vz * vx;
    vz += vx * vy;
    x = vx;
    y = vy;
    z = vz;
}
// shuffled_scrambled_sobol_2d (sobol.h:119-129)
__device__ __forceinline__ float2 sobol2d(uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2)
{
    pcg3d(p0, p1, p2);
    uint32_t v = lk_permutation(__brev(index), p0);
    return make_float2(random_float(nested_uniform_scramble(v, p1)),
                       random_float(nested_uniform_scramble(pascal(v), p2)));
}

// PCG32 (main_gpu.cu:51-82)
struct Pcg {
    uint64_t state, inc;
    __device__ __forceinline__ Pcg(uint64_t seed, uint64_t seq)
    {
        state = 0;
        inc = (seq << 1u) | 1u;
        next();
        state += seed;
        next();
    }
    __device__ __forceinline__ uint32_t next()
    {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
    }
    __device__ __forceinline__ float uniformf() { return __uint_as_float((next() >> 9) | 0x3f800000u) - 1.0f; }
};

// FP32 sin and cos of phi in [0, 2*pi]: Cody-Waite reduction by pi/2 (split
// in three float parts), then the Taylor polynomials of sin (to r^9) and cos
// (to r^10) on [-pi/4, pi/4], all in fused multiply-adds. The same formula is
// evaluated on the host by the oracle, so sample directions agree bit for bit;
// its error is within 2 ulp of the true values over the sample range.
__device__ __forceinline__ void sincos_portable(float phi, float& s, float& c)
{
    const float kPio2Hi = 1.57079637050628662109375f;
    const float kPio2Mid = -4.371138828673792886547744274139404296875e-8f;
    const float kPio2Lo = -1.71512451000588187280393448475e-15f;
    float k = rintf(phi * 0.636619772367581343f);
    float r = fmaf(-k, kPio2Hi, phi);
    r = fmaf(-k, kPio2Mid, r);
    r = fmaf(-k, kPio2Lo, r);
    float r2 = r * r;
    float ps = fmaf(r2, (float)(1.0 / 362880.0), (float)(-1.0 / 5040.0));
    ps = fmaf(ps, r2, (float)(1.0 / 120.0));
    ps = fmaf(ps, r2, (float)(-1.0 / 6.0));
    float sr = fmaf(ps * r2, r, r);
    float pc = fmaf(r2, (float)(-1.0 / 3628800.0), (float)(1.0 / 40320.0));
    pc = fmaf(pc, r2, (float)(-1.0 / 720.0));
    pc = fmaf(pc, r2, (float)(1.0 / 24.0));
    pc = fmaf(pc, r2, -0.5f);
    float cr = fmaf(pc, r2, 1.0f);
    int q = ((int)k) & 3;
    if (q == 0) {
        s = sr;
        c = cr;
    } else if (q == 1) {
        s = cr;
        c = -sr;
    } else if (q == 2) {
        s = -sr;
        c = -cr;
    } else {
        s = -cr;
        c = sr;
    }
}

constexpr float kPi = 3.14159265358979323846f;

// sampleHemisphereCosWeighted (main_gpu.cu:24-36) with the portable sincos.
__device__ __forceinline__ f3 sample_hemisphere(float xi0, float xi1)
{
    float phi = xi0 * 2.0f * kPi;
    float r = sqrtf(xi1);
    float sp, cp;
    sincos_portable(phi, sp, cp);
    float x = cp * r;
    float z = sp * r;
    float y = sqrtf(fmaxf(1.0f - r * r, 0.0f));
    return mk(x, y, z);
}

// GetOrthonormalBasis (main_gpu.cu:39-45; Duff et al. 2017)
__device__ __forceinline__ void onb(f3 z, f3& xaxis, f3& yaxis)
{
    const float sign = copysignf(1.0f, z.z);
    const float a = -1.0f / (sign + z.z);
    const float b = z.x * z.y * a;
    xaxis = mk(1.0f + sign * z.x * z.x * a, sign * b, -sign * z.x);
    yaxis = mk(b, sign + z.y * z.y * a, -z.y);
}

// packRGBA (main_gpu.cu:17-22): alpha is not stored.
__device__ __forceinline__ uint32_t pack_rgba(float r, float g, float b)
{
    int x = clampi(f2i_host(r * 255.0f + 0.5f), 0, 255);
    int y = clampi(f2i_host(g * 255.0f + 0.5f), 0, 255);
    int z = clampi(f2i_host(b * 255.0f + 0.5f), 0, 255);
    return ((uint32_t)z << 16) | ((uint32_t)y << 8) | (uint32_t)x;
}

struct Camera {
    f3 origin, right, up;
};
// RayGenerator::shoot (camera.h:24-31)
__device__ __forceinline__ void shoot(const Camera& cam, float u, float v, f3& ro, f3& rd)
{
    f3 from = cam.origin;
    f3 forward = normalize(cross(cam.up, cam.right));
    f3 to = cam.origin + forward + lerp(-cam.right, cam.right, u) + lerp(cam.up, -cam.up, v);
    ro = from;
    rd = to - from;
}

// ------------------------------------------------------------ quantised tree
// 32-byte nodes with 8-bit child boxes (see mlbvh_qnode in mlbvh.h). Boxes
// are decoded with directed rounding (lower corners down, upper corners up),
// so every decoded box contains the FP32 box it came from and the traversal
// visits every leaf the FP32 traversal would need.
constexpr uint32_t kQIndexMask = 0x7FFFFFu;  // 23-bit index / leaf position
constexpr uint32_t kQMaxLeaves = 1u << 23;

__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }  // e in [-126, 127]

// Plane code q under scale 2^E stands for V = 2^E (1 + q / 2^15): one byte
// permute writes q (byte k of `codes`) into mantissa byte 1 of the bits of
// 2^E, which gives V exactly. A plane is base + V. Used by the quantised
// binary nodes and the quantised 4-wide slots alike.
__device__ __forceinline__ float qw_value(uint32_t codes, uint32_t scaleBits, int k)
{
    return __uint_as_float(__byte_perm(codes, scaleBits, 0x7604u | ((uint32_t)k << 4)));
}
// The quantisers keep every base below 2^60 and every scale at most 2^59
// (else the tree's status word sends its rays to a walk without the FMA
// form), so every plane lies below 2^61. A ray whose |inv| and |ro|
// components are below 2^62 then keeps every term of the FMA form (V inv + C,
// C = base inv - ro inv) below 2^125, in the float range (qwide_ray_fits,
// tested once per ray). Other rays (in practice those with a zero direction
// component, whose inverse the reference clamps to +-FLT_MAX) take a walk
// without it.
constexpr float kQBaseLimit = 1.152921504606846976e18f;  // 2^60
constexpr float kQRayLimit = 4.611686018427387904e18f;   // 2^62
__device__ __forceinline__ bool qwide_ray_fits(f3 ro, f3 inv)
{
    return fmaxf(fmaxf(fabsf(inv.x), fabsf(inv.y)), fmaxf(fabsf(inv.z), fmaxf(fmaxf(fabsf(ro.x), fabsf(ro.y)),
                                                                               fabsf(ro.z)))) < kQRayLimit;
}
// Relative margins of the quantised slab test: 2^-22 below the entry and
// 2^-21 above the exit (see qnode_test and qwide_visit).
constexpr float kQEntryMargin = 2.384185791015625e-07f;
constexpr float kQExitMargin = 4.76837158203125e-07f;

// The per-walk parameters of the quantised binary tree: its scale exponent
// EB (mlbvh_qheader::eBase), its status word, and whether this ray takes the
// FMA form (status 0 and qwide_ray_fits).
struct QParams {
    int eb;
    uint32_t status;
    bool fma;
};
__device__ __forceinline__ QParams qparams(const mlbvh_qheader* __restrict__ header, f3 ro, f3 inv)
{
    const int eb = __ldg(&header->eBase);
    const uint32_t status = __ldg(&header->status);
    return QParams{eb, status, status == 0u && qwide_ray_fits(ro, inv)};
}

// A quantised node's words: base (3 floats), the codes of axis x, y, z (bytes
// child 0 lower, child 0 upper, child 1 lower, child 1 upper), the child
// words (bits 23-30 the axis exponents as k = EB - E, 5 bits each: child 0
// k_x | k_y bits 0-2, child 1 k_y bits 3-4 | k_z). One 32-byte load.
struct QNodeWords {
    f3 base;
    uint32_t q[3];
    uint32_t c0, c1;       // leaf flag | 23-bit index
    uint32_t scale[3];     // bits of 2^E per axis
};
__device__ __forceinline__ QNodeWords load_qnode(const mlbvh_qnode* __restrict__ qnodes, uint32_t i, int eb)
{
    float4 a, b;
    ldg32(reinterpret_cast<const float4*>(qnodes + i), a, b);
    QNodeWords n;
    n.base = mk(a.x, a.y, a.z);
    n.q[0] = __float_as_uint(a.w);
    n.q[1] = __float_as_uint(b.x);
    n.q[2] = __float_as_uint(b.y);
    const uint32_t w6 = __float_as_uint(b.z), w7 = __float_as_uint(b.w);
    const uint32_t code = ((w6 >> 23) & 0xFFu) | (((w7 >> 23) & 0x7Fu) << 8);
    const int e127 = eb + 127;
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2) n.scale[a2] = (uint32_t)(e127 - (int)((code >> (5 * a2)) & 31u)) << 23;
    n.c0 = w6 & (kLeafBit | kQIndexMask);
    n.c1 = w7 & (kLeafBit | kQIndexMask);
    return n;
}
// Child c's decoded box: base + V with V exact, the sum rounded down for the
// lower planes and up for the upper ones, so it contains the exact box.
__device__ __forceinline__ void qnode_box(const QNodeWords& n, int c, f3& lo, f3& hi)
{
    lo = mk(__fadd_rd(n.base.x, qw_value(n.q[0], n.scale[0], 2 * c)),
            __fadd_rd(n.base.y, qw_value(n.q[1], n.scale[1], 2 * c)),
            __fadd_rd(n.base.z, qw_value(n.q[2], n.scale[2], 2 * c)));
    hi = mk(__fadd_ru(n.base.x, qw_value(n.q[0], n.scale[0], 2 * c + 1)),
            __fadd_ru(n.base.y, qw_value(n.q[1], n.scale[1], 2 * c + 1)),
            __fadd_ru(n.base.z, qw_value(n.q[2], n.scale[2], 2 * c + 1)));
}

// The slab test of both children of a quantised node: (entry, exit) per
// child, clipped to [max(0, tmin), hitT]; a child passes when entry <= exit.
// FMA form (qp.fma): a plane's distance along the ray, (base + V - ro) inv,
// is one FMA, V inv + C, with C = base inv - ro inv bounding (base - ro) inv
// from below for near planes (ro inv rounded up, the FMA rounded down) and
// from above for far planes (ro inv rounded down, the FMA rounded up); the
// plane's FMA is rounded the same way. On an axis whose inv is positive the
// near plane is the lower one, on one whose inv is negative the upper one.
// The entry (the largest near distance) is moved down by 2^-22 of itself and
// the exit (the smallest far one) up by 2^-21 of itself, which covers the
// reference slab's own rounding on the exact box (two roundings per distance,
// then its 1.00000024 factor on the exit and that product's rounding); the
// codes were rounded outward too, so the test passes wherever the reference's
// passes on the exact box. Otherwise the reference's slabs on the decoded
// boxes (qnode_box), conservative at any magnitude. A tree with a
// non-finite coordinate (status bit 1) lets every box pass.
// kPacked takes both children's planes as packed FP32 pairs (the same
// values); the any-hit walks use it (AO rays 1.7 % faster), the closest-hit
// walks do not (camera rays 3.8 % slower with it).
template <bool kPacked>
__device__ __forceinline__ float4 qnode_test(const QNodeWords& n, const QParams& qp, f3 ro, f3 inv, float tmin,
                                             float hitT)
{
    if (qp.status & 2u) {
        const float lo = fmaxf(0.0f, tmin);
        return make_float4(lo, hitT, lo, hitT);
    }
    if (qp.fma) {
        const float cnx = __fmaf_rd(n.base.x, inv.x, -__fmul_ru(ro.x, inv.x));
        const float cny = __fmaf_rd(n.base.y, inv.y, -__fmul_ru(ro.y, inv.y));
        const float cnz = __fmaf_rd(n.base.z, inv.z, -__fmul_ru(ro.z, inv.z));
        const float cfx = __fmaf_ru(n.base.x, inv.x, -__fmul_rd(ro.x, inv.x));
        const float cfy = __fmaf_ru(n.base.y, inv.y, -__fmul_rd(ro.y, inv.y));
        const float cfz = __fmaf_ru(n.base.z, inv.z, -__fmul_rd(ro.z, inv.z));
        // per axis the codes ordered (near, far) for each child: where inv is
        // negative the upper plane is the near one, so its byte pairs swap
        const uint32_t qx = __byte_perm(n.q[0], 0u, inv.x < 0.0f ? 0x2301u : 0x3210u);
        const uint32_t qy = __byte_perm(n.q[1], 0u, inv.y < 0.0f ? 0x2301u : 0x3210u);
        const uint32_t qz = __byte_perm(n.q[2], 0u, inv.z < 0.0f ? 0x2301u : 0x3210u);
        const float lo = fmaxf(0.0f, tmin);
        if constexpr (kPacked) {
            // both children side by side: per axis and side one packed FMA
            // (sm_100) over their planes (codes 0 and 2 near, 1 and 3 far)
            const float2 nx = __ffma2_rd(make_float2(qw_value(qx, n.scale[0], 0), qw_value(qx, n.scale[0], 2)),
                                         make_float2(inv.x, inv.x), make_float2(cnx, cnx));
            const float2 ny = __ffma2_rd(make_float2(qw_value(qy, n.scale[1], 0), qw_value(qy, n.scale[1], 2)),
                                         make_float2(inv.y, inv.y), make_float2(cny, cny));
            const float2 nz = __ffma2_rd(make_float2(qw_value(qz, n.scale[2], 0), qw_value(qz, n.scale[2], 2)),
                                         make_float2(inv.z, inv.z), make_float2(cnz, cnz));
            const float2 fx2 = __ffma2_ru(make_float2(qw_value(qx, n.scale[0], 1), qw_value(qx, n.scale[0], 3)),
                                          make_float2(inv.x, inv.x), make_float2(cfx, cfx));
            const float2 fy2 = __ffma2_ru(make_float2(qw_value(qy, n.scale[1], 1), qw_value(qy, n.scale[1], 3)),
                                          make_float2(inv.y, inv.y), make_float2(cfy, cfy));
            const float2 fz2 = __ffma2_ru(make_float2(qw_value(qz, n.scale[2], 1), qw_value(qz, n.scale[2], 3)),
                                          make_float2(inv.z, inv.z), make_float2(cfz, cfz));
            const float2 en = make_float2(fmaxf(fmaxf(nx.x, ny.x), nz.x), fmaxf(fmaxf(nx.y, ny.y), nz.y));
            // entry - 2^-22 entry rounded down: the same as with |entry|
            // wherever entry >= 0, and both are negative (clipped to lo >= 0)
            // elsewhere
            const float2 em = __ffma2_rd(en, make_float2(-kQEntryMargin, -kQEntryMargin), en);
            const float exa = fminf(fminf(fx2.x, fy2.x), fz2.x), exb = fminf(fminf(fx2.y, fy2.y), fz2.y);
            return make_float4(fmaxf(em.x, lo), fminf(__fmaf_ru(fabsf(exa), kQExitMargin, exa), hitT),
                               fmaxf(em.y, lo), fminf(__fmaf_ru(fabsf(exb), kQExitMargin, exb), hitT));
        } else {
            float r[4];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const float en = fmaxf(fmaxf(__fmaf_rd(qw_value(qx, n.scale[0], 2 * c), inv.x, cnx),
                                             __fmaf_rd(qw_value(qy, n.scale[1], 2 * c), inv.y, cny)),
                                       __fmaf_rd(qw_value(qz, n.scale[2], 2 * c), inv.z, cnz));
                const float ex = fminf(fminf(__fmaf_ru(qw_value(qx, n.scale[0], 2 * c + 1), inv.x, cfx),
                                             __fmaf_ru(qw_value(qy, n.scale[1], 2 * c + 1), inv.y, cfy)),
                                       __fmaf_ru(qw_value(qz, n.scale[2], 2 * c + 1), inv.z, cfz));
                r[2 * c] = fmaxf(__fmaf_rd(fabsf(en), -kQEntryMargin, en), lo);
                r[2 * c + 1] = fminf(__fmaf_ru(fabsf(ex), kQExitMargin, ex), hitT);
            }
            return make_float4(r[0], r[1], r[2], r[3]);
        }
    }
    f3 lo0, hi0, lo1, hi1;
    qnode_box(n, 0, lo0, hi0);
    qnode_box(n, 1, lo1, hi1);
    const float2 a = slab(ro, inv, lo0, hi0, tmin, hitT), b = slab(ro, inv, lo1, hi1, tmin, hitT);
    return make_float4(a.x, a.y, b.x, b.y);
}

// The reference's own test of a leaf: its slabs (minimum_lbvh.h:82-96) on the
// triangle's FP32 box, as its parent node stores it. A quantised walk reaches
// every leaf the FP32 walk reaches and a few more (its boxes are larger); a
// hit it finds counts only if the triangle's exact box passes, which makes the
// hits it can find those of the FP32 walk: for FP32 boxes the slab test is
// monotone, so a leaf box that passes implies every ancestor box passes too.
// A miss needs no check, so the check runs on hits only.
__device__ __forceinline__ bool leaf_box_passes(f3 ro, f3 inv, f3 v0, f3 v1, f3 v2, float tmin, float hitT)
{
    const f3 lo = smin3(smin3(smin3(mk(kFltMax, kFltMax, kFltMax), v0), v1), v2);
    const f3 hi = smax3(smax3(smax3(mk(-kFltMax, -kFltMax, -kFltMax), v0), v1), v2);
    const float2 t = slab(ro, inv, lo, hi, tmin, hitT);
    return t.x <= t.y;
}

// Stack-free walk over the quantised tree: the state machine of
// intersect_stackfree (minimum_lbvh.h:981-1061), with "came from the parent"
// recognised as "came from neither child" so that the parent word is read
// only when the walk moves up. quantised_step advances it by one leaf test or
// internal-node visit and returns true when the walk is over; nu counts
// parent-word loads. The node test is qnode_test (qp from qparams).
template <bool kAny, bool kCount>
__device__ __forceinline__ bool quantised_step(uint32_t& curr, uint32_t& prev, HitRecord& hit,
                                               const mlbvh_qnode* __restrict__ qnodes,
                                               const uint32_t* __restrict__ parents,
                                               const mlbvh_qtri* __restrict__ qtris, const QParams& qp, f3 ro, f3 rd,
                                               f3 inv, float tmin, uint32_t& nv, uint32_t& nt, uint32_t& nu)
{
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const float4* t = reinterpret_cast<const float4*>(qtris + (curr & kQIndexMask));
        const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        const f3 v0 = mk(a.x, a.y, a.z), v1 = mk(a.w, b.x, b.y), v2 = mk(b.z, b.w, c.x);
        float tt, u, v;
        f3 ng;
        if (intersect_triangle(tt, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2) &&
            leaf_box_passes(ro, inv, v0, v1, v2, tmin, hit.t)) {
            hit.t = tt;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = __float_as_uint(c.y);
            if (kAny) return true;
        }
        const uint32_t s = curr;
        curr = prev;
        prev = s;
        return curr == kInvalid;
    }
    if (kCount) ++nv;
    const QNodeWords nd = load_qnode(qnodes, curr, qp.eb);
    const float4 r = qnode_test<kAny>(nd, qp, ro, inv, tmin, hit.t);  // packed pairs on any-hit walks
    const float2 rl = make_float2(r.x, r.y), rr = make_float2(r.z, r.w);
    const bool hitL = rl.x <= rl.y, hitR = rr.x <= rr.y;
    uint32_t nearN = nd.c0, farN = nd.c1;
    int nHits = 0;
    if (hitL && hitR) {
        if (rr.x < rl.x) {
            nearN = nd.c1;
            farN = nd.c0;
        }
        nHits = 2;
    } else if (hitL || hitR) {
        nHits = 1;
        nearN = hitR ? farN : nearN;
    }
    const bool fromParent = prev != nd.c0 && prev != nd.c1;
    uint32_t next = kInvalid;
    bool up;
    if (fromParent) {
        up = nHits == 0;
        next = nearN;
    } else if (prev == nearN) {
        up = nHits != 2;
        next = farN;
    } else {
        up = true;
    }
    if (up) {
        if (kCount) ++nu;
        next = __ldg(parents + curr);
    }
    prev = curr;
    curr = next;
    return curr == kInvalid;
}

// The same walk with a stack of pending far children instead of revisits.
// At a node whose two child boxes are hit, the far child and its entry
// distance are pushed and the near child is entered; when a subtree is done,
// entries are popped and an entry is entered iff its entry distance is still
// <= hit.t. That is exactly when the stack-free walk, back at the parent from
// the near child, finds both boxes still hit: a box's entry distance does not
// depend on hit.t, and the near entry never exceeds the far one. So leaves
// are tested in the same order against the same hit.t and the Hit record is
// the stack-free walk's bit for bit, with each internal node loaded once
// instead of up to three times and no parent loads.
//
// The stack holds kDepth entries of this thread at stack[d * stride]
// (shared memory, one column per thread). A push onto a full stack hands the
// walk to the stack-free state machine at (near child, this node), marked by
// depth = -1; climbing through the parents, it re-derives every entry still
// on the stack. Start a walk with curr = root, depth = 0.
template <bool kAny, bool kCount, int kDepth>
__device__ __forceinline__ bool quantised_replay_step(uint32_t& curr, uint32_t& prev, int& depth,
                                                      typename ReplayStack<kAny>::Entry* stack,
                                                      int stride, HitRecord& hit,
                                                      const mlbvh_qnode* __restrict__ qnodes,
                                                      const uint32_t* __restrict__ parents,
                                                      const mlbvh_qtri* __restrict__ qtris, const QParams& qp, f3 ro,
                                                      f3 rd, f3 inv, float tmin, uint32_t& nv, uint32_t& nt,
                                                      uint32_t& nu)
{
    if (depth < 0)
        return quantised_step<kAny, kCount>(curr, prev, hit, qnodes, parents, qtris, qp, ro, rd, inv, tmin, nv, nt, nu);
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const float4* t = reinterpret_cast<const float4*>(qtris + (curr & kQIndexMask));
        const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        const f3 v0 = mk(a.x, a.y, a.z), v1 = mk(a.w, b.x, b.y), v2 = mk(b.z, b.w, c.x);
        float tt, u, v;
        f3 ng;
        if (intersect_triangle(tt, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2) &&
            leaf_box_passes(ro, inv, v0, v1, v2, tmin, hit.t)) {
            hit.t = tt;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = __float_as_uint(c.y);
            if (kAny) return true;
        }
    } else {
        if (kCount) ++nv;
        const QNodeWords nd = load_qnode(qnodes, curr, qp.eb);
        const float4 r = qnode_test<kAny>(nd, qp, ro, inv, tmin, hit.t);  // packed pairs on any-hit walks
        const float2 rl = make_float2(r.x, r.y), rr = make_float2(r.z, r.w);
        const bool hitL = rl.x <= rl.y, hitR = rr.x <= rr.y;
        if (hitL && hitR) {
            const bool swap = rr.x < rl.x;
            const uint32_t nearN = swap ? nd.c1 : nd.c0, farN = swap ? nd.c0 : nd.c1;
            if (depth == kDepth) {  // full: continue as the stack-free walk
                depth = -1;
                prev = curr;
                curr = nearN;
                return false;
            }
            if constexpr (kAny)
                stack[depth * stride] = farN;
            else
                stack[depth * stride] = make_uint2(farN, __float_as_uint(swap ? rl.x : rr.x));
            ++depth;
            curr = nearN;
            return false;
        }
        if (hitL || hitR) {
            curr = hitL ? nd.c0 : nd.c1;
            return false;
        }
    }
    if constexpr (kAny) {
        if (depth == 0) return true;
        curr = stack[--depth * stride];
        return false;
    } else {
        while (depth > 0) {
            const uint2 e = stack[--depth * stride];
            if (__uint_as_float(e.y) <= hit.t) {
                curr = e.x;
                return false;
            }
        }
        return true;
    }
}

template <bool kAny, bool kCount = false>
__device__ __forceinline__ void trace_quantised(HitRecord& hit, const mlbvh_qnode* __restrict__ qnodes,
                                                const uint32_t* __restrict__ parents,
                                                const mlbvh_qtri* __restrict__ qtris, uint32_t root,
                                                const QParams& qp, f3 ro, f3 rd, f3 inv, float tmin,
                                                uint32_t* visits = nullptr, uint32_t* tests = nullptr,
                                                uint32_t* ups = nullptr)
{
    uint32_t curr = root, prev = kInvalid, nv = 0, nt = 0, nu = 0;
    for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
        if (quantised_step<kAny, kCount>(curr, prev, hit, qnodes, parents, qtris, qp, ro, rd, inv, tmin, nv, nt, nu))
            break;
    if (kCount) {
        *visits += nv;
        *tests += nt;
        *ups += nu;
    }
}


// ------------------------------------------------------- the 4-wide tree
// mlbvh_wnode / mlbvh_qwnode (include/mlbvh.h): slot i is the expansion of
// binary internal node i into at most four children with the binary tree's
// own boxes (mlbvh_wnode), or those boxes with 8-bit planes rounded outward
// (mlbvh_qwnode). Only any-hit rays walk it: a leaf whose box passes the
// slab test is reached through boxes that contain it and therefore pass too
// (the slab test is monotone in the box: every operation rounds to nearest,
// which preserves order), and only leaves whose own box passes are tested (on
// the quantised slots, a hit counts only if the leaf's exact box passes,
// leaf_box_passes), so a ray finds a hit exactly when intersect_stackfree's
// any-hit walk does.
constexpr uint32_t kWideEmpty = 0xFFFFFFFFu;  // an empty child slot
constexpr int kWideDepth = 24;                // stack entries per ray

__device__ __forceinline__ float wpick(const float4& v, int k)
{
    return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}
__device__ __forceinline__ uint32_t wpick(const uint4& v, int k)
{
    return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}

// One visit: which non-empty children pass (bit mask), the nearest of them
// (entry distance, ties to the lower slot; -1 if none), the child words and
// every child's entry distance (the closest-hit walk orders by them).
struct WideVisit {
    uint32_t pass;
    int best;
    uint4 ch;
    float entry[4];
};
// FP32 slot: three 32-byte plane loads and the 16-byte child words.
// kPacked computes the slabs as packed FP32 pairs (the same values); the
// closest-hit walk uses it (camera rays 4 % faster), the any-hit walk does not
// (AO rays 5 % slower with it). The same holds for qwide_visit (2 % faster,
// 3.5 % slower).
template <bool kPacked>
__device__ __forceinline__ WideVisit wide_visit(const mlbvh_wnode* __restrict__ wnodes, uint32_t i, f3 ro, f3 inv,
                                                float tmin, float hitT)
{
    const float4* p = reinterpret_cast<const float4*>(wnodes + i);
    float4 lx, hx, ly, hy, lz, hz;
    ldg32(p, lx, hx);
    ldg32(p + 2, ly, hy);
    ldg32(p + 4, lz, hz);
    WideVisit w{0u, -1, __ldg(reinterpret_cast<const uint4*>(p + 6)), {}};
    float bestT = 0.0f;
    // kPacked: slab() on two children at a time, each plane's difference and
    // product as packed FP32 pairs (sm_100), rounded to nearest per
    // component, so every distance is the scalar slab's bit for bit
    float en4[4], ex4[4];
    if constexpr (kPacked) {
        const float2 nrx = make_float2(-ro.x, -ro.x), nry = make_float2(-ro.y, -ro.y), nrz = make_float2(-ro.z, -ro.z);
        const float2 ix = make_float2(inv.x, inv.x), iy = make_float2(inv.y, inv.y), iz = make_float2(inv.z, inv.z);
#pragma unroll
        for (int p = 0; p < 4; p += 2) {
            const float2 t0x = __fmul2_rn(__fadd2_rn(make_float2(wpick(lx, p), wpick(lx, p + 1)), nrx), ix);
            const float2 t1x = __fmul2_rn(__fadd2_rn(make_float2(wpick(hx, p), wpick(hx, p + 1)), nrx), ix);
            const float2 t0y = __fmul2_rn(__fadd2_rn(make_float2(wpick(ly, p), wpick(ly, p + 1)), nry), iy);
            const float2 t1y = __fmul2_rn(__fadd2_rn(make_float2(wpick(hy, p), wpick(hy, p + 1)), nry), iy);
            const float2 t0z = __fmul2_rn(__fadd2_rn(make_float2(wpick(lz, p), wpick(lz, p + 1)), nrz), iz);
            const float2 t1z = __fmul2_rn(__fadd2_rn(make_float2(wpick(hz, p), wpick(hz, p + 1)), nrz), iz);
            const float2 rmax = __fmul2_rn(
                make_float2(fminf(fminf(fmaxf(t0x.x, t1x.x), fmaxf(t0y.x, t1y.x)), fmaxf(t0z.x, t1z.x)),
                            fminf(fminf(fmaxf(t0x.y, t1x.y), fmaxf(t0y.y, t1y.y)), fmaxf(t0z.y, t1z.y))),
                make_float2(1.00000024f, 1.00000024f));
            en4[p] = fmaxf(fmaxf(fmaxf(fmaxf(fminf(t0x.x, t1x.x), fminf(t0y.x, t1y.x)), fminf(t0z.x, t1z.x)), 0.0f),
                           tmin);
            en4[p + 1] = fmaxf(
                fmaxf(fmaxf(fmaxf(fminf(t0x.y, t1x.y), fminf(t0y.y, t1y.y)), fminf(t0z.y, t1z.y)), 0.0f), tmin);
            ex4[p] = fminf(rmax.x, hitT);
            ex4[p + 1] = fminf(rmax.y, hitT);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float2 r;
        if constexpr (kPacked)
            r = make_float2(en4[k], ex4[k]);
        else
            r = slab(ro, inv, mk(wpick(lx, k), wpick(ly, k), wpick(lz, k)),
                     mk(wpick(hx, k), wpick(hy, k), wpick(hz, k)), tmin, hitT);
        w.entry[k] = r.x;
        if (wpick(w.ch, k) != kWideEmpty && r.x <= r.y) {
            w.pass |= 1u << k;
            if (w.best < 0 || r.x < bestT) {
                w.best = k;
                bestT = r.x;
            }
        }
    }
    return w;
}

// Quantised slot (two 32-byte loads): per axis a base and a scale 2^E, the
// planes at base + V (qw_value). The distance of a plane along the ray,
// (base + V - ro) inv, is one FMA per plane: V inv + C, where C = base inv - ro inv bounds (base - ro) inv from
// below for near planes (ro inv rounded up, the FMA rounded down) and from
// above for far planes (ro inv rounded down, the FMA rounded up); the plane's
// FMA is rounded the same way. On an axis whose inv is positive the near
// plane is the lower one, on one whose inv is negative the upper one (inv is
// never 0). A child's entry is the largest of its near distances, its exit
// the smallest far one, each moved outward by a relative margin (entry -
// 2^-22 |entry| rounded down, exit + 2^-21 |exit| rounded up) that covers
// the reference slab's own rounding on the exact box (two roundings per
// distance, then the 1.00000024 factor on the exit and its rounding). The
// codes were rounded outward too, so entry <= the reference's entry and exit
// >= its exit: the test passes wherever the reference's passes on the exact
// box. Every rounding is directed, so a distance that overflows stays on its
// conservative side (an FMA rounded down gives FLT_MAX or -inf).
template <bool kPacked>
__device__ __forceinline__ WideVisit qwide_visit(const mlbvh_qwnode* __restrict__ qw, uint32_t i, f3 ro, f3 inv,
                                                 float tmin, float hitT)
{
    const float4* p = reinterpret_cast<const float4*>(qw + i);
    float4 a, b, c, d;
    ldg32(p, a, b);
    ldg32(p + 2, c, d);
    const uint32_t sx = __float_as_uint(a.w), sy = __float_as_uint(b.x), sz = __float_as_uint(b.y);
    const bool fx = inv.x < 0.0f, fy = inv.y < 0.0f, fz = inv.z < 0.0f;
    const uint32_t qxl = __float_as_uint(b.z), qxh = __float_as_uint(b.w), qyl = __float_as_uint(c.x),
                   qyh = __float_as_uint(c.y), qzl = __float_as_uint(c.z), qzh = __float_as_uint(c.w);
    const uint32_t nqx = fx ? qxh : qxl, fqx = fx ? qxl : qxh;
    const uint32_t nqy = fy ? qyh : qyl, fqy = fy ? qyl : qyh;
    const uint32_t nqz = fz ? qzh : qzl, fqz = fz ? qzl : qzh;
    const float cnx = __fmaf_rd(a.x, inv.x, -__fmul_ru(ro.x, inv.x));
    const float cny = __fmaf_rd(a.y, inv.y, -__fmul_ru(ro.y, inv.y));
    const float cnz = __fmaf_rd(a.z, inv.z, -__fmul_ru(ro.z, inv.z));
    const float cfx = __fmaf_ru(a.x, inv.x, -__fmul_rd(ro.x, inv.x));
    const float cfy = __fmaf_ru(a.y, inv.y, -__fmul_rd(ro.y, inv.y));
    const float cfz = __fmaf_ru(a.z, inv.z, -__fmul_rd(ro.z, inv.z));
    const float lo = fmaxf(0.0f, tmin);
    WideVisit w{0u, -1, make_uint4(__float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z),
                                   __float_as_uint(d.w)), {}};
    float bestT = 0.0f;
    // kPacked: two children at a time, per axis and side one packed FMA
    // (sm_100) over the pair's planes and one for the pair's entry margins
    float en4[4], ex4[4];
    if constexpr (kPacked) {
        const float2 ix = make_float2(inv.x, inv.x), iy = make_float2(inv.y, inv.y), iz = make_float2(inv.z, inv.z);
#pragma unroll
        for (int p = 0; p < 4; p += 2) {
            const float2 nx = __ffma2_rd(make_float2(qw_value(nqx, sx, p), qw_value(nqx, sx, p + 1)), ix,
                                         make_float2(cnx, cnx));
            const float2 ny = __ffma2_rd(make_float2(qw_value(nqy, sy, p), qw_value(nqy, sy, p + 1)), iy,
                                         make_float2(cny, cny));
            const float2 nz = __ffma2_rd(make_float2(qw_value(nqz, sz, p), qw_value(nqz, sz, p + 1)), iz,
                                         make_float2(cnz, cnz));
            const float2 fx2 = __ffma2_ru(make_float2(qw_value(fqx, sx, p), qw_value(fqx, sx, p + 1)), ix,
                                          make_float2(cfx, cfx));
            const float2 fy2 = __ffma2_ru(make_float2(qw_value(fqy, sy, p), qw_value(fqy, sy, p + 1)), iy,
                                          make_float2(cfy, cfy));
            const float2 fz2 = __ffma2_ru(make_float2(qw_value(fqz, sz, p), qw_value(fqz, sz, p + 1)), iz,
                                          make_float2(cfz, cfz));
            const float2 en = make_float2(fmaxf(fmaxf(nx.x, ny.x), nz.x), fmaxf(fmaxf(nx.y, ny.y), nz.y));
            // entry - 2^-22 entry rounded down: the same as with |entry|
            // wherever entry >= 0, and both are negative (clipped to lo >= 0)
            // elsewhere
            const float2 em = __ffma2_rd(en, make_float2(-kQEntryMargin, -kQEntryMargin), en);
            const float exa = fminf(fminf(fx2.x, fy2.x), fz2.x), exb = fminf(fminf(fx2.y, fy2.y), fz2.y);
            en4[p] = fmaxf(em.x, lo);
            en4[p + 1] = fmaxf(em.y, lo);
            ex4[p] = fminf(__fmaf_ru(fabsf(exa), kQExitMargin, exa), hitT);
            ex4[p + 1] = fminf(__fmaf_ru(fabsf(exb), kQExitMargin, exb), hitT);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float en = fmaxf(fmaxf(__fmaf_rd(qw_value(nqx, sx, k), inv.x, cnx),
                                         __fmaf_rd(qw_value(nqy, sy, k), inv.y, cny)),
                                   __fmaf_rd(qw_value(nqz, sz, k), inv.z, cnz));
            const float ex = fminf(fminf(__fmaf_ru(qw_value(fqx, sx, k), inv.x, cfx),
                                         __fmaf_ru(qw_value(fqy, sy, k), inv.y, cfy)),
                                   __fmaf_ru(qw_value(fqz, sz, k), inv.z, cfz));
            en4[k] = fmaxf(__fmaf_rd(fabsf(en), -kQEntryMargin, en), lo);
            ex4[k] = fminf(__fmaf_ru(fabsf(ex), kQExitMargin, ex), hitT);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float entry = en4[k], exit = ex4[k];
        w.entry[k] = entry;
        if (wpick(w.ch, k) != kWideEmpty && entry <= exit) {
            w.pass |= 1u << k;
            if (w.best < 0 || entry < bestT) {
                w.best = k;
                bestT = entry;
            }
        }
    }
    return w;
}

// One step of the any-hit walk over the wide tree (FP32 slots, or quantised
// slots with kQuant): a leaf test (leaf-ordered triangles) or a slot visit.
// At a slot, every non-empty child whose box passes is taken: the nearest
// entry first, the others pushed in slot order. A visit whose pushes would
// overflow the stack (kWideDepth entries, shared memory, `stride` apart)
// restarts the ray with the stack-free walk over the binary tree from
// `binaryRoot` (depth < 0 from then on; ++nr). Returns true when the walk is
// over (a hit, or nothing left).
template <bool kCount, bool kQuant, class Slot>
__device__ __forceinline__ bool wide_any_step(uint32_t& curr, uint32_t& prev, int& depth, uint32_t* stack, int stride,
                                              HitRecord& hit, const Slot* __restrict__ slots,
                                              const mlbvh_internal_node* __restrict__ nodes,
                                              const float* __restrict__ tris, const mlbvh_qtri* __restrict__ leafTris,
                                              uint32_t binaryRoot, f3 ro, f3 rd, f3 inv, float tmin, uint32_t& nv,
                                              uint32_t& nt, uint32_t& nr)
{
    if (depth < 0) return stackfree_step<true, kCount, true>(curr, prev, hit, nodes, tris, ro, rd, inv, tmin, nv, nt);
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const float4* t = reinterpret_cast<const float4*>(leafTris + (curr & ~kLeafBit));
        const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        const f3 v0 = mk(a.x, a.y, a.z), v1 = mk(a.w, b.x, b.y), v2 = mk(b.z, b.w, c.x);
        float tt, u, v;
        f3 ng;
        if (intersect_triangle(tt, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2) &&
            (!kQuant || leaf_box_passes(ro, inv, v0, v1, v2, tmin, hit.t))) {
            hit.t = tt;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = __float_as_uint(c.y);
            return true;
        }
    } else {
        if (kCount) ++nv;
        WideVisit w;
        if constexpr (kQuant)
            w = qwide_visit<false>(slots, curr, ro, inv, tmin, hit.t);
        else
            w = wide_visit<false>(slots, curr, ro, inv, tmin, hit.t);
        if (w.pass) {
            const uint32_t others = w.pass & ~(1u << w.best);
            if (depth + __popc(others) > kWideDepth) {
                if (kCount) ++nr;
                depth = -1;
                curr = binaryRoot;
                prev = kInvalid;
                return false;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (others & (1u << k)) stack[depth++ * stride] = wpick(w.ch, k);
            curr = wpick(w.ch, w.best);
            return false;
        }
    }
    if (depth == 0) return true;
    curr = stack[--depth * stride];
    return false;
}

// The closest-hit walk over the wide tree (FP32 slots, or quantised slots
// with kQuant). At a slot, the children whose box passes are entered in the
// order of their sort keys, nearest first: the key of child k is the bits of
// its entry distance (>= 0) with the two lowest bits replaced by k, so entries
// within four ulps go in slot order. The others are pushed farthest first,
// each with its key's distance (at most its entry), and a popped child is
// entered only if that distance is still <= hit.t (a box whose entry lies
// beyond hit.t fails the slab test). A triangle hit at t <= hit.t (the
// reference's inclusive test) replaces the hit; on the quantised slots only
// if the leaf's exact box passes the slab test too. A visit whose pushes would
// overflow the stack (kWideDepth entries of {child, distance}, `stride` apart)
// continues with the closest-hit stack-free walk over the binary tree from
// `binaryRoot`, keeping the hit found so far (depth < 0 from then on; ++nr).
// The hit found is intersect_stackfree's wherever the nearest hit triangle's
// own box passes the slab test at that triangle's distance (a box holds its
// triangle, and the boxes above it pass whenever it does, so the walk enters
// it whatever the order); the order decides only between hits at
// bit-identical t, and where the rounded slabs exclude the hit point from its
// triangle's box. Returns true when the walk is over.
__device__ __forceinline__ uint32_t wide_sort_key(const WideVisit& w, int k)
{
    return (w.pass & (1u << k)) ? ((__float_as_uint(w.entry[k]) & 0x7FFFFFFCu) | (uint32_t)k) : 0xFFFFFFFFu;
}
template <bool kCount, bool kQuant, class Slot>
__device__ __forceinline__ bool wide_closest_step(uint32_t& curr, uint32_t& prev, int& depth, uint2* stack,
                                                  int stride, HitRecord& hit, const Slot* __restrict__ slots,
                                                  const mlbvh_internal_node* __restrict__ nodes,
                                                  const float* __restrict__ tris,
                                                  const mlbvh_qtri* __restrict__ leafTris, uint32_t binaryRoot, f3 ro,
                                                  f3 rd, f3 inv, float tmin, uint32_t& nv, uint32_t& nt,
                                                  uint32_t& nr)
{
    if (depth < 0) return stackfree_step<false, kCount, true>(curr, prev, hit, nodes, tris, ro, rd, inv, tmin, nv, nt);
    if (curr & kLeafBit) {
        if (kCount) ++nt;
        const float4* t = reinterpret_cast<const float4*>(leafTris + (curr & ~kLeafBit));
        const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        const f3 v0 = mk(a.x, a.y, a.z), v1 = mk(a.w, b.x, b.y), v2 = mk(b.z, b.w, c.x);
        float tt, u, v;
        f3 ng;
        if (intersect_triangle(tt, u, v, ng, tmin, hit.t, ro, rd, v0, v1, v2) &&
            (!kQuant || leaf_box_passes(ro, inv, v0, v1, v2, tmin, hit.t))) {
            hit.t = tt;
            hit.u = u;
            hit.v = v;
            hit.ng = ng;
            hit.tri = __float_as_uint(c.y);
        }
    } else {
        if (kCount) ++nv;
        WideVisit w;
        if constexpr (kQuant)
            w = qwide_visit<true>(slots, curr, ro, inv, tmin, hit.t);
        else
            w = wide_visit<true>(slots, curr, ro, inv, tmin, hit.t);
        if (w.pass) {
            const int np = __popc(w.pass);
            if (depth + np - 1 > kWideDepth) {
                if (kCount) ++nr;
                depth = -1;
                curr = binaryRoot;
                prev = kInvalid;
                return false;
            }
            // sort the four keys (a five-exchange network); non-passing children sort last
            uint32_t k0 = wide_sort_key(w, 0), k1 = wide_sort_key(w, 1), k2 = wide_sort_key(w, 2),
                     k3 = wide_sort_key(w, 3), x;
            x = min(k0, k1); k1 = max(k0, k1); k0 = x;
            x = min(k2, k3); k3 = max(k2, k3); k2 = x;
            x = min(k0, k2); k2 = max(k0, k2); k0 = x;
            x = min(k1, k3); k3 = max(k1, k3); k1 = x;
            x = min(k1, k2); k2 = max(k1, k2); k1 = x;
            if (np == 4) stack[depth++ * stride] = make_uint2(wpick(w.ch, (int)(k3 & 3u)), k3 & 0x7FFFFFFCu);
            if (np >= 3) stack[depth++ * stride] = make_uint2(wpick(w.ch, (int)(k2 & 3u)), k2 & 0x7FFFFFFCu);
            if (np >= 2) stack[depth++ * stride] = make_uint2(wpick(w.ch, (int)(k1 & 3u)), k1 & 0x7FFFFFFCu);
            curr = wpick(w.ch, (int)(k0 & 3u));
            return false;
        }
    }
    while (depth > 0) {
        const uint2 e = stack[--depth * stride];
        if (__uint_as_float(e.y) <= hit.t) {
            curr = e.x;
            return false;
        }
    }
    return true;
}

}  // namespace mlbvh
