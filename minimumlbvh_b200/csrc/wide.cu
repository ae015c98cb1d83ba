// The 4-wide tree (no reference counterpart): a regrouping of the binary tree
// that intersect_stackfree walks (minimum_lbvh.h:981-1061) with the same
// leaves and the same boxes, so that a ray loads half as many nodes in a
// chain (any-hit and closest-hit walks). Slot i of the wide array is the expansion of
// binary internal node i, written by one thread with no order between slots:
// the walk starts at the root's slot and only ever follows child indices,
// which name the slots of their own expansions.
#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {
namespace {

constexpr int kWideThreads = 256;
// threads per CTA of the wide trace kernel (build-time override for sweeps: -DMLBVH_WIDE_TRACE_THREADS=...)
#ifndef MLBVH_WIDE_TRACE_THREADS
#define MLBVH_WIDE_TRACE_THREADS 128
#endif
constexpr int kWideTraceThreads = MLBVH_WIDE_TRACE_THREADS;

struct WideKid {
    uint32_t name;  // internal index, kLeafBit | leaf position, or kWideEmpty
    f3 lo, hi;
};

__device__ __forceinline__ float half_area(f3 lo, f3 hi)
{
    const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    float a = dx * dy;
    a = a + dy * dz;
    a = a + dz * dx;
    return a;
}

// Leaf children of binary node p are named by leaf position: the left one is
// leaf p, the right one leaf p + 1 (mlbvh_leaf_triangles' order).
__device__ __forceinline__ void binary_children(const mlbvh_internal_node* __restrict__ nodes, uint32_t p, WideKid& a,
                                                WideKid& b)
{
    const NodeView nd = load_node<true>(nodes, p);
    a = WideKid{(nd.c0 & kLeafBit) ? (kLeafBit | p) : nd.c0, nd.lo0, nd.hi0};
    b = WideKid{(nd.c1 & kLeafBit) ? (kLeafBit | (p + 1)) : nd.c1, nd.lo1, nd.hi1};
}

// Slot i: start from binary node i's two children; twice, replace the
// internal child of largest surface area (ties: the lower slot) by its two
// children, keeping the left-to-right leaf order. The area is summed in the
// fixed order dx dy + dy dz + dz dx (the oracle does the same), so the
// regrouping, and with it every slot, is deterministic.
__global__ void __launch_bounds__(kWideThreads)
    k_wide_collapse(const mlbvh_internal_node* __restrict__ nodes, uint32_t nInternal, mlbvh_wnode* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInternal) return;
    WideKid kid[4];
    binary_children(nodes, i, kid[0], kid[1]);
    kid[2].name = kid[3].name = kWideEmpty;
    kid[2].lo = kid[2].hi = kid[3].lo = kid[3].hi = mk(0.0f, 0.0f, 0.0f);
    int count = 2;
#pragma unroll
    for (int round = 0; round < 2; ++round) {
        int pick = -1;
        float best = 0.0f;
#pragma unroll
        for (int k = 0; k < 3 + round; ++k)
            if (k < count && !(kid[k].name & kLeafBit)) {
                const float a = half_area(kid[k].lo, kid[k].hi);
                if (pick < 0 || a > best) {
                    pick = k;
                    best = a;
                }
            }
        if (pick >= 0) {
            WideKid a, b;
            uint32_t p = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k == pick) p = kid[k].name;
            binary_children(nodes, p, a, b);
            // kid[pick] becomes a, b; the kids after it move one slot up
            WideKid next[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                next[k] = k < pick ? kid[k] : k == pick ? a : k == pick + 1 ? b : kid[k > 0 ? k - 1 : 0];
#pragma unroll
            for (int k = 0; k < 4; ++k) kid[k] = next[k];
            ++count;
        }
    }
    float4* dst = reinterpret_cast<float4*>(out + i);
    dst[0] = make_float4(kid[0].lo.x, kid[1].lo.x, kid[2].lo.x, kid[3].lo.x);
    dst[1] = make_float4(kid[0].hi.x, kid[1].hi.x, kid[2].hi.x, kid[3].hi.x);
    dst[2] = make_float4(kid[0].lo.y, kid[1].lo.y, kid[2].lo.y, kid[3].lo.y);
    dst[3] = make_float4(kid[0].hi.y, kid[1].hi.y, kid[2].hi.y, kid[3].hi.y);
    dst[4] = make_float4(kid[0].lo.z, kid[1].lo.z, kid[2].lo.z, kid[3].lo.z);
    dst[5] = make_float4(kid[0].hi.z, kid[1].hi.z, kid[2].hi.z, kid[3].hi.z);
    reinterpret_cast<uint4*>(dst)[6] = make_uint4(kid[0].name, kid[1].name, kid[2].name, kid[3].name);
    reinterpret_cast<uint4*>(dst)[7] = make_uint4(0u, 0u, 0u, 0u);
}

// Quantises one axis of a slot: base, power-of-two scale 2^E and the codes
// of the children in `valid` (byte k of qlo / qhi). A lower code q satisfies
// base + 2^E (1 + q / 2^15) <= lo and an upper code >= hi, in exact
// arithmetic: every step rounds toward that side. E is the smallest exponent
// (>= -111, so that 2^(E-15) stays a normal number) whose codes fit 8 bits.
// An axis whose base would reach 2^60 or whose scale would exceed 2^59
// (coordinates beyond about 1e18) counts as not quantised.
__device__ __forceinline__ bool quantise_axis(const float lo[4], const float hi[4], uint32_t valid, float& base,
                                              float& scale, uint32_t& qlo, uint32_t& qhi)
{
    base = scale = 0.0f;
    qlo = qhi = 0u;
    float nlo = kFltMax, nhi = -kFltMax;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (valid & (1u << k)) {
            nlo = fminf(nlo, lo[k]);
            nhi = fmaxf(nhi, hi[k]);
        }
    if (!(isfinite(nlo) && isfinite(nhi) && nlo <= nhi)) return false;
    const float m = __fdiv_ru(__fsub_ru(nhi, nlo), 255.0f);  // >= extent / 255
    int e = -111;
    if (m > 0.0f) {
        int k;
        const float f = frexpf(m, &k);  // m = f 2^k, f in [0.5, 1)
        e = max(e, (f == 0.5f ? k - 1 : k) + 15);
    }
    for (; e <= 127; ++e) {
        scale = pow2f(e);
        base = __fsub_rd(nlo, scale);
        if (!isfinite(base)) return false;
        const float toCode = pow2f(15 - e);
        bool fits = true;
        qlo = qhi = 0u;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (valid & (1u << k)) {
                const float ql = floorf(__fmul_rd(__fsub_rd(__fsub_rd(lo[k], base), scale), toCode));
                const float qh = ceilf(__fmul_ru(__fsub_ru(__fsub_ru(hi[k], base), scale), toCode));
                if (!(qh <= 255.0f)) fits = false;
                qlo |= (uint32_t)fminf(fmaxf(ql, 0.0f), 255.0f) << (8 * k);
                qhi |= (uint32_t)fminf(fmaxf(qh, 0.0f), 255.0f) << (8 * k);
            }
        // the walks' FMA form relies on bases below 2^60 and scales of at most 2^59 (qwide_ray_fits)
        if (fits) return fabsf(base) < kQBaseLimit && e <= 59;
    }
    return false;
}

// One thread per slot: the FP32 slot's planes quantised axis by axis; a slot
// that cannot be quantised sets *status.
__global__ void __launch_bounds__(kWideThreads)
    k_wide_quantise(const mlbvh_wnode* __restrict__ wnodes, uint32_t nSlots, mlbvh_qwnode* __restrict__ out,
                    uint32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nSlots) return;
    const float4* p = reinterpret_cast<const float4*>(wnodes + i);
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(p + 6));
    uint32_t valid = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (wpick(ch, k) != kWideEmpty) valid |= 1u << k;
    float base[3], scale[3];
    uint32_t q[6];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float4 l = __ldg(p + 2 * a), h = __ldg(p + 2 * a + 1);
        const float lo[4] = {l.x, l.y, l.z, l.w}, hi[4] = {h.x, h.y, h.z, h.w};
        ok = quantise_axis(lo, hi, valid, base[a], scale[a], q[2 * a], q[2 * a + 1]) && ok;
    }
    if (!ok) atomicOr(status, 1u);
    float4* dst = reinterpret_cast<float4*>(out + i);
    dst[0] = make_float4(base[0], base[1], base[2], scale[0]);
    dst[1] = make_float4(scale[1], scale[2], __uint_as_float(q[0]), __uint_as_float(q[1]));
    dst[2] = make_float4(__uint_as_float(q[2]), __uint_as_float(q[3]), __uint_as_float(q[4]), __uint_as_float(q[5]));
    reinterpret_cast<uint4*>(dst)[3] = ch;
}

// One thread per ray, any-hit (wide_any_step) or closest-hit
// (wide_closest_step), over FP32 slots or (kQuant) quantised slots. counts
// (may be null): per ray, node visits, triangle tests and restarts at
// counts[i], counts[n + i], counts[2n + i]. status (quantised slots): nonzero
// sends every ray to the stack-free walk over the binary tree; so does a ray
// that qwide_ray_fits rejects.
template <bool kAny, bool kCount, bool kQuant, class Slot>
__global__ void __launch_bounds__(kWideTraceThreads)
    k_trace_wide(const Slot* __restrict__ slots, const uint32_t* __restrict__ status,
                 const mlbvh_internal_node* __restrict__ nodes, const mlbvh_node_index* __restrict__ rootPtr,
                 const float* __restrict__ tris, const mlbvh_qtri* __restrict__ leafTris,
                 const float4* __restrict__ rays, float4* __restrict__ hits, uint32_t n,
                 uint32_t* __restrict__ counts)
{
    using Entry = typename ReplayStack<kAny>::Entry;
    __shared__ Entry s_stack[kWideDepth][kWideTraceThreads];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
    const f3 ro = mk(a.x, a.y, a.z), rd = mk(b.x, b.y, b.z);
    HitRecord hit;
    hit.t = b.w;
    hit.u = 0.0f;
    hit.v = 0.0f;
    hit.ng = mk(0.0f, 0.0f, 0.0f);
    hit.tri = 0xFFFFFFFFu;
    const uint32_t root = __ldg(rootPtr);
    const f3 inv = inv_rd(rd);
    uint32_t nv = 0, nt = 0, nr = 0;
    uint32_t curr = (root & kLeafBit) ? kLeafBit : root, prev = kInvalid;
    int depth = 0;
    if (kQuant && (__ldg(status) != 0u || !qwide_ray_fits(ro, inv))) {
        curr = root;
        depth = -1;
    }
    for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps) {
        bool done;
        if constexpr (kAny)
            done = wide_any_step<kCount, kQuant>(curr, prev, depth, &s_stack[0][threadIdx.x], kWideTraceThreads, hit,
                                                 slots, nodes, tris, leafTris, root, ro, rd, inv, a.w, nv, nt, nr);
        else
            done = wide_closest_step<kCount, kQuant>(curr, prev, depth, &s_stack[0][threadIdx.x], kWideTraceThreads,
                                                     hit, slots, nodes, tris, leafTris, root, ro, rd, inv, a.w, nv,
                                                     nt, nr);
        if (done) break;
    }
    hits[2 * (size_t)i] = make_float4(hit.t, 0.0f, hit.u, hit.v);
    hits[2 * (size_t)i + 1] = make_float4(hit.ng.x, hit.ng.y, hit.ng.z, __uint_as_float(hit.tri));
    if (kCount) {
        counts[i] = nv;
        counts[n + i] = nt;
        counts[2 * (size_t)n + i] = nr;
    }
}

inline bool aligned128(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 127u) == 0; }

}  // namespace

mlbvh_status build_wide(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, uint32_t n,
                        mlbvh_wnode* dWide, cudaStream_t stream)
{
    if (n == 0) return fail(MLBVH_ERR_INVALID_ARG, "no triangles");
    if (n == 1) return MLBVH_OK;
    if (!dNodes || !dRoot || !dWide) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned32(dNodes) || !aligned16(dRoot) || !aligned128(dWide))
        return fail(MLBVH_ERR_INVALID_ARG, "nodes must be 32-byte and wide nodes 128-byte aligned");
    const uint32_t m = n - 1;
    k_wide_collapse<<<(m + kWideThreads - 1) / kWideThreads, kWideThreads, 0, stream>>>(dNodes, m, dWide);
    MLBVH_CHECK_LAUNCH("k_wide_collapse");
    return MLBVH_OK;
}

namespace {

template <bool kQuant, class Slot>
mlbvh_status launch_trace_wide(const Slot* dSlots, const uint32_t* dStatus, const mlbvh_internal_node* dNodes,
                               const mlbvh_node_index* dRoot, const mlbvh_triangle* dTris,
                               const mlbvh_qtri* dLeafTris, const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays,
                               int rayQuery, uint32_t* dCounts, cudaStream_t stream)
{
    if (nRays == 0) return MLBVH_OK;
    if (rayQuery != MLBVH_RAY_QUERY_ANY && rayQuery != MLBVH_RAY_QUERY_CLOSEST)
        return fail(MLBVH_ERR_INVALID_ARG, "rayQuery must be MLBVH_RAY_QUERY_CLOSEST or MLBVH_RAY_QUERY_ANY");
    if (!dRoot || !dTris || !dLeafTris || !dRays || !dHits || (kQuant && !dStatus))
        return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!(kQuant ? aligned32(dSlots) : aligned128(dSlots)) || !aligned32(dNodes) || !aligned16(dRoot) ||
        !aligned16(dTris) || !aligned16(dLeafTris) || !aligned16(dRays) || !aligned16(dHits) || !aligned16(dCounts) ||
        !aligned16(dStatus))
        return fail(MLBVH_ERR_INVALID_ARG,
                    "device pointers misaligned (wide slots 128 B, quantised slots and nodes 32 B, others 16 B)");
    if (nRays >= (1u << 30) && dCounts) return fail(MLBVH_ERR_INVALID_ARG, "nRays must be below 2^30 with counts");
    const unsigned blocks = (nRays + kWideTraceThreads - 1) / kWideTraceThreads;
    const float4* rays = reinterpret_cast<const float4*>(dRays);
    float4* hits = reinterpret_cast<float4*>(dHits);
    const float* tris = reinterpret_cast<const float*>(dTris);
    const bool any = rayQuery == MLBVH_RAY_QUERY_ANY;
    if (any && dCounts)
        k_trace_wide<true, true, kQuant><<<blocks, kWideTraceThreads, 0, stream>>>(
            dSlots, dStatus, dNodes, dRoot, tris, dLeafTris, rays, hits, nRays, dCounts);
    else if (any)
        k_trace_wide<true, false, kQuant><<<blocks, kWideTraceThreads, 0, stream>>>(
            dSlots, dStatus, dNodes, dRoot, tris, dLeafTris, rays, hits, nRays, nullptr);
    else if (dCounts)
        k_trace_wide<false, true, kQuant><<<blocks, kWideTraceThreads, 0, stream>>>(
            dSlots, dStatus, dNodes, dRoot, tris, dLeafTris, rays, hits, nRays, dCounts);
    else
        k_trace_wide<false, false, kQuant><<<blocks, kWideTraceThreads, 0, stream>>>(
            dSlots, dStatus, dNodes, dRoot, tris, dLeafTris, rays, hits, nRays, nullptr);
    MLBVH_CHECK_LAUNCH("k_trace_wide");
    return MLBVH_OK;
}

}  // namespace

mlbvh_status trace_wide(const mlbvh_wnode* dWide, const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                        const mlbvh_triangle* dTris, const mlbvh_qtri* dLeafTris, const mlbvh_ray* dRays,
                        mlbvh_hit* dHits, uint32_t nRays, int rayQuery, uint32_t* dCounts, cudaStream_t stream)
{
    return launch_trace_wide<false>(dWide, static_cast<const uint32_t*>(nullptr), dNodes, dRoot, dTris, dLeafTris,
                                    dRays, dHits, nRays, rayQuery, dCounts, stream);
}

mlbvh_status trace_wide_quantised(const mlbvh_qwnode* dQWide, const uint32_t* dStatus,
                                  const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                                  const mlbvh_triangle* dTris, const mlbvh_qtri* dLeafTris, const mlbvh_ray* dRays,
                                  mlbvh_hit* dHits, uint32_t nRays, int rayQuery, uint32_t* dCounts,
                                  cudaStream_t stream)
{
    return launch_trace_wide<true>(dQWide, dStatus, dNodes, dRoot, dTris, dLeafTris, dRays, dHits, nRays, rayQuery,
                                   dCounts, stream);
}

mlbvh_status quantise_wide(const mlbvh_wnode* dWide, uint32_t n, mlbvh_qwnode* dQWide, uint32_t* dStatus,
                           cudaStream_t stream)
{
    if (n == 0) return fail(MLBVH_ERR_INVALID_ARG, "no triangles");
    if (!dStatus) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dStatus)) return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    cudaError_t e = cudaMemsetAsync(dStatus, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    if (n == 1) return MLBVH_OK;
    if (!dWide || !dQWide) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned128(dWide) || !aligned32(dQWide))
        return fail(MLBVH_ERR_INVALID_ARG, "wide slots must be 128-byte and quantised slots 32-byte aligned");
    const uint32_t m = n - 1;
    k_wide_quantise<<<(m + kWideThreads - 1) / kWideThreads, kWideThreads, 0, stream>>>(dWide, m, dQWide, dStatus);
    MLBVH_CHECK_LAUNCH("k_wide_quantise");
    return MLBVH_OK;
}

}  // namespace mlbvh
