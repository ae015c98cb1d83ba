// Ray queries over the reference node layout: one thread per ray.
//
// Replaces the per-ray device calls of intersect_stackfree (minimum_lbvh.h:
// 981-1061), intersect_escape_link (:1063-1137) and intersect_stackfull
// (:912-973) with a single launch; MLBVH_TRAVERSAL_REPLAY gives
// intersect_stackfree's Hit records through the replay walk. Rays and hits move as 2 x 16-byte vectors,
// nodes as 4 x 16-byte read-only loads.
#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {

namespace {

// Threads per CTA: a CTA holds its slot until its longest ray is done, so
// smaller CTAs free slots sooner (measured on 1M camera rays of the 4M soup,
// replay / stack-free walk: 128 threads 0.552 / 0.689 ms, 64 0.505 / 0.690,
// 32 0.522 / 0.719; on 1M random rays 1.38 / 1.61, 1.275 / 1.58, 1.29 / 1.65).
// Build-time override for sweeps: -DMLBVH_TRACE_THREADS.
#ifndef MLBVH_TRACE_THREADS
#define MLBVH_TRACE_THREADS 64
#endif
constexpr int kTraceThreads = MLBVH_TRACE_THREADS;

constexpr int kReplayDepth = 16;  // stack entries per ray of the replay walk

template <int kMode, bool kAny>
__global__ void __launch_bounds__(kTraceThreads)
    k_trace(const mlbvh_internal_node* __restrict__ nodes, const mlbvh_node_index* __restrict__ rootPtr,
            const float* __restrict__ tris, const float4* __restrict__ rays, float4* __restrict__ hits, uint32_t n)
{
    __shared__ typename ReplayStack<kAny>::Entry s_stack[kMode == MLBVH_TRAVERSAL_REPLAY ? kReplayDepth : 1]
                                                        [kTraceThreads];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
    const f3 ro = mk(a.x, a.y, a.z), rd = mk(b.x, b.y, b.z);
    const float tmin = a.w;
    HitRecord hit;
    hit.t = b.w;
    hit.u = 0.0f;
    hit.v = 0.0f;
    hit.ng = mk(0.0f, 0.0f, 0.0f);
    hit.tri = 0xFFFFFFFFu;
    const uint32_t root = __ldg(rootPtr);
    const f3 inv = inv_rd(rd);
    if (kMode == MLBVH_TRAVERSAL_ESCAPE_LINK) {
        trace_escape<kAny>(hit, nodes, tris, root, ro, rd, inv, tmin);
    } else if (kMode == MLBVH_TRAVERSAL_REPLAY) {
        uint32_t curr = root, prev = kInvalid, nv = 0, nt = 0;
        int depth = 0;
        for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
            if (stackfree_replay_step<kAny, false, kReplayDepth>(curr, prev, depth, &s_stack[0][threadIdx.x],
                                                                 kTraceThreads, hit, nodes, tris, ro, rd, inv, tmin,
                                                                 nv, nt))
                break;
    } else if (kMode == MLBVH_TRAVERSAL_STACKFULL) {
        uint32_t stack[64];
        trace_stackfull(hit, nodes, tris, root, ro, rd, inv, tmin, stack, 64);
    } else {
        trace_stackfree<kAny, false, true>(hit, nodes, tris, root, ro, rd, inv, tmin);
    }
    hits[2 * (size_t)i] = make_float4(hit.t, 0.0f, hit.u, hit.v);
    hits[2 * (size_t)i + 1] = make_float4(hit.ng.x, hit.ng.y, hit.ng.z, __uint_as_float(hit.tri));
}

}  // namespace

mlbvh_status trace(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, const mlbvh_triangle* dTris,
                   const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays, int rayQuery, int traversal,
                   cudaStream_t stream)
{
    if (nRays == 0) return MLBVH_OK;
    if (!dRoot || !dTris || !dRays || !dHits) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned32(dNodes) || !aligned16(dRoot) || !aligned16(dTris) || !aligned16(dRays) || !aligned16(dHits))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned (node arrays 32-byte)");
    if (rayQuery != MLBVH_RAY_QUERY_CLOSEST && rayQuery != MLBVH_RAY_QUERY_ANY)
        return fail(MLBVH_ERR_INVALID_ARG, "rayQuery must be MLBVH_RAY_QUERY_CLOSEST or MLBVH_RAY_QUERY_ANY");
    const bool any = rayQuery == MLBVH_RAY_QUERY_ANY;
    const unsigned blocks = (nRays + kTraceThreads - 1) / kTraceThreads;
    const float* tris = reinterpret_cast<const float*>(dTris);
    const float4* rays = reinterpret_cast<const float4*>(dRays);
    float4* hits = reinterpret_cast<float4*>(dHits);
    switch (traversal) {
    case MLBVH_TRAVERSAL_STACKFREE:
        if (any)
            k_trace<MLBVH_TRAVERSAL_STACKFREE, true><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        else
            k_trace<MLBVH_TRAVERSAL_STACKFREE, false><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        break;
    case MLBVH_TRAVERSAL_ESCAPE_LINK:
        if (any)
            k_trace<MLBVH_TRAVERSAL_ESCAPE_LINK, true><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        else
            k_trace<MLBVH_TRAVERSAL_ESCAPE_LINK, false><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        break;
    case MLBVH_TRAVERSAL_REPLAY:
        if (any)
            k_trace<MLBVH_TRAVERSAL_REPLAY, true><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        else
            k_trace<MLBVH_TRAVERSAL_REPLAY, false><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        break;
    case MLBVH_TRAVERSAL_STACKFULL:
        k_trace<MLBVH_TRAVERSAL_STACKFULL, false><<<blocks, kTraceThreads, 0, stream>>>(dNodes, dRoot, tris, rays, hits, nRays);
        break;
    default:
        return fail(MLBVH_ERR_INVALID_ARG, "unknown traversal");
    }
    MLBVH_CHECK_LAUNCH("k_trace");
    return MLBVH_OK;
}

}  // namespace mlbvh
