// The quantised tree: 32-byte nodes with 8-bit child boxes (no reference
// counterpart), made from a tree built by build.cu, and its ray query.
//
// k_quantise: one thread per internal node. Per axis the node stores a base b
// and a scale 2^E; code q stands for the plane b + 2^E (1 + q / 2^15) (the
// form of the quantised 4-wide slots, decoded with one byte permute), lower
// planes rounded down and upper ones up in exact arithmetic. E is the
// smallest exponent in [EB - 31, EB] whose codes fit 8 bits, stored as the
// 5-bit code k = EB - E, where EB (tree_scale_exponent) is chosen from the
// root box so that every node's codes fit at E = EB. Leaves move to sorted
// (leaf) order: a left leaf child of node j is leaf j, a right leaf child is
// leaf j+1 (node j splits leaves j and j+1).
#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {

namespace {

constexpr int kQuantiseThreads = 256;
// Threads per CTA of k_trace_quantised: a CTA holds its slot until its longest
// ray is done (1M camera / random rays of the 4M soup, replay walk: 128 threads
// 0.599 / 1.59 ms, 64 0.578 / 1.52, 32 0.604 / 1.57). Build-time override for
// sweeps: -DMLBVH_QTRACE_THREADS.
#ifndef MLBVH_QTRACE_THREADS
#define MLBVH_QTRACE_THREADS 64
#endif
constexpr int kTraceThreads = MLBVH_QTRACE_THREADS;

__device__ __forceinline__ void leaf_box(const float* __restrict__ tris, uint32_t t, f3& lo, f3& hi)
{
    f3 v0, v1, v2;
    load_triangle(tris, t, v0, v1, v2);
    lo = smin3(smin3(smin3(mk(kFltMax, kFltMax, kFltMax), v0), v1), v2);
    hi = smax3(smax3(smax3(mk(-kFltMax, -kFltMax, -kFltMax), v0), v1), v2);
}

// ceil(log2(x)) for finite x > 0; -150 for 0
__device__ __forceinline__ int ceil_log2f(float x)
{
    if (!(x > 0.0f)) return -150;
    int k;
    const float f = frexpf(x, &k);  // x = f 2^k, f in [0.5, 1)
    return f == 0.5f ? k - 1 : k;
}

// The tree's scale exponent EB from the root box's largest extent D and
// largest coordinate magnitude R: EB = max(ceil(log2 D) + 9, ceil(log2 R) -
// 13, -111). At E = EB a code's extent term stays below 64 steps of
// 2^(E - 15) and the rounding of the base (b = nlo - 2^E rounded down, at
// most R + 2^E in size) below 33 steps, so every node's codes fit 8 bits.
// finite = false for a non-finite root box or an EB above 127.
__device__ __forceinline__ int tree_scale_exponent(const mlbvh_internal_node* __restrict__ nodes,
                                                   const float* __restrict__ tris, uint32_t root, bool& finite)
{
    f3 lo, hi;
    if (root & kLeafBit) {
        leaf_box(tris, root & ~kLeafBit, lo, hi);
    } else {
        const NodeView nd = load_node(nodes, root);
        lo = smin3(nd.lo0, nd.lo1);
        hi = smax3(nd.hi0, nd.hi1);
    }
    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    float d = 0.0f, r = 0.0f;
    finite = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!(isfinite(l[a]) && isfinite(h[a]))) finite = false;
        d = fmaxf(d, __fsub_ru(h[a], l[a]));
        r = fmaxf(r, fmaxf(fabsf(l[a]), fabsf(h[a])));
    }
    if (!finite || !isfinite(d)) {
        finite = false;
        return 0;
    }
    const int e = max(max(ceil_log2f(d) + 9, ceil_log2f(r) - 13), -111);
    finite = e <= 127;  // a scale 2^E must be a float
    return finite ? e : 0;
}

// One axis of a node: base, exponent E in [eLo, eHi] and the four codes
// (byte 0 child 0 lower, 1 child 0 upper, 2 child 1 lower, 3 child 1 upper)
// with base + 2^E (1 + q / 2^15) <= the lower and >= the upper plane in exact
// arithmetic (every step rounds toward that side), E the smallest in range
// whose codes fit. false when no E in range fits or a plane is not finite
// (base 0, E = eHi and codes 0xFF00FF00 then).
__device__ __forceinline__ bool quantise_axis2(const float lo[2], const float hi[2], int eLo, int eHi, float& base,
                                               int& E, uint32_t& codes)
{
    base = 0.0f;
    E = eHi;
    codes = 0xFF00FF00u;
    const float nlo = fminf(lo[0], lo[1]), nhi = fmaxf(hi[0], hi[1]);
    if (!(isfinite(lo[0]) && isfinite(lo[1]) && isfinite(hi[0]) && isfinite(hi[1]) && nlo <= nhi)) return false;
    const float m = __fdiv_ru(__fsub_ru(nhi, nlo), 255.0f);  // >= extent / 255
    int e = -111;
    if (m > 0.0f) e = max(e, ceil_log2f(m) + 15);
    e = max(e, eLo);
    for (; e <= eHi; ++e) {
        const float sc = pow2f(e);
        const float b = __fsub_rd(nlo, sc);
        if (!isfinite(b)) return false;
        const float toCode = pow2f(15 - e);
        bool fits = true;
        uint32_t q = 0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const float ql = floorf(__fmul_rd(__fsub_rd(__fsub_rd(lo[c], b), sc), toCode));
            const float qh = ceilf(__fmul_ru(__fsub_ru(__fsub_ru(hi[c], b), sc), toCode));
            if (!(qh <= 255.0f)) fits = false;
            q |= (uint32_t)fminf(fmaxf(ql, 0.0f), 255.0f) << (16 * c);
            q |= (uint32_t)fminf(fmaxf(qh, 0.0f), 255.0f) << (16 * c + 8);
        }
        if (fits) {
            base = b;
            E = e;
            codes = q;
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ void write_qtri(mlbvh_qtri* __restrict__ qtris, uint32_t pos, const float* __restrict__ tris,
                                           uint32_t t)
{
    const float* src = tris + 9ull * t;
    float4* dst = reinterpret_cast<float4*>(qtris + pos);
    dst[0] = make_float4(__ldg(src + 0), __ldg(src + 1), __ldg(src + 2), __ldg(src + 3));
    dst[1] = make_float4(__ldg(src + 4), __ldg(src + 5), __ldg(src + 6), __ldg(src + 7));
    dst[2] = make_float4(__ldg(src + 8), __uint_as_float(t), 0.0f, 0.0f);
}

// header->status must be 0 before the launch (the threads OR bits into it):
// bit 0 a base of 2^60 or more or a scale above 2^59, bit 1 a non-finite
// coordinate (or a scale exponent above 127).
__global__ void __launch_bounds__(kQuantiseThreads)
    k_quantise(const mlbvh_internal_node* __restrict__ nodes, const mlbvh_node_index* __restrict__ rootPtr,
               const float* __restrict__ tris, uint32_t n, mlbvh_qnode* __restrict__ qnodes,
               uint32_t* __restrict__ parents, mlbvh_qtri* __restrict__ qtris, mlbvh_qheader* __restrict__ header)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t root = __ldg(rootPtr);
    bool finite;
    const int eb = tree_scale_exponent(nodes, tris, root, finite);
    if (i == 0) {
        header->root = (root & kLeafBit) ? kLeafBit : root;
        header->eBase = eb;
        header->nTriangles = n;
        if (!finite) atomicOr(&header->status, 2u);
        if (root & kLeafBit) write_qtri(qtris, 0, tris, root & ~kLeafBit);
    }
    if (i + 1 >= n) return;
    const NodeView nd = load_node(nodes, i);
    const float lo0[3] = {nd.lo0.x, nd.lo0.y, nd.lo0.z}, hi0[3] = {nd.hi0.x, nd.hi0.y, nd.hi0.z};
    const float lo1[3] = {nd.lo1.x, nd.lo1.y, nd.lo1.z}, hi1[3] = {nd.hi1.x, nd.hi1.y, nd.hi1.z};
    const int eLo = max(-111, eb - 31);
    uint32_t code = 0, status = 0, q[3];
    float base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float l2[2] = {lo0[a], lo1[a]}, h2[2] = {hi0[a], hi1[a]};
        int e = eb;
        base[a] = 0.0f;
        q[a] = 0xFF00FF00u;
        if (!finite || !quantise_axis2(l2, h2, eLo, eb, base[a], e, q[a]))
            status |= 2u;
        else if (!(fabsf(base[a]) < kQBaseLimit && e <= 59))
            status |= 1u;
        code |= (uint32_t)(eb - e) << (5 * a);
    }
    if (status) atomicOr(&header->status, status);
    uint32_t c0 = nd.c0, c1 = nd.c1;
    if (c0 & kLeafBit) {
        write_qtri(qtris, i, tris, c0 & ~kLeafBit);
        c0 = kLeafBit | i;
    }
    if (c1 & kLeafBit) {
        write_qtri(qtris, i + 1, tris, c1 & ~kLeafBit);
        c1 = kLeafBit | (i + 1);
    }
    c0 |= (code & 0xFFu) << 23;
    c1 |= ((code >> 8) & 0x7Fu) << 23;
    float4* dst = reinterpret_cast<float4*>(qnodes + i);
    dst[0] = make_float4(base[0], base[1], base[2], __uint_as_float(q[0]));
    dst[1] = make_float4(__uint_as_float(q[1]), __uint_as_float(q[2]), __uint_as_float(c0), __uint_as_float(c1));
    parents[i] = nd.parent;
}

// Leaf-ordered triangles alone (the qtris of k_quantise): one thread per
// internal node j writes its leaf children, leaf j (left) and j + 1 (right).
__global__ void __launch_bounds__(kQuantiseThreads)
    k_leaf_tris(const mlbvh_internal_node* __restrict__ nodes, const mlbvh_node_index* __restrict__ rootPtr,
                const float* __restrict__ tris, uint32_t n, mlbvh_qtri* __restrict__ leafTris)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (n == 1) {
        if (j == 0) write_qtri(leafTris, 0, tris, __ldg(rootPtr) & ~kLeafBit);
        return;
    }
    if (j + 1 >= n) return;
    const uint32_t c0 = __ldg(&nodes[j].children[0]), c1 = __ldg(&nodes[j].children[1]);
    if (c0 & kLeafBit) write_qtri(leafTris, j, tris, c0 & ~kLeafBit);
    if (c1 & kLeafBit) write_qtri(leafTris, j + 1, tris, c1 & ~kLeafBit);
}

// One thread per ray. kDepth = 0: the stack-free walk (trace_quantised);
// otherwise the replay walk with a kDepth-entry stack per thread in shared
// memory (quantised_replay_step), which returns the same Hit records.
// counts (may be null): per ray, internal-node visits, triangle tests and
// parent loads at counts[i], counts[n + i], counts[2n + i].
template <bool kAny, int kDepth, bool kCount>
__global__ void __launch_bounds__(kTraceThreads)
    k_trace_quantised(const mlbvh_qnode* __restrict__ qnodes, const uint32_t* __restrict__ parents,
                      const mlbvh_qtri* __restrict__ qtris, const mlbvh_qheader* __restrict__ header,
                      const float4* __restrict__ rays, float4* __restrict__ hits, uint32_t n,
                      uint32_t* __restrict__ counts)
{
    __shared__ typename ReplayStack<kAny>::Entry s_stack[kDepth > 0 ? kDepth : 1][kTraceThreads];
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
    const uint32_t root = __ldg(&header->root);
    const f3 inv = inv_rd(rd);
    const QParams qp = qparams(header, ro, inv);
    uint32_t nv = 0, nt = 0, nu = 0;
    if (kDepth == 0) {
        trace_quantised<kAny, kCount>(hit, qnodes, parents, qtris, root, qp, ro, rd, inv, a.w, &nv, &nt, &nu);
    } else {
        uint32_t curr = root, prev = kInvalid;
        int depth = 0;
        for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
            if (quantised_replay_step<kAny, kCount, kDepth>(curr, prev, depth, &s_stack[0][threadIdx.x],
                                                            kTraceThreads, hit, qnodes, parents, qtris, qp, ro, rd,
                                                            inv, a.w, nv, nt, nu))
                break;
    }
    hits[2 * (size_t)i] = make_float4(hit.t, 0.0f, hit.u, hit.v);
    hits[2 * (size_t)i + 1] = make_float4(hit.ng.x, hit.ng.y, hit.ng.z, __uint_as_float(hit.tri));
    if (kCount) {
        counts[i] = nv;
        counts[n + i] = nt;
        counts[2 * (size_t)n + i] = nu;
    }
}

template <bool kAny, int kDepth>
void launch_trace_quantised(unsigned blocks, cudaStream_t stream, const mlbvh_qnode* q, const uint32_t* p,
                            const mlbvh_qtri* t, const mlbvh_qheader* h, const float4* rays, float4* hits, uint32_t n,
                            uint32_t* counts)
{
    if (counts)
        k_trace_quantised<kAny, kDepth, true><<<blocks, kTraceThreads, 0, stream>>>(q, p, t, h, rays, hits, n, counts);
    else
        k_trace_quantised<kAny, kDepth, false><<<blocks, kTraceThreads, 0, stream>>>(q, p, t, h, rays, hits, n,
                                                                                    nullptr);
}

template <bool kAny>
void launch_trace_quantised_depth(int depth, unsigned blocks, cudaStream_t stream, const mlbvh_qnode* q,
                                  const uint32_t* p, const mlbvh_qtri* t, const mlbvh_qheader* h, const float4* rays,
                                  float4* hits, uint32_t n, uint32_t* counts)
{
    switch (depth) {
    case 0: launch_trace_quantised<kAny, 0>(blocks, stream, q, p, t, h, rays, hits, n, counts); break;
    case 1: launch_trace_quantised<kAny, 1>(blocks, stream, q, p, t, h, rays, hits, n, counts); break;
    case 4: launch_trace_quantised<kAny, 4>(blocks, stream, q, p, t, h, rays, hits, n, counts); break;
    default: launch_trace_quantised<kAny, 16>(blocks, stream, q, p, t, h, rays, hits, n, counts); break;
    }
}

}  // namespace

mlbvh_status quantise(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, const mlbvh_triangle* dTris,
                      uint32_t n, mlbvh_qnode* dQNodes, uint32_t* dQParents, mlbvh_qtri* dQTris,
                      mlbvh_qheader* dQHeader, cudaStream_t stream)
{
    if (n == 0 || n > kQMaxLeaves) return fail(MLBVH_ERR_INVALID_ARG, "nTriangles must be in [1, 2^23]");
    if (!dRoot || !dTris || !dQTris || !dQHeader || (n > 1 && (!dNodes || !dQNodes || !dQParents)))
        return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dNodes) || !aligned16(dRoot) || !aligned16(dTris) || !aligned32(dQNodes) || !aligned16(dQParents) ||
        !aligned16(dQTris) || !aligned16(dQHeader))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned (node arrays 32-byte)");
    const uint32_t threads = n > 1 ? n - 1 : 1;
    const cudaError_t e = cudaMemsetAsync(&dQHeader->status, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    k_quantise<<<(threads + kQuantiseThreads - 1) / kQuantiseThreads, kQuantiseThreads, 0, stream>>>(
        dNodes, dRoot, reinterpret_cast<const float*>(dTris), n, dQNodes, dQParents, dQTris, dQHeader);
    MLBVH_CHECK_LAUNCH("k_quantise");
    return MLBVH_OK;
}

mlbvh_status leaf_triangles(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                            const mlbvh_triangle* dTris, uint32_t n, mlbvh_qtri* dLeafTris, cudaStream_t stream)
{
    if (n == 0 || n >= (1u << 31)) return fail(MLBVH_ERR_INVALID_ARG, "nTriangles must be in [1, 2^31)");
    if (!dRoot || !dTris || !dLeafTris || (n > 1 && !dNodes)) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dNodes) || !aligned16(dRoot) || !aligned16(dTris) || !aligned16(dLeafTris))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    const uint32_t threads = n > 1 ? n - 1 : 1;
    k_leaf_tris<<<(threads + kQuantiseThreads - 1) / kQuantiseThreads, kQuantiseThreads, 0, stream>>>(
        dNodes, dRoot, reinterpret_cast<const float*>(dTris), n, dLeafTris);
    MLBVH_CHECK_LAUNCH("k_leaf_tris");
    return MLBVH_OK;
}

mlbvh_status trace_quantised(const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                             const mlbvh_qheader* dQHeader, const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays,
                             int rayQuery, int stackDepth, uint32_t* dCounts, cudaStream_t stream)
{
    if (nRays == 0) return MLBVH_OK;
    if (!dQTris || !dQHeader || !dRays || !dHits) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned32(dQNodes) || !aligned16(dQParents) || !aligned16(dQTris) || !aligned16(dQHeader) ||
        !aligned16(dRays) || !aligned16(dHits) || !aligned16(dCounts))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (rayQuery != MLBVH_RAY_QUERY_CLOSEST && rayQuery != MLBVH_RAY_QUERY_ANY)
        return fail(MLBVH_ERR_INVALID_ARG, "rayQuery must be MLBVH_RAY_QUERY_CLOSEST or MLBVH_RAY_QUERY_ANY");
    if (stackDepth != 0 && stackDepth != 1 && stackDepth != 4 && stackDepth != 16)
        return fail(MLBVH_ERR_INVALID_ARG, "stackDepth must be 0, 1, 4 or 16");
    if (nRays >= (1u << 30) && dCounts) return fail(MLBVH_ERR_INVALID_ARG, "nRays must be below 2^30 with counts");
    const unsigned blocks = (nRays + kTraceThreads - 1) / kTraceThreads;
    const float4* rays = reinterpret_cast<const float4*>(dRays);
    float4* hits = reinterpret_cast<float4*>(dHits);
    if (rayQuery == MLBVH_RAY_QUERY_ANY)
        launch_trace_quantised_depth<true>(stackDepth, blocks, stream, dQNodes, dQParents, dQTris, dQHeader, rays, hits,
                                           nRays, dCounts);
    else
        launch_trace_quantised_depth<false>(stackDepth, blocks, stream, dQNodes, dQParents, dQTris, dQHeader, rays,
                                            hits, nRays, dCounts);
    MLBVH_CHECK_LAUNCH("k_trace_quantised");
    return MLBVH_OK;
}

}  // namespace mlbvh
