// minimum_lbvh.h — C++ host and device API of minimumlbvh_b200 with the
// reference's names, types and call shapes (MinimumLBVH's minimum_lbvh.h),
// built on the C ABI of mlbvh.h. Code written against the reference's
// BVHGPUBuilder / OnesweepSort / intersect_* compiles against this header:
//
//   reference (minimum_lbvh.h)                        here
//   Triangle, AABB, NodeIndex, InternalNode,          same names, same bytes
//     IndexedMorton, Hit  (:207-282, 502-506, 890-896)  (static_asserts below)
//   BUILD_OPTION, RAY_QUERY (:42-46, 975-979)         same enumerators
//   invRd, hashPCG (:898-909)                         same (device)
//   intersect_stackfree / _escape_link / _stackfull   same signatures (device),
//     (:981, :1063, :912)                               one shared implementation
//                                                       with the library kernels
//   BVHGPUBuilder(kernelPath, includeDir) (:729)      same; the paths are ignored
//   BVHGPUBuilder::build(tris, n, opt, sorter, stream) same; calls mlbvh_build
//     (:783)
//   m_internals, m_rootNode, m_sceneAABB,             same members (device
//     m_nTriangles (:876-884)                           pointers), same meaning
//   tinyhiponesweep::OnesweepSort(device) (:575)      owns the build scratch
//
// Differences, by design: build() neither prints its time nor synchronises
// (the reference's DeviceStopwatch does both, :785-870); errors abort with the
// library's message, as the reference's host asserts abort (:23); the query
// functions take rays with t in [0, hit->t] exactly as the reference's.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "mlbvh.h"
#ifdef __CUDACC__
#include "mlbvh_device.cuh"
#endif

#define MINIMUM_LBVH_FLT_MAX 3.402823466e+38F

namespace minimum_lbvh {

enum BUILD_OPTION { BUILD_OPTION_USE_NORMAL = 1, BUILD_OPTION_CPU_PARALLEL = 2 };
enum RAY_QUERY { RAY_QUERY_CLOSEST, RAY_QUERY_ANY };

struct Triangle {
    float3 vs[3];
};
struct AABB {
    float3 lower;
    float3 upper;
};
struct NodeIndex {
    __host__ __device__ NodeIndex() : m_index(0), m_isLeaf(0) {}
    __host__ __device__ NodeIndex(uint32_t index, bool isLeaf) : m_index(index), m_isLeaf(isLeaf) {}
    uint32_t m_index : 31;
    uint32_t m_isLeaf : 1;
    __host__ __device__ static NodeIndex invalid() { return NodeIndex(0x7FFFFFFF, false); }
};
__host__ __device__ inline bool operator==(NodeIndex a, NodeIndex b)
{
    return a.m_index == b.m_index && a.m_isLeaf == b.m_isLeaf;
}
__host__ __device__ inline bool operator!=(NodeIndex a, NodeIndex b) { return !(a == b); }
struct InternalNode {
    NodeIndex children[2];
    AABB aabbs[2];
    NodeIndex parent;
    uint32_t context;
};
struct IndexedMorton {
    uint32_t morton;
    uint32_t index;
};
struct Hit {
    float t = MINIMUM_LBVH_FLT_MAX;
    float2 uv = {};
    float3 ng = {};
    uint32_t triangleIndex = 0xFFFFFFFF;
};

static_assert(sizeof(Triangle) == sizeof(mlbvh_triangle) && sizeof(Triangle) == 36, "Triangle layout");
static_assert(sizeof(AABB) == sizeof(mlbvh_aabb) && sizeof(AABB) == 24, "AABB layout");
static_assert(sizeof(NodeIndex) == 4, "NodeIndex layout");
static_assert(sizeof(InternalNode) == sizeof(mlbvh_internal_node) && sizeof(InternalNode) == 64, "InternalNode layout");
static_assert(sizeof(Hit) == sizeof(mlbvh_hit) && sizeof(Hit) == 32, "Hit layout");
static_assert(offsetof(Hit, uv) == 8 && offsetof(Hit, ng) == 16 && offsetof(Hit, triangleIndex) == 28, "Hit offsets");

#ifdef __CUDACC__
// ------------------------------------------------------------ device queries
__device__ inline float3 invRd(float3 rd)
{
    mlbvh::f3 r = mlbvh::inv_rd(mlbvh::mk(rd.x, rd.y, rd.z));
    return make_float3(r.x, r.y, r.z);
}
__device__ inline uint32_t hashPCG(uint32_t v) { return mlbvh::hash_pcg(v); }

namespace detail {
__device__ inline mlbvh::HitRecord to_record(const Hit* h)
{
    mlbvh::HitRecord r;
    r.t = h->t;
    r.u = h->uv.x;
    r.v = h->uv.y;
    r.ng = mlbvh::mk(h->ng.x, h->ng.y, h->ng.z);
    r.tri = h->triangleIndex;
    return r;
}
__device__ inline void from_record(Hit* h, const mlbvh::HitRecord& r)
{
    h->t = r.t;
    h->uv = make_float2(r.u, r.v);
    h->ng = make_float3(r.ng.x, r.ng.y, r.ng.z);
    h->triangleIndex = r.tri;
}
__device__ inline uint32_t bits(NodeIndex n) { return n.m_index | (n.m_isLeaf ? 0x80000000u : 0u); }
__device__ inline mlbvh::f3 f(float3 v) { return mlbvh::mk(v.x, v.y, v.z); }
}  // namespace detail

// intersect_stackfree (minimum_lbvh.h:981)
__device__ inline void intersect_stackfree(Hit* hit, const InternalNode* nodes, const Triangle* triangles,
                                           NodeIndex node, float3 ro, float3 rd, float3 one_over_rd,
                                           RAY_QUERY rayQuery = RAY_QUERY_CLOSEST)
{
    mlbvh::HitRecord r = detail::to_record(hit);
    auto n = reinterpret_cast<const mlbvh_internal_node*>(nodes);
    auto t = reinterpret_cast<const float*>(triangles);
    if (rayQuery == RAY_QUERY_ANY)
        mlbvh::trace_stackfree<true>(r, n, t, detail::bits(node), detail::f(ro), detail::f(rd), detail::f(one_over_rd),
                                     0.0f);
    else
        mlbvh::trace_stackfree<false>(r, n, t, detail::bits(node), detail::f(ro), detail::f(rd),
                                      detail::f(one_over_rd), 0.0f);
    detail::from_record(hit, r);
}

// intersect_escape_link (minimum_lbvh.h:1063)
__device__ inline void intersect_escape_link(Hit* hit, const InternalNode* nodes, const Triangle* triangles,
                                             NodeIndex node, float3 ro, float3 rd, float3 one_over_rd,
                                             RAY_QUERY rayQuery = RAY_QUERY_CLOSEST)
{
    mlbvh::HitRecord r = detail::to_record(hit);
    auto n = reinterpret_cast<const mlbvh_internal_node*>(nodes);
    auto t = reinterpret_cast<const float*>(triangles);
    if (rayQuery == RAY_QUERY_ANY)
        mlbvh::trace_escape<true>(r, n, t, detail::bits(node), detail::f(ro), detail::f(rd), detail::f(one_over_rd),
                                  0.0f);
    else
        mlbvh::trace_escape<false>(r, n, t, detail::bits(node), detail::f(ro), detail::f(rd), detail::f(one_over_rd),
                                   0.0f);
    detail::from_record(hit, r);
}

// intersect_stackfull (minimum_lbvh.h:912): the caller's stack must hold the
// tree depth; `capacity` bounds it here (the reference does not check).
__device__ inline void intersect_stackfull(Hit* hit, const InternalNode* nodes, const Triangle* triangles,
                                           NodeIndex rootNode, float3 ro, float3 rd, float3 one_over_rd,
                                           NodeIndex* stack, int capacity = 1 << 30)
{
    mlbvh::HitRecord r = detail::to_record(hit);
    mlbvh::trace_stackfull(r, reinterpret_cast<const mlbvh_internal_node*>(nodes),
                           reinterpret_cast<const float*>(triangles), detail::bits(rootNode), detail::f(ro),
                           detail::f(rd), detail::f(one_over_rd), 0.0f, reinterpret_cast<uint32_t*>(stack), capacity);
    detail::from_record(hit, r);
}
#endif  // __CUDACC__

namespace detail {
inline void check(mlbvh_status s, const char* what)
{
    if (s != MLBVH_OK) {
        std::fprintf(stderr, "minimum_lbvh: %s failed (%d): %s\n", what, (int)s, mlbvh_last_error_string());
        std::abort();
    }
}
inline void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "minimum_lbvh: %s failed: %s\n", what, cudaGetErrorString(e));
        std::abort();
    }
}
}  // namespace detail

}  // namespace minimum_lbvh

namespace tinyhiponesweep {

// OnesweepSort (tinyhiponesweep.h:572-748): here the owner of the build's
// device scratch (histograms, look-back words, key/index ping-pong buffers),
// grown on demand and freed with the object.
class OnesweepSort {
public:
    explicit OnesweepSort(int device = 0) : m_device(device) {}
    ~OnesweepSort()
    {
        if (m_scratch) cudaFree(m_scratch);
    }
    OnesweepSort(const OnesweepSort&) = delete;
    void operator=(const OnesweepSort&) = delete;

    void* reserve(size_t bytes, cudaStream_t stream)
    {
        if (bytes > m_bytes) {
            if (m_scratch) minimum_lbvh::detail::check(cudaFreeAsync(m_scratch, stream), "cudaFreeAsync");
            minimum_lbvh::detail::check(cudaMallocAsync(&m_scratch, bytes, stream), "cudaMallocAsync");
            m_bytes = bytes;
        }
        return m_scratch;
    }
    void* scratch() const { return m_scratch; }
    size_t bytes() const { return m_bytes; }

private:
    int m_device;
    void* m_scratch = nullptr;
    size_t m_bytes = 0;
};

}  // namespace tinyhiponesweep

namespace minimum_lbvh {

// BVHGPUBuilder (minimum_lbvh.h:726-885).
class BVHGPUBuilder {
public:
    BVHGPUBuilder(const char* kernel = nullptr, const char* includeDir = nullptr)
    {
        (void)kernel;  // the reference compiles minimum_lbvh.cu at run time from here;
        (void)includeDir;  // this library's kernels are compiled ahead of time
        detail::check(cudaMalloc((void**)&m_sceneAABB, sizeof(AABB)), "cudaMalloc");
        detail::check(cudaMalloc((void**)&m_rootNode, 16), "cudaMalloc");
    }
    ~BVHGPUBuilder()
    {
        if (m_internals) cudaFree(m_internals);
        cudaFree(m_rootNode);
        cudaFree(m_sceneAABB);
    }
    BVHGPUBuilder(const BVHGPUBuilder&) = delete;
    void operator=(const BVHGPUBuilder&) = delete;

    void build(const Triangle* triangles, int nTriangles, uint32_t buildOption, tinyhiponesweep::OnesweepSort& sorter,
               cudaStream_t stream)
    {
        reserve_nodes(nTriangles, stream);
        const size_t bytes = mlbvh_build_scratch_bytes((uint32_t)nTriangles);
        void* scratch = sorter.reserve(bytes, stream);
        detail::check(mlbvh_build(reinterpret_cast<const mlbvh_triangle*>(triangles), (uint32_t)nTriangles,
                                  buildOption, reinterpret_cast<mlbvh_internal_node*>(m_internals),
                                  reinterpret_cast<mlbvh_node_index*>(m_rootNode),
                                  reinterpret_cast<mlbvh_aabb*>(m_sceneAABB), scratch, bytes, stream),
                      "mlbvh_build");
    }
    // The higher-quality build, counterpart of BVHCPUBuilder::buildByEmbree
    // (minimum_lbvh.h:594-656) on the GPU: PLOC with neighbourhood radius
    // `radius`, the same members and node conventions as build().
    void buildByPLOC(const Triangle* triangles, int nTriangles, uint32_t buildOption,
                     tinyhiponesweep::OnesweepSort& sorter, cudaStream_t stream, int radius = 8)
    {
        reserve_nodes(nTriangles, stream);
        const size_t bytes = mlbvh_build_ploc_scratch_bytes((uint32_t)nTriangles);
        void* scratch = sorter.reserve(bytes, stream);
        detail::check(mlbvh_build_ploc(reinterpret_cast<const mlbvh_triangle*>(triangles), (uint32_t)nTriangles,
                                       buildOption, radius, reinterpret_cast<mlbvh_internal_node*>(m_internals),
                                       reinterpret_cast<mlbvh_node_index*>(m_rootNode),
                                       reinterpret_cast<mlbvh_aabb*>(m_sceneAABB), scratch, bytes, stream),
                      "mlbvh_build_ploc");
    }
    bool empty() const { return m_nTriangles == 0; }

    AABB* m_sceneAABB = nullptr;
    InternalNode* m_internals = nullptr;
    NodeIndex* m_rootNode = nullptr;
    int m_nTriangles = 0;

private:
    void reserve_nodes(int nTriangles, cudaStream_t stream)
    {
        m_nTriangles = nTriangles;
        const size_t nodes = nTriangles > 1 ? (size_t)nTriangles - 1 : 1;
        if (nodes > m_capacity) {
            if (m_internals) detail::check(cudaFreeAsync(m_internals, stream), "cudaFreeAsync");
            detail::check(cudaMallocAsync((void**)&m_internals, sizeof(InternalNode) * nodes, stream),
                          "cudaMallocAsync");
            m_capacity = nodes;
        }
    }
    size_t m_capacity = 0;
};

}  // namespace minimum_lbvh
