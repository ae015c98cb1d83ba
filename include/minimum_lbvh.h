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
//   BVHCPUBuilder::build(tris, n, opt) (:512)         same call and members
//     m_internals, m_deltas, m_rootNode (:666-668),     (host std::vectors, a
//     empty(), validate() (:657-664)                    host NodeIndex); the
//                                                       build runs on the GPU
//
// Differences, by design: BVHGPUBuilder::build() neither prints its time nor
// synchronises (the reference's DeviceStopwatch does both, :785-870), so a
// bounded device wait that gave up is reported by status(stream), which
// synchronises; errors abort with the library's message, as the reference's
// host asserts abort (:23); the query functions take rays with t in
// [0, hit->t] exactly as the reference's. BVHCPUBuilder keeps the reference's
// host-side results, but there is no CPU build: it uploads the triangles,
// builds on the GPU and copies the tree back, synchronously. The reference's
// intersect_* are host+device functions (:5-24); here they are device-only,
// since nothing of this library runs the path on the CPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>
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
        m_scratch = scratch;
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
        m_scratch = scratch;
    }
    // Synchronises `stream` and reports on the last build (build or
    // buildByPLOC): MLBVH_ERR_TIMEOUT if one of its bounded device waits gave
    // up (the tree is then unusable; build again), else MLBVH_OK. The
    // reference's build synchronised on return and had no such waits; this
    // one returns after the launches, so call status() where the reference's
    // caller relied on a finished build. The scratch is the sorter's, so
    // the sorter must not have run another build since.
    mlbvh_status status(cudaStream_t stream) const
    {
        if (!m_scratch) return MLBVH_ERR_INVALID_ARG;
        return mlbvh_scratch_status(m_scratch, stream);
    }
    bool empty() const { return m_nTriangles == 0; }

    AABB* m_sceneAABB = nullptr;
    InternalNode* m_internals = nullptr;
    NodeIndex* m_rootNode = nullptr;
    int m_nTriangles = 0;

private:
    const void* m_scratch = nullptr;  // the scratch of the last build, for status()
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

// BVHCPUBuilder (minimum_lbvh.h:509-669): the reference's host-side build
// API, with the tree in host memory (m_internals, m_deltas, m_rootNode) for
// callers that read it on the host, as main.cpp:246-249 does. The build runs
// on the GPU (device `device`, its own stream): build() uploads the host
// triangles, runs mlbvh_build_ex and copies nodes, deltas and root back, and
// returns when they are there. Its tree is the GPU build's, i.e. the
// reference's with equal Morton keys in triangle-index order (the reference's
// CPU build sorts with std::sort, whose order of equal keys is unspecified;
// its GPU build sorts stably, as here). BUILD_OPTION_CPU_PARALLEL is accepted
// and has no effect. Device buffers are kept for the next build and freed
// with the object. Errors (and a bounded device wait that gave up) abort
// with the library's message, as the reference's host asserts abort.
class BVHCPUBuilder {
public:
    explicit BVHCPUBuilder(int device = 0) : m_device(device) {}
    ~BVHCPUBuilder()
    {
        if (!m_stream) return;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(m_device);
        cudaFree(m_dTriangles);
        cudaFree(m_dInternals);
        cudaFree(m_dRoot);
        cudaFree(m_dDeltas);
        cudaFree(m_dScratch);
        cudaStreamDestroy(m_stream);
        cudaSetDevice(prev);
    }
    BVHCPUBuilder(const BVHCPUBuilder&) = delete;
    void operator=(const BVHCPUBuilder&) = delete;

    void build(const Triangle* triangles, int nTriangles, uint32_t buildOption)
    {
        m_internals.clear();
        m_deltas.clear();
        m_rootNode = NodeIndex();
        if (nTriangles <= 0) return;  // the reference requires nTriangles >= 1 (:515)
        const uint32_t n = (uint32_t)nTriangles;
        int prev = 0;
        detail::check(cudaGetDevice(&prev), "cudaGetDevice");
        detail::check(cudaSetDevice(m_device), "cudaSetDevice");
        if (!m_stream) detail::check(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        grow(&m_dTriangles, &m_trianglesBytes, sizeof(Triangle) * n);
        grow(&m_dInternals, &m_internalsBytes, sizeof(InternalNode) * (n > 1 ? n - 1 : 1));
        grow(&m_dRoot, &m_rootBytes, 16);
        grow(&m_dDeltas, &m_deltasBytes, n);
        grow(&m_dScratch, &m_scratchBytes, mlbvh_build_scratch_bytes(n));
        detail::check(cudaMemcpyAsync(m_dTriangles, triangles, sizeof(Triangle) * n, cudaMemcpyHostToDevice, m_stream),
                      "cudaMemcpyAsync");
        detail::check(mlbvh_build_ex(static_cast<const mlbvh_triangle*>(m_dTriangles), n, buildOption,
                                     n > 1 ? static_cast<mlbvh_internal_node*>(m_dInternals) : nullptr,
                                     static_cast<mlbvh_node_index*>(m_dRoot), nullptr, nullptr, nullptr,
                                     static_cast<uint8_t*>(m_dDeltas), m_dScratch, m_scratchBytes, m_stream),
                      "mlbvh_build_ex");
        detail::check(mlbvh_scratch_status(m_dScratch, m_stream), "BVHCPUBuilder::build");
        m_internals.resize(n - 1);
        m_deltas.resize(n - 1);
        if (n > 1) {
            detail::check(cudaMemcpyAsync(m_internals.data(), m_dInternals, sizeof(InternalNode) * (n - 1),
                                          cudaMemcpyDeviceToHost, m_stream),
                          "cudaMemcpyAsync");
            detail::check(cudaMemcpyAsync(m_deltas.data(), m_dDeltas, n - 1, cudaMemcpyDeviceToHost, m_stream),
                          "cudaMemcpyAsync");
        }
        detail::check(cudaMemcpyAsync(&m_rootNode, m_dRoot, sizeof(NodeIndex), cudaMemcpyDeviceToHost, m_stream),
                      "cudaMemcpyAsync");
        detail::check(cudaStreamSynchronize(m_stream), "cudaStreamSynchronize");
        detail::check(cudaSetDevice(prev), "cudaSetDevice");
    }
    bool empty() const { return m_internals.empty(); }
    // validate_lbvh (minimum_lbvh.h:415-426) from the root with maxDelta 255:
    // every internal node's split delta is at most its parent's. Walked with
    // an explicit stack (a chain of equal keys makes the tree as deep as the
    // chain is long); aborts on a violation, as the reference's assert does.
    void validate() const
    {
        if (m_rootNode.m_isLeaf || m_internals.empty()) return;
        std::vector<std::pair<NodeIndex, int>> todo{{m_rootNode, 255}};
        while (!todo.empty()) {
            const std::pair<NodeIndex, int> top = todo.back();
            todo.pop_back();
            if (top.first.m_isLeaf) continue;
            const uint32_t i = top.first.m_index;
            if (i >= m_internals.size() || (int)m_deltas[i] > top.second) {
                std::fprintf(stderr, "minimum_lbvh: BVHCPUBuilder::validate failed at node %u\n", i);
                std::abort();
            }
            todo.push_back({m_internals[i].children[0], (int)m_deltas[i]});
            todo.push_back({m_internals[i].children[1], (int)m_deltas[i]});
        }
    }

    NodeIndex m_rootNode;
    std::vector<InternalNode> m_internals;
    std::vector<uint8_t> m_deltas;

private:
    void grow(void** p, size_t* have, size_t need)
    {
        if (need <= *have) return;
        if (*p) detail::check(cudaFree(*p), "cudaFree");
        *p = nullptr;
        detail::check(cudaMalloc(p, need), "cudaMalloc");
        *have = need;
    }
    int m_device;
    cudaStream_t m_stream = nullptr;
    void* m_dTriangles = nullptr;
    void* m_dInternals = nullptr;
    void* m_dRoot = nullptr;
    void* m_dDeltas = nullptr;
    void* m_dScratch = nullptr;
    size_t m_trianglesBytes = 0, m_internalsBytes = 0, m_rootBytes = 0, m_deltasBytes = 0, m_scratchBytes = 0;
};

}  // namespace minimum_lbvh
