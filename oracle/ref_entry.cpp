// Test infrastructure only: the C entry points of oracle/_ref/libmlbvh_ref.so.
//
// This translation unit compiles the REFERENCE's own sources, unmodified and
// read where they lie (-I points at the reference checkout; nothing is copied),
// with the three Linux shim headers in oracle/ref_shims/:
//   minimum_lbvh.h   Morton coding, build_lbvh, BVHCPUBuilder, traversals
//   main_gpu.cu      the normal/ao/pt/pack shading kernels, compiled as host C++
//   camera.h, sobol.h
// It exists to pin oracle/mlbvh_oracle.c (the restatement the tests use as the
// checker) against the reference itself, and to serve as the timed CPU
// baseline. Nothing in the product links it.
//
// Build: oracle/Makefile (g++ -std=c++17 -O2 -ffp-contract=off -mlzcnt -mbmi).

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstring>
#include <cmath>
#include <cstdint>
#include <climits>
#include <thread>
#include <vector>

using std::fmax;

// Host stand-ins for the CUDA launch built-ins, so that the reference's
// kernels in main_gpu.cu run as plain functions, one call per thread.
#define __device__
#define __global__
struct OracleDim3 { unsigned int x, y, z; };
static thread_local OracleDim3 threadIdx, blockIdx, blockDim;

#include "minimum_lbvh.h"
#include "main_gpu.cu"

using namespace minimum_lbvh;

static_assert(sizeof(Triangle) == 36, "Triangle is 36 B");
static_assert(sizeof(InternalNode) == 64, "InternalNode is 64 B");
static_assert(sizeof(Hit) == 32, "Hit is 32 B");
static_assert(sizeof(RayGenerator) == 36, "RayGenerator is 9 floats");
static_assert(sizeof(TriangleAttrib) == 60, "TriangleAttrib is 60 B");

namespace
{
unsigned hw_threads()
{
    return concurrency::oracle_thread_count();
}

template <class F>
void parallel_rows(int n, F f)
{
    concurrency::parallel_for(0, n, f);
}

// Runs a 2D reference kernel body over every (x, y) of the image, as the
// reference's 16x16-block launch would, without its out-of-range threads.
template <class K>
void launch2d(int w, int h, K kernel)
{
    parallel_rows(h, [&](int y) {
        blockDim = {16, 16, 1};
        for (int x = 0; x < w; ++x)
        {
            blockIdx = {(unsigned)(x / 16), (unsigned)(y / 16), 0};
            threadIdx = {(unsigned)(x % 16), (unsigned)(y % 16), 0};
            kernel();
        }
    });
}
} // namespace

extern "C" {

int ref_version(void) { return 1; }
int ref_threads(void) { return (int)hw_threads(); }

// BVHCPUBuilder::build exactly as the reference runs it (minimum_lbvh.h:512),
// including its unstable std::sort. Outputs nodes [n-1], deltas [n-1], root.
void ref_cpu_builder(const Triangle* tris, int n, uint32_t option,
                     InternalNode* nodes, uint8_t* deltas, uint32_t* root)
{
    BVHCPUBuilder b;
    b.build(tris, n, option);
    b.validate();
    if (n > 1)
    {
        memcpy(nodes, b.m_internals.data(), sizeof(InternalNode) * (n - 1));
        memcpy(deltas, b.m_deltas.data(), n - 1);
    }
    memcpy(root, &b.m_rootNode, 4);
}

// BVHCPUBuilder::build (minimum_lbvh.h:512-592) with one change: the keys are
// ordered by std::stable_sort, i.e. by (morton, triangle index), the order the
// reference's GPU radix sort (a stable LSD sort, minimum_lbvh.h:833) produces.
// Everything else calls the reference's own functions. keys/indices receive the
// sorted IndexedMorton array; nThreads 0 means all host threads.
void ref_build_stable(const Triangle* tris, int n, uint32_t option,
                      InternalNode* nodes, uint8_t* deltas, uint32_t* root,
                      uint32_t* keys, uint32_t* indices, float* sceneAABB,
                      int parallel)
{
    std::vector<InternalNode> internals(n > 1 ? n - 1 : 0);
    for (auto& node : internals) node.context = 0xFFFFFFFF;
    std::vector<uint8_t> d(n > 1 ? n - 1 : 0);

    AABB scene;
    scene.setEmpty();
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 3; ++j) scene.extend(tris[i].vs[j]);

    std::vector<IndexedMorton> mortons(n);
    for (int i = 0; i < n; i++)
    {
        Triangle tri = tris[i];
        float3 center = (tri.vs[0] + tri.vs[1] + tri.vs[2]) / 3.0f;
        if (option & BUILD_OPTION_USE_NORMAL)
        {
            float3 ng = normalOf(tri);
            AABB unit = {{-1, -1, -1}, {+1, +1, +1}};
            uint32_t nMorton = (uint32_t)(unit.encodeMortonCode(ng) >> 31);
            uint32_t pMorton = (uint32_t)(scene.encodeMortonCode(center) >> 31);
            mortons[i].morton = (pMorton & 0xFFFFFFC0) | (nMorton >> 26);
        }
        else
        {
            mortons[i].morton = (uint32_t)(scene.encodeMortonCode(center) >> 31);
        }
        mortons[i].index = i;
    }
    std::stable_sort(mortons.begin(), mortons.end(),
                     [](IndexedMorton a, IndexedMorton b) { return a.morton < b.morton; });
    for (size_t i = 0; i + 1 < mortons.size(); i++)
        d[i] = delta(mortons[i].morton, mortons[i + 1].morton);

    NodeIndex rootNode(0, true);
    if (n == 1)
    {
        // build_lbvh writes internals[0].parent for a single leaf, out of
        // bounds of an empty array; the root of a 1-triangle tree is leaf 0.
        rootNode = NodeIndex(mortons[0].index, true);
    }
    else if (parallel)
    {
        concurrency::parallel_for(size_t(0), mortons.size(), [&](uint32_t i_leaf) {
            build_lbvh(&rootNode, internals.data(), tris, n, d.data(), i_leaf, mortons[i_leaf].index);
        });
    }
    else
    {
        for (uint32_t i_leaf = 0; i_leaf < mortons.size(); i_leaf++)
            build_lbvh(&rootNode, internals.data(), tris, n, d.data(), i_leaf, mortons[i_leaf].index);
    }
    if (n > 1)
    {
        validate_lbvh(rootNode, internals.data(), d.data(), 255);
        memcpy(nodes, internals.data(), sizeof(InternalNode) * (n - 1));
        memcpy(deltas, d.data(), n - 1);
    }
    memcpy(root, &rootNode, 4);
    for (int i = 0; i < n; i++)
    {
        if (keys) keys[i] = mortons[i].morton;
        if (indices) indices[i] = mortons[i].index;
    }
    if (sceneAABB) memcpy(sceneAABB, &scene, sizeof(AABB));
}

// The toy 8-key tree of main.cpp:60-109 over caller-given keys (leaf i keeps
// index i, no triangles), built serially; asserts validate_lbvh.
void ref_toy_tree(const uint32_t* mortons, int n, InternalNode* nodes, uint8_t* deltas, uint32_t* root)
{
    std::vector<uint8_t> d(n - 1);
    for (int i = 0; i + 1 < n; i++) d[i] = delta(mortons[i], mortons[i + 1]);
    std::vector<InternalNode> internals(n - 1);
    for (auto& node : internals) node.context = 0xFFFFFFFF;
    NodeIndex rootNode;
    for (uint32_t i_leaf = 0; i_leaf < (uint32_t)n; i_leaf++)
        build_lbvh(&rootNode, internals.data(), nullptr, n, d.data(), i_leaf, i_leaf);
    validate_lbvh(rootNode, internals.data(), d.data(), INT_MAX);
    memcpy(nodes, internals.data(), sizeof(InternalNode) * (n - 1));
    memcpy(deltas, d.data(), n - 1);
    memcpy(root, &rootNode, 4);
}

// Traces rays[i] = {ro.xyz, tmin, rd.xyz, tmax} (tmin must be 0: the
// reference's queries have no near limit) with the reference's
// traversals: mode 0 intersect_stackfree (minimum_lbvh.h:981), 1
// intersect_escape_link (:1063), 2 intersect_stackfull (:912, closest only).
void ref_trace(const InternalNode* nodes, const Triangle* tris, uint32_t root,
               const float* rays, int nRays, int query, int mode, Hit* hits)
{
    NodeIndex rootNode;
    memcpy(&rootNode, &root, 4);
    concurrency::parallel_for(0, nRays, [&](int i) {
        const float* r = rays + 8 * (size_t)i;
        float3 ro = make_float3(r[0], r[1], r[2]);
        float3 rd = make_float3(r[4], r[5], r[6]);
        Hit hit;
        hit.t = r[7];
        if (mode == 0)
            intersect_stackfree(&hit, nodes, tris, rootNode, ro, rd, invRd(rd), (RAY_QUERY)query);
        else if (mode == 1)
            intersect_escape_link(&hit, nodes, tris, rootNode, ro, rd, invRd(rd), (RAY_QUERY)query);
        else
        {
            NodeIndex stack[128];
            intersect_stackfull(&hit, nodes, tris, rootNode, ro, rd, invRd(rd), stack);
        }
        // copy the fields into a zeroed record so the padding word is 0
        unsigned char* out = reinterpret_cast<unsigned char*>(hits + i);
        memset(out, 0, sizeof(Hit));
        memcpy(out + offsetof(Hit, t), &hit.t, 4);
        memcpy(out + offsetof(Hit, uv), &hit.uv, 8);
        memcpy(out + offsetof(Hit, ng), &hit.ng, 12);
        memcpy(out + offsetof(Hit, triangleIndex), &hit.triangleIndex, 4);
    });
}

// RayGenerator::lookat (camera.h:10-22); writes m_origin, m_right, m_up.
void ref_lookat(const float* eye, const float* center, const float* up, float fovy,
                int w, int h, float* out9)
{
    RayGenerator g;
    g.lookat(make_float3(eye[0], eye[1], eye[2]), make_float3(center[0], center[1], center[2]),
             make_float3(up[0], up[1], up[2]), fovy, w, h);
    memcpy(out9, &g, sizeof(RayGenerator));
}

// RayGenerator::shoot (camera.h:24-31) for pixel (x, y) of a w x h image with
// no sub-pixel offset, as the normal/ao kernels call it.
void ref_shoot(const float* cam9, int w, int h, int x, int y, float* ro, float* rd)
{
    RayGenerator g;
    memcpy(&g, cam9, sizeof(RayGenerator));
    float3 o, d;
    g.shoot(&o, &d, (float)x / w, (float)y / h);
    memcpy(ro, &o, 12);
    memcpy(rd, &d, 12);
}

// The reference's ao kernel (main_gpu.cu:111-177) run on the host over a
// w x h image: 16 samples, ray length 1.0, packed RGBA8 output.
void ref_ao(uint32_t* pixels, int w, int h, const float* cam9, uint32_t root,
            const InternalNode* nodes, const Triangle* tris, int useSobol)
{
    RayGenerator g;
    memcpy(&g, cam9, sizeof(RayGenerator));
    NodeIndex rootNode;
    memcpy(&rootNode, &root, 4);
    int2 size = {w, h};
    launch2d(w, h, [&]() { ao(pixels, size, g, &rootNode, nodes, tris, useSobol); });
}

// The reference's ao kernel body (main_gpu.cu:121-176) with the sample count,
// AO ray length and Sobol seed as parameters, over rows [rowBegin, rowEnd),
// using the reference's own RayGenerator::shoot, intersect_stackfree,
// sobol::shuffled_scrambled_sobol_2d, sampleHemisphereCosWeighted and
// GetOrthonormalBasis. occluded[pixel] = AO rays that hit (0xFFFFFFFF on a
// primary miss). stats[0] += rays traced. Used as the timed CPU baseline on
// the workloads whose AO parameters differ from the reference's fixed ones.
void ref_ao_param(uint32_t* occluded, int w, int h, const float* cam9, uint32_t root,
                  const InternalNode* nodes, const Triangle* tris, int nSample, float length,
                  uint32_t seed, int rowBegin, int rowEnd, uint64_t* stats)
{
    RayGenerator g;
    memcpy(&g, cam9, sizeof(RayGenerator));
    NodeIndex rootNode;
    memcpy(&rootNode, &root, 4);
    std::atomic<uint64_t> rays(0);
    concurrency::parallel_for(rowBegin, rowEnd, [&](int yi) {
        uint64_t local = 0;
        for (int xi = 0; xi < w; ++xi)
        {
            int pixel = xi + yi * w;
            float3 ro, rd;
            g.shoot(&ro, &rd, (float)xi / w, (float)yi / h);
            Hit hit;
            intersect_stackfree(&hit, nodes, tris, rootNode, ro, rd, invRd(rd));
            ++local;
            if (hit.t == MINIMUM_LBVH_FLT_MAX)
            {
                occluded[pixel] = 0xFFFFFFFF;
                continue;
            }
            float3 n = normalize(hit.ng);
            if (0.0f < dot(n, rd)) n = -n;
            float3 xaxis, zaxis;
            GetOrthonormalBasis(n, &xaxis, &zaxis);
            float3 ao_origin = ro + rd * hit.t + n * 0.001f;
            uint32_t count = 0;
            for (int i = 0; i < nSample; i++)
            {
                float2 random;
                sobol::shuffled_scrambled_sobol_2d(&random.x, &random.y, i, xi, yi, seed);
                float3 dirLocal = sampleHemisphereCosWeighted(random.x, random.y);
                float3 dir = xaxis * dirLocal.x + zaxis * dirLocal.z + n * dirLocal.y;
                Hit h2;
                h2.t = length;
                intersect_stackfree(&h2, nodes, tris, rootNode, ao_origin, dir, invRd(dir), RAY_QUERY_ANY);
                ++local;
                if (h2.t != length) ++count;
            }
            occluded[pixel] = count;
        }
        rays += local;
    });
    if (stats) stats[0] += rays.load();
}

// The reference's normal kernel (main_gpu.cu:84-109) on the host.
void ref_normal(uint32_t* pixels, int w, int h, const float* cam9, uint32_t root,
                const InternalNode* nodes, const Triangle* tris)
{
    RayGenerator g;
    memcpy(&g, cam9, sizeof(RayGenerator));
    NodeIndex rootNode;
    memcpy(&rootNode, &root, 4);
    int2 size = {w, h};
    launch2d(w, h, [&]() { normal(pixels, size, g, &rootNode, nodes, tris); });
}

// One progressive pt launch (main_gpu.cu:179-272) on the host: reads and
// updates the float4 accumulators (w = spp so far).
void ref_pt(uint32_t* pixels, float* accum4, int w, int h, const float* cam9, uint32_t root,
            const InternalNode* nodes, const Triangle* tris, const float* attribs15,
            int useSobol, int maxSPP)
{
    RayGenerator g;
    memcpy(&g, cam9, sizeof(RayGenerator));
    NodeIndex rootNode;
    memcpy(&rootNode, &root, 4);
    int2 size = {w, h};
    launch2d(w, h, [&]() {
        pt(pixels, (float4*)accum4, size, g, &rootNode, nodes, tris,
           (const TriangleAttrib*)attribs15, useSobol, maxSPP);
    });
}

// The pack kernel (main_gpu.cu:273-286) on the host.
void ref_pack(uint32_t* pixels, const float* accum4, int n)
{
    blockDim = {256, 1, 1};
    for (int i = 0; i < n; ++i)
    {
        blockIdx = {(unsigned)(i / 256), 0, 0};
        threadIdx = {(unsigned)(i % 256), 0, 0};
        pack(pixels, (float4*)accum4, n);
    }
}

// sobol::shuffled_scrambled_sobol_2d (sobol.h:119-129).
void ref_sobol(uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2, float* xy)
{
    sobol::shuffled_scrambled_sobol_2d(&xy[0], &xy[1], index, p0, p1, p2);
}

// The reference's Morton and bit utilities (minimum_lbvh.h:99-195).
uint64_t ref_splat3(uint32_t a) { return splat3(a); }
uint32_t ref_compact3(uint64_t m) { return compact3(m); }
uint64_t ref_encode_morton(uint32_t x, uint32_t y, uint32_t z) { return encodeMortonCode(x, y, z); }
uint64_t ref_encode_morton_naive(uint32_t x, uint32_t y, uint32_t z) { return encodeMortonCode_Naive(x, y, z); }
int ref_clz(uint32_t x) { return clz(x); }
int ref_clz64(uint64_t x) { return clz64(x); }
int ref_ffs(uint32_t x) { return ffs(x); }
int ref_ffs64(uint64_t x) { return ffs64(x); }
uint32_t ref_hash_pcg(uint32_t v) { return hashPCG(v); }

// AABB::encodeMortonCode (minimum_lbvh.h:246-251) of one point.
uint64_t ref_aabb_morton(const float* lower, const float* upper, const float* p)
{
    AABB b;
    b.lower = make_float3(lower[0], lower[1], lower[2]);
    b.upper = make_float3(upper[0], upper[1], upper[2]);
    return b.encodeMortonCode(make_float3(p[0], p[1], p[2]));
}

} // extern "C"
