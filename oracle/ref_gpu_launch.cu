// Baseline infrastructure only: a launcher for the reference's OWN GPU kernels
// (minimum_lbvh.cu: getSceneAABB, buildMortons, computeDeltas, build;
// main_gpu.cu: ao, pt), compiled unmodified for sm_100a from the reference
// checkout by oracle/Makefile (nothing is copied) into
// oracle/_ref/libmlbvh_ref_gpu.so. The reference launches them through Orochi
// (minimum_lbvh.h:783-871, main_gpu.cpp:337-350), which is not available; this
// file launches them through the CUDA runtime with the reference's own grid
// and block shapes. It serves the reference-GPU baseline leg of bench.py;
// nothing in the product links it.
//
// Left out on purpose: the reference's Onesweep sort (tinyhiponesweep.h). Its
// tile index is blockIdx.x (:236) and its look-back and tail waits (:341-409)
// spin without a bound, relying on in-order block dispatch; a stall there
// would hang a shared GPU. The caller passes keys sorted by this project's
// sort (bit-identical to the reference's stable order) instead.
//
// Guards against the reference's known launch defects:
//   * build: the grid covers ceil((n-1)/256) blocks of 256 threads for n leaves
//     (minimum_lbvh.h:859-862), which skips the last leaf when (n-1) % 256 == 0
//     and leaves an incomplete tree; such n are refused.
//   * ao, pt: the bounds test is `w <= x && h <= y` (main_gpu.cu:116, 184), so
//     threads past one edge write past the image; the pixel (accumulator)
//     buffer must cover the whole padded grid (ceil(w/16) * 16 by
//     ceil(h/16) * 16 pixels), checked here.
// The reference's headers first: under nvcc, helper_math.h declares the
// fixed-width integer types itself (helper_math.h:46-53), which a prior
// <cstdint> would contradict.
#include "minimum_lbvh.h"
#include "camera.h"

#include <cuda_runtime.h>

using namespace minimum_lbvh;

// main_gpu.cu:10-15 (global scope); the launcher only passes the pointer on.
struct TriangleAttrib;

extern "C" __global__ void getSceneAABB(AABB* sceneAABB, const Triangle* triangles, int nTriangles);
extern "C" __global__ void buildMortons(IndexedMorton* indexedMortons, const Triangle* triangles, int nTriangles,
                                        const AABB* sceneAABB, uint32_t buildOption);
extern "C" __global__ void computeDeltas(uint8_t* deltas, const IndexedMorton* indexedMortons, int nTriangles);
extern "C" __global__ void build(NodeIndex* rootNode, InternalNode* internals, const Triangle* triangles,
                                 int nTriangles, uint8_t* deltas, const IndexedMorton* indexedMortons);
extern "C" __global__ void ao(uint32_t* pixels, int2 imageSize, RayGenerator rayGenerator, const NodeIndex* rootNode,
                              const InternalNode* internals, const Triangle* triangles, int useSobol);
extern "C" __global__ void pt(uint32_t* pixels, float4* accumulators, int2 imageSize, RayGenerator rayGenerator,
                              const NodeIndex* rootNode, const InternalNode* internals, const Triangle* triangles,
                              const TriangleAttrib* triangleAttribs, int useSobol, int maxSPP);

namespace {

unsigned blocks_of(long long n, int per) { return (unsigned)((n + per - 1) / per); }

int status_of(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }

}  // namespace

extern "C" {

// getSceneAABB after resetting the box to empty (minimum_lbvh.h:803-818).
int refgpu_scene_aabb(void* dScene, const void* dTris, int n, void* stream)
{
    if (n < 1) return -1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the empty box in static storage, as the reference keeps it (minimum_lbvh.h:803-804);
    // AABB::setEmpty (:229-233) is device-only, so the fields are set here
    static AABB empty;
    empty.lower = make_float3(+MINIMUM_LBVH_FLT_MAX, +MINIMUM_LBVH_FLT_MAX, +MINIMUM_LBVH_FLT_MAX);
    empty.upper = make_float3(-MINIMUM_LBVH_FLT_MAX, -MINIMUM_LBVH_FLT_MAX, -MINIMUM_LBVH_FLT_MAX);
    cudaError_t e = cudaMemcpyAsync(dScene, &empty, sizeof(AABB), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return status_of(e);
    getSceneAABB<<<blocks_of(n, 256), 256, 0, s>>>(static_cast<AABB*>(dScene), static_cast<const Triangle*>(dTris),
                                                   n);
    return status_of(cudaGetLastError());
}

// buildMortons (minimum_lbvh.h:820-832): unsorted IndexedMorton pairs.
int refgpu_mortons(void* dMortons, const void* dTris, int n, const void* dScene, uint32_t option, void* stream)
{
    if (n < 1) return -1;
    buildMortons<<<blocks_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<IndexedMorton*>(dMortons), static_cast<const Triangle*>(dTris), n,
        static_cast<const AABB*>(dScene), option);
    return status_of(cudaGetLastError());
}

// computeDeltas, the 0xFF fill of the nodes and build (minimum_lbvh.h:836-863)
// over sorted pairs.
int refgpu_deltas_and_build(void* dRoot, void* dNodes, const void* dTris, int n, void* dDeltas,
                            const void* dSortedMortons, void* stream)
{
    if (n < 2 || (n - 1) % 256 == 0) return -1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    computeDeltas<<<blocks_of(n - 1, 256), 256, 0, s>>>(static_cast<uint8_t*>(dDeltas),
                                                         static_cast<const IndexedMorton*>(dSortedMortons), n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(dNodes, 0xFF, sizeof(InternalNode) * (size_t)(n - 1), s);
    if (e != cudaSuccess) return status_of(e);
    build<<<blocks_of(n - 1, 256), 256, 0, s>>>(static_cast<NodeIndex*>(dRoot), static_cast<InternalNode*>(dNodes),
                                                 static_cast<const Triangle*>(dTris), n,
                                                 static_cast<uint8_t*>(dDeltas),
                                                 static_cast<const IndexedMorton*>(dSortedMortons));
    return status_of(cudaGetLastError());
}

// ao with 16 x 16 blocks over ceil(w/16) x ceil(h/16) (main_gpu.cpp:337-350).
// camera: origin, right, up (RayGenerator, camera.h:5-8). bufferPixels must
// be at least the padded grid's pixel count.
int refgpu_ao(void* dPixels, long long bufferPixels, int w, int h, const float* camera, const void* dRoot,
              const void* dNodes, const void* dTris, int useSobol, void* stream)
{
    if (w < 1 || h < 1) return -1;
    const long long padded = (long long)blocks_of(w, 16) * 16 * (long long)blocks_of(h, 16) * 16;
    if (bufferPixels < padded) return -2;
    RayGenerator gen;
    gen.m_origin = make_float3(camera[0], camera[1], camera[2]);
    gen.m_right = make_float3(camera[3], camera[4], camera[5]);
    gen.m_up = make_float3(camera[6], camera[7], camera[8]);
    const dim3 grid(blocks_of(w, 16), blocks_of(h, 16), 1), block(16, 16, 1);
    ao<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<uint32_t*>(dPixels), make_int2(w, h), gen, static_cast<const NodeIndex*>(dRoot),
        static_cast<const InternalNode*>(dNodes), static_cast<const Triangle*>(dTris), useSobol);
    return status_of(cudaGetLastError());
}

// pt with 16 x 16 blocks (main_gpu.cpp:355-368): one progressive pass over
// the float4 accumulators (w = samples so far). attribs: TriangleAttrib
// (main_gpu.cu:10-15). bufferPixels as for refgpu_ao.
int refgpu_pt(void* dAccum, long long bufferPixels, int w, int h, const float* camera, const void* dRoot,
              const void* dNodes, const void* dTris, const void* dAttribs, int useSobol, int maxSPP, void* stream)
{
    if (w < 1 || h < 1) return -1;
    const long long padded = (long long)blocks_of(w, 16) * 16 * (long long)blocks_of(h, 16) * 16;
    if (bufferPixels < padded) return -2;
    RayGenerator gen;
    gen.m_origin = make_float3(camera[0], camera[1], camera[2]);
    gen.m_right = make_float3(camera[3], camera[4], camera[5]);
    gen.m_up = make_float3(camera[6], camera[7], camera[8]);
    const dim3 grid(blocks_of(w, 16), blocks_of(h, 16), 1), block(16, 16, 1);
    pt<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        nullptr, static_cast<float4*>(dAccum), make_int2(w, h), gen, static_cast<const NodeIndex*>(dRoot),
        static_cast<const InternalNode*>(dNodes), static_cast<const Triangle*>(dTris),
        static_cast<const TriangleAttrib*>(dAttribs), useSobol, maxSPP);
    return status_of(cudaGetLastError());
}

}  // extern "C"
