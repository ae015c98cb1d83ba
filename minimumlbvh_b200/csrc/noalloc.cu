// mlbvh_build_noalloc: the build of mlbvh_build for callers that may not
// allocate device memory (see include/mlbvh.h). Its scratch is the file-scope
// device array below, resident on every GPU that loads this library until
// the process exits.
//
// Host code cannot use g_noallocScratch as a device pointer: its name is a
// host-side stand-in. The device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and cached; kernels receive
// that address. The build zeroes its own counters, histograms and look-back
// words on every call and resets its hand-off words, so the array needs no
// clearing between calls; it keeps the last call's contents, and calls that
// overlap on the GPU (in different streams) race on it.
#include <mutex>

#include "capi_internal.h"

namespace mlbvh {

namespace {

constexpr uint32_t kNoAllocMaxTriangles = 65536;
constexpr size_t kNoAllocScratchBytes = 2u << 20;  // 2 MiB >= mlbvh_build_scratch_bytes(65536)
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noallocScratch[kNoAllocScratchBytes];

std::mutex g_noallocMutex;
void* g_noallocAddress[kMaxDevices] = {};

// The device address of g_noallocScratch on the current device, looked up on
// the first call made with that device current.
mlbvh_status noalloc_scratch(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(MLBVH_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noallocMutex);
    if (!g_noallocAddress[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
        g_noallocAddress[dev] = p;
    }
    *out = g_noallocAddress[dev];
    return MLBVH_OK;
}

}  // namespace

}  // namespace mlbvh

using namespace mlbvh;

extern "C" mlbvh_status mlbvh_build_noalloc(const mlbvh_triangle* dTriangles, uint32_t nTriangles,
                                            uint32_t buildOption, mlbvh_internal_node* dInternals,
                                            mlbvh_node_index* dRootNode, mlbvh_aabb* dSceneAABB, void* stream)
{
    clear_error();
    if (nTriangles > kNoAllocMaxTriangles)
        return fail(MLBVH_ERR_INVALID_ARG, "mlbvh_build_noalloc supports at most 65536 triangles");
    if (build_scratch_bytes(nTriangles) > kNoAllocScratchBytes)
        return fail(MLBVH_ERR_INVALID_ARG, "built-in scratch smaller than the build needs");
    void* scratch = nullptr;
    if (mlbvh_status s = noalloc_scratch(&scratch)) return s;
    return build(dTriangles, nTriangles, buildOption, dInternals, dRootNode, dSceneAABB, nullptr, nullptr, nullptr,
                 scratch, kNoAllocScratchBytes, reinterpret_cast<cudaStream_t>(stream), 0);
}
