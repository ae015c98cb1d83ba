// mlbvh_build_noalloc: the build of mlbvh_build for callers that may not
// allocate device memory (see include/mlbvh.h). Its scratch is the file-scope
// device array below, resident on every GPU that loads this library until
// the process exits.
//
// Host code cannot use g_noallocScratch as a device pointer: its name is a
// host-side stand-in. The device address is looked up with
// cudaGetSymbolAddress, with the device current, on the first call made in
// each CUDA context, and cached together with that context's id: a context
// that is destroyed and created again (cudaDeviceReset, a driver-API context
// of the caller's) reloads this library's module, possibly at another
// address, and its first call looks the address up again. Kernels receive the
// cached address. The build zeroes its own counters, histograms and look-back
// words on every call and resets its hand-off words, so the array needs no
// clearing between calls; it keeps the last call's contents, and calls that
// overlap on the GPU (in different streams) race on it. Its first word is the
// build's error word, which mlbvh_scratch_status(NULL, stream) reads.
#include <cuda.h>

#include <mutex>

#include "capi_internal.h"

namespace mlbvh {

namespace {

constexpr uint32_t kNoAllocMaxTriangles = 65536;
constexpr size_t kNoAllocScratchBytes = 2u << 20;  // 2 MiB >= mlbvh_build_scratch_bytes(65536)
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noallocScratch[kNoAllocScratchBytes];

// The driver's cuCtxGetCurrent / cuCtxGetId, fetched through the runtime so
// that the library needs no link against libcuda.
using CtxGetCurrentFn = CUresult(CUDAAPI*)(CUcontext*);
using CtxGetIdFn = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);

struct CachedAddress {
    unsigned long long context = 0;  // cuCtxGetId of the context the address was taken in; 0: none
    void* address = nullptr;
};

std::mutex g_noallocMutex;
CachedAddress g_noallocAddress[kMaxDevices];
CtxGetCurrentFn g_ctxGetCurrent = nullptr;
CtxGetIdFn g_ctxGetId = nullptr;

mlbvh_status driver_entry_points()
{
    if (g_ctxGetCurrent && g_ctxGetId) return MLBVH_OK;
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound, qb = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &a, 12000, cudaEnableDefault, &qa);
    if (e == cudaSuccess) e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &b, 12000, cudaEnableDefault, &qb);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
        return fail(MLBVH_ERR_CUDA, "the CUDA driver offers no cuCtxGetCurrent / cuCtxGetId");
    g_ctxGetCurrent = reinterpret_cast<CtxGetCurrentFn>(a);
    g_ctxGetId = reinterpret_cast<CtxGetIdFn>(b);
    return MLBVH_OK;
}

// The id of the context current on this thread for device `dev`, making the
// device's primary context current first where none is (the runtime would do
// the same on its next call).
mlbvh_status current_context_id(int dev, unsigned long long* id)
{
    CUcontext ctx = nullptr;
    if (g_ctxGetCurrent(&ctx) != CUDA_SUCCESS) return fail(MLBVH_ERR_CUDA, "cuCtxGetCurrent failed");
    if (!ctx) {
        cudaError_t e = cudaSetDevice(dev);
        if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
        if (g_ctxGetCurrent(&ctx) != CUDA_SUCCESS || !ctx) return fail(MLBVH_ERR_CUDA, "no current CUDA context");
    }
    if (g_ctxGetId(ctx, id) != CUDA_SUCCESS) return fail(MLBVH_ERR_CUDA, "cuCtxGetId failed");
    return MLBVH_OK;
}

// The device address of g_noallocScratch in the current context. With
// `lookup` false, a context in which no build has looked it up yet gives
// nullptr (nothing to report on).
mlbvh_status noalloc_scratch(void** out, bool lookup)
{
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(MLBVH_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noallocMutex);
    if (mlbvh_status s = driver_entry_points()) return s;
    unsigned long long ctx = 0;
    if (mlbvh_status s = current_context_id(dev, &ctx)) return s;
    CachedAddress& c = g_noallocAddress[dev];
    if (c.context != ctx || !c.address) {
        if (!lookup) return MLBVH_OK;
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
        c.context = ctx;
        c.address = p;
    }
    *out = c.address;
    return MLBVH_OK;
}

}  // namespace

mlbvh_status noalloc_scratch_status(cudaStream_t stream)
{
    void* scratch = nullptr;
    if (mlbvh_status s = noalloc_scratch(&scratch, false)) return s;
    if (!scratch)
        return fail(MLBVH_ERR_INVALID_ARG,
                    "null scratch pointer, and no mlbvh_build_noalloc call in this device's current context");
    return scratch_status(scratch, stream);
}

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
    if (mlbvh_status s = noalloc_scratch(&scratch, true)) return s;
    return build(dTriangles, nTriangles, buildOption, dInternals, dRootNode, dSceneAABB, nullptr, nullptr, nullptr,
                 scratch, kNoAllocScratchBytes, reinterpret_cast<cudaStream_t>(stream), spin_limit());
}
