// mlbvh_read_probe: a measurement hook (no reference counterpart). It reads a
// device buffer with the load the traversal kernels use for their nodes
// (32 bytes per instruction, ld.global.nc.v8: through L1 and L2), so that a
// caller timing it with CUDA events gets the bandwidth those loads achieve
// from wherever the buffer lives: a buffer of a few tens of MB stays in the
// 126 MB L2 (beyond the L1s), one of GBs streams from HBM. Two patterns:
//   streaming   consecutive threads read consecutive 32-byte sectors (a warp
//               reads 1 KB per instruction), grid-stride, `passes` sweeps;
//   gather      every load hits a pseudo-random 32-byte sector, as the
//               traversal's node and triangle loads do (each lane its own
//               line); independent loads, eight in flight per thread.
#include <algorithm>

#include "capi_internal.h"

namespace mlbvh {

namespace {

constexpr int kProbeThreads = 256;

__device__ __forceinline__ uint32_t ld32_xor(const void* p)
{
    uint32_t a, b, c, d, e, f, g, h;
    asm volatile("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(a), "=r"(b), "=r"(c), "=r"(d), "=r"(e), "=r"(f), "=r"(g), "=r"(h)
                 : "l"(p));
    return a ^ b ^ c ^ d ^ e ^ f ^ g ^ h;
}

__device__ __forceinline__ uint32_t mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(kProbeThreads)
    k_read_stream(const unsigned char* __restrict__ buf, size_t nSectors, uint32_t passes, uint32_t* sink)
{
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t T = (size_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    for (uint32_t p = 0; p < passes; ++p) {
        size_t s = t;
        for (; s + 3 * T < nSectors; s += 4 * T)
            acc ^= ld32_xor(buf + 32 * s) ^ ld32_xor(buf + 32 * (s + T)) ^ ld32_xor(buf + 32 * (s + 2 * T)) ^
                   ld32_xor(buf + 32 * (s + 3 * T));
        for (; s < nSectors; s += T) acc ^= ld32_xor(buf + 32 * s);
    }
    if (acc == 0x9e3779b9u) sink[t & 1023] = acc;  // keeps the loads; practically never written
}

// nSectors is a power of two; every thread issues `loads` loads (a multiple of 8).
__global__ void __launch_bounds__(kProbeThreads)
    k_read_gather(const unsigned char* __restrict__ buf, uint32_t sectorMask, uint32_t loads, uint32_t* sink)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    uint32_t h = mix(t * 0x9e3779b9u + 1u);
    for (uint32_t k = 0; k < loads; k += 8) {
        uint32_t idx[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            h = mix(h + (uint32_t)j);
            idx[j] = h & sectorMask;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc ^= ld32_xor(buf + 32ull * idx[j]);
    }
    if (acc == 0x9e3779b9u) sink[t & 1023] = acc;
}

}  // namespace

}  // namespace mlbvh

using namespace mlbvh;

extern "C" mlbvh_status mlbvh_read_probe(const void* dBuffer, size_t bytes, int pattern, uint32_t loads,
                                         uint32_t* dSink, size_t* bytesRead, void* stream)
{
    clear_error();
    if (!dBuffer || !dSink || !bytesRead) return fail(MLBVH_ERR_INVALID_ARG, "null buffer, sink or bytesRead");
    if (!aligned32(dBuffer) || !aligned16(dSink)) return fail(MLBVH_ERR_INVALID_ARG, "buffer must be 32-byte aligned");
    if (bytes < 32 * 1024 || bytes % 32) return fail(MLBVH_ERR_INVALID_ARG, "bytes must be a multiple of 32, >= 32 KiB");
    if (loads == 0) return fail(MLBVH_ERR_INVALID_ARG, "loads must be positive");
    const int sms = device_sm_count();
    int dev = 0, perSM = 0;
    cudaGetDevice(&dev);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned char* buf = static_cast<const unsigned char*>(dBuffer);
    const size_t nSectors = bytes / 32;
    if (pattern == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_read_stream, kProbeThreads, 0);
        const int blocks = sms * std::max(perSM, 1);
        k_read_stream<<<blocks, kProbeThreads, 0, s>>>(buf, nSectors, loads, dSink);
        MLBVH_CHECK_LAUNCH("k_read_stream");
        *bytesRead = 32 * nSectors * (size_t)loads;
    } else if (pattern == 1) {
        if (nSectors & (nSectors - 1)) return fail(MLBVH_ERR_INVALID_ARG, "gather needs bytes = 32 * 2^k");
        if (nSectors > (1ull << 32)) return fail(MLBVH_ERR_INVALID_ARG, "gather buffer beyond 128 GiB");
        if (loads % 8) return fail(MLBVH_ERR_INVALID_ARG, "gather loads per thread must be a multiple of 8");
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_read_gather, kProbeThreads, 0);
        const int blocks = sms * std::max(perSM, 1);
        k_read_gather<<<blocks, kProbeThreads, 0, s>>>(buf, (uint32_t)(nSectors - 1), loads, dSink);
        MLBVH_CHECK_LAUNCH("k_read_gather");
        *bytesRead = 32ull * loads * (size_t)blocks * kProbeThreads;
    } else {
        return fail(MLBVH_ERR_INVALID_ARG, "pattern must be 0 (streaming) or 1 (gather)");
    }
    return MLBVH_OK;
}
