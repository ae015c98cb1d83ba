// LBVH build on B200: scene bounds, Morton keys + digit histograms, a
// stable Onesweep LSD radix sort, and the agglomerative bottom-up build.
//
// Replaces BVHGPUBuilder::build (minimum_lbvh.h:783-871), its kernels
// (minimum_lbvh.cu:38-120) and OnesweepSort (tinyhiponesweep.h:592-668).
//
// Launch chain on one stream (no host synchronisation):
//   k_scene_bounds   per-CTA partial bounds of all vertices; zeroes the
//                    sort's counters, histograms and look-back words
//   k_keys           reduces the partial bounds, writes the 32-bit Morton key
//                    of every triangle and accumulates the four 8-bit digit
//                    histograms; resets the build's hand-off words
//   k_onesweep x4    one stable pass per digit: warp multisplit, decoupled
//                    look-back over per-tile digit counts, scatter through
//                    shared memory so that runs of one digit store coalesced
//   k_build          one thread per sorted leaf climbs to the root
//                    (build_lbvh, minimum_lbvh.h:284-361)
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"
#include "climb.cuh"
#include "onesweep.cuh"

namespace mlbvh {

namespace {

constexpr int kBoundsThreads = 256;
constexpr int kBoundsMaxBlocks = 1024;
constexpr int kKeysThreads = 256;
constexpr int kSortTile = sort::kTile;  // 4096 keys per tile
constexpr int kBuildThreads = (int)kTileLeaves;
constexpr uint32_t kDefaultSpinLimit = 1u << 22;

// Scratch layout of one build (offsets from the caller's dScratch). The
// leading region [header, partials) is zeroed by k_scene_bounds on every build.
struct BuildLayout {
    size_t header;     // u32 error word, u32 tile counters[4]
    size_t histogram;  // 4 x 256 u32
    size_t lookback;   // 4 x tiles x 256 u32
    size_t partials;   // kBoundsMaxBlocks x 8 floats
    size_t keysA, keysB, valsA, valsB;
    size_t handoff;  // n u32
    size_t deltas;   // n u8
    size_t total;
    uint32_t tiles;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

BuildLayout build_layout(uint32_t n)
{
    BuildLayout L;
    L.tiles = (n + kSortTile - 1) / kSortTile;
    size_t o = 0;
    L.header = o;
    o += 256;
    L.histogram = o;
    o = align256(o + sizeof(uint32_t) * 4 * 256);
    L.lookback = o;
    o = align256(o + sizeof(uint32_t) * 4 * 256 * (size_t)L.tiles);
    L.partials = o;
    o = align256(o + sizeof(float) * 8 * kBoundsMaxBlocks);
    L.keysA = o;
    o = align256(o + sizeof(uint32_t) * (size_t)n);
    L.keysB = o;
    o = align256(o + sizeof(uint32_t) * (size_t)n);
    L.valsA = o;
    o = align256(o + sizeof(uint32_t) * (size_t)n);
    L.valsB = o;
    o = align256(o + sizeof(uint32_t) * (size_t)n);
    L.handoff = o;
    o = align256(o + sizeof(uint32_t) * (size_t)n);
    L.deltas = o;
    o = align256(o + (size_t)n);
    L.total = o;
    return L;
}


// ------------------------------------------------------------ kernels

// Partial bounds of the vertex soup per CTA. The triangles are read as a flat
// float array in 48-byte groups (three float4 = four vertices, axis pattern
// x y z x | y z x y | z x y z), then the scalar tail. Also zeroes the
// counters, histograms and look-back words the sort passes rely on.
__global__ void __launch_bounds__(kBoundsThreads)
    k_scene_bounds(const float* __restrict__ tris, uint32_t n, float* __restrict__ partials,
                   uint32_t* __restrict__ zeroBegin, size_t zeroWords)
{
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t nthreads = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i < zeroWords; i += nthreads) zeroBegin[i] = 0u;

    float lo[3] = {kFltMax, kFltMax, kFltMax};
    float hi[3] = {-kFltMax, -kFltMax, -kFltMax};
    const size_t nFloats = (size_t)n * 9;
    const size_t nGroups = nFloats / 12;
    const float4* t4 = reinterpret_cast<const float4*>(tris);
    for (size_t g = tid; g < nGroups; g += nthreads) {
        float4 a = __ldg(t4 + 3 * g), b = __ldg(t4 + 3 * g + 1), c = __ldg(t4 + 3 * g + 2);
        lo[0] = fminf(lo[0], fminf(fminf(a.x, a.w), fminf(b.z, c.y)));
        hi[0] = fmaxf(hi[0], fmaxf(fmaxf(a.x, a.w), fmaxf(b.z, c.y)));
        lo[1] = fminf(lo[1], fminf(fminf(a.y, b.x), fminf(b.w, c.z)));
        hi[1] = fmaxf(hi[1], fmaxf(fmaxf(a.y, b.x), fmaxf(b.w, c.z)));
        lo[2] = fminf(lo[2], fminf(fminf(a.z, b.y), fminf(c.x, c.w)));
        hi[2] = fmaxf(hi[2], fmaxf(fmaxf(a.z, b.y), fmaxf(c.x, c.w)));
    }
    for (size_t j = nGroups * 12 + tid; j < nFloats; j += nthreads) {
        float v = __ldg(tris + j);
        int ax = (int)(j % 3);
        lo[ax] = fminf(lo[ax], v);
        hi[ax] = fmaxf(hi[ax], v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    __shared__ float s_box[kBoundsThreads / 32][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            s_box[warp][a] = lo[a];
            s_box[warp][3 + a] = hi[a];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        float v = s_box[0][threadIdx.x];
        for (int w = 1; w < kBoundsThreads / 32; ++w)
            v = threadIdx.x < 3 ? fminf(v, s_box[w][threadIdx.x]) : fmaxf(v, s_box[w][threadIdx.x]);
        partials[blockIdx.x * 8 + threadIdx.x] = v;
    }
}

// Morton key per triangle (buildMortons, minimum_lbvh.cu:68-92) plus the four
// digit histograms of the sort. Triangles are staged through shared memory
// with 16-byte loads, 256 triangles (2304 floats) per step.
__global__ void __launch_bounds__(kKeysThreads)
    k_keys(const float* __restrict__ tris, uint32_t n, uint32_t option, const float* __restrict__ partials,
           int nPartials, uint32_t* __restrict__ keys, uint32_t* __restrict__ histogram,
           uint32_t* __restrict__ handoff, mlbvh_aabb* __restrict__ sceneOut)
{
    __shared__ float s_scene[6];
    __shared__ uint32_t s_hist[4][256];
    __shared__ __align__(16) float s_tri[kKeysThreads * 9];  // written with 16-byte stores

    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) (&s_hist[0][0])[i] = 0u;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        float lo[3] = {kFltMax, kFltMax, kFltMax}, hi[3] = {-kFltMax, -kFltMax, -kFltMax};
        for (int p = lane; p < nPartials; p += 32)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], partials[p * 8 + a]);
                hi[a] = fmaxf(hi[a], partials[p * 8 + 3 + a]);
            }
        for (int o = 16; o > 0; o >>= 1)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
            }
        if (lane == 0)
            for (int a = 0; a < 3; ++a) {
                s_scene[a] = lo[a];
                s_scene[3 + a] = hi[a];
            }
    }
    __syncthreads();
    if (blockIdx.x == 0 && sceneOut && threadIdx.x < 6) {
        float* out = reinterpret_cast<float*>(sceneOut);
        out[threadIdx.x] = s_scene[threadIdx.x];
    }
    const f3 lower = mk(s_scene[0], s_scene[1], s_scene[2]);
    const f3 upper = mk(s_scene[3], s_scene[4], s_scene[5]);

    const size_t gthreads = (size_t)gridDim.x * blockDim.x;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i + 1 < n; i += gthreads) handoff[i] = 0xFFFFFFFFu;

    const uint32_t nTiles = (n + kKeysThreads - 1) / kKeysThreads;
    for (uint32_t tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
        const size_t fbase = (size_t)tile * kKeysThreads * 9;
        const size_t fcount = min((size_t)kKeysThreads * 9, (size_t)n * 9 - fbase);
        const float4* src4 = reinterpret_cast<const float4*>(tris + fbase);
        const int n4 = (int)(fcount / 4);
        __syncthreads();
        for (int j = threadIdx.x; j < n4; j += kKeysThreads) reinterpret_cast<float4*>(s_tri)[j] = __ldg(src4 + j);
        for (int j = n4 * 4 + threadIdx.x; j < (int)fcount; j += kKeysThreads) s_tri[j] = __ldg(tris + fbase + j);
        __syncthreads();
        const uint32_t i = tile * kKeysThreads + threadIdx.x;
        if (i < n) {
            const float* t = s_tri + threadIdx.x * 9;
            f3 v0 = mk(t[0], t[1], t[2]), v1 = mk(t[3], t[4], t[5]), v2 = mk(t[6], t[7], t[8]);
            f3 center = (v0 + v1 + v2) / 3.0f;
            uint32_t key;
            if (option & MLBVH_BUILD_OPTION_USE_NORMAL) {
                f3 ng = normalize(cross(v1 - v0, v2 - v0));
                uint32_t nMorton = morton32(mk(-1, -1, -1), mk(1, 1, 1), ng);
                uint32_t pMorton = morton32(lower, upper, center);
                key = (pMorton & 0xFFFFFFC0u) | (nMorton >> 26);
            } else {
                key = morton32(lower, upper, center);
            }
            keys[i] = key;
#pragma unroll
            for (int d = 0; d < 4; ++d) atomicAdd(&s_hist[d][(key >> (8 * d)) & 255u], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(&histogram[i], c);
    }
}


// One thread per sorted leaf of the single-mesh build, one CTA per tile of
// kTileLeaves leaves (climb_tile: the tile's own nodes meet in shared memory).
static_assert(kBuildThreads == (int)kTileLeaves, "one thread per leaf of a tile");
__global__ void __launch_bounds__(kBuildThreads)
    k_build(const float* __restrict__ tris, uint32_t n, const uint32_t* __restrict__ sortedKeys,
            const uint32_t* __restrict__ sortedIdx, mlbvh_internal_node* __restrict__ nodes,
            uint32_t* __restrict__ handoff, mlbvh_node_index* __restrict__ root, uint8_t* __restrict__ deltas)
{
    __shared__ TileClimbShared sh;
    const uint32_t t0 = blockIdx.x * kTileLeaves;
    const uint32_t i = t0 + threadIdx.x;
    // tri >= n only after a sort whose bounded wait gave up (error word set)
    const uint32_t tri = i < n ? sortedIdx[i] : 0xFFFFFFFFu;
    f3 lo = mk(0.0f, 0.0f, 0.0f), hi = lo;
    if (tri < n) leaf_box(tris, n, tri, lo, hi);
    tile_climb_prepare(sh, sortedKeys, n, t0, 0u, n);
    if (tri >= n) return;
    climb_tile(sh, t0, n, i, tri, lo, hi, sortedKeys, nodes, handoff, root, deltas);
}

}  // namespace

size_t build_scratch_bytes(uint32_t n) { return build_layout(n).total; }

mlbvh_status sort_leaves(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, mlbvh_aabb* dScene,
                         uint32_t* dKeysOut, uint32_t* dIdxOut, uint8_t* dDeltasOut, void* dScratch,
                         cudaStream_t stream, uint32_t spinLimit, SortedLeaves* out)
{
    const BuildLayout L = build_layout(n);
    if (spinLimit == 0) spinLimit = kDefaultSpinLimit;
    char* s = static_cast<char*>(dScratch);
    uint32_t* header = reinterpret_cast<uint32_t*>(s + L.header);
    float* partials = reinterpret_cast<float*>(s + L.partials);
    uint32_t* hist = reinterpret_cast<uint32_t*>(s + L.histogram);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(s + L.lookback);
    uint32_t* keysA = reinterpret_cast<uint32_t*>(s + L.keysA);
    uint32_t* keysB = reinterpret_cast<uint32_t*>(s + L.keysB);
    uint32_t* valsA = reinterpret_cast<uint32_t*>(s + L.valsA);
    uint32_t* valsB = reinterpret_cast<uint32_t*>(s + L.valsB);
    uint32_t* handoff = reinterpret_cast<uint32_t*>(s + L.handoff);
    uint32_t* keysFinal = dKeysOut ? dKeysOut : keysA;
    uint32_t* valsFinal = dIdxOut ? dIdxOut : valsA;
    const float* tris = reinterpret_cast<const float*>(dTris);

    const int sms = device_sm_count();
    const size_t zeroWords = (L.partials - L.header) / 4;
    int boundsBlocks = (int)std::min<size_t>((size_t)kBoundsMaxBlocks,
                                             std::max<size_t>(1, ((size_t)n * 9 / 12 + kBoundsThreads - 1) / kBoundsThreads));
    boundsBlocks = std::min(boundsBlocks, 4 * sms);
    k_scene_bounds<<<boundsBlocks, kBoundsThreads, 0, stream>>>(tris, n, partials, header, zeroWords);
    MLBVH_CHECK_LAUNCH("k_scene_bounds");
    const int keysBlocks = std::max(1, std::min<int>((n + kKeysThreads - 1) / kKeysThreads, 8 * sms));
    k_keys<<<keysBlocks, kKeysThreads, 0, stream>>>(tris, n, option, partials, boundsBlocks, keysA, hist, handoff,
                                                    dScene);
    MLBVH_CHECK_LAUNCH("k_keys");

    uint32_t* kin = keysA;
    uint32_t* vin = valsA;
    constexpr size_t kSmem = sort::Shape<8>::kSmemBytes;
    for (int pass = 0; pass < 4; ++pass) {
        uint32_t* kout = (pass == 3) ? keysFinal : (pass % 2 == 0 ? keysB : keysA);
        uint32_t* vout = (pass == 3) ? valsFinal : (pass % 2 == 0 ? valsB : valsA);
        const sort::SingleSegment seg{n, L.tiles, hist + 256 * pass};
        uint32_t* lb = lookback + (size_t)pass * L.tiles * 256;
        if (pass == 0)
            sort::k_onesweep<8, true><<<L.tiles, sort::kThreads, kSmem, stream>>>(kin, kout, nullptr, vout, 8 * pass,
                                                                                seg, lb, header + 1 + pass, header,
                                                                                spinLimit);
        else
            sort::k_onesweep<8, false><<<L.tiles, sort::kThreads, kSmem, stream>>>(kin, kout, vin, vout, 8 * pass,
                                                                                 seg, lb, header + 1 + pass, header,
                                                                                 spinLimit);
        MLBVH_CHECK_LAUNCH("k_onesweep");
        kin = kout;
        vin = vout;
    }
    out->keys = keysFinal;
    out->indices = valsFinal;
    out->error = header;
    out->handoff = handoff;
    out->deltas = dDeltasOut ? dDeltasOut : reinterpret_cast<uint8_t*>(s + L.deltas);
    out->spinLimit = spinLimit;
    return MLBVH_OK;
}

mlbvh_status build(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, mlbvh_internal_node* dNodes,
                   mlbvh_node_index* dRoot, mlbvh_aabb* dScene, uint32_t* dKeysOut, uint32_t* dIdxOut,
                   uint8_t* dDeltasOut, void* dScratch, size_t scratchBytes, cudaStream_t stream, uint32_t spinLimit)
{
    if (n == 0 || n >= (1u << 30)) return fail(MLBVH_ERR_INVALID_ARG, "nTriangles must be in [1, 2^30)");
    if (!dTris || !dRoot || !dScratch) return fail(MLBVH_ERR_INVALID_ARG, "null triangles, root or scratch pointer");
    if (n > 1 && !dNodes) return fail(MLBVH_ERR_INVALID_ARG, "null internal-node pointer");
    if (!aligned16(dTris) || !aligned16(dNodes) || !aligned16(dScratch) || !aligned16(dRoot) || !aligned16(dScene) ||
        !aligned16(dKeysOut) || !aligned16(dIdxOut) || !aligned16(dDeltasOut))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (scratchBytes < build_layout(n).total)
        return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_build_scratch_bytes(n)");
    SortedLeaves sl;
    mlbvh_status st = sort_leaves(dTris, n, option, dScene, dKeysOut, dIdxOut, dDeltasOut, dScratch, stream,
                                  spinLimit, &sl);
    if (st != MLBVH_OK) return st;
    ProfileEvents ev = take_profile_events();
    if (ev.start) cudaEventRecord(ev.start, stream);
    k_build<<<(n + kBuildThreads - 1) / kBuildThreads, kBuildThreads, 0, stream>>>(
        reinterpret_cast<const float*>(dTris), n, sl.keys, sl.indices, dNodes, sl.handoff, dRoot, sl.deltas);
    MLBVH_CHECK_LAUNCH("k_build");
    if (ev.stop) cudaEventRecord(ev.stop, stream);
    return MLBVH_OK;
}

mlbvh_status scratch_status(const void* dScratch, cudaStream_t stream)
{
    if (!dScratch) return fail(MLBVH_ERR_INVALID_ARG, "null scratch pointer");
    uint32_t word = 0;
    cudaError_t e = cudaMemcpyAsync(&word, dScratch, sizeof(word), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    if (word & 2u)
        return fail(MLBVH_ERR_INVALID_ARG, "batch triangle offsets are not 0 = o[0] < o[1] < ... < o[nMeshes] = "
                                           "nTriangles; nothing was built");
    if (word) return fail(MLBVH_ERR_TIMEOUT, "a bounded device wait gave up; the output of that call is unusable");
    return MLBVH_OK;
}

}  // namespace mlbvh
