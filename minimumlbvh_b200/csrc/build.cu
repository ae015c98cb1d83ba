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

namespace mlbvh {

namespace {

constexpr int kBoundsThreads = 256;
constexpr int kBoundsMaxBlocks = 1024;
constexpr int kKeysThreads = 256;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kBuildThreads = 256;
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
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

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t exch_acq_rel(uint32_t* p, uint32_t v)
{
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan256(uint32_t v, uint32_t* s_warp /*8 entries*/)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < warp; ++w) base += s_warp[w];
    __syncthreads();
    return base + inc - v;
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

// One stable counting pass of the LSD sort over digit (key >> shift) & 255.
// Tile t (4096 keys, ticketed in launch order so every tile a CTA waits on has
// already started) ranks its keys with an 8-ballot warp multisplit, publishes
// its per-digit counts, and resolves its global offsets by decoupled look-back
// over earlier tiles (Merrill & Garland; Adinets & Merrill, "Onesweep", 2022).
// Every wait is bounded: on expiry the error word is set and the pass goes on
// with a wrong prefix instead of hanging.
template <bool kFirst>
__global__ void __launch_bounds__(kSortThreads)
    k_onesweep(const uint32_t* __restrict__ keysIn, uint32_t* __restrict__ keysOut,
               const uint32_t* __restrict__ valsIn, uint32_t* __restrict__ valsOut, uint32_t n, int shift,
               const uint32_t* __restrict__ digitCounts, uint32_t* __restrict__ lookback,
               uint32_t* __restrict__ tileCounter, uint32_t* __restrict__ errorWord, uint32_t spinLimit)
{
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warpHist[kSortWarps][256];
    __shared__ uint32_t s_tileExcl[256];
    __shared__ uint32_t s_dest[256];
    __shared__ uint32_t s_scan[kSortWarps];
    __shared__ uint32_t s_keys[kSortTile];
    __shared__ uint32_t s_vals[kSortTile];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tileCounter, 1u);
    for (int i = tid; i < kSortWarps * 256; i += kSortThreads) (&s_warpHist[0][0])[i] = 0u;
    // global base offset of each digit for this pass
    const uint32_t digitBase = block_exclusive_scan256(digitCounts[tid], s_scan);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * (uint32_t)kSortTile + (uint32_t)warp * (kSortItems * 32);

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        const bool valid = idx < n;
        key[k] = valid ? __ldg(keysIn + idx) : 0xFFFFFFFFu;
        val[k] = kFirst ? idx : (valid ? __ldg(valsIn + idx) : 0u);
    }
    const uint32_t lanesBelow = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        const uint32_t d = (key[k] >> shift) & 255u;
        uint32_t peers = __ballot_sync(0xffffffffu, idx < n);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t m = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? m : ~m;
        }
        const uint32_t before = s_warpHist[warp][d];
        rank[k] = before + __popc(peers & lanesBelow);
        __syncwarp();
        if (idx < n && lane == __ffs(peers) - 1) s_warpHist[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // per digit (one per thread): warp offsets and the tile's count
    const uint32_t d = (uint32_t)tid;
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = s_warpHist[w][d];
        s_warpHist[w][d] = count;
        count += c;
    }
    uint32_t* myWord = lookback + (size_t)tile * 256 + d;
    uint32_t prefix = 0;
    if (tile == 0) {
        st_relaxed(myWord, kFlagPrefix | count);
    } else {
        st_relaxed(myWord, kFlagAggregate | count);
        int t = (int)tile - 1;
        while (t >= 0) {
            const uint32_t* w = lookback + (size_t)t * 256 + d;
            uint32_t word = ld_relaxed(w);
            uint32_t spins = 0;
            while ((word >> 30) == 0u) {
                if (++spins > spinLimit) {
                    atomicOr(errorWord, 1u);
                    word = kFlagPrefix;
                    break;
                }
                __nanosleep(32);
                word = ld_relaxed(w);
            }
            prefix += word & kValueMask;
            if ((word >> 30) == 2u) break;
            --t;
        }
        st_relaxed(myWord, kFlagPrefix | ((prefix + count) & kValueMask));
    }
    const uint32_t excl = block_exclusive_scan256(count, s_scan);
    s_tileExcl[d] = excl;
    s_dest[d] = digitBase + prefix - excl;
    __syncthreads();

    // place every key at its tile-sorted position in shared memory
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        if (idx < n) {
            const uint32_t dk = (key[k] >> shift) & 255u;
            const uint32_t pos = s_tileExcl[dk] + s_warpHist[warp][dk] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
    const uint32_t tileStart = tile * (uint32_t)kSortTile;
    const uint32_t count_in_tile = min((uint32_t)kSortTile, n - tileStart);
    for (uint32_t i = tid; i < count_in_tile; i += kSortThreads) {
        const uint32_t k = s_keys[i];
        const uint32_t dst = s_dest[(k >> shift) & 255u] + i;
        if (dst < n) {  // always true unless a bounded wait gave up (error word set)
            keysOut[dst] = k;
            valsOut[dst] = s_vals[i];
        }
    }
}

__device__ __forceinline__ uint32_t delta_at(const uint32_t* __restrict__ keys, uint32_t i)
{
    return split_delta(keys[i], keys[i + 1]);
}

// build_lbvh (minimum_lbvh.h:284-361), one thread per sorted leaf. The
// hand-off word per internal node lives in its own array (reset by k_keys)
// and is exchanged with acquire-release semantics, so the first walker's
// child slot is visible to the second; the sibling bounds are then read from
// L2. The merged box is formed as max/min(box of child 1, box of child 0)
// whichever walker arrives second, which is the order the reference's serial
// CPU build produces (its second arrival always comes from the right).
__global__ void __launch_bounds__(kBuildThreads)
    k_build(const float* __restrict__ tris, uint32_t n, const uint32_t* __restrict__ sortedKeys,
            const uint32_t* __restrict__ sortedIdx, mlbvh_internal_node* __restrict__ nodes,
            uint32_t* __restrict__ handoff, mlbvh_node_index* __restrict__ root, uint8_t* __restrict__ deltas)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t nInternals = n - 1;
    const uint32_t tri = sortedIdx[i];
    if (tri >= n) return;  // only after a sort whose bounded wait gave up (error word set)
    if (deltas && i < nInternals) deltas[i] = (uint8_t)delta_at(sortedKeys, i);

    f3 v0, v1, v2;
    load_triangle(tris, tri, v0, v1, v2);
    f3 lo = mk(kFltMax, kFltMax, kFltMax), hi = mk(-kFltMax, -kFltMax, -kFltMax);
    lo = smin3(lo, v0);
    hi = smax3(hi, v0);
    lo = smin3(lo, v1);
    hi = smax3(hi, v1);
    lo = smin3(lo, v2);
    hi = smax3(hi, v2);

    uint32_t leafLower = i, leafUpper = i;
    uint32_t node = tri | kLeafBit;
    while (leafUpper - leafLower < nInternals) {
        const uint32_t deltaL = 0 < leafLower ? delta_at(sortedKeys, leafLower - 1) : 0xFFFFFFFFu;
        const uint32_t deltaR = leafUpper < nInternals ? delta_at(sortedKeys, leafUpper) : 0xFFFFFFFFu;
        const int goLeft = deltaL < deltaR ? 1 : 0;
        const uint32_t parent = goLeft ? leafLower - 1 : leafUpper;

        mlbvh_internal_node* p = nodes + parent;
        p->children[goLeft] = node;
        float* box = p->aabbs[goLeft].lower;
        box[0] = lo.x;
        box[1] = lo.y;
        box[2] = lo.z;
        box[3] = hi.x;
        box[4] = hi.y;
        box[5] = hi.z;
        if (!(node & kLeafBit)) nodes[node].parent = parent;

        uint32_t other = exch_acq_rel(handoff + parent, goLeft ? leafUpper : leafLower);
        if (other == 0xFFFFFFFFu) return;  // first arrival: the sibling finishes this node

        leafLower = min(leafLower, other);
        leafUpper = max(leafUpper, other);
        p->context = leafUpper < nInternals ? leafUpper : 0xFFFFFFFFu;
        const float* ob = p->aabbs[goLeft ^ 1].lower;
        const f3 olo = mk(__ldcg(ob + 0), __ldcg(ob + 1), __ldcg(ob + 2));
        const f3 ohi = mk(__ldcg(ob + 3), __ldcg(ob + 4), __ldcg(ob + 5));
        if (goLeft) {  // this walker is child 1
            lo = smin3(lo, olo);
            hi = smax3(hi, ohi);
        } else {
            lo = smin3(olo, lo);
            hi = smax3(ohi, hi);
        }
        node = parent;
    }
    *root = node;
    if (!(node & kLeafBit)) nodes[node].parent = kInvalid;
}

}  // namespace

size_t build_scratch_bytes(uint32_t n) { return build_layout(n).total; }

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
    const BuildLayout L = build_layout(n);
    if (scratchBytes < L.total) return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_build_scratch_bytes(n)");
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
    uint8_t* deltas = dDeltasOut ? dDeltasOut : reinterpret_cast<uint8_t*>(s + L.deltas);
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
    for (int pass = 0; pass < 4; ++pass) {
        uint32_t* kout = (pass == 3) ? keysFinal : (pass % 2 == 0 ? keysB : keysA);
        uint32_t* vout = (pass == 3) ? valsFinal : (pass % 2 == 0 ? valsB : valsA);
        if (pass == 0)
            k_onesweep<true><<<L.tiles, kSortThreads, 0, stream>>>(kin, kout, nullptr, vout, n, 8 * pass,
                                                                    hist + 256 * pass, lookback + (size_t)pass * L.tiles * 256,
                                                                    header + 1 + pass, header, spinLimit);
        else
            k_onesweep<false><<<L.tiles, kSortThreads, 0, stream>>>(kin, kout, vin, vout, n, 8 * pass,
                                                                     hist + 256 * pass, lookback + (size_t)pass * L.tiles * 256,
                                                                     header + 1 + pass, header, spinLimit);
        MLBVH_CHECK_LAUNCH("k_onesweep");
        kin = kout;
        vin = vout;
    }
    ProfileEvents ev = take_profile_events();
    if (ev.start) cudaEventRecord(ev.start, stream);
    k_build<<<(n + kBuildThreads - 1) / kBuildThreads, kBuildThreads, 0, stream>>>(tris, n, keysFinal, valsFinal, dNodes,
                                                                                   handoff, dRoot, deltas);
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
    if (word) return fail(MLBVH_ERR_TIMEOUT, "a bounded device wait gave up; the output of that call is unusable");
    return MLBVH_OK;
}

}  // namespace mlbvh
