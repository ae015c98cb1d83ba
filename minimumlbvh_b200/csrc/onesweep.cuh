// One stable LSD radix-sort pass of (32-bit key, 32-bit value) pairs, shared
// by the single-mesh build (one segment: the whole array) and the batched
// build (one segment per mesh, sorted independently in the same launch).
//
// The pass is Onesweep (Adinets & Merrill, "Onesweep: A Faster Least
// Significant Digit Radix Sort for GPUs", 2022) over tiles of 4096 keys:
// a tile ranks its keys with a warp multisplit (one ballot per digit bit),
// publishes its per-digit counts, resolves its global offsets by decoupled
// look-back over the earlier tiles of its segment, then scatters through
// shared memory so that runs of one digit store coalesced. Tiles are
// ticketed in launch order (an atomic counter), so every tile a CTA waits on
// belongs to a CTA that has already started. Every wait is bounded: after
// spinLimit polls the error word is set and the pass goes on with a wrong
// prefix instead of hanging; the scatter then drops out-of-segment indices.
//
// This replaces the reference's onesweep_count / onesweep_reorder
// (tinyhiponesweep.h:136-192, 204-502), which sort 8-byte IndexedMorton
// structs as 64-bit keys over bits [0, 32) with 8-bit digits; here keys and
// values are separate arrays, the digit width is 8 or 11 bits, and a tile
// never straddles a segment.
#pragma once

#include <cstdint>

namespace mlbvh {
namespace sort {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096 keys per tile
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;

template <int kBits>
struct Shape {
    static_assert(kBits == 8 || kBits == 11, "digit width must be 8 or 11 bits");
    static constexpr int kBins = 1 << kBits;
    static constexpr int kDigitsPerThread = kBins / kThreads;
    static constexpr int kPasses = (32 + kBits - 1) / kBits;
    // dynamic shared memory: per-warp digit counts (reused for the scatter
    // destinations), tile-exclusive digit offsets, staged keys and values
    static constexpr size_t kSmemBytes = sizeof(uint32_t) * ((size_t)kWarps * kBins + kBins + 2 * (size_t)kTile);
};

// One segment as a tile sees it.
struct Segment {
    uint32_t start;            // first key of the segment
    uint32_t len;              // keys in the segment
    uint32_t firstTile;        // tile id of the segment's first tile
    const uint32_t* counts;    // the segment's digit counts for this pass (kBins)
};

// The whole array is one segment of n keys; tile ids 0 .. ceil(n / kTile) - 1.
struct SingleSegment {
    uint32_t n;
    uint32_t tiles;
    const uint32_t* counts;
    __device__ __forceinline__ bool resolve(uint32_t tile, Segment& s) const
    {
        if (tile >= tiles) return false;
        s.start = 0;
        s.len = n;
        s.firstTile = 0;
        s.counts = counts;
        return true;
    }
};

// Segment m holds keys [offsets[m], offsets[m + 1]) and tiles
// [tileStart[m], tileStart[m + 1]); every segment has at least one key, so
// tileStart is strictly increasing and tileStart[nSegments] is the number of
// tiles. Digit counts of segment m for this pass sit at counts + m * stride.
struct MeshSegments {
    const uint32_t* offsets;
    const uint32_t* tileStart;
    uint32_t nSegments;
    const uint32_t* counts;
    uint32_t stride;
    __device__ __forceinline__ bool resolve(uint32_t tile, Segment& s) const
    {
        if (tile >= __ldcg(tileStart + nSegments)) return false;
        uint32_t lo = 0, hi = nSegments;  // tileStart[lo] <= tile < tileStart[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldcg(tileStart + mid) <= tile)
                lo = mid;
            else
                hi = mid;
        }
        s.start = __ldcg(offsets + lo);
        s.len = __ldcg(offsets + lo + 1) - s.start;
        s.firstTile = __ldcg(tileStart + lo);
        s.counts = counts + (size_t)lo * stride;
        return true;
    }
};

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

// Exclusive scan of one value per thread over a block of kThreads threads;
// *total receives the sum over the block.
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* s_warp /*kWarps*/, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t base = 0, sum = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t x = s_warp[w];
        base += w < warp ? x : 0u;
        sum += x;
    }
    __syncthreads();
    *total = sum;
    return base + inc - v;
}

// One pass over digit (key >> shift) & (2^kBits - 1). Launch with at least
// as many CTAs as tiles (extra CTAs exit), kThreads threads and
// Shape<kBits>::kSmemBytes of dynamic shared memory. kFirst: the values are
// the keys' positions within their segment (valsIn unused). The 8-bit passes
// are held to three resident CTAs per SM (at most 85 registers): the pass is
// latency-bound and more tiles in flight shorten it (measured 3 % on a 4M
// build); the 11-bit passes are limited by shared memory to two anyway.
template <int kBits, bool kFirst, class Segments>
__global__ void __launch_bounds__(kThreads, kBits == 8 ? 3 : 1)
    k_onesweep(const uint32_t* __restrict__ keysIn, uint32_t* __restrict__ keysOut,
               const uint32_t* __restrict__ valsIn, uint32_t* __restrict__ valsOut, int shift, Segments segs,
               uint32_t* __restrict__ lookback, uint32_t* __restrict__ tileCounter, uint32_t* __restrict__ errorWord,
               uint32_t spinLimit)
{
    using S = Shape<kBits>;
    constexpr int kBins = S::kBins, kDPT = S::kDigitsPerThread;
    constexpr uint32_t kMask = (uint32_t)kBins - 1u;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* s_warpHist = smem;                  // [kWarps][kBins]
    uint32_t* s_tileExcl = smem + kWarps * kBins;  // [kBins]
    uint32_t* s_keys = s_tileExcl + kBins;         // [kTile]
    uint32_t* s_vals = s_keys + kTile;             // [kTile]
    __shared__ uint32_t s_tile, s_ok;
    __shared__ Segment s_seg;
    __shared__ uint32_t s_scan[kWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const uint32_t t = atomicAdd(tileCounter, 1u);
        Segment sg;
        s_ok = segs.resolve(t, sg) ? 1u : 0u;
        s_seg = sg;
        s_tile = t;
    }
    for (int i = tid; i < kWarps * kBins; i += kThreads) s_warpHist[i] = 0u;
    __syncthreads();
    if (!s_ok) return;
    const uint32_t tile = s_tile;
    const Segment seg = s_seg;
    const uint32_t chunk = tile - seg.firstTile;

    // global start of every digit of this thread (digit d = j * kThreads + tid)
    uint32_t digitBase[kDPT], count[kDPT];
    {
        uint32_t running = seg.start;
#pragma unroll
        for (int j = 0; j < kDPT; ++j) {
            uint32_t total;
            const uint32_t excl = block_scan(__ldg(seg.counts + j * kThreads + tid), s_scan, &total);
            digitBase[j] = running + excl;
            running += total;
        }
    }

    const uint32_t localBase = chunk * (uint32_t)kTile + (uint32_t)warp * (kItems * 32);
    uint32_t key[kItems], val[kItems], rank[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t li = localBase + k * 32 + lane;
        const bool valid = li < seg.len;
        key[k] = valid ? __ldg(keysIn + seg.start + li) : 0xFFFFFFFFu;
        val[k] = kFirst ? li : (valid ? __ldg(valsIn + seg.start + li) : 0u);
    }
    const uint32_t lanesBelow = (1u << lane) - 1u;
    uint32_t* myHist = s_warpHist + warp * kBins;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t li = localBase + k * 32 + lane;
        const uint32_t d = (key[k] >> shift) & kMask;
        uint32_t peers = __ballot_sync(0xffffffffu, li < seg.len);
#pragma unroll
        for (int b = 0; b < kBits; ++b) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t m = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? m : ~m;
        }
        const uint32_t before = myHist[d];
        rank[k] = before + __popc(peers & lanesBelow);
        __syncwarp();
        if (li < seg.len && lane == __ffs(peers) - 1) myHist[d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // per digit: offsets of the warps within the tile, and the tile's count
#pragma unroll
    for (int j = 0; j < kDPT; ++j) {
        const int d = j * kThreads + tid;
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t x = s_warpHist[w * kBins + d];
            s_warpHist[w * kBins + d] = c;
            c += x;
        }
        count[j] = c;
    }

    // decoupled look-back over the earlier tiles of this segment
    uint32_t prefix[kDPT];
#pragma unroll
    for (int j = 0; j < kDPT; ++j) {
        prefix[j] = 0;
        st_relaxed(lookback + (size_t)tile * kBins + j * kThreads + tid,
                   (chunk == 0 ? kFlagPrefix : kFlagAggregate) | count[j]);
    }
    if (chunk != 0) {
        uint32_t done = 0;
        constexpr uint32_t kAll = (1u << kDPT) - 1u;
        for (uint32_t t = tile - 1;; --t) {
            const uint32_t* row = lookback + (size_t)t * kBins + tid;
            uint32_t w[kDPT];
#pragma unroll
            for (int j = 0; j < kDPT; ++j) w[j] = ((done >> j) & 1u) ? kFlagPrefix : ld_relaxed(row + j * kThreads);
            uint32_t spins = 0;
            for (;;) {
                bool pending = false;
#pragma unroll
                for (int j = 0; j < kDPT; ++j) pending |= (w[j] >> 30) == 0u;
                if (!pending) break;
                if (++spins > spinLimit) {
                    atomicOr(errorWord, 1u);
#pragma unroll
                    for (int j = 0; j < kDPT; ++j)
                        if ((w[j] >> 30) == 0u) w[j] = kFlagPrefix;
                    break;
                }
                __nanosleep(32);
#pragma unroll
                for (int j = 0; j < kDPT; ++j)
                    if ((w[j] >> 30) == 0u) w[j] = ld_relaxed(row + j * kThreads);
            }
#pragma unroll
            for (int j = 0; j < kDPT; ++j)
                if (!((done >> j) & 1u)) {
                    prefix[j] += w[j] & kValueMask;
                    if ((w[j] >> 30) == 2u) done |= 1u << j;
                }
            if (done == kAll || t == seg.firstTile) break;
        }
#pragma unroll
        for (int j = 0; j < kDPT; ++j)
            st_relaxed(lookback + (size_t)tile * kBins + j * kThreads + tid,
                       kFlagPrefix | ((prefix[j] + count[j]) & kValueMask));
    }

    // tile-exclusive digit offsets; destination of tile position i of digit d
    // is dest[d] + i
    uint32_t dest[kDPT];
    {
        uint32_t running = 0;
#pragma unroll
        for (int j = 0; j < kDPT; ++j) {
            uint32_t total;
            const uint32_t excl = running + block_scan(count[j], s_scan, &total);
            running += total;
            s_tileExcl[j * kThreads + tid] = excl;
            dest[j] = digitBase[j] + prefix[j] - excl;
        }
    }
    __syncthreads();

    // place every key at its tile-sorted position in shared memory
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t li = localBase + k * 32 + lane;
        if (li < seg.len) {
            const uint32_t dk = (key[k] >> shift) & kMask;
            const uint32_t pos = s_tileExcl[dk] + myHist[dk] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kDPT; ++j) s_warpHist[j * kThreads + tid] = dest[j];
    __syncthreads();
    const uint32_t inTile = min((uint32_t)kTile, seg.len - chunk * (uint32_t)kTile);
    for (uint32_t i = tid; i < inTile; i += kThreads) {
        const uint32_t k = s_keys[i];
        const uint32_t dst = s_warpHist[(k >> shift) & kMask] + i;
        if (dst - seg.start < seg.len) {  // always true unless a bounded wait gave up (error word set)
            keysOut[dst] = k;
            valsOut[dst] = s_vals[i];
        }
    }
}

}  // namespace sort
}  // namespace mlbvh
