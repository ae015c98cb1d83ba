// Batched form (no reference counterpart): many independent meshes of uneven
// size built by one launch chain, and their rays drained by one persistent
// work-queue traversal kernel.
//
// Every mesh's tree is bit-identical to what mlbvh_build makes of that mesh
// alone: the same Morton keys over the mesh's own bounds, the same stable
// sort order (key, then position in the mesh), the same agglomerative climb.
// Meshes are laid out back to back: mesh m owns triangles [o[m], o[m+1]),
// internal nodes [o[m] - m, o[m+1] - m - 1) and root roots[m]; node and leaf
// indices inside a tree are local to its mesh.
//
// Build chain on one stream (no host synchronisation):
//   k_batch_plan      one CTA: checks the offsets, numbers every mesh's sort
//                     tiles (4096 triangles each, never straddling a mesh),
//                     resets the per-mesh bounds and the tile tickets
//   k_batch_bounds    per tile: bounds of its triangles, merged into the
//                     mesh's bounds with order-preserving integer atomics;
//                     zeroes the histograms and look-back words
//   k_batch_keys      per tile: Morton keys over the mesh's bounds, digit
//                     histograms per mesh, reset of the hand-off words
//   k_onesweep x P    segmented Onesweep passes (onesweep.cuh), one segment
//                     per mesh; P = 4 (8-bit digits) or 3 (11-bit digits)
//   k_batch_build     one thread per sorted leaf: the tile climb of mlbvh_build
//
// Traversal: k_batch_trace is persistent (one grid of resident CTAs). A warp
// takes `queueChunk` consecutive rays per atomic on the queue counter and
// hands them to its idle lanes; every lane walks its own ray one node per
// loop iteration (the stack-free walk of intersect_stackfree, or the replay
// walk that gives the same Hit records from a stack of pending far children)
// and takes the next ray as soon as it finishes, so lanes never wait for the
// longest ray of the warp. Rays find their mesh through the ray offsets.
#include <algorithm>
#include <cstring>
#include <vector>

#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"
#include "climb.cuh"
#include "onesweep.cuh"

namespace mlbvh {

namespace {

constexpr int kPlanThreads = 1024;
constexpr int kTileThreads = 256;  // bounds / keys kernels: one CTA per sort tile
constexpr int kStageTris = 256;    // triangles staged in shared memory per step
constexpr int kBuildThreads = (int)kTileLeaves;  // build: one CTA per tile of the climb
constexpr uint32_t kDefaultSpinLimit = 1u << 22;
constexpr uint32_t kMaxMeshes = 1u << 20;
// error word bits: 1 a bounded wait gave up (set by sort::k_onesweep), 2 bad offsets
constexpr uint32_t kErrOffsets = 2u;

// header words
constexpr int kHdrError = 0;
constexpr int kHdrTickets = 1;  // 4 tile tickets, one per sort pass
constexpr int kHdrQueue = 8;    // traversal queue counter

struct BatchLayout {
    size_t header;     // 64 u32
    size_t tileStart;  // nMeshes + 1 u32
    size_t bounds;     // nMeshes x 6 u32 (order-preserving integer form)
    size_t histogram;  // nMeshes x passes x bins u32
    size_t lookback;   // passes x maxTiles x bins u32
    size_t zeroEnd;    // [histogram, zeroEnd) is zeroed by k_batch_bounds
    size_t keysA, keysB, valsA, valsB, handoff;
    size_t total;
    uint32_t maxTiles;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

BatchLayout batch_layout(uint32_t nMeshes, uint32_t n, int bits)
{
    const int bins = 1 << bits, passes = (32 + bits - 1) / bits;
    BatchLayout L;
    L.maxTiles = (uint32_t)((n + (uint32_t)sort::kTile - 1) / (uint32_t)sort::kTile) + nMeshes;
    size_t o = 0;
    L.header = o;
    o += 256;
    L.tileStart = o;
    o = align256(o + sizeof(uint32_t) * ((size_t)nMeshes + 1));
    L.bounds = o;
    o = align256(o + sizeof(uint32_t) * 6 * (size_t)nMeshes);
    L.histogram = o;
    o = align256(o + sizeof(uint32_t) * (size_t)nMeshes * passes * bins);
    L.lookback = o;
    o = align256(o + sizeof(uint32_t) * (size_t)passes * L.maxTiles * bins);
    L.zeroEnd = o;
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
    L.total = o;
    return L;
}

// IEEE floats as unsigned integers in the same order (negative values
// reversed below the positive ones), so that atomicMin / atomicMax on the
// integers are min / max on the floats; -0 orders below +0.
__device__ __forceinline__ uint32_t ordered(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// Mesh of sorted position / tile / ray x: the largest m with off[m] <= x,
// for off[0] <= x < off[count].
__device__ __forceinline__ uint32_t find_segment(const uint32_t* __restrict__ off, uint32_t count, uint32_t x)
{
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Exclusive scan over a block of kPlanThreads threads; *total gets the sum.
__device__ __forceinline__ uint32_t plan_scan(uint32_t v, uint32_t* s_warp /*32*/, uint32_t* total)
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
    if (warp == 0) {
        uint32_t w = s_warp[lane], wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        s_warp[lane] = wi - w;
        if (lane == 31) s_warp[32] = wi;
    }
    __syncthreads();
    const uint32_t r = s_warp[warp] + inc - v;
    *total = s_warp[32];
    __syncthreads();
    return r;
}

// Checks o[0] = 0, o[nMeshes] = n and o[m+1] > o[m] (every mesh non-empty);
// numbers the sort tiles of every mesh (tileStart = exclusive prefix of
// ceil(n_m / 4096), tileStart[nMeshes] = total, 0 on bad offsets); resets the
// mesh bounds, the error word and the tile tickets.
__global__ void __launch_bounds__(kPlanThreads)
    k_batch_plan(const uint32_t* __restrict__ off, uint32_t nMeshes, uint32_t n, uint32_t* __restrict__ header,
                 uint32_t* __restrict__ tileStart, uint32_t* __restrict__ bounds)
{
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_bad;
    if (threadIdx.x == 0) s_bad = (__ldg(off) != 0u || __ldg(off + nMeshes) != n) ? 1u : 0u;
    if (threadIdx.x < 8) header[threadIdx.x] = 0u;  // error word and tile tickets
    if (threadIdx.x == kHdrQueue) header[kHdrQueue] = 0u;
    __syncthreads();
    for (uint32_t m = threadIdx.x; m < nMeshes; m += kPlanThreads)
        if (__ldg(off + m + 1) <= __ldg(off + m)) s_bad = 1u;
    __syncthreads();
    const bool bad = s_bad != 0u;
    uint32_t running = 0;
    for (uint32_t m0 = 0; m0 < nMeshes; m0 += kPlanThreads) {
        const uint32_t m = m0 + threadIdx.x;
        uint32_t tiles = 0;
        if (!bad && m < nMeshes) {
            const uint32_t len = __ldg(off + m + 1) - __ldg(off + m);
            tiles = (len + (uint32_t)sort::kTile - 1) / (uint32_t)sort::kTile;
        }
        uint32_t total;
        const uint32_t excl = plan_scan(tiles, s_warp, &total);
        if (m < nMeshes) tileStart[m] = running + excl;
        running += total;
    }
    if (threadIdx.x == 0) {
        tileStart[nMeshes] = running;
        if (bad) header[kHdrError] = kErrOffsets;
    }
    for (uint32_t i = threadIdx.x; i < 6 * nMeshes; i += kPlanThreads) bounds[i] = (i % 6) < 3 ? 0xFFFFFFFFu : 0u;
}

// Copies floats [f0, f0 + count) of src into s[0, count) with 16-byte loads
// over the aligned span that covers them (src is 16-byte aligned and holds
// fEnd floats).
__device__ __forceinline__ void stage_floats(float* s, const float* __restrict__ src, size_t f0, int count,
                                             size_t fEnd)
{
    const size_t a0 = f0 & ~(size_t)3;
    const int lead = (int)(f0 - a0);
    const int n4 = (lead + count + 3) >> 2;
    for (int j = threadIdx.x; j < n4; j += blockDim.x) {
        const size_t g = a0 + 4 * (size_t)j;
        float v[4];
        if (g + 4 <= fEnd) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(src + g));
            v[0] = x.x;
            v[1] = x.y;
            v[2] = x.z;
            v[3] = x.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = g + k < fEnd ? __ldg(src + g + k) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int o = 4 * j + k - lead;
            if (o >= 0 && o < count) s[o] = v[k];
        }
    }
}

// The tile a CTA works on: mesh, the mesh's triangle range, the tile's range.
struct TileWork {
    uint32_t mesh, start, len, first, count;
};
__device__ __forceinline__ bool tile_work(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tileStart,
                                          uint32_t nMeshes, uint32_t tile, TileWork& w)
{
    if (tile >= __ldg(tileStart + nMeshes)) return false;
    w.mesh = find_segment(tileStart, nMeshes, tile);
    w.start = __ldg(off + w.mesh);
    w.len = __ldg(off + w.mesh + 1) - w.start;
    w.first = (tile - __ldg(tileStart + w.mesh)) * (uint32_t)sort::kTile;
    w.count = min((uint32_t)sort::kTile, w.len - w.first);
    return true;
}

// Per tile: the bounds of its triangles' vertices, merged into the mesh's.
// Every CTA also zeroes its share of [zeroBegin, zeroBegin + zeroWords).
__global__ void __launch_bounds__(kTileThreads)
    k_batch_bounds(const float* __restrict__ tris, uint32_t n, const uint32_t* __restrict__ off, uint32_t nMeshes,
                   const uint32_t* __restrict__ tileStart, uint32_t* __restrict__ bounds,
                   uint32_t* __restrict__ zeroBegin, size_t zeroWords)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < zeroWords; i += (size_t)gridDim.x * blockDim.x)
        zeroBegin[i] = 0u;
    TileWork w;
    if (!tile_work(off, tileStart, nMeshes, blockIdx.x, w)) return;
    __shared__ __align__(16) float s_tri[kStageTris * 9];
    __shared__ float s_box[kTileThreads / 32][6];
    float lo[3] = {kFltMax, kFltMax, kFltMax}, hi[3] = {-kFltMax, -kFltMax, -kFltMax};
    for (uint32_t b = 0; b < w.count; b += kStageTris) {
        const int cnt = (int)min((uint32_t)kStageTris, w.count - b);
        __syncthreads();
        stage_floats(s_tri, tris, 9 * ((size_t)w.start + w.first + b), 9 * cnt, 9 * (size_t)n);
        __syncthreads();
        if ((int)threadIdx.x < cnt) {
            const float* t = s_tri + 9 * threadIdx.x;
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    lo[a] = fminf(lo[a], t[3 * v + a]);
                    hi[a] = fmaxf(hi[a], t[3 * v + a]);
                }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            s_box[warp][a] = lo[a];
            s_box[warp][3 + a] = hi[a];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        float v = s_box[0][threadIdx.x];
        for (int k = 1; k < kTileThreads / 32; ++k)
            v = threadIdx.x < 3 ? fminf(v, s_box[k][threadIdx.x]) : fmaxf(v, s_box[k][threadIdx.x]);
        uint32_t* dst = bounds + 6 * (size_t)w.mesh + threadIdx.x;
        if (threadIdx.x < 3)
            atomicMin(dst, ordered(v));
        else
            atomicMax(dst, ordered(v));
    }
}

// Per tile: Morton keys over the mesh's bounds (buildMortons,
// minimum_lbvh.cu:68-92, as k_keys of the single-mesh build), the mesh's
// digit histograms for every pass, and the reset of the tile's hand-off
// words. The first tile of a mesh also writes the mesh's AABB.
template <int kBits>
__global__ void __launch_bounds__(kTileThreads)
    k_batch_keys(const float* __restrict__ tris, uint32_t n, uint32_t option, const uint32_t* __restrict__ off,
                 uint32_t nMeshes, const uint32_t* __restrict__ tileStart, const uint32_t* __restrict__ bounds,
                 uint32_t* __restrict__ keys, uint32_t* __restrict__ histogram, uint32_t* __restrict__ handoff,
                 mlbvh_aabb* __restrict__ meshAABBs)
{
    using S = sort::Shape<kBits>;
    constexpr int kBins = S::kBins, kPasses = S::kPasses;
    constexpr uint32_t kMask = (uint32_t)kBins - 1u;
    __shared__ uint32_t s_hist[kPasses * kBins];
    __shared__ __align__(16) float s_tri[kStageTris * 9];
    TileWork w;
    if (!tile_work(off, tileStart, nMeshes, blockIdx.x, w)) return;
    for (int i = threadIdx.x; i < kPasses * kBins; i += kTileThreads) s_hist[i] = 0u;
    const uint32_t* mb = bounds + 6 * (size_t)w.mesh;
    if (w.first == 0 && meshAABBs && threadIdx.x < 6)
        reinterpret_cast<float*>(meshAABBs + w.mesh)[threadIdx.x] = unordered(__ldcg(mb + threadIdx.x));
    const f3 lower = mk(unordered(__ldcg(mb)), unordered(__ldcg(mb + 1)), unordered(__ldcg(mb + 2)));
    const f3 upper = mk(unordered(__ldcg(mb + 3)), unordered(__ldcg(mb + 4)), unordered(__ldcg(mb + 5)));
    // hand-off words of the mesh's internal nodes [first, first + count) ∩ [0, len - 1)
    uint32_t* ho = handoff + (w.start - w.mesh);
    for (uint32_t j = w.first + threadIdx.x; j < w.first + w.count && j + 1 < w.len; j += kTileThreads)
        ho[j] = 0xFFFFFFFFu;

    for (uint32_t b = 0; b < w.count; b += kStageTris) {
        const int cnt = (int)min((uint32_t)kStageTris, w.count - b);
        __syncthreads();
        stage_floats(s_tri, tris, 9 * ((size_t)w.start + w.first + b), 9 * cnt, 9 * (size_t)n);
        __syncthreads();
        if ((int)threadIdx.x < cnt) {
            const float* t = s_tri + 9 * threadIdx.x;
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
            keys[w.start + w.first + b + threadIdx.x] = key;
#pragma unroll
            for (int p = 0; p < kPasses; ++p) atomicAdd(&s_hist[p * kBins + ((key >> (kBits * p)) & kMask)], 1u);
        }
    }
    __syncthreads();
    uint32_t* h = histogram + (size_t)w.mesh * kPasses * kBins;
    for (int i = threadIdx.x; i < kPasses * kBins; i += kTileThreads) {
        const uint32_t c = s_hist[i];
        if (c) atomicAdd(h + i, c);
    }
}


// build_lbvh (minimum_lbvh.h:284-361), one thread per sorted leaf: the tile
// climb of the single-mesh build, over tiles of kTileLeaves consecutive leaves
// of the whole batch. A tile may hold the end of one mesh and the start of the
// next: the delta across a mesh boundary is staged as infinite (the value each
// mesh's climb gives the deltas outside its range), so each node's range, and
// with it its interior test, stays inside its mesh.
static_assert(kBuildThreads == (int)kTileLeaves, "one thread per leaf of a tile");
__global__ void __launch_bounds__(kBuildThreads)
    k_batch_build(const float* __restrict__ tris, uint32_t n, const uint32_t* __restrict__ off, uint32_t nMeshes,
                  const uint32_t* __restrict__ sortedKeys, const uint32_t* __restrict__ sortedIdx,
                  mlbvh_internal_node* __restrict__ allNodes, uint32_t* __restrict__ allHandoff,
                  mlbvh_node_index* __restrict__ roots, const uint32_t* __restrict__ header)
{
    __shared__ TileClimbShared sh;
    if (__ldcg(header + kHdrError) & kErrOffsets) return;  // the whole CTA: the plan's word is set before
    const uint32_t t0 = blockIdx.x * kTileLeaves;
    const uint32_t g = t0 + threadIdx.x;
    uint32_t m = 0, start = n, end = n, tri = 0xFFFFFFFFu;
    f3 lo = mk(0.0f, 0.0f, 0.0f), hi = lo;
    if (g < n) {
        m = find_segment(off, nMeshes, g);
        start = __ldg(off + m);
        end = __ldg(off + m + 1);
        tri = sortedIdx[g];
        // tri >= the mesh's size only after a sort whose bounded wait gave up (error word set)
        if (tri < end - start) leaf_box(tris + 9 * (size_t)start, end - start, tri, lo, hi);
    }
    tile_climb_prepare(sh, sortedKeys, n, t0, start, end);
    if (g >= n || tri >= end - start) return;
    climb_tile(sh, t0 - start, end - start, g - start, tri, lo, hi, sortedKeys + start, allNodes + (start - m),
               allHandoff + (start - m), roots + m, nullptr);
}

// The persistent traversal (see the file comment). Hits are written as
// mlbvh_trace writes them; ray i of the batch belongs to the mesh m with
// rayOff[m] <= i < rayOff[m+1].
constexpr int kBatchReplayDepth = 16;  // stack entries per lane of the replay walk

template <bool kAny, bool kReplay>
__global__ void __launch_bounds__(512)
    k_batch_trace(const mlbvh_internal_node* __restrict__ nodes, const mlbvh_node_index* __restrict__ roots,
                  const float* __restrict__ tris, const uint32_t* __restrict__ triOff,
                  const float4* __restrict__ rays, const uint32_t* __restrict__ rayOff, uint32_t nMeshes,
                  uint32_t nRays, float4* __restrict__ hits, uint32_t* __restrict__ queue,
                  const uint32_t* __restrict__ header, uint32_t chunk, uint32_t refill)
{
    if (__ldcg(header + kHdrError)) return;  // the build failed: its trees must not be walked
    // replay walk: kBatchReplayDepth stack entries per lane in dynamic shared memory, one column per thread
    extern __shared__ __align__(16) unsigned char s_replay[];
    using Entry = typename ReplayStack<kAny>::Entry;
    Entry* const stack = reinterpret_cast<Entry*>(s_replay) + threadIdx.x;
    int depth = 0;
    const int lane = threadIdx.x & 31;
    const uint32_t lanesBelow = (1u << lane) - 1u;
    uint32_t poolNext = 0, poolEnd = 0, poolMesh = 0;  // warp-uniform: rays taken, not yet handed out
    bool exhausted = false;                            // warp-uniform: the queue is empty
    bool live = false;
    uint32_t ray = 0, curr = 0, prev = 0, steps = 0, nv = 0, nt = 0, leaves = 1;
    const mlbvh_internal_node* mn = nodes;
    const float* mt = tris;
    f3 ro = mk(0, 0, 0), rd = ro, inv = ro;
    float tmin = 0.0f;
    HitRecord hit;
    hit.t = 0.0f;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !live);
        if (idle) {
            if (poolNext >= poolEnd && !exhausted && ((uint32_t)__popc(idle) >= refill || idle == 0xffffffffu)) {
                uint32_t base = 0, m = 0;
                if (lane == 0) {
                    base = atomicAdd(queue, chunk);
                    if (base < nRays) m = find_segment(rayOff, nMeshes, base);
                }
                base = __shfl_sync(0xffffffffu, base, 0);
                m = __shfl_sync(0xffffffffu, m, 0);
                if (base >= nRays) {
                    exhausted = true;
                } else {
                    poolNext = base;
                    poolEnd = min(base + chunk, nRays);
                    poolMesh = m;
                }
            }
            if (poolNext < poolEnd) {
                const uint32_t avail = poolEnd - poolNext;
                const uint32_t rank = __popc(idle & lanesBelow);
                if (!live && rank < avail) {
                    ray = poolNext + rank;
                    uint32_t m = poolMesh;
                    while (m + 1 < nMeshes && __ldg(rayOff + m + 1) <= ray) ++m;
                    const uint32_t start = __ldg(triOff + m);
                    leaves = __ldg(triOff + m + 1) - start;
                    mn = nodes + (start - m);
                    mt = tris + 9 * (size_t)start;
                    const float4 a = __ldg(rays + 2 * (size_t)ray), b = __ldg(rays + 2 * (size_t)ray + 1);
                    ro = mk(a.x, a.y, a.z);
                    rd = mk(b.x, b.y, b.z);
                    tmin = a.w;
                    inv = inv_rd(rd);
                    hit.t = b.w;
                    hit.u = 0.0f;
                    hit.v = 0.0f;
                    hit.ng = mk(0.0f, 0.0f, 0.0f);
                    hit.tri = 0xFFFFFFFFu;
                    curr = __ldg(roots + m);
                    prev = kInvalid;
                    depth = 0;
                    steps = 0;
                    live = true;
                }
                poolNext += min((uint32_t)__popc(idle), avail);
            }
        }
        if (!__any_sync(0xffffffffu, live)) {
            if (exhausted) break;
            continue;
        }
        if (live) {
            // an index outside the mesh's tree (possible only in a corrupt tree) ends the walk
            const bool inTree = (curr & kLeafBit) ? (curr & ~kLeafBit) < leaves : curr + 1 < leaves;
            bool done = !inTree;
            if (!done) {
                if constexpr (kReplay)
                    done = stackfree_replay_step<kAny, false, kBatchReplayDepth>(curr, prev, depth, stack, blockDim.x,
                                                                                  hit, mn, mt, ro, rd, inv, tmin, nv,
                                                                                  nt);
                else
                    done = stackfree_step<kAny, false, true>(curr, prev, hit, mn, mt, ro, rd, inv, tmin, nv, nt);
            }
            if (done || ++steps >= kMaxTraversalSteps) {
                hits[2 * (size_t)ray] = make_float4(hit.t, 0.0f, hit.u, hit.v);
                hits[2 * (size_t)ray + 1] = make_float4(hit.ng.x, hit.ng.y, hit.ng.z, __uint_as_float(hit.tri));
                live = false;
            }
        }
    }
}

// The replay traversal's dynamic shared memory can exceed 48 KB (512 threads,
// closest hit: 64 KB); allow it once per device.
void prepare_trace()
{
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev]) return;
    const int smem = kBatchReplayDepth * 512 * 8;
    cudaFuncSetAttribute(k_batch_trace<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_batch_trace<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int kBits>
void prepare_sort()
{
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev]) return;
    constexpr int smem = (int)sort::Shape<kBits>::kSmemBytes;
    cudaFuncSetAttribute(sort::k_onesweep<kBits, true, sort::MeshSegments>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(sort::k_onesweep<kBits, false, sort::MeshSegments>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int kBits>
mlbvh_status launch_build(const mlbvh_batch& B, const BatchLayout& L, cudaStream_t stream, uint32_t spinLimit)
{
    using S = sort::Shape<kBits>;
    constexpr int kBins = S::kBins, kPasses = S::kPasses;
    prepare_sort<kBits>();
    char* s = static_cast<char*>(B.dScratch);
    uint32_t* header = reinterpret_cast<uint32_t*>(s + L.header);
    uint32_t* tileStart = reinterpret_cast<uint32_t*>(s + L.tileStart);
    uint32_t* bounds = reinterpret_cast<uint32_t*>(s + L.bounds);
    uint32_t* hist = reinterpret_cast<uint32_t*>(s + L.histogram);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(s + L.lookback);
    uint32_t* keysA = reinterpret_cast<uint32_t*>(s + L.keysA);
    uint32_t* keysB = reinterpret_cast<uint32_t*>(s + L.keysB);
    uint32_t* valsA = reinterpret_cast<uint32_t*>(s + L.valsA);
    uint32_t* valsB = reinterpret_cast<uint32_t*>(s + L.valsB);
    uint32_t* handoff = reinterpret_cast<uint32_t*>(s + L.handoff);
    const float* tris = reinterpret_cast<const float*>(B.dTriangles);
    const uint32_t* off = B.dMeshTriangleOffsets;
    const uint32_t nm = B.nMeshes, n = B.nTriangles;

    k_batch_plan<<<1, kPlanThreads, 0, stream>>>(off, nm, n, header, tileStart, bounds);
    MLBVH_CHECK_LAUNCH("k_batch_plan");
    const size_t zeroWords = (L.zeroEnd - L.histogram) / 4;
    k_batch_bounds<<<L.maxTiles, kTileThreads, 0, stream>>>(tris, n, off, nm, tileStart, bounds, hist, zeroWords);
    MLBVH_CHECK_LAUNCH("k_batch_bounds");
    k_batch_keys<kBits><<<L.maxTiles, kTileThreads, 0, stream>>>(tris, n, B.buildOption, off, nm, tileStart, bounds,
                                                                 keysA, hist, handoff, B.dMeshAABBs);
    MLBVH_CHECK_LAUNCH("k_batch_keys");
    uint32_t* kin = keysA;
    uint32_t* vin = valsA;
    for (int pass = 0; pass < kPasses; ++pass) {
        uint32_t* kout = (pass % 2 == 0) ? keysB : keysA;
        uint32_t* vout = (pass % 2 == 0) ? valsB : valsA;
        const sort::MeshSegments segs{off, tileStart, nm, hist + (size_t)pass * kBins, (uint32_t)(kPasses * kBins)};
        uint32_t* lb = lookback + (size_t)pass * L.maxTiles * kBins;
        if (pass == 0)
            sort::k_onesweep<kBits, true><<<L.maxTiles, sort::kThreads, S::kSmemBytes, stream>>>(
                kin, kout, nullptr, vout, kBits * pass, segs, lb, header + kHdrTickets + pass, header, spinLimit);
        else
            sort::k_onesweep<kBits, false><<<L.maxTiles, sort::kThreads, S::kSmemBytes, stream>>>(
                kin, kout, vin, vout, kBits * pass, segs, lb, header + kHdrTickets + pass, header, spinLimit);
        MLBVH_CHECK_LAUNCH("k_onesweep");
        kin = kout;
        vin = vout;
    }
    const ProfileEvents ev = take_profile_events();
    if (ev.start) cudaEventRecord(ev.start, stream);
    k_batch_build<<<(n + kBuildThreads - 1) / kBuildThreads, kBuildThreads, 0, stream>>>(
        tris, n, off, nm, kin, vin, B.dInternals, handoff, B.dRootNodes, header);
    MLBVH_CHECK_LAUNCH("k_batch_build");
    if (ev.stop) cudaEventRecord(ev.stop, stream);
    return MLBVH_OK;
}

mlbvh_status check_params(const mlbvh_batch_params& p)
{
    if (p.digitBits != 8 && p.digitBits != 11) return fail(MLBVH_ERR_INVALID_ARG, "digitBits must be 8 or 11");
    if (p.traceBlock != 64 && p.traceBlock != 128 && p.traceBlock != 256 && p.traceBlock != 512)
        return fail(MLBVH_ERR_INVALID_ARG, "traceBlock must be 64, 128, 256 or 512");
    if (p.queueChunk < 1 || p.queueChunk > 65536) return fail(MLBVH_ERR_INVALID_ARG, "queueChunk must be in [1, 65536]");
    if (p.refillLanes < 1 || p.refillLanes > 32) return fail(MLBVH_ERR_INVALID_ARG, "refillLanes must be in [1, 32]");
    if (p.walk != 0 && p.walk != 1) return fail(MLBVH_ERR_INVALID_ARG, "walk must be 0 (stack-free) or 1 (replay)");
    return MLBVH_OK;
}

mlbvh_status check_geometry(const mlbvh_batch& B)
{
    if (B.nMeshes == 0 || B.nMeshes > kMaxMeshes) return fail(MLBVH_ERR_INVALID_ARG, "nMeshes must be in [1, 2^20]");
    if (B.nTriangles < B.nMeshes || B.nTriangles >= (1u << 30))
        return fail(MLBVH_ERR_INVALID_ARG, "nTriangles must be in [nMeshes, 2^30)");
    if (!B.dTriangles || !B.dMeshTriangleOffsets || !B.dRootNodes || !B.dScratch)
        return fail(MLBVH_ERR_INVALID_ARG, "null triangles, offsets, roots or scratch pointer");
    if (B.nTriangles > B.nMeshes && !B.dInternals) return fail(MLBVH_ERR_INVALID_ARG, "null internal-node pointer");
    if (!aligned16(B.dTriangles) || !aligned16(B.dMeshTriangleOffsets) || !aligned32(B.dInternals) ||
        !aligned16(B.dRootNodes) || !aligned16(B.dMeshAABBs) || !aligned16(B.dScratch))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned (node arrays 32-byte)");
    return MLBVH_OK;
}

}  // namespace

size_t batch_scratch_bytes(uint32_t nMeshes, uint32_t n)
{
    if (nMeshes == 0 || nMeshes > kMaxMeshes || n < nMeshes || n >= (1u << 30)) return 0;
    return std::max(batch_layout(nMeshes, n, 8).total, batch_layout(nMeshes, n, 11).total);
}

void batch_params_default(mlbvh_batch_params* p)
{
    p->digitBits = 8;
    p->traceBlock = 128;
    p->queueChunk = 64;
    p->refillLanes = 8;
    p->walk = 1;
}

mlbvh_status build_batched(const mlbvh_batch& B, const mlbvh_batch_params& P, cudaStream_t stream)
{
    if (mlbvh_status s = check_geometry(B)) return s;
    if (mlbvh_status s = check_params(P)) return s;
    if (B.scratchBytes < batch_scratch_bytes(B.nMeshes, B.nTriangles))
        return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_batch_scratch_bytes");
    const BatchLayout L = batch_layout(B.nMeshes, B.nTriangles, P.digitBits);
    return P.digitBits == 11 ? launch_build<11>(B, L, stream, kDefaultSpinLimit)
                             : launch_build<8>(B, L, stream, kDefaultSpinLimit);
}

mlbvh_status trace_batched(const mlbvh_batch& B, const mlbvh_batch_params& P, cudaStream_t stream)
{
    if (mlbvh_status s = check_geometry(B)) return s;
    if (mlbvh_status s = check_params(P)) return s;
    if (B.nRays == 0) return MLBVH_OK;
    if (B.nRays >= (1u << 31)) return fail(MLBVH_ERR_INVALID_ARG, "nRays must be below 2^31");
    if (!B.dRays || !B.dMeshRayOffsets || !B.dHits) return fail(MLBVH_ERR_INVALID_ARG, "null rays, ray offsets or hits");
    if (!aligned16(B.dRays) || !aligned16(B.dMeshRayOffsets) || !aligned16(B.dHits))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (B.rayQuery != MLBVH_RAY_QUERY_CLOSEST && B.rayQuery != MLBVH_RAY_QUERY_ANY)
        return fail(MLBVH_ERR_INVALID_ARG, "rayQuery must be MLBVH_RAY_QUERY_CLOSEST or MLBVH_RAY_QUERY_ANY");
    if (B.scratchBytes < batch_scratch_bytes(B.nMeshes, B.nTriangles))
        return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_batch_scratch_bytes");
    uint32_t* header = static_cast<uint32_t*>(B.dScratch);
    cudaError_t e = cudaMemsetAsync(header + kHdrQueue, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    const bool any = B.rayQuery == MLBVH_RAY_QUERY_ANY;
    const bool replay = P.walk == 1;
    auto kernel = any ? (replay ? k_batch_trace<true, true> : k_batch_trace<true, false>)
                      : (replay ? k_batch_trace<false, true> : k_batch_trace<false, false>);
    const size_t smem = replay ? (size_t)kBatchReplayDepth * P.traceBlock * (any ? 4 : 8) : 0;
    prepare_trace();
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, P.traceBlock, smem) != cudaSuccess || perSm <= 0)
        perSm = 1;
    const int grid = perSm * device_sm_count();
    kernel<<<grid, P.traceBlock, smem, stream>>>(B.dInternals, B.dRootNodes, reinterpret_cast<const float*>(B.dTriangles),
                                              B.dMeshTriangleOffsets, reinterpret_cast<const float4*>(B.dRays),
                                              B.dMeshRayOffsets, B.nMeshes, B.nRays,
                                              reinterpret_cast<float4*>(B.dHits), header + kHdrQueue, header,
                                              (uint32_t)P.queueChunk, (uint32_t)P.refillLanes);
    MLBVH_CHECK_LAUNCH("k_batch_trace");
    return MLBVH_OK;
}

// ------------------------------------------------------------------ graphs

}  // namespace mlbvh

struct mlbvh_batch_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace mlbvh {

mlbvh_status batch_graph_create(const mlbvh_batch& B, const mlbvh_batch_params& P, int stages,
                                mlbvh_batch_graph** out)
{
    if (!out) return fail(MLBVH_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (stages < 1 || stages > 3) return fail(MLBVH_ERR_INVALID_ARG, "stages must be 1 (build), 2 (trace) or 3 (both)");
    if (mlbvh_status s = check_geometry(B)) return s;
    if (mlbvh_status s = check_params(P)) return s;
    // kernel attributes are set outside the capture
    prepare_trace();
    if (P.digitBits == 11)
        prepare_sort<11>();
    else
        prepare_sort<8>();
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    }
    mlbvh_status st = MLBVH_OK;
    if (stages & 1) st = build_batched(B, P, cs);
    if (st == MLBVH_OK && (stages & 2)) st = trace_batched(B, P, cs);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (st != MLBVH_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    }
    mlbvh_batch_graph* g = new mlbvh_batch_graph;
    g->graph = graph;
    g->exec = exec;
    *out = g;
    return MLBVH_OK;
}

mlbvh_status batch_graph_launch(mlbvh_batch_graph* g, cudaStream_t stream)
{
    if (!g) return fail(MLBVH_ERR_INVALID_ARG, "null graph");
    const cudaError_t e = cudaGraphLaunch(g->exec, stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    return MLBVH_OK;
}

void batch_graph_destroy(mlbvh_batch_graph* g)
{
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

// --------------------------------------------------------------- autotuner

namespace {

// Median device time of `reps` runs of fn on `stream`, after one warm-up run.
template <class Fn>
mlbvh_status time_median(Fn fn, cudaStream_t stream, int reps, float* ms)
{
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        if (a) cudaEventDestroy(a);
        return fail(MLBVH_ERR_CUDA, "cudaEventCreate failed");
    }
    std::vector<float> t;
    mlbvh_status st = fn();
    for (int r = 0; st == MLBVH_OK && r < reps; ++r) {
        cudaEventRecord(a, stream);
        st = fn();
        cudaEventRecord(b, stream);
        if (st != MLBVH_OK) break;
        const cudaError_t e = cudaEventSynchronize(b);
        if (e != cudaSuccess) {
            st = fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
            break;
        }
        float x = 0.0f;
        cudaEventElapsedTime(&x, a, b);
        t.push_back(x);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != MLBVH_OK) return st;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return MLBVH_OK;
}

}  // namespace

mlbvh_status batch_autotune(const mlbvh_batch& B, mlbvh_batch_params* out, float* bestBuildMs, float* bestTraceMs,
                            cudaStream_t stream)
{
    if (!out) return fail(MLBVH_ERR_INVALID_ARG, "null output pointer");
    mlbvh_batch_params best;
    batch_params_default(&best);
    if (mlbvh_status s = check_geometry(B)) return s;
    const int reps = 3;
    // digit width of the build's sort
    float bestB = 1e30f;
    for (int bits : {8, 11}) {
        mlbvh_batch_params p = best;
        p.digitBits = bits;
        float ms = 0.0f;
        if (mlbvh_status s = time_median([&] { return build_batched(B, p, stream); }, stream, reps, &ms)) return s;
        if (ms < bestB) {
            bestB = ms;
            best.digitBits = bits;
        }
    }
    // the build's output must stand for the traversal candidates: rebuild with the winner
    if (mlbvh_status s = build_batched(B, best, stream)) return s;
    float bestT = 0.0f;
    if (B.nRays > 0) {
        // coordinate descent: block size, then queue chunk, then refill threshold
        auto try_trace = [&](mlbvh_batch_params p, float* ms) {
            return time_median([&] { return trace_batched(B, p, stream); }, stream, 1, ms);
        };
        if (mlbvh_status s = try_trace(best, &bestT)) return s;
        const int walks[] = {0, 1}, blocks[] = {64, 128, 256, 512}, chunks[] = {32, 64, 128, 256, 512},
                  refills[] = {1, 4, 8, 16};
        for (int axis = 0; axis < 4; ++axis) {
            const int* vals = axis == 0 ? walks : axis == 1 ? blocks : axis == 2 ? chunks : refills;
            const int count = axis == 0 ? 2 : axis == 1 ? 4 : axis == 2 ? 5 : 4;
            for (int k = 0; k < count; ++k) {
                mlbvh_batch_params p = best;
                int& field = axis == 0 ? p.walk : axis == 1 ? p.traceBlock : axis == 2 ? p.queueChunk : p.refillLanes;
                if (field == vals[k]) continue;
                field = vals[k];
                float ms = 0.0f;
                if (mlbvh_status s = try_trace(p, &ms)) return s;
                if (ms < bestT) {
                    bestT = ms;
                    best = p;
                }
            }
        }
    }
    *out = best;
    if (bestBuildMs) *bestBuildMs = bestB;
    if (bestTraceMs) *bestTraceMs = bestT;
    return MLBVH_OK;
}

}  // namespace mlbvh
