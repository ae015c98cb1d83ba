// Higher-quality build on B200: parallel locally-ordered clustering (PLOC;
// Meister and Bittner, "Parallel Locally-Ordered Clustering for Bounding
// Volume Hierarchy Construction", 2018) over the Morton order of the LBVH
// build, written into the same InternalNode array as build.cu.
//
// The reference's higher-quality build is Embree's SAH builder behind
// BVHCPUBuilder::buildByEmbree (minimum_lbvh.h:594-656): binary nodes, one
// triangle per leaf, boxes of both children in each node, root parent
// invalid. Here the nodes are numbered in in-order (node j lies between the
// j-th and (j+1)-th leaf of a left-to-right walk), as build_lbvh's are, so
// a left leaf child of node j is leaf j, a right one leaf j + 1, and context
// (the escape index intersect_escape_link reads) is the in-order index of
// the subtree's last leaf when below n - 1, else ~0, exactly build_lbvh's
// convention: every walk, the leaf-ordered triangles, the 4-wide regrouping
// and the quantisers take this tree unchanged.
//
// Clustering rule (the oracle states the same): a cluster's nearest
// neighbour among the r clusters on either side minimises the half area of
// the union box (area_key: union by fminf / fmaxf, dx*dy + dy*dz + dz*dx, a
// NaN area counted as +inf), ties to the smaller position: a strict order on pairs,
// so the closest pair overall is mutual and every iteration merges. Once an
// iteration has removed fewer than 1/64 of the clusters, later iterations
// break exact ties first by the smaller pair_hash of the two positions (still
// a strict order), so runs of equal union areas (duplicated or collinear
// triangles) pair up about a quarter at a time instead of one pair per run;
// and if such an iteration still removes fewer than 1/64 (a chain of growing
// gaps, each cluster nearest to the one before it), the next iteration pairs
// positions 2k and 2k + 1 outright, so every build ends in O(log n)
// iterations. Mutual nearest neighbours merge into the lower position;
// survivors keep order.
//
// Launch chain on one stream (no host synchronisation):
//   k_scene_bounds, k_keys, k_onesweep x4   build.cu's chain (sorted leaves)
//   k_ploc_init   cluster i = sorted leaf i (box, id, one leaf); zeroes the
//                 look-back words and the control block
//   k_ploc        one cooperative launch (every CTA resident), three phases:
//     grid phase, while more than kTailClusters clusters remain: tiles of
//       kTile - 2r clusters; a tile stages its clusters and 2r on each side
//       in shared memory, finds the nearest neighbours of its clusters and of
//       r on each side (kTile positions, four consecutive per thread, radius
//       unrolled at compile time for 4, 8, 16 and 32), keeps or merges, and
//       finds where its survivors and new nodes go by decoupled look-back
//       (the whole CTA reading 256 earlier tiles per step) over the earlier
//       tiles of the iteration; a grid barrier ends the iteration;
//     tail: CTA 0 finishes the last clusters in shared memory;
//     placement, top-down from the root without barriers: each node's
//       in-order index is its first leaf's in-order index (handed down by its
//       parent) plus its left child's leaf count minus one; warps take the
//       nodes in descending creation order (parents before children) and a
//       lane places its node once its parent has handed the first leaf down.
//
// Every wait is bounded: a look-back or barrier wait that gives up sets the
// build's error word (reported by mlbvh_scratch_status), skips its writes,
// and the kernel returns at the next barrier. Data written by another CTA in
// the same launch is read through L2 (ld.global.cg / .relaxed.gpu), never L1.
#include <algorithm>

#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"
#include "climb.cuh"
#include "onesweep.cuh"

namespace mlbvh {

namespace {

constexpr int kPlocThreads = sort::kThreads;  // 256 (block_scan's width)
constexpr int kPer = 4;                       // clusters per thread in a tile
constexpr uint32_t kTile = kPlocThreads * kPer;
constexpr uint32_t kTailClusters = kTile;
constexpr int kMaxRadius = 32;
constexpr uint32_t kSpan = kTile + 2 * kMaxRadius;  // staged clusters per tile (kTile - 2r + 4r)
// Shared-memory slot of staged cluster k: one pad slot after every four, so
// that lanes reading clusters four apart (each thread owns four consecutive
// positions) hit distinct banks.
__host__ __device__ constexpr uint32_t pad(uint32_t k) { return k + (k >> 2); }
constexpr uint32_t kSpanP = pad(kSpan);
constexpr size_t kPlocSmem = (size_t)kSpanP * (2 * sizeof(float4) + sizeof(uint32_t));
constexpr int kInitThreads = 256;
constexpr uint32_t kPlaceChunk = 128;  // placement positions a warp takes at a time
constexpr uint32_t kUnset = 0xFFFFFFFFu;
constexpr int kMaxCtasPerSm = 4;

constexpr unsigned long long kFlagAggregate = 1ull << 62;
constexpr unsigned long long kFlagInclusive = 2ull << 62;
constexpr unsigned long long kValueMask = (1ull << 62) - 1;
constexpr int kMergeShift = 31;  // packed counts: survivors bits 0-30, merges bits 31-61
constexpr unsigned long long kCountMask = (1ull << 31) - 1;

// clusters / merged after grid-phase iteration k sit in slot (k + 1) & 1: the
// last tile of iteration k writes them while a CTA without tiles may still be
// reading slot k & 1, and cannot read slot (k + 1) & 1 before the barrier.
struct PlocControl {
    uint32_t barrierCount, barrierGen;
    uint32_t clusters[2], merged[2];
    uint32_t placeNext;  // next position of the placement order to hand out
};

struct PlocArgs {
    float4* clusters[2];  // per cluster {lo.xyz, id} {hi.xyz, leaf count}
    float4* tmp;          // per new node, creation order: {lo0, id0} {hi0, id1} {lo1, cnt0} {hi1, cnt1}
    unsigned long long* info;  // per new node: in-order index of its first leaf | parent's in-order index << 32
                               // (first leaf ~0: not handed down yet)
    unsigned long long* flags;  // 2 x maxTiles look-back words
    PlocControl* ctl;
    uint32_t* error;
    mlbvh_internal_node* out;
    mlbvh_node_index* root;
    uint32_t n, maxTiles, radius, spinLimit;
};

// Scratch after build.cu's layout.
struct PlocLayout {
    size_t control, flags, clustersA, clustersB, tmp, info, total;
    uint32_t maxTiles;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

PlocLayout ploc_layout(uint32_t n)
{
    PlocLayout L;
    L.maxTiles = (n + (kTile - 2 * kMaxRadius) - 1) / (kTile - 2 * kMaxRadius);
    size_t o = align256(build_scratch_bytes(n));
    L.control = o;
    o += 256;
    L.flags = o;
    o = align256(o + sizeof(unsigned long long) * 2 * (size_t)L.maxTiles);
    L.clustersA = o;
    o = align256(o + 32 * (size_t)n);
    L.clustersB = o;
    o = align256(o + 32 * (size_t)n);
    L.tmp = o;
    o = align256(o + 64 * (size_t)n);
    L.info = o;
    o = align256(o + 8 * (size_t)n);
    L.total = o;
    return L;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }

// Half area of the union of boxes a and b as an order key: union by
// fminf / fmaxf (a NaN operand is ignored), area dx*dy + dy*dz + dz*dx, key
// the bits of min(|area|, +inf): a zero area of either sign is 0, a NaN
// area counts as +inf, and the key is symmetric in a and b.
__device__ __forceinline__ uint32_t area_key(f3 alo, f3 ahi, f3 blo, f3 bhi)
{
    const float dx = __fsub_rn(fmaxf(ahi.x, bhi.x), fminf(alo.x, blo.x));
    const float dy = __fsub_rn(fmaxf(ahi.y, bhi.y), fminf(alo.y, blo.y));
    const float dz = __fsub_rn(fmaxf(ahi.z, bhi.z), fminf(alo.z, blo.z));
    const float a = __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
    return __float_as_uint(fminf(fabsf(a), __int_as_float(0x7f800000)));
}

// A symmetric mix of a pair's two positions (integer hashing in the style of
// MurmurHash3's finaliser), the tie-break once ties stall the clustering.
__device__ __forceinline__ uint32_t pair_hash(uint32_t a, uint32_t b)
{
    const uint32_t lo = min(a, b), hi = max(a, b);
    uint32_t h = lo * 0x9E3779B1u ^ hi * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}

// Once ties stall the clustering: among the candidates of position p (window
// [jFirst, jEnd), staged from `base`) whose key equals the minimum bestA, the
// one with the smallest pair_hash, the smaller position on equal hashes. A
// second, plain scan, so that the unrolled search above keeps its registers.
__device__ __noinline__ uint32_t resolve_tie(uint32_t p, uint32_t bestA, uint32_t bestJ, int jFirst, int jEnd,
                                             uint32_t base, const float4* sLo, const float4* sHi)
{
    const f3 plo = xyz(sLo[pad(p - base)]), phi = xyz(sHi[pad(p - base)]);
    uint32_t bestH = pair_hash(p, bestJ);
    for (int j = jFirst; j < jEnd; ++j) {
        if ((uint32_t)j == p || (uint32_t)j == bestJ) continue;
        if (area_key(plo, phi, xyz(sLo[pad(j - base)]), xyz(sHi[pad(j - base)])) != bestA) continue;
        const uint32_t h = pair_hash(p, (uint32_t)j);
        if (h < bestH || (h == bestH && (uint32_t)j < bestJ)) {
            bestH = h;
            bestJ = (uint32_t)j;
        }
    }
    return bestJ;
}

// Nearest neighbours of the kPer consecutive positions p0 .. p0 + kPer - 1
// (those in [first, end) are written to sNN); clusters [base, staged) are in
// sLo/sHi, and staged covers r past end or reaches the last cluster. Each
// staged box of the window is read from shared memory once for all kPer
// positions; positions and window are clamped to the staged clusters (the
// positions cut off that way are not written). Keys are at most +inf's bits,
// so the first candidate always beats the initial 0xFFFFFFFF and ascending j
// keeps the smaller position on ties.
__device__ __forceinline__ void nearest_group(uint32_t p0, uint32_t first, uint32_t end, uint32_t base,
                                              uint32_t staged, int r, const float4* sLo, const float4* sHi,
                                              uint32_t* sNN)
{
    f3 plo[kPer], phi[kPer];
    uint32_t bestA[kPer], bestJ[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = min(p0 + q, staged - 1);
        plo[q] = xyz(sLo[pad(p - base)]);
        phi[q] = xyz(sHi[pad(p - base)]);
        bestA[q] = 0xFFFFFFFFu;
        bestJ[q] = 0xFFFFFFFFu;
    }
    const int jFirst = (int)p0 > r ? (int)p0 - r : 0;
    const int jEnd = (int)p0 + kPer + r < (int)staged ? (int)p0 + kPer + r : (int)staged;
    for (int j = jFirst; j < jEnd; ++j) {
        const f3 jlo = xyz(sLo[pad(j - base)]), jhi = xyz(sHi[pad(j - base)]);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int d = j - (int)(p0 + q);
            if (d == 0 || d < -r || d > r) continue;
            const uint32_t a = area_key(plo[q], phi[q], jlo, jhi);
            if (a < bestA[q]) {
                bestA[q] = a;
                bestJ[q] = (uint32_t)j;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = p0 + q;
        if (p >= first && p < end) sNN[pad(p - base)] = bestJ[q];
    }
}

// nearest_group with the radius fixed at compile time, for groups whose whole
// window [p0 - R, p0 + kPer - 1 + R] is staged: the loops unroll and every
// window test resolves at compile time.
template <int R>
__device__ __forceinline__ void nearest_fixed(uint32_t p0, uint32_t first, uint32_t end, uint32_t base,
                                              const float4* sLo, const float4* sHi, uint32_t* sNN)
{
    f3 plo[kPer], phi[kPer];
    uint32_t bestA[kPer], bestJ[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        plo[q] = xyz(sLo[pad(p0 + q - base)]);
        phi[q] = xyz(sHi[pad(p0 + q - base)]);
        bestA[q] = 0xFFFFFFFFu;
        bestJ[q] = 0u;
    }
    const uint32_t j0 = p0 - R;
#pragma unroll
    for (int k = 0; k < 2 * R + kPer; ++k) {
        const f3 jlo = xyz(sLo[pad(j0 + k - base)]), jhi = xyz(sHi[pad(j0 + k - base)]);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int d = k - R - q;
            if (d == 0 || d < -R || d > R) continue;
            const uint32_t a = area_key(plo[q], phi[q], jlo, jhi);
            if (a < bestA[q]) {
                bestA[q] = a;
                bestJ[q] = j0 + k;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = p0 + q;
        if (p >= first && p < end) sNN[pad(p - base)] = bestJ[q];
    }
}

template <int R>
__device__ __forceinline__ void nearest(uint32_t p0, uint32_t first, uint32_t end, uint32_t base, uint32_t staged,
                                        int r, const float4* sLo, const float4* sHi, uint32_t* sNN)
{
    if (R > 0 && p0 >= base + R && p0 + kPer - 1 + R < staged)
        nearest_fixed<R>(p0, first, end, base, sLo, sHi, sNN);
    else
        nearest_group(p0, first, end, base, staged, r, sLo, sHi, sNN);
}

// A pairing iteration: position 2k's neighbour is 2k + 1 and the other way
// round; an odd last cluster points back and stays (tiles start at even
// positions, so no pair straddles two tiles).
__device__ __forceinline__ void pair_partners(uint32_t p0, uint32_t first, uint32_t end, uint32_t base, uint32_t C,
                                              uint32_t* sNN)
{
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = p0 + q;
        if (p < first || p >= end) continue;
        sNN[pad(p - base)] = (p ^ 1u) < C ? p ^ 1u : (p > 0 ? p - 1 : p);
    }
}

// The tie pass of the kPer positions p0 .. (those in [first, end)) once ties
// stall the clustering: each keeps, among its window's candidates with the
// key of the neighbour found, the one with the smallest pair_hash (the window
// as nearest_group clamps it). Run after the search, so the unrolled search
// keeps its registers; it reads boxes and writes only its own entries.
__device__ __forceinline__ void resolve_ties(uint32_t p0, uint32_t first, uint32_t end, uint32_t base,
                                             uint32_t staged, int r, const float4* sLo, const float4* sHi,
                                             uint32_t* sNN)
{
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = p0 + q;
        if (p < first || p >= end) continue;
        const uint32_t j = sNN[pad(p - base)];
        const uint32_t key = area_key(xyz(sLo[pad(p - base)]), xyz(sHi[pad(p - base)]), xyz(sLo[pad(j - base)]),
                                      xyz(sHi[pad(j - base)]));
        sNN[pad(p - base)] = resolve_tie(p, key, j, (int)p > r ? (int)p - r : 0,
                                         (int)p + r + 1 < (int)staged ? (int)p + r + 1 : (int)staged, base, sLo, sHi);
    }
}

// Keep / merge decisions of the kPer positions p0 .. (those below end).
struct Decision {
    uint32_t keepMask, mergeMask;
};
__device__ __forceinline__ Decision decide(uint32_t p0, uint32_t end, uint32_t base, const uint32_t* sNN)
{
    Decision dc{0u, 0u};
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t p = p0 + q;
        if (p >= end) continue;
        const uint32_t j = sNN[pad(p - base)];
        const bool mutual = sNN[pad(j - base)] == p;
        if (!mutual || p < j) dc.keepMask |= 1u << q;
        if (mutual && p < j) dc.mergeMask |= 1u << q;
    }
    return dc;
}

// Writes the new node m (creation order) that merges clusters p (lower) and
// j and returns the merged cluster in (lo, hi).
__device__ __forceinline__ void merge_pair(float4* __restrict__ tmp, uint32_t m, float4 plo, float4 phi, float4 jlo,
                                           float4 jhi, float4& lo, float4& hi)
{
    float4* t = tmp + 4ull * m;
    t[0] = make_float4(plo.x, plo.y, plo.z, plo.w);                    // lo0, id0
    t[1] = make_float4(phi.x, phi.y, phi.z, jlo.w);                    // hi0, id1
    t[2] = make_float4(jlo.x, jlo.y, jlo.z, phi.w);                    // lo1, cnt0
    t[3] = make_float4(jhi.x, jhi.y, jhi.z, jhi.w);                    // hi1, cnt1
    const f3 l = smin3(xyz(plo), xyz(jlo)), h = smax3(xyz(phi), xyz(jhi));
    lo = make_float4(l.x, l.y, l.z, __uint_as_float(m));
    hi = make_float4(h.x, h.y, h.z, __uint_as_float(__float_as_uint(phi.w) + __float_as_uint(jhi.w)));
}

// Exclusive prefix of tile t's packed counts over tiles 0 .. t-1 of this
// iteration, by the whole CTA (every thread gets it): each step reads the
// 256 tiles below `top` at once and stops at the nearest one that holds an
// inclusive prefix, so a tile that is k tiles into its round of the grid
// takes k / 256 + 1 steps. ok = false when a wait gave up.
struct LookbackShared {
    unsigned long long sum[sort::kWarps];
    int stop[sort::kWarps];
};
__device__ unsigned long long lookback(unsigned long long* flags, uint32_t t, unsigned long long agg, uint32_t* error,
                                       uint32_t spinLimit, bool& ok, LookbackShared& sh)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (t == 0) {
        if (tid == 0) st_relaxed64(&flags[0], kFlagInclusive | agg);
        return 0;
    }
    if (tid == 0) st_relaxed64(&flags[t], kFlagAggregate | agg);
    unsigned long long excl = 0;
    int64_t top = (int64_t)t - 1;
    for (;;) {
        const int64_t k = top - tid;
        unsigned long long v = k >= 0 ? ld_relaxed64(&flags[k]) : kFlagInclusive;
        uint32_t spins = 0;
        while (__syncthreads_or((v >> 62) == 0)) {
            if (++spins > spinLimit) {
                if (tid == 0) atomicOr(error, 1u);
                ok = false;
                if ((v >> 62) == 0) v = kFlagInclusive;
                break;
            }
            __nanosleep(32);
            if ((v >> 62) == 0) v = ld_relaxed64(&flags[k]);
        }
        // the nearest inclusive tile is the lowest thread holding one
        const uint32_t incl = __ballot_sync(0xffffffffu, (v >> 62) == 2);
        if (lane == 0) sh.stop[warp] = incl ? warp * 32 + __ffs(incl) - 1 : kPlocThreads;
        __syncthreads();
        int stop = kPlocThreads;
#pragma unroll
        for (int w = 0; w < sort::kWarps; ++w) stop = min(stop, sh.stop[w]);
        unsigned long long mine = tid <= stop ? (v & kValueMask) : 0ull;
#pragma unroll
        for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if (lane == 0) sh.sum[warp] = mine;
        __syncthreads();
#pragma unroll
        for (int w = 0; w < sort::kWarps; ++w) excl += sh.sum[w];
        __syncthreads();  // sh is reused by the next step
        if (stop < kPlocThreads) break;
        top -= kPlocThreads;
    }
    if (tid == 0) st_relaxed64(&flags[t], kFlagInclusive | (excl + agg));
    return excl;
}

// Grid-wide barrier over the cooperative launch. Returns false (in every
// thread of the CTA) when its wait gave up or the error word is set.
__device__ bool grid_barrier(PlocControl* ctl, uint32_t* error, uint32_t spinLimit, int* sFlag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gen = ld_acquire(&ctl->barrierGen);
        __threadfence();
        bool ok = true;
        if (atomicAdd(&ctl->barrierCount, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->barrierCount, 0u);
            __threadfence();
            st_release(&ctl->barrierGen, gen + 1);
        } else {
            uint32_t spins = 0;
            while (ld_acquire(&ctl->barrierGen) == gen) {
                if (++spins > spinLimit) {
                    atomicOr(error, 1u);
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        *sFlag = ok && ld_acquire(error) == 0;
    }
    __syncthreads();
    return *sFlag != 0;
}

// What a node's placement reads that does not depend on its parent: its
// creation record and the left-leaf counts of its internal children. Loaded
// before the lane waits for the parent's hand-down.
struct NodeRecord {
    float4 t0, t1, t2, t3;  // {lo0, id0} {hi0, id1} {lo1, cnt0} {hi1, cnt1}
    uint32_t left0, left1;  // left-leaf counts of internal children 0 / 1
};
__device__ __forceinline__ NodeRecord load_record(const PlocArgs& a, uint32_t m)
{
    NodeRecord r;
    const float4* t = a.tmp + 4ull * m;
    r.t0 = __ldcg(t);
    r.t1 = __ldcg(t + 1);
    r.t2 = __ldcg(t + 2);
    r.t3 = __ldcg(t + 3);
    const uint32_t id0 = __float_as_uint(r.t0.w), id1 = __float_as_uint(r.t1.w), nInternal = a.n - 1;
    r.left0 = (!(id0 & kLeafBit) && id0 < nInternal) ? __float_as_uint(__ldcg(&a.tmp[4ull * id0 + 2].w)) : 0u;
    r.left1 = (!(id1 & kLeafBit) && id1 < nInternal) ? __float_as_uint(__ldcg(&a.tmp[4ull * id1 + 2].w)) : 0u;
    return r;
}

// Places node `rec` given its hand-down word `in` (first leaf's in-order
// index | parent's in-order index << 32): the 64-byte InternalNode at its
// in-order index, and the hand-down words of its internal children (one
// 8-byte store each, read whole by the child's lane).
__device__ __forceinline__ void place_node(const PlocArgs& a, const NodeRecord& rec, unsigned long long in)
{
    const uint32_t first = (uint32_t)in, parent = (uint32_t)(in >> 32);
    const uint32_t id0 = __float_as_uint(rec.t0.w), id1 = __float_as_uint(rec.t1.w);
    const uint32_t cnt0 = __float_as_uint(rec.t2.w), cnt1 = __float_as_uint(rec.t3.w);
    const uint32_t nInternal = a.n - 1;
    const uint32_t rank = first + cnt0 - 1;
    const uint32_t last = first + cnt0 + cnt1 - 1;
    if (rank >= nInternal) return;  // only after a wait gave up (error word set)
    uint32_t c0 = id0, c1 = id1;
    if (!(id0 & kLeafBit) && id0 < nInternal) {
        c0 = first + rec.left0 - 1;
        st_relaxed64(a.info + id0, (unsigned long long)first | (unsigned long long)rank << 32);
    }
    if (!(id1 & kLeafBit) && id1 < nInternal) {
        const uint32_t off1 = first + cnt0;
        c1 = off1 + rec.left1 - 1;
        st_relaxed64(a.info + id1, (unsigned long long)off1 | (unsigned long long)rank << 32);
    }
    float4* o = reinterpret_cast<float4*>(a.out + rank);
    o[0] = make_float4(__uint_as_float(c0), __uint_as_float(c1), rec.t0.x, rec.t0.y);
    o[1] = make_float4(rec.t0.z, rec.t1.x, rec.t1.y, rec.t1.z);
    o[2] = make_float4(rec.t2.x, rec.t2.y, rec.t2.z, rec.t3.x);
    o[3] = make_float4(rec.t3.y, rec.t3.z, __uint_as_float(parent), __uint_as_float(last < nInternal ? last : 0xFFFFFFFFu));
    if (parent == kInvalid) *a.root = rank;
}

// Placement of all n - 1 nodes, in descending creation order (a parent is
// always created after its children): a warp takes kPlaceChunk positions at a
// time, 32 per step; each lane loads its node's record, then places the node
// once the node's hand-down word is set, and lanes of one step that wait on
// each other resolve over the step's rounds. The lowest unplaced position
// always has its parent placed and every CTA is resident, so each wait ends;
// it is still bounded.
__device__ void place_all(const PlocArgs& a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t total = a.n - 1;
    for (;;) {
        uint32_t c0 = 0;
        if (lane == 0) c0 = atomicAdd(&a.ctl->placeNext, kPlaceChunk);
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        if (c0 >= total) return;
        for (uint32_t step = 0; step < kPlaceChunk; step += 32) {
            const uint32_t pos = c0 + step + lane;
            bool done = pos >= total;
            const uint32_t m = done ? 0u : total - 1 - pos;
            NodeRecord rec;
            if (!done) rec = load_record(a, m);
            uint32_t spins = 0;
            while (!__all_sync(0xffffffffu, done)) {
                if (!done) {
                    const unsigned long long in = ld_relaxed64(a.info + m);
                    if ((uint32_t)in != kUnset) {
                        place_node(a, rec, in);
                        done = true;
                    }
                }
                __syncwarp();
                if (!__all_sync(0xffffffffu, done)) {
                    if (++spins > a.spinLimit) {
                        if (lane == 0) atomicOr(a.error, 1u);
                        return;
                    }
                    __nanosleep(32);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kInitThreads)
    k_ploc_init(const float* __restrict__ tris, const uint32_t* __restrict__ sortedIdx, uint32_t n,
                float4* __restrict__ clusters, unsigned long long* __restrict__ flags, uint32_t nFlags,
                PlocControl* __restrict__ ctl, unsigned long long* __restrict__ info)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = g; i < nFlags; i += stride) flags[i] = 0ull;
    for (uint32_t i = g; i + 1 < n; i += stride) info[i] = ~0ull;
    if (g == 0) {
        ctl->barrierCount = 0;
        ctl->barrierGen = 0;
        ctl->clusters[0] = ctl->clusters[1] = n;
        ctl->merged[0] = ctl->merged[1] = 0;
        ctl->placeNext = 0;
    }
    for (uint32_t i = g; i < n; i += stride) {
        uint32_t tri = sortedIdx[i];
        if (tri >= n) tri = 0;  // only after a sort whose bounded wait gave up (error word set)
        f3 lo, hi;
        leaf_box(tris, n, tri, lo, hi);
        clusters[2ull * i] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(kLeafBit | tri));
        clusters[2ull * i + 1] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(1u));
    }
}

// R: the radius when it is one of the compiled-in values (its groups take the
// unrolled search), 0 for any radius (the generic search everywhere).
template <int R>
__global__ void __launch_bounds__(kPlocThreads, 3) k_ploc(PlocArgs a)
{
    extern __shared__ float4 smem[];
    float4* sLo = smem;
    float4* sHi = smem + kSpanP;
    uint32_t* sNN = reinterpret_cast<uint32_t*>(smem + 2 * kSpanP);
    __shared__ uint32_t sWarp[sort::kWarps];
    __shared__ LookbackShared sLook;
    __shared__ int sFlag;
    const int tid = threadIdx.x;
    const int r = R > 0 ? R : (int)a.radius;
    const uint32_t tileClusters = kTile - 2u * r;  // the search range of a tile is kTile positions

    uint32_t C = a.n, merged = 0, iter = 0;
    int cur = 0;
    bool hashTies = false, pairNext = false;  // the same in every CTA: they follow the cluster counts
    // ------------------------------------------------------------ grid phase
    while (C > kTailClusters) {
        const bool pairs = pairNext;
        const uint32_t tiles = (C + tileClusters - 1) / tileClusters;
        unsigned long long* flags = a.flags + (size_t)(iter & 1) * a.maxTiles;
        unsigned long long* nextFlags = a.flags + (size_t)((iter + 1) & 1) * a.maxTiles;
        const float4* src = cur ? a.clusters[1] : a.clusters[0];
        float4* dst = cur ? a.clusters[0] : a.clusters[1];
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
            const uint32_t s = t * tileClusters, e = min(s + tileClusters, C);
            const uint32_t base = s > 2u * r ? s - 2u * r : 0u;
            const uint32_t stagedEnd = min(C, e + 2u * r);
            __syncthreads();  // the previous tile's shared-memory reads are done
            for (uint32_t k = tid; k < stagedEnd - base; k += kPlocThreads) {
                sLo[pad(k)] = __ldcg(src + 2ull * (base + k));
                sHi[pad(k)] = __ldcg(src + 2ull * (base + k) + 1);
            }
            __syncthreads();
            const uint32_t nnFirst = s > (uint32_t)r ? s - r : 0u, nnEnd = min(C, e + r);
            {
                const uint32_t g0 = nnFirst + kPer * tid;  // nnEnd - nnFirst <= kTile: one group per thread
                if (g0 < nnEnd) {
                    if (pairs)
                        pair_partners(g0, nnFirst, nnEnd, base, C, sNN);
                    else
                        nearest<R>(g0, nnFirst, nnEnd, base, stagedEnd, r, sLo, sHi, sNN);
                }
            }
            __syncthreads();
            if (hashTies && !pairs) {  // uniform over the grid
                const uint32_t g0 = nnFirst + kPer * tid;
                if (g0 < nnEnd) resolve_ties(g0, nnFirst, nnEnd, base, stagedEnd, r, sLo, sHi, sNN);
                __syncthreads();
            }
            const uint32_t p0 = s + kPer * tid;
            const Decision dc = decide(p0, e, base, sNN);
            uint32_t total;
            const uint32_t before = sort::block_scan(__popc(dc.keepMask) | __popc(dc.mergeMask) << 16, sWarp, &total);
            const unsigned long long agg =
                (unsigned long long)(total & 0xFFFFu) | (unsigned long long)(total >> 16) << kMergeShift;
            bool ok = true;
            const unsigned long long pre = lookback(flags, t, agg, a.error, a.spinLimit, ok, sLook);
            if (tid == 0) {
                nextFlags[t] = 0ull;
                if (t == tiles - 1) {
                    const uint32_t survivors = (uint32_t)(pre & kCountMask) + (total & 0xFFFFu);
                    const uint32_t mergedAfter = merged + (uint32_t)((pre >> kMergeShift) & kCountMask) + (total >> 16);
                    a.ctl->clusters[(iter + 1) & 1] = survivors;
                    a.ctl->merged[(iter + 1) & 1] = mergedAfter;
                }
            }
            if (!ok) continue;  // uniform: every thread took the same waits
            uint32_t outPos = (uint32_t)(pre & kCountMask) + (before & 0xFFFFu);
            uint32_t node = merged + (uint32_t)((pre >> kMergeShift) & kCountMask) + (before >> 16);
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (!((dc.keepMask >> q) & 1u)) continue;
                const uint32_t p = p0 + q;
                float4 lo = sLo[pad(p - base)], hi = sHi[pad(p - base)];
                if ((dc.mergeMask >> q) & 1u) {
                    const uint32_t j = sNN[pad(p - base)];
                    if (node < a.n - 1)
                        merge_pair(a.tmp, node, lo, hi, sLo[pad(j - base)], sHi[pad(j - base)], lo, hi);
                    ++node;
                }
                if (outPos < C) {
                    dst[2ull * outPos] = lo;
                    dst[2ull * outPos + 1] = hi;
                }
                ++outPos;
            }
        }
        if (!grid_barrier(a.ctl, a.error, a.spinLimit, &sFlag)) return;
        cur ^= 1;
        ++iter;
        // counts only shrink (every iteration merges); the clamps keep a wrong
        // count from reaching past the buffers
        const uint32_t next = min(C, ld_acquire(&a.ctl->clusters[iter & 1]));
        if ((unsigned long long)(C - next) * 64ull < C) {
            pairNext = hashTies;
            hashTies = true;
        } else {
            pairNext = false;
        }
        C = next;
        merged = min(a.n - 1, ld_acquire(&a.ctl->merged[iter & 1]));
    }

    // ------------------------------------------------------------------ tail
    if (blockIdx.x == 0) {
        const float4* src = cur ? a.clusters[1] : a.clusters[0];
        for (uint32_t k = tid; k < C; k += kPlocThreads) {
            sLo[pad(k)] = __ldcg(src + 2ull * k);
            sHi[pad(k)] = __ldcg(src + 2ull * k + 1);
        }
        __syncthreads();
        while (C > 1) {
            const bool pairs = pairNext;
            {
                const uint32_t g0 = kPer * tid;  // C <= kTile: one group per thread
                if (g0 < C) {
                    if (pairs)
                        pair_partners(g0, 0, C, 0, C, sNN);
                    else
                        nearest<R>(g0, 0, C, 0, C, r, sLo, sHi, sNN);
                }
            }
            __syncthreads();
            if (hashTies && !pairs) {
                const uint32_t g0 = kPer * tid;
                if (g0 < C) resolve_ties(g0, 0, C, 0, C, r, sLo, sHi, sNN);
                __syncthreads();
            }
            const uint32_t p0 = kPer * tid;
            const Decision dc = decide(p0, C, 0, sNN);
            uint32_t total;
            const uint32_t before = sort::block_scan(__popc(dc.keepMask) | __popc(dc.mergeMask) << 16, sWarp, &total);
            float4 keepLo[kPer], keepHi[kPer];
            uint32_t node = merged + (before >> 16);
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                keepLo[q] = keepHi[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (!((dc.keepMask >> q) & 1u)) continue;
                const uint32_t p = p0 + q;
                keepLo[q] = sLo[pad(p)];
                keepHi[q] = sHi[pad(p)];
                if ((dc.mergeMask >> q) & 1u) {
                    const uint32_t j = sNN[pad(p)];
                    if (node < a.n - 1)
                        merge_pair(a.tmp, node, keepLo[q], keepHi[q], sLo[pad(j)], sHi[pad(j)], keepLo[q], keepHi[q]);
                    ++node;
                }
            }
            __syncthreads();  // every read of this iteration's clusters is done
            uint32_t outPos = before & 0xFFFFu;
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
                if (!((dc.keepMask >> q) & 1u)) continue;
                sLo[pad(outPos)] = keepLo[q];
                sHi[pad(outPos)] = keepHi[q];
                ++outPos;
            }
            merged += total >> 16;
            const uint32_t next = total & 0xFFFFu;
            if ((unsigned long long)(C - next) * 64ull < C) {
                pairNext = hashTies;
                hashTies = true;
            } else {
                pairNext = false;
            }
            C = next;
            __syncthreads();
        }
        // the root (the last node made) has the first leaf and no parent
        if (tid == 0 && merged > 0)
            st_relaxed64(a.info + merged - 1, (unsigned long long)kInvalid << 32);
    }
    if (!grid_barrier(a.ctl, a.error, a.spinLimit, &sFlag)) return;

    // ------------------------------------------------------------- placement
    place_all(a);
}

// The cooperative launch of k_ploc<R> with as many CTAs as can be resident
// (at most kMaxCtasPerSm per multiprocessor, at most one per first-iteration
// tile).
template <int R>
mlbvh_status launch_ploc(PlocArgs& a, uint32_t firstTiles, cudaStream_t stream)
{
    cudaError_t e = cudaFuncSetAttribute(k_ploc<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPlocSmem);
    int perSm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ploc<R>, kPlocThreads, kPlocSmem);
    if (e != cudaSuccess) return fail(MLBVH_ERR_LAUNCH, cudaGetErrorString(e));
    if (perSm < 1) return fail(MLBVH_ERR_LAUNCH, "k_ploc does not fit on a multiprocessor");
    const uint32_t sms = (uint32_t)device_sm_count();
    const int grid = (int)std::max<uint32_t>(
        1u, std::min<uint32_t>(firstTiles, (uint32_t)std::min(perSm, kMaxCtasPerSm) * sms));
    void* args[] = {&a};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_ploc<R>), dim3(grid), dim3(kPlocThreads), args,
                                    kPlocSmem, stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_LAUNCH, cudaGetErrorString(e));
    return MLBVH_OK;
}

}  // namespace

size_t build_ploc_scratch_bytes(uint32_t n) { return ploc_layout(n).total; }

mlbvh_status build_ploc(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, int radius,
                        mlbvh_internal_node* dNodes, mlbvh_node_index* dRoot, mlbvh_aabb* dScene, void* dScratch,
                        size_t scratchBytes, cudaStream_t stream, uint32_t spinLimit)
{
    if (n == 0 || n >= (1u << 30)) return fail(MLBVH_ERR_INVALID_ARG, "nTriangles must be in [1, 2^30)");
    if (radius < 1 || radius > kMaxRadius) return fail(MLBVH_ERR_INVALID_ARG, "radius must be in [1, 32]");
    if (!dTris || !dRoot || !dScratch) return fail(MLBVH_ERR_INVALID_ARG, "null triangles, root or scratch pointer");
    if (n > 1 && !dNodes) return fail(MLBVH_ERR_INVALID_ARG, "null internal-node pointer");
    if (!aligned16(dTris) || !aligned16(dNodes) || !aligned16(dScratch) || !aligned16(dRoot) || !aligned16(dScene))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    const PlocLayout L = ploc_layout(n);
    if (scratchBytes < L.total)
        return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_build_ploc_scratch_bytes(n)");
    if (n == 1)  // one leaf: every builder's tree
        return build(dTris, n, option, dNodes, dRoot, dScene, nullptr, nullptr, nullptr, dScratch, scratchBytes,
                     stream, spinLimit);

    SortedLeaves sl;
    mlbvh_status st = sort_leaves(dTris, n, option, dScene, nullptr, nullptr, nullptr, dScratch, stream, spinLimit, &sl);
    if (st != MLBVH_OK) return st;

    char* s = static_cast<char*>(dScratch);
    PlocArgs a;
    a.clusters[0] = reinterpret_cast<float4*>(s + L.clustersA);
    a.clusters[1] = reinterpret_cast<float4*>(s + L.clustersB);
    a.tmp = reinterpret_cast<float4*>(s + L.tmp);
    a.info = reinterpret_cast<unsigned long long*>(s + L.info);
    a.flags = reinterpret_cast<unsigned long long*>(s + L.flags);
    a.ctl = reinterpret_cast<PlocControl*>(s + L.control);
    a.error = sl.error;
    a.out = dNodes;
    a.root = dRoot;
    a.n = n;
    a.maxTiles = L.maxTiles;
    a.radius = (uint32_t)radius;
    a.spinLimit = sl.spinLimit;

    const int sms = device_sm_count();
    const int initBlocks = std::max(1, std::min<int>((n + kInitThreads - 1) / kInitThreads, 8 * sms));
    k_ploc_init<<<initBlocks, kInitThreads, 0, stream>>>(reinterpret_cast<const float*>(dTris), sl.indices, n,
                                                         a.clusters[0], a.flags, 2 * L.maxTiles, a.ctl, a.info);
    MLBVH_CHECK_LAUNCH("k_ploc_init");

    ProfileEvents ev = take_profile_events();
    if (ev.start) cudaEventRecord(ev.start, stream);
    const uint32_t firstTiles = (n + (kTile - 2u * radius) - 1) / (kTile - 2u * radius);
    switch (radius) {
        case 4: st = launch_ploc<4>(a, firstTiles, stream); break;
        case 8: st = launch_ploc<8>(a, firstTiles, stream); break;
        case 16: st = launch_ploc<16>(a, firstTiles, stream); break;
        case 32: st = launch_ploc<32>(a, firstTiles, stream); break;
        default: st = launch_ploc<0>(a, firstTiles, stream); break;
    }
    if (st != MLBVH_OK) return st;
    if (ev.stop) cudaEventRecord(ev.stop, stream);
    return MLBVH_OK;
}

}  // namespace mlbvh
