// Shading on B200: the reference's normal / ao / pt / pack kernels
// (main_gpu.cu:84-286) restated over this library's traversal.
//
// AO runs in three kernels: k_ao_primary traces one closest-hit ray per pixel
// and appends each hit pixel (AO origin and facing normal) to a queue, so no
// later work is spent on missed pixels; k_ao_rays is a persistent kernel in
// which every lane owns one queued pixel at a time and steps its any-hit rays
// one node per iteration, refilling idle lanes from the queue (no lane waits
// for the longest ray of its warp); k_ao_finish turns the per-pixel occlusion
// counts into the packed image.
#include <algorithm>

#include <type_traits>

#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {

namespace {

constexpr int kTileW = 16, kTileH = 8;  // 128-thread pixel tile: 4 warps of 8 x 4 pixels
constexpr int kAoThreads = 128;

// Build-time overrides for tuning sweeps (-DMLBVH_AO_START_BATCH=...).
#ifndef MLBVH_AO_START_BATCH
#define MLBVH_AO_START_BATCH 8
#endif
#ifndef MLBVH_AO_STEPS_PER_ROUND
#define MLBVH_AO_STEPS_PER_ROUND 3
#endif
#ifndef MLBVH_AO_WIDE_STEPS_PER_ROUND
#define MLBVH_AO_WIDE_STEPS_PER_ROUND 2
#endif
#ifndef MLBVH_AO_QWIDE_STEPS_PER_ROUND
#define MLBVH_AO_QWIDE_STEPS_PER_ROUND 1
#endif
#ifndef MLBVH_AO_MIN_BLOCKS
#define MLBVH_AO_MIN_BLOCKS 8
#endif
#ifndef MLBVH_AO_QUANT_MIN_BLOCKS
#define MLBVH_AO_QUANT_MIN_BLOCKS 9
#endif
// resident CTAs per SM of the AO kernel over quantised 4-wide slots (swept: 9
// and 10, at 56 and 48 registers, ran 3 and 4 % slower than 8 at 63)
#ifndef MLBVH_AO_QWIDE_MIN_BLOCKS
#define MLBVH_AO_QWIDE_MIN_BLOCKS 8
#endif
// the stack-free walk's own (swept: 4 steps and a batch of 16 lanes beat 3 and
// 8 by 1.7 %; a batch of 24 loses 7 %)
// the wide trees' refill batch (swept 4-16: 8 is best for the quantised slots,
// within 1 % of the best for the FP32 ones)
#ifndef MLBVH_AO_WIDE_START_BATCH
#define MLBVH_AO_WIDE_START_BATCH 8
#endif
#ifndef MLBVH_AO_PLAIN_STEPS_PER_ROUND
#define MLBVH_AO_PLAIN_STEPS_PER_ROUND 4
#endif
#ifndef MLBVH_AO_PLAIN_START_BATCH
#define MLBVH_AO_PLAIN_START_BATCH 16
#endif
constexpr int kFinishThreads = 256;

struct AoRecord {
    float ox, oy, oz;
    float nx, ny, nz;
    uint32_t pixel;
    uint32_t pad;  // replay forms: the node AO rays of this pixel start from (ball_start)
};

struct RenderLayout {
    size_t header;  // u32 queue count, u32 pad, u64 work counter
    size_t records;
    size_t counts;
    size_t total;
};
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
RenderLayout render_layout(int w, int h)
{
    RenderLayout L;
    const size_t px = (size_t)w * (size_t)h;
    L.header = 0;
    L.records = 256;
    L.counts = align256(L.records + sizeof(AoRecord) * px);
    L.total = align256(L.counts + sizeof(uint32_t) * px);
    return L;
}

__device__ __forceinline__ Camera to_camera(const mlbvh_ray_generator& g)
{
    Camera c;
    c.origin = mk(g.origin[0], g.origin[1], g.origin[2]);
    c.right = mk(g.right[0], g.right[1], g.right[2]);
    c.up = mk(g.up[0], g.up[1], g.up[2]);
    return c;
}

__device__ __forceinline__ bool tile_pixel(int w, int h, int& xi, int& yi)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    xi = blockIdx.x * kTileW + (lane & 7) + 8 * (warp & 1);
    yi = blockIdx.y * kTileH + (lane >> 3) + 4 * (warp >> 1);
    return xi < w && yi < h;
}

// The path tracer's own tiles: kPtWarps warps of 8 x 4 pixels (1: 8 x 4,
// 2: 16 x 4, 4: 16 x 8, the other kernels' tile). A CTA holds its slot until
// its longest path is done, and Russian roulette makes path lengths differ
// widely; measured on the bench's PT pass (replay walk): 0.615 / 0.621 / 0.626
// ms (build-time override for sweeps: -DMLBVH_PT_WARPS).
#ifndef MLBVH_PT_WARPS
#define MLBVH_PT_WARPS 1
#endif
constexpr int kPtWarps = MLBVH_PT_WARPS;
static_assert(kPtWarps == 1 || kPtWarps == 2 || kPtWarps == 4, "1, 2 or 4 warps per path-tracing tile");
constexpr int kPtThreads = 32 * kPtWarps;
constexpr int kPtTileW = kPtWarps >= 2 ? 16 : 8, kPtTileH = kPtWarps == 4 ? 8 : 4;
__device__ __forceinline__ bool pt_pixel(int w, int h, int& xi, int& yi)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    xi = blockIdx.x * kPtTileW + (lane & 7) + 8 * (warp & 1);
    yi = blockIdx.y * kPtTileH + (lane >> 3) + 4 * (warp >> 1);
    return xi < w && yi < h;
}

// PCG32 jump-ahead by `delta` steps (Brown, "Random Number Generation with
// Arbitrary Strides", 1994), so that AO sample i can start at draw 2i.
__device__ __forceinline__ void pcg_advance(Pcg& r, uint64_t delta)
{
    uint64_t curMult = 6364136223846793005ULL, curPlus = r.inc, accMult = 1, accPlus = 0;
    while (delta > 0) {
        if (delta & 1) {
            accMult *= curMult;
            accPlus = accPlus * curMult + curPlus;
        }
        curPlus = (curMult + 1) * curPlus;
        curMult *= curMult;
        delta >>= 1;
    }
    r.state = accMult * r.state + accPlus;
}

// Traversal counters of the counting variants: visits = internal-node loads,
// tests = triangle tests, ups = parent-word loads (quantised tree only).
struct Counts {
    uint32_t visits = 0, tests = 0, ups = 0;
};

// Adds per-thread counts to stats[1] (node visits), [2] (triangle tests) and
// [5] (parent loads) with one atomic per warp; AO rays also to [3], [4], [6].
__device__ __forceinline__ void add_stats(unsigned long long* stats, const Counts& c, bool aoRays)
{
    unsigned long long v = c.visits, t = c.tests, u = c.ups;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        t += __shfl_xor_sync(0xffffffffu, t, o);
        u += __shfl_xor_sync(0xffffffffu, u, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(stats + 1, v);
        atomicAdd(stats + 2, t);
        atomicAdd(stats + 5, u);
        if (aoRays) {
            atomicAdd(stats + 3, v);
            atomicAdd(stats + 4, t);
            atomicAdd(stats + 6, u);
        }
    }
}

// The cube around an AO origin that holds every point an AO ray of length
// radius can reach (directions are unit vectors), widened by 0.1% of the
// radius plus 1e-6 of the coordinates' magnitude and rounded outward, so
// that it also holds the hit points the triangle test can report.
struct AoBall {
    f3 lo, hi;
};
__device__ __forceinline__ AoBall ao_ball(f3 o, float radius)
{
    const float mag = __fadd_ru(__fadd_ru(fabsf(o.x), fabsf(o.y)), __fadd_ru(fabsf(o.z), radius));
    const float r = __fadd_ru(__fmul_ru(radius, 1.001f), __fmul_ru(mag, 1e-6f));
    return AoBall{mk(__fsub_rd(o.x, r), __fsub_rd(o.y, r), __fsub_rd(o.z, r)),
                  mk(__fadd_ru(o.x, r), __fadd_ru(o.y, r), __fadd_ru(o.z, r))};
}
__device__ __forceinline__ bool box_meets(f3 lo, f3 hi, const AoBall& b)
{
    return lo.x <= b.hi.x && lo.y <= b.hi.y && lo.z <= b.hi.z && hi.x >= b.lo.x && hi.y >= b.lo.y && hi.z >= b.lo.z;
}

// The tree formats and walks the AO kernels run over: the reference node
// layout with the stack-free walk (kWalk 0), the replay walk (kWalk 1: the
// same Hit records from a stack of pending far children), or the replay walk
// over leaf-ordered 48-byte triangles (kWalk 2); and the quantised tree with
// the replay walk. Primary rays of the replay forms take the closest-hit
// replay walk (pstack: 16 entries per thread in shared memory).
constexpr int kReplayDepth = 16;
template <int kWalk>
struct PlainTreeT {
    const mlbvh_internal_node* nodes;
    const float* tris;
    const mlbvh_node_index* rootPtr;
    const mlbvh_qtri* leafTris;  // kWalk 2 only
    struct Ctx {
        uint32_t root;  // kWalk 2: a leaf root is named by its position, 0
    };
    __device__ __forceinline__ Ctx context() const
    {
        const uint32_t r = __ldg(rootPtr);
        return Ctx{(kWalk == 2 && (r & kLeafBit)) ? kLeafBit : r};
    }
    static constexpr int kStack = kWalk > 0 ? kReplayDepth : 0;
    static constexpr int kPrimaryStack = kStack;  // closest-hit replay stack of primary rays
    static constexpr int kMinBlocks = kWalk == 0 ? 10 : MLBVH_AO_MIN_BLOCKS;
    static constexpr int kSteps = kWalk == 0 ? MLBVH_AO_PLAIN_STEPS_PER_ROUND : MLBVH_AO_STEPS_PER_ROUND;
    static constexpr int kStartBatch = kWalk == 0 ? MLBVH_AO_PLAIN_START_BATCH : MLBVH_AO_START_BATCH;
    // Replay forms: the node where AO rays from the ball's centre start. From
    // the root, while exactly one child's box meets the ball, go down into it;
    // stop where both do (or at a leaf). Every leaf an AO ray of the pixel can
    // hit lies below that node; kInvalid: no box meets the ball, nothing can be
    // hit. Leaves are named as the walk names them.
    __device__ __forceinline__ uint32_t ball_start(const Ctx& c, const AoBall& b) const
    {
        uint32_t curr = c.root;
        for (uint32_t steps = 0; !(curr & kLeafBit) && steps < kMaxTraversalSteps; ++steps) {
            const NodeView nd = load_node<true>(nodes, curr);
            const bool m0 = box_meets(nd.lo0, nd.hi0, b), m1 = box_meets(nd.lo1, nd.hi1, b);
            if (m0 && m1) return curr;
            if (!m0 && !m1) return kInvalid;
            const uint32_t child = m0 ? nd.c0 : nd.c1;
            curr = (kWalk == 2 && (child & kLeafBit)) ? (kLeafBit | (curr + (m0 ? 0u : 1u))) : child;
        }
        return curr;
    }
    template <bool kAny, bool kCount, class Entry>
    __device__ __forceinline__ bool walk(uint32_t& curr, uint32_t& prev, int& depth, Entry* stack, int stride,
                                         HitRecord& hit, f3 ro, f3 rd, f3 inv, Counts& n) const
    {
        if constexpr (kWalk == 2)
            return stackfree_replay_step_lo<kAny, kCount, kReplayDepth>(curr, prev, depth, stack, stride, hit, nodes,
                                                                        tris, leafTris, ro, rd, inv, 0.0f, n.visits,
                                                                        n.tests);
        else if constexpr (kWalk == 1)
            return stackfree_replay_step<kAny, kCount, kReplayDepth>(curr, prev, depth, stack, stride, hit, nodes, tris,
                                                                     ro, rd, inv, 0.0f, n.visits, n.tests);
        else
            return stackfree_step<kAny, kCount, true>(curr, prev, hit, nodes, tris, ro, rd, inv, 0.0f, n.visits,
                                                      n.tests);
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ void trace(const Ctx& c, HitRecord& hit, f3 ro, f3 rd, Counts& n, uint2* pstack,
                                          int stride) const
    {
        if constexpr (kWalk == 0) {
            trace_stackfree<kAny, kCount, true>(hit, nodes, tris, c.root, ro, rd, inv_rd(rd), 0.0f, &n.visits,
                                                &n.tests);
        } else {
            static_assert(!kAny, "primary rays are closest-hit");
            const f3 inv = inv_rd(rd);
            uint32_t curr = c.root, prev = kInvalid;
            int depth = 0;
            for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
                if (walk<false, kCount>(curr, prev, depth, pstack, stride, hit, ro, rd, inv, n)) break;
        }
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ bool step(const Ctx&, uint32_t& curr, uint32_t& prev, int& depth, uint32_t* stack,
                                         HitRecord& hit, f3 ro, f3 rd, f3 inv, Counts& n, bool fits) const
    {
        static_assert(kWalk == 0 || kAny, "AO rays are any-hit");
        return walk<kAny, kCount>(curr, prev, depth, stack, kAoThreads, hit, ro, rd, inv, n);
    }
};
using PlainTree = PlainTreeT<0>;
using PlainReplayTree = PlainTreeT<1>;
using PlainReplayLeafTree = PlainTreeT<2>;
struct QuantTree {
    const mlbvh_qnode* qnodes;
    const uint32_t* parents;
    const mlbvh_qtri* qtris;
    const mlbvh_qheader* header;
    struct Ctx {
        uint32_t root;
        int eb;
        uint32_t status;
    };
    __device__ __forceinline__ Ctx context() const
    {
        return Ctx{__ldg(&header->root), __ldg(&header->eBase), __ldg(&header->status)};
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ void trace(const Ctx& c, HitRecord& hit, f3 ro, f3 rd, Counts& n, uint2* pstack,
                                          int stride) const
    {
        static_assert(!kAny, "primary rays are closest-hit");
        const f3 inv = inv_rd(rd);
        const QParams qp{c.eb, c.status, c.status == 0u && qwide_ray_fits(ro, inv)};
        uint32_t curr = c.root, prev = kInvalid;
        int depth = 0;
        for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
            if (quantised_replay_step<false, kCount, kStack>(curr, prev, depth, pstack, stride, hit, qnodes, parents,
                                                            qtris, qp, ro, rd, inv, 0.0f, n.visits, n.tests, n.ups))
                break;
    }
    // the replay walk: the stack-free walk's leaf order with a stack of
    // kStack pending far children per lane (shared memory) instead of revisits;
    // only any-hit steps are taken (AO rays)
    static constexpr int kStack = 16;
    static constexpr int kPrimaryStack = kStack;
    static constexpr int kMinBlocks = MLBVH_AO_QUANT_MIN_BLOCKS;
    __device__ __forceinline__ uint32_t ball_start(const Ctx& c, const AoBall& b) const
    {
        if (c.status & 2u) return c.root;  // every box passes: no box bounds the ball
        uint32_t curr = c.root;
        for (uint32_t steps = 0; !(curr & kLeafBit) && steps < kMaxTraversalSteps; ++steps) {
            const QNodeWords nd = load_qnode(qnodes, curr, c.eb);
            f3 lo0, hi0, lo1, hi1;
            qnode_box(nd, 0, lo0, hi0);
            qnode_box(nd, 1, lo1, hi1);
            const bool m0 = box_meets(lo0, hi0, b), m1 = box_meets(lo1, hi1, b);
            if (m0 && m1) return curr;
            if (!m0 && !m1) return kInvalid;
            curr = m0 ? nd.c0 : nd.c1;
        }
        return curr;
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ bool step(const Ctx& c, uint32_t& curr, uint32_t& prev, int& depth, uint32_t* stack,
                                         HitRecord& hit, f3 ro, f3 rd, f3 inv, Counts& n, bool fits) const
    {
        const QParams qp{c.eb, c.status, c.status == 0u && fits};
        return quantised_replay_step<kAny, kCount, kStack>(curr, prev, depth, stack, kAoThreads, hit, qnodes, parents,
                                                           qtris, qp, ro, rd, inv, 0.0f, n.visits, n.tests, n.ups);
    }
};

// The 4-wide tree for AO rays (any-hit, wide_any_step) over FP32 slots or
// (kQuant) quantised slots; primary rays on the binary tree's replay walk over
// leaf-ordered triangles (closest hit, the stack-free walk's Hit records).
// Context: the walk's root (a leaf root is leaf position 0), the binary root
// as the reference names it (the restart of a ray whose wide stack would
// overflow) and, for quantised slots, whether they are unusable (every AO ray
// then takes the stack-free walk over the binary tree).
template <bool kQuant>
struct WideTreeT {
    using Slot = typename std::conditional<kQuant, mlbvh_qwnode, mlbvh_wnode>::type;
    PlainReplayLeafTree binary;
    const Slot* slots;
    const uint32_t* status;  // quantised slots only
    struct Ctx {
        uint32_t root, binaryRoot;
        bool fallback;
    };
    static constexpr int kStack = kWideDepth;
    static constexpr int kPrimaryStack = PlainReplayLeafTree::kStack;
    static constexpr int kSteps = kQuant ? MLBVH_AO_QWIDE_STEPS_PER_ROUND : MLBVH_AO_WIDE_STEPS_PER_ROUND;
    static constexpr int kStartBatch = MLBVH_AO_WIDE_START_BATCH;
    static constexpr int kMinBlocks = kQuant ? MLBVH_AO_QWIDE_MIN_BLOCKS : MLBVH_AO_MIN_BLOCKS;
    __device__ __forceinline__ Ctx context() const
    {
        const uint32_t r = __ldg(binary.rootPtr);
        return Ctx{(r & kLeafBit) ? kLeafBit : r, r, kQuant && __ldg(status) != 0u};
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ void trace(const Ctx& c, HitRecord& hit, f3 ro, f3 rd, Counts& n, uint2* pstack,
                                          int stride) const
    {
        binary.template trace<kAny, kCount>(PlainReplayLeafTree::Ctx{c.root}, hit, ro, rd, n, pstack, stride);
    }
    // From the root, while exactly one child's box meets the ball, go down
    // into it; stop where several do (or at a leaf); kInvalid where none does.
    // Quantised slots are tested on their decoded boxes, which contain the
    // exact ones.
    __device__ __forceinline__ uint32_t ball_start(const Ctx& c, const AoBall& b) const
    {
        if (c.fallback) return c.root;
        uint32_t curr = c.root;
        for (uint32_t steps = 0; !(curr & kLeafBit) && steps < kMaxTraversalSteps; ++steps) {
            const float4* p = reinterpret_cast<const float4*>(slots + curr);
            int meets = 0;
            uint32_t only = kInvalid;
            if constexpr (kQuant) {
                float4 a, q, c2, d;
                ldg32(p, a, q);
                ldg32(p + 2, c2, d);
                const uint32_t sx = __float_as_uint(a.w), sy = __float_as_uint(q.x), sz = __float_as_uint(q.y);
                const uint4 ch = make_uint4(__float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z),
                                            __float_as_uint(d.w));
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const f3 lo = mk(__fadd_rd(a.x, qw_value(__float_as_uint(q.z), sx, k)),
                                     __fadd_rd(a.y, qw_value(__float_as_uint(c2.x), sy, k)),
                                     __fadd_rd(a.z, qw_value(__float_as_uint(c2.z), sz, k)));
                    const f3 hi = mk(__fadd_ru(a.x, qw_value(__float_as_uint(q.w), sx, k)),
                                     __fadd_ru(a.y, qw_value(__float_as_uint(c2.y), sy, k)),
                                     __fadd_ru(a.z, qw_value(__float_as_uint(c2.w), sz, k)));
                    if (wpick(ch, k) != kWideEmpty && box_meets(lo, hi, b)) {
                        ++meets;
                        only = wpick(ch, k);
                    }
                }
            } else {
                float4 lx, hx, ly, hy, lz, hz;
                ldg32(p, lx, hx);
                ldg32(p + 2, ly, hy);
                ldg32(p + 4, lz, hz);
                const uint4 ch = __ldg(reinterpret_cast<const uint4*>(p + 6));
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (wpick(ch, k) != kWideEmpty && box_meets(mk(wpick(lx, k), wpick(ly, k), wpick(lz, k)),
                                                                mk(wpick(hx, k), wpick(hy, k), wpick(hz, k)), b)) {
                        ++meets;
                        only = wpick(ch, k);
                    }
            }
            if (meets == 0) return kInvalid;
            if (meets > 1) return curr;
            curr = only;
        }
        return curr;
    }
    template <bool kAny, bool kCount>
    __device__ __forceinline__ bool step(const Ctx& c, uint32_t& curr, uint32_t& prev, int& depth, uint32_t* stack,
                                         HitRecord& hit, f3 ro, f3 rd, f3 inv, Counts& n, bool fits) const
    {
        static_assert(kAny, "AO rays are any-hit");
        // unusable slots, or a ray outside qwide_ray_fits: the stack-free walk from the binary root
        if (kQuant && (c.fallback || !fits) && depth >= 0) {
            depth = -1;
            curr = c.binaryRoot;
            prev = kInvalid;
        }
        return wide_any_step<kCount, kQuant>(curr, prev, depth, stack, kAoThreads, hit, slots, binary.nodes,
                                             binary.tris, binary.leafTris, c.binaryRoot, ro, rd, inv, 0.0f, n.visits,
                                             n.tests, n.ups);
    }
};
using WideTree = WideTreeT<false>;
using QuantWideTree = WideTreeT<true>;

// Primary rays of ao (main_gpu.cu:121-144): closest hit, flip the normal
// towards the viewer, AO origin p + n * 1e-3.
template <class Tree, bool kCount>
__global__ void __launch_bounds__(kTileW* kTileH)
    k_ao_primary(mlbvh_ray_generator gen, int w, int h, float radius, Tree tree, AoRecord* __restrict__ records,
                 uint32_t* __restrict__ queueCount, uint32_t* __restrict__ counts, unsigned long long* __restrict__ stats)
{
    __shared__ uint2 s_pstack[Tree::kPrimaryStack > 0 ? Tree::kPrimaryStack : 1][kTileW * kTileH];
    Counts cnt;
    int xi, yi;
    const bool inside = tile_pixel(w, h, xi, yi);
    bool isHit = false;
    AoRecord rec;
    if (inside) {
        const Camera cam = to_camera(gen);
        const int pixel = xi + yi * w;
        f3 ro, rd;
        shoot(cam, (float)xi / (float)w, (float)yi / (float)h, ro, rd);
        HitRecord hit;
        hit.t = kFltMax;
        hit.tri = 0xFFFFFFFFu;
        tree.template trace<false, kCount>(tree.context(), hit, ro, rd, cnt, &s_pstack[0][threadIdx.x],
                                           kTileW * kTileH);
        if (hit.t == kFltMax) {
            counts[pixel] = 0xFFFFFFFFu;
        } else {
            f3 n = normalize(hit.ng);
            if (0.0f < dot(n, rd)) n = -n;
            const f3 o = ro + rd * hit.t + n * 0.001f;
            uint32_t start = 0u;
            if constexpr (Tree::kStack > 0) start = tree.ball_start(tree.context(), ao_ball(o, radius));
            rec = AoRecord{o.x, o.y, o.z, n.x, n.y, n.z, (uint32_t)pixel, start};
            counts[pixel] = 0u;
            isHit = true;
        }
    }
    if (kCount) add_stats(stats, cnt, false);
    // warp-aggregated append to the hit queue
    const uint32_t mask = __ballot_sync(0xffffffffu, isHit);
    if (mask == 0u) return;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == __ffs(mask) - 1) base = atomicAdd(queueCount, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
    if (isHit) {
        float4* dst = reinterpret_cast<float4*>(records + base + __popc(mask & ((1u << lane) - 1u)));
        dst[0] = make_float4(rec.ox, rec.oy, rec.oz, rec.nx);
        dst[1] = make_float4(rec.ny, rec.nz, __uint_as_float(rec.pixel), __uint_as_float(rec.pad));
    }
}

// AO rays (main_gpu.cu:146-173), scheduled per lane. A work item is one AO
// sample of one hit pixel, item i = (queue entry i / nSamples, sample
// i % nSamples). A warp takes kChunk consecutive items per atomic on the work
// counter, so its lanes mostly trace samples of the same pixel: rays from one
// origin share their upper paths, and the warp's node loads coalesce. Each
// lane traces its own ray one node (or leaf) per loop iteration and takes the
// next item as soon as it is free, so lanes never wait for the longest ray of
// their warp. Setting a ray up (Sobol point, hemisphere direction, reciprocal
// direction) costs about as much as several traversal steps, so free lanes
// take items once kStartBatch of them are free (or none is busy), and the
// set-up runs for many lanes at once. An occluded ray adds one to its pixel's
// count; the lanes of a warp add per pixel with one atomic.
constexpr int kChunk = 64;
constexpr int kStartBatch = MLBVH_AO_START_BATCH;
// Traversal steps per lane between two refill checks: a tree's kSteps (the
// wide tree's steps are about twice as long: 2; its quantised steps longer
// still: 1, measured 2 % faster than 2), else kStepsPerRound.
constexpr int kStepsPerRound = MLBVH_AO_STEPS_PER_ROUND;
template <class Tree, class = void>
struct StepsOf {
    static constexpr int value = kStepsPerRound;
};
template <class Tree>
struct StepsOf<Tree, decltype((void)Tree::kSteps)> {
    static constexpr int value = Tree::kSteps;
};
// Resident CTAs per SM the kernel is compiled for: a tree's kMinBlocks, else
// MLBVH_AO_MIN_BLOCKS (8: at most 64 registers, 32 warps per SM). The
// stack-free walk fits 10 (48 registers) without spills and gains from the
// extra warps; the stack and wide walks spill below 64 registers.
template <class Tree, class = void>
struct StartBatchOf {
    static constexpr int value = kStartBatch;
};
template <class Tree>
struct StartBatchOf<Tree, decltype((void)Tree::kStartBatch)> {
    static constexpr int value = Tree::kStartBatch;
};
template <class Tree, class = void>
struct MinBlocksOf {
    static constexpr int value = MLBVH_AO_MIN_BLOCKS;
};
template <class Tree>
struct MinBlocksOf<Tree, decltype((void)Tree::kMinBlocks)> {
    static constexpr int value = Tree::kMinBlocks;
};

template <class Tree, bool kCount>
__global__ void __launch_bounds__(kAoThreads, MinBlocksOf<Tree>::value)
    k_ao_rays(const AoRecord* __restrict__ records, const uint32_t* __restrict__ queueCount,
              unsigned long long* __restrict__ workCounter, int w, int nSamples, float radius, uint32_t seed,
              int useSobol, Tree tree, uint32_t* __restrict__ counts, unsigned long long* __restrict__ stats)
{
    Counts cnt;
    const int lane = threadIdx.x & 31;
    const uint32_t lanesBelow = (1u << lane) - 1u;
    const unsigned long long total = (unsigned long long)(*queueCount) * (unsigned long long)nSamples;
    const typename Tree::Ctx ctx = tree.context();
    __shared__ uint32_t s_stack[Tree::kStack > 0 ? Tree::kStack : 1][kAoThreads];  // AO rays are any-hit
    uint32_t* const stack = &s_stack[0][threadIdx.x];
    unsigned long long poolNext = 0, poolEnd = 0;  // warp-uniform: items taken, not yet handed out
    bool exhausted = false;                        // warp-uniform: the work counter is past the end
    bool live = false;                             // this lane has a ray in flight
    uint32_t pixel = 0, curr = 0, prev = 0, steps = 0;
    int depth = 0;
    f3 origin = mk(0, 0, 0), dir = origin, inv = origin;
    bool fits = true;  // qwide_ray_fits of this lane's ray (the quantised trees use it)
    HitRecord hit;
    hit.t = radius;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !live);
        if (idle == 0xffffffffu || (uint32_t)__popc(idle) >= (uint32_t)StartBatchOf<Tree>::value) {
            if (poolNext >= poolEnd && !exhausted) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(workCounter, (unsigned long long)kChunk);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= total) {
                    exhausted = true;
                } else {
                    poolNext = base;
                    poolEnd = min(base + (unsigned long long)kChunk, total);
                }
            }
            if (poolNext < poolEnd) {
                const unsigned long long avail = poolEnd - poolNext;
                const uint32_t rank = __popc(idle & lanesBelow);
                if (!live && rank < avail) {  // start item poolNext + rank
                    const unsigned long long item = poolNext + rank;
                    const uint32_t entry = (uint32_t)(item / (uint32_t)nSamples);
                    const uint32_t s = (uint32_t)(item - (unsigned long long)entry * (uint32_t)nSamples);
                    const float4* rp = reinterpret_cast<const float4*>(records + entry);
                    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
                    origin = mk(r0.x, r0.y, r0.z);
                    const f3 n = mk(r0.w, r1.x, r1.y);
                    pixel = __float_as_uint(r1.z);
                    const uint32_t start = Tree::kStack > 0 ? __float_as_uint(r1.w) : ctx.root;
                    f3 xaxis, zaxis;
                    onb(n, xaxis, zaxis);
                    float2 rnd;
                    if (useSobol) {
                        rnd = sobol2d(s, pixel % (uint32_t)w, pixel / (uint32_t)w, seed);
                    } else {
                        Pcg rng(hash_pcg(pixel), 0);
                        pcg_advance(rng, 2ull * s);
                        rnd.x = rng.uniformf();
                        rnd.y = rng.uniformf();
                    }
                    const f3 dl = sample_hemisphere(rnd.x, rnd.y);
                    dir = xaxis * dl.x + zaxis * dl.z + n * dl.y;
                    inv = inv_rd(dir);
                    fits = qwide_ray_fits(origin, inv);
                    hit.t = radius;
                    hit.tri = 0xFFFFFFFFu;
                    curr = start;
                    prev = kInvalid;
                    depth = 0;
                    steps = 0;
                    live = start != kInvalid;  // kInvalid: no box within the AO radius, the ray misses
                }
                poolNext += min((unsigned long long)__popc(idle), avail);
            }
        }
        if (!__any_sync(0xffffffffu, live)) {
            if (exhausted) break;
            continue;
        }
        // up to StepsOf<Tree> steps per loop iteration: the refill and vote
        // overhead of an iteration is shared by several steps
        bool occluded = false;
#pragma unroll
        for (int rep = 0; rep < StepsOf<Tree>::value; ++rep)
            if (live) {
                if (tree.template step<true, kCount>(ctx, curr, prev, depth, stack, hit, origin, dir, inv, cnt,
                                                     fits) ||
                    ++steps >= kMaxTraversalSteps) {
                    live = false;
                    occluded = hit.t != radius;
                }
            }
        // one atomic per pixel among the lanes whose ray just ended occluded
        uint32_t pending = __ballot_sync(0xffffffffu, occluded);
        while (pending) {
            const int leader = __ffs(pending) - 1;
            const uint32_t p = __shfl_sync(0xffffffffu, pixel, leader);
            const uint32_t same = __ballot_sync(0xffffffffu, occluded && pixel == p);
            if (lane == leader) atomicAdd(counts + p, (uint32_t)__popc(same));
            pending &= ~same;
        }
    }
    if (kCount) add_stats(stats, cnt, true);
}

// The tail of ao (main_gpu.cu:169-176): ao accumulates 1/nSample per occluded
// ray in float (so it equals the reference's sum), gamma 1/2.2, pack.
__global__ void __launch_bounds__(kFinishThreads)
    k_ao_finish(const uint32_t* __restrict__ counts, int nPixels, int nSamples, uint32_t* __restrict__ pixels,
                uint32_t* __restrict__ occludedOut, const uint32_t* __restrict__ queueCount,
                unsigned long long* __restrict__ stats)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && stats) *stats = (unsigned long long)nPixels + (unsigned long long)(*queueCount) * nSamples;
    if (p >= nPixels) return;
    const uint32_t c = counts[p];
    uint32_t rgba;
    if (c == 0xFFFFFFFFu) {
        rgba = pack_rgba(0.0f, 0.0f, 0.0f);
    } else {
        float ao = 0.0f;
        const float step = 1.0f / (float)nSamples;
        for (uint32_t k = 0; k < c; ++k) ao += step;
        const float brightness = powf(1.0f - ao, 1.0f / 2.2f);
        rgba = pack_rgba(brightness, brightness, brightness);
    }
    if (pixels) pixels[p] = rgba;
    if (occludedOut) occludedOut[p] = c;
}

// normal (main_gpu.cu:84-109)
__global__ void __launch_bounds__(kTileW* kTileH)
    k_normal(uint32_t* __restrict__ pixels, mlbvh_ray_generator gen, int w, int h,
             const mlbvh_node_index* __restrict__ rootPtr, const mlbvh_internal_node* __restrict__ nodes,
             const float* __restrict__ tris)
{
    int xi, yi;
    if (!tile_pixel(w, h, xi, yi)) return;
    const Camera cam = to_camera(gen);
    f3 ro, rd;
    shoot(cam, (float)xi / (float)w, (float)yi / (float)h, ro, rd);
    HitRecord hit;
    hit.t = kFltMax;
    hit.tri = 0xFFFFFFFFu;
    trace_stackfree<false, false, true>(hit, nodes, tris, __ldg(rootPtr), ro, rd, inv_rd(rd), 0.0f);
    uint32_t rgba;
    if (hit.t != kFltMax) {
        const f3 n = normalize(hit.ng);
        const f3 c = (n + mk(1.0f, 1.0f, 1.0f)) * 0.5f;
        rgba = pack_rgba(c.x, c.y, c.z);
    } else {
        rgba = pack_rgba(0.0f, 0.0f, 0.0f);
    }
    pixels[xi + yi * w] = rgba;
}

struct PtRandom {
    int useSobol;
    uint32_t iteration, xi, yi, dim;
    Pcg rng;
    __device__ __forceinline__ float2 next()
    {
        if (useSobol) return sobol2d(iteration, xi, yi, dim++);
        float2 r;
        r.x = rng.uniformf();
        r.y = rng.uniformf();
        return r;
    }
};

// pt (main_gpu.cu:179-272): one progressive sample per pixel. Tree: the
// walk of every closest-hit ray (PlainTree: intersect_stackfree as the
// reference; the replay trees: the same Hit records from a per-thread stack
// of pending far children in shared memory), so the accumulators are the same.
template <class Tree>
__global__ void __launch_bounds__(kPtThreads)
    k_pt(float4* __restrict__ accum, mlbvh_ray_generator gen, int w, int h, Tree tree,
         const float* __restrict__ attribs, int useSobol, int maxSPP, int maxDepth)
{
    __shared__ uint2 s_pstack[Tree::kPrimaryStack > 0 ? Tree::kPrimaryStack : 1][kPtThreads];
    uint2* const pstack = &s_pstack[0][threadIdx.x];
    Counts cnt;
    int xi, yi;
    if (!pt_pixel(w, h, xi, yi)) return;
    const Camera cam = to_camera(gen);
    const int pixel = xi + yi * w;
    float4 acc = accum[pixel];
    const int iteration = (int)acc.w;
    PtRandom rr{useSobol, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, 0u,
                Pcg(hash_pcg(hash_pcg((uint32_t)pixel) + (uint32_t)iteration), 0)};
    const typename Tree::Ctx ctx = tree.context();
    float2 rnd = rr.next();
    f3 ro, rd;
    shoot(cam, ((float)xi + rnd.x) / (float)w, ((float)yi + rnd.y) / (float)h, ro, rd);
    f3 color = mk(0.0f, 0.0f, 0.0f);
    f3 throughput = mk(1.0f, 1.0f, 1.0f);
    HitRecord hit;
    hit.t = kFltMax;
    hit.tri = 0xFFFFFFFFu;
    tree.template trace<false, false>(ctx, hit, ro, rd, cnt, pstack, kPtThreads);
    if (hit.t != kFltMax)
        for (int depth = 0; depth < maxDepth; depth++) {
            const float2 r2 = rr.next();
            const f3 hit_p = ro + rd * hit.t;
            f3 hit_n = normalize(hit.ng);
            if (0.0f < dot(hit_n, rd)) hit_n = -hit_n;
            const float* at = attribs + 15 * (size_t)hit.tri;
            const f3 refl = mk(__ldg(at + 9), __ldg(at + 10), __ldg(at + 11));
            const f3 emis = mk(__ldg(at + 12), __ldg(at + 13), __ldg(at + 14));
            color = color + throughput * emis;
            f3 xaxis, zaxis;
            onb(hit_n, xaxis, zaxis);
            const f3 dl = sample_hemisphere(r2.x, r2.y);
            const f3 next_ro = hit_p + hit_n * 0.0001f;
            const f3 next_rd = xaxis * dl.x + zaxis * dl.z + hit_n * dl.y;
            throughput = throughput * refl;
            const float rrThreshold = 0.25f;
            const float maxComp = smax(smax(throughput.x, throughput.y), throughput.z);
            const float p = smin(maxComp / rrThreshold, 1.0f);
            if (p < rr.next().x) break;
            throughput = throughput / p;
            hit.t = kFltMax;
            hit.u = hit.v = 0.0f;
            hit.ng = mk(0.0f, 0.0f, 0.0f);
            hit.tri = 0xFFFFFFFFu;
            tree.template trace<false, false>(ctx, hit, next_ro, next_rd, cnt, pstack, kPtThreads);
            if (hit.t == kFltMax) break;
            ro = next_ro;
            rd = next_rd;
        }
    if (iteration < maxSPP) {
        acc.x += color.x;
        acc.y += color.y;
        acc.z += color.z;
        acc.w += 1.0f;
        accum[pixel] = acc;
    }
}

// pack (main_gpu.cu:273-286)
__global__ void k_pack(uint32_t* __restrict__ pixels, const float4* __restrict__ accum, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = accum[i];
    pixels[i] = pack_rgba(powf(a.x / a.w, 1.0f / 2.2f), powf(a.y / a.w, 1.0f / 2.2f), powf(a.z / a.w, 1.0f / 2.2f));
}

dim3 tile_grid(int w, int h) { return dim3((w + kTileW - 1) / kTileW, (h + kTileH - 1) / kTileH); }

mlbvh_status check_image(int w, int h)
{
    if (w <= 0 || h <= 0 || (long long)w * (long long)h >= (1ll << 31))
        return fail(MLBVH_ERR_INVALID_ARG, "image size must be positive and below 2^31 pixels");
    return MLBVH_OK;
}

template <class Tree>
int ao_ray_blocks()
{
    static int blocksPerSm = 0;
    if (blocksPerSm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_ao_rays<Tree, false>, kAoThreads, 0) != cudaSuccess ||
            b <= 0)
            b = 8;
        blocksPerSm = b;
    }
    return blocksPerSm * device_sm_count();
}

// The AO launch chain over either tree format (arguments already checked).
template <class Tree>
mlbvh_status launch_ao(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                       const Tree& tree, int useSobol, int nSamples, float radius, uint32_t seed,
                       unsigned long long* dStats, void* dScratch, size_t scratchBytes, cudaStream_t stream)
{
    const RenderLayout L = render_layout(w, h);
    if (scratchBytes < L.total) return fail(MLBVH_ERR_INVALID_ARG, "scratch smaller than mlbvh_render_scratch_bytes");
    char* s = static_cast<char*>(dScratch);
    uint32_t* header = reinterpret_cast<uint32_t*>(s + L.header);
    AoRecord* records = reinterpret_cast<AoRecord*>(s + L.records);
    uint32_t* counts = reinterpret_cast<uint32_t*>(s + L.counts);
    unsigned long long* work = reinterpret_cast<unsigned long long*>(s + L.header + 8);

    cudaError_t e = cudaMemsetAsync(header, 0, 16, stream);  // queue count, 64-bit work counter
    if (e == cudaSuccess && dStats) e = cudaMemsetAsync(dStats, 0, 8 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return fail(MLBVH_ERR_CUDA, cudaGetErrorString(e));
    const dim3 grid = tile_grid(w, h);
    if (dStats)
        k_ao_primary<Tree, true><<<grid, kTileW * kTileH, 0, stream>>>(cam, w, h, radius, tree, records, header, counts,
                                                                       dStats);
    else
        k_ao_primary<Tree, false><<<grid, kTileW * kTileH, 0, stream>>>(cam, w, h, radius, tree, records, header, counts,
                                                                        nullptr);
    MLBVH_CHECK_LAUNCH("k_ao_primary");
    ProfileEvents ev = take_profile_events();
    if (ev.start) cudaEventRecord(ev.start, stream);
    if (dStats)
        k_ao_rays<Tree, true><<<ao_ray_blocks<Tree>(), kAoThreads, 0, stream>>>(
            records, header, work, w, nSamples, radius, seed, useSobol, tree, counts, dStats);
    else
        k_ao_rays<Tree, false><<<ao_ray_blocks<Tree>(), kAoThreads, 0, stream>>>(
            records, header, work, w, nSamples, radius, seed, useSobol, tree, counts, nullptr);
    MLBVH_CHECK_LAUNCH("k_ao_rays");
    if (ev.stop) cudaEventRecord(ev.stop, stream);
    const int px = w * h;
    k_ao_finish<<<(px + kFinishThreads - 1) / kFinishThreads, kFinishThreads, 0, stream>>>(
        counts, px, nSamples, dPixels, dOccluded, header, dStats);
    MLBVH_CHECK_LAUNCH("k_ao_finish");
    return MLBVH_OK;
}

mlbvh_status check_ao_args(int w, int h, int nSamples, const void* dPixels, const void* dOccluded,
                           const void* dScratch, const unsigned long long* dStats)
{
    if (mlbvh_status s = check_image(w, h)) return s;
    if (nSamples <= 0 || nSamples > 65536) return fail(MLBVH_ERR_INVALID_ARG, "nSamples must be in [1, 65536]");
    if (!dScratch) return fail(MLBVH_ERR_INVALID_ARG, "null scratch pointer");
    if (!aligned16(dPixels) || !aligned16(dOccluded) || !aligned16(dScratch) ||
        (reinterpret_cast<uintptr_t>(dStats) & 7u))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    return MLBVH_OK;
}

}  // namespace

size_t render_scratch_bytes(int w, int h)
{
    if (w <= 0 || h <= 0) return 0;
    return render_layout(w, h).total;
}

mlbvh_status render_normal(uint32_t* dPixels, int w, int h, const mlbvh_ray_generator& cam,
                           const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                           const mlbvh_triangle* dTris, cudaStream_t stream)
{
    if (mlbvh_status s = check_image(w, h)) return s;
    if (!dPixels || !dRoot || !dTris) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dPixels) || !aligned16(dRoot) || !aligned32(dNodes) || !aligned16(dTris))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    k_normal<<<tile_grid(w, h), kTileW * kTileH, 0, stream>>>(dPixels, cam, w, h, dRoot, dNodes,
                                                              reinterpret_cast<const float*>(dTris));
    MLBVH_CHECK_LAUNCH("k_normal");
    return MLBVH_OK;
}

mlbvh_status render_ao(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                       const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                       int useSobol, int nSamples, float radius, uint32_t seed, unsigned long long* dStats,
                       void* dScratch, size_t scratchBytes, int traversal, const mlbvh_qtri* dLeafTris,
                       cudaStream_t stream)
{
    if (mlbvh_status s = check_ao_args(w, h, nSamples, dPixels, dOccluded, dScratch, dStats)) return s;
    if (!dRoot || !dTris) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dRoot) || !aligned32(dNodes) || !aligned16(dTris))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (!aligned16(dLeafTris)) return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (traversal == MLBVH_TRAVERSAL_REPLAY && dLeafTris) {
        const PlainReplayLeafTree tree{dNodes, reinterpret_cast<const float*>(dTris), dRoot, dLeafTris};
        return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                         scratchBytes, stream);
    }
    if (traversal == MLBVH_TRAVERSAL_REPLAY) {
        const PlainReplayTree tree{dNodes, reinterpret_cast<const float*>(dTris), dRoot, nullptr};
        return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                         scratchBytes, stream);
    }
    if (traversal != MLBVH_TRAVERSAL_STACKFREE)
        return fail(MLBVH_ERR_INVALID_ARG, "AO traversal must be MLBVH_TRAVERSAL_STACKFREE or MLBVH_TRAVERSAL_REPLAY");
    const PlainTree tree{dNodes, reinterpret_cast<const float*>(dTris), dRoot, nullptr};
    return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                     scratchBytes, stream);
}

mlbvh_status render_ao_wide(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                            const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                            const mlbvh_triangle* dTris, const mlbvh_wnode* dWide, const mlbvh_qtri* dLeafTris,
                            int useSobol, int nSamples, float radius, uint32_t seed, unsigned long long* dStats,
                            void* dScratch, size_t scratchBytes, cudaStream_t stream)
{
    if (mlbvh_status s = check_ao_args(w, h, nSamples, dPixels, dOccluded, dScratch, dStats)) return s;
    if (!dRoot || !dTris || !dLeafTris) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dRoot) || !aligned32(dNodes) || !aligned16(dTris) || !aligned16(dLeafTris) ||
        (reinterpret_cast<uintptr_t>(dWide) & 127u))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers misaligned (wide nodes 128 B, nodes 32 B, others 16 B)");
    const WideTree tree{PlainReplayLeafTree{dNodes, reinterpret_cast<const float*>(dTris), dRoot, dLeafTris}, dWide,
                        nullptr};
    return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                     scratchBytes, stream);
}

mlbvh_status render_ao_wide_quantised(uint32_t* dPixels, uint32_t* dOccluded, int w, int h,
                                      const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                                      const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                                      const mlbvh_qwnode* dQWide, const uint32_t* dStatus,
                                      const mlbvh_qtri* dLeafTris, int useSobol, int nSamples, float radius,
                                      uint32_t seed, unsigned long long* dStats, void* dScratch, size_t scratchBytes,
                                      cudaStream_t stream)
{
    if (mlbvh_status s = check_ao_args(w, h, nSamples, dPixels, dOccluded, dScratch, dStats)) return s;
    if (!dRoot || !dTris || !dLeafTris || !dStatus) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dRoot) || !aligned32(dNodes) || !aligned16(dTris) || !aligned16(dLeafTris) ||
        !aligned16(dStatus) || !aligned32(dQWide))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers misaligned (quantised slots and nodes 32 B, others 16 B)");
    const QuantWideTree tree{PlainReplayLeafTree{dNodes, reinterpret_cast<const float*>(dTris), dRoot, dLeafTris},
                             dQWide, dStatus};
    return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                     scratchBytes, stream);
}

mlbvh_status render_ao_quantised(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                                 const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                 const mlbvh_qheader* dQHeader, int useSobol, int nSamples, float radius,
                                 uint32_t seed, unsigned long long* dStats, void* dScratch, size_t scratchBytes,
                                 cudaStream_t stream)
{
    if (mlbvh_status s = check_ao_args(w, h, nSamples, dPixels, dOccluded, dScratch, dStats)) return s;
    if (!dQTris || !dQHeader) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned32(dQNodes) || !aligned16(dQParents) || !aligned16(dQTris) || !aligned16(dQHeader))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    const QuantTree tree{dQNodes, dQParents, dQTris, dQHeader};
    return launch_ao(dPixels, dOccluded, w, h, cam, tree, useSobol, nSamples, radius, seed, dStats, dScratch,
                     scratchBytes, stream);
}

mlbvh_status render_pt(float* dAccum, int w, int h, const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                       const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                       const mlbvh_triangle_attrib* dAttribs, int useSobol, int maxSPP, int maxDepth,
                       cudaStream_t stream, int traversal, const mlbvh_qtri* dLeafTris)
{
    if (mlbvh_status s = check_image(w, h)) return s;
    if (!dAccum || !dRoot || !dTris || !dAttribs) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dAccum) || !aligned16(dRoot) || !aligned32(dNodes) || !aligned16(dTris) || !aligned16(dAttribs) ||
        !aligned16(dLeafTris))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    if (maxDepth < 0) return fail(MLBVH_ERR_INVALID_ARG, "maxDepth must be >= 0");
    if (traversal != MLBVH_TRAVERSAL_STACKFREE && traversal != MLBVH_TRAVERSAL_REPLAY)
        return fail(MLBVH_ERR_INVALID_ARG, "PT traversal must be MLBVH_TRAVERSAL_STACKFREE or MLBVH_TRAVERSAL_REPLAY");
    float4* acc = reinterpret_cast<float4*>(dAccum);
    const float* tris = reinterpret_cast<const float*>(dTris);
    const float* at = reinterpret_cast<const float*>(dAttribs);
    const dim3 grid((unsigned)((w + kPtTileW - 1) / kPtTileW), (unsigned)((h + kPtTileH - 1) / kPtTileH));
    if (traversal == MLBVH_TRAVERSAL_REPLAY && dLeafTris)
        k_pt<<<grid, kPtThreads, 0, stream>>>(acc, cam, w, h, PlainReplayLeafTree{dNodes, tris, dRoot, dLeafTris},
                                                   at, useSobol, maxSPP, maxDepth);
    else if (traversal == MLBVH_TRAVERSAL_REPLAY)
        k_pt<<<grid, kPtThreads, 0, stream>>>(acc, cam, w, h, PlainReplayTree{dNodes, tris, dRoot, nullptr}, at,
                                                   useSobol, maxSPP, maxDepth);
    else
        k_pt<<<grid, kPtThreads, 0, stream>>>(acc, cam, w, h, PlainTree{dNodes, tris, dRoot, nullptr}, at,
                                                   useSobol, maxSPP, maxDepth);
    MLBVH_CHECK_LAUNCH("k_pt");
    return MLBVH_OK;
}

mlbvh_status pack(uint32_t* dPixels, const float* dAccum, int n, cudaStream_t stream)
{
    if (n <= 0) return n == 0 ? MLBVH_OK : fail(MLBVH_ERR_INVALID_ARG, "negative pixel count");
    if (!dPixels || !dAccum) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(dPixels) || !aligned16(dAccum))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    k_pack<<<(n + 255) / 256, 256, 0, stream>>>(dPixels, reinterpret_cast<const float4*>(dAccum), n);
    MLBVH_CHECK_LAUNCH("k_pack");
    return MLBVH_OK;
}

}  // namespace mlbvh
