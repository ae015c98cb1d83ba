/* Test infrastructure only — the oracle (checker) for the MinimumLBVH hot path.
 *
 * Plain-C restatement of the reference's CPU algorithm. Each function cites
 * the reference file:line it follows. Compiled with -ffp-contract=off so that
 * every float expression rounds exactly as the reference's host build does
 * (one rounding per written operation, in source order). See mlbvh_oracle.h.
 */
#define _GNU_SOURCE
#include "mlbvh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_FLT_MAX 3.402823466e+38F /* minimum_lbvh.h:37 */
#define ORC_MORTON_MAX 0x1FFFFF      /* minimum_lbvh.h:38 */
#define ORC_INVALID 0x7FFFFFFFu      /* NodeIndex::invalid(), minimum_lbvh.h:261-264 */
#define ORC_LEAF_BIT 0x80000000u

int orc_version(void) { return 1; }

/* ------------------------------------------------------------------ threads */
static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static int orc_threads(void)
{
    if (g_threads > 0) return g_threads;
    const char* env = getenv("MLBVH_ORACLE_THREADS");
    if (env && atoi(env) > 0) return atoi(env);
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

typedef void (*orc_range_fn)(void* ctx, uint32_t begin, uint32_t end);
typedef struct {
    orc_range_fn fn;
    void* ctx;
    uint32_t n, chunk;
    uint32_t next; /* atomic */
} orc_pool_job;

static void* orc_worker(void* p)
{
    orc_pool_job* job = (orc_pool_job*)p;
    for (;;)
    {
        uint32_t b = __atomic_fetch_add(&job->next, job->chunk, __ATOMIC_RELAXED);
        if (b >= job->n) break;
        uint32_t e = b + job->chunk < job->n ? b + job->chunk : job->n;
        job->fn(job->ctx, b, e);
    }
    return NULL;
}

static void orc_parallel_for(uint32_t n, uint32_t chunk, orc_range_fn fn, void* ctx)
{
    int nt = orc_threads();
    if (n == 0) return;
    if (nt <= 1 || n <= chunk)
    {
        fn(ctx, 0, n);
        return;
    }
    orc_pool_job job = {fn, ctx, n, chunk, 0};
    pthread_t th[256];
    if (nt > 256) nt = 256;
    int started = 0;
    for (int i = 1; i < nt; ++i)
        if (pthread_create(&th[started], NULL, orc_worker, &job) == 0) started++;
    orc_worker(&job);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
}

/* --------------------------------------------------------------- float math
 * helper_math.h host semantics: fminf/fmaxf are selects (helper_math.h:134-142),
 * rsqrtf is 1/sqrtf (:154-157), normalize is v * rsqrtf(dot(v, v)) (:1437). */
static inline float smin(float a, float b) { return a < b ? a : b; }
static inline float smax(float a, float b) { return a > b ? a : b; }
static inline orc_f3 f3(float x, float y, float z) { orc_f3 r = {x, y, z}; return r; }
static inline orc_f3 add3(orc_f3 a, orc_f3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline orc_f3 sub3(orc_f3 a, orc_f3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline orc_f3 mul3(orc_f3 a, orc_f3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline orc_f3 muls(orc_f3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
static inline orc_f3 smul(float s, orc_f3 a) { return f3(s * a.x, s * a.y, s * a.z); }
static inline orc_f3 divs(orc_f3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
static inline orc_f3 div3(orc_f3 a, orc_f3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline orc_f3 neg3(orc_f3 a) { return f3(-a.x, -a.y, -a.z); }
static inline orc_f3 min3(orc_f3 a, orc_f3 b) { return f3(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
static inline orc_f3 max3(orc_f3 a, orc_f3 b) { return f3(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }
static inline float dot3(orc_f3 a, orc_f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline orc_f3 cross3(orc_f3 a, orc_f3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline orc_f3 normalize3(orc_f3 v)
{
    float invLen = 1.0f / sqrtf(dot3(v, v));
    return muls(v, invLen);
}
/* helper_math.h:1266 lerp(a, b, t) = a + t*(b-a) */
static inline orc_f3 lerp3(orc_f3 a, orc_f3 b, float t) { return add3(a, smul(t, sub3(b, a))); }
static inline float compMin(orc_f3 v) { return smin(smin(v.x, v.y), v.z); } /* minimum_lbvh.h:73 */
static inline float compMax(orc_f3 v) { return smax(smax(v.x, v.y), v.z); } /* minimum_lbvh.h:77 */
static inline float clampf(float f, float a, float b) { return smax(a, smin(f, b)); } /* helper_math.h:1280 */
static inline int clampi(int f, int a, int b)
{
    int m = f < b ? f : b;
    return a > m ? a : m;
}
/* float -> int conversion as x86 cvttss2si does it (the reference's host
 * build): truncation, and 0x80000000 for NaN or out-of-range values. */
static inline int f2i_x86(float x)
{
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return (int)0x80000000u;
    return (int)x;
}

/* -------------------------------------------------------- bits and Morton */
int orc_clz(uint32_t x) { return x ? __builtin_clz(x) : 32; }          /* minimum_lbvh.h:99 */
int orc_clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }      /* minimum_lbvh.h:107 */
int orc_ffs(uint32_t x) { return x ? __builtin_ctz(x) + 1 : 0; }       /* minimum_lbvh.h:117 */
int orc_ffs64(uint64_t x) { return x ? __builtin_ctzll(x) + 1 : 0; }   /* minimum_lbvh.h:128 */
int orc_delta(uint32_t a, uint32_t b) { return 32 - orc_clz(a ^ b); } /* minimum_lbvh.h:140 */

/* minimum_lbvh.h:149-160: bit i of x, y, z lands at bit 3i, 3i+1, 3i+2. */
uint64_t orc_encode_morton_naive(uint32_t x, uint32_t y, uint32_t z)
{
    uint64_t code = 0;
    for (uint64_t i = 0; i < 64 / 3; ++i)
    {
        code |= ((uint64_t)(x & (1u << i)) << (2 * i + 0)) |
                ((uint64_t)(y & (1u << i)) << (2 * i + 1)) |
                ((uint64_t)(z & (1u << i)) << (2 * i + 2));
    }
    return code;
}

/* minimum_lbvh.h:173-182: spreads the low 21 bits of a three apart by
 * successive shift-or-mask steps (the usual magic-number dilation). */
uint64_t orc_splat3(uint32_t a)
{
    uint64_t x = a & 0x1fffffu;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

/* minimum_lbvh.h:162-171: the inverse of splat3. */
uint32_t orc_compact3(uint64_t m)
{
    uint64_t x = m & 0x1249249249249249ull;
    x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
    x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
    x = (x ^ (x >> 8)) & 0x001f0000ff0000ffull;
    x = (x ^ (x >> 16)) & 0x001f00000000ffffull;
    x = (x ^ (x >> 32)) & 0x1fffffull;
    return (uint32_t)x;
}

uint64_t orc_encode_morton(uint32_t x, uint32_t y, uint32_t z) /* minimum_lbvh.h:190 */
{
    return orc_splat3(x) | orc_splat3(y) << 1 | orc_splat3(z) << 2;
}

void orc_decode_morton(uint64_t m, uint32_t* x, uint32_t* y, uint32_t* z) /* :184 */
{
    *x = orc_compact3(m);
    *y = orc_compact3(m >> 1);
    *z = orc_compact3(m >> 2);
}

/* AABB::encodeMortonCode (minimum_lbvh.h:246-251): quantise
 * (p - lower) / (upper - lower) * 2^21, truncate, clamp to [0, 2^21 - 1]. */
uint64_t orc_aabb_morton(const orc_aabb* box, orc_f3 p)
{
    orc_f3 q = muls(div3(sub3(p, box->lower), sub3(box->upper, box->lower)), (float)(ORC_MORTON_MAX + 1));
    int cx = clampi(f2i_x86(q.x), 0, ORC_MORTON_MAX);
    int cy = clampi(f2i_x86(q.y), 0, ORC_MORTON_MAX);
    int cz = clampi(f2i_x86(q.z), 0, ORC_MORTON_MAX);
    return orc_encode_morton((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}

/* ------------------------------------------------------------------ build */
static void aabb_set_empty(orc_aabb* b) /* minimum_lbvh.h:229-233 */
{
    b->lower = f3(ORC_FLT_MAX, ORC_FLT_MAX, ORC_FLT_MAX);
    b->upper = f3(-ORC_FLT_MAX, -ORC_FLT_MAX, -ORC_FLT_MAX);
}
static void aabb_extend_p(orc_aabb* b, orc_f3 p) /* :234-238 */
{
    b->lower = min3(b->lower, p);
    b->upper = max3(b->upper, p);
}
static void aabb_extend_b(orc_aabb* b, const orc_aabb* o) /* :240-244 */
{
    b->lower = min3(b->lower, o->lower);
    b->upper = max3(b->upper, o->upper);
}

/* BVHCPUBuilder::build scene-AABB loop (minimum_lbvh.h:522-532). */
void orc_scene_aabb(const orc_triangle* tris, uint32_t n, orc_aabb* out)
{
    orc_aabb s;
    aabb_set_empty(&s);
    for (uint32_t i = 0; i < n; i++)
        for (int j = 0; j < 3; ++j) aabb_extend_p(&s, tris[i].v[j]);
    *out = s;
}

/* Morton keys (minimum_lbvh.h:534-553; device twin minimum_lbvh.cu:68-92):
 * centroid (v0 + v1 + v2) / 3, top 32 of the 63-bit code; with
 * BUILD_OPTION_USE_NORMAL the low 6 bits are the normal's code. */
void orc_morton_keys(const orc_triangle* tris, uint32_t n, uint32_t option,
                     const orc_aabb* scene, uint32_t* keys)
{
    for (uint32_t i = 0; i < n; i++)
    {
        orc_triangle tri = tris[i];
        orc_f3 center = divs(add3(add3(tri.v[0], tri.v[1]), tri.v[2]), 3.0f);
        if (option & 1u)
        {
            orc_f3 ng = normalize3(cross3(sub3(tri.v[1], tri.v[0]), sub3(tri.v[2], tri.v[0])));
            orc_aabb unit = {{-1, -1, -1}, {+1, +1, +1}};
            uint32_t nMorton = (uint32_t)(orc_aabb_morton(&unit, ng) >> 31);
            uint32_t pMorton = (uint32_t)(orc_aabb_morton(scene, center) >> 31);
            keys[i] = (pMorton & 0xFFFFFFC0u) | (nMorton >> 26);
        }
        else
        {
            keys[i] = (uint32_t)(orc_aabb_morton(scene, center) >> 31);
        }
    }
}

/* Stable sort of (key, value) pairs by key: a four-pass LSD counting sort,
 * i.e. the (morton, original index) order a stable sort of the reference's
 * IndexedMorton array gives (minimum_lbvh.h:554 sorts with std::sort; the
 * reference GPU path sorts the same array with a stable LSD radix sort,
 * minimum_lbvh.h:833). */
void orc_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n)
{
    uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* v2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *ks = keys, *vs = values, *kd = k2, *vd = v2;
    for (int pass = 0; pass < 4; ++pass)
    {
        uint32_t count[257];
        memset(count, 0, sizeof(count));
        int shift = pass * 8;
        for (uint32_t i = 0; i < n; ++i) count[((ks[i] >> shift) & 255u) + 1]++;
        for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
        for (uint32_t i = 0; i < n; ++i)
        {
            uint32_t d = (ks[i] >> shift) & 255u;
            uint32_t o = count[d]++;
            kd[o] = ks[i];
            vd[o] = vs[i];
        }
        uint32_t* t = ks; ks = kd; kd = t;
        t = vs; vs = vd; vd = t;
    }
    /* four passes: the result is back in the caller's arrays */
    free(k2);
    free(v2);
}

/* build_lbvh (minimum_lbvh.h:284-361): one walker per sorted leaf climbs
 * bottom-up; at each step the parent is the internal node on the side with the
 * smaller neighbouring delta (internal node i splits leaves i and i+1); the
 * first walker to reach a parent leaves its range bound in `context` and stops,
 * the second merges ranges and bounds and continues. Serial here: the result
 * is the same for any walker order. */
static void build_walk(uint32_t* rootNode, orc_node* internals, const orc_triangle* triangles,
                       uint32_t nTriangles, const uint8_t* deltas, uint32_t i_leaf, uint32_t triangleIndex)
{
    uint32_t nInternals = nTriangles - 1;
    uint32_t nDeltas = nInternals;
    uint32_t leaf_lower = i_leaf, leaf_upper = i_leaf;
    uint32_t node = triangleIndex | ORC_LEAF_BIT;

    orc_aabb aabb;
    aabb_set_empty(&aabb);
    if (triangles)
        for (int j = 0; j < 3; ++j) aabb_extend_p(&aabb, triangles[triangleIndex].v[j]);

    int isRoot = 1;
    while (leaf_upper - leaf_lower < nInternals)
    {
        uint32_t deltaL = 0 < leaf_lower ? deltas[leaf_lower - 1] : 0xFFFFFFFFu;
        uint32_t deltaR = leaf_upper < nDeltas ? deltas[leaf_upper] : 0xFFFFFFFFu;
        int goLeft = deltaL < deltaR ? 1 : 0;
        uint32_t parent = goLeft ? (leaf_lower - 1) : leaf_upper;

        internals[parent].children[goLeft] = node;
        internals[parent].aabbs[goLeft] = aabb;
        if (!(node & ORC_LEAF_BIT)) internals[node].parent = parent;

        uint32_t index = goLeft ? leaf_upper : leaf_lower;
        uint32_t old = internals[parent].context; /* the exchange (:330-336) */
        internals[parent].context = index;
        index = old;
        if (index == 0xFFFFFFFFu)
        {
            isRoot = 0;
            break;
        }
        leaf_lower = leaf_lower < index ? leaf_lower : index;
        leaf_upper = leaf_upper < index ? index : leaf_upper;
        internals[parent].context = leaf_upper < nInternals ? leaf_upper : 0xFFFFFFFFu;
        node = parent;
        orc_aabb other = internals[parent].aabbs[goLeft ^ 1];
        aabb_extend_b(&aabb, &other);
    }
    if (isRoot)
    {
        *rootNode = node;
        if (!(node & ORC_LEAF_BIT)) internals[node].parent = ORC_INVALID;
    }
}

int orc_build_from_keys(const uint32_t* sorted_keys, const uint32_t* sorted_indices,
                        const orc_triangle* tris, uint32_t n,
                        orc_node* nodes, uint8_t* deltas, uint32_t* root)
{
    if (n == 0) return -1;
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        memset(&nodes[i], 0, sizeof(orc_node));
        nodes[i].context = 0xFFFFFFFFu; /* minimum_lbvh.h:514-519 */
        deltas[i] = (uint8_t)orc_delta(sorted_keys[i], sorted_keys[i + 1]); /* :556-561 */
    }
    for (uint32_t i = 0; i < n; ++i)
        build_walk(root, nodes, tris, n, deltas, i, sorted_indices[i]);
    return 0;
}

/* BVHCPUBuilder::build (minimum_lbvh.h:512-592) with the stable key order. */
int orc_build(const orc_triangle* tris, uint32_t n, uint32_t option,
              orc_node* nodes, uint8_t* deltas, uint32_t* root,
              uint32_t* keys_out, uint32_t* indices_out, orc_aabb* scene_out)
{
    if (n == 0) return -1;
    orc_aabb scene;
    orc_scene_aabb(tris, n, &scene);
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * n);
    orc_morton_keys(tris, n, option, &scene, keys);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    orc_sort_pairs(keys, idx, n);
    int rc = orc_build_from_keys(keys, idx, tris, n, nodes, deltas, root);
    if (keys_out) memcpy(keys_out, keys, sizeof(uint32_t) * n);
    if (indices_out) memcpy(indices_out, idx, sizeof(uint32_t) * n);
    if (scene_out) *scene_out = scene;
    free(keys);
    free(idx);
    return rc;
}

/* ------------------------------------------------------------ PLOC build
 * The higher-quality builder. The reference's is Embree's SAH build
 * (BVHCPUBuilder::buildByEmbree, minimum_lbvh.h:594-656: one triangle per
 * leaf, binary nodes written into the same InternalNode array, root parent
 * invalid); Embree is a binary-only dependency. This is the published
 * parallel locally-ordered clustering (Meister and Bittner, "Parallel
 * Locally-Ordered Clustering for Bounding Volume Hierarchy Construction",
 * 2018) restated over the stable Morton order of orc_build:
 *   - clusters start as the leaves in sorted order;
 *   - each cluster's nearest neighbour is sought among the `radius` clusters
 *     on either side by the half surface area of the union box (the union by
 *     fminf / fmaxf, which ignore a NaN operand; area dx*dy + dy*dz + dz*dx;
 *     the order key is the bit pattern of min(|area|, +inf), so a zero area
 *     of either sign is 0 and a NaN area counts as +inf); ties go to the
 *     smaller position. That is a strict order on pairs, so the closest pair
 *     overall is always mutual and every iteration merges at least once. Once
 *     an iteration has removed fewer than 1/64 of the clusters, every later
 *     iteration breaks exact ties first by the smaller ploc_pair_hash of the
 *     pair's two positions (still a strict order): where all union areas are
 *     equal (duplicated or collinear triangles) ties to the smaller position
 *     merge only the first pair of a run per iteration, the hash about a
 *     quarter of the clusters. If an iteration that already breaks ties by
 *     the hash still removes fewer than 1/64 of the clusters (a chain of
 *     strictly growing gaps, where every cluster's nearest neighbour is the
 *     one before it), the next iteration pairs positions 2k and 2k + 1
 *     outright, halving the count; so every build ends in O(log n)
 *     iterations;
 *   - mutual nearest neighbours merge into the lower position, all other
 *     clusters stay, and the survivors keep their order.
 * Nodes are then numbered in in-order (node j between the j-th and the
 * (j+1)-th leaf of a left-to-right walk), as build_lbvh's are, so the
 * leaf-order conventions of the other walks hold; context is the in-order
 * index of the subtree's last leaf when below n - 1, else ~0 (the escape
 * index intersect_escape_link reads, minimum_lbvh.h:1090-1122). */
static uint32_t ploc_area_key(const orc_aabb* a0, const orc_aabb* a1)
{
    float lx = fminf(a0->lower.x, a1->lower.x), ly = fminf(a0->lower.y, a1->lower.y);
    float lz = fminf(a0->lower.z, a1->lower.z);
    float hx = fmaxf(a0->upper.x, a1->upper.x), hy = fmaxf(a0->upper.y, a1->upper.y);
    float hz = fmaxf(a0->upper.z, a1->upper.z);
    float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    float a = fminf(fabsf(dx * dy + dy * dz + dz * dx), INFINITY);
    uint32_t k;
    memcpy(&k, &a, 4);
    return k;
}

/* A symmetric mix of the two positions of a pair (integer hashing in the
 * style of MurmurHash3's finaliser). */
static uint32_t ploc_pair_hash(uint32_t a, uint32_t b)
{
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    uint32_t h = lo * 0x9E3779B1u ^ hi * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}

typedef struct {
    uint32_t id[2];
    orc_aabb box[2];
    uint32_t cnt[2];
} ploc_node;

int orc_build_ploc(const orc_triangle* tris, uint32_t n, uint32_t option, int radius, orc_node* nodes,
                   uint32_t* root)
{
    if (n == 0 || radius < 1) return -1;
    orc_aabb scene;
    orc_scene_aabb(tris, n, &scene);
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * n);
    orc_morton_keys(tris, n, option, &scene, keys);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    orc_sort_pairs(keys, idx, n);
    free(keys);
    if (n == 1)
    {
        *root = ORC_LEAF_BIT | idx[0];
        free(idx);
        return 0;
    }
    orc_aabb* box[2] = {(orc_aabb*)malloc(sizeof(orc_aabb) * n), (orc_aabb*)malloc(sizeof(orc_aabb) * n)};
    uint32_t* id[2] = {(uint32_t*)malloc(4ull * n), (uint32_t*)malloc(4ull * n)};
    uint32_t* cnt[2] = {(uint32_t*)malloc(4ull * n), (uint32_t*)malloc(4ull * n)};
    uint32_t* nn = (uint32_t*)malloc(4ull * n);
    ploc_node* tmp = (ploc_node*)malloc(sizeof(ploc_node) * (n - 1));
    for (uint32_t i = 0; i < n; ++i)
    {
        aabb_set_empty(&box[0][i]);
        for (int j = 0; j < 3; ++j) aabb_extend_p(&box[0][i], tris[idx[i]].v[j]);
        id[0][i] = ORC_LEAF_BIT | idx[i];
        cnt[0][i] = 1;
    }
    free(idx);
    uint32_t C = n, created = 0;
    int cur = 0, iterations = 0, hashTies = 0, pairNext = 0;
    const uint32_t r = (uint32_t)radius;
    while (C > 1)
    {
        const orc_aabb* b = box[cur];
        const int pairs = pairNext;
        for (uint32_t p = 0; p < C && pairs; ++p)  /* position 2k with 2k + 1; an odd last one stays */
            nn[p] = (p ^ 1u) < C ? p ^ 1u : (p > 0 ? p - 1 : p);
        for (uint32_t p = 0; p < C && !pairs; ++p)
        {
            uint32_t bestA = 0xFFFFFFFFu, bestJ = 0;
            uint32_t lo = p > r ? p - r : 0, hi = p + r < C - 1 ? p + r : C - 1;
            for (uint32_t j = lo; j <= hi; ++j)
            {
                if (j == p) continue;
                uint32_t a = ploc_area_key(&b[p], &b[j]);
                if (a < bestA || (a == bestA && hashTies && ploc_pair_hash(p, j) < ploc_pair_hash(p, bestJ)))
                {
                    bestA = a;
                    bestJ = j;
                }
            }
            nn[p] = bestJ;
        }
        uint32_t w = 0;
        for (uint32_t p = 0; p < C; ++p)
        {
            uint32_t j = nn[p];
            int mutual = nn[j] == p;
            if (mutual && j < p) continue;
            if (mutual)
            {
                ploc_node* t = &tmp[created];
                t->id[0] = id[cur][p];
                t->id[1] = id[cur][j];
                t->box[0] = b[p];
                t->box[1] = b[j];
                t->cnt[0] = cnt[cur][p];
                t->cnt[1] = cnt[cur][j];
                box[cur ^ 1][w].lower = min3(b[p].lower, b[j].lower);
                box[cur ^ 1][w].upper = max3(b[p].upper, b[j].upper);
                id[cur ^ 1][w] = created++;
                cnt[cur ^ 1][w] = cnt[cur][p] + cnt[cur][j];
            }
            else
            {
                box[cur ^ 1][w] = b[p];
                id[cur ^ 1][w] = id[cur][p];
                cnt[cur ^ 1][w] = cnt[cur][p];
            }
            ++w;
        }
        if ((uint64_t)(C - w) * 64 < C)
        {
            if (hashTies) pairNext = 1;
            hashTies = 1;
        }
        else
            pairNext = 0;
        C = w;
        cur ^= 1;
        ++iterations;
    }
    /* in-order numbering, parents before children (creation order reversed) */
    uint32_t* off = (uint32_t*)malloc(4ull * (n - 1));
    uint32_t* par = (uint32_t*)malloc(4ull * (n - 1));
    off[created - 1] = 0;
    par[created - 1] = ORC_INVALID;
    for (uint32_t m = created; m-- > 0;)
    {
        const ploc_node* t = &tmp[m];
        uint32_t rank = off[m] + t->cnt[0] - 1;
        uint32_t last = off[m] + t->cnt[0] + t->cnt[1] - 1;
        orc_node* o = &nodes[rank];
        for (int c = 0; c < 2; ++c)
        {
            uint32_t ch = t->id[c];
            uint32_t co = c == 0 ? off[m] : off[m] + t->cnt[0];
            if (ch & ORC_LEAF_BIT)
                o->children[c] = ch;
            else
            {
                o->children[c] = co + tmp[ch].cnt[0] - 1;
                off[ch] = co;
                par[ch] = rank;
            }
            o->aabbs[c] = t->box[c];
        }
        o->parent = par[m];
        o->context = last < n - 1 ? last : 0xFFFFFFFFu;
        if (par[m] == ORC_INVALID) *root = rank;
    }
    free(off);
    free(par);
    for (int k = 0; k < 2; ++k)
    {
        free(box[k]);
        free(id[k]);
        free(cnt[k]);
    }
    free(nn);
    free(tmp);
    return iterations;
}

static double half_area(const orc_aabb* b)
{
    double dx = (double)b->upper.x - b->lower.x, dy = (double)b->upper.y - b->lower.y,
           dz = (double)b->upper.z - b->lower.z;
    return dx * dy + dy * dz + dz * dx;
}

double orc_sah_cost(const orc_node* nodes, uint32_t n, uint32_t root)
{
    if (n < 2) return 1.0;
    orc_aabb rb;
    rb.lower = min3(nodes[root].aabbs[0].lower, nodes[root].aabbs[1].lower);
    rb.upper = max3(nodes[root].aabbs[0].upper, nodes[root].aabbs[1].upper);
    double sum = 0.0;
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        const orc_aabb* b = nodes[i].aabbs;
        orc_aabb u;
        u.lower = min3(b[0].lower, b[1].lower);
        u.upper = max3(b[0].upper, b[1].upper);
        sum += half_area(&u);
        for (int c = 0; c < 2; ++c)
            if (nodes[i].children[c] & ORC_LEAF_BIT) sum += half_area(&b[c]);
    }
    return sum / half_area(&rb);
}

/* validate_lbvh (minimum_lbvh.h:415-426), iterative; returns 1 when every
 * child's split delta is <= its parent's. */
int orc_validate(const orc_node* nodes, const uint8_t* deltas, uint32_t n, uint32_t root, int maxDelta)
{
    if (n <= 1) return 1;
    uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * 2 * n);
    int* limit = (int*)malloc(sizeof(int) * 2 * n);
    size_t sp = 0;
    int ok = 1;
    stack[sp] = root;
    limit[sp++] = maxDelta;
    while (sp && ok)
    {
        --sp;
        uint32_t node = stack[sp];
        int lim = limit[sp];
        if (node & ORC_LEAF_BIT) continue;
        if (node >= n - 1) { ok = 0; break; }
        int d = deltas[node];
        if (d > lim) { ok = 0; break; }
        for (int c = 0; c < 2; ++c)
        {
            stack[sp] = nodes[node].children[c];
            limit[sp++] = d;
        }
    }
    free(stack);
    free(limit);
    return ok;
}

/* Structural check: every leaf reached exactly once from the root, parent
 * links consistent, each child's box inside its parent's, leaf boxes equal to
 * their triangle's bounds. Returns 1 when all hold. */
int orc_check_tree(const orc_node* nodes, const orc_triangle* tris, uint32_t n, uint32_t root)
{
    if (n == 1) return root == ORC_LEAF_BIT;
    uint8_t* seen = (uint8_t*)calloc(n, 1);
    uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * n);
    size_t sp = 0;
    int ok = (root & ORC_LEAF_BIT) == 0 && root < n - 1 && nodes[root].parent == ORC_INVALID;
    uint32_t visited = 0;
    if (ok) stack[sp++] = root;
    while (sp && ok)
    {
        uint32_t node = stack[--sp];
        visited++;
        for (int c = 0; c < 2 && ok; ++c)
        {
            uint32_t ch = nodes[node].children[c];
            const orc_aabb* b = &nodes[node].aabbs[c];
            if (ch & ORC_LEAF_BIT)
            {
                uint32_t t = ch & ~ORC_LEAF_BIT;
                if (t >= n || seen[t]) { ok = 0; break; }
                seen[t] = 1;
                orc_aabb tb;
                aabb_set_empty(&tb);
                for (int j = 0; j < 3; ++j) aabb_extend_p(&tb, tris[t].v[j]);
                if (memcmp(&tb, b, sizeof(tb)) != 0) ok = 0;
            }
            else
            {
                if (ch >= n - 1 || nodes[ch].parent != node) { ok = 0; break; }
                const orc_aabb* cb = &nodes[ch].aabbs[0];
                const orc_aabb* cb1 = &nodes[ch].aabbs[1];
                if (cb->lower.x < b->lower.x || cb->lower.y < b->lower.y || cb->lower.z < b->lower.z ||
                    cb->upper.x > b->upper.x || cb->upper.y > b->upper.y || cb->upper.z > b->upper.z ||
                    cb1->lower.x < b->lower.x || cb1->lower.y < b->lower.y || cb1->lower.z < b->lower.z ||
                    cb1->upper.x > b->upper.x || cb1->upper.y > b->upper.y || cb1->upper.z > b->upper.z)
                    ok = 0;
                stack[sp++] = ch;
            }
        }
    }
    for (uint32_t i = 0; i < n && ok; ++i)
        if (!seen[i]) ok = 0;
    if (ok && visited != n - 1) ok = 0;
    free(seen);
    free(stack);
    return ok;
}

/* ---------------------------------------------------------------- queries */
/* slabs (minimum_lbvh.h:82-96): entry/exit of the ray against one box, the
 * exit inflated by 1.00000024 (robust traversal), clipped to [0, knownHitT]. */
static inline void slabs(orc_f3 ro, orc_f3 inv, const orc_aabb* b, float knownHitT, float* rmin, float* rmax)
{
    orc_f3 t0 = mul3(sub3(b->lower, ro), inv);
    orc_f3 t1 = mul3(sub3(b->upper, ro), inv);
    orc_f3 tmin = min3(t0, t1);
    orc_f3 tmax = max3(t0, t1);
    float region_min = compMax(tmin);
    float region_max = compMin(tmax) * 1.00000024f;
    region_min = smax(region_min, 0.0f);
    region_max = smin(region_max, knownHitT);
    *rmin = region_min;
    *rmax = region_max;
}

/* intersectRayTriangle (minimum_lbvh.h:363-413). */
static inline int intersect_tri(float* tOut, float* uOut, float* vOut, orc_f3* ngOut, float t_min, float t_max,
                                orc_f3 ro, orc_f3 rd, orc_f3 v0, orc_f3 v1, orc_f3 v2)
{
    orc_f3 e0 = sub3(v1, v0);
    orc_f3 e1 = sub3(v2, v1);
    orc_f3 ng = cross3(e0, e1);
    float t = dot3(sub3(v0, ro), ng) / dot3(ng, rd);
    if (t_min <= t && t <= t_max)
    {
        orc_f3 e2 = sub3(v0, v2);
        orc_f3 ro2 = muls(ro, 2.0f);
        float u_vol = dot3(cross3(e2, sub3(add3(v0, v2), ro2)), rd);
        float v_vol = dot3(cross3(e0, sub3(add3(v1, v0), ro2)), rd);
        float w_vol = dot3(cross3(e1, sub3(add3(v2, v1), ro2)), rd);
        if (smin(smin(u_vol, v_vol), w_vol) < 0.0f && 0.0f < smax(smax(u_vol, v_vol), w_vol)) return 0;
        float vol = u_vol + v_vol + w_vol;
        *tOut = t;
        *uOut = u_vol / vol;
        *vOut = v_vol / vol;
        *ngOut = ng;
        return 1;
    }
    return 0;
}

/* invRd (minimum_lbvh.h:898-901) */
static inline orc_f3 inv_rd(orc_f3 rd)
{
    orc_f3 r = f3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    return f3(clampf(r.x, -ORC_FLT_MAX, ORC_FLT_MAX), clampf(r.y, -ORC_FLT_MAX, ORC_FLT_MAX),
              clampf(r.z, -ORC_FLT_MAX, ORC_FLT_MAX));
}

static inline int is_leaf(uint32_t n) { return (n & ORC_LEAF_BIT) != 0; }
static inline uint32_t idx_of(uint32_t n) { return n & ~ORC_LEAF_BIT; }

static inline void leaf_test(orc_hit* hit, const orc_triangle* tris, uint32_t leaf, orc_f3 ro, orc_f3 rd,
                             float tmin, int* hitOut, uint32_t* triTests)
{
    float t, u, v;
    orc_f3 ng;
    const orc_triangle* tri = &tris[idx_of(leaf)];
    (*triTests)++;
    *hitOut = 0;
    if (intersect_tri(&t, &u, &v, &ng, tmin, hit->t, ro, rd, tri->v[0], tri->v[1], tri->v[2]))
    {
        hit->t = t;
        hit->u = u;
        hit->v = v;
        hit->triangleIndex = idx_of(leaf);
        hit->ng = ng;
        *hitOut = 1;
    }
}

/* intersect_stackfree (minimum_lbvh.h:981-1061): parent-pointer traversal.
 * Coming from the parent, go to the near hit child (entry order, ties to the
 * left) or back up; coming from the near child, go to the far child if both
 * boxes are still hit, else up; coming from the far child, go up. */
static void stackfree_walk(orc_hit* hit, const orc_node* nodes, const orc_triangle* tris, uint32_t curr,
                           uint32_t prev, orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, int anyHit,
                           uint32_t* nodeVisits, uint32_t* triTests)
{
    while (curr != ORC_INVALID)
    {
        if (is_leaf(curr))
        {
            int h;
            leaf_test(hit, tris, curr, ro, rd, tmin, &h, triTests);
            if (h && anyHit) break;
            uint32_t t = curr; curr = prev; prev = t;
            continue;
        }
        (*nodeVisits)++;
        const orc_node* nd = &nodes[curr];
        float lmin, lmax, rmin, rmax;
        slabs(ro, inv, &nd->aabbs[0], hit->t, &lmin, &lmax);
        slabs(ro, inv, &nd->aabbs[1], hit->t, &rmin, &rmax);
        lmin = smax(lmin, tmin);
        rmin = smax(rmin, tmin);
        int hitL = lmin <= lmax, hitR = rmin <= rmax;
        uint32_t parent = nd->parent, near = nd->children[0], far = nd->children[1];
        int nHits = 0;
        if (hitL && hitR)
        {
            if (rmin < lmin) { uint32_t t = near; near = far; far = t; }
            nHits = 2;
        }
        else if (hitL || hitR)
        {
            nHits = 1;
            near = hitR ? far : near;
        }
        uint32_t next;
        if (prev == parent) next = 0 < nHits ? near : parent;
        else if (prev == near) next = nHits == 2 ? far : parent;
        else next = parent;
        prev = curr;
        curr = next;
    }
}

static void trace_stackfree(orc_hit* hit, const orc_node* nodes, const orc_triangle* tris, uint32_t root,
                            orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, int anyHit,
                            uint32_t* nodeVisits, uint32_t* triTests)
{
    stackfree_walk(hit, nodes, tris, root, ORC_INVALID, ro, rd, inv, tmin, anyHit, nodeVisits, triTests);
}

/* stackfree_replay_step (include/mlbvh_device.cuh): intersect_stackfree's
 * leaf order and hit.t updates without its revisits. Where both child boxes
 * are hit, the far child and its entry distance are pushed and the near child
 * entered; when a subtree is done, entries are popped, and an entry is entered
 * iff its entry distance is still <= hit.t -- exactly when the stack-free
 * walk, back at the parent from the near child, finds both boxes still hit
 * (an entry distance does not depend on hit.t, and the near entry never
 * exceeds the far one). A push onto a full stack (depth entries) hands over
 * to the stack-free walk at (near child, this node). */
static void trace_replay(orc_hit* hit, const orc_node* nodes, const orc_triangle* tris, uint32_t root, orc_f3 ro,
                         orc_f3 rd, orc_f3 inv, float tmin, int anyHit, int depth, uint32_t* nodeVisits,
                         uint32_t* triTests)
{
    uint32_t stackNode[64];
    float stackEntry[64];
    int top = 0;
    uint32_t curr = root;
    for (;;)
    {
        int pop = 0;
        if (is_leaf(curr))
        {
            int h;
            leaf_test(hit, tris, curr, ro, rd, tmin, &h, triTests);
            if (h && anyHit) return;
            pop = 1;
        }
        else
        {
            (*nodeVisits)++;
            const orc_node* nd = &nodes[curr];
            float lmin, lmax, rmin, rmax;
            slabs(ro, inv, &nd->aabbs[0], hit->t, &lmin, &lmax);
            slabs(ro, inv, &nd->aabbs[1], hit->t, &rmin, &rmax);
            lmin = smax(lmin, tmin);
            rmin = smax(rmin, tmin);
            int hitL = lmin <= lmax, hitR = rmin <= rmax;
            if (hitL && hitR)
            {
                uint32_t nearN = nd->children[0], farN = nd->children[1];
                float farEntry = rmin;
                if (rmin < lmin) { nearN = nd->children[1]; farN = nd->children[0]; farEntry = lmin; }
                if (top == depth)
                {
                    stackfree_walk(hit, nodes, tris, nearN, curr, ro, rd, inv, tmin, anyHit, nodeVisits, triTests);
                    return;
                }
                stackNode[top] = farN;
                stackEntry[top] = farEntry;
                ++top;
                curr = nearN;
            }
            else if (hitL || hitR)
                curr = nd->children[hitL ? 0 : 1];
            else
                pop = 1;
        }
        if (pop)
        {
            for (;;)
            {
                if (top == 0) return;
                --top;
                if (stackEntry[top] <= hit->t) { curr = stackNode[top]; break; }
            }
        }
    }
}

/* intersect_escape_link (minimum_lbvh.h:1063-1137): ropes through `context`
 * (the index of the node covering the next leaf range). The reference reads
 * nodes[prev] at a leaf; a leaf root (one triangle) is tested directly here. */
static void trace_escape(orc_hit* hit, const orc_node* nodes, const orc_triangle* tris, uint32_t root,
                         orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, int anyHit,
                         uint32_t* nodeVisits, uint32_t* triTests)
{
    if (is_leaf(root))
    {
        int h;
        leaf_test(hit, tris, root, ro, rd, tmin, &h, triTests);
        return;
    }
    uint32_t curr = root, prev = ORC_INVALID;
    while (curr != ORC_INVALID)
    {
        if (is_leaf(curr))
        {
            int h;
            leaf_test(hit, tris, curr, ro, rd, tmin, &h, triTests);
            if (h && anyHit) break;
            if (nodes[idx_of(prev)].children[0] == curr)
            {
                uint32_t t = curr; curr = prev; prev = t;
                continue;
            }
            uint32_t ioi = nodes[idx_of(prev)].context;
            uint32_t next = ioi != 0xFFFFFFFFu ? ioi : ORC_INVALID;
            prev = curr;
            curr = next;
            continue;
        }
        (*nodeVisits)++;
        const orc_node* nd = &nodes[curr];
        uint32_t parent = nd->parent;
        const orc_aabb* box;
        uint32_t hitChild, miss;
        if (prev == parent)
        {
            box = &nd->aabbs[0];
            hitChild = nd->children[0];
            miss = curr;
        }
        else
        {
            box = &nd->aabbs[1];
            hitChild = nd->children[1];
            uint32_t ioi = nd->context;
            miss = ioi != 0xFFFFFFFFu ? ioi : ORC_INVALID;
        }
        float rmin, rmax;
        slabs(ro, inv, box, hit->t, &rmin, &rmax);
        rmin = smax(rmin, tmin);
        uint32_t next = rmin <= rmax ? hitChild : miss;
        prev = curr;
        curr = next;
    }
}

/* intersect_stackfull (minimum_lbvh.h:912-973): explicit stack, far child
 * pushed. Closest hit only, as in the reference. */
static void trace_stackfull(orc_hit* hit, const orc_node* nodes, const orc_triangle* tris, uint32_t root,
                            orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin,
                            uint32_t* nodeVisits, uint32_t* triTests)
{
    uint32_t stack[64];
    int sp = 0;
    uint32_t node = root;
    while (node != ORC_INVALID)
    {
        if (is_leaf(node))
        {
            int h;
            leaf_test(hit, tris, node, ro, rd, tmin, &h, triTests);
            node = sp == 0 ? ORC_INVALID : stack[--sp];
            continue;
        }
        (*nodeVisits)++;
        const orc_node* nd = &nodes[node];
        float lmin, lmax, rmin, rmax;
        slabs(ro, inv, &nd->aabbs[0], hit->t, &lmin, &lmax);
        slabs(ro, inv, &nd->aabbs[1], hit->t, &rmin, &rmax);
        lmin = smax(lmin, tmin);
        rmin = smax(rmin, tmin);
        int hitL = lmin <= lmax, hitR = rmin <= rmax;
        if (hitL && hitR)
        {
            uint32_t nearN = nd->children[0], farN = nd->children[1];
            if (rmin < lmin) { uint32_t t = nearN; nearN = farN; farN = t; }
            node = nearN;
            if (sp < 64) stack[sp++] = farN;
        }
        else if (hitL || hitR)
            node = nd->children[hitL ? 0 : 1];
        else
            node = sp == 0 ? ORC_INVALID : stack[--sp];
    }
}

static inline void hit_init(orc_hit* h, float tmax)
{
    memset(h, 0, sizeof(*h));
    h->t = tmax;
    h->triangleIndex = 0xFFFFFFFFu;
}

typedef struct {
    const orc_node* nodes;
    const orc_triangle* tris;
    uint32_t root;
    const orc_ray* rays;
    int query, mode;
    orc_hit* hits;
    uint32_t *nodeVisits, *triTests;
    int depth; /* stack entries of the replay walk (mode 3) */
} trace_ctx;

static void trace_range(void* p, uint32_t b, uint32_t e)
{
    trace_ctx* c = (trace_ctx*)p;
    for (uint32_t i = b; i < e; ++i)
    {
        const orc_ray* r = &c->rays[i];
        orc_f3 ro = f3(r->ro[0], r->ro[1], r->ro[2]);
        orc_f3 rd = f3(r->rd[0], r->rd[1], r->rd[2]);
        orc_hit hit;
        hit_init(&hit, r->tmax);
        uint32_t nv = 0, nt = 0;
        orc_f3 inv = inv_rd(rd);
        if (c->mode == 1)
            trace_escape(&hit, c->nodes, c->tris, c->root, ro, rd, inv, r->tmin, c->query == 1, &nv, &nt);
        else if (c->mode == 2)
            trace_stackfull(&hit, c->nodes, c->tris, c->root, ro, rd, inv, r->tmin, &nv, &nt);
        else if (c->mode == 3)
            trace_replay(&hit, c->nodes, c->tris, c->root, ro, rd, inv, r->tmin, c->query == 1, c->depth, &nv, &nt);
        else
            trace_stackfree(&hit, c->nodes, c->tris, c->root, ro, rd, inv, r->tmin, c->query == 1, &nv, &nt);
        c->hits[i] = hit;
        if (c->nodeVisits) c->nodeVisits[i] = nv;
        if (c->triTests) c->triTests[i] = nt;
    }
}

void orc_trace(const orc_node* nodes, const orc_triangle* tris, uint32_t root,
               const orc_ray* rays, uint32_t nRays, int query, int mode,
               orc_hit* hits, uint32_t* nodeVisits, uint32_t* triTests)
{
    trace_ctx c = {nodes, tris, root, rays, query, mode, hits, nodeVisits, triTests, 16};
    orc_parallel_for(nRays, 1024, trace_range, &c);
}

void orc_trace_replay(const orc_node* nodes, const orc_triangle* tris, uint32_t root, const orc_ray* rays,
                      uint32_t nRays, int query, int depth, orc_hit* hits, uint32_t* nodeVisits, uint32_t* triTests)
{
    trace_ctx c = {nodes, tris, root, rays, query, 3, hits, nodeVisits, triTests,
                   depth < 1 ? 1 : depth > 64 ? 64 : depth};
    orc_parallel_for(nRays, 1024, trace_range, &c);
}

/* ------------------------------------------------------- the 4-wide tree */
/* No reference counterpart: csrc/wide.cu (k_wide_collapse) and
 * wide_any_step (include/mlbvh_device.cuh). A wide node is 32 words: per
 * axis a, words 8a..8a+3 the lower and 8a+4..8a+7 the upper bounds of
 * children 0-3; words 24-27 the children (internal index, leaf position with
 * bit 31, or 0xFFFFFFFF for an empty slot); 28-31 zero. */
#define ORC_WIDE_EMPTY 0xFFFFFFFFu
#define ORC_WIDE_DEPTH 24

typedef struct {
    uint32_t name;
    orc_aabb box;
} wide_kid;

static float wide_area(const orc_aabb* b)
{
    float dx = b->upper.x - b->lower.x, dy = b->upper.y - b->lower.y, dz = b->upper.z - b->lower.z;
    float a = dx * dy;
    a = a + dy * dz;
    a = a + dz * dx;
    return a;
}

static wide_kid wide_child(const orc_node* nodes, uint32_t p, int side)
{
    wide_kid k;
    uint32_t c = nodes[p].children[side];
    k.name = is_leaf(c) ? (ORC_LEAF_BIT | (p + (uint32_t)side)) : c;
    k.box = nodes[p].aabbs[side];
    return k;
}

/* Slot i: binary node i's children; twice, the internal child of largest
 * area (ties: the lower slot) replaced by its two children in place. */
void orc_build_wide(const orc_node* nodes, uint32_t n, uint32_t* out)
{
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        wide_kid kid[4];
        int count = 2;
        kid[0] = wide_child(nodes, i, 0);
        kid[1] = wide_child(nodes, i, 1);
        for (int round = 0; round < 2; ++round)
        {
            int pick = -1;
            float best = 0.0f;
            for (int k = 0; k < count; ++k)
            {
                if (is_leaf(kid[k].name)) continue;
                float a = wide_area(&kid[k].box);
                if (pick < 0 || a > best) { pick = k; best = a; }
            }
            if (pick < 0) break;
            uint32_t p = kid[pick].name;
            for (int k = count; k > pick + 1; --k) kid[k] = kid[k - 1];
            kid[pick] = wide_child(nodes, p, 0);
            kid[pick + 1] = wide_child(nodes, p, 1);
            ++count;
        }
        uint32_t* w = out + 32 * (size_t)i;
        memset(w, 0, 32 * sizeof(uint32_t));
        for (int k = 0; k < 4; ++k)
        {
            if (k >= count) { w[24 + k] = ORC_WIDE_EMPTY; continue; }
            const float lo[3] = {kid[k].box.lower.x, kid[k].box.lower.y, kid[k].box.lower.z};
            const float hi[3] = {kid[k].box.upper.x, kid[k].box.upper.y, kid[k].box.upper.z};
            for (int a = 0; a < 3; ++a)
            {
                memcpy(&w[8 * a + k], &lo[a], 4);
                memcpy(&w[8 * a + 4 + k], &hi[a], 4);
            }
            w[24 + k] = kid[k].name;
        }
    }
}

/* ----- quantised slots (csrc/wide.cu: quantise_axis, k_wide_quantise) */
static int leaf_box_passes(orc_f3 ro, orc_f3 inv, const orc_f3* v, float tmin, float hitT);

/* a + b rounded down (up != 0: up), as __fadd_rd / __fadd_ru: the nearest sum
 * and its exact error (TwoSum) decide the step. */
static float add_dir(float a, float b, int up)
{
    float s = a + b;
    if (!isfinite(s)) return s;
    /* an exact zero sum is -0 when rounding down unless both operands are +0
     * (IEEE 754); rounding up gives the nearest sum's zero */
    if (s == 0.0f && !up && (a != 0.0f || b != 0.0f || signbit(a) || signbit(b))) return -0.0f;
    float bb = s - a;
    float err = (a - (s - bb)) + (b - bb);
    if (up) return err > 0.0f ? nextafterf(s, INFINITY) : s;
    return err < 0.0f ? nextafterf(s, -INFINITY) : s;
}
/* a * b rounded down / up (the double product of two floats is exact) */
static float mul_dir(float a, float b, int up)
{
    double p = (double)a * (double)b;
    float f = (float)p;
    if (up) return (double)f < p ? nextafterf(f, INFINITY) : f;
    return (double)f > p ? nextafterf(f, -INFINITY) : f;
}
/* a * b + c with one rounding, down (up != 0: up), as __fmaf_rd / __fmaf_ru
 * (fma.rm / fma.rp): the double product of two floats is exact, TwoSum gives
 * the exact sum as s + e, and the float nearest s is stepped once toward the
 * rounding side if it lies beyond s + e. An exact zero sum of opposite signs
 * is -0 when rounding down, +0 when rounding up (IEEE 754). */
static float fma_dir(float a, float b, float c, int up)
{
    if (isinf(c)) return c;
    const double p = (double)a * (double)b;
    const double s = p + (double)c;
    const double bb = s - p;
    const double e = (p - (s - bb)) + ((double)c - bb);
    if (s == 0.0 && e == 0.0)
    {
        if (signbit(p) && signbit(c)) return -0.0f;
        if (!signbit(p) && !signbit(c)) return 0.0f;
        return up ? 0.0f : -0.0f;
    }
    const float f = (float)s;
    const double diff = (double)f - s; /* exact: f and s are within one float ulp (or f is infinite) */
    if (up) return diff < e ? nextafterf(f, INFINITY) : f;
    return diff > e ? nextafterf(f, -INFINITY) : f;
}
/* Test hook: fma_dir exported (tests/test_oracle_walks.py checks it against
 * exact rational arithmetic). */
float orc_fma_dir(float a, float b, float c, int up) { return fma_dir(a, b, c, up); }
/* a / b rounded up (b = 255 here: the product q * 255 is exact in double) */
static float div_up(float a, float b)
{
    float q = a / b;
    return (double)q * (double)b < (double)a ? nextafterf(q, INFINITY) : q;
}
static float pow2_of(int e)
{
    uint32_t u = (uint32_t)(127 + e) << 23;
    float f;
    memcpy(&f, &u, 4);
    return f;
}
/* the plane value of code q under scale 2^E: 2^E (1 + q / 2^15) */
static float qw_value(uint32_t codes, uint32_t scaleBits, int k)
{
    uint32_t u = scaleBits | (((codes >> (8 * k)) & 255u) << 8);
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static int quantise_axis(const float lo[4], const float hi[4], uint32_t valid, float* base, float* scale,
                         uint32_t* qlo, uint32_t* qhi)
{
    *base = *scale = 0.0f;
    *qlo = *qhi = 0u;
    float nlo = ORC_FLT_MAX, nhi = -ORC_FLT_MAX;
    for (int k = 0; k < 4; ++k)
        if (valid & (1u << k))
        {
            nlo = fminf(nlo, lo[k]);
            nhi = fmaxf(nhi, hi[k]);
        }
    if (!(isfinite(nlo) && isfinite(nhi) && nlo <= nhi)) return 0;
    float m = div_up(add_dir(nhi, -nlo, 1), 255.0f);
    int e = -111;
    if (m > 0.0f)
    {
        int k;
        float f = frexpf(m, &k);
        int c = (f == 0.5f ? k - 1 : k) + 15;
        if (c > e) e = c;
    }
    for (; e <= 127; ++e)
    {
        float sc = pow2_of(e);
        float b = add_dir(nlo, -sc, 0);
        if (!isfinite(b)) return 0;
        float toCode = pow2_of(15 - e);
        int fits = 1;
        uint32_t ql_all = 0, qh_all = 0;
        for (int k = 0; k < 4; ++k)
        {
            if (!(valid & (1u << k))) continue;
            float ql = floorf(mul_dir(add_dir(add_dir(lo[k], -b, 0), -sc, 0), toCode, 0));
            float qh = ceilf(mul_dir(add_dir(add_dir(hi[k], -b, 1), -sc, 1), toCode, 1));
            if (!(qh <= 255.0f)) fits = 0;
            ql_all |= (uint32_t)fminf(fmaxf(ql, 0.0f), 255.0f) << (8 * k);
            qh_all |= (uint32_t)fminf(fmaxf(qh, 0.0f), 255.0f) << (8 * k);
        }
        *base = b;
        *scale = sc;
        *qlo = ql_all;
        *qhi = qh_all;
        if (fits) return fabsf(b) < 1.152921504606846976e18f && e <= 59; /* base < 2^60, scale <= 2^59 */
    }
    return 0;
}

/* 16 words per slot: base x y z, scale x y z, codes (x lo, x hi, y lo, y hi,
 * z lo, z hi), children. Returns 1 when every slot was quantised. */
int orc_quantise_wide(const uint32_t* wide, uint32_t n, uint32_t* out)
{
    int ok = 1;
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        const uint32_t* w = wide + 32 * (size_t)i;
        uint32_t* o = out + 16 * (size_t)i;
        uint32_t valid = 0;
        for (int k = 0; k < 4; ++k)
            if (w[24 + k] != ORC_WIDE_EMPTY) valid |= 1u << k;
        for (int a = 0; a < 3; ++a)
        {
            float lo[4], hi[4], b, sc;
            memcpy(lo, &w[8 * a], 16);
            memcpy(hi, &w[8 * a + 4], 16);
            ok &= quantise_axis(lo, hi, valid, &b, &sc, &o[6 + 2 * a], &o[7 + 2 * a]);
            memcpy(&o[a], &b, 4);
            memcpy(&o[3 + a], &sc, 4);
        }
        memcpy(&o[12], &w[24], 16);
    }
    return ok;
}

/* The slab test on planes given relative to the ray origin (slabs with
 * lower - ro, upper - ro already formed). */
static inline void slabs_offsets(orc_f3 dlo, orc_f3 dhi, orc_f3 inv, float knownHitT, float* rmin, float* rmax)
{
    orc_f3 t0 = mul3(dlo, inv);
    orc_f3 t1 = mul3(dhi, inv);
    float region_min = compMax(min3(t0, t1));
    float region_max = compMin(max3(t0, t1)) * 1.00000024f;
    *rmin = smax(region_min, 0.0f);
    *rmax = smin(region_max, knownHitT);
}

/* The slab test of child k of a quantised slot w (csrc/wide.cu layout:
 * base[3], scale[3], then per axis the lower and upper plane codes, then the
 * child words), as qwide_visit (include/mlbvh_device.cuh) forms it: per axis
 * the near plane (lower where inv > 0, upper where inv < 0) and the far plane
 * at V inv + C, C = base inv - ro inv, near planes rounded down with ro inv
 * rounded up, far planes rounded up with ro inv rounded down; entry = the
 * largest near distance moved down by 2^-22 of itself, exit = the smallest far
 * one moved up by 2^-21 of itself, then clipped to [max(0, tmin), hitT]. */
/* qwide_ray_fits: every |inv| and |ro| component below 2^62, which keeps the
 * FMA form in the float range given the quantiser's bound (bases below 2^60,
 * scales at most 2^59); other rays take the stack-free walk over the binary
 * tree instead of the quantised slots */
static int qwide_ray_fits(orc_f3 ro, orc_f3 inv)
{
    const float lim = 4.611686018427387904e18f; /* 2^62 */
    return fabsf(inv.x) < lim && fabsf(inv.y) < lim && fabsf(inv.z) < lim && fabsf(ro.x) < lim &&
           fabsf(ro.y) < lim && fabsf(ro.z) < lim;
}
#define ORC_Q_ENTRY_MARGIN 2.384185791015625e-07f
#define ORC_Q_EXIT_MARGIN 4.76837158203125e-07f
static void qwide_child(const uint32_t* w, int k, orc_f3 ro, orc_f3 inv, float tmin, float hitT, float* entry,
                        float* exitOut)
{
    float base[3];
    memcpy(base, w, 12);
    const float r[3] = {ro.x, ro.y, ro.z}, iv[3] = {inv.x, inv.y, inv.z};
    float en = 0.0f, ex = 0.0f;
    for (int a = 0; a < 3; ++a)
    {
        const int neg = iv[a] < 0.0f;
        const uint32_t qn = w[6 + 2 * a + neg], qf = w[6 + 2 * a + (1 - neg)];
        const float cn = fma_dir(base[a], iv[a], -mul_dir(r[a], iv[a], 1), 0);
        const float cf = fma_dir(base[a], iv[a], -mul_dir(r[a], iv[a], 0), 1);
        const float tn = fma_dir(qw_value(qn, w[3 + a], k), iv[a], cn, 0);
        const float tf = fma_dir(qw_value(qf, w[3 + a], k), iv[a], cf, 1);
        en = a ? smax(en, tn) : tn;
        ex = a ? smin(ex, tf) : tf;
    }
    *entry = smax(fma_dir(fabsf(en), -ORC_Q_ENTRY_MARGIN, en, 0), smax(0.0f, tmin));
    *exitOut = smin(fma_dir(fabsf(ex), ORC_Q_EXIT_MARGIN, ex, 1), hitT);
}

/* Which children of wide slot `curr` pass the slab test (FP32 slots: the
 * reference's slabs on the exact boxes; quantised slots: qwide_child), with
 * each child's entry distance. Returns the number that pass. */
static int wide_children(const uint32_t* wide, const uint32_t* qwide, uint32_t curr, orc_f3 ro, orc_f3 inv,
                         float tmin, float hitT, int pass[4], float entry[4], const uint32_t** chOut)
{
    const uint32_t* w = qwide ? qwide + 16 * (size_t)curr : wide + 32 * (size_t)curr;
    const uint32_t* ch = qwide ? w + 12 : w + 24;
    int npass = 0;
    for (int k = 0; k < 4; ++k)
    {
        pass[k] = 0;
        entry[k] = 0.0f;
        float rmin, rmax;
        if (qwide)
            qwide_child(w, k, ro, inv, tmin, hitT, &rmin, &rmax);
        else
        {
            orc_aabb b;
            memcpy(&b.lower.x, &w[k], 4);
            memcpy(&b.upper.x, &w[4 + k], 4);
            memcpy(&b.lower.y, &w[8 + k], 4);
            memcpy(&b.upper.y, &w[12 + k], 4);
            memcpy(&b.lower.z, &w[16 + k], 4);
            memcpy(&b.upper.z, &w[20 + k], 4);
            slabs(ro, inv, &b, hitT, &rmin, &rmax);
            rmin = smax(rmin, tmin);
        }
        entry[k] = rmin;
        if (ch[k] != ORC_WIDE_EMPTY && rmin <= rmax)
        {
            pass[k] = 1;
            ++npass;
        }
    }
    *chOut = ch;
    return npass;
}

/* The any-hit walk over the wide tree from `start` (a wide slot or leaf
 * position; ORC_INVALID: nothing to test). leafIndex maps leaf positions to
 * triangle indices. Children whose box passes: the nearest entry first (ties
 * to the lower slot), the others pushed in slot order; a visit whose pushes
 * would overflow ORC_WIDE_DEPTH entries restarts with the stack-free walk
 * from binaryRoot. */
static void trace_wide_any(orc_hit* hit, const uint32_t* wide, const uint32_t* qwide, const orc_node* nodes,
                           const orc_triangle* tris, const uint32_t* leafIndex, uint32_t start, uint32_t binaryRoot,
                           orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, uint32_t* visits, uint32_t* tests,
                           uint32_t* restarts)
{
    uint32_t stack[ORC_WIDE_DEPTH];
    int top = 0;
    uint32_t curr = start;
    if (start == ORC_INVALID) return;
    for (;;)
    {
        if (is_leaf(curr))
        {
            const orc_triangle* tri = &tris[leafIndex[idx_of(curr)]];
            orc_hit probe = *hit;
            int h;
            leaf_test(&probe, tris, ORC_LEAF_BIT | leafIndex[idx_of(curr)], ro, rd, tmin, &h, tests);
            if (h && (!qwide || leaf_box_passes(ro, inv, tri->v, tmin, hit->t)))
            {
                *hit = probe;
                return;
            }
        }
        else
        {
            (*visits)++;
            const uint32_t* ch;
            int pass[4], best = -1;
            float entry[4], bestT = 0.0f;
            const int npass = wide_children(wide, qwide, curr, ro, inv, tmin, hit->t, pass, entry, &ch);
            for (int k = 0; k < 4; ++k)
                if (pass[k] && (best < 0 || entry[k] < bestT)) { best = k; bestT = entry[k]; }
            if (best >= 0)
            {
                if (top + npass - 1 > ORC_WIDE_DEPTH)
                {
                    (*restarts)++;
                    stackfree_walk(hit, nodes, tris, binaryRoot, ORC_INVALID, ro, rd, inv, tmin, 1, visits, tests);
                    return;
                }
                for (int k = 0; k < 4; ++k)
                    if (pass[k] && k != best) stack[top++] = ch[k];
                curr = ch[best];
                continue;
            }
        }
        if (top == 0) return;
        curr = stack[--top];
    }
}

/* The closest-hit walk over the wide tree (wide_closest_step,
 * include/mlbvh_device.cuh): at a slot the passing children in the order of
 * their sort keys (entry bits with the two lowest replaced by the slot), the
 * nearest entered, the others pushed farthest first with their key's
 * distance; a popped child is entered only if that distance is <= hit.t;
 * every triangle hit at t <= hit.t replaces the hit (quantised slots: only if
 * the leaf's exact box passes too); a visit whose pushes would overflow
 * ORC_WIDE_DEPTH entries continues with the closest-hit stack-free walk from
 * binaryRoot, keeping the hit. */
static uint32_t wide_sort_key(int pass, float entry, int k)
{
    uint32_t u;
    memcpy(&u, &entry, 4);
    return pass ? ((u & 0x7FFFFFFCu) | (uint32_t)k) : 0xFFFFFFFFu;
}
static void trace_wide_closest(orc_hit* hit, const uint32_t* wide, const uint32_t* qwide, const orc_node* nodes,
                               const orc_triangle* tris, const uint32_t* leafIndex, uint32_t start,
                               uint32_t binaryRoot, orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, uint32_t* visits,
                               uint32_t* tests, uint32_t* restarts)
{
    uint32_t stackNode[ORC_WIDE_DEPTH], stackKey[ORC_WIDE_DEPTH];
    int top = 0;
    uint32_t curr = start;
    if (start == ORC_INVALID) return;
    for (;;)
    {
        int descend = 0;
        if (is_leaf(curr))
        {
            const orc_triangle* tri = &tris[leafIndex[idx_of(curr)]];
            orc_hit probe = *hit;
            int h;
            leaf_test(&probe, tris, ORC_LEAF_BIT | leafIndex[idx_of(curr)], ro, rd, tmin, &h, tests);
            if (h && (!qwide || leaf_box_passes(ro, inv, tri->v, tmin, hit->t))) *hit = probe;
        }
        else
        {
            (*visits)++;
            const uint32_t* ch;
            int pass[4];
            float entry[4];
            const int npass = wide_children(wide, qwide, curr, ro, inv, tmin, hit->t, pass, entry, &ch);
            if (npass > 0)
            {
                if (top + npass - 1 > ORC_WIDE_DEPTH)
                {
                    (*restarts)++;
                    stackfree_walk(hit, nodes, tris, binaryRoot, ORC_INVALID, ro, rd, inv, tmin, 0, visits, tests);
                    return;
                }
                uint32_t key[4];
                for (int k = 0; k < 4; ++k) key[k] = wide_sort_key(pass[k], entry[k], k);
                for (int i = 1; i < 4; ++i) /* insertion sort, ascending */
                    for (int j = i; j > 0 && key[j] < key[j - 1]; --j)
                    {
                        uint32_t x = key[j];
                        key[j] = key[j - 1];
                        key[j - 1] = x;
                    }
                for (int r = npass - 1; r >= 1; --r)
                {
                    stackNode[top] = ch[key[r] & 3u];
                    stackKey[top++] = key[r] & 0x7FFFFFFCu;
                }
                curr = ch[key[0] & 3u];
                descend = 1;
            }
        }
        if (descend) continue;
        for (;;)
        {
            if (top == 0) return;
            --top;
            float d;
            memcpy(&d, &stackKey[top], 4);
            if (d <= hit->t)
            {
                curr = stackNode[top];
                break;
            }
        }
    }
}

/* leaf position -> triangle index of a built tree (n leaves) */
static void leaf_positions(const orc_node* nodes, uint32_t n, uint32_t root, uint32_t* leafIndex)
{
    if (n == 1) { leafIndex[0] = idx_of(root); return; }
    for (uint32_t j = 0; j + 1 < n; ++j)
    {
        if (is_leaf(nodes[j].children[0])) leafIndex[j] = idx_of(nodes[j].children[0]);
        if (is_leaf(nodes[j].children[1])) leafIndex[j + 1] = idx_of(nodes[j].children[1]);
    }
}

typedef struct {
    const uint32_t* wide;
    const uint32_t* qwide; /* quantised slots, or NULL */
    int fallback;          /* the quantised slots are unusable: the stack-free walk for every ray */
    const orc_node* nodes;
    const orc_triangle* tris;
    const uint32_t* leafIndex;
    uint32_t root;
    const orc_ray* rays;
    orc_hit* hits;
    uint32_t *visits, *tests, *restarts;
    int any; /* any-hit (1) or closest-hit (0) rays */
} wide_ctx;

static void wide_range(void* p, uint32_t b, uint32_t e)
{
    wide_ctx* c = (wide_ctx*)p;
    for (uint32_t i = b; i < e; ++i)
    {
        const orc_ray* r = &c->rays[i];
        orc_f3 ro = f3(r->ro[0], r->ro[1], r->ro[2]);
        orc_f3 rd = f3(r->rd[0], r->rd[1], r->rd[2]);
        orc_hit hit;
        hit_init(&hit, r->tmax);
        uint32_t nv = 0, nt = 0, nr = 0;
        uint32_t start = is_leaf(c->root) ? ORC_LEAF_BIT : c->root;
        if (c->fallback || (c->qwide && !qwide_ray_fits(ro, inv_rd(rd))))
            stackfree_walk(&hit, c->nodes, c->tris, c->root, ORC_INVALID, ro, rd, inv_rd(rd), r->tmin, c->any, &nv,
                           &nt);
        else if (c->any)
            trace_wide_any(&hit, c->wide, c->qwide, c->nodes, c->tris, c->leafIndex, start, c->root, ro, rd,
                           inv_rd(rd), r->tmin, &nv, &nt, &nr);
        else
            trace_wide_closest(&hit, c->wide, c->qwide, c->nodes, c->tris, c->leafIndex, start, c->root, ro, rd,
                               inv_rd(rd), r->tmin, &nv, &nt, &nr);
        c->hits[i] = hit;
        if (c->visits) c->visits[i] = nv;
        if (c->tests) c->tests[i] = nt;
        if (c->restarts) c->restarts[i] = nr;
    }
}

void orc_trace_wide(const uint32_t* wide, const orc_node* nodes, const orc_triangle* tris, uint32_t n, uint32_t root,
                    const orc_ray* rays, uint32_t nRays, orc_hit* hits, uint32_t* visits, uint32_t* tests,
                    uint32_t* restarts, int query)
{
    uint32_t* leafIndex = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    leaf_positions(nodes, n, root, leafIndex);
    wide_ctx c = {wide, NULL, 0, nodes, tris, leafIndex, root, rays, hits, visits, tests, restarts, query != 0};
    orc_parallel_for(nRays, 1024, wide_range, &c);
    free(leafIndex);
}

void orc_trace_wide_quantised(const uint32_t* qwide, int fallback, const orc_node* nodes, const orc_triangle* tris,
                              uint32_t n, uint32_t root, const orc_ray* rays, uint32_t nRays, orc_hit* hits,
                              uint32_t* visits, uint32_t* tests, uint32_t* restarts, int query)
{
    uint32_t* leafIndex = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    leaf_positions(nodes, n, root, leafIndex);
    wide_ctx c = {NULL, qwide, fallback, nodes, tris, leafIndex, root, rays, hits, visits, tests, restarts,
                  query != 0};
    orc_parallel_for(nRays, 1024, wide_range, &c);
    free(leafIndex);
}

/* ----------------------------------------------------------------- camera */
/* RayGenerator::lookat (camera.h:10-22) */
void orc_lookat(orc_f3 eye, orc_f3 center, orc_f3 up, float fovy, int w, int h, orc_camera* cam)
{
    orc_f3 f = normalize3(sub3(center, eye));
    orc_f3 s = normalize3(cross3(f, up));
    orc_f3 u = cross3(s, f);
    float tanThetaY = tanf(fovy * 0.5f);
    float tanThetaX = tanThetaY / (float)h * (float)w;
    cam->origin = eye;
    cam->right = muls(s, tanThetaX);
    cam->up = muls(u, tanThetaY);
}

/* RayGenerator::shoot (camera.h:24-31) */
void orc_shoot(const orc_camera* cam, float u, float v, orc_f3* ro, orc_f3* rd)
{
    orc_f3 from = cam->origin;
    orc_f3 forward = normalize3(cross3(cam->up, cam->right));
    orc_f3 to = add3(add3(add3(cam->origin, forward), lerp3(neg3(cam->right), cam->right, u)),
                     lerp3(cam->up, neg3(cam->up), v));
    *ro = from;
    *rd = sub3(to, from);
}

/* ---------------------------------------------------------------- samples */
static inline uint32_t reverse_bits(uint32_t v) /* sobol.h:18-30 */
{
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
    v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
    return (v >> 16) | (v << 16);
}
/* Laine-Karras style hash permutation (sobol.h:31-39, "Practical Hash-based
 * Owen Scrambling", JCGT 2020). */
static inline uint32_t lk_permutation(uint32_t x, uint32_t seed)
{
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
static inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) /* sobol.h:40-46 */
{
    return reverse_bits(lk_permutation(reverse_bits(x), seed));
}
/* Pascal-matrix product giving Sobol's second dimension (sobol.h:51-59). */
static inline uint32_t pascal(uint32_t v)
{
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    return v;
}
static inline float random_float(uint32_t u) /* sobol.h:62-72: top 24 bits / 2^24 */
{
    return (float)(u >> 8) / (float)((0xFFFFFFFFu >> 8) + 1);
}
uint32_t orc_hash_pcg(uint32_t v) /* sobol.h:76-81, minimum_lbvh.h:904-909 */
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
static inline void pcg3d(uint32_t* x, uint32_t* y, uint32_t* z) /* sobol.h:83-107 */
{
    uint32_t vx = *x * 1664525u + 1013904223u;
    uint32_t vy = *y * 1664525u + 1013904223u;
    uint32_t vz = *z * 1664525u + 1013904223u;
    vx += vy * vz;
    vy += vz * vx;
    vz += vx * vy;
    vx ^= vx >> 16;
    vy ^= vy >> 16;
    vz ^= vz >> 16;
    vx += vy * vz;
    vy += vz * vx;
    vz += vx * vy;
    *x = vx;
    *y = vy;
    *z = vz;
}
/* shuffled_scrambled_sobol_2d (sobol.h:119-129) */
void orc_sobol(uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2, float* x, float* y)
{
    pcg3d(&p0, &p1, &p2);
    uint32_t v = lk_permutation(reverse_bits(index), p0);
    *x = random_float(nested_uniform_scramble(v, p1));
    *y = random_float(nested_uniform_scramble(pascal(v), p2));
}

/* PCG32 (main_gpu.cu:51-82, the pcg-random.org minimal generator). */
typedef struct { uint64_t state, inc; } orc_pcg;
static inline uint32_t pcg_next(orc_pcg* r)
{
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
}
static inline void pcg_init(orc_pcg* r, uint64_t seed, uint64_t seq)
{
    r->state = 0;
    r->inc = (seq << 1u) | 1u;
    pcg_next(r);
    r->state += seed;
    pcg_next(r);
}
static inline float pcg_float(orc_pcg* r)
{
    uint32_t bits = (pcg_next(r) >> 9) | 0x3f800000u;
    float v;
    memcpy(&v, &bits, 4);
    return v - 1.0f;
}

/* The project's portable FP32 sincos (shared formula with the CUDA kernels):
 * Cody-Waite reduction by pi/2 split in three float parts, then the Taylor
 * polynomials of sin (to r^9) and cos (to r^10) on [-pi/4, pi/4], evaluated
 * with fused multiply-adds so that host and device round identically. */
#define ORC_PIO2_HI 1.57079637050628662109375f
#define ORC_PIO2_MID -4.371138828673792886547744274139404296875e-8f
#define ORC_PIO2_LO -1.71512451000588187280393448475e-15f
void orc_sincos(float phi, float* s, float* c)
{
    float k = rintf(phi * 0.636619772367581343f);
    float r = fmaf(-k, ORC_PIO2_HI, phi);
    r = fmaf(-k, ORC_PIO2_MID, r);
    r = fmaf(-k, ORC_PIO2_LO, r);
    float r2 = r * r;
    float ps = fmaf(r2, (float)(1.0 / 362880.0), (float)(-1.0 / 5040.0));
    ps = fmaf(ps, r2, (float)(1.0 / 120.0));
    ps = fmaf(ps, r2, (float)(-1.0 / 6.0));
    float sr = fmaf(ps * r2, r, r);
    float pc = fmaf(r2, (float)(-1.0 / 3628800.0), (float)(1.0 / 40320.0));
    pc = fmaf(pc, r2, (float)(-1.0 / 720.0));
    pc = fmaf(pc, r2, (float)(1.0 / 24.0));
    pc = fmaf(pc, r2, -0.5f);
    float cr = fmaf(pc, r2, 1.0f);
    int q = ((int)k) & 3;
    if (q == 0) { *s = sr; *c = cr; }
    else if (q == 1) { *s = cr; *c = -sr; }
    else if (q == 2) { *s = -sr; *c = -cr; }
    else { *s = -cr; *c = sr; }
}

#define ORC_PI 3.14159265358979323846f
/* sampleHemisphereCosWeighted (main_gpu.cu:24-36) */
static inline orc_f3 sample_hemisphere(float xi0, float xi1, int trig)
{
    float phi = xi0 * 2.0f * ORC_PI;
    float r = sqrtf(xi1);
    float sp, cp;
    if (trig == ORC_TRIG_LIBM) { cp = cosf(phi); sp = sinf(phi); }
    else orc_sincos(phi, &sp, &cp);
    float x = cp * r;
    float z = sp * r;
    float y = sqrtf(fmaxf(1.0f - r * r, 0.0f));
    return f3(x, y, z);
}
/* GetOrthonormalBasis (main_gpu.cu:39-45; Duff et al. 2017) */
static inline void onb(orc_f3 z, orc_f3* xaxis, orc_f3* yaxis)
{
    const float sign = copysignf(1.0f, z.z);
    const float a = -1.0f / (sign + z.z);
    const float b = z.x * z.y * a;
    *xaxis = f3(1.0f + sign * z.x * z.x * a, sign * b, -sign * z.x);
    *yaxis = f3(b, sign + z.y * z.y * a, -z.y);
}
/* packRGBA (main_gpu.cu:17-22): (int)(c * 255 + 0.5) clamped, alpha not stored */
static inline uint32_t pack_rgba(float r, float g, float b, float a)
{
    int x = clampi(f2i_x86(r * 255.0f + 0.5f), 0, 255);
    int y = clampi(f2i_x86(g * 255.0f + 0.5f), 0, 255);
    int z = clampi(f2i_x86(b * 255.0f + 0.5f), 0, 255);
    (void)a;
    return ((uint32_t)z << 16) | ((uint32_t)y << 8) | (uint32_t)x;
}

/* -------------------------------------------------------------------- AO */
typedef struct {
    uint32_t *pixels, *occluded;
    int w, h;
    const orc_camera* cam;
    uint32_t root;
    const orc_node* nodes;
    const orc_triangle* tris;
    int useSobol, nSamples;
    float radius;
    uint32_t seed;
    int trig, rowBegin;
    uint64_t* counters;
} ao_ctx;

/* ao (main_gpu.cu:111-177), per pixel, with nSample, ray length and the
 * Sobol p2 seed as parameters (the reference fixes 16, 1.0 and 12345). */
static void ao_rows(void* p, uint32_t b, uint32_t e)
{
    ao_ctx* c = (ao_ctx*)p;
    uint64_t visits = 0, tests = 0, rays = 0;
    for (uint32_t row = b; row < e; ++row)
    {
        int yi = c->rowBegin + (int)row;
        for (int xi = 0; xi < c->w; ++xi)
        {
            int pixel = xi + yi * c->w;
            orc_f3 ro, rd;
            orc_shoot(c->cam, (float)xi / (float)c->w, (float)yi / (float)c->h, &ro, &rd);
            orc_hit hit;
            hit_init(&hit, ORC_FLT_MAX);
            uint32_t nv = 0, nt = 0;
            trace_stackfree(&hit, c->nodes, c->tris, c->root, ro, rd, inv_rd(rd), 0.0f, 0, &nv, &nt);
            rays++;
            if (hit.t == ORC_FLT_MAX)
            {
                if (c->pixels) c->pixels[pixel] = pack_rgba(0, 0, 0, 1);
                if (c->occluded) c->occluded[pixel] = 0xFFFFFFFFu;
                visits += nv;
                tests += nt;
                continue;
            }
            orc_f3 n = normalize3(hit.ng);
            if (0.0f < dot3(n, rd)) n = neg3(n);
            orc_f3 xaxis, zaxis;
            onb(n, &xaxis, &zaxis);
            orc_f3 ao_origin = add3(add3(ro, muls(rd, hit.t)), muls(n, 0.001f));
            orc_pcg rng;
            pcg_init(&rng, orc_hash_pcg((uint32_t)pixel), 0);
            float ao = 0.0f;
            uint32_t count = 0;
            for (int i = 0; i < c->nSamples; i++)
            {
                float rx, ry;
                if (c->useSobol == 1) orc_sobol((uint32_t)i, (uint32_t)xi, (uint32_t)yi, c->seed, &rx, &ry);
                else if (c->useSobol == 2) { ry = pcg_float(&rng); rx = pcg_float(&rng); }
                else { rx = pcg_float(&rng); ry = pcg_float(&rng); }
                orc_f3 dl = sample_hemisphere(rx, ry, c->trig);
                orc_f3 dir = add3(add3(muls(xaxis, dl.x), muls(zaxis, dl.z)), muls(n, dl.y));
                orc_hit h2;
                hit_init(&h2, c->radius);
                trace_stackfree(&h2, c->nodes, c->tris, c->root, ao_origin, dir, inv_rd(dir), 0.0f, 1, &nv, &nt);
                rays++;
                if (h2.t != c->radius)
                {
                    ao += 1.0f / (float)c->nSamples;
                    count++;
                }
            }
            visits += nv;
            tests += nt;
            float brightness = powf(1.0f - ao, 1.0f / 2.2f);
            if (c->pixels) c->pixels[pixel] = pack_rgba(brightness, brightness, brightness, 1.0f);
            if (c->occluded) c->occluded[pixel] = count;
        }
    }
    if (c->counters)
    {
        __atomic_fetch_add(&c->counters[0], visits, __ATOMIC_RELAXED);
        __atomic_fetch_add(&c->counters[1], tests, __ATOMIC_RELAXED);
        __atomic_fetch_add(&c->counters[2], rays, __ATOMIC_RELAXED);
    }
}

void orc_render_ao(uint32_t* pixels, uint32_t* occluded, int w, int h, const orc_camera* cam,
                   uint32_t root, const orc_node* nodes, const orc_triangle* tris,
                   int useSobol, int nSamples, float radius, uint32_t seed, int trig,
                   int rowBegin, int rowEnd, uint64_t* counters)
{
    if (rowEnd <= 0 || rowEnd > h) rowEnd = h;
    if (rowBegin < 0) rowBegin = 0;
    if (rowEnd <= rowBegin) return;
    ao_ctx c = {pixels, occluded, w, h, cam, root, nodes, tris, useSobol, nSamples, radius, seed, trig, rowBegin, counters};
    orc_parallel_for((uint32_t)(rowEnd - rowBegin), 1, ao_rows, &c);
}

/* ---------------------------------------------------------------- normal */
typedef struct {
    uint32_t* pixels;
    int w, h;
    const orc_camera* cam;
    uint32_t root;
    const orc_node* nodes;
    const orc_triangle* tris;
} normal_ctx;

/* normal (main_gpu.cu:84-109) */
static void normal_rows(void* p, uint32_t b, uint32_t e)
{
    normal_ctx* c = (normal_ctx*)p;
    for (uint32_t yi = b; yi < e; ++yi)
        for (int xi = 0; xi < c->w; ++xi)
        {
            int pixel = xi + (int)yi * c->w;
            orc_f3 ro, rd;
            orc_shoot(c->cam, (float)xi / (float)c->w, (float)yi / (float)c->h, &ro, &rd);
            orc_hit hit;
            hit_init(&hit, ORC_FLT_MAX);
            uint32_t nv = 0, nt = 0;
            trace_stackfree(&hit, c->nodes, c->tris, c->root, ro, rd, inv_rd(rd), 0.0f, 0, &nv, &nt);
            if (hit.t != ORC_FLT_MAX)
            {
                orc_f3 n = normalize3(hit.ng);
                orc_f3 col = muls(add3(n, f3(1.0f, 1.0f, 1.0f)), 0.5f);
                c->pixels[pixel] = pack_rgba(col.x, col.y, col.z, 1.0f);
            }
            else
                c->pixels[pixel] = pack_rgba(0, 0, 0, 1);
        }
}

void orc_render_normal(uint32_t* pixels, int w, int h, const orc_camera* cam, uint32_t root,
                       const orc_node* nodes, const orc_triangle* tris)
{
    normal_ctx c = {pixels, w, h, cam, root, nodes, tris};
    orc_parallel_for((uint32_t)h, 1, normal_rows, &c);
}

/* -------------------------------------------------------------------- PT */
typedef struct {
    float* accum4;
    int w, h;
    const orc_camera* cam;
    uint32_t root;
    const orc_node* nodes;
    const orc_triangle* tris;
    const float* attribs;
    int useSobol, maxSPP, maxDepth, trig;
} pt_ctx;

typedef struct {
    int useSobol, iteration, xi, yi, dimLevel;
    orc_pcg rng;
} pt_random;

static inline void pt_next(pt_random* r, float* x, float* y)
{
    if (r->useSobol == 1)
        orc_sobol((uint32_t)r->iteration, (uint32_t)r->xi, (uint32_t)r->yi, (uint32_t)(r->dimLevel++), x, y);
    else if (r->useSobol == 2)
    {
        *y = pcg_float(&r->rng);
        *x = pcg_float(&r->rng);
    }
    else
    {
        *x = pcg_float(&r->rng);
        *y = pcg_float(&r->rng);
    }
}

/* pt (main_gpu.cu:179-272): one sample per pixel, emission accumulated along
 * a cosine-sampled path, Russian roulette against max(throughput)/0.25. */
static void pt_rows(void* p, uint32_t b, uint32_t e)
{
    pt_ctx* c = (pt_ctx*)p;
    for (uint32_t yrow = b; yrow < e; ++yrow)
        for (int xi = 0; xi < c->w; ++xi)
        {
            int yi = (int)yrow;
            int pixel = xi + yi * c->w;
            float* acc = c->accum4 + 4 * (size_t)pixel;
            int iteration = (int)acc[3];
            pt_random rr;
            rr.useSobol = c->useSobol;
            rr.iteration = iteration;
            rr.xi = xi;
            rr.yi = yi;
            rr.dimLevel = 0;
            pcg_init(&rr.rng, orc_hash_pcg(orc_hash_pcg((uint32_t)pixel) + (uint32_t)iteration), 0);
            float rx, ry;
            pt_next(&rr, &rx, &ry);
            orc_f3 ro, rd;
            orc_shoot(c->cam, ((float)xi + rx) / (float)c->w, ((float)yi + ry) / (float)c->h, &ro, &rd);
            orc_f3 color = f3(0, 0, 0);
            orc_f3 throughput = f3(1, 1, 1);
            orc_hit hit;
            hit_init(&hit, ORC_FLT_MAX);
            uint32_t nv = 0, nt = 0;
            trace_stackfree(&hit, c->nodes, c->tris, c->root, ro, rd, inv_rd(rd), 0.0f, 0, &nv, &nt);
            if (hit.t != ORC_FLT_MAX)
                for (int depth = 0; depth < c->maxDepth; depth++)
                {
                    float r0, r1;
                    pt_next(&rr, &r0, &r1);
                    orc_f3 hit_p = add3(ro, muls(rd, hit.t));
                    orc_f3 hit_n = normalize3(hit.ng);
                    if (0.0f < dot3(hit_n, rd)) hit_n = neg3(hit_n);
                    const float* at = c->attribs + 15 * (size_t)hit.triangleIndex;
                    orc_f3 refl = f3(at[9], at[10], at[11]);
                    orc_f3 emis = f3(at[12], at[13], at[14]);
                    color = add3(color, mul3(throughput, emis));
                    orc_f3 xaxis, zaxis;
                    onb(hit_n, &xaxis, &zaxis);
                    orc_f3 dl = sample_hemisphere(r0, r1, c->trig);
                    orc_f3 next_ro = add3(hit_p, muls(hit_n, 0.0001f));
                    orc_f3 next_rd = add3(add3(muls(xaxis, dl.x), muls(zaxis, dl.z)), muls(hit_n, dl.y));
                    throughput = mul3(throughput, refl);
                    const float rrThreshold = 0.25f;
                    float maxComp = smax(smax(throughput.x, throughput.y), throughput.z);
                    float pr = smin(maxComp / rrThreshold, 1.0f);
                    float q0, q1;
                    pt_next(&rr, &q0, &q1);
                    if (pr < q0) break;
                    throughput = divs(throughput, pr);
                    hit_init(&hit, ORC_FLT_MAX);
                    trace_stackfree(&hit, c->nodes, c->tris, c->root, next_ro, next_rd, inv_rd(next_rd), 0.0f, 0,
                                    &nv, &nt);
                    if (hit.t == ORC_FLT_MAX) break;
                    ro = next_ro;
                    rd = next_rd;
                }
            if (iteration < c->maxSPP)
            {
                acc[0] += color.x;
                acc[1] += color.y;
                acc[2] += color.z;
                acc[3] += 1.0f;
            }
        }
}

void orc_render_pt(float* accum4, int w, int h, const orc_camera* cam, uint32_t root,
                   const orc_node* nodes, const orc_triangle* tris, const float* attribs15,
                   int useSobol, int maxSPP, int maxDepth, int trig)
{
    pt_ctx c = {accum4, w, h, cam, root, nodes, tris, attribs15, useSobol, maxSPP, maxDepth, trig};
    orc_parallel_for((uint32_t)h, 1, pt_rows, &c);
}

/* pack (main_gpu.cu:273-286) */
void orc_pack(uint32_t* pixels, const float* accum4, int n)
{
    for (int i = 0; i < n; ++i)
    {
        const float* a = accum4 + 4 * (size_t)i;
        pixels[i] = pack_rgba(powf(a[0] / a[3], 1.0f / 2.2f), powf(a[1] / a[3], 1.0f / 2.2f),
                              powf(a[2] / a[3], 1.0f / 2.2f), 1.0f);
    }
}

/* ------------------------------------------------------------ quantised tree
 * Restates csrc/quantise.cu and the quantised walks of the device header (this
 * node format has no reference counterpart; its checker is this code plus
 * the FP32 traversal above, whose closest hits it must reproduce). The
 * directed roundings are those of the quantised slots above (add_dir,
 * mul_dir, fma_dir). */
#define ORC_QMASK 0x7FFFFFu

static void tri_box(const orc_triangle* t, orc_aabb* b)
{
    aabb_set_empty(b);
    for (int j = 0; j < 3; ++j) aabb_extend_p(b, t->v[j]);
}

/* ceil(log2(x)) for finite x > 0; -150 for 0 */
static int ceil_log2(float x)
{
    if (!(x > 0.0f)) return -150;
    int k;
    const float f = frexpf(x, &k); /* x = f 2^k, f in [0.5, 1) */
    return f == 0.5f ? k - 1 : k;
}

/* The tree's scale exponent EB (quantise.cu: tree_scale_exponent): every
 * node's axis scale is 2^E with E in [max(-111, EB - 31), EB]. From the root
 * box's largest extent D and largest coordinate magnitude R, EB = max(ceil(log2
 * D) + 9, ceil(log2 R) - 13, -111): at E = EB the extent term of a code stays
 * below 64 steps and the rounding of the base below 33, so every node's codes
 * fit 8 bits. Returns 0 (and *ok = 0) for a non-finite root box or an EB
 * above 127. */
static int tree_scale_exponent(const orc_aabb* rb, int* ok)
{
    const float lo[3] = {rb->lower.x, rb->lower.y, rb->lower.z}, hi[3] = {rb->upper.x, rb->upper.y, rb->upper.z};
    float d = 0.0f, r = 0.0f;
    for (int a = 0; a < 3; ++a)
    {
        if (!(isfinite(lo[a]) && isfinite(hi[a]))) { *ok = 0; return 0; }
        d = fmaxf(d, add_dir(hi[a], -lo[a], 1));
        r = fmaxf(r, fmaxf(fabsf(lo[a]), fabsf(hi[a])));
    }
    if (!isfinite(d)) { *ok = 0; return 0; }
    int e = ceil_log2(d) + 9;
    const int e2 = ceil_log2(r) - 13;
    if (e2 > e) e = e2;
    if (e < -111) e = -111;
    *ok = e <= 127; /* a scale 2^E must be a float */
    return *ok ? e : 0;
}

/* One axis of a node (quantise.cu: quantise_axis2): base, exponent E in
 * [eLo, eHi] and the four codes (byte 0 child 0 lower, 1 child 0 upper,
 * 2 child 1 lower, 3 child 1 upper) with base + 2^E (1 + q / 2^15) <= the
 * lower and >= the upper plane in exact arithmetic (every step rounds toward
 * that side), E the smallest in range whose codes fit 8 bits. Returns 0 when
 * no E in range fits or a plane is not finite (then *codes, clamped, must not
 * be used). */
static int quantise_axis2(const float lo[2], const float hi[2], int eLo, int eHi, float* base, int* E,
                          uint32_t* codes)
{
    *base = 0.0f;
    *E = eHi;
    *codes = 0xFF00FF00u;
    const float nlo = fminf(lo[0], lo[1]), nhi = fmaxf(hi[0], hi[1]);
    if (!(isfinite(lo[0]) && isfinite(lo[1]) && isfinite(hi[0]) && isfinite(hi[1]) && nlo <= nhi)) return 0;
    const float m = div_up(add_dir(nhi, -nlo, 1), 255.0f);
    int e = -111;
    if (m > 0.0f)
    {
        const int c = ceil_log2(m) + 15;
        if (c > e) e = c;
    }
    if (e < eLo) e = eLo;
    for (; e <= eHi; ++e)
    {
        const float sc = pow2_of(e);
        const float b = add_dir(nlo, -sc, 0);
        if (!isfinite(b)) return 0;
        const float toCode = pow2_of(15 - e);
        int fits = 1;
        uint32_t q = 0;
        for (int c = 0; c < 2; ++c)
        {
            const float ql = floorf(mul_dir(add_dir(add_dir(lo[c], -b, 0), -sc, 0), toCode, 0));
            const float qh = ceilf(mul_dir(add_dir(add_dir(hi[c], -b, 1), -sc, 1), toCode, 1));
            if (!(qh <= 255.0f)) fits = 0;
            q |= (uint32_t)fminf(fmaxf(ql, 0.0f), 255.0f) << (16 * c);
            q |= (uint32_t)fminf(fmaxf(qh, 0.0f), 255.0f) << (16 * c + 8);
        }
        if (fits)
        {
            *base = b;
            *E = e;
            *codes = q;
            return 1;
        }
    }
    return 0;
}

/* k_quantise (csrc/quantise.cu). qnodes: 8 words per node (base x y z; the
 * codes of axis x, y, z, one word each; the child words, bits 23-30 holding
 * the axis exponents as k = EB - E, 5 bits each: child 0 k_x | k_y bits 0-2,
 * child 1 k_y bits 3-4 | k_z); qtris: 12 words per leaf; header: root, EB,
 * n, status (bit 0: some node's base or scale lies beyond the walks' FMA form,
 * bit 1: a non-finite coordinate). Returns 0. */
int orc_quantise(const orc_node* nodes, uint32_t root, const orc_triangle* tris, uint32_t n,
                 uint32_t* qnodes, uint32_t* parents, uint32_t* qtris, uint32_t* header)
{
    orc_aabb rb;
    if (root & ORC_LEAF_BIT) tri_box(&tris[root & ~ORC_LEAF_BIT], &rb);
    else
    {
        rb.lower = min3(nodes[root].aabbs[0].lower, nodes[root].aabbs[1].lower);
        rb.upper = max3(nodes[root].aabbs[0].upper, nodes[root].aabbs[1].upper);
    }
    int finite = 1;
    const int eb = tree_scale_exponent(&rb, &finite);
    uint32_t status = finite ? 0u : 2u;
    header[0] = (root & ORC_LEAF_BIT) ? ORC_LEAF_BIT : root;
    memcpy(&header[1], &eb, 4);
    header[2] = n;
#define PUT_QTRI(pos, t)                                                  \
    do {                                                                  \
        memcpy(qtris + 12 * (size_t)(pos), &tris[t], 36);                 \
        qtris[12 * (size_t)(pos) + 9] = (t);                              \
        qtris[12 * (size_t)(pos) + 10] = 0;                               \
        qtris[12 * (size_t)(pos) + 11] = 0;                               \
    } while (0)
    if (root & ORC_LEAF_BIT) PUT_QTRI(0, root & ~ORC_LEAF_BIT);
    const int eLo = eb - 31 < -111 ? -111 : eb - 31;
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        const orc_node* nd = &nodes[i];
        const float lo[2][3] = {{nd->aabbs[0].lower.x, nd->aabbs[0].lower.y, nd->aabbs[0].lower.z},
                                {nd->aabbs[1].lower.x, nd->aabbs[1].lower.y, nd->aabbs[1].lower.z}};
        const float hi[2][3] = {{nd->aabbs[0].upper.x, nd->aabbs[0].upper.y, nd->aabbs[0].upper.z},
                                {nd->aabbs[1].upper.x, nd->aabbs[1].upper.y, nd->aabbs[1].upper.z}};
        uint32_t code = 0, q[3];
        float base[3];
        for (int a = 0; a < 3; ++a)
        {
            const float l2[2] = {lo[0][a], lo[1][a]}, h2[2] = {hi[0][a], hi[1][a]};
            int e = eb;
            base[a] = 0.0f;
            q[a] = 0xFF00FF00u;
            if (!finite || !quantise_axis2(l2, h2, eLo, eb, &base[a], &e, &q[a])) status |= 2u;
            else if (!(fabsf(base[a]) < 1.152921504606846976e18f && e <= 59)) status |= 1u; /* 2^60, 2^59 */
            code |= (uint32_t)(eb - e) << (5 * a);
        }
        uint32_t c0 = nd->children[0], c1 = nd->children[1];
        if (c0 & ORC_LEAF_BIT) { PUT_QTRI(i, c0 & ~ORC_LEAF_BIT); c0 = ORC_LEAF_BIT | i; }
        if (c1 & ORC_LEAF_BIT) { PUT_QTRI(i + 1, c1 & ~ORC_LEAF_BIT); c1 = ORC_LEAF_BIT | (i + 1); }
        c0 |= (code & 0xFFu) << 23;
        c1 |= ((code >> 8) & 0x7Fu) << 23;
        uint32_t* w = qnodes + 8 * (size_t)i;
        memcpy(&w[0], base, 12);
        w[3] = q[0];
        w[4] = q[1];
        w[5] = q[2];
        w[6] = c0;
        w[7] = c1;
        parents[i] = nd->parent;
    }
    header[3] = status;
#undef PUT_QTRI
    return 0;
}

/* The scale bits 2^E of each axis of node w (E = EB - k). */
static inline void qnode_scales(const uint32_t* w, int eb, uint32_t s[3])
{
    const uint32_t code = ((w[6] >> 23) & 0xFFu) | (((w[7] >> 23) & 0x7Fu) << 8);
    for (int a = 0; a < 3; ++a) s[a] = (uint32_t)(eb - (int)((code >> (5 * a)) & 31u) + 127) << 23;
}

/* The decoded child boxes (load_qnode): base + V, V = 2^E (1 + q / 2^15)
 * exact, the sum rounded down for lower planes and up for upper ones. */
static inline void qnode_boxes(const uint32_t* w, int eb, orc_aabb* b0, orc_aabb* b1)
{
    uint32_t s[3];
    qnode_scales(w, eb, s);
    float base[3], l[2][3], h[2][3];
    memcpy(base, w, 12);
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 2; ++c)
        {
            l[c][a] = add_dir(base[a], qw_value(w[3 + a], s[a], 2 * c), 0);
            h[c][a] = add_dir(base[a], qw_value(w[3 + a], s[a], 2 * c + 1), 1);
        }
    b0->lower = f3(l[0][0], l[0][1], l[0][2]);
    b0->upper = f3(h[0][0], h[0][1], h[0][2]);
    b1->lower = f3(l[1][0], l[1][1], l[1][2]);
    b1->upper = f3(h[1][0], h[1][1], h[1][2]);
}

/* Checks that every child box of the quantised tree, in exact arithmetic
 * (base + V: rounded up it is <= a lower plane iff the exact sum is, rounded
 * down >= an upper one iff the exact sum is), contains the FP32 child box of
 * the same node. Returns 1 when all do (and the tree is usable: status bit 1
 * clear). */
int orc_check_quantised(const orc_node* nodes, uint32_t n, const uint32_t* qnodes, const uint32_t* header)
{
    int eb;
    memcpy(&eb, &header[1], 4);
    if (header[3] & 2u) return 0;
    for (uint32_t i = 0; i + 1 < n; ++i)
    {
        const uint32_t* w = qnodes + 8 * (size_t)i;
        uint32_t s[3];
        qnode_scales(w, eb, s);
        float base[3];
        memcpy(base, w, 12);
        for (int c = 0; c < 2; ++c)
        {
            const orc_aabb* e = &nodes[i].aabbs[c];
            const float el[3] = {e->lower.x, e->lower.y, e->lower.z}, eh[3] = {e->upper.x, e->upper.y, e->upper.z};
            for (int a = 0; a < 3; ++a)
            {
                if (add_dir(base[a], qw_value(w[3 + a], s[a], 2 * c), 1) > el[a]) return 0;
                if (add_dir(base[a], qw_value(w[3 + a], s[a], 2 * c + 1), 0) < eh[a]) return 0;
            }
        }
    }
    return 1;
}

typedef struct {
    const uint32_t *qnodes, *parents, *qtris;
    uint32_t root;
    int eb;          /* the tree's scale exponent EB */
    uint32_t status; /* header[3] */
    const orc_ray* rays;
    int query;
    orc_hit* hits;
    uint32_t *visits, *tests, *ups;
    int stackDepth; /* 0: stack-free walk; 1..64: replay walk with that many stack entries */
} qtrace_ctx;

/* leaf_box_passes (include/mlbvh_device.cuh): on a hit in a quantised walk,
 * the reference's slabs on the triangle's FP32 box must pass as well. */
static int leaf_box_passes(orc_f3 ro, orc_f3 inv, const orc_f3* v, float tmin, float hitT)
{
    orc_aabb b;
    aabb_set_empty(&b);
    for (int j = 0; j < 3; ++j) aabb_extend_p(&b, v[j]);
    float e, x;
    slabs(ro, inv, &b, hitT, &e, &x);
    e = smax(e, tmin);
    return e <= x;
}

/* qnode_test (include/mlbvh_device.cuh): the slab test of both children of
 * quantised node w, as entry / exit pairs clipped to [max(0, tmin), hitT].
 * fma (a ray for which qwide_ray_fits holds, in a tree whose status is 0):
 * per axis the near plane (lower where inv > 0, upper where inv < 0) and the
 * far plane at V inv + C, C = base inv - ro inv, near planes rounded down
 * with ro inv rounded up, far planes up with ro inv rounded down; the entry
 * (largest near distance) moved down by 2^-22 of itself, the exit (smallest
 * far distance) up by 2^-21 of itself, as the quantised slots do. Otherwise
 * the reference's slabs on the decoded boxes (qnode_boxes). Status bit 1 (a
 * non-finite coordinate): every box passes. */
static void qnode_test(const qtrace_ctx* c, const uint32_t* w, orc_f3 ro, orc_f3 inv, float tmin, float hitT, int fma,
                       float* lmin, float* lmax, float* rmin, float* rmax)
{
    if (c->status & 2u)
    {
        *lmin = *rmin = smax(0.0f, tmin);
        *lmax = *rmax = hitT;
        return;
    }
    if (fma)
    {
        uint32_t sb[3];
        qnode_scales(w, c->eb, sb);
        float base[3];
        memcpy(base, w, 12);
        const float r[3] = {ro.x, ro.y, ro.z}, iv[3] = {inv.x, inv.y, inv.z};
        float e[2], x[2];
        for (int k = 0; k < 2; ++k)
        {
            float en = 0.0f, ex = 0.0f;
            for (int a = 0; a < 3; ++a)
            {
                const int neg = iv[a] < 0.0f;
                const float cn = fma_dir(base[a], iv[a], -mul_dir(r[a], iv[a], 1), 0);
                const float cf = fma_dir(base[a], iv[a], -mul_dir(r[a], iv[a], 0), 1);
                const float tn = fma_dir(qw_value(w[3 + a], sb[a], 2 * k + neg), iv[a], cn, 0);
                const float tf = fma_dir(qw_value(w[3 + a], sb[a], 2 * k + 1 - neg), iv[a], cf, 1);
                en = a ? smax(en, tn) : tn;
                ex = a ? smin(ex, tf) : tf;
            }
            e[k] = smax(fma_dir(fabsf(en), -ORC_Q_ENTRY_MARGIN, en, 0), smax(0.0f, tmin));
            x[k] = smin(fma_dir(fabsf(ex), ORC_Q_EXIT_MARGIN, ex, 1), hitT);
        }
        *lmin = e[0];
        *lmax = x[0];
        *rmin = e[1];
        *rmax = x[1];
        return;
    }
    orc_aabb b0, b1;
    qnode_boxes(w, c->eb, &b0, &b1);
    slabs(ro, inv, &b0, hitT, lmin, lmax);
    slabs(ro, inv, &b1, hitT, rmin, rmax);
    *lmin = smax(*lmin, tmin);
    *rmin = smax(*rmin, tmin);
}

/* trace_quantised (include/mlbvh_device.cuh): the stack-free state machine
 * over quantised nodes; "came from the parent" is "came from neither child",
 * and the parent word is read only when moving up. */
static void qtrace_walk(const qtrace_ctx* c, orc_hit* hit, orc_f3 ro, orc_f3 rd, orc_f3 inv, float tmin, uint32_t curr,
                        uint32_t prev, uint32_t* nv, uint32_t* nt, uint32_t* nu)
{
    const int fma = c->status == 0u && qwide_ray_fits(ro, inv);
    while (curr != ORC_INVALID)
    {
        if (curr & ORC_LEAF_BIT)
        {
            (*nt)++;
            const uint32_t* q = c->qtris + 12 * (size_t)(curr & ORC_QMASK);
            orc_f3 v[3];
            memcpy(v, q, 36);
            float t, u, vv;
            orc_f3 ng;
            if (intersect_tri(&t, &u, &vv, &ng, tmin, hit->t, ro, rd, v[0], v[1], v[2]) &&
                leaf_box_passes(ro, inv, v, tmin, hit->t))
            {
                hit->t = t;
                hit->u = u;
                hit->v = vv;
                hit->ng = ng;
                hit->triangleIndex = q[9];
                if (c->query == 1) break;
            }
            uint32_t s = curr;
            curr = prev;
            prev = s;
            continue;
        }
        (*nv)++;
        const uint32_t* w = c->qnodes + 8 * (size_t)curr;
        uint32_t c0 = w[6] & (ORC_LEAF_BIT | ORC_QMASK), c1 = w[7] & (ORC_LEAF_BIT | ORC_QMASK);
        float lmin, lmax, rmin, rmax;
        qnode_test(c, w, ro, inv, tmin, hit->t, fma, &lmin, &lmax, &rmin, &rmax);
        int hitL = lmin <= lmax, hitR = rmin <= rmax;
        uint32_t nearN = c0, farN = c1;
        int nHits = 0;
        if (hitL && hitR)
        {
            if (rmin < lmin) { nearN = c1; farN = c0; }
            nHits = 2;
        }
        else if (hitL || hitR)
        {
            nHits = 1;
            nearN = hitR ? farN : nearN;
        }
        int fromParent = prev != c0 && prev != c1, up;
        uint32_t next = ORC_INVALID;
        if (fromParent) { up = nHits == 0; next = nearN; }
        else if (prev == nearN) { up = nHits != 2; next = farN; }
        else up = 1;
        if (up) { (*nu)++; next = c->parents[curr]; }
        prev = curr;
        curr = next;
    }
}

static void qtrace_one(const qtrace_ctx* c, orc_hit* hit, orc_f3 ro, orc_f3 rd, float tmin, uint32_t* nv, uint32_t* nt,
                       uint32_t* nu)
{
    qtrace_walk(c, hit, ro, rd, inv_rd(rd), tmin, c->root, ORC_INVALID, nv, nt, nu);
}

/* quantised_replay_step (include/mlbvh_device.cuh): the same walk with a
 * stack of pending far children (node, entry distance) instead of revisits.
 * At a node whose two child boxes are hit, the far child is pushed and the
 * near child entered; when a subtree is done, entries are popped and an entry
 * is entered iff its entry distance is still <= hit.t, which is exactly when
 * the stack-free walk, back at the parent, finds both boxes still hit (the
 * near entry never exceeds the far one). So leaves are tested in the same
 * order against the same hit.t. A push onto a full stack (depth entries)
 * hands the walk to the stack-free state machine at (near child, parent),
 * which re-derives every pending entry on its way up. */
static void qreplay_one(const qtrace_ctx* c, int depth, orc_hit* hit, orc_f3 ro, orc_f3 rd, float tmin, uint32_t* nv,
                        uint32_t* nt, uint32_t* nu)
{
    orc_f3 inv = inv_rd(rd);
    const int fma = c->status == 0u && qwide_ray_fits(ro, inv);
    uint32_t stackNode[64];
    float stackEntry[64];
    int top = 0;
    uint32_t curr = c->root;
    for (;;)
    {
        int pop = 0;
        if (curr & ORC_LEAF_BIT)
        {
            (*nt)++;
            const uint32_t* q = c->qtris + 12 * (size_t)(curr & ORC_QMASK);
            orc_f3 v[3];
            memcpy(v, q, 36);
            float t, u, vv;
            orc_f3 ng;
            if (intersect_tri(&t, &u, &vv, &ng, tmin, hit->t, ro, rd, v[0], v[1], v[2]) &&
                leaf_box_passes(ro, inv, v, tmin, hit->t))
            {
                hit->t = t;
                hit->u = u;
                hit->v = vv;
                hit->ng = ng;
                hit->triangleIndex = q[9];
                if (c->query == 1) return;
            }
            pop = 1;
        }
        else
        {
            (*nv)++;
            const uint32_t* w = c->qnodes + 8 * (size_t)curr;
            uint32_t c0 = w[6] & (ORC_LEAF_BIT | ORC_QMASK), c1 = w[7] & (ORC_LEAF_BIT | ORC_QMASK);
            float lmin, lmax, rmin, rmax;
            qnode_test(c, w, ro, inv, tmin, hit->t, fma, &lmin, &lmax, &rmin, &rmax);
            int hitL = lmin <= lmax, hitR = rmin <= rmax;
            if (hitL && hitR)
            {
                uint32_t nearN = c0, farN = c1;
                float farEntry = rmin;
                if (rmin < lmin) { nearN = c1; farN = c0; farEntry = lmin; }
                if (top == depth)
                {
                    qtrace_walk(c, hit, ro, rd, inv, tmin, nearN, curr, nv, nt, nu);
                    return;
                }
                stackNode[top] = farN;
                stackEntry[top] = farEntry;
                ++top;
                curr = nearN;
            }
            else if (hitL || hitR)
                curr = hitL ? c0 : c1;
            else
                pop = 1;
        }
        if (pop)
        {
            for (;;)
            {
                if (top == 0) return;
                --top;
                if (stackEntry[top] <= hit->t) { curr = stackNode[top]; break; }
            }
        }
    }
}

static void qtrace_range(void* p, uint32_t b, uint32_t e)
{
    qtrace_ctx* c = (qtrace_ctx*)p;
    for (uint32_t i = b; i < e; ++i)
    {
        const orc_ray* r = &c->rays[i];
        orc_hit hit;
        hit_init(&hit, r->tmax);
        uint32_t nv = 0, nt = 0, nu = 0;
        if (c->stackDepth > 0)
            qreplay_one(c, c->stackDepth, &hit, f3(r->ro[0], r->ro[1], r->ro[2]), f3(r->rd[0], r->rd[1], r->rd[2]),
                        r->tmin, &nv, &nt, &nu);
        else
            qtrace_one(c, &hit, f3(r->ro[0], r->ro[1], r->ro[2]), f3(r->rd[0], r->rd[1], r->rd[2]), r->tmin, &nv, &nt,
                       &nu);
        c->hits[i] = hit;
        if (c->visits) c->visits[i] = nv;
        if (c->tests) c->tests[i] = nt;
        if (c->ups) c->ups[i] = nu;
    }
}

void orc_trace_quantised(const uint32_t* qnodes, const uint32_t* parents, const uint32_t* qtris, const uint32_t* header,
                         const orc_ray* rays, uint32_t nRays, int query, orc_hit* hits, uint32_t* visits,
                         uint32_t* tests, uint32_t* ups)
{
    qtrace_ctx c;
    c.qnodes = qnodes;
    c.parents = parents;
    c.qtris = qtris;
    c.root = header[0];
    memcpy(&c.eb, &header[1], 4);
    c.status = header[3];
    c.rays = rays;
    c.query = query;
    c.hits = hits;
    c.visits = visits;
    c.tests = tests;
    c.ups = ups;
    c.stackDepth = 0;
    orc_parallel_for(nRays, 1024, qtrace_range, &c);
}

void orc_trace_quantised_replay(const uint32_t* qnodes, const uint32_t* parents, const uint32_t* qtris,
                                const uint32_t* header, const orc_ray* rays, uint32_t nRays, int query, int stackDepth,
                                orc_hit* hits, uint32_t* visits, uint32_t* tests, uint32_t* ups)
{
    qtrace_ctx c;
    c.qnodes = qnodes;
    c.parents = parents;
    c.qtris = qtris;
    c.root = header[0];
    memcpy(&c.eb, &header[1], 4);
    c.status = header[3];
    c.rays = rays;
    c.query = query;
    c.hits = hits;
    c.visits = visits;
    c.tests = tests;
    c.ups = ups;
    c.stackDepth = stackDepth < 1 ? 1 : stackDepth > 64 ? 64 : stackDepth;
    orc_parallel_for(nRays, 1024, qtrace_range, &c);
}

/* ------------------------------------------------ differentiable path trace
 * Restates csrc/adjoint.cu (no reference counterpart). The path geometry
 * (hits, directions) is computed in FP32 exactly as the kernels do, so the
 * paths are the GPU's; the radiance and the gradient are accumulated either
 * in FP32 in the kernels' order (for bit-exact image parity) or in FP64 (the
 * FP64 host adjoint and the finite differences). */
#define ORC_MAX_BOUNCES 8

static int diff_path(uint32_t* tri, int bounces, uint32_t s, int xi, int yi, int w, int h, const orc_camera* cam,
                     uint32_t root, const orc_node* nodes, const orc_triangle* tris)
{
    float jx, jy;
    orc_sobol(s, (uint32_t)xi, (uint32_t)yi, 0u, &jx, &jy);
    orc_f3 ro, rd;
    orc_shoot(cam, ((float)xi + jx) / (float)w, ((float)yi + jy) / (float)h, &ro, &rd);
    orc_hit hit;
    hit_init(&hit, ORC_FLT_MAX);
    uint32_t nv = 0, nt = 0;
    trace_stackfree(&hit, nodes, tris, root, ro, rd, inv_rd(rd), 0.0f, 0, &nv, &nt);
    if (hit.t == ORC_FLT_MAX) return 0;
    int count = 0;
    for (int d = 0; d <= bounces; ++d)
    {
        tri[count++] = hit.triangleIndex;
        if (d == bounces) break;
        orc_f3 p = add3(ro, muls(rd, hit.t));
        orc_f3 n = normalize3(hit.ng);
        if (0.0f < dot3(n, rd)) n = neg3(n);
        orc_f3 xaxis, zaxis;
        onb(n, &xaxis, &zaxis);
        float r0, r1;
        orc_sobol(s, (uint32_t)xi, (uint32_t)yi, (uint32_t)(1 + d), &r0, &r1);
        orc_f3 dl = sample_hemisphere(r0, r1, ORC_TRIG_PORTABLE);
        ro = add3(p, muls(n, 0.0001f));
        rd = add3(add3(muls(xaxis, dl.x), muls(zaxis, dl.z)), muls(n, dl.y));
        hit_init(&hit, ORC_FLT_MAX);
        trace_stackfree(&hit, nodes, tris, root, ro, rd, inv_rd(rd), 0.0f, 0, &nv, &nt);
        if (hit.t == ORC_FLT_MAX) break;
    }
    return count;
}

typedef struct {
    int w, h, spp, bounces;
    const orc_camera* cam;
    uint32_t root;
    const orc_node* nodes;
    const orc_triangle* tris;
    const float* albedo32;
    const float* emission32;
    const double* albedo64;
    const double* emission64;
    float* image32;
    double* image64;
    const double* gradImage;
    double* grad;
} diff_ctx;

static void atomic_add_double(double* p, double v)
{
    uint64_t old = __atomic_load_n((uint64_t*)p, __ATOMIC_RELAXED), upd;
    do
    {
        double cur;
        memcpy(&cur, &old, 8);
        cur += v;
        memcpy(&upd, &cur, 8);
    } while (!__atomic_compare_exchange_n((uint64_t*)p, &old, upd, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
}

/* k_pt_diff_render gives each pixel a warp: lane l sums the radiance of
 * samples l, l + 32, ... in order, and the pixel's sum is the pairwise tree of
 * the lanes' sums in lane order, ((p0 + p1) + (p2 + p3)) + ... */
#define ORC_DIFF_LANES 32
static void diff_rows(void* p, uint32_t b, uint32_t e)
{
    diff_ctx* c = (diff_ctx*)p;
    uint32_t tri[ORC_MAX_BOUNCES + 1];
    for (uint32_t y = b; y < e; ++y)
        for (int x = 0; x < c->w; ++x)
        {
            int px = x + (int)y * c->w;
            float part32[ORC_DIFF_LANES] = {0.0f};
            double sum64 = 0.0;
            double g = c->gradImage ? c->gradImage[px] / (double)c->spp : 0.0;
            for (int s = 0; s < c->spp; ++s)
            {
                int n = diff_path(tri, c->bounces, (uint32_t)s, x, (int)y, c->w, c->h, c->cam, c->root, c->nodes, c->tris);
                if (c->image32)
                {
                    float thr = 1.0f, L = 0.0f;
                    float coll[ORC_MAX_BOUNCES + 1];
                    for (int d = 0; d < n; ++d)
                    {
                        coll[d] = thr * c->emission32[tri[d]];
                        if (d < c->bounces) thr = thr * c->albedo32[tri[d]];
                    }
                    for (int d = 0; d < n; ++d) L += coll[d];
                    part32[s % ORC_DIFF_LANES] += L; /* the pixel's lane s % 32, its samples in order */
                }
                if (c->image64 || c->grad)
                {
                    double thr = 1.0, coll[ORC_MAX_BOUNCES + 1];
                    for (int d = 0; d < n; ++d)
                    {
                        coll[d] = thr * c->emission64[tri[d]];
                        thr *= c->albedo64[tri[d]];
                    }
                    if (c->image64)
                        for (int d = 0; d < n; ++d) sum64 += coll[d];
                    if (c->grad && g != 0.0)
                    {
                        double after = 0.0;
                        for (int j = n - 1; j >= 0; --j)
                        {
                            if (j < c->bounces && after != 0.0)
                                atomic_add_double(&c->grad[tri[j]], g * after / c->albedo64[tri[j]]);
                            after += coll[j];
                        }
                    }
                }
            }
            if (c->image32)
            {
                for (int width = ORC_DIFF_LANES; width > 1; width /= 2)
                    for (int i = 0; i < width / 2; ++i) part32[i] = part32[2 * i] + part32[2 * i + 1];
                c->image32[px] = part32[0] / (float)c->spp;
            }
            if (c->image64) c->image64[px] = sum64 / (double)c->spp;
        }
}

/* k_pt_diff_render in FP32 (bit-exact with the kernel) and/or FP64. */
void orc_pt_diff_render(float* image32, double* image64, int w, int h, int spp, int bounces, const orc_camera* cam,
                        uint32_t root, const orc_node* nodes, const orc_triangle* tris, const float* albedo32,
                        const float* emission32, const double* albedo64, const double* emission64)
{
    diff_ctx c = {w, h, spp, bounces, cam, root, nodes, tris, albedo32, emission32, albedo64, emission64,
                  image32, image64, NULL, NULL};
    orc_parallel_for((uint32_t)h, 1, diff_rows, &c);
}

/* The FP64 host adjoint: grad[t] += sum over paths of dLoss/dI_p / spp *
 * (radiance collected after each scattering at t) / albedo[t]. */
void orc_pt_diff_adjoint(double* grad, const double* gradImage, int w, int h, int spp, int bounces,
                         const orc_camera* cam, uint32_t root, const orc_node* nodes, const orc_triangle* tris,
                         const double* albedo64, const double* emission64)
{
    diff_ctx c = {w, h, spp, bounces, cam, root, nodes, tris, NULL, NULL, albedo64, emission64, NULL, NULL,
                  gradImage, grad};
    orc_parallel_for((uint32_t)h, 1, diff_rows, &c);
}
