/*
 * mlbvh.h — the C-ABI boundary of minimumlbvh_b200, the B200 (sm_100a)
 * implementation of MinimumLBVH's build and query path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and is
 * stream-ordered: device buffers are owned by the caller, nothing is
 * allocated, and nothing synchronises unless stated. `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream). Device
 * pointers must be 16-byte aligned, and node arrays that a query reads
 * (mlbvh_internal_node, mlbvh_qnode) 32-byte aligned, as cudaMalloc returns
 * them (checked; MLBVH_ERR_INVALID_ARG).
 *
 * Data layouts are byte-identical to the reference's minimum_lbvh.h types so
 * that buffers built here can be handed to code written against it:
 *   mlbvh_triangle       = minimum_lbvh::Triangle      (minimum_lbvh.h:207-210) 36 B
 *   mlbvh_aabb           = minimum_lbvh::AABB          (minimum_lbvh.h:217-252) 24 B
 *   mlbvh_node_index     = minimum_lbvh::NodeIndex     (minimum_lbvh.h:254-265)  4 B
 *                          bits 0-30 index, bit 31 leaf flag; 0x7FFFFFFF = invalid
 *   mlbvh_internal_node  = minimum_lbvh::InternalNode  (minimum_lbvh.h:276-282) 64 B
 *   mlbvh_hit            = minimum_lbvh::Hit           (minimum_lbvh.h:890-896) 32 B
 *   mlbvh_ray_generator  = RayGenerator                (camera.h:3-32)          36 B
 *   mlbvh_triangle_attrib= TriangleAttrib              (main_gpu.cu:10-15)      60 B
 */
#ifndef MLBVH_H
#define MLBVH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLBVH_VERSION 1

#if defined(__GNUC__)
#define MLBVH_API __attribute__((visibility("default")))
#else
#define MLBVH_API
#endif

typedef enum mlbvh_status {
    MLBVH_OK = 0,
    MLBVH_ERR_INVALID_ARG = 1, /* null/misaligned pointer, bad size, scratch too small */
    MLBVH_ERR_OOM = 2,         /* reserved for callers' allocation wrappers */
    MLBVH_ERR_TIMEOUT = 3,     /* a bounded device-side wait gave up (see mlbvh_scratch_status) */
    MLBVH_ERR_LAUNCH = 4,      /* a kernel launch failed */
    MLBVH_ERR_CUDA = 5         /* another CUDA runtime error */
} mlbvh_status;

enum {
    MLBVH_BUILD_OPTION_USE_NORMAL = 1,  /* BUILD_OPTION_USE_NORMAL, minimum_lbvh.h:44 */
    MLBVH_BUILD_OPTION_CPU_PARALLEL = 2 /* accepted and ignored: the build always runs on the GPU */
};
enum { MLBVH_RAY_QUERY_CLOSEST = 0, MLBVH_RAY_QUERY_ANY = 1 }; /* RAY_QUERY, minimum_lbvh.h:975 */
enum {
    MLBVH_TRAVERSAL_STACKFREE = 0,   /* intersect_stackfree,   minimum_lbvh.h:981  */
    MLBVH_TRAVERSAL_ESCAPE_LINK = 1, /* intersect_escape_link, minimum_lbvh.h:1063 */
    MLBVH_TRAVERSAL_STACKFULL = 2,   /* intersect_stackfull,   minimum_lbvh.h:912  */
    /* intersect_stackfree's Hit records (bit for bit, ties included) from a walk
     * that keeps pending far children on a 16-entry stack instead of revisiting
     * nodes through their parents; no reference counterpart */
    MLBVH_TRAVERSAL_REPLAY = 3
};

typedef struct mlbvh_triangle { float vs[3][3]; } mlbvh_triangle;
typedef struct mlbvh_aabb { float lower[3]; float upper[3]; } mlbvh_aabb;
typedef uint32_t mlbvh_node_index;
typedef struct mlbvh_internal_node {
    mlbvh_node_index children[2];
    mlbvh_aabb aabbs[2];
    mlbvh_node_index parent;
    uint32_t context; /* upper bound of the leaf range after the build (0xFFFFFFFF at the top) */
} mlbvh_internal_node;
typedef struct mlbvh_hit {
    float t; /* FLT_MAX (3.402823466e+38f) when nothing was hit */
    uint32_t _pad;
    float uv[2];
    float ng[3];
    uint32_t triangleIndex; /* 0xFFFFFFFF when nothing was hit */
} mlbvh_hit;
/* A query ray. The reference's intersect_* take (ro, rd) with the initial
 * hit.t as the far limit and 0 as the near one; tmin = 0 gives exactly that. */
typedef struct mlbvh_ray { float ro[3]; float tmin; float rd[3]; float tmax; } mlbvh_ray;
typedef struct mlbvh_ray_generator { float origin[3]; float right[3]; float up[3]; } mlbvh_ray_generator;
typedef struct mlbvh_triangle_attrib {
    float shadingNormals[3][3];
    float reflectance[3];
    float emissive[3];
} mlbvh_triangle_attrib;

/* The quantised tree (no reference counterpart; a replacement node format for
 * the same topology, 32 bytes instead of 64):
 *   base       per axis a the base b_a (FP32); axis a has the scale 2^E_a
 *   q[4*a+0..3] the 8-bit codes of axis a: child 0 lower, child 0 upper,
 *              child 1 lower, child 1 upper. Code q stands for the plane
 *              b_a + 2^E_a (1 + q / 2^15); lower planes lie at or below the
 *              exact child box, upper ones at or above it (exact arithmetic)
 *   child[c]   bit 31 leaf flag; bits 0-22 internal-node index or leaf
 *              position; bits 23-30 carry the three 5-bit axis codes
 *              k_a = eBase - E_a (child[0]: k_x | k_y bits 0-2; child[1]:
 *              k_y bits 3-4 | k_z)
 * Parents live in a separate array (read only when the walk moves up).
 * Leaves are stored in sorted (leaf) order as mlbvh_qtri: the triangle's three
 * FP32 corners, unchanged, and its original index. */
typedef struct mlbvh_qnode {
    float base[3];
    uint8_t q[12];
    uint32_t child[2];
} mlbvh_qnode;
typedef struct mlbvh_qtri {
    float v[9];
    uint32_t triangleIndex;
    uint32_t _pad[2];
} mlbvh_qtri;
typedef struct mlbvh_qheader {
    uint32_t root;   /* bit 31 leaf flag, bits 0-22 index */
    int32_t eBase;   /* the scale exponent of axis code k = 0: E = eBase - k */
    uint32_t nTriangles;
    uint32_t status; /* bit 0: a base of 2^60 or more or a scale above 2^59 (the walks then
                        test the decoded boxes with the reference's slabs); bit 1: a
                        non-finite coordinate, or a root box so large that its scale
                        exponent would exceed 127 (about 1e36; every box then passes) */
} mlbvh_qheader;

/* The 4-wide tree for any-hit rays (no reference counterpart): a 4-wide
 * regrouping of the same binary tree. Slot i holds the expansion of binary
 * internal node i: its two children, then repeatedly the internal child of
 * largest surface area replaced by its two children, until four children or
 * only leaves are left. Child boxes are the binary tree's own (exact FP32),
 * stored per axis (axis[a].lo[c], axis[a].hi[c] for child c). child[c] is an
 * internal-node index (which is also the slot of that node's expansion), a
 * leaf position with bit 31 set (leaf j = left leaf child of binary node j or
 * right leaf child of node j - 1, as in mlbvh_leaf_triangles), or 0xFFFFFFFF
 * for an empty slot. Every leaf whose box passes a ray's slab test is reached
 * through boxes that pass too (a box contains its descendants' boxes and the
 * slab test is monotone in the box), so an any-hit walk over this tree finds
 * a hit exactly when intersect_stackfree's any-hit walk does. */
typedef struct mlbvh_wnode {
    struct {
        float lo[4], hi[4];
    } axis[3];         /* axis[a].lo[c], axis[a].hi[c]: 32 bytes per axis */
    uint32_t child[4];
    uint32_t _pad[4];  /* zero */
} mlbvh_wnode;         /* 128 bytes, 128-byte aligned */

/* The 4-wide tree with 8-bit child planes (no reference counterpart): the
 * slots of mlbvh_wnode in 64 bytes. Per axis a, a base and a power of two
 * scale; plane code q stands for base[a] + scale[a] * (1 + q / 32768). Lower
 * plane codes are rounded down and upper ones up (and decoded with the same
 * directed rounding), so a decoded child box contains the exact one. */
typedef struct mlbvh_qwnode {
    float base[3];
    float scale[3];
    uint8_t q[3][2][4]; /* q[a][0][c], q[a][1][c]: lower, upper plane of child c on axis a */
    uint32_t child[4];  /* as in mlbvh_wnode */
} mlbvh_qwnode;         /* 64 bytes, 32-byte aligned */

/* Library version (MLBVH_VERSION) and the message of the last error raised on
 * the calling host thread ("" if none). */
MLBVH_API int mlbvh_version(void);
MLBVH_API const char* mlbvh_last_error_string(void);

/* ---------------------------------------------------------------- build ---
 * Replaces BVHGPUBuilder::build (minimum_lbvh.h:783-871) and the
 * OnesweepSort it drives (tinyhiponesweep.h:592-668). Scene AABB, Morton keys
 * (minimum_lbvh.cu:38-92), a stable LSD radix sort of (key, triangle index),
 * deltas (minimum_lbvh.cu:94-102) and the agglomerative build
 * (minimum_lbvh.h:284-361) run as a chain of kernels on `stream`.
 *
 * dInternals receives nTriangles-1 nodes, *dRootNode the root (a leaf when
 * nTriangles == 1). dSceneAABB may be NULL. dScratch must hold
 * mlbvh_build_scratch_bytes(nTriangles) bytes; its contents need no
 * initialisation and must not be shared by builds in flight at the same time.
 * 1 <= nTriangles < 2^30. */
MLBVH_API size_t mlbvh_build_scratch_bytes(uint32_t nTriangles);
MLBVH_API mlbvh_status mlbvh_build(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption,
                         mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode,
                         mlbvh_aabb* dSceneAABB, void* dScratch, size_t scratchBytes, void* stream);

/* mlbvh_build plus the intermediate arrays the reference keeps or prints:
 * the sorted Morton keys and triangle indices (IndexedMorton after
 * OnesweepSort, minimum_lbvh.h:833) and the split deltas (BVHCPUBuilder::
 * m_deltas, minimum_lbvh.h:668). Each of the three may be NULL. */
MLBVH_API mlbvh_status mlbvh_build_ex(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption,
                            mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode,
                            mlbvh_aabb* dSceneAABB, uint32_t* dSortedKeys, uint32_t* dSortedIndices,
                            uint8_t* dDeltas, void* dScratch, size_t scratchBytes, void* stream);

/* mlbvh_build without the scratch argument, for callers that must not
 * allocate device memory: plugins whose host application owns all GPU memory
 * through its own allocator, and real-time loops that cannot afford
 * cudaMalloc's implicit device synchronisation or its failure mid-frame. This
 * entry point has no counterpart in the reference (whose builder allocates
 * and frees its temporaries on every build).
 * Its scratch is a fixed 2 MiB device array inside this library, held by
 * every GPU that loads the library until the process exits; it limits the
 * build to nTriangles <= 65536 (larger sizes return MLBVH_ERR_INVALID_ARG).
 * The caller still passes the triangles and the output buffers. The first
 * call in each CUDA context of a device (the first call on the device, and
 * again after cudaDeviceReset) looks up the array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture. Every call shares the one array, which keeps
 * the last call's contents: calls that overlap on the GPU (e.g. on two
 * streams) race and must be serialised by the caller. Nothing is allocated
 * or freed. Like mlbvh_build it does not synchronise; whether a bounded wait
 * of the last call on this device gave up (its tree is then unusable) is
 * reported by mlbvh_scratch_status(NULL, stream), and mlbvh_set_spin_limit
 * applies to it as to mlbvh_build. */
MLBVH_API mlbvh_status mlbvh_build_noalloc(const mlbvh_triangle* dTriangles, uint32_t nTriangles,
                                           uint32_t buildOption, mlbvh_internal_node* dInternals,
                                           mlbvh_node_index* dRootNode, mlbvh_aabb* dSceneAABB, void* stream);

/* The higher-quality build: the counterpart of BVHCPUBuilder::buildByEmbree
 * (minimum_lbvh.h:594-656, Embree's SAH builder with one triangle per leaf
 * written into the same InternalNode array). Parallel locally-ordered
 * clustering over the Morton order of mlbvh_build (same keys, buildOption
 * included): each cluster merges with its nearest neighbour, by the area of
 * the union box, among the `radius` clusters on either side (1-32; 8 is a
 * good default) when that choice is mutual, until one cluster remains. The
 * output has mlbvh_build's form exactly: n - 1 nodes numbered in in-order (a
 * left leaf child of node j is leaf j of the in-order, a right one leaf
 * j + 1), parent links, the root's parent invalid, context the escape index
 * of intersect_escape_link, so every walk and every other entry point takes
 * it. Its boxes cost less to traverse (a smaller surface-area sum) at a
 * longer build. One cooperative launch after the sort (it can be captured in
 * a CUDA graph); needs mlbvh_build_ploc_scratch_bytes(n) bytes of scratch;
 * timeouts are reported by mlbvh_scratch_status like mlbvh_build's. */
MLBVH_API size_t mlbvh_build_ploc_scratch_bytes(uint32_t nTriangles);
MLBVH_API mlbvh_status mlbvh_build_ploc(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption,
                                        int radius, mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode,
                                        mlbvh_aabb* dSceneAABB, void* dScratch, size_t scratchBytes, void* stream);

/* Test hook: the number of polls after which a bounded device wait of the
 * builds that this host thread starts afterwards (mlbvh_build, _ex, _ploc,
 * _noalloc) gives up; 0 restores each build's default (a second or so). A wait that
 * gives up sets the build's error word and the build ends without hanging
 * (its output is then unusable); mlbvh_scratch_status reports it. Lets tests
 * make a wait run out without a device fault. */
MLBVH_API void mlbvh_set_spin_limit(uint32_t polls);

/* Synchronises `stream`, then reports MLBVH_ERR_TIMEOUT if a bounded wait of
 * the last build that used dScratch gave up (its output is then unusable),
 * else MLBVH_OK. dScratch = NULL asks the same of the last
 * mlbvh_build_noalloc on the current device (its built-in scratch);
 * MLBVH_ERR_INVALID_ARG when there was none in the current context. */
MLBVH_API mlbvh_status mlbvh_scratch_status(const void* dScratch, void* stream);

/* ---------------------------------------------------------------- query ---
 * Replaces the per-ray calls of intersect_stackfree / intersect_escape_link /
 * intersect_stackfull (minimum_lbvh.h:981, 1063, 912) with one launch over
 * nRays rays. hits[i] follows minimum_lbvh::Hit; for RAY_QUERY_ANY the first
 * hit found stops the ray. The stackful traversal has no any-hit mode in the
 * reference and answers closest hits. */
MLBVH_API mlbvh_status mlbvh_trace(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                         const mlbvh_triangle* dTriangles, const mlbvh_ray* dRays, mlbvh_hit* dHits,
                         uint32_t nRays, int rayQuery, int traversal, void* stream);

/* ------------------------------------------------------- quantised form ---
 * No reference counterpart. mlbvh_quantise converts a tree built by
 * mlbvh_build (same topology) into 32-byte nodes with 8-bit child boxes
 * rounded outward, a parent array and leaf-ordered triangles:
 * dQNodes nTriangles-1 entries, dQParents nTriangles-1, dQTris nTriangles,
 * one dQHeader. 1 <= nTriangles <= 2^23. The triangle test stays FP32 and
 * identical, so closest hits equal the FP32 tree's except where two triangles
 * return bit-identical t (the later-visited wins in both). */
MLBVH_API mlbvh_status mlbvh_quantise(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                                      const mlbvh_triangle* dTriangles, uint32_t nTriangles, mlbvh_qnode* dQNodes,
                                      uint32_t* dQParents, mlbvh_qtri* dQTris, mlbvh_qheader* dQHeader, void* stream);
/* mlbvh_trace over the quantised tree. The walk visits leaves in the order
 * of intersect_stackfree's state machine; a 16-entry stack of pending far
 * children per ray replaces its revisits (same Hit records, fewer node loads). */
MLBVH_API mlbvh_status mlbvh_trace_quantised(const mlbvh_qnode* dQNodes, const uint32_t* dQParents,
                                             const mlbvh_qtri* dQTris, const mlbvh_qheader* dQHeader,
                                             const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays, int rayQuery,
                                             void* stream);
/* mlbvh_trace_quantised with the walk chosen: stackDepth 0 = the stack-free
 * walk (parent loads instead of a stack), 1, 4 or 16 = that many stack entries
 * per ray (a full stack hands over to the stack-free walk). All give the same
 * Hit records. dCounts (may be NULL; 3 * nRays words, nRays < 2^30) receives
 * per ray the internal-node visits, triangle tests and parent loads at
 * [i], [nRays + i], [2 nRays + i]. */
MLBVH_API mlbvh_status mlbvh_trace_quantised_ex(const mlbvh_qnode* dQNodes, const uint32_t* dQParents,
                                                const mlbvh_qtri* dQTris, const mlbvh_qheader* dQHeader,
                                                const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays,
                                                int rayQuery, int stackDepth, uint32_t* dCounts, void* stream);
/* mlbvh_render_ao over the quantised tree; same arguments otherwise. */
MLBVH_API mlbvh_status mlbvh_render_ao_quantised(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                                 const mlbvh_ray_generator* camera, const mlbvh_qnode* dQNodes,
                                                 const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                                 const mlbvh_qheader* dQHeader, int useSobol, int nSamples,
                                                 float radius, uint32_t sobolSeed, unsigned long long* dStats,
                                                 void* dScratch, size_t scratchBytes, void* stream);

/* --------------------------------------------------------- batched form ---
 * No reference counterpart (the reference builds one mesh per
 * BVHGPUBuilder::build call). Many independent meshes of uneven size, laid
 * out back to back, are built by one launch chain, and a batch of rays, each
 * aimed at one mesh, is drained by one persistent work-queue kernel.
 *
 * Layout: mesh m owns triangles [o[m], o[m+1]) of dTriangles (o =
 * dMeshTriangleOffsets, nMeshes + 1 device words, o[0] = 0, o[nMeshes] =
 * nTriangles, every mesh at least one triangle), internal nodes
 * [o[m] - m, o[m+1] - m - 1) of dInternals (nTriangles - nMeshes nodes in
 * all), and dRootNodes[m]. Node and leaf indices inside a tree are local to
 * its mesh, and every tree is bit-identical to mlbvh_build of that mesh alone.
 * Rays [r[m], r[m+1]) of dRays (r = dMeshRayOffsets, nondecreasing, r[0] = 0,
 * r[nMeshes] = nRays) query mesh m; dHits[i] is ray i's hit as mlbvh_trace
 * writes it, with the triangle index local to the mesh.
 * Bad triangle offsets are detected on the device: nothing is built or
 * traced, and mlbvh_scratch_status(dScratch) reports MLBVH_ERR_INVALID_ARG. */
typedef struct mlbvh_batch {
    const mlbvh_triangle* dTriangles;
    const uint32_t* dMeshTriangleOffsets;
    uint32_t nMeshes;    /* 1 .. 2^20 */
    uint32_t nTriangles; /* nMeshes .. 2^30 - 1 */
    uint32_t buildOption;
    int rayQuery;        /* MLBVH_RAY_QUERY_CLOSEST or _ANY */
    mlbvh_internal_node* dInternals;
    mlbvh_node_index* dRootNodes;
    mlbvh_aabb* dMeshAABBs; /* nMeshes, may be NULL */
    const mlbvh_ray* dRays;
    const uint32_t* dMeshRayOffsets;
    uint32_t nRays;         /* below 2^31 */
    uint32_t _pad;
    mlbvh_hit* dHits;
    void* dScratch;         /* mlbvh_batch_scratch_bytes(nMeshes, nTriangles); build and trace of one batch share it */
    size_t scratchBytes;
} mlbvh_batch;

/* Launch parameters, chosen by mlbvh_batch_autotune; results do not depend
 * on them (only the time does). */
typedef struct mlbvh_batch_params {
    int digitBits;   /* radix digit width of the build's sort: 8 (4 passes) or 11 (3 passes) */
    int traceBlock;  /* threads per CTA of the traversal kernel: 64, 128, 256 or 512 */
    int queueChunk;  /* rays a warp takes from the queue per atomic: 1 .. 65536 */
    int refillLanes; /* idle lanes of a warp that trigger taking more rays: 1 .. 32 */
    int walk;        /* 0: intersect_stackfree's walk; 1: the replay walk (same Hit records, fewer node loads) */
} mlbvh_batch_params;

typedef struct mlbvh_batch_graph mlbvh_batch_graph; /* opaque */

MLBVH_API size_t mlbvh_batch_scratch_bytes(uint32_t nMeshes, uint32_t nTriangles);
/* Defaults: 8-bit digits, 128 threads, chunks of 64 rays, refill at 8 idle lanes, replay walk. */
MLBVH_API void mlbvh_batch_params_default(mlbvh_batch_params* params);
/* Builds every mesh's tree (params may be NULL: the defaults). */
MLBVH_API mlbvh_status mlbvh_build_batched(const mlbvh_batch* batch, const mlbvh_batch_params* params, void* stream);
/* Traces every ray against its mesh's tree (built by mlbvh_build_batched with
 * the same dScratch, whose header it reads). */
MLBVH_API mlbvh_status mlbvh_trace_batched(const mlbvh_batch* batch, const mlbvh_batch_params* params, void* stream);
/* Times candidate parameters on this batch (the digit width on the build,
 * then walk, block size, queue chunk and refill threshold on the traversal, one at
 * a time) and writes the fastest to *params; *buildMs / *traceMs (may be
 * NULL) receive their median times. Runs the build and the traversal many
 * times, overwriting the outputs, and synchronises `stream`. */
MLBVH_API mlbvh_status mlbvh_batch_autotune(const mlbvh_batch* batch, mlbvh_batch_params* params, float* buildMs,
                                            float* traceMs, void* stream);
/* Captures the build (stages = 1), the traversal (2) or both (3) of this
 * batch into a CUDA graph. The graph keeps the batch's pointers and sizes;
 * each launch reads the buffers' contents at that time, so new triangles or
 * rays of the same sizes need no new capture. */
MLBVH_API mlbvh_status mlbvh_batch_graph_create(const mlbvh_batch* batch, const mlbvh_batch_params* params,
                                                int stages, mlbvh_batch_graph** graph);
MLBVH_API mlbvh_status mlbvh_batch_graph_launch(mlbvh_batch_graph* graph, void* stream);
MLBVH_API void mlbvh_batch_graph_destroy(mlbvh_batch_graph* graph);

/* --------------------------------------------------------------- shading ---
 * The reference's shading kernels (main_gpu.cu), one launch chain each.
 * `camera` is a HOST pointer (passed by value to the kernels, as the
 * reference passes RayGenerator). Pixels are packed RGBA8 as packRGBA writes
 * them (main_gpu.cu:17-22). */

/* normal (main_gpu.cu:84-109) */
MLBVH_API mlbvh_status mlbvh_render_normal(uint32_t* dPixels, int width, int height, const mlbvh_ray_generator* camera,
                                 const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                                 const mlbvh_triangle* dTriangles, void* stream);

/* ao (main_gpu.cu:111-177) with the sample count, AO ray length and the Sobol
 * scramble seed as parameters (the reference fixes 16, 1.0f and 12345).
 * dOccluded (may be NULL) receives per pixel the number of AO rays that hit
 * something, or 0xFFFFFFFF where the primary ray missed; linear AO is
 * dOccluded / nSamples. The sample directions use this library's FP32 sincos
 * instead of CUDA's cosf/sinf, so that the host oracle can reproduce them bit
 * for bit. dScratch holds mlbvh_render_scratch_bytes(width, height) bytes.
 * dStats (may be NULL; 8 device uint64) receives {rays traced (primary + AO),
 * internal-node visits, triangle tests, the AO rays' share of those visits,
 * the AO rays' share of those tests, parent-word loads (quantised tree only),
 * the AO rays' share of those, 0}; counting runs a slower kernel variant, so
 * leave it NULL when timing. */
MLBVH_API size_t mlbvh_render_scratch_bytes(int width, int height);
MLBVH_API mlbvh_status mlbvh_render_ao(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                             const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                             const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                             int useSobol, int nSamples, float radius, uint32_t sobolSeed,
                             unsigned long long* dStats, void* dScratch, size_t scratchBytes, void* stream);

/* mlbvh_render_ao with the walk of its rays chosen: MLBVH_TRAVERSAL_STACKFREE
 * (what mlbvh_render_ao runs) or MLBVH_TRAVERSAL_REPLAY (the same occlusion
 * counts and pixels from fewer node loads; primary rays too). With REPLAY,
 * dLeafTriangles (may be NULL) is the tree's triangles in leaf order from
 * mlbvh_leaf_triangles: 16-byte aligned records read with three vector loads
 * instead of nine scalar ones, same results. No reference counterpart. With
 * dStats, node visits are those of the chosen walk. */
MLBVH_API mlbvh_status mlbvh_render_ao_ex(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                          const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                          const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                          int useSobol, int nSamples, float radius, uint32_t sobolSeed, int traversal,
                                          const mlbvh_qtri* dLeafTriangles, unsigned long long* dStats,
                                          void* dScratch, size_t scratchBytes, void* stream);
/* The triangles of a built tree in leaf (sorted) order as 48-byte mlbvh_qtri
 * records (corners and original index), nTriangles of them: leaf j is the
 * left leaf child of internal node j or the right leaf child of node j - 1.
 * The same array mlbvh_quantise writes. No reference counterpart. */
MLBVH_API mlbvh_status mlbvh_leaf_triangles(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                                            const mlbvh_triangle* dTriangles, uint32_t nTriangles,
                                            mlbvh_qtri* dLeafTriangles, void* stream);

/* The 4-wide tree of a built tree: nTriangles - 1 mlbvh_wnode slots (none
 * for one triangle), 128-byte aligned. No reference counterpart. */
MLBVH_API mlbvh_status mlbvh_build_wide(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                                        uint32_t nTriangles, mlbvh_wnode* dWideNodes, void* stream);
/* Rays over the 4-wide tree, one thread per ray. MLBVH_RAY_QUERY_ANY: a ray
 * has a hit exactly when mlbvh_trace's any-hit walk finds one; the Hit record
 * is that of the first triangle this walk finds (the reference's walk may
 * stop at another one). MLBVH_RAY_QUERY_CLOSEST: children are entered nearest
 * first and pending ones skipped once beyond hit.t; the Hit record is
 * intersect_stackfree's, except that where two triangles meet the ray at
 * bit-identical t either may report. dLeafTriangles from
 * mlbvh_leaf_triangles. A ray whose stack (24 entries) would overflow
 * continues with the stack-free walk over dInternals / dTriangles, keeping
 * its hit. dCounts (may be NULL; 3 * nRays words,
 * nRays < 2^30) receives per ray the node visits (wide nodes, then binary
 * nodes after a restart), triangle tests and restarts at [i], [nRays + i],
 * [2 nRays + i]. */
MLBVH_API mlbvh_status mlbvh_trace_wide(const mlbvh_wnode* dWideNodes, const mlbvh_internal_node* dInternals,
                                        const mlbvh_node_index* dRootNode, const mlbvh_triangle* dTriangles,
                                        const mlbvh_qtri* dLeafTriangles, const mlbvh_ray* dRays, mlbvh_hit* dHits,
                                        uint32_t nRays, int rayQuery, uint32_t* dCounts, void* stream);
/* The quantised slots of a 4-wide tree: nTriangles - 1 mlbvh_qwnode (none for
 * one triangle), 32-byte aligned, from the FP32 slots of mlbvh_build_wide.
 * *dStatus (one device word) becomes 0 when every slot was quantised, 1 when
 * one could not be (non-finite planes, or coordinates beyond about 1e18); the
 * quantised walks then take the stack-free walk over the binary tree for
 * every ray (the same answers, slower). No reference counterpart. */
MLBVH_API mlbvh_status mlbvh_quantise_wide(const mlbvh_wnode* dWideNodes, uint32_t nTriangles,
                                           mlbvh_qwnode* dQWideNodes, uint32_t* dStatus, void* stream);
/* mlbvh_trace_wide over the quantised slots (either query; a hit counts only
 * where the triangle's exact box passes the slab test as well, so the answers
 * are mlbvh_trace_wide's). A ray with a direction component of magnitude
 * below 2^-62 (the reference clamps its inverse to +-FLT_MAX) or an origin
 * coordinate of 2^62 or more takes the stack-free walk over dInternals
 * instead, as every ray does when *dStatus is set. */
MLBVH_API mlbvh_status mlbvh_trace_wide_quantised(const mlbvh_qwnode* dQWideNodes, const uint32_t* dStatus,
                                                  const mlbvh_internal_node* dInternals,
                                                  const mlbvh_node_index* dRootNode, const mlbvh_triangle* dTriangles,
                                                  const mlbvh_qtri* dLeafTriangles, const mlbvh_ray* dRays,
                                                  mlbvh_hit* dHits, uint32_t nRays, int rayQuery, uint32_t* dCounts,
                                                  void* stream);
/* mlbvh_render_ao_wide over the quantised slots (the same occlusion counts). */
MLBVH_API mlbvh_status mlbvh_render_ao_wide_quantised(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                                      const mlbvh_ray_generator* camera,
                                                      const mlbvh_node_index* dRootNode,
                                                      const mlbvh_internal_node* dInternals,
                                                      const mlbvh_triangle* dTriangles,
                                                      const mlbvh_qwnode* dQWideNodes, const uint32_t* dStatus,
                                                      const mlbvh_qtri* dLeafTriangles, int useSobol, int nSamples,
                                                      float radius, uint32_t sobolSeed, unsigned long long* dStats,
                                                      void* dScratch, size_t scratchBytes, void* stream);
/* mlbvh_render_ao with the AO rays over the 4-wide tree (any-hit, so every
 * occlusion count is mlbvh_render_ao's) and the primary rays on the replay
 * walk over the binary tree (the stack-free walk's Hit records). AO rays of a
 * pixel start at the deepest wide node whose subtree holds every leaf within
 * their reach. With dStats, node visits count wide nodes for AO rays. */
MLBVH_API mlbvh_status mlbvh_render_ao_wide(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                            const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                            const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                            const mlbvh_wnode* dWideNodes, const mlbvh_qtri* dLeafTriangles,
                                            int useSobol, int nSamples, float radius, uint32_t sobolSeed,
                                            unsigned long long* dStats, void* dScratch, size_t scratchBytes,
                                            void* stream);

/* One progressive path-tracing pass (pt, main_gpu.cu:179-272): reads and
 * updates dAccumulators (float4 per pixel, w = samples so far). maxDepth is
 * the bounce limit (the reference uses 1024). */
MLBVH_API mlbvh_status mlbvh_render_pt(float* dAccumulators, int width, int height, const mlbvh_ray_generator* camera,
                             const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                             const mlbvh_triangle* dTriangles, const mlbvh_triangle_attrib* dAttribs,
                             int useSobol, int maxSPP, int maxDepth, void* stream);
/* mlbvh_render_pt with the walk of its closest-hit rays chosen:
 * MLBVH_TRAVERSAL_STACKFREE (what mlbvh_render_pt runs) or
 * MLBVH_TRAVERSAL_REPLAY (the same Hit records, so the same accumulators,
 * from fewer node loads; dLeafTriangles from mlbvh_leaf_triangles may be
 * NULL). No reference counterpart. */
MLBVH_API mlbvh_status mlbvh_render_pt_ex(float* dAccumulators, int width, int height,
                                          const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                          const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                          const mlbvh_triangle_attrib* dAttribs, int useSobol, int maxSPP,
                                          int maxDepth, int traversal, const mlbvh_qtri* dLeafTriangles,
                                          void* stream);

/* ------------------------------------------------ differentiable path trace ---
 * No reference counterpart (the reference's pt, main_gpu.cu:179-272, is not
 * differentiable). A fixed-depth, Russian-roulette-free variant of pt with
 * grey per-triangle albedo dAlbedo[t] and emission dEmission[t]:
 *   I_p = 1/spp sum_s sum_{d=0..bounces} e(t_d) prod_{j<d} a(t_j)
 * over spp Owen-Sobol paths per pixel (dimension 0 jitters the pixel,
 * dimension 1 + d samples bounce d). mlbvh_pt_diff_render writes the float
 * image; mlbvh_pt_diff_adjoint ADDS dLoss/dAlbedo to dGradAlbedo (zero it
 * first) given dLoss/dImage, by replaying every path from its sample index
 * instead of storing it (path replay). 0 <= bounces <= 8. */
MLBVH_API mlbvh_status mlbvh_pt_diff_render(float* dImage, int width, int height, int spp, int bounces,
                                            const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                            const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                            const float* dAlbedo, const float* dEmission, void* stream);
MLBVH_API mlbvh_status mlbvh_pt_diff_adjoint(float* dGradAlbedo, const float* dGradImage, int width, int height,
                                             int spp, int bounces, const mlbvh_ray_generator* camera,
                                             const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                                             const mlbvh_triangle* dTriangles, const float* dAlbedo,
                                             const float* dEmission, void* stream);

/* pack (main_gpu.cu:273-286): accumulator / spp, gamma 1/2.2, RGBA8. */
MLBVH_API mlbvh_status mlbvh_pack(uint32_t* dPixels, const float* dAccumulators, int n, void* stream);

/* ------------------------------------------------------------ OBJ scenes ---
 * A host-side OBJ / MTL reader giving the path tracer's input as the
 * reference's scene loop does (main_gpu.cpp:209-282, over a third-party OBJ
 * library there): one triangle and one TriangleAttrib per triangle, with the
 * corner normals, reflectance = the material's Kd, emissive = its Ke, or
 * reflectance 0.5 and no emission without a material. Quads are split along
 * the shorter diagonal, larger faces into fans. The mesh lives in host memory
 * until mlbvh_obj_free; copy the arrays to the device for mlbvh_build and
 * mlbvh_render_pt. Errors: MLBVH_ERR_INVALID_ARG (file missing, bad corner). */
typedef struct mlbvh_obj_mesh mlbvh_obj_mesh; /* opaque */
MLBVH_API mlbvh_status mlbvh_obj_load(const char* path, mlbvh_obj_mesh** mesh);
MLBVH_API uint32_t mlbvh_obj_triangle_count(const mlbvh_obj_mesh* mesh);
MLBVH_API const mlbvh_triangle* mlbvh_obj_triangles(const mlbvh_obj_mesh* mesh);
MLBVH_API const mlbvh_triangle_attrib* mlbvh_obj_attribs(const mlbvh_obj_mesh* mesh);
MLBVH_API void mlbvh_obj_free(mlbvh_obj_mesh* mesh);

/* Profiling hook (no reference counterpart; the reference times whole calls
 * with its DeviceStopwatch, minimum_lbvh.h:693-724): the next mlbvh_render_ao,
 * mlbvh_build or mlbvh_build_batched on this host thread records the two
 * cudaEvent_t handles around its dominant kernel (the AO-ray kernel, resp. the
 * agglomerative build kernel). NULL, NULL cancels. */
MLBVH_API void mlbvh_profile_events(void* startEvent, void* stopEvent);

/* Measurement hook (no reference counterpart): one launch that reads dBuffer
 * with the traversal kernels' node load (32 bytes per instruction through L1
 * and L2), so that CUDA events around it give the bandwidth such loads reach
 * from where the buffer lives (tens of MB: L2; GBs: HBM). pattern 0 streams:
 * consecutive threads read consecutive 32-byte sectors, `loads` sweeps over
 * the buffer; pattern 1 gathers: each thread makes `loads` (a multiple of 8)
 * loads of pseudo-random sectors (bytes must then be 32 * 2^k). *bytesRead
 * (host) receives the bytes the launch reads. dSink: 1024 device words that
 * keep the loads from being optimised away (practically never written).
 * bytes: a multiple of 32, at least 32 KiB; dBuffer 32-byte aligned. */
MLBVH_API mlbvh_status mlbvh_read_probe(const void* dBuffer, size_t bytes, int pattern, uint32_t loads,
                                        uint32_t* dSink, size_t* bytesRead, void* stream);

/* RayGenerator::lookat (camera.h:10-22), on the host. */
MLBVH_API mlbvh_status mlbvh_camera_lookat(mlbvh_ray_generator* out, const float eye[3], const float center[3],
                                 const float up[3], float fovy, int width, int height);

#ifdef __cplusplus
}
#endif
#endif /* MLBVH_H */
