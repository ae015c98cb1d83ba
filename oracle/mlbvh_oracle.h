/* Test infrastructure only — the oracle (checker) for the MinimumLBVH hot path.
 *
 * A plain-C restatement of the reference's CPU algorithm, used by tests/,
 * __graft_entry__.smoke() and the CPU-baseline legs of bench.py as the thing
 * GPU results are compared against. The product never links it.
 *
 * Pinned against the reference itself: tests/test_oracle_pin.py runs the same
 * inputs through oracle/_ref/libmlbvh_ref.so (the reference's own sources
 * compiled by oracle/Makefile) and through the committed fixtures in
 * tests/golden/ (generated from that library by tests/golden/gen_golden.py).
 *
 * Layouts are the reference's (minimum_lbvh.h:207-282, 502-506, 890-896):
 *   Triangle 36 B, AABB 24 B, NodeIndex 4 B (31-bit index, leaf bit 31),
 *   InternalNode 64 B, Hit 32 B (t@0 uv@8 ng@16 triangleIndex@28),
 *   RayGenerator 36 B (camera.h:5-8), TriangleAttrib 60 B (main_gpu.cu:10-15).
 */
#ifndef MLBVH_ORACLE_H
#define MLBVH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y, z; } orc_f3;
typedef struct { orc_f3 v[3]; } orc_triangle;
typedef struct { orc_f3 lower, upper; } orc_aabb;
typedef struct {
    uint32_t children[2];
    orc_aabb aabbs[2];
    uint32_t parent;
    uint32_t context;
} orc_node;
typedef struct {
    float t;
    uint32_t pad;
    float u, v;
    orc_f3 ng;
    uint32_t triangleIndex;
} orc_hit;
typedef struct { orc_f3 origin, right, up; } orc_camera;
typedef struct {
    float ro[3];
    float tmin;
    float rd[3];
    float tmax;
} orc_ray;

/* Trigonometry used for the cosine-weighted hemisphere sample:
 * ORC_TRIG_LIBM is the reference's cosf/sinf (main_gpu.cu:30-31);
 * ORC_TRIG_PORTABLE is the project's own FP32 sincos that the CUDA kernels
 * also use, so that GPU and oracle agree bit for bit. */
enum { ORC_TRIG_LIBM = 0, ORC_TRIG_PORTABLE = 1 };

int orc_version(void);
void orc_set_threads(int n);

/* minimum_lbvh.h:99-147, 149-195 */
int orc_clz(uint32_t x);
int orc_clz64(uint64_t x);
int orc_ffs(uint32_t x);
int orc_ffs64(uint64_t x);
int orc_delta(uint32_t a, uint32_t b);
uint64_t orc_splat3(uint32_t a);
uint32_t orc_compact3(uint64_t m);
uint64_t orc_encode_morton(uint32_t x, uint32_t y, uint32_t z);
uint64_t orc_encode_morton_naive(uint32_t x, uint32_t y, uint32_t z);
void orc_decode_morton(uint64_t m, uint32_t* x, uint32_t* y, uint32_t* z);
uint64_t orc_aabb_morton(const orc_aabb* box, orc_f3 p);

/* Build (minimum_lbvh.h:512-592, stable key order) */
void orc_scene_aabb(const orc_triangle* tris, uint32_t n, orc_aabb* out);
void orc_morton_keys(const orc_triangle* tris, uint32_t n, uint32_t option,
                     const orc_aabb* scene, uint32_t* keys);
void orc_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n);
int orc_build(const orc_triangle* tris, uint32_t n, uint32_t option,
              orc_node* nodes, uint8_t* deltas, uint32_t* root,
              uint32_t* keys_out, uint32_t* indices_out, orc_aabb* scene_out);
int orc_build_from_keys(const uint32_t* sorted_keys, const uint32_t* sorted_indices,
                        const orc_triangle* tris, uint32_t n,
                        orc_node* nodes, uint8_t* deltas, uint32_t* root);
int orc_validate(const orc_node* nodes, const uint8_t* deltas, uint32_t n, uint32_t root, int maxDelta);
/* The higher-quality builder (csrc/ploc.cu; the reference's is Embree's SAH
 * build behind the same InternalNode array, minimum_lbvh.h:594-656):
 * parallel locally-ordered clustering over orc_build's sorted order with
 * neighbourhood radius `radius`, nodes numbered in in-order. Returns the
 * number of clustering iterations (0 for n == 1), negative on bad input. */
int orc_build_ploc(const orc_triangle* tris, uint32_t n, uint32_t option, int radius, orc_node* nodes,
                   uint32_t* root);
/* Surface-area cost of a tree: sum over internal nodes of their box's
 * half area plus, over leaves, that of their box, each over the root box's
 * half area (unit costs for a node visit and a triangle test). */
double orc_sah_cost(const orc_node* nodes, uint32_t n, uint32_t root);
int orc_check_tree(const orc_node* nodes, const orc_triangle* tris, uint32_t n, uint32_t root);

/* Queries (minimum_lbvh.h:898-1137); mode 0 stack-free, 1 escape-link,
 * 2 stackful. counters (nullable) receive per-ray node visits, triangle tests. */
void orc_trace(const orc_node* nodes, const orc_triangle* tris, uint32_t root,
               const orc_ray* rays, uint32_t nRays, int query, int mode,
               orc_hit* hits, uint32_t* nodeVisits, uint32_t* triTests);
/* The replay walk (stackfree_replay_step): intersect_stackfree's hits with a
 * stack of `depth` (1..64) pending far children instead of revisits. mode 3
 * of orc_trace is this walk with 16 entries. */
void orc_trace_replay(const orc_node* nodes, const orc_triangle* tris, uint32_t root, const orc_ray* rays,
                      uint32_t nRays, int query, int depth, orc_hit* hits, uint32_t* nodeVisits, uint32_t* triTests);

/* The 4-wide tree (no reference counterpart; csrc/wide.cu): 32 words per
 * slot, n - 1 slots. orc_trace_wide: any-hit (query 1) or closest-hit
 * (query 0) rays over it (restarting with the stack-free walk where its
 * 24-entry stack would overflow); per ray the wide-node (then binary-node)
 * visits, triangle tests and restarts. */
void orc_build_wide(const orc_node* nodes, uint32_t n, uint32_t* out);
void orc_trace_wide(const uint32_t* wide, const orc_node* nodes, const orc_triangle* tris, uint32_t n, uint32_t root,
                    const orc_ray* rays, uint32_t nRays, orc_hit* hits, uint32_t* visits, uint32_t* tests,
                    uint32_t* restarts, int query);
/* Quantised slots (16 words each; csrc/wide.cu): returns 1 when every slot
 * was quantised. orc_trace_wide_quantised walks them (a hit counts only where
 * the triangle's exact box passes too); fallback != 0: the stack-free walk
 * for every ray, as the kernels do when a slot could not be quantised. */
int orc_quantise_wide(const uint32_t* wide, uint32_t n, uint32_t* out);
/* a * b + c rounded once, down (up = 0) or up (up = 1): the emulation of
 * __fmaf_rd / __fmaf_ru the quantised walks use (exported for its test). */
float orc_fma_dir(float a, float b, float c, int up);
void orc_trace_wide_quantised(const uint32_t* qwide, int fallback, const orc_node* nodes, const orc_triangle* tris,
                              uint32_t n, uint32_t root, const orc_ray* rays, uint32_t nRays, orc_hit* hits,
                              uint32_t* visits, uint32_t* tests, uint32_t* restarts, int query);

/* Camera (camera.h:10-31) */
void orc_lookat(orc_f3 eye, orc_f3 center, orc_f3 up, float fovy, int w, int h, orc_camera* cam);
void orc_shoot(const orc_camera* cam, float u, float v, orc_f3* ro, orc_f3* rd);

/* Samples (sobol.h:18-129, main_gpu.cu:24-82) */
void orc_sobol(uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2, float* x, float* y);
uint32_t orc_hash_pcg(uint32_t v);
void orc_sincos(float phi, float* s, float* c);

/* Sample streams: useSobol 1 = Owen-scrambled Sobol (sobol.h:119); 0 = PCG32
 * with the first draw of each pair as x, the order the CUDA kernels use; 2 =
 * PCG32 with the second draw as x, the order g++ gives the reference's
 * make_float2(rng.uniformf(), rng.uniformf()) (C++ leaves it unspecified).
 *
 * AO (main_gpu.cu:111-177) with sample count, radius and Sobol seed as
 * parameters. occluded[pixel] = number of AO rays that hit (0xFFFFFFFF where
 * the primary ray missed); pixels = packed RGBA8 as the reference writes it.
 * Counters (nullable, 2 entries) accumulate node visits and triangle tests
 * over all rays; nRays receives primary + AO ray count. */
void orc_render_ao(uint32_t* pixels, uint32_t* occluded, int w, int h, const orc_camera* cam,
                   uint32_t root, const orc_node* nodes, const orc_triangle* tris,
                   int useSobol, int nSamples, float radius, uint32_t seed, int trig,
                   int rowBegin, int rowEnd, uint64_t* counters);

/* One progressive path-tracing pass (main_gpu.cu:179-272) and pack (:273-286). */
void orc_render_pt(float* accum4, int w, int h, const orc_camera* cam, uint32_t root,
                   const orc_node* nodes, const orc_triangle* tris, const float* attribs15,
                   int useSobol, int maxSPP, int maxDepth, int trig);
void orc_pack(uint32_t* pixels, const float* accum4, int n);
void orc_render_normal(uint32_t* pixels, int w, int h, const orc_camera* cam, uint32_t root,
                       const orc_node* nodes, const orc_triangle* tris);

/* Quantised tree (no reference counterpart): the conversion and traversal of
 * csrc/quantise.cu and the device header, word for word. qnodes 8 words per
 * internal node, parents 1, qtris 12 words per leaf, header 4 words. */
int orc_quantise(const orc_node* nodes, uint32_t root, const orc_triangle* tris, uint32_t n,
                 uint32_t* qnodes, uint32_t* parents, uint32_t* qtris, uint32_t* header);
int orc_check_quantised(const orc_node* nodes, uint32_t n, const uint32_t* qnodes, const uint32_t* header);
void orc_trace_quantised(const uint32_t* qnodes, const uint32_t* parents, const uint32_t* qtris, const uint32_t* header,
                         const orc_ray* rays, uint32_t nRays, int query, orc_hit* hits, uint32_t* visits,
                         uint32_t* tests, uint32_t* ups);
/* The quantised walk with a stack of stackDepth (1..64) pending far children
 * replacing the revisits (quantised_replay_step); same hits as
 * orc_trace_quantised, fewer node visits. */
void orc_trace_quantised_replay(const uint32_t* qnodes, const uint32_t* parents, const uint32_t* qtris,
                                const uint32_t* header, const orc_ray* rays, uint32_t nRays, int query, int stackDepth,
                                orc_hit* hits, uint32_t* visits, uint32_t* tests, uint32_t* ups);

/* Differentiable path tracing (no reference counterpart): the render and
 * path-replay adjoint of csrc/adjoint.cu. image32 (nullable) is the kernel's
 * FP32 image bit for bit; image64 (nullable) and the adjoint accumulate in
 * FP64 over the same FP32 path geometry. */
void orc_pt_diff_render(float* image32, double* image64, int w, int h, int spp, int bounces, const orc_camera* cam,
                        uint32_t root, const orc_node* nodes, const orc_triangle* tris, const float* albedo32,
                        const float* emission32, const double* albedo64, const double* emission64);
void orc_pt_diff_adjoint(double* grad, const double* gradImage, int w, int h, int spp, int bounces,
                         const orc_camera* cam, uint32_t root, const orc_node* nodes, const orc_triangle* tris,
                         const double* albedo64, const double* emission64);

#ifdef __cplusplus
}
#endif
#endif
