// Differentiable path tracing with a path-replay adjoint (no reference
// counterpart): the gradient of an image loss with respect to per-triangle
// albedo, for the fixed-depth, Russian-roulette-free estimator
//
//   I_p = 1/spp * sum_s L(path_s),   L = sum_{d=0..B} e(t_d) * prod_{j<d} a(t_j)
//
// where t_0 is the primary hit, t_1..t_B the hits after B cosine-sampled
// bounces, e the per-triangle emission and a the per-triangle (grey) albedo.
// Path geometry is that of pt (main_gpu.cu:179-272): Owen-Sobol sample
// streams (dimension 0 for the pixel jitter, 1 + d for bounce d), normals
// facing the incoming ray, origin offset n * 1e-4, Lambertian bounce whose
// cosine/pdf cancels so the throughput is multiplied by the albedo.
//
// The adjoint replays every path from its sample index (paths are never
// stored; Vicini et al., "Path Replay Backpropagation", 2021): with c_d the
// radiance collected at vertex d, dL/da(t_j) = (sum_{d>j} c_d) / a(t_j), and
// grad[t_j] += dLoss/dI_p / spp * that, scattered with atomic adds.
#include "capi_internal.h"
#include "../../include/mlbvh_device.cuh"

namespace mlbvh {

namespace {

// Threads per CTA: one pixel's warp (measured forward / adjoint ms: 22.6 / 18.0
// against 22.6 / 18.3 for 64 and 22.7 / 19.1 for 128, where a CTA holds its
// slot until its slowest pixel is done); compiled for 768 threads per SM (80
// registers). Build-time override for sweeps: -DMLBVH_DIFF_THREADS.
#ifndef MLBVH_DIFF_THREADS
#define MLBVH_DIFF_THREADS 32
#endif
constexpr int kDiffThreads = MLBVH_DIFF_THREADS;
constexpr int kMaxBounces = 8;
// Lanes per pixel: one warp per pixel, lane l tracing samples l, l + 32, ...
// in order; the render adds the lanes' partial sums as a pairwise tree in lane
// order ((p0 + p1) + (p2 + p3)) + ... . Measured on the differentiation
// workload (forward / adjoint ms): one thread per pixel 35.3 / 32.3 (2.3 waves
// of long CTAs, the last on a third of the SMs), 2 lanes 30.1 / 27.1, 4 lanes
// 26.5 / 23.3, 8 lanes 24.4 / 21.0, 16 lanes 23.2 / 19.6, 32 lanes 22.7 / 18.3:
// a pixel's samples start from nearby rays, so its warp walks the same nodes.
// (Build-time override for sweeps: -DMLBVH_DIFF_LANES=2, 4, 8 or 16.)
#ifndef MLBVH_DIFF_LANES
#define MLBVH_DIFF_LANES 32
#endif
constexpr int kLanesPerPixel = MLBVH_DIFF_LANES;
static_assert(kDiffThreads % kLanesPerPixel == 0, "a pixel's lanes share a warp");
constexpr int kDiffStack = 16;  // replay-walk stack entries per thread (shared memory)

// intersect_stackfree's closest hit (minimum_lbvh.h:981-1061) through the
// replay walk (stackfree_replay_step): the same Hit record, ties included,
// with every internal node loaded once. `stack` is this thread's column of a
// kDiffStack x kDiffThreads shared-memory array.
__device__ __forceinline__ void trace_closest(HitRecord& hit, const mlbvh_internal_node* __restrict__ nodes,
                                              const float* __restrict__ tris, uint32_t root, f3 ro, f3 rd,
                                              uint2* stack)
{
    const f3 inv = inv_rd(rd);
    uint32_t curr = root, prev = kInvalid, nv = 0, nt = 0;
    int depth = 0;
    for (uint32_t steps = 1; steps < kMaxTraversalSteps; ++steps)
        if (stackfree_replay_step<false, false, kDiffStack>(curr, prev, depth, stack, kDiffThreads, hit, nodes, tris,
                                                             ro, rd, inv, 0.0f, nv, nt))
            break;
}

struct PathVertex {
    uint32_t tri;
    float collected;  // throughput * emission at this vertex
};

// Traces the path of sample s of pixel (xi, yi). kStore: fills v (at most
// bounces + 1 vertices) and returns the vertex count; otherwise adds the
// collected radiance, vertex by vertex in path order, to *L (the same sum the
// forward render forms from v) and keeps no vertices.
template <bool kStore>
__device__ __forceinline__ int trace_path(PathVertex* v, float* L, int bounces, uint32_t s, int xi, int yi, int w, int h,
                                          const Camera& cam, uint32_t root, const mlbvh_internal_node* __restrict__ nodes,
                                          const float* __restrict__ tris, const float* __restrict__ albedo,
                                          const float* __restrict__ emission, uint2* stack)
{
    const float2 jitter = sobol2d(s, (uint32_t)xi, (uint32_t)yi, 0u);
    f3 ro, rd;
    shoot(cam, ((float)xi + jitter.x) / (float)w, ((float)yi + jitter.y) / (float)h, ro, rd);
    HitRecord hit;
    hit.t = kFltMax;
    hit.tri = 0xFFFFFFFFu;
    trace_closest(hit, nodes, tris, root, ro, rd, stack);
    if (hit.t == kFltMax) return 0;
    float throughput = 1.0f;
    int count = 0;
    for (int d = 0; d <= bounces; ++d) {
        const uint32_t t = hit.tri;
        const float collected = throughput * __ldg(emission + t);
        if (kStore) {
            v[count].tri = t;
            v[count].collected = collected;
        } else {
            *L += collected;
        }
        ++count;
        if (d == bounces) break;
        const f3 p = ro + rd * hit.t;
        f3 n = normalize(hit.ng);
        if (0.0f < dot(n, rd)) n = -n;
        f3 xaxis, zaxis;
        onb(n, xaxis, zaxis);
        const float2 r = sobol2d(s, (uint32_t)xi, (uint32_t)yi, (uint32_t)(1 + d));
        const f3 dl = sample_hemisphere(r.x, r.y);
        ro = p + n * 0.0001f;
        rd = xaxis * dl.x + zaxis * dl.z + n * dl.y;
        throughput = throughput * __ldg(albedo + t);
        hit.t = kFltMax;
        hit.tri = 0xFFFFFFFFu;
        trace_closest(hit, nodes, tris, root, ro, rd, stack);
        if (hit.t == kFltMax) break;
    }
    return count;
}

__device__ __forceinline__ Camera camera_of(const mlbvh_ray_generator& g)
{
    Camera c;
    c.origin = mk(g.origin[0], g.origin[1], g.origin[2]);
    c.right = mk(g.right[0], g.right[1], g.right[2]);
    c.up = mk(g.up[0], g.up[1], g.up[2]);
    return c;
}

__global__ void __launch_bounds__(kDiffThreads, 768 / kDiffThreads)
    k_pt_diff_render(float* __restrict__ image, int w, int h, int spp, int bounces, mlbvh_ray_generator gen,
                     const mlbvh_node_index* __restrict__ rootPtr, const mlbvh_internal_node* __restrict__ nodes,
                     const float* __restrict__ tris, const float* __restrict__ albedo,
                     const float* __restrict__ emission)
{
    __shared__ uint2 s_stack[kDiffStack][kDiffThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = t / kLanesPerPixel, lane = t % kLanesPerPixel;
    const bool valid = p < w * h;  // every lane takes part in the shuffles below
    float sum = 0.0f;
    if (valid) {
        const int xi = p % w, yi = p / w;
        const Camera cam = camera_of(gen);
        const uint32_t root = __ldg(rootPtr);
        for (int s = lane; s < spp; s += kLanesPerPixel) {
            float L = 0.0f;
            trace_path<false>(nullptr, &L, bounces, (uint32_t)s, xi, yi, w, h, cam, root, nodes, tris, albedo,
                              emission, &s_stack[0][threadIdx.x]);
            sum += L;
        }
    }
    // the pairwise tree in lane order: after step o every lane holds the sum of
    // its aligned group of 2o lanes, the same bits on each (a + b == b + a)
#pragma unroll
    for (int o = 1; o < kLanesPerPixel; o <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (valid && lane == 0) image[p] = sum / (float)spp;
}

__global__ void __launch_bounds__(kDiffThreads, 768 / kDiffThreads)
    k_pt_diff_adjoint(float* __restrict__ grad, const float* __restrict__ gradImage, int w, int h, int spp,
                      int bounces, mlbvh_ray_generator gen, const mlbvh_node_index* __restrict__ rootPtr,
                      const mlbvh_internal_node* __restrict__ nodes, const float* __restrict__ tris,
                      const float* __restrict__ albedo, const float* __restrict__ emission)
{
    __shared__ uint2 s_stack[kDiffStack][kDiffThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = t / kLanesPerPixel, lane = t % kLanesPerPixel;
    if (p >= w * h) return;
    const float g = __ldg(gradImage + p) / (float)spp;
    if (g == 0.0f) return;
    const int xi = p % w, yi = p / w;
    const Camera cam = camera_of(gen);
    const uint32_t root = __ldg(rootPtr);
    PathVertex v[kMaxBounces + 1];
    for (int s = lane; s < spp; s += kLanesPerPixel) {
        const int n = trace_path<true>(v, nullptr, bounces, (uint32_t)s, xi, yi, w, h, cam, root, nodes, tris, albedo,
                                       emission, &s_stack[0][threadIdx.x]);
        // suffix sums of the collected radiance: the part of L that depends on
        // the albedo of vertex j is everything collected after it
        float after = 0.0f;
        for (int j = n - 1; j >= 0; --j) {
            if (j < bounces && after != 0.0f) {
                const uint32_t tj = v[j].tri;
                atomicAdd(grad + tj, g * after / __ldg(albedo + tj));
            }
            after += v[j].collected;
        }
    }
}

mlbvh_status check_diff_args(int w, int h, int spp, int bounces, const void* a, const void* b, const void* c,
                             const void* d, const void* e)
{
    if (w <= 0 || h <= 0 || (long long)w * h >= (1ll << 31)) return fail(MLBVH_ERR_INVALID_ARG, "bad image size");
    if (spp <= 0) return fail(MLBVH_ERR_INVALID_ARG, "spp must be positive");
    if (bounces < 0 || bounces > kMaxBounces) return fail(MLBVH_ERR_INVALID_ARG, "bounces must be in [0, 8]");
    if (!a || !b || !c || !d || !e) return fail(MLBVH_ERR_INVALID_ARG, "null pointer");
    if (!aligned16(a) || !aligned16(b) || !aligned16(c) || !aligned16(d) || !aligned16(e))
        return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    return MLBVH_OK;
}

}  // namespace

mlbvh_status pt_diff_render(float* dImage, int w, int h, int spp, int bounces, const mlbvh_ray_generator& cam,
                            const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                            const mlbvh_triangle* dTris, const float* dAlbedo, const float* dEmission,
                            cudaStream_t stream)
{
    if (mlbvh_status s = check_diff_args(w, h, spp, bounces, dImage, dRoot, dTris, dAlbedo, dEmission)) return s;
    if (!aligned32(dNodes)) return fail(MLBVH_ERR_INVALID_ARG, "device pointers must be 16-byte aligned");
    const long long threads = (long long)w * h * kLanesPerPixel;
    if (threads >= (1ll << 31)) return fail(MLBVH_ERR_INVALID_ARG, "bad image size");
    k_pt_diff_render<<<(unsigned)((threads + kDiffThreads - 1) / kDiffThreads), kDiffThreads, 0, stream>>>(
        dImage, w, h, spp, bounces, cam, dRoot, dNodes, reinterpret_cast<const float*>(dTris), dAlbedo, dEmission);
    MLBVH_CHECK_LAUNCH("k_pt_diff_render");
    return MLBVH_OK;
}

mlbvh_status pt_diff_adjoint(float* dGrad, const float* dGradImage, int w, int h, int spp, int bounces,
                             const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                             const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris, const float* dAlbedo,
                             const float* dEmission, cudaStream_t stream)
{
    if (mlbvh_status s = check_diff_args(w, h, spp, bounces, dGrad, dRoot, dTris, dAlbedo, dEmission)) return s;
    if (!dGradImage || !aligned16(dGradImage) || !aligned32(dNodes))
        return fail(MLBVH_ERR_INVALID_ARG, "null or misaligned pointer");
    const long long threads = (long long)w * h * kLanesPerPixel;
    if (threads >= (1ll << 31)) return fail(MLBVH_ERR_INVALID_ARG, "bad image size");
    k_pt_diff_adjoint<<<(unsigned)((threads + kDiffThreads - 1) / kDiffThreads), kDiffThreads, 0, stream>>>(
        dGrad, dGradImage, w, h, spp, bounces, cam, dRoot, dNodes, reinterpret_cast<const float*>(dTris), dAlbedo,
        dEmission);
    MLBVH_CHECK_LAUNCH("k_pt_diff_adjoint");
    return MLBVH_OK;
}

}  // namespace mlbvh
