// The extern "C" entry points declared in include/mlbvh.h: argument
// checks, error strings, and dispatch to the kernels of build.cu, trace.cu
// and shade.cu. No entry point allocates device memory or synchronises,
// except mlbvh_scratch_status, which synchronises by design.
#include <cmath>
#include <cstring>
#include <string>

#include "capi_internal.h"

namespace mlbvh {

namespace {
thread_local std::string g_lastError;
}

mlbvh_status fail(mlbvh_status status, const char* message)
{
    g_lastError = message ? message : "";
    return status;
}
void clear_error() { g_lastError.clear(); }

namespace {
thread_local ProfileEvents g_profile;
thread_local uint32_t g_spinLimit = 0;  // 0: each build's default
}
void set_profile_events(cudaEvent_t start, cudaEvent_t stop)
{
    g_profile.start = start;
    g_profile.stop = stop;
}
uint32_t spin_limit() { return g_spinLimit; }
ProfileEvents take_profile_events()
{
    ProfileEvents e = g_profile;
    g_profile = ProfileEvents{};
    return e;
}

int device_sm_count()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

}  // namespace mlbvh

using namespace mlbvh;

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

int mlbvh_version(void) { return MLBVH_VERSION; }

const char* mlbvh_last_error_string(void) { return g_lastError.c_str(); }

size_t mlbvh_build_scratch_bytes(uint32_t nTriangles) { return build_scratch_bytes(nTriangles); }

size_t mlbvh_build_ploc_scratch_bytes(uint32_t nTriangles) { return build_ploc_scratch_bytes(nTriangles); }

void mlbvh_set_spin_limit(uint32_t polls) { g_spinLimit = polls; }

mlbvh_status mlbvh_build_ploc(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption, int radius,
                              mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode, mlbvh_aabb* dSceneAABB,
                              void* dScratch, size_t scratchBytes, void* stream)
{
    clear_error();
    return build_ploc(dTriangles, nTriangles, buildOption, radius, dInternals, dRootNode, dSceneAABB, dScratch,
                      scratchBytes, as_stream(stream), g_spinLimit);
}

mlbvh_status mlbvh_build(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption,
                         mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode, mlbvh_aabb* dSceneAABB,
                         void* dScratch, size_t scratchBytes, void* stream)
{
    clear_error();
    return build(dTriangles, nTriangles, buildOption, dInternals, dRootNode, dSceneAABB, nullptr, nullptr, nullptr,
                 dScratch, scratchBytes, as_stream(stream), g_spinLimit);
}

mlbvh_status mlbvh_build_ex(const mlbvh_triangle* dTriangles, uint32_t nTriangles, uint32_t buildOption,
                            mlbvh_internal_node* dInternals, mlbvh_node_index* dRootNode, mlbvh_aabb* dSceneAABB,
                            uint32_t* dSortedKeys, uint32_t* dSortedIndices, uint8_t* dDeltas, void* dScratch,
                            size_t scratchBytes, void* stream)
{
    clear_error();
    return build(dTriangles, nTriangles, buildOption, dInternals, dRootNode, dSceneAABB, dSortedKeys, dSortedIndices,
                 dDeltas, dScratch, scratchBytes, as_stream(stream), g_spinLimit);
}

mlbvh_status mlbvh_scratch_status(const void* dScratch, void* stream)
{
    clear_error();
    if (!dScratch) return noalloc_scratch_status(as_stream(stream));
    return scratch_status(dScratch, as_stream(stream));
}

mlbvh_status mlbvh_trace(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                         const mlbvh_triangle* dTriangles, const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays,
                         int rayQuery, int traversal, void* stream)
{
    clear_error();
    return trace(dInternals, dRootNode, dTriangles, dRays, dHits, nRays, rayQuery, traversal, as_stream(stream));
}

size_t mlbvh_render_scratch_bytes(int width, int height) { return render_scratch_bytes(width, height); }

mlbvh_status mlbvh_render_normal(uint32_t* dPixels, int width, int height, const mlbvh_ray_generator* camera,
                                 const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                                 const mlbvh_triangle* dTriangles, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_normal(dPixels, width, height, *camera, dRootNode, dInternals, dTriangles, as_stream(stream));
}

mlbvh_status mlbvh_render_ao(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                             const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                             const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles, int useSobol,
                             int nSamples, float radius, uint32_t sobolSeed, unsigned long long* dStats,
                             void* dScratch, size_t scratchBytes, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_ao(dPixels, dOccluded, width, height, *camera, dRootNode, dInternals, dTriangles, useSobol, nSamples,
                     radius, sobolSeed, dStats, dScratch, scratchBytes, MLBVH_TRAVERSAL_STACKFREE, nullptr,
                     as_stream(stream));
}

mlbvh_status mlbvh_render_ao_ex(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles, int useSobol,
                                int nSamples, float radius, uint32_t sobolSeed, int traversal,
                                const mlbvh_qtri* dLeafTriangles, unsigned long long* dStats, void* dScratch,
                                size_t scratchBytes, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_ao(dPixels, dOccluded, width, height, *camera, dRootNode, dInternals, dTriangles, useSobol, nSamples,
                     radius, sobolSeed, dStats, dScratch, scratchBytes, traversal, dLeafTriangles, as_stream(stream));
}

mlbvh_status mlbvh_leaf_triangles(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                                  const mlbvh_triangle* dTriangles, uint32_t nTriangles, mlbvh_qtri* dLeafTriangles,
                                  void* stream)
{
    clear_error();
    return leaf_triangles(dInternals, dRootNode, dTriangles, nTriangles, dLeafTriangles, as_stream(stream));
}

mlbvh_status mlbvh_build_wide(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                              uint32_t nTriangles, mlbvh_wnode* dWideNodes, void* stream)
{
    clear_error();
    return build_wide(dInternals, dRootNode, nTriangles, dWideNodes, as_stream(stream));
}

mlbvh_status mlbvh_trace_wide(const mlbvh_wnode* dWideNodes, const mlbvh_internal_node* dInternals,
                              const mlbvh_node_index* dRootNode, const mlbvh_triangle* dTriangles,
                              const mlbvh_qtri* dLeafTriangles, const mlbvh_ray* dRays, mlbvh_hit* dHits,
                              uint32_t nRays, int rayQuery, uint32_t* dCounts, void* stream)
{
    clear_error();
    return trace_wide(dWideNodes, dInternals, dRootNode, dTriangles, dLeafTriangles, dRays, dHits, nRays, rayQuery,
                      dCounts, as_stream(stream));
}

mlbvh_status mlbvh_render_ao_wide(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                  const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                  const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                  const mlbvh_wnode* dWideNodes, const mlbvh_qtri* dLeafTriangles, int useSobol,
                                  int nSamples, float radius, uint32_t sobolSeed, unsigned long long* dStats,
                                  void* dScratch, size_t scratchBytes, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_ao_wide(dPixels, dOccluded, width, height, *camera, dRootNode, dInternals, dTriangles, dWideNodes,
                          dLeafTriangles, useSobol, nSamples, radius, sobolSeed, dStats, dScratch, scratchBytes,
                          as_stream(stream));
}

mlbvh_status mlbvh_quantise_wide(const mlbvh_wnode* dWideNodes, uint32_t nTriangles, mlbvh_qwnode* dQWideNodes,
                                 uint32_t* dStatus, void* stream)
{
    clear_error();
    return quantise_wide(dWideNodes, nTriangles, dQWideNodes, dStatus, as_stream(stream));
}

mlbvh_status mlbvh_trace_wide_quantised(const mlbvh_qwnode* dQWideNodes, const uint32_t* dStatus,
                                        const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                                        const mlbvh_triangle* dTriangles, const mlbvh_qtri* dLeafTriangles,
                                        const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays, int rayQuery,
                                        uint32_t* dCounts, void* stream)
{
    clear_error();
    return trace_wide_quantised(dQWideNodes, dStatus, dInternals, dRootNode, dTriangles, dLeafTriangles, dRays, dHits,
                                nRays, rayQuery, dCounts, as_stream(stream));
}

mlbvh_status mlbvh_render_ao_wide_quantised(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                            const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                            const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                            const mlbvh_qwnode* dQWideNodes, const uint32_t* dStatus,
                                            const mlbvh_qtri* dLeafTriangles, int useSobol, int nSamples,
                                            float radius, uint32_t sobolSeed, unsigned long long* dStats,
                                            void* dScratch, size_t scratchBytes, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_ao_wide_quantised(dPixels, dOccluded, width, height, *camera, dRootNode, dInternals, dTriangles,
                                    dQWideNodes, dStatus, dLeafTriangles, useSobol, nSamples, radius, sobolSeed,
                                    dStats, dScratch, scratchBytes, as_stream(stream));
}

mlbvh_status mlbvh_render_pt(float* dAccumulators, int width, int height, const mlbvh_ray_generator* camera,
                             const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                             const mlbvh_triangle* dTriangles, const mlbvh_triangle_attrib* dAttribs, int useSobol,
                             int maxSPP, int maxDepth, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_pt(dAccumulators, width, height, *camera, dRootNode, dInternals, dTriangles, dAttribs, useSobol,
                     maxSPP, maxDepth, as_stream(stream));
}

mlbvh_status mlbvh_render_pt_ex(float* dAccumulators, int width, int height, const mlbvh_ray_generator* camera,
                                const mlbvh_node_index* dRootNode, const mlbvh_internal_node* dInternals,
                                const mlbvh_triangle* dTriangles, const mlbvh_triangle_attrib* dAttribs,
                                int useSobol, int maxSPP, int maxDepth, int traversal,
                                const mlbvh_qtri* dLeafTriangles, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_pt(dAccumulators, width, height, *camera, dRootNode, dInternals, dTriangles, dAttribs, useSobol,
                     maxSPP, maxDepth, as_stream(stream), traversal, dLeafTriangles);
}

mlbvh_status mlbvh_quantise(const mlbvh_internal_node* dInternals, const mlbvh_node_index* dRootNode,
                            const mlbvh_triangle* dTriangles, uint32_t nTriangles, mlbvh_qnode* dQNodes,
                            uint32_t* dQParents, mlbvh_qtri* dQTris, mlbvh_qheader* dQHeader, void* stream)
{
    clear_error();
    return quantise(dInternals, dRootNode, dTriangles, nTriangles, dQNodes, dQParents, dQTris, dQHeader,
                    as_stream(stream));
}

mlbvh_status mlbvh_trace_quantised(const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                   const mlbvh_qheader* dQHeader, const mlbvh_ray* dRays, mlbvh_hit* dHits,
                                   uint32_t nRays, int rayQuery, void* stream)
{
    clear_error();
    return trace_quantised(dQNodes, dQParents, dQTris, dQHeader, dRays, dHits, nRays, rayQuery, 16, nullptr,
                           as_stream(stream));
}

mlbvh_status mlbvh_trace_quantised_ex(const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                      const mlbvh_qheader* dQHeader, const mlbvh_ray* dRays, mlbvh_hit* dHits,
                                      uint32_t nRays, int rayQuery, int stackDepth, uint32_t* dCounts, void* stream)
{
    clear_error();
    return trace_quantised(dQNodes, dQParents, dQTris, dQHeader, dRays, dHits, nRays, rayQuery, stackDepth, dCounts,
                           as_stream(stream));
}

mlbvh_status mlbvh_render_ao_quantised(uint32_t* dPixels, uint32_t* dOccluded, int width, int height,
                                       const mlbvh_ray_generator* camera, const mlbvh_qnode* dQNodes,
                                       const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                       const mlbvh_qheader* dQHeader, int useSobol, int nSamples, float radius,
                                       uint32_t sobolSeed, unsigned long long* dStats, void* dScratch,
                                       size_t scratchBytes, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return render_ao_quantised(dPixels, dOccluded, width, height, *camera, dQNodes, dQParents, dQTris, dQHeader,
                               useSobol, nSamples, radius, sobolSeed, dStats, dScratch, scratchBytes,
                               as_stream(stream));
}

mlbvh_status mlbvh_pt_diff_render(float* dImage, int width, int height, int spp, int bounces,
                                  const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                  const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                  const float* dAlbedo, const float* dEmission, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return pt_diff_render(dImage, width, height, spp, bounces, *camera, dRootNode, dInternals, dTriangles, dAlbedo,
                          dEmission, as_stream(stream));
}

mlbvh_status mlbvh_pt_diff_adjoint(float* dGradAlbedo, const float* dGradImage, int width, int height, int spp,
                                   int bounces, const mlbvh_ray_generator* camera, const mlbvh_node_index* dRootNode,
                                   const mlbvh_internal_node* dInternals, const mlbvh_triangle* dTriangles,
                                   const float* dAlbedo, const float* dEmission, void* stream)
{
    clear_error();
    if (!camera) return fail(MLBVH_ERR_INVALID_ARG, "null camera");
    return pt_diff_adjoint(dGradAlbedo, dGradImage, width, height, spp, bounces, *camera, dRootNode, dInternals,
                           dTriangles, dAlbedo, dEmission, as_stream(stream));
}

size_t mlbvh_batch_scratch_bytes(uint32_t nMeshes, uint32_t nTriangles)
{
    return batch_scratch_bytes(nMeshes, nTriangles);
}

void mlbvh_batch_params_default(mlbvh_batch_params* params)
{
    if (params) batch_params_default(params);
}

static const mlbvh_batch_params& params_or_default(const mlbvh_batch_params* p, mlbvh_batch_params& storage)
{
    if (p) return *p;
    batch_params_default(&storage);
    return storage;
}

mlbvh_status mlbvh_build_batched(const mlbvh_batch* batch, const mlbvh_batch_params* params, void* stream)
{
    clear_error();
    if (!batch) return fail(MLBVH_ERR_INVALID_ARG, "null batch");
    mlbvh_batch_params d;
    return build_batched(*batch, params_or_default(params, d), as_stream(stream));
}

mlbvh_status mlbvh_trace_batched(const mlbvh_batch* batch, const mlbvh_batch_params* params, void* stream)
{
    clear_error();
    if (!batch) return fail(MLBVH_ERR_INVALID_ARG, "null batch");
    mlbvh_batch_params d;
    return trace_batched(*batch, params_or_default(params, d), as_stream(stream));
}

mlbvh_status mlbvh_batch_autotune(const mlbvh_batch* batch, mlbvh_batch_params* params, float* buildMs,
                                  float* traceMs, void* stream)
{
    clear_error();
    if (!batch) return fail(MLBVH_ERR_INVALID_ARG, "null batch");
    return batch_autotune(*batch, params, buildMs, traceMs, as_stream(stream));
}

mlbvh_status mlbvh_batch_graph_create(const mlbvh_batch* batch, const mlbvh_batch_params* params, int stages,
                                      mlbvh_batch_graph** graph)
{
    clear_error();
    if (!batch) return fail(MLBVH_ERR_INVALID_ARG, "null batch");
    mlbvh_batch_params d;
    return batch_graph_create(*batch, params_or_default(params, d), stages, graph);
}

mlbvh_status mlbvh_batch_graph_launch(mlbvh_batch_graph* graph, void* stream)
{
    clear_error();
    return batch_graph_launch(graph, as_stream(stream));
}

void mlbvh_batch_graph_destroy(mlbvh_batch_graph* graph) { batch_graph_destroy(graph); }

void mlbvh_profile_events(void* startEvent, void* stopEvent)
{
    set_profile_events(reinterpret_cast<cudaEvent_t>(startEvent), reinterpret_cast<cudaEvent_t>(stopEvent));
}

mlbvh_status mlbvh_pack(uint32_t* dPixels, const float* dAccumulators, int n, void* stream)
{
    clear_error();
    return pack(dPixels, dAccumulators, n, as_stream(stream));
}

// RayGenerator::lookat (camera.h:10-22) on the host; the host compiler runs
// with -ffp-contract=off, so this rounds as the reference's host build does.
mlbvh_status mlbvh_camera_lookat(mlbvh_ray_generator* out, const float eye[3], const float center[3],
                                 const float up[3], float fovy, int width, int height)
{
    clear_error();
    if (!out || !eye || !center || !up || width <= 0 || height <= 0)
        return fail(MLBVH_ERR_INVALID_ARG, "null pointer or non-positive image size");
    auto sub = [](const float* a, const float* b, float* r) {
        r[0] = a[0] - b[0];
        r[1] = a[1] - b[1];
        r[2] = a[2] - b[2];
    };
    auto cross = [](const float* a, const float* b, float* r) {
        float x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
        r[0] = x;
        r[1] = y;
        r[2] = z;
    };
    auto normalize = [](float* v) {
        float d = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        float inv = 1.0f / std::sqrt(d);
        v[0] = v[0] * inv;
        v[1] = v[1] * inv;
        v[2] = v[2] * inv;
    };
    float f[3], s[3], u[3];
    sub(center, eye, f);
    normalize(f);
    cross(f, up, s);
    normalize(s);
    cross(s, f, u);
    float tanThetaY = std::tan(fovy * 0.5f);
    float tanThetaX = tanThetaY / (float)height * (float)width;
    for (int i = 0; i < 3; ++i) {
        out->origin[i] = eye[i];
        out->right[i] = s[i] * tanThetaX;
        out->up[i] = u[i] * tanThetaY;
    }
    return MLBVH_OK;
}

}  // extern "C"
