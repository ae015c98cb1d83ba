// Internal declarations shared by the translation units of libmlbvh_b200.so.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mlbvh.h"

namespace mlbvh {

// Records the message for mlbvh_last_error_string() on this host thread and
// returns the status.
mlbvh_status fail(mlbvh_status status, const char* message);
void clear_error();
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
// Node arrays are read with 32-byte loads.
inline bool aligned32(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; }
int device_sm_count();

// CUDA events (cudaEvent_t) that the next render_ao / build call on this host
// thread records around its dominant kernel; taking them clears them.
struct ProfileEvents {
    cudaEvent_t start = nullptr, stop = nullptr;
};
void set_profile_events(cudaEvent_t start, cudaEvent_t stop);
ProfileEvents take_profile_events();

#define MLBVH_CHECK_LAUNCH(name)                                                              \
    do {                                                                                      \
        cudaError_t e_ = cudaGetLastError();                                                  \
        if (e_ != cudaSuccess) return ::mlbvh::fail(MLBVH_ERR_LAUNCH, cudaGetErrorString(e_)); \
    } while (0)

size_t build_scratch_bytes(uint32_t n);
mlbvh_status build(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, mlbvh_internal_node* dNodes,
                   mlbvh_node_index* dRoot, mlbvh_aabb* dScene, uint32_t* dKeysOut, uint32_t* dIdxOut,
                   uint8_t* dDeltasOut, void* dScratch, size_t scratchBytes, cudaStream_t stream, uint32_t spinLimit);
mlbvh_status scratch_status(const void* dScratch, cudaStream_t stream);
// The bounded-wait poll count set by mlbvh_set_spin_limit on this host thread
// (0: each build's default).
uint32_t spin_limit();
// scratch_status of mlbvh_build_noalloc's built-in array in the current
// context (noalloc.cu).
mlbvh_status noalloc_scratch_status(cudaStream_t stream);

// The build chain up to the sorted leaves (scene bounds, keys, four stable
// sort passes), shared by build() and build_ploc(); the caller has checked
// the arguments. Pointers into the caller's scratch (or its outputs).
struct SortedLeaves {
    const uint32_t* keys;     // n sorted Morton keys
    const uint32_t* indices;  // n triangle indices in that order
    uint32_t* error;          // the build's error word (scratch offset 0)
    uint32_t* handoff;        // n words, zeroed for build_lbvh's hand-off
    uint8_t* deltas;          // n bytes
    uint32_t spinLimit;       // polls per bounded wait
};
mlbvh_status sort_leaves(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, mlbvh_aabb* dScene,
                         uint32_t* dKeysOut, uint32_t* dIdxOut, uint8_t* dDeltasOut, void* dScratch,
                         cudaStream_t stream, uint32_t spinLimit, SortedLeaves* out);

size_t build_ploc_scratch_bytes(uint32_t n);
mlbvh_status build_ploc(const mlbvh_triangle* dTris, uint32_t n, uint32_t option, int radius,
                        mlbvh_internal_node* dNodes, mlbvh_node_index* dRoot, mlbvh_aabb* dScene, void* dScratch,
                        size_t scratchBytes, cudaStream_t stream, uint32_t spinLimit);

mlbvh_status trace(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, const mlbvh_triangle* dTris,
                   const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays, int rayQuery, int traversal,
                   cudaStream_t stream);

size_t render_scratch_bytes(int w, int h);
mlbvh_status render_normal(uint32_t* dPixels, int w, int h, const mlbvh_ray_generator& cam,
                           const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                           const mlbvh_triangle* dTris, cudaStream_t stream);
mlbvh_status render_ao(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                       const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                       int useSobol, int nSamples, float radius, uint32_t seed, unsigned long long* dStats,
                       void* dScratch, size_t scratchBytes, int traversal, const mlbvh_qtri* dLeafTris,
                       cudaStream_t stream);
mlbvh_status leaf_triangles(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                            const mlbvh_triangle* dTris, uint32_t n, mlbvh_qtri* dLeafTris, cudaStream_t stream);
mlbvh_status build_wide(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, uint32_t n,
                        mlbvh_wnode* dWide, cudaStream_t stream);
mlbvh_status trace_wide(const mlbvh_wnode* dWide, const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                        const mlbvh_triangle* dTris, const mlbvh_qtri* dLeafTris, const mlbvh_ray* dRays,
                        mlbvh_hit* dHits, uint32_t nRays, int rayQuery, uint32_t* dCounts, cudaStream_t stream);
mlbvh_status quantise_wide(const mlbvh_wnode* dWide, uint32_t n, mlbvh_qwnode* dQWide, uint32_t* dStatus,
                           cudaStream_t stream);
mlbvh_status trace_wide_quantised(const mlbvh_qwnode* dQWide, const uint32_t* dStatus,
                                  const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot,
                                  const mlbvh_triangle* dTris, const mlbvh_qtri* dLeafTris, const mlbvh_ray* dRays,
                                  mlbvh_hit* dHits, uint32_t nRays, int rayQuery, uint32_t* dCounts,
                                  cudaStream_t stream);
mlbvh_status render_ao_wide_quantised(uint32_t* dPixels, uint32_t* dOccluded, int w, int h,
                                      const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                                      const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                                      const mlbvh_qwnode* dQWide, const uint32_t* dStatus,
                                      const mlbvh_qtri* dLeafTris, int useSobol, int nSamples, float radius,
                                      uint32_t seed, unsigned long long* dStats, void* dScratch, size_t scratchBytes,
                                      cudaStream_t stream);
mlbvh_status render_ao_wide(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                            const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                            const mlbvh_triangle* dTris, const mlbvh_wnode* dWide, const mlbvh_qtri* dLeafTris,
                            int useSobol, int nSamples, float radius, uint32_t seed, unsigned long long* dStats,
                            void* dScratch, size_t scratchBytes, cudaStream_t stream);
mlbvh_status render_ao_quantised(uint32_t* dPixels, uint32_t* dOccluded, int w, int h, const mlbvh_ray_generator& cam,
                                 const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                                 const mlbvh_qheader* dQHeader, int useSobol, int nSamples, float radius,
                                 uint32_t seed, unsigned long long* dStats, void* dScratch, size_t scratchBytes,
                                 cudaStream_t stream);
mlbvh_status quantise(const mlbvh_internal_node* dNodes, const mlbvh_node_index* dRoot, const mlbvh_triangle* dTris,
                      uint32_t n, mlbvh_qnode* dQNodes, uint32_t* dQParents, mlbvh_qtri* dQTris,
                      mlbvh_qheader* dQHeader, cudaStream_t stream);
mlbvh_status trace_quantised(const mlbvh_qnode* dQNodes, const uint32_t* dQParents, const mlbvh_qtri* dQTris,
                             const mlbvh_qheader* dQHeader, const mlbvh_ray* dRays, mlbvh_hit* dHits, uint32_t nRays,
                             int rayQuery, int stackDepth, uint32_t* dCounts, cudaStream_t stream);
mlbvh_status render_pt(float* dAccum, int w, int h, const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                       const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris,
                       const mlbvh_triangle_attrib* dAttribs, int useSobol, int maxSPP, int maxDepth,
                       cudaStream_t stream, int traversal = MLBVH_TRAVERSAL_STACKFREE,
                       const mlbvh_qtri* dLeafTris = nullptr);
mlbvh_status pack(uint32_t* dPixels, const float* dAccum, int n, cudaStream_t stream);
mlbvh_status pt_diff_render(float* dImage, int w, int h, int spp, int bounces, const mlbvh_ray_generator& cam,
                            const mlbvh_node_index* dRoot, const mlbvh_internal_node* dNodes,
                            const mlbvh_triangle* dTris, const float* dAlbedo, const float* dEmission,
                            cudaStream_t stream);
mlbvh_status pt_diff_adjoint(float* dGrad, const float* dGradImage, int w, int h, int spp, int bounces,
                             const mlbvh_ray_generator& cam, const mlbvh_node_index* dRoot,
                             const mlbvh_internal_node* dNodes, const mlbvh_triangle* dTris, const float* dAlbedo,
                             const float* dEmission, cudaStream_t stream);

size_t batch_scratch_bytes(uint32_t nMeshes, uint32_t n);
void batch_params_default(mlbvh_batch_params* p);
mlbvh_status build_batched(const mlbvh_batch& B, const mlbvh_batch_params& P, cudaStream_t stream);
mlbvh_status trace_batched(const mlbvh_batch& B, const mlbvh_batch_params& P, cudaStream_t stream);
mlbvh_status batch_autotune(const mlbvh_batch& B, mlbvh_batch_params* out, float* bestBuildMs, float* bestTraceMs,
                            cudaStream_t stream);
mlbvh_status batch_graph_create(const mlbvh_batch& B, const mlbvh_batch_params& P, int stages,
                                mlbvh_batch_graph** out);
mlbvh_status batch_graph_launch(mlbvh_batch_graph* g, cudaStream_t stream);
void batch_graph_destroy(mlbvh_batch_graph* g);
mlbvh_status obj_load(const char* path, mlbvh_obj_mesh** out);

}  // namespace mlbvh
