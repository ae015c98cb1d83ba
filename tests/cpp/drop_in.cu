// A program written against the reference's API (BVHGPUBuilder, OnesweepSort,
// intersect_stackfree / intersect_escape_link inside the caller's own kernel),
// compiled against include/minimum_lbvh.h and linked with libmlbvh_b200.so.
// Used by tests/test_gpu_dropin.py:
//   drop_in <triangles.bin> <rays.bin> <out.bin> [ploc radius, 0 = LBVH] [timeout]
// triangles.bin: n x 36 B; rays.bin: m x 32 B (ro, tmin, rd, tmax);
// out.bin: root (4 B), nodes ((n-1) x 64 B), stack-free hits (m x 32 B),
// escape-link any-hit hits (m x 32 B).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "minimum_lbvh.h"

using namespace minimum_lbvh;

__global__ void user_trace(Hit* out, Hit* outAny, const float4* rays, int m, const NodeIndex* rootNode,
                           const InternalNode* internals, const Triangle* triangles)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    float4 a = rays[2 * i], b = rays[2 * i + 1];
    float3 ro = make_float3(a.x, a.y, a.z), rd = make_float3(b.x, b.y, b.z);
    Hit hit;
    hit.t = b.w;
    intersect_stackfree(&hit, internals, triangles, *rootNode, ro, rd, invRd(rd));
    out[i] = hit;
    Hit any;
    any.t = b.w;
    intersect_escape_link(&any, internals, triangles, *rootNode, ro, rd, invRd(rd), RAY_QUERY_ANY);
    outAny[i] = any;
}

static std::vector<char> load(const char* path)
{
    std::vector<char> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    v.resize(std::ftell(f));
    std::fseek(f, 0, SEEK_SET);
    if (std::fread(v.data(), 1, v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

// With the bounded device waits cut to one poll (mlbvh_set_spin_limit, a
// test hook), builds whose waits give up must say so through
// BVHGPUBuilder::status. Returns the number of MLBVH_ERR_TIMEOUT reports in
// `tries` builds, or -1 on any status other than that and MLBVH_OK. The spin
// limit is restored before returning; the caller then builds once more with
// the default limit, and that tree is the one checked.
static int count_timeouts(BVHGPUBuilder& builder, tinyhiponesweep::OnesweepSort& onesweep, const Triangle* dTris,
                          int n, cudaStream_t stream, int ploc, int tries)
{
    int timeouts = 0;
    mlbvh_set_spin_limit(1);
    for (int i = 0; i < tries; ++i) {
        if (ploc)
            builder.buildByPLOC(dTris, n, 0, onesweep, stream, ploc);
        else
            builder.build(dTris, n, 0, onesweep, stream);
        const mlbvh_status s = builder.status(stream);
        if (s == MLBVH_ERR_TIMEOUT)
            ++timeouts;
        else if (s != MLBVH_OK)
            timeouts = -1000;
    }
    mlbvh_set_spin_limit(0);
    return timeouts < 0 ? -1 : timeouts;
}

int main(int argc, char** argv)
{
    // argv[4] (optional): a PLOC radius; the tree then comes from buildByPLOC.
    // argv[5] (optional): "timeout" first runs builds with one-poll waits
    // (count_timeouts) and prints how many reported MLBVH_ERR_TIMEOUT.
    if (argc < 4 || argc > 6) return 2;
    std::vector<char> tris = load(argv[1]), rays = load(argv[2]);
    const int n = (int)(tris.size() / sizeof(Triangle)), m = (int)(rays.size() / 32);
    if (n < 2 || m < 1) return 3;
    Triangle* dTris;
    float4* dRays;
    Hit *dHits, *dAny;
    cudaMalloc(&dTris, tris.size());
    cudaMalloc(&dRays, rays.size());
    cudaMalloc(&dHits, sizeof(Hit) * m);
    cudaMalloc(&dAny, sizeof(Hit) * m);
    cudaMemcpy(dTris, tris.data(), tris.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dRays, rays.data(), rays.size(), cudaMemcpyHostToDevice);

    cudaStream_t stream;
    cudaStreamCreate(&stream);
    tinyhiponesweep::OnesweepSort onesweep(0);
    BVHGPUBuilder builder("unused/minimum_lbvh.cu", "unused/");
    const int ploc = argc >= 5 ? std::atoi(argv[4]) : 0;
    if (argc == 6 && std::string(argv[5]) == "timeout") {
        const int timeouts = count_timeouts(builder, onesweep, dTris, n, stream, ploc, 3);
        if (timeouts < 0) return 6;
        std::printf("drop_in: %d of 3 builds with one-poll waits reported MLBVH_ERR_TIMEOUT\n", timeouts);
    }
    if (ploc)
        builder.buildByPLOC(dTris, n, 0, onesweep, stream, ploc);
    else
        builder.build(dTris, n, 0, onesweep, stream);
    if (builder.status(stream) != MLBVH_OK) return 7;
    user_trace<<<(m + 127) / 128, 128, 0, stream>>>(dHits, dAny, dRays, m, builder.m_rootNode, builder.m_internals, dTris);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return 4;

    std::vector<char> out(4 + sizeof(InternalNode) * (n - 1) + 2 * sizeof(Hit) * m);
    cudaMemcpy(out.data(), builder.m_rootNode, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(out.data() + 4, builder.m_internals, sizeof(InternalNode) * (n - 1), cudaMemcpyDeviceToHost);
    cudaMemcpy(out.data() + 4 + sizeof(InternalNode) * (n - 1), dHits, sizeof(Hit) * m, cudaMemcpyDeviceToHost);
    cudaMemcpy(out.data() + 4 + sizeof(InternalNode) * (n - 1) + sizeof(Hit) * m, dAny, sizeof(Hit) * m,
               cudaMemcpyDeviceToHost);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 5;
    std::fwrite(out.data(), 1, out.size(), f);
    std::fclose(f);
    std::printf("drop_in: %d triangles, %d rays\n", n, m);
    return 0;
}
