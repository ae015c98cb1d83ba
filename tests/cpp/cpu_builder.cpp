// A host-only C++ program written against the reference's BVHCPUBuilder
// (minimum_lbvh.h:509-669), as its viewer uses it (main.cpp:246-249: build
// when empty, validate, then read the nodes on the host). Compiled with g++
// against include/minimum_lbvh.h and linked with libmlbvh_b200.so and
// cudart; the build itself runs on the GPU. Used by tests/test_gpu_dropin.py:
//   cpu_builder <triangles.bin> <out.bin> [option]
// out.bin: root (4 B), nodes ((n-1) x 64 B), deltas (n-1 B), then the number
// of leaves reached from the root by a host walk over m_internals (4 B).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "minimum_lbvh.h"

static std::vector<minimum_lbvh::Triangle> load(const char* path)
{
    std::vector<minimum_lbvh::Triangle> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize(bytes / sizeof(minimum_lbvh::Triangle));
    if (std::fread(v.data(), sizeof(minimum_lbvh::Triangle), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

int main(int argc, char** argv)
{
    if (argc != 3 && argc != 4) return 2;
    std::vector<minimum_lbvh::Triangle> triangles = load(argv[1]);
    if (triangles.empty()) return 3;
    const uint32_t option = argc == 4 ? (uint32_t)std::atoi(argv[3]) : minimum_lbvh::BUILD_OPTION_CPU_PARALLEL;

    minimum_lbvh::BVHCPUBuilder builder;
    if (builder.empty()) {
        builder.build(triangles.data(), triangles.size(), option);
        builder.validate();
    }

    // host-side use of the tree: count the leaves below the root
    uint32_t leaves = 0;
    std::vector<minimum_lbvh::NodeIndex> todo{builder.m_rootNode};
    while (!todo.empty()) {
        minimum_lbvh::NodeIndex node = todo.back();
        todo.pop_back();
        if (node.m_isLeaf) {
            ++leaves;
            continue;
        }
        todo.push_back(builder.m_internals[node.m_index].children[0]);
        todo.push_back(builder.m_internals[node.m_index].children[1]);
    }

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 5;
    std::fwrite(&builder.m_rootNode, 4, 1, f);
    std::fwrite(builder.m_internals.data(), sizeof(minimum_lbvh::InternalNode), builder.m_internals.size(), f);
    std::fwrite(builder.m_deltas.data(), 1, builder.m_deltas.size(), f);
    std::fwrite(&leaves, 4, 1, f);
    std::fclose(f);
    std::printf("cpu_builder: %zu triangles, %u leaves\n", triangles.size(), leaves);
    return 0;
}
