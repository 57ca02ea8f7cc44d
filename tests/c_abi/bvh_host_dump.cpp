// Builds the host wide BVH (raymond_b200/csrc/bvh_build.cpp) of a triangle
// soup read from a file and writes the nodes and leaf-ordered triangles, so
// the CPU tests can check the builder's tree without a GPU.
//   bvh_host_dump in.f32 nodes.bin tris.bin   (in: n x 9 floats, v0 v1 v2)
#include <cstdio>
#include <vector>

#include "bvh_build.h"

int main(int argc, char **argv) {
    if (argc != 4) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    std::vector<float> in;
    float buf[9];
    while (std::fread(buf, sizeof(float), 9, f) == 9) in.insert(in.end(), buf, buf + 9);
    std::fclose(f);
    const size_t n = in.size() / 9;
    std::vector<float> v0(3 * n), v1(3 * n), v2(3 * n);
    std::vector<uint32_t> inst(n, 0), prim(n);
    for (size_t i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) {
            v0[3 * i + k] = in[9 * i + k];
            v1[3 * i + k] = in[9 * i + 3 + k];
            v2[3 * i + k] = in[9 * i + 6 + k];
        }
        prim[i] = (uint32_t)i;
    }
    rmdhost::GpuWideBvh bvh;
    rmdhost::buildWideBvh(v0, v1, v2, inst, prim, bvh);
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 4;
    std::fwrite(bvh.nodes.data(), sizeof(rmdhost::GpuWideNode), bvh.nodes.size(), o);
    std::fclose(o);
    o = std::fopen(argv[3], "wb");
    if (!o) return 5;
    std::fwrite(bvh.tris.data(), sizeof(float), bvh.tris.size(), o);
    std::fclose(o);
    return 0;
}
