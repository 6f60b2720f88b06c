// The C++ adapter (include/dmap_b200.hpp) used the way the reference's
// callers use ObjectIntersector (traversal_test_util.cpp:13-19): one unit
// quad of two base triangles displaced by a height grid read from a file,
// rays read from a file; every ray through the single-ray intersect() and
// all rays through intersect_batch(). Writes both answers for comparison.
// Usage: adapter_quad <nodes> <heights.f32> <rays.f64> <out.f64>
#include "dmap_b200.hpp"

#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

template <typename T> std::vector<T> read_all(const char *path)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    std::vector<T> v((size_t)f.tellg() / sizeof(T));
    f.seekg(0);
    f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
    return v;
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        std::cerr << "usage: adapter_quad <nodes> <heights.f32> <rays.f64> <out.f64>\n";
        return 2;
    }
    try {
        int nodes = std::atoi(argv[1]);
        std::vector<float> heights = read_all<float>(argv[2]);
        std::vector<double> rays = read_all<double>(argv[3]);
        const int64_t n = (int64_t)rays.size() / 8;
        dmapgpu::Context ctx(0);
        dmapgpu::DisplacementAsset asset(ctx, heights.data(), nodes);
        const dmapgpu::vec3d z = {0.0, 0.0, 1.0};
        std::vector<dmapgpu::BaseTriangleDesc> tris = {
            {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, z, z, z, {0, 0}, {1, 0}, {0, 1}},
            {{1, 1, 0}, {0, 1, 0}, {1, 0, 0}, z, z, z, {1, 1}, {0, 1}, {1, 0}},
        };
        dmapgpu::ObjectIntersector isect(ctx, tris, asset);
        dmapgpu::TraversalOptions options;
        // per ray: found, triangle, t, st, bary, ng (single call), then the batch's t and triangle
        std::vector<double> out((size_t)n * 12);
        std::vector<dmap_hit64> batch((size_t)n);
        isect.intersect_batch(rays.data(), n, options, batch.data());
        for (int64_t k = 0; k < n; ++k) {
            const double *r = &rays[8 * k];
            dmapgpu::DisplacedHit hit;
            int tri = -1;
            bool found = isect.intersect({r[0], r[1], r[2]}, {r[3], r[4], r[5]}, r[6], r[7], options, hit, tri);
            double *o = &out[12 * k];
            o[0] = found ? 1.0 : 0.0;
            o[1] = tri;
            o[2] = found ? hit.t : 0.0;
            o[3] = hit.st[0], o[4] = hit.st[1], o[5] = hit.bary[0], o[6] = hit.bary[1];
            o[7] = hit.ng[0], o[8] = hit.ng[1], o[9] = hit.ng[2];
            o[10] = batch[k].tri >= 0 ? batch[k].t : 0.0;
            o[11] = batch[k].tri;
        }
        std::ofstream f(argv[4], std::ios::binary);
        f.write(reinterpret_cast<const char *>(out.data()), (std::streamsize)(out.size() * sizeof(double)));
    } catch (const dmapgpu::Error &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    return 0;
}
