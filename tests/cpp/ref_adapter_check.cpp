// The drop-in adapter (include/dmap_b200_reference.hpp) against the
// reference's own ObjectIntersector, built from the reference sources in
// place with the oracle's stand-in headers (oracle/Makefile ref_adapter).
// TEST INFRASTRUCTURE: tests/test_ref_adapter.py writes the input and reads
// the output.
//
// Input (little-endian): int32 W, int32 build (0 fold, 1 direct), int32
// repeat, double scale, double offset, W*W doubles (node grid), int32 n_tri,
// n_tri*24 doubles (p0 p1 p2 m0 m1 m2 t0 t1 t2), int32 n_rays, n_rays*8
// doubles (o, d, t_min, t_max).
// Output: per ray, for the reference, the adapter's single-ray call and its
// batch call, 12 doubles (t, st, bary, ng, i, j, triangle; t = inf on a
// miss) and, for the single-ray calls, the 6 counters of each.
#include "displaced_intersector.h"
#include "taylor_pyramid.h"

#include "dmap_b200_reference.hpp"

#include <cmath>
#include <cstdio>
#include <vector>

namespace
{
template <typename T>
bool get(FILE *f, T *p, size_t n)
{
    return fread(p, sizeof(T), n, f) == n;
}

void put_hit(std::vector<double> &out, bool found, const dmap::DisplacedHit &h, int tri)
{
    double v[12] = {INFINITY, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -1.0, 0.0};
    if (found) {
        double w[12] = {h.t, h.st[0], h.st[1], h.bary[0], h.bary[1], h.ng[0], h.ng[1], h.ng[2],
                        (double)h.i, (double)h.j, (double)tri, 0.0};
        for (int q = 0; q < 12; ++q)
            v[q] = w[q];
    }
    out.insert(out.end(), v, v + 12);
}

void put_stats(std::vector<double> &out, const dmap::TraversalStats &s)
{
    double v[6] = {(double)s.triangle_tests, (double)s.node_tests, (double)s.leaf_tests, (double)s.sub_squares,
                   (double)s.node_tests_after_hit, (double)s.leaf_tests_after_hit};
    out.insert(out.end(), v, v + 6);
}
} // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: ref_adapter_check IN OUT\n");
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f)
        return 2;
    int W = 0, build = 0, repeat = 0, n_tri = 0, n_rays = 0;
    double scale = 1.0, offset = 0.0;
    bool ok = get(f, &W, 1) && get(f, &build, 1) && get(f, &repeat, 1) && get(f, &scale, 1) && get(f, &offset, 1);
    std::vector<double> values(ok ? (size_t)W * W : 0);
    ok = ok && get(f, values.data(), values.size()) && get(f, &n_tri, 1);
    std::vector<double> tri_rec(ok ? (size_t)n_tri * 24 : 0);
    ok = ok && get(f, tri_rec.data(), tri_rec.size()) && get(f, &n_rays, 1);
    std::vector<double> rays(ok ? (size_t)n_rays * 8 : 0);
    ok = ok && get(f, rays.data(), rays.size());
    fclose(f);
    if (!ok) {
        fprintf(stderr, "bad input\n");
        return 2;
    }

    dmap::HeightGrid field;
    field.W = field.H = W;
    field.values = values.data();
    field.scale = scale;
    field.offset = offset;
    field.repeat = repeat != 0;
    dmap::TaylorPyramid pyramid(field, build ? dmap::PyramidBuild::Direct : dmap::PyramidBuild::Fold);
    std::vector<dmap::BaseTriangle> tris;
    for (int k = 0; k < n_tri; ++k) {
        const double *r = &tri_rec[24 * (size_t)k];
        auto v3 = [&](int o) { return ks::vec3d(r[o], r[o + 1], r[o + 2]); };
        auto v2 = [&](int o) { return ks::vec2d(r[o], r[o + 1]); };
        tris.emplace_back(v3(0), v3(3), v3(6), v3(9), v3(12), v3(15), v2(18), v2(20), v2(22));
    }

    dmap::ObjectIntersector reference(tris, pyramid, field);
    dmap::GpuObjectIntersector gpu(tris, pyramid, field);
    dmap::TraversalOptions options;

    std::vector<double> out;
    out.reserve((size_t)n_rays * 48);
    std::vector<dmap::DisplacedHit> batch(n_rays);
    std::vector<int> batch_tri(n_rays);
    gpu.intersect_batch(rays.data(), n_rays, options, batch.data(), batch_tri.data());
    for (int k = 0; k < n_rays; ++k) {
        const double *r = &rays[8 * (size_t)k];
        ks::vec3d o(r[0], r[1], r[2]), d(r[3], r[4], r[5]);
        dmap::DisplacedHit h_ref, h_gpu;
        int t_ref = -1, t_gpu = -1;
        dmap::TraversalStats s_ref, s_gpu;
        bool f_ref = reference.intersect(o, d, r[6], r[7], options, h_ref, t_ref, &s_ref);
        bool f_gpu = gpu.intersect(o, d, r[6], r[7], options, h_gpu, t_gpu, &s_gpu);
        put_hit(out, f_ref, h_ref, t_ref);
        put_hit(out, f_gpu, h_gpu, t_gpu);
        put_hit(out, batch_tri[k] >= 0, batch[k], batch_tri[k]);
        put_stats(out, s_ref);
        put_stats(out, s_gpu);
    }
    FILE *g = fopen(argv[2], "wb");
    if (!g || fwrite(out.data(), sizeof(double), out.size(), g) != out.size())
        return 2;
    fclose(g);
    printf("ref_adapter_check: %d rays over %d triangles\n", n_rays, n_tri);
    return 0;
}
