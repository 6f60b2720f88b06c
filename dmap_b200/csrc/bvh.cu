// Host build of the triangle tree that the nearest-first candidate order
// walks (bvh.cuh gives the layout and the traversal).
//
// The triangles are sorted by the Morton code of their FP32 box centres
// (10 bits per axis over the scene's box, ties to the lower index), then the
// sorted list is split top down: a range of at most kLeaf triangles is a
// leaf, a larger one splits where the surface-area cost
// A(left) n(left) + A(right) n(right) along the list is smallest (ties to the
// split nearest the middle), past depth kSahDepth at the middle, so the depth
// stays below the traversal stack for any scene. A node's child boxes are
// the exact unions of their triangles' outward FP32 boxes; beside the nodes
// the smallest and largest triangle index under each child (the index
// order's bounds) are kept as 4 ints per node.
#include "launch.h"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace dmapk
{
namespace
{

constexpr int kLeaf = 4;      // triangles per leaf, at most (the leaf reference holds counts 1..8)
constexpr int kSahDepth = 24; // below this depth the splits are midpoints
constexpr int kMaxDepth = 63; // the device stack holds 64 entries

struct Box3
{
    float lo[3], hi[3];
};

Box3 empty_box()
{
    return {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
}

void grow(Box3 &b, const Box3 &c)
{
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(b.lo[a], c.lo[a]);
        b.hi[a] = std::max(b.hi[a], c.hi[a]);
    }
}

double half_area(const Box3 &b)
{
    const double x = (double)b.hi[0] - b.lo[0], y = (double)b.hi[1] - b.lo[1], z = (double)b.hi[2] - b.lo[2];
    if (!(x >= 0.0 && y >= 0.0 && z >= 0.0))
        return 0.0;
    return x * y + y * z + z * x;
}

float int_as_float(int i)
{
    float f;
    std::memcpy(&f, &i, sizeof f);
    return f;
}

struct Builder
{
    const std::vector<Box3> &box; // in list order
    const std::vector<int> &tri;  // the triangle at each list position
    std::vector<float> &nodes;
    std::vector<int> &range;      // per node: min0, max0, min1, max1
    std::vector<double> right; // scratch: suffix areas
    int depth_max = 0;

    Box3 range_box(int lo, int hi) const
    {
        Box3 b = empty_box();
        for (int k = lo; k < hi; ++k)
            grow(b, box[k]);
        return b;
    }

    int split(int lo, int hi, int depth)
    {
        const int n = hi - lo, mid = lo + n / 2;
        if (depth >= kSahDepth)
            return mid;
        // suffix areas, then a sweep from the left
        Box3 r = empty_box();
        for (int k = hi - 1; k > lo; --k) {
            grow(r, box[k]);
            right[k] = half_area(r);
        }
        Box3 l = empty_box();
        int best = mid;
        double best_cost = INFINITY;
        for (int k = lo + 1; k < hi; ++k) {
            grow(l, box[k - 1]);
            const double cost = half_area(l) * (k - lo) + right[k] * (hi - k);
            if (cost < best_cost || (cost == best_cost && std::abs(k - mid) < std::abs(best - mid))) {
                best_cost = cost;
                best = k;
            }
        }
        return best;
    }

    // The subtree over list positions [lo, hi): its reference, its box and
    // the smallest and largest triangle index in it.
    int build(int lo, int hi, int depth, Box3 &out, int &min_tri, int &max_tri)
    {
        depth_max = std::max(depth_max, depth);
        if (hi - lo <= kLeaf) {
            out = range_box(lo, hi);
            min_tri = *std::min_element(tri.begin() + lo, tri.begin() + hi);
            max_tri = *std::max_element(tri.begin() + lo, tri.begin() + hi);
            return ~((lo << 3) | (hi - lo - 1));
        }
        const int s = split(lo, hi, depth);
        const size_t v = nodes.size() / 16;
        nodes.resize(nodes.size() + 16, 0.0f);
        range.resize(range.size() + 4, 0);
        Box3 b0, b1;
        int m0, m1, x0, x1;
        const int c0 = build(lo, s, depth + 1, b0, m0, x0);
        const int c1 = build(s, hi, depth + 1, b1, m1, x1);
        float *p = nodes.data() + 16 * v;
        for (int a = 0; a < 3; ++a) {
            p[a] = b0.lo[a];
            p[3 + a] = b0.hi[a];
            p[6 + a] = b1.lo[a];
            p[9 + a] = b1.hi[a];
        }
        p[12] = int_as_float(c0);
        p[13] = int_as_float(c1);
        int *r = range.data() + 4 * v;
        r[0] = m0;
        r[1] = x0;
        r[2] = m1;
        r[3] = x1;
        min_tri = std::min(m0, m1);
        max_tri = std::max(x0, x1);
        out = b0;
        grow(out, b1);
        return (int)v;
    }
};

} // namespace

int build_bvh(const dmapdev::TriDev32 *t32, int n_tri, std::vector<float> &nodes, std::vector<float> &tri_box,
              std::vector<int> &range)
{
    nodes.clear();
    tri_box.clear();
    range.clear();
    if (n_tri <= 0 || n_tri >= (1 << 28))
        return -1;
    // Morton order of the box centres
    float slo[3] = {INFINITY, INFINITY, INFINITY}, shi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < n_tri; ++k)
        for (int a = 0; a < 3; ++a) {
            slo[a] = std::min(slo[a], t32[k].box_lo[a]);
            shi[a] = std::max(shi[a], t32[k].box_hi[a]);
        }
    std::vector<std::pair<uint32_t, int>> code(n_tri);
    for (int k = 0; k < n_tri; ++k) {
        uint32_t m = 0;
        for (int a = 0; a < 3; ++a) {
            const double c = 0.5 * ((double)t32[k].box_lo[a] + (double)t32[k].box_hi[a]);
            const double ext = (double)shi[a] - (double)slo[a];
            const double f = ext > 0.0 ? (c - (double)slo[a]) / ext : 0.0;
            const uint32_t q = (uint32_t)std::min(1023.0, std::max(0.0, f * 1023.0));
            for (int bit = 0; bit < 10; ++bit)
                m |= ((q >> bit) & 1u) << (3 * bit + (2 - a));
        }
        code[k] = {m, k};
    }
    std::sort(code.begin(), code.end());
    std::vector<Box3> box(n_tri);
    std::vector<int> tri(n_tri);
    tri_box.resize((size_t)8 * n_tri);
    for (int k = 0; k < n_tri; ++k) {
        const int t = code[k].second;
        tri[k] = t;
        for (int a = 0; a < 3; ++a) {
            box[k].lo[a] = t32[t].box_lo[a];
            box[k].hi[a] = t32[t].box_hi[a];
            tri_box[8 * (size_t)k + a] = t32[t].box_lo[a];
            tri_box[8 * (size_t)k + 4 + a] = t32[t].box_hi[a];
        }
        tri_box[8 * (size_t)k + 3] = int_as_float(t);
        tri_box[8 * (size_t)k + 7] = 0.0f;
    }
    Builder b{box, tri, nodes, range, std::vector<double>(n_tri + 1, 0.0)};
    Box3 all;
    if (n_tri <= kLeaf) {
        // the root is always an inner node: the triangles, and a leaf whose
        // empty box no ray meets
        nodes.assign(16, 0.0f);
        all = b.range_box(0, n_tri);
        const Box3 none = empty_box();
        for (int a = 0; a < 3; ++a) {
            nodes[a] = all.lo[a];
            nodes[3 + a] = all.hi[a];
            nodes[6 + a] = none.lo[a];
            nodes[9 + a] = none.hi[a];
        }
        nodes[12] = int_as_float(~(n_tri - 1));
        nodes[13] = int_as_float(~0);
        range = {*std::min_element(tri.begin(), tri.end()), *std::max_element(tri.begin(), tri.end()), n_tri, -1};
        return 1;
    }
    int min_tri, max_tri;
    b.build(0, n_tri, 0, all, min_tri, max_tri);
    return b.depth_max < kMaxDepth ? b.depth_max : -1;
}

} // namespace dmapk
