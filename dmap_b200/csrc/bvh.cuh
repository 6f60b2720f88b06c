// The candidate orders over a bounding volume hierarchy of the scene's
// triangles, for scenes of more than 256 triangles.
//
// Both orders are fixed by a key per triangle: the nearest-first order's
// FP64 box entry (order.cuh), the index order's own index (the reference's
// flat loop). A ray's next triangle is the smallest (key, index) past the
// cursor among the triangles whose float box the ray still meets with its
// current t_max. A lane keeps a sorted buffer of the
// kNearBuf smallest candidates past a scan cursor, found by one traversal of
// the tree (bvh_refill), and takes them in order, re-testing each box with
// the current t_max when it comes up (t_max only shrinks, so a candidate
// that fails then stays out, as it would for a full scan). Every triangle
// the buffer does not hold comes after its last entry, so once the buffer is
// spent the next refill starts past that entry; a buffer that came back with
// fewer than kNearBuf entries held every candidate left. The picks are
// therefore the ones a scan over every triangle makes, in the same order.
//
// Tree layout (built on the host, bvh.cu): node v is 16 floats, the boxes of
// its two children (lo0, hi0, lo1, hi1) and their references (as int bits):
// >= 0 an inner node, < 0 a leaf ~(first << 3 | (count - 1)) over positions
// first .. first + count - 1 of the triangle list. The list holds per
// position two float4: (lo, triangle index as int bits) and (hi, 0), the
// triangle's own outward FP32 box. Beside the nodes, 4 ints per node hold
// the smallest and largest triangle index under each child (min0, max0,
// min1, max1). Node 0 is the root.
#pragma once
#include "box32.cuh"
#include "order.cuh"

namespace d32
{

constexpr int kNearBuf = 8;   // candidates one refill keeps
constexpr int kBvhStack = 64; // the host build keeps the depth below this

// A lane's buffered candidates: n < 0 none (the next pick refills from the
// ray's own cursor), else n sorted entries of which pos are taken.
struct NearBuf
{
    double key[kNearBuf];
    int tri[kNearBuf];
    int n, pos;
};

struct BvhView
{
    const float4 *nodes;
    const float4 *tri_box;
    const int4 *range;
    int n_nodes;
};

// A subtree's bound as a key: the entry distance, or (index order) the
// smallest index under it, stored as int bits.
template <bool NEAR>
__device__ __forceinline__ double bound_of(float e)
{
    return NEAR ? (double)e : (double)__float_as_int(e);
}

// The kNearBuf smallest (key, index) past (sk, sidx) among the triangles
// whose float box the ray meets within [tmin_f, tmf], sorted, into bk / bt;
// NEAR: the keys are the FP64 box entries, else the indices themselves.
// Returns how many there are (kNearBuf: more may follow the last), or -1
// when the traversal overran its stack or its visit budget (neither happens
// for a tree the host built). Subtrees are entered smallest bound first and
// skipped when the ray misses their box or when their bound (a lower bound
// of their triangles' keys: the box entry, or the smallest index under them)
// is past the buffer's last entry once it is full, and when they lie wholly
// before the cursor: in the index order every index under them is at most
// the cursor's; in the nearest order their exit bound is before the cursor
// (a triangle with a key past its box's exit meets the ray nowhere, and one
// with a key before the cursor was taken already).
template <bool NEAR>
__device__ __noinline__ int bvh_refill(const BvhView v, const TriDev *__restrict__ tris64, const double *o,
                                       const double *d, const double *inv, double t_min, const float *of,
                                       const float *df, const float *invf, float tmin_f, float tmf, double sk,
                                       int sidx, double *bk, int *bt)
{
    int n = 0;
    int sref[kBvhStack];
    float se[kBvhStack];
    int sp = 0;
    int ref = 0;
    const int budget = 2 * v.n_nodes + 2;
    for (int visit = 0; visit < budget; ++visit) {
        if (ref >= 0) {
            const float4 *p = v.nodes + 4 * (int64_t)ref;
            const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), q = __ldg(p + 3);
            const float lo0[3] = {a.x, a.y, a.z}, hi0[3] = {a.w, b.x, b.y};
            const float lo1[3] = {b.z, b.w, c.x}, hi1[3] = {c.y, c.z, c.w};
            float e0 = tmin_f, x0 = tmf, e1 = tmin_f, x1 = tmf;
            bool p0 = node_range(lo0, hi0, of, df, invf, tmin_f, e0, x0);
            bool p1 = node_range(lo1, hi1, of, df, invf, tmin_f, e1, x1);
            // the children's bounds: entry distances, or (index order) their
            // smallest indices as int bits in the float slots, with the
            // largest ones in place of the exits
            if (!NEAR) {
                const int4 ix = __ldg(v.range + ref);
                e0 = __int_as_float(ix.x);
                x0 = __int_as_float(ix.y);
                e1 = __int_as_float(ix.z);
                x1 = __int_as_float(ix.w);
            }
            // past the buffer's last entry, or wholly before the cursor (the
            // exit with a margin far above the FP64 rounding of the keys)
            auto keep = [&](float e, float x) {
                if (n == kNearBuf && bound_of<NEAR>(e) > bk[kNearBuf - 1])
                    return false;
                if (!NEAR)
                    return (double)__float_as_int(x) > sk;
                return !((double)x + 1.52587890625e-05 * fmax(1.0, fabs((double)x)) < sk);
            };
            p0 = p0 && keep(e0, x0);
            p1 = p1 && keep(e1, x1);
            const int c0 = __float_as_int(q.x), c1 = __float_as_int(q.y);
            if (p0 && p1) {
                if (sp == kBvhStack)
                    return -1;
                const bool first0 = bound_of<NEAR>(e0) <= bound_of<NEAR>(e1);
                sref[sp] = first0 ? c1 : c0;
                se[sp] = first0 ? e1 : e0;
                ++sp;
                ref = first0 ? c0 : c1;
                continue;
            }
            if (p0 || p1) {
                ref = p0 ? c0 : c1;
                continue;
            }
        } else {
            const int leaf = ~ref, first = leaf >> 3, cnt = (leaf & 7) + 1;
            for (int k = first; k < first + cnt; ++k) {
                const float4 l = __ldg(v.tri_box + 2 * (int64_t)k), h = __ldg(v.tri_box + 2 * (int64_t)k + 1);
                const float blo[3] = {l.x, l.y, l.z}, bhi[3] = {h.x, h.y, h.z};
                const int t = __float_as_int(l.w);
                double key = (double)t;
                if (!NEAR && (!d64::after_cursor(key, t, sk, sidx) ||
                              (n == kNearBuf && !d64::before_best(key, t, bk[kNearBuf - 1], bt[kNearBuf - 1]))))
                    continue; // the index tests first: they need no box
                float e = tmin_f, tt = tmf;
                if (!box_range(blo, bhi, of, df, invf, e, tt))
                    continue;
                if (NEAR) {
                    if (n == kNearBuf && (double)e > bk[kNearBuf - 1])
                        continue;
                    key = d64::entry_key(tris64[t], o, d, inv, t_min);
                    if (!d64::after_cursor(key, t, sk, sidx))
                        continue;
                    if (n == kNearBuf && !d64::before_best(key, t, bk[kNearBuf - 1], bt[kNearBuf - 1]))
                        continue;
                }
                int j = n < kNearBuf ? n++ : kNearBuf - 1;
                for (; j > 0 && d64::before_best(key, t, bk[j - 1], bt[j - 1]); --j) {
                    bk[j] = bk[j - 1];
                    bt[j] = bt[j - 1];
                }
                bk[j] = key;
                bt[j] = t;
            }
        }
        // the next pushed subtree that can still hold one of the smallest
        for (;;) {
            if (sp == 0)
                return n;
            --sp;
            if (n == kNearBuf && bound_of<NEAR>(se[sp]) > bk[kNearBuf - 1])
                continue;
            ref = sref[sp];
            break;
        }
    }
    return -1;
}

// The ray's next triangle in the order (NEAR: nearest first, else index),
// or -1 when none is left (also on a traversal overrun, which sets `err`).
// On a pick the cursor (ckey, cidx) moves to it and t1 is the exit bound of
// its box test.
template <bool NEAR>
__device__ __forceinline__ int near_next(NearBuf &b, const BvhView v, const TriDev32 *__restrict__ tris32,
                                         const TriDev *__restrict__ tris64, const double *o, const double *d,
                                         const double *inv, double t_min, const float *of, const float *df,
                                         const float *invf, float tmin_f, float tmf, double &ckey, int &cidx,
                                         float &t1, bool &err)
{
    // each refill starts past the previous one's last entry: at most one per
    // kNearBuf triangles (a leaf holds at most 4, so fewer than n_nodes + 4)
    for (int refill = 0; refill <= v.n_nodes + 4; ++refill) {
        while (b.pos < b.n) {
            const int t = b.tri[b.pos];
            const double k = b.key[b.pos];
            ++b.pos;
            float e = tmin_f, tt = tmf;
            if (box_range(tris32[t].box_lo, tris32[t].box_hi, of, df, invf, e, tt)) {
                ckey = k;
                cidx = t;
                t1 = tt;
                return t;
            }
        }
        if (b.n >= 0 && b.n < kNearBuf)
            return -1;
        // every candidate not buffered comes after the last buffered one
        const bool own = b.n < 0;
        const double sk = own ? ckey : b.key[kNearBuf - 1];
        const int si = own ? cidx : b.tri[kNearBuf - 1];
        b.n = bvh_refill<NEAR>(v, tris64, o, d, inv, t_min, of, df, invf, tmin_f, tmf, sk, si, b.key, b.tri);
        b.pos = 0;
        if (b.n < 0)
            break;
    }
    b.n = 0;
    err = true;
    return -1;
}

} // namespace d32
