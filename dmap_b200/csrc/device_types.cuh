// Device-side records shared by the kernels of dmap_b200.
//
// HBM layout
//   node grid   (W x W) values of the asset's dtype, row pitch `pitch`
//               elements (a multiple of 16 bytes so TMA can tile it)
//   pyramid64   per level l (m = n_leaf >> l cells per side), row-major
//               [j*m + i], 8 doubles per cell (h0 gu gv r ru rv h_min h_max):
//               64 B, the reference's TaylorNode (taylor_pyramid.h:63-66)
//   pyramid32   the same cells as 8 floats (32 B = one DRAM sector) rounded
//               outward: h0/gu/gv to nearest with r/ru/rv widened by the
//               rounding, h_min down, h_max up
//   triangles   one TriDev (FP64) and one TriDev32 (FP32) record each
#pragma once
#include <cmath>
#include <cstdint>

namespace dmapdev
{

constexpr int kMaxLevels = 24;

struct AssetDev
{
    const void *nodes;   // node grid
    int dtype;           // 0 f32, 1 f16, 2 f64, 3 bf16
    int W;               // nodes per side (2^L + 1)
    int pitch;           // elements per row
    int n_leaf;          // 2^L
    int n_levels;        // L + 1
    int repeat;
    double scale, offset;
    const double *pyr64; // may be null
    const float *pyr32;
    int64_t level_off[kMaxLevels]; // first cell of each level
};

// One base triangle with everything the FP64 walk reads
// (BaseTriangle, TangentFrame, UvTriangle, DisplacedIntersector fields).
struct TriDev
{
    double q0[3], e1[3], e2[3], m0[3], Mu[3], Mv[3];
    double t0[2], t1[2], t2[2];
    double J[2][2];
    double A[3][3]; // to_tangent
    double ng[3];
    double wn[3];           // winding normal (p1 - p0) x (p2 - p0)
    double un[3][2], ud[3]; // inward edge normals and offsets
    double lo[2], hi[2];    // texture-space bounding box of the domain
    double residual_tol;
    double box_lo[3], box_hi[3];
    double h_min, h_max;
    int root_level, n_roots, asset, status;
    int roots_i[4], roots_j[4];
    // 1 + the index of the non-rigid instance the triangle belongs to
    // (instance.cuh), 0 for a triangle placed in world space
    int inst, inst_pad;
};

// The FP32 record: the same geometry rounded to float, plus the FP64 frame
// origin and matrix for the per-ray transform.
struct TriDev32
{
    float e1[3], e2[3], m0[3], Mu[3], Mv[3];
    float q0f[3];
    float t0[2], t1[2], t2[2];
    float J[2][2];
    float Af[3][3];        // to_tangent rounded to nearest
    float un[3][2], ud[3]; // domain edges (exact for dyadic texture coordinates)
    float lo[2], hi[2];
    float box_lo[3], box_hi[3]; // object AABB widened outward
    float residual_tol;
    float newton_tol;      // FP32 acceptance tolerance of the Newton residual
    float mean_edge;
    int root_level, n_roots, asset, pad;
    int roots_i[4], roots_j[4];
    double A[3][3];        // to_tangent in double for the ray transform
    double q0[3];
    // The interpolated normal in tangent space, A N(s,t) = a0 + s au + t av,
    // and |N(s,t)|^2 = qc + 2 s q1 + 2 t q2 + s^2 q11 + 2 s t q12 + t^2 q22,
    // rounded from double; rowsum[i] = sum_j |A_ij| bounds |A n| for a unit n.
    float a0[3], au[3], av[3];
    float qc, q1, q2, q11, q12, q22;
    float rowsum[3];
};

// Device status word bits (written with atomicOr).
constexpr unsigned kStatusCapped = 1u;
constexpr unsigned kStatusBadInput = 2u;

// A ray the query cannot answer: a non-finite origin or direction
// component, a zero direction, or a NaN t_min / t_max. Such a ray is
// answered as a miss (the reference has no defined result for it).
__host__ __device__ __forceinline__ bool ray_unanswerable(const double *o, const double *d, double t_min,
                                                          double t_max)
{
    bool bad = t_min != t_min || t_max != t_max || (d[0] == 0.0 && d[1] == 0.0 && d[2] == 0.0);
#pragma unroll
    for (int a = 0; a < 3; ++a)
        bad = bad || !(fabs(o[a]) <= 1.7976931348623157e308) || !(fabs(d[a]) <= 1.7976931348623157e308);
    return bad;
}

// An unanswerable ray is replaced by one that every box test rejects
// (t_min > t_max), so every kernel answers it as a miss without a branch of
// its own.
__host__ __device__ __forceinline__ void sanitize_ray(double *o, double *d, double &t_min, double &t_max)
{
    if (ray_unanswerable(o, d, t_min, t_max)) {
        o[0] = o[1] = o[2] = 0.0;
        d[0] = 1.0;
        d[1] = d[2] = 0.0;
        t_min = 1.0;
        t_max = 0.0;
    }
}

// Hit records, laid out as dmap_hit32 / dmap_hit64 of include/dmap_b200.h.
struct Hit32
{
    float t, st[2], bary[2], ng[3];
    int32_t tri, i, j, flags;
};
struct Hit64
{
    double t, st[2], bary[2], ng[3];
    int32_t tri, i, j, flags;
};

} // namespace dmapdev

// Hit flag bits, as DMAP_HIT_* of include/dmap_b200.h (which defines the
// same names when it is included first).
#ifndef DMAP_HIT_FP64_LEAF
#define DMAP_HIT_FP64_LEAF 1 // the root came from the FP64 certified Newton leaf
#endif
#ifndef DMAP_HIT_CAPPED
#define DMAP_HIT_CAPPED 2 // a walk cap of the query ran out for this ray
#endif
#ifndef DMAP_HIT_POLISHED
#define DMAP_HIT_POLISHED 4 // an FP32 leaf root refined by FP64 Newton (ill-conditioned Jacobian)
#endif

// Per-ray counter slots (TraversalStats), as DMAP_ST_* of include/dmap_b200.h.
enum
{
    DMAP_ST_TRI = 0,
    DMAP_ST_NODE = 1,
    DMAP_ST_LEAF = 2,
    DMAP_ST_SUB = 3,
    DMAP_ST_NEWTON = 4,
    DMAP_ST_NAH = 5,
    DMAP_ST_LAH = 6,
    DMAP_ST_N = 8
};
