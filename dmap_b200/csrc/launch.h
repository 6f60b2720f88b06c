// Host-side launchers of the device kernels (one per translation unit), called
// by the C-ABI layer in api.cu.
#pragma once
#include "device_types.cuh"
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace dmapk
{

// Per-query options as the kernels read them.
struct QueryOpts
{
    int bound, slab_max_level, leaf, mode;
    double polish_cond;
    int ray_dtype, hit_dtype; // 0 f32, 2 f64
    int precision;            // DMAP_PRECISION_*
    int schedule;             // DMAP_SCHEDULE_*
    int rounds;               // wavefront: walk/leaf rounds before the inline-leaf drain
    int blocks_per_sm;        // wavefront walk: 128-thread CTAs per SM (0: the walk's compiled occupancy)
    int order = 1;            // DMAP_ORDER_*: 0 index order, 1 nearest box entry first
    int guard_cap = 1 << 26;  // FP32 walk: cells one triangle walk may visit before it gives up
    int leaf_precision = 0;   // FP32 walk: DMAP_PRECISION_F64 (the reference's leaf) or _F32 (leaf32.cuh)
    // When set, the number of rays is read here on the device when the query
    // runs (at most the n the launch is given, which sizes grids and scratch):
    // stages of a device-driven pipeline pass counts they produced themselves.
    const long long *n_dev = nullptr;
    // Scenes of more than 256 triangles: the tree over the triangles' FP32
    // boxes that both candidate orders walk (bvh.cuh gives the layout), bvh_n_nodes
    // inner nodes of 4 float4, 2 float4 per triangle list position.
    // Non-rigid instances: kInstDoubles per instance (instance.cuh), indexed
    // by TriDev::inst - 1; null when the scene has none.
    const double *inst_xf = nullptr;
    const float4 *bvh_nodes = nullptr;
    const float4 *bvh_tri = nullptr;
    const int4 *bvh_range = nullptr;
    int bvh_n_nodes = 0;
    // The scene's opacity filter (dmap_scene_set_opacity): op_h rows of op_w
    // mask texels, 0 transparent; op_tri flags the triangles it covers
    // (nullptr: every one); the object uv map of the crossings' coordinates.
    const unsigned char *op_mask = nullptr;
    const unsigned char *op_tri = nullptr;
    int op_w = 0, op_h = 0, op_flip = 0;
    double op_scale[2] = {1.0, 1.0}, op_offset[2] = {0.0, 0.0};
};

constexpr int kMaxRounds = 32;
// Counters of a wavefront scratch: 4 per round (kMaxRounds + 1 rounds), then
// the length of the filter's rerun list.
constexpr int kWaveCounters = 4 * (kMaxRounds + 1) + 1;

// Device scratch of the wavefront schedule for up to `capacity` rays: the
// parked walk states, two ray queues (resume in / resume out), the leaf
// jobs, the counters, and the rays a filtered scene answers again on the
// filter's own schedule (a crossing the filter rejects was taken).
struct WaveScratch
{
    void *state = nullptr;
    int *queue[2] = {nullptr, nullptr};
    void *leaves = nullptr;
    unsigned long long *counters = nullptr;
    int *rerun = nullptr;
    int64_t capacity = 0;
};
size_t wave_state_bytes();
size_t wave_leaf_bytes();
// Kernel launches one FP32 query makes under these options.
int walk32_launches(const QueryOpts &opt);

// Pyramid build (pyramid.cu). `tmap` is an encoded CUtensorMap over the node
// grid (128 bytes), `tile` the leaf cells per CTA side. Writes the FP64
// levels without the offset into pyr64 and the outward-rounded FP32 levels
// with it into pyr32.
// all64: write every FP64 level (the FP64 pyramid is kept); otherwise only
// the levels the fold launches read back, which are scratch.
cudaError_t launch_pyramid(const void *tmap, const dmapdev::AssetDev &a, int tile, double *pyr64, float *pyr32,
                           unsigned *status, cudaStream_t stream, bool all64 = true);

// The Direct build (taylor_pyramid.cpp:151-202): every level from the node
// grid. hull_scratch holds 32 bytes per pyramid cell plus 32768 x 32 bytes
// of partial hulls; 2 or 3 launches per level (direct_launches).
int direct_launches(int n_leaf);
cudaError_t launch_pyramid_direct(const dmapdev::AssetDev &a, double *pyr64, float *pyr32, void *hull_scratch,
                                  cudaStream_t stream, bool all64);

// Per-triangle setup (setup.cu) over records of `stride` doubles: vertex
// records (kVertexRecord) or BaseTriangle chart records (kChartRecord).
constexpr int kVertexRecord = 24;
constexpr int kChartRecord = 37;
cudaError_t launch_setup(const double *tris_dev, int stride, const int *tri_asset_dev,
                         const dmapdev::AssetDev *assets_dev, int n_tri, dmapdev::TriDev *out,
                         dmapdev::TriDev32 *out32, unsigned *status, cudaStream_t stream);

// The tree over the triangles' FP32 boxes for the candidate orders
// (bvh.cu; the layout is bvh.cuh's): 16 floats per inner node, 8 per
// triangle list position, 4 ints of child index ranges per inner node. Returns the tree's depth, or -1 when it would not
// fit the traversal stack.
int build_bvh(const dmapdev::TriDev32 *t32, int n_tri, std::vector<float> &nodes, std::vector<float> &tri_box,
              std::vector<int> &range);

// The FP64 walk, one thread per ray over every triangle (walk64.cu).
cudaError_t launch_walk64(const dmapdev::TriDev *tris, int n_tri, const dmapdev::AssetDev *assets, const void *rays,
                          int64_t n, const QueryOpts &opt, void *hits, int64_t *stats, unsigned *status,
                          cudaStream_t stream);

// The FP32 walk (walk32.cu). The wavefront schedule needs `ws` sized for n
// rays; the launcher zeroes its counters (and `stats`) on `stream`.
cudaError_t launch_walk32(const dmapdev::TriDev32 *tris32, const dmapdev::TriDev *tris64, int n_tri,
                          const dmapdev::AssetDev *assets, const void *rays, int64_t n, const QueryOpts &opt,
                          void *hits, int64_t *stats, unsigned *status, const WaveScratch &ws, cudaStream_t stream);

} // namespace dmapk
