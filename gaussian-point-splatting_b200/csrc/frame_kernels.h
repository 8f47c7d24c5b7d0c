// Internal interface between the frame driver (renderer.cu) and the sm_100a kernels
// (frame_kernels.cu).  Nothing here crosses the C-ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gps_math.cuh"
#include "gps_scene.cuh"

namespace gps {

// Per-surviving-Gaussian data the splat needs, produced once by the preprocess (the
// reference recomputes this per point, gaussian_point_splatting.cu:416-423).  64 bytes:
//   a = (pixel_mean.x, pixel_mean.y, c0, c1)   Cholesky factor of cov2d
//   b = (c2, conic.x, conic.y, conic.z)
//   c = (opacity, colour.r, colour.g, colour.b) colour is the SH evaluation of this frame
//   d = (min.x | min.y << 16, max.x | max.y << 16, key.lo, key.hi)  key = depth28<<36 | rgb36
struct SplatRecord {
    float4 a, b, c;
    uint4 d;
};

// Hi-Z max-depth pyramid layout (depth_mip_chain.cuh:10-71).
struct HizView {
    float* mip;
    int width, height, levels;
    uint64_t mip_size;
    int level_w[16];
    int level_h[16];
    uint64_t level_off[16];
    unsigned* done;        // block counter of the one-launch build (zero between builds)
};

// Fixed-size contiguous Gaussian blocks with AABBs (gaussian_bvh.cuh:8-53).
struct BlockView {
    const float4* nodes;   // 2 float4 per node: (min.xyz, begin bits), (max.xyz, count bits)
    uint32_t* culled;      // one bit per node, 32 nodes per word
    uint32_t node_count;
    uint32_t words;
    uint32_t per_block;    // Gaussians per block
    uint32_t* chunk_count; // visible-chunk counter, reset by the block cull
};

// Device-side counters of one render pass, readable by later kernels without a host sync.
struct PassCounters {
    uint32_t survivors;    // Gaussians with at least one point
    uint32_t total_points; // sum of point counts (u32, wraps like the reference)
    uint32_t points;       // min(total_points, max_number_of_points)
    uint32_t truncated;    // 1 if the point budget clipped the tail
    uint32_t scan_timeouts;  // always 0: no device-side wait can give up
    uint32_t loaded;         // Gaussians whose attributes the pass's preprocess read (after the
                             // block cull and pass 2's previous-mask test); 0 without a tally
    uint32_t crowded;        // 1 if a screen bin held more than kBinCrowded survivors: the
                             // pass is walked in Gaussian order
    uint32_t pad;
};

struct FrameConst {
    mat4 vp, view, cam;
    vec2 tan_fov, focal;
    int up_width, up_height;
    int num_passes;        // samples per pixel
    int ss;                // supersampling factor
    int k_points;          // points per thread in the splat (ss*ss or 1)
    float near_plane, far_plane;
    vec4 planes[6];
    int use_unbiased;
    int reduce_point_count;
    int cull_small;
    int enable_occlusion;
    int enable_hier;
    int width, height;
};

struct PreprocessArgs {
    FrameConst fc;
    int frame_seed;
    int only_previously_occluded;
    uint32_t n;
    uint32_t* counts;
    uint32_t* mask_cur;
    const uint32_t* mask_prev;
    SplatRecord* records;
    HizView hiz;
    BlockView blocks;
    const uint32_t* chunk_list;   // 32-Gaussian chunks with a visible block (null: every chunk)
    const uint32_t* chunk_count;
    int immediate_threshold;      // > 0: splat Gaussians of <= this many points in the preprocess
    uint64_t* buffer;             // splat buffer (immediate splatting only)
    // When mask_iter is set, mask_cur / mask_prev are mask_pair[it & 1] / mask_pair[(it + 1) & 1]
    // for the device-side pass counter it (see ScanArgs::mask_iter).
    uint32_t* mask_pair[2];
    const uint32_t* mask_iter;
    uint32_t* loaded;             // tally of Gaussians whose attributes were read (null: none)
    // Pass workload accumulated here (render path; null: not accumulated): per scan tile of
    // 2^tile_shift Gaussians, survivors in the high and points (mod 2^32) in the low word; per
    // screen bin, survivors << 32 | points.  Both are zero on entry.
    unsigned long long* tile_totals;
    int tile_shift;
    unsigned long long* bins;
    int bin_shift, bins_x, bins_y;
    int bin_sub_log2;  // each screen bin has 2^bin_sub_log2 cursors (see kBinSubs)
    uint32_t bin_count;  // bins_x * bins_y
};

struct ScanArgs {
    const uint32_t* counts;
    const uint32_t* mask;
    // Survivor masks A/B and the device-side pass counter choosing between them (null: `mask`
    // is used as given).  The counter advances after a pass only when its point total is
    // non-zero: WorkloadDistributor::build returns before iteration++ when it has no samples
    // (workload_distributor.cu:107-111,145), so the next pass reuses the same mask pair order.
    const uint32_t* mask_pair[2];
    uint32_t* mask_iter;
    uint32_t n;
    uint32_t max_points;
    uint32_t tile_points;        // points per splat tile
    uint32_t* surv_gid;          // [n] compacted Gaussian ids of survivors
    uint32_t* surv_start;        // [n] first point of each survivor
    uint32_t* tile_first_rank;   // [ceil(max_points / tile_points) + 1]
    unsigned long long* tile_state;  // [scan tiles] tile totals, then tile prefixes
    PassCounters* counters;
    uint32_t* loaded;            // the preprocess's tally: moved into counters->loaded and reset
    // Screen binning in the downsweep (render path; null bins: Gaussian order): the bin scan runs
    // beside the tile scan, and the downsweep scatters the survivors into bin order
    unsigned long long* bins;
    uint32_t nbins;
    int bin_shift, bins_x, bins_y, up_width, up_height;
    int bin_sub_log2;            // cursors per screen bin, log2 (see kBinSubs)
    uint32_t bin_count;          // bins_x * bins_y (nbins = bin_count << bin_sub_log2)
    const SplatRecord* records;
    uint32_t* sorted_gid;        // [n] survivors in bin order
    uint32_t* sorted_pstart;     //     their first points (reference point indices)
    uint32_t* sorted_qstart;     //     their first walk positions in bin order
    uint32_t bin_crowded;        // survivors of one bin past which the pass keeps Gaussian order
};

struct SplatArgs {
    FrameConst fc;
    int frame_seed;
    const SplatRecord* records;
    const uint32_t* surv_gid;        // survivors in Gaussian order: a walk position is a point index
    const uint32_t* surv_start;      // first point of each survivor (monotone)
    const uint32_t* tile_first_rank;
    const PassCounters* counters;
    uint64_t* buffer;
    uint32_t n;
    // Screen-binned order (null sorted_gid, or a truncated pass: Gaussian order): survivor i's
    // points are the reference's point indices sorted_pstart[i] + (q - sorted_qstart[i]).
    const uint32_t* sorted_gid;
    const uint32_t* sorted_qstart;
    const uint32_t* sorted_pstart;
    // cleared for the next pass once this pass's workload is consumed (null: nothing)
    unsigned long long* clear_a;
    uint32_t clear_a_words;
    unsigned long long* clear_b;
    uint32_t clear_b_words;
    uint32_t* mask_iter;             // advanced after a pass with points (null: not here)
};

// Screen bins: the splat walks a pass's survivors grouped by the 64x64 splat-buffer tile (or
// block of tiles, for very large views) that holds their pixel mean, so that blocks running at
// the same time write a compact part of the buffer.  Only the order changes: every point keeps
// its reference point index (its seed) and the min is order-free.
constexpr uint32_t kMaxBins = 16384;  // screen bins per pass (bins widen beyond 8192 x 8192 pixels)
#ifndef GPS_BIN_CROWDED
#define GPS_BIN_CROWDED 131072
#endif
// Survivors of one bin past which binning costs more than it saves: each takes its place with
// an atomic on one of the bin's cursors, and those serialise.  The environment
// variable GPS_BIN_CROWDED overrides it when a renderer is created.
constexpr uint32_t kBinCrowded = GPS_BIN_CROWDED;
// Cursors per screen bin (at most; fewer where bins x cursors would pass kMaxBins): a survivor
// takes its place on cursor (its 32-Gaussian chunk mod kBinSubs), so that the survivors of one
// bin spread their atomics over that many addresses.  Cursor k of bin b is stored at word
// k * bin_count + b, so that a bin's cursors sit in different cache lines (L2 slices), while the
// order takes them as (b, k): a bin's cursors are consecutive and the walk still takes the bin
// as a unit.
#ifndef GPS_BIN_SUBS
#define GPS_BIN_SUBS 4
#endif
constexpr uint32_t kBinSubs = GPS_BIN_SUBS;  // a power of two, at most 4 (the bin scan's words per thread)
#ifndef GPS_SPLAT_BINNED
#define GPS_SPLAT_BINNED 1
#endif
// Views whose splat buffer is smaller than this are walked in Gaussian order: their buffer
// stays in L2 whatever the order, and their few bins (60 at 640x360) would put every cursor
// atomic of the pass on a handful of cache lines.
#ifndef GPS_BIN_MIN_BUFFER_MB
#define GPS_BIN_MIN_BUFFER_MB 64
#endif
constexpr uint64_t kBinMinBufferBytes = (uint64_t)GPS_BIN_MIN_BUFFER_MB << 20;
#ifndef GPS_BIN_SHIFT
#define GPS_BIN_SHIFT 6  // log2 of the bin width in pixels: one 64x64 splat-buffer tile
#endif
GPS_HD uint32_t screen_bin(float pmx, float pmy, int up_width, int up_height, int bin_shift, int bins_x, int bins_y) {
    const float x = fminf(fmaxf(pmx, 0.0f), (float)(up_width - 1));  // NaN -> 0
    const float y = fminf(fmaxf(pmy, 0.0f), (float)(up_height - 1));
    const int bx = min((int)x >> bin_shift, bins_x - 1);
    const int by = min((int)y >> bin_shift, bins_y - 1);
    return (uint32_t)(by * bins_x + bx);
}

struct ResolveArgs {
    const uint64_t* buffer;
    float* color;          // float3 per pixel (may be null for depth-only)
    float* depth;
    int width, height, num_passes, ss;
    uint64_t entries;
    float near_plane, far_plane;
    uint64_t initial_value;
};

// launchers (all asynchronous on `stream`)
void launch_block_cull(const BlockView& b, const FrameConst& fc, const HizView& hiz, cudaStream_t stream);
// Lists the 32-Gaussian chunks that hold at least one unculled block and zeroes the survivor
// mask words of the others.
// Zeroes the survivor-mask words of chunks without a visible block in the current mask: mask_a,
// or the one of (mask_a, mask_b) that *mask_iter selects when mask_iter is set.
void launch_visible_chunks(const BlockView& b, uint32_t n, uint32_t* list, uint32_t* mask_a, uint32_t* mask_b,
                           const uint32_t* mask_iter, cudaStream_t stream);
void launch_preprocess_fp32(const PreprocessArgs& a, const SceneFP32& s, cudaStream_t stream);
void launch_preprocess_compressed(const PreprocessArgs& a, const SceneCompressed& s, cudaStream_t stream);
void launch_preprocess_half(const PreprocessArgs& a, const SceneHalf& s, cudaStream_t stream);
// half-precision scenes (load time)
void launch_encode_half(const float4* pos_op, const float4* rot, const float4* scale, const float4* sh, uint32_t n,
                        float4* origin, uint4* rec, uint4* scl, uint4* acq, cudaStream_t stream);
void launch_translate_origins(const float4* src, uint32_t count, float dx, float dz, float4* dst, cudaStream_t stream);
void launch_tile_nodes(const float4* src, uint32_t src_pb, uint32_t src_n, uint32_t pb, uint32_t copies,
                       const float2* offsets, uint64_t total, float4* dst, uint32_t nodes, cudaStream_t stream);
void launch_scan(const ScanArgs& a, uint32_t scan_tiles, cudaStream_t stream);
// The render path's scan over the tile totals the preprocess accumulated: the tile scan (and the
// bin scan), then the downsweep that compacts the survivors, bins them and finds each splat
// tile's first survivor.  Two launches.
void launch_scan_fused(const ScanArgs& a, cudaStream_t stream);
int scan_tile_shift(uint32_t n);
uint32_t scan_tile_count(uint32_t n);
constexpr uint32_t kScanTileGaussians = 16384;  // Gaussians per scan tile (counts are padded to it)
void launch_splat(const SplatArgs& a, int grid, int block, cudaStream_t stream);
void launch_clear(uint64_t* buf, uint64_t entries, uint64_t value, cudaStream_t stream);
void launch_resolve(const ResolveArgs& a, bool depth_only, cudaStream_t stream);
void launch_hiz_build(const HizView& h, const float* depth, int min_levels, cudaStream_t stream);
void launch_block_bounds(const float4* pos_op, const float4* rot, const float4* scale, uint32_t n,
                         uint32_t per_block, float4* nodes, cudaStream_t stream);
// Scene order on the device: order[j] = the input index of the j-th Gaussian in 3D Morton order
// of the means, the order the host reorder (morton_sort) gives, key for key and tie for tie.
// Allocates its own scratch; synchronizes the stream.
cudaError_t morton_order_device(const float4* pos_op, uint32_t n, uint32_t* order, cudaStream_t stream);
// dst[j * per + k] = src[order[j] * per + k]
void launch_gather_rows(const float4* src, const uint32_t* order, uint32_t n, uint32_t per, float4* dst,
                        cudaStream_t stream);
void launch_taa(uint8_t* image, float* out_color, const float* cur_color, const float* prev_color,
                const float* cur_depth, const float* prev_depth, const mat4& reproj, float blend, int width, int height,
                int frame_number, cudaStream_t stream);
void launch_progressive(uint8_t* image, float* cur_color, float* accum, int width, int height, int frames,
                        cudaStream_t stream);
int splat_grid_size(int block);

}  // namespace gps
