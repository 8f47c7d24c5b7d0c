// sm_100a kernels of the Gaussian point-splatting frame path.
//
//   block cull    gaussian_bvh.cu:215-329          one thread per block node, warp ballot
//   preprocess    gaussian_point_splatting.cu:17-65,147-307
//   scan          workload_distributor.cu:52-145   tile reduce -> tile scan -> downsweep that
//                                                  compacts survivors and keeps P on the device
//   splat         gaussian_point_splatting.cu:67-141,383-432  persistent, tile-of-points blocks
//   clear/resolve gaussian_point_splatting.cu:484-548,580-585
//   Hi-Z          depth_mip_chain.cu:7-145, depth_mip_chain.cuh:172-215
//   TAA/progress  post_processing_kernels.cuh:108-285
//
// Every floating-point expression that decides a sample position, a count or a packed
// value follows the reference's expression shape (see gps_math.cuh) so that the 64-bit
// splat buffer is bit-identical to the reference kernels' for the same inputs.
#include <type_traits>
#include <cstdio>
#include <mutex>
#include <string>
#include "../../include/gps_b200.h"
#include "frame_kernels.h"
#include "gps_rng.cuh"
#include "host_io.hpp"

namespace gps {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;   // per thread and round
constexpr int kScanRoundsMax = 4;  // a thread covers kScanItems * rounds consecutive Gaussians:
                                   // 1 round (4096-Gaussian tiles) below kScanBigScene, else 4
constexpr uint32_t kScanTile = kScanThreads * kScanItems * kScanRoundsMax;  // largest tile, 16384
constexpr uint32_t kScanTileSmall = kScanThreads * kScanItems;             // 4096
constexpr uint32_t kScanBigScene = 32u << 20;

// ---------------------------------------------------------------------------------
// Hi-Z query (depth_mip_chain.cuh:172-215, the non-tree variant the reference compiles)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ bool hiz_occluded(const HizView& c, float depth, ivec2 mn, ivec2 mx) {
    mn.x = max(0, mn.x);
    mn.y = max(0, mn.y);
    mx.x = min(c.width - 1, mx.x);
    mx.y = min(c.height - 1, mx.y);
    int w = mx.x - mn.x + 1;
    int h = mx.y - mn.y + 1;
    int d = max(w, h);
    int lod = (int)ceilf(log2f((float)d / 2.0f));
    lod = min(max(lod, 0), c.levels - 1);
    int l = (c.levels - 1) - lod;
    const int wl = c.level_w[l];
    const int hl = c.level_h[l];
    int tile_w = max(1, min(c.width, 1 << (c.levels - l - 1)));
    int tile_h = max(1, min(c.height, 1 << (c.levels - l - 1)));
    int tx0 = max(0, min(wl - 1, mn.x / tile_w));
    int ty0 = max(0, min(hl - 1, mn.y / tile_h)) * wl;
    int tx1 = max(0, min(wl - 1, mx.x / tile_w));
    int ty1 = max(0, min(hl - 1, mx.y / tile_h)) * wl;
    const float* base = c.mip + c.level_off[l];
    float zmax = fmaxf(base[tx0 + ty0], fmaxf(base[tx1 + ty0], fmaxf(base[tx0 + ty1], base[tx1 + ty1])));
    return zmax < depth;
}

__device__ __forceinline__ bool block_culled(const BlockView& b, uint32_t g) {
    uint32_t node = g / b.per_block;
    return ((__ldg(&b.culled[node >> 5]) >> (node & 31)) & 1u) != 0u;
}

__device__ __forceinline__ bool mask_bit(const uint32_t* m, uint32_t g) {
    return ((__ldg(&m[g >> 5]) >> (g & 31)) & 1u) != 0u;
}

// ---------------------------------------------------------------------------------
// Block cull (gaussian_bvh.cu:215-329)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ bool aabb_outside_frustum(vec3 bmin, vec3 bmax, const vec4* planes) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const vec3 n = make_v3(planes[i].x, planes[i].y, planes[i].z);
        const float d = planes[i].w;
        vec3 v = make_v3(n.x >= 0.0f ? bmax.x : bmin.x, n.y >= 0.0f ? bmax.y : bmin.y, n.z >= 0.0f ? bmax.z : bmin.z);
        if (dot(n, v) + d < 0.0f) return true;
    }
    return false;
}

__device__ __forceinline__ bool aabb_project_bounds(vec3 bmin, vec3 bmax, const mat4& vp, int width, int height,
                                                    ivec2& out_min, ivec2& out_max, float& out_depth) {
    vec3 corners[8] = {{bmin.x, bmin.y, bmin.z}, {bmax.x, bmin.y, bmin.z}, {bmin.x, bmax.y, bmin.z},
                       {bmax.x, bmax.y, bmin.z}, {bmin.x, bmin.y, bmax.z}, {bmax.x, bmin.y, bmax.z},
                       {bmin.x, bmax.y, bmax.z}, {bmax.x, bmax.y, bmax.z}};
    int minx = width - 1, miny = height - 1, maxx = 0, maxy = 0;
    float min_depth = 1e30f;
    bool any_front = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        vec4 clip = vp * make_v4(corners[i].x, corners[i].y, corners[i].z, 1.0f);
        if (clip.w <= 0.0f) continue;
        any_front = true;
        vec3 ndc = make_v3(clip.x / clip.w, clip.y / clip.w, clip.z / clip.w);
        int px = int((ndc.x * 0.5f + 0.5f) * width);
        int py = int((ndc.y * 0.5f + 0.5f) * height);
        minx = min(minx, px);
        miny = min(miny, py);
        maxx = max(maxx, px);
        maxy = max(maxy, py);
        min_depth = fminf(min_depth, ndc.z);
    }
    if (!any_front) return false;
    minx = max(minx, 0);
    miny = max(miny, 0);
    maxx = min(maxx, width - 1);
    maxy = min(maxy, height - 1);
    if (minx > maxx || miny > maxy) return false;
    out_min = {minx, miny};
    out_max = {maxx, maxy};
    out_depth = min_depth;
    return true;
}

__global__ void __launch_bounds__(256) block_cull_kernel(BlockView b, FrameConst fc, HizView hiz) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx == 0 && b.chunk_count) *b.chunk_count = 0u;
    const uint32_t word = (idx & ~31u) >> 5;
    if (word >= b.words) return;
    bool culled = false;
    if (idx < b.node_count) {
        float4 lo = __ldg(&b.nodes[2 * idx]);
        float4 hi = __ldg(&b.nodes[2 * idx + 1]);
        vec3 bmin = make_v3(lo.x, lo.y, lo.z), bmax = make_v3(hi.x, hi.y, hi.z);
        if (aabb_outside_frustum(bmin, bmax, fc.planes)) {
            culled = true;
        } else if (fc.enable_occlusion) {
            ivec2 mn, mx;
            float front;
            if (aabb_project_bounds(bmin, bmax, fc.vp, hiz.width, hiz.height, mn, mx, front))
                culled = hiz_occluded(hiz, front, mn, mx);
        }
    }
    __syncwarp();
    unsigned m = __ballot_sync(0xffffffffu, culled);
    if ((threadIdx.x & 31) == 0) b.culled[word] = m;
}

// Chunks of 32 Gaussians (one survivor-mask word each) that contain an unculled block, appended
// warp by warp; culled chunks get their mask word zeroed here, since the preprocess skips them.
__global__ void __launch_bounds__(256) visible_chunks_kernel(BlockView b, uint32_t n, uint32_t* __restrict__ list,
                                                             uint32_t* mask_cur, uint32_t* mask_b,
                                                             const uint32_t* __restrict__ mask_iter) {
    if (mask_iter && (*mask_iter & 1u)) mask_cur = mask_b;  // with mask_iter, mask_cur arrives as mask A
    const uint32_t chunks = (n + 31u) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < chunks; base += stride) {
        const uint32_t c = base + lane;
        bool vis = false;
        if (c < chunks) {
            const uint32_t g1 = min((c << 5) + 31u, n - 1u);
            for (uint32_t node = (c << 5) / b.per_block, last = g1 / b.per_block; node <= last && !vis; ++node)
                vis = ((__ldg(&b.culled[node >> 5]) >> (node & 31u)) & 1u) == 0u;
            if (!vis) mask_cur[c] = 0u;
        }
        const unsigned m = __ballot_sync(0xffffffffu, vis);
        if (m == 0u) continue;
        uint32_t slot = 0;
        if (lane == (uint32_t)(__ffs(m) - 1)) slot = atomicAdd(b.chunk_count, (uint32_t)__popc(m));
        slot = __shfl_sync(0xffffffffu, slot, __ffs(m) - 1);
        if (vis) list[slot + (uint32_t)__popc(m & ((1u << lane) - 1u))] = c;
    }
}

// ---------------------------------------------------------------------------------
// Preprocess (gaussian_point_splatting.cu:17-65 + 147-307)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void splat_samples_biased(u32x2& seed, const SplatRecord& rec, const FrameConst& fc,
                                                     uint64_t* __restrict__ buffer);
__device__ __forceinline__ void splat_samples_unbiased(u32x2& seed, const SplatRecord& rec, const FrameConst& fc,
                                                       uint64_t* __restrict__ buffer);

// One Gaussian: true if it splats this pass (record and count written).  kImmediate: a
// Gaussian of at most a.immediate_threshold points is splatted here instead, its samples
// drawn from the seed state the point count left (ENABLE_IMMEDIATE_SPLATTING,
// gaussian_point_splatting.cu:272-287), and it is no survivor.
template <class Scene, bool kImmediate>
__device__ __forceinline__ bool preprocess_one(const PreprocessArgs& a, const Scene& scene, uint32_t gi,
                                               const uint32_t* __restrict__ mask_prev, bool& loaded,
                                               uint32_t& out_points, uint32_t& out_bin) {
    const int idx = (int)gi;
    const FrameConst& fc = a.fc;
    bool splats = false;
    loaded = false;
    out_points = 0;
    out_bin = 0xFFFFFFFFu;
    do {
        if (idx >= (int)a.n) break;
        if (fc.enable_hier && block_culled(a.blocks, (uint32_t)idx)) break;
        if (a.only_previously_occluded && mask_bit(mask_prev, (uint32_t)idx)) break;
        loaded = true;
        u32x2 seed = make_seed((uint32_t)idx, (uint32_t)a.frame_seed);
        float opacity = scene.opacity((uint32_t)idx);
        if (opacity <= 0.0f) break;

        vec3 mean, scale;
        vec4 quat;
        scene.geometry((uint32_t)idx, mean, quat, scale);
        // loadAndTransformGaussian
        vec3 view_mean = transform_point4x3(mean, fc.view);
        float view_z = view_mean.z;
        if (-view_z <= 0.2f) break;
        vec4 proj_mean = fc.vp * make_v4(mean.x, mean.y, mean.z, 1.0f);
        proj_mean = proj_mean * (1.0f / proj_mean.w);
        if (proj_mean.z < -1.0f || proj_mean.z > 1.0f) break;
        mat3 cov = scale_rot_to_cov(scale, quat);
        vec3 cov2d = compute_cov2d(fc.view, cov, mean, fc.tan_fov, fc.focal);
        const float dil = 0.3f * (float)fc.ss * (float)fc.ss;
        cov2d = cov2d + make_v3(dil, 0.0f, dil);
        float det = cov2d.x * cov2d.z - cov2d.y * cov2d.y;
        double det64 = 0.0;
        bool precise = false;
        if constexpr (Scene::kFp64Conic) {
            if (det < 1.0e-3f * cov2d.x * cov2d.z) {  // a*c - b^2 cancels: recompute in FP64
                det64 = (double)cov2d.x * (double)cov2d.z - (double)cov2d.y * (double)cov2d.y;
                det = (float)det64;
                precise = true;
            }
        }
        if (det <= 0.0f) break;
        vec2 pixel_mean = make_v2((proj_mean.x * 0.5f + 0.5f) * (float)fc.up_width,
                                  (proj_mean.y * 0.5f + 0.5f) * (float)fc.up_height);
        ivec2 pmin, pmax;
        if (!gaussian_tile_bounds(pmin, pmax, {fc.up_width, fc.up_height}, cov2d, pixel_mean)) break;

        if (pmin.x >= fc.up_width || pmin.y >= fc.up_height || pmax.x < 0 || pmax.y < 0) break;
        if (fc.cull_small) {
            float trace = cov2d.x + cov2d.z;
            float half = 0.5f * trace;
            float term2 = __fsqrt_rn(fmaxf(0.1f, half * half - det));
            float e1 = half + term2;
            float e2 = half - term2;
            if (e1 < 0.02f || e2 < 0.02f) break;
        }
        constexpr float kTwoPi = 2.0f * 3.14159265358979323846f;
        float importance;
        float s_det = __fsqrt_rn(det);
        if (fc.use_unbiased) importance = kTwoPi * s_det * dilog(opacity);
        else importance = opacity * kTwoPi * s_det;

        if (fc.enable_occlusion) {
            ivec2 qmin = {pmin.x / fc.ss, pmin.y / fc.ss};
            ivec2 qmax = {pmax.x / fc.ss, pmax.y / fc.ss};
            if (hiz_occluded(a.hiz, proj_mean.z, qmin, qmax)) break;
        }
        const float kf = (float)fc.k_points;  // ss^2 x POINTS_PER_KERNEL, 1, or the K override
        uint32_t num_points;
        if (fc.use_unbiased) num_points = poisson(seed, importance);
        else num_points = (uint32_t)stochastic_round(importance, pcg2d(seed).x);
        if (kf > 1) num_points = (uint32_t)stochastic_round((float)num_points / kf, pcg2d(seed).x);
        if (num_points <= 0) break;
        uint32_t cap = (uint32_t)(fc.up_width * fc.up_height / (2 * kf));
        num_points = (cap < num_points) ? cap : num_points;

        vec3 campos = make_v3(fc.cam.c[3].x, fc.cam.c[3].y, fc.cam.c[3].z);
        vec3 color = scene.color((uint32_t)idx, mean, campos);

        // per-Gaussian prologue of splatGaussianPoint (gaussian_point_splatting.cu:88-96)
        const uint64_t view_depth_bits = depth_key(view_z, fc.near_plane, fc.far_plane) << kDepthShift;
        vec3 conic;
        if (precise) conic = make_v3((float)(cov2d.z / det64), (float)(-cov2d.y / det64), (float)(cov2d.x / det64));
        else conic = conic_of(cov2d, 1.0f / det);
        const float c0 = __fsqrt_rn(cov2d.x);
        const float c1 = cov2d.y / c0;
        const float c2 = __fsqrt_rn(cov2d.z - c1 * c1);
        uint32_t r12 = (uint32_t)(color.x * 255.0f) & 0xFFFu;
        uint32_t g12 = (uint32_t)(color.y * 255.0f) & 0xFFFu;
        uint32_t b12 = (uint32_t)(color.z * 255.0f) & 0xFFFu;
        uint64_t key = view_depth_bits | (uint64_t(r12) << 24) | (uint64_t(g12) << 12) | uint64_t(b12);

        SplatRecord rec;
        rec.a = make_float4(pixel_mean.x, pixel_mean.y, c0, c1);
        rec.b = make_float4(c2, conic.x, conic.y, conic.z);
        rec.c = make_float4(opacity, color.x, color.y, color.z);
        rec.d = make_uint4((uint32_t)pmin.x | ((uint32_t)pmin.y << 16), (uint32_t)pmax.x | ((uint32_t)pmax.y << 16),
                           (uint32_t)key, (uint32_t)(key >> 32));
        if constexpr (kImmediate) {
            if ((int)num_points <= a.immediate_threshold) {
                for (uint32_t pt = 0; pt < num_points; ++pt) {
                    if (fc.use_unbiased) splat_samples_unbiased(seed, rec, fc, a.buffer);
                    else splat_samples_biased(seed, rec, fc, a.buffer);
                }
                a.counts[idx] = 0;
                break;
            }
        }
        a.records[idx] = rec;
        a.counts[idx] = num_points;
        out_points = num_points;
        if (a.bins)
            out_bin = screen_bin(pixel_mean.x, pixel_mean.y, fc.up_width, fc.up_height, a.bin_shift, a.bins_x, a.bins_y);
        splats = true;
    } while (false);
    return splats;
}

// Persistent over 32-Gaussian chunks (one mask word each): a warp takes chunk after chunk, so
// a pass over a mostly culled scene costs a bit test per Gaussian, not a thread-block launch
// per 256 Gaussians.
template <class Scene, bool kImmediate>
__global__ void __launch_bounds__(256) preprocess_kernel(PreprocessArgs a, Scene scene) {
    uint32_t* mask_cur = a.mask_cur;
    const uint32_t* mask_prev = a.mask_prev;
    if (a.mask_iter) {
        const bool odd = (*a.mask_iter & 1u) != 0u;
        mask_cur = odd ? a.mask_pair[1] : a.mask_pair[0];
        mask_prev = odd ? a.mask_pair[0] : a.mask_pair[1];
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t first = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    uint32_t loaded_tally = 0;  // this warp's Gaussians whose attributes were read
    // this warp's running survivor / point totals of one scan tile, flushed on a tile change
    uint32_t tile = 0xFFFFFFFFu, tile_s = 0, tile_p = 0;
    auto flush_tile = [&]() {
        if (lane == 0 && tile != 0xFFFFFFFFu && tile_s) {
            // two 32-bit halves: the point total wraps mod 2^32 without carrying into the count
            uint32_t* w = reinterpret_cast<uint32_t*>(a.tile_totals + tile);
            atomicAdd(w, tile_p);
            atomicAdd(w + 1, tile_s);
        }
    };
    auto chunk = [&](uint32_t c) {
        bool loaded;
        uint32_t pts, bin;
        const bool splats = preprocess_one<Scene, kImmediate>(a, scene, (c << 5) + lane, mask_prev, loaded, pts, bin);
        const unsigned m = __ballot_sync(0xffffffffu, splats);
        loaded_tally += (uint32_t)__popc(__ballot_sync(0xffffffffu, loaded));
        if (lane == 0) mask_cur[c] = m;
        if (a.tile_totals && m) {
            const uint32_t t = (c << 5) >> a.tile_shift;
            if (t != tile) {
                flush_tile();
                tile = t;
                tile_s = tile_p = 0;
            }
            tile_s += (uint32_t)__popc(m);
            tile_p += __reduce_add_sync(0xffffffffu, pts);
        }
        if (a.bins && m) {  // one atomic per distinct bin cursor among the warp's survivors
            bin += (c & ((1u << a.bin_sub_log2) - 1u)) * a.bin_count;  // this chunk's cursor of each bin
            unsigned todo = m;
            while (todo) {
                const uint32_t key = __shfl_sync(0xffffffffu, bin, __ffs(todo) - 1);
                const unsigned members = __ballot_sync(0xffffffffu, ((todo >> lane) & 1u) && bin == key);
                const uint32_t sum = __reduce_add_sync(0xffffffffu, ((members >> lane) & 1u) ? pts : 0u);
                if (lane == 0) atomicAdd(a.bins + key, ((unsigned long long)__popc(members) << 32) | sum);
                todo &= ~members;
            }
        }
    };
    if (a.chunk_list) {
        const uint32_t count = *a.chunk_count;
        if (a.tile_totals) {  // contiguous ranges of the (ascending) list, so tile totals merge
            const uint32_t per = (count + warps - 1) / warps;
            const uint32_t b = first * per, e = min(count, b + per);
            // the next chunk's attributes are prefetched into L2 while this one is worked on
            // (256M town: preprocess 1.149 -> 1.130 ms/frame)
            uint32_t next = b < e ? __ldg(a.chunk_list + b) : 0u;
            for (uint32_t i = b; i < e; ++i) {
                const uint32_t c = next;
                if (i + 1 < e) {
                    next = __ldg(a.chunk_list + i + 1);
                    const uint32_t g = (next << 5) + lane;
                    if (g < a.n) scene.prefetch(g);
                }
                chunk(c);
            }
        } else {
            for (uint32_t i = first; i < count; i += warps) chunk(__ldg(a.chunk_list + i));
        }
    } else {
        const uint32_t chunks = (a.n + 31u) >> 5;
        if (a.tile_totals) {
            const uint32_t per = (chunks + warps - 1) / warps;
            const uint32_t b = first * per, e = min(chunks, b + per);
            for (uint32_t c = b; c < e; ++c) chunk(c);
        } else {
            for (uint32_t c = first; c < chunks; c += warps) chunk(c);
        }
    }
    flush_tile();
    if (a.loaded && lane == 0 && loaded_tally) atomicAdd(a.loaded, loaded_tally);
}

// ---------------------------------------------------------------------------------
// Scan over (survivor count, point count) pairs in three fully parallel launches: per-tile
// totals, one block scanning the tile totals, a downsweep writing the compacted survivors
// (replaces workload_distributor.cu:62-145: 3 blocking D2H copies, an exclusive scan, a
// scatter and a P-long max-scan).  Tile word: [63:32] survivors, [31:0] points (mod 2^32 like
// the reference's u32 offsets).  No block waits on another, so there is no spin at all.
// ---------------------------------------------------------------------------------

// One round of a thread's Gaussians (16 consecutive): its mask bits and point counts.
__device__ __forceinline__ uint32_t scan_load(const ScanArgs& a, const uint32_t* __restrict__ mask, uint32_t base,
                                              uint32_t cnt[kScanItems]) {
    uint32_t bits = 0;
    if (base < a.n) {
        bits = (__ldg(&mask[base >> 5]) >> (base & 31)) & 0xFFFFu;
        if (a.n - base < (uint32_t)kScanItems) bits &= (1u << (a.n - base)) - 1u;
    }
#pragma unroll
    for (int q = 0; q < kScanItems / 4; ++q) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if ((bits >> (4 * q)) & 0xFu) v = __ldg(reinterpret_cast<const uint4*>(a.counts + base) + q);
        cnt[4 * q + 0] = ((bits >> (4 * q + 0)) & 1u) ? v.x : 0u;
        cnt[4 * q + 1] = ((bits >> (4 * q + 1)) & 1u) ? v.y : 0u;
        cnt[4 * q + 2] = ((bits >> (4 * q + 2)) & 1u) ? v.z : 0u;
        cnt[4 * q + 3] = ((bits >> (4 * q + 3)) & 1u) ? v.w : 0u;
    }
    return bits;
}

// Block-wide exclusive scan of (survivors, points) pairs; also returns the block totals.
template <int kThreads>
__device__ __forceinline__ void block_scan_pair(uint32_t s, uint32_t p, uint32_t& ex_s, uint32_t& ex_p,
                                                uint32_t& tot_s, uint32_t& tot_p) {
    __shared__ uint32_t w_s[kThreads / 32], w_p[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t is = s, ip = p;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t vs = __shfl_up_sync(0xffffffffu, is, o);
        const uint32_t vp = __shfl_up_sync(0xffffffffu, ip, o);
        if (lane >= o) {
            is += vs;
            ip += vp;
        }
    }
    if (lane == 31) {
        w_s[warp] = is;
        w_p[warp] = ip;
    }
    __syncthreads();
    uint32_t off_s = 0, off_p = 0, all_s = 0, all_p = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        if (w < warp) {
            off_s += w_s[w];
            off_p += w_p[w];
        }
        all_s += w_s[w];
        all_p += w_p[w];
    }
    ex_s = off_s + is - s;
    ex_p = off_p + ip - p;
    tot_s = all_s;
    tot_p = all_p;
}

// Pass 1 of the scan: every tile's survivor and point totals, fully parallel.
template <int kScanRounds>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(ScanArgs a) {
    const uint32_t* mask = a.mask;  // (a select, not a runtime index into the parameter array)
    if (a.mask_iter) mask = (*a.mask_iter & 1u) ? a.mask_pair[1] : a.mask_pair[0];
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * (kScanThreads * kScanItems * kScanRounds) + threadIdx.x * (kScanItems * kScanRounds);
    uint32_t surv = 0, pts = 0;
#pragma unroll
    for (int q = 0; q < kScanRounds; ++q) {
        uint32_t cnt[kScanItems];
        surv += __popc(scan_load(a, mask, base + q * kScanItems, cnt));
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) pts += cnt[i];
    }
    uint32_t ex_s, ex_p, tot_s, tot_p;
    block_scan_pair<kScanThreads>(surv, pts, ex_s, ex_p, tot_s, tot_p);
    if (threadIdx.x == 0) a.tile_state[tile] = ((unsigned long long)tot_s << 32) | tot_p;
}

// Pass 2: one block turns the tile totals into exclusive tile prefixes (in place) and writes
// the pass counters (points mod 2^32, like the reference's u32 offsets).  The tile words go
// through shared memory in rounds of kTileScanThreads * 4 with coalesced loads and stores;
// each thread scans 4 consecutive words and a block scan plus a running carry joins them.
constexpr int kTileScanThreads = 1024;
constexpr int kTileScanPer = 4;
static_assert(kBinSubs <= (uint32_t)kTileScanPer && (kBinSubs & (kBinSubs - 1u)) == 0u,
              "a scan thread's words must hold whole bins");

// One block: exclusive prefix of `count` packed (survivors << 32 | points) words in place,
// through shared memory in coalesced rounds; returns the totals.
// Scans words_g in the order of its logical index L; with sub_log2 > 0, word L is stored at
// (L mod 2^sub_log2) * stride + L / 2^sub_log2 (the bin cursors' layout).
__device__ __forceinline__ void scan_words_inplace(unsigned long long* words_g, uint32_t count, uint32_t& total_s,
                                                   uint32_t& total_p, uint32_t* max_s = nullptr,
                                                   uint32_t sub_log2 = 0, uint32_t stride = 0) {
    auto at = [&](uint32_t L) -> uint32_t {
        return sub_log2 ? (L & ((1u << sub_log2) - 1u)) * stride + (L >> sub_log2) : L;
    };
    __shared__ unsigned long long words[kTileScanThreads * kTileScanPer];
    __shared__ uint32_t s_max;
    constexpr uint32_t kRound = kTileScanThreads * kTileScanPer;
    uint32_t carry_s = 0, carry_p = 0, my_max = 0;
    if (threadIdx.x == 0) s_max = 0;
    for (uint32_t r0 = 0; r0 < count; r0 += kRound) {
        for (uint32_t i = threadIdx.x; i < kRound; i += kTileScanThreads)
            words[i] = r0 + i < count ? words_g[at(r0 + i)] : 0ull;
        __syncthreads();
        uint32_t s = 0, p = 0, group = 0;
#pragma unroll
        for (int k = 0; k < kTileScanPer; ++k) {
            const unsigned long long v = words[threadIdx.x * kTileScanPer + k];
            s += (uint32_t)(v >> 32);
            p += (uint32_t)v;
            group += (uint32_t)(v >> 32);
            if ((((uint32_t)k + 1u) & ((1u << sub_log2) - 1u)) == 0u) {  // a whole bin's cursors
                my_max = max(my_max, group);
                group = 0;
            }
        }
        uint32_t ex_s, ex_p, tot_s, tot_p;
        block_scan_pair<kTileScanThreads>(s, p, ex_s, ex_p, tot_s, tot_p);
        ex_s += carry_s;
        ex_p += carry_p;
#pragma unroll
        for (int k = 0; k < kTileScanPer; ++k) {
            const unsigned long long v = words[threadIdx.x * kTileScanPer + k];
            words[threadIdx.x * kTileScanPer + k] = ((unsigned long long)ex_s << 32) | ex_p;
            ex_s += (uint32_t)(v >> 32);
            ex_p += (uint32_t)v;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kRound && r0 + i < count; i += kTileScanThreads) words_g[at(r0 + i)] = words[i];
        carry_s += tot_s;
        carry_p += tot_p;
        __syncthreads();
    }
    total_s = carry_s;
    total_p = carry_p;
    if (max_s) {  // the largest survivor count of one bin (2^sub_log2 consecutive words)
        my_max = __reduce_max_sync(0xffffffffu, my_max);
        if ((threadIdx.x & 31u) == 0u) atomicMax(&s_max, my_max);
        __syncthreads();
        *max_s = s_max;
    }
}

// Pass 2: block 0 turns the tile totals into exclusive tile prefixes (in place) and writes the
// pass counters (points mod 2^32, like the reference's u32 offsets); block 1, when the pass is
// screen-binned, does the same for the bin histogram.
__global__ void __launch_bounds__(kTileScanThreads) scan_tiles_kernel(ScanArgs a, uint32_t num_tiles) {
    uint32_t carry_s, carry_p;
    if (blockIdx.x == 1) {
        uint32_t most = 0;
        scan_words_inplace(a.bins, a.nbins, carry_s, carry_p, &most, (uint32_t)a.bin_sub_log2, a.bin_count);
        // a bin crowded past bin_crowded survivors would serialise the downsweep on its
        // cursors: the pass is then walked in Gaussian order
        if (threadIdx.x == 0) a.counters->crowded = most > a.bin_crowded ? 1u : 0u;
        return;
    }
    scan_words_inplace(a.tile_state, num_tiles, carry_s, carry_p);
    if (threadIdx.x == 0) {
        a.counters->survivors = carry_s;
        a.counters->total_points = carry_p;
        a.counters->points = carry_p < a.max_points ? carry_p : a.max_points;
        a.counters->truncated = carry_p > a.max_points ? 1u : 0u;
        a.counters->scan_timeouts = 0u;
        a.counters->loaded = a.loaded ? *a.loaded : 0u;
        if (a.loaded) *a.loaded = 0u;  // the next pass's preprocess tallies from zero
        a.counters->pad = 0u;
        if (!a.bins) a.counters->crowded = 0u;
    }
}

// Pass 3: each tile rescans its Gaussians from its prefix and writes the compacted survivor
// ids and first points.
template <int kScanRounds>
__global__ void __launch_bounds__(kScanThreads) scan_write_kernel(ScanArgs a) {
    const uint32_t* mask = a.mask;  // (a select, not a runtime index into the parameter array)
    if (a.mask_iter) mask = (*a.mask_iter & 1u) ? a.mask_pair[1] : a.mask_pair[0];
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * (kScanThreads * kScanItems * kScanRounds) + threadIdx.x * (kScanItems * kScanRounds);
    uint32_t surv = 0, pts = 0;
#pragma unroll
    for (int q = 0; q < kScanRounds; ++q) {
        uint32_t cnt[kScanItems];
        surv += __popc(scan_load(a, mask, base + q * kScanItems, cnt));
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) pts += cnt[i];
    }
    uint32_t ex_s, ex_p, tot_s, tot_p;
    block_scan_pair<kScanThreads>(surv, pts, ex_s, ex_p, tot_s, tot_p);
    if (surv == 0u) return;
    const unsigned long long pre = a.tile_state[tile];
    uint32_t r = (uint32_t)(pre >> 32) + ex_s;
    uint32_t pt = (uint32_t)pre + ex_p;
    for (int q = 0; q < kScanRounds; ++q) {  // again, now writing (the counts come from L1/L2)
        uint32_t cnt[kScanItems];
        const uint32_t b = base + q * kScanItems;
        const uint32_t bits = scan_load(a, mask, b, cnt);
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            if ((bits >> i) & 1u) {
                a.surv_gid[r] = b + i;
                a.surv_start[r] = pt;
                ++r;
                pt += cnt[i];
            }
        }
    }
}

// The render path's downsweep: as scan_write_kernel, and then for every survivor the splat's
// work order.  Screen-binned (bins set, pass not truncated): the survivor takes its slot and
// first walk position from one of its bin's cursors with one 64-bit atomic, so that slot and position
// stay consistent and positions increase with the slot; otherwise the Gaussian order itself,
// with the points past P dropped as the reference drops them.  Either way the survivor then
// records itself as the owner of every 256-point splat tile that starts inside its points.
// (tiles starting at or past P are never walked, and the array holds max_points / 256 + 2)
__device__ __forceinline__ void own_tiles(uint32_t* __restrict__ tile_first_rank, uint64_t first, uint64_t count,
                                          uint32_t rank, uint32_t P) {
    const uint64_t end = min(first + count, (uint64_t)P);
    for (uint64_t t = (first + 255u) >> 8; (t << 8) < end; ++t) tile_first_rank[t] = rank;
}

template <int kScanRounds>
__global__ void __launch_bounds__(kScanThreads) scan_write_fused_kernel(ScanArgs a) {
    const uint32_t tile = blockIdx.x;
    // a tile without survivors (its exclusive survivor prefix equals the next tile's) has
    // nothing to write: culled regions of the scene cost two loads, not a pass over their masks
    // (256M town: scan 0.586 -> 0.548 ms/frame)
    {
        const uint32_t s0 = (uint32_t)(a.tile_state[tile] >> 32);
        const uint32_t s1 = tile + 1u < gridDim.x ? (uint32_t)(a.tile_state[tile + 1u] >> 32) : a.counters->survivors;
        if (s0 == s1) return;
    }
    const uint32_t* mask = a.mask;
    if (a.mask_iter) mask = (*a.mask_iter & 1u) ? a.mask_pair[1] : a.mask_pair[0];
    const uint32_t base = tile * (kScanThreads * kScanItems * kScanRounds) + threadIdx.x * (kScanItems * kScanRounds);
    uint32_t surv = 0, pts = 0;
#pragma unroll
    for (int q = 0; q < kScanRounds; ++q) {
        uint32_t cnt[kScanItems];
        surv += __popc(scan_load(a, mask, base + q * kScanItems, cnt));
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) pts += cnt[i];
    }
    uint32_t ex_s, ex_p, tot_s, tot_p;
    block_scan_pair<kScanThreads>(surv, pts, ex_s, ex_p, tot_s, tot_p);
    if (surv == 0u) return;
    const uint32_t P = a.counters->points;
    const bool binned = a.bins && a.counters->truncated == 0u && a.counters->crowded == 0u;
    const unsigned long long pre = a.tile_state[tile];
    uint32_t r = (uint32_t)(pre >> 32) + ex_s;
    uint32_t pt = (uint32_t)pre + ex_p;
    for (int q = 0; q < kScanRounds; ++q) {  // again, now writing (the counts come from L1/L2)
        uint32_t cnt[kScanItems];
        const uint32_t b = base + q * kScanItems;
        const uint32_t bits = scan_load(a, mask, b, cnt);
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            if ((bits >> i) & 1u) {
                const uint32_t g = b + i;
                a.surv_gid[r] = g;
                a.surv_start[r] = pt;
                if (binned) {
                    const float2 pm = __ldg(reinterpret_cast<const float2*>(a.records + g));
                    const uint32_t bin = screen_bin(pm.x, pm.y, a.up_width, a.up_height, a.bin_shift, a.bins_x, a.bins_y) +
                                         ((g >> 5) & ((1u << a.bin_sub_log2) - 1u)) * a.bin_count;
                    const unsigned long long old = atomicAdd(a.bins + bin, (1ull << 32) | cnt[i]);
                    const uint32_t slot = (uint32_t)(old >> 32);
                    a.sorted_gid[slot] = g;
                    a.sorted_pstart[slot] = pt;
                    a.sorted_qstart[slot] = (uint32_t)old;
                    own_tiles(a.tile_first_rank, (uint32_t)old, cnt[i], slot, P);
                } else if (pt < P) {
                    own_tiles(a.tile_first_rank, pt, cnt[i], r, P);
                }
                ++r;
                pt += cnt[i];
            }
        }
    }
}

// First survivor of every splat tile: tile t (points [t*tile_points, ...)) starts inside the
// survivor with the largest rank whose first point is <= t*tile_points.  One thread per tile,
// a binary search over the survivors' first points (monotone below 2^32 points per pass).  A
// survivor can own thousands of tiles (a Gaussian right in front of the camera), so this is
// done per tile rather than per survivor.
__global__ void __launch_bounds__(256) tile_owner_kernel(const uint32_t* __restrict__ surv_start,
                                                         uint32_t* __restrict__ tile_first_rank,
                                                         const PassCounters* __restrict__ counters,
                                                         uint32_t tile_points, uint32_t* __restrict__ mask_iter) {
    const uint32_t points = counters->points;
    const uint32_t survivors = counters->survivors;
    if (mask_iter && points > 0 && blockIdx.x == 0 && threadIdx.x == 0) *mask_iter += 1u;
    if (points == 0 || survivors == 0) return;
    const uint32_t tiles = (uint32_t)(((unsigned long long)points + tile_points - 1) / tile_points);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += gridDim.x * blockDim.x) {
        const uint32_t target = t * tile_points;
        uint32_t lo = 0, hi = survivors - 1;
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo + 1) >> 1);
            if (__ldg(surv_start + mid) <= target) lo = mid;
            else hi = mid - 1;
        }
        tile_first_rank[t] = lo;
    }
}

// ---------------------------------------------------------------------------------
// Splat (gaussian_point_splatting.cu:67-141 with num_points = 1, 383-432)
// ---------------------------------------------------------------------------------
constexpr int kSplatTile = 256;

__device__ __forceinline__ void atomic_add_color(unsigned long long* address, uint64_t value) {
    // post_processing_kernels.cuh:13-42 with add_if_equal = true
    const uint64_t target_depth = value & kDepthMask;
    unsigned long long old = *address, assumed;
    do {
        assumed = old;
        uint64_t assumed_depth = assumed & kDepthMask;
        uint64_t new_value = value;
        if (target_depth > assumed_depth) return;
        if (target_depth == assumed_depth) {
            uint64_t new_lower = (assumed & kColorMask) + (value & kColorMask);
            new_value = (assumed & kDepthMask) | (new_lower & kColorMask);
        }
        old = atomicCAS(address, assumed, (unsigned long long)new_value);
    } while (assumed != old);
}

// Biased mode (use_unbiased_2d_splatting = false): samples in the reference's order, each
// pre-tested and colour-added before the next one is drawn.
// One point's samples from `seed` onwards (the seed advances, as splatGaussianPoint's does).
__device__ __forceinline__ void splat_samples_biased(u32x2& seed, const SplatRecord& rec, const FrameConst& fc,
                                                     uint64_t* __restrict__ buffer) {
    const vec2 pixel_mean = make_v2(rec.a.x, rec.a.y);
    const float c0 = rec.a.z, c1 = rec.a.w, c2 = rec.b.x;
    const vec3 conic = make_v3(rec.b.y, rec.b.z, rec.b.w);
    const float opacity = rec.c.x;
    const int minx = (int)(rec.d.x & 0xFFFFu), miny = (int)(rec.d.x >> 16);
    const int maxx = (int)(rec.d.y & 0xFFFFu), maxy = (int)(rec.d.y >> 16);
    const uint64_t key = (uint64_t)rec.d.z | ((uint64_t)rec.d.w << 32);
    const uint64_t view_depth_bits = key & kDepthMask;
    const int k = fc.k_points;
    const int samples = fc.num_passes * k;
    for (int p = 0; p < samples; ++p) {
        vec2 u = pcg2d(seed);
        vec2 xy = box_muller(u.x, u.y);
        vec2 pixel = make_v2(pixel_mean.x + c0 * xy.x, pixel_mean.y + c1 * xy.x + c2 * xy.y);
        pixel = make_v2(floorf(pixel.x), floorf(pixel.y));
        int x = (int)pixel.x;
        int y = (int)pixel.y;
        vec2 delta = make_v2(pixel_mean.x - pixel.x, pixel_mean.y - pixel.y);
        if (x < minx || x >= maxx || y < miny || y >= maxy) continue;
        float gw = gaussian_value(conic, delta);
        float alpha = opacity * gw;
        if (alpha < 1.0f / 255.0f) continue;
        int index = splat_index(x, y, p / k, fc.num_passes, fc.up_width, fc.up_height);
        unsigned long long* slot = reinterpret_cast<unsigned long long*>(buffer + index);
        if ((uint64_t)__ldcg(slot) <= view_depth_bits) continue;
        atomic_add_color(slot, key);
    }
}

__device__ __forceinline__ void splat_point_biased(uint32_t point, const SplatRecord& rec, const FrameConst& fc,
                                                   int frame_seed, uint64_t* __restrict__ buffer) {
    u32x2 seed = make_seed(point, (uint32_t)frame_seed);
    splat_samples_biased(seed, rec, fc, buffer);
}

// Unbiased mode (the default): the same sample stream, drawn kSplatBatch samples at a time.
// Each batch computes its slots first, then issues their pre-test loads together (several
// loads in flight per thread instead of one), then the atomicMins.  Order does not matter for
// a min, and a slot is skipped only when it already holds a value <= this Gaussian's key, the
// exact condition under which atomicMin would leave it unchanged (the reference skips when
// the slot is <= the depth bits alone, a subset of these cases), so the buffer is identical.
// Slot values only decrease during the kernel, so an L1-cached (possibly stale, hence larger)
// pre-test value can only cause an extra atomic, never a wrong skip.
#ifndef GPS_SPLAT_BATCH
#define GPS_SPLAT_BATCH 4
#endif
// Pre-test before the atomic: 1 = L1-cached load, 2 = L2 load, 0 = none (every live sample
// issues its atomicMin; the buffer is the same in all three).  On the 16M-Gaussian town orbit
// (1080p, ss 2, 4 spp) the L1-cached pre-test measured fastest on B200 (splat 2.04 ms/frame vs
// 2.07 with the L2 load and 2.25 with none): it drops the atomics whose slot already holds a
// nearer or equal key, and an L1 hit costs less than the atomic it saves.
#ifndef GPS_SPLAT_PRETEST
#define GPS_SPLAT_PRETEST 1
#endif
#ifndef GPS_SPLAT_PIPELINE
#define GPS_SPLAT_PIPELINE 1
#endif
// 1: a sample's in-tile Morton code comes from a 64-entry shared-memory table of spread 6-bit
// coordinates (two table loads) instead of two 4-step bit spreads; the codes are identical.
// Measured on the 16M-Gaussian town orbit (1080p, ss 2, 4 spp): splat 1.90 vs 1.96 ms/frame.
#ifndef GPS_SPLAT_MORTON_LUT
#define GPS_SPLAT_MORTON_LUT 1
#endif
constexpr int kSplatBatch = GPS_SPLAT_BATCH;

__device__ __forceinline__ void splat_samples_unbiased(u32x2& seed, const SplatRecord& rec, const FrameConst& fc,
                                                       uint64_t* __restrict__ buffer) {
    const vec2 pixel_mean = make_v2(rec.a.x, rec.a.y);
    const float c0 = rec.a.z, c1 = rec.a.w, c2 = rec.b.x;
    const vec3 conic = make_v3(rec.b.y, rec.b.z, rec.b.w);
    const float opacity = rec.c.x;
    const int minx = (int)(rec.d.x & 0xFFFFu), miny = (int)(rec.d.x >> 16);
    const int maxx = (int)(rec.d.y & 0xFFFFu), maxy = (int)(rec.d.y >> 16);
    const unsigned long long key = (unsigned long long)rec.d.z | ((unsigned long long)rec.d.w << 32);
    // the per-Gaussian factors of correctedBoxMuller (random.cuh:132-141), evaluated once
    const float inv_alpha = 1.0f / fmaxf(opacity, 1.e-37f);
    const float li2_alpha = dilog(opacity);
    const int k = fc.k_points;
    const int samples = fc.num_passes * k;
    const int passes = fc.num_passes;
    const int tiles_per_row = (fc.up_width + kTileSize - 1) >> kTileBits;
    int p = 0, j = 0;
    for (int s0 = 0; s0 < samples; s0 += kSplatBatch) {
        uint32_t slot[kSplatBatch];
        uint32_t live = 0;
#pragma unroll
        for (int b = 0; b < kSplatBatch; ++b) {
            slot[b] = 0;
            if (s0 + b < samples) {
                vec2 u = pcg2d(seed);
                float a = inv_alpha * inv_dilog((1.0f - u.x) * li2_alpha);
                a = gclamp(a, 1.e-37f, 1.0f);
                float r = __fsqrt_rn(fmaxf(-2.0f * __logf(a), 0.0f));
                float theta = 2.0f * kPiF * u.y;
                float sn, cs;
                __sincosf(theta, &sn, &cs);
                vec2 xy = make_v2(r * cs, r * sn);
                vec2 pixel = make_v2(pixel_mean.x + c0 * xy.x, pixel_mean.y + c1 * xy.x + c2 * xy.y);
                pixel = make_v2(floorf(pixel.x), floorf(pixel.y));
                int x = (int)pixel.x;
                int y = (int)pixel.y;
                vec2 delta = make_v2(pixel_mean.x - pixel.x, pixel_mean.y - pixel.y);
                if (x >= minx && x < maxx && y >= miny && y < maxy) {
                    float alpha = opacity * gaussian_value(conic, delta);
                    if (!(alpha < 1.0f / 255.0f)) {
                        const uint32_t code = morton_encode((uint32_t)(x & (kTileSize - 1)), (uint32_t)(y & (kTileSize - 1)));
                        const uint32_t tile = (uint32_t)((y >> kTileBits) * tiles_per_row + (x >> kTileBits));
                        slot[b] = (tile * (uint32_t)(kTileSize * kTileSize) + code) * (uint32_t)passes + (uint32_t)p;
                        live |= 1u << b;
                    }
                }
                if (++j == k) {
                    j = 0;
                    ++p;
                }
            }
        }
#if GPS_SPLAT_PRETEST
        unsigned long long seen[kSplatBatch];
#pragma unroll
        for (int b = 0; b < kSplatBatch; ++b) {
            const unsigned long long* at = reinterpret_cast<const unsigned long long*>(buffer) + slot[b];
            seen[b] = ((live >> b) & 1u) ? (GPS_SPLAT_PRETEST == 1 ? __ldca(at) : __ldcg(at)) : 0ull;
        }
#pragma unroll
        for (int b = 0; b < kSplatBatch; ++b)
            if (((live >> b) & 1u) && seen[b] > key)
                atomicMin(reinterpret_cast<unsigned long long*>(buffer) + slot[b], key);
#else
#pragma unroll
        for (int b = 0; b < kSplatBatch; ++b)
            if ((live >> b) & 1u) atomicMin(reinterpret_cast<unsigned long long*>(buffer) + slot[b], key);
#endif
    }
}

__device__ __forceinline__ void splat_point_unbiased(uint32_t point, const SplatRecord& rec, const FrameConst& fc,
                                                     int frame_seed, uint64_t* __restrict__ buffer) {
    u32x2 seed = make_seed(point, (uint32_t)frame_seed);
    splat_samples_unbiased(seed, rec, fc, buffer);
}

// The same stream with K (points per thread per pass, ss*ss) known at compile time: the K
// samples of a pass are drawn without branches (bounds and alpha tests become predicates), so
// their independent transcendental chains can be interleaved, then the live ones are splatted.
struct SampleConst {
    vec2 pixel_mean;
    float c0, c1, c2, opacity, inv_alpha, li2_alpha;
    vec3 conic;
    int minx, miny, maxx, maxy;
    uint32_t span_x, span_y;  // max(maxx - minx, 0), max(maxy - miny, 0)
    int tiles_per_row, passes;
    const uint32_t* spread;  // shared-memory Morton table (GPS_SPLAT_MORTON_LUT)
};

__device__ __forceinline__ bool draw_sample(u32x2& seed, const SampleConst& c, int p, uint32_t& slot) {
    const vec2 u = pcg2d(seed);
    float a = c.inv_alpha * inv_dilog((1.0f - u.x) * c.li2_alpha);
    a = gclamp(a, 1.e-37f, 1.0f);
    const float r = __fsqrt_rn(fmaxf(-2.0f * __logf(a), 0.0f));
    const float theta = 2.0f * kPiF * u.y;
    float sn, cs;
    __sincosf(theta, &sn, &cs);
    const vec2 xy = make_v2(r * cs, r * sn);
    vec2 pixel = make_v2(c.pixel_mean.x + c.c0 * xy.x, c.pixel_mean.y + c.c1 * xy.x + c.c2 * xy.y);
    pixel = make_v2(floorf(pixel.x), floorf(pixel.y));
    const int x = (int)pixel.x;
    const int y = (int)pixel.y;
    const vec2 delta = make_v2(c.pixel_mean.x - pixel.x, c.pixel_mean.y - pixel.y);
    // minx <= x < maxx as one unsigned compare (x - minx wraps to a large value below minx):
    // splat 1.572 -> 1.563 ms/frame on the 16M orbit
    const bool inside = ((uint32_t)x - (uint32_t)c.minx < c.span_x) & ((uint32_t)y - (uint32_t)c.miny < c.span_y);
    const float alpha = c.opacity * gaussian_value(c.conic, delta);
#if GPS_SPLAT_MORTON_LUT
    const uint32_t code = c.spread[x & (kTileSize - 1)] | (c.spread[y & (kTileSize - 1)] << 1);
#else
    const uint32_t code = morton_encode((uint32_t)(x & (kTileSize - 1)), (uint32_t)(y & (kTileSize - 1)));
#endif
    const uint32_t tile = (uint32_t)((y >> kTileBits) * c.tiles_per_row + (x >> kTileBits));
    slot = (tile * (uint32_t)(kTileSize * kTileSize) + code) * (uint32_t)c.passes + (uint32_t)p;
    return inside & !(alpha < 1.0f / 255.0f);
}

#ifndef GPS_SPLAT_PAIRED
#define GPS_SPLAT_PAIRED 1  // splat 1.547 -> 1.461 ms/frame (16M)
#endif
// The K samples of a pass drawn two at a time: the random words come off the seed in stream
// order, and the floating-point steps two samples share (the opacity-corrected inverse dilog
// polynomial, the Box-Muller products, the pixel position and its offset, the Gaussian weight)
// run as sm_100 paired FP32 instructions (FFMA2 / FMUL2 / FADD2), each lane rounded as the
// scalar instruction would.  The transcendental and per-lane steps stay scalar.  Same values
// as draw_sample, bit for bit.
template <int K>
__device__ __forceinline__ void draw_samples_paired(u32x2& seed, const SampleConst& c, int p, uint32_t* slot,
                                                    bool* live) {
    static_assert(K % 2 == 0, "samples are drawn in pairs");
    const float2 one = make_float2(1.0f, 1.0f);
    const float2 li2 = make_float2(c.li2_alpha, c.li2_alpha);
    const float2 inva = make_float2(c.inv_alpha, c.inv_alpha);
    const float2 c0 = make_float2(c.c0, c.c0), c1 = make_float2(c.c1, c.c1), c2 = make_float2(c.c2, c.c2);
    const float2 pmx = make_float2(c.pixel_mean.x, c.pixel_mean.x), pmy = make_float2(c.pixel_mean.y, c.pixel_mean.y);
#pragma unroll
    for (int j = 0; j < K; j += 2) {
        u32x2 s0 = pcg2d_step(seed);
        u32x2 s1 = pcg2d_step(s0);
        seed = s1;
        const float2 rk = make_float2(kRecip2e32, kRecip2e32);
        const float2 ux = __fmul2_rn(make_float2((float)s0.x, (float)s1.x), rk);
        const float2 uy = __fmul2_rn(make_float2((float)s0.y, (float)s1.y), rk);
        // inv_dilog((1 - u.x) * Li2(alpha)) (random.cuh:110-127, 132-141)
        const float2 x = __fmul2_rn(__fadd2_rn(one, make_float2(-ux.x, -ux.y)), li2);
        const float2 t = make_float2(fminf(x.x / kLi2Max, 1.0f), fminf(x.y / kLi2Max, 1.0f));
        float2 y = make_float2(-1.27463503e+01f, -1.27463503e+01f);
        y = __ffma2_rn(y, t, make_float2(5.88993459e+01f, 5.88993459e+01f));
        y = __ffma2_rn(y, t, make_float2(-1.16025780e+02f, -1.16025780e+02f));
        y = __ffma2_rn(y, t, make_float2(1.26945827e+02f, 1.26945827e+02f));
        y = __ffma2_rn(y, t, make_float2(-8.43108826e+01f, -8.43108826e+01f));
        y = __ffma2_rn(y, t, make_float2(3.48799862e+01f, 3.48799862e+01f));
        y = __ffma2_rn(y, t, make_float2(-8.89606235e+00f, -8.89606235e+00f));
        y = __ffma2_rn(y, t, make_float2(1.38640936e+00f, 1.38640936e+00f));
        y = __ffma2_rn(y, t, make_float2(-7.80640876e-01f, -7.80640876e-01f));
        y = __ffma2_rn(y, t, make_float2(1.64841888e+00f, 1.64841888e+00f));
        y = __ffma2_rn(y, t, make_float2(-2.82836687e-05f, -2.82836687e-05f));
        const float2 a2 = __fmul2_rn(inva, y);
        float r[2], sn[2], cs[2];
        // -2 log(a) and the angle 2 pi u: one product each, paired (scaling by -2 is exact, so
        // the pair equals the scalar (lg2(a) ln2) (-2) however the scalar form groups it)
        const float2 lg = __fmul2_rn(make_float2(-2.0f, -2.0f), make_float2(__logf(gclamp(a2.x, 1.e-37f, 1.0f)),
                                                                             __logf(gclamp(a2.y, 1.e-37f, 1.0f))));
        const float2 th = __fmul2_rn(make_float2(2.0f * kPiF, 2.0f * kPiF), uy);
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            r[l] = __fsqrt_rn(fmaxf(l ? lg.y : lg.x, 0.0f));
            __sincosf(l ? th.y : th.x, &sn[l], &cs[l]);
        }
        const float2 rr = make_float2(r[0], r[1]);
        const float2 xyx = __fmul2_rn(rr, make_float2(cs[0], cs[1]));
        const float2 xyy = __fmul2_rn(rr, make_float2(sn[0], sn[1]));
        const float2 px = __ffma2_rn(c0, xyx, pmx);
        const float2 py = __ffma2_rn(c2, xyy, __ffma2_rn(c1, xyx, pmy));
        const float2 fx = make_float2(floorf(px.x), floorf(px.y)), fy = make_float2(floorf(py.x), floorf(py.y));
        const float2 dx = __fadd2_rn(pmx, make_float2(-fx.x, -fx.y));
        const float2 dy = __fadd2_rn(pmy, make_float2(-fy.x, -fy.y));
        // gaussian_value (linalg.cuh:309-317) on both samples.  Its sums of two products are fused
        // as the compiler contracts them, the left product into the FMA: x*x-part first
        // (fma(cx dx, dx, (cz dy) dy)), then fma(-0.5, quad, -((cy dx) dy)).  The tests pin this:
        // fusing the right-hand products instead changed one entry of the 4K parity case.
        const float2 cx = make_float2(c.conic.x, c.conic.x), cyv = make_float2(c.conic.y, c.conic.y),
                     cz = make_float2(c.conic.z, c.conic.z);
        const float2 quad = __ffma2_rn(__fmul2_rn(cx, dx), dx, __fmul2_rn(__fmul2_rn(cz, dy), dy));
        const float2 hh = __fmul2_rn(__fmul2_rn(cyv, dx), dy);
        const float2 sig = __ffma2_rn(make_float2(-0.5f, -0.5f), quad, make_float2(-hh.x, -hh.y));
        const float2 gv = make_float2(sig.x > 0.f ? 0.0f : __expf(sig.x), sig.y > 0.f ? 0.0f : __expf(sig.y));
        const float2 al = __fmul2_rn(make_float2(c.opacity, c.opacity), gv);
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int xi = (int)(l ? fx.y : fx.x);
            const int yi = (int)(l ? fy.y : fy.x);
            const bool inside = ((uint32_t)xi - (uint32_t)c.minx < c.span_x) & ((uint32_t)yi - (uint32_t)c.miny < c.span_y);
            const float alpha = l ? al.y : al.x;
#if GPS_SPLAT_MORTON_LUT
            const uint32_t code = c.spread[xi & (kTileSize - 1)] | (c.spread[yi & (kTileSize - 1)] << 1);
#else
            const uint32_t code = morton_encode((uint32_t)(xi & (kTileSize - 1)), (uint32_t)(yi & (kTileSize - 1)));
#endif
            const uint32_t tile = (uint32_t)((yi >> kTileBits) * c.tiles_per_row + (xi >> kTileBits));
            slot[j + l] = (tile * (uint32_t)(kTileSize * kTileSize) + code) * (uint32_t)c.passes + (uint32_t)p;
            live[j + l] = inside & !(alpha < 1.0f / 255.0f);
        }
    }
}

template <int K>
__device__ __forceinline__ void splat_point_unbiased_k(uint32_t point, const SplatRecord& rec, const FrameConst& fc,
                                                       int frame_seed, uint64_t* __restrict__ buffer,
                                                       const uint32_t* spread) {
    u32x2 seed = make_seed(point, (uint32_t)frame_seed);
    SampleConst c;
    c.spread = spread;
    c.pixel_mean = make_v2(rec.a.x, rec.a.y);
    c.c0 = rec.a.z;
    c.c1 = rec.a.w;
    c.c2 = rec.b.x;
    c.conic = make_v3(rec.b.y, rec.b.z, rec.b.w);
    c.opacity = rec.c.x;
    c.minx = (int)(rec.d.x & 0xFFFFu);
    c.miny = (int)(rec.d.x >> 16);
    c.maxx = (int)(rec.d.y & 0xFFFFu);
    c.maxy = (int)(rec.d.y >> 16);
    c.span_x = (uint32_t)max(c.maxx - c.minx, 0);
    c.span_y = (uint32_t)max(c.maxy - c.miny, 0);
    // the per-Gaussian factors of correctedBoxMuller (random.cuh:132-141), evaluated once
    c.inv_alpha = 1.0f / fmaxf(c.opacity, 1.e-37f);
    c.li2_alpha = dilog(c.opacity);
    c.passes = fc.num_passes;
    c.tiles_per_row = (fc.up_width + kTileSize - 1) >> kTileBits;
    const unsigned long long key = (unsigned long long)rec.d.z | ((unsigned long long)rec.d.w << 32);
    unsigned long long* buf = reinterpret_cast<unsigned long long*>(buffer);
#if GPS_SPLAT_PRETEST && GPS_SPLAT_PIPELINE
    // Software-pipelined over passes: pass p+1's samples are drawn and their pre-test loads
    // issued before pass p's atomics consume its loads, so the load latency hides behind the
    // next pass's arithmetic.  Samples are still drawn in stream order.
    uint32_t sa[K], sb[K];
    bool la[K], lb[K];
    unsigned long long va[K], vb[K];
    auto draw = [&](int p, uint32_t* sl, bool* lv, unsigned long long* vv) {
#if GPS_SPLAT_PAIRED
        if constexpr (K % 2 == 0) {
            draw_samples_paired<K>(seed, c, p, sl, lv);
        } else {
#pragma unroll
            for (int j = 0; j < K; ++j) lv[j] = draw_sample(seed, c, p, sl[j]);
        }
#else
#pragma unroll
        for (int j = 0; j < K; ++j) lv[j] = draw_sample(seed, c, p, sl[j]);
#endif
#pragma unroll
        for (int j = 0; j < K; ++j)
            vv[j] = lv[j] ? (GPS_SPLAT_PRETEST == 1 ? __ldca(buf + sl[j]) : __ldcg(buf + sl[j])) : 0ull;
    };
    auto commit = [&](const uint32_t* sl, const bool* lv, const unsigned long long* vv) {
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (lv[j] && vv[j] > key) atomicMin(buf + sl[j], key);
    };
    if (c.passes > 0) draw(0, sa, la, va);
    for (int p = 0; p < c.passes; p += 2) {
        if (p + 1 < c.passes) draw(p + 1, sb, lb, vb);
        commit(sa, la, va);
        if (p + 1 < c.passes) {
            if (p + 2 < c.passes) draw(p + 2, sa, la, va);
            commit(sb, lb, vb);
        }
    }
#else
    for (int p = 0; p < c.passes; ++p) {
        uint32_t slot[K];
        bool live[K];
#pragma unroll
        for (int j = 0; j < K; ++j) live[j] = draw_sample(seed, c, p, slot[j]);
#pragma unroll
        for (int j = 0; j < K; ++j) {
#if GPS_SPLAT_PRETEST
            if (live[j] && (GPS_SPLAT_PRETEST == 1 ? __ldca(buf + slot[j]) : __ldcg(buf + slot[j])) > key) atomicMin(buf + slot[j], key);
#else
            if (live[j]) atomicMin(buf + slot[j], key);
#endif
        }
    }
#endif
}

// Points per thread between two block barriers: a block takes kSplatRounds consecutive 256-point
// tiles at once, with one survivor-start window of kSplatRounds * 256 entries (the survivors
// owning those points are the first tile's owner and at most that many more).  Fewer barriers
// mean less time waiting for a block's slowest warp: on the 16M-Gaussian town orbit (1080p,
// ss 2, 4 spp) the splat took 1.90 ms/frame with 1 round, 1.854 with 2 and 1.849 with 4.  With
// more than one round the kernel is held to 64 registers (4 blocks per SM) by its launch bounds.
#ifndef GPS_SPLAT_ROUNDS
#define GPS_SPLAT_ROUNDS 4
#endif
constexpr int kSplatRounds = GPS_SPLAT_ROUNDS;
constexpr int kSplatWindow = kSplatTile * kSplatRounds;

// K > 0: unbiased splatting with K points per thread per pass; K = 0: any other setting.
template <int K>
#ifndef GPS_SPLAT_MIN_BLOCKS
#define GPS_SPLAT_MIN_BLOCKS 4
#endif
// (K = 8 keeps two passes of eight samples in flight: more registers, fewer resident blocks)
__global__ void __launch_bounds__(kSplatTile, kSplatRounds > 1 ? (K >= 8 ? 2 : GPS_SPLAT_MIN_BLOCKS) : 1) splat_kernel(SplatArgs a) {
    __shared__ uint32_t s_start[kSplatWindow];
    __shared__ uint32_t s_spread[kTileSize];
    if (GPS_SPLAT_MORTON_LUT && threadIdx.x < kTileSize) s_spread[threadIdx.x] = morton_spread(threadIdx.x);
    const uint32_t points = a.counters->points;
    const uint32_t survivors = a.counters->survivors;
    // the pass's work order: screen bins unless the scan had to truncate the pass or a bin was
    // too crowded to sort into
    const bool binned = a.sorted_gid && a.counters->truncated == 0u && a.counters->crowded == 0u;
    const uint32_t* __restrict__ gids = binned ? a.sorted_gid : a.surv_gid;
    const uint32_t* __restrict__ first_q = binned ? a.sorted_qstart : a.surv_start;
    const uint32_t* __restrict__ point_base = binned ? a.sorted_pstart : nullptr;
    // the preprocess of the next pass accumulates into these; nothing here reads them
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.clear_a_words; i += gridDim.x * blockDim.x)
        a.clear_a[i] = 0ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.clear_b_words; i += gridDim.x * blockDim.x)
        a.clear_b[i] = 0ull;
    if (a.mask_iter && points > 0u && blockIdx.x == 0 && threadIdx.x == 0) *a.mask_iter += 1u;
    // splats walk position q0 + threadIdx.x of a tile whose survivor starts are in `starts`
    auto splat_tile_point = [&](uint32_t q0, uint32_t r0, const uint32_t* starts, int window, int lo0, int hi0) {
        const uint32_t q = q0 + threadIdx.x;
        if (q < points && starts[0] <= q) {
            int lo = lo0, hi = hi0;  // largest k with starts[k] <= q
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (starts[mid] <= q) lo = mid;
                else hi = mid - 1;
            }
            // the reference's point index (the seed): the walk position itself in Gaussian
            // order, the survivor's first point plus the offset in screen-bin order
            const uint32_t p = point_base ? __ldg(&point_base[r0 + lo]) + (q - starts[lo]) : q;
            const uint32_t g = __ldg(&gids[r0 + lo]);
            if (g < a.n) {  // always true unless the scan gave up (device_timeouts)
                const float4* rp = reinterpret_cast<const float4*>(a.records + g);
                SplatRecord rec;
                rec.a = __ldg(rp + 0);
                rec.b = __ldg(rp + 1);
                rec.c = __ldg(rp + 2);
                rec.d = __ldg(reinterpret_cast<const uint4*>(rp + 3));
                if constexpr (K > 0) {
                    splat_point_unbiased_k<K>(p, rec, a.fc, a.frame_seed, a.buffer, s_spread);
                } else {
                    if (a.fc.use_unbiased) splat_point_unbiased(p, rec, a.fc, a.frame_seed, a.buffer);
                    else splat_point_biased(p, rec, a.fc, a.frame_seed, a.buffer);
                }
            }
        }
    };
    auto start_of = [&](uint32_t r0, uint32_t k) {
        const uint32_t r = r0 + k;
        return (r0 < survivors && r < survivors) ? first_q[r] : 0xFFFFFFFFu;
    };
    // grouped tiles only while there are at least two groups per block; a small pass keeps one
    // tile per barrier so that its points still spread over every block
    auto walk = [&](auto rounds_c) {
        constexpr uint32_t rounds = decltype(rounds_c)::value;
        constexpr uint32_t group_points = kSplatTile * rounds;
        for (uint32_t group = blockIdx.x; (unsigned long long)group * group_points < points; group += gridDim.x) {
            const uint32_t r0 = a.tile_first_rank[group * rounds];
#pragma unroll
            for (uint32_t q = 0; q < rounds; ++q)
                s_start[q * kSplatTile + threadIdx.x] = start_of(r0, q * kSplatTile + threadIdx.x);
            __syncthreads();
            for (uint32_t q = 0; q < rounds; ++q) {
                // the tile's points belong to the owners of its first point and of the next
                // tile's first point, and to those between: the owner search starts from that
                // range (splat 1.562 -> 1.545 ms/frame on the 16M orbit)
                const uint32_t t = group * rounds + q;
                int hi0 = (int)group_points - 1;
                const int lo0 = min((int)(__ldg(&a.tile_first_rank[t]) - r0), hi0);
                if ((unsigned long long)(t + 1) * kSplatTile < points)
                    hi0 = max(lo0, min((int)(__ldg(&a.tile_first_rank[t + 1]) - r0), hi0));
                splat_tile_point(group * group_points + q * kSplatTile, r0, s_start, (int)group_points, lo0, hi0);
            }
            __syncthreads();
        }
    };
    if ((unsigned long long)points >= 2ull * gridDim.x * kSplatWindow)
        walk(std::integral_constant<uint32_t, (uint32_t)kSplatRounds>{});
    else
        walk(std::integral_constant<uint32_t, 1u>{});
}

// ---------------------------------------------------------------------------------
// Clear and resolve (gaussian_point_splatting.cu:484-548, 580-585)
// ---------------------------------------------------------------------------------
__global__ void clear_kernel(ulonglong2* __restrict__ buf, uint64_t pairs, unsigned long long value) {
    const ulonglong2 v = make_ulonglong2(value, value);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < pairs; i += (uint64_t)gridDim.x * blockDim.x)
        buf[i] = v;
}

// Where resolve_pixel reads entry i of the splat buffer from.
struct GlobalEntries {
    const uint64_t* buffer;
    __device__ __forceinline__ uint64_t operator()(int i) const {
        return __ldg(reinterpret_cast<const unsigned long long*>(buffer) + i);
    }
};
struct StagedEntries {  // a contiguous run of the buffer copied to shared memory, one pad
    const uint64_t* stage;  // word after every pixel's samples (stride = run + 1)
    int first;
    int run_log2;
    __device__ __forceinline__ uint64_t operator()(int i) const {
        const int w = i - first;
        return stage[w + (w >> run_log2)];
    }
};

// One output pixel: the mean colour of its SS x SS x spp samples and their nearest NDC depth,
// in the reference's loop order.  The depth arithmetic is kept in exactly this form (and
// loop shape) because the reference's result depends on how the compiler evaluates it under
// fast math; the parity tests check it bit for bit.
template <bool kDepthOnly, class Src>
__device__ __forceinline__ void resolve_pixel(const ResolveArgs& a, int x, int y, Src src) {
    const uint32_t idx = (uint32_t)(y * a.width + x);
    const int bx = x * a.ss, by = y * a.ss;
    const int up_w = a.width * a.ss, up_h = a.height * a.ss;
    float depth = 1e9f;
    vec3 color = make_v3(0.0f, 0.0f, 0.0f);
    for (int dx = 0; dx < a.ss; dx++)
        for (int dy = 0; dy < a.ss; dy++)
            for (int p = 0; p < a.num_passes; ++p) {
                int i = splat_index(bx + dx, by + dy, p, a.num_passes, up_w, up_h);
                if ((uint64_t)(int64_t)i >= a.entries) continue;
                uint64_t val = src(i);
                float view_depth = view_depth_from_key((val >> 36ull) & kDepthMax, a.near_plane, a.far_plane);
                float z_ndc = view_to_projected_depth(view_depth, a.near_plane, a.far_plane);
                depth = gmin(depth, z_ndc);
                if (kDepthOnly) continue;
                color.x += (float)((val >> 24) & 0xFFFu) / 255.0f;
                color.y += (float)((val >> 12) & 0xFFFu) / 255.0f;
                color.z += (float)((val >> 0) & 0xFFFu) / 255.0f;
            }
    float inv_passes = 1.0f / (float)(a.num_passes * a.ss * a.ss);
    if (!kDepthOnly) {
        a.color[3 * idx + 0] = color.x * inv_passes;
        a.color[3 * idx + 1] = color.y * inv_passes;
        a.color[3 * idx + 2] = color.z * inv_passes;
    }
    a.depth[idx] = depth;
}

// Row-major pixels (any supersampling factor).
template <bool kDepthOnly>
__global__ void __launch_bounds__(256) resolve_kernel(ResolveArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.width || y >= a.height) return;
    resolve_pixel<kDepthOnly>(a, x, y, GlobalEntries{a.buffer});
}

// Power-of-two supersampling: the pixels of each 64x64 splat tile in Morton order.  An
// output pixel's sub-pixels are then one contiguous Morton range, its samples one contiguous
// run of the buffer, and a warp reads 32 consecutive runs (4 KB at SS 2, 4 spp) instead of
// runs scattered over a tile.
__device__ __forceinline__ uint32_t morton_compact(uint32_t a) {
    a &= 0x55555555u;
    a = (a | (a >> 1)) & 0x33333333u;
    a = (a | (a >> 2)) & 0x0F0F0F0Fu;
    a = (a | (a >> 4)) & 0x00FF00FFu;
    a = (a | (a >> 8)) & 0x0000FFFFu;
    return a;
}

template <bool kDepthOnly>
__global__ void __launch_bounds__(256) resolve_morton_kernel(ResolveArgs a, int ss_log2) {
    const uint32_t tile_px = (uint32_t)kTileSize >> ss_log2;
    const uint32_t per_tile_log2 = 2u * (uint32_t)(kTileBits - ss_log2);
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tile = g >> per_tile_log2;
    const uint32_t m = g & ((1u << per_tile_log2) - 1u);
    const uint32_t tiles_per_row = (uint32_t)((a.width * a.ss + kTileSize - 1) >> kTileBits);
    const int x = (int)((tile % tiles_per_row) * tile_px + morton_compact(m));
    const int y = (int)((tile / tiles_per_row) * tile_px + morton_compact(m >> 1));
    if (x >= a.width || y >= a.height) return;
    resolve_pixel<kDepthOnly>(a, x, y, GlobalEntries{a.buffer});
}

// Staged variant: a block's pixels are consecutive in Morton-tile order, so their samples are
// one contiguous run of the buffer (px_per_block x SS*SS*spp entries, at most 48 KB).  The
// block copies the run to shared memory with coalesced 16-byte loads, all in flight at once,
// then each thread resolves its pixel from shared memory with the same per-pixel code.  A pad
// word after each pixel's samples keeps the threads of a warp, which read samples a whole
// pixel run apart, on different banks.  Used when SS*SS*spp is a power of two >= 2.
constexpr int kResolveStageBytes = 48 * 1024;
#ifndef GPS_RESOLVE_REVERSED
#define GPS_RESOLVE_REVERSED 1
#endif
#ifndef GPS_RESOLVE_PIXELS
#define GPS_RESOLVE_PIXELS 64
#endif

template <bool kDepthOnly>
__global__ void __launch_bounds__(256) resolve_staged_kernel(ResolveArgs a, int ss_log2, int run_log2) {
    extern __shared__ uint64_t stage[];
    const uint32_t run = 1u << run_log2;                            // entries per pixel
    // blocks take the buffer from its end: the splat walks screen bins (buffer tiles) in
    // ascending order, so the tiles it touched last are the ones still in L2
    const uint32_t bid = GPS_RESOLVE_REVERSED ? gridDim.x - 1u - blockIdx.x : blockIdx.x;
    const uint32_t g0 = bid * blockDim.x;
    const uint64_t first = (uint64_t)g0 * run;
    uint64_t last = first + (uint64_t)blockDim.x * run;
    if (last > a.entries) last = a.entries;
    const uint32_t chunks = (uint32_t)((last - first) / 2);        // first and last are even
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(a.buffer + first);
    for (uint32_t i = threadIdx.x; i < chunks; i += blockDim.x) {
        const ulonglong2 q = __ldcs(src + i);
        const uint32_t w = 2u * i;                                  // both words in one pixel run
        const uint32_t d = w + (w >> run_log2);
        stage[d] = q.x;
        stage[d + 1] = q.y;
    }
    __syncthreads();
    const uint32_t tile_px = (uint32_t)kTileSize >> ss_log2;
    const uint32_t per_tile_log2 = 2u * (uint32_t)(kTileBits - ss_log2);
    const uint32_t g = g0 + threadIdx.x;
    const uint32_t tile = g >> per_tile_log2;
    const uint32_t m = g & ((1u << per_tile_log2) - 1u);
    const uint32_t tiles_per_row = (uint32_t)((a.width * a.ss + kTileSize - 1) >> kTileBits);
    const int x = (int)((tile % tiles_per_row) * tile_px + morton_compact(m));
    const int y = (int)((tile / tiles_per_row) * tile_px + morton_compact(m >> 1));
    if (x >= a.width || y >= a.height) return;
    resolve_pixel<kDepthOnly>(a, x, y, StagedEntries{stage, (int)first, run_log2});
}

// ---------------------------------------------------------------------------------
// Hi-Z chain (depth_mip_chain.cu:7-67)
// ---------------------------------------------------------------------------------
// The whole chain in one launch.  A 16x16-thread block covers a 64x64 tile of the depth image:
// each thread copies its 4x4 texels into the finest level and reduces them in registers to
// the next two levels (2x2, then 1), the block reduces its 16x16 results through four more
// levels in shared memory, and the block that finishes last (a counter, no waiting) reduces
// the remaining coarse levels.  Every texel is the min/max of the same finest texels as with
// one launch per level, so the chain is identical.  Level j from the finest (j = 1, 2, ...)
// reduces with min while j <= min_levels, else with max.
constexpr int kHizThreads = 16;                  // threads per block edge
constexpr int kHizTile = 4 * kHizThreads;        // finest texels per block edge

__device__ __forceinline__ float hiz_op(bool use_min, float a, float b) { return use_min ? fminf(a, b) : fmaxf(a, b); }

__global__ void __launch_bounds__(kHizThreads * kHizThreads) hiz_build_kernel(HizView c, const float* __restrict__ src,
                                                                               int min_levels) {
    __shared__ float sm[kHizThreads * kHizThreads];
    __shared__ int s_last;
    const int L = c.levels - 1;
    const int tx = threadIdx.x % kHizThreads, ty = threadIdx.x / kHizThreads;
    const int gx = blockIdx.x * kHizThreads + tx, gy = blockIdx.y * kHizThreads + ty;  // coords at level L-2
    const int W = c.level_w[L], H = c.level_h[L];
    float f[4][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = 4 * gx + u, y = 4 * gy + v;
            f[v][u] = 0.0f;
            if (x < W && y < H) {
                f[v][u] = src[(uint64_t)y * W + x];
                c.mip[c.level_off[L] + (uint64_t)y * W + x] = f[v][u];
            }
        }
    float r = 0.0f;  // this thread's texel at the last level reduced so far
    bool have = false;
    if (L >= 1) {
        const int l = L - 1;
        const bool use_min = 0 < min_levels;
        const int wl = c.level_w[l], hl = c.level_h[l];
        float q[2][2];
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                float acc = use_min ? INFINITY : -INFINITY;
#pragma unroll
                for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                    for (int dx = 0; dx < 2; ++dx)
                        if (4 * gx + 2 * i + dx < W && 4 * gy + 2 * j + dy < H) acc = hiz_op(use_min, acc, f[2 * j + dy][2 * i + dx]);
                q[j][i] = acc;
                const int x = 2 * gx + i, y = 2 * gy + j;
                if (x < wl && y < hl) c.mip[c.level_off[l] + (uint64_t)y * wl + x] = acc;
            }
        if (L >= 2) {
            const int l2 = L - 2;
            const bool use_min2 = 1 < min_levels;
            float acc = use_min2 ? INFINITY : -INFINITY;
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int i = 0; i < 2; ++i)
                    if (2 * gx + i < wl && 2 * gy + j < hl) acc = hiz_op(use_min2, acc, q[j][i]);
            r = acc;
            have = true;
            if (gx < c.level_w[l2] && gy < c.level_h[l2]) c.mip[c.level_off[l2] + (uint64_t)gy * c.level_w[l2] + gx] = acc;
        }
    }
    const int shared_levels = have ? min(4, L - 2) : 0;   // levels L-3 .. L-6 in shared memory
    if (have) sm[ty * kHizThreads + tx] = r;
    __syncthreads();
    for (int j = 1; j <= shared_levels; ++j) {
        const int l = L - 2 - j;
        const bool use_min = (j + 1) < min_levels;
        const int half = kHizThreads >> j;
        const int wf = c.level_w[l + 1], hf = c.level_h[l + 1];
        const bool act = tx < half && ty < half;
        const int bx = blockIdx.x * half + tx, by = blockIdx.y * half + ty;
        float acc = use_min ? INFINITY : -INFINITY;
        if (act) {
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                    if (2 * bx + dx < wf && 2 * by + dy < hf) acc = hiz_op(use_min, acc, sm[(2 * ty + dy) * kHizThreads + 2 * tx + dx]);
        }
        __syncthreads();
        if (act) {
            sm[ty * kHizThreads + tx] = acc;
            if (bx < c.level_w[l] && by < c.level_h[l]) c.mip[c.level_off[l] + (uint64_t)by * c.level_w[l] + bx] = acc;
        }
        __syncthreads();
    }
    const int done_levels = (L >= 2 ? 2 : L) + shared_levels;   // levels below L written so far
    if (done_levels >= L) return;                                // the whole chain fits one block
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(c.done, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int l = L - done_levels - 1; l >= 0; --l) {
        const bool use_min = (L - 1 - l) < min_levels;
        const int wl = c.level_w[l], hl = c.level_h[l];
        const int wf = c.level_w[l + 1], hf = c.level_h[l + 1];
        const float* fine = c.mip + c.level_off[l + 1];
        for (int i = threadIdx.x; i < wl * hl; i += blockDim.x) {
            const int x = i % wl, y = i / wl;
            float acc = use_min ? INFINITY : -INFINITY;
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int fx = 2 * x + dx, fy = 2 * y + dy;
                    if (fx < wf && fy < hf) acc = hiz_op(use_min, acc, __ldcg(fine + (uint64_t)fy * wf + fx));
                }
            c.mip[c.level_off[l] + (uint64_t)y * wl + x] = acc;
        }
        __threadfence_block();
        __syncthreads();
    }
    if (threadIdx.x == 0) *c.done = 0u;
}

// ---------------------------------------------------------------------------------
// Half-precision scene: encode from the FP32 arrays, tile copies (load time)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
    return (uint32_t)__half_as_ushort(__float2half_rn(lo)) | ((uint32_t)__half_as_ushort(__float2half_rn(hi)) << 16);
}

// origin of every kHalfOriginBlock Gaussians: the centre of their means' bounding box, and in w
// the step of the 16-bit fixed-point offsets from it (the largest half-extent / 32767)
__global__ void half_origins_kernel(const float4* __restrict__ pos_op, uint32_t n, float4* __restrict__ origin) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t begin = b * kHalfOriginBlock;
    if (begin >= n) return;
    const uint32_t end = min(begin + kHalfOriginBlock, n);
    float3 lo = make_float3(INFINITY, INFINITY, INFINITY), hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t g = begin; g < end; ++g) {
        const float4 p = pos_op[g];
        lo = make_float3(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z));
        hi = make_float3(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z));
    }
    const float3 o = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
    const float h = fmaxf(fmaxf(fmaxf(hi.x - o.x, o.x - lo.x), fmaxf(hi.y - o.y, o.y - lo.y)),
                          fmaxf(hi.z - o.z, o.z - lo.z));
    const float k = __fdiv_rn(h, 32767.0f);
    origin[b] = make_float4(o.x, o.y, o.z, k >= 1.0e-30f ? k : 0.0f);
}

__device__ __forceinline__ uint32_t fixed16(float v, float o, float k) {
    const int q = k > 0.0f ? max(-32767, min(32767, __float2int_rn(__fdiv_rn(v - o, k)))) : 0;
    return (uint32_t)q & 0xFFFFu;
}

__global__ void encode_half_kernel(const float4* __restrict__ pos_op, const float4* __restrict__ rot,
                                   const float4* __restrict__ scale, const float4* __restrict__ sh,
                                   const float4* __restrict__ origin, uint32_t n, uint4* __restrict__ rec,
                                   uint4* __restrict__ scl, uint4* __restrict__ acq) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const float4 p = pos_op[g], q = rot[g], c = scale[g], o = origin[g / kHalfOriginBlock];
    const uint32_t op16 = (uint32_t)__half_as_ushort(__float2half_rn(p.w));
    rec[g] = make_uint4(fixed16(p.x, o.x, o.w) | (fixed16(p.y, o.y, o.w) << 16), fixed16(p.z, o.z, o.w) | (op16 << 16),
                        pack_h2(q.x, q.y), pack_h2(q.z, q.w));
    float v[48];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const float4 t = sh[(size_t)g * 12 + i];
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
    }
    // AC terms: 8-bit integers on a per-band scale (band 1: AC 0-8, band 2: 9-23, band 3: 24-44),
    // scale = the band's max |c| / 127 rounded up to bf16, so that every |c| / scale <= 127
    float mb[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int e = 0; e < 45; ++e) {
        const int b = e < 9 ? 0 : (e < 24 ? 1 : 2);
        mb[b] = fmaxf(mb[b], fabsf(v[3 + e]));
    }
    uint32_t sb[3];
    float sc[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const uint32_t bits = __float_as_uint(mb[b] / 127.0f);
        sb[b] = (bits >> 16) + ((bits & 0xFFFFu) ? 1u : 0u);
        sc[b] = __uint_as_float(sb[b] << 16);
    }
    scl[g] = make_uint4(pack_h2(c.x, c.y), pack_h2(c.z, v[0]), pack_h2(v[1], v[2]), sb[0] | (sb[1] << 16));
    uint32_t w[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) w[i] = 0u;
#pragma unroll
    for (int e = 0; e < 45; ++e) {
        const float k = sc[e < 9 ? 0 : (e < 24 ? 1 : 2)];
        const int q = k > 0.0f ? max(-127, min(127, __float2int_rn(__fdiv_rn(v[3 + e], k)))) : 0;
        w[e >> 2] |= ((uint32_t)q & 0xFFu) << (8 * (e & 3));
    }
    w[11] |= sb[2] << 8;  // bytes 45-46: band 3's scale
#pragma unroll
    for (int i = 0; i < 3; ++i) acq[(size_t)g * 3 + i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}

// copies of a half scene: origins of copy k = source origins + (dx[k], 0, dz[k])
__global__ void translate_origins_kernel(const float4* __restrict__ src, uint32_t count, float dx, float dz,
                                         float4* __restrict__ dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 o = src[i];
    dst[i] = make_float4(o.x + dx, o.y, o.z + dz, o.w);
}

// cull blocks of the tiled scene: node j covers Gaussians [j*pb, j*pb+pb) inside one copy and is
// the union of the source nodes it spans, translated with its copy
__global__ void tile_nodes_kernel(const float4* __restrict__ src, uint32_t src_pb, uint32_t src_n, uint32_t pb,
                                  uint32_t copies, const float2* __restrict__ offsets, uint64_t total,
                                  float4* __restrict__ dst, uint32_t nodes) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nodes) return;
    const uint64_t begin = (uint64_t)j * pb;
    const uint64_t end = min(begin + pb, total);
    const uint32_t k = (uint32_t)(begin / src_n);
    const uint32_t s0 = (uint32_t)((begin - (uint64_t)k * src_n) / src_pb);
    const uint32_t s1 = (uint32_t)((end - 1 - (uint64_t)k * src_n) / src_pb);
    float3 lo = make_float3(INFINITY, INFINITY, INFINITY), hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t s = s0; s <= s1; ++s) {
        const float4 a = src[2 * s], b = src[2 * s + 1];
        lo = make_float3(fminf(lo.x, a.x), fminf(lo.y, a.y), fminf(lo.z, a.z));
        hi = make_float3(fmaxf(hi.x, b.x), fmaxf(hi.y, b.y), fmaxf(hi.z, b.z));
    }
    const float2 t = offsets[k];
    dst[2 * j] = make_float4(lo.x + t.x, lo.y, lo.z + t.y, __uint_as_float((uint32_t)begin));
    dst[2 * j + 1] = make_float4(hi.x + t.x, hi.y, hi.z + t.y, __uint_as_float((uint32_t)(end - begin)));
}

// ---------------------------------------------------------------------------------
// Block AABBs at load time (gaussian_bvh.cu:111-144).  The reference computes these on the
// host in IEEE single precision without fused multiply-adds; the _rn intrinsics below keep
// nvcc from contracting, so the boxes are bit-identical to the host computation.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ void host_order_cov_diag(vec3 s, vec4 q, float out[3]) {
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    float qxx = rmul(x, x), qyy = rmul(y, y), qzz = rmul(z, z);
    float qxz = rmul(x, z), qxy = rmul(x, y), qyz = rmul(y, z);
    float qwx = rmul(w, x), qwy = rmul(w, y), qwz = rmul(w, z);
    float r[3][3];
    r[0][0] = rsub(1.0f, rmul(2.0f, radd(qyy, qzz)));
    r[0][1] = rmul(2.0f, radd(qxy, qwz));
    r[0][2] = rmul(2.0f, rsub(qxz, qwy));
    r[1][0] = rmul(2.0f, rsub(qxy, qwz));
    r[1][1] = rsub(1.0f, rmul(2.0f, radd(qxx, qzz)));
    r[1][2] = rmul(2.0f, radd(qyz, qwx));
    r[2][0] = rmul(2.0f, radd(qxz, qwy));
    r[2][1] = rmul(2.0f, rsub(qyz, qwx));
    r[2][2] = rsub(1.0f, rmul(2.0f, radd(qxx, qyy)));
    // M = R * S, column j = (R0*S[j].x + R1*S[j].y) + R2*S[j].z with S diagonal
    float sd[3][3] = {{s.x, 0.0f, 0.0f}, {0.0f, s.y, 0.0f}, {0.0f, 0.0f, s.z}};
    float m[3][3];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            m[j][i] = radd(radd(rmul(r[0][i], sd[j][0]), rmul(r[1][i], sd[j][1])), rmul(r[2][i], sd[j][2]));
    // cov = M * M^T: cov[j][i] = (M0[i]*M[0][j] + M1[i]*M[1][j]) + M2[i]*M[2][j]; diagonal only
    for (int i = 0; i < 3; ++i)
        out[i] = radd(radd(rmul(m[0][i], m[0][i]), rmul(m[1][i], m[1][i])), rmul(m[2][i], m[2][i]));
}

__global__ void block_bounds_kernel(const float4* __restrict__ pos_op, const float4* __restrict__ rot,
                                    const float4* __restrict__ scale, uint32_t n, uint32_t per_block,
                                    float4* __restrict__ nodes, uint32_t node_count) {
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= node_count) return;
    const uint32_t begin = node * per_block;
    const uint32_t end = min(begin + per_block, n);
    float bmin[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float bmax[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (uint32_t g = begin; g < end; ++g) {
        float4 p = pos_op[g], q = rot[g], s = scale[g];
        float d[3];
        host_order_cov_diag(make_v3(s.x, s.y, s.z), make_v4(q.x, q.y, q.z, q.w), d);
        float mean[3] = {p.x, p.y, p.z};
        for (int i = 0; i < 3; ++i) {
            float ext = rmul(kTruncationStd, __fsqrt_rn(d[i]));
            float lo = rsub(mean[i], ext), hi = radd(mean[i], ext);
            bmin[i] = (lo < bmin[i]) ? lo : bmin[i];
            bmax[i] = (bmax[i] < hi) ? hi : bmax[i];
        }
    }
    nodes[2 * node] = make_float4(bmin[0], bmin[1], bmin[2], __uint_as_float(begin));
    nodes[2 * node + 1] = make_float4(bmax[0], bmax[1], bmax[2], __uint_as_float(end - begin));
}

// ---------------------------------------------------------------------------------
// Post-processing (post_processing_kernels.cuh:108-285)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
__device__ __forceinline__ vec3 mix3s(vec3 x, vec3 y, float a) {
    return make_v3(mixf(x.x, y.x, a), mixf(x.y, y.y, a), mixf(x.z, y.z, a));
}
__device__ __forceinline__ vec3 ld3(const float* p, int i) { return make_v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// temporalRender reads the 3x3 neighbourhood of the current colour buffer while other threads
// overwrite that same buffer with blended results, so its output depends on thread order.
// Here the blended colour goes to a separate buffer (out_color, never aliasing cur_color): the
// neighbourhood is always the unblended current frame and the result is deterministic.
__global__ void taa_kernel(uint8_t* __restrict__ image, float* __restrict__ out_color,
                           const float* __restrict__ cur_color,
                           const float* __restrict__ prev_color, const float* __restrict__ cur_depth,
                           const float* __restrict__ prev_depth, mat4 reproj, float blend, int width, int height,
                           int frame_number) {
    // 32 x 8 pixel blocks: a block's 3 x 3 neighbourhood reads stay within 10 rows of L1
    // (TAA 0.042 -> 0.038 ms at 1080p)
    const int x = blockIdx.x * 32 + (int)(threadIdx.x & 31u);
    const int y = blockIdx.y * 8 + (int)(threadIdx.x >> 5);
    if (x >= width || y >= height) return;
    const int idx = y * width + x;
    vec3 color = ld3(cur_color, idx);
    float depth = cur_depth[idx];
    if (frame_number > 0) {
        vec4 clip = make_v4((x + 0.5f) / width * 2.0f - 1.0f, (y + 0.5f) / height * 2.0f - 1.0f, depth, 1.0f);
        vec4 prev = reproj * clip;
        prev = make_v4(prev.x / prev.w, prev.y / prev.w, prev.z / prev.w, prev.w / prev.w);
        float px = (prev.x * 0.5f + 0.5f) * width - 0.5f;
        float py = (prev.y * 0.5f + 0.5f) * height - 0.5f;
        if (px >= 0 && px < width && py >= 0 && py < height) {
            // bilinearSampleCombined
            int x0 = (int)floorf(px), y0 = (int)floorf(py);
            int x1 = x0 + 1, y1 = y0 + 1;
            x0 = (x0 < 0) ? 0 : ((x0 >= width) ? width - 1 : x0);
            y0 = (y0 < 0) ? 0 : ((y0 >= height) ? height - 1 : y0);
            x1 = (x1 < 0) ? 0 : ((x1 >= width) ? width - 1 : x1);
            y1 = (y1 < 0) ? 0 : ((y1 >= height) ? height - 1 : y1);
            float tx = px - floorf(px);
            float ty = py - floorf(py);
            int i00 = y0 * width + x0, i10 = y0 * width + x1, i01 = y1 * width + x0, i11 = y1 * width + x1;
            (void)prev_depth;
            vec3 top = mix3s(ld3(prev_color, i00), ld3(prev_color, i10), tx);
            vec3 bottom = mix3s(ld3(prev_color, i01), ld3(prev_color, i11), tx);
            vec3 hist = mix3s(top, bottom, ty);
            // computeNeighborhoodMinMax
            vec3 nmin = make_v3(1e9f, 1e9f, 1e9f), nmax = make_v3(-1e9f, -1e9f, -1e9f);
            for (int dy = -1; dy <= 1; dy++) {
                int yy = y + dy;
                if (yy < 0 || yy >= height) continue;
                for (int dx = -1; dx <= 1; dx++) {
                    int xx = x + dx;
                    if (xx < 0 || xx >= width) continue;
                    vec3 c = ld3(cur_color, yy * width + xx);
                    nmin = make_v3(gmin(nmin.x, c.x), gmin(nmin.y, c.y), gmin(nmin.z, c.z));
                    nmax = make_v3(gmax(nmax.x, c.x), gmax(nmax.y, c.y), gmax(nmax.z, c.z));
                }
            }
            vec3 h = make_v3(gclamp(hist.x, nmin.x - 0.05f, nmax.x + 0.05f), gclamp(hist.y, nmin.y - 0.05f, nmax.y + 0.05f),
                             gclamp(hist.z, nmin.z - 0.05f, nmax.z + 0.05f));
            color = mix3s(color, h, blend);
        }
    }
    out_color[3 * idx + 0] = color.x;
    out_color[3 * idx + 1] = color.y;
    out_color[3 * idx + 2] = color.z;
    vec3 o = make_v3(gclamp(color.x, 0.0f, 1.0f) * 255.0f, gclamp(color.y, 0.0f, 1.0f) * 255.0f,
                     gclamp(color.z, 0.0f, 1.0f) * 255.0f);
    image[3 * idx + 0] = (uint8_t)roundf(o.x);
    image[3 * idx + 1] = (uint8_t)roundf(o.y);
    image[3 * idx + 2] = (uint8_t)roundf(o.z);
}

__global__ void progressive_kernel(uint8_t* __restrict__ image, float* __restrict__ cur, float* __restrict__ accum,
                                   int width, int height, int frames) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= width * height) return;
    vec3 color = ld3(cur, idx);
    if (frames > 1) color = color + ld3(accum, idx);
    cur[3 * idx + 0] = color.x;
    cur[3 * idx + 1] = color.y;
    cur[3 * idx + 2] = color.z;
    accum[3 * idx + 0] = 0.0f;
    accum[3 * idx + 1] = 0.0f;
    accum[3 * idx + 2] = 0.0f;
    color = color * (255.0f / (float)frames);
    color = make_v3(gclamp(color.x, 0.0f, 255.0f), gclamp(color.y, 0.0f, 255.0f), gclamp(color.z, 0.0f, 255.0f));
    image[3 * idx + 0] = (uint8_t)roundf(color.x);
    image[3 * idx + 1] = (uint8_t)roundf(color.y);
    image[3 * idx + 2] = (uint8_t)roundf(color.z);
}

int g_num_sms = 0;

}  // namespace

// ---------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------
namespace {
template <typename... KArgs, typename... Args>
void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args... args) {
    kernel<<<grid, block, smem, stream>>>(args...);
}
}  // namespace

void launch_block_cull(const BlockView& b, const FrameConst& fc, const HizView& hiz, cudaStream_t stream) {
    if (b.node_count == 0) return;
    uint32_t threads = b.words * 32;
    launch_k(block_cull_kernel, (threads + 255) / 256, 256, 0, stream, b, fc, hiz);
}

void launch_visible_chunks(const BlockView& b, uint32_t n, uint32_t* list, uint32_t* mask_a, uint32_t* mask_b,
                           const uint32_t* mask_iter, cudaStream_t stream) {
    if (n == 0) return;
    const uint32_t chunks = (n + 31u) >> 5;
    const uint32_t want = (chunks + 255u) / 256u;
    launch_k(visible_chunks_kernel, want < 1184u ? want : 1184u, 256, 0, stream, b, n, list, mask_a, mask_b, mask_iter);
}

// Resident blocks of the persistent preprocess on this device, capped by the work.
template <class Scene, bool kImmediate>
int preprocess_grid_size(uint32_t n) {
    static int per_sm = 0;
    if (per_sm == 0) {
        int blocks = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, preprocess_kernel<Scene, kImmediate>, 256, 0);
        per_sm = blocks < 1 ? 1 : blocks;
    }
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const uint64_t want = ((uint64_t)n + 255) / 256;
    const uint64_t cap = (uint64_t)g_num_sms * (uint64_t)per_sm;
    return (int)(want < cap ? want : cap);
}

template <class Scene>
void launch_preprocess(const PreprocessArgs& a, const Scene& s, cudaStream_t stream) {
    if (a.n == 0) return;
    if (a.immediate_threshold > 0)
        launch_k(preprocess_kernel<Scene, true>, preprocess_grid_size<Scene, true>(a.n), 256, 0, stream, a, s);
    else
        launch_k(preprocess_kernel<Scene, false>, preprocess_grid_size<Scene, false>(a.n), 256, 0, stream, a, s);
}

void launch_preprocess_fp32(const PreprocessArgs& a, const SceneFP32& s, cudaStream_t stream) {
    launch_preprocess(a, s, stream);
}

void launch_preprocess_half(const PreprocessArgs& a, const SceneHalf& s, cudaStream_t stream) {
    launch_preprocess(a, s, stream);
}

void launch_preprocess_compressed(const PreprocessArgs& a, const SceneCompressed& s, cudaStream_t stream) {
    launch_preprocess(a, s, stream);
}

static_assert(kScanTile == kScanTileGaussians, "scan tile size");
// tile words a scan of n Gaussians may use (the small-tile count, an upper bound)
uint32_t scan_tile_count(uint32_t n) { return (uint32_t)(((uint64_t)n + kScanTileSmall - 1) / kScanTileSmall); }

int scan_tile_shift(uint32_t n) { return n >= kScanBigScene ? 14 : 12; }

void launch_scan_fused(const ScanArgs& a, cudaStream_t stream) {
    if (a.n == 0) {
        cudaMemsetAsync(a.counters, 0, sizeof(PassCounters), stream);
        return;
    }
    const bool big = a.n >= kScanBigScene;
    const uint32_t tiles = (uint32_t)(((uint64_t)a.n + (big ? kScanTile : kScanTileSmall) - 1) / (big ? kScanTile : kScanTileSmall));
    launch_k(scan_tiles_kernel, a.bins ? 2 : 1, kTileScanThreads, 0, stream, a, tiles);
    if (big) launch_k(scan_write_fused_kernel<kScanRoundsMax>, tiles, kScanThreads, 0, stream, a);
    else launch_k(scan_write_fused_kernel<1>, tiles, kScanThreads, 0, stream, a);
}

void launch_scan(const ScanArgs& a, uint32_t scan_tiles, cudaStream_t stream) {
    if (scan_tiles == 0 || a.n == 0) {
        cudaMemsetAsync(a.counters, 0, sizeof(PassCounters), stream);
        return;
    }
    if (a.n >= kScanBigScene) {  // fewer, larger tiles: four rounds per thread
        const uint32_t tiles = (uint32_t)(((uint64_t)a.n + kScanTile - 1) / kScanTile);
        launch_k(scan_reduce_kernel<kScanRoundsMax>, tiles, kScanThreads, 0, stream, a);
        launch_k(scan_tiles_kernel, 1, kTileScanThreads, 0, stream, a, tiles);
        launch_k(scan_write_kernel<kScanRoundsMax>, tiles, kScanThreads, 0, stream, a);
    } else {
        const uint32_t tiles = (uint32_t)(((uint64_t)a.n + kScanTileSmall - 1) / kScanTileSmall);
        launch_k(scan_reduce_kernel<1>, tiles, kScanThreads, 0, stream, a);
        launch_k(scan_tiles_kernel, 1, kTileScanThreads, 0, stream, a, tiles);
        launch_k(scan_write_kernel<1>, tiles, kScanThreads, 0, stream, a);
    }
    const uint64_t max_tiles = ((uint64_t)a.max_points + a.tile_points - 1) / a.tile_points;
    const uint64_t want = (max_tiles + 255) / 256;
    const int owner_grid = (int)(want < 1184 ? (want ? want : 1) : 1184);  // 148 SMs x 8
    launch_k(tile_owner_kernel, owner_grid, 256, 0, stream, a.surv_start, a.tile_first_rank, a.counters, a.tile_points,
             a.mask_iter);
}

template <int K>
int splat_blocks_per_sm() {
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, splat_kernel<K>, kSplatTile, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

int splat_grid_size(int block) {
    (void)block;
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return g_num_sms * splat_blocks_per_sm<0>();
}

void launch_splat(const SplatArgs& a, int grid, int block, cudaStream_t stream) {
    (void)block;
    if (g_num_sms == 0) splat_grid_size(kSplatTile);
    // a persistent grid: as many blocks as fit on the device at once
    if (a.fc.use_unbiased && a.fc.k_points == 4) {
        launch_k(splat_kernel<4>, g_num_sms * splat_blocks_per_sm<4>(), kSplatTile, 0, stream, a);
    } else if (a.fc.use_unbiased && a.fc.k_points == 2) {
        launch_k(splat_kernel<2>, g_num_sms * splat_blocks_per_sm<2>(), kSplatTile, 0, stream, a);
    } else if (a.fc.use_unbiased && a.fc.k_points == 8) {
        launch_k(splat_kernel<8>, g_num_sms * splat_blocks_per_sm<8>(), kSplatTile, 0, stream, a);
    } else if (a.fc.use_unbiased && a.fc.k_points == 1) {
        launch_k(splat_kernel<1>, g_num_sms * splat_blocks_per_sm<1>(), kSplatTile, 0, stream, a);
    } else {
        launch_k(splat_kernel<0>, grid, kSplatTile, 0, stream, a);
    }
}

void launch_clear(uint64_t* buf, uint64_t entries, uint64_t value, cudaStream_t stream) {
    uint64_t pairs = entries / 2;
    int grid = (int)((pairs + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    if (grid < 1) grid = 1;
    launch_k(clear_kernel, grid, 256, 0, stream, reinterpret_cast<ulonglong2*>(buf), pairs, value);
    if (entries & 1) cudaMemcpyAsync(buf + entries - 1, &buf[0], 8, cudaMemcpyDeviceToDevice, stream);
}

void launch_resolve(const ResolveArgs& a, bool depth_only, cudaStream_t stream) {
    int ss_log2 = -1;
    for (int l = 0; l <= 3; ++l)
        if (a.ss == (1 << l)) ss_log2 = l;
    if (ss_log2 >= 0) {
        const uint64_t tiles = ((uint64_t)(a.width * a.ss + kTileSize - 1) >> kTileBits) *
                               ((uint64_t)(a.height * a.ss + kTileSize - 1) >> kTileBits);
        const uint64_t threads = tiles << (2 * (kTileBits - ss_log2));
        const uint32_t run = (uint32_t)(a.ss * a.ss * a.num_passes);
        int run_log2 = -1;
        for (int l = 1; l <= 12; ++l)
            if (run == (1u << l)) run_log2 = l;
        const uint32_t run_bytes = (run + 1u) * 8u;                 // with the pad word
        uint32_t px = GPS_RESOLVE_PIXELS;  // pixels (threads) per block
        while (px > 32 && px * run_bytes > (uint32_t)kResolveStageBytes) px >>= 1;
        if (run_log2 > 0 && px * run_bytes <= (uint32_t)kResolveStageBytes && (uint64_t)a.entries <= 0x7FFFFFFFull) {
            const unsigned grid = (unsigned)((threads + px - 1) / px);
            const size_t smem = (size_t)px * run_bytes;
            if (depth_only) launch_k(resolve_staged_kernel<true>, grid, px, smem, stream, a, ss_log2, run_log2);
            else launch_k(resolve_staged_kernel<false>, grid, px, smem, stream, a, ss_log2, run_log2);
            return;
        }
        const unsigned grid = (unsigned)((threads + 255) / 256);
        if (depth_only) launch_k(resolve_morton_kernel<true>, grid, 256, 0, stream, a, ss_log2);
        else launch_k(resolve_morton_kernel<false>, grid, 256, 0, stream, a, ss_log2);
        return;
    }
    dim3 block(16, 16);
    dim3 grid((a.width + 15) / 16, (a.height + 15) / 16);
    if (depth_only) launch_k(resolve_kernel<true>, grid, block, 0, stream, a);
    else launch_k(resolve_kernel<false>, grid, block, 0, stream, a);
}

void launch_hiz_build(const HizView& h, const float* depth, int min_levels, cudaStream_t stream) {
    const int L = h.levels - 1;
    dim3 grid((h.level_w[L] + kHizTile - 1) / kHizTile, (h.level_h[L] + kHizTile - 1) / kHizTile);
    launch_k(hiz_build_kernel, grid, kHizThreads * kHizThreads, 0, stream, h, depth, min_levels);
}

void launch_encode_half(const float4* pos_op, const float4* rot, const float4* scale, const float4* sh, uint32_t n,
                        float4* origin, uint4* rec, uint4* scl, uint4* acq, cudaStream_t stream) {
    if (n == 0) return;
    const uint32_t blocks = (n + kHalfOriginBlock - 1) / kHalfOriginBlock;
    half_origins_kernel<<<(blocks + 255) / 256, 256, 0, stream>>>(pos_op, n, origin);
    encode_half_kernel<<<(n + 255) / 256, 256, 0, stream>>>(pos_op, rot, scale, sh, origin, n, rec, scl, acq);
}

void launch_translate_origins(const float4* src, uint32_t count, float dx, float dz, float4* dst, cudaStream_t stream) {
    if (count) translate_origins_kernel<<<(count + 255) / 256, 256, 0, stream>>>(src, count, dx, dz, dst);
}

void launch_tile_nodes(const float4* src, uint32_t src_pb, uint32_t src_n, uint32_t pb, uint32_t copies,
                       const float2* offsets, uint64_t total, float4* dst, uint32_t nodes, cudaStream_t stream) {
    if (nodes) tile_nodes_kernel<<<(nodes + 255) / 256, 256, 0, stream>>>(src, src_pb, src_n, pb, copies, offsets, total, dst, nodes);
}

void launch_block_bounds(const float4* pos_op, const float4* rot, const float4* scale, uint32_t n,
                         uint32_t per_block, float4* nodes, cudaStream_t stream) {
    uint32_t node_count = (n + per_block - 1) / per_block;
    if (node_count == 0) return;
    block_bounds_kernel<<<(node_count + 255) / 256, 256, 0, stream>>>(pos_op, rot, scale, n, per_block, nodes,
                                                                       node_count);
}

void launch_taa(uint8_t* image, float* out_color, const float* cur_color, const float* prev_color,
                const float* cur_depth, const float* prev_depth, const mat4& reproj, float blend, int width, int height,
                int frame_number, cudaStream_t stream) {
    const dim3 grid((unsigned)((width + 31) / 32), (unsigned)((height + 7) / 8));
    launch_k(taa_kernel, grid, 256, 0, stream, image, out_color, cur_color, prev_color, cur_depth, prev_depth, reproj,
             blend, width, height, frame_number);
}

void launch_progressive(uint8_t* image, float* cur_color, float* accum, int width, int height, int frames,
                        cudaStream_t stream) {
    int n = width * height;
    launch_k(progressive_kernel, (n + 255) / 256, 256, 0, stream, image, cur_color, accum, width, height, frames);
}

// ---------------------------------------------------------------------------------
// Allocation-free point scan.
//
// Some callers cannot allocate device memory at the moment they need the scan: code running
// inside a CUDA-graph capture or a stream-ordered pipeline where cudaMalloc would synchronise
// the device, a host with a fixed device-memory pool or budget enforced by its own allocator,
// or a plugin host that owns every buffer and forbids its plugins from allocating. For them
// the scan's only scratch — the survivor and point totals of every scan tile — lives
// in this file-scope device array, and the caller passes all inputs and outputs. The array is
// shared by every call on a device and keeps the previous call's contents; each call rewrites
// every word it reads before reading it (tile totals, then prefixes); calls that overlap on the GPU
// (different streams, or host threads on the same device) race on it and must be serialised.
// ---------------------------------------------------------------------------------
constexpr uint32_t kNoAllocScanMaxTiles = 65536;  // 512 KiB of tile words
constexpr uint64_t kNoAllocScanMaxGaussians = 1ull << 28;  // the stated limit
static_assert(kNoAllocScanMaxGaussians / kScanTileSmall <= kNoAllocScanMaxTiles, "scratch too small");
static __device__ __align__(256) unsigned long long g_noalloc_scan_scratch[kNoAllocScanMaxTiles + 1];

namespace {
// The array's device address belongs to the module as loaded into one CUDA context: a driver
// API context other than the device's primary one, or the primary context re-created after
// cudaDeviceReset, loads the module again at another address.  So the cache is keyed on the
// current context's ID (cuCtxGetId: unique for the life of the process, never reused), fetched
// through the runtime's driver entry points so the library needs no libcuda link.
struct NoAllocScratchEntry {
    unsigned long long ctx_id;
    unsigned long long* ptr;
};
constexpr int kNoAllocCacheSlots = 64;
std::mutex g_noalloc_mutex;
NoAllocScratchEntry g_noalloc_cache[kNoAllocCacheSlots] = {};
int g_noalloc_cache_next = 0;
using CuCtxGetCurrentFn = int (*)(void**);
using CuCtxGetIdFn = int (*)(void*, unsigned long long*);

bool current_context_id(unsigned long long& id) {
    static CuCtxGetCurrentFn get_current = nullptr;
    static CuCtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
            q0 != cudaDriverEntryPointSuccess || !f0)
            return false;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || !f1)
            return false;
        get_current = reinterpret_cast<CuCtxGetCurrentFn>(f0);
        get_id = reinterpret_cast<CuCtxGetIdFn>(f1);
    }
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, &id) == 0;
}
}  // namespace

}  // namespace gps

extern "C" gps_status gps_workload_scan_noalloc(const uint32_t* d_counts, const uint32_t* d_mask, uint32_t n,
                                                uint32_t max_points, uint32_t* d_surv_gid, uint32_t* d_surv_start,
                                                uint32_t* d_tile_first_rank, uint32_t* d_counters8, void* stream) {
    using namespace gps;
    const uint64_t tiles64 = ((uint64_t)n + kScanTile - 1) / kScanTile;
    if ((uint64_t)n > kNoAllocScanMaxGaussians) {
        set_last_error("gps_workload_scan_noalloc: " + std::to_string(n) + " Gaussians exceed the fixed scratch's limit of " +
                       std::to_string((unsigned long long)kNoAllocScanMaxGaussians) + " Gaussians");
        return GPS_ERR_SIZE;
    }
    const uint32_t tiles = (uint32_t)tiles64;
    if ((n && (!d_counts || !d_mask || !d_surv_gid || !d_surv_start)) || !d_tile_first_rank || !d_counters8) {
        set_last_error("gps_workload_scan_noalloc: null argument");
        return GPS_ERR_INVALID_ARGUMENT;
    }
    if ((reinterpret_cast<uintptr_t>(d_counts) & 15u) != 0 || (reinterpret_cast<uintptr_t>(d_counters8) & 3u) != 0) {
        set_last_error("gps_workload_scan_noalloc: d_counts must be 16-byte aligned, d_counters8 4-byte aligned");
        return GPS_ERR_INVALID_ARGUMENT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_last_error(std::string("gps_workload_scan_noalloc: no usable current device: ") + cudaGetErrorString(e));
        return GPS_ERR_CUDA;
    }
    // An error left pending by earlier, unrelated work is reported as such and left in place
    // for the caller's own check; it is not taken for a failure of this scan.
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("gps_workload_scan_noalloc: a CUDA error from earlier work is pending: ") +
                       cudaGetErrorString(e));
        return GPS_ERR_CUDA;
    }
    unsigned long long* scratch = nullptr;
    {
        // Once per context, with it current: the host-side name of a __device__ array is not a
        // device address, the address must be looked up.
        unsigned long long ctx_id = 0;
        const bool have_id = current_context_id(ctx_id);
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (have_id)
            for (const NoAllocScratchEntry& en : g_noalloc_cache)
                if (en.ptr && en.ctx_id == ctx_id) scratch = en.ptr;
        if (!scratch) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
            if (e != cudaSuccess) {
                set_last_error(std::string("gps_workload_scan_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
                return GPS_ERR_CUDA;
            }
            scratch = static_cast<unsigned long long*>(p);
            if (have_id) {  // without a context ID the address is looked up on every call
                g_noalloc_cache[g_noalloc_cache_next] = {ctx_id, scratch};
                g_noalloc_cache_next = (g_noalloc_cache_next + 1) % kNoAllocCacheSlots;
            }
        }
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    ScanArgs a{};
    a.counts = d_counts;
    a.mask = d_mask;
    a.n = n;
    a.max_points = max_points;
    a.tile_points = 256;
    a.surv_gid = d_surv_gid;
    a.surv_start = d_surv_start;
    a.tile_first_rank = d_tile_first_rank;
    a.tile_state = scratch;
    a.counters = reinterpret_cast<PassCounters*>(d_counters8);
    launch_scan(a, tiles, st);  // writes every tile word and all eight counters
    e = cudaGetLastError();  // nothing was pending before the launches: this is theirs
    if (e != cudaSuccess) {
        set_last_error(std::string("gps_workload_scan_noalloc: ") + cudaGetErrorString(e));
        return GPS_ERR_CUDA;
    }
    return GPS_OK;
}

// ---------------------------------------------------------------------------------
// Scene order on the device: 3D Morton order of the Gaussian means, the same order as the host
// reorder (host_scene.cpp morton_sort: keys from the scene's bounding box, 21 bits per axis,
// a stable sort), computed with round-to-nearest arithmetic so that every key is the host's.
// ---------------------------------------------------------------------------------
#include <cub/device/device_radix_sort.cuh>

namespace gps {
namespace {

__device__ __forceinline__ uint32_t ordered_bits(float f) {  // monotone float -> uint32 map
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_ordered_bits(uint32_t b) {
    return __uint_as_float((b & 0x80000000u) ? (b & 0x7FFFFFFFu) : ~b);
}

__global__ void __launch_bounds__(256) mean_bounds_kernel(const float4* __restrict__ pos, uint32_t n,
                                                          uint32_t* __restrict__ bounds6) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = __ldg(pos + i);
        const float f[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (f[c] != f[c]) continue;  // NaN never wins the host's comparisons
            const uint32_t v = ordered_bits(f[c]);
            lo[c] = min(lo[c], v);
            hi[c] = max(hi[c], v);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = min(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = max(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
        if ((threadIdx.x & 31u) == 0u) {
            atomicMin(bounds6 + c, lo[c]);
            atomicMax(bounds6 + 3 + c, hi[c]);
        }
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t v) {  // bit b -> bit 3b
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__global__ void __launch_bounds__(256) morton_keys_kernel(const float4* __restrict__ pos, uint32_t n,
                                                          const uint32_t* __restrict__ bounds6,
                                                          unsigned long long* __restrict__ keys,
                                                          uint32_t* __restrict__ index) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(pos + i);
    const float v[3] = {p.x, p.y, p.z};
    uint32_t q[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float mn = from_ordered_bits(bounds6[c]), mx = from_ordered_bits(bounds6[3 + c]);
        const float den = __fsub_rn(mx, mn), num = __fsub_rn(v[c], mn);
        const float rel = den != 0.0f ? __fdiv_rn(num, den) : 0.0f;
        q[c] = (uint32_t)__float2int_rz(__fmul_rn(rel, (float)((1 << 21) - 1)));
    }
    keys[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
    index[i] = i;
}

template <class T>
__global__ void __launch_bounds__(256) gather_kernel(const T* __restrict__ src, const uint32_t* __restrict__ order,
                                                     uint32_t n, uint32_t per, T* __restrict__ dst) {
    const uint64_t total = (uint64_t)n * per;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = j / per, k = j - i * per;
        dst[j] = __ldg(src + (uint64_t)__ldg(order + i) * per + k);
    }
}

}  // namespace

cudaError_t morton_order_device(const float4* pos, uint32_t n, uint32_t* order, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t* bounds6 = nullptr;
    unsigned long long *keys = nullptr, *keys_out = nullptr;
    uint32_t* index = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    const uint32_t init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    cudaError_t e = cudaMalloc(&bounds6, 6 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&keys, (size_t)n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&keys_out, (size_t)n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&index, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bounds6, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        mean_bounds_kernel<<<148 * 8, 256, 0, st>>>(pos, n, bounds6);
        morton_keys_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, n, bounds6, keys, index);
        e = cudaGetLastError();
    }
    // 63 key bits; the radix sort is stable, so equal keys keep their input order as the
    // host's std::stable_sort does
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_out, index, order, (int)n, 0, 63, st);
    if (e == cudaSuccess) e = cudaMalloc(&temp, temp_bytes);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_out, index, order, (int)n, 0, 63, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(temp);
    cudaFree(index);
    cudaFree(keys_out);
    cudaFree(keys);
    cudaFree(bounds6);
    return e;
}

void launch_gather_rows(const float4* src, const uint32_t* order, uint32_t n, uint32_t per, float4* dst, cudaStream_t st) {
    if (n) gather_kernel<float4><<<148 * 8, 256, 0, st>>>(src, order, n, per, dst);
}

}  // namespace gps
