/*
 * gps_b200 — C-ABI of the B200-native Gaussian point-splatting frame path.
 *
 * Drop-in boundary for the reference's render pass (PeterZs/gaussian-point-splatting):
 *   class RenderPass { virtual void render(glm::vec3* d_image, float* d_depth,
 *                                          const RenderSettings&) = 0; }
 *     src/core/rendering/render_pass.cuh:17-24, implemented by GaussianPointSplatting
 *     (src/core/rendering/passes/gaussian_point_splatting.cuh:34-71, .cu:599-816).
 * Plain pointers and sizes only; every call returns a gps_status and never traps or
 * aborts.  Device pointers are CUDA global-memory addresses on the current device; the
 * `stream` arguments are cudaStream_t values passed as void* (NULL = legacy stream).
 */
#ifndef GPS_B200_H
#define GPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPS_B200_ABI_VERSION 1

typedef enum gps_status {
    GPS_OK = 0,
    GPS_ERR_INVALID_ARGUMENT = 1,
    GPS_ERR_IO = 2,             /* file missing / unreadable / short read */
    GPS_ERR_FORMAT = 3,         /* malformed PLY header or camera JSON */
    GPS_ERR_CUDA = 4,           /* a CUDA runtime call failed */
    GPS_ERR_OUT_OF_MEMORY = 5,
    GPS_ERR_SIZE = 6,           /* request exceeds a supported size */
    GPS_ERR_DEVICE_TIMEOUT = 7  /* a bounded device-side wait gave up */
} gps_status;

/* Scene storage formats on the device. */
typedef enum gps_scene_format {
    GPS_SCENE_FP32 = 0,        /* GPUGaussianSceneUncompressed (gaussian_types.cuh:548-646) */
    GPS_SCENE_COMPRESSED = 1,  /* GPUGaussianSceneCompressed, the reference's default build
                                  (config.h:15, gaussian_types.cuh:421-541) */
    GPS_SCENE_HALF = 2         /* this library's own storage, no counterpart in the reference:
                                  positions as 16-bit fixed-point offsets from a 16-Gaussian block
                                  origin, FP16 opacity, rotation, scale and SH DC term, int8 SH
                                  AC terms on one bf16 scale per SH band; 80 bytes per Gaussian
                                  (FP32: 240), decoded to FP32, near-degenerate 2D covariances
                                  inverted in FP64.  Not bit-exact with the reference by design. */
} gps_scene_format;

typedef enum gps_accumulation {
    GPS_ACCUM_PROGRESSIVE = 0, /* AccumulationMode::ProgressiveRendering */
    GPS_ACCUM_TAA = 1,         /* AccumulationMode::TAA */
    GPS_ACCUM_NONE = 2         /* AccumulationMode::None */
} gps_accumulation;

/*
 * Render settings: the fields of RenderSettings (src/render_settings.cuh:36-103) that the
 * frame path reads, with the same defaults (gps_settings_default).
 */
typedef struct gps_settings {
    int32_t width, height;                      /* resolution (1920 x 1080) */
    int32_t supersampling_factor;               /* 2 */
    int32_t samples_per_pixel;                  /* render_pass_count, 1 */
    int32_t max_number_of_points;               /* 250000000 */
    float fovy;                                 /* degrees, 45 */
    float near_view_plane, far_view_plane;      /* 0.2, 10000 */
    int32_t enable_hierarchical_culling;        /* 1 */
    int32_t fully_disable_hierarchical_culling; /* 0 */
    int32_t enable_occlusion_culling;           /* 1 */
    int32_t occlusion_culling_min_reduce_count; /* 0 */
    int32_t cull_small_gaussians;               /* 0 */
    int32_t use_unbiased_2d_splatting;          /* 1 */
    int32_t reduce_point_count;                 /* 1: K = ss^2 points per thread; 0 = --one-point-per-thread */
    float background[3];                        /* 0,0,0 */
    int32_t accumulation_mode;                  /* gps_accumulation, progressive */
    int32_t sort_morton_order;                  /* 0 */
    /* immediate_splat_threshold: Gaussians of at most this many points are splatted inside
     * the preprocess (ENABLE_IMMEDIATE_SPLATTING, gaussian_point_splatting.cu:272-287).  The
     * reference compiles the option out by default, hence 0 = off here; its menu default,
     * when compiled in, is 8. */
    int32_t immediate_splat_threshold;          /* 0 */
    /* points_per_thread (K): not in the reference, which fixes K = ss^2 x POINTS_PER_KERNEL
     * (1 with reduce_point_count off).  > 0 overrides it: a Gaussian's Poisson count is divided
     * by K and each point draws K samples per spp pass, so the estimator is unchanged and the
     * work moves between points and samples (the batch autotuner's knob).  0 = the reference's
     * rule; renders with the same K are bit-identical to each other. */
    int32_t points_per_thread;                  /* 0 */
} gps_settings;

/* One frame's camera: what RenderSettings carries per frame (render_settings.cuh:94-105). */
typedef struct gps_camera {
    float view[16];            /* cameraViewMatrix, column-major */
    float proj[16];            /* cameraProjectionMatrix, column-major */
    float position[3];         /* cameraPosition */
    float frustum_planes[24];  /* 6 x (nx, ny, nz, d), left,right,bottom,top,near,far */
    int32_t frame;             /* settings.frame (seeds, A/B buffers) */
    int32_t camera_moved;      /* resets progressive accumulation */
} gps_camera;

/* One entry of a 3DGS cameras.json (src/utils/camera_loader.cuh:29-40). */
typedef struct gps_camera_state {
    int32_t id;
    int32_t width, height;
    float position[3];
    float rotation[9];         /* rows as stored in the JSON (camera-to-world basis rows) */
    float fx, fy;
    char img_name[64];
} gps_camera_state;

/* Per-frame statistics (render_settings.cuh:23-34) plus device-side counters. */
typedef struct gps_stats {
    int32_t num_points_one, num_points_two;         /* P of pass 1 / pass 2 */
    int32_t num_gaussians_one, num_gaussians_two;   /* Gaussians scanned per pass */
    int32_t survivors_one, survivors_two;           /* Gaussians with >= 1 point per pass */
    uint32_t total_points_one, total_points_two;    /* before the max_number_of_points clamp */
    int32_t truncated;                              /* 1 if the point budget clipped a pass */
    int32_t device_timeouts;                        /* bounded waits that gave up (0 normally) */
    int32_t kernel_launches;                        /* kernels the last frame launched */
    int32_t gaussians_read_one, gaussians_read_two; /* Gaussians whose attributes the preprocess
                                                       read per pass (after the block cull and
                                                       pass 2's previous-mask test) */
    int32_t screen_order_one, screen_order_two;     /* 1 if the pass's splat walked its survivors
                                                       in screen-bin order, 0 in Gaussian order
                                                       (a splat buffer under 64 MB, a
                                                       budget-truncated pass, or a bin crowded
                                                       past 131,072 survivors; the environment
                                                       variable GPS_BIN_CROWDED, read when a
                                                       renderer is created, overrides that
                                                       count).  The order changes no output. */
} gps_stats;

typedef struct gps_scene gps_scene;
typedef struct gps_renderer gps_renderer;
typedef struct gps_camera_path gps_camera_path;

/* ---- version / errors -------------------------------------------------------------- */
int32_t gps_abi_version(void);
/* Last error message of the calling thread ("" if none). */
const char* gps_last_error(void);

/* ---- settings (render_settings.cuh:36-103, parse_args.cuh:21-127) ------------------- */
void gps_settings_default(gps_settings* s);
/* Parses the reference's CLI flags (--resolution W H, --supersampling-factor, ...).
 * model_path/camera_path receive --model-path / --camera-path (may be NULL). */
gps_status gps_settings_parse_args(int32_t argc, const char* const* argv, gps_settings* s,
                                   char* model_path, size_t model_path_cap,
                                   char* camera_path, size_t camera_path_cap);

/* ---- scenes (gaussian_loader.cu:282-427, gaussian_types.cuh:442-503,568-608) ---------
 * gps_scene_load_ply accepts a .ply file or a 3DGS output directory
 * (point_cloud/<alphabetically last>/point_cloud.ply, render_settings.cuh:137-227).
 * presorted_out (may be NULL) receives 1 if the file carries the bvh_sorted_order comment. */
gps_status gps_scene_load_ply(const char* path, int32_t format, int32_t sort_morton_order,
                              gps_scene** out, int32_t* presorted_out);
/* Builds a scene from host Gaussians in the reference's CPUGaussian layout
 * (gaussian_types.cuh:89-100): 59 floats each = mean[3], sh[48], opacity (activated),
 * scale[3] (activated), rotation[4] (normalised, rot_0..rot_3). */
gps_status gps_scene_from_host(const float* gaussians, uint64_t count, int32_t format,
                               int32_t presorted, gps_scene** out);
/* gps_scene_from_host after the --sort-morton-order reorder (gaussian_loader.cu:363-424):
 * sort_morton_order 0 keeps the given order, 1 reorders on the host, 2 on the device (keys,
 * stable radix sort and gather in HBM).  1 and 2 give the identical order.  The same values
 * select the reorder in gps_scene_load_ply, where a file carrying the bvh_sorted_order
 * comment keeps its order. */
gps_status gps_scene_from_host_sorted(const float* gaussians, uint64_t count, int32_t format,
                                      int32_t sort_morton_order, gps_scene** out);
/* The reorder's permutation: order[j] = the input index of the j-th Gaussian in 3D Morton
 * order of the means (21 bits per axis over the means' bounding box, ties in input order);
 * computed on the host (on_device = 0) or on the device. */
gps_status gps_morton_order(const float* gaussians, uint64_t count, int32_t on_device, uint32_t* order);
/* A new GPS_SCENE_HALF scene holding `copies` translated copies of a GPS_SCENE_HALF scene (copy
 * k moved by (offsets_xz[2k], 0, offsets_xz[2k+1])), built on the device; the culling blocks
 * follow the reference's size rule for the new count (like GaussianEditor::Repeat,
 * src/core/gaussians/editor/gaussian_editor.cu:37-65, followed by build_fixed_blocks). */
gps_status gps_scene_tile(const gps_scene* src, int32_t copies, const float* offsets_xz, gps_scene** out);
uint64_t gps_scene_count(const gps_scene* scene);
int32_t gps_scene_format_of(const gps_scene* scene);
void gps_scene_free(gps_scene* scene);
/* Writes host Gaussians (CPUGaussian layout) as a 3DGS binary PLY with normals
 * (gaussian_loader.cu:480-562); comments are '\n'-separated (may be NULL). */
gps_status gps_ply_write(const char* path, const float* gaussians, uint64_t count, const char* comments);
/* Reads a PLY into host memory in CPUGaussian layout (count first with out = NULL). */
gps_status gps_ply_read(const char* path, float* out, uint64_t capacity, uint64_t* count, int32_t* presorted);

/* ---- renderer = GaussianPointSplatting (gaussian_point_splatting.cu:599-816) -------- */
gps_status gps_renderer_create(gps_scene* scene, const gps_settings* settings, gps_renderer** out);
void gps_renderer_free(gps_renderer* r);
/* RenderPass::render: writes the W x H float3 image and float NDC depth (caller-owned
 * device buffers).  No host synchronisation and no allocation inside. */
gps_status gps_render_frame(gps_renderer* r, const gps_camera* cam, float* d_image_rgb, float* d_depth,
                            void* stream);
/* Forgets the previous frame (its Hi-Z depth chain): the next gps_render_frame renders as the
 * first frame of a newly created renderer would, e.g. after a camera cut.  Asynchronous on
 * `stream`. */
gps_status gps_renderer_reset(gps_renderer* r, void* stream);
/* Statistics of the last frame; waits for that frame's work on its stream. */
gps_status gps_renderer_stats(gps_renderer* r, gps_stats* out);
/* Per-stage GPU timing with CUDA events on the frame's stream (off by default).  Stages:
 * 0 clear, 1 block cull, 2 preprocess, 3 scan, 4 splat, 5 resolve, 6 Hi-Z, 7 post-process;
 * out_ms[8] receives the accumulated milliseconds, out_launches[8] (may be NULL) the kernel
 * launches per stage, since enabling or the last reset. */
gps_status gps_renderer_enable_timing(gps_renderer* r, int32_t enable);
gps_status gps_renderer_stage_times(gps_renderer* r, float* out_ms, uint64_t* out_launches, int32_t reset);
/* The current 64-bit splat buffer (depth28 << 36 | rgb36, Morton 64x64 tiles, spp innermost). */
gps_status gps_renderer_splat_buffer(gps_renderer* r, const uint64_t** d_buffer, uint64_t* entries);
/* Per-frame constants the renderer derived from the camera (gaussian_point_splatting.cu:605-615):
 * out[0:16] view-projection, out[16:32] camera-to-world, out[32:34] tan_fov, out[34:36] focal. */
gps_status gps_renderer_derived(gps_renderer* r, const gps_camera* cam, float* out36);
/* Device views of the last pass's workload for parity checks: counts[N] (valid where the
 * mask bit is set), mask words of the last two passes, survivors' Gaussian ids and first
 * points, the Hi-Z chain, per-Gaussian colours (float3 inside 64-byte records), block mask. */
typedef struct gps_debug_view {
    const uint32_t* counts;
    const uint32_t* mask_last;
    const uint32_t* mask_other;
    const uint32_t* surv_gid;
    const uint32_t* surv_start;
    uint32_t survivors;
    uint32_t points;
    const float* records;       /* 16 floats per Gaussian */
    const float* hiz;
    uint64_t hiz_size;
    const uint32_t* block_culled;
    uint32_t block_words;
    const float* block_nodes;   /* 8 floats per node: min.xyz, begin bits, max.xyz, count bits */
    uint32_t block_count;
    uint32_t per_block;
} gps_debug_view;
gps_status gps_renderer_debug_view(gps_renderer* r, gps_debug_view* out);

/* ---- measured peaks -------------------------------------------------------------------
 * No counterpart in the reference: the rate of 64-bit atomicMin on random addresses of a
 * caller-owned device buffer of `entries` words (< 2^32; overwritten), best of `repeats`
 * timed launches on `stream` (blocking).  The splat's unit of work is one such operation per
 * live sample, so this is the roofline its achieved rate is compared with. */
gps_status gps_measure_atomic_min_rate(uint64_t* d_buf, uint64_t entries, int32_t repeats, double* atomics_per_second,
                                       void* stream);

/* ---- allocation-free point scan ------------------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that cannot allocate
 * device memory when they run the scan — inside a CUDA-graph capture or a stream-ordered
 * pipeline where cudaMalloc would synchronise, under a host that enforces its own fixed
 * device-memory budget, or as a plugin whose host owns every buffer.  It computes one render
 * pass's workload (what gps_render_frame computes internally, the reference's
 * WorkloadDistributor::build): the exclusive point offsets of the Gaussians whose mask bit is
 * set, compacted.  It allocates nothing: its scratch (the per-tile totals of the scan) is a fixed 512 KiB device array
 * inside the library, so n is limited to 268,435,456 Gaussians (larger n: GPS_ERR_SIZE).
 *   d_counts            n point counts (only entries whose mask bit is set are used); 16-byte
 *                       aligned and readable up to n rounded up to a multiple of 4
 *   d_mask              ceil(n / 32) mask words (bit i of word w = Gaussian 32*w + i)
 *   d_surv_gid/start    outputs, n entries each: the Gaussian id and first point of every
 *                       Gaussian with its bit set, in Gaussian order
 *   d_tile_first_rank   output, max_points / 256 + 2 entries: first survivor of each 256-point tile
 *   d_counters8         output, 8 words: survivors, total points (mod 2^32),
 *                       points = min(total, max_points), truncated flag, 0, 0, 0, 0
 * The first call in a CUDA context (the device's primary context, or a driver-API context
 * made current by the caller) looks the scratch array's address up in that context and keeps
 * it, keyed on the context's unique ID; make that first call before any stream capture.  A
 * context re-created after cudaDeviceReset is a new context and gets its own lookup.  An
 * error already pending from earlier work is reported (GPS_ERR_CUDA) and left pending.  All
 * calls in a context share the array; each call writes every word of it that it reads before
 * reading it, and calls that overlap on the GPU race on it — serialise them (one stream at a
 * time). */
gps_status gps_workload_scan_noalloc(const uint32_t* d_counts, const uint32_t* d_mask, uint32_t n,
                                     uint32_t max_points, uint32_t* d_surv_gid, uint32_t* d_surv_start,
                                     uint32_t* d_tile_first_rank, uint32_t* d_counters8, void* stream);

/* ---- batched multi-view rendering ----------------------------------------------------
 * Many views of one scene per call, each with its own camera, resolution and samples per
 * pixel, written to caller-owned device buffers.  Each view is rendered as the first frame of
 * a fresh gps_render_frame renderer would render it (no temporal Hi-Z reuse), so its image and
 * depth are bit-identical to that plain render.  Views run on `workers` internal streams that
 * fork from and join back into `stream`, so views too small to fill the GPU overlap.  Workers
 * hold per-Gaussian scratch sized for the scene and a splat buffer sized for the largest view
 * (max_width x max_height at max_spp); views beyond that capacity return GPS_ERR_SIZE.  The
 * other fields of `settings` (supersampling, culling, K mode, planes, fovy, background) apply to
 * every view. */
typedef struct gps_view {
    gps_camera camera;
    int32_t width, height;       /* output resolution of this view */
    int32_t samples_per_pixel;
    float* d_image;              /* width * height float3 (device) */
    float* d_depth;              /* width * height float NDC depth (device) */
} gps_view;
typedef struct gps_batch gps_batch;
gps_status gps_batch_create(gps_scene* scene, const gps_settings* settings, int32_t max_width, int32_t max_height,
                            int32_t max_spp, int32_t workers, gps_batch** out);
void gps_batch_free(gps_batch* b);
/* Enqueues every view; returns without waiting for the GPU. */
gps_status gps_batch_render(gps_batch* b, const gps_view* views, int32_t count, void* stream);
/* Number of workers used by gps_batch_render (1 .. the number created). */
gps_status gps_batch_set_workers(gps_batch* b, int32_t workers);
int32_t gps_batch_workers(const gps_batch* b);
/* Points per thread K of every view (gps_settings.points_per_thread; 0 = the reference's rule).
 * Each view stays bit-identical to a plain render with the same K. */
gps_status gps_batch_set_points_per_thread(gps_batch* b, int32_t k);
/* enable != 0: gps_batch_render replays the batch from a CUDA graph: the fork/join launch
 * sequence is captured on a private stream, and a batch whose layout (view sizes, samples,
 * worker assignment, K) matches the previous one updates the executable graph's parameters
 * (the cameras) with cudaGraphExecUpdate instead of instantiating it again; the graph is
 * launched on the caller's stream.  Results are identical to the direct launches. */
gps_status gps_batch_use_graph(gps_batch* b, int32_t enable);
gps_status gps_batch_graph_stats(const gps_batch* b, int64_t* instantiations, int64_t* updates);
/* The autotuner over K in {1, 2, 4, 8} and, for each, the worker count (gps_batch_autotune);
 * leaves the batch at the fastest pair. */
gps_status gps_batch_autotune_k(gps_batch* b, const gps_view* views, int32_t count, int32_t rounds, void* stream,
                                int32_t* chosen_workers, int32_t* chosen_k, float* ms);
/* Autotuner: times `rounds` renders of the batch for each worker count 1, 2, 4, ... up to the
 * number created (CUDA events on `stream`), keeps the fastest and returns it in *chosen and its
 * time per batch in *ms (either may be NULL).  Synchronises `stream`. */
gps_status gps_batch_autotune(gps_batch* b, const gps_view* views, int32_t count, int32_t rounds, void* stream,
                              int32_t* chosen, float* ms);

/* ---- serving: a request loop over resident scenes -------------------------------------
 * Render requests (scene, camera, resolution, spp) are submitted from any host thread and
 * queued; a dispatcher thread of the server admits them, first come first served, onto
 * `workers` GPU workers (each with its own stream, per-Gaussian scratch for the largest
 * scene and a splat buffer for the largest view) as soon as a worker is free, so requests
 * that arrive while others are on the GPU start as slots free up and their work overlaps on
 * the device.  A request larger than the workers' capacity completes with GPS_ERR_SIZE.  Each
 * request is rendered as a fresh renderer's first frame (like gps_batch_render), so its result
 * does not depend on what else is in flight.  The device current at gps_server_create is used. */
typedef struct gps_request {
    uint64_t id;                 /* caller's tag, returned in the completion */
    int32_t scene;               /* index into the scenes passed to gps_server_create */
    gps_camera camera;
    int32_t width, height, samples_per_pixel;
    float* d_image;              /* width * height float3, or NULL to render into the worker's buffer */
    float* d_depth;              /* width * height float, or NULL */
} gps_request;
typedef struct gps_completion {
    uint64_t id;
    int32_t status;              /* gps_status of this request */
    int32_t worker;
    double queued_ms;            /* submit -> admitted to a worker */
    double latency_ms;           /* submit -> its GPU work seen finished */
} gps_completion;
typedef struct gps_server gps_server;
gps_status gps_server_create(gps_scene* const* scenes, int32_t n_scenes, const gps_settings* settings,
                             int32_t max_width, int32_t max_height, int32_t max_spp, int32_t workers,
                             gps_server** out);
/* Admission budget: a request joins the requests in flight only while their splat buffers
 * together hold at most `max_inflight_entries` entries (W*ss x H*ss x spp, rounded up to 64x64
 * tiles); a request above the budget runs alone.  Large views saturate the GPU by themselves
 * and only slow each other down when overlapped, small ones fill it together.  0 = no limit.
 * Default: 67,108,864 entries (two 1920x1080 views at ss 2 and 4 spp). */
gps_status gps_server_set_admission(gps_server* s, uint64_t max_inflight_entries);
/* Queues one request; thread-safe and never waits for the GPU. */
gps_status gps_server_submit(gps_server* s, const gps_request* req);
/* Moves up to `capacity` completions (oldest first) to `out`; returns how many. */
int32_t gps_server_poll(gps_server* s, gps_completion* out, int32_t capacity);
/* Waits until every submitted request has completed (GPS_ERR_DEVICE_TIMEOUT after timeout_s). */
gps_status gps_server_drain(gps_server* s, double timeout_s);
/* Drains, stops the dispatcher and frees the workers (the scenes stay the caller's). */
void gps_server_free(gps_server* s);

/* ---- RenderServer post-process (render_server.cu:122-157) ---------------------------- */
/* temporalRender (post_processing_kernels.cuh:222-285): reprojects history through reproj
 * (column-major), clamps it to the 3x3 neighbourhood of the current colour +-0.05, blends,
 * writes the blended colour to d_out_color and u8 RGB to d_image_u8.  The reference blends in
 * place, which races with the neighbourhood reads of adjacent threads; d_out_color must be a
 * different buffer from d_cur_color, which makes the result deterministic. */
gps_status gps_post_taa(uint8_t* d_image_u8, float* d_out_color, const float* d_cur_color,
                        const float* d_prev_color, const float* d_cur_depth, const float* d_prev_depth,
                        const float* reproj16, float blend, int32_t width, int32_t height,
                        int32_t frame_number, void* stream);
/* progressiveRender: cur += accum (frames > 1), accum = 0, u8 = round(clamp(cur*255/frames)). */
gps_status gps_post_progressive(uint8_t* d_image_u8, float* d_cur_color, float* d_accum, int32_t width,
                                int32_t height, int32_t frames, void* stream);

/* ---- headless frame loop = RenderServer::renderFrame without GL -------------------- */
/* Owns the colour/depth ping-pong buffers and the u8 output; reproduces the reference's
 * buffer rotation (including its depth-slot order) and accumulation counter. */
typedef struct gps_frame_loop gps_frame_loop;
gps_status gps_frame_loop_create(gps_renderer* r, gps_frame_loop** out);
void gps_frame_loop_free(gps_frame_loop* l);
/* Renders one frame and post-processes it; d_image_u8 may be NULL (internal buffer). */
gps_status gps_frame_loop_step(gps_frame_loop* l, const gps_camera* cam, void* stream);
/* Copies the last u8 RGB frame (W*H*3 bytes) to host memory. */
gps_status gps_frame_loop_read(gps_frame_loop* l, uint8_t* host_rgb, void* stream);
/* The same copy without waiting: it runs on the loop's own copy stream once the last frame on
 * `stream` is done, while the next frames render (u8 frames alternate between two buffers; a
 * step waits only if it would overwrite a frame still being copied).  host_rgb should be pinned
 * and must stay untouched until gps_frame_loop_read_wait returns. */
gps_status gps_frame_loop_read_async(gps_frame_loop* l, uint8_t* host_rgb, void* stream);
/* Waits for every copy started by gps_frame_loop_read_async. */
gps_status gps_frame_loop_read_wait(gps_frame_loop* l);
/* Device buffers of ping-pong slot `slot` (0 or 1): frame f renders its colour into slot
 * f % 2 and its depth into slot 1 - f % 2 (render_server.cu:87-92).  Slot 2 (TAA mode):
 * the last frame's resolved colour before TAA blended it (no depth). */
gps_status gps_frame_loop_buffers(gps_frame_loop* l, int32_t slot, const uint8_t** d_u8, const float** d_color,
                                  const float** d_depth);

/* ---- evaluation workflow (main.cu:72-120, render_server.cu:162-315) ----------------- */
/* 8-bit RGB PNG (stbi_write_png in save_image_to_disk); flip_rows != 0 writes the last row
 * first, as save_image_to_disk does with the frame it reads back. */
gps_status gps_write_png(const char* path, const uint8_t* host_rgb, int32_t width, int32_t height, int32_t flip_rows);
/* write_pfm: "PF\n<w> <h>\n-1.0\n", then the W*H*3 floats in memory order. */
gps_status gps_write_pfm(const char* path, const float* host_rgb, int32_t width, int32_t height);
/* export_pfm_from_buffer: the colour buffer the last step resolved into, divided by the
 * accumulated frame count (the running mean in progressive mode), as a PFM file. */
gps_status gps_frame_loop_export_pfm(gps_frame_loop* l, const char* path, void* stream);
/* The --create-evaluation-screenshots run without the viewer: for each camera of the path
 * (0 .. min(count - 1, max_eval_count), the reference's stopping rule), progressive frames
 * restart at 1 (camera_moved), and after frame t of each spp target t the u8 frame is written
 * to <out_dir>/<img_name>_spp%04d.png (rows flipped, as the reference saves them; "cam<i>"
 * when the camera has no name), plus a .pfm of the running mean when write_pfm != 0.
 * spp_targets NULL = {1, 4, 16, 64, 256, 1024}; targets must increase.  Frame numbers
 * (seeds, ping-pong slots) run on from first_frame across cameras.  Renders on the default
 * stream and returns when the files are written. */
gps_status gps_evaluate(gps_frame_loop* l, const gps_camera_path* path, const char* out_dir,
                        const int32_t* spp_targets, int32_t num_targets, int32_t max_eval_count,
                        int32_t first_frame, int32_t write_pfm, int32_t* frames_rendered);

/* ---- cameras (camera_loader.cu:62-150, main.cu:141-157, camera.cpp:88-156) ---------- */
gps_status gps_camera_path_load(const char* json_path, gps_camera_path** out);
int32_t gps_camera_path_count(const gps_camera_path* p);
gps_status gps_camera_path_get(const gps_camera_path* p, int32_t index, gps_camera_state* out);
void gps_camera_path_free(gps_camera_path* p);
/* Applies fromCameraState's resolution/fovy override rules to *settings (when
 * override_camera_settings == 0) and fills *cam with view, projection, planes, position. */
gps_status gps_camera_from_state(const gps_camera_state* state, gps_settings* settings,
                                 int32_t override_camera_settings, int32_t* can_override_resolution,
                                 int32_t frame, gps_camera* cam);
/* Builds view/projection/planes from a camera position and camera-to-world basis
 * (columns right, up, back), as the viewer does each frame (main.cu:141-157). */
gps_status gps_camera_from_pose(const float position[3], const float basis_cols[9],
                                const gps_settings* settings, int32_t frame, gps_camera* cam);

#ifdef __cplusplus
}
#endif
#endif /* GPS_B200_H */
