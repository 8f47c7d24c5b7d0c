// Frame driver and C-ABI of the B200-native Gaussian point-splatting path.
//
// gps_render_frame reproduces GaussianPointSplatting::render
// (src/core/rendering/passes/gaussian_point_splatting.cu:599-737): clear, pass 1 (block
// cull -> preprocess -> scan -> splat), optionally depth-only resolve -> Hi-Z -> pass 2 over
// the Gaussians that did not splat in pass 1, final resolve, Hi-Z for the next frame.
// Unlike the reference it performs no host synchronisation and no allocation per frame:
// the point count P stays on the device (the splat kernel reads it), so the whole frame is
// a fixed sequence of asynchronous launches on the caller's stream.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <deque>
#include <condition_variable>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/gps_b200.h"
#include "frame_kernels.h"
#include "host_images.hpp"
#include "host_io.hpp"

using namespace gps;

namespace {

struct CudaError : std::exception {
    std::string msg;
    explicit CudaError(std::string m) : msg(std::move(m)) {}
    const char* what() const noexcept override { return msg.c_str(); }
};

#define GPS_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
T* dev_alloc(size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) + " bytes: " + cudaGetErrorString(e));
    }
    return static_cast<T*>(p);
}

struct DevFree {
    void operator()(void* p) const {
        if (p) cudaFree(p);
    }
};
template <class T>
using dptr = std::unique_ptr<T, DevFree>;

gps_status fail(gps_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

mat4 mat4_from(const float* m) {
    mat4 r;
    for (int c = 0; c < 4; ++c) r.c[c] = make_v4(m[4 * c], m[4 * c + 1], m[4 * c + 2], m[4 * c + 3]);
    return r;
}
void mat4_to(const mat4& m, float* out) {
    for (int c = 0; c < 4; ++c) {
        out[4 * c] = m.c[c].x;
        out[4 * c + 1] = m.c[c].y;
        out[4 * c + 2] = m.c[c].z;
        out[4 * c + 3] = m.c[c].w;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------
// scene
// ---------------------------------------------------------------------------------
struct gps_scene {
    int format = GPS_SCENE_FP32;
    uint64_t n = 0;
    bool presorted = false;
    // FP32 arrays (FP32 format)
    dptr<float4> pos_op, rot, scale, sh;
    // compressed arrays
    dptr<uint4> geom, sh_ac;
    dptr<uint8_t> opac;
    dptr<float4> sh_dc;
    // half-precision arrays
    dptr<uint4> h_rec, h_scl, h_ac;
    dptr<float4> h_origin;
    SceneBounds bounds{};
    // fixed-size blocks for the hierarchical cull (computed from the FP32 values, like
    // build_fixed_blocks on the host CPUGaussian array)
    dptr<float4> block_nodes;
    uint32_t per_block = 4;
    uint32_t block_count = 0;
};

namespace {

void check_order(cudaError_t e) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw CudaError(std::string("cudaMalloc in the device Morton reorder: ") + cudaGetErrorString(e));
    }
    if (e != cudaSuccess) throw CudaError(std::string("device Morton reorder: ") + cudaGetErrorString(e));
}

// The Morton order of host Gaussians computed on the device (only the means travel).
void device_morton_order(const CpuGaussian* g, uint64_t n, uint32_t* order_host) {
    if (n == 0) return;
    std::vector<float4> pos(n);
    for (uint64_t i = 0; i < n; ++i) pos[i] = make_float4(g[i].mean[0], g[i].mean[1], g[i].mean[2], 0.0f);
    dptr<float4> d_pos(dev_alloc<float4>(n));
    dptr<uint32_t> d_order(dev_alloc<uint32_t>(n));
    GPS_CUDA(cudaMemcpy(d_pos.get(), pos.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    check_order(morton_order_device(d_pos.get(), (uint32_t)n, d_order.get(), 0));
    GPS_CUDA(cudaMemcpy(order_host, d_order.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
}

// device_sort: put the uploaded Gaussians in Morton order on the device (FP32 and HALF
// scenes; the same order as morton_sort on the host).
void scene_upload(gps_scene* s, const CpuGaussian* g, uint64_t n, bool device_sort) {
    s->n = n;
    s->per_block = gaussians_per_block(n);
    s->block_count = (uint32_t)((n + s->per_block - 1) / s->per_block);
    // repack into 16-byte SoA in chunks through two pinned staging halves: a chunk is repacked on
    // every host core while the previous one is copied
    const uint64_t chunk = 1u << 19;
    float4* stage = nullptr;
    GPS_CUDA(cudaMallocHost(&stage, 2 * chunk * sizeof(float4) * 15));
    std::unique_ptr<float4, void (*)(float4*)> stage_guard(stage, [](float4* p) { cudaFreeHost(p); });
    cudaStream_t cs = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    GPS_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    struct CopyState {
        cudaStream_t s;
        cudaEvent_t* e;
        ~CopyState() {
            if (s) cudaStreamSynchronize(s);
            for (int i = 0; i < 2; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
            if (s) cudaStreamDestroy(s);
        }
    } copy_state{cs, ev};
    for (int i = 0; i < 2; ++i) GPS_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    float4* d_pos = dev_alloc<float4>(n);
    s->pos_op.reset(d_pos);
    float4* d_rot = dev_alloc<float4>(n);
    s->rot.reset(d_rot);
    float4* d_scale = dev_alloc<float4>(n);
    s->scale.reset(d_scale);
    float4* d_sh = nullptr;
    if (s->format == GPS_SCENE_FP32 || s->format == GPS_SCENE_HALF) {
        d_sh = dev_alloc<float4>(n * 12);
        s->sh.reset(d_sh);
    }
    uint64_t k = 0;
    for (uint64_t b = 0; b < n; b += chunk, ++k) {
        const uint64_t e = std::min(n, b + chunk), m = e - b;
        float4* buf = stage + (k & 1) * chunk * 15;
        if (k >= 2) GPS_CUDA(cudaEventSynchronize(ev[k & 1]));  // its previous copy is done
        float4* sp = buf;
        float4* sr = buf + chunk;
        float4* ss = buf + 2 * chunk;
        float4* sh = buf + 3 * chunk;
        const bool with_sh = d_sh != nullptr;
        parallel_ranges(m, [&](uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; ++i) {
                const CpuGaussian& q = g[b + i];
                sp[i] = make_float4(q.mean[0], q.mean[1], q.mean[2], q.opacity);
                sr[i] = make_float4(q.rot[0], q.rot[1], q.rot[2], q.rot[3]);
                ss[i] = make_float4(q.scale[0], q.scale[1], q.scale[2], 0.0f);
                if (with_sh) std::memcpy(sh + i * 12, q.sh, sizeof(float) * 48);
            }
        });
        GPS_CUDA(cudaMemcpyAsync(d_pos + b, sp, m * sizeof(float4), cudaMemcpyHostToDevice, cs));
        GPS_CUDA(cudaMemcpyAsync(d_rot + b, sr, m * sizeof(float4), cudaMemcpyHostToDevice, cs));
        GPS_CUDA(cudaMemcpyAsync(d_scale + b, ss, m * sizeof(float4), cudaMemcpyHostToDevice, cs));
        if (d_sh) GPS_CUDA(cudaMemcpyAsync(d_sh + b * 12, sh, m * 12 * sizeof(float4), cudaMemcpyHostToDevice, cs));
        GPS_CUDA(cudaEventRecord(ev[k & 1], cs));
    }
    GPS_CUDA(cudaStreamSynchronize(cs));
    if (device_sort && n > 1) {
        dptr<uint32_t> order(dev_alloc<uint32_t>(n));
        check_order(morton_order_device(d_pos, (uint32_t)n, order.get(), 0));
        auto regather = [&](dptr<float4>& arr, uint32_t per) {
            float4* dst = dev_alloc<float4>(n * per);
            launch_gather_rows(arr.get(), order.get(), (uint32_t)n, per, dst, 0);
            GPS_CUDA(cudaGetLastError());
            GPS_CUDA(cudaDeviceSynchronize());
            arr.reset(dst);
        };
        regather(s->pos_op, 1);
        regather(s->rot, 1);
        regather(s->scale, 1);
        if (d_sh) regather(s->sh, 12);
        d_pos = s->pos_op.get();
        d_rot = s->rot.get();
        d_scale = s->scale.get();
        d_sh = s->sh.get();
    }
    float4* nodes = dev_alloc<float4>((size_t)s->block_count * 2);
    s->block_nodes.reset(nodes);
    launch_block_bounds(d_pos, d_rot, d_scale, (uint32_t)n, s->per_block, nodes, 0);
    GPS_CUDA(cudaGetLastError());
    if (s->format == GPS_SCENE_HALF) {
        s->h_rec.reset(dev_alloc<uint4>(n));
        s->h_scl.reset(dev_alloc<uint4>(n));
        s->h_ac.reset(dev_alloc<uint4>(n * 3));
        s->h_origin.reset(dev_alloc<float4>((n + kHalfOriginBlock - 1) / kHalfOriginBlock));
        launch_encode_half(d_pos, d_rot, d_scale, d_sh, (uint32_t)n, s->h_origin.get(), s->h_rec.get(), s->h_scl.get(),
                           s->h_ac.get(), 0);
        GPS_CUDA(cudaGetLastError());
        GPS_CUDA(cudaDeviceSynchronize());
        s->pos_op.reset();
        s->rot.reset();
        s->scale.reset();
        s->sh.reset();
    }
    if (s->format == GPS_SCENE_COMPRESSED) {
        s->bounds = compute_scene_bounds(g, n);
        std::vector<uint4> geom(n), ac(n * 3);
        std::vector<uint8_t> op(n);
        std::vector<float4> dc(n);
        encode_compressed(g, n, s->bounds, geom.data(), op.data(), dc.data(), ac.data());
        s->geom.reset(dev_alloc<uint4>(n));
        s->sh_ac.reset(dev_alloc<uint4>(n * 3));
        s->opac.reset(dev_alloc<uint8_t>(n));
        s->sh_dc.reset(dev_alloc<float4>(n));
        GPS_CUDA(cudaMemcpy(s->geom.get(), geom.data(), n * sizeof(uint4), cudaMemcpyHostToDevice));
        GPS_CUDA(cudaMemcpy(s->sh_ac.get(), ac.data(), n * 3 * sizeof(uint4), cudaMemcpyHostToDevice));
        GPS_CUDA(cudaMemcpy(s->opac.get(), op.data(), n, cudaMemcpyHostToDevice));
        GPS_CUDA(cudaMemcpy(s->sh_dc.get(), dc.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
        GPS_CUDA(cudaDeviceSynchronize());
        // the compressed renderer needs no FP32 geometry once the blocks exist
        s->pos_op.reset();
        s->rot.reset();
        s->scale.reset();
    }
    GPS_CUDA(cudaDeviceSynchronize());
}

}  // namespace

// ---------------------------------------------------------------------------------
// renderer
// ---------------------------------------------------------------------------------
// Optional per-stage timing: CUDA events recorded between the stages of each frame on the
// frame's own stream; intervals are accumulated when read (or when the event pool fills).
enum Stage { kStClear, kStCull, kStPreprocess, kStScan, kStSplat, kStResolve, kStHiz, kStPost, kStCount };

struct StageTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<int> stage;  // stage that starts at event i (-1: frame end)
    size_t used = 0;
    double total_ms[kStCount] = {0};
    uint64_t launches[kStCount] = {0};
    int frames = 0;
    ~StageTimer() {
        for (auto e : pool) cudaEventDestroy(e);
    }
    void drain() {
        if (used == 0) return;
        cudaEventSynchronize(pool[used - 1]);
        for (size_t i = 0; i + 1 < used; ++i) {
            if (stage[i] < 0) continue;
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, pool[i], pool[i + 1]) == cudaSuccess) total_ms[stage[i]] += ms;
        }
        used = 0;
    }
    void mark(int st, cudaStream_t s) {
        if (!on) return;
        if (used == pool.size()) {
            // keep the last event as the start of the next interval
            cudaEvent_t last = pool[used - 1];
            int last_stage = stage[used - 1];
            drain();
            std::swap(pool[0], pool[pool.size() - 1]);
            (void)last;
            stage[0] = last_stage;
            used = 1;
        }
        stage[used] = st;
        cudaEventRecord(pool[used], s);
        ++used;
    }
};

struct gps_renderer {
    StageTimer timer;
    uint64_t frame_launches = 0;  // kernels launched by the last frame
    gps_scene* scene = nullptr;
    gps_settings s{};
    int up_w = 0, up_h = 0;
    uint64_t entries = 0;
    uint32_t n = 0, n_pad = 0;
    dptr<uint64_t> buffer;
    dptr<uint32_t> counts, mask[2], surv_gid, surv_start, tile_first_rank, culled, chunk_list, chunk_count, loaded;
    dptr<SplatRecord> records;
    dptr<unsigned long long> tile_state;
    dptr<unsigned long long> bins;  // screen-bin histogram / cursors, kMaxBins + 1 words
    dptr<uint32_t> sorted_gid, sorted_pstart, sorted_qstart;  // survivors in screen-bin order
    uint32_t bin_crowded = kBinCrowded;  // see kBinCrowded
    dptr<PassCounters> counters;  // [2]: pass 1, pass 2
    dptr<float> mip;
    dptr<unsigned> hiz_done;
    HizView hiz{};
    uint32_t scan_tiles = 0;
    uint64_t cap_entries = 0;     // splat-buffer and Hi-Z capacity (a batch worker renders
    uint64_t cap_mip = 0;         // views of different sizes within these)
    uint32_t cap_n = 0;           // per-Gaussian scratch capacity (a server worker renders any
    uint32_t cap_blocks = 0;      // resident scene up to these sizes)
    dptr<uint32_t> mask_iter;     // device pass counter selecting the survivor mask pair
    int splat_grid = 0;
    PassCounters* host_counters = nullptr;  // pinned [2]
    cudaEvent_t done = nullptr;
    bool have_frame = false;
    bool second_pass_last = false;
    ~gps_renderer() {
        if (host_counters) cudaFreeHost(host_counters);
        if (done) cudaEventDestroy(done);
    }
};

namespace {

void hiz_layout(HizView& h, int w, int hgt) {
    h.width = w;
    h.height = hgt;
    int max_dim = std::max(w, hgt), e = 0;
    while ((1 << e) < max_dim) ++e;
    h.levels = e + 1;
    uint64_t off = 0;
    for (int l = 0; l < h.levels; ++l) {
        int fe = h.levels - 1;
        h.level_w[l] = std::max(1, (w + (1 << (fe - l)) - 1) >> (fe - l));
        h.level_h[l] = std::max(1, (hgt + (1 << (fe - l)) - 1) >> (fe - l));
        h.level_off[l] = off;
        off += (uint64_t)h.level_w[l] * (uint64_t)h.level_h[l];
    }
    h.mip_size = off;
}

__global__ void fill_f32(float* p, uint64_t n, float v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) p[i] = v;
}

FrameConst make_frame_const(const gps_renderer* r, const gps_camera* cam) {
    FrameConst fc{};
    mat4 view = mat4_from(cam->view), proj = mat4_from(cam->proj);
    mat4 vp, cm;
    vec2 tan_fov, focal;
    derive_frame(view, proj, r->s.width, r->s.height, r->s.supersampling_factor, r->s.fovy, vp, cm, tan_fov, focal);
    fc.vp = vp;
    fc.view = view;
    fc.cam = cm;
    fc.tan_fov = tan_fov;
    fc.focal = focal;
    fc.up_width = r->up_w;
    fc.up_height = r->up_h;
    fc.num_passes = r->s.samples_per_pixel;
    fc.ss = r->s.supersampling_factor;
    fc.k_points = !r->s.reduce_point_count ? 1
                  : r->s.points_per_thread > 0 ? r->s.points_per_thread : fc.ss * fc.ss * kPointsPerKernel;
    fc.near_plane = r->s.near_view_plane;
    fc.far_plane = r->s.far_view_plane;
    for (int i = 0; i < 6; ++i)
        fc.planes[i] = make_v4(cam->frustum_planes[4 * i], cam->frustum_planes[4 * i + 1], cam->frustum_planes[4 * i + 2],
                               cam->frustum_planes[4 * i + 3]);
    fc.use_unbiased = r->s.use_unbiased_2d_splatting ? 1 : 0;
    fc.reduce_point_count = r->s.reduce_point_count ? 1 : 0;
    fc.cull_small = r->s.cull_small_gaussians ? 1 : 0;
    fc.enable_occlusion = r->s.enable_occlusion_culling ? 1 : 0;
    fc.enable_hier = (r->s.enable_hierarchical_culling && !r->s.fully_disable_hierarchical_culling) ? 1 : 0;
    fc.width = r->s.width;
    fc.height = r->s.height;
    return fc;
}

BlockView block_view(gps_renderer* r) {
    BlockView b{};
    b.nodes = r->scene->block_nodes.get();
    b.culled = r->culled.get();
    b.chunk_count = r->chunk_count.get();
    b.node_count = r->scene->block_count;
    b.words = (b.node_count + 31) / 32;
    b.per_block = r->scene->per_block;
    return b;
}

void count_launch(gps_renderer* r, int stage, uint64_t n = 1) {
    r->frame_launches += n;
    r->timer.launches[stage] += n;
}

// Whether the view's passes walk their survivors in screen-bin order (see kBinMinBufferBytes).
bool screen_binned(const gps_renderer* r) {
    return GPS_SPLAT_BINNED != 0 && r->entries * sizeof(uint64_t) >= kBinMinBufferBytes;
}

void render_pass(gps_renderer* r, const FrameConst& fc, int frame, bool first, cudaStream_t st) {
    const int frame_seed = 4 * frame + (first ? 0 : 2);
    BlockView blocks = block_view(r);
    const bool listed = fc.enable_hier && blocks.node_count;
    if (listed) {
        r->timer.mark(kStCull, st);
        launch_block_cull(blocks, fc, r->hiz, st);
        launch_visible_chunks(blocks, r->n, r->chunk_list.get(), r->mask[0].get(), r->mask[1].get(),
                              r->mask_iter.get(), st);
        count_launch(r, kStCull, 2);
    }
    r->timer.mark(kStPreprocess, st);
    PreprocessArgs pa{};
    pa.fc = fc;
    pa.frame_seed = frame_seed;
    pa.only_previously_occluded = first ? 0 : 1;
    pa.n = r->n;
    pa.counts = r->counts.get();
    pa.mask_pair[0] = r->mask[0].get();
    pa.mask_pair[1] = r->mask[1].get();
    pa.mask_iter = r->mask_iter.get();
    pa.records = r->records.get();
    pa.hiz = r->hiz;
    pa.blocks = blocks;
    pa.chunk_list = listed ? r->chunk_list.get() : nullptr;
    pa.chunk_count = listed ? r->chunk_count.get() : nullptr;
    pa.immediate_threshold = r->s.immediate_splat_threshold;
    pa.buffer = r->buffer.get();
    pa.loaded = r->loaded.get();
    // screen bins for this view: one 64x64 splat-buffer tile each, wider for very large views
    const bool binned = screen_binned(r);
    int bin_shift = GPS_BIN_SHIFT;
    while ((uint64_t)((fc.up_width + (1 << bin_shift) - 1) >> bin_shift) *
               (uint64_t)((fc.up_height + (1 << bin_shift) - 1) >> bin_shift) > kMaxBins)
        ++bin_shift;
    const int bins_x = (fc.up_width + (1 << bin_shift) - 1) >> bin_shift;
    const int bins_y = (fc.up_height + (1 << bin_shift) - 1) >> bin_shift;
    int bin_sub_log2 = 0;  // cursors per bin, within kMaxBins words
    while ((1u << (bin_sub_log2 + 1)) <= kBinSubs && ((uint64_t)bins_x * bins_y << (bin_sub_log2 + 1)) <= kMaxBins)
        ++bin_sub_log2;
    const uint32_t nbins = (uint32_t)(bins_x * bins_y) << bin_sub_log2;
    pa.tile_totals = r->tile_state.get();
    pa.tile_shift = scan_tile_shift(r->n);
    pa.bins = binned ? r->bins.get() : nullptr;
    pa.bin_shift = bin_shift;
    pa.bin_sub_log2 = bin_sub_log2;
    pa.bin_count = (uint32_t)(bins_x * bins_y);
    pa.bins_x = bins_x;
    pa.bins_y = bins_y;
    if (r->scene->format == GPS_SCENE_FP32) {
        SceneFP32 s{r->scene->pos_op.get(), r->scene->rot.get(), r->scene->scale.get(), r->scene->sh.get(), r->n};
        launch_preprocess_fp32(pa, s, st);
    } else if (r->scene->format == GPS_SCENE_HALF) {
        SceneHalf s{r->scene->h_rec.get(), r->scene->h_scl.get(), r->scene->h_ac.get(), r->scene->h_origin.get(), r->n};
        launch_preprocess_half(pa, s, st);
    } else {
        SceneCompressed s{};
        s.geom = r->scene->geom.get();
        s.opac = r->scene->opac.get();
        s.sh_dc = r->scene->sh_dc.get();
        s.sh_ac = r->scene->sh_ac.get();
        s.bounds = r->scene->bounds;
        s.n = r->n;
        launch_preprocess_compressed(pa, s, st);
    }
    count_launch(r, kStPreprocess);
    r->timer.mark(kStScan, st);
    PassCounters* pc = r->counters.get() + (first ? 0 : 1);
    ScanArgs sa{};
    sa.counts = r->counts.get();
    sa.mask_pair[0] = r->mask[0].get();
    sa.mask_pair[1] = r->mask[1].get();
    sa.mask_iter = r->mask_iter.get();
    sa.n = r->n;
    sa.max_points = (uint32_t)std::max(0, r->s.max_number_of_points);
    sa.tile_points = 256;
    sa.surv_gid = r->surv_gid.get();
    sa.surv_start = r->surv_start.get();
    sa.tile_first_rank = r->tile_first_rank.get();
    sa.tile_state = r->tile_state.get();
    sa.counters = pc;
    sa.loaded = r->loaded.get();
    sa.bins = binned ? r->bins.get() : nullptr;
    sa.bin_crowded = r->bin_crowded;
    sa.nbins = nbins;
    sa.bin_shift = bin_shift;
    sa.bin_sub_log2 = bin_sub_log2;
    sa.bin_count = (uint32_t)(bins_x * bins_y);
    sa.bins_x = bins_x;
    sa.bins_y = bins_y;
    sa.up_width = fc.up_width;
    sa.up_height = fc.up_height;
    sa.records = r->records.get();
    sa.sorted_gid = r->sorted_gid.get();
    sa.sorted_pstart = r->sorted_pstart.get();
    sa.sorted_qstart = r->sorted_qstart.get();
    launch_scan_fused(sa, st);
    count_launch(r, kStScan, 2);  // tile (and bin) scan, downsweep with binning and tile owners
    r->timer.mark(kStSplat, st);
    SplatArgs sp{};
    sp.fc = fc;
    sp.frame_seed = frame_seed + 1;
    sp.records = r->records.get();
    sp.surv_gid = r->surv_gid.get();
    sp.surv_start = r->surv_start.get();
    sp.sorted_gid = binned ? r->sorted_gid.get() : nullptr;
    sp.sorted_qstart = r->sorted_qstart.get();
    sp.sorted_pstart = r->sorted_pstart.get();
    sp.tile_first_rank = r->tile_first_rank.get();
    sp.counters = pc;
    sp.buffer = r->buffer.get();
    sp.n = r->n;
    sp.clear_a = r->tile_state.get();
    sp.clear_a_words = std::max<uint32_t>(r->scan_tiles, 1);
    sp.clear_b = binned ? r->bins.get() : nullptr;
    sp.clear_b_words = binned ? nbins : 0u;
    sp.mask_iter = r->mask_iter.get();
    launch_splat(sp, r->splat_grid, 256, st);
    count_launch(r, kStSplat);
}

}  // namespace

// ---------------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------------
extern "C" {

int32_t gps_abi_version(void) { return GPS_B200_ABI_VERSION; }
const char* gps_last_error(void) { return last_error(); }

void gps_settings_default(gps_settings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->width = 1920;
    s->height = 1080;
    s->supersampling_factor = 2;
    s->samples_per_pixel = 1;
    s->max_number_of_points = 250000000;
    s->fovy = 45.0f;
    s->near_view_plane = 0.2f;
    s->far_view_plane = 10000.0f;
    s->enable_hierarchical_culling = 1;
    s->fully_disable_hierarchical_culling = 0;
    s->enable_occlusion_culling = 1;
    s->occlusion_culling_min_reduce_count = 0;
    s->cull_small_gaussians = 0;
    s->use_unbiased_2d_splatting = 1;
    s->reduce_point_count = 1;
    s->accumulation_mode = GPS_ACCUM_PROGRESSIVE;
    s->sort_morton_order = 0;
    s->immediate_splat_threshold = 0;
    s->points_per_thread = 0;
}

gps_status gps_settings_parse_args(int32_t argc, const char* const* argv, gps_settings* s, char* model_path,
                                   size_t model_cap, char* camera_path, size_t camera_cap) {
    if (!s || (argc > 0 && !argv)) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    auto need = [&](int i, int k) { return i + k < argc; };
    auto put = [](char* dst, size_t cap, const char* v) {
        if (dst && cap) {
            std::strncpy(dst, v, cap - 1);
            dst[cap - 1] = 0;
        }
    };
    try {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a == "--background" && need(i, 3)) {
                for (int k = 0; k < 3; ++k) s->background[k] = std::stof(argv[++i]);
            } else if (a == "--fovy" && need(i, 1)) {
                s->fovy = std::stof(argv[++i]);
            } else if ((a == "--near-view-plane" || a == "--near_view_plane") && need(i, 1)) {
                s->near_view_plane = std::stof(argv[++i]);
            } else if ((a == "--far-view-plane" || a == "--far_view_plane") && need(i, 1)) {
                s->far_view_plane = std::stof(argv[++i]);
            } else if ((a == "--samples-per-pixel" || a == "--samples_per_pixel") && need(i, 1)) {
                s->samples_per_pixel = std::stoi(argv[++i]);
            } else if ((a == "--max-number-of-points" || a == "--max_number_of_points") && need(i, 1)) {
                s->max_number_of_points = std::stoi(argv[++i]);
            } else if ((a == "--supersampling-factor" || a == "--supersampling_factor") && need(i, 1)) {
                s->supersampling_factor = std::stoi(argv[++i]);
            } else if (a == "--resolution" && need(i, 2)) {
                s->width = (int)std::stof(argv[++i]);
                s->height = (int)std::stof(argv[++i]);
            } else if ((a == "--set-target-width" || a == "--set_target_width") && need(i, 1)) {
                s->width = std::stoi(argv[++i]);
            } else if (a == "--cull-small") {
                s->cull_small_gaussians = 1;
            } else if (a == "--one_point_per_thread" || a == "--one-point-per-thread") {
                s->reduce_point_count = 0;
            } else if (a == "--disable_hierarchical_culling" || a == "--disable-hierarchical-culling") {
                s->enable_hierarchical_culling = 0;
            } else if (a == "--disable_occlusion_culling" || a == "--disable-occlusion-culling") {
                s->enable_occlusion_culling = 0;
            } else if (a == "--sort_morton_order" || a == "--sort-morton-order") {
                s->sort_morton_order = 1;
            } else if (a == "--taa") {
                s->accumulation_mode = GPS_ACCUM_TAA;
            } else if ((a == "--cameras-path" || a == "--camera-path") && need(i, 1)) {
                put(camera_path, camera_cap, argv[++i]);
            } else if (a == "--model-path" && need(i, 1)) {
                put(model_path, model_cap, argv[++i]);
            }
            // other viewer flags (--disable-gui, --run-tests, ...) are accepted and ignored,
            // as the reference ignores unknown ones (parse_args.cuh:120-122)
        }
    } catch (const std::exception& e) {
        return fail(GPS_ERR_INVALID_ARGUMENT, std::string("bad numeric argument: ") + e.what());
    }
    return GPS_OK;
}

// sort: 0 keeps the given order, 1 reorders on the host (morton_sort), 2 on the device.
static gps_status scene_create(std::vector<CpuGaussian>& g, int32_t format, bool presorted, gps_scene** out,
                               int32_t sort = 0) {
    if (format != GPS_SCENE_FP32 && format != GPS_SCENE_COMPRESSED && format != GPS_SCENE_HALF)
        return fail(GPS_ERR_INVALID_ARGUMENT, "unknown scene format");
    if (g.size() >= (1ull << 30)) return fail(GPS_ERR_SIZE, "scenes are limited to 2^30 Gaussians");
    auto s = std::make_unique<gps_scene>();
    s->format = format;
    s->presorted = presorted;
    try {
        if (sort == 1) morton_sort(g);
        bool device_sort = sort == 2;
        if (device_sort && format == GPS_SCENE_COMPRESSED) {
            // the compressed encoding is made on the host: order the host copy by the device's keys
            std::vector<uint32_t> order(g.size());
            device_morton_order(g.data(), g.size(), order.data());
            std::vector<CpuGaussian> tmp(g.size());
            for (size_t j = 0; j < g.size(); ++j) tmp[j] = g[order[j]];
            g.swap(tmp);
            device_sort = false;
        }
        scene_upload(s.get(), g.data(), g.size(), device_sort);
    } catch (const CudaError& e) {
        return fail(std::string(e.what()).find("cudaMalloc") != std::string::npos ? GPS_ERR_OUT_OF_MEMORY : GPS_ERR_CUDA, e.what());
    }
    *out = s.release();
    return GPS_OK;
}

gps_status gps_scene_load_ply(const char* path, int32_t format, int32_t sort_morton_order, gps_scene** out,
                              int32_t* presorted_out) {
    if (!path || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::string resolved;
    int rc = resolve_model_path(path, resolved);
    if (rc) return (gps_status)rc;
    std::vector<CpuGaussian> g;
    std::vector<std::string> comments;
    rc = ply_read(resolved, g, comments);
    if (rc) return (gps_status)rc;
    bool presorted = has_bvh_sorted_comment(comments);
    if (presorted_out) *presorted_out = presorted ? 1 : 0;
    // a file written in BVH order keeps it (gaussian_loader.cu:363)
    return scene_create(g, format, presorted, out, presorted ? 0 : (sort_morton_order == 2 ? 2 : sort_morton_order ? 1 : 0));
}

gps_status gps_scene_from_host(const float* gaussians, uint64_t count, int32_t format, int32_t presorted,
                               gps_scene** out) {
    if (!out || (!gaussians && count)) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::vector<CpuGaussian> g(count);
    if (count) std::memcpy(g.data(), gaussians, count * sizeof(CpuGaussian));
    return scene_create(g, format, presorted != 0, out);
}

gps_status gps_scene_from_host_sorted(const float* gaussians, uint64_t count, int32_t format, int32_t sort_morton_order,
                                      gps_scene** out) {
    if (!out || (!gaussians && count)) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    if (sort_morton_order < 0 || sort_morton_order > 2) return fail(GPS_ERR_INVALID_ARGUMENT, "sort_morton_order must be 0, 1 or 2");
    *out = nullptr;
    std::vector<CpuGaussian> g(count);
    if (count) std::memcpy(g.data(), gaussians, count * sizeof(CpuGaussian));
    return scene_create(g, format, false, out, sort_morton_order);
}

gps_status gps_morton_order(const float* gaussians, uint64_t count, int32_t on_device, uint32_t* order) {
    if ((!gaussians || !order) && count) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    if (count >= (1ull << 30)) return fail(GPS_ERR_SIZE, "scenes are limited to 2^30 Gaussians");
    const CpuGaussian* g = reinterpret_cast<const CpuGaussian*>(gaussians);
    if (!on_device) {
        morton_order(g, count, order);
        return GPS_OK;
    }
    try {
        device_morton_order(g, count, order);
    } catch (const CudaError& e) {
        return fail(std::string(e.what()).find("cudaMalloc") != std::string::npos ? GPS_ERR_OUT_OF_MEMORY : GPS_ERR_CUDA, e.what());
    }
    return GPS_OK;
}

uint64_t gps_scene_count(const gps_scene* scene) { return scene ? scene->n : 0; }
int32_t gps_scene_format_of(const gps_scene* scene) { return scene ? scene->format : -1; }

gps_status gps_scene_tile(const gps_scene* src, int32_t copies, const float* offsets_xz, gps_scene** out) {
    if (!src || !offsets_xz || !out || copies < 1) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    *out = nullptr;
    if (src->format != GPS_SCENE_HALF) return fail(GPS_ERR_INVALID_ARGUMENT, "only GPS_SCENE_HALF scenes can be tiled");
    const uint64_t n = src->n, total = n * (uint64_t)copies;
    if (total >= (1ull << 30)) return fail(GPS_ERR_SIZE, "scenes are limited to 2^30 Gaussians");
    if (n % kHalfOriginBlock) return fail(GPS_ERR_INVALID_ARGUMENT, "the source count must be a multiple of 16");
    auto s = std::make_unique<gps_scene>();
    s->format = GPS_SCENE_HALF;
    s->n = total;
    s->presorted = src->presorted;
    uint32_t pb = gaussians_per_block(total);
    if (n % pb || pb % src->per_block) pb = src->per_block;   // blocks must not straddle copies
    s->per_block = pb;
    s->block_count = (uint32_t)((total + pb - 1) / pb);
    try {
        const uint64_t ob = n / kHalfOriginBlock;
        s->h_rec.reset(dev_alloc<uint4>(total));
        s->h_scl.reset(dev_alloc<uint4>(total));
        s->h_ac.reset(dev_alloc<uint4>(total * 3));
        s->h_origin.reset(dev_alloc<float4>(ob * copies));
        s->block_nodes.reset(dev_alloc<float4>((size_t)s->block_count * 2));
        dptr<float2> offs(dev_alloc<float2>(copies));
        GPS_CUDA(cudaMemcpy(offs.get(), offsets_xz, sizeof(float2) * copies, cudaMemcpyHostToDevice));
        for (int32_t k = 0; k < copies; ++k) {
            GPS_CUDA(cudaMemcpy(s->h_rec.get() + k * n, src->h_rec.get(), n * sizeof(uint4), cudaMemcpyDeviceToDevice));
            GPS_CUDA(cudaMemcpy(s->h_scl.get() + k * n, src->h_scl.get(), n * sizeof(uint4), cudaMemcpyDeviceToDevice));
            GPS_CUDA(cudaMemcpy(s->h_ac.get() + k * n * 3, src->h_ac.get(), n * 3 * sizeof(uint4), cudaMemcpyDeviceToDevice));
            launch_translate_origins(src->h_origin.get(), (uint32_t)ob, offsets_xz[2 * k], offsets_xz[2 * k + 1],
                                     s->h_origin.get() + k * ob, 0);
        }
        launch_tile_nodes(src->block_nodes.get(), src->per_block, (uint32_t)n, pb, (uint32_t)copies, offs.get(), total,
                          s->block_nodes.get(), s->block_count, 0);
        GPS_CUDA(cudaGetLastError());
        GPS_CUDA(cudaDeviceSynchronize());
    } catch (const CudaError& e) {
        return fail(std::string(e.what()).find("cudaMalloc") != std::string::npos ? GPS_ERR_OUT_OF_MEMORY : GPS_ERR_CUDA, e.what());
    }
    *out = s.release();
    return GPS_OK;
}
void gps_scene_free(gps_scene* scene) { delete scene; }

gps_status gps_ply_write(const char* path, const float* gaussians, uint64_t count, const char* comments) {
    if (!path || (!gaussians && count)) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<std::string> cs;
    if (comments) {
        std::string c = comments, cur;
        for (char ch : c) {
            if (ch == '\n') {
                if (!cur.empty()) cs.push_back(cur);
                cur.clear();
            } else cur += ch;
        }
        if (!cur.empty()) cs.push_back(cur);
    }
    int rc = ply_write(path, reinterpret_cast<const CpuGaussian*>(gaussians), count, cs);
    return (gps_status)rc;
}

gps_status gps_ply_read(const char* path, float* out, uint64_t capacity, uint64_t* count, int32_t* presorted) {
    if (!path || !count) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::string resolved;
    int rc = resolve_model_path(path, resolved);
    if (rc) return (gps_status)rc;
    std::vector<std::string> comments;
    uint64_t n = 0;
    rc = out ? ply_read_into(resolved, reinterpret_cast<CpuGaussian*>(out), capacity, n, comments)
             : ply_count(resolved, n, comments);  // count only: the header alone
    *count = n;
    if (rc) return (gps_status)rc;
    if (presorted) *presorted = has_bvh_sorted_comment(comments) ? 1 : 0;
    return GPS_OK;
}

}  // extern "C"

namespace {

gps_status check_view_size(const gps_settings& s, uint64_t* entries_out) {
    if (s.width <= 0 || s.height <= 0 || s.supersampling_factor <= 0 || s.samples_per_pixel <= 0)
        return fail(GPS_ERR_INVALID_ARGUMENT, "resolution, supersampling factor and samples per pixel must be positive");
    const uint64_t up_w = (uint64_t)s.width * s.supersampling_factor, up_h = (uint64_t)s.height * s.supersampling_factor;
    if (up_w > 65504 || up_h > 65504) return fail(GPS_ERR_SIZE, "supersampled resolution above 65504 pixels per axis");
    const uint64_t entries = splat_buffer_entries((int)up_w, (int)up_h, s.samples_per_pixel);
    if (entries >= (1ull << 31)) return fail(GPS_ERR_SIZE, "splat buffer above 2^31 entries");
    *entries_out = entries;
    return GPS_OK;
}

// Makes r render width x height at spp samples per pixel from now on, within its capacity.
gps_status configure_view(gps_renderer* r, int32_t width, int32_t height, int32_t spp) {
    gps_settings s = r->s;
    s.width = width;
    s.height = height;
    s.samples_per_pixel = spp;
    uint64_t entries = 0;
    gps_status st = check_view_size(s, &entries);
    if (st != GPS_OK) return st;
    HizView h = r->hiz;
    hiz_layout(h, width, height);
    if (entries > r->cap_entries || h.mip_size > r->cap_mip)
        return fail(GPS_ERR_SIZE, "view of " + std::to_string(width) + "x" + std::to_string(height) + " at " +
                                      std::to_string(spp) + " spp exceeds the renderer's capacity");
    r->s = s;
    r->up_w = width * s.supersampling_factor;
    r->up_h = height * s.supersampling_factor;
    r->entries = entries;
    r->hiz = h;
    return GPS_OK;
}

// A renderer for `settings` whose splat buffer and Hi-Z also fit views of `capacity`'s size and
// whose per-Gaussian scratch also fits scenes of up to cap_n Gaussians in cap_blocks blocks.
gps_status create_renderer(gps_scene* scene, const gps_settings* settings, const gps_settings* capacity,
                           gps_renderer** out, uint64_t cap_n = 0, uint32_t cap_blocks = 0) {
    if (!scene || !settings || !capacity || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    const gps_settings& s = *settings;
    uint64_t cap_entries = 0;
    const gps_status cs = check_view_size(*capacity, &cap_entries);
    if (cs != GPS_OK) return cs;
    HizView cap_hiz{};
    hiz_layout(cap_hiz, capacity->width, capacity->height);
    if (s.width <= 0 || s.height <= 0 || s.supersampling_factor <= 0 || s.samples_per_pixel <= 0)
        return fail(GPS_ERR_INVALID_ARGUMENT, "resolution, supersampling factor and samples per pixel must be positive");
    if (!(s.far_view_plane > s.near_view_plane) || !(s.fovy > 0.0f))
        return fail(GPS_ERR_INVALID_ARGUMENT, "need far > near and fovy > 0");
    if (s.points_per_thread < 0 || s.points_per_thread > 64)
        return fail(GPS_ERR_INVALID_ARGUMENT, "points_per_thread must be 0 (the reference's rule) or 1..64");
    const uint64_t up_w = (uint64_t)s.width * s.supersampling_factor, up_h = (uint64_t)s.height * s.supersampling_factor;
    if (up_w > 65504 || up_h > 65504) return fail(GPS_ERR_SIZE, "supersampled resolution above 65504 pixels per axis");
    const uint64_t entries = splat_buffer_entries((int)up_w, (int)up_h, s.samples_per_pixel);
    if (entries >= (1ull << 31)) return fail(GPS_ERR_SIZE, "splat buffer above 2^31 entries");
    auto r = std::make_unique<gps_renderer>();
    r->scene = scene;
    r->s = s;
    r->up_w = (int)up_w;
    r->up_h = (int)up_h;
    r->entries = entries;
    r->cap_n = (uint32_t)std::max<uint64_t>(scene->n, cap_n);
    r->cap_blocks = std::max<uint32_t>(scene->block_count, cap_blocks);
    r->n = r->cap_n;  // size the per-Gaussian arrays for the capacity, then bind the scene
    r->scan_tiles = scan_tile_count(r->n);
    r->n_pad = r->scan_tiles * kScanTileGaussians;
    r->cap_entries = std::max(entries, cap_entries);
    if (const char* v = std::getenv("GPS_BIN_CROWDED")) r->bin_crowded = (uint32_t)std::strtoul(v, nullptr, 10);
    try {
        r->buffer.reset(dev_alloc<uint64_t>(r->cap_entries));
        r->counts.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n_pad, 16)));
        GPS_CUDA(cudaMemset(r->counts.get(), 0, sizeof(uint32_t) * std::max<uint32_t>(r->n_pad, 16)));
        const uint32_t words = (r->n + 31) / 32;
        for (int i = 0; i < 2; ++i) {
            r->mask[i].reset(dev_alloc<uint32_t>(words + 1));
            GPS_CUDA(cudaMemset(r->mask[i].get(), 0, sizeof(uint32_t) * (words + 1)));
        }
        r->mask_iter.reset(dev_alloc<uint32_t>(1));
        GPS_CUDA(cudaMemset(r->mask_iter.get(), 0, sizeof(uint32_t)));
        r->records.reset(dev_alloc<SplatRecord>(std::max<uint32_t>(r->n, 1)));
        r->surv_gid.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n, 1)));
        r->surv_start.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n, 1)));
        r->sorted_gid.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n, 1)));
        r->sorted_pstart.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n, 1)));
        r->sorted_qstart.reset(dev_alloc<uint32_t>(std::max<uint32_t>(r->n, 1)));
        r->bins.reset(dev_alloc<unsigned long long>(kMaxBins + 1));

        GPS_CUDA(cudaMemset(r->bins.get(), 0, sizeof(unsigned long long) * (kMaxBins + 1)));
        const uint64_t max_pts = (uint64_t)std::max(0, s.max_number_of_points);
        r->tile_first_rank.reset(dev_alloc<uint32_t>(max_pts / 256 + 2));
        r->tile_state.reset(dev_alloc<unsigned long long>(std::max<uint32_t>(r->scan_tiles, 1)));
        // the preprocess accumulates each pass's tile totals here; the splat clears them after use
        GPS_CUDA(cudaMemset(r->tile_state.get(), 0, sizeof(unsigned long long) * std::max<uint32_t>(r->scan_tiles, 1)));
        r->counters.reset(dev_alloc<PassCounters>(2));
        GPS_CUDA(cudaMemset(r->counters.get(), 0, sizeof(PassCounters) * 2));
        const uint32_t bwords = (r->cap_blocks + 31) / 32;
        r->culled.reset(dev_alloc<uint32_t>(bwords + 1));
        r->chunk_list.reset(dev_alloc<uint32_t>(words + 1));
        r->chunk_count.reset(dev_alloc<uint32_t>(1));
        GPS_CUDA(cudaMemset(r->chunk_count.get(), 0, sizeof(uint32_t)));
        r->loaded.reset(dev_alloc<uint32_t>(1));
        GPS_CUDA(cudaMemset(r->loaded.get(), 0, sizeof(uint32_t)));
        GPS_CUDA(cudaMemset(r->culled.get(), 0, sizeof(uint32_t) * (bwords + 1)));
        hiz_layout(r->hiz, s.width, s.height);
        r->cap_mip = std::max(r->hiz.mip_size, cap_hiz.mip_size);
        r->mip.reset(dev_alloc<float>(r->cap_mip));
        r->hiz.mip = r->mip.get();
        r->hiz_done.reset(dev_alloc<unsigned>(1));
        GPS_CUDA(cudaMemset(r->hiz_done.get(), 0, sizeof(unsigned)));
        r->hiz.done = r->hiz_done.get();
        // the reference leaves its Hi-Z uninitialised before the first frame; +inf here
        // means "nothing occluded" for frame 1
        fill_f32<<<148 * 4, 256>>>(r->mip.get(), r->cap_mip, INFINITY);
        GPS_CUDA(cudaGetLastError());
        GPS_CUDA(cudaMallocHost(&r->host_counters, sizeof(PassCounters) * 2));
        std::memset(r->host_counters, 0, sizeof(PassCounters) * 2);
        GPS_CUDA(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming));
        r->splat_grid = splat_grid_size(256);
        GPS_CUDA(cudaDeviceSynchronize());
    } catch (const CudaError& e) {
        return fail(std::string(e.what()).find("cudaMalloc") != std::string::npos ? GPS_ERR_OUT_OF_MEMORY : GPS_ERR_CUDA, e.what());
    }
    r->n = (uint32_t)scene->n;
    r->scan_tiles = scan_tile_count(r->n);
    r->n_pad = r->scan_tiles * kScanTileGaussians;
    *out = r.release();
    return GPS_OK;
}

// Points r at another resident scene whose sizes fit its per-Gaussian scratch.
gps_status bind_scene(gps_renderer* r, gps_scene* scene) {
    if (scene->n > r->cap_n || scene->block_count > r->cap_blocks)
        return fail(GPS_ERR_SIZE, "scene larger than the renderer's per-Gaussian capacity");
    r->scene = scene;
    r->n = (uint32_t)scene->n;
    r->scan_tiles = scan_tile_count(r->n);
    r->n_pad = r->scan_tiles * kScanTileGaussians;
    return GPS_OK;
}

gps_status render_frame_impl(gps_renderer* r, const gps_camera* cam, float* d_image, float* d_depth, cudaStream_t st);

}  // namespace

extern "C" {

gps_status gps_renderer_create(gps_scene* scene, const gps_settings* settings, gps_renderer** out) {
    return create_renderer(scene, settings, settings, out);
}

void gps_renderer_free(gps_renderer* r) {
    if (r) cudaDeviceSynchronize();
    delete r;
}

gps_status gps_render_frame(gps_renderer* r, const gps_camera* cam, float* d_image, float* d_depth, void* stream) {
    if (!r || !cam || !d_image || !d_depth) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    return render_frame_impl(r, cam, d_image, d_depth, as_stream(stream));
}

}  // extern "C"

namespace {
gps_status render_frame_impl(gps_renderer* r, const gps_camera* cam, float* d_image, float* d_depth, cudaStream_t st) {
    const FrameConst fc = make_frame_const(r, cam);
    const uint64_t bg = 0xFFFFFFF000000000ull |
                        rgb_to_36bits(make_v3(r->s.background[0], r->s.background[1], r->s.background[2]));
    r->frame_launches = 0;
    r->timer.mark(kStClear, st);
    launch_clear(r->buffer.get(), r->entries, bg, st);
    count_launch(r, kStClear);
    if (r->n > 0) render_pass(r, fc, cam->frame, true, st);
    ResolveArgs ra{};
    ra.buffer = r->buffer.get();
    ra.color = d_image;
    ra.depth = d_depth;
    ra.width = r->s.width;
    ra.height = r->s.height;
    ra.num_passes = r->s.samples_per_pixel;
    ra.ss = r->s.supersampling_factor;
    ra.entries = r->entries;
    ra.near_plane = r->s.near_view_plane;
    ra.far_plane = r->s.far_view_plane;
    ra.initial_value = bg;
    r->second_pass_last = false;
    if (r->s.enable_occlusion_culling) {
        r->timer.mark(kStResolve, st);
        launch_resolve(ra, true, st);
        count_launch(r, kStResolve);
        r->timer.mark(kStHiz, st);
        launch_hiz_build(r->hiz, d_depth, r->s.occlusion_culling_min_reduce_count, st);
        count_launch(r, kStHiz);
        if (r->n > 0) {
            render_pass(r, fc, cam->frame, false, st);
            r->second_pass_last = true;
        }
    } else {
        cudaMemsetAsync(r->counters.get() + 1, 0, sizeof(PassCounters), st);
    }
    r->timer.mark(kStResolve, st);
    launch_resolve(ra, false, st);
    count_launch(r, kStResolve);
    if (r->s.enable_occlusion_culling) {
        r->timer.mark(kStHiz, st);
        launch_hiz_build(r->hiz, d_depth, r->s.occlusion_culling_min_reduce_count, st);
        count_launch(r, kStHiz);
    }
    r->timer.mark(-1, st);
    cudaMemcpyAsync(r->host_counters, r->counters.get(), sizeof(PassCounters) * 2, cudaMemcpyDeviceToHost, st);
    cudaEventRecord(r->done, st);
    r->have_frame = true;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GPS_ERR_CUDA, std::string("frame launch failed: ") + cudaGetErrorString(e));
    return GPS_OK;
}
}  // namespace

extern "C" {

gps_status gps_renderer_reset(gps_renderer* r, void* stream) {
    if (!r) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    fill_f32<<<148, 256, 0, as_stream(stream)>>>(r->mip.get(), r->hiz.mip_size, INFINITY);
    cudaMemsetAsync(r->mask_iter.get(), 0, sizeof(uint32_t), as_stream(stream));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_renderer_stats(gps_renderer* r, gps_stats* out) {
    if (!r || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    if (!r->have_frame) return GPS_OK;
    cudaError_t e = cudaEventSynchronize(r->done);
    if (e != cudaSuccess) return fail(GPS_ERR_CUDA, std::string("frame failed: ") + cudaGetErrorString(e));
    const PassCounters* c = r->host_counters;
    out->num_points_one = (int32_t)c[0].points;
    out->num_points_two = (int32_t)c[1].points;
    out->num_gaussians_one = (int32_t)r->n;
    out->num_gaussians_two = r->s.enable_occlusion_culling ? (int32_t)r->n : 0;
    out->survivors_one = (int32_t)c[0].survivors;
    out->survivors_two = (int32_t)c[1].survivors;
    out->total_points_one = c[0].total_points;
    out->total_points_two = c[1].total_points;
    out->truncated = (int32_t)(c[0].truncated | c[1].truncated);
    out->device_timeouts = (int32_t)(c[0].scan_timeouts + c[1].scan_timeouts);
    out->kernel_launches = (int32_t)r->frame_launches;
    out->gaussians_read_one = (int32_t)c[0].loaded;
    out->gaussians_read_two = (int32_t)c[1].loaded;
    const bool binned = screen_binned(r);
    out->screen_order_one = (binned && c[0].points && !c[0].truncated && !c[0].crowded) ? 1 : 0;
    out->screen_order_two = (binned && c[1].points && !c[1].truncated && !c[1].crowded) ? 1 : 0;
    if (out->device_timeouts) return fail(GPS_ERR_DEVICE_TIMEOUT, "a device-side look-back wait gave up");
    return GPS_OK;
}

gps_status gps_renderer_enable_timing(gps_renderer* r, int32_t enable) {
    if (!r) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    StageTimer& t = r->timer;
    if (enable && t.pool.empty()) {
        t.pool.resize(4096);
        t.stage.assign(4096, -1);
        for (auto& e : t.pool) {
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return fail(GPS_ERR_CUDA, cudaGetErrorString(err));
        }
    }
    t.drain();
    t.on = enable != 0;
    return GPS_OK;
}

gps_status gps_renderer_stage_times(gps_renderer* r, float* out_ms, uint64_t* out_launches, int32_t reset) {
    if (!r || !out_ms) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    r->timer.drain();
    for (int i = 0; i < kStCount; ++i) {
        out_ms[i] = (float)r->timer.total_ms[i];
        if (out_launches) out_launches[i] = r->timer.launches[i];
    }
    if (reset) {
        for (int i = 0; i < kStCount; ++i) {
            r->timer.total_ms[i] = 0.0;
            r->timer.launches[i] = 0;
        }
    }
    return GPS_OK;
}

gps_status gps_renderer_splat_buffer(gps_renderer* r, const uint64_t** d_buffer, uint64_t* entries) {
    if (!r || !d_buffer || !entries) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *d_buffer = r->buffer.get();
    *entries = r->entries;
    return GPS_OK;
}

gps_status gps_renderer_derived(gps_renderer* r, const gps_camera* cam, float* out36) {
    if (!r || !cam || !out36) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    FrameConst fc = make_frame_const(r, cam);
    mat4_to(fc.vp, out36);
    mat4_to(fc.cam, out36 + 16);
    out36[32] = fc.tan_fov.x;
    out36[33] = fc.tan_fov.y;
    out36[34] = fc.focal.x;
    out36[35] = fc.focal.y;
    return GPS_OK;
}

gps_status gps_renderer_debug_view(gps_renderer* r, gps_debug_view* out) {
    if (!r || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    if (r->have_frame) {
        cudaError_t e = cudaEventSynchronize(r->done);
        if (e != cudaSuccess) return fail(GPS_ERR_CUDA, cudaGetErrorString(e));
    }
    out->counts = r->counts.get();
    // the reference's getWeightsMaskPrevious / Current after the frame: mask[(it + 1) % 2] is the
    // last pass's mask whenever that pass had points (the counter advanced after it)
    uint32_t it = 0;
    cudaError_t ce = cudaMemcpy(&it, r->mask_iter.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return fail(GPS_ERR_CUDA, cudaGetErrorString(ce));
    out->mask_last = r->mask[(it + 1) % 2].get();
    out->mask_other = r->mask[it % 2].get();
    out->surv_gid = r->surv_gid.get();
    out->surv_start = r->surv_start.get();
    const PassCounters& c = r->host_counters[r->second_pass_last ? 1 : 0];
    out->survivors = c.survivors;
    out->points = c.points;
    out->records = reinterpret_cast<const float*>(r->records.get());
    out->hiz = r->mip.get();
    out->hiz_size = r->hiz.mip_size;
    out->block_culled = r->culled.get();
    out->block_words = (r->scene->block_count + 31) / 32;
    out->block_nodes = reinterpret_cast<const float*>(r->scene->block_nodes.get());
    out->block_count = r->scene->block_count;
    out->per_block = r->scene->per_block;
    return GPS_OK;
}

gps_status gps_post_taa(uint8_t* d_image_u8, float* d_out_color, const float* d_cur_color, const float* d_prev_color,
                        const float* d_cur_depth, const float* d_prev_depth, const float* reproj16, float blend,
                        int32_t width, int32_t height, int32_t frame_number, void* stream) {
    if (!d_image_u8 || !d_out_color || !d_cur_color || !d_prev_color || !d_cur_depth || !reproj16 || width <= 0 ||
        height <= 0)
        return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    if (d_out_color == d_cur_color) return fail(GPS_ERR_INVALID_ARGUMENT, "d_out_color must not alias d_cur_color");
    launch_taa(d_image_u8, d_out_color, d_cur_color, d_prev_color, d_cur_depth, d_prev_depth, mat4_from(reproj16), blend,
               width, height, frame_number, as_stream(stream));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_post_progressive(uint8_t* d_image_u8, float* d_cur_color, float* d_accum, int32_t width,
                                int32_t height, int32_t frames, void* stream) {
    if (!d_image_u8 || !d_cur_color || !d_accum || width <= 0 || height <= 0 || frames <= 0)
        return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    launch_progressive(d_image_u8, d_cur_color, d_accum, width, height, frames, as_stream(stream));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// batched multi-view rendering
// ---------------------------------------------------------------------------------
struct gps_batch {
    gps_settings s{};
    std::vector<gps_renderer*> workers;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joined;
    cudaEvent_t forked = nullptr;
    int active = 1;
    // CUDA-graph replay: the batch's whole fork/join launch sequence, captured on a private
    // stream; a batch with the same view layout refreshes the executable graph's parameters
    // (cameras) with cudaGraphExecUpdate instead of instantiating a new one
    bool use_graph = false;
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int64_t> exec_layout;
    int64_t graph_instantiations = 0, graph_updates = 0;
    ~gps_batch() {
        cudaDeviceSynchronize();
        if (exec) cudaGraphExecDestroy(exec);
        if (capture) cudaStreamDestroy(capture);
        for (gps_renderer* w : workers) delete w;
        for (cudaStream_t st : streams) cudaStreamDestroy(st);
        for (cudaEvent_t e : joined) cudaEventDestroy(e);
        if (forked) cudaEventDestroy(forked);
    }
};

namespace {

// Renders one view on worker w as a fresh renderer's first frame would.
gps_status render_view(gps_renderer* w, const gps_view& v, cudaStream_t st) {
    gps_status rc = configure_view(w, v.width, v.height, v.samples_per_pixel);
    if (rc != GPS_OK) return rc;
    if (w->s.enable_occlusion_culling) fill_f32<<<148, 256, 0, st>>>(w->mip.get(), w->hiz.mip_size, INFINITY);
    cudaMemsetAsync(w->mask_iter.get(), 0, sizeof(uint32_t), st);
    return render_frame_impl(w, &v.camera, v.d_image, v.d_depth, st);
}

// Longest-processing-time-first assignment of views to workers by estimated cost (buffer
// entries cleared and resolved, plus a per-view share for the culling and preprocess).
std::vector<int> assign_views(const gps_batch* b, const gps_view* views, int32_t count, uint64_t n_gaussians) {
    std::vector<std::pair<double, int>> cost(count);
    const double ss = b->s.supersampling_factor;
    for (int i = 0; i < count; ++i)
        cost[i] = {(double)views[i].width * views[i].height * ss * ss * views[i].samples_per_pixel + 0.05 * (double)n_gaussians, i};
    std::sort(cost.begin(), cost.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<double> load(b->active, 0.0);
    std::vector<int> owner(count, 0);
    for (const auto& c : cost) {
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        owner[c.second] = w;
        load[w] += c.first;
    }
    return owner;
}

}  // namespace

extern "C" {

gps_status gps_batch_create(gps_scene* scene, const gps_settings* settings, int32_t max_width, int32_t max_height,
                            int32_t max_spp, int32_t workers, gps_batch** out) {
    if (!scene || !settings || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (workers < 1 || workers > 64) return fail(GPS_ERR_INVALID_ARGUMENT, "workers must be 1..64");
    auto b = std::make_unique<gps_batch>();
    b->s = *settings;
    gps_settings cap = *settings;
    cap.width = max_width;
    cap.height = max_height;
    cap.samples_per_pixel = max_spp;
    for (int i = 0; i < workers; ++i) {
        gps_renderer* w = nullptr;
        gps_status rc = create_renderer(scene, &cap, &cap, &w);
        if (rc != GPS_OK) return rc;
        b->workers.push_back(w);
        cudaStream_t st = nullptr;
        cudaEvent_t e = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return fail(GPS_ERR_CUDA, "stream or event creation failed");
        b->streams.push_back(st);
        b->joined.push_back(e);
    }
    if (cudaEventCreateWithFlags(&b->forked, cudaEventDisableTiming) != cudaSuccess)
        return fail(GPS_ERR_CUDA, "event creation failed");
    b->active = workers;
    *out = b.release();
    return GPS_OK;
}

void gps_batch_free(gps_batch* b) { delete b; }

gps_status gps_batch_set_workers(gps_batch* b, int32_t workers) {
    if (!b || workers < 1 || workers > (int32_t)b->workers.size()) return fail(GPS_ERR_INVALID_ARGUMENT, "bad worker count");
    b->active = workers;
    return GPS_OK;
}

int32_t gps_batch_workers(const gps_batch* b) { return b ? b->active : 0; }

namespace {
// The batch's launch sequence on `st`: fork to the workers' streams, each view as a fresh
// renderer's first frame on its worker, join back.
gps_status batch_enqueue(gps_batch* b, const gps_view* views, int32_t count, const std::vector<int>& owner,
                         cudaStream_t st) {
    cudaEventRecord(b->forked, st);
    for (int w = 0; w < b->active; ++w) cudaStreamWaitEvent(b->streams[w], b->forked, 0);
    gps_status rc = GPS_OK;
    for (int i = 0; i < count && rc == GPS_OK; ++i) rc = render_view(b->workers[owner[i]], views[i], b->streams[owner[i]]);
    for (int w = 0; w < b->active; ++w) {
        cudaEventRecord(b->joined[w], b->streams[w]);
        cudaStreamWaitEvent(st, b->joined[w], 0);
    }
    return rc;
}
}  // namespace

gps_status gps_batch_render(gps_batch* b, const gps_view* views, int32_t count, void* stream) {
    if (!b || (count > 0 && !views) || count < 0) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < count; ++i)
        if (!views[i].d_image || !views[i].d_depth) return fail(GPS_ERR_INVALID_ARGUMENT, "view without output buffers");
    cudaStream_t st = as_stream(stream);
    const std::vector<int> owner = assign_views(b, views, count, b->workers[0]->n);
    gps_status rc = GPS_OK;
    if (!b->use_graph) {
        rc = batch_enqueue(b, views, count, owner, st);
    } else {
        // the layout a captured graph can be refreshed for: worker count, K, and per view its
        // size, samples and worker (the same launches in the same order)
        std::vector<int64_t> layout = {count, b->active, b->s.points_per_thread};
        for (int i = 0; i < count; ++i) {
            layout.push_back(views[i].width);
            layout.push_back(views[i].height);
            layout.push_back(views[i].samples_per_pixel);
            layout.push_back(owner[i]);
        }
        if (cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(GPS_ERR_CUDA, "batch graph capture could not start");
        rc = batch_enqueue(b, views, count, owner, b->capture);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->capture, &g);
        if (rc == GPS_OK && (ce != cudaSuccess || !g)) rc = fail(GPS_ERR_CUDA, std::string("batch graph capture failed: ") + cudaGetErrorString(ce));
        if (rc == GPS_OK && b->exec && layout == b->exec_layout) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(b->exec, g, &info) == cudaSuccess) {
                ++b->graph_updates;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
        } else if (rc == GPS_OK && b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        if (rc == GPS_OK && !b->exec) {
            if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
                b->exec = nullptr;
                rc = fail(GPS_ERR_CUDA, "batch graph instantiation failed");
            } else {
                b->exec_layout = layout;
                ++b->graph_instantiations;
            }
        }
        if (g) cudaGraphDestroy(g);
        if (rc == GPS_OK && cudaGraphLaunch(b->exec, st) != cudaSuccess) rc = fail(GPS_ERR_CUDA, "batch graph launch failed");
    }
    if (rc != GPS_OK) return rc;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, std::string("batch launch failed: ") + cudaGetErrorString(e));
}

gps_status gps_batch_use_graph(gps_batch* b, int32_t enable) {
    if (!b) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    if (enable && !b->capture && cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) != cudaSuccess)
        return fail(GPS_ERR_CUDA, "stream creation failed");
    b->use_graph = enable != 0;
    return GPS_OK;
}

gps_status gps_batch_graph_stats(const gps_batch* b, int64_t* instantiations, int64_t* updates) {
    if (!b) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    if (instantiations) *instantiations = b->graph_instantiations;
    if (updates) *updates = b->graph_updates;
    return GPS_OK;
}

gps_status gps_batch_set_points_per_thread(gps_batch* b, int32_t k) {
    if (!b || k < 0 || k > 64) return fail(GPS_ERR_INVALID_ARGUMENT, "points_per_thread must be 0..64");
    b->s.points_per_thread = k;
    for (gps_renderer* w : b->workers) w->s.points_per_thread = k;
    return GPS_OK;
}

gps_status gps_batch_autotune_k(gps_batch* b, const gps_view* views, int32_t count, int32_t rounds, void* stream,
                                int32_t* chosen_workers, int32_t* chosen_k, float* ms) {
    if (!b || rounds < 1) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    const int32_t ks[] = {1, 2, 4, 8};
    int best_w = 1, best_k = b->s.points_per_thread;
    float best_ms = 0.0f;
    bool have = false;
    gps_status rc = GPS_OK;
    for (int32_t k : ks) {
        rc = gps_batch_set_points_per_thread(b, k);
        if (rc != GPS_OK) break;
        int32_t w = 1;
        float t = 0.0f;
        rc = gps_batch_autotune(b, views, count, rounds, stream, &w, &t);
        if (rc != GPS_OK) break;
        if (!have || t < best_ms) {
            have = true;
            best_w = w;
            best_k = k;
            best_ms = t;
        }
    }
    gps_batch_set_points_per_thread(b, best_k);
    b->active = best_w;
    if (chosen_workers) *chosen_workers = best_w;
    if (chosen_k) *chosen_k = best_k;
    if (ms) *ms = best_ms;
    return rc;
}

gps_status gps_batch_autotune(gps_batch* b, const gps_view* views, int32_t count, int32_t rounds, void* stream,
                              int32_t* chosen, float* ms) {
    if (!b || rounds < 1) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    cudaStream_t st = as_stream(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 1;
    float best_ms = 0.0f;
    gps_status rc = GPS_OK;
    for (int w = 1; w <= (int)b->workers.size() && rc == GPS_OK; w *= 2) {
        b->active = w;
        rc = gps_batch_render(b, views, count, stream);  // warm-up at this width
        cudaEventRecord(e0, st);
        for (int r = 0; r < rounds && rc == GPS_OK; ++r) rc = gps_batch_render(b, views, count, stream);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        t /= (float)rounds;
        if (w == 1 || t < best_ms) {
            best = w;
            best_ms = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->active = best;
    if (chosen) *chosen = best;
    if (ms) *ms = best_ms;
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// serving: request queue, dispatcher thread, GPU workers
// ---------------------------------------------------------------------------------
struct gps_server {
    using clock = std::chrono::steady_clock;
    struct Pending {
        gps_request req;
        clock::time_point submitted;
    };
    struct Worker {
        gps_renderer* r = nullptr;
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        dptr<float> img, dep;          // outputs of requests that bring none
        bool busy = false;
        Pending job{};
        uint64_t entries = 0;          // splat-buffer entries of the request in flight
        clock::time_point admitted;
    };
    std::vector<gps_scene*> scenes;
    std::vector<Worker> workers;
    int device = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Pending> queue;
    std::deque<gps_completion> done;
    uint64_t submitted = 0, completed = 0;
    uint64_t max_inflight = 67108864ull;   // admission budget in splat-buffer entries (0 = none)
    uint64_t inflight = 0;
    int ss = 1;
    bool stop = false;
    std::thread dispatcher;
    ~gps_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (dispatcher.joinable()) dispatcher.join();
        cudaDeviceSynchronize();
        for (Worker& w : workers) {
            delete w.r;
            if (w.st) cudaStreamDestroy(w.st);
            if (w.ev) cudaEventDestroy(w.ev);
        }
    }
};

namespace {

double ms_between(gps_server::clock::time_point a, gps_server::clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Called with the lock held.
void finish(gps_server* sv, const gps_server::Pending& p, int worker, gps_status st,
            gps_server::clock::time_point admitted) {
    const auto now = gps_server::clock::now();
    sv->done.push_back(gps_completion{p.req.id, (int32_t)st, worker, ms_between(p.submitted, admitted),
                                      ms_between(p.submitted, now)});
    ++sv->completed;
    sv->cv.notify_all();
}

gps_status start_request(gps_server* sv, gps_server::Worker& w, const gps_request& q) {
    if (q.scene < 0 || q.scene >= (int32_t)sv->scenes.size()) return fail(GPS_ERR_INVALID_ARGUMENT, "no such scene");
    gps_status rc = bind_scene(w.r, sv->scenes[q.scene]);
    if (rc != GPS_OK) return rc;
    gps_view v{};
    v.camera = q.camera;
    v.width = q.width;
    v.height = q.height;
    v.samples_per_pixel = q.samples_per_pixel;
    v.d_image = q.d_image ? q.d_image : w.img.get();
    v.d_depth = q.d_depth ? q.d_depth : w.dep.get();
    rc = render_view(w.r, v, w.st);
    if (rc != GPS_OK) return rc;
    cudaEventRecord(w.ev, w.st);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

void dispatch_loop(gps_server* sv) {
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    for (;;) {
        bool progressed = false, busy = false;
        for (size_t i = 0; i < sv->workers.size(); ++i) {
            gps_server::Worker& w = sv->workers[i];
            if (!w.busy) continue;
            const cudaError_t q = cudaEventQuery(w.ev);
            if (q == cudaErrorNotReady) {
                busy = true;
                continue;
            }
            finish(sv, w.job, (int)i, q == cudaSuccess ? GPS_OK : GPS_ERR_CUDA, w.admitted);
            w.busy = false;
            sv->inflight -= w.entries;
            progressed = true;
        }
        for (size_t i = 0; i < sv->workers.size() && !sv->queue.empty(); ++i) {
            gps_server::Worker& w = sv->workers[i];
            if (w.busy) continue;
            const gps_request& head = sv->queue.front().req;
            const uint64_t need = head.width > 0 && head.height > 0 && head.samples_per_pixel > 0
                                      ? splat_buffer_entries(head.width * sv->ss, head.height * sv->ss, head.samples_per_pixel)
                                      : 0;
            if (sv->inflight > 0 && sv->max_inflight > 0 && sv->inflight + need > sv->max_inflight) break;  // FIFO: wait
            gps_server::Pending p = sv->queue.front();
            sv->queue.pop_front();
            lk.unlock();  // launch without blocking submitters
            const auto admitted = gps_server::clock::now();
            const gps_status rc = start_request(sv, w, p.req);
            lk.lock();
            if (rc == GPS_OK) {
                w.busy = true;
                w.job = p;
                w.admitted = admitted;
                w.entries = need;
                sv->inflight += need;
                busy = true;
            } else {
                finish(sv, p, (int)i, rc, admitted);
            }
            progressed = true;
        }
        if (sv->stop && sv->queue.empty() && !busy) break;
        if (progressed) continue;
        if (busy) {  // poll the workers' events again shortly
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
        } else {
            sv->cv.wait_for(lk, std::chrono::milliseconds(5), [&] { return sv->stop || !sv->queue.empty(); });
        }
    }
}

}  // namespace

extern "C" {

gps_status gps_server_create(gps_scene* const* scenes, int32_t n_scenes, const gps_settings* settings,
                             int32_t max_width, int32_t max_height, int32_t max_spp, int32_t workers,
                             gps_server** out) {
    if (!scenes || n_scenes < 1 || !settings || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (workers < 1 || workers > 64) return fail(GPS_ERR_INVALID_ARGUMENT, "workers must be 1..64");
    auto sv = std::make_unique<gps_server>();
    uint64_t cap_n = 0;
    uint32_t cap_blocks = 0;
    for (int i = 0; i < n_scenes; ++i) {
        if (!scenes[i]) return fail(GPS_ERR_INVALID_ARGUMENT, "null scene");
        sv->scenes.push_back(scenes[i]);
        cap_n = std::max<uint64_t>(cap_n, scenes[i]->n);
        cap_blocks = std::max(cap_blocks, scenes[i]->block_count);
    }
    cudaGetDevice(&sv->device);
    sv->ss = settings->supersampling_factor > 0 ? settings->supersampling_factor : 1;
    gps_settings cap = *settings;
    cap.width = max_width;
    cap.height = max_height;
    cap.samples_per_pixel = max_spp;
    sv->workers.resize(workers);
    for (gps_server::Worker& w : sv->workers) {
        gps_status rc = create_renderer(scenes[0], &cap, &cap, &w.r, cap_n, cap_blocks);
        if (rc != GPS_OK) return rc;
        try {
            w.img.reset(dev_alloc<float>((size_t)max_width * max_height * 3));
            w.dep.reset(dev_alloc<float>((size_t)max_width * max_height));
        } catch (const CudaError& e) {
            return fail(GPS_ERR_OUT_OF_MEMORY, e.what());
        }
        if (cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming) != cudaSuccess)
            return fail(GPS_ERR_CUDA, "stream or event creation failed");
    }
    gps_server* raw = sv.get();
    raw->dispatcher = std::thread(dispatch_loop, raw);
    *out = sv.release();
    return GPS_OK;
}

gps_status gps_server_set_admission(gps_server* s, uint64_t max_inflight_entries) {
    if (!s) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    s->max_inflight = max_inflight_entries;
    return GPS_OK;
}

gps_status gps_server_submit(gps_server* s, const gps_request* req) {
    if (!s || !req) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->queue.push_back(gps_server::Pending{*req, gps_server::clock::now()});
        ++s->submitted;
    }
    s->cv.notify_all();
    return GPS_OK;
}

int32_t gps_server_poll(gps_server* s, gps_completion* out, int32_t capacity) {
    if (!s || !out || capacity <= 0) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    int32_t n = 0;
    while (n < capacity && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    return n;
}

gps_status gps_server_drain(gps_server* s, double timeout_s) {
    if (!s) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                   [&] { return s->completed == s->submitted; });
    return ok ? GPS_OK : fail(GPS_ERR_DEVICE_TIMEOUT, "requests still in flight after the drain timeout");
}

void gps_server_free(gps_server* s) { delete s; }

}  // extern "C"

// ---------------------------------------------------------------------------------
// headless frame loop (RenderServer::renderFrame, render_server.cu:86-157, without GL)
// ---------------------------------------------------------------------------------
struct gps_frame_loop {
    gps_renderer* r = nullptr;
    dptr<float> color[2], depth[2];
    dptr<float> taa_out;  // TAA writes here, then swaps with the current colour slot
    dptr<uint8_t> u8[2];  // u8 frames alternate, so one can be read back while the next renders
    int cur = 0;          // u8 slot of the last frame
    int last_color = 0;   // colour slot the last frame resolved (and accumulated) into
    cudaStream_t copy = nullptr;      // read-back stream of gps_frame_loop_read_async
    cudaEvent_t framed = nullptr;     // end of the last frame, on the caller's stream
    cudaEvent_t read_done[2] = {nullptr, nullptr};
    bool reading[2] = {false, false};
    int progressive_frames = 0;
    mat4 prev_vp{};
    ~gps_frame_loop() {
        if (copy) cudaStreamSynchronize(copy);
        if (copy) cudaStreamDestroy(copy);
        if (framed) cudaEventDestroy(framed);
        for (cudaEvent_t e : read_done)
            if (e) cudaEventDestroy(e);
    }
};

extern "C" {

gps_status gps_frame_loop_create(gps_renderer* r, gps_frame_loop** out) {
    if (!r || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    auto l = std::make_unique<gps_frame_loop>();
    l->r = r;
    const size_t px = (size_t)r->s.width * r->s.height;
    try {
        for (int i = 0; i < 2; ++i) {
            l->color[i].reset(dev_alloc<float>(px * 3));
            l->depth[i].reset(dev_alloc<float>(px));
            GPS_CUDA(cudaMemset(l->color[i].get(), 0, px * 3 * sizeof(float)));
            GPS_CUDA(cudaMemset(l->depth[i].get(), 0, px * sizeof(float)));
        }
        for (int i = 0; i < 2; ++i) {
            l->u8[i].reset(dev_alloc<uint8_t>(px * 3));
            GPS_CUDA(cudaMemset(l->u8[i].get(), 0, px * 3));
            GPS_CUDA(cudaEventCreateWithFlags(&l->read_done[i], cudaEventDisableTiming));
        }
        l->taa_out.reset(dev_alloc<float>(px * 3));
        GPS_CUDA(cudaStreamCreateWithFlags(&l->copy, cudaStreamNonBlocking));
        GPS_CUDA(cudaEventCreateWithFlags(&l->framed, cudaEventDisableTiming));
    } catch (const CudaError& e) {
        return fail(GPS_ERR_OUT_OF_MEMORY, e.what());
    }
    for (int c = 0; c < 4; ++c) l->prev_vp.c[c] = make_v4(c == 0, c == 1, c == 2, c == 3);
    *out = l.release();
    return GPS_OK;
}

void gps_frame_loop_free(gps_frame_loop* l) { delete l; }

gps_status gps_frame_loop_step(gps_frame_loop* l, const gps_camera* cam, void* stream) {
    if (!l || !cam) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    gps_renderer* r = l->r;
    const int a = cam->frame % 2, b = 1 - a;
    gps_status st = gps_render_frame(r, cam, l->color[a].get(), l->depth[b].get(), stream);
    if (st != GPS_OK) return st;
    const int w = r->s.width, h = r->s.height;
    mat4 view = mat4_from(cam->view), proj = mat4_from(cam->proj);
    const int slot = 1 - l->cur;  // write the other u8 frame; wait if it is still being read back
    if (l->reading[slot]) {
        cudaStreamWaitEvent(as_stream(stream), l->read_done[slot], 0);
        l->reading[slot] = false;
    }
    uint8_t* u8 = l->u8[slot].get();
    r->timer.mark(kStPost, as_stream(stream));
    r->frame_launches += 1;
    r->timer.launches[kStPost] += 1;
    if (r->s.accumulation_mode == GPS_ACCUM_TAA) {
        l->progressive_frames++;
        mat4 model = affine_inverse(view);
        mat4 delta = mat4_mul(mat4_mul(l->prev_vp, model), inverse4(proj));
        launch_taa(u8, l->taa_out.get(), l->color[a].get(), l->color[b].get(), l->depth[a].get(),
                   l->depth[b].get(), delta, 0.9f, w, h, l->progressive_frames, as_stream(stream));
        std::swap(l->color[a], l->taa_out);
    } else {
        if (cam->camera_moved || r->s.accumulation_mode == GPS_ACCUM_NONE) l->progressive_frames = 1;
        else l->progressive_frames++;
        launch_progressive(u8, l->color[a].get(), l->color[b].get(), w, h, l->progressive_frames,
                           as_stream(stream));
    }
    r->timer.mark(-1, as_stream(stream));
    l->cur = slot;
    l->last_color = a;
    l->prev_vp = mat4_mul(proj, view);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_frame_loop_read(gps_frame_loop* l, uint8_t* host_rgb, void* stream) {
    if (!l || !host_rgb) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    const size_t bytes = (size_t)l->r->s.width * l->r->s.height * 3;
    cudaError_t e = cudaMemcpyAsync(host_rgb, l->u8[l->cur].get(), bytes, cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_frame_loop_read_async(gps_frame_loop* l, uint8_t* host_rgb, void* stream) {
    if (!l || !host_rgb) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    const size_t bytes = (size_t)l->r->s.width * l->r->s.height * 3;
    const int slot = l->cur;
    cudaEventRecord(l->framed, as_stream(stream));
    cudaStreamWaitEvent(l->copy, l->framed, 0);
    cudaError_t e = cudaMemcpyAsync(host_rgb, l->u8[slot].get(), bytes, cudaMemcpyDeviceToHost, l->copy);
    if (e == cudaSuccess) e = cudaEventRecord(l->read_done[slot], l->copy);
    l->reading[slot] = true;
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_frame_loop_read_wait(gps_frame_loop* l) {
    if (!l) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaStreamSynchronize(l->copy);
    l->reading[0] = l->reading[1] = false;
    return e == cudaSuccess ? GPS_OK : fail(GPS_ERR_CUDA, cudaGetErrorString(e));
}

gps_status gps_frame_loop_buffers(gps_frame_loop* l, int32_t slot, const uint8_t** d_u8, const float** d_color,
                                  const float** d_depth) {
    if (!l || slot < 0 || slot > 2) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    if (d_u8) *d_u8 = l->u8[l->cur].get();
    if (slot == 2) {
        // resolved colour of the last frame before TAA blended it (TAA mode only)
        if (d_color) *d_color = l->taa_out.get();
        if (d_depth) *d_depth = nullptr;
        return GPS_OK;
    }
    if (d_color) *d_color = l->color[slot].get();
    if (d_depth) *d_depth = l->depth[slot].get();
    return GPS_OK;
}

// ---- evaluation workflow --------------------------------------------------------------

gps_status gps_write_png(const char* path, const uint8_t* host_rgb, int32_t width, int32_t height, int32_t flip_rows) {
    if (!path || !host_rgb || width <= 0 || height <= 0) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    const int rc = write_png(path, host_rgb, width, height, flip_rows != 0);
    if (rc == 3) return fail(GPS_ERR_IO, std::string("cannot write ") + path);
    return rc ? fail(GPS_ERR_INVALID_ARGUMENT, "PNG encoding failed") : GPS_OK;
}

gps_status gps_write_pfm(const char* path, const float* host_rgb, int32_t width, int32_t height) {
    if (!path || !host_rgb || width <= 0 || height <= 0) return fail(GPS_ERR_INVALID_ARGUMENT, "bad argument");
    return write_pfm(path, host_rgb, width, height) ? fail(GPS_ERR_IO, std::string("cannot write ") + path) : GPS_OK;
}

gps_status gps_frame_loop_export_pfm(gps_frame_loop* l, const char* path, void* stream) {
    if (!l || !path) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    const int w = l->r->s.width, h = l->r->s.height;
    const size_t n = (size_t)w * h * 3;
    std::vector<float> host(n);
    cudaError_t e = cudaMemcpyAsync(host.data(), l->color[l->last_color].get(), n * sizeof(float),
                                    cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return fail(GPS_ERR_CUDA, cudaGetErrorString(e));
    // export_pfm_from_buffer: colour / float(numFrames), per component
    const float frames = (float)(l->progressive_frames > 0 ? l->progressive_frames : 1);
    for (size_t i = 0; i < n; ++i) host[i] = host[i] / frames;
    return gps_write_pfm(path, host.data(), w, h);
}

gps_status gps_evaluate(gps_frame_loop* l, const gps_camera_path* path, const char* out_dir,
                        const int32_t* spp_targets, int32_t num_targets, int32_t max_eval_count,
                        int32_t first_frame, int32_t write_pfm_too, int32_t* frames_rendered) {
    if (!l || !path || !out_dir) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    static const int32_t kDefaultTargets[] = {1, 4, 16, 64, 256, 1024};  // main.cu:72
    if (!spp_targets) {
        spp_targets = kDefaultTargets;
        num_targets = 6;
    }
    if (num_targets <= 0 || max_eval_count < 0) return fail(GPS_ERR_INVALID_ARGUMENT, "bad evaluation targets");
    for (int i = 0; i < num_targets; ++i)
        if (spp_targets[i] < 1 || (i > 0 && spp_targets[i] <= spp_targets[i - 1]))
            return fail(GPS_ERR_INVALID_ARGUMENT, "spp targets must be positive and increasing");
    if (!make_dirs(out_dir)) return fail(GPS_ERR_IO, std::string("cannot create ") + out_dir);
    gps_renderer* r = l->r;
    const int w = r->s.width, h = r->s.height;
    std::vector<uint8_t> rgb((size_t)w * h * 3);
    const int cameras = gps_camera_path_count(path);
    int frame = first_frame, rendered = 0;
    // main.cu:95-107: after camera c finishes, the run ends if c >= count - 1 or c >= max_eval_count
    for (int c = 0; c < cameras; ++c) {
        gps_camera_state st;
        gps_status rc = gps_camera_path_get(path, c, &st);
        if (rc != GPS_OK) return rc;
        gps_settings s = r->s;
        int32_t can_override = 0;  // the resolution is fixed once the renderer exists
        std::string name = st.img_name[0] ? std::string(st.img_name) : "cam" + std::to_string(c);
        int next = 0;
        for (int f = 1; f <= spp_targets[num_targets - 1]; ++f, ++frame) {
            gps_camera cam;
            rc = gps_camera_from_state(&st, &s, 0, &can_override, frame, &cam);
            if (rc != GPS_OK) return rc;
            cam.camera_moved = f == 1;
            rc = gps_frame_loop_step(l, &cam, nullptr);
            if (rc != GPS_OK) return rc;
            ++rendered;
            if (f != spp_targets[next]) continue;
            char suffix[16];
            std::snprintf(suffix, sizeof(suffix), "_spp%04d", f);
            const std::string stem = std::string(out_dir) + "/" + name + suffix;
            rc = gps_frame_loop_read(l, rgb.data(), nullptr);
            if (rc == GPS_OK) rc = gps_write_png((stem + ".png").c_str(), rgb.data(), w, h, 1);
            if (rc == GPS_OK && write_pfm_too) rc = gps_frame_loop_export_pfm(l, (stem + ".pfm").c_str(), nullptr);
            if (rc != GPS_OK) return rc;
            ++next;
        }
        if (c >= cameras - 1 || c >= max_eval_count) break;
    }
    if (frames_rendered) *frames_rendered = rendered;
    return GPS_OK;
}

// ---- cameras --------------------------------------------------------------------------
}  // extern "C"

struct gps_camera_path {
    std::vector<CameraState> states;
};

extern "C" {

gps_status gps_camera_path_load(const char* json_path, gps_camera_path** out) {
    if (!json_path || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto p = std::make_unique<gps_camera_path>();
    int rc = load_cameras(json_path, p->states);
    if (rc) return (gps_status)rc;
    *out = p.release();
    return GPS_OK;
}

int32_t gps_camera_path_count(const gps_camera_path* p) { return p ? (int32_t)p->states.size() : 0; }

gps_status gps_camera_path_get(const gps_camera_path* p, int32_t index, gps_camera_state* out) {
    if (!p || !out) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    if (index < 0 || index >= (int32_t)p->states.size()) return fail(GPS_ERR_INVALID_ARGUMENT, "camera index out of range");
    const CameraState& c = p->states[index];
    std::memset(out, 0, sizeof(*out));
    out->id = c.id;
    out->width = c.width;
    out->height = c.height;
    for (int i = 0; i < 3; ++i) out->position[i] = c.position[i];
    for (int i = 0; i < 9; ++i) out->rotation[i] = c.rotation[i];
    out->fx = c.fx;
    out->fy = c.fy;
    std::strncpy(out->img_name, c.img_name.c_str(), sizeof(out->img_name) - 1);
    return GPS_OK;
}

void gps_camera_path_free(gps_camera_path* p) { delete p; }

static void fill_camera(const CameraMatrices& m, int32_t frame, gps_camera* cam) {
    std::memset(cam, 0, sizeof(*cam));
    mat4_to(m.view, cam->view);
    mat4_to(m.proj, cam->proj);
    cam->position[0] = m.position.x;
    cam->position[1] = m.position.y;
    cam->position[2] = m.position.z;
    for (int i = 0; i < 6; ++i) {
        cam->frustum_planes[4 * i] = m.planes[i].x;
        cam->frustum_planes[4 * i + 1] = m.planes[i].y;
        cam->frustum_planes[4 * i + 2] = m.planes[i].z;
        cam->frustum_planes[4 * i + 3] = m.planes[i].w;
    }
    cam->frame = frame;
}

gps_status gps_camera_from_state(const gps_camera_state* state, gps_settings* settings, int32_t override_camera_settings,
                                 int32_t* can_override_resolution, int32_t frame, gps_camera* cam) {
    if (!state || !settings || !cam) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    // basis = transpose(rotation) where rotation's glm columns are the JSON rows
    mat3 rot_glm;
    for (int c = 0; c < 3; ++c) rot_glm.c[c] = make_v3(state->rotation[3 * c], state->rotation[3 * c + 1], state->rotation[3 * c + 2]);
    mat3 basis = transpose(rot_glm);
    float q[4];
    quat_from_basis(basis, q);
    if (!override_camera_settings) {
        int can = can_override_resolution ? *can_override_resolution : 1;
        if (can) {
            float aspect_yx = (float)state->height / (float)state->width;
            float rx = roundf((float)settings->width);
            float ry = roundf((float)settings->width * aspect_yx);
            settings->width = (int)rx;
            settings->height = (int)ry;
            if (can_override_resolution) *can_override_resolution = 0;
        }
        settings->fovy = focal_to_fov_deg(state->fy, state->height);
    }
    float aspect = (float)settings->width / (float)settings->height;
    CameraMatrices m = camera_matrices(make_v3(state->position[0], state->position[1], state->position[2]), q,
                                       settings->fovy, aspect, settings->near_view_plane, settings->far_view_plane);
    fill_camera(m, frame, cam);
    return GPS_OK;
}

gps_status gps_camera_from_pose(const float position[3], const float basis_cols[9], const gps_settings* settings,
                                int32_t frame, gps_camera* cam) {
    if (!position || !basis_cols || !settings || !cam) return fail(GPS_ERR_INVALID_ARGUMENT, "null argument");
    mat3 basis;
    for (int c = 0; c < 3; ++c) basis.c[c] = make_v3(basis_cols[3 * c], basis_cols[3 * c + 1], basis_cols[3 * c + 2]);
    float q[4];
    quat_from_basis(basis, q);
    float aspect = (float)settings->width / (float)settings->height;
    CameraMatrices m = camera_matrices(make_v3(position[0], position[1], position[2]), q, settings->fovy, aspect,
                                       settings->near_view_plane, settings->far_view_plane);
    fill_camera(m, frame, cam);
    return GPS_OK;
}

}  // extern "C"
