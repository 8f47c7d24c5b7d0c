// Headless driver around the reference's own CUDA frame path (test infrastructure only).
//
// This translation unit is compiled by oracle/ref/build_ref.sh against the reference
// sources where they lie; it is never part of the shipped library.  It includes the
// reference's gaussian_point_splatting.cu directly so that the per-frame driver, the
// workload distributor, the Hi-Z chain and the block cull run exactly as the reference
// compiles them, and it adds only what the GL viewer would otherwise provide:
//   * RenderSettings filled from a binary camera file (view, proj, planes, frame index),
//   * the RenderServer post-process step (temporalRender / progressiveRender) with the
//     same colour/depth ping-pong as render_server.cu:86-157,
//   * dumps of every observable per-frame buffer as .npy files,
//   * a known-answer mode that evaluates the reference's device RNG / packing helpers.
//
// Modes:
//   ref_harness render <ply> <outdir> <camfile> [options]
//   ref_harness kat <outdir>
//   ref_harness camera <cameras.json> <outdir> <width> <height> <fovy> <near> <far> <override>
#define private public
#define protected public
#include "core/rendering/passes/gaussian_point_splatting.cu"
#undef private
#undef protected

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include <chrono>

// ---------------------------------------------------------------------------------
// .npy writer
// ---------------------------------------------------------------------------------
static void write_npy(const std::string& path, const void* data, size_t count, const char* descr,
                      size_t elem_size, const std::vector<size_t>& shape_in = {}) {
    std::vector<size_t> shape = shape_in.empty() ? std::vector<size_t>{count} : shape_in;
    std::string dict = "{'descr': '";
    dict += descr;
    dict += "', 'fortran_order': False, 'shape': (";
    for (size_t i = 0; i < shape.size(); ++i) {
        dict += std::to_string(shape[i]);
        if (shape.size() == 1 || i + 1 < shape.size()) dict += ",";
        if (i + 1 < shape.size()) dict += " ";
    }
    dict += "), }";
    size_t total = 10 + dict.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    dict.append(pad, ' ');
    dict += "\n";
    std::ofstream f(path, std::ios::binary);
    f.write("\x93NUMPY\x01\x00", 8);
    uint16_t hl = (uint16_t)dict.size();
    f.write(reinterpret_cast<const char*>(&hl), 2);
    f.write(dict.data(), dict.size());
    f.write(reinterpret_cast<const char*>(data), count * elem_size);
}

template <typename T>
static std::vector<T> d2h(const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Order-independent 64-bit checksum of a u64 buffer (sum of mixed (value, index) pairs).
static uint64_t buffer_checksum(const std::vector<uint64_t>& v) {
    uint64_t s = 0;
    for (size_t i = 0; i < v.size(); ++i) s += splitmix64(v[i] ^ (uint64_t(i) * 0xD1B54A32D192ED03ull));
    return s;
}

struct CamRecord {  // binary layout of one frame in the camera file (all little-endian)
    float view[16];
    float proj[16];
    float position[3];
    float planes[24];
    int32_t frame;
    int32_t camera_moved;
};

static glm::mat4 to_mat4(const float* m) {
    glm::mat4 r;
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) r[c][rr] = m[c * 4 + rr];
    return r;
}

static void put_mat4(std::vector<float>& out, const glm::mat4& m) {
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) out.push_back(m[c][r]);
}

// temporalRender (post_processing_kernels.cuh:222-285) blends each pixel in place while its
// neighbours read the same buffer for the 3x3 clamp, so its output depends on thread order.
// This runs the UNMODIFIED kernel so that no read can see a blended value: nine launches, one
// per pixel class (x mod 3, y mod 3), each on a fresh copy of the unblended colour buffer and
// with NaN current depth everywhere outside the class.  A NaN depth reprojects to NaN, fails
// the kernel's bounds test and writes the pixel's own unchanged colour back; pixels of one
// class are at least 3 apart, so none reads another's blended value.  The class pixels of the
// nine launches are assembled into the colour buffer and the u8 image.
static void temporal_render_race_free(unsigned char* d_u8, glm::vec3* d_cur, const glm::vec3* d_prev, const float* d_cur_depth,
                                      const float* d_prev_depth, const glm::mat4& reprojection, int W, int H, int frame_number) {
    const size_t npx = size_t(W) * H;
    std::vector<glm::vec3> pre(npx), out(npx);
    std::vector<float> depth(npx), masked(npx);
    std::vector<unsigned char> u8(npx * 3), u8_out(npx * 3);
    cudaMemcpy(pre.data(), d_cur, npx * sizeof(glm::vec3), cudaMemcpyDeviceToHost);
    cudaMemcpy(depth.data(), d_cur_depth, npx * sizeof(float), cudaMemcpyDeviceToHost);
    float* d_masked = nullptr;
    cudaMalloc(&d_masked, npx * sizeof(float));
    dim3 block(256), grid((unsigned)((npx + 255) / 256));
    for (int cls = 0; cls < 9; ++cls) {
        const int cx = cls % 3, cy = cls / 3;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                masked[size_t(y) * W + x] = (x % 3 == cx && y % 3 == cy) ? depth[size_t(y) * W + x] : NAN;
        cudaMemcpy(d_masked, masked.data(), npx * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d_cur, pre.data(), npx * sizeof(glm::vec3), cudaMemcpyHostToDevice);
        temporalRender<<<grid, block>>>(d_u8, d_cur, d_prev, d_masked, d_prev_depth, reprojection, 0.9f, W, H, frame_number);
        std::vector<glm::vec3> got(npx);
        cudaMemcpy(got.data(), d_cur, npx * sizeof(glm::vec3), cudaMemcpyDeviceToHost);
        cudaMemcpy(u8.data(), d_u8, npx * 3, cudaMemcpyDeviceToHost);
        for (int y = cy; y < H; y += 3)
            for (int x = cx; x < W; x += 3) {
                const size_t i = size_t(y) * W + x;
                out[i] = got[i];
                u8_out[3 * i + 0] = u8[3 * i + 0];
                u8_out[3 * i + 1] = u8[3 * i + 1];
                u8_out[3 * i + 2] = u8[3 * i + 2];
            }
    }
    cudaMemcpy(d_cur, out.data(), npx * sizeof(glm::vec3), cudaMemcpyHostToDevice);
    cudaMemcpy(d_u8, u8_out.data(), npx * 3, cudaMemcpyHostToDevice);
    cudaFree(d_masked);
}

static int run_render(int argc, char** argv) {
    if (argc < 5) { fprintf(stderr, "usage: render <ply> <outdir> <camfile> [opts]\n"); return 2; }
    std::string ply = argv[2], outdir = argv[3], camfile = argv[4];
    RenderSettings s;
    s.statistics = new Statistics();
    s.model_path = ply;
    s.render_gui = false;
    int frames_to_dump = 1 << 30;
    bool dump_full = true, timing = false, dump_post = true;
    int warmup = 0;
    bool taa_race_free = false;
    for (int i = 5; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--res") { s.resolution.x = atoi(argv[++i]); s.resolution.y = atoi(argv[++i]); }
        else if (a == "--ss") s.supersampling_factor = atoi(argv[++i]);
        else if (a == "--spp") s.render_pass_count = atoi(argv[++i]);
        else if (a == "--max-points") s.max_number_of_points = atoi(argv[++i]);
        else if (a == "--near") s.near_view_plane = (float)atof(argv[++i]);
        else if (a == "--far") s.far_view_plane = (float)atof(argv[++i]);
        else if (a == "--fovy") s.fovy = (float)atof(argv[++i]);
        else if (a == "--one-point-per-thread") s.reduce_point_count = false;
        else if (a == "--disable-hierarchical-culling") s.enable_hierarchical_culling = false;
        else if (a == "--fully-disable-hierarchical-culling") s.fully_disable_hierarchical_culling = true;
        else if (a == "--disable-occlusion-culling") s.enable_occlusion_culling = false;
        else if (a == "--cull-small") s.cull_small_gaussians = true;
        else if (a == "--biased") s.use_unbiased_2d_splatting = false;
        else if (a == "--min-reduce") s.occlusion_culling_min_reduce_count = atoi(argv[++i]);
        else if (a == "--background") { s.backgroundColor.x = (float)atof(argv[++i]); s.backgroundColor.y = (float)atof(argv[++i]); s.backgroundColor.z = (float)atof(argv[++i]); }
        else if (a == "--taa") s.accumulationMode = AccumulationMode::TAA;
        else if (a == "--taa-race-free") { s.accumulationMode = AccumulationMode::TAA; taa_race_free = true; }
        else if (a == "--no-accumulation") s.accumulationMode = AccumulationMode::None;
        else if (a == "--sort-morton-order") s.sort_morton_order = true;
        else if (a == "--immediate-threshold") s.immediate_splat_threshold = atoi(argv[++i]);
        else if (a == "--dump-frames") frames_to_dump = atoi(argv[++i]);
        else if (a == "--checksum-only") dump_full = false;
        else if (a == "--no-post-dump") dump_post = false;
        else if (a == "--time") timing = true;
        else if (a == "--warmup") warmup = atoi(argv[++i]);
        else { fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }

    std::vector<CamRecord> cams;
    {
        std::ifstream f(camfile, std::ios::binary);
        if (!f) { fprintf(stderr, "cannot open %s\n", camfile.c_str()); return 2; }
        CamRecord r;
        while (f.read(reinterpret_cast<char*>(&r), sizeof(r))) cams.push_back(r);
    }
    if (cams.empty()) { fprintf(stderr, "no camera records\n"); return 2; }

    auto t_load0 = std::chrono::steady_clock::now();
    GaussianPointSplatting* gps = new GaussianPointSplatting(s);
    cudaDeviceSynchronize();
    auto t_load1 = std::chrono::steady_clock::now();
    fprintf(stderr, "reference scene ready in %.2f s (N=%d)\n",
            std::chrono::duration<double>(t_load1 - t_load0).count(), gps->numGaussians);

    // host scene exactly as the reference loaded (and possibly reordered) it
    write_npy(outdir + "/scene_cpu.npy", gps->gaussians.data(), gps->gaussians.size() * 59, "<f4", 4,
              {gps->gaussians.size(), 59});
#ifdef USE_COMPRESSED_GAUSSIANS
    {
        auto& sc = gps->gpuGaussianScene;
        size_t n = sc.numGaussians;
        std::vector<uint32_t> geom = d2h(reinterpret_cast<uint32_t*>(sc.d_gaussians), n * 4);
        std::vector<uint8_t> op = d2h(sc.d_opacities, n);
        std::vector<uint8_t> shs = d2h(reinterpret_cast<uint8_t*>(sc.d_shs), n * sizeof(CompactSH));
        write_npy(outdir + "/scene_geom.npy", geom.data(), geom.size(), "<u4", 4, {n, 4});
        write_npy(outdir + "/scene_opacity.npy", op.data(), op.size(), "|u1", 1);
        write_npy(outdir + "/scene_compact_sh.npy", shs.data(), shs.size(), "|u1", 1, {n, sizeof(CompactSH)});
        write_npy(outdir + "/scene_bounds.npy", &sc.sceneBounds, sizeof(GaussianSceneBounds) / 4, "<f4", 4);
    }
#endif
    // The reference never initialises its Hi-Z buffer before the first frame; start it at
    // +inf ("nothing occluded") so that frame 1 is defined.
    {
        std::vector<float> inf(gps->depthMipChain.view.mip_size, INFINITY);
        cudaMemcpy(gps->depthMipChain.view.d_mip, inf.data(), inf.size() * sizeof(float), cudaMemcpyHostToDevice);
    }

    const int W = s.resolution.x, H = s.resolution.y;
    glm::vec3* d_color[2];
    float* d_depth[2];
    unsigned char* d_u8 = nullptr;
    for (int i = 0; i < 2; ++i) {
        cudaMalloc(&d_color[i], size_t(W) * H * sizeof(glm::vec3));
        cudaMalloc(&d_depth[i], size_t(W) * H * sizeof(float));
        cudaMemset(d_color[i], 0, size_t(W) * H * sizeof(glm::vec3));
        cudaMemset(d_depth[i], 0, size_t(W) * H * sizeof(float));
    }
    cudaMalloc(&d_u8, size_t(W) * H * 3);
    int numProgressiveFrames = 0;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    std::vector<float> frame_ms;

    for (size_t fi = 0; fi < cams.size(); ++fi) {
        const CamRecord& c = cams[fi];
        s.cameraViewMatrix = to_mat4(c.view);
        s.cameraProjectionMatrix = to_mat4(c.proj);
        s.cameraPosition = glm::vec3(c.position[0], c.position[1], c.position[2]);
        for (int p = 0; p < 6; ++p)
            s.frustumPlanes[p] = glm::vec4(c.planes[p * 4 + 0], c.planes[p * 4 + 1], c.planes[p * 4 + 2], c.planes[p * 4 + 3]);
        s.frame = c.frame;
        s.cameraMoved = c.camera_moved != 0;
        s.copyToGPU();

        // RenderServer::renderFrame (render_server.cu:86-157), minus GL interop.
        int a = s.frame % 2;
        int b = 1 - a;
        cudaEventRecord(ev0);
        gps->render(d_color[a], d_depth[b], s);
        std::vector<float> pre_post;
        if (dump_full && (int)fi < frames_to_dump) pre_post = d2h(reinterpret_cast<float*>(d_color[a]), size_t(W) * H * 3);
        {
            dim3 blockSize(256);
            dim3 gridSize((W * H + blockSize.x - 1) / blockSize.x);
            if (s.accumulationMode == AccumulationMode::TAA) {
                numProgressiveFrames++;
                glm::mat4 modelMat = glm::affineInverse(s.cameraViewMatrix);
                glm::mat4 deltaMatrix = s.previousViewProjectionMatrix * modelMat * glm::inverse(s.cameraProjectionMatrix);
                if (taa_race_free)
                    temporal_render_race_free(d_u8, d_color[a], d_color[b], d_depth[a], d_depth[b], deltaMatrix, W, H,
                                              numProgressiveFrames);
                else
                    temporalRender<<<gridSize, blockSize>>>(d_u8, d_color[a], d_color[b], d_depth[a], d_depth[b],
                                                            deltaMatrix, 0.9f, W, H, numProgressiveFrames);
            } else {
                if (s.cameraMoved || s.accumulationMode == AccumulationMode::None) numProgressiveFrames = 1;
                else numProgressiveFrames++;
                progressiveRender<<<gridSize, blockSize>>>(d_u8, d_color[a], d_color[b], W, H, numProgressiveFrames);
            }
        }
        cudaEventRecord(ev1);
        cudaEventSynchronize(ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        if ((int)fi >= warmup) frame_ms.push_back(ms);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 3; }

        // main.cu:176 — previous view-projection for the next frame's TAA
        glm::mat4 vp_prev = s.cameraProjectionMatrix * s.cameraViewMatrix;

        if ((int)fi < frames_to_dump) {
            char pre[512];
            snprintf(pre, sizeof(pre), "%s/f%03zu_", outdir.c_str(), fi);
            std::string P(pre);
            // derived per-frame constants, computed exactly as render() does (gps.cu:605-615)
            {
                auto vMatrix = s.cameraViewMatrix;
                auto camMatrix = glm::affineInverse(vMatrix);
                auto vpMatrix = s.cameraProjectionMatrix * vMatrix;
                float r = s.get_aspectXY();
                float t_f_y = glm::tan(glm::radians(s.fovy) * 0.5f);
                float fovx = 2.0f * glm::atan(t_f_y * r);
                float t_f_x = glm::tan(fovx * 0.5f);
                glm::vec2 tan_fov{ t_f_x, t_f_y };
                glm::vec2 focal{ s.resolution.x * s.supersampling_factor / (2.0f * tan_fov.x),
                                 s.resolution.y * s.supersampling_factor / (2.0f * tan_fov.y) };
                std::vector<float> dv;
                put_mat4(dv, vpMatrix);
                put_mat4(dv, camMatrix);
                dv.push_back(tan_fov.x); dv.push_back(tan_fov.y);
                dv.push_back(focal.x); dv.push_back(focal.y);
                glm::mat4 modelMat = glm::affineInverse(s.cameraViewMatrix);
                put_mat4(dv, s.previousViewProjectionMatrix * modelMat * glm::inverse(s.cameraProjectionMatrix));
                write_npy(P + "derived.npy", dv.data(), dv.size(), "<f4", 4);
            }
            uint64_t* cur = gps->get_current_image_buffer(s.frame);
            std::vector<uint64_t> buf = d2h(cur, gps->imageBufferSize);
            uint64_t cs = buffer_checksum(buf);
            write_npy(P + "buffer_checksum.npy", &cs, 1, "<u8", 8);
            if (dump_full) write_npy(P + "buffer.npy", buf.data(), buf.size(), "<u8", 8);

            std::vector<float> img = d2h(reinterpret_cast<float*>(d_color[a]), size_t(W) * H * 3);
            std::vector<float> dep = d2h(d_depth[b], size_t(W) * H);
            write_npy(P + "image.npy", img.data(), img.size(), "<f4", 4, {size_t(H), size_t(W), 3});
            if (!pre_post.empty())
                write_npy(P + "image_pre_post.npy", pre_post.data(), pre_post.size(), "<f4", 4, {size_t(H), size_t(W), 3});
            write_npy(P + "depth.npy", dep.data(), dep.size(), "<f4", 4, {size_t(H), size_t(W)});
            if (dump_post) {
                std::vector<uint8_t> u8 = d2h(d_u8, size_t(W) * H * 3);
                write_npy(P + "post_u8.npy", u8.data(), u8.size(), "|u1", 1, {size_t(H), size_t(W), 3});
            }
            std::vector<float> mip = d2h(gps->depthMipChain.view.d_mip, gps->depthMipChain.view.mip_size);
            write_npy(P + "hiz.npy", mip.data(), mip.size(), "<f4", 4);

            WorkloadDistributor* wd = gps->pointsWorkload;
            size_t N = gps->numGaussians;
            std::vector<uint32_t> offs = d2h(wd->weights.device_data(), N);
            std::vector<uint32_t> mcur = d2h(wd->getWeightsMaskCurrent().device_data(), (N + 31) / 32);
            std::vector<uint32_t> mprev = d2h(wd->getWeightsMaskPrevious().device_data(), (N + 31) / 32);
            uint32_t P_pts = wd->num_samples;
            std::vector<uint32_t> idx = d2h(wd->indices.device_data(), P_pts);
            write_npy(P + "offsets.npy", offs.data(), offs.size(), "<u4", 4);
            // after build() the iteration counter has advanced: "previous" is the mask the last pass wrote
            write_npy(P + "mask_last.npy", mprev.data(), mprev.size(), "<u4", 4);
            write_npy(P + "mask_other.npy", mcur.data(), mcur.size(), "<u4", 4);
            write_npy(P + "indices.npy", idx.data(), idx.size(), "<u4", 4);
            std::vector<float> col = d2h(reinterpret_cast<float*>(gps->gpuGaussianScene.d_colors), N * 3);
            write_npy(P + "colors.npy", col.data(), col.size(), "<f4", 4, {N, 3});
            int32_t st[6] = { s.statistics->numPointsOne, s.statistics->numPointsTwo,
                              s.statistics->numGaussiansOne, s.statistics->numGaussiansTwo,
                              (int32_t)P_pts, (int32_t)wd->iteration };
            write_npy(P + "stats.npy", st, 6, "<i4", 4);
            if (gps->gaussianBVH.dev.d_culledMask) {
                auto& dv = gps->gaussianBVH.dev;
                std::vector<uint32_t> cm = d2h(dv.d_culledMask, dv.culledMaskSize);
                write_npy(P + "culled.npy", cm.data(), cm.size(), "<u4", 4);
            }
        }
        s.previousViewProjectionMatrix = vp_prev;
    }
    if (timing) {
        double sum = 0;
        for (float m : frame_ms) sum += m;
        printf("{\"frames\": %zu, \"ms_per_frame\": %.4f}\n", frame_ms.size(), frame_ms.empty() ? 0.0 : sum / frame_ms.size());
    }
    // static scene tables that never change per frame
    {
        if (gps->gaussianBVH.dev.d_nodes) {
            auto& dv = gps->gaussianBVH.dev;
            std::vector<float> nodes = d2h(reinterpret_cast<float*>(dv.d_nodes), size_t(dv.nodeCount) * 8);
            write_npy(outdir + "/bvh_nodes.npy", nodes.data(), nodes.size(), "<f4", 4, {size_t(dv.nodeCount), 8});
            uint32_t gpb = dv.gaussians_per_block;
            write_npy(outdir + "/bvh_gpb.npy", &gpb, 1, "<u4", 4);
        }
    }
    delete gps;
    return 0;
}

// ---------------------------------------------------------------------------------
// Per-Gaussian intermediates of the reference's preprocess for a list of Gaussian ids
// (stage-by-stage debugging of parity): 48 floats per id, see probe layout below.
// ---------------------------------------------------------------------------------
constexpr int kProbeFloats = 48;

__global__ void probe_kernel(GPUGaussianScene scene, const uint32_t* ids, int m, glm::mat4 vp, glm::mat4 v,
                             glm::mat4 cam, glm::vec2 tan_fov, glm::vec2 focal, int upw, int uph, int ss,
                             int frame_seed, float* out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    uint32_t idx = ids[t];
    float* o = out + (size_t)t * kProbeFloats;
    for (int i = 0; i < kProbeFloats; ++i) o[i] = 0.0f;
    GaussianGeometry gg = scene.get_gaussian_transform(idx);
    o[0] = gg.mean.x; o[1] = gg.mean.y; o[2] = gg.mean.z;
    o[3] = gg.quat.x; o[4] = gg.quat.y; o[5] = gg.quat.z; o[6] = gg.quat.w;
    o[7] = gg.scale.x; o[8] = gg.scale.y; o[9] = gg.scale.z;
    float opacity = scene.get_opacity(idx);
    o[10] = opacity;
    glm::mat3 cov = CudaMath::scale_rot_to_cov(gg.scale, gg.quat);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) o[16 + 3 * c + r] = cov[c][r];
    GaussianGeometry g2;
    glm::vec4 proj_mean;
    glm::vec2 pixel_mean;
    glm::vec3 cov2d;
    glm::ivec2 mn, mx;
    float det = 0, view_z = 0;
    bool ok = loadAndTransformGaussian(scene, idx, vp, v, tan_fov, focal, upw, uph, ss, g2, proj_mean, pixel_mean, cov2d,
                                       mn, mx, det, view_z);
    o[11] = view_z;
    o[12] = proj_mean.x; o[13] = proj_mean.y; o[14] = proj_mean.z; o[15] = proj_mean.w;
    o[25] = cov2d.x; o[26] = cov2d.y; o[27] = cov2d.z;
    o[28] = det;
    o[29] = pixel_mean.x; o[30] = pixel_mean.y;
    o[31] = (float)mn.x; o[32] = (float)mn.y; o[33] = (float)mx.x; o[34] = (float)mx.y;
    o[47] = ok ? 1.0f : 0.0f;
    if (!ok) return;
    constexpr float TWO_PI = 2.0f * 3.14159265358979323846f;
    float s_det = __fsqrt_rn(det);
    float dl = Random::dilog(opacity);
    float importance = TWO_PI * s_det * dl;
    o[35] = s_det;
    o[36] = dl;
    o[37] = importance;
    uint2 seed = Random::makeSeed(idx, frame_seed);
    uint32_t np = Random::poisson(seed, importance);
    o[38] = (float)np;
    float K = (float)(ss * ss);
    if (K > 1) np = Random::stochastic_round(static_cast<float>(np) / K, Random::pcg2d(seed).x);
    o[39] = (float)np;
    glm::vec3 campos = glm::vec3(cam[3]);
    glm::vec3 col = scene.get_sh(idx, 4, gg.mean, campos);
    o[40] = col.x; o[41] = col.y; o[42] = col.z;
    glm::vec3 conic = CudaMath::conic(cov2d, 1.0f / det);
    o[43] = conic.x; o[44] = conic.y; o[45] = conic.z;
    o[46] = cov2d.y / __fsqrt_rn(cov2d.x);
}

static int run_probe(int argc, char** argv) {
    if (argc < 6) { fprintf(stderr, "usage: probe <ply> <outdir> <camfile> <ids.u32> [opts]\n"); return 2; }
    RenderSettings s;
    s.statistics = new Statistics();
    s.model_path = argv[2];
    std::string outdir = argv[3];
    std::vector<CamRecord> cams;
    {
        std::ifstream f(argv[4], std::ios::binary);
        CamRecord r;
        while (f.read(reinterpret_cast<char*>(&r), sizeof(r))) cams.push_back(r);
    }
    std::vector<uint32_t> ids;
    {
        std::ifstream f(argv[5], std::ios::binary);
        uint32_t v;
        while (f.read(reinterpret_cast<char*>(&v), 4)) ids.push_back(v);
    }
    for (int i = 6; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--res") { s.resolution.x = atoi(argv[++i]); s.resolution.y = atoi(argv[++i]); }
        else if (a == "--ss") s.supersampling_factor = atoi(argv[++i]);
        else if (a == "--fovy") s.fovy = (float)atof(argv[++i]);
        else if (a == "--fully-disable-hierarchical-culling") s.fully_disable_hierarchical_culling = true;
    }
    if (cams.empty() || ids.empty()) return 2;
    GaussianPointSplatting* gps = new GaussianPointSplatting(s);
    const CamRecord& c = cams[0];
    s.cameraViewMatrix = to_mat4(c.view);
    s.cameraProjectionMatrix = to_mat4(c.proj);
    auto vMatrix = s.cameraViewMatrix;
    auto camMatrix = glm::affineInverse(vMatrix);
    auto vpMatrix = s.cameraProjectionMatrix * vMatrix;
    float r = s.get_aspectXY();
    float t_f_y = glm::tan(glm::radians(s.fovy) * 0.5f);
    float fovx = 2.0f * glm::atan(t_f_y * r);
    float t_f_x = glm::tan(fovx * 0.5f);
    glm::vec2 tan_fov{ t_f_x, t_f_y };
    glm::vec2 focal{ s.resolution.x * s.supersampling_factor / (2.0f * tan_fov.x),
                     s.resolution.y * s.supersampling_factor / (2.0f * tan_fov.y) };
    uint32_t* d_ids;
    float* d_out;
    cudaMalloc(&d_ids, ids.size() * 4);
    cudaMalloc(&d_out, ids.size() * kProbeFloats * 4);
    cudaMemcpy(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice);
    int m = (int)ids.size();
    probe_kernel<<<(m + 127) / 128, 128>>>(gps->gpuGaussianScene, d_ids, m, vpMatrix, vMatrix, camMatrix, tan_fov, focal,
                                          s.resolution.x * s.supersampling_factor, s.resolution.y * s.supersampling_factor,
                                          s.supersampling_factor, 4 * c.frame, d_out);
    cudaDeviceSynchronize();
    std::vector<float> out = d2h(d_out, ids.size() * kProbeFloats);
    write_npy(outdir + "/probe.npy", out.data(), out.size(), "<f4", 4, {ids.size(), (size_t)kProbeFloats});
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 3; }
    return 0;
}

// ---------------------------------------------------------------------------------
// One point's samples through the reference's device functions (loadAndTransformGaussian,
// Random::pcg2d / correctedBoxMuller, the splatGaussianPoint position expression), with the
// intermediates written out: 12 floats per sample (parity debugging).
// ---------------------------------------------------------------------------------
__global__ void sample_probe_kernel(GPUGaussianScene scene, uint32_t g, uint32_t point, int frame_seed, glm::mat4 vp,
                                    glm::mat4 v, glm::vec2 tan_fov, glm::vec2 focal, int upw, int uph, int ss,
                                    int samples, float* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    GaussianGeometry gg;
    glm::vec4 proj_mean;
    glm::vec2 pixel_mean;
    glm::vec3 cov2d;
    glm::ivec2 mn, mx;
    float det = 0, view_z = 0;
    if (!loadAndTransformGaussian(scene, g, vp, v, tan_fov, focal, upw, uph, ss, gg, proj_mean, pixel_mean, cov2d, mn, mx,
                                  det, view_z))
        return;
    const float opacity = scene.get_opacity(g);
    const float c0 = __fsqrt_rn(cov2d.x);
    const float c1 = cov2d.y / c0;
    const float c2 = __fsqrt_rn(cov2d.z - c1 * c1);
    uint2 seed = Random::makeSeed(point, frame_seed);
    for (int q = 0; q < samples; ++q) {
        float2 u = Random::pcg2d(seed);
        float2 xy = Random::correctedBoxMuller(u.x, u.y, opacity);
        glm::vec2 pixel(pixel_mean.x + c0 * xy.x, pixel_mean.y + c1 * xy.x + c2 * xy.y);
        float* o = out + 12 * q;
        o[0] = u.x; o[1] = u.y; o[2] = xy.x; o[3] = xy.y; o[4] = pixel.x; o[5] = pixel.y;
        o[6] = pixel_mean.x; o[7] = pixel_mean.y; o[8] = c0; o[9] = c1; o[10] = c2; o[11] = opacity;
    }
}

static int run_sample_probe(int argc, char** argv) {
    if (argc < 8) { fprintf(stderr, "usage: sampleprobe <ply> <outdir> <camfile> <gaussian> <point> <frame_seed> [opts]\n"); return 2; }
    RenderSettings s;
    s.statistics = new Statistics();
    s.model_path = argv[2];
    std::string outdir = argv[3];
    std::vector<CamRecord> cams;
    {
        std::ifstream f(argv[4], std::ios::binary);
        CamRecord r;
        while (f.read(reinterpret_cast<char*>(&r), sizeof(r))) cams.push_back(r);
    }
    const uint32_t g = (uint32_t)strtoul(argv[5], nullptr, 10);
    const uint32_t point = (uint32_t)strtoul(argv[6], nullptr, 10);
    const int frame_seed = atoi(argv[7]);
    for (int i = 8; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--res") { s.resolution.x = atoi(argv[++i]); s.resolution.y = atoi(argv[++i]); }
        else if (a == "--ss") s.supersampling_factor = atoi(argv[++i]);
        else if (a == "--spp") s.render_pass_count = atoi(argv[++i]);
        else if (a == "--fovy") s.fovy = (float)atof(argv[++i]);
    }
    if (cams.empty()) return 2;
    GaussianPointSplatting* gps = new GaussianPointSplatting(s);
    if (g >= (uint32_t)gps->numGaussians) { fprintf(stderr, "gaussian out of range\n"); return 2; }
    const CamRecord& c = cams[0];
    s.cameraViewMatrix = to_mat4(c.view);
    s.cameraProjectionMatrix = to_mat4(c.proj);
    auto vMatrix = s.cameraViewMatrix;
    auto vpMatrix = s.cameraProjectionMatrix * vMatrix;
    float r = s.get_aspectXY();
    float t_f_y = glm::tan(glm::radians(s.fovy) * 0.5f);
    float fovx = 2.0f * glm::atan(t_f_y * r);
    float t_f_x = glm::tan(fovx * 0.5f);
    glm::vec2 tan_fov{ t_f_x, t_f_y };
    glm::vec2 focal{ s.resolution.x * s.supersampling_factor / (2.0f * tan_fov.x),
                     s.resolution.y * s.supersampling_factor / (2.0f * tan_fov.y) };
    const int samples = s.render_pass_count * s.supersampling_factor * s.supersampling_factor;
    float* d_out;
    cudaMalloc(&d_out, sizeof(float) * 12 * samples);
    cudaMemset(d_out, 0, sizeof(float) * 12 * samples);
    sample_probe_kernel<<<1, 32>>>(gps->gpuGaussianScene, g, point, frame_seed, vpMatrix, vMatrix, tan_fov, focal,
                                   s.resolution.x * s.supersampling_factor, s.resolution.y * s.supersampling_factor,
                                   s.supersampling_factor, samples, d_out);
    cudaDeviceSynchronize();
    std::vector<float> out = d2h(d_out, (size_t)12 * samples);
    write_npy(outdir + "/sample_probe.npy", out.data(), out.size(), "<f4", 4, {(size_t)samples, 12});
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 3; }
    return 0;
}

// ---------------------------------------------------------------------------------
// The reference's own splat kernel (splatGaussianPointsKernel, unmodified) over a given
// point -> Gaussian index array and frame seed, into a freshly cleared buffer: where exactly
// the reference puts the samples of chosen points (parity debugging).  Writes the entries that
// differ from the clear value as (index, value) pairs.
// ---------------------------------------------------------------------------------
static int run_splat_points(int argc, char** argv) {
    if (argc < 7) { fprintf(stderr, "usage: splatpoints <ply> <outdir> <camfile> <indices.u32> <frame_seed> [opts]\n"); return 2; }
    RenderSettings s;
    s.statistics = new Statistics();
    s.model_path = argv[2];
    std::string outdir = argv[3];
    std::vector<CamRecord> cams;
    {
        std::ifstream f(argv[4], std::ios::binary);
        CamRecord r;
        while (f.read(reinterpret_cast<char*>(&r), sizeof(r))) cams.push_back(r);
    }
    std::vector<uint32_t> ids;
    {
        std::ifstream f(argv[5], std::ios::binary);
        uint32_t v;
        while (f.read(reinterpret_cast<char*>(&v), 4)) ids.push_back(v);
    }
    const int frame_seed = atoi(argv[6]);
    for (int i = 7; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--res") { s.resolution.x = atoi(argv[++i]); s.resolution.y = atoi(argv[++i]); }
        else if (a == "--ss") s.supersampling_factor = atoi(argv[++i]);
        else if (a == "--spp") s.render_pass_count = atoi(argv[++i]);
        else if (a == "--fovy") s.fovy = (float)atof(argv[++i]);
        else if (a == "--near") s.near_view_plane = (float)atof(argv[++i]);
        else if (a == "--far") s.far_view_plane = (float)atof(argv[++i]);
    }
    if (cams.empty() || ids.empty()) return 2;
    GaussianPointSplatting* gps = new GaussianPointSplatting(s);
    if (ids.size() > 0) {
        uint32_t mx = 0;
        for (uint32_t v : ids) mx = v > mx ? v : mx;
        if (mx >= (uint32_t)gps->numGaussians) { fprintf(stderr, "index %u out of range\n", mx); return 2; }
    }
    const CamRecord& c = cams[0];
    s.cameraViewMatrix = to_mat4(c.view);
    s.cameraProjectionMatrix = to_mat4(c.proj);
    auto vMatrix = s.cameraViewMatrix;
    auto camMatrix = glm::affineInverse(vMatrix);
    auto vpMatrix = s.cameraProjectionMatrix * vMatrix;
    float r = s.get_aspectXY();
    float t_f_y = glm::tan(glm::radians(s.fovy) * 0.5f);
    float fovx = 2.0f * glm::atan(t_f_y * r);
    float t_f_x = glm::tan(fovx * 0.5f);
    glm::vec2 tan_fov{ t_f_x, t_f_y };
    glm::vec2 focal{ s.resolution.x * s.supersampling_factor / (2.0f * tan_fov.x),
                     s.resolution.y * s.supersampling_factor / (2.0f * tan_fov.y) };
    const int upw = s.resolution.x * s.supersampling_factor, uph = s.resolution.y * s.supersampling_factor;
    const size_t tiles = size_t((upw + 63) / 64) * size_t((uph + 63) / 64);
    const size_t entries = tiles * 4096 * size_t(s.render_pass_count);
    const uint64_t clear = 0xFFFFFFF000000000ull;
    std::vector<uint64_t> init(entries, clear);
    uint64_t* d_buf;
    uint32_t* d_ids;
    cudaMalloc(&d_buf, entries * 8);
    cudaMalloc(&d_ids, ids.size() * 4);
    cudaMemcpy(d_buf, init.data(), entries * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice);
    const int n = (int)ids.size();
    splatGaussianPointsKernel<<<(n + 255) / 256, 256>>>(gps->gpuGaussianScene, d_ids, d_buf, vpMatrix, vMatrix, camMatrix,
                                                       tan_fov, focal, upw, uph, s.render_pass_count, frame_seed, n,
                                                       s.near_view_plane, s.far_view_plane, s.use_unbiased_2d_splatting,
                                                       s.reduce_point_count, s.supersampling_factor);
    cudaDeviceSynchronize();
    std::vector<uint64_t> buf = d2h(d_buf, entries);
    std::vector<uint64_t> pairs;
    for (size_t i = 0; i < entries; ++i)
        if (buf[i] != clear) { pairs.push_back(i); pairs.push_back(buf[i]); }
    write_npy(outdir + "/splat_points.npy", pairs.data(), pairs.size(), "<u8", 8, {pairs.size() / 2, 2});
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 3; }
    return 0;
}

// ---------------------------------------------------------------------------------
// Known-answer vectors from the reference's device helpers
// ---------------------------------------------------------------------------------
__global__ void kat_kernel(const uint32_t* idx, const uint32_t* frame, const float* fin, int n,
                           uint32_t* seeds, uint32_t* pcg, float* pcgf, float* dl, float* idl,
                           float* bm, float* cbm, uint32_t* pois, int* sround) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint2 s = Random::makeSeed(idx[i], frame[i]);
    seeds[2 * i] = s.x; seeds[2 * i + 1] = s.y;
    uint2 q = Random::pcg2d_uint(s);
    pcg[2 * i] = q.x; pcg[2 * i + 1] = q.y;
    uint2 st = s;
    float2 u = Random::pcg2d(st);
    pcgf[2 * i] = u.x; pcgf[2 * i + 1] = u.y;
    float x = fin[i];
    dl[i] = Random::dilog(x);
    idl[i] = Random::inv_dilog(x * LI2_MAX);
    float2 b = Random::boxMuller(u.x, u.y);
    bm[2 * i] = b.x; bm[2 * i + 1] = b.y;
    float2 cb = Random::correctedBoxMuller(u.x, u.y, x);
    cbm[2 * i] = cb.x; cbm[2 * i + 1] = cb.y;
    uint2 ps = s;
    pois[i] = Random::poisson(ps, 0.05f + 60.0f * x);
    sround[i] = Random::stochastic_round(10.0f * x, u.y);
}

__global__ void kat_mem_kernel(const int* xs, const int* ys, const int* ps, int n, int npass, int w, int h, int* out,
                               const float* depths, uint64_t* dbits, float nearp, float farp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = posToMemory(xs[i], ys[i], ps[i], npass, w, h);
    dbits[i] = CudaMath::convert_view_depth(depths[i], nearp, farp);
}

static int run_kat(int argc, char** argv) {
    if (argc < 3) return 2;
    std::string outdir = argv[2];
    const int n = 4096;
    std::vector<uint32_t> idx(n), fr(n);
    std::vector<float> fin(n);
    uint64_t st = 12345;
    for (int i = 0; i < n; ++i) {
        st = splitmix64(st);
        idx[i] = (i < 1024) ? uint32_t(i) : uint32_t(st);
        fr[i] = (i < 2048) ? uint32_t(i % 7) : uint32_t(st >> 32);
        fin[i] = (i + 0.5f) / n;
    }
    uint32_t *d_idx, *d_fr, *d_seeds, *d_pcg, *d_pois;
    float *d_fin, *d_pcgf, *d_dl, *d_idl, *d_bm, *d_cbm;
    int* d_sr;
    cudaMalloc(&d_idx, n * 4); cudaMalloc(&d_fr, n * 4); cudaMalloc(&d_fin, n * 4);
    cudaMalloc(&d_seeds, n * 8); cudaMalloc(&d_pcg, n * 8); cudaMalloc(&d_pcgf, n * 8);
    cudaMalloc(&d_dl, n * 4); cudaMalloc(&d_idl, n * 4); cudaMalloc(&d_bm, n * 8); cudaMalloc(&d_cbm, n * 8);
    cudaMalloc(&d_pois, n * 4); cudaMalloc(&d_sr, n * 4);
    cudaMemcpy(d_idx, idx.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_fr, fr.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_fin, fin.data(), n * 4, cudaMemcpyHostToDevice);
    kat_kernel<<<(n + 255) / 256, 256>>>(d_idx, d_fr, d_fin, n, d_seeds, d_pcg, d_pcgf, d_dl, d_idl, d_bm, d_cbm, d_pois, d_sr);
    cudaDeviceSynchronize();
    write_npy(outdir + "/kat_idx.npy", idx.data(), n, "<u4", 4);
    write_npy(outdir + "/kat_frame.npy", fr.data(), n, "<u4", 4);
    write_npy(outdir + "/kat_x.npy", fin.data(), n, "<f4", 4);
    auto s = d2h(d_seeds, 2 * n); write_npy(outdir + "/kat_seed.npy", s.data(), 2 * n, "<u4", 4, {size_t(n), 2});
    auto p = d2h(d_pcg, 2 * n); write_npy(outdir + "/kat_pcg.npy", p.data(), 2 * n, "<u4", 4, {size_t(n), 2});
    auto pf = d2h(d_pcgf, 2 * n); write_npy(outdir + "/kat_pcgf.npy", pf.data(), 2 * n, "<f4", 4, {size_t(n), 2});
    auto dl = d2h(d_dl, n); write_npy(outdir + "/kat_dilog.npy", dl.data(), n, "<f4", 4);
    auto idl = d2h(d_idl, n); write_npy(outdir + "/kat_invdilog.npy", idl.data(), n, "<f4", 4);
    auto bm = d2h(d_bm, 2 * n); write_npy(outdir + "/kat_boxmuller.npy", bm.data(), 2 * n, "<f4", 4, {size_t(n), 2});
    auto cbm = d2h(d_cbm, 2 * n); write_npy(outdir + "/kat_cboxmuller.npy", cbm.data(), 2 * n, "<f4", 4, {size_t(n), 2});
    auto po = d2h(d_pois, n); write_npy(outdir + "/kat_poisson.npy", po.data(), n, "<u4", 4);
    auto sr = d2h(d_sr, n); write_npy(outdir + "/kat_sround.npy", sr.data(), n, "<i4", 4);

    // posToMemory / depth quantisation
    const int m = 4096, npass = 3, w = 200, h = 130;
    std::vector<int> xs(m), ys(m), ps(m);
    std::vector<float> dep(m);
    for (int i = 0; i < m; ++i) {
        st = splitmix64(st);
        xs[i] = int(st % w); ys[i] = int((st >> 20) % h); ps[i] = int((st >> 40) % npass);
        dep[i] = -(0.1f + 200.0f * float(i) / m);
    }
    int *d_xs, *d_ys, *d_ps, *d_out;
    float* d_dep;
    uint64_t* d_db;
    cudaMalloc(&d_xs, m * 4); cudaMalloc(&d_ys, m * 4); cudaMalloc(&d_ps, m * 4); cudaMalloc(&d_out, m * 4);
    cudaMalloc(&d_dep, m * 4); cudaMalloc(&d_db, m * 8);
    cudaMemcpy(d_xs, xs.data(), m * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_ys, ys.data(), m * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_ps, ps.data(), m * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_dep, dep.data(), m * 4, cudaMemcpyHostToDevice);
    kat_mem_kernel<<<(m + 255) / 256, 256>>>(d_xs, d_ys, d_ps, m, npass, w, h, d_out, d_dep, d_db, 0.2f, 150.0f);
    cudaDeviceSynchronize();
    write_npy(outdir + "/kat_mem_x.npy", xs.data(), m, "<i4", 4);
    write_npy(outdir + "/kat_mem_y.npy", ys.data(), m, "<i4", 4);
    write_npy(outdir + "/kat_mem_p.npy", ps.data(), m, "<i4", 4);
    auto o = d2h(d_out, m); write_npy(outdir + "/kat_mem_index.npy", o.data(), m, "<i4", 4);
    write_npy(outdir + "/kat_depth_in.npy", dep.data(), m, "<f4", 4);
    auto db = d2h(d_db, m); write_npy(outdir + "/kat_depth_bits.npy", db.data(), m, "<u8", 8);
    // host-side colour packing of the background (sh.cuh vec3To36Bits)
    std::vector<uint64_t> bg;
    for (int i = 0; i < 64; ++i) {
        glm::vec3 c(float(i) / 63.0f, float((i * 7) % 64) / 63.0f * 1.5f, float((i * 13) % 64) / 63.0f * 0.25f);
        bg.push_back(CudaMath::vec3To36Bits(c));
    }
    write_npy(outdir + "/kat_bg36.npy", bg.data(), bg.size(), "<u8", 8);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 3; }
    return 0;
}

// ---------------------------------------------------------------------------------
// Camera path → matrices, as the viewer computes them (camera_loader.cu:62-90, main.cu:141-157)
// ---------------------------------------------------------------------------------
static int run_camera(int argc, char** argv) {
    if (argc < 10) return 2;
    RenderSettings s;
    s.statistics = new Statistics();
    s.camera_path = argv[2];
    std::string outdir = argv[3];
    s.resolution.x = atoi(argv[4]);
    s.resolution.y = atoi(argv[5]);
    s.fovy = (float)atof(argv[6]);
    s.near_view_plane = (float)atof(argv[7]);
    s.far_view_plane = (float)atof(argv[8]);
    s.override_camera_settings = atoi(argv[9]) != 0;
    s.load_camera();
    std::vector<float> out;
    std::vector<int32_t> res;
    for (size_t i = 0; i < s.camera_states.size(); ++i) {
        s.load_camera_state((int)i);
        s.cameraPosition = s.camera.getTransform().getPosition();
        s.cameraViewMatrix = glm::scale(glm::mat4(1.0f), glm::vec3(1.0f, -1.0f, -1.0f)) * s.camera.getViewMatrix() * s.sceneMatrix;
        float aspect = s.get_aspectXY();
        s.cameraProjectionMatrix = s.camera.getProjectionMatrix(s.fovy, aspect, s.near_view_plane, s.far_view_plane);
        auto planes = s.camera.getFrustumPlanesFromViewMatrix(s.fovy, s.cameraViewMatrix, aspect, s.near_view_plane, s.far_view_plane);
        put_mat4(out, s.cameraViewMatrix);
        put_mat4(out, s.cameraProjectionMatrix);
        for (auto& p : planes) { out.push_back(p.x); out.push_back(p.y); out.push_back(p.z); out.push_back(p.w); }
        out.push_back(s.cameraPosition.x); out.push_back(s.cameraPosition.y); out.push_back(s.cameraPosition.z);
        out.push_back(s.fovy);
        res.push_back(s.resolution.x); res.push_back(s.resolution.y);
    }
    size_t n = s.camera_states.size();
    write_npy(outdir + "/camera_matrices.npy", out.data(), out.size(), "<f4", 4, {n, size_t(16 + 16 + 24 + 3 + 1)});
    write_npy(outdir + "/camera_resolution.npy", res.data(), res.size(), "<i4", 4, {n, 2});
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: ref_harness render|kat|camera ...\n"); return 2; }
    std::string mode = argv[1];
    if (mode == "render") return run_render(argc, argv);
    if (mode == "kat") return run_kat(argc, argv);
    if (mode == "camera") return run_camera(argc, argv);
    if (mode == "probe") return run_probe(argc, argv);
    if (mode == "splatpoints") return run_splat_points(argc, argv);
    if (mode == "sampleprobe") return run_sample_probe(argc, argv);
    fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
