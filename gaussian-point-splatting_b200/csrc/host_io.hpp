// Host-side boundary of the frame path: the 3DGS PLY reader/writer, scene encodings,
// settings and camera math.  Everything here runs once per load or once per frame on the
// CPU, in IEEE single precision without fused multiply-adds (compiled with
// -ffp-contract=off), in the same operation order as the reference's host code, so that
// the values handed to the kernels are bit-identical to the reference's.
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>
#include "gps_math.cuh"
#include "gps_scene.cuh"

namespace gps {

// CPUGaussian (gaussian_types.cuh:89-100): 59 floats, 236 bytes.
struct CpuGaussian {
    float mean[3];
    float sh[48];
    float opacity;
    float scale[3];
    float rot[4];
};
static_assert(sizeof(CpuGaussian) == 236, "CpuGaussian must match the reference layout");

// ---- host threads ------------------------------------------------------------------
// f(begin, end) over [0, n) split across the host's cores (one range below 65,536 items).
void parallel_ranges(uint64_t n, const std::function<void(uint64_t, uint64_t)>& f);

// ---- errors ------------------------------------------------------------------------
void set_last_error(const std::string& msg);
const char* last_error();

// ---- PLY (gaussian_loader.cu:115-245,282-427,480-562, ply_comments.h) ---------------
// Returns 0 on success, otherwise a gps_status value (see include/gps_b200.h).
int ply_read(const std::string& path, std::vector<CpuGaussian>& out, std::vector<std::string>& comments);
// The vertex count and comments from the header alone.
int ply_count(const std::string& path, uint64_t& count, std::vector<std::string>& comments);
// Reads into caller memory of `capacity` Gaussians (the next chunk is read while the current one
// is converted); count receives the vertex count.
int ply_read_into(const std::string& path, CpuGaussian* out, uint64_t capacity, uint64_t& count,
                  std::vector<std::string>& comments);
int ply_write(const std::string& path, const CpuGaussian* g, uint64_t n, const std::vector<std::string>& comments);
bool has_bvh_sorted_comment(const std::vector<std::string>& comments);
// 3DGS output directory -> point_cloud/<alphabetically last>/point_cloud.ply
// (render_settings.cuh:137-199); a file path is returned unchanged.
int resolve_model_path(const std::string& in, std::string& out);
// --sort-morton-order reorder (gaussian_loader.cu:363-424)
void morton_sort(std::vector<CpuGaussian>& g);
// The permutation morton_sort applies: order[j] = the input index of the j-th Gaussian.
void morton_order(const CpuGaussian* g, uint64_t n, uint32_t* order);

// ---- compressed scene encoding (gaussian_types.cuh:127-320, sh.cuh:28-39) ------------
SceneBounds compute_scene_bounds(const CpuGaussian* g, uint64_t n);
void encode_compressed(const CpuGaussian* g, uint64_t n, const SceneBounds& b, uint4* geom, uint8_t* opac,
                       float4* sh_dc, uint4* sh_ac);

// ---- blocks for the hierarchical cull (gaussian_bvh.cu:171-172) ----------------------
uint32_t gaussians_per_block(uint64_t n);

// ---- camera (camera.cpp:88-156, camera.h:39-47, camera_loader.cu:62-90, main.cu:141-157)
struct CameraState {
    int id = 0;
    std::string img_name;
    int width = 0, height = 0;
    float position[3] = {0, 0, 0};
    float rotation[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // JSON rows
    float fx = 0, fy = 0;
};
int load_cameras(const std::string& path, std::vector<CameraState>& out);
float focal_to_fov_deg(float focal, int pixels);
float fov_deg_to_focal(float fovdeg, int pixels);

struct CameraMatrices {
    mat4 view, proj;
    vec4 planes[6];
    vec3 position;
};
// Camera pose given as position + quaternion (glm order w, x, y, z) of the camera transform.
CameraMatrices camera_matrices(vec3 position, const float quat_wxyz[4], float fovy, float aspect, float near_plane,
                               float far_plane);
// glm::quat_cast of a basis given by its columns (c[0], c[1], c[2]).
void quat_from_basis(const mat3& basis, float quat_wxyz[4]);

// ---- per-frame derived constants (gaussian_point_splatting.cu:605-615) --------------
mat4 affine_inverse(const mat4& m);
mat4 inverse4(const mat4& m);
mat4 mat4_mul(const mat4& a, const mat4& b);
void derive_frame(const mat4& view, const mat4& proj, int width, int height, int ss, float fovy, mat4& vp, mat4& cam,
                  vec2& tan_fov, vec2& focal);

}  // namespace gps
