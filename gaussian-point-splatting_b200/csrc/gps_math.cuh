// Small fixed-size vector/matrix types for the splatting frame path.
//
// Bit-exact parity with the reference kernels (which use glm 1.0.2 compiled with nvcc
// -use_fast_math) requires the same floating-point operation sequence, not merely the same
// mathematics: every product, sum and its association below follows the order in which
// the reference evaluates it (column-major matrices; mat*vec = (c0*x + c1*y) + (c2*z + c3*w);
// mat3*mat3 column j = (A0*Bj.x + A1*Bj.y) + A2*Bj.z; dot3 = (x*x' + y*y') + z*z'), so that
// nvcc contracts the same multiply-adds.  Matrix zeros that the reference carries through
// (e.g. the third column of the EWA Jacobian) are carried through here too.
//
// Reference call sites mirrored here:
//   linalg.cuh:211-249 (transformPoint4x3, computeCov2D), :251-296 (bounds), :301-317
//   (conic, gaussian_value), :319-342 (quat_to_rotmat, scale_rot_to_cov), :406-420 (depth).
// All paths are src/core/math/linalg.cuh of PeterZs/gaussian-point-splatting.
#pragma once
#include <cmath>
#include <cstdint>
#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

#if defined(__CUDACC__)
#define GPS_HD __host__ __device__ __forceinline__
#define GPS_D __device__ __forceinline__
#else
#define GPS_HD inline
#define GPS_D inline
#endif

namespace gps {

// ---- packing constants of the 64-bit splat word (reference config.h:36-48) ----------
constexpr uint64_t kColorBits = 36ull;
constexpr uint64_t kDepthBits = 28ull;
constexpr uint64_t kDepthMax = (1ull << kDepthBits) - 1;
constexpr uint64_t kDepthShift = kColorBits;
constexpr uint64_t kColorMask = (1ull << kColorBits) - 1;
constexpr uint64_t kDepthMask = kDepthMax << kDepthShift;
constexpr int kTileBits = 6;               // Morton-ordered 64x64 tiles
constexpr int kTileSize = 1 << kTileBits;
constexpr float kTruncationStd = 3.0f;     // GAUSSIAN_TRUNCATION_STD
constexpr int kPointsPerKernel = 1;        // POINTS_PER_KERNEL
constexpr float kMaxOpacity = 1.0f;        // MAX_GAUSSIAN_OPACITY

struct vec2 { float x, y; };
struct vec3 { float x, y, z; };
struct vec4 { float x, y, z, w; };
struct ivec2 { int x, y; };
struct mat3 { vec3 c[3]; };  // c[column]
struct mat4 { vec4 c[4]; };

// glm's scalar min/max/clamp semantics: min = (y < x) ? y : x, max = (x < y) ? y : x
GPS_HD float gmin(float x, float y) { return (y < x) ? y : x; }
GPS_HD float gmax(float x, float y) { return (x < y) ? y : x; }
GPS_HD float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }

GPS_HD vec2 make_v2(float x, float y) { vec2 r; r.x = x; r.y = y; return r; }
GPS_HD vec3 make_v3(float x, float y, float z) { vec3 r; r.x = x; r.y = y; r.z = z; return r; }
GPS_HD vec4 make_v4(float x, float y, float z, float w) { vec4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }

GPS_HD vec3 operator+(vec3 a, vec3 b) { return make_v3(a.x + b.x, a.y + b.y, a.z + b.z); }
GPS_HD vec3 operator-(vec3 a, vec3 b) { return make_v3(a.x - b.x, a.y - b.y, a.z - b.z); }
GPS_HD vec3 operator*(vec3 a, float s) { return make_v3(a.x * s, a.y * s, a.z * s); }
GPS_HD vec3 operator*(float s, vec3 a) { return make_v3(s * a.x, s * a.y, s * a.z); }
GPS_HD vec3 operator*(vec3 a, vec3 b) { return make_v3(a.x * b.x, a.y * b.y, a.z * b.z); }
GPS_HD vec4 operator*(vec4 a, float s) { return make_v4(a.x * s, a.y * s, a.z * s, a.w * s); }
GPS_HD vec4 operator*(vec4 a, vec4 b) { return make_v4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
GPS_HD vec4 operator+(vec4 a, vec4 b) { return make_v4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
GPS_HD vec4 operator-(vec4 a, vec4 b) { return make_v4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

// (x*x' + y*y') + z*z'
GPS_HD float dot(vec3 a, vec3 b) {
    vec3 t = a * b;
    return t.x + t.y + t.z;
}
// (x*x' + y*y') + (z*z' + w*w')
GPS_HD float dot(vec4 a, vec4 b) {
    vec4 t = a * b;
    return (t.x + t.y) + (t.z + t.w);
}

GPS_HD mat3 mat3_from_cols(vec3 a, vec3 b, vec3 c) { mat3 m; m.c[0] = a; m.c[1] = b; m.c[2] = c; return m; }
GPS_HD mat3 mat3_identity(float d) {
    return mat3_from_cols(make_v3(d, 0.0f, 0.0f), make_v3(0.0f, d, 0.0f), make_v3(0.0f, 0.0f, d));
}
GPS_HD mat3 mat3_of(const mat4& m) {  // upper-left 3x3
    return mat3_from_cols(make_v3(m.c[0].x, m.c[0].y, m.c[0].z), make_v3(m.c[1].x, m.c[1].y, m.c[1].z),
                          make_v3(m.c[2].x, m.c[2].y, m.c[2].z));
}
GPS_HD mat3 transpose(const mat3& m) {
    return mat3_from_cols(make_v3(m.c[0].x, m.c[1].x, m.c[2].x), make_v3(m.c[0].y, m.c[1].y, m.c[2].y),
                          make_v3(m.c[0].z, m.c[1].z, m.c[2].z));
}
// (c0*x + c1*y) + c2*z
GPS_HD vec3 operator*(const mat3& m, vec3 v) {
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}
// column j = (A0*Bj.x + A1*Bj.y) + A2*Bj.z
GPS_HD mat3 operator*(const mat3& a, const mat3& b) {
    mat3 r;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        vec3 t = a.c[0] * b.c[j].x;
        t = t + a.c[1] * b.c[j].y;
        t = t + a.c[2] * b.c[j].z;
        r.c[j] = t;
    }
    return r;
}
// (c0*x + c1*y) + (c2*z + c3*w)
GPS_HD vec4 operator*(const mat4& m, vec4 v) {
    vec4 m0 = m.c[0] * v.x;
    vec4 m1 = m.c[1] * v.y;
    vec4 a0 = m0 + m1;
    vec4 m2 = m.c[2] * v.z;
    vec4 m3 = m.c[3] * v.w;
    vec4 a1 = m2 + m3;
    return a0 + a1;
}
// column j = ((A0*Bj.x + A1*Bj.y) + A2*Bj.z) + A3*Bj.w
GPS_HD mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r;
    for (int j = 0; j < 4; ++j) {
        vec4 t = a.c[0] * b.c[j].x;
        t = t + a.c[1] * b.c[j].y;
        t = t + a.c[2] * b.c[j].z;
        t = t + a.c[3] * b.c[j].w;
        r.c[j] = t;
    }
    return r;
}

// linalg.cuh:211-215
GPS_HD vec3 transform_point4x3(vec3 p, const mat4& m) {
    const mat3 b = mat3_of(m);
    vec3 o = make_v3(m.c[3].x, m.c[3].y, m.c[3].z);
    return b * p + o;
}

// Rotation from a quaternion stored (w, x, y, z) in the four lanes (3DGS rot_0..rot_3 order),
// linalg.cuh:319-321 feeding glm's quaternion-to-matrix conversion.
GPS_HD mat3 quat_to_rotmat(vec4 q) {
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    float qxx = x * x, qyy = y * y, qzz = z * z;
    float qxz = x * z, qxy = x * y, qyz = y * z;
    float qwx = w * x, qwy = w * y, qwz = w * z;
    mat3 r = mat3_identity(1.0f);
    r.c[0].x = 1.0f - 2.0f * (qyy + qzz);
    r.c[0].y = 2.0f * (qxy + qwz);
    r.c[0].z = 2.0f * (qxz - qwy);
    r.c[1].x = 2.0f * (qxy - qwz);
    r.c[1].y = 1.0f - 2.0f * (qxx + qzz);
    r.c[1].z = 2.0f * (qyz + qwx);
    r.c[2].x = 2.0f * (qxz + qwy);
    r.c[2].y = 2.0f * (qyz - qwx);
    r.c[2].z = 1.0f - 2.0f * (qxx + qyy);
    return r;
}

// linalg.cuh:324-342: Sigma = (R S)(R S)^T with S = diag(scale)
#if defined(__CUDA_ARCH__)
// On the device the 3D covariance is spelled out with round-to-nearest intrinsics, which the
// compiler never contracts or reorders, in the rounding pattern of the reference's compiled
// quaternion-to-matrix and M * M^T (glm's mat3_cast and mat3 product): which products are
// rounded on their own and which are fused into the following add.  Left to the compiler, the
// same expressions contract differently inside different kernels; in the preprocess that gave
// 1-ulp different off-diagonal terms for about a third of the Gaussians, hence 1-ulp different
// sample positions.  The pattern was fitted against the reference's own kernels (bit-identical
// covariances for every survivor of a 2M-Gaussian town frame, up to the sign of exact zeros,
// which fast-math code does not preserve).
GPS_D mat3 scale_rot_to_cov(vec3 scale, vec4 quat) {
    const float w = quat.x, x = quat.y, y = quat.z, z = quat.w;
    const float qxx = __fmul_rn(x, x), qyy = __fmul_rn(y, y), qzz = __fmul_rn(z, z);
    const float qxz = __fmul_rn(x, z), qxy = __fmul_rn(x, y), qyz = __fmul_rn(y, z);
    const float qwx = __fmul_rn(w, x), qwy = __fmul_rn(w, y), qwz = __fmul_rn(w, z);
    (void)qxx;
    mat3 r;  // columns, as glm::toMat3
    r.c[0].x = __fsub_rn(1.0f, __fmul_rn(2.0f, __fadd_rn(qyy, qzz)));
    r.c[0].y = __fmul_rn(2.0f, __fmaf_rn(x, y, qwz));
    r.c[0].z = __fmul_rn(2.0f, __fmaf_rn(x, z, -qwy));
    r.c[1].x = __fmul_rn(2.0f, __fmaf_rn(x, y, -qwz));
    r.c[1].y = __fsub_rn(1.0f, __fmul_rn(2.0f, __fmaf_rn(x, x, qzz)));
    r.c[1].z = __fmul_rn(2.0f, __fmaf_rn(w, x, qyz));
    r.c[2].x = __fmul_rn(2.0f, __fmaf_rn(x, z, qwy));
    r.c[2].y = __fmul_rn(2.0f, __fmaf_rn(-w, x, qyz));
    r.c[2].z = __fsub_rn(1.0f, __fmul_rn(2.0f, __fmaf_rn(x, x, qyy)));
    const float sc[3] = {scale.x, scale.y, scale.z};
    float m[3][3];  // m[k][i] = M column k, row i = R column k, row i * scale_k
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        m[k][0] = __fmul_rn(r.c[k].x, sc[k]);
        m[k][1] = __fmul_rn(r.c[k].y, sc[k]);
        m[k][2] = __fmul_rn(r.c[k].z, sc[k]);
    }
    // (M M^T)[c][i] = (M[0][i] M[0][c] + M[1][i] M[1][c]) + M[2][i] M[2][c]: the middle product
    // rounded, the first and last fused
    auto el = [&](int c, int i) {
        return __fmaf_rn(m[2][i], m[2][c], __fmaf_rn(m[0][i], m[0][c], __fmul_rn(m[1][i], m[1][c])));
    };
    mat3 out;
    out.c[0] = make_v3(el(0, 0), el(0, 1), el(0, 2));
    out.c[1] = make_v3(out.c[0].y, el(1, 1), el(1, 2));
    out.c[2] = make_v3(out.c[0].z, out.c[1].z, el(2, 2));
    return out;
}
#else
GPS_HD mat3 scale_rot_to_cov(vec3 scale, vec4 quat) {
    mat3 r = quat_to_rotmat(quat);
    mat3 s = mat3_identity(1.0f);
    s.c[0].x = scale.x;
    s.c[1].y = scale.y;
    s.c[2].z = scale.z;
    mat3 m = r * s;
    return m * transpose(m);
}
#endif

// linalg.cuh:221-249: EWA projection of the 3D covariance (Zwicker et al. 2002, eq. 29/31),
// returns (cov[0][0], cov[0][1], cov[1][1]).
GPS_HD vec3 compute_cov2d(const mat4& view, const mat3& cov3d, vec3 mean, vec2 tan_fov, vec2 focal) {
    const mat3 w = mat3_of(view);
    vec3 t = transform_point4x3(mean, view);
    const float limx = 1.3f * tan_fov.x;
    const float limy = 1.3f * tan_fov.y;
    const float txtz = t.x / t.z;
    const float tytz = t.y / t.z;
    t.x = fminf(limx, fmaxf(-limx, txtz)) * t.z;
    t.y = fminf(limy, fmaxf(-limy, tytz)) * t.z;
    mat3 j = mat3_from_cols(make_v3(focal.x / t.z, 0.0f, -(focal.x * t.x) / (t.z * t.z)),
                            make_v3(0.0f, focal.y / t.z, -(focal.y * t.y) / (t.z * t.z)),
                            make_v3(0.0f, 0.0f, 0.0f));
    mat3 tm = transpose(w) * j;
    mat3 cov = transpose(tm) * cov3d * tm;
    return make_v3(cov.c[0].x, cov.c[0].y, cov.c[1].y);
}

// linalg.cuh:251-296: 3-sigma extent rounded out to 16-pixel tiles and clamped to the screen.
GPS_D bool gaussian_tile_bounds(ivec2& out_min, ivec2& out_max, ivec2 resolution, vec3 cov2d, vec2 pixel_mean) {
    const int tile = 16;
    float a = cov2d.x;
    float c = cov2d.z;
#if defined(__CUDA_ARCH__)
    ivec2 ext = {(int)ceilf(kTruncationStd * __fsqrt_rn(a)), (int)ceilf(kTruncationStd * __fsqrt_rn(c))};
#else
    ivec2 ext = {(int)ceilf(kTruncationStd * sqrtf(a)), (int)ceilf(kTruncationStd * sqrtf(c))};
#endif
    vec2 mn = make_v2(pixel_mean.x - (float)ext.x, pixel_mean.y - (float)ext.y);
    vec2 mx = make_v2(pixel_mean.x + (float)ext.x, pixel_mean.y + (float)ext.y);
    int tile_min_x = (int)floorf(mn.x / tile);
    int tile_min_y = (int)floorf(mn.y / tile);
    int tile_max_x = (int)ceilf(mx.x / tile);
    int tile_max_y = (int)ceilf(mx.y / tile);
    int tiles_x = (resolution.x + tile - 1) / tile;
    int tiles_y = (resolution.y + tile - 1) / tile;
    if (tile_max_x <= 0 || tile_max_y <= 0 || tile_min_x >= tiles_x || tile_min_y >= tiles_y) return false;
    tile_min_x = (int)fmaxf((float)tile_min_x, 0.0f);
    tile_min_y = (int)fmaxf((float)tile_min_y, 0.0f);
    tile_max_x = (int)fminf((float)tile_max_x, (float)tiles_x);
    tile_max_y = (int)fminf((float)tile_max_y, (float)tiles_y);
    out_min.x = tile_min_x * tile;
    out_min.y = tile_min_y * tile;
    out_max.x = tile_max_x * tile;
    out_max.y = tile_max_y * tile;
    return true;
}

// linalg.cuh:301-307
GPS_HD vec3 conic_of(vec3 cov2d, float inv_det) {
    return make_v3(cov2d.z * inv_det, -cov2d.y * inv_det, cov2d.x * inv_det);
}

// linalg.cuh:406-411: 28-bit linear view-depth key
GPS_HD float view_depth_from_key(uint64_t depth, float near_plane, float far_plane) {
    return -(((float)depth / (float)kDepthMax) * (far_plane - near_plane) + near_plane);
}
GPS_HD uint64_t depth_key(float depth, float near_plane, float far_plane) {
    float t = gclamp((fabsf(depth) - near_plane) / (far_plane - near_plane), 0.0f, 1.0f);
    return ((uint64_t)(t * (float)kDepthMax)) & kDepthMax;
}
// linalg.cuh:413-420
GPS_HD float view_to_projected_depth(float z_view, float near_plane, float far_plane) {
    float a = (far_plane + near_plane) / (far_plane - near_plane);
    float b = (2.0f * far_plane * near_plane) / (far_plane - near_plane);
    return a + b / z_view;
}

// post_processing_kernels.cuh:71-104: 64x64 Morton tiles, samples-per-pixel innermost.
GPS_HD uint32_t morton_spread(uint32_t a) {
    a = (a | (a << 8)) & 0x00FF00FFu;
    a = (a | (a << 4)) & 0x0F0F0F0Fu;
    a = (a | (a << 2)) & 0x33333333u;
    a = (a | (a << 1)) & 0x55555555u;
    return a;
}
GPS_HD uint32_t morton_encode(uint32_t x, uint32_t y) { return morton_spread(x) | (morton_spread(y) << 1); }
GPS_HD int splat_index(int x, int y, int p, int num_passes, int width, int height) {
    const int tx = x >> kTileBits;
    const int ty = y >> kTileBits;
    const int lx = x & (kTileSize - 1);
    const int ly = y & (kTileSize - 1);
    const uint32_t code = morton_encode((uint32_t)lx, (uint32_t)ly);
    const int tiles_per_row = (width + kTileSize - 1) >> kTileBits;
    (void)height;
    const int tile_index = ty * tiles_per_row + tx;
    return (tile_index * kTileSize * kTileSize + (int)code) * num_passes + p;
}
// Entries of the padded splat buffer (gaussian_point_splatting.cu:749-760), as size_t.
GPS_HD uint64_t splat_buffer_entries(int up_width, int up_height, int num_passes) {
    uint64_t tx = (uint64_t)((up_width + kTileSize - 1) >> kTileBits);
    uint64_t ty = (uint64_t)((up_height + kTileSize - 1) >> kTileBits);
    return tx * ty * (uint64_t)kTileSize * kTileSize * (uint64_t)num_passes;
}

// sh.cuh:124-133: background colour to three 12-bit channels (truncating, HDR headroom)
GPS_HD uint64_t rgb_to_36bits(vec3 rgb) {
    const float a = 255.0f;
    return (((uint64_t)(rgb.x * a) & 0xFFFu) << 24) | (((uint64_t)(rgb.y * a) & 0xFFFu) << 12) |
           ((uint64_t)(rgb.z * a) & 0xFFFu);
}

}  // namespace gps
