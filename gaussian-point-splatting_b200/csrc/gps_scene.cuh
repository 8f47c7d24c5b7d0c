// Device-resident Gaussian scene formats and their per-Gaussian accessors.
//
//   SceneFP32       — the reference's GPUGaussianSceneUncompressed
//                     (src/core/gaussians/gaussian_types.cuh:548-646), stored here as
//                     16-byte-aligned structure-of-arrays so that every attribute is fetched
//                     with 128-bit loads: pos_op = (mean.xyz, opacity), rot = (w,x,y,z),
//                     scale = (sx,sy,sz,0), sh = 12 float4 (48 interleaved RGB coefficients).
//   SceneCompressed — the reference's default GPUGaussianSceneCompressed
//                     (gaussian_types.cuh:173-374,421-541): 16-byte quantised geometry,
//                     u8 opacity, compact SH (FP32 DC + 45 u8 AC, scene-wide min/max).
//
// Accessors return exactly the values the reference accessors return; the colour
// evaluation follows sh.cuh:191-223 (FP32) and sh.cuh:41-47,55-96,257-273 (compact).
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include "gps_math.cuh"

namespace gps {

// GaussianSceneBounds (gaussian_types.cuh:127-171), the dequantisation ranges.
struct SceneBounds {
    vec3 min_pos, max_pos;
    vec3 min_scale, max_scale;  // log-encoded
    vec3 min_sh[15], max_sh[15];
};

constexpr float kShC0 = 0.28209479177387814f;
constexpr float kShC1 = 0.4886025119029199f;

#if defined(__CUDACC__)

GPS_D vec3 normalize(vec3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
GPS_D vec3 vmax0(vec3 v) { return make_v3(gmax(v.x, 0.0f), gmax(v.y, 0.0f), gmax(v.z, 0.0f)); }

// sh.cuh:191-223 with deg = 3 (the preprocess asks for degree 4, which evaluates all bands)
GPS_D vec3 color_from_sh_fp32(vec3 pos, vec3 campos, const float* shs) {
    vec3 dir = pos - campos;
    dir = normalize(dir);
#define GPS_SH(i) make_v3(shs[3 * (i)], shs[3 * (i) + 1], shs[3 * (i) + 2])
    vec3 result = kShC0 * GPS_SH(0);
    float x = dir.x, y = dir.y, z = dir.z;
    result = result - kShC1 * y * GPS_SH(1) + kShC1 * z * GPS_SH(2) - kShC1 * x * GPS_SH(3);
    float xx = x * x, yy = y * y, zz = z * z;
    float xy = x * y, yz = y * z, xz = x * z;
    result = result + (1.0925484305920792f * xy * GPS_SH(4) + -1.0925484305920792f * yz * GPS_SH(5) +
                       0.31539156525252005f * (2.0f * zz - xx - yy) * GPS_SH(6) +
                       -1.0925484305920792f * xz * GPS_SH(7) + 0.5462742152960396f * (xx - yy) * GPS_SH(8));
    result = result + (-0.5900435899266435f * y * (3.0f * xx - yy) * GPS_SH(9) +
                       2.890611442640554f * xy * z * GPS_SH(10) +
                       -0.4570457994644658f * y * (4.0f * zz - xx - yy) * GPS_SH(11) +
                       0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * GPS_SH(12) +
                       -0.4570457994644658f * x * (4.0f * zz - xx - yy) * GPS_SH(13) +
                       1.445305721320277f * z * (xx - yy) * GPS_SH(14) +
                       -0.5900435899266435f * x * (xx - 3.0f * yy) * GPS_SH(15));
#undef GPS_SH
    result = result + make_v3(0.5f, 0.5f, 0.5f);
    return vmax0(result);
}

// sh.cuh:55-96: real SH basis to band 3, Sloan's recurrence ordering
GPS_D void eval_sh_basis_l3(float out[16], vec3 dir) {
    float x, y, z, z2, c0, s0, c1, s1, d, a, b;
    x = dir.x;
    y = dir.y;
    z = dir.z;
    z2 = z * z;
    d = 0.282094792f;
    out[0] = d;
    d = 0.488602512f * z;
    out[2] = d;
    a = z2 - 0.333333333f;
    d = 0.946174696f * a;
    out[6] = d;
    b = z * (a - 0.266666667f);
    d = 1.865881663f * b;
    out[12] = d;
    c1 = x;
    s1 = y;
    d = -0.488602512f;
    out[1] = s1 * d;
    out[3] = c1 * d;
    d = -1.092548431f * z;
    out[5] = s1 * d;
    out[7] = c1 * d;
    a = z2 - 0.2f;
    d = -2.285228997f * a;
    out[11] = s1 * d;
    out[13] = c1 * d;
    c0 = x * c1 - y * s1;
    s0 = y * c1 + x * s1;
    d = 0.546274215f;
    out[4] = s0 * d;
    out[8] = c0 * d;
    d = 1.445305721f * z;
    out[10] = s0 * d;
    out[14] = c0 * d;
    c1 = x * c0 - y * s0;
    s1 = y * c0 + x * s0;
    d = -0.59004359f;
    out[9] = s1 * d;
    out[15] = c1 * d;
}

// glm::mix(x, y, a) = x*(1-a) + y*a.  In the reference build nvcc fuses one of the two
// products into the multiply-add and keeps the other rounded, and which one differs per
// vector component of the position and log-scale dequantisation (established by comparing
// every Gaussian's decoded position against the reference kernels' outputs).  The two forms
// are therefore written out explicitly:
//   kFuseSecond: fma(y, a, round(x*(1-a)))      kFuseFirst: fma(x, 1-a, round(y*a))
constexpr int kFuseFirst = 0, kFuseSecond = 1;
template <int kForm>
GPS_D float mix_form(float x, float y, float a) {
    if (kForm == kFuseSecond) return __fmaf_rn(y, a, __fmul_rn(x, 1.0f - a));
    return __fmaf_rn(x, 1.0f - a, __fmul_rn(y, a));
}
// position and log-scale dequantisation (gaussian_types.cuh:346,371)
GPS_D vec3 mix_dequant(vec3 x, vec3 y, vec3 a) {
    return make_v3(mix_form<kFuseFirst>(x.x, y.x, a.x), mix_form<kFuseSecond>(x.y, y.y, a.y),
                   mix_form<kFuseSecond>(x.z, y.z, a.z));
}
// compact SH dequantisation (sh.cuh:46)
GPS_D vec3 mix_sh(vec3 x, vec3 y, vec3 a) {
    return make_v3(mix_form<kFuseFirst>(x.x, y.x, a.x), mix_form<kFuseFirst>(x.y, y.y, a.y),
                   mix_form<kFuseFirst>(x.z, y.z, a.z));
}

#endif  // __CUDACC__

#if defined(__CUDACC__)
// Asks L2 for the line holding p (no register, no wait): the preprocess touches the next chunk's
// attributes this way while it works on the current chunk.
GPS_D void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
#endif

struct SceneFP32 {
    const float4* __restrict__ pos_op;
    const float4* __restrict__ rot;
    const float4* __restrict__ scale;
    const float4* __restrict__ sh;
    uint32_t n;
    static constexpr bool kFp64Conic = false;

#if defined(__CUDACC__)
    GPS_D float opacity(uint32_t g) const {
        return gmin(__ldg(&pos_op[g]).w, kMaxOpacity);
    }
    GPS_D void prefetch(uint32_t g) const {
        prefetch_l2(pos_op + g);
        prefetch_l2(rot + g);
        prefetch_l2(scale + g);
    }
    GPS_D void geometry(uint32_t g, vec3& mean, vec4& quat, vec3& s) const {
        float4 a = __ldg(&pos_op[g]);
        float4 q = __ldg(&rot[g]);
        float4 c = __ldg(&scale[g]);
        mean = make_v3(a.x, a.y, a.z);
        quat = make_v4(q.x, q.y, q.z, q.w);
        s = make_v3(c.x, c.y, c.z);
    }
    GPS_D vec3 color(uint32_t g, vec3 mean, vec3 campos) const {
        float shs[48];
        const float4* src = sh + (size_t)g * 12;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            float4 v = __ldg(&src[i]);
            shs[4 * i + 0] = v.x;
            shs[4 * i + 1] = v.y;
            shs[4 * i + 2] = v.z;
            shs[4 * i + 3] = v.w;
        }
        return color_from_sh_fp32(mean, campos, shs);
    }
#endif
};

// Quantised geometry words (gaussian_types.cuh:173-181) + u8 opacity + compact SH.
// Compact SH is stored as two arrays: dc (float4: DC rgb, unused lane) and ac (3 x uint4 =
// 48 bytes holding the 45 AC bytes in the reference's order, 3 trailing pad bytes).
struct SceneCompressed {
    const uint4* __restrict__ geom;
    const uint8_t* __restrict__ opac;
    const float4* __restrict__ sh_dc;
    const uint4* __restrict__ sh_ac;
    SceneBounds bounds;
    uint32_t n;
    static constexpr bool kFp64Conic = false;

#if defined(__CUDACC__)
    GPS_D float opacity(uint32_t g) const {
        return gmin((float)__ldg(&opac[g]) / 255.0f, kMaxOpacity);
    }
    GPS_D void prefetch(uint32_t g) const {
        prefetch_l2(geom + g);
        if ((g & 31u) == 0u) prefetch_l2(opac + g);
    }
    // gaussian_types.cuh:322-374
    GPS_D void geometry(uint32_t g, vec3& mean, vec4& quat, vec3& s) const {
        uint4 q = __ldg(&geom[g]);
        uint32_t px = q.x & 0x7FFFFFu;
        uint32_t py_low9 = (q.x >> 23) & 0x1FFu;
        uint32_t py_high13 = q.y & 0x1FFFu;
        uint32_t pz_low19 = (q.y >> 13) & 0x7FFFFu;
        uint32_t pz_high4 = q.z & 0xFu;
        uint32_t py = py_low9 | (py_high13 << 9);
        uint32_t pz = pz_low19 | (pz_high4 << 19);
        float fx = float(px) / float((1u << 23) - 1u);
        float fy = float(py) / float((1u << 22) - 1u);
        float fz = float(pz) / float((1u << 23) - 1u);
        mean = mix_dequant(bounds.min_pos, bounds.max_pos, make_v3(fx, fy, fz));

        uint32_t rx = (q.z >> 4) & 0x3FFu;
        uint32_t ry = (q.z >> 14) & 0x3FFu;
        uint32_t rz_low8 = (q.z >> 24) & 0xFFu;
        uint32_t rz_high2 = q.w & 0x3u;
        uint32_t rz = rz_low8 | (rz_high2 << 8);
        vec3 vr = make_v3((float)rx / 1023.0f, (float)ry / 1023.0f, (float)rz / 1023.0f);
        vec3 v = make_v3(vr.x * 2.0f - 1.0f, vr.y * 2.0f - 1.0f, vr.z * 2.0f - 1.0f);
        // quat_iem (gaussian_types.cuh:215-235), device branch
        float d = v.x * v.x + v.y * v.y + v.z * v.z;
        float t = rsqrtf(d + 1e-8f);
        float a = 1.57079632679f * t * d;
        float sn = __sinf(a);
        float cs = __cosf(a);
        float k = sn * t;
        quat = make_v4(k * v.x, k * v.y, k * v.z, cs);

        uint32_t sx = (q.w >> 2) & 0x3FFu;
        uint32_t sy = (q.w >> 12) & 0x3FFu;
        uint32_t sz = (q.w >> 22) & 0x3FFu;
        vec3 st = make_v3((float)sx / 1023.0f, (float)sy / 1023.0f, (float)sz / 1023.0f);
        vec3 ls = mix_dequant(bounds.min_scale, bounds.max_scale, st);
        s = make_v3(__expf(ls.x), __expf(ls.y), __expf(ls.z));
    }
    // sh.cuh:257-273 with CompactSH::get (sh.cuh:41-47)
    GPS_D vec3 color(uint32_t g, vec3 mean, vec3 campos) const {
        vec3 dir = mean - campos;
        dir = normalize(dir);
        float e[16];
        eval_sh_basis_l3(e, dir);
        float4 dc = __ldg(&sh_dc[g]);
        uint32_t w[12];
        const uint4* src = sh_ac + (size_t)g * 3;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            uint4 u = __ldg(&src[i]);
            w[4 * i + 0] = u.x;
            w[4 * i + 1] = u.y;
            w[4 * i + 2] = u.z;
            w[4 * i + 3] = u.w;
        }
        vec3 result = make_v3(0.0f, 0.0f, 0.0f);
        result = result + e[0] * make_v3(dc.x, dc.y, dc.z);
#pragma unroll
        for (int i = 1; i < 16; ++i) {
            const int j = i - 1;
            const float r = 1.0f / 255.0f;
            int b0 = 3 * j, b1 = 3 * j + 1, b2 = 3 * j + 2;
            uint32_t q0 = (w[b0 >> 2] >> (8 * (b0 & 3))) & 0xFFu;
            uint32_t q1 = (w[b1 >> 2] >> (8 * (b1 & 3))) & 0xFFu;
            uint32_t q2 = (w[b2 >> 2] >> (8 * (b2 & 3))) & 0xFFu;
            vec3 vq = make_v3((float)(int)q0 * r, (float)(int)q1 * r, (float)(int)q2 * r);
            vec3 c = mix_sh(bounds.min_sh[j], bounds.max_sh[j], vq);
            result = result + e[i] * c;
        }
        result = result + make_v3(0.5f, 0.5f, 0.5f);
        return vmax0(result);
    }
#endif
};

// Half-precision storage (this library's own format, no counterpart in the reference), 80 bytes
// per Gaussian, decoded to FP32 for all arithmetic:
//   rec   uint4 : position as 16-bit fixed-point offsets (x, y, z) from its block origin in
//                 steps of the origin's w, FP16 opacity, FP16 rotation (w, x, y, z)
//   scl   uint4 : FP16 scale (x, y, z), FP16 SH DC term (r, g, b), bf16 AC scales k1, k2
//   ac    3 x uint4 : the 45 AC SH coefficients (FP32 layout order 3..47) as int8 q with
//                 value = q * k_band (band 1: AC 0-8, band 2: 9-23, band 3: 24-44;
//                 k_band = max |AC of the band| / 127, rounded up to bf16); bytes 45-46 hold
//                 k3, byte 47 is zero
//   origin float4 per kHalfOriginBlock Gaussians: the centre of the block's means and the step
//                 w = largest half-extent / 32767 (16 bits over the block's extent, where
//                 FP16 offsets keep 11; the offsets' rounding moved thin coplanar Gaussians
//                 in front of one another)
// The DC term carries most of a Gaussian's colour, so it keeps 11 significant bits.
constexpr uint32_t kHalfOriginBlock = 16;

struct SceneHalf {
    const uint4* __restrict__ rec;
    const uint4* __restrict__ scl;
    const uint4* __restrict__ ac;
    const float4* __restrict__ origin;
    uint32_t n;
    // near-degenerate 2D covariances (det small against a*c) are inverted in FP64
    static constexpr bool kFp64Conic = true;

#if defined(__CUDACC__)
    static GPS_D float h(uint32_t word, int hi) {
        return __half2float(__ushort_as_half((unsigned short)(hi ? (word >> 16) : (word & 0xFFFFu))));
    }
    GPS_D float opacity(uint32_t g) const { return gmin(h(__ldg(&rec[g]).y, 1), kMaxOpacity); }
    GPS_D void prefetch(uint32_t g) const {
        prefetch_l2(rec + g);
        prefetch_l2(scl + g);
    }
    GPS_D void geometry(uint32_t g, vec3& mean, vec4& quat, vec3& s) const {
        const uint4 r = __ldg(&rec[g]);
        const uint4 c = __ldg(&scl[g]);
        const float4 o = __ldg(&origin[g / kHalfOriginBlock]);
        mean = make_v3(o.x + (float)(int16_t)(r.x & 0xFFFFu) * o.w, o.y + (float)(int16_t)(r.x >> 16) * o.w,
                       o.z + (float)(int16_t)(r.y & 0xFFFFu) * o.w);
        quat = make_v4(h(r.z, 0), h(r.z, 1), h(r.w, 0), h(r.w, 1));
        s = make_v3(h(c.x, 0), h(c.x, 1), h(c.y, 0));
    }
    GPS_D vec3 color(uint32_t g, vec3 mean, vec3 campos) const {
        float shs_[48];
        const uint4 c = __ldg(&scl[g]);
        shs_[0] = h(c.y, 1);
        shs_[1] = h(c.z, 0);
        shs_[2] = h(c.z, 1);
        const uint4* src = ac + (size_t)g * 3;
        const uint4 a0 = __ldg(&src[0]), a1 = __ldg(&src[1]), a2 = __ldg(&src[2]);
        const uint32_t w[12] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
        const float k1 = __uint_as_float(c.w << 16), k2 = __uint_as_float(c.w & 0xFFFF0000u);
        const float k3 = __uint_as_float((w[11] << 8) & 0xFFFF0000u);
#pragma unroll
        for (int e = 0; e < 45; ++e) {
            const int q = (int)(int8_t)((w[e >> 2] >> (8 * (e & 3))) & 0xFFu);
            shs_[3 + e] = (float)q * (e < 9 ? k1 : (e < 24 ? k2 : k3));
        }
        return color_from_sh_fp32(mean, campos, shs_);
    }
#endif
};

}  // namespace gps
