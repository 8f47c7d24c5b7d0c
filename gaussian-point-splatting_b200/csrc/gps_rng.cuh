// Counter-based sampling for the stochastic splat: seeds, the 2D PCG hash, Box-Muller and
// its opacity-corrected variant, the dilogarithm polynomial pair, Poisson (Giles' QN3) and
// stochastic rounding.  The integer parts are exact restatements of the reference
// (src/core/random/random.cuh:162-215); the floating-point parts evaluate the same
// expressions with the same CUDA intrinsics (__logf, __sincosf, __fsqrt_rn, __float2int_rn),
// which is what the sample streams' bit-exactness depends on.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gps_math.cuh"

namespace gps {

constexpr float kRecip2e32 = 2.3283064365387e-10f;     // random.cuh:13
constexpr float kLi2Max = 1.6449340668482264f;         // Li2(1) = pi^2/6, random.cuh:108
constexpr float kPiF = 3.141592654f;                   // CUDART_PI_F

struct u32x2 { uint32_t x, y; };

// random.cuh:192-199
GPS_HD uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// random.cuh:201-215: per-(index, frame) 2x32-bit state
GPS_HD u32x2 make_seed(uint32_t idx, uint32_t frame) {
    const uint32_t c1 = 0x9E3779B9u, c2 = 0xBB67AE85u, c3 = 0x3C6EF372u, c4 = 0xA54FF53Au;
    uint32_t h1 = hash32(idx ^ (frame * c1));
    uint32_t h2 = hash32((idx * c2) ^ frame);
    h1 ^= (h2 * c3);
    h2 ^= (h1 * c4);
    u32x2 r;
    r.x = h1;
    r.y = h2;
    return r;
}

// random.cuh:162-178
GPS_HD u32x2 pcg2d_step(u32x2 s) {
    s.x = s.x * 1664525u + 1013904223u;
    s.y = s.y * 1664525u + 1013904223u;
    s.x += s.y * 1664525u;
    s.y += s.x * 1664525u;
    s.x ^= s.x >> 16u;
    s.y ^= s.y >> 16u;
    s.x += s.y * 1664525u;
    s.y += s.x * 1664525u;
    s.x ^= s.x >> 16u;
    s.y ^= s.y >> 16u;
    return s;
}

// random.cuh:181-184: advance the state and return two uniforms in [0,1)
GPS_HD vec2 pcg2d(u32x2& s) {
    s = pcg2d_step(s);
    return make_v2((float)s.x * kRecip2e32, (float)s.y * kRecip2e32);
}

// random.cuh:186-190
GPS_HD int stochastic_round(float x, float u) {
    int base = (int)floorf(x);
    float frac = x - (float)base;
    int r = (u < frac) ? (base + 1) : base;
    return r < 0 ? 0 : r;
}

#if defined(__CUDACC__)
// random.cuh:88-104: polynomial fit of Li2 on [0,1] plus the (1-x)log(1-x) term
GPS_D float dilog(float x) {
    float y = -6.09201442e-01f;
    y = fmaf(y, x, 1.79126616e+00f);
    y = fmaf(y, x, -2.14953223e+00f);
    y = fmaf(y, x, 1.26304372e+00f);
    y = fmaf(y, x, -4.59069895e-01f);
    y = fmaf(y, x, -1.87417414e-01f);
    y = fmaf(y, x, 1.99603130e+00f);
    y = fmaf(y, x, 5.99669467e-05f);
    float s = 1.0f - x;
    if (s > 0.0f) y += s * __logf(fmaxf(s, 1e-37f));
    return y;
}

// random.cuh:110-127: polynomial inverse of Li2 over [0, pi^2/6]
GPS_D float inv_dilog(float x) {
    float t = fminf(x / kLi2Max, 1.0f);
    float y = -1.27463503e+01f;
    y = fmaf(y, t, 5.88993459e+01f);
    y = fmaf(y, t, -1.16025780e+02f);
    y = fmaf(y, t, 1.26945827e+02f);
    y = fmaf(y, t, -8.43108826e+01f);
    y = fmaf(y, t, 3.48799862e+01f);
    y = fmaf(y, t, -8.89606235e+00f);
    y = fmaf(y, t, 1.38640936e+00f);
    y = fmaf(y, t, -7.80640876e-01f);
    y = fmaf(y, t, 1.64841888e+00f);
    y = fmaf(y, t, -2.82836687e-05f);
    return y;
}

GPS_D float clamp_unit_log(float u) { return gclamp(u, 1.e-37f, 1.0f); }

// random.cuh:69-75
GPS_D vec2 box_muller(float u1, float u2) {
    float r = __fsqrt_rn(fmaxf(-2.0f * __logf(clamp_unit_log(u1)), 0.0f));
    float theta = 2.0f * kPiF * u2;
    float s, c;
    __sincosf(theta, &s, &c);
    return make_v2(r * c, r * s);
}

// random.cuh:132-141: radius drawn so that the opacity test after it is unbiased
GPS_D vec2 corrected_box_muller(float u1, float u2, float alpha) {
    float a = 1.0f / fmaxf(alpha, 1.e-37f) * inv_dilog((1.0f - u1) * dilog(alpha));
    a = gclamp(a, 1.e-37f, 1.0f);
    float r = __fsqrt_rn(fmaxf(-2.0f * __logf(a), 0.0f));
    float theta = 2.0f * kPiF * u2;
    float s, c;
    __sincosf(theta, &s, &c);
    return make_v2(r * c, r * s);
}

// poisson.cuh:12-38: Giles (2016) Algorithm 955, QN3 normal asymptotic approximation
GPS_D uint32_t poisson(u32x2& state, float lambda) {
    vec2 u = pcg2d(state);
    float w = box_muller(u.x, u.y).x;
    float w2 = w * w;
    float w3 = w2 * w;
    float w4 = w2 * w2;
    float s = __fsqrt_rn(lambda);
    float inv_s = 1.0f / s;
    float inv_l = 1.0f / lambda;
    float kf = lambda + s * w + (w2 - 1.0f) / 6.0f;
    kf += inv_s * (-(1.0f / 36.0f) * w - (1.0f / 72.0f) * w3);
    kf += inv_l * (-(8.0f / 405.0f) + (7.0f / 810.0f) * w2 + (1.0f / 270.0f) * w4);
    int ki = __float2int_rn(kf);
    return (uint32_t)max(ki, 0);
}

// linalg.cuh:309-317
GPS_D float gaussian_value(vec3 conic, vec2 delta) {
    const float sigma = -0.5f * (conic.x * delta.x * delta.x + conic.z * delta.y * delta.y) - conic.y * delta.x * delta.y;
    if (sigma > 0.f) return 0.0f;
    return __expf(sigma);
}
#endif

}  // namespace gps
