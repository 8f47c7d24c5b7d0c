// CPU oracle of the Gaussian point-splatting frame path — TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference's algorithm (PeterZs/gaussian-point-splatting),
// used by tests/ and by bench.py's CPU-baseline leg to check the CUDA path; nothing in the library
// links or calls it.  It follows, step by step:
//   frame driver        src/core/rendering/passes/gaussian_point_splatting.cu:599-737
//   preprocess          gaussian_point_splatting.cu:17-65, 147-307
//   workload scan       src/core/random/workload/workload_distributor.cu:52-145
//   splat               gaussian_point_splatting.cu:67-141, 383-432
//   resolve / clear     gaussian_point_splatting.cu:484-548, 580-585, 620-621
//   RNG / Poisson       src/core/random/random.cuh:69-215, src/core/random/poisson.cuh:12-38
//   math                src/core/math/linalg.cuh:211-317, 339-342, 406-420
//   SH                  src/core/math/sh.cuh:28-51, 55-96, 124-133, 191-223, 257-273
//   scene formats       src/core/gaussians/gaussian_types.cuh:173-374, 421-653
//   addressing          src/core/rendering/passes/post_processing_kernels.cuh:71-104
//   post                post_processing_kernels.cuh:108-285
//   Hi-Z                src/core/rendering/occlusion/depth_mip_chain.cu:7-145, .cuh:172-215
//   block cull          src/core/rendering/occlusion/gaussian_bvh.cu:111-195, 215-329
//
// Arithmetic: IEEE single precision, no contraction (built with -ffp-contract=off), and
// correctly rounded libm functions in place of the GPU's approximate intrinsics (__logf,
// __expf, __sincosf, lg2.approx, approximate division).  The integer layer — seeds, PCG,
// Morton addressing, packing, scan, point->Gaussian map — is exact; floating-point results
// agree with the GPU to a few ulps, so sample-level outputs are compared with tolerances.
// The reference's own polynomial fmaf() evaluations are kept as fmaf (exact on both sides).
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/gps_b200.h"

// The estimator's arithmetic type: float for the FP32 oracle (what the CUDA path is checked against),
// double for the FP64 build (ORACLE_FP64, liboracle64.so) used to state arithmetic error.  The
// integer layer (seeds, PCG, Morton addressing, packing, scan) is the same in both; scene storage,
// the depth chain and the culling blocks stay FP32 in both.
#ifdef ORACLE_FP64
typedef double real;
#else
typedef float real;
#endif


namespace {

// ---------------------------------------------------------------------------------
// small math (column-major), same association as the reference
// ---------------------------------------------------------------------------------
struct V2 { real x, y; };
struct V3 { real x, y, z; };
struct V4 { real x, y, z, w; };
struct M3 { V3 c[3]; };
struct M4 { V4 c[4]; };

inline real gmin(real x, real y) { return (y < x) ? y : x; }
inline real gmax(real x, real y) { return (x < y) ? y : x; }
inline real gclamp(real x, real lo, real hi) { return gmin(gmax(x, lo), hi); }
inline V3 v3(real x, real y, real z) { return {x, y, z}; }
inline V4 v4(real x, real y, real z, real w) { return {x, y, z, w}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, real s) { return {a.x * s, a.y * s, a.z * s}; }
inline V4 add(V4 a, V4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline V4 mul(V4 a, real s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline real dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline M3 mat3_of(const M4& m) {
    return {{{m.c[0].x, m.c[0].y, m.c[0].z}, {m.c[1].x, m.c[1].y, m.c[1].z}, {m.c[2].x, m.c[2].y, m.c[2].z}}};
}
inline M3 transpose(const M3& m) {
    return {{{m.c[0].x, m.c[1].x, m.c[2].x}, {m.c[0].y, m.c[1].y, m.c[2].y}, {m.c[0].z, m.c[1].z, m.c[2].z}}};
}
inline V3 mul(const M3& m, V3 v) { return add(add(mul(m.c[0], v.x), mul(m.c[1], v.y)), mul(m.c[2], v.z)); }
inline M3 mul(const M3& a, const M3& b) {
    M3 r;
    for (int j = 0; j < 3; ++j) r.c[j] = add(add(mul(a.c[0], b.c[j].x), mul(a.c[1], b.c[j].y)), mul(a.c[2], b.c[j].z));
    return r;
}
inline V4 mul(const M4& m, V4 v) {
    return add(add(mul(m.c[0], v.x), mul(m.c[1], v.y)), add(mul(m.c[2], v.z), mul(m.c[3], v.w)));
}
inline M4 mul(const M4& a, const M4& b) {
    M4 r;
    for (int j = 0; j < 4; ++j)
        r.c[j] = add(add(add(mul(a.c[0], b.c[j].x), mul(a.c[1], b.c[j].y)), mul(a.c[2], b.c[j].z)), mul(a.c[3], b.c[j].w));
    return r;
}
M4 m4_from(const float* p) {
    M4 m;
    for (int c = 0; c < 4; ++c) m.c[c] = v4(p[4 * c], p[4 * c + 1], p[4 * c + 2], p[4 * c + 3]);
    return m;
}
inline real el(const M4& m, int c, int r) { const V4& v = m.c[c]; return r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w; }
inline real el3(const M3& m, int c, int r) { const V3& v = m.c[c]; return r == 0 ? v.x : r == 1 ? v.y : v.z; }

M3 inverse3(const M3& m) {
    auto e = [&](int c, int r) { return el3(m, c, r); };
    real od = 1.0f / (+e(0, 0) * (e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2)) - e(1, 0) * (e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2)) +
                       e(2, 0) * (e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2)));
    real i[3][3];
    i[0][0] = +(e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2));
    i[1][0] = -(e(1, 0) * e(2, 2) - e(2, 0) * e(1, 2));
    i[2][0] = +(e(1, 0) * e(2, 1) - e(2, 0) * e(1, 1));
    i[0][1] = -(e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2));
    i[1][1] = +(e(0, 0) * e(2, 2) - e(2, 0) * e(0, 2));
    i[2][1] = -(e(0, 0) * e(2, 1) - e(2, 0) * e(0, 1));
    i[0][2] = +(e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2));
    i[1][2] = -(e(0, 0) * e(1, 2) - e(1, 0) * e(0, 2));
    i[2][2] = +(e(0, 0) * e(1, 1) - e(1, 0) * e(0, 1));
    M3 r;
    for (int c = 0; c < 3; ++c) r.c[c] = v3(i[c][0] * od, i[c][1] * od, i[c][2] * od);
    return r;
}
M4 affine_inverse(const M4& m) {
    M3 inv = inverse3(mat3_of(m));
    M3 neg;
    for (int c = 0; c < 3; ++c) neg.c[c] = v3(-inv.c[c].x, -inv.c[c].y, -inv.c[c].z);
    V3 t = mul(neg, v3(m.c[3].x, m.c[3].y, m.c[3].z));
    M4 r;
    for (int c = 0; c < 3; ++c) r.c[c] = v4(inv.c[c].x, inv.c[c].y, inv.c[c].z, 0.0f);
    r.c[3] = v4(t.x, t.y, t.z, 1.0f);
    return r;
}

// ---------------------------------------------------------------------------------
// RNG (random.cuh), exact integer layer
// ---------------------------------------------------------------------------------
struct Seed { uint32_t x, y; };
inline uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
inline Seed make_seed(uint32_t idx, uint32_t frame) {
    uint32_t h1 = hash32(idx ^ (frame * 0x9E3779B9u));
    uint32_t h2 = hash32((idx * 0xBB67AE85u) ^ frame);
    h1 ^= (h2 * 0x3C6EF372u);
    h2 ^= (h1 * 0xA54FF53Au);
    return {h1, h2};
}
inline Seed pcg_step(Seed s) {
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
inline V2 pcg2d(Seed& s) {
    s = pcg_step(s);
    return {(real)s.x * 2.3283064365387e-10f, (real)s.y * 2.3283064365387e-10f};
}
inline int stochastic_round(real x, real u) {
    int base = (int)std::floor(x);
    real frac = x - (real)base;
    int r = (u < frac) ? base + 1 : base;
    return r < 0 ? 0 : r;
}
real dilog(real x) {
    real y = -6.09201442e-01f;
    y = std::fmaf(y, x, 1.79126616e+00f);
    y = std::fmaf(y, x, -2.14953223e+00f);
    y = std::fmaf(y, x, 1.26304372e+00f);
    y = std::fmaf(y, x, -4.59069895e-01f);
    y = std::fmaf(y, x, -1.87417414e-01f);
    y = std::fmaf(y, x, 1.99603130e+00f);
    y = std::fmaf(y, x, 5.99669467e-05f);
    real s = 1.0f - x;
    if (s > 0.0f) y += s * std::log(std::fmax(s, 1e-37f));
    return y;
}
real inv_dilog(real x) {
    real t = std::fmin(x / 1.6449340668482264f, 1.0f);
    real y = -1.27463503e+01f;
    y = std::fmaf(y, t, 5.88993459e+01f);
    y = std::fmaf(y, t, -1.16025780e+02f);
    y = std::fmaf(y, t, 1.26945827e+02f);
    y = std::fmaf(y, t, -8.43108826e+01f);
    y = std::fmaf(y, t, 3.48799862e+01f);
    y = std::fmaf(y, t, -8.89606235e+00f);
    y = std::fmaf(y, t, 1.38640936e+00f);
    y = std::fmaf(y, t, -7.80640876e-01f);
    y = std::fmaf(y, t, 1.64841888e+00f);
    y = std::fmaf(y, t, -2.82836687e-05f);
    return y;
}
constexpr real kTwoPiF = 2.0f * 3.141592654f;
V2 box_muller(real u1, real u2) {
    real r = std::sqrt(std::fmax(-2.0f * std::log(gclamp(u1, 1.e-37f, 1.0f)), 0.0f));
    real th = kTwoPiF * u2;
    return {r * std::cos(th), r * std::sin(th)};
}
V2 corrected_box_muller(real u1, real u2, real alpha) {
    real a = 1.0f / std::fmax(alpha, 1.e-37f) * inv_dilog((1.0f - u1) * dilog(alpha));
    a = gclamp(a, 1.e-37f, 1.0f);
    real r = std::sqrt(std::fmax(-2.0f * std::log(a), 0.0f));
    real th = kTwoPiF * u2;
    return {r * std::cos(th), r * std::sin(th)};
}
uint32_t poisson(Seed& st, real lambda) {
    V2 u = pcg2d(st);
    real w = box_muller(u.x, u.y).x;
    real w2 = w * w, w3 = w2 * w, w4 = w2 * w2;
    real s = std::sqrt(lambda);
    real inv_s = 1.0f / s, inv_l = 1.0f / lambda;
    real kf = lambda + s * w + (w2 - 1.0f) / 6.0f;
    kf += inv_s * (-(1.0f / 36.0f) * w - (1.0f / 72.0f) * w3);
    kf += inv_l * (-(8.0f / 405.0f) + (7.0f / 810.0f) * w2 + (1.0f / 270.0f) * w4);
    long ki = std::lrint(kf);  // round half to even like __float2int_rn
    return (uint32_t)(ki < 0 ? 0 : ki);
}

// ---------------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------------
M3 quat_to_rotmat(V4 q) {
    const real w = q.x, x = q.y, y = q.z, z = q.w;
    real qxx = x * x, qyy = y * y, qzz = z * z, qxz = x * z, qxy = x * y, qyz = y * z, qwx = w * x, qwy = w * y, qwz = w * z;
    M3 r;
    r.c[0] = v3(1.0f - 2.0f * (qyy + qzz), 2.0f * (qxy + qwz), 2.0f * (qxz - qwy));
    r.c[1] = v3(2.0f * (qxy - qwz), 1.0f - 2.0f * (qxx + qzz), 2.0f * (qyz + qwx));
    r.c[2] = v3(2.0f * (qxz + qwy), 2.0f * (qyz - qwx), 1.0f - 2.0f * (qxx + qyy));
    return r;
}
M3 scale_rot_to_cov(V3 s, V4 q) {
    M3 r = quat_to_rotmat(q);
    M3 sm = {{{s.x, 0.0f, 0.0f}, {0.0f, s.y, 0.0f}, {0.0f, 0.0f, s.z}}};
    M3 m = mul(r, sm);
    return mul(m, transpose(m));
}
V3 transform_point4x3(V3 p, const M4& m) { return add(mul(mat3_of(m), p), v3(m.c[3].x, m.c[3].y, m.c[3].z)); }
V3 compute_cov2d(const M4& view, const M3& cov3d, V3 mean, V2 tan_fov, V2 focal) {
    M3 w = mat3_of(view);
    V3 t = transform_point4x3(mean, view);
    real limx = 1.3f * tan_fov.x, limy = 1.3f * tan_fov.y;
    real txtz = t.x / t.z, tytz = t.y / t.z;
    t.x = std::fmin(limx, std::fmax(-limx, txtz)) * t.z;
    t.y = std::fmin(limy, std::fmax(-limy, tytz)) * t.z;
    M3 j = {{{focal.x / t.z, 0.0f, -(focal.x * t.x) / (t.z * t.z)}, {0.0f, focal.y / t.z, -(focal.y * t.y) / (t.z * t.z)}, {0.0f, 0.0f, 0.0f}}};
    M3 tm = mul(transpose(w), j);
    M3 cov = mul(mul(transpose(tm), cov3d), tm);
    return v3(cov.c[0].x, cov.c[0].y, cov.c[1].y);
}
bool tile_bounds(int& mnx, int& mny, int& mxx, int& mxy, int resx, int resy, V3 cov2d, V2 pm) {
    const int tile = 16;
    int ex = (int)std::ceil(3.0f * std::sqrt(cov2d.x)), ey = (int)std::ceil(3.0f * std::sqrt(cov2d.z));
    real lox = pm.x - (real)ex, loy = pm.y - (real)ey, hix = pm.x + (real)ex, hiy = pm.y + (real)ey;
    int tmnx = (int)std::floor(lox / tile), tmny = (int)std::floor(loy / tile);
    int tmxx = (int)std::ceil(hix / tile), tmxy = (int)std::ceil(hiy / tile);
    int tx = (resx + tile - 1) / tile, ty = (resy + tile - 1) / tile;
    if (tmxx <= 0 || tmxy <= 0 || tmnx >= tx || tmny >= ty) return false;
    tmnx = std::max(tmnx, 0);
    tmny = std::max(tmny, 0);
    tmxx = std::min(tmxx, tx);
    tmxy = std::min(tmxy, ty);
    mnx = tmnx * tile;
    mny = tmny * tile;
    mxx = tmxx * tile;
    mxy = tmxy * tile;
    return true;
}
inline uint64_t depth_key(real d, real n, real f) {
    real t = gclamp((std::fabs(d) - n) / (f - n), 0.0f, 1.0f);
    return ((uint64_t)(t * 268435456.0f)) & 0xFFFFFFFull;
}
inline real view_depth_from_key(uint64_t d, real n, real f) { return -(((real)d / 268435456.0f) * (f - n) + n); }
inline real view_to_ndc(real z, real n, real f) {
    real a = (f + n) / (f - n), b = (2.0f * f * n) / (f - n);
    return a + b / z;
}
inline uint32_t spread(uint32_t a) {
    a = (a | (a << 8)) & 0x00FF00FFu;
    a = (a | (a << 4)) & 0x0F0F0F0Fu;
    a = (a | (a << 2)) & 0x33333333u;
    a = (a | (a << 1)) & 0x55555555u;
    return a;
}
inline int64_t splat_index(int x, int y, int p, int np, int w) {
    int tx = x >> 6, ty = y >> 6, lx = x & 63, ly = y & 63;
    uint32_t code = spread((uint32_t)lx) | (spread((uint32_t)ly) << 1);
    int64_t tpr = (w + 63) >> 6;
    return ((int64_t)(ty * tpr + tx) * 4096 + code) * np + p;
}
inline uint64_t rgb36(V3 c) {
    return (((uint64_t)(c.x * 255.0f) & 0xFFF) << 24) | (((uint64_t)(c.y * 255.0f) & 0xFFF) << 12) | ((uint64_t)(c.z * 255.0f) & 0xFFF);
}

V3 normalize3(V3 v) { return mul(v, 1.0f / std::sqrt(dot3(v, v))); }

V3 sh_color_fp32(V3 pos, V3 campos, const float* sh) {
    V3 dir = normalize3(sub(pos, campos));
    auto S = [&](int i) { return v3(sh[3 * i], sh[3 * i + 1], sh[3 * i + 2]); };
    const real C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
    V3 r = mul(S(0), C0);
    real x = dir.x, y = dir.y, z = dir.z;
    r = sub(add(sub(r, mul(S(1), C1 * y)), mul(S(2), C1 * z)), mul(S(3), C1 * x));
    real xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    V3 b2 = add(add(add(add(mul(S(4), 1.0925484305920792f * xy), mul(S(5), -1.0925484305920792f * yz)),
                        mul(S(6), 0.31539156525252005f * (2.0f * zz - xx - yy))),
                    mul(S(7), -1.0925484305920792f * xz)),
                mul(S(8), 0.5462742152960396f * (xx - yy)));
    r = add(r, b2);
    V3 b3 = mul(S(9), -0.5900435899266435f * y * (3.0f * xx - yy));
    b3 = add(b3, mul(S(10), 2.890611442640554f * xy * z));
    b3 = add(b3, mul(S(11), -0.4570457994644658f * y * (4.0f * zz - xx - yy)));
    b3 = add(b3, mul(S(12), 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy)));
    b3 = add(b3, mul(S(13), -0.4570457994644658f * x * (4.0f * zz - xx - yy)));
    b3 = add(b3, mul(S(14), 1.445305721320277f * z * (xx - yy)));
    b3 = add(b3, mul(S(15), -0.5900435899266435f * x * (xx - 3.0f * yy)));
    r = add(r, b3);
    r = add(r, v3(0.5f, 0.5f, 0.5f));
    return v3(gmax(r.x, 0.0f), gmax(r.y, 0.0f), gmax(r.z, 0.0f));
}

// ---------------------------------------------------------------------------------
// the oracle context: one scene + settings + frame state
// ---------------------------------------------------------------------------------
struct Gaussian {  // the caller's CPUGaussian layout, kept in FP32
    float mean[3];
    float sh[48];
    float opacity;
    float scale[3];
    float rot[4];
};

struct Hiz {
    int w = 0, h = 0, levels = 0;
    std::vector<int> lw, lh;
    std::vector<size_t> off;
    std::vector<float> mip;  // depth chain, FP32 like the caller's depth image
};

struct Record {
    real pm[2], c0, c1, c2, conic[3], opacity;
    int mnx, mny, mxx, mxy;
    uint64_t key;
    real color[3];
};

struct Ctx {
    std::vector<Gaussian> g;
    gps_settings s;
    int up_w, up_h;
    size_t entries;
    std::vector<uint64_t> buffer;
    std::vector<uint32_t> counts, mask[2], block_culled;
    std::vector<Record> rec;
    std::vector<float> nodes;  // 6 per node (min xyz, max xyz), FP32 like the reference's blocks
    uint32_t per_block = 4, node_count = 0;
    uint32_t iteration = 0;
    Hiz hiz;
    int threads = 1;
    // last pass workload
    std::vector<uint32_t> surv_gid, surv_start;
    uint32_t points = 0, total = 0;
    uint32_t pts_pass[2] = {0, 0};
};

// Dynamic chunks (about 64 per thread) taken from a shared counter: the work per item is very
// uneven (a survivor's point count, a culled vs visible chunk), so equal static ranges leave
// most threads idle behind the densest one.
template <class F>
void par_for(int threads, size_t n, F f) {
    if (threads <= 1 || n < 1024) {
        f(0, n);
        return;
    }
    const size_t grain = std::max<size_t>(16, n / ((size_t)threads * 64));
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const size_t b = next.fetch_add(grain, std::memory_order_relaxed);
            if (b >= n) return;
            f(b, std::min(n, b + grain));
        }
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < threads; ++t) ts.emplace_back(worker);
    worker();
    for (auto& t : ts) t.join();
}

void hiz_init(Hiz& h, int w, int hh) {
    h.w = w;
    h.h = hh;
    int e = 0;
    while ((1 << e) < std::max(w, hh)) ++e;
    h.levels = e + 1;
    h.lw.resize(h.levels);
    h.lh.resize(h.levels);
    h.off.resize(h.levels);
    size_t o = 0;
    for (int l = 0; l < h.levels; ++l) {
        int fe = h.levels - 1;
        h.lw[l] = std::max(1, (w + (1 << (fe - l)) - 1) >> (fe - l));
        h.lh[l] = std::max(1, (hh + (1 << (fe - l)) - 1) >> (fe - l));
        h.off[l] = o;
        o += (size_t)h.lw[l] * h.lh[l];
    }
    h.mip.assign(o, INFINITY);
}

void hiz_build(Hiz& h, const float* depth, int min_levels) {
    int fl = h.levels - 1;
    std::memcpy(&h.mip[h.off[fl]], depth, sizeof(float) * (size_t)h.lw[fl] * h.lh[fl]);
    for (int l = h.levels - 2; l >= 0; --l) {
        bool use_min = ((h.levels - 2) - l) < min_levels;
        int wl = h.lw[l], hl = h.lh[l], wf = h.lw[l + 1], hf = h.lh[l + 1];
        for (int y = 0; y < hl; ++y)
            for (int x = 0; x < wl; ++x) {
                float v = use_min ? INFINITY : -INFINITY;
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) {
                        int fx = 2 * x + dx, fy = 2 * y + dy;
                        if (fx < wf && fy < hf) {
                            float f = h.mip[h.off[l + 1] + (size_t)fy * wf + fx];
                            v = use_min ? std::fmin(v, f) : std::fmax(v, f);
                        }
                    }
                h.mip[h.off[l] + (size_t)y * wl + x] = v;
            }
    }
}

bool hiz_occluded(const Hiz& c, real depth, int mnx, int mny, int mxx, int mxy) {
    mnx = std::max(0, mnx);
    mny = std::max(0, mny);
    mxx = std::min(c.w - 1, mxx);
    mxy = std::min(c.h - 1, mxy);
    int d = std::max(mxx - mnx + 1, mxy - mny + 1);
    int lod = (int)std::ceil(std::log2((real)d / 2.0f));
    lod = std::min(std::max(lod, 0), c.levels - 1);
    int l = (c.levels - 1) - lod;
    int wl = c.lw[l], hl = c.lh[l];
    int tw = std::max(1, std::min(c.w, 1 << (c.levels - l - 1)));
    int th = std::max(1, std::min(c.h, 1 << (c.levels - l - 1)));
    int tx0 = std::max(0, std::min(wl - 1, mnx / tw)), ty0 = std::max(0, std::min(hl - 1, mny / th)) * wl;
    int tx1 = std::max(0, std::min(wl - 1, mxx / tw)), ty1 = std::max(0, std::min(hl - 1, mxy / th)) * wl;
    const float* b = &c.mip[c.off[l]];
    float z = std::fmax(b[tx0 + ty0], std::fmax(b[tx1 + ty0], std::fmax(b[tx0 + ty1], b[tx1 + ty1])));
    return z < depth;
}

struct FrameC {
    M4 vp, view, cam;
    V2 tan_fov, focal;
    V4 planes[6];
};

FrameC derive(const Ctx& c, const gps_camera* cam) {
    FrameC f;
    f.view = m4_from(cam->view);
    M4 proj = m4_from(cam->proj);
    f.cam = affine_inverse(f.view);
    f.vp = mul(proj, f.view);
    real r = (real)c.s.width / (real)c.s.height;
    real tfy = std::tan(c.s.fovy * 0.01745329251994329576923690768489f * 0.5f);
    real fovx = 2.0f * std::atan(tfy * r);
    real tfx = std::tan(fovx * 0.5f);
    f.tan_fov = {tfx, tfy};
    f.focal = {(real)(c.s.width * c.s.supersampling_factor) / (2.0f * tfx), (real)(c.s.height * c.s.supersampling_factor) / (2.0f * tfy)};
    for (int i = 0; i < 6; ++i)
        f.planes[i] = v4(cam->frustum_planes[4 * i], cam->frustum_planes[4 * i + 1], cam->frustum_planes[4 * i + 2], cam->frustum_planes[4 * i + 3]);
    return f;
}

void block_cull(Ctx& c, const FrameC& f) {
    uint32_t words = (c.node_count + 31) / 32;
    c.block_culled.assign(words, 0);
    for (uint32_t i = 0; i < c.node_count; ++i) {
        V3 mn = v3(c.nodes[6 * i], c.nodes[6 * i + 1], c.nodes[6 * i + 2]);
        V3 mx = v3(c.nodes[6 * i + 3], c.nodes[6 * i + 4], c.nodes[6 * i + 5]);
        bool culled = false;
        for (int p = 0; p < 6; ++p) {
            V3 n = v3(f.planes[p].x, f.planes[p].y, f.planes[p].z);
            V3 v = v3(n.x >= 0 ? mx.x : mn.x, n.y >= 0 ? mx.y : mn.y, n.z >= 0 ? mx.z : mn.z);
            if (dot3(n, v) + f.planes[p].w < 0.0f) { culled = true; break; }
        }
        if (!culled && c.s.enable_occlusion_culling) {
            int minx = c.hiz.w - 1, miny = c.hiz.h - 1, maxx = 0, maxy = 0;
            real md = 1e30f;
            bool any = false;
            for (int k = 0; k < 8; ++k) {
                V4 p = v4((k & 1) ? mx.x : mn.x, (k & 2) ? mx.y : mn.y, (k & 4) ? mx.z : mn.z, 1.0f);
                V4 cl = mul(f.vp, p);
                if (cl.w <= 0.0f) continue;
                any = true;
                real nx = cl.x / cl.w, ny = cl.y / cl.w, nz = cl.z / cl.w;
                int px = (int)((nx * 0.5f + 0.5f) * c.hiz.w), py = (int)((ny * 0.5f + 0.5f) * c.hiz.h);
                minx = std::min(minx, px);
                miny = std::min(miny, py);
                maxx = std::max(maxx, px);
                maxy = std::max(maxy, py);
                md = std::fmin(md, nz);
            }
            if (any) {
                minx = std::max(minx, 0);
                miny = std::max(miny, 0);
                maxx = std::min(maxx, c.hiz.w - 1);
                maxy = std::min(maxy, c.hiz.h - 1);
                if (!(minx > maxx || miny > maxy)) culled = hiz_occluded(c.hiz, md, minx, miny, maxx, maxy);
            }
        }
        if (culled) c.block_culled[i >> 5] |= 1u << (i & 31);
    }
}

// Geometry of Gaussian idx (loadAndTransformGaussian + the splat's per-Gaussian prologue):
// fills everything of the record except the colour; false if the Gaussian is rejected.
bool geometry_record(const Ctx& c, const FrameC& f, uint32_t idx, Record& r, real& ndc_z, real& det_out,
                     V3& cov2d_out) {
    const gps_settings& s = c.s;
    const Gaussian& g = c.g[idx];
    V3 mean = v3(g.mean[0], g.mean[1], g.mean[2]);
    V3 view_mean = transform_point4x3(mean, f.view);
    real view_z = view_mean.z;
    if (-view_z <= 0.2f) return false;
    V4 pmn = mul(f.vp, v4(mean.x, mean.y, mean.z, 1.0f));
    pmn = mul(pmn, 1.0f / pmn.w);
    if (pmn.z < -1.0f || pmn.z > 1.0f) return false;
    M3 cov = scale_rot_to_cov(v3(g.scale[0], g.scale[1], g.scale[2]), v4(g.rot[0], g.rot[1], g.rot[2], g.rot[3]));
    V3 cov2d = compute_cov2d(f.view, cov, mean, f.tan_fov, f.focal);
    real dil = 0.3f * (real)s.supersampling_factor * (real)s.supersampling_factor;
    cov2d = v3(cov2d.x + dil, cov2d.y + 0.0f, cov2d.z + dil);
    real det = cov2d.x * cov2d.z - cov2d.y * cov2d.y;
    if (det <= 0.0f) return false;
    V2 pm = {(pmn.x * 0.5f + 0.5f) * (real)c.up_w, (pmn.y * 0.5f + 0.5f) * (real)c.up_h};
    int mnx, mny, mxx, mxy;
    if (!tile_bounds(mnx, mny, mxx, mxy, c.up_w, c.up_h, cov2d, pm)) return false;
    r.pm[0] = pm.x;
    r.pm[1] = pm.y;
    r.c0 = std::sqrt(cov2d.x);
    r.c1 = cov2d.y / r.c0;
    r.c2 = std::sqrt(cov2d.z - r.c1 * r.c1);
    real inv_det = 1.0f / det;
    r.conic[0] = cov2d.z * inv_det;
    r.conic[1] = -cov2d.y * inv_det;
    r.conic[2] = cov2d.x * inv_det;
    r.opacity = gmin(g.opacity, 1.0f);
    r.mnx = mnx;
    r.mny = mny;
    r.mxx = mxx;
    r.mxy = mxy;
    r.key = depth_key(view_z, s.near_view_plane, s.far_view_plane) << 36;
    ndc_z = pmn.z;
    det_out = det;
    cov2d_out = cov2d;
    return true;
}

void record_color(const Ctx& c, const FrameC& f, uint32_t idx, Record& r) {
    const Gaussian& g = c.g[idx];
    V3 campos = v3(f.cam.c[3].x, f.cam.c[3].y, f.cam.c[3].z);
    V3 col = sh_color_fp32(v3(g.mean[0], g.mean[1], g.mean[2]), campos, g.sh);
    r.color[0] = col.x;
    r.color[1] = col.y;
    r.color[2] = col.z;
    r.key = (r.key & (0xFFFFFFFull << 36)) | rgb36(col);
}

void splat_samples(Ctx& c, Seed& seed, const Record& r);

// One preprocess of Gaussian idx; returns the point count (0 = no points) and fills rec.
// With immediate_splat_threshold > 0, a Gaussian of at most that many points is splatted here
// from the seed state the point count left, and counts as no points
// (ENABLE_IMMEDIATE_SPLATTING, gaussian_point_splatting.cu:272-287, splatGaussianPoint :67-141).
uint32_t preprocess_one(Ctx& c, const FrameC& f, uint32_t idx, int frame_seed, bool only_prev,
                        const std::vector<uint32_t>& mask_prev, Record& r) {
    const gps_settings& s = c.s;
    Seed seed = make_seed(idx, (uint32_t)frame_seed);
    bool hier = s.enable_hierarchical_culling && !s.fully_disable_hierarchical_culling;
    if (hier) {
        uint32_t node = idx / c.per_block;
        if ((c.block_culled[node >> 5] >> (node & 31)) & 1u) return 0;
    }
    if (only_prev && ((mask_prev[idx >> 5] >> (idx & 31)) & 1u)) return 0;
    real opacity = gmin(c.g[idx].opacity, 1.0f);
    if (opacity <= 0.0f) return 0;
    real ndc_z, det;
    V3 cov2d;
    if (!geometry_record(c, f, idx, r, ndc_z, det, cov2d)) return 0;
    if (r.mnx >= c.up_w || r.mny >= c.up_h || r.mxx < 0 || r.mxy < 0) return 0;
    if (s.cull_small_gaussians) {
        real half = 0.5f * (cov2d.x + cov2d.z);
        real t2 = std::sqrt(std::fmax(0.1f, half * half - det));
        if (half + t2 < 0.02f || half - t2 < 0.02f) return 0;
    }
    real sdet = std::sqrt(det);
    const real two_pi = 2.0f * 3.14159265358979323846f;
    real importance = s.use_unbiased_2d_splatting ? two_pi * sdet * dilog(opacity) : opacity * two_pi * sdet;
    const int ss = s.supersampling_factor;
    if (s.enable_occlusion_culling && hiz_occluded(c.hiz, ndc_z, r.mnx / ss, r.mny / ss, r.mxx / ss, r.mxy / ss))
        return 0;
    real k = (real)(s.points_per_thread > 0 ? s.points_per_thread : ss * ss);
    if (!s.reduce_point_count) k = 1.0f;
    uint32_t n = s.use_unbiased_2d_splatting ? poisson(seed, importance) : (uint32_t)stochastic_round(importance, pcg2d(seed).x);
    if (k > 1) n = (uint32_t)stochastic_round((real)n / k, pcg2d(seed).x);
    if (n == 0) return 0;
    uint32_t cap = (uint32_t)(c.up_w * c.up_h / (2 * k));
    n = std::min(n, cap);
    record_color(c, f, idx, r);
    if (s.immediate_splat_threshold > 0 && (int)n <= s.immediate_splat_threshold) {
        for (uint32_t pt = 0; pt < n; ++pt) splat_samples(c, seed, r);
        return 0;
    }
    return n;
}

void preprocess_pass(Ctx& c, const FrameC& f, int frame_seed, bool first) {
    uint32_t n = (uint32_t)c.g.size();
    std::vector<uint32_t>& cur = c.mask[c.iteration % 2];
    const std::vector<uint32_t>& prev = c.mask[(c.iteration + 1) % 2];
    std::fill(cur.begin(), cur.end(), 0u);
    // words are independent: split by 32-Gaussian words
    par_for(c.threads, (n + 31) / 32, [&](size_t wb, size_t we) {
        for (size_t w = wb; w < we; ++w) {
            uint32_t bits = 0;
            for (uint32_t i = (uint32_t)w * 32; i < std::min<uint32_t>(n, (uint32_t)w * 32 + 32); ++i) {
                Record r;
                uint32_t np = preprocess_one(c, f, i, frame_seed, !first, prev, r);
                if (np > 0) {
                    c.counts[i] = np;
                    c.rec[i] = r;
                    bits |= 1u << (i & 31);
                }
            }
            cur[w] = bits;
        }
    });
}

void scan_pass(Ctx& c) {
    uint32_t n = (uint32_t)c.g.size();
    const std::vector<uint32_t>& cur = c.mask[c.iteration % 2];
    c.surv_gid.clear();
    c.surv_start.clear();
    uint32_t pt = 0;
    for (uint32_t i = 0; i < n; ++i)
        if ((cur[i >> 5] >> (i & 31)) & 1u) {
            c.surv_gid.push_back(i);
            c.surv_start.push_back(pt);
            pt += c.counts[i];
        }
    c.total = pt;
    c.points = std::min<uint32_t>(pt, (uint32_t)std::max(0, c.s.max_number_of_points));
}

inline void atomic_min64(uint64_t* p, uint64_t v) {
    auto* a = reinterpret_cast<std::atomic<uint64_t>*>(p);
    uint64_t old = a->load(std::memory_order_relaxed);
    while (old > v && !a->compare_exchange_weak(old, v, std::memory_order_relaxed)) {
    }
}
inline void atomic_add_color(uint64_t* p, uint64_t v) {
    const uint64_t dm = 0xFFFFFFFull << 36, cm = (1ull << 36) - 1;
    auto* a = reinterpret_cast<std::atomic<uint64_t>*>(p);
    uint64_t old = a->load(std::memory_order_relaxed);
    for (;;) {
        uint64_t td = v & dm, ad = old & dm, nv = v;
        if (td > ad) return;
        if (td == ad) nv = (old & dm) | (((old & cm) + (v & cm)) & cm);
        if (a->compare_exchange_weak(old, nv, std::memory_order_relaxed)) return;
    }
}

// One point's samples from `seed` onwards (splatGaussianPoint's inner loop, :98-139).
void splat_samples(Ctx& c, Seed& seed, const Record& r) {
    const gps_settings& s = c.s;
    int k = !s.reduce_point_count ? 1 : s.points_per_thread > 0 ? s.points_per_thread : s.supersampling_factor * s.supersampling_factor;
    const int np = s.samples_per_pixel;
    const uint64_t vdb = r.key & (0xFFFFFFFull << 36);
    for (int q = 0; q < np * k; ++q) {
        V2 u = pcg2d(seed);
        V2 xy = s.use_unbiased_2d_splatting ? corrected_box_muller(u.x, u.y, r.opacity) : box_muller(u.x, u.y);
        real px = std::floor(r.pm[0] + r.c0 * xy.x), py = std::floor(r.pm[1] + r.c1 * xy.x + r.c2 * xy.y);
        int x = (int)px, y = (int)py;
        real dx = r.pm[0] - px, dy = r.pm[1] - py;
        if (x < r.mnx || x >= r.mxx || y < r.mny || y >= r.mxy) continue;
        real sig = -0.5f * (r.conic[0] * dx * dx + r.conic[2] * dy * dy) - r.conic[1] * dx * dy;
        real gw = sig > 0.0f ? 0.0f : std::exp(sig);
        if (r.opacity * gw < 1.0f / 255.0f) continue;
        int64_t idx = splat_index(x, y, q / k, np, c.up_w);
        uint64_t* slot = &c.buffer[(size_t)idx];
        if (reinterpret_cast<std::atomic<uint64_t>*>(slot)->load(std::memory_order_relaxed) <= vdb) continue;
        if (s.use_unbiased_2d_splatting) atomic_min64(slot, r.key);
        else atomic_add_color(slot, r.key);
    }
}

void splat_point(Ctx& c, uint32_t p, const Record& r, int frame_seed) {
    Seed seed = make_seed(p, (uint32_t)frame_seed);
    splat_samples(c, seed, r);
}

void splat_pass(Ctx& c, int frame_seed, const uint32_t* gid, const uint32_t* start, uint32_t survivors, uint32_t points,
                const Record* recs) {
    par_for(c.threads, survivors, [&](size_t b, size_t e) {
        for (size_t r = b; r < e; ++r) {
            uint32_t p0 = start[r];
            uint32_t p1 = (r + 1 < survivors) ? start[r + 1] : points;
            if (p1 > points) p1 = points;
            for (uint32_t p = p0; p < p1; ++p) splat_point(c, p, recs[gid[r]], frame_seed);
        }
    });
}

void resolve(const Ctx& c, float* color, float* depth, bool depth_only) {
    const gps_settings& s = c.s;
    const int w = s.width, h = s.height, ss = s.supersampling_factor, np = s.samples_per_pixel;
    par_for(c.threads, (size_t)h, [&](size_t yb, size_t ye) {
        for (size_t y = yb; y < ye; ++y)
            for (int x = 0; x < w; ++x) {
                real d = 1e9f, cr = 0, cg = 0, cb = 0;
                for (int dx = 0; dx < ss; ++dx)
                    for (int dy = 0; dy < ss; ++dy)
                        for (int p = 0; p < np; ++p) {
                            int64_t i = splat_index(x * ss + dx, (int)y * ss + dy, p, np, c.up_w);
                            uint64_t v = c.buffer[(size_t)i];
                            real vd = view_depth_from_key((v >> 36) & 0xFFFFFFFull, s.near_view_plane, s.far_view_plane);
                            d = gmin(d, view_to_ndc(vd, s.near_view_plane, s.far_view_plane));
                            if (depth_only) continue;
                            cr += (real)((v >> 24) & 0xFFF) / 255.0f;
                            cg += (real)((v >> 12) & 0xFFF) / 255.0f;
                            cb += (real)(v & 0xFFF) / 255.0f;
                        }
                real inv = 1.0f / (real)(np * ss * ss);
                size_t idx = y * w + x;
                if (!depth_only) {
                    color[3 * idx] = cr * inv;
                    color[3 * idx + 1] = cg * inv;
                    color[3 * idx + 2] = cb * inv;
                }
                depth[idx] = d;
            }
    });
}

void render_pass(Ctx& c, const FrameC& f, int frame, bool first, int pass) {
    int fs = 4 * frame + (first ? 0 : 2);
    bool hier = c.s.enable_hierarchical_culling && !c.s.fully_disable_hierarchical_culling;
    if (hier) block_cull(c, f);
    preprocess_pass(c, f, fs, first);
    scan_pass(c);
    c.pts_pass[pass] = c.points;
    splat_pass(c, fs + 1, c.surv_gid.data(), c.surv_start.data(), (uint32_t)c.surv_gid.size(), c.points, c.rec.data());
    // WorkloadDistributor::build returns before iteration++ when the pass has no samples
    // (workload_distributor.cu:107-111,145): the mask pair keeps its order
    if (c.points > 0) c.iteration++;
}

}  // namespace

extern "C" {

struct oracle_ctx;

// Scene in CPUGaussian layout (59 floats each, already activated), settings as the C-ABI's.
oracle_ctx* oracle_create(const float* gaussians, uint64_t n, const gps_settings* s, int threads) {
    Ctx* c = new Ctx();
    c->g.resize(n);
    std::memcpy(c->g.data(), gaussians, n * sizeof(Gaussian));
    c->s = *s;
    c->up_w = s->width * s->supersampling_factor;
    c->up_h = s->height * s->supersampling_factor;
    size_t tx = (size_t)((c->up_w + 63) >> 6), ty = (size_t)((c->up_h + 63) >> 6);
    c->entries = tx * ty * 4096 * (size_t)s->samples_per_pixel;
    c->buffer.assign(c->entries, 0);
    c->counts.assign(n, 0);
    c->mask[0].assign((n + 31) / 32 + 1, 0);
    c->mask[1].assign((n + 31) / 32 + 1, 0);
    c->rec.resize(n);
    c->threads = std::max(1, threads);
    hiz_init(c->hiz, s->width, s->height);
    // fixed blocks (gaussian_bvh.cu:111-144,171-172) in IEEE host arithmetic
    float v = std::floor((float)n / 1e6f);
    c->per_block = (uint32_t)(int)gmax(4.0f, v);
    c->node_count = (uint32_t)((n + c->per_block - 1) / c->per_block);
    c->nodes.resize((size_t)c->node_count * 6);
    for (uint32_t b = 0; b < c->node_count; ++b) {
        float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint64_t i = (uint64_t)b * c->per_block; i < std::min<uint64_t>(n, (uint64_t)(b + 1) * c->per_block); ++i) {
            const Gaussian& g = c->g[i];
            M3 cov = scale_rot_to_cov(v3(g.scale[0], g.scale[1], g.scale[2]), v4(g.rot[0], g.rot[1], g.rot[2], g.rot[3]));
            float d[3] = {(float)cov.c[0].x, (float)cov.c[1].y, (float)cov.c[2].z};
            for (int k = 0; k < 3; ++k) {
                float e = 3.0f * std::sqrt(d[k]);
                float lo = g.mean[k] - e, hi = g.mean[k] + e;
                mn[k] = gmin(mn[k], lo);
                mx[k] = gmax(mx[k], hi);
            }
        }
        for (int k = 0; k < 3; ++k) {
            c->nodes[6 * b + k] = mn[k];
            c->nodes[6 * b + 3 + k] = mx[k];
        }
    }
    return reinterpret_cast<oracle_ctx*>(c);
}

void oracle_free(oracle_ctx* h) { delete reinterpret_cast<Ctx*>(h); }

// gaussian_point_splatting.cu:599-737 on the CPU; image is W*H*3 floats, depth W*H.
void oracle_render_frame(oracle_ctx* h, const gps_camera* cam, float* image, float* depth) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    FrameC f = derive(c, cam);
    uint64_t bg = 0xFFFFFFF000000000ull | rgb36(v3(c.s.background[0], c.s.background[1], c.s.background[2]));
    std::fill(c.buffer.begin(), c.buffer.end(), bg);
    c.pts_pass[0] = c.pts_pass[1] = 0;
    render_pass(c, f, cam->frame, true, 0);
    if (c.s.enable_occlusion_culling) {
        resolve(c, image, depth, true);
        hiz_build(c.hiz, depth, c.s.occlusion_culling_min_reduce_count);
        render_pass(c, f, cam->frame, false, 1);
    }
    resolve(c, image, depth, false);
    if (c.s.enable_occlusion_culling) hiz_build(c.hiz, depth, c.s.occlusion_culling_min_reduce_count);
}

// Splats an externally supplied workload (survivor ids, first points, total P) with this
// oracle's own per-Gaussian records of the given camera; the buffer is cleared first when
// clear != 0.  This isolates the per-sample arithmetic from count differences.
void oracle_splat_workload(oracle_ctx* h, const gps_camera* cam, int frame_seed, const uint32_t* surv_gid,
                           const uint32_t* surv_start, uint32_t survivors, uint32_t points, int clear) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    FrameC f = derive(c, cam);
    if (clear) {
        uint64_t bg = 0xFFFFFFF000000000ull | rgb36(v3(c.s.background[0], c.s.background[1], c.s.background[2]));
        std::fill(c.buffer.begin(), c.buffer.end(), bg);
    }
    par_for(c.threads, survivors, [&](size_t b, size_t e) {
        for (size_t r = b; r < e; ++r) {
            uint32_t g = surv_gid[r];
            Record rec;
            real ndc_z, det;
            V3 cov2d;
            if (geometry_record(c, f, g, rec, ndc_z, det, cov2d)) record_color(c, f, g, rec);
            else rec.mnx = rec.mny = rec.mxx = rec.mxy = 0;  // rejected here: no sample can land
            c.rec[g] = rec;
        }
    });
    splat_pass(c, frame_seed, surv_gid, surv_start, survivors, points, c.rec.data());
}

// One preprocess pass only (no splat); outputs counts (valid where the mask bit is set),
// the mask words, and per-Gaussian colours (3 floats, valid where the mask bit is set).
void oracle_preprocess(oracle_ctx* h, const gps_camera* cam, int first_pass, uint32_t* counts, uint32_t* mask,
                       float* colors) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    FrameC f = derive(c, cam);
    bool hier = c.s.enable_hierarchical_culling && !c.s.fully_disable_hierarchical_culling;
    if (hier) block_cull(c, f);
    preprocess_pass(c, f, 4 * cam->frame + (first_pass ? 0 : 2), first_pass != 0);
    const std::vector<uint32_t>& cur = c.mask[c.iteration % 2];
    size_t n = c.g.size();
    std::memcpy(mask, cur.data(), sizeof(uint32_t) * ((n + 31) / 32));
    for (size_t i = 0; i < n; ++i) {
        counts[i] = c.counts[i];
        colors[3 * i] = c.rec[i].color[0];
        colors[3 * i + 1] = c.rec[i].color[1];
        colors[3 * i + 2] = c.rec[i].color[2];
    }
    c.iteration++;
}

void oracle_get_buffer(oracle_ctx* h, uint64_t* out) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    std::memcpy(out, c.buffer.data(), c.buffer.size() * sizeof(uint64_t));
}
uint64_t oracle_buffer_entries(oracle_ctx* h) { return reinterpret_cast<Ctx*>(h)->entries; }
void oracle_get_hiz(oracle_ctx* h, float* out) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    std::memcpy(out, c.hiz.mip.data(), c.hiz.mip.size() * sizeof(float));
}
uint64_t oracle_hiz_size(oracle_ctx* h) { return reinterpret_cast<Ctx*>(h)->hiz.mip.size(); }
void oracle_last_workload(oracle_ctx* h, uint32_t* points_pass, uint32_t* survivors, uint32_t* total) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    points_pass[0] = c.pts_pass[0];
    points_pass[1] = c.pts_pass[1];
    *survivors = (uint32_t)c.surv_gid.size();
    *total = c.total;
}
void oracle_get_survivors(oracle_ctx* h, uint32_t* gid, uint32_t* start) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    std::memcpy(gid, c.surv_gid.data(), c.surv_gid.size() * 4);
    std::memcpy(start, c.surv_start.data(), c.surv_start.size() * 4);
}
void oracle_get_blocks(oracle_ctx* h, float* nodes6, uint32_t* per_block, uint32_t* count) {
    Ctx& c = *reinterpret_cast<Ctx*>(h);
    std::memcpy(nodes6, c.nodes.data(), c.nodes.size() * 4);
    *per_block = c.per_block;
    *count = c.node_count;
}

// ---- known-answer helpers (exact integer layer + reference float helpers) ------------
void oracle_kat(const uint32_t* idx, const uint32_t* frame, const float* x, int n, uint32_t* seeds, uint32_t* pcg,
                float* pcgf, float* dl, float* idl, uint32_t* pois, int32_t* sround) {
    for (int i = 0; i < n; ++i) {
        Seed s = make_seed(idx[i], frame[i]);
        seeds[2 * i] = s.x;
        seeds[2 * i + 1] = s.y;
        Seed q = pcg_step(s);
        pcg[2 * i] = q.x;
        pcg[2 * i + 1] = q.y;
        Seed st = s;
        V2 u = pcg2d(st);
        pcgf[2 * i] = u.x;
        pcgf[2 * i + 1] = u.y;
        dl[i] = dilog(x[i]);
        idl[i] = inv_dilog(x[i] * 1.6449340668482264f);
        Seed ps = s;
        pois[i] = poisson(ps, 0.05f + 60.0f * x[i]);
        sround[i] = stochastic_round(10.0f * x[i], u.y);
    }
}
void oracle_splat_index(const int32_t* xs, const int32_t* ys, const int32_t* ps, int n, int npass, int w, int64_t* out) {
    for (int i = 0; i < n; ++i) out[i] = splat_index(xs[i], ys[i], ps[i], npass, w);
}
void oracle_depth_key(const float* d, int n, float nearp, float farp, uint64_t* out) {
    for (int i = 0; i < n; ++i) out[i] = depth_key(d[i], nearp, farp);
}
void oracle_rgb36(const float* rgb, int n, uint64_t* out) {
    for (int i = 0; i < n; ++i) out[i] = rgb36(v3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
}

}  // extern "C"
