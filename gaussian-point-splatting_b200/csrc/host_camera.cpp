// Camera path JSON, camera matrices and the per-frame constants the renderer derives.
//
// Operation order follows the reference's host code (glm 1.0.2 scalar paths):
//   camera_loader.cu:26-41,62-90,123-150  cameras.json -> CameraState -> pose
//   transform.cpp:21-44, camera.cpp:88-98,126-156  model/view/projection/planes
//   main.cu:141-157                                per-frame view = diag(1,-1,-1,1)*view
//   gaussian_point_splatting.cu:605-615            vp, camera-to-world, tan_fov, focal
//   camera.h:39-47                                 focal <-> fov
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include "host_io.hpp"

namespace gps {

namespace {
constexpr int kStatusIo = 2;
constexpr int kStatusFormat = 3;

// ---- a small JSON reader (objects, arrays, numbers, strings, literals) --------------
struct JValue {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    double num = 0.0;
    bool b = false;
    std::string str;
    std::vector<JValue> arr;
    std::vector<std::pair<std::string, JValue>> obj;
    const JValue* get(const std::string& k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct JParser {
    const std::string& s;
    size_t i = 0;
    std::string err;
    explicit JParser(const std::string& src) : s(src) {}
    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    bool fail(const char* m) {
        if (err.empty()) err = std::string(m) + " at offset " + std::to_string(i);
        return false;
    }
    bool parse(JValue& v, int depth = 0) {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (i >= s.size()) return fail("unexpected end");
        char c = s[i];
        if (c == '{') {
            v.kind = JValue::Object;
            ++i;
            ws();
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            for (;;) {
                ws();
                JValue key;
                if (i >= s.size() || s[i] != '"') return fail("expected key");
                if (!parse_string(key.str)) return false;
                ws();
                if (i >= s.size() || s[i] != ':') return fail("expected ':'");
                ++i;
                JValue val;
                if (!parse(val, depth + 1)) return false;
                v.obj.emplace_back(key.str, std::move(val));
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == '}') { ++i; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JValue::Array;
            ++i;
            ws();
            if (i < s.size() && s[i] == ']') { ++i; return true; }
            for (;;) {
                JValue val;
                if (!parse(val, depth + 1)) return false;
                v.arr.push_back(std::move(val));
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == ']') { ++i; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JValue::String;
            return parse_string(v.str);
        }
        if (s.compare(i, 4, "true") == 0) { v.kind = JValue::Bool; v.b = true; i += 4; return true; }
        if (s.compare(i, 5, "false") == 0) { v.kind = JValue::Bool; v.b = false; i += 5; return true; }
        if (s.compare(i, 4, "null") == 0) { v.kind = JValue::Null; i += 4; return true; }
        const char* begin = s.c_str() + i;
        char* end = nullptr;
        double d = std::strtod(begin, &end);
        if (end == begin) return fail("invalid value");
        v.kind = JValue::Number;
        v.num = d;
        i += (size_t)(end - begin);
        return true;
    }
    bool parse_string(std::string& out) {
        ++i;  // opening quote
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) {
                char e = s[i + 1];
                if (e == 'n') out += '\n';
                else if (e == 't') out += '\t';
                else if (e == 'u' && i + 5 < s.size()) { out += '?'; i += 4; }
                else out += e;
                i += 2;
            } else {
                out += s[i++];
            }
        }
        if (i >= s.size()) return fail("unterminated string");
        ++i;
        return true;
    }
};

bool num_of(const JValue* v, float& out) {
    if (!v || v->kind != JValue::Number) return false;
    out = (float)v->num;
    return true;
}
bool int_of(const JValue* v, int& out) {
    if (!v || v->kind != JValue::Number) return false;
    out = (int)v->num;
    return true;
}

// host mat4 helpers, glm's scalar order
mat4 mat4_identity() {
    mat4 m;
    for (int c = 0; c < 4; ++c) m.c[c] = make_v4(c == 0, c == 1, c == 2, c == 3);
    return m;
}
vec4 v4_add(vec4 a, vec4 b) { return make_v4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
vec4 v4_sub(vec4 a, vec4 b) { return make_v4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
vec4 v4_mul(vec4 a, float s) { return make_v4(a.x * s, a.y * s, a.z * s, a.w * s); }
vec4 v4_div(vec4 a, float s) { return make_v4(a.x / s, a.y / s, a.z / s, a.w / s); }

mat4 translate(const mat4& m, vec3 v) {
    mat4 r = m;
    vec4 t = v4_mul(m.c[0], v.x);
    t = v4_add(t, v4_mul(m.c[1], v.y));
    t = v4_add(t, v4_mul(m.c[2], v.z));
    t = v4_add(t, m.c[3]);
    r.c[3] = t;
    return r;
}
mat4 scale4(const mat4& m, vec3 v) {
    mat4 r;
    r.c[0] = v4_mul(m.c[0], v.x);
    r.c[1] = v4_mul(m.c[1], v.y);
    r.c[2] = v4_mul(m.c[2], v.z);
    r.c[3] = m.c[3];
    return r;
}
mat4 mat4_from_mat3(const mat3& m) {
    mat4 r;
    r.c[0] = make_v4(m.c[0].x, m.c[0].y, m.c[0].z, 0.0f);
    r.c[1] = make_v4(m.c[1].x, m.c[1].y, m.c[1].z, 0.0f);
    r.c[2] = make_v4(m.c[2].x, m.c[2].y, m.c[2].z, 0.0f);
    r.c[3] = make_v4(0.0f, 0.0f, 0.0f, 1.0f);
    return r;
}
// glm::mat3_cast for a quaternion (w, x, y, z)
mat3 mat3_cast(const float q[4]) {
    const float w = q[0], x = q[1], y = q[2], z = q[3];
    vec4 qq = make_v4(x, y, z, w);
    (void)qq;
    float qxx = x * x, qyy = y * y, qzz = z * z;
    float qxz = x * z, qxy = x * y, qyz = y * z;
    float qwx = w * x, qwy = w * y, qwz = w * z;
    mat3 r;
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
// glm::inverse(mat3), scalar path (func_matrix.inl inv3x3<false>)
mat3 inverse3(const mat3& m) {
    auto e = [&](int c, int r) { return (r == 0) ? m.c[c].x : (r == 1) ? m.c[c].y : m.c[c].z; };
    float one_over_det = 1.0f / (+e(0, 0) * (e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2)) -
                                 e(1, 0) * (e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2)) +
                                 e(2, 0) * (e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2)));
    float inv[3][3];
    inv[0][0] = +(e(1, 1) * e(2, 2) - e(2, 1) * e(1, 2));
    inv[1][0] = -(e(1, 0) * e(2, 2) - e(2, 0) * e(1, 2));
    inv[2][0] = +(e(1, 0) * e(2, 1) - e(2, 0) * e(1, 1));
    inv[0][1] = -(e(0, 1) * e(2, 2) - e(2, 1) * e(0, 2));
    inv[1][1] = +(e(0, 0) * e(2, 2) - e(2, 0) * e(0, 2));
    inv[2][1] = -(e(0, 0) * e(2, 1) - e(2, 0) * e(0, 1));
    inv[0][2] = +(e(0, 1) * e(1, 2) - e(1, 1) * e(0, 2));
    inv[1][2] = -(e(0, 0) * e(1, 2) - e(1, 0) * e(0, 2));
    inv[2][2] = +(e(0, 0) * e(1, 1) - e(1, 0) * e(0, 1));
    mat3 r;
    for (int c = 0; c < 3; ++c) r.c[c] = make_v3(inv[c][0] * one_over_det, inv[c][1] * one_over_det, inv[c][2] * one_over_det);
    return r;
}
mat4 perspective(float fovy, float aspect, float z_near, float z_far) {
    float t = std::tan(fovy / 2.0f);
    mat4 r;
    for (int c = 0; c < 4; ++c) r.c[c] = make_v4(0, 0, 0, 0);
    r.c[0].x = 1.0f / (aspect * t);
    r.c[1].y = 1.0f / t;
    r.c[2].z = -(z_far + z_near) / (z_far - z_near);
    r.c[2].w = -1.0f;
    r.c[3].z = -(2.0f * z_far * z_near) / (z_far - z_near);
    return r;
}
float radians(float deg) { return deg * 0.01745329251994329576923690768489f; }
}  // namespace

mat4 mat4_mul(const mat4& a, const mat4& b) {
    mat4 r;
    for (int j = 0; j < 4; ++j) {
        vec4 t = v4_mul(a.c[0], b.c[j].x);
        t = v4_add(t, v4_mul(a.c[1], b.c[j].y));
        t = v4_add(t, v4_mul(a.c[2], b.c[j].z));
        t = v4_add(t, v4_mul(a.c[3], b.c[j].w));
        r.c[j] = t;
    }
    return r;
}

// glm::affineInverse(mat4) (gtc/matrix_inverse.inl)
mat4 affine_inverse(const mat4& m) {
    mat3 inv = inverse3(mat3_of(m));
    mat3 neg;
    for (int c = 0; c < 3; ++c) neg.c[c] = make_v3(-inv.c[c].x, -inv.c[c].y, -inv.c[c].z);
    vec3 t = make_v3(m.c[3].x, m.c[3].y, m.c[3].z);
    vec3 nt = neg.c[0] * t.x + neg.c[1] * t.y + neg.c[2] * t.z;
    mat4 r;
    r.c[0] = make_v4(inv.c[0].x, inv.c[0].y, inv.c[0].z, 0.0f);
    r.c[1] = make_v4(inv.c[1].x, inv.c[1].y, inv.c[1].z, 0.0f);
    r.c[2] = make_v4(inv.c[2].x, inv.c[2].y, inv.c[2].z, 0.0f);
    r.c[3] = make_v4(nt.x, nt.y, nt.z, 1.0f);
    return r;
}

// glm::inverse(mat4) (func_matrix.inl compute_inverse<4,4>)
mat4 inverse4(const mat4& mm) {
    auto m = [&](int c, int r) { const vec4& v = mm.c[c]; return r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w; };
    float c00 = m(2, 2) * m(3, 3) - m(3, 2) * m(2, 3);
    float c02 = m(1, 2) * m(3, 3) - m(3, 2) * m(1, 3);
    float c03 = m(1, 2) * m(2, 3) - m(2, 2) * m(1, 3);
    float c04 = m(2, 1) * m(3, 3) - m(3, 1) * m(2, 3);
    float c06 = m(1, 1) * m(3, 3) - m(3, 1) * m(1, 3);
    float c07 = m(1, 1) * m(2, 3) - m(2, 1) * m(1, 3);
    float c08 = m(2, 1) * m(3, 2) - m(3, 1) * m(2, 2);
    float c10 = m(1, 1) * m(3, 2) - m(3, 1) * m(1, 2);
    float c11 = m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2);
    float c12 = m(2, 0) * m(3, 3) - m(3, 0) * m(2, 3);
    float c14 = m(1, 0) * m(3, 3) - m(3, 0) * m(1, 3);
    float c15 = m(1, 0) * m(2, 3) - m(2, 0) * m(1, 3);
    float c16 = m(2, 0) * m(3, 2) - m(3, 0) * m(2, 2);
    float c18 = m(1, 0) * m(3, 2) - m(3, 0) * m(1, 2);
    float c19 = m(1, 0) * m(2, 2) - m(2, 0) * m(1, 2);
    float c20 = m(2, 0) * m(3, 1) - m(3, 0) * m(2, 1);
    float c22 = m(1, 0) * m(3, 1) - m(3, 0) * m(1, 1);
    float c23 = m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1);
    vec4 f0 = make_v4(c00, c00, c02, c03), f1 = make_v4(c04, c04, c06, c07), f2 = make_v4(c08, c08, c10, c11);
    vec4 f3 = make_v4(c12, c12, c14, c15), f4 = make_v4(c16, c16, c18, c19), f5 = make_v4(c20, c20, c22, c23);
    vec4 v0 = make_v4(m(1, 0), m(0, 0), m(0, 0), m(0, 0));
    vec4 v1 = make_v4(m(1, 1), m(0, 1), m(0, 1), m(0, 1));
    vec4 v2 = make_v4(m(1, 2), m(0, 2), m(0, 2), m(0, 2));
    vec4 v3 = make_v4(m(1, 3), m(0, 3), m(0, 3), m(0, 3));
    auto mul = [](vec4 a, vec4 b) { return make_v4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); };
    vec4 i0 = v4_add(v4_sub(mul(v1, f0), mul(v2, f1)), mul(v3, f2));
    vec4 i1 = v4_add(v4_sub(mul(v0, f0), mul(v2, f3)), mul(v3, f4));
    vec4 i2 = v4_add(v4_sub(mul(v0, f1), mul(v1, f3)), mul(v3, f5));
    vec4 i3 = v4_add(v4_sub(mul(v0, f2), mul(v1, f4)), mul(v2, f5));
    vec4 sa = make_v4(+1, -1, +1, -1), sb = make_v4(-1, +1, -1, +1);
    mat4 inv;
    inv.c[0] = mul(i0, sa);
    inv.c[1] = mul(i1, sb);
    inv.c[2] = mul(i2, sa);
    inv.c[3] = mul(i3, sb);
    vec4 row0 = make_v4(inv.c[0].x, inv.c[1].x, inv.c[2].x, inv.c[3].x);
    vec4 d0 = mul(mm.c[0], row0);
    float d1 = (d0.x + d0.y) + (d0.z + d0.w);
    float one_over = 1.0f / d1;
    for (int c = 0; c < 4; ++c) inv.c[c] = v4_mul(inv.c[c], one_over);
    return inv;
}

void quat_from_basis(const mat3& m, float q[4]) {
    auto e = [&](int c, int r) { return (r == 0) ? m.c[c].x : (r == 1) ? m.c[c].y : m.c[c].z; };
    float fx = e(0, 0) - e(1, 1) - e(2, 2);
    float fy = e(1, 1) - e(0, 0) - e(2, 2);
    float fz = e(2, 2) - e(0, 0) - e(1, 1);
    float fw = e(0, 0) + e(1, 1) + e(2, 2);
    int bi = 0;
    float fb = fw;
    if (fx > fb) { fb = fx; bi = 1; }
    if (fy > fb) { fb = fy; bi = 2; }
    if (fz > fb) { fb = fz; bi = 3; }
    float big = std::sqrt(fb + 1.0f) * 0.5f;
    float mult = 0.25f / big;
    switch (bi) {
        case 0: q[0] = big; q[1] = (e(1, 2) - e(2, 1)) * mult; q[2] = (e(2, 0) - e(0, 2)) * mult; q[3] = (e(0, 1) - e(1, 0)) * mult; break;
        case 1: q[0] = (e(1, 2) - e(2, 1)) * mult; q[1] = big; q[2] = (e(0, 1) + e(1, 0)) * mult; q[3] = (e(2, 0) + e(0, 2)) * mult; break;
        case 2: q[0] = (e(2, 0) - e(0, 2)) * mult; q[1] = (e(0, 1) + e(1, 0)) * mult; q[2] = big; q[3] = (e(1, 2) + e(2, 1)) * mult; break;
        default: q[0] = (e(0, 1) - e(1, 0)) * mult; q[1] = (e(2, 0) + e(0, 2)) * mult; q[2] = (e(1, 2) + e(2, 1)) * mult; q[3] = big; break;
    }
}

float focal_to_fov_deg(float focal, int pixels) {
    float fovr = (float)(2.0 * (double)atanf(0.5f * (float)pixels / focal));
    return fovr * 57.2957795f;
}
float fov_deg_to_focal(float fovdeg, int pixels) {
    float fovr = (float)((double)fovdeg * 0.01745329);
    return (float)((double)pixels / (2.0 * (double)tanf((float)((double)fovr / 2.0))));
}

CameraMatrices camera_matrices(vec3 position, const float quat_wxyz[4], float fovy, float aspect, float near_plane,
                               float far_plane) {
    // Transform::getModelMatrix: translate(I, pos) * mat4_cast(rot) * scale(1)
    mat4 model = translate(mat4_identity(), position);
    model = mat4_mul(model, mat4_from_mat3(mat3_cast(quat_wxyz)));
    model = scale4(model, make_v3(1.0f, 1.0f, 1.0f));
    mat4 cam_view = affine_inverse(model);
    mat4 flip = scale4(mat4_identity(), make_v3(1.0f, -1.0f, -1.0f));
    CameraMatrices out;
    out.view = mat4_mul(mat4_mul(flip, cam_view), mat4_identity());
    out.proj = perspective(radians(fovy), aspect, near_plane, far_plane);
    // getFrustumPlanesFromViewMatrix
    mat4 vp = mat4_mul(perspective(radians(fovy), aspect, near_plane, far_plane), out.view);
    mat4 t;
    for (int c = 0; c < 4; ++c) {
        const float* col = &vp.c[c].x;
        (void)col;
    }
    auto el = [&](int c, int r) { const vec4& v = vp.c[c]; return r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w; };
    for (int c = 0; c < 4; ++c) t.c[c] = make_v4(el(0, c), el(1, c), el(2, c), el(3, c));
    out.planes[0] = v4_add(t.c[3], t.c[0]);
    out.planes[1] = v4_sub(t.c[3], t.c[0]);
    out.planes[2] = v4_add(t.c[3], t.c[1]);
    out.planes[3] = v4_sub(t.c[3], t.c[1]);
    out.planes[4] = v4_add(t.c[3], t.c[2]);
    out.planes[5] = v4_sub(t.c[3], t.c[2]);
    for (auto& p : out.planes) {
        vec3 n = make_v3(p.x, p.y, p.z);
        float len = std::sqrt(dot(n, n));
        if (len > 0.0f) p = v4_div(p, len);
    }
    out.position = position;
    return out;
}

void derive_frame(const mat4& view, const mat4& proj, int width, int height, int ss, float fovy, mat4& vp, mat4& cam,
                  vec2& tan_fov, vec2& focal) {
    cam = affine_inverse(view);
    vp = mat4_mul(proj, view);
    float r = (float)width / (float)height;
    float t_f_y = std::tan(radians(fovy) * 0.5f);
    float fovx = 2.0f * std::atan(t_f_y * r);
    float t_f_x = std::tan(fovx * 0.5f);
    tan_fov = make_v2(t_f_x, t_f_y);
    focal = make_v2((float)(width * ss) / (2.0f * tan_fov.x), (float)(height * ss) / (2.0f * tan_fov.y));
}

int load_cameras(const std::string& path, std::vector<CameraState>& out) {
    std::ifstream f(path);
    if (!f.is_open()) {
        set_last_error("unable to open camera file: " + path);
        return kStatusIo;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    JParser p(text);
    JValue root;
    if (!p.parse(root)) {
        set_last_error("camera JSON parse error: " + p.err);
        return kStatusFormat;
    }
    if (root.kind != JValue::Array) {
        set_last_error("camera JSON must be an array of camera objects");
        return kStatusFormat;
    }
    std::vector<CameraState> cams;
    for (auto& e : root.arr) {
        CameraState c;
        const JValue* pos = e.get("position");
        const JValue* rot = e.get("rotation");
        const JValue* name = e.get("img_name");
        if (e.kind != JValue::Object || !int_of(e.get("id"), c.id) || !int_of(e.get("width"), c.width) ||
            !int_of(e.get("height"), c.height) || !num_of(e.get("fx"), c.fx) || !num_of(e.get("fy"), c.fy) || !pos ||
            pos->kind != JValue::Array || pos->arr.size() < 3 || !rot || rot->kind != JValue::Array ||
            rot->arr.size() < 3 || !name || name->kind != JValue::String) {
            set_last_error("camera entry is missing id/img_name/width/height/position/rotation/fx/fy");
            return kStatusFormat;
        }
        c.img_name = name->str;
        for (int k = 0; k < 3; ++k)
            if (!num_of(&pos->arr[k], c.position[k])) { set_last_error("bad camera position"); return kStatusFormat; }
        for (int r = 0; r < 3; ++r) {
            const JValue& row = rot->arr[r];
            if (row.kind != JValue::Array || row.arr.size() < 3) { set_last_error("bad camera rotation"); return kStatusFormat; }
            for (int k = 0; k < 3; ++k)
                if (!num_of(&row.arr[k], c.rotation[3 * r + k])) { set_last_error("bad camera rotation"); return kStatusFormat; }
        }
        cams.push_back(c);
    }
    std::stable_sort(cams.begin(), cams.end(), [](const CameraState& a, const CameraState& b) { return a.id < b.id; });
    out.swap(cams);
    return 0;
}

}  // namespace gps
