// 3DGS binary PLY I/O and the reference's compressed scene encoding (host side).
//
// PLY semantics follow gaussian_loader.cu:115-245 (header-driven field offsets, any
// property order, opacity = sigmoid, scale = exp, rotation = normalize(rot_0..rot_3) kept
// in (w,x,y,z) lane order, f_rest channel-major -> interleaved RGB per coefficient, missing
// f_rest -> zero) and :480-562 (writer with normals).  The encoder follows
// gaussian_types.cuh:127-320 and sh.cuh:28-39 operation by operation.
#include <algorithm>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <numeric>
#include <sstream>
#include <thread>
#include "host_io.hpp"

namespace gps {

namespace {
thread_local std::string g_last_error;

constexpr int kStatusIo = 2;
constexpr int kStatusFormat = 3;
constexpr int kStatusSize = 6;

float sigmoid_ref(float x) {
    float v = 1.0f / (1.0f + std::exp(-x));
    return gclamp(v, 0.0f, 1.0f);
}

// glm::normalize(vec4) on the host: v * (1 / sqrt((x*x + y*y) + (z*z + w*w)))
void normalize4(float v[4]) {
    float d = (v[0] * v[0] + v[1] * v[1]) + (v[2] * v[2] + v[3] * v[3]);
    float inv = 1.0f / std::sqrt(d);
    for (int i = 0; i < 4; ++i) v[i] = v[i] * inv;
}

size_t ply_type_size(const std::string& t) {
    if (t == "double" || t == "float64" || t == "int64" || t == "uint64") return 8;
    if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
    if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
    return 4;
}

constexpr size_t kMissing = SIZE_MAX;

struct Offsets {
    size_t x = kMissing, y = kMissing, z = kMissing;
    size_t dc[3] = {kMissing, kMissing, kMissing};
    std::vector<size_t> rest;
    size_t opacity = kMissing;
    size_t scale[3] = {kMissing, kMissing, kMissing};
    size_t rot[4] = {kMissing, kMissing, kMissing, kMissing};
    size_t record = 0;
};

float getf(const uint8_t* rec, size_t off) {
    if (off == kMissing) return 0.0f;
    float v;
    std::memcpy(&v, rec + off, 4);
    return v;
}

void record_to_gaussian(const uint8_t* rec, const Offsets& o, CpuGaussian& g) {
    g.mean[0] = getf(rec, o.x);
    g.mean[1] = getf(rec, o.y);
    g.mean[2] = getf(rec, o.z);
    g.opacity = sigmoid_ref(getf(rec, o.opacity));
    for (int i = 0; i < 3; ++i) g.scale[i] = std::exp(getf(rec, o.scale[i]));
    for (int i = 0; i < 4; ++i) g.rot[i] = getf(rec, o.rot[i]);
    normalize4(g.rot);
    for (int i = 0; i < 3; ++i) g.sh[i] = getf(rec, o.dc[i]);
    const bool have_rest = o.rest.size() >= 45;
    for (int j = 1; j < 16; ++j) {
        int r = j - 1;
        g.sh[j * 3 + 0] = have_rest ? getf(rec, o.rest[r]) : 0.0f;
        g.sh[j * 3 + 1] = have_rest ? getf(rec, o.rest[r + 15]) : 0.0f;
        g.sh[j * 3 + 2] = have_rest ? getf(rec, o.rest[r + 30]) : 0.0f;
    }
}

template <class F>
void parallel_for(uint64_t n, F f) {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 65536) nt = 1;
    std::vector<std::thread> ts;
    uint64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        uint64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back([=]() { f(b, e); });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

void parallel_ranges(uint64_t n, const std::function<void(uint64_t, uint64_t)>& f) { parallel_for(n, f); }

namespace {

uint64_t morton3d21(int x, int y, int z) {
    uint64_t code = 0;
    for (int bit = 0; bit < 21; ++bit) {
        code |= (uint64_t(x & (1 << bit)) << (2 * bit + 0));
        code |= (uint64_t(y & (1 << bit)) << (2 * bit + 1));
        code |= (uint64_t(z & (1 << bit)) << (2 * bit + 2));
    }
    return code;
}

// static_cast<uint8_t>(float) as the reference's host build evaluates it: truncation via a
// 32-bit conversion, keeping the low byte (NaN converts to 0).
uint8_t float_to_u8_trunc(float v) {
    if (std::isnan(v)) return 0;
    return (uint8_t)(int32_t)v;
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

bool has_bvh_sorted_comment(const std::vector<std::string>& comments) {
    return std::any_of(comments.begin(), comments.end(), [](const std::string& c) { return c == "bvh_sorted_order"; });
}

int resolve_model_path(const std::string& in, std::string& out) {
    namespace fs = std::filesystem;
    fs::path mp(in);
    std::error_code ec;
    if (fs::is_directory(mp, ec)) {
        fs::path pc = mp / "point_cloud";
        if (!fs::exists(pc, ec)) {
            set_last_error("model directory has no 'point_cloud' subfolder: " + pc.string());
            return kStatusIo;
        }
        fs::path best;
        bool found = false;
        for (auto& e : fs::directory_iterator(pc, ec)) {
            if (!e.is_directory()) continue;
            if (!found || e.path().filename().string() > best.filename().string()) {
                best = e.path();
                found = true;
            }
        }
        if (!found) {
            set_last_error("no subfolders inside " + pc.string());
            return kStatusIo;
        }
        fs::path cand = best / "point_cloud.ply";
        if (!fs::exists(cand, ec)) {
            set_last_error("alphabetically last folder has no point_cloud.ply: " + cand.string());
            return kStatusIo;
        }
        out = cand.string();
        return 0;
    }
    if (!fs::exists(mp, ec)) {
        set_last_error("model path does not exist: " + in);
        return kStatusIo;
    }
    out = in;
    return 0;
}

namespace {

// The header of a binary little-endian 3DGS PLY: property offsets, vertex count, comments; the
// stream is left at the first record.  Returns 0 or a gps_status value.
int ply_header(std::ifstream& f, const std::string& path, Offsets& o, size_t& count, std::vector<std::string>& comments) {
    comments.clear();
    count = 0;
    size_t off = 0;
    bool in_vertex = false, saw_end = false, saw_magic = false, binary_le = false;
    std::string line;
    while (std::getline(f, line)) {
        auto first = line.find_first_not_of(" \t\r\n");
        if (first != std::string::npos) line = line.substr(first);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line == "ply") { saw_magic = true; continue; }
        if (line.rfind("format", 0) == 0) { binary_le = line.find("binary_little_endian") != std::string::npos; continue; }
        if (line.rfind("comment", 0) == 0) { comments.push_back(line.size() > 8 ? line.substr(8) : std::string()); continue; }
        if (line.rfind("element", 0) == 0) {
            std::istringstream iss(line);
            std::string kw, name;
            size_t c = 0;
            iss >> kw >> name >> c;
            in_vertex = (name == "vertex");
            if (in_vertex) count = c;
            continue;
        }
        if (line.rfind("property", 0) == 0) {
            if (!in_vertex) continue;
            std::istringstream iss(line);
            std::string kw, type, name;
            iss >> kw >> type >> name;
            if (name.empty()) continue;
            size_t sz = ply_type_size(type);
            if (name == "x") o.x = off;
            else if (name == "y") o.y = off;
            else if (name == "z") o.z = off;
            else if (name == "f_dc_0") o.dc[0] = off;
            else if (name == "f_dc_1") o.dc[1] = off;
            else if (name == "f_dc_2") o.dc[2] = off;
            else if (name == "opacity") o.opacity = off;
            else if (name == "scale_0") o.scale[0] = off;
            else if (name == "scale_1") o.scale[1] = off;
            else if (name == "scale_2") o.scale[2] = off;
            else if (name == "rot_0") o.rot[0] = off;
            else if (name == "rot_1") o.rot[1] = off;
            else if (name == "rot_2") o.rot[2] = off;
            else if (name == "rot_3") o.rot[3] = off;
            else if (name.rfind("f_rest_", 0) == 0) {
                char* end = nullptr;
                long idx = std::strtol(name.c_str() + 7, &end, 10);
                if (end && *end == 0 && idx >= 0 && idx < 4096) {
                    if ((size_t)idx >= o.rest.size()) o.rest.resize(idx + 1, kMissing);
                    o.rest[idx] = off;
                }
            }
            off += sz;
            continue;
        }
        if (line == "end_header") { saw_end = true; break; }
    }
    o.record = off;
    if (!saw_magic || !saw_end) {
        set_last_error("not a PLY file or header not terminated: " + path);
        return kStatusFormat;
    }
    if (!binary_le) {
        set_last_error("only binary_little_endian PLY is supported: " + path);
        return kStatusFormat;
    }
    if (count == 0) {
        set_last_error("header missing or zero vertex count: " + path);
        return kStatusFormat;
    }
    if (o.x == kMissing || o.y == kMissing || o.z == kMissing) { set_last_error("missing position fields (x/y/z)"); return kStatusFormat; }
    if (o.dc[0] == kMissing || o.dc[1] == kMissing || o.dc[2] == kMissing) { set_last_error("missing DC spherical harmonic fields (f_dc_0/1/2)"); return kStatusFormat; }
    if (o.opacity == kMissing) { set_last_error("missing opacity field"); return kStatusFormat; }
    for (int i = 0; i < 3; ++i) if (o.scale[i] == kMissing) { set_last_error("missing scale field(s)"); return kStatusFormat; }
    for (int i = 0; i < 4; ++i) if (o.rot[i] == kMissing) { set_last_error("missing rotation field(s)"); return kStatusFormat; }
    for (size_t i = 0; i < o.rest.size() && i < 45; ++i)
        if (o.rest.size() >= 45 && o.rest[i] == kMissing) { set_last_error("f_rest fields are not contiguous"); return kStatusFormat; }

    return 0;
}

int ply_open(const std::string& path, std::ifstream& f) {
    f.open(path, std::ios::binary);
    if (!f.is_open()) {
        set_last_error("failed to open file: " + path);
        return kStatusIo;
    }
    return 0;
}

}  // namespace

int ply_count(const std::string& path, uint64_t& count, std::vector<std::string>& comments) {
    std::ifstream f;
    int rc = ply_open(path, f);
    if (rc) return rc;
    Offsets o;
    size_t c = 0;
    rc = ply_header(f, path, o, c, comments);
    count = c;
    return rc;
}

int ply_read_into(const std::string& path, CpuGaussian* out, uint64_t capacity, uint64_t& count,
                  std::vector<std::string>& comments) {
    std::ifstream f;
    int rc = ply_open(path, f);
    if (rc) return rc;
    Offsets o;
    size_t c = 0;
    rc = ply_header(f, path, o, c, comments);
    if (rc) return rc;
    count = c;
    if (capacity < c) {
        set_last_error("output capacity too small");
        return kStatusSize;
    }
    // records in 64 MiB chunks: the next chunk is read while the current one is converted on
    // every core
    const size_t per = std::max<size_t>(1, ((size_t)64 << 20) / o.record);
    std::vector<uint8_t> buf[2];
    auto read_chunk = [&](size_t b, std::vector<uint8_t>& into) -> bool {
        const size_t m = std::min(per, c - b);
        into.resize(m * o.record);
        f.read(reinterpret_cast<char*>(into.data()), (std::streamsize)into.size());
        return (size_t)f.gcount() == into.size();
    };
    if (!read_chunk(0, buf[0])) {
        set_last_error("short read: expected " + std::to_string(c) + " records in " + path);
        return kStatusIo;
    }
    for (size_t b = 0, k = 0; b < c; b += per, k ^= 1) {
        const size_t m = std::min(per, c - b);
        bool next_ok = true;
        std::thread reader;
        if (b + per < c) reader = std::thread([&, b, k]() { next_ok = read_chunk(b + per, buf[k ^ 1]); });
        const uint8_t* src = buf[k].data();
        parallel_for(m, [&](uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; ++i) record_to_gaussian(src + i * o.record, o, out[b + i]);
        });
        if (reader.joinable()) reader.join();
        if (!next_ok) {
            set_last_error("short read: expected " + std::to_string(c) + " records in " + path);
            return kStatusIo;
        }
    }
    return 0;
}

int ply_read(const std::string& path, std::vector<CpuGaussian>& out, std::vector<std::string>& comments) {
    uint64_t count = 0;
    int rc = ply_count(path, count, comments);
    if (rc) return rc;
    out.resize(count);
    return ply_read_into(path, out.data(), count, count, comments);
}

int ply_write(const std::string& path, const CpuGaussian* g, uint64_t n, const std::vector<std::string>& comments) {
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) {
        set_last_error("failed to open file for writing: " + path);
        return kStatusIo;
    }
    std::ostringstream h;
    h << "ply\nformat binary_little_endian 1.0\n";
    for (auto& c : comments) h << "comment " << c << "\n";
    h << "element vertex " << n << "\n"
      << "property float x\nproperty float y\nproperty float z\n"
      << "property float nx\nproperty float ny\nproperty float nz\n"
      << "property float f_dc_0\nproperty float f_dc_1\nproperty float f_dc_2\n";
    for (int i = 0; i < 45; ++i) h << "property float f_rest_" << i << "\n";
    h << "property float opacity\n"
      << "property float scale_0\nproperty float scale_1\nproperty float scale_2\n"
      << "property float rot_0\nproperty float rot_1\nproperty float rot_2\nproperty float rot_3\n"
      << "end_header\n";
    std::string hs = h.str();
    f.write(hs.data(), (std::streamsize)hs.size());
    const size_t chunk = 1 << 16;
    std::vector<float> rec(chunk * 62);
    for (uint64_t b = 0; b < n; b += chunk) {
        uint64_t e = std::min<uint64_t>(n, b + chunk);
        for (uint64_t i = b; i < e; ++i) {
            float* r = &rec[(i - b) * 62];
            const CpuGaussian& q = g[i];
            r[0] = q.mean[0]; r[1] = q.mean[1]; r[2] = q.mean[2];
            r[3] = 0.0f; r[4] = 0.0f; r[5] = 0.0f;
            r[6] = q.sh[0]; r[7] = q.sh[1]; r[8] = q.sh[2];
            for (int j = 1; j < 16; ++j) {
                int k = j - 1;
                r[9 + k] = q.sh[j * 3 + 0];
                r[9 + k + 15] = q.sh[j * 3 + 1];
                r[9 + k + 30] = q.sh[j * 3 + 2];
            }
            r[54] = std::log(q.opacity / (1.0f - q.opacity));
            r[55] = std::log(q.scale[0]); r[56] = std::log(q.scale[1]); r[57] = std::log(q.scale[2]);
            r[58] = q.rot[0]; r[59] = q.rot[1]; r[60] = q.rot[2]; r[61] = q.rot[3];
        }
        f.write(reinterpret_cast<const char*>(rec.data()), (std::streamsize)((e - b) * 62 * sizeof(float)));
    }
    if (!f) {
        set_last_error("write failed: " + path);
        return kStatusIo;
    }
    return 0;
}

void morton_order(const CpuGaussian* g, uint64_t n, uint32_t* order) {
    if (n == 0) return;
    vec3 mn = make_v3(FLT_MAX, FLT_MAX, FLT_MAX), mx = make_v3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint64_t i = 0; i < n; ++i) {
        const CpuGaussian& q = g[i];
        mn = make_v3(gmin(mn.x, q.mean[0]), gmin(mn.y, q.mean[1]), gmin(mn.z, q.mean[2]));
        mx = make_v3(gmax(mx.x, q.mean[0]), gmax(mx.y, q.mean[1]), gmax(mx.z, q.mean[2]));
    }
    std::vector<uint64_t> key(n);
    parallel_for(n, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            float rel[3], den[3] = {mx.x - mn.x, mx.y - mn.y, mx.z - mn.z};
            float num[3] = {g[i].mean[0] - mn.x, g[i].mean[1] - mn.y, g[i].mean[2] - mn.z};
            for (int c = 0; c < 3; ++c) rel[c] = den[c] != 0.0f ? num[c] / den[c] : 0.0f;
            const float s = float((1 << 21) - 1);
            key[i] = morton3d21((int)(rel[0] * s), (int)(rel[1] * s), (int)(rel[2] * s));
        }
    });
    std::iota(order, order + n, 0u);
    std::stable_sort(order, order + n, [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
}

void morton_sort(std::vector<CpuGaussian>& g) {
    const size_t n = g.size();
    if (n == 0) return;
    std::vector<uint32_t> idx(n);
    morton_order(g.data(), n, idx.data());
    std::vector<CpuGaussian> tmp(n);
    for (size_t j = 0; j < n; ++j) tmp[j] = g[idx[j]];
    g.swap(tmp);
}

uint32_t gaussians_per_block(uint64_t n) {
    // glm::max(4.0f, glm::floor(N / float(1e6)))
    float v = std::floor((float)n / 1e6f);
    return (uint32_t)(int)gmax(4.0f, v);
}

SceneBounds compute_scene_bounds(const CpuGaussian* g, uint64_t n) {
    auto fresh = []() {
        SceneBounds b;
        const float lo = -FLT_MAX, hi = FLT_MAX;
        b.max_pos = make_v3(lo, lo, lo);
        b.min_pos = make_v3(hi, hi, hi);
        b.max_scale = make_v3(lo, lo, lo);
        b.min_scale = make_v3(hi, hi, hi);
        for (int i = 0; i < 15; ++i) {
            b.max_sh[i] = make_v3(lo, lo, lo);
            b.min_sh[i] = make_v3(hi, hi, hi);
        }
        return b;
    };
    // gmin / gmax keep the running value unless the new one is strictly smaller / larger (and a
    // NaN never is), so a fold keeps the earliest extreme value.  Folding contiguous ranges in
    // parallel and then the ranges' results left to right keeps the same one: the result is the
    // sequential fold's, bit for bit (signed zeros included).
    auto vmax = [](vec3 a, vec3 c) { return make_v3(gmax(a.x, c.x), gmax(a.y, c.y), gmax(a.z, c.z)); };
    auto vmin = [](vec3 a, vec3 c) { return make_v3(gmin(a.x, c.x), gmin(a.y, c.y), gmin(a.z, c.z)); };
    auto merge = [&](SceneBounds& b, const SceneBounds& c) {
        b.max_pos = vmax(b.max_pos, c.max_pos);
        b.min_pos = vmin(b.min_pos, c.min_pos);
        b.max_scale = vmax(b.max_scale, c.max_scale);
        b.min_scale = vmin(b.min_scale, c.min_scale);
        for (int j = 0; j < 15; ++j) {
            b.max_sh[j] = vmax(b.max_sh[j], c.max_sh[j]);
            b.min_sh[j] = vmin(b.min_sh[j], c.min_sh[j]);
        }
    };
    auto fold = [&](uint64_t lo_i, uint64_t hi_i, SceneBounds& b) {
        for (uint64_t i = lo_i; i < hi_i; ++i) {
            vec3 m = make_v3(g[i].mean[0], g[i].mean[1], g[i].mean[2]);
            b.max_pos = vmax(b.max_pos, m);
            b.min_pos = vmin(b.min_pos, m);
            vec3 ls = make_v3(std::log(g[i].scale[0]), std::log(g[i].scale[1]), std::log(g[i].scale[2]));
            b.max_scale = vmax(b.max_scale, ls);
            b.min_scale = vmin(b.min_scale, ls);
            for (int j = 0; j < 15; ++j) {
                vec3 s = make_v3(g[i].sh[3 * j + 3], g[i].sh[3 * j + 4], g[i].sh[3 * j + 5]);
                b.max_sh[j] = vmax(b.max_sh[j], s);
                b.min_sh[j] = vmin(b.min_sh[j], s);
            }
        }
    };
    const uint64_t ranges = n < 65536 ? 1 : std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<SceneBounds> part(ranges, fresh());
    const uint64_t per = (n + ranges - 1) / ranges;
    std::vector<std::thread> ts;
    for (uint64_t r = 0; r < ranges; ++r)
        ts.emplace_back([&, r]() { fold(std::min(n, r * per), std::min(n, (r + 1) * per), part[r]); });
    for (auto& t : ts) t.join();
    SceneBounds b = fresh();
    for (const SceneBounds& p : part) merge(b, p);
    const float margin = 0.001f;
    b.max_pos = make_v3(b.max_pos.x + margin, b.max_pos.y + margin, b.max_pos.z + margin);
    b.min_pos = make_v3(b.min_pos.x - margin, b.min_pos.y - margin, b.min_pos.z - margin);
    return b;
}

namespace {
// quat_fem (gaussian_types.cuh:201-210) on the host: 2/pi is a double there (M_PI from
// <cmath>), atan of a float argument is atanf, and the product is rounded once to float.
vec3 quat_fem_host(const float q[4]) {
    float w = q[3];
    float a = 1.0f - w * w;
    float b = 1.0f / std::sqrt(a + 1.0e-12f);
    float k = a * b;
    float s = (float)((2.0f / 3.14159265358979323846) * (double)std::atan(k / w) * (double)b);
    return make_v3(s * q[0], s * q[1], s * q[2]);
}
}  // namespace

void encode_compressed(const CpuGaussian* g, uint64_t n, const SceneBounds& b, uint4* geom, uint8_t* opac,
                       float4* sh_dc, uint4* sh_ac) {
    parallel_for(n, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            const CpuGaussian& q = g[i];
            // opacity byte (gaussian_types.cuh:196-199)
            opac[i] = (uint8_t)(fminf(fmaxf(q.opacity, 0.0f), 1.0f) * 255.0f + 0.5f);
            // position
            float t[3];
            const float mn[3] = {b.min_pos.x, b.min_pos.y, b.min_pos.z};
            const float mx[3] = {b.max_pos.x, b.max_pos.y, b.max_pos.z};
            for (int c = 0; c < 3; ++c) t[c] = gclamp((q.mean[c] - mn[c]) / (mx[c] - mn[c]), 0.0f, 1.0f);
            uint32_t px = (uint32_t)(t[0] * (float)((1u << 23) - 1u));
            uint32_t py = (uint32_t)(t[1] * (float)((1u << 22) - 1u));
            uint32_t pz = (uint32_t)(t[2] * (float)((1u << 23) - 1u));
            // rotation
            float r[4] = {q.rot[0], q.rot[1], q.rot[2], q.rot[3]};
            normalize4(r);
            if (r[3] < 0.0f)
                for (int c = 0; c < 4; ++c) r[c] = -r[c];
            vec3 v = quat_fem_host(r);
            float vr[3] = {gclamp((v.x + 1.0f) * 0.5f, 0.0f, 1.0f), gclamp((v.y + 1.0f) * 0.5f, 0.0f, 1.0f),
                           gclamp((v.z + 1.0f) * 0.5f, 0.0f, 1.0f)};
            uint32_t rx = (uint32_t)(vr[0] * 1023.0f), ry = (uint32_t)(vr[1] * 1023.0f), rz = (uint32_t)(vr[2] * 1023.0f);
            // scale
            const float smn[3] = {b.min_scale.x, b.min_scale.y, b.min_scale.z};
            const float smx[3] = {b.max_scale.x, b.max_scale.y, b.max_scale.z};
            uint32_t s[3];
            for (int c = 0; c < 3; ++c) {
                float ls = std::log(q.scale[c]);
                float st = gclamp((ls - smn[c]) / (smx[c] - smn[c]), 0.0f, 1.0f);
                s[c] = (uint32_t)(st * 1023.0f);
            }
            uint32_t py_low9 = py & 0x1FFu, py_high13 = (py >> 9) & 0x1FFFu;
            uint32_t pz_low19 = pz & 0x7FFFFu, pz_high4 = (pz >> 19) & 0xFu;
            uint32_t rz_low8 = rz & 0xFFu, rz_high2 = (rz >> 8) & 0x3u;
            uint4 w;
            w.x = (px & 0x7FFFFFu) | (py_low9 << 23);
            w.y = (py_high13 & 0x1FFFu) | (pz_low19 << 13);
            w.z = (pz_high4 & 0xFu) | ((rx & 0x3FFu) << 4) | ((ry & 0x3FFu) << 14) | ((rz_low8 & 0xFFu) << 24);
            w.w = (rz_high2 & 0x3u) | ((s[0] & 0x3FFu) << 2) | ((s[1] & 0x3FFu) << 12) | ((s[2] & 0x3FFu) << 22);
            geom[i] = w;
            // compact SH (sh.cuh:29-39)
            sh_dc[i] = make_float4(q.sh[0], q.sh[1], q.sh[2], 0.0f);
            uint8_t bytes[48] = {0};
            for (int j = 0; j < 15; ++j) {
                float c3[3];
                const float lo3[3] = {b.min_sh[j].x, b.min_sh[j].y, b.min_sh[j].z};
                const float hi3[3] = {b.max_sh[j].x, b.max_sh[j].y, b.max_sh[j].z};
                for (int c = 0; c < 3; ++c) {
                    c3[c] = (q.sh[3 * j + 3 + c] - lo3[c]) / (hi3[c] - lo3[c]);
                    bytes[3 * j + c] = float_to_u8_trunc(gclamp(c3[c] * 255.0f, 0.0f, 255.0f));
                }
            }
            uint4* dst = sh_ac + i * 3;
            std::memcpy(dst, bytes, 48);
        }
    });
}

}  // namespace gps
