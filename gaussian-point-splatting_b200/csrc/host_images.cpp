// Image files of the evaluation workflow: 8-bit RGB PNG (the reference's stbi_write_png call,
// render_server.cu:269-315) and 32-bit float RGB PFM (write_pfm, render_server.cu:196-208),
// plus the directory creation they need.  PNG rows are filtered with filter type 0 and
// compressed by zlib; chunk CRCs come from zlib's crc32.
#include "host_images.hpp"

#include <sys/stat.h>
#include <sys/types.h>
#include <zlib.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace gps {
namespace {

void put_be32(std::vector<uint8_t>& out, uint32_t v) {
    out.push_back((uint8_t)(v >> 24));
    out.push_back((uint8_t)(v >> 16));
    out.push_back((uint8_t)(v >> 8));
    out.push_back((uint8_t)v);
}

void put_chunk(std::vector<uint8_t>& out, const char type[4], const uint8_t* data, size_t n) {
    put_be32(out, (uint32_t)n);
    const size_t at = out.size();
    out.insert(out.end(), type, type + 4);
    if (n) out.insert(out.end(), data, data + n);
    const uLong crc = crc32(crc32(0L, Z_NULL, 0), out.data() + at, (uInt)(n + 4));
    put_be32(out, (uint32_t)crc);
}

bool write_all(const std::string& path, const void* data, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, n, f) == n;
    return (std::fclose(f) == 0) && ok;
}

}  // namespace

bool make_dirs(const std::string& dir) {
    if (dir.empty()) return true;
    std::string cur;
    size_t i = 0;
    while (i <= dir.size()) {
        const size_t j = dir.find('/', i);
        const size_t end = j == std::string::npos ? dir.size() : j;
        cur = dir.substr(0, end);
        if (!cur.empty() && ::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
        if (j == std::string::npos) break;
        i = j + 1;
    }
    struct stat st;
    return ::stat(dir.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

int encode_png(const uint8_t* rgb, int width, int height, bool flip_rows, std::vector<uint8_t>& out) {
    if (!rgb || width <= 0 || height <= 0) return 1;
    const size_t row = (size_t)width * 3;
    std::vector<uint8_t> raw((row + 1) * (size_t)height);
    for (int y = 0; y < height; ++y) {
        const int src = flip_rows ? height - 1 - y : y;
        uint8_t* dst = raw.data() + (row + 1) * (size_t)y;
        dst[0] = 0;  // filter type None
        std::memcpy(dst + 1, rgb + row * (size_t)src, row);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return 2;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    out.assign(sig, sig + 8);
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(2);  // colour type: RGB
    ihdr.push_back(0);  // deflate
    ihdr.push_back(0);  // adaptive filtering
    ihdr.push_back(0);  // no interlace
    put_chunk(out, "IHDR", ihdr.data(), ihdr.size());
    put_chunk(out, "IDAT", z.data(), zlen);
    put_chunk(out, "IEND", nullptr, 0);
    return 0;
}

int write_png(const std::string& path, const uint8_t* rgb, int width, int height, bool flip_rows) {
    std::vector<uint8_t> png;
    const int rc = encode_png(rgb, width, height, flip_rows, png);
    if (rc) return rc;
    return write_all(path, png.data(), png.size()) ? 0 : 3;
}

int write_pfm(const std::string& path, const float* rgb, int width, int height) {
    if (!rgb || width <= 0 || height <= 0) return 1;
    char header[64];
    const int n = std::snprintf(header, sizeof(header), "PF\n%d %d\n-1.0\n", width, height);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return 3;
    bool ok = std::fwrite(header, 1, (size_t)n, f) == (size_t)n;
    const size_t count = (size_t)width * height * 3;
    ok = ok && std::fwrite(rgb, sizeof(float), count, f) == count;
    return (std::fclose(f) == 0 && ok) ? 0 : 3;
}

}  // namespace gps
