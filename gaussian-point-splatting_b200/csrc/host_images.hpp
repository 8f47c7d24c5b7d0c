// PNG / PFM writers for the evaluation workflow (render_server.cu:196-315).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace gps {

// mkdir -p; true if `dir` exists as a directory afterwards.
bool make_dirs(const std::string& dir);
// 8-bit RGB, rows top to bottom unless flip_rows.  Returns 0, 1 (bad argument) or 2 (zlib).
int encode_png(const uint8_t* rgb, int width, int height, bool flip_rows, std::vector<uint8_t>& out);
// encode_png to a file; 3 = I/O error.
int write_png(const std::string& path, const uint8_t* rgb, int width, int height, bool flip_rows);
// "PF\n<w> <h>\n-1.0\n" then the floats in memory order (little-endian scale, as the reference).
int write_pfm(const std::string& path, const float* rgb, int width, int height);

}  // namespace gps
