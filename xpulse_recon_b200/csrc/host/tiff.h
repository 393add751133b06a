// tiff.h -- single-channel 32-bit floating-point TIFF reading and writing.
//
// The reference reads and writes such files through TinyTIFF
// (src/reconstruction/dataset/data_loader.hpp:209-237, dataset.hpp:243-269).  This
// is an independent implementation of the TIFF 6.0 baseline subset needed here:
// uncompressed, strip-organised, one sample per pixel, SampleFormat 3 (IEEE float),
// 32 bits per sample, either byte order.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace xpr {

struct TiffInfo {
    uint32_t width = 0, height = 0;
    uint16_t bits = 0, sample_format = 1, samples = 1, compression = 1;
};

// Reads the header of `path`.  Returns false (with *err set) when the file is not a TIFF.
bool tiff_info(const std::string &path, TiffInfo *info, std::string *err);
// Reads a float32 image; throws std::runtime_error on any problem.
std::vector<float> tiff_read_f32(const std::string &path, uint32_t *width, uint32_t *height);
// Writes a little-endian single-strip float32 TIFF; throws std::runtime_error.
void tiff_write_f32(const std::string &path, const float *data, uint32_t width, uint32_t height);

}  // namespace xpr
