// Internal: image decoding and resampling for dataset loading, and a small JSON reader.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace gs::detail {

struct Image {
  uint32_t width = 0, height = 0, channels = 0;
  std::vector<uint8_t> data;  // row-major, `channels` bytes per pixel
};

// PNG (8 or 16 bits per sample, grey / grey+alpha / RGB / RGBA / palette, not interlaced),
// binary PPM (P6) / PGM (P5) or JPEG (decoded on the GPU by nvJPEG: decode_jpeg), converted
// to `channels` (1: grey or the alpha channel's source for masks, 4: RGBA with alpha 255
// where the file has none). Throws std::runtime_error for other formats and for JPEG files
// when no GPU can decode them.
Image decode_image(const std::vector<uint8_t>& bytes, uint32_t channels);

// A JPEG file decoded by nvJPEG on the current CUDA device (baseline and progressive,
// any chroma subsampling), as `channels` (1: luma, 4: RGBA with alpha 255). The decode
// runs on the GPU; the pixels come back to host memory. Throws std::runtime_error with
// nvJPEG's status when the file or the device cannot be decoded.
Image decode_jpeg(const std::vector<uint8_t>& bytes, uint32_t channels);

// A depth map: a single-channel PNG (16- or 8-bit) or PGM (P5, maxval up to 65535), raw
// samples in the file's units (the capture's depth_unit_scale_factor converts them).
struct Depth16 {
  uint32_t width = 0, height = 0;
  std::vector<uint16_t> data;
};
Depth16 decode_depth16(const std::vector<uint8_t>& bytes);

// Area resampling (each output pixel is the coverage-weighted mean of the input pixels it
// covers), rounded to the nearest level.
std::vector<uint8_t> resize_area(const uint8_t* src, uint32_t w, uint32_t h, uint32_t channels, uint32_t out_w,
                                 uint32_t out_h);

// A parsed JSON value (objects keep their keys sorted; duplicate keys keep the last).
struct Json {
  enum class Type { Null, Bool, Number, String, Array, Object } type = Type::Null;
  bool boolean = false;
  double number = 0.0;
  std::string string;
  std::vector<Json> array;
  std::map<std::string, Json> object;

  const Json* find(const std::string& key) const;
  double number_or(const std::string& key, double fallback) const;
  std::string string_or(const std::string& key, const std::string& fallback) const;
};
Json parse_json(const std::string& text);  // throws std::runtime_error with the offset

}  // namespace gs::detail
