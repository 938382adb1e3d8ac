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

// PNG (8 or 16 bits per sample, grey / grey+alpha / RGB / RGBA / palette, not interlaced)
// or binary PPM (P6) / PGM (P5), converted to `channels` (1: grey or the alpha channel's
// source for masks, 4: RGBA with alpha 255 where the file has none). Throws
// std::runtime_error for other formats (libgs_host has no JPEG decoder).
Image decode_image(const std::vector<uint8_t>& bytes, uint32_t channels);

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
