// PNG / PNM decoding, area resampling and JSON parsing for dataset loading.
#include "image_io.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cctype>
#include <stdexcept>

#include <zlib.h>

namespace gs::detail {

namespace {

uint32_t be32(const uint8_t* p) { return uint32_t(p[0]) << 24 | uint32_t(p[1]) << 16 | uint32_t(p[2]) << 8 | p[3]; }

// Samples (8-bit, already reduced from 16) of one pixel -> the requested channel count.
void convert(const uint8_t* px, uint32_t src_channels, uint32_t channels, uint8_t* out) {
  const bool grey = src_channels <= 2;
  const uint8_t r = px[0], g = grey ? px[0] : px[1], b = grey ? px[0] : px[2];
  const uint8_t a = src_channels == 2 ? px[1] : (src_channels == 4 ? px[3] : 255);
  if (channels == 1) {
    out[0] = grey ? px[0] : uint8_t((uint32_t(r) * 299u + uint32_t(g) * 587u + uint32_t(b) * 114u + 500u) / 1000u);
  } else {
    out[0] = r;
    out[1] = g;
    out[2] = b;
    out[3] = a;
  }
}

// A PNG's unfiltered samples (big-endian when 16-bit) and the header fields that say how
// to read them.
struct PngRaster {
  uint32_t w = 0, h = 0, samples = 0;
  int depth = 0, type = -1;
  std::vector<uint8_t> px, palette, palette_alpha;
};

PngRaster read_png(const std::vector<uint8_t>& f) {
  PngRaster r;
  std::vector<uint8_t> idat;
  for (size_t at = 8; at + 12 <= f.size();) {
    const uint32_t len = be32(&f[at]);
    if (at + 12 + size_t(len) > f.size()) throw std::runtime_error("PNG: truncated chunk");
    const char* kind = reinterpret_cast<const char*>(&f[at + 4]);
    const uint8_t* d = &f[at + 8];
    if (std::memcmp(kind, "IHDR", 4) == 0) {
      if (len < 13) throw std::runtime_error("PNG: bad IHDR");
      r.w = be32(d);
      r.h = be32(d + 4);
      r.depth = d[8];
      r.type = d[9];
      if (d[12] != 0) throw std::runtime_error("PNG: interlaced images are not supported");
    } else if (std::memcmp(kind, "PLTE", 4) == 0) {
      r.palette.assign(d, d + len);
    } else if (std::memcmp(kind, "tRNS", 4) == 0) {
      r.palette_alpha.assign(d, d + len);
    } else if (std::memcmp(kind, "IDAT", 4) == 0) {
      idat.insert(idat.end(), d, d + len);
    } else if (std::memcmp(kind, "IEND", 4) == 0) {
      break;
    }
    at += 12 + size_t(len);
  }
  if (r.w == 0 || r.h == 0) throw std::runtime_error("PNG: no IHDR");
  switch (r.type) {
    case 0: r.samples = 1; break;
    case 2: r.samples = 3; break;
    case 3: r.samples = 1; break;
    case 4: r.samples = 2; break;
    case 6: r.samples = 4; break;
    default: throw std::runtime_error("PNG: bad colour type");
  }
  if (!(r.depth == 8 || (r.depth == 16 && r.type != 3)))
    throw std::runtime_error("PNG: only 8- and 16-bit samples are supported");
  const size_t bpp = r.samples * size_t(r.depth / 8), stride = bpp * r.w;
  std::vector<uint8_t> raw((stride + 1) * r.h);
  uLongf got = uLongf(raw.size());
  if (uncompress(raw.data(), &got, idat.data(), uLong(idat.size())) != Z_OK || got != raw.size())
    throw std::runtime_error("PNG: bad image data");
  // Undo the per-row filters (None, Sub, Up, Average, Paeth) in place.
  r.px.resize(stride * r.h);
  for (uint32_t y = 0; y < r.h; ++y) {
    const uint8_t filter = raw[y * (stride + 1)];
    const uint8_t* in = &raw[y * (stride + 1) + 1];
    uint8_t* row = &r.px[y * stride];
    const uint8_t* up = y > 0 ? &r.px[(y - 1) * stride] : nullptr;
    for (size_t i = 0; i < stride; ++i) {
      const int a = i >= bpp ? row[i - bpp] : 0, b = up ? up[i] : 0, c = (up && i >= bpp) ? up[i - bpp] : 0;
      int v = in[i];
      switch (filter) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) / 2; break;
        case 4: {
          const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
          v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
          break;
        }
        default: throw std::runtime_error("PNG: bad filter type");
      }
      row[i] = uint8_t(v);
    }
  }
  return r;
}

Image decode_png(const std::vector<uint8_t>& f, uint32_t channels) {
  const PngRaster r = read_png(f);
  const size_t bpp = r.samples * size_t(r.depth / 8);
  Image img;
  img.width = r.w;
  img.height = r.h;
  img.channels = channels;
  img.data.resize(size_t(r.w) * r.h * channels);
  for (size_t p = 0; p < size_t(r.w) * r.h; ++p) {
    uint8_t s[4];
    const uint32_t step = uint32_t(r.depth / 8);
    for (uint32_t k = 0; k < r.samples; ++k) s[k] = r.px[p * bpp + k * step];  // 16-bit: the high byte
    if (r.type == 3) {
      const uint32_t i = s[0];
      if (size_t(i) * 3 + 2 >= r.palette.size()) throw std::runtime_error("PNG: palette index out of range");
      const uint8_t rgba[4] = {r.palette[i * 3], r.palette[i * 3 + 1], r.palette[i * 3 + 2],
                               i < r.palette_alpha.size() ? r.palette_alpha[i] : uint8_t(255)};
      convert(rgba, 4, channels, &img.data[p * channels]);
    } else {
      convert(s, r.samples, channels, &img.data[p * channels]);
    }
  }
  return img;
}

Image decode_pnm(const std::vector<uint8_t>& f, uint32_t channels) {
  const bool colour = f[1] == '6';
  size_t at = 2;
  uint32_t v[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k) {
    while (at < f.size() && (std::isspace(f[at]) || f[at] == '#')) {
      if (f[at] == '#')
        while (at < f.size() && f[at] != '\n') ++at;
      else
        ++at;
    }
    while (at < f.size() && std::isdigit(f[at])) v[k] = v[k] * 10 + uint32_t(f[at++] - '0');
  }
  ++at;  // the single whitespace after maxval
  const uint32_t src = colour ? 3 : 1;
  if (v[2] != 255 || at + size_t(v[0]) * v[1] * src > f.size()) throw std::runtime_error("PNM: unsupported or truncated");
  Image img;
  img.width = v[0];
  img.height = v[1];
  img.channels = channels;
  img.data.resize(size_t(v[0]) * v[1] * channels);
  for (size_t p = 0; p < size_t(v[0]) * v[1]; ++p) convert(&f[at + p * src], src, channels, &img.data[p * channels]);
  return img;
}

// Weights of the input samples each output sample covers, along one axis.
struct Span {
  uint32_t first;
  std::vector<float> weights;
};
std::vector<Span> spans(uint32_t in, uint32_t out) {
  std::vector<Span> s(out);
  const double scale = double(in) / double(out);
  for (uint32_t o = 0; o < out; ++o) {
    const double lo = o * scale, hi = (o + 1) * scale;
    s[o].first = uint32_t(std::floor(lo));
    for (uint32_t i = s[o].first; i < in && double(i) < hi; ++i) {
      const double cover = std::min(hi, double(i + 1)) - std::max(lo, double(i));
      s[o].weights.push_back(float(cover / scale));
    }
  }
  return s;
}

}  // namespace

Image decode_image(const std::vector<uint8_t>& bytes, uint32_t channels) {
  if (channels != 1 && channels != 4) throw std::runtime_error("decode_image: 1 or 4 channels");
  static const uint8_t kPng[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (bytes.size() >= 8 && std::memcmp(bytes.data(), kPng, 8) == 0) return decode_png(bytes, channels);
  if (bytes.size() >= 3 && bytes[0] == 'P' && (bytes[1] == '5' || bytes[1] == '6')) return decode_pnm(bytes, channels);
  if (bytes.size() >= 3 && bytes[0] == 0xff && bytes[1] == 0xd8) return decode_jpeg(bytes, channels);
  throw std::runtime_error("unknown image format");
}

Depth16 decode_depth16(const std::vector<uint8_t>& bytes) {
  static const uint8_t kPng[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  Depth16 d;
  if (bytes.size() >= 8 && std::memcmp(bytes.data(), kPng, 8) == 0) {
    const PngRaster r = read_png(bytes);
    if (r.type != 0) throw std::runtime_error("depth PNG: not a single grey channel");
    d.width = r.w;
    d.height = r.h;
    d.data.resize(size_t(r.w) * r.h);
    for (size_t p = 0; p < d.data.size(); ++p)
      d.data[p] = r.depth == 16 ? uint16_t(uint32_t(r.px[p * 2]) << 8 | r.px[p * 2 + 1]) : uint16_t(r.px[p]);
    return d;
  }
  if (bytes.size() >= 3 && bytes[0] == 'P' && bytes[1] == '5') {
    size_t at = 2;
    uint32_t v[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
      while (at < bytes.size() && (std::isspace(bytes[at]) || bytes[at] == '#')) {
        if (bytes[at] == '#')
          while (at < bytes.size() && bytes[at] != '\n') ++at;
        else
          ++at;
      }
      while (at < bytes.size() && std::isdigit(bytes[at])) v[k] = v[k] * 10 + uint32_t(bytes[at++] - '0');
    }
    ++at;
    const size_t each = v[2] > 255 ? 2 : 1;
    if (v[2] == 0 || v[2] > 65535 || at + size_t(v[0]) * v[1] * each > bytes.size())
      throw std::runtime_error("depth PGM: unsupported or truncated");
    d.width = v[0];
    d.height = v[1];
    d.data.resize(size_t(v[0]) * v[1]);
    for (size_t p = 0; p < d.data.size(); ++p)
      d.data[p] = each == 2 ? uint16_t(uint32_t(bytes[at + 2 * p]) << 8 | bytes[at + 2 * p + 1]) : bytes[at + p];
    return d;
  }
  throw std::runtime_error("depth map: not a 16-bit PNG or PGM");
}

std::vector<uint8_t> resize_area(const uint8_t* src, uint32_t w, uint32_t h, uint32_t channels, uint32_t out_w,
                                 uint32_t out_h) {
  if (w == out_w && h == out_h) return std::vector<uint8_t>(src, src + size_t(w) * h * channels);
  const std::vector<Span> sx = spans(w, out_w), sy = spans(h, out_h);
  std::vector<float> rows(size_t(out_w) * h * channels);
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < out_w; ++x)
      for (uint32_t c = 0; c < channels; ++c) {
        float acc = 0.0f;
        for (size_t k = 0; k < sx[x].weights.size(); ++k)
          acc += sx[x].weights[k] * src[(size_t(y) * w + sx[x].first + k) * channels + c];
        rows[(size_t(y) * out_w + x) * channels + c] = acc;
      }
  std::vector<uint8_t> out(size_t(out_w) * out_h * channels);
  for (uint32_t y = 0; y < out_h; ++y)
    for (uint32_t x = 0; x < out_w; ++x)
      for (uint32_t c = 0; c < channels; ++c) {
        float acc = 0.0f;
        for (size_t k = 0; k < sy[y].weights.size(); ++k)
          acc += sy[y].weights[k] * rows[((sy[y].first + k) * out_w + x) * channels + c];
        out[(size_t(y) * out_w + x) * channels + c] = uint8_t(std::lround(std::min(std::max(acc, 0.0f), 255.0f)));
      }
  return out;
}

// ---- JSON ----

const Json* Json::find(const std::string& key) const {
  if (type != Type::Object) return nullptr;
  const auto it = object.find(key);
  return it == object.end() ? nullptr : &it->second;
}

double Json::number_or(const std::string& key, double fallback) const {
  const Json* v = find(key);
  return v != nullptr && v->type == Type::Number ? v->number : fallback;
}

std::string Json::string_or(const std::string& key, const std::string& fallback) const {
  const Json* v = find(key);
  return v != nullptr && v->type == Type::String ? v->string : fallback;
}

namespace {

struct Parser {
  const std::string& s;
  size_t at = 0;

  [[noreturn]] void error(const char* what) const {
    throw std::runtime_error(std::string("JSON: ") + what + " at offset " + std::to_string(at));
  }
  void space() {
    while (at < s.size() && std::isspace(static_cast<unsigned char>(s[at]))) ++at;
  }
  bool eat(char c) {
    space();
    if (at < s.size() && s[at] == c) {
      ++at;
      return true;
    }
    return false;
  }
  std::string text() {
    if (!eat('"')) error("expected a string");
    std::string out;
    while (at < s.size() && s[at] != '"') {
      char c = s[at++];
      if (c == '\\') {
        if (at >= s.size()) error("bad escape");
        c = s[at++];
        switch (c) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (at + 4 > s.size()) error("bad \\u escape");
            const unsigned cp = unsigned(std::stoul(s.substr(at, 4), nullptr, 16));
            at += 4;
            if (cp < 0x80) {
              out += char(cp);
            } else if (cp < 0x800) {
              out += char(0xc0 | (cp >> 6));
              out += char(0x80 | (cp & 0x3f));
            } else {
              out += char(0xe0 | (cp >> 12));
              out += char(0x80 | ((cp >> 6) & 0x3f));
              out += char(0x80 | (cp & 0x3f));
            }
            break;
          }
          default: out += c;  // \" \\ \/
        }
      } else {
        out += c;
      }
    }
    if (at >= s.size()) error("unterminated string");
    ++at;
    return out;
  }
  Json value() {
    space();
    if (at >= s.size()) error("unexpected end");
    Json v;
    const char c = s[at];
    if (c == '{') {
      ++at;
      v.type = Json::Type::Object;
      if (eat('}')) return v;
      do {
        std::string key = text();
        if (!eat(':')) error("expected ':'");
        v.object[key] = value();
      } while (eat(','));
      if (!eat('}')) error("expected '}'");
    } else if (c == '[') {
      ++at;
      v.type = Json::Type::Array;
      if (eat(']')) return v;
      do v.array.push_back(value());
      while (eat(','));
      if (!eat(']')) error("expected ']'");
    } else if (c == '"') {
      v.type = Json::Type::String;
      v.string = text();
    } else if (s.compare(at, 4, "true") == 0 || s.compare(at, 5, "false") == 0) {
      v.type = Json::Type::Bool;
      v.boolean = s[at] == 't';
      at += v.boolean ? 4 : 5;
    } else if (s.compare(at, 4, "null") == 0) {
      at += 4;
    } else {
      size_t used = 0;
      try {
        v.number = std::stod(s.substr(at, 64), &used);
      } catch (const std::exception&) {
        error("bad value");
      }
      v.type = Json::Type::Number;
      at += used;
    }
    return v;
  }
};

}  // namespace

Json parse_json(const std::string& text) {
  Parser p{text};
  Json v = p.value();
  p.space();
  if (p.at != text.size()) p.error("trailing characters");
  return v;
}

}  // namespace gs::detail
