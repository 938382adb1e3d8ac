// JPEG frames for dataset loading, decoded on the GPU by nvJPEG (the CUDA toolkit's JPEG
// decoder): the entropy decoding, dequantisation, inverse DCT, chroma upsampling and
// colour conversion run on the device, and the interleaved RGB result is copied back.
#include <cuda_runtime.h>
#include <nvjpeg.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "image_io.h"

namespace gs::detail {

namespace {

void nvjpeg_ok(nvjpegStatus_t s, const char* what) {
  if (s != NVJPEG_STATUS_SUCCESS) throw std::runtime_error(std::string("JPEG: ") + what + " (nvJPEG status " + std::to_string(int(s)) + ")");
}

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("JPEG: ") + what + ": " + cudaGetErrorString(e));
}

// One decoder per process, created on first use with the caller's current device.
struct Decoder {
  nvjpegHandle_t handle = nullptr;
  nvjpegJpegState_t state = nullptr;
  Decoder() {
    nvjpeg_ok(nvjpegCreateSimple(&handle), "no decoder (nvjpegCreateSimple)");
    const nvjpegStatus_t s = nvjpegJpegStateCreate(handle, &state);
    if (s != NVJPEG_STATUS_SUCCESS) {
      nvjpegDestroy(handle);
      nvjpeg_ok(s, "nvjpegJpegStateCreate");
    }
  }
  ~Decoder() {
    if (state) nvjpegJpegStateDestroy(state);
    if (handle) nvjpegDestroy(handle);
  }
};

std::mutex g_mutex;
Decoder* g_decoder = nullptr;  // kept until exit (destroying it at exit races the CUDA runtime's teardown)

// A device buffer freed on every path.
struct DeviceBytes {
  unsigned char* p = nullptr;
  ~DeviceBytes() {
    if (p) cudaFree(p);
  }
};

}  // namespace

Image decode_jpeg(const std::vector<uint8_t>& bytes, uint32_t channels) {
  if (channels != 1 && channels != 4) throw std::runtime_error("decode_jpeg: 1 or 4 channels");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_decoder == nullptr) g_decoder = new Decoder();
  int components = 0;
  nvjpegChromaSubsampling_t subsampling;
  int widths[NVJPEG_MAX_COMPONENT] = {}, heights[NVJPEG_MAX_COMPONENT] = {};
  nvjpeg_ok(nvjpegGetImageInfo(g_decoder->handle, bytes.data(), bytes.size(), &components, &subsampling, widths, heights),
            "not a decodable JPEG");
  const uint32_t w = uint32_t(widths[0]), h = uint32_t(heights[0]);
  if (w == 0 || h == 0) throw std::runtime_error("JPEG: empty image");
  DeviceBytes rgb;
  cuda_ok(cudaMalloc(&rgb.p, size_t(w) * h * 3), "device buffer");
  nvjpegImage_t out{};
  out.channel[0] = rgb.p;
  out.pitch[0] = size_t(w) * 3;
  nvjpeg_ok(nvjpegDecode(g_decoder->handle, g_decoder->state, bytes.data(), bytes.size(), NVJPEG_OUTPUT_RGBI, &out,
                         nullptr),
            "decode");
  std::vector<uint8_t> host(size_t(w) * h * 3);
  cuda_ok(cudaMemcpy(host.data(), rgb.p, host.size(), cudaMemcpyDeviceToHost), "copy back");
  Image img;
  img.width = w;
  img.height = h;
  img.channels = channels;
  img.data.resize(size_t(w) * h * channels);
  for (size_t p = 0; p < size_t(w) * h; ++p) {
    const uint8_t* s = &host[p * 3];
    uint8_t* d = &img.data[p * channels];
    if (channels == 1) {
      // A single-component JPEG comes back as equal R, G, B: its luma.
      d[0] = uint8_t((uint32_t(s[0]) * 299u + uint32_t(s[1]) * 587u + uint32_t(s[2]) * 114u + 500u) / 1000u);
    } else {
      d[0] = s[0];
      d[1] = s[1];
      d[2] = s[2];
      d[3] = 255;
    }
  }
  return img;
}

}  // namespace gs::detail
