// gs_sort_pairs_noalloc: the library's stable radix sort of (key, value) pairs for callers
// that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: host runtimes that hand all device memory to their
// own pool and forbid allocations outside it, plugins that run inside such a runtime and
// get only the buffers it passes them, and tight loops where an allocation's implicit
// device synchronisation costs more than the sort. For them this entry point sorts
// buffers the caller already owns and takes its scratch — the alternate key/value
// buffers, the digit histograms and the per-tile digit counts — from one file-scope
// device array of fixed size instead of allocating it. Every GPU
// that loads the library holds that array (about 8.3 MB) until the process exits.
//
// The first call on a device does the set-up (the array's device address, looked up with
// that device current) and should come before any stream capture. All calls share the
// array, which keeps the last call's contents; calls that overlap on the GPU race.
#include <mutex>
#include <string>

#include "gs_kernels.h"

namespace {

constexpr uint32_t kMaxItems = 1u << 20;  // GS_SORT_NOALLOC_MAX_ITEMS
constexpr uint32_t kMaxTiles = (kMaxItems + gsk::kSortTile - 1u) / gsk::kSortTile;
// Word offsets of the scratch parts.
constexpr size_t kAltKeys = 0;
constexpr size_t kAltVals = kAltKeys + kMaxItems;
constexpr size_t kHist = kAltVals + kMaxItems;
constexpr size_t kTileCounts = kHist + 4 * 256;
constexpr size_t kWords = kTileCounts + size_t(kMaxTiles) * 256;

// The scratch. Host code must not take this name as a device address: it is a host-side
// stand-in for the symbol. The device address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) uint32_t g_sort_scratch[kWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

namespace gsk {
// The thread's error message of libgs_cuda (api.cu).
void set_last_error(const std::string& message);
}  // namespace gsk

extern "C" int gs_sort_pairs_noalloc(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t key_bits, void* stream) {
  auto failed = [](int code, const std::string& message) {
    gsk::set_last_error(message);
    return code;
  };
  if (n > kMaxItems)
    return failed(GS_ERR_INVALID, "gs_sort_pairs_noalloc: " + std::to_string(n) + " pairs exceed the maximum of " +
                                      std::to_string(kMaxItems));
  if (key_bits == 0u || key_bits > 32u) return failed(GS_ERR_INVALID, "gs_sort_pairs_noalloc: key_bits must be 1..32");
  if (n > 0u && (keys == nullptr || values == nullptr)) return failed(GS_ERR_INVALID, "gs_sort_pairs_noalloc: null buffer");
  // A launch error the caller left pending on this thread is not this call's: report it as
  // such and leave it in place, rather than return it later as a failed sort.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: a CUDA error was pending before the call: ") +
                                   cudaGetErrorString(e));
  int device = 0;
  e = cudaGetDevice(&device);
  if (e != cudaSuccess) return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: ") + cudaGetErrorString(e));
  if (device < 0 || device >= kMaxDevices) return failed(GS_ERR_INVALID, "gs_sort_pairs_noalloc: device index too large");
  uint32_t* base = nullptr;
  {
    // Set-up, once per device, with that device current: the scratch's device address.
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[device] == nullptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sort_scratch);
      if (e != cudaSuccess)
        return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[device] = static_cast<uint32_t*>(p);
    }
    base = g_scratch_ptr[device];
  }
  if (n <= 1u) return GS_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  gsk::SortScratch s;
  s.hist = base + kHist;
  s.tile_counts = base + kTileCounts;
  s.count_tiles = kMaxTiles;
  // The array keeps the previous call's contents; the sort clears its histograms and
  // overwrites the tile counts it reads, so nothing needs clearing here.
  const bool in_alt = gsk::radix_sort_pairs(s, keys, values, base + kAltKeys, base + kAltVals, nullptr, n,
                                            int(key_bits), st, nullptr);
  e = cudaGetLastError();  // the sort's launches
  if (e != cudaSuccess)
    return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: sort launch: ") + cudaGetErrorString(e));
  if (in_alt) {
    e = cudaMemcpyAsync(keys, base + kAltKeys, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(values, base + kAltVals, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess)
      return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: copy back: ") + cudaGetErrorString(e));
  }
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return failed(GS_ERR_CUDA, std::string("gs_sort_pairs_noalloc: ") + cudaGetErrorString(e));
  gsk::set_last_error("");
  return GS_OK;
}
