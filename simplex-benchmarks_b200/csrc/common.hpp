// Shared host-side utilities: error reporting and checked CUDA calls.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>

namespace sfem {

// Error raised anywhere below the C ABI; converted to a status code plus a
// message readable through fem_last_error_string().
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);
const char* last_error();

}  // namespace sfem

#define SFEM_REQUIRE(cond, code, msg)                                   \
  do {                                                                  \
    if (!(cond)) throw ::sfem::Error((code), std::string(msg));         \
  } while (0)

#ifdef __CUDACC__
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "../../include/simplex_fem.h"
#define SFEM_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw ::sfem::Error(FEM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace sfem {
inline std::mutex& device_setup_mutex() {
  static std::mutex m;
  return m;
}
// Per-device one-time set-up (kernel attributes are set per device): runs
// init() the first time it is called with `mask` while device `dev` is
// current.  Bit d of the mask stands for device d (ordinals of 64 and above
// are refused); it is set only after init() has finished, and concurrent
// first callers wait for it, so no caller launches a kernel before its
// attributes are in place.  If init() throws, the device stays unconfigured.
template <class F>
inline void once_per_device(std::atomic<uint64_t>& mask, int dev, F&& init) {
  if (dev < 0 || dev >= 64) throw Error(FEM_ERR_INTERNAL, "device ordinal out of range (0..63)");
  const uint64_t bit = uint64_t(1) << dev;
  if (mask.load(std::memory_order_acquire) & bit) return;
  std::lock_guard<std::mutex> lock(device_setup_mutex());
  if (mask.load(std::memory_order_relaxed) & bit) return;
  init();
  mask.fetch_or(bit, std::memory_order_release);
}
}  // namespace sfem
#endif
