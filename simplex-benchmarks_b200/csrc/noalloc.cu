// DG / Helmholtz vmult whose scratch lives in a fixed, file-scope device array.
//
// What the call provides: it allocates no device memory, and it does not use
// the operator's own scratch buffer (the published face normal derivatives,
// which fem_op_create allocates once with the operator's other tables).  The
// scratch comes instead from g_static_scratch below, a static device array
// that exists on every GPU that loads this library, from module load until
// process exit, whether or not this call is ever made (16 MiB per GPU).
//
// Who needs it: callers that cannot call cudaMalloc where they set up their
// per-apply working memory - an application whose memory pool (a framework's
// caching allocator, a pre-reserved arena) owns the rest of the device, or one
// that must not add a device allocation per concurrent apply.  fem_op_vmult
// allocates nothing at the call either; the difference is that every apply
// through this entry point shares one library-owned buffer instead of the
// operator's.  Creating the operator still allocates its tables.
//
// Limits and rules:
//   - at most kStaticScratchBytes (16 MiB) of scratch (traces of whole 128-cell
//     blocks): DG P3 FP64 up to 87,296
//     cells (e.g. 24^3 x 6 = 82,944); larger problems are rejected with FEM_ERR_ARG;
//   - every call shares the one array and leaves its contents behind; the
//     scratch is fully written before it is read in each call, so nothing has
//     to start at zero;
//   - calls whose kernels overlap on the GPU (other streams, other threads)
//     race on the array and give wrong results: order them on one stream;
//   - the array's device address is looked up (cudaGetSymbolAddress, with the
//     device current) on every call made outside stream capture, so it stays
//     right after a device reset; a call made while `stream` is capturing uses
//     the address found by the last uncaptured call on that device, so make one
//     call on each device before capturing.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "handles.hpp"

namespace sfem {
namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device.  In host code the
// symbol only names a host-side shadow; its device address must be looked up.
// Outside stream capture the lookup is repeated (it is cheap), so a context
// that was reset and re-created never gets a stale address; under capture the
// last looked-up address of the device is used.
void* static_scratch_address(cudaStream_t stream) {
  int dev = -1;
  SFEM_CUDA(cudaGetDevice(&dev));
  SFEM_REQUIRE(dev >= 0 && dev < kMaxDevices, FEM_ERR_INTERNAL, "device ordinal out of range");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SFEM_CUDA(cudaStreamIsCapturing(stream, &cap));
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap != cudaStreamCaptureStatusNone) {
    SFEM_REQUIRE(g_scratch_ptr[dev] != nullptr, FEM_ERR_STATE,
                 "fem_op_vmult_static_scratch: make one call on this device before stream capture");
    return g_scratch_ptr[dev];
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess || p == nullptr)
    throw Error(FEM_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
  g_scratch_ptr[dev] = p;
  return p;
}

}  // namespace
}  // namespace sfem

extern "C" int fem_op_vmult_static_scratch(fem_op* op, void* dst, const void* src, void* stream) {
  return sfem::guarded([&] {
    SFEM_REQUIRE_PTR(op);
    SFEM_REQUIRE_PTR(dst);
    SFEM_REQUIRE_PTR(src);
    SFEM_REQUIRE(dst != src, FEM_ERR_ARG, "vmult: dst and src must not alias");
    SFEM_REQUIRE(op->op->cfg.kind != FEM_CG, FEM_ERR_ARG,
                 "fem_op_vmult_static_scratch: only DG and Helmholtz operators use scratch");
    const size_t need = op->op->scratch_bytes();
    SFEM_REQUIRE(need <= sfem::kStaticScratchBytes, FEM_ERR_ARG,
                 "fem_op_vmult_static_scratch: operator needs " + std::to_string(need) +
                     " bytes of scratch, more than the static maximum of " +
                     std::to_string(sfem::kStaticScratchBytes) + " bytes");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* scratch = sfem::static_scratch_address(s);
    op->op->vmult_with_scratch(dst, src, scratch, sfem::kStaticScratchBytes, s);
  });
}
