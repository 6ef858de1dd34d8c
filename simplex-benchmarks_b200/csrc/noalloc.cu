// DG / Helmholtz vmult whose scratch lives in a fixed, file-scope device array.
//
// Why: fem_op_vmult uses a scratch buffer (the published face normal
// derivatives) that fem_op_create obtains with cudaMalloc.  Some callers must
// not allocate device memory: an application whose memory pool (a framework's
// caching allocator, a pre-reserved arena) already owns the whole device, or a
// latency-bound loop where cudaMalloc/cudaFree, which may synchronise the
// device and take unbounded time, are not allowed.  fem_op_vmult_static_scratch
// gives them the same product with the scratch taken from g_static_scratch
// below, a static device array that exists on every GPU that loads this
// library, from module load until process exit.
//
// Limits and rules:
//   - at most kStaticScratchBytes (16 MiB) of scratch: DG P3 FP64 up to 87,381
//     cells (e.g. 24^3 x 6 = 82,944); larger problems are rejected with FEM_ERR_ARG;
//   - every call shares the one array and leaves its contents behind; the
//     scratch is fully written before it is read in each call, so nothing has
//     to start at zero;
//   - calls whose kernels overlap on the GPU (other streams, other threads)
//     race on the array and give wrong results: order them on one stream;
//   - on each device, the first call looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture.
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
void* static_scratch_address() {
  int dev = -1;
  SFEM_CUDA(cudaGetDevice(&dev));
  SFEM_REQUIRE(dev >= 0 && dev < kMaxDevices, FEM_ERR_INTERNAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error(FEM_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
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
    void* scratch = sfem::static_scratch_address();
    op->op->vmult_with_scratch(dst, src, scratch, sfem::kStaticScratchBytes, static_cast<cudaStream_t>(stream));
  });
}
