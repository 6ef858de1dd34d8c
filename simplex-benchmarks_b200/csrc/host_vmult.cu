// vmult on vectors in host memory (fem_op_vmult_host).
//
// The reference's operator is applied to deal.II vectors that live in host
// memory (Operator::vmult(dst, src), CG/cells_batched/application.cc:1154-1176,
// DG/cells_batched/application.cc:1303-1316).  A drop-in that keeps those
// vectors on the host has to move src to the device and dst back on every
// call; on a PCIe-attached GPU those two copies take far longer than the
// operator itself (DG P3 on 32^3 x 6 tets: 2 x 31.5 MB against ~90 us).
//
// The copies of consecutive vectors are therefore pipelined through two
// device staging pairs owned by the operator and three streams:
//   copy-in  stream: src_i -> stage_src[i % 2]
//   compute  stream: stage_dst[i % 2] = A stage_src[i % 2]
//   copy-out stream: stage_dst[i % 2] -> dst_i
// so that (with pinned host memory, which copies asynchronously) the copy-in
// of vector i+1, the apply of vector i and the copy-out of vector i-1 run at
// the same time on the two PCIe directions and the SMs.  Events order the
// reuse of a staging buffer after the work of vector i-2 that read it.  All
// three streams first wait for the caller's stream, and the caller's stream
// waits for the last copy-out, so the call behaves as one operation enqueued
// on `stream`.
#include "host_vmult.hpp"

namespace sfem {

struct HostPipe {
  DevBuf<unsigned char> src[2], dst[2];
  cudaStream_t st[3] = {nullptr, nullptr, nullptr};  // copy-in, compute, copy-out
  cudaEvent_t start = nullptr, loaded[2] = {}, computed[2] = {}, stored[2] = {};
  HostPipe() {
    for (auto& s : st) SFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    SFEM_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    for (int b = 0; b < 2; ++b) {
      SFEM_CUDA(cudaEventCreateWithFlags(&loaded[b], cudaEventDisableTiming));
      SFEM_CUDA(cudaEventCreateWithFlags(&computed[b], cudaEventDisableTiming));
      SFEM_CUDA(cudaEventCreateWithFlags(&stored[b], cudaEventDisableTiming));
    }
  }
  ~HostPipe() {
    for (int b = 0; b < 2; ++b) {
      if (loaded[b]) cudaEventDestroy(loaded[b]);
      if (computed[b]) cudaEventDestroy(computed[b]);
      if (stored[b]) cudaEventDestroy(stored[b]);
    }
    if (start) cudaEventDestroy(start);
    for (auto& s : st)
      if (s) cudaStreamDestroy(s);
  }
};

void vmult_host(Operator& op, int n, void* const* dst, const void* const* src, cudaStream_t s) {
  SFEM_REQUIRE(n >= 1, FEM_ERR_ARG, "vmult_host: n must be >= 1");
  for (int i = 0; i < n; ++i)
    SFEM_REQUIRE(dst[i] != nullptr && src[i] != nullptr, FEM_ERR_ARG, "vmult_host: null host vector");
  const size_t bytes = size_t(op.m) * op.elem_size();
  if (!op.host_pipe) op.host_pipe = std::make_shared<HostPipe>();
  HostPipe& h = *op.host_pipe;
  for (int b = 0; b < 2; ++b) {
    if (h.src[b].n != bytes) h.src[b].alloc(bytes);
    if (h.dst[b].n != bytes) h.dst[b].alloc(bytes);
  }
  cudaStream_t in = h.st[0], comp = h.st[1], out = h.st[2];
  SFEM_CUDA(cudaEventRecord(h.start, s));
  for (cudaStream_t q : h.st) SFEM_CUDA(cudaStreamWaitEvent(q, h.start, 0));
  // a previous call may have been joined into another caller stream: order the
  // staging buffers after its last apply and copy-outs (waiting for an event
  // that was never recorded returns at once)
  for (int b = 0; b < 2; ++b) {
    SFEM_CUDA(cudaStreamWaitEvent(in, h.computed[b], 0));
    SFEM_CUDA(cudaStreamWaitEvent(comp, h.stored[b], 0));
  }
  for (int i = 0; i < n; ++i) {
    const int b = i & 1;
    if (i >= 2) SFEM_CUDA(cudaStreamWaitEvent(in, h.computed[b], 0));  // vector i-2 no longer reads src[b]
    SFEM_CUDA(cudaMemcpyAsync(h.src[b].p, src[i], bytes, cudaMemcpyHostToDevice, in));
    SFEM_CUDA(cudaEventRecord(h.loaded[b], in));
    SFEM_CUDA(cudaStreamWaitEvent(comp, h.loaded[b], 0));
    if (i >= 2) SFEM_CUDA(cudaStreamWaitEvent(comp, h.stored[b], 0));  // dst[b] of vector i-2 copied out
    op.vmult(h.dst[b].p, h.src[b].p, comp);
    SFEM_CUDA(cudaEventRecord(h.computed[b], comp));
    SFEM_CUDA(cudaStreamWaitEvent(out, h.computed[b], 0));
    SFEM_CUDA(cudaMemcpyAsync(dst[i], h.dst[b].p, bytes, cudaMemcpyDeviceToHost, out));
    SFEM_CUDA(cudaEventRecord(h.stored[b], out));
  }
  // the copy-out stream is in order: its last event covers every vector
  SFEM_CUDA(cudaStreamWaitEvent(s, h.stored[(n - 1) & 1], 0));
}

}  // namespace sfem
