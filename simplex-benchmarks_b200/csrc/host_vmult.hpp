// vmult on vectors in host memory, pipelined over several vectors (see
// host_vmult.cu).
#pragma once
#include <cuda_runtime.h>

#include "operator.hpp"

namespace sfem {

// dst[i] = A src[i] for i < n, all vectors in host memory; enqueued on s.
void vmult_host(Operator& op, int n, void* const* dst, const void* const* src, cudaStream_t s);

}  // namespace sfem
