// Vector kernels of the solvers and the multigrid cycle (FP64 and FP32).
//
// These replace the deal.II LinearAlgebra::distributed::Vector operations
// used by SolverCG, PreconditionChebyshev and MGTransferGlobalCoarsening
// (add/sadd/equ/scale, dot products, norms).  Reductions are two-stage with a
// fixed block order, so results are bitwise reproducible.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sfem {

constexpr int kReduceBlocks = 592;  // 4 x 148 SMs
constexpr int kReduceThreads = 256;

template <typename To, typename Ti>
__global__ void vec_convert(int64_t n, const Ti* __restrict__ in, To* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = To(in[i]);
}

// y = a x + b y
template <typename T>
__global__ void vec_axpby(int64_t n, T a, const T* __restrict__ x, T b, T* __restrict__ y) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// r = b - t
template <typename T>
__global__ void vec_residual(int64_t n, const T* __restrict__ b, const T* __restrict__ t, T* __restrict__ r) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    r[i] = b[i] - t[i];
}

// z = invd .* r
template <typename T>
__global__ void vec_scale(int64_t n, const T* __restrict__ invd, const T* __restrict__ r, T* __restrict__ z) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    z[i] = invd[i] * r[i];
}

// block partial sums of x.y (double accumulation), then one block sums the partials
template <typename T>
__global__ void __launch_bounds__(kReduceThreads) vec_dot_partial(int64_t n, const T* __restrict__ x,
                                                                  const T* __restrict__ y, double* partial) {
  __shared__ double s[kReduceThreads];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    acc += double(x[i]) * double(y[i]);
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

static __global__ void __launch_bounds__(kReduceThreads) reduce_partials(int n, const double* partial, double* out) {
  __shared__ double s[kReduceThreads];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// Chebyshev, first step from a zero initial guess: d = c P b, x = d
template <typename T>
__global__ void cheb_first_zero(int64_t n, T c, const T* __restrict__ invd, const T* __restrict__ b,
                                T* __restrict__ d, T* __restrict__ x) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T v = c * invd[i] * b[i];
    d[i] = v;
    x[i] = v;
  }
}

// Chebyshev step: d = f1 d + f2 P (b - t), x += d   (t = A x); FIRST: the
// first step from a nonzero x, d = f2 P (b - t) (d is not read)
template <typename T, bool FIRST = false>
__global__ void cheb_step(int64_t n, T f1, T f2, const T* __restrict__ invd, const T* __restrict__ b,
                          const T* __restrict__ t, T* __restrict__ d, T* __restrict__ x) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const T v = (FIRST ? T(0) : f1 * d[i]) + f2 * invd[i] * (b[i] - t[i]);
    d[i] = v;
    x[i] += v;
  }
}

// y[r] += sum_k val[k] x[col[k]]  (CSR rows; used for prolongation and, with
// the transposed matrix, for restriction)
template <typename T>
__global__ void csr_spmv_add(int64_t nrows, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                             const double* __restrict__ val, const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < nrows; r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t a = rowptr[r], e = rowptr[r + 1];
    if (a == e) continue;
    double acc = 0.0;
    for (int64_t k = a; k < e; ++k) acc += val[k] * double(x[col[k]]);
    y[r] += T(acc);
  }
}

// y = A x for a small dense FP64 matrix (coarse-grid solve), one warp per row
template <typename T>
__global__ void dense_matvec(int n, const double* __restrict__ A, const T* __restrict__ x, T* __restrict__ y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  double acc = 0.0;
  for (int j = lane; j < n; j += 32) acc += A[int64_t(warp) * n + j] * double(x[j]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) y[warp] = T(acc);
}

// CG update with the step read on the device: alpha = sc[rz] / sc[pq];
// nothing is updated unless sc[pq] is finite and positive (the host reads
// sc[pq] after the step and reports the breakdown)
static __global__ void cg_update_xr_dev(int64_t n, const double* __restrict__ sc, int rz, int pq,
                                        const double* __restrict__ p, const double* __restrict__ q,
                                        double* __restrict__ x, double* __restrict__ r) {
  const double den = sc[pq];
  if (!(den > 0) || !isfinite(den)) return;
  const double alpha = sc[rz] / den;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] += alpha * p[i];
    r[i] -= alpha * q[i];
  }
}

// p = a z + beta p with beta = (sc[num] - (sub >= 0 ? sc[sub] : 0)) / sc[den], read on the device
static __global__ void cg_update_p_dev(int64_t n, double a, const double* __restrict__ sc, int num, int sub, int den,
                                       const double* __restrict__ z, double* __restrict__ p) {
  const double beta = (sub >= 0 ? sc[num] - sc[sub] : sc[num]) / sc[den];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = a * z[i] + beta * p[i];
}

// x += (sc[0]/sc[1]) z  (step 0 unless sc[1] > 0); the ratio stays on the device
template <typename T>
__global__ void axpy_ratio(int64_t n, const double* __restrict__ sc, const T* __restrict__ z, T* __restrict__ x) {
  const double den = sc[1];
  const T w = den > 0.0 ? T(sc[0] / den) : T(0);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] += w * z[i];
}

// r = b - (sc[0]/sc[1]) q
template <typename T>
__global__ void residual_ratio(int64_t n, const double* __restrict__ sc, const T* __restrict__ b,
                               const T* __restrict__ q, T* __restrict__ r) {
  const double den = sc[1];
  const T w = den > 0.0 ? T(sc[0] / den) : T(0);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    r[i] = b[i] - w * q[i];
}

inline unsigned grid_for(int64_t n, int bs = 256, unsigned cap = 148 * 16) {
  const int64_t b = (n + bs - 1) / bs;
  return unsigned(b < cap ? (b > 0 ? b : 1) : cap);
}

}  // namespace sfem
