// Per-cell MLP of the learned smoother: 29 -> 64 -> 64 -> 20, GELU (tanh form), BF16
// weights, FP32 accumulation.  No counterpart in the reference (its finest
// level is always smoothed by PreconditionChebyshev).
//
// Inputs of a cell K: the 20 P3 residual values r_K / s_K (s_K = ||r_K||_2)
// and the 9 entries of J_K / h_K (h_K = |det J_K|^(1/3)); output o (20); the
// correction is (s_K / h_K) o, so the map is scale-equivariant in r and in
// the mesh size (the Laplace stiffness scales like h).  Corrections are
// assembled with inverse-multiplicity weights (additive Schwarz with one
// cell per subdomain).
//
// Parameter layout (FP32 master copy and its BF16 image):
//   W1 [64][29], b1 [64], W2 [64][64], b2 [64], W3 [20][64], b3 [20]
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mlp_dims.hpp"

namespace sfem {

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
// (Hendrycks & Gimpel), and its derivative.
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanhf(0.7978845608028654f * (x + 0.044715f * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}
// the same GELU with the hardware tanh approximation (tensor-core epilogues)
// (6 instructions: u = x (c1 + c2 x^2), y = h + h tanh(u), h = x / 2)
__device__ __forceinline__ float gelu_fast(float x) {
  const float u = x * fmaf(0.7978845608028654f * 0.044715f, x * x, 0.7978845608028654f);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  const float h = 0.5f * x;
  return fmaf(h, t, h);
}

// FP32 master -> BF16 image
__global__ void mlp_round_weights(int n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wb[i] = __float2bfloat16(w[i]);
}

// stage the BF16 weights in shared memory as FP32
__device__ __forceinline__ void mlp_load_weights(float* sw, const __nv_bfloat16* __restrict__ wb) {
  for (int i = threadIdx.x; i < MLPDims::NPARAM; i += blockDim.x) sw[i] = __bfloat162float(wb[i]);
}

// forward of one sample; a1/a2 are the pre-activations (kept for backward)
__device__ __forceinline__ void mlp_forward(const float* sw, const float (&x)[MLPDims::NIN], float (&a1)[MLPDims::NH],
                                            float (&a2)[MLPDims::NH], float (&o)[MLPDims::NOUT]) {
  using D = MLPDims;
  float h[D::NH];
#pragma unroll 4
  for (int j = 0; j < D::NH; ++j) {
    float acc = sw[D::OFF_B1 + j];
#pragma unroll
    for (int i = 0; i < D::NIN; ++i) acc = fmaf(sw[D::OFF_W1 + j * D::NIN + i], x[i], acc);
    a1[j] = acc;
  }
#pragma unroll
  for (int j = 0; j < D::NH; ++j) h[j] = gelu(a1[j]);
#pragma unroll 4
  for (int j = 0; j < D::NH; ++j) {
    float acc = sw[D::OFF_B2 + j];
#pragma unroll
    for (int i = 0; i < D::NH; ++i) acc = fmaf(sw[D::OFF_W2 + j * D::NH + i], h[i], acc);
    a2[j] = acc;
  }
#pragma unroll
  for (int j = 0; j < D::NH; ++j) h[j] = gelu(a2[j]);
#pragma unroll 4
  for (int j = 0; j < D::NOUT; ++j) {
    float acc = sw[D::OFF_B3 + j];
#pragma unroll
    for (int i = 0; i < D::NH; ++i) acc = fmaf(sw[D::OFF_W3 + j * D::NH + i], h[i], acc);
    o[j] = acc;
  }
}

// Fused learned smoothing step on a P3 CG level: z += sum_K w (s_K/h_K) MLP(r_K/s_K, J_K/h_K).
// dofs: [20][n_cells] (-1 at constrained DoFs), feat: [n_cells][10] = J/h (9) and 1/h,
// winv: inverse multiplicity [m].
template <typename T>
__global__ void __launch_bounds__(128) mlp_smooth_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
                                                         const float* __restrict__ feat,
                                                         const float* __restrict__ winv,
                                                         const __nv_bfloat16* __restrict__ wb,
                                                         const T* __restrict__ r, T* __restrict__ z) {
  using D = MLPDims;
  __shared__ float sw[D::NPARAM];
  mlp_load_weights(sw, wb);
  __syncthreads();
  for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < n_cells;
       c += int64_t(gridDim.x) * blockDim.x) {
    float x[D::NIN];
    int32_t g[D::NR];
    float s2 = 0.0f;
#pragma unroll
    for (int i = 0; i < D::NR; ++i) {
      g[i] = dofs[i * n_cells + c];
      x[i] = g[i] >= 0 ? float(r[g[i]]) : 0.0f;
      s2 += x[i] * x[i];
    }
    if (s2 == 0.0f) continue;
    const float s = sqrtf(s2), is = 1.0f / s;
#pragma unroll
    for (int i = 0; i < D::NR; ++i) x[i] *= is;
#pragma unroll
    for (int k = 0; k < D::NJ; ++k) x[D::NR + k] = feat[c * 10 + k];
    const float scale = s * feat[c * 10 + 9];
    float a1[D::NH], a2[D::NH], o[D::NOUT];
    mlp_forward(sw, x, a1, a2, o);
#pragma unroll
    for (int i = 0; i < D::NR; ++i)
      if (g[i] >= 0) atomicAdd(z + g[i], T(scale * o[i] * winv[g[i]]));
  }
}

// One optimisation step's gradient over a batch: loss = mean_b ||o_b - y_b||^2.
// X [n][29], Y [n][20]; grad (FP32, zeroed by the caller) accumulates dLoss/dW
// (of the BF16 weights); loss_sum accumulates the summed loss.
__global__ void __launch_bounds__(128) mlp_grad_kernel(int n, const float* __restrict__ X,
                                                       const float* __restrict__ Y,
                                                       const __nv_bfloat16* __restrict__ wb, float* __restrict__ grad,
                                                       float* __restrict__ loss_sum, float inv_batch) {
  using D = MLPDims;
  extern __shared__ float smem_f[];  // 2 * NPARAM floats (dynamic, > 48 KB)
  float* sw = smem_f;
  float* sg = smem_f + D::NPARAM;
  mlp_load_weights(sw, wb);
  for (int i = threadIdx.x; i < D::NPARAM; i += blockDim.x) sg[i] = 0.0f;
  __syncthreads();
  float lsum = 0.0f;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    float x[D::NIN], a1[D::NH], a2[D::NH], o[D::NOUT];
#pragma unroll
    for (int i = 0; i < D::NIN; ++i) x[i] = X[int64_t(b) * D::NIN + i];
    mlp_forward(sw, x, a1, a2, o);
    float dlo[D::NOUT];
#pragma unroll
    for (int j = 0; j < D::NOUT; ++j) {
      const float d = o[j] - Y[int64_t(b) * D::NOUT + j];
      lsum += d * d;
      dlo[j] = 2.0f * d * inv_batch;
    }
    // layer 3
    float h2[D::NH], dh[D::NH];
#pragma unroll
    for (int i = 0; i < D::NH; ++i) {
      h2[i] = gelu(a2[i]);
      dh[i] = 0.0f;
    }
    for (int j = 0; j < D::NOUT; ++j) {
      atomicAdd(&sg[D::OFF_B3 + j], dlo[j]);
#pragma unroll
      for (int i = 0; i < D::NH; ++i) {
        atomicAdd(&sg[D::OFF_W3 + j * D::NH + i], dlo[j] * h2[i]);
        dh[i] = fmaf(sw[D::OFF_W3 + j * D::NH + i], dlo[j], dh[i]);
      }
    }
    // layer 2
#pragma unroll
    for (int i = 0; i < D::NH; ++i) dh[i] *= gelu_grad(a2[i]);
    float h1[D::NH], dh1[D::NH];
#pragma unroll
    for (int i = 0; i < D::NH; ++i) {
      h1[i] = gelu(a1[i]);
      dh1[i] = 0.0f;
    }
    for (int j = 0; j < D::NH; ++j) {
      atomicAdd(&sg[D::OFF_B2 + j], dh[j]);
#pragma unroll
      for (int i = 0; i < D::NH; ++i) {
        atomicAdd(&sg[D::OFF_W2 + j * D::NH + i], dh[j] * h1[i]);
        dh1[i] = fmaf(sw[D::OFF_W2 + j * D::NH + i], dh[j], dh1[i]);
      }
    }
    // layer 1
    for (int j = 0; j < D::NH; ++j) {
      const float d = dh1[j] * gelu_grad(a1[j]);
      atomicAdd(&sg[D::OFF_B1 + j], d);
#pragma unroll
      for (int i = 0; i < D::NIN; ++i) atomicAdd(&sg[D::OFF_W1 + j * D::NIN + i], d * x[i]);
    }
  }
  atomicAdd(loss_sum, lsum);
  __syncthreads();
  for (int i = threadIdx.x; i < D::NPARAM; i += blockDim.x)
    if (sg[i] != 0.0f) atomicAdd(grad + i, sg[i]);
}

// forward only, for evaluation: O [n][20]
__global__ void __launch_bounds__(128) mlp_forward_kernel(int n, const float* __restrict__ X,
                                                          const __nv_bfloat16* __restrict__ wb, float* __restrict__ O) {
  using D = MLPDims;
  __shared__ float sw[D::NPARAM];
  mlp_load_weights(sw, wb);
  __syncthreads();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    float x[D::NIN], a1[D::NH], a2[D::NH], o[D::NOUT];
#pragma unroll
    for (int i = 0; i < D::NIN; ++i) x[i] = X[int64_t(b) * D::NIN + i];
    mlp_forward(sw, x, a1, a2, o);
#pragma unroll
    for (int j = 0; j < D::NOUT; ++j) O[int64_t(b) * D::NOUT + j] = o[j];
  }
}

// Adam (decoupled weight decay off)
__global__ void mlp_adam_kernel(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// Training samples from a solver state: for the selected cells, X = (r_K/s, J/h)
// and Y = e_K h / s (normalised error), constrained DoFs as zeros.
template <typename T>
__global__ void mlp_extract_kernel(int n_sel, const int32_t* __restrict__ sel, int64_t n_cells,
                                   const int32_t* __restrict__ dofs, const float* __restrict__ feat,
                                   const T* __restrict__ r, const T* __restrict__ e, float* __restrict__ X,
                                   float* __restrict__ Y, int32_t* __restrict__ valid) {
  using D = MLPDims;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_sel) return;
  const int64_t c = sel[b];
  float rr[D::NR], ee[D::NR], s2 = 0.0f;
  for (int i = 0; i < D::NR; ++i) {
    const int32_t g = dofs[i * n_cells + c];
    rr[i] = g >= 0 ? float(r[g]) : 0.0f;
    ee[i] = g >= 0 ? float(e[g]) : 0.0f;
    s2 += rr[i] * rr[i];
  }
  const float s = sqrtf(s2);
  valid[b] = s > 0.0f;
  const float is = s > 0.0f ? 1.0f / s : 0.0f, h = 1.0f / feat[c * 10 + 9];
  for (int i = 0; i < D::NR; ++i) {
    X[int64_t(b) * D::NIN + i] = rr[i] * is;
    Y[int64_t(b) * D::NOUT + i] = ee[i] * h * is;
  }
  for (int k = 0; k < D::NJ; ++k) X[int64_t(b) * D::NIN + D::NR + k] = feat[c * 10 + k];
}

}  // namespace sfem
