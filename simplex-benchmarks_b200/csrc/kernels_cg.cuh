// Continuous Galerkin Laplace cell kernel (sm_100a).
//
// Restates the reference's fused cell loop do_cell_integral_masked_gather
// (CG/cells_batched/application.cc:1237-1416): masked gather of the cell DoFs
// (constrained -> 0, :1278-1306), reference-gradient contraction (:1314),
// affine metric w_q J^-1 J^-T |J| (:1333-1360), transposed contraction
// (:1381) and scatter-add that skips constrained DoFs (:1391-1412).
//
// B200 form: one thread per cell, cells in hierarchical order, all shape
// matrices are compile-time constants (ref_kernels.cuh) so the contractions
// are pure register FMAs.  The gradient of a P_p function is represented
// exactly in the P_{p-1} nodal basis and integrated with the P_{p-1}
// reference mass, which is the minimal exact "quadrature" for affine cells
// (the reference's QGaussSimplex(p+1) is exact for the same integrand).
#pragma once
#include <cstdint>

#include "ref_kernels.cuh"

namespace sfem {

// G = |det J| J^-1 J^-T stored as (00, 11, 22, 01, 02, 12); w_b = sum_a G_ab g_a
template <int KQ, typename T>
__device__ __forceinline__ void apply_metric(const T (&G)[6], const T* g, T* w) {
#pragma unroll
  for (int m = 0; m < KQ; ++m) {
    const T g0 = g[m], g1 = g[KQ + m], g2 = g[2 * KQ + m];
    w[m] = G[0] * g0 + G[3] * g1 + G[4] * g2;
    w[KQ + m] = G[3] * g0 + G[1] * g1 + G[5] * g2;
    w[2 * KQ + m] = G[4] * g0 + G[5] * g1 + G[2] * g2;
  }
}

// Local Laplace stiffness of one cell applied to u: y = A_K u.
template <int P, typename T>
__device__ __forceinline__ void cg_local_apply(const T (&G)[6], const T (&u)[gen::Ops<P>::K],
                                               T (&y)[gen::Ops<P>::K]) {
  using O = gen::Ops<P>;
  T g[3 * O::KQ];
  O::grad(u, g);
  T w[3 * O::KQ];
  apply_metric<O::KQ>(G, g, w);
  T h[3 * O::KQ];
#pragma unroll
  for (int a = 0; a < 3; ++a) O::massQ(w + a * O::KQ, h + a * O::KQ);
#pragma unroll
  for (int i = 0; i < O::K; ++i) y[i] = T(0);
  O::gradT(h, y);
}

// dst must be zero on entry except at constrained rows, which this kernel
// sets to src (ones on the constrained diagonal).
// dofs: [K][n_cells], -1 marks a constrained DoF (masked gather/scatter).
// geo:  [6][n_cells] metric G.
template <int P, typename T>
__global__ void __launch_bounds__(128) cg_cell_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
                                                      const T* __restrict__ geo, const T* __restrict__ src,
                                                      T* __restrict__ dst, int64_t n_constrained,
                                                      const int32_t* __restrict__ constrained) {
  using O = gen::Ops<P>;
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c < n_constrained) {
    const int32_t i = constrained[c];
    dst[i] = src[i];
  }
  if (c >= n_cells) return;
  int32_t idx[O::K];
  T u[O::K];
#pragma unroll
  for (int i = 0; i < O::K; ++i) {
    idx[i] = __ldg(dofs + i * n_cells + c);
    u[i] = idx[i] >= 0 ? __ldg(src + idx[i]) : T(0);
  }
  T G[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) G[k] = __ldg(geo + k * n_cells + c);
  T y[O::K];
  cg_local_apply<P>(G, u, y);
#pragma unroll
  for (int i = 0; i < O::K; ++i)
    if (idx[i] >= 0) atomicAdd(dst + idx[i], y[i]);
}

// Diagonal of the assembled operator: sum over cells of (A_K)_ii, constrained
// rows get 1 (ones on the diagonal).  dst zero on entry.
template <int P, typename T>
__global__ void __launch_bounds__(128) cg_diagonal_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
                                                          const T* __restrict__ geo, T* __restrict__ dst,
                                                          int64_t n_constrained,
                                                          const int32_t* __restrict__ constrained) {
  using O = gen::Ops<P>;
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c < n_constrained) dst[constrained[c]] = T(1);
  if (c >= n_cells) return;
  T G[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) G[k] = geo[k * n_cells + c];
  for (int i = 0; i < O::K; ++i) {
    const int32_t gi = dofs[i * n_cells + c];
    if (gi < 0) continue;
    T u[O::K], y[O::K];
#pragma unroll
    for (int j = 0; j < O::K; ++j) u[j] = j == i ? T(1) : T(0);
    cg_local_apply<P>(G, u, y);
    T yi = T(0);
#pragma unroll
    for (int j = 0; j < O::K; ++j)
      if (j == i) yi = y[j];
    atomicAdd(dst + gi, yi);
  }
}

}  // namespace sfem
