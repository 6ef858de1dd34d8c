// TF32 tensor-core form of the CG Laplace cell operator, for the FP32
// multigrid levels (sm_100a).
//
// The cell operator of cg_local_apply, y = sum_ab G_ab D_a^T MQ D_b u, is
// rewritten over the 6 independent metric entries c = (00,11,22,01,02,12):
//   y_i = sum_c G_c (S_c u)_i,   S_aa = D_a^T MQ D_a,
//   S_ab = D_a^T MQ D_b + D_b^T MQ D_a (a < b),
// so a tile of 128 cells is one dense product Z = U [128 x K] * B^T with
// B = [S_0; ...; S_5] ([6K x K], the same for every cell): a tcgen05.mma of
// kind::tf32 with U (the gathered cell DoFs, TF32-rounded) and B in shared
// memory and Z (FP32) in tensor memory.  The epilogue reads the thread's row
// of Z with tcgen05.ld, forms y_i = sum_c G_c Z[c K + i] in FP32 and scatters
// y with atomics, as cg_cell_kernel does.  TF32 keeps 10 mantissa bits, so
// the operator is accurate to ~1e-3 relative: meant for multigrid levels (a
// preconditioner), never for the outer FP64 operator.
//
// Persistent grid, 128 threads (one tile of 128 cells per iteration) per CTA,
// at most 512 / TMEM_COLS CTAs per SM.  The mbarrier wait is bounded; on a
// timeout the CTA sets *status, waits (bounded) for its MMAs and returns.
#pragma once
#include <cstdint>

#include "kernels_cg.cuh"
#include "tcgen05.cuh"

namespace sfem {

template <int P>
struct CGTcShape {
  static constexpr int K = gen::Ops<P>::K;
  static constexpr int KPAD = (K + 7) / 8 * 8;    // TF32 MMA K step is 8
  static constexpr int N = 6 * K;
  static constexpr int NPAD = (N + 15) / 16 * 16;  // M = 128 needs N % 16 == 0
  static constexpr int TMEM_COLS = NPAD <= 32 ? 32 : NPAD <= 64 ? 64 : NPAD <= 128 ? 128 : 256;
  static constexpr int OFF_B = 0;                          // B [NPAD x KPAD], K-major
  static constexpr int OFF_A = OFF_B + NPAD * KPAD * 4;    // A [128 x KPAD], K-major
  static constexpr int OFF_BAR = OFF_A + 128 * KPAD * 4;   // mbarrier + tensor-memory address
  static constexpr int SMEM_BYTES = OFF_BAR + 16;
};

namespace tc {
// byte offset of 32-bit element (row, k) of an R-row K-major operand
__device__ __forceinline__ int kmajor_off32(int row, int k, int R) {
  return (k >> 2) * (R * 16) + row * 16 + (k & 3) * 4;
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
}  // namespace tc

// dofs [K][n_cells] (-1: constrained), geo [6][n_cells], Bg [NPAD][KPAD]
// (TF32 values, zero padded), dst zero on entry except constrained rows
// (set to src here).
template <int P>
__global__ void __launch_bounds__(128) cg_cell_tc_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
                                                         const float* __restrict__ geo, const float* __restrict__ Bg,
                                                         const float* __restrict__ src, float* __restrict__ dst,
                                                         int64_t n_constrained,
                                                         const int32_t* __restrict__ constrained,
                                                         int* __restrict__ status) {
  using S = CGTcShape<P>;
  using namespace tc;
  constexpr int K = S::K, KPAD = S::KPAD, NPAD = S::NPAD;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + S::OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::OFF_BAR + 8);
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t bar = smem_u32(bar_p);

  for (int64_t i = blockIdx.x * int64_t(128) + t; i < n_constrained; i += int64_t(gridDim.x) * 128) {
    const int32_t g = constrained[i];
    dst[g] = src[g];
  }
  for (int e = t; e < NPAD * KPAD; e += 128)
    *reinterpret_cast<float*>(smem + S::OFF_B + kmajor_off32(e / KPAD, e % KPAD, NPAD)) = __ldg(Bg + e);
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(uint32_t(S::TMEM_COLS))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
  const uint32_t base = smem_u32(smem);
  const uint32_t idesc = idesc_tf32(128, NPAD);

  uint32_t phase = 0;
  bool failed = false;
  const int64_t n_tiles = (n_cells + 127) / 128;
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t c = tile * 128 + t;
    const bool live = c < n_cells;
    int32_t idx[K];
    float u[KPAD], G[6];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      idx[i] = live ? __ldg(dofs + i * n_cells + c) : -1;
      u[i] = idx[i] >= 0 ? __ldg(src + idx[i]) : 0.0f;
    }
#pragma unroll
    for (int i = K; i < KPAD; ++i) u[i] = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = live ? __ldg(geo + k * n_cells + c) : 0.0f;
    // row t of A: KPAD TF32 values in 16-byte K chunks
#pragma unroll
    for (int ch = 0; ch < KPAD / 4; ++ch) {
      const uint4 q = make_uint4(to_tf32(u[4 * ch]), to_tf32(u[4 * ch + 1]), to_tf32(u[4 * ch + 2]),
                                 to_tf32(u[4 * ch + 3]));
      *reinterpret_cast<uint4*>(smem + S::OFF_A + ch * (128 * 16) + t * 16) = q;
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    bool ok = true;
    if (t == 0) {
      tc_after_sync();
#pragma unroll
      for (int ks = 0; ks < KPAD / 8; ++ks) {
        const uint64_t da = smem_desc(base + S::OFF_A + ks * 2 * (128 * 16), 128 * 16, 128);
        const uint64_t db = smem_desc(base + S::OFF_B + ks * 2 * (NPAD * 16), NPAD * 16, 128);
        mma_tf32(tmem, da, db, idesc, ks > 0 ? 1u : 0u);
      }
      mma_commit(bar);
      ok = bar_wait(bar, phase);
      tc_before_sync();
    }
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    tc_after_sync();
    float y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) y[i] = 0.0f;
#pragma unroll
    for (int q = 0; q < NPAD / 32; ++q) {
      float v[32];
      tmem_ld32(trow + 32 * q, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int n = 32 * q + j;
        if (n < 6 * K) y[n % K] = fmaf(G[n / K], v[j], y[n % K]);
      }
    }
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (idx[i] >= 0) atomicAdd(dst + idx[i], y[i]);
    // the next tile's MMAs (issued after its block barrier) overwrite the accumulator
    tc_before_sync();
  }
  if (failed && t == 0) {
    atomicOr(status, 1);
    bar_wait(bar, phase ^ 1u);
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(S::TMEM_COLS))
                 : "memory");
}

}  // namespace sfem
