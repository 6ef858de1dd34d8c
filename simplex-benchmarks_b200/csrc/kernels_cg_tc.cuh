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

// Cube-block form of the TF32 tensor-core operator (FP32 multigrid levels):
// the cube kernel's structure (cg_cube_pipe_kernel: one CTA per 4 x 4 x 4-hex
// cube, one gather per distinct DoF, bank-scheduled DoF reduction) with the
// per-tet contraction on the tensor cores instead of CUDA-core FMAs.  The
// cube's 384 tets are three M = 128 tiles of one A operand [384 x KPAD]
// (TF32, built in shared memory from the gathered DoF values); B holds the
// reference matrices S_c and the metric components are split into PASSES
// passes of CPP components, so that the accumulators of the three tiles fit
// NP columns each: Z_tile = A_tile B_pass^T in tensor memory, then every
// thread forms y_i += sum_c G_c Z[c K + i] from its row (tcgen05.ld).  At most
// 512 / TMEM_COLS CTAs per SM: the host pads the dynamic shared memory so that
// no more fit.  Every mbarrier wait is bounded; on a timeout the CTA sets
// *status, waits (bounded) for its MMAs and returns.
template <int P>
struct CubeTcShape {
  static constexpr int K = gen::Ops<P>::K;
  static constexpr int KPAD = (K + 7) / 8 * 8;          // TF32 MMA K step is 8
  static constexpr int CPP = P == 3 ? 3 : 6;             // metric components per pass
  static constexpr int PASSES = 6 / CPP;
  static constexpr int NP = (CPP * K + 15) / 16 * 16;    // MMA N of a pass
  static constexpr int NBROWS = PASSES * NP;             // rows of B
  static constexpr int TMEM_COLS = 3 * NP <= 128 ? 128 : 256;
  static constexpr int MAX_CTAS = 512 / TMEM_COLS;       // per SM
  static constexpr int OFF_B = 0;                        // B [NBROWS x KPAD], K-major
  static constexpr int OFF_A = OFF_B + NBROWS * KPAD * 4;  // A [384 x KPAD], K-major
  static constexpr int OFF_BAR = OFF_A + 384 * KPAD * 4;   // mbarrier + tensor-memory address
  static constexpr int OFF_U = OFF_BAR + 16;               // [2][NB] DoF values, then yr
  static constexpr size_t smem_bytes(int NB, int KP) { return OFF_U + (2 * size_t(NB) + 384 * size_t(KP) + 32) * 4; }
};

template <int P, int NB, int KP>
__global__ void __launch_bounds__(384, CubeTcShape<P>::MAX_CTAS > 2 ? 2 : CubeTcShape<P>::MAX_CTAS)
    cg_cube_tc_kernel(int64_t n_blocks, const int16_t* __restrict__ tmapv, const int32_t* __restrict__ bdof,
                      const uint32_t* __restrict__ ritem, const int16_t* __restrict__ cslot8,
                      const float* __restrict__ geo, const float* __restrict__ Bg, const float* __restrict__ src,
                      float* __restrict__ dst, int64_t n_constrained, const int32_t* __restrict__ constrained,
                      int* __restrict__ status) {
  using S = CubeTcShape<P>;
  using namespace tc;
  constexpr int K = S::K, KPAD = S::KPAD, NP = S::NP, CPP = S::CPP;
  constexpr int KV = (K + 7) / 8 * 8;
  constexpr int NJ = (NB + 383) / 384;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + S::OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::OFF_BAR + 8);
  float* ubuf = reinterpret_cast<float*>(smem + S::OFF_U);  // [2][NB]
  float* yr = ubuf + 2 * NB;                                // [384][KP], then 32 zero slots
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t bar = smem_u32(bar_p);
  if (t < 32) yr[384 * KP + t] = 0.0f;
  const int64_t stride = gridDim.x;
  const int64_t n_cells = n_blocks * 384;
  for (int64_t i = blockIdx.x * int64_t(384) + t; i < n_constrained; i += stride * 384) {
    const int32_t g = constrained[i];
    dst[g] = src[g];
  }
  for (int e = t; e < S::NBROWS * KPAD; e += 384)
    *reinterpret_cast<float*>(smem + S::OFF_B + kmajor_off32(e / KPAD, e % KPAD, S::NBROWS)) = __ldg(Bg + e);
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
  // warp w owns rows 32 (w % 4) .. of tile w / 4, whose accumulator starts at column NP (w / 4)
  const uint32_t trow = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t((warp >> 2) * NP);
  const uint32_t base = smem_u32(smem);
  const uint32_t idesc = idesc_tf32(128, NP);

  auto load_codes = [&](int64_t b, int32_t (&code)[NJ]) {
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      const int j = t + 384 * q;
      code[q] = (b < n_blocks && j < NB) ? __ldg(bdof + b * NB + j) : -1;
    }
  };
  auto issue_gather = [&](const int32_t (&code)[NJ], int buf, bool valid) {
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      const int j = t + 384 * q;
      if (!valid || j >= NB) continue;
      float* d = ubuf + buf * NB + j;
      if (code[q] < 0) {
        *d = 0.0f;
      } else {
        const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(d));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(src + (code[q] & 0x3FFFFFFF))
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto load_geo = [&](int64_t bq, float (&G)[6]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = bq < n_blocks ? __ldg(geo + k * n_cells + bq * 384 + t) : 0.0f;
  };

  uint32_t phase = 0;
  bool failed = false;
  int64_t b = blockIdx.x;
  int32_t code_cur[NJ], code_nxt[NJ];
  float G[6], Gn[6];
  load_codes(b, code_cur);
  issue_gather(code_cur, 0, b < n_blocks);
  load_codes(b + stride, code_nxt);
  load_geo(b, G);
  for (int k = 0; b < n_blocks; ++k, b += stride) {
    const int buf = k & 1;
    issue_gather(code_nxt, buf ^ 1, b + stride < n_blocks);
#pragma unroll
    for (int q = 0; q < NJ; ++q) code_cur[q] = code_nxt[q];
    load_codes(b + 2 * stride, code_nxt);
    load_geo(b + stride, Gn);
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // this cube's gather
    __syncthreads();
    // row t of A: the tet's DoF values as TF32, in 16-byte K chunks
    {
      const float* ub = ubuf + buf * NB;
      const uint4* tm = reinterpret_cast<const uint4*>(tmapv) + t;
      float u[KV];
#pragma unroll
      for (int q = 0; q < KV / 8; ++q) {
        const uint4 w = __ldg(tm + 384 * q);
        const uint32_t wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          u[8 * q + 2 * h] = 8 * q + 2 * h < K ? ub[wv[h] & 0xFFFFu] : 0.0f;
          u[8 * q + 2 * h + 1] = 8 * q + 2 * h + 1 < K ? ub[wv[h] >> 16] : 0.0f;
        }
      }
#pragma unroll
      for (int ch = 0; ch < KPAD / 4; ++ch)
        *reinterpret_cast<uint4*>(smem + S::OFF_A + ch * (384 * 16) + t * 16) =
            make_uint4(to_tf32(u[4 * ch]), to_tf32(u[4 * ch + 1]), to_tf32(u[4 * ch + 2]), to_tf32(u[4 * ch + 3]));
    }
    float y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) y[i] = 0.0f;
#pragma unroll
    for (int p = 0; p < S::PASSES; ++p) {
      // A is written (pass 0) / every thread has read the previous pass's accumulators
      fence_async_smem();
      tc_before_sync();
      __syncthreads();
      bool ok = true;
      if (t == 0) {
        tc_after_sync();
#pragma unroll
        for (int tl = 0; tl < 3; ++tl)
#pragma unroll
          for (int ks = 0; ks < KPAD / 8; ++ks) {
            const uint64_t da = smem_desc(base + S::OFF_A + tl * (128 * 16) + ks * 2 * (384 * 16), 384 * 16, 128);
            const uint64_t db =
                smem_desc(base + S::OFF_B + p * (NP * 16) + ks * 2 * (S::NBROWS * 16), S::NBROWS * 16, 128);
            mma_tf32(tmem + uint32_t(tl * NP), da, db, idesc, ks > 0 ? 1u : 0u);
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
#pragma unroll
      for (int q = 0; q < NP / 32; ++q) {
        float v[32];
        tmem_ld32(trow + 32 * q, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = 32 * q + j;
          if (n < CPP * K) y[n % K] = fmaf(G[p * CPP + n / K], v[j], y[n % K]);
        }
      }
    }
    if (failed) break;
#pragma unroll
    for (int i = 0; i < K; ++i) yr[t * KP + i] = y[i];
    tc_before_sync();  // the next cube's MMAs overwrite the accumulators after the next barriers
    __syncthreads();
    cube_reduce<float, NB>(t, bdof + b * NB, ritem, cslot8, yr, dst);
#pragma unroll
    for (int k6 = 0; k6 < 6; ++k6) G[k6] = Gn[k6];
  }
  if (failed && t == 0) {
    atomicOr(status, 1);
    bar_wait(bar, phase ^ 1u);  // the MMAs of the timed-out commit
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(S::TMEM_COLS))
                 : "memory");
}

}  // namespace sfem
