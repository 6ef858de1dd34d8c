// Tensor-core (tcgen05) inference of the learned smoother's MLP, sm_100a.
//
// A CTA runs GROUPS = 4 independent groups of 128 threads that share one
// copy of the weights; each group owns a tile of 128 cells (the MMA's M
// dimension), its own tensor-memory columns, mbarrier and named barrier.
// Thread t of a group builds row t of the BF16 input tile in shared memory (the
// normalised residual of cell t plus J/h, padded 29 -> 32).  The group's thread 0 issues
// the tcgen05.mma instructions of each layer (BF16 operands from shared
// memory, FP32 accumulators in tensor memory) and commits them to the
// group's mbarrier.  Every thread then reads its own accumulator row back with
// tcgen05.ld, adds the bias, applies GELU (tanh form, hardware tanh) and
// writes the BF16 activation row that feeds the next layer:
//
//   layer 1: [128 x 32] x W1^T [32 x 64]   (2 MMAs of K = 16)
//   layer 2: [128 x 64] x W2^T [64 x 64]   (4 MMAs)
//   layer 3: [128 x 64] x W3^T [64 x 32]   (4 MMAs; outputs 20..31 are padding)
//
// The weights stay in shared memory for the CTA's lifetime (persistent grid).
// Operand layout: K-major, no swizzle.  A core matrix is 8 rows x 16 bytes;
// for an R-row operand, element (row, k) lives at byte
//   (k / 8) * (R * 16) + row * 16 + (k % 8) * 2,
// so adjacent core matrices along K are R * 16 bytes apart (leading byte
// offset) and adjacent 8-row groups 128 bytes apart (stride byte offset).
//
// MODE 0: fused smoother, z += (s_K / h_K) * winv * MLP(r_K / s_K, J_K / h_K)
//         (the same map as mlp_smooth_kernel, computed with BF16 activations).
// MODE 1: dense forward O [n][20] = MLP(X [n][29]), used to test the kernel.
//
// Every mbarrier wait is bounded; on a timeout the CTA sets *status, waits
// (bounded) for its MMAs in flight, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "mlp.cuh"
#include "mlp_dims.hpp"
#include "tcgen05.cuh"

namespace sfem {
namespace tc {

constexpr int TILE = 128;       // cells per tile (MMA M)
constexpr int K1 = 32;          // 29 inputs padded to a multiple of 16
constexpr int N3 = 32;          // 20 outputs padded to a multiple of 16
constexpr int GROUPS = 4;       // independent 128-row tile pipelines per CTA
constexpr int THREADS = 128 * GROUPS;
constexpr int TMEM_COLS = 64 * GROUPS;  // one 64-column FP32 accumulator per group, reused by the layers
constexpr int XH_BYTES = TILE * 64 * 2;           // per group: input tile [128 x 32], then activations [128 x 64]
constexpr int OFF_XH = 0;                         // GROUPS x XH_BYTES
constexpr int OFF_W1 = OFF_XH + GROUPS * XH_BYTES; // W1 [64 x 32] (shared by the groups)
constexpr int OFF_W2 = OFF_W1 + 64 * K1 * 2;      // W2 [64 x 64]
constexpr int OFF_W3 = OFF_W2 + 64 * 64 * 2;      // W3 [32 x 64]
constexpr int OFF_B = OFF_W3 + N3 * 64 * 2;       // b1[64], b2[64], b3[32] as float
constexpr int OFF_BAR = OFF_B + 160 * 4;          // GROUPS mbarriers (8 B each) + tensor-memory address
constexpr int SMEM_BYTES = OFF_BAR + 8 * GROUPS + 16;

// named barrier of one 128-thread group (ids 1..GROUPS; 0 is __syncthreads)
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool group_sync_or(int id, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(id)
      : "memory");
  return r != 0;
}

// 8 values of one row as one 16-byte K chunk (bf16) of an R-row operand
__device__ __forceinline__ void store_chunk(unsigned char* base, int row, int c, int R, const float* v) {
  __align__(16) __nv_bfloat162 p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4*>(base + c * (R * 16) + row * 16) = *reinterpret_cast<const uint4*>(p);
}

// issue the K / 16 MMAs of one layer: A [128 x K] at a_off, B [N x K] at b_off
__device__ __forceinline__ void issue_layer(const unsigned char* smem, uint32_t tmem, int a_off, int b_off, int K,
                                            int N, uint32_t bar) {
  const uint32_t base = smem_u32(smem);
  const uint32_t idesc = idesc_bf16(TILE, N);
  for (int kk = 0; kk < K / 16; ++kk) {
    const uint64_t da = smem_desc(base + a_off + kk * 2 * (TILE * 16), TILE * 16, 128);
    const uint64_t db = smem_desc(base + b_off + kk * 2 * (N * 16), N * 16, 128);
    mma_bf16(tmem, da, db, idesc, kk > 0 ? 1u : 0u);
  }
  mma_commit(bar);
}

}  // namespace tc

// MODE 0 (smoother): dofs [20][n] (-1 at constrained DoFs), feat [n][10]
// (J/h and 1/h), winv [m], r in, z += correction.  MODE 1: X [n][29] in
// (passed as feat), O [n][20] out (passed as zout); dofs/winv/r unused.
template <int MODE, typename T>
__global__ void __launch_bounds__(tc::THREADS, 2) mlp_tc_kernel(int64_t n, const int32_t* __restrict__ dofs,
                                                               const float* __restrict__ feat,
                                                               const float* __restrict__ winv,
                                                               const __nv_bfloat16* __restrict__ wb,
                                                               const T* __restrict__ r, T* __restrict__ z,
                                                               float* __restrict__ zout, int* __restrict__ status) {
  using D = MLPDims;
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char smem[];
  float* sb = reinterpret_cast<float*>(smem + OFF_B);
  uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + OFF_BAR + 8 * GROUPS);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int grp = tid >> 7, t = tid & 127;  // group and row within the group's tile
  const int gbar = 1 + grp;                 // the group's named barrier
  const uint32_t bar = smem_u32(bar_p + grp);
  const int xh = OFF_XH + grp * XH_BYTES;   // the group's input / activation tile

  // weights -> shared memory (K-major, zero padding), biases as float
  for (int i = tid; i < 64 * K1; i += THREADS) {
    const int nn = i / K1, k = i % K1;
    const __nv_bfloat16 v = k < D::NIN ? wb[D::OFF_W1 + nn * D::NIN + k] : __float2bfloat16(0.0f);
    *reinterpret_cast<__nv_bfloat16*>(smem + OFF_W1 + kmajor_off(nn, k, 64)) = v;
  }
  for (int i = tid; i < 64 * 64; i += THREADS) {
    const int nn = i / 64, k = i % 64;
    *reinterpret_cast<__nv_bfloat16*>(smem + OFF_W2 + kmajor_off(nn, k, 64)) = wb[D::OFF_W2 + nn * 64 + k];
  }
  for (int i = tid; i < N3 * 64; i += THREADS) {
    const int nn = i / 64, k = i % 64;
    const __nv_bfloat16 v = nn < D::NOUT ? wb[D::OFF_W3 + nn * 64 + k] : __float2bfloat16(0.0f);
    *reinterpret_cast<__nv_bfloat16*>(smem + OFF_W3 + kmajor_off(nn, k, N3)) = v;
  }
  for (int i = tid; i < 160; i += THREADS)
    sb[i] = i < 64 ? __bfloat162float(wb[D::OFF_B1 + i])
            : i < 128 ? __bfloat162float(wb[D::OFF_B2 + i - 64])
            : i < 128 + D::NOUT ? __bfloat162float(wb[D::OFF_B3 + i - 128]) : 0.0f;
  if (tid < GROUPS) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar_p + tid)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(uint32_t(TMEM_COLS))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *tslot + 64 * grp;                              // the group's accumulator columns
  const uint32_t trow = tmem + (uint32_t((warp & 3) * 32) << 16);  // this warp's 32 accumulator lanes

  uint32_t phase = 0;
  bool failed = false;
  const int64_t n_tiles = (n + TILE - 1) / TILE;
  for (int64_t tile = int64_t(blockIdx.x) * GROUPS + grp; tile < n_tiles; tile += int64_t(gridDim.x) * GROUPS) {
    const int64_t c = tile * TILE + t;
    const bool live = c < n;
    if (MODE == 0) {
      // the next tile's DoF-index rows (20 x 512 B) and features (128 x 40 B)
      // into L2, one 128-byte line per thread, while this tile runs
      const int64_t c1 = (tile + int64_t(gridDim.x) * GROUPS) * TILE;
      if (c1 < n) {
        const void* line = nullptr;
        if (t < 4 * D::NR) {
          const int64_t e = c1 + 32 * (t & 3);
          if (e < n) line = dofs + (t >> 2) * n + e;
        } else if (t < 4 * D::NR + 40) {
          const int64_t e = c1 * 10 + 32 * (t - 4 * D::NR);
          if (e < n * 10) line = feat + e;
        }
        if (line) asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
      }
    }
    // ---- input row
    float x[K1];
    float scale = 0.0f;
#pragma unroll
    for (int i = 0; i < K1; ++i) x[i] = 0.0f;
    if (MODE == 0) {
      float s2 = 0.0f;
#pragma unroll
      for (int i = 0; i < D::NR; ++i) {
        const int32_t gi = live ? __ldg(dofs + i * n + c) : -1;
        x[i] = gi >= 0 ? float(r[gi]) : 0.0f;
        s2 += x[i] * x[i];
      }
      if (s2 > 0.0f) {
        const float s = sqrtf(s2), is = 1.0f / s;
#pragma unroll
        for (int i = 0; i < D::NR; ++i) x[i] *= is;
#pragma unroll
        for (int k = 0; k < D::NJ; ++k) x[D::NR + k] = __ldg(feat + c * 10 + k);
        scale = s * __ldg(feat + c * 10 + 9);
      } else {
#pragma unroll
        for (int i = 0; i < D::NR; ++i) x[i] = 0.0f;
      }
    } else if (live) {
#pragma unroll
      for (int i = 0; i < D::NIN; ++i) x[i] = __ldg(feat + c * D::NIN + i);
    }
#pragma unroll
    for (int ch = 0; ch < K1 / 8; ++ch) store_chunk(smem + xh, t, ch, TILE, x + 8 * ch);

    // ---- three layers (the activations overwrite the input tile once the
    // layer-1 MMAs that read it have completed)
    float v[32];
#pragma unroll 1
    for (int layer = 0; layer < 3; ++layer) {
      fence_async_smem();
      tc_before_sync();
      group_sync(gbar);
      if (t == 0) {
        tc_after_sync();
        if (layer == 0) issue_layer(smem, tmem, xh, OFF_W1, K1, 64, bar);
        else if (layer == 1) issue_layer(smem, tmem, xh, OFF_W2, 64, 64, bar);
        else issue_layer(smem, tmem, xh, OFF_W3, 64, N3, bar);
      }
      // one thread polls the group's mbarrier; the others wait at its barrier
      bool ok = true;
      if (t == 0) {
        ok = bar_wait(bar, phase);
        tc_before_sync();
      }
      phase ^= 1u;
      if (group_sync_or(gbar, !ok)) {
        failed = true;
        break;
      }
      tc_after_sync();
      if (layer < 2) {
        // 32 accumulator columns at a time: bias, GELU, BF16 row chunks for the next layer
        const float* bias = sb + 64 * layer;
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
          tmem_ld32(trow + 32 * half, v);
          const float4* b4 = reinterpret_cast<const float4*>(bias + 32 * half);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 bq = b4[q];
            v[4 * q] = gelu_fast(v[4 * q] + bq.x);
            v[4 * q + 1] = gelu_fast(v[4 * q + 1] + bq.y);
            v[4 * q + 2] = gelu_fast(v[4 * q + 2] + bq.z);
            v[4 * q + 3] = gelu_fast(v[4 * q + 3] + bq.w);
          }
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) store_chunk(smem + xh, t, 4 * half + ch, TILE, v + 8 * ch);
        }
      } else {
        tmem_ld32(trow, v);
      }
    }
    if (failed) break;
    // ---- output row (the DoF indices are read again: they are still in L2)
    {
      const float4* b4 = reinterpret_cast<const float4*>(sb + 128);
#pragma unroll
      for (int q = 0; q < D::NOUT / 4; ++q) {
        const float4 bq = b4[q];
        v[4 * q] += bq.x;
        v[4 * q + 1] += bq.y;
        v[4 * q + 2] += bq.z;
        v[4 * q + 3] += bq.w;
      }
    }
    if (MODE == 0) {
      if (scale != 0.0f) {
#pragma unroll
        for (int i = 0; i < D::NR; ++i) {
          const int32_t gi = __ldg(dofs + i * n + c);
          if (gi >= 0) atomicAdd(z + gi, T(scale * v[i] * __ldg(winv + gi)));
        }
      }
    } else if (live) {
#pragma unroll
      for (int j = 0; j < D::NOUT; ++j) zout[c * D::NOUT + j] = v[j];
    }
    // the next tile's layer-1 MMA overwrites the accumulator read above
    tc_before_sync();
  }
  if (failed && t == 0) {
    atomicOr(status, 1);
    bar_wait(bar, phase ^ 1u);  // the MMAs of the timed-out commit
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tslot), "r"(uint32_t(TMEM_COLS))
                 : "memory");
}

}  // namespace sfem
