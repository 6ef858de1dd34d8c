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

// L1 cache policies of the cube kernels' loads: the tables every cube reads
// (tet maps, reduce schedules) are kept (evict_last); the per-cube metric and
// DoF codes are read once and not allocated in L1, so they do not push the
// tables out.  The asm is volatile and every call sits under an explicit
// bounds test: a non-volatile asm load counts as side-effect free, and the
// compiler may then execute it ahead of the test that guards its address.
__device__ __forceinline__ uint4 ld_keep(const uint4* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::evict_last.v4.u32 {%0, %1, %2, %3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p));
  return v;
}
__device__ __forceinline__ uint32_t ld_keep(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::evict_last.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) {
  int32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

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
template <int P, typename T, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) cg_cell_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
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

// Vector Laplacian with NC interleaved components (global index NC g + comp
// of node DoF g), the optimized kernels of the reference's components-batched
// CG operator (CG/components_batched/application.cc:1025-1216: the scalar
// metric applied to every component).  One thread per cell: the node table
// is read once and the cell's NC K values gathered, every component runs the
// fused local operator, results added atomically.  constrained lists vector
// indices (rows dst = src).
template <int P, typename T, int NC>
__global__ void __launch_bounds__(128) cg_cell_vec_kernel(int64_t n_cells, const int32_t* __restrict__ dofs,
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
#pragma unroll
  for (int i = 0; i < O::K; ++i) idx[i] = __ldg(dofs + i * n_cells + c);
  T G[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) G[k] = __ldg(geo + k * n_cells + c);
#pragma unroll 1
  for (int comp = 0; comp < NC; ++comp) {
    T u[O::K], y[O::K];
#pragma unroll
    for (int i = 0; i < O::K; ++i) u[i] = idx[i] >= 0 ? __ldg(src + int64_t(NC) * idx[i] + comp) : T(0);
    cg_local_apply<P>(G, u, y);
#pragma unroll
    for (int i = 0; i < O::K; ++i)
      if (idx[i] >= 0) atomicAdd(dst + int64_t(NC) * idx[i] + comp, y[i]);
  }
}

// the scalar diagonal d (node DoFs) repeated on every component
template <typename T, int NC>
__global__ void expand_components(int64_t n, const T* __restrict__ d, T* __restrict__ out) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int comp = 0; comp < NC; ++comp) out[NC * i + comp] = d[i];
}

// Dense element matrices of the cell operator, mats[c][r][i] = (A_K)_ri, one
// thread per cell applying the local operator to each unit vector (set-up of
// the assembled-matrix comparison; constraints are applied at assembly).
template <int P, typename T>
__global__ void __launch_bounds__(128) cg_element_matrix_kernel(int64_t n_cells, const T* __restrict__ geo,
                                                                T* __restrict__ mats) {
  using O = gen::Ops<P>;
  constexpr int K = O::K;
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n_cells) return;
  T G[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) G[k] = __ldg(geo + k * n_cells + c);
  T* m = mats + c * K * K;
  for (int i = 0; i < K; ++i) {
    T u[K], y[K];
#pragma unroll
    for (int j = 0; j < K; ++j) u[j] = j == i ? T(1) : T(0);
    cg_local_apply<P>(G, u, y);
#pragma unroll
    for (int r = 0; r < K; ++r) m[r * K + i] = y[r];
  }
}

// y = A x for a CSR matrix, LANES threads per row (partial sums reduced with
// warp shuffles); the assembled-matrix baseline of the matrix-free vmult.
template <typename T, int LANES>
__global__ void __launch_bounds__(256) csr_spmv_kernel(int64_t n_rows, const int64_t* __restrict__ row_ptr,
                                                       const int32_t* __restrict__ col, const T* __restrict__ val,
                                                       const T* __restrict__ x, T* __restrict__ y) {
  const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t row = t / LANES;
  const int lane = int(t % LANES);
  T s = T(0);
  if (row < n_rows) {
    const int64_t b = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
    for (int64_t k = b + lane; k < e; k += LANES) s += __ldg(val + k) * __ldg(x + __ldg(col + k));
  }
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LANES);
  if (row < n_rows && lane == 0) y[row] = s;
}

// Macro-element form for Kuhn meshes: one thread per hex, i.e. the 6
// consecutive tets that subdivide it.  The 6 tets share most of their DoFs
// (P1: 8 distinct of 24, P2: 27 of 60, P3: 64 of 120), so the thread gathers
// each distinct DoF once into its shared-memory row, applies the 6 cell
// operators from there, accumulates their results in a second row, and
// issues one global atomic per distinct DoF: 2-3x fewer L2 atomics and
// gathers than cg_cell_kernel, and no cooperation between threads.
// hdofs: [H][n_hex] global DoF of hex-local DoF k (-1: constrained);
// hgeo:  [6 * 6][n_hex] metric value k of tet q at row 6 q + k (coalesced per hex);
// map: hex-local index of local DoF i of tet q (the same for every hex: it
// only depends on the Kuhn subdivision and the vertex ordering).
// Dynamic shared memory: 2 * BS * HexRow<H>::S values.
struct HexMap {
  int8_t m[6][20];
};

template <int H>
struct HexRow {
  static constexpr int S = (H % 2) ? H : H + 1;  // odd stride: per-thread rows in distinct banks
};

template <int P, typename T, int H, int BS>
__global__ void __launch_bounds__(BS) cg_hex_kernel(int64_t n_hex, const int32_t* __restrict__ hdofs,
                                                    const __grid_constant__ HexMap map, const T* __restrict__ hgeo,
                                                    const T* __restrict__ src, T* __restrict__ dst,
                                                    int64_t n_constrained, const int32_t* __restrict__ constrained) {
  using O = gen::Ops<P>;
  constexpr int S = HexRow<H>::S;
  extern __shared__ __align__(16) unsigned char smem_hex[];
  const int t = threadIdx.x;
  T* u = reinterpret_cast<T*>(smem_hex) + t * S;
  T* y = reinterpret_cast<T*>(smem_hex) + (BS + t) * S;
  for (int64_t i = blockIdx.x * int64_t(BS) + t; i < n_constrained; i += int64_t(gridDim.x) * BS) {
    const int32_t g = constrained[i];
    dst[g] = src[g];
  }
  const int64_t h = blockIdx.x * int64_t(BS) + t;
  if (h >= n_hex) return;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const int32_t g = __ldg(hdofs + k * n_hex + h);
    u[k] = g >= 0 ? __ldg(src + g) : T(0);
    y[k] = T(0);
  }
  // P1/P2: all 6 tets unrolled, so the 36 metric loads are issued together;
  // P3 (register-heavy) keeps a rolled loop
#pragma unroll(P <= 2 ? 6 : 1)
  for (int q = 0; q < 6; ++q) {
    T G[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(hgeo + (6 * q + k) * n_hex + h);
    T ut[O::K], yt[O::K];
#pragma unroll
    for (int i = 0; i < O::K; ++i) ut[i] = u[map.m[q][i]];
    cg_local_apply<P>(G, ut, yt);
#pragma unroll
    for (int i = 0; i < O::K; ++i) y[map.m[q][i]] += yt[i];
  }
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const int32_t g = __ldg(hdofs + k * n_hex + h);
    if (g >= 0) atomicAdd(dst + g, y[k]);
  }
}

// DoF reduction of one cube (cube kernels): thread t sums the contributions of
// its reduce slots n = 384 r + t from the per-tet result rows yr, in the order
// of its cslot8 steps, and writes each DoF once (store for cube-interior DoFs,
// atomic on the cube surface).  bd: the cube's row of bdof.
template <typename T, int NB>
__device__ __forceinline__ void cube_reduce(int t, const int32_t* __restrict__ bd, const uint32_t* __restrict__ ritem,
                                            const int16_t* __restrict__ cslot8, const T* yr, T* __restrict__ dst) {
  constexpr int NJ = (NB + 383) / 384;
#pragma unroll 1
  for (int r = 0; r < NJ; ++r) {
    const int n = 384 * r + t;
    if (n >= NB) break;
    const int32_t code = __ldg(bd + n);
    if (code < 0) continue;
    const uint32_t item = __ldg(ritem + n);
    const uint4* grp = reinterpret_cast<const uint4*>(cslot8) + (item >> 8);
    const int steps = int(item & 0xFFu);  // per lane; the same for every lane in schedule 1
    T sum = T(0);
    for (int q = 0; 8 * q < steps; ++q) {
      const uint4 w = __ldg(grp + 32 * q);
      const uint32_t wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int h = 0; h < 8; ++h)
        if (8 * q + h < steps) sum += yr[(h & 1) ? (wv[h >> 1] >> 16) : (wv[h >> 1] & 0xFFFFu)];
    }
    const int32_t g = code & 0x3FFFFFFF;
    if (code & 0x40000000) dst[g] = sum;
    else atomicAdd(dst + g, sum);
  }
}

// The same reduction for cg_cube_pipe_kernel: the cube's DoF codes of this
// thread come from registers; reduce items from registers when `items` is
// given (else loaded, kept in L1), schedules loaded with L1::evict_last.
template <typename T, int NB>
__device__ __forceinline__ void cube_reduce_regs(int t, const int32_t (&codes)[(NB + 383) / 384],
                                                 const uint32_t* __restrict__ ritem,
                                                 const uint32_t (*items)[(NB + 383) / 384],
                                                 const int16_t* __restrict__ cslot8, const T* yr,
                                                 T* __restrict__ dst) {
  constexpr int NJ = (NB + 383) / 384;
#pragma unroll
  for (int r = 0; r < NJ; ++r) {
    const int n = 384 * r + t;
    if (n >= NB) break;
    const int32_t code = codes[r];
    if (code < 0) continue;
    const uint32_t item = items ? (*items)[r] : ld_keep(ritem + n);
    const uint4* grp = reinterpret_cast<const uint4*>(cslot8) + (item >> 8);
    const int steps = int(item & 0xFFu);  // per lane; the same for every lane in schedule 1
    T sum = T(0);
    for (int q = 0; 8 * q < steps; ++q) {
      const uint4 w = ld_keep(grp + 32 * q);
      const uint32_t wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int h = 0; h < 8; ++h)
        if (8 * q + h < steps) sum += yr[(h & 1) ? (wv[h >> 1] >> 16) : (wv[h >> 1] & 0xFFFFu)];
    }
    const int32_t g = code & 0x3FFFFFFF;
    if (code & 0x40000000) dst[g] = sum;
    else atomicAdd(dst + g, sum);
  }
}

// Cube-block form for Kuhn meshes whose hexes come in Morton order: 64
// consecutive hexes (384 tets) form a 4 x 4 x 4 cube, and every cube has the
// same local structure, so one set of small tables serves all cubes.  One
// thread per tet:
//   1. the cube's distinct DoFs (P1 125, P2 729, P3 2197) are gathered once
//      into shared memory;
//   2. each thread applies its tet's operator and writes its K results to its
//      shared-memory row;
//   3. each distinct DoF sums its contributions and is written back once: a
//      plain store when only this cube touches it, else one atomic.
// About 6 atomics per hex for P2 (27 with cg_hex_kernel, 60 with
// cg_cell_kernel) and one gather per distinct DoF.  The kernel is bound by L1 /
// shared-memory transactions, so the tables are packed for 16-byte loads and
// laid out [row][thread] (a warp reads one contiguous 512-byte row):
// cube DoFs are numbered by reduce slot n = 384 r + t (thread t gathers and
// reduces slot n in round r; a warp-round holds 32 DoFs with similar
// contribution counts);
// tmapv  [KV/8][384] x 8: slot of tet t's local DoF i (KV = K rounded up to 8)
// bdof   [n_blocks][NB] global DoF | (interior << 30), -1 at constrained DoFs
// ritem  [NB]: steps of the warp-round | (first cslot8 entry << 8)
// cslot8 per warp-round [groups][32] x 8: the row slot (t * KP + i) each
//        lane reads at each step, or a zero slot 384 KP + z; the steps are
//        scheduled so that no two lanes of a step read the same bank
// Persistent and software-pipelined: a CTA walks cubes b0, b0 + G, b0 + 2G,
// ...  While it computes cube k, the gather of cube k+1
// is already in flight as cp.async copies into the second of two shared
// buffers, the DoF codes of cube k+2 and the tet metric of cube k+1 are being
// loaded into registers, and the atomics of cube k-1 drain.  Buffer reuse is
// ordered by the two block barriers of every iteration (a buffer is refilled
// only after the barrier that follows its last read).
// The tet metric of the next cube arrives one of two ways (cube_metric_smem):
// loaded into registers one cube ahead, or streamed into shared memory with
// 16-byte cp.async copies issued after the apply of the current cube (its six
// [384] rows are contiguous in geo), landing during the reduction.  The second
// frees the prefetch registers but takes 6 x 384 values of shared memory, which
// the L1 cache loses: measured on B200 it is faster for P3 FP32 (130 against
// 136 us on 64^3) and P1 FP64 (155 against 177 us on 128^3), slower for P2
// FP64 (421 against 396 us) and P3 FP64, and no faster for P2 FP32.
// Shared memory: ((6 x 384) + 2 NB + 384 KP + NZ) values, NZ = 16 zero slots
// for 8-byte values (bank pairs), 32 for 4-byte values.
template <int P, typename T>
__host__ __device__ constexpr bool cube_metric_smem() {
  return (P == 3 && sizeof(T) == 4) || (P == 1 && sizeof(T) == 8);
}
// Resident CTAs per SM of the cube kernel (its register cap).  P2 FP64 runs
// two CTAs with up to 85 registers: with three (56 registers) the DoF codes
// of the current cube spill (measured on B200, 128^3: 356 us with two CTAs,
// 404 us with three).
template <int P, typename T>
__host__ __device__ constexpr int cube_min_ctas() {
  return (P == 2 && sizeof(T) == 8) ? 2 : P <= 2 ? 3 : (sizeof(T) == 4 ? 2 : 1);
}

template <int P, typename T, int NB, int KP>
__global__ void __launch_bounds__(384, cube_min_ctas<P, T>())
    cg_cube_pipe_kernel(int64_t n_blocks, const int16_t* __restrict__ tmapv, const int32_t* __restrict__ bdof,
                        const uint32_t* __restrict__ ritem, const int16_t* __restrict__ cslot8,
                        const T* __restrict__ geo, const T* __restrict__ src, T* __restrict__ dst, int64_t n_constrained, const int32_t* __restrict__ constrained) {
  using O = gen::Ops<P>;
  constexpr int K = O::K;
  constexpr int KV = (K + 7) / 8 * 8;
  constexpr int NJ = (NB + 383) / 384;  // cube DoFs gathered per thread
  constexpr bool GS = cube_metric_smem<P, T>();
  extern __shared__ __align__(16) unsigned char smem_cube[];
  T* sg = reinterpret_cast<T*>(smem_cube);  // GS: [6][384] metric of the cube
  T* ubuf = sg + (GS ? 6 * 384 : 0);        // [2][NB]
  T* yr = ubuf + 2 * NB;                    // [384][KP], then the zero slots
  const int t = threadIdx.x;
  if (t < (sizeof(T) == 8 ? 16 : 32)) yr[384 * KP + t] = T(0);
  const int64_t stride = gridDim.x;
  const int64_t n_cells = n_blocks * 384;
  for (int64_t i = blockIdx.x * int64_t(384) + t; i < n_constrained; i += stride * 384) {
    const int32_t g = constrained[i];
    dst[g] = src[g];
  }
  auto load_codes = [&](int64_t b, int32_t (&code)[NJ]) {
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      const int j = t + 384 * q;
      code[q] = -1;
      if (b < n_blocks && j < NB) code[q] = ld_stream(bdof + b * NB + j);
    }
  };
  // cp.async of this thread's share of cube DoF values into buffer `buf`
  auto issue_gather = [&](const int32_t (&code)[NJ], int buf, bool valid) {
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      const int j = t + 384 * q;
      if (!valid || j >= NB) continue;
      T* d = ubuf + buf * NB + j;
      if (code[q] < 0) {
        *d = T(0);
      } else {
        const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(d));
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(src + (code[q] & 0x3FFFFFFF)),
                     "n"(sizeof(T))
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // GS: cp.async (16 bytes, L2 only) of cube bq's metric rows into sg
  auto issue_geo = [&](int64_t bq) {
    constexpr int CH = 384 * int(sizeof(T)) / 16;  // 16-byte chunks per row
    if (GS && bq < n_blocks)
      for (int e = t; e < 6 * CH; e += 384) {
        const int k = e / CH, ch = e % CH;
        const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(sg + k * 384 + ch * (16 / sizeof(T))));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa),
                     "l"(geo + k * n_cells + bq * 384 + ch * (16 / int(sizeof(T))))
                     : "memory");
      }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // !GS: the metric of cube bq into registers
  auto load_geo = [&](int64_t bq, T (&G)[6]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      G[k] = T(0);
      if (bq < n_blocks) G[k] = ld_stream(geo + k * n_cells + bq * 384 + t);
    }
  };

  int64_t b = blockIdx.x;
  int32_t code_cur[NJ], code_nxt[NJ], code_nn[NJ];  // DoF codes of cubes k, k+1, k+2
  // HOIST: the tet map and reduce items are the same for every cube; with two
  // or fewer CTAs per SM there are registers to hold them across the loop
  constexpr bool HOIST = cube_min_ctas<P, T>() <= 2;
  uint4 tmv[KV / 8];
  uint32_t items[NJ];
  if (HOIST) {
#pragma unroll
    for (int q = 0; q < KV / 8; ++q) tmv[q] = ld_keep(reinterpret_cast<const uint4*>(tmapv) + t + 384 * q);
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      items[q] = 0u;
      if (384 * q + t < NB) items[q] = ld_keep(ritem + 384 * q + t);
    }
  }
  T Gc[6], Gn[6];
  load_codes(b, code_cur);
  issue_gather(code_cur, 0, b < n_blocks);
  if (GS) issue_geo(b);
  else load_geo(b, Gc);
  load_codes(b + stride, code_nxt);
  for (int k = 0; b < n_blocks; ++k, b += stride) {
    const int buf = k & 1;
    const bool more = b + stride < n_blocks;
    // gather of the next cube, codes of the one after (and !GS: metric of the next)
    issue_gather(code_nxt, buf ^ 1, more);
    load_codes(b + 2 * stride, code_nn);
    if (!GS) load_geo(b + stride, Gn);
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // this cube's gather (GS: and metric)
    __syncthreads();
    {
      T G[6];
#pragma unroll
      for (int k6 = 0; k6 < 6; ++k6) G[k6] = GS ? sg[k6 * 384 + t] : Gc[k6];
      const T* ub = ubuf + buf * NB;
      const uint4* tm = reinterpret_cast<const uint4*>(tmapv) + t;  // unused when HOIST
      int ti[KV];
#pragma unroll
      for (int q = 0; q < KV / 8; ++q) {
        const uint4 w = HOIST ? tmv[q] : ld_keep(tm + 384 * q);
        const uint32_t wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          ti[8 * q + 2 * h] = int(wv[h] & 0xFFFFu);
          ti[8 * q + 2 * h + 1] = int(wv[h] >> 16);
        }
      }
      T ut[K], yt[K];
#pragma unroll
      for (int i = 0; i < K; ++i) ut[i] = ub[ti[i]];
      cg_local_apply<P>(G, ut, yt);
#pragma unroll
      for (int i = 0; i < K; ++i) yr[t * KP + i] = yt[i];
    }
    __syncthreads();
    if (GS) issue_geo(b + stride);  // every thread has read this cube's metric
    cube_reduce_regs<T, NB>(t, code_cur, ritem, HOIST ? &items : nullptr, cslot8, yr, dst);
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
      code_cur[q] = code_nxt[q];
      code_nxt[q] = code_nn[q];
    }
    if (!GS) {
#pragma unroll
      for (int k6 = 0; k6 < 6; ++k6) Gc[k6] = Gn[k6];
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
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
