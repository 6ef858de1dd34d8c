// Discontinuous Galerkin SIPG Laplace (+ optional mass) kernels (sm_100a).
//
// Operator restated (generic form DG/cells_batched/application.cc:1349-1490,
// Helmholtz application_helmholtz.cc:611-733,841-882):
//   a(u,v) = sum_K [ m (u,v)_K + (grad u, grad v)_K ]
//          + sum_F int_F ( sigma [u][v] - {d_n u}[v] - 1/2 [u] d_n v^- - 1/2 [u] d_n v^+ )
//   interior: [u] = u^- - u^+, {d_n u} = (d_n u^- + d_n u^+)/2, n = outward normal of K^-
//   boundary (weak homogeneous Dirichlet, u^+ = -u^-, d_n u^+ = d_n u^-):
//            test_by_value = 2 sigma u - d_n u, test by normal derivative = -u
//
// Element-centric, deterministic, no atomics: every cell writes its own DoF
// block once.  Two passes per vmult:
//   A (trace pass):       q_f = 2|F| d_n u on face f at the P_{p-1} face nodes,
//                         for all 4 faces of every cell (published in Q):
//                         dg_trace_tma_kernel (scalar problems, bulk copies),
//                         dg_trace_blk_kernel (scalar, unaligned vectors),
//                         dg_trace_kernel (3-component problems);
//   B (dg_apply_kernel):  cell term + the complete face terms of the cell's 4
//                         faces, reading the neighbour's face values from src and
//                         its published q from Q.
// For scalar problems B is launched as a programmatic dependent of A: its
// CTAs start while A's last blocks run, load what does not depend on A, and
// wait for A's grid before they read Q (pdl_trigger / pdl_wait).
// The reference instead sweeps faces in 576 (f_int,f_ext,o_int,o_ext) buckets
// and scatters into both sides (DG/cells_batched/application.cc:1738-2431);
// sorting every cell's vertices by global id removes the orientation part of
// that bucket key, and the element-centric form removes the scatter.
//
// Memory: one thread per cell, BS cells per CTA.  A CTA's cells are
// contiguous, so their DoF blocks are one contiguous range: it is copied into
// shared memory with coalesced loads, into rows padded to an odd number of
// words (conflict-free per-thread reads), and the results leave the same way.
// Q is [cell][4][NC][NFQ] rows for 3-component problems and block-major for
// scalar ones (see dg_trace_blk_kernel).  Neighbours inside the CTA are read
// from shared memory, the others from L2.  Each cell's geometry and neighbour
// ids are requested before its block is staged, so their latency overlaps
// the staging rather than the compute.
//
// Geometry per cell (structure of arrays, n_cells stride):
//   [0..5]  G = |det J| J^-1 J^-T           (00,11,22,01,02,12)
//   [6..9]  s_f = sigma_f |F_f|              (penalty times face area)
//   [10]    m |det J|                         (only when the mass term is on)
// The area-weighted face normals follow from G without storage:
//   J^-1 (2|F_f| n_f) = -G grad_xi(lambda_f),  grad_xi(lambda_0) = (-1,-1,-1),
//   grad_xi(lambda_i) = e_{i-1}.
#pragma once
#include <cstdint>

#include "kernels_cg.cuh"
#include "ref_kernels.cuh"
#include "tcgen05.cuh"

namespace sfem {

constexpr int kMaxBatch = 40;

template <typename T>
struct DGProblem {
  const T* geo;       // [n_geo][n_cells]
  const int32_t* nb;  // [4][n_cells]
  const int8_t* nbf;  // [4][n_cells]
  const T* src;       // [n_cells][NC][K]
  T* dst;
  T* Q;               // [n_cells][4][NC][NFQ], or block-major (see dg_trace_blk_kernel)
  int64_t n_cells;
};

// Several independent problems in one launch.  Work is split in CTA-sized
// blocks of cells that never straddle two problems; block_begin[] is the
// prefix sum of the blocks per problem.  Passed as a __grid_constant__ kernel
// parameter.
template <typename T>
struct DGBatch {
  int32_t n;
  int64_t block_begin[kMaxBatch + 1];
  DGProblem<T> p[kMaxBatch];
};

template <typename T>
__device__ __forceinline__ int find_problem(const DGBatch<T>& b, int64_t blk) {
  int lo = 0, hi = b.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.block_begin[mid] <= blk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// row stride (in elements) of a staged per-cell block of n values: odd, so
// that 32 threads reading their own rows hit 32 different banks
__host__ __device__ constexpr int padded(int n) { return (n % 2) ? n : n + 1; }

template <int P, int NC>
struct DGShape {
  using O = gen::Ops<P>;
  static constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  static constexpr int U = NC * K;           // values per cell
  static constexpr int QN = 4 * NC * NFQ;    // published traces per cell
  static constexpr int US = padded(U);       // staged row strides
  static constexpr int QS = padded(QN);
};

// asynchronous global -> shared copies of one element (LDGSTS)
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Programmatic dependent launch (sm_90 and later).  The trace pass lets the
// apply pass of the same vmult launch while it still runs; the apply pass
// does the work that does not read the traces (its geometry, neighbour ids,
// src rows, optionally the cell term) and then waits for the whole trace grid
// - its completion and the visibility of its stores - before it reads Q.  A
// kernel launched without the programmatic-serialization attribute returns
// from the wait at once.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// J^-1 (2|F_f| n_f) for local face f
template <typename T>
__device__ __forceinline__ void face_cf(const T (&G)[6], int f, T (&cf)[3]) {
  if (f == 0) {
    cf[0] = G[0] + G[3] + G[4];
    cf[1] = G[3] + G[1] + G[5];
    cf[2] = G[4] + G[5] + G[2];
  } else if (f == 1) {
    cf[0] = -G[0]; cf[1] = -G[3]; cf[2] = -G[4];
  } else if (f == 2) {
    cf[0] = -G[3]; cf[1] = -G[1]; cf[2] = -G[5];
  } else {
    cf[0] = -G[4]; cf[1] = -G[5]; cf[2] = -G[2];
  }
}

// coalesced copy of `rows` rows of N contiguous values into padded rows.  A
// full block from a 16-byte aligned source takes 16-byte loads, all issued
// before the first shared-memory store (N / (16 / sizeof(T)) per thread in
// flight); other blocks copy value by value.
template <int N, int S, int BS, typename T>
__device__ __forceinline__ void stage_in(T* __restrict__ sm, const T* __restrict__ g, int rows) {
  constexpr int V = 16 / int(sizeof(T));  // values per 16-byte load
  if constexpr (N % V == 0) {
    if (rows == BS && (reinterpret_cast<uintptr_t>(g) & 15u) == 0) {
      constexpr int PER = N / V;  // 16-byte loads per thread
      uint4 w[PER];
#pragma unroll
      for (int k = 0; k < PER; ++k) w[k] = __ldg(reinterpret_cast<const uint4*>(g) + k * BS + threadIdx.x);
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const T* v = reinterpret_cast<const T*>(&w[k]);
        const int e0 = (k * BS + threadIdx.x) * V;
#pragma unroll
        for (int q = 0; q < V; ++q) sm[((e0 + q) / N) * S + ((e0 + q) % N)] = v[q];
      }
      return;
    }
  }
  const int total = rows * N;
  for (int e = threadIdx.x; e < total; e += BS) sm[(e / N) * S + (e % N)] = __ldg(g + e);
}
// the reverse copy; full blocks to a 16-byte aligned destination take 16-byte stores
template <int N, int S, int BS, typename T>
__device__ __forceinline__ void stage_out(T* __restrict__ g, const T* __restrict__ sm, int rows) {
  constexpr int V = 16 / int(sizeof(T));
  if constexpr (N % V == 0) {
    if (rows == BS && (reinterpret_cast<uintptr_t>(g) & 15u) == 0) {
      constexpr int PER = N / V;
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int e0 = (k * BS + threadIdx.x) * V;
        uint4 w;
        T* v = reinterpret_cast<T*>(&w);
#pragma unroll
        for (int q = 0; q < V; ++q) v[q] = sm[((e0 + q) / N) * S + ((e0 + q) % N)];
        reinterpret_cast<uint4*>(g)[k * BS + threadIdx.x] = w;
      }
      return;
    }
  }
  const int total = rows * N;
  for (int e = threadIdx.x; e < total; e += BS) g[e] = sm[(e / N) * S + (e % N)];
}

// ---- block-major traces (scalar problems) ------------------------------------------------------
// The staged forms below publish traces as rows [cell][4][NC][NFQ].  For
// scalar problems the one-thread-per-cell forms store them block-major,
//   Q[b][k][l]: block b of kQB = 128 cells, trace k = f * NFQ + m, local cell l,
// so that the trace pass needs no shared memory (each thread reads its own
// row with 16-byte loads and every trace k is one coalesced store across the
// block), the apply pass copies its CTA's traces as QN contiguous runs, and a
// thread's own traces sit at stride BS in shared memory (bank-conflict free).
// A neighbour in another block is read at Q[nb / 128][k][nb % 128].
constexpr int kQB = 128;

// N values from p into v: 16-byte loads when p and the row allow it
template <int N, typename T>
__device__ __forceinline__ void load_row(const T* __restrict__ p, T (&v)[N]) {
  constexpr int V = 16 / int(sizeof(T));
  if constexpr (N % V == 0) {
    if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
#pragma unroll
      for (int k = 0; k < N / V; ++k) {
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(p) + k);
        const T* e = reinterpret_cast<const T*>(&w);
#pragma unroll
        for (int q = 0; q < V; ++q) v[k * V + q] = e[q];
      }
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = __ldg(p + i);
}

// Traces of the CTA's cells c0 .. c0 + nloc - 1 (BS cells inside one block of
// kQB, c0 a multiple of BS) into shared memory [QN][BS]; all loads in flight
// before the first store.
template <int QN, int BS, typename T>
__device__ __forceinline__ void stage_q_blk(T* __restrict__ sq, const T* __restrict__ Q, int64_t c0, int nloc) {
  static_assert(kQB % BS == 0, "a CTA's cells lie in one trace block");
  const T* base = Q + (c0 / kQB) * (QN * kQB) + (c0 % kQB);
  const int l = threadIdx.x;
  if (l < nloc) {
    T v[QN];
#pragma unroll
    for (int k = 0; k < QN; ++k) v[k] = __ldg(base + k * kQB + l);
#pragma unroll
    for (int k = 0; k < QN; ++k) sq[k * BS + l] = v[k];
  }
}

// trace k of `cell` in the block-major layout
template <int QN, typename T>
__device__ __forceinline__ const T* q_blk_ptr(const T* Q, int64_t cell, int k) {
  return Q + (cell / kQB) * (QN * kQB) + int64_t(k) * kQB + cell % kQB;
}

// Pass 1 for scalar problems, block-major: one thread per cell, no shared memory.
template <int P, typename T>
__global__ void __launch_bounds__(kQB) dg_trace_blk_kernel(const __grid_constant__ DGBatch<T> batch,
                                                           int64_t n_blocks) {
  using O = gen::Ops<P>;
  constexpr int K = O::K, KQ = O::KQ, NFQ = O::NFQ, QN = 4 * NFQ;
  pdl_trigger();
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t lb = blk - batch.block_begin[pi];
    const int64_t c = lb * kQB + threadIdx.x;
    if (c >= pr.n_cells) continue;
    const int64_t n = pr.n_cells;
    T G[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
    T u[K];
    load_row<K>(pr.src + c * K, u);
    T g[3 * KQ];
    O::grad(u, g);
    T* q = pr.Q + lb * (QN * kQB) + threadIdx.x;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      T cf[3];
      face_cf(G, f, cf);
#pragma unroll
      for (int m = 0; m < NFQ; ++m) {
        const int nq = O::fnq(f, m);
        q[(f * NFQ + m) * kQB] = cf[0] * g[nq] + cf[1] * g[KQ + nq] + cf[2] * g[2 * KQ + nq];
      }
    }
  }
}

// ---- the same pass fed by bulk copies ----------------------------------------------------------
// Persistent CTAs of kQB threads; a ring of NS stages, each holding one
// block's src rows ([kQB][K], dense) and its metric ([6][kQB]).  Thread 0
// issues cp.async.bulk copies (global -> shared, no multicast, completion on
// the stage's mbarrier) for block k + NS as soon as every thread is done with
// block k, so NS blocks are always in flight while one computes.  The host
// uses it when every copy starts 16-byte aligned and moves whole 16-byte units
// (src rows of the last block included; the metric copies are whole blocks,
// which the geometry's rows past the metric keep inside the allocation).
// Every mbarrier wait is bounded: on a timeout the CTA stops, waits (bounded)
// for the copies it issued and sets *status.
template <typename T, int K, int NS>
struct TraceTmaShape {
  static constexpr int U_BYTES = kQB * K * int(sizeof(T));
  static constexpr int G_BYTES = 6 * kQB * int(sizeof(T));
  static constexpr int STAGE = U_BYTES + G_BYTES;
  static constexpr int OFF_BAR = NS * STAGE;
  static constexpr int SMEM = OFF_BAR + 8 * NS;
  static_assert(U_BYTES % 16 == 0 && G_BYTES % 16 == 0, "bulk copies move 16-byte units");
};

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// global -> shared bulk copy without multicast, completion counted on `bar`
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int P, typename T, int NS>
__global__ void __launch_bounds__(kQB) dg_trace_tma_kernel(const __grid_constant__ DGBatch<T> batch, int64_t n_blocks,
                                                           int* __restrict__ status) {
  using O = gen::Ops<P>;
  constexpr int K = O::K, KQ = O::KQ, NFQ = O::NFQ, QN = 4 * NFQ;
  using S = TraceTmaShape<T, K, NS>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x;
  const uint32_t bar0 = tc::smem_u32(smem_raw + S::OFF_BAR);
  const int64_t first = blockIdx.x, stride = gridDim.x;
  const int64_t mine = first < n_blocks ? (n_blocks - 1 - first) / stride + 1 : 0;
  // thread 0: copies of this CTA's k-th block into stage k % NS
  auto issue = [&](int64_t k) {
    const int64_t blk = first + k * stride;
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * kQB;
    const int64_t rest = pr.n_cells - c0;
    const uint32_t ub = uint32_t(rest < kQB ? rest : int64_t(kQB)) * K * sizeof(T);
    const int s = int(k % NS);
    unsigned char* st = smem_raw + s * S::STAGE;
    const uint32_t bar = bar0 + 8 * s;
    mbar_expect_tx(bar, ub + S::G_BYTES);
    bulk_g2s(tc::smem_u32(st), pr.src + c0 * K, ub, bar);
#pragma unroll
    for (int i = 0; i < 6; ++i)
      bulk_g2s(tc::smem_u32(st + S::U_BYTES + i * kQB * sizeof(T)), pr.geo + i * pr.n_cells + c0,
               kQB * sizeof(T), bar);
  };
  if (t == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(bar0 + 8 * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int64_t k = 0; k < NS && k < mine; ++k) issue(k);
  }
  pdl_trigger();
  __syncthreads();
  int64_t done = 0;  // blocks whose stage wait completed
  bool ok = true;
  for (int64_t k = 0; k < mine; ++k) {
    const int s = int(k % NS);
    if (!tc::bar_wait(bar0 + 8 * s, uint32_t((k / NS) & 1))) ok = false;
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    done = k + 1;
    const int64_t blk = first + k * stride;
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t lb = blk - batch.block_begin[pi];
    if (lb * kQB + t < pr.n_cells) {
      const T* su = reinterpret_cast<const T*>(smem_raw + s * S::STAGE);
      const T* sg = reinterpret_cast<const T*>(smem_raw + s * S::STAGE + S::U_BYTES);
      T G[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) G[i] = sg[i * kQB + t];
      T u[K];
      constexpr int V = 16 / int(sizeof(T));
      if constexpr ((K * sizeof(T)) % 16 == 0) {
#pragma unroll
        for (int q = 0; q < K / V; ++q) {
          const uint4 w = reinterpret_cast<const uint4*>(su + t * K)[q];
          const T* e = reinterpret_cast<const T*>(&w);
#pragma unroll
          for (int r = 0; r < V; ++r) u[q * V + r] = e[r];
        }
      } else {
#pragma unroll
        for (int i = 0; i < K; ++i) u[i] = su[t * K + i];
      }
      T g[3 * KQ];
      O::grad(u, g);
      T* q = pr.Q + lb * (QN * kQB) + t;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        T cf[3];
        face_cf(G, f, cf);
#pragma unroll
        for (int m = 0; m < NFQ; ++m) {
          const int nq = O::fnq(f, m);
          q[(f * NFQ + m) * kQB] = cf[0] * g[nq] + cf[1] * g[KQ + nq] + cf[2] * g[2 * KQ + nq];
        }
      }
    }
    __syncthreads();  // stage s is free
    if (t == 0 && k + NS < mine) issue(k + NS);
  }
  if (!ok && t == 0) {
    // wait (bounded) for the copies still in flight, then report
    for (int64_t k = done; k < mine && k < done + NS; ++k) tc::bar_wait(bar0 + 8 * int(k % NS), uint32_t((k / NS) & 1));
    atomicExch(status, 1);
  }
}

// Publish q_f = 2|F_f| d_n u (own outward normal) at the P_{p-1} nodes of every face.
template <int P, int NC, int BS, typename T>
__global__ void __launch_bounds__(BS) dg_trace_kernel(const __grid_constant__ DGBatch<T> batch, int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S = DGShape<P, NC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [BS][US]
  T* sq = su + BS * S::US;                 // [BS][QS]
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * BS;
    const int nloc = int(pr.n_cells - c0 < BS ? pr.n_cells - c0 : int64_t(BS));
    __syncthreads();
    stage_in<S::U, S::US, BS>(su, pr.src + c0 * S::U, nloc);
    __syncthreads();
    const int t = threadIdx.x;
    if (t < nloc) {
      const int64_t c = c0 + t;
      const int64_t n = pr.n_cells;
      T G[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
#pragma unroll
      for (int comp = 0; comp < NC; ++comp) {
        T u[O::K];
#pragma unroll
        for (int i = 0; i < O::K; ++i) u[i] = su[t * S::US + comp * O::K + i];
        T g[3 * O::KQ];
        O::grad(u, g);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          T cf[3];
          face_cf(G, f, cf);
#pragma unroll
          for (int m = 0; m < O::NFQ; ++m) {
            const int nq = O::fnq(f, m);
            sq[t * S::QS + (f * NC + comp) * O::NFQ + m] =
                cf[0] * g[nq] + cf[1] * g[O::KQ + nq] + cf[2] * g[2 * O::KQ + nq];
          }
        }
      }
    }
    __syncthreads();
    stage_out<S::QN, S::QS, BS>(pr.Q + c0 * S::QN, sq, nloc);
  }
}

// Cell term of one component: h = MQ (G grad u) (the gradient test before
// the face terms) and y = m|J| MP u (or 0).  u: the component's K values.
template <int P, bool MASS, typename T>
__device__ __forceinline__ void dg_cell_term(const T* u, const T (&G)[6], T md, T (&h)[3 * gen::Ops<P>::KQ],
                                             T (&y)[gen::Ops<P>::K]) {
  using O = gen::Ops<P>;
  constexpr int K = O::K, KQ = O::KQ;
  T uu[K];
#pragma unroll
  for (int i = 0; i < K; ++i) uu[i] = u[i];
  T g[3 * KQ];
  O::grad(uu, g);
  T w[3 * KQ];
  apply_metric<KQ>(G, g, w);
#pragma unroll
  for (int a = 0; a < 3; ++a) O::massQ(w + a * KQ, h + a * KQ);
#pragma unroll
  for (int i = 0; i < K; ++i) y[i] = T(0);
  if (MASS) O::massP(uu, md, y);
}

// The four faces' terms of one component added to the cell term (h, y),
// then y += D^T h.  Arguments as for dg_cell_component.
template <int P, int NC, bool HAVE_NB, typename T, bool XS = false, bool BQ = false, int BSQ = 1>
__device__ __forceinline__ void dg_face_terms(const DGProblem<T>& pr, int64_t c0, int comp,
                                              const T* us, const T* qs, const T* su, const T* sq, int nloc,
                                              const T (&G)[6], const T (&sf)[4],
                                              const int32_t (&nb)[4], const int (&nbf)[4],
                                              T (&h)[3 * gen::Ops<P>::KQ], T (&y)[gen::Ops<P>::K],
                                              const T* xs = nullptr, const int (*slot)[4] = nullptr) {
  using O = gen::Ops<P>;
  using S = DGShape<P, NC>;
  constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  static_assert(!BQ || NC == 1, "block-major traces are for scalar problems");
  constexpr int QST = BQ ? BSQ : 1;  // stride of a cell's consecutive traces in shared memory
  const T* u = us + comp * K;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    T cf[3];
    face_cf(G, f, cf);
    const T* qm = qs + (BQ ? f * NFQ * BSQ : (f * NC + comp) * NFQ);
    T j[NF], avg[NFQ];
    if (nb[f] >= 0) {
      if (XS && (*slot)[f] >= 0) {
        const T* xn = xs + (*slot)[f] * (NF + NFQ);
#pragma unroll
        for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)] - xn[i];
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * (qm[m * QST] - xn[NF + m]);
      } else if (HAVE_NB) {
        const int64_t lc = int64_t(nb[f]) - c0;
        const T* un;
        const T* qn;
        int qns;  // stride of the neighbour's consecutive traces
        if (lc >= 0 && lc < nloc) {
          un = su + lc * S::US + comp * K;
          qn = BQ ? sq + nbf[f] * NFQ * BSQ + lc : sq + lc * S::QS + (nbf[f] * NC + comp) * NFQ;
          qns = QST;
        } else {
          un = pr.src + (int64_t(nb[f]) * NC + comp) * K;
          qn = BQ ? q_blk_ptr<4 * NFQ>(pr.Q, nb[f], nbf[f] * NFQ)
                  : pr.Q + ((int64_t(nb[f]) * 4 + nbf[f]) * NC + comp) * NFQ;
          qns = BQ ? kQB : 1;
        }
#pragma unroll
        for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)] - un[O::fn_runtime(nbf[f], i)];
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * (qm[m * QST] - qn[m * qns]);
      } else {
#pragma unroll
        for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)];
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * qm[m * QST];
      }
    } else {
      // boundary face: u+ = -u-, d_n u+ = d_n u-
#pragma unroll
      for (int i = 0; i < NF; ++i) j[i] = T(2) * u[O::fn(f, i)];
#pragma unroll
      for (int m = 0; m < NFQ; ++m) avg[m] = T(0.5) * qm[m * QST];
    }
    // value test: sigma|F| MFPP j - MFPQ avg
    T t[NF];
    O::facePP(j, t);
#pragma unroll
    for (int i = 0; i < NF; ++i) t[i] *= sf[f];
#pragma unroll
    for (int m = 0; m < NFQ; ++m) avg[m] = -avg[m];
    O::facePQ(avg, t);
#pragma unroll
    for (int i = 0; i < NF; ++i) y[O::fn(f, i)] += t[i];
    // gradient test: h_a += -1/4 cf_a MFQP j
    T r[NFQ];
    O::faceQP(j, r);
#pragma unroll
    for (int m = 0; m < NFQ; ++m) {
      const int nq = O::fnq(f, m);
      const T rm = T(-0.25) * r[m];
      h[nq] += cf[0] * rm;
      h[KQ + nq] += cf[1] * rm;
      h[2 * KQ + nq] += cf[2] * rm;
    }
  }
  O::gradT(h, y);
}

// Own-cell terms plus face terms for one component.  u and qm come from the
// staged rows of this cell (`us`, `qs`); HAVE_NB reads the neighbour traces
// (from shared memory when the neighbour is in this CTA, rows su/sq),
// otherwise they are zero (diagonal).
// XS: `xs` points at this cell's staged cross-block neighbour data, one row
// of XROW values per face slot (slot[f] < 0: not staged): the neighbour's
// face values already in this cell's face-node order, then its traces.
// BQ (scalar): the traces are block-major, staged as [QN][BSQ] (qs = sq + this
// cell's local index), and a neighbour in another block is read from pr.Q in
// the block-major layout.
template <int P, int NC, bool MASS, bool HAVE_NB, typename T, bool XS = false, bool BQ = false, int BSQ = 1>
__device__ __forceinline__ void dg_cell_component(const DGProblem<T>& pr, int64_t c0, int comp,
                                                  const T* us, const T* qs, const T* su, const T* sq, int nloc,
                                                  const T (&G)[6], const T (&sf)[4], T md,
                                                  const int32_t (&nb)[4], const int (&nbf)[4],
                                                  T (&y)[gen::Ops<P>::K], const T* xs = nullptr,
                                                  const int (*slot)[4] = nullptr) {
  T h[3 * gen::Ops<P>::KQ];
  dg_cell_term<P, MASS>(us + comp * gen::Ops<P>::K, G, md, h, y);
  dg_face_terms<P, NC, HAVE_NB, T, XS, BQ, BSQ>(pr, c0, comp, us, qs, su, sq, nloc, G, sf, nb, nbf, h, y, xs,
                                                slot);
}

template <typename T>
struct CellData {
  T G[6], sf[4], md;
  int32_t nb[4];
  int nbf[4];
};

template <bool MASS, typename T>
__device__ __forceinline__ void load_cell(const DGProblem<T>& pr, int64_t c, CellData<T>& d) {
  const int64_t n = pr.n_cells;
#pragma unroll
  for (int k = 0; k < 6; ++k) d.G[k] = __ldg(pr.geo + k * n + c);
#pragma unroll
  for (int f = 0; f < 4; ++f) d.sf[f] = __ldg(pr.geo + (6 + f) * n + c);
  d.md = MASS ? __ldg(pr.geo + 10 * n + c) : T(0);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    d.nb[f] = __ldg(pr.nb + f * n + c);
    d.nbf[f] = __ldg(pr.nbf + f * n + c);
  }
}

// MINB: minimum resident CTAs per SM (register cap).  ALIAS (NC == 1): the
// results stay in registers until every thread of the CTA is done reading the
// staged src rows, then reuse those rows for the coalesced write-out, so the
// CTA needs no separate result rows (less shared memory, more CTAs per SM).
// BQ (NC == 1): block-major traces (dg_trace_blk_kernel), staged as [QN][BS].
// PDLM: launched as a programmatic dependent of the trace pass.  1: the
// geometry and the src rows are loaded before the wait for the trace grid;
// 2 (scalar, block-major traces): the cell term is computed before the wait
// as well, and the traces are staged after it.
template <int P, int NC, bool MASS, int BS, typename T, int MINB = (BS == 64 ? 6 : 1), bool ALIAS = false,
          bool BQ = false, int PDLM = 0>
__global__ void __launch_bounds__(BS, MINB) dg_apply_kernel(const __grid_constant__ DGBatch<T> batch,
                                                            int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S = DGShape<P, NC>;
  static_assert(!ALIAS || NC == 1, "result aliasing holds one component in registers");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [BS][US]  src rows
  T* sq = su + BS * S::US;                 // [BS][QS]  published traces
  T* sy = ALIAS ? su : sq + BS * S::QS;    // [BS][US]  results
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * BS;
    const int nloc = int(pr.n_cells - c0 < BS ? pr.n_cells - c0 : int64_t(BS));
    const int t = threadIdx.x;
    // the cell's geometry and neighbours are requested before the block's
    // rows, so their latency overlaps the staging instead of the compute
    CellData<T> d;
    if (t < nloc) load_cell<MASS>(pr, c0 + t, d);
    __syncthreads();
    stage_in<S::U, S::US, BS>(su, pr.src + c0 * S::U, nloc);
    if constexpr (PDLM == 2) {
      static_assert(NC == 1 && BQ, "cell term before the wait: scalar problems, block-major traces");
      __syncthreads();  // src rows staged
      T h[3 * O::KQ], y[O::K];
      if (t < nloc) dg_cell_term<P, MASS>(su + t * S::US, d.G, d.md, h, y);
      pdl_wait();
      stage_q_blk<S::QN, BS>(sq, pr.Q, c0, nloc);
      __syncthreads();
      if (t < nloc)
        dg_face_terms<P, NC, true, T, false, BQ, BS>(pr, c0, 0, su + t * S::US, sq + t, su, sq, nloc, d.G, d.sf, d.nb,
                                                     d.nbf, h, y);
      if (ALIAS) __syncthreads();  // every thread is done with the staged src rows
      if (t < nloc) {
#pragma unroll
        for (int i = 0; i < O::K; ++i) sy[t * S::US + i] = y[i];
      }
      __syncthreads();
      stage_out<S::U, S::US, BS>(pr.dst + c0 * S::U, sy, nloc);
      continue;
    }
    if constexpr (PDLM == 1) pdl_wait();
    if constexpr (BQ) stage_q_blk<S::QN, BS>(sq, pr.Q, c0, nloc);
    else stage_in<S::QN, S::QS, BS>(sq, pr.Q + c0 * S::QN, nloc);
    __syncthreads();
    const T* qs = BQ ? sq + t : sq + t * S::QS;  // this cell's traces
    if (ALIAS) {
      T y[O::K];
      if (t < nloc) {
        dg_cell_component<P, NC, MASS, true, T, false, BQ, BS>(pr, c0, 0, su + t * S::US, qs, su, sq, nloc, d.G,
                                                                d.sf, d.md, d.nb, d.nbf, y);
      }
      __syncthreads();  // every thread is done with the staged src rows
      if (t < nloc) {
#pragma unroll
        for (int i = 0; i < O::K; ++i) sy[t * S::US + i] = y[i];
      }
    } else if (t < nloc) {
#pragma unroll 1
      for (int comp = 0; comp < NC; ++comp) {
        T y[O::K];
        dg_cell_component<P, NC, MASS, true, T, false, BQ, BS>(pr, c0, comp, su + t * S::US, qs, su, sq, nloc,
                                                                d.G, d.sf, d.md, d.nb, d.nbf, y);
#pragma unroll
        for (int i = 0; i < O::K; ++i) sy[t * S::US + comp * O::K + i] = y[i];
      }
    }
    __syncthreads();
    stage_out<S::U, S::US, BS>(pr.dst + c0 * S::U, sy, nloc);
  }
}

// Apply with the cross-block neighbour data prefetched (scalar problems).
// Faces whose neighbour lies outside the CTA's BS cells read the neighbour's
// face values and published traces from global memory, one dependent load
// chain per face, which a thread-per-cell kernel at 2 warps per scheduler
// cannot hide.  Here, while the CTA stages its own rows, every thread also
// issues cp.async copies of its cross-block faces' neighbour data (face
// values permuted into its own face-node order, then the traces) into
// compact shared-memory rows: a CTA-wide prefix sum over the cross faces
// gives the rows, up to XCAP of them; faces past XCAP (rare) keep the direct
// global reads.  All copies are in flight together and land before the
// compute starts.
template <int P, int BS, int XCAP, typename T>
__global__ void __launch_bounds__(BS, 1) dg_apply_xp_kernel(const __grid_constant__ DGBatch<T> batch,
                                                            int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S = DGShape<P, 1>;
  constexpr int XROW = O::NF + O::NFQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [BS][US]  src rows
  T* sq = su + BS * S::US;                 // [BS][QS]  published traces
  T* sy = sq + BS * S::QS;                 // [BS][US]  results
  T* sx = sy + BS * S::US;                 // [XCAP][XROW] cross-block neighbour rows
  __shared__ int warp_tot[BS / 32];
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * BS;
    const int nloc = int(pr.n_cells - c0 < BS ? pr.n_cells - c0 : int64_t(BS));
    const int t = threadIdx.x;
    const int64_t n = pr.n_cells;
    CellData<T> d;
    int cross = 0;  // bit f: face f has its neighbour outside this CTA
    if (t < nloc) {
      load_cell<false>(pr, c0 + t, d);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int64_t lc = int64_t(d.nb[f]) - c0;
        if (d.nb[f] >= 0 && (lc < 0 || lc >= nloc)) cross |= 1 << f;
      }
    }
    // CTA-wide exclusive prefix sum of the cross-face counts
    const int cnt = __popc(cross);
    const int lane = t & 31, warp = t >> 5;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    __syncthreads();  // the previous block is done with every shared buffer
    if (lane == 31) warp_tot[warp] = incl;
    stage_in<S::U, S::US, BS>(su, pr.src + c0 * S::U, nloc);
    stage_in<S::QN, S::QS, BS>(sq, pr.Q + c0 * S::QN, nloc);
    __syncthreads();
    int base = incl - cnt;
    for (int w = 0; w < warp; ++w) base += warp_tot[w];
    int slot[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      slot[f] = -1;
      if (cross >> f & 1) {
        if (base < XCAP) {
          slot[f] = base;
          T* dst = sx + base * XROW;
          const int nf = d.nbf[f];
          const T* un = pr.src + int64_t(d.nb[f]) * O::K;
          const T* qn = pr.Q + (int64_t(d.nb[f]) * 4 + nf) * O::NFQ;
#pragma unroll
          for (int i = 0; i < O::NF; ++i) cp_async_elem(dst + i, un + O::fn_runtime(nf, i));
#pragma unroll
          for (int m = 0; m < O::NFQ; ++m) cp_async_elem(dst + O::NF + m, qn + m);
        }
        ++base;
      }
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (t < nloc) {
      T y[O::K];
      dg_cell_component<P, 1, false, true, T, true>(pr, c0, 0, su + t * S::US, sq + t * S::QS, su, sq, nloc, d.G,
                                                   d.sf, d.md, d.nb, d.nbf, y, sx, &slot);
#pragma unroll
      for (int i = 0; i < O::K; ++i) sy[t * S::US + i] = y[i];
    }
    __syncthreads();
    stage_out<S::U, S::US, BS>(pr.dst + c0 * S::U, sy, nloc);
  }
}

// Weak homogeneous Dirichlet terms of a CG operator on boundary face F of
// each listed cell (the CG levels of the reference's DG multigrid,
// DG/cells_batched/application_phc.cc:1799-1832): test by value 2 sigma u -
// d_n u, test by normal derivative -u, with sf = sigma |F|.  One thread per
// boundary face; the cell's DoFs come from the CG table [K][n_cells] and the
// results are added atomically.  diag: the diagonal of those terms instead
// (each local basis function applied on its own, x unused).
template <int P, int F, typename T>
__global__ void __launch_bounds__(128) cg_weak_boundary_kernel(int64_t n, const int32_t* __restrict__ cells,
                                                               const T* __restrict__ sfs, int64_t n_cells,
                                                               const int32_t* __restrict__ dofs,
                                                               const T* __restrict__ geo, const T* __restrict__ x,
                                                               T* __restrict__ dst, bool diag) {
  using O = gen::Ops<P>;
  constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  const int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (e >= n) return;
  const int64_t c = cells[e];
  const T sf = sfs[e];
  T G[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) G[k] = geo[k * n_cells + c];
  T cf[3];
  face_cf(G, F, cf);
  int32_t dof[K];
#pragma unroll
  for (int i = 0; i < K; ++i) dof[i] = dofs[int64_t(i) * n_cells + c];
  // y = B u for the local boundary operator B of face F
  auto apply = [&](const T (&u)[K], T (&y)[K]) {
    T g[3 * KQ];
    O::grad(u, g);
    T j[NF], avg[NFQ];
#pragma unroll
    for (int i = 0; i < NF; ++i) j[i] = T(2) * u[O::fn(F, i)];
#pragma unroll
    for (int m = 0; m < NFQ; ++m) {
      const int nq = O::fnq(F, m);
      avg[m] = T(-0.5) * (cf[0] * g[nq] + cf[1] * g[KQ + nq] + cf[2] * g[2 * KQ + nq]);
    }
    T t[NF];
    O::facePP(j, t);
#pragma unroll
    for (int i = 0; i < NF; ++i) t[i] *= sf;
    O::facePQ(avg, t);
#pragma unroll
    for (int i = 0; i < K; ++i) y[i] = T(0);
#pragma unroll
    for (int i = 0; i < NF; ++i) y[O::fn(F, i)] += t[i];
    T r[NFQ];
    O::faceQP(j, r);
    T h[3 * KQ];
#pragma unroll
    for (int q = 0; q < 3 * KQ; ++q) h[q] = T(0);
#pragma unroll
    for (int m = 0; m < NFQ; ++m) {
      const int nq = O::fnq(F, m);
      const T rm = T(-0.25) * r[m];
      h[nq] += cf[0] * rm;
      h[KQ + nq] += cf[1] * rm;
      h[2 * KQ + nq] += cf[2] * rm;
    }
    O::gradT(h, y);
  };
  if (!diag) {
    T u[K], y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) u[i] = dof[i] >= 0 ? x[dof[i]] : T(0);
    apply(u, y);
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (dof[i] >= 0) atomicAdd(dst + dof[i], y[i]);
  } else {
    for (int i = 0; i < K; ++i) {
      T u[K], y[K];
#pragma unroll
      for (int k = 0; k < K; ++k) u[k] = k == i ? T(1) : T(0);
      apply(u, y);
      T yi = T(0);
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k == i) yi = y[k];
      if (dof[i] >= 0) atomicAdd(dst + dof[i], yi);
    }
  }
}

// Diagonal of the DG operator: (A)_ii = own-cell terms applied to e_i, with
// the own traces of e_i formed on the fly and the neighbour traces zero.
// Set-up only: plain per-thread code, 128 cells per block of work.
template <int P, int NC, bool MASS, typename T>
__global__ void __launch_bounds__(128) dg_diagonal_kernel(const __grid_constant__ DGBatch<T> batch,
                                                          int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S1 = DGShape<P, 1>;
  constexpr int BS = 128;
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c = (blk - batch.block_begin[pi]) * BS + threadIdx.x;
    if (c >= pr.n_cells) continue;
    CellData<T> d;
    load_cell<MASS>(pr, c, d);
    for (int i = 0; i < O::K; ++i) {
      T e[S1::US];
      T q[S1::QS];
#pragma unroll
      for (int j = 0; j < O::K; ++j) e[j] = j == i ? T(1) : T(0);
      {
        T g[3 * O::KQ];
        T uu[O::K];
#pragma unroll
        for (int j = 0; j < O::K; ++j) uu[j] = e[j];
        O::grad(uu, g);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          T cf[3];
          face_cf(d.G, f, cf);
#pragma unroll
          for (int m = 0; m < O::NFQ; ++m) {
            const int nq = O::fnq(f, m);
            q[f * O::NFQ + m] = cf[0] * g[nq] + cf[1] * g[O::KQ + nq] + cf[2] * g[2 * O::KQ + nq];
          }
        }
      }
      T y[O::K];
      // the diagonal is the same for every component
      dg_cell_component<P, 1, MASS, false, T>(pr, 0, 0, e, q, nullptr, nullptr, 0, d.G, d.sf, d.md, d.nb, d.nbf,
                                              y);
      T yi = T(0);
#pragma unroll
      for (int j = 0; j < O::K; ++j)
        if (j == i) yi = y[j];
      for (int comp = 0; comp < NC; ++comp) pr.dst[(c * NC + comp) * O::K + i] = yi;
    }
  }
}

}  // namespace sfem
