// Warp-role DG kernels (sm_100a): 32 cells per CTA, 4 warps, lane = cell.
//
// Same operator and two-pass structure as kernels_dg.cuh (trace, then apply),
// but the work of one cell is split over the 4 warps of the CTA so that no
// thread carries a whole cell's state (the thread-per-cell form needs ~110
// doubles per thread and runs at 2 warps per scheduler, latency bound on its
// neighbour loads):
//   apply, per CTA:
//     0  warp f issues cp.async copies of the neighbour data of face f of its
//        32 cells (u^+ at the face nodes, published q^+) into shared memory;
//        they land while the CTA stages its own rows and contracts gradients;
//   per component:
//     A  warps a = 0..2 contract the reference gradient component a (g_a = D_a u);
//        warp f then computes the face-f terms: jump/average, value test
//        t_f = s_f MFPP j - MFPQ avg and r_f = MFQP j;
//     B  warps a = 0..2: h_a = MQ (G g)_a - 1/4 sum_f cf_f[a] r_f;
//     C  warp w produces output nodes [w*PART, (w+1)*PART): y_i = (D^T h)_i +
//        sum over faces through i of t_f (+ m|J| (MP u)_i).
//   trace: warps a = 0..2 contract g_a, then warp f publishes q_f.
// Every choice of face, component and node is warp-uniform, so the generated
// straight-line code runs without divergence.  Shared memory rows indexed by
// lane are either [value][cell] (stride 32, consecutive lanes) or
// [cell][value] with an odd row stride; both are bank-conflict free.  Rows
// used by a contraction are first copied to registers, so every shared value
// is loaded once per thread.
#pragma once
#include <cstdint>

#include "kernels_dg.cuh"

namespace sfem {

template <int P, int NC>
struct DG3 {
  using O = gen::Ops<P>;
  using S = DGShape<P, NC>;
  static constexpr int CELLS = 32, THREADS = 128;
  static constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  static constexpr int US = S::US, QS = S::QS, U = S::U, QN = S::QN;
  static constexpr int PART = (K + 3) / 4;
  static constexpr int NV = NF + NFQ;  // neighbour values per face and component
  // shared memory layout (elements)
  static constexpr int OFF_U = 0;                          // [CELLS][US]
  static constexpr int OFF_Q = OFF_U + CELLS * US;         // [CELLS][QS]
  static constexpr int OFF_T = OFF_Q + CELLS * QS;         // [4*NF][CELLS]
  static constexpr int OFF_R = OFF_T + 4 * NF * CELLS;     // [4*NFQ][CELLS]
  static constexpr int OFF_G = OFF_R + 4 * NFQ * CELLS;    // [3*KQ][CELLS]
  static constexpr int OFF_Y = OFF_G + 3 * KQ * CELLS;     // [CELLS][US]
  static constexpr int OFF_N = OFF_Y + CELLS * US;         // [4][NC][NV][CELLS]
  static constexpr int APPLY_ELEMS = OFF_N + 4 * NC * NV * CELLS;
  static constexpr int TRACE_ELEMS = CELLS * US + 3 * KQ * CELLS + CELLS * QS;
};

// cf_f[a] = (J^-1 2|F_f| n_f)_a from the symmetric metric G
template <typename T>
__device__ __forceinline__ T cf_comp(const T (&G)[6], int f, int a) {
  const T g[3][3] = {{G[0], G[3], G[4]}, {G[3], G[1], G[5]}, {G[4], G[5], G[2]}};
  if (f == 0) return g[a][0] + g[a][1] + g[a][2];
  return -g[a][f - 1];
}

// neighbour data of face F (all components) -> shared memory, by the face-F warp
template <int P, int NC, int F, typename T>
__device__ __forceinline__ void dg3_prefetch(const DGProblem<T>& pr, int l, T* sm, int32_t nb, int nbf) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  if (nb < 0) return;
  const T* un = pr.src + int64_t(nb) * D::U;
  const T* qn = pr.Q + (int64_t(nb) * 4 + nbf) * NC * D::NFQ;
#pragma unroll
  for (int comp = 0; comp < NC; ++comp) {
    T* dst = sm + D::OFF_N + ((F * NC + comp) * D::NV) * D::CELLS + l;
#pragma unroll
    for (int i = 0; i < D::NF; ++i) cp_async_elem(dst + i * D::CELLS, un + comp * D::K + O::fn_runtime(nbf, i));
#pragma unroll
    for (int m = 0; m < D::NFQ; ++m) cp_async_elem(dst + (D::NF + m) * D::CELLS, qn + comp * D::NFQ + m);
  }
}

template <int P, int NC, int F, typename T>
__device__ __forceinline__ void dg3_face(int l, int comp, T* sm, T sf, int32_t nb) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  const T* u = sm + D::OFF_U + l * D::US + comp * D::K;
  const T* qm = sm + D::OFF_Q + l * D::QS + (F * NC + comp) * D::NFQ;
  T j[D::NF], avg[D::NFQ];
  if (nb >= 0) {
    const T* nv = sm + D::OFF_N + ((F * NC + comp) * D::NV) * D::CELLS + l;
#pragma unroll
    for (int i = 0; i < D::NF; ++i) j[i] = u[O::fn(F, i)] - nv[i * D::CELLS];
#pragma unroll
    for (int m = 0; m < D::NFQ; ++m) avg[m] = T(-0.25) * (qm[m] - nv[(D::NF + m) * D::CELLS]);
  } else {
#pragma unroll
    for (int i = 0; i < D::NF; ++i) j[i] = T(2) * u[O::fn(F, i)];
#pragma unroll
    for (int m = 0; m < D::NFQ; ++m) avg[m] = T(-0.5) * qm[m];
  }
  T t[D::NF];
  O::facePP(j, t);
#pragma unroll
  for (int i = 0; i < D::NF; ++i) t[i] *= sf;
  O::facePQ(avg, t);
#pragma unroll
  for (int i = 0; i < D::NF; ++i) sm[D::OFF_T + (F * D::NF + i) * D::CELLS + l] = t[i];
  T r[D::NFQ];
  O::faceQP(j, r);
#pragma unroll
  for (int m = 0; m < D::NFQ; ++m) sm[D::OFF_R + (F * D::NFQ + m) * D::CELLS + l] = r[m];
}

// g_A = D_A u into sG rows (u read once into registers)
template <int P, int NC, int A, typename T>
__device__ __forceinline__ void dg3_grad(int l, int comp, T* sm) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  const T* u = sm + D::OFF_U + l * D::US + comp * D::K;
  T uu[D::K];
#pragma unroll
  for (int i = 0; i < D::K; ++i) uu[i] = u[i];
  T g[D::KQ];
#pragma unroll
  for (int m = 0; m < D::KQ; ++m) g[m] = O::grad_row(A * D::KQ + m, uu, 1);
#pragma unroll
  for (int m = 0; m < D::KQ; ++m) sm[D::OFF_G + (A * D::KQ + m) * D::CELLS + l] = g[m];
}

// h_A = MQ (G g)_A - 1/4 sum_f cf_f[A] r_f  (returned in registers)
template <int P, int NC, int A, typename T>
__device__ __forceinline__ void dg3_h(int l, const T* sm, const T (&G)[6], T (&h)[DG3<P, NC>::KQ]) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  constexpr int KQ = D::KQ;
  const T ga = G[A == 0 ? 0 : A == 1 ? 3 : 4], gb = G[A == 0 ? 3 : A == 1 ? 1 : 5],
          gc = G[A == 0 ? 4 : A == 1 ? 5 : 2];
  T w[KQ];
  const T* g = sm + D::OFF_G + l;
#pragma unroll
  for (int m = 0; m < KQ; ++m)
    w[m] = ga * g[(0 * KQ + m) * D::CELLS] + gb * g[(1 * KQ + m) * D::CELLS] + gc * g[(2 * KQ + m) * D::CELLS];
#pragma unroll
  for (int m = 0; m < KQ; ++m) h[m] = O::massQ_row(m, w);
  const T* r = sm + D::OFF_R + l;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const T c = T(-0.25) * cf_comp(G, f, A);
#pragma unroll
    for (int m = 0; m < KQ; ++m) {
      const int pos = O::faceq_pos(f, m);
      if (pos >= 0) h[m] += c * r[(f * D::NFQ + pos) * D::CELLS];
    }
  }
}

// outputs i in [W*PART, (W+1)*PART) of component comp
template <int P, int NC, bool MASS, int W, typename T>
__device__ __forceinline__ void dg3_out(int l, int comp, T* sm, T md) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  T hh[3 * D::KQ];
#pragma unroll
  for (int r = 0; r < 3 * D::KQ; ++r) hh[r] = sm[D::OFF_G + r * D::CELLS + l];
  T uu[D::K];
  if (MASS) {
#pragma unroll
    for (int i = 0; i < D::K; ++i) uu[i] = sm[D::OFF_U + l * D::US + comp * D::K + i];
  }
  const T* t = sm + D::OFF_T + l;
#pragma unroll
  for (int k = 0; k < D::PART; ++k) {
    const int i = W * D::PART + k;
    if (i < D::K) {
      T y = O::gradT_row(i, hh, 1);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int pos = O::face_pos(f, i);
        if (pos >= 0) y += t[(f * D::NF + pos) * D::CELLS];
      }
      if (MASS) y += md * O::massP_row(i, uu, 1);
      sm[D::OFF_Y + l * D::US + comp * D::K + i] = y;
    }
  }
}

template <int P, int NC, bool MASS, typename T>
__global__ void __launch_bounds__(128, 4) dg3_apply_kernel(const __grid_constant__ DGBatch<T> batch,
                                                           int64_t n_blocks) {
  using D = DG3<P, NC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * D::CELLS;
    const int nloc = int(pr.n_cells - c0 < D::CELLS ? pr.n_cells - c0 : int64_t(D::CELLS));
    const bool valid = l < nloc;
    const int64_t c = c0 + (valid ? l : 0);
    const int64_t n = pr.n_cells;
    __syncthreads();  // previous block's shared memory reads are done
    const int32_t nb = valid ? __ldg(pr.nb + warp * n + c) : -1;
    const int nbf = __ldg(pr.nbf + warp * n + c);
    switch (warp) {
      case 0: dg3_prefetch<P, NC, 0>(pr, l, sm, nb, nbf); break;
      case 1: dg3_prefetch<P, NC, 1>(pr, l, sm, nb, nbf); break;
      case 2: dg3_prefetch<P, NC, 2>(pr, l, sm, nb, nbf); break;
      default: dg3_prefetch<P, NC, 3>(pr, l, sm, nb, nbf); break;
    }
    cp_async_commit();
    stage_in<D::U, D::US, D::THREADS>(sm + D::OFF_U, pr.src + c0 * D::U, nloc);
    stage_in<D::QN, D::QS, D::THREADS>(sm + D::OFF_Q, pr.Q + c0 * D::QN, nloc);
    T G[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
    const T sf = __ldg(pr.geo + (6 + warp) * n + c);
    const T md = MASS ? __ldg(pr.geo + 10 * n + c) : T(0);
    __syncthreads();
#pragma unroll 1
    for (int comp = 0; comp < NC; ++comp) {
      if (valid) {
        switch (warp) {
          case 0: dg3_grad<P, NC, 0>(l, comp, sm); break;
          case 1: dg3_grad<P, NC, 1>(l, comp, sm); break;
          case 2: dg3_grad<P, NC, 2>(l, comp, sm); break;
          default: break;
        }
      }
      cp_async_wait_all();  // this thread's neighbour copies have landed
      if (valid) {
        switch (warp) {
          case 0: dg3_face<P, NC, 0>(l, comp, sm, sf, nb); break;
          case 1: dg3_face<P, NC, 1>(l, comp, sm, sf, nb); break;
          case 2: dg3_face<P, NC, 2>(l, comp, sm, sf, nb); break;
          default: dg3_face<P, NC, 3>(l, comp, sm, sf, nb); break;
        }
      }
      __syncthreads();
      T h[D::KQ];
      if (valid && warp < 3) {
        if (warp == 0) dg3_h<P, NC, 0>(l, sm, G, h);
        else if (warp == 1) dg3_h<P, NC, 1>(l, sm, G, h);
        else dg3_h<P, NC, 2>(l, sm, G, h);
      }
      __syncthreads();
      if (valid && warp < 3) {
#pragma unroll
        for (int m = 0; m < D::KQ; ++m) sm[D::OFF_G + (warp * D::KQ + m) * D::CELLS + l] = h[m];
      }
      __syncthreads();
      if (valid) {
        switch (warp) {
          case 0: dg3_out<P, NC, MASS, 0>(l, comp, sm, md); break;
          case 1: dg3_out<P, NC, MASS, 1>(l, comp, sm, md); break;
          case 2: dg3_out<P, NC, MASS, 2>(l, comp, sm, md); break;
          default: dg3_out<P, NC, MASS, 3>(l, comp, sm, md); break;
        }
      }
      __syncthreads();
    }
    stage_out<D::U, D::US, D::THREADS>(pr.dst + c0 * D::U, sm + D::OFF_Y, nloc);
  }
}

// trace pass: g_A = D_A u of the staged row into sg
template <int P, int NC, int A, typename T>
__device__ __forceinline__ void dg3_grad_rows(int l, int comp, const T* su, T* sg) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  T uu[D::K];
#pragma unroll
  for (int i = 0; i < D::K; ++i) uu[i] = su[l * D::US + comp * D::K + i];
#pragma unroll
  for (int m = 0; m < D::KQ; ++m) sg[(A * D::KQ + m) * D::CELLS + l] = O::grad_row(A * D::KQ + m, uu, 1);
}

// trace pass: q_F = sum_a cf_F[a] g_a at the P_{p-1} nodes of face F
template <int P, int NC, int F, typename T>
__device__ __forceinline__ void dg3_publish(int l, int comp, const T* sg, T* sq, const T (&cf)[3]) {
  using D = DG3<P, NC>;
  using O = typename D::O;
#pragma unroll
  for (int m = 0; m < D::NFQ; ++m) {
    const int nq = O::fnq(F, m);
    sq[l * D::QS + (F * NC + comp) * D::NFQ + m] = cf[0] * sg[(0 * D::KQ + nq) * D::CELLS + l] +
                                                   cf[1] * sg[(1 * D::KQ + nq) * D::CELLS + l] +
                                                   cf[2] * sg[(2 * D::KQ + nq) * D::CELLS + l];
  }
}

template <int P, int NC, typename T>
__global__ void __launch_bounds__(128, 8) dg3_trace_kernel(const __grid_constant__ DGBatch<T> batch,
                                                           int64_t n_blocks) {
  using D = DG3<P, NC>;
  using O = typename D::O;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  T* su = sm;                                 // [CELLS][US]
  T* sg = sm + D::CELLS * D::US;              // [3*KQ][CELLS]
  T* sq = sg + 3 * D::KQ * D::CELLS;          // [CELLS][QS]
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * D::CELLS;
    const int nloc = int(pr.n_cells - c0 < D::CELLS ? pr.n_cells - c0 : int64_t(D::CELLS));
    __syncthreads();
    stage_in<D::U, D::US, D::THREADS>(su, pr.src + c0 * D::U, nloc);
    const bool valid = l < nloc;
    const int64_t c = c0 + (valid ? l : 0);
    T cf[3];
    {
      T G[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * pr.n_cells + c);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        switch (warp) {
          case 0: cf[a] = cf_comp(G, 0, a); break;
          case 1: cf[a] = cf_comp(G, 1, a); break;
          case 2: cf[a] = cf_comp(G, 2, a); break;
          default: cf[a] = cf_comp(G, 3, a); break;
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int comp = 0; comp < NC; ++comp) {
      if (valid) {
        switch (warp) {
          case 0: dg3_grad_rows<P, NC, 0>(l, comp, su, sg); break;
          case 1: dg3_grad_rows<P, NC, 1>(l, comp, su, sg); break;
          case 2: dg3_grad_rows<P, NC, 2>(l, comp, su, sg); break;
          default: break;
        }
      }
      __syncthreads();
      if (valid) {
        switch (warp) {
          case 0: dg3_publish<P, NC, 0>(l, comp, sg, sq, cf); break;
          case 1: dg3_publish<P, NC, 1>(l, comp, sg, sq, cf); break;
          case 2: dg3_publish<P, NC, 2>(l, comp, sg, sq, cf); break;
          default: dg3_publish<P, NC, 3>(l, comp, sg, sq, cf); break;
        }
      }
      __syncthreads();
    }
    stage_out<D::QN, D::QS, D::THREADS>(pr.Q + c0 * D::QN, sq, nloc);
  }
}

}  // namespace sfem
