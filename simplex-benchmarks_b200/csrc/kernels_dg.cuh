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
//   A (dg_trace_kernel):  q_f = 2|F| d_n u on face f at the P_{p-1} face nodes,
//                         for all 4 faces of every cell (published in Q);
//   B (dg_apply_kernel):  cell term + the complete face terms of the cell's 4
//                         faces, reading the neighbour's face values from src and
//                         its published q from Q.
// The reference instead sweeps faces in 576 (f_int,f_ext,o_int,o_ext) buckets
// and scatters into both sides (DG/cells_batched/application.cc:1738-2431);
// sorting every cell's vertices by global id removes the orientation part of
// that bucket key, and the element-centric form removes the scatter.
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

namespace sfem {

constexpr int kMaxBatch = 40;

template <typename T>
struct DGProblem {
  const T* geo;       // [n_geo][n_cells]
  const int32_t* nb;  // [4][n_cells]
  const int8_t* nbf;  // [4][n_cells]
  const T* src;       // [n_cells][NC][K]
  T* dst;
  T* Q;               // [n_cells][4][NC][NFQ]
  int64_t n_cells;
};

// Several independent problems in one launch; begin[] is the prefix sum of
// their cell counts.  Passed by value as a kernel parameter.
template <typename T>
struct DGBatch {
  int32_t n;
  int64_t begin[kMaxBatch + 1];
  DGProblem<T> p[kMaxBatch];
};

template <typename T>
__device__ __forceinline__ int find_problem(const DGBatch<T>& b, int64_t gc) {
  int lo = 0, hi = b.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.begin[mid] <= gc) lo = mid; else hi = mid - 1;
  }
  return lo;
}

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

// Publish q_f = 2|F_f| d_n u (own outward normal) at the P_{p-1} nodes of every face.
template <int P, int NC, typename T>
__global__ void __launch_bounds__(128) dg_trace_kernel(const __grid_constant__ DGBatch<T> batch, int64_t n_total) {
  using O = gen::Ops<P>;
  for (int64_t gc = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gc < n_total;
       gc += int64_t(gridDim.x) * blockDim.x) {
    const int pi = find_problem(batch, gc);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c = gc - batch.begin[pi];
    const int64_t n = pr.n_cells;
    T G[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
#pragma unroll
    for (int comp = 0; comp < NC; ++comp) {
      T u[O::K];
      const T* s = pr.src + (c * NC + comp) * O::K;
#pragma unroll
      for (int i = 0; i < O::K; ++i) u[i] = __ldg(s + i);
      T g[3 * O::KQ];
      O::grad(u, g);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        T cf[3];
        face_cf(G, f, cf);
        T* q = pr.Q + ((c * 4 + f) * NC + comp) * O::NFQ;
#pragma unroll
        for (int m = 0; m < O::NFQ; ++m) {
          const int nq = O::fnq(f, m);
          q[m] = cf[0] * g[nq] + cf[1] * g[O::KQ + nq] + cf[2] * g[2 * O::KQ + nq];
        }
      }
    }
  }
}

// Own-cell terms for one component; with HAVE_NB the neighbour traces come
// from src/Q, otherwise (diagonal) they are zero.
template <int P, int NC, bool MASS, bool HAVE_NB, typename T>
__device__ __forceinline__ void dg_cell_component(const DGProblem<T>& pr, int64_t c, int comp,
                                                  const T (&G)[6], const T (&sf)[4], T md,
                                                  const int32_t (&nb)[4], const int (&nbf)[4],
                                                  const T (&u)[gen::Ops<P>::K], T (&y)[gen::Ops<P>::K]) {
  using O = gen::Ops<P>;
  constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  T g[3 * KQ];
  O::grad(u, g);
  T h[3 * KQ];
  {
    T w[3 * KQ];
    apply_metric<KQ>(G, g, w);
#pragma unroll
    for (int a = 0; a < 3; ++a) O::massQ(w + a * KQ, h + a * KQ);
  }
#pragma unroll
  for (int i = 0; i < K; ++i) y[i] = T(0);
  if (MASS) O::massP(u, md, y);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    T cf[3];
    face_cf(G, f, cf);
    T qm[NFQ];
#pragma unroll
    for (int m = 0; m < NFQ; ++m) {
      const int nq = O::fnq(f, m);
      qm[m] = cf[0] * g[nq] + cf[1] * g[KQ + nq] + cf[2] * g[2 * KQ + nq];
    }
    T j[NF], avg[NFQ];
    if (nb[f] >= 0) {
      // interior face: jump and average with the neighbour's published trace
      if (HAVE_NB) {
        const T* us = pr.src + (int64_t(nb[f]) * NC + comp) * K;
        const T* qs = pr.Q + ((int64_t(nb[f]) * 4 + nbf[f]) * NC + comp) * NFQ;
#pragma unroll
        for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)] - __ldg(us + O::fn_runtime(nbf[f], i));
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * (qm[m] - __ldg(qs + m));
      } else {
#pragma unroll
        for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)];
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * qm[m];
      }
    } else {
      // boundary face: u+ = -u-, d_n u+ = d_n u-
#pragma unroll
      for (int i = 0; i < NF; ++i) j[i] = T(2) * u[O::fn(f, i)];
#pragma unroll
      for (int m = 0; m < NFQ; ++m) avg[m] = T(0.5) * qm[m];
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

template <int P, int NC, bool MASS, typename T>
__global__ void __launch_bounds__(128) dg_apply_kernel(const __grid_constant__ DGBatch<T> batch, int64_t n_total) {
  using O = gen::Ops<P>;
  for (int64_t gc = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gc < n_total;
       gc += int64_t(gridDim.x) * blockDim.x) {
    const int pi = find_problem(batch, gc);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c = gc - batch.begin[pi];
    const int64_t n = pr.n_cells;
    T G[6], sf[4];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
#pragma unroll
    for (int f = 0; f < 4; ++f) sf[f] = __ldg(pr.geo + (6 + f) * n + c);
    const T md = MASS ? __ldg(pr.geo + 10 * n + c) : T(0);
    int32_t nb[4];
    int nbf[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      nb[f] = __ldg(pr.nb + f * n + c);
      nbf[f] = __ldg(pr.nbf + f * n + c);
    }
#pragma unroll 1
    for (int comp = 0; comp < NC; ++comp) {
      T u[O::K], y[O::K];
      const T* s = pr.src + (c * NC + comp) * O::K;
#pragma unroll
      for (int i = 0; i < O::K; ++i) u[i] = __ldg(s + i);
      dg_cell_component<P, NC, MASS, true>(pr, c, comp, G, sf, md, nb, nbf, u, y);
      T* d = pr.dst + (c * NC + comp) * O::K;
#pragma unroll
      for (int i = 0; i < O::K; ++i) d[i] = y[i];
    }
  }
}

// Diagonal of the DG operator: (A)_ii = own-cell terms applied to e_i.
template <int P, int NC, bool MASS, typename T>
__global__ void __launch_bounds__(128) dg_diagonal_kernel(const __grid_constant__ DGBatch<T> batch, int64_t n_total) {
  using O = gen::Ops<P>;
  for (int64_t gc = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gc < n_total;
       gc += int64_t(gridDim.x) * blockDim.x) {
    const int pi = find_problem(batch, gc);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c = gc - batch.begin[pi];
    const int64_t n = pr.n_cells;
    T G[6], sf[4];
    for (int k = 0; k < 6; ++k) G[k] = pr.geo[k * n + c];
    for (int f = 0; f < 4; ++f) sf[f] = pr.geo[(6 + f) * n + c];
    const T md = MASS ? pr.geo[10 * n + c] : T(0);
    int32_t nb[4];
    int nbf[4];
    for (int f = 0; f < 4; ++f) {
      nb[f] = pr.nb[f * n + c];
      nbf[f] = pr.nbf[f * n + c];
    }
    for (int i = 0; i < O::K; ++i) {
      T u[O::K], y[O::K];
#pragma unroll
      for (int j = 0; j < O::K; ++j) u[j] = j == i ? T(1) : T(0);
      dg_cell_component<P, NC, MASS, false>(pr, c, 0, G, sf, md, nb, nbf, u, y);
      T yi = T(0);
#pragma unroll
      for (int j = 0; j < O::K; ++j)
        if (j == i) yi = y[j];
      for (int comp = 0; comp < NC; ++comp) pr.dst[(c * NC + comp) * O::K + i] = yi;
    }
  }
}

}  // namespace sfem
