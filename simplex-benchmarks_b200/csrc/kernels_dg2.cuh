// Phase-split DG SIPG kernels (sm_100a): the same operator as kernels_dg.cuh,
// arranged so that no thread holds a whole cell's state at once.
//
// The thread-per-cell apply of kernels_dg.cuh keeps the cell's gradient test
// h (3 x KQ values), its result y (K values), the geometry and the face
// temporaries live across the four face terms: for DG P3 that is more than
// the 168 registers a 6-CTA launch allows, and ptxas spills ~0.5 KB per
// thread, which the L1 (mostly given to the staged rows) cannot hold.
// Here one CTA of BS contiguous cells runs three phases per block:
//   A  own cell: g = grad u; the cell's own traces q_f = 2|F_f| d_n u on all
//      four faces go to shared memory (sq), so neighbours in the same CTA take
//      them from there instead of from the published Q; h = MQ (G g) goes to
//      shared memory (sh);
//   B  faces (after a CTA barrier): jump / average with the neighbour's
//      values and trace - shared memory for neighbours inside the CTA, src
//      and Q in global memory for the others - value tests into y (registers)
//      and gradient tests into sh;
//   C  y += D^T h (h read back from sh), then the results replace the staged
//      src rows once every thread is done with them, and leave with coalesced
//      16-byte stores.
// dg_trace_cross_kernel publishes q_f only for faces whose neighbour lies in
// another block of BS cells (the only traces the apply reads from Q), so the
// trace pass writes about a quarter of the full trace array for BS = 64.
// Scalar problems (NC == 1) only; the multi-component operators keep the
// kernels of kernels_dg.cuh.
#pragma once
#include <cstdint>

#include "kernels_dg.cuh"

namespace sfem {

// YS: the results also live in shared memory (their own rows) while the
// faces run, instead of registers.
template <int P, bool YS = false>
struct DG2Shape {
  using O = gen::Ops<P>;
  static constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  static constexpr int US = padded(K);        // staged src rows (results at the end)
  static constexpr int QS = padded(4 * NFQ);  // own traces of the four faces
  static constexpr int HS = padded(3 * KQ);   // gradient test h
  static constexpr int ELEMS = US + QS + HS + (YS ? US : 0);  // shared values per cell
};

// own traces of the four faces from the gradient g, into q[4][NFQ]
template <int P, typename T>
__device__ __forceinline__ void traces_from_grad(const T (&G)[6], const T* g, T* q) {
  using O = gen::Ops<P>;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    T cf[3];
    face_cf(G, f, cf);
#pragma unroll
    for (int m = 0; m < O::NFQ; ++m) {
      const int nq = O::fnq(f, m);
      q[f * O::NFQ + m] = cf[0] * g[nq] + cf[1] * g[O::KQ + nq] + cf[2] * g[2 * O::KQ + nq];
    }
  }
}

// Publish q_f for the faces whose neighbour is outside this cell's block of BS.
template <int P, int BS, typename T>
__global__ void __launch_bounds__(BS) dg_trace_cross_kernel(const __grid_constant__ DGBatch<T> batch,
                                                            int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S = DG2Shape<P>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [BS][US]
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * BS;
    const int nloc = int(pr.n_cells - c0 < BS ? pr.n_cells - c0 : int64_t(BS));
    __syncthreads();
    stage_in<O::K, S::US, BS>(su, pr.src + c0 * O::K, nloc);
    __syncthreads();
    const int t = threadIdx.x;
    if (t < nloc) {
      const int64_t c = c0 + t;
      const int64_t n = pr.n_cells;
      int32_t nb[4];
      bool cross[4], any = false;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        nb[f] = __ldg(pr.nb + f * n + c);
        const int64_t lc = int64_t(nb[f]) - c0;
        cross[f] = nb[f] >= 0 && (lc < 0 || lc >= nloc);
        any |= cross[f];
      }
      if (any) {
        T G[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
        T u[O::K];
#pragma unroll
        for (int i = 0; i < O::K; ++i) u[i] = su[t * S::US + i];
        T g[3 * O::KQ];
        O::grad(u, g);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          if (!cross[f]) continue;
          T cf[3];
          face_cf(G, f, cf);
          T* q = pr.Q + (c * 4 + f) * O::NFQ;
#pragma unroll
          for (int m = 0; m < O::NFQ; ++m) {
            const int nq = O::fnq(f, m);
            q[m] = cf[0] * g[nq] + cf[1] * g[O::KQ + nq] + cf[2] * g[2 * O::KQ + nq];
          }
        }
      }
    }
  }
}

template <int P, bool MASS, int BS, typename T, int MINB, bool YS = false>
__global__ void __launch_bounds__(BS, MINB) dg_apply2_kernel(const __grid_constant__ DGBatch<T> batch,
                                                             int64_t n_blocks) {
  using O = gen::Ops<P>;
  using S = DG2Shape<P, YS>;
  constexpr int K = O::K, KQ = O::KQ, NF = O::NF, NFQ = O::NFQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [BS][US]  src rows, then results
  T* sq = su + BS * S::US;                 // [BS][QS]  own traces
  T* sh = sq + BS * S::QS;                 // [BS][HS]  gradient test
  T* sy = sh + BS * S::HS;                 // [BS][US]  results (YS)
  for (int64_t blk = blockIdx.x; blk < n_blocks; blk += gridDim.x) {
    const int pi = find_problem(batch, blk);
    const DGProblem<T>& pr = batch.p[pi];
    const int64_t c0 = (blk - batch.block_begin[pi]) * BS;
    const int nloc = int(pr.n_cells - c0 < BS ? pr.n_cells - c0 : int64_t(BS));
    const int64_t n = pr.n_cells;
    const int t = threadIdx.x;
    const int64_t c = c0 + t;
    __syncthreads();
    stage_in<K, S::US, BS>(su, pr.src + c0 * K, nloc);
    __syncthreads();
    T G[6], sf[4];
    int32_t nb[4];
    int nbf[4];
    // ---- A: own gradient, traces, metric and cell mass of the gradient; the
    // face data are loaded first so that they arrive during the contractions
    if (t < nloc) {
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        nb[f] = __ldg(pr.nb + f * n + c);
        nbf[f] = __ldg(pr.nbf + f * n + c);
        sf[f] = __ldg(pr.geo + (6 + f) * n + c);
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) G[k] = __ldg(pr.geo + k * n + c);
      T g[3 * KQ];
      {
        T u[K];
#pragma unroll
        for (int i = 0; i < K; ++i) u[i] = su[t * S::US + i];
        O::grad(u, g);
      }
      traces_from_grad<P>(G, g, sq + t * S::QS);
      T w[3 * KQ];
      apply_metric<KQ>(G, g, w);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        T h[KQ];
        O::massQ(w + a * KQ, h);
#pragma unroll
        for (int m = 0; m < KQ; ++m) sh[t * S::HS + a * KQ + m] = h[m];
      }
    }
    __syncthreads();
    // ---- B: face terms
    T y[K];
    if (t < nloc) {
      const T* u = su + t * S::US;
      const T* qs = sq + t * S::QS;
      T* hs = sh + t * S::HS;
      T* ys = sy + t * S::US;
#pragma unroll
      for (int i = 0; i < K; ++i) y[i] = T(0);
      if (MASS) {
        T uu[K];
#pragma unroll
        for (int i = 0; i < K; ++i) uu[i] = u[i];
        O::massP(uu, __ldg(pr.geo + 10 * n + c), y);
      }
      if (YS) {
#pragma unroll
        for (int i = 0; i < K; ++i) ys[i] = y[i];
      }
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int32_t nbc = nb[f];
        T cf[3];
        face_cf(G, f, cf);
        const T* qm = qs + f * NFQ;
        T j[NF], avg[NFQ];
        if (nbc >= 0) {
          const int nf = nbf[f];
          const int64_t lc = int64_t(nbc) - c0;
          const T* un;
          const T* qn;
          if (lc >= 0 && lc < nloc) {
            un = su + lc * S::US;
            qn = sq + lc * S::QS + nf * NFQ;
          } else {
            un = pr.src + int64_t(nbc) * K;
            qn = pr.Q + (int64_t(nbc) * 4 + nf) * NFQ;
          }
#pragma unroll
          for (int i = 0; i < NF; ++i) j[i] = u[O::fn(f, i)] - un[O::fn_runtime(nf, i)];
#pragma unroll
          for (int m = 0; m < NFQ; ++m) avg[m] = T(0.25) * (qm[m] - qn[m]);
        } else {
#pragma unroll
          for (int i = 0; i < NF; ++i) j[i] = T(2) * u[O::fn(f, i)];
#pragma unroll
          for (int m = 0; m < NFQ; ++m) avg[m] = T(0.5) * qm[m];
        }
        T tt[NF];
        O::facePP(j, tt);
#pragma unroll
        for (int i = 0; i < NF; ++i) tt[i] *= sf[f];
#pragma unroll
        for (int m = 0; m < NFQ; ++m) avg[m] = -avg[m];
        O::facePQ(avg, tt);
        if (YS) {
#pragma unroll
          for (int i = 0; i < NF; ++i) ys[O::fn(f, i)] += tt[i];
        } else {
#pragma unroll
          for (int i = 0; i < NF; ++i) y[O::fn(f, i)] += tt[i];
        }
        T r[NFQ];
        O::faceQP(j, r);
#pragma unroll
        for (int m = 0; m < NFQ; ++m) {
          const int nq = O::fnq(f, m);
          const T rm = T(-0.25) * r[m];
          hs[nq] += cf[0] * rm;
          hs[KQ + nq] += cf[1] * rm;
          hs[2 * KQ + nq] += cf[2] * rm;
        }
      }
      // ---- C: y += D^T h
      if (YS) {
#pragma unroll
        for (int i = 0; i < K; ++i) y[i] = ys[i];
      }
      T h[3 * KQ];
#pragma unroll
      for (int e = 0; e < 3 * KQ; ++e) h[e] = hs[e];
      O::gradT(h, y);
    }
    __syncthreads();  // every thread is done with the staged src rows and traces
    if (t < nloc) {
#pragma unroll
      for (int i = 0; i < K; ++i) su[t * S::US + i] = y[i];
    }
    __syncthreads();
    stage_out<K, S::US, BS>(pr.dst + c0 * K, su, nloc);
  }
}

}  // namespace sfem
