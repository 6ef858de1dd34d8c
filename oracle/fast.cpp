/*
 * fast.cpp - the reference's OPTIMIZED CPU vmult, restated for the CPU
 * baseline.
 *
 * TEST INFRASTRUCTURE ONLY: bench.py times it as the CPU baseline and as the
 * reference arm, tests/ check it against the scalar oracle (oracle.c).  The
 * product never links or calls it.
 *
 * What it restates (the hand-optimised MatrixFree paths of the reference):
 *   CG  cells:  CG/cells_batched/application.cc:1237-1416 (masked gather,
 *               apply_matrix_vector_product over a batch of cell batches,
 *               affine metric at every quadrature point, transposed product,
 *               masked scatter-add), constrained rows = identity (:1160-1176)
 *   DG  cells:  DG/cells_batched/application.cc:1493-1735 (contiguous cell
 *               blocks, same batched products)
 *   DG  faces:  DG/cells_batched/application.cc:1738-2431 (faces grouped by
 *               (face_no_int, face_no_ext, orientations), values and
 *               gradients of both sides at the face points, SIPG flux,
 *               transposed products, scatter-add to both cells) and the
 *               boundary faces :2436-2845 (weak Dirichlet, u+ = -u-)
 *   Helmholtz:  DG/components_batched/application_helmholtz.cc:611-632,
 *               672-733, 841-882 (mass + Laplace per component, sigma from
 *               the two sides' 1/h normal to the face)
 *
 * Layout of the computation, as in the reference:
 *   - cells (faces) in batches of 8 SIMD lanes (VectorizedArray<double> with
 *     AVX-512); 4 batches at a time go through each dense shape-matrix
 *     product, so every matrix entry loaded is used 4 x 8 times;
 *   - shape matrices are dense [n_q*3][k] (gradients) and [n_q][k] (values)
 *     at the quadrature points; face matrices per local face number.  Every
 *     cell lists its vertices in ascending global id, so both sides of a face
 *     see its points in the same order and the orientation part of the
 *     reference's 576 face groups is always the identity: faces are grouped
 *     by (face_no_int, face_no_ext) only;
 *   - OpenMP threads take contiguous ranges of cell batches, as MPI ranks
 *     take contiguous ranges of the z-ordered cells in the reference.  DoFs
 *     (CG) or cells (DG faces) that receive contributions from two threads
 *     go through per-thread buffers that are summed afterwards, the analogue
 *     of the reference's ghost entries and compress(add).
 * Quadrature: the smallest positive symmetric rules exact for the integrands
 * (fast_rules.h, made by gen_rules.py); the reference's QGaussSimplex(p+1)
 * has at least as many points, so this port does no more work per cell.
 */
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "fast_rules.h"

extern "C" int oracle_basis(int32_t degree, const double* xi, double* values, double* grads);

namespace {

constexpr int L = 8;  // SIMD lanes (doubles per 512-bit vector)
typedef double V __attribute__((vector_size(64)));
constexpr int NB = 4;  // cell batches per matrix product

inline V splat(double a) { return V{a, a, a, a, a, a, a, a}; }

constexpr int k_of(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

struct Rule {
  int n = 0;
  std::vector<double> xi;  // [n][3] reference coordinates (tet) or [n][2] (triangle, barycentric 1, 2)
  std::vector<double> w;   // sums to the element measure (1/6 tet, 1/2 triangle)
};

Rule tet_rule(int n, const double (*pts)[4], const double* w) {
  Rule r;
  r.n = n;
  for (int q = 0; q < n; ++q) {
    for (int a = 1; a < 4; ++a) r.xi.push_back(pts[q][a]);
    r.w.push_back(w[q] / 6.0);
  }
  return r;
}
Rule tri_rule(int n, const double (*pts)[3], const double* w) {
  Rule r;
  r.n = n;
  for (int q = 0; q < n; ++q) {
    r.xi.push_back(pts[q][0]);
    r.xi.push_back(pts[q][1]);
    r.xi.push_back(pts[q][2]);
    r.w.push_back(w[q]);  // times the face area at run time
  }
  return r;
}

// The three local vertices of face f of the reference tet, ascending.
void face_vertices(int f, int fv[3]) {
  int m = 0;
  for (int v = 0; v < 4; ++v)
    if (v != f) fv[m++] = v;
}
const double kRefV[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

struct Params {
  int32_t degree, kind, n_components, penalty;
  double mass;
  int32_t n_threads;
};

enum { KIND_CG = 0, KIND_DG = 1, KIND_HELMHOLTZ = 2 };

struct FaceBatch {
  int32_t cm[L], cp[L];  // cells on both sides (-1: empty lane); cp unused on the boundary
  V nm[3], np[3];        // J^-1 n of both sides (n = outward normal of the minus side)
  V sigma, area;
};

struct Ctx {
  Params prm;
  int K = 0, NC = 1, nq = 0, nqf = 0;
  int64_t n_cells = 0, n_dofs = 0, n_batches = 0;
  // cell batches
  std::vector<int32_t> bcell;  // [n_batches][L] cell ids (-1: empty lane)
  std::vector<V> metric;       // [n_batches][6] G = |det J| J^-1 J^-T
  std::vector<V> mscale;       // [n_batches] mass * |det J| (Helmholtz)
  std::vector<int32_t> bdofs;  // CG: [n_batches][K][L] (-1: constrained or empty)
  std::vector<int32_t> constrained_list;
  // shape tables at the cell points
  std::vector<double> D;   // [nq*3][K]
  std::vector<double> Vq;  // [nq][K]
  std::vector<double> wq;  // [nq]
  // face tables per local face: values [4][nqf][K], gradients [4][nqf*3][K]
  std::vector<double> Vf, Df, wf;
  // threads: batch ranges, their faces by bucket, shared targets
  int nt = 1;
  std::vector<int64_t> tb;                   // [nt+1] batch ranges
  std::vector<std::vector<FaceBatch>> tint;  // per thread: interior face batches, grouped by bucket
  std::vector<std::vector<int8_t>> tint_f;   // per batch: (f-, f+) packed as 4 f- + f+
  std::vector<std::vector<FaceBatch>> tbnd;
  std::vector<std::vector<int8_t>> tbnd_f;
  std::vector<int32_t> owner;   // thread of each cell (DG) / unused (CG)
  std::vector<int64_t> shared;  // DG: shared cell id per cell; CG: shared DoF id per DoF (-1: private)
  int64_t n_shared = 0;
  std::vector<int64_t> shared_list;  // the shared cells / DoFs
  std::vector<std::vector<double>> tbuf;  // per thread [n_shared][width]
};

// Small dense product over NB cell batches: out[b][r] = sum_c M[r][c] in[b][c].
// Two rows at a time, so each input vector loaded feeds two FMAs.
template <int ROWS, int COLS>
inline void mv(const double* __restrict M, const V (*__restrict in)[COLS], V (*__restrict out)[ROWS]) {
  int r = 0;
  for (; r + 1 < ROWS; r += 2) {
    V a0 = splat(0), a1 = splat(0), a2 = splat(0), a3 = splat(0);
    V b0 = splat(0), b1 = splat(0), b2 = splat(0), b3 = splat(0);
    for (int c = 0; c < COLS; ++c) {
      const V m = splat(M[r * COLS + c]), n = splat(M[(r + 1) * COLS + c]);
      const V x0 = in[0][c], x1 = in[1][c], x2 = in[2][c], x3 = in[3][c];
      a0 += m * x0; a1 += m * x1; a2 += m * x2; a3 += m * x3;
      b0 += n * x0; b1 += n * x1; b2 += n * x2; b3 += n * x3;
    }
    out[0][r] = a0; out[1][r] = a1; out[2][r] = a2; out[3][r] = a3;
    out[0][r + 1] = b0; out[1][r + 1] = b1; out[2][r + 1] = b2; out[3][r + 1] = b3;
  }
  for (; r < ROWS; ++r) {
    V s0 = splat(0), s1 = splat(0), s2 = splat(0), s3 = splat(0);
    for (int c = 0; c < COLS; ++c) {
      const V m = splat(M[r * COLS + c]);
      s0 += m * in[0][c]; s1 += m * in[1][c]; s2 += m * in[2][c]; s3 += m * in[3][c];
    }
    out[0][r] = s0; out[1][r] = s1; out[2][r] = s2; out[3][r] = s3;
  }
}
// transposed: out[b][c] (+)= sum_r M[r][c] in[b][r], two columns at a time
template <int ROWS, int COLS, bool ADD>
inline void mvT(const double* __restrict M, const V (*__restrict in)[ROWS], V (*__restrict out)[COLS]) {
  int c = 0;
  for (; c + 1 < COLS; c += 2) {
    V a0 = ADD ? out[0][c] : splat(0), a1 = ADD ? out[1][c] : splat(0), a2 = ADD ? out[2][c] : splat(0),
      a3 = ADD ? out[3][c] : splat(0);
    V b0 = ADD ? out[0][c + 1] : splat(0), b1 = ADD ? out[1][c + 1] : splat(0),
      b2 = ADD ? out[2][c + 1] : splat(0), b3 = ADD ? out[3][c + 1] : splat(0);
    for (int r = 0; r < ROWS; ++r) {
      const V m = splat(M[r * COLS + c]), n = splat(M[r * COLS + c + 1]);
      const V x0 = in[0][r], x1 = in[1][r], x2 = in[2][r], x3 = in[3][r];
      a0 += m * x0; a1 += m * x1; a2 += m * x2; a3 += m * x3;
      b0 += n * x0; b1 += n * x1; b2 += n * x2; b3 += n * x3;
    }
    out[0][c] = a0; out[1][c] = a1; out[2][c] = a2; out[3][c] = a3;
    out[0][c + 1] = b0; out[1][c + 1] = b1; out[2][c + 1] = b2; out[3][c + 1] = b3;
  }
  for (; c < COLS; ++c) {
    V s0 = ADD ? out[0][c] : splat(0), s1 = ADD ? out[1][c] : splat(0), s2 = ADD ? out[2][c] : splat(0),
      s3 = ADD ? out[3][c] : splat(0);
    for (int r = 0; r < ROWS; ++r) {
      const V m = splat(M[r * COLS + c]);
      s0 += m * in[0][r]; s1 += m * in[1][r]; s2 += m * in[2][r]; s3 += m * in[3][r];
    }
    out[0][c] = s0; out[1][c] = s1; out[2][c] = s2; out[3][c] = s3;
  }
}

// ---- cell term ------------------------------------------------------------
template <int P, int NQ, int NCOMP, bool MASS, bool CG>
void cell_batches(const Ctx& c, int t, const double* src, double* dst) {
  constexpr int K = k_of(P);
  const int64_t b0 = c.tb[t], b1 = c.tb[t + 1];
  std::vector<double>& buf = const_cast<std::vector<double>&>(c.tbuf[t]);
  alignas(64) V u[NB][K], g[NB][NQ * 3], y[NB][K], vq[NB][NQ];
  for (int64_t b = b0; b < b1; b += NB) {
    const int nb = int(std::min<int64_t>(NB, b1 - b));
    for (int comp = 0; comp < NCOMP; ++comp) {
      // gather (masked for CG, contiguous blocks for DG)
      for (int j = 0; j < NB; ++j) {
        const int64_t bb = b + j;
        for (int i = 0; i < K; ++i) {
          alignas(64) double lane[L];
          for (int v = 0; v < L; ++v) {
            double val = 0.0;
            if (j < nb) {
              if (CG) {
                const int32_t d = c.bdofs[(bb * K + i) * L + v];
                val = d >= 0 ? src[d] : 0.0;
              } else {
                const int32_t cell = c.bcell[bb * L + v];
                val = cell >= 0 ? src[(int64_t(cell) * NCOMP + comp) * K + i] : 0.0;
              }
            }
            lane[v] = val;
          }
          std::memcpy(&u[j][i], lane, sizeof(V));
        }
      }
      mv<NQ * 3, K>(c.D.data(), u, g);
      for (int j = 0; j < NB; ++j) {
        const int64_t bb = std::min<int64_t>(b + j, b1 - 1);
        const V* G = &c.metric[6 * bb];
        for (int q = 0; q < NQ; ++q) {
          const V w = splat(c.wq[q]);
          const V gx = g[j][3 * q], gy = g[j][3 * q + 1], gz = g[j][3 * q + 2];
          g[j][3 * q] = w * (G[0] * gx + G[3] * gy + G[4] * gz);
          g[j][3 * q + 1] = w * (G[3] * gx + G[1] * gy + G[5] * gz);
          g[j][3 * q + 2] = w * (G[4] * gx + G[5] * gy + G[2] * gz);
        }
      }
      mvT<NQ * 3, K, false>(c.D.data(), g, y);
      if (MASS) {
        mv<NQ, K>(c.Vq.data(), u, vq);
        for (int j = 0; j < NB; ++j) {
          const int64_t bb = std::min<int64_t>(b + j, b1 - 1);
          for (int q = 0; q < NQ; ++q) vq[j][q] *= splat(c.wq[q]) * c.mscale[bb];
        }
        mvT<NQ, K, true>(c.Vq.data(), vq, y);
      }
      // scatter
      for (int j = 0; j < nb; ++j) {
        const int64_t bb = b + j;
        for (int i = 0; i < K; ++i) {
          alignas(64) double lane[L];
          std::memcpy(lane, &y[j][i], sizeof(V));
          for (int v = 0; v < L; ++v) {
            if (CG) {
              const int32_t d = c.bdofs[(bb * K + i) * L + v];
              if (d < 0) continue;
              const int64_t s = c.shared[d];
              if (s < 0) dst[d] += lane[v];
              else buf[s] += lane[v];
            } else {
              const int32_t cell = c.bcell[bb * L + v];
              if (cell >= 0) dst[(int64_t(cell) * NCOMP + comp) * K + i] = lane[v];
            }
          }
        }
      }
    }
  }
}

// ---- face terms -------------------------------------------------------------
template <int P, int NQF, int NCOMP, bool BOUNDARY>
void face_batches(const Ctx& c, int t, const double* src, double* dst) {
  constexpr int K = k_of(P);
  const std::vector<FaceBatch>& fb = BOUNDARY ? c.tbnd[t] : c.tint[t];
  const std::vector<int8_t>& ff = BOUNDARY ? c.tbnd_f[t] : c.tint_f[t];
  std::vector<double>& buf = const_cast<std::vector<double>&>(c.tbuf[t]);
  const int W = NCOMP * K;
  alignas(64) V um[NB][K], up[NB][K], vm[NB][NQF], vp[NB][NQF], gm[NB][NQF * 3], gp[NB][NQF * 3];
  alignas(64) V tv[NB][NQF], tgm[NB][NQF * 3], tgp[NB][NQF * 3], ym[NB][K], yp[NB][K];
  const size_t nfb = fb.size();
  size_t i0 = 0;
  while (i0 < nfb) {
    // up to NB batches of the same bucket
    size_t i1 = i0 + 1;
    while (i1 < nfb && i1 - i0 < size_t(NB) && ff[i1] == ff[i0]) ++i1;
    const int nb = int(i1 - i0);
    const int fmi = ff[i0] >> 2, fpi = ff[i0] & 3;
    const double* Vm = &c.Vf[size_t(fmi) * NQF * K];
    const double* Dm = &c.Df[size_t(fmi) * NQF * 3 * K];
    const double* Vp = &c.Vf[size_t(fpi) * NQF * K];
    const double* Dp = &c.Df[size_t(fpi) * NQF * 3 * K];
    for (int comp = 0; comp < NCOMP; ++comp) {
      for (int j = 0; j < NB; ++j) {
        const FaceBatch& B = fb[i0 + std::min(j, nb - 1)];
        for (int i = 0; i < K; ++i) {
          alignas(64) double lm[L], lp[L];
          for (int v = 0; v < L; ++v) {
            const int32_t a = B.cm[v];
            lm[v] = (j < nb && a >= 0) ? src[(int64_t(a) * NCOMP + comp) * K + i] : 0.0;
            if (!BOUNDARY) {
              const int32_t p = B.cp[v];
              lp[v] = (j < nb && p >= 0) ? src[(int64_t(p) * NCOMP + comp) * K + i] : 0.0;
            }
          }
          std::memcpy(&um[j][i], lm, sizeof(V));
          if (!BOUNDARY) std::memcpy(&up[j][i], lp, sizeof(V));
        }
      }
      mv<NQF, K>(Vm, um, vm);
      mv<NQF * 3, K>(Dm, um, gm);
      if (!BOUNDARY) {
        mv<NQF, K>(Vp, up, vp);
        mv<NQF * 3, K>(Dp, up, gp);
      }
      for (int j = 0; j < NB; ++j) {
        const FaceBatch& B = fb[i0 + std::min(j, nb - 1)];
        for (int q = 0; q < NQF; ++q) {
          const V jxw = B.area * splat(c.wf[q]);
          const V dnm = B.nm[0] * gm[j][3 * q] + B.nm[1] * gm[j][3 * q + 1] + B.nm[2] * gm[j][3 * q + 2];
          V jump, avg;
          if (BOUNDARY) {
            jump = splat(2.0) * vm[j][q];
            avg = dnm;
          } else {
            const V dnp = B.np[0] * gp[j][3 * q] + B.np[1] * gp[j][3 * q + 1] + B.np[2] * gp[j][3 * q + 2];
            jump = vm[j][q] - vp[j][q];
            avg = splat(0.5) * (dnm + dnp);
          }
          tv[j][q] = (B.sigma * jump - avg) * jxw;
          const V tg = splat(-0.5) * jump * jxw;
          for (int a = 0; a < 3; ++a) {
            tgm[j][3 * q + a] = tg * B.nm[a];
            if (!BOUNDARY) tgp[j][3 * q + a] = tg * B.np[a];
          }
        }
      }
      mvT<NQF, K, false>(Vm, tv, ym);
      mvT<NQF * 3, K, true>(Dm, tgm, ym);
      if (!BOUNDARY) {
        for (int j = 0; j < NB; ++j)
          for (int q = 0; q < NQF; ++q) tv[j][q] = -tv[j][q];
        mvT<NQF, K, false>(Vp, tv, yp);
        mvT<NQF * 3, K, true>(Dp, tgp, yp);
      }
      for (int j = 0; j < nb; ++j) {
        const FaceBatch& B = fb[i0 + j];
        for (int i = 0; i < K; ++i) {
          alignas(64) double lm[L], lp[L];
          std::memcpy(lm, &ym[j][i], sizeof(V));
          if (!BOUNDARY) std::memcpy(lp, &yp[j][i], sizeof(V));
          for (int v = 0; v < L; ++v) {
            const int32_t a = B.cm[v];
            if (a < 0) continue;
            dst[(int64_t(a) * NCOMP + comp) * K + i] += lm[v];  // the minus cell is always this thread's
            if (!BOUNDARY) {
              const int32_t p = B.cp[v];
              const int64_t s = c.shared[p];
              if (s < 0) dst[(int64_t(p) * NCOMP + comp) * K + i] += lp[v];
              else buf[size_t(s) * W + comp * K + i] += lp[v];
            }
          }
        }
      }
    }
    i0 = i1;
  }
}

template <int P, int NQ, int NQF, int NCOMP, bool MASS>
void vmult_dg(Ctx& c, const double* src, double* dst) {
  const int W = NCOMP * k_of(P);
#pragma omp parallel num_threads(c.nt)
  {
    const int t = omp_get_thread_num();
    std::fill(c.tbuf[t].begin(), c.tbuf[t].end(), 0.0);
    cell_batches<P, NQ, NCOMP, MASS, false>(c, t, src, dst);
    face_batches<P, NQF, NCOMP, false>(c, t, src, dst);
    face_batches<P, NQF, NCOMP, true>(c, t, src, dst);
#pragma omp barrier
#pragma omp for schedule(static)
    for (int64_t s = 0; s < c.n_shared; ++s) {
      double* d = dst + c.shared_list[s] * W;
      for (int tt = 0; tt < c.nt; ++tt) {
        const double* b = &c.tbuf[tt][size_t(s) * W];
        for (int i = 0; i < W; ++i) d[i] += b[i];
      }
    }
  }
}

template <int P, int NQ>
void vmult_cg(Ctx& c, const double* src, double* dst) {
#pragma omp parallel num_threads(c.nt)
  {
    const int t = omp_get_thread_num();
    std::fill(c.tbuf[t].begin(), c.tbuf[t].end(), 0.0);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < c.n_dofs; ++i) dst[i] = 0.0;
    cell_batches<P, NQ, 1, false, true>(c, t, src, dst);
#pragma omp barrier
#pragma omp for schedule(static)
    for (int64_t s = 0; s < c.n_shared; ++s) {
      double acc = 0.0;
      for (int tt = 0; tt < c.nt; ++tt) acc += c.tbuf[tt][s];
      dst[c.shared_list[s]] = acc;
    }
#pragma omp for schedule(static)
    for (int64_t i = 0; i < int64_t(c.constrained_list.size()); ++i)
      dst[c.constrained_list[i]] = src[c.constrained_list[i]];
  }
}

// ---- set-up -------------------------------------------------------------------
struct Geo {
  double J[3][3], Ji[3][3], det;
};
Geo geometry(const double* x, const int32_t* cv) {
  Geo g;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) g.J[i][j] = x[3 * int64_t(cv[j + 1]) + i] - x[3 * int64_t(cv[0]) + i];
  const double(&J)[3][3] = g.J;
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  g.det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / g.det;
  g.Ji[0][0] = c00 * id;
  g.Ji[1][0] = c01 * id;
  g.Ji[2][0] = c02 * id;
  g.Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  g.Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  g.Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  g.Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  g.Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  g.Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return g;
}

// outward unit normal and area of local face f
void face_normal(const double* x, const int32_t* cv, int f, double n[3], double& area) {
  int fv[3];
  face_vertices(f, fv);
  const double* p0 = &x[3 * int64_t(cv[fv[0]])];
  const double* p1 = &x[3 * int64_t(cv[fv[1]])];
  const double* p2 = &x[3 * int64_t(cv[fv[2]])];
  const double* o = &x[3 * int64_t(cv[f])];
  double a[3], b[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = p1[i] - p0[i];
    b[i] = p2[i] - p0[i];
  }
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  area = 0.5 * len;
  double dot = 0;
  for (int i = 0; i < 3; ++i) dot += cr[i] * (o[i] - p0[i]);
  const double s = dot > 0 ? -1.0 / len : 1.0 / len;
  for (int i = 0; i < 3; ++i) n[i] = cr[i] * s;
}

void shape_tables(Ctx& c, const Rule& cell, const Rule& face) {
  const int K = c.K, p = c.prm.degree;
  c.nq = cell.n;
  c.nqf = face.n;
  c.D.assign(size_t(cell.n) * 3 * K, 0.0);
  c.Vq.assign(size_t(cell.n) * K, 0.0);
  c.wq = cell.w;
  std::vector<double> val(K), grad(3 * K);
  for (int q = 0; q < cell.n; ++q) {
    oracle_basis(p, &cell.xi[3 * q], val.data(), grad.data());
    for (int i = 0; i < K; ++i) {
      c.Vq[size_t(q) * K + i] = val[i];
      for (int a = 0; a < 3; ++a) c.D[(size_t(q) * 3 + a) * K + i] = grad[3 * i + a];
    }
  }
  c.Vf.assign(size_t(4) * face.n * K, 0.0);
  c.Df.assign(size_t(4) * face.n * 3 * K, 0.0);
  c.wf = face.w;
  for (int f = 0; f < 4; ++f) {
    int fv[3];
    face_vertices(f, fv);
    for (int q = 0; q < face.n; ++q) {
      double xi[3] = {0, 0, 0};
      for (int m = 0; m < 3; ++m)
        for (int a = 0; a < 3; ++a) xi[a] += face.xi[3 * q + m] * kRefV[fv[m]][a];
      oracle_basis(p, xi, val.data(), grad.data());
      for (int i = 0; i < K; ++i) {
        c.Vf[(size_t(f) * face.n + q) * K + i] = val[i];
        for (int a = 0; a < 3; ++a) c.Df[((size_t(f) * face.n + q) * 3 + a) * K + i] = grad[3 * i + a];
      }
    }
  }
}

}  // namespace

extern "C" {

struct fast_ctx;

int fast_create(const Params* prm, int64_t nv, const double* x, int64_t nc, const int32_t* cells,
                const int32_t* nb, const int8_t* nbf, const int32_t* cell_dofs, const uint8_t* constrained,
                int64_t n_dofs, fast_ctx** out) {
  (void)nv;
  if (!prm || !out || prm->degree < 1 || prm->degree > 3) return 1;
  if (prm->kind == KIND_HELMHOLTZ && prm->degree > 2) return 1;  // no positive degree-6 rule in the table
  auto c = std::make_unique<Ctx>();
  c->prm = *prm;
  const int p = prm->degree;
  const int K = k_of(p);
  c->K = K;
  c->NC = prm->kind == KIND_HELMHOLTZ ? std::max(1, prm->n_components) : 1;
  if (c->NC != 1 && c->NC != 3) return 1;
  c->n_cells = nc;
  c->nt = prm->n_threads > 0 ? prm->n_threads : omp_get_max_threads();
  const bool mass = prm->kind == KIND_HELMHOLTZ;
  // rules: Laplace cell 2p-2, mass 2p; faces 2p
  Rule cell, face;
  const int need = mass ? 2 * p : 2 * p - 2;
  if (need <= 1) cell = tet_rule(kRule_tet1_n, kRule_tet1_pts, kRule_tet1_w);
  else if (need <= 2) cell = tet_rule(kRule_tet4_n, kRule_tet4_pts, kRule_tet4_w);
  else cell = tet_rule(kRule_tet14_n, kRule_tet14_pts, kRule_tet14_w);
  if (p == 1) face = tri_rule(kRule_tri3_n, kRule_tri3_pts, kRule_tri3_w);
  else if (p == 2) face = tri_rule(kRule_tri6_n, kRule_tri6_pts, kRule_tri6_w);
  else face = tri_rule(kRule_tri12_n, kRule_tri12_pts, kRule_tri12_w);
  shape_tables(*c, cell, face);

  c->n_batches = (nc + L - 1) / L;
  const int64_t nbt = c->n_batches;
  c->bcell.assign(size_t(nbt) * L, -1);
  for (int64_t i = 0; i < nc; ++i) c->bcell[i] = int32_t(i);
  c->metric.assign(size_t(nbt) * 6, splat(0));
  c->mscale.assign(size_t(nbt), splat(0));
  std::vector<Geo> geo(nc);
  for (int64_t i = 0; i < nc; ++i) geo[i] = geometry(x, cells + 4 * i);
  for (int64_t i = 0; i < nc; ++i) {
    const Geo& g = geo[i];
    const double ad = std::fabs(g.det);
    double G[6];
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) {
      double s = 0;
      for (int e = 0; e < 3; ++e) s += g.Ji[ia[k]][e] * g.Ji[ib[k]][e];
      G[k] = s * ad;
    }
    for (int k = 0; k < 6; ++k) c->metric[6 * (i / L) + k][i % L] = G[k];
    c->mscale[i / L][i % L] = prm->mass * ad;
  }

  // thread ranges over cell batches (whole batches of NB)
  const int nt = c->nt;
  c->tb.assign(nt + 1, 0);
  const int64_t groups = (nbt + NB - 1) / NB;
  for (int t = 0; t <= nt; ++t) c->tb[t] = std::min<int64_t>(nbt, (groups * t / nt) * NB);
  std::vector<int32_t> owner(nc);
  for (int t = 0; t < nt; ++t)
    for (int64_t b = c->tb[t]; b < c->tb[t + 1]; ++b)
      for (int v = 0; v < L; ++v)
        if (b * L + v < nc) owner[b * L + v] = t;

  if (prm->kind == KIND_CG) {
    c->n_dofs = n_dofs;
    c->bdofs.assign(size_t(nbt) * K * L, -1);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < K; ++k) {
        const int32_t d = cell_dofs[int64_t(K) * i + k];
        c->bdofs[((i / L) * K + k) * L + i % L] = constrained[d] ? -1 : d;
      }
    for (int64_t d = 0; d < n_dofs; ++d)
      if (constrained[d]) c->constrained_list.push_back(int32_t(d));
    // a DoF is shared when cells of two threads touch it
    std::vector<int32_t> first(n_dofs, -1);
    std::vector<uint8_t> multi(n_dofs, 0);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < K; ++k) {
        const int32_t d = cell_dofs[int64_t(K) * i + k];
        if (first[d] < 0) first[d] = owner[i];
        else if (first[d] != owner[i]) multi[d] = 1;
      }
    c->shared.assign(n_dofs, -1);
    for (int64_t d = 0; d < n_dofs; ++d)
      if (multi[d] && !constrained[d]) {
        c->shared[d] = int64_t(c->shared_list.size());
        c->shared_list.push_back(d);
      }
    c->n_shared = int64_t(c->shared_list.size());
    c->tbuf.assign(nt, std::vector<double>(std::max<int64_t>(1, c->n_shared), 0.0));
    c->tint.resize(nt);
    c->tbnd.resize(nt);
    *out = reinterpret_cast<fast_ctx*>(c.release());
    return 0;
  }

  // DG: SIPG penalty (DG/cells_batched/application.cc:1191-1245) or the
  // Helmholtz sigma (application_helmholtz.cc:1329-1333, 857-859)
  c->n_dofs = nc * c->NC * K;
  const double factor = prm->penalty == 1 ? double((p + 1) * (p + 1)) : double((p + 1) * (p + 3)) / 3.0;
  std::vector<double> tau(nc), area(4 * size_t(nc)), ih(4 * size_t(nc));
  std::vector<double> nrm(12 * size_t(nc));
  for (int64_t i = 0; i < nc; ++i) {
    const double ad = std::fabs(geo[i].det);
    double surf = 0;
    for (int f = 0; f < 4; ++f) {
      double a;
      face_normal(x, cells + 4 * i, f, &nrm[12 * i + 3 * f], a);
      area[4 * i + f] = a;
      ih[4 * i + f] = 2.0 * a / ad;
      surf += a * (nb[4 * i + f] < 0 ? 1.0 : 0.5);
    }
    tau[i] = surf / (ad / 6.0);
  }
  auto sigma_of = [&](int64_t i, int f) {
    const int32_t o = nb[4 * i + f];
    if (mass) return o >= 0 ? factor * 0.5 * (ih[4 * i + f] + ih[4 * size_t(o) + nbf[4 * i + f]]) : factor * ih[4 * i + f];
    return o >= 0 ? factor * std::max(tau[i], tau[o]) : factor * tau[i];
  };
  auto jin = [&](int64_t i, const double n[3], V* out, int v) {
    // J^-1 n: the reference-space direction whose product with grad_xi is d_n
    for (int a = 0; a < 3; ++a) {
      double s = 0;
      for (int e = 0; e < 3; ++e) s += geo[i].Ji[a][e] * n[e];
      out[a][v] = s;
    }
  };
  // faces owned by the thread of the minus cell (the lower id); 16 buckets
  c->tint.resize(nt);
  c->tint_f.resize(nt);
  c->tbnd.resize(nt);
  c->tbnd_f.resize(nt);
  c->shared.assign(nc, -1);
  for (int t = 0; t < nt; ++t) {
    std::vector<std::vector<std::pair<int32_t, int8_t>>> bucket(16), bbucket(4);
    const int64_t c0 = c->tb[t] * L, c1 = std::min<int64_t>(nc, c->tb[t + 1] * L);
    for (int64_t i = c0; i < c1; ++i)
      for (int f = 0; f < 4; ++f) {
        const int32_t o = nb[4 * i + f];
        if (o < 0) bbucket[f].push_back({int32_t(i), int8_t(f)});
        else if (o > i) bucket[4 * f + nbf[4 * i + f]].push_back({int32_t(i), int8_t(f)});
      }
    for (int bk = 0; bk < 16; ++bk) {
      const auto& lst = bucket[bk];
      for (size_t s = 0; s < lst.size(); s += L) {
        FaceBatch B;
        for (int a = 0; a < 3; ++a) B.nm[a] = B.np[a] = splat(0);
        B.sigma = B.area = splat(0);
        for (int v = 0; v < L; ++v) {
          B.cm[v] = B.cp[v] = -1;
          if (s + v >= lst.size()) continue;
          const int64_t i = lst[s + v].first;
          const int f = lst[s + v].second;
          const int32_t o = nb[4 * i + f];
          B.cm[v] = int32_t(i);
          B.cp[v] = o;
          const double* n = &nrm[12 * i + 3 * f];
          jin(i, n, B.nm, v);
          jin(o, n, B.np, v);
          B.sigma[v] = sigma_of(i, f);
          B.area[v] = area[4 * i + f];
          if (owner[o] != t && c->shared[o] < 0) {
            c->shared[o] = int64_t(c->shared_list.size());
            c->shared_list.push_back(o);
          }
        }
        c->tint[t].push_back(B);
        c->tint_f[t].push_back(int8_t(bk));
      }
    }
    for (int f = 0; f < 4; ++f) {
      const auto& lst = bbucket[f];
      for (size_t s = 0; s < lst.size(); s += L) {
        FaceBatch B;
        for (int a = 0; a < 3; ++a) B.nm[a] = B.np[a] = splat(0);
        B.sigma = B.area = splat(0);
        for (int v = 0; v < L; ++v) {
          B.cm[v] = B.cp[v] = -1;
          if (s + v >= lst.size()) continue;
          const int64_t i = lst[s + v].first;
          B.cm[v] = int32_t(i);
          jin(i, &nrm[12 * i + 3 * f], B.nm, v);
          B.sigma[v] = sigma_of(i, f);
          B.area[v] = area[4 * i + f];
        }
        c->tbnd[t].push_back(B);
        c->tbnd_f[t].push_back(int8_t(4 * f + f));
      }
    }
  }
  c->n_shared = int64_t(c->shared_list.size());
  c->tbuf.assign(nt, std::vector<double>(std::max<int64_t>(1, c->n_shared * c->NC * K), 0.0));
  *out = reinterpret_cast<fast_ctx*>(c.release());
  return 0;
}

void fast_destroy(fast_ctx* ctx) { delete reinterpret_cast<Ctx*>(ctx); }

int64_t fast_n_dofs(const fast_ctx* ctx) { return reinterpret_cast<const Ctx*>(ctx)->n_dofs; }

int fast_info(const fast_ctx* ctx, int32_t* nq, int32_t* nqf, int32_t* lanes, int32_t* threads) {
  const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
  if (nq) *nq = c->nq;
  if (nqf) *nqf = c->nqf;
  if (lanes) *lanes = L;
  if (threads) *threads = c->nt;
  return 0;
}

// diagonal of the CG operator (constrained rows 1): sum over cells of
// w_q (D_q phi_i)^T G (D_q phi_i), the Jacobi entries of the smoother
int fast_diagonal(fast_ctx* ctx, double* diag) {
  Ctx& c = *reinterpret_cast<Ctx*>(ctx);
  if (c.prm.kind != KIND_CG) return 1;
  const int K = c.K, nq = c.nq;
  // per local node i and metric component k: sum_q w_q g_a g_b
  std::vector<double> S(size_t(K) * 6, 0.0);
  const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
  for (int i = 0; i < K; ++i)
    for (int q = 0; q < nq; ++q)
      for (int k = 0; k < 6; ++k) {
        const double ga = c.D[(size_t(q) * 3 + ia[k]) * K + i], gb = c.D[(size_t(q) * 3 + ib[k]) * K + i];
        S[size_t(i) * 6 + k] += c.wq[q] * ga * gb * (ia[k] == ib[k] ? 1.0 : 2.0);
      }
  std::fill(diag, diag + c.n_dofs, 0.0);
  for (int64_t b = 0; b < c.n_batches; ++b)
    for (int v = 0; v < L; ++v) {
      if (c.bcell[b * L + v] < 0) continue;
      for (int i = 0; i < K; ++i) {
        const int32_t d = c.bdofs[(b * K + i) * L + v];
        if (d < 0) continue;
        double s = 0;
        for (int k = 0; k < 6; ++k) s += S[size_t(i) * 6 + k] * c.metric[6 * b + k][v];
        diag[d] += s;
      }
    }
  for (int32_t d : c.constrained_list) diag[d] = 1.0;
  return 0;
}

int fast_vmult(fast_ctx* ctx, const double* src, double* dst) {
  Ctx& c = *reinterpret_cast<Ctx*>(ctx);
  const int p = c.prm.degree;
  if (c.prm.kind == KIND_CG) {
    if (p == 1) vmult_cg<1, 1>(c, src, dst);
    else if (p == 2) vmult_cg<2, 4>(c, src, dst);
    else vmult_cg<3, 14>(c, src, dst);
    return 0;
  }
  if (c.prm.kind == KIND_DG) {
    if (p == 1) vmult_dg<1, 1, 3, 1, false>(c, src, dst);
    else if (p == 2) vmult_dg<2, 4, 6, 1, false>(c, src, dst);
    else vmult_dg<3, 14, 12, 1, false>(c, src, dst);
    return 0;
  }
  if (c.NC == 3) {
    if (p == 1) vmult_dg<1, 4, 3, 3, true>(c, src, dst);
    else vmult_dg<2, 14, 6, 3, true>(c, src, dst);
  } else {
    if (p == 1) vmult_dg<1, 4, 3, 1, true>(c, src, dst);
    else vmult_dg<2, 14, 6, 1, true>(c, src, dst);
  }
  return 0;
}

}  // extern "C"
