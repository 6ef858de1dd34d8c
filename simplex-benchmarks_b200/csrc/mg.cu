// Hybrid p/h multigrid (V-cycle, Chebyshev-Jacobi smoothing, dense FP64
// coarse solve) and preconditioned CG.
//
// Level sequence (MultigridPreconditioner ctor, CG/cells_batched/application_ph.cc:1769-1907):
//   order PH: P1 on the coarsest mesh ... P1 on the fine mesh, then P2 ... Pp on the fine mesh
//   order HP (application_hp.cc:1819-1843): P1 ... Pp on the coarsest mesh, then Pp on finer meshes
// Transfers (MGTwoLevelTransfer): prolongation is the nodal interpolation of the
// coarse function at the fine nodes; restriction is its transpose.
// Smoother (PreconditionChebyshev + DiagonalMatrix, application_ph.cc:1909-1932):
//   Chebyshev of degree d around the Jacobi-preconditioned operator, lambda_max
//   from a CG/Lanczos estimate times a safety factor, lambda_min = lambda_max/range.
// Coarse grid: the reference uses Trilinos ML AMG on the level-0 matrix
//   (application_ph.cc:1934-1946); here the level-0 matrix (125 DoFs at 4^3)
//   is assembled in FP64 and inverted densely.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "learned.hpp"
#include "mg.hpp"
#include "ref_tables.h"
#include "vector_kernels.cuh"

namespace sfem {

namespace {

int k_of_deg(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

// ---------------------------------------------------------------- transfers
// One fine cell: coarse parent cell, local interpolation matrix id and the
// bit mask of the fine local nodes this cell owns (first touch), so that
// every fine DoF is written by exactly one cell.
struct TransferHost {
  int Kf = 0, Kc = 0;
  std::vector<int32_t> parent;
  std::vector<uint8_t> mat_id;
  std::vector<uint32_t> owner;
  std::vector<double> mats;  // [n_mat][Kf][Kc]
};

template <typename T>
__global__ void transfer_prolongate_add(int64_t nf, int Kf, int Kc, const int32_t* __restrict__ parent,
                                        const uint8_t* __restrict__ mid, const uint32_t* __restrict__ owner,
                                        const double* __restrict__ mats, const int32_t* __restrict__ fdofs,
                                        const int32_t* __restrict__ cdofs, int64_t nc, const T* __restrict__ xc,
                                        T* __restrict__ xf) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nf) return;
  const uint32_t ow = owner[c];
  if (!ow) return;
  const int64_t pc = parent[c];
  const double* M = mats + int64_t(mid[c]) * Kf * Kc;
  double xl[20];
  for (int j = 0; j < Kc; ++j) {
    const int32_t g = cdofs[j * nc + pc];
    xl[j] = g >= 0 ? double(xc[g]) : 0.0;
  }
  for (int i = 0; i < Kf; ++i) {
    if (!((ow >> i) & 1u)) continue;
    const int32_t g = fdofs[i * nf + c];
    if (g < 0) continue;
    double acc = 0.0;
    for (int j = 0; j < Kc; ++j) acc += M[i * Kc + j] * xl[j];
    xf[g] += T(acc);
  }
}

template <typename T>
__global__ void transfer_restrict_add(int64_t nf, int Kf, int Kc, const int32_t* __restrict__ parent,
                                      const uint8_t* __restrict__ mid, const uint32_t* __restrict__ owner,
                                      const double* __restrict__ mats, const int32_t* __restrict__ fdofs,
                                      const int32_t* __restrict__ cdofs, int64_t nc, const T* __restrict__ xf,
                                      T* __restrict__ xc) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nf) return;
  const uint32_t ow = owner[c];
  if (!ow) return;
  const int64_t pc = parent[c];
  const double* M = mats + int64_t(mid[c]) * Kf * Kc;
  double rl[20];
  for (int i = 0; i < Kf; ++i) {
    rl[i] = 0.0;
    if ((ow >> i) & 1u) {
      const int32_t g = fdofs[i * nf + c];
      if (g >= 0) rl[i] = double(xf[g]);
    }
  }
  for (int j = 0; j < Kc; ++j) {
    const int32_t g = cdofs[j * nc + pc];
    if (g < 0) continue;
    double acc = 0.0;
    for (int i = 0; i < Kf; ++i) acc += M[i * Kc + j] * rl[i];
    if (acc != 0.0) atomicAdd(xc + g, T(acc));
  }
}

// The same two transfers with the local matrix shape known at compile time
// (every p and h pair of the ladders): fully unrolled loops over registers.
template <typename T, int KF, int KC>
__global__ void __launch_bounds__(128) transfer_prolongate_add_k(int64_t nf, const int32_t* __restrict__ parent,
                                                                 const uint8_t* __restrict__ mid,
                                                                 const uint32_t* __restrict__ owner,
                                                                 const double* __restrict__ mats,
                                                                 const int32_t* __restrict__ fdofs,
                                                                 const int32_t* __restrict__ cdofs, int64_t nc,
                                                                 const T* __restrict__ xc, T* __restrict__ xf) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nf) return;
  const uint32_t ow = __ldg(owner + c);
  if (!ow) return;
  const int64_t pc = __ldg(parent + c);
  const double* M = mats + int64_t(__ldg(mid + c)) * KF * KC;
  double xl[KC];
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    const int32_t g = __ldg(cdofs + j * nc + pc);
    xl[j] = g >= 0 ? double(__ldg(xc + g)) : 0.0;
  }
#pragma unroll
  for (int i = 0; i < KF; ++i) {
    if (!((ow >> i) & 1u)) continue;
    const int32_t g = __ldg(fdofs + i * nf + c);
    if (g < 0) continue;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < KC; ++j) acc += __ldg(M + i * KC + j) * xl[j];
    xf[g] += T(acc);
  }
}

template <typename T, int KF, int KC>
__global__ void __launch_bounds__(128) transfer_restrict_add_k(int64_t nf, const int32_t* __restrict__ parent,
                                                               const uint8_t* __restrict__ mid,
                                                               const uint32_t* __restrict__ owner,
                                                               const double* __restrict__ mats,
                                                               const int32_t* __restrict__ fdofs,
                                                               const int32_t* __restrict__ cdofs, int64_t nc,
                                                               const T* __restrict__ xf, T* __restrict__ xc) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nf) return;
  const uint32_t ow = __ldg(owner + c);
  if (!ow) return;
  const int64_t pc = __ldg(parent + c);
  const double* M = mats + int64_t(__ldg(mid + c)) * KF * KC;
  double rl[KF];
#pragma unroll
  for (int i = 0; i < KF; ++i) {
    rl[i] = 0.0;
    if ((ow >> i) & 1u) {
      const int32_t g = __ldg(fdofs + i * nf + c);
      if (g >= 0) rl[i] = double(__ldg(xf + g));
    }
  }
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    const int32_t g = __ldg(cdofs + j * nc + pc);
    if (g < 0) continue;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < KF; ++i) acc += __ldg(M + i * KC + j) * rl[i];
    if (acc != 0.0) atomicAdd(xc + g, T(acc));
  }
}

// p-transfers on one mesh (every cell is its own parent, one embedding
// matrix): the matrix travels as a kernel parameter, so the unrolled
// products read it as constant-bank operands instead of issuing a load per
// entry (the forms above spend most of their time waiting on those loads).
template <int KF, int KC>
struct XferMat {
  double m[KF * KC];
};

template <typename T, int KF, int KC>
__global__ void __launch_bounds__(128) transfer_p_prolongate_k(int64_t n, const uint32_t* __restrict__ owner,
                                                               const __grid_constant__ XferMat<KF, KC> M,
                                                               const int32_t* __restrict__ fdofs,
                                                               const int32_t* __restrict__ cdofs,
                                                               const T* __restrict__ xc, T* __restrict__ xf) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  const uint32_t ow = __ldg(owner + c);
  if (!ow) return;
  double xl[KC];
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    const int32_t g = __ldg(cdofs + j * n + c);
    xl[j] = g >= 0 ? double(__ldg(xc + g)) : 0.0;
  }
#pragma unroll
  for (int i = 0; i < KF; ++i) {
    if (!((ow >> i) & 1u)) continue;
    const int32_t g = __ldg(fdofs + i * n + c);
    if (g < 0) continue;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < KC; ++j) acc += M.m[i * KC + j] * xl[j];
    xf[g] += T(acc);
  }
}

template <typename T, int KF, int KC>
__global__ void __launch_bounds__(128) transfer_p_restrict_k(int64_t n, const uint32_t* __restrict__ owner,
                                                             const __grid_constant__ XferMat<KF, KC> M,
                                                             const int32_t* __restrict__ fdofs,
                                                             const int32_t* __restrict__ cdofs,
                                                             const T* __restrict__ xf, T* __restrict__ xc) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  const uint32_t ow = __ldg(owner + c);
  if (!ow) return;
  double rl[KF];
#pragma unroll
  for (int i = 0; i < KF; ++i) {
    rl[i] = 0.0;
    if ((ow >> i) & 1u) {
      const int32_t g = __ldg(fdofs + i * n + c);
      if (g >= 0) rl[i] = double(__ldg(xf + g));
    }
  }
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    const int32_t g = __ldg(cdofs + j * n + c);
    if (g < 0) continue;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < KF; ++i) acc += M.m[i * KC + j] * rl[i];
    if (acc != 0.0) atomicAdd(xc + g, T(acc));
  }
}

// DG p-transfer on one mesh: cell-local embedding P_{p-1} -> P_p, no sharing
// (DG/cells_batched/application_phc.cc:3396-3475 builds the same two-level
// transfer with MGTwoLevelTransfer on FE_SimplexDGP).  Layout [cell][K].
template <typename T>
__global__ void dg_p_prolongate_add(int64_t n, int Kf, int Kc, const double* __restrict__ emb,
                                    const T* __restrict__ xc, T* __restrict__ xf) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  double xl[20];
  for (int j = 0; j < Kc; ++j) xl[j] = double(xc[c * Kc + j]);
  for (int i = 0; i < Kf; ++i) {
    double acc = 0.0;
    for (int j = 0; j < Kc; ++j) acc += emb[i * Kc + j] * xl[j];
    xf[c * Kf + i] += T(acc);
  }
}

template <typename T>
__global__ void dg_p_restrict_add(int64_t n, int Kf, int Kc, const double* __restrict__ emb,
                                  const T* __restrict__ xf, T* __restrict__ xc) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  double rl[20];
  for (int i = 0; i < Kf; ++i) rl[i] = double(xf[c * Kf + i]);
  for (int j = 0; j < Kc; ++j) {
    double acc = 0.0;
    for (int i = 0; i < Kf; ++i) acc += emb[i * Kc + j] * rl[i];
    xc[c * Kc + j] += T(acc);
  }
}

// c-transfer between CG P_q and DG P_q on the same mesh
// (DG/cells_batched/application_phc.cc:3476-3552): prolongation copies the
// continuous nodal values into every cell (0 at constrained nodes),
// restriction sums the cells' values back (its transpose).
template <typename T>
__global__ void c_prolongate_add(int64_t n, int K, const int32_t* __restrict__ cdofs, const T* __restrict__ xcg,
                                 T* __restrict__ xdg) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  for (int i = 0; i < K; ++i) {
    const int32_t g = cdofs[i * n + c];
    if (g >= 0) xdg[c * K + i] += xcg[g];
  }
}

template <typename T>
__global__ void c_restrict_add(int64_t n, int K, const int32_t* __restrict__ cdofs, const T* __restrict__ xdg,
                               T* __restrict__ xcg) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n) return;
  for (int i = 0; i < K; ++i) {
    const int32_t g = cdofs[i * n + c];
    if (g >= 0) atomicAdd(xcg + g, xdg[c * K + i]);
  }
}

// basis of P_p at reference point xi
void eval_basis(int p, const double xi[3], double* out) {
  auto ev = [&](auto tag) {
    using Tb = decltype(tag);
    constexpr int NM = sizeof(Tb::MONO) / sizeof(Tb::MONO[0]);
    for (int i = 0; i < Tb::K; ++i) {
      double v = 0;
      for (int m = 0; m < NM; ++m)
        v += Tb::COEF[i][m] * std::pow(xi[0], Tb::MONO[m][0]) * std::pow(xi[1], Tb::MONO[m][1]) *
             std::pow(xi[2], Tb::MONO[m][2]);
      out[i] = v;
    }
  };
  if (p == 1) ev(ref::Tables<1>{});
  else if (p == 2) ev(ref::Tables<2>{});
  else ev(ref::Tables<3>{});
}

const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

int kuhn_type(const double f[3]) {
  int best = 0;
  for (int t = 0; t < 6; ++t)
    if (f[kPerm[t][0]] >= f[kPerm[t][1]] && f[kPerm[t][1]] >= f[kPerm[t][2]]) {
      best = t;
      break;
    }
  return best;
}

std::vector<uint32_t> owner_masks(const std::vector<int32_t>& cell_dofs, int K, int64_t n_cells, int64_t n_dofs) {
  std::vector<uint8_t> seen(n_dofs, 0);
  std::vector<uint32_t> own(n_cells, 0);
  for (int64_t c = 0; c < n_cells; ++c)
    for (int i = 0; i < K; ++i) {
      const int32_t g = cell_dofs[K * c + i];
      if (!seen[g]) {
        seen[g] = 1;
        own[c] |= 1u << i;
      }
    }
  return own;
}

// p-transfer on one mesh: P_{p-1} -> P_p through the embedding table
TransferHost make_p_transfer(const Operator& fine) {
  TransferHost t;
  const int p = fine.cfg.degree;
  t.Kf = k_of_deg(p);
  t.Kc = k_of_deg(p - 1);
  t.parent.resize(fine.n_cells);
  for (int64_t c = 0; c < fine.n_cells; ++c) t.parent[c] = int32_t(c);
  t.mat_id.assign(fine.n_cells, 0);
  t.owner = owner_masks(fine.cell_dofs, t.Kf, fine.n_cells, fine.m);
  t.mats.resize(size_t(t.Kf) * t.Kc);
  for (int i = 0; i < t.Kf; ++i)
    for (int j = 0; j < t.Kc; ++j)
      t.mats[i * t.Kc + j] = p == 2 ? ref::Tables<2>::EMB[i][j] : ref::Tables<3>::EMB[i][j];
  return t;
}

// h-transfer between nested Kuhn meshes (coarse n, fine 2n), same degree:
// every fine cell lies in one coarse cell; the coarse basis is evaluated at
// the fine nodes in the lattice (parametric) coordinates of the two grids.
TransferHost make_h_transfer(const Operator& fine, const Operator& coarse) {
  const Mesh& mf = *fine.mesh;
  const Mesh& mc = *coarse.mesh;
  const int p = fine.cfg.degree;
  TransferHost t;
  t.Kf = t.Kc = k_of_deg(p);
  for (int a = 0; a < 3; ++a)
    SFEM_REQUIRE(mf.desc.n[a] == 2 * mc.desc.n[a], FEM_ERR_ARG, "h-transfer: fine mesh must be the 2x refinement");
  // coarse cell by (hex, Kuhn type)
  const int ncx = mc.desc.n[0], ncy = mc.desc.n[1];
  std::vector<int32_t> cell_of(6 * size_t(mc.n_cells / 6), -1);
  for (int64_t c = 0; c < mc.n_cells; ++c) {
    double cen[3] = {0, 0, 0};
    for (int v = 0; v < 4; ++v) {
      const auto L = mc.vertex_lattice(mc.cell_vertices[4 * c + v]);
      for (int a = 0; a < 3; ++a) cen[a] += 0.25 * L[a];
    }
    int h[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
      h[a] = int(std::floor(cen[a]));
      f[a] = cen[a] - h[a];
    }
    const int64_t hex = h[0] + int64_t(ncx) * (h[1] + int64_t(ncy) * h[2]);
    cell_of[6 * hex + kuhn_type(f)] = int32_t(c);
  }
  t.parent.resize(mf.n_cells);
  t.mat_id.resize(mf.n_cells);
  t.owner = owner_masks(fine.cell_dofs, t.Kf, fine.n_cells, fine.m);
  using Key = std::vector<int>;
  std::map<Key, int> cache;
  const int K = t.Kf;
  for (int64_t c = 0; c < mf.n_cells; ++c) {
    std::array<int, 3> fl[4];
    double cen[3] = {0, 0, 0};
    for (int v = 0; v < 4; ++v) {
      fl[v] = mf.vertex_lattice(mf.cell_vertices[4 * c + v]);
      for (int a = 0; a < 3; ++a) cen[a] += 0.125 * fl[v][a];  // coarse units: /2
    }
    int h[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
      h[a] = int(std::floor(cen[a]));
      f[a] = cen[a] - h[a];
    }
    const int type = kuhn_type(f);
    const int64_t hex = h[0] + int64_t(ncx) * (h[1] + int64_t(ncy) * h[2]);
    const int32_t pc = cell_of[6 * hex + type];
    SFEM_REQUIRE(pc >= 0, FEM_ERR_INTERNAL, "h-transfer: parent cell not found");
    t.parent[c] = pc;
    // key: fine vertex lattice offsets and parent vertex offsets (fine units) from fine vertex 0
    Key key;
    std::array<int, 3> cl[4];
    for (int v = 0; v < 4; ++v) cl[v] = mc.vertex_lattice(mc.cell_vertices[4 * int64_t(pc) + v]);
    for (int v = 0; v < 4; ++v)
      for (int a = 0; a < 3; ++a) key.push_back(fl[v][a] - fl[0][a]);
    for (int v = 0; v < 4; ++v)
      for (int a = 0; a < 3; ++a) key.push_back(2 * cl[v][a] - fl[0][a]);
    auto it = cache.find(key);
    if (it == cache.end()) {
      SFEM_REQUIRE(cache.size() < 255, FEM_ERR_INTERNAL, "h-transfer: too many local matrices");
      const int id = int(cache.size());
      cache[key] = id;
      // Kuhn vertex order of the parent: 0, e_p0, e_p0+e_p1, 111 relative to its hex
      int kv[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 1}};
      kv[1][kPerm[type][0]] = 1;
      kv[2][kPerm[type][0]] = 1;
      kv[2][kPerm[type][1]] = 1;
      int local_of_kuhn[4];
      for (int q = 0; q < 4; ++q) {
        local_of_kuhn[q] = -1;
        for (int v = 0; v < 4; ++v)
          if (cl[v][0] == h[0] + kv[q][0] && cl[v][1] == h[1] + kv[q][1] && cl[v][2] == h[2] + kv[q][2])
            local_of_kuhn[q] = v;
        SFEM_REQUIRE(local_of_kuhn[q] >= 0, FEM_ERR_INTERNAL, "h-transfer: parent vertex mismatch");
      }
      t.mats.resize(size_t(id + 1) * K * K);
      const int* lat = nullptr;
      for (int i = 0; i < K; ++i) {
        lat = p == 1 ? ref::Tables<1>::LATTICE[i] : p == 2 ? ref::Tables<2>::LATTICE[i] : ref::Tables<3>::LATTICE[i];
        double X[3] = {0, 0, 0};  // fine node, coarse lattice units
        for (int v = 0; v < 4; ++v)
          for (int a = 0; a < 3; ++a) X[a] += double(lat[v]) / p * fl[v][a] * 0.5;
        double fr[3];
        for (int a = 0; a < 3; ++a) fr[a] = X[a] - h[a];
        const int* pm = kPerm[type];
        const double lk[4] = {1.0 - fr[pm[0]], fr[pm[0]] - fr[pm[1]], fr[pm[1]] - fr[pm[2]], fr[pm[2]]};
        double lam[4];
        for (int q = 0; q < 4; ++q) lam[local_of_kuhn[q]] = lk[q];
        const double xi[3] = {lam[1], lam[2], lam[3]};
        double phi[20];
        eval_basis(p, xi, phi);
        for (int j = 0; j < K; ++j) {
          const double v = std::fabs(phi[j]) < 1e-14 ? 0.0 : phi[j];
          t.mats[(size_t(id) * K + i) * K + j] = v;
        }
      }
      it = cache.find(key);
    }
    t.mat_id[c] = uint8_t(it->second);
  }
  return t;
}

// Mesh with n/2 hexes whose vertices are the fine mesh's vertices at even lattice points
std::unique_ptr<Mesh> coarsen_mesh(const Mesh& fine) {
  MeshDescription d = fine.desc;
  for (int a = 0; a < 3; ++a) {
    SFEM_REQUIRE(d.n[a] % 2 == 0, FEM_ERR_ARG, "multigrid: mesh size must be divisible by 2 per level");
    d.n[a] /= 2;
  }
  d.jitter = 0.0;
  auto m = std::make_unique<Mesh>(build_kuhn_mesh(d));
  for (int k = 0; k <= d.n[2]; ++k)
    for (int j = 0; j <= d.n[1]; ++j)
      for (int i = 0; i <= d.n[0]; ++i) {
        const int64_t vc = m->vertex_id(i, j, k), vf = fine.vertex_id(2 * i, 2 * j, 2 * k);
        for (int a = 0; a < 3; ++a) m->x[3 * vc + a] = fine.x[3 * vf + a];
      }
  m->desc.jitter = fine.desc.jitter;
  return m;
}

// largest eigenvalue of the symmetric tridiagonal matrix (bisection on Sturm counts)
double tridiag_max_eig(const std::vector<double>& a, const std::vector<double>& b) {
  const int n = int(a.size());
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0) + (i + 1 < n ? std::fabs(b[i]) : 0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto count_below = [&](double x) {
    int cnt = 0;
    double d = 1.0;
    for (int i = 0; i < n; ++i) {
      d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
      if (d == 0.0) d = -1e-300;
      if (d < 0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= n) hi = mid; else lo = mid;
  }
  return hi;
}

template <typename T>
class MultigridImpl final : public Multigrid {
 public:
  struct Level {
    const Mesh* mesh = nullptr;
    int kind = FEM_CG;
    // transfer from level-1: cell-based CG p/h, DG embedding, or CG -> DG
    enum { T_NONE, T_CG, T_DGP, T_C } ttype = T_NONE;
    std::unique_ptr<Operator> op;
    DevBuf<T> inv_diag, x, b, r, t, d;
    double lmax = 0, lmin = 0;
    int degree = 1;
    int hexes = 1;
    // transfer from level-1 (absent on level 0)
    int Kf = 0, Kc = 0;
    DevBuf<int32_t> parent;
    DevBuf<uint8_t> mat_id;
    DevBuf<uint32_t> owner;
    DevBuf<double> mats;
    std::vector<double> mats_host;  // p-transfers: the embedding matrix as a kernel parameter
  };
  std::vector<std::unique_ptr<Mesh>> meshes_;  // owned h-level meshes
  std::vector<Level> levels_;
  DevBuf<double> coarse_inv_;
  int coarse_n_ = 0;
  DevBuf<double> d_in_, d_out_, partial_, scal_, step_;
  DevBuf<T> cc_rhs_, cc_y_;  // coarse-correction work vectors (level below the finest)
  cudaGraph_t graph_[2] = {nullptr, nullptr};      // [0] Chebyshev, [1] learned finest level
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
  cudaStream_t cap_stream_ = nullptr;
  int64_t fine_m_ = 0;
  LearnedSmoother* learned_ = nullptr;
  bool use_learned_ = false;
  bool fallback_enabled_ = false;

  MultigridImpl(const Operator& fine, const MGParams& prm) {
    params = prm;
    SFEM_REQUIRE((fine.cfg.kind == FEM_CG || fine.cfg.kind == FEM_DG) && fine.cfg.n_components == 1 && fine.mesh,
                 FEM_ERR_ARG, "multigrid: fine operator must be CG or DG (one component)");
    SFEM_REQUIRE(prm.c_transfer == 0 || prm.c_transfer == 1, FEM_ERR_ARG, "multigrid: c_transfer must be 0 or 1");
    SFEM_REQUIRE(prm.smoother_degree >= 1 && prm.smoother_degree <= 32, FEM_ERR_ARG, "multigrid: smoother degree");
    const Mesh& mf = *fine.mesh;
    SFEM_REQUIRE(mf.structured, FEM_ERR_ARG,
                 "multigrid: the h-levels need a Kuhn box mesh (fem_mesh_create), not a mesh from arrays");
    fine_m_ = fine.m;
    // number of h-levels
    int H = 0;
    {
      int n = mf.desc.n[0];
      SFEM_REQUIRE(mf.desc.n[1] == n && mf.desc.n[2] == n, FEM_ERR_ARG, "multigrid: cubic meshes only");
      SFEM_REQUIRE(prm.coarse_n >= 1 && n % prm.coarse_n == 0, FEM_ERR_ARG, "multigrid: coarse_n must divide n");
      int r = n / prm.coarse_n;
      while (r > 1) {
        SFEM_REQUIRE(r % 2 == 0, FEM_ERR_ARG, "multigrid: n / coarse_n must be a power of 2");
        r /= 2;
        ++H;
      }
    }
    // meshes from fine (index 0) to coarsest (index H)
    std::vector<const Mesh*> mesh_of(H + 1);
    mesh_of[0] = &mf;
    for (int k = 1; k <= H; ++k) {
      meshes_.push_back(coarsen_mesh(*mesh_of[k - 1]));
      mesh_of[k] = meshes_.back().get();
    }
    const int p = fine.cfg.degree;
    const bool dg = fine.cfg.kind == FEM_DG;
    // CG ladder up to degree pc on the fine mesh, then (DG) DG levels pc .. p
    const int pc = dg && prm.c_transfer == 0 ? 1 : p;
    struct Spec {
      const Mesh* mesh;
      int degree, kind;
    };
    std::vector<Spec> seq;  // coarse -> fine
    if (prm.order == MG_ORDER_PH) {
      for (int k = H; k >= 0; --k) seq.push_back({mesh_of[k], 1, FEM_CG});
      for (int q = 2; q <= pc; ++q) seq.push_back({&mf, q, FEM_CG});
    } else {
      for (int q = 1; q <= pc; ++q) seq.push_back({mesh_of[H], q, FEM_CG});
      for (int k = H - 1; k >= 0; --k) seq.push_back({mesh_of[k], pc, FEM_CG});
    }
    if (dg)
      for (int q = pc; q <= p; ++q) seq.push_back({&mf, q, FEM_DG});
    levels_.resize(seq.size());
    OpConfig cfg;
    cfg.precision = std::is_same<T, double>::value ? FEM_FP64 : FEM_FP32;
    cfg.penalty = fine.cfg.penalty;
    for (size_t l = 0; l < seq.size(); ++l) {
      Level& L = levels_[l];
      L.mesh = seq[l].mesh;
      L.degree = seq[l].degree;
      L.kind = seq[l].kind;
      L.hexes = L.mesh->desc.n[0];
      cfg.degree = L.degree;
      cfg.kind = L.kind;
      cfg.kernel_variant = prm.tensor_cores && L.kind == FEM_CG && cfg.precision == FEM_FP32 ? 8 : 0;
      cfg.weak_bc = prm.weak_cg_levels && L.kind == FEM_CG;
      L.op = make_operator(*L.mesh, cfg);
      const int64_t m = L.op->m;
      L.inv_diag.alloc(m);
      L.x.alloc(m);
      L.b.alloc(m);
      L.r.alloc(m);
      L.t.alloc(m);
      L.d.alloc(m);
      L.op->inverse_diagonal(L.inv_diag.p, nullptr);
    }
    SFEM_REQUIRE(levels_.back().op->m == fine.m, FEM_ERR_INTERNAL, "multigrid: top level does not match the fine operator");
    // transfers
    for (size_t l = 1; l < levels_.size(); ++l) {
      Level& F = levels_[l];
      const Level& Cl = levels_[l - 1];
      if (F.kind == FEM_DG && Cl.kind == FEM_DG) {
        F.ttype = Level::T_DGP;
        F.Kf = k_of_deg(F.degree);
        F.Kc = k_of_deg(Cl.degree);
        std::vector<double> emb(size_t(F.Kf) * F.Kc);
        for (int i = 0; i < F.Kf; ++i)
          for (int j = 0; j < F.Kc; ++j)
            emb[i * F.Kc + j] = F.degree == 2 ? ref::Tables<2>::EMB[i][j] : ref::Tables<3>::EMB[i][j];
        F.mats.upload(emb);
        continue;
      }
      if (F.kind == FEM_DG) {
        SFEM_REQUIRE(Cl.kind == FEM_CG && Cl.degree == F.degree && Cl.mesh == F.mesh, FEM_ERR_INTERNAL,
                     "multigrid: c-transfer needs CG and DG of one degree on one mesh");
        F.ttype = Level::T_C;
        F.Kf = F.Kc = k_of_deg(F.degree);
        continue;
      }
      F.ttype = Level::T_CG;
      TransferHost th = F.mesh == Cl.mesh ? make_p_transfer(*F.op) : make_h_transfer(*F.op, *Cl.op);
      F.Kf = th.Kf;
      F.Kc = th.Kc;
      F.parent.upload(th.parent);
      F.mat_id.upload(th.mat_id);
      F.owner.upload(th.owner);
      F.mats.upload(th.mats);
      if (F.mesh == Cl.mesh) F.mats_host = th.mats;
    }
    partial_.alloc(kReduceBlocks);
    scal_.alloc(1);
    step_.alloc(2);
    // smoother spectra
    for (size_t l = 1; l < levels_.size(); ++l) estimate_eigenvalues(levels_[l]);
    build_coarse();
    d_in_.alloc(fine.m);
    d_out_.alloc(fine.m);
    SFEM_CUDA(cudaDeviceSynchronize());
  }

  ~MultigridImpl() override {
    for (int k = 0; k < 2; ++k) {
      if (exec_[k]) cudaGraphExecDestroy(exec_[k]);
      if (graph_[k]) cudaGraphDestroy(graph_[k]);
    }
    if (cap_stream_) cudaStreamDestroy(cap_stream_);
  }

  void set_learned(LearnedSmoother* s, bool fallback) override {
    if (s) {
      const Level& top = levels_.back();
      SFEM_REQUIRE(top.degree == 3 && top.kind == FEM_CG, FEM_ERR_ARG,
                   "learned smoother: the finest level must be CG P3");
    }
    learned_ = s;
    use_learned_ = s != nullptr;
    fallback_enabled_ = fallback;
    if (exec_[1]) {
      cudaGraphExecDestroy(exec_[1]);
      cudaGraphDestroy(graph_[1]);
      exec_[1] = nullptr;
      graph_[1] = nullptr;
    }
  }
  bool fallback_to_chebyshev() override {
    if (!use_learned_ || !fallback_enabled_) return false;
    use_learned_ = false;
    return true;
  }
  bool learned_active() const override { return use_learned_; }

  double dot(const T* x, const T* y, int64_t n, cudaStream_t s) {
    vec_dot_partial<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, x, y, partial_.p);
    reduce_partials<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, partial_.p, scal_.p);
    double h = 0;
    SFEM_CUDA(cudaMemcpyAsync(&h, scal_.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    SFEM_CUDA(cudaStreamSynchronize(s));
    return h;
  }

  // Jacobi-preconditioned CG steps give the Lanczos tridiagonal of D^-1 A
  void estimate_eigenvalues(Level& L) {
    const int64_t m = L.op->m;
    cudaStream_t s = nullptr;
    // deterministic start vector in [-1, 1], zero at constrained DoFs
    std::vector<T> h(m);
    uint64_t st = 0x9e3779b97f4a7c15ULL;
    for (int64_t i = 0; i < m; ++i) {
      st ^= st << 13;
      st ^= st >> 7;
      st ^= st << 17;
      const bool fixed = !L.op->constrained.empty() && L.op->constrained[i];
      h[i] = fixed ? T(0) : T(double(st >> 11) * (2.0 / 9007199254740992.0) - 1.0);
    }
    L.r.upload(h);  // r = b (x = 0)
    const unsigned g = grid_for(m);
    vec_scale<T><<<g, 256, 0, s>>>(m, L.inv_diag.p, L.r.p, L.d.p);  // z
    SFEM_CUDA(cudaMemcpyAsync(L.x.p, L.d.p, sizeof(T) * m, cudaMemcpyDeviceToDevice, s));  // p = z
    double rz = dot(L.r.p, L.d.p, m, s);
    std::vector<double> alpha, beta;
    for (int it = 0; it < params.eig_iterations && rz > 0; ++it) {
      L.op->vmult(L.t.p, L.x.p, s);  // q = A p
      const double pq = dot(L.x.p, L.t.p, m, s);
      if (!(pq > 0)) break;
      const double a = rz / pq;
      alpha.push_back(a);
      vec_axpby<T><<<g, 256, 0, s>>>(m, T(-a), L.t.p, T(1), L.r.p);        // r -= a q
      vec_scale<T><<<g, 256, 0, s>>>(m, L.inv_diag.p, L.r.p, L.d.p);       // z = D^-1 r
      const double rz_new = dot(L.r.p, L.d.p, m, s);
      const double bt = rz_new / rz;
      beta.push_back(bt);
      vec_axpby<T><<<g, 256, 0, s>>>(m, T(1), L.d.p, T(bt), L.x.p);       // p = z + b p
      rz = rz_new;
    }
    const int k = int(alpha.size());
    SFEM_REQUIRE(k > 0, FEM_ERR_INTERNAL, "multigrid: eigenvalue estimate failed");
    std::vector<double> da(k), ob(k > 1 ? k - 1 : 0);
    for (int i = 0; i < k; ++i) {
      da[i] = 1.0 / alpha[i] + (i > 0 ? beta[i - 1] / alpha[i - 1] : 0.0);
      if (i + 1 < k) ob[i] = std::sqrt(beta[i]) / alpha[i];
    }
    L.lmax = params.eig_safety * tridiag_max_eig(da, ob);
    L.lmin = L.lmax / params.smoothing_range;
  }

  void build_coarse() {
    const Level& L0 = levels_[0];
    OpConfig cfg = L0.op->cfg;
    cfg.precision = FEM_FP64;
    cfg.kernel_variant = 0;
    auto op64 = make_operator(*L0.mesh, cfg);
    const int n = int(op64->m);
    SFEM_REQUIRE(n <= 8192, FEM_ERR_ARG, "multigrid: coarse level too large for the dense solve");
    coarse_n_ = n;
    DevBuf<double> e(n), y(n);
    std::vector<double> A(size_t(n) * n), col(n);
    std::vector<double> unit(n, 0.0);
    for (int j = 0; j < n; ++j) {
      unit[j] = 1.0;
      e.upload(unit);
      unit[j] = 0.0;
      op64->vmult(y.p, e.p, nullptr);
      SFEM_CUDA(cudaMemcpy(col.data(), y.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
      for (int i = 0; i < n; ++i) A[size_t(i) * n + j] = col[i];
    }
    // Gauss-Jordan inverse with partial pivoting
    std::vector<double> inv(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i) inv[size_t(i) * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
      int piv = c;
      for (int r = c + 1; r < n; ++r)
        if (std::fabs(A[size_t(r) * n + c]) > std::fabs(A[size_t(piv) * n + c])) piv = r;
      SFEM_REQUIRE(std::fabs(A[size_t(piv) * n + c]) > 1e-300, FEM_ERR_INTERNAL, "multigrid: singular coarse matrix");
      if (piv != c)
        for (int k = 0; k < n; ++k) {
          std::swap(A[size_t(c) * n + k], A[size_t(piv) * n + k]);
          std::swap(inv[size_t(c) * n + k], inv[size_t(piv) * n + k]);
        }
      const double d = A[size_t(c) * n + c];
      for (int k = 0; k < n; ++k) {
        A[size_t(c) * n + k] /= d;
        inv[size_t(c) * n + k] /= d;
      }
      for (int r = 0; r < n; ++r)
        if (r != c) {
          const double f = A[size_t(r) * n + c];
          if (f == 0.0) continue;
          for (int k = 0; k < n; ++k) {
            A[size_t(r) * n + k] -= f * A[size_t(c) * n + k];
            inv[size_t(r) * n + k] -= f * inv[size_t(c) * n + k];
          }
        }
    }
    coarse_inv_.upload(inv);
  }

  int n_levels() const override { return int(levels_.size()); }
  int64_t level_m(int l) const override { return levels_.at(l).op->m; }
  int level_degree(int l) const override { return levels_.at(l).degree; }
  int level_hexes(int l) const override { return levels_.at(l).hexes; }
  double level_lambda_max(int l) const override { return levels_.at(l).lmax; }
  Operator& level_operator(int l) override { return *levels_.at(l).op; }

  void level_vmult(int l, void* dst, const void* src, cudaStream_t s) override {
    levels_.at(l).op->vmult(dst, src, s);
  }

  void smooth(int l, void* xv, const void* bv, bool zero_init, cudaStream_t s) override {
    Level& L = levels_.at(l);
    SFEM_REQUIRE(l > 0, FEM_ERR_ARG, "smooth: level 0 is solved, not smoothed");
    T* x = static_cast<T*>(xv);
    const T* b = static_cast<const T*>(bv);
    const int64_t m = L.op->m;
    const unsigned g = grid_for(m);
    const double theta = 0.5 * (L.lmax + L.lmin), delta = 0.5 * (L.lmax - L.lmin);
    double rho = delta / theta;
    if (zero_init) {
      cheb_first_zero<T><<<g, 256, 0, s>>>(m, T(1.0 / theta), L.inv_diag.p, b, L.d.p, x);
    } else {
      L.op->vmult(L.t.p, x, s);
      cheb_step<T, true><<<g, 256, 0, s>>>(m, T(0), T(1.0 / theta), L.inv_diag.p, b, L.t.p, L.d.p, x);
    }
    for (int k = 1; k < params.smoother_degree; ++k) {
      const double rho_new = 1.0 / (2.0 * theta / delta - rho);
      L.op->vmult(L.t.p, x, s);
      cheb_step<T><<<g, 256, 0, s>>>(m, T(rho_new * rho), T(2.0 * rho_new / delta), L.inv_diag.p, b, L.t.p,
                                     L.d.p, x);
      rho = rho_new;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  template <int KF, int KC>
  static XferMat<KF, KC> xfer_mat(const Level& F) {
    SFEM_REQUIRE(F.mats_host.size() == size_t(KF) * KC, FEM_ERR_INTERNAL, "multigrid: p-transfer matrix shape");
    XferMat<KF, KC> M;
    std::memcpy(M.m, F.mats_host.data(), sizeof(M.m));
    return M;
  }

  void prolongate_add(int l, void* dst, const void* src, cudaStream_t s) override {
    Level& F = levels_.at(l);
    SFEM_REQUIRE(l > 0, FEM_ERR_ARG, "prolongate: level must be >= 1");
    const Level& Cl = levels_[l - 1];
    const unsigned grid = unsigned((F.op->n_cells + 127) / 128);
    if (F.ttype == Level::T_DGP) {
      dg_p_prolongate_add<T><<<grid, 128, 0, s>>>(F.op->n_cells, F.Kf, F.Kc, F.mats.p, static_cast<const T*>(src),
                                                  static_cast<T*>(dst));
      SFEM_CUDA(cudaGetLastError());
      return;
    }
    if (F.ttype == Level::T_C) {
      c_prolongate_add<T><<<grid, 128, 0, s>>>(F.op->n_cells, F.Kf, Cl.op->device_dof_table(),
                                               static_cast<const T*>(src), static_cast<T*>(dst));
      SFEM_CUDA(cudaGetLastError());
      return;
    }
#define SFEM_PXFER(KF_, KC_)                                                                               \
  if (F.Kf == KF_ && F.Kc == KC_) {                                                                        \
    transfer_p_prolongate_k<T, KF_, KC_><<<grid, 128, 0, s>>>(                                             \
        F.op->n_cells, F.owner.p, xfer_mat<KF_, KC_>(F), F.op->device_dof_table(), Cl.op->device_dof_table(), \
        static_cast<const T*>(src), static_cast<T*>(dst));                                                 \
    SFEM_CUDA(cudaGetLastError());                                                                        \
    return;                                                                                               \
  }
    if (!F.mats_host.empty()) {
      SFEM_PXFER(20, 10) SFEM_PXFER(10, 4)
    }
#undef SFEM_PXFER
#define SFEM_XFER(KF_, KC_)                                                                                \
  if (F.Kf == KF_ && F.Kc == KC_) {                                                                        \
    transfer_prolongate_add_k<T, KF_, KC_><<<grid, 128, 0, s>>>(                                           \
        F.op->n_cells, F.parent.p, F.mat_id.p, F.owner.p, F.mats.p, F.op->device_dof_table(),               \
        Cl.op->device_dof_table(), Cl.op->n_cells, static_cast<const T*>(src), static_cast<T*>(dst));       \
    SFEM_CUDA(cudaGetLastError());                                                                        \
    return;                                                                                               \
  }
    SFEM_XFER(20, 10) SFEM_XFER(10, 4) SFEM_XFER(4, 4) SFEM_XFER(10, 10) SFEM_XFER(20, 20)
#undef SFEM_XFER
    transfer_prolongate_add<T><<<grid, 128, 0, s>>>(
        F.op->n_cells, F.Kf, F.Kc, F.parent.p, F.mat_id.p, F.owner.p, F.mats.p, F.op->device_dof_table(),
        Cl.op->device_dof_table(), Cl.op->n_cells, static_cast<const T*>(src), static_cast<T*>(dst));
    SFEM_CUDA(cudaGetLastError());
  }

  void restrict_add(int l, void* dst, const void* src, cudaStream_t s) override {
    Level& F = levels_.at(l);
    SFEM_REQUIRE(l > 0, FEM_ERR_ARG, "restrict: level must be >= 1");
    const Level& Cl = levels_[l - 1];
    const unsigned grid = unsigned((F.op->n_cells + 127) / 128);
    if (F.ttype == Level::T_DGP) {
      dg_p_restrict_add<T><<<grid, 128, 0, s>>>(F.op->n_cells, F.Kf, F.Kc, F.mats.p, static_cast<const T*>(src),
                                                static_cast<T*>(dst));
      SFEM_CUDA(cudaGetLastError());
      return;
    }
    if (F.ttype == Level::T_C) {
      c_restrict_add<T><<<grid, 128, 0, s>>>(F.op->n_cells, F.Kf, Cl.op->device_dof_table(),
                                             static_cast<const T*>(src), static_cast<T*>(dst));
      SFEM_CUDA(cudaGetLastError());
      return;
    }
#define SFEM_PXFER(KF_, KC_)                                                                               \
  if (F.Kf == KF_ && F.Kc == KC_) {                                                                        \
    transfer_p_restrict_k<T, KF_, KC_><<<grid, 128, 0, s>>>(                                               \
        F.op->n_cells, F.owner.p, xfer_mat<KF_, KC_>(F), F.op->device_dof_table(), Cl.op->device_dof_table(), \
        static_cast<const T*>(src), static_cast<T*>(dst));                                                 \
    SFEM_CUDA(cudaGetLastError());                                                                        \
    return;                                                                                               \
  }
    if (!F.mats_host.empty()) {
      SFEM_PXFER(20, 10) SFEM_PXFER(10, 4)
    }
#undef SFEM_PXFER
#define SFEM_XFER(KF_, KC_)                                                                                \
  if (F.Kf == KF_ && F.Kc == KC_) {                                                                        \
    transfer_restrict_add_k<T, KF_, KC_><<<grid, 128, 0, s>>>(                                             \
        F.op->n_cells, F.parent.p, F.mat_id.p, F.owner.p, F.mats.p, F.op->device_dof_table(),               \
        Cl.op->device_dof_table(), Cl.op->n_cells, static_cast<const T*>(src), static_cast<T*>(dst));       \
    SFEM_CUDA(cudaGetLastError());                                                                        \
    return;                                                                                               \
  }
    SFEM_XFER(20, 10) SFEM_XFER(10, 4) SFEM_XFER(4, 4) SFEM_XFER(10, 10) SFEM_XFER(20, 20)
#undef SFEM_XFER
    transfer_restrict_add<T><<<grid, 128, 0, s>>>(
        F.op->n_cells, F.Kf, F.Kc, F.parent.p, F.mat_id.p, F.owner.p, F.mats.p, F.op->device_dof_table(),
        Cl.op->device_dof_table(), Cl.op->n_cells, static_cast<const T*>(src), static_cast<T*>(dst));
    SFEM_CUDA(cudaGetLastError());
  }

  void coarse_solve(void* dst, const void* src, cudaStream_t s) override {
    dense_matvec<T><<<unsigned((coarse_n_ * 32 + 255) / 256), 256, 0, s>>>(
        coarse_n_, coarse_inv_.p, static_cast<const T*>(src), static_cast<T*>(dst));
    SFEM_CUDA(cudaGetLastError());
  }

  // b_l given, x_l = V_l(b_l)
  void cycle(int l, cudaStream_t s) {
    Level& L = levels_[l];
    if (l == 0) {
      coarse_solve(L.x.p, L.b.p, s);
      return;
    }
    const int64_t m = L.op->m;
    const unsigned g = grid_for(m);
    const bool learned = use_learned_ && l == int(levels_.size()) - 1;
    if (learned) {
      SFEM_CUDA(cudaMemsetAsync(L.x.p, 0, sizeof(T) * m, s));
      if (params.learned_steps & 1) {
        // pre-smoothing from zero: x = w z, z = S(b), w = (b,z)/(z,Az); r = b - w Az
        learned_step(L, L.b.p, s);
        residual_ratio<T><<<g, 256, 0, s>>>(m, step_.p, L.b.p, L.t.p, L.r.p);
      } else {
        SFEM_CUDA(cudaMemcpyAsync(L.r.p, L.b.p, sizeof(T) * m, cudaMemcpyDeviceToDevice, s));
      }
    } else {
      smooth(l, L.x.p, L.b.p, true, s);
      L.op->vmult(L.t.p, L.x.p, s);
      vec_residual<T><<<g, 256, 0, s>>>(m, L.b.p, L.t.p, L.r.p);
    }
    Level& C = levels_[l - 1];
    SFEM_CUDA(cudaMemsetAsync(C.b.p, 0, sizeof(T) * C.op->m, s));
    restrict_add(l, C.b.p, L.r.p, s);
    cycle(l - 1, s);
    prolongate_add(l, L.x.p, C.x.p, s);
    if (learned) {
      if (!(params.learned_steps & 2)) return;
      // post-smoothing: one energy-optimal step along S(b - A x)
      L.op->vmult(L.t.p, L.x.p, s);
      vec_residual<T><<<g, 256, 0, s>>>(m, L.b.p, L.t.p, L.r.p);
      learned_step(L, L.r.p, s);
    } else {
      smooth(l, L.x.p, L.b.p, false, s);
    }
  }

  // Learned smoothing step for residual r: z = S(r) (into L.d), A z (into L.t),
  // x += w z with the energy-optimal w = (r,z)/(z,Az); step_ keeps (r,z),(z,Az)
  // on the device so the step needs no host synchronisation (graph capturable).
  // Any direction z with (r,z) > 0 then lowers the A-norm of the error.
  void learned_step(Level& L, const T* r, cudaStream_t s) {
    const int64_t m = L.op->m;
    SFEM_CUDA(cudaMemsetAsync(L.d.p, 0, sizeof(T) * m, s));
    learned_->apply(*L.op, r, L.d.p, s);
    L.op->vmult(L.t.p, L.d.p, s);
    vec_dot_partial<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(m, r, L.d.p, partial_.p);
    reduce_partials<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, partial_.p, step_.p);
    vec_dot_partial<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(m, L.d.p, L.t.p, partial_.p);
    reduce_partials<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, partial_.p, step_.p + 1);
    axpy_ratio<T><<<grid_for(m), 256, 0, s>>>(m, step_.p, L.d.p, L.x.p);
    SFEM_CUDA(cudaGetLastError());
  }

  void on_solve_start() override { use_learned_ = learned_ != nullptr; }

  void coarse_correction(const double* r, double* x, int iterations, cudaStream_t s) override {
    const int top = int(levels_.size()) - 1;
    SFEM_REQUIRE(top >= 1, FEM_ERR_STATE, "coarse correction needs two levels");
    SFEM_REQUIRE(iterations >= 1, FEM_ERR_ARG, "coarse correction: iterations >= 1");
    Level& L = levels_[top];
    Level& C = levels_[top - 1];
    const int64_t m = L.op->m, mc = C.op->m;
    if (cc_rhs_.n != size_t(mc)) {
      cc_rhs_.alloc(mc);
      cc_y_.alloc(mc);
    }
    vec_convert<T, double><<<grid_for(m), 256, 0, s>>>(m, r, L.r.p);
    SFEM_CUDA(cudaMemsetAsync(cc_rhs_.p, 0, sizeof(T) * mc, s));
    restrict_add(top, cc_rhs_.p, L.r.p, s);
    SFEM_CUDA(cudaMemsetAsync(cc_y_.p, 0, sizeof(T) * mc, s));
    // y += V(R r - A_c y): V-cycle iteration on the level below
    for (int it = 0; it < iterations; ++it) {
      C.op->vmult(C.t.p, cc_y_.p, s);
      vec_residual<T><<<grid_for(mc), 256, 0, s>>>(mc, cc_rhs_.p, C.t.p, C.b.p);
      cycle(top - 1, s);
      vec_axpby<T><<<grid_for(mc), 256, 0, s>>>(mc, T(1), C.x.p, T(1), cc_y_.p);
    }
    SFEM_CUDA(cudaMemsetAsync(L.x.p, 0, sizeof(T) * m, s));
    prolongate_add(top, L.x.p, cc_y_.p, s);
    vec_convert<double, T><<<grid_for(m), 256, 0, s>>>(m, L.x.p, x);
    SFEM_CUDA(cudaGetLastError());
  }

  void run_cycle(cudaStream_t s) {
    Level& top = levels_.back();
    const int64_t m = top.op->m;
    vec_convert<T, double><<<grid_for(m), 256, 0, s>>>(m, d_in_.p, top.b.p);
    cycle(int(levels_.size()) - 1, s);
    vec_convert<double, T><<<grid_for(m), 256, 0, s>>>(m, top.x.p, d_out_.p);
    SFEM_CUDA(cudaGetLastError());
  }

  void vcycle(double* dst, const double* src, cudaStream_t s) override {
    SFEM_CUDA(cudaMemcpyAsync(d_in_.p, src, sizeof(double) * fine_m_, cudaMemcpyDeviceToDevice, s));
    if (params.use_graph) {
      const int mode = use_learned_ ? 1 : 0;
      if (!exec_[mode]) {
        // one eager cycle sets up kernel attributes and bindings, then capture
        run_cycle(s);
        SFEM_CUDA(cudaStreamSynchronize(s));
        if (!cap_stream_) SFEM_CUDA(cudaStreamCreateWithFlags(&cap_stream_, cudaStreamNonBlocking));
        SFEM_CUDA(cudaStreamBeginCapture(cap_stream_, cudaStreamCaptureModeThreadLocal));
        run_cycle(cap_stream_);
        SFEM_CUDA(cudaStreamEndCapture(cap_stream_, &graph_[mode]));
        SFEM_CUDA(cudaGraphInstantiate(&exec_[mode], graph_[mode], 0));
      }
      SFEM_CUDA(cudaGraphLaunch(exec_[mode], s));
    } else {
      run_cycle(s);
    }
    SFEM_CUDA(cudaMemcpyAsync(dst, d_out_.p, sizeof(double) * fine_m_, cudaMemcpyDeviceToDevice, s));
  }
};

}  // namespace

std::unique_ptr<Multigrid> make_multigrid(const Operator& fine, const MGParams& p) {
  if (p.precision == FEM_FP64) return std::make_unique<MultigridImpl<double>>(fine, p);
  SFEM_REQUIRE(p.precision == FEM_FP32, FEM_ERR_ARG, "multigrid: precision must be FEM_FP64 or FEM_FP32");
  return std::make_unique<MultigridImpl<float>>(fine, p);
}

// ------------------------------------------------------------------- PCG ----
CGSolver::CGSolver(Operator& A, Preconditioner* M, bool flexible) : A_(A), M_(M), flexible_(flexible) {
  SFEM_REQUIRE(A.cfg.precision == FEM_FP64, FEM_ERR_ARG, "cg: the outer operator must be FP64");
  const int64_t m = A.m;
  r_.alloc(m);
  z_.alloc(m);
  p_.alloc(m);
  q_.alloc(m);
  if (flexible) zold_.alloc(m);
  partial_.alloc(kReduceBlocks + 1);
  sc_.alloc(8);
  SFEM_CUDA(cudaMallocHost(&host_, 2 * sizeof(double)));
}

CGSolver::~CGSolver() {
  if (host_) cudaFreeHost(host_);
}

void CGSolver::dot_to(const double* x, const double* y, int slot, cudaStream_t s) {
  vec_dot_partial<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(A_.m, x, y, partial_.p);
  reduce_partials<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, partial_.p, sc_.p + slot);
}

double CGSolver::dot(const double* x, const double* y, cudaStream_t s) {
  vec_dot_partial<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(A_.m, x, y, partial_.p);
  reduce_partials<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, partial_.p, partial_.p + kReduceBlocks);
  SFEM_CUDA(cudaMemcpyAsync(host_, partial_.p + kReduceBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
  SFEM_CUDA(cudaStreamSynchronize(s));
  return *host_;
}

SolveInfo CGSolver::solve(double* x, const double* b, double rtol, int maxit, cudaStream_t s) {
  SolveInfo info;
  const int64_t m = A_.m;
  const unsigned g = grid_for(m);
  if (M_) M_->on_solve_start();
  // r = b - A x
  A_.vmult(q_.p, x, s);
  vec_residual<double><<<g, 256, 0, s>>>(m, b, q_.p, r_.p);
  const double bnorm = std::sqrt(dot(b, b, s));
  double rr = dot(r_.p, r_.p, s);
  info.r0 = std::sqrt(rr);
  info.rn = info.r0;
  const double target = rtol * (bnorm > 0 ? bnorm : 1.0);
  if (!std::isfinite(rr)) {
    info.status = FEM_ERR_NONFINITE;
    return info;
  }
  if (info.r0 <= target) return info;
  auto precondition = [&](double* zz, const double* rr_) {
    if (M_) M_->apply(zz, rr_, s);
    else SFEM_CUDA(cudaMemcpyAsync(zz, rr_, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
  };
  precondition(z_.p, r_.p);
  SFEM_CUDA(cudaMemcpyAsync(p_.p, z_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
  // alpha and beta stay on the device: one host read per iteration, of
  // (p,Ap) and (r,r) together, for the breakdown and convergence checks
  constexpr int kPQ = 2, kRR = 3, kRZOLD = 4;
  int cur = 0;  // slot of (r,z) of this iteration; 1 - cur: the next one
  dot_to(r_.p, z_.p, cur, s);
  double prev_rn = info.r0;
  info.status = FEM_ERR_NOT_CONVERGED;
  for (int it = 1; it <= maxit; ++it) {
    A_.vmult(q_.p, p_.p, s);
    dot_to(p_.p, q_.p, kPQ, s);
    cg_update_xr_dev<<<g, 256, 0, s>>>(m, sc_.p, cur, kPQ, p_.p, q_.p, x, r_.p);
    dot_to(r_.p, r_.p, kRR, s);
    SFEM_CUDA(cudaMemcpyAsync(host_, sc_.p + kPQ, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SFEM_CUDA(cudaStreamSynchronize(s));
    const double pq = host_[0];
    rr = host_[1];
    if (!std::isfinite(pq)) {
      info.status = FEM_ERR_NONFINITE;
      info.iterations = it;
      break;
    }
    if (!(pq > 0)) {
      info.status = FEM_ERR_BREAKDOWN;
      info.iterations = it;
      break;
    }
    info.iterations = it;
    info.rn = std::sqrt(rr);
    if (!std::isfinite(rr)) {
      info.status = FEM_ERR_NONFINITE;
      break;
    }
    if (info.rn <= target) {
      info.status = FEM_OK;
      break;
    }
    // a cycle that reduced the residual by less than 2x: fall back if the preconditioner can
    if (M_ && !info.fallback_iteration && info.rn > 0.5 * prev_rn && M_->on_poor_reduction())
      info.fallback_iteration = it;
    prev_rn = info.rn;
    if (flexible_) SFEM_CUDA(cudaMemcpyAsync(zold_.p, z_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
    precondition(z_.p, r_.p);
    dot_to(r_.p, z_.p, 1 - cur, s);
    if (flexible_) dot_to(r_.p, zold_.p, kRZOLD, s);
    // p = z + beta p, beta = (r,z)_new / (r,z), or ((r,z)_new - (r,z_old)) / (r,z)
    cg_update_p_dev<<<g, 256, 0, s>>>(m, 1.0, sc_.p, 1 - cur, flexible_ ? kRZOLD : -1, cur, z_.p, p_.p);
    cur = 1 - cur;
  }
  SFEM_CUDA(cudaGetLastError());
  return info;
}

JacobiPreconditioner::JacobiPreconditioner(Operator& A) {
  inv_.alloc(A.m);
  A.inverse_diagonal(inv_.p, nullptr);
  SFEM_CUDA(cudaDeviceSynchronize());
}

void JacobiPreconditioner::apply(double* dst, const double* src, cudaStream_t s) {
  vec_scale<double><<<grid_for(int64_t(inv_.n)), 256, 0, s>>>(int64_t(inv_.n), inv_.p, src, dst);
  SFEM_CUDA(cudaGetLastError());
}

}  // namespace sfem
