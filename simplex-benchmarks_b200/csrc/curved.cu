// Curvilinear (non-affine) CG Laplace operator on quadratic geometry.
//
// The reference keeps a per-quadrature-point Jacobian for cells that are not
// affine and applies  JxW_q J_q^-1 J_q^-T  at every point
// (CG/cells_batched/application.cc:1361-1376; deal.II's MappingFE on a
// manifold, e.g. use_manifold in DG/components_batched/application.cc:1547).
// Here a curved mesh (fem_mesh_curve) carries a P2 geometry per cell: its 4
// vertices and 6 edge nodes.  The operator stores, per cell and quadrature
// point q, the symmetric metric G_q = w_q |det J_q| J_q^-1 J_q^-T (6 values),
// and one thread per cell runs gather -> for each q: reference gradients
// (D_q, dense [3][K]), metric, transposed gradients -> atomic scatter.  On
// curved cells the integrand is not a polynomial, so the quadrature is part
// of the operator: collapsed Gauss-Legendre (Stroud conical product) with
// p + 1 points per direction, (p + 1)^3 per cell.
#include <cmath>
#include <memory>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "kernels_cg.cuh"
#include "operator.hpp"
#include "ref_tables.h"

namespace sfem {
namespace {

inline unsigned grid_for(int64_t n, int bs) { return unsigned((std::max<int64_t>(n, 1) + bs - 1) / bs); }

template <int P, typename T>
__global__ void __launch_bounds__(128) cg_curved_kernel(int64_t n_cells, int nq, const int32_t* __restrict__ dofs,
                                                        const T* __restrict__ gq, const T* __restrict__ D,
                                                        const T* __restrict__ src, T* __restrict__ dst,
                                                        int64_t n_constrained, const int32_t* __restrict__ constrained) {
  constexpr int K = gen::Ops<P>::K;
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c < n_constrained) {
    const int32_t i = constrained[c];
    dst[i] = src[i];
  }
  if (c >= n_cells) return;
  int32_t idx[K];
  T u[K], y[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    idx[i] = __ldg(dofs + i * n_cells + c);
    u[i] = idx[i] >= 0 ? __ldg(src + idx[i]) : T(0);
    y[i] = T(0);
  }
  for (int q = 0; q < nq; ++q) {
    const T* Dq = D + q * 3 * K;  // the same address in every lane: broadcast loads
    T g0 = T(0), g1 = T(0), g2 = T(0);
#pragma unroll
    for (int i = 0; i < K; ++i) {
      g0 += __ldg(Dq + i) * u[i];
      g1 += __ldg(Dq + K + i) * u[i];
      g2 += __ldg(Dq + 2 * K + i) * u[i];
    }
    T G[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) G[k] = __ldg(gq + (int64_t(q) * 6 + k) * n_cells + c);
    const T w0 = G[0] * g0 + G[3] * g1 + G[4] * g2;
    const T w1 = G[3] * g0 + G[1] * g1 + G[5] * g2;
    const T w2 = G[4] * g0 + G[5] * g1 + G[2] * g2;
#pragma unroll
    for (int i = 0; i < K; ++i) y[i] += __ldg(Dq + i) * w0 + __ldg(Dq + K + i) * w1 + __ldg(Dq + 2 * K + i) * w2;
  }
#pragma unroll
  for (int i = 0; i < K; ++i)
    if (idx[i] >= 0) atomicAdd(dst + idx[i], y[i]);
}

template <int P, typename T>
__global__ void __launch_bounds__(128) cg_curved_diagonal_kernel(int64_t n_cells, int nq,
                                                                 const int32_t* __restrict__ dofs,
                                                                 const T* __restrict__ gq, const T* __restrict__ D,
                                                                 T* __restrict__ dst, int64_t n_constrained,
                                                                 const int32_t* __restrict__ constrained) {
  constexpr int K = gen::Ops<P>::K;
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c < n_constrained) dst[constrained[c]] = T(1);
  if (c >= n_cells) return;
  for (int i = 0; i < K; ++i) {
    const int32_t gi = dofs[i * n_cells + c];
    if (gi < 0) continue;
    T s = T(0);
    for (int q = 0; q < nq; ++q) {
      const T* Dq = D + q * 3 * K;
      const T a = Dq[i], b = Dq[K + i], e = Dq[2 * K + i];
      const T* G = gq;
      const int64_t o = int64_t(q) * 6;
      const T G0 = G[(o + 0) * n_cells + c], G1 = G[(o + 1) * n_cells + c], G2 = G[(o + 2) * n_cells + c];
      const T G3 = G[(o + 3) * n_cells + c], G4 = G[(o + 4) * n_cells + c], G5 = G[(o + 5) * n_cells + c];
      s += a * (G0 * a + G3 * b + G4 * e) + b * (G3 * a + G1 * b + G5 * e) + e * (G4 * a + G5 * b + G2 * e);
    }
    atomicAdd(dst + gi, s);
  }
}

// Gauss-Legendre nodes and weights on [0, 1] (Newton on the three-term
// recurrence of the Legendre polynomials)
void gauss_legendre(int n, std::vector<double>& t, std::vector<double>& w) {
  t.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 200; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) {
        p0 = 1.0;
        p1 = z;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
      const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = pk;
    }
    if (n == 1) p0 = 1.0;
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    t[i] = 0.5 * (1.0 - z);
    w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

// gradients of the P_q Lagrange basis at xi, grad[i][d]
template <int Q>
void basis_grad(const double xi[3], std::vector<double>& grad) {
  using Tb = ref::Tables<Q>;
  constexpr int NM = sizeof(Tb::MONO) / sizeof(Tb::MONO[0]);
  grad.assign(3 * Tb::K, 0.0);
  for (int i = 0; i < Tb::K; ++i)
    for (int m = 0; m < NM; ++m) {
      const double cf = Tb::COEF[i][m];
      if (cf == 0.0) continue;
      const int e[3] = {Tb::MONO[m][0], Tb::MONO[m][1], Tb::MONO[m][2]};
      for (int d = 0; d < 3; ++d) {
        if (e[d] == 0) continue;
        double v = cf * e[d];
        for (int a = 0; a < 3; ++a) v *= std::pow(xi[a], a == d ? e[a] - 1 : e[a]);
        grad[3 * i + d] += v;
      }
    }
}

template <typename T>
class CGCurvedOperator final : public Operator {
 public:
  DevBuf<int32_t> d_dofs;         // [K][n_cells], -1 = constrained
  DevBuf<T> d_gq;                 // [nq][6][n_cells]
  DevBuf<T> d_D;                  // [nq][3][K] reference gradients at the points
  DevBuf<int32_t> d_constrained;
  int nq = 0;

  CGCurvedOperator(const Mesh& mesh, const OpConfig& c) {
    cfg = c;
    const int p = cfg.degree;
    SFEM_REQUIRE(mesh.curved && int64_t(mesh.edge_x.size()) == 18 * mesh.n_cells, FEM_ERR_INTERNAL,
                 "curved operator: mesh has no edge geometry");
    const CGDofs dofs = build_cg_dofs(mesh, p);
    K = dofs.K;
    n_cells = mesh.n_cells;
    m = dofs.n_dofs;
    n_interior_faces = mesh.n_interior_faces;
    n_boundary_faces = mesh.n_boundary_faces;
    cell_dofs = dofs.cell_dofs;
    constrained = dofs.constrained;
    support = dofs.support;
    std::vector<int32_t> idx(size_t(K) * n_cells), cl;
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int i = 0; i < K; ++i) {
        const int32_t g = dofs.cell_dofs[K * cc + i];
        idx[size_t(i) * n_cells + cc] = dofs.constrained[g] ? -1 : g;
      }
    for (int64_t i = 0; i < m; ++i)
      if (constrained[i]) cl.push_back(int32_t(i));
    d_dofs.upload(idx);
    d_constrained.upload(cl);
    // collapsed Gauss-Legendre rule, p + 1 points per direction
    const int n1 = p + 1;
    std::vector<double> t, w;
    gauss_legendre(n1, t, w);
    std::vector<std::array<double, 3>> xq;
    std::vector<double> wq;
    for (int a = 0; a < n1; ++a)
      for (int b = 0; b < n1; ++b)
        for (int e = 0; e < n1; ++e) {
          const double u = t[a], v = t[b], s = t[e];
          xq.push_back({u, v * (1 - u), s * (1 - u) * (1 - v)});
          wq.push_back(w[a] * w[b] * w[e] * (1 - u) * (1 - u) * (1 - v));
        }
    nq = int(xq.size());
    // reference gradients of the solution basis (P_p) and the geometry basis (P2)
    std::vector<T> D(size_t(nq) * 3 * K);
    std::vector<double> gs, gg;
    std::vector<std::vector<double>> geo_grad(nq);
    for (int q = 0; q < nq; ++q) {
      if (p == 1) basis_grad<1>(xq[q].data(), gs);
      else if (p == 2) basis_grad<2>(xq[q].data(), gs);
      else basis_grad<3>(xq[q].data(), gs);
      for (int i = 0; i < K; ++i)
        for (int d = 0; d < 3; ++d) D[(size_t(q) * 3 + d) * K + i] = T(gs[3 * i + d]);
      basis_grad<2>(xq[q].data(), geo_grad[q]);
    }
    d_D.upload(D);
    std::vector<T> gqh(size_t(nq) * 6 * n_cells);
#pragma omp parallel for schedule(static)
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      // geometry nodes in the P2 node order: vertices, then edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
      double X[10][3];
      for (int v = 0; v < 4; ++v)
        for (int a = 0; a < 3; ++a) X[v][a] = mesh.x[3 * int64_t(mesh.cell_vertices[4 * cc + v]) + a];
      for (int e = 0; e < 6; ++e)
        for (int a = 0; a < 3; ++a) X[4 + e][a] = mesh.edge_x[18 * cc + 3 * e + a];
      for (int q = 0; q < nq; ++q) {
        double J[3][3] = {};
        for (int k = 0; k < 10; ++k)
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) J[i][j] += X[k][i] * geo_grad[q][3 * k + j];
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        double Ji[3][3];
        const double id = 1.0 / det;
        Ji[0][0] = c00 * id;
        Ji[1][0] = c01 * id;
        Ji[2][0] = c02 * id;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
        static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
        for (int k = 0; k < 6; ++k) {
          double s = 0;
          for (int e = 0; e < 3; ++e) s += Ji[ia[k]][e] * Ji[ib[k]][e];
          gqh[(size_t(q) * 6 + k) * n_cells + cc] = T(wq[q] * std::fabs(det) * s);
        }
      }
    }
    d_gq.upload(gqh);
  }

  void vmult(void* dst, const void* src, cudaStream_t s) override {
    vmult_phase(dst, src, 1, s);
    vmult_phase(dst, src, 2, s);
  }

  void vmult_phase(void* dst, const void* src, int phase, cudaStream_t s) override {
    T* d = static_cast<T*>(dst);
    const T* x = static_cast<const T*>(src);
    if (phase == 1) {
      SFEM_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * m, s));
      return;
    }
    const unsigned grid = grid_for(std::max<int64_t>(n_cells, int64_t(d_constrained.n)), 128);
    switch (cfg.degree) {
      case 1: cg_curved_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, x, d, d_constrained.n, d_constrained.p); break;
      case 2: cg_curved_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, x, d, d_constrained.n, d_constrained.p); break;
      case 3: cg_curved_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, x, d, d_constrained.n, d_constrained.p); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  void diagonal(void* diag, cudaStream_t s) override {
    T* d = static_cast<T*>(diag);
    SFEM_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * m, s));
    const unsigned grid = grid_for(std::max<int64_t>(n_cells, int64_t(d_constrained.n)), 128);
    switch (cfg.degree) {
      case 1: cg_curved_diagonal_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, d, d_constrained.n, d_constrained.p); break;
      case 2: cg_curved_diagonal_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, d, d_constrained.n, d_constrained.p); break;
      case 3: cg_curved_diagonal_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, nq, d_dofs.p, d_gq.p, d_D.p, d, d_constrained.n, d_constrained.p); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  const int32_t* device_dof_table() const override { return d_dofs.p; }

  void rhs(const RhsDesc&, void*, cudaStream_t) override {
    throw Error(FEM_ERR_ARG, "rhs: not provided on curved meshes");
  }

  void work(double& flops, double& bytes) const override {
    flops = 2.0 * nq * (6.0 * K + 15.0) * double(n_cells);
    const double sz = double(sizeof(T));
    bytes = 2 * sz * double(m) + 4.0 * K * double(n_cells) + 6.0 * nq * sz * double(n_cells);
  }
};

}  // namespace

std::unique_ptr<Operator> make_curved_cg_operator(const Mesh& mesh, const OpConfig& cfg) {
  SFEM_REQUIRE(cfg.n_components == 1 && !cfg.weak_bc, FEM_ERR_ARG,
               "curved meshes: scalar CG with strong constraints only");
  SFEM_REQUIRE(cfg.kernel_variant == 0 || cfg.kernel_variant == 1, FEM_ERR_ARG,
               "curved meshes: the per-quadrature-point cell kernel only");
  if (cfg.precision == FEM_FP64) return std::make_unique<CGCurvedOperator<double>>(mesh, cfg);
  return std::make_unique<CGCurvedOperator<float>>(mesh, cfg);
}

}  // namespace sfem
