// Right-hand side assembly b_i = (f, phi_i) on the GPU.
//
// Replaces Operator::rhs / rhs_range (CG/cells_batched/application_ph.cc:
// 1361-1367,1435-1458): the reference integrates its analytic load with
// FEEvaluation at QGaussSimplex(p+1) points; here every cell integrates the
// load with a collapsed Gauss-Legendre rule of p+3 points per direction
// (exact for polynomials of degree 2p+3) and scatters into the DoFs,
// skipping constrained ones (CG) as deal.II's integrate_scatter does.
#include <cmath>
#include <vector>

#include "operator.hpp"
#include "ref_tables.h"

namespace sfem {

double rhs_value(const RhsDesc& r, const double* x) {
  double f = 0.0;
  for (int m = 0; m < r.n_modes; ++m) {
    if (r.kind == 0) {
      f += r.amp[m] * std::sin(r.k[m][0] * x[0] + r.k[m][1] * x[1] + r.k[m][2] * x[2]);
    } else {
      f += r.amp[m] * std::sin(r.k[m][0] * x[0]) * std::sin(r.k[m][1] * x[1]) * std::sin(r.k[m][2] * x[2]);
    }
  }
  return f;
}

namespace {

constexpr int kMaxQ = 6 * 6 * 6;

struct RhsTables {
  int nq;
  double w[kMaxQ];
  double xi[kMaxQ][3];
  double phi[kMaxQ][20];
};

// Gauss-Legendre points and weights on [0,1] (Newton on the Legendre recurrence)
void gauss_legendre01(int n, double* t, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) p0 = 1.0;
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    t[i] = 0.5 * (1.0 - z);
    w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

template <int P>
void basis_values(const double xi[3], double* phi) {
  using Tb = ref::Tables<P>;
  constexpr int NM = sizeof(Tb::MONO) / sizeof(Tb::MONO[0]);
  for (int i = 0; i < Tb::K; ++i) {
    double v = 0;
    for (int m = 0; m < NM; ++m)
      v += Tb::COEF[i][m] * std::pow(xi[0], Tb::MONO[m][0]) * std::pow(xi[1], Tb::MONO[m][1]) *
           std::pow(xi[2], Tb::MONO[m][2]);
    phi[i] = v;
  }
}

RhsTables make_tables(int p) {
  RhsTables t{};
  const int n = p + 3;
  double g[8], gw[8];
  gauss_legendre01(n, g, gw);
  int q = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c) {
        const double u = g[a], v = g[b], s = g[c];
        t.xi[q][0] = u;
        t.xi[q][1] = v * (1 - u);
        t.xi[q][2] = s * (1 - u) * (1 - v);
        t.w[q] = gw[a] * gw[b] * gw[c] * (1 - u) * (1 - u) * (1 - v);
        if (p == 1) basis_values<1>(t.xi[q], t.phi[q]);
        else if (p == 2) basis_values<2>(t.xi[q], t.phi[q]);
        else basis_values<3>(t.xi[q], t.phi[q]);
        ++q;
      }
  t.nq = q;
  return t;
}

__global__ void rhs_kernel(int64_t n_cells, int K, int NC, const double* __restrict__ x,
                           const int32_t* __restrict__ cells, const int32_t* __restrict__ idx /* [n][K] or null */,
                           const RhsTables* __restrict__ tab, const RhsDesc rd, double* __restrict__ b) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= n_cells) return;
  double x0[3], J[3][3];
  const int32_t* cv = cells + 4 * c;
  for (int d = 0; d < 3; ++d) x0[d] = x[3 * int64_t(cv[0]) + d];
  for (int j = 0; j < 3; ++j)
    for (int d = 0; d < 3; ++d) J[d][j] = x[3 * int64_t(cv[j + 1]) + d] - x0[d];
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double loc[20];
  for (int i = 0; i < K; ++i) loc[i] = 0.0;
  for (int q = 0; q < tab->nq; ++q) {
    double X[3];
    for (int d = 0; d < 3; ++d) X[d] = x0[d] + J[d][0] * tab->xi[q][0] + J[d][1] * tab->xi[q][1] + J[d][2] * tab->xi[q][2];
    double f = 0.0;
    for (int m = 0; m < rd.n_modes; ++m) {
      if (rd.kind == 0)
        f += rd.amp[m] * sin(rd.k[m][0] * X[0] + rd.k[m][1] * X[1] + rd.k[m][2] * X[2]);
      else
        f += rd.amp[m] * sin(rd.k[m][0] * X[0]) * sin(rd.k[m][1] * X[1]) * sin(rd.k[m][2] * X[2]);
    }
    const double wf = tab->w[q] * fabs(det) * f;
    for (int i = 0; i < K; ++i) loc[i] += wf * tab->phi[q][i];
  }
  if (idx) {
    for (int i = 0; i < K; ++i) {
      const int32_t g = idx[c * K + i];
      if (g >= 0) atomicAdd(b + g, loc[i]);
    }
  } else {
    for (int comp = 0; comp < NC; ++comp)
      for (int i = 0; i < K; ++i) b[(c * NC + comp) * K + i] = loc[i];
  }
}

template <typename To>
__global__ void convert_out(int64_t n, const double* in, To* out) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = To(in[i]);
}

}  // namespace

void Operator::rhs(const RhsDesc& rd, void* dst, cudaStream_t s) {
  SFEM_REQUIRE(mesh != nullptr, FEM_ERR_STATE, "rhs: operator has no mesh");
  SFEM_REQUIRE(rd.n_modes >= 0 && rd.n_modes <= 16, FEM_ERR_ARG, "rhs: 0..16 modes");
  const RhsTables tab = make_tables(cfg.degree);
  DevBuf<RhsTables> d_tab(1);
  d_tab.upload(&tab, 1);
  DevBuf<double> d_x;
  d_x.upload(mesh->x);
  DevBuf<int32_t> d_cells;
  d_cells.upload(mesh->cell_vertices);
  DevBuf<int32_t> d_idx;
  if (cfg.kind == FEM_CG) {
    std::vector<int32_t> idx(cell_dofs.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = constrained[cell_dofs[i]] ? -1 : cell_dofs[i];
    d_idx.upload(idx);
  }
  DevBuf<double> b(m);
  SFEM_CUDA(cudaMemsetAsync(b.p, 0, sizeof(double) * m, s));
  rhs_kernel<<<unsigned((n_cells + 127) / 128), 128, 0, s>>>(n_cells, K, cfg.n_components, d_x.p, d_cells.p,
                                                             d_idx.p, d_tab.p, rd, b.p);
  SFEM_CUDA(cudaGetLastError());
  if (cfg.precision == FEM_FP64) {
    SFEM_CUDA(cudaMemcpyAsync(dst, b.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
  } else {
    convert_out<float><<<unsigned((m + 255) / 256), 256, 0, s>>>(m, b.p, static_cast<float*>(dst));
    SFEM_CUDA(cudaGetLastError());
  }
  // temporaries are freed when this returns: finish using them first
  SFEM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace sfem
