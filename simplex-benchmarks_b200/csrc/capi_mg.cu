// extern "C" entry points: loads, multigrid hierarchy, preconditioned CG.
#include <cstring>
#include <vector>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "handles.hpp"

namespace {
using sfem::guarded;

sfem::RhsDesc to_desc(const fem_rhs_desc* f) {
  SFEM_REQUIRE(f->n_modes >= 0 && f->n_modes <= 16, FEM_ERR_ARG, "rhs: n_modes must be 0..16");
  SFEM_REQUIRE(f->kind == FEM_RHS_PLANE_WAVES || f->kind == FEM_RHS_SINE_PRODUCTS, FEM_ERR_ARG, "rhs: bad kind");
  sfem::RhsDesc d;
  d.kind = f->kind;
  d.n_modes = f->n_modes;
  for (int m = 0; m < 16; ++m) {
    d.amp[m] = f->amp[m];
    for (int a = 0; a < 3; ++a) d.k[m][a] = f->k[m][a];
  }
  return d;
}
}  // namespace

extern "C" {

int fem_op_rhs(fem_op* op, const fem_rhs_desc* f, void* dst, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(op);
    SFEM_REQUIRE_PTR(f);
    SFEM_REQUIRE_PTR(dst);
    op->op->rhs(to_desc(f), dst, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_interpolate(fem_op* op, const fem_rhs_desc* f, void* dst, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(op);
    SFEM_REQUIRE_PTR(f);
    SFEM_REQUIRE_PTR(dst);
    const sfem::RhsDesc d = to_desc(f);
    const sfem::Operator& o = *op->op;
    const int nc = o.cfg.n_components;
    const int64_t npts = o.m / nc;
    std::vector<double> v(o.m);
    const int K = o.K;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < npts; ++i) {
      const double val = sfem::rhs_value(d, &o.support[3 * i]);
      if (o.cfg.kind == FEM_CG) {
        v[i] = val;
      } else {
        const int64_t c = i / K, loc = i % K;
        for (int comp = 0; comp < nc; ++comp) v[(c * nc + comp) * K + loc] = val;
      }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (o.cfg.precision == FEM_FP64) {
      SFEM_CUDA(cudaMemcpyAsync(dst, v.data(), sizeof(double) * o.m, cudaMemcpyHostToDevice, s));
    } else {
      std::vector<float> w(v.begin(), v.end());
      SFEM_CUDA(cudaMemcpyAsync(dst, w.data(), sizeof(float) * o.m, cudaMemcpyHostToDevice, s));
      SFEM_CUDA(cudaStreamSynchronize(s));
    }
    SFEM_CUDA(cudaStreamSynchronize(s));
  });
}

int fem_mg_params_default(fem_mg_params* p) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(p);
    std::memset(p, 0, sizeof(*p));
    sfem::MGParams d;
    p->order = d.order;
    p->precision = d.precision;
    p->smoother_degree = d.smoother_degree;
    p->eig_iterations = d.eig_iterations;
    p->smoothing_range = d.smoothing_range;
    p->eig_safety = d.eig_safety;
    p->coarse_n = d.coarse_n;
    p->use_graph = d.use_graph;
    p->c_transfer = d.c_transfer;
    p->learned_steps = d.learned_steps;
    p->tensor_cores = d.tensor_cores;
    p->weak_cg_levels = d.weak_cg_levels;
  });
}

int fem_mg_create(fem_op* fine, const fem_mg_params* p, fem_mg** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(fine);
    SFEM_REQUIRE_PTR(out);
    sfem::MGParams prm;
    if (p) {
      prm.order = p->order;
      prm.precision = p->precision;
      prm.smoother_degree = p->smoother_degree;
      prm.eig_iterations = p->eig_iterations;
      prm.smoothing_range = p->smoothing_range;
      prm.eig_safety = p->eig_safety;
      prm.coarse_n = p->coarse_n;
      prm.use_graph = p->use_graph;
      prm.c_transfer = p->c_transfer;
      prm.learned_steps = p->learned_steps;
      prm.tensor_cores = p->tensor_cores;
      prm.weak_cg_levels = p->weak_cg_levels;
    }
    SFEM_REQUIRE(prm.weak_cg_levels == 0 || (prm.weak_cg_levels == 1 && fine->op->cfg.kind == FEM_DG), FEM_ERR_ARG,
                 "mg: weak_cg_levels must be 0, or 1 for a FEM_DG fine operator");
    SFEM_REQUIRE(prm.learned_steps >= 1 && prm.learned_steps <= 3, FEM_ERR_ARG, "mg: learned_steps must be 1..3");
    SFEM_REQUIRE(prm.order == FEM_MG_PH || prm.order == FEM_MG_HP, FEM_ERR_ARG, "mg: order must be PH or HP");
    SFEM_REQUIRE(prm.eig_iterations >= 1 && prm.smoothing_range > 1 && prm.eig_safety >= 1, FEM_ERR_ARG,
                 "mg: bad smoother parameters");
    auto h = std::make_unique<fem_mg>();
    h->mg = sfem::make_multigrid(*fine->op, prm);
    *out = h.release();
  });
}

int fem_mg_destroy(fem_mg* mg) {
  return guarded([&] { delete mg; });
}

int fem_mg_n_levels(const fem_mg* mg, int32_t* n) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    SFEM_REQUIRE_PTR(n);
    *n = mg->mg->n_levels();
  });
}

int fem_mg_level_info(const fem_mg* mg, int32_t level, uint64_t* m, int32_t* degree, int32_t* hexes,
                      double* lambda_max) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    SFEM_REQUIRE(level >= 0 && level < mg->mg->n_levels(), FEM_ERR_ARG, "mg: level out of range");
    if (m) *m = uint64_t(mg->mg->level_m(level));
    if (degree) *degree = mg->mg->level_degree(level);
    if (hexes) *hexes = mg->mg->level_hexes(level);
    if (lambda_max) *lambda_max = mg->mg->level_lambda_max(level);
  });
}

int fem_mg_level_kind(const fem_mg* mg, int32_t level, int32_t* kind) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    SFEM_REQUIRE_PTR(kind);
    SFEM_REQUIRE(level >= 0 && level < mg->mg->n_levels(), FEM_ERR_ARG, "mg: level out of range");
    *kind = mg->mg->level_operator(level).cfg.kind;
  });
}

int fem_mg_vcycle(fem_mg* mg, double* dst, const double* src, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    SFEM_REQUIRE_PTR(dst);
    SFEM_REQUIRE_PTR(src);
    mg->mg->vcycle(dst, src, static_cast<cudaStream_t>(stream));
  });
}

#define MG_LEVEL_CHECK(lo)                                                                          \
  SFEM_REQUIRE_PTR(mg);                                                                             \
  SFEM_REQUIRE(level >= (lo) && level < mg->mg->n_levels(), FEM_ERR_ARG, "mg: level out of range")

int fem_mg_level_vmult(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream) {
  return guarded([&] {
    MG_LEVEL_CHECK(0);
    mg->mg->level_vmult(level, dst, src, static_cast<cudaStream_t>(stream));
  });
}

int fem_mg_smooth(fem_mg* mg, int32_t level, void* x, const void* b, int32_t zero_initial, void* stream) {
  return guarded([&] {
    MG_LEVEL_CHECK(1);
    mg->mg->smooth(level, x, b, zero_initial != 0, static_cast<cudaStream_t>(stream));
  });
}

int fem_mg_prolongate_add(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream) {
  return guarded([&] {
    MG_LEVEL_CHECK(1);
    mg->mg->prolongate_add(level, dst, src, static_cast<cudaStream_t>(stream));
  });
}

int fem_mg_restrict_add(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream) {
  return guarded([&] {
    MG_LEVEL_CHECK(1);
    mg->mg->restrict_add(level, dst, src, static_cast<cudaStream_t>(stream));
  });
}

int fem_mg_coarse_solve(fem_mg* mg, void* dst, const void* src, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    mg->mg->coarse_solve(dst, src, static_cast<cudaStream_t>(stream));
  });
}

int fem_cg_create(fem_op* op, fem_mg* mg, int32_t precond, int32_t flexible, fem_cg** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(op);
    SFEM_REQUIRE_PTR(out);
    auto h = std::make_unique<fem_cg>();
    sfem::Preconditioner* P = nullptr;
    if (precond == FEM_PRECOND_MG) {
      SFEM_REQUIRE_PTR(mg);
      SFEM_REQUIRE(mg->mg->level_m(mg->mg->n_levels() - 1) == op->op->m, FEM_ERR_ARG,
                   "cg: multigrid was built for another operator");
      h->own_precond = std::make_unique<sfem::MGPreconditioner>(*mg->mg);
      P = h->own_precond.get();
    } else if (precond == FEM_PRECOND_JACOBI) {
      h->own_precond = std::make_unique<sfem::JacobiPreconditioner>(*op->op);
      P = h->own_precond.get();
    } else {
      SFEM_REQUIRE(precond == FEM_PRECOND_NONE, FEM_ERR_ARG, "cg: unknown preconditioner");
    }
    h->solver = std::make_unique<sfem::CGSolver>(*op->op, P, flexible != 0);
    *out = h.release();
  });
}

int fem_cg_destroy(fem_cg* cg) {
  return guarded([&] { delete cg; });
}

int fem_cg_solve(fem_cg* cg, double* x, const double* b, double rtol, int32_t max_iterations,
                 fem_solve_info* info, void* stream) {
  int status = FEM_OK;
  const int rc = guarded([&] {
    SFEM_REQUIRE_PTR(cg);
    SFEM_REQUIRE_PTR(x);
    SFEM_REQUIRE_PTR(b);
    SFEM_REQUIRE(rtol > 0 && max_iterations > 0, FEM_ERR_ARG, "cg: rtol and max_iterations must be positive");
    const sfem::SolveInfo si = cg->solver->solve(x, b, rtol, max_iterations, static_cast<cudaStream_t>(stream));
    if (info) {
      info->iterations = si.iterations;
      info->status = si.status;
      info->initial_residual = si.r0;
      info->final_residual = si.rn;
      info->fallback_iteration = si.fallback_iteration;
      info->reserved = 0;
    }
    status = si.status;
  });
  if (rc != FEM_OK) return rc;
  if (status != FEM_OK) sfem::set_last_error("cg: not converged (see fem_solve_info.status)");
  return status;
}

}  // extern "C"
