// extern "C" entry points of include/simplex_fem.h.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "autotune.hpp"
#include "host_vmult.hpp"
#include "handles.hpp"

namespace sfem {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
}  // namespace sfem

namespace {
using sfem::guarded;
#define REQUIRE_PTR(p) SFEM_REQUIRE_PTR(p)
}  // namespace

extern "C" {

const char* fem_last_error_string(void) { return sfem::last_error(); }

int fem_version(int32_t* major, int32_t* minor) {
  return guarded([&] {
    REQUIRE_PTR(major);
    REQUIRE_PTR(minor);
    *major = 0;
    *minor = 1;
  });
}

int fem_mesh_create(const fem_mesh_desc* desc, fem_mesh** out) {
  return guarded([&] {
    REQUIRE_PTR(desc);
    REQUIRE_PTR(out);
    sfem::MeshDescription d;
    for (int a = 0; a < 3; ++a) {
      d.n[a] = desc->n[a];
      d.lo[a] = desc->lo[a];
      d.hi[a] = desc->hi[a];
    }
    d.jitter = desc->jitter;
    d.seed = desc->seed;
    auto m = std::make_unique<fem_mesh>();
    m->mesh = sfem::build_kuhn_mesh(d);
    *out = m.release();
  });
}

int fem_mesh_create_from_arrays(int64_t n_vertices, const double* xyz, int64_t n_cells, const int32_t* cell_vertices,
                                int32_t reorder, fem_mesh** out) {
  return guarded([&] {
    REQUIRE_PTR(xyz);
    REQUIRE_PTR(cell_vertices);
    REQUIRE_PTR(out);
    auto m = std::make_unique<fem_mesh>();
    m->mesh = sfem::build_mesh_from_arrays(n_vertices, xyz, n_cells, cell_vertices, reorder);
    *out = m.release();
  });
}

int fem_mesh_read_vtk(const char* path, int32_t reorder, fem_mesh** out) {
  return guarded([&] {
    REQUIRE_PTR(path);
    REQUIRE_PTR(out);
    auto m = std::make_unique<fem_mesh>();
    m->mesh = sfem::read_vtk_mesh(path, reorder);
    *out = m.release();
  });
}

int fem_mesh_curve(fem_mesh* mesh, double amplitude) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    sfem::curve_mesh(mesh->mesh, amplitude);
  });
}

int fem_mesh_copy_edge_nodes(const fem_mesh* mesh, double* xyz) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(xyz);
    SFEM_REQUIRE(mesh->mesh.curved, FEM_ERR_STATE, "fem_mesh_copy_edge_nodes: the mesh is not curved");
    std::memcpy(xyz, mesh->mesh.edge_x.data(), mesh->mesh.edge_x.size() * sizeof(double));
  });
}

int fem_mesh_copy_input_cells(const fem_mesh* mesh, int64_t* input_cell) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(input_cell);
    const sfem::Mesh& m = mesh->mesh;
    for (int64_t c = 0; c < m.n_cells; ++c) input_cell[c] = m.input_cell.empty() ? c : m.input_cell[c];
  });
}

int fem_mesh_destroy(fem_mesh* mesh) {
  return guarded([&] { delete mesh; });
}

int fem_mesh_sizes(const fem_mesh* mesh, int64_t* n_vertices, int64_t* n_cells, int64_t* n_interior_faces,
                   int64_t* n_boundary_faces) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    if (n_vertices) *n_vertices = mesh->mesh.n_vertices;
    if (n_cells) *n_cells = mesh->mesh.n_cells;
    if (n_interior_faces) *n_interior_faces = mesh->mesh.n_interior_faces;
    if (n_boundary_faces) *n_boundary_faces = mesh->mesh.n_boundary_faces;
  });
}

int fem_mesh_copy_vertices(const fem_mesh* mesh, double* xyz) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(xyz);
    std::memcpy(xyz, mesh->mesh.x.data(), mesh->mesh.x.size() * sizeof(double));
  });
}

int fem_mesh_copy_cells(const fem_mesh* mesh, int32_t* cells) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(cells);
    std::memcpy(cells, mesh->mesh.cell_vertices.data(), mesh->mesh.cell_vertices.size() * sizeof(int32_t));
  });
}

int fem_mesh_copy_neighbors(const fem_mesh* mesh, int32_t* nb, int8_t* nbf) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    if (nb) std::memcpy(nb, mesh->mesh.nb.data(), mesh->mesh.nb.size() * sizeof(int32_t));
    if (nbf) std::memcpy(nbf, mesh->mesh.nbf.data(), mesh->mesh.nbf.size() * sizeof(int8_t));
  });
}

int fem_mesh_cg_dofs(const fem_mesh* mesh, int32_t degree, int64_t* n_dofs, int32_t* cell_dofs,
                     uint8_t* constrained) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(n_dofs);
    sfem::CGDofs d = sfem::build_cg_dofs(mesh->mesh, degree);
    *n_dofs = d.n_dofs;
    if (cell_dofs) std::memcpy(cell_dofs, d.cell_dofs.data(), d.cell_dofs.size() * sizeof(int32_t));
    if (constrained) std::memcpy(constrained, d.constrained.data(), d.constrained.size());
  });
}

}  // extern "C"

namespace sfem {
bool valid_variant(int kind, int v) {
  if (kind == FEM_CG) return v >= 0 && v <= 8;
  return (v >= 0 && v <= 5) || v == 7 || v == 9 || v == 11;
}

// fem_op_params -> OpConfig, with the checks of fem_op_create
OpConfig op_config(int32_t degree, int32_t kind, int32_t precision, const fem_op_params* params) {
    OpConfig cfg;
    cfg.degree = degree;
    cfg.kind = kind;
    cfg.precision = precision;
    if (kind == FEM_HELMHOLTZ) {
      cfg.mass = 1e5;
      cfg.n_components = 3;
    }
    if (params) {
      if (kind == FEM_HELMHOLTZ) {
        cfg.mass = params->mass_coefficient;
        cfg.n_components = params->n_components > 0 ? params->n_components : 3;
      } else if (kind == FEM_CG) {
        cfg.n_components = params->n_components > 0 ? params->n_components : 1;
      }
      cfg.penalty = params->penalty;
      cfg.kernel_variant = params->kernel_variant;
      SFEM_REQUIRE(params->weak_boundary == 0 || (params->weak_boundary == 1 && kind == FEM_CG), FEM_ERR_ARG,
                   "weak_boundary must be 0, or 1 for FEM_CG operators");
      cfg.weak_bc = params->weak_boundary == 1;
      SFEM_REQUIRE(valid_variant(kind, cfg.kernel_variant), FEM_ERR_ARG,
                   "kernel_variant must be 0..8 (CG) or 0..5, 7, 9, 11 (DG, Helmholtz)");
      SFEM_REQUIRE((cfg.kernel_variant != 4 && cfg.kernel_variant != 8) || kind != FEM_CG || precision == FEM_FP32,
                   FEM_ERR_ARG, "CG kernel_variant 4 and 8 (TF32 tensor cores) are for FP32 operators");
      SFEM_REQUIRE(cfg.penalty == FEM_PENALTY_REFERENCE || cfg.penalty == FEM_PENALTY_SQUARE, FEM_ERR_ARG,
                   "penalty must be FEM_PENALTY_REFERENCE or FEM_PENALTY_SQUARE");
    }
    return cfg;
}
}  // namespace sfem

extern "C" {

int fem_op_create(fem_mesh* mesh, int32_t degree, int32_t kind, int32_t precision, const fem_op_params* params,
                  fem_op** out) {
  return guarded([&] {
    REQUIRE_PTR(mesh);
    REQUIRE_PTR(out);
    const sfem::OpConfig cfg = sfem::op_config(degree, kind, precision, params);
    auto o = std::make_unique<fem_op>();
    o->op = sfem::make_operator(mesh->mesh, cfg);
    *out = o.release();
  });
}

int fem_op_element_matrices(fem_op* op, void* mats, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(mats);
    op->op->element_matrices(mats, static_cast<cudaStream_t>(stream));
  });
}

int fem_csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col, const void* val, const void* x, void* y,
                 int32_t precision, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(row_ptr);
    REQUIRE_PTR(col);
    REQUIRE_PTR(val);
    REQUIRE_PTR(x);
    REQUIRE_PTR(y);
    SFEM_REQUIRE(n_rows >= 0, FEM_ERR_ARG, "fem_csr_spmv: n_rows must be >= 0");
    SFEM_REQUIRE(precision == FEM_FP64 || precision == FEM_FP32, FEM_ERR_ARG, "fem_csr_spmv: bad precision");
    SFEM_REQUIRE(x != y, FEM_ERR_ARG, "fem_csr_spmv: x and y must not alias");
    sfem::csr_spmv(n_rows, row_ptr, col, val, x, y, precision, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_destroy(fem_op* op) {
  return guarded([&] { delete op; });
}

int fem_op_m(const fem_op* op, uint64_t* m) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(m);
    *m = uint64_t(op->op->m);
  });
}

int fem_op_info(const fem_op* op, int32_t* degree, int32_t* kind, int32_t* precision, int32_t* dofs_per_cell,
                int64_t* n_cells, int32_t* n_components) {
  return guarded([&] {
    REQUIRE_PTR(op);
    const auto& o = *op->op;
    if (degree) *degree = o.cfg.degree;
    if (kind) *kind = o.cfg.kind;
    if (precision) *precision = o.cfg.precision;
    if (dofs_per_cell) *dofs_per_cell = o.K;
    if (n_cells) *n_cells = o.n_cells;
    if (n_components) *n_components = o.cfg.n_components;
  });
}

int fem_op_copy_dof_map(const fem_op* op, int32_t* cell_dofs) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(cell_dofs);
    const auto& o = *op->op;
    if (o.cfg.kind == FEM_CG) {
      std::memcpy(cell_dofs, o.cell_dofs.data(), o.cell_dofs.size() * sizeof(int32_t));
    } else {
      const int64_t nk = int64_t(o.K) * o.cfg.n_components;
      for (int64_t c = 0; c < o.n_cells; ++c)
        for (int64_t i = 0; i < nk; ++i) cell_dofs[c * nk + i] = int32_t(c * nk + i);
    }
  });
}

int fem_op_copy_constrained(const fem_op* op, uint8_t* mask) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(mask);
    std::memcpy(mask, op->op->constrained.data(), op->op->constrained.size());
  });
}

int fem_op_copy_support_points(const fem_op* op, double* xyz) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(xyz);
    std::memcpy(xyz, op->op->support.data(), op->op->support.size() * sizeof(double));
  });
}

int fem_op_vmult(fem_op* op, void* dst, const void* src, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(dst);
    REQUIRE_PTR(src);
    SFEM_REQUIRE(dst != src, FEM_ERR_ARG, "vmult: dst and src must not alias");
    op->op->vmult(dst, src, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_vmult_phase(fem_op* op, void* dst, const void* src, int32_t phase, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(dst);
    REQUIRE_PTR(src);
    SFEM_REQUIRE(phase == 1 || phase == 2, FEM_ERR_ARG, "vmult_phase: phase must be 1 or 2");
    op->op->vmult_phase(dst, src, phase, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_Tvmult(fem_op* op, void* dst, const void* src, void* stream) {
  return fem_op_vmult(op, dst, src, stream);
}

int fem_op_compute_inverse_diagonal(fem_op* op, void* diag, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(diag);
    op->op->inverse_diagonal(diag, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_compute_diagonal(fem_op* op, void* diag, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(diag);
    op->op->diagonal(diag, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_vmult_host(fem_op* op, int32_t n, void* const* dst_host, const void* const* src_host, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(dst_host);
    REQUIRE_PTR(src_host);
    sfem::vmult_host(*op->op, n, dst_host, src_host, static_cast<cudaStream_t>(stream));
  });
}

int fem_op_set_kernel_variant(fem_op* op, int32_t variant) {
  return guarded([&] {
    REQUIRE_PTR(op);
    SFEM_REQUIRE(sfem::valid_variant(op->op->cfg.kind, variant), FEM_ERR_ARG,
                 "kernel_variant must be 0..8 (CG) or 0..5, 7, 9, 11 (DG, Helmholtz)");
    SFEM_REQUIRE((variant != 4 && variant != 8) || op->op->cfg.kind != FEM_CG || op->op->cfg.precision == FEM_FP32,
                 FEM_ERR_ARG, "CG kernel_variant 4 and 8 (TF32 tensor cores) are for FP32 operators");
    op->op->cfg.kernel_variant = variant;
  });
}

int fem_op_work(const fem_op* op, double* flops, double* bytes) {
  return guarded([&] {
    REQUIRE_PTR(op);
    double f = 0, b = 0;
    op->op->work(f, b);
    if (flops) *flops = f;
    if (bytes) *bytes = b;
  });
}

int fem_op_status(fem_op* op, int32_t* status) {
  return guarded([&] {
    REQUIRE_PTR(op);
    REQUIRE_PTR(status);
    *status = op->op->status(true);
  });
}

int fem_batch_create(fem_op* const* ops, int32_t n_ops, fem_batch** out) {
  return guarded([&] {
    REQUIRE_PTR(ops);
    REQUIRE_PTR(out);
    std::vector<sfem::Operator*> v;
    for (int i = 0; i < n_ops; ++i) {
      REQUIRE_PTR(ops[i]);
      v.push_back(ops[i]->op.get());
    }
    auto b = std::make_unique<fem_batch>();
    b->batch = sfem::make_batch(v);
    *out = b.release();
  });
}

int fem_batch_destroy(fem_batch* batch) {
  return guarded([&] { delete batch; });
}

int fem_op_autotune(fem_op* op, int32_t reps, int32_t use_cache, int32_t* variant, int32_t* cached,
                    double* us) {
  return guarded([&] {
    REQUIRE_PTR(op);
    const sfem::TuneResult r = sfem::autotune(*op->op, reps, use_cache != 0);
    if (variant) *variant = r.variant;
    if (cached) *cached = r.cached ? 1 : 0;
    if (us)
      for (int i = 0; i < 8; ++i) us[i] = i < int(r.us.size()) ? r.us[i] : 0.0;
  });
}

int fem_batch_autotune(fem_batch* batch, int32_t reps, int32_t use_cache, int32_t* variant, int32_t* cached,
                       double* us) {
  return guarded([&] {
    REQUIRE_PTR(batch);
    const sfem::TuneResult r = batch->batch->tune(reps, use_cache != 0);
    if (variant) *variant = r.variant;
    if (cached) *cached = r.cached ? 1 : 0;
    if (us)
      for (int i = 0; i < 8; ++i) us[i] = i < int(r.us.size()) ? r.us[i] : 0.0;
  });
}

int fem_batch_set_kernel_variant(fem_batch* batch, int32_t variant) {
  return guarded([&] {
    REQUIRE_PTR(batch);
    batch->batch->set_variant(variant);
  });
}

int fem_autotune_cache(const char* path) {
  return guarded([&] { sfem::tune_set_cache_file(path ? std::string(path) : std::string()); });
}

int fem_batch_vmult(fem_batch* batch, void* const* dst, const void* const* src, void* stream) {
  return guarded([&] {
    REQUIRE_PTR(batch);
    REQUIRE_PTR(dst);
    REQUIRE_PTR(src);
    batch->batch->vmult(dst, src, static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
