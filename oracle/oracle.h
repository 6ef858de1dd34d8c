/*
 * oracle.h - CPU restatement of the reference's matrix-free operators.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (libsimplexfem.so) never links or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load liboracle.so, as the checker.
 *
 * Parity status: UNPINNED against the reference itself.  The reference's
 * arithmetic lives in deal.II (FEEvaluation / FEFaceEvaluation, git revision
 * 5037bf40bd, README.md:29), which is not vendored and cannot be built here
 * (no deal.II, Trilinos or MPI), and the reference ships no golden vectors or
 * tests.  The oracle is pinned instead by known-answer tests derived from the
 * mathematics (tests/golden/make_golden.py: exact rational element matrices,
 * constant/linear null spaces, symmetry) and by two different quadrature
 * rules agreeing to rounding.
 *
 * What it restates (generic deal.II path, FEEvaluation semantics):
 *   CG Laplace:  CG/cells_batched/application.cc:1206-1234 (cell integral),
 *                :1154-1163 (constrained rows = identity, masked gather),
 *                :1333-1360 (affine metric J^-1 J^-T |J| w_q)
 *   DG SIPG:     DG/cells_batched/application.cc:1349-1490 (cell, face, boundary),
 *                :1191-1245 (penalty (p+1)(p+d)/d * surface/volume, max of both sides)
 *   Helmholtz:   DG/components_batched/application_helmholtz.cc:611-632 (mass 1e5 +
 *                Laplace), :672-733 (face, sigma from 1/h normal to the face),
 *                :841-882 (boundary)
 * with quadrature in physical space (face points are generated from one
 * side and mapped into the other cell by inverting its affine map), so no
 * face orientation convention is shared with the product.
 */
#ifndef SFEM_ORACLE_H
#define SFEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_CG 0
#define ORACLE_DG 1
#define ORACLE_HELMHOLTZ 2

typedef struct oracle_params {
  int32_t degree;       /* 1..3 */
  int32_t kind;         /* ORACLE_CG / ORACLE_DG / ORACLE_HELMHOLTZ */
  int32_t n_components; /* DG/Helmholtz: fields per cell (DoF layout [cell][comp][k]) */
  int32_t penalty;      /* 0: (p+1)(p+3)/3, 1: (p+1)^2 */
  double mass;          /* Helmholtz mass coefficient */
  int32_t quad_points;  /* Gauss points per collapsed direction (0: degree + 2) */
  int32_t n_threads;    /* OpenMP threads (0: all) */
  int32_t weak_bc;      /* CG: weak (Nitsche) homogeneous Dirichlet on boundary faces, no constrained
                           DoFs (the CG levels of DG/cells_batched/application_phc.cc:1799-1832) */
} oracle_params;

typedef struct oracle_ctx oracle_ctx;

/* cell_dofs/constrained/n_dofs are used for CG only (cell_dofs [n_cells][k]). */
int oracle_create(const oracle_params* prm, int64_t n_vertices, const double* x, int64_t n_cells,
                  const int32_t* cells, const int32_t* cell_dofs, const uint8_t* constrained,
                  int64_t n_dofs, oracle_ctx** out);
void oracle_destroy(oracle_ctx* ctx);
int64_t oracle_n_dofs(const oracle_ctx* ctx);
/* dst = A src */
int oracle_vmult(oracle_ctx* ctx, const double* src, double* dst);
/* the contributions of cells [c0, c1) only (DG: their DoF blocks; CG: dst is
 * zeroed, then those cells scatter) - a bounded sample for timing */
int oracle_vmult_cells(oracle_ctx* ctx, const double* src, double* dst, int64_t c0, int64_t c1);
/* diagonal of A (constrained CG rows: 1) */
int oracle_diagonal(oracle_ctx* ctx, double* diag);
/* dense element matrix of cell c (own-cell terms only, no neighbour coupling),
 * k*nc x k*nc row-major */
int oracle_cell_matrix(oracle_ctx* ctx, int64_t c, double* mat);
/* CG numbering check: every global DoF must map to one physical point from
 * every cell that references it, and be constrained iff it lies on the box
 * boundary.  Returns the number of violations (0 = consistent). */
int64_t oracle_check_cg_numbering(oracle_ctx* ctx, const double* lo, const double* hi);
/* reference basis value / gradient (for known-answer tests) */
int oracle_basis(int32_t degree, const double* xi, double* values, double* grads);
/* The benchmark mesh, restated independently of the product (mesh.c): Kuhn
 * tets of an n[0] x n[1] x n[2] hex box in Morton hex order, vertices
 * jittered from an MT19937-64 stream.  Caller-allocated outputs:
 * x [(n0+1)(n1+1)(n2+1)][3], cells/nb/nbf [6 n0 n1 n2][4].  Returns 0 on success. */
int oracle_kuhn_mesh(const int32_t n[3], const double lo[3], const double hi[3], double jitter, uint64_t seed,
                     double* x, int32_t* cells, int32_t* nb, int8_t* nbf);
/* First-touch continuous P_degree numbering and Dirichlet mask of a mesh with
 * sorted cell vertices.  Returns n_dofs (negative on error); with cell_dofs ==
 * NULL only counts.  cell_dofs [n_cells][k], constrained [n_dofs]. */
int64_t oracle_cg_numbering(int64_t n_vertices, int64_t n_cells, const int32_t* cells, const int32_t* nb,
                            int32_t degree, int32_t* cell_dofs, uint8_t* constrained);
/* CG on curved cells: quadratic geometry from the cells' vertices and their
 * edge nodes [n_cells][6][3] (edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3));
 * the cell integrals then use the Jacobian at every quadrature point
 * (CG/cells_batched/application.cc:1361-1376). */
int oracle_set_p2_geometry(oracle_ctx* ctx, const double* edge_nodes);
/* quadrature sizes actually used */
int oracle_quadrature_sizes(const oracle_ctx* ctx, int32_t* n_cell_points, int32_t* n_face_points);

#ifdef __cplusplus
}
#endif
#endif
