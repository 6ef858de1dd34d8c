/*
 * simplex_fem.h - C ABI of the B200 matrix-free tetrahedral FEM engine.
 *
 * The functions below replace the operator / preconditioner / solver
 * interface that the reference benchmark programs build on deal.II:
 *
 *   Operator<dim,Number>            CG/cells_batched/application.cc:1040-1582
 *                                   DG/cells_batched/application.cc:1156-2858
 *                                   DG/components_batched/application_helmholtz.cc:434-1765
 *   MultigridPreconditioner         CG/cells_batched/application_ph.cc:1754-2023
 *                                   DG/cells_batched/application_phc.cc:3396-3667
 *   SolverCG + PreconditionMG       CG/cells_batched/application_ph.cc:1949-1980
 *
 * Conventions
 *   - Every function returns an int status: FEM_OK (0) or one of FEM_ERR_*.
 *     fem_last_error_string() gives the message of the last failure on the
 *     calling thread.
 *   - Handles are opaque.  A handle is not thread-safe; use one stream per
 *     handle at a time.
 *   - Vector arguments are DEVICE pointers (cudaMalloc'd by the caller or by
 *     fem_vector_alloc) of the operator's number type (double for FEM_FP64,
 *     float for FEM_FP32) and length m().  `stream` is a cudaStream_t passed
 *     as void* (NULL = legacy default stream).
 *   - The library owns the device memory it allocates for meshes, operators,
 *     multigrid hierarchies and solvers; the caller owns vectors.
 *   - Host-copy functions (fem_*_copy_*) write into caller-provided host
 *     buffers and exist for inspection and testing.
 */
#ifndef SIMPLEX_FEM_H
#define SIMPLEX_FEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FEM_OK 0
#define FEM_ERR_ARG 1            /* invalid argument */
#define FEM_ERR_CUDA 2           /* a CUDA runtime call failed */
#define FEM_ERR_STATE 3          /* call not valid in the handle's state */
#define FEM_ERR_NOT_CONVERGED 4  /* iterative solver hit its iteration limit */
#define FEM_ERR_BREAKDOWN 5      /* CG breakdown: p^T A p <= 0 */
#define FEM_ERR_NONFINITE 6      /* NaN/Inf met in a residual or dot product */
#define FEM_ERR_INTERNAL 7

/* ---- enums ------------------------------------------------------------- */
enum fem_kind {
  FEM_CG = 0,        /* continuous Lagrange, Laplace, homogeneous Dirichlet (strong) */
  FEM_DG = 1,        /* discontinuous Lagrange, SIPG Laplace, weak Dirichlet */
  FEM_HELMHOLTZ = 2  /* DG, n_components fields, mass + SIPG Laplace */
};
enum fem_precision { FEM_FP64 = 0, FEM_FP32 = 1 };
enum fem_penalty {
  FEM_PENALTY_REFERENCE = 0, /* (p+1)(p+d)/d * surface/volume (DG/cells_batched/application.cc:1193-1245) */
  FEM_PENALTY_SQUARE = 1     /* (p+1)^2 * surface/volume */
};

typedef struct fem_mesh fem_mesh;
typedef struct fem_op fem_op;
typedef struct fem_batch fem_batch;
typedef struct fem_mg fem_mg;
typedef struct fem_mlp fem_mlp;

/* Kuhn-subdivided box: n[0]*n[1]*n[2] hexes x 6 tets, interior vertices
 * jittered by U[-jitter*h, jitter*h] per axis from std::mt19937_64(seed).
 * Replaces GridGenerator::subdivided_hyper_cube_with_simplices +
 * refine_global (CG/cells_batched/application.cc:1762-1770). */
typedef struct fem_mesh_desc {
  int32_t n[3];
  double lo[3];
  double hi[3];
  double jitter;
  uint64_t seed;
} fem_mesh_desc;

typedef struct fem_op_params {
  double mass_coefficient; /* FEM_HELMHOLTZ: factor of the mass term (reference: 1e5) */
  int32_t n_components;    /* FEM_HELMHOLTZ: number of fields (reference: 3); others: 1 */
  int32_t penalty;         /* FEM_DG: enum fem_penalty */
  int32_t kernel_variant;  /* 0: tuned default; DG/Helmholtz: 1 thread per cell x128 cells per
                              CTA, 2 thread per cell x64, 3 warp roles x32, 4 thread per cell
                              x64 with results in registers (scalar) and 8 CTAs per SM, 5 thread
                              per cell x64 with 5 CTAs per SM; CG: 1 thread per
                              cell, 2 thread per Kuhn hex (6 tets, one atomic per distinct
                              DoF), 3 CTA per 4x4x4-hex Morton cube (stores for cube-interior
                              DoFs); each falls back to the next simpler form where the mesh
                              lacks the pattern; default P1 3 (FP64) / 2 (FP32), P2 3, P3 3;
                              4: FP32 CG on the TF32 tensor cores (tcgen05 kind::tf32, cell
                              operator as one [128 cells x K] x [K x 6K] product; ~1e-3
                              relative accuracy, for multigrid levels); CG 5, 6, 7: the cube
                              kernel (3) with its DoF reduction read in contribution order
                              (5), bank-scheduled with the same steps per warp (6) or
                              bank-scheduled with per-lane steps (7); 3 takes the fastest
                              measured on B200 (6 for FP64 P1 and P2, else 5); CG 8:
                              FP32 on the TF32 tensor cores per cube (the cube kernel
                              with each tile of 128 tets as one tcgen05 product;
                              variant 4 on meshes without whole cubes) */
  int32_t weak_boundary;   /* FEM_CG: 1 = weak (Nitsche) homogeneous Dirichlet on the boundary
                              faces (2 sigma u v - d_n u v - u d_n v, sigma = (p+1)(p+3)/3 *
                              surface/volume) and no constrained DoFs, as the CG levels of the
                              reference's DG multigrid (DG/cells_batched/application_phc.cc:
                              1799-1832); 0 = strong constraints (default) */
  int32_t reserved[4];
} fem_op_params;

/* ---- library ----------------------------------------------------------- */
const char* fem_last_error_string(void);
int fem_version(int32_t* major, int32_t* minor);

/* ---- mesh -------------------------------------------------------------- */
int fem_mesh_create(const fem_mesh_desc* desc, fem_mesh** out);
/* Unstructured tetrahedral mesh from arrays (the reference reads one with
 * GridIn::read_vtk and reorders it with SparsityTools::reorder_hierarchical,
 * CG/cells_batched/application.cc:1696-1757).  Cells may list their vertices
 * in any order (stored sorted by vertex id; orientation does not matter).
 * reorder = 1: cells in Morton order of their centroids (the hierarchical
 * order the kernels' locality relies on); 0: input order.  Degenerate cells,
 * vertex ids out of range and faces shared by more than two cells are
 * FEM_ERR_ARG.  Such meshes take the per-cell kernels; multigrid needs a
 * Kuhn box (fem_mesh_create). */
int fem_mesh_create_from_arrays(int64_t n_vertices, const double* xyz /* [n_vertices][3] */, int64_t n_cells,
                                const int32_t* cell_vertices /* [n_cells][4] */, int32_t reorder, fem_mesh** out);
/* The same from a legacy ASCII VTK unstructured grid of tetrahedra (VTK cell type 10). */
int fem_mesh_read_vtk(const char* path, int32_t reorder, fem_mesh** out);
/* Curvilinear geometry (the reference's non-affine cells, MappingFE on a
 * manifold: CG/cells_batched/application.cc:1361-1376,
 * DG/components_batched/application.cc:1547): every point x of the mesh's
 * bounding box moves to x + amplitude * prod_d sin(pi xi_d) * (hi - lo), xi in
 * [0,1]^3 the box coordinates (the box boundary stays), and every cell gets a
 * quadratic geometry (its moved vertices and moved edge midpoints).  FEM_CG
 * operators on a curved mesh apply a per-quadrature-point metric (collapsed
 * Gauss-Legendre rule, p + 1 points per direction); DG / Helmholtz operators,
 * partitions and multigrid need affine meshes.  |amplitude| < 0.5; an
 * amplitude that inverts a cell is FEM_ERR_ARG. */
int fem_mesh_curve(fem_mesh* mesh, double amplitude);
/* edge geometry nodes of a curved mesh, [n_cells][6][3] in the edge order
 * (0,1),(0,2),(0,3),(1,2),(1,3),(2,3) of the sorted cell vertices */
int fem_mesh_copy_edge_nodes(const fem_mesh* mesh, double* xyz);
/* input index of every cell of a mesh from arrays (identity for Kuhn meshes) */
int fem_mesh_copy_input_cells(const fem_mesh* mesh, int64_t* input_cell /* [n_cells] */);
int fem_mesh_destroy(fem_mesh* mesh);
int fem_mesh_sizes(const fem_mesh* mesh, int64_t* n_vertices, int64_t* n_cells,
                   int64_t* n_interior_faces, int64_t* n_boundary_faces);
int fem_mesh_copy_vertices(const fem_mesh* mesh, double* xyz /* [n_vertices][3] */);
int fem_mesh_copy_cells(const fem_mesh* mesh, int32_t* cell_vertices /* [n_cells][4] */);
int fem_mesh_copy_neighbors(const fem_mesh* mesh, int32_t* nb /* [n_cells][4] */,
                            int8_t* nb_face /* [n_cells][4] */);

/* Host-only continuous P_degree numbering of the mesh (first touch in the
 * hierarchical cell order) and its homogeneous Dirichlet mask; no GPU needed.
 * Call with cell_dofs == NULL and constrained == NULL to query n_dofs.
 * Replaces DoFHandler::distribute_dofs + DoFRenumbering::matrix_free_data_locality
 * + VectorTools::interpolate_boundary_values (CG/cells_batched/application.cc:1809-1838). */
int fem_mesh_cg_dofs(const fem_mesh* mesh, int32_t degree, int64_t* n_dofs,
                     int32_t* cell_dofs /* [n_cells][dofs_per_cell] */,
                     uint8_t* constrained /* [n_dofs] */);

/* ---- operator ------------------------------------------------------------
 * fem_op_create replaces Operator::reinit (CG/cells_batched/application.cc:1056-1128,
 * DG/cells_batched/application.cc:1170-1277, application_helmholtz.cc:450-510).
 * CG operators keep ones on the constrained diagonal (reinit(..., true),
 * CG/cells_batched/application.cc:1842). */
int fem_op_create(fem_mesh* mesh, int32_t degree, int32_t kind, int32_t precision,
                  const fem_op_params* params /* may be NULL */, fem_op** out);
int fem_op_destroy(fem_op* op);
/* Operator::m() (CG/cells_batched/application.cc:1131-1139) */
int fem_op_m(const fem_op* op, uint64_t* m);
int fem_op_info(const fem_op* op, int32_t* degree, int32_t* kind, int32_t* precision,
                int32_t* dofs_per_cell, int64_t* n_cells, int32_t* n_components);
/* CG: global DoF of local node i of cell c, [n_cells][dofs_per_cell];
 * DG: the identity layout c*n_components*dofs_per_cell + comp*dofs_per_cell + i. */
int fem_op_copy_dof_map(const fem_op* op, int32_t* cell_dofs);
int fem_op_copy_constrained(const fem_op* op, uint8_t* mask /* [m] */);
int fem_op_copy_support_points(const fem_op* op, double* xyz /* [m/n_components][3] */);
/* Operator::vmult_masked_gather / vmult_manual / vmult
 * (CG/cells_batched/application.cc:1167-1176, DG/cells_batched/application.cc:1319-1332,
 * application_helmholtz.cc:567-580): dst = A src.  dst and src must not alias. */
int fem_op_vmult(fem_op* op, void* dst, const void* src, void* stream);
/* dst_host[i] = A src_host[i] for i < n, on vectors in HOST memory (the
 * reference's Operator::vmult on deal.II host vectors,
 * CG/cells_batched/application.cc:1154-1176, DG/cells_batched/
 * application.cc:1303-1316): each src is copied to the device, the operator
 * applied and dst copied back.  Enqueued on `stream` (asynchronous: the host
 * buffers must stay valid, and dst is ready, when the stream passes the
 * call).  The operator keeps two device staging pairs (4 x m values, made by
 * the first call) and its own copy-in, compute and copy-out streams, so with
 * pinned host memory the copy-in of vector i+1, the apply of vector i and the
 * copy-out of vector i-1 overlap.  Pageable host memory works, with copies
 * that do not overlap. */
int fem_op_vmult_host(fem_op* op, int32_t n, void* const* dst_host, const void* const* src_host, void* stream);
/* Same product as fem_op_vmult for FEM_DG / FEM_HELMHOLTZ operators, with
 * the face-trace scratch taken from a 16 MiB static device array inside this
 * library instead of the operator's own buffer.  No counterpart in the
 * reference.  The call allocates nothing (nor does fem_op_vmult at the call;
 * fem_op_create allocates the operator's tables and its own scratch once).
 * It serves callers that cannot call cudaMalloc where they set up per-apply
 * working memory (a framework's memory pool owns the device): every apply
 * through it shares the one library-owned array.  The array is held on every
 * GPU that loads the library, until exit, whether or not the call is used.
 * Operators needing more scratch are rejected with FEM_ERR_ARG (DG P3 FP64:
 * up to 87,296 cells).  All calls share the array, so calls that overlap on
 * the GPU race; order them on one stream.  Each call outside stream capture
 * looks up the array's device address; a call under capture reuses the last
 * one, so make one call on the device before capturing. */
int fem_op_vmult_static_scratch(fem_op* op, void* dst, const void* src, void* stream);
/* Operator::Tvmult (CG/cells_batched/application.cc:1193-1197): the operator is symmetric. */
int fem_op_Tvmult(fem_op* op, void* dst, const void* src, void* stream);
/* Operator::compute_inverse_diagonal (CG/cells_batched/application_ph.cc:1382-1404):
 * 1/diag, 1 where |diag| < 1e-10. */
int fem_op_compute_inverse_diagonal(fem_op* op, void* inv_diag, void* stream);
/* MatrixFreeTools::compute_diagonal / Operator::get_diagonal
 * (application_helmholtz.cc:588-600). */
int fem_op_compute_diagonal(fem_op* op, void* diag, void* stream);
/* One phase of vmult, for per-kernel timing: CG phase 1 zeroes dst and
 * phase 2 runs the fused cell kernel; DG/Helmholtz phase 1 publishes the
 * face normal derivatives and phase 2 runs the fused cell+face kernel.
 * Running phase 1 then phase 2 equals fem_op_vmult. */
int fem_op_vmult_phase(fem_op* op, void* dst, const void* src, int32_t phase, void* stream);
/* Switch the kernel form of an existing operator (same meaning as
 * fem_op_params.kernel_variant); used by the autotuner.  No counterpart in
 * the reference (deal.II picks its vectorisation at compile time). */
int fem_op_set_kernel_variant(fem_op* op, int32_t variant);
/* ---- assembled-matrix comparison -----------------------------------------
 * The reference compares its matrix-free vmult with a Trilinos sparse
 * matrix-vector product on the same DoFs (CG/cells_batched/application.cc:
 * 1944-1988).  fem_op_element_matrices writes the dense cell matrices of a
 * FEM_CG operator to device memory [n_cells][K][K] (operator precision,
 * unconstrained; the caller assembles them with fem_op_copy_dof_map and the
 * constrained mask: constrained rows and columns dropped, ones on their
 * diagonal).  fem_csr_spmv is y = A x for a device CSR matrix (row_ptr int64
 * [n_rows + 1], col int32, val and vectors in `precision`). */
int fem_op_element_matrices(fem_op* op, void* mats, void* stream);
int fem_csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col, const void* val, const void* x,
                 void* y, int32_t precision, void* stream);
/* Algorithmic work of one vmult: flops and bytes of the fused kernels. */
int fem_op_work(const fem_op* op, double* flops, double* bytes);
/* Device-side status of the operator's kernels since the last call, then
 * cleared: bit 0 = a kernel gave up on a bounded wait (a tensor-core CG
 * kernel, or the bulk-copy trace pass of a DG / Helmholtz operator); that
 * vmult's result is invalid.  Synchronises with the device.  No counterpart
 * in the reference (its kernels have no bounded waits). */
int fem_op_status(fem_op* op, int32_t* status);

/* ---- domain decomposition (one rank per GPU) -----------------------------
 * Replaces the reference's distributed triangulation with a z-order
 * partition (parallel::fullydistributed::Triangulation,
 * CG/cells_batched/application.cc:1773-1801) and the ghost handling of its
 * MPI-distributed vectors inside MatrixFree::cell_loop / loop
 * (update_ghost_values before, compress(add) after; DG/cells_batched/
 * application.cc:1303-1316).  Part r of n_parts owns a contiguous range of
 * the hierarchical cell order (cut at 4x4x4-hex cubes or hexes when possible).
 * Its local vectors hold [owned entries | ghost entries]: CG DoFs (a DoF
 * belongs to the part of the first cell touching it) or DG cell blocks (the
 * ghosts are the face neighbours of the part's cells).  For each peer, the
 * send list (local indices of owned entries the peer holds as ghosts) and the
 * receive list (local indices of ghosts the peer owns) are in ascending
 * global index, so they match entry by entry.  Before each vmult the caller
 * copies send -> peer's recv (ghost update); after a CG vmult it adds the
 * ghost entries back into their owners' entries along the same lists
 * (compress) and may clear them.  The partition itself is host-only. */
typedef struct fem_part fem_part;
int fem_part_create(const fem_mesh* mesh, int32_t degree, int32_t kind, int32_t n_components, int32_t n_parts,
                    int32_t part, fem_part** out);
int fem_part_destroy(fem_part* part);
int fem_part_sizes(const fem_part* part, int64_t* n_owned, int64_t* n_ghost, int64_t* n_global,
                   int64_t* cell_begin, int64_t* cell_end, int32_t* n_peers);
/* global vector index of every local entry, [n_owned + n_ghost] */
int fem_part_global_index(const fem_part* part, int64_t* gidx);
/* peer i (ascending rank): its rank and the lengths of its send / receive lists */
int fem_part_peer(const fem_part* part, int32_t i, int32_t* rank, int64_t* n_send, int64_t* n_recv);
int fem_part_halo(const fem_part* part, int32_t i, int64_t* send /* [n_send] */, int64_t* recv /* [n_recv] */);
/* The part's local operator on its local vectors (m() = n_owned + n_ghost):
 * the owned rows of dst are the global operator's rows once the ghosts of src
 * are up to date (CG: after the compress); DG ghost rows hold no meaning.
 * The partition may be destroyed afterwards. */
int fem_op_create_part(const fem_part* part, int32_t precision, const fem_op_params* params, fem_op** out);

/* ---- loads --------------------------------------------------------------
 * f(x) = sum_m amp[m] sin(k[m] . x)           (kind FEM_RHS_PLANE_WAVES)
 *      = sum_m amp[m] prod_d sin(k[m][d] x_d)  (kind FEM_RHS_SINE_PRODUCTS) */
enum { FEM_RHS_PLANE_WAVES = 0, FEM_RHS_SINE_PRODUCTS = 1 };
typedef struct fem_rhs_desc {
  int32_t kind;
  int32_t n_modes; /* <= 16 */
  double k[16][3];
  double amp[16];
} fem_rhs_desc;
/* Operator::rhs (CG/cells_batched/application_ph.cc:1361-1367,1435-1458):
 * dst_i = (f, phi_i); 0 on constrained CG DoFs; every DG component gets f. */
int fem_op_rhs(fem_op* op, const fem_rhs_desc* f, void* dst, void* stream);
/* nodal interpolant of f (VectorTools::interpolate; reference error checks
 * application_ph.cc:2210-2213) */
int fem_op_interpolate(fem_op* op, const fem_rhs_desc* f, void* dst, void* stream);

/* ---- hybrid multigrid ----------------------------------------------------
 * MultigridPreconditioner (CG/cells_batched/application_ph.cc:1754-2023):
 * levels P1 on the coarsest mesh .. P1 on the fine mesh, then P2 .. Pp
 * (FEM_MG_PH, application_ph.cc) or P1 .. Pp on the coarsest mesh, then Pp on
 * finer meshes (FEM_MG_HP, application_hp.cc:1819-1843); Chebyshev-Jacobi
 * smoothing; dense FP64 coarse solve; optional CUDA-graph V-cycle.  The fine
 * operator must be FEM_CG on a cubic mesh with n / coarse_n a power of two;
 * the mesh must outlive the hierarchy. */
enum { FEM_MG_PH = 0, FEM_MG_HP = 1 };
typedef struct fem_mg_params {
  int32_t order;            /* FEM_MG_PH / FEM_MG_HP */
  int32_t precision;        /* level precision: FEM_FP32 (mixed) or FEM_FP64 */
  int32_t smoother_degree;  /* Chebyshev degree (reference 5, benchmark 3) */
  int32_t eig_iterations;   /* CG steps of the eigenvalue estimate (10) */
  double smoothing_range;   /* lambda_max / lambda_min (20) */
  double eig_safety;        /* lambda_max = safety * estimate (1.2) */
  int32_t coarse_n;         /* hexes per direction on the coarsest level (4) */
  int32_t use_graph;        /* capture the V-cycle as a CUDA graph (1) */
  int32_t c_transfer;       /* FEM_DG fine operators: 0 = DG P_p .. P_1 then CG P_1 (phc),
                               1 = CG P_p right below DG P_p, then the CG ladder of `order`
                               (cph / chp; DG/cells_batched/application_phc.cc:3396-3652) */
  int32_t learned_steps;    /* learned finest-level smoothing per V-cycle: 1 pre, 2 post, 3 both (3) */
  int32_t tensor_cores;     /* FP32 CG levels apply their operator with TF32 tensor-core
                               contractions (kernel variant 8: per cube, or per cell on
                               levels without whole cubes; operator accurate to ~1e-3) */
  int32_t weak_cg_levels;   /* FEM_DG fine operators: 1 = the CG levels use weak boundary terms
                               and no constrained DoFs (the reference's phc/cph/chp hierarchy,
                               DG/cells_batched/application_phc.cc:1737-1744,1799-1832);
                               0 = strong Dirichlet constraints (default) */
} fem_mg_params;
int fem_mg_params_default(fem_mg_params* p);
int fem_mg_create(fem_op* fine, const fem_mg_params* p, fem_mg** out);
int fem_mg_destroy(fem_mg* mg);
int fem_mg_n_levels(const fem_mg* mg, int32_t* n);
int fem_mg_level_info(const fem_mg* mg, int32_t level, uint64_t* m, int32_t* degree, int32_t* hexes,
                      double* lambda_max);
/* FEM_CG or FEM_DG: the kind of a level's operator (DG hierarchies have both) */
int fem_mg_level_kind(const fem_mg* mg, int32_t level, int32_t* kind);
/* PreconditionMG::vmult: dst = V(src), FP64 vectors of the fine operator */
int fem_mg_vcycle(fem_mg* mg, double* dst, const double* src, void* stream);
/* MG hooks on level-precision vectors of length level m: mg::Matrix::vmult,
 * MGSmootherPrecondition::smooth, MGTwoLevelTransfer::prolongate_and_add /
 * restrict_and_add (level -> level-1), MGCoarseGridBase::operator()
 * (application_ph.cc:1714-1746) */
int fem_mg_level_vmult(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream);
int fem_mg_smooth(fem_mg* mg, int32_t level, void* x, const void* b, int32_t zero_initial, void* stream);
int fem_mg_prolongate_add(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream);
int fem_mg_restrict_add(fem_mg* mg, int32_t level, void* dst, const void* src, void* stream);
int fem_mg_coarse_solve(fem_mg* mg, void* dst, const void* src, void* stream);

/* ---- preconditioned CG ---------------------------------------------------
 * SolverCG (application_ph.cc:1949-1980) on an FP64 operator; stops when
 * ||r|| <= rtol ||b||.  status: FEM_OK, FEM_ERR_NOT_CONVERGED,
 * FEM_ERR_BREAKDOWN (p^T A p <= 0) or FEM_ERR_NONFINITE; on a breakdown or a
 * non-finite p^T A p, x and r keep the previous iterate.  The step lengths
 * stay on the device; the host reads p^T A p and r^T r back once per
 * iteration (it synchronises with `stream` there). */
enum { FEM_PRECOND_NONE = 0, FEM_PRECOND_JACOBI = 1, FEM_PRECOND_MG = 2 };
typedef struct fem_solve_info {
  int32_t iterations;
  int32_t status;
  double initial_residual;
  double final_residual;
  int32_t fallback_iteration; /* iteration at which a learned smoother was replaced by
                                 Chebyshev (0: never) */
  int32_t reserved;
} fem_solve_info;
typedef struct fem_cg fem_cg;
/* flexible != 0: Polak-Ribiere beta (flexible CG, for variable preconditioners) */
int fem_cg_create(fem_op* op, fem_mg* mg /* FEM_PRECOND_MG only */, int32_t precond, int32_t flexible,
                  fem_cg** out);
int fem_cg_destroy(fem_cg* cg);
int fem_cg_solve(fem_cg* cg, double* x, const double* b, double rtol, int32_t max_iterations,
                 fem_solve_info* info, void* stream);

/* ---- learned finest-level smoother ----------------------------------------
 * No counterpart in the reference (its levels are always smoothed by
 * PreconditionChebyshev).  A per-cell MLP 29 -> 64 -> 64 -> 20 (GELU, BF16
 * weights, FP32 accumulation) maps a P3 cell's residual r_K / ||r_K|| and its
 * Jacobian J_K / h_K to a correction scaled by ||r_K|| / h_K; corrections are
 * assembled with inverse-multiplicity weights.  Trained on residual/error
 * pairs of the multigrid-preconditioned CG on Kuhn meshes; used on the finest
 * level of a P3 hierarchy inside flexible CG, with Chebyshev as fallback when
 * one outer iteration reduces the residual by less than a factor 2. */
typedef struct fem_mlp_train_params {
  int32_t n_sizes;      /* number of data meshes (<= 4) */
  int32_t sizes[4];     /* hexes per direction (16, 32) */
  int32_t rhs_per_size; /* random sin-mode loads per mesh (seeds seed + 100 size + i) */
  int32_t iterates;     /* MG-CG iterates per solve taken as samples */
  int32_t samples;      /* total residual/error cell samples (200000) */
  int32_t epochs;
  int32_t batch;
  float lr;             /* Adam learning rate */
  double jitter;
  uint64_t seed;
  double noise_fraction;     /* share of samples from white-noise errors e with r = A e (0) */
  int32_t coarse_iterations; /* V-cycle iterations of the coarse-grid correction removed from the
                                solver's errors before they become targets (12) */
  int32_t reserved;
} fem_mlp_train_params;
typedef struct fem_mlp_train_info {
  int32_t samples;
  int32_t reserved;
  double loss_first; /* mean loss of the first epoch */
  double loss_last;
  double seconds;
} fem_mlp_train_info;
int fem_mlp_create(uint64_t seed, fem_mlp** out);
int fem_mlp_destroy(fem_mlp* mlp);
int fem_mlp_n_params(int32_t* n);
int fem_mlp_get_weights(const fem_mlp* mlp, float* host /* [n_params] */);
int fem_mlp_set_weights(fem_mlp* mlp, const float* host);
int fem_mlp_train_params_default(fem_mlp_train_params* p);
int fem_mlp_generate_and_train(fem_mlp* mlp, const fem_mlp_train_params* p, fem_mlp_train_info* info);
/* training on device samples X [n][29], Y [n][20] */
int fem_mlp_train(fem_mlp* mlp, const float* X, const float* Y, int32_t n, int32_t epochs, int32_t batch, float lr,
                  uint64_t seed, fem_mlp_train_info* info);
/* gradient of mean ||MLP(X) - Y||^2 w.r.t. the (BF16-rounded) weights, device grad [n_params] */
int fem_mlp_gradient(fem_mlp* mlp, const float* X, const float* Y, int32_t n, float* grad, double* loss,
                     void* stream);
int fem_mlp_forward(fem_mlp* mlp, const float* X, float* O, int32_t n, void* stream);
/* The same forward on the tensor cores (tcgen05 MMAs, BF16 operands, FP32
 * accumulators, BF16 activations between the layers): the kernel the
 * smoother uses when tensor cores are on.  No counterpart in the reference. */
int fem_mlp_forward_tc(fem_mlp* mlp, const float* X, float* O, int32_t n, void* stream);
/* smoothing on the tensor cores (on != 0, default) or on the CUDA cores */
int fem_mlp_set_tensor_cores(fem_mlp* mlp, int32_t on);
/* *timed_out = 1 if a tensor-core launch gave up on a bounded wait since the
 * last call (the results of that launch are then invalid); synchronises */
int fem_mlp_status(fem_mlp* mlp, int32_t* timed_out);
int fem_mlp_save(const fem_mlp* mlp, const char* path);
int fem_mlp_load(const char* path, fem_mlp** out);
/* use mlp on the finest level of mg (NULL: back to Chebyshev); fallback != 0
 * re-enables Chebyshev after the first poor outer iteration */
int fem_mg_set_learned_smoother(fem_mg* mg, fem_mlp* mlp, int32_t fallback);

/* ---- batched multi-problem launch (components-batched Helmholtz etc.) ----
 * All operators must share kind, degree, precision and n_components.  One
 * persistent launch per phase covers every problem. */
int fem_batch_create(fem_op* const* ops, int32_t n_ops, fem_batch** out);
int fem_batch_destroy(fem_batch* batch);
int fem_batch_vmult(fem_batch* batch, void* const* dst, const void* const* src, void* stream);
int fem_batch_set_kernel_variant(fem_batch* batch, int32_t variant);

/* ---- autotuner -------------------------------------------------------------
 * Times every kernel variant (cells per CTA, thread or warp roles per cell;
 * fem_op_params.kernel_variant) of an operator or a batch with CUDA events
 * (median of `reps` launches after 2 warm-ups, on zero input), keeps the
 * fastest and returns it in *variant.  us[8] receives the median time per
 * variant 1..8 (0 = not a candidate; CG's approximate TF32 variant 4 is
 * never a candidate, and CG's cube variant 3 is timed as 5, 6 and 7).  With use_cache != 0 a choice recorded for
 * the same (kind, degree, precision, components, log2 cells, GPU name) is
 * applied without timing (*cached = 1).  fem_autotune_cache sets a file that
 * keeps the choices across processes (JSON lines; NULL = memory only).
 * No counterpart in the reference (deal.II fixes its vectorisation at compile
 * time).  Synchronises with the device; allocates two vectors per problem. */
int fem_op_autotune(fem_op* op, int32_t reps, int32_t use_cache, int32_t* variant, int32_t* cached, double* us);
int fem_batch_autotune(fem_batch* batch, int32_t reps, int32_t use_cache, int32_t* variant, int32_t* cached,
                       double* us);
int fem_autotune_cache(const char* path);

#ifdef __cplusplus
}
#endif
#endif /* SIMPLEX_FEM_H */
