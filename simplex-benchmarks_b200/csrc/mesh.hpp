// Tetrahedral mesh, adjacency and DoF numbering (host side).
//
// The mesh is the Kuhn (Freudenthal) subdivision of an nx*ny*nz hexahedral
// grid: every hex is cut into 6 tetrahedra that share its main diagonal.  It
// stands in for deal.II's GridGenerator::subdivided_hyper_cube_with_simplices
// + refine_global (CG/cells_batched/application.cc:1762-1770), which cuts each
// hex into 5 tets; the 6-tet cut keeps the mesh nested under refinement
// (needed by h-multigrid) and is what the benchmark configurations specify.
//
// Cell order is hierarchical: hexes in Morton (Z-curve) order, the 6 tets of
// a hex contiguous.  This plays the role of the reference's z-order partition
// and DoFRenumbering::matrix_free_data_locality
// (CG/cells_batched/application.cc:1773-1780,1828): consecutive cells share
// vertices, so gathers from a thread block stay in a few cache lines.
//
// Every cell lists its 4 vertices sorted by global vertex id.  Two cells that
// share an edge or a face therefore walk it in the same direction, which makes
// CG edge/face DoFs and DG face quadrature consistent without orientation
// codes (the reference carries deal.II's face orientation instead,
// DG/cells_batched/application.cc:1755-1782).
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace sfem {

struct MeshDescription {
  int n[3] = {1, 1, 1};        // hexes per direction
  double lo[3] = {0, 0, 0};    // box corner
  double hi[3] = {1, 1, 1};    // opposite box corner
  double jitter = 0.0;         // interior vertices move by U[-jitter*h, jitter*h] per axis
  uint64_t seed = 0;           // seed of the std::mt19937_64 stream used for the jitter
};

struct Mesh {
  MeshDescription desc;
  int64_t n_vertices = 0;
  int64_t n_cells = 0;
  std::vector<double> x;            // [n_vertices][3] coordinates
  std::vector<int32_t> cell_vertices;  // [n_cells][4], ascending global vertex id
  std::vector<int32_t> cell_hex;    // [n_cells] lexicographic hex index the tet came from
  std::vector<int32_t> nb;          // [n_cells][4] neighbour across local face f (-1: boundary)
  std::vector<int8_t> nbf;          // [n_cells][4] local face index of f inside the neighbour
  int64_t n_interior_faces = 0;
  int64_t n_boundary_faces = 0;
  bool structured = false;          // a Kuhn box (hex / cube kernels, h-multigrid)
  bool curved = false;              // quadratic geometry: edge_x holds the edge nodes
  std::vector<double> edge_x;       // [n_cells][6][3] geometry nodes of edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
  std::vector<int64_t> input_cell;  // meshes from arrays: input index of every cell

  // lexicographic vertex index of lattice point (i,j,k)
  int64_t vertex_id(int i, int j, int k) const {
    return i + (int64_t)(desc.n[0] + 1) * (j + (int64_t)(desc.n[1] + 1) * k);
  }
  std::array<int, 3> vertex_lattice(int64_t v) const {
    const int64_t nx = desc.n[0] + 1, ny = desc.n[1] + 1;
    return {int(v % nx), int((v / nx) % ny), int(v / (nx * ny))};
  }
};

Mesh build_kuhn_mesh(const MeshDescription& d);

// Curvilinear geometry: every point x of the mesh's bounding box moves to
// x + amplitude * prod_d sin(pi xi_d) * (hi - lo), xi the box coordinates in
// [0,1]^3 (the box boundary stays), and every cell gets a quadratic
// (P2) geometry: its moved vertices and the moved midpoints of its straight
// edges.  Cells whose orientation would flip are rejected.
void curve_mesh(Mesh& m, double amplitude);

// Face neighbours (nb, nbf) and face counts of a mesh with sorted cell vertices.
void build_face_adjacency(Mesh& m);

// Unstructured tetrahedral mesh from vertex and cell arrays (any vertex order
// per cell; the cells are stored with sorted vertices).  reorder = 1 puts the
// cells in Morton order of their centroids, 0 keeps the input order.
Mesh build_mesh_from_arrays(int64_t n_vertices, const double* x, int64_t n_cells, const int32_t* cells,
                            int reorder);

// Legacy ASCII VTK unstructured grid (POINTS, CELLS, CELL_TYPES; tetrahedra,
// VTK cell type 10, only), the format GridIn::read_vtk reads in the reference.
Mesh read_vtk_mesh(const std::string& path, int reorder);

// Affine geometry of one tet: J = [x1-x0, x2-x0, x3-x0] (J_ij = dx_i/dxi_j).
struct CellGeometry {
  double J[3][3];
  double Jinv[3][3];
  double det;   // signed
};
CellGeometry cell_geometry(const Mesh& m, int64_t c);

// Area of local face f of cell c and its outward unit normal.
void face_area_normal(const Mesh& m, int64_t c, int f, double& area, double n[3]);

// Continuous Lagrange P_p numbering (first touch in cell order), homogeneous
// Dirichlet constraints on every node that lies on a boundary face.
struct CGDofs {
  int degree = 1;
  int K = 4;
  int64_t n_dofs = 0;
  std::vector<int32_t> cell_dofs;     // [n_cells][K]
  std::vector<uint8_t> constrained;   // [n_dofs]
  std::vector<double> support;        // [n_dofs][3] node positions
};
CGDofs build_cg_dofs(const Mesh& m, int degree);

}  // namespace sfem
