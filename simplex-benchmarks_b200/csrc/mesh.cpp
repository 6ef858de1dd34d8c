// Kuhn tetrahedral mesh, face adjacency and continuous DoF numbering.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <random>
#include <string>

#include "common.hpp"
#include "ref_tables.h"
#include "../../include/simplex_fem.h"

namespace sfem {

namespace {

// Morton key of (i,j,k) with 21 bits per axis.
uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton3(uint64_t i, uint64_t j, uint64_t k) {
  return spread3(i) | (spread3(j) << 1) | (spread3(k) << 2);
}

// vertex -> incident cells (CSR)
struct Incidence {
  std::vector<int64_t> start;
  std::vector<int32_t> cells;
};
Incidence vertex_cells(const Mesh& m) {
  Incidence inc;
  inc.start.assign(m.n_vertices + 1, 0);
  for (int64_t c = 0; c < m.n_cells; ++c)
    for (int v = 0; v < 4; ++v) inc.start[m.cell_vertices[4 * c + v] + 1]++;
  for (int64_t v = 0; v < m.n_vertices; ++v) inc.start[v + 1] += inc.start[v];
  inc.cells.resize(inc.start[m.n_vertices]);
  std::vector<int64_t> pos(inc.start.begin(), inc.start.end() - 1);
  for (int64_t c = 0; c < m.n_cells; ++c)
    for (int v = 0; v < 4; ++v) inc.cells[pos[m.cell_vertices[4 * c + v]]++] = (int32_t)c;
  return inc;
}

const int kEdges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

}  // namespace

Mesh build_kuhn_mesh(const MeshDescription& d) {
  for (int a = 0; a < 3; ++a) {
    SFEM_REQUIRE(d.n[a] >= 1 && d.n[a] <= 1024, FEM_ERR_ARG, "mesh: n must be in [1,1024]");
    SFEM_REQUIRE(d.hi[a] > d.lo[a], FEM_ERR_ARG, "mesh: hi must exceed lo");
  }
  SFEM_REQUIRE(d.jitter >= 0.0 && d.jitter < 0.25, FEM_ERR_ARG, "mesh: jitter must be in [0,0.25)");
  Mesh m;
  m.desc = d;
  const int nx = d.n[0], ny = d.n[1], nz = d.n[2];
  m.n_vertices = int64_t(nx + 1) * (ny + 1) * (nz + 1);
  const int64_t n_hex = int64_t(nx) * ny * nz;
  SFEM_REQUIRE(6 * n_hex < (int64_t(1) << 31), FEM_ERR_ARG, "mesh: too many cells for int32 ids");
  m.n_cells = 6 * n_hex;
  double h[3];
  for (int a = 0; a < 3; ++a) h[a] = (d.hi[a] - d.lo[a]) / d.n[a];

  // vertices, lexicographic; interior vertices jittered from one mt19937_64 stream
  m.x.resize(3 * m.n_vertices);
  std::mt19937_64 rng(d.seed);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const int64_t v = m.vertex_id(i, j, k);
        const int idx[3] = {i, j, k};
        const bool interior = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
        for (int a = 0; a < 3; ++a) {
          double pos = d.lo[a] + idx[a] * h[a];
          if (d.jitter > 0) {
            // uniform in [0,1) from the top 53 bits, mapped to [-jitter h, jitter h)
            const double u = double(rng() >> 11) * (1.0 / 9007199254740992.0);
            if (interior) pos += (2.0 * u - 1.0) * d.jitter * h[a];
          }
          m.x[3 * v + a] = pos;
        }
      }

  // hexes in Morton order
  std::vector<std::pair<uint64_t, int64_t>> hexes;
  hexes.reserve(n_hex);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        hexes.push_back({morton3(i, j, k), i + int64_t(nx) * (j + int64_t(ny) * k)});
  std::sort(hexes.begin(), hexes.end());

  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  m.cell_vertices.resize(4 * m.n_cells);
  m.cell_hex.resize(m.n_cells);
  int64_t c = 0;
  for (const auto& hx : hexes) {
    const int64_t lin = hx.second;
    const int i = int(lin % nx), j = int((lin / nx) % ny), k = int(lin / (int64_t(nx) * ny));
    for (int t = 0; t < 6; ++t) {
      int off[3] = {0, 0, 0};
      int32_t vs[4];
      vs[0] = (int32_t)m.vertex_id(i, j, k);
      for (int s = 0; s < 2; ++s) {
        off[perms[t][s]] = 1;
        vs[s + 1] = (int32_t)m.vertex_id(i + off[0], j + off[1], k + off[2]);
      }
      vs[3] = (int32_t)m.vertex_id(i + 1, j + 1, k + 1);
      std::sort(vs, vs + 4);
      for (int v = 0; v < 4; ++v) m.cell_vertices[4 * c + v] = vs[v];
      m.cell_hex[c] = (int32_t)lin;
      ++c;
    }
  }

  build_face_adjacency(m);
  m.structured = true;
  return m;
}

void build_face_adjacency(Mesh& m) {
  // face adjacency: a face is found from its lowest vertex; the other two
  // vertices identify it among the faces incident to that vertex.
  Incidence inc = vertex_cells(m);
  m.nb.assign(4 * m.n_cells, -1);
  m.nbf.assign(4 * m.n_cells, -1);
  struct Pending { int32_t b, c2; int32_t cell; int8_t f; };
  std::vector<Pending> local;
  for (int64_t a = 0; a < m.n_vertices; ++a) {
    local.clear();
    for (int64_t s = inc.start[a]; s < inc.start[a + 1]; ++s) {
      const int32_t cc = inc.cells[s];
      const int32_t* cv = &m.cell_vertices[4 * int64_t(cc)];
      for (int f = 0; f < 4; ++f) {
        int32_t fv[3];
        int q = 0;
        for (int v = 0; v < 4; ++v)
          if (v != f) fv[q++] = cv[v];
        if (fv[0] != a) continue;
        bool matched = false;
        for (auto& p : local) {
          if (p.b == fv[1] && p.c2 == fv[2]) {
            SFEM_REQUIRE(p.cell >= 0, FEM_ERR_ARG, "mesh: a face is shared by more than two cells");
            m.nb[4 * int64_t(cc) + f] = p.cell;
            m.nbf[4 * int64_t(cc) + f] = p.f;
            m.nb[4 * int64_t(p.cell) + p.f] = cc;
            m.nbf[4 * int64_t(p.cell) + p.f] = (int8_t)f;
            p.cell = -1;  // a face has at most two cells
            matched = true;
            break;
          }
        }
        if (!matched) local.push_back({fv[1], fv[2], cc, (int8_t)f});
      }
    }
  }
  m.n_boundary_faces = m.n_interior_faces = 0;
  for (int64_t i = 0; i < 4 * m.n_cells; ++i) {
    if (m.nb[i] < 0)
      m.n_boundary_faces++;
    else
      m.n_interior_faces++;
  }
  m.n_interior_faces /= 2;
}

Mesh build_mesh_from_arrays(int64_t n_vertices, const double* x, int64_t n_cells, const int32_t* cells,
                            int reorder) {
  SFEM_REQUIRE(n_vertices >= 4 && n_cells >= 1, FEM_ERR_ARG, "mesh: need at least 4 vertices and 1 cell");
  SFEM_REQUIRE(n_vertices < (int64_t(1) << 31) && n_cells < (int64_t(1) << 31), FEM_ERR_ARG,
               "mesh: too many vertices or cells for int32 ids");
  SFEM_REQUIRE(reorder == 0 || reorder == 1, FEM_ERR_ARG, "mesh: reorder must be 0 (input order) or 1 (Morton)");
  Mesh m;
  m.desc.n[0] = m.desc.n[1] = m.desc.n[2] = 0;
  m.n_vertices = n_vertices;
  m.n_cells = n_cells;
  m.x.assign(x, x + 3 * n_vertices);
  // hierarchical cell order: Morton order of the cell centroids on a 2^21 grid
  // over the bounding box (the role of SparsityTools::reorder_hierarchical
  // and DoFRenumbering::matrix_free_data_locality in the reference,
  // CG/cells_batched/application.cc:1696-1757,1828)
  std::vector<int64_t> order(n_cells);
  for (int64_t c = 0; c < n_cells; ++c) order[c] = c;
  for (int64_t c = 0; c < n_cells; ++c)
    for (int v = 0; v < 4; ++v)
      SFEM_REQUIRE(cells[4 * c + v] >= 0 && cells[4 * c + v] < n_vertices, FEM_ERR_ARG,
                   "mesh: cell " + std::to_string(c) + " names a vertex out of range");
  if (reorder == 1) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t v = 0; v < n_vertices; ++v)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], x[3 * v + a]);
        hi[a] = std::max(hi[a], x[3 * v + a]);
      }
    std::vector<uint64_t> key(n_cells);
    for (int64_t c = 0; c < n_cells; ++c) {
      uint64_t q[3];
      for (int a = 0; a < 3; ++a) {
        double s = 0;
        for (int v = 0; v < 4; ++v) s += x[3 * int64_t(cells[4 * c + v]) + a];
        const double t = (s / 4 - lo[a]) / std::max(hi[a] - lo[a], 1e-300);
        q[a] = uint64_t(std::min(std::max(t, 0.0), 1.0) * double((1 << 21) - 1));
      }
      key[c] = morton3(q[0], q[1], q[2]);
    }
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  }
  m.cell_vertices.resize(4 * n_cells);
  m.cell_hex.resize(n_cells);
  m.input_cell.resize(n_cells);
  for (int64_t c = 0; c < n_cells; ++c) {
    int32_t vs[4];
    for (int v = 0; v < 4; ++v) vs[v] = cells[4 * order[c] + v];
    std::sort(vs, vs + 4);
    SFEM_REQUIRE(vs[0] != vs[1] && vs[1] != vs[2] && vs[2] != vs[3], FEM_ERR_ARG,
                 "mesh: cell " + std::to_string(order[c]) + " repeats a vertex");
    for (int v = 0; v < 4; ++v) m.cell_vertices[4 * c + v] = vs[v];
    m.cell_hex[c] = int32_t(c);  // no hex structure: every cell its own macro cell
    m.input_cell[c] = order[c];
  }
  for (int64_t c = 0; c < n_cells; ++c) {
    const CellGeometry g = cell_geometry(m, c);
    SFEM_REQUIRE(std::fabs(g.det) > 0.0 && std::isfinite(g.det), FEM_ERR_ARG,
                 "mesh: cell " + std::to_string(m.input_cell[c]) + " is degenerate");
  }
  build_face_adjacency(m);
  return m;
}

void curve_mesh(Mesh& m, double amplitude) {
  SFEM_REQUIRE(!m.curved, FEM_ERR_STATE, "curve: the mesh is already curved");
  SFEM_REQUIRE(std::isfinite(amplitude) && std::fabs(amplitude) < 0.5, FEM_ERR_ARG,
               "curve: |amplitude| must be below 0.5");
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t v = 0; v < m.n_vertices; ++v)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], m.x[3 * v + a]);
      hi[a] = std::max(hi[a], m.x[3 * v + a]);
    }
  auto phi = [&](const double* x, double* out) {
    double s = amplitude;
    for (int a = 0; a < 3; ++a) s *= std::sin(M_PI * (x[a] - lo[a]) / (hi[a] - lo[a]));
    for (int a = 0; a < 3; ++a) out[a] = x[a] + s * (hi[a] - lo[a]);
  };
  std::vector<double> sign(m.n_cells);
  for (int64_t c = 0; c < m.n_cells; ++c) sign[c] = cell_geometry(m, c).det > 0 ? 1.0 : -1.0;
  m.edge_x.resize(18 * size_t(m.n_cells));
  for (int64_t c = 0; c < m.n_cells; ++c)
    for (int e = 0; e < 6; ++e) {
      double mid[3];
      for (int a = 0; a < 3; ++a)
        mid[a] = 0.5 * (m.x[3 * int64_t(m.cell_vertices[4 * c + kEdges[e][0]]) + a] +
                        m.x[3 * int64_t(m.cell_vertices[4 * c + kEdges[e][1]]) + a]);
      phi(mid, &m.edge_x[18 * c + 3 * e]);
    }
  std::vector<double> moved(m.x.size());
  for (int64_t v = 0; v < m.n_vertices; ++v) phi(&m.x[3 * v], &moved[3 * v]);
  m.x.swap(moved);
  for (int64_t c = 0; c < m.n_cells; ++c) {
    const double det = cell_geometry(m, c).det;
    SFEM_REQUIRE(det * sign[c] > 0, FEM_ERR_ARG, "curve: the amplitude inverts cell " + std::to_string(c));
  }
  m.curved = true;
  m.structured = false;  // the h-levels of the multigrid are affine Kuhn meshes
}

Mesh read_vtk_mesh(const std::string& path, int reorder) {
  std::ifstream in(path);
  SFEM_REQUIRE(in.good(), FEM_ERR_ARG, "vtk: cannot open " + path);
  std::string line;
  std::vector<double> x;
  std::vector<int32_t> cells;
  std::vector<int> types;
  int64_t np = -1;
  bool ascii = false;
  std::string tok;
  while (in >> tok) {
    if (tok == "ASCII") {
      ascii = true;
    } else if (tok == "BINARY") {
      throw Error(FEM_ERR_ARG, "vtk: only ASCII legacy files are read");
    } else if (tok == "DATASET") {
      in >> tok;
      SFEM_REQUIRE(tok == "UNSTRUCTURED_GRID", FEM_ERR_ARG, "vtk: DATASET must be UNSTRUCTURED_GRID");
    } else if (tok == "POINTS") {
      std::string type;
      in >> np >> type;
      SFEM_REQUIRE(np > 0, FEM_ERR_ARG, "vtk: bad POINTS count");
      x.resize(3 * np);
      for (auto& v : x) SFEM_REQUIRE(bool(in >> v), FEM_ERR_ARG, "vtk: short POINTS section");
    } else if (tok == "CELLS") {
      int64_t nc = 0, size = 0;
      in >> nc >> size;
      SFEM_REQUIRE(nc > 0 && size >= 5 * nc, FEM_ERR_ARG, "vtk: bad CELLS header");
      cells.reserve(4 * nc);
      for (int64_t c = 0; c < nc; ++c) {
        int64_t k = 0;
        SFEM_REQUIRE(bool(in >> k), FEM_ERR_ARG, "vtk: short CELLS section");
        SFEM_REQUIRE(k == 4, FEM_ERR_ARG, "vtk: only tetrahedra (4 vertices per cell) are read");
        for (int v = 0; v < 4; ++v) {
          int64_t id = 0;
          SFEM_REQUIRE(bool(in >> id), FEM_ERR_ARG, "vtk: short CELLS section");
          cells.push_back(int32_t(id));
        }
      }
    } else if (tok == "CELL_TYPES") {
      int64_t nt = 0;
      in >> nt;
      types.resize(nt);
      for (auto& t : types) SFEM_REQUIRE(bool(in >> t), FEM_ERR_ARG, "vtk: short CELL_TYPES section");
    } else if (tok == "CELL_DATA" || tok == "POINT_DATA") {
      break;  // attached data is not needed
    }
  }
  SFEM_REQUIRE(ascii, FEM_ERR_ARG, "vtk: not an ASCII legacy VTK file");
  SFEM_REQUIRE(np > 0 && !cells.empty(), FEM_ERR_ARG, "vtk: POINTS and CELLS are required");
  SFEM_REQUIRE(types.empty() || int64_t(types.size()) * 4 == int64_t(cells.size()), FEM_ERR_ARG,
               "vtk: CELL_TYPES count differs from CELLS");
  for (int t : types) SFEM_REQUIRE(t == 10, FEM_ERR_ARG, "vtk: only VTK_TETRA (type 10) cells are read");
  return build_mesh_from_arrays(np, x.data(), int64_t(cells.size() / 4), cells.data(), reorder);
}

CellGeometry cell_geometry(const Mesh& m, int64_t c) {
  CellGeometry g;
  const int32_t* cv = &m.cell_vertices[4 * c];
  const double* x0 = &m.x[3 * int64_t(cv[0])];
  for (int jj = 0; jj < 3; ++jj) {
    const double* xj = &m.x[3 * int64_t(cv[jj + 1])];
    for (int i = 0; i < 3; ++i) g.J[i][jj] = xj[i] - x0[i];
  }
  const double(&J)[3][3] = g.J;
  g.det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
          J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  const double id = 1.0 / g.det;
  g.Jinv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  g.Jinv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  g.Jinv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  g.Jinv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  g.Jinv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  g.Jinv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  g.Jinv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  g.Jinv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  g.Jinv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return g;
}

void face_area_normal(const Mesh& m, int64_t c, int f, double& area, double n[3]) {
  const int32_t* cv = &m.cell_vertices[4 * c];
  int q = 0;
  const double* p[3];
  for (int v = 0; v < 4; ++v)
    if (v != f) p[q++] = &m.x[3 * int64_t(cv[v])];
  const double* opp = &m.x[3 * int64_t(cv[f])];
  double a[3], b[3];
  for (int i = 0; i < 3; ++i) {
    a[i] = p[1][i] - p[0][i];
    b[i] = p[2][i] - p[0][i];
  }
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  area = 0.5 * len;
  double dot = 0;
  for (int i = 0; i < 3; ++i) dot += cr[i] * (opp[i] - p[0][i]);
  const double s = dot > 0 ? -1.0 / len : 1.0 / len;  // point away from the opposite vertex
  for (int i = 0; i < 3; ++i) n[i] = cr[i] * s;
}

namespace {
template <int P>
void number_cg(const Mesh& m, CGDofs& d) {
  using T = ref::Tables<P>;
  constexpr int K = T::K;
  d.K = K;
  d.cell_dofs.assign(K * m.n_cells, -1);
  // edge and face ids from the lowest vertex (sorted cell vertices make every
  // local edge (i<j) and face walk upwards in global id)
  Incidence inc = vertex_cells(m);
  std::vector<int32_t> cell_edge(6 * m.n_cells, -1), cell_face(4 * m.n_cells, -1);
  int64_t n_edges = 0, n_faces = 0;
  std::vector<std::pair<int32_t, int32_t>> loc_e;
  std::vector<std::pair<std::pair<int32_t, int32_t>, int32_t>> loc_f;
  for (int64_t a = 0; a < m.n_vertices; ++a) {
    loc_e.clear();
    loc_f.clear();
    for (int64_t s = inc.start[a]; s < inc.start[a + 1]; ++s) {
      const int32_t cc = inc.cells[s];
      const int32_t* cv = &m.cell_vertices[4 * int64_t(cc)];
      for (int e = 0; e < 6; ++e) {
        if (cv[kEdges[e][0]] != a) continue;
        const int32_t b = cv[kEdges[e][1]];
        int32_t id = -1;
        for (auto& pr : loc_e)
          if (pr.first == b) id = pr.second;
        if (id < 0) {
          id = (int32_t)n_edges++;
          loc_e.push_back({b, id});
        }
        cell_edge[6 * int64_t(cc) + e] = id;
      }
      if (P >= 3) {
        for (int f = 0; f < 4; ++f) {
          int32_t fv[3];
          int q = 0;
          for (int v = 0; v < 4; ++v)
            if (v != f) fv[q++] = cv[v];
          if (fv[0] != a) continue;
          int32_t id = -1;
          for (auto& pr : loc_f)
            if (pr.first.first == fv[1] && pr.first.second == fv[2]) id = pr.second;
          if (id < 0) {
            id = (int32_t)n_faces++;
            loc_f.push_back({{fv[1], fv[2]}, id});
          }
          cell_face[4 * int64_t(cc) + f] = id;
        }
      }
    }
  }
  // first-touch numbering in cell order
  std::vector<int32_t> vdof(m.n_vertices, -1), edof(n_edges, -1), fdof(n_faces, -1);
  int64_t next = 0;
  for (int64_t c = 0; c < m.n_cells; ++c) {
    const int32_t* cv = &m.cell_vertices[4 * c];
    for (int i = 0; i < K; ++i) {
      const int* a = T::LATTICE[i];
      int nz = 0, first = -1, second = -1, zero = -1;
      for (int v = 0; v < 4; ++v) {
        if (a[v] > 0) {
          if (first < 0) first = v; else if (second < 0) second = v;
          nz++;
        } else {
          zero = v;
        }
      }
      int32_t dof;
      if (nz == 1) {
        int32_t& r = vdof[cv[first]];
        if (r < 0) r = (int32_t)next++;
        dof = r;
      } else if (nz == 2) {
        int e = 0;
        for (; e < 6; ++e)
          if (kEdges[e][0] == first && kEdges[e][1] == second) break;
        int32_t& r = edof[cell_edge[6 * c + e]];
        if (r < 0) {
          r = (int32_t)next;
          next += P - 1;
        }
        dof = r + (a[second] - 1);
      } else {
        // P3: one node per face
        int32_t& r = fdof[cell_face[4 * c + zero]];
        if (r < 0) r = (int32_t)next++;
        dof = r;
      }
      d.cell_dofs[K * c + i] = dof;
    }
  }
  SFEM_REQUIRE(next < (int64_t(1) << 31), FEM_ERR_ARG, "dofs: too many DoFs for int32 indices");
  d.n_dofs = next;
  d.constrained.assign(d.n_dofs, 0);
  d.support.assign(3 * d.n_dofs, 0.0);
  for (int64_t c = 0; c < m.n_cells; ++c) {
    const int32_t* cv = &m.cell_vertices[4 * c];
    for (int i = 0; i < K; ++i) {
      const int32_t g = d.cell_dofs[K * c + i];
      for (int a = 0; a < 3; ++a) {
        double s = 0;
        for (int v = 0; v < 4; ++v) s += T::LATTICE[i][v] * m.x[3 * int64_t(cv[v]) + a];
        d.support[3 * int64_t(g) + a] = s / P;
      }
    }
    for (int f = 0; f < 4; ++f)
      if (m.nb[4 * c + f] < 0)
        for (int i = 0; i < T::NF; ++i) d.constrained[d.cell_dofs[K * c + T::FN[f][i]]] = 1;
  }
}
}  // namespace

CGDofs build_cg_dofs(const Mesh& m, int degree) {
  CGDofs d;
  d.degree = degree;
  switch (degree) {
    case 1: number_cg<1>(m, d); break;
    case 2: number_cg<2>(m, d); break;
    case 3: number_cg<3>(m, d); break;
    default: throw Error(FEM_ERR_ARG, "dofs: degree must be 1, 2 or 3");
  }
  return d;
}

}  // namespace sfem
