// Domain decomposition of a mesh over ranks: see partition.hpp.
#include "partition.hpp"

#include <algorithm>
#include <unordered_map>

#include "../../include/simplex_fem.h"
#include "common.hpp"

namespace sfem {

void part_range(int64_t n_cells, int n_parts, int part, int64_t& begin, int64_t& end) {
  // cut at whole 4x4x4-hex cubes (384 tets) or whole hexes when there are enough
  int64_t unit = 1;
  if (n_cells % 384 == 0 && n_cells / 384 >= n_parts) unit = 384;
  else if (n_cells % 6 == 0 && n_cells / 6 >= n_parts) unit = 6;
  const int64_t units = n_cells / unit;
  begin = units * part / n_parts * unit;
  end = part + 1 == n_parts ? n_cells : units * (part + 1) / n_parts * unit;
}

namespace {

struct Parts {
  std::vector<int64_t> begin;  // [n_parts + 1]
  int of(int64_t c) const {
    return int(std::upper_bound(begin.begin(), begin.end(), c) - begin.begin()) - 1;
  }
};

// local mesh with the vertices of the global one and the listed cells;
// neighbour ids mapped to local ids, -2 where the neighbour is not local
std::shared_ptr<Mesh> local_mesh(const Mesh& g, const std::vector<int32_t>& cells,
                                 const std::vector<int32_t>& loc_of_global) {
  auto m = std::make_shared<Mesh>();
  m->desc = g.desc;
  m->n_vertices = g.n_vertices;
  m->x = g.x;
  m->n_cells = int64_t(cells.size());
  m->cell_vertices.resize(4 * cells.size());
  m->cell_hex.resize(cells.size());
  m->nb.resize(4 * cells.size());
  m->nbf.resize(4 * cells.size());
  for (size_t l = 0; l < cells.size(); ++l) {
    const int64_t c = cells[l];
    m->cell_hex[l] = g.cell_hex[c];
    for (int f = 0; f < 4; ++f) {
      m->cell_vertices[4 * l + f] = g.cell_vertices[4 * c + f];
      const int32_t o = g.nb[4 * c + f];
      m->nb[4 * l + f] = o < 0 ? -1 : (loc_of_global[o] >= 0 ? loc_of_global[o] : -2);
      m->nbf[4 * l + f] = g.nbf[4 * c + f];
      if (m->nb[4 * l + f] == -1) m->n_boundary_faces++;
      else m->n_interior_faces++;
    }
  }
  m->n_interior_faces /= 2;
  return m;
}

void build_cg(const Mesh& mesh, const Parts& parts, Partition& P) {
  const CGDofs g = build_cg_dofs(mesh, P.degree);
  const int K = g.K;
  const int64_t nd = g.n_dofs;
  P.n_global = nd;
  // owner: the part of the first cell that touches the DoF
  std::vector<int32_t> owner(nd, -1);
  for (int64_t c = 0; c < mesh.n_cells; ++c) {
    const int q = parts.of(c);
    for (int i = 0; i < K; ++i) {
      int32_t& o = owner[g.cell_dofs[K * c + i]];
      if (o < 0) o = q;
    }
  }
  const int r = P.part;
  std::vector<int32_t> loc(nd, -1);
  std::vector<int64_t> owned, ghosts;
  for (int64_t d = 0; d < nd; ++d)
    if (owner[d] == r) owned.push_back(d);
  for (int64_t c = P.cell_begin; c < P.cell_end; ++c)
    for (int i = 0; i < K; ++i) {
      const int32_t d = g.cell_dofs[K * c + i];
      if (owner[d] != r && loc[d] != -2) {
        loc[d] = -2;
        ghosts.push_back(d);
      }
    }
  std::sort(ghosts.begin(), ghosts.end(), [&](int64_t a, int64_t b) {
    return owner[a] != owner[b] ? owner[a] < owner[b] : a < b;
  });
  P.n_owned = int64_t(owned.size());
  P.n_ghost = int64_t(ghosts.size());
  P.gidx = owned;
  P.gidx.insert(P.gidx.end(), ghosts.begin(), ghosts.end());
  for (size_t l = 0; l < P.gidx.size(); ++l) loc[P.gidx[l]] = int32_t(l);
  // entries of this part that other parts touch (their ghosts), per part
  std::vector<std::vector<int64_t>> send(P.n_parts);
  for (int q = 0; q < P.n_parts; ++q) {
    if (q == r) continue;
    for (int64_t c = parts.begin[q]; c < parts.begin[q + 1]; ++c)
      for (int i = 0; i < K; ++i) {
        const int32_t d = g.cell_dofs[K * c + i];
        if (owner[d] == r) send[q].push_back(d);
      }
    std::sort(send[q].begin(), send[q].end());
    send[q].erase(std::unique(send[q].begin(), send[q].end()), send[q].end());
  }
  for (int q = 0; q < P.n_parts; ++q) {
    if (q == r) continue;
    PartPeer peer;
    peer.rank = q;
    for (int64_t d : send[q]) peer.send.push_back(loc[d]);
    for (int64_t d : ghosts)
      if (owner[d] == q) peer.recv.push_back(loc[d]);
    if (!peer.send.empty() || !peer.recv.empty()) P.peers.push_back(std::move(peer));
  }
  // local operator data
  std::vector<int32_t> cells;
  for (int64_t c = P.cell_begin; c < P.cell_end; ++c) cells.push_back(int32_t(c));
  std::vector<int32_t> loc_cell(mesh.n_cells, -1);
  for (size_t l = 0; l < cells.size(); ++l) loc_cell[cells[l]] = int32_t(l);
  P.local = local_mesh(mesh, cells, loc_cell);
  const int64_t nl = int64_t(P.gidx.size());
  P.dofs.degree = P.degree;
  P.dofs.K = K;
  P.dofs.n_dofs = nl;
  P.dofs.cell_dofs.resize(size_t(K) * cells.size());
  for (size_t l = 0; l < cells.size(); ++l)
    for (int i = 0; i < K; ++i) P.dofs.cell_dofs[K * l + i] = loc[g.cell_dofs[K * int64_t(cells[l]) + i]];
  P.dofs.constrained.resize(nl);
  P.dofs.support.resize(3 * size_t(nl));
  P.identity.assign(nl, 0);
  for (int64_t l = 0; l < nl; ++l) {
    const int64_t d = P.gidx[l];
    P.dofs.constrained[l] = g.constrained[d];
    for (int a = 0; a < 3; ++a) P.dofs.support[3 * l + a] = g.support[3 * d + a];
    P.identity[l] = l < P.n_owned && g.constrained[d];
  }
}

void build_dg(const Mesh& mesh, const Parts& parts, Partition& P) {
  const int K = (P.degree + 1) * (P.degree + 2) * (P.degree + 3) / 6;
  const int64_t W = int64_t(K) * P.n_components;
  const int r = P.part;
  P.n_global = mesh.n_cells * W;
  std::vector<int32_t> cells, ghosts;
  std::vector<int32_t> loc(mesh.n_cells, -1);
  for (int64_t c = P.cell_begin; c < P.cell_end; ++c) cells.push_back(int32_t(c));
  for (int64_t c = P.cell_begin; c < P.cell_end; ++c)
    for (int f = 0; f < 4; ++f) {
      const int32_t o = mesh.nb[4 * c + f];
      if (o >= 0 && (o < P.cell_begin || o >= P.cell_end) && loc[o] != -2) {
        loc[o] = -2;
        ghosts.push_back(o);
      }
    }
  std::sort(ghosts.begin(), ghosts.end(), [&](int32_t a, int32_t b) {
    const int qa = parts.of(a), qb = parts.of(b);
    return qa != qb ? qa < qb : a < b;
  });
  const int64_t n_own_cells = int64_t(cells.size());
  cells.insert(cells.end(), ghosts.begin(), ghosts.end());
  for (size_t l = 0; l < cells.size(); ++l) loc[cells[l]] = int32_t(l);
  P.n_owned = n_own_cells * W;
  P.n_ghost = int64_t(ghosts.size()) * W;
  P.gidx.resize(cells.size() * W);
  for (size_t l = 0; l < cells.size(); ++l)
    for (int64_t k = 0; k < W; ++k) P.gidx[l * W + k] = int64_t(cells[l]) * W + k;
  // owned cells that are face neighbours of another part's cells
  std::vector<std::vector<int32_t>> send(P.n_parts);
  for (int64_t c = P.cell_begin; c < P.cell_end; ++c)
    for (int f = 0; f < 4; ++f) {
      const int32_t o = mesh.nb[4 * c + f];
      if (o < 0 || (o >= P.cell_begin && o < P.cell_end)) continue;
      send[parts.of(o)].push_back(int32_t(c));
    }
  for (int q = 0; q < P.n_parts; ++q) {
    if (q == r) continue;
    std::sort(send[q].begin(), send[q].end());
    send[q].erase(std::unique(send[q].begin(), send[q].end()), send[q].end());
    PartPeer peer;
    peer.rank = q;
    for (int32_t c : send[q])
      for (int64_t k = 0; k < W; ++k) peer.send.push_back(int64_t(loc[c]) * W + k);
    for (int32_t c : ghosts)
      if (parts.of(c) == q)
        for (int64_t k = 0; k < W; ++k) peer.recv.push_back(int64_t(loc[c]) * W + k);
    if (!peer.send.empty() || !peer.recv.empty()) P.peers.push_back(std::move(peer));
  }
  P.local = local_mesh(mesh, cells, loc);
}

}  // namespace

Partition build_partition(const Mesh& mesh, int degree, int kind, int n_components, int n_parts, int part) {
  SFEM_REQUIRE(degree >= 1 && degree <= 3, FEM_ERR_ARG, "partition: degree must be 1, 2 or 3");
  SFEM_REQUIRE(kind == FEM_CG || kind == FEM_DG || kind == FEM_HELMHOLTZ, FEM_ERR_ARG, "partition: unknown kind");
  SFEM_REQUIRE(n_parts >= 1 && part >= 0 && part < n_parts, FEM_ERR_ARG, "partition: need 0 <= part < n_parts");
  SFEM_REQUIRE(mesh.n_cells >= n_parts, FEM_ERR_ARG, "partition: fewer cells than parts");
  SFEM_REQUIRE(!mesh.curved, FEM_ERR_ARG, "partition: curved meshes are not partitioned");
  SFEM_REQUIRE(kind == FEM_CG ? n_components == 1 : (n_components == 1 || n_components == 3), FEM_ERR_ARG,
               "partition: n_components must be 1 (CG, DG) or 1 / 3 (Helmholtz)");
  Partition P;
  P.kind = kind;
  P.degree = degree;
  P.n_components = n_components;
  P.n_parts = n_parts;
  P.part = part;
  Parts parts;
  parts.begin.resize(n_parts + 1);
  for (int q = 0; q < n_parts; ++q) {
    int64_t b, e;
    part_range(mesh.n_cells, n_parts, q, b, e);
    parts.begin[q] = b;
    parts.begin[q + 1] = e;
  }
  P.cell_begin = parts.begin[part];
  P.cell_end = parts.begin[part + 1];
  SFEM_REQUIRE(P.cell_end > P.cell_begin, FEM_ERR_ARG, "partition: empty part");
  if (kind == FEM_CG) build_cg(mesh, parts, P);
  else build_dg(mesh, parts, P);
  return P;
}

}  // namespace sfem
