// Domain decomposition of a mesh over ranks (host side, no GPU needed).
//
// The reference distributes its triangulation over MPI ranks by z-order
// (parallel::fullydistributed::Triangulation with a z-order partition,
// CG/cells_batched/application.cc:1773-1801) and exchanges ghost values inside
// MatrixFree::cell_loop / loop (update_ghost_values before the cell and face
// integrals, compress(VectorOperation::add) after them, DG:
// DG/cells_batched/application.cc:1303-1316).  Here a part is a contiguous
// range of the hierarchical (Morton) cell order, cut at 4x4x4-hex cube
// boundaries when the mesh has enough cubes, so that every part keeps the
// cube and hex kernels.
//
// Local vector layout of part r (the operator built on it works on it):
//   [ owned entries | ghost entries ]
//   CG: DoFs; a DoF belongs to the part of the first cell (in cell order) that
//       touches it; the ghosts are the DoFs of r's cells owned elsewhere.
//   DG: whole cell blocks (n_components x k values); the ghosts are the
//       face neighbours of r's cells in other parts.
// Owned entries keep the global order; ghosts are sorted by (owner, global
// index).  For every peer the send list (owned entries the peer holds as
// ghosts) and the receive list (ghosts the peer owns) are both in ascending
// global index, so they match entry by entry on the two sides.
//   ghost update (before vmult): owner -> ghost copy along these lists;
//   CG compress (after vmult):   ghost -> owner add along the same lists.
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "mesh.hpp"

namespace sfem {

struct PartPeer {
  int rank = 0;
  std::vector<int64_t> send;  // local indices of owned entries, ascending global index
  std::vector<int64_t> recv;  // local indices of ghost entries, ascending global index
};

struct Partition {
  int kind = 0, degree = 1, n_components = 1, n_parts = 1, part = 0;
  int64_t cell_begin = 0, cell_end = 0;  // owned cells [begin, end) of the global order
  int64_t n_owned = 0, n_ghost = 0;      // local vector entries
  int64_t n_global = 0;                  // global vector length
  std::vector<int64_t> gidx;             // global index of every local entry
  std::vector<PartPeer> peers;           // ascending rank
  // the local mesh the operator runs on: CG the owned cells; DG the owned
  // cells then the ghost cells (nb = -2 on faces to cells outside it)
  std::shared_ptr<Mesh> local;
  CGDofs dofs;                     // CG: local numbering, global constraints
  std::vector<uint8_t> identity;   // CG: owned constrained DoFs (rows dst = src)
};

// cell range of part `part` of `n_parts` over n_cells cells
void part_range(int64_t n_cells, int n_parts, int part, int64_t& begin, int64_t& end);

Partition build_partition(const Mesh& mesh, int degree, int kind, int n_components, int n_parts, int part);

}  // namespace sfem
