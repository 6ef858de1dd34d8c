// extern "C" entry points of the domain decomposition (partition.hpp).
#include <cstring>
#include <memory>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "handles.hpp"

namespace {
using sfem::guarded;
}

extern "C" {

int fem_part_create(const fem_mesh* mesh, int32_t degree, int32_t kind, int32_t n_components, int32_t n_parts,
                    int32_t part, fem_part** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mesh);
    SFEM_REQUIRE_PTR(out);
    auto p = std::make_unique<fem_part>();
    p->p = sfem::build_partition(mesh->mesh, degree, kind, n_components > 0 ? n_components : 1, n_parts, part);
    *out = p.release();
  });
}

int fem_part_destroy(fem_part* part) {
  return guarded([&] { delete part; });
}

int fem_part_sizes(const fem_part* part, int64_t* n_owned, int64_t* n_ghost, int64_t* n_global, int64_t* cell_begin,
                   int64_t* cell_end, int32_t* n_peers) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(part);
    const sfem::Partition& P = part->p;
    if (n_owned) *n_owned = P.n_owned;
    if (n_ghost) *n_ghost = P.n_ghost;
    if (n_global) *n_global = P.n_global;
    if (cell_begin) *cell_begin = P.cell_begin;
    if (cell_end) *cell_end = P.cell_end;
    if (n_peers) *n_peers = int32_t(P.peers.size());
  });
}

int fem_part_global_index(const fem_part* part, int64_t* gidx) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(part);
    SFEM_REQUIRE_PTR(gidx);
    std::memcpy(gidx, part->p.gidx.data(), part->p.gidx.size() * sizeof(int64_t));
  });
}

int fem_part_peer(const fem_part* part, int32_t i, int32_t* rank, int64_t* n_send, int64_t* n_recv) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(part);
    SFEM_REQUIRE(i >= 0 && i < int32_t(part->p.peers.size()), FEM_ERR_ARG, "fem_part_peer: peer index out of range");
    const sfem::PartPeer& q = part->p.peers[i];
    if (rank) *rank = q.rank;
    if (n_send) *n_send = int64_t(q.send.size());
    if (n_recv) *n_recv = int64_t(q.recv.size());
  });
}

int fem_part_halo(const fem_part* part, int32_t i, int64_t* send, int64_t* recv) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(part);
    SFEM_REQUIRE(i >= 0 && i < int32_t(part->p.peers.size()), FEM_ERR_ARG, "fem_part_halo: peer index out of range");
    const sfem::PartPeer& q = part->p.peers[i];
    if (send) std::memcpy(send, q.send.data(), q.send.size() * sizeof(int64_t));
    if (recv) std::memcpy(recv, q.recv.data(), q.recv.size() * sizeof(int64_t));
  });
}

int fem_op_create_part(const fem_part* part, int32_t precision, const fem_op_params* params, fem_op** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(part);
    SFEM_REQUIRE_PTR(out);
    const sfem::Partition& P = part->p;
    sfem::OpConfig cfg = sfem::op_config(P.degree, P.kind, precision, params);
    if (P.kind == FEM_HELMHOLTZ) cfg.n_components = P.n_components;
    SFEM_REQUIRE(cfg.n_components == P.n_components, FEM_ERR_ARG,
                 "fem_op_create_part: n_components differs from the partition's");
    auto o = std::make_unique<fem_op>();
    o->op = sfem::make_local_operator(P.local, &P.dofs, &P.identity, cfg);
    SFEM_REQUIRE(o->op->m == P.n_owned + P.n_ghost, FEM_ERR_INTERNAL, "partition: local vector length");
    *out = o.release();
  });
}

}  // extern "C"
