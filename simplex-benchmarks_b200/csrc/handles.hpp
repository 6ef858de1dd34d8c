// Definitions of the opaque C ABI handles (shared by the extern "C" files).
#pragma once
#include <memory>

#include "learned.hpp"
#include "mesh.hpp"
#include "mg.hpp"
#include "operator.hpp"
#include "partition.hpp"

struct fem_mesh {
  sfem::Mesh mesh;
};
struct fem_op {
  std::unique_ptr<sfem::Operator> op;
};
struct fem_part {
  sfem::Partition p;
};
struct fem_batch {
  std::unique_ptr<sfem::Batch> batch;
};
struct fem_mg {
  std::unique_ptr<sfem::Multigrid> mg;
};
struct fem_mlp {
  std::unique_ptr<sfem::LearnedSmoother> s;
};
struct fem_cg {
  std::unique_ptr<sfem::Preconditioner> own_precond;
  std::unique_ptr<sfem::CGSolver> solver;
};

namespace sfem {
OpConfig op_config(int32_t degree, int32_t kind, int32_t precision, const fem_op_params* params);

// Runs f, converting exceptions into a status code and the last-error string.
template <class F>
int guarded(F&& f) {
  try {
    f();
    return FEM_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return FEM_ERR_INTERNAL;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FEM_ERR_INTERNAL;
  }
}
}  // namespace sfem

#define SFEM_REQUIRE_PTR(p) SFEM_REQUIRE((p) != nullptr, FEM_ERR_ARG, #p " is NULL")
