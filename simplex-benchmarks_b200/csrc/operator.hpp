// Matrix-free operators on the GPU: the object behind fem_op.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "mesh.hpp"

namespace sfem {

// Owning device buffer.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      cudaError_t e = cudaMalloc(&p, count * sizeof(T));
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        throw Error(FEM_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      }
    }
  }
  void upload(const T* host, size_t count) {
    if (count != n) alloc(count);
    if (count) {
      cudaError_t e = cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) throw Error(FEM_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    }
  }
  void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct OpConfig {
  int degree = 2;
  int kind = FEM_CG;
  int precision = FEM_FP64;
  double mass = 0.0;
  int n_components = 1;
  int penalty = FEM_PENALTY_REFERENCE;
  int kernel_variant = 0;  // 0: tuned default (see fem_op_params.kernel_variant)
  bool weak_bc = false;    // CG: weak (Nitsche) Dirichlet on the boundary faces, no constrained DoFs
};

struct HostPipe;  // staging buffers and streams of vmult_host (host_vmult.cu)

class Operator {
 public:
  virtual ~Operator() = default;
  std::shared_ptr<HostPipe> host_pipe;  // created by the first vmult_host
  OpConfig cfg;
  const Mesh* mesh = nullptr;  // the mesh the operator was built on (must outlive it)
  std::shared_ptr<const Mesh> owned_mesh;  // set when the operator keeps its own (partition-local) mesh
  int K = 0;               // DoFs per cell and component
  int64_t n_cells = 0;
  int64_t m = 0;           // vector length
  int64_t n_interior_faces = 0, n_boundary_faces = 0;
  std::vector<int32_t> cell_dofs;    // host copy of the dof map (CG)
  std::vector<uint8_t> constrained;  // host mask [m]
  std::vector<double> support;       // host support points [m/NC][3]

  size_t elem_size() const { return cfg.precision == FEM_FP64 ? 8 : 4; }
  virtual void vmult(void* dst, const void* src, cudaStream_t s) = 0;
  // phase 1 / phase 2 of vmult (see fem_op_vmult_phase)
  virtual void vmult_phase(void* dst, const void* src, int phase, cudaStream_t s) = 0;
  virtual void diagonal(void* diag, cudaStream_t s) = 0;
  // CG: device table [K][n_cells] of global DoFs, -1 at constrained ones
  virtual const int32_t* device_dof_table() const { return nullptr; }
  // Device scratch one vmult needs (DG: the published face traces; CG: none).
  virtual size_t scratch_bytes() const { return 0; }
  // vmult with the scratch supplied by the caller instead of the operator's own.
  virtual void vmult_with_scratch(void* dst, const void* src, void* scratch, size_t bytes, cudaStream_t s) {
    throw Error(FEM_ERR_ARG, "this operator kind uses no scratch memory");
  }
  void inverse_diagonal(void* diag, cudaStream_t s);
  // CG: dense element matrices of the cell operator, device [n_cells][K][K]
  virtual void element_matrices(void* out, cudaStream_t s) {
    throw Error(FEM_ERR_ARG, "element matrices: CG operators only");
  }
  // device-side status bits of the operator's kernels since the last call
  // (bit 0: a tensor-core kernel gave up on a bounded wait); clear resets them
  virtual int status(bool clear) { return 0; }
  // flops of the fused kernels and algorithmic bytes (src+dst once, index and
  // geometry data once) of one vmult
  virtual void work(double& flops, double& bytes) const = 0;
  // dst = (f, v_i) for the load described by `rhs` (CG: 0 on constrained DoFs)
  virtual void rhs(const struct RhsDesc& rhs, void* dst, cudaStream_t s);
};

// f(x) = sum_m amp[m] sin(k[m] . x)            (kind 0, sum of plane waves)
//      = sum_m amp[m] prod_d sin(k[m][d] x_d)   (kind 1, products)
struct RhsDesc {
  int kind = 0;
  int n_modes = 0;
  double k[16][3] = {};
  double amp[16] = {};
};
double rhs_value(const RhsDesc& r, const double* x);

std::unique_ptr<Operator> make_operator(const Mesh& mesh, const OpConfig& cfg);
// CG Laplace on a curved mesh (per-quadrature-point metric, curved.cu)
std::unique_ptr<Operator> make_curved_cg_operator(const Mesh& mesh, const OpConfig& cfg);
// Operator on a partition-local mesh it keeps alive: CG takes the given
// numbering (dofs) and identity rows; DG / Helmholtz read nb == -2 as an
// interior face whose neighbour is not in the local mesh.
std::unique_ptr<Operator> make_local_operator(std::shared_ptr<const Mesh> mesh, const CGDofs* dofs,
                                              const std::vector<uint8_t>* identity, const OpConfig& cfg);

// Outcome of an autotuning run (autotune.hpp).
struct TuneResult {
  int variant = 0;
  bool cached = false;
  std::vector<double> us;  // median us per candidate (index = variant - 1), 0 = not timed
};

// Batched multi-problem DG launch.
class Batch {
 public:
  virtual ~Batch() = default;
  virtual void vmult(void* const* dst, const void* const* src, cudaStream_t s) = 0;
  // time the kernel variants on the whole batch and keep the fastest
  virtual TuneResult tune(int reps, bool use_cache) = 0;
  virtual int variant() const = 0;
  virtual void set_variant(int v) = 0;
};
std::unique_ptr<Batch> make_batch(const std::vector<Operator*>& ops);

// y = A x for a CSR matrix on the device (row_ptr int64, col int32)
void csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col, const void* val, const void* x, void* y,
              int precision, cudaStream_t s);

}  // namespace sfem
