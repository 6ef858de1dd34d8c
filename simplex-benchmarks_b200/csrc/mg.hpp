// Hybrid (p/h/c) multigrid V-cycle and the preconditioned CG solver.
//
// Replaces MultigridPreconditioner (CG/cells_batched/application_ph.cc:
// 1754-2023, h-then-p order application_hp.cc:1735-2008; DG p/c/h orders
// DG/cells_batched/application_phc.cc:3396-3652) and SolverCG +
// PreconditionMG (application_ph.cc:1949-1980).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "operator.hpp"

namespace sfem {

enum MGOrder { MG_ORDER_PH = 0, MG_ORDER_HP = 1 };

struct MGParams {
  int order = MG_ORDER_PH;      // p-coarsening first, then h (reference _ph); or h first (_hp)
  int precision = FEM_FP32;     // level operators, smoothers and transfers
  int smoother_degree = 3;      // Chebyshev degree (reference: 5)
  double smoothing_range = 20;  // lambda_min = lambda_max / range
  int eig_iterations = 10;      // CG steps of the eigenvalue estimate
  double eig_safety = 1.2;      // lambda_max = safety * estimate
  int coarse_n = 4;             // hexes per direction of the coarsest mesh
  int use_graph = 1;            // capture the V-cycle in a CUDA graph
  // DG fine operators: degree at which the DG levels hand over to CG levels
  // on the same mesh (c-transfer).  0: DG P_p .. P_1, then CG P_1 (the
  // reference's phc order); 1: CG P_p right below DG P_p, then the CG p/h
  // ladder of `order` (cph with FEM_MG_PH, chp with FEM_MG_HP).
  int c_transfer = 0;
  // finest-level learned smoothing steps per V-cycle: 1 pre, 2 post, 3 both
  int learned_steps = 3;
  // FP32 CG levels apply their operator on the TF32 tensor cores
  // (cg_cell_tc_kernel, kernel variant 4)
  int tensor_cores = 0;
  // DG fine operators: the CG levels take weak (Nitsche) boundary terms and no
  // constrained DoFs, as in the reference's DG multigrid
  int weak_cg_levels = 0;
};

class Multigrid {
 public:
  virtual ~Multigrid() = default;
  MGParams params;
  virtual int n_levels() const = 0;
  virtual int64_t level_m(int l) const = 0;
  virtual int level_degree(int l) const = 0;
  virtual int level_hexes(int l) const = 0;
  virtual double level_lambda_max(int l) const = 0;
  // dst = V(src), FP64 vectors of the fine operator
  virtual void vcycle(double* dst, const double* src, cudaStream_t s) = 0;
  // level hooks (level-precision vectors of length level_m)
  virtual void level_vmult(int l, void* dst, const void* src, cudaStream_t s) = 0;
  virtual void smooth(int l, void* x, const void* b, bool zero_initial, cudaStream_t s) = 0;
  virtual void prolongate_add(int l, void* dst, const void* src, cudaStream_t s) = 0;  // l-1 -> l
  virtual void restrict_add(int l, void* dst, const void* src, cudaStream_t s) = 0;    // l -> l-1
  virtual void coarse_solve(void* dst, const void* src, cudaStream_t s) = 0;
  virtual Operator& level_operator(int l) = 0;
  // finest-level smoothing by a learned per-cell MLP (nullptr: Chebyshev);
  // with fallback the Chebyshev smoother returns on the first poor cycle
  virtual void set_learned(class LearnedSmoother* s, bool fallback) = 0;
  // switch back to Chebyshev (returns true if the learned smoother was active)
  virtual bool fallback_to_chebyshev() = 0;
  virtual bool learned_active() const = 0;
  // a new outer solve starts: a learned smoother that fell back is used again
  virtual void on_solve_start() = 0;
  // x = P y, y ~ A_c^-1 R r by `iterations` V-cycle iterations on the level below
  // the finest: the coarse-grid correction of the FP64 fine residual r (no
  // finest-level smoothing); with enough iterations r - A x is A-orthogonal to
  // the coarse space
  virtual void coarse_correction(const double* r, double* x, int iterations, cudaStream_t s) = 0;
};

std::unique_ptr<Multigrid> make_multigrid(const Operator& fine, const MGParams& p);

struct SolveInfo {
  int iterations = 0;
  int status = 0;  // FEM_OK, FEM_ERR_NOT_CONVERGED, FEM_ERR_BREAKDOWN, FEM_ERR_NONFINITE
  double r0 = 0, rn = 0;
  int fallback_iteration = 0;  // iteration at which a learned smoother was replaced (0: never)
};

// Preconditioner interface for the CG solver (FP64 vectors of the fine operator)
class Preconditioner {
 public:
  virtual ~Preconditioner() = default;
  virtual void apply(double* dst, const double* src, cudaStream_t s) = 0;
  // the outer iteration reduced the residual by less than 2x: change strategy
  // if the preconditioner has another one (returns true if it did)
  virtual bool on_poor_reduction() { return false; }
  virtual void on_solve_start() {}
};

class CGSolver {
 public:
  // flexible: Polak-Ribiere beta (for preconditioners that change between applications)
  CGSolver(Operator& A, Preconditioner* M, bool flexible);
  ~CGSolver();
  CGSolver(const CGSolver&) = delete;
  CGSolver& operator=(const CGSolver&) = delete;
  SolveInfo solve(double* x, const double* b, double rtol, int maxit, cudaStream_t s);
  double dot(const double* x, const double* y, cudaStream_t s);

 private:
  // (x, y) into the device scalar sc_[slot], no host synchronisation
  void dot_to(const double* x, const double* y, int slot, cudaStream_t s);
  Operator& A_;
  Preconditioner* M_;
  bool flexible_;
  DevBuf<double> r_, z_, p_, q_, zold_, partial_;
  // device scalars of the iteration: [0],[1] (r,z) of this and the next
  // iteration (alternating), [2] (p,Ap), [3] (r,r), [4] (r,z_old)
  DevBuf<double> sc_;
  double* host_ = nullptr;  // pinned: (p,Ap), (r,r) read back once per iteration
};

class MGPreconditioner final : public Preconditioner {
 public:
  explicit MGPreconditioner(Multigrid& mg) : mg_(mg) {}
  void apply(double* dst, const double* src, cudaStream_t s) override { mg_.vcycle(dst, src, s); }
  bool on_poor_reduction() override { return mg_.fallback_to_chebyshev(); }
  void on_solve_start() override { mg_.on_solve_start(); }

 private:
  Multigrid& mg_;
};

class JacobiPreconditioner final : public Preconditioner {
 public:
  explicit JacobiPreconditioner(Operator& A);
  void apply(double* dst, const double* src, cudaStream_t s) override;

 private:
  DevBuf<double> inv_;
};

}  // namespace sfem
