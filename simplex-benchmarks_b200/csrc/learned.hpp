// Learned finest-level smoother (per-cell MLP) for the hybrid multigrid.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "mlp_dims.hpp"
#include "operator.hpp"

namespace sfem {

struct TrainParams {
  int n_sizes = 2;
  int sizes[4] = {16, 32, 0, 0};  // hexes per direction of the data meshes
  int rhs_per_size = 4;           // random sin-mode loads per mesh (seeds 1000+)
  int iterates = 6;               // MG-CG iterates per solve used as samples
  int samples = 200000;
  int epochs = 30;
  int batch = 2048;
  float lr = 2e-3f;
  double jitter = 0.1;
  uint64_t seed = 1000;
  // fraction of the samples taken from white-noise errors e (r = A e) on the
  // same meshes: high-frequency errors, the part a smoother has to remove
  double noise_fraction = 0.0;
  // V-cycle iterations of the coarse-grid correction removed from the solver's
  // errors before they become targets
  int coarse_iterations = 12;
};

struct TrainStats {
  int samples = 0;
  double loss_first = 0, loss_last = 0;
  double seconds = 0;
};

class LearnedSmoother {
 public:
  explicit LearnedSmoother(uint64_t seed);
  static constexpr int NP = MLPDims::NPARAM;
  std::vector<float> host_weights() const;
  void set_weights(const std::vector<float>& w);
  // z += S(r) on a P3 CG operator's DoF vectors (T = float or double)
  void apply(const Operator& op, const void* r, void* z, cudaStream_t s);
  // training on device arrays X [n][29], Y [n][20]
  TrainStats train(const float* X, const float* Y, int n, int epochs, int batch, float lr, uint64_t seed);
  // the whole pipeline: data from MG-CG solves on Kuhn meshes, then training
  TrainStats generate_and_train(const TrainParams& p);
  // gradient of mean ||o - y||^2 over n samples (device arrays); grad on device [NP]
  double gradient(const float* X, const float* Y, int n, float* grad, cudaStream_t s);
  void forward(const float* X, float* O, int n, cudaStream_t s);
  // the same forward on the tensor cores (tcgen05, BF16 activations)
  void forward_tc(const float* X, float* O, int n, cudaStream_t s);
  // smoothing on the tensor cores (default) or on the CUDA cores
  void set_tensor_cores(bool on) { tensor_cores_ = on; }
  bool tensor_cores() const { return tensor_cores_; }
  // 1 if a tensor-core launch gave up on a bounded wait since the last call
  int status(bool clear);
  void save(const std::string& path) const;
  static std::unique_ptr<LearnedSmoother> load(const std::string& path);
  const __nv_bfloat16* bf16() const { return wb_.p; }

 private:
  struct Bound {
    DevBuf<float> feat;  // [n_cells][10]
    DevBuf<float> winv;  // [m]
  };
  Bound& bind(const Operator& op);
  void round_weights(cudaStream_t s);
  DevBuf<float> w_, m_, v_, g_, loss_;
  DevBuf<__nv_bfloat16> wb_;
  DevBuf<int> status_;
  bool tensor_cores_ = true;
  int adam_t_ = 0;
  std::map<const Operator*, std::unique_ptr<Bound>> bound_;
};

}  // namespace sfem
