// extern "C" entry points of the learned smoother.
#include <cstring>
#include <vector>

#include "../../include/simplex_fem.h"
#include "common.hpp"
#include "handles.hpp"

namespace {
using sfem::guarded;

void fill_info(const sfem::TrainStats& st, fem_mlp_train_info* info) {
  if (!info) return;
  std::memset(info, 0, sizeof(*info));
  info->samples = st.samples;
  info->loss_first = st.loss_first;
  info->loss_last = st.loss_last;
  info->seconds = st.seconds;
}
}  // namespace

extern "C" {

int fem_mlp_create(uint64_t seed, fem_mlp** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(out);
    auto h = std::make_unique<fem_mlp>();
    h->s = std::make_unique<sfem::LearnedSmoother>(seed);
    *out = h.release();
  });
}

int fem_mlp_destroy(fem_mlp* mlp) {
  return guarded([&] { delete mlp; });
}

int fem_mlp_n_params(int32_t* n) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(n);
    *n = sfem::MLPDims::NPARAM;
  });
}

int fem_mlp_get_weights(const fem_mlp* mlp, float* host) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(host);
    const std::vector<float> w = mlp->s->host_weights();
    std::memcpy(host, w.data(), sizeof(float) * w.size());
  });
}

int fem_mlp_set_weights(fem_mlp* mlp, const float* host) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(host);
    mlp->s->set_weights(std::vector<float>(host, host + sfem::MLPDims::NPARAM));
  });
}

int fem_mlp_train_params_default(fem_mlp_train_params* p) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(p);
    std::memset(p, 0, sizeof(*p));
    sfem::TrainParams d;
    p->n_sizes = d.n_sizes;
    for (int i = 0; i < 4; ++i) p->sizes[i] = d.sizes[i];
    p->rhs_per_size = d.rhs_per_size;
    p->iterates = d.iterates;
    p->samples = d.samples;
    p->epochs = d.epochs;
    p->batch = d.batch;
    p->lr = d.lr;
    p->jitter = d.jitter;
    p->seed = d.seed;
    p->noise_fraction = d.noise_fraction;
    p->coarse_iterations = d.coarse_iterations;
  });
}

int fem_mlp_generate_and_train(fem_mlp* mlp, const fem_mlp_train_params* p, fem_mlp_train_info* info) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(p);
    sfem::TrainParams t;
    t.n_sizes = p->n_sizes;
    for (int i = 0; i < 4; ++i) t.sizes[i] = p->sizes[i];
    t.rhs_per_size = p->rhs_per_size;
    t.iterates = p->iterates;
    t.samples = p->samples;
    t.epochs = p->epochs;
    t.batch = p->batch;
    t.lr = p->lr;
    t.jitter = p->jitter;
    t.seed = p->seed;
    t.noise_fraction = p->noise_fraction;
    t.coarse_iterations = p->coarse_iterations;
    SFEM_REQUIRE(t.coarse_iterations >= 1 && t.coarse_iterations <= 100, FEM_ERR_ARG,
                 "mlp: coarse_iterations in [1,100]");
    SFEM_REQUIRE(t.noise_fraction >= 0 && t.noise_fraction <= 1, FEM_ERR_ARG, "mlp: noise_fraction in [0,1]");
    for (int i = 0; i < t.n_sizes; ++i)
      SFEM_REQUIRE(t.sizes[i] >= 4 && t.sizes[i] <= 128, FEM_ERR_ARG, "mlp: data mesh sizes must be in [4,128]");
    fill_info(mlp->s->generate_and_train(t), info);
  });
}

int fem_mlp_train(fem_mlp* mlp, const float* X, const float* Y, int32_t n, int32_t epochs, int32_t batch, float lr,
                  uint64_t seed, fem_mlp_train_info* info) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(X);
    SFEM_REQUIRE_PTR(Y);
    fill_info(mlp->s->train(X, Y, n, epochs, batch, lr, seed), info);
  });
}

int fem_mlp_gradient(fem_mlp* mlp, const float* X, const float* Y, int32_t n, float* grad, double* loss,
                     void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(X);
    SFEM_REQUIRE_PTR(Y);
    SFEM_REQUIRE_PTR(grad);
    SFEM_REQUIRE(n > 0, FEM_ERR_ARG, "mlp: n must be positive");
    const double l = mlp->s->gradient(X, Y, n, grad, static_cast<cudaStream_t>(stream));
    if (loss) *loss = l;
  });
}

int fem_mlp_forward(fem_mlp* mlp, const float* X, float* O, int32_t n, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(X);
    SFEM_REQUIRE_PTR(O);
    mlp->s->forward(X, O, n, static_cast<cudaStream_t>(stream));
  });
}

int fem_mlp_forward_tc(fem_mlp* mlp, const float* X, float* O, int32_t n, void* stream) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(X);
    SFEM_REQUIRE_PTR(O);
    mlp->s->forward_tc(X, O, n, static_cast<cudaStream_t>(stream));
  });
}

int fem_mlp_set_tensor_cores(fem_mlp* mlp, int32_t on) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    mlp->s->set_tensor_cores(on != 0);
  });
}

int fem_mlp_status(fem_mlp* mlp, int32_t* timed_out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(timed_out);
    *timed_out = mlp->s->status(true);
  });
}

int fem_mlp_save(const fem_mlp* mlp, const char* path) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mlp);
    SFEM_REQUIRE_PTR(path);
    mlp->s->save(path);
  });
}

int fem_mlp_load(const char* path, fem_mlp** out) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(path);
    SFEM_REQUIRE_PTR(out);
    auto h = std::make_unique<fem_mlp>();
    h->s = sfem::LearnedSmoother::load(path);
    *out = h.release();
  });
}

int fem_mg_set_learned_smoother(fem_mg* mg, fem_mlp* mlp, int32_t fallback) {
  return guarded([&] {
    SFEM_REQUIRE_PTR(mg);
    mg->mg->set_learned(mlp ? mlp->s.get() : nullptr, fallback != 0);
  });
}

}  // extern "C"
