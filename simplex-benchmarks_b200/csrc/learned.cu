// Learned finest-level smoother: weights, binding to a P3 level, training on
// residual/error pairs produced by the multigrid-preconditioned CG itself.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "learned.hpp"
#include "mg.hpp"
#include "mlp.cuh"
#include "mlp_tc.cuh"
#include "vector_kernels.cuh"

namespace sfem {

namespace {

__global__ void gather_rows(int n, int width, const int32_t* __restrict__ perm, const float* __restrict__ in,
                            float* __restrict__ out) {
  const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (t >= int64_t(n) * width) return;
  const int64_t r = t / width, c = t % width;
  out[t] = in[int64_t(perm[r]) * width + c];
}

// persistent tensor-core launch: 2 CTAs of 4 groups per SM (each CTA holds
// 256 of the 512 tensor-memory columns and 89 KB of shared memory)
template <int MODE, typename T>
void launch_tc(int64_t n, const int32_t* dofs, const float* feat, const float* winv, const __nv_bfloat16* wb,
               const T* r, T* z, float* zout, int* status, cudaStream_t s) {
  static std::atomic<uint64_t> configured{0};
  auto kern = mlp_tc_kernel<MODE, T>;
  int dev = 0, sms = 0;
  SFEM_CUDA(cudaGetDevice(&dev));
  once_per_device(configured, dev, [&] {
    SFEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
  });
  SFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t tiles = (n + tc::TILE - 1) / tc::TILE;
  const int64_t groups = (tiles + tc::GROUPS - 1) / tc::GROUPS;
  const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(groups, int64_t(sms) * 2)));
  kern<<<grid, tc::THREADS, tc::SMEM_BYTES, s>>>(n, dofs, feat, winv, wb, r, z, zout, status);
  SFEM_CUDA(cudaGetLastError());
}

uint64_t fnv1a(const void* data, size_t n) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint64_t h = 1469598103934665603ULL;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}

}  // namespace

LearnedSmoother::LearnedSmoother(uint64_t seed) {
  using D = MLPDims;
  std::vector<float> w(NP, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / (rows + cols));
    for (int i = 0; i < rows * cols; ++i) {
      const double u = double(rng() >> 11) * (1.0 / 9007199254740992.0);
      w[off + i] = float((2.0 * u - 1.0) * a);
    }
  };
  fill(D::OFF_W1, D::NH, D::NIN);
  fill(D::OFF_W2, D::NH, D::NH);
  fill(D::OFF_W3, D::NOUT, D::NH);
  w_.alloc(NP);
  m_.alloc(NP);
  v_.alloc(NP);
  g_.alloc(NP);
  loss_.alloc(1);
  wb_.alloc(NP);
  status_.alloc(1);
  SFEM_CUDA(cudaMemset(status_.p, 0, sizeof(int)));
  set_weights(w);
}

std::vector<float> LearnedSmoother::host_weights() const {
  std::vector<float> h(NP);
  SFEM_CUDA(cudaMemcpy(h.data(), w_.p, sizeof(float) * NP, cudaMemcpyDeviceToHost));
  return h;
}

void LearnedSmoother::set_weights(const std::vector<float>& w) {
  SFEM_REQUIRE(int(w.size()) == NP, FEM_ERR_ARG, "mlp: wrong number of parameters");
  w_.upload(w);
  SFEM_CUDA(cudaMemset(m_.p, 0, sizeof(float) * NP));
  SFEM_CUDA(cudaMemset(v_.p, 0, sizeof(float) * NP));
  adam_t_ = 0;
  round_weights(nullptr);
  SFEM_CUDA(cudaDeviceSynchronize());
}

void LearnedSmoother::round_weights(cudaStream_t s) {
  mlp_round_weights<<<(NP + 255) / 256, 256, 0, s>>>(NP, w_.p, wb_.p);
  SFEM_CUDA(cudaGetLastError());
}

LearnedSmoother::Bound& LearnedSmoother::bind(const Operator& op) {
  auto it = bound_.find(&op);
  if (it != bound_.end()) return *it->second;
  SFEM_REQUIRE(op.cfg.kind == FEM_CG && op.cfg.degree == 3 && op.mesh, FEM_ERR_ARG,
               "learned smoother: needs a CG P3 operator");
  auto b = std::make_unique<Bound>();
  const Mesh& mesh = *op.mesh;
  std::vector<float> feat(10 * size_t(op.n_cells));
  for (int64_t c = 0; c < op.n_cells; ++c) {
    const CellGeometry g = cell_geometry(mesh, c);
    const double h = std::cbrt(std::fabs(g.det));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) feat[10 * c + 3 * i + j] = float(g.J[i][j] / h);
    feat[10 * c + 9] = float(1.0 / h);
  }
  std::vector<int> count(op.m, 0);
  for (size_t i = 0; i < op.cell_dofs.size(); ++i) count[op.cell_dofs[i]]++;
  std::vector<float> winv(op.m);
  for (int64_t i = 0; i < op.m; ++i) winv[i] = count[i] ? 1.0f / count[i] : 0.0f;
  b->feat.upload(feat);
  b->winv.upload(winv);
  auto& ref = *b;
  bound_[&op] = std::move(b);
  return ref;
}

void LearnedSmoother::apply(const Operator& op, const void* r, void* z, cudaStream_t s) {
  Bound& b = bind(op);
  if (tensor_cores_) {
    if (op.cfg.precision == FEM_FP64)
      launch_tc<0, double>(op.n_cells, op.device_dof_table(), b.feat.p, b.winv.p, wb_.p,
                           static_cast<const double*>(r), static_cast<double*>(z), nullptr, status_.p, s);
    else
      launch_tc<0, float>(op.n_cells, op.device_dof_table(), b.feat.p, b.winv.p, wb_.p,
                          static_cast<const float*>(r), static_cast<float*>(z), nullptr, status_.p, s);
    return;
  }
  const unsigned grid = unsigned(std::min<int64_t>((op.n_cells + 127) / 128, 148 * 8));
  if (op.cfg.precision == FEM_FP64)
    mlp_smooth_kernel<double><<<grid, 128, 0, s>>>(op.n_cells, op.device_dof_table(), b.feat.p, b.winv.p, wb_.p,
                                                   static_cast<const double*>(r), static_cast<double*>(z));
  else
    mlp_smooth_kernel<float><<<grid, 128, 0, s>>>(op.n_cells, op.device_dof_table(), b.feat.p, b.winv.p, wb_.p,
                                                  static_cast<const float*>(r), static_cast<float*>(z));
  SFEM_CUDA(cudaGetLastError());
}

double LearnedSmoother::gradient(const float* X, const float* Y, int n, float* grad, cudaStream_t s) {
  static std::atomic<uint64_t> configured{0};
  const int smem = 2 * NP * int(sizeof(float));
  int dev = 0;
  SFEM_CUDA(cudaGetDevice(&dev));
  once_per_device(configured, dev, [&] {
    SFEM_CUDA(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  });
  SFEM_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * NP, s));
  SFEM_CUDA(cudaMemsetAsync(loss_.p, 0, sizeof(float), s));
  const int grid = std::min((n + 127) / 128, 148 * 2);
  mlp_grad_kernel<<<grid, 128, smem, s>>>(n, X, Y, wb_.p, grad, loss_.p, 1.0f / float(n));
  SFEM_CUDA(cudaGetLastError());
  float h = 0;
  SFEM_CUDA(cudaMemcpyAsync(&h, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, s));
  SFEM_CUDA(cudaStreamSynchronize(s));
  return double(h) / n;
}

void LearnedSmoother::forward(const float* X, float* O, int n, cudaStream_t s) {
  const int grid = std::max(1, std::min((n + 127) / 128, 148 * 8));
  mlp_forward_kernel<<<grid, 128, 0, s>>>(n, X, wb_.p, O);
  SFEM_CUDA(cudaGetLastError());
}

void LearnedSmoother::forward_tc(const float* X, float* O, int n, cudaStream_t s) {
  SFEM_REQUIRE(n >= 0, FEM_ERR_ARG, "mlp: negative sample count");
  launch_tc<1, float>(n, nullptr, X, nullptr, wb_.p, nullptr, nullptr, O, status_.p, s);
}

int LearnedSmoother::status(bool clear) {
  int v = 0;
  SFEM_CUDA(cudaMemcpy(&v, status_.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (clear && v) SFEM_CUDA(cudaMemset(status_.p, 0, sizeof(int)));
  return v;
}

TrainStats LearnedSmoother::train(const float* X, const float* Y, int n, int epochs, int batch, float lr,
                                  uint64_t seed) {
  using D = MLPDims;
  SFEM_REQUIRE(n > 0 && epochs > 0 && batch > 0, FEM_ERR_ARG, "mlp: bad training parameters");
  const auto t0 = std::chrono::steady_clock::now();
  TrainStats st;
  st.samples = n;
  DevBuf<float> Xp(size_t(n) * D::NIN), Yp(size_t(n) * D::NOUT);
  DevBuf<int32_t> perm(n);
  std::vector<int32_t> hp(n);
  for (int i = 0; i < n; ++i) hp[i] = i;
  std::mt19937_64 rng(seed);
  cudaStream_t s = nullptr;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(hp.begin(), hp.end(), rng);
    perm.upload(hp);
    gather_rows<<<unsigned((int64_t(n) * D::NIN + 255) / 256), 256, 0, s>>>(n, D::NIN, perm.p, X, Xp.p);
    gather_rows<<<unsigned((int64_t(n) * D::NOUT + 255) / 256), 256, 0, s>>>(n, D::NOUT, perm.p, Y, Yp.p);
    double ep_loss = 0;
    int nb = 0;
    for (int off = 0; off + batch <= n || (off < n && nb == 0); off += batch) {
      const int cnt = std::min(batch, n - off);
      ep_loss += gradient(Xp.p + int64_t(off) * D::NIN, Yp.p + int64_t(off) * D::NOUT, cnt, g_.p, s);
      ++adam_t_;
      const float c1 = 1.0f / (1.0f - std::pow(b1, float(adam_t_)));
      const float c2 = 1.0f / (1.0f - std::pow(b2, float(adam_t_)));
      mlp_adam_kernel<<<(NP + 255) / 256, 256, 0, s>>>(NP, w_.p, g_.p, m_.p, v_.p, lr, b1, b2, eps, c1, c2);
      round_weights(s);
      ++nb;
    }
    ep_loss /= std::max(nb, 1);
    if (ep == 0) st.loss_first = ep_loss;
    st.loss_last = ep_loss;
  }
  SFEM_CUDA(cudaDeviceSynchronize());
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

TrainStats LearnedSmoother::generate_and_train(const TrainParams& p) {
  using D = MLPDims;
  SFEM_REQUIRE(p.n_sizes >= 1 && p.n_sizes <= 4 && p.rhs_per_size >= 1 && p.iterates >= 1 && p.samples > 0,
               FEM_ERR_ARG, "mlp: bad data parameters");
  const int per_state = std::max(1, p.samples / (p.n_sizes * p.rhs_per_size * p.iterates));
  const int total = per_state * p.n_sizes * p.rhs_per_size * p.iterates;
  DevBuf<float> X(size_t(total) * D::NIN), Y(size_t(total) * D::NOUT);
  DevBuf<int32_t> valid(size_t(per_state) * p.iterates), sel(size_t(per_state) * p.iterates);
  int filled = 0;
  std::mt19937_64 rng(p.seed);
  cudaStream_t s = nullptr;
  for (int si = 0; si < p.n_sizes; ++si) {
    for (int ri = 0; ri < p.rhs_per_size; ++ri) {
      const uint64_t rhs_seed = p.seed + uint64_t(si) * 100 + ri;
      MeshDescription md;
      for (int a = 0; a < 3; ++a) md.n[a] = p.sizes[si];
      md.jitter = p.jitter;
      md.seed = rhs_seed;
      Mesh mesh = build_kuhn_mesh(md);
      OpConfig cfg;
      cfg.degree = 3;
      cfg.kind = FEM_CG;
      cfg.precision = FEM_FP64;
      auto op = make_operator(mesh, cfg);
      MGParams mp;
      mp.precision = FEM_FP32;
      auto mg = make_multigrid(*op, mp);
      MGPreconditioner pre(*mg);
      CGSolver solver(*op, &pre, false);
      RhsDesc rd;
      rd.kind = 0;
      rd.n_modes = 8;
      std::mt19937_64 krng(rhs_seed);
      for (int m = 0; m < 8; ++m) {
        for (int a = 0; a < 3; ++a) rd.k[m][a] = 1.0 + 5.0 * double(krng() >> 11) * (1.0 / 9007199254740992.0);
        rd.amp[m] = 1.0;
      }
      const int64_t m = op->m;
      DevBuf<double> b(m), xs(m), x(m), r(m), e(m), cc(m);
      op->rhs(rd, b.p, s);
      SFEM_CUDA(cudaMemsetAsync(xs.p, 0, sizeof(double) * m, s));
      solver.solve(xs.p, b.p, 1e-12, 200, s);
      Bound& bd = bind(*op);
      auto take = [&](int count, const double* rr, const double* ee) {
        std::vector<int32_t> hs(count);
        for (auto& c : hs) c = int32_t(rng() % uint64_t(op->n_cells));
        SFEM_CUDA(cudaMemcpy(sel.p, hs.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice));
        mlp_extract_kernel<double><<<(count + 127) / 128, 128, 0, s>>>(
            count, sel.p, op->n_cells, op->device_dof_table(), bd.feat.p, rr, ee, X.p + int64_t(filled) * D::NIN,
            Y.p + int64_t(filled) * D::NOUT, valid.p);
        SFEM_CUDA(cudaGetLastError());
        SFEM_CUDA(cudaStreamSynchronize(s));
        filled += count;
      };
      const int n_noise = int(std::lround(p.noise_fraction * per_state * p.iterates));
      const int n_solver_each = (per_state * p.iterates - n_noise) / p.iterates;
      if (n_noise > 0) {
        // white-noise error field (zero on constrained DoFs) and its residual
        std::vector<double> hn(m);
        for (int64_t i = 0; i < m; ++i)
          hn[i] = op->constrained[i] ? 0.0 : 2.0 * double(rng() >> 11) * (1.0 / 9007199254740992.0) - 1.0;
        e.upload(hn);
        op->vmult(r.p, e.p, s);
        take(n_noise, r.p, e.p);
      }
      for (int k = 0; k < p.iterates && n_solver_each > 0; ++k) {
        SFEM_CUDA(cudaMemsetAsync(x.p, 0, sizeof(double) * m, s));
        if (k > 0) solver.solve(x.p, b.p, 1e-30, k, s);
        op->vmult(r.p, x.p, s);
        vec_residual<double><<<grid_for(m), 256, 0, s>>>(m, b.p, r.p, r.p);  // r = b - A x
        SFEM_CUDA(cudaMemcpyAsync(e.p, xs.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        vec_axpby<double><<<grid_for(m), 256, 0, s>>>(m, -1.0, x.p, 1.0, e.p);  // e = x* - x
        // what the smoother has to remove: the part left after the (accurate)
        // coarse-grid correction x_cc of this residual, e - x_cc, with residual
        // r - A x_cc: the component outside the coarse space
        mg->coarse_correction(r.p, x.p, p.coarse_iterations, s);
        vec_axpby<double><<<grid_for(m), 256, 0, s>>>(m, -1.0, x.p, 1.0, e.p);
        op->vmult(cc.p, x.p, s);
        vec_axpby<double><<<grid_for(m), 256, 0, s>>>(m, -1.0, cc.p, 1.0, r.p);
        take(n_solver_each, r.p, e.p);
      }
      SFEM_CUDA(cudaStreamSynchronize(s));
      bound_.erase(op.get());
    }
  }
  return train(X.p, Y.p, filled, p.epochs, p.batch, p.lr, p.seed + 7);
}

void LearnedSmoother::save(const std::string& path) const {
  const std::vector<float> w = host_weights();
  std::ofstream f(path, std::ios::binary);
  SFEM_REQUIRE(f.good(), FEM_ERR_ARG, "mlp: cannot write " + path);
  std::ostringstream hdr;
  hdr << "{\"format\":\"simplexfem-mlp-1\",\"layers\":[29,64,64,20],\"activation\":\"gelu\",\"params\":" << NP
      << ",\"dtype\":\"float32\",\"fnv1a64\":" << fnv1a(w.data(), sizeof(float) * NP) << "}\n";
  const std::string h = hdr.str();
  f.write(h.data(), std::streamsize(h.size()));
  f.write(reinterpret_cast<const char*>(w.data()), std::streamsize(sizeof(float) * NP));
  SFEM_REQUIRE(f.good(), FEM_ERR_ARG, "mlp: write failed for " + path);
}

std::unique_ptr<LearnedSmoother> LearnedSmoother::load(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  SFEM_REQUIRE(f.good(), FEM_ERR_ARG, "mlp: cannot read " + path);
  std::string hdr;
  std::getline(f, hdr);
  SFEM_REQUIRE(hdr.find("simplexfem-mlp-1") != std::string::npos, FEM_ERR_ARG, "mlp: not a weight file");
  std::vector<float> w(NP);
  f.read(reinterpret_cast<char*>(w.data()), std::streamsize(sizeof(float) * NP));
  SFEM_REQUIRE(f.gcount() == std::streamsize(sizeof(float) * NP), FEM_ERR_ARG, "mlp: truncated weight file");
  const auto pos = hdr.find("\"fnv1a64\":");
  SFEM_REQUIRE(pos != std::string::npos, FEM_ERR_ARG, "mlp: header without checksum");
  const uint64_t want = std::stoull(hdr.substr(pos + 10));
  SFEM_REQUIRE(want == fnv1a(w.data(), sizeof(float) * NP), FEM_ERR_ARG, "mlp: checksum mismatch");
  auto s = std::make_unique<LearnedSmoother>(0);
  s->set_weights(w);
  return s;
}

}  // namespace sfem
