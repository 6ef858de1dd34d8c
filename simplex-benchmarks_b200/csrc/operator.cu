// Operator set-up (geometry, penalties, index tables) and kernel dispatch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "kernels_cg.cuh"
#include "kernels_cg_tc.cuh"
#include "kernels_dg.cuh"
#include "kernels_dg2.cuh"
#include "kernels_dg3.cuh"
#include "autotune.hpp"
#include "operator.hpp"
#include "ref_tables.h"

namespace sfem {

namespace {

template <typename T>
__global__ void inverse_diagonal_kernel(int64_t n, T* d) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) {
    const T v = d[i];
    d[i] = fabs(double(v)) > 1e-10 ? T(1) / v : T(1);
  }
}

inline unsigned blocks_for(int64_t n, int bs) { return unsigned((n + bs - 1) / bs); }

template <int P>
int nnz_grad() {
  int z = 0;
  using Tb = ref::Tables<P>;
  for (int a = 0; a < 3; ++a)
    for (int m = 0; m < Tb::KQ; ++m)
      for (int i = 0; i < Tb::K; ++i) z += Tb::D[a][m][i] != 0.0;
  return z;
}
int nnz_grad_rt(int p) { return p == 1 ? nnz_grad<1>() : p == 2 ? nnz_grad<2>() : nnz_grad<3>(); }
int kq_of(int p) { return p == 1 ? 1 : p == 2 ? 4 : 10; }
int k_of(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
int nf_of(int p) { return (p + 1) * (p + 2) / 2; }
int nfq_of(int p) { return p == 1 ? 1 : p * (p + 1) / 2; }

// metric G = |det J| J^-1 J^-T as (00,11,22,01,02,12)
void metric(const CellGeometry& g, double G[6]) {
  const double ad = std::fabs(g.det);
  auto mm = [&](int a, int b) {
    double s = 0;
    for (int c = 0; c < 3; ++c) s += g.Jinv[a][c] * g.Jinv[b][c];
    return ad * s;
  };
  G[0] = mm(0, 0); G[1] = mm(1, 1); G[2] = mm(2, 2);
  G[3] = mm(0, 1); G[4] = mm(0, 2); G[5] = mm(1, 2);
}

// ------------------------------------------------------------------ CG ----
template <typename T>
class CGOperator final : public Operator {
 public:
  DevBuf<int32_t> d_dofs;        // [K][n_cells], -1 = constrained
  DevBuf<T> d_geo;               // [6][n_cells]
  DevBuf<int32_t> d_constrained; // constrained DoF list
  // macro-element (hex) tables of cg_hex_kernel; empty when the mesh is not
  // 6 consecutive Kuhn tets per hex with one common DoF pattern
  DevBuf<int32_t> d_hdofs;       // [H][n_hex]
  DevBuf<T> d_hgeo;              // [36][n_hex]: metric of tet q at rows 6 q .. 6 q + 5
  HexMap hex_map{};
  int64_t n_hex = 0;
  int hex_H = 0;

  static int hex_dofs(int p) { return p == 1 ? 8 : p == 2 ? 27 : 64; }

  // TF32 tensor-core tables (variant 4, FP32 operators): B = [S_0; ..; S_5]
  DevBuf<float> d_btc;
  DevBuf<int> d_status;
  int tc_grid = 0;

  // (S_c)_ij of the cell operator y = sum_c G_c S_c u over the metric
  // components c = (00,11,22,01,02,12): S_aa = D_a^T MQ D_a,
  // S_ab = D_a^T MQ D_b + D_b^T MQ D_a
  template <int P>
  static double stiffness_S(int c, int i, int j) {
    using Tb = ref::Tables<P>;
    constexpr int KQ = Tb::KQ;
    static const int ca[6] = {0, 1, 2, 0, 0, 1}, cb[6] = {0, 1, 2, 1, 2, 2};
    auto E = [&](int a, int b) {
      double s = 0;
      for (int m = 0; m < KQ; ++m)
        for (int q = 0; q < KQ; ++q) s += Tb::D[a][m][i] * Tb::MQ[m][q] * Tb::D[b][q][j];
      return s;
    };
    return ca[c] == cb[c] ? E(ca[c], cb[c]) : E(ca[c], cb[c]) + E(cb[c], ca[c]);
  }
  // round to TF32 (10 mantissa bits, nearest, ties away)
  static float tf32_round(double v) {
    float f = float(v);
    uint32_t bits;
    std::memcpy(&bits, &f, 4);
    bits = (bits + 0x1000u) & 0xFFFFE000u;
    std::memcpy(&f, &bits, 4);
    return f;
  }

  template <int P>
  void build_tc_tables() {
    using Sh = CGTcShape<P>;
    std::vector<float> B(size_t(Sh::NPAD) * Sh::KPAD, 0.0f);
    for (int c = 0; c < 6; ++c)
      for (int i = 0; i < Sh::K; ++i)
        for (int j = 0; j < Sh::K; ++j) B[size_t(c * Sh::K + i) * Sh::KPAD + j] = tf32_round(stiffness_S<P>(c, i, j));
    d_btc.upload(B);
    int dev = 0, sms = 0, occ = 0;
    SFEM_CUDA(cudaGetDevice(&dev));
    SFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cg_cell_tc_kernel<P>, 128, Sh::SMEM_BYTES));
    occ = std::min(occ, 512 / Sh::TMEM_COLS);  // tensor-memory columns per SM
    SFEM_REQUIRE(occ > 0, FEM_ERR_CUDA, "CG tensor-core kernel does not fit on an SM");
    tc_grid = int(std::min<int64_t>((n_cells + 127) / 128, int64_t(sms) * occ));
  }

  int status(bool clear) override {
    if (!d_status.p) return 0;
    int v = 0;
    SFEM_CUDA(cudaMemcpy(&v, d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear && v) SFEM_CUDA(cudaMemset(d_status.p, 0, sizeof(int)));
    return v;
  }

  // cube-block tables of cg_cube_kernel (blocks of 64 hexes = 384 tets)
  DevBuf<int16_t> d_tmapv, d_cslot8[3];
  DevBuf<uint32_t> d_ritem[3];
  DevBuf<int32_t> d_bdof;
  int64_t n_blocks = 0;
  int cube_NB = 0;
  static int cube_nb(int p) { return p == 1 ? 125 : p == 2 ? 729 : 2197; }
  static int cube_kp(int k) { return (k % 2) ? k : k + 1; }

  void build_cube_tables(const CGDofs& dofs) {
    if (n_cells == 0 || n_cells % 384 != 0) return;
    const int NB = cube_nb(cfg.degree), KP = cube_kp(K);
    const int64_t nbk = n_cells / 384;
    // cube-local numbering by first occurrence over (tet, local DoF)
    auto local = [&](int64_t b, std::vector<int16_t>& tm, std::vector<int32_t>& order,
                     std::unordered_map<int32_t, int>& at) -> bool {
      order.clear();
      at.clear();
      tm.resize(size_t(384) * K);
      for (int t = 0; t < 384; ++t)
        for (int i = 0; i < K; ++i) {
          const int32_t g = dofs.cell_dofs[size_t(K) * (384 * b + t) + i];
          auto it = at.find(g);
          int j;
          if (it == at.end()) {
            j = int(order.size());
            if (j >= NB) return false;
            at.emplace(g, j);
            order.push_back(g);
          } else {
            j = it->second;
          }
          tm[t * K + i] = int16_t(j);
        }
      return int(order.size()) == NB;
    };
    std::vector<int16_t> tm0;
    std::vector<int32_t> ord0;
    std::unordered_map<int32_t, int> at0;
    if (!local(0, tm0, ord0, at0)) return;
    // contribution lists and their sizes (identical in every block)
    std::vector<std::vector<int16_t>> contrib(NB);
    for (int t = 0; t < 384; ++t)
      for (int i = 0; i < K; ++i) contrib[tm0[t * K + i]].push_back(int16_t(t * KP + i));
    // reduce slots: slot n = 384 r + 32 w + l is gathered and reduced by lane
    // l of warp w in round r.  DoFs sorted by contribution groups of 8
    // (most first; first-occurrence order inside a class, which keeps the
    // global addresses of a warp's gathers and stores close) form chunks of
    // 32 that fill one warp-round each, so the lanes of a warp loop over the
    // same number of groups; the chunks are dealt longest-first to the
    // least-loaded warp, which balances the warps up to the block barrier.
    std::vector<int> jorder(NB), slot_of(NB), dof_at(NB);
    for (int j = 0; j < NB; ++j) jorder[j] = j;
    std::stable_sort(jorder.begin(), jorder.end(), [&](int a, int b2) {
      return (contrib[a].size() + 7) / 8 > (contrib[b2].size() + 7) / 8;
    });
    {
      constexpr int NW = 12;
      const int NJr = (NB + 383) / 384, nch = (NB + 31) / 32;
      std::vector<int> cap(NW, 0), used(NW, 0), load(NW, 0), base(nch, -1);
      for (int r = 0; r < NJr; ++r)
        for (int w = 0; w < NW; ++w) {
          const int len = std::max(0, std::min(32, NB - (384 * r + 32 * w)));
          if (len == 32) ++cap[w];
          else if (len > 0) base[nch - 1] = 384 * r + 32 * w;  // the one partial chunk
        }
      auto cost = [&](int c) {
        int mx = 0;
        for (int e = 32 * c; e < std::min(NB, 32 * c + 32); ++e) mx = std::max(mx, int(contrib[jorder[e]].size()));
        return mx + 2 * ((mx + 7) / 8) + 4;
      };
      std::vector<int> corder;
      for (int c = 0; c < nch; ++c)
        if (base[c] < 0) corder.push_back(c);
      std::stable_sort(corder.begin(), corder.end(), [&](int a, int b2) { return cost(a) > cost(b2); });
      for (int c : corder) {
        int w = -1;
        for (int v = 0; v < NW; ++v)
          if (used[v] < cap[v] && (w < 0 || load[v] < load[w])) w = v;
        SFEM_REQUIRE(w >= 0, FEM_ERR_INTERNAL, "cube tables: no warp-round left for a chunk");
        base[c] = 384 * used[w] + 32 * w;
        ++used[w];
        load[w] += cost(c);
      }
      for (int e = 0; e < NB; ++e) {
        slot_of[jorder[e]] = base[e / 32] + e % 32;
        dof_at[base[e / 32] + e % 32] = jorder[e];
      }
    }
    std::vector<int32_t> count(m, 0);
    for (size_t i = 0; i < dofs.cell_dofs.size(); ++i) ++count[dofs.cell_dofs[i]];
    std::vector<int32_t> bd(size_t(NB) * nbk);
    bool ok = true;
#pragma omp parallel
    {
      std::vector<int16_t> tm;
      std::vector<int32_t> ord;
      std::unordered_map<int32_t, int> at;
      at.reserve(4 * NB);
#pragma omp for schedule(dynamic, 16)
      for (int64_t b = 0; b < nbk; ++b) {
        if (!ok) continue;
        if (!local(b, tm, ord, at) || tm != tm0) {
          ok = false;
          continue;
        }
        for (int n = 0; n < NB; ++n) {
          const int j = dof_at[n];
          const int32_t g = ord[j];
          const bool interior = count[g] == int(contrib[j].size());
          bd[size_t(b) * NB + n] = dofs.constrained[g] ? -1 : (g | (interior ? 0x40000000 : 0));
        }
      }
    }
    if (!ok || m >= (int64_t(1) << 30)) return;
    // packed tables, laid out so that a warp reads 16 consecutive bytes per
    // lane:
    //   tmapv  [KV/8][384] x 8 int16: slot of tet t's local DoF i (KV = K
    //          rounded up to 8, padding entries 0);
    //   cslot8 per warp-round, [groups][32 lanes] x 8 int16: the row slot
    //          (t' * KP + i) each lane reads at each step;
    //   ritem  [NB]: steps of the lane | (first cslot8 entry << 8).
    // Three reduce schedules (kernel variants 5, 6, 7):
    //   0  each lane reads its contributions in (tet, local DoF) order;
    //   1  bank-scheduled, the same steps for every lane of a warp-round;
    //   2  bank-scheduled, each lane stops after its last contribution.
    // Bank-scheduled steps come from an edge colouring of the bipartite
    // multigraph lanes x shared-memory banks (one edge per contribution): a
    // bipartite multigraph of maximum degree D has a proper D-edge-colouring
    // (Konig), found here by alternating-path recolouring.  Colour = step, so
    // no two lanes of one step hit the same bank and every step is one
    // shared-memory wavefront (per half-warp for 8-byte values).  A lane with
    // nothing to add at a step reads one of the zero slots 384 * KP + z (one
    // per bank), in a bank that no other lane of the step uses.
    const int KV = (K + 7) / 8 * 8;
    std::vector<int16_t> tmv(size_t(384) * KV, 0);
    for (int t = 0; t < 384; ++t)
      for (int i = 0; i < K; ++i) tmv[(size_t(i / 8) * 384 + t) * 8 + i % 8] = int16_t(slot_of[tm0[t * K + i]]);
    const int nbank = sizeof(T) == 8 ? 16 : 32;  // 8-byte values: 16 bank pairs per half-warp
    const int span = sizeof(T) == 8 ? 16 : 32;   // lanes that share one wavefront
    SFEM_REQUIRE(384 * KP + 32 < 32768, FEM_ERR_INTERNAL, "cube tables exceed their index bits");
    for (int mode = 0; mode < 3; ++mode) {
      std::vector<int16_t> c8;
      std::vector<uint32_t> items(NB);
      for (int n0 = 0; n0 < NB; n0 += 32) {
        const int len = std::min(32, NB - n0);
        std::vector<std::vector<int>> step_slot(32);  // per lane: slot at each step, -1 = none
        for (int h0 = 0; h0 < len; h0 += span) {
          const int h1 = std::min(len, h0 + span);
          if (mode == 0) {
            for (int l = h0; l < h1; ++l)
              for (int16_t v : contrib[dof_at[n0 + l]]) step_slot[l].push_back(v);
            continue;
          }
          std::vector<std::pair<int, int>> edges;  // (lane in span, slot)
          std::vector<int> degl(span, 0), degb(nbank, 0);
          for (int l = h0; l < h1; ++l)
            for (int16_t v : contrib[dof_at[n0 + l]]) {
              edges.emplace_back(l - h0, v);
              ++degl[l - h0];
              ++degb[v % nbank];
            }
          const int D = std::max(*std::max_element(degl.begin(), degl.end()),
                                 *std::max_element(degb.begin(), degb.end()));
          std::vector<int> Lc(size_t(span) * D, -1), Bc(size_t(nbank) * D, -1), col(edges.size(), -1);
          auto lc = [&](int u, int c) -> int& { return Lc[size_t(u) * D + c]; };
          auto bc = [&](int v, int c) -> int& { return Bc[size_t(v) * D + c]; };
          for (size_t e = 0; e < edges.size(); ++e) {
            const int u = edges[e].first, v = edges[e].second % nbank;
            int a = 0, c2 = 0;
            while (lc(u, a) >= 0) ++a;
            while (bc(v, c2) >= 0) ++c2;
            if (a != c2 && bc(v, a) >= 0) {
              // swap colours a and c2 along the alternating path that leaves bank v by colour a
              std::vector<int> path;
              bool at_bank = true;
              int node = v, c = a;
              for (;;) {
                const int ed = at_bank ? bc(node, c) : lc(node, c);
                if (ed < 0) break;
                path.push_back(ed);
                node = at_bank ? edges[ed].first : edges[ed].second % nbank;
                at_bank = !at_bank;
                c = c == a ? c2 : a;
              }
              for (int ed : path) {
                lc(edges[ed].first, col[ed]) = -1;
                bc(edges[ed].second % nbank, col[ed]) = -1;
              }
              for (int ed : path) {
                col[ed] = col[ed] == a ? c2 : a;
                lc(edges[ed].first, col[ed]) = ed;
                bc(edges[ed].second % nbank, col[ed]) = ed;
              }
            }
            SFEM_REQUIRE(lc(u, a) < 0 && bc(v, a) < 0, FEM_ERR_INTERNAL, "cube tables: edge colouring failed");
            col[e] = a;
            lc(u, a) = int(e);
            bc(v, a) = int(e);
          }
          for (size_t e = 0; e < edges.size(); ++e) {
            std::vector<int>& st = step_slot[h0 + edges[e].first];
            if (int(st.size()) <= col[e]) st.resize(col[e] + 1, -1);
            st[col[e]] = edges[e].second;
          }
        }
        int S = 0;
        for (int l = 0; l < len; ++l) S = std::max(S, int(step_slot[l].size()));
        SFEM_REQUIRE(S > 0 && S < 256, FEM_ERR_INTERNAL, "cube tables: step count out of range");
        std::vector<int> steps(len);
        for (int l = 0; l < len; ++l) {
          steps[l] = mode == 1 ? S : int(step_slot[l].size());
          step_slot[l].resize(S, -1);
        }
        // gaps: a zero slot in a bank that no lane of the span reads at that step
        for (int h0 = 0; h0 < len; h0 += span) {
          const int h1 = std::min(len, h0 + span);
          for (int st = 0; st < S; ++st) {
            std::vector<char> busy(nbank, 0);
            for (int l = h0; l < h1; ++l)
              if (step_slot[l][st] >= 0) busy[step_slot[l][st] % nbank] = 1;
            const int f = int(std::find(busy.begin(), busy.end(), 0) - busy.begin());
            for (int l = h0; l < h1; ++l)
              if (step_slot[l][st] < 0) step_slot[l][st] = 384 * KP + ((f % nbank - 384 * KP) % nbank + nbank) % nbank;
          }
        }
        const size_t e0 = c8.size() / 8;
        c8.resize(c8.size() + size_t((S + 7) / 8) * 32 * 8, int16_t(384 * KP));
        for (int l = 0; l < len; ++l) {
          for (int e = 0; e < S; ++e) c8[((e0 + size_t(e / 8) * 32) + l) * 8 + e % 8] = int16_t(step_slot[l][e]);
          items[n0 + l] = uint32_t(steps[l]) | (uint32_t(e0 + l) << 8);
        }
      }
      SFEM_REQUIRE(c8.size() / 8 < (size_t(1) << 24), FEM_ERR_INTERNAL, "cube tables exceed their index bits");
      d_ritem[mode].upload(items);
      d_cslot8[mode].upload(c8);
    }
    d_tmapv.upload(tmv);
    d_bdof.upload(bd);
    n_blocks = nbk;
    cube_NB = NB;
  }

  void launch_tc_cell(const T* x, T* d, cudaStream_t s) {
    const float* xf = reinterpret_cast<const float*>(x);
    float* df = reinterpret_cast<float*>(d);
    switch (cfg.degree) {
      case 1: cg_cell_tc_kernel<1><<<tc_grid, 128, CGTcShape<1>::SMEM_BYTES, s>>>(n_cells, d_dofs.p, reinterpret_cast<const float*>(d_geo.p), d_btc.p, xf, df, d_constrained.n, d_constrained.p, d_status.p); break;
      case 2: cg_cell_tc_kernel<2><<<tc_grid, 128, CGTcShape<2>::SMEM_BYTES, s>>>(n_cells, d_dofs.p, reinterpret_cast<const float*>(d_geo.p), d_btc.p, xf, df, d_constrained.n, d_constrained.p, d_status.p); break;
      case 3: cg_cell_tc_kernel<3><<<tc_grid, 128, CGTcShape<3>::SMEM_BYTES, s>>>(n_cells, d_dofs.p, reinterpret_cast<const float*>(d_geo.p), d_btc.p, xf, df, d_constrained.n, d_constrained.p, d_status.p); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  int cube_grid = 0;
  template <int P, int NB, int KP>
  static size_t cube_smem() {
    return ((cube_metric_smem<P, T>() ? 6 * 384 : 0) + 2 * size_t(NB) + 384 * size_t(KP) + (sizeof(T) == 8 ? 16 : 32)) *
           sizeof(T);
  }
  template <int P, int NB, int KP>
  void setup_cube() {
    auto kern = cg_cube_pipe_kernel<P, T, NB, KP>;
    SFEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(cube_smem<P, NB, KP>())));
    int dev = 0, sms = 0, occ = 0;
    SFEM_CUDA(cudaGetDevice(&dev));
    SFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 384, cube_smem<P, NB, KP>()));
    SFEM_REQUIRE(occ > 0, FEM_ERR_CUDA, "CG cube kernel does not fit on an SM");
    cube_grid = int(std::min<int64_t>(n_blocks, int64_t(sms) * occ));
  }
  template <int P, int NB, int KP>
  void launch_cube(const T* x, T* d, int sched, cudaStream_t s) {
    cg_cube_pipe_kernel<P, T, NB, KP><<<unsigned(cube_grid), 384, cube_smem<P, NB, KP>(), s>>>(
        n_blocks, d_tmapv.p, d_bdof.p, d_ritem[sched].p, d_cslot8[sched].p, d_geo.p, x, d, d_constrained.n,
        d_constrained.p);
  }

  // TF32 tensor-core cube kernel (variant 8, FP32 operators with cube tables):
  // B rows p NP + n = (S_c)_i. for c = p CPP + n / K, i = n % K
  DevBuf<float> d_bcube;
  int cube_tc_grid = 0;
  size_t cube_tc_smem = 0;
  template <int P, int NB, int KP>
  void setup_cube_tc() {
    using Sh = CubeTcShape<P>;
    std::vector<float> B(size_t(Sh::NBROWS) * Sh::KPAD, 0.0f);
    for (int p = 0; p < Sh::PASSES; ++p)
      for (int n = 0; n < Sh::CPP * Sh::K; ++n)
        for (int j = 0; j < Sh::K; ++j)
          B[size_t(p * Sh::NP + n) * Sh::KPAD + j] = tf32_round(stiffness_S<P>(p * Sh::CPP + n / Sh::K, n % Sh::K, j));
    d_bcube.upload(B);
    auto kern = cg_cube_tc_kernel<P, NB, KP>;
    int dev = 0, sms = 0, occ = 0;
    SFEM_CUDA(cudaGetDevice(&dev));
    SFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // more CTAs per SM than the tensor memory holds would wait in tcgen05.alloc
    // for another CTA to finish: pad the shared memory until they cannot fit
    size_t smem = Sh::smem_bytes(NB, KP);
    for (;;) {
      SFEM_REQUIRE(smem <= 227 * 1024, FEM_ERR_CUDA, "CG tensor-core cube kernel: no shared-memory size fits");
      SFEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      SFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 384, smem));
      if (occ <= Sh::MAX_CTAS) break;
      smem += 4096;
    }
    SFEM_REQUIRE(occ > 0, FEM_ERR_CUDA, "CG tensor-core cube kernel does not fit on an SM");
    cube_tc_smem = smem;
    cube_tc_grid = int(std::min<int64_t>(n_blocks, int64_t(sms) * occ));
  }
  template <int P, int NB, int KP>
  void launch_cube_tc(const T* x, T* d, int sched, cudaStream_t s) {
    cg_cube_tc_kernel<P, NB, KP><<<unsigned(cube_tc_grid), 384, cube_tc_smem, s>>>(
        n_blocks, d_tmapv.p, d_bdof.p, d_ritem[sched].p, d_cslot8[sched].p, reinterpret_cast<const float*>(d_geo.p),
        d_bcube.p, reinterpret_cast<const float*>(x), reinterpret_cast<float*>(d), d_constrained.n, d_constrained.p,
        d_status.p);
  }

  void build_hex_tables(const Mesh& mesh, const CGDofs& dofs, const std::vector<T>& geo) {
    if (n_cells == 0 || n_cells % 6 != 0 || int64_t(mesh.cell_hex.size()) != n_cells) return;
    const int64_t nh = n_cells / 6;
    const int H = hex_dofs(cfg.degree);
    // hex-local numbering by first occurrence over (tet, local DoF)
    auto local_map = [&](int64_t h, int8_t (&mm)[6][20], std::vector<int32_t>& order) -> bool {
      order.clear();
      for (int q = 0; q < 6; ++q) {
        if (mesh.cell_hex[6 * h + q] != mesh.cell_hex[6 * h]) return false;
        for (int i = 0; i < K; ++i) {
          const int32_t g = dofs.cell_dofs[size_t(K) * (6 * h + q) + i];
          int k = 0;
          while (k < int(order.size()) && order[k] != g) ++k;
          if (k == int(order.size())) {
            if (k >= H) return false;
            order.push_back(g);
          }
          mm[q][i] = int8_t(k);
        }
      }
      return int(order.size()) == H;
    };
    HexMap m0{};
    std::vector<int32_t> ord0;
    if (!local_map(0, m0.m, ord0)) return;
    std::vector<int32_t> hd(size_t(H) * nh);
    bool ok = true;
#pragma omp parallel
    {
      std::vector<int32_t> ord;
      int8_t mm[6][20];
#pragma omp for schedule(static)
      for (int64_t h = 0; h < nh; ++h) {
        if (!ok) continue;
        bool same = local_map(h, mm, ord);
        for (int q = 0; q < 6 && same; ++q)
          for (int i = 0; i < K; ++i) same = same && mm[q][i] == m0.m[q][i];
        if (!same) {
          ok = false;
          continue;
        }
        for (int k = 0; k < H; ++k) hd[size_t(k) * nh + h] = dofs.constrained[ord[k]] ? -1 : ord[k];
      }
    }
    if (!ok) return;
    std::vector<T> hg(36 * size_t(nh));
#pragma omp parallel for schedule(static)
    for (int64_t h = 0; h < nh; ++h)
      for (int q = 0; q < 6; ++q)
        for (int k = 0; k < 6; ++k) hg[size_t(6 * q + k) * nh + h] = geo[size_t(k) * n_cells + 6 * h + q];
    d_hgeo.upload(hg);
    d_hdofs.upload(hd);
    hex_map = m0;
    n_hex = nh;
    hex_H = H;
  }

  CGOperator(const Mesh& mesh, const OpConfig& c) : CGOperator(mesh, build_cg_dofs(mesh, c.degree), nullptr, c) {}

  // Operator on the cells of `mesh` with a given numbering: dofs.constrained
  // masks the gather and scatter, `identity` (default: dofs.constrained)
  // lists the rows that get dst = src.  A partition's local operator passes
  // the global constraints of its owned and ghost DoFs and only the owned
  // constrained DoFs as identity rows.
  CGOperator(const Mesh& mesh, CGDofs dofs, const std::vector<uint8_t>* identity, const OpConfig& c) {
    cfg = c;
    if (cfg.weak_bc) {
      // weak (Nitsche) Dirichlet: no DoF is constrained, boundary faces carry
      // the penalty terms instead
      std::fill(dofs.constrained.begin(), dofs.constrained.end(), uint8_t(0));
      identity = nullptr;
    }
    K = dofs.K;
    n_cells = mesh.n_cells;
    m = dofs.n_dofs;
    n_interior_faces = mesh.n_interior_faces;
    n_boundary_faces = mesh.n_boundary_faces;
    cell_dofs = dofs.cell_dofs;
    constrained = dofs.constrained;
    support = dofs.support;
    std::vector<int32_t> idx(size_t(K) * n_cells);
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int i = 0; i < K; ++i) {
        const int32_t g = dofs.cell_dofs[K * cc + i];
        idx[size_t(i) * n_cells + cc] = dofs.constrained[g] ? -1 : g;
      }
    d_dofs.upload(idx);
    std::vector<T> geo(6 * size_t(n_cells));
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      double G[6];
      metric(cell_geometry(mesh, cc), G);
      for (int k = 0; k < 6; ++k) geo[size_t(k) * n_cells + cc] = T(G[k]);
    }
    d_geo.upload(geo);
    std::vector<int32_t> cl;
    const std::vector<uint8_t>& id_rows = identity ? *identity : constrained;
    SFEM_REQUIRE(int64_t(id_rows.size()) == m, FEM_ERR_INTERNAL, "CG: identity mask size");
    for (int64_t i = 0; i < m; ++i)
      if (id_rows[i]) cl.push_back(int32_t(i));
    d_constrained.upload(cl);
    build_hex_tables(mesh, dofs, geo);
    build_cube_tables(dofs);
    if (cfg.weak_bc) build_weak_boundary(mesh);
    d_status.alloc(1);
    SFEM_CUDA(cudaMemset(d_status.p, 0, sizeof(int)));
    if (std::is_same<T, float>::value && n_cells > 0) {
      switch (cfg.degree) {
        case 1: build_tc_tables<1>(); break;
        case 2: build_tc_tables<2>(); break;
        case 3: build_tc_tables<3>(); break;
      }
    }
    if (cube_NB) {
      switch (cfg.degree) {
        case 1: setup_cube<1, 125, 5>(); break;
        case 2: setup_cube<2, 729, 11>(); break;
        case 3: setup_cube<3, 2197, 21>(); break;
      }
      if (std::is_same<T, float>::value) {
        switch (cfg.degree) {
          case 1: setup_cube_tc<1, 125, 5>(); break;
          case 2: setup_cube_tc<2, 729, 11>(); break;
          case 3: setup_cube_tc<3, 2197, 21>(); break;
        }
      }
    }
    if (hex_H) {
      switch (cfg.degree) {
        case 1: setup_hex<1, 8>(); break;
        case 2: setup_hex<2, 27>(); break;
        case 3: setup_hex<3, 64>(); break;
      }
    }
  }

  static constexpr int kHexBS = 64;
  template <int P, int H>
  static size_t hex_smem() { return 2 * size_t(kHexBS) * HexRow<H>::S * sizeof(T); }
  template <int P, int H>
  void setup_hex() {
    SFEM_CUDA(cudaFuncSetAttribute(cg_hex_kernel<P, T, H, kHexBS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(hex_smem<P, H>())));
  }
  template <int P, int H>
  void launch_hex(const T* x, T* d, cudaStream_t s) {
    const unsigned grid = blocks_for(std::max<int64_t>(n_hex, 1), kHexBS);
    cg_hex_kernel<P, T, H, kHexBS><<<grid, kHexBS, hex_smem<P, H>(), s>>>(
        n_hex, d_hdofs.p, hex_map, d_hgeo.p, x, d, d_constrained.n, d_constrained.p);
  }

  void vmult(void* dst, const void* src, cudaStream_t s) override {
    vmult_phase(dst, src, 1, s);
    vmult_phase(dst, src, 2, s);
  }

  void vmult_phase(void* dst, const void* src, int phase, cudaStream_t s) override {
    T* d = static_cast<T*>(dst);
    const T* x = static_cast<const T*>(src);
    if (phase == 1) {
      SFEM_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * m, s));
      return;
    }
    apply_cells(x, d, s);
    if (cfg.weak_bc) apply_boundary(x, d, false, s);
  }

  // weak (Nitsche) boundary terms: boundary faces grouped by local face number
  DevBuf<int32_t> d_bcell[4];
  DevBuf<T> d_bsf[4];

  void build_weak_boundary(const Mesh& mesh) {
    const int p = cfg.degree;
    const double factor = double((p + 1) * (p + 3)) / 3.0;
    std::vector<int32_t> cells[4];
    std::vector<T> sf[4];
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      const double vol = std::fabs(cell_geometry(mesh, cc).det) / 6.0;
      double area[4], surf = 0;
      for (int f = 0; f < 4; ++f) {
        double nrm[3];
        face_area_normal(mesh, cc, f, area[f], nrm);
        surf += area[f] * (mesh.nb[4 * cc + f] == -1 ? 1.0 : 0.5);
      }
      const double tau = surf / vol;  // surface / volume (DG/cells_batched/application_phc.cc:1284-1313)
      for (int f = 0; f < 4; ++f)
        if (mesh.nb[4 * cc + f] == -1) {
          cells[f].push_back(int32_t(cc));
          sf[f].push_back(T(factor * tau * area[f]));
        }
    }
    for (int f = 0; f < 4; ++f) {
      d_bcell[f].upload(cells[f]);
      d_bsf[f].upload(sf[f]);
    }
  }

  template <int P>
  void launch_boundary(const T* x, T* d, bool diag, cudaStream_t s) {
    auto go = [&](auto fc) {
      constexpr int F = decltype(fc)::value;
      const int64_t nb = int64_t(d_bcell[F].n);
      if (!nb) return;
      cg_weak_boundary_kernel<P, F, T><<<blocks_for(nb, 128), 128, 0, s>>>(nb, d_bcell[F].p, d_bsf[F].p, n_cells,
                                                                          d_dofs.p, d_geo.p, x, d, diag);
    };
    go(std::integral_constant<int, 0>{});
    go(std::integral_constant<int, 1>{});
    go(std::integral_constant<int, 2>{});
    go(std::integral_constant<int, 3>{});
  }

  void apply_boundary(const T* x, T* d, bool diag, cudaStream_t s) {
    switch (cfg.degree) {
      case 1: launch_boundary<1>(x, d, diag, s); break;
      case 2: launch_boundary<2>(x, d, diag, s); break;
      case 3: launch_boundary<3>(x, d, diag, s); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  void apply_cells(const T* x, T* d, cudaStream_t s) {
    // default (variant 0), measured on B200: P1 per cube in FP64 and per hex
    // in FP32, P2 per cube, P3 per cube in FP32 and per cell in FP64; per cell on meshes too small to give
    // every SM two cubes (or two CTAs of hexes), where the coarser forms
    // leave SMs idle
    int v = cfg.kernel_variant;
    if (v == 8) {
      // TF32 tensor cores per cube; per cell (variant 4) without whole cubes
      SFEM_REQUIRE(d_btc.p != nullptr, FEM_ERR_ARG, "CG kernel variant 8 (TF32 tensor cores) needs an FP32 operator");
      if (cube_NB && cube_tc_grid) {
        switch (cfg.degree) {
          case 1: launch_cube_tc<1, 125, 5>(x, d, 0, s); break;
          case 2: launch_cube_tc<2, 729, 11>(x, d, 0, s); break;
          case 3: launch_cube_tc<3, 2197, 21>(x, d, 0, s); break;
        }
        SFEM_CUDA(cudaGetLastError());
        return;
      }
      v = 4;
    }
    if (v == 4) {
      SFEM_REQUIRE(d_btc.p != nullptr, FEM_ERR_ARG, "CG kernel variant 4 (TF32 tensor cores) needs an FP32 operator");
      launch_tc_cell(x, d, s);
      return;
    }
    if (v == 0) {
      constexpr int64_t kFill = 2 * 148;
      // measured on B200: P3 FP64 64^3 cube 171 against 190 us per cell
      v = cfg.degree == 1 ? (sizeof(T) == 8 ? 3 : 2) : 3;
      if (v == 3 && n_blocks < kFill) v = 2;
      if (v == 2 && n_hex < kFill * kHexBS) v = 1;
    }
    // cube reduce schedule: variants 5, 6, 7 pick one; variant 3 takes the
    // one measured fastest on B200 (FP64 P1 and P2: bank-scheduled with
    // uniform steps, 144 against 157 us and 380 against 380-413 us on 128^3;
    // FP32 and P3: contribution order)
    int sched = v >= 5 ? v - 5 : (sizeof(T) == 8 && cfg.degree <= 2 ? 1 : 0);
    if (v >= 5) v = 3;
    if (v == 3 && cube_NB) {
      switch (cfg.degree) {
        case 1: launch_cube<1, 125, 5>(x, d, sched, s); break;
        case 2: launch_cube<2, 729, 11>(x, d, sched, s); break;
        case 3: launch_cube<3, 2197, 21>(x, d, sched, s); break;
      }
      SFEM_CUDA(cudaGetLastError());
      return;
    }
    // variant 2 (and 3 without whole cubes): one thread per hex; the cell
    // kernel on meshes without the common hex pattern
    if ((v == 2 || v == 3) && hex_H) {
      switch (cfg.degree) {
        case 1: launch_hex<1, 8>(x, d, s); break;
        case 2: launch_hex<2, 27>(x, d, s); break;
        case 3: launch_hex<3, 64>(x, d, s); break;
      }
      SFEM_CUDA(cudaGetLastError());
      return;
    }
    const int64_t n = std::max<int64_t>(n_cells, int64_t(d_constrained.n));
    const unsigned grid = blocks_for(n, 128);
    switch (cfg.degree) {
      case 1: cg_cell_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p); break;
      case 2: cg_cell_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p); break;
      case 3:
        // P3 in FP64: registers capped for 4 CTAs per SM (measured faster on B200)
        if (sizeof(T) == 8) cg_cell_kernel<3, T, 4><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p);
        else cg_cell_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p);
        break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  void diagonal(void* diag, cudaStream_t s) override {
    T* d = static_cast<T*>(diag);
    SFEM_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * m, s));
    const int64_t n = std::max<int64_t>(n_cells, int64_t(d_constrained.n));
    const unsigned grid = blocks_for(n, 128);
    switch (cfg.degree) {
      case 1: cg_diagonal_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, d, d_constrained.n, d_constrained.p); break;
      case 2: cg_diagonal_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, d, d_constrained.n, d_constrained.p); break;
      case 3: cg_diagonal_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, d, d_constrained.n, d_constrained.p); break;
    }
    SFEM_CUDA(cudaGetLastError());
    if (cfg.weak_bc) apply_boundary(nullptr, d, true, s);
  }

  const int32_t* device_dof_table() const override { return d_dofs.p; }

  void element_matrices(void* out, cudaStream_t s) override {
    T* m = static_cast<T*>(out);
    const unsigned grid = blocks_for(std::max<int64_t>(n_cells, 1), 128);
    switch (cfg.degree) {
      case 1: cg_element_matrix_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, d_geo.p, m); break;
      case 2: cg_element_matrix_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, d_geo.p, m); break;
      case 3: cg_element_matrix_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, d_geo.p, m); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  void work(double& flops, double& bytes) const override {
    const int p = cfg.degree, kq = kq_of(p);
    const double per_cell = 2.0 * (2 * nnz_grad_rt(p) + 9 * kq + 3 * kq * kq);
    flops = per_cell * double(n_cells);
    const double s = double(sizeof(T));
    bytes = 2 * s * double(m) + 4.0 * K * double(n_cells) + 6 * s * double(n_cells);
  }
};

// ------------------------------------------------------- CG, 3 components --
// Vector Laplacian with the components of every node DoF interleaved
// (index 3 g + comp), as the reference's components-batched CG operator
// (CG/components_batched/application.cc:778-1611, FESystem of dim
// FE_SimplexP).  Homogeneous Dirichlet on every component of the boundary
// nodes.  Cell kernel only.
template <typename T>
class CGVectorOperator final : public Operator {
 public:
  static constexpr int NC = 3;
  DevBuf<int32_t> d_dofs;         // [K][n_cells] node DoFs, -1 = constrained
  DevBuf<T> d_geo;                // [6][n_cells]
  DevBuf<int32_t> d_constrained;  // constrained vector indices
  int64_t n_nodes = 0;
  std::vector<int32_t> node_dofs;  // [n_cells][K]

  CGVectorOperator(const Mesh& mesh, const OpConfig& c) {
    cfg = c;
    const CGDofs dofs = build_cg_dofs(mesh, cfg.degree);
    K = dofs.K;
    n_cells = mesh.n_cells;
    n_nodes = dofs.n_dofs;
    m = NC * n_nodes;
    n_interior_faces = mesh.n_interior_faces;
    n_boundary_faces = mesh.n_boundary_faces;
    node_dofs = dofs.cell_dofs;
    cell_dofs.resize(size_t(NC) * K * n_cells);
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int comp = 0; comp < NC; ++comp)
        for (int i = 0; i < K; ++i)
          cell_dofs[(cc * NC + comp) * K + i] = NC * dofs.cell_dofs[K * cc + i] + comp;
    constrained.assign(m, 0);
    std::vector<int32_t> cl;
    for (int64_t g = 0; g < n_nodes; ++g)
      if (dofs.constrained[g])
        for (int comp = 0; comp < NC; ++comp) {
          constrained[NC * g + comp] = 1;
          cl.push_back(int32_t(NC * g + comp));
        }
    support = dofs.support;
    std::vector<int32_t> idx(size_t(K) * n_cells);
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int i = 0; i < K; ++i) {
        const int32_t g = dofs.cell_dofs[K * cc + i];
        idx[size_t(i) * n_cells + cc] = dofs.constrained[g] ? -1 : g;
      }
    d_dofs.upload(idx);
    std::vector<T> geo(6 * size_t(n_cells));
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      double G[6];
      metric(cell_geometry(mesh, cc), G);
      for (int k = 0; k < 6; ++k) geo[size_t(k) * n_cells + cc] = T(G[k]);
    }
    d_geo.upload(geo);
    d_constrained.upload(cl);
  }

  void vmult(void* dst, const void* src, cudaStream_t s) override {
    vmult_phase(dst, src, 1, s);
    vmult_phase(dst, src, 2, s);
  }

  void vmult_phase(void* dst, const void* src, int phase, cudaStream_t s) override {
    T* d = static_cast<T*>(dst);
    const T* x = static_cast<const T*>(src);
    if (phase == 1) {
      SFEM_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * m, s));
      return;
    }
    const unsigned grid = blocks_for(std::max<int64_t>(n_cells, int64_t(d_constrained.n)), 128);
    switch (cfg.degree) {
      case 1: cg_cell_vec_kernel<1, T, NC><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p); break;
      case 2: cg_cell_vec_kernel<2, T, NC><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p); break;
      case 3: cg_cell_vec_kernel<3, T, NC><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, x, d, d_constrained.n, d_constrained.p); break;
    }
    SFEM_CUDA(cudaGetLastError());
  }

  void diagonal(void* diag, cudaStream_t s) override {
    DevBuf<T> dn(n_nodes);
    SFEM_CUDA(cudaMemsetAsync(dn.p, 0, sizeof(T) * n_nodes, s));
    std::vector<int32_t> cn;
    for (int64_t g = 0; g < n_nodes; ++g)
      if (constrained[NC * g]) cn.push_back(int32_t(g));
    DevBuf<int32_t> d_cn;
    d_cn.upload(cn);
    const unsigned grid = blocks_for(std::max<int64_t>(n_cells, int64_t(cn.size())), 128);
    switch (cfg.degree) {
      case 1: cg_diagonal_kernel<1, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, dn.p, d_cn.n, d_cn.p); break;
      case 2: cg_diagonal_kernel<2, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, dn.p, d_cn.n, d_cn.p); break;
      case 3: cg_diagonal_kernel<3, T><<<grid, 128, 0, s>>>(n_cells, d_dofs.p, d_geo.p, dn.p, d_cn.n, d_cn.p); break;
    }
    expand_components<T, NC><<<blocks_for(std::max<int64_t>(n_nodes, 1), 256), 256, 0, s>>>(
        n_nodes, dn.p, static_cast<T*>(diag));
    SFEM_CUDA(cudaGetLastError());
    SFEM_CUDA(cudaStreamSynchronize(s));  // the temporaries are freed on return
  }

  void rhs(const RhsDesc& rd, void* dst, cudaStream_t s) override {
    throw Error(FEM_ERR_ARG, "rhs: not provided for the 3-component CG operator");
  }

  void work(double& flops, double& bytes) const override {
    const int p = cfg.degree, kq = kq_of(p);
    flops = NC * 2.0 * (2 * nnz_grad_rt(p) + 9 * kq + 3 * kq * kq) * double(n_cells);
    const double sz = double(sizeof(T));
    bytes = 2 * sz * double(m) + 4.0 * K * double(n_cells) + 6 * sz * double(n_cells);
  }
};

// ------------------------------------------------------------------ DG ----
template <typename T>
class DGOperator final : public Operator {
 public:
  DevBuf<T> d_geo;      // [6 + 4 + (mass?1:0)][n_cells]
  DevBuf<int32_t> d_nb; // [4][n_cells]
  DevBuf<int8_t> d_nbf; // [4][n_cells]
  DevBuf<T> d_Q;        // published face normal derivatives: [n_cells][4][NC][NFQ], or block-major
                        // (scalar problems, 1-thread-per-cell forms), for whole 128-cell blocks
  DevBuf<int> d_status; // timeouts of the bounded waits in the bulk-copy trace pass
  bool has_mass = false;

  DGOperator(const Mesh& mesh, const OpConfig& c) {
    cfg = c;
    const int p = cfg.degree;
    K = k_of(p);
    n_cells = mesh.n_cells;
    m = int64_t(K) * cfg.n_components * n_cells;
    n_interior_faces = mesh.n_interior_faces;
    n_boundary_faces = mesh.n_boundary_faces;
    has_mass = cfg.kind == FEM_HELMHOLTZ;
    constrained.assign(m, 0);
    support.resize(3 * size_t(K) * n_cells);
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      const int32_t* cv = &mesh.cell_vertices[4 * cc];
      for (int i = 0; i < K; ++i)
        for (int a = 0; a < 3; ++a) {
          double sum = 0;
          for (int v = 0; v < 4; ++v) {
            const int lat = p == 1 ? ref::Tables<1>::LATTICE[i][v]
                                   : p == 2 ? ref::Tables<2>::LATTICE[i][v] : ref::Tables<3>::LATTICE[i][v];
            sum += lat * mesh.x[3 * size_t(cv[v]) + a];
          }
          support[3 * (size_t(K) * cc + i) + a] = sum / p;
        }
    }
    const int n_geo = has_mass ? 11 : 10;
    std::vector<T> geo(size_t(n_geo) * n_cells);
    // per-cell quantities for the penalty
    std::vector<double> tau(n_cells), inv_h(4 * size_t(n_cells)), area(4 * size_t(n_cells));
    std::vector<double> absdet(n_cells);
    for (int64_t cc = 0; cc < n_cells; ++cc) {
      const CellGeometry g = cell_geometry(mesh, cc);
      absdet[cc] = std::fabs(g.det);
      double G[6];
      metric(g, G);
      for (int k = 0; k < 6; ++k) geo[size_t(k) * n_cells + cc] = T(G[k]);
      if (has_mass) geo[size_t(10) * n_cells + cc] = T(cfg.mass * absdet[cc]);
      double surf = 0;
      for (int f = 0; f < 4; ++f) {
        double a, nrm[3];
        face_area_normal(mesh, cc, f, a, nrm);
        area[4 * cc + f] = a;
        inv_h[4 * cc + f] = 2.0 * a / absdet[cc];  // |grad lambda_f| = 1/h_f
        surf += a * (mesh.nb[4 * cc + f] == -1 ? 1.0 : 0.5);  // -2: interior, neighbour not local
      }
      tau[cc] = surf / (absdet[cc] / 6.0);
    }
    const double factor = cfg.penalty == FEM_PENALTY_SQUARE ? double((p + 1) * (p + 1))
                                                            : double((p + 1) * (p + 3)) / 3.0;
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int f = 0; f < 4; ++f) {
        const int32_t nbc = mesh.nb[4 * cc + f];
        double sigma;
        if (cfg.kind == FEM_HELMHOLTZ) {
          // 1/h normal to the face, averaged over both sides
          // (application_helmholtz.cc:1329-1333 and :857-859 on the boundary)
          sigma = nbc >= 0 ? factor * 0.5 * (inv_h[4 * cc + f] + inv_h[4 * size_t(nbc) + mesh.nbf[4 * cc + f]])
                           : factor * inv_h[4 * cc + f];
        } else {
          // max of the two cells' surface/volume (DG/cells_batched/application.cc:1377-1379)
          sigma = nbc >= 0 ? factor * std::max(tau[cc], tau[nbc]) : factor * tau[cc];
        }
        geo[size_t(6 + f) * n_cells + cc] = T(sigma * area[4 * cc + f]);
      }
    d_geo.upload(geo);
    std::vector<int32_t> nb(4 * size_t(n_cells));
    std::vector<int8_t> nbf(4 * size_t(n_cells));
    for (int64_t cc = 0; cc < n_cells; ++cc)
      for (int f = 0; f < 4; ++f) {
        nb[size_t(f) * n_cells + cc] = std::max(mesh.nb[4 * cc + f], -1);
        nbf[size_t(f) * n_cells + cc] = mesh.nbf[4 * cc + f] < 0 ? 0 : mesh.nbf[4 * cc + f];
      }
    d_nb.upload(nb);
    d_nbf.upload(nbf);
    d_Q.alloc(size_t((n_cells + kQB - 1) / kQB * kQB) * 4 * cfg.n_components * nfq_of(p));
    d_status.alloc(1);
    SFEM_CUDA(cudaMemset(d_status.p, 0, sizeof(int)));
  }

  int status(bool clear) override {
    int v = 0;
    SFEM_CUDA(cudaMemcpy(&v, d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear && v) SFEM_CUDA(cudaMemset(d_status.p, 0, sizeof(int)));
    return v;
  }

  DGProblem<T> problem(const void* src, void* dst) const {
    DGProblem<T> pr;
    pr.geo = d_geo.p;
    pr.nb = d_nb.p;
    pr.nbf = d_nbf.p;
    pr.src = static_cast<const T*>(src);
    pr.dst = static_cast<T*>(dst);
    pr.Q = d_Q.p;
    pr.n_cells = n_cells;
    return pr;
  }

  void vmult(void* dst, const void* src, cudaStream_t s) override {
    const DGProblem<T> pr = problem(src, dst);
    launch_dg(cfg, &pr, 1, s, 0, d_status.p);
  }

  void vmult_phase(void* dst, const void* src, int phase, cudaStream_t s) override {
    const DGProblem<T> pr = problem(src, dst);
    launch_dg(cfg, &pr, 1, s, phase, d_status.p);
  }

  size_t scratch_bytes() const override { return d_Q.n * sizeof(T); }

  void vmult_with_scratch(void* dst, const void* src, void* scratch, size_t bytes, cudaStream_t s) override {
    SFEM_REQUIRE(bytes >= scratch_bytes(), FEM_ERR_ARG, "vmult: scratch too small");
    DGProblem<T> pr = problem(src, dst);
    pr.Q = static_cast<T*>(scratch);
    launch_dg(cfg, &pr, 1, s, 0, d_status.p);
  }

  void diagonal(void* diag, cudaStream_t s) override {
    const DGProblem<T> pr = problem(nullptr, diag);
    launch_dg(cfg, &pr, 1, s, 3, d_status.p);
  }

  void work(double& flops, double& bytes) const override {
    const int p = cfg.degree, kq = kq_of(p), nf = nf_of(p), nfq = nfq_of(p), nz = nnz_grad_rt(p);
    const double trace = 2.0 * (nz + 12 * nfq);
    double apply = 2.0 * (2 * nz + 9 * kq + 3 * kq * kq) +
                   4 * 2.0 * (3 * nfq + nf + nf * nf + nf + 2 * nf * nfq + 3 * nfq + 3 * nfq);
    if (has_mass) apply += 2.0 * (K * K + K);
    flops = (trace + apply) * cfg.n_components * double(n_cells);
    const double s = double(sizeof(T));
    bytes = 2 * s * double(m) + 6 * s * double(n_cells) + double(n_interior_faces) * (8 + s) +
            double(n_boundary_faces) * (4 + s);
  }

  // Dispatch over n problems.  what: 0 trace+apply, 1 trace, 2 apply, 3 diagonal.
  // status: device word set by the bounded waits of the bulk-copy trace pass.
  static void launch_dg(const OpConfig& cfg, const DGProblem<T>* probs, int n, cudaStream_t s, int what,
                        int* status) {
    const bool mass = cfg.kind == FEM_HELMHOLTZ;
    const int nc = cfg.n_components;
    SFEM_REQUIRE(nc == 1 || nc == 3, FEM_ERR_ARG, "DG: n_components must be 1 or 3");
    SFEM_REQUIRE(n >= 1 && n <= kMaxBatch, FEM_ERR_ARG, "DG: 1..40 problems per launch");
    const int variant = cfg.kernel_variant > 0 ? cfg.kernel_variant : default_variant(cfg.degree, nc);
#define SFEM_DG_CASE(P, NC, MASS)                                                       \
  if (cfg.degree == P && nc == NC && mass == MASS) {                                    \
    run<P, NC, MASS>(probs, n, s, what, variant, status);                               \
    return;                                                                             \
  }
    SFEM_DG_CASE(1, 1, false) SFEM_DG_CASE(2, 1, false) SFEM_DG_CASE(3, 1, false)
    SFEM_DG_CASE(1, 1, true) SFEM_DG_CASE(2, 1, true) SFEM_DG_CASE(3, 1, true)
    SFEM_DG_CASE(1, 3, true) SFEM_DG_CASE(2, 3, true) SFEM_DG_CASE(3, 3, true)
    SFEM_DG_CASE(1, 3, false) SFEM_DG_CASE(2, 3, false) SFEM_DG_CASE(3, 3, false)
#undef SFEM_DG_CASE
    throw Error(FEM_ERR_ARG, "DG: unsupported degree/components combination");
  }

  // kernel forms: 1 thread per cell, 128 cells per CTA; 2 thread per cell, 64
  // cells per CTA; 3 warp roles, 32 cells per CTA
  // (measured on B200: scalar P3 runs best register-capped at 64 cells per CTA,
  // the 3-component forms at 128 cells per CTA)
  // measured on B200 (DG P3 32^3, medians of 25 L2-flushed vmults): FP64
  // 82.9 us with 128 cells per CTA against 85.0 us with 64; FP32 44.1 us with
  // the results in registers and 8 CTAs per SM against 52.2 us; 128 cells per
  // CTA otherwise
  static int default_variant(int p, int nc) { return (nc == 1 && p == 3 && sizeof(T) == 4) ? 4 : 1; }

  static DGBatch<T> make_batch(const DGProblem<T>* probs, int n, int bs, int64_t& n_blocks) {
    DGBatch<T> b;
    b.n = n;
    b.block_begin[0] = 0;
    for (int i = 0; i < n; ++i) {
      b.p[i] = probs[i];
      b.block_begin[i + 1] = b.block_begin[i] + (probs[i].n_cells + bs - 1) / bs;
    }
    n_blocks = b.block_begin[n];
    return b;
  }

  template <class K>
  static void opt_in_smem(K kernel, size_t bytes, std::atomic<uint64_t>& configured) {
    int dev = 0;
    SFEM_CUDA(cudaGetDevice(&dev));
    once_per_device(configured, dev, [&] {
      SFEM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    });
  }

  // The bulk-copy trace pass needs every copy 16-byte aligned and a whole
  // number of 16-byte units: src rows (the last block's included) and the
  // metric rows of the geometry.
  template <int P>
  static bool trace_tma_ok(const DGProblem<T>* probs, int n) {
    for (int i = 0; i < n; ++i) {
      const DGProblem<T>& pr = probs[i];
      if ((reinterpret_cast<uintptr_t>(pr.src) | reinterpret_cast<uintptr_t>(pr.geo)) & 15u) return false;
      if ((size_t(pr.n_cells) * sizeof(T)) % 16 != 0) return false;  // metric row starts
      if ((size_t(pr.n_cells % kQB) * k_of(P) * sizeof(T)) % 16 != 0) return false;
    }
    return true;
  }
  template <int P>
  static void run_trace_tma(const DGBatch<T>& b, int64_t n_blocks, cudaStream_t s, int* status) {
    constexpr int NS = 3;
    using S = TraceTmaShape<T, gen::Ops<P>::K, NS>;
    auto kern = dg_trace_tma_kernel<P, T, NS>;
    static std::atomic<uint64_t> conf{0};
    static int grid_per_dev[64] = {};
    int dev = 0;
    SFEM_CUDA(cudaGetDevice(&dev));
    once_per_device(conf, dev, [&] {
      SFEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
      int sms = 0, occ = 0;
      SFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      SFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kQB, S::SMEM));
      SFEM_REQUIRE(occ > 0, FEM_ERR_CUDA, "DG trace pass does not fit on an SM");
      grid_per_dev[dev] = sms * occ;
    });
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(n_blocks, grid_per_dev[dev]));
    kern<<<unsigned(grid), kQB, S::SMEM, s>>>(b, n_blocks, status);
  }

  // PDLM > 0 (scalar problems): the apply pass is launched as a programmatic
  // dependent of the trace pass (see dg_apply_kernel)
  template <int P, int NC, bool MASS, int BS, int MINB = (BS == 64 ? 6 : 1), bool ALIAS = false, int PDLM = 0>
  static void run_cell(const DGProblem<T>* probs, int n, cudaStream_t s, int what, int* status) {
    using S = DGShape<P, NC>;
    int64_t n_blocks = 0;
    const DGBatch<T> b = make_batch(probs, n, BS, n_blocks);
    const size_t sm_trace = size_t(BS) * (S::US + S::QS) * sizeof(T);
    // scalar problems: block-major traces (no shared memory in the trace pass)
    constexpr bool BQ = NC == 1;
    const size_t sm_apply = size_t(BS) * ((ALIAS ? 1 : 2) * S::US + S::QS) * sizeof(T);
    static std::atomic<uint64_t> conf_t{0}, conf_a{0};
    auto apply = dg_apply_kernel<P, NC, MASS, BS, T, MINB, ALIAS, BQ, (BQ ? PDLM : 0)>;
    opt_in_smem(apply, sm_apply, conf_a);
    if (what != 2) {
      if constexpr (BQ) {
        int64_t nbt = 0;
        const DGBatch<T> bt = make_batch(probs, n, kQB, nbt);
        if (trace_tma_ok<P>(probs, n)) run_trace_tma<P>(bt, nbt, s, status);
        else dg_trace_blk_kernel<P, T><<<unsigned(nbt), kQB, 0, s>>>(bt, nbt);
      } else {
        opt_in_smem(dg_trace_kernel<P, NC, BS, T>, sm_trace, conf_t);
        dg_trace_kernel<P, NC, BS, T><<<unsigned(n_blocks), BS, sm_trace, s>>>(b, n_blocks);
      }
    }
    if (what == 1) return;
    if (BQ && PDLM > 0 && what == 0) {
      // the trace pass just launched on this stream is the only producer the
      // apply pass may overlap: everything else it reads was complete before
      // the trace pass started
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3(unsigned(n_blocks));
      lc.blockDim = dim3(BS);
      lc.dynamicSmemBytes = sm_apply;
      lc.stream = s;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      SFEM_CUDA(cudaLaunchKernelEx(&lc, apply, b, n_blocks));
    } else {
      apply<<<unsigned(n_blocks), BS, sm_apply, s>>>(b, n_blocks);
    }
  }

  // trace + apply with the cross-block neighbour data prefetched (scalar problems)
  template <int P, int BS, int XCAP>
  static void run_xp(const DGProblem<T>* probs, int n, cudaStream_t s, int what) {
    using S = DGShape<P, 1>;
    using O = gen::Ops<P>;
    int64_t n_blocks = 0;
    const DGBatch<T> b = make_batch(probs, n, BS, n_blocks);
    const size_t sm_trace = size_t(BS) * (S::US + S::QS) * sizeof(T);
    const size_t sm_apply = (size_t(BS) * (2 * S::US + S::QS) + size_t(XCAP) * (O::NF + O::NFQ)) * sizeof(T);
    static std::atomic<uint64_t> conf_t{0}, conf_a{0};
    auto trace = dg_trace_kernel<P, 1, BS, T>;
    auto apply = dg_apply_xp_kernel<P, BS, XCAP, T>;
    opt_in_smem(trace, sm_trace, conf_t);
    opt_in_smem(apply, sm_apply, conf_a);
    if (what != 2) trace<<<unsigned(n_blocks), BS, sm_trace, s>>>(b, n_blocks);
    if (what != 1) apply<<<unsigned(n_blocks), BS, sm_apply, s>>>(b, n_blocks);
  }

  // phase-split scalar kernels (kernels_dg2.cuh): cross-block trace + apply
  template <int P, bool MASS, int BS, int MINB, bool YS = false>
  static void run_split(const DGProblem<T>* probs, int n, cudaStream_t s, int what) {
    using S = DG2Shape<P, YS>;
    int64_t n_blocks = 0;
    const DGBatch<T> b = make_batch(probs, n, BS, n_blocks);
    const size_t sm_trace = size_t(BS) * S::US * sizeof(T);
    const size_t sm_apply = size_t(BS) * S::ELEMS * sizeof(T);
    static std::atomic<uint64_t> conf_t{0}, conf_a{0};
    auto trace = dg_trace_cross_kernel<P, BS, T>;
    auto apply = dg_apply2_kernel<P, MASS, BS, T, MINB, YS>;
    opt_in_smem(trace, sm_trace, conf_t);
    opt_in_smem(apply, sm_apply, conf_a);
    if (what != 2) trace<<<unsigned(n_blocks), BS, sm_trace, s>>>(b, n_blocks);
    if (what != 1) apply<<<unsigned(n_blocks), BS, sm_apply, s>>>(b, n_blocks);
  }

  template <int P, int NC, bool MASS>
  static void run_warp(const DGProblem<T>* probs, int n, cudaStream_t s, int what) {
    using D = DG3<P, NC>;
    int64_t n_blocks = 0;
    const DGBatch<T> b = make_batch(probs, n, D::CELLS, n_blocks);
    const size_t sm_trace = size_t(D::TRACE_ELEMS) * sizeof(T);
    const size_t sm_apply = size_t(D::APPLY_ELEMS) * sizeof(T);
    static std::atomic<uint64_t> conf_t{0}, conf_a{0};
    opt_in_smem(dg3_trace_kernel<P, NC, T>, sm_trace, conf_t);
    opt_in_smem(dg3_apply_kernel<P, NC, MASS, T>, sm_apply, conf_a);
    if (what != 2) dg3_trace_kernel<P, NC, T><<<unsigned(n_blocks), D::THREADS, sm_trace, s>>>(b, n_blocks);
    if (what != 1) dg3_apply_kernel<P, NC, MASS, T><<<unsigned(n_blocks), D::THREADS, sm_apply, s>>>(b, n_blocks);
  }

  template <int P, int NC, bool MASS>
  static void run(const DGProblem<T>* probs, int n, cudaStream_t s, int what, int variant, int* status) {
    if (what == 3) {
      int64_t n_blocks = 0;
      const DGBatch<T> b = make_batch(probs, n, 128, n_blocks);
      dg_diagonal_kernel<P, NC, MASS, T><<<unsigned(n_blocks), 128, 0, s>>>(b, n_blocks);
    } else if (variant == 1) {
      // scalar problems: the apply pass loads its geometry and src rows while
      // the trace pass finishes (B200, DG P3 FP64 32^3: 68.5 -> 64.5 us per vmult)
      run_cell<P, NC, MASS, 128, 1, false, 1>(probs, n, s, what, status);
    } else if (variant == 2) {
      run_cell<P, NC, MASS, 64>(probs, n, s, what, status);
    } else if (variant == 3) {
      run_warp<P, NC, MASS>(probs, n, s, what);
    } else if (variant == 5) {
      // 64 cells per CTA, 5 CTAs per SM (up to 204 registers: no spills for P3)
      run_cell<P, NC, MASS, 64, 5, false>(probs, n, s, what, status);
    } else if (variant == 4) {
      // 64 cells per CTA, results aliased onto the staged src rows (scalar
      // problems), registers capped for 8 CTAs per SM; for scalar problems the
      // cell term is computed while the trace pass finishes (B200, DG P3 FP32
      // 32^3: 41.8 -> 38.0 us per vmult)
      if (NC == 1) run_cell<P, NC, MASS, 64, 8, (NC == 1), 2>(probs, n, s, what, status);
      else run_cell<P, NC, MASS, 64, 8, false>(probs, n, s, what, status);
    } else if (variant == 7 || variant == 9) {
      // phase-split scalar kernels (kernels_dg2.cuh): 7 results in registers,
      // 64 cells x 5 CTAs per SM; 9 results in shared memory, 64 cells x 4
      // CTAs (no spills); multi-component problems take the 128-cell form
      if constexpr (NC == 1) {
        if (variant == 7) run_split<P, MASS, 64, 5>(probs, n, s, what);
        else run_split<P, MASS, 64, 4, true>(probs, n, s, what);
      } else {
        run_cell<P, NC, MASS, 128>(probs, n, s, what, status);
      }
    } else if (variant == 11) {
      // 128 cells per CTA with the cross-block neighbour data prefetched into
      // shared memory; multi-component and mass problems take the 128-cell form
      if constexpr (NC == 1 && !MASS) run_xp<P, 128, 192>(probs, n, s, what);
      else run_cell<P, NC, MASS, 128>(probs, n, s, what, status);
    } else {
      throw Error(FEM_ERR_ARG, "DG: kernel variant must be 0..5, 7, 9 or 11");
    }
    SFEM_CUDA(cudaGetLastError());
  }
};

template <typename T>
class DGBatchImpl final : public Batch {
 public:
  std::vector<DGOperator<T>*> ops;
  // an operator listed more than once (several right-hand sides on one mesh)
  // gets a trace scratch of its own for every repeat: the two passes of one
  // launch must not share it between problems
  std::vector<DevBuf<T>> extra_q;
  std::vector<int> q_of;  // -1: the operator's own scratch, else index into extra_q
  OpConfig cfg;
  explicit DGBatchImpl(const std::vector<Operator*>& o) {
    SFEM_REQUIRE(!o.empty() && int(o.size()) <= kMaxBatch, FEM_ERR_ARG, "batch: 1..40 operators");
    cfg = o[0]->cfg;
    for (auto* op : o) {
      auto* d = dynamic_cast<DGOperator<T>*>(op);
      SFEM_REQUIRE(d != nullptr, FEM_ERR_ARG, "batch: only DG/Helmholtz operators of one precision");
      SFEM_REQUIRE(d->cfg.degree == cfg.degree && d->cfg.kind == cfg.kind &&
                       d->cfg.n_components == cfg.n_components,
                   FEM_ERR_ARG, "batch: operators must share kind, degree and components");
      int repeat = -1;
      for (auto* prev : ops)
        if (prev == d) repeat = 0;
      if (repeat == 0) {
        extra_q.emplace_back(d->scratch_bytes() / sizeof(T));
        repeat = int(extra_q.size()) - 1;
      }
      q_of.push_back(repeat);
      ops.push_back(d);
    }
  }
  void vmult(void* const* dst, const void* const* src, cudaStream_t s) override {
    DGProblem<T> probs[kMaxBatch];
    for (size_t i = 0; i < ops.size(); ++i) {
      probs[i] = ops[i]->problem(src[i], dst[i]);
      if (q_of[i] >= 0) probs[i].Q = extra_q[q_of[i]].p;
    }
    DGOperator<T>::launch_dg(cfg, probs, int(ops.size()), s, 0, ops[0]->d_status.p);
  }
  int variant() const override { return cfg.kernel_variant; }
  void set_variant(int v) override {
    SFEM_REQUIRE(v >= 0 && v <= 11 && v != 6 && v != 8 && v != 10, FEM_ERR_ARG,
                 "batch: kernel variant must be 0..5, 7, 9 or 11");
    cfg.kernel_variant = v;
  }
  TuneResult tune(int reps, bool use_cache) override {
    TuneResult res;
    res.us.assign(5, 0.0);
    int64_t cells = 0;
    for (auto* o : ops) cells += o->n_cells;
    const std::string key = "batch" + std::to_string(ops.size()) + "," + tune_key(cfg, cells);
    if (use_cache) {
      const int v = tune_lookup(key);
      if (v > 0) {
        cfg.kernel_variant = v;
        res.variant = v;
        res.cached = true;
        return res;
      }
    }
    std::vector<DevBuf<T>> bufs;
    std::vector<void*> d(ops.size());
    std::vector<const void*> x(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) {
      bufs.emplace_back(size_t(ops[i]->m));
      bufs.emplace_back(size_t(ops[i]->m));
      SFEM_CUDA(cudaMemset(bufs[2 * i].p, 0, sizeof(T) * ops[i]->m));
    }
    for (size_t i = 0; i < ops.size(); ++i) {
      x[i] = bufs[2 * i].p;
      d[i] = bufs[2 * i + 1].p;
    }
    cudaStream_t s = nullptr;
    SFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const int keep = cfg.kernel_variant;
    double best = 1e300;
    try {
      for (int v : tune_candidates(cfg)) {
        cfg.kernel_variant = v;
        const double us = time_launches([&](cudaStream_t st) { vmult(d.data(), x.data(), st); }, reps, s);
        res.us[v - 1] = us;
        if (us < best) {
          best = us;
          res.variant = v;
        }
      }
    } catch (...) {
      cfg.kernel_variant = keep;
      cudaStreamDestroy(s);
      throw;
    }
    cudaStreamDestroy(s);
    cfg.kernel_variant = res.variant;
    tune_store(key, res.variant, res.us);
    return res;
  }
};

}  // namespace

void Operator::inverse_diagonal(void* diag, cudaStream_t s) {
  diagonal(diag, s);
  const unsigned grid = blocks_for(m, 256);
  if (cfg.precision == FEM_FP64)
    inverse_diagonal_kernel<double><<<grid, 256, 0, s>>>(m, static_cast<double*>(diag));
  else
    inverse_diagonal_kernel<float><<<grid, 256, 0, s>>>(m, static_cast<float*>(diag));
  SFEM_CUDA(cudaGetLastError());
}

std::unique_ptr<Operator> make_operator(const Mesh& mesh, const OpConfig& cfg) {
  SFEM_REQUIRE(cfg.degree >= 1 && cfg.degree <= 3, FEM_ERR_ARG, "operator: degree must be 1, 2 or 3");
  SFEM_REQUIRE(cfg.precision == FEM_FP64 || cfg.precision == FEM_FP32, FEM_ERR_ARG, "operator: bad precision");
  std::unique_ptr<Operator> op;
  if (mesh.curved) {
    SFEM_REQUIRE(cfg.kind == FEM_CG, FEM_ERR_ARG,
                 "curved meshes: CG operators only (the DG face terms are affine in this library)");
    op = make_curved_cg_operator(mesh, cfg);
  } else if (cfg.kind == FEM_CG) {
    SFEM_REQUIRE(cfg.n_components == 1 || cfg.n_components == 3, FEM_ERR_ARG, "CG: n_components must be 1 or 3");
    if (cfg.n_components == 3) {
      SFEM_REQUIRE(!cfg.weak_bc && (cfg.kernel_variant == 0 || cfg.kernel_variant == 1), FEM_ERR_ARG,
                   "CG with 3 components: strong constraints and the cell kernel only");
      if (cfg.precision == FEM_FP64) op = std::make_unique<CGVectorOperator<double>>(mesh, cfg);
      else op = std::make_unique<CGVectorOperator<float>>(mesh, cfg);
    } else if (cfg.precision == FEM_FP64) {
      op = std::make_unique<CGOperator<double>>(mesh, cfg);
    } else {
      op = std::make_unique<CGOperator<float>>(mesh, cfg);
    }
  } else if (cfg.kind == FEM_DG || cfg.kind == FEM_HELMHOLTZ) {
    if (cfg.precision == FEM_FP64) op = std::make_unique<DGOperator<double>>(mesh, cfg);
    else op = std::make_unique<DGOperator<float>>(mesh, cfg);
  } else {
    throw Error(FEM_ERR_ARG, "operator: unknown kind");
  }
  op->mesh = &mesh;
  return op;
}

void csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col, const void* val, const void* x, void* y,
              int precision, cudaStream_t s) {
  constexpr int LANES = 8;
  const unsigned grid = blocks_for(std::max<int64_t>(n_rows, 1) * LANES, 256);
  if (precision == FEM_FP64)
    csr_spmv_kernel<double, LANES><<<grid, 256, 0, s>>>(n_rows, row_ptr, col, static_cast<const double*>(val),
                                                        static_cast<const double*>(x), static_cast<double*>(y));
  else
    csr_spmv_kernel<float, LANES><<<grid, 256, 0, s>>>(n_rows, row_ptr, col, static_cast<const float*>(val),
                                                       static_cast<const float*>(x), static_cast<float*>(y));
  SFEM_CUDA(cudaGetLastError());
}

std::unique_ptr<Operator> make_local_operator(std::shared_ptr<const Mesh> mesh, const CGDofs* dofs,
                                              const std::vector<uint8_t>* identity, const OpConfig& cfg) {
  SFEM_REQUIRE(cfg.degree >= 1 && cfg.degree <= 3, FEM_ERR_ARG, "operator: degree must be 1, 2 or 3");
  SFEM_REQUIRE(cfg.precision == FEM_FP64 || cfg.precision == FEM_FP32, FEM_ERR_ARG, "operator: bad precision");
  std::unique_ptr<Operator> op;
  if (cfg.kind == FEM_CG) {
    SFEM_REQUIRE(dofs && identity, FEM_ERR_INTERNAL, "CG local operator needs its numbering");
    if (cfg.precision == FEM_FP64) op = std::make_unique<CGOperator<double>>(*mesh, *dofs, identity, cfg);
    else op = std::make_unique<CGOperator<float>>(*mesh, *dofs, identity, cfg);
  } else {
    op = make_operator(*mesh, cfg);
  }
  op->mesh = mesh.get();
  op->owned_mesh = std::move(mesh);
  return op;
}

std::unique_ptr<Batch> make_batch(const std::vector<Operator*>& ops) {
  SFEM_REQUIRE(!ops.empty(), FEM_ERR_ARG, "batch: empty");
  if (ops[0]->cfg.precision == FEM_FP64) return std::make_unique<DGBatchImpl<double>>(ops);
  return std::make_unique<DGBatchImpl<float>>(ops);
}

}  // namespace sfem
