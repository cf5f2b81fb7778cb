// ww3-gpu_b200/csrc/abi_sur.cpp
// The learned DIA surrogate behind the C ABI: a BF16 MLP trained on the device by this
// library's own forward and backward kernels (mlp_gemm.cu, mlp_ops.cu), and the gated W3SNL1
// entry that uses it, with the plain DIA as the fallback for every rejected point.
//
// The reference has no learned component; the function the surrogate stands in for is W3SNL1
// (ww3-gpu kokkos/src/ww_kokkos/snl1_team.hpp:351-497), whose batch entry ww_snl1
// (ww_kokkos_c.hpp:102-118) the gated entry mirrors argument for argument.
//
// Two layers of entries:
//   ww_mlp_*  a plain MLP (din -> dh -> dh -> dh -> dout, GELU, BF16 weights and activations,
//             FP32 accumulation and master weights, AdamW), by handle. Tests check its GEMMs
//             and gradients against CPU references through these.
//   ww_sur_*  the surrogate of one DIA grid: synthetic training data labelled by the plain DIA
//             kernel, training, gate calibration against the FP64 DIA, and ww_snl1_gated.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "mlp.cuh"
#include "mlp_ops.cuh"
#include "snl1_kernel.cuh"
#include "snl1_tables.hpp"
#include "wwb_common.hpp"

namespace wwb {
bool snl1_grid_dev(int igrid, Snl1Dev* out);                                        // abi_snl1.cpp
bool snl1_grid_config(int igrid, Snl1Config* cfg, std::vector<float>* sig);         // abi_snl1.cpp

namespace {
using bf16 = __nv_bfloat16;
using namespace mlp;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    reset();
    if (count == 0) return;
    WWB_CHECK(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void zero(cudaStream_t st) {
    if (p) WWB_CHECK(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  }
};

Status g_mlp_status;
Status g_sur_status;

struct Layer {
  int n = 0, k = 0, nvalid = 0;  // weight n x k; rows >= nvalid stay zero
  DBuf<float> w, m, v, g, b, bm, bv, bg;
  DBuf<bf16> wb, wt;
};

/// Tile width of a GEMM whose output has n columns.
int pick_bn(int n) {
  for (int bn : {256, 192, 128, 64})
    if (n % bn == 0) return bn;
  return 0;
}

/// Reduction split of a weight-gradient GEMM: enough work units to fill the SMs.
int pick_splits(int tiles, int kblocks) {
  int sms = runtime().sm_count > 0 ? runtime().sm_count : 148;
  int s = 1;
  while (tiles * s < sms && kblocks % (2 * s) == 0 && kblocks / (2 * s) >= 4) s *= 2;
  return s;
}

struct Mlp {
  int din = 0, dh = 0, dout = 0, nvalid = 0, cap = 0;
  Layer L[4];
  // training activations (cap rows)
  DBuf<bf16> x0, x0t, z[3], act[3], actt[3], g4, g4t, gh[3], ght[3];
  DBuf<float> out, tb;
  // inference activations (icap rows)
  int icap = 0;
  DBuf<bf16> ix0, ih[2];
  DBuf<float> iout;
  DBuf<int> err;
  DBuf<float> loss;  // 3 accumulators
  long long step = 0;
  cudaStream_t st = nullptr;
  ~Mlp() {
    if (st) cudaStreamDestroy(st);
  }
};

void mlp_alloc(Mlp& m, int din, int dh, int dout, int nvalid, int cap, uint64_t seed) {
  m.din = din;
  m.dh = dh;
  m.dout = dout;
  m.nvalid = nvalid;
  m.cap = cap;
  WWB_CHECK(cudaStreamCreateWithFlags(&m.st, cudaStreamNonBlocking));
  const int dims[5] = {din, dh, dh, dh, dout};
  for (int l = 0; l < 4; ++l) {
    Layer& L = m.L[l];
    L.n = dims[l + 1];
    L.k = dims[l];
    L.nvalid = l == 3 ? std::min(dout, nvalid + 1) : L.n;  // + the error-head row
    const size_t nw = static_cast<size_t>(L.n) * L.k;
    L.w.alloc(nw);
    L.m.alloc(nw);
    L.v.alloc(nw);
    L.g.alloc(nw);
    L.wb.alloc(nw);
    L.wt.alloc(nw);
    L.b.alloc(L.n);
    L.bm.alloc(L.n);
    L.bv.alloc(L.n);
    L.bg.alloc(L.n);
    L.m.zero(m.st);
    L.v.zero(m.st);
    L.g.zero(m.st);
    L.b.zero(m.st);
    L.bm.zero(m.st);
    L.bv.zero(m.st);
    L.bg.zero(m.st);
    init_weights(seed + 1000003ull * (l + 1), L.n, L.k, L.nvalid, l == 3 ? 0.5f : 1.0f, L.w.p,
                 L.wb.p, L.wt.p, m.st);
  }
  const size_t c = static_cast<size_t>(cap);
  m.x0.alloc(c * din);
  m.x0t.alloc(c * din);
  for (int i = 0; i < 3; ++i) {
    m.z[i].alloc(c * dh);
    m.act[i].alloc(c * dh);
    m.actt[i].alloc(c * dh);
    m.gh[i].alloc(c * dh);
    m.ght[i].alloc(c * dh);
  }
  m.g4.alloc(c * dout);
  m.g4t.alloc(c * dout);
  m.out.alloc(c * dout);
  m.err.alloc(1);
  m.err.zero(m.st);
  m.loss.alloc(3);
  WWB_CHECK(cudaStreamSynchronize(m.st));
}

void mlp_infer_alloc(Mlp& m, int rows) {
  if (rows <= m.icap) return;
  const size_t c = static_cast<size_t>(rows);
  m.ix0.alloc(c * m.din);
  m.ih[0].alloc(c * m.dh);
  m.ih[1].alloc(c * m.dh);
  m.iout.alloc(c * m.dout);
  m.icap = rows;
}

/// Inference GEMMs of at least this many rows would run with paired tiles (two CTAs of a
/// cluster per 256-row tile, cta_group::2). At the surrogate's shapes (65,536 x 1024 x 1024 and
/// x 1344) the paired kernel measured slower than one CTA per 128-row tile (the main loop is not
/// short of shared-memory bandwidth; the epilogue is the limit), so the threshold keeps it off;
/// ww_mlp_gemm's mode + 16 runs it.
constexpr int kPairRows = 1 << 30;  // measured slower on B200 at these shapes: kept off
int infer_pair(int rows) { return rows >= kPairRows ? 1 : 0; }

GemmArgs args(int M, int N, int K, const Mlp& m) {
  GemmArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.bn = pick_bn(N);
  g.splits = 1;
  g.err = m.err.p;
  return g;
}

void run_gemm(int mode, const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t st) {
  const char* why = nullptr;
  if (!gemm_shape_ok(g, a, b, &why)) throw CudaError(cudaErrorInvalidValue, why);
  gemm(mode, g, a, b, st);
}

/// Inference forward of rows [0, rows) of x (default m.ix0) into out (default m.iout; fp32,
/// dout columns).
void mlp_forward_infer(Mlp& m, int rows, cudaStream_t st, const bf16* x = nullptr,
                       float* out = nullptr) {
  const bf16* in = x ? x : m.ix0.p;
  int kin = m.din;
  for (int l = 0; l < 3; ++l) {
    GemmArgs g = args(rows, m.dh, kin, m);
    g.pair = infer_pair(rows);
    g.bias = m.L[l].b.p;
    g.out = m.ih[l & 1].p;
    g.ldo = m.dh;
    run_gemm(kEpiGeluInfer, g, make_operand(in, rows, kin, kin, kBM),
             make_operand(m.L[l].wb.p, m.dh, kin, kin, gemm_b_box(g)), st);
    in = m.ih[l & 1].p;
    kin = m.dh;
  }
  GemmArgs g = args(rows, m.dout, m.dh, m);
  g.pair = infer_pair(rows);
  g.bias = m.L[3].b.p;
  g.out_f32 = out ? out : m.iout.p;
  g.ldo = m.dout;
  run_gemm(kEpiF32, g, make_operand(in, rows, m.dh, m.dh, kBM),
           make_operand(m.L[3].wb.p, m.dout, m.dh, m.dh, gemm_b_box(g)), st);
}

/// One training step on rows [0, rows) of m.x0 (bf16) and targets t (rows x ldt fp32):
/// forward with the training epilogues, loss and output gradient, backward, then AdamW when
/// `apply`. `sg` carries the surrogate's loss terms (null: plain MSE).
void mlp_train_step(Mlp& m, int rows, const float* t, int ldt, const SurGrid* sg,
                    const float* ps, const LossWeights& lw, const Adam* adam, float* loss,
                    cudaStream_t st) {
  if (rows % 128 != 0 || rows > m.cap)
    throw CudaError(cudaErrorInvalidValue, "training batch must be a multiple of 128 within capacity");
  const int cap = m.cap;
  transpose(m.x0.p, rows, m.din, m.din, m.x0t.p, cap, st);
  // Forward.
  const bf16* in = m.x0.p;
  int kin = m.din;
  for (int l = 0; l < 3; ++l) {
    GemmArgs g = args(rows, m.dh, kin, m);
    g.bias = m.L[l].b.p;
    g.out = m.act[l].p;
    g.out_t = m.actt[l].p;
    g.aux = m.z[l].p;
    g.ldo = m.dh;
    g.ldt = cap;
    run_gemm(kEpiGeluTrain, g, make_operand(in, rows, kin, kin, kBM),
             make_operand(m.L[l].wb.p, m.dh, kin, kin, g.bn), st);
    in = m.act[l].p;
    kin = m.dh;
  }
  {
    GemmArgs g = args(rows, m.dout, m.dh, m);
    g.bias = m.L[3].b.p;
    g.out_f32 = m.out.p;
    g.ldo = m.dout;
    run_gemm(kEpiF32, g, make_operand(in, rows, m.dh, m.dh, kBM),
             make_operand(m.L[3].wb.p, m.dout, m.dh, m.dh, g.bn), st);
  }
  // Loss and dL/dout.
  SurGrid plain{};
  plain.dout = m.dout;
  plain.nth = 1;
  loss_grad(sg ? *sg : plain, lw, rows, m.nvalid, m.out.p, m.dout, t, ldt, sg ? ps : nullptr,
            m.g4.p, m.dout, loss, st);
  transpose(m.g4.p, rows, m.dout, m.dout, m.g4t.p, cap, st);
  // Backward: layer l's input gradient G (rows x n_l) and its transpose GT (n_l x rows).
  const bf16* G = m.g4.p;
  const bf16* GT = m.g4t.p;
  for (int l = 3; l >= 0; --l) {
    Layer& L = m.L[l];
    const bf16* XT = l == 0 ? m.x0t.p : m.actt[l - 1].p;  // layer input, transposed (k x rows)
    {  // dW = G^T X: (n x rows) . (k x rows)^T
      GemmArgs g = args(L.n, L.k, rows, m);
      const int tiles = ((L.n + kBM - 1) / kBM) * (L.k / g.bn);
      g.splits = pick_splits(tiles, rows / kBK);
      g.out_f32 = L.g.p;
      g.ldo = L.k;
      run_gemm(kEpiAtomic, g, make_operand(GT, L.n, rows, cap, kBM),
               make_operand(XT, L.k, rows, cap, g.bn), st);
    }
    colsum(GT, L.n, rows, cap, L.bg.p, st);
    if (l == 0) break;
    {  // dX = G W, times GELU'(z) of the layer below: (rows x n) . (k x n)^T
      GemmArgs g = args(rows, L.k, L.n, m);
      g.aux = m.z[l - 1].p;
      g.out = m.gh[l - 1].p;
      g.out_t = m.ght[l - 1].p;
      g.ldo = L.k;
      g.ldt = cap;
      run_gemm(kEpiDGelu, g, make_operand(G, rows, L.n, L.n, kBM),
               make_operand(L.wt.p, L.k, L.n, L.n, g.bn), st);
    }
    G = m.gh[l - 1].p;
    GT = m.ght[l - 1].p;
  }
  if (adam) {
    for (int l = 0; l < 4; ++l) {
      Layer& L = m.L[l];
      adamw(*adam, L.n, L.k, L.w.p, L.m.p, L.v.p, L.g.p, L.wb.p, L.wt.p, st);
      adamw_vec(*adam, L.n, L.b.p, L.bm.p, L.bv.p, L.bg.p, st);
    }
  }
}

Adam adam_at(long long step, float lr, float wd) {
  Adam h{};
  h.lr = lr;
  h.beta1 = 0.9f;
  h.beta2 = 0.999f;
  h.eps = 1e-8f;
  h.wd = wd;
  h.c1 = static_cast<float>(1.0 - std::pow(0.9, static_cast<double>(step)));
  h.c2 = static_cast<float>(1.0 - std::pow(0.999, static_cast<double>(step)));
  return h;
}

size_t mlp_param_count(const Mlp& m) {
  size_t n = 0;
  for (const Layer& L : m.L) n += static_cast<size_t>(L.n) * L.k + L.n;
  return n;
}

/// Copies parameters (or with grads=true the last gradients) between the device and a host
/// array laid out layer by layer as W (n x k, row-major) then b (n).
void mlp_params(Mlp& m, float* host, bool to_host, bool grads) {
  size_t o = 0;
  for (Layer& L : m.L) {
    const size_t nw = static_cast<size_t>(L.n) * L.k;
    float* w = grads ? L.g.p : L.w.p;
    float* b = grads ? L.bg.p : L.b.p;
    if (to_host) {
      WWB_CHECK(cudaMemcpyAsync(host + o, w, nw * 4, cudaMemcpyDeviceToHost, m.st));
      WWB_CHECK(cudaMemcpyAsync(host + o + nw, b, L.n * 4, cudaMemcpyDeviceToHost, m.st));
    } else {
      WWB_CHECK(cudaMemcpyAsync(w, host + o, nw * 4, cudaMemcpyHostToDevice, m.st));
      WWB_CHECK(cudaMemcpyAsync(b, host + o + nw, L.n * 4, cudaMemcpyHostToDevice, m.st));
      to_bf16(L.w.p, L.n, L.k, L.wb.p, L.wt.p, m.st);
    }
    o += nw + L.n;
  }
  WWB_CHECK(cudaStreamSynchronize(m.st));
}

int take_err(Mlp& m) {
  int v = 0;
  WWB_CHECK(cudaMemcpyAsync(&v, m.err.p, sizeof(int), cudaMemcpyDeviceToHost, m.st));
  WWB_CHECK(cudaStreamSynchronize(m.st));
  if (v) WWB_CHECK(cudaMemset(m.err.p, 0, sizeof(int)));
  return v;
}

std::map<int, std::unique_ptr<Mlp>>& mlps() {
  static auto* m = new std::map<int, std::unique_ptr<Mlp>>();
  return *m;
}

// ------------------------------------------------------------------------------ the surrogate

constexpr int kInferRows = 65536;  // inference chunk (the activations of one chunk stay resident)

struct Sur {
  Snl1Dev dia{};
  Snl1Config cfg{};
  std::vector<float> sig;
  Mlp net;
  SurGrid g{};
  DBuf<float> rowscale;
  // dataset: normalised inputs, targets and per-point scales (2 NK floats each)
  long long n_data = 0, n_train = 0;
  DBuf<bf16> xs;
  DBuf<float> ts, pss, tb_ps;
  // inference scratch (per chunk)
  DBuf<float> ps, gv, gsum, head;
  DBuf<int> shift, rej, nrej, nrej_total;
  DBuf<int> rej_all;  ///< the rejected points of one gated call (all its chunks)
  GateParams gate{0.05f, 1e30f};
  LossWeights lw{0.0f, 0.0f, 1};
  // FP64 judge
  DiaF64 f64{};
  bool f64_ok = false;
  DBuf<double> af11d, sigd;
  // host-pointer entry: three chunk slots, copies in and out overlapping the compute
  struct Pipe {
    static constexpr int kSlots = 3;
    /// Rows of D per chunk that come back packed (the rejected points'); a chunk with more
    /// rejected points brings its whole D back.
    static constexpr int kDRows = kInferRows / 8;
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    cudaEvent_t copied[kSlots] = {}, computed[kSlots] = {}, drained[kSlots] = {};
    DBuf<float> a[kSlots], cg[kSlots], kd[kSlots], s[kSlots], d[kSlots], dc[kSlots];
    DBuf<int> dl[kSlots], dn[kSlots];
    float* h_dc[kSlots] = {};  ///< page-locked: the packed D rows of the slot's chunk
    int* h_dl[kSlots] = {};    ///< their point indices in the chunk
    int* h_dn[kSlots] = {};    ///< the chunk's count of rejected points
    bool ready = false;
    ~Pipe() {
      for (int k = 0; k < kSlots; ++k) {
        if (copied[k]) cudaEventDestroy(copied[k]);
        if (computed[k]) cudaEventDestroy(computed[k]);
        if (drained[k]) cudaEventDestroy(drained[k]);
        if (h_dc[k]) cudaFreeHost(h_dc[k]);
        if (h_dl[k]) cudaFreeHost(h_dl[k]);
        if (h_dn[k]) cudaFreeHost(h_dn[k]);
      }
      for (cudaStream_t x : {in, comp, out})
        if (x) cudaStreamDestroy(x);
    }
  } pipe;
  /// A side stream for the D zeros of a gated call, so they overlap the network's GEMMs (which
  /// leave most of the HBM bandwidth unused) instead of adding a pass of their own.
  struct Side {
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    void make() {
      if (st) return;
      WWB_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      WWB_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
      WWB_CHECK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    }
    ~Side() {
      if (fork) cudaEventDestroy(fork);
      if (join) cudaEventDestroy(join);
      if (st) cudaStreamDestroy(st);
    }
  } side;
};

std::map<int, std::unique_ptr<Sur>>& surs() {
  static auto* m = new std::map<int, std::unique_ptr<Sur>>();
  return *m;
}

Sur* find_sur(int igrid) {
  auto it = surs().find(igrid);
  if (it == surs().end() || !runtime().ready) {
    g_sur_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_sur: no surrogate for this grid");
    return nullptr;
  }
  return it->second.get();
}

void sur_scratch(Sur& s, int rows) {
  mlp_infer_alloc(s.net, rows);
  if (s.shift.n < static_cast<size_t>(rows)) {
    s.ps.alloc(static_cast<size_t>(rows) * 2 * s.g.nk);
    s.gv.alloc(static_cast<size_t>(rows) * 2);
    s.gsum.alloc(static_cast<size_t>(rows) * 2);
    s.head.alloc(rows);
    s.shift.alloc(rows);
    s.rej.alloc(rows);
  }
  if (s.rej_all.n < static_cast<size_t>(rows)) s.rej_all.alloc(rows);
  if (!s.nrej.p) {
    s.nrej.alloc(1);
    s.nrej_total.alloc(1);
  }
}

/// Whether the output layer runs the TMA-store epilogue (kEpiSurOutTma): when the spectral grid
/// suits it, unless WW_B200_SUR_EPILOGUE=6 asks for the row-by-row one (kEpiSurOut; the same
/// S bits, for comparisons).
bool sur_tma_epilogue(const Sur& s) {
  const char* e = std::getenv("WW_B200_SUR_EPILOGUE");
  if (e != nullptr && std::strcmp(e, "6") == 0) return false;
  return sur_tma_ok(s.g.nk, s.g.nth);
}

/// One chunk (n <= kInferRows points) through the network with the fused output epilogue:
/// S and D of every point, then the gate: rejected points listed in s.rej and counted in s.nrej
/// (zeroed here), or, with `rej` given, appended as base + index to rej at the count *rej_n.
void sur_chunk_out(Sur& s, int n, const float* a, const float* cg, const float* kd, float* so,
                   float* dd, int* accepted, float* gv, const GateParams& gate, int* total,
                   cudaStream_t st, int* rej = nullptr, int* rej_n = nullptr, int base = 0) {
  Mlp& m = s.net;
  // The inputs, and zeros for the gate sums the output epilogue adds to (D is zeroed by the
  // caller).
  prep(s.g, n, a, cg, kd, m.ix0.p, m.din, s.ps.p, s.shift.p, st, nullptr, s.gsum.p);
  const bf16* in = m.ix0.p;
  int kin = m.din;
  for (int l = 0; l < 3; ++l) {
    GemmArgs g = args(n, m.dh, kin, m);
    g.pair = infer_pair(n);
    g.bias = m.L[l].b.p;
    g.out = m.ih[l & 1].p;
    g.ldo = m.dh;
    run_gemm(kEpiGeluInfer, g, make_operand(in, n, kin, kin, kBM),
             make_operand(m.L[l].wb.p, m.dh, kin, kin, gemm_b_box(g)), st);
    in = m.ih[l & 1].p;
    kin = m.dh;
  }
  GemmArgs g = args(n, m.dout, m.dh, m);
  g.pair = infer_pair(n);
  g.bias = m.L[3].b.p;
  g.ldo = m.dout;
  g.sur = SurOut{s.ps.p, s.shift.p, s.rowscale.p, so, dd, s.head.p, s.gsum.p, s.g.nspec,
                 s.g.nth, s.g.nk};
  const char* why = nullptr;
  if (sur_tma_epilogue(s) && !g.pair) {
    // Tiles of four frequency rows, each quarter rotated in shared memory and stored by TMA;
    // N padded to whole tiles (B's rows past DOUT read as zeros).
    g.bn = 4 * s.g.nth;
    g.N = (m.dout + g.bn - 1) / g.bn * g.bn;
    g.ldo = g.N;  // S goes through the store map; the row stride check is moot
    g.b_rows = m.dout;
    const CUtensorMap smap = make_store_map(so, n, s.g.nspec, g.bn);
    g.store = &smap;
    if (!sur_out_ok(g, &why)) throw CudaError(cudaErrorInvalidValue, why);
    run_gemm(kEpiSurOutTma, g, make_operand(in, n, m.dh, m.dh, kBM),
             make_operand(m.L[3].wb.p, m.dout, m.dh, m.dh, g.bn), st);
  } else {
    if (!sur_out_ok(g, &why)) throw CudaError(cudaErrorInvalidValue, why);
    run_gemm(kEpiSurOut, g, make_operand(in, n, m.dh, m.dh, kBM),
             make_operand(m.L[3].wb.p, m.dout, m.dh, m.dh, gemm_b_box(g)), st);
  }
  if (rej == nullptr) {
    WWB_CHECK(cudaMemsetAsync(s.nrej.p, 0, sizeof(int), st));
    rej = s.rej.p;
    rej_n = s.nrej.p;
  }
  gate_points(gate, n, s.gsum.p, s.head.p, accepted, gv, rej, rej_n, total, st, base);
}

/// The surrogate's S for npts points (device arrays) into s/d, gated, with the plain DIA on the
/// rejected points; accepted (optional) gets 1/0 per point.
void sur_apply(Sur& s, int npts, const float* a, const float* cg, const float* kd, float* so,
               float* dd, int* accepted, const GateParams& gate, cudaStream_t st, bool fallback,
               bool reset_count = true) {
  const int nspec = s.g.nspec, nk = s.g.nk;
  sur_scratch(s, std::min(npts, kInferRows));
  if (s.rej_all.n < static_cast<size_t>(npts)) s.rej_all.alloc(npts);
  if (reset_count) WWB_CHECK(cudaMemsetAsync(s.nrej_total.p, 0, sizeof(int), st));
  // Every chunk's rejected points go into one list of the call's points, so the plain DIA runs
  // once on all of them (one launch that fills the GPU) instead of once per chunk.
  WWB_CHECK(cudaMemsetAsync(s.nrej.p, 0, sizeof(int), st));
  // D = 0 for every point (the surrogate does not model the diagonal term), on the side stream
  // while the network runs; the plain DIA overwrites the rejected points' D after it.
  s.side.make();
  WWB_CHECK(cudaEventRecord(s.side.fork, st));
  WWB_CHECK(cudaStreamWaitEvent(s.side.st, s.side.fork, 0));
  WWB_CHECK(cudaMemsetAsync(dd, 0, static_cast<size_t>(npts) * nspec * sizeof(float), s.side.st));
  WWB_CHECK(cudaEventRecord(s.side.join, s.side.st));
  for (int p0 = 0; p0 < npts; p0 += kInferRows) {
    const int n = std::min(kInferRows, npts - p0);
    sur_chunk_out(s, n, a + static_cast<size_t>(p0) * nspec, cg + static_cast<size_t>(p0) * nk,
                  kd + p0, so + static_cast<size_t>(p0) * nspec,
                  dd + static_cast<size_t>(p0) * nspec, accepted ? accepted + p0 : nullptr,
                  nullptr, gate, s.nrej_total.p, st, s.rej_all.p, s.nrej.p, p0);
  }
  WWB_CHECK(cudaStreamWaitEvent(st, s.side.join, 0));
  if (fallback && !launch_snl1_list(s.dia, npts, s.rej_all.p, s.nrej.p, a, cg, kd, so, dd,
                                    nullptr, st))
    throw CudaError(cudaErrorInvalidValue, "gated DIA: the pair and band kernels cannot run this grid");
}

void build_f64(Sur& s) {
  Snl1Tables t;
  if (!build_snl1_tables(s.cfg, s.sig.data(), t)) return;
  Snl1WeightsF64 w;
  if (!build_snl1_weights_f64(s.cfg, s.sig.data(), t, w)) return;
  s.af11d.alloc(w.af11_row.size());
  WWB_CHECK(cudaMemcpy(s.af11d.p, w.af11_row.data(), w.af11_row.size() * 8, cudaMemcpyHostToDevice));
  std::vector<double> sd(s.sig.begin(), s.sig.end());
  s.sigd.alloc(sd.size());
  WWB_CHECK(cudaMemcpy(s.sigd.p, sd.data(), sd.size() * 8, cudaMemcpyHostToDevice));
  DiaF64& f = s.f64;
  f.nk = s.cfg.nk;
  f.nth = s.cfg.nth;
  f.nfr = t.nfr;
  f.nfrhgh = t.nfrhgh;
  f.nfrchg = t.nfrchg;
  f.nspec = t.nspec;
  f.nspecx = t.nspecx;
  f.dal1 = w.dal1;
  f.dal2 = w.dal2;
  f.dal3 = w.dal3;
  for (int j = 0; j < 8; ++j) {
    f.awg[j] = w.awg[j];
    f.swg[j] = w.swg[j];
  }
  f.snlc1 = s.cfg.snlc1;
  f.kdcon = s.cfg.kdcon;
  f.kdmn = s.cfg.kdmn;
  f.snls1 = s.cfg.snls1;
  f.snls2 = s.cfg.snls2;
  f.snls3 = s.cfg.snls3;
  f.fachfe = s.cfg.fachfe;
  f.dth = s.cfg.dth;
  f.xfr = s.cfg.xfr;
  f.ipim = s.dia.ipim;
  f.ic = s.dia.ic;
  f.af11 = s.af11d.p;
  f.sig = s.sigd.p;
  s.f64_ok = dia_f64_smem(f) <= 227 * 1024;
}

/// The per-row target scales from host values.
void set_rowscale(Sur& s, const std::vector<float>& rs) {
  WWB_CHECK(cudaMemcpy(s.rowscale.p, rs.data(), rs.size() * 4, cudaMemcpyHostToDevice));
}

int sur_fail(int code, const char* what) { return g_sur_status.fail(code, what); }

}  // namespace

void release_sur_contexts() {
  surs().clear();
  mlps().clear();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

// ------------------------------------------------------------------------------ ww_mlp_*

int ww_mlp_create(int din, int dh, int dout, int nvalid, int cap, unsigned long long seed,
                  int* handle) {
  try {
    if (!runtime().ready) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_mlp_create before ww_kokkos_init");
    if (!handle || din <= 0 || dh <= 0 || dout <= 0 || din % 64 || dh % 64 || dout % 64 ||
        nvalid <= 0 || nvalid > dout || cap <= 0 || cap % 128)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                               "ww_mlp_create: widths must be positive multiples of 64, nvalid in "
                               "(0, dout], capacity a multiple of 128");
    auto m = std::make_unique<Mlp>();
    mlp_alloc(*m, din, dh, dout, nvalid, cap, seed);
    const int h = mlps().empty() ? 1 : mlps().rbegin()->first + 1;
    mlps()[h] = std::move(m);
    *handle = h;
    g_mlp_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_mlp_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

int ww_mlp_destroy(int handle) {
  auto it = mlps().find(handle);
  if (it == mlps().end()) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_mlp_destroy: unknown handle");
  mlps().erase(it);
  g_mlp_status.ok();
  return WW_KOKKOS_OK;
}

long long ww_mlp_param_count(int handle) {
  auto it = mlps().find(handle);
  return it == mlps().end() ? -1 : static_cast<long long>(mlp_param_count(*it->second));
}

static int mlp_copy(int handle, float* host, bool to_host, bool grads, const char* who) {
  try {
    auto it = mlps().find(handle);
    if (it == mlps().end()) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, who);
    if (!host) return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, who);
    mlp_params(*it->second, host, to_host, grads);
    g_mlp_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_mlp_set_params(int handle, const float* host) {
  return mlp_copy(handle, const_cast<float*>(host), false, false, "ww_mlp_set_params");
}
int ww_mlp_get_params(int handle, float* host) {
  return mlp_copy(handle, host, true, false, "ww_mlp_get_params");
}
int ww_mlp_get_grads(int handle, float* host) {
  return mlp_copy(handle, host, true, true, "ww_mlp_get_grads");
}

int ww_mlp_train_step(int handle, int rows, const void* x, const float* t, int ldt, float lr,
                      float wd, int apply, float* loss3) {
  try {
    auto it = mlps().find(handle);
    if (it == mlps().end()) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_mlp_train_step: unknown handle");
    Mlp& m = *it->second;
    if (!x || !t || rows <= 0 || rows % 128 || rows > m.cap || ldt < m.nvalid || ldt % 4)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_train_step: bad shape");
    WWB_CHECK(cudaMemcpyAsync(m.x0.p, x, static_cast<size_t>(rows) * m.din * 2,
                              cudaMemcpyDeviceToDevice, m.st));
    m.loss.zero(m.st);
    // The weight gradients accumulate (split reductions add into them): start from zero, so
    // each call reports and applies one step's gradient.
    for (Layer& L : m.L) L.g.zero(m.st);
    Adam h{};
    if (apply) h = adam_at(++m.step, lr, wd);
    mlp_train_step(m, rows, t, ldt, nullptr, nullptr, LossWeights{0.0f, 0.0f, 0},
                   apply ? &h : nullptr, m.loss.p, m.st);
    if (loss3) WWB_CHECK(cudaMemcpyAsync(loss3, m.loss.p, 12, cudaMemcpyDeviceToHost, m.st));
    if (take_err(m)) return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, "ww_mlp_train_step: a GEMM wait gave up");
    g_mlp_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_mlp_forward(int handle, int rows, const void* x, float* out) {
  try {
    auto it = mlps().find(handle);
    if (it == mlps().end()) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_mlp_forward: unknown handle");
    Mlp& m = *it->second;
    if (!x || !out || rows <= 0) return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_forward: bad shape");
    mlp_infer_alloc(m, rows);
    WWB_CHECK(cudaMemcpyAsync(m.ix0.p, x, static_cast<size_t>(rows) * m.din * 2,
                              cudaMemcpyDeviceToDevice, m.st));
    mlp_forward_infer(m, rows, m.st);
    WWB_CHECK(cudaMemcpyAsync(out, m.iout.p, static_cast<size_t>(rows) * m.dout * 4,
                              cudaMemcpyDeviceToDevice, m.st));
    if (take_err(m)) return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, "ww_mlp_forward: a GEMM wait gave up");
    g_mlp_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_mlp_gemm(int mode, int M, int N, int K, int bn, int splits, const void* a, int lda,
                const void* b, int ldb, const float* bias, void* out, void* out_t, void* aux,
                float* out_f32, int ldo, int ldt, void* stream) {
  try {
    if (!runtime().ready) return g_mlp_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_mlp_gemm before ww_kokkos_init");
    static int* err = nullptr;
    if (!err) {
      WWB_CHECK(cudaMalloc(&err, sizeof(int)));
      WWB_CHECK(cudaMemset(err, 0, sizeof(int)));
    }
    const bool paired = (mode & 16) != 0;
    mode &= ~16;
    GemmArgs g{};
    g.pair = paired ? 1 : 0;
    g.M = M;
    g.N = N;
    g.K = K;
    g.bn = bn;
    g.splits = splits;
    g.bias = bias;
    g.out = static_cast<bf16*>(out);
    g.out_t = static_cast<bf16*>(out_t);
    g.aux = static_cast<bf16*>(aux);
    g.out_f32 = out_f32;
    g.ldo = ldo;
    g.ldt = ldt;
    g.err = err;
    if (!a || !b || lda % 8 || ldb % 8 || lda < K || ldb < K)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_gemm: operand strides");
    const bool needs_bias = mode == kEpiGeluTrain || mode == kEpiGeluInfer || mode == kEpiF32;
    const bool needs_out = mode == kEpiGeluTrain || mode == kEpiGeluInfer || mode == kEpiDGelu;
    const bool needs_f32 = mode == kEpiF32 || mode == kEpiAtomic;
    const bool needs_aux = mode == kEpiGeluTrain || mode == kEpiDGelu;
    if ((needs_bias && !bias) || (needs_out && !out) || (needs_f32 && !out_f32) ||
        (needs_aux && !aux) || mode < kEpiGeluTrain || mode > kEpiAtomic)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_gemm: missing operand for the epilogue");
    if (mode != kEpiAtomic && splits != 1)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_gemm: split reductions need the atomic epilogue");
    const Operand oa = make_operand(static_cast<const bf16*>(a), M, K, lda, kBM);
    if (paired && mode != kEpiGeluInfer && mode != kEpiF32)
      return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mlp_gemm: paired tiles for modes 2 and 3 only");
    const Operand ob = make_operand(static_cast<const bf16*>(b), N, K, ldb,
                                    bn > 0 ? gemm_b_box(g) : 64);
    const char* why = nullptr;
    if (!gemm_shape_ok(g, oa, ob, &why)) return g_mlp_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, why);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    gemm(mode, g, oa, ob, st);
    int v = 0;
    WWB_CHECK(cudaMemcpyAsync(&v, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    WWB_CHECK(cudaStreamSynchronize(st));
    if (v) {
      WWB_CHECK(cudaMemset(err, 0, sizeof(int)));
      return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, "ww_mlp_gemm: a wait gave up");
    }
    g_mlp_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_mlp_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_mlp_last_error(void) { return g_mlp_status.get(); }

// ------------------------------------------------------------------------------ ww_sur_*

int ww_sur_init(int igrid, int nhidden, unsigned long long seed) {
  try {
    if (!runtime().ready) return sur_fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_sur_init before ww_kokkos_init");
    auto s = std::make_unique<Sur>();
    if (!snl1_grid_dev(igrid, &s->dia) || !snl1_grid_config(igrid, &s->cfg, &s->sig))
      return sur_fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                      "ww_sur_init: grid needs ww_snl1_init with the row-shift tables first");
    if (nhidden <= 0 || nhidden % 64)
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_init: hidden width must be a positive multiple of 64");
    const int nk = s->cfg.nk, nth = s->cfg.nth, nspec = nk * nth;
    if (nk > 64 || nth > 64) return sur_fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_sur_init: NK or NTH above 64");
    const int din = (nspec + 2 + 63) / 64 * 64;
    const int dout = (nspec + 1 + 63) / 64 * 64;  // + the error head
    mlp_alloc(s->net, din, nhidden, dout, nspec, 8192, seed);
    s->rowscale.alloc(nk);
    set_rowscale(*s, std::vector<float>(nk, 1.0f));
    SurGrid& g = s->g;
    g.nk = nk;
    g.nth = nth;
    g.nspec = nspec;
    g.din = din;
    g.dout = dout;
    g.sig = s->dia.sig;
    g.rowscale = s->rowscale.p;
    g.snlc1 = s->cfg.snlc1;
    g.kdcon = s->cfg.kdcon;
    g.kdmn = s->cfg.kdmn;
    g.snls1 = s->cfg.snls1;
    g.snls2 = s->cfg.snls2;
    g.snls3 = s->cfg.snls3;
    g.dth = s->cfg.dth;
    g.xfr = s->cfg.xfr;
    build_f64(*s);
    surs()[igrid] = std::move(s);
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

int ww_sur_synth(int igrid, int npts, unsigned long long seed, float bimodal, float dmin,
                 float dmax, long long p0, float* a, float* cg, float* kdmean, void* stream) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (npts < 0 || (npts > 0 && (!a || !cg || !kdmean)) || !(dmin > 0) || dmax < dmin)
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_synth: bad arguments");
    synth(s->g, SynthDraw{seed, bimodal, dmin, dmax}, p0, npts, a, cg, kdmean,
          static_cast<cudaStream_t>(stream));
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_dataset(int igrid, long long npts, long long holdout, unsigned long long seed,
                   float bimodal, float dmin, float dmax) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (npts <= 0 || holdout < 0 || holdout >= npts || !(dmin > 0) || dmax < dmin)
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_dataset: bad arguments");
    const int nspec = s->g.nspec, nk = s->g.nk, din = s->net.din;
    cudaStream_t st = s->net.st;
    constexpr int kChunk = 65536;
    DBuf<float> a, cg, kd, so, dd;
    DBuf<int> sh;
    a.alloc(static_cast<size_t>(kChunk) * nspec);
    cg.alloc(static_cast<size_t>(kChunk) * nk);
    kd.alloc(kChunk);
    so.alloc(static_cast<size_t>(kChunk) * nspec);
    dd.alloc(static_cast<size_t>(kChunk) * nspec);
    sh.alloc(kChunk);
    s->xs.alloc(static_cast<size_t>(npts) * din);
    s->ts.alloc(static_cast<size_t>(npts) * nspec);
    s->pss.alloc(static_cast<size_t>(npts) * 2 * nk);
    const SynthDraw draw{seed, bimodal, dmin, dmax};
    for (long long p0 = 0; p0 < npts; p0 += kChunk) {
      const int n = static_cast<int>(std::min<long long>(kChunk, npts - p0));
      synth(s->g, draw, p0, n, a.p, cg.p, kd.p, st);
      launch_snl1(snl1_pair_ok(s->dia) ? kSnl1Pair : snl1_band_ok(s->dia) ? kSnl1Band : kSnl1Gather,
                  s->dia, n, a.p, cg.p, kd.p,
                  so.p, dd.p, st);
      float* const psc = s->pss.p + static_cast<size_t>(p0) * 2 * nk;
      prep(s->g, n, a.p, cg.p, kd.p, s->xs.p + static_cast<size_t>(p0) * din, din, psc, sh.p, st);
      if (p0 == 0) {  // the target scale per frequency row, from the first chunk
        DBuf<double> acc;
        DBuf<unsigned long long> cnt;
        acc.alloc(nk);
        cnt.alloc(1);
        acc.zero(st);
        cnt.zero(st);
        rowscale_acc(s->g, n, so.p, psc, acc.p, cnt.p, st);
        std::vector<double> h(nk);
        unsigned long long c = 0;
        WWB_CHECK(cudaMemcpyAsync(h.data(), acc.p, nk * 8, cudaMemcpyDeviceToHost, st));
        WWB_CHECK(cudaMemcpyAsync(&c, cnt.p, 8, cudaMemcpyDeviceToHost, st));
        WWB_CHECK(cudaStreamSynchronize(st));
        std::vector<float> rs(nk, 1.0f);
        double mx = 0;
        for (int k = 0; k < nk; ++k) {
          const double r = c ? std::sqrt(h[k] / (static_cast<double>(c) * s->g.nth)) : 1.0;
          rs[k] = static_cast<float>(r);
          mx = std::max(mx, r);
        }
        for (int k = 0; k < nk; ++k)
          if (!(rs[k] > 1e-6 * mx)) rs[k] = static_cast<float>(mx > 0 ? 1e-6 * mx : 1.0);
        set_rowscale(*s, rs);
      }
      targets(s->g, n, so.p, psc, sh.p, s->ts.p + static_cast<size_t>(p0) * nspec, nspec, st);
    }
    WWB_CHECK(cudaStreamSynchronize(st));
    if (snl1_take_error() != 0) return sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_sur_dataset: a DIA wait gave up");
    s->n_data = npts;
    s->n_train = npts - holdout;
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_loss_weights(int igrid, float mu, float lambda) {
  Sur* s = find_sur(igrid);
  if (!s) return g_sur_status.get();
  if (!(mu >= 0) || !(lambda >= 0)) return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_loss_weights: negative weight");
  s->lw.mu = mu;
  s->lw.lambda = lambda;
  s->lw.head = 1;
  g_sur_status.ok();
  return WW_KOKKOS_OK;
}

int ww_sur_train(int igrid, int steps, int batch, float lr, float lr_end, float wd,
                 unsigned long long seed, float* losses) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    Mlp& m = s->net;
    if (s->n_train <= 0) return sur_fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_sur_train before ww_sur_dataset");
    if (steps < 0 || batch <= 0 || batch % 128 || batch > m.cap || !(lr > 0))
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_train: batch must be a multiple of 128 up to 8192");
    cudaStream_t st = m.st;
    if (!s->ts.p) return sur_fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_sur_train: no dataset");
    m.tb.alloc(static_cast<size_t>(m.cap) * s->g.nspec);
    s->tb_ps.alloc(static_cast<size_t>(m.cap) * 2 * s->g.nk);
    DBuf<float> hist;
    hist.alloc(static_cast<size_t>(std::max(steps, 1)) * 3);
    hist.zero(st);
    const int warm = std::min(200, std::max(1, steps / 20));
    for (int i = 0; i < steps; ++i) {
      // Warm-up, then cosine decay from lr to lr_end.
      double rate = lr;
      if (i < warm) rate = lr * (i + 1) / warm;
      else {
        const double f = static_cast<double>(i - warm) / std::max(1, steps - warm);
        rate = lr_end + 0.5 * (lr - lr_end) * (1.0 + std::cos(3.141592653589793 * f));
      }
      const uint64_t draw = (seed ^ 0x5DEECE66Dull) * 6364136223846793005ull + static_cast<uint64_t>(i) + 1;
      gather_batch(batch, s->n_train, draw | 1ull, 0, s->xs.p, m.din, s->ts.p, s->g.nspec,
                   s->pss.p, 2 * s->g.nk, m.x0.p, m.tb.p, s->tb_ps.p, st);
      const Adam h = adam_at(++m.step, static_cast<float>(rate), wd);
      mlp_train_step(m, batch, m.tb.p, s->g.nspec, &s->g, s->tb_ps.p, s->lw, &h,
                     hist.p + static_cast<size_t>(i) * 3, st);
    }
    if (losses && steps > 0)
      WWB_CHECK(cudaMemcpyAsync(losses, hist.p, static_cast<size_t>(steps) * 12, cudaMemcpyDeviceToHost, st));
    if (take_err(m)) return sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_sur_train: a GEMM wait gave up");
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_eval(int igrid, long long p0, int npts, float* loss3) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    Mlp& m = s->net;
    if (p0 < 0 || npts <= 0 || p0 + npts > s->n_data || !loss3)
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_eval: rows outside the dataset");
    cudaStream_t st = m.st;
    mlp_infer_alloc(m, std::min(npts, kInferRows));
    DBuf<float> acc;
    acc.alloc(3);
    double tot[3] = {0, 0, 0};
    for (long long q = 0; q < npts; q += kInferRows) {
      const int n = static_cast<int>(std::min<long long>(kInferRows, npts - q));
      acc.zero(st);
      WWB_CHECK(cudaMemcpyAsync(m.ix0.p, s->xs.p + static_cast<size_t>(p0 + q) * m.din,
                                static_cast<size_t>(n) * m.din * 2, cudaMemcpyDeviceToDevice, st));
      mlp_forward_infer(m, n, st);
      // The loss kernel's gradient output is scratch here (the inference input buffer's rows).
      DBuf<bf16> gs;
      gs.alloc(static_cast<size_t>(n) * m.dout);
      LossWeights lw = s->lw;
      loss_grad(s->g, lw, n, s->g.nspec, m.iout.p, m.dout,
                s->ts.p + static_cast<size_t>(p0 + q) * s->g.nspec, s->g.nspec,
                s->pss.p + static_cast<size_t>(p0 + q) * 2 * s->g.nk, gs.p, m.dout, acc.p, st);
      float h[3];
      WWB_CHECK(cudaMemcpyAsync(h, acc.p, 12, cudaMemcpyDeviceToHost, st));
      WWB_CHECK(cudaStreamSynchronize(st));
      // The loss kernel averages over its n rows; weight each chunk by its rows.
      for (int j = 0; j < 3; ++j) tot[j] += static_cast<double>(h[j]) * n;
    }
    for (int j = 0; j < 3; ++j) loss3[j] = static_cast<float>(tot[j] / npts);
    if (take_err(m)) return sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_sur_eval: a GEMM wait gave up");
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_gate(int igrid, float energy, float log_err) {
  Sur* s = find_sur(igrid);
  if (!s) return g_sur_status.get();
  if (!(energy >= 0)) return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_gate: negative threshold");
  s->gate.energy = energy;
  s->gate.log_err = log_err;
  g_sur_status.ok();
  return WW_KOKKOS_OK;
}

void ww_snl1_gated(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                   float* s, float* d, int* accepted, void* stream) {
  try {
    Sur* sp = find_sur(igrid);
    if (!sp) return;
    if (npts < 0) {
      sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gated: npts is negative");
      return;
    }
    if (npts == 0) {
      g_sur_status.ok();
      return;
    }
    if (!a || !cg || !kdmean || !s || !d) {
      sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gated: null array pointer");
      return;
    }
    sur_apply(*sp, npts, a, cg, kdmean, s, d, accepted, sp->gate, static_cast<cudaStream_t>(stream),
              true);
    g_sur_status.ok();
  } catch (const std::exception& e) {
    sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_snl1_gated_host(int igrid, int npts, const float* a, const float* cg,
                        const float* kdmean, float* s, float* d) {
  try {
    Sur* sp = find_sur(igrid);
    if (!sp) return;
    if (npts < 0) {
      sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gated_host: npts is negative");
      return;
    }
    if (npts == 0) {
      g_sur_status.ok();
      return;
    }
    if (!a || !cg || !kdmean || !s || !d) {
      sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gated_host: null array pointer");
      return;
    }
    Sur& S = *sp;
    auto& P = S.pipe;
    const size_t nspec = S.g.nspec, nk = S.g.nk;
    if (!P.ready) {
      WWB_CHECK(cudaStreamCreateWithFlags(&P.in, cudaStreamNonBlocking));
      WWB_CHECK(cudaStreamCreateWithFlags(&P.comp, cudaStreamNonBlocking));
      WWB_CHECK(cudaStreamCreateWithFlags(&P.out, cudaStreamNonBlocking));
      for (int k = 0; k < Sur::Pipe::kSlots; ++k) {
        WWB_CHECK(cudaEventCreateWithFlags(&P.copied[k], cudaEventDisableTiming));
        WWB_CHECK(cudaEventCreateWithFlags(&P.computed[k], cudaEventDisableTiming));
        WWB_CHECK(cudaEventCreateWithFlags(&P.drained[k], cudaEventDisableTiming));
        P.a[k].alloc(kInferRows * nspec);
        P.cg[k].alloc(kInferRows * nk);
        P.kd[k].alloc(kInferRows);
        P.s[k].alloc(kInferRows * nspec);
        P.d[k].alloc(kInferRows * nspec);
        P.dc[k].alloc(static_cast<size_t>(Sur::Pipe::kDRows) * nspec);
        P.dl[k].alloc(Sur::Pipe::kDRows);
        P.dn[k].alloc(1);
        WWB_CHECK(cudaHostAlloc(&P.h_dc[k], sizeof(float) * Sur::Pipe::kDRows * nspec,
                                cudaHostAllocDefault));
        WWB_CHECK(cudaHostAlloc(&P.h_dl[k], sizeof(int) * Sur::Pipe::kDRows, cudaHostAllocDefault));
        WWB_CHECK(cudaHostAlloc(&P.h_dn[k], sizeof(int), cudaHostAllocDefault));
      }
      P.ready = true;
    }
    timers::Region t_call("snl1.gated.call");
    // D is zero for the accepted points (the surrogate does not model the diagonal term): host
    // threads clear the caller's D while the device works, and only the rejected points' rows
    // cross the bus, packed on the device (at most kDRows a chunk; a chunk with more brings its
    // whole D). S crosses whole.
    const size_t dbytes = static_cast<size_t>(npts) * nspec * sizeof(float);
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthr = static_cast<int>(std::max(1u, std::min(16u, hw == 0 ? 4u : hw)));
    std::vector<std::thread> zeroers;
    try {
      for (int t = 0; t < nthr; ++t) {
        const size_t b0 = dbytes * t / nthr, b1 = dbytes * (t + 1) / nthr;
        zeroers.emplace_back([=] { std::memset(reinterpret_cast<char*>(d) + b0, 0, b1 - b0); });
      }
    } catch (...) {  // a thread that could not start: the started ones finish first
      for (auto& th : zeroers) th.join();
      throw;
    }
    bool zeroed = false;
    auto join_zeroers = [&] {
      if (zeroed) return;
      for (auto& th : zeroers) th.join();
      zeroed = true;
    };
    // The rejected rows of chunk cc (slot k) into the caller's D, once its copies are done.
    auto place_d = [&](int cc, int k) {
      WWB_CHECK(cudaEventSynchronize(P.drained[k]));
      join_zeroers();
      const size_t p0 = static_cast<size_t>(cc) * kInferRows;
      const size_t n = std::min(static_cast<size_t>(kInferRows), static_cast<size_t>(npts) - p0);
      const int cnt = *P.h_dn[k];
      if (cnt <= Sur::Pipe::kDRows) {
        for (int i = 0; i < cnt; ++i)
          std::memcpy(d + (p0 + static_cast<size_t>(P.h_dl[k][i])) * nspec,
                      P.h_dc[k] + static_cast<size_t>(i) * nspec, nspec * sizeof(float));
      } else {
        WWB_CHECK(cudaMemcpy(d + p0 * nspec, P.d[k].p, n * nspec * sizeof(float),
                             cudaMemcpyDeviceToHost));
      }
    };
    // Chunk c: copy in on `in`, compute on `comp`, copy out on `out`, slot c % 3; a slot is
    // refilled only after its previous chunk's results left and its D rows were placed.
    int c = 0;
    int placed = 0;  // chunks whose D rows are in the caller's D
    try {
      for (int p0 = 0; p0 < npts; p0 += kInferRows, ++c) {
        const int k = c % Sur::Pipe::kSlots;
        if (c >= Sur::Pipe::kSlots) place_d(placed++, k);
        const size_t n = static_cast<size_t>(std::min(kInferRows, npts - p0));
        WWB_CHECK(cudaStreamWaitEvent(P.in, P.drained[k], 0));
        WWB_CHECK(cudaMemcpyAsync(P.a[k].p, a + p0 * nspec, n * nspec * 4, cudaMemcpyHostToDevice, P.in));
        WWB_CHECK(cudaMemcpyAsync(P.cg[k].p, cg + p0 * nk, n * nk * 4, cudaMemcpyHostToDevice, P.in));
        WWB_CHECK(cudaMemcpyAsync(P.kd[k].p, kdmean + p0, n * 4, cudaMemcpyHostToDevice, P.in));
        WWB_CHECK(cudaEventRecord(P.copied[k], P.in));
        WWB_CHECK(cudaStreamWaitEvent(P.comp, P.copied[k], 0));
        sur_apply(S, static_cast<int>(n), P.a[k].p, P.cg[k].p, P.kd[k].p, P.s[k].p, P.d[k].p,
                  nullptr, S.gate, P.comp, true, c == 0);
        gather_listed_rows(S.nrej.p, S.rej_all.p, Sur::Pipe::kDRows, static_cast<int>(nspec),
                           P.d[k].p, P.dc[k].p, P.dl[k].p, P.dn[k].p, P.comp);
        WWB_CHECK(cudaEventRecord(P.computed[k], P.comp));
        WWB_CHECK(cudaStreamWaitEvent(P.out, P.computed[k], 0));
        WWB_CHECK(cudaMemcpyAsync(s + p0 * nspec, P.s[k].p, n * nspec * 4, cudaMemcpyDeviceToHost, P.out));
        WWB_CHECK(cudaMemcpyAsync(P.h_dn[k], P.dn[k].p, sizeof(int), cudaMemcpyDeviceToHost, P.out));
        WWB_CHECK(cudaMemcpyAsync(P.h_dl[k], P.dl[k].p, sizeof(int) * Sur::Pipe::kDRows,
                                  cudaMemcpyDeviceToHost, P.out));
        WWB_CHECK(cudaMemcpyAsync(P.h_dc[k], P.dc[k].p,
                                  sizeof(float) * Sur::Pipe::kDRows * nspec,
                                  cudaMemcpyDeviceToHost, P.out));
        WWB_CHECK(cudaEventRecord(P.drained[k], P.out));
      }
      for (; placed < c; ++placed) place_d(placed, placed % Sur::Pipe::kSlots);
    } catch (...) {
      join_zeroers();
      throw;
    }
    WWB_CHECK(cudaStreamSynchronize(P.out));
    WWB_CHECK(cudaStreamSynchronize(P.comp));
    if (take_err(S.net)) {
      sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1_gated_host: a GEMM wait gave up");
      return;
    }
    if (snl1_take_error() != 0) {
      sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1_gated_host: a DIA wait gave up");
      return;
    }
    g_sur_status.ok();
  } catch (const std::exception& e) {
    sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_fallback_count(int igrid, void* stream) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return -1;
    if (!s->nrej_total.p) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int v = 0;
    WWB_CHECK(cudaMemcpyAsync(&v, s->nrej_total.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    WWB_CHECK(cudaStreamSynchronize(st));
    if (take_err(s->net)) {
      sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1_gated: a GEMM wait gave up");
      return -1;
    }
    if (snl1_take_error() != 0) {
      sur_fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1_gated: a DIA wait gave up");
      return -1;
    }
    return v;
  } catch (const std::exception& e) {
    sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
    return -1;
  }
}

int ww_sur_forward(int igrid, int rows, const void* x, float* out, void* stream) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (rows <= 0 || !x || !out) return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_forward: bad arguments");
    mlp_infer_alloc(s->net, rows);
    mlp_forward_infer(s->net, rows, static_cast<cudaStream_t>(stream), static_cast<const bf16*>(x),
                      out);
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_judge(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                 const float* s_cand, double* stats, double* s64, double* d64, void* stream) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (!s->f64_ok) return sur_fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_sur_judge: no FP64 tables for this grid");
    if (npts < 0 || (npts > 0 && (!a || !cg || !kdmean || !stats)))
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_judge: bad arguments");
    dia_f64_judge(s->f64, npts, a, cg, kdmean, s_cand, stats, s64, d64,
                  static_cast<cudaStream_t>(stream));
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_calibrate(int igrid, int npts, unsigned long long seed, float bimodal, float dmin,
                     float dmax, float energy, float target_err, float* out) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (!s->f64_ok) return sur_fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_sur_calibrate: no FP64 tables");
    if (npts <= 0 || !(target_err > 0) || !(energy >= 0) || !out)
      return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_calibrate: bad arguments");
    const int nspec = s->g.nspec, nk = s->g.nk;
    cudaStream_t st = s->net.st;
    DBuf<float> a, cg, kd, so, dd;
    DBuf<double> stats;
    DBuf<int> acc;
    a.alloc(static_cast<size_t>(npts) * nspec);
    cg.alloc(static_cast<size_t>(npts) * nk);
    kd.alloc(npts);
    so.alloc(static_cast<size_t>(npts) * nspec);
    dd.alloc(static_cast<size_t>(npts) * nspec);
    stats.alloc(static_cast<size_t>(npts) * 10);
    acc.alloc(npts);
    synth(s->g, SynthDraw{seed, bimodal, dmin, dmax}, 0, npts, a.p, cg.p, kd.p, st);
    // Every point through the network (no gate, no fallback), then its head and error.
    std::vector<float> head(npts), res(npts);
    const GateParams open{1e30f, 1e30f};
    std::vector<double> st_h(static_cast<size_t>(npts) * 10);
    for (int p0 = 0; p0 < npts; p0 += kInferRows) {
      const int n = std::min(kInferRows, npts - p0);
      sur_scratch(*s, n);
      sur_chunk_out(*s, n, a.p + static_cast<size_t>(p0) * nspec,
                    cg.p + static_cast<size_t>(p0) * nk, kd.p + p0,
                    so.p + static_cast<size_t>(p0) * nspec, dd.p + static_cast<size_t>(p0) * nspec,
                    nullptr, s->gv.p, open, nullptr, st);
      // The gate's two inputs per point: the head (column NSPEC) and the energy residual.
      std::vector<float> gv(static_cast<size_t>(n) * 2);
      WWB_CHECK(cudaMemcpyAsync(gv.data(), s->gv.p, gv.size() * 4, cudaMemcpyDeviceToHost, st));
      WWB_CHECK(cudaStreamSynchronize(st));
      for (int i = 0; i < n; ++i) {
        head[p0 + i] = gv[2 * i];
        res[p0 + i] = gv[2 * i + 1];
      }
    }
    dia_f64_judge(s->f64, npts, a.p, cg.p, kd.p, so.p, stats.p, nullptr, nullptr, st);
    WWB_CHECK(cudaMemcpyAsync(st_h.data(), stats.p, st_h.size() * 8, cudaMemcpyDeviceToHost, st));
    WWB_CHECK(cudaStreamSynchronize(st));
    // Points the energy test passes, in order of predicted error; accept the longest prefix
    // whose summed band Hs-tendency error stays within target_err per point of the whole set
    // (a rejected point is computed by the plain DIA, whose error is counted as zero).
    std::vector<int> order;
    for (int i = 0; i < npts; ++i)
      if (res[i] <= energy) order.push_back(i);
    std::sort(order.begin(), order.end(), [&](int x, int y) { return head[x] < head[y]; });
    // The error of a point: the band-resolved Hs-tendency error, sum over frequency bands of
    // |band tendency - FP64 band tendency| over sum of |FP64 band tendency|.
    auto err_of = [&](int i) {
      const double* o = st_h.data() + static_cast<size_t>(i) * 10;
      return o[5] > 0 ? o[4] / o[5] : 0.0;
    };
    double sum = 0;
    int take = 0;
    for (size_t j = 0; j < order.size(); ++j) {
      const double e = err_of(order[j]);
      if ((sum + e) > target_err * npts) break;
      sum += e;
      take = static_cast<int>(j + 1);
    }
    float thr = -1e30f;
    if (take > 0) {
      thr = head[order[take - 1]];
      // ties: a threshold equal to the next head would take it too; step just below it.
      if (take < static_cast<int>(order.size()) && head[order[take]] == thr) thr = std::nextafter(thr, -1e30f);
    }
    s->gate.energy = energy;
    s->gate.log_err = thr;
    double all = 0;
    for (int i = 0; i < npts; ++i) all += err_of(i);
    out[0] = thr;
    out[1] = static_cast<float>(take) / npts;
    out[2] = static_cast<float>(sum / npts);
    out[3] = static_cast<float>(all / npts);
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

long long ww_sur_param_count(int igrid) {
  auto it = surs().find(igrid);
  return it == surs().end() ? -1 : static_cast<long long>(mlp_param_count(it->second->net)) + it->second->cfg.nk;
}

int ww_sur_get_params(int igrid, float* host) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (!host) return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_get_params: null");
    mlp_params(s->net, host, true, false);
    WWB_CHECK(cudaMemcpy(host + mlp_param_count(s->net), s->rowscale.p, s->cfg.nk * 4, cudaMemcpyDeviceToHost));
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_set_params(int igrid, const float* host) {
  try {
    Sur* s = find_sur(igrid);
    if (!s) return g_sur_status.get();
    if (!host) return sur_fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sur_set_params: null");
    mlp_params(s->net, const_cast<float*>(host), false, false);
    const float* rs = host + mlp_param_count(s->net);
    set_rowscale(*s, std::vector<float>(rs, rs + s->cfg.nk));
    g_sur_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return sur_fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_sur_last_error(void) { return g_sur_status.get(); }

}  // extern "C"
