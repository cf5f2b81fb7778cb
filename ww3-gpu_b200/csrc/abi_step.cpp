// ww3-gpu_b200/csrc/abi_step.cpp
// ww_step_begin / ww_step_end / ww_step_run / ww_step_free: a whole time step on a grid's
// resident VA recorded once and replayed as one CUDA graph (see step.hpp).
//
// What W3WAVE does between two output times on a PR3 grid is, per time step, W3KTP3 on every
// sea point, W3XYP3 on every spectral component, W3KTP3 again and W3SRCE on every sea point
// (ww3-gpu kokkos/src/ww_kokkos/wave_w3wave.hpp:577-800 orders them; the fork calls the C
// entries ww_ktp3_batch_va, ww_xyp3_batch_va and ww_srce_batch_va one after another). Their
// host work (validation, derived maps, copies of the grid's arrays) depends only on the grid
// and the recorded arguments, so it is done once while recording; the replay is launches only.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "st4_srce.cuh"
#include "step.hpp"
#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {

struct StepRecorder {
  bool recording = false;
  std::vector<std::function<void(cudaStream_t)>> ops;
  std::vector<std::shared_ptr<void>> srce_jobs;  ///< per op: its W3SRCE job (SrceRecorded) or null
  std::vector<std::shared_ptr<void>> keep;
  cudaStream_t stage = nullptr;  ///< staging stream of the recorded calls
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nops = 0;
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void clear() {
    drop_graph();
    ops.clear();
    srce_jobs.clear();
    keep.clear();
    recording = false;
    nops = 0;
  }
  ~StepRecorder() {
    clear();
    if (stage) cudaStreamDestroy(stage);
  }
};

namespace {

Status g_step;

/// Tables replaced while a recorded step may still read them.
std::vector<void*>& retired() {
  static auto* v = new std::vector<void*>();
  return *v;
}

std::map<int, std::unique_ptr<StepRecorder>>& recs() {
  static auto* m = new std::map<int, std::unique_ptr<StepRecorder>>();
  return *m;
}

StepRecorder* find(int igrid) {
  auto it = recs().find(igrid);
  return it == recs().end() ? nullptr : it->second.get();
}

/// Several grids' recorded steps merged into one graph (ww_steps_fuse): every grid's calls
/// before its W3SRCE batch, one W3SRCE launch over all the grids' points, then the calls after.
struct FusedSteps {
  std::vector<int> grids;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  SrceJob* jobs = nullptr;  ///< device copy of the jobs
  SrceWork work;
  int total = 0;
  void clear() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (jobs) cudaFree(jobs);
    work.release();
    exec = nullptr;
    graph = nullptr;
    jobs = nullptr;
    grids.clear();
    total = 0;
  }
  ~FusedSteps() { clear(); }
};

FusedSteps& fused() {
  static auto* f = new FusedSteps();
  return *f;
}

/// A grid's recorded step changes or goes: a fused graph that holds it goes too.
void drop_fused_with(int igrid) {
  FusedSteps& f = fused();
  for (int g : f.grids)
    if (g == igrid) {
      f.clear();
      return;
    }
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    return g_step.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return g_step.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

}  // namespace

StepRecorder* step_recorder(int igrid) {
  StepRecorder* r = find(igrid);
  return (r && r->recording) ? r : nullptr;
}

void step_keep(StepRecorder* r, std::shared_ptr<void> obj) { r->keep.push_back(std::move(obj)); }

void step_add(StepRecorder* r, std::function<void(cudaStream_t)> op,
              std::shared_ptr<void> srce_job) {
  r->ops.push_back(std::move(op));
  r->srce_jobs.push_back(std::move(srce_job));
}

cudaStream_t step_stream(StepRecorder* r) { return r->stage; }

namespace {
bool any_step() {
  for (auto& kv : recs())
    if (kv.second && (kv.second->graph || kv.second->recording)) return true;
  return false;
}
void flush_retired() {
  for (void* p : retired()) cudaFree(p);
  retired().clear();
}
}  // namespace

void free_table(void* p) {
  if (p == nullptr) return;
  if (any_step()) {
    retired().push_back(p);
  } else {
    cudaFree(p);
  }
}

void release_steps() {
  fused().clear();
  recs().clear();
  flush_retired();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_step_begin(int igrid) {
  return guarded([&] {
    if (!runtime().ready) return g_step.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    auto& r = recs()[igrid];
    if (!r) r = std::make_unique<StepRecorder>();
    if (r->recording) return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_step_begin: already recording");
    // Recording again replaces the grid's step (and a fused graph that holds it).
    drop_fused_with(igrid);
    r->clear();
    if (!r->stage) WWB_CHECK(cudaStreamCreateWithFlags(&r->stage, cudaStreamNonBlocking));
    r->recording = true;
    g_step.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_step_end(int igrid) {
  return guarded([&] {
    StepRecorder* r = find(igrid);
    if (!r || !r->recording) return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_step_end: not recording");
    r->recording = false;
    cudaStream_t cap = nullptr;
    WWB_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    // Relaxed: the launchers look up occupancies and set function attributes, which are not
    // stream work; they allocate nothing here (the recorded calls reserved their buffers).
    WWB_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
    bool failed = false;
    try {
      for (auto& op : r->ops) op(cap);
    } catch (...) {
      failed = true;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (failed || e != cudaSuccess || g == nullptr) {
      if (g) cudaGraphDestroy(g);
      r->clear();
      return g_step.fail(WW_KOKKOS_ERR_KERNEL, "ww_step_end: the step's launches could not be captured");
    }
    r->graph = g;
    WWB_CHECK(cudaGraphInstantiate(&r->exec, r->graph, 0));
    r->nops = static_cast<int>(r->ops.size());
    g_step.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_step_run(int igrid, int nrep, void* stream) {
  return guarded([&] {
    StepRecorder* r = find(igrid);
    if (!r || r->recording || !r->exec)
      return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_step_run: no recorded step for this grid");
    if (nrep < 0) return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_step_run: nrep < 0");
    // The host may have written its VA since the last call (ww_va_host_write): upload first.
    if (nrep > 0)
      if (int rc = va_device_current(igrid); rc != WW_KOKKOS_OK)
        return g_step.fail(rc, "ww_step_run: the grid's VA could not be made current on the device");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : runtime().stream;
    for (int i = 0; i < nrep; ++i) WWB_CHECK(cudaGraphLaunch(r->exec, s));
    if (nrep > 0) va_device_written(igrid);
    if (!stream) WWB_CHECK(cudaStreamSynchronize(s));
    g_step.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_steps_run(const int* igrids, int ngrids, int nrep, void* stream) {
  return guarded([&] {
    if (igrids == nullptr || ngrids < 1 || nrep < 0)
      return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_run: bad grid list or nrep");
    std::vector<StepRecorder*> rs;
    for (int k = 0; k < ngrids; ++k) {
      for (int j = 0; j < k; ++j)
        if (igrids[j] == igrids[k])
          return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_run: a grid is listed twice");
      StepRecorder* r = find(igrids[k]);
      if (!r || r->recording || !r->exec)
        return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_run: a grid has no recorded step");
      rs.push_back(r);
    }
    // The grids' graphs one after another on one stream: a graph of all the grids' steps, as
    // branches side by side or chained, measured slower (the grids' persistent W3SRCE launches
    // compete for the same SMs when side by side).
    if (nrep > 0)
      for (int k = 0; k < ngrids; ++k)
        if (int rc = va_device_current(igrids[k]); rc != WW_KOKKOS_OK)
          return g_step.fail(rc, "ww_steps_run: a grid's VA could not be made current on the device");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : runtime().stream;
    const FusedSteps& f = fused();
    const bool use_fused =
        f.exec != nullptr && f.grids == std::vector<int>(igrids, igrids + ngrids);
    for (int i = 0; i < nrep; ++i) {
      if (use_fused) {
        WWB_CHECK(cudaGraphLaunch(f.exec, s));
      } else {
        for (StepRecorder* r : rs) WWB_CHECK(cudaGraphLaunch(r->exec, s));
      }
    }
    if (nrep > 0)
      for (int k = 0; k < ngrids; ++k) va_device_written(igrids[k]);
    if (!stream) WWB_CHECK(cudaStreamSynchronize(s));
    g_step.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_steps_fuse(const int* igrids, int ngrids) {
  return guarded([&] {
    FusedSteps& f = fused();
    f.clear();
    if (ngrids == 0) {
      g_step.ok();
      return static_cast<int>(WW_KOKKOS_OK);
    }
    if (igrids == nullptr || ngrids < 1)
      return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_fuse: bad grid list");
    std::vector<StepRecorder*> rs;
    std::vector<int> at;  // index of each grid's W3SRCE batch among its recorded calls
    std::vector<SrceJob> jobs;
    pt::SrceLayout L{};
    int total = 0;
    for (int k = 0; k < ngrids; ++k) {
      for (int j = 0; j < k; ++j)
        if (igrids[j] == igrids[k])
          return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_fuse: a grid is listed twice");
      StepRecorder* r = find(igrids[k]);
      if (!r || r->recording || !r->exec)
        return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_fuse: a grid has no recorded step");
      int idx = -1, count = 0;
      for (size_t i = 0; i < r->srce_jobs.size(); ++i)
        if (r->srce_jobs[i]) {
          idx = static_cast<int>(i);
          ++count;
        }
      if (count != 1)
        return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_steps_fuse: every grid's step needs exactly one W3SRCE batch");
      const auto* rec = static_cast<const SrceRecorded*>(r->srce_jobs[idx].get());
      if (k == 0) L = rec->L;
      if (std::memcmp(&L, &rec->L, sizeof L) != 0)
        return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_steps_fuse: the grids' W3SRCE working sets differ (spectral grid or ST4 tables)");
      SrceJob j = rec->job;
      j.first = total;
      if (static_cast<long long>(total) + j.npts > (1LL << 30))
        return g_step.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_steps_fuse: too many points");
      total += j.npts;
      jobs.push_back(j);
      rs.push_back(r);
      at.push_back(idx);
    }
    WWB_CHECK(cudaMalloc(&f.jobs, jobs.size() * sizeof(SrceJob)));
    WWB_CHECK(cudaMemcpy(f.jobs, jobs.data(), jobs.size() * sizeof(SrceJob), cudaMemcpyHostToDevice));
    srce_multi_reserve(L, total, f.work);
    f.total = total;
    cudaStream_t cap = nullptr;
    WWB_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    WWB_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
    bool failed = false;
    try {
      for (size_t k = 0; k < rs.size(); ++k)
        for (int i = 0; i < at[k]; ++i) rs[k]->ops[i](cap);
      launch_srce_multi(f.jobs, static_cast<int>(jobs.size()), total, L, f.work, cap);
      for (size_t k = 0; k < rs.size(); ++k)
        for (size_t i = at[k] + 1; i < rs[k]->ops.size(); ++i) rs[k]->ops[i](cap);
    } catch (...) {
      failed = true;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (failed || e != cudaSuccess || g == nullptr) {
      if (g) cudaGraphDestroy(g);
      f.clear();
      return g_step.fail(WW_KOKKOS_ERR_KERNEL, "ww_steps_fuse: the launches could not be captured");
    }
    f.graph = g;
    WWB_CHECK(cudaGraphInstantiate(&f.exec, f.graph, 0));
    f.grids.assign(igrids, igrids + ngrids);
    g_step.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_step_free(int igrid) {
  drop_fused_with(igrid);
  StepRecorder* r = find(igrid);
  if (r) r->clear();
  if (!any_step()) flush_retired();
  g_step.ok();
  return WW_KOKKOS_OK;
}

int ww_step_nodes(int igrid) {
  StepRecorder* r = find(igrid);
  if (!r || !r->graph) return -1;
  size_t n = 0;
  if (cudaGraphGetNodes(r->graph, nullptr, &n) != cudaSuccess) return -1;
  return static_cast<int>(n);
}

int ww_step_ops(int igrid) {
  StepRecorder* r = find(igrid);
  return r ? static_cast<int>(r->ops.size()) : -1;
}

}  // extern "C"
