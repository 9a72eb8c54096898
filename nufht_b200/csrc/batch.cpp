// Many independent transforms in one CUDA-graph launch (no counterpart in the reference,
// which transforms one problem per call).
//
// The items' device plans run their usual kernel sequences, captured once into a graph whose
// branches execute concurrently: items are grouped by plan (a plan's workspace serves one
// transform at a time), and the groups are dealt to the branches longest first, each to the
// branch with the least estimated work so far.  With branches = 0 the branch count is tuned
// at creation by timing the graph for 1, 2, 4, ... 32 branches on the items' own buffers.
//
// The graph records each plan's workspace pointers and cuFFT plans.  So the batch holds a
// reference to every plan (a plan outlives its handle while a batch uses it) and pins it:
// while pinned, a standalone run that needs a larger workspace gets new buffers and the old
// ones stay allocated for the graph; cuFFT plans are kept per batch width and never remade.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "capi_internal.h"
#include "executor.h"
#include "nufht_b200.h"

using hankel::DevicePlan;

struct NufhtB200Batch {
  int device = 0;
  std::vector<NufhtB200BatchItem> items;
  std::vector<std::shared_ptr<DevicePlan>> item_plan;  // plan of each item
  std::vector<std::shared_ptr<DevicePlan>> plans;      // distinct plans of the items, pinned
  int branches = 0;
  long kernel_nodes = 0;
  float tuned_ms = 0.0f;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cudaStream_t> streams;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;

  void release_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~NufhtB200Batch() {
    release_graph();
    for (auto& D : plans) {
      std::lock_guard<std::mutex> lk(D->mu);
      D->unpin();
    }
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
  }
};

namespace {

// Estimated device work of one item (multiply-adds; Bessel evaluations weighted as ~16).
double item_cost(const DevicePlan& D, const NufhtB200BatchItem& it) {
  double st[12];
  hankel::plan_stats(D, st, 12);
  const double B = it.batch;
  return B * st[10] * (st[3] + st[4]) + B * st[10] * st[9] / 4.0 + (16.0 + B) * st[5] +
         B * st[11] * (st[6] + st[7]);
}

int ensure_streams(NufhtB200Batch* b, int n) {
  while ((int)b->streams.size() < n) {
    cudaStream_t s;
    cudaEvent_t e;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return NUFHT_E_CUDA;
    b->streams.push_back(s);
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return NUFHT_E_CUDA;
    b->joins.push_back(e);
  }
  if (!b->fork && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    return NUFHT_E_CUDA;
  return 0;
}

// Capture all items into a graph with `nb` concurrent branches.
int capture(NufhtB200Batch* b, int nb) {
  b->release_graph();
  int rc = ensure_streams(b, nb);
  if (rc) return rc;
  // group items by plan, costliest group first, each to the least loaded branch
  std::map<DevicePlan*, std::vector<int>> groups;
  std::map<DevicePlan*, double> gcost;
  for (int i = 0; i < (int)b->items.size(); ++i) {
    DevicePlan* D = b->item_plan[i].get();
    groups[D].push_back(i);
    gcost[D] += item_cost(*D, b->items[i]);
  }
  std::vector<DevicePlan*> order;
  for (auto& kv : groups) order.push_back(kv.first);
  std::sort(order.begin(), order.end(), [&](DevicePlan* a, DevicePlan* c) { return gcost[a] > gcost[c]; });
  std::vector<double> load(nb, 0.0);
  std::vector<std::vector<int>> lanes(nb);
  for (DevicePlan* D : order) {
    int br = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[br] += gcost[D];
    for (int i : groups[D]) lanes[br].push_back(i);
  }
  const bool timing = hankel::g_phase_timing.exchange(false);
  cudaStream_t s0 = b->streams[0];
  rc = 0;
  if (cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    hankel::g_phase_timing.store(timing);
    return NUFHT_E_CUDA;
  }
  if (cudaEventRecord(b->fork, s0) != cudaSuccess) rc = NUFHT_E_CUDA;
  for (int br = 1; br < nb && !rc; ++br)
    if (cudaStreamWaitEvent(b->streams[br], b->fork, 0) != cudaSuccess) rc = NUFHT_E_CUDA;
  for (int br = 0; br < nb && !rc; ++br) {
    for (int i : lanes[br]) {
      const NufhtB200BatchItem& it = b->items[i];
      DevicePlan* D = b->item_plan[i].get();
      std::lock_guard<std::mutex> lk(D->mu);
      rc = D->run(it.cs, it.ld_cs, it.gs, it.ld_gs, it.batch, b->streams[br], true);
      if (rc) break;
    }
  }
  for (int br = 1; br < nb; ++br) {
    if (cudaEventRecord(b->joins[br], b->streams[br]) != cudaSuccess && !rc) rc = NUFHT_E_CUDA;
    if (cudaStreamWaitEvent(s0, b->joins[br], 0) != cudaSuccess && !rc) rc = NUFHT_E_CUDA;
  }
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(s0, &g);
  hankel::g_phase_timing.store(timing);
  if (rc || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc ? rc : NUFHT_E_CUDA;
  }
  b->graph = g;
  if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
    b->release_graph();
    return NUFHT_E_CUDA;
  }
  b->branches = nb;
  size_t nn = 0;
  cudaGraphGetNodes(b->graph, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) cudaGraphGetNodes(b->graph, nodes.data(), &nn);
  b->kernel_nodes = 0;
  for (cudaGraphNode_t node : nodes) {
    cudaGraphNodeType ty;
    if (cudaGraphNodeGetType(node, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++b->kernel_nodes;
  }
  return 0;
}

// Device time of one graph launch (median of 3, after one warm launch).
int time_graph(NufhtB200Batch* b, float* ms) {
  cudaStream_t s = b->streams[0];
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return NUFHT_E_CUDA;
  std::vector<float> t;
  int rc = 0;
  for (int r = 0; r < 4 && !rc; ++r) {
    if (cudaEventRecord(e0, s) != cudaSuccess || cudaGraphLaunch(b->exec, s) != cudaSuccess ||
        cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      rc = NUFHT_E_CUDA;
      break;
    }
    float v = 0.0f;
    cudaEventElapsedTime(&v, e0, e1);
    if (r > 0) t.push_back(v);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return 0;
}

}  // namespace

extern "C" {

int nufht_b200_batch_create(NufhtB200Batch** out, const NufhtB200BatchItem* items, int count, int branches) {
  if (!out) return -200;
  *out = nullptr;
  if (!items || count <= 0 || branches < 0) return -400;
  int device = -1;
  for (int i = 0; i < count; ++i) {
    const NufhtB200BatchItem& it = items[i];
    if (!it.plan || !it.cs || !it.gs || it.batch <= 0) return -400;
    const DevicePlan* D = it.plan->dp.get();
    if (it.ld_cs < D->m || it.ld_gs < D->n) return -401;
    if (device < 0) device = D->device;
    if (D->device != device) return -400;  // one GPU per batch
  }
  std::unique_ptr<NufhtB200Batch> b(new NufhtB200Batch);
  b->device = device;
  b->items.assign(items, items + count);
  for (const NufhtB200BatchItem& it : b->items) b->item_plan.push_back(it.plan->dp);
  if (cudaSetDevice(device) != cudaSuccess) return NUFHT_E_CUDA;
  int rc = ensure_streams(b.get(), 1);
  if (rc) return rc;
  // The warm-up below runs the plans on the batch's own stream: work the caller queued on
  // these plans elsewhere (any stream) must have finished, or the two would share a workspace.
  if (cudaDeviceSynchronize() != cudaSuccess) return NUFHT_E_CUDA;
  // One ordinary pass first, widest items first: sizes every workspace for its plan's widest
  // item, makes the FFT plans of every width and sets kernel attributes, so that nothing
  // allocates while the graph is captured (items that share a plan may differ in width).
  std::vector<int> warm(count);
  std::iota(warm.begin(), warm.end(), 0);
  std::stable_sort(warm.begin(), warm.end(),
                   [&](int a, int c) { return b->items[a].batch > b->items[c].batch; });
  for (int i : warm) {
    const NufhtB200BatchItem& it = b->items[i];
    DevicePlan* D = b->item_plan[i].get();
    std::lock_guard<std::mutex> lk(D->mu);
    if ((rc = D->run(it.cs, it.ld_cs, it.gs, it.ld_gs, it.batch, b->streams[0], true))) return rc;
  }
  if (cudaStreamSynchronize(b->streams[0]) != cudaSuccess) return NUFHT_E_CUDA;
  // Pin the plans before the first capture (the destructor unpins them).
  for (const std::shared_ptr<DevicePlan>& D : b->item_plan) {
    if (std::find(b->plans.begin(), b->plans.end(), D) != b->plans.end()) continue;
    std::lock_guard<std::mutex> lk(D->mu);
    D->pin();
    b->plans.push_back(D);
  }
  if (branches > 0) {
    if ((rc = capture(b.get(), std::min(branches, count)))) return rc;
  } else {
    int best = 1;
    float best_ms = 0.0f;
    for (int nb = 1; nb <= 32 && nb <= count; nb *= 2) {
      if ((rc = capture(b.get(), nb))) return rc;
      float ms = 0.0f;
      if ((rc = time_graph(b.get(), &ms))) return rc;
      if (nb == 1 || ms < best_ms) {
        best = nb;
        best_ms = ms;
      }
    }
    if ((rc = capture(b.get(), best))) return rc;
    b->tuned_ms = best_ms;
  }
  *out = b.release();
  return 0;
}

int nufht_b200_batch_launch(NufhtB200Batch* b, void* stream) {
  if (!b || !b->exec) return -400;
  if (cudaSetDevice(b->device) != cudaSuccess) return NUFHT_E_CUDA;
  if (cudaGraphLaunch(b->exec, (cudaStream_t)stream) != cudaSuccess) return NUFHT_E_CUDA;
  hankel::g_launch_counter.fetch_add(b->kernel_nodes, std::memory_order_relaxed);
  return 0;
}

int nufht_b200_batch_info(const NufhtB200Batch* b, int* branches, float* tuned_ms, long* kernel_nodes) {
  if (!b) return -400;
  if (branches) *branches = b->branches;
  if (tuned_ms) *tuned_ms = b->tuned_ms;
  if (kernel_nodes) *kernel_nodes = b->kernel_nodes;
  return 0;
}

void nufht_b200_batch_destroy(NufhtB200Batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  delete b;
}

int nufht_b200_plan_buffers(const NufhtDevicePlan* plan, const void** grid, int* retired, int* pins) {
  if (!plan) return -400;
  DevicePlan* D = plan->dp.get();
  std::lock_guard<std::mutex> lk(D->mu);
  if (grid) *grid = D->d_grid;
  if (retired) *retired = (int)D->retired.size();
  if (pins) *pins = D->pins;
  return 0;
}

}  // extern "C"
