// runner.cpp -- see runner.h.
#include "runner.h"

namespace pmhd {

cudaError_t Runner::enqueue_steps(int nsteps) const {
  const Batch& b = batch[choice.ty_idx];
  for (int n = 0; n < nsteps; n++) {
    const int p = n & 1;
    cudaError_t e = pre_step ? pre_step(p) : cudaSuccess;
    if (e != cudaSuccess) return e;
    if (hancock) {
      if (!single) return cudaErrorNotSupported;
      e = kt->hancock(precision, hlld, 0, *single, p, stream);
      if (e == cudaSuccess) e = kt->hancock(precision, hlld, 1, *single, p, stream);
    } else if (!parts.empty()) {
      for (int st = 1; st <= 2 && e == cudaSuccess; st++)
        for (size_t q = 0; q < parts.size() && e == cudaSuccess; q++)
          e = kt->stage(precision, hlld, st, parts[q].ty_idx, parts[q].batch, single, p, parts[q].grid, stream);
    } else {
      e = kt->stage(precision, hlld, 1, choice.ty_idx, b, single, p, choice.grid, stream);
      if (e == cudaSuccess) e = kt->stage(precision, hlld, 2, choice.ty_idx, b, single, p, choice.grid, stream);
    }
    if (e != cudaSuccess) return e;
    if (post_step) {
      e = post_step(p);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int Runner::graph(int nsteps, cudaGraphExec_t* out) {
  const int plan = parts.empty() ? -1 : plan_id_;
  for (auto& g : graphs_)
    if (g.steps == nsteps && g.ty_idx == choice.ty_idx && g.grid == choice.grid && g.plan == plan) {
      *out = g.exec;
      return 0;
    }
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
  cudaError_t e = enqueue_steps(nsteps);
  cudaError_t e2 = cudaStreamEndCapture(stream, &graph);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return -1;
  }
  Graph g{nsteps, choice.ty_idx, choice.grid, plan, nullptr};
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return -1;
  graphs_.push_back(g);
  *out = g.exec;
  return 0;
}

cudaError_t Runner::tune(int steps, TuneResult* res) {
  steps += steps & 1;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const LaunchChoice saved = choice;
  LaunchChoice best = saved;
  float best_ms = -1.f, default_ms = -1.f;
  int ncand = 0;
  cudaError_t err = cudaSuccess;
  for (int ty = 0; ty < kNumTileHeights && err == cudaSuccess; ty++) {
    const int occ = kt->ctas_per_sm(precision, hlld, ty, single == nullptr);
    for (int k = occ; k >= 1 && err == cudaSuccess; k--) {
      choice.ty_idx = ty;
      choice.grid = k == occ ? 0 : sms * k;
      cudaEventRecord(e0, stream);
      err = enqueue_steps(steps);
      cudaEventRecord(e1, stream);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)steps;
      ncand++;
      if (ty == 0 && k == occ) default_ms = ms;
      if (best_ms < 0.f || ms < best_ms) {
        best_ms = ms;
        best = choice;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  choice = err == cudaSuccess ? best : saved;
  if (res) {
    res->best = choice;
    res->candidates = ncand;
    res->best_ms_per_step = best_ms;
    res->default_ms_per_step = default_ms;
  }
  return err;
}

void Runner::release() {
  for (auto& g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

}  // namespace pmhd
