// runner.h -- launch plans, CUDA-graph cache and the kernel-variant autotuner
// shared by the single-grid solver (solver.cpp) and the ensemble
// (ensemble.cpp).
#ifndef PMHD_RUNNER_H
#define PMHD_RUNNER_H

#include <cuda_runtime.h>

#include <functional>
#include <vector>

#include "kernel_api.h"

namespace pmhd {

// Which compiled stage-kernel variant runs and with how many persistent CTAs.
struct LaunchChoice {
  int ty_idx = 0;  // index into kTileHeights
  int grid = 0;    // persistent CTAs; 0 = SM count x resident CTAs
};

struct TuneResult {
  LaunchChoice best;
  int candidates = 0;
  float best_ms_per_step = 0.f;
  float default_ms_per_step = 0.f;  // the untuned choice (32 x 8, full occupancy)
};

// One work list of a multi-part launch plan (an ensemble whose size classes
// run different tile heights): its tile height, persistent CTAs and tiles.
struct LaunchPart {
  int ty_idx = 0;
  int grid = 0;  // 0 = SM count x resident CTAs
  Batch batch;
};

class Runner {
 public:
  const KernelTable* kt = nullptr;
  int precision = 0;
  int hlld = 1;
  cudaStream_t stream = nullptr;
  Batch batch[kNumTileHeights];
  const Member* single = nullptr;  // host copy of a one-grid batch's member, or nullptr
  LaunchChoice choice;
  // Multi-part plan: when non-empty, a step launches stage 1 of every part,
  // then stage 2 of every part (parts hold disjoint members), instead of one
  // launch per stage with `choice`.  Change it through set_parts().
  std::vector<LaunchPart> parts;
  void set_parts(const std::vector<LaunchPart>& p) {
    parts = p;
    plan_id_++;
  }
  int hancock = 0;  // MUSCL-Hancock steps (single grid) instead of SSPRK2 stages
  // Optional work enqueued before and after every step (argument: the
  // step's parity), captured into the graphs with the stage launches.
  std::function<cudaError_t(int)> pre_step, post_step;

  // Enqueues `nsteps` steps (two stage launches each, parity 0, 1, 0, ...).
  cudaError_t enqueue_steps(int nsteps) const;
  // Cached CUDA graph of `nsteps` steps for the current choice.
  int graph(int nsteps, cudaGraphExec_t* out);
  // Times every variant (tile height x CTAs per SM) on `steps` live steps
  // each (an even number), keeps the fastest in `choice`.  The variants
  // compute identical results, so the timed steps are ordinary steps of the
  // run.  Returns cudaSuccess or the first CUDA error.
  cudaError_t tune(int steps, TuneResult* res);
  void release();

 private:
  struct Graph {
    int steps, ty_idx, grid, plan;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs_;
  int plan_id_ = 0;
};

}  // namespace pmhd

#endif
