// solver_internal.h -- access to a pmhd_solver's device state for other
// parts of the library (the learned coarse-grid correction); not exported
// through include/pmhd.h.
#ifndef PMHD_SOLVER_INTERNAL_H
#define PMHD_SOLVER_INTERNAL_H

#include <cuda_runtime.h>

#include <functional>

#include "kernel_api.h"
#include "pmhd.h"

namespace pmhd {

struct SolverView {
  void* u = nullptr;   // SoA state: variable k, ghosted cell (gi, gj) at u[k*plane + gj*pitch + gi]
  void* u1 = nullptr;  // stage-1 buffer, same layout
  int pitch = 0;
  long long plane = 0;
  int nx = 0, ny = 0;
  double dx = 0, dy = 0, gamma = 0;
  int precision = 0;
  cudaStream_t stream = nullptr;
  Ctrl* ctrl = nullptr;
  const KernelTable* kt = nullptr;
};

bool solver_view(pmhd_solver* s, SolverView* v);

// Work enqueued before / after every step of the solver's graphs (argument:
// the step's parity); empty functions remove it.  Cached graphs are rebuilt.
void solver_set_step_hooks(pmhd_solver* s, std::function<cudaError_t(int)> pre,
                           std::function<cudaError_t(int)> post);

}  // namespace pmhd

#endif
