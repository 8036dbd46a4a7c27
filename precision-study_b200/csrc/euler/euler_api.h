// euler_api.h -- device control block and launchers of the Euler sibling's
// kernels (euler_kernels.cu, compiled as namespaces exact and fast).
#ifndef PMHD_EULER_API_H
#define PMHD_EULER_API_H

#include <cuda_runtime.h>

namespace pmhd {
namespace euler {

// Time control of a 2D run, double-buffered by the launch parity p (t, step)
// and triple-buffered by the step count (max signal speeds along x and y, as
// ordered bit patterns of positive doubles).
struct EulerCtrl {
  double t[2];
  long long step[2];
  unsigned long long sx[3], sy[3];
  double t_end;  // compared with t in binary64 (t_end holds a value of the run's type unless wide_time)
  long long step_limit;
  int stop;       // the reference's "dt <= 0 or t + dt == t" exit was taken
  int wide_time;  // binary64 CFL and end-time arithmetic of the shock-bubble program (euler2d_cpu.cpp:165, :306)
  double cfl;     // the CFL number as binary64 (used when wide_time)
};

#define PMHD_EULER_DECLARE(NS)                                                                                      \
  namespace NS {                                                                                                    \
  cudaError_t prepare();                                                                                            \
  cudaError_t step2d(int fp32, int hll, const void* uin, void* uout, int nx, int ny, int pitch, long long plane,    \
                     double dx, double dy, double cfl, EulerCtrl* ctrl, int p, cudaStream_t s);                     \
  cudaError_t speed2d(int fp32, const void* u, int nx, int ny, int pitch, long long plane, EulerCtrl* ctrl,         \
                      int slot, cudaStream_t s);                                                                    \
  cudaError_t run1d(int fp32, int hll, void* u, void* f, int n, double t_end, long long max_iters, double* out_t,   \
                    long long* out_steps, int* err, cudaStream_t s);                                                \
  }
PMHD_EULER_DECLARE(exact)
PMHD_EULER_DECLARE(fast)
#undef PMHD_EULER_DECLARE

}  // namespace euler
}  // namespace pmhd

#endif
