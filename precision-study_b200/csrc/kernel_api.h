// kernel_api.h -- host-side interface of the pmhd CUDA kernels.
//
// The kernels are compiled twice from the same source: once with IEEE
// arithmetic and floating-point contraction disabled (-fmad=false, table
// "exact", the bit-parity mode against the reference CPU build) and once for
// speed (table "fast": FMA contraction, and binary32 division and square
// root with the hardware's approximate instructions, at most 2 ulp; binary64
// arithmetic stays IEEE apart from contraction).  solver.cpp picks a table
// per handle.
#ifndef PMHD_KERNEL_API_H
#define PMHD_KERNEL_API_H

#include <cuda_runtime.h>

namespace pmhd {

struct Ctrl;

enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1, PREC_MIXED = 2 };

// Arguments of one stage launch; the input planes come in as a TMA tensor map.
struct StageArgs {
  const void* u_in;   // stage input planes (U in stage 1, U1 in stage 2)
  void* u_out;        // stage output planes (U1 in stage 1, U in stage 2)
  const void* u_old;  // stage 2: U^n (the same buffer as u_out, read per cell)
  Ctrl* ctrl;
  long long plane;    // elements per plane
  int nx, ny, pitch;
  int parity;         // step parity: Ctrl slot read by this launch
  int muscl;          // 1: MUSCL reconstruction, 0: first order
  int bc[4];          // x low, x high, y low, y high
  double gamma, tol, cfl, alpha, dx, dy;  // cfl, dx, dy exact in the time type
};

struct KernelTable {
  const char* name;
  // Sets dynamic shared-memory limits; call once per process and device.
  cudaError_t (*init)();
  // One SSPRK2 stage (1 or 2) over the whole grid.
  cudaError_t (*stage)(int precision, int hlld, int stage, const void* tmap_in, const StageArgs& a,
                       cudaStream_t s);
  // Max signal speed of the interior of `u` into ctrl->chbits[slot].
  cudaError_t (*speed)(int precision, const void* u, long long plane, int nx, int ny, int pitch, double gamma,
                       Ctrl* ctrl, int slot, cudaStream_t s);
  // Caller AoS buffer (device copy) <-> SoA planes with ghost cells.
  cudaError_t (*aos_to_soa)(int precision, const void* aos, int layout, void* u, long long plane, int nx, int ny,
                            int pitch, const int bc[4], cudaStream_t s);
  cudaError_t (*soa_to_aos)(int precision, const void* u, long long plane, int nx, int ny, int pitch, int layout,
                            void* aos, cudaStream_t s);
  // Tile shape of the stage kernel and its dynamic shared memory per CTA.
  void (*tile)(int precision, int* tx, int* ty, size_t* smem_bytes);
};

const KernelTable& kernel_table_exact();
const KernelTable& kernel_table_fast();

}  // namespace pmhd

#endif  // PMHD_KERNEL_API_H
