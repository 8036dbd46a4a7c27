// kernel_api.h -- host-side interface of the pmhd CUDA kernels.
//
// The kernels are compiled twice from the same source: once with IEEE
// arithmetic and floating-point contraction disabled (-fmad=false, table
// "exact", the bit-parity mode against the reference CPU build) and once for
// speed (table "fast": FMA contraction, and binary32 division and square
// root with the hardware's approximate instructions, at most 2 ulp; binary64
// arithmetic stays IEEE apart from contraction).  solver.cpp, ensemble.cpp
// and noalloc.cu pick a table per run.
//
// A stage launch works on a *batch*: one or more independent grids
// ("members", each with its own size, gamma, boundaries, time step and
// control block) whose 32 x TY tiles form one work list walked by
// persistent CTAs.  A single solver is a batch of one member.
#ifndef PMHD_KERNEL_API_H
#define PMHD_KERNEL_API_H

#include <cuda.h>
#include <cuda_runtime.h>

namespace pmhd {

struct Ctrl;

enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1, PREC_MIXED = 2 };

// Tile heights compiled into the library (tile width is 32).  Index into
// Member::tm and the Batch tile tables; index 0 is the default.
#ifndef PMHD_TY0
#define PMHD_TY0 19
#endif
constexpr int kTileHeights[2] = {PMHD_TY0, 8};
constexpr int kNumTileHeights = 2;
// A batched stage launch hands its CTAs runs of this many consecutive tiles.
constexpr int kBatchRun = 16;

// One grid of a batch; lives in device memory (64-byte aligned for the TMA
// descriptors).
struct alignas(64) Member {
  CUtensorMap tm[kNumTileHeights][2];  // [tile height][U, U1]: stage-1 / stage-2 inputs
  void* u;            // U planes (stage-1 input, stage-2 output)
  void* u1;           // U1 planes (stage-1 output, stage-2 input)
  Ctrl* ctrl;         // this grid's control block
  long long plane;    // elements per plane
  int nx, ny, pitch;
  int muscl;          // 1: MUSCL reconstruction, 0: first order
  int bc[4];          // x low, x high, y low, y high
  double gamma, tol;
  double cfl, alpha, dx, dy;  // exact in the precision's time type
  double inv_dx, inv_dy;      // 1 / dx, 1 / dy divided in the precision's time type
};

// The work list of one tile height.
struct Batch {
  const Member* members;   // device array of nmembers
  const int* tile_member;  // device array: global tile -> member (nullptr: all tiles are member 0)
  const int* member_tile0; // device array: first global tile of each member (nullptr: 0)
  int nmembers;
  int ntiles;
};

struct KernelTable {
  const char* name;
  // Sets dynamic shared-memory limits; call once per process and device.
  cudaError_t (*init)();
  // One SSPRK2 stage (1 or 2) over every member of the batch.  `ty_idx`
  // selects the tile height (kTileHeights), `grid` the number of persistent
  // CTAs (<= 0: SM count x resident CTAs), `parity` the step's Ctrl slot.
  // `single` != nullptr: a one-grid batch whose member is passed by value
  // (host copy; only b.ntiles is used); nullptr: the members of `b`.
  cudaError_t (*stage)(int precision, int hlld, int stage, int ty_idx, const Batch& b, const Member* single,
                       int parity, int grid, cudaStream_t s);
  // Resident stage CTAs per SM of a kernel variant (from the occupancy API).
  int (*ctas_per_sm)(int precision, int hlld, int ty_idx, int batched);
  // Max signal speed of the interior of `u` into ctrl->chbits[slot].
  cudaError_t (*speed)(int precision, const void* u, long long plane, int nx, int ny, int pitch, double gamma,
                       Ctrl* ctrl, int slot, cudaStream_t s);
  // Caller AoS buffer (device copy) <-> SoA planes with ghost cells.
  cudaError_t (*aos_to_soa)(int precision, const void* aos, int layout, void* u, long long plane, int nx, int ny,
                            int pitch, const int bc[4], cudaStream_t s);
  cudaError_t (*soa_to_aos)(int precision, const void* u, long long plane, int nx, int ny, int pitch, int layout,
                            void* aos, cudaStream_t s);
  // Shared memory per CTA of the stage kernel with tile height kTileHeights[ty_idx].
  size_t (*stage_smem)(int precision, int ty_idx);
  // One MUSCL-Hancock step of a single grid: part 0 = the control prologue,
  // part 1 = the step (reads m.u for parity 0 / m.u1 for parity 1, writes
  // the other).  fp64 and fp32 only.
  cudaError_t (*hancock)(int precision, int hlld, int part, const Member& m, int parity, cudaStream_t s);
};

const KernelTable& kernel_table_exact();
const KernelTable& kernel_table_fast();

// Fills the TMA descriptors of a member whose u, u1, plane, nx, ny and pitch
// are set (member_setup.cpp).  Returns false if the driver entry point is
// missing or an encoding fails.
bool encode_member_tmaps(Member& m, size_t elem_bytes);

// Fills the time-type constants of a member from a configuration's physical
// values, rounding to binary32 first when `fp32` (the reference's Real).
void set_member_physics(Member& m, double x_min, double x_max, double y_min, double y_max, double gamma,
                        double tol, double cfl, double alpha, int muscl, const int bc[4], bool fp32);

}  // namespace pmhd

#endif  // PMHD_KERNEL_API_H
