// common.cuh -- device-side definitions shared by the pmhd kernels.
//
// State layout in HBM (per solver handle): structure of arrays, one plane
// per conserved variable k = 0..8 (rho, mx, my, mz, E, Bx, By, Bz, psi).
// A plane holds (ny + 4) rows of `pitch` elements; interior cell (i, j)
// lives at row j + 2, column i + 2, and the two ghost layers on every side
// are written by the kernels themselves (no boundary-condition kernels).
// `pitch` is nx + 4 rounded up to 16 elements so every row and every plane
// starts on a 128-byte (fp64) / 64-byte (fp32) boundary, as TMA requires.
#ifndef PMHD_COMMON_CUH
#define PMHD_COMMON_CUH

#include <cstdint>
#include <cuda_runtime.h>

namespace pmhd {

constexpr int GHOST = 2;
constexpr int NVAR = 9;
constexpr int BAD_NONE = 0x7fffffff;

// Boundary kinds per side (x low, x high, y low, y high).
enum BcKind : int { BC_PERIODIC = 0, BC_REFLECT = 1, BC_TRANSMISSIVE = 2 };

// Device-resident control block.  Slots [2] are double-buffered by step
// parity: the kernels of step n read slot n&1 and write slot (n&1)^1, so no
// kernel ever reads a word that another block of the same launch writes.
struct Ctrl {
  double t[2];                  // simulation time before the step
  long long step[2];            // steps taken before the step
  unsigned long long chbits[2]; // bit pattern of max signal speed (>= 0)
  double t_end;                 // stop when !(t < t_end)
  long long step_limit;         // stop when step >= step_limit
  int halted;                   // set after a stage reported a bad cell
  int bad1, bad2;               // min flat index of an unusable cell per stage
  int err;                      // device-side error (bounded wait expired)
  long long bad_step;           // step at which a bad cell was found
  double last_ch, last_dt;      // ch and dt of the last step taken
  unsigned long long degenerate, nonphysical;  // HLLD fallbacks this advance
  unsigned long long active_stage_launches;    // stage launches that did work
  double t_bad;                 // time at the start of the failing step (Hancock)
  // Test hook of the bounded-wait path, 0 in normal runs.  When > 0, a
  // one-grid stage launch issues no input load for its first tile and waits
  // for it at most this many polls, so every CTA takes the wait-expired exit
  // with nothing in flight.  Set by the host from PMHD_TEST_STALL_POLLS.
  int test_stall;
};

enum DeviceErr : int { DERR_NONE = 0, DERR_TMA_TIMEOUT = 1 };

// ---- shared-memory barrier + TMA (sm_90+/sm_100a PTX) --------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns false if the phase did not
// complete within `max_iters` polls (each poll may suspend the thread for a
// hardware-defined interval); the caller then records an error and leaves.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_iters) {
  for (uint32_t it = 0; it < max_iters; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3-D tiled TMA load (no multicast) of box {x, y, z} into shared memory,
// completing on `bar` with the box's byte count.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Prefetches a TMA box (same coordinates as tma_load_3d) into L2.
__device__ __forceinline__ void tma_prefetch_3d(const void* tmap, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(tmap), "r"(x), "r"(y),
               "r"(z)
               : "memory");
}

// Orders this CTA's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

// ---- reductions ----------------------------------------------------------

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  return v;
}

__device__ __forceinline__ unsigned warp_sum_u32(unsigned v) { return __reduce_add_sync(0xffffffffu, v); }

// Positive doubles order like their bit patterns.  Zero, -0.0 and NaN map
// to 0 so they never win the max (NaN would otherwise sort above +inf).
__device__ __forceinline__ unsigned long long speed_bits(double v) {
  return (v > 0.0) ? static_cast<unsigned long long>(__double_as_longlong(v)) : 0ull;
}

}  // namespace pmhd

#endif  // PMHD_COMMON_CUH
