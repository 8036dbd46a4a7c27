// stage_kernels.cuh -- the fused SSPRK2 stage kernel and its helpers.
//
// One launch performs one SSPRK2 stage of the 2D ideal-MHD + mixed-GLM
// finite-volume step for every grid of a batch (reference: the kernel chain
// bcX/bcY -> fluxX -> fluxY -> rhs -> stage1/stage2 of
// src/mhd/mhd2d_glm_gpu.cu:141-321, plus speedKernel/rateKernel :171-222
// for the next step's CFL reduction).  Per 32 x TY output tile:
//
//   1. TMA loads the stage input tile with its 2-cell halo, all nine SoA
//      planes, into shared memory (one 3-D box, no multicast).  CTAs are
//      persistent and load their next tile while they compute the current
//      one.
//   2. Every tile cell is recovered to primitives once (the reference
//      recovers each cell up to 8 times, once per stencil use; the result of
//      a recovery depends only on the cell, so this is bit-identical).
//   3. One thread per interface: MUSCL reconstruction of the two adjacent
//      cells from shared memory, then the GLM + HLLD (or HLL) Riemann flux.
//      Interfaces shared with the neighbouring tile are computed by both
//      tiles, but counted only by the tile to their right/top.
//   4. One thread per cell: flux divergence, psi damping, the SSPRK2
//      combination, the usability check, the store (including this cell's
//      ghost copies for the boundary conditions) and, in stage 2, the
//      signal speed of the new state for the next step's CFL max.
//
// Time stepping state lives in each grid's device control block (Ctrl); the
// kernels derive ch, dt and the stop condition from it, so many steps can be
// replayed from one CUDA graph without returning to the host, and the grids
// of a batch advance with their own time steps.
//
// Precision policies:
//   PolF64   storage, recovery, flux and update in binary64
//   PolF32   storage, recovery, flux and update in binary32
//   PolMixed storage, recovery (one reciprocal of the density), flux
//            divergence scaling and update in binary64; reconstruction,
//            Riemann flux, flux differences and CFL speed in binary32
#ifndef PMHD_STAGE_KERNELS_CUH
#define PMHD_STAGE_KERNELS_CUH

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernel_api.h"
#include "pmhd/point.hpp"

#ifndef PMHD_KNS
#error "PMHD_KNS (kernel namespace: exact or fast) must be defined"
#endif

// PMHD_FAST_FLUX = 1 in the performance build (see Makefile): the HLLD
// performance arithmetic, the binary64 MUSCL faces go to the Riemann solver
// as primitives (glm_flux_prim), and tiles whose cells are all usable skip
// the face usability tests of the reconstruction (cell_usable_fast).  0 in
// the parity build.
#ifndef PMHD_FAST_FLUX
#define PMHD_FAST_FLUX 0
#endif

namespace pmhd {
namespace PMHD_KNS {

struct PolF64 {
  using S = double;  // storage
  using R = double;  // reconstruction / Riemann flux
  using TT = double; // time, dt, dx
  static constexpr bool kMixed = false;
};
struct PolF32 {
  using S = float;
  using R = float;
  using TT = float;
  static constexpr bool kMixed = false;
};
struct PolMixed {
  using S = double;
  using R = float;
  using TT = double;
  static constexpr bool kMixed = true;
};

constexpr int TX = 32;                    // tile width: one warp per tile row
constexpr int NTA = 256;                  // threads per CTA of the auxiliary kernels
constexpr uint32_t kWaitIters = 1u << 22; // bound on mbarrier polls

// Geometry of a 32 x TY tile: TY warps own one tile row each, one more warp
// handles the tile's bottom row of y-interfaces and left column of
// x-interfaces.
template <int TY_>
struct Geo {
  static constexpr int TY = TY_;
  static constexpr int HX = TX + 4, HY = TY + 4;  // tile with halo
  static constexpr int TC = HX * HY;              // cells per loaded tile
  static constexpr int NW = TY + 1;               // warps per CTA
  static constexpr int NT = NW * 32;              // threads per CTA
  static constexpr int FXN = TY * (TX + 1);       // x-interfaces per tile
  static constexpr int GYN = (TY + 1) * TX;       // y-interfaces per tile
  static_assert(TY <= 32, "the extra warp covers the left column");
};

constexpr size_t align128(size_t b) { return (b + 127) & ~size_t(127); }

// Per-policy, per-tile-height launch tuning, measured on B200 at Orszag-Tang
// 4096^2 (the stage kernel is issue-bound, so these trade occupancy against
// registers and shared memory):
//   nbuf  input tile buffers: 1 = the next tile's TMA load reuses the buffer
//         as soon as the current tile is recovered (the update then reads
//         its own cell from global memory, an L2 hit); 2 = double buffering
//         (the update reads shared memory);
//   minb  resident CTAs per SM the register allocation is sized for.
// 32 x 8 tiles: fp64 1 buffer / 2 CTAs (a small spill beats halving the
// resident warps), fp32 1 / 3, mixed 2 / 2.  The default tile is 32 x 19
// with one CTA per SM: 20 warps, five on each of the SM's four schedulers,
// whose 16 K-register files then allow 96 registers a thread.  A 32 x 16
// tile has 17 warps (5 / 4 / 4 / 4 per scheduler, so the same 96-register
// cap with fewer warps), a 32 x 15 tile 16 warps at 128 registers.  At
// 4096^2 (performance build) 32 x 19 runs mixed 5.91, fp64 2.42, fp32 6.68 G
// zone-cycles/s against 5.25 / 2.20 / 6.04 at 32 x 16 and 5.90 / 2.28 / 6.69
// at 32 x 15; it also recomputes the fewest halo interfaces and recoveries
// (2.08 interface solves and 1.34 recoveries per cell; 32 x 16: 2.09 / 1.41;
// 32 x 8: 2.16 / 1.63).  32 x 4 tiles keep about the same threads per SM as
// 32 x 8.  PMHD_NBUF / PMHD_MINB_R32 / PMHD_MINB_R64 override the 32 x 8
// values for tuning experiments.
template <class Pol, int TY>
struct Tune {
  static constexpr bool r64 = sizeof(typename Pol::R) == 8;
#ifdef PMHD_NBUF
  static constexpr int nbuf = PMHD_NBUF;
#else
  static constexpr int nbuf = Pol::kMixed ? 2 : 1;
#endif
#ifdef PMHD_MINB_R64
  static constexpr int minb_r64 = PMHD_MINB_R64;
#else
  static constexpr int minb_r64 = 2;
#endif
#ifdef PMHD_MINB_R32
  static constexpr int minb_r32 = PMHD_MINB_R32;
#else
  static constexpr int minb_r32 = Pol::kMixed ? 2 : 3;
#endif
  static constexpr int minb8 = r64 ? minb_r64 : minb_r32;
  static constexpr int minb = TY == 8 ? minb8 : (TY == 4 ? (minb8 * 9) / 5 : 1);
};

template <class Pol, int TY>
struct Smem {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using G = Geo<TY>;
  static constexpr int NBUF = Tune<Pol, TY>::nbuf;
  static constexpr size_t u_bytes = sizeof(S) * NVAR * G::TC;  // TMA box size
  static constexpr size_t u_stride = align128(u_bytes);         // per buffer
  static constexpr size_t p_off = u_stride * NBUF;
  static constexpr size_t fx_off = p_off + align128(sizeof(R) * NVAR * G::TC);
  static constexpr size_t gy_off = fx_off + align128(sizeof(R) * NVAR * G::FXN);
  static constexpr size_t total = gy_off + align128(sizeof(R) * NVAR * G::GYN);
};

// Performance build: whether a recovered cell may take part in a limited
// reconstruction (positive density and pressure, all nine values finite; a
// sum is non-finite exactly when a term is, barring overflow, which only
// makes the test stricter).  When every cell of a tile is usable, every
// minmod-limited face is usable too -- a face lies between the cell value and
// the midpoint towards a neighbour, so it stays above the floors (up to the
// rounding of that one operation) and finite -- and the tile skips the face
// tests of the reference (reconstructPrimitiveDev, mhd2d_glm_gpu.cu:81-95).
// A tile with any unusable cell runs them.
template <class R>
__device__ __forceinline__ bool cell_usable_fast(const R* P) {
  R sum = P[0];
#pragma unroll
  for (int k = 1; k < NVAR; k++) sum += P[k];
  return P[RHO] > rho_floor<R>() && P[EN] > p_floor<R>() && vfinite(sum);
}

// Primitive recovery of one cell in the storage precision.  PolF64/PolF32
// follow the reference (stateToPrimitiveDev, mhd2d_glm_gpu.cu:53-58: three
// divisions by the density).  PolMixed is this project's variant: one
// binary64 reciprocal of the density and three products, the pressure from
// total energy in the reference's association order.
template <class Pol>
__device__ __forceinline__ void recover_cell(const typename Pol::S* U, typename Pol::S* P,
                                             const Phys<typename Pol::S>& ph) {
  if constexpr (Pol::kMixed) {
    const double rho = fmax(U[RHO], 1.0e-12);
    // Performance build: Newton-refined reciprocal (within binary64 rounding).
    const double inv = PMHD_FAST_FLUX ? rcp_newton(rho) : 1.0 / rho;
    const double vx = U[MX] * inv, vy = U[MY] * inv, vz = U[MZ] * inv;
    const double bx = U[BX], by = U[BY], bz = U[BZ];
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double b2 = bx * bx + by * by + bz * bz;
    P[RHO] = rho;
    P[MX] = vx;
    P[MY] = vy;
    P[MZ] = vz;
    P[EN] = ph.gm1 * (U[EN] - 0.5 * rho * v2 - 0.5 * b2);
    P[BX] = bx;
    P[BY] = by;
    P[BZ] = bz;
    P[PSI] = U[PSI];
  } else if (PMHD_FAST_FLUX) {
    // Performance build: one reciprocal of the density for the velocities.
    using S = typename Pol::S;
    const S rho = vmax(U[RHO], rho_floor<S>());
    const S inv = fast_rcp(rho);
    const S vx = U[MX] * inv, vy = U[MY] * inv, vz = U[MZ] * inv;
    const S bx = U[BX], by = U[BY], bz = U[BZ];
    P[RHO] = rho;
    P[MX] = vx;
    P[MY] = vy;
    P[MZ] = vz;
    P[EN] = ph.gm1 * (U[EN] - (S)0.5 * rho * (vx * vx + vy * vy + vz * vz) - (S)0.5 * (bx * bx + by * by + bz * bz));
    P[BX] = bx;
    P[BY] = by;
    P[BZ] = bz;
    P[PSI] = U[PSI];
  } else {
    state_to_prim9<typename Pol::S>(U, P, ph);
  }
}

// Ghost copies of interior index i (0 <= i < n) along one axis, in ghosted
// coordinates, with whether the copy is a mirror image (reflecting wall).
// Follows the ghost fill of the reference (mhd2d_glm_gpu.cu:141-168) for
// periodic sides, extended with reflecting and transmissive sides.
__device__ __forceinline__ int ghost_targets(int i, int n, int lo, int hi, int pos[4], bool flip[4]) {
  int m = 0;
  pos[m] = i + GHOST;
  flip[m++] = false;
  if (lo == BC_PERIODIC) {
    if (i >= n - 2) { pos[m] = i - n + 2; flip[m++] = false; }
  } else if (lo == BC_REFLECT) {
    if (i < 2) { pos[m] = 1 - i; flip[m++] = true; }
  } else if (i == 0) {
    pos[m] = 0; flip[m++] = false;
    pos[m] = 1; flip[m++] = false;
  }
  if (hi == BC_PERIODIC) {
    if (i < 2) { pos[m] = n + 2 + i; flip[m++] = false; }
  } else if (hi == BC_REFLECT) {
    if (i >= n - 2) { pos[m] = 2 * n + 1 - i; flip[m++] = true; }
  } else if (i == n - 1) {
    pos[m] = n + 2; flip[m++] = false;
    pos[m] = n + 3; flip[m++] = false;
  }
  return m;
}

// Store one interior cell and all of its ghost copies.
template <class S>
__device__ __forceinline__ void store_cell(S* u, long long plane, int pitch, int i, int j, int nx, int ny,
                                           const int bc[4], const S* v) {
  const size_t own = (size_t)(j + GHOST) * pitch + (i + GHOST);
#pragma unroll
  for (int k = 0; k < NVAR; k++) u[(size_t)k * plane + own] = v[k];
  const bool edge = (i < 2) | (i >= nx - 2) | (j < 2) | (j >= ny - 2);
  if (!edge) return;
  int px[4], py[4];
  bool fx[4], fy[4];
  const int mx = ghost_targets(i, nx, bc[0], bc[1], px, fx);
  const int my = ghost_targets(j, ny, bc[2], bc[3], py, fy);
  for (int a = 0; a < mx; a++)
    for (int b = 0; b < my; b++) {
      if (a == 0 && b == 0) continue;
      const size_t o = (size_t)py[b] * pitch + px[a];
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        S w = v[k];
        if (fx[a] && (k == MX || k == BX)) w = -w;
        if (fy[b] && (k == MY || k == BY)) w = -w;
        u[(size_t)k * plane + o] = w;
      }
    }
}

// Face states and Riemann flux of one interface, always computed in x-normal
// slot order, from the tile's primitives in shared memory (MUSCL) or its
// conserved states (first order).  A y-interface is solved exactly as the
// reference solves it: the stencil is read with the x and y slots of
// velocity/momentum and field swapped (mhdRotateYToX, mhd_common.hpp:381-391),
// the x-direction routine runs, and the caller stores the flux back through
// the same swap (mhdRotateFluxXToY, :395-405).  Reconstruction is per
// component and the primitive->conserved sums are order-independent, so this
// equals the reference bit for bit.  One copy of the flux code then serves
// both directions, which keeps the kernel's hot loop inside the instruction
// cache.
//   base   tile index of the cell two steps upwind of the interface
//   stride 1 (x) or HX (y)
//   o1/o2  plane offsets of the normal / first tangential velocity slot
//   o5/o6  plane offsets of the normal / first tangential field slot
//   checks whether the reconstruction runs the reference's face usability
//          tests (always in the parity build; in the performance build only
//          in tiles with an unusable cell, see cell_usable_fast)
template <class Pol, bool HLLD, int TC>
__device__ __forceinline__ int face_flux(const typename Pol::R* sP, bool checks, int base, int stride, int o1,
                                         int o2, int o5, int o6, int muscl, const GlmK<typename Pol::R>& gk,
                                         const Phys<typename Pol::R>& ph, typename Pol::R* F) {
  using R = typename Pol::R;
  const int off[NVAR] = {0, o1, o2, 3 * TC, 4 * TC, o5, o6, 7 * TC, 8 * TC};
  R UL[NVAR], UR[NVAR];
  if (muscl) {
    R Pm[NVAR], P0[NVAR], P1[NVAR], P2[NVAR], Pa[NVAR], Pb[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      const R* q = sP + off[k] + base;
      Pm[k] = q[0];
      P0[k] = q[stride];
      P1[k] = q[2 * stride];
      P2[k] = q[3 * stride];
    }
    // Pa: right face of cell 0, Pb: left face of cell 1.
    if (PMHD_FAST_FLUX && !checks) {
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        const R d1 = P1[k] - P0[k];
        Pa[k] = P0[k] + (R)0.5 * minmod_fast(P0[k] - Pm[k], d1);
        Pb[k] = P1[k] - (R)0.5 * minmod_fast(d1, P2[k] - P1[k]);
      }
    } else {
      R Pl[NVAR];
      recon_cell<R>(Pm, P0, P1, Pl, Pa);
      recon_cell<R>(P0, P1, P2, Pb, Pl);
    }
#if PMHD_FAST_FLUX
    // Performance build: the face primitives go to the solver directly
    // (glm_flux_fast), no primitive -> conserved -> primitive trip.
    return glm_flux_fast<R, 0>(Pa, Pb, gk, HLLD, F, ph);
#else
    prim9_to_state<R>(Pa, UL, ph);
    prim9_to_state<R>(Pb, UR, ph);
#endif
  } else {  // first order: sP holds the conserved states
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      UL[k] = sP[off[k] + base + stride];
      UR[k] = sP[off[k] + base + 2 * stride];
    }
  }
  return glm_flux<R, 0, PMHD_FAST_FLUX != 0>(UL, UR, gk.ch, HLLD, F, ph);
}

// Per-member step values (uniform for all tiles of a member in one launch).
template <class Pol>
struct StepVals {
  typename Pol::R ch;
  typename Pol::TT t, dt;
  long long step;
  bool active;
  int bad_prev;
};

// Reads a member's control slot and derives ch, dt and whether it steps.
template <class Pol, int STAGE>
__device__ __forceinline__ StepVals<Pol> step_values(const Member& m, int p) {
  using R = typename Pol::R;
  using TT = typename Pol::TT;
  const Ctrl* c = m.ctrl;
  StepVals<Pol> v;
  const double t_raw = c->t[p];
  v.step = c->step[p];
  v.bad_prev = (STAGE == 1) ? c->bad2 : c->bad1;
  v.active = !c->halted && !c->err && v.bad_prev == BAD_NONE && (TT)t_raw < (TT)c->t_end && v.step < c->step_limit;
  v.ch = vmax((R)__longlong_as_double((long long)c->chbits[p]), (R)1.0e-12);
  v.t = (TT)t_raw;
  // max over cells of max(s_x, ch)/dx + max(s_y, ch)/dy equals ch/dx + ch/dy
  // because ch is the maximum of every s_x and s_y (mhd2d_glm_gpu.cu:485-500).
  const TT max_rate = (TT)v.ch / (TT)m.dx + (TT)v.ch / (TT)m.dy;
  TT dt = (TT)m.cfl / max_rate;
  const TT t_end = (TT)c->t_end;
  if (v.t + dt > t_end) dt = t_end - v.t;
  v.dt = dt;
  return v;
}

// Work accumulated by a CTA for the member it is currently processing;
// flushed with one atomic per warp when the member changes and at the end.
struct MemberAcc {
  int member;
  unsigned n_deg, n_np;
  unsigned long long sp_bits;
};

template <bool HLLD, int STAGE>
__device__ __forceinline__ void flush_acc(MemberAcc& acc, const Member* members, int lane, int p) {
  if (acc.member < 0) return;
  Ctrl* c = members[acc.member].ctrl;
  if (HLLD) {
    const unsigned d = warp_sum_u32(acc.n_deg), np = warp_sum_u32(acc.n_np);
    if (lane == 0 && d) atomicAdd(&c->degenerate, (unsigned long long)d);
    if (lane == 0 && np) atomicAdd(&c->nonphysical, (unsigned long long)np);
  }
  if (STAGE == 2) {
    const unsigned long long mbits = warp_max_u64(acc.sp_bits);
    if (lane == 0 && mbits) atomicMax(&c->chbits[p ^ 1], mbits);
  }
  acc.n_deg = acc.n_np = 0;
  acc.sp_bits = 0;
}

// The member's once-per-launch control updates, done by the thread that
// processes (or skips) the member's first tile.
template <class Pol, int STAGE>
__device__ __forceinline__ void member_bookkeeping(const Member& m, const StepVals<Pol>& v, int p) {
  Ctrl* c = m.ctrl;
  if (!v.active) {  // carry the slot forward so the other parity also stops
    c->t[p ^ 1] = c->t[p];
    c->step[p ^ 1] = c->step[p];
    c->chbits[p ^ 1] = c->chbits[p];
    if (v.bad_prev != BAD_NONE || c->err) c->halted = 1;
    return;
  }
  atomicAdd(&c->active_stage_launches, 1ull);
  if (STAGE == 1) {
    c->chbits[p ^ 1] = 0ull;  // stage 2 of this step accumulates into it
  } else {
    c->t[p ^ 1] = (double)(v.t + v.dt);
    c->step[p ^ 1] = v.step + 1;
    c->last_ch = (double)v.ch;
    c->last_dt = (double)v.dt;
  }
}

// Whether a member steps in this launch (step_values without the arithmetic).
template <class Pol, int STAGE>
__device__ __forceinline__ bool member_active(const Member& m, int p) {
  using TT = typename Pol::TT;
  const Ctrl* c = m.ctrl;
  const int bad_prev = (STAGE == 1) ? c->bad2 : c->bad1;
  return !c->halted && !c->err && bad_prev == BAD_NONE && (TT)c->t[p] < (TT)c->t_end && c->step[p] < c->step_limit;
}

// BATCHED = false: one grid, passed by value as a kernel parameter (its
// scalars are then constant-bank operands and its TMA descriptors live in
// parameter space); `b` only supplies the tile count.  BATCHED = true: the
// members of `b`, read from device memory per tile.
template <class Pol, int STAGE, bool HLLD, int TY, bool BATCHED>
__global__ void __launch_bounds__(Geo<TY>::NT, Tune<Pol, TY>::minb)
    stage_kernel(const __grid_constant__ Member m0, const Batch b, const int p) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using G = Geo<TY>;
  constexpr int HX = G::HX, TC = G::TC, NT = G::NT, FXN = G::FXN, GYN = G::GYN;
  constexpr int NBUF = Tune<Pol, TY>::nbuf;
  constexpr int TI = kTileHeights[0] == TY ? 0 : 1;  // index into Member::tm
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw + Smem<Pol, TY>::p_off);
  R* sFx = reinterpret_cast<R*>(smem_raw + Smem<Pol, TY>::fx_off);
  R* sGy = reinterpret_cast<R*>(smem_raw + Smem<Pol, TY>::gy_off);
  __shared__ __align__(8) uint64_t bar[NBUF];
  auto ubuf = [&](int k) { return reinterpret_cast<S*>(smem_raw + (size_t)k * Smem<Pol, TY>::u_stride); };

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  auto member_of = [&](int t) { return BATCHED ? b.tile_member[t] : 0; };
  auto tile0_of = [&](int mi) { return BATCHED ? b.member_tile0[mi] : 0; };
  auto member = [&](int mi) -> const Member& { return BATCHED ? b.members[mi] : m0; };

  // One grid that does not step this launch: nothing to load.
  if (!BATCHED && !member_active<Pol, STAGE>(m0, p)) {
    if (blockIdx.x == 0 && tid == 0) member_bookkeeping<Pol, STAGE>(m0, step_values<Pol, STAGE>(m0, p), p);
    return;
  }

  // Tile order.  One grid: tile blockIdx.x, then every gridDim.x-th.  A
  // batch: runs of kBatchRun consecutive tiles, run blockIdx.x, then
  // every gridDim.x-th run -- consecutive tiles of a CTA then mostly share
  // a member, so its descriptor, control slot and step values are re-read
  // once per member run instead of once per tile, while members that stop
  // early still leave their tiles spread over all CTAs.
  auto first_tile = [&]() { return BATCHED ? (int)blockIdx.x * kBatchRun : (int)blockIdx.x; };
  auto after = [&](int t) {
    if constexpr (BATCHED)
      return (t + 1) % kBatchRun != 0 ? t + 1 : t + 1 + ((int)gridDim.x - 1) * kBatchRun;
    else
      return t + (int)gridDim.x;
  };
  // Next tile of this CTA, from t on, whose member steps; members that do
  // not step get their bookkeeping from whoever meets their tile 0.
  int active_mi = -1;  // member last found stepping (batch)
  auto next_active = [&](int t) {
    if constexpr (BATCHED) {
      for (; t < b.ntiles; t = after(t)) {
        const int mi = member_of(t);
        if (mi == active_mi) return t;
        const Member& mm = b.members[mi];
        if (member_active<Pol, STAGE>(mm, p)) {
          active_mi = mi;
          return t;
        }
        if (t == tile0_of(mi) && tid == 0) member_bookkeeping<Pol, STAGE>(mm, step_values<Pol, STAGE>(mm, p), p);
      }
      return b.ntiles;
    } else {
      return t < b.ntiles ? t : b.ntiles;
    }
  };
  auto issue = [&](int t, int k) {
    const int mi = member_of(t);
    const Member& mm = member(mi);
    const int lt = t - tile0_of(mi);
    const int tiles_x = (mm.nx + TX - 1) / TX;
    mbar_arrive_expect_tx(&bar[k], (uint32_t)Smem<Pol, TY>::u_bytes);
    tma_load_3d(ubuf(k), &mm.tm[TI][STAGE - 1], &bar[k], (lt % tiles_x) * TX, (lt / tiles_x) * TY, 0);
  };

  if (tid == 0) {
    for (int k = 0; k < NBUF; k++) mbar_init(&bar[k], 1);
    fence_barrier_init();
  }
  __syncthreads();
  // Test hook (Ctrl::test_stall): no first load, a short wait, the error exit.
  const int stall = BATCHED ? 0 : m0.ctrl->test_stall;
  int tile = next_active(first_tile());
  if (tid == 0 && tile < b.ntiles && stall == 0) issue(tile, 0);
  MemberAcc acc = {-1, 0, 0, 0ull};
  StepVals<Pol> v = step_values<Pol, STAGE>(member(BATCHED ? (tile < b.ntiles ? member_of(tile) : 0) : 0), p);

  for (int it = 0; tile < b.ntiles; it++) {
    const int mi = member_of(tile);
    const Member& m = member(mi);
    if (mi != acc.member) {
      flush_acc<HLLD, STAGE>(acc, BATCHED ? b.members : &m0, lane, p);
      acc.member = mi;
      if (BATCHED) v = step_values<Pol, STAGE>(m, p);
    }
    const int lt = tile - tile0_of(mi);
    const int tiles_x = (m.nx + TX - 1) / TX;
    const int i0 = (lt % tiles_x) * TX, j0 = (lt / tiles_x) * TY;
    const Phys<R> phR = Phys<R>::make(m.gamma, m.tol);
    const Phys<S> phS = Phys<S>::make(m.gamma, m.tol);
    const int cb = it % NBUF;                        // buffer of this tile
    const uint32_t par = (uint32_t)(it / NBUF) & 1;  // its mbarrier phase
    S* sU = ubuf(cb);
    const bool got =
        __syncthreads_and(mbar_wait_bounded(&bar[cb], par, stall > 0 ? (uint32_t)stall : kWaitIters));
    if (!got) {
      if (tid == 0) atomicExch(&m.ctrl->err, (int)DERR_TMA_TIMEOUT);
      // Let an issued copy land before leaving (the test hook issued none).
      if (stall == 0) mbar_wait_bounded(&bar[cb], par, kWaitIters);
      return;
    }

    // ---- recovery, once per tile cell (halo corners are never used) -------
    // First order needs no primitives: the conserved states are staged.
    bool usable = true;  // performance build: this thread's cells (cell_usable_fast)
    for (int q = tid; q < TC; q += NT) {
      const int cx = q % HX, cy = q / HX;
      if ((cx < 2 || cx >= TX + 2) && (cy < 2 || cy >= TY + 2)) continue;
      S U9[NVAR], P9[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) U9[k] = sU[k * TC + q];
      if (m.muscl) {
        recover_cell<Pol>(U9, P9, phS);
      } else {
#pragma unroll
        for (int k = 0; k < NVAR; k++) P9[k] = U9[k];
      }
      R PR[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        PR[k] = (R)P9[k];
        sP[k * TC + q] = PR[k];
      }
      if (PMHD_FAST_FLUX && m.muscl) usable = usable && cell_usable_fast<R>(PR);
    }
    const bool all_usable = __syncthreads_and(usable);
    const bool checks = !PMHD_FAST_FLUX || !all_usable;
    // The next tile goes into the buffer no thread reads any more: this one
    // (just recovered) or, double-buffered, the previous tile's.
    const int next = next_active(after(tile));
    if (tid == 0 && next < b.ntiles) {
      fence_proxy_async_smem();  // order earlier reads of that buffer before the async overwrite
      issue(next, (it + 1) % NBUF);
    }
    // Stage 2 also reads U^n of its cells in the update: start bringing this
    // tile's box of it into L2 now, so the update finds it there.
    if (STAGE == 2 && tid == 32) tma_prefetch_3d(&m.tm[TI][0], i0, j0, 0);

    // ---- interface fluxes --------------------------------------------------
    // Warps 0..TY-1 own one tile row each: lane tx computes the x-interface
    // to the right of cell (tx, ty), then the y-interface above it.  The last
    // warp computes the tile's bottom row of y-interfaces, then its left
    // column of x-interfaces.  Every warp runs two rounds, each round one
    // direction for the whole warp, through one (not unrolled) copy of the
    // flux code.
#pragma unroll 1
    for (int r = 0; r < 2; r++) {
      int axis, fx, fy;
      if (warp < TY) {
        axis = r;
        fx = r ? lane : lane + 1;
        fy = r ? warp + 1 : warp;
      } else {
        axis = 1 - r;
        fx = r ? 0 : lane;
        fy = r ? lane : 0;
        if (r == 1 && lane >= TY) continue;
      }
      // x: interface between cells (i0+fx-1, j0+fy) and (i0+fx, j0+fy)
      // y: interface between cells (i0+fx, j0+fy-1) and (i0+fx, j0+fy)
      const bool valid = axis ? (j0 + fy <= m.ny && i0 + fx < m.nx) : (i0 + fx <= m.nx && j0 + fy < m.ny);
      if (!valid) continue;
      const int base = axis ? fy * HX + fx + 2 : (fy + 2) * HX + fx;
      const int stride = axis ? HX : 1;
      const int o1 = (axis ? 2 : 1) * TC, o2 = (axis ? 1 : 2) * TC;
      const int o5 = (axis ? 6 : 5) * TC, o6 = (axis ? 5 : 6) * TC;
      R F[NVAR];
      const int st = face_flux<Pol, HLLD, TC>(sP, checks, base, stride, o1, o2, o5, o6, m.muscl, GlmK<R>::make(v.ch), phR, F);
      R* out = axis ? sGy : sFx;
      const int n_out = axis ? GYN : FXN;
      const int item = axis ? fy * TX + fx : fy * (TX + 1) + fx;
      const int p1 = axis ? 2 : 1, p2 = axis ? 1 : 2, p5 = axis ? 6 : 5, p6 = axis ? 5 : 6;
      out[0 * n_out + item] = F[0];
      out[p1 * n_out + item] = F[1];
      out[p2 * n_out + item] = F[2];
      out[3 * n_out + item] = F[3];
      out[4 * n_out + item] = F[4];
      out[p5 * n_out + item] = F[5];
      out[p6 * n_out + item] = F[6];
      out[7 * n_out + item] = F[7];
      out[8 * n_out + item] = F[8];
      if (HLLD && ((axis ? fy : fx) >= 1 || (axis ? j0 : i0) == 0)) {
        acc.n_deg += (st == HLLD_FALLBACK_DEGENERATE);
        acc.n_np += (st == HLLD_FALLBACK_NONPHYSICAL);
      }
    }
    __syncthreads();

    // ---- divergence, update, checks, store, next-step speed ---------------
    const int tx = lane, ty = warp;
    const int gi = i0 + tx, gj = j0 + ty;
    if (warp < TY && gi < m.nx && gj < m.ny) {
      const size_t gidx = (size_t)(gj + GHOST) * m.pitch + (gi + GHOST);
      const int lc = (ty + 2) * HX + tx + 2;
      const S* u_in = static_cast<const S*>(STAGE == 1 ? m.u : m.u1);
      S* u_out = static_cast<S*>(STAGE == 1 ? m.u1 : m.u);
      S Un[NVAR];
      if constexpr (!Pol::kMixed) {
        // Reference order (mhd2d_glm_gpu.cu:282-285, :299, :316-317); the
        // performance build multiplies by 1 / dx, 1 / dy (Member) instead of
        // dividing.
        const R damping = v.ch / vmax((R)m.alpha, (R)1.0e-12);
        const R dxR = (R)m.dx, dyR = (R)m.dy, dtR = (R)v.dt;
        const R idxR = (R)m.inv_dx, idyR = (R)m.inv_dy;
#pragma unroll
        for (int k = 0; k < NVAR; k++) {
          const R uin = NBUF == 2 ? sU[k * TC + lc] : u_in[(size_t)k * m.plane + gidx];
          const R dfx = sFx[k * FXN + ty * (TX + 1) + tx + 1] - sFx[k * FXN + ty * (TX + 1) + tx];
          const R dgy = sGy[k * GYN + (ty + 1) * TX + tx] - sGy[k * GYN + ty * TX + tx];
          R rhs = PMHD_FAST_FLUX ? -dfx * idxR - dgy * idyR : -dfx / dxR - dgy / dyR;
          if (k == PSI) rhs -= damping * uin;
          if (STAGE == 1) {
            Un[k] = uin + dtR * rhs;
          } else {
            const S uold = static_cast<const S*>(m.u)[(size_t)k * m.plane + gidx];
            Un[k] = (R)0.5 * uold + (R)0.5 * (uin + dtR * rhs);
          }
        }
      } else {
        // Binary32 fluxes and their differences, binary64 scaling and
        // accumulation (m.inv_dx = 1.0 / dx in binary64, set on the host).
        const double damping = (double)v.ch / fmax(m.alpha, 1.0e-12);
#pragma unroll
        for (int k = 0; k < NVAR; k++) {
          const double uin = NBUF == 2 ? sU[k * TC + lc] : u_in[(size_t)k * m.plane + gidx];
          const float dfx = sFx[k * FXN + ty * (TX + 1) + tx + 1] - sFx[k * FXN + ty * (TX + 1) + tx];
          const float dgy = sGy[k * GYN + (ty + 1) * TX + tx] - sGy[k * GYN + ty * TX + tx];
          double rhs = -(double)dfx * m.inv_dx - (double)dgy * m.inv_dy;
          if (k == PSI) rhs -= damping * uin;
          if (STAGE == 1) {
            Un[k] = uin + (double)v.dt * rhs;
          } else {
            const double uold = static_cast<const double*>(m.u)[(size_t)k * m.plane + gidx];
            Un[k] = 0.5 * uold + 0.5 * (uin + (double)v.dt * rhs);
          }
        }
      }
      // stateIsUsable (mhd2d_glm_gpu.cu:74-79); its recovery doubles as the
      // recovery of the next step's CFL speed (speedKernel, :171-195).
      S P9[NVAR];
      recover_cell<Pol>(Un, P9, phS);
      if (!(Un[RHO] > rho_floor<S>()) || !prim9_usable<S>(P9)) {
        atomicMin(STAGE == 1 ? &m.ctrl->bad1 : &m.ctrl->bad2, gj * m.nx + gi);
        m.ctrl->bad_step = v.step;
      }
      store_cell<S>(u_out, m.plane, m.pitch, gi, gj, m.nx, m.ny, m.bc, Un);
      if (STAGE == 2) {
        R Pr[NVAR];
#pragma unroll
        for (int k = 0; k < NVAR; k++) Pr[k] = (R)P9[k];
        const unsigned long long sb =
            speed_bits((double)(PMHD_FAST_FLUX ? cell_speed_fast<R>(Pr, phR) : cell_speed<R>(Pr, phR)));
        acc.sp_bits = sb > acc.sp_bits ? sb : acc.sp_bits;
      }
    }
    if (lt == 0 && tid == 0) member_bookkeeping<Pol, STAGE>(m, v, p);
    tile = next;
  }
  flush_acc<HLLD, STAGE>(acc, BATCHED ? b.members : &m0, lane, p);
}

// ---- initial CFL speed: max over interior cells into chbits[slot] ----------
template <class Pol>
__global__ void __launch_bounds__(NTA) speed_kernel(const typename Pol::S* __restrict__ u, long long plane, int nx,
                                                   int ny, int pitch, double gamma, Ctrl* c, int slot) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  const Phys<S> phS = Phys<S>::make(gamma, 0.0);
  const Phys<R> phR = Phys<R>::make(gamma, 0.0);
  unsigned long long m = 0;
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)NTA + threadIdx.x; q < n; q += (long long)gridDim.x * NTA) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t g = (size_t)(j + GHOST) * pitch + (i + GHOST);
    S U9[NVAR], P9[NVAR];
    R Pr[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) U9[k] = u[(size_t)k * plane + g];
    recover_cell<Pol>(U9, P9, phS);
#pragma unroll
    for (int k = 0; k < NVAR; k++) Pr[k] = (R)P9[k];
    const unsigned long long b =
        speed_bits((double)(PMHD_FAST_FLUX ? cell_speed_fast<R>(Pr, phR) : cell_speed<R>(Pr, phR)));
    m = b > m ? b : m;
  }
  __shared__ unsigned long long red[NTA / 32];
  m = warp_max_u64(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NTA / 32; w++) m = red[w] > m ? red[w] : m;
    if (m) atomicMax(&c->chbits[slot], m);
  }
}

// ---- layout conversion between the caller's AoS buffer and the SoA planes --
// AoS layout 0: interior only, [ny][nx][9]; layout 1: the reference's
// ghosted array, [(ny+4)][(nx+4)][9] (ghost values are rebuilt from the
// boundary conditions on input).
template <class S>
__global__ void __launch_bounds__(NTA) aos_to_soa_kernel(const S* __restrict__ aos, int layout, S* u, long long plane,
                                                        int nx, int ny, int pitch, int bc0, int bc1, int bc2,
                                                        int bc3) {
  const int bc[4] = {bc0, bc1, bc2, bc3};
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)NTA + threadIdx.x; q < n; q += (long long)gridDim.x * NTA) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t src = layout == 0 ? (size_t)q * NVAR : ((size_t)(j + GHOST) * (nx + 4) + (i + GHOST)) * NVAR;
    S v[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) v[k] = aos[src + k];
    store_cell<S>(u, plane, pitch, i, j, nx, ny, bc, v);
  }
}

template <class S>
__global__ void __launch_bounds__(NTA) soa_to_aos_kernel(const S* __restrict__ u, long long plane, int nx, int ny,
                                                        int pitch, int layout, S* __restrict__ aos) {
  const int wx = layout == 0 ? nx : nx + 4, wy = layout == 0 ? ny : ny + 4, off = layout == 0 ? GHOST : 0;
  const long long n = (long long)wx * wy;
  for (long long q = blockIdx.x * (long long)NTA + threadIdx.x; q < n; q += (long long)gridDim.x * NTA) {
    const int i = (int)(q % wx), j = (int)(q / wx);
    const size_t g = (size_t)(j + off) * pitch + (i + off);
#pragma unroll
    for (int k = 0; k < NVAR; k++) aos[(size_t)q * NVAR + k] = u[(size_t)k * plane + g];
  }
}

}  // namespace PMHD_KNS
}  // namespace pmhd

#endif  // PMHD_STAGE_KERNELS_CUH
