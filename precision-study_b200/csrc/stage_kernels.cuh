// stage_kernels.cuh -- the fused SSPRK2 stage kernel and its helpers.
//
// One launch performs one SSPRK2 stage of the 2D ideal-MHD + mixed-GLM
// finite-volume step for the whole grid (reference: the kernel chain
// bcX/bcY -> fluxX -> fluxY -> rhs -> stage1/stage2 of
// src/mhd/mhd2d_glm_gpu.cu:141-321, plus speedKernel/rateKernel :171-222
// for the next step's CFL reduction).  Per CTA and 32 x 8 output tile:
//
//   1. TMA loads the stage input tile with its 2-cell halo, all nine SoA
//      planes, into shared memory (one 3-D box, no multicast).  CTAs are
//      persistent (SM count x resident CTAs) and load their next tile while
//      they compute the current one.
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
// Time stepping state lives in the device control block (Ctrl); the kernels
// derive ch, dt and the stop condition from it, so many steps can be
// replayed from one CUDA graph without returning to the host.
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

#ifndef PMHD_TILE_Y
#define PMHD_TILE_Y 8
#endif
constexpr int TX = 32, TY = PMHD_TILE_Y;  // output tile
constexpr int HX = TX + 4, HY = TY + 4;   // tile with halo
constexpr int TC = HX * HY;               // cells per loaded tile
constexpr int NCELL = TX * TY;            // output cells per tile
constexpr int NW = NCELL / 32 + 1;        // warps per CTA: one per tile row + one
constexpr int NT = NW * 32;               // threads per stage CTA (288)
constexpr int NTA = 256;                  // threads per CTA of the auxiliary kernels
constexpr int FXN = TY * (TX + 1);        // x-interfaces per tile
constexpr int GYN = (TY + 1) * TX;        // y-interfaces per tile
constexpr uint32_t kWaitIters = 1u << 22; // bound on mbarrier polls
static_assert(TX == 32, "one warp per tile row");

constexpr size_t align128(size_t b) { return (b + 127) & ~size_t(127); }

// Per-policy launch tuning, measured on B200 at Orszag-Tang 4096^2 (the
// stage kernel is issue-bound, so these trade occupancy against registers
// and shared memory):
//   nbuf  input tile buffers: 1 = the next tile's TMA load reuses the buffer
//         as soon as the current tile is recovered (the update then reads
//         its own cell from global memory, an L2 hit); 2 = double buffering
//         (the update reads shared memory);
//   minb  resident CTAs per SM the register allocation is sized for.
// fp64: 1 buffer, 2 CTAs (a small spill beats halving the resident warps);
// fp32: 1 buffer, 3 CTAs; mixed: 2 buffers (its binary64 tile is large),
// 2 CTAs.  PMHD_NBUF / PMHD_MINB_R32 / PMHD_MINB_R64 override for tuning.
template <class Pol>
struct Tune {
  static constexpr bool r64 = sizeof(typename Pol::R) == 8;
#ifdef PMHD_NBUF
  static constexpr int nbuf = PMHD_NBUF;
#else
  static constexpr int nbuf = Pol::kMixed ? 2 : 1;
#endif
#if defined(PMHD_MINB_R32) && defined(PMHD_MINB_R64)
  static constexpr int minb = r64 ? PMHD_MINB_R64 : PMHD_MINB_R32;
#elif defined(PMHD_MINB_R32)
  static constexpr int minb = r64 ? 2 : PMHD_MINB_R32;
#elif defined(PMHD_MINB_R64)
  static constexpr int minb = r64 ? PMHD_MINB_R64 : (Pol::kMixed ? 2 : 3);
#else
  static constexpr int minb = r64 ? 2 : (Pol::kMixed ? 2 : 3);
#endif
};

template <class Pol>
struct Smem {
  using S = typename Pol::S;
  using R = typename Pol::R;
  static constexpr int NBUF = Tune<Pol>::nbuf;
  static constexpr size_t u_bytes = sizeof(S) * NVAR * TC;  // TMA box size
  static constexpr size_t u_stride = align128(u_bytes);      // per buffer
  static constexpr size_t p_off = u_stride * NBUF;
  static constexpr size_t fx_off = p_off + align128(sizeof(R) * NVAR * TC);
  static constexpr size_t gy_off = fx_off + align128(sizeof(R) * NVAR * FXN);
  static constexpr size_t total = gy_off + align128(sizeof(R) * NVAR * GYN);
};

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
    const double inv = 1.0 / rho;
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
// conserved states (first order).  A y-interface is solved exactly as the reference solves it:
// the stencil is read with the x and y slots of velocity/momentum and field
// swapped (mhdRotateYToX, mhd_common.hpp:381-391), the x-direction routine
// runs, and the caller stores the flux back through the same swap
// (mhdRotateFluxXToY, :395-405).  Reconstruction is per component and the
// primitive->conserved sums are order-independent, so this equals the
// reference bit for bit.  One copy of the flux code then serves both
// directions, which keeps the kernel's hot loop inside the instruction cache.
//   base   tile index of the cell two steps upwind of the interface
//   stride 1 (x) or HX (y)
//   o1/o2  plane offsets of the normal / first tangential velocity slot
//   o5/o6  plane offsets of the normal / first tangential field slot
template <class Pol, bool HLLD>
__device__ __forceinline__ int face_flux(const typename Pol::R* sP, int base, int stride, int o1, int o2, int o5,
                                         int o6, int muscl,
                                         typename Pol::R ch, const Phys<typename Pol::R>& ph,
                                         typename Pol::R* F) {
  using R = typename Pol::R;
  const int off[NVAR] = {0, o1, o2, 3 * TC, 4 * TC, o5, o6, 7 * TC, 8 * TC};
  R UL[NVAR], UR[NVAR];
  if (muscl) {
    R Pm[NVAR], P0[NVAR], P1[NVAR], P2[NVAR], Pl[NVAR], Pr[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      const R* q = sP + off[k] + base;
      Pm[k] = q[0];
      P0[k] = q[stride];
      P1[k] = q[2 * stride];
      P2[k] = q[3 * stride];
    }
    recon_cell<R>(Pm, P0, P1, Pl, Pr);
    prim9_to_state<R>(Pr, UL, ph);
    recon_cell<R>(P0, P1, P2, Pl, Pr);
    prim9_to_state<R>(Pl, UR, ph);
  } else {  // first order: sP holds the conserved states
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      UL[k] = sP[off[k] + base + stride];
      UR[k] = sP[off[k] + base + 2 * stride];
    }
  }
  return glm_flux<R, 0>(UL, UR, ch, HLLD, F, ph);
}

template <class Pol, int STAGE, bool HLLD>
__global__ void __launch_bounds__(NT, Tune<Pol>::minb)
    stage_kernel(const __grid_constant__ CUtensorMap tmap_in, const StageArgs a) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using TT = typename Pol::TT;
  constexpr int NBUF = Tune<Pol>::nbuf;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw + Smem<Pol>::p_off);
  R* sFx = reinterpret_cast<R*>(smem_raw + Smem<Pol>::fx_off);
  R* sGy = reinterpret_cast<R*>(smem_raw + Smem<Pol>::gy_off);
  __shared__ __align__(8) uint64_t bar[NBUF];
  __shared__ unsigned long long red_speed[NW];
  __shared__ unsigned red_deg[NW], red_np[NW];
  auto ubuf = [&](int b) { return reinterpret_cast<S*>(smem_raw + (size_t)b * Smem<Pol>::u_stride); };

  const int tid = threadIdx.x;
  const bool leader = (blockIdx.x == 0 && tid == 0);
  Ctrl* c = a.ctrl;
  const int p = a.parity;

  // ---- step control: identical decision in every thread of the grid -----
  const double t_raw = c->t[p];
  const long long step = c->step[p];
  const int bad_prev = (STAGE == 1) ? c->bad2 : c->bad1;
  const bool active = !c->halted && !c->err && bad_prev == BAD_NONE && (TT)t_raw < (TT)c->t_end &&
                      step < c->step_limit;
  if (!active) {
    if (leader) {  // carry the slot forward so the other parity also stops
      c->t[p ^ 1] = c->t[p];
      c->step[p ^ 1] = c->step[p];
      c->chbits[p ^ 1] = c->chbits[p];
      if (bad_prev != BAD_NONE || c->err) c->halted = 1;
    }
    return;
  }
  if (tid == 0) prefetch_tmap(&tmap_in);

  const Phys<R> phR = Phys<R>::make(a.gamma, a.tol);
  const Phys<S> phS = Phys<S>::make(a.gamma, a.tol);
  const R ch = vmax((R)__longlong_as_double((long long)c->chbits[p]), (R)1.0e-12);
  const TT t = (TT)t_raw;
  const TT dxT = (TT)a.dx, dyT = (TT)a.dy;
  // max over cells of max(s_x, ch)/dx + max(s_y, ch)/dy equals ch/dx + ch/dy
  // because ch is the maximum of every s_x and s_y (mhd2d_glm_gpu.cu:485-500).
  const TT max_rate = (TT)ch / dxT + (TT)ch / dyT;
  TT dt = (TT)a.cfl / max_rate;
  const TT t_end = (TT)c->t_end;
  if (t + dt > t_end) dt = t_end - t;

  // ---- persistent loop over tiles, next tile's TMA load in flight ---------
  // The CTA owns tiles blockIdx.x, blockIdx.x + gridDim.x, ...  As soon as a
  // tile's cells are recovered into sP, sU is free and the next tile's load
  // is issued, so the load overlaps this tile's flux and update phases.
  const int tiles_x = (a.nx + TX - 1) / TX;
  const int ntiles = tiles_x * ((a.ny + TY - 1) / TY);
  int tile = blockIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  unsigned n_deg = 0, n_np = 0;
  unsigned long long sp_bits = 0;
  const S* u_in = static_cast<const S*>(a.u_in);
  if (tid == 0) {
    for (int b = 0; b < NBUF; b++) mbar_init(&bar[b], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0 && tile < ntiles) {
    mbar_arrive_expect_tx(&bar[0], (uint32_t)Smem<Pol>::u_bytes);
    tma_load_3d(ubuf(0), &tmap_in, &bar[0], (tile % tiles_x) * TX, (tile / tiles_x) * TY, 0);
  }
  for (int it = 0; tile < ntiles; it++, tile += gridDim.x) {
    const int i0 = (tile % tiles_x) * TX, j0 = (tile / tiles_x) * TY;
    const int cb = it % NBUF;                        // buffer of this tile
    const uint32_t par = (uint32_t)(it / NBUF) & 1;  // its mbarrier phase
    S* sU = ubuf(cb);
    const bool got = __syncthreads_and(mbar_wait_bounded(&bar[cb], par, kWaitIters));
    if (!got) {
      if (tid == 0) atomicExch(&c->err, (int)DERR_TMA_TIMEOUT);
      mbar_wait_bounded(&bar[cb], par, kWaitIters);  // let the copy land before leaving
      return;
    }

    // ---- recovery, once per tile cell (halo corners are never used) -------
    // First order needs no primitives: the conserved states are staged.
    for (int q = tid; q < TC; q += NT) {
      const int cx = q % HX, cy = q / HX;
      if ((cx < 2 || cx >= TX + 2) && (cy < 2 || cy >= TY + 2)) continue;
      S U9[NVAR], P9[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) U9[k] = sU[k * TC + q];
      if (a.muscl) {
        recover_cell<Pol>(U9, P9, phS);
      } else {
#pragma unroll
        for (int k = 0; k < NVAR; k++) P9[k] = U9[k];
      }
#pragma unroll
      for (int k = 0; k < NVAR; k++) sP[k * TC + q] = (R)P9[k];
    }
    __syncthreads();
    // The next tile goes into the buffer no thread reads any more: this
    // one (just recovered) or, double-buffered, the previous tile's.
    if (tid == 0 && tile + (int)gridDim.x < ntiles) {
      const int nt = tile + gridDim.x, nb = (it + 1) % NBUF;
      fence_proxy_async_smem();  // order earlier reads of that buffer before the async overwrite
      mbar_arrive_expect_tx(&bar[nb], (uint32_t)Smem<Pol>::u_bytes);
      tma_load_3d(ubuf(nb), &tmap_in, &bar[nb], (nt % tiles_x) * TX, (nt / tiles_x) * TY, 0);
    }

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
      const bool valid = axis ? (j0 + fy <= a.ny && i0 + fx < a.nx) : (i0 + fx <= a.nx && j0 + fy < a.ny);
      if (!valid) continue;
      const int base = axis ? fy * HX + fx + 2 : (fy + 2) * HX + fx;
      const int stride = axis ? HX : 1;
      const int o1 = (axis ? 2 : 1) * TC, o2 = (axis ? 1 : 2) * TC;
      const int o5 = (axis ? 6 : 5) * TC, o6 = (axis ? 5 : 6) * TC;
      R F[NVAR];
      const int st = face_flux<Pol, HLLD>(sP, base, stride, o1, o2, o5, o6, a.muscl, ch, phR, F);
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
        n_deg += (st == HLLD_FALLBACK_DEGENERATE);
        n_np += (st == HLLD_FALLBACK_NONPHYSICAL);
      }
    }
    __syncthreads();

    // ---- divergence, update, checks, store, next-step speed ---------------
    const int tx = lane, ty = warp;
    const int gi = i0 + tx, gj = j0 + ty;
    if (warp < TY && gi < a.nx && gj < a.ny) {
      const size_t gidx = (size_t)(gj + GHOST) * a.pitch + (gi + GHOST);
      S Un[NVAR];
      if constexpr (!Pol::kMixed) {
        // Reference order (mhd2d_glm_gpu.cu:282-285, :299, :316-317).
        const R damping = ch / vmax((R)a.alpha, (R)1.0e-12);
#pragma unroll
        for (int k = 0; k < NVAR; k++) {
          const R uin = NBUF == 2 ? sU[k * TC + (ty + 2) * HX + tx + 2] : u_in[(size_t)k * a.plane + gidx];
          R rhs = -(sFx[k * FXN + ty * (TX + 1) + tx + 1] - sFx[k * FXN + ty * (TX + 1) + tx]) / (R)dxT -
                  (sGy[k * GYN + (ty + 1) * TX + tx] - sGy[k * GYN + ty * TX + tx]) / (R)dyT;
          if (k == PSI) rhs -= damping * uin;
          if (STAGE == 1) {
            Un[k] = uin + (R)dt * rhs;
          } else {
            const S uold = static_cast<const S*>(a.u_old)[(size_t)k * a.plane + gidx];
            Un[k] = (R)0.5 * uold + (R)0.5 * (uin + (R)dt * rhs);
          }
        }
      } else {
        // Binary32 fluxes and their differences, binary64 scaling and
        // accumulation.
        const double damping = (double)ch / fmax(a.alpha, 1.0e-12);
        const double inv_dx = 1.0 / a.dx, inv_dy = 1.0 / a.dy;
#pragma unroll
        for (int k = 0; k < NVAR; k++) {
          const double uin = NBUF == 2 ? sU[k * TC + (ty + 2) * HX + tx + 2] : u_in[(size_t)k * a.plane + gidx];
          const float dfx = sFx[k * FXN + ty * (TX + 1) + tx + 1] - sFx[k * FXN + ty * (TX + 1) + tx];
          const float dgy = sGy[k * GYN + (ty + 1) * TX + tx] - sGy[k * GYN + ty * TX + tx];
          double rhs = -(double)dfx * inv_dx - (double)dgy * inv_dy;
          if (k == PSI) rhs -= damping * uin;
          if (STAGE == 1) {
            Un[k] = uin + (double)dt * rhs;
          } else {
            const double uold = static_cast<const double*>(a.u_old)[(size_t)k * a.plane + gidx];
            Un[k] = 0.5 * uold + 0.5 * (uin + (double)dt * rhs);
          }
        }
      }
      // stateIsUsable (mhd2d_glm_gpu.cu:74-79); its recovery doubles as the
      // recovery of the next step's CFL speed (speedKernel, :171-195).
      S P9[NVAR];
      recover_cell<Pol>(Un, P9, phS);
      if (!(Un[RHO] > rho_floor<S>()) || !prim9_usable<S>(P9)) {
        atomicMin(STAGE == 1 ? &c->bad1 : &c->bad2, gj * a.nx + gi);
        c->bad_step = step;
      }
      store_cell<S>(static_cast<S*>(a.u_out), a.plane, a.pitch, gi, gj, a.nx, a.ny, a.bc, Un);
      if (STAGE == 2) {
        R Pr[NVAR];
#pragma unroll
        for (int k = 0; k < NVAR; k++) Pr[k] = (R)P9[k];
        const unsigned long long b = speed_bits((double)cell_speed<R>(Pr, phR));
        sp_bits = b > sp_bits ? b : sp_bits;
      }
    }
  }

  // ---- block reductions, one atomic per CTA ----------------------------------
  if (HLLD) {
    const unsigned d = warp_sum_u32(n_deg), np = warp_sum_u32(n_np);
    if (lane == 0) {
      red_deg[warp] = d;
      red_np[warp] = np;
    }
  }
  if (STAGE == 2) {
    const unsigned long long m = warp_max_u64(sp_bits);
    if (lane == 0) red_speed[warp] = m;
  }
  __syncthreads();
  if (tid == 0) {
    if (HLLD) {
      unsigned d = 0, np = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) {
        d += red_deg[w];
        np += red_np[w];
      }
      if (d) atomicAdd(&c->degenerate, (unsigned long long)d);
      if (np) atomicAdd(&c->nonphysical, (unsigned long long)np);
    }
    if (STAGE == 2) {
      unsigned long long m = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) m = red_speed[w] > m ? red_speed[w] : m;
      if (m) atomicMax(&c->chbits[p ^ 1], m);
    }
  }
  if (leader) {
    atomicAdd(&c->active_stage_launches, 1ull);
    if (STAGE == 1) {
      c->chbits[p ^ 1] = 0ull;  // stage 2 of this step accumulates into it
    } else {
      c->t[p ^ 1] = (double)(t + dt);
      c->step[p ^ 1] = step + 1;
      c->last_ch = (double)ch;
      c->last_dt = (double)dt;
    }
  }
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
    const unsigned long long b = speed_bits((double)cell_speed<R>(Pr, phR));
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
