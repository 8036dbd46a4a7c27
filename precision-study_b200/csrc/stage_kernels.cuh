// stage_kernels.cuh -- the fused SSPRK2 stage kernel and its helpers.
//
// One launch performs one SSPRK2 stage of the 2D ideal-MHD + mixed-GLM
// finite-volume step for the whole grid (reference: the kernel chain
// bcX/bcY -> fluxX -> fluxY -> rhs -> stage1/stage2 of
// src/mhd/mhd2d_glm_gpu.cu:141-321, plus speedKernel/rateKernel :171-222
// for the next step's CFL reduction).  Per CTA and 32 x 8 output tile:
//
//   1. TMA loads the stage input tile with its 2-cell halo, all nine SoA
//      planes, into shared memory (one 3-D box, no multicast).
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
//   PolMixed storage, recovery, flux divergence and update in binary64;
//            reconstruction, Riemann flux and CFL speed in binary32
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

constexpr int TX = 32, TY = 8;            // output tile
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

template <class Pol>
struct Smem {
  using S = typename Pol::S;
  using R = typename Pol::R;
  static constexpr size_t u_bytes = sizeof(S) * NVAR * TC;  // TMA box size
  static constexpr size_t p_off = align128(u_bytes);
  static constexpr size_t fx_off = p_off + align128(sizeof(R) * NVAR * TC);
  static constexpr size_t gy_off = fx_off + align128(sizeof(R) * NVAR * FXN);
  static constexpr size_t total = gy_off + align128(sizeof(R) * NVAR * GYN);
};

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

// Face states and Riemann flux of one interface.  `base` is the tile index
// of the cell two steps upwind of the interface; `stride` is 1 (x) or HX (y).
template <class Pol, int AX, bool HLLD>
__device__ __forceinline__ int face_flux(const typename Pol::S* sU, const typename Pol::R* sP, int base,
                                         int stride, int muscl, typename Pol::R ch,
                                         const Phys<typename Pol::R>& ph, typename Pol::R* F) {
  using R = typename Pol::R;
  R UL[NVAR], UR[NVAR];
  if (muscl) {
    R Pm[NVAR], P0[NVAR], P1[NVAR], P2[NVAR], Pl[NVAR], Pr[NVAR];
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      const R* q = sP + k * TC + base;
      Pm[k] = q[0];
      P0[k] = q[stride];
      P1[k] = q[2 * stride];
      P2[k] = q[3 * stride];
    }
    recon_cell<R>(Pm, P0, P1, Pl, Pr);
    prim9_to_state<R>(Pr, UL, ph);
    recon_cell<R>(P0, P1, P2, Pl, Pr);
    prim9_to_state<R>(Pl, UR, ph);
  } else {
#pragma unroll
    for (int k = 0; k < NVAR; k++) {
      UL[k] = (R)sU[k * TC + base + stride];
      UR[k] = (R)sU[k * TC + base + 2 * stride];
    }
  }
  return glm_flux<R, AX>(UL, UR, ch, HLLD, F, ph);
}

// Resident CTAs per SM the register allocation is sized for: two for the
// binary32-flux policies; one for binary64, whose HLLD needs more registers
// than two resident CTAs leave per thread (spilling costs more than the lost
// occupancy).
template <class Pol>
struct StageMinBlocks {
  static constexpr int value = sizeof(typename Pol::R) == 8 ? 1 : 2;
};

template <class Pol, int STAGE, bool HLLD>
__global__ void __launch_bounds__(NT, StageMinBlocks<Pol>::value)
    stage_kernel(const __grid_constant__ CUtensorMap tmap_in, const StageArgs a) {
  using S = typename Pol::S;
  using R = typename Pol::R;
  using TT = typename Pol::TT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S* sU = reinterpret_cast<S*>(smem_raw);
  R* sP = reinterpret_cast<R*>(smem_raw + Smem<Pol>::p_off);
  R* sFx = reinterpret_cast<R*>(smem_raw + Smem<Pol>::fx_off);
  R* sGy = reinterpret_cast<R*>(smem_raw + Smem<Pol>::gy_off);
  __shared__ __align__(8) uint64_t bar;
  __shared__ unsigned long long red_speed[NW];
  __shared__ unsigned red_deg[NW], red_np[NW];

  const int tid = threadIdx.x;
  const bool leader = (blockIdx.x == 0 && blockIdx.y == 0 && tid == 0);
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

  // ---- 1. TMA tile load ---------------------------------------------------
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar, (uint32_t)Smem<Pol>::u_bytes);
    tma_load_3d(sU, &tmap_in, &bar, i0, j0, 0);
  }
  const bool got = __syncthreads_and(mbar_wait_bounded(&bar, 0, kWaitIters));
  if (!got) {
    if (tid == 0) atomicExch(&c->err, (int)DERR_TMA_TIMEOUT);
    mbar_wait_bounded(&bar, 0, kWaitIters);  // let the copy land before leaving
    return;
  }

  // ---- 2. recovery, once per tile cell (halo corners are never used) -------
  if (a.muscl) {
    for (int q = tid; q < TC; q += NT) {
      const int cx = q % HX, cy = q / HX;
      if ((cx < 2 || cx >= TX + 2) && (cy < 2 || cy >= TY + 2)) continue;
      S U9[NVAR], P9[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) U9[k] = sU[k * TC + q];
      state_to_prim9<S>(U9, P9, phS);
#pragma unroll
      for (int k = 0; k < NVAR; k++) sP[k * TC + q] = (R)P9[k];
    }
    __syncthreads();
  }

  // ---- 3. interface fluxes --------------------------------------------------
  // Warps 0..TY-1 own one tile row each: lane tx computes the x-interface to
  // the right of cell (tx, ty), then the y-interface above it.  The last warp
  // computes the tile's bottom row of y-interfaces, then its left column of
  // x-interfaces.  Every warp runs two rounds of one direction each, so no
  // warp lags at the barrier and no warp mixes the two code paths.
  const int warp = tid >> 5, lane = tid & 31;
  unsigned n_deg = 0, n_np = 0;
  auto x_face = [&](int fx, int fy) {
    const int gi = i0 + fx;  // interface between cells gi-1 and gi
    if (gi > a.nx || j0 + fy >= a.ny) return;
    R F[NVAR];
    const int st = face_flux<Pol, 0, HLLD>(sU, sP, (fy + 2) * HX + fx, 1, a.muscl, ch, phR, F);
#pragma unroll
    for (int k = 0; k < NVAR; k++) sFx[k * FXN + fy * (TX + 1) + fx] = F[k];
    if (HLLD && (fx >= 1 || i0 == 0)) {
      n_deg += (st == HLLD_FALLBACK_DEGENERATE);
      n_np += (st == HLLD_FALLBACK_NONPHYSICAL);
    }
  };
  auto y_face = [&](int fx, int fy) {
    const int gj = j0 + fy;  // interface between rows gj-1 and gj
    if (gj > a.ny || i0 + fx >= a.nx) return;
    R F[NVAR];
    const int st = face_flux<Pol, 1, HLLD>(sU, sP, fy * HX + fx + 2, HX, a.muscl, ch, phR, F);
#pragma unroll
    for (int k = 0; k < NVAR; k++) sGy[k * GYN + fy * TX + fx] = F[k];
    if (HLLD && (fy >= 1 || j0 == 0)) {
      n_deg += (st == HLLD_FALLBACK_DEGENERATE);
      n_np += (st == HLLD_FALLBACK_NONPHYSICAL);
    }
  };
  if (warp < TY) {
    x_face(lane + 1, warp);
    y_face(lane, warp + 1);
  } else {
    y_face(lane, 0);
    if (lane < TY) x_face(0, lane);
  }
  __syncthreads();

  // ---- 4. divergence, update, checks, store, next-step speed ---------------
  const int tx = lane, ty = warp;
  const int gi = i0 + tx, gj = j0 + ty;
  unsigned long long sp_bits = 0;
  if (warp < TY && gi < a.nx && gj < a.ny) {
    const int lc = (ty + 2) * HX + (tx + 2);
    const size_t gidx = (size_t)(gj + GHOST) * a.pitch + (gi + GHOST);
    S Un[NVAR];
    if constexpr (!Pol::kMixed) {
      // Reference order (mhd2d_glm_gpu.cu:282-285, :299, :316-317).
      const R damping = ch / vmax((R)a.alpha, (R)1.0e-12);
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        const R uin = sU[k * TC + lc];
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
      // Binary32 fluxes, binary64 divergence and accumulation.
      const double damping = (double)ch / fmax(a.alpha, 1.0e-12);
      const double inv_dx = 1.0 / a.dx, inv_dy = 1.0 / a.dy;
#pragma unroll
      for (int k = 0; k < NVAR; k++) {
        const double uin = sU[k * TC + lc];
        const double dfx = (double)sFx[k * FXN + ty * (TX + 1) + tx + 1] - (double)sFx[k * FXN + ty * (TX + 1) + tx];
        const double dgy = (double)sGy[k * GYN + (ty + 1) * TX + tx] - (double)sGy[k * GYN + ty * TX + tx];
        double rhs = -dfx * inv_dx - dgy * inv_dy;
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
    state_to_prim9<S>(Un, P9, phS);
    if (!(Un[RHO] > rho_floor<S>()) || !prim9_usable<S>(P9)) {
      atomicMin(STAGE == 1 ? &c->bad1 : &c->bad2, gj * a.nx + gi);
      c->bad_step = step;
    }
    store_cell<S>(static_cast<S*>(a.u_out), a.plane, a.pitch, gi, gj, a.nx, a.ny, a.bc, Un);
    if (STAGE == 2) {
      R Pr[NVAR];
#pragma unroll
      for (int k = 0; k < NVAR; k++) Pr[k] = (R)P9[k];
      sp_bits = speed_bits((double)cell_speed<R>(Pr, phR));
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
    state_to_prim9<S>(U9, P9, phS);
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
