// euler_kernels.cu -- the Euler sibling on sm_100a: one fused kernel per
// dimensionally split 2D step (both sweeps of the reference's
// MUSCL-Hancock + HLLC / HLL step, src/euler/riemann2d_cpu.cpp:295-309, in
// one pass over HBM), its initial max-speed reduction, and a one-CTA kernel
// that runs a whole 1D Riemann problem (src/euler/riemann1d_cpu.cpp:95-196).
//
// 2D step kernel.  A CTA of 512 threads owns a 32 x TY tile of output cells
// (TY = 16 or 12 fp64, 32 fp32).  It loads the conservative state of a
// (TY + 4) x 36 region around it (2 cells of halo,
// indices clamped at the walls: the reference's transmissive ghost copies,
// riemann2d_cpu.cpp:160-182), and runs the first sweep on the part of the
// region the second sweep needs (all rows for x-then-y, all columns for
// y-then-x), then the second sweep on the tile; each sweep is
// reconstruction + Hancock of every cell's two faces, one flux per
// interface, and the conservative update, staged in shared memory.  The
// order alternates with the step count (even: x then y).  The next step's
// max signal speeds come from the epilogue (one atomicMax per CTA), so the
// time step never needs a separate pass.
//
// Compiled twice (see Makefile): PMHD_EKNS=exact with -fmad=false (bit
// parity with the reference CPU build) and PMHD_EKNS=fast (contraction,
// approximate binary32 division / square root).
#include <cuda_runtime.h>

#include <cstdint>

#include "euler/euler_api.h"
#include "pmhd/euler.hpp"

#ifndef PMHD_EKNS
#error "PMHD_EKNS must name the build flavour (exact or fast)"
#endif

namespace pmhd {
namespace euler {
namespace PMHD_EKNS {

namespace {

// Point arithmetic of the build: the reference's expressions (exact build,
// bit parity) or the performance forms (fast build, PMHD_EULER_FAST).
#if PMHD_EULER_FAST
namespace pf = ::pmhd::euler::fastform;
template <class T>
__device__ __forceinline__ void k_c2p(const T U[4], T W[4]) {
  pf::cons_to_prim(U, W);
}
template <class T, int NI, int TI>
__device__ __forceinline__ void k_hancock_pair(const T l[4], const T r[4], T lh[4], T rh[4], T fac) {
  pf::hancock_pair<T, NI, TI>(l, r, lh, rh, fac);
}
template <class T, int NI, int TI, bool HLL>
__device__ __forceinline__ void k_flux(const T a[4], const T b[4], T f[4]) {
  if (HLL)
    pf::hll_flux<T, NI, TI>(a, b, f);
  else
    pf::hllc_flux<T, NI, TI>(a, b, f);
}
template <class T>
__device__ __forceinline__ void k_speeds(const T U[4], T& sx, T& sy) {
  pf::cell_speeds(U, sx, sy);
}
#else
template <class T>
__device__ __forceinline__ void k_c2p(const T U[4], T W[4]) {
  cons_to_prim(U, W);
}
template <class T, int NI, int TI>
__device__ __forceinline__ void k_hancock_pair(const T l[4], const T r[4], T lh[4], T rh[4], T fac) {
  hancock<T, NI, TI>(l, l, r, lh, fac);
  hancock<T, NI, TI>(r, l, r, rh, fac);
}
template <class T, int NI, int TI, bool HLL>
__device__ __forceinline__ void k_flux(const T a[4], const T b[4], T f[4]) {
  if (HLL)
    hll_flux<T, NI, TI>(a, b, f);
  else
    hllc_flux<T, NI, TI>(a, b, f);
}
// riemann2d_cpu.cpp:200-210: |u| + c, |v| + c from the primitives.
template <class T>
__device__ __forceinline__ void k_speeds(const T U[4], T& sx, T& sy) {
  T W[4];
  cons_to_prim(U, W);
  const T cs = sound_speed(W[3], W[0]);
  sx = std::fabs(W[1]) + cs;
  sy = std::fabs(W[2]) + cs;
}
#endif

constexpr int NV = 4;

constexpr int TW = 32;  // tile width (cells)
constexpr int RW = TW + 4;

__device__ __forceinline__ unsigned long long speed_bits(double v) {
  return v > 0.0 ? (unsigned long long)__double_as_longlong(v) : 0ull;
}
__device__ __forceinline__ double bits_speed(unsigned long long b) { return __longlong_as_double((long long)b); }

__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

template <class T, int TY>
struct Tile {
  static constexpr int RH = TY + 4;
  static constexpr int N = RH * RW;  // cells of the region
  T U[NV][N];
  T W[NV][N];   // primitives
  T HL[NV][N];  // Hancock-evolved left (lower) face of each cell; then the interface fluxes
  T HR[NV][N];  // ... right (upper) face
};

// Where the last sweep's updated cells go: the output state (interior cells
// only) and the running maxima of the next step's signal speeds.
template <class T>
struct TileOut {
  T* __restrict__ u;
  long long plane;
  int pitch, i0, j0, nx, ny;
  unsigned long long bx, by;
};

// One sweep over the region cells [r0, r1) x [c0, c1) that are updated;
// DIR 0 = x (along c), 1 = y (along r).  Needs W valid on the cells within
// 2 of them along DIR.  The update phase also does what follows it: the
// first sweep (LAST = false) forms the primitives of each updated cell for
// the second sweep's reconstruction; the last one stores the tile and
// reduces the signal speeds.  (Region rows or columns beyond a wall hold
// copies of the edge cells, and a sweep along them gives the edge cell's
// result bit for bit, so their primitives are the refreshed ghost copies of
// the reference's applyBC between the sweeps.)
template <class T, int TY, int DIR, bool HLL, bool LAST>
__device__ __forceinline__ void sweep(Tile<T, TY>& s, int r0, int r1, int c0, int c1, T fac, T ratio,
                                      TileOut<T>& out) {
  constexpr int NI = DIR == 0 ? 1 : 2, TI = DIR == 0 ? 2 : 1;
  const int step = DIR == 0 ? 1 : RW;
  // Hancock faces of the cells one beyond the updated ones along DIR.
  const int hr0 = DIR == 1 ? r0 - 1 : r0, hr1 = DIR == 1 ? r1 + 1 : r1;
  const int hc0 = DIR == 0 ? c0 - 1 : c0, hc1 = DIR == 0 ? c1 + 1 : c1;
  const int hw = hc1 - hc0, hn = (hr1 - hr0) * hw;
  for (int q = threadIdx.x; q < hn; q += blockDim.x) {
    const int id = (hr0 + q / hw) * RW + hc0 + q % hw;
    T l[NV], r[NV], lh[NV], rh[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) muscl_recon(s.W[k][id - step], s.W[k][id], s.W[k][id + step], l[k], r[k]);
    k_hancock_pair<T, NI, TI>(l, r, lh, rh, fac);
#pragma unroll
    for (int k = 0; k < NV; k++) {
      s.HL[k][id] = lh[k];
      s.HR[k][id] = rh[k];
    }
  }
  __syncthreads();
  // Interface fluxes: F at cell id = flux between id - step and id, for the
  // updated cells and the one past them; stored over HL[id], which only this
  // thread reads.
  const int fr1 = DIR == 1 ? r1 + 1 : r1, fc1 = DIR == 0 ? c1 + 1 : c1;
  const int fw = fc1 - c0, fn = (fr1 - r0) * fw;
  for (int q = threadIdx.x; q < fn; q += blockDim.x) {
    const int id = (r0 + q / fw) * RW + c0 + q % fw;
    T a[NV], b[NV], f[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      a[k] = s.HR[k][id - step];
      b[k] = s.HL[k][id];
    }
    k_flux<T, NI, TI, HLL>(a, b, f);
#pragma unroll
    for (int k = 0; k < NV; k++) s.HL[k][id] = f[k];
  }
  __syncthreads();
  const int uw = c1 - c0, un = (r1 - r0) * uw;
  for (int q = threadIdx.x; q < un; q += blockDim.x) {
    const int r = r0 + q / uw, c = c0 + q % uw, id = r * RW + c;
    T U4[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) U4[k] = s.U[k][id] - ratio * (s.HL[k][id + step] - s.HL[k][id]);
    if (!LAST) {
      T W4[NV];
      k_c2p(U4, W4);
#pragma unroll
      for (int k = 0; k < NV; k++) {
        s.U[k][id] = U4[k];
        s.W[k][id] = W4[k];
      }
    } else {
      const int i = out.i0 + c - 2, j = out.j0 + r - 2;
      if (i < out.nx && j < out.ny) {
#pragma unroll
        for (int k = 0; k < NV; k++) out.u[k * out.plane + (long long)j * out.pitch + i] = U4[k];
        T vx, vy;
        k_speeds(U4, vx, vy);
        const unsigned long long sx = speed_bits((double)vx), sy = speed_bits((double)vy);
        out.bx = sx > out.bx ? sx : out.bx;
        out.by = sy > out.by ? sy : out.by;
      }
    }
  }
  if (!LAST) __syncthreads();
}

// Registers: 64 per thread for 1024 / NT resident CTAs (the shared-memory
// limit of the tile shapes below).
template <class T, int TY, int NT, int MINB, bool HLL>
__global__ void __launch_bounds__(NT, MINB) step_kernel(const T* __restrict__ uin, T* __restrict__ uout, int nx, int ny,
                                                   int pitch, long long plane, T dx, T dy, T cfl, EulerCtrl* ctrl,
                                                   int p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Tile<T, TY>& s = *reinterpret_cast<Tile<T, TY>*>(smem_raw);
  constexpr int RH = TY + 4;
  const int i0 = blockIdx.x * TW, j0 = blockIdx.y * TY;
  // Step control (every CTA reads the same slots; block (0,0) writes the
  // other parity and the speed slot two steps ahead).
  const T t = (T)ctrl->t[p];
  const long long n = ctrl->step[p];
  // t and t + dt are values of type T, so their tests against t_end are
  // exact in binary64 whichever type t_end has.
  bool active = !ctrl->stop && (double)t < ctrl->t_end && n < ctrl->step_limit;
  T dt = (T)0;
  if (active) {
    const T mx = (T)bits_speed(ctrl->sx[n % 3]), my = (T)bits_speed(ctrl->sy[n % 3]);
    const T m = vmin(dx / mx, dy / my);
    dt = ctrl->wide_time ? (T)(ctrl->cfl * (double)m) : cfl * m;
    if ((double)(T)(t + dt) > ctrl->t_end) dt = ctrl->wide_time ? (T)(ctrl->t_end - (double)t) : (T)ctrl->t_end - t;
    if (!(dt > (T)0.0) || t + dt == t) active = false;  // riemann2d_cpu.cpp:298, euler2d_cpu.cpp:309
  }
  const bool leader = blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0;
  if (!active) {
    if (leader) {
      ctrl->t[p ^ 1] = ctrl->t[p];
      ctrl->step[p ^ 1] = n;
      if (!((double)t < ctrl->t_end) || n >= ctrl->step_limit) {
      } else {
        ctrl->stop = 1;
      }
    }
    // Carry the state to the output buffer.
    for (int q = threadIdx.x; q < TW * TY; q += blockDim.x) {
      const int i = i0 + q % TW, j = j0 + q / TW;
      if (i < nx && j < ny)
#pragma unroll
        for (int k = 0; k < NV; k++) uout[k * plane + (long long)j * pitch + i] = uin[k * plane + (long long)j * pitch + i];
    }
    return;
  }
  if (leader) {
    ctrl->t[p ^ 1] = (double)(t + dt);
    ctrl->step[p ^ 1] = n + 1;
    ctrl->sx[(n + 2) % 3] = 0ull;
    ctrl->sy[(n + 2) % 3] = 0ull;
  }
  // Region load with wall clamping, and the primitives of every region cell
  // (same thread, so no barrier between them).  (Measured: asynchronous
  // global -> shared copies of the region, issued ahead of the step-control
  // reads, were 11 % slower in binary64 and no faster in binary32.)
  for (int q = threadIdx.x; q < RH * RW; q += blockDim.x) {
    const int r = q / RW, c = q % RW;
    int j = j0 - 2 + r, i = i0 - 2 + c;
    j = j < 0 ? 0 : (j >= ny ? ny - 1 : j);
    i = i < 0 ? 0 : (i >= nx ? nx - 1 : i);
    T U4[NV], W4[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      U4[k] = uin[k * plane + (long long)j * pitch + i];
      s.U[k][q] = U4[k];
    }
    k_c2p(U4, W4);
#pragma unroll
    for (int k = 0; k < NV; k++) s.W[k][q] = W4[k];
  }
  __syncthreads();
  const T facx = (T)0.5 * dt / dx, facy = (T)0.5 * dt / dy, rx = dt / dx, ry = dt / dy;
  TileOut<T> out{uout, plane, pitch, i0, j0, nx, ny, 0ull, 0ull};
  if (n % 2 == 0) {
    // x sweep on every region row (columns 2..TW+1), then y sweep on the tile.
    sweep<T, TY, 0, HLL, false>(s, 0, RH, 2, TW + 2, facx, rx, out);
    sweep<T, TY, 1, HLL, true>(s, 2, TY + 2, 2, TW + 2, facy, ry, out);
  } else {
    sweep<T, TY, 1, HLL, false>(s, 2, TY + 2, 0, RW, facy, ry, out);
    sweep<T, TY, 0, HLL, true>(s, 2, TY + 2, 2, TW + 2, facx, rx, out);
  }
  unsigned long long bx = out.bx, by = out.by;
  bx = warp_max(bx);
  by = warp_max(by);
  if ((threadIdx.x & 31) == 0) {
    if (bx) atomicMax(&ctrl->sx[(n + 1) % 3], bx);
    if (by) atomicMax(&ctrl->sy[(n + 1) % 3], by);
  }
}

template <class T>
__global__ void __launch_bounds__(256) speed_kernel(const T* __restrict__ u, int nx, int ny, int pitch,
                                                    long long plane, EulerCtrl* ctrl, int slot) {
  unsigned long long bx = 0, by = 0;
  for (long long q = blockIdx.x * 256LL + threadIdx.x; q < (long long)nx * ny; q += (long long)gridDim.x * 256) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    T U4[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) U4[k] = u[k * plane + (long long)j * pitch + i];
    T vx, vy;
    k_speeds(U4, vx, vy);
    const unsigned long long sx = speed_bits((double)vx), sy = speed_bits((double)vy);
    bx = sx > bx ? sx : bx;
    by = sy > by ? sy : by;
  }
  bx = warp_max(bx);
  by = warp_max(by);
  if ((threadIdx.x & 31) == 0) {
    if (bx) atomicMax(&ctrl->sx[slot], bx);
    if (by) atomicMax(&ctrl->sy[slot], by);
  }
}

// The whole 1D run in one CTA (riemann1d_cpu.cpp:95-196); arrays in global
// memory (tiny, L1/L2-resident).  u = [3][N+4] with ghosts, f = [3][N+4].
template <class T, bool HLL>
__global__ void __launch_bounds__(1024) riemann1d_kernel(T* __restrict__ u, T* __restrict__ f, int N, T t_end,
                                                         long long max_iters, double* __restrict__ out_t,
                                                         long long* __restrict__ out_steps, int* __restrict__ err) {
  const int GH = 2, TOT = N + 4;
  T* U0 = u;
  T* U1 = u + TOT;
  T* U2 = u + 2 * TOT;
  T* F0 = f;
  T* F1 = f + TOT;
  T* F2 = f + 2 * TOT;
  const T DX = ((T)1.0 - (T)0.0) / (T)N, CFL = (T)0.8;
  __shared__ unsigned long long red[32];
  T t = (T)0.0;
  long long step = 0;
  while (t < t_end) {
    if (step >= max_iters) {  // the reference has no such limit; a GPU loop must
      if (threadIdx.x == 0) *err = 1;
      break;
    }
    if (threadIdx.x < GH) {
      const int g = threadIdx.x, ir = TOT - 1 - g, in = TOT - 1 - GH;
      U0[g] = U0[GH];
      U1[g] = U1[GH];
      U2[g] = U2[GH];
      U0[ir] = U0[in];
      U1[ir] = U1[in];
      U2[ir] = U2[in];
    }
    unsigned long long m = 0;
    for (int i = GH + threadIdx.x; i < N + GH; i += blockDim.x) {
      const unsigned long long b = speed_bits((double)speed_1d(U0[i], U1[i], U2[i]));
      m = b > m ? b : m;
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = red[w] > m ? red[w] : m;
    const T ms = (T)bits_speed(m);
    T dt = CFL * DX / ms;
    if (t + dt > t_end) dt = t_end - t;
    const T fac = (T)0.5 * dt / DX;
    for (int i = GH - 1 + threadIdx.x; i < N + GH; i += blockDim.x) {
      T Wq[4][3];
#pragma unroll
      for (int q = 0; q < 4; q++) cons_to_prim_1d(U0[i - 1 + q], U1[i - 1 + q], U2[i - 1 + q], Wq[q]);
      T Lf[3], Rf[3], L0[3], R0[3], Lh[3], Oh[3], fl[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        muscl_recon(Wq[0][k], Wq[1][k], Wq[2][k], Lf[k], Rf[k]);
        muscl_recon(Wq[1][k], Wq[2][k], Wq[3][k], L0[k], R0[k]);
      }
      hancock_1d(Rf, Lf, Rf, Lh, fac);
      hancock_1d(L0, L0, R0, Oh, fac);
      if (HLL)
        hll_flux_1d(Lh, Oh, fl);
      else
        hllc_flux_1d(Lh, Oh, fl);
      F0[i] = fl[0];
      F1[i] = fl[1];
      F2[i] = fl[2];
    }
    __syncthreads();
    const T ratio = dt / DX;
    for (int i = GH + threadIdx.x; i < N + GH; i += blockDim.x) {
      U0[i] -= ratio * (F0[i] - F0[i - 1]);
      U1[i] -= ratio * (F1[i] - F1[i - 1]);
      U2[i] -= ratio * (F2[i] - F2[i - 1]);
    }
    __syncthreads();
    t += dt;
    step++;
  }
  if (threadIdx.x == 0) {
    *out_t = (double)t;
    *out_steps = step;
  }
}

template <class T, int TY, int NT, int MINB, bool HLL>
cudaError_t launch_step(const void* uin, void* uout, int nx, int ny, int pitch, long long plane, double dx, double dy,
                        double cfl, EulerCtrl* ctrl, int p, cudaStream_t s) {
  auto k = step_kernel<T, TY, NT, MINB, HLL>;  // shared-memory limit set by prepare()
  const size_t smem = sizeof(Tile<T, TY>);
  const dim3 grid((nx + TW - 1) / TW, (ny + TY - 1) / TY);
  k<<<grid, NT, smem, s>>>(static_cast<const T*>(uin), static_cast<T*>(uout), nx, ny, pitch, plane, (T)dx, (T)dy,
                           (T)cfl, ctrl, p);
  return cudaGetLastError();
}

template <class T, int TY, int NT, int MINB>
cudaError_t allow_smem() {
  cudaError_t e = cudaFuncSetAttribute(step_kernel<T, TY, NT, MINB, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Tile<T, TY>));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(step_kernel<T, TY, NT, MINB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(Tile<T, TY>));
  return e;
}

template <class T, int TY, int NT, int MINB>
cudaError_t launch_any(int hll, const void* uin, void* uout, int nx, int ny, int pitch, long long plane, double dx,
                       double dy, double cfl, EulerCtrl* ctrl, int p, cudaStream_t s) {
  return hll ? launch_step<T, TY, NT, MINB, true>(uin, uout, nx, ny, pitch, plane, dx, dy, cfl, ctrl, p, s)
             : launch_step<T, TY, NT, MINB, false>(uin, uout, nx, ny, pitch, plane, dx, dy, cfl, ctrl, p, s);
}

}  // namespace

// Tile shapes (measured at 4096^2, performance build): 32 x 16 cells for fp64
// and 32 x 32 for fp32, 512 threads, two CTAs (32 warps) per SM at 64
// registers (shared memory: 92 KB / 83 KB for the four region arrays).
// Against 32 x 8 (fp64) / 32 x 16 (fp32) tiles of 256 threads at four CTAs
// per SM: the same occupancy with less halo re-work and half the block
// barriers per cell (fp64 +15 %, fp32 +17 %).  Measured and not kept at
// 4096^2: fp64 32 x 12 (-6 %), fp64 32 x 10 with 320 threads at three CTAs
// per SM (-18 %), fp32 32 x 28 / 32 x 24 at three CTAs per SM (-13 % / -20 %).  fp64 grids whose 32 x 16 tiling fills less than one wave
// of two CTAs per SM take 32 x 12 tiles (the 500 x 197 shock-bubble: 46.1 ->
// 41.3 ms).
constexpr int kThreads = 512;

cudaError_t prepare() {
  cudaError_t e = allow_smem<double, 16, kThreads, 2>();
  if (e == cudaSuccess) e = allow_smem<double, 12, kThreads, 2>();
  if (e == cudaSuccess) e = allow_smem<float, 32, kThreads, 2>();
  return e;
}

cudaError_t step2d(int fp32, int hll, const void* uin, void* uout, int nx, int ny, int pitch, long long plane,
                   double dx, double dy, double cfl, EulerCtrl* ctrl, int p, cudaStream_t s) {
  if (fp32) return launch_any<float, 32, kThreads, 2>(hll, uin, uout, nx, ny, pitch, plane, dx, dy, cfl, ctrl, p, s);
  const long long tiles16 = (long long)((nx + TW - 1) / TW) * ((ny + 15) / 16);
  if (tiles16 < 2 * 148)
    return launch_any<double, 12, kThreads, 2>(hll, uin, uout, nx, ny, pitch, plane, dx, dy, cfl, ctrl, p, s);
  return launch_any<double, 16, kThreads, 2>(hll, uin, uout, nx, ny, pitch, plane, dx, dy, cfl, ctrl, p, s);
}

cudaError_t speed2d(int fp32, const void* u, int nx, int ny, int pitch, long long plane, EulerCtrl* ctrl, int slot,
                    cudaStream_t s) {
  const long long n = (long long)nx * ny;
  long long g = (n + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  if (fp32)
    speed_kernel<float><<<(unsigned)g, 256, 0, s>>>(static_cast<const float*>(u), nx, ny, pitch, plane, ctrl, slot);
  else
    speed_kernel<double><<<(unsigned)g, 256, 0, s>>>(static_cast<const double*>(u), nx, ny, pitch, plane, ctrl, slot);
  return cudaGetLastError();
}

cudaError_t run1d(int fp32, int hll, void* u, void* f, int n, double t_end, long long max_iters, double* out_t,
                  long long* out_steps, int* err, cudaStream_t s) {
  if (fp32) {
    if (hll)
      riemann1d_kernel<float, true><<<1, 1024, 0, s>>>(static_cast<float*>(u), static_cast<float*>(f), n, (float)t_end,
                                                       max_iters, out_t, out_steps, err);
    else
      riemann1d_kernel<float, false><<<1, 1024, 0, s>>>(static_cast<float*>(u), static_cast<float*>(f), n,
                                                        (float)t_end, max_iters, out_t, out_steps, err);
  } else {
    if (hll)
      riemann1d_kernel<double, true><<<1, 1024, 0, s>>>(static_cast<double*>(u), static_cast<double*>(f), n, t_end,
                                                        max_iters, out_t, out_steps, err);
    else
      riemann1d_kernel<double, false><<<1, 1024, 0, s>>>(static_cast<double*>(u), static_cast<double*>(f), n, t_end,
                                                         max_iters, out_t, out_steps, err);
  }
  return cudaGetLastError();
}

}  // namespace PMHD_EKNS
}  // namespace euler
}  // namespace pmhd
