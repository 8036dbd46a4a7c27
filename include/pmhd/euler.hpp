// euler.hpp -- per-point numerics of the Euler sibling (gamma = 1.4): sound
// speed, primitive <-> conservative, MUSCL (minmod) reconstruction, the
// Hancock half-step, and the HLLC / HLL fluxes with Davis wave speeds, for
// 2D (rho, u, v, p) and 1D (rho, u, p) states; host and device.
//
// Same arithmetic as the reference's include/euler/euler_common.hpp:29-91
// and include/euler/riemann.hpp:38-447, including its mixed-precision
// expressions: gamma is a double constant there, so in a binary32 build
// every expression that contains it is evaluated in binary64 and rounded
// once on assignment.  T = double or float; G is that double constant.
#ifndef PMHD_EULER_HPP
#define PMHD_EULER_HPP

#include <cmath>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace pmhd {
namespace euler {

constexpr double G = 1.4;

template <class T>
__host__ __device__ inline T vmin(T a, T b) {
#ifdef __CUDA_ARCH__
  return fmin(a, b);
#else
  return (b < a) ? b : a;
#endif
}
template <class T>
__host__ __device__ inline T vmax(T a, T b) {
#ifdef __CUDA_ARCH__
  return fmax(a, b);
#else
  return (a < b) ? b : a;
#endif
}

// euler_common.hpp:29-36 (binary64 sqrt of a binary64 argument)
template <class T>
__host__ __device__ inline T sound_speed(T p, T rho) {
  return (T)std::sqrt(G * p / rho);
}

// euler_common.hpp:42-50
template <class T>
__host__ __device__ inline T minmod(T a, T b) {
  if (a * b <= (T)0.0) return (T)0.0;
  return (std::fabs(a) < std::fabs(b)) ? a : b;
}

// euler_common.hpp:67-75
template <class T>
__host__ __device__ inline void cons_to_prim(const T U[4], T W[4]) {
  const T r = U[0];
  W[0] = r;
  W[1] = U[1] / r;
  W[2] = U[2] / r;
  W[3] = (T)((G - (T)1.0) * (U[3] - (T)0.5 * (U[1] * U[1] + U[2] * U[2]) / r));
}

// euler_common.hpp:83-90
template <class T>
__host__ __device__ inline void prim_to_cons(const T W[4], T U[4]) {
  U[0] = W[0];
  U[1] = W[0] * W[1];
  U[2] = W[0] * W[2];
  U[3] = (T)(W[3] / (G - (T)1.0) + (T)0.5 * W[0] * (W[1] * W[1] + W[2] * W[2]));
}

// riemann.hpp:38-43
template <class T>
__host__ __device__ inline void muscl_recon(T qm, T q0, T qp, T& ql, T& qr) {
  const T slope = minmod(q0 - qm, qp - q0);
  ql = q0 - (T)0.5 * slope;
  qr = q0 + (T)0.5 * slope;
}

// riemann.hpp:60-88.  NI / TI: index of the normal / tangential velocity.
template <class T, int NI, int TI>
__host__ __device__ inline void hancock(const T Wface[4], const T Wlf[4], const T Wrf[4], T Wh[4], T factor) {
  T Uf[4];
  prim_to_cons(Wface, Uf);
  const T rL = Wlf[0], uL = Wlf[NI], vL = Wlf[TI], pL = Wlf[3];
  const T rR = Wrf[0], uR = Wrf[NI], vR = Wrf[TI], pR = Wrf[3];
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rL * (uL * uL + vL * vL));
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rR * (uR * uR + vR * vR));
  T dF[4];
  dF[0] = rR * uR - rL * uL;
  dF[NI] = (rR * uR * uR + pR) - (rL * uL * uL + pL);
  dF[TI] = rR * uR * vR - rL * uL * vL;
  dF[3] = (ER + pR) * uR - (EL + pL) * uL;
  T Uh[4];
#pragma unroll
  for (int k = 0; k < 4; k++) Uh[k] = Uf[k] - factor * dF[k];
  cons_to_prim(Uh, Wh);
}

// Tangential momentum flux: the reference's x-direction HLLC multiplies it
// as rho * u_n * u_t, its y-direction one as rho * u_t * u_n.
template <class T, int NI>
__host__ __device__ inline T tangential_flux(T rho, T un, T ut) {
  return NI == 1 ? rho * un * ut : rho * ut * un;
}

// riemann.hpp:98-150 (x, NI = 1) and :158-210 (y, NI = 2): HLLC with Davis
// wave speeds.
template <class T, int NI, int TI>
__host__ __device__ inline void hllc_flux(const T WL[4], const T WR[4], T f[4]) {
  const T rhoL = WL[0], uL = WL[NI], vL = WL[TI], pL = WL[3];
  const T rhoR = WR[0], uR = WR[NI], vR = WR[TI], pR = WR[3];
  const T cL = sound_speed(pL, rhoL), cR = sound_speed(pR, rhoR);
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T denom = rhoL * (SL - uL) - rhoR * (SR - uR);
  const T Ss = (pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR)) / denom;
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rhoL * (uL * uL + vL * vL));
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rhoR * (uR * uR + vR * vR));
  if (SL > (T)0.0) {
    f[0] = rhoL * uL;
    f[NI] = rhoL * uL * uL + pL;
    f[TI] = tangential_flux<T, NI>(rhoL, uL, vL);
    f[3] = (EL + pL) * uL;
  } else if (Ss > (T)0.0) {
    const T coeff = rhoL * (SL - uL) / (SL - Ss);
    const T U0 = coeff, U1 = coeff * Ss, U2 = coeff * vL;
    const T U3 = coeff * (EL / rhoL + (Ss - uL) * (Ss + pL / (rhoL * (SL - uL))));
    f[0] = rhoL * uL + SL * (U0 - rhoL);
    f[NI] = (rhoL * uL * uL + pL) + SL * (U1 - rhoL * uL);
    f[TI] = tangential_flux<T, NI>(rhoL, uL, vL) + SL * (U2 - rhoL * vL);
    f[3] = (EL + pL) * uL + SL * (U3 - EL);
  } else if (SR > (T)0.0) {
    const T coeff = rhoR * (SR - uR) / (SR - Ss);
    const T U0 = coeff, U1 = coeff * Ss, U2 = coeff * vR;
    const T U3 = coeff * (ER / rhoR + (Ss - uR) * (Ss + pR / (rhoR * (SR - uR))));
    f[0] = rhoR * uR + SR * (U0 - rhoR);
    f[NI] = (rhoR * uR * uR + pR) + SR * (U1 - rhoR * uR);
    f[TI] = tangential_flux<T, NI>(rhoR, uR, vR) + SR * (U2 - rhoR * vR);
    f[3] = (ER + pR) * uR + SR * (U3 - ER);
  } else {
    f[0] = rhoR * uR;
    f[NI] = rhoR * uR * uR + pR;
    f[TI] = tangential_flux<T, NI>(rhoR, uR, vR);
    f[3] = (ER + pR) * uR;
  }
}

// riemann.hpp:388-432 (HLL, Davis wave speeds).
template <class T, int NI, int TI>
__host__ __device__ inline void hll_flux(const T WL[4], const T WR[4], T f[4]) {
  const T rhoL = WL[0], uL = WL[NI], vL = WL[TI], pL = WL[3];
  const T rhoR = WR[0], uR = WR[NI], vR = WR[TI], pR = WR[3];
  const T cL = sound_speed(pL, rhoL), cR = sound_speed(pR, rhoR);
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rhoL * (uL * uL + vL * vL));
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rhoR * (uR * uR + vR * vR));
  T FL[4], FR[4], UL[4], UR[4];
  FL[0] = rhoL * uL;
  FR[0] = rhoR * uR;
  FL[NI] = rhoL * uL * uL + pL;
  FR[NI] = rhoR * uR * uR + pR;
  FL[TI] = rhoL * uL * vL;
  FR[TI] = rhoR * uR * vR;
  FL[3] = (EL + pL) * uL;
  FR[3] = (ER + pR) * uR;
  UL[0] = rhoL;
  UR[0] = rhoR;
  UL[NI] = rhoL * uL;
  UR[NI] = rhoR * uR;
  UL[TI] = rhoL * vL;
  UR[TI] = rhoR * vR;
  UL[3] = EL;
  UR[3] = ER;
  if (SL > (T)0.0) {
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = FL[k];
  } else if (SR > (T)0.0) {
    const T inv = (T)1.0 / (SR - SL);
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) * inv;
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = FR[k];
  }
}

// ---- 1D (rho, u, p) ---------------------------------------------------------

// Primitive state of a 1D conservative cell as the reference's 1D driver
// computes it for reconstruction (src/euler/riemann1d_cpu.cpp:138-143).
template <class T>
__host__ __device__ inline void cons_to_prim_1d(T rho, T ru, T E, T W[3]) {
  W[0] = rho;
  W[1] = ru / rho;
  W[2] = (T)((G - (T)1.0) * (E - (T)0.5 * ru * ru / rho));
}

// |u| + c of a 1D cell as the reference computes the time step
// (src/euler/riemann1d_cpu.cpp:117-123).
template <class T>
__host__ __device__ inline T speed_1d(T rho, T ru, T E) {
  const T u = ru / rho;
  const T p = (T)((G - (T)1.0) * (E - (T)0.5 * rho * u * u));
  return std::fabs(u) + sound_speed(p, rho);
}

// Hancock half-step of a 1D face (src/euler/riemann1d_cpu.cpp:160-177).
template <class T>
__host__ __device__ inline void hancock_1d(const T Wf[3], const T Wlf[3], const T Wrf[3], T Wh[3], T factor) {
  const T Uf[3] = {Wf[0], Wf[0] * Wf[1], (T)(Wf[2] / (G - (T)1.0) + (T)0.5 * Wf[0] * Wf[1] * Wf[1])};
  const T rL = Wlf[0], uL = Wlf[1], pL = Wlf[2];
  const T rR = Wrf[0], uR = Wrf[1], pR = Wrf[2];
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rL * uL * uL);
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rR * uR * uR);
  T dF[3];
  dF[0] = rR * uR - rL * uL;
  dF[1] = (rR * uR * uR + pR) - (rL * uL * uL + pL);
  dF[2] = (ER + pR) * uR - (EL + pL) * uL;
  T Uh[3];
#pragma unroll
  for (int k = 0; k < 3; k++) Uh[k] = Uf[k] - factor * dF[k];
  Wh[0] = Uh[0];
  Wh[1] = Uh[1] / Uh[0];
  Wh[2] = (T)((G - (T)1.0) * (Uh[2] - (T)0.5 * Uh[1] * Uh[1] / Uh[0]));
}

// riemann.hpp:290-343
template <class T>
__host__ __device__ inline void hllc_flux_1d(const T WL[3], const T WR[3], T f[3]) {
  const T rhoL = WL[0], uL = WL[1], pL = WL[2];
  const T rhoR = WR[0], uR = WR[1], pR = WR[2];
  const T cL = sound_speed(pL, rhoL), cR = sound_speed(pR, rhoR);
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T denom = rhoL * (SL - uL) - rhoR * (SR - uR);
  const T Ss = (pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR)) / denom;
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rhoL * uL * uL);
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rhoR * uR * uR);
  if (SL > (T)0.0) {
    f[0] = rhoL * uL;
    f[1] = rhoL * uL * uL + pL;
    f[2] = (EL + pL) * uL;
  } else if (Ss > (T)0.0) {
    const T coeff = rhoL * (SL - uL) / (SL - Ss);
    const T U0 = coeff, U1 = coeff * Ss;
    const T U2 = coeff * (EL / rhoL + (Ss - uL) * (Ss + pL / (rhoL * (SL - uL))));
    f[0] = rhoL * uL + SL * (U0 - rhoL);
    f[1] = (rhoL * uL * uL + pL) + SL * (U1 - rhoL * uL);
    f[2] = (EL + pL) * uL + SL * (U2 - EL);
  } else if (SR > (T)0.0) {
    const T coeff = rhoR * (SR - uR) / (SR - Ss);
    const T U0 = coeff, U1 = coeff * Ss;
    const T U2 = coeff * (ER / rhoR + (Ss - uR) * (Ss + pR / (rhoR * (SR - uR))));
    f[0] = rhoR * uR + SR * (U0 - rhoR);
    f[1] = (rhoR * uR * uR + pR) + SR * (U1 - rhoR * uR);
    f[2] = (ER + pR) * uR + SR * (U2 - ER);
  } else {
    f[0] = rhoR * uR;
    f[1] = rhoR * uR * uR + pR;
    f[2] = (ER + pR) * uR;
  }
}

// riemann.hpp:346-378
template <class T>
__host__ __device__ inline void hll_flux_1d(const T WL[3], const T WR[3], T f[3]) {
  const T rhoL = WL[0], uL = WL[1], pL = WL[2];
  const T rhoR = WR[0], uR = WR[1], pR = WR[2];
  const T cL = sound_speed(pL, rhoL), cR = sound_speed(pR, rhoR);
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T EL = (T)(pL / (G - (T)1.0) + (T)0.5 * rhoL * uL * uL);
  const T ER = (T)(pR / (G - (T)1.0) + (T)0.5 * rhoR * uR * uR);
  const T FL[3] = {rhoL * uL, rhoL * uL * uL + pL, (EL + pL) * uL};
  const T FR[3] = {rhoR * uR, rhoR * uR * uR + pR, (ER + pR) * uR};
  const T UL[3] = {rhoL, rhoL * uL, EL};
  const T UR[3] = {rhoR, rhoR * uR, ER};
  if (SL > (T)0.0) {
#pragma unroll
    for (int k = 0; k < 3; k++) f[k] = FL[k];
  } else if (SR > (T)0.0) {
    const T inv = (T)1.0 / (SR - SL);
#pragma unroll
    for (int k = 0; k < 3; k++) f[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) * inv;
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) f[k] = FR[k];
  }
}

// ---- performance forms (the fast build's 2D kernels) -------------------------
// The same scheme with cheaper arithmetic, not bit-identical to the reference:
//   * every expression in the run's type T (the reference evaluates the gamma
//     expressions of its binary32 build in binary64);
//   * one reciprocal per density or divisor, shared by its quotients, and
//     1 / (gamma - 1) as the constant 2.5 (binary64: the IEEE reciprocal;
//     binary32: the hardware's approximate reciprocal and square root);
//   * the two Hancock faces of a cell share one flux difference (it depends
//     only on the two face states, riemann.hpp:60-88 forms it twice);
//   * the HLLC star energy as coeff (E/rho + (S* - u) S*) + (S* - u) p / (S - S*),
//     the reference's coeff (E/rho + (S* - u)(S* + p / (rho (S - u)))) with
//     coeff = rho (S - u) / (S - S*) distributed.
#if defined(__CUDACC__)
namespace fastform {

__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double root(double x) { return sqrt(x); }
__device__ __forceinline__ float root(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <class T>
__device__ __forceinline__ void cons_to_prim(const T U[4], T W[4]) {
  const T ri = rcp(U[0]);
  W[0] = U[0];
  W[1] = U[1] * ri;
  W[2] = U[2] * ri;
  W[3] = (T)0.4 * (U[3] - (T)0.5 * (U[1] * W[1] + U[2] * W[2]));
}

// |u| + c and |v| + c of a conservative cell (the time-step reduction).
template <class T>
__device__ __forceinline__ void cell_speeds(const T U[4], T& sx, T& sy) {
  const T ri = rcp(U[0]);
  const T u = U[1] * ri, v = U[2] * ri;
  const T p = (T)0.4 * (U[3] - (T)0.5 * (U[1] * u + U[2] * v));
  const T c = root((T)1.4 * p * ri);
  sx = std::fabs(u) + c;
  sy = std::fabs(v) + c;
}

// Both Hancock-evolved faces of a cell from its reconstructed left / right
// (lower / upper) face primitives.
template <class T, int NI, int TI>
__device__ __forceinline__ void hancock_pair(const T Wl[4], const T Wr[4], T Lh[4], T Rh[4], T fac) {
  const T rL = Wl[0], uL = Wl[NI], vL = Wl[TI], pL = Wl[3];
  const T rR = Wr[0], uR = Wr[NI], vR = Wr[TI], pR = Wr[3];
  const T mL = rL * uL, mR = rR * uR;
  const T EL = pL * (T)2.5 + (T)0.5 * rL * (uL * uL + vL * vL);
  const T ER = pR * (T)2.5 + (T)0.5 * rR * (uR * uR + vR * vR);
  T dF[4], UL[4], UR[4];
  dF[0] = mR - mL;
  dF[NI] = (mR * uR + pR) - (mL * uL + pL);
  dF[TI] = mR * vR - mL * vL;
  dF[3] = (ER + pR) * uR - (EL + pL) * uL;
  UL[0] = rL, UL[NI] = mL, UL[TI] = rL * vL, UL[3] = EL;
  UR[0] = rR, UR[NI] = mR, UR[TI] = rR * vR, UR[3] = ER;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    UL[k] -= fac * dF[k];
    UR[k] -= fac * dF[k];
  }
  cons_to_prim(UL, Lh);
  cons_to_prim(UR, Rh);
}

template <class T, int NI, int TI>
__device__ __forceinline__ void hllc_flux(const T WL[4], const T WR[4], T f[4]) {
  const T rhoL = WL[0], uL = WL[NI], vL = WL[TI], pL = WL[3];
  const T rhoR = WR[0], uR = WR[NI], vR = WR[TI], pR = WR[3];
  const T riL = rcp(rhoL), riR = rcp(rhoR);
  const T cL = root((T)1.4 * pL * riL), cR = root((T)1.4 * pR * riR);
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T aL = rhoL * (SL - uL), aR = rhoR * (SR - uR);
  const T Ss = (pR - pL + aL * uL - aR * uR) * rcp(aL - aR);
  const T mL = rhoL * uL, mR = rhoR * uR;
  const T EL = pL * (T)2.5 + (T)0.5 * rhoL * (uL * uL + vL * vL);
  const T ER = pR * (T)2.5 + (T)0.5 * rhoR * (uR * uR + vR * vR);
  if (SL > (T)0.0) {
    f[0] = mL;
    f[NI] = mL * uL + pL;
    f[TI] = mL * vL;
    f[3] = (EL + pL) * uL;
  } else if (Ss > (T)0.0) {
    const T d = rcp(SL - Ss), coeff = aL * d, su = Ss - uL;
    const T U3 = coeff * (EL * riL + su * Ss) + su * pL * d;
    f[0] = mL + SL * (coeff - rhoL);
    f[NI] = (mL * uL + pL) + SL * (coeff * Ss - mL);
    f[TI] = mL * vL + SL * (coeff * vL - rhoL * vL);
    f[3] = (EL + pL) * uL + SL * (U3 - EL);
  } else if (SR > (T)0.0) {
    const T d = rcp(SR - Ss), coeff = aR * d, su = Ss - uR;
    const T U3 = coeff * (ER * riR + su * Ss) + su * pR * d;
    f[0] = mR + SR * (coeff - rhoR);
    f[NI] = (mR * uR + pR) + SR * (coeff * Ss - mR);
    f[TI] = mR * vR + SR * (coeff * vR - rhoR * vR);
    f[3] = (ER + pR) * uR + SR * (U3 - ER);
  } else {
    f[0] = mR;
    f[NI] = mR * uR + pR;
    f[TI] = mR * vR;
    f[3] = (ER + pR) * uR;
  }
}

template <class T, int NI, int TI>
__device__ __forceinline__ void hll_flux(const T WL[4], const T WR[4], T f[4]) {
  const T rhoL = WL[0], uL = WL[NI], vL = WL[TI], pL = WL[3];
  const T rhoR = WR[0], uR = WR[NI], vR = WR[TI], pR = WR[3];
  const T cL = root((T)1.4 * pL * rcp(rhoL)), cR = root((T)1.4 * pR * rcp(rhoR));
  const T SL = vmin(uL - cL, uR - cR);
  const T SR = vmax(uL + cL, uR + cR);
  const T mL = rhoL * uL, mR = rhoR * uR;
  const T EL = pL * (T)2.5 + (T)0.5 * rhoL * (uL * uL + vL * vL);
  const T ER = pR * (T)2.5 + (T)0.5 * rhoR * (uR * uR + vR * vR);
  T FL[4], FR[4], UL[4], UR[4];
  FL[0] = mL, FR[0] = mR;
  FL[NI] = mL * uL + pL, FR[NI] = mR * uR + pR;
  FL[TI] = mL * vL, FR[TI] = mR * vR;
  FL[3] = (EL + pL) * uL, FR[3] = (ER + pR) * uR;
  UL[0] = rhoL, UR[0] = rhoR;
  UL[NI] = mL, UR[NI] = mR;
  UL[TI] = rhoL * vL, UR[TI] = rhoR * vR;
  UL[3] = EL, UR[3] = ER;
  if (SL > (T)0.0) {
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = FL[k];
  } else if (SR > (T)0.0) {
    const T inv = rcp(SR - SL);
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) * inv;
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = FR[k];
  }
}

}  // namespace fastform
#endif

}  // namespace euler
}  // namespace pmhd

#endif  // PMHD_EULER_HPP
