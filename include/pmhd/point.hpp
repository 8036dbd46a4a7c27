// pmhd/point.hpp -- header-only per-point ideal-MHD + mixed-GLM numerics,
// compiled both as host code (g++) and as device code (nvcc, sm_100a).
//
// This is the B200 build's replacement for the reference's header-only
// Real/HD layer (include/base.hpp, include/mhd/mhd_common.hpp,
// include/mhd/mhd_glm_common.hpp).  Differences in form, not in arithmetic:
//   * every function is a template on the arithmetic type T, so one source
//     serves the binary64, binary32 and mixed-precision kernels;
//   * gamma and the HLLD tolerance are runtime values (Phys<T>) so batched
//     runs can mix gamma = 5/3 and gamma = 2 in one launch;
//   * the normal direction is a template parameter AX (0 = x, 1 = y).  The
//     reference solves y-faces by permuting the state into x order, calling
//     the x routine and permuting back (mhd_common.hpp:381-405, :658-667);
//     here the routine reads the permuted slots directly, which performs the
//     same operations on the same values.
// Each expression keeps the reference's association order, so with
// contraction disabled (-fmad=false on device, -ffp-contract=off on host)
// the binary64 results are bit-identical to the reference CPU build.
//
// The reference-named compatibility API (mhdHlldFluxX, mhdGlmFluxY, ...)
// lives in pmhd/compat/mhd/mhd_glm_common.hpp on top of this file.
#ifndef PMHD_POINT_HPP
#define PMHD_POINT_HPP

#include <cmath>

#if defined(__CUDACC__)
#define PMHD_HD __host__ __device__ __forceinline__
#else
#define PMHD_HD inline
#endif

namespace pmhd {

// Conserved slots (reference MHDIndex + MHD_GLM_PSI, mhd_common.hpp:81-90,
// mhd_glm_common.hpp:26-27).  Primitive slots reuse 1..4 for vx, vy, vz, p.
enum Slot : int { RHO = 0, MX = 1, MY = 2, MZ = 3, EN = 4, BX = 5, BY = 6, BZ = 7, PSI = 8 };
constexpr int NV8 = 8;
constexpr int NV9 = 9;

// HLLD status codes (mhd_common.hpp:438-440).
enum HlldStatus : int { HLLD_OK = 0, HLLD_FALLBACK_DEGENERATE = 1, HLLD_FALLBACK_NONPHYSICAL = 2 };

template <class T>
struct Phys {
  T gamma;    // ratio of specific heats
  T gm1;      // gamma - 1, evaluated as (gamma - 1) in T
  T tol;      // HLLD relative degeneracy tolerance
  T inv_gm1;  // 1 / gm1 (performance-build forms only)
  PMHD_HD static Phys make(double g, double tolerance) {
    Phys p;
    p.gamma = (T)g;
    p.gm1 = p.gamma - (T)1.0;
    p.tol = (T)tolerance;
    p.inv_gm1 = (T)1.0 / p.gm1;
    return p;
  }
};

template <class T> PMHD_HD T rho_floor() { return (T)1.0e-12; }
template <class T> PMHD_HD T p_floor() { return (T)1.0e-12; }

// max/min/abs/sqrt: device uses fmax/fmin (as the reference device path
// does), host uses the std::max/std::min comparison form.
template <class T> PMHD_HD T vmax(T a, T b) {
#ifdef __CUDA_ARCH__
  return fmax(a, b);
#else
  return (a < b) ? b : a;
#endif
}
template <class T> PMHD_HD T vmin(T a, T b) {
#ifdef __CUDA_ARCH__
  return fmin(a, b);
#else
  return (b < a) ? b : a;
#endif
}
template <class T> PMHD_HD T vabs(T a) {
#ifdef __CUDA_ARCH__
  return fabs(a);
#else
  return std::fabs(a);
#endif
}
template <class T> PMHD_HD T vsqrt(T a) {
#ifdef __CUDA_ARCH__
  return sqrt(a);
#else
  return std::sqrt(a);
#endif
}
// Finite test in the value's own type (the reference converts to double
// first; for a float that is the same predicate).
template <class T> PMHD_HD bool vfinite(T a) {
#ifdef __CUDA_ARCH__
  return isfinite(a);
#else
  return std::isfinite(a);
#endif
}

// Slot map of a normal direction: n = normal, t1/t2 = tangential.
template <int AX>
struct Dir {
  static constexpr int vn = AX ? MY : MX, vt1 = AX ? MX : MY, vt2 = MZ;
  static constexpr int bn = AX ? BY : BX, bt1 = AX ? BX : BY, bt2 = BZ;
};

// Minmod limiter (mhd_common.hpp:140-143).
template <class T> PMHD_HD T minmod(T a, T b) {
  if (a * b <= (T)0.0) return (T)0.0;
  return (vabs(a) < vabs(b)) ? a : b;
}

// W -> U, 8 slots (mhd_common.hpp:149-173), sums in x, y, z order.
template <class T>
PMHD_HD void prim_to_cons(const T* W, T* U, const Phys<T>& ph) {
  const T rho = W[RHO], vx = W[MX], vy = W[MY], vz = W[MZ], p = W[EN];
  const T bx = W[BX], by = W[BY], bz = W[BZ];
  const T v2 = vx * vx + vy * vy + vz * vz;
  const T b2 = bx * bx + by * by + bz * bz;
  U[RHO] = rho;
  U[MX] = rho * vx;
  U[MY] = rho * vy;
  U[MZ] = rho * vz;
  U[EN] = p / ph.gm1 + (T)0.5 * rho * v2 + (T)0.5 * b2;
  U[BX] = bx;
  U[BY] = by;
  U[BZ] = bz;
}

// U -> W, 8 slots (mhd_common.hpp:178-201).  AX selects the summation order
// of |v|^2 and |B|^2 (normal, t1, t2), which is what the reference's
// rotated y-direction calls compute.
template <class T, int AX = 0>
PMHD_HD void cons_to_prim(const T* U, T* W, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T rho = vmax(U[RHO], rho_floor<T>());
  const T vn = U[D::vn] / rho, vt1 = U[D::vt1] / rho, vt2 = U[D::vt2] / rho;
  const T bn = U[D::bn], bt1 = U[D::bt1], bt2 = U[D::bt2];
  const T v2 = vn * vn + vt1 * vt1 + vt2 * vt2;
  const T b2 = bn * bn + bt1 * bt1 + bt2 * bt2;
  const T p = ph.gm1 * (U[EN] - (T)0.5 * rho * v2 - (T)0.5 * b2);
  W[RHO] = rho;
  W[D::vn] = vn;
  W[D::vt1] = vt1;
  W[D::vt2] = vt2;
  W[EN] = p;
  W[D::bn] = bn;
  W[D::bt1] = bt1;
  W[D::bt2] = bt2;
}

// Fast magnetosonic speed along AX (mhd_common.hpp:206-238).
template <class T, int AX>
PMHD_HD T fast_speed(const T* W, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T rho = vmax(W[RHO], rho_floor<T>());
  const T p = vmax(W[EN], p_floor<T>());
  const T bn = W[D::bn], bt1 = W[D::bt1], bt2 = W[D::bt2];
  const T a2 = ph.gamma * p / rho;
  const T b2 = (bn * bn + bt1 * bt1 + bt2 * bt2) / rho;
  const T can2 = bn * bn / rho;
  T disc = (a2 + b2) * (a2 + b2) - (T)4.0 * a2 * can2;
  disc = vmax(disc, (T)0.0);
  const T cf2 = (T)0.5 * (a2 + b2 + vsqrt(disc));
  return vsqrt(vmax(cf2, (T)0.0));
}

// Physical ideal-MHD flux along AX from primitives W and total energy e
// (mhdFluxXW / mhdFluxYW, mhd_common.hpp:247-308).
template <class T, int AX>
PMHD_HD void phys_flux(const T* W, T e, T* F) {
  using D = Dir<AX>;
  const T rho = W[RHO], vn = W[D::vn], vt1 = W[D::vt1], vt2 = W[D::vt2], p = W[EN];
  const T bn = W[D::bn], bt1 = W[D::bt1], bt2 = W[D::bt2];
  const T b2 = bn * bn + bt1 * bt1 + bt2 * bt2;
  const T ptot = p + (T)0.5 * b2;
  const T vdotb = vn * bn + vt1 * bt1 + vt2 * bt2;
  F[RHO] = rho * vn;
  F[D::vn] = rho * vn * vn + ptot - bn * bn;
  F[D::vt1] = rho * vn * vt1 - bn * bt1;
  F[D::vt2] = rho * vn * vt2 - bn * bt2;
  F[EN] = (e + ptot) * vn - bn * vdotb;
  F[D::bn] = (T)0.0;
  F[D::bt1] = vn * bt1 - bn * vt1;
  F[D::bt2] = vn * bt2 - bn * vt2;
}

// HLL flux along AX (mhdHllFluxX / mhdHllFluxY, mhd_common.hpp:323-377).
template <class T, int AX>
PMHD_HD void hll_flux(const T* UL, const T* UR, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  T WL[NV8], WR[NV8], FL[NV8], FR[NV8];
  cons_to_prim<T, AX>(UL, WL, ph);
  cons_to_prim<T, AX>(UR, WR, ph);
  phys_flux<T, AX>(WL, UL[EN], FL);
  phys_flux<T, AX>(WR, UR[EN], FR);
  const T cfL = fast_speed<T, AX>(WL, ph);
  const T cfR = fast_speed<T, AX>(WR, ph);
  const T sL = vmin(WL[D::vn] - cfL, WR[D::vn] - cfR);
  const T sR = vmax(WL[D::vn] + cfL, WR[D::vn] + cfR);
  if (sL >= (T)0.0) {
#pragma unroll
    for (int k = 0; k < NV8; k++) F[k] = FL[k];
  } else if (sR <= (T)0.0) {
#pragma unroll
    for (int k = 0; k < NV8; k++) F[k] = FR[k];
  } else {
    const T denom = sR - sL;
#pragma unroll
    for (int k = 0; k < NV8; k++) F[k] = (sR * FL[k] - sL * FR[k] + sL * sR * (UR[k] - UL[k])) / denom;
  }
}

// Scale-aware smallness test (mhdHlldIsSmall, mhd_common.hpp:417-419).
template <class T> PMHD_HD bool hlld_small(T v, T scale, const Phys<T>& ph) {
  return vabs(v) <= ph.tol * scale;
}

// Positive density and pressure; the negated comparison also rejects NaN
// (mhdConservedHasPositivePressure, mhd_common.hpp:426-431).
template <class T, int AX>
PMHD_HD bool positive_state(const T* U, const Phys<T>& ph) {
  if (!(U[RHO] > rho_floor<T>())) return false;
  T W[NV8];
  cons_to_prim<T, AX>(U, W, ph);
  return (W[RHO] > rho_floor<T>() && W[EN] > p_floor<T>());
}

// Star state behind an outer fast wave of speed s (mhdHlldStarStateX,
// mhd_common.hpp:445-511).  bn is the (shared) normal field.  vts receives
// the star tangential velocities.
//
// FAST = true (the performance build only, never the parity build): the same
// state with two reciprocals instead of six divisions, and the positivity
// test from the star primitives already at hand instead of a conserved ->
// primitive recovery (equal up to rounding).
template <class T, int AX, bool FAST = false>
PMHD_HD int hlld_star(const T* U, const T* W, T s, T sm, T pt_star, T bn, T* Us, T* vts, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T rho = vmax(W[RHO], rho_floor<T>());
  const T vn = W[D::vn], vt1 = W[D::vt1], vt2 = W[D::vt2];
  const T p = vmax(W[EN], p_floor<T>());
  const T bt1 = W[D::bt1], bt2 = W[D::bt2];
  const T e = U[EN];
  const T smv = s - vn;
  const T sms = s - sm;
  const T wave_scale = vmax(vabs(s), vabs(sm));
  if (hlld_small(sms, wave_scale, ph)) return HLLD_FALLBACK_DEGENERATE;
  T rho_s, vt1_s, vt2_s, bt1_s, bt2_s, e_s;
  const T b2 = bn * bn + bt1 * bt1 + bt2 * bt2;
  const T pt = p + (T)0.5 * b2;
  const T vdotb = vn * bn + vt1 * bt1 + vt2 * bt2;
  if (FAST) {
    const T inv_sms = (T)1.0 / sms;
    rho_s = rho * smv * inv_sms;
    if (rho_s <= rho_floor<T>()) return HLLD_FALLBACK_NONPHYSICAL;
    const T denom = rho * smv * sms - bn * bn;
    const T denom_scale = vabs(rho * smv * sms) + bn * bn;
    if (hlld_small(denom, denom_scale, ph)) return HLLD_FALLBACK_DEGENERATE;
    const T inv_den = (T)1.0 / denom;
    const T cb = bn * (sm - vn) * inv_den;
    const T fb = (rho * smv * smv - bn * bn) * inv_den;
    vt1_s = vt1 - bt1 * cb;
    vt2_s = vt2 - bt2 * cb;
    bt1_s = bt1 * fb;
    bt2_s = bt2 * fb;
    const T vbs = sm * bn + vt1_s * bt1_s + vt2_s * bt2_s;
    e_s = (smv * e - pt * vn + pt_star * sm + bn * (vdotb - vbs)) * inv_sms;
  } else {
    rho_s = rho * smv / sms;
    if (rho_s <= rho_floor<T>()) return HLLD_FALLBACK_NONPHYSICAL;
    const T denom = rho * smv * sms - bn * bn;
    const T denom_scale = vabs(rho * smv * sms) + bn * bn;
    if (hlld_small(denom, denom_scale, ph)) return HLLD_FALLBACK_DEGENERATE;
    const T common = sm - vn;
    vt1_s = vt1 - bn * bt1 * common / denom;
    vt2_s = vt2 - bn * bt2 * common / denom;
    bt1_s = bt1 * (rho * smv * smv - bn * bn) / denom;
    bt2_s = bt2 * (rho * smv * smv - bn * bn) / denom;
    const T vbs = sm * bn + vt1_s * bt1_s + vt2_s * bt2_s;
    e_s = (smv * e - pt * vn + pt_star * sm + bn * (vdotb - vbs)) / sms;
  }
  Us[RHO] = rho_s;
  Us[D::vn] = rho_s * sm;
  Us[D::vt1] = rho_s * vt1_s;
  Us[D::vt2] = rho_s * vt2_s;
  Us[EN] = e_s;
  Us[D::bn] = bn;
  Us[D::bt1] = bt1_s;
  Us[D::bt2] = bt2_s;
  vts[0] = vt1_s;
  vts[1] = vt2_s;
  if (FAST) {
    const T v2 = sm * sm + vt1_s * vt1_s + vt2_s * vt2_s;
    const T b2s = bn * bn + bt1_s * bt1_s + bt2_s * bt2_s;
    const T p_s = ph.gm1 * (e_s - (T)0.5 * rho_s * v2 - (T)0.5 * b2s);
    return (p_s > p_floor<T>()) ? HLLD_OK : HLLD_FALLBACK_NONPHYSICAL;
  }
  return positive_state<T, AX>(Us, ph) ? HLLD_OK : HLLD_FALLBACK_NONPHYSICAL;
}

// HLLD flux along AX (Miyoshi & Kusano 2005 with the reference's
// scale-aware guards; mhdHlldFluxX, mhd_common.hpp:518-654).  Degenerate or
// non-physical intermediate states fall back to HLL at this interface and
// return the reason.
//
// Same arithmetic as the reference, arranged for a GPU thread: the HLL
// fallback has a single call site, and only the physical flux of the side
// the final formula uses is evaluated (the reference evaluates both up
// front; the unused one never reaches F).  The side test `sm >= 0` selects
// the same branch as the reference's chain sLs >= 0 / sm >= 0 / sRs >= 0
// because sLs <= sm <= sRs, and NaN reaches the same last branch.
//
// hlld_core takes the primitives of both sides as well; FAST as for
// hlld_star (tangential star velocities reused, reciprocals, positivity of
// the double-star states from their primitives).
template <class T, int AX, bool FAST = false>
PMHD_HD int hlld_core(const T* UL, const T* WL, const T* UR, const T* WR, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T cfL = fast_speed<T, AX>(WL, ph);
  const T cfR = fast_speed<T, AX>(WR, ph);
  const T sL = vmin(WL[D::vn] - cfL, WR[D::vn] - cfR);
  const T sR = vmax(WL[D::vn] + cfL, WR[D::vn] + cfR);
  if (sL >= (T)0.0) {
    phys_flux<T, AX>(WL, UL[EN], F);
    return HLLD_OK;
  }
  if (sR <= (T)0.0) {
    phys_flux<T, AX>(WR, UR[EN], F);
    return HLLD_OK;
  }
  int status = HLLD_OK;
  do {
    const T rhoL = vmax(WL[RHO], rho_floor<T>());
    const T rhoR = vmax(WR[RHO], rho_floor<T>());
    const T vnL = WL[D::vn], vnR = WR[D::vn];
    const T bn = (T)0.5 * (WL[D::bn] + WR[D::bn]);
    const T b2L = bn * bn + WL[D::bt1] * WL[D::bt1] + WL[D::bt2] * WL[D::bt2];
    const T b2R = bn * bn + WR[D::bt1] * WR[D::bt1] + WR[D::bt2] * WR[D::bt2];
    const T ptL = vmax(WL[EN], p_floor<T>()) + (T)0.5 * b2L;
    const T ptR = vmax(WR[EN], p_floor<T>()) + (T)0.5 * b2R;
    const T denom_sm = rhoR * (sR - vnR) - rhoL * (sL - vnL);
    const T denom_sm_scale = vabs(rhoR * (sR - vnR)) + vabs(rhoL * (sL - vnL));
    const T b_scale = vsqrt(vmax(b2L, b2R));
    if (hlld_small(denom_sm, denom_sm_scale, ph) || hlld_small(bn, b_scale, ph)) {
      status = HLLD_FALLBACK_DEGENERATE;
      break;
    }
    const T sm = (rhoR * vnR * (sR - vnR) - rhoL * vnL * (sL - vnL) + ptL - ptR) / denom_sm;
    const T ptsL = ptL + rhoL * (sL - vnL) * (sm - vnL);
    const T ptsR = ptR + rhoR * (sR - vnR) * (sm - vnR);
    const T pts = (T)0.5 * (ptsL + ptsR);
    T ULs[NV8], URs[NV8], vtL[2], vtR[2];
    const int stL = hlld_star<T, AX, FAST>(UL, WL, sL, sm, pts, bn, ULs, vtL, ph);
    const int stR = hlld_star<T, AX, FAST>(UR, WR, sR, sm, pts, bn, URs, vtR, ph);
    if (stL != HLLD_OK || stR != HLLD_OK) {
      status = (stL != HLLD_OK) ? stL : stR;
      break;
    }
    const T sqL = vsqrt(vmax(ULs[RHO], rho_floor<T>()));
    const T sqR = vsqrt(vmax(URs[RHO], rho_floor<T>()));
    const T sgn = (bn < (T)0.0) ? (T)-1.0 : (T)1.0;
    const T sLs = sm - vabs(bn) / sqL;
    const T sRs = sm + vabs(bn) / sqR;
    const T den = sqL + sqR;
    if (den <= (T)0.0) {
      status = HLLD_FALLBACK_DEGENERATE;
      break;
    }
    const T vt1Ls = FAST ? vtL[0] : ULs[D::vt1] / ULs[RHO], vt2Ls = FAST ? vtL[1] : ULs[D::vt2] / ULs[RHO];
    const T bt1Ls = ULs[D::bt1], bt2Ls = ULs[D::bt2];
    const T vt1Rs = FAST ? vtR[0] : URs[D::vt1] / URs[RHO], vt2Rs = FAST ? vtR[1] : URs[D::vt2] / URs[RHO];
    const T bt1Rs = URs[D::bt1], bt2Rs = URs[D::bt2];
    T vt1D, vt2D, bt1D, bt2D;
    if (FAST) {
      const T inv_den = (T)1.0 / den;
      vt1D = (sqL * vt1Ls + sqR * vt1Rs + sgn * (bt1Rs - bt1Ls)) * inv_den;
      vt2D = (sqL * vt2Ls + sqR * vt2Rs + sgn * (bt2Rs - bt2Ls)) * inv_den;
      bt1D = (sqL * bt1Rs + sqR * bt1Ls + sgn * sqL * sqR * (vt1Rs - vt1Ls)) * inv_den;
      bt2D = (sqL * bt2Rs + sqR * bt2Ls + sgn * sqL * sqR * (vt2Rs - vt2Ls)) * inv_den;
    } else {
      vt1D = (sqL * vt1Ls + sqR * vt1Rs + sgn * (bt1Rs - bt1Ls)) / den;
      vt2D = (sqL * vt2Ls + sqR * vt2Rs + sgn * (bt2Rs - bt2Ls)) / den;
      bt1D = (sqL * bt1Rs + sqR * bt1Ls + sgn * sqL * sqR * (vt1Rs - vt1Ls)) / den;
      bt2D = (sqL * bt2Rs + sqR * bt2Ls + sgn * sqL * sqR * (vt2Rs - vt2Ls)) / den;
    }
    const T vbD = sm * bn + vt1D * bt1D + vt2D * bt2D;
    const T vbLs = sm * bn + vt1Ls * bt1Ls + vt2Ls * bt2Ls;
    const T vbRs = sm * bn + vt1Rs * bt1Rs + vt2Rs * bt2Rs;
    // Double-star states differ from the star states only in the tangential
    // slots and the energy.
    T ULD[NV8], URD[NV8];
#pragma unroll
    for (int k = 0; k < NV8; k++) {
      ULD[k] = ULs[k];
      URD[k] = URs[k];
    }
    ULD[D::vt1] = ULD[RHO] * vt1D;
    ULD[D::vt2] = ULD[RHO] * vt2D;
    ULD[D::bt1] = bt1D;
    ULD[D::bt2] = bt2D;
    URD[D::vt1] = URD[RHO] * vt1D;
    URD[D::vt2] = URD[RHO] * vt2D;
    URD[D::bt1] = bt1D;
    URD[D::bt2] = bt2D;
    ULD[EN] = ULs[EN] - sgn * sqL * (vbLs - vbD);
    URD[EN] = URs[EN] + sgn * sqR * (vbRs - vbD);
    bool positive;
    if (FAST) {
      const T v2D = sm * sm + vt1D * vt1D + vt2D * vt2D;
      const T b2D = bn * bn + bt1D * bt1D + bt2D * bt2D;
      const T pLD = ph.gm1 * (ULD[EN] - (T)0.5 * ULD[RHO] * v2D - (T)0.5 * b2D);
      const T pRD = ph.gm1 * (URD[EN] - (T)0.5 * URD[RHO] * v2D - (T)0.5 * b2D);
      positive = ULD[RHO] > rho_floor<T>() && URD[RHO] > rho_floor<T>() && pLD > p_floor<T>() && pRD > p_floor<T>();
    } else {
      positive = positive_state<T, AX>(ULD, ph) && positive_state<T, AX>(URD, ph);
    }
    if (!positive) {
      status = HLLD_FALLBACK_NONPHYSICAL;
      break;
    }
    if (sm >= (T)0.0) {
      phys_flux<T, AX>(WL, UL[EN], F);
      if (sLs >= (T)0.0) {
#pragma unroll
        for (int k = 0; k < NV8; k++) F[k] = F[k] + sL * (ULs[k] - UL[k]);
      } else {
#pragma unroll
        for (int k = 0; k < NV8; k++) F[k] = F[k] + sL * (ULs[k] - UL[k]) + sLs * (ULD[k] - ULs[k]);
      }
    } else {
      phys_flux<T, AX>(WR, UR[EN], F);
      if (sRs >= (T)0.0) {
#pragma unroll
        for (int k = 0; k < NV8; k++) F[k] = F[k] + sR * (URs[k] - UR[k]) + sRs * (URD[k] - URs[k]);
      } else {
#pragma unroll
        for (int k = 0; k < NV8; k++) F[k] = F[k] + sR * (URs[k] - UR[k]);
      }
    }
    return HLLD_OK;
  } while (false);
  hll_flux<T, AX>(UL, UR, F, ph);
  return status;
}

template <class T, int AX, bool FAST = false>
PMHD_HD int hlld_flux(const T* UL, const T* UR, T* F, const Phys<T>& ph) {
  T WL[NV8], WR[NV8];
  cons_to_prim<T, AX>(UL, WL, ph);
  cons_to_prim<T, AX>(UR, WR, ph);
  return hlld_core<T, AX, FAST>(UL, WL, UR, WR, F, ph);
}

// Mixed-GLM interface flux along AX (mhdGlmNormalState + mhdGlmFluxX/Y,
// mhd_glm_common.hpp:55-126): upwind B_n* and psi* of the linear GLM
// subsystem, HLLD (or HLL) on the 8 MHD slots with B_n = B_n* on both sides,
// F[B_n] = psi*, F[psi] = ch^2 B_n*.
//
// FAST selects the performance-build HLLD arithmetic (hlld_core).
template <class T, int AX, bool FAST = false>
PMHD_HD int glm_flux(const T* UL, const T* UR, T ch, bool use_hlld, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T ch_safe = vmax(ch, (T)1.0e-12);
  const T bnL = UL[D::bn], bnR = UR[D::bn], psiL = UL[PSI], psiR = UR[PSI];
  const T bns = (T)0.5 * (bnL + bnR) - (T)0.5 * (psiR - psiL) / ch_safe;
  const T psis = (T)0.5 * (psiL + psiR) - (T)0.5 * ch_safe * (bnR - bnL);
  T a[NV8], b[NV8];
#pragma unroll
  for (int k = 0; k < NV8; k++) {
    a[k] = UL[k];
    b[k] = UR[k];
  }
  a[D::bn] = bns;
  b[D::bn] = bns;
  int status = HLLD_OK;
  if (use_hlld)
    status = hlld_flux<T, AX, FAST>(a, b, F, ph);
  else
    hll_flux<T, AX>(a, b, F, ph);
  F[D::bn] = psis;
  F[PSI] = ch * ch * bns;
  return status;
}

// GLM-augmented physical flux along AX of a 9-slot conserved state: the
// ideal-MHD flux (recovered with AX's summation order, i.e. the reference's
// rotation for y), F[B_n] = psi, F[psi] = ch^2 B_n.  Used by the MUSCL-Hancock
// predictor.
template <class T, int AX>
PMHD_HD void glm_phys_flux(const T* U, T ch, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  T W[NV8];
  cons_to_prim<T, AX>(U, W, ph);
  phys_flux<T, AX>(W, U[EN], F);
  F[D::bn] = U[PSI];
  F[PSI] = ch * ch * U[D::bn];
}

// glm_flux from the two face PRIMITIVES (9 slots, as reconstructed), for the
// performance build: the conserved states are formed once, the primitives
// the flux needs are the face primitives with B_n replaced by B_n* and the
// pressure shifted by gm1 * (B_n^2 - B_n*^2) / 2 (what recovering them from
// the modified conserved state gives, up to rounding), so the Riemann solver
// recovers nothing.
template <class T, int AX>
PMHD_HD int glm_flux_prim(const T* PL, const T* PR, T ch, bool use_hlld, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T ch_safe = vmax(ch, (T)1.0e-12);
  const T bnL = PL[D::bn], bnR = PR[D::bn], psiL = PL[PSI], psiR = PR[PSI];
  const T bns = (T)0.5 * (bnL + bnR) - (T)0.5 * (psiR - psiL) / ch_safe;
  const T psis = (T)0.5 * (psiL + psiR) - (T)0.5 * ch_safe * (bnR - bnL);
  T UL[NV8], UR[NV8];
  prim_to_cons<T>(PL, UL, ph);
  prim_to_cons<T>(PR, UR, ph);
  UL[D::bn] = bns;
  UR[D::bn] = bns;
  int status = HLLD_OK;
  if (use_hlld) {
    T WL[NV8], WR[NV8];
#pragma unroll
    for (int k = 0; k < NV8; k++) {
      WL[k] = PL[k];
      WR[k] = PR[k];
    }
    WL[D::bn] = bns;
    WR[D::bn] = bns;
    WL[EN] = PL[EN] + (T)0.5 * ph.gm1 * (bnL - bns) * (bnL + bns);
    WR[EN] = PR[EN] + (T)0.5 * ph.gm1 * (bnR - bns) * (bnR + bns);
    status = hlld_core<T, AX, true>(UL, WL, UR, WR, F, ph);
  } else {
    hll_flux<T, AX>(UL, UR, F, ph);
  }
  F[D::bn] = psis;
  F[PSI] = ch * ch * bns;
  return status;
}

// ---- 9-slot helpers of the 2D driver (mhd2d_glm_cpu.cpp:90-161) ----------

// Conserved -> primitive with psi carried in slot 8.
template <class T>
PMHD_HD void state_to_prim9(const T* U, T* P, const Phys<T>& ph) {
  cons_to_prim<T, 0>(U, P, ph);
  P[PSI] = U[PSI];
}

template <class T>
PMHD_HD void prim9_to_state(const T* P, T* U, const Phys<T>& ph) {
  prim_to_cons<T>(P, U, ph);
  U[PSI] = P[PSI];
}

// Positive floors and all nine slots finite (primitiveIsUsable).
template <class T>
PMHD_HD bool prim9_usable(const T* P) {
  if (P[RHO] <= rho_floor<T>() || P[EN] <= p_floor<T>()) return false;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < NV9; k++) ok = ok && vfinite(P[k]);
  return ok;
}

// stateIsUsable: density above the floor before recovery, then the
// primitive test.
template <class T>
PMHD_HD bool state_usable(const T* U, const Phys<T>& ph) {
  if (U[RHO] <= rho_floor<T>()) return false;
  T P[NV9];
  state_to_prim9<T>(U, P, ph);
  return prim9_usable<T>(P);
}

// Limited linear reconstruction of one cell from its two neighbours along an
// axis: Pl = left face, Pr = right face; first order when either face is
// unusable (reconstructPrimitive).
template <class T>
PMHD_HD void recon_cell(const T* Pm, const T* P0, const T* Pp, T* Pl, T* Pr) {
#pragma unroll
  for (int k = 0; k < NV9; k++) {
    const T slope = minmod(P0[k] - Pm[k], Pp[k] - P0[k]);
    Pl[k] = P0[k] - (T)0.5 * slope;
    Pr[k] = P0[k] + (T)0.5 * slope;
  }
  if (!prim9_usable<T>(Pl) || !prim9_usable<T>(Pr)) {
#pragma unroll
    for (int k = 0; k < NV9; k++) {
      Pl[k] = P0[k];
      Pr[k] = P0[k];
    }
  }
}

// Signal speed of one cell, max(|vx| + cf_x, |vy| + cf_y).
template <class T>
PMHD_HD T cell_speed(const T* P, const Phys<T>& ph) {
  const T sx = vabs(P[MX]) + fast_speed<T, 0>(P, ph);
  const T sy = vabs(P[MY]) + fast_speed<T, 1>(P, ph);
  return vmax(sx, sy);
}

// ---- performance-build forms ------------------------------------------------
//
// The kernels of the performance build (never the parity build) use the forms
// below: the same HLLD / HLL + GLM algorithm, rearranged so a GPU thread issues
// fewer instructions.  Equal to the reference forms above up to rounding:
//   * reciprocals instead of divisions: one per density, wave-speed
//     difference and denominator, shared by every quotient of that divisor
//     (binary32: the hardware's approximate reciprocal, <= 1 ulp);
//   * the Riemann problem is posed on primitives plus total energy: the face
//     primitives of the reconstruction go in directly (the reference forms
//     conserved states and recovers primitives again), the pressure carries
//     the GLM change of B_n as gm1 (B_n^2 - B_n*^2) / 2 (what the recovery of
//     the modified conserved state gives), and a conserved component is
//     formed only where a flux difference needs it;
//   * the field-smallness guard |B_n| <= tol sqrt(max(b2L, b2R)) is tested
//     squared, and the star-state positivity tests use the star primitives at
//     hand (as the FAST forms above).

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float fast_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float fast_rsqrt(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float fast_sqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#else
inline float fast_rcp(float x) { return 1.0f / x; }
inline float fast_rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float fast_sqrt(float x) { return std::sqrt(x); }
#endif
PMHD_HD double fast_rcp(double x) { return 1.0 / x; }
PMHD_HD double fast_rsqrt(double x) { return 1.0 / vsqrt(x); }
PMHD_HD double fast_sqrt(double x) { return vsqrt(x); }

// Binary64 reciprocal by two Newton-Raphson steps r <- r + r (1 - x r) from
// the binary32 approximate reciprocal (relative error ~2^-22 -> ~2^-44 ->
// below binary64 rounding); for 1e-30 < |x| < 1e30.
PMHD_HD double rcp_newton(double x) {
#if defined(__CUDA_ARCH__)
  double r = (double)fast_rcp((float)x);
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
#else
  return 1.0 / x;
#endif
}

// GLM constants of one stage, uniform over a launch: ch, max(ch, 1e-12),
// 0.5 / max(ch, 1e-12) and ch^2.
template <class T>
struct GlmK {
  T ch, ch_safe, half_inv, ch2;
  PMHD_HD static GlmK make(T c) {
    GlmK k;
    k.ch = c;
    k.ch_safe = vmax(c, (T)1.0e-12);
    k.half_inv = (T)0.5 * fast_rcp(k.ch_safe);
    k.ch2 = c * c;
    return k;
  }
};

// One side of an interface in normal/tangential components, after the GLM
// substitution B_n := B_n*.
template <class T>
struct RSide {
  T rho, inv, vn, vt1, vt2, p, bt1, bt2, e, bt2s;  // bt2s = bt1^2 + bt2^2
};

template <class T, int AX>
PMHD_HD RSide<T> rside(const T* P, T bn0, T bns, const Phys<T>& ph) {
  using D = Dir<AX>;
  RSide<T> s;
  s.rho = vmax(P[RHO], rho_floor<T>());
  s.inv = fast_rcp(s.rho);
  s.vn = P[D::vn];
  s.vt1 = P[D::vt1];
  s.vt2 = P[D::vt2];
  s.bt1 = P[D::bt1];
  s.bt2 = P[D::bt2];
  s.bt2s = s.bt1 * s.bt1 + s.bt2 * s.bt2;
  const T v2 = s.vn * s.vn + s.vt1 * s.vt1 + s.vt2 * s.vt2;
  const T p0 = P[EN];
  s.e = p0 * ph.inv_gm1 + (T)0.5 * s.rho * v2 + (T)0.5 * (bn0 * bn0 + s.bt2s);
  s.p = p0 + (T)0.5 * ph.gm1 * (bn0 - bns) * (bn0 + bns);
  return s;
}

// Fast magnetosonic speed along the normal (fast_speed with one reciprocal).
template <class T>
PMHD_HD T rside_cf(const RSide<T>& s, T bn2, const Phys<T>& ph) {
  const T a2 = ph.gamma * vmax(s.p, p_floor<T>()) * s.inv;
  const T b2 = (bn2 + s.bt2s) * s.inv;
  const T can2 = bn2 * s.inv;
  const T sum = a2 + b2;
  const T disc = vmax(sum * sum - (T)4.0 * a2 * can2, (T)0.0);
  return fast_sqrt(vmax((T)0.5 * (sum + fast_sqrt(disc)), (T)0.0));
}

// Physical flux of one side (slots in AX order; F[B_n] is left to the caller).
template <class T, int AX>
PMHD_HD void rside_flux(const RSide<T>& s, T bn, T bn2, T* F) {
  using D = Dir<AX>;
  const T ptot = s.p + (T)0.5 * (bn2 + s.bt2s);
  const T vdotb = s.vn * bn + s.vt1 * s.bt1 + s.vt2 * s.bt2;
  const T mn = s.rho * s.vn;
  F[RHO] = mn;
  F[D::vn] = mn * s.vn + ptot - bn2;
  F[D::vt1] = mn * s.vt1 - bn * s.bt1;
  F[D::vt2] = mn * s.vt2 - bn * s.bt2;
  F[EN] = (s.e + ptot) * s.vn - bn * vdotb;
  F[D::bt1] = s.vn * s.bt1 - bn * s.vt1;
  F[D::bt2] = s.vn * s.bt2 - bn * s.vt2;
}

// HLL along AX from two sides and their outer wave speeds sL < 0 < sR.
template <class T, int AX>
PMHD_HD void rside_hll(const RSide<T>& L, const RSide<T>& R, T bn, T bn2, T sL, T sR, T* F) {
  using D = Dir<AX>;
  T FL[NV8], FR[NV8];
  rside_flux<T, AX>(L, bn, bn2, FL);
  rside_flux<T, AX>(R, bn, bn2, FR);
  const T inv = fast_rcp(sR - sL);
  const T ss = sL * sR;
  F[RHO] = (sR * FL[RHO] - sL * FR[RHO] + ss * (R.rho - L.rho)) * inv;
  F[D::vn] = (sR * FL[D::vn] - sL * FR[D::vn] + ss * (R.rho * R.vn - L.rho * L.vn)) * inv;
  F[D::vt1] = (sR * FL[D::vt1] - sL * FR[D::vt1] + ss * (R.rho * R.vt1 - L.rho * L.vt1)) * inv;
  F[D::vt2] = (sR * FL[D::vt2] - sL * FR[D::vt2] + ss * (R.rho * R.vt2 - L.rho * L.vt2)) * inv;
  F[EN] = (sR * FL[EN] - sL * FR[EN] + ss * (R.e - L.e)) * inv;
  F[D::bt1] = (sR * FL[D::bt1] - sL * FR[D::bt1] + ss * (R.bt1 - L.bt1)) * inv;
  F[D::bt2] = (sR * FL[D::bt2] - sL * FR[D::bt2] + ss * (R.bt2 - L.bt2)) * inv;
}

// Star state of one side (hlld_star): density, tangential velocity and field,
// energy, and v.B; returns the status.
template <class T>
struct RStar {
  T rho, vt1, vt2, bt1, bt2, e, vb;
};

template <class T>
PMHD_HD int rside_star(const RSide<T>& s, T sw, T sm, T pt, T pts, T bn, T bn2, RStar<T>& o, const Phys<T>& ph) {
  const T smv = sw - s.vn;
  const T sms = sw - sm;
  if (hlld_small(sms, vmax(vabs(sw), vabs(sm)), ph)) return HLLD_FALLBACK_DEGENERATE;
  const T inv_sms = fast_rcp(sms);
  const T d = s.rho * smv;
  o.rho = d * inv_sms;
  if (o.rho <= rho_floor<T>()) return HLLD_FALLBACK_NONPHYSICAL;
  const T dsms = d * sms;
  const T denom = dsms - bn2;
  if (hlld_small(denom, vabs(dsms) + bn2, ph)) return HLLD_FALLBACK_DEGENERATE;
  const T inv_den = fast_rcp(denom);
  const T cb = bn * (sm - s.vn) * inv_den;
  const T fb = (d * smv - bn2) * inv_den;
  o.vt1 = s.vt1 - s.bt1 * cb;
  o.vt2 = s.vt2 - s.bt2 * cb;
  o.bt1 = s.bt1 * fb;
  o.bt2 = s.bt2 * fb;
  const T vdotb = s.vn * bn + s.vt1 * s.bt1 + s.vt2 * s.bt2;
  o.vb = sm * bn + o.vt1 * o.bt1 + o.vt2 * o.bt2;
  o.e = (smv * s.e - pt * s.vn + pts * sm + bn * (vdotb - o.vb)) * inv_sms;
  const T v2 = sm * sm + o.vt1 * o.vt1 + o.vt2 * o.vt2;
  const T b2 = bn2 + o.bt1 * o.bt1 + o.bt2 * o.bt2;
  const T ps = ph.gm1 * (o.e - (T)0.5 * o.rho * v2 - (T)0.5 * b2);
  return (ps > p_floor<T>()) ? HLLD_OK : HLLD_FALLBACK_NONPHYSICAL;
}

// F += sw (Us - U) for one side (slots in AX order; the B_n jump is zero).
template <class T, int AX>
PMHD_HD void rside_jump(const RSide<T>& s, const RStar<T>& st, T sm, T sw, T* F) {
  using D = Dir<AX>;
  F[RHO] += sw * (st.rho - s.rho);
  F[D::vn] += sw * (st.rho * sm - s.rho * s.vn);
  F[D::vt1] += sw * (st.rho * st.vt1 - s.rho * s.vt1);
  F[D::vt2] += sw * (st.rho * st.vt2 - s.rho * s.vt2);
  F[EN] += sw * (st.e - s.e);
  F[D::bt1] += sw * (st.bt1 - s.bt1);
  F[D::bt2] += sw * (st.bt2 - s.bt2);
}

// F += sws (UD - Us) (density and normal momentum do not jump).
template <class T, int AX>
PMHD_HD void rside_jump2(const RStar<T>& st, T vt1D, T vt2D, T bt1D, T bt2D, T eD, T sws, T* F) {
  using D = Dir<AX>;
  const T sr = sws * st.rho;
  F[D::vt1] += sr * (vt1D - st.vt1);
  F[D::vt2] += sr * (vt2D - st.vt2);
  F[EN] += sws * (eD - st.e);
  F[D::bt1] += sws * (bt1D - st.bt1);
  F[D::bt2] += sws * (bt2D - st.bt2);
}

// One side from a 9-slot CONSERVED state (the Riemann problem of evolved
// conserved faces): the recovery cons_to_prim performs on the state with
// B_n := B_n*, with one reciprocal of the density.
template <class T, int AX>
PMHD_HD RSide<T> rside_cons(const T* U, T bns, const Phys<T>& ph) {
  using D = Dir<AX>;
  RSide<T> s;
  s.rho = vmax(U[RHO], rho_floor<T>());
  s.inv = fast_rcp(s.rho);
  s.vn = U[D::vn] * s.inv;
  s.vt1 = U[D::vt1] * s.inv;
  s.vt2 = U[D::vt2] * s.inv;
  s.bt1 = U[D::bt1];
  s.bt2 = U[D::bt2];
  s.bt2s = s.bt1 * s.bt1 + s.bt2 * s.bt2;
  const T v2 = s.vn * s.vn + s.vt1 * s.vt1 + s.vt2 * s.vt2;
  s.e = U[EN];
  s.p = ph.gm1 * (s.e - (T)0.5 * s.rho * v2 - (T)0.5 * (bns * bns + s.bt2s));
  return s;
}

template <class T, int AX>
PMHD_HD int hlld_core_fast(const RSide<T>& L, const RSide<T>& R, T bn, bool use_hlld, T* F, const Phys<T>& ph);

// GLM + HLLD (or HLL) interface flux along AX from the two face primitives
// (9 slots as reconstructed): the performance-build form of glm_flux /
// glm_flux_prim, same statuses.  F receives all nine slots.
template <class T, int AX>
PMHD_HD int glm_flux_fast(const T* PL, const T* PR, const GlmK<T>& g, bool use_hlld, T* F, const Phys<T>& ph) {
  using D = Dir<AX>;
  const T bnL0 = PL[D::bn], bnR0 = PR[D::bn], psiL = PL[PSI], psiR = PR[PSI];
  const T bn = (T)0.5 * (bnL0 + bnR0) - (psiR - psiL) * g.half_inv;
  F[D::bn] = (T)0.5 * (psiL + psiR) - (T)0.5 * g.ch_safe * (bnR0 - bnL0);
  F[PSI] = g.ch2 * bn;
  return hlld_core_fast<T, AX>(rside<T, AX>(PL, bnL0, bn, ph), rside<T, AX>(PR, bnR0, bn, ph), bn, use_hlld, F,
                               ph);
}

// The same from the two 9-slot conserved face states (performance-build form
// of glm_flux).
template <class T, int AX>
PMHD_HD int glm_flux_fast_cons(const T* UL, const T* UR, const GlmK<T>& g, bool use_hlld, T* F,
                               const Phys<T>& ph) {
  using D = Dir<AX>;
  const T bnL0 = UL[D::bn], bnR0 = UR[D::bn], psiL = UL[PSI], psiR = UR[PSI];
  const T bn = (T)0.5 * (bnL0 + bnR0) - (psiR - psiL) * g.half_inv;
  F[D::bn] = (T)0.5 * (psiL + psiR) - (T)0.5 * g.ch_safe * (bnR0 - bnL0);
  F[PSI] = g.ch2 * bn;
  return hlld_core_fast<T, AX>(rside_cons<T, AX>(UL, bn, ph), rside_cons<T, AX>(UR, bn, ph), bn, use_hlld, F, ph);
}

// HLLD (or HLL) on the eight MHD slots between two sides sharing the normal
// field bn; writes every slot of F but B_n and psi.
template <class T, int AX>
PMHD_HD int hlld_core_fast(const RSide<T>& L, const RSide<T>& R, T bn, bool use_hlld, T* F, const Phys<T>& ph) {
  const T bn2 = bn * bn;
  const T cfL = rside_cf<T>(L, bn2, ph), cfR = rside_cf<T>(R, bn2, ph);
  const T sL = vmin(L.vn - cfL, R.vn - cfR);
  const T sR = vmax(L.vn + cfL, R.vn + cfR);
  if (sL >= (T)0.0) {
    rside_flux<T, AX>(L, bn, bn2, F);
    return HLLD_OK;
  }
  if (sR <= (T)0.0) {
    rside_flux<T, AX>(R, bn, bn2, F);
    return HLLD_OK;
  }
  int status = HLLD_OK;
  if (use_hlld) {
    do {
      const T b2L = bn2 + L.bt2s, b2R = bn2 + R.bt2s;
      const T ptL = vmax(L.p, p_floor<T>()) + (T)0.5 * b2L;
      const T ptR = vmax(R.p, p_floor<T>()) + (T)0.5 * b2R;
      const T dL = L.rho * (sL - L.vn), dR = R.rho * (sR - R.vn);
      const T denom_sm = dR - dL;
      if (hlld_small(denom_sm, vabs(dR) + vabs(dL), ph) || bn2 <= ph.tol * ph.tol * vmax(b2L, b2R)) {
        status = HLLD_FALLBACK_DEGENERATE;
        break;
      }
      const T sm = (dR * R.vn - dL * L.vn + ptL - ptR) * fast_rcp(denom_sm);
      const T pts = (T)0.5 * ((ptL + dL * (sm - L.vn)) + (ptR + dR * (sm - R.vn)));
      RStar<T> Ls, Rs;
      const int stL = rside_star<T>(L, sL, sm, ptL, pts, bn, bn2, Ls, ph);
      const int stR = rside_star<T>(R, sR, sm, ptR, pts, bn, bn2, Rs, ph);
      if (stL != HLLD_OK || stR != HLLD_OK) {
        status = (stL != HLLD_OK) ? stL : stR;
        break;
      }
      const T isqL = fast_rsqrt(Ls.rho), isqR = fast_rsqrt(Rs.rho);
      const T sqL = Ls.rho * isqL, sqR = Rs.rho * isqR;
      const T sgn = (bn < (T)0.0) ? (T)-1.0 : (T)1.0;
      const T abn = vabs(bn);
      const T sLs = sm - abn * isqL, sRs = sm + abn * isqR;
      const T den = sqL + sqR;
      if (den <= (T)0.0) {
        status = HLLD_FALLBACK_DEGENERATE;
        break;
      }
      const T inv = fast_rcp(den);
      const T sq2 = sgn * sqL * sqR;
      const T vt1D = (sqL * Ls.vt1 + sqR * Rs.vt1 + sgn * (Rs.bt1 - Ls.bt1)) * inv;
      const T vt2D = (sqL * Ls.vt2 + sqR * Rs.vt2 + sgn * (Rs.bt2 - Ls.bt2)) * inv;
      const T bt1D = (sqL * Rs.bt1 + sqR * Ls.bt1 + sq2 * (Rs.vt1 - Ls.vt1)) * inv;
      const T bt2D = (sqL * Rs.bt2 + sqR * Ls.bt2 + sq2 * (Rs.vt2 - Ls.vt2)) * inv;
      const T vbD = sm * bn + vt1D * bt1D + vt2D * bt2D;
      const T eLD = Ls.e - sgn * sqL * (Ls.vb - vbD);
      const T eRD = Rs.e + sgn * sqR * (Rs.vb - vbD);
      const T v2D = sm * sm + vt1D * vt1D + vt2D * vt2D;
      const T b2D = bn2 + bt1D * bt1D + bt2D * bt2D;
      const T pLD = ph.gm1 * (eLD - (T)0.5 * Ls.rho * v2D - (T)0.5 * b2D);
      const T pRD = ph.gm1 * (eRD - (T)0.5 * Rs.rho * v2D - (T)0.5 * b2D);
      if (!(pLD > p_floor<T>() && pRD > p_floor<T>())) {
        status = HLLD_FALLBACK_NONPHYSICAL;
        break;
      }
      if (sm >= (T)0.0) {
        rside_flux<T, AX>(L, bn, bn2, F);
        rside_jump<T, AX>(L, Ls, sm, sL, F);
        if (sLs < (T)0.0) rside_jump2<T, AX>(Ls, vt1D, vt2D, bt1D, bt2D, eLD, sLs, F);
      } else {
        rside_flux<T, AX>(R, bn, bn2, F);
        rside_jump<T, AX>(R, Rs, sm, sR, F);
        if (sRs >= (T)0.0) rside_jump2<T, AX>(Rs, vt1D, vt2D, bt1D, bt2D, eRD, sRs, F);
      }
      return HLLD_OK;
    } while (false);
  }
  rside_hll<T, AX>(L, R, bn, bn2, sL, sR, F);
  return status;
}

// GLM-augmented physical flux along AX of a face given by its primitives P
// and total energy e (glm_phys_flux without recovering the primitives from
// the conserved state).
template <class T, int AX>
PMHD_HD void glm_phys_flux_prim(const T* P, T e, T ch2, T* F) {
  using D = Dir<AX>;
  phys_flux<T, AX>(P, e, F);
  F[D::bn] = P[PSI];
  F[PSI] = ch2 * P[D::bn];
}

// state_usable with one reciprocal of the density: density and pressure
// above the floors, all nine slots finite.
template <class T>
PMHD_HD bool state_usable_fast(const T* U, const Phys<T>& ph) {
  if (!(U[RHO] > rho_floor<T>())) return false;
  const T inv = fast_rcp(U[RHO]);
  const T m2 = U[MX] * U[MX] + U[MY] * U[MY] + U[MZ] * U[MZ];
  const T b2 = U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ];
  const T p = ph.gm1 * (U[EN] - (T)0.5 * m2 * inv - (T)0.5 * b2);
  T sum = U[0];
#pragma unroll
  for (int k = 1; k < NV9; k++) sum += U[k];
  return p > p_floor<T>() && vfinite(sum) && vfinite(p);
}

// Signal speed of one cell (cell_speed with one reciprocal of the density).
template <class T>
PMHD_HD T cell_speed_fast(const T* P, const Phys<T>& ph) {
  const T inv = fast_rcp(vmax(P[RHO], rho_floor<T>()));
  const T a2 = ph.gamma * vmax(P[EN], p_floor<T>()) * inv;
  const T bx2 = P[BX] * P[BX], by2 = P[BY] * P[BY];
  const T b2 = (bx2 + by2 + P[BZ] * P[BZ]) * inv;
  const T sum = a2 + b2, s2 = sum * sum, a4 = (T)4.0 * a2 * inv;
  const T cfx = fast_sqrt(vmax((T)0.5 * (sum + fast_sqrt(vmax(s2 - a4 * bx2, (T)0.0))), (T)0.0));
  const T cfy = fast_sqrt(vmax((T)0.5 * (sum + fast_sqrt(vmax(s2 - a4 * by2, (T)0.0))), (T)0.0));
  return vmax(vabs(P[MX]) + cfx, vabs(P[MY]) + cfy);
}

// Minmod as min/max selections: minmod(a, b) = max(min(a, b), min(max(a, b),
// 0)); the same value as minmod() for finite arguments.
template <class T>
PMHD_HD T minmod_fast(T a, T b) {
  return vmax(vmin(a, b), vmin(vmax(a, b), (T)0.0));
}

}  // namespace pmhd

#endif  // PMHD_POINT_HPP
