// Drop-in for the reference's header-only Real/HD point interface.
//
// Code written against the reference's include/mhd/mhd_glm_common.hpp (which
// includes mhd_common.hpp and base.hpp) compiles unchanged against this
// header by putting include/pmhd/compat first on the include path.  The same
// knobs apply: USE_FLOAT selects Real = float, MHD_GAMMA_VALUE and
// MHD_HLLD_TOLERANCE_VALUE are compile-time constants with the reference's
// defaults (2.0 and 1e-6).  Every function forwards to the templates of
// pmhd/point.hpp with the macro values, so results and status codes equal
// the reference's.
//
// Names and signatures mirror include/base.hpp:21-31,
// include/mhd/mhd_common.hpp:46-667 and include/mhd/mhd_glm_common.hpp:26-126.
#ifndef PMHD_COMPAT_MHD_GLM_COMMON_HPP
#define PMHD_COMPAT_MHD_GLM_COMMON_HPP

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

#ifdef USE_FLOAT
typedef float Real;
#else
typedef double Real;
#endif

#include "../../point.hpp"

#ifndef MHD_GAMMA_VALUE
#define MHD_GAMMA_VALUE 2.0
#endif
#ifndef MHD_HLLD_TOLERANCE_VALUE
#define MHD_HLLD_TOLERANCE_VALUE 1.0e-6
#endif

static const int MHD_NVAR = 8;
static const Real MHD_GAMMA = (Real)MHD_GAMMA_VALUE;
static const Real MHD_RHO_FLOOR = (Real)1.0e-12;
static const Real MHD_P_FLOOR = (Real)1.0e-12;
static const int MHD_GLM_NVAR = 9;
static const int MHD_GLM_PSI = 8;
static const int MHD_HLLD_OK = pmhd::HLLD_OK;
static const int MHD_HLLD_FALLBACK_DEGENERATE = pmhd::HLLD_FALLBACK_DEGENERATE;
static const int MHD_HLLD_FALLBACK_NONPHYSICAL = pmhd::HLLD_FALLBACK_NONPHYSICAL;

enum MHDIndex { MHD_RHO = 0, MHD_MX = 1, MHD_MY = 2, MHD_MZ = 3, MHD_E = 4, MHD_BX = 5, MHD_BY = 6, MHD_BZ = 7 };
enum MHDPrimIndex {
  MHD_PR_RHO = 0, MHD_PR_VX = 1, MHD_PR_VY = 2, MHD_PR_VZ = 3,
  MHD_PR_P = 4, MHD_PR_BX = 5, MHD_PR_BY = 6, MHD_PR_BZ = 7
};

__host__ __device__ inline pmhd::Phys<Real> mhdCompatPhys() {
  pmhd::Phys<Real> p;
  p.gamma = MHD_GAMMA;
  p.gm1 = MHD_GAMMA - (Real)1.0;
  p.tol = (Real)MHD_HLLD_TOLERANCE_VALUE;
  return p;
}

__host__ __device__ inline Real mhdMax(Real a, Real b) { return pmhd::vmax(a, b); }
__host__ __device__ inline Real mhdMin(Real a, Real b) { return pmhd::vmin(a, b); }
__host__ __device__ inline Real mhdAbs(Real a) { return pmhd::vabs(a); }
__host__ __device__ inline Real mhdSqrt(Real a) { return pmhd::vsqrt(a); }
__host__ __device__ inline Real mhdMinmod(Real a, Real b) { return pmhd::minmod(a, b); }
__host__ __device__ inline void mhdPrimToCons(const Real W[8], Real U[8]) {
  pmhd::prim_to_cons<Real>(W, U, mhdCompatPhys());
}
__host__ __device__ inline void mhdConsToPrim(const Real U[8], Real W[8]) {
  pmhd::cons_to_prim<Real, 0>(U, W, mhdCompatPhys());
}
__host__ __device__ inline Real mhdFastSpeedX(const Real W[8]) {
  return pmhd::fast_speed<Real, 0>(W, mhdCompatPhys());
}
__host__ __device__ inline Real mhdFastSpeedY(const Real W[8]) {
  return pmhd::fast_speed<Real, 1>(W, mhdCompatPhys());
}
__host__ __device__ inline void mhdFluxXW(const Real W[8], Real e, Real F[8]) {
  pmhd::phys_flux<Real, 0>(W, e, F);
}
__host__ __device__ inline void mhdFluxYW(const Real W[8], Real e, Real G[8]) {
  pmhd::phys_flux<Real, 1>(W, e, G);
}
__host__ __device__ inline void mhdFluxX(const Real U[8], Real F[8]) {
  Real W[8];
  mhdConsToPrim(U, W);
  mhdFluxXW(W, U[MHD_E], F);
}
__host__ __device__ inline void mhdFluxY(const Real U[8], Real G[8]) {
  Real W[8];
  mhdConsToPrim(U, W);
  mhdFluxYW(W, U[MHD_E], G);
}
__host__ __device__ inline void mhdHllFluxX(const Real UL[8], const Real UR[8], Real F[8]) {
  pmhd::hll_flux<Real, 0>(UL, UR, F, mhdCompatPhys());
}
__host__ __device__ inline void mhdHllFluxY(const Real UL[8], const Real UR[8], Real G[8]) {
  pmhd::hll_flux<Real, 1>(UL, UR, G, mhdCompatPhys());
}
__host__ __device__ inline void mhdRotateYToX(const Real Uy[8], Real Ux[8]) {
  const int perm[8] = {0, 2, 1, 3, 4, 6, 5, 7};
  for (int k = 0; k < 8; k++) Ux[k] = Uy[perm[k]];
}
__host__ __device__ inline void mhdRotateFluxXToY(const Real Fx[8], Real Gy[8]) {
  mhdRotateYToX(Fx, Gy);
}
__host__ __device__ inline Real mhdSignNonZero(Real a) { return (a < (Real)0.0) ? (Real)-1.0 : (Real)1.0; }
__host__ __device__ inline Real mhdHlldTolerance() { return (Real)MHD_HLLD_TOLERANCE_VALUE; }
__host__ __device__ inline bool mhdHlldIsSmall(Real value, Real scale) {
  return pmhd::hlld_small(value, scale, mhdCompatPhys());
}
__host__ __device__ inline bool mhdConservedHasPositivePressure(const Real U[8]) {
  return pmhd::positive_state<Real, 0>(U, mhdCompatPhys());
}
__host__ __device__ inline int mhdHlldStarStateX(const Real U[8], const Real W[8], Real s, Real sm,
                                                 Real pt_star, Real bx, Real Ustar[8]) {
  Real vts[2];
  return pmhd::hlld_star<Real, 0>(U, W, s, sm, pt_star, bx, Ustar, vts, mhdCompatPhys());
}
__host__ __device__ inline int mhdHlldFluxX(const Real UL[8], const Real UR[8], Real F[8]) {
  return pmhd::hlld_flux<Real, 0>(UL, UR, F, mhdCompatPhys());
}
__host__ __device__ inline int mhdHlldFluxY(const Real UL[8], const Real UR[8], Real G[8]) {
  return pmhd::hlld_flux<Real, 1>(UL, UR, G, mhdCompatPhys());
}
__host__ __device__ inline void mhdGlmExtractMhdState(const Real U9[9], Real U8[8]) {
  for (int k = 0; k < 8; k++) U8[k] = U9[k];
}
__host__ __device__ inline void mhdGlmPrimToCons(const Real W[8], Real psi, Real U9[9]) {
  mhdPrimToCons(W, U9);
  U9[MHD_GLM_PSI] = psi;
}
__host__ __device__ inline void mhdGlmConsToPrim(const Real U9[9], Real W[8], Real& psi) {
  mhdConsToPrim(U9, W);
  psi = U9[MHD_GLM_PSI];
}
__host__ __device__ inline void mhdGlmNormalState(Real bnL, Real bnR, Real psiL, Real psiR, Real ch,
                                                  Real& bnStar, Real& psiStar) {
  const Real ch_safe = pmhd::vmax(ch, (Real)1.0e-12);
  bnStar = (Real)0.5 * (bnL + bnR) - (Real)0.5 * (psiR - psiL) / ch_safe;
  psiStar = (Real)0.5 * (psiL + psiR) - (Real)0.5 * ch_safe * (bnR - bnL);
}
__host__ __device__ inline int mhdGlmFluxX(const Real UL[9], const Real UR[9], Real ch, bool use_hlld,
                                           Real F[9]) {
  return pmhd::glm_flux<Real, 0>(UL, UR, ch, use_hlld, F, mhdCompatPhys());
}
__host__ __device__ inline int mhdGlmFluxY(const Real UL[9], const Real UR[9], Real ch, bool use_hlld,
                                           Real G[9]) {
  return pmhd::glm_flux<Real, 1>(UL, UR, ch, use_hlld, G, mhdCompatPhys());
}

#endif  // PMHD_COMPAT_MHD_GLM_COMMON_HPP
