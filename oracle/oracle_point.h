/*
 * oracle_point.h -- TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into
 * the product library or the CLI.
 *
 * Plain-C restatement of the reference's per-point ideal-MHD + mixed-GLM
 * numerics.  This file is a C "template": pmhd_oracle.c includes it once per
 * arithmetic type with
 *     OT   -- the arithmetic type (double or float)
 *     OS   -- the name suffix (f64 or f32)
 * defined, producing e.g. or_hlld_x_f64() and or_hlld_x_f32().
 *
 * Every expression keeps the reference's operation order (left-to-right
 * association of + - * /, no reciprocal-multiply) so that the f64 build is
 * bit-identical to the reference CPU build.  Comparisons use the std::max /
 * std::min semantics of the reference CPU path.  Physical constants (gamma,
 * HLLD tolerance) are runtime parameters here; the reference makes them
 * compile-time constants (include/mhd/mhd_common.hpp:52-79), which produces
 * the same bits because (gamma - 1) and tol*scale are evaluated identically.
 *
 * Reference anchors (paths inside the reference project):
 *   include/mhd/mhd_common.hpp      -- 8-variable MHD point functions
 *   include/mhd/mhd_glm_common.hpp  -- 9-variable GLM extension
 */

#define OR_CAT2(a, b) a##_##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define OF(name) OR_CAT(name, OS)

/* Physical parameters of one run. */
typedef struct {
  OT gamma;
  OT tol;
} OF(or_phys);

/* std::max(a,b) / std::min(a,b) semantics (mhd_common.hpp:106-120, host branch). */
static inline OT OF(or_max)(OT a, OT b) { return (a < b) ? b : a; }
static inline OT OF(or_min)(OT a, OT b) { return (b < a) ? b : a; }
static inline OT OF(or_abs)(OT a) { return (OT)fabs((double)a); }
static inline OT OF(or_sqrt)(OT a) { return (OT)sqrt((double)a); }

#define OR_RHO_FLOOR ((OT)1.0e-12)
#define OR_P_FLOOR ((OT)1.0e-12)

/* mhdMinmod, mhd_common.hpp:140-143 */
static inline OT OF(or_minmod)(OT a, OT b) {
  if (a * b <= (OT)0.0) return (OT)0.0;
  return (OF(or_abs)(a) < OF(or_abs)(b)) ? a : b;
}

/* mhdPrimToCons, mhd_common.hpp:149-173 */
static void OF(or_prim_to_cons)(const OT W[8], OT U[8], const OF(or_phys) * ph) {
  OT rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
  OT bx = W[5], by = W[6], bz = W[7];
  OT v2 = vx * vx + vy * vy + vz * vz;
  OT b2 = bx * bx + by * by + bz * bz;
  U[0] = rho;
  U[1] = rho * vx;
  U[2] = rho * vy;
  U[3] = rho * vz;
  U[4] = p / (ph->gamma - (OT)1.0) + (OT)0.5 * rho * v2 + (OT)0.5 * b2;
  U[5] = bx;
  U[6] = by;
  U[7] = bz;
}

/* mhdConsToPrim, mhd_common.hpp:178-201 */
static void OF(or_cons_to_prim)(const OT U[8], OT W[8], const OF(or_phys) * ph) {
  OT rho = OF(or_max)(U[0], OR_RHO_FLOOR);
  OT vx = U[1] / rho, vy = U[2] / rho, vz = U[3] / rho;
  OT bx = U[5], by = U[6], bz = U[7];
  OT v2 = vx * vx + vy * vy + vz * vz;
  OT b2 = bx * bx + by * by + bz * bz;
  OT p = (ph->gamma - (OT)1.0) * (U[4] - (OT)0.5 * rho * v2 - (OT)0.5 * b2);
  W[0] = rho; W[1] = vx; W[2] = vy; W[3] = vz; W[4] = p;
  W[5] = bx; W[6] = by; W[7] = bz;
}

/* mhdFastSpeedX / mhdFastSpeedY, mhd_common.hpp:206-238.  bn is the field
 * component along the direction (W[5] for x, W[6] for y). */
static OT OF(or_fast_speed)(const OT W[8], OT bn, const OF(or_phys) * ph) {
  OT rho = OF(or_max)(W[0], OR_RHO_FLOOR);
  OT p = OF(or_max)(W[4], OR_P_FLOOR);
  OT bx = W[5], by = W[6], bz = W[7];
  OT a2 = ph->gamma * p / rho;
  OT b2 = (bx * bx + by * by + bz * bz) / rho;
  OT can2 = bn * bn / rho;
  OT disc = (a2 + b2) * (a2 + b2) - (OT)4.0 * a2 * can2;
  disc = OF(or_max)(disc, (OT)0.0);
  OT cf2 = (OT)0.5 * (a2 + b2 + OF(or_sqrt)(disc));
  return OF(or_sqrt)(OF(or_max)(cf2, (OT)0.0));
}

/* mhdFluxXW, mhd_common.hpp:247-270 */
static void OF(or_flux_x_w)(const OT W[8], OT e, OT F[8]) {
  OT rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
  OT bx = W[5], by = W[6], bz = W[7];
  OT b2 = bx * bx + by * by + bz * bz;
  OT ptot = p + (OT)0.5 * b2;
  OT vdotb = vx * bx + vy * by + vz * bz;
  F[0] = rho * vx;
  F[1] = rho * vx * vx + ptot - bx * bx;
  F[2] = rho * vx * vy - bx * by;
  F[3] = rho * vx * vz - bx * bz;
  F[4] = (e + ptot) * vx - bx * vdotb;
  F[5] = (OT)0.0;
  F[6] = vx * by - bx * vy;
  F[7] = vx * bz - bx * vz;
}

/* mhdFluxYW, mhd_common.hpp:285-308 */
static void OF(or_flux_y_w)(const OT W[8], OT e, OT G[8]) {
  OT rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
  OT bx = W[5], by = W[6], bz = W[7];
  OT b2 = bx * bx + by * by + bz * bz;
  OT ptot = p + (OT)0.5 * b2;
  OT vdotb = vx * bx + vy * by + vz * bz;
  G[0] = rho * vy;
  G[1] = rho * vy * vx - by * bx;
  G[2] = rho * vy * vy + ptot - by * by;
  G[3] = rho * vy * vz - by * bz;
  G[4] = (e + ptot) * vy - by * vdotb;
  G[5] = vy * bx - by * vx;
  G[6] = (OT)0.0;
  G[7] = vy * bz - by * vz;
}

/* mhdHllFluxX (dir 0) / mhdHllFluxY (dir 1), mhd_common.hpp:323-377 */
static void OF(or_hll)(const OT UL[8], const OT UR[8], OT F[8], int dir,
                       const OF(or_phys) * ph) {
  OT WL[8], WR[8], FL[8], FR[8];
  int k;
  OF(or_cons_to_prim)(UL, WL, ph);
  OF(or_cons_to_prim)(UR, WR, ph);
  int vn = dir ? 2 : 1;
  int bnk = dir ? 6 : 5;
  if (dir) {
    OF(or_flux_y_w)(WL, UL[4], FL);
    OF(or_flux_y_w)(WR, UR[4], FR);
  } else {
    OF(or_flux_x_w)(WL, UL[4], FL);
    OF(or_flux_x_w)(WR, UR[4], FR);
  }
  OT cfL = OF(or_fast_speed)(WL, WL[bnk], ph);
  OT cfR = OF(or_fast_speed)(WR, WR[bnk], ph);
  OT sL = OF(or_min)(WL[vn] - cfL, WR[vn] - cfR);
  OT sR = OF(or_max)(WL[vn] + cfL, WR[vn] + cfR);
  if (sL >= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FL[k];
  } else if (sR <= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FR[k];
  } else {
    OT denom = sR - sL;
    for (k = 0; k < 8; k++)
      F[k] = (sR * FL[k] - sL * FR[k] + sL * sR * (UR[k] - UL[k])) / denom;
  }
}

static int OF(or_small)(OT v, OT scale, const OF(or_phys) * ph) {
  return OF(or_abs)(v) <= ph->tol * scale; /* mhdHlldIsSmall, mhd_common.hpp:417-419 */
}

/* mhdConservedHasPositivePressure, mhd_common.hpp:426-431 */
static int OF(or_positive)(const OT U[8], const OF(or_phys) * ph) {
  OT W[8];
  if (!(U[0] > OR_RHO_FLOOR)) return 0;
  OF(or_cons_to_prim)(U, W, ph);
  return (W[0] > OR_RHO_FLOOR && W[4] > OR_P_FLOOR);
}

/* mhdHlldStarStateX, mhd_common.hpp:445-511 */
static int OF(or_star)(const OT U[8], const OT W[8], OT s, OT sm, OT pt_star,
                       OT bx, OT Us[8], const OF(or_phys) * ph) {
  OT rho = OF(or_max)(W[0], OR_RHO_FLOOR);
  OT vx = W[1], vy = W[2], vz = W[3];
  OT p = OF(or_max)(W[4], OR_P_FLOOR);
  OT by = W[6], bz = W[7];
  OT e = U[4];
  OT smv = s - vx;
  OT sms = s - sm;
  OT wave_scale = OF(or_max)(OF(or_abs)(s), OF(or_abs)(sm));
  if (OF(or_small)(sms, wave_scale, ph)) return 1;
  OT rho_s = rho * smv / sms;
  if (rho_s <= OR_RHO_FLOOR) return 2;
  OT denom = rho * smv * sms - bx * bx;
  OT denom_scale = OF(or_abs)(rho * smv * sms) + bx * bx;
  if (OF(or_small)(denom, denom_scale, ph)) return 1;
  OT common = sm - vx;
  OT vy_s = vy - bx * by * common / denom;
  OT vz_s = vz - bx * bz * common / denom;
  OT by_s = by * (rho * smv * smv - bx * bx) / denom;
  OT bz_s = bz * (rho * smv * smv - bx * bx) / denom;
  OT b2 = bx * bx + by * by + bz * bz;
  OT pt = p + (OT)0.5 * b2;
  OT vdotb = vx * bx + vy * by + vz * bz;
  OT vsbs = sm * bx + vy_s * by_s + vz_s * bz_s;
  OT e_s = (smv * e - pt * vx + pt_star * sm + bx * (vdotb - vsbs)) / sms;
  Us[0] = rho_s;
  Us[1] = rho_s * sm;
  Us[2] = rho_s * vy_s;
  Us[3] = rho_s * vz_s;
  Us[4] = e_s;
  Us[5] = bx;
  Us[6] = by_s;
  Us[7] = bz_s;
  return OF(or_positive)(Us, ph) ? 0 : 2;
}

/* mhdHlldFluxX, mhd_common.hpp:518-654.  Returns 0 ok, 1 degenerate, 2
 * non-physical (the last two fall back to HLL). */
static int OF(or_hlld_x)(const OT UL[8], const OT UR[8], OT F[8],
                         const OF(or_phys) * ph) {
  OT WL[8], WR[8], FL[8], FR[8];
  int k;
  OF(or_cons_to_prim)(UL, WL, ph);
  OF(or_cons_to_prim)(UR, WR, ph);
  OF(or_flux_x_w)(WL, UL[4], FL);
  OF(or_flux_x_w)(WR, UR[4], FR);
  OT cfL = OF(or_fast_speed)(WL, WL[5], ph);
  OT cfR = OF(or_fast_speed)(WR, WR[5], ph);
  OT sL = OF(or_min)(WL[1] - cfL, WR[1] - cfR);
  OT sR = OF(or_max)(WL[1] + cfL, WR[1] + cfR);
  if (sL >= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FL[k];
    return 0;
  }
  if (sR <= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FR[k];
    return 0;
  }
  OT rhoL = OF(or_max)(WL[0], OR_RHO_FLOOR);
  OT rhoR = OF(or_max)(WR[0], OR_RHO_FLOOR);
  OT vxL = WL[1], vxR = WR[1];
  OT bx = (OT)0.5 * (WL[5] + WR[5]);
  OT b2L = bx * bx + WL[6] * WL[6] + WL[7] * WL[7];
  OT b2R = bx * bx + WR[6] * WR[6] + WR[7] * WR[7];
  OT ptL = OF(or_max)(WL[4], OR_P_FLOOR) + (OT)0.5 * b2L;
  OT ptR = OF(or_max)(WR[4], OR_P_FLOOR) + (OT)0.5 * b2R;
  OT denom_sm = rhoR * (sR - vxR) - rhoL * (sL - vxL);
  OT denom_sm_scale = OF(or_abs)(rhoR * (sR - vxR)) + OF(or_abs)(rhoL * (sL - vxL));
  OT b_scale = OF(or_sqrt)(OF(or_max)(b2L, b2R));
  if (OF(or_small)(denom_sm, denom_sm_scale, ph) || OF(or_small)(bx, b_scale, ph)) {
    OF(or_hll)(UL, UR, F, 0, ph);
    return 1;
  }
  OT sm = (rhoR * vxR * (sR - vxR) - rhoL * vxL * (sL - vxL) + ptL - ptR) / denom_sm;
  OT ptsL = ptL + rhoL * (sL - vxL) * (sm - vxL);
  OT ptsR = ptR + rhoR * (sR - vxR) * (sm - vxR);
  OT pts = (OT)0.5 * (ptsL + ptsR);
  OT ULs[8], URs[8];
  int stL = OF(or_star)(UL, WL, sL, sm, pts, bx, ULs, ph);
  int stR = OF(or_star)(UR, WR, sR, sm, pts, bx, URs, ph);
  if (stL != 0 || stR != 0) {
    OF(or_hll)(UL, UR, F, 0, ph);
    return (stL != 0) ? stL : stR;
  }
  OT sqL = OF(or_sqrt)(OF(or_max)(ULs[0], OR_RHO_FLOOR));
  OT sqR = OF(or_sqrt)(OF(or_max)(URs[0], OR_RHO_FLOOR));
  OT sgn = (bx < (OT)0.0) ? (OT)-1.0 : (OT)1.0;
  OT sLs = sm - OF(or_abs)(bx) / sqL;
  OT sRs = sm + OF(or_abs)(bx) / sqR;
  OT den = sqL + sqR;
  if (den <= (OT)0.0) {
    OF(or_hll)(UL, UR, F, 0, ph);
    return 1;
  }
  OT vyLs = ULs[2] / ULs[0], vzLs = ULs[3] / ULs[0];
  OT byLs = ULs[6], bzLs = ULs[7];
  OT vyRs = URs[2] / URs[0], vzRs = URs[3] / URs[0];
  OT byRs = URs[6], bzRs = URs[7];
  OT vyD = (sqL * vyLs + sqR * vyRs + sgn * (byRs - byLs)) / den;
  OT vzD = (sqL * vzLs + sqR * vzRs + sgn * (bzRs - bzLs)) / den;
  OT byD = (sqL * byRs + sqR * byLs + sgn * sqL * sqR * (vyRs - vyLs)) / den;
  OT bzD = (sqL * bzRs + sqR * bzLs + sgn * sqL * sqR * (vzRs - vzLs)) / den;
  OT ULD[8], URD[8];
  for (k = 0; k < 8; k++) { ULD[k] = ULs[k]; URD[k] = URs[k]; }
  ULD[2] = ULD[0] * vyD; ULD[3] = ULD[0] * vzD; ULD[6] = byD; ULD[7] = bzD;
  URD[2] = URD[0] * vyD; URD[3] = URD[0] * vzD; URD[6] = byD; URD[7] = bzD;
  OT vbLD = sm * bx + vyD * byD + vzD * bzD;
  OT vbLs = sm * bx + vyLs * byLs + vzLs * bzLs;
  OT vbRD = vbLD;
  OT vbRs = sm * bx + vyRs * byRs + vzRs * bzRs;
  ULD[4] = ULs[4] - sgn * sqL * (vbLs - vbLD);
  URD[4] = URs[4] + sgn * sqR * (vbRs - vbRD);
  if (!OF(or_positive)(ULD, ph) || !OF(or_positive)(URD, ph)) {
    OF(or_hll)(UL, UR, F, 0, ph);
    return 2;
  }
  if (sLs >= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FL[k] + sL * (ULs[k] - UL[k]);
  } else if (sm >= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FL[k] + sL * (ULs[k] - UL[k]) + sLs * (ULD[k] - ULs[k]);
  } else if (sRs >= (OT)0.0) {
    for (k = 0; k < 8; k++) F[k] = FR[k] + sR * (URs[k] - UR[k]) + sRs * (URD[k] - URs[k]);
  } else {
    for (k = 0; k < 8; k++) F[k] = FR[k] + sR * (URs[k] - UR[k]);
  }
  return 0;
}

/* mhdRotateYToX / mhdRotateFluxXToY (mhd_common.hpp:381-405): swap the x and
 * y slots of momentum and field.  The permutation is its own inverse. */
static void OF(or_swap_xy)(const OT a[8], OT b[8]) {
  b[0] = a[0]; b[1] = a[2]; b[2] = a[1]; b[3] = a[3];
  b[4] = a[4]; b[5] = a[6]; b[6] = a[5]; b[7] = a[7];
}

/* mhdHlldFluxY, mhd_common.hpp:658-667 */
static int OF(or_hlld_y)(const OT UL[8], const OT UR[8], OT G[8],
                         const OF(or_phys) * ph) {
  OT a[8], b[8], f[8];
  OF(or_swap_xy)(UL, a);
  OF(or_swap_xy)(UR, b);
  int st = OF(or_hlld_x)(a, b, f, ph);
  OF(or_swap_xy)(f, G);
  return st;
}

/* mhdGlmNormalState + mhdGlmFluxX/Y, mhd_glm_common.hpp:55-126.  dir 0 = x,
 * 1 = y.  Returns the HLLD status (always 0 for HLL). */
static int OF(or_glm_flux)(const OT UL[9], const OT UR[9], OT ch, int use_hlld,
                           int dir, OT F[9], const OF(or_phys) * ph) {
  int bn = dir ? 6 : 5;
  OT ch_safe = OF(or_max)(ch, (OT)1.0e-12);
  OT bnL = UL[bn], bnR = UR[bn], psiL = UL[8], psiR = UR[8];
  OT bns = (OT)0.5 * (bnL + bnR) - (OT)0.5 * (psiR - psiL) / ch_safe;
  OT psis = (OT)0.5 * (psiL + psiR) - (OT)0.5 * ch_safe * (bnR - bnL);
  OT a[8], b[8], f[8];
  int k, st = 0;
  for (k = 0; k < 8; k++) { a[k] = UL[k]; b[k] = UR[k]; }
  a[bn] = bns;
  b[bn] = bns;
  if (use_hlld) {
    st = dir ? OF(or_hlld_y)(a, b, f, ph) : OF(or_hlld_x)(a, b, f, ph);
  } else {
    OF(or_hll)(a, b, f, dir, ph);
  }
  for (k = 0; k < 8; k++) F[k] = f[k];
  F[bn] = psis;
  F[8] = ch * ch * bns;
  return st;
}

/* stateToPrimitive (mhd2d_glm_cpu.cpp:90-96): 9-slot primitive with psi. */
static void OF(or_state_to_prim9)(const OT U[9], OT P[9], const OF(or_phys) * ph) {
  OF(or_cons_to_prim)(U, P, ph);
  P[8] = U[8];
}

/* primitiveToState (mhd2d_glm_cpu.cpp:98-103) */
static void OF(or_prim9_to_state)(const OT P[9], OT U[9], const OF(or_phys) * ph) {
  OF(or_prim_to_cons)(P, U, ph);
  U[8] = P[8];
}

/* primitiveIsUsable (mhd2d_glm_cpu.cpp:105-111) */
static int OF(or_prim9_usable)(const OT P[9]) {
  int k;
  if (P[0] <= OR_RHO_FLOOR || P[4] <= OR_P_FLOOR) return 0;
  for (k = 0; k < 9; k++)
    if (!isfinite((double)P[k])) return 0;
  return 1;
}

/* stateIsUsable (mhd2d_glm_cpu.cpp:113-118) */
static int OF(or_state_usable)(const OT U[9], const OF(or_phys) * ph) {
  OT P[9];
  if (U[0] <= OR_RHO_FLOOR) return 0;
  OF(or_state_to_prim9)(U, P, ph);
  return OF(or_prim9_usable)(P);
}

/* reconstructPrimitive (mhd2d_glm_cpu.cpp:144-161): minmod slopes on all 9
 * primitives, first-order fallback when either face is unusable. */
static void OF(or_recon)(const OT Pm[9], const OT P0[9], const OT Pp[9],
                         OT Pl[9], OT Pr[9]) {
  int k;
  for (k = 0; k < 9; k++) {
    OT slope = OF(or_minmod)(P0[k] - Pm[k], Pp[k] - P0[k]);
    Pl[k] = P0[k] - (OT)0.5 * slope;
    Pr[k] = P0[k] + (OT)0.5 * slope;
  }
  if (!OF(or_prim9_usable)(Pl) || !OF(or_prim9_usable)(Pr)) {
    for (k = 0; k < 9; k++) { Pl[k] = P0[k]; Pr[k] = P0[k]; }
  }
}

/* Signal speed of one cell: max(|vx|+cfx, |vy|+cfy) (mhd2d_glm_cpu.cpp:298-301). */
static OT OF(or_cell_speed)(const OT P[9], const OF(or_phys) * ph) {
  OT sx = OF(or_abs)(P[1]) + OF(or_fast_speed)(P, P[5], ph);
  OT sy = OF(or_abs)(P[2]) + OF(or_fast_speed)(P, P[6], ph);
  return OF(or_max)(sx, sy);
}

#undef OF
#undef OR_CAT
#undef OR_CAT2
#undef OR_RHO_FLOOR
#undef OR_P_FLOOR
