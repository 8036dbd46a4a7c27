/* euler_oracle.h -- CPU restatement of the reference's Euler sibling (the
 * 1D and 2D MUSCL-Hancock + HLLC / HLL drivers), instantiated for binary64
 * (ET = double, EF = f64) and binary32 (ET = float, EF = f32) by
 * euler_oracle.c.  TEST INFRASTRUCTURE ONLY: used by tests/ as the checker
 * of the GPU Euler kernels, never by the product.
 *
 * Follows src/euler/riemann1d_cpu.cpp:95-214,
 * src/euler/riemann2d_cpu.cpp:108-330 and src/euler/euler2d_cpu.cpp:53-398
 * (same loops, ghost handling and
 * expression order, gamma a binary64 constant as in
 * include/euler/config.hpp:43) with the point functions of
 * include/euler/euler_common.hpp and include/euler/riemann.hpp. */
#define EG 1.4
#define ECAT2(a, b) a##_##b
#define ECAT(a, b) ECAT2(a, b)
#define EN(name) ECAT(name, EF)

static ET EN(eo_min)(ET a, ET b) { return (b < a) ? b : a; }
static ET EN(eo_max)(ET a, ET b) { return (a < b) ? b : a; }
static ET EN(eo_sound)(ET p, ET rho) { return (ET)sqrt(EG * p / rho); }
static ET EN(eo_minmod)(ET a, ET b) {
  if (a * b <= (ET)0.0) return (ET)0.0;
  return (fabs(a) < fabs(b)) ? a : b;
}
static void EN(eo_c2p)(const ET U[4], ET W[4]) {
  ET r = U[0];
  W[0] = r;
  W[1] = U[1] / r;
  W[2] = U[2] / r;
  W[3] = (ET)((EG - (ET)1.0) * (U[3] - (ET)0.5 * (U[1] * U[1] + U[2] * U[2]) / r));
}
static void EN(eo_p2c)(const ET W[4], ET U[4]) {
  U[0] = W[0];
  U[1] = W[0] * W[1];
  U[2] = W[0] * W[2];
  U[3] = (ET)(W[3] / (EG - (ET)1.0) + (ET)0.5 * W[0] * (W[1] * W[1] + W[2] * W[2]));
}
static void EN(eo_recon)(ET qm, ET q0, ET qp, ET* ql, ET* qr) {
  ET s = EN(eo_minmod)(q0 - qm, qp - q0);
  *ql = q0 - (ET)0.5 * s;
  *qr = q0 + (ET)0.5 * s;
}
/* riemann.hpp:60-88 */
static void EN(eo_hancock)(const ET Wf[4], const ET Wl[4], const ET Wr[4], ET Wh[4], ET fac, int n, int tt) {
  ET Uf[4], dF[4], Uh[4];
  int k;
  EN(eo_p2c)(Wf, Uf);
  ET rL = Wl[0], uL = Wl[n], vL = Wl[tt], pL = Wl[3];
  ET rR = Wr[0], uR = Wr[n], vR = Wr[tt], pR = Wr[3];
  ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rL * (uL * uL + vL * vL));
  ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rR * (uR * uR + vR * vR));
  dF[0] = rR * uR - rL * uL;
  dF[n] = (rR * uR * uR + pR) - (rL * uL * uL + pL);
  dF[tt] = rR * uR * vR - rL * uL * vL;
  dF[3] = (ER + pR) * uR - (EL + pL) * uL;
  for (k = 0; k < 4; k++) Uh[k] = Uf[k] - fac * dF[k];
  EN(eo_c2p)(Uh, Wh);
}
/* riemann.hpp:98-150 (x) and :158-210 (y): the y form multiplies the
 * tangential momentum flux as rho * u_t * u_n, the x form as rho * u_n * u_t. */
static ET EN(eo_tflux)(ET rho, ET un, ET ut, int n) { return n == 1 ? rho * un * ut : rho * ut * un; }
static void EN(eo_hllc)(const ET WL[4], const ET WR[4], ET f[4], int n, int tt) {
  ET rhoL = WL[0], uL = WL[n], vL = WL[tt], pL = WL[3];
  ET rhoR = WR[0], uR = WR[n], vR = WR[tt], pR = WR[3];
  ET cL = EN(eo_sound)(pL, rhoL), cR = EN(eo_sound)(pR, rhoR);
  ET SL = EN(eo_min)(uL - cL, uR - cR), SR = EN(eo_max)(uL + cL, uR + cR);
  ET denom = rhoL * (SL - uL) - rhoR * (SR - uR);
  ET Ss = (pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR)) / denom;
  ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rhoL * (uL * uL + vL * vL));
  ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rhoR * (uR * uR + vR * vR));
  if (SL > (ET)0.0) {
    f[0] = rhoL * uL;
    f[n] = rhoL * uL * uL + pL;
    f[tt] = EN(eo_tflux)(rhoL, uL, vL, n);
    f[3] = (EL + pL) * uL;
  } else if (Ss > (ET)0.0) {
    ET c = rhoL * (SL - uL) / (SL - Ss);
    ET U0 = c, U1 = c * Ss, U2 = c * vL, U3 = c * (EL / rhoL + (Ss - uL) * (Ss + pL / (rhoL * (SL - uL))));
    ET f0 = rhoL * uL, f1 = rhoL * uL * uL + pL, f2 = EN(eo_tflux)(rhoL, uL, vL, n), f3 = (EL + pL) * uL;
    f[0] = f0 + SL * (U0 - rhoL);
    f[n] = f1 + SL * (U1 - rhoL * uL);
    f[tt] = f2 + SL * (U2 - rhoL * vL);
    f[3] = f3 + SL * (U3 - EL);
  } else if (SR > (ET)0.0) {
    ET c = rhoR * (SR - uR) / (SR - Ss);
    ET U0 = c, U1 = c * Ss, U2 = c * vR, U3 = c * (ER / rhoR + (Ss - uR) * (Ss + pR / (rhoR * (SR - uR))));
    ET f0 = rhoR * uR, f1 = rhoR * uR * uR + pR, f2 = EN(eo_tflux)(rhoR, uR, vR, n), f3 = (ER + pR) * uR;
    f[0] = f0 + SR * (U0 - rhoR);
    f[n] = f1 + SR * (U1 - rhoR * uR);
    f[tt] = f2 + SR * (U2 - rhoR * vR);
    f[3] = f3 + SR * (U3 - ER);
  } else {
    f[0] = rhoR * uR;
    f[n] = rhoR * uR * uR + pR;
    f[tt] = EN(eo_tflux)(rhoR, uR, vR, n);
    f[3] = (ER + pR) * uR;
  }
}
/* riemann.hpp:388-432 */
static void EN(eo_hll)(const ET WL[4], const ET WR[4], ET f[4], int n, int tt) {
  ET rhoL = WL[0], uL = WL[n], vL = WL[tt], pL = WL[3];
  ET rhoR = WR[0], uR = WR[n], vR = WR[tt], pR = WR[3];
  ET cL = EN(eo_sound)(pL, rhoL), cR = EN(eo_sound)(pR, rhoR);
  ET SL = EN(eo_min)(uL - cL, uR - cR), SR = EN(eo_max)(uL + cL, uR + cR);
  ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rhoL * (uL * uL + vL * vL));
  ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rhoR * (uR * uR + vR * vR));
  ET FL[4], FR[4], UL[4], UR[4];
  int k;
  FL[0] = rhoL * uL; FR[0] = rhoR * uR;
  FL[n] = rhoL * uL * uL + pL; FR[n] = rhoR * uR * uR + pR;
  FL[tt] = rhoL * uL * vL; FR[tt] = rhoR * uR * vR;
  FL[3] = (EL + pL) * uL; FR[3] = (ER + pR) * uR;
  UL[0] = rhoL; UR[0] = rhoR;
  UL[n] = rhoL * uL; UR[n] = rhoR * uR;
  UL[tt] = rhoL * vL; UR[tt] = rhoR * vR;
  UL[3] = EL; UR[3] = ER;
  if (SL > (ET)0.0) {
    for (k = 0; k < 4; k++) f[k] = FL[k];
  } else if (SR > (ET)0.0) {
    ET inv = (ET)1.0 / (SR - SL);
    for (k = 0; k < 4; k++) f[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) * inv;
  } else {
    for (k = 0; k < 4; k++) f[k] = FR[k];
  }
}

/* riemann.hpp:290-343 (1D HLLC) */
static void EN(eo_hllc1)(const ET WL[3], const ET WR[3], ET f[3]) {
  ET rhoL = WL[0], uL = WL[1], pL = WL[2], rhoR = WR[0], uR = WR[1], pR = WR[2];
  ET cL = EN(eo_sound)(pL, rhoL), cR = EN(eo_sound)(pR, rhoR);
  ET SL = EN(eo_min)(uL - cL, uR - cR), SR = EN(eo_max)(uL + cL, uR + cR);
  ET denom = rhoL * (SL - uL) - rhoR * (SR - uR);
  ET Ss = (pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR)) / denom;
  ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rhoL * uL * uL);
  ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rhoR * uR * uR);
  if (SL > (ET)0.0) {
    f[0] = rhoL * uL; f[1] = rhoL * uL * uL + pL; f[2] = (EL + pL) * uL;
  } else if (Ss > (ET)0.0) {
    ET c = rhoL * (SL - uL) / (SL - Ss);
    ET U0 = c, U1 = c * Ss, U2 = c * (EL / rhoL + (Ss - uL) * (Ss + pL / (rhoL * (SL - uL))));
    ET f0 = rhoL * uL, f1 = rhoL * uL * uL + pL, f2 = (EL + pL) * uL;
    f[0] = f0 + SL * (U0 - rhoL); f[1] = f1 + SL * (U1 - rhoL * uL); f[2] = f2 + SL * (U2 - EL);
  } else if (SR > (ET)0.0) {
    ET c = rhoR * (SR - uR) / (SR - Ss);
    ET U0 = c, U1 = c * Ss, U2 = c * (ER / rhoR + (Ss - uR) * (Ss + pR / (rhoR * (SR - uR))));
    ET f0 = rhoR * uR, f1 = rhoR * uR * uR + pR, f2 = (ER + pR) * uR;
    f[0] = f0 + SR * (U0 - rhoR); f[1] = f1 + SR * (U1 - rhoR * uR); f[2] = f2 + SR * (U2 - ER);
  } else {
    f[0] = rhoR * uR; f[1] = rhoR * uR * uR + pR; f[2] = (ER + pR) * uR;
  }
}
/* riemann.hpp:346-378 (1D HLL) */
static void EN(eo_hll1)(const ET WL[3], const ET WR[3], ET f[3]) {
  ET rhoL = WL[0], uL = WL[1], pL = WL[2], rhoR = WR[0], uR = WR[1], pR = WR[2];
  ET cL = EN(eo_sound)(pL, rhoL), cR = EN(eo_sound)(pR, rhoR);
  ET SL = EN(eo_min)(uL - cL, uR - cR), SR = EN(eo_max)(uL + cL, uR + cR);
  ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rhoL * uL * uL);
  ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rhoR * uR * uR);
  ET FL[3] = {rhoL * uL, rhoL * uL * uL + pL, (EL + pL) * uL}, FR[3] = {rhoR * uR, rhoR * uR * uR + pR, (ER + pR) * uR};
  ET UL[3] = {rhoL, rhoL * uL, EL}, UR[3] = {rhoR, rhoR * uR, ER};
  int k;
  if (SL > (ET)0.0) {
    for (k = 0; k < 3; k++) f[k] = FL[k];
  } else if (SR > (ET)0.0) {
    ET inv = (ET)1.0 / (SR - SL);
    for (k = 0; k < 3; k++) f[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) * inv;
  } else {
    for (k = 0; k < 3; k++) f[k] = FR[k];
  }
}

/* Liska-Wendroff quadrant states (riemann2d_cpu.cpp:54-76): rho, u, v, p for
 * Q1 (x>=.5,y>=.5), Q2 (x<.5,y>=.5), Q3 (x<.5,y<.5), Q4; and T_end. */
static int EN(eo_lw_config)(int id, ET q[4][4], ET* t_end) {
  static const double c3[4][4] = {{0.5197, -0.6259, -0.3109, 0.4}, {1.0, 0.1, -0.3109, 1.0},
                                  {0.8, 0.1, 0.4276, 0.4}, {0.5197, -0.6259, 0.4276, 0.4}};
  static const double c6[4][4] = {{1.0, 0.75, -0.5, 1.0}, {2.0, 0.75, 0.5, 1.0},
                                  {1.0, -0.75, 0.5, 1.0}, {3.0, -0.75, -0.5, 1.0}};
  static const double c12[4][4] = {{0.5313, 0.0, 0.0, 0.4}, {1.0, 0.7276, 0.0, 1.0},
                                   {0.8, 0.0, 0.0, 1.0}, {1.0, 0.0, 0.7276, 1.0}};
  const double(*c)[4] = id == 3 ? c3 : id == 6 ? c6 : id == 12 ? c12 : 0;
  int a, b;
  if (!c) return 0;
  for (a = 0; a < 4; a++)
    for (b = 0; b < 4; b++) q[a][b] = (ET)c[a][b];
  *t_end = id == 12 ? (ET)0.25 : (ET)0.3;
  return 1;
}

/* Problem id of the shock-bubble program (src/euler/euler2d_cpu.cpp). */
#ifndef EO_SHOCK_BUBBLE
#define EO_SHOCK_BUBBLE 100
#endif

/* The 2D driver behind eo_riemann2d and eo_shock_bubble: NX x NY cells,
 * CFL 0.8, transmissive walls, dimensionally split steps alternating x-y /
 * y-x.  prob = 3, 6, 12 (riemann2d_cpu.cpp:108-330, [0,1]^2, every scalar
 * of type ET) or EO_SHOCK_BUBBLE (euler2d_cpu.cpp:109-398: 0.225 x 0.089 m;
 * include/euler/config.hpp gives the domain, CFL_NUM and T_END as binary64
 * literals, so in the binary32 build the cell centres, the time step
 * (CFL_NUM * min(...)) and every test against T_END are binary64
 * expressions rounded to ET where they are stored). */
static long long EN(eo_run2d)(int NX, int NY, int prob, int hll, double t_end_in, long long max_steps, ET* out,
                              ET* t_out) {
  const int GH = 2, TX = NX + 4, TY = NY + 4;
  const size_t SZ = (size_t)TX * TY;
  const int sb = prob == EO_SHOCK_BUBBLE;
  ET q[4][4], T_end = (ET)0;
  double T_endd = 0.0;
  ET *rho, *ru, *rv, *E, *W[4], *WL[4], *WR[4], *WLh[4], *WRh[4], *F[4];
  ET* blk;
  int i, j, k, g;
  long long step = 0;
  ET t = (ET)0.0;
  /* config.hpp:56-57: DX = (Real)(X_MAX - X_MIN) / (Real)NX; riemann2d: ((Real)1 - (Real)0) / N. */
  const ET dx = sb ? (ET)(0.225 - 0.0) / (ET)NX : ((ET)1.0 - (ET)0.0) / (ET)NX;
  const ET dy = sb ? (ET)(0.089 - 0.0) / (ET)NY : ((ET)1.0 - (ET)0.0) / (ET)NY, cfl = (ET)0.8;
  if (NX < 2 || NY < 2) return -1;
  if (sb) {
    T_endd = t_end_in > 0.0 ? t_end_in : 0.0011741;
  } else {
    if (!EN(eo_lw_config)(prob, q, &T_end)) return -1;
    if (t_end_in > 0.0) T_end = (ET)t_end_in;
  }
  blk = (ET*)calloc(SZ * 24, sizeof(ET));
  if (!blk) return -1;
  rho = blk; ru = blk + SZ; rv = blk + 2 * SZ; E = blk + 3 * SZ;
  for (k = 0; k < 4; k++) {
    W[k] = blk + (4 + k) * SZ; WL[k] = blk + (8 + k) * SZ; WR[k] = blk + (12 + k) * SZ;
    WLh[k] = blk + (16 + k) * SZ; WRh[k] = blk + (20 + k) * SZ;
    F[k] = WL[k]; /* the flux reuses the reconstruction buffers (not read after Hancock) */
  }
#define ID(i_, j_) ((size_t)(j_) * TX + (i_))
  if (sb) {
    /* euler2d_cpu.cpp:114-150: Rankine-Hugoniot post-shock state of a Mach
     * 1.22 shock in air (ET arithmetic), a helium bubble of radius 2.5 cm at
     * (3.5 cm, 4.45 cm), the shock at x = 0.5 cm. */
    const ET M = (ET)1.22, gm = (ET)1.4, rho1 = (ET)1.29, p1 = (ET)101325.0;
    const ET c1 = (ET)sqrt(gm * p1 / rho1);
    const ET rho2 = rho1 * ((gm + 1) * M * M) / ((gm - 1) * M * M + 2);
    const ET p2 = p1 * (2 * gm * M * M - (gm - 1)) / (gm + 1);
    const ET u2 = c1 * M * (1 - rho1 / rho2);
    const ET R2 = (ET)(0.025 * 0.025);
    for (j = 0; j < TY; j++) {
      const ET y = (ET)(0.0 + (j - GH + 0.5) * (double)dy);
      for (i = 0; i < TX; i++) {
        const ET x = (ET)(0.0 + (i - GH + 0.5) * (double)dx);
        const ET dxb = (ET)((double)x - 0.035), dyb = (ET)((double)y - 0.089 / 2.0);
        const ET d2 = dxb * dxb + dyb * dyb;
        ET Wc[4], Uc[4];
        size_t id = ID(i, j);
        if (d2 < R2) {
          Wc[0] = (ET)0.214; Wc[1] = (ET)0.0; Wc[2] = (ET)0.0; Wc[3] = p1;
        } else if ((double)x < 0.005) {
          Wc[0] = rho2; Wc[1] = u2; Wc[2] = (ET)0.0; Wc[3] = p2;
        } else {
          Wc[0] = rho1; Wc[1] = (ET)0.0; Wc[2] = (ET)0.0; Wc[3] = p1;
        }
        for (k = 0; k < 4; k++) W[k][id] = Wc[k];
        EN(eo_p2c)(Wc, Uc);
        rho[id] = Uc[0]; ru[id] = Uc[1]; rv[id] = Uc[2]; E[id] = Uc[3];
      }
    }
  } else {
    for (j = 0; j < TY; j++) {
      ET y = (ET)0.0 + (j - GH + (ET)0.5) * dy;
      for (i = 0; i < TX; i++) {
        ET x = (ET)0.0 + (i - GH + (ET)0.5) * dx;
        const ET* s = (x >= (ET)0.5 && y >= (ET)0.5) ? q[0] : (x < (ET)0.5 && y >= (ET)0.5) ? q[1]
                    : (x < (ET)0.5 && y < (ET)0.5) ? q[2] : q[3];
        ET Wc[4] = {s[0], s[1], s[2], s[3]}, Uc[4];
        size_t id = ID(i, j);
        for (k = 0; k < 4; k++) W[k][id] = Wc[k];
        EN(eo_p2c)(Wc, Uc);
        rho[id] = Uc[0]; ru[id] = Uc[1]; rv[id] = Uc[2]; E[id] = Uc[3];
      }
    }
  }
#define BC()                                                                                   \
  do {                                                                                         \
    for (j = GH; j < NY + GH; j++)                                                              \
      for (g = 0; g < GH; g++) {                                                               \
        size_t gL = ID(g, j), iL = ID(GH, j), gR = ID(TX - 1 - g, j), iR = ID(TX - 1 - GH, j); \
        rho[gL] = rho[iL]; ru[gL] = ru[iL]; rv[gL] = rv[iL]; E[gL] = E[iL];                    \
        rho[gR] = rho[iR]; ru[gR] = ru[iR]; rv[gR] = rv[iR]; E[gR] = E[iR];                    \
      }                                                                                        \
    for (g = 0; g < GH; g++)                                                                   \
      for (i = 0; i < TX; i++) {                                                               \
        size_t gB = ID(i, g), iB = ID(i, GH), gT = ID(i, TY - 1 - g), iT = ID(i, TY - 1 - GH); \
        rho[gB] = rho[iB]; ru[gB] = ru[iB]; rv[gB] = rv[iB]; E[gB] = E[iB];                    \
        rho[gT] = rho[iT]; ru[gT] = ru[iT]; rv[gT] = rv[iT]; E[gT] = E[iT];                    \
      }                                                                                        \
  } while (0)
#define C2P()                                                         \
  do {                                                                \
    for (size_t id_ = 0; id_ < SZ; id_++) {                           \
      ET U4[4] = {rho[id_], ru[id_], rv[id_], E[id_]}, W4[4];         \
      EN(eo_c2p)(U4, W4);                                             \
      for (k = 0; k < 4; k++) W[k][id_] = W4[k];                      \
    }                                                                 \
  } while (0)
  BC();
  while ((sb ? (double)t < T_endd : t < T_end) && (max_steps < 0 || step < max_steps)) {
    ET mx = (ET)0, my = (ET)0, dt;
    int pass;
    C2P();
    for (j = GH; j < NY + GH; j++)
      for (i = GH; i < NX + GH; i++) {
        size_t id = ID(i, j);
        ET c = EN(eo_sound)(W[3][id], W[0][id]);
        mx = EN(eo_max)(mx, (ET)fabs(W[1][id]) + c);
        my = EN(eo_max)(my, (ET)fabs(W[2][id]) + c);
      }
    if (sb) {
      /* euler2d_cpu.cpp:165 and :306-309 */
      dt = (ET)(0.8 * (double)EN(eo_min)(dx / mx, dy / my));
      if ((double)(ET)(t + dt) > T_endd) dt = (ET)(T_endd - (double)t);
    } else {
      dt = cfl * EN(eo_min)(dx / mx, dy / my);
      if (t + dt > T_end) dt = T_end - t;
    }
    if (dt <= (ET)0.0 || t + dt == t) break;
    for (pass = 0; pass < 2; pass++) {
      const int xsweep = ((step % 2 == 0) ? pass == 0 : pass == 1);
      if (pass == 1) C2P();
      if (xsweep) {
        ET fac = (ET)0.5 * dt / dx, rx = dt / dx;
        for (j = GH; j < NY + GH; j++)
          for (i = 1; i < TX - 1; i++) {
            size_t id = ID(i, j), a = ID(i - 1, j), b = ID(i + 1, j);
            for (k = 0; k < 4; k++) EN(eo_recon)(W[k][a], W[k][id], W[k][b], &WL[k][id], &WR[k][id]);
          }
        for (j = GH; j < NY + GH; j++)
          for (i = 1; i < TX - 1; i++) {
            size_t id = ID(i, j);
            ET l[4] = {WL[0][id], WL[1][id], WL[2][id], WL[3][id]}, r[4] = {WR[0][id], WR[1][id], WR[2][id], WR[3][id]};
            ET lh[4], rh[4];
            EN(eo_hancock)(l, l, r, lh, fac, 1, 2);
            EN(eo_hancock)(r, l, r, rh, fac, 1, 2);
            for (k = 0; k < 4; k++) { WLh[k][id] = lh[k]; WRh[k][id] = rh[k]; }
          }
        for (j = GH; j < NY + GH; j++)
          for (i = GH - 1; i < NX + GH; i++) {
            size_t a = ID(i, j), b = ID(i + 1, j);
            ET l[4] = {WRh[0][a], WRh[1][a], WRh[2][a], WRh[3][a]}, r[4] = {WLh[0][b], WLh[1][b], WLh[2][b], WLh[3][b]};
            ET f[4];
            if (hll) EN(eo_hll)(l, r, f, 1, 2); else EN(eo_hllc)(l, r, f, 1, 2);
            for (k = 0; k < 4; k++) F[k][a] = f[k];
          }
        for (j = GH; j < NY + GH; j++)
          for (i = GH; i < NX + GH; i++) {
            size_t id = ID(i, j), il = ID(i - 1, j);
            rho[id] -= rx * (F[0][id] - F[0][il]);
            ru[id] -= rx * (F[1][id] - F[1][il]);
            rv[id] -= rx * (F[2][id] - F[2][il]);
            E[id] -= rx * (F[3][id] - F[3][il]);
          }
      } else {
        ET fac = (ET)0.5 * dt / dy, ry = dt / dy;
        for (j = 1; j < TY - 1; j++)
          for (i = GH; i < NX + GH; i++) {
            size_t id = ID(i, j), a = ID(i, j - 1), b = ID(i, j + 1);
            for (k = 0; k < 4; k++) EN(eo_recon)(W[k][a], W[k][id], W[k][b], &WL[k][id], &WR[k][id]);
          }
        for (j = 1; j < TY - 1; j++)
          for (i = GH; i < NX + GH; i++) {
            size_t id = ID(i, j);
            ET l[4] = {WL[0][id], WL[1][id], WL[2][id], WL[3][id]}, r[4] = {WR[0][id], WR[1][id], WR[2][id], WR[3][id]};
            ET lh[4], rh[4];
            EN(eo_hancock)(l, l, r, lh, fac, 2, 1);
            EN(eo_hancock)(r, l, r, rh, fac, 2, 1);
            for (k = 0; k < 4; k++) { WLh[k][id] = lh[k]; WRh[k][id] = rh[k]; }
          }
        for (j = GH - 1; j < NY + GH; j++)
          for (i = GH; i < NX + GH; i++) {
            size_t a = ID(i, j), b = ID(i, j + 1);
            ET l[4] = {WRh[0][a], WRh[1][a], WRh[2][a], WRh[3][a]}, r[4] = {WLh[0][b], WLh[1][b], WLh[2][b], WLh[3][b]};
            ET f[4];
            if (hll) EN(eo_hll)(l, r, f, 2, 1); else EN(eo_hllc)(l, r, f, 2, 1);
            for (k = 0; k < 4; k++) F[k][a] = f[k];
          }
        for (j = GH; j < NY + GH; j++)
          for (i = GH; i < NX + GH; i++) {
            size_t id = ID(i, j), ib = ID(i, j - 1);
            rho[id] -= ry * (F[0][id] - F[0][ib]);
            ru[id] -= ry * (F[1][id] - F[1][ib]);
            rv[id] -= ry * (F[2][id] - F[2][ib]);
            E[id] -= ry * (F[3][id] - F[3][ib]);
          }
      }
      BC();
    }
    t += dt;
    step++;
  }
  C2P();
  for (j = 0; j < NY; j++)
    for (i = 0; i < NX; i++)
      for (k = 0; k < 4; k++) out[((size_t)j * NX + i) * 4 + k] = W[k][ID(i + GH, j + GH)];
  if (t_out) *t_out = t;
#undef BC
#undef C2P
#undef ID
  free(blk);
  return step;
}

/* 2D Riemann problem, NX x NY on [0,1]^2 (the reference runs N x N), CFL
 * 0.8, transmissive walls (riemann2d_cpu.cpp:108-330).  max_steps < 0: run
 * to T_end (t_end < 0: the configuration's).  out: primitive interior
 * [NY][NX][4] (rho, u, v, p).  Returns the step count, or -1 on a bad
 * configuration / allocation. */
long long EN(eo_riemann2d)(int NX, int NY, int cfg_id, int hll, ET t_end_in, long long max_steps, ET* out,
                           ET* t_out) {
  if (cfg_id == EO_SHOCK_BUBBLE) return -1;
  return EN(eo_run2d)(NX, NY, cfg_id, hll, (double)t_end_in, max_steps, out, t_out);
}

/* Shock-bubble problem (euler2d_cpu.cpp, Haas-Sturtevant: Mach 1.22 shock in
 * air on a helium bubble; the reference grid is 500 x 197) on NX x NY cells of
 * the 0.225 x 0.089 m domain, to T_END = 0.0011741 s (t_end <= 0) or t_end.
 * Arguments and result as eo_riemann2d. */
long long EN(eo_shock_bubble)(int NX, int NY, int hll, double t_end_in, long long max_steps, ET* out, ET* t_out) {
  return EN(eo_run2d)(NX, NY, EO_SHOCK_BUBBLE, hll, t_end_in, max_steps, out, t_out);
}

/* Toro test states (riemann1d_cpu.cpp:43-62): rhoL uL pL rhoR uR pR T_end x0. */
static int EN(eo_toro)(int id, ET s[8]) {
  static const double tc[5][8] = {{1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.25, 0.5},
                                  {1.0, -2.0, 0.4, 1.0, 2.0, 0.4, 0.15, 0.5},
                                  {1.0, 0.0, 1000.0, 1.0, 0.0, 0.01, 0.012, 0.5},
                                  {1.0, 0.0, 0.01, 1.0, 0.0, 100.0, 0.035, 0.5},
                                  {5.99924, 19.5975, 460.894, 5.99242, -6.19633, 46.0950, 0.035, 0.4}};
  int k;
  if (id < 1 || id > 5) return 0;
  for (k = 0; k < 8; k++) s[k] = (ET)tc[id - 1][k];
  return 1;
}

/* 1D Riemann problem (riemann1d_cpu.cpp:95-214): N cells on [0,1], CFL 0.8.
 * out: interior [N][3] = rho, u, p as the reference writes them.  Returns
 * the step count or -1. */
long long EN(eo_riemann1d)(int N, int test_id, int hll, ET* out, ET* t_out) {
  const int GH = 2, TOT = N + 4;
  ET s[8];
  ET *U0, *U1, *U2, *F0, *F1, *F2, *blk;
  const ET DX = ((ET)1.0 - (ET)0.0) / (ET)N, CFL = (ET)0.8;
  ET t = (ET)0.0;
  long long step = 0;
  int i, g, k;
  if (!EN(eo_toro)(test_id, s) || N < 2) return -1;
  blk = (ET*)calloc((size_t)TOT * 6, sizeof(ET));
  if (!blk) return -1;
  U0 = blk; U1 = blk + TOT; U2 = blk + 2 * TOT; F0 = blk + 3 * TOT; F1 = blk + 4 * TOT; F2 = blk + 5 * TOT;
  for (i = 0; i < TOT; i++) {
    ET x = (ET)0.0 + (ET)(i - GH + 0.5) * DX;
    ET rho, u, p;
    if (x < s[7]) { rho = s[0]; u = s[1]; p = s[2]; } else { rho = s[3]; u = s[4]; p = s[5]; }
    U0[i] = rho;
    U1[i] = rho * u;
    U2[i] = (ET)(p / (EG - (ET)1.0) + (ET)0.5 * rho * u * u);
  }
  while (t < s[6]) {
    ET ms = (ET)0.0, dt, fac, ratio;
    for (g = 0; g < GH; g++) {
      int ir = TOT - 1 - g, in = TOT - 1 - GH;
      U0[g] = U0[GH]; U1[g] = U1[GH]; U2[g] = U2[GH];
      U0[ir] = U0[in]; U1[ir] = U1[in]; U2[ir] = U2[in];
    }
    for (i = GH; i < N + GH; i++) {
      ET rho = U0[i], ru = U1[i], E = U2[i];
      ET u = ru / rho;
      ET p = (ET)((EG - (ET)1.0) * (E - (ET)0.5 * rho * u * u));
      ET c = EN(eo_sound)(p, rho);
      ms = EN(eo_max)(ms, (ET)fabs(u) + c);
    }
    dt = CFL * DX / ms;
    if (t + dt > s[6]) dt = s[6] - t;
    fac = (ET)0.5 * dt / DX;
    for (i = GH - 1; i < N + GH; i++) {
      ET Wq[4][3], Lf[3], Rf[3], L0[3], R0[3], Lh[3], Oh[3], f[3];
      int q2;
      for (q2 = 0; q2 < 4; q2++) {
        int idx = i - 1 + q2;
        ET rho = U0[idx], ru = U1[idx], E = U2[idx];
        Wq[q2][0] = rho;
        Wq[q2][1] = ru / rho;
        Wq[q2][2] = (ET)((EG - (ET)1.0) * (E - (ET)0.5 * ru * ru / rho));
      }
      for (k = 0; k < 3; k++) {
        EN(eo_recon)(Wq[0][k], Wq[1][k], Wq[2][k], &Lf[k], &Rf[k]);
        EN(eo_recon)(Wq[1][k], Wq[2][k], Wq[3][k], &L0[k], &R0[k]);
      }
      /* hancock1d (riemann1d_cpu.cpp:160-177) of WL's right face and W0's left face */
      {
        const ET* fcs[2] = {Rf, L0};
        const ET* lfs[2] = {Lf, L0};
        const ET* rfs[2] = {Rf, R0};
        ET* outs[2] = {Lh, Oh};
        int h;
        for (h = 0; h < 2; h++) {
          const ET* Wf = fcs[h];
          const ET* Wl = lfs[h];
          const ET* Wr = rfs[h];
          ET Uf[3] = {Wf[0], Wf[0] * Wf[1], (ET)(Wf[2] / (EG - (ET)1.0) + (ET)0.5 * Wf[0] * Wf[1] * Wf[1])};
          ET rL = Wl[0], uL = Wl[1], pL = Wl[2], rR = Wr[0], uR = Wr[1], pR = Wr[2];
          ET EL = (ET)(pL / (EG - (ET)1.0) + (ET)0.5 * rL * uL * uL);
          ET ER = (ET)(pR / (EG - (ET)1.0) + (ET)0.5 * rR * uR * uR);
          ET dF[3], Uh[3];
          dF[0] = rR * uR - rL * uL;
          dF[1] = (rR * uR * uR + pR) - (rL * uL * uL + pL);
          dF[2] = (ER + pR) * uR - (EL + pL) * uL;
          for (k = 0; k < 3; k++) Uh[k] = Uf[k] - fac * dF[k];
          outs[h][0] = Uh[0];
          outs[h][1] = Uh[1] / Uh[0];
          outs[h][2] = (ET)((EG - (ET)1.0) * (Uh[2] - (ET)0.5 * Uh[1] * Uh[1] / Uh[0]));
        }
      }
      if (hll) EN(eo_hll1)(Lh, Oh, f); else EN(eo_hllc1)(Lh, Oh, f);
      F0[i] = f[0]; F1[i] = f[1]; F2[i] = f[2];
    }
    ratio = dt / DX;
    for (i = GH; i < N + GH; i++) {
      U0[i] -= ratio * (F0[i] - F0[i - 1]);
      U1[i] -= ratio * (F1[i] - F1[i - 1]);
      U2[i] -= ratio * (F2[i] - F2[i - 1]);
    }
    t += dt;
    step++;
  }
  for (i = 0; i < N; i++) {
    ET rho = U0[i + GH], ru = U1[i + GH], E = U2[i + GH];
    ET u = ru / rho;
    out[i * 3 + 0] = rho;
    out[i * 3 + 1] = u;
    out[i * 3 + 2] = (ET)((EG - (ET)1.0) * (E - (ET)0.5 * rho * u * u));
  }
  if (t_out) *t_out = t;
  free(blk);
  return step;
}

#undef EN
#undef ECAT
#undef ECAT2
#undef EG
