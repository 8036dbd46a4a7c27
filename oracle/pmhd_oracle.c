/*
 * pmhd_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this library (liboracle.so), and only as the checker or the timed CPU
 * baseline.  The product (libpmhd.so, the CLI) never links or calls it.
 *
 * A plain-C restatement of the reference's serial 2D ideal-MHD + mixed-GLM
 * solver (src/mhd/mhd2d_glm_cpu.cpp with the point numerics of
 * include/mhd/mhd_common.hpp and include/mhd/mhd_glm_common.hpp), built for
 * binary64 (suffix _f64) and binary32 (suffix _f32), plus a restatement of
 * this project's mixed-precision variant (suffix _mixed), which has no
 * counterpart in the reference:
 *   - state storage, primitive recovery from total energy (one binary64
 *     reciprocal of the density, then products), the SSPRK2 accumulation
 *     and the flux divergence scaling in binary64;
 *   - reconstruction, the GLM+HLLD/HLL Riemann flux, the difference of
 *     neighbouring interface fluxes and the CFL signal speed in binary32.
 *
 * Pinning: the f64/f32 restatements are checked in tests/ against golden
 * vectors made by the reference's own headers and against output files of
 * the reference CPU solver compiled from its sources (recipe: oracle/Makefile,
 * outputs in oracle/_ref/).  The mixed restatement has no reference; it is
 * pinned indirectly (its binary32 kernels are the pinned f32 point functions
 * and its binary64 parts are the pinned f64 ones).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pmhd_oracle.h"

/* Source index (ghosted coordinates) of ghost g on one side of an axis of n
 * interior cells.  low != 0: ghost at position g (0 outermost); else ghost at
 * position n + 2 + g. */
static int or_bc_src(int kind, int g, int n, int low) {
  if (kind == OR_BC_PERIODIC) return low ? n + g : 2 + g;
  if (kind == OR_BC_REFLECT) return low ? 3 - g : n + 1 - g;
  return low ? 2 : n + 1; /* transmissive: copy the edge cell */
}

#define OT double
#define OS f64
#include "oracle_point.h"
#include "oracle_step.h"
#undef OT
#undef OS

#define OT float
#define OS f32
#include "oracle_point.h"
#include "oracle_step.h"
#undef OT
#undef OS

/* ------------------------------------------------------------------------ */
/* Mixed-precision variant (this project's design; no reference counterpart) */

/* Face states of one interface from binary32 primitives (MUSCL or first
 * order).  P32 holds the binary32 primitives of every cell (9 per cell). */
static void or_mixed_face_states(const double* U, const float* P32, int c, int step,
                                 int muscl, float UL[9], float UR[9],
                                 const or_phys_f32* ph) {
  int k;
  if (!muscl) {
    for (k = 0; k < 9; k++) {
      UL[k] = (float)U[c * 9 + k];
      UR[k] = (float)U[(c + step) * 9 + k];
    }
    return;
  }
  float Pl0[9], Pr0[9], Pl1[9], Pr1[9];
  or_recon_f32(&P32[(c - step) * 9], &P32[c * 9], &P32[(c + step) * 9], Pl0, Pr0);
  or_recon_f32(&P32[c * 9], &P32[(c + step) * 9], &P32[(c + 2 * step) * 9], Pl1, Pr1);
  or_prim9_to_state_f32(Pr0, UL, ph);
  or_prim9_to_state_f32(Pl1, UR, ph);
}

/* Binary64 primitive recovery of the mixed variant: density floor, one
 * reciprocal of the density, velocities as products, pressure from total
 * energy in the reference's association order. */
static void or_mixed_prim9(const double* U, double* P, double gm1) {
  double rho = or_max_f64(U[0], 1.0e-12);
  double inv = 1.0 / rho;
  double vx = U[1] * inv, vy = U[2] * inv, vz = U[3] * inv;
  double bx = U[5], by = U[6], bz = U[7];
  double v2 = vx * vx + vy * vy + vz * vz;
  double b2 = bx * bx + by * by + bz * bz;
  P[0] = rho; P[1] = vx; P[2] = vy; P[3] = vz;
  P[4] = gm1 * (U[4] - 0.5 * rho * v2 - 0.5 * b2);
  P[5] = bx; P[6] = by; P[7] = bz; P[8] = U[8];
}

/* stateIsUsable with the mixed recovery. */
static int or_mixed_usable(const double* U, double gm1) {
  double P[9];
  if (U[0] <= 1.0e-12) return 0;
  or_mixed_prim9(U, P, gm1);
  return or_prim9_usable_f64(P);
}

static int or_mixed_all_usable(const double* U, int nx, int ny, int* bi, int* bj, double gm1) {
  const int nxt = nx + 4;
  int i, j;
  for (j = 2; j < ny + 2; j++)
    for (i = 2; i < nx + 2; i++)
      if (!or_mixed_usable(&U[((size_t)j * nxt + i) * 9], gm1)) {
        *bi = i - 2;
        *bj = j - 2;
        return 0;
      }
  return 1;
}

/* Binary64 recovery of every cell, rounded to binary32. */
static void or_mixed_recover(const double* U, float* P32, size_t ncell, double gm1) {
  size_t c;
  int k;
  for (c = 0; c < ncell; c++) {
    double P[9];
    or_mixed_prim9(&U[c * 9], P, gm1);
    for (k = 0; k < 9; k++) P32[c * 9 + k] = (float)P[k];
  }
}

static void or_mixed_rhs(const double* Uc, const float* P32, double* rhs, float* Fx,
                         float* Gy, int nx, int ny, double inv_dx, double inv_dy,
                         int muscl, int hlld, float ch, double alpha, or_stats* st,
                         const or_phys_f32* ph) {
  const int G = 2, nxt = nx + 4;
  const double damping = (double)ch / or_max_f64(alpha, 1.0e-12);
  int i, j, k;
  for (j = G; j < ny + G; j++)
    for (i = G - 1; i < nx + G; i++) {
      float UL[9], UR[9], F[9];
      int c = j * nxt + i;
      or_mixed_face_states(Uc, P32, c, 1, muscl, UL, UR, ph);
      int s = or_glm_flux_f32(UL, UR, ch, hlld, 0, F, ph);
      if (hlld) {
        st->x_evals++;
        if (s == 1) st->degenerate++;
        if (s == 2) st->nonphysical++;
      }
      for (k = 0; k < 9; k++) Fx[c * 9 + k] = F[k];
    }
  for (j = G - 1; j < ny + G; j++)
    for (i = G; i < nx + G; i++) {
      float UL[9], UR[9], F[9];
      int c = j * nxt + i;
      or_mixed_face_states(Uc, P32, c, nxt, muscl, UL, UR, ph);
      int s = or_glm_flux_f32(UL, UR, ch, hlld, 1, F, ph);
      if (hlld) {
        st->y_evals++;
        if (s == 1) st->degenerate++;
        if (s == 2) st->nonphysical++;
      }
      for (k = 0; k < 9; k++) Gy[c * 9 + k] = F[k];
    }
  for (j = G; j < ny + G; j++)
    for (i = G; i < nx + G; i++) {
      int id = j * nxt + i, im = id - 1, jm = id - nxt;
      for (k = 0; k < 9; k++) {
        float dfx = Fx[id * 9 + k] - Fx[im * 9 + k];
        float dgy = Gy[id * 9 + k] - Gy[jm * 9 + k];
        rhs[id * 9 + k] = -(double)dfx * inv_dx - (double)dgy * inv_dy;
      }
      rhs[id * 9 + 8] -= damping * Uc[id * 9 + 8];
    }
}

static float or_mixed_max_speed(const float* P32, int nx, int ny, const or_phys_f32* ph) {
  const int nxt = nx + 4;
  float m = 0.0f;
  int i, j;
  for (j = 2; j < ny + 2; j++)
    for (i = 2; i < nx + 2; i++) m = or_max_f32(m, or_cell_speed_f32(&P32[(j * nxt + i) * 9], ph));
  return m;
}

int or_run_mixed(const or_config* cfg, double* U, or_stats* st) {
  const int nx = cfg->nx, ny = cfg->ny, nxt = nx + 4;
  const size_t ncell = (size_t)nxt * (ny + 4), n = ncell * 9;
  or_phys_f32 ph32;
  const double gm1 = cfg->gamma - 1.0;
  ph32.gamma = (float)cfg->gamma;
  ph32.tol = (float)cfg->hlld_tol;
  const double dx = (cfg->x_max - cfg->x_min) / (double)nx;
  const double dy = (cfg->y_max - cfg->y_min) / (double)ny;
  const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
  double* U1 = (double*)malloc(n * sizeof(double));
  double* Uc = (double*)malloc(n * sizeof(double));
  double* rhs = (double*)calloc(n, sizeof(double));
  float* P32 = (float*)calloc(n, sizeof(float));
  float* Fx = (float*)calloc(n, sizeof(float));
  float* Gy = (float*)calloc(n, sizeof(float));
  int rc = 0, i, j, k;
  double t = st->t;
  memcpy(U1, U, n * sizeof(double));
  or_apply_bc_f64(U, nx, ny, cfg->bc);
  while (t < cfg->t_end && (cfg->max_steps < 0 || st->steps < cfg->max_steps)) {
    or_mixed_recover(U, P32, ncell, gm1);
    float ch = or_max_f32(or_mixed_max_speed(P32, nx, ny, &ph32), 1.0e-12f);
    st->ch_last = (double)ch;
    double dt = cfg->cfl / ((double)ch / dx + (double)ch / dy);
    if (t + dt > cfg->t_end) dt = cfg->t_end - t;
    memcpy(Uc, U, n * sizeof(double));
    or_apply_bc_f64(Uc, nx, ny, cfg->bc);
    or_mixed_recover(Uc, P32, ncell, gm1);
    or_mixed_rhs(Uc, P32, rhs, Fx, Gy, nx, ny, inv_dx, inv_dy, cfg->use_muscl,
                 cfg->use_hlld, ch, cfg->alpha, st, &ph32);
    for (j = 2; j < ny + 2; j++)
      for (i = 2; i < nx + 2; i++) {
        size_t id = ((size_t)j * nxt + i) * 9;
        for (k = 0; k < 9; k++) U1[id + k] = U[id + k] + dt * rhs[id + k];
      }
    or_apply_bc_f64(U1, nx, ny, cfg->bc);
    if (!or_mixed_all_usable(U1, nx, ny, &st->bad_i, &st->bad_j, gm1)) { rc = 3; break; }
    memcpy(Uc, U1, n * sizeof(double));
    or_mixed_recover(Uc, P32, ncell, gm1);
    or_mixed_rhs(Uc, P32, rhs, Fx, Gy, nx, ny, inv_dx, inv_dy, cfg->use_muscl,
                 cfg->use_hlld, ch, cfg->alpha, st, &ph32);
    for (j = 2; j < ny + 2; j++)
      for (i = 2; i < nx + 2; i++) {
        size_t id = ((size_t)j * nxt + i) * 9;
        for (k = 0; k < 9; k++)
          U[id + k] = 0.5 * U[id + k] + 0.5 * (U1[id + k] + dt * rhs[id + k]);
      }
    or_apply_bc_f64(U, nx, ny, cfg->bc);
    if (!or_mixed_all_usable(U, nx, ny, &st->bad_i, &st->bad_j, gm1)) { rc = 4; break; }
    t += dt;
    st->steps++;
  }
  st->t = t;
  st->status = rc;
  free(U1); free(Uc); free(rhs); free(P32); free(Fx); free(Gy);
  return rc;
}

/* Mixed-precision MUSCL-Hancock variant (this project's design; no
 * reference counterpart): the binary64 recovery of every cell rounded to
 * binary32, the binary32 faces, half-step predictor and GLM fluxes of the
 * f32 Hancock restatement (oracle_step.h) from those primitives, and the
 * binary64 update of the mixed SSPRK2 variant (binary32 flux differences,
 * binary64 scaling, psi damping and accumulation), once per step. */
static void or_mixed_hancock_cell(const float* P32, int c, int nxt, float hx, float hy, float ch, float hdamp,
                                  float HXL[9], float HXR[9], float HYL[9], float HYR[9],
                                  const or_phys_f32* ph) {
  float Pxl[9], Pxr[9], Pyl[9], Pyr[9];
  float F[4][9], corr[9];
  float* faces[4] = {HXL, HXR, HYL, HYR};
  int k, f;
  or_recon_f32(&P32[(c - 1) * 9], &P32[c * 9], &P32[(c + 1) * 9], Pxl, Pxr);
  or_recon_f32(&P32[(c - nxt) * 9], &P32[c * 9], &P32[(c + nxt) * 9], Pyl, Pyr);
  or_prim9_to_state_f32(Pxl, HXL, ph);
  or_prim9_to_state_f32(Pxr, HXR, ph);
  or_prim9_to_state_f32(Pyl, HYL, ph);
  or_prim9_to_state_f32(Pyr, HYR, ph);
  for (f = 0; f < 4; f++) or_glm_phys_flux_f32(faces[f], ch, f >= 2, F[f], ph);
  for (k = 0; k < 9; k++) corr[k] = hx * (F[1][k] - F[0][k]) + hy * (F[3][k] - F[2][k]);
  for (f = 0; f < 4; f++) {
    float h[9];
    for (k = 0; k < 9; k++) h[k] = faces[f][k] - corr[k];
    h[8] = h[8] - hdamp * faces[f][8];
    if (or_state_usable_f32(h, ph))
      for (k = 0; k < 9; k++) faces[f][k] = h[k];
  }
}

int or_run_hancock_mixed(const or_config* cfg, double* U, or_stats* st) {
  const int nx = cfg->nx, ny = cfg->ny, nxt = nx + 4, G = 2;
  const size_t cells = (size_t)nxt * (ny + 4), n = cells * 9;
  or_phys_f32 ph32;
  const double gm1 = cfg->gamma - 1.0;
  ph32.gamma = (float)cfg->gamma;
  ph32.tol = (float)cfg->hlld_tol;
  const double dx = (cfg->x_max - cfg->x_min) / (double)nx;
  const double dy = (cfg->y_max - cfg->y_min) / (double)ny;
  const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
  float* P32 = (float*)calloc(n, sizeof(float));
  float* H = (float*)calloc(n * 4, sizeof(float));
  float* Fx = (float*)calloc(n, sizeof(float));
  float* Gy = (float*)calloc(n, sizeof(float));
  float *HXL = H, *HXR = H + n, *HYL = H + 2 * n, *HYR = H + 3 * n;
  int rc = 0, i, j, k;
  double t = st->t;
  or_apply_bc_f64(U, nx, ny, cfg->bc);
  while (t < cfg->t_end && (cfg->max_steps < 0 || st->steps < cfg->max_steps)) {
    or_mixed_recover(U, P32, cells, gm1);
    const float ch = or_max_f32(or_mixed_max_speed(P32, nx, ny, &ph32), 1.0e-12f);
    st->ch_last = (double)ch;
    double dt = cfg->cfl / ((double)ch / dx + (double)ch / dy);
    if (t + dt > cfg->t_end) dt = cfg->t_end - t;
    const double damping = (double)ch / or_max_f64(cfg->alpha, 1.0e-12);
    const float hx = (float)(0.5 * dt / dx), hy = (float)(0.5 * dt / dy), hdamp = (float)(0.5 * dt * damping);
    for (j = G - 1; j < ny + G + 1; j++)
      for (i = G - 1; i < nx + G + 1; i++) {
        int c = j * nxt + i;
        if ((j < G || j >= ny + G) && (i < G || i >= nx + G)) continue; /* corners: unused */
        or_mixed_hancock_cell(P32, c, nxt, hx, hy, ch, hdamp, &HXL[c * 9], &HXR[c * 9], &HYL[c * 9], &HYR[c * 9],
                              &ph32);
      }
    for (j = G; j < ny + G; j++)
      for (i = G - 1; i < nx + G; i++) {
        int c = j * nxt + i;
        int s = or_glm_flux_f32(&HXR[c * 9], &HXL[(c + 1) * 9], ch, cfg->use_hlld, 0, &Fx[c * 9], &ph32);
        if (cfg->use_hlld) {
          st->x_evals++;
          if (s == 1) st->degenerate++;
          if (s == 2) st->nonphysical++;
        }
      }
    for (j = G - 1; j < ny + G; j++)
      for (i = G; i < nx + G; i++) {
        int c = j * nxt + i;
        int s = or_glm_flux_f32(&HYR[c * 9], &HYL[(c + nxt) * 9], ch, cfg->use_hlld, 1, &Gy[c * 9], &ph32);
        if (cfg->use_hlld) {
          st->y_evals++;
          if (s == 1) st->degenerate++;
          if (s == 2) st->nonphysical++;
        }
      }
    for (j = G; j < ny + G; j++)
      for (i = G; i < nx + G; i++) {
        int id = j * nxt + i, im = id - 1, jm = id - nxt;
        for (k = 0; k < 9; k++) {
          float dfx = Fx[id * 9 + k] - Fx[im * 9 + k];
          float dgy = Gy[id * 9 + k] - Gy[jm * 9 + k];
          double rhs = -(double)dfx * inv_dx - (double)dgy * inv_dy;
          if (k == 8) rhs -= damping * U[id * 9 + 8];
          U[id * 9 + k] = U[id * 9 + k] + dt * rhs;
        }
      }
    or_apply_bc_f64(U, nx, ny, cfg->bc);
    if (!or_mixed_all_usable(U, nx, ny, &st->bad_i, &st->bad_j, gm1)) { rc = 3; break; }
    t += dt;
    st->steps++;
  }
  st->t = t;
  st->status = rc;
  free(P32); free(H); free(Fx); free(Gy);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Initial conditions restated from mhd2d_glm_cpu.cpp:486-505 (Orszag-Tang)  */
/* and mhd2d_glm_gpu.cu:421-441 (the reference's doubly periodic KH), in     */
/* both precisions.  Output: ghosted AoS conserved state.                    */

#define OR_IC_BODY(T, SIN, EXP, TANH, ACOS, SQRT)                                  \
  const int G = 2, nxt = nx + 4, nyt = ny + 4;                                     \
  const T dx = ((T)x_max - (T)x_min) / (T)nx;                                      \
  const T dy = ((T)y_max - (T)y_min) / (T)ny;                                      \
  const T pi = ACOS((T)-1.0);                                                      \
  const T two_pi = (T)2.0 * pi;                                                    \
  const T inv_sqrt_4pi = (T)1.0 / SQRT((T)4.0 * pi);                               \
  int i, j, k;                                                                     \
  for (j = 0; j < nyt; j++)                                                        \
    for (i = 0; i < nxt; i++) {                                                    \
      T x = (T)x_min + ((T)(i - G) + (T)0.5) * dx;                                 \
      T y = (T)y_min + ((T)(j - G) + (T)0.5) * dy;                                 \
      T P[9];                                                                      \
      if (problem == 1) {                                                          \
        const T a = (T)0.025, sigma = (T)0.05, delta = (T)0.01;                    \
        T S = (T)0.5 * (TANH((y - (T)0.25) / a) - TANH((y - (T)0.75) / a));         \
        T g1 = (y - (T)0.25) / sigma;                                              \
        T g2 = (y - (T)0.75) / sigma;                                              \
        P[0] = (T)1.0 + S;                                                         \
        P[1] = -(T)0.5 + S;                                                        \
        P[2] = delta * SIN((T)2.0 * two_pi * x) *                                  \
               (EXP(-(T)0.5 * g1 * g1) + EXP(-(T)0.5 * g2 * g2));                  \
        P[3] = (T)0.0;                                                             \
        P[4] = (T)2.5;                                                             \
        P[5] = (T)0.2;                                                             \
        P[6] = (T)0.0;                                                             \
        P[7] = (T)0.0;                                                             \
        P[8] = (T)0.0;                                                             \
      } else {                                                                     \
        P[0] = (T)25.0 / ((T)36.0 * pi);                                           \
        P[1] = -SIN(two_pi * y);                                                   \
        P[2] = SIN(two_pi * x);                                                    \
        P[3] = (T)0.0;                                                             \
        P[4] = (T)5.0 / ((T)12.0 * pi);                                            \
        P[5] = -SIN(two_pi * y) * inv_sqrt_4pi;                                    \
        P[6] = SIN((T)2.0 * two_pi * x) * inv_sqrt_4pi;                            \
        P[7] = (T)0.0;                                                             \
        P[8] = (T)0.0;                                                             \
      }                                                                            \
      T Uc[9];                                                                     \
      PRIM2STATE(P, Uc);                                                           \
      for (k = 0; k < 9; k++) U[((size_t)j * nxt + i) * 9 + k] = Uc[k];            \
    }

void or_init_ref_problem_f64(int problem, int nx, int ny, double x_min, double x_max,
                             double y_min, double y_max, double gamma, double* U) {
  or_phys_f64 ph = {gamma, 0.0};
#define PRIM2STATE(P, Uc) or_prim9_to_state_f64(P, Uc, &ph)
  OR_IC_BODY(double, sin, exp, tanh, acos, sqrt)
#undef PRIM2STATE
}

void or_init_ref_problem_f32(int problem, int nx, int ny, double x_min, double x_max,
                             double y_min, double y_max, double gamma, float* U) {
  or_phys_f32 ph = {(float)gamma, 0.0f};
#define PRIM2STATE(P, Uc) or_prim9_to_state_f32(P, Uc, &ph)
  OR_IC_BODY(float, sinf, expf, tanhf, acosf, sqrtf)
#undef PRIM2STATE
}

/* ------------------------------------------------------------------------ */
/* Data lines of the reference's .dat output (mhd2d_glm_cpu.cpp:645-672):   */
/* "x y rho vx vy vz p Bx By Bz E divB psi", j outer, i inner, scientific    */
/* with max_digits10 digits.  Header lines ('#') are not produced: the       */
/* reference's regression gate hashes data lines only.                       */

int or_write_dat_lines_f64(const char* path, int nx, int ny, double x_min, double x_max,
                           double y_min, double y_max, double gamma, const double* U) {
  FILE* f = fopen(path, "w");
  if (!f) return 5;
  or_phys_f64 ph = {gamma, 0.0};
  const int nxt = nx + 4;
  const double dx = (x_max - x_min) / (double)nx, dy = (y_max - y_min) / (double)ny;
  int i, j;
  for (j = 2; j < ny + 2; j++)
    for (i = 2; i < nx + 2; i++) {
      const double* c = &U[((size_t)j * nxt + i) * 9];
      double W[8];
      or_cons_to_prim_f64(c, W, &ph);
      double x = x_min + ((double)(i - 2) + 0.5) * dx;
      double y = y_min + ((double)(j - 2) + 0.5) * dy;
      double divb = (U[((size_t)j * nxt + i + 1) * 9 + 5] - U[((size_t)j * nxt + i - 1) * 9 + 5]) / (2.0 * dx)
                  + (U[((size_t)(j + 1) * nxt + i) * 9 + 6] - U[((size_t)(j - 1) * nxt + i) * 9 + 6]) / (2.0 * dy);
      fprintf(f, "%.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n",
              x, y, W[0], W[1], W[2], W[3], W[4], W[5], W[6], W[7], c[4], divb, c[8]);
    }
  fclose(f);
  return 0;
}

int or_write_dat_lines_f32(const char* path, int nx, int ny, double x_min, double x_max,
                           double y_min, double y_max, double gamma, const float* U) {
  FILE* f = fopen(path, "w");
  if (!f) return 5;
  or_phys_f32 ph = {(float)gamma, 0.0f};
  const int nxt = nx + 4;
  const float dx = ((float)x_max - (float)x_min) / (float)nx;
  const float dy = ((float)y_max - (float)y_min) / (float)ny;
  int i, j;
  for (j = 2; j < ny + 2; j++)
    for (i = 2; i < nx + 2; i++) {
      const float* c = &U[((size_t)j * nxt + i) * 9];
      float W[8];
      or_cons_to_prim_f32(c, W, &ph);
      float x = (float)x_min + ((float)(i - 2) + 0.5f) * dx;
      float y = (float)y_min + ((float)(j - 2) + 0.5f) * dy;
      float divb = (U[((size_t)j * nxt + i + 1) * 9 + 5] - U[((size_t)j * nxt + i - 1) * 9 + 5]) / (2.0f * dx)
                 + (U[((size_t)(j + 1) * nxt + i) * 9 + 6] - U[((size_t)(j - 1) * nxt + i) * 9 + 6]) / (2.0f * dy);
      fprintf(f, "%.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e\n",
              (double)x, (double)y, (double)W[0], (double)W[1], (double)W[2], (double)W[3],
              (double)W[4], (double)W[5], (double)W[6], (double)W[7], (double)c[4],
              (double)divb, (double)c[8]);
    }
  fclose(f);
  return 0;
}
