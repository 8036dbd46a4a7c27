/*
 * oracle_step.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * C "template" (instantiated by pmhd_oracle.c with OT/OS defined) restating the
 * reference's serial 2D MHD+GLM SSPRK2 step loop, src/mhd/mhd2d_glm_cpu.cpp:
 *   applyPeriodicBoundary          :120-142
 *   xFaceStates / yFaceStates      :163-229
 *   computeRhs                     :231-287
 *   maxPhysicalSignalSpeed         :289-305
 *   maxSignalRate                  :307-326
 *   allInteriorStatesUsable        :328-345
 *   main loop                      :513-570
 * State layout is the reference's AoS with 2 ghost layers:
 *   U[((j * (nx + 4)) + i) * 9 + k].
 * Extensions beyond the reference (used only by non-reference problems):
 * per-side reflecting / transmissive boundaries and a step limit.
 */

#define OR_CAT2(a, b) a##_##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define OF(name) OR_CAT(name, OS)

/* Ghost fill in the reference's two-pass order: x ghosts for interior rows,
 * then y ghosts for every column (corners included). */
static void OF(or_apply_bc)(OT* U, int nx, int ny, const int bc[4]) {
  const int G = 2, nxt = nx + 4;
  int i, j, g, k;
  for (j = G; j < ny + G; j++) {
    for (g = 0; g < G; g++) {
      int dl = j * nxt + g, dr = j * nxt + nx + G + g;
      int sl = or_bc_src(bc[0], g, nx, 1);
      int sr = or_bc_src(bc[1], g, nx, 0);
      for (k = 0; k < 9; k++) {
        OT vl = U[(j * nxt + sl) * 9 + k];
        OT vr = U[(j * nxt + sr) * 9 + k];
        if (bc[0] == OR_BC_REFLECT && (k == 1 || k == 5)) vl = -vl;
        if (bc[1] == OR_BC_REFLECT && (k == 1 || k == 5)) vr = -vr;
        U[dl * 9 + k] = vl;
        U[dr * 9 + k] = vr;
      }
    }
  }
  for (i = 0; i < nxt; i++) {
    for (g = 0; g < G; g++) {
      int dl = g * nxt + i, dr = (ny + G + g) * nxt + i;
      int sl = or_bc_src(bc[2], g, ny, 1);
      int sr = or_bc_src(bc[3], g, ny, 0);
      for (k = 0; k < 9; k++) {
        OT vl = U[(sl * nxt + i) * 9 + k];
        OT vr = U[(sr * nxt + i) * 9 + k];
        if (bc[2] == OR_BC_REFLECT && (k == 2 || k == 6)) vl = -vl;
        if (bc[3] == OR_BC_REFLECT && (k == 2 || k == 6)) vr = -vr;
        U[dl * 9 + k] = vl;
        U[dr * 9 + k] = vr;
      }
    }
  }
}

/* Face states of the interface between cells a=(i,j) and b=a+step, where
 * step is +1 (x) or +(nx+4) (y) in cell units (xFaceStates/yFaceStates). */
static void OF(or_face_states)(const OT* U, int c, int step, int muscl,
                               OT UL[9], OT UR[9], const OF(or_phys) * ph) {
  int k;
  if (!muscl) {
    for (k = 0; k < 9; k++) { UL[k] = U[c * 9 + k]; UR[k] = U[(c + step) * 9 + k]; }
    return;
  }
  OT Pm[9], P0[9], P1[9], P2[9], Pl0[9], Pr0[9], Pl1[9], Pr1[9];
  OF(or_state_to_prim9)(&U[(c - step) * 9], Pm, ph);
  OF(or_state_to_prim9)(&U[c * 9], P0, ph);
  OF(or_state_to_prim9)(&U[(c + step) * 9], P1, ph);
  OF(or_state_to_prim9)(&U[(c + 2 * step) * 9], P2, ph);
  OF(or_recon)(Pm, P0, P1, Pl0, Pr0);
  OF(or_recon)(P0, P1, P2, Pl1, Pr1);
  OF(or_prim9_to_state)(Pr0, UL, ph);
  OF(or_prim9_to_state)(Pl1, UR, ph);
}

/* computeRhs (mhd2d_glm_cpu.cpp:231-287).  Uc is the stage input with ghosts
 * already filled; Fx/Gy are scratch of the full ghosted size. */
static void OF(or_rhs)(const OT* Uc, OT* rhs, OT* Fx, OT* Gy, int nx, int ny,
                       OT dx, OT dy, int muscl, int hlld, OT ch, OT alpha,
                       or_stats* st, const OF(or_phys) * ph) {
  const int G = 2, nxt = nx + 4;
  const OT damping = ch / OF(or_max)(alpha, (OT)1.0e-12);
  int i, j, k;
  for (j = G; j < ny + G; j++) {
    for (i = G - 1; i < nx + G; i++) {
      OT UL[9], UR[9], F[9];
      int c = j * nxt + i;
      OF(or_face_states)(Uc, c, 1, muscl, UL, UR, ph);
      int s = OF(or_glm_flux)(UL, UR, ch, hlld, 0, F, ph);
      if (hlld) {
        st->x_evals++;
        if (s == 1) st->degenerate++;
        if (s == 2) st->nonphysical++;
      }
      for (k = 0; k < 9; k++) Fx[c * 9 + k] = F[k];
    }
  }
  for (j = G - 1; j < ny + G; j++) {
    for (i = G; i < nx + G; i++) {
      OT UL[9], UR[9], F[9];
      int c = j * nxt + i;
      OF(or_face_states)(Uc, c, nxt, muscl, UL, UR, ph);
      int s = OF(or_glm_flux)(UL, UR, ch, hlld, 1, F, ph);
      if (hlld) {
        st->y_evals++;
        if (s == 1) st->degenerate++;
        if (s == 2) st->nonphysical++;
      }
      for (k = 0; k < 9; k++) Gy[c * 9 + k] = F[k];
    }
  }
  for (j = G; j < ny + G; j++) {
    for (i = G; i < nx + G; i++) {
      int id = j * nxt + i, im = id - 1, jm = id - nxt;
      for (k = 0; k < 9; k++)
        rhs[id * 9 + k] = -(Fx[id * 9 + k] - Fx[im * 9 + k]) / dx
                          - (Gy[id * 9 + k] - Gy[jm * 9 + k]) / dy;
      rhs[id * 9 + 8] -= damping * Uc[id * 9 + 8];
    }
  }
}

/* First unusable interior cell in j-major order; 1 if all usable. */
static int OF(or_all_usable)(const OT* U, int nx, int ny, int* bi, int* bj,
                             const OF(or_phys) * ph) {
  const int G = 2, nxt = nx + 4;
  int i, j;
  for (j = G; j < ny + G; j++)
    for (i = G; i < nx + G; i++)
      if (!OF(or_state_usable)(&U[(j * nxt + i) * 9], ph)) {
        *bi = i - G;
        *bj = j - G;
        return 0;
      }
  return 1;
}

/* Max physical signal speed over the interior (maxPhysicalSignalSpeed). */
static OT OF(or_max_speed)(const OT* U, int nx, int ny, const OF(or_phys) * ph) {
  const int G = 2, nxt = nx + 4;
  OT m = (OT)0.0;
  int i, j;
  for (j = G; j < ny + G; j++)
    for (i = G; i < nx + G; i++) {
      OT P[9];
      OF(or_state_to_prim9)(&U[(j * nxt + i) * 9], P, ph);
      m = OF(or_max)(m, OF(or_cell_speed)(P, ph));
    }
  return m;
}

/* maxSignalRate (mhd2d_glm_cpu.cpp:307-326) */
static OT OF(or_max_rate)(const OT* U, int nx, int ny, OT dx, OT dy, OT ch,
                          const OF(or_phys) * ph) {
  const int G = 2, nxt = nx + 4;
  OT m = (OT)0.0;
  int i, j;
  for (j = G; j < ny + G; j++)
    for (i = G; i < nx + G; i++) {
      OT P[9];
      OF(or_state_to_prim9)(&U[(j * nxt + i) * 9], P, ph);
      OT sx = OF(or_max)(OF(or_abs)(P[1]) + OF(or_fast_speed)(P, P[5], ph), ch);
      OT sy = OF(or_max)(OF(or_abs)(P[2]) + OF(or_fast_speed)(P, P[6], ph), ch);
      m = OF(or_max)(m, sx / dx + sy / dy);
    }
  return m;
}

/* The reference time loop (mhd2d_glm_cpu.cpp:513-570) on a ghosted AoS state
 * U (in/out).  Returns 0, or the reference exit code 2/3/4. */
int OF(or_run)(const or_config* cfg, OT* U, or_stats* st) {
  const int nx = cfg->nx, ny = cfg->ny, nxt = nx + 4;
  const size_t n = (size_t)nxt * (ny + 4) * 9;
  OF(or_phys) ph;
  ph.gamma = (OT)cfg->gamma;
  ph.tol = (OT)cfg->hlld_tol;
  const OT dx = ((OT)cfg->x_max - (OT)cfg->x_min) / (OT)nx;
  const OT dy = ((OT)cfg->y_max - (OT)cfg->y_min) / (OT)ny;
  const OT cfl = (OT)cfg->cfl, alpha = (OT)cfg->alpha, t_end = (OT)cfg->t_end;
  OT* U1 = (OT*)malloc(n * sizeof(OT));
  OT* Uc = (OT*)malloc(n * sizeof(OT));
  OT* rhs = (OT*)calloc(n, sizeof(OT));
  OT* Fx = (OT*)calloc(n, sizeof(OT));
  OT* Gy = (OT*)calloc(n, sizeof(OT));
  int rc = 0, i, j, k;
  OT t = (OT)st->t;
  memcpy(U1, U, n * sizeof(OT));
  OF(or_apply_bc)(U, nx, ny, cfg->bc);
  while (t < t_end && (cfg->max_steps < 0 || st->steps < cfg->max_steps)) {
    OT ch = OF(or_max)(OF(or_max_speed)(U, nx, ny, &ph), (OT)1.0e-12);
    st->ch_last = (double)ch;
    OT max_rate = OF(or_max_rate)(U, nx, ny, dx, dy, ch, &ph);
    if (max_rate <= (OT)0.0) { rc = 2; break; }
    OT dt = cfl / max_rate;
    if (t + dt > t_end) dt = t_end - t;
    /* stage 1 (the reference passes U by value and fills its ghosts) */
    memcpy(Uc, U, n * sizeof(OT));
    OF(or_apply_bc)(Uc, nx, ny, cfg->bc);
    OF(or_rhs)(Uc, rhs, Fx, Gy, nx, ny, dx, dy, cfg->use_muscl, cfg->use_hlld,
               ch, alpha, st, &ph);
    for (j = 2; j < ny + 2; j++)
      for (i = 2; i < nx + 2; i++) {
        size_t id = ((size_t)j * nxt + i) * 9;
        for (k = 0; k < 9; k++) U1[id + k] = U[id + k] + dt * rhs[id + k];
      }
    OF(or_apply_bc)(U1, nx, ny, cfg->bc);
    if (!OF(or_all_usable)(U1, nx, ny, &st->bad_i, &st->bad_j, &ph)) { rc = 3; break; }
    /* stage 2 */
    memcpy(Uc, U1, n * sizeof(OT));
    OF(or_apply_bc)(Uc, nx, ny, cfg->bc);
    OF(or_rhs)(Uc, rhs, Fx, Gy, nx, ny, dx, dy, cfg->use_muscl, cfg->use_hlld,
               ch, alpha, st, &ph);
    for (j = 2; j < ny + 2; j++)
      for (i = 2; i < nx + 2; i++) {
        size_t id = ((size_t)j * nxt + i) * 9;
        for (k = 0; k < 9; k++)
          U[id + k] = (OT)0.5 * U[id + k] + (OT)0.5 * (U1[id + k] + dt * rhs[id + k]);
      }
    OF(or_apply_bc)(U, nx, ny, cfg->bc);
    if (!OF(or_all_usable)(U, nx, ny, &st->bad_i, &st->bad_j, &ph)) { rc = 4; break; }
    t += dt;
    st->steps++;
  }
  st->t = (double)t;
  st->status = rc;
  free(U1); free(Uc); free(rhs); free(Fx); free(Gy);
  return rc;
}

/* ---- 2D MUSCL-Hancock variant (order "hancock") ----------------------------
 * No 2D reference exists: this is the unsplit 2D extension of the reference's
 * 1D Hancock predictor (mhd1d_cpu.cpp:203-235) on the 2D GLM solver's
 * reconstruction, fluxes and update (mhd2d_glm_cpu.cpp:231-287): the four
 * reconstructed faces of a cell advance by half a step with the cell's GLM
 * flux differences in x and y (and half a step of psi damping), falling back
 * to the unevolved face when the result is unusable; one interface flux per
 * face from the evolved states; U += dt * rhs once per step. */

/* Physical flux along dir of a 9-slot state with the GLM terms: the y flux
 * is the x flux of the slot-swapped state (the reference's rotation). */
static void OF(or_glm_phys_flux)(const OT U[9], OT ch, int dir, OT F[9], const OF(or_phys) * ph) {
  OT a[8], W[8], f[8];
  int k;
  if (dir) OF(or_swap_xy)(U, a); else for (k = 0; k < 8; k++) a[k] = U[k];
  OF(or_cons_to_prim)(a, W, ph);
  OF(or_flux_x_w)(W, a[4], f);
  f[5] = U[8];
  if (dir) OF(or_swap_xy)(f, F); else for (k = 0; k < 8; k++) F[k] = f[k];
  F[8] = ch * ch * a[5];
}

/* Half-step faces of one cell: Hx/Hy hold left/right (bottom/top) states. */
static void OF(or_hancock_cell)(const OT* U, int c, int nxt, OT hx, OT hy, OT ch, OT hdamp, OT HXL[9], OT HXR[9],
                                OT HYL[9], OT HYR[9], const OF(or_phys) * ph) {
  OT P0[9], Pw[9], Pe[9], Ps[9], Pn[9], Pxl[9], Pxr[9], Pyl[9], Pyr[9];
  OT F[4][9], corr[9];
  OT* faces[4] = {HXL, HXR, HYL, HYR};
  int k, f;
  OF(or_state_to_prim9)(&U[c * 9], P0, ph);
  OF(or_state_to_prim9)(&U[(c - 1) * 9], Pw, ph);
  OF(or_state_to_prim9)(&U[(c + 1) * 9], Pe, ph);
  OF(or_state_to_prim9)(&U[(c - nxt) * 9], Ps, ph);
  OF(or_state_to_prim9)(&U[(c + nxt) * 9], Pn, ph);
  OF(or_recon)(Pw, P0, Pe, Pxl, Pxr);
  OF(or_recon)(Ps, P0, Pn, Pyl, Pyr);
  OF(or_prim9_to_state)(Pxl, HXL, ph);
  OF(or_prim9_to_state)(Pxr, HXR, ph);
  OF(or_prim9_to_state)(Pyl, HYL, ph);
  OF(or_prim9_to_state)(Pyr, HYR, ph);
  for (f = 0; f < 4; f++) OF(or_glm_phys_flux)(faces[f], ch, f >= 2, F[f], ph);
  for (k = 0; k < 9; k++) corr[k] = hx * (F[1][k] - F[0][k]) + hy * (F[3][k] - F[2][k]);
  for (f = 0; f < 4; f++) {
    OT h[9];
    for (k = 0; k < 9; k++) h[k] = faces[f][k] - corr[k];
    h[8] = h[8] - hdamp * faces[f][8];
    if (OF(or_state_usable)(h, ph))
      for (k = 0; k < 9; k++) faces[f][k] = h[k];
  }
}

int OF(or_run_hancock)(const or_config* cfg, OT* U, or_stats* st) {
  const int nx = cfg->nx, ny = cfg->ny, nxt = nx + 4, G = 2;
  const size_t cells = (size_t)nxt * (ny + 4), n = cells * 9;
  OF(or_phys) ph;
  ph.gamma = (OT)cfg->gamma;
  ph.tol = (OT)cfg->hlld_tol;
  const OT dx = ((OT)cfg->x_max - (OT)cfg->x_min) / (OT)nx;
  const OT dy = ((OT)cfg->y_max - (OT)cfg->y_min) / (OT)ny;
  const OT cfl = (OT)cfg->cfl, alpha = (OT)cfg->alpha, t_end = (OT)cfg->t_end;
  OT* H = (OT*)calloc(n * 4, sizeof(OT));
  OT* Fx = (OT*)calloc(n, sizeof(OT));
  OT* Gy = (OT*)calloc(n, sizeof(OT));
  OT *HXL = H, *HXR = H + n, *HYL = H + 2 * n, *HYR = H + 3 * n;
  int rc = 0, i, j, k;
  OT t = (OT)st->t;
  OF(or_apply_bc)(U, nx, ny, cfg->bc);
  while (t < t_end && (cfg->max_steps < 0 || st->steps < cfg->max_steps)) {
    OT ch = OF(or_max)(OF(or_max_speed)(U, nx, ny, &ph), (OT)1.0e-12);
    st->ch_last = (double)ch;
    OT max_rate = OF(or_max_rate)(U, nx, ny, dx, dy, ch, &ph);
    if (max_rate <= (OT)0.0) { rc = 2; break; }
    OT dt = cfl / max_rate;
    if (t + dt > t_end) dt = t_end - t;
    const OT damping = ch / OF(or_max)(alpha, (OT)1.0e-12);
    const OT hx = (OT)0.5 * dt / dx, hy = (OT)0.5 * dt / dy, hdamp = (OT)0.5 * dt * damping;
    for (j = G - 1; j < ny + G + 1; j++)
      for (i = G - 1; i < nx + G + 1; i++) {
        int c = j * nxt + i;
        if ((j < G || j >= ny + G) && (i < G || i >= nx + G)) continue; /* corners: unused */
        OF(or_hancock_cell)(U, c, nxt, hx, hy, ch, hdamp, &HXL[c * 9], &HXR[c * 9], &HYL[c * 9], &HYR[c * 9], &ph);
      }
    for (j = G; j < ny + G; j++)
      for (i = G - 1; i < nx + G; i++) {
        int c = j * nxt + i;
        int s = OF(or_glm_flux)(&HXR[c * 9], &HXL[(c + 1) * 9], ch, cfg->use_hlld, 0, &Fx[c * 9], &ph);
        if (cfg->use_hlld) {
          st->x_evals++;
          if (s == 1) st->degenerate++;
          if (s == 2) st->nonphysical++;
        }
      }
    for (j = G - 1; j < ny + G; j++)
      for (i = G; i < nx + G; i++) {
        int c = j * nxt + i;
        int s = OF(or_glm_flux)(&HYR[c * 9], &HYL[(c + nxt) * 9], ch, cfg->use_hlld, 1, &Gy[c * 9], &ph);
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
          OT rhs = -(Fx[id * 9 + k] - Fx[im * 9 + k]) / dx - (Gy[id * 9 + k] - Gy[jm * 9 + k]) / dy;
          if (k == 8) rhs -= damping * U[id * 9 + 8];
          U[id * 9 + k] = U[id * 9 + k] + dt * rhs;
        }
      }
    OF(or_apply_bc)(U, nx, ny, cfg->bc);
    if (!OF(or_all_usable)(U, nx, ny, &st->bad_i, &st->bad_j, &ph)) { rc = 3; break; }
    t += dt;
    st->steps++;
  }
  st->t = (double)t;
  st->status = rc;
  free(H); free(Fx); free(Gy);
  return rc;
}

/* Exported per-point entry points (used to pin the restatement against the
 * reference's own headers through golden vectors). */
void OF(or_point_cons_to_prim)(const OT U[8], OT W[8], double gamma) {
  OF(or_phys) ph = {(OT)gamma, (OT)0};
  OF(or_cons_to_prim)(U, W, &ph);
}
void OF(or_point_prim_to_cons)(const OT W[8], OT U[8], double gamma) {
  OF(or_phys) ph = {(OT)gamma, (OT)0};
  OF(or_prim_to_cons)(W, U, &ph);
}
OT OF(or_point_fast_speed)(const OT W[8], int dir, double gamma) {
  OF(or_phys) ph = {(OT)gamma, (OT)0};
  return OF(or_fast_speed)(W, dir ? W[6] : W[5], &ph);
}
void OF(or_point_hll)(const OT UL[8], const OT UR[8], OT F[8], int dir, double gamma) {
  OF(or_phys) ph = {(OT)gamma, (OT)0};
  OF(or_hll)(UL, UR, F, dir, &ph);
}
int OF(or_point_hlld)(const OT UL[8], const OT UR[8], OT F[8], int dir,
                      double gamma, double tol) {
  OF(or_phys) ph = {(OT)gamma, (OT)tol};
  return dir ? OF(or_hlld_y)(UL, UR, F, &ph) : OF(or_hlld_x)(UL, UR, F, &ph);
}
int OF(or_point_glm_flux)(const OT UL[9], const OT UR[9], double ch, int use_hlld,
                          int dir, OT F[9], double gamma, double tol) {
  OF(or_phys) ph = {(OT)gamma, (OT)tol};
  return OF(or_glm_flux)(UL, UR, (OT)ch, use_hlld, dir, F, &ph);
}
void OF(or_point_recon)(const OT Pm[9], const OT P0[9], const OT Pp[9], OT Pl[9], OT Pr[9]) {
  OF(or_recon)(Pm, P0, Pp, Pl, Pr);
}
void OF(or_fill_ghosts)(const or_config* cfg, OT* U) { OF(or_apply_bc)(U, cfg->nx, cfg->ny, cfg->bc); }
OT OF(or_point_minmod)(OT a, OT b) { return OF(or_minmod)(a, b); }
int OF(or_point_positive)(const OT U[8], double gamma) {
  OF(or_phys) ph = {(OT)gamma, (OT)0};
  return OF(or_positive)(U, &ph);
}

#undef OF
#undef OR_CAT
#undef OR_CAT2
