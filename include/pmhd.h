/*
 * pmhd.h -- C ABI of libpmhd.so, the B200 (sm_100a) 2D ideal-MHD + mixed-GLM
 * finite-volume solver.
 *
 * The reference exposes this path only as a command-line program and a
 * header-only point interface; it has no library API.  Each entry point
 * below replaces one piece of the reference's host driver
 * src/mhd/mhd2d_glm_gpu.cu (paths are inside the reference project):
 *
 *   pmhd_config_default / pmhd_create   argv parsing + cudaMalloc of the
 *                                       state arrays (mhd2d_glm_gpu.cu:353-472)
 *   pmhd_init_problem                   host initial conditions + H2D copy
 *                                       + first applyBC (:414-474)
 *   pmhd_set_state / pmhd_get_state     the H2D / D2H state copies (:473, :546)
 *   pmhd_advance                        the time loop while (t < t_end)
 *                                       (:482-537): CFL reduction, two SSPRK2
 *                                       stages, positivity checks
 *   pmhd_get_stats                      step count, t, c_h(last) and the HLLD
 *                                       fallback counters printed at :548-589
 *   pmhd_diagnostics                    divB / psi norms (:556-574)
 *   pmhd_write_dat                      the .dat output file (:591-648)
 *   pmhd_destroy                        the cudaFree calls (:650-651)
 *   pmhd_strerror                       the stderr messages of the exit codes
 *
 * Conventions
 *   - Every function returns an int status: PMHD_OK (0) or a pmhd_status
 *     code.  Codes 1..9 mirror the reference program's exit codes; the
 *     library never calls exit().
 *   - State buffers passed in or out are HOST memory owned by the caller, in
 *     the reference's array-of-structures order: conserved variables
 *     (rho, rho*vx, rho*vy, rho*vz, E, Bx, By, Bz, psi) innermost, then i,
 *     then j.  Element type: double for PMHD_FP64 and PMHD_MIXED, float for
 *     PMHD_FP32.  Device memory is owned by the handle.
 *   - A handle is used by one host thread at a time and runs on its own CUDA
 *     stream; distinct handles are independent.
 */
#ifndef PMHD_H
#define PMHD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMHD_ABI_VERSION 1

typedef enum {
  PMHD_OK = 0,
  PMHD_ERR_ARG = 1,          /* invalid argument (reference exit code 1)        */
  PMHD_ERR_RATE = 2,         /* non-positive maximum signal rate (exit code 2)  */
  PMHD_ERR_STAGE1 = 3,       /* non-physical state after RK stage 1 (code 3)    */
  PMHD_ERR_STAGE2 = 4,       /* non-physical state after RK stage 2 (code 4)    */
  PMHD_ERR_IO = 5,           /* cannot open the output file (code 5)            */
  PMHD_ERR_CUDA = 9,         /* CUDA runtime error (code 9)                     */
  PMHD_ERR_TIMEOUT = -1,     /* a bounded device-side wait expired              */
  PMHD_ERR_NOMEM = -2,       /* device allocation failed                        */
  PMHD_ERR_UNSUPPORTED = -3, /* configuration not supported by the library     */
  PMHD_ERR_NODEVICE = -4     /* no CUDA device of compute capability 10.0       */
} pmhd_status;

typedef enum { PMHD_FP64 = 0, PMHD_FP32 = 1, PMHD_MIXED = 2 } pmhd_precision;
typedef enum { PMHD_BC_PERIODIC = 0, PMHD_BC_REFLECT = 1, PMHD_BC_TRANSMISSIVE = 2 } pmhd_bc;
/* PMHD_ORDER_HANCOCK: MUSCL reconstruction + Hancock half-step predictor, one
 * stage per step (no counterpart in the reference's 2D program; the 2D form
 * of its 1D predictor, src/mhd/mhd1d_cpu.cpp:203-235).  All three precision
 * policies; single grids only (not ensembles or pmhd_advance_noalloc). */
typedef enum { PMHD_ORDER_FIRST = 0, PMHD_ORDER_MUSCL = 1, PMHD_ORDER_HANCOCK = 2 } pmhd_order;
typedef enum { PMHD_SOLVER_HLL = 0, PMHD_SOLVER_HLLD = 1, PMHD_SOLVER_HLLC = 2 /* Euler */ } pmhd_solver_kind;
typedef enum {
  PMHD_PROBLEM_ORSZAG_TANG = 0, /* mhd2d_glm_gpu.cu:443-451, unit periodic box        */
  PMHD_PROBLEM_KH_REF = 1,      /* the reference's doubly periodic double shear layer */
  PMHD_PROBLEM_KH_REFLECT = 2,  /* single shear layer, x periodic, y reflecting       */
  PMHD_PROBLEM_BRIO_WU_2D = 3,  /* Brio-Wu Riemann problem, interface rotated         */
  PMHD_PROBLEM_BRIO_WU_TORUS = 4 /* Brio-Wu states in bands of slope k/m, periodic    */
} pmhd_problem;
typedef enum { PMHD_LAYOUT_INTERIOR = 0, PMHD_LAYOUT_GHOSTED = 1 } pmhd_layout;

typedef struct {
  int nx, ny;                       /* interior cells                          */
  double x_min, x_max, y_min, y_max;
  double gamma;                     /* ratio of specific heats                 */
  double hlld_tol;                  /* HLLD relative degeneracy tolerance      */
  double cfl;                       /* CFL number, 0 < cfl < 1                 */
  double alpha;                     /* GLM damping parameter, rate = c_h/alpha */
  int order;                        /* pmhd_order (MUSCL + SSPRK2, first, Hancock) */
  int solver;                       /* pmhd_solver_kind                        */
  int precision;                    /* pmhd_precision                          */
  int exact;                        /* 1: IEEE kernels without FMA contraction
                                       (bit-parity mode); 0: fast kernels (FMA,
                                       approximate binary32 div/sqrt)         */
  int bc[4];                        /* x low, x high, y low, y high (pmhd_bc)  */
  int device;                       /* CUDA device ordinal                     */
  int steps_per_graph;              /* steps captured per CUDA graph, 0 = auto */
  int autotune;                     /* 1: the first pmhd_advance that runs at least
                                       32 steps times every stage-kernel variant
                                       (32x19 / 32x8 tiles x resident CTAs per SM)
                                       on 2 live steps each and keeps the fastest
                                       (an ensemble: per grid size, see below);
                                       results do not depend on the variant.
                                       0: 32x19 tiles, all resident CTAs.      */
} pmhd_config;

typedef struct {
  long long steps;                  /* steps taken since creation / set_state */
  double t;                         /* current simulation time                */
  double ch_last;                   /* c_h of the last step taken             */
  double dt_last;                   /* dt of the last step taken              */
  unsigned long long x_evals;       /* HLLD flux evaluations, x interfaces    */
  unsigned long long y_evals;       /* HLLD flux evaluations, y interfaces    */
  unsigned long long degenerate;    /* HLLD -> HLL fallbacks, degenerate      */
  unsigned long long nonphysical;   /* HLLD -> HLL fallbacks, non-physical    */
  int status;                       /* status of the last advance             */
  int bad_i, bad_j;                 /* first unusable cell (status 3 or 4)    */
  long long bad_step;               /* step index of that failure             */
  unsigned long long kernel_launches; /* kernels that did work, total        */
  double device_ms;                 /* GPU time of the last pmhd_advance, from
                                       CUDA events on the handle's stream     */
  int tile_height;                  /* stage-kernel tile height in use (19, 8) */
  int ctas;                         /* persistent CTAs per stage launch        */
  unsigned long long zone_cycles;   /* cells x steps of the last advance
                                       (summed over ensemble members)         */
} pmhd_stats;

typedef struct pmhd_solver pmhd_solver;

/* Fills the reference CLI defaults: 128 x 128 on [0,1]^2, gamma 5/3, HLLD
 * tolerance 1e-4, CFL 0.25, alpha 0.18, MUSCL, HLLD, fp64, FMA, periodic. */
int pmhd_config_default(pmhd_config* cfg);

/* Allocates the device state for cfg on cfg->device.  *out is NULL on error. */
int pmhd_create(const pmhd_config* cfg, pmhd_solver** out);

int pmhd_destroy(pmhd_solver* s);

/* Builds problem `problem` on the host and uploads it; resets t and the
 * step count to 0.  params may be NULL (defaults) or point to:
 *   ORSZAG_TANG:   params[0] = field amplitude factor B0 (1 = reference)
 *   KH_REF:        params[0] = shear-layer width (the reference's 0.025)
 *   KH_REFLECT:    params[0] = shear-layer width (0.05), params[1] = Bx (0.1)
 *   BRIO_WU_2D:    params[0] = interface angle in radians (0)
 *   BRIO_WU_TORUS: params[0] = k, params[1] = m (integers >= 0, not both 0;
 *                  default 1, 2): the interface normal is (m/Lx, k/Ly), the
 *                  Brio-Wu left state fills half of each of the bands of one
 *                  period m x + k y along it, so the pattern is periodic on the
 *                  box and every band edge is a Brio-Wu (or mirrored) jump
 * gamma, domain and boundary kinds are taken from the handle's config. */
int pmhd_init_problem(pmhd_solver* s, int problem, const double* params, int nparams);

/* Fills a caller-owned host buffer with problem `problem` for configuration
 * cfg, without a device: GHOSTED layout, (ny+4)*(nx+4)*9 elements of the
 * precision's element type.  Same states as pmhd_init_problem uploads. */
int pmhd_problem_state(const pmhd_config* cfg, int problem, const double* params, int nparams, void* host);

/* Copies a host state into the solver and resets t and the step count.
 * layout INTERIOR: ny*nx*9 values; GHOSTED: (ny+4)*(nx+4)*9 values (the
 * reference's array; ghost values are rebuilt from the boundary kinds). */
int pmhd_set_state(pmhd_solver* s, const void* host, int layout);

/* Copies the current state to host memory (layout as for set_state; the
 * GHOSTED form includes the ghost values the solver holds). */
int pmhd_get_state(pmhd_solver* s, void* host, int layout);

/* Sets the simulation time and step count (e.g. after set_state of a
 * restart). */
int pmhd_set_time(pmhd_solver* s, double t, long long steps);

/* Advances while t < t_end and fewer than max_steps steps were taken in this
 * call (max_steps < 0: no step limit).  Returns PMHD_OK, or PMHD_ERR_STAGE1 /
 * PMHD_ERR_STAGE2 with stats->bad_i/bad_j/bad_step set.  stats may be NULL. */
int pmhd_advance(pmhd_solver* s, double t_end, long long max_steps, pmhd_stats* stats);

int pmhd_get_stats(const pmhd_solver* s, pmhd_stats* stats);

/* divB L1, divB Linf and psi Linf of the current state, computed on the host
 * exactly as the reference does (central differences, mhd2d_glm_gpu.cu:556-574). */
int pmhd_diagnostics(pmhd_solver* s, double out[3]);

/* Writes the reference .dat file (header lines + one data line per cell:
 * x y rho vx vy vz p Bx By Bz E divB psi).  title: first header line without
 * the leading "# "; order/solver/precision names go into the second line. */
int pmhd_write_dat(pmhd_solver* s, const char* path, const char* title);

/* Restart files (no counterpart in the reference, which only writes .dat
 * output): pmhd_write_restart stores the state (the GHOSTED layout, in the
 * precision's element type), the time and the step count in a small binary
 * file ("PMHDRST1", int32 nx, ny, precision, element bytes, double t, int64
 * steps, values); pmhd_read_restart loads one into a handle of the same grid
 * and precision (PMHD_ERR_ARG otherwise, PMHD_ERR_IO on a bad file).  A run
 * resumed from a restart gives the same bits as one that never stopped. */
int pmhd_write_restart(pmhd_solver* s, const char* path);
int pmhd_read_restart(pmhd_solver* s, const char* path);

/* Output file name the reference would use for this configuration:
 * {prob}_glm_{order}_{solver}_{fp64|fp32|mixed}_N{nx}x{ny}.dat */
int pmhd_dat_filename(const pmhd_solver* s, const char* prob_base, char* buf, size_t len);

const char* pmhd_strerror(int status);

/* Copies the configuration a handle was created with. */
int pmhd_get_config(const pmhd_solver* s, pmhd_config* cfg);

/* ---- Ensembles: many independent grids advanced by the same launches -------
 * No counterpart in the reference (it runs one grid per process).  Every
 * member has its own grid size, domain, gamma, boundary kinds, initial
 * condition and end time, and advances with its own CFL time step; all
 * members' tiles form one work list of one persistent stage launch per SSPRK2
 * stage, replayed from CUDA graphs.  With autotune, every grid size is timed
 * on its own and the sizes that choose the same tile height share one work
 * list: a stage is then one launch per chosen tile height.  The common
 * configuration supplies
 * precision, exact, order, solver, cfl, alpha, hlld_tol, device,
 * steps_per_graph and autotune (its nx, ny, domain, gamma and bc are
 * ignored).  Each member gives the same results as a single pmhd_solver run
 * of it. */
typedef struct {
  int nx, ny;
  double x_min, x_max, y_min, y_max;
  double gamma;
  int bc[4];            /* x low, x high, y low, y high (pmhd_bc)              */
  int problem;          /* pmhd_problem building the initial state             */
  int nparams;          /* parameters of that problem (see pmhd_init_problem)  */
  double params[4];
  double t_end;         /* the member stops when !(t < t_end)                  */
} pmhd_member_desc;

typedef struct pmhd_ensemble pmhd_ensemble;

/* Fills out[0..n-1] with the benchmark ensemble: square grids drawn uniformly
 * from {64, 128, 256, 512}; even members Orszag-Tang with the field scaled by
 * B0 ~ U[0.5, 1.5] (gamma 5/3, periodic, t_end 0.5), odd members the Brio-Wu
 * tube (gamma 2, t_end 0.1) with its interface rotated by an angle
 * ~ U[0, pi/2]; the draws come from splitmix64 seeded with `seed` (three
 * draws per member: size, amplitude or angle, spare). */
int pmhd_ensemble_describe_default(int n, unsigned long long seed, pmhd_member_desc* out);

int pmhd_ensemble_create(const pmhd_config* common, const pmhd_member_desc* members, int n, pmhd_ensemble** out);

/* Advances every member until its t_end, or by at most max_steps steps per
 * member in this call (max_steps < 0: no limit).  total: steps = the largest
 * member step count, zone_cycles and HLLD counters summed, kernel_launches =
 * kernels enqueued (stage launches with or without work, CFL reductions),
 * device_ms, tile_height / ctas of the kernel variant; status = the first
 * failing member's status (PMHD_OK if none).  Per-member statistics
 * (pmhd_ensemble_member_stats) count that member's stage launches with work. */
int pmhd_ensemble_advance(pmhd_ensemble* e, long long max_steps, pmhd_stats* total);

int pmhd_ensemble_member_stats(const pmhd_ensemble* e, int k, pmhd_stats* st);
int pmhd_ensemble_get_state(pmhd_ensemble* e, int k, void* host, int layout);
int pmhd_ensemble_destroy(pmhd_ensemble* e);

/* ---- Learned coarse-grid correction: network building blocks --------------
 * No counterpart in the reference (its learned part exists only as a plan).
 * BF16 tensor-core (tcgen05) 3x3 convolutions over device NHWC bf16 images
 * [batch][h][w][channels], periodic in y and x; weights [c_out][9][c_in],
 * tap t = (dy+1)*3 + (dx+1), out(y,x) = sum_t W[t] x(y+dy, x+dx) + bias.
 * Enqueued on `stream` (a cudaStream_t, NULL = default) and synchronised
 * before returning; all pointers are device pointers, 16-byte aligned.
 *   PMHD_CONV_GELU:   out0 = z (bf16), out1 = gelu(z) (bf16), (c_in, c_out) = (32, 32);
 *                     gelu is the tanh form z / (1 + exp(-2 sqrt(2/pi) (z + 0.044715 z^3)))
 *   PMHD_CONV_LINEAR: out0 = fp32 result, (32, 16)
 *   PMHD_CONV_DGELU:  backward to the input of a GELU layer: x = the
 *                     layer's output gradient (c_in = its outputs), weight =
 *                     its weights transposed to [c_out][9][c_in], z_prev =
 *                     the previous layer's z; out0 = that z's gradient
 *                     (bf16); (16, 32) or (32, 32)
 * PMHD_ERR_UNSUPPORTED for other channel counts, PMHD_ERR_TIMEOUT when a
 * bounded wait in the kernel expired. */
typedef enum { PMHD_CONV_GELU = 0, PMHD_CONV_LINEAR = 1, PMHD_CONV_DGELU = 2 } pmhd_conv_mode;
int pmhd_conv3x3(int mode, const void* x, int batch, int h, int w, int c_in, const void* weight, const float* bias,
                 int c_out, const void* z_prev, void* out0, void* out1, void* stream);

/* Weight and bias gradients of a 3x3 layer: dweight[co][t][ci] +=
 * sum_p dz[p][co] x[p + tap t][ci], dbias[co] += sum_p dz[p][co] (dbias may
 * be NULL); fp32 accumulation.  (c_in, c_out) = (32, 32) or (32, 16). */
int pmhd_conv3x3_wgrad(const void* x, const void* dz, int batch, int h, int w, int c_in, int c_out, float* dweight,
                       float* dbias, void* stream);

/* Training loss of the correction network and its gradient with respect to
 * the network output, over `batch` periodic h x w images; device pointers:
 * out and tgt [batch][h][w][16] fp32, dz [batch][h][w][16] bf16 (16-byte
 * aligned).  Channels 0-4, 6, 7 are compared directly with tgt; channel 5 is
 * a potential A whose central-difference curl, dBx = cy (A(y+1) - A(y-1)),
 * dBy = -cx (A(x+1) - A(x-1)), is compared with tgt channels 8 and 9:
 * loss = sum of the nine squared differences / (9 batch h w).  *loss (host)
 * receives the loss.  Synchronises `stream` before returning. */
int pmhd_learned_loss_grad(const float* out, const float* tgt, int batch, int h, int w, float cx, float cy, void* dz,
                           double* loss, void* stream);

/* ---- Learned coarse-grid correction -------------------------------------------
 * No counterpart in the reference.  A periodic problem runs on a coarse grid
 * (nx x ny) with the plain solver; after every step a small network (four
 * 3x3 convolutions, 32 channels, GELU; BF16 tensor-core kernels with fp32
 * accumulation) predicts the difference between the fine solution (refine x
 * finer, restricted by block averages) and the coarse step, from the coarse
 * state and its step increment, in quantities that keep the corrected state
 * physical: log ratios of density and pressure, velocity increments, and a
 * potential whose central-difference curl corrects B_x and B_y (so the
 * central-difference div B does not change).  The correction is applied only
 * when the corrected state keeps positive density and pressure and its
 * ||div B||_1 grows by at most div_tol relative to the uncorrected step;
 * otherwise the plain coarse step stands (counted as a rejection).  Training
 * pairs come
 * from the solver itself (pmhd_learned_generate: fine and coarse runs of a
 * problem); training runs on the device with the project's own forward and
 * backward kernels and Adam.  All four boundaries are periodic; states are
 * fp64 (precision PMHD_FP64 or PMHD_MIXED for both solvers). */
typedef struct pmhd_learned pmhd_learned;

typedef struct {
  int nx, ny;                 /* coarse grid (even sizes)                        */
  int refine;                 /* fine / coarse ratio of the training pairs (4)   */
  double x_min, x_max, y_min, y_max;
  double gamma, cfl, alpha;
  int precision;              /* PMHD_FP64 or PMHD_MIXED                         */
  int device;
  int max_pairs;              /* capacity of the pair store (512)                */
  unsigned long long seed;    /* weight initialisation and minibatch order       */
  double div_tol;             /* allowed relative growth of ||div B||_1 (0.5)    */
  double relax;               /* fraction of the predicted correction applied
                                 (0.25; the full correction compounds its error
                                 into an unstable run)                         */
  double train_noise;         /* std of Gaussian noise added to the normalised
                                 network inputs in training (0.03; 0: none)   */
  double shrink;              /* soft threshold on the normalised network
                                 outputs: only the part beyond +-shrink is
                                 applied (0: all of it)                        */
} pmhd_learned_config;

typedef struct {
  long long steps;            /* coarse (or fine) steps taken                    */
  double t;
  long long accepted;         /* corrections applied                             */
  long long rejected_positivity, rejected_divergence;
  double device_ms;           /* device time of the time loop                    */
  double wall_ms;             /* wall-clock time of the time loop                */
  int status;
} pmhd_learned_stats;

int pmhd_learned_config_default(pmhd_learned_config* cfg);
int pmhd_learned_create(const pmhd_learned_config* cfg, pmhd_learned** out);
int pmhd_learned_destroy(pmhd_learned* L);

/* Runs `problem` (params as for pmhd_init_problem) on the fine grid to
 * t_end; before every coarse step it restricts the fine state, takes one
 * plain coarse step from it, advances the fine run to the same time and
 * stores (before, coarse step, restricted fine) as a pair every `every`
 * steps, until the store is full.  *added (may be NULL) = pairs stored. */
int pmhd_learned_generate(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int every,
                          int* added);
/* As pmhd_learned_generate, but the coarse run keeps its own state after the
 * first step (the restricted fine state is loaded once): pairs along the
 * plain coarse trajectory, the states a corrected run meets, each with the
 * restricted fine state at the same time as its target. */
int pmhd_learned_generate_rollout(pmhd_learned* L, int problem, const double* params, int nparams, double t_end,
                                  int every, int* added);
/* As pmhd_learned_generate_rollout, but the coarse run is corrected by the
 * current network (as in pmhd_learned_run) after every step: pairs along the
 * trajectory the trained correction itself produces, each with the
 * restricted fine state at the same time as its target (data aggregation
 * against the correction's own compounding error).  Needs a trained network
 * (PMHD_ERR_ARG otherwise). */
int pmhd_learned_generate_corrected(pmhd_learned* L, int problem, const double* params, int nparams, double t_end,
                                    int every, int* added);
int pmhd_learned_num_pairs(const pmhd_learned* L);

/* `iters` Adam steps (cosine decay from lr) on minibatches of `batch` pairs
 * drawn uniformly; losses (may be NULL, `iters` floats) receives the
 * minibatch loss (see pmhd_learned_loss_grad; targets normalised by their
 * root mean square) per step.  The
 * input/output normalisation is fixed from the pairs at the first call. */
int pmhd_learned_train(pmhd_learned* L, int iters, int batch, double lr, float* losses);

/* Coarse run of `problem` from the restricted fine initial state to t_end,
 * corrected (use_net = 1) or plain (0); host_out (may be NULL) receives the
 * final coarse interior state, [ny][nx][9] doubles. */
int pmhd_learned_run(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int use_net,
                     double* host_out, pmhd_learned_stats* stats);

/* Fine run at `refine` x the coarse resolution, restricted onto the coarse
 * grid at t_end (the yardstick of the coarse runs); host_out as above. */
int pmhd_learned_fine_run(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int refine,
                          double* host_out, pmhd_learned_stats* stats);

/* Network weights and normalisation to / from a file. */
int pmhd_learned_save(const pmhd_learned* L, const char* path);
int pmhd_learned_load(pmhd_learned* L, const char* path);

/* ---- Euler sibling (gamma = 1.4) -------------------------------------------------
 * The reference's 1D and 2D MUSCL-Hancock + HLLC / HLL Euler programs
 * (src/euler/riemann1d_cpu.cpp, src/euler/riemann2d_cpu.cpp): same problems,
 * CFL 0.8, transmissive walls, dimensionally split 2D steps alternating x-y
 * and y-x.  solver: PMHD_SOLVER_HLLC or PMHD_SOLVER_HLL; precision:
 * PMHD_FP64 or PMHD_FP32; exact = 1 gives the reference CPU build's bits. */
typedef struct pmhd_euler2d pmhd_euler2d;

typedef struct {
  long long steps;
  double t;
  double device_ms;    /* device time of the steps of this call */
  int status;
} pmhd_euler_stats;

/* config of pmhd_euler2d_create for the shock-bubble program
 * (src/euler/euler2d_cpu.cpp; Haas-Sturtevant: a Mach 1.22 shock in air
 * meets a helium bubble, 0.225 x 0.089 m, reference grid 500 x 197, end time
 * 0.0011741 s).  Its constants are binary64 literals
 * (include/euler/config.hpp), so in binary32 the cell centres, the CFL
 * product and the end-time tests are binary64 expressions, as there. */
enum { PMHD_EULER_SHOCK_BUBBLE = 100 };

/* nx x ny grid on [0,1]^2 holding Liska-Wendroff configuration `config`
 * (3, 6 or 12; riemann2d_cpu.cpp:54-76), or the shock-bubble domain
 * (config PMHD_EULER_SHOCK_BUBBLE). */
int pmhd_euler2d_create(int nx, int ny, int config, int solver, int precision, int exact, int device,
                        pmhd_euler2d** out);
/* Advances until t_end (< 0: the configuration's end time) or max_steps
 * steps (< 0: no limit). */
int pmhd_euler2d_advance(pmhd_euler2d* e, double t_end, long long max_steps, pmhd_euler_stats* stats);
/* Primitive state (rho, u, v, p) of the interior, [ny][nx][4] values of the
 * precision's type. */
int pmhd_euler2d_get_prim(pmhd_euler2d* e, void* host);
int pmhd_euler2d_destroy(pmhd_euler2d* e);

/* Toro test `test` (1-5; riemann1d_cpu.cpp:43-62) on n cells of [0,1] to its
 * end time, in one kernel launch; host_out (may be NULL): [n][3] = rho, u, p
 * of the precision's type, as the reference writes them. */
int pmhd_euler1d_run(int n, int test, int solver, int precision, int exact, int device, void* host_out,
                     pmhd_euler_stats* stats);

/* ---- Allocation-free time loop ----------------------------------------------
 * No counterpart in the reference: its program always cudaMallocs five state
 * arrays.  For callers that must not allocate device memory while they run
 * (a process that pre-carves all GPU memory into its own pool, an allocator
 * hook that forbids cudaMalloc after start-up, a fixed memory plan that must
 * not fail mid-run).  Advances the caller's state like pmhd_advance, but with
 * no handle and no allocation: d_in and d_out are the caller's DEVICE buffers
 * of ny*nx*9 elements in the PMHD_LAYOUT_INTERIOR order (double for fp64 and
 * mixed, float for fp32; they may be the same buffer); t0 and step0 are the
 * time and step count d_in is at; stream is a cudaStream_t (NULL = the
 * default stream).  The working state lives in one array compiled into the
 * library, PMHD_NOALLOC_SCRATCH_BYTES long, that every GPU using this entry
 * point keeps until exit.  Grids whose working state does not fit --
 * 2048 + 2 * round_up_256(9 * (ny+4) * round_up(nx+4, 16) * element size)
 * bytes (a control block and grid descriptor, then two states), up to 586^2
 * cells in fp64/mixed and 828^2 in fp32 -- are rejected with
 * PMHD_ERR_UNSUPPORTED.  All calls share that array: calls that overlap on
 * the GPU race; serialise them.
 * The array and the kernels' code are placed in device memory when the
 * CUDA runtime loads this library's device code on a device.  Under lazy
 * module loading (the CUDA 12 default) that happens during the FIRST call on
 * each device, which also looks up the array's address with that device
 * current: that first call does allocate (the array plus the code), so make
 * it -- for example a one-step call (max_steps = 1) with the same precision,
 * solver and build on a scratch copy of the state -- before the caller hands
 * all remaining device memory to its own pool, and before any stream
 * capture.  Later calls allocate nothing.  stats: as pmhd_advance (steps/t
 * are totals including step0/t0; device_ms is not measured, 0). */
#define PMHD_NOALLOC_SCRATCH_BYTES (48u << 20)
int pmhd_advance_noalloc(const pmhd_config* cfg, const void* d_in, void* d_out, double t0, long long step0,
                         double t_end, long long max_steps, void* stream, pmhd_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* PMHD_H */
