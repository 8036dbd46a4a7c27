/*
 * pmhd_oracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle's C interface.
 * Loaded by tests/ (ctypes), __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg.  Never part of the product.
 */
#ifndef PMHD_ORACLE_H
#define PMHD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_BC_PERIODIC = 0, OR_BC_REFLECT = 1, OR_BC_TRANSMISSIVE = 2 };

typedef struct {
  int nx, ny;
  double x_min, x_max, y_min, y_max;
  double gamma, hlld_tol, cfl, alpha, t_end;
  int use_muscl, use_hlld;
  int bc[4]; /* x low, x high, y low, y high */
  int max_steps; /* < 0: no limit */
} or_config;

typedef struct {
  int steps;     /* in: steps already taken; out: total */
  int status;    /* 0, or the reference exit code 2/3/4 */
  int bad_i, bad_j;
  double t;      /* in: start time; out: final time */
  double ch_last;
  unsigned long long x_evals, y_evals, degenerate, nonphysical;
} or_stats;

int or_run_f64(const or_config* cfg, double* U, or_stats* st);
int or_run_f32(const or_config* cfg, float* U, or_stats* st);
int or_run_mixed(const or_config* cfg, double* U, or_stats* st);
/* The 2D MUSCL-Hancock variant (oracle_step.h): one predictor-corrector
 * stage per step instead of SSPRK2; exit code 3 on an unusable cell. */
int or_run_hancock_f64(const or_config* cfg, double* U, or_stats* st);
int or_run_hancock_f32(const or_config* cfg, float* U, or_stats* st);
int or_run_hancock_mixed(const or_config* cfg, double* U, or_stats* st);

void or_fill_ghosts_f64(const or_config* cfg, double* U);
void or_fill_ghosts_f32(const or_config* cfg, float* U);

void or_init_ref_problem_f64(int problem, int nx, int ny, double x_min, double x_max,
                             double y_min, double y_max, double gamma, double* U);
void or_init_ref_problem_f32(int problem, int nx, int ny, double x_min, double x_max,
                             double y_min, double y_max, double gamma, float* U);
int or_write_dat_lines_f64(const char* path, int nx, int ny, double x_min, double x_max,
                           double y_min, double y_max, double gamma, const double* U);
int or_write_dat_lines_f32(const char* path, int nx, int ny, double x_min, double x_max,
                           double y_min, double y_max, double gamma, const float* U);

#ifdef __cplusplus
}
#endif
#endif
