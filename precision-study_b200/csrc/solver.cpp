// solver.cpp -- implementation of the pmhd C ABI (include/pmhd.h).
//
// One handle = one grid on one device: two SoA state buffers (U and the
// stage-1 result U1), a device control block, two TMA tensor maps (one per
// stage input), a private CUDA stream and cached CUDA graphs that replay a
// fixed number of steps.  The time loop never waits on the host per step:
// ch, dt and the stop condition are computed on the device, steps past the
// stop condition are no-ops, and the host only polls the control block once
// per graph replay.
#include <cuda.h>
#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernel_api.h"
#include "pmhd.h"
#include "problems.h"
#include "runner.h"
#include "solver_internal.h"

using namespace pmhd;

namespace {

std::mutex g_init_mu;
bool g_init_done[64][2];

}  // namespace

struct pmhd_solver {
  pmhd_config cfg;
  const KernelTable* kt = nullptr;
  cudaStream_t stream = nullptr;
  size_t elem = 8;
  int pitch = 0;
  long long plane = 0;
  void* dU = nullptr;
  void* dU1 = nullptr;
  Ctrl* dCtrl = nullptr;
  Ctrl* hCtrl = nullptr;  // pinned mirror
  Member* dMember = nullptr;  // this grid as a one-member batch
  Member hMember;             // its host copy (passed by value to the kernels)
  Runner run;
  bool tuned = false;
  TuneResult tune_result;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // host view of the run
  double t = 0.0;
  long long steps = 0;
  pmhd_stats stats;
  bool failed = false;
};

namespace pmhd {

bool solver_view(pmhd_solver* s, SolverView* v) {
  if (!s || !v) return false;
  v->u = s->dU;
  v->u1 = s->dU1;
  v->pitch = s->pitch;
  v->plane = s->plane;
  v->nx = s->cfg.nx;
  v->ny = s->cfg.ny;
  v->dx = (s->cfg.x_max - s->cfg.x_min) / s->cfg.nx;
  v->dy = (s->cfg.y_max - s->cfg.y_min) / s->cfg.ny;
  v->gamma = s->cfg.gamma;
  v->precision = s->cfg.precision;
  v->stream = s->stream;
  v->ctrl = s->dCtrl;
  v->kt = s->kt;
  return true;
}

void solver_set_step_hooks(pmhd_solver* s, std::function<cudaError_t(int)> pre,
                           std::function<cudaError_t(int)> post) {
  if (!s) return;
  cudaStreamSynchronize(s->stream);
  s->run.release();
  s->run.pre_step = std::move(pre);
  s->run.post_step = std::move(post);
}

}  // namespace pmhd

namespace {

#define PMHD_CU(call)                          \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return PMHD_ERR_CUDA; \
  } while (0)

bool is_fp32(const pmhd_solver* s) { return s->cfg.precision == PMHD_FP32; }

// Values the reference computes in its Real type (float for the fp32 build).
double to_time_type(const pmhd_solver* s, double v) { return is_fp32(s) ? (double)(float)v : v; }

int get_graph(pmhd_solver* s, int nsteps, cudaGraphExec_t* out) {
  return s->run.graph(nsteps, out) == 0 ? PMHD_OK : PMHD_ERR_CUDA;
}

int check_args(const pmhd_config* c) {
  if (!c) return PMHD_ERR_ARG;
  if (c->nx < 4 || c->ny < 4) return PMHD_ERR_ARG;
  if ((long long)c->nx * c->ny > (long long)INT_MAX) return PMHD_ERR_ARG;
  if (!(c->x_max > c->x_min) || !(c->y_max > c->y_min)) return PMHD_ERR_ARG;
  if (!(c->cfl > 0.0) || !(c->cfl < 1.0)) return PMHD_ERR_ARG;
  if (!(c->alpha > 0.0)) return PMHD_ERR_ARG;
  if (!(c->gamma > 1.0)) return PMHD_ERR_ARG;
  if (!(c->hlld_tol >= 0.0)) return PMHD_ERR_ARG;
  if (c->order != PMHD_ORDER_FIRST && c->order != PMHD_ORDER_MUSCL && c->order != PMHD_ORDER_HANCOCK)
    return PMHD_ERR_ARG;
  if (c->solver != PMHD_SOLVER_HLL && c->solver != PMHD_SOLVER_HLLD) return PMHD_ERR_ARG;
  if (c->precision < PMHD_FP64 || c->precision > PMHD_MIXED) return PMHD_ERR_ARG;
  for (int k = 0; k < 4; k++)
    if (c->bc[k] < PMHD_BC_PERIODIC || c->bc[k] > PMHD_BC_TRANSMISSIVE) return PMHD_ERR_ARG;
  if ((c->bc[0] == PMHD_BC_PERIODIC) != (c->bc[1] == PMHD_BC_PERIODIC)) return PMHD_ERR_ARG;
  if ((c->bc[2] == PMHD_BC_PERIODIC) != (c->bc[3] == PMHD_BC_PERIODIC)) return PMHD_ERR_ARG;
  if (c->steps_per_graph < 0 || (c->steps_per_graph & 1)) return PMHD_ERR_ARG;
  return PMHD_OK;
}

void reset_run(pmhd_solver* s) {
  s->t = 0.0;
  s->steps = 0;
  s->failed = false;
  std::memset(&s->stats, 0, sizeof(s->stats));
  s->stats.bad_i = s->stats.bad_j = -1;
  s->stats.bad_step = -1;
}

template <class T>
int upload_host_state(pmhd_solver* s, const T* host, int layout) {
  const size_t n = layout == PMHD_LAYOUT_INTERIOR ? (size_t)s->cfg.nx * s->cfg.ny * 9
                                                  : (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  PMHD_CU(cudaMemcpyAsync(s->dU1, host, n * sizeof(T), cudaMemcpyHostToDevice, s->stream));
  PMHD_CU(s->kt->aos_to_soa(s->cfg.precision, s->dU1, layout, s->dU, s->plane, s->cfg.nx, s->cfg.ny, s->pitch,
                            s->cfg.bc, s->stream));
  PMHD_CU(cudaStreamSynchronize(s->stream));
  return PMHD_OK;
}

template <class T>
int download_state(pmhd_solver* s, T* host, int layout) {
  const size_t n = layout == PMHD_LAYOUT_INTERIOR ? (size_t)s->cfg.nx * s->cfg.ny * 9
                                                  : (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  PMHD_CU(s->kt->soa_to_aos(s->cfg.precision, s->dU, s->plane, s->cfg.nx, s->cfg.ny, s->pitch, layout, s->dU1,
                            s->stream));
  PMHD_CU(cudaMemcpyAsync(host, s->dU1, n * sizeof(T), cudaMemcpyDeviceToHost, s->stream));
  PMHD_CU(cudaStreamSynchronize(s->stream));
  return PMHD_OK;
}

ProblemGrid grid_of(const pmhd_solver* s) {
  ProblemGrid g;
  g.nx = s->cfg.nx;
  g.ny = s->cfg.ny;
  g.x_min = s->cfg.x_min;
  g.x_max = s->cfg.x_max;
  g.y_min = s->cfg.y_min;
  g.y_max = s->cfg.y_max;
  g.gamma = s->cfg.gamma;
  return g;
}

}  // namespace

extern "C" {

int pmhd_config_default(pmhd_config* c) {
  if (!c) return PMHD_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->nx = 128;
  c->ny = 128;
  c->x_min = 0.0;
  c->x_max = 1.0;
  c->y_min = 0.0;
  c->y_max = 1.0;
  c->gamma = 5.0 / 3.0;
  c->hlld_tol = 1.0e-4;
  c->cfl = 0.25;
  c->alpha = 0.18;
  c->order = PMHD_ORDER_MUSCL;
  c->solver = PMHD_SOLVER_HLLD;
  c->precision = PMHD_FP64;
  c->exact = 0;
  for (int k = 0; k < 4; k++) c->bc[k] = PMHD_BC_PERIODIC;
  c->device = 0;
  c->steps_per_graph = 0;
  return PMHD_OK;
}

int pmhd_create(const pmhd_config* cfg, pmhd_solver** out) {
  if (!out) return PMHD_ERR_ARG;
  *out = nullptr;
  int rc = check_args(cfg);
  if (rc != PMHD_OK) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0) {
    cudaGetLastError();
    return PMHD_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  PMHD_CU(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major != 10 || prop.minor != 0) return PMHD_ERR_NODEVICE;  // sm_100a code only
  PMHD_CU(cudaSetDevice(cfg->device));

  pmhd_solver* s = new (std::nothrow) pmhd_solver();
  if (!s) return PMHD_ERR_NOMEM;
  s->cfg = *cfg;
  if (s->cfg.steps_per_graph == 0) s->cfg.steps_per_graph = 32;
  s->kt = cfg->exact ? &kernel_table_exact() : &kernel_table_fast();
  {
    std::lock_guard<std::mutex> lk(g_init_mu);
    const int dev = cfg->device & 63, which = cfg->exact ? 1 : 0;
    if (!g_init_done[dev][which]) {
      if (s->kt->init() != cudaSuccess) {
        delete s;
        return PMHD_ERR_CUDA;
      }
      g_init_done[dev][which] = true;
    }
  }
  s->elem = cfg->precision == PMHD_FP32 ? 4 : 8;
  s->pitch = ((cfg->nx + 4) + 15) / 16 * 16;
  s->plane = (long long)s->pitch * (cfg->ny + 4);
  const size_t bytes = (size_t)9 * s->plane * s->elem;
  reset_run(s);
  rc = PMHD_OK;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) rc = PMHD_ERR_CUDA;
  if (rc == PMHD_OK && (cudaMalloc(&s->dU, bytes) != cudaSuccess || cudaMalloc(&s->dU1, bytes) != cudaSuccess))
    rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMalloc(&s->dCtrl, sizeof(Ctrl)) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMallocHost(&s->hCtrl, sizeof(Ctrl)) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && (cudaMemsetAsync(s->dU, 0, bytes, s->stream) != cudaSuccess ||
                        cudaMemsetAsync(s->dU1, 0, bytes, s->stream) != cudaSuccess ||
                        cudaMemsetAsync(s->dCtrl, 0, sizeof(Ctrl), s->stream) != cudaSuccess))
    rc = PMHD_ERR_CUDA;
  if (rc == PMHD_OK && (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess))
    rc = PMHD_ERR_CUDA;
  if (rc == PMHD_OK && cudaMalloc(&s->dMember, sizeof(Member)) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK) {
    Member m;
    std::memset(&m, 0, sizeof(m));
    m.u = s->dU;
    m.u1 = s->dU1;
    m.ctrl = s->dCtrl;
    m.plane = s->plane;
    m.nx = cfg->nx;
    m.ny = cfg->ny;
    m.pitch = s->pitch;
    set_member_physics(m, cfg->x_min, cfg->x_max, cfg->y_min, cfg->y_max, cfg->gamma, cfg->hlld_tol, cfg->cfl,
                       cfg->alpha, cfg->order == PMHD_ORDER_MUSCL ? 1 : 0, cfg->bc, is_fp32(s));
    if (!encode_member_tmaps(m, s->elem)) rc = PMHD_ERR_CUDA;
    // Stream-ordered (the solver's stream does not wait for the legacy stream).
    if (rc == PMHD_OK && (cudaMemcpyAsync(s->dMember, &m, sizeof(m), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
                          cudaStreamSynchronize(s->stream) != cudaSuccess))
      rc = PMHD_ERR_CUDA;
    s->hMember = m;
    s->run.single = &s->hMember;
    s->run.kt = s->kt;
    s->run.precision = cfg->precision;
    s->run.hlld = cfg->solver == PMHD_SOLVER_HLLD ? 1 : 0;
    s->run.hancock = cfg->order == PMHD_ORDER_HANCOCK ? 1 : 0;
    s->run.stream = s->stream;
    for (int t = 0; t < kNumTileHeights; t++) {
      Batch& b = s->run.batch[t];
      b.members = s->dMember;
      b.tile_member = nullptr;
      b.member_tile0 = nullptr;
      b.nmembers = 1;
      b.ntiles = ((cfg->nx + 31) / 32) * ((cfg->ny + kTileHeights[t] - 1) / kTileHeights[t]);
    }
  }
  if (rc == PMHD_OK && cudaStreamSynchronize(s->stream) != cudaSuccess) rc = PMHD_ERR_CUDA;
  if (rc != PMHD_OK) {
    cudaGetLastError();
    pmhd_destroy(s);
    return rc;
  }
  *out = s;
  return PMHD_OK;
}

int pmhd_destroy(pmhd_solver* s) {
  if (!s) return PMHD_OK;
  cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  s->run.release();
  if (s->dMember) cudaFree(s->dMember);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->dU) cudaFree(s->dU);
  if (s->dU1) cudaFree(s->dU1);
  if (s->dCtrl) cudaFree(s->dCtrl);
  if (s->hCtrl) cudaFreeHost(s->hCtrl);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return PMHD_OK;
}

int pmhd_get_config(const pmhd_solver* s, pmhd_config* cfg) {
  if (!s || !cfg) return PMHD_ERR_ARG;
  *cfg = s->cfg;
  return PMHD_OK;
}

int pmhd_set_state(pmhd_solver* s, const void* host, int layout) {
  if (!s || !host || (layout != PMHD_LAYOUT_INTERIOR && layout != PMHD_LAYOUT_GHOSTED)) return PMHD_ERR_ARG;
  PMHD_CU(cudaSetDevice(s->cfg.device));
  reset_run(s);
  if (is_fp32(s)) return upload_host_state<float>(s, static_cast<const float*>(host), layout);
  return upload_host_state<double>(s, static_cast<const double*>(host), layout);
}

int pmhd_get_state(pmhd_solver* s, void* host, int layout) {
  if (!s || !host || (layout != PMHD_LAYOUT_INTERIOR && layout != PMHD_LAYOUT_GHOSTED)) return PMHD_ERR_ARG;
  PMHD_CU(cudaSetDevice(s->cfg.device));
  if (is_fp32(s)) return download_state<float>(s, static_cast<float*>(host), layout);
  return download_state<double>(s, static_cast<double*>(host), layout);
}

int pmhd_set_time(pmhd_solver* s, double t, long long steps) {
  if (!s || steps < 0 || !std::isfinite(t)) return PMHD_ERR_ARG;
  s->t = to_time_type(s, t);
  s->steps = steps;
  s->stats.t = s->t;
  s->stats.steps = steps;
  return PMHD_OK;
}

int pmhd_problem_state(const pmhd_config* cfg, int problem, const double* params, int nparams, void* host) {
  if (!host || nparams < 0 || check_args(cfg) != PMHD_OK) return PMHD_ERR_ARG;
  ProblemGrid g;
  g.nx = cfg->nx;
  g.ny = cfg->ny;
  g.x_min = cfg->x_min;
  g.x_max = cfg->x_max;
  g.y_min = cfg->y_min;
  g.y_max = cfg->y_max;
  g.gamma = cfg->gamma;
  const size_t n = (size_t)(cfg->nx + 4) * (cfg->ny + 4) * 9;
  if (cfg->precision == PMHD_FP32) {
    std::vector<float> U;
    if (!init_problem_host<float>(g, problem, params, nparams, U)) return PMHD_ERR_ARG;
    std::memcpy(host, U.data(), n * sizeof(float));
  } else {
    std::vector<double> U;
    if (!init_problem_host<double>(g, problem, params, nparams, U)) return PMHD_ERR_ARG;
    std::memcpy(host, U.data(), n * sizeof(double));
  }
  return PMHD_OK;
}

int pmhd_init_problem(pmhd_solver* s, int problem, const double* params, int nparams) {
  if (!s || nparams < 0) return PMHD_ERR_ARG;
  const size_t n = (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  if (is_fp32(s)) {
    std::vector<float> U(n);
    int rc = pmhd_problem_state(&s->cfg, problem, params, nparams, U.data());
    return rc != PMHD_OK ? rc : pmhd_set_state(s, U.data(), PMHD_LAYOUT_GHOSTED);
  }
  std::vector<double> U(n);
  int rc = pmhd_problem_state(&s->cfg, problem, params, nparams, U.data());
  return rc != PMHD_OK ? rc : pmhd_set_state(s, U.data(), PMHD_LAYOUT_GHOSTED);
}

int pmhd_advance(pmhd_solver* s, double t_end, long long max_steps, pmhd_stats* stats) {
  if (!s || std::isnan(t_end)) return PMHD_ERR_ARG;
  if (s->failed) {
    if (stats) *stats = s->stats;
    return s->stats.status;
  }
  PMHD_CU(cudaSetDevice(s->cfg.device));
  Ctrl& h = *s->hCtrl;
  std::memset(&h, 0, sizeof(h));
  h.t[0] = h.t[1] = s->t;
  h.step[0] = h.step[1] = s->steps;
  h.t_end = to_time_type(s, t_end);
  h.step_limit = max_steps < 0 ? LLONG_MAX : s->steps + max_steps;
  h.bad1 = h.bad2 = BAD_NONE;
  // Test hook of the bounded-wait error path (see Ctrl::test_stall): the
  // SSPRK2 stage kernels time out on purpose, with no load in flight.
  if (const char* e = std::getenv("PMHD_TEST_STALL_POLLS")) {
    const long v = std::strtol(e, nullptr, 10);
    h.test_stall = (v > 0 && v < (1L << 20)) ? (int)v : 0;
  }
  PMHD_CU(cudaMemcpyAsync(s->dCtrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice, s->stream));
  PMHD_CU(cudaEventRecord(s->ev0, s->stream));
  // CFL speed of the initial state; later steps get it from stage 2.
  PMHD_CU(s->kt->speed(s->cfg.precision, s->dU, s->plane, s->cfg.nx, s->cfg.ny, s->pitch, s->cfg.gamma, s->dCtrl,
                       0, s->stream));
  const int big = s->cfg.steps_per_graph;
  long long tune_steps = 0;
  if (s->cfg.autotune && !s->run.hancock && !s->tuned && (max_steps < 0 || max_steps >= 32)) {
    // Live steps timed per kernel variant; identical results for every variant.
    const int per = 2;
    PMHD_CU(s->run.tune(per, &s->tune_result));
    tune_steps = (long long)per * s->tune_result.candidates;
    s->tuned = true;
  }
  if (max_steps >= 0) {
    // Known step budget: replay exactly enough steps, then check once.
    long long left = max_steps - tune_steps;
    if (left < 0) left = 0;
    left += left & 1;
    cudaGraphExec_t gb = nullptr, g2 = nullptr;
    if (left >= big) {
      int rc = get_graph(s, big, &gb);
      if (rc != PMHD_OK) return rc;
    }
    int rc = get_graph(s, 2, &g2);
    if (rc != PMHD_OK) return rc;
    while (left >= big) {
      PMHD_CU(cudaGraphLaunch(gb, s->stream));
      left -= big;
    }
    while (left > 0) {
      PMHD_CU(cudaGraphLaunch(g2, s->stream));
      left -= 2;
    }
    PMHD_CU(cudaEventRecord(s->ev1, s->stream));
    PMHD_CU(cudaMemcpyAsync(&h, s->dCtrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream));
    PMHD_CU(cudaStreamSynchronize(s->stream));
    if (!h.halted && !h.err && h.bad1 == BAD_NONE && h.bad2 == BAD_NONE && h.t[0] < h.t_end &&
        h.step[0] < h.step_limit) {
      // A budget above the graph plan cannot happen; keep going defensively.
      return PMHD_ERR_CUDA;
    }
  } else {
    // Time-limited: replay graphs, polling the control block one replay
    // behind so the device never idles waiting for the host.
    cudaGraphExec_t gb = nullptr;
    int rc = get_graph(s, big, &gb);
    if (rc != PMHD_OK) return rc;
    Ctrl* poll = nullptr;
    PMHD_CU(cudaMallocHost(&poll, 2 * sizeof(Ctrl)));
    cudaEvent_t evs[2];
    cudaEventCreateWithFlags(&evs[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&evs[1], cudaEventDisableTiming);
    int issued = 0;
    bool done = false;
    cudaError_t err = cudaSuccess;
    auto issue = [&]() {
      const int b = issued & 1;
      if (err == cudaSuccess) err = cudaGraphLaunch(gb, s->stream);
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(&poll[b], s->dCtrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream);
      if (err == cudaSuccess) err = cudaEventRecord(evs[b], s->stream);
      issued++;
    };
    issue();
    for (int k = 0; !done && err == cudaSuccess; k++) {
      issue();
      if (err == cudaSuccess) err = cudaEventSynchronize(evs[k & 1]);
      const Ctrl& c = poll[k & 1];
      done = c.halted || c.err || c.bad1 != BAD_NONE || c.bad2 != BAD_NONE || !(c.t[0] < c.t_end);
    }
    if (err == cudaSuccess) err = cudaEventRecord(s->ev1, s->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&h, s->dCtrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s->stream);
    cudaEventDestroy(evs[0]);
    cudaEventDestroy(evs[1]);
    cudaFreeHost(poll);
    if (err != cudaSuccess) return PMHD_ERR_CUDA;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  const long long done_steps = h.step[0] - s->steps;
  const int hlld = s->cfg.solver == PMHD_SOLVER_HLLD;
  // Flux passes: two per SSPRK2 step, one per Hancock step.
  const int per_step = s->run.hancock ? 1 : 2;
  long long stages = per_step * done_steps;
  int status = PMHD_OK;
  if (h.err) {
    status = PMHD_ERR_TIMEOUT;
  } else if (h.bad1 != BAD_NONE) {
    status = PMHD_ERR_STAGE1;
    stages += 1;
    s->stats.bad_i = h.bad1 % s->cfg.nx;
    s->stats.bad_j = h.bad1 / s->cfg.nx;
  } else if (h.bad2 != BAD_NONE) {
    status = PMHD_ERR_STAGE2;
    stages += 2;
    s->stats.bad_i = h.bad2 % s->cfg.nx;
    s->stats.bad_j = h.bad2 / s->cfg.nx;
  }
  if (status == PMHD_ERR_STAGE1 || status == PMHD_ERR_STAGE2) s->stats.bad_step = h.bad_step;
  if (hlld) {
    s->stats.x_evals += (unsigned long long)stages * (unsigned long long)(s->cfg.nx + 1) * s->cfg.ny;
    s->stats.y_evals += (unsigned long long)stages * (unsigned long long)s->cfg.nx * (s->cfg.ny + 1);
    s->stats.degenerate += h.degenerate;
    s->stats.nonphysical += h.nonphysical;
  }
  s->stats.kernel_launches += h.active_stage_launches + 1;
  if (done_steps > 0 || status != PMHD_OK) {
    s->stats.ch_last = h.last_ch;
    s->stats.dt_last = h.last_dt;
  }
  s->t = h.t[0];
  s->steps = h.step[0];
  if (s->run.hancock && status == PMHD_ERR_STAGE1) {
    // The failing Hancock step's launch already advanced the control slots;
    // report the state the failure left, at the step and time it started
    // (as the SSPRK2 path and the reference do).
    s->t = h.t_bad;
    s->steps = h.bad_step;
  }
  s->stats.t = s->t;
  s->stats.steps = s->steps;
  s->stats.status = status;
  s->stats.device_ms = ms;
  s->stats.zone_cycles = (unsigned long long)done_steps * (unsigned long long)s->cfg.nx * s->cfg.ny;
  s->stats.tile_height = kTileHeights[s->run.choice.ty_idx];
  {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->cfg.device);
    const int def = sms * s->kt->ctas_per_sm(s->cfg.precision, s->run.hlld, s->run.choice.ty_idx, 0);
    const int g = s->run.choice.grid > 0 ? s->run.choice.grid : def;
    const int nt = s->run.batch[s->run.choice.ty_idx].ntiles;
    s->stats.ctas = g < nt ? g : nt;
  }
  if (status != PMHD_OK) s->failed = true;
  if (stats) *stats = s->stats;
  return status;
}

int pmhd_get_stats(const pmhd_solver* s, pmhd_stats* stats) {
  if (!s || !stats) return PMHD_ERR_ARG;
  *stats = s->stats;
  return PMHD_OK;
}

int pmhd_diagnostics(pmhd_solver* s, double out[3]) {
  if (!s || !out) return PMHD_ERR_ARG;
  const ProblemGrid g = grid_of(s);
  const size_t n = (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  if (is_fp32(s)) {
    std::vector<float> U(n);
    int rc = pmhd_get_state(s, U.data(), PMHD_LAYOUT_GHOSTED);
    if (rc != PMHD_OK) return rc;
    diagnostics_host<float>(g, U, out);
  } else {
    std::vector<double> U(n);
    int rc = pmhd_get_state(s, U.data(), PMHD_LAYOUT_GHOSTED);
    if (rc != PMHD_OK) return rc;
    diagnostics_host<double>(g, U, out);
  }
  return PMHD_OK;
}

static const char* precision_name(int p) { return p == PMHD_FP32 ? "fp32" : (p == PMHD_MIXED ? "mixed" : "fp64"); }

int pmhd_dat_filename(const pmhd_solver* s, const char* prob_base, char* buf, size_t len) {
  if (!s || !prob_base || !buf || len == 0) return PMHD_ERR_ARG;
  const int n = std::snprintf(buf, len, "%s_glm_%s_%s_%s_N%dx%d.dat", prob_base,
                              s->cfg.order == PMHD_ORDER_MUSCL ? "muscl" : (s->cfg.order == PMHD_ORDER_HANCOCK ? "hancock" : "first"),
                              s->cfg.solver == PMHD_SOLVER_HLLD ? "hlld" : "hll", precision_name(s->cfg.precision),
                              s->cfg.nx, s->cfg.ny);
  return (n < 0 || (size_t)n >= len) ? PMHD_ERR_ARG : PMHD_OK;
}

int pmhd_write_restart(pmhd_solver* s, const char* path) {
  if (!s || !path) return PMHD_ERR_ARG;
  const size_t n = (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  std::vector<unsigned char> buf(n * s->elem);
  const int rc = pmhd_get_state(s, buf.data(), PMHD_LAYOUT_GHOSTED);
  if (rc != PMHD_OK) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return PMHD_ERR_IO;
  const int hdr[4] = {s->cfg.nx, s->cfg.ny, s->cfg.precision, (int)s->elem};
  const double t = s->t;
  const long long steps = s->steps;
  bool ok = std::fwrite("PMHDRST1", 1, 8, f) == 8 && std::fwrite(hdr, sizeof(int), 4, f) == 4 &&
            std::fwrite(&t, sizeof(t), 1, f) == 1 && std::fwrite(&steps, sizeof(steps), 1, f) == 1 &&
            std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PMHD_OK : PMHD_ERR_IO;
}

int pmhd_read_restart(pmhd_solver* s, const char* path) {
  if (!s || !path) return PMHD_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return PMHD_ERR_IO;
  char magic[8];
  int hdr[4];
  double t = 0.0;
  long long steps = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PMHDRST1", 8) == 0 &&
            std::fread(hdr, sizeof(int), 4, f) == 4 && std::fread(&t, sizeof(t), 1, f) == 1 &&
            std::fread(&steps, sizeof(steps), 1, f) == 1;
  if (!ok) {
    std::fclose(f);
    return PMHD_ERR_IO;
  }
  if (hdr[0] != s->cfg.nx || hdr[1] != s->cfg.ny || hdr[2] != s->cfg.precision || hdr[3] != (int)s->elem) {
    std::fclose(f);
    return PMHD_ERR_ARG;
  }
  const size_t n = (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  std::vector<unsigned char> buf(n * s->elem);
  ok = std::fread(buf.data(), 1, buf.size(), f) == buf.size();
  std::fclose(f);
  if (!ok) return PMHD_ERR_IO;
  int rc = pmhd_set_state(s, buf.data(), PMHD_LAYOUT_GHOSTED);
  if (rc == PMHD_OK) rc = pmhd_set_time(s, t, steps);
  return rc;
}

int pmhd_write_dat(pmhd_solver* s, const char* path, const char* title) {
  if (!s || !path) return PMHD_ERR_ARG;
  const ProblemGrid g = grid_of(s);
  const size_t n = (size_t)(s->cfg.nx + 4) * (s->cfg.ny + 4) * 9;
  std::vector<double> Ud;
  std::vector<float> Uf;
  int rc = is_fp32(s) ? (Uf.resize(n), pmhd_get_state(s, Uf.data(), PMHD_LAYOUT_GHOSTED))
                      : (Ud.resize(n), pmhd_get_state(s, Ud.data(), PMHD_LAYOUT_GHOSTED));
  if (rc != PMHD_OK) return rc;
  std::FILE* f = std::fopen(path, "w");
  if (!f) return PMHD_ERR_IO;
  // Header lines in the reference's default stream formatting (:610-627).
  std::ostringstream hd;
  const bool f32 = is_fp32(s);
  auto real = [&](double v) -> std::string {
    std::ostringstream o;
    if (f32)
      o << (float)v;
    else
      o << v;
    return o.str();
  };
  const char* order =
      s->cfg.order == PMHD_ORDER_MUSCL ? "muscl" : (s->cfg.order == PMHD_ORDER_HANCOCK ? "hancock" : "first");
  const char* solver = s->cfg.solver == PMHD_SOLVER_HLLD ? "hlld" : "hll";
  hd << "# " << (title ? title : "Orszag-Tang ideal MHD with mixed GLM (GPU)") << "\n";
  hd << "# nx " << s->cfg.nx << " ny " << s->cfg.ny << " t " << real(s->t) << " gamma " << real(s->cfg.gamma)
     << " cfl " << real(s->cfg.cfl) << " order " << order << " solver " << solver << " alpha "
     << real(s->cfg.alpha) << " ch_last " << real(s->stats.ch_last) << "\n";
  if (s->cfg.solver == PMHD_SOLVER_HLLD) {
    const unsigned long long ev = s->stats.x_evals + s->stats.y_evals;
    const unsigned long long fb = s->stats.degenerate + s->stats.nonphysical;
    const double frac = ev > 0 ? (double)fb / (double)ev : 0.0;
    hd << "# hlld_evaluations " << ev << " hlld_tolerance " << real(s->cfg.hlld_tol) << " hlld_x_evaluations "
       << s->stats.x_evals << " hlld_y_evaluations " << s->stats.y_evals << " hlld_fallbacks " << fb
       << " hlld_degenerate " << s->stats.degenerate << " hlld_nonphysical " << s->stats.nonphysical
       << " hlld_fallback_fraction " << frac << "\n";
  }
  hd << "# columns: x y rho vx vy vz p Bx By Bz E divB psi\n";
  const std::string hs = hd.str();
  bool ok = std::fwrite(hs.data(), 1, hs.size(), f) == hs.size();
  ok = ok && (f32 ? write_dat_body<float>(f, g, Uf) : write_dat_body<double>(f, g, Ud));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PMHD_OK : PMHD_ERR_IO;
}

const char* pmhd_strerror(int status) {
  switch (status) {
    case PMHD_OK: return "ok";
    case PMHD_ERR_ARG: return "invalid argument";
    case PMHD_ERR_RATE: return "non-positive maximum signal rate";
    case PMHD_ERR_STAGE1: return "non-physical RK stage";
    case PMHD_ERR_STAGE2: return "non-physical state";
    case PMHD_ERR_IO: return "failed to open output file";
    case PMHD_ERR_CUDA: return "CUDA error";
    case PMHD_ERR_TIMEOUT: return "device-side wait timed out";
    case PMHD_ERR_NOMEM: return "device allocation failed";
    case PMHD_ERR_UNSUPPORTED: return "unsupported configuration";
    case PMHD_ERR_NODEVICE: return "no compute-capability 10.0 CUDA device";
    default: return "unknown status";
  }
}

}  // extern "C"
