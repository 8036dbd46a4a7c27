// euler.cpp -- pmhd_euler2d_* / pmhd_euler1d_run (include/pmhd.h): host side
// of the Euler sibling.  Initial states follow the reference programs
// (src/euler/riemann2d_cpu.cpp:117-134, src/euler/euler2d_cpu.cpp:109-150,
// src/euler/riemann1d_cpu.cpp:95-112) with the same arithmetic; the 2D time loop replays CUDA graphs of
// fused split steps (state ping-ponged between two SoA buffers) and polls
// the device control block one replay behind.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "euler/euler_api.h"
#include "pmhd.h"
#include "pmhd/euler.hpp"

using namespace pmhd::euler;

struct pmhd_euler2d {
  int nx = 0, ny = 0, pitch = 0, config = 0, hll = 0, fp32 = 0, exact = 0, device = 0, wide_time = 0;
  long long plane = 0;
  size_t elem = 8;
  double dx = 0, dy = 0, cfl = 0, t_end_cfg = 0;
  void* u[2] = {nullptr, nullptr};
  EulerCtrl* dctrl = nullptr;
  EulerCtrl* hctrl = nullptr;  // pinned, [3]: upload + two poll slots
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp[2] = {nullptr, nullptr};
  cudaGraphExec_t graph_big = nullptr, graph_two = nullptr;
  int big = 32;
  double t = 0.0;
  long long steps = 0;
  bool stopped = false;
};

namespace {

#define E_CU(call)                 \
  do {                             \
    if ((call) != cudaSuccess) {   \
      cudaGetLastError();          \
      return PMHD_ERR_CUDA;        \
    }                              \
  } while (0)

std::mutex g_mu;
bool g_prepared[64][2];

int prepare_device(int dev, int exact) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (dev < 0 || dev >= 64) return PMHD_ERR_ARG;
  if (g_prepared[dev][exact]) return PMHD_OK;
  const cudaError_t e = exact ? exact::prepare() : fast::prepare();
  if (e != cudaSuccess) return PMHD_ERR_CUDA;
  g_prepared[dev][exact] = true;
  return PMHD_OK;
}

int check_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return PMHD_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PMHD_ERR_CUDA;
  if (prop.major != 10 || prop.minor != 0) return PMHD_ERR_NODEVICE;
  return cudaSetDevice(device) == cudaSuccess ? PMHD_OK : PMHD_ERR_CUDA;
}

// Liska-Wendroff quadrant states (rho, u, v, p) Q1..Q4 and end time.
bool lw_config(int id, double q[4][4], double* t_end) {
  static const double c3[4][4] = {{0.5197, -0.6259, -0.3109, 0.4}, {1.0, 0.1, -0.3109, 1.0},
                                  {0.8, 0.1, 0.4276, 0.4}, {0.5197, -0.6259, 0.4276, 0.4}};
  static const double c6[4][4] = {{1.0, 0.75, -0.5, 1.0}, {2.0, 0.75, 0.5, 1.0},
                                  {1.0, -0.75, 0.5, 1.0}, {3.0, -0.75, -0.5, 1.0}};
  static const double c12[4][4] = {{0.5313, 0.0, 0.0, 0.4}, {1.0, 0.7276, 0.0, 1.0},
                                   {0.8, 0.0, 0.0, 1.0}, {1.0, 0.0, 0.7276, 1.0}};
  const double(*c)[4] = id == 3 ? c3 : id == 6 ? c6 : id == 12 ? c12 : nullptr;
  if (!c) return false;
  std::memcpy(q, c, sizeof(c3));
  *t_end = id == 12 ? 0.25 : 0.3;
  return true;
}

template <class T>
void init_2d(const pmhd_euler2d* e, const double qd[4][4], std::vector<unsigned char>& buf) {
  buf.assign((size_t)4 * e->plane * sizeof(T), 0);
  T* u = reinterpret_cast<T*>(buf.data());
  T q[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) q[a][b] = (T)qd[a][b];
  const T dx = ((T)1.0 - (T)0.0) / (T)e->nx, dy = ((T)1.0 - (T)0.0) / (T)e->ny;
  for (int j = 0; j < e->ny; j++) {
    const T y = (T)0.0 + (j + (T)0.5) * dy;
    for (int i = 0; i < e->nx; i++) {
      const T x = (T)0.0 + (i + (T)0.5) * dx;
      const T* s = (x >= (T)0.5 && y >= (T)0.5) ? q[0] : (x < (T)0.5 && y >= (T)0.5) ? q[1]
                 : (x < (T)0.5 && y < (T)0.5) ? q[2] : q[3];
      T U[4];
      prim_to_cons(s, U);
      for (int k = 0; k < 4; k++) u[(size_t)k * e->plane + (size_t)j * e->pitch + i] = U[k];
    }
  }
}

// Shock-bubble initial state (euler2d_cpu.cpp:109-150): the post-shock state
// of a Mach 1.22 shock in air from the Rankine-Hugoniot relations (T
// arithmetic), a helium bubble of radius 2.5 cm centred at (3.5, 4.45) cm,
// the shock at x = 0.5 cm.  Cell centres and the comparisons with the
// binary64 constants are binary64 expressions, as in the reference.
template <class T>
void init_shock_bubble(const pmhd_euler2d* e, std::vector<unsigned char>& buf) {
  buf.assign((size_t)4 * e->plane * sizeof(T), 0);
  T* u = reinterpret_cast<T*>(buf.data());
  const T M = (T)1.22, g = (T)1.4, rho1 = (T)1.29, p1 = (T)101325.0;
  const T c1 = std::sqrt(g * p1 / rho1);
  const T rho2 = rho1 * ((g + 1) * M * M) / ((g - 1) * M * M + 2);
  const T p2 = p1 * (2 * g * M * M - (g - 1)) / (g + 1);
  const T u2 = c1 * M * (1 - rho1 / rho2);
  const T R2 = (T)(0.025 * 0.025);
  const double dx = (double)e->dx, dy = (double)e->dy;
  for (int j = 0; j < e->ny; j++) {
    const T y = (T)(0.0 + (j + 0.5) * dy);
    for (int i = 0; i < e->nx; i++) {
      const T x = (T)(0.0 + (i + 0.5) * dx);
      const T dxb = (T)((double)x - 0.035), dyb = (T)((double)y - 0.089 / 2.0);
      const T d2 = dxb * dxb + dyb * dyb;
      T W[4];
      if (d2 < R2) {
        W[0] = (T)0.214, W[1] = (T)0.0, W[2] = (T)0.0, W[3] = p1;
      } else if ((double)x < 0.005) {
        W[0] = rho2, W[1] = u2, W[2] = (T)0.0, W[3] = p2;
      } else {
        W[0] = rho1, W[1] = (T)0.0, W[2] = (T)0.0, W[3] = p1;
      }
      T U[4];
      prim_to_cons(W, U);
      for (int k = 0; k < 4; k++) u[(size_t)k * e->plane + (size_t)j * e->pitch + i] = U[k];
    }
  }
}

cudaError_t enqueue_steps(pmhd_euler2d* e, int nsteps) {
  for (int k = 0; k < nsteps; k++) {
    const int p = k & 1;
    const cudaError_t r =
        e->exact ? exact::step2d(e->fp32, e->hll, e->u[p], e->u[p ^ 1], e->nx, e->ny, e->pitch, e->plane, e->dx,
                                 e->dy, e->cfl, e->dctrl, p, e->stream)
                 : fast::step2d(e->fp32, e->hll, e->u[p], e->u[p ^ 1], e->nx, e->ny, e->pitch, e->plane, e->dx, e->dy,
                                e->cfl, e->dctrl, p, e->stream);
    if (r != cudaSuccess) return r;
  }
  return cudaSuccess;
}

int build_graph(pmhd_euler2d* e, int nsteps, cudaGraphExec_t* out) {
  if (*out) return PMHD_OK;
  cudaGraph_t g = nullptr;
  E_CU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e1 = enqueue_steps(e, nsteps);
  const cudaError_t e2 = cudaStreamEndCapture(e->stream, &g);
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return PMHD_ERR_CUDA;
  }
  const cudaError_t e3 = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  return e3 == cudaSuccess ? PMHD_OK : PMHD_ERR_CUDA;
}

template <class T>
void prims_from_cons(const std::vector<unsigned char>& buf, const pmhd_euler2d* e, void* host) {
  const T* u = reinterpret_cast<const T*>(buf.data());
  T* out = static_cast<T*>(host);
  for (int j = 0; j < e->ny; j++)
    for (int i = 0; i < e->nx; i++) {
      T U[4], W[4];
      for (int k = 0; k < 4; k++) U[k] = u[(size_t)k * e->plane + (size_t)j * e->pitch + i];
      cons_to_prim(U, W);
      for (int k = 0; k < 4; k++) out[((size_t)j * e->nx + i) * 4 + k] = W[k];
    }
}

// Toro test states rhoL uL pL rhoR uR pR T_end x0 (riemann1d_cpu.cpp:43-62).
bool toro(int id, double s[8]) {
  static const double tc[5][8] = {{1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.25, 0.5},
                                  {1.0, -2.0, 0.4, 1.0, 2.0, 0.4, 0.15, 0.5},
                                  {1.0, 0.0, 1000.0, 1.0, 0.0, 0.01, 0.012, 0.5},
                                  {1.0, 0.0, 0.01, 1.0, 0.0, 100.0, 0.035, 0.5},
                                  {5.99924, 19.5975, 460.894, 5.99242, -6.19633, 46.0950, 0.035, 0.4}};
  if (id < 1 || id > 5) return false;
  std::memcpy(s, tc[id - 1], sizeof(tc[0]));
  return true;
}

template <class T>
void init_1d(int n, const double sd[8], std::vector<unsigned char>& buf) {
  const int GH = 2, TOT = n + 4;
  buf.assign((size_t)3 * TOT * sizeof(T), 0);
  T* u = reinterpret_cast<T*>(buf.data());
  T s[8];
  for (int k = 0; k < 8; k++) s[k] = (T)sd[k];
  const T DX = ((T)1.0 - (T)0.0) / (T)n;
  for (int i = 0; i < TOT; i++) {
    const T x = (T)0.0 + (T)(i - GH + 0.5) * DX;
    T rho, uu, p;
    if (x < s[7]) {
      rho = s[0];
      uu = s[1];
      p = s[2];
    } else {
      rho = s[3];
      uu = s[4];
      p = s[5];
    }
    u[i] = rho;
    u[TOT + i] = rho * uu;
    u[2 * TOT + i] = (T)(p / (G - (T)1.0) + (T)0.5 * rho * uu * uu);
  }
}

template <class T>
void out_1d(const std::vector<unsigned char>& buf, int n, void* host) {
  const int GH = 2, TOT = n + 4;
  const T* u = reinterpret_cast<const T*>(buf.data());
  T* o = static_cast<T*>(host);
  for (int i = 0; i < n; i++) {
    const T rho = u[GH + i], ru = u[TOT + GH + i], E = u[2 * TOT + GH + i];
    const T uu = ru / rho;
    o[i * 3 + 0] = rho;
    o[i * 3 + 1] = uu;
    o[i * 3 + 2] = (T)((G - (T)1.0) * (E - (T)0.5 * rho * uu * uu));
  }
}

}  // namespace

extern "C" {

int pmhd_euler2d_destroy(pmhd_euler2d* e) {
  if (!e) return PMHD_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph_big) cudaGraphExecDestroy(e->graph_big);
  if (e->graph_two) cudaGraphExecDestroy(e->graph_two);
  for (int b = 0; b < 2; b++) {
    if (e->u[b]) cudaFree(e->u[b]);
    if (e->evp[b]) cudaEventDestroy(e->evp[b]);
  }
  if (e->dctrl) cudaFree(e->dctrl);
  if (e->hctrl) cudaFreeHost(e->hctrl);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return PMHD_OK;
}

int pmhd_euler2d_create(int nx, int ny, int config, int solver, int precision, int exact, int device,
                        pmhd_euler2d** out) {
  if (!out) return PMHD_ERR_ARG;
  *out = nullptr;
  double q[4][4], t_end = 0.0011741;  // euler2d: T_END (include/euler/config.hpp)
  const bool sb = config == PMHD_EULER_SHOCK_BUBBLE;
  if (nx < 2 || ny < 2 || (long long)nx * ny > (1LL << 31) || (!sb && !lw_config(config, q, &t_end)))
    return PMHD_ERR_ARG;
  if (solver != PMHD_SOLVER_HLL && solver != PMHD_SOLVER_HLLC) return PMHD_ERR_ARG;
  if (precision != PMHD_FP64 && precision != PMHD_FP32) return PMHD_ERR_ARG;
  int rc = check_device(device);
  if (rc != PMHD_OK) return rc;
  rc = prepare_device(device, exact ? 1 : 0);
  if (rc != PMHD_OK) return rc;
  pmhd_euler2d* e = new (std::nothrow) pmhd_euler2d();
  if (!e) return PMHD_ERR_NOMEM;
  e->nx = nx;
  e->ny = ny;
  e->pitch = (nx + 31) / 32 * 32;
  e->plane = (long long)e->pitch * ny;
  e->config = config;
  e->hll = solver == PMHD_SOLVER_HLL;
  e->fp32 = precision == PMHD_FP32;
  e->exact = exact ? 1 : 0;
  e->device = device;
  e->elem = e->fp32 ? 4 : 8;
  e->t_end_cfg = t_end;
  e->wide_time = sb ? 1 : 0;
  // Domain lengths: [0,1]^2, or the shock-bubble's X_MAX - X_MIN and Y_MAX - Y_MIN
  // (binary64 differences, rounded to the run's type as config.hpp's DX / DY do).
  const double lx = sb ? 0.225 - 0.0 : 1.0, ly = sb ? 0.089 - 0.0 : 1.0;
  std::vector<unsigned char> host;
  if (e->fp32) {
    const float dx = (float)lx / (float)nx, dy = (float)ly / (float)ny;
    e->dx = dx;
    e->dy = dy;
    e->cfl = sb ? 0.8 : (double)0.8f;
    if (sb)
      init_shock_bubble<float>(e, host);
    else
      init_2d<float>(e, q, host);
  } else {
    e->dx = lx / nx;
    e->dy = ly / ny;
    e->cfl = 0.8;
    if (sb)
      init_shock_bubble<double>(e, host);
    else
      init_2d<double>(e, q, host);
  }
  const size_t bytes = (size_t)4 * e->plane * e->elem;
  bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&e->u[0], bytes) == cudaSuccess && cudaMalloc(&e->u[1], bytes) == cudaSuccess &&
            cudaMalloc(&e->dctrl, sizeof(EulerCtrl)) == cudaSuccess &&
            cudaMallocHost(&e->hctrl, 3 * sizeof(EulerCtrl)) == cudaSuccess &&
            cudaEventCreate(&e->ev0) == cudaSuccess && cudaEventCreate(&e->ev1) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->evp[0], cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->evp[1], cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(e->u[0], host.data(), bytes, cudaMemcpyHostToDevice, e->stream) == cudaSuccess &&
       cudaMemsetAsync(e->u[1], 0, bytes, e->stream) == cudaSuccess &&
       cudaStreamSynchronize(e->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    pmhd_euler2d_destroy(e);
    return PMHD_ERR_NOMEM;
  }
  *out = e;
  return PMHD_OK;
}

int pmhd_euler2d_advance(pmhd_euler2d* e, double t_end, long long max_steps, pmhd_euler_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!e) return PMHD_ERR_ARG;
  E_CU(cudaSetDevice(e->device));
  if (t_end < 0) t_end = e->t_end_cfg;
  if (e->fp32 && !e->wide_time) t_end = (double)(float)t_end;
  EulerCtrl& h = e->hctrl[0];
  std::memset(&h, 0, sizeof(h));
  h.t[0] = h.t[1] = e->t;
  h.step[0] = h.step[1] = e->steps;
  h.t_end = t_end;
  h.step_limit = max_steps < 0 ? LLONG_MAX : e->steps + max_steps;
  h.stop = e->stopped ? 1 : 0;
  h.wide_time = e->wide_time;
  h.cfl = e->cfl;
  E_CU(cudaMemcpyAsync(e->dctrl, &h, sizeof(h), cudaMemcpyHostToDevice, e->stream));
  E_CU(cudaEventRecord(e->ev0, e->stream));
  const int slot = (int)(e->steps % 3);
  E_CU(e->exact ? exact::speed2d(e->fp32, e->u[0], e->nx, e->ny, e->pitch, e->plane, e->dctrl, slot, e->stream)
                : fast::speed2d(e->fp32, e->u[0], e->nx, e->ny, e->pitch, e->plane, e->dctrl, slot, e->stream));
  if (build_graph(e, e->big, &e->graph_big) != PMHD_OK || build_graph(e, 2, &e->graph_two) != PMHD_OK)
    return PMHD_ERR_CUDA;
  auto finished = [&](const EulerCtrl& c) {
    return c.stop || !(c.t[0] < c.t_end) || c.step[0] >= c.step_limit;
  };
  if (max_steps >= 0) {
    long long left = max_steps + (max_steps & 1);
    for (; left >= e->big; left -= e->big) E_CU(cudaGraphLaunch(e->graph_big, e->stream));
    for (; left > 0; left -= 2) E_CU(cudaGraphLaunch(e->graph_two, e->stream));
  } else {
    long long issued = 0;
    auto issue = [&]() -> cudaError_t {
      const int b = (int)(issued & 1);
      cudaError_t r = cudaGraphLaunch(e->graph_big, e->stream);
      if (r == cudaSuccess)
        r = cudaMemcpyAsync(&e->hctrl[1 + b], e->dctrl, sizeof(EulerCtrl), cudaMemcpyDeviceToHost, e->stream);
      if (r == cudaSuccess) r = cudaEventRecord(e->evp[b], e->stream);
      issued++;
      return r;
    };
    E_CU(issue());
    for (long long k = 0;; k++) {
      E_CU(issue());
      E_CU(cudaEventSynchronize(e->evp[k & 1]));
      if (finished(e->hctrl[1 + (k & 1)])) break;
    }
  }
  E_CU(cudaEventRecord(e->ev1, e->stream));
  E_CU(cudaMemcpyAsync(&e->hctrl[1], e->dctrl, sizeof(EulerCtrl), cudaMemcpyDeviceToHost, e->stream));
  E_CU(cudaStreamSynchronize(e->stream));
  const EulerCtrl& c = e->hctrl[1];
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e->ev0, e->ev1);
  const long long done = c.step[0] - e->steps;
  e->t = c.t[0];
  e->steps = c.step[0];
  e->stopped = c.stop != 0;
  if (stats) {
    stats->steps = e->steps;
    stats->t = e->t;
    stats->device_ms = ms;
    stats->status = PMHD_OK;
  }
  (void)done;
  return PMHD_OK;
}

int pmhd_euler2d_get_prim(pmhd_euler2d* e, void* host) {
  if (!e || !host) return PMHD_ERR_ARG;
  E_CU(cudaSetDevice(e->device));
  std::vector<unsigned char> buf((size_t)4 * e->plane * e->elem);
  // Graphs hold an even number of steps, so the state is always in u[0].
  E_CU(cudaMemcpyAsync(buf.data(), e->u[0], buf.size(), cudaMemcpyDeviceToHost, e->stream));
  E_CU(cudaStreamSynchronize(e->stream));
  if (e->fp32)
    prims_from_cons<float>(buf, e, host);
  else
    prims_from_cons<double>(buf, e, host);
  return PMHD_OK;
}

int pmhd_euler1d_run(int n, int test, int solver, int precision, int exact, int device, void* host_out,
                     pmhd_euler_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  double s[8];
  if (n < 2 || n > (1 << 24) || !toro(test, s)) return PMHD_ERR_ARG;
  if (solver != PMHD_SOLVER_HLL && solver != PMHD_SOLVER_HLLC) return PMHD_ERR_ARG;
  if (precision != PMHD_FP64 && precision != PMHD_FP32) return PMHD_ERR_ARG;
  int rc = check_device(device);
  if (rc != PMHD_OK) return rc;
  const int fp32 = precision == PMHD_FP32, hll = solver == PMHD_SOLVER_HLL;
  const size_t elem = fp32 ? 4 : 8;
  std::vector<unsigned char> host;
  if (fp32)
    init_1d<float>(n, s, host);
  else
    init_1d<double>(n, s, host);
  const double t_end = fp32 ? (double)(float)s[6] : s[6];
  void *du = nullptr, *df = nullptr, *dscr = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  struct Scratch {
    double t;
    long long steps;
    int err;
  };
  Scratch hs{};
  rc = PMHD_OK;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&du, host.size()) != cudaSuccess ||
      cudaMalloc(&df, host.size()) != cudaSuccess || cudaMalloc(&dscr, sizeof(Scratch)) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = PMHD_ERR_NOMEM;
  Scratch* d = static_cast<Scratch*>(dscr);
  if (rc == PMHD_OK) {
    cudaError_t r = cudaMemcpyAsync(du, host.data(), host.size(), cudaMemcpyHostToDevice, st);
    if (r == cudaSuccess) r = cudaMemsetAsync(df, 0, host.size(), st);
    if (r == cudaSuccess) r = cudaMemsetAsync(dscr, 0, sizeof(Scratch), st);
    if (r == cudaSuccess) r = cudaEventRecord(e0, st);
    const long long max_iters = 50000000LL;
    if (r == cudaSuccess)
      r = exact ? exact::run1d(fp32, hll, du, df, n, t_end, max_iters, &d->t, &d->steps, &d->err, st)
                : fast::run1d(fp32, hll, du, df, n, t_end, max_iters, &d->t, &d->steps, &d->err, st);
    if (r == cudaSuccess) r = cudaEventRecord(e1, st);
    if (r == cudaSuccess) r = cudaMemcpyAsync(&hs, dscr, sizeof(Scratch), cudaMemcpyDeviceToHost, st);
    if (r == cudaSuccess) r = cudaMemcpyAsync(host.data(), du, host.size(), cudaMemcpyDeviceToHost, st);
    if (r == cudaSuccess) r = cudaStreamSynchronize(st);
    if (r != cudaSuccess) rc = PMHD_ERR_CUDA;
  }
  if (rc == PMHD_OK) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (stats) {
      stats->steps = hs.steps;
      stats->t = hs.t;
      stats->device_ms = ms;
      stats->status = hs.err ? PMHD_ERR_TIMEOUT : PMHD_OK;
    }
    if (hs.err) rc = PMHD_ERR_TIMEOUT;
    if (host_out) {
      if (fp32)
        out_1d<float>(host, n, host_out);
      else
        out_1d<double>(host, n, host_out);
    }
  }
  cudaGetLastError();
  if (du) cudaFree(du);
  if (df) cudaFree(df);
  if (dscr) cudaFree(dscr);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  (void)elem;
  return rc;
}

}  // extern "C"
