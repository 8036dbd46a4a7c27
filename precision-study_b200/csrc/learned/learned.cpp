// learned.cpp -- pmhd_learned_*: the learned coarse-grid correction's
// runtime (declared in include/pmhd.h): the training-pair store filled from
// fine and coarse solver runs, device training with the project's own BF16
// tensor-core forward / backward kernels and Adam (one CUDA graph per
// iteration), and corrected coarse runs in which the correction is captured
// into the solver's own step graphs through its step hooks.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "learned/conv.h"
#include "learned/net.h"
#include "pmhd.h"
#include "solver_internal.h"

using namespace pmhd;
using namespace pmhd::learned;

struct pmhd_learned {
  pmhd_learned_config cfg;
  cudaStream_t stream = nullptr;
  NetLayout L;
  NetWeights w{};
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  Norm hnorm{};
  Norm* dnorm = nullptr;
  bool have_norm = false;
  int npairs = 0;
  size_t pair_elems = 0;  // doubles per stored state
  double* px = nullptr;   // states before the coarse step, AoS interior, [max_pairs]
  double* py = nullptr;   // after the plain coarse step
  double* pz = nullptr;   // restricted fine state at the same time
  int* err = nullptr;     // device error word of the convolution kernels
  int trains = 0;
};

namespace {

#define L_CU(call)                                   \
  do {                                               \
    if ((call) != cudaSuccess) {                     \
      cudaGetLastError();                            \
      return PMHD_ERR_CUDA;                          \
    }                                                \
  } while (0)

unsigned long long splitmix64(unsigned long long& x) {
  unsigned long long z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
double uniform01(unsigned long long& x) { return ((double)(splitmix64(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
double normal01(unsigned long long& x) {  // Box-Muller
  const double u1 = uniform01(x), u2 = uniform01(x);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

pmhd_config solver_config(const pmhd_learned_config& c, int factor) {
  pmhd_config s;
  pmhd_config_default(&s);
  s.nx = c.nx * factor;
  s.ny = c.ny * factor;
  s.x_min = c.x_min;
  s.x_max = c.x_max;
  s.y_min = c.y_min;
  s.y_max = c.y_max;
  s.gamma = c.gamma;
  s.cfl = c.cfl;
  s.alpha = c.alpha;
  s.precision = c.precision;
  s.device = c.device;
  for (int k = 0; k < 4; k++) s.bc[k] = PMHD_BC_PERIODIC;
  s.autotune = 0;
  return s;
}

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}

// RAII owner of a solver handle.
struct SolverHandle {
  pmhd_solver* s = nullptr;
  ~SolverHandle() {
    if (s) pmhd_destroy(s);
  }
};

// Restricted fine initial state of `problem` loaded into the coarse solver.
int load_restricted_ic(pmhd_learned* L, pmhd_solver* coarse, int problem, const double* params, int nparams,
                       double* scratch) {
  const pmhd_config fc = solver_config(L->cfg, L->cfg.refine);
  SolverHandle f;
  int rc = pmhd_create(&fc, &f.s);
  if (rc != PMHD_OK) return rc;
  rc = pmhd_init_problem(f.s, problem, params, nparams);
  if (rc != PMHD_OK) return rc;
  SolverView vf, vc;
  solver_view(f.s, &vf);
  solver_view(coarse, &vc);
  L_CU(restrict_state(vf.u, vf.pitch, vf.plane, vf.nx, vf.ny, L->cfg.refine, scratch, vc.stream));
  L_CU(load_periodic(scratch, vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, vc.stream));
  L_CU(cudaStreamSynchronize(vc.stream));
  return pmhd_set_time(coarse, 0.0, 0);
}

void fill_stats(pmhd_learned_stats* out, const pmhd_stats& st, double wall_ms) {
  if (!out) return;
  out->steps = st.steps;
  out->t = st.t;
  out->device_ms = st.device_ms;
  out->wall_ms = wall_ms;
  out->status = st.status;
}

// Every copy and memset below is stream-ordered on the stream whose kernels
// use the memory: the library's streams are non-blocking, so they are not
// ordered after the legacy default stream.
int check_err(pmhd_learned* L, cudaStream_t s) {
  int h = 0;
  L_CU(cudaMemcpyAsync(&h, L->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  L_CU(cudaStreamSynchronize(s));
  return h ? PMHD_ERR_TIMEOUT : PMHD_OK;
}

// Device buffers of the per-step correction of one coarse grid.
struct CorrBuffers {
  CorrState cs{};
  std::vector<void*> owned;
  // plane: elements per SoA plane of the coarse solver; pix = nx * ny.
  int alloc(const pmhd_learned* L, long long plane, long long pix, cudaStream_t s) {
    auto grab = [&](cudaError_t e, void* p) {
      owned.push_back(p);
      return e == cudaSuccess;
    };
    bool ok = grab(dalloc(&cs.before, (size_t)kNVar * plane), cs.before);
    ok = ok && grab(dalloc(&cs.cand, (size_t)pix * kNVar), cs.cand);
    ok = ok && grab(dalloc(&cs.x, (size_t)pix * kFeat), cs.x) && grab(dalloc(&cs.z1, (size_t)pix * kWidth), cs.z1);
    ok = ok && grab(dalloc(&cs.a1, (size_t)pix * kWidth), cs.a1) && grab(dalloc(&cs.z2, (size_t)pix * kWidth), cs.z2);
    ok = ok && grab(dalloc(&cs.a2, (size_t)pix * kWidth), cs.a2) && grab(dalloc(&cs.out, (size_t)pix * kOut), cs.out);
    ok = ok && grab(dalloc(&cs.z3, (size_t)pix * kWidth), cs.z3) && grab(dalloc(&cs.a3, (size_t)pix * kWidth), cs.a3);
    ok = ok && grab(dalloc(&cs.flags, 4), cs.flags) && grab(dalloc(&cs.sums, kCorrSums), cs.sums);
    ok = ok && grab(dalloc(&cs.counters, 4), cs.counters) && grab(dalloc(&cs.accept, 4), cs.accept);
    if (!ok) {
      cudaGetLastError();
      return PMHD_ERR_NOMEM;
    }
    cs.norm = L->dnorm;
    cs.relax = L->cfg.relax;
    cs.shrink = L->cfg.shrink;
    cudaError_t e = cudaMemsetAsync(cs.flags, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cs.sums, 0, kCorrSums * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cs.counters, 0, 4 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? PMHD_OK : PMHD_ERR_CUDA;
  }
  ~CorrBuffers() {
    for (void* p : owned)
      if (p) cudaFree(p);
  }
};

// The network on one coarse grid: features of (u after the step, the state
// before it) -> four convolutions -> cs.out.
cudaError_t net_infer(const NetLayout& N, const NetWeights& W, const CorrState& cs, const void* u, int pitch,
                      long long plane, int nx, int ny, int* err, cudaStream_t s) {
  cudaError_t r = features(soa_view(u, pitch, plane), soa_view(cs.before, pitch, plane), 1, nx, ny, cs.norm, cs.x, s);
  if (r == cudaSuccess)
    r = conv3x3(CONV_GELU, cs.x, 1, ny, nx, kFeat, W.wf[0], W.theta + N.b_off[0], kWidth, nullptr, cs.z1, cs.a1, err,
                s);
  if (r == cudaSuccess)
    r = conv3x3(CONV_GELU, cs.a1, 1, ny, nx, kWidth, W.wf[1], W.theta + N.b_off[1], kWidth, nullptr, cs.z2, cs.a2, err,
                s);
  if (r == cudaSuccess)
    r = conv3x3(CONV_GELU, cs.a2, 1, ny, nx, kWidth, W.wf[2], W.theta + N.b_off[2], kWidth, nullptr, cs.z3, cs.a3, err,
                s);
  if (r == cudaSuccess)
    r = conv3x3(CONV_LINEAR, cs.a3, 1, ny, nx, kWidth, W.wf[3], W.theta + N.b_off[3], kOut, nullptr, cs.out, nullptr,
                err, s);
  return r;
}

}  // namespace

extern "C" {

int pmhd_learned_config_default(pmhd_learned_config* c) {
  if (!c) return PMHD_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->nx = c->ny = 64;
  c->refine = 4;
  c->x_min = 0.0;
  c->x_max = 1.0;
  c->y_min = 0.0;
  c->y_max = 1.0;
  c->gamma = 5.0 / 3.0;
  c->cfl = 0.25;
  c->alpha = 0.18;
  c->precision = PMHD_MIXED;
  c->device = 0;
  c->max_pairs = 512;
  c->seed = 1;
  c->div_tol = 0.5;
  c->relax = 0.25;
  c->train_noise = 0.03;
  c->shrink = 0.0;
  return PMHD_OK;
}

int pmhd_learned_destroy(pmhd_learned* L) {
  if (!L) return PMHD_OK;
  cudaSetDevice(L->cfg.device);
  if (L->stream) cudaStreamSynchronize(L->stream);
  void* ptrs[] = {L->w.theta, L->grad, L->m, L->v, L->dnorm, L->px, L->py, L->pz, L->err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int l = 0; l < kLayers; l++) {
    if (L->w.wf[l]) cudaFree(L->w.wf[l]);
    if (L->w.wb[l]) cudaFree(L->w.wb[l]);
  }
  if (L->stream) cudaStreamDestroy(L->stream);
  delete L;
  return PMHD_OK;
}

int pmhd_learned_create(const pmhd_learned_config* cfg, pmhd_learned** out) {
  if (!out) return PMHD_ERR_ARG;
  *out = nullptr;
  if (!cfg || cfg->nx < 8 || cfg->ny < 8 || cfg->refine < 2 || cfg->refine > 16 || cfg->max_pairs < 1 ||
      !(cfg->x_max > cfg->x_min) || !(cfg->y_max > cfg->y_min) || !(cfg->gamma > 1.0) || !(cfg->cfl > 0.0) ||
      !(cfg->cfl < 1.0) || !(cfg->alpha > 0.0) || !(cfg->div_tol >= 0.0) ||
      !(cfg->relax >= 0.0) || !(cfg->relax <= 1.0) || !(cfg->train_noise >= 0.0) ||
      !(cfg->shrink >= 0.0))
    return PMHD_ERR_ARG;
  if (cfg->precision != PMHD_FP64 && cfg->precision != PMHD_MIXED) return PMHD_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
    cudaGetLastError();
    return PMHD_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  L_CU(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major != 10 || prop.minor != 0) return PMHD_ERR_NODEVICE;
  L_CU(cudaSetDevice(cfg->device));
  pmhd_learned* L = new (std::nothrow) pmhd_learned();
  if (!L) return PMHD_ERR_NOMEM;
  L->cfg = *cfg;
  L->L = net_layout();
  if (conv_prepare() != cudaSuccess) {
    cudaGetLastError();
    delete L;
    return PMHD_ERR_CUDA;
  }
  const int np = L->L.n_params;
  L->pair_elems = (size_t)cfg->nx * cfg->ny * kNVar;
  bool ok = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && dalloc(&L->w.theta, np) == cudaSuccess && dalloc(&L->grad, np) == cudaSuccess &&
       dalloc(&L->m, np) == cudaSuccess && dalloc(&L->v, np) == cudaSuccess && dalloc(&L->dnorm, 1) == cudaSuccess &&
       dalloc(&L->err, 1) == cudaSuccess;
  for (int l = 0; ok && l < kLayers; l++) {
    const size_t n = (size_t)L->L.cout[l] * 9 * L->L.cin[l];
    ok = dalloc(&L->w.wf[l], n) == cudaSuccess && dalloc(&L->w.wb[l], n) == cudaSuccess;
  }
  const size_t pbytes = (size_t)cfg->max_pairs * L->pair_elems;
  ok = ok && dalloc(&L->px, pbytes) == cudaSuccess && dalloc(&L->py, pbytes) == cudaSuccess &&
       dalloc(&L->pz, pbytes) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    pmhd_learned_destroy(L);
    return PMHD_ERR_NOMEM;
  }
  // He-normal weights over the inputs in use; unused inputs and outputs 0;
  // the last layer starts near zero so the untrained correction is ~0.
  std::vector<float> th(np, 0.f);
  unsigned long long st = cfg->seed;
  const int used_in[kLayers] = {2 * kNVar, kWidth, kWidth, kWidth}, used_out[kLayers] = {kWidth, kWidth, kWidth, 8};
  for (int l = 0; l < kLayers; l++) {
    const double sd = (l < kLayers - 1 ? std::sqrt(2.0 / (9.0 * used_in[l]))
                                       : 0.01 * std::sqrt(1.0 / (9.0 * used_in[l])));
    for (int co = 0; co < L->L.cout[l]; co++)
      for (int t = 0; t < 9; t++)
        for (int ci = 0; ci < L->L.cin[l]; ci++) {
          const double r = normal01(st);
          if (co < used_out[l] && ci < used_in[l])
            th[L->L.w_off[l] + (co * 9 + t) * L->L.cin[l] + ci] = (float)(sd * r);
        }
  }
  int rc = PMHD_OK;
  cudaStream_t s = L->stream;
  if (cudaMemcpyAsync(L->w.theta, th.data(), np * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(L->grad, 0, np * sizeof(float), s) != cudaSuccess ||
      cudaMemsetAsync(L->m, 0, np * sizeof(float), s) != cudaSuccess ||
      cudaMemsetAsync(L->v, 0, np * sizeof(float), s) != cudaSuccess ||
      cudaMemsetAsync(L->err, 0, sizeof(int), s) != cudaSuccess ||
      weights_to_bf16(L->L, L->w, L->stream) != cudaSuccess || cudaStreamSynchronize(L->stream) != cudaSuccess)
    rc = PMHD_ERR_CUDA;
  if (rc != PMHD_OK) {
    cudaGetLastError();
    pmhd_learned_destroy(L);
    return rc;
  }
  *out = L;
  return PMHD_OK;
}

int pmhd_learned_num_pairs(const pmhd_learned* L) { return L ? L->npairs : 0; }

}  // extern "C"

namespace {

// Training pairs (before, plain coarse step, restricted fine state at the
// same time) along a fine run.  mode PAIRS_FINE: every coarse step starts
// from the restricted fine state; PAIRS_ROLLOUT: the coarse run keeps its own
// state after the first step (the plain coarse trajectory); PAIRS_CORRECTED:
// the coarse run is corrected by the current network after every step (the
// states a corrected run meets, DAgger-style data aggregation).  The target
// is always the restricted fine state at the same time.
enum PairMode { PAIRS_FINE = 0, PAIRS_ROLLOUT = 1, PAIRS_CORRECTED = 2 };

int generate_pairs(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int every,
                   int* added, int mode) {
  if (added) *added = 0;
  if (!L || every < 1 || !(t_end > 0.0)) return PMHD_ERR_ARG;
  if (mode == PAIRS_CORRECTED && !L->have_norm) return PMHD_ERR_ARG;  // needs a trained network
  const bool rollout = mode != PAIRS_FINE;
  L_CU(cudaSetDevice(L->cfg.device));
  const int r = L->cfg.refine;
  const pmhd_config fc = solver_config(L->cfg, r), cc = solver_config(L->cfg, 1);
  SolverHandle f, c;
  int rc = pmhd_create(&fc, &f.s);
  if (rc == PMHD_OK) rc = pmhd_create(&cc, &c.s);
  if (rc == PMHD_OK) rc = pmhd_init_problem(f.s, problem, params, nparams);
  if (rc != PMHD_OK) return rc;
  SolverView vf, vc;
  solver_view(f.s, &vf);
  solver_view(c.s, &vc);
  CorrBuffers cb;
  if (mode == PAIRS_CORRECTED) {
    rc = cb.alloc(L, vc.plane, (long long)vc.nx * vc.ny, vc.stream);
    if (rc != PMHD_OK) return rc;
  }
  const size_t state_bytes = (size_t)kNVar * vc.plane * sizeof(double);
  double *cur = nullptr, *nxt = nullptr, *yy = nullptr;
  if (dalloc(&cur, L->pair_elems) != cudaSuccess || dalloc(&nxt, L->pair_elems) != cudaSuccess ||
      dalloc(&yy, L->pair_elems) != cudaSuccess) {
    cudaFree(cur);
    cudaFree(nxt);
    cudaGetLastError();
    return PMHD_ERR_NOMEM;
  }
  const size_t bytes = L->pair_elems * sizeof(double);
  double t = 0.0;
  long long k = 0;
  int n_added = 0;
  cudaError_t e = restrict_state(vf.u, vf.pitch, vf.plane, vf.nx, vf.ny, r, cur, vf.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(vf.stream);
  while (e == cudaSuccess && rc == PMHD_OK && t < t_end && L->npairs < L->cfg.max_pairs) {
    if (!rollout || k == 0) {
      e = load_periodic(cur, vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, vc.stream);
    } else {
      e = store_interior(vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, cur, vc.stream);
    }
    if (e == cudaSuccess && mode == PAIRS_CORRECTED)
      e = cudaMemcpyAsync(cb.cs.before, vc.u, state_bytes, cudaMemcpyDeviceToDevice, vc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(vc.stream);
    if (e != cudaSuccess) break;
    pmhd_set_time(c.s, t, 0);
    pmhd_stats sc, sf;
    rc = pmhd_advance(c.s, t_end, 1, &sc);
    if (rc != PMHD_OK) break;
    const double t1 = sc.t;
    e = store_interior(vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, yy, vc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(vc.stream);
    if (e != cudaSuccess) break;
    rc = pmhd_advance(f.s, t1, -1, &sf);
    if (rc != PMHD_OK) break;
    e = restrict_state(vf.u, vf.pitch, vf.plane, vf.nx, vf.ny, r, nxt, vf.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(vf.stream);
    if (e != cudaSuccess) break;
    if (k % every == 0) {
      const size_t off = (size_t)L->npairs * L->pair_elems;
      e = cudaMemcpyAsync(L->px + off, cur, bytes, cudaMemcpyDeviceToDevice, vf.stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L->py + off, yy, bytes, cudaMemcpyDeviceToDevice, vf.stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L->pz + off, nxt, bytes, cudaMemcpyDeviceToDevice, vf.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(vf.stream);
      L->npairs++;
      n_added++;
    }
    if (mode == PAIRS_CORRECTED) {
      // The network's correction of this step, applied in place to the
      // coarse state the next iteration starts from (checked as in a run).
      e = net_infer(L->L, L->w, cb.cs, vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, L->err, vc.stream);
      if (e == cudaSuccess)
        e = correct_step(cb.cs, vc.u, vc.pitch, vc.plane, vc.nx, vc.ny, vc.dx, vc.dy, vc.gamma, L->cfg.div_tol,
                         nullptr, nullptr, 0, vc.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(vc.stream);
      if (e != cudaSuccess) break;
    }
    double* tmp = cur;
    cur = nxt;
    nxt = tmp;
    t = t1;
    k++;
  }
  cudaFree(cur);
  cudaFree(nxt);
  cudaFree(yy);
  if (added) *added = n_added;
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PMHD_ERR_CUDA;
  }
  return rc;
}

}  // namespace

extern "C" {

int pmhd_learned_generate(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int every,
                          int* added) {
  return generate_pairs(L, problem, params, nparams, t_end, every, added, PAIRS_FINE);
}

int pmhd_learned_generate_rollout(pmhd_learned* L, int problem, const double* params, int nparams, double t_end,
                                  int every, int* added) {
  return generate_pairs(L, problem, params, nparams, t_end, every, added, PAIRS_ROLLOUT);
}

int pmhd_learned_generate_corrected(pmhd_learned* L, int problem, const double* params, int nparams, double t_end,
                                    int every, int* added) {
  return generate_pairs(L, problem, params, nparams, t_end, every, added, PAIRS_CORRECTED);
}

int pmhd_learned_train(pmhd_learned* L, int iters, int batch, double lr, float* losses) {
  if (!L || iters < 1 || batch < 1 || !(lr > 0.0)) return PMHD_ERR_ARG;
  if (L->npairs < 1) return PMHD_ERR_ARG;
  L_CU(cudaSetDevice(L->cfg.device));
  const int nx = L->cfg.nx, ny = L->cfg.ny, np = L->npairs;
  const long long pix = (long long)nx * ny, P = pix * batch;
  cudaStream_t s = L->stream;
  // Normalisation from all pairs, fixed at the first training.
  if (!L->have_norm) {
    double* dsum = nullptr;
    L_CU(dalloc(&dsum, kMomentSums));
    L_CU(cudaMemsetAsync(dsum, 0, kMomentSums * sizeof(double), s));
    L_CU(moments(aos_view(L->px, nx, ny), aos_view(L->py, nx, ny), aos_view(L->pz, nx, ny), np, nx, ny, L->cfg.gamma,
                 dsum, s));
    double h[kMomentSums];
    L_CU(cudaMemcpyAsync(h, dsum, sizeof(h), cudaMemcpyDeviceToHost, s));
    L_CU(cudaStreamSynchronize(s));
    cudaFree(dsum);
    const double n = (double)np * pix;
    for (int g = 0; g < 2; g++)
      for (int k = 0; k < kNVar; k++) {
        const double mean = h[g * kNVar + k] / n;
        const double var = std::fmax(h[2 * kNVar + g * kNVar + k] / n - mean * mean, 0.0);
        const double sd = std::sqrt(var);
        const bool live = sd > 1e-12 * (1.0 + std::fabs(mean));
        L->hnorm.mu[g * kNVar + k] = (float)mean;
        L->hnorm.inv_sig[g * kNVar + k] = live ? (float)(1.0 / sd) : 0.f;
      }
    // Corrections: scale only (root mean square), no shift.  Both field
    // components share one scale so the curl of the potential is one map.
    double rms[kNOutQ];
    for (int k = 0; k < kNOutQ; k++) rms[k] = std::sqrt(std::fmax(h[4 * kNVar + kNOutQ + k] / n, 0.0));
    const double rb = std::sqrt(0.5 * (rms[TGT_DBX] * rms[TGT_DBX] + rms[TGT_DBY] * rms[TGT_DBY]));
    rms[TGT_DBX] = rms[TGT_DBY] = rb;
    const double dx = (L->cfg.x_max - L->cfg.x_min) / nx, dy = (L->cfg.y_max - L->cfg.y_min) / ny;
    rms[OUT_A] = rb * std::fmin(dx, dy);
    for (int k = 0; k < kNOutQ; k++) {
      const bool lv = rms[k] > 1e-14;
      L->hnorm.sig_out[k] = lv ? (float)rms[k] : 0.f;
      L->hnorm.inv_out[k] = lv ? (float)(1.0 / rms[k]) : 0.f;
    }
    L->hnorm.cx = rb > 1e-14 ? (float)(rms[OUT_A] / (2.0 * dx * rb)) : 0.f;
    L->hnorm.cy = rb > 1e-14 ? (float)(rms[OUT_A] / (2.0 * dy * rb)) : 0.f;
    L_CU(cudaMemcpyAsync(L->dnorm, &L->hnorm, sizeof(Norm), cudaMemcpyHostToDevice, s));
    L_CU(cudaStreamSynchronize(s));
    L->have_norm = true;
  }
  // Network inputs and targets of every pair.
  __nv_bfloat16 *feat_all = nullptr, *xb = nullptr, *z1 = nullptr, *a1 = nullptr, *z2 = nullptr, *a2 = nullptr,
                *z3 = nullptr, *a3 = nullptr, *dz4 = nullptr, *dz3 = nullptr, *dz2 = nullptr, *dz1 = nullptr;
  float *tgt_all = nullptr, *tb = nullptr, *out = nullptr, *hist = nullptr;
  int *sched = nullptr, *it = nullptr;
  std::vector<void*> owned;
  auto grab = [&](cudaError_t e, void* p) {
    owned.push_back(p);
    return e == cudaSuccess;
  };
  bool ok = grab(dalloc(&feat_all, (size_t)np * pix * kFeat), feat_all);
  ok = ok && grab(dalloc(&tgt_all, (size_t)np * pix * kOut), tgt_all);
  ok = ok && grab(dalloc(&xb, (size_t)P * kFeat), xb) && grab(dalloc(&tb, (size_t)P * kOut), tb);
  ok = ok && grab(dalloc(&z1, (size_t)P * kWidth), z1) && grab(dalloc(&a1, (size_t)P * kWidth), a1);
  ok = ok && grab(dalloc(&z2, (size_t)P * kWidth), z2) && grab(dalloc(&a2, (size_t)P * kWidth), a2);
  ok = ok && grab(dalloc(&z3, (size_t)P * kWidth), z3) && grab(dalloc(&a3, (size_t)P * kWidth), a3);
  ok = ok && grab(dalloc(&out, (size_t)P * kOut), out) && grab(dalloc(&dz4, (size_t)P * kOut), dz4);
  ok = ok && grab(dalloc(&dz3, (size_t)P * kWidth), dz3);
  ok = ok && grab(dalloc(&dz2, (size_t)P * kWidth), dz2) && grab(dalloc(&dz1, (size_t)P * kWidth), dz1);
  ok = ok && grab(dalloc(&hist, (size_t)iters), hist) && grab(dalloc(&sched, (size_t)iters * batch), sched);
  ok = ok && grab(dalloc(&it, 1), it);
  auto release = [&]() {
    for (void* p : owned)
      if (p) cudaFree(p);
  };
  if (!ok) {
    cudaGetLastError();
    release();
    return PMHD_ERR_NOMEM;
  }
  std::vector<int> hs((size_t)iters * batch);
  unsigned long long rs = L->cfg.seed * 0x2545F4914F6CDD1Dull + (unsigned long long)(++L->trains);
  for (auto& q : hs) q = (int)(splitmix64(rs) % (unsigned long long)np);
  cudaError_t e = cudaMemcpyAsync(sched, hs.data(), hs.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, (size_t)iters * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(it, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(L->err, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = features(aos_view(L->py, nx, ny), aos_view(L->px, nx, ny), np, nx, ny, L->dnorm, feat_all, s);
  if (e == cudaSuccess)
    e = targets(aos_view(L->py, nx, ny), aos_view(L->pz, nx, ny), np, nx, ny, L->dnorm, L->cfg.gamma, tgt_all, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  // One training iteration, captured once and replayed.
  const NetLayout& N = L->L;
  float* th = L->w.theta;
  float* g = L->grad;
  auto iteration = [&]() -> cudaError_t {
    cudaError_t r = gather_pairs(sched, it, batch, feat_all, tgt_all, pix, xb, tb, s);
    if (r == cudaSuccess && L->cfg.train_noise > 0.0)
      r = input_noise(xb, P, (float)L->cfg.train_noise, it, L->cfg.seed, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_GELU, xb, batch, ny, nx, kFeat, L->w.wf[0], th + N.b_off[0], kWidth, nullptr, z1, a1, L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_GELU, a1, batch, ny, nx, kWidth, L->w.wf[1], th + N.b_off[1], kWidth, nullptr, z2, a2, L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_GELU, a2, batch, ny, nx, kWidth, L->w.wf[2], th + N.b_off[2], kWidth, nullptr, z3, a3, L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_LINEAR, a3, batch, ny, nx, kWidth, L->w.wf[3], th + N.b_off[3], kOut, nullptr, out, nullptr,
                  L->err, s);
    if (r == cudaSuccess) r = loss_grad(out, tb, batch, nx, ny, L->dnorm, dz4, hist, it, s);
    if (r == cudaSuccess) r = conv3x3_wgrad(a3, dz4, batch, ny, nx, kWidth, kOut, g + N.w_off[3], g + N.b_off[3], L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_DGELU, dz4, batch, ny, nx, kOut, L->w.wb[3], nullptr, kWidth, z3, dz3, nullptr, L->err, s);
    if (r == cudaSuccess) r = conv3x3_wgrad(a2, dz3, batch, ny, nx, kWidth, kWidth, g + N.w_off[2], g + N.b_off[2], L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_DGELU, dz3, batch, ny, nx, kWidth, L->w.wb[2], nullptr, kWidth, z2, dz2, nullptr, L->err, s);
    if (r == cudaSuccess) r = conv3x3_wgrad(a1, dz2, batch, ny, nx, kWidth, kWidth, g + N.w_off[1], g + N.b_off[1], L->err, s);
    if (r == cudaSuccess)
      r = conv3x3(CONV_DGELU, dz2, batch, ny, nx, kWidth, L->w.wb[1], nullptr, kWidth, z1, dz1, nullptr, L->err, s);
    if (r == cudaSuccess) r = conv3x3_wgrad(xb, dz1, batch, ny, nx, kFeat, kWidth, g + N.w_off[0], g + N.b_off[0], L->err, s);
    if (r == cudaSuccess) r = adam(N, L->w, g, L->m, L->v, it, iters, (float)lr, s);
    if (r == cudaSuccess) r = increment(it, s);
    return r;
  };
  // The first iteration runs eagerly, the rest replay its graph.
  if (e == cudaSuccess) e = iteration();
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess && iters > 1) {
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t e1 = iteration();
      const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      e = e1 != cudaSuccess ? e1 : e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    for (int i = 1; e == cudaSuccess && i < iters; i++) e = cudaGraphLaunch(exec, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && losses)
    e = cudaMemcpyAsync(losses, hist, (size_t)iters * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  release();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorNotSupported ? PMHD_ERR_UNSUPPORTED : PMHD_ERR_CUDA;
  }
  return check_err(L, s);
}

int pmhd_learned_run(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int use_net,
                     double* host_out, pmhd_learned_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!L || !(t_end > 0.0)) return PMHD_ERR_ARG;
  if (use_net && !L->have_norm) return PMHD_ERR_ARG;  // untrained
  L_CU(cudaSetDevice(L->cfg.device));
  const pmhd_config cc = solver_config(L->cfg, 1);
  SolverHandle c;
  int rc = pmhd_create(&cc, &c.s);
  if (rc != PMHD_OK) return rc;
  SolverView vc;
  solver_view(c.s, &vc);
  const int nx = vc.nx, ny = vc.ny;
  const long long pix = (long long)nx * ny;
  CorrBuffers cb;
  rc = cb.alloc(L, vc.plane, pix, vc.stream);
  if (rc != PMHD_OK) return rc;
  const CorrState cs = cb.cs;
  if (cudaMemsetAsync(L->err, 0, sizeof(int), vc.stream) != cudaSuccess ||
      cudaStreamSynchronize(vc.stream) != cudaSuccess)
    return PMHD_ERR_CUDA;
  rc = load_restricted_ic(L, c.s, problem, params, nparams, cs.cand);
  if (rc != PMHD_OK) return rc;
  cudaError_t e = cudaSuccess;
  if (use_net) {
    const NetLayout N = L->L;
    const NetWeights W = L->w;
    const double div_tol = L->cfg.div_tol;
    int* err = L->err;
    const size_t state_bytes = (size_t)kNVar * vc.plane * sizeof(double);
    auto pre = [=](int) -> cudaError_t {
      return cudaMemcpyAsync(cs.before, vc.u, state_bytes, cudaMemcpyDeviceToDevice, vc.stream);
    };
    auto post = [=](int p) -> cudaError_t {
      cudaStream_t s = vc.stream;
      cudaError_t r = net_infer(N, W, cs, vc.u, vc.pitch, vc.plane, nx, ny, err, s);
      if (r == cudaSuccess)
        r = correct_step(cs, vc.u, vc.pitch, vc.plane, nx, ny, vc.dx, vc.dy, vc.gamma, div_tol, vc.ctrl, vc.ctrl, p, s);
      if (r == cudaSuccess)
        r = vc.kt->speed(vc.precision, vc.u, vc.plane, nx, ny, vc.pitch, vc.gamma, vc.ctrl, p ^ 1, s);
      return r;
    };
    solver_set_step_hooks(c.s, pre, post);
  }
  pmhd_stats st;
  const auto t0 = std::chrono::steady_clock::now();
  rc = pmhd_advance(c.s, t_end, -1, &st);
  const auto t1 = std::chrono::steady_clock::now();
  fill_stats(stats, st, std::chrono::duration<double, std::milli>(t1 - t0).count());
  if (rc == PMHD_OK && host_out) {
    e = store_interior(vc.u, vc.pitch, vc.plane, nx, ny, cs.cand, vc.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, cs.cand, (size_t)pix * kNVar * sizeof(double),
                                              cudaMemcpyDeviceToHost, vc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(vc.stream);
    if (e != cudaSuccess) rc = PMHD_ERR_CUDA;
  }
  if (rc == PMHD_OK && use_net && stats) {
    unsigned long long h[4];
    if (cudaMemcpyAsync(h, cs.counters, sizeof(h), cudaMemcpyDeviceToHost, vc.stream) == cudaSuccess &&
        cudaStreamSynchronize(vc.stream) == cudaSuccess) {
      stats->accepted = (long long)h[0];
      stats->rejected_positivity = (long long)h[1];
      stats->rejected_divergence = (long long)h[2];
    }
  }
  if (use_net) solver_set_step_hooks(c.s, nullptr, nullptr);
  if (rc == PMHD_OK) rc = check_err(L, vc.stream);
  return rc;
}

int pmhd_learned_fine_run(pmhd_learned* L, int problem, const double* params, int nparams, double t_end, int refine,
                          double* host_out, pmhd_learned_stats* stats) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!L || !(t_end > 0.0) || refine < 1 || refine > 32) return PMHD_ERR_ARG;
  L_CU(cudaSetDevice(L->cfg.device));
  const pmhd_config fc = solver_config(L->cfg, refine);
  SolverHandle f;
  int rc = pmhd_create(&fc, &f.s);
  if (rc == PMHD_OK) rc = pmhd_init_problem(f.s, problem, params, nparams);
  if (rc != PMHD_OK) return rc;
  pmhd_stats st;
  const auto t0 = std::chrono::steady_clock::now();
  rc = pmhd_advance(f.s, t_end, -1, &st);
  const auto t1 = std::chrono::steady_clock::now();
  fill_stats(stats, st, std::chrono::duration<double, std::milli>(t1 - t0).count());
  if (rc != PMHD_OK || !host_out) return rc;
  SolverView vf;
  solver_view(f.s, &vf);
  double* tmp = nullptr;
  L_CU(dalloc(&tmp, L->pair_elems));
  cudaError_t e = restrict_state(vf.u, vf.pitch, vf.plane, vf.nx, vf.ny, refine, tmp, vf.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host_out, tmp, L->pair_elems * sizeof(double), cudaMemcpyDeviceToHost, vf.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(vf.stream);
  cudaFree(tmp);
  return e == cudaSuccess ? PMHD_OK : PMHD_ERR_CUDA;
}

// File: "PMHDNET3", int32 n_params, Norm, n_params floats (four layers,
// physical-quantity outputs).
int pmhd_learned_save(const pmhd_learned* L, const char* path) {
  if (!L || !path || !L->have_norm) return PMHD_ERR_ARG;
  std::vector<float> th(L->L.n_params);
  if (cudaMemcpyAsync(th.data(), L->w.theta, th.size() * sizeof(float), cudaMemcpyDeviceToHost, L->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(L->stream) != cudaSuccess)
    return PMHD_ERR_CUDA;
  FILE* f = std::fopen(path, "wb");
  if (!f) return PMHD_ERR_IO;
  const int n = L->L.n_params;
  bool ok = std::fwrite("PMHDNET3", 1, 8, f) == 8 && std::fwrite(&n, sizeof(int), 1, f) == 1 &&
            std::fwrite(&L->hnorm, sizeof(Norm), 1, f) == 1 &&
            std::fwrite(th.data(), sizeof(float), th.size(), f) == th.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PMHD_OK : PMHD_ERR_IO;
}

int pmhd_learned_load(pmhd_learned* L, const char* path) {
  if (!L || !path) return PMHD_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return PMHD_ERR_IO;
  char magic[8];
  int n = 0;
  Norm nm;
  std::vector<float> th(L->L.n_params);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PMHDNET3", 8) == 0 &&
            std::fread(&n, sizeof(int), 1, f) == 1 && n == L->L.n_params &&
            std::fread(&nm, sizeof(Norm), 1, f) == 1 && std::fread(th.data(), sizeof(float), th.size(), f) == th.size();
  std::fclose(f);
  if (!ok) return PMHD_ERR_IO;
  L_CU(cudaSetDevice(L->cfg.device));
  L->hnorm = nm;
  L->have_norm = true;
  L_CU(cudaMemcpyAsync(L->dnorm, &nm, sizeof(Norm), cudaMemcpyHostToDevice, L->stream));
  L_CU(cudaMemcpyAsync(L->w.theta, th.data(), th.size() * sizeof(float), cudaMemcpyHostToDevice, L->stream));
  L_CU(weights_to_bf16(L->L, L->w, L->stream));
  L_CU(cudaStreamSynchronize(L->stream));
  return PMHD_OK;
}

}  // extern "C"
