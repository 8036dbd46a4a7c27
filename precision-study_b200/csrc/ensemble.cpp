// ensemble.cpp -- pmhd_ensemble_*: many independent grids advanced by the
// same persistent stage launches (declared in include/pmhd.h).
//
// Device layout: one allocation for every member's two state buffers (SoA
// planes as for a single solver, each member starting on a 256-byte
// boundary), one array of control blocks, one array of Member descriptors
// (TMA maps for both tile heights, pointers, physics) and, per tile height,
// the work list tables tile -> member and member -> first tile.  A member
// whose stage reports an unusable cell halts alone; the others go on.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernel_api.h"
#include "pmhd.h"
#include "runner.h"

using namespace pmhd;

struct pmhd_ensemble {
  pmhd_config cfg;
  std::vector<pmhd_member_desc> desc;
  const KernelTable* kt = nullptr;
  cudaStream_t stream = nullptr;
  size_t elem = 8;
  std::vector<Member> hm;          // host copies of the descriptors
  std::vector<size_t> state_off;   // byte offset of each member's U in dState
  void* dState = nullptr;
  Ctrl* dCtrl = nullptr;
  Ctrl* hCtrl = nullptr;           // pinned mirror, n entries
  Ctrl* hPoll = nullptr;           // pinned, 2n entries: polls one replay behind
  cudaEvent_t evPoll[2] = {nullptr, nullptr};
  Member* dMembers = nullptr;
  int* dTiles[kNumTileHeights] = {nullptr, nullptr};
  int* dTile0[kNumTileHeights] = {nullptr, nullptr};
  Runner run;
  bool tuned = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<pmhd_stats> mstats;  // per member, cumulative
  std::vector<double> t;
  std::vector<long long> steps;
  std::vector<char> failed;        // member halted on an unusable cell
  bool broken = false;             // a CUDA error or device timeout
  std::vector<int> member_ty;      // tile-height index each member runs with
  std::vector<int*> plan_lists;    // device work lists of the per-size plan
};

namespace {

#define PMHD_E(call)                                 \
  do {                                               \
    if ((call) != cudaSuccess) return PMHD_ERR_CUDA; \
  } while (0)

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

bool member_ok(const pmhd_member_desc& d) {
  if (d.nx < 4 || d.ny < 4 || (long long)d.nx * d.ny > (long long)INT_MAX / 2) return false;
  if (!(d.x_max > d.x_min) || !(d.y_max > d.y_min) || !(d.gamma > 1.0) || std::isnan(d.t_end)) return false;
  for (int k = 0; k < 4; k++)
    if (d.bc[k] < PMHD_BC_PERIODIC || d.bc[k] > PMHD_BC_TRANSMISSIVE) return false;
  if ((d.bc[0] == PMHD_BC_PERIODIC) != (d.bc[1] == PMHD_BC_PERIODIC)) return false;
  if ((d.bc[2] == PMHD_BC_PERIODIC) != (d.bc[3] == PMHD_BC_PERIODIC)) return false;
  if (d.nparams < 0 || d.nparams > 4) return false;
  return true;
}

bool common_ok(const pmhd_config* c) {
  if (!c) return false;
  if (!(c->cfl > 0.0) || !(c->cfl < 1.0) || !(c->alpha > 0.0) || !(c->hlld_tol >= 0.0)) return false;
  if (c->order != PMHD_ORDER_FIRST && c->order != PMHD_ORDER_MUSCL) return false;
  if (c->solver != PMHD_SOLVER_HLL && c->solver != PMHD_SOLVER_HLLD) return false;
  if (c->precision < PMHD_FP64 || c->precision > PMHD_MIXED) return false;
  if (c->steps_per_graph < 0 || (c->steps_per_graph & 1)) return false;
  return true;
}

// splitmix64 (Steele, Lea and Flood; constants as published by Vigna): the
// state advances by the golden-ratio increment and the output goes through
// two xor-shift-multiply rounds.
unsigned long long splitmix64(unsigned long long& x) {
  unsigned long long z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
double uniform01(unsigned long long& x) { return (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0); }

int gcd(int a, int b) { return b == 0 ? a : gcd(b, a % b); }

// The band slope k/m (k, m <= 4, coprime) whose angle atan2(k, m) is
// nearest to `angle`.
void snap_slope(double angle, int* kk, int* mm) {
  double best = 1e30;
  for (int k = 0; k <= 4; k++)
    for (int m = 0; m <= 4; m++) {
      if (k + m == 0 || gcd(k, m) != 1) continue;
      const double d = std::fabs(std::atan2((double)k, (double)m) - angle);
      if (d < best) {
        best = d;
        *kk = k;
        *mm = m;
      }
    }
}

pmhd_config member_config(const pmhd_ensemble* e, int k) {
  pmhd_config c = e->cfg;
  const pmhd_member_desc& d = e->desc[k];
  c.nx = d.nx;
  c.ny = d.ny;
  c.x_min = d.x_min;
  c.x_max = d.x_max;
  c.y_min = d.y_min;
  c.y_max = d.y_max;
  c.gamma = d.gamma;
  for (int q = 0; q < 4; q++) c.bc[q] = d.bc[q];
  return c;
}

double time_type(const pmhd_ensemble* e, double v) {
  return e->cfg.precision == PMHD_FP32 ? (double)(float)v : v;
}

// Work list (tile -> member, member -> first tile) of the members `ms` at
// tile height index t, copied to new device arrays.
cudaError_t make_work_list(pmhd_ensemble* e, const std::vector<int>& ms, int t, Batch* b, int** d_tiles,
                           int** d_tile0) {
  const int n = (int)e->desc.size();
  std::vector<int> tiles, tile0(n, 0);
  for (int k : ms) {
    tile0[k] = (int)tiles.size();
    const long long nt = (long long)((e->desc[k].nx + 31) / 32) *
                         ((e->desc[k].ny + kTileHeights[t] - 1) / kTileHeights[t]);
    tiles.insert(tiles.end(), (size_t)nt, k);
  }
  *d_tiles = nullptr;
  *d_tile0 = nullptr;
  cudaError_t err = cudaMalloc(d_tiles, sizeof(int) * tiles.size());
  if (err == cudaSuccess) err = cudaMalloc(d_tile0, sizeof(int) * n);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(*d_tiles, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(*d_tile0, tile0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  b->members = e->dMembers;
  b->tile_member = *d_tiles;
  b->member_tile0 = *d_tile0;
  b->nmembers = n;
  b->ntiles = (int)tiles.size();
  return err;
}

// The autotuner of an ensemble: every size class (members of one grid size)
// is timed on its own -- two live steps of only that class's members per
// kernel variant (tile height x resident CTAs per SM); the variants compute
// identical results, so these are ordinary steps of those members -- and
// keeps its fastest variant.  The classes that chose the same tile height
// then share one work list, whose CTA count is that of its largest class by
// cells; a step launches each such part's stage 1, then each part's stage 2.
// Returns the fewest tuning steps any member took (for step budgets) and
// adds the launches made to *launched.
cudaError_t tune_by_size(pmhd_ensemble* e, long long* min_steps, long long* launched) {
  const int n = (int)e->desc.size();
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  std::vector<std::pair<int, int>> keys;
  std::vector<std::vector<int>> classes;
  for (int k = 0; k < n; k++) {
    const std::pair<int, int> key(e->desc[k].nx, e->desc[k].ny);
    size_t c = 0;
    while (c < keys.size() && keys[c] != key) c++;
    if (c == keys.size()) {
      keys.push_back(key);
      classes.emplace_back();
    }
    classes[c].push_back(k);
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  std::vector<LaunchPart> best(classes.size());
  cudaError_t err = cudaSuccess;
  *min_steps = -1;
  for (size_t c = 0; c < classes.size() && err == cudaSuccess; c++) {
    float best_ms = -1.f;
    long long steps = 0;
    for (int t = 0; t < kNumTileHeights && err == cudaSuccess; t++) {
      LaunchPart part;
      part.ty_idx = t;
      int *dt = nullptr, *d0 = nullptr;
      err = make_work_list(e, classes[c], t, &part.batch, &dt, &d0);
      const int occ = e->kt->ctas_per_sm(e->cfg.precision, e->run.hlld, t, 1);
      for (int k = occ; k >= 1 && err == cudaSuccess; k--) {
        part.grid = k == occ ? 0 : sms * k;
        e->run.set_parts(std::vector<LaunchPart>(1, part));
        cudaEventRecord(e0, e->stream);
        err = e->run.enqueue_steps(2);
        cudaEventRecord(e1, e->stream);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        steps += 2;
        *launched += 4;
        if (best_ms < 0.f || ms < best_ms) {
          best_ms = ms;
          best[c] = part;
        }
      }
      cudaStreamSynchronize(e->stream);
      if (dt) cudaFree(dt);
      if (d0) cudaFree(d0);
    }
    if (*min_steps < 0 || steps < *min_steps) *min_steps = steps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) {
    e->run.set_parts(std::vector<LaunchPart>());
    return err;
  }
  // One part per chosen tile height.
  std::vector<LaunchPart> parts;
  for (int t = 0; t < kNumTileHeights && err == cudaSuccess; t++) {
    std::vector<int> ms;
    long long top_cells = -1;
    int grid = 0;
    for (size_t c = 0; c < classes.size(); c++) {
      if (best[c].ty_idx != t) continue;
      const long long cells = (long long)keys[c].first * keys[c].second * (long long)classes[c].size();
      if (cells > top_cells) {
        top_cells = cells;
        grid = best[c].grid;
      }
    }
    for (int k = 0; k < n; k++) {
      size_t c = 0;
      while (keys[c] != std::pair<int, int>(e->desc[k].nx, e->desc[k].ny)) c++;
      if (best[c].ty_idx == t) {
        ms.push_back(k);
        e->member_ty[k] = t;
      }
    }
    if (ms.empty()) continue;
    LaunchPart part;
    part.ty_idx = t;
    part.grid = grid;
    int *dt = nullptr, *d0 = nullptr;
    err = make_work_list(e, ms, t, &part.batch, &dt, &d0);
    if (dt) e->plan_lists.push_back(dt);
    if (d0) e->plan_lists.push_back(d0);
    parts.push_back(part);
  }
  e->run.set_parts(err == cudaSuccess ? parts : std::vector<LaunchPart>());
  return err;
}

bool finished(const Ctrl& c) { return !(c.t[0] < c.t_end) || c.step[0] >= c.step_limit; }
bool failing(const Ctrl& c) { return c.halted || c.bad1 != BAD_NONE || c.bad2 != BAD_NONE; }

}  // namespace

extern "C" {

int pmhd_ensemble_describe_default(int n, unsigned long long seed, pmhd_member_desc* out) {
  if (n < 0 || (n > 0 && !out)) return PMHD_ERR_ARG;
  static const int sizes[4] = {64, 128, 256, 512};
  unsigned long long st = seed;
  const double half_pi = 0.5 * std::acos(-1.0);
  for (int k = 0; k < n; k++) {
    pmhd_member_desc& d = out[k];
    std::memset(&d, 0, sizeof(d));
    const double u_size = uniform01(st), u_par = uniform01(st);
    (void)uniform01(st);  // spare draw: member k always uses draws 3k .. 3k+2
    int si = (int)(u_size * 4.0);
    if (si > 3) si = 3;
    d.nx = d.ny = sizes[si];
    d.x_min = 0.0;
    d.x_max = 1.0;
    d.y_min = 0.0;
    d.y_max = 1.0;
    for (int q = 0; q < 4; q++) d.bc[q] = PMHD_BC_PERIODIC;
    if ((k & 1) == 0) {
      d.gamma = 5.0 / 3.0;
      d.problem = PMHD_PROBLEM_ORSZAG_TANG;
      d.nparams = 1;
      d.params[0] = 0.5 + u_par;
      d.t_end = 0.5;
    } else {
      int kk = 1, mm = 2;
      snap_slope(u_par * half_pi, &kk, &mm);
      d.gamma = 2.0;
      d.problem = PMHD_PROBLEM_BRIO_WU_TORUS;
      d.nparams = 2;
      d.params[0] = kk;
      d.params[1] = mm;
      d.t_end = 0.1;
    }
  }
  return PMHD_OK;
}

int pmhd_ensemble_destroy(pmhd_ensemble* e) {
  if (!e) return PMHD_OK;
  cudaSetDevice(e->cfg.device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  e->run.release();
  for (int* d : e->plan_lists) cudaFree(d);
  for (int t = 0; t < kNumTileHeights; t++) {
    if (e->dTiles[t]) cudaFree(e->dTiles[t]);
    if (e->dTile0[t]) cudaFree(e->dTile0[t]);
  }
  if (e->dMembers) cudaFree(e->dMembers);
  if (e->dCtrl) cudaFree(e->dCtrl);
  if (e->dState) cudaFree(e->dState);
  if (e->hCtrl) cudaFreeHost(e->hCtrl);
  if (e->hPoll) cudaFreeHost(e->hPoll);
  for (int b = 0; b < 2; b++)
    if (e->evPoll[b]) cudaEventDestroy(e->evPoll[b]);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return PMHD_OK;
}

int pmhd_ensemble_create(const pmhd_config* common, const pmhd_member_desc* members, int n, pmhd_ensemble** out) {
  if (!out) return PMHD_ERR_ARG;
  *out = nullptr;
  if (!common_ok(common) || n <= 0 || !members) return PMHD_ERR_ARG;
  for (int k = 0; k < n; k++)
    if (!member_ok(members[k])) return PMHD_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || common->device < 0 || common->device >= ndev) {
    cudaGetLastError();
    return PMHD_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  PMHD_E(cudaGetDeviceProperties(&prop, common->device));
  if (prop.major != 10 || prop.minor != 0) return PMHD_ERR_NODEVICE;
  PMHD_E(cudaSetDevice(common->device));
  pmhd_ensemble* e = new (std::nothrow) pmhd_ensemble();
  if (!e) return PMHD_ERR_NOMEM;
  e->cfg = *common;
  if (e->cfg.steps_per_graph == 0) e->cfg.steps_per_graph = 32;
  e->desc.assign(members, members + n);
  e->kt = common->exact ? &kernel_table_exact() : &kernel_table_fast();
  e->elem = common->precision == PMHD_FP32 ? 4 : 8;
  e->mstats.assign(n, pmhd_stats());
  for (auto& st : e->mstats) {
    std::memset(&st, 0, sizeof(st));
    st.bad_i = st.bad_j = -1;
    st.bad_step = -1;
  }
  e->t.assign(n, 0.0);
  e->steps.assign(n, 0);
  e->failed.assign(n, 0);
  e->member_ty.assign(n, 0);
  int rc = PMHD_OK;
  if (e->kt->init() != cudaSuccess) rc = PMHD_ERR_CUDA;
  // Layout of the member states.
  e->hm.assign(n, Member());
  e->state_off.assign(n, 0);
  size_t total = 0;
  for (int k = 0; k < n; k++) {
    Member& m = e->hm[k];
    std::memset(&m, 0, sizeof(m));
    m.nx = members[k].nx;
    m.ny = members[k].ny;
    m.pitch = ((m.nx + 4) + 15) / 16 * 16;
    m.plane = (long long)m.pitch * (m.ny + 4);
    e->state_off[k] = total;
    total += 2 * round256((size_t)9 * m.plane * e->elem);
  }
  if (rc == PMHD_OK && cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) rc = PMHD_ERR_CUDA;
  if (rc == PMHD_OK && cudaMalloc(&e->dState, total) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMalloc(&e->dCtrl, sizeof(Ctrl) * n) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMalloc(&e->dMembers, sizeof(Member) * n) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMallocHost(&e->hCtrl, sizeof(Ctrl) * n) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && cudaMallocHost(&e->hPoll, 2 * sizeof(Ctrl) * n) != cudaSuccess) rc = PMHD_ERR_NOMEM;
  if (rc == PMHD_OK && (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess ||
                        cudaEventCreateWithFlags(&e->evPoll[0], cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventCreateWithFlags(&e->evPoll[1], cudaEventDisableTiming) != cudaSuccess))
    rc = PMHD_ERR_CUDA;
  if (rc == PMHD_OK && (cudaMemsetAsync(e->dState, 0, total, e->stream) != cudaSuccess ||
                        cudaMemsetAsync(e->dCtrl, 0, sizeof(Ctrl) * n, e->stream) != cudaSuccess))
    rc = PMHD_ERR_CUDA;
  // Descriptors.
  for (int k = 0; rc == PMHD_OK && k < n; k++) {
    Member& m = e->hm[k];
    const pmhd_member_desc& d = members[k];
    unsigned char* base = static_cast<unsigned char*>(e->dState) + e->state_off[k];
    m.u = base;
    m.u1 = base + round256((size_t)9 * m.plane * e->elem);
    m.ctrl = e->dCtrl + k;
    set_member_physics(m, d.x_min, d.x_max, d.y_min, d.y_max, d.gamma, common->hlld_tol, common->cfl, common->alpha,
                       common->order == PMHD_ORDER_MUSCL ? 1 : 0, d.bc, common->precision == PMHD_FP32);
    if (!encode_member_tmaps(m, e->elem)) rc = PMHD_ERR_CUDA;
  }
  if (rc == PMHD_OK &&
      cudaMemcpyAsync(e->dMembers, e->hm.data(), sizeof(Member) * n, cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
    rc = PMHD_ERR_CUDA;
  // Work lists: each member's tiles, members in order, per tile height.
  std::vector<int> tiles, tile0;
  for (int t = 0; rc == PMHD_OK && t < kNumTileHeights; t++) {
    tiles.clear();
    tile0.assign(n, 0);
    for (int k = 0; k < n; k++) {
      tile0[k] = (int)tiles.size();
      const long long nt =
          (long long)((members[k].nx + 31) / 32) * ((members[k].ny + kTileHeights[t] - 1) / kTileHeights[t]);
      if ((long long)tiles.size() + nt > (long long)INT_MAX) {
        rc = PMHD_ERR_UNSUPPORTED;
        break;
      }
      tiles.insert(tiles.end(), (size_t)nt, k);
    }
    if (rc != PMHD_OK) break;
    if (cudaMalloc(&e->dTiles[t], sizeof(int) * tiles.size()) != cudaSuccess ||
        cudaMalloc(&e->dTile0[t], sizeof(int) * n) != cudaSuccess) {
      rc = PMHD_ERR_NOMEM;
      break;
    }
    // Stream-ordered copies, finished before the host vectors are reused.
    if (cudaMemcpyAsync(e->dTiles[t], tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, e->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(e->dTile0[t], tile0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
      rc = PMHD_ERR_CUDA;
    Batch& b = e->run.batch[t];
    b.members = e->dMembers;
    b.tile_member = e->dTiles[t];
    b.member_tile0 = e->dTile0[t];
    b.nmembers = n;
    b.ntiles = (int)tiles.size();
  }
  e->run.kt = e->kt;
  e->run.precision = common->precision;
  e->run.hlld = common->solver == PMHD_SOLVER_HLLD ? 1 : 0;
  e->run.stream = e->stream;
  e->run.single = nullptr;
  // Initial states: built on the host, uploaded through the member's U1.
  for (int k = 0; rc == PMHD_OK && k < n; k++) {
    const pmhd_config c = member_config(e, k);
    const pmhd_member_desc& d = members[k];
    const size_t cnt = (size_t)(d.nx + 4) * (d.ny + 4) * 9;
    std::vector<unsigned char> host(cnt * e->elem);
    rc = pmhd_problem_state(&c, d.problem, d.nparams ? d.params : nullptr, d.nparams, host.data());
    if (rc != PMHD_OK) break;
    const Member& m = e->hm[k];
    if (cudaMemcpyAsync(m.u1, host.data(), host.size(), cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
        e->kt->aos_to_soa(common->precision, m.u1, PMHD_LAYOUT_GHOSTED, m.u, m.plane, m.nx, m.ny, m.pitch, d.bc,
                          e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
      rc = PMHD_ERR_CUDA;
  }
  if (rc != PMHD_OK) {
    cudaGetLastError();
    pmhd_ensemble_destroy(e);
    return rc;
  }
  *out = e;
  return PMHD_OK;
}

int pmhd_ensemble_advance(pmhd_ensemble* e, long long max_steps, pmhd_stats* total) {
  if (!e) return PMHD_ERR_ARG;
  const int n = (int)e->desc.size();
  if (e->broken) {
    if (total) {
      std::memset(total, 0, sizeof(*total));
      total->status = PMHD_ERR_CUDA;
    }
    return PMHD_ERR_CUDA;
  }
  PMHD_E(cudaSetDevice(e->cfg.device));
  for (int k = 0; k < n; k++) {
    Ctrl& h = e->hCtrl[k];
    std::memset(&h, 0, sizeof(h));
    h.t[0] = h.t[1] = e->t[k];
    h.step[0] = h.step[1] = e->steps[k];
    h.t_end = time_type(e, e->desc[k].t_end);
    h.step_limit = max_steps < 0 ? LLONG_MAX : e->steps[k] + max_steps;
    h.halted = e->failed[k];  // a failed member stays frozen
    h.bad1 = h.bad2 = BAD_NONE;
  }
  PMHD_E(cudaMemcpyAsync(e->dCtrl, e->hCtrl, sizeof(Ctrl) * n, cudaMemcpyHostToDevice, e->stream));
  PMHD_E(cudaEventRecord(e->ev0, e->stream));
  for (int k = 0; k < n; k++) {
    const Member& m = e->hm[k];
    PMHD_E(e->kt->speed(e->cfg.precision, m.u, m.plane, m.nx, m.ny, m.pitch, m.gamma, m.ctrl, 0, e->stream));
  }
  long long tune_steps = 0, launched = n;  // kernels enqueued: n CFL reductions so far
  if (e->cfg.autotune && !e->tuned && (max_steps < 0 || max_steps >= 32)) {
    // Live steps timed per size class and kernel variant (tune_by_size).
    PMHD_E(tune_by_size(e, &tune_steps, &launched));
    e->tuned = true;
  }
  const int big = e->cfg.steps_per_graph;
  const long long per_step = 2LL * (e->run.parts.empty() ? 1 : (long long)e->run.parts.size());
  // Done when every member has finished or failed, or on a device timeout.
  auto all_done = [n](const Ctrl* cs) {
    for (int k = 0; k < n; k++)
      if (cs[k].err) return true;
    for (int k = 0; k < n; k++)
      if (!failing(cs[k]) && !finished(cs[k])) return false;
    return true;
  };
  if (max_steps >= 0) {
    // Known step budget: replay exactly enough steps, no host round trips.
    long long left = max_steps - tune_steps;
    if (left < 0) left = 0;
    left += left & 1;
    cudaGraphExec_t gb = nullptr, g2 = nullptr;
    if (left >= big && e->run.graph(big, &gb) != 0) return PMHD_ERR_CUDA;
    if (e->run.graph(2, &g2) != 0) return PMHD_ERR_CUDA;
    for (; left >= big; left -= big, launched += per_step * big) PMHD_E(cudaGraphLaunch(gb, e->stream));
    for (; left > 0; left -= 2, launched += 2 * per_step) PMHD_E(cudaGraphLaunch(g2, e->stream));
  } else {
    // Time-limited: replay graphs, polling the control blocks one replay
    // behind so the device never idles waiting for the host.
    cudaGraphExec_t gb = nullptr;
    if (e->run.graph(big, &gb) != 0) return PMHD_ERR_CUDA;
    long long issued = 0;
    auto issue = [&]() -> cudaError_t {
      const int b = (int)(issued & 1);
      cudaError_t err = cudaGraphLaunch(gb, e->stream);
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(e->hPoll + (size_t)b * n, e->dCtrl, sizeof(Ctrl) * n, cudaMemcpyDeviceToHost,
                              e->stream);
      if (err == cudaSuccess) err = cudaEventRecord(e->evPoll[b], e->stream);
      issued++;
      launched += per_step * big;
      return err;
    };
    PMHD_E(issue());
    for (long long k = 0;; k++) {
      PMHD_E(issue());
      PMHD_E(cudaEventSynchronize(e->evPoll[k & 1]));
      if (all_done(e->hPoll + (size_t)(k & 1) * n)) break;
    }
  }
  PMHD_E(cudaEventRecord(e->ev1, e->stream));
  PMHD_E(cudaMemcpyAsync(e->hCtrl, e->dCtrl, sizeof(Ctrl) * n, cudaMemcpyDeviceToHost, e->stream));
  PMHD_E(cudaStreamSynchronize(e->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e->ev0, e->ev1);
  pmhd_stats tot;
  std::memset(&tot, 0, sizeof(tot));
  tot.bad_i = tot.bad_j = -1;
  tot.bad_step = -1;
  const int hlld = e->cfg.solver == PMHD_SOLVER_HLLD;
  int status = PMHD_OK;
  for (int k = 0; k < n; k++) {
    const Ctrl& h = e->hCtrl[k];
    pmhd_stats& st = e->mstats[k];
    const pmhd_member_desc& d = e->desc[k];
    const long long done = h.step[0] - e->steps[k];
    long long stages = 2 * done;
    int mst = PMHD_OK;
    if (h.err) {
      mst = PMHD_ERR_TIMEOUT;
      e->broken = true;
    } else if (!e->failed[k] && (h.bad1 != BAD_NONE || h.bad2 != BAD_NONE)) {
      const int bad = h.bad1 != BAD_NONE ? h.bad1 : h.bad2;
      mst = h.bad1 != BAD_NONE ? PMHD_ERR_STAGE1 : PMHD_ERR_STAGE2;
      stages += h.bad1 != BAD_NONE ? 1 : 2;
      st.bad_i = bad % d.nx;
      st.bad_j = bad / d.nx;
      st.bad_step = h.bad_step;
      e->failed[k] = 1;
    }
    if (hlld) {
      st.x_evals += (unsigned long long)stages * (unsigned long long)(d.nx + 1) * d.ny;
      st.y_evals += (unsigned long long)stages * (unsigned long long)d.nx * (d.ny + 1);
      st.degenerate += h.degenerate;
      st.nonphysical += h.nonphysical;
    }
    st.kernel_launches += h.active_stage_launches + 1;
    if (done > 0 || mst != PMHD_OK) {
      st.ch_last = h.last_ch;
      st.dt_last = h.last_dt;
    }
    e->t[k] = h.t[0];
    e->steps[k] = h.step[0];
    st.t = h.t[0];
    st.steps = h.step[0];
    if (mst != PMHD_OK || !e->failed[k]) st.status = mst;
    st.zone_cycles = (unsigned long long)done * (unsigned long long)d.nx * d.ny;
    st.device_ms = ms;
    st.tile_height = kTileHeights[e->run.parts.empty() ? e->run.choice.ty_idx : e->member_ty[k]];
    if (mst != PMHD_OK && status == PMHD_OK) {
      status = mst;
      tot.bad_i = st.bad_i;
      tot.bad_j = st.bad_j;
      tot.bad_step = st.bad_step;
    }
    tot.steps = st.steps > tot.steps ? st.steps : tot.steps;
    tot.t = st.t > tot.t ? st.t : tot.t;
    tot.zone_cycles += st.zone_cycles;
    tot.x_evals += st.x_evals;
    tot.y_evals += st.y_evals;
    tot.degenerate += st.degenerate;
    tot.nonphysical += st.nonphysical;
  }
  tot.kernel_launches = (unsigned long long)launched;
  tot.status = status;
  tot.device_ms = ms;
  {
    // The launch plan's largest part (by tiles) stands for the ensemble's
    // tile height and CTA count; each member reports its own tile height.
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->cfg.device);
    std::vector<LaunchPart> plan = e->run.parts;
    if (plan.empty()) {
      LaunchPart one;
      one.ty_idx = e->run.choice.ty_idx;
      one.grid = e->run.choice.grid;
      one.batch = e->run.batch[one.ty_idx];
      plan.push_back(one);
    }
    size_t top = 0;
    for (size_t q = 1; q < plan.size(); q++)
      if (plan[q].batch.ntiles > plan[top].batch.ntiles) top = q;
    const int def = sms * e->kt->ctas_per_sm(e->cfg.precision, e->run.hlld, plan[top].ty_idx, 1);
    const int g = plan[top].grid > 0 ? plan[top].grid : def;
    const int nt = plan[top].batch.ntiles;
    tot.tile_height = kTileHeights[plan[top].ty_idx];
    tot.ctas = g < nt ? g : nt;
  }
  for (int k = 0; k < n; k++) e->mstats[k].ctas = tot.ctas;
  if (total) *total = tot;
  return status;
}

int pmhd_ensemble_member_stats(const pmhd_ensemble* e, int k, pmhd_stats* st) {
  if (!e || !st || k < 0 || k >= (int)e->desc.size()) return PMHD_ERR_ARG;
  *st = e->mstats[k];
  return PMHD_OK;
}

int pmhd_ensemble_get_state(pmhd_ensemble* e, int k, void* host, int layout) {
  if (!e || !host || k < 0 || k >= (int)e->desc.size()) return PMHD_ERR_ARG;
  if (layout != PMHD_LAYOUT_INTERIOR && layout != PMHD_LAYOUT_GHOSTED) return PMHD_ERR_ARG;
  PMHD_E(cudaSetDevice(e->cfg.device));
  const Member& m = e->hm[k];
  const size_t cnt = layout == PMHD_LAYOUT_INTERIOR ? (size_t)m.nx * m.ny * 9 : (size_t)(m.nx + 4) * (m.ny + 4) * 9;
  PMHD_E(e->kt->soa_to_aos(e->cfg.precision, m.u, m.plane, m.nx, m.ny, m.pitch, layout, m.u1, e->stream));
  PMHD_E(cudaMemcpyAsync(host, m.u1, cnt * e->elem, cudaMemcpyDeviceToHost, e->stream));
  PMHD_E(cudaStreamSynchronize(e->stream));
  return PMHD_OK;
}

}  // extern "C"
