// noalloc.cu -- pmhd_advance_noalloc: the time loop without any device
// allocation.
//
// Who needs it: code that must not allocate GPU memory while it runs --
// for example a caller that has carved all device memory into its own pool
// up front (a serving process or a coupled multiphysics code with a fixed
// memory plan), a caller running under an allocator hook that forbids
// cudaMalloc after start-up, or code that must not risk an allocation
// failure half way through a run.  The regular path (pmhd_create) allocates
// two state buffers and a control block per handle; this entry point
// instead works on the caller's own device buffers and keeps its working
// state -- the stage-1 state, the step state in the solver's padded planar
// layout and the control block -- in one fixed array compiled into the
// library (`g_noalloc_scratch`, 48 MiB, see PMHD_NOALLOC_SCRATCH_BYTES).
//
// Properties (also stated in include/pmhd.h):
//   * The array is a static __device__ object: every GPU on which this entry
//     point runs holds it until the process exits.  The CUDA runtime places
//     it in device memory when it loads this library's device code on that
//     GPU; with lazy module loading (the CUDA 12 default) that is the first
//     call's cudaGetSymbolAddress and first kernel launches, so the FIRST
//     call on a device allocates (the array and the kernels' code) and must
//     come before the caller gives the rest of the device memory to its own
//     pool.  Later calls allocate nothing.
//   * Grids are limited to what fits in it: kHeadBytes (2048: the control
//     block and the grid descriptor) plus two states of 9 x (ny + 4) x
//     round_up(nx + 4, 16) elements (8 bytes in fp64 / mixed, 4 in fp32),
//     each rounded up to 256 bytes.  Up to 586^2 cells in fp64 / mixed and
//     828^2 in fp32.  Larger grids are rejected with PMHD_ERR_UNSUPPORTED
//     before anything is launched.
//   * Every call shares the array and it keeps the last call's contents;
//     each call rewrites the control block and the whole state before using
//     them.  Calls that overlap on the GPU (from several host threads or
//     streams at once) race on the array and give wrong results: serialise
//     them.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and sets the kernels' shared-memory limits,
//     with that device current; make that first call before any stream
//     capture.
//   * It calls no cudaMalloc / cudaFree / graph instantiation and no library
//     routine that allocates: kernels are launched directly on the caller's
//     stream and the control block is read back into a host stack variable.
#include <cuda.h>
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "kernel_api.h"
#include "pmhd.h"

using namespace pmhd;

namespace {

constexpr size_t kScratchBytes = (size_t)PMHD_NOALLOC_SCRATCH_BYTES;
constexpr size_t kCtrlBytes = 256;    // control block slot
constexpr size_t kMemberOff = 256;    // grid descriptor (TMA maps, pointers)
constexpr size_t kHeadBytes = 2048;   // control block + descriptor
static_assert(sizeof(Ctrl) <= kCtrlBytes, "control block must fit its slot");
static_assert(kMemberOff + sizeof(Member) <= kHeadBytes, "grid descriptor must fit its slot");

// The fixed working memory of pmhd_advance_noalloc (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
  bool done = false;
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch
};
std::mutex g_mu;
DeviceSetup g_setup[64];

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// Same validation as pmhd_create.
bool config_ok(const pmhd_config* c) {
  if (!c || c->nx < 4 || c->ny < 4 || (long long)c->nx * c->ny > (long long)INT_MAX) return false;
  if (!(c->x_max > c->x_min) || !(c->y_max > c->y_min)) return false;
  if (!(c->cfl > 0.0) || !(c->cfl < 1.0) || !(c->alpha > 0.0) || !(c->gamma > 1.0)) return false;
  if (!(c->hlld_tol >= 0.0)) return false;
  if (c->order != PMHD_ORDER_FIRST && c->order != PMHD_ORDER_MUSCL) return false;
  if (c->solver != PMHD_SOLVER_HLL && c->solver != PMHD_SOLVER_HLLD) return false;
  if (c->precision < PMHD_FP64 || c->precision > PMHD_MIXED) return false;
  for (int k = 0; k < 4; k++)
    if (c->bc[k] < PMHD_BC_PERIODIC || c->bc[k] > PMHD_BC_TRANSMISSIVE) return false;
  if ((c->bc[0] == PMHD_BC_PERIODIC) != (c->bc[1] == PMHD_BC_PERIODIC)) return false;
  if ((c->bc[2] == PMHD_BC_PERIODIC) != (c->bc[3] == PMHD_BC_PERIODIC)) return false;
  return true;
}

// Once per device, with that device current: the array's device address
// and the kernels' shared-memory attributes.
int setup_device(int dev, unsigned char** base) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceSetup& d = g_setup[dev & 63];
  if (!d.done) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return PMHD_ERR_CUDA;
    if (kernel_table_exact().init() != cudaSuccess || kernel_table_fast().init() != cudaSuccess)
      return PMHD_ERR_CUDA;
    d.base = static_cast<unsigned char*>(p);
    d.done = true;
  }
  *base = d.base;
  return PMHD_OK;
}

}  // namespace

namespace {
size_t scratch_needed(const pmhd_config* cfg) {
  const size_t elem = cfg->precision == PMHD_FP32 ? 4 : 8;
  const size_t pitch = ((size_t)(cfg->nx + 4) + 15) / 16 * 16;
  const size_t plane = pitch * (size_t)(cfg->ny + 4);
  return kHeadBytes + 2 * round256(9 * plane * elem);
}
}  // namespace

extern "C" int pmhd_advance_noalloc(const pmhd_config* cfg, const void* d_in, void* d_out, double t0,
                                    long long step0, double t_end, long long max_steps, void* stream,
                                    pmhd_stats* stats) {
  if (!config_ok(cfg) || !d_in || !d_out || std::isnan(t_end) || !std::isfinite(t0) || step0 < 0)
    return PMHD_ERR_ARG;
  if (scratch_needed(cfg) > kScratchBytes) return PMHD_ERR_UNSUPPORTED;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess) return PMHD_ERR_NODEVICE;
  if (prop.major != 10 || prop.minor != 0) return PMHD_ERR_NODEVICE;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return PMHD_ERR_CUDA;
  unsigned char* base = nullptr;
  int rc = setup_device(cfg->device, &base);
  if (rc != PMHD_OK) return rc;

  const bool f32 = cfg->precision == PMHD_FP32;
  const size_t elem = f32 ? 4 : 8;
  const int nx = cfg->nx, ny = cfg->ny;
  const int pitch = ((nx + 4) + 15) / 16 * 16;
  const long long plane = (long long)pitch * (ny + 4);
  Ctrl* dctrl = reinterpret_cast<Ctrl*>(base);
  Member* dmember = reinterpret_cast<Member*>(base + kMemberOff);
  void* dU = base + kHeadBytes;
  void* dU1 = base + kHeadBytes + round256(9 * (size_t)plane * elem);
  const KernelTable& kt = cfg->exact ? kernel_table_exact() : kernel_table_fast();
  Member hm;
  std::memset(&hm, 0, sizeof(hm));
  hm.u = dU;
  hm.u1 = dU1;
  hm.ctrl = dctrl;
  hm.plane = plane;
  hm.nx = nx;
  hm.ny = ny;
  hm.pitch = pitch;
  set_member_physics(hm, cfg->x_min, cfg->x_max, cfg->y_min, cfg->y_max, cfg->gamma, cfg->hlld_tol, cfg->cfl,
                     cfg->alpha, cfg->order == PMHD_ORDER_MUSCL ? 1 : 0, cfg->bc, f32);
  if (!encode_member_tmaps(hm, elem)) return PMHD_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Batch batch;
  batch.members = dmember;
  batch.tile_member = nullptr;
  batch.member_tile0 = nullptr;
  batch.nmembers = 1;
  batch.ntiles = ((nx + 31) / 32) * ((ny + kTileHeights[0] - 1) / kTileHeights[0]);

  // Values the reference holds in its Real type.
  auto tt = [&](double v) { return f32 ? (double)(float)v : v; };

  // Control block: everything that must start at zero is rewritten here.
  Ctrl h;
  std::memset(&h, 0, sizeof(h));
  h.t[0] = h.t[1] = tt(t0);
  h.step[0] = h.step[1] = step0;
  h.t_end = tt(t_end);
  h.step_limit = max_steps < 0 ? LLONG_MAX : step0 + max_steps;
  h.bad1 = h.bad2 = BAD_NONE;
#define PMHD_NA(call)                               \
  do {                                              \
    if ((call) != cudaSuccess) return PMHD_ERR_CUDA; \
  } while (0)
  PMHD_NA(cudaMemcpyAsync(dctrl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  PMHD_NA(cudaMemcpyAsync(dmember, &hm, sizeof(hm), cudaMemcpyHostToDevice, s));
  PMHD_NA(kt.aos_to_soa(cfg->precision, d_in, PMHD_LAYOUT_INTERIOR, dU, plane, nx, ny, pitch, cfg->bc, s));
  PMHD_NA(kt.speed(cfg->precision, dU, plane, nx, ny, pitch, cfg->gamma, dctrl, 0, s));

  const int hlld = cfg->solver == PMHD_SOLVER_HLLD ? 1 : 0;
  // Steps are launched in pairs (parity 0 then 1) so the final values land
  // in control slot 0; a step past the stop condition is a no-op.
  auto launch_pairs = [&](long long pairs) -> int {
    for (long long q = 0; q < pairs; q++)
      for (int par = 0; par < 2; par++) {
        if (kt.stage(cfg->precision, hlld, 1, 0, batch, &hm, par, 0, s) != cudaSuccess) return PMHD_ERR_CUDA;
        if (kt.stage(cfg->precision, hlld, 2, 0, batch, &hm, par, 0, s) != cudaSuccess) return PMHD_ERR_CUDA;
      }
    return PMHD_OK;
  };
  // Chunks of 16 step pairs, each followed by a look at the control block,
  // so a large step cap used only as a safety bound queues no more launches
  // than the run needs (steps past the stop condition are no-ops).
  Ctrl r;
  long long pairs_left = max_steps >= 0 ? (max_steps + 1) / 2 : LLONG_MAX;
  std::memcpy(&r, &h, sizeof(r));
  while (pairs_left > 0) {
    const long long chunk = pairs_left < 16 ? pairs_left : 16;
    if ((rc = launch_pairs(chunk)) != PMHD_OK) return rc;
    pairs_left -= chunk;
    PMHD_NA(cudaMemcpyAsync(&r, dctrl, sizeof(r), cudaMemcpyDeviceToHost, s));
    PMHD_NA(cudaStreamSynchronize(s));
    if (r.halted || r.err || r.bad1 != BAD_NONE || r.bad2 != BAD_NONE || !(r.t[0] < r.t_end) ||
        !(r.step[0] < r.step_limit))
      break;
  }
  PMHD_NA(kt.soa_to_aos(cfg->precision, dU, plane, nx, ny, pitch, PMHD_LAYOUT_INTERIOR, d_out, s));
  PMHD_NA(cudaStreamSynchronize(s));
#undef PMHD_NA

  int status = PMHD_OK;
  long long stages = 2 * (r.step[0] - step0);
  pmhd_stats out;
  std::memset(&out, 0, sizeof(out));
  out.bad_i = out.bad_j = -1;
  out.bad_step = -1;
  if (r.err) {
    status = PMHD_ERR_TIMEOUT;
  } else if (r.bad1 != BAD_NONE || r.bad2 != BAD_NONE) {
    const int bad = r.bad1 != BAD_NONE ? r.bad1 : r.bad2;
    status = r.bad1 != BAD_NONE ? PMHD_ERR_STAGE1 : PMHD_ERR_STAGE2;
    stages += r.bad1 != BAD_NONE ? 1 : 2;
    out.bad_i = bad % nx;
    out.bad_j = bad / nx;
    out.bad_step = r.bad_step;
  }
  out.steps = r.step[0];
  out.t = r.t[0];
  out.ch_last = r.last_ch;
  out.dt_last = r.last_dt;
  if (hlld) {
    out.x_evals = (unsigned long long)stages * (unsigned long long)(nx + 1) * ny;
    out.y_evals = (unsigned long long)stages * (unsigned long long)nx * (ny + 1);
    out.degenerate = r.degenerate;
    out.nonphysical = r.nonphysical;
  }
  out.kernel_launches = r.active_stage_launches + 1;
  out.zone_cycles = (unsigned long long)(r.step[0] - step0) * (unsigned long long)nx * ny;
  out.status = status;
  if (stats) *stats = out;
  return status;
}
