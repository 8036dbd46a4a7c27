// kernels.cu -- instantiates the pmhd kernels for every precision policy and
// tile height and exposes them through a KernelTable.  Built twice by the
// Makefile:
//   -DPMHD_KNS=exact -fmad=false                  -> kernel_table_exact()
//   -DPMHD_KNS=fast  -fmad=true -prec-div=false -prec-sqrt=false
//                                                 -> kernel_table_fast()
#include <mutex>

#include "stage_kernels.cuh"

namespace pmhd {
namespace PMHD_KNS {

#include "hancock_kernel.cuh"  // no includes of its own; lives in this namespace

template <class Pol, int STAGE, bool HLLD, int TY, bool BATCHED>
static cudaError_t set_smem_attr() {
  return cudaFuncSetAttribute(stage_kernel<Pol, STAGE, HLLD, TY, BATCHED>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Smem<Pol, TY>::total);
}

template <class Pol, int TY, bool BATCHED>
static cudaError_t init_pol_ty_b() {
  cudaError_t e;
  if ((e = set_smem_attr<Pol, 1, true, TY, BATCHED>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<Pol, 2, true, TY, BATCHED>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<Pol, 1, false, TY, BATCHED>()) != cudaSuccess) return e;
  return set_smem_attr<Pol, 2, false, TY, BATCHED>();
}

template <class Pol, int TY>
static cudaError_t init_pol_ty() {
  cudaError_t e = init_pol_ty_b<Pol, TY, false>();
  return e != cudaSuccess ? e : init_pol_ty_b<Pol, TY, true>();
}

template <class Pol>
static cudaError_t init_pol() {
  cudaError_t e;
  if ((e = init_pol_ty<Pol, kTileHeights[0]>()) != cudaSuccess) return e;
  return init_pol_ty<Pol, kTileHeights[1]>();
}

template <class Pol, bool HLLD>
static cudaError_t init_hancock() {
  const int smem = (int)sizeof(HancockTileOf<Pol>);
  cudaError_t e = cudaFuncSetAttribute(hancock_kernel<Pol, HLLD>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if constexpr (HancockPersistent<Pol>::on) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(hancock_persistent_kernel<Pol, HLLD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem);
  }
  return e;
}

static cudaError_t init() {
  cudaError_t e;
  if ((e = init_pol<PolF64>()) != cudaSuccess) return e;
  if ((e = init_pol<PolF32>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolF64, true>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolF64, false>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolF32, true>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolF32, false>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolMixed, true>()) != cudaSuccess) return e;
  if ((e = init_hancock<PolMixed, false>()) != cudaSuccess) return e;
  return init_pol<PolMixed>();
}

static int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

template <class Pol, bool HLLD, int TY, bool BATCHED>
static int occupancy() {
  static int per_sm = -1;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (per_sm < 0) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage_kernel<Pol, 1, HLLD, TY, BATCHED>, Geo<TY>::NT,
                                                  Smem<Pol, TY>::total);
    per_sm = nb > 0 ? nb : 1;
  }
  return per_sm;
}

template <class Pol, bool HLLD, int TY, bool BATCHED>
static void launch_one(int stage, const Batch& b, const Member& m0, int parity, int grid, cudaStream_t s) {
  const size_t smem = Smem<Pol, TY>::total;
  if (stage == 1)
    stage_kernel<Pol, 1, HLLD, TY, BATCHED><<<grid, Geo<TY>::NT, smem, s>>>(m0, b, parity);
  else
    stage_kernel<Pol, 2, HLLD, TY, BATCHED><<<grid, Geo<TY>::NT, smem, s>>>(m0, b, parity);
}

template <class Pol, int TY>
static int occ_pol_ty(int hlld, bool batched) {
  if (batched) return hlld ? occupancy<Pol, true, TY, true>() : occupancy<Pol, false, TY, true>();
  return hlld ? occupancy<Pol, true, TY, false>() : occupancy<Pol, false, TY, false>();
}

template <class Pol, int TY>
static cudaError_t launch_stage_pol(int hlld, int stage, const Batch& b, const Member* single, int parity, int grid,
                                    cudaStream_t s) {
  if (b.ntiles <= 0) return cudaSuccess;
  const bool batched = single == nullptr;
  if (grid <= 0) grid = sm_count() * occ_pol_ty<Pol, TY>(hlld, batched);
  const int units = batched ? (b.ntiles + kBatchRun - 1) / kBatchRun : b.ntiles;  // tiles or runs of tiles
  if (grid > units) grid = units;
  static const Member empty = {};
  const Member& m0 = batched ? empty : *single;
  if (hlld) {
    if (batched)
      launch_one<Pol, true, TY, true>(stage, b, m0, parity, grid, s);
    else
      launch_one<Pol, true, TY, false>(stage, b, m0, parity, grid, s);
  } else {
    if (batched)
      launch_one<Pol, false, TY, true>(stage, b, m0, parity, grid, s);
    else
      launch_one<Pol, false, TY, false>(stage, b, m0, parity, grid, s);
  }
  return cudaGetLastError();
}

template <class Pol>
static cudaError_t launch_stage_ty(int hlld, int stage, int ty_idx, const Batch& b, const Member* single, int parity,
                                   int grid, cudaStream_t s) {
  return ty_idx == 0 ? launch_stage_pol<Pol, kTileHeights[0]>(hlld, stage, b, single, parity, grid, s)
                     : launch_stage_pol<Pol, kTileHeights[1]>(hlld, stage, b, single, parity, grid, s);
}

static cudaError_t launch_stage(int precision, int hlld, int stage, int ty_idx, const Batch& b, const Member* single,
                                int parity, int grid, cudaStream_t s) {
  if (ty_idx < 0 || ty_idx >= kNumTileHeights) return cudaErrorInvalidValue;
  switch (precision) {
    case PREC_FP64: return launch_stage_ty<PolF64>(hlld, stage, ty_idx, b, single, parity, grid, s);
    case PREC_FP32: return launch_stage_ty<PolF32>(hlld, stage, ty_idx, b, single, parity, grid, s);
    case PREC_MIXED: return launch_stage_ty<PolMixed>(hlld, stage, ty_idx, b, single, parity, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class Pol>
static int occ_pol(int hlld, int ty_idx, bool batched) {
  return ty_idx == 0 ? occ_pol_ty<Pol, kTileHeights[0]>(hlld, batched)
                     : occ_pol_ty<Pol, kTileHeights[1]>(hlld, batched);
}

static int ctas_per_sm(int precision, int hlld, int ty_idx, int batched) {
  switch (precision) {
    case PREC_FP64: return occ_pol<PolF64>(hlld, ty_idx, batched != 0);
    case PREC_FP32: return occ_pol<PolF32>(hlld, ty_idx, batched != 0);
    default: return occ_pol<PolMixed>(hlld, ty_idx, batched != 0);
  }
}

static size_t stage_smem(int precision, int ty_idx) {
  const bool t8 = ty_idx == 0;
  switch (precision) {
    case PREC_FP64: return t8 ? Smem<PolF64, kTileHeights[0]>::total : Smem<PolF64, kTileHeights[1]>::total;
    case PREC_FP32: return t8 ? Smem<PolF32, kTileHeights[0]>::total : Smem<PolF32, kTileHeights[1]>::total;
    default: return t8 ? Smem<PolMixed, kTileHeights[0]>::total : Smem<PolMixed, kTileHeights[1]>::total;
  }
}

static int grid_for(long long n) {
  long long b = (n + NTA - 1) / NTA;
  if (b > 148 * 64) b = 148 * 64;
  return (int)(b < 1 ? 1 : b);
}

static cudaError_t launch_speed(int precision, const void* u, long long plane, int nx, int ny, int pitch,
                                double gamma, Ctrl* ctrl, int slot, cudaStream_t s) {
  const int g = grid_for((long long)nx * ny);
  switch (precision) {
    case PREC_FP64:
      speed_kernel<PolF64><<<g, NTA, 0, s>>>(static_cast<const double*>(u), plane, nx, ny, pitch, gamma, ctrl, slot);
      break;
    case PREC_FP32:
      speed_kernel<PolF32><<<g, NTA, 0, s>>>(static_cast<const float*>(u), plane, nx, ny, pitch, gamma, ctrl, slot);
      break;
    case PREC_MIXED:
      speed_kernel<PolMixed><<<g, NTA, 0, s>>>(static_cast<const double*>(u), plane, nx, ny, pitch, gamma, ctrl,
                                              slot);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

static cudaError_t launch_aos_to_soa(int precision, const void* aos, int layout, void* u, long long plane, int nx,
                                     int ny, int pitch, const int bc[4], cudaStream_t s) {
  const int g = grid_for((long long)nx * ny);
  if (precision == PREC_FP32)
    aos_to_soa_kernel<float><<<g, NTA, 0, s>>>(static_cast<const float*>(aos), layout, static_cast<float*>(u), plane,
                                               nx, ny, pitch, bc[0], bc[1], bc[2], bc[3]);
  else
    aos_to_soa_kernel<double><<<g, NTA, 0, s>>>(static_cast<const double*>(aos), layout, static_cast<double*>(u),
                                                plane, nx, ny, pitch, bc[0], bc[1], bc[2], bc[3]);
  return cudaGetLastError();
}

static cudaError_t launch_soa_to_aos(int precision, const void* u, long long plane, int nx, int ny, int pitch,
                                     int layout, void* aos, cudaStream_t s) {
  const long long n = layout == 0 ? (long long)nx * ny : (long long)(nx + 4) * (ny + 4);
  const int g = grid_for(n);
  if (precision == PREC_FP32)
    soa_to_aos_kernel<float><<<g, NTA, 0, s>>>(static_cast<const float*>(u), plane, nx, ny, pitch, layout,
                                               static_cast<float*>(aos));
  else
    soa_to_aos_kernel<double><<<g, NTA, 0, s>>>(static_cast<const double*>(u), plane, nx, ny, pitch, layout,
                                                static_cast<double*>(aos));
  return cudaGetLastError();
}

template <class Pol>
static cudaError_t hancock_pol(int hlld, int part, const Member& m, int parity, cudaStream_t s) {
  if (part == 0) {
    hancock_begin_kernel<Pol><<<1, 32, 0, s>>>(m, parity);
    return cudaGetLastError();
  }
  constexpr int TYH = HancockTileOf<Pol>::TYH;
  const int ntiles = ((m.nx + TX - 1) / TX) * ((m.ny + TYH - 1) / TYH);
  const size_t smem = sizeof(HancockTileOf<Pol>);
  if constexpr (HancockPersistent<Pol>::on) {
    // Persistent: the SMs x the resident CTAs, at most one per tile.
    static int per_sm = -1;
    if (per_sm < 0) {
      int nb = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, hancock_persistent_kernel<Pol, true>, 256, smem);
      per_sm = nb > 0 ? nb : 1;
    }
    int grid = sm_count() * per_sm;
    if (grid > ntiles) grid = ntiles;
    if (hlld)
      hancock_persistent_kernel<Pol, true><<<grid, 256, smem, s>>>(m, parity);
    else
      hancock_persistent_kernel<Pol, false><<<grid, 256, smem, s>>>(m, parity);
  } else {
    if (hlld)
      hancock_kernel<Pol, true><<<ntiles, 256, smem, s>>>(m, parity);
    else
      hancock_kernel<Pol, false><<<ntiles, 256, smem, s>>>(m, parity);
  }
  return cudaGetLastError();
}

static cudaError_t launch_hancock(int precision, int hlld, int part, const Member& m, int parity, cudaStream_t s) {
  switch (precision) {
    case PREC_FP64: return hancock_pol<PolF64>(hlld, part, m, parity, s);
    case PREC_FP32: return hancock_pol<PolF32>(hlld, part, m, parity, s);
    case PREC_MIXED: return hancock_pol<PolMixed>(hlld, part, m, parity, s);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace PMHD_KNS

#define PMHD_STR2(x) #x
#define PMHD_STR(x) PMHD_STR2(x)
#define PMHD_TABLE_FN2(n) kernel_table_##n
#define PMHD_TABLE_FN(n) PMHD_TABLE_FN2(n)

const KernelTable& PMHD_TABLE_FN(PMHD_KNS)() {
  static const KernelTable t = {PMHD_STR(PMHD_KNS),          PMHD_KNS::init,
                                PMHD_KNS::launch_stage,      PMHD_KNS::ctas_per_sm,
                                PMHD_KNS::launch_speed,      PMHD_KNS::launch_aos_to_soa,
                                PMHD_KNS::launch_soa_to_aos, PMHD_KNS::stage_smem,
                                PMHD_KNS::launch_hancock};
  return t;
}

}  // namespace pmhd
