// kernels.cu -- instantiates the pmhd kernels for every precision policy and
// exposes them through a KernelTable.  Built twice by the Makefile:
//   -DPMHD_KNS=exact -fmad=false                  -> kernel_table_exact()
//   -DPMHD_KNS=fast  -fmad=true -prec-div=false -prec-sqrt=false
//                                                 -> kernel_table_fast()
#include "stage_kernels.cuh"

namespace pmhd {
namespace PMHD_KNS {

template <class Pol, int STAGE, bool HLLD>
static cudaError_t set_smem_attr() {
  return cudaFuncSetAttribute(stage_kernel<Pol, STAGE, HLLD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Smem<Pol>::total);
}

template <class Pol>
static cudaError_t init_pol() {
  cudaError_t e;
  if ((e = set_smem_attr<Pol, 1, true>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<Pol, 2, true>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<Pol, 1, false>()) != cudaSuccess) return e;
  return set_smem_attr<Pol, 2, false>();
}

static cudaError_t init() {
  cudaError_t e;
  if ((e = init_pol<PolF64>()) != cudaSuccess) return e;
  if ((e = init_pol<PolF32>()) != cudaSuccess) return e;
  return init_pol<PolMixed>();
}

// Persistent grid: every SM holds as many stage CTAs as fit, capped by the
// number of tiles.
template <class Pol, int STAGE, bool HLLD>
static int persistent_grid(int ntiles) {
  static int per_sm = -1, sms = 0;
  if (per_sm < 0) {
    int dev = 0, nb = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage_kernel<Pol, STAGE, HLLD>, NT, Smem<Pol>::total);
    per_sm = nb > 0 ? nb : 1;
  }
  const int g = sms * per_sm;
  return g < ntiles ? g : ntiles;
}

template <class Pol>
static cudaError_t launch_stage_pol(int hlld, int stage, const void* tmap_in, const StageArgs& a, cudaStream_t s) {
  const int ntiles = ((a.nx + TX - 1) / TX) * ((a.ny + TY - 1) / TY);
  const size_t smem = Smem<Pol>::total;
  const CUtensorMap& tm = *static_cast<const CUtensorMap*>(tmap_in);
  if (hlld) {
    if (stage == 1)
      stage_kernel<Pol, 1, true><<<persistent_grid<Pol, 1, true>(ntiles), NT, smem, s>>>(tm, a);
    else
      stage_kernel<Pol, 2, true><<<persistent_grid<Pol, 2, true>(ntiles), NT, smem, s>>>(tm, a);
  } else {
    if (stage == 1)
      stage_kernel<Pol, 1, false><<<persistent_grid<Pol, 1, false>(ntiles), NT, smem, s>>>(tm, a);
    else
      stage_kernel<Pol, 2, false><<<persistent_grid<Pol, 2, false>(ntiles), NT, smem, s>>>(tm, a);
  }
  return cudaGetLastError();
}

static cudaError_t launch_stage(int precision, int hlld, int stage, const void* tmap_in, const StageArgs& a,
                                cudaStream_t s) {
  switch (precision) {
    case PREC_FP64: return launch_stage_pol<PolF64>(hlld, stage, tmap_in, a, s);
    case PREC_FP32: return launch_stage_pol<PolF32>(hlld, stage, tmap_in, a, s);
    case PREC_MIXED: return launch_stage_pol<PolMixed>(hlld, stage, tmap_in, a, s);
    default: return cudaErrorInvalidValue;
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

static void tile(int precision, int* tx, int* ty, size_t* smem) {
  *tx = TX;
  *ty = TY;
  *smem = precision == PREC_FP64 ? Smem<PolF64>::total
                                 : (precision == PREC_FP32 ? Smem<PolF32>::total : Smem<PolMixed>::total);
}

}  // namespace PMHD_KNS

#define PMHD_STR2(x) #x
#define PMHD_STR(x) PMHD_STR2(x)
#define PMHD_TABLE_FN2(n) kernel_table_##n
#define PMHD_TABLE_FN(n) PMHD_TABLE_FN2(n)

const KernelTable& PMHD_TABLE_FN(PMHD_KNS)() {
  static const KernelTable t = {PMHD_STR(PMHD_KNS),        PMHD_KNS::init,         PMHD_KNS::launch_stage,
                                PMHD_KNS::launch_speed,    PMHD_KNS::launch_aos_to_soa, PMHD_KNS::launch_soa_to_aos,
                                PMHD_KNS::tile};
  return t;
}

}  // namespace pmhd
