// member_setup.cpp -- host helpers shared by the solver front ends: TMA
// descriptors and time-type constants of one batch member.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "kernel_api.h"

namespace pmhd {

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

}  // namespace

bool encode_member_tmaps(Member& m, size_t elem) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  // Planes of (ny + 4) rows x pitch; the box is a tile with its 2-cell halo
  // and all nine variables.  x (the innermost coordinate) is always a
  // multiple of 32 elements, so every copy starts 16-byte aligned.
  const cuuint64_t dims[3] = {(cuuint64_t)m.nx + 4, (cuuint64_t)m.ny + 4, 9};
  const cuuint64_t strides[2] = {(cuuint64_t)m.pitch * elem, (cuuint64_t)m.plane * elem};
  const cuuint32_t estr[3] = {1, 1, 1};
  void* bufs[2] = {m.u, m.u1};
  for (int t = 0; t < kNumTileHeights; t++) {
    const cuuint32_t box[3] = {32 + 4, (cuuint32_t)kTileHeights[t] + 4, 9};
    for (int k = 0; k < 2; k++) {
      CUresult r = enc(&m.tm[t][k], elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                       bufs[k], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return false;
    }
  }
  return true;
}

void set_member_physics(Member& m, double x_min, double x_max, double y_min, double y_max, double gamma, double tol,
                        double cfl, double alpha, int muscl, const int bc[4], bool fp32) {
  if (fp32) {
    m.dx = (double)(((float)x_max - (float)x_min) / (float)m.nx);
    m.dy = (double)(((float)y_max - (float)y_min) / (float)m.ny);
    m.cfl = (double)(float)cfl;
    m.alpha = (double)(float)alpha;
    m.inv_dx = (double)(1.0f / (float)m.dx);
    m.inv_dy = (double)(1.0f / (float)m.dy);
  } else {
    m.dx = (x_max - x_min) / (double)m.nx;
    m.dy = (y_max - y_min) / (double)m.ny;
    m.cfl = cfl;
    m.alpha = alpha;
    m.inv_dx = 1.0 / m.dx;
    m.inv_dy = 1.0 / m.dy;
  }
  m.gamma = gamma;
  m.tol = tol;
  m.muscl = muscl;
  for (int k = 0; k < 4; k++) m.bc[k] = bc[k];
}

}  // namespace pmhd
