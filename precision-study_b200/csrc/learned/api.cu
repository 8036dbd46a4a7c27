// api.cu -- C ABI of the learned correction's building blocks
// (pmhd_conv3x3, pmhd_conv3x3_wgrad, pmhd_learned_loss_grad; declared in
// include/pmhd.h).
#include <cuda_runtime.h>

#include <cstdint>

#include "learned/conv.h"
#include "learned/net.h"
#include "pmhd.h"

namespace {

__device__ int g_conv_err;  // set by a kernel whose bounded wait expired

// Device address of the error word; the first call on a device also sets the
// kernels' shared-memory limits there.
int* error_word() {
  static int prepared_dev = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  if (dev != prepared_dev) {
    if (pmhd::learned::conv_prepare() != cudaSuccess) return nullptr;
    prepared_dev = dev;
  }
  int* p = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_conv_err) != cudaSuccess) return nullptr;
  return p;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int finish(cudaError_t e, int* err, cudaStream_t s) {
  if (e == cudaErrorNotSupported) return PMHD_ERR_UNSUPPORTED;
  if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PMHD_ERR_CUDA;
  }
  int h = 0;
  if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PMHD_ERR_CUDA;
  return h ? PMHD_ERR_TIMEOUT : PMHD_OK;
}

}  // namespace

extern "C" {

int pmhd_conv3x3(int mode, const void* x, int batch, int h, int w, int c_in, const void* weight, const float* bias,
                 int c_out, const void* z_prev, void* out0, void* out1, void* stream) {
  if (batch < 1 || h < 1 || w < 1 || (long long)batch * h * w > (1LL << 31)) return PMHD_ERR_ARG;
  if (!x || !weight || !out0 || !aligned16(x) || !aligned16(weight) || !aligned16(out0)) return PMHD_ERR_ARG;
  if (mode == PMHD_CONV_GELU && (!bias || !out1 || !aligned16(out1))) return PMHD_ERR_ARG;
  if (mode == PMHD_CONV_LINEAR && !bias) return PMHD_ERR_ARG;
  if (mode == PMHD_CONV_DGELU && (!z_prev || !aligned16(z_prev))) return PMHD_ERR_ARG;
  if (mode < PMHD_CONV_GELU || mode > PMHD_CONV_DGELU) return PMHD_ERR_ARG;
  int* err = error_word();
  if (!err) return PMHD_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return PMHD_ERR_CUDA;
  const cudaError_t e = pmhd::learned::conv3x3(mode, static_cast<const __nv_bfloat16*>(x), batch, h, w, c_in,
                                               static_cast<const __nv_bfloat16*>(weight), bias, c_out,
                                               static_cast<const __nv_bfloat16*>(z_prev), out0, out1, err, s);
  return finish(e, err, s);
}

int pmhd_conv3x3_wgrad(const void* x, const void* dz, int batch, int h, int w, int c_in, int c_out, float* dweight,
                       float* dbias, void* stream) {
  if (batch < 1 || h < 1 || w < 1 || (long long)batch * h * w > (1LL << 31)) return PMHD_ERR_ARG;
  if (!x || !dz || !dweight || !aligned16(x) || !aligned16(dz)) return PMHD_ERR_ARG;
  int* err = error_word();
  if (!err) return PMHD_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return PMHD_ERR_CUDA;
  const cudaError_t e = pmhd::learned::conv3x3_wgrad(static_cast<const __nv_bfloat16*>(x),
                                                     static_cast<const __nv_bfloat16*>(dz), batch, h, w, c_in, c_out,
                                                     dweight, dbias, err, s);
  return finish(e, err, s);
}

int pmhd_learned_loss_grad(const float* out, const float* tgt, int batch, int h, int w, float cx, float cy, void* dz,
                           double* loss, void* stream) {
  if (batch < 1 || h < 1 || w < 1 || (long long)batch * h * w > (1LL << 31)) return PMHD_ERR_ARG;
  if (!out || !tgt || !dz || !loss || !aligned16(dz)) return PMHD_ERR_ARG;
  using namespace pmhd::learned;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Norm hn{};
  hn.cx = cx;
  hn.cy = cy;
  Norm* dn = nullptr;
  float* hist = nullptr;
  int* it = nullptr;
  cudaError_t e = cudaMalloc(&dn, sizeof(Norm));
  if (e == cudaSuccess) e = cudaMalloc(&hist, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&it, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dn, &hn, sizeof(Norm), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(it, 0, sizeof(int), s);
  if (e == cudaSuccess) e = loss_grad(out, tgt, batch, w, h, dn, static_cast<__nv_bfloat16*>(dz), hist, it, s);
  float hl = 0.f;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hl, hist, sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dn);
  cudaFree(hist);
  cudaFree(it);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PMHD_ERR_CUDA;
  }
  *loss = hl;
  return PMHD_OK;
}

}  // extern "C"
