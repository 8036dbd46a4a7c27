// conv.h -- launchers of the BF16 tensor-core 3x3 convolutions (conv.cu).
#ifndef PMHD_LEARNED_CONV_H
#define PMHD_LEARNED_CONV_H

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pmhd {
namespace learned {

enum ConvMode : int { CONV_GELU = 0, CONV_LINEAR = 1, CONV_DGELU = 2 };
enum : int { PMHD_LEARNED_ERR_TIMEOUT = 1 };

// Sets the kernels' shared-memory limits on the current device; call once
// per device before the first launch (and before any stream capture).
cudaError_t conv_prepare();

// One 3x3 periodic convolution over NHWC bf16 images (see conv.cu).
//   CONV_GELU:   out0 = z = conv(x) + bias (bf16), out1 = gelu(z) (bf16)
//   CONV_LINEAR: out0 = conv(x) + bias (fp32)
//   CONV_DGELU:  out0 = (transposed conv of x) * gelu'(zprev) (bf16); wt is
//                the layer's weight transposed to [c_out][9][c_in] with c_in
//                = the layer's outputs
// Supported (c_in, c_out): GELU (32, 32); LINEAR (32, 16); DGELU (16, 32),
// (32, 32).  cudaErrorNotSupported otherwise.  *err is set (non-zero) when
// a bounded wait of the kernel expired.
cudaError_t conv3x3(int mode, const __nv_bfloat16* x, int batch, int h, int w, int c_in, const __nv_bfloat16* wt,
                    const float* bias, int c_out, const __nv_bfloat16* zprev, void* out0, void* out1, int* err,
                    cudaStream_t s);

// dw[co][t][ci] += sum_p dz[p][co] x[p + tap t][ci]; db[co] += sum_p dz[p][co]
// (db may be null).  Supported (c_in, c_out): (32, 32), (32, 16).
cudaError_t conv3x3_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dz, int batch, int h, int w, int c_in,
                          int c_out, float* dw, float* db, int* err, cudaStream_t s);

}  // namespace learned
}  // namespace pmhd

#endif  // PMHD_LEARNED_CONV_H
