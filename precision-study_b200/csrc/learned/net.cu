// net.cu -- kernels of the learned coarse-grid correction other than the
// convolutions: network inputs / targets from fp64 solver states, the loss
// gradient, Adam with bf16 weight copies, minibatch gathering, restriction
// of fine states, and the checked application of a correction inside a
// solver step (candidate, positivity and divergence checks, decision,
// commit with periodic ghost cells).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "learned/net.h"

namespace pmhd {
namespace learned {

NetLayout net_layout() {
  NetLayout L{};
  const int cin[3] = {kFeat, kWidth, kWidth}, cout[3] = {kWidth, kWidth, kOut};
  int off = 0;
  for (int l = 0; l < 3; l++) {
    L.cin[l] = cin[l];
    L.cout[l] = cout[l];
    L.w_off[l] = off;
    off += cout[l] * 9 * cin[l];
    L.b_off[l] = off;
    off += cout[l];
  }
  L.n_params = off;
  return L;
}

namespace {

__device__ __forceinline__ double sv(const StateView& s, long long b, int k, int i, int j) {
  return s.u[s.offset + b * s.bstride + k * s.vstride + j * s.jstride + i * s.istride];
}

// Whether the step of parity p was taken and left a usable state.
__device__ __forceinline__ bool step_taken(const Ctrl* c, int p) {
  return c->step[p ^ 1] != c->step[p] && !c->halted && !c->err && c->bad1 == BAD_NONE && c->bad2 == BAD_NONE;
}

__global__ void features_kernel(StateView after, StateView before, int batch, int nx, int ny,
                                const Norm* __restrict__ norm, __nv_bfloat16* __restrict__ x) {
  const long long P = (long long)batch * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long b = r / ny;
    __align__(16) __nv_bfloat16 f[kFeat];
#pragma unroll
    for (int k = 0; k < kNVar; k++) {
      const double a = sv(after, b, k, i, j), d = a - sv(before, b, k, i, j);
      f[k] = __float2bfloat16_rn(((float)a - norm->mu[k]) * norm->inv_sig[k]);
      f[kNVar + k] = __float2bfloat16_rn(((float)d - norm->mu[kNVar + k]) * norm->inv_sig[kNVar + k]);
    }
#pragma unroll
    for (int k = 2 * kNVar; k < kFeat; k++) f[k] = __float2bfloat16_rn(0.f);
    uint4* dst = reinterpret_cast<uint4*>(x + q * kFeat);
#pragma unroll
    for (int v = 0; v < kFeat / 8; v++) dst[v] = reinterpret_cast<const uint4*>(f)[v];
  }
}

__global__ void targets_kernel(StateView after, StateView fine, int batch, int nx, int ny,
                               const Norm* __restrict__ norm, float* __restrict__ tgt) {
  const long long P = (long long)batch * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long b = r / ny;
    float* o = tgt + q * kOut;
#pragma unroll
    for (int k = 0; k < kNVar; k++) {
      const double d = sv(fine, b, k, i, j) - sv(after, b, k, i, j);
      o[k] = (float)d * norm->inv_out[k];
    }
#pragma unroll
    for (int k = kNVar; k < kOut; k++) o[k] = 0.f;
  }
}

__global__ void moments_kernel(StateView before, StateView after, StateView fine, int batch, int nx, int ny,
                               double* __restrict__ sums) {
  __shared__ double part[6 * kNVar];
  for (int k = threadIdx.x; k < 6 * kNVar; k += blockDim.x) part[k] = 0.0;
  __syncthreads();
  double acc[6 * kNVar];
#pragma unroll
  for (int k = 0; k < 6 * kNVar; k++) acc[k] = 0.0;
  const long long P = (long long)batch * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long b = r / ny;
#pragma unroll
    for (int k = 0; k < kNVar; k++) {
      const double a = sv(after, b, k, i, j);
      const double v[3] = {a, a - sv(before, b, k, i, j), sv(fine, b, k, i, j) - a};
#pragma unroll
      for (int g = 0; g < 3; g++) {
        acc[g * kNVar + k] += v[g];
        acc[3 * kNVar + g * kNVar + k] += v[g] * v[g];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6 * kNVar; k++) atomicAdd(&part[k], acc[k]);
  __syncthreads();
  for (int k = threadIdx.x; k < 6 * kNVar; k += blockDim.x) atomicAdd(&sums[k], part[k]);
}

__global__ void loss_grad_kernel(const float* __restrict__ out, const float* __restrict__ tgt, long long P,
                                 __nv_bfloat16* __restrict__ dz, float* __restrict__ loss_hist,
                                 const int* __restrict__ it) {
  const float scale = 2.0f / (float)(P * kNVar);
  float part = 0.f;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 g[kOut];
#pragma unroll
    for (int k = 0; k < kOut; k++) {
      float d = 0.f;
      if (k < kNVar) d = out[q * kOut + k] - tgt[q * kOut + k];
      part += d * d;
      g[k] = __float2bfloat16_rn(scale * d);
    }
    uint4* dst = reinterpret_cast<uint4*>(dz + q * kOut);
    dst[0] = reinterpret_cast<const uint4*>(g)[0];
    dst[1] = reinterpret_cast<const uint4*>(g)[1];
  }
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    atomicAdd(loss_hist + *it, s / (float)(P * kNVar));
  }
}

// Writes the bf16 forward and transposed copies of parameter e (if e is a
// weight).
__device__ __forceinline__ void write_bf16(const NetLayout& L, const NetWeights& w, int e, float th) {
#pragma unroll
  for (int l = 0; l < 3; l++) {
    const int n = L.cout[l] * 9 * L.cin[l];
    const int q = e - L.w_off[l];
    if (q >= 0 && q < n) {
      const int co = q / (9 * L.cin[l]), rem = q - co * 9 * L.cin[l];
      const int t = rem / L.cin[l], ci = rem - t * L.cin[l];
      const __nv_bfloat16 bv = __float2bfloat16_rn(th);
      w.wf[l][q] = bv;
      w.wb[l][(ci * 9 + t) * L.cout[l] + co] = bv;
    }
  }
}

// Adam (beta 0.9 / 0.999, eps 1e-8) with a cosine learning-rate decay to 5 %
// over `iters` steps; zeroes the gradient it consumed.
__global__ void adam_kernel(NetLayout L, NetWeights w, float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, const int* __restrict__ it, int iters, float lr) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= L.n_params) return;
  const float b1 = 0.9f, b2 = 0.999f;
  const int t = *it + 1;
  const float g = grad[e];
  grad[e] = 0.f;
  const float mm = b1 * m[e] + (1.f - b1) * g;
  const float vv = b2 * v[e] + (1.f - b2) * g * g;
  m[e] = mm;
  v[e] = vv;
  const float frac = fminf((float)t / (float)iters, 1.f);
  const float lr_t = lr * (0.05f + 0.95f * 0.5f * (1.f + cospif(frac)));
  const float mh = mm / (1.f - powf(b1, (float)t));
  const float vh = vv / (1.f - powf(b2, (float)t));
  const float th = w.theta[e] - lr_t * mh / (sqrtf(vh) + 1e-8f);
  w.theta[e] = th;
  write_bf16(L, w, e, th);
}

__global__ void to_bf16_kernel(NetLayout L, NetWeights w) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < L.n_params) write_bf16(L, w, e, w.theta[e]);
}

__global__ void gather_kernel(const int* __restrict__ schedule, const int* __restrict__ it, int batch,
                              const uint4* __restrict__ feat_all, const uint4* __restrict__ tgt_all,
                              long long n16_feat, long long n16_tgt, uint4* __restrict__ feat,
                              uint4* __restrict__ tgt) {
  const long long per = n16_feat + n16_tgt;
  const int base = *it * batch;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < per * batch;
       q += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(q / per);
    const long long r = q - (long long)b * per;
    const long long pair = schedule[base + b];
    if (r < n16_feat)
      feat[b * n16_feat + r] = feat_all[pair * n16_feat + r];
    else
      tgt[b * n16_tgt + (r - n16_feat)] = tgt_all[pair * n16_tgt + (r - n16_feat)];
  }
}

__global__ void increment_kernel(int* it) { *it += 1; }

__global__ void restrict_kernel(const double* __restrict__ fu, int fpitch, long long fplane, int fnx, int r,
                                int nx, int ny, double* __restrict__ coarse) {
  const long long n = (long long)nx * ny * kNVar;
  const double inv = 1.0 / ((double)r * r);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % kNVar);
    const long long c = q / kNVar;
    const int I = (int)(c % nx), J = (int)(c / nx);
    double s = 0.0;
    for (int b = 0; b < r; b++)
      for (int a = 0; a < r; a++) s += fu[k * fplane + (long long)(J * r + b + 2) * fpitch + (I * r + a + 2)];
    coarse[q] = s * inv;
  }
  (void)fnx;
}

__global__ void load_periodic_kernel(const double* __restrict__ aos, double* __restrict__ u, int pitch,
                                     long long plane, int nx, int ny) {
  const long long n = (long long)(nx + 4) * (ny + 4);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int gi = (int)(q % (nx + 4)), gj = (int)(q / (nx + 4));
    const int si = (gi - 2 + nx) % nx, sj = (gj - 2 + ny) % ny;
#pragma unroll
    for (int k = 0; k < kNVar; k++) u[k * plane + (long long)gj * pitch + gi] = aos[((long long)sj * nx + si) * kNVar + k];
  }
}

__global__ void store_interior_kernel(const double* __restrict__ u, int pitch, long long plane, int nx, int ny,
                                      double* __restrict__ aos) {
  const long long n = (long long)nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
#pragma unroll
    for (int k = 0; k < kNVar; k++) aos[q * kNVar + k] = u[k * plane + (long long)(j + 2) * pitch + (i + 2)];
  }
}

// Candidate = state after the step + sig_out * network output; flags a
// cell whose density or pressure is not positive (or not finite).
__global__ void candidate_kernel(const double* __restrict__ u, int pitch, long long plane, int nx, int ny,
                                 const float* __restrict__ out, const Norm* __restrict__ norm, double gamma,
                                 double* __restrict__ cand, int* __restrict__ flags, const Ctrl* __restrict__ c,
                                 int p) {
  if (!step_taken(c, p)) return;
  const long long n = (long long)nx * ny;
  int bad = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    double U[kNVar];
#pragma unroll
    for (int k = 0; k < kNVar; k++) {
      U[k] = u[k * plane + (long long)(j + 2) * pitch + (i + 2)] + (double)norm->sig_out[k] * (double)out[q * kOut + k];
      cand[q * kNVar + k] = U[k];
    }
    const double rho = U[0];
    const double ke = 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rho;
    const double me = 0.5 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]);
    const double pr = (gamma - 1.0) * (U[4] - ke - me);
    if (!(rho > 0.0) || !(pr > 0.0) || !isfinite(pr)) bad = 1;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1);
}

// sums[0] += ||divB||_1 of the state after the step, sums[1] += that of the
// candidate (central differences, periodic, times the cell area).
__global__ void divnorm_kernel(const double* __restrict__ u, int pitch, long long plane, int nx, int ny,
                               const double* __restrict__ cand, double dx, double dy, double* __restrict__ sums,
                               const Ctrl* __restrict__ c, int p) {
  if (!step_taken(c, p)) return;
  const long long n = (long long)nx * ny;
  double s0 = 0.0, s1 = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const long long g = (long long)(j + 2) * pitch + (i + 2);
    const double d0 = (u[5 * plane + g + 1] - u[5 * plane + g - 1]) / (2.0 * dx) +
                      (u[6 * plane + g + pitch] - u[6 * plane + g - pitch]) / (2.0 * dy);
    const int ip = (i + 1) % nx, im = (i + nx - 1) % nx, jp = (j + 1) % ny, jm = (j + ny - 1) % ny;
    const double d1 = (cand[((long long)j * nx + ip) * kNVar + 5] - cand[((long long)j * nx + im) * kNVar + 5]) / (2.0 * dx) +
                      (cand[((long long)jp * nx + i) * kNVar + 6] - cand[((long long)jm * nx + i) * kNVar + 6]) / (2.0 * dy);
    s0 += fabs(d0);
    s1 += fabs(d1);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], s0 * dx * dy);
    atomicAdd(&sums[1], s1 * dx * dy);
  }
}

__global__ void decide_kernel(int* __restrict__ flags, double* __restrict__ sums, double div_tol,
                              unsigned long long* __restrict__ counters, int* __restrict__ accept, Ctrl* c, int p) {
  int acc = 0;
  if (step_taken(c, p)) {
    if (flags[0]) {
      counters[1]++;
    } else if (sums[1] > (1.0 + div_tol) * sums[0] + 1e-12) {
      counters[2]++;
    } else {
      counters[0]++;
      acc = 1;
      c->chbits[p ^ 1] = 0ull;  // the next step's speed is recomputed from the corrected state
    }
  }
  *accept = acc;
  flags[0] = 0;
  sums[0] = sums[1] = 0.0;
}

__global__ void commit_kernel(const double* __restrict__ cand, double* __restrict__ u, int pitch, long long plane,
                              int nx, int ny, const int* __restrict__ accept) {
  if (!*accept) return;
  const long long n = (long long)(nx + 4) * (ny + 4);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int gi = (int)(q % (nx + 4)), gj = (int)(q / (nx + 4));
    const int si = (gi - 2 + nx) % nx, sj = (gj - 2 + ny) % ny;
#pragma unroll
    for (int k = 0; k < kNVar; k++) u[k * plane + (long long)gj * pitch + gi] = cand[((long long)sj * nx + si) * kNVar + k];
  }
}

unsigned grid_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  if (g > 148LL * 16) g = 148LL * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace

cudaError_t features(const StateView& after, const StateView& before, int batch, int nx, int ny, const Norm* norm,
                     __nv_bfloat16* x, cudaStream_t s) {
  features_kernel<<<grid_for((long long)batch * nx * ny, 256), 256, 0, s>>>(after, before, batch, nx, ny, norm, x);
  return cudaGetLastError();
}

cudaError_t targets(const StateView& after, const StateView& fine, int batch, int nx, int ny, const Norm* norm,
                    float* tgt, cudaStream_t s) {
  targets_kernel<<<grid_for((long long)batch * nx * ny, 256), 256, 0, s>>>(after, fine, batch, nx, ny, norm, tgt);
  return cudaGetLastError();
}

cudaError_t moments(const StateView& before, const StateView& after, const StateView& fine, int batch, int nx,
                    int ny, double* sums, cudaStream_t s) {
  moments_kernel<<<grid_for((long long)batch * nx * ny, 128), 128, 0, s>>>(before, after, fine, batch, nx, ny, sums);
  return cudaGetLastError();
}

cudaError_t loss_grad(const float* out, const float* tgt, long long P, __nv_bfloat16* dz, float* loss_hist,
                      const int* it, cudaStream_t s) {
  loss_grad_kernel<<<grid_for(P, 256), 256, 0, s>>>(out, tgt, P, dz, loss_hist, it);
  return cudaGetLastError();
}

cudaError_t adam(const NetLayout& L, NetWeights w, float* grad, float* m, float* v, const int* it, int iters,
                 float lr, cudaStream_t s) {
  adam_kernel<<<(L.n_params + 255) / 256, 256, 0, s>>>(L, w, grad, m, v, it, iters, lr);
  return cudaGetLastError();
}

cudaError_t weights_to_bf16(const NetLayout& L, NetWeights w, cudaStream_t s) {
  to_bf16_kernel<<<(L.n_params + 255) / 256, 256, 0, s>>>(L, w);
  return cudaGetLastError();
}

cudaError_t gather_pairs(const int* schedule, const int* it, int batch, const __nv_bfloat16* feat_all,
                         const float* tgt_all, long long pix_per_pair, __nv_bfloat16* feat, float* tgt,
                         cudaStream_t s) {
  const long long n16f = pix_per_pair * kFeat * 2 / 16, n16t = pix_per_pair * kOut * 4 / 16;
  gather_kernel<<<grid_for((n16f + n16t) * batch, 256), 256, 0, s>>>(
      schedule, it, batch, reinterpret_cast<const uint4*>(feat_all), reinterpret_cast<const uint4*>(tgt_all), n16f,
      n16t, reinterpret_cast<uint4*>(feat), reinterpret_cast<uint4*>(tgt));
  return cudaGetLastError();
}

cudaError_t increment(int* it, cudaStream_t s) {
  increment_kernel<<<1, 1, 0, s>>>(it);
  return cudaGetLastError();
}

cudaError_t restrict_state(const void* fine_u, int fpitch, long long fplane, int fnx, int fny, int r, double* coarse,
                           cudaStream_t s) {
  const int nx = fnx / r, ny = fny / r;
  restrict_kernel<<<grid_for((long long)nx * ny * kNVar, 256), 256, 0, s>>>(static_cast<const double*>(fine_u), fpitch,
                                                                             fplane, fnx, r, nx, ny, coarse);
  return cudaGetLastError();
}

cudaError_t load_periodic(const double* aos, void* u, int pitch, long long plane, int nx, int ny, cudaStream_t s) {
  load_periodic_kernel<<<grid_for((long long)(nx + 4) * (ny + 4), 256), 256, 0, s>>>(aos, static_cast<double*>(u),
                                                                                      pitch, plane, nx, ny);
  return cudaGetLastError();
}

cudaError_t store_interior(const void* u, int pitch, long long plane, int nx, int ny, double* aos, cudaStream_t s) {
  store_interior_kernel<<<grid_for((long long)nx * ny, 256), 256, 0, s>>>(static_cast<const double*>(u), pitch, plane,
                                                                          nx, ny, aos);
  return cudaGetLastError();
}

cudaError_t correct_step(const CorrState& cs, void* u, int pitch, long long plane, int nx, int ny, double dx,
                         double dy, double gamma, double div_tol, const Ctrl* ctrl, Ctrl* ctrl_w, int p,
                         cudaStream_t s) {
  double* ud = static_cast<double*>(u);
  const long long n = (long long)nx * ny;
  candidate_kernel<<<grid_for(n, 256), 256, 0, s>>>(ud, pitch, plane, nx, ny, cs.out, cs.norm, gamma, cs.cand,
                                                    cs.flags, ctrl, p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  divnorm_kernel<<<grid_for(n, 256), 256, 0, s>>>(ud, pitch, plane, nx, ny, cs.cand, dx, dy, cs.sums, ctrl, p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  decide_kernel<<<1, 1, 0, s>>>(cs.flags, cs.sums, div_tol, cs.counters, cs.accept, ctrl_w, p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  commit_kernel<<<grid_for((long long)(nx + 4) * (ny + 4), 256), 256, 0, s>>>(cs.cand, ud, pitch, plane, nx, ny,
                                                                              cs.accept);
  return cudaGetLastError();
}

}  // namespace learned
}  // namespace pmhd
