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
  const int cin[kLayers] = {kFeat, kWidth, kWidth, kWidth}, cout[kLayers] = {kWidth, kWidth, kWidth, kOut};
  int off = 0;
  for (int l = 0; l < kLayers; l++) {
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

// Whether the step of parity p was taken and left a usable state (no
// control block: a correction applied outside a solver step, always).
__device__ __forceinline__ bool step_taken(const Ctrl* c, int p) {
  if (c == nullptr) return true;
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

// Primitives of one cell of a state view (rho, vx, vy, vz, p, Bx, By, Bz, psi).
__device__ __forceinline__ void prim_at(const StateView& s, long long b, int i, int j, double gamma, double* w) {
  double U[kNVar];
#pragma unroll
  for (int k = 0; k < kNVar; k++) U[k] = sv(s, b, k, i, j);
  const double inv = 1.0 / U[0];
  w[0] = U[0];
  w[1] = U[1] * inv;
  w[2] = U[2] * inv;
  w[3] = U[3] * inv;
  w[4] = (gamma - 1.0) * (U[4] - 0.5 * U[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) -
                          0.5 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]));
  w[5] = U[5];
  w[6] = U[6];
  w[7] = U[7];
  w[8] = U[8];
}

// Target quantities (Out order) of the change from state a to state f; the
// logarithms need positive densities and pressures (usable states), else 0.
__device__ __forceinline__ void target_q(const double* a, const double* f, double* q) {
  q[OUT_LRHO] = (a[0] > 0.0 && f[0] > 0.0) ? log(f[0] / a[0]) : 0.0;
  q[OUT_V] = f[1] - a[1];
  q[OUT_V + 1] = f[2] - a[2];
  q[OUT_V + 2] = f[3] - a[3];
  q[OUT_LP] = (a[4] > 0.0 && f[4] > 0.0) ? log(f[4] / a[4]) : 0.0;
  q[OUT_A] = 0.0;
  q[OUT_BZ] = f[7] - a[7];
  q[OUT_PSI] = f[8] - a[8];
  q[TGT_DBX] = f[5] - a[5];
  q[TGT_DBY] = f[6] - a[6];
}

__global__ void targets_kernel(StateView after, StateView fine, int batch, int nx, int ny,
                               const Norm* __restrict__ norm, double gamma, float* __restrict__ tgt) {
  const long long P = (long long)batch * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long b = r / ny;
    double a[kNVar], f[kNVar], t[kNOutQ];
    prim_at(after, b, i, j, gamma, a);
    prim_at(fine, b, i, j, gamma, f);
    target_q(a, f, t);
    float* o = tgt + q * kOut;
#pragma unroll
    for (int k = 0; k < kNOutQ; k++) o[k] = (float)t[k] * norm->inv_out[k];
#pragma unroll
    for (int k = kNOutQ; k < kOut; k++) o[k] = 0.f;
  }
}

__global__ void moments_kernel(StateView before, StateView after, StateView fine, int batch, int nx, int ny,
                               double gamma, double* __restrict__ sums) {
  constexpr int NS = kMomentSums;
  __shared__ double part[NS];
  for (int k = threadIdx.x; k < NS; k += blockDim.x) part[k] = 0.0;
  __syncthreads();
  double acc[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) acc[k] = 0.0;
  const long long P = (long long)batch * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long b = r / ny;
#pragma unroll
    for (int k = 0; k < kNVar; k++) {
      const double a = sv(after, b, k, i, j), d = a - sv(before, b, k, i, j);
      acc[k] += a;
      acc[kNVar + k] += d;
      acc[2 * kNVar + k] += a * a;
      acc[3 * kNVar + k] += d * d;
    }
    double pa[kNVar], pf[kNVar], t[kNOutQ];
    prim_at(after, b, i, j, gamma, pa);
    prim_at(fine, b, i, j, gamma, pf);
    target_q(pa, pf, t);
#pragma unroll
    for (int k = 0; k < kNOutQ; k++) {
      acc[4 * kNVar + k] += t[k];
      acc[4 * kNVar + kNOutQ + k] += t[k] * t[k];
    }
  }
#pragma unroll
  for (int k = 0; k < NS; k++) atomicAdd(&part[k], acc[k]);
  __syncthreads();
  for (int k = threadIdx.x; k < NS; k += blockDim.x) atomicAdd(&sums[k], part[k]);
}

// Loss over the nine trained quantities: the seven direct channels and the
// two field components, the latter through the curl of OUT_A (periodic on
// each image).  With rx(q) = cy (A(q+j) - A(q-j)) - t_bx(q) and
// ry(q) = -cx (A(q+i) - A(q-i)) - t_by(q), the gradient with respect to A at
// q collects the terms of the four neighbours whose curls contain it.
__global__ void loss_grad_kernel(const float* __restrict__ out, const float* __restrict__ tgt, int batch, int nx,
                                 int ny, const Norm* __restrict__ norm, __nv_bfloat16* __restrict__ dz,
                                 float* __restrict__ loss_hist, const int* __restrict__ it) {
  const long long P = (long long)batch * nx * ny;
  const float scale = 2.0f / (float)(P * 9);
  const float cx = norm->cx, cy = norm->cy;
  float part = 0.f;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny);
    const long long img = r / ny;
    auto at = [&](int ii, int jj) -> long long {
      ii = (ii % nx + nx) % nx;
      jj = (jj % ny + ny) % ny;
      return (img * ny + jj) * nx + ii;
    };
    auto A = [&](int ii, int jj) { return out[at(ii, jj) * kOut + OUT_A]; };
    auto rx = [&](int ii, int jj) { return cy * (A(ii, jj + 1) - A(ii, jj - 1)) - tgt[at(ii, jj) * kOut + TGT_DBX]; };
    auto ry = [&](int ii, int jj) { return -cx * (A(ii + 1, jj) - A(ii - 1, jj)) - tgt[at(ii, jj) * kOut + TGT_DBY]; };
    __align__(16) __nv_bfloat16 g[kOut];
#pragma unroll
    for (int k = 0; k < kOut; k++) {
      float d = 0.f;
      if (k < 8 && k != OUT_A) d = out[q * kOut + k] - tgt[q * kOut + k];
      part += d * d;
      g[k] = __float2bfloat16_rn(scale * d);
    }
    const float rxq = rx(i, j), ryq = ry(i, j);
    part += rxq * rxq + ryq * ryq;
    const float ga = cy * (rx(i, j - 1) - rx(i, j + 1)) + cx * (ry(i + 1, j) - ry(i - 1, j));
    g[OUT_A] = __float2bfloat16_rn(scale * ga);
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
    atomicAdd(loss_hist + *it, s / (float)(P * 9));
  }
}

// Writes the bf16 forward and transposed copies of parameter e (if e is a
// weight).
__device__ __forceinline__ void write_bf16(const NetLayout& L, const NetWeights& w, int e, float th) {
#pragma unroll
  for (int l = 0; l < kLayers; l++) {
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

// splitmix64 finaliser as a counter-based hash (published mixing constants).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void input_noise_kernel(__nv_bfloat16* __restrict__ x, long long n, float sigma,
                                   const int* __restrict__ it, unsigned long long seed) {
  const unsigned long long base = mix64(seed ^ (0x9e3779b97f4a7c15ull * (unsigned long long)(*it + 1)));
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long q = e / (2 * kNVar), c = e % (2 * kNVar);
    const unsigned long long h = mix64(base + (unsigned long long)e);
    // Box-Muller from two 24-bit uniforms in (0, 1).
    const float u1 = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
    const float u2 = ((float)((h >> 16) & 0xFFFFFF) + 0.5f) * (1.0f / 16777216.0f);
    const float g = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
    __nv_bfloat16* p = x + q * kFeat + c;
    *p = __float2bfloat16_rn(__bfloat162float(*p) + sigma * g);
  }
}

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

// Candidate = the state after the step corrected by the network output:
// density and pressure scaled by exp(correction) (the exponent clamped to
// [-2, 2]), velocities, B_z and psi shifted, B_x and B_y shifted by the
// central-difference curl of the potential (periodic).  Accumulates the
// domain sums of the changes of the conserved quantities (sums[2..]).
__constant__ int kConserved[kNConserved] = {0, 1, 2, 3, 4, 7};

__global__ void candidate_kernel(const double* __restrict__ u, int pitch, long long plane, int nx, int ny,
                                 const float* __restrict__ out, const Norm* __restrict__ norm, double gamma,
                                 double dx, double dy, double relax, double shrink, double* __restrict__ cand,
                                 double* __restrict__ sums, const Ctrl* __restrict__ c, int p) {
  if (!step_taken(c, p)) return;
  const long long n = (long long)nx * ny;
  double dsum[kNConserved] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // Soft threshold: sign(o) max(|o| - shrink, 0) of a normalised output.
  auto shr = [shrink](float o) {
    const double a = fabs((double)o) - shrink;
    return a > 0.0 ? copysign(a, (double)o) : 0.0;
  };
  const double sA = relax * norm->sig_out[OUT_A];
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    double U[kNVar];
#pragma unroll
    for (int k = 0; k < kNVar; k++) U[k] = u[k * plane + (long long)(j + 2) * pitch + (i + 2)];
    const float* o = out + q * kOut;
    auto sig = [&](int k) { return relax * (double)norm->sig_out[k] * shr(o[k]); };
    auto clamp2 = [](double x) { return x < -2.0 ? -2.0 : (x > 2.0 ? 2.0 : x); };
    const double rho = U[0], inv = 1.0 / rho;
    const double vx = U[1] * inv, vy = U[2] * inv, vz = U[3] * inv;
    const double pr = (gamma - 1.0) * (U[4] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) -
                                       0.5 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]));
    const double rho1 = rho * exp(clamp2(sig(OUT_LRHO)));
    const double vx1 = vx + sig(OUT_V), vy1 = vy + sig(OUT_V + 1), vz1 = vz + sig(OUT_V + 2);
    const double p1 = pr * exp(clamp2(sig(OUT_LP)));
    const int ip = (i + 1) % nx, im = (i + nx - 1) % nx, jp = (j + 1) % ny, jm = (j + ny - 1) % ny;
    const double a_n = sA * shr(out[((long long)jp * nx + i) * kOut + OUT_A]);
    const double a_s = sA * shr(out[((long long)jm * nx + i) * kOut + OUT_A]);
    const double a_e = sA * shr(out[((long long)j * nx + ip) * kOut + OUT_A]);
    const double a_w = sA * shr(out[((long long)j * nx + im) * kOut + OUT_A]);
    const double bx1 = U[5] + (a_n - a_s) / (2.0 * dy), by1 = U[6] - (a_e - a_w) / (2.0 * dx);
    const double bz1 = U[7] + sig(OUT_BZ), psi1 = U[8] + sig(OUT_PSI);
    double* C = cand + q * kNVar;
    C[0] = rho1;
    C[1] = rho1 * vx1;
    C[2] = rho1 * vy1;
    C[3] = rho1 * vz1;
    C[4] = p1 / (gamma - 1.0) + 0.5 * rho1 * (vx1 * vx1 + vy1 * vy1 + vz1 * vz1) +
           0.5 * (bx1 * bx1 + by1 * by1 + bz1 * bz1);
    C[5] = bx1;
    C[6] = by1;
    C[7] = bz1;
    C[8] = psi1;
#pragma unroll
    for (int k = 0; k < kNConserved; k++) dsum[k] += C[kConserved[k]] - U[kConserved[k]];
  }
#pragma unroll
  for (int k = 0; k < kNConserved; k++) {
    double v = dsum[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sums[2 + k], v);
  }
}

// The restricted fine state and the coarse state conserve the same totals on
// the periodic grid, so the true correction of a conserved quantity has zero
// mean: its domain mean is removed from the candidate (a systematic bias of
// the network would otherwise build up step after step).  Then flags a cell
// whose density or pressure is not positive (or not finite).
__global__ void conserve_kernel(double* __restrict__ cand, int nx, int ny, double gamma,
                                const double* __restrict__ sums, int* __restrict__ flags,
                                const Ctrl* __restrict__ c, int p) {
  if (!step_taken(c, p)) return;
  const long long n = (long long)nx * ny;
  double mean[kNConserved];
#pragma unroll
  for (int k = 0; k < kNConserved; k++) mean[k] = sums[2 + k] / (double)n;
  int bad = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    double* C = cand + q * kNVar;
#pragma unroll
    for (int k = 0; k < kNConserved; k++) C[kConserved[k]] -= mean[k];
    const double rho = C[0];
    const double pr = (gamma - 1.0) * (C[4] - 0.5 * (C[1] * C[1] + C[2] * C[2] + C[3] * C[3]) / rho -
                                       0.5 * (C[5] * C[5] + C[6] * C[6] + C[7] * C[7]));
    if (!(rho > 0.0) || !(pr > 0.0) || !isfinite(C[4]) || !isfinite(C[1] + C[2] + C[3] + C[5] + C[6] + C[8]))
      bad = 1;
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
      if (c) c->chbits[p ^ 1] = 0ull;  // the next step's speed is recomputed from the corrected state
    }
  }
  *accept = acc;
  flags[0] = 0;
  for (int k = 0; k < kCorrSums; k++) sums[k] = 0.0;
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
                    double gamma, float* tgt, cudaStream_t s) {
  targets_kernel<<<grid_for((long long)batch * nx * ny, 256), 256, 0, s>>>(after, fine, batch, nx, ny, norm, gamma,
                                                                            tgt);
  return cudaGetLastError();
}

cudaError_t moments(const StateView& before, const StateView& after, const StateView& fine, int batch, int nx,
                    int ny, double gamma, double* sums, cudaStream_t s) {
  moments_kernel<<<grid_for((long long)batch * nx * ny, 128), 128, 0, s>>>(before, after, fine, batch, nx, ny, gamma,
                                                                            sums);
  return cudaGetLastError();
}

cudaError_t loss_grad(const float* out, const float* tgt, int batch, int nx, int ny, const Norm* norm,
                      __nv_bfloat16* dz, float* loss_hist, const int* it, cudaStream_t s) {
  loss_grad_kernel<<<grid_for((long long)batch * nx * ny, 256), 256, 0, s>>>(out, tgt, batch, nx, ny, norm, dz,
                                                                              loss_hist, it);
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

cudaError_t input_noise(__nv_bfloat16* x, long long P, float sigma, const int* it, unsigned long long seed,
                        cudaStream_t s) {
  const long long n = P * 2 * kNVar;
  input_noise_kernel<<<grid_for(n, 256), 256, 0, s>>>(x, n, sigma, it, seed);
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
  candidate_kernel<<<grid_for(n, 256), 256, 0, s>>>(ud, pitch, plane, nx, ny, cs.out, cs.norm, gamma, dx, dy,
                                                    cs.relax, cs.shrink, cs.cand, cs.sums, ctrl, p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  conserve_kernel<<<grid_for(n, 256), 256, 0, s>>>(cs.cand, nx, ny, gamma, cs.sums, cs.flags, ctrl, p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
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
