// conv.cu -- BF16 tensor-core (tcgen05, accumulators in tensor memory) 3x3
// convolutions of the learned coarse-grid correction: forward with bias and
// GELU, forward linear, backward to the input through the previous layer's
// GELU, and the weight gradient.  Images are NHWC bf16 tensors
// [batch][h][w][channels], periodic in y and x (the coarse grids they come
// from are periodic).  Weights are [c_out][9][c_in] with tap t = (dy+1)*3 +
// (dx+1): out(y, x) = sum_t W[t] x(y+dy, x+dx) (cross-correlation).
//
// Implicit GEMM.  Forward / backward-data: M = 128 output pixels x N = c_out
// channels, K = 9 taps x c_in channels.  Row kernels (width a multiple of
// 128, height of 8): a row tile's input is staged once, each tap's operand
// is a shifted descriptor into it, one thread issues 8 rows x 9 * c_in / 16
// tcgen05.mma, eight warps run the epilogue -- one CTA per tile, or (from
// two tiles per SM) a persistent CTA per SM whose producer, MMA and
// epilogue warps pipeline the tiles.  Gather kernel (other shapes):
// one CTA per 128 pixels gathers the 9 shifted copies of its pixels' input
// vectors (periodic wrap) into K-major tiles, one thread issues 9 * c_in / 16
// tcgen05.mma, the four warps read the 128 x N accumulator back with
// tcgen05.ld and run the epilogue.  Weight gradient: D[(t, c_in)][c_out] =
// sum over pixels of x(p + tap) dz(p)^T, K = pixels: blocks of 8 pixels x 8
// channels are transposed in registers into K-major tiles, three M = 128
// tiles accumulate over 64-pixel chunks, CTAs sum with fp32 atomics.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdlib>

#include "learned/conv.h"
#include "learned/umma.cuh"

namespace pmhd {
namespace learned {

namespace {

constexpr uint32_t kWaitPolls = 1u << 22;

// GELU in the tanh form, 0.5 z (1 + tanh(y)) with y = sqrt(2/pi) (z + 0.044715
// z^3), written as z s with s = 1 / (1 + exp(-2 y)): one hardware exp2 and
// one reciprocal, and the left tail keeps its relative accuracy (s is never
// formed as a difference).  Its derivative: s + z s (1 - s) dy2/dz.
constexpr float kGeluA = 1.5957691216057308f;     // 2 sqrt(2 / pi)
constexpr float kGeluB = 0.071354816272737f;      // 2 sqrt(2 / pi) 0.044715
constexpr float kLog2e = 1.4426950408889634f;
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float gelu_sigmoid(float z) {
  const float y2 = z * (kGeluA + kGeluB * z * z);
  return rcp_approx(1.0f + ex2_approx(-y2 * kLog2e));
}
__device__ __forceinline__ float gelu(float z) { return z * gelu_sigmoid(z); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float s = gelu_sigmoid(z);
  return s + z * s * (1.0f - s) * (kGeluA + 3.0f * kGeluB * z * z);
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ uint32_t word_of(const uint4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Row `ch` of the 8 x 8 bf16 transpose of v[0..7] (v[q] = 8 channels of
// pixel q): the 8 pixels' values of channel ch, pixel q in halfword q.
__device__ __forceinline__ uint4 transpose_row(const uint4 (&v)[8], int ch) {
  const uint32_t sel = (ch & 1) ? 0x7632u : 0x5410u;
  const int wi = ch >> 1;
  uint4 r;
  r.x = __byte_perm(word_of(v[0], wi), word_of(v[1], wi), sel);
  r.y = __byte_perm(word_of(v[2], wi), word_of(v[3], wi), sel);
  r.z = __byte_perm(word_of(v[4], wi), word_of(v[5], wi), sel);
  r.w = __byte_perm(word_of(v[6], wi), word_of(v[7], wi), sel);
  return r;
}

// Bounded wait for the MMA batch; on expiry record the error and wait once
// more (bounded) so tensor memory is not released under a running MMA.
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t parity, int* err) {
  bool ok = mbar_wait_bounded(bar, parity, kWaitPolls);
  ok = __all_sync(0xffffffffu, ok);
  if (!ok) {
    if ((threadIdx.x & 31) == 0) atomicExch(err, PMHD_LEARNED_ERR_TIMEOUT);
    mbar_wait_bounded(bar, parity, kWaitPolls);
  }
  return ok;
}

// Epilogue of one output pixel p from its CO fp32 accumulators; `bias` is
// the CTA's 16-byte-aligned shared copy (unused by CONV_DGELU).
template <int CO, int EPI>
__device__ __forceinline__ void epilogue(const float (&acc)[CO], long long p, const float* __restrict__ bias,
                                         const __nv_bfloat16* __restrict__ zprev, void* __restrict__ out0,
                                         void* __restrict__ out1) {
  if (EPI == CONV_GELU) {
    __nv_bfloat16* z = static_cast<__nv_bfloat16*>(out0) + p * CO;
    __nv_bfloat16* a = static_cast<__nv_bfloat16*>(out1) + p * CO;
#pragma unroll
    for (int c8 = 0; c8 < CO / 8; c8++) {
      __align__(16) __nv_bfloat162 zb[4], ab[4];
      const float4 b0 = reinterpret_cast<const float4*>(bias)[c8 * 2];
      const float4 b1 = reinterpret_cast<const float4*>(bias)[c8 * 2 + 1];
      const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float z0 = acc[c8 * 8 + 2 * q] + bb[2 * q];
        const float z1 = acc[c8 * 8 + 2 * q + 1] + bb[2 * q + 1];
        zb[q] = __floats2bfloat162_rn(z0, z1);
        ab[q] = __floats2bfloat162_rn(gelu(z0), gelu(z1));
      }
      *reinterpret_cast<uint4*>(z + c8 * 8) = *reinterpret_cast<const uint4*>(zb);
      *reinterpret_cast<uint4*>(a + c8 * 8) = *reinterpret_cast<const uint4*>(ab);
    }
  } else if (EPI == CONV_LINEAR) {
    float* o = static_cast<float*>(out0) + p * CO;
#pragma unroll
    for (int c4 = 0; c4 < CO / 4; c4++) {
      const float4 b = reinterpret_cast<const float4*>(bias)[c4];
      float4 v;
      v.x = acc[c4 * 4 + 0] + b.x;
      v.y = acc[c4 * 4 + 1] + b.y;
      v.z = acc[c4 * 4 + 2] + b.z;
      v.w = acc[c4 * 4 + 3] + b.w;
      *reinterpret_cast<float4*>(o + c4 * 4) = v;
    }
  } else {
    const __nv_bfloat16* zp = zprev + p * CO;
    __nv_bfloat16* d = static_cast<__nv_bfloat16*>(out0) + p * CO;
#pragma unroll
    for (int c8 = 0; c8 < CO / 8; c8++) {
      const uint4 zv = *reinterpret_cast<const uint4*>(zp + c8 * 8);
      const __nv_bfloat16* zs = reinterpret_cast<const __nv_bfloat16*>(&zv);
      __align__(16) __nv_bfloat16 db[8];
#pragma unroll
      for (int q = 0; q < 8; q++) db[q] = __float2bfloat16_rn(acc[c8 * 8 + q] * gelu_grad(__bfloat162float(zs[q])));
      *reinterpret_cast<uint4*>(d + c8 * 8) = *reinterpret_cast<const uint4*>(db);
    }
  }
}

// B operand: the weights [CO][9 CG], K-groups of 8 (16-byte vectors) at
// kLboB = CO * 16; thread t of nt.
template <int CG, int CO>
__device__ __forceinline__ void stage_weights(unsigned char* sB, const __nv_bfloat16* __restrict__ wt, int t,
                                              int nt) {
  constexpr int K = 9 * CG;
  for (int c = t; c < CO * (K / 8); c += nt) {
    const int n = c / (K / 8), g = c - n * (K / 8);
    const uint4 v = *reinterpret_cast<const uint4*>(wt + (size_t)n * K + g * 8);
    *reinterpret_cast<uint4*>(sB + n * 16 + g * CO * 16) = v;
  }
}

template <int CG, int CO>
struct ConvSmem {
  static constexpr int K = 9 * CG;
  static constexpr uint32_t kATap = 128u * CG * 2u;  // bytes of one tap tile
  static constexpr uint32_t kLboA = 128u * 16u;      // K-group stride of A
  static constexpr uint32_t kBytesB = (uint32_t)CO * K * 2u;
  static constexpr uint32_t kLboB = (uint32_t)CO * 16u;
  static constexpr uint32_t kOffB = 9u * kATap;
  static constexpr uint32_t kOffBar = kOffB + kBytesB;
  static constexpr uint32_t kBytes = kOffBar + 16u;
};

// EPI: CONV_GELU   out0 = z (bf16), out1 = gelu(z) (bf16), z = acc + bias
//      CONV_LINEAR out0 = acc + bias (fp32)
//      CONV_DGELU  out0 = acc * gelu'(zprev) (bf16); taps mirrored (the
//                  transposed convolution of the backward pass)
template <int CG, int CO, int EPI>
__global__ void __launch_bounds__(128) conv3x3_kernel(const __nv_bfloat16* __restrict__ x,
                                                      const __nv_bfloat16* __restrict__ wt,
                                                      const float* __restrict__ bias,
                                                      const __nv_bfloat16* __restrict__ zprev, int batch, int h,
                                                      int w, void* __restrict__ out0, void* __restrict__ out1,
                                                      int* __restrict__ err) {
  using S = ConvSmem<CG, CO>;
  constexpr uint32_t kCols = umma::tmem_cols(CO);
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + S::kOffB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S::kOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::kOffBar + 8);
  __shared__ __align__(16) float sbias[CO];
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long P = (long long)batch * h * w;
  const long long p0 = (long long)blockIdx.x * 128;
  if (tid < CO) sbias[tid] = EPI == CONV_DGELU ? 0.0f : bias[tid];

  if (warp == 0) {
    umma::tmem_alloc(tslot, kCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  stage_weights<CG, CO>(sB, wt, tid, 128);
  // A operand: for each tap, the 128 pixels' shifted input vectors.
  for (int c = tid; c < 9 * 128 * (CG / 8); c += 128) {
    const int g = c % (CG / 8);
    const int m = (c / (CG / 8)) % 128;
    const int t = c / (128 * (CG / 8));
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    const long long p = p0 + m;
    if (p < P) {
      const int x0 = (int)(p % w);
      const long long r = p / w;
      const int y0 = (int)(r % h);
      const long long b = r / h;
      int dy = t / 3 - 1, dx = t % 3 - 1;
      if (EPI == CONV_DGELU) {
        dy = -dy;
        dx = -dx;
      }
      const int yy = wrap(y0 + dy, h), xx = wrap(x0 + dx, w);
      v = *reinterpret_cast<const uint4*>(x + ((b * h + yy) * (long long)w + xx) * CG + g * 8);
    }
    *reinterpret_cast<uint4*>(sA + t * S::kATap + m * 16 + g * S::kLboA) = v;
  }
  fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    constexpr uint32_t idesc = umma::idesc_bf16(128, CO, false, false);
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll 1
    for (int t = 0; t < 9; t++)
#pragma unroll
      for (int kc = 0; kc < CG / 16; kc++) {
        const uint64_t da = umma::desc(a0 + t * S::kATap + kc * 2 * S::kLboA, S::kLboA, 128);
        const uint64_t db = umma::desc(b0 + (t * (CG / 8) + kc * 2) * S::kLboB, S::kLboB, 128);
        umma::mma_bf16(tmem, da, db, idesc, (t | kc) ? 1u : 0u);
      }
    umma::commit(bar);
  }
  __syncwarp();
  const bool ok = wait_mma(bar, 0, err);
  umma::fence_after_sync();
  if (ok) {
    float acc[CO];
#pragma unroll
    for (int c8 = 0; c8 < CO / 8; c8++) umma::ld8(tmem + ((uint32_t)(warp * 32) << 16) + c8 * 8, acc + c8 * 8);
    const long long p = p0 + tid;
    if (p < P) epilogue<CO, EPI>(acc, p, sbias, zprev, out0, out1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, kCols);
  }
}

constexpr int kRowPix = 128;               // output pixels of a row segment (M)
constexpr int kRows = 8;                   // output rows per tile
constexpr int kRowPitch = kRowPix + 2;     // staged pixels per input row
constexpr int kRowThreads = 256;
constexpr uint32_t kRowLboA = (uint32_t)(kRows + 2) * kRowPitch * 16u;  // channel-group stride of A

template <int CG, int CO>
struct RowSmem {
  static constexpr int K = 9 * CG;
  static constexpr uint32_t kBytesA = (uint32_t)(CG / 8) * kRowLboA;
  static constexpr uint32_t kOffB = (kBytesA + 127u) & ~127u;
  static constexpr uint32_t kBytesB = (uint32_t)CO * K * 2u;
  static constexpr uint32_t kOffBar = kOffB + kBytesB;
  static constexpr uint32_t kBytes = kOffBar + 16u;
  // Shared memory requested per CTA: at least enough that no more CTAs fit
  // on an SM (228 KB) than its 512 tensor-memory columns hold; eight CTAs of
  // 256 threads are the thread limit anyway.
  static constexpr uint32_t kTmemCols = umma::tmem_cols(kRows * CO);
  static constexpr uint32_t kMaxCtas = 512u / kTmemCols;
  static constexpr uint32_t kMinBytes = kMaxCtas >= 8u ? 0u : (228u * 1024u) / (kMaxCtas + 1u) + 1024u;
  static constexpr uint32_t kLaunchBytes = kBytes > kMinBytes ? kBytes : kMinBytes;
};

// A row tile: image bb, output rows y0 .. y0 + kRows - 1, pixels x0 .. x0 + 127.
struct RowTile {
  long long bb;
  int y0, x0;
};
__device__ __forceinline__ RowTile row_tile(long long tile, int h, int w) {
  const int segs = w / kRowPix, rblocks = h / kRows;
  RowTile t;
  t.x0 = (int)(tile % segs) * kRowPix;
  t.y0 = (int)((tile / segs) % rblocks) * kRows;
  t.bb = tile / ((long long)segs * rblocks);
  return t;
}

// A operand of a row tile: input rows y0 - 1 .. y0 + kRows, pixels
// x0 - 1 .. x0 + 128 (periodic), one 16-byte channel group per item
// (consecutive items are consecutive 16-byte words of the NHWC input), by
// asynchronous copies from thread t of nt; the caller waits for them.
template <int CG>
__device__ __forceinline__ void stage_row_tile(unsigned char* sA, const __nv_bfloat16* __restrict__ x,
                                               const RowTile& rt, int h, int w, int t, int nt) {
  for (int c = t; c < (kRows + 2) * kRowPitch * (CG / 8); c += nt) {
    const int g = c % (CG / 8);
    const int px = (c / (CG / 8)) % kRowPitch;
    const int r = c / ((CG / 8) * kRowPitch);
    const int yy = wrap(rt.y0 - 1 + r, h), xx = wrap(rt.x0 - 1 + px, w);
    const uint32_t dst = smem_u32(sA + g * kRowLboA + (r * kRowPitch + px) * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                 "l"(x + ((rt.bb * h + yy) * (long long)w + xx) * CG + g * 8)
                 : "memory");
  }
}

// The row tile's MMAs, issued by one thread: for output row r and tap
// (dy, dx) (mirrored for CONV_DGELU) the A operand is the staged tile seen
// from pixel 1 + dx of staged row r + 1 + dy -- a shift of the descriptor's
// start address; accumulators of row r at d0 + r * CO.
template <int CG, int CO, int EPI>
__device__ __forceinline__ void issue_row_mmas(uint32_t a0, uint32_t b0, uint32_t d0) {
  constexpr uint32_t idesc = umma::idesc_bf16(128, CO, false, false);
  constexpr uint32_t kLboB = (uint32_t)CO * 16u;
#pragma unroll 1
  for (int r = 0; r < kRows; r++)
#pragma unroll 1
    for (int t = 0; t < 9; t++) {
      int dy = t / 3 - 1, dx = t % 3 - 1;
      if (EPI == CONV_DGELU) {
        dy = -dy;
        dx = -dx;
      }
      const uint32_t at = a0 + (uint32_t)(((r + 1 + dy) * kRowPitch + 1 + dx) * 16);
#pragma unroll
      for (int kc = 0; kc < CG / 16; kc++) {
        const uint64_t da = umma::desc(at + kc * 2 * kRowLboA, kRowLboA, 128);
        const uint64_t db = umma::desc(b0 + (t * (CG / 8) + kc * 2) * kLboB, kLboB, 128);
        umma::mma_bf16(d0 + (uint32_t)(r * CO), da, db, idesc, (t | kc) ? 1u : 0u);
      }
    }
}

// Reads a row tile's accumulators back (tensor-memory columns from tbase)
// and runs the epilogue: warp `warp` of `nwarps` owns lane quarter warp % 4
// (pixels 32 q .. 32 q + 31) of rows warp / 4, warp / 4 + nwarps / 4, ...
template <int CO, int EPI>
__device__ __forceinline__ void drain_row_tile(uint32_t tbase, int warp, int lane, int nwarps, const RowTile& rt,
                                               int h, int w, const float* __restrict__ sbias,
                                               const __nv_bfloat16* __restrict__ zprev, void* __restrict__ out0,
                                               void* __restrict__ out1) {
  const int q = warp & 3;
  for (int r = warp >> 2; r < kRows; r += nwarps / 4) {
    float acc[CO];
#pragma unroll
    for (int c8 = 0; c8 < CO / 8; c8++)
      umma::ld8(tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(r * CO + c8 * 8), acc + c8 * 8);
    const long long p = (rt.bb * h + rt.y0 + r) * (long long)w + rt.x0 + q * 32 + lane;
    epilogue<CO, EPI>(acc, p, sbias, zprev, out0, out1);
  }
}

// Row kernel (forward / backward-data when the width is a multiple of 128
// and the height of 8), one CTA of 8 warps per row tile of kRows image rows
// x 128 pixels.  It stages the (kRows + 2) x 130 input pixels around them
// once (periodic wrap), channel-group-interleaved: group g of 8 channels at
// g * kRowLboA, then row, then pixel at 16 bytes -- the K-major no-swizzle
// layout of an M = 128 operand whose rows are pixels, so the nine taps need
// no copies (issue_row_mmas).  Accumulators: 128 lanes x CO columns per row,
// kRows rows side by side in tensor memory.  (Measured at batch 8 x 512^2:
// 8, 4 and 2 rows per CTA -- two to four CTAs per SM -- run equally fast.)
template <int CG, int CO, int EPI>
__global__ void __launch_bounds__(kRowThreads) conv3x3_rows_kernel(const __nv_bfloat16* __restrict__ x,
                                                                   const __nv_bfloat16* __restrict__ wt,
                                                                   const float* __restrict__ bias,
                                                                   const __nv_bfloat16* __restrict__ zprev,
                                                                   int batch, int h, int w,
                                                                   void* __restrict__ out0, void* __restrict__ out1,
                                                                   int* __restrict__ err) {
  using S = RowSmem<CG, CO>;
  constexpr uint32_t kCols = S::kTmemCols;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + S::kOffB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S::kOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::kOffBar + 8);
  __shared__ __align__(16) float sbias[CO];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const RowTile rt = row_tile(blockIdx.x, h, w);
  (void)batch;

  if (warp == 0) {
    umma::tmem_alloc(tslot, kCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  if (tid < CO) sbias[tid] = EPI == CONV_DGELU ? 0.0f : bias[tid];
  stage_weights<CG, CO>(sB, wt, tid, kRowThreads);
  stage_row_tile<CG>(sA, x, rt, h, w, tid, kRowThreads);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    issue_row_mmas<CG, CO, EPI>(smem_u32(sA), smem_u32(sB), tmem);
    umma::commit(bar);
  }
  __syncwarp();
  const bool ok = wait_mma(bar, 0, err);
  umma::fence_after_sync();
  if (ok) drain_row_tile<CO, EPI>(tmem, warp, lane, kRowThreads / 32, rt, h, w, sbias, zprev, out0, out1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, kCols);
  }
}

// Persistent, warp-specialised form of the row kernel: one CTA per SM
// loops over the row tiles; four producer warps stage tile k + 1 (16-byte
// asynchronous copies) while one thread issues tile k's MMAs and eight
// warps drain tile k - 1 from tensor memory.  Two staging buffers and two
// accumulator buffers; the hand-offs are mbarriers:
//   full[b]   producers -> MMA      staging buffer b holds its tile
//   empty[b]  MMA commit -> producers  the MMAs that read buffer b are done
//   tfull[b]  MMA commit -> epilogue   accumulator buffer b is complete
//   tempty[b] epilogue -> MMA          accumulator buffer b has been read
// Every wait is bounded; on expiry the CTA records the error and leaves.
constexpr int kPipeEpiWarps = 8, kPipeProdWarps = 4;
constexpr int kPipeThreads = 32 * (kPipeEpiWarps + kPipeProdWarps + 1);

template <int CG, int CO>
struct PipeSmem {
  using R = RowSmem<CG, CO>;
  static constexpr uint32_t kStage = (R::kBytesA + 127u) & ~127u;  // one staging buffer (A operand)
  static constexpr uint32_t kOffB = 2u * kStage;
  static constexpr uint32_t kOffBar = (kOffB + R::kBytesB + 7u) & ~7u;
  static constexpr uint32_t kBytes = kOffBar + 8u * 8u + 16u;
  static constexpr uint32_t kColsBuf = umma::tmem_cols(kRows * CO);
  static constexpr uint32_t kTmemCols = 2u * kColsBuf;
  // At most 512 / kTmemCols CTAs per SM (see RowSmem).
  static constexpr uint32_t kMaxCtas = 512u / kTmemCols;
  static constexpr uint32_t kMinBytes = (228u * 1024u) / (kMaxCtas + 1u) + 1024u;
  static constexpr uint32_t kLaunchBytes = kBytes > kMinBytes ? kBytes : kMinBytes;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait agreed by the whole warp.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity) {
  return __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity, kWaitPolls));
}

template <int CG, int CO, int EPI>
__global__ void __launch_bounds__(kPipeThreads, 1) conv3x3_pipe_kernel(const __nv_bfloat16* __restrict__ x,
                                                                       const __nv_bfloat16* __restrict__ wt,
                                                                       const float* __restrict__ bias,
                                                                       const __nv_bfloat16* __restrict__ zprev,
                                                                       int batch, int h, int w,
                                                                       void* __restrict__ out0,
                                                                       void* __restrict__ out1,
                                                                       int* __restrict__ err) {
  using S = PipeSmem<CG, CO>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sB = smem + S::kOffB;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::kOffBar);
  uint64_t* empty = full + 2;
  uint64_t* tfull = full + 4;
  uint64_t* tempty = full + 6;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 8);
  __shared__ __align__(16) float sbias[CO];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long ntiles = (long long)batch * (h / kRows) * (w / kRowPix);

  if (warp == 0) {
    umma::tmem_alloc(tslot, S::kTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    for (int b = 0; b < 2; b++) {
      mbar_init(full + b, kPipeProdWarps * 32);
      mbar_init(empty + b, 1);
      mbar_init(tfull + b, 1);
      mbar_init(tempty + b, kPipeEpiWarps * 32);
    }
    fence_barrier_init();
  }
  if (tid < CO) sbias[tid] = EPI == CONV_DGELU ? 0.0f : bias[tid];
  stage_weights<CG, CO>(sB, wt, tid, kPipeThreads);
  fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp >= kPipeEpiWarps && warp < kPipeEpiWarps + kPipeProdWarps) {
    // Producers: stage tile k into buffer k % 2 once the MMAs of tile k - 2
    // (the buffer's previous tile) are done.
    const int pt = tid - kPipeEpiWarps * 32;
    int k = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
      const int b = k & 1;
      if (k >= 2 && !warp_wait(empty + b, (uint32_t)((k >> 1) - 1) & 1u)) {
        ok = false;
        break;
      }
      stage_row_tile<CG>(smem + b * S::kStage, x, row_tile(tile, h, w), h, w, pt, kPipeProdWarps * 32);
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      fence_proxy_async_smem();
      mbar_arrive(full + b);
    }
  } else if (warp == kPipeEpiWarps + kPipeProdWarps) {
    // MMA issuer: tile k from buffer k % 2 into accumulator buffer k % 2
    // once the epilogue has read that buffer's previous tile (k - 2).
    int k = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
      const int b = k & 1;
      if (!warp_wait(full + b, (uint32_t)(k >> 1) & 1u) ||
          (k >= 2 && !warp_wait(tempty + b, (uint32_t)((k >> 1) - 1) & 1u))) {
        ok = false;
        break;
      }
      umma::fence_after_sync();
      if (lane == 0) {
        issue_row_mmas<CG, CO, EPI>(smem_u32(smem + b * S::kStage), smem_u32(sB),
                                    tmem + (uint32_t)b * S::kColsBuf);
        umma::commit(tfull + b);
        umma::commit(empty + b);
      }
      __syncwarp();
    }
    // The last two tiles' commits on empty[] have arrived before the CTA
    // leaves (those phases are the newest of their barriers).
    for (int kk = k - 2; ok && kk < k; kk++)
      if (kk >= 0 && !warp_wait(empty + (kk & 1), (uint32_t)(kk >> 1) & 1u)) ok = false;
  } else {
    // Epilogue warps: tile k from accumulator buffer k % 2.
    int k = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
      const int b = k & 1;
      if (!warp_wait(tfull + b, (uint32_t)(k >> 1) & 1u)) {
        ok = false;
        break;
      }
      umma::fence_after_sync();
      drain_row_tile<CO, EPI>(tmem + (uint32_t)b * S::kColsBuf, warp, lane, kPipeEpiWarps, row_tile(tile, h, w), h,
                              w, sbias, zprev, out0, out1);
      umma::fence_before_sync();
      mbar_arrive(tempty + b);
    }
  }
  if (!ok && lane == 0) atomicExch(err, PMHD_LEARNED_ERR_TIMEOUT);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, S::kTmemCols);
  }
}

template <int CIN, int CO>
struct WgradSmem {
  static constexpr int M = 9 * CIN;
  static constexpr int MT = (M + 127) / 128;           // M = 128 tiles
  static constexpr int KC = 64;                        // pixels per chunk
  static constexpr uint32_t kLboA = MT * 16u * 128u;   // K-group (8 pixels) stride of A
  static constexpr uint32_t kBytesA = (KC / 8) * kLboA;
  static constexpr uint32_t kLboB = (CO / 8) * 128u;
  static constexpr uint32_t kBytesB = (KC / 8) * kLboB;
  static constexpr uint32_t kOffBar = kBytesA + kBytesB;
  static constexpr uint32_t kBytes = kOffBar + 16u;
};

// dW[co][t][ci] += sum_p dz[p][co] * x[p + tap t][ci] over this CTA's pixel
// chunks; accumulator tile i (rows m = 128 i + lane, m = t * CIN + ci) sits
// in tensor-memory columns [32 i, 32 i + CO).
template <int CIN, int CO>
__global__ void __launch_bounds__(128) wgrad_kernel(const __nv_bfloat16* __restrict__ x,
                                                    const __nv_bfloat16* __restrict__ dz, int batch, int h, int w,
                                                    float* __restrict__ dw, int* __restrict__ err) {
  using S = WgradSmem<CIN, CO>;
  constexpr uint32_t kCols = umma::tmem_cols(32 * S::MT);
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + S::kBytesA;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S::kOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::kOffBar + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long P = (long long)batch * h * w;
  const long long nchunks = (P + S::KC - 1) / S::KC;

  if (warp == 0) {
    umma::tmem_alloc(tslot, kCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  // Rows M .. 128*MT-1 of A stay zero.
  constexpr int kPadGroups = S::MT * 16 - S::M / 8;
  for (int c = tid; c < (S::KC / 8) * kPadGroups * 8; c += 128) {
    const int kg = c / (kPadGroups * 8), r = c - kg * kPadGroups * 8;
    *reinterpret_cast<uint4*>(sA + kg * S::kLboA + (S::M / 8) * 128 + r * 16) = make_uint4(0u, 0u, 0u, 0u);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = umma::idesc_bf16(128, CO, false, false);
  const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
  uint32_t phase = 0;
  bool ok = true, any = false;
  for (long long ch = blockIdx.x; ch < nchunks && ok; ch += gridDim.x) {
    const long long p0 = ch * S::KC;
    // A: blocks of 8 pixels x 8 channels, transposed in registers so that
    // each row (one tap and channel) holds 8 consecutive pixels (K-major).
    for (int c = tid; c < 9 * (S::KC / 8) * (CIN / 8); c += 128) {
      const int g = c % (CIN / 8);
      const int kg = (c / (CIN / 8)) % (S::KC / 8);
      const int t = c / ((S::KC / 8) * (CIN / 8));
      uint4 v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        v[q] = make_uint4(0u, 0u, 0u, 0u);
        const long long p = p0 + kg * 8 + q;
        if (p < P) {
          const int x0 = (int)(p % w);
          const long long r = p / w;
          const int y0 = (int)(r % h);
          const long long b = r / h;
          const int yy = wrap(y0 + t / 3 - 1, h), xx = wrap(x0 + t % 3 - 1, w);
          v[q] = *reinterpret_cast<const uint4*>(x + ((b * h + yy) * (long long)w + xx) * CIN + g * 8);
        }
      }
#pragma unroll
      for (int ch = 0; ch < 8; ch++) {
        const int m = t * CIN + g * 8 + ch;
        *reinterpret_cast<uint4*>(sA + (m / 8) * 128 + (m % 8) * 16 + kg * S::kLboA) = transpose_row(v, ch);
      }
    }
    // B: the output gradient, the same way (rows = output channels).
    for (int c = tid; c < (S::KC / 8) * (CO / 8); c += 128) {
      const int g = c % (CO / 8), kg = c / (CO / 8);
      uint4 v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const long long p = p0 + kg * 8 + q;
        v[q] = p < P ? *reinterpret_cast<const uint4*>(dz + p * CO + g * 8) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int ch = 0; ch < 8; ch++)
        *reinterpret_cast<uint4*>(sB + g * 128 + ch * 16 + kg * S::kLboB) = transpose_row(v, ch);
    }
    fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < S::KC / 16; kk++)
#pragma unroll
        for (int i = 0; i < S::MT; i++) {
          const uint64_t da = umma::desc(a0 + i * 2048 + kk * 2 * S::kLboA, S::kLboA, 128);
          const uint64_t db = umma::desc(b0 + kk * 2 * S::kLboB, S::kLboB, 128);
          umma::mma_bf16(tmem + 32 * i, da, db, idesc, (any || kk) ? 1u : 0u);
        }
      umma::commit(bar);
    }
    __syncwarp();
    ok = wait_mma(bar, phase, err);
    phase ^= 1u;
    any = true;
    umma::fence_after_sync();
    ok = __syncthreads_and(ok);  // every warp agrees before the tiles are rewritten
  }
  if (any && ok) {
#pragma unroll 1
    for (int i = 0; i < S::MT; i++) {
      float acc[CO];
#pragma unroll
      for (int c8 = 0; c8 < CO / 8; c8++)
        umma::ld8(tmem + ((uint32_t)(warp * 32) << 16) + 32 * i + c8 * 8, acc + c8 * 8);
      const int m = 128 * i + tid;
      if (m < S::M)
#pragma unroll
        for (int co = 0; co < CO; co++) atomicAdd(dw + (size_t)co * S::M + m, acc[co]);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, kCols);
  }
}

// db[co] += sum_p dz[p][co].
template <int CO>
__global__ void __launch_bounds__(256) bias_grad_kernel(const __nv_bfloat16* __restrict__ dz, long long P,
                                                        float* __restrict__ db) {
  __shared__ float part[CO];
  if (threadIdx.x < CO) part[threadIdx.x] = 0.f;
  __syncthreads();
  const int c = threadIdx.x % CO;
  float s = 0.f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P * CO; i += (long long)gridDim.x * blockDim.x)
    s += __bfloat162float(dz[(i / CO) * CO + c]);
  atomicAdd(&part[c], s);
  __syncthreads();
  if (threadIdx.x < CO) atomicAdd(db + threadIdx.x, part[threadIdx.x]);
}

template <class K>
cudaError_t set_smem(K kernel, uint32_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

int g_sms = 0;  // SM count of the device the kernels were prepared on

// Images whose width is a multiple of 128 and height a multiple of kRows take
// the row kernels (the tile is staged once; taps are descriptor shifts) --
// the persistent pipelined one from two row tiles per SM, else one CTA per
// tile -- others the gather kernel.
template <int CG, int CO, int EPI>
cudaError_t launch_conv(const __nv_bfloat16* x, int batch, int h, int w, const __nv_bfloat16* wt, const float* bias,
                        const __nv_bfloat16* zprev, void* out0, void* out1, int* err, cudaStream_t s) {
  if (w % kRowPix == 0 && h % kRows == 0) {
    const long long tiles = (long long)batch * (h / kRows) * (w / kRowPix);
    const int sms = g_sms > 0 ? g_sms : 148;
    // Test hook: PMHD_CONV_MAX_CTAS > 0 selects the persistent kernel on any
    // row shape with at most that many CTAs, so small images still give each
    // CTA several tiles (both buffers reused, barrier phases flipping).
    const char* hook_env = getenv("PMHD_CONV_MAX_CTAS");
    const long long hook = hook_env ? atoll(hook_env) : 0;
    if (hook > 0 || tiles >= 2LL * sms) {
      // Persistent, pipelined: pays off from two tiles per SM (8 x 512^2:
      // 210 -> 182 us); one tile per CTA gains nothing from the pipeline.
      long long grid = tiles < sms ? tiles : sms;
      if (hook > 0 && grid > hook) grid = hook;
      conv3x3_pipe_kernel<CG, CO, EPI><<<(unsigned)grid, kPipeThreads, PipeSmem<CG, CO>::kLaunchBytes, s>>>(
          x, wt, bias, zprev, batch, h, w, out0, out1, err);
      return cudaGetLastError();
    }
    const long long ctas = (long long)batch * (h / kRows) * (w / kRowPix);
    conv3x3_rows_kernel<CG, CO, EPI><<<(unsigned)ctas, kRowThreads, RowSmem<CG, CO>::kLaunchBytes, s>>>(
        x, wt, bias, zprev, batch, h, w, out0, out1, err);
    return cudaGetLastError();
  }
  using S = ConvSmem<CG, CO>;
  auto k = conv3x3_kernel<CG, CO, EPI>;
  const long long P = (long long)batch * h * w;
  const unsigned grid = (unsigned)((P + 127) / 128);
  k<<<grid, 128, S::kBytes, s>>>(x, wt, bias, zprev, batch, h, w, out0, out1, err);
  return cudaGetLastError();
}

template <int CIN, int CO>
cudaError_t launch_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dz, int batch, int h, int w, float* dw,
                         float* db, int* err, cudaStream_t s) {
  using S = WgradSmem<CIN, CO>;
  auto k = wgrad_kernel<CIN, CO>;
  const int sms = g_sms > 0 ? g_sms : 148;
  const long long P = (long long)batch * h * w;
  const long long nchunks = (P + S::KC - 1) / S::KC;
  // Up to 4 CTAs per SM fit both shared memory and the 512 tensor-memory
  // columns; each CTA takes several chunks so the atomics stay few.
  long long grid = nchunks < 2LL * sms ? nchunks : 2LL * sms;
  if (grid < 1) grid = 1;
  k<<<(unsigned)grid, 128, S::kBytes, s>>>(x, dz, batch, h, w, dw, err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !db) return e;
  const long long tot = P * CO;
  long long bg = (tot + 255) / 256;
  if (bg > 4LL * sms) bg = 4LL * sms;
  if (bg < 1) bg = 1;
  bias_grad_kernel<CO><<<(unsigned)bg, 256, 0, s>>>(dz, P, db);
  return cudaGetLastError();
}

}  // namespace

cudaError_t conv_prepare() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = set_smem(conv3x3_kernel<32, 32, CONV_GELU>, ConvSmem<32, 32>::kBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_kernel<32, 16, CONV_LINEAR>, ConvSmem<32, 16>::kBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_kernel<16, 32, CONV_DGELU>, ConvSmem<16, 32>::kBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_kernel<32, 32, CONV_DGELU>, ConvSmem<32, 32>::kBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_rows_kernel<32, 32, CONV_GELU>, RowSmem<32, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_pipe_kernel<32, 32, CONV_GELU>, PipeSmem<32, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_rows_kernel<32, 16, CONV_LINEAR>, RowSmem<32, 16>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_pipe_kernel<32, 16, CONV_LINEAR>, PipeSmem<32, 16>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_rows_kernel<16, 32, CONV_DGELU>, RowSmem<16, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_pipe_kernel<16, 32, CONV_DGELU>, PipeSmem<16, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_rows_kernel<32, 32, CONV_DGELU>, RowSmem<32, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(conv3x3_pipe_kernel<32, 32, CONV_DGELU>, PipeSmem<32, 32>::kLaunchBytes);
  if (e == cudaSuccess) e = set_smem(wgrad_kernel<32, 32>, WgradSmem<32, 32>::kBytes);
  if (e == cudaSuccess) e = set_smem(wgrad_kernel<32, 16>, WgradSmem<32, 16>::kBytes);
  return e;
}

cudaError_t conv3x3(int mode, const __nv_bfloat16* x, int batch, int h, int w, int c_in, const __nv_bfloat16* wt,
                    const float* bias, int c_out, const __nv_bfloat16* zprev, void* out0, void* out1, int* err,
                    cudaStream_t s) {
  if (mode == CONV_GELU && c_in == 32 && c_out == 32)
    return launch_conv<32, 32, CONV_GELU>(x, batch, h, w, wt, bias, zprev, out0, out1, err, s);
  if (mode == CONV_LINEAR && c_in == 32 && c_out == 16)
    return launch_conv<32, 16, CONV_LINEAR>(x, batch, h, w, wt, bias, zprev, out0, out1, err, s);
  if (mode == CONV_DGELU && c_in == 16 && c_out == 32)
    return launch_conv<16, 32, CONV_DGELU>(x, batch, h, w, wt, bias, zprev, out0, out1, err, s);
  if (mode == CONV_DGELU && c_in == 32 && c_out == 32)
    return launch_conv<32, 32, CONV_DGELU>(x, batch, h, w, wt, bias, zprev, out0, out1, err, s);
  return cudaErrorNotSupported;
}

cudaError_t conv3x3_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dz, int batch, int h, int w, int c_in,
                          int c_out, float* dw, float* db, int* err, cudaStream_t s) {
  if (c_in == 32 && c_out == 32) return launch_wgrad<32, 32>(x, dz, batch, h, w, dw, db, err, s);
  if (c_in == 32 && c_out == 16) return launch_wgrad<32, 16>(x, dz, batch, h, w, dw, db, err, s);
  return cudaErrorNotSupported;
}

}  // namespace learned
}  // namespace pmhd
