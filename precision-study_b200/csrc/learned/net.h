// net.h -- the learned coarse-grid correction's non-convolution kernels
// (net.cu): features and targets from solver states, loss, Adam, restriction
// of fine states, and the checked application of a correction.
#ifndef PMHD_LEARNED_NET_H
#define PMHD_LEARNED_NET_H

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace pmhd {
namespace learned {

constexpr int kNVar = 9;
constexpr int kFeat = 32;   // input channels (18 used: state and step increment)
constexpr int kWidth = 32;  // hidden channels
constexpr int kOut = 16;    // output channels (8 used: the correction, see Out)
constexpr int kLayers = 4;  // 3x3 layers: 3 x (32 -> 32, GELU), 32 -> 16 linear

// Output channels: the correction in quantities that keep it physical.
//   OUT_LRHO / OUT_LP  log(rho_new / rho), log(p_new / p): positive by
//                      construction;
//   OUT_V..OUT_V+2     velocity increments;
//   OUT_A              a vector potential A_z: the field changes by its
//                      central-difference curl (dBx = dA/dy, dBy = -dA/dx), which
//                      leaves the central-difference div B unchanged;
//   OUT_BZ, OUT_PSI    increments of B_z and psi.
// Target channels 8 and 9 hold the field change (dBx, dBy) the curl of OUT_A
// is trained against.
enum Out : int { OUT_LRHO = 0, OUT_V = 1, OUT_LP = 4, OUT_A = 5, OUT_BZ = 6, OUT_PSI = 7, TGT_DBX = 8, TGT_DBY = 9 };
constexpr int kNOutQ = 10;  // target quantities (channels 0..9; 5 unused)

// fp64 state of `batch` grids: variable k of interior cell (i, j) of grid b at
// u[offset + b*bstride + k*vstride + j*jstride + i*istride].
struct StateView {
  const double* u;
  long long offset, bstride, vstride, jstride, istride;
};

inline StateView soa_view(const void* u, int pitch, long long plane) {
  return StateView{static_cast<const double*>(u), 2LL * pitch + 2, 0, plane, pitch, 1};
}
inline StateView aos_view(const void* u, int nx, int ny) {
  return StateView{static_cast<const double*>(u), 0, (long long)nx * ny * kNVar, 1, (long long)nx * kNVar, kNVar};
}

// Normalisation of the network's inputs and outputs.
struct Norm {
  float mu[2 * kNVar], inv_sig[2 * kNVar];  // features: state, step increment
  // Scale of each target quantity (0 / 0: not corrected).  For OUT_A the scale
  // is that of the potential, sig_out[TGT_DBX] * min(dx, dy).
  float sig_out[kNOutQ], inv_out[kNOutQ];
  // curl of the normalised potential in normalised field units:
  // dBx_n = cy * (A_n[j+1] - A_n[j-1]), dBy_n = -cx * (A_n[i+1] - A_n[i-1]).
  float cx, cy;
};

// Four 3x3 layers: 32 -> 32 -> 32 -> 32 (GELU) -> 16 (linear).
struct NetLayout {
  int w_off[kLayers], b_off[kLayers];  // offsets into the fp32 parameter vector
  int cin[kLayers], cout[kLayers];
  int n_params;
};
NetLayout net_layout();

// Device pointers of one set of network weights.
struct NetWeights {
  float* theta;                  // fp32 parameters (weights then bias per layer)
  __nv_bfloat16* wf[kLayers];    // bf16 [cout][9][cin] (forward)
  __nv_bfloat16* wb[kLayers];    // bf16 [cin][9][cout] (backward to the input)
};

// Per-step work of a corrected run.
// Conserved quantities whose correction is made mean-free over the periodic
// grid: rho, the three momenta, E, B_z (B_x and B_y change by a curl, whose
// mean is zero already).
constexpr int kNConserved = 6;
constexpr int kCorrSums = 2 + kNConserved;

struct CorrState {
  double* before;      // SoA copy of the state before the step (solver layout)
  double* cand;        // AoS interior candidate state
  __nv_bfloat16* x;    // features [ny][nx][32]
  __nv_bfloat16* z1, *a1, *z2, *a2, *z3, *a3;
  float* out;          // network output [ny][nx][16]
  // flags[0]: candidate not positive; sums[0..1]: ||divB||_1 after the step
  // and of the candidate, sums[2 + k]: domain sum of the candidate's change
  // of conserved quantity kConserved[k] (kCorrSums doubles); counters[0..2]:
  // accepted, rejected (positivity), rejected (divergence); accept: this
  // step's decision.
  int* flags;
  double* sums;
  unsigned long long* counters;
  int* accept;
  const Norm* norm;    // device copy
  double relax;        // fraction of the predicted correction applied
  double shrink;       // soft threshold on the normalised outputs
};

cudaError_t features(const StateView& after, const StateView& before, int batch, int nx, int ny, const Norm* norm,
                     __nv_bfloat16* x, cudaStream_t s);
// Normalised target quantities (Out) of the step from `after` to `fine`.
cudaError_t targets(const StateView& after, const StateView& fine, int batch, int nx, int ny, const Norm* norm,
                    double gamma, float* tgt, cudaStream_t s);
// sums[0..17] += per-variable sums of (after, after - before), sums[18..35]
// += their squares; sums[36..45] += sums of the target quantities (Out,
// unnormalised) from `after` to `fine`, sums[46..55] += their squares.
constexpr int kMomentSums = 56;
cudaError_t moments(const StateView& before, const StateView& after, const StateView& fine, int batch, int nx,
                    int ny, double gamma, double* sums, cudaStream_t s);
// Mean squared error over the target quantities (the field through the curl
// of OUT_A, periodic on each nx x ny image of the batch) and its gradient
// with respect to the output.
cudaError_t loss_grad(const float* out, const float* tgt, int batch, int nx, int ny, const Norm* norm,
                      __nv_bfloat16* dz, float* loss_hist, const int* it, cudaStream_t s);
cudaError_t adam(const NetLayout& L, NetWeights w, float* grad, float* m, float* v, const int* it, int iters,
                 float lr, cudaStream_t s);
cudaError_t weights_to_bf16(const NetLayout& L, NetWeights w, cudaStream_t s);
cudaError_t gather_pairs(const int* schedule, const int* it, int batch, const __nv_bfloat16* feat_all,
                         const float* tgt_all, long long pix_per_pair, __nv_bfloat16* feat, float* tgt,
                         cudaStream_t s);
cudaError_t increment(int* it, cudaStream_t s);
// Adds N(0, sigma^2) to the used input channels (0 .. 2 * kNVar - 1) of P
// pixels of a feature batch; the draws depend on (seed, *it, element).
cudaError_t input_noise(__nv_bfloat16* x, long long P, float sigma, const int* it, unsigned long long seed,
                        cudaStream_t s);
// Block average of a fine SoA state (factor r) into a coarse AoS interior.
cudaError_t restrict_state(const void* fine_u, int fpitch, long long fplane, int fnx, int fny, int r, double* coarse,
                           cudaStream_t s);
// AoS interior -> solver SoA with periodic ghost cells.
cudaError_t load_periodic(const double* aos, void* u, int pitch, long long plane, int nx, int ny, cudaStream_t s);
// Solver SoA interior -> AoS interior.
cudaError_t store_interior(const void* u, int pitch, long long plane, int nx, int ny, double* aos, cudaStream_t s);

// The correction of one step at parity p: candidate, checks, decision,
// commit (see net.cu); ctrl tells whether the step was taken.
cudaError_t correct_step(const CorrState& cs, void* u, int pitch, long long plane, int nx, int ny, double dx,
                         double dy, double gamma, double div_tol, const Ctrl* ctrl, Ctrl* ctrl_w, int p,
                         cudaStream_t s);

}  // namespace learned
}  // namespace pmhd

#endif  // PMHD_LEARNED_NET_H
