// problems.cpp -- host-side initial conditions, diagnostics and .dat output.
//
// Compiled with -ffp-contract=off: the Orszag-Tang and reference-KH states
// must be bit-identical to the reference's host code (same libm calls, same
// expression order) for the bit-parity mode to reproduce its output files.
#include "problems.h"

#include <cmath>
#include <cstdio>

#include "pmhd.h"
#include "pmhd/point.hpp"

namespace pmhd {

namespace {

template <class T>
T t_sin(T x) { return std::sin(x); }
template <class T>
T t_exp(T x) { return std::exp(x); }
template <class T>
T t_tanh(T x) { return std::tanh(x); }

}  // namespace

template <class T>
bool init_problem_host(const ProblemGrid& g, int problem, const double* params, int nparams, std::vector<T>& U) {
  const int nx = g.nx, ny = g.ny, G = 2, nxt = nx + 4, nyt = ny + 4;
  U.assign((size_t)nxt * nyt * 9, (T)0);
  const Phys<T> ph = Phys<T>::make(g.gamma, 0.0);
  const T x_min = (T)g.x_min, x_max = (T)g.x_max, y_min = (T)g.y_min, y_max = (T)g.y_max;
  const T dx = (x_max - x_min) / (T)nx;
  const T dy = (y_max - y_min) / (T)ny;
  // Constants as in mhd2d_glm_gpu.cu:398-400.
  const T pi = std::acos((T)-1.0);
  const T two_pi = (T)2.0 * pi;
  const T inv_sqrt_4pi = (T)1.0 / std::sqrt((T)4.0 * pi);
  auto par = [&](int k, double d) { return (params && nparams > k) ? params[k] : d; };
  const T b0 = (T)par(0, 1.0);                 // Orszag-Tang field factor
  const T width = (T)par(0, 0.05);             // KH_REFLECT shear width
  const T kh_bx = (T)par(1, 0.1);              // KH_REFLECT parallel field
  const double angle = par(0, 0.0);            // BRIO_WU_2D interface angle
  const T cth = (T)std::cos(angle), sth = (T)std::sin(angle);
  // BRIO_WU_TORUS: band slope k/m; unit normal and tangent of the bands.
  const double kb = par(0, 1.0), mb = par(1, 2.0);
  if (problem == PMHD_PROBLEM_BRIO_WU_TORUS &&
      (kb < 0 || mb < 0 || kb != std::floor(kb) || mb != std::floor(mb) || kb + mb == 0 || kb > 64 || mb > 64))
    return false;
  const double nxb = mb / (g.x_max - g.x_min), nyb = kb / (g.y_max - g.y_min);
  const double nlen = std::sqrt(nxb * nxb + nyb * nyb);
  const T bnx = (T)(nxb / nlen), bny = (T)(nyb / nlen);
  // Band edges at phases 1/(4 n) and 1/2 + 1/(4 n), n = max(nx, ny): on a
  // square grid with even n no cell centre lies on an edge.
  const double phase0 = 0.25 / (double)(nx > ny ? nx : ny);
  for (int j = 0; j < nyt; j++) {
    for (int i = 0; i < nxt; i++) {
      const T x = x_min + ((T)(i - G) + (T)0.5) * dx;
      const T y = y_min + ((T)(j - G) + (T)0.5) * dy;
      T P[9];
      switch (problem) {
        case PMHD_PROBLEM_ORSZAG_TANG:  // mhd2d_glm_gpu.cu:443-451
          P[0] = (T)25.0 / ((T)36.0 * pi);
          P[1] = -t_sin(two_pi * y);
          P[2] = t_sin(two_pi * x);
          P[3] = (T)0.0;
          P[4] = (T)5.0 / ((T)12.0 * pi);
          P[5] = -t_sin(two_pi * y) * inv_sqrt_4pi;
          P[6] = t_sin((T)2.0 * two_pi * x) * inv_sqrt_4pi;
          if (b0 != (T)1.0) {
            P[5] = P[5] * b0;
            P[6] = P[6] * b0;
          }
          P[7] = (T)0.0;
          P[8] = (T)0.0;
          break;
        case PMHD_PROBLEM_KH_REF: {  // mhd2d_glm_gpu.cu:421-441
          // params[0]: the shear-layer width (the reference's 0.025 when absent).
          const T a = (params && nparams > 0) ? (T)params[0] : (T)0.025, sigma = (T)0.05, delta = (T)0.01;
          const T S = (T)0.5 * (t_tanh((y - (T)0.25) / a) - t_tanh((y - (T)0.75) / a));
          const T g1 = (y - (T)0.25) / sigma;
          const T g2 = (y - (T)0.75) / sigma;
          P[0] = (T)1.0 + S;
          P[1] = -(T)0.5 + S;
          P[2] = delta * t_sin((T)2.0 * two_pi * x) * (t_exp(-(T)0.5 * g1 * g1) + t_exp(-(T)0.5 * g2 * g2));
          P[3] = (T)0.0;
          P[4] = (T)2.5;
          P[5] = (T)0.2;
          P[6] = (T)0.0;
          P[7] = (T)0.0;
          P[8] = (T)0.0;
          break;
        }
        case PMHD_PROBLEM_KH_REFLECT:  // single shear layer on [0,1] x [-1,1]
          P[0] = (T)1.0;
          P[1] = (T)0.5 * t_tanh(y / width);
          P[2] = (T)0.01 * t_sin(two_pi * x) * t_exp(-y * y / (T)0.01);
          P[3] = (T)0.0;
          P[4] = (T)1.0;
          P[5] = kh_bx;
          P[6] = (T)0.0;
          P[7] = (T)0.0;
          P[8] = (T)0.0;
          break;
        case PMHD_PROBLEM_BRIO_WU_2D: {  // mhd1d_cpu.cpp:283-295 states, rotated
          const T s = (x - (T)0.5 * (x_min + x_max)) * cth + (y - (T)0.5 * (y_min + y_max)) * sth;
          const bool left = s < (T)0.0;
          const T bn = (T)0.75, bt = left ? (T)1.0 : (T)-1.0;
          P[0] = left ? (T)1.0 : (T)0.125;
          P[1] = (T)0.0;
          P[2] = (T)0.0;
          P[3] = (T)0.0;
          P[4] = left ? (T)1.0 : (T)0.1;
          P[5] = bn * cth - bt * sth;
          P[6] = bn * sth + bt * cth;
          P[7] = (T)0.0;
          P[8] = (T)0.0;
          break;
        }
        case PMHD_PROBLEM_BRIO_WU_TORUS: {  // mhd1d_cpu.cpp:283-295 states in periodic bands
          const double xc = g.x_min + ((i - G) + 0.5) * (g.x_max - g.x_min) / nx;
          const double yc = g.y_min + ((j - G) + 0.5) * (g.y_max - g.y_min) / ny;
          double phs = mb * (xc - g.x_min) / (g.x_max - g.x_min) + kb * (yc - g.y_min) / (g.y_max - g.y_min) - phase0;
          phs -= std::floor(phs);
          const bool left = phs < 0.5;
          const T bn = (T)0.75, bt = left ? (T)1.0 : (T)-1.0;
          P[0] = left ? (T)1.0 : (T)0.125;
          P[1] = (T)0.0;
          P[2] = (T)0.0;
          P[3] = (T)0.0;
          P[4] = left ? (T)1.0 : (T)0.1;
          P[5] = bn * bnx - bt * bny;
          P[6] = bn * bny + bt * bnx;
          P[7] = (T)0.0;
          P[8] = (T)0.0;
          break;
        }
        default:
          return false;
      }
      prim9_to_state<T>(P, &U[((size_t)j * nxt + i) * 9], ph);
    }
  }
  return true;
}

template <class T>
void diagnostics_host(const ProblemGrid& g, const std::vector<T>& U, double out[3]) {
  // mhd2d_glm_gpu.cu:556-572
  const int nx = g.nx, ny = g.ny, nxt = nx + 4;
  const T dx = ((T)g.x_max - (T)g.x_min) / (T)nx;
  const T dy = ((T)g.y_max - (T)g.y_min) / (T)ny;
  auto at = [&](int i, int j, int k) { return U[((size_t)j * nxt + i) * 9 + k]; };
  T l1 = (T)0.0, linf = (T)0.0, plinf = (T)0.0;
  for (int j = 2; j < ny + 2; j++)
    for (int i = 2; i < nx + 2; i++) {
      const T divb = (at(i + 1, j, BX) - at(i - 1, j, BX)) / ((T)2.0 * dx) +
                     (at(i, j + 1, BY) - at(i, j - 1, BY)) / ((T)2.0 * dy);
      l1 += vabs(divb);
      linf = vmax(linf, vabs(divb));
      plinf = vmax(plinf, vabs(at(i, j, PSI)));
    }
  l1 /= (T)(nx * ny);
  out[0] = (double)l1;
  out[1] = (double)linf;
  out[2] = (double)plinf;
}

template <class T>
bool write_dat_body(std::FILE* f, const ProblemGrid& g, const std::vector<T>& U) {
  // mhd2d_glm_gpu.cu:628-647: scientific with max_digits10 digits
  const int nx = g.nx, ny = g.ny, nxt = nx + 4;
  const Phys<T> ph = Phys<T>::make(g.gamma, 0.0);
  const T x_min = (T)g.x_min, y_min = (T)g.y_min;
  const T dx = ((T)g.x_max - x_min) / (T)nx;
  const T dy = ((T)g.y_max - y_min) / (T)ny;
  const char* fmt = sizeof(T) == 8 ? "%.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n"
                                   : "%.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e\n";
  auto at = [&](int i, int j, int k) { return U[((size_t)j * nxt + i) * 9 + k]; };
  for (int j = 2; j < ny + 2; j++)
    for (int i = 2; i < nx + 2; i++) {
      const T* c = &U[((size_t)j * nxt + i) * 9];
      T W[9];
      cons_to_prim<T, 0>(c, W, ph);
      const T x = x_min + ((T)(i - 2) + (T)0.5) * dx;
      const T y = y_min + ((T)(j - 2) + (T)0.5) * dy;
      const T divb = (at(i + 1, j, BX) - at(i - 1, j, BX)) / ((T)2.0 * dx) +
                     (at(i, j + 1, BY) - at(i, j - 1, BY)) / ((T)2.0 * dy);
      if (std::fprintf(f, fmt, (double)x, (double)y, (double)W[0], (double)W[1], (double)W[2], (double)W[3],
                       (double)W[4], (double)W[5], (double)W[6], (double)W[7], (double)c[EN], (double)divb,
                       (double)c[PSI]) < 0)
        return false;
    }
  return true;
}

template bool init_problem_host<double>(const ProblemGrid&, int, const double*, int, std::vector<double>&);
template bool init_problem_host<float>(const ProblemGrid&, int, const double*, int, std::vector<float>&);
template void diagnostics_host<double>(const ProblemGrid&, const std::vector<double>&, double[3]);
template void diagnostics_host<float>(const ProblemGrid&, const std::vector<float>&, double[3]);
template bool write_dat_body<double>(std::FILE*, const ProblemGrid&, const std::vector<double>&);
template bool write_dat_body<float>(std::FILE*, const ProblemGrid&, const std::vector<float>&);

}  // namespace pmhd
