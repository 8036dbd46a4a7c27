// euler2d_gpu -- drop-in replacement for the reference's shock-bubble
// program (src/euler/euler2d_cuda.cu, main at :290-392; its serial twin is
// src/euler/euler2d_cpu.cpp), running on libpmhd.so.
//
//   euler2d_gpu            (no arguments, as the reference)
//
// Haas-Sturtevant shock-bubble: a Mach 1.22 shock in air meets a helium
// bubble; 500 x 197 cells of 0.225 x 0.089 m, MUSCL-Hancock + HLLC, CFL 0.8,
// transmissive walls, to t = 0.0011741 s.  The same stdout lines as the
// reference's CUDA program (grid, domain, end time, the shock states, a
// progress line every 100 steps, "Done. Steps:", "Execution Time:", "Saved")
// and the same .dat file $OUTDIR/gpu_shock_bubble.dat (default
// results/euler/2d/<fp64|fp32>): a "# Time" line, then "x y rho u v p" per
// cell in scientific notation with max_digits10 digits, x outermost, a blank
// line after each column.
//
// The reference builds one binary per precision; here the program name
// picks it ("_fp32": binary32, anything else binary64) and PMHD_PRECISION
// (fp64|fp32) overrides it.  PMHD_EXACT=1 selects the kernels built without
// FMA contraction, whose data lines equal the reference CPU program's bit for
// bit (the reference's CUDA program takes its time step as CFL / max(...)
// instead of CFL * min(...) and is compiled with contraction, so its own bits
// differ from both).  Exit codes as the reference's: 0, and 1 (EXIT_FAILURE,
// its CUDA_CHECK) when the device cannot be used or a CUDA call fails; like
// the reference, an output file that cannot be written is reported and the
// program still exits 0.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "pmhd.h"

namespace {

constexpr int kNx = 500, kNy = 197;
constexpr double kTEnd = 0.0011741;

bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

// euler2d_cuda.cu:365-392 (writeOutput): cell centres are binary64
// expressions of the compile-time constants, stored in the run's type.
template <class T>
bool write_dat(const std::string& path, const std::vector<T>& w, T t) {
  std::ofstream out(path);
  if (!out) return false;
  out << "# Time = " << t << "\n";
  out << std::scientific;
  out.precision(std::numeric_limits<T>::max_digits10);
  const T dx = (T)(0.225 - 0.0) / (T)kNx, dy = (T)(0.089 - 0.0) / (T)kNy;
  for (int i = 0; i < kNx; i++) {
    const T x = (T)(0.0 + (i + 0.5) * (double)dx);
    for (int j = 0; j < kNy; j++) {
      const T y = (T)(0.0 + (j + 0.5) * (double)dy);
      const T* c = &w[((size_t)j * kNx + i) * 4];
      out << x << " " << y << " " << c[0] << " " << c[1] << " " << c[2] << " " << c[3] << "\n";
    }
    out << "\n";
  }
  return (bool)out;
}

}  // namespace

int main(int argc, char* argv[]) {
  (void)argc;
  int precision = ends_with(argv[0], "_fp32") ? PMHD_FP32 : PMHD_FP64;
  if (const char* e = std::getenv("PMHD_PRECISION")) {
    const std::string v = e;
    if (v == "fp32") precision = PMHD_FP32;
    else if (v == "fp64") precision = PMHD_FP64;
  }
  const char* ex = std::getenv("PMHD_EXACT");
  const int exact = ex && std::atoi(ex) != 0;
  const bool fp32 = precision == PMHD_FP32;

  std::printf("Grid: %d x %d (with %d ghost -> %d x %d)\n", kNx, kNy, 2, kNx + 4, kNy + 4);
  std::printf("Domain: x=[%.3f, %.3f], y=[%.3f, %.3f]\n", 0.0, 0.225, 0.0, 0.089);
  std::printf("T_end = %.7f s\n\n", kTEnd);
  // The shock states as the reference prints them (euler2d_cuda.cu:231-243).
  {
    const double g = 1.4, M = 1.22, rho1 = 1.29, p1 = 101325.0;
    const double c1 = std::sqrt(g * p1 / rho1);
    const double rho2 = rho1 * ((g + 1) * M * M) / ((g - 1) * M * M + 2);
    const double p2 = p1 * (2 * g * M * M - (g - 1)) / (g + 1);
    const double u2 = c1 * M * (1.0 - rho1 / rho2);
    std::printf("===== Shock-Bubble Problem (CUDA) =====\n");
    std::printf("Pre-shock:  rho=%.4f, p=%.1f\n", rho1, p1);
    std::printf("Post-shock: rho=%.4f, p=%.1f, u=%.4f\n", rho2, p2, u2);
    std::printf("=======================================\n");
  }

  pmhd_euler2d* e = nullptr;
  int rc = pmhd_euler2d_create(kNx, kNy, PMHD_EULER_SHOCK_BUBBLE, PMHD_SOLVER_HLLC, precision, exact, 0, &e);
  if (rc != PMHD_OK) {
    std::fprintf(stderr, "pmhd_euler2d_create: %s\n", pmhd_strerror(rc));
    return EXIT_FAILURE;
  }
  std::printf("Starting CUDA simulation...\n");
  const auto t0 = std::chrono::high_resolution_clock::now();
  pmhd_euler_stats st{};
  long long printed = 0;
  // Chunks of 100 steps, so the progress line comes every 100 steps as in
  // the reference (the end of the run stops a chunk early).
  for (;;) {
    const long long before = st.steps;
    rc = pmhd_euler2d_advance(e, -1.0, 100, &st);
    if (rc != PMHD_OK) break;
    if (st.steps % 100 == 0 && st.steps > printed) {
      std::printf("Step %lld: t = %.6e\n", st.steps, st.t);
      printed = st.steps;
    }
    if (st.steps - before < 100) break;
  }
  const auto t1 = std::chrono::high_resolution_clock::now();
  if (rc != PMHD_OK) {
    std::fprintf(stderr, "pmhd_euler2d_advance: %s\n", pmhd_strerror(rc));
    pmhd_euler2d_destroy(e);
    return EXIT_FAILURE;
  }
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("\nDone. Steps: %lld\n", st.steps);
  std::printf("Execution Time: %.2f ms (%.4f s)\n", ms, ms / 1000.0);

  const char* prec_name = fp32 ? "fp32" : "fp64";
  const char* out_env = std::getenv("OUTDIR");
  const std::string out_dir = out_env ? std::string(out_env) : std::string("results/euler/2d/") + prec_name;
  std::string cmd = "mkdir -p '" + out_dir + "' 2>/dev/null";
  if (std::system(cmd.c_str()) != 0) {
    // The reference ignores this too; the open below reports it.
  }
  std::ostringstream fname;
  fname << out_dir << "/gpu_shock_bubble.dat";
  bool ok = false;
  if (fp32) {
    std::vector<float> w((size_t)kNx * kNy * 4);
    ok = pmhd_euler2d_get_prim(e, w.data()) == PMHD_OK && write_dat<float>(fname.str(), w, (float)st.t);
  } else {
    std::vector<double> w((size_t)kNx * kNy * 4);
    ok = pmhd_euler2d_get_prim(e, w.data()) == PMHD_OK && write_dat<double>(fname.str(), w, st.t);
  }
  if (!ok) std::fprintf(stderr, "could not write %s\n", fname.str().c_str());
  std::printf("Saved %s (t=%.6e)\n", fname.str().c_str(), st.t);
  pmhd_euler2d_destroy(e);
  return 0;
}
