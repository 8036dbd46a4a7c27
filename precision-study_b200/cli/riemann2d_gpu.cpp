// riemann2d_gpu -- drop-in replacement for the reference's 2D Riemann
// program (src/euler/riemann2d_gpu.cu, main at :323-470; its serial twin is
// src/euler/riemann2d_cpu.cpp), running on libpmhd.so.
//
//   riemann2d_gpu [N [config_id]]
//
// Liska-Wendroff configuration 3, 6 or 12 (default 6) on an N x N grid of
// [0,1]^2 (default 400), MUSCL-Hancock + HLLC, CFL 0.8, transmissive walls,
// dimensionally split steps alternating x-y / y-x, to the configuration's end
// time.  The same stdout lines as the reference's GPU program (the header, a
// progress line every 200 steps, "Done. Steps: ...   Wall: ... s",
// "Saved: ...") and the same .dat file
// $OUTDIR/riemann2d_<config name>_hllc_<N>.dat (default
// results/euler/2d/<fp64|fp32>/gpu): "x y rho u v p" per cell in scientific
// notation with max_digits10 digits, y outermost, no header.
//
// The program name picks the precision ("_fp32": binary32, anything else
// binary64; PMHD_PRECISION overrides).  PMHD_EXACT=1 selects the kernels built
// without FMA contraction, whose output equals the reference CPU program's
// bit for bit (the reference's GPU program takes its time step as
// CFL / max(...) instead of CFL * min(...) and is compiled with contraction,
// so its own bits differ from both).  Exit codes as the reference's: 1 for a
// bad configuration id and when the device cannot be used or a CUDA call
// fails (its CUDA_CHECK), else 0.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "pmhd.h"

namespace {

bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

// riemann2d_cpu.cpp:56-79: names and end times of the configurations.
const char* config_name(int id) {
  return id == 3 ? "cfg3_4shocks" : id == 6 ? "cfg6_4contacts" : id == 12 ? "cfg12_2S2C" : nullptr;
}

// riemann2d_gpu.cu:299-318 (writeOutput2D): y outermost, cell centres in the
// run's type.
template <class T>
bool write_dat(const std::string& path, const std::vector<T>& w, int n) {
  std::ofstream out(path);
  if (!out) return false;
  out << std::scientific;
  out.precision(std::numeric_limits<T>::max_digits10);
  const T dx = ((T)1.0 - (T)0.0) / (T)n;
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < n; i++) {
      const T x = (T)0.0 + (T)(i + 0.5) * dx;
      const T y = (T)0.0 + (T)(j + 0.5) * dx;
      const T* c = &w[((size_t)j * n + i) * 4];
      out << x << " " << y << " " << c[0] << " " << c[1] << " " << c[2] << " " << c[3] << "\n";
    }
  }
  return (bool)out;
}

template <class T>
int run(int n, int cfg_id, bool exact, const char* prec_name) {
  const T dx = ((T)1.0 - (T)0.0) / (T)n;
  const T t_end = cfg_id == 12 ? (T)0.25 : (T)0.3;
  std::cout << "===== 2D Riemann GPU =====\n"
            << "Config:    " << config_name(cfg_id) << "  (id=" << cfg_id << ")\n"
            << "Solver:    HLLC\n"
            << "Precision: " << prec_name << "\n"
            << "Grid:      " << n << " x " << n << "  dx=" << dx << "\n"
            << "T_end:     " << t_end << "\n";
  std::cout.flush();
  pmhd_euler2d* e = nullptr;
  int rc = pmhd_euler2d_create(n, n, cfg_id, PMHD_SOLVER_HLLC, sizeof(T) == 4 ? PMHD_FP32 : PMHD_FP64, exact ? 1 : 0,
                               0, &e);
  if (rc != PMHD_OK) {
    std::fprintf(stderr, "pmhd_euler2d_create: %s\n", pmhd_strerror(rc));
    return EXIT_FAILURE;
  }
  const auto t0 = std::chrono::high_resolution_clock::now();
  pmhd_euler_stats st{};
  // Chunks of 200 steps for the reference's progress line.
  for (;;) {
    const long long before = st.steps;
    rc = pmhd_euler2d_advance(e, -1.0, 200, &st);
    if (rc != PMHD_OK) break;
    if (st.steps - before == 200) std::cout << "Step " << st.steps << ": t = " << (T)st.t << "\n";
    if (st.steps - before < 200) break;
  }
  const auto t1 = std::chrono::high_resolution_clock::now();
  if (rc != PMHD_OK) {
    std::fprintf(stderr, "pmhd_euler2d_advance: %s\n", pmhd_strerror(rc));
    pmhd_euler2d_destroy(e);
    return EXIT_FAILURE;
  }
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::cout << "Done. Steps: " << st.steps << "   Wall: " << ms / 1000.0 << " s\n";
  const char* out_env = std::getenv("OUTDIR");
  const std::string out_dir =
      out_env ? std::string(out_env) : std::string("results/euler/2d/") + prec_name + "/gpu";
  const std::string cmd = "mkdir -p '" + out_dir + "' 2>/dev/null";
  if (std::system(cmd.c_str()) != 0) {
    // The reference ignores this too; the open below reports it.
  }
  std::ostringstream fname;
  fname << out_dir << "/riemann2d_" << config_name(cfg_id) << "_hllc_" << n << ".dat";
  std::vector<T> w((size_t)n * n * 4);
  const bool ok = pmhd_euler2d_get_prim(e, w.data()) == PMHD_OK && write_dat<T>(fname.str(), w, n);
  if (!ok) std::fprintf(stderr, "could not write %s\n", fname.str().c_str());
  std::cout << "Saved: " << fname.str() << "\n";
  pmhd_euler2d_destroy(e);
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  int n = 400, cfg_id = 6;
  if (argc > 1) n = std::atoi(argv[1]);
  if (argc > 2) cfg_id = std::atoi(argv[2]);
  if (!config_name(cfg_id)) {
    std::cerr << "Error: config_id must be 3, 6, or 12\n";
    return 1;
  }
  bool fp32 = ends_with(argv[0], "_fp32");
  if (const char* p = std::getenv("PMHD_PRECISION")) {
    const std::string v = p;
    if (v == "fp32") fp32 = true;
    else if (v == "fp64") fp32 = false;
  }
  const char* ex = std::getenv("PMHD_EXACT");
  const bool exact = ex && std::atoi(ex) != 0;
  return fp32 ? run<float>(n, cfg_id, exact, "fp32") : run<double>(n, cfg_id, exact, "fp64");
}
