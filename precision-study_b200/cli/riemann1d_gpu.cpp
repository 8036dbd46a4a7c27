// riemann1d_gpu -- drop-in replacement for the reference's 1D Riemann
// program (src/euler/riemann1d_gpu.cu, main at :206-325; its serial twin is
// src/euler/riemann1d_cpu.cpp), running on libpmhd.so.
//
//   riemann1d_gpu [N [test_id [hllc|hll]]]
//
// Toro's test `test_id` (1-5, default 1) on N cells of [0,1] (default 200),
// MUSCL-Hancock + HLLC or HLL, CFL 0.8, transmissive ends, to the test's end
// time -- the whole run is one kernel launch.  The same stdout lines as the
// reference's GPU program (the header, "Done. Steps:", "Saved:") and the same
// .dat file $OUTDIR/toro<id>_<solver>_<fp64|fp32>_<N>.dat (default
// results/euler/gpu/<fp64|fp32>): "x rho u p" per cell in scientific
// notation with max_digits10 digits.
//
// The program name picks the precision ("_fp32": binary32, anything else
// binary64; PMHD_PRECISION overrides).  PMHD_EXACT=1 selects the kernels built
// without FMA contraction, whose output equals the reference CPU program's
// bit for bit.  Exit codes as the reference's: 1 for a bad test id, an output
// file that cannot be opened, or when the device cannot be used or a CUDA
// call fails (its CUDA_CHECK), else 0.
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

// riemann1d_gpu.cu:45-66: Toro's table 4.1 names.
const char* const kTestNames[5] = {"Sod", "123_problem", "Left_blast", "Right_blast", "Two_shocks"};

template <class T>
int run(int n, int test_id, const std::string& solver, bool exact, const char* prec_name) {
  const bool hll = solver == "hll" || solver == "HLL";
  const T dx = ((T)1.0 - (T)0.0) / (T)n;
  std::cout << "===== 1D Riemann GPU =====\n"
            << "Test:      " << kTestNames[test_id - 1] << "  (id=" << test_id << ")\n"
            << "Solver:    " << (hll ? "HLL" : "HLLC") << "\n"
            << "Precision: " << prec_name << "\n"
            << "N=" << n << "  dx=" << dx << "\n";
  std::cout.flush();
  std::vector<T> w((size_t)n * 3);
  pmhd_euler_stats st{};
  const int rc = pmhd_euler1d_run(n, test_id, hll ? PMHD_SOLVER_HLL : PMHD_SOLVER_HLLC,
                                  sizeof(T) == 4 ? PMHD_FP32 : PMHD_FP64, exact ? 1 : 0, 0, w.data(), &st);
  if (rc != PMHD_OK) {
    std::fprintf(stderr, "pmhd_euler1d_run: %s\n", pmhd_strerror(rc));
    return EXIT_FAILURE;
  }
  std::cout << "Done. Steps: " << st.steps << "\n";
  const char* out_env = std::getenv("OUTDIR");
  const std::string dir = out_env ? std::string(out_env) : std::string("results/euler/gpu/") + prec_name;
  const std::string cmd = "mkdir -p '" + dir + "' 2>/dev/null";
  if (std::system(cmd.c_str()) != 0) {
    // The reference ignores this too; the open below reports it.
  }
  std::ostringstream fname;
  fname << dir << "/toro" << test_id << "_" << solver << "_" << prec_name << "_" << n << ".dat";
  std::ofstream out(fname.str());
  if (!out) {
    std::cerr << "Cannot open: " << fname.str() << "\n";
    return 1;
  }
  out << std::scientific;
  out.precision(std::numeric_limits<T>::max_digits10);
  for (int i = 0; i < n; i++) {
    const T x = (T)0.0 + (T)(i + 0.5) * dx;
    out << x << " " << w[i * 3 + 0] << " " << w[i * 3 + 1] << " " << w[i * 3 + 2] << "\n";
  }
  out.close();
  std::cout << "Saved: " << fname.str() << "\n";
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  int n = 200, test_id = 1;
  std::string solver = "hllc";
  if (argc > 1) n = std::atoi(argv[1]);
  if (argc > 2) test_id = std::atoi(argv[2]);
  if (argc > 3) solver = argv[3];
  if (test_id < 1 || test_id > 5) {
    std::cerr << "Error: test_id must be 1-5\n";
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
  return fp32 ? run<float>(n, test_id, solver, exact, "fp32") : run<double>(n, test_id, solver, exact, "fp64");
}
