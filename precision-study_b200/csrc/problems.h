// problems.h -- host-side initial conditions and .dat output helpers.
#ifndef PMHD_PROBLEMS_H
#define PMHD_PROBLEMS_H

#include <cstddef>
#include <string>
#include <vector>

namespace pmhd {

struct ProblemGrid {
  int nx, ny;
  double x_min, x_max, y_min, y_max, gamma;
};

// Fills a ghosted AoS state [(ny+4)][(nx+4)][9] of element type T with
// problem `problem` (pmhd_problem).  Returns false for an unknown problem.
template <class T>
bool init_problem_host(const ProblemGrid& g, int problem, const double* params, int nparams, std::vector<T>& U);

// divB L1, divB Linf, psi Linf of a ghosted AoS state.
template <class T>
void diagnostics_host(const ProblemGrid& g, const std::vector<T>& U, double out[3]);

// Writes the data lines of the reference .dat format for a ghosted state.
template <class T>
bool write_dat_body(std::FILE* f, const ProblemGrid& g, const std::vector<T>& U);

}  // namespace pmhd

#endif
