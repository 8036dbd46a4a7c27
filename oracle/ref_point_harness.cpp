// ref_point_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// This project's driver around the reference's header-only point functions
// (include/mhd/mhd_common.hpp, include/mhd/mhd_glm_common.hpp).  It is
// compiled by oracle/Makefile against the reference tree (never copied here)
// into oracle/_ref/, and run by tests/golden/make_golden.py to record golden
// input/output vectors for the oracle and the CUDA point functions.
//
// Protocol (binary, native endianness, Real = double or float per build):
//   stdin : int32 n, then n records { int32 op; Real in[19]; }
//           in[0..8] = left state, in[9..17] = right state, in[18] = ch
//   stdout: n records { int32 status; Real out[9]; }
#include "mhd/mhd_glm_common.hpp"

#include <cstdint>
#include <cstdio>
#include <vector>

int main() {
  int32_t n = 0;
  if (std::fread(&n, sizeof(n), 1, stdin) != 1) return 1;
  for (int32_t r = 0; r < n; r++) {
    int32_t op = 0;
    Real in[19];
    if (std::fread(&op, sizeof(op), 1, stdin) != 1) return 1;
    if (std::fread(in, sizeof(Real), 19, stdin) != 19) return 1;
    const Real* a = in;
    const Real* b = in + 9;
    Real ch = in[18];
    Real out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int32_t status = 0;
    switch (op) {
      case 0: mhdConsToPrim(a, out); break;
      case 1: mhdPrimToCons(a, out); break;
      case 2: out[0] = mhdFastSpeedX(a); break;
      case 3: out[0] = mhdFastSpeedY(a); break;
      case 4: mhdHllFluxX(a, b, out); break;
      case 5: mhdHllFluxY(a, b, out); break;
      case 6: status = mhdHlldFluxX(a, b, out); break;
      case 7: status = mhdHlldFluxY(a, b, out); break;
      case 8: status = mhdGlmFluxX(a, b, ch, true, out); break;
      case 9: status = mhdGlmFluxY(a, b, ch, true, out); break;
      case 10: status = mhdGlmFluxX(a, b, ch, false, out); break;
      case 11: status = mhdGlmFluxY(a, b, ch, false, out); break;
      case 12: out[0] = mhdMinmod(a[0], b[0]); break;
      case 13: status = mhdConservedHasPositivePressure(a) ? 1 : 0; break;
      default: status = -1; break;
    }
    std::fwrite(&status, sizeof(status), 1, stdout);
    std::fwrite(out, sizeof(Real), 9, stdout);
  }
  return 0;
}
