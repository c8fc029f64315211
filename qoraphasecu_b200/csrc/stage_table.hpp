// The stage-major twiddle table of the register-resident line transforms
// (line_fft.cuh), shared by the device code that reads it and the host code
// that builds it.
#pragma once

#include "common.cuh"

namespace qpb {

// Radices of the register-resident transform of a line of L points and the
// size of its stage-major twiddle table.
struct StageGeometry {
  int stages = 0;  // 0: no register-resident transform for this length
  int radix[3] = {1, 1, 1};
  int count = 0;   // entries of the stage-major twiddle table
};

// The geometry for line length L (stages 0 unless L is a power of two in
// 16..1024).
StageGeometry stage_geometry(int L);

// Exponent e (the entry is W_L^e) of entry i < g.count of the stage-major
// table: stage 1 (NS = R0, radix R1) first, then stage 2 (NS = R0 R1, radix
// R2), each (r - 1) NS + k for r = 1..R-1, k < NS, with e = r k L / (NS R).
QPB_HD int stage_twiddle_exponent(const StageGeometry& g, int L, int i) {
  int ns = g.radix[0];
  int radix = g.radix[1];
  if (i >= (radix - 1) * ns) {
    i -= (radix - 1) * ns;
    ns *= radix;
    radix = g.radix[2];
  }
  const int r = i / ns + 1;
  const int k = i % ns;
  return r * k * (L / (ns * radix));
}

}  // namespace qpb
