// gen_d12.cc -- build-time generator of the D12 wavelet table.
//
// The D12 mass-assignment stencil samples a tabulated wavelet (reference
// cc/particle_mesh/d12.h:13-147) that has no closed form; the numbers are
// reference data, so they are read from the reference header at build time
// instead of being copied into this repository.  This program includes that
// header (path given with -I<reference>/cc), runs its setup_wavelet()
// transpose (d12.h:149-155) and prints wave[] as exact hexadecimal floating
// literals for csrc/_gen/d12_table.inc.
#include <cstdio>

#include "particle_mesh/d12.h"

int main() {
  setup_wavelet();
  for (int i = 0; i < WCELLS * WAVESAMPLE; ++i) std::printf("%a,\n", wave[i]);
  return 0;
}
