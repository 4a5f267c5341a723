// Internal interface between the state I/O (state_io.cu) and the immersed
// boundary (ib.cu) translation units.  Not part of the C ABI.
#pragma once

#include <cstdint>

struct ilbm_ib;

namespace ilbm {

// Device arrays that carry an IB object's state from one step to the next.
// Everything else it holds (band fields, CSR operator, stored inverse) is
// rebuilt from these and from its creation parameters.
struct IBState {
  int64_t n = 0;       // markers
  int dim = 0;
  int geometry = 0;    // geometry_type of the creation parameters
  int coupling = 0;    // coupling_method
  double *xyz = nullptr, *uvw = nullptr, *F = nullptr;  // 3n each
  double *fsum = nullptr;  // 3: last marker force sum
  double *X = nullptr;     // 3n: CG start of the next solve, or NULL
  double *Xh = nullptr;    // 3n: the solution before it (extrapolated start), or NULL
  bool cg_warm = false;
  bool cg_hist2 = false;
};

void ib_state(ilbm_ib *ib, IBState *out);
void ib_set_cg_warm(ilbm_ib *ib, bool warm, bool hist2);
}  // namespace ilbm
