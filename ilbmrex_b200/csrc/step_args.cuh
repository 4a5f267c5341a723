// Kernel arguments of one box of a level step, shared by the level-step
// kernels (lbm_step.cu), the immersed boundary (ib.cu) and the batch engine
// (batch.cu), which keeps one StepArgs per case and buffer parity in device
// memory.
#pragma once

#include <stdint.h>

namespace ilbm {

constexpr int kMaxLevelBoxes = 64;

struct StepArgs {
  // box valid region and allocated lower corners
  int lo[3], hi[3];
  int fgl[3];  // allocated lower corner of f arrays
  int mgl[3];  // allocated lower corner of macro / force arrays
  int64_t fs0, fs1, fs2;
  int64_t ms0, ms1, ms2;
  const void *f_in;
  void *f_out;
  const void *macro_in;
  const void *force;
  const void *force_prev;
  // level
  int dlo[3], dhi[3];
  int periodic[3];
  int bclo[3], bchi[3];
  double bvlo[3][4], bvhi[3][4];
  double tau;
  int self_fill;
  int use_uniform;
  double uf[3];
  int flo[3], fhi[3];
  float f16_scale;
  float om32, omh32;  // 1/tau and 1 - 1/(2 tau) rounded to float, from the host
  // per-direction element offsets: q*fs2 (load) and c_q + q*fs2 (push target)
  int32_t loff[27], doff[27];
  // cells handled by this launch: [rlo, rhi], minus [slo, shi] when use_skip
  int rlo[3], rhi[3];
  int slo[3], shi[3];
  int use_skip;
  int ghost_slices;          // leading z-slices of the k_step grid that run ghost_push
  int act_lo[3], act_hi[3];  // face returns outgoing populations (wrap / reflect)
  int nlb;
  int lb[kMaxLevelBoxes][6];
  // with use_mbox, macro_in holds stored values only on [mblo, mbhi]; cells
  // outside recover rho, u from f^n and F^{n-1}
  int use_mbox;
  int mblo[3], mbhi[3];
};

// the cell's rho, u come from macro_in (else from its populations)
__device__ __forceinline__ bool stored_macro_at(const StepArgs &a, int i, int j, int k) {
  if (!a.macro_in) return false;
  if (!a.use_mbox) return true;
  return i >= a.mblo[0] && i <= a.mbhi[0] && j >= a.mblo[1] && j <= a.mbhi[1] && k >= a.mblo[2] &&
         k <= a.mbhi[2];
}

// One work item of the batched level step (k_step_batch): a row segment of
// blockDim.x cells of case c starting at (i0, j, k), or, when i0 < 0, chunk
// (-1 - i0) of the case's ghost shell push, which has j chunks in all.
struct StepTile {
  int c, i0, j, k;
};

// Support band of an immersed body on a case's level (EV: 3 velocity
// components, RHO: density, EFI: 3 spread-force components, zeroed by the
// batched band macro when set; all band-sized).
struct BandDesc {
  int blo[3], bn[3];
  int64_t nb;
  double *EV, *RHO, *EFI;
};

// Work lists of the batched immersed-body stages: one entry per marker
// (case, marker) and tiles of kItemTile band cells of one case (case, first
// cell), so an item finds its case with one load.
struct ItemRef {
  int c, u;
};
constexpr int kItemTile = 256;

}  // namespace ilbm
