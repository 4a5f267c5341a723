// Internal interface between the batch engine (batch.cu) and the level-step
// (lbm_step.cu) and immersed-boundary (ib.cu) translation units.  Not part
// of the C ABI.
#pragma once

#include <vector>

#include "ilbm_common.cuh"
#include "step_args.cuh"

struct ilbm_ib;

namespace ilbm {

// ---- lbm_step.cu --------------------------------------------------------
// the level step with a stored-macro box (the two-level hierarchy's coarse
// level); mlo / mhi NULL: ilbm_level_step.  part 0: the whole step; 1 / 2:
// its two halves along the box's last dimension (one box; the ghost push
// runs with the first, macro_out after the second)
int level_step_impl(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const ilbm_level_params *p,
                    const int *mlo, const int *mhi, int part);
// StepArgs of one batched case (self-filled ghosts, one box = domain)
int batch_case_args(const ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                    StepArgs *out);
// ghost-push chunks of w threads one case needs
int batch_ghost_chunks(const ilbm_ctx *ctx, const StepArgs &a, int w);
// k_step_batch over a tile table (w threads per block, `blocks` persistent
// blocks); cases with steps[c] >= limit[c] are skipped
int batch_step_launch(ilbm_ctx *ctx, const StepArgs *d_args, const StepTile *d_tiles, int ntiles,
                      int w, int blocks, const int *steps, const int *limit, cudaStream_t st);
// band macro of every case's body over its band tiles (same skipping)
int batch_band_macro_launch(ilbm_ctx *ctx, const StepArgs *d_args, const BandDesc *d_bands,
                            const ItemRef *d_tiles, int ntiles, const int *steps, const int *limit,
                            cudaStream_t st);
// resident blocks of w threads per SM of k_step_batch
int batch_step_occupancy(const ilbm_ctx *ctx, int w, int *per_sm);

// ---- forces.cu ------------------------------------------------------------
// the Eulerian force sum of ilbm_force_integrals enqueued on ctx->stream; the
// three sums land at *d_sum (context scratch, with 8 spare doubles after
// them) when the stream gets there; with fsum set, the same final launch also
// packs a force record (the sums, fsum[0..2], status[0..1] as doubles) at
// rec_dst (a device-accessible address) or, without it, at *d_sum + 8
int force_sum_enqueue(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const int lo[3],
                      const int hi[3], double **d_sum, const double *fsum = nullptr,
                      const int *status = nullptr, double *rec_dst = nullptr);
// one box's force record (region sum, fsum, status) written to rec (device-
// accessible) by launches on stream st, using the caller's scratch of at
// least force_record_scratch() doubles
size_t force_record_scratch();
int force_record_on(ilbm_ctx *ctx, const ilbm_box &box, const int lo[3], const int hi[3],
                    const double *fsum, const int *status, double *rec, double *scr,
                    cudaStream_t st);
// the body's force record on stream st (the context's side stream, after
// the body's forcing chain queued there, or its main stream): rec is
// device-accessible; records ctx->ev_rec on st after it
int ib_record_on(ilbm_ib *ib, const ilbm_box &box, const int lo[3], const int hi[3], double *rec,
                 cudaStream_t st);

// ---- ib.cu ----------------------------------------------------------------
// ilbm_advance_level in two halves: begin starts the body's update_forcing
// (on the side stream, after the work queued so far on the main stream, when
// it may overlap), end runs the level step of the cells outside the body's
// band and then the band.  Work the caller queues in between on the main
// stream overlaps the body's forcing.
struct AdvanceSplit {
  ilbm_level_params q;  // the level's parameters with the body's force region
  int lo[3], hi[3];     // the body's band
  bool serial;          // no overlap: forcing first, then the whole step
};
int advance_begin(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p, ilbm_ib *ib,
                  double dt, double time, AdvanceSplit *sp);
int advance_end(ilbm_ctx *ctx, const ilbm_box *box, const AdvanceSplit *sp);
struct IBBatch;

struct IBBatchCase {
  ilbm_ib *ib;     // NULL: a case without an immersed body
  double dt;       // time step of the case's level
  double time0;    // time of the case's next step
  int kin_steps;   // length of its kinematics table (>= limit, >= 1)
  int limit;       // steps the case may take in this batch (it stops there)
};

// device tables for a set of cases; fails if a body has not taken its first
// step through ilbm_advance_level / ilbm_ib_update_forcing, or uses several
// MDF iterations
int ib_batch_create(ilbm_ctx *ctx, const std::vector<IBBatchCase> &cases, int rec_slots,
                    IBBatch **out);
void ib_batch_destroy(IBBatch *b);
// update_forcing of every case for one step; d_args: the step's StepArgs table
int ib_batch_forcing(IBBatch *b, const StepArgs *d_args, cudaStream_t s);
// per-case force record of the step and step counter + 1
int ib_batch_record(IBBatch *b, const StepArgs *d_args, cudaStream_t s);
// record rings (ncase x rec_slots x 8 doubles), step counters (ncase) and
// status words (ncase) to the host; synchronises s
int ib_batch_read(IBBatch *b, std::vector<double> &rec, std::vector<int> &steps,
                  std::vector<int> &status, cudaStream_t s);
int ib_batch_rec_slots(const IBBatch *b);
// device step counters and limits (one int per case)
const int *ib_batch_steps(const IBBatch *b);
const int *ib_batch_limits(const IBBatch *b);

}  // namespace ilbm
