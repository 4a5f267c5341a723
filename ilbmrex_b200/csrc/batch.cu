// Batch engine: many independent single-level cases (each one box equal to
// its level domain, self-filled ghosts) advanced together on one GPU.
//
// Per step the whole batch costs a fixed number of launches, whatever the
// number of cases: the immersed-boundary stages run once each over the
// concatenated markers / band cells of every case (ib.cu), and the fused
// collide-stream of every cell of every case is one persistent kernel that
// walks a tile table of row segments and ghost-push chunks (k_step_batch,
// lbm_step.cu).  Two consecutive steps (the two population buffers swap
// roles) are captured once as a CUDA graph and replayed.  The tile width and
// the number of resident blocks come from ilbm_batch_tune, which times the
// candidates on the batch itself.
//
// There is no counterpart in the reference: it advances one case per run.
#include <algorithm>
#include <cstring>
#include <vector>

#include "batch_internal.h"

using namespace ilbm;

struct ilbm_batch {
  struct Case {
    int id;
    ilbm_box box;
    ilbm_level_params p;
    ilbm_ib *ib;
    double dt, time;   // time of the case's next step
    int max_steps;     // steps the caller may still ask for (kinematics table)
    int parity;        // buffers of the state at the last build: 0 as in box, 1 swapped
    int64_t steps;     // steps taken inside this batch
    int64_t cells;
    std::vector<double> rec;  // 8 doubles per step taken in the batch
  };
  ilbm_ctx *ctx = nullptr;
  std::vector<Case> cases;
  int next_id = 1;
  int rec_slots = 256;
  int tile_w = 128, ctas_per_sm = 0;  // 0: as many as fit
  int sms = 0;
  // built state
  bool built = false;
  int phase = 0;    // slot of the next step (a case's state: parity ^ (its steps & 1))
  int pending = 0;  // steps since the record rings were drained
  StepArgs *d_args = nullptr;  // [2][ncase]
  StepTile *d_tiles = nullptr;
  int ntiles = 0, blocks = 0;
  IBBatch *ibb = nullptr;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int64_t graph_launches[2] = {0, 0};
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

namespace {

void free_built(ilbm_batch *b) {
  for (int i = 0; i < 2; ++i)
    if (b->gexec[i]) {
      cudaGraphExecDestroy(b->gexec[i]);
      b->gexec[i] = nullptr;
    }
  ilbm_ctx_free(b->ctx, b->d_args);  // stream-ordered: after the steps that read them
  ilbm_ctx_free(b->ctx, b->d_tiles);
  b->d_args = nullptr;
  b->d_tiles = nullptr;
  ib_batch_destroy(b->ibb);
  b->ibb = nullptr;
  b->built = false;
}

// copy the record rings into the per-case histories
int drain(ilbm_batch *b) {
  if (!b->built || !b->ibb) return ILBM_OK;
  std::vector<double> rec;
  std::vector<int> steps, status;
  int rc = ib_batch_read(b->ibb, rec, steps, status, b->ctx->stream);
  if (rc) return rc;
  const int R = ib_batch_rec_slots(b->ibb);
  for (size_t c = 0; c < b->cases.size(); ++c) {
    auto &k = b->cases[c];
    const int64_t have = (int64_t)k.rec.size() / 8 - k.steps;  // taken in this build, stored
    for (int64_t s = have; s < steps[c]; ++s) {
      const double *r = rec.data() + ((size_t)c * R + (size_t)(s % R)) * 8;
      k.rec.insert(k.rec.end(), r, r + 8);
    }
  }
  b->pending = 0;
  for (size_t c = 0; c < b->cases.size(); ++c) {
    if (status[c] & 1) {
      set_error("batch: an IB stencil left its support band");
      return ILBM_ERR_RANGE;
    }
    if (status[c] & 2) {
      set_error("batch: an IVC operator exceeded its nonzero capacity");
      return ILBM_ERR_SOLVER;
    }
    if (status[c] & 4) {
      set_error("batch: an IVC conjugate gradient did not converge");
      return ILBM_ERR_SOLVER;
    }
    if (status[c] & 16) {
      set_error("batch: a case ran past the steps it was added for (max_steps)");
      return ILBM_ERR_RANGE;
    }
  }
  return ILBM_OK;
}

// fold the steps taken since the last build into each case (time, parity,
// step count) before the tables are rebuilt
int settle(ilbm_batch *b) {
  if (!b->built) return ILBM_OK;
  int rc = drain(b);
  if (rc) return rc;
  for (auto &k : b->cases) {
    const int64_t taken = (int64_t)k.rec.size() / 8 - k.steps;
    for (int64_t s = 0; s < taken; ++s) k.time += k.dt;  // as the single path accumulates it
    k.steps += taken;
    k.max_steps -= (int)taken;
    k.parity ^= (int)(taken & 1);  // a case that stopped early keeps its own parity
  }
  b->phase = 0;
  free_built(b);
  return ILBM_OK;
}

ilbm_box slot_box(const ilbm_batch::Case &k, int q) {
  ilbm_box x = k.box;
  if (q) {
    std::swap(x.f_in, x.f_out);
    std::swap(x.force, x.force_prev);
  }
  return x;
}

int build(ilbm_batch *b) {
  if (b->built) return ILBM_OK;
  ilbm_ctx *ctx = b->ctx;
  const int nc = (int)b->cases.size();
  if (nc == 0) {
    b->built = true;
    return ILBM_OK;
  }
  std::vector<StepArgs> args(2 * (size_t)nc);
  std::vector<IBBatchCase> ibc(nc);
  int rc;
  for (int c = 0; c < nc; ++c) {
    const auto &k = b->cases[c];
    for (int s = 0; s < 2; ++s) {
      const ilbm_box x = slot_box(k, k.parity ^ s);
      ilbm_level_params p = k.p;
      if (k.ib) {
        int lo[3], hi[3];
        ilbm_ib_force_region(k.ib, lo, hi);
        for (int d = 0; d < 3; ++d) {
          p.force_lo[d] = lo[d];
          p.force_hi[d] = hi[d];
        }
      }
      if ((rc = batch_case_args(ctx, x, &p, &args[(size_t)s * nc + c]))) return rc;
    }
    ibc[c] = IBBatchCase{k.ib, k.dt, k.time, std::max(1, k.max_steps), std::max(0, k.max_steps)};
  }
  // tile table: every case's ghost-push chunks first (strided, slow), then
  // its row segments; the kernel's block b takes entries b, b + blocks, ...
  // When every case has the same number of steps left (none sits out before
  // the batch is re-tabled), each case owns a share of the blocks
  // proportional to its rows and its row segments are dealt round by round
  // over its own blocks, so a block stays in one case (its arguments copied
  // to shared memory once) while the case's blocks sweep neighbouring rows
  // together; the ghost chunks are then padded to a whole number of rounds
  // and entries with c = -1 fill the rounds (skipped).  Otherwise the row
  // segments follow case after case, so that the blocks of a case that has
  // finished its steps take the other cases' segments.
  const int W = b->tile_w;
  int per_sm = 0;
  if ((rc = batch_step_occupancy(ctx, W, &per_sm))) return rc;
  if (per_sm < 1) {
    set_error("batch: the level-step kernel does not fit this tile width");
    return ILBM_ERR_UNSUPPORTED;
  }
  const int use = (b->ctas_per_sm > 0) ? std::min(b->ctas_per_sm, per_sm) : per_sm;
  std::vector<StepTile> tiles;
  for (int c = 0; c < nc; ++c) {
    const int nch = batch_ghost_chunks(ctx, args[c], W);
    for (int ch = 0; ch < nch; ++ch) tiles.push_back(StepTile{c, -1 - ch, nch, 0});
  }
  std::vector<std::vector<StepTile>> rows(nc);
  int64_t nrow = 0;
  for (int c = 0; c < nc; ++c) {
    const StepArgs &a = args[c];
    for (int k = a.lo[2]; k <= a.hi[2]; ++k)
      for (int j = a.lo[1]; j <= a.hi[1]; ++j)
        for (int i0 = a.lo[0]; i0 <= a.hi[0]; i0 += W) rows[c].push_back(StepTile{c, i0, j, k});
    nrow += (int64_t)rows[c].size();
  }
  const int G = (int)std::max<int64_t>(1, std::min<int64_t>(nrow + (int64_t)tiles.size(),
                                                            (int64_t)use * b->sms));
  b->blocks = G;
  bool same_steps = true;
  for (int c = 1; c < nc; ++c) same_steps = same_steps && b->cases[c].max_steps == b->cases[0].max_steps;
  if (nc <= G && same_steps) {
    // blocks per case: proportional to its rows, at least one (largest remainders)
    std::vector<int> nb(nc, 1);
    int left = G - nc;
    std::vector<std::pair<double, int>> rem;
    for (int c = 0; c < nc; ++c) {
      const double share = nrow ? double(left) * double(rows[c].size()) / double(nrow) : 0.0;
      nb[c] += (int)share;
      rem.push_back({share - (int)share, c});
    }
    int given = 0;
    for (int c = 0; c < nc; ++c) given += nb[c] - 1;
    std::sort(rem.begin(), rem.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    for (int q = 0; q < left - given && q < (int)rem.size(); ++q) nb[rem[q].second]++;
    int64_t rounds = 0;
    for (int c = 0; c < nc; ++c)
      rounds = std::max<int64_t>(rounds, ((int64_t)rows[c].size() + nb[c] - 1) / nb[c]);
    while (tiles.size() % G) tiles.push_back(StepTile{-1, 0, 0, 0});
    std::vector<int> owner(G), first(nc + 1, 0);
    for (int c = 0; c < nc; ++c) first[c + 1] = first[c] + nb[c];
    for (int c = 0; c < nc; ++c)
      for (int s = first[c]; s < first[c + 1]; ++s) owner[s] = c;
    for (int64_t r = 0; r < rounds; ++r)
      for (int s = 0; s < G; ++s) {
        const int c = owner[s];
        const int64_t i = r * nb[c] + (s - first[c]);
        tiles.push_back(i < (int64_t)rows[c].size() ? rows[c][(size_t)i] : StepTile{-1, 0, 0, 0});
      }
  } else {
    for (int c = 0; c < nc; ++c) tiles.insert(tiles.end(), rows[c].begin(), rows[c].end());
  }
  b->ntiles = (int)tiles.size();
  // stream-ordered tables (pageable sources are staged before the copies return)
  cudaError_t e = ilbm_ctx_malloc(ctx, (void **)&b->d_args, args.size() * sizeof(StepArgs));
  if (e == cudaSuccess) e = ilbm_ctx_malloc(ctx, (void **)&b->d_tiles, tiles.size() * sizeof(StepTile));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_args, args.data(), args.size() * sizeof(StepArgs), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_tiles, tiles.data(), tiles.size() * sizeof(StepTile), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e != cudaSuccess) {
    free_built(b);
    return cuda_fail(e, "batch tables");
  }
  if ((rc = ib_batch_create(ctx, ibc, b->rec_slots, &b->ibb))) {
    free_built(b);
    return rc;
  }
  b->built = true;
  b->phase = 0;
  b->pending = 0;
  return ILBM_OK;
}

// one step of every case, buffers of `slot`
int step_slot(ilbm_batch *b, int slot) {
  const int nc = (int)b->cases.size();
  const StepArgs *a = b->d_args + (size_t)slot * nc;
  int rc = ib_batch_forcing(b->ibb, a, b->ctx->stream);
  if (rc) return rc;
  if ((rc = batch_step_launch(b->ctx, a, b->d_tiles, b->ntiles, b->tile_w, b->blocks,
                              ib_batch_steps(b->ibb), ib_batch_limits(b->ibb), b->ctx->stream)))
    return rc;
  return ib_batch_record(b->ibb, a, b->ctx->stream);
}

// graph of two steps starting at slot `first`
int ensure_graph(ilbm_batch *b, int first) {
  if (b->gexec[first]) return ILBM_OK;
  cudaStream_t s = b->ctx->stream;
  cudaGraph_t g = nullptr;
  const int64_t l0 = b->ctx->launches;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
  int rc = step_slot(b, first);
  if (!rc) rc = step_slot(b, first ^ 1);
  e = cudaStreamEndCapture(s, &g);
  b->graph_launches[first] = b->ctx->launches - l0;
  b->ctx->launches = l0;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
  e = cudaGraphInstantiate(&b->gexec[first], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
  return ILBM_OK;
}

int advance(ilbm_batch *b, int n) {
  int rc = build(b);
  if (rc) return rc;
  if (b->cases.empty()) return ILBM_OK;
  while (n > 0) {
    const int room = b->rec_slots - b->pending;
    int k = std::min(n, room);
    n -= k;
    b->pending += k;
    while (k >= 2) {
      if ((rc = ensure_graph(b, b->phase))) return rc;
      cudaError_t e = cudaGraphLaunch(b->gexec[b->phase], b->ctx->stream);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph launch");
      b->ctx->launches += b->graph_launches[b->phase];
      k -= 2;
    }
    if (k == 1) {
      if ((rc = step_slot(b, b->phase))) return rc;
      b->phase ^= 1;
    }
    if (b->pending >= b->rec_slots && (rc = drain(b))) return rc;
  }
  return ILBM_OK;
}

ilbm_batch::Case *find_case(ilbm_batch *b, int id) {
  for (auto &k : b->cases)
    if (k.id == id) return &k;
  return nullptr;
}

}  // namespace

extern "C" {

int ilbm_batch_create(ilbm_ctx *ctx, int rec_slots, ilbm_batch **out) {
  if (!ctx || !out) {
    set_error("ilbm_batch_create: null argument");
    return ILBM_ERR_ARG;
  }
  auto *b = new ilbm_batch();
  b->ctx = ctx;
  b->rec_slots = std::max(2, rec_slots > 0 ? rec_slots : 256);
  cudaSetDevice(ctx->device);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaError_t e = cudaEventCreate(&b->ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev[1]);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "ilbm_batch_create");
  }
  *out = b;
  return ILBM_OK;
}

int ilbm_batch_destroy(ilbm_batch *b) {
  if (!b) return ILBM_OK;
  cudaStreamSynchronize(b->ctx->stream);
  free_built(b);
  for (auto &e : b->ev)
    if (e) cudaEventDestroy(e);
  delete b;
  return ILBM_OK;
}

int ilbm_batch_add(ilbm_batch *b, const ilbm_box *box, const ilbm_level_params *p, ilbm_ib *ib,
                   double dt, double time, int max_steps, int *case_id) {
  if (!b || !box || !p || !case_id) {
    set_error("ilbm_batch_add: null argument");
    return ILBM_ERR_ARG;
  }
  StepArgs probe;
  int rc = batch_case_args(b->ctx, *box, p, &probe);
  if (rc) return rc;
  if (ib && (!box->force || !box->force_prev)) {
    set_error("ilbm_batch_add: a case with a body needs force and force_prev");
    return ILBM_ERR_ARG;
  }
  if ((rc = settle(b))) return rc;
  ilbm_batch::Case k;
  k.id = b->next_id++;
  k.box = *box;
  k.p = *p;
  k.ib = ib;
  k.dt = dt;
  k.time = time;
  k.max_steps = std::max(0, max_steps);
  k.parity = 0;
  k.steps = 0;
  k.cells = 1;
  for (int d = 0; d < b->ctx->dim; ++d) k.cells *= (int64_t)(box->hi[d] - box->lo[d] + 1);
  b->cases.push_back(std::move(k));
  *case_id = b->cases.back().id;
  return ILBM_OK;
}

int ilbm_batch_remove(ilbm_batch *b, int case_id) {
  if (!b || !find_case(b, case_id)) {
    set_error("ilbm_batch_remove: unknown case");
    return ILBM_ERR_ARG;
  }
  int rc = settle(b);
  if (rc) return rc;
  for (size_t c = 0; c < b->cases.size(); ++c)
    if (b->cases[c].id == case_id) {
      b->cases.erase(b->cases.begin() + c);
      break;
    }
  return ILBM_OK;
}

int ilbm_batch_step(ilbm_batch *b, int nsteps) {
  if (!b || nsteps < 0) {
    set_error("ilbm_batch_step: bad argument");
    return ILBM_ERR_ARG;
  }
  return advance(b, nsteps);
}

int ilbm_batch_case_state(ilbm_batch *b, int case_id, int *parity, int64_t *steps_done,
                          double *time) {
  ilbm_batch::Case *k = b ? find_case(b, case_id) : nullptr;
  if (!k) {
    set_error("ilbm_batch_case_state: unknown case");
    return ILBM_ERR_ARG;
  }
  int rc = drain(b);
  if (rc) return rc;
  const int64_t taken = (int64_t)k->rec.size() / 8 - k->steps;
  double t = k->time;
  for (int64_t s = 0; s < taken; ++s) t += k->dt;
  if (parity) *parity = k->parity ^ (int)(taken & 1);
  if (steps_done) *steps_done = k->steps + taken;
  if (time) *time = t;
  return ILBM_OK;
}

int ilbm_batch_records(ilbm_batch *b, int case_id, double *out, int max_rec, int *nrec) {
  ilbm_batch::Case *k = b ? find_case(b, case_id) : nullptr;
  if (!k || !nrec) {
    set_error("ilbm_batch_records: unknown case or null argument");
    return ILBM_ERR_ARG;
  }
  int rc = drain(b);
  if (rc) return rc;
  const int have = (int)(k->rec.size() / 8);
  const int n = out ? std::min(have, std::max(0, max_rec)) : 0;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < 6; ++c) out[r * 6 + c] = k->rec[(size_t)(have - n + r) * 8 + c];
  *nrec = out ? n : have;
  return ILBM_OK;
}

int ilbm_batch_set_tiles(ilbm_batch *b, int tile_w, int ctas_per_sm) {
  if (!b || (tile_w != 64 && tile_w != 128 && tile_w != 256) || ctas_per_sm < 0) {
    set_error("ilbm_batch_set_tiles: tile_w must be 64, 128 or 256, ctas_per_sm >= 0");
    return ILBM_ERR_ARG;
  }
  int rc = settle(b);
  if (rc) return rc;
  b->tile_w = tile_w;
  b->ctas_per_sm = ctas_per_sm;
  return ILBM_OK;
}

int ilbm_batch_tune(ilbm_batch *b, int trial_steps, int *tile_w, int *ctas_per_sm,
                    float *ms_per_step) {
  if (!b || trial_steps < 2) {
    set_error("ilbm_batch_tune: trial_steps must be >= 2");
    return ILBM_ERR_ARG;
  }
  if (b->cases.empty()) {
    set_error("ilbm_batch_tune: empty batch");
    return ILBM_ERR_ARG;
  }
  trial_steps += trial_steps & 1;  // whole graph replays
  float best = 1e30f;
  int bw = b->tile_w, bc = b->ctas_per_sm;
  for (int w : {64, 128, 256}) {
    int per_sm = 0;
    int rc = batch_step_occupancy(b->ctx, w, &per_sm);
    if (rc) return rc;
    for (int cps = per_sm; cps >= 1 && cps >= per_sm - 2; --cps) {
      if ((rc = ilbm_batch_set_tiles(b, w, cps))) return rc;
      if ((rc = advance(b, 2))) return rc;  // build, capture, warm
      cudaEventRecord(b->ev[0], b->ctx->stream);
      if ((rc = advance(b, trial_steps))) return rc;
      cudaEventRecord(b->ev[1], b->ctx->stream);
      cudaError_t e = cudaEventSynchronize(b->ev[1]);
      if (e != cudaSuccess) return cuda_fail(e, "ilbm_batch_tune");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
      ms /= float(trial_steps);
      if (ms < best) {
        best = ms;
        bw = w;
        bc = cps;
      }
    }
  }
  int rc = ilbm_batch_set_tiles(b, bw, bc);
  if (rc) return rc;
  if (tile_w) *tile_w = bw;
  if (ctas_per_sm) *ctas_per_sm = bc;
  if (ms_per_step) *ms_per_step = best;
  return ILBM_OK;
}

int ilbm_batch_progress(ilbm_batch *b, int max_cases, int *ids, int64_t *steps_done,
                        int *remaining, int *ncase) {
  if (!b || !ncase) {
    set_error("ilbm_batch_progress: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = drain(b);
  if (rc) return rc;
  const int n = std::min((int)b->cases.size(), std::max(0, max_cases));
  for (int c = 0; c < n; ++c) {
    const auto &k = b->cases[c];
    const int64_t taken = (int64_t)k.rec.size() / 8 - k.steps;
    if (ids) ids[c] = k.id;
    if (steps_done) steps_done[c] = k.steps + taken;
    if (remaining) remaining[c] = std::max(0, k.max_steps - (int)taken);
  }
  *ncase = (int)b->cases.size();
  return ILBM_OK;
}

int ilbm_batch_size(ilbm_batch *b, int *ncase, int64_t *cells) {
  if (!b) return ILBM_ERR_ARG;
  int64_t n = 0;
  for (auto &k : b->cases) n += k.cells;
  if (ncase) *ncase = (int)b->cases.size();
  if (cells) *cells = n;
  return ILBM_OK;
}

}  // extern "C"
