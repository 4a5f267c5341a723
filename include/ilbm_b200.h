/*
 * ilbm_b200.h -- C ABI of the B200 (sm_100a) level-step library for the
 * iLBMReX per-level hot path.
 *
 * The reference has no plugin or FFI for this path: its seam is a set of C++
 * member calls inside one binary.  Each entry point below replaces one of
 * them (reference paths are relative to the reference project root):
 *
 *   ilbm_level_step        AmrCoreLBM::AdvancePhiAtLevel, the collide /
 *                          bounce-back / stream / macro passes
 *                          (Source/Core/AdvanceLBMAtLevel.cpp:20-21, 196-386)
 *                          with the ghost fill of FillPatchMesoscopic
 *                          (Source/Core/AmrCoreLBM.cpp:1531-1628 using
 *                          mesoscopicBcFill, Source/BC/bc_fill.H:303-347)
 *   ilbm_compute_macro     calculateMacroForcing pass
 *                          (Source/LBM/calculateMacroForcing.H:9-32,
 *                          Source/Core/AdvanceLBMAtLevel.cpp:382-386)
 *   ilbm_init_equilibrium  AmrCoreLBM::InitEquilibrium
 *                          (Source/Core/AmrCoreLBM.cpp:2117-2164)
 *   ilbm_ib_create         IBMarkerDF::IBMarkerDF + build_markers
 *                          (Source/IBM/IBMarkerDF.H:68-70,
 *                          Source/IBM/IBMarkerDF.cpp:190-497)
 *   ilbm_ib_update_forcing IBMarkerDF::update_forcing
 *                          (Source/IBM/IBMarkerDF.H:76-87,
 *                          Source/IBM/IBMarkerDF.cpp:1522-1917)
 *   ilbm_ib_last_marker_force_sum / ilbm_ib_num_markers
 *                          IBMarkerDF::last_marker_force_sum / num_markers
 *                          (Source/IBM/IBMarkerDF.H:90-91)
 *   ilbm_force_integrals   the Eulerian forcing integral of
 *                          AmrCoreLBM::ComputeIBForce
 *                          (Source/Core/AmrCoreLBM.cpp:489-509)
 *   ilbm_momentum_exchange IBForceEval::ComputeMomentumExchangeBodyForce
 *                          (Source/IBM/IBForceEval.H:24-32,
 *                          Source/IBM/IBForceEval.cpp:28-191)
 *
 * Conventions
 *   - The caller owns every field buffer (device memory).  The library never
 *     frees caller memory; it allocates only internal scratch inside a
 *     context or IB object.
 *   - Every call returns ILBM_OK (0) or a negative status and never aborts.
 *     ilbm_last_error() returns the message of the last failure on the
 *     calling thread.
 *   - Calls are asynchronous on the context's stream, except the ones that
 *     return host values (force sums, integrals, marker counts), which
 *     synchronise that stream.
 *   - One context per host thread / stream.  There is no global mutable state
 *     apart from the per-thread error message.
 *
 * Field layout (AMReX Array4): element (i,j,k,n) of a box whose allocated
 * (grown) region starts at glo = lo - ngrow lives at
 *     ptr[(i-glo.x) + (j-glo.y)*s0 + (k-glo.z)*s1 + n*s2]
 * with (s0,s1,s2) the box's jstride, kstride and component stride.  In 2D the
 * k index is 0 and glo.z = 0.
 *
 * Storage forms (ilbm_create):
 *   ILBM_STORAGE_F64         populations f_q stored and collided in double;
 *                            macro/force arrays are double.
 *   ILBM_STORAGE_F32_SHIFT   stored g_q = f_q - w_q in float, collided in
 *                            float; macro/force arrays are float.
 *   ILBM_STORAGE_F16_SCALED  stored h_q = (f_q - w_q) * scale / w_q in IEEE
 *                            half, collided in float; macro/force float.
 */
#ifndef ILBM_B200_H
#define ILBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ILBM_OK 0
#define ILBM_ERR_ARG (-1)
#define ILBM_ERR_CUDA (-2)
#define ILBM_ERR_UNSUPPORTED (-3)
#define ILBM_ERR_NOMEM (-4)
#define ILBM_ERR_SOLVER (-5)
#define ILBM_ERR_RANGE (-6)

#define ILBM_STORAGE_F64 0
#define ILBM_STORAGE_F32_SHIFT 1
#define ILBM_STORAGE_F16_SCALED 2

/* AMReX BCType codes accepted on non-periodic faces */
#define ILBM_BC_INT_DIR 0
#define ILBM_BC_FOEXTRAP 2
#define ILBM_BC_EXT_DIR 3
#define ILBM_BC_USER_1 1001
#define ILBM_BC_USER_2 1002

#define ILBM_MAX_Q 27

typedef struct ilbm_ctx ilbm_ctx;
typedef struct ilbm_ib ilbm_ib;

/* Discrete velocity set as the reference reads it from its deck
 * (lbm2d|lbm3d.{ndir,wis,wim,dirx,diry,dirz}, AmrCoreLBM.cpp:1212-1236).
 * Must be D2Q9, D3Q19 or D3Q27 in the reference decks' direction order. */
typedef struct {
  int dim;
  int q;
  double cx[ILBM_MAX_Q], cy[ILBM_MAX_Q], cz[ILBM_MAX_Q];
  double wis[ILBM_MAX_Q], wim[ILBM_MAX_Q];
} ilbm_lattice;

/* One box of a level (one FAB of f_old/f_new/macro/forcing in AMReX terms). */
typedef struct {
  int lo[3], hi[3]; /* valid region, inclusive, level index space */
  int ngrow_f;      /* ghost width allocated around f_in / f_out (>= 1; the ghost
                       layer of f_out is scratch written by edge cells) */
  int ngrow_m;      /* ghost width allocated around macro / force arrays */
  int64_t fstride[3]; /* f arrays: j, k, component strides (elements) */
  int64_t mstride[3]; /* macro / force arrays: j, k, component strides */
  void *f_in;       /* f^n (storage type); ghost layer 1 read in caller mode only */
  void *f_out;      /* f^{n+1} on valid cells (storage type) */
  void *macro_in;   /* rho,u,v,w at step n (real type) or NULL (recomputed) */
  void *macro_out;  /* rho,u,v,w at step n+1 (real type) or NULL */
  void *force;      /* F^n = dt*rho*a (3 comps, real type) or NULL */
  void *force_prev; /* F^{n-1} (3 comps) used when macro_in == NULL, or NULL */
} ilbm_box;

#define ILBM_GHOST_SELF 0   /* the library synthesises physical/periodic ghosts; one box = domain */
#define ILBM_GHOST_CALLER 1 /* caller filled f_in/macro_in/force ghosts (AMReX FillPatch) */

typedef struct {
  double tau;
  int domain_lo[3], domain_hi[3];
  int periodic[3];
  int bc_lo[3], bc_hi[3];
  double bc_val_lo[3][4]; /* per dim: rho, ux, uy, uz (BCBuf lo_*) */
  double bc_val_hi[3][4]; /* per dim: rho, ux, uy, uz (BCBuf hi_*) */
  int ghost_mode;
  int use_uniform_force;     /* lbm.prescribed_force, applied where force == NULL */
  double uniform_force[3];
  int force_lo[3], force_hi[3]; /* cells outside this region have zero force
                                   (both force and force_prev); ignored for uniform */
  double f16_scale;          /* ILBM_STORAGE_F16_SCALED only; 0 selects the default */
  /* ILBM_GHOST_CALLER: boxes of the whole level, to classify ghost cells as
   * covered (collided like the neighbour's valid cell) or not (kept). */
  const int *level_boxes; /* host array of nlevel_boxes * 6 ints (lo xyz, hi xyz) or NULL */
  int nlevel_boxes;
} ilbm_level_params;

/* ---- context ------------------------------------------------------------ */
/* The context owns a stream (or uses cuda_stream), a high-priority side
 * stream for the immersed-boundary chain, and a device memory pool from which
 * IB objects and batches allocate in stream order. */
int ilbm_create(const ilbm_lattice *lat, int storage, int device, void *cuda_stream,
                ilbm_ctx **out);
int ilbm_destroy(ilbm_ctx *ctx);
const char *ilbm_last_error(void);
int ilbm_sync(ilbm_ctx *ctx);
void *ilbm_stream(ilbm_ctx *ctx);
/* CUDA events on the context stream, for device-side timing (slots 0..8207;
 * slots from 16 up are created on first use). */
int ilbm_event_record(ilbm_ctx *ctx, int slot);
int ilbm_event_elapsed_ms(ilbm_ctx *ctx, int slot_a, int slot_b, float *ms);
/* number of kernels this context has launched since creation (a graph
 * replay counts the kernels it holds) */
int64_t ilbm_kernel_launches(const ilbm_ctx *ctx);
/* CUDA graphs of a context's steps (no counterpart in the reference, whose
 * steps are host loops over ParallelFor launches).  Between ilbm_graph_begin
 * and ilbm_graph_end the launches that calls on the context issue (level
 * steps, hierarchy steps, the body's forcing, on the context's stream and its
 * side stream) are recorded instead of run; ilbm_graph_launch replays them on
 * the context's stream, as one submission, with the arguments they were
 * recorded with: the buffers, boxes and parameters must be the same at every
 * replay (a hierarchy's buffers are back in place after two coarse steps), and
 * whatever the recorded calls keep on the device (a body's solver history)
 * carries on from replay to replay.  Calls that synchronise, read results back
 * or allocate cannot be recorded: they fail, the capture is invalidated, and
 * ilbm_graph_end reports it (ILBM_ERR_CUDA) and ends the capture.  A recorded
 * step must therefore not be the first one of a level or body (which builds
 * the body's tables and allocates).  ilbm_kernel_launches counts recorded
 * kernels only when they are replayed. */
typedef struct ilbm_graph ilbm_graph;
int ilbm_graph_begin(ilbm_ctx *ctx);
int ilbm_graph_end(ilbm_ctx *ctx, ilbm_graph **out);
int ilbm_graph_launch(ilbm_ctx *ctx, const ilbm_graph *g);
int ilbm_graph_destroy(ilbm_graph *g);
/* storage element size in bytes and real (macro/force) element size */
int ilbm_storage_bytes(const ilbm_ctx *ctx, int *storage_bytes, int *real_bytes);

/* ---- level step --------------------------------------------------------- */
/* One level step on nbox boxes: BGK collision with Guo forcing on valid cells,
 * halfway bounce-back for user_1 faces and streaming into f_out (each cell
 * pushes its post-collision populations to its neighbours, which gives the
 * same f_out as the reference's pull stream), with the reference's ghost
 * semantics.  If macro_out is set, rho/u of f^{n+1} are
 * written as well (calculateMacroForcing with F^n). */
int ilbm_level_step(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox,
                    const ilbm_level_params *p);
/* rho,u,v,w of f (valid cells of region [lo,hi] clipped to the box) with the
 * half-force shift of F (force array, uniform force or zero). */
int ilbm_compute_macro(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                       const void *f, const void *force, void *macro_out,
                       const int lo[3], const int hi[3]);
/* f = f_eq(rho,u) over the whole allocated box (valid + ngrow_f ghosts),
 * written to both f_in and f_out (InitEquilibrium). macro_in must cover the
 * same region (ngrow_m >= ngrow_f). */
int ilbm_init_equilibrium(ilbm_ctx *ctx, const ilbm_box *box);

/* ---- marker direct-forcing IBM ----------------------------------------- */
typedef struct {
  int dim;
  int n_cell[3];
  double prob_lo[3], prob_hi[3];
  int periodic[3];
  int bc_lo[3], bc_hi[3];
  double bc_val_lo[3][4], bc_val_hi[3][4];
} ilbm_level_geom;

typedef struct {
  /* MarkerIBParams, Source/IBM/MarkerIBParams.H:8-132 */
  int coupling_method; /* 0 explicit, 1 ivc (wu_shu), 2 explicit_diag */
  int delta_type;      /* 0/4: 4-point, 1/3: 3-point */
  int loop_ns;
  double mdf_relax;
  double explicit_diag_eps;
  int geometry_type;   /* 0 cylinder/sphere, 1 box, 2 user-defined pitching NACA */
  double box_xlo, box_xhi, box_ylo, box_yhi, box_zlo, box_zhi, box_ds;
  int box_lid_only;
  double box_lid_ux, box_lid_uy, box_lid_uz, box_wall_tol;
  int n_marker;
  double rd;
  double ubx, uby, ubz, omx, omy, omz;
  double ivc_diag_reg;
  int ivc_rebuild_matrix;
  int renormalize_delta;
  double x0, y0, z0, R; /* ibm.x0,y0,z0,R */
  /* user-defined pitching NACA 00xx (Examples/Pitching_airfoil/
   * IBMUserDefinedGeometry.H:14-20, 59-175); pivot_x moves the pivot along
   * the chord (0 = leading edge, as in the reference). */
  double airfoil_chord, airfoil_thickness;
  double pitch_mean, pitch_amplitude, pitch_frequency, pitch_phase, pivot_x;
} ilbm_ib_params;

int ilbm_ib_create(ilbm_ctx *ctx, const ilbm_ib_params *p, const ilbm_level_geom *g,
                   ilbm_ib **out);
/* Frees the body's device arrays in stream order on its context's stream
 * (after the work queued there and on the side stream); it does not
 * synchronise the device.  Destroy IB objects and batches before their
 * context. */
int ilbm_ib_destroy(ilbm_ib *ib);
int ilbm_ib_num_markers(const ilbm_ib *ib, int64_t *n);
/* Lower/upper corner (inclusive) of the cells whose force the IB may write. */
int ilbm_ib_force_region(const ilbm_ib *ib, int lo[3], int hi[3]);
/* update_forcing on a level held in nbox boxes (IBMarkerDF::update_forcing,
 * Source/IBM/IBMarkerDF.H:76-87, IBMarkerDF.cpp:1522-1917): reads rho, u of
 * every cell of the body's support band and writes box->force = dt*rho*a on
 * the valid cells of the force region (ilbm_ib_force_region).  Cells of the
 * force arrays outside that region are not touched (keep them zero).
 *   - One box that covers the level domain (self-filled or caller-filled
 *     ghosts), or one box whose valid cells hold the whole band: rho, u come
 *     from box->macro_in (two filled ghost layers) when set, else from f_in
 *     and force_prev.
 *   - Any other level (ILBM_GHOST_CALLER, e.g. an AMReX level cut by
 *     max_grid_size): a band cell takes rho, u from the box whose valid
 *     region holds it (the reference's EulerVel + FillBoundary,
 *     IBMarkerDF.cpp:1541-1566, 702-703), else from the caller-filled ghost
 *     of a box whose grown arrays reach it (macro_in grown by ngrow_m, or
 *     f_in / force_prev).  The force of a band cell goes to its box and, as
 *     the reference's FillBoundary of the force before the collision does
 *     (Source/Core/AdvanceLBMAtLevel.cpp:187-194), into the ghost cells of
 *     every other box whose grown force array holds the cell or a periodic
 *     image of it; force spread outside every box's valid cells is dropped
 *     (SumBoundary, IBMarkerDF.cpp:1511).  The boxes that meet the band are
 *     copied to the device in stream order; their arrays must stay valid
 *     until the call's work has run. */
int ilbm_ib_update_forcing(ilbm_ib *ib, const ilbm_box *boxes, int nbox,
                           const ilbm_level_params *p, double dt, double time);
/* One whole AdvancePhiAtLevel of a level with an immersed body
 * (Source/Core/AdvanceLBMAtLevel.cpp:20-394): update_forcing into box->force,
 * then the level step with that force.  In self-fill mode the IB chain runs on
 * a high-priority side stream concurrently with the collide-stream of every
 * cell outside the IB band (those cells carry no IB force), and the band
 * cells follow once the force is ready.  p's force region is set from the IB.
 * ib may be NULL (plain level step). */
int ilbm_advance_level(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                       ilbm_ib *ib, double dt, double time);
/* sum over markers of F*dv from the last update_forcing (synchronises) */
int ilbm_ib_last_marker_force_sum(ilbm_ib *ib, double out[3]);
/* iterations of the last IVC conjugate-gradient solve (synchronises); the
 * diagnostic counterpart of ibm.ivc_verbose (IBMarkerDF.cpp:1302-1313);
 * 0 when the system is solved through the stored inverse */
int ilbm_ib_solver_stats(ilbm_ib *ib, int *cg_iterations);
/* How the implicit-velocity-correction system A F = b is solved.
 * The reference factorises A = dv*S*S^T + reg*I once by dense LU and
 * back-substitutes each step while the markers stay put
 * (Source/IBM/IBMarkerDF.cpp:1015-1070, 1131, 1248-1300).  ILBM_IVC_DENSE
 * is the device counterpart: A^-1 is formed once per body (in-place
 * Gauss-Jordan on the GPU, n*n doubles, n <= ILBM_IVC_DENSE_MAX) and each step
 * solves with one dense matvec.  ILBM_IVC_CG solves every step by
 * preconditioned CG on the sparse operator (used for moving markers and
 * ivc_rebuild_matrix > 0), started from the linear extrapolation of the
 * body's last two solutions (the body keeps them, with their count, on the
 * device, so its own solves and a batch's alternate freely; selecting a
 * solver restarts from zero).  ILBM_IVC_AUTO (the default) takes the
 * stored inverse whenever it applies.  Selecting ILBM_IVC_DENSE where it does
 * not apply returns ILBM_ERR_UNSUPPORTED. */
#define ILBM_IVC_AUTO 0
#define ILBM_IVC_CG 1
#define ILBM_IVC_DENSE 2
#define ILBM_IVC_DENSE_MAX 8192
int ilbm_ib_set_ivc_solver(ilbm_ib *ib, int solver);
/* marker positions / interpolated velocity / force: n*3 doubles each, or NULL */
int ilbm_ib_markers(ilbm_ib *ib, double *xyz, double *uvw, double *force);

/* ---- force evaluation ---------------------------------------------------- */
/* Sum of boxes[b].force (3 components, the real type) over the valid cells of
 * every box inside [lo, hi] (NULL: whole boxes); 3 doubles, synchronous.  The
 * Eulerian forcing integral of ComputeIBForce is this sum times -dV/dt
 * (Source/Core/AmrCoreLBM.cpp:489-509).  The summation order is fixed for a
 * given list of boxes, so repeated calls return identical bits. */
int ilbm_force_integrals(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const int lo[3],
                         const int hi[3], double out_sum[3]);
/* The same sum as ilbm_force_integrals over one box whose force array is
 * `force`, for callers that cannot allocate
 * device memory while they run (no counterpart in the reference).  Hosts
 * such as AMReX reserve most of the device memory in their own arena at
 * start-up, serving loops admit work against a fixed memory budget, and
 * cudaMalloc / cudaFree can synchronise the device; ilbm_force_integrals
 * grows the context's scratch with cudaMalloc on first use, this call never
 * allocates: its partial sums live in a fixed array inside the library.
 *   - Limit: the clipped region may hold at most 8,388,608 cells (2048
 *     chunks of up to 4096 cells); larger regions return ILBM_ERR_RANGE
 *     without launching anything.
 *   - The first call on a device does a one-time set-up (it looks up the
 *     array's device address, which may load the library's device code on
 *     that device); make it before any stream capture begins.  The address
 *     is cached for the life of the process: a process that resets a device
 *     (cudaDeviceReset) must not call this entry point on that device again.
 *   - There is one array per device: calls that overlap on a device (from
 *     two host threads, or on two contexts of the same device) race on it
 *     and give wrong sums.  Each call synchronises the context's stream
 *     before returning, so calls from one host thread never overlap.
 *   - Results may differ from ilbm_force_integrals in the last bits (the
 *     partial sums are grouped differently); repeated calls on the same
 *     region return identical bits. */
int ilbm_force_integrals_noalloc(ilbm_ctx *ctx, const ilbm_box *box, const void *force,
                                 const int lo[3], const int hi[3], double out_sum[3]);
/* The force record of a step, without synchronising (no counterpart in the
 * reference, whose ComputeIBForce returns the sums at once,
 * Source/Core/AmrCoreLBM.cpp:456-631): enqueues on the context's stream the
 * Eulerian sum of ilbm_force_integrals (boxes[b].force over [lo, hi]) and
 * copies it, the
 * body's last marker force sum (ilbm_ib_last_marker_force_sum) and the body's
 * two status words into out[8] = {Eulerian sum (3), marker sum (3),
 * status word 0, status word 1}.  out should be pinned host memory (or device
 * memory), which the sums' last kernel writes directly (other memory gets a
 * copy on the stream); the values are there once the stream passes this point (an event
 * recorded after the call, or ilbm_sync), so a host can issue the next step
 * before it reads this one's record.  Status bits as reported by
 * ilbm_ib_last_marker_force_sum: word 0 bit 0 a stencil left the band, bit 1
 * the IVC operator's nonzero capacity, bit 2 CG not converged; word 1 bit 3 a
 * non-positive pivot of the stored inverse.  The next call on the context
 * reuses the record's device slot after this copy, in stream order. */
int ilbm_force_record_async(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, ilbm_ib *ib,
                            const int lo[3], const int hi[3], double *out);
/* Link-wise momentum exchange (IBForceEval::ComputeMomentumExchangeBodyForce,
 * Source/IBM/IBForceEval.H:24-32, IBForceEval.cpp:28-191) on the populations
 * boxes[b].f_in of a level held in nbox boxes, for a circle / sphere body
 * (x0, y0, z0, R); out = the reaction force on the body (3, synchronous).
 * Each fluid->solid link of a valid cell counts once; the opposite population
 * of the solid cell comes from the box whose valid region holds it (the
 * domain wrapped along periodic directions), else from the ghost layer of
 * the cell's own box, and a link neither reaches is left out.  With one box
 * covering the domain this is the reference's loop; summation order is
 * fixed for a given list of boxes. */
int ilbm_momentum_exchange(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox,
                           const ilbm_level_params *p, double x0, double y0, double z0, double R,
                           const double prob_lo[3], const double dx[3], int one_sided,
                           double out[3]);

/* ---- derived fields and refinement tags ---------------------------------- */
/* UpdateDerivedMacroFields / visPara (Source/Core/AmrCoreLBM.cpp:105-168,
 * Source/LBM/visPara.H:10-54) for a level held in one box with self-filled
 * ghosts: vorticity (2D: dv/dx - du/dy; 3D: |curl u|) by central differences
 * of the velocity of f (with the half force of force_prev, which may be
 * NULL) FillPatched one cell out, and pressure (rho - 1)/3, written on valid
 * cells into vor / pres (macro-array layout of `box`, real type; either may
 * be NULL); *vort_max = the largest vorticity of the level (ErrorEst's
 * vortMax, AmrCoreLBM.cpp:1047).  dx: the level's cell sizes.  Synchronises. */
int ilbm_derived_fields(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                        const void *f, const void *force_prev, const double dx[3], void *vor,
                        void *pres, double *vort_max);
/* ErrorEst tags (AmrCoreLBM.cpp:988-1185, Tagging.H:12-18): on every valid
 * cell, 0 inside the no-refine x zones (within no_refine_xlo of prob_lo[0] or
 * no_refine_xhi of prob_hi[0], when either is > 0), else 1 where |vor| >
 * threshold (the caller's thresholdRatio * vortMax) or, with use_box, where the
 * cell centre lies in [box_lo, box_hi] (the body refinement region), else 0.
 * levelset: NULL, or {x0, y0, z0, R, n_cells_band, dx_min} of a cylinder /
 * sphere body (the cylinder-geometry branch, AmrCoreLBM.cpp:1073-1132 with
 * levelset_tagging, Tagging.H:27-35): a cell is also tagged where the signed
 * distance |x - x0| - R of its centre is below (n_cells_band + 0.5) * dx_min,
 * which takes in the body's interior.  The reference uses n_cells_band = 5.
 * tags: device array of one byte per valid cell, i fastest; *ntagged = count.
 * Synchronises. */
int ilbm_tag_cells(ilbm_ctx *ctx, const ilbm_box *box, const void *vor, double threshold,
                   int use_box, const double box_lo[3], const double box_hi[3],
                   double no_refine_xlo, double no_refine_xhi, const double prob_lo[3],
                   const double prob_hi[3], const double dx[3], const double *levelset,
                   void *tags, int64_t *ntagged);

/* ---- static two-level hierarchy ------------------------------------------
 * A coarse level equal to its domain (ILBM_GHOST_SELF) and one fine box of
 * refinement ratio 2 (ILBM_GHOST_CALLER, fine domain = the coarse domain
 * refined by 2, box lo even and hi odd in fine indices, at least two coarse
 * cells inside every face of the domain), advanced as
 * AmrCoreLBM::timeStepWithSubcycling does for max_level = 1
 * (Source/Core/AmrCoreLBM.cpp:1690-1755):
 *   1. the coarse level steps by dt (coarse->f_in, macro_in -> f_out,
 *      macro_out);
 *   2. the fine level steps twice by dt/2 at t and t + dt/2; before each
 *      substep every fine ghost cell gets the coarse macro fields at the
 *      substep's time (old, new, or their linear time interpolation,
 *      GetDataMacro :2239-2269), interpolated by cell-conservative linear
 *      interpolation with monotonised-central limited slopes (AMReX's
 *      cell_cons_interp in FillPatchMacro :2166-2198), and ghost populations
 *      equal to the equilibrium of that state (FillPatchMesoscopic's
 *      coarse-fine overwrite, :1566-1626).  The body `ib` (or NULL) lives
 *      on the fine level (AdvanceLBMAtLevel.cpp:30, 73-93);
 *   3. average-down of ratio 2 (AverageDownTo :1519-1527) of the fine
 *      populations and macro fields onto coarse->f_out / macro_out.
 * Stored macro fields: the coarse level's macro_in / macro_out hold them on
 * the covered cells grown by two coarse cells (what average-down writes and
 * the fine ghost fill reads); elsewhere, and on the fine level, rho and u are
 * recovered from f^n and F^{n-1}, which equals the stored value.  The first
 * step after initialisation (flags ILBM_TWO_LEVEL_FIRST_STEP) instead reads
 * both levels' initial macro fields everywhere (coarse->macro_in,
 * fine->macro_in).  With a body, its forcing for the first substep overlaps
 * the coarse step.
 * Buffers: the fine level's f_in holds the new fine state on return (two
 * substeps swap f_in / f_out twice), force / force_prev hold the first /
 * second substep's forces; the caller swaps the coarse in / out pairs.
 * Asynchronous on the context's stream. */
#define ILBM_TWO_LEVEL_FIRST_STEP 1
int ilbm_advance_two_level(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                           const ilbm_box *fine, const ilbm_level_params *pf, ilbm_ib *ib,
                           double dt, double time, int flags);

/* ilbm_advance_two_level followed by the step's force record (ib must not be
 * NULL), taken as ilbm_force_record_async takes it (region [lo, hi] of the
 * fine level's force
 * of the second substep, fine->force_prev on return; the body's last marker
 * force sum; its two status words) into out[8], with the same values: when
 * out is pinned host memory (or memory of this device) the record's kernels
 * run on the context's side stream right after the second substep's forcing,
 * beside the rest of the step, which only reads what they read, and write out
 * directly; the step's end on the context's stream waits for them, so out is
 * ready once the stream passes this call.  Other memory gets the step, then
 * ilbm_force_record_async.  Replaces the caller's ilbm_advance_two_level +
 * ilbm_force_record_async pair (ComputeIBForce after the finest level's
 * substeps, Source/Core/AmrCoreLBM.cpp:456-631). */
int ilbm_advance_two_level_recorded(ilbm_ctx *ctx, const ilbm_box *coarse,
                                    const ilbm_level_params *pc, const ilbm_box *fine,
                                    const ilbm_level_params *pf, ilbm_ib *ib, double dt,
                                    double time, int flags, const int lo[3], const int hi[3],
                                    double *out);
/* average-down alone (InitData's AverageDown after the levels are made,
 * AmrCoreLBM.cpp:710-720): fine f_in / macro_in onto coarse f_in / macro_in,
 * for any two adjacent levels of a hierarchy (the coarse one self-filled and
 * equal to its domain, or one box in caller mode holding the fine box two
 * coarse cells inside it) */
int ilbm_average_down(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                      const ilbm_box *fine, const ilbm_level_params *pf);

/* ---- static hierarchy of any depth --------------------------------------
 * nlev levels (2..8), one box each: level 0 equal to its domain
 * (ILBM_GHOST_SELF), level l > 0 a box of the domain of level l-1 refined by
 * 2 (ILBM_GHOST_CALLER, lo even and hi odd, coarsened at least two cells
 * inside the box of level l-1), advanced as AmrCoreLBM::
 * timeStepWithSubcycling does (Source/Core/AmrCoreLBM.cpp:1690-1755): a
 * level's step by its dt (dt / 2^l), then two substeps of level l+1 at t and
 * t + dt/2 whose ghost cells are filled from level l's macro fields at that
 * time (as ilbm_advance_two_level's fine level), then the average-down of
 * level l+1 onto level l (AverageDownTo, :1519-1527); recursively.  The body
 * `ib` (or NULL) lives on the finest level, whose steps overlap its forcing
 * chain with the cells outside its band.
 * Buffers: every level with a finer one carries stored macro fields
 * (macro_in, macro_out; kept on the finer box coarsened and grown by two
 * cells after the first step); the finest level's f_in, and every finer
 * level's f_in / macro_in, hold the new state on return (an even number of
 * steps swaps them back); level 0's new state is in its f_out / macro_out and
 * the caller swaps that pair.  force / force_prev of the finest level: the
 * force of its last substep is in force_prev on return.  With flags
 * ILBM_HIERARCHY_FIRST_STEP each level's first step reads its initial macro
 * fields everywhere (after ilbm_init_equilibrium and ilbm_average_down from
 * the finest level up).  nlev = 2 is the schedule of ilbm_advance_two_level
 * without its overlap of the coarse step with the fine level's forcing.
 * Asynchronous on the context's stream. */
#define ILBM_HIERARCHY_FIRST_STEP 1
int ilbm_advance_hierarchy(ilbm_ctx *ctx, int nlev, const ilbm_box *boxes,
                           const ilbm_level_params *params, ilbm_ib *ib, double dt, double time,
                           int flags);

/* ---- state I/O ----------------------------------------------------------
 * Checkpoint and restart of one level box (and its immersed body): the
 * checkpoint the reference declares but leaves as commented-out stubs
 * (AmrCoreLBM::WriteCheckpointFile / ReadCheckpointFile,
 * Source/Core/AmrCoreLBM.cpp:1932-2115), in a format of this library: a
 * header, then sections of valid-cell data (component-major, i fastest) in
 * the storage's own bits, each closed by a 64-bit word hash.  A restart from
 * it continues bit for bit where the saved run left off.
 *   box->f_in          f^n (saved / restored, storage type)
 *   box->macro_in      rho,u,v,w when the next step still reads the stored
 *                      macro fields (the first step after initialisation),
 *                      else NULL; on restore it may be given for a file
 *                      without them (flags then says so)
 *   box->force_prev    F^{n-1} (3 comps) of a level with a body, else NULL
 *   ib                 the body (marker positions, velocities and forces,
 *                      last force sum, the CG start vector), or NULL; on
 *                      restore it must have been created with the same
 *                      parameters on the same level
 *   f16 storage keeps its raw half bits: restore with the same f16_scale.
 * Both synchronise the context's stream.  Errors: ILBM_ERR_IO (file, short
 * read, hash mismatch), ILBM_ERR_ARG (the file does not match the lattice,
 * storage, box, body or the sections asked for).  A read is checked section
 * by section as it is restored: when ilbm_checkpoint_read fails with
 * ILBM_ERR_IO after its header was accepted, the box arrays and the body may
 * already be partly overwritten and are undefined; restore them from
 * another checkpoint or re-initialise them. */
#define ILBM_ERR_IO (-7)
#define ILBM_CKPT_MACRO 1 /* flags: the file holds stored macro fields */
#define ILBM_CKPT_FORCE 2 /*        F^{n-1} */
#define ILBM_CKPT_BODY 4  /*        an immersed body */
typedef struct {
  int64_t istep;     /* steps taken by the level */
  double time;       /* time of the next step */
  double user[16];   /* caller state carried with the checkpoint */
  int flags;         /* read: ILBM_CKPT_* of the file (ignored on write) */
} ilbm_checkpoint_meta;
int ilbm_checkpoint_write(ilbm_ctx *ctx, const ilbm_box *box, ilbm_ib *ib,
                          const ilbm_checkpoint_meta *meta, const char *path);
int ilbm_checkpoint_read(ilbm_ctx *ctx, const ilbm_box *box, ilbm_ib *ib,
                         ilbm_checkpoint_meta *meta, const char *path);

/* AMReX plotfile of one level held in one box (AmrCoreLBM::WritePlotFile,
 * PlotFileMF and PlotFileVarNames, Source/Core/AmrCoreLBM.cpp:1756-1930, which
 * call AMReX's WriteMultiLevelPlotfile): the directory `dir` gets Header,
 * Level_0/Cell_H and Level_0/Cell_D_00000 ("HyperCLaw-V1.1", one FAB of
 * little-endian doubles), readable by AMReX-based tools.  Components: rho,
 * ux, uy, uz, vor, Pressure (macro of f^n with the half force of F^{n-1},
 * vorticity and pressure as ilbm_derived_fields), f_new_0 .. f_new_{Q-1}
 * (unshifted populations), and with `levelset` set, phi = |x - c| - R of a
 * cylinder / sphere body, whose interior (phi < 0) then shows the body
 * velocity and zero vorticity (PlotFileMF's masking).  Self-filled ghosts,
 * box equal to the domain; uses box->f_in and box->force_prev.
 * Synchronises. */
typedef struct {
  double prob_lo[3], prob_hi[3], dx[3];
  double time;
  int istep;
  int levelset;          /* 1: append phi and mask the body interior */
  double ls_center[3];
  double ls_radius;
  double body_u[3];      /* ubx, uby, ubz */
} ilbm_plot_info;
int ilbm_plotfile_write(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                        const ilbm_plot_info *info, const char *dir);

/* ---- batch engine (no counterpart in the reference) ---------------------
 * Many independent single-level cases of the context's lattice and storage
 * form, advanced together: per step one launch per immersed-boundary stage
 * for all cases and one persistent collide-stream kernel over a tile table of
 * every case's cells; two consecutive steps are replayed as a CUDA graph.
 * A case is one box equal to its level domain with self-filled ghosts
 * (ILBM_GHOST_SELF).  It joins after its first step has been taken through
 * ilbm_advance_level (which reads the stored macro fields and builds the IVC
 * operator); from then on its state lives in the buffers of `box`, whose
 * f_in/f_out and force/force_prev swap every step.  Bodies use one MDF
 * iteration.  Adding, removing or re-tiling settles the batch (synchronises
 * and rebuilds its tables at the next step). */
typedef struct ilbm_batch ilbm_batch;
/* rec_slots: per-case force records kept on the device between read-backs
 * (0 selects 256) */
int ilbm_batch_create(ilbm_ctx *ctx, int rec_slots, ilbm_batch **out);
int ilbm_batch_destroy(ilbm_batch *b);
/* time: time of the case's next step; max_steps: steps the case may take in
 * the batch (sizes the pitching-kinematics table) */
int ilbm_batch_add(ilbm_batch *b, const ilbm_box *box, const ilbm_level_params *p, ilbm_ib *ib,
                   double dt, double time, int max_steps, int *case_id);
int ilbm_batch_remove(ilbm_batch *b, int case_id);
/* advances every case by nsteps, each case stopping once it has taken the
 * max_steps it was added with (asynchronous, except for record read-backs
 * every rec_slots steps) */
int ilbm_batch_step(ilbm_batch *b, int nsteps);
/* parity 0: box.f_in (with box.force_prev holding F^{n-1}) hold the current
 * state, 1: box.f_out (with box.force); synchronises */
int ilbm_batch_case_state(ilbm_batch *b, int case_id, int *parity, int64_t *steps_done,
                          double *time);
/* the case's per-step force records, oldest first, 6 doubles each: Eulerian
 * force sum over the IB force region (3) and marker force sum (3); with out
 * NULL, *nrec = number available.  Synchronises. */
int ilbm_batch_records(ilbm_batch *b, int case_id, double *out, int max_rec, int *nrec);
/* tile width (threads per block: 64, 128, 256) and resident blocks per SM
 * (0: as many as fit) of the batched collide-stream */
int ilbm_batch_set_tiles(ilbm_batch *b, int tile_w, int ctas_per_sm);
/* times every tile width and block count on the batch itself (advancing every
 * case by the trial steps of each candidate) and keeps the fastest */
int ilbm_batch_tune(ilbm_batch *b, int trial_steps, int *tile_w, int *ctas_per_sm,
                    float *ms_per_step);
int ilbm_batch_size(ilbm_batch *b, int *ncase, int64_t *cells);
/* ids, steps taken and steps remaining of the first max_cases cases (any of
 * the arrays may be NULL), *ncase = number of cases; one synchronisation */
int ilbm_batch_progress(ilbm_batch *b, int max_cases, int *ids, int64_t *steps_done,
                        int *remaining, int *ncase);

#ifdef __cplusplus
}
#endif
#endif /* ILBM_B200_H */
