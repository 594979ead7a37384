/*
 * rbsim.h -- C ABI of librbsim.so, the B200 solver hot path of river-basin-sim.
 *
 * The reference path is Python driving NVIDIA Warp kernels behind a scheme module
 * with two calls (solver/core/schemes.py:1-26, :41-52):
 *     compute_dt(state, alpha, dt_max) -> float
 *     step(state, dt, rain, rain_scale, t)      (LI adds limit=True)
 * plus the point-source injector (solver/processes/inflow.py:167), the Exner
 * activation (solver/processes/morphology.py:223) and the float64 mass ledger
 * (solver/core/massbalance.py:66). This header is what a ctypes binding of that
 * seam calls. Conventions:
 *   - Every buffer is caller-owned device memory (raw pointers; nothing here
 *     frees or allocates device memory). Library scratch lives in a caller-
 *     allocated workspace sized by rb_*_workspace_bytes and zeroed once by
 *     rb_workspace_init.
 *   - Layout: row-major float32, cells (ny, nx), x-faces (ny, nx+1),
 *     y-faces (ny+1, nx) (solver/core/grid.py:9-31). qx > 0 flows +x, qy > 0 flows
 *     +y (increasing row index).
 *   - Fields that neighbouring cells read (h, qx, qy; h, hu, hv) are double
 *     buffered: a step reads buffer [cur] and writes buffer [cur ^ 1]. The caller
 *     flips `cur` after a successful step.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream). Calls are
 *     asynchronous unless documented as synchronising; calls on one workspace
 *     must not overlap.
 *   - Return value: RB_OK (0) or a negative RB_ERR_*; rb_last_error() gives the
 *     message of the calling thread's last failure.
 */
#ifndef RBSIM_H
#define RBSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB_OK 0
#define RB_ERR_ARG (-1)      /* bad shape, size or pointer (the reference raises ValueError) */
#define RB_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define RB_ERR_DEVICE (-3)   /* a kernel raised a device error bit (see RB_DEVERR_*) */
#define RB_ERR_TIMEOUT (-4)  /* a bounded device wait expired */
#define RB_ERR_STEP (-5)     /* non-positive or non-finite timestep (scheduler.py:221-227) */

/* Device error bits, OR-ed into the workspace error word. */
#define RB_DEVERR_NONFINITE 1u /* a step produced a NaN/inf depth */
#define RB_DEVERR_CLOCK 2u     /* the device clock produced a non-positive timestep */
#define RB_DEVERR_STEPS 4u     /* the device clock hit its step budget before its target */
#define RB_DEVERR_TIMEOUT 8u   /* a bounded device wait (a tensor-memory copy) gave up */

/* Edge order of every per-edge array: north, south, east, west (state.py:35). */
enum { RB_EDGE_NORTH = 0, RB_EDGE_SOUTH = 1, RB_EDGE_EAST = 2, RB_EDGE_WEST = 3 };
/* Edge kinds (state.py:84-96). */
enum { RB_BC_CLOSED = 0, RB_BC_OPEN = 1, RB_BC_STAGE = 2 };

/* Local-inertial state: the arrays of solver/core/state.py:38-96 that the step
 * touches. Optional physics is armed by a non-NULL pointer, as the reference arms
 * it by presence (state.py:98-171, sediment.py:658). */
typedef struct rb_li_fields {
  int32_t ny, nx;
  double dx;                 /* Grid.dx (grid.py:52-63) */
  float *h[2];               /* depth (ny, nx), double buffered */
  float *qx[2];              /* x-face discharge (ny, nx+1), double buffered */
  float *qy[2];              /* y-face discharge (ny+1, nx), double buffered */
  const float *z;            /* bed (ny, nx) */
  const float *n;            /* Manning roughness (ny, nx) */
  float *h_comp;             /* Kahan residue of areal sources (sources.py), or NULL */
  const float *rain_field;   /* rain rate field m/s (state.py:106), or NULL */
  const float *infil;        /* infiltration rate m/s (state.py:98), or NULL */
  int32_t bc[4];             /* RB_BC_* per edge; LI honours closed and open */
  /* Morphology (sediment.py:549-571); d50 == NULL leaves the bed static. */
  const float *d50;
  float *qs_int_x, *qs_comp_x; /* (ny, nx+1) transport integral + Kahan residue */
  float *qs_int_y, *qs_comp_y; /* (ny+1, nx) */
  /* Sub-grid channels (solver/core/channels.py:182-312); chan_w == NULL: unarmed.
   * Geometry per cell (w = d = 0 where there is no channel; callers validate as
   * channels.py:214-262 does); the split face discharges are double buffered
   * like qx / qy: the step reads [cur] and writes [cur ^ 1]. */
  const float *chan_w, *chan_d, *chan_n; /* (ny, nx) width m, bank-full depth m, roughness */
  float *qx_ch[2], *qx_fp[2];            /* (ny, nx+1) channel / floodplain x-face discharge */
  float *qy_ch[2], *qy_fp[2];            /* (ny+1, nx) */
} rb_li_fields;

/* HLLC state (state.py:52-57, hllc.py:96-152). */
typedef struct rb_hllc_fields {
  int32_t ny, nx;
  double dx;
  float *h[2], *hu[2], *hv[2]; /* (ny, nx), double buffered */
  const float *z, *n;
  float *h_comp;
  const float *rain_field;
  const float *infil;
  int32_t bc[4];               /* closed = reflective wall, open = transmissive + banked,
                                  fixed_stage = prescribed-surface ghost + banked */
} rb_hllc_fields;

/* Per-step forcing, as the reference passes it to step(): dt and rain in float64
 * host precision (each kernel rounds them exactly where the reference does). */
typedef struct rb_step_args {
  double dt;          /* seconds */
  double rain;        /* uniform rain rate, m/s (scalar path) */
  double rain_scale;  /* temporal multiplier of the rain field */
  int32_t limit;      /* LI donor limiter (local_inertial.py:551); ignored by HLLC */
  int32_t reserved;
  double stage[4];    /* HLLC fixed_stage surface per edge at t + dt/2 (hllc.py:1308-1312) */
} rb_step_args;

/* --- workspace ----------------------------------------------------------- */
/* Bytes of library scratch a domain of this size needs (reduction slots, the
 * error word, per-tile float64 ledger partials, HLLC stage-1 state). */
size_t rb_li_workspace_bytes(int32_t ny, int32_t nx);
size_t rb_hllc_workspace_bytes(int32_t ny, int32_t nx);
/* Zero a workspace (ledger partials, error word). Asynchronous on `stream`. */
int rb_workspace_init(void *ws, size_t bytes, void *stream);

/* --- local-inertial scheme (solver/core/local_inertial.py) ------------------ */
/* One step: replaces step() (local_inertial.py:547-727): eta, both face updates
 * with semi-implicit Manning, closed edges, donor limiter, bedload integral,
 * continuity, compensated or plain rain, infiltration and open-edge sinks, fused
 * in one launch. Infiltration and open-edge losses are banked into the
 * workspace ledger (replacing the per-cell float64 loss_cum). */
int rb_li_step(const rb_li_fields *f, int32_t cur, const rb_step_args *a, void *ws, void *stream);
/* Replaces compute_dt() (local_inertial.py:515-544). Synchronising: reduces
 * max(h) of buffer [cur] on the device and returns dt in *dt_out (host). */
int rb_li_compute_dt(const rb_li_fields *f, int32_t cur, double alpha, double dt_max, void *ws, void *stream,
                     double *dt_out);

/* --- HLLC scheme (solver/core/hllc.py) ---------------------------------- */
/* One SSP-RK2 step: replaces step() (hllc.py:1272-1373) in two launches (one
 * per Heun stage). Open and fixed_stage boundary flux and infiltration are
 * banked into the workspace ledger (replacing loss_cum). */
int rb_hllc_step(const rb_hllc_fields *f, int32_t cur, const rb_step_args *a, void *ws, void *stream);
/* One Heun stage of rb_hllc_step (stage 1: U^n -> U1 in the workspace; stage 2:
 * (U^n, U1) -> U^{n+1} with friction and sources). rb_hllc_step == stage 1 then
 * stage 2; split so a caller can time or interleave the two launches. */
int rb_hllc_stage(const rb_hllc_fields *f, int32_t cur, const rb_step_args *a, void *ws, void *stream,
                  int32_t stage);
/* Replaces compute_dt() (hllc.py:972-990). Synchronising. */
int rb_hllc_compute_dt(const rb_hllc_fields *f, int32_t cur, double alpha, double dt_max, void *ws, void *stream,
                       double *dt_out);

/* --- sources, morphology, ledger ---------------------------------------- */
/* Point sources: replaces the _inject_point_sources[_c] launch of
 * InflowInjector.apply (inflow.py:74-113, :183-199). comp == NULL adds plainly.
 * rows / cols (device, nsrc each) must name distinct cells inside the ny x nx grid, as
 * InflowInjector checks on the host; a source outside the grid adds nothing. */
int rb_inject_points(float *h, int32_t ny, int32_t nx, int32_t nsrc, const int32_t *rows, const int32_t *cols,
                     const float *add_depth, float *comp, void *stream);
/* Exner activation: replaces exner_update + rebuild_bed (sediment.py:383-441) as
 * launched by MorphologyProcess.advance (morphology.py:261-270); then zeroes the
 * transport integrals and keeps their Kahan residue (sediment.py:513-524). */
int rb_exner_apply(int32_t ny, int32_t nx, double dx, float *qs_int_x, float *qs_int_y, const float *dz_lo,
                   const float *dz_hi, float inv_one_minus_p, double *dz_cum, double *dz_unapplied, const float *z0,
                   float *z, void *stream);
/* Ledger outflow: the float64 sum of everything banked into the workspace
 * ledger since rb_workspace_init, in metres of depth summed over cells (the
 * reference's loss_cum.sum(), massbalance.py:173-177). Synchronising. */
int rb_ledger_loss(void *ws, int32_t ny, int32_t nx, void *stream, double *out);
/* Deterministic float64 sum of a float32 field (the stored-volume term,
 * massbalance.py:292-295), fixed reduction order. Synchronising. */
int rb_sum_f64(const float *x, int64_t n, void *ws, size_t ws_bytes, void *stream, double *out);
/* Read and clear the workspace device error word. Synchronising. */
int rb_read_device_error(void *ws, void *stream, uint32_t *err_out);

/* --- device-resident clock ----------------------------------------------------
 * The run loop of solver/run.py:369-388 with the scheduler of
 * solver/scheduler.py:171-246, moved onto the device: a one-thread plan kernel
 * turns the max the previous step folded into the clock into compute_dt's dt,
 * clamps it with fill_span to the next sync time, gates the rain and banks its
 * volume, all in float64 in the reference's operation order, so K steps run
 * without host round trips and can be captured in a CUDA graph. The clock lives
 * in the workspace. Point sources (inflow.py:167-200) and fixed_stage curves
 * (boundaries.py:199-220) are sampled on the device from tables in device memory. */
typedef struct rb_clock_config {
  double alpha, dt_max;      /* compute_dt arguments */
  double t0;                 /* simulated time of the current state */
  const double *sync;        /* device array, ascending: output times, forcing
                                breakpoints, slow-process activations, end time
                                (scheduler.py:136-147); must outlive the clock */
  int32_t nsync;
  int32_t rain_is_field;     /* 0: uniform rain_rate; 1: the state's rain field */
  double rain_rate;          /* m/s while t < rain_until - 1e-6 (run.py:378) */
  double rain_until;         /* rain duration, s */
  double rain_field_sum;     /* float64 sum of the rain field, m/s (run.py:276) */
  int32_t limit;             /* LI donor limiter */
  int32_t nsrc;              /* point sources (0: none) */
  const int32_t *src_cell;   /* device, nsrc: row * nx + col, distinct cells (one outside the grid adds nothing) */
  const int32_t *knot_off;   /* device, nsrc + 1: source k's hydrograph knots are [off[k], off[k+1]) */
  const double *knot_t;      /* device: knot times (s), non-decreasing per source */
  const double *knot_q;      /* device: knot discharges (m^3/s) */
  float *src_comp;           /* device, nsrc: Kahan residue per source, or NULL for the plain add */
  int32_t stage_off[5];      /* fixed_stage curve of edge e: stage_t/v[off[e] .. off[e+1]) (empty: none) */
  int32_t reserved;
  const double *stage_t;     /* device: curve knot times */
  const double *stage_v;     /* device: curve levels (m, stepping datum) */
} rb_clock_config;

typedef struct rb_clock_state {
  double t;            /* simulated time of the committed state */
  double dt;           /* the last planned step */
  double rain_volume;  /* areal rain banked since start, m^3 (ledger add_rain_step) */
  double inflow_volume; /* point-source volume requested since start, m^3 (InflowInjector.apply) */
  int32_t cur;         /* the buffer holding the state */
  int32_t steps;       /* steps taken since start */
  uint32_t err;        /* RB_DEVERR_* bits raised by the clock or the steps */
  int32_t reserved;
} rb_clock_state;

/* Arm the clock for the state in buffer [cur] (seeds compute_dt's reduction).
 * Not capturable: copies the configuration from host memory. */
int rb_li_clock_start(const rb_li_fields *f, int32_t cur, const rb_clock_config *cfg, void *ws, void *stream);
int rb_hllc_clock_start(const rb_hllc_fields *f, int32_t cur, const rb_clock_config *cfg, void *ws, void *stream);
/* Re-seed compute_dt's reduction from the state in buffer [cur] after something
 * outside the clocked steps changed it between spans (a reservoir transfer,
 * solver/processes/reservoir.py:215-263, runs between ticks and the reference's
 * next compute_dt reads the changed state). Capturable. */
int rb_li_clock_reseed(const rb_li_fields *f, int32_t cur, void *ws, void *stream);
int rb_hllc_clock_reseed(const rb_hllc_fields *f, int32_t cur, void *ws, void *stream);
/* Let the clock run until t_target (a sync time) or max_steps more steps. Capturable. */
int rb_clock_set_target(void *ws, double t_target, int32_t max_steps, void *stream);
/* One plan (commit the previous step, plan the next). Capturable. */
int rb_clock_plan(void *ws, void *stream);
/* One clocked launch: a no-op when the plan stopped the clock. Capturable. */
int rb_li_step_clocked(const rb_li_fields *f, void *ws, void *stream);
int rb_hllc_stage_clocked(const rb_hllc_fields *f, int32_t stage, void *ws, void *stream);
/* The planned step's point-source injection into buffer [cur] of (h0, h1). Capturable. */
int rb_clock_inflow(const float *h0, const float *h1, void *ws, void *stream);
/* nsteps x (plan, [point sources when with_sources], step). Capturable. */
int rb_li_enqueue_steps(const rb_li_fields *f, int32_t nsteps, int32_t with_sources, void *ws, void *stream);
int rb_hllc_enqueue_steps(const rb_hllc_fields *f, int32_t nsteps, int32_t with_sources, void *ws, void *stream);
/* Commit the last planned step and read the clock. Synchronising. */
int rb_clock_read(void *ws, void *stream, rb_clock_state *out);

/* --- ensembles and serving ------------------------------------------------------
 * Many independent domains (local inertial and HLLC mixed) stepped together: each
 * keeps its own fields, workspace and device clock (its own dt, rain and target),
 * and one persistent kernel per scheme walks the (domain, tile) work-list of all of
 * them; a domain whose clock has stopped costs one early return per tile. A
 * domain's arithmetic is exactly that of rb_li_step / rb_hllc_step, so its result
 * does not depend on the batch it is in. No reference counterpart: the reference
 * runs one scenario per process (solver/run.py:530). The ensemble workspace
 * (clocks, parameter blocks, tile maps) is caller-allocated, sized by the layout. */
typedef struct rb_ensemble_layout {
  int32_t ndom, n_li, n_hllc;
  int32_t li_variant, hllc_variant;  /* tile shapes: LI 0 = 32x16, 1 = 32x8, 2 = 64x8, 3 = 32x32; HLLC 0 = 32x16, 1 = 32x8, 2 = 32x32 */
  int32_t li_grid, hllc_grid;        /* persistent grid sizes (set by rb_ensemble_init) */
  int32_t reserved;
  int64_t li_tiles, hllc_tiles;
  int64_t off_clocks, off_li, off_hllc, off_map_li, off_map_hllc, off_targets, bytes;
} rb_ensemble_layout;

/* Host only: the workspace layout of ndom domains (scheme 0 = LI, 1 = HLLC). */
int rb_ensemble_layout_make(int32_t ndom, const int32_t *scheme, const int32_t *ny, const int32_t *nx,
                            int32_t li_variant, int32_t hllc_variant, rb_ensemble_layout *out);
/* Fill the ensemble workspace from each domain's fields (li[] for the LI domains
 * and hl[] for the HLLC domains, in domain order), its own workspace (dom_ws[d],
 * sized by rb_*_workspace_bytes), clock configuration (no point sources or stage
 * curves) and current buffer; seeds every domain's dt reduction. Synchronising. */
int rb_ensemble_init(rb_ensemble_layout *L, void *ens, const int32_t *scheme, const rb_li_fields *li,
                     const rb_hllc_fields *hl, void *const *dom_ws, const rb_clock_config *cfg, const int32_t *cur,
                     void *stream);
/* Per-domain span targets (host arrays). Synchronising. */
int rb_ensemble_set_targets(const rb_ensemble_layout *L, void *ens, const double *t_target, const int32_t *max_steps,
                            void *stream);
/* nsteps x (plan every clock, LI tiles, HLLC stage 1 tiles, HLLC stage 2 tiles). Capturable. */
int rb_ensemble_enqueue(const rb_ensemble_layout *L, void *ens, int32_t nsteps, void *stream);
/* Commit and read every domain's clock into out[ndom]. Synchronising. */
int rb_ensemble_read(const rb_ensemble_layout *L, void *ens, rb_clock_state *out, void *stream);

/* --- kernel tuning -------------------------------------------------------------
 * No counterpart in the reference. A process-wide choice among the HLLC stage
 * kernel's variants (tile shape, block size, faces per work item, load batching;
 * 7 stages interior tiles with tensor-memory copies, falling back to plain loads
 * where a row is not a multiple of 16 bytes; 8 does the same with one persistent block
 * per resident slot that prefetches the halo of its next tile). Every variant computes bit-identical
 * results; this is a speed knob only, read at each launch (a captured graph keeps
 * the variant it was captured with). The library starts with the variant measured
 * fastest on B200 (6: 32 x 32 tiles, 640 threads). */
int rb_hllc_set_kernel_variant(int32_t variant);
int rb_hllc_kernel_variants(int32_t *count);
/* The same for the local-inertial step (tile 32 x 16, 32 x 32, 64 x 16, 32 x 8, and
 * 32 x 16 held to 48 registers; a state with sub-grid channels always uses 32 x 16).
 * The library starts with variant 1 (32 x 32 tiles, 512 threads). */
int rb_li_set_kernel_variant(int32_t variant);
int rb_li_kernel_variants(int32_t *count);

/* --- arithmetic of the step kernels ---------------------------------------------
 * No counterpart in the reference. A process-wide choice of the arithmetic the
 * single-domain local-inertial step and HLLC stage kernels run with:
 *  RB_ARITH_EXACT (the default): one IEEE rounding per operation in the
 *    reference's expression order, no fused multiply-add, IEEE division and square
 *    root, deterministic powers -- bit-identical to the CPU oracle;
 *  RB_ARITH_FAST: the same kernels built with contracted multiply-adds and the
 *    hardware's approximate division, square root and powers, the arithmetic of a
 *    GPU build of the reference; it agrees with the exact build to the solver
 *    tolerance, not bit for bit. Compensated (Kahan) additions stay exact.
 * Read at each launch (a captured graph keeps the mode it was captured with).
 * Ensembles always run the exact arithmetic. */
#define RB_ARITH_EXACT 0
#define RB_ARITH_FAST 1
int rb_set_arith_mode(int32_t mode);
int rb_arith_mode(int32_t *mode);
/* The launch configuration in force now: LI kernel variant, HLLC kernel variant and
 * arithmetic mode. A host that caches captured graphs keys them on it, since a graph
 * keeps the kernels it was captured with. */
int rb_launch_config(int32_t *li_variant, int32_t *hllc_variant, int32_t *arith_mode);

/* --- reservoir release (solver/processes/reservoir.py) -------------------------
 * Boxes are inclusive (r0, c0, r1, c1), as Structure.pool / .outlet. h is the
 * current depth buffer, modified in place between steps. */
/* reservoir.py:97-121 _withdraw_pool: h -= h * scale over the pool box (scale in
 * [0, 1]); taken (device, (r1-r0+1) x (c1-c0+1) float64) receives each cell's exact
 * float64 depth removed, for the host to sum as reservoir.py:246 does. */
int rb_reservoir_withdraw(float *h, int32_t ny, int32_t nx, int32_t r0, int32_t c0, int32_t r1, int32_t c1,
                          float scale, double *taken, void *stream);
/* reservoir.py:124-144 _deliver_release: h += float32(add_depth) over the outlet box;
 * the rounding shortfall (add_depth - actual gain, summed over the box) is banked in
 * the workspace's loss ledger, where the reference banks it in loss_cum. */
int rb_reservoir_deliver(float *h, int32_t ny, int32_t nx, int32_t r0, int32_t c0, int32_t r1, int32_t c1,
                         double add_depth, void *ws, void *stream);

/* --- a step that allocates nothing ---------------------------------------------
 * No counterpart in the reference. rb_hllc_step with its scratch in a static
 * device array inside the library instead of a caller-allocated workspace, for
 * callers that cannot allocate device memory: hosts whose own allocator owns all
 * device memory (an embedding engine, a plugin host that forbids allocation after
 * start-up), a framework whose allocator is frozen while it records a CUDA graph,
 * or a loop that cannot take cudaMalloc's implicit device synchronisation.
 * Limit: 1,048,576 cells (e.g. 1024 x 1024); larger grids return RB_ERR_ARG.
 * The array (~14 MiB) is held until exit by every GPU that loads the library's
 * device code; under CUDA's lazy module loading (the default since CUDA 12.2) a
 * GPU loads it, and so reserves the array, at the first call on that GPU. Make
 * that first call at start-up: before any stream capture on the device (it looks
 * up the array's address with cudaGetSymbolAddress) and before the host's own
 * allocator takes the rest of the memory. Every call shares the array: the loss
 * ledger is cleared at the start of each call, and calls that overlap on the GPU
 * race. If loss_out (device, one double) is given, it receives the depth this step
 * banked through open / fixed_stage edges and infiltration (metres summed over
 * cells). A step that produces a non-finite state sets RB_DEVERR_NONFINITE in the
 * array's error word, which stays set until rb_hllc_noalloc_read_error reads it.
 * Calls no allocation routine. */
int rb_hllc_step_noalloc(const rb_hllc_fields *f, int32_t cur, const rb_step_args *a, double *loss_out,
                         void *stream);
/* The error bits rb_hllc_step_noalloc calls on the current device have set since
 * the last read (RB_DEVERR_*), then cleared. Synchronises `stream`. No counterpart
 * in the reference (its kernels raise no device-side errors). */
int rb_hllc_noalloc_read_error(uint32_t *err_out, void *stream);

/* --- diagnostics ------------------------------------------------------------ */
/* Message of this thread's last failed call (empty if none). Returns its length. */
int rb_last_error(char *buf, size_t n);
/* Library version and the SM architecture it was built for (e.g. 100). */
int rb_version(int32_t *major, int32_t *minor, int32_t *sm_arch);

#ifdef __cplusplus
}
#endif

#endif /* RBSIM_H */
