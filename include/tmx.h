/*
 * tmx.h -- C ABI of the B200 T-mixer solver (coupled D3Q19 lattice Boltzmann:
 * flow plus reactive species A + B -> C in two coupled boxes).
 *
 * The reference (Tmixer.cpp) has no library interface: main() calls five
 * void(void) phase functions on global arrays once per step
 * (Tmixer.cpp:10467-10475) and fixes the case with #defines
 * (Tmixer.cpp:76-149).  Each entry point below names the reference code it
 * replaces.  Plain pointers and sizes only; no CUDA or torch types.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative TMX_E* code; the text
 *     of the last error on the calling thread is returned by tmx_last_error().
 *   - Boxes: 0 = inlet channel ("I", inx x iny x nz), 1 = mixing channel
 *     ("M", mnx x mny x nz).  Host arrays are in the reference's [i][j][k]
 *     order over nodes 1..n (k fastest), i.e. shape (nx, ny, nz) row-major.
 *   - A handle owns all of its device memory and one CUDA stream; use one
 *     handle from one host thread at a time.  Different handles may run
 *     concurrently.
 */
#ifndef TMX_H
#define TMX_H

#ifdef __cplusplus
extern "C" {
#endif

#define TMX_ABI_VERSION 1

#define TMX_OK 0
#define TMX_E_INVALID (-1)  /* invalid case or argument */
#define TMX_E_NOMEM (-2)    /* device or host allocation failed */
#define TMX_E_CUDA (-3)     /* CUDA runtime error */
#define TMX_E_STATE (-4)    /* call out of order (e.g. step before init) */
#define TMX_E_NONFINITE (-5) /* non-finite value found in the state */

/* arithmetic of the state and of the step */
#define TMX_FP64 0 /* plain form: FP64 storage and arithmetic, bit-exact with the reference */
#define TMX_FP32 1 /* FP32 storage and arithmetic */
#define TMX_FP16 2 /* FP32 arithmetic; populations stored in FP16 as their non-equilibrium part, next to FP32 moments */

/* field ids of tmx_fields */
#define TMX_RHO 0
#define TMX_UX 1
#define TMX_UY 2
#define TMX_UZ 3
#define TMX_CA 4
#define TMX_CB 5
#define TMX_CC 6

/* Case parameters: the reference's compile-time constants as runtime values.
 *   inx, iny, nz        Tmixer.cpp:122-134   inlet box size
 *   mnx, mny            Tmixer.cpp:140-143   mixing box size
 *   ia                  Tmixer.cpp:1374      first inlet column over the opening;
 *                                            ib = ia + mnx - 1 (Tmixer.cpp:1375)
 *   tau                 Tmixer.cpp:84        flow relaxation time
 *   tau_a, tau_b, tau_c Tmixer.cpp:86-88     species relaxation times
 *   rho0, rho_out       Tmixer.cpp:101-103   initial and outlet density
 *   c_in[s][n]          Tmixer.cpp:90-97     species s (A,B,C) at inlet n (1,2)
 *   rateconst           Tmixer.cpp:99        A + B -> C rate constant
 *   umean               Tmixer.cpp:107       mean of the inlet-1 duct profile
 *   precision           TMX_FP64, TMX_FP32 or TMX_FP16 (no counterpart in the reference,
 *                       which is FP64 throughout)
 * Requirements: all sizes >= 3, 2 <= ia, ia + mnx - 1 <= inx - 1. */
typedef struct tmx_case {
    int inx, iny, nz;
    int mnx, mny;
    int ia;
    double tau;
    double tau_a, tau_b, tau_c;
    double rho0, rho_out;
    double c_in[3][2];
    double rateconst;
    double umean;
    int precision;
} tmx_case;

typedef struct tmx_handle tmx_handle;

/* ABI version of the loaded library (TMX_ABI_VERSION). */
int tmx_abi_version(void);

/* Text of the last error on the calling thread ("" if none). */
const char *tmx_last_error(void);

/* Fill *out with the reference's hard-coded case (Tmixer.cpp:76-149, with
 * taua = taub = taup = 0.5*((2*tau-1)/3 + 1), Tmixer.cpp:86-88). */
int tmx_case_reference(tmx_case *out);

/* Fill *out with a T-mixer of width W in the layout of the benchmark
 * configurations (no counterpart in the reference, whose sizes are fixed):
 * inlet 8W x W x W, mixing 2W x 4W x W, opening x = 3W+1..5W, tau_a = tau_b =
 * tau_c = tau_c, species A = 1 at inlet 1 and B = 1 at inlet 2, rho0 = rho_out
 * = rho, rate constant k.  The reference's duct profile is scaled by mean
 * (Umean); here umean is chosen so that the profile's maximum is u_max. */
int tmx_case_wlayout(int W, double u_max, double tau_f, double tau_c, double k, double rho, tmx_case *out);

/* Validate a case; returns TMX_E_INVALID with a message if it cannot run. */
int tmx_case_check(const tmx_case *c);

/* Device bytes tmx_create would allocate for this case. */
int tmx_case_footprint(const tmx_case *c, long long *bytes);

/* Allocate the device state of one solve on CUDA device `device`.
 * Replaces allocateMemory() (Tmixer.cpp:711-1081). */
int tmx_create(const tmx_case *c, int device, tmx_handle **out);

/* Inlet profile, initial macroscopic state and initial distributions.
 * Replaces GenerateInletVelocity() (Tmixer.cpp:1426-1539), initialization()
 * (:1544-1585), equilibrium() (:1589-1831) and
 * initialize_distribution_function() (:1835-2018). */
int tmx_init(tmx_handle *h);

/* Advance nsteps full steps.  Each step equals one pass of the reference's
 * loop body: equilibrium, collision, streaming, boundary_conditions,
 * calculate_velocity_density (Tmixer.cpp:10469-10475).  Asynchronous on the
 * handle's stream; the macroscopic fields of the last step are kept. */
int tmx_step(tmx_handle *h, int nsteps);

/* Wait for all work queued on the handle. */
int tmx_sync(tmx_handle *h);

/* Number of steps completed since tmx_init. */
long long tmx_steps_done(const tmx_handle *h);

/* The case a handle was created with. */
int tmx_case_of(const tmx_handle *h, tmx_case *out);

/* Checkpoint and restore of a solve's device state (no counterpart in the
 * reference, which only writes text output): everything the next step reads
 * (the populations held between steps, the previous step's densities, the
 * FP16 form's moment records), the macroscopic fields of the last step and
 * the inlet profiles, behind a header with the case, the form and the step
 * count.  The buffer is host memory of tmx_checkpoint_size bytes, portable
 * between handles and batch slots (tmx_batch_checkpoint / tmx_batch_restore)
 * of the same case and form.  A restored solve continues bit for bit as the
 * saved one would have; tmx_restore replaces the state of a created handle
 * (it need not be initialised) and sets its step count. */
int tmx_checkpoint_size(const tmx_handle *h, long long *bytes);
int tmx_checkpoint(tmx_handle *h, void *buf, long long bytes);
int tmx_restore(tmx_handle *h, const void *buf, long long bytes);

/* Copy one macroscopic field of one box after the last step into host memory
 * (nx*ny*nz doubles).  The arrays rho/ux/uy/uz/grho/hrho/prho (and mrho, mux,
 * ... for the mixing box) of calculate_velocity_density() (Tmixer.cpp:9352-9656),
 * as written out by write_Domain_Data() (Tmixer.cpp:10028-10064). */
int tmx_fields(tmx_handle *h, int box, int field, double *host_out);

/* Copy the populations held between steps (post-collision, i.e. the
 * reference's fn/gn/hn/pn arrays, Tmixer.cpp:9661-9860, that the next step
 * streams) of field fld (0 flow, 1 A, 2 B, 3 C) of one box:
 * 19*nx*ny*nz doubles, direction-major. */
int tmx_populations(tmx_handle *h, int box, int fld, double *host_out);

/* Mixing quality after the last step: (mny + iny) rows of
 * {row, mean cA, mean cB, mean cC, I_A, I_B, I_C}, mixing rows 1..mny then
 * inlet rows 1..iny over the opening; outlet_im[3] = I_A, I_B, I_C of mixing
 * row 1 (may be NULL).  The numbers write_MixingQuality() prints
 * (Tmixer.cpp:10161-10409), with its running maxima starting at 0. */
int tmx_mixing(tmx_handle *h, double *rows_out, double *outlet_im);

/* tmx_mixing without any allocation, host or device, in the call: the same
 * rows, bit for bit, from a fixed 512 KiB scratch array in the library's
 * static device memory, finished on the device and copied straight into
 * rows_out.  No counterpart in the reference.  For callers that must not
 * allocate while they poll the mixing quality, such as a monitor thread
 * that may not take the heap lock or a host that accounts for every byte of
 * device memory itself.  The call launches on the handle's stream, so such
 * a monitor thread still uses the handle under the one-thread-at-a-time rule
 * above: it must take turns with the thread that steps the handle.
 *   - At most 4096 rows (mny + iny <= 4096); larger cases get TMX_E_INVALID
 *     (use tmx_mixing).
 *   - The first call on each device resolves the scratch address there
 *     (cudaGetSymbolAddress); make it before capturing any stream on that
 *     device.  That lookup runs once per device and process: if it fails,
 *     every later call on that device returns the same error until the
 *     process exits.
 *   - The scratch is shared by every handle of the process on that device:
 *     calls that overlap in time on one device race and must be serialised
 *     by the caller. */
int tmx_mixing_static(tmx_handle *h, double *rows_out, double *outlet_im);

/* Pressure and specific power after the last step: the numbers
 * write_Pressure_Power() prints (Tmixer.cpp:9866-10027), in lattice units,
 * computed in FP64 on the device in the reference's summation order.
 *   pressure_rows[(mny+iny)*3]  {row, p, p - p_top}: p = mean density / 3 over
 *       mixing row 1..mny, then inlet row 1..iny over x = ia..ib (row number
 *       j + mny); p_top = the same over inlet row iny
 *   pressure_x[inx*2]           {i, p}: mean density / 3 over the inlet box's
 *       cross-section at x = i
 *   power_rows[(mny-2)*5]       {j, cross-section rate, total rate, the same
 *       two summed over every x}: 2 vis <deformation rate> over mixing row
 *       j = 2..mny-1 (vis = (2 tau - 1)/6).  The first two reproduce the
 *       reference, whose x loop assigns instead of adding (only x = mnx-1
 *       enters its sums); the last two add every x.
 *   units[2]                    the reference's factors P0 and Pw0 (its
 *       Tmixer.cpp:189-196 with length = inx) that turn p and the rates into
 *       pascal and W/kg as it prints them. */
int tmx_pressure_power(tmx_handle *h, double *pressure_rows, double *pressure_x, double *power_rows,
                       double units[2]);

/* The reference's Tecplot text files, written from the state after the last
 * step with the reference's own line formats (byte-identical to the
 * reference's files for the FP64 form):
 *   TMX_FILE_DOMAIN    Domain_Data: every node of both boxes
 *                      (write_Domain_Data, Tmixer.cpp:10028-10064)
 *   TMX_FILE_PVC       Data_P_V_C: the mid-depth plane and five cross-sections
 *                      (write_Data_P_V_C, :10065-10160); the sections at fixed
 *                      rows 600, mny-1 and 775-mny are left out where the row
 *                      is outside its box (the reference reads outside its
 *                      arrays there)
 *   TMX_FILE_PRESSURE  Pressure (write_Pressure_Power, :9866-10027)
 *   TMX_FILE_MIXING    MixingQuality (write_MixingQuality, :10161-10409)
 * The reference names them Domain_Data_<itr>.dat etc.; path is the caller's. */
#define TMX_FILE_DOMAIN 0
#define TMX_FILE_PVC 1
#define TMX_FILE_PRESSURE 2
#define TMX_FILE_MIXING 3
int tmx_write_file(tmx_handle *h, int kind, const char *path);

/* FP64 totals over both boxes after the last step: out[0] = sum rho,
 * out[1..3] = sum cA, cB, cC, out[4] = sum (cA + cB + cC), out[5] = outlet
 * flux sum(rho*uy) over mixing row 1, out[6] = number of non-finite values in
 * the fields, out[7] = fluid nodes.  No counterpart in the reference. */
int tmx_sums(tmx_handle *h, double out[8]);

/* The inlet profiles Uin1, Uin2 as the reference keeps them
 * ((iny+3) x (nz+3) doubles each, Tmixer.cpp:703-704). */
int tmx_inlet_profile(tmx_handle *h, double *uin1, double *uin2);

/* Run nsteps steps with CUDA events around every kernel launch on the
 * handle's stream and return the summed device times (ms) of the bulk
 * (interior) kernel, of the boundary kernels and of the whole step loop.
 * The interior kernel runs after the boundary kernels here in every form
 * (tmx_step overlaps them in the FP32 and FP16 forms), so that each time is
 * that of its kernels alone.  Benchmark support; no counterpart in the
 * reference. */
int tmx_step_timed(tmx_handle *h, int nsteps, double *ms_bulk, double *ms_boundary, double *ms_total);

/* Run nsteps steps exactly as tmx_step does, between two CUDA events recorded
 * on the handle's stream, wait for them, and return the elapsed device time
 * (ms).  Benchmark support; no counterpart in the reference. */
int tmx_time_steps(tmx_handle *h, int nsteps, double *ms);

/* The memory-traffic ceiling of the interior kernels' access pattern on
 * device `device`: kernels that move exactly the bytes of a lattice update of
 * form `precision` (the 19 direction planes read at the upstream neighbours
 * and written at the node: FP64 1216 B, FP32 608 B, FP16 304 B plus the
 * 32-byte moment record read and written = 368 B), in the forms' layouts,
 * with no arithmetic, over an x-fastest box of at least `nodes` nodes (at
 * least 3 x 32768, at most 2^30), ping-ponging two buffers as the step does.
 * Tries 1, 2, 4 and 8 blocks of 256 threads per SM, `reps` timed launches
 * each after 3 untimed ones, and returns the best rate in *gbs (GB/s of
 * those bytes) and its blocks per SM.  Allocates and frees its own buffers.
 * Benchmark support (the denominator beside the plain copy bandwidth); no
 * counterpart in the reference. */
int tmx_pattern_ceiling(int precision, long long nodes, int reps, int device, double *gbs, int *blocks_per_sm);

/* Launch shape of the interior (bulk) kernel; no counterpart in the
 * reference.  kind TMX_SHAPE_FLAT: one thread per node over the flat node
 * range (every form; zchunk ignored).  The sweep shapes (FP16 form only):
 * blocks of 32 x TY threads own tiles of as many nodes of one box and walk
 * them through zchunk planes (zchunk >= 1), the writers' moment records
 * staged in shared memory: TMX_SHAPE_SWEEP8 (TY 8), TMX_SHAPE_SWEEP4 (TY 4).
 * Every shape gives the same results bit for bit.  Default: TMX_SHAPE_SWEEP4
 * with zchunk 8 for the FP16 form (set by tmx_create), TMX_SHAPE_FLAT for the
 * others. */
#define TMX_SHAPE_FLAT 0
#define TMX_SHAPE_SWEEP8 1
#define TMX_SHAPE_SWEEP4 2
int tmx_set_shape(tmx_handle *h, int kind, int zchunk);

/* Node counts: out[0] fluid nodes (both boxes), out[1] interior nodes,
 * out[2] boundary nodes, out[3] device bytes allocated. */
int tmx_counts(const tmx_handle *h, long long out[4]);

/* Free the handle and its device memory.  Replaces deallocateMemory()
 * (Tmixer.cpp:1083-1366). */
void tmx_destroy(tmx_handle *h);

/* ------------------------------------------------------------------------
 * Batched engine: many mixers of uneven size and parameters stepped together,
 * each step one launch per kernel kind over all of them (a persistent bulk
 * kernel over a concatenated cell-block list, and persistent boundary kernels
 * over the concatenated boundary-node lists), with the step captured as a
 * CUDA graph.  The reference runs one case per process and has no
 * counterpart for any of these functions.  One batch is used from one host
 * thread at a time.
 * ------------------------------------------------------------------------ */
typedef struct tmx_batch tmx_batch;

/* Device bytes one mixer of this case takes in a batch. */
int tmx_batch_footprint(const tmx_case *c, long long *bytes);

/* Create a batch of the given precision (every case added must have it)
 * whose mixers share one device arena of budget_bytes, allocated here. */
int tmx_batch_create(int precision, long long budget_bytes, int device, tmx_batch **out);

/* Admit one mixer: carve its state from the arena (TMX_E_NOMEM if no free
 * range of its footprint is left), compute its inlet profiles and initial
 * state (as tmx_init does), and return its slot number.  It joins the next
 * step of the batch. */
int tmx_batch_add(tmx_batch *b, const tmx_case *c, int *slot);

/* Retire a mixer and return its range to the arena; the slot number may be
 * reused by a later tmx_batch_add. */
int tmx_batch_remove(tmx_batch *b, int slot);

/* Checkpoint one mixer of the batch (format and size as tmx_checkpoint), and
 * admit a mixer from a checkpoint of case c (taken from a handle or a batch
 * slot): it continues bit for bit as the saved one would have, from the saved
 * step count. */
int tmx_batch_checkpoint_size(const tmx_batch *b, int slot, long long *bytes);
int tmx_batch_checkpoint(tmx_batch *b, int slot, void *buf, long long bytes);
int tmx_batch_restore(tmx_batch *b, const tmx_case *c, const void *buf, long long bytes, int *slot);

/* Advance every mixer of the batch by nsteps steps (asynchronous).  With
 * write_macro_last the last step also writes the macroscopic fields that
 * tmx_batch_fields and tmx_batch_outlet_im read. */
int tmx_batch_step(tmx_batch *b, int nsteps, int write_macro_last);

/* Wait for the batch's queued work. */
int tmx_batch_sync(tmx_batch *b);

/* Slot numbers in use (at most cap written to slots; *n = how many there are). */
int tmx_batch_slots(const tmx_batch *b, int *slots, int cap, int *n);

/* Steps taken by the mixer in a slot since it was admitted (-1 if unused). */
long long tmx_batch_slot_steps(const tmx_batch *b, int slot);

/* Outlet mixing quality of n mixers: I_A, I_B, I_C of mixing row 1, as the
 * first row of tmx_mixing, into im_out[3*e .. 3*e+2] for slots[e].  Reads the
 * macroscopic fields of the last step that wrote them; waits for the result. */
int tmx_batch_outlet_im(tmx_batch *b, const int *slots, int n, double *im_out);

/* Health of n mixers: bad[e] = 1 if mixer slots[e] has a non-finite density,
 * velocity or concentration in the macroscopic fields of the last step that
 * wrote them (checked on the device over all its nodes), else 0. */
int tmx_batch_health(tmx_batch *b, const int *slots, int n, int *bad);

/* One macroscopic field of one box of one mixer, as tmx_fields. */
int tmx_batch_fields(tmx_batch *b, int slot, int box, int field, double *host_out);

/* out[0] mixers, out[1] their fluid nodes, out[2] arena bytes, out[3] free
 * arena bytes, out[4] bulk threads per block, out[5] nodes per cell block,
 * out[6] batch steps taken, out[7] bytes of the batch's work lists. */
int tmx_batch_info(const tmx_batch *b, long long out[8]);

/* Set the bulk kernel's launch shape: threads per block (128, 256 or 512) and
 * nodes per cell block (a multiple of it). */
int tmx_batch_set_shape(tmx_batch *b, int threads, int cells);

/* Autotune the launch shape on the batch's current mixers: time
 * steps_per_trial steps of every shape of the interior kernel (the flat
 * kernel's (threads, cells) choices; for the FP16 form also every sweep
 * shape with 4, 8, 16 or 32 planes per tile, i.e. nodes per thread), keep
 * the fastest, then with it the boundary kernels' grid (1, 2 or 4 blocks per
 * SM or as many as fit) and order (beside the interior kernel or before it,
 * tmx_batch_set_boundary), keep the fastest, then
 * start every mixer again from its initial state.  Returns the threads per
 * block, the nodes per cell block (flat) or per tile (sweep), and the time
 * per step (ms); tmx_batch_shape and tmx_batch_boundary tell what won. */
int tmx_batch_tune(tmx_batch *b, int steps_per_trial, int *threads_out, int *cells_out, double *ms_out);

/* Use one of the FP16 form's sweep kernels for the interior: kind a
 * TMX_SHAPE_SWEEP* shape, zchunk planes per tile (see tmx_set_shape).
 * tmx_batch_set_shape switches back to the flat kernel.  No counterpart in
 * the reference. */
int tmx_batch_set_sweep(tmx_batch *b, int kind, int zchunk);

/* The boundary (face and edge) kernels' persistent grid: blocks_per_sm
 * blocks of 128 threads per SM, at most as many as fit; 0 (the default): as
 * many as fit.  after = 1 runs the interior kernel after them, 0 (the
 * default) beside them; the FP64 form always runs it after them.
 * tmx_batch_boundary returns the face kernel's blocks per SM in use and the
 * order (after may be NULL).  No counterpart in the reference. */
int tmx_batch_set_boundary(tmx_batch *b, int blocks_per_sm, int after);
int tmx_batch_boundary(const tmx_batch *b, int *blocks_per_sm, int *after);

/* The interior kernel's shape: out[0] TMX_SHAPE_*,
 * out[1] threads per block, out[2] nodes per cell block of the flat kernel,
 * out[3] planes per sweep tile. */
int tmx_batch_shape(const tmx_batch *b, int out[4]);

/* Run nsteps steps between two CUDA events on the batch's stream and return
 * the elapsed device time (ms). */

/* Run nsteps steps (without the captured graphs) with CUDA events around the
 * interior kernel and around the boundary kernels, the interior kernel after
 * the boundary kernels in every form so that each time is that of its
 * kernels alone, and return the summed device times (ms) and that of the
 * whole loop.  Benchmark support; no counterpart in the reference. */
int tmx_batch_step_timed(tmx_batch *b, int nsteps, double *ms_interior, double *ms_boundary, double *ms_total);
int tmx_batch_time_steps(tmx_batch *b, int nsteps, double *ms);

/* Free the batch, its arena and its mixers. */
void tmx_batch_destroy(tmx_batch *b);

/* ------------------------------------------------------------------------
 * Served form: a request loop over a batch (continuous batching).  Requests
 * arrive over time; each is admitted as soon as it has arrived, every
 * earlier request has been admitted and its footprint fits in the batch's
 * free arena; admitted mixers step together; every check_every steps the
 * outlet mixing index of each is read and a mixer is retired once, over its
 * last window steps, every species' index was non-zero (the species have
 * reached the outlet) and moved by less than tol, or after max_steps; a
 * retired mixer's range is back-filled by the next request.  No
 * counterpart in the reference.
 * ------------------------------------------------------------------------ */
typedef struct tmx_request {
    tmx_case c;
    double arrival; /* seconds after the start of the loop */
    int max_steps;  /* retire after this many steps at most */
    int window;     /* convergence window (steps), a multiple of check_every */
    double tol;     /* convergence tolerance of the outlet mixing index */
} tmx_request;

typedef struct tmx_served {
    int status;         /* 0 converged, 1 stopped at max_steps, TMX_E_NOMEM larger than the whole budget,
                           TMX_E_NONFINITE retired because its state became non-finite */
    int slot;           /* batch slot it ran in */
    long long steps;    /* steps taken */
    double admitted;    /* seconds after the start */
    double finished;    /* seconds after the start (time to solution = finished - arrival) */
    double outlet_im[3]; /* outlet I_A, I_B, I_C when retired */
} tmx_served;

typedef struct tmx_serve_opts {
    int check_every; /* steps between convergence checks */
    int max_active;  /* at most this many mixers at once (0: no limit but the budget) */
} tmx_serve_opts;

/* summary[0] makespan (s, from the start to the last retirement), [1] lattice
 * updates (fluid nodes x steps, all requests), [2] aggregate MLUPS, [3] p50
 * and [4] p99 time to solution (s), [5] most mixers at once, [6] time-weighted
 * mean mixers at once, [7] convergence checks made. */
int tmx_serve(tmx_batch *b, const tmx_request *reqs, int n, const tmx_serve_opts *opts, tmx_served *out,
              double summary[8]);

/* The same loop over an engine given as callbacks (for testing the scheduler
 * without a GPU, or driving another engine).  Each callback returns 0 or a
 * TMX_E_* code; add returns TMX_E_NOMEM when the mixer does not fit now. */
typedef struct tmx_serve_ops {
    void *ctx;
    int (*footprint)(void *ctx, const tmx_case *c, long long *bytes);
    long long (*capacity)(void *ctx);
    int (*add)(void *ctx, const tmx_case *c, int *slot);
    int (*remove)(void *ctx, int slot);
    int (*step)(void *ctx, int nsteps);
    int (*outlet_im)(void *ctx, const int *slots, int n, double *im);
    double (*now)(void *ctx);
    void (*wait_until)(void *ctx, double t);
    /* optional (may be NULL): bad[e] = 1 for a mixer whose state is no longer
     * finite; such a mixer is retired at once with status TMX_E_NONFINITE */
    int (*health)(void *ctx, const int *slots, int n, int *bad);
} tmx_serve_ops;

int tmx_serve_with(const tmx_serve_ops *ops, const tmx_request *reqs, int n, const tmx_serve_opts *opts,
                   tmx_served *out, double summary[8]);

#ifdef __cplusplus
}
#endif
#endif /* TMX_H */
