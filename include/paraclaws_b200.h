/*
 * paraclaws_b200.h -- C ABI of the B200-native wave-propagation finite-volume step.
 *
 * The drop-in boundary for paraCLAWs' hot path: the Fortran host keeps read_solver_control,
 * the user equation module and the time loop of main.f90, and binds these entry points with
 * iso_c_binding (one bind(C) interface per function below).  Plain C types only; all arrays
 * are caller-owned host buffers; every call returns an int status (PCL_OK = 0, errors < 0).
 *
 * Threading: one host thread per context; each context owns one CUDA stream and its device
 * memory.  The only state shared between contexts is the static device scratch of
 * pcl_solve_dimensional_split_noalloc.
 *
 * State layout at the boundary is the reference's: vars(3, -1:m_xi+2, -1:m_eta+2) column-major
 * (domain/SMOD_domain_allocation.f90:94), (h, hu, hv) fastest.  Inside the context the state is
 * held as SoA planes in device memory; the transpose happens only in upload/download.
 */
#ifndef PARACLAWS_B200_H
#define PARACLAWS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PCL_OK 0
#define PCL_ERR_NAN (-1)        /* NaN in a flux Jacobian (examples/2D_dam_break/cartesian/SMOD_jakobian.f90:55-70) */
#define PCL_ERR_NEG_DEPTH (-2)  /* h < 0: complex eigenvalues (utility/SMOD_eigenvalue_problem.f90:72-83) */
#define PCL_ERR_TIMEOUT (-3)    /* a bounded device wait gave up */
#define PCL_ERR_OOM (-4)        /* device or pinned-host allocation failed */
#define PCL_ERR_BADARG (-5)     /* invalid settings or arguments */
#define PCL_ERR_CUDA (-6)       /* CUDA runtime error */
#define PCL_ERR_FATAL_DT (-7)   /* end_program in updateTime (time_control/MOD_time_control.f90:213-231) */
#define PCL_ERR_IO (-8)         /* control.in / custom.in unreadable, or a snapshot file unwritable */
#define PCL_ERR_FULL (-9)       /* batch: no free slot or over the memory budget */
#define PCL_ERR_USER (-10)      /* a device hook (user boundary condition, source term) failed */

/* precision forms (custom.in) */
#define PCL_PREC_FP64 0   /* bit-compatible FP64 path (the drop-in) */
#define PCL_PREC_MIXED 1  /* FP32 flux/limiter arithmetic, FP64 state, FP64 dt and sums */

/* boundary-condition codes (user_subroutines/SMOD_boundary_conditions.f90:13) */
#define PCL_BC_WALL 1          /* BC_USER slot: reflective wall in this library */
#define PCL_BC_ZERO_GRADIENT 2
#define PCL_BC_CONST_GRADIENT 3

/* Everything read_solver_control reads from control.in (utility/MOD_IO.f90:61-94), in that
   order, plus the settings this library reads from custom.in (the reference leaves custom.in
   unread: custom_settings.py:16-22). */
typedef struct pcl_solver_control {
  int num_equations, num_dimensions, num_ghost, num_aux, num_waves;
  int number_of_snapshots;
  int adaptive_timestepping;
  int higher_order_flux_correction;
  int use_limiter;
  int limiter_method;
  int m_xi, m_eta;
  int bc_xi_lower, bc_xi_upper, bc_eta_lower, bc_eta_upper;
  int precision_mode;           /* custom.in */
  int initial_condition;        /* custom.in: 0 file, 1 circular dam */
  double t_start, t_final, dt_initial, cfl_limit, dt_min, dt_max;
  double dt_max_growth_ratio, dt_min_shrink_ratio;
  double xi_min, xi_max, eta_min, eta_max;
  double grav;                  /* custom.in; the reference sets it in SMOD_setup.f90:21 */
  double dam_radius, dam_h_in, dam_h_out, dam_x0, dam_y0;  /* custom.in */
  long long max_accepted_steps; /* custom.in: 0 = run to t_final only */
} pcl_solver_control;

typedef struct pcl_ctx pcl_ctx;

/* Per-run counters of a context. */
typedef struct pcl_run_stats {
  long long attempts, accepted, rejected;
  long long launches;           /* kernels this context has launched so far */
  double time, dt, dt_previous, cfl;
  int snapshot_index, done, status, last_ierr;
} pcl_run_stats;

/* One attempted step as main.f90:265-271 reports it. */
typedef struct pcl_step_record {
  double dt, cfl, time, dt_next;
  int ierr, snapshot_index;
} pcl_step_record;

/* ---- configuration ---- */

/* Fill *out with the reference defaults (control_settings.py:21-105; grav = real(9.81)). */
void pcl_default_control(pcl_solver_control* out);

/* Parse control.in (28 list-directed records, utility/MOD_IO.f90:55-94) and, if custom_in is
   not NULL and exists, custom.in as this library defines it.  Replaces read_solver_control's
   reads. */
int pcl_read_solver_control(const char* control_in, const char* custom_in, pcl_solver_control* out);

/* ---- context lifecycle ---- */

/* Allocate the device state of one grid on `device`, build the mesh metrics
   (domain/SMOD_mesh_manipulation.f90:14-178) and initialise the time control
   (time_control/MOD_time_control.f90:70-151).  Replaces the allocations of main.f90:125-151. */
int pcl_create(const pcl_solver_control* ctl, int device, pcl_ctx** out);
int pcl_destroy(pcl_ctx* ctx);

/* Copy the state in and out (reference layout, see top).  upload_state also makes it the
   current solution of every rotation buffer. */
int pcl_upload_state(pcl_ctx* ctx, const double* vars);
int pcl_download_state(pcl_ctx* ctx, double* vars);

/* set_initial_conditions of the dam-break example on the device
   (examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:34-46): h = dam_h_in where
   sqrt(x^2 + y^2) < dam_radius at the cell centre (shifted by dam_x0, dam_y0), else dam_h_out,
   hu = hv = 0, on the whole padded block.  Needs initial_condition = 1. */
int pcl_initial_condition(pcl_ctx* ctx);

/* ---- snapshots (main.f90:178 and :256-268, writeData of utility/MOD_IO.f90:397-460) ---- */

/* The device-resident loop of pcl_advance, stopped after the accepted attempt whose time reaches
   the next snapshot time (main.f90:256-258), with that step's ghost fill done: the state is what
   the reference passes to writeData.  Returns at time_final, the accepted-step cap or an error as
   pcl_advance does; stats->snapshot_index tells which snapshot was reached. */
int pcl_advance_to_snapshot(pcl_ctx* ctx, pcl_run_stats* stats);

/* writeData for the current state: <output_dir>/<time as F20.10, left-adjusted>/rank_0/qout.dat
   with one record per cell of the padded block (j outer, i inner) holding h, hu, hv in the
   reference's format(50e26.16), and aout.dat with num_aux zeros per cell (the shallow-water
   module never sets its aux fields).  The state is transposed on the device and copied
   asynchronously into a pinned buffer; a host thread then formats and writes the files while
   the caller may go on stepping.  wait != 0 returns after the files are written; otherwise
   pcl_snapshot_wait (or the next pcl_write_snapshot, or pcl_destroy) joins the writer. */
int pcl_write_snapshot(pcl_ctx* ctx, const char* output_dir, int wait);
int pcl_snapshot_wait(pcl_ctx* ctx);

/* One value in the E26.16 field of that format, NUL-terminated (out holds 27 chars). */
int pcl_format_e26_16(double value, char* out);

/* ---- user boundary condition (code 1, BC_USER of SMOD_boundary_conditions.f90:13) ---- */

/* What a device hook (user boundary condition, source term) sees: the context's device state,
   the current-buffer index and the attempt's flags. */
typedef struct pcl_device_view {
  double* state;               /* device: rotation buffer b, plane p (shallow water: 0 h, 1 hu,
                                  2 hv) at state + b*buffer_stride + p*plane_stride */
  long long buffer_stride;     /* doubles */
  long long plane_stride;      /* doubles */
  int pitch;                   /* doubles per row: cell (i, j), i, j = -1 .. m+2, at (j+1)*pitch + (i+1) */
  int m_xi, m_eta;
  int centre_stride;           /* centre of column i at xi_centre[(i+1)*centre_stride], row j likewise */
  const double* xi_centre;     /* device */
  const double* eta_centre;    /* device */
  const int* current_buffer;   /* device int: index of the buffer holding the current solution */
  const int* attempt_accepted; /* device int: 1 when the attempt just taken was accepted */
  const double* step_dt;       /* device double: dt of that attempt */
  int num_equations;           /* planes per rotation buffer (control.in's num_equations) */
} pcl_device_view;
typedef pcl_device_view pcl_bc_view;

/* The reference leaves BC_USER unimplemented (it aborts, SMOD_boundary_conditions.f90:83-211);
   this library fills it with a reflective wall unless a hook is set.  The hook enqueues the
   caller's own device work on `stream` (a cudaStream_t) for the sides in `sides` (bit 0 xi low,
   1 xi high, 2 eta low, 3 eta high: those coded 1) and returns 0, or nonzero on failure
   (PCL_ERR_USER).  It must only enqueue: the library calls it wherever it fills ghosts, also
   while capturing the CUDA graphs of pcl_advance, where the fill of every attempt is in the
   graph and must do nothing on the device unless *attempt_accepted == 1.  force = 1 marks a
   fill that always runs (pcl_update_rank_boundaries).  The current buffer changes every
   accepted step, so device code reads *current_buffer.  Corner ghosts are never read. */
typedef int (*pcl_user_bc_fn)(const pcl_bc_view* view, int sides, int force, void* stream, void* user);
int pcl_set_user_bc(pcl_ctx* ctx, pcl_user_bc_fn fn, void* user);

/* ---- source term (integrate_source_term, solver/MOD_solve.f90:295-336) ---- */

/* The reference integrates a user source_function phi by forward Euler, q_p += phi_p * dt, on
   the interior cells after an accepted attempt and before the ghost fill (main.f90:238).  The
   dam break's phi is 0, a no-op the library skips.  A source hook enqueues the caller's own
   kernel doing that update on `stream`; `*step_dt` on the device is the attempt's dt.  The hook
   runs from pcl_integrate_source_term (force = 1) and inside the device loop's graphs after
   every attempt's time control (force = 0: do nothing on the device unless
   *attempt_accepted == 1).  Returns 0, or nonzero on failure (PCL_ERR_USER). */
typedef int (*pcl_source_fn)(const pcl_device_view* view, int force, void* stream, void* user);
int pcl_set_source_hook(pcl_ctx* ctx, pcl_source_fn fn, void* user);

/* ---- equation modules (getJakobi interface, user_subroutines/MOD_user_subroutines.f90) ---- */

/* The reference builds one equation module into the program (a USER_DIR jakobian submodule
   replaces the example's).  This library compiles its modules in and takes one per context:
     PCL_EQ_SHALLOW_WATER          the dam-break module (examples/2D_dam_break/cartesian/
                                   SMOD_jakobian.f90:44-53), specialised kernels; the default
     PCL_EQ_SHALLOW_WATER_GENERIC  the same Jacobian through the generic path
     PCL_EQ_ACOUSTICS              linear acoustics, q = (p, u, v), params (K, rho)
   The generic path runs the reference's step for the module's Jacobian: flux J(q).q in dgemv
   order, HLL with the largest |eigenvalue| of both cells (closed form per module), the limiter
   and the correction on the three components.  params: shallow water takes g (default: the
   control's grav), acoustics K and rho (both > 0).  FP64 contexts on uniform grids only. */
#define PCL_EQ_SHALLOW_WATER 0
#define PCL_EQ_SHALLOW_WATER_GENERIC 1
#define PCL_EQ_ACOUSTICS 2
int pcl_set_equation(pcl_ctx* ctx, int module, const double* params, int nparams);

/* Shape of the FP64 eta sweep, a schedule that never changes results.  PCL_SHAPE_AUTO (the
   default) and PCL_SHAPE_BAND run the bands (shared-memory phases along the columns of narrow
   column bands); PCL_SHAPE_WINDOW runs column windows (one thread per column over a strip of
   rows).  For the specialised shallow-water module the bands need g in [2^-20, 2^20]; outside
   it the windows run.  Applies to every equation module's FP64 path. */
#define PCL_SHAPE_AUTO 0
#define PCL_SHAPE_WINDOW 1
#define PCL_SHAPE_BAND 2
int pcl_set_sweep_shape(pcl_ctx* ctx, int eta_shape);
/* The shape the FP64 eta sweep runs for this context's grid (PCL_SHAPE_WINDOW or
   PCL_SHAPE_BAND), with PCL_SHAPE_AUTO resolved. */
int pcl_get_sweep_shape(pcl_ctx* ctx, int* eta_shape);

/* ---- mapped (curvilinear) grids ---- */

/* Mesh metrics of a mapped grid, as finalize_mesh leaves them in the reference
   (domain/SMOD_mesh_manipulation.f90:147-173; MOD_domain.f90:68-78): capacity(i,j),
   length_ratio_xi(1,i,j) (the xi face between cells i-1 and i) and length_ratio_eta(1,i,j) (the
   eta face between cells j-1 and j), each a column-major (m_xi+4) x (m_eta+4) array with lower
   bounds -1, i.e. the reference's own arrays.  The FP64 sweeps then read them per cell
   (solver/MOD_solve.f90:211-233, MOD_flux_correction.f90:162-181).  A Fortran host passes the
   arrays its finalize_mesh computed.  FP64 contexts only (PCL_ERR_BADARG otherwise).  The
   device dam-break initial condition (pcl_initial_condition) uses computational coordinates;
   a mapped grid's initial state is uploaded by the host. */
int pcl_set_mesh_metrics(pcl_ctx* ctx, const double* capacity, const double* length_ratio_xi,
                         const double* length_ratio_eta);

/* map_to_physical_coordinates (user_subroutines/SMOD_coordinate_mapping.f90:35-43): (xi, eta) ->
   (x, y). */
typedef void (*pcl_map_fn)(double xi, double eta, double* x, double* y, void* user);

/* The three metric arrays of pcl_set_mesh_metrics computed on the host from a coordinate mapping
   (NULL: the identity), in the reference's order: corners of initialize_computational_coordinates
   (SMOD_mesh_manipulation.f90:14-56), face length ratio NORM2(face)/delta and the shoelace area
   over delta_xi*delta_eta.  NORM2 of a face vector (a, b) is |a| when b = 0, |b| when a = 0 and
   sqrt(a*a + b*b) otherwise (the Fortran intrinsic's rounding on skewed faces is
   compiler-defined).  Outputs as in pcl_set_mesh_metrics.  Allocates nothing on the device. */
int pcl_compute_mesh_metrics(const pcl_solver_control* ctl, pcl_map_fn map, void* user, double* capacity,
                             double* length_ratio_xi, double* length_ratio_eta);

/* ---- the hot path, one call per reference routine ---- */

/* update_rank_boundaries (user_subroutines/SMOD_boundary_conditions.f90:17-56): on-device
   ghost fill of the current solution; no halo exchange (one GPU holds the whole grid). */
int pcl_update_rank_boundaries(pcl_ctx* ctx);

/* solve_dimensional_split (solver/MOD_solve.f90:23-175): one attempted step with the current
   dt: xi sweep, validity, eta sweep, validity.  *ierr = 1 accepted (the new solution is
   current) or -1 rejected (the pre-step solution stays current, as after main.f90:221).
   Updates the time control's CFL like update_max_CFL. */
int pcl_solve_dimensional_split(pcl_ctx* ctx, int* ierr);

/* solution = solution_old (main.f90:221).  A rejected attempt never overwrites the current
   buffer, so this only has to exist for call-for-call parity; it is a no-op. */
int pcl_restore_solution(pcl_ctx* ctx);

/* integrate_source_term (solver/MOD_solve.f90:295-336) with the default source phi = 0
   (user_subroutines/SMOD_source_function.f90:27): q + 0*dt, a no-op for finite q. */
int pcl_integrate_source_term(pcl_ctx* ctx);

/* ---- time control (time_control/MOD_time_control.f90), device resident ---- */
int pcl_update_time(pcl_ctx* ctx, int step_valid);   /* updateTime :153-243 */
int pcl_reset_cfl(pcl_ctx* ctx);                      /* reset_CFL :270-279 */
int pcl_advance_snapshot_index(pcl_ctx* ctx);         /* advance_snapshot_index :254-260 */
int pcl_set_dt(pcl_ctx* ctx, double dt);              /* host override of dt (tests) */
int pcl_get_time(pcl_ctx* ctx, double* time);
int pcl_get_dt(pcl_ctx* ctx, double* dt);             /* get_dt :290-297 */
int pcl_get_previous_dt(pcl_ctx* ctx, double* dt);    /* get_previous_dt :299-306 */
int pcl_get_cfl(pcl_ctx* ctx, double* cfl);           /* get_CFL :281-288 */
int pcl_get_snapshot_index(pcl_ctx* ctx, int* idx);   /* get_snapshot_index :308-315 */
int pcl_get_snapshot_time(pcl_ctx* ctx, int idx, double* t); /* snapshot_intervals(idx) */

/* ---- the whole main loop on the device ---- */

/* Run main.f90:193-283 (solve, reject/restore, ghost fill, updateTime, snapshot index,
   reset_CFL) without a host round trip per step, in CUDA graphs of `chunk` attempts, until
   time >= t_final, the accepted-step cap, an error, or max_attempts (0: no cap).  Every
   attempt is logged on the device (pcl_get_step_log).  *stats may be NULL. */
int pcl_advance(pcl_ctx* ctx, long long max_attempts, pcl_run_stats* stats);
int pcl_get_stats(pcl_ctx* ctx, pcl_run_stats* stats);
/* time_control%initialize again (MOD_time_control.f90:70-151) and clear the counters and the
   step log: with pcl_upload_state, restarts a run on the same context. */
int pcl_reset_time_control(pcl_ctx* ctx);
/* Diagnostic: run `reps` device-loop attempts with a CUDA event around every kernel and return
   the mean duration of each kernel kind in avg_ms[] (FP64: xi sweep, eta sweep, time control,
   ghost fill; mixed: fused sweep, time control, ghost fill); *nkinds = entries written.  The
   attempts advance the run: on a context that reaches its end time or accepted-step cap during
   them, the remaining kernels return at once and the means come out too short. */
int pcl_profile_kernels(pcl_ctx* ctx, int reps, double* avg_ms, int* nkinds);
/* Copy up to cap records of the device step log; *n = records logged so far. */
int pcl_get_step_log(pcl_ctx* ctx, pcl_step_record* out, long long cap, long long* n);

/* ---- batching form ----
   No counterpart in the reference (one run = one grid there).  Many independent grids of
   uneven size ("instances"), each with its own control.in settings, state and adaptive dt
   (its own time_control), advanced together by ONE persistent kernel launch per attempted step
   (captured in CUDA graphs).  Each launch runs, for every instance that is not done, exactly
   what pcl_advance runs for one attempt (sweeps, accept/reject, updateTime, snapshot index,
   ghost fill), with bit-identical results.  Instances can be added and removed between steps. */
typedef struct pcl_batch pcl_batch;

/* precision: PCL_PREC_FP64 or PCL_PREC_MIXED (every instance of a batch uses it). */
int pcl_batch_create(int device, int precision, int max_instances, pcl_batch** out);
int pcl_batch_destroy(pcl_batch* batch);
/* device bytes one instance with these settings holds (state buffers, tables, control, log) */
long long pcl_batch_instance_bytes(const pcl_solver_control* ctl);
/* Allocate a slot, upload the state (reference layout) -- or, with vars = NULL and
   initial_condition = 1, build the dam-break state on the device -- and fill its ghosts: *slot
   receives its id.  PCL_ERR_FULL when no slot is free. */
int pcl_batch_add(pcl_batch* batch, const pcl_solver_control* ctl, const double* vars, int* slot);
int pcl_batch_remove(pcl_batch* batch, int slot);
/* nsteps attempted steps of every instance not done (persistent launches, graphs of 16). */
int pcl_batch_step(pcl_batch* batch, int nsteps);
/* done[slot] (1 done, 0 running, -1 free slot) and status[slot] (PCL_* code) of every slot;
   arrays of max_instances entries. */
int pcl_batch_poll(pcl_batch* batch, int* done, int* status);
int pcl_batch_stats(pcl_batch* batch, int slot, pcl_run_stats* stats);
int pcl_batch_download(pcl_batch* batch, int slot, double* vars);
int pcl_batch_get_step_log(pcl_batch* batch, int slot, pcl_step_record* out, long long cap, long long* n);
/* Schedule of the persistent kernel (set by the autotuner): rows per mixed work item (0, the
   default: chosen from the instances each time they change), rows per FP64 xi item (default 8),
   rows per FP64 eta item (a chunk of a 4-column band, default 124: 32 rows per step, the first
   step filling a 4-row halo), CTAs per SM (0: the occupancy limit).  Results do not depend on
   it. */
int pcl_batch_set_schedule(pcl_batch* batch, int tile_rows, int x_rows, int y_rows, int blocks_per_sm);
int pcl_batch_info(pcl_batch* batch, int* n_used, int* n_done, long long* cells, long long* device_bytes);
void* pcl_batch_get_stream(pcl_batch* batch);

/* ---- precision form support ---- */

/* FP64 sums of h, hu and hv over the interior cells of the current solution (mass and
   momentum; multiply by d_xi*d_eta for the integrals).  Rows are summed on the device and the
   row partials added on the host in row order, so the result is reproducible.  No counterpart
   in the reference (it has no conservation diagnostics). */
int pcl_conservation_sums(pcl_ctx* ctx, double* sums3);

/* Rows per work item of the fused mixed-precision kernel (default 128 where that still makes
   four waves of CTAs, else 64).  No effect on results: every cell's arithmetic is independent
   of the tiling. */
int pcl_set_tile_rows(pcl_ctx* ctx, int rows);

/* ---- one step without device allocation ---- */

/* No counterpart in the reference.  One attempted FP64 step -- the xi and eta sweeps and the
   accept/reject test of pcl_solve_dimensional_split, bit-identical to it -- for callers that
   cannot allocate device memory: hosts whose device memory belongs to another allocator, step
   loops that must not pay the device-wide synchronisation of cudaMalloc/cudaFree, or jobs that
   must account for all device memory up front.  It allocates nothing: its scratch (the
   intermediate state, mesh tables and control block) is one static device array in the library,
   held by every GPU that loads the library (about 1.6 MB) until exit, which limits the grid to
   m_xi, m_eta <= 128 (larger grids return PCL_ERR_BADARG).
   - d_state_in / d_state_out: caller-owned device memory, three planes (h, hu, hv), each of
     m_eta+4 rows of ld >= m_xi+4 doubles, plane p at base + p*ld*(m_eta+4), cell (i, j) of the
     padded block (i, j = -1 .. m+2) at row j+1, column i+1.  The input's ghost cells must be
     filled (pcl_update_rank_boundaries semantics).  The output gets the new interior plus the
     input's ghost cells, and is written only when *ierr = 1.
   - dt: the step size; ctl supplies the grid, limiter, boundary codes, grav, cfl_limit and
     dt_min_shrink_ratio (precision_mode must be FP64).  *cfl receives the attempt's CFL.
     Uniform grids and the built-in shallow-water module only: mapped meshes
     (pcl_set_mesh_metrics) and other equation modules (pcl_set_equation) belong to contexts
     and do not apply here.
   - stream: a cudaStream_t or NULL; the call synchronises it before returning.  The caller's
     current device is restored on return.
   The first call on a device looks up the array's device address (once per device); make that
   first call before any stream capture.  The address belongs to the device's primary context:
   after a cudaDeviceReset of that device, do not call this entry point on it again in the same
   process.  All calls share the array and it keeps the last call's contents; calls that overlap
   on the GPU race on it. */
int pcl_solve_dimensional_split_noalloc(const pcl_solver_control* ctl, int device, void* stream,
                                        const double* d_state_in, double* d_state_out, long long ld,
                                        double dt, double* cfl, int* ierr);

/* ---- self-checks of the FP64 sweeps' arithmetic shortcuts (no counterpart in the reference) ----
   The FP64 sweeps take quotients that share a denominator from one correctly rounded reciprocal
   (Markstein's correction, two steps), and skip the limiter's division where phi saturates; both
   give the same bits as the plain IEEE operations.  These run the shortcut and the plain form side
   by side on the current device and count results that differ in any bit. */
/* a[k] / b[k] against the shared-reciprocal quotient for every pair inside the method's range
   (|a|, |b|, |a/b| in [2^-960, 2^960], or a = 0); *checked = pairs in range. */
int pcl_check_quotients(const double* a, const double* b, long long n, long long* mismatches, long long* checked);
/* the same on n pseudo-random pairs generated on the device from seed */
int pcl_check_quotients_random(long long n, unsigned long long seed, long long* mismatches, long long* checked);
/* cell flux + HLL of both sweep directions, fast against plain division, on n random cell pairs
   across the range the sweeps admit (h, |hu|, |hv| in [2^-64, 2^64), momenta also 0), with
   gravity grav; the limiter with and without the saturation shortcut on waves made from them. */
int pcl_check_flux_paths(long long n, unsigned long long seed, double grav, long long* flux_mismatches,
                         long long* fast_pairs, long long* limiter_mismatches);

/* ---- tests of the bounded-wait timeout path (no counterpart in the reference) ----
   Every inter-CTA or copy-completion wait in the library is bounded; when one gives up, the
   kernel records PCL_ERR_TIMEOUT, the attempt is void (the current solution stays as it was)
   and the context or batch stays usable.  These switches make a wait run out on purpose, with
   a short bound, so that path can be tested; both are off by default and set only from here.
   Neither faults nor hangs the GPU: the wait is for a flag that nothing sets, and it ends at
   its bound. */
/* FP64 batch: the eta items of `slot` wait for one xi item more than the step has (slot -1:
   off); spin_limit bounds every eta item's wait in polls of ~64 ns (0: the default, ~1 s).
   pcl_batch_step then returns PCL_ERR_TIMEOUT and the slot's status is PCL_ERR_TIMEOUT. */
int pcl_batch_inject_stall(pcl_batch* batch, int slot, unsigned spin_limit);
/* Mixed-precision context: the bulk copy of state row `row` (-1 .. m_eta+2) into the fused
   kernel's shared-memory ring is never issued, and its waits give up after `probes` probes
   (row -1: off, the normal build runs again). */
int pcl_inject_copy_stall(pcl_ctx* ctx, int row, unsigned probes);

/* ---- utilities ---- */
int pcl_synchronize(pcl_ctx* ctx);
void* pcl_get_stream(pcl_ctx* ctx);                   /* the context's cudaStream_t */
long long pcl_state_doubles(const pcl_ctx* ctx);      /* 3*(m_xi+4)*(m_eta+4) */
long long pcl_device_bytes(const pcl_ctx* ctx);       /* device memory held by the context */
int pcl_get_io_bytes(pcl_ctx* ctx, long long* h2d, long long* d2h); /* bytes copied so far */
int pcl_host_alloc(void** ptr, long long bytes);      /* pinned host buffer */
int pcl_host_free(void* ptr);
const char* pcl_status_string(int status);
int pcl_version(void);

#ifdef __cplusplus
}
#endif
#endif
