/*
 * fdtd_b200.h -- C ABI of libfdtd_b200.so, the B200 engine for the FDTD hot path
 * of QJohn2017/3D_FDTD.
 *
 * Drop-in: the library exports the reference's own FDTD (timefield3d.h) and taper
 * adjoint (adjoint3d.h) entry points with the same names, by-value struct
 * arguments and meaning, so a program written against the reference links
 * against this library instead of timefield3d.o and adjoint3d.o and keeps the
 * reference's complex.o, matrix.o and mode.o.  The struct layouts below are
 * identical to the reference's (timefield3d.h:15-27, mode.h:13-22,
 * matrix.h:11-16, complex.h:11-15, adjoint3d.h:37-58).  If a translation unit
 * also includes the reference's headers, include those first: the type blocks
 * here are skipped when the reference's include guards are already defined.
 *
 * What changes behind the same calls:
 *   - field state lives on the GPU; psi.fields is a host mirror refreshed by
 *     timefield3d_get_fields, timefield3d_get_edge_fields and
 *     timefield3d_sync_host;
 *   - materials stay host-authoritative: the timefield3d_set_* rasterisers write
 *     psi.ep/mu/sig on the host exactly as the reference does, and the next
 *     device operation uploads them;
 *   - calls queue GPU work on the grid's own stream and return; only calls
 *     that return data to the host wait for it;
 *   - errors never abort: every entry point records a status, read with
 *     fdtd_last_error().  There is no CPU fallback: without a usable GPU the
 *     device entry points fail with FDTD_ERR_NO_DEVICE and print why.
 *
 * Extensions (no reference counterpart) are grouped at the end: precision
 * (the reference's FP64 or FP32 fields), CPML boundary, point sources, probes,
 * multi-wavelength overlap monitors, a scheduled mode source and a captured
 * multi-step run.
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference-compatible types (layouts identical to the reference) ---- */
#ifndef _complex_h
struct complex_ { double re, im; };                       /* complex.h:11-15 */
typedef struct complex_ complex;
#endif
#ifndef _matrix_h
struct matrix_ { int i, j; complex *m; };                 /* matrix.h:11-16 */
typedef struct matrix_ matrix;
#endif
#ifndef _mode_h
struct mode_ { int i, j; double disc; matrix pml; matrix ep; matrix mu; matrix fields; }; /* mode.h:13-22 */
typedef struct mode_ mode;
#endif
#ifndef _timefield3d_h
struct timefield3d_ {                                     /* timefield3d.h:15-27 */
    int i, j, k;
    double disc;
    float *ep;
    float *mu;
    float *sig;
    double *fields;
    double *old_fields;
    complex *fourier_fields;
    float *sources;
};
typedef struct timefield3d_ timefield3d;
#endif
#ifndef _adjoint3d_h
struct adjoint3d_taper_ {                                 /* adjoint3d.h:37-58 */
    double ep;
    double mu;
    int seg_num;
    int start;
    int end;
    int bottom;
    int top;
    int duration;
    int *left;
    int *right;
    double *forward_fields;
    double *adjoint_fields;
    double *ep_gradient;
    double *left_grad;
    double *right_grad;
};
typedef struct adjoint3d_taper_ adjoint3d_taper;
#endif

/* =========================================================================
 * Reference entry points (timefield3d.h).  Each replaces the reference
 * function of the same name; the cited line is its declaration.
 * ========================================================================= */

/* timefield3d.h:30 -- allocates host mirrors; the device grid is created on first use */
timefield3d timefield3d_new(int i, int j, int k, double disc);
/* timefield3d.h:31 */
void timefield3d_free(timefield3d psi);
/* timefield3d.h:32 -- copies materials and current fields into a new grid */
timefield3d timefield3d_copy(timefield3d psi);
/* timefield3d.h:33 -- zeroes fields, boundary memory, sources, running DFTs, monitors */
void timefield3d_zero_fields(timefield3d psi);
/* timefield3d.h:34 -- waits for the grid, returns a malloc'd AoS double copy */
double *timefield3d_get_fields(timefield3d psi);
/* timefield3d.h:35 -- same, only the 2-cell shell filled (other entries unspecified) */
double *timefield3d_get_edge_fields(timefield3d psi);
/* timefield3d.h:36 -- snapshot of the 2-cell shell used by the Mur boundary */
void timefield3d_update_old_edge_fields(timefield3d psi);

/* timefield3d.h:39-53 -- gnuplot plots in the reference.  No graphics here: each
 * call writes the slice as raw float64 (header: int n1, int n2) to
 * $FDTD_PLOT_DIR/<name>_<index>.bin when FDTD_PLOT_DIR is set, else does nothing. */
void timefield3d_plot_Ex_x_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ex_y_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ex_z_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ey_x_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ey_y_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ey_z_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ez_x_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ez_y_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ez_z_slice(timefield3d psi, int slice_index);
void timefield3d_plot_Ex_x_slice_fourier(timefield3d psi, int slice_index);
void timefield3d_plot_Ex_y_slice_fourier(timefield3d psi, int slice_index);
void timefield3d_plot_Ex_z_slice_fourier(timefield3d psi, int slice_index);
void timefield3d_plot_permittivity_x_slice(timefield3d psi, int slice_index);
void timefield3d_plot_permittivity_y_slice(timefield3d psi, int slice_index);
void timefield3d_plot_permittivity_z_slice(timefield3d psi, int slice_index);

/* timefield3d.h:56-70 -- material rasterisers; host arrays, uploaded on next device use */
void timefield3d_set_background(timefield3d psi, float ep, float mu);
void timefield3d_set_top_half_plane(timefield3d psi, float ep, float mu, int bottom);
void timefield3d_set_background_permittivity(timefield3d psi, float ep);
void timefield3d_set_background_permeability(timefield3d psi, float mu);
void timefield3d_set_background_electric_conductivity(timefield3d psi, float sig);
void timefield3d_set_background_magnetic_conductivity(timefield3d psi, float sig);
void timefield3d_set_background_complex_permittivity(timefield3d psi, double omega, float real_ep, float imag_ep);
void timefield3d_set_prism_permittivity(timefield3d psi, float ep, int start_x, int end_x, int start_y, int end_y, int start_z, int end_z);
void timefield3d_set_prism_electric_conductivity(timefield3d psi, float sig, int start_x, int end_x, int start_y, int end_y, int start_z, int end_z);
void timefield3d_set_prism_complex_permittivity(timefield3d psi, double omega, float real_ep, float imag_ep, int start_x, int end_x, int start_y, int end_y, int start_z, int end_z);
void timefield3d_set_waveguide(timefield3d psi, float ep, int start_x, int end_x, int start_z, int end_z, int bottom, int top);
void timefield3d_set_taper(timefield3d psi, double ep, double mu, int start_left, int start_right, int end_left, int end_right, int start_z, int end_z, int bottom, int top);

/* timefield3d.h:73-76 -- explicit (non-semi-implicit) interior updates, whole grid */
void timefield3d_apply_H_timestep(timefield3d psi, double delta_t);
void timefield3d_apply_E_timestep(timefield3d psi, double delta_t);
/* timefield3d.h:75-76 -- semi-implicit interior update of z in [start+1, stop-1) */
void timefield3d_apply_H_timestep_zsection(timefield3d psi, double delta_t, int start_index, int stop_index);
void timefield3d_apply_E_timestep_zsection(timefield3d psi, double delta_t, int start_index, int stop_index);
/* timefield3d.h:77-80 -- Mur boundary; old_field is an AoS shell copy from
 * timefield3d_get_edge_fields (host).  The zsection forms use psi.old_fields,
 * i.e. the snapshot taken by timefield3d_update_old_edge_fields. */
void timefield3d_apply_H_first_order_abc(timefield3d psi, double *old_field, double delta_t);
void timefield3d_apply_E_first_order_abc(timefield3d psi, double *old_field, double delta_t);
void timefield3d_apply_H_first_order_abc_zsection(timefield3d psi, double delta_t, int start_index, int stop_index);
void timefield3d_apply_E_first_order_abc_zsection(timefield3d psi, double delta_t, int start_index, int stop_index);
/* timefield3d.h:81 -- explicit-update step: shell copy, E, E-ABC, H, H-ABC */
void timefield3d_apply_timestep(timefield3d psi, double delta_t);
/* timefield3d.h:82-83 -- the semi-implicit step the reference driver uses
 * (timefield3d.c:2787-2849).  With the CPML extension enabled the Mur passes
 * are replaced by the CPML terms inside the update. */
void timefield3d_apply_timestep_omp(timefield3d psi, double delta_t);
void timefield3d_apply_timestep_omp_full(timefield3d psi, double delta_t);
/* timefield3d.h:84-89 -- running single-frequency DFT, on device (complex double) */
void timefield3d_update_fourier_fields(timefield3d psi, double phase);
void timefield3d_update_fourier_fields_y_slice(timefield3d psi, double phase, int slice_index);
void timefield3d_update_fourier_fields_zsection(timefield3d psi, double phase, int start_index, int stop_index);
void timefield3d_update_fourier_fields_y_slice_zsection(timefield3d psi, double phase, int slice_index, int start_index, int stop_index);
void timefield3d_update_fourier_fields_omp(timefield3d psi, double phase);
void timefield3d_update_fourier_fields_y_slice_omp(timefield3d psi, double phase, int slice_index);

/* timefield3d.h:95-96 -- mode plane sources.  The mode is power-normalised in
 * place on first use (as the reference does on every call) and kept on the
 * device; see timefield3d_release_mode. */
void timefield3d_mode_source(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode, double phase, double amplitude, int reverse);
void timefield3d_mode_source_adjoint(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode, double phase, int reverse);
/* timefield3d.h:97-98 -- Gaussian-beam sources: not provided (FDTD_ERR_UNSUPPORTED) */
void timefield3d_TE_gaussian_source(timefield3d psi, int center_x, int center_y, int center_z, double width, double omega, double phase, double amplitude);
void timefield3d_TM_gaussian_source(timefield3d psi, int center_x, int center_y, int center_z, double width, double omega, double phase, double amplitude);
/* timefield3d.h:101 -- instantaneous mode overlap on plane z; adds e^{i phase} x
 * overlap to *cumulative_overlap.  Waits for the grid (it returns a value). */
complex timefield3d_mode_overlap(timefield3d psi, int center_x, int center_y, int center_z, mode overlap_mode, double phase, int reverse, complex *cumulative_overlap);
/* timefield3d.h:104 -- binarised permittivity slice writer (host) */
void timefield3d_file_write_permittivity_y_slice(timefield3d psi, char *filename, int left, int right, int start, int end, int y_slice, double ep_min, double ep_max);

/* =========================================================================
 * Reference entry points (adjoint3d.h, taper part).  Edge-field storage lives
 * on the device (E components only, the precision of the grid); the host
 * arrays forward_fields/adjoint_fields are filled only by
 * adjoint3d_taper_sync_host.
 * ========================================================================= */
/* adjoint3d.h:60 */
adjoint3d_taper adjoint3d_taper_new(double ep, double mu, int seg_num, int start, int end, int *left, int *right, int bottom, int top, int duration);
/* adjoint3d.h:61 (host raster, adjoint3d.c:243-257) */
void adjoint3d_taper_insert(timefield3d psi, adjoint3d_taper taper);
/* adjoint3d.h:62-63 -- gather E on the rasterised edge pixels at time index timestep */
void adjoint3d_taper_store_forward_fields(adjoint3d_taper taper, timefield3d main_fields, int timestep);
void adjoint3d_taper_store_adjoint_fields(adjoint3d_taper taper, timefield3d main_fields, int timestep);
/* adjoint3d.h:64 -- sum_t sum_{m<3} E_fwd E_adj on the device in FP64; fills taper.ep_gradient */
void adjoint3d_taper_calculate_ep_gradient(adjoint3d_taper taper);
/* adjoint3d.h:65 -- hat-weighted vertex gradients (host, from taper.ep_gradient) */
void adjoint3d_taper_calculate_gradients_from_ep_gradient(adjoint3d_taper taper, double ep_diff);
/* adjoint3d.h:68-69 -- integer-pixel edge updates (host) */
int adjoint3d_taper_update_symmetric(adjoint3d_taper taper, double improvement_goal, double disc, int min_width);
int adjoint3d_taper_update_asymmetric(adjoint3d_taper taper, double improvement_goal, double disc, int min_width);
/* adjoint3d.c:42 defines the reference's release function as adjointd3d_free (its
 * header says adjoint3d_free); this library releases tapers with: */
void adjoint3d_taper_free(adjoint3d_taper taper);

/* =========================================================================
 * Extensions (no reference counterpart)
 * ========================================================================= */
enum fdtd_status {
    FDTD_OK = 0,
    FDTD_ERR_NO_DEVICE = 1,     /* no CUDA device or driver */
    FDTD_ERR_CUDA = 2,          /* a CUDA call failed */
    FDTD_ERR_ARG = 3,           /* invalid argument or unknown grid */
    FDTD_ERR_ALLOC = 4,         /* host or device allocation failed */
    FDTD_ERR_UNSUPPORTED = 5,   /* entry point or combination not provided */
    FDTD_ERR_TIMEOUT = 6,       /* a bounded device wait gave up */
    FDTD_ERR_NONFINITE = 7      /* NaN/Inf found in materials */
};
enum fdtd_precision { FDTD_F64 = 0, FDTD_F32 = 1 };
/* FP32 grids with mu = 1, no magnetic loss and a CPML or PEC boundary run one of
 * five kernel designs: flat (one thread per cell, separate E and H launches),
 * flat4 (separate E and H launches, four x cells per thread with 16-byte
 * accesses; nx % 4 == 0), fused (one launch per step streaming z-planes through
 * shared memory) or wave (flat4's cell updates, but timefield3d_run executes
 * whole chunks of steps -- monitors and scheduled source included -- in one
 * persistent launch ordered as a wavefront in z, so a sweep's planes stay in
 * L2; runs with probes or bound taper stores, and single steps, use flat4).
 * stream (one launch per step: each thread block streams a band of rows
 * through its planes, E and H of a plane in one pass, reading each array once
 * and writing the other field set; nx % 4 == 0, fewer than 2^31 cells).  AUTO picks stream where the
 * grid allows it, else flat4 where nx allows, else flat.  wave's fields are
 * bit-identical to flat4's; stream's agree with flat4's to float rounding. */
enum fdtd_yee_variant {
    FDTD_YEE_AUTO = 0, FDTD_YEE_FLAT = 1, FDTD_YEE_FUSED = 2, FDTD_YEE_FLAT4 = 3, FDTD_YEE_WAVE = 4,
    FDTD_YEE_STREAM = 5
};
enum fdtd_boundary { FDTD_BOUNDARY_MUR = 0, FDTD_BOUNDARY_CPML = 1, FDTD_BOUNDARY_PEC = 2 };

/* status of the last failing call on this thread (sticky until cleared) */
int fdtd_last_error(void);
const char *fdtd_last_error_message(void);
const char *fdtd_error_string(int code);
void fdtd_clear_error(void);
int fdtd_device_count(void);
const char *fdtd_version(void);

/* Grid configuration.  Precision FDTD_F64 (default) reproduces the reference's
 * double fields; FDTD_F32 keeps fields and update coefficients in float.
 * Changing precision or boundary keeps the current fields. */
int timefield3d_set_precision(timefield3d psi, int precision);
int timefield3d_set_boundary(timefield3d psi, int boundary);
/* kernel design of the FP32 fast path (enum fdtd_yee_variant); results agree to FP32 rounding */
int timefield3d_set_yee_variant(timefield3d psi, int variant);
/* FDTD_YEE_WAVE: steps per persistent launch (default 64), steps per sweep
 * (default 16; a sweep keeps about 4 x steps_per_sweep planes live) and blocks
 * of work per ticket (default 2; a ticket's synchronisation is paid once per
 * group).  No reference counterpart.  steps_per_launch in [1, 4096],
 * steps_per_sweep in [1, steps_per_launch], blocks_per_ticket in [1, 64];
 * anything else is FDTD_ERR_ARG. */
int timefield3d_set_wave_steps(timefield3d psi, int steps_per_launch, int steps_per_sweep, int blocks_per_ticket);
/* The work-item table of one FDTD_YEE_WAVE launch (host computation, no device
 * work), for inspection and tests.  No reference counterpart.  Grid nx x ny x nz
 * (nx % 4 == 0), CPML thickness (0: none), monitors on planes job_z[0..njobs),
 * nparts overlap partials per monitor.  Writes 9 ints per item into out
 * (capacity cap items; out may be null to count): first ticket, descriptor
 * (kind 0 E / 1 H / 2 overlaps | plane << 2 | step << 17), blocks of work,
 * then three (counter, required count) pairs, counter -1 for none.  Returns the item count
 * and the ticket total, or -1 on invalid input. */
int fdtd_wave_schedule(int nx, int ny, int nz, int cpml_cells, int steps, int sweep, int blocks_per_ticket,
                       const int *job_z, int njobs, int nparts, int *out, int cap, int *tickets);
/* The tile plan of the FDTD_YEE_STREAM kernel (host computation, no device
 * work), for inspection and tests.  No reference counterpart.  Grid
 * nx x ny x nz, CPML thickness (0: none), lossy != 0 when the E update has
 * loss coefficients, nsm streaming multiprocessors.  Writes 4 ints per tile
 * into tiles (capacity cap tiles; null to count): first owned row, owned rows,
 * first owned plane, one past the last owned plane; and the block's row
 * capacity, threads and dynamic shared memory.  Returns the tile count, or -1
 * when the grid cannot use the kernel or on invalid input. */
int fdtd_stream_plan(int nx, int ny, int nz, int cpml_cells, int lossy, int nsm, int *tiles, int cap, int *ty,
                     int *threads, long long *smem_bytes);
/* CPML of `thickness` cells on every face, polynomial grading `order`;
 * sigma_max <= 0 selects 0.8 (order+1)/disc; kappa_max >= 1; alpha_max >= 0.
 * Profiles depend on delta_t and are rebuilt when the step size changes.
 * Implies timefield3d_set_boundary(psi, FDTD_BOUNDARY_CPML). */
int timefield3d_set_cpml(timefield3d psi, int thickness, int order, double sigma_max, double kappa_max, double alpha_max);

/* host mirror <-> device */
int timefield3d_sync_host(timefield3d psi);       /* device fields -> psi.fields (waits) */
int timefield3d_sync_device(timefield3d psi);     /* psi.fields, ep, mu, sig, sources -> device */
int timefield3d_synchronize(timefield3d psi);     /* waits for all queued work */
/* one source sample, without touching the rest of the sources (component m = 0..5) */
int timefield3d_set_source_value(timefield3d psi, int i, int j, int k, int m, float value);
/* one field value (waits) */
double timefield3d_get_field_value(timefield3d psi, int i, int j, int k, int m);

/* Probes: after every step, component m at (i,j,k) is appended on the device.
 * read copies the first `count` samples of probe `id` into out (waits). */
int timefield3d_add_probe(timefield3d psi, int i, int j, int k, int m, int capacity);
int timefield3d_read_probe(timefield3d psi, int id, double *out, int count);
int timefield3d_clear_probes(timefield3d psi);

/* Mode-overlap monitors: after every step n (0-based count of steps already
 * taken when the step started) the instantaneous overlap of
 * timefield3d_mode_overlap is formed on the device and accumulated as
 * O_l += e^{i omega_l n delta_t} o(n), in FP64 with compensated summation, for
 * each of n_freq angular frequencies.  Returns the monitor id (>= 0) or -1. */
int timefield3d_add_overlap_monitor(timefield3d psi, int center_x, int center_y, int center_z, mode overlap_mode, int reverse, int n_freq, const double *omega);
int timefield3d_read_overlap_monitor(timefield3d psi, int id, complex *out);   /* n_freq values (waits) */
int timefield3d_clear_monitors(timefield3d psi);
/* number of completed steps since the last timefield3d_zero_fields */
long long timefield3d_step_count(timefield3d psi);

/* Scheduled mode source: before step n the plane source of
 * timefield3d_mode_source (adjoint = 0) or timefield3d_mode_source_adjoint
 * (adjoint = 1) is written with amplitude[n] and phase[n], n < nsteps.
 * Applied by timefield3d_run. */
int timefield3d_set_source_schedule(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode, int reverse, int adjoint, int nsteps, const double *amplitude, const double *phase);
int timefield3d_clear_source_schedule(timefield3d psi);
/* Exact discrete adjoint of an overlap monitor.  No reference counterpart:
 * it replaces the reference driver's CW adjoint (3d_fdtd.c:143-165 with
 * timefield3d_mode_source_adjoint) when the gradient must equal the derivative
 * of the simulated objective.  For a forward run of nsteps steps from zero
 * fields whose monitor (this mode at center_x/y/z, `reverse` as for
 * timefield3d_add_overlap_monitor) accumulates O(omega), and the objective
 * F = Re(w O) with w = weight_re + i weight_im (F = |O| at the forward design:
 * w = conj(O)/|O|), this schedules the adjoint sources so that
 * timefield3d_run(psi, delta_t, nsteps + 1) from zero fields runs the exact
 * adjoint of the leapfrog scheme (the transposed step is the same step with H
 * negated); a spline store bound with which = 1, t0 = nsteps, dir = -1 then
 * holds the adjoint fields for fdtd_spline_store_gradient_exact.  The CPML
 * terms run forward in the adjoint too, so the result is exact up to the
 * absorber's reflection. */
int timefield3d_set_exact_adjoint_schedule(timefield3d psi, int center_x, int center_y, int center_z,
                                           mode monitor_mode, int reverse, int nsteps, double omega, double delta_t,
                                           double weight_re, double weight_im);
/* Bind a taper's edge store to timefield3d_run: after step n the edge fields
 * are stored at time index t0 + dir*n (which = 0 forward, 1 adjoint). */
int adjoint3d_taper_bind_store(adjoint3d_taper taper, timefield3d psi, int which, int t0, int dir);
int adjoint3d_taper_unbind_store(adjoint3d_taper taper, timefield3d psi);
/* nsteps x (scheduled source, timefield3d_apply_timestep_omp_full, probes,
 * monitors, bound taper stores), captured in CUDA graphs; returns at once. */
int timefield3d_run(timefield3d psi, double delta_t, int nsteps);

/* forget the device copy of a mode (call after editing mode.fields in place) */
int timefield3d_release_mode(mode m);

/* CUDA device used by grids created afterwards on this thread */
int fdtd_set_device(int device);
/* kernels this library has launched so far (graph replays counted per kernel) */
long long fdtd_launch_count(void);
/* Waveguide eigenmode on the GPU in FP64: the reference's restarted Arnoldi
 * beta^2 solver, mode_solve_beta_squared (mode.c:3461-3616), same arguments
 * and meaning; fills psi->fields (6 components, H-normalised) and returns
 * beta.  A different name because the reference's mode.o, which a program
 * keeps linking for mode_new and friends, already defines the original.
 * Starts from the reference's rand() vector; stops, like the reference, when
 * |n_eff| changes by less than tol between restarts (at most 5000 restarts,
 * else FDTD_ERR_TIMEOUT).  On failure returns 0 with the status set. */
complex fdtd_mode_solve_beta_squared(mode *psi, double omega, double tol, mode *prev_modes, int prev_num, int size,
                                     int confinement, int lateral_symmetry);
/* restarts the last fdtd_mode_solve_beta_squared took (no reference counterpart) */
int fdtd_mode_solve_restarts(void);
/* One application of the beta^2 operator, mode_apply_beta_squared_operator
 * (mode.c:2796-2943), on the GPU: out.fields = B in.fields (Hx, Hy on interior
 * cells; every other entry 0).  The reference returns a new mode with in's
 * materials; here the caller passes `out` of the same size (its ep/mu/pml are
 * not touched).  Bit-identical to the reference for the same input. */
int fdtd_mode_apply_beta_squared(mode in, double omega, mode out);

/* ---- spline taper (no reference counterpart; generalises timefield3d_set_taper,
 * timefield3d.c:1511-1535, and the taper gradient, adjoint3d.c:339-418) ------
 * Width on plane k: natural cubic spline through `ncontrol` widths (um) placed
 * evenly on [start_z, end_z - 1].  The core spans x in
 * [center_x - w/(2 disc), center_x + w/(2 disc)) (cell units, cell i covers
 * [i, i+1)) on rows [bottom, top); a cell covered by a fraction f gets
 * ep_old + f (ep - ep_old) (mu alike, all 3 components), fully covered cells
 * get ep exactly, so integer edges fill exactly like timefield3d_set_taper. */
/* weights[(k - start_z) * ncontrol + c]: weight of width c in width(k) */
int fdtd_spline_basis(int ncontrol, int start_z, int end_z, double *weights);
/* rasterise (host arrays, and the device copy directly when it is current) */
int timefield3d_set_spline_taper(timefield3d psi, double ep, double mu, int ncontrol, const double *widths,
                                 double center_x, int start_z, int end_z, int bottom, int top);
/* Edge store for the adjoint gradient of a spline taper: E at the cell holding
 * each core edge and at its two x neighbours, per row and plane
 * ([k][j][edge][3], edge 0 right, 1 left; cells floor(x)-1, floor(x),
 * floor(x)+1), for
 * `duration` steps, forward and adjoint, on the GPU.  Bind it to a grid like
 * adjoint3d_taper_bind_store (which 0 forward / 1 adjoint; after step n of
 * timefield3d_run it stores at t0 + dir*n); unbind before freeing. */
typedef struct fdtd_spline_store_ *fdtd_spline_store;
fdtd_spline_store fdtd_spline_store_new(timefield3d psi, int ncontrol, const double *widths, double center_x,
                                        int start_z, int end_z, int bottom, int top, int duration);
int fdtd_spline_store_bind(fdtd_spline_store store, timefield3d psi, int which, int t0, int dir);
int fdtd_spline_store_unbind(fdtd_spline_store store, timefield3d psi);
/* grad[c] = sum_k sum_j W[k][c] / (2 disc) (g_right + g_left) ep_diff with
 * g = sum_t sum_m E_fwd E_adj at the edge cells; cell_gradient (optional,
 * 6*(top-bottom)*(end_z-start_z) values, the store's cell order) receives g */
int fdtd_spline_store_gradient(fdtd_spline_store store, double ep_diff, double *grad, double *cell_gradient);
/* dF/d(control width) for a forward store (which 0, t0 0, dir 1) and an adjoint
 * store from timefield3d_set_exact_adjoint_schedule: per edge cell
 * g = -sum_n sum_m adj[n] (fwd[n] - fwd[n-1]) (dF/deps of the cell), then the
 * spline-weighted reduction of fdtd_spline_store_gradient.  No fitted or
 * omitted constant: the derivative of the simulated objective.  No reference
 * counterpart (generalises adjoint3d.c:339-418). */
int fdtd_spline_store_gradient_exact(fdtd_spline_store store, double ep_diff, double *grad, double *cell_gradient);
/* The same adjoint fields applied to a finite step: grad[c] = sum over the
 * stored cells of g (eps(w + delta e_c) - eps(w - delta e_c)) / (2 delta), with
 * eps from the fill rule at both ends of the step.  It differs from the
 * derivative where the step moves an edge across a cell boundary (the fill is
 * only piecewise linear in the width), and it is what a central difference of
 * the simulated objective with step +-delta measures, to second order.  delta
 * (um) may move an edge by at most one cell.  No reference counterpart. */
int fdtd_spline_store_gradient_step(fdtd_spline_store store, double ep_diff, double delta, double *grad);
void fdtd_spline_store_free(fdtd_spline_store store);

/* BF16 GEMM on the tcgen05 tensor cores (no reference counterpart; the
 * surrogate network's contractions).  Device pointers, queued on `stream`:
 *   pre = alpha A B^T + beta C32 + bias, Z32 = pre, post = act(pre) (0 identity,
 *   1 GELU), C32 = post (FP32), C16 = post (BF16); any output may be NULL.
 * A is M x K, B is N x K, both row-major with K contiguous (lda, ldb and K
 * multiples of 8, operands 16-byte aligned); FP32 accumulation in tensor
 * memory.  *err (device int) is set if a bounded internal wait gave up. */
int fdtd_gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
                   float alpha, float beta, float *C32, int ldc32, void *C16, int ldc16, float *Z32, int ldz,
                   int *err, void *stream);

/* Surrogate network of the taper optimiser (no reference counterpart): MLP
 * n_in -> hidden x3 -> n_out, GELU, BF16 weights and activations with FP32
 * accumulation on the tensor cores, FP32 master weights and Adam.  Host
 * arrays, row-major [batch][n]; batch a multiple of 8.  Parameters in flat
 * order W1 [hidden][n_in], b1, W2, b2, W3, b3, W4 [n_out][hidden], b4. */
void *fdtd_mlp_new(int n_in, int hidden, int n_out, unsigned long long seed);
long long fdtd_mlp_param_count(void *net);
int fdtd_mlp_get_params(void *net, float *params);
int fdtd_mlp_set_params(void *net, const float *params);   /* also resets Adam */
int fdtd_mlp_forward(void *net, const float *x, int batch, float *y);
/* gradients of the mean squared error (no update) */
int fdtd_mlp_gradients(void *net, const float *x, const float *target, int batch, float *grad, double *loss);
/* forward, backward and one Adam step (beta 0.9 / 0.999, eps 1e-8) */
int fdtd_mlp_train_step(void *net, const float *x, const float *target, int batch, float lr, double *loss);
/* dx = (dy/dx)^T dy for each row */
int fdtd_mlp_input_gradient(void *net, const float *x, const float *dy, int batch, float *dx);
void fdtd_mlp_free(void *net);

/* Checkpoint / resume (no reference counterpart): the current fields, CPML
 * auxiliaries, step counters, overlap-monitor accumulators and source planes
 * of a grid, in one file.  Loading needs a grid of the same size, precision,
 * boundary (CPML thickness) and number of monitors with the same frequency
 * counts, set up by the caller as before (materials, modes, schedules);
 * continuing from a loaded checkpoint gives the same results, bit for bit, as
 * never stopping.  Taper edge stores are not included. */
int timefield3d_checkpoint_save(timefield3d psi, const char *path);
int timefield3d_checkpoint_load(timefield3d psi, const char *path);
/* Host-side fault injection for tests: the next n device allocations of the
 * grid engine report FDTD_ERR_ALLOC without touching the GPU (0 clears). */
void fdtd_inject_allocation_failures(int n);

/* Self-test of the engine's bounded device waits (no reference counterpart):
 * one block waits, with the routine the TMA pipeline uses, on a barrier that
 * nothing arrives on.  Expected result FDTD_ERR_TIMEOUT after about
 * limit_seconds (0 < limit <= 10), reported like a real pipeline timeout, with
 * the CUDA context still usable; *elapsed_seconds = the device-side wait. */
int fdtd_wait_selftest(double limit_seconds, double *elapsed_seconds);
/* Candidate sweep: advance `ngrids` grids together, grid i by nsteps[i] steps
 * (uneven counts allowed), in persistent launches of up to steps_per_launch
 * steps that run every grid's one-pass Yee update, monitors and scheduled
 * source (captured as one CUDA graph on the library's sweep stream; returns
 * at once, each grid's stream continues after it).  No reference counterpart:
 * the reference runs one design at a time (3d_fdtd.c:93-202).  Each grid is
 * set up as for timefield3d_run (FP32, CPML of the same thickness on all or
 * PEC walls on all, the same loss, nx a multiple of 4, no probes or bound
 * stores) and ends exactly as timefield3d_run would leave it.  Tile shape:
 * band_rows caps the rows of a band (0: as many as shared memory allows);
 * tiles_per_sm sets how many tiles per SM the grids are cut into per step
 * (in (0, 16]; the blocks take the tiles of all grids from one queue, longest
 * first, so finer tiles balance better).  At most 48 grids per call.  A grid barrier that waits more than 1 s ends the launch;
 * the grids then report FDTD_ERR_TIMEOUT at their next synchronising call. */
int fdtd_sweep_run(const timefield3d *grids, int ngrids, double delta_t, const int *nsteps, int steps_per_launch,
                   int band_rows, double tiles_per_sm);
/* runs the sweep's grid barrier on a barrier nothing can complete, with a
 * limit of limit_seconds (in (0, 10]); returns FDTD_ERR_TIMEOUT when the wait
 * gave up as designed and the context stays usable.  No reference counterpart. */
int fdtd_sweep_barrier_selftest(double limit_seconds);
/* the grid's CUDA stream (cudaStream_t), for callers that order work or time it */
void *timefield3d_get_stream(timefield3d psi);
/* upload psi.ep/mu/sig now (otherwise done on the next device use after a change) */
int timefield3d_upload_materials(timefield3d psi);
/* Kernel timing: while on (on = k > 0), every captured step of one graph
 * replay of timefield3d_run in k records a CUDA event pair around its Yee
 * update (E and H kernels, boundary included); the other replays run without
 * events.  on = 0 turns it off; negative is an argument error.  Read returns
 * the summed milliseconds and the number of timed steps, then resets. */
int timefield3d_set_kernel_timing(timefield3d psi, int on);
int timefield3d_read_kernel_timing(timefield3d psi, double *total_ms, long long *count);

/* Mode overlap of one z-plane that allocates nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory -- code running
 * while a stream is captured into a CUDA graph, applications that own a fixed
 * device-memory budget, loops that cannot afford cudaMalloc's implicit
 * synchronisation -- this computes the instantaneous overlap of
 * timefield3d_mode_overlap (timefield3d.c:3176-3233) entirely from
 * caller-owned device memory: ex, ey, hx, hy point to the nx*ny values of one
 * z-plane (x fastest; double for FDTD_F64, float for FDTD_F32), mode_fields
 * to the 6*mode_i*mode_j complex values of a power-normalised mode in the
 * layout of mode.fields.m, result to one complex that receives
 * -disc^2/2 * sum; ratio = disc / mode disc.  mode_fields and result must
 * be 16-byte aligned (cudaMalloc'd memory is) and ex..hy aligned to their
 * element size; other pointers are refused with FDTD_ERR_ARG before any
 * launch.  Work is queued on `stream`
 * (a cudaStream_t, or NULL for the default stream); the call returns at once.
 * Scratch is a fixed file-scope device array of one partial per plane row:
 * ny may be at most 8192 (larger planes are rejected with FDTD_ERR_ARG).  The
 * first call on each device looks the array's address up; make that first
 * call before any stream capture.  Calls share the array, so calls that can
 * run concurrently on the GPU race; order them on one stream. */
int fdtd_mode_overlap_plane_noalloc(const void *ex, const void *ey, const void *hx, const void *hy, int precision,
                                    int nx, int ny, int center_x, int center_y, const complex *mode_fields,
                                    int mode_i, int mode_j, double ratio, int reverse, double disc,
                                    complex *result, void *stream);
/* copy the device edge storage into taper.forward_fields/adjoint_fields in the
 * reference layout [t][k][j][edge][6] (E components; H left zero) */
int adjoint3d_taper_sync_host(adjoint3d_taper taper);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_B200_H */
