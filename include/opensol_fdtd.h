/*
 * opensol_fdtd.h -- C ABI of the B200 FDTD engine (libopensol_fdtd.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status (OS_OK = 0) and never aborts; the message
 * of the last failure on the calling thread is read with os_fdtd_last_error.  A handle owns its device buffers and
 * one CUDA stream; calls on one handle come from one host thread.  Host pointers are copied in (the caller may reuse
 * them on return); "_device" variants take device pointers the caller keeps alive.
 *
 * Arrays are C-contiguous row-major exactly as open_sol holds them: 2D (nx, ny) with idx = i * ny + j, 3D
 * (nx, ny, nz) with idx = (i * ny + j) * nz + k.  All field arithmetic is float32, evaluated in open_sol's order with
 * no fused multiply-add, so results equal open_sol's CPU backend bit for bit.
 *
 * Each function names the open_sol interface it replaces (file:line inside the open_sol project).
 */
#ifndef OPENSOL_FDTD_H
#define OPENSOL_FDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    OS_OK = 0,
    OS_ERR_INVALID = 1,     /* bad argument or configuration (open_sol raises ValueError / TypeError there) */
    OS_ERR_CUDA = 2,        /* a CUDA call failed (RuntimeError) */
    OS_ERR_NO_MEMORY = 3,   /* device allocation failed */
    OS_ERR_STATE = 4        /* call out of order (e.g. advance before coefficients are set) */
};

/* CPML side bits, open_sol FACES order (open_sol/core/constants.py:18). */
enum { OS_SIDE_X_LO = 1, OS_SIDE_X_HI = 2, OS_SIDE_Y_LO = 4, OS_SIDE_Y_HI = 8, OS_SIDE_Z_LO = 16, OS_SIDE_Z_HI = 32 };

/* Field components of os_fdtd2d_read_field / write_field. */
enum { OS_EZ = 0, OS_HX = 1, OS_HY = 2 };

/* Copies the calling thread's last error message (NUL-terminated, truncated to n) into buf; returns its length. */
int os_fdtd_last_error(char *buf, size_t n);

/* Library version (major * 10000 + minor * 100 + patch). */
int os_fdtd_version(void);

/* Device memory of destroyed 2D engines is kept in a process-wide pool and handed to new engines of the same array
 * sizes (after the old engine's queued work has finished), so engines created and destroyed while others run call
 * neither cudaMalloc nor cudaFree, which waits for the whole device.  At most 16 GiB is kept; os_fdtd_pool_trim frees
 * the pooled memory.  No open_sol counterpart (open_sol relies on cupy's memory pool). */
int os_fdtd_pool_trim(void);

/* Page-locked host memory for material arrays and read-back buffers (cudaHostAlloc), so host<->device copies run at
 * full PCIe / C2C rate.  No open_sol counterpart (open_sol's cupy pool allocates device memory only). */
int os_fdtd_host_alloc(size_t bytes, void **out);
int os_fdtd_host_free(void *ptr);

/* ----------------------------------------------------------------------------------------------------------------
 * 2D E_z polarisation engine (E_z, H_x, H_y): replaces FDTDEngine2D_Ez (open_sol/physics/em/solvers/fdtd_ez_2d.py:11)
 * with its BoundaryManager / CPMLSided state (open_sol/physics/em/boundaries.py:376, 689).
 * ---------------------------------------------------------------------------------------------------------------- */
typedef struct OsFdtd2D OsFdtd2D;

typedef struct {
    int32_t nx, ny;              /* total grid incl. CPML cells (Domain.uniform pads them: core/domain.py:180-197) */
    int32_t periodic_x, periodic_y;
    int32_t npml;                /* CPML cells per active side (BoundaryConfig.cpml_npml) */
    int32_t cpml_sides;          /* OS_SIDE_* bits of the CPML faces */
    int32_t device;              /* CUDA device ordinal */
} OsGrid2D;

/* Zeroed fields, psi slabs and spectra on `device`: FDTDEngine2D_Ez.__init__ (fdtd_ez_2d.py:20-52) plus
 * CPMLSided.__init__ (boundaries.py:694-730).  Refuses a grid that cannot hold its CPML layers plus two rows
 * (cpml_axis_profiles, boundaries.py:604-608). */
int os_fdtd2d_create(const OsGrid2D *grid, OsFdtd2D **out);
int os_fdtd2d_destroy(OsFdtd2D *h);

/* Kappa-folded 1D curl spacings (nx,) (nx,) (ny,) (ny,): _curl_spacings (fdtd_2d_base.py:76-84). */
int os_fdtd2d_set_spacings(OsFdtd2D *h, const float *inv_dx_e, const float *inv_dx_h, const float *inv_dy_e,
                           const float *inv_dy_h);

/* E / H update coefficients from the float32 material arrays (nx, ny): e_coefficients / h_coefficients
 * (fdtd_ez_2d_kernels.py:314-353) evaluated on the device.  sigma_e NULL = lossless (ca = 1 is not stored); mu_r and
 * sigma_m NULL = vacuum permeability everywhere (da = 1, db = dt / mu0 uniform, not stored). */
int os_fdtd2d_set_materials(OsFdtd2D *h, const float *eps_r, const float *sigma_e, const float *mu_r,
                            const float *sigma_m, float dt, float eps0, float mu0);

/* The same from precomputed coefficient arrays (nx, ny): ca NULL = 1; da/db NULL = the uniform values. */
int os_fdtd2d_set_coefficients(OsFdtd2D *h, const float *ca, const float *cb, const float *da, const float *db,
                               float da_uniform, float db_uniform);

/* Copies the device cb (nx, ny) to the host: the calibration input of SheetCurrentCalibration.apply
 * (physics/em/sources.py:582-602). */
int os_fdtd2d_read_cb(OsFdtd2D *h, float *cb);

/* ----------------------------------------------------------------------------------------------------------------
 * 2D H_z polarisation (H_z at the cell centres, E_x on the hi-y faces, E_y on the hi-x faces): replaces
 * FDTDEngine2D_Hz (open_sol/physics/em/solvers/fdtd_hz_2d.py:12).  An OsFdtd2D made by os_fdtd2d_hz_create takes
 * the same spacing, CPML, line-source, flux-line, sample-interval, advance, read/write, reset and stream calls as an
 * E_z engine, with these meanings: a line source adds to E_x (axis 0, the hi-y faces of y-cell `position`) or E_y
 * (axis 1, the hi-x faces of x-cell `position`) after the E update (TangentialSheetCurrentSource,
 * physics/em/sources.py:469-480); a flux line samples E_y (normal 0) or E_x (normal 1) with H_z
 * (FluxMonitor 'hz', physics/em/monitors.py:350-362); field components are OS_HZ_HZ / OS_HZ_EX / OS_HZ_EY.
 * os_fdtd2d_configure takes variant 1 (default: per step an interior kernel over the box of plain cells, tile_rows
 * rows per CTA, 0 = chosen per grid, and a border kernel over the rest) or 0 (one H_z and one E kernel per step) with
 * steps_per_launch 1 or 2: with 2, on a grid without conductivity or magnetic cells whose rows are a multiple of 4
 * cells, the interior box advances two steps per launch and the border two single steps through a scratch field set
 * (allocated by this call), except where the next step is a DFT sample step or field probes are set; results are
 * bit-identical either way.  The E_z-only calls (set_materials,
 * set_coefficients, read_cb, autotune, plan_info, batch, adjoint) return OS_ERR_STATE on an H_z handle and the
 * H_z-only calls below on an E_z handle.
 * ---------------------------------------------------------------------------------------------------------------- */
enum { OS_HZ_HZ = 0, OS_HZ_EX = 1, OS_HZ_EY = 2 };

/* Zeroed H_z engine: FDTDEngine2D_Hz.__init__ (fdtd_hz_2d.py:24-92) with the same grid checks as os_fdtd2d_create. */
int os_fdtd2d_hz_create(const OsGrid2D *grid, OsFdtd2D **out);

/* E face coefficients ca_x, cb_x (E_x faces) and ca_y, cb_y (E_y faces) from the float32 cell arrays (nx, ny) and
 * the float32 face shares lower_x, upper_x (nx,) and lower_y, upper_y (ny,): e_face_coefficients
 * (fdtd_hz_2d_kernels.py:196-277, face_shares yee_grid.py:119-125); da / db as os_fdtd2d_set_materials.  sigma_e
 * NULL = lossless; mu_r, sigma_m NULL = vacuum permeability.  A lossless grid with eps_xx = eps_yy, every eps > 0,
 * and vacuum permeability keeps one eps_r word per cell and the step kernel evaluates cb = dt / (face eps eps0)
 * itself (the same bits as the stored form). */
int os_fdtd2d_hz_set_materials(OsFdtd2D *h, const float *eps_xx, const float *eps_yy, const float *sigma_e,
                               const float *mu_r, const float *sigma_m, const float *lower_x, const float *upper_x,
                               const float *lower_y, const float *upper_y, float dt, float eps0, float mu0);

/* Copies cb_x and cb_y (nx, ny) to the host (the face coefficients SheetCurrentCalibration.apply reads for a
 * TangentialSheetCurrentSource, physics/em/sources.py:586-590). */
int os_fdtd2d_hz_read_cb(OsFdtd2D *h, float *cb_x, float *cb_y);

/* 1 when the lossless one-word-per-cell form is active, else 0.  No open_sol counterpart. */
int os_fdtd2d_hz_form(OsFdtd2D *h, int32_t *lossless_form);

/* Cells the variant-1 step gives the interior kernel and the border kernel.  No open_sol counterpart. */
int os_fdtd2d_hz_plan(OsFdtd2D *h, int64_t *interior_cells, int64_t *border_cells);

/* One CPML side (a single OS_SIDE_* bit): psi recursion rows b, a and bulk curl spacing of its cell-centre (_e) and
 * hi-face (_h) rows, npml each (_cpml_row_set, boundaries.py:671-686; rows from cpml_side_rows, :570-576). */
int os_fdtd2d_set_cpml_side(OsFdtd2D *h, int32_t side, const float *b_e, const float *a_e, const float *inv_e,
                            const float *b_h, const float *a_h, const float *inv_h);

/* Soft E_z line source: axis 0 = line along x at y-cell `position`, 1 = along y at x-cell `position`, half-open
 * span [lo, hi), calibrated float32 profile (hi - lo,): LineSource (core/sources.py:190-229).  At most 16. */
int os_fdtd2d_add_line_source(OsFdtd2D *h, int32_t axis, int32_t position, int32_t lo, int32_t hi,
                              const float *profile, int32_t *source_id);
int os_fdtd2d_set_line_profile(OsFdtd2D *h, int32_t source_id, const float *profile);

/* Flux line: E_z and the tangential H (H_y for normal_axis 0, H_x for 1) on cells [lo, hi) of x-cell (normal 0) or
 * y-cell (normal 1) `position`, nf frequencies, complex128 running DFTs: FluxMonitor (physics/em/monitors.py:325).
 * At most 8. */
int os_fdtd2d_add_flux_line(OsFdtd2D *h, int32_t normal_axis, int32_t position, int32_t lo, int32_t hi, int32_t nf,
                            int32_t *monitor_id);

/* Field-map running DFT over the cell box [x_start, x_stop) x [y_start, y_stop): DFTMonitor (physics/em/
 * monitors.py:248-322).  downsample s >= 1 samples every s-th cell along x and y from the middle of the first s-cell
 * block (dft_sample_slice, monitors.py:152-155); nf frequencies; complex64 sums updated at every DFT sample step with
 * the chunk's phase table, whose rows follow the flux lines' rows, per map in add order.  E_z handle: E_z, (nf, mx,
 * my), one phase table per map.  H_z handle: H_z, E_x and E_y collocated to the cell centres ((3, nf, mx, my)), two
 * phase tables per map (at t, then at t - dt/2 for H_z).  A blocked advance ends a launch on every sample step when
 * a map exists.  Not in batched advances. */
int os_fdtd2d_add_dft_map(OsFdtd2D *h, int32_t x_start, int32_t x_stop, int32_t y_start, int32_t y_stop,
                          int32_t downsample, int32_t nf, int32_t *map_id);

/* Spectra of a field map as float pairs: (nf, mx, my) complex64 (DFTMonitor.ez_dft), or (3, nf, mx, my) on an H_z
 * handle (hz_dft, ex_dft, ey_dft). */
int os_fdtd2d_read_dft_map(OsFdtd2D *h, int32_t map_id, float *spectra);

/* +x plane wave in vacuum on a total-field box of E_z cells [x0, x1) x [y0, y1): TFSFSource (physics/em/sources.py:
 * 206-350).  The host computes, as the reference does, the 1D incident line of aux_cells cells (the box's first
 * column at aux index aux_x0, the soft source at source_index), its H and E coefficients aux_coef_h (aux_cells - 1)
 * and aux_coef_e (aux_cells), the Mur end coefficients, and the side coefficients, 4 floats each: E_z handle, coef_h
 * = H_y rows x0 - 1, x1 - 1 and H_x columns y0 - 1, y1 - 1, coef_e[0..1] = E_z rows x0, x1 - 1; H_z handle
 * (TFSFSourceHz, sources.py:352-379: the incident line holds E_y on its faces and H_z at its centres), coef_h[0..1] =
 * H_z rows x0, x1 - 1, coef_e = E_y rows x0 - 1, x1 - 1 and E_x columns y0 - 1, y1 - 1.  Each step: the H side
 * corrections and the incident H update after the H update, the E side corrections and the incident E update (soft
 * source from row n_lines + box of the chunk's value table) after the E update and the line sources.  An engine with
 * a box advances with the per-half-step kernels.  Not in batched advances or the adjoint.  At most 4. */
int os_fdtd2d_add_tfsf(OsFdtd2D *h, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t aux_cells, int32_t aux_x0,
                       int32_t source_index, const float *coef_h, const float *coef_e, float mur_lo, float mur_hi,
                       const float *aux_coef_h, const float *aux_coef_e, int32_t *tfsf_id);

/* Dispersive pole on the cell box [i0, i1) x [j0, j1) (FDTDEngine2D_Ez.add_drude / add_lorentz, fdtd_ez_2d.py:
 * 123-163): kind 0 Drude (J += damping J + drive E^n before the E update, E -= cb J_total after it on the union box of
 * the Drude poles), kind 1 Lorentz (dP += damping dP - restoring P + drive E^n, P += dP; E -= cb inv_dt dP), with the
 * host's float32 ADE coefficients (DrudePole / LorentzPole.ade_coefficients) and drive = the box's cell mask times the
 * drive coefficient ((i1 - i0) x (j1 - j0) floats); inv_dt = float32(1 / dt).  Poles act in add order, Drude before
 * Lorentz, ahead of the line sources.  An engine with poles advances with the per-half-step kernels.  E_z engines only;
 * not in batched advances or the adjoint.  At most 32. */
int os_fdtd2d_add_pole(OsFdtd2D *h, int32_t kind, int32_t i0, int32_t i1, int32_t j0, int32_t j1, float damping,
                       float restoring, const float *drive, float inv_dt, int32_t *pole_id);

/* Dispersive pole on one E face set of an H_z engine (FDTDEngine2D_Hz.add_drude / add_lorentz, fdtd_hz_2d.py:441-472,
 * updates and corrections :286-325): component 0 = E_x (hi-y faces), 1 = E_y (hi-x faces), on the face box
 * [i0, i1) x [j0, j1); drive = float32(drive coefficient) x the face weight of each face of the box (the width-
 * weighted face average of the pole's cell mask, _pole_faces :547-570).  Kind 0 Drude: J += damping J + drive E^n
 * before the E update, E -= cb J after it; kind 1 Lorentz: dP += damping dP - restoring P + drive E^n, P += dP,
 * E -= cb inv_dt dP; cb of the face set.  Face sets act in add order, all Drude sets before all Lorentz ones, the
 * corrections ahead of the sheet sources.  An engine with poles advances with the per-half-step kernels.  H_z
 * engines only; not in batched advances.  At most 64 face sets. */
int os_fdtd2d_hz_add_pole(OsFdtd2D *h, int32_t kind, int32_t component, int32_t i0, int32_t i1, int32_t j0,
                          int32_t j1, float damping, float restoring, const float *drive, float inv_dt,
                          int32_t *pole_id);

/* Field probe: one component (OS_EZ / OS_HX / OS_HY, or OS_HZ_* on an H_z handle) of cell (ix, iy) recorded after
 * every step from the current one on: FieldProbe.record at t_full (core/monitors.py:194-243, fdtd_2d_base.py:481-487).
 * At most 8.  On an E_z handle the blocked launches stage the probes' cells at every step (same values as one step
 * per launch) while flux lines and probes together number at most 8, else an advance with probes runs one step per
 * launch; on an H_z handle two-step launches record the first step by stepping the probe cells again from the
 * launch's input.  Not in batched advances; os_fdtd2d_advance_noalloc
 * refuses a chunk for which the probes' rows would have to grow. */
int os_fdtd2d_add_probe(OsFdtd2D *h, int32_t ix, int32_t iy, int32_t component, int32_t *probe_id);

/* The probe's values since it was added (or since the last reset), one per step, float32; *n_values = their count
 * (values may be NULL to ask for it). */
int os_fdtd2d_read_probe(OsFdtd2D *h, int32_t probe_id, float *values, int64_t max_values, int64_t *n_values);

/* Steps between DFT samples (dft_sample_interval, physics/em/monitors.py:177-191). */
int os_fdtd2d_set_sample_interval(OsFdtd2D *h, int64_t sample_interval);

/* n_steps Yee steps (FDTDEngine2D_Ez.advance, fdtd_ez_2d.py:71-119, repeated): line_values (n_sources, n_steps)
 * float32 amplitude * temporal(t + dt/2) per step (core/sources.py:221-223); phases: for every monitor in add
 * order, (n_samples, nf) complex64 as float pairs for samples first_sample .. first_sample + n_samples - 1 (sample q
 * is taken after engine step q * sample_interval; monitors.py:22-24,219-220).  Asynchronous on the handle's stream. */
int os_fdtd2d_advance(OsFdtd2D *h, int64_t n_steps, const float *line_values, int64_t first_sample,
                      int64_t n_samples, const float *phases);

/* Floats in the fixed device scratch of os_fdtd2d_advance_noalloc (1 MiB), and the device ordinals it serves. */
#define OS_FDTD_NOALLOC_MAX_FLOATS 262144
#define OS_FDTD_MAX_DEVICES 64

/* os_fdtd2d_advance without any device allocation; no open_sol counterpart.  Same arguments, checks and results as os_fdtd2d_advance, but the chunk's tables go
 * to a fixed file-scope device array of OS_FDTD_NOALLOC_MAX_FLOATS floats instead of the handle's grow-only
 * buffers: for callers that must not allocate mid-run (jobs sharing a GPU on several streams, where cudaFree's
 * device-wide wait would stall the others; jobs held to a fixed memory budget).  Refusals, each with nothing run:
 * n_sources * n_steps source values plus the phase floats (counted only when phases is given, rounded to 64 after
 * the values) must fit, else OS_ERR_INVALID; profiling must be off, and field probes must already have rows for the
 * chunk (advance once with os_fdtd2d_advance to reserve them), else OS_ERR_STATE.  The first call per device looks
 * the array up (it may load the module), so make it before any stream capture; the address is kept for the life of
 * the process, so do not call it again on a device after cudaDeviceReset.  One array per device and process: calls
 * whose device work may overlap (unordered streams) race on it. */
int os_fdtd2d_advance_noalloc(OsFdtd2D *h, int64_t n_steps, const float *line_values, int64_t first_sample,
                              int64_t n_samples, const float *phases);

/* Kernel choice: variant 1 (default) advances steps_per_launch (1..4) Yee steps per launch with temporally blocked,
 * double-buffered kernels, tile_rows rows per interior tile (0, the default: chosen from the grid so that the tiles
 * fill the device's warp slots once, 8..128 rows) and the frame around the interior advanced one step per launch;
 * variant 2 the same with the blocked general kernel on the frame; variant 0 launches one H and one E kernel per
 * step.
 * Every choice gives bit-identical results.  No open_sol counterpart (open_sol launches per half step). */
int os_fdtd2d_configure(OsFdtd2D *h, int32_t variant, int32_t steps_per_launch, int32_t tile_rows);

/* Test hook of the bounded waits, no open_sol counterpart (0, the default: off).  With wait_ns > 0 the next blocked
 * advances make one warp of the interior kernel wait on an mbarrier that nothing completes, for at most wait_ns
 * nanoseconds (<= 2 s), and give up as a real wait does: the handle's error flag is set, that warp's tile is not
 * written, and the next synchronising call returns OS_ERR_CUDA (the flag cleared).  The context stays usable: reset
 * and advance again. */
int os_fdtd2d_set_stall_probe(OsFdtd2D *h, int64_t wait_ns);

/* Kernels the last os_fdtd2d_advance launched. */
int os_fdtd2d_launch_count(OsFdtd2D *h, int64_t *launches);

/* Profiling: with `on`, every kernel of the following advances is bracketed by CUDA events; kernel_times returns the
 * summed device milliseconds and launch count of one kind over the last advance (0 interior blocked kernel, 1 general
 * blocked kernel, 2 DFT kernel, 3 per-step kernel pair).  While profiling, the frame / border kernels run on the
 * handle's stream ahead of the interior kernel instead of beside it, so each event pair times one kernel alone and the
 * shares compare with a serialised launch list.  No open_sol counterpart. */
int os_fdtd2d_set_profiling(OsFdtd2D *h, int32_t on);

/* Autotuner of the interior tile height: times `repeats` launches of steps_per_launch steps for every candidate
 * rows-per-tile, in three interleaved rounds (each candidate keeps its fastest), on the live fields (trial launches
 * write the idle buffer set, which is not swapped in, so the simulation state is unchanged), keeps the fastest as
 * the engine's tile_rows and returns it with its time per launch.  No open_sol counterpart. */
int os_fdtd2d_autotune(OsFdtd2D *h, int32_t steps_per_launch, const int32_t *candidates, int32_t n_candidates,
                       int32_t repeats, int32_t *best_rows, float *best_ms);

/* The blocked kernels' plan for steps_per_launch: cells of the interior rectangle and tiles (warps) of the interior
 * and general kernels.  No open_sol counterpart. */
int os_fdtd2d_plan_info(OsFdtd2D *h, int32_t steps_per_launch, int64_t *interior_cells, int64_t *interior_tiles,
                        int64_t *general_tiles);
int os_fdtd2d_kernel_times(OsFdtd2D *h, int32_t kind, double *total_ms, int64_t *launches);

/* Engine steps taken since create / reset (FDTDEngine2D_Ez.n_step). */
int os_fdtd2d_step_count(OsFdtd2D *h, int64_t *n_step);

/* Spectra of a flux line: (nf, hi - lo) complex128 as double pairs, E then H (_LineSpectra.host, monitors.py:240). */
int os_fdtd2d_read_flux_spectra(OsFdtd2D *h, int32_t monitor_id, double *e_spectra, double *h_spectra);

/* Field copies (nx, ny) float32 (solution_state / restore_solution, fdtd_2d_base.py:419-456). */
int os_fdtd2d_read_field(OsFdtd2D *h, int32_t component, float *out);
int os_fdtd2d_write_field(OsFdtd2D *h, int32_t component, const float *in);

/* Zero fields, psi slabs and spectra and the step count (Fields2D.reset, fields.py:32-36). */
int os_fdtd2d_reset(OsFdtd2D *h);

/* Waits for the handle's stream. */
int os_fdtd2d_synchronize(OsFdtd2D *h);

/* Launch on the caller's CUDA stream (a cudaStream_t; NULL = back to the handle's own stream).  The new stream waits
 * on the device for the work already queued on the previous one (an event; the host does not wait).  The caller keeps that stream alive while the handle uses it: set the
 * handle back (NULL) before destroying the stream; os_fdtd2d_destroy itself never touches a caller's stream.  No
 * open_sol counterpart: the B200 hook for torch streams. */
int os_fdtd2d_set_stream(OsFdtd2D *h, void *cuda_stream);

/* Device milliseconds of the dominant field kernels over the last os_fdtd2d_advance (CUDA events on the handle's
 * stream around its launches; 0 before the first advance). */
int os_fdtd2d_last_advance_ms(OsFdtd2D *h, float *ms);

/* Batched advance of several 2D simulations on one device (the serving loop's step; no open_sol counterpart: open_sol
 * steps one simulation at a time).  Every T steps, one border launch and one interior launch per template
 * configuration cover the tiles of all jobs, and one launch folds all their DFT samples; each job's results equal
 * those of os_fdtd2d_advance.  Jobs must use the blocked kernels with the same steps per launch and be on the batch's
 * stream (os_fdtd2d_set_stream(job, stream of os_fdtd2d_batch_stream)).  line_values / first_samples / n_samples /
 * phases: per job, as os_fdtd2d_advance takes them. */
typedef struct OsFdtd2DBatch OsFdtd2DBatch;
int os_fdtd2d_batch_create(int32_t device, OsFdtd2DBatch **out);
int os_fdtd2d_batch_destroy(OsFdtd2DBatch *b);
int os_fdtd2d_batch_stream(OsFdtd2DBatch *b, void **stream);
int os_fdtd2d_batch_advance(OsFdtd2DBatch *b, OsFdtd2D *const *handles, int32_t n_jobs, int64_t n_steps,
                            const float *const *line_values, const int64_t *first_samples, const int64_t *n_samples,
                            const float *const *phases);
/* Device milliseconds and kernel launches of the last batched advance (waits for it). */
int os_fdtd2d_batch_last_ms(OsFdtd2DBatch *b, float *ms, int64_t *launches);

/* Discrete adjoint of a 2D simulation for d(objective)/d(eps_r) on a design box (no open_sol counterpart: open_sol has
 * no FDTD adjoint).  Checkpoint slots of the full state (fields and psi of the live buffers) are filled by
 * os_fdtd2d_adjoint_save during the forward run; os_fdtd2d_adjoint_segment restores a slot, recomputes n_steps from
 * it with the per-step kernels while recording E over the box, then runs the transposed steps backward through the
 * segment: at the steps source_steps (increasing, indices within the segment) the adjoint sources dJ/de and dJ/dh
 * of DFT samples of flux line monitor_id enter (n_sources x line cells each), and the box accumulates
 * sum lambda_E (E^{n+1} - E^n) in float64 (os_fdtd2d_adjoint_gradient; dJ/deps_r = -that / eps_r where
 * cb = dt / (eps_r eps0)).  Segments run last to first after os_fdtd2d_adjoint_reset; the live fields hold the
 * recomputed state afterwards (reset the simulation before another forward run). */
typedef struct OsAdjoint2D OsAdjoint2D;
int os_fdtd2d_adjoint_create(OsFdtd2D *h, int32_t box_i0, int32_t box_i1, int32_t box_j0, int32_t box_j1,
                             int32_t n_slots, int32_t segment_steps, OsAdjoint2D **out);
int os_fdtd2d_adjoint_destroy(OsAdjoint2D *a);
int os_fdtd2d_adjoint_save(OsAdjoint2D *a, int32_t slot);
int os_fdtd2d_adjoint_reset(OsAdjoint2D *a);
int os_fdtd2d_adjoint_segment(OsAdjoint2D *a, int32_t slot, int64_t step0, int32_t n_steps, const float *line_values,
                              int32_t monitor_id, int32_t n_sources, const int32_t *source_steps,
                              const float *source_e, const float *source_h);
int os_fdtd2d_adjoint_gradient(OsAdjoint2D *a, double *out);

/* ----------------------------------------------------------------------------------------------------------------
 * 3D engine (E_x..H_z): replaces FDTDEngine3D (open_sol/physics/em3d/engine3d.py:157) for a Cartesian grid, one real
 * field set (no Bloch phase) and float32 fields.  Fields (nx, ny, nz) z contiguous, idx = (i * ny + j) * nz + k.
 * ---------------------------------------------------------------------------------------------------------------- */
typedef struct OsFdtd3D OsFdtd3D;

/* Field components of os_fdtd3d_read_field / write_field. */
enum { OS_EX = 0, OS_EY = 1, OS_EZ3 = 2, OS_HX3 = 3, OS_HY3 = 4, OS_HZ3 = 5 };

typedef struct {
    int32_t nx, ny, nz;          /* total grid incl. CPML cells (Domain3D.uniform pads them: core/domain3d.py:55-65) */
    int32_t periodic[3];         /* periodic axes (BoundaryConfig3D.periodic, boundaries3d.py:97-98) */
    int32_t device;              /* CUDA device ordinal */
} OsGrid3D;

/* Zeroed fields on `device`: FDTDEngine3D.__init__ (engine3d.py:162-263) and Fields3D. */
int os_fdtd3d_create(const OsGrid3D *grid, OsFdtd3D **out);
int os_fdtd3d_destroy(OsFdtd3D *h);

/* Kappa-folded curl spacings inv_e (1 / cell width) and inv_h (1 / hi-face spacing, 0 on the last row of an open
 * axis) per axis (engine3d.py:189-203), and the hi-face shares as one array wl_x, wu_x, wl_y, wu_y, wl_z, wu_z
 * (face_shares, physics/em/yee_grid.py:119-125; engine3d.py:204-205). */
int os_fdtd3d_set_rows(OsFdtd3D *h, const float *inv_e_x, const float *inv_e_y, const float *inv_e_z,
                       const float *inv_h_x, const float *inv_h_y, const float *inv_h_z, const float *shares);

/* uint16 material id per cell and the per-id float32 tables (eps per E component with the PEC id at eps -1, sigma_e,
 * mu_r, sigma_m): FDTDEngine3D.rebuild_materials (engine3d.py:337-369, material_index3d.py:131).  The H coefficients
 * da / db per id are derived on the device (edge_coefficients, physics/em3d/kernels3d.py:44-54). */
int os_fdtd3d_set_materials(OsFdtd3D *h, const uint16_t *material_id, int32_t n_ids, const float *t_ex,
                            const float *t_ey, const float *t_ez, const float *t_sig, const float *t_mu,
                            const float *t_sm, float dt);

/* CPML layers of one axis (0, 1, 2): row maps grid row -> psi row (-1 outside), recursion b and gain per psi row, for
 * the E ('e' rows at cell centres) and H ('h' rows at hi faces) kinds: CPMLAxis3D (boundaries3d.py:192-243).  The psi
 * slabs (n_rows x the other two axes, two components per kind) are allocated and zeroed. */
int os_fdtd3d_set_cpml_axis(OsFdtd3D *h, int32_t axis, int32_t n_rows, const int32_t *row_map_e, const float *b_e,
                            const float *gain_e, const int32_t *row_map_h, const float *b_h, const float *gain_h);

/* cb of E component comp on the face of cell (i, j, k): box_face_cb_3d for one cell (kernels3d.py:745-779), the
 * dipole calibration input (DipoleSource3D.calibrate, sources3d.py:56-61).  Synchronous. */
int os_fdtd3d_face_cb(OsFdtd3D *h, int32_t comp, int32_t i, int32_t j, int32_t k, float *cb);

/* Electric dipole on E component comp of cell (i, j, k): E += FP32(s(t + dt/2)) * weight after every E update
 * (DipoleSource3D.inject, sources3d.py:69-75).  At most 16. */
int os_fdtd3d_add_dipole(OsFdtd3D *h, int32_t comp, int32_t i, int32_t j, int32_t k, float weight,
                         int32_t *dipole_id);
int os_fdtd3d_set_dipole_weight(OsFdtd3D *h, int32_t dipole_id, float weight);

/* A flux monitor of nf frequencies (PlaneFlux3D / FluxBox3D, physics/em3d/monitors3d.py:42-162) and its (E, H) pairs:
 * E component e_comp averaged over the layers edge - 1 and edge along normal_axis, H component h_comp on layer
 * edge - 1, over the box origin / extent of the two tangential axes (extent 1 along the normal); complex128 running
 * DFTs (nf, cells) for E and H, cells in grid axis order. */
int os_fdtd3d_add_flux_monitor(OsFdtd3D *h, int32_t nf, int32_t *monitor_id);
int os_fdtd3d_add_flux_pair(OsFdtd3D *h, int32_t monitor_id, int32_t e_comp, int32_t h_comp, int32_t normal_axis,
                            int32_t edge, const int32_t *origin, const int32_t *extent, int32_t *pair_id);
int os_fdtd3d_set_sample_interval(OsFdtd3D *h, int64_t sample_interval);

/* n_steps Yee steps (FDTDEngine3D.advance, engine3d.py:497-554, repeated): dipole_values (n_dipoles, n_steps) float32
 * amplitude FP32(temporal(t + dt/2)) per step; phases: per sample, for every monitor in add order, nf complex64 as
 * float pairs (sample q is taken after engine step q * sample_interval), samples first_sample .. first_sample +
 * n_samples - 1.  Asynchronous on the handle's stream. */
int os_fdtd3d_advance(OsFdtd3D *h, int64_t n_steps, const float *dipole_values, int64_t first_sample,
                      int64_t n_samples, const float *phases);

int os_fdtd3d_read_field(OsFdtd3D *h, int32_t component, float *out);
int os_fdtd3d_write_field(OsFdtd3D *h, int32_t component, const float *in);

/* Spectra of one pair: (nf, cells) complex128 as double pairs, E then H (PlaneFlux3D._pairs e_dft / h_dft). */
int os_fdtd3d_read_flux_pair(OsFdtd3D *h, int32_t pair_id, double *e_spectra, double *h_spectra);

/* Zero fields, psi and spectra; step count back to 0. */
int os_fdtd3d_reset(OsFdtd3D *h);
int os_fdtd3d_synchronize(OsFdtd3D *h);
int os_fdtd3d_set_stream(OsFdtd3D *h, void *cuda_stream);

/* x planes each block of the H / E kernels streams (chosen from the grid at create; results do not depend on it). */
int os_fdtd3d_set_x_chunk(OsFdtd3D *h, int32_t planes);

/* Step form (results bit-identical; no counterpart in open_sol, which has one form): 0 = the H and the E kernel over
 * the whole grid in place; 1 = one fused H + E kernel over every cell but the outermost layer of each axis plus the
 * two-kernel update of that layer, on two field sets and two CPML psi sets swapped every step (twice the field memory,
 * a third less DRAM traffic per step); 2 = form 1 with each x plane of a tile staged in shared memory by tensor copies
 * (rows of a multiple of 8 cells, at least 48; other grids run form 1); 3 (the default) = form 1 with the lean staged
 * kernel (four cells a thread; z rows of a multiple of 4 cells and at least 144, y at least 17, at most 255 z CPML
 * rows; other grids run form 0). */
int os_fdtd3d_set_variant(OsFdtd3D *h, int32_t variant);

/* Launch shape of the fused kernel of forms 1-3, -1..4 (tile rows and the blocks per SM its registers are cut for;
 * -1: the form's default); speed only, results bit-identical. */
int os_fdtd3d_set_fused_config(OsFdtd3D *h, int32_t config);

/* The fused box (i0, i1, j0, j1, k0, k1) and whether the next advance uses it (*fused = 1). */
int os_fdtd3d_interior(OsFdtd3D *h, int32_t *box6, int32_t *fused);
int os_fdtd3d_last_advance_ms(OsFdtd3D *h, float *ms);
int os_fdtd3d_launch_count(OsFdtd3D *h, int64_t *launches);
int os_fdtd3d_step_count(OsFdtd3D *h, int64_t *n_step);

#ifdef __cplusplus
}
#endif
#endif /* OPENSOL_FDTD_H */
