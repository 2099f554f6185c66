/*
 * pmpic_gpu.h -- C ABI of libpmpic_gpu.so, the B200 implementation of the PMPIC
 * per-timestep hot path.
 *
 * The reference (EPCCed/pmpic, Fortran + MPI) runs its hot path as five MONC
 * components whose timestep callbacks the timestepper calls rksteps (= 4) times
 * per model step, in the integrator group order of global_config:43:
 *   vort2vel -> vorticity_tendency -> rk4_integrator -> parcel_splitting -> parcel_mixing
 * Each component exports `<name>_get_descriptor()` with init / timestep /
 * finalise procedure pointers taking `type(model_state_type)`
 * (model_core/src/components/monc_component.F90:51-107).  This header declares
 * the C entry points that new versions of those five component modules bind
 * through `iso_c_binding`: one entry point per timestep
 * callback, plus context set-up, parcel/grid transfer and step information.
 *
 * Conventions
 *  - Every call is synchronous from the caller's view and returns PMPIC_OK (0)
 *    or a negative PMPIC_ERR_* code; pmpic_last_error() gives the message.  The
 *    reference aborts (`error stop`) in the same situations; the Fortran shim
 *    turns a non-zero return into `error stop`.
 *  - Device memory is owned by the context.  Host pointers are borrowed for the
 *    duration of a call.  Parcel state stays on the device between callbacks.
 *  - A context is not thread-safe: one host thread per context (the reference
 *    runs MPI_THREAD_SERIALIZED and calls callbacks from the master thread).
 *  - Parcel slots are 0-based here (Fortran slot n is C slot n-1).
 *  - Grids are exchanged dense, x fastest: physical (nz+1) x ny x nx; spectral
 *    (nz+1) x (ny+2) x (nx+2) in the reference's four-reals-per-mode layout.
 */
#ifndef PMPIC_GPU_H
#define PMPIC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------- */
#define PMPIC_OK              0
#define PMPIC_ERR_CONFIG     -1  /* invalid configuration (sizes, origin, capacity) */
#define PMPIC_ERR_CAPACITY   -2  /* max_parcels reached: parcel_splitting.F90:90-93, parcel_mixing.F90:196-199, haloswap.F90:705-708 */
#define PMPIC_ERR_OUT_OF_BOX -3  /* parcel outside the grid: parcel_interpolation.F90:222-237 */
#define PMPIC_ERR_ZERO_PIVOT -4  /* tridiagonal zero pivot: fft_ops.F90:642-645 */
#define PMPIC_ERR_BACKFILL   -5  /* mixing backfill ran below slot 1 (reference reads keep(0)) */
#define PMPIC_ERR_TIMEOUT    -6  /* a bounded device wait gave up */
#define PMPIC_ERR_CUDA       -7  /* CUDA runtime error */
#define PMPIC_ERR_ARG        -8  /* invalid argument */
#define PMPIC_ERR_STATE      -9  /* call not valid in the current state */
#define PMPIC_ERR_TOO_LARGE -10  /* size beyond a fixed static maximum (pmpic_par2grid_static) */

/* ---- precision forms ---------------------------------------------------- */
#define PMPIC_FP64  0            /* plain FP64 throughout (the reference's DEFAULT_PRECISION) */
#define PMPIC_MIXED 1            /* FP32 fields, grids, transforms and RK4; positions as integer cell
                                    index + FP32 offset; FP64 zero mode */

/* ---- parcel property ids (parcels.F90:19-34) ----------------------------- */
enum {
  PMPIC_PROP_X = 0, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R,
  PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT, PMPIC_PROP_DRDT,
  PMPIC_PROP_H, PMPIC_PROP_B, PMPIC_PROP_VOL, PMPIC_PROP_STRETCH, PMPIC_PROP_TAG, PMPIC_PROP_BTOT,
  PMPIC_PROP_XO, PMPIC_PROP_YO, PMPIC_PROP_ZO, PMPIC_PROP_XF, PMPIC_PROP_YF, PMPIC_PROP_ZF,
  PMPIC_PROP_PO, PMPIC_PROP_QO, PMPIC_PROP_RO, PMPIC_PROP_PF, PMPIC_PROP_QF, PMPIC_PROP_RF,
  PMPIC_NPROP
};

/* ---- grid ids (state.F90:38-67; vorticity_tendency.F90:90-91) ----------- */
enum {
  PMPIC_GRID_U = 0, PMPIC_GRID_V, PMPIC_GRID_W, PMPIC_GRID_P, PMPIC_GRID_Q, PMPIC_GRID_R,
  PMPIC_GRID_B, PMPIC_GRID_DP, PMPIC_GRID_DQ, PMPIC_GRID_DR, PMPIC_GRID_VOL, PMPIC_GRID_HG,
  PMPIC_NGRID
};
enum { PMPIC_SPEC_U = 0, PMPIC_SPEC_V, PMPIC_SPEC_W, PMPIC_NSPEC };  /* u_s, v_s, w_s */

typedef struct pmpic_ctx pmpic_ctx;

/* Model configuration: the hot-path keys of config.mcf / global_config. */
typedef struct pmpic_config {
  int32_t nx, ny, nz;              /* cell counts (config keys nx, ny, nz); nz+1 z points (setup_grid.F90:51) */
  double xmin, xmax, ymin, ymax, zmin, zmax;  /* domain; the origins must be 0 (the reference adds a non-zero origin twice) */
  double dtm, dtmax;               /* rk4_integrator.F90:38-41 */
  double timestep_prefactor;       /* vorticity_tendency.F90:96 */
  int64_t max_parcels;             /* parcelsetup_base max_parcels */
  int32_t precision;               /* PMPIC_FP64 or PMPIC_MIXED */
  int32_t device;                  /* CUDA device ordinal */
} pmpic_config;

/* Per-step counters, copied to the host once per call of pmpic_get_step_info. */
typedef struct pmpic_step_info {
  int64_t n_parcels;               /* numparcels_local */
  double dtm;                      /* state%dtm after the dt rule */
  int32_t limiter;                 /* 0 dtmax, 1 velocity (vort2vel.F90:368), 2 vorticity (vorticity_tendency.F90:300) */
  int64_t n_split;                 /* parcels split in the last splitting call */
  int64_t n_removed;               /* nremove of the last mixing call */
  int64_t n_added;                 /* nadd of the last mixing call */
  int64_t n_migrated;              /* parcels re-slotted by the last parcel haloswap */
  double vol_sum, hvol_sum, bvol_sum;  /* domain totals of vol, h*vol and b*vol over the parcels by a
                                          compensated FP64 reduction (both forms), taken after each
                                          acting mixing call and by pmpic_conserved_sums; the reference
                                          checks mixing by them (parcel_mixing.F90:87-103, :409-418) */
  int32_t error;                   /* sticky device error word (PMPIC_ERR_*) */
  char message[160];
} pmpic_step_info;

/* ---- context ------------------------------------------------------------ */
/* Replaces the initialisation callbacks of the five components plus the
 * setup_grid / parcelsetup_base allocation (setup_grid.F90:116-144,
 * parcelsetup_base.F90:63-81, rk4_integrator.F90:33-78, vort2vel.F90:46-90,
 * vorticity_tendency.F90:52-99, parcel_mixing.F90:46-64). */
int  pmpic_create(const pmpic_config* cfg, pmpic_ctx** out);
/* Replaces the finalisation callbacks (e.g. rk4_integrator.F90:321-337). */
void pmpic_destroy(pmpic_ctx* ctx);
const char* pmpic_last_error(const pmpic_ctx* ctx);

/* ---- parcel transfer (setup, restart and dumps; not on the timestep path) -- */
/* Sets numparcels_local = n and the 11 prognostic properties of slots 0..n-1;
 * the RK4 arrays and tendencies of those slots are set to zero and a sticky
 * device error from an earlier call is cleared. */
int pmpic_upload_parcels(pmpic_ctx* ctx, int64_t n,
                         const double* x, const double* y, const double* z,
                         const double* p, const double* q, const double* r,
                         const double* b, const double* h, const double* vol,
                         const double* stretch, const double* tag);
/* Copies slots 0..n-1 (n = numparcels_local, returned in *n) of the same 11
 * properties; any pointer may be NULL. Fails if capacity < n. */
int pmpic_download_parcels(pmpic_ctx* ctx, int64_t capacity, int64_t* n,
                           double* x, double* y, double* z, double* p, double* q, double* r,
                           double* b, double* h, double* vol, double* stretch, double* tag);
/* Generic property access over slots 0..n-1 (n <= max_parcels). */
int pmpic_set_property(pmpic_ctx* ctx, int prop, int64_t n, const double* src);
int pmpic_get_property(pmpic_ctx* ctx, int prop, int64_t n, double* dst);
int pmpic_set_count(pmpic_ctx* ctx, int64_t n);
int pmpic_get_count(pmpic_ctx* ctx, int64_t* n);

/* ---- component timestep callbacks (one call each, as the timestepper does) -- */
int pmpic_vort2vel(pmpic_ctx* ctx);              /* vort2vel.F90:98-400 */
int pmpic_vorticity_tendency(pmpic_ctx* ctx);    /* vorticity_tendency.F90:107-334 */
int pmpic_rk4_integrator(pmpic_ctx* ctx);        /* rk4_integrator.F90:95-319 (+ parcel_haloswap) */
int pmpic_parcel_splitting(pmpic_ctx* ctx);      /* parcel_splitting.F90:47-168 */
int pmpic_parcel_mixing(pmpic_ctx* ctx);         /* parcel_mixing.F90:68-431 */
/* (The kept-class grids of construct_grids go to the vol, b, hg, p, q, r grids as in the
 * reference.  A call that removes no parcel makes the vol grid in full and the b, hg, p, q, r
 * sums only at the corners of new parcels' cells, the only points mixing reads; elsewhere
 * those five grids are left as scratch.) */
/* nsteps model steps: the integrator group run rksteps (=4) times per step
 * (timestepper.F90:89-106 with global_config:43's group contents). */
int pmpic_step(pmpic_ctx* ctx, int nsteps);

/* The reference's test components for the parcel migration path (FP64
 * contexts; PMPIC_ERR_STATE on a mixed one):
 * euler_integrator timestep (euler_integrator.F90:53-86): x, y, z, p, q, r
 * += tendency * dtm, then the parcel haloswap;
 * prescribed_parcel_velocity timestep (velocity.F90:96-255): dxdt, dydt, dzdt
 * set from the profile (PMPIC_VELOCITY_*, the reference's velocity_profile
 * codes) at each parcel's position, with x0, y0 the domain centre and r0 an
 * eighth of its x extent (:66-69); and its initialisation's quadrant tags on
 * one process (:72-84: tag = 2 [y > y0] + [x > x0]). */
#define PMPIC_VELOCITY_SHEAR 0        /* dydt = tanh((x - x0) / r0) */
#define PMPIC_VELOCITY_NORTH 1        /* 1..8: the compass directions N, NE, E, SE, S, SW, W, NW */
#define PMPIC_VELOCITY_NORTH_WEST 8
#define PMPIC_VELOCITY_CYLINDRICAL 9  /* a Gaussian vortex about (x0, y0) */
#define PMPIC_VELOCITY_EVACUATE 10    /* flow out of (x/4, y/4) into (3x/4, 3y/4) */
int pmpic_euler_integrator(pmpic_ctx* ctx);
int pmpic_prescribed_velocity(pmpic_ctx* ctx, int profile);
int pmpic_prescribed_velocity_tag(pmpic_ctx* ctx);
int pmpic_get_step_info(pmpic_ctx* ctx, pmpic_step_info* info);
/* The domain totals of vol, h*vol and b*vol over the current parcels now
 * (sums[0..2]; also left in pmpic_step_info): every product split exactly and
 * summed in double-double in a fixed order, so the result is the FP64 rounding
 * of the exact total and repeats bit for bit.  The diagnostic sums around
 * mixing of parcel_mixing.F90:87-103 and :409-418. */
int pmpic_conserved_sums(pmpic_ctx* ctx, double sums[3]);

/* Component iteration counters (vort2vel, vorticity_tendency, rk4 stage,
 * splitting, mixing) -- the modules' `iteration` / `rkstep` save variables. */
int pmpic_get_counters(pmpic_ctx* ctx, int32_t counters[5]);
int pmpic_set_counters(pmpic_ctx* ctx, const int32_t counters[5]);
int pmpic_set_dtm(pmpic_ctx* ctx, double dtm);

/* ---- grid transfer (diagnostics, writebinary-style dumps, tests) ---------- */
int pmpic_download_grid(pmpic_ctx* ctx, int grid, double* dst);      /* (nz+1) x ny x nx */
int pmpic_upload_grid(pmpic_ctx* ctx, int grid, const double* src);
int pmpic_download_spectral(pmpic_ctx* ctx, int spec, double* dst);  /* (nz+1) x (ny+2) x (nx+2) */

/* ---- kernel-level entry points (the model-core routines the components call) */
/* cache_parcel_interp_weights (parcel_interpolation.F90:186-262): writes the
 * interior cell id ((k-1)*ny + (j-3))*nx + (i-3) of slots 0..n-1. */
int pmpic_op_cell_ids(pmpic_ctx* ctx, int32_t* cells);
/* par2grid (parcel_interpolation.F90:336-481) of a property into a grid. */
int pmpic_op_par2grid(pmpic_ctx* ctx, int prop, int grid);
/* grid2par (parcel_interpolation.F90:267-332) of a grid into a property. */
int pmpic_op_grid2par(pmpic_ctx* ctx, int grid, int prop);
/* perform_forward_3dfft / perform_backwards_3dfft (pencilfft.F90:151-212). */
int pmpic_op_fft_forward(pmpic_ctx* ctx, const double* phys, double* spec);
int pmpic_op_fft_backward(pmpic_ctx* ctx, const double* spec, double* phys);
/* fft_ops.F90: diffx :204-302, diffy :305-401, spectral_filter :176-197,
 * diffz :419-483 (bot/top may be NULL; else (ny+2) x (nx+2)), laplinv :505-601. */
int pmpic_op_diffx(pmpic_ctx* ctx, const double* in, double* out);
int pmpic_op_diffy(pmpic_ctx* ctx, const double* in, double* out);
int pmpic_op_filter(pmpic_ctx* ctx, const double* in, double* out);
int pmpic_op_diffz(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top);
int pmpic_op_laplinv(pmpic_ctx* ctx, double* inout, int df_zero_on_boundary);
/* parcel_haloswap (parcels/haloswap.F90:109-289), single-GPU semantics. */
int pmpic_op_parcel_haloswap(pmpic_ctx* ctx);

/* par2grid (parcel_interpolation.F90:336-481) of nf (1, 3 or 4) properties into
 * nf grids with one set of weights, in the context's precision (the mixed form
 * takes FP32 properties only). */
int pmpic_op_par2grid_multi(pmpic_ctx* ctx, int nf, const int* props, const int* grids);
/* grid2par (parcel_interpolation.F90:267-332) of ng (1, 3 or 6) grids into ng
 * properties at the current positions. */
int pmpic_op_grid2par_multi(pmpic_ctx* ctx, int ng, const int* grids, const int* props);
/* The inversion of vort2vel.F90:139-320 alone, on the gridded vorticity
 * already in grids p, q, r: velocity into u, v, w, corrected vorticity into
 * p, q, r, filtered spectra into u_s, v_s, w_s.  Both precisions. */
int pmpic_op_vort2vel_grids(pmpic_ctx* ctx);
/* Renumbers parcel slots into cell order (cell id z fastest, slot order kept
 * inside a cell), moving every property.  No counterpart in the reference,
 * whose slot order is part of its integer bookkeeping: use it where slot
 * numbering does not matter (e.g. after set-up, before a run) to make the
 * parcel gathers of par2grid and the RK4 stage contiguous.  Allocates a
 * temporary device buffer of n doubles. */
int pmpic_sort_parcels(pmpic_ctx* ctx);

/* par2grid without a context and without allocation.  No counterpart in the
 * reference: an addition for callers that cannot allocate device memory when
 * they call it, such as a host model whose device memory is all handed to its
 * own pool allocator, or one that forbids cudaMalloc (which can synchronize the
 * device) inside its time step.  Same arithmetic and result as pmpic_op_par2grid (binning
 * parcel_interpolation.F90:186-262, par2grid :336-481) of one field with volume
 * weights over an nx x ny x nz box, x in [0,lx), y in [0,ly), z in [0,lz) (the
 * reference's binning rule k < nz rejects z = lz).  nx, ny >= 4 and nz >= 3,
 * as pmpic_create requires, else PMPIC_ERR_ARG.  x, y, z, vol, field are n
 * device doubles; out receives the dense (nz+1) x ny x nx grid on the device.
 * Scratch is one fixed static device array (about 7 MB per device):
 * n <= 131072, nx*ny*nz <= 32768 and ceil(nz/16)*nx*ny <= 4096, else
 * PMPIC_ERR_TOO_LARGE with nothing launched.  The call clears its own counters,
 * runs on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * synchronizes that stream before returning; PMPIC_ERR_OUT_OF_BOX if a parcel
 * is outside the box.
 *  - Calls that overlap on one device share the scratch and race: serialize
 *    them (one stream, or synchronize between calls).
 *  - The first call on a device, made with that device current, looks up the
 *    scratch array's device address (cudaGetSymbolAddress); make that first
 *    call before any stream capture begins. */
int pmpic_par2grid_static(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                          int64_t n, const double* x, const double* y, const double* z,
                          const double* vol, const double* field, double* out, void* stream);

/* ---- dumps and restart in the reference's binary stream format ------------- */
/* A parcel dump of writebinary.F90:149-199: time, the domain bounds, the count
 * (int64), then x, y, z, p, q, r, dxdt, dydt, dzdt, dpdt, dqdt, drdt, h, b, vol,
 * stretch, tag as FP64 arrays (native byte order).  The reference's reader and
 * post-processing tools read it as one rank's file. */
int pmpic_write_parcels(pmpic_ctx* ctx, const char* path, double time);
/* Restart from a parcel dump (readfromfile_parcelsetup.F90:169-290): the
 * parcels of the file inside this domain, in file order, replace the current
 * parcels (append = 0) or follow them (append != 0, one call per file of a
 * multi-rank dump); *time (may be NULL) receives the dump's time. */
int pmpic_read_parcels(pmpic_ctx* ctx, const char* path, int append, double* time);
/* A grid dump of writebinary.F90:201-299: p, q, r, b, h gridded afresh from the
 * parcels, hgliq = max(0, hg - exp(-z)), b + 12.5 hgliq, written with u, v, w
 * and vol as FP64, z fastest.  The model's own grids are not changed. */
int pmpic_write_grids(pmpic_ctx* ctx, const char* path, double time);
/* The NetCDF files of writenetcdf.F90 (write_ncgrid_file :225-308,
 * write_parcels_to_file :310-439), one process, in the NetCDF classic
 * 64-bit-offset format (the reference writes NetCDF-4; netCDF readers open
 * both).  time is stored as given (the reference stores time + dtm); timestep
 * is the model step number; dtm is the context's.  Grid file: dimensions
 * time, z (nz+1), y, x; variables time, z, y, x, then u, v, w, p, q, r,
 * b (+12.5 hgliq), hg, hgliq, vol over (time, x, y, z) gridded as in
 * pmpic_write_grids, then timestep and dtm.  Parcel file: dimensions time and
 * the unlimited nparcel; records parcel (1..n) and the 17 properties of
 * pmpic_write_parcels (stretch under the reference's key "stetch"); the
 * index bounds x_start .. z_end; timestep and dtm. */
int pmpic_write_grids_netcdf(pmpic_ctx* ctx, const char* path, double time, int32_t timestep);
int pmpic_write_parcels_netcdf(pmpic_ctx* ctx, const char* path, double time, int32_t timestep);
/* The same files from host arrays: fields[10] each (nz+1)*ny*nx values, z
 * fastest, on [0,lx) x [0,ly) x [0,lz]; props[17] each n values in the order
 * x, y, z, p, q, r, dxdt, dydt, dzdt, dpdt, dqdt, drdt, h, b, vol, stretch, tag. */
int pmpic_netcdf_write_grids(const char* path, int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                             double time, int32_t timestep, double dtm, const double* const* fields);
int pmpic_netcdf_write_parcels(const char* path, int32_t nx, int32_t ny, int32_t nz, int64_t n, double time,
                               int32_t timestep, double dtm, const double* const* props);

/* ---- ensembles (no counterpart in the reference, which runs one model per job) --
 * A batch of independent plumes of uneven grid sizes and parcel counts on one
 * GPU.  Every member is a full context (its own stream, its own device state):
 * set it up with the single-context calls on pmpic_ensemble_member(e, i).
 * pmpic_ensemble_step advances every member nsteps model steps, members running
 * concurrently (a pool of host threads, largest members first). */
typedef struct pmpic_ensemble pmpic_ensemble;
/* n members with one configuration each; all on the same device. */
int  pmpic_ensemble_create(int n, const pmpic_config* cfgs, pmpic_ensemble** out);
void pmpic_ensemble_destroy(pmpic_ensemble* e);
pmpic_ctx* pmpic_ensemble_member(pmpic_ensemble* e, int i);
/* Host threads stepping members at once; 0 (the default) tunes the number
 * online: the first steps of the next run try 2, 4, 8, 16, 32, 64 threads, one
 * step each, and the rest of the run uses the fastest.  1 runs the members
 * one after another (the sequential baseline). */
int  pmpic_ensemble_set_concurrency(pmpic_ensemble* e, int threads);
/* Tile tuning: for each distinct grid size, the par2grid row-pass column
 * segment (8, 16, 32 or 64 columns per warp) with the shortest time, timed on
 * a member's own parcels; no member state changes (grids p, q, r, b are
 * overwritten, as the next vort2vel does anyway). */
int  pmpic_ensemble_autotune(pmpic_ensemble* e);
/* nsteps model steps of every member; *device_ms (may be NULL) receives the
 * device time from the first member's start to the last member's end. */
int  pmpic_ensemble_step(pmpic_ensemble* e, int nsteps, float* device_ms);
/* The tuning in use: host threads, and per member the par2grid segment. */
int  pmpic_ensemble_tuning(pmpic_ensemble* e, int* threads, int32_t* xseg_per_member);
/* Columns per x segment of the par2grid row pass of one context (default 64). */
int  pmpic_set_p2g_segment(pmpic_ctx* ctx, int xseg);

/* ---- instrumentation ------------------------------------------------------ */
/* Named timers after the reference's timer_mod (register_routine_for_timing /
 * timer_start / timer_stop, model_core/src/utils/timer.F90:110-245), backed by
 * CUDA events on the context's stream: cache_weights, par2grid, grid2par,
 * fft_fwd_tot, fft_inv_tot, diffz, laplinv, vort2vel, vort_tend,
 * RK4_all_steps, Par_HSWP_entire, splitting, mixing, step, rk4_kernel (the RK4
 * stage kernel alone).  Enabling resets. */
int pmpic_timing(pmpic_ctx* ctx, int enable);
int pmpic_timer_count(void);
const char* pmpic_timer_name(int id);
int pmpic_timer_read(pmpic_ctx* ctx, int id, double* total_ms, int64_t* calls);
/* Number of kernels this context has launched since creation. */
int pmpic_launch_count(pmpic_ctx* ctx, int64_t* n);
/* CUDA events recorded on the context's stream (slots 0..7), for timing a
 * region of calls on the device; elapsed time in milliseconds. */
int pmpic_event_record(pmpic_ctx* ctx, int slot);
int pmpic_event_elapsed(pmpic_ctx* ctx, int slot_a, int slot_b, float* ms);
/* Page-lock (pin) an existing host buffer for fast transfers, and release it. */
int pmpic_pin_host(void* ptr, size_t bytes);
int pmpic_unpin_host(void* ptr);

/* ---- parcel set-up (new set-up components; not on the graded path) -------- */
/* Jittered thermal plume: sub^3 parcels per cell on a sub-lattice jittered by
 * U(+-jitter) sub-spacings (Philox4x32-10 keyed by seed and parcel index),
 * vol = cell volume / sub^3, zero vorticity, tag = parcel index.  Buoyancy
 * b = max(0, z - z_strat) * n2 + excess * cos^2(pi r / (2 radius)) inside the
 * thermal; humidity h = h_in inside, h_env0 * (1 - z / Lz) outside.
 * Parcels are ordered cell by cell (x outer, then y, then z) and, inside a
 * cell, sub-lattice point by point (x outer, z inner), the order of
 * basic_parcelsetup.F90:90-118. */
typedef struct pmpic_thermal_params {
  int32_t nx, ny, nz;
  double lx, ly, lz;
  int32_t sub;            /* parcels per cell per direction (2) */
  double jitter;          /* jitter amplitude in sub-spacings (0.25) */
  uint64_t seed;
  double xc, yc, zc, radius, excess;
  double h_in, h_env0;
  double z_strat, n2;
} pmpic_thermal_params;
int64_t pmpic_setup_count(const pmpic_thermal_params* prm);
int pmpic_setup_thermal(const pmpic_thermal_params* prm, int64_t n,
                        double* x, double* y, double* z, double* p, double* q, double* r,
                        double* b, double* h, double* vol, double* stretch, double* tag);
/* The same thermal written on the device into the context's parcel state
 * (either form), replacing it: the parcels of pmpic_setup_thermal, positions,
 * h, vol and tag bit for bit, b within the rounding of the device cos; the
 * count is pmpic_setup_count(prm). */
int pmpic_setup_thermal_device(pmpic_ctx* ctx, const pmpic_thermal_params* prm);

/* basic_parcelsetup initialisation (basic_parcelsetup.F90:22-134), one
 * process, written on the device into the context's parcel state (either
 * form), replacing it: parcels_per_cell_dir^3 parcels per cell at the centres
 * of a regular sub-lattice, cell by cell (x outer, z inner), vol = 1, the
 * other properties zero.  PMPIC_ERR_CAPACITY if they exceed max_parcels. */
int pmpic_setup_basic(pmpic_ctx* ctx, int32_t parcels_per_cell_dir);

/* plume_parcelsetup initialisation (plume_parcelsetup.F90:58-334), one
 * process, written on the device into the context's parcel state (either
 * form), replacing it.  Plume parcels (4^3 per cell on a lattice, inside a
 * sphere of radius r_plume * lambda resting on z = 0 at the domain centre)
 * take the first *n_plume slots; environment parcels (2^3 per cell, outside
 * the sphere) follow, in the reference's loop order.  Sets x, y, z, b, h and
 * vol as the reference does; the other properties are zero.  The reference's
 * parameter checks (:86-131) return PMPIC_ERR_ARG, and so does a plume that
 * reaches above the domain top; too many parcels return PMPIC_ERR_CAPACITY. */
typedef struct pmpic_plume_params {
  double lambda;       /* scale height (config key lambda) */
  double H;            /* relative humidity of the environment, < 1 (H) */
  double z_c;          /* the plume's humidity is exp(-z_c) (z_c) */
  double mu;           /* environment humidity / plume humidity, in (H, 1] (mu) */
  double z_d, z_m;     /* the stratified layer's buoyancy gradient levels (z_d, z_m) */
  double r_plume;      /* plume radius in scale heights (r_plume) */
  double e_values[3];  /* buoyancy perturbation coefficients (e_values) */
} pmpic_plume_params;
int pmpic_setup_plume(pmpic_ctx* ctx, const pmpic_plume_params* prm, int64_t* n_plume);

#ifdef __cplusplus
}
#endif
#endif /* PMPIC_GPU_H */
