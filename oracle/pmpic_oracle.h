/*
 * pmpic_oracle.h -- CPU restatement of the PMPIC per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker and the timed
 * CPU baseline for the B200 library in pmpic_b200/.  Only tests/, the smoke()
 * entry point and bench.py's cpu_baseline / --impl reference legs may load it.
 * The product path never calls it.
 *
 * It restates, in FP64 and with the reference's serial loop orders, the Fortran
 * routines of EPCCed/pmpic that the integrator group runs every substep:
 *   model_core/src/parcels/parcel_interpolation.F90   (binning, par2grid, grid2par)
 *   model_core/src/communication/MPIC_Haloswap.F90     (grid halo copy / sum, 1 rank)
 *   model_core/src/parcels/haloswap.F90                (parcel migration, 1 rank)
 *   model_core/src/fft/pencilfft.F90, ffte_mod.F90     (semi-spectral transforms)
 *   model_core/src/fft/fft_ops.F90                     (diffx/y/z, laplinv, filter)
 *   components/vort2vel, vorticity_tendency, rk4_integrator,
 *   components/parcel_splitting, parcel_mixing
 * Each function in pmpic_oracle.cpp cites the file:line it follows.
 *
 * Parity status: the interpolation, z-solver, mixing and splitting restatements
 * are pinned by the reference's own known-answer tests (grid2partest linear
 * fields, analytic laplinv potentials, mixing conservation, split geometry,
 * migration count conservation) re-implemented under tests/.  FFT output bits
 * are not pinned by any reference fixture; the transform is checked against
 * numpy.fft instead.
 */
#ifndef PMPIC_ORACLE_H
#define PMPIC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* Property ids: identical numbering to include/pmpic_gpu.h (PMPIC_PROP_*). */
enum {
  ORC_X = 0, ORC_Y, ORC_Z, ORC_P, ORC_Q, ORC_R,
  ORC_DXDT, ORC_DYDT, ORC_DZDT, ORC_DPDT, ORC_DQDT, ORC_DRDT,
  ORC_H, ORC_B, ORC_VOL, ORC_STRETCH, ORC_TAG, ORC_BTOT,
  ORC_XO, ORC_YO, ORC_ZO, ORC_XF, ORC_YF, ORC_ZF,
  ORC_PO, ORC_QO, ORC_RO, ORC_PF, ORC_QF, ORC_RF,
  ORC_NPROP
};

/* Grid ids (physical grids, returned as interior (Nz+1) x Ny x Nx, x fastest). */
enum {
  ORC_GU = 0, ORC_GV, ORC_GW, ORC_GP, ORC_GQ, ORC_GR, ORC_GB,
  ORC_GDP, ORC_GDQ, ORC_GDR, ORC_GVOL, ORC_GHG, ORC_NGRID
};
/* Spectral ids ((Nz+1) x (Ny+2) x (Nx+2), x' fastest). */
enum { ORC_SU = 0, ORC_SV, ORC_SW, ORC_NSPEC };

typedef struct orc_step_info {
  int64_t n_parcels;
  double dtm;
  int limiter;          /* 0 = dtmax, 1 = velocity, 2 = vorticity */
  int64_t n_split;
  int64_t n_removed;
  int64_t n_added;
  int64_t n_migrated;   /* parcels re-slotted by the last parcel haloswap */
  int error;
  char message[160];
} orc_step_info;

orc_ctx* orc_create(int nx, int ny, int nz,
                    double xmin, double xmax, double ymin, double ymax,
                    double zmin, double zmax,
                    double dtm, double dtmax, double timestep_prefactor,
                    int64_t max_parcels);
void orc_destroy(orc_ctx*);
int  orc_error(const orc_ctx*, char* msg, int len);
void orc_set_threads(int n);

int     orc_set_count(orc_ctx*, int64_t n);
int64_t orc_count(const orc_ctx*);
int     orc_set_prop(orc_ctx*, int prop, const double* src, int64_t n);   /* slots 0..n-1 */
int     orc_get_prop(const orc_ctx*, int prop, double* dst, int64_t n);   /* slots 0..n-1 */
int     orc_get_grid(const orc_ctx*, int grid, double* dst);
int     orc_set_grid(orc_ctx*, int grid, const double* src);
int     orc_get_spec(const orc_ctx*, int spec, double* dst);
void    orc_get_step_info(const orc_ctx*, orc_step_info*);

/* Kernel-level entry points (used by the parity tests). */
int orc_cache_weights(orc_ctx*, int32_t* cells /* may be NULL */);
int orc_par2grid(orc_ctx*, int prop, int grid);
int orc_grid2par(orc_ctx*, int grid, int prop);
int orc_fft_forward(orc_ctx*, const double* phys, double* spec);
int orc_fft_backward(orc_ctx*, const double* spec, double* phys);
int orc_diffx(orc_ctx*, const double* in, double* out);
int orc_diffy(orc_ctx*, const double* in, double* out);
int orc_diffz(orc_ctx*, const double* in, double* out, const double* bot, const double* top);
int orc_laplinv(orc_ctx*, double* inout, int df_zero_on_boundary);
int orc_filter(orc_ctx*, const double* in, double* out);
int orc_parcel_haloswap(orc_ctx*);
int orc_kx_ky_k2(orc_ctx*, double* kx, double* ky, double* k2, double* filt);

/* Component callbacks (one call = one timestep callback of the component). */
int orc_vort2vel(orc_ctx*);
/* vort2vel.F90:139-320 alone: the inversion of the gridded vorticity (grids p, q, r). */
int orc_vort2vel_grids(orc_ctx*);
int orc_vorticity_tendency(orc_ctx*);
int orc_rk4_integrator(orc_ctx*);
int orc_parcel_splitting(orc_ctx*);
int orc_parcel_mixing(orc_ctx*);
/* One full model step: the integrator group executed rksteps (=4) times. */
int orc_step(orc_ctx*);
/* test components: euler_integrator.F90:53-86 and prescribed_parcel_velocity
 * (velocity.F90:59-255; profile 0 shear, 1-8 the compass directions N .. NW,
 * 9 cylindrical, 10 evacuate) */
int orc_euler_integrator(orc_ctx*);
int orc_prescribed_velocity(orc_ctx*, int profile);
int orc_prescribed_velocity_tag(orc_ctx*);
/* plume_parcelsetup initialisation (plume_parcelsetup.F90:58-334), one
 * process: prm = {lambda, H, z_c, mu, z_d, z_m, r_plume, e_values(1:3)};
 * replaces the parcels; *n_plume = the parcels of the plume (slots first). */
int orc_plume_setup(orc_ctx*, const double* prm, int64_t* n_plume);
/* basic_parcelsetup initialisation (basic_parcelsetup.F90:22-134), one
 * process: n_per_dir^3 parcels per cell on a regular sub-lattice, vol = 1. */
int orc_basic_setup(orc_ctx*, int n_per_dir);
/* The jittered thermal of the benchmark workloads (no counterpart in the
 * reference): prm = {sub, jitter, xc, yc, zc, radius, excess, h_in, h_env0,
 * z_strat, n2}; sub^3 parcels per cell jittered by U(+-jitter) sub-spacings
 * (Philox4x32-10 keyed by seed and parcel index), vol = cell volume / sub^3,
 * tag = parcel index, b and h of the thermal and its environment. */
int orc_thermal_setup(orc_ctx*, const double* prm, uint64_t seed);
/* The domain totals of vol, h*vol and b*vol over the parcels (the diagnostic
 * sums of parcel_mixing.F90:87-103, :409-418), compensated FP64. */
int orc_conserved_sums(const orc_ctx*, double* out3);

/* Component iteration counters (vort2vel, vorticity_tendency, rk4 stage,
 * splitting, mixing), for re-synchronising with another implementation. */
void orc_get_counters(const orc_ctx*, int* counters5);
void orc_set_counters(orc_ctx*, const int* counters5);
void orc_set_dtm(orc_ctx*, double dtm);

#ifdef __cplusplus
}
#endif
#endif
