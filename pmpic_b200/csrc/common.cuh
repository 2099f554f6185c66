// common.cuh -- shared definitions of the B200 PMPIC library (libpmpic_gpu.so).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pmpic_gpu.h"

#define PMPIC_CUDA(call)                                                     \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return pmpic::cuda_fail(ctx, e_, #call, __LINE__); \
  } while (0)

namespace pmpic {

// Fortran single-precision literals promoted to double (fft_ops.F90:427-429,
// :512-513, parcel_splitting.F90:71,79, vort2vel.F90:237-238).
// f4div(1.f, 6.f) is the REAL(4) quotient 1./6. widened to REAL(8).
__host__ __device__ constexpr double f4div(float a, float b) { return (double)(a / b); }
__host__ __device__ constexpr double f4(float a) { return (double)a; }

// Device error word values (sticky until read by pmpic_get_step_info).
enum { DEV_OK = 0 };

// Stockham FFT plan for one transform length (radix 4, 2, 3, 5 stages).
constexpr int FFT_MAX_STAGES = 16;
struct FftPlan {
  int n;
  int nst;
  int radix[FFT_MAX_STAGES];
  int tw_off[FFT_MAX_STAGES];  // offset (in double2) of each stage's twiddle table
  int n1, n2;                  // four-step split n = n1 * n2 (0: generic Stockham path)
  int tw4_off;                 // offset of the four-step twiddles W_n^(n2 k1), [n2 * n1 + k1]
};

// Geometry of one rank covering the whole domain (setup_grid.F90:45-104,
// parcel_interpolation.F90:76-136, haloswap.F90:296-318, :531-552).
struct Geom {
  int Nx, Ny, Nz, nzp;          // cells, and Nz+1 z points
  int sx, sy;                   // spectral extents Nx+2, Ny+2
  int64_t ncell;                // Nx*Ny*Nz
  int64_t nphys;                // (Nz+1)*Ny*Nx
  int64_t nspec;                // (Nz+1)*(Ny+2)*(Nx+2)
  double dx, dy, dz;
  double pxmin, pymin, pzmin;   // first halo point coordinate (-2dx, -2dy, 0)
  double pzmax;                 // Nz*dz (z reflection limit)
  double hxmin, hxmax, hymin, hymax;  // x_coords(3), x_coords(Nx+3), y likewise
  double xshift_e, xshift_w, yshift_n, yshift_s;
  double xc0, yc0, zc0;         // x_coords(1), y_coords(1), z_coords(1)
  double vmin;                  // dx*dy*dz/6/6/6 (parcel_mixing.F90:54)
  double rNz, rNy;              // 1/Nz, 1/Ny (cell id decoding)
};

// Cell ids are z fastest: id = (i*Ny + j)*Nz + k.  Decoding divides by Nz and
// Ny through the reciprocals (the product's quotient is exact or one off,
// corrected by the remainder's sign).
__device__ __forceinline__ void cell_decode(const Geom& g, int32_t id, int& i, int& j, int& k) {
  int t = __double2int_rz((double)id * g.rNz);
  int r = id - t * g.Nz;
  if (r < 0) { --t; r += g.Nz; } else if (r >= g.Nz) { ++t; r -= g.Nz; }
  k = r;
  int q = __double2int_rz((double)t * g.rNy);
  int s = t - q * g.Ny;
  if (s < 0) { --q; s += g.Ny; } else if (s >= g.Ny) { ++q; s -= g.Ny; }
  j = s;
  i = q;
}
__host__ __device__ __forceinline__ int32_t cell_encode(const Geom& g, int i, int j, int k) {
  return (int32_t)(((int64_t)i * g.Ny + j) * g.Nz + k);
}

// Interior cell id of a parcel and its fractional offsets, restating
// cache_parcel_interp_weights (parcel_interpolation.F90:214-237) bit for bit:
// i = floor((x-xmin)/dx)+1 and delx = ((x-xmin)-(i-1)dx)/dx with the halo
// origin xmin = -2dx; the interior cell is i-3 (x), j-3 (y), k-1 (z).
// A parcel one ulp below x = Lx is not wrapped by the parcel haloswap
// (x < x_coords(Nx+3)) yet bins to the halo cell i = Nx+3 with delx = 0; the
// reference then puts its weight on the halo point that par2grid_haloswap
// folds onto x = 0, which is interior cell 0 here.  Anything else outside the
// interior is an error (the reference aborts).
__device__ __forceinline__ bool bin_parcel(const Geom& g, double xp, double yp, double zp, int& ci, int& cj,
                                           int& ck, double& delx, double& dely, double& delz) {
  double fi = floor(__ddiv_rn(__dsub_rn(xp, g.pxmin), g.dx));
  double fj = floor(__ddiv_rn(__dsub_rn(yp, g.pymin), g.dy));
  double fk = floor(__ddiv_rn(__dsub_rn(zp, g.pzmin), g.dz));
  if (!(fi >= 2.0 && fi <= 2.0 + g.Nx && fj >= 2.0 && fj <= 2.0 + g.Ny && fk >= 0.0 && fk < (double)g.Nz))
    return false;
  int i = (int)fi + 1, j = (int)fj + 1, k = (int)fk + 1;
  delx = __ddiv_rn(__dsub_rn(__dsub_rn(xp, g.pxmin), __dmul_rn((double)(i - 1), g.dx)), g.dx);
  dely = __ddiv_rn(__dsub_rn(__dsub_rn(yp, g.pymin), __dmul_rn((double)(j - 1), g.dy)), g.dy);
  delz = __ddiv_rn(__dsub_rn(__dsub_rn(zp, g.pzmin), __dmul_rn((double)(k - 1), g.dz)), g.dz);
  if (delx > 1.0 || delx < 0.0 || dely > 1.0 || dely < 0.0 || delz > 1.0 || delz < 0.0) return false;
  ci = i - 3;
  cj = j - 3;
  ck = k - 1;
  if (ci == g.Nx) ci = 0;
  if (cj == g.Ny) cj = 0;
  return true;
}

// one integer atomic per distinct cell of the warp (neighbouring slots mostly
// share a cell): the per-cell histogram of the binning
__device__ __forceinline__ void count_cell(int32_t id, int32_t* __restrict__ count) {
  const unsigned act = __activemask();
  const unsigned same = __match_any_sync(act, id);
  if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&count[id], __popc(same));
}

// ---- mixed-precision form --------------------------------------------------
// Positions of the mixed form are an integer cell index plus an FP32 offset
// inside the cell in cell units, x = (i + f) * dx, so a parcel's absolute
// position never loses bits as it moves.  Three arrays carry them:
//  * the current position x, y, z (the reference's parcel x, y, z): the cell
//    id in ctx->cell (i, j, k packed z fastest; x and y wrapped into the
//    domain, z reflected at the walls) and the three offsets as FP32 in the
//    X, Y, Z property slots.  f lies in [0, 1); the one exception is f = 1 in
//    cell Nz-1, a parcel exactly on the top wall (the reference bins z = zmax
//    with delz = 1 in the last cell).  The cell id is at once the binning of
//    par2grid: the current cell is known wherever the position is.
//  * xo, yo, zo, the RK4 step's start (rk4_integrator.F90:125-127): a CellOff
//    {int32 index, FP32 offset} per axis in the 8-byte XO, YO, ZO slots, the
//    index unwrapped (the parcel haloswap shifts it by whole periods);
//  * xf, yf, zf as the FP32 displacement from xo in cell units (bounded by the
//    step's motion, dt |u| / dx) in the XF, YF, ZF slots.
struct __align__(8) CellOff {
  int32_t i;
  float f;
};
// a + d cell units, renormalised so that f is in [0, 1)
__device__ __forceinline__ CellOff co_add(CellOff a, float d) {
  const float t = a.f + d;
  const float fl = floorf(t);
  CellOff r;
  r.i = a.i + (int)fl;
  r.f = t - fl;
  if (r.f >= 1.0f) {  // t just below an integer, rounded up by the subtraction
    r.f -= 1.0f;
    r.i += 1;
  }
  return r;
}
// mirror of a z component at the walls z = 0 and z = nz (haloswap.F90:440-456)
__device__ __forceinline__ CellOff co_reflect(CellOff a, int nz) {
  if (a.i < 0) {  // -(i + f) = (-i - 1) + (1 - f)
    a.i = -a.i - 1;
    a.f = 1.0f - a.f;
  } else if (a.i > nz || (a.i == nz && a.f > 0.0f)) {  // 2 nz - (i + f)
    a.i = 2 * nz - a.i - 1;
    a.f = 1.0f - a.f;
  }
  if (a.f >= 1.0f) {
    a.f -= 1.0f;
    a.i += 1;
  }
  if (a.i == nz && a.f == 0.0f) {  // on the top wall: last cell, offset 1
    a.i = nz - 1;
    a.f = 1.0f;
  }
  return a;
}
// an index wrapped into [0, n) (one period at most away on the path; any
// integer here)
__device__ __forceinline__ int wrap_index(int i, int n) {
  if (i >= n) i -= n;
  else if (i < 0) i += n;
  if ((unsigned)i >= (unsigned)n) i = ((i % n) + n) % n;
  return i;
}
// the storage kinds of the properties on the mixed form
enum MixedKind {
  MK_F32 = 0,  // FP32 value in the first half of the allocation
  MK_CUR = 1,  // x, y, z: FP32 offset (with the cell id in ctx->cell)
  MK_BASE = 2, // xo, yo, zo: CellOff in the 8-byte slot
  MK_DISP = 3, // xf, yf, zf: FP32 displacement from xo in cell units
  MK_F64 = 4   // tag: FP64
};
__host__ __device__ __forceinline__ int mixed_kind(int pid) {
  switch (pid) {
    case PMPIC_PROP_X: case PMPIC_PROP_Y: case PMPIC_PROP_Z: return MK_CUR;
    case PMPIC_PROP_XO: case PMPIC_PROP_YO: case PMPIC_PROP_ZO: return MK_BASE;
    case PMPIC_PROP_XF: case PMPIC_PROP_YF: case PMPIC_PROP_ZF: return MK_DISP;
    case PMPIC_PROP_TAG: return MK_F64;
    default: return MK_F32;
  }
}
// whether a property is a position component on the mixed form
__host__ __device__ __forceinline__ bool mixed_is_pos(int pid) {
  const int k = mixed_kind(pid);
  return k == MK_CUR || k == MK_BASE || k == MK_DISP;
}
// element size of a property on the mixed form
__host__ __device__ __forceinline__ int mixed_elem_bytes(int pid) {
  const int k = mixed_kind(pid);
  return (k == MK_BASE || k == MK_F64) ? 8 : 4;
}
// an FP64 coordinate v as cell index + FP32 offset for cell size d (index not wrapped)
__device__ __forceinline__ CellOff co_from_double(double v, double d) {
  const double u = v / d;
  const double fl = floor(u);
  CellOff c;
  c.i = (int)fl;
  c.f = (float)(u - fl);
  if (c.f >= 1.0f) {
    c.f = 0.0f;
    c.i += 1;
  }
  return c;
}
// a current position from FP64 coordinates: x and y wrapped into the domain,
// z reflected at the walls (what the parcel haloswap does to a parcel outside);
// false if z lies beyond the reach of one reflection
__device__ __forceinline__ bool cur_from_double(const Geom& g, double x, double y, double z, int32_t& id, float& fx,
                                                float& fy, float& fz) {
  CellOff cx = co_from_double(x, g.dx), cy = co_from_double(y, g.dy), cz = co_from_double(z, g.dz);
  cx.i = wrap_index(cx.i, g.Nx);
  cy.i = wrap_index(cy.i, g.Ny);
  cz = co_reflect(cz, g.Nz);
  const bool ok = cz.i >= 0 && cz.i < g.Nz && cz.f >= 0.f && cz.f <= 1.f;
  if (!ok) cz = CellOff{0, 0.f};
  id = cell_encode(g, cx.i, cy.i, cz.i);
  fx = cx.f;
  fy = cy.f;
  fz = cz.f;
  return ok;
}

// Device-side step counters and error word.
struct DevInfo {
  int error;
  int pad;
  long long n_parcels;     // current numparcels (device copy)
  long long n_split;
  long long n_removed;
  long long n_added;
  long long n_migrated;
  long long n_zero;        // mixing: number of keep==0 slots
  long long n_kept;        // mixing: number of keep==1 slots
  double dtm;
  double umax2, vmax2, wmax2, omax2;  // squared maxima (order-free reductions)
  int limiter;
  int pad2;
  double sums[3];          // compensated totals of vol, h*vol, b*vol (conserved.cu)
};
// blocks of the first pass of the conserved sums (its partials buffer holds 6 doubles each)
constexpr int CS_BLOCKS = 148 * 4;

// Named timers, after the reference's timer_mod handles (e.g.
// parcel_interpolation.F90:144-148, pencilfft.F90:104-108, fft_ops.F90:157-160,
// rk4_integrator.F90:71-75), backed by CUDA events on the context's stream.
enum TimerId {
  T_CACHE = 0, T_P2G, T_G2P, T_FFTF, T_FFTI, T_DIFFZ, T_LAPLINV, T_V2V, T_VT, T_RK4, T_HSWP, T_SPLIT,
  T_MIX, T_STEP, T_RK4K, T_NT
};

}  // namespace pmpic

struct pmpic_ctx;
namespace pmpic {
struct TimerScope {
  pmpic_ctx* c;
  int id;
  int e0;
  TimerScope(pmpic_ctx* ctx, int id);
  ~TimerScope();
};
}  // namespace pmpic

// ---------------------------------------------------------------------------
// Context (host struct; device pointers inside)
// ---------------------------------------------------------------------------
struct pmpic_ctx {
  pmpic_config cfg;
  bool mixed;                // PMPIC_MIXED: FP32 bulk, int cell + FP32 offset positions
  int p2g_xseg;              // columns per x segment of the par2grid row pass (tunable)
  pmpic::Geom g;
  int device;
  cudaStream_t stream;
  std::string err;
  // parcels: NPROP arrays of capacity cap
  int64_t cap;
  int64_t n;                 // numparcels (host mirror, valid between calls)
  double* parcels;           // NPROP * cap
  int32_t* cell;             // cap: interior cell id per slot, z fastest: (i*Ny + j)*Nz + k
  double* del;               // 3 x cap: cached delx, dely, delz per slot
  bool sorted_valid;         // cell ids, offsets and cell lists match the current positions
  bool in_step;              // inside pmpic_step: no caller code runs between the callbacks
  bool split_follows;        // pmpic_step: a split that acts follows this RK4 stage
  bool stretch_advanced;     // mixed form: the last RK4 stage advanced the stretch property
                             // (parcel_splitting.F90:64-73) for the split that follows
  bool in_domain;            // every parcel is inside the domain (set by the parcel haloswap,
                             // cleared by any change of positions): a split moves only its own
  bool count_ready;          // mixed form: cell ids and per-cell counts were written by the
                             // last RK4 stage and haloswap, so binning starts at the scan
  bool btot_grid_ready;      // gspare holds par2grid(btot) of the current substep
  bool pending_uvw;          // vort2vel's grid2par of u, v, w not yet applied
  bool pending_pqr;          // vorticity_tendency's grid2par of dp, dq, dr not yet applied
  bool dir_ready;            // dir[] and the z reflection done for the current positions
  double* gspare;            // spare physical grid
  int32_t* sorted;           // cap: slot indices sorted by cell
  double* rowpart;           // par2grid row partials (rowpart_bytes)
  double* gpack;             // 6 x nphys: the RK4 gather grids packed z fastest (parcels.cu)
  double* lapcp;             // laplinv's Thomas factor tables (spectral.cu laplinv_tables;
                             // FP32 values on the mixed form)
  int32_t* cell_count;       // ncell + 1
  int32_t* cell_start;       // ncell + 1
  int32_t* cell_fill;        // ncell
  int32_t* keep;             // cap (mixing)
  int32_t* aux;              // cap (scans / migration lists)
  int32_t* aux2;             // 2*nbmax + cap (compaction block counts, offsets, lists)
  int64_t nbmax;             // max compaction blocks: ceil(max(cap, ncell)/1024) + 8
  int8_t* dir;               // cap (haloswap direction)
  double* swapbuf;           // staging for migrating parcels (29 doubles each)
  int64_t swapcap;
  void* scan_tmp;            // block sums for scans
  // physical grids (dense (Nz+1) x Ny x Nx)
  double* grid[PMPIC_NGRID];
  double* gwork[5];          // dudx, dwdx, dvdy, dwdy, ap
  double* mixres[6];         // residual grids vres..rres
  int32_t* npercell;         // ncell
  int32_t* newslot;          // ncell: slot of the new parcel of a cell or -1
  uint8_t* near;             // ncell (mixing): cell within one of a cell with a removed or a
                             // new parcel (its corners may hold residuals)
  int32_t* whint;            // cap/256 + 1: per RK4 CTA, where its gather window is staged: the
                             // cell its first parcel moved to at the last stage (mixed form), or
                             // the one the last binning found (FP64 path)
  double* newportion;        // ncell: portion of the new parcel of a cell
  // spectral arrays
  double* spec[PMPIC_NSPEC]; // u_s, v_s, w_s
  double* sa, *sb, *sc, *sd, *se, *sf, *sas, *sbs, *sscratch;
  double* fftmid;            // (Nz+1) x (Ny+2) x Nx
  double* ftw;               // twiddle tables (x plan first, then y plan), double2
  float* ftw32;              // the same twiddles as float2 (mixed-precision form)
  float* wn32;               // FP32 kx, ky, k2, filter tables and diffz factors
  double* hsum;              // FP64 horizontal sums of p and q per level (mixed form's zero mode)
  double* stage64;           // mixed form: FP64 staging of host transfers (stage_n values, two halves)
  int64_t stage_n;
  cudaStream_t xstream;      // mixed form: the host copies of the staged transfers
  cudaEvent_t xfull[2];      // a staging half holds its chunk (its producer is done)
  cudaEvent_t xfree[2];      // a staging half has been read (its consumer is done)
  int ftw_off_x, ftw_off_y;
  pmpic::FftPlan plan_x, plan_y;
  // small per-column data
  double* kx, *ky, *k2, *filt;  // (Ny+2) x (Nx+2)
  double* bt;                // atop, abot, btop, bbot: 4 x (Ny+2)(Nx+2)
  double* zmode;             // ubar, vbar: 2 x (Nz+1)
  double* csum;              // 6 x CS_BLOCKS: partials of the conserved sums
  // info
  pmpic::DevInfo* dinfo;     // device
  pmpic::DevInfo* hinfo;     // pinned host
  int counters[5];           // it_v2v, it_vt, rkstep, it_split, it_mix
  double dtm;
  pmpic_step_info info;
  // instrumentation
  int64_t nlaunch;           // kernels launched by this context
  bool timing;               // named timers enabled
  std::vector<cudaEvent_t> evpool;
  std::vector<int> evfree;
  std::vector<std::pair<int, int>> pending[pmpic::T_NT];
  double tms[pmpic::T_NT];
  int64_t tcalls[pmpic::T_NT];
  cudaEvent_t marks[8];      // pmpic_event_record slots
};

namespace pmpic {
int cuda_fail(pmpic_ctx* ctx, cudaError_t e, const char* what, int line);
int set_error(pmpic_ctx* ctx, int code, const std::string& msg);
inline double* prop(pmpic_ctx* ctx, int p) { return ctx->parcels + (size_t)p * (size_t)ctx->cap; }
// the mixed form's views of the same property arrays
inline float* propf(pmpic_ctx* ctx, int p) { return (float*)prop(ctx, p); }
inline CellOff* propc(pmpic_ctx* ctx, int p) { return (CellOff*)prop(ctx, p); }
// the mixed form's current position: cell ids, and the offsets of one axis
inline float* curoff(pmpic_ctx* ctx, int axis) { return propf(ctx, PMPIC_PROP_X + axis); }

// kernels / launchers (interp.cu)
int bin_and_sort(pmpic_ctx* ctx);
int par2grid_multi(pmpic_ctx* ctx, const double* const* fields, int nf, double* const* out, bool btot_from_bhz);
int grid2par_multi(pmpic_ctx* ctx, const double* const* grids, int ng, double* const* out);
int par2grid_multi_m(pmpic_ctx* ctx, const float* const* fields, int nf, float* const* out, bool btot_from_bhz = false);
int grid2par_multi_m(pmpic_ctx* ctx, const float* const* grids, int ng, float* const* out);
int cell_ids(pmpic_ctx* ctx, int32_t* dcells);
size_t rowpart_bytes(const Geom& g);
// host FP64 <-> property pid of slots off..off+n-1 (NULL src: zeros), in the
// context's precision, stream-ordered (ctx.cu)
int prop_upload(pmpic_ctx* ctx, int pid, int64_t off, int64_t n, const double* src);
int prop_download(pmpic_ctx* ctx, int pid, int64_t off, int64_t n, double* dst);
// fft.cu
// Elementwise operators fused into an inverse transform: one on its spectral
// input, applied as the first (x) pass reads it, and one on its physical
// output, applied as the last (y) pass writes it.  Each repeats the arithmetic
// of the separate operator kernel it replaces (same operands, same order), so
// fused and unfused sequences give the same bits.
enum SpecOpKind {
  SPEC_PLAIN = 0,
  SPEC_DX,    // diffx (fft_ops.F90:266-295) of the input, tab = kx
  SPEC_DY,    // diffy (fft_ops.F90:366-394) of the input, tab = ky
  SPEC_FILT,  // the de-aliasing filter (fft_ops.F90:176-197), tab = filt
  SPEC_VEL    // a velocity spectrum of vort2vel.F90:254-315 (see k_vel), no input array
};
template <class R>
struct SpecIn {
  int op = SPEC_PLAIN;
  const R* tab = nullptr;
  // SPEC_VEL: component vmode (0 u, 1 v, 2 w) from e, c (u, v) or a, b (w);
  // its filtered copy is stored to fs; zbar is the mean flow of u or v
  int vmode = 0;
  const R *e = nullptr, *c = nullptr, *a = nullptr, *b = nullptr;
  const R *kx = nullptr, *ky = nullptr, *filt = nullptr;
  R* fs = nullptr;
  const double* zbar = nullptr;
};
enum PhysOpKind {
  PHYS_STORE = 0,
  PHYS_ADD_MUL,      // o = o + in0 * v
  PHYS_ADD_MUL_SUM,  // o = o + in0 * (in1 + v)
  PHYS_NEG_ADD_MUL,  // o = -o + in0 * v
  PHYS_DQ_DR         // o = o + in0 * (-in1 + v); o2 = in1 in3 + in2 v + in0 (-in4) + in0 (-in5)
};
template <class R>
struct PhysOut {
  int op = PHYS_STORE;
  int store = 1;  // the transformed field itself is stored too
  R* o = nullptr;
  R* o2 = nullptr;
  const R* in[6] = {};
};
int fft_init(pmpic_ctx* ctx);
int fft_forward(pmpic_ctx* ctx, const double* phys, double* spec);
int fft_backward(pmpic_ctx* ctx, const double* spec, double* phys);
int fft_forward(pmpic_ctx* ctx, const float* phys, float* spec);
int fft_backward(pmpic_ctx* ctx, const float* spec, float* phys);
int fft_backward(pmpic_ctx* ctx, const double* spec, double* phys, const SpecIn<double>& si,
                 const PhysOut<double>& po);
int fft_backward(pmpic_ctx* ctx, const float* spec, float* phys, const SpecIn<float>& si,
                 const PhysOut<float>& po);
// spectral.cu
int spec_diffx(pmpic_ctx* ctx, const double* in, double* out);
int spec_diffy(pmpic_ctx* ctx, const double* in, double* out);
int spec_filter(pmpic_ctx* ctx, const double* in, double* out);
int spec_diffz(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top);
int spec_laplinv(pmpic_ctx* ctx, double* inout, bool df0);
int vort2vel_spectral(pmpic_ctx* ctx);
int vorticity_tendency_grids(pmpic_ctx* ctx);
int field_max(pmpic_ctx* ctx, bool first_substep_v2v, bool first_substep_vt);
// parcels.cu
int rk4_stage(pmpic_ctx* ctx, int stage);
int parcel_haloswap(pmpic_ctx* ctx);
int splitting(pmpic_ctx* ctx);
int mixing(pmpic_ctx* ctx);
int compute_btot(pmpic_ctx* ctx);
int euler_step(pmpic_ctx* ctx);
int prescribed_velocity(pmpic_ctx* ctx, int profile, bool tags);
int setup_plume(pmpic_ctx* ctx, const pmpic_plume_params* prm, int64_t* n_plume);
int setup_thermal_device(pmpic_ctx* ctx, const pmpic_thermal_params* prm);
int setup_basic(pmpic_ctx* ctx, int n_per_dir);
int flush_gathers(pmpic_ctx* ctx);
int sync_info(pmpic_ctx* ctx);
// conserved.cu: the compensated totals of vol, h*vol, b*vol into dinfo->sums
int conserved_sums(pmpic_ctx* ctx);
}  // namespace pmpic
