// ctx.cu -- the C ABI of libpmpic_gpu.so (include/pmpic_gpu.h): context
// set-up, transfers, and the five component timestep callbacks of the
// reference's integrator group.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace pmpic {

int spectral_init(pmpic_ctx* ctx);
int scan_excl(pmpic_ctx* ctx, const int32_t* in, int64_t n, int32_t* out);

int cuda_fail(pmpic_ctx* ctx, cudaError_t e, const char* what, int line) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "CUDA error %s at ctx.cu/%d: %s", cudaGetErrorString(e), line, what);
  if (ctx) ctx->err = buf;
  return PMPIC_ERR_CUDA;
}

int set_error(pmpic_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

static const char* err_text(int code) {
  switch (code) {
    case PMPIC_ERR_CAPACITY: return "maximum parcel count reached";
    case PMPIC_ERR_OUT_OF_BOX: return "parcel out of box";
    case PMPIC_ERR_ZERO_PIVOT: return "zero pivot in tridiagonal solver";
    case PMPIC_ERR_BACKFILL: return "mixing backfill ran out of kept parcels";
    case PMPIC_ERR_TIMEOUT: return "device wait timed out";
    default: return "device error";
  }
}

// Copy the device info block to the host; report a sticky device error.
int sync_info(pmpic_ctx* ctx) {
  PMPIC_CUDA(cudaMemcpyAsync(ctx->hinfo, ctx->dinfo, sizeof(DevInfo), cudaMemcpyDeviceToHost, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  const DevInfo& h = *ctx->hinfo;
  ctx->dtm = h.dtm;
  ctx->info.dtm = h.dtm;
  ctx->info.limiter = h.limiter;
  ctx->info.n_migrated = h.n_migrated;
  ctx->info.vol_sum = h.sums[0];
  ctx->info.hvol_sum = h.sums[1];
  ctx->info.bvol_sum = h.sums[2];
  ctx->info.n_parcels = ctx->n;
  if (h.error != 0) {
    ctx->info.error = h.error;
    return set_error(ctx, h.error, err_text(h.error));
  }
  return 0;
}

static const char* kTimerNames[T_NT] = {"cache_weights", "par2grid", "grid2par", "fft_fwd_tot",
                                        "fft_inv_tot",   "diffz",    "laplinv",  "vort2vel",
                                        "vort_tend",     "RK4_all_steps", "Par_HSWP_entire", "splitting",
                                        "mixing",        "step", "rk4_kernel"};

static int take_event(pmpic_ctx* c) {
  if (c->evfree.empty()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    c->evpool.push_back(e);
    return (int)c->evpool.size() - 1;
  }
  int i = c->evfree.back();
  c->evfree.pop_back();
  return i;
}

TimerScope::TimerScope(pmpic_ctx* ctx, int tid) : c(ctx), id(tid), e0(-1) {
  if (!c->timing) return;
  e0 = take_event(c);
  if (e0 >= 0) cudaEventRecord(c->evpool[e0], c->stream);
}
TimerScope::~TimerScope() {
  if (e0 < 0) return;
  int e1 = take_event(c);
  if (e1 < 0) return;
  cudaEventRecord(c->evpool[e1], c->stream);
  c->pending[id].push_back({e0, e1});
}

// fold recorded event pairs into the accumulated times
static void drain_timers(pmpic_ctx* c) {
  cudaStreamSynchronize(c->stream);
  for (int t = 0; t < T_NT; ++t) {
    for (auto& pr : c->pending[t]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->evpool[pr.first], c->evpool[pr.second]) == cudaSuccess) c->tms[t] += ms;
      c->tcalls[t] += 1;
      c->evfree.push_back(pr.first);
      c->evfree.push_back(pr.second);
    }
    c->pending[t].clear();
  }
}

}  // namespace pmpic

using namespace pmpic;

namespace {

template <class T>
int dalloc(pmpic_ctx* ctx, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc", __LINE__);
  return 0;
}

void free_all(pmpic_ctx* c) {
  void* ptrs[] = {c->parcels, c->rowpart,  c->gpack,    c->lapcp,    c->cell,     c->del,       c->gspare,     c->sorted,    c->cell_count, c->cell_start, c->cell_fill, c->keep,
                  c->aux,     c->aux2,     c->dir,       c->swapbuf,    c->scan_tmp,   c->npercell,  c->newslot,
                  c->newportion, c->sa,    c->sb,        c->sc,         c->sd,         c->se,        c->sf,
                  c->sas,     c->sbs,      c->sscratch,  c->fftmid,     c->ftw,        c->ftw32,      c->wn32,       c->hsum,       c->stage64,        c->kx,        c->ky,
                  c->k2,      c->filt,     c->bt,        c->zmode,      c->csum,       c->near,       c->whint,      c->dinfo};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < PMPIC_NGRID; ++i)
    if (c->grid[i]) cudaFree(c->grid[i]);
  for (int i = 0; i < 5; ++i)
    if (c->gwork[i]) cudaFree(c->gwork[i]);
  for (int i = 0; i < 6; ++i)
    if (c->mixres[i]) cudaFree(c->mixres[i]);
  for (int i = 0; i < PMPIC_NSPEC; ++i)
    if (c->spec[i]) cudaFree(c->spec[i]);
  if (c->hinfo) cudaFreeHost(c->hinfo);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  for (int i = 0; i < 8; ++i)
    if (c->marks[i]) cudaEventDestroy(c->marks[i]);
  for (int i = 0; i < 2; ++i) {
    if (c->xfull[i]) cudaEventDestroy(c->xfull[i]);
    if (c->xfree[i]) cudaEventDestroy(c->xfree[i]);
  }
  if (c->xstream) cudaStreamDestroy(c->xstream);
  if (c->stream) cudaStreamDestroy(c->stream);
}

bool smooth235(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  while (n % 5 == 0) n /= 5;
  return n == 1;
}

// wavenumbers and filter (fft_ops.F90:111-140) with the reference's arithmetic
void wavenumbers(const pmpic_config& cfg, const Geom& g, std::vector<double>& kx, std::vector<double>& ky,
                 std::vector<double>& k2, std::vector<double>& filt) {
  const int sx = g.sx, sy = g.sy;
  double lx = g.dx * (double)g.Nx, ly = g.dy * (double)g.Ny;
  const double kxm = (double)((float)g.Nx / 2.0f) / lx, kym = (double)((float)g.Ny / 2.0f) / ly;
  double ksqmax = kxm * kxm + kym * kym;
  ksqmax = ksqmax * 2.0 / 9.0;
  const double twopi = 8.0 * std::atan(1.0);
  kx.resize((size_t)sx * sy); ky.resize(kx.size()); k2.resize(kx.size()); filt.resize(kx.size());
  for (int jp = 0; jp < sy; ++jp)
    for (int ip = 0; ip < sx; ++ip) {
      double xval = (double)(ip / 2) / lx;
      double yval = (double)(jp / 2) / ly;
      size_t o = (size_t)jp * sx + ip;
      double kk = xval * xval + yval * yval;
      filt[o] = (kk > ksqmax) ? 0.0 : 1.0;
      kx[o] = xval * twopi;
      ky[o] = yval * twopi;
      k2[o] = kk * twopi * twopi;
    }
  (void)cfg;
}

}  // namespace

extern "C" {

int pmpic_create(const pmpic_config* cfg, pmpic_ctx** out) {
  if (!cfg || !out) return PMPIC_ERR_ARG;
  *out = nullptr;
  if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 3 || (cfg->nx & 1) || (cfg->ny & 1) || !smooth235(cfg->nx) ||
      !smooth235(cfg->ny) || cfg->max_parcels <= 0 || cfg->max_parcels >= (int64_t)0x7fffffff ||
      (cfg->precision != PMPIC_FP64 && cfg->precision != PMPIC_MIXED))
    return PMPIC_ERR_CONFIG;
  // cell ids and grid offsets are 32-bit: the largest grid, the spectral one, must fit
  if ((int64_t)(cfg->nz + 1) * (cfg->ny + 2) * (cfg->nx + 2) >= (int64_t)0x7fffffff) return PMPIC_ERR_CONFIG;
  if (cfg->xmin != 0.0 || cfg->ymin != 0.0 || cfg->zmin != 0.0 || !(cfg->xmax > 0) || !(cfg->ymax > 0) ||
      !(cfg->zmax > 0))
    return PMPIC_ERR_CONFIG;
  pmpic_ctx* ctx = new pmpic_ctx();
  std::memset((void*)&ctx->g, 0, sizeof(ctx->g));
  ctx->cfg = *cfg;
  ctx->mixed = cfg->precision == PMPIC_MIXED;
  ctx->p2g_xseg = 64;
  ctx->device = cfg->device;
  ctx->parcels = nullptr;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
    delete ctx;
    return PMPIC_ERR_CUDA;
  }
  // geometry (setup_grid.F90:73-95; parcel_interpolation.F90:104-136)
  Geom& g = ctx->g;
  g.Nx = cfg->nx; g.Ny = cfg->ny; g.Nz = cfg->nz; g.nzp = cfg->nz + 1;
  g.sx = g.Nx + 2; g.sy = g.Ny + 2;
  g.ncell = (int64_t)g.Nx * g.Ny * g.Nz;
  g.nphys = (int64_t)g.nzp * g.Ny * g.Nx;
  g.nspec = (int64_t)g.nzp * g.sy * g.sx;
  g.dx = (cfg->xmax - cfg->xmin) / (double)g.Nx;
  g.dy = (cfg->ymax - cfg->ymin) / (double)g.Ny;
  g.dz = (cfg->zmax - cfg->zmin) / (double)(g.nzp - 1);
  g.pxmin = (double)(-2) * g.dx + cfg->xmin;
  g.pymin = (double)(-2) * g.dy + cfg->ymin;
  g.pzmin = 0.0 * g.dz + cfg->zmin;
  g.pzmax = (double)(g.nzp - 1) * g.dz;
  g.xc0 = g.pxmin; g.yc0 = g.pymin; g.zc0 = g.pzmin;
  g.hxmin = g.pxmin + 2.0 * g.dx;                   // x_coords(hx+1)
  g.hxmax = g.pxmin + (double)(g.Nx + 2) * g.dx;    // x_coords(nx-hx+1)
  g.hymin = g.pymin + 2.0 * g.dy;
  g.hymax = g.pymin + (double)(g.Ny + 2) * g.dy;
  const double topx = cfg->xmax - g.dx, topy = cfg->ymax - g.dy;  // setup_grid.F90:92-93
  g.xshift_e = cfg->xmin - topx - g.dx;             // haloswap.F90:531-535
  g.xshift_w = topx - cfg->xmin + g.dx;             // :536-540
  g.yshift_n = cfg->ymin - topy - g.dy;             // :542-546
  g.yshift_s = topy - cfg->ymin + g.dy;             // :547-551
  g.vmin = g.dx * g.dy * g.dz / 6. / 6. / 6.;       // parcel_mixing.F90:54
  g.rNz = 1.0 / (double)g.Nz;
  g.rNy = 1.0 / (double)g.Ny;
  ctx->cap = cfg->max_parcels;
  ctx->n = 0;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->pending_uvw = ctx->pending_pqr = ctx->dir_ready = false;
  ctx->split_follows = ctx->stretch_advanced = ctx->in_step = false;
  ctx->nbmax = (std::max<int64_t>(ctx->cap, g.ncell) + 1023) / 1024 + 8;
  int64_t sc = 2LL * (g.Nx + g.Ny) * (int64_t)g.nzp * 32;
  ctx->swapcap = std::min<int64_t>(ctx->cap, std::max<int64_t>(1 << 20, sc));
  int rc = 0;
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) rc = cuda_fail(ctx, e, "stream", __LINE__);
  const size_t cap = (size_t)ctx->cap;
  if (!rc) rc = dalloc(ctx, &ctx->parcels, (size_t)PMPIC_NPROP * cap);
  if (!rc) rc = dalloc(ctx, &ctx->cell, cap);
  if (!rc && !ctx->mixed) rc = dalloc(ctx, &ctx->del, 3 * cap);  // the mixed form's offsets live in its positions
  if (!rc) rc = dalloc(ctx, &ctx->gspare, (size_t)g.nphys);
  if (!rc) rc = dalloc(ctx, &ctx->sorted, cap);
  if (!rc) rc = dalloc(ctx, (char**)&ctx->rowpart, rowpart_bytes(g));
  if (!rc) rc = dalloc(ctx, &ctx->gpack, 6 * (size_t)g.nphys);  // the six RK4 gather grids
  ctx->stage_n = std::min<int64_t>(ctx->cap, (int64_t)1 << 24);
  if (!rc && ctx->mixed) rc = dalloc(ctx, &ctx->stage64, (size_t)ctx->stage_n);
  if (!rc && ctx->mixed) {  // the staged transfers' copy stream: copies overlap the conversions
    e = cudaStreamCreateWithFlags(&ctx->xstream, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
      e = cudaEventCreateWithFlags(&ctx->xfull[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->xfree[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "copy stream", __LINE__);
  }
  if (!rc) rc = dalloc(ctx, &ctx->keep, cap);
  if (!rc) rc = dalloc(ctx, &ctx->aux, cap);
  if (!rc) rc = dalloc(ctx, &ctx->aux2, 2 * (size_t)ctx->nbmax + cap);
  if (!rc) rc = dalloc(ctx, &ctx->dir, cap);
  if (!rc) rc = dalloc(ctx, &ctx->cell_count, (size_t)g.ncell + 1);
  if (!rc) rc = dalloc(ctx, &ctx->cell_start, (size_t)g.ncell + 1);
  if (!rc) rc = dalloc(ctx, &ctx->cell_fill, (size_t)g.ncell);
  if (!rc) rc = dalloc(ctx, &ctx->swapbuf, (size_t)ctx->swapcap * 30);  // 29 properties (+ the mixed form's cell id)
  if (!rc) rc = dalloc(ctx, (int32_t**)&ctx->scan_tmp, (size_t)(std::max<int64_t>(std::max<int64_t>(g.ncell, ctx->cap), ctx->nbmax) / 4096 + 64));
  for (int i = 0; i < PMPIC_NGRID && !rc; ++i) rc = dalloc(ctx, &ctx->grid[i], (size_t)g.nphys);
  for (int i = 0; i < 5 && !rc; ++i) rc = dalloc(ctx, &ctx->gwork[i], (size_t)g.nphys);
  for (int i = 0; i < 6 && !rc; ++i) rc = dalloc(ctx, &ctx->mixres[i], (size_t)g.nphys);
  if (!rc) rc = dalloc(ctx, &ctx->npercell, (size_t)g.ncell);
  if (!rc) rc = dalloc(ctx, &ctx->newslot, (size_t)g.ncell);
  if (!rc) rc = dalloc(ctx, &ctx->near, (size_t)g.ncell);
  if (!rc) rc = dalloc(ctx, &ctx->whint, (size_t)cap / 256 + 1);
  if (!rc) rc = dalloc(ctx, &ctx->newportion, (size_t)g.ncell);
  for (int i = 0; i < PMPIC_NSPEC && !rc; ++i) rc = dalloc(ctx, &ctx->spec[i], (size_t)g.nspec);
  double** sp[] = {&ctx->sa, &ctx->sb, &ctx->sc, &ctx->sd, &ctx->se, &ctx->sf, &ctx->sas, &ctx->sbs};
  for (double** p : sp)
    if (!rc) rc = dalloc(ctx, p, (size_t)g.nspec);
  if (!rc) rc = dalloc(ctx, &ctx->sscratch, (size_t)g.nspec + 6 * (size_t)g.nzp);
  if (!rc) rc = dalloc(ctx, &ctx->fftmid, (size_t)g.nzp * g.sy * g.Nx);
  const size_t cols = (size_t)g.sx * g.sy;
  if (!rc) rc = dalloc(ctx, &ctx->kx, cols);
  if (!rc) rc = dalloc(ctx, &ctx->ky, cols);
  if (!rc) rc = dalloc(ctx, &ctx->k2, cols);
  if (!rc) rc = dalloc(ctx, &ctx->filt, cols);
  if (!rc) rc = dalloc(ctx, &ctx->bt, 4 * cols);
  if (!rc) rc = dalloc(ctx, &ctx->zmode, 2 * (size_t)g.nzp);
  if (!rc) rc = dalloc(ctx, &ctx->csum, 6 * (size_t)CS_BLOCKS);
  if (!rc) rc = dalloc(ctx, (char**)&ctx->dinfo, sizeof(DevInfo) + 64 * sizeof(int32_t));
  if (!rc) {
    e = cudaMallocHost((void**)&ctx->hinfo, sizeof(DevInfo));
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMallocHost", __LINE__);
  }
  if (!rc) {
    // zero-initialised state: every slot of every property starts at 0
    e = cudaMemset(ctx->parcels, 0, sizeof(double) * (size_t)PMPIC_NPROP * cap);
    if (e == cudaSuccess) e = cudaMemset(ctx->dinfo, 0, sizeof(DevInfo) + 64 * sizeof(int32_t));
    for (int i = 0; i < PMPIC_NGRID && e == cudaSuccess; ++i) e = cudaMemset(ctx->grid[i], 0, sizeof(double) * g.nphys);
    if (e == cudaSuccess && ctx->whint) e = cudaMemset(ctx->whint, 0, sizeof(int32_t) * ((size_t)cap / 256 + 1));
    for (int i = 0; i < PMPIC_NSPEC && e == cudaSuccess; ++i) e = cudaMemset(ctx->spec[i], 0, sizeof(double) * g.nspec);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemset", __LINE__);
  }
  if (!rc) {
    std::vector<double> kx, ky, k2, filt;
    wavenumbers(*cfg, g, kx, ky, k2, filt);
    cudaMemcpy(ctx->kx, kx.data(), sizeof(double) * cols, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->ky, ky.data(), sizeof(double) * cols, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->k2, k2.data(), sizeof(double) * cols, cudaMemcpyHostToDevice);
    e = cudaMemcpy(ctx->filt, filt.data(), sizeof(double) * cols, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "wavenumbers", __LINE__);
  }
  if (!rc) rc = fft_init(ctx);
  if (!rc) rc = spectral_init(ctx);
  if (!rc) {
    DevInfo h{};
    h.dtm = cfg->dtm;  // rk4_integrator.F90:38-41
    e = cudaMemcpy(ctx->dinfo, &h, sizeof(DevInfo), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "dinfo", __LINE__);
  }
  for (int i = 0; i < 8 && !rc; ++i) {
    e = cudaEventCreate(&ctx->marks[i]);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaEventCreate", __LINE__);
  }
  ctx->dtm = cfg->dtm;
  ctx->counters[0] = 0; ctx->counters[1] = 0; ctx->counters[2] = 1; ctx->counters[3] = 0; ctx->counters[4] = 0;
  std::memset(&ctx->info, 0, sizeof(ctx->info));
  ctx->info.dtm = cfg->dtm;
  if (rc) {
    free_all(ctx);
    delete ctx;
    return rc;
  }
  *out = ctx;
  return PMPIC_OK;
}

void pmpic_destroy(pmpic_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
}

const char* pmpic_last_error(const pmpic_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// ---- the mixed form's property and grid conversions ---------------------------------
namespace {
// Host FP64 values into one property of the mixed form (kinds of mixed_kind):
// FP32 values; the tag as FP64; xo as {index, offset}; xf as the displacement
// from the slot's xo; a current position component as the offset, with the
// axis's index written into the slot's cell id (x, y wrapped into the domain,
// z reflected at the walls, as the parcel haloswap would; a z beyond one
// reflection is reported out of box).
struct ConvIn {
  int kind, axis;
  double d;             // cell size along the axis
  const CellOff* base;  // MK_DISP: the axis's xo
  int32_t* cell;        // MK_CUR: the cell ids
  DevInfo* info;
};
__global__ void k_conv_in(Geom g, int64_t n, const double* __restrict__ src, void* __restrict__ dst, ConvIn c) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double v = src ? src[t] : 0.0;
  switch (c.kind) {
    case MK_F32: ((float*)dst)[t] = (float)v; break;
    case MK_F64: ((double*)dst)[t] = v; break;
    case MK_BASE: ((CellOff*)dst)[t] = co_from_double(v, c.d); break;
    case MK_DISP: {
      const CellOff b = c.base[t];
      ((float*)dst)[t] = (float)(v / c.d - ((double)b.i + (double)b.f));
      break;
    }
    default: {  // MK_CUR
      int ijk[3] = {0, 0, 0};
      const int32_t id = c.cell[t];
      if (id >= 0 && id < g.ncell) cell_decode(g, id, ijk[0], ijk[1], ijk[2]);
      CellOff a = co_from_double(v, c.d);
      if (c.axis == 0) a.i = wrap_index(a.i, g.Nx);
      else if (c.axis == 1) a.i = wrap_index(a.i, g.Ny);
      else {
        a = co_reflect(a, g.Nz);
        if (!(a.i >= 0 && a.i < g.Nz && a.f >= 0.f && a.f <= 1.f)) {
          atomicCAS(&c.info->error, 0, PMPIC_ERR_OUT_OF_BOX);
          a = CellOff{0, 0.f};
        }
      }
      ijk[c.axis] = a.i;
      c.cell[t] = cell_encode(g, ijk[0], ijk[1], ijk[2]);
      ((float*)dst)[t] = a.f;
    }
  }
}
struct ConvOut {
  int kind, axis;
  double d;
  const CellOff* base;   // MK_DISP
  const int32_t* cell;   // MK_CUR
};
__global__ void k_conv_out(Geom g, int64_t n, const void* __restrict__ src, double* __restrict__ dst, ConvOut c) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  switch (c.kind) {
    case MK_F32: dst[t] = (double)((const float*)src)[t]; break;
    case MK_F64: dst[t] = ((const double*)src)[t]; break;
    case MK_BASE: {
      const CellOff b = ((const CellOff*)src)[t];
      dst[t] = ((double)b.i + (double)b.f) * c.d;
      break;
    }
    case MK_DISP: {
      const CellOff b = c.base[t];
      dst[t] = ((double)b.i + (double)b.f + (double)((const float*)src)[t]) * c.d;
      break;
    }
    default: {  // MK_CUR
      int ijk[3] = {0, 0, 0};
      cell_decode(g, c.cell[t], ijk[0], ijk[1], ijk[2]);
      dst[t] = ((double)ijk[c.axis] + (double)((const float*)src)[t]) * c.d;
    }
  }
}
__global__ void k_f2d(int64_t n, const float* __restrict__ src, double* __restrict__ dst) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (double)src[t];
}
__global__ void k_d2f(int64_t n, const double* __restrict__ src, float* __restrict__ dst) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (float)src[t];
}
unsigned cblk(int64_t n) { return (unsigned)((n + 255) / 256); }

int axis_of(int pid) {
  if (pid == PMPIC_PROP_X || pid == PMPIC_PROP_XO || pid == PMPIC_PROP_XF) return 0;
  if (pid == PMPIC_PROP_Y || pid == PMPIC_PROP_YO || pid == PMPIC_PROP_YF) return 1;
  return 2;
}
double cell_size(const Geom& g, int axis) { return axis == 0 ? g.dx : (axis == 1 ? g.dy : g.dz); }
}  // namespace

// host FP64 values (NULL: zeros) into property pid of slots off..off+n-1, in
// the context's precision; stream-ordered
}  // extern "C"

int pmpic::prop_upload(pmpic_ctx* ctx, int pid, int64_t off, int64_t n, const double* src) {
  if (n <= 0) return 0;
  if (!ctx->mixed) {
    if (src) PMPIC_CUDA(cudaMemcpyAsync(prop(ctx, pid) + off, src, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    else PMPIC_CUDA(cudaMemsetAsync(prop(ctx, pid) + off, 0, sizeof(double) * n, ctx->stream));
    return 0;
  }
  const size_t es = (size_t)mixed_elem_bytes(pid);
  const int kind = mixed_kind(pid);
  if (!src && (kind == MK_F32 || kind == MK_F64 || kind == MK_BASE)) {
    PMPIC_CUDA(cudaMemsetAsync((char*)prop(ctx, pid) + es * off, 0, es * n, ctx->stream));
    return 0;
  }
  ConvIn c;
  c.kind = kind;
  c.axis = axis_of(pid);
  c.d = cell_size(ctx->g, c.axis);
  c.info = ctx->dinfo;
  char* base = (char*)prop(ctx, pid) + es * off;
  // chunks alternate between the staging halves: the copy stream fills one
  // while the context's stream converts the other
  const int64_t h = std::max<int64_t>(ctx->stage_n / 2, 1);
  for (int64_t c0 = 0, i = 0; c0 < n; c0 += h, ++i) {
    const int64_t len = std::min<int64_t>(h, n - c0);
    double* buf = ctx->stage64 + (i & 1) * h;
    c.base = propc(ctx, PMPIC_PROP_XO + c.axis) + off + c0;
    c.cell = ctx->cell + off + c0;
    if (src) {
      PMPIC_CUDA(cudaStreamWaitEvent(ctx->xstream, ctx->xfree[i & 1], 0));  // its last conversion is done
      PMPIC_CUDA(cudaMemcpyAsync(buf, src + c0, sizeof(double) * len, cudaMemcpyHostToDevice, ctx->xstream));
      PMPIC_CUDA(cudaEventRecord(ctx->xfull[i & 1], ctx->xstream));
      PMPIC_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->xfull[i & 1], 0));
    }
    k_conv_in<<<cblk(len), 256, 0, ctx->stream>>>(ctx->g, len, src ? buf : nullptr, base + es * c0, c);
    ++ctx->nlaunch;
    if (src) PMPIC_CUDA(cudaEventRecord(ctx->xfree[i & 1], ctx->stream));
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
// property pid of slots off..off+n-1 into host FP64 values; stream-ordered
int pmpic::prop_download(pmpic_ctx* ctx, int pid, int64_t off, int64_t n, double* dst) {
  if (n <= 0) return 0;
  if (!ctx->mixed) {
    PMPIC_CUDA(cudaMemcpyAsync(dst, prop(ctx, pid) + off, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    return 0;
  }
  const size_t es = (size_t)mixed_elem_bytes(pid);
  ConvOut c;
  c.kind = mixed_kind(pid);
  c.axis = axis_of(pid);
  c.d = cell_size(ctx->g, c.axis);
  const char* base = (const char*)prop(ctx, pid) + es * off;
  // chunks alternate between the staging halves: the context's stream
  // converts one while the copy stream empties the other
  const int64_t h = std::max<int64_t>(ctx->stage_n / 2, 1);
  for (int64_t c0 = 0, i = 0; c0 < n; c0 += h, ++i) {
    const int64_t len = std::min<int64_t>(h, n - c0);
    double* buf = ctx->stage64 + (i & 1) * h;
    c.base = propc(ctx, PMPIC_PROP_XO + c.axis) + off + c0;
    c.cell = ctx->cell + off + c0;
    PMPIC_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->xfree[i & 1], 0));  // its last copy is done
    k_conv_out<<<cblk(len), 256, 0, ctx->stream>>>(ctx->g, len, base + es * c0, buf, c);
    ++ctx->nlaunch;
    PMPIC_CUDA(cudaEventRecord(ctx->xfull[i & 1], ctx->stream));
    PMPIC_CUDA(cudaStreamWaitEvent(ctx->xstream, ctx->xfull[i & 1], 0));
    PMPIC_CUDA(cudaMemcpyAsync(dst + c0, buf, sizeof(double) * len, cudaMemcpyDeviceToHost, ctx->xstream));
    PMPIC_CUDA(cudaEventRecord(ctx->xfree[i & 1], ctx->xstream));
  }
  // the context's stream waits for the copies, so a caller synchronizing it finds the values on the host
  for (int i = 0; i < 2; ++i) PMPIC_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->xfree[i], 0));
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

extern "C" {

static int put_prop(pmpic_ctx* ctx, int pid, int64_t n, const double* src) {
  return prop_upload(ctx, pid, 0, n, src);
}
static int get_prop(pmpic_ctx* ctx, int pid, int64_t n, double* dst) { return prop_download(ctx, pid, 0, n, dst); }

int pmpic_set_count(pmpic_ctx* ctx, int64_t n) {
  if (!ctx) return PMPIC_ERR_ARG;
  if (n < 0 || n > ctx->cap) return set_error(ctx, PMPIC_ERR_CAPACITY, "parcel count exceeds max_parcels");
  cudaSetDevice(ctx->device);
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  ctx->n = n;
  ctx->info.n_parcels = n;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->dir_ready = false;
  return PMPIC_OK;
}
int pmpic_get_count(pmpic_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return PMPIC_ERR_ARG;
  *n = ctx->n;
  return PMPIC_OK;
}

int pmpic_set_property(pmpic_ctx* ctx, int p, int64_t n, const double* src) {
  if (!ctx || p < 0 || p >= PMPIC_NPROP || n < 0 || n > ctx->cap || (!src && n > 0)) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  ctx->dir_ready = false;
  int rc = put_prop(ctx, p, n, src);
  if (rc) return rc;
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  return PMPIC_OK;
}
int pmpic_get_property(pmpic_ctx* ctx, int p, int64_t n, double* dst) {
  if (!ctx || p < 0 || p >= PMPIC_NPROP || n < 0 || n > ctx->cap || (!dst && n > 0)) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  int rc = get_prop(ctx, p, n, dst);
  if (rc) return rc;
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return PMPIC_OK;
}

static const int kIO[11] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P,       PMPIC_PROP_Q,  PMPIC_PROP_R,
                            PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_VOL, PMPIC_PROP_STRETCH, PMPIC_PROP_TAG};

int pmpic_upload_parcels(pmpic_ctx* ctx, int64_t n, const double* x, const double* y, const double* z,
                         const double* p, const double* q, const double* r, const double* b, const double* h,
                         const double* vol, const double* stretch, const double* tag) {
  if (!ctx) return PMPIC_ERR_ARG;
  if (n < 0 || n > ctx->cap) return set_error(ctx, PMPIC_ERR_CAPACITY, "parcel count exceeds max_parcels");
  const double* src[11] = {x, y, z, p, q, r, b, h, vol, stretch, tag};
  cudaSetDevice(ctx->device);
  ctx->pending_uvw = ctx->pending_pqr = false;  // a new state
  ctx->dir_ready = false;
  for (int i = 0; i < 11; ++i) {
    int rc = put_prop(ctx, kIO[i], n, src[i]);
    if (rc) return rc;
  }
  const int zero[] = {PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT,
                      PMPIC_PROP_DRDT, PMPIC_PROP_BTOT, PMPIC_PROP_XO,   PMPIC_PROP_YO,   PMPIC_PROP_ZO,
                      PMPIC_PROP_XF,   PMPIC_PROP_YF,   PMPIC_PROP_ZF,   PMPIC_PROP_PO,   PMPIC_PROP_QO,
                      PMPIC_PROP_RO,   PMPIC_PROP_PF,   PMPIC_PROP_QF,   PMPIC_PROP_RF};
  for (int pid : zero) {
    int rc = put_prop(ctx, pid, n, nullptr);
    if (rc) return rc;
  }
  // a new state clears the sticky device error word
  PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->error, 0, sizeof(int), ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->n = n;
  ctx->info.n_parcels = n;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  return PMPIC_OK;
}

int pmpic_download_parcels(pmpic_ctx* ctx, int64_t capacity, int64_t* n, double* x, double* y, double* z, double* p,
                           double* q, double* r, double* b, double* h, double* vol, double* stretch, double* tag) {
  if (!ctx) return PMPIC_ERR_ARG;
  if (n) *n = ctx->n;
  if (capacity < ctx->n) return set_error(ctx, PMPIC_ERR_ARG, "download capacity below parcel count");
  double* dst[11] = {x, y, z, p, q, r, b, h, vol, stretch, tag};
  cudaSetDevice(ctx->device);
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  for (int i = 0; i < 11; ++i)
    if (dst[i]) {
      int rc = get_prop(ctx, kIO[i], ctx->n, dst[i]);
      if (rc) return rc;
    }
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return PMPIC_OK;
}

int pmpic_download_grid(pmpic_ctx* ctx, int grid, double* dst) {
  if (!ctx || grid < 0 || grid >= PMPIC_NGRID || !dst) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->mixed) {  // FP32 grid widened into the spare grid first
    k_f2d<<<cblk(ctx->g.nphys), 256, 0, ctx->stream>>>(ctx->g.nphys, (const float*)ctx->grid[grid], ctx->gspare);
    ++ctx->nlaunch;
    ctx->btot_grid_ready = false;  // gspare is overwritten
    PMPIC_CUDA(cudaMemcpyAsync(dst, ctx->gspare, sizeof(double) * ctx->g.nphys, cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    PMPIC_CUDA(cudaMemcpyAsync(dst, ctx->grid[grid], sizeof(double) * ctx->g.nphys, cudaMemcpyDeviceToHost, ctx->stream));
  }
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return PMPIC_OK;
}
int pmpic_upload_grid(pmpic_ctx* ctx, int grid, const double* src) {
  if (!ctx || grid < 0 || grid >= PMPIC_NGRID || !src) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->mixed) {
    PMPIC_CUDA(cudaMemcpyAsync(ctx->gspare, src, sizeof(double) * ctx->g.nphys, cudaMemcpyHostToDevice, ctx->stream));
    k_d2f<<<cblk(ctx->g.nphys), 256, 0, ctx->stream>>>(ctx->g.nphys, ctx->gspare, (float*)ctx->grid[grid]);
    ++ctx->nlaunch;
    ctx->btot_grid_ready = false;
  } else {
    PMPIC_CUDA(cudaMemcpyAsync(ctx->grid[grid], src, sizeof(double) * ctx->g.nphys, cudaMemcpyHostToDevice, ctx->stream));
  }
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return PMPIC_OK;
}
int pmpic_download_spectral(pmpic_ctx* ctx, int spec, double* dst) {
  if (!ctx || spec < 0 || spec >= PMPIC_NSPEC || !dst) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->mixed) {
    k_f2d<<<cblk(ctx->g.nspec), 256, 0, ctx->stream>>>(ctx->g.nspec, (const float*)ctx->spec[spec], ctx->sscratch);
    ++ctx->nlaunch;
    PMPIC_CUDA(cudaMemcpyAsync(dst, ctx->sscratch, sizeof(double) * ctx->g.nspec, cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    PMPIC_CUDA(cudaMemcpyAsync(dst, ctx->spec[spec], sizeof(double) * ctx->g.nspec, cudaMemcpyDeviceToHost, ctx->stream));
  }
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return PMPIC_OK;
}

int pmpic_get_counters(pmpic_ctx* ctx, int32_t c[5]) {
  if (!ctx || !c) return PMPIC_ERR_ARG;
  for (int i = 0; i < 5; ++i) c[i] = ctx->counters[i];
  return PMPIC_OK;
}
int pmpic_set_counters(pmpic_ctx* ctx, const int32_t c[5]) {
  if (!ctx || !c || c[2] < 1 || c[2] > 4) return PMPIC_ERR_ARG;
  for (int i = 0; i < 5; ++i) ctx->counters[i] = c[i];
  return PMPIC_OK;
}
int pmpic_set_dtm(pmpic_ctx* ctx, double dtm) {
  if (!ctx) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  PMPIC_CUDA(cudaMemcpyAsync(&ctx->dinfo->dtm, &dtm, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->dtm = dtm;
  ctx->info.dtm = dtm;
  return PMPIC_OK;
}

int pmpic_get_step_info(pmpic_ctx* ctx, pmpic_step_info* info) {
  if (!ctx || !info) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = sync_info(ctx);
  *info = ctx->info;
  info->n_parcels = ctx->n;
  info->error = rc ? rc : 0;
  std::snprintf(info->message, sizeof(info->message), "%s", ctx->err.c_str());
  return rc;
}

int pmpic_conserved_sums(pmpic_ctx* ctx, double sums[3]) {
  if (!ctx || !sums) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = conserved_sums(ctx);
  if (!rc) rc = sync_info(ctx);
  if (rc) return rc;
  sums[0] = ctx->info.vol_sum;
  sums[1] = ctx->info.hvol_sum;
  sums[2] = ctx->info.bvol_sum;
  return PMPIC_OK;
}

// ---- component callbacks --------------------------------------------------------
// Internal forms without the trailing error check; the public entry points
// check the sticky device error word once per call.

static int do_vort2vel(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_V2V);
  int rc;
  if ((rc = flush_gathers(ctx))) return rc;
  // vort2vel.F90:117-121: binning and par2grid of p, q, r with one set of
  // weights.  The par2grid(btot) of vorticity_tendency.F90:121-129 uses the
  // same weights and parcel state, so it runs in the same pass into a spare
  // grid that the vorticity_tendency callback adopts.  The binning of a
  // mixing call that moved, removed and added no parcel is still current.
  if (!ctx->sorted_valid)
    if ((rc = bin_and_sort(ctx))) return rc;
  // The pass computes the btot property (vorticity_tendency.F90:121-126) as it
  // stages each parcel and stores it.
  if (ctx->mixed) {
    const float* f[4] = {propf(ctx, PMPIC_PROP_P), propf(ctx, PMPIC_PROP_Q), propf(ctx, PMPIC_PROP_R), nullptr};
    float* o[4] = {(float*)ctx->grid[PMPIC_GRID_P], (float*)ctx->grid[PMPIC_GRID_Q], (float*)ctx->grid[PMPIC_GRID_R],
                   (float*)ctx->gspare};
    if ((rc = par2grid_multi_m(ctx, f, 4, o, true))) return rc;
  } else {
    const double* f[4] = {prop(ctx, PMPIC_PROP_P), prop(ctx, PMPIC_PROP_Q), prop(ctx, PMPIC_PROP_R), nullptr};
    double* o[4] = {ctx->grid[PMPIC_GRID_P], ctx->grid[PMPIC_GRID_Q], ctx->grid[PMPIC_GRID_R], ctx->gspare};
    if ((rc = par2grid_multi(ctx, f, 4, o, true))) return rc;
  }
  ctx->btot_grid_ready = true;
  if ((rc = vort2vel_spectral(ctx))) return rc;
  // :325-327: the grid2par of u, v, w is deferred into the rk4 pass (or to
  // the next call that observes the tendencies)
  ctx->pending_uvw = true;
  if (ctx->counters[0] % 4 == 0)
    if ((rc = field_max(ctx, true, false))) return rc;  // :329-372
  ctx->counters[0]++;
  return 0;
}

static int do_vorticity_tendency(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_VT);
  int rc;
  if (ctx->pending_pqr) {  // a second call without rk4 in between: apply the first
    bool u = ctx->pending_uvw;  // u, v, w stay pending
    ctx->pending_uvw = false;
    if ((rc = flush_gathers(ctx))) return rc;
    ctx->pending_uvw = u;
  }
  // par2grid(btot) (:129): computed by vort2vel's pass when the state is unchanged
  if (ctx->btot_grid_ready && ctx->sorted_valid) {
    // :121-126, the btot property: written by that pass
    std::swap(ctx->grid[PMPIC_GRID_B], ctx->gspare);
  } else {
    if ((rc = compute_btot(ctx))) return rc;
    if (!ctx->sorted_valid)
      if ((rc = bin_and_sort(ctx))) return rc;
    if (ctx->mixed) {
      const float* f[1] = {propf(ctx, PMPIC_PROP_BTOT)};
      float* o[1] = {(float*)ctx->grid[PMPIC_GRID_B]};
      if ((rc = par2grid_multi_m(ctx, f, 1, o))) return rc;
    } else {
      const double* f[1] = {nullptr};
      double* o[1] = {ctx->grid[PMPIC_GRID_B]};
      if ((rc = par2grid_multi(ctx, f, 1, o, true))) return rc;
    }
  }
  ctx->btot_grid_ready = false;
  if ((rc = vorticity_tendency_grids(ctx))) return rc;
  // :273-275: the grid2par of dp, dq, dr is deferred like vort2vel's
  ctx->pending_pqr = true;
  if (ctx->counters[1] % 4 == 0)
    if ((rc = field_max(ctx, false, true))) return rc;  // :277-313
  ctx->counters[1]++;
  return 0;
}

static int do_rk4(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_RK4);
  ctx->btot_grid_ready = false;
  int rc;
  if ((rc = rk4_stage(ctx, ctx->counters[2]))) return rc;
  ctx->counters[2] = ctx->counters[2] < 4 ? ctx->counters[2] + 1 : 1;  // rk4_integrator.F90:311-315
  return parcel_haloswap(ctx);                                          // :317
}

static int do_split(pmpic_ctx* ctx) {
  int rc = 0;
  if (ctx->counters[3] % 4 == 3) {  // parcel_splitting.F90:59
    TimerScope ts(ctx, T_SPLIT);
    rc = splitting(ctx);
  }
  ctx->counters[3]++;
  return rc;
}

static int do_mix(pmpic_ctx* ctx) {
  int rc = 0;
  if (ctx->counters[4] % 4 == 3) {  // parcel_mixing.F90:77
    TimerScope ts(ctx, T_MIX);
    rc = mixing(ctx);
    // the diagnostic totals after mixing (parcel_mixing.F90:409-418)
    if (!rc) rc = conserved_sums(ctx);
  }
  ctx->counters[4]++;
  return rc;
}

#define PMPIC_ENTRY(body)                 \
  if (!ctx) return PMPIC_ERR_ARG;         \
  cudaSetDevice(ctx->device);             \
  int rc_ = (body);                       \
  if (rc_) return rc_;                    \
  return sync_info(ctx);

int pmpic_euler_integrator(pmpic_ctx* ctx) { PMPIC_ENTRY(euler_step(ctx)) }
int pmpic_prescribed_velocity(pmpic_ctx* ctx, int profile) { PMPIC_ENTRY(prescribed_velocity(ctx, profile, false)) }
int pmpic_prescribed_velocity_tag(pmpic_ctx* ctx) { PMPIC_ENTRY(prescribed_velocity(ctx, 0, true)) }
int pmpic_setup_plume(pmpic_ctx* ctx, const pmpic_plume_params* prm, int64_t* n_plume) {
  if (!prm) return PMPIC_ERR_ARG;
  PMPIC_ENTRY(setup_plume(ctx, prm, n_plume))
}
int pmpic_setup_basic(pmpic_ctx* ctx, int32_t parcels_per_cell_dir) {
  PMPIC_ENTRY(setup_basic(ctx, parcels_per_cell_dir))
}
int pmpic_setup_thermal_device(pmpic_ctx* ctx, const pmpic_thermal_params* prm) {
  if (!prm) return PMPIC_ERR_ARG;
  PMPIC_ENTRY(setup_thermal_device(ctx, prm))
}
int pmpic_vort2vel(pmpic_ctx* ctx) { PMPIC_ENTRY(do_vort2vel(ctx)) }
int pmpic_vorticity_tendency(pmpic_ctx* ctx) { PMPIC_ENTRY(do_vorticity_tendency(ctx)) }
int pmpic_rk4_integrator(pmpic_ctx* ctx) { PMPIC_ENTRY(do_rk4(ctx)) }
int pmpic_parcel_splitting(pmpic_ctx* ctx) { PMPIC_ENTRY(do_split(ctx)) }
int pmpic_parcel_mixing(pmpic_ctx* ctx) { PMPIC_ENTRY(do_mix(ctx)) }

int pmpic_step(pmpic_ctx* ctx, int nsteps) {
  if (!ctx || nsteps < 0) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  for (int s = 0; s < nsteps; ++s) {
    TimerScope ts(ctx, T_STEP);
    for (int sub = 0; sub < 4; ++sub) {
      int rc;
      if ((rc = do_vort2vel(ctx))) return rc;
      if ((rc = do_vorticity_tendency(ctx))) return rc;
      // the last stage of a step can advance the stretch for the split that
      // follows; the earlier stages' tendencies are dead (store_tendencies)
      ctx->split_follows = ctx->counters[3] % 4 == 3;
      // another stage follows within this call, with no split in between
      ctx->in_step = ctx->counters[2] < 4 && !ctx->split_follows && !(s == nsteps - 1 && sub == 3);
      rc = do_rk4(ctx);
      ctx->split_follows = false;
      ctx->in_step = false;
      if (rc) return rc;
      if ((rc = do_split(ctx))) return rc;
      if ((rc = do_mix(ctx))) return rc;
    }
    int rc = sync_info(ctx);
    if (rc) return rc;
  }
  return PMPIC_OK;
}

// ---- kernel-level entry points ----------------------------------------------------
int pmpic_op_cell_ids(pmpic_ctx* ctx, int32_t* cells) {
  if (!ctx || !cells) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  {
    int frc = flush_gathers(ctx);
    if (frc) return frc;
  }
  int rc = cell_ids(ctx, ctx->aux);
  if (rc) return rc;
  PMPIC_CUDA(cudaMemcpyAsync(cells, ctx->aux, sizeof(int32_t) * ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_info(ctx);
}

int pmpic_op_par2grid(pmpic_ctx* ctx, int p, int grid) {
  if (!ctx || p < 0 || p >= PMPIC_NPROP || grid < 0 || grid >= PMPIC_NGRID) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  {
    int frc = flush_gathers(ctx);
    if (frc) return frc;
  }
  int rc = bin_and_sort(ctx);
  if (rc) return rc;
  const double* f[1] = {prop(ctx, p)};
  double* o[1] = {ctx->grid[grid]};
  if ((rc = par2grid_multi(ctx, f, 1, o, false))) return rc;
  return sync_info(ctx);
}

int pmpic_op_grid2par(pmpic_ctx* ctx, int grid, int p) {
  if (!ctx || p < 0 || p >= PMPIC_NPROP || grid < 0 || grid >= PMPIC_NGRID) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  {
    int frc = flush_gathers(ctx);
    if (frc) return frc;
  }
  const double* gr[1] = {ctx->grid[grid]};
  double* out[1] = {prop(ctx, p)};
  int rc = grid2par_multi(ctx, gr, 1, out);
  if (rc) return rc;
  return sync_info(ctx);
}

// host <-> device helpers for the spectral test entry points
static int h2d(pmpic_ctx* ctx, double* d, const double* h, size_t n) {
  PMPIC_CUDA(cudaMemcpyAsync(d, h, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}
static int d2h(pmpic_ctx* ctx, double* h, const double* d, size_t n) {
  PMPIC_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int pmpic_op_fft_forward(pmpic_ctx* ctx, const double* phys, double* spec) {
  if (!ctx || !phys || !spec) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = h2d(ctx, ctx->gwork[0], phys, ctx->g.nphys))) return rc;
  if ((rc = fft_forward(ctx, ctx->gwork[0], ctx->sa))) return rc;
  return d2h(ctx, spec, ctx->sa, ctx->g.nspec);
}
int pmpic_op_fft_backward(pmpic_ctx* ctx, const double* spec, double* phys) {
  if (!ctx || !phys || !spec) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = h2d(ctx, ctx->sa, spec, ctx->g.nspec))) return rc;
  if ((rc = fft_backward(ctx, ctx->sa, ctx->gwork[0]))) return rc;
  return d2h(ctx, phys, ctx->gwork[0], ctx->g.nphys);
}

typedef int (*spec_op)(pmpic_ctx*, const double*, double*);
static int spec_unary(pmpic_ctx* ctx, const double* in, double* out, spec_op op) {
  if (!ctx || !in || !out) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = h2d(ctx, ctx->sa, in, ctx->g.nspec))) return rc;
  if ((rc = op(ctx, ctx->sa, ctx->sb))) return rc;
  return d2h(ctx, out, ctx->sb, ctx->g.nspec);
}
int pmpic_op_diffx(pmpic_ctx* ctx, const double* in, double* out) { return spec_unary(ctx, in, out, spec_diffx); }
int pmpic_op_diffy(pmpic_ctx* ctx, const double* in, double* out) { return spec_unary(ctx, in, out, spec_diffy); }
int pmpic_op_filter(pmpic_ctx* ctx, const double* in, double* out) { return spec_unary(ctx, in, out, spec_filter); }
int pmpic_op_diffz(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top) {
  if (!ctx || !in || !out || ((bot == nullptr) != (top == nullptr))) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  int rc;
  const size_t cols = (size_t)ctx->g.sx * ctx->g.sy;
  if ((rc = h2d(ctx, ctx->sa, in, ctx->g.nspec))) return rc;
  const double *db = nullptr, *dt = nullptr;
  if (bot) {
    if ((rc = h2d(ctx, ctx->bt, bot, cols))) return rc;
    if ((rc = h2d(ctx, ctx->bt + cols, top, cols))) return rc;
    db = ctx->bt;
    dt = ctx->bt + cols;
  }
  if ((rc = spec_diffz(ctx, ctx->sa, ctx->sb, db, dt))) return rc;
  return d2h(ctx, out, ctx->sb, ctx->g.nspec);
}
int pmpic_op_laplinv(pmpic_ctx* ctx, double* inout, int df0) {
  if (!ctx || !inout) return PMPIC_ERR_ARG;
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "kernel-level FP64 operator on a mixed-precision context");
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = h2d(ctx, ctx->sa, inout, ctx->g.nspec))) return rc;
  if ((rc = spec_laplinv(ctx, ctx->sa, df0 != 0))) return rc;
  if ((rc = d2h(ctx, inout, ctx->sa, ctx->g.nspec))) return rc;
  return sync_info(ctx);
}
int pmpic_op_vort2vel_grids(pmpic_ctx* ctx) {
  if (!ctx) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = vort2vel_spectral(ctx);
  if (rc) return rc;
  return sync_info(ctx);
}

int pmpic_op_par2grid_multi(pmpic_ctx* ctx, int nf, const int* props, const int* grids) {
  if (!ctx || !props || !grids || (nf != 1 && nf != 3 && nf != 4)) return PMPIC_ERR_ARG;
  for (int q = 0; q < nf; ++q)
    if (props[q] < 0 || props[q] >= PMPIC_NPROP || grids[q] < 0 || grids[q] >= PMPIC_NGRID) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = flush_gathers(ctx);
  if (rc) return rc;
  if ((rc = bin_and_sort(ctx))) return rc;
  if (ctx->mixed) {
    const float* f[4];
    float* o[4];
    for (int q = 0; q < nf; ++q) {
      if (mixed_elem_bytes(props[q]) != 4) return set_error(ctx, PMPIC_ERR_ARG, "par2grid of a position or tag");
      f[q] = propf(ctx, props[q]);
      o[q] = (float*)ctx->grid[grids[q]];
    }
    rc = par2grid_multi_m(ctx, f, nf, o);
  } else {
    const double* f[4];
    double* o[4];
    for (int q = 0; q < nf; ++q) {
      f[q] = prop(ctx, props[q]);
      o[q] = ctx->grid[grids[q]];
    }
    rc = par2grid_multi(ctx, f, nf, o, false);
  }
  if (rc) return rc;
  ctx->btot_grid_ready = false;
  return sync_info(ctx);
}

int pmpic_op_grid2par_multi(pmpic_ctx* ctx, int ng, const int* grids, const int* props) {
  if (!ctx || !props || !grids || (ng != 1 && ng != 3 && ng != 6)) return PMPIC_ERR_ARG;
  for (int q = 0; q < ng; ++q)
    if (props[q] < 0 || props[q] >= PMPIC_NPROP || grids[q] < 0 || grids[q] >= PMPIC_NGRID) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = flush_gathers(ctx);
  if (rc) return rc;
  if (ctx->mixed) {
    const float* gr[6];
    float* o[6];
    for (int q = 0; q < ng; ++q) {
      if (mixed_elem_bytes(props[q]) != 4) return set_error(ctx, PMPIC_ERR_ARG, "grid2par into a position or tag");
      gr[q] = (const float*)ctx->grid[grids[q]];
      o[q] = propf(ctx, props[q]);
    }
    rc = grid2par_multi_m(ctx, gr, ng, o);  // reports positions outside the grid
  } else {
    const double* gr[6];
    double* o[6];
    for (int q = 0; q < ng; ++q) {
      gr[q] = ctx->grid[grids[q]];
      o[q] = prop(ctx, props[q]);
    }
    rc = grid2par_multi(ctx, gr, ng, o);
  }
  if (rc) return rc;
  return sync_info(ctx);
}

namespace {
__global__ void k_permute(int64_t n, const int32_t* __restrict__ perm, const void* __restrict__ src,
                          void* __restrict__ dst, int es) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  if (es == 8) ((double*)dst)[q] = ((const double*)src)[perm[q]];
  else ((float*)dst)[q] = ((const float*)src)[perm[q]];
}
}  // namespace

int pmpic_sort_parcels(pmpic_ctx* ctx) {
  if (!ctx) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = flush_gathers(ctx);
  if (rc) return rc;
  const int64_t n = ctx->n;
  if (n == 0) return PMPIC_OK;
  if ((rc = bin_and_sort(ctx))) return rc;
  if ((rc = sync_info(ctx))) return rc;  // every parcel binned (else out of box)
  void* tmp = nullptr;
  PMPIC_CUDA(cudaMalloc(&tmp, sizeof(double) * (size_t)n));
  // every property, and on the mixed form the cell ids (part of its positions)
  for (int p = 0; p <= PMPIC_NPROP && !rc; ++p) {
    if (p == PMPIC_NPROP && !ctx->mixed) break;
    void* col = p < PMPIC_NPROP ? (void*)prop(ctx, p) : (void*)ctx->cell;
    const int es = p == PMPIC_NPROP ? 4 : (ctx->mixed ? mixed_elem_bytes(p) : 8);
    k_permute<<<cblk(n), 256, 0, ctx->stream>>>(n, ctx->sorted, col, tmp, es);
    ++ctx->nlaunch;
    cudaError_t e = cudaMemcpyAsync(col, tmp, (size_t)es * n, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemcpyAsync", __LINE__);
  }
  cudaStreamSynchronize(ctx->stream);
  cudaFree(tmp);
  if (rc) return rc;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->dir_ready = false;
  return sync_info(ctx);
}

int pmpic_op_parcel_haloswap(pmpic_ctx* ctx) {
  if (!ctx) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  {
    int frc = flush_gathers(ctx);
    if (frc) return frc;
  }
  int rc = parcel_haloswap(ctx);
  if (rc) return rc;
  return sync_info(ctx);
}

// ---- instrumentation -------------------------------------------------------------
int pmpic_timing(pmpic_ctx* ctx, int enable) {
  if (!ctx) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  drain_timers(ctx);
  for (int t = 0; t < T_NT; ++t) {
    ctx->tms[t] = 0.0;
    ctx->tcalls[t] = 0;
  }
  ctx->timing = enable != 0;
  return PMPIC_OK;
}
int pmpic_timer_count(void) { return T_NT; }
const char* pmpic_timer_name(int id) { return (id >= 0 && id < T_NT) ? kTimerNames[id] : ""; }
int pmpic_timer_read(pmpic_ctx* ctx, int id, double* total_ms, int64_t* calls) {
  if (!ctx || id < 0 || id >= T_NT) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  drain_timers(ctx);
  if (total_ms) *total_ms = ctx->tms[id];
  if (calls) *calls = ctx->tcalls[id];
  return PMPIC_OK;
}
int pmpic_launch_count(pmpic_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return PMPIC_ERR_ARG;
  *n = ctx->nlaunch;
  return PMPIC_OK;
}
int pmpic_event_record(pmpic_ctx* ctx, int slot) {
  if (!ctx || slot < 0 || slot >= 8) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  PMPIC_CUDA(cudaEventRecord(ctx->marks[slot], ctx->stream));
  return PMPIC_OK;
}
int pmpic_event_elapsed(pmpic_ctx* ctx, int a, int b, float* ms) {
  if (!ctx || a < 0 || a >= 8 || b < 0 || b >= 8 || !ms) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  PMPIC_CUDA(cudaEventSynchronize(ctx->marks[b]));
  PMPIC_CUDA(cudaEventElapsedTime(ms, ctx->marks[a], ctx->marks[b]));
  return PMPIC_OK;
}
int pmpic_pin_host(void* ptr, size_t bytes) {
  if (!ptr || bytes == 0) return PMPIC_ERR_ARG;
  return cudaHostRegister(ptr, bytes, cudaHostRegisterDefault) == cudaSuccess ? PMPIC_OK : PMPIC_ERR_CUDA;
}
int pmpic_unpin_host(void* ptr) {
  if (!ptr) return PMPIC_ERR_ARG;
  return cudaHostUnregister(ptr) == cudaSuccess ? PMPIC_OK : PMPIC_ERR_CUDA;
}

}  // extern "C"
