// setup.cu -- parcel initial conditions generated on the device.
//
// Set-up components write the context's parcel state directly in HBM (FP64
// or the mixed form's cell index + FP32 offset), so that a 10^8-parcel start
// is not bound by host generation and a PCIe upload:
//  * the reference's basic_parcelsetup (basic_parcelsetup.F90:22-134): a
//    regular sub-lattice of n^3 parcels per cell, vol = 1;
//  * the reference's plume_parcelsetup (plume_parcelsetup.F90:58-334): a
//    spherical plume on a 4^3-per-cell lattice and the environment on a
//    2^3-per-cell lattice outside it, in the reference's slot order;
//  * the jittered thermal of the benchmark workloads (the same Philox stream
//    and formula as the host generator pmpic_setup_thermal).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "thermal.h"

namespace pmpic {
namespace {

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// one property value into slot s, in the context's precision; a position as
// its three components at once (the mixed form packs them into a cell id and
// three offsets)
struct ParcelSink {
  double* base;  // ctx->parcels
  int64_t cap;
  bool mixed;
  Geom g;
  int32_t* cell;    // the mixed form's cell ids
  DevInfo* info;
  __device__ __forceinline__ void put(int pid, int64_t s, double v) const {
    double* col = base + (size_t)pid * (size_t)cap;
    if (!mixed || pid == PMPIC_PROP_TAG) col[s] = v;
    else ((float*)col)[s] = (float)v;
  }
  __device__ __forceinline__ void put_xyz(int64_t s, double x, double y, double z) const {
    if (!mixed) {
      base[(size_t)PMPIC_PROP_X * cap + s] = x;
      base[(size_t)PMPIC_PROP_Y * cap + s] = y;
      base[(size_t)PMPIC_PROP_Z * cap + s] = z;
      return;
    }
    int32_t id;
    float fx, fy, fz;
    if (!cur_from_double(g, x, y, z, id, fx, fy, fz)) atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    cell[s] = id;
    ((float*)(base + (size_t)PMPIC_PROP_X * cap))[s] = fx;
    ((float*)(base + (size_t)PMPIC_PROP_Y * cap))[s] = fy;
    ((float*)(base + (size_t)PMPIC_PROP_Z * cap))[s] = fz;
  }
};

ParcelSink sink_of(pmpic_ctx* ctx) {
  ParcelSink k;
  k.base = ctx->parcels;
  k.cap = ctx->cap;
  k.mixed = ctx->mixed;
  k.g = ctx->g;
  k.cell = ctx->cell;
  k.info = ctx->dinfo;
  return k;
}

// The two lattices of plume_parcelsetup as columns (i, j) walked along k:
// columns [0, npl) are the plume's (i outer, j inner, :209-240), columns
// [npl, npl + nbg) the environment's (:255-297).  Coordinates come from
// tables built on the host by the reference's repeated additions.
struct PlumeLattice {
  int64_t npl, nbg;       // column counts
  int jpl, jbg;           // columns per i (4 Ny, 2 Ny)
  int kpl, kbg;           // points per column (ceiling(2 r / dzplume), 2 (nz-1))
  const double* xpl;      // [4 Nx] x of the plume lattice
  const double* ypl;      // [4 Ny]
  const double* zpl;      // [kpl]
  const double* xbg;      // [2 Nx]
  const double* ybg;      // [2 Ny]
  const double* zbg;      // [kbg]
  const double* bbg;      // [kbg] environment buoyancy per level (:274-283)
  const double* hbg;      // [kbg] environment humidity per level
  double xc, yc, zc, rr;  // plume centre, r^2
  double b_pl, h_pl, e1, e2, e3, vol_pl, vol_bg;
};

// the acceptance test of a lattice point, in the reference's operand order:
// inside the plume (:216), outside it for the environment (:263)
__device__ __forceinline__ bool plume_accept(const PlumeLattice& L, int64_t col, int k, double& xp, double& yp,
                                             double& zp) {
  if (col < L.npl) {
    xp = L.xpl[col / L.jpl] - L.xc;
    yp = L.ypl[col % L.jpl] - L.yc;
    zp = L.zpl[k] - L.zc;
    return zp * zp + xp * xp + yp * yp <= L.rr;
  }
  const int64_t c = col - L.npl;
  xp = L.xbg[c / L.jbg] - L.xc;
  yp = L.ybg[c % L.jbg] - L.yc;
  zp = L.zbg[k] - L.zc;
  return zp * zp + yp * yp + xp * xp > L.rr;
}

// one warp per column: the number of accepted points
__global__ void k_plume_count(PlumeLattice L, int32_t* __restrict__ count) {
  const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (col >= L.npl + L.nbg) return;
  const int kn = col < L.npl ? L.kpl : L.kbg;
  int total = 0;
  for (int k0 = 0; k0 < kn; k0 += 32) {
    const int k = k0 + lane;
    double xp, yp, zp;
    const bool ok = k < kn && plume_accept(L, col, k, xp, yp, zp);
    total += __popc(__ballot_sync(0xffffffffu, ok));
  }
  if (lane == 0) count[col] = total;
}

// one warp per column: the accepted points into slots off[col] + rank, in k
// order, with the properties of :220-226 and :270-286
__global__ void k_plume_write(PlumeLattice L, const int64_t* __restrict__ off, ParcelSink out) {
  const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (col >= L.npl + L.nbg) return;
  const bool plume = col < L.npl;
  const int kn = plume ? L.kpl : L.kbg;
  int64_t s0 = off[col];
  for (int k0 = 0; k0 < kn; k0 += 32) {
    const int k = k0 + lane;
    double xp = 0, yp = 0, zp = 0;
    const bool ok = k < kn && plume_accept(L, col, k, xp, yp, zp);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      const int64_t s = s0 + __popc(m & ((1u << lane) - 1u));
      if (plume) {
        out.put_xyz(s, L.xpl[col / L.jpl], L.ypl[col % L.jpl], L.zpl[k]);
        out.put(PMPIC_PROP_B, s, L.b_pl * (1. + L.e1 * xp * yp + L.e2 * xp * zp + L.e3 * yp * zp));
        out.put(PMPIC_PROP_H, s, L.h_pl);
        out.put(PMPIC_PROP_VOL, s, L.vol_pl);
      } else {
        const int64_t c = col - L.npl;
        out.put_xyz(s, L.xbg[c / L.jbg], L.ybg[c % L.jbg], L.zbg[k]);
        out.put(PMPIC_PROP_B, s, L.bbg[k]);
        out.put(PMPIC_PROP_H, s, L.hbg[k]);
        out.put(PMPIC_PROP_VOL, s, L.vol_bg);
      }
    }
    s0 += __popc(m);
  }
}

// the jittered thermal, one thread per parcel (the host generator's formula)
__global__ void k_thermal(pmpic_thermal_params prm, ThermalGeom tg, int64_t n, ParcelSink out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const ThermalParcel p = thermal_parcel(prm, tg, t);
  out.put_xyz(t, p.x, p.y, p.z);
  out.put(PMPIC_PROP_B, t, p.b);
  out.put(PMPIC_PROP_H, t, p.h);
  out.put(PMPIC_PROP_VOL, t, tg.v0);
  out.put(PMPIC_PROP_TAG, t, (double)t);
}

// basic_parcelsetup (basic_parcelsetup.F90:91-115), one thread per parcel in
// the reference's order (cell by cell, x outer, then the sub-lattice, x
// outer); x_coords(n) = pxmin + (n - 1) dx + bottom as in
// parcel_interpolation.F90:126-136, interior cells from index 3 in x and y
// (halo 2) and 1 in z
struct BasicLattice {
  int Nx, Ny, Nz, s;
  double pxmin, pymin, pzmin, dx, dy, dz, bx, by, bz;
};
__device__ __forceinline__ double lattice_coord(double pmin, int n, double d, double b) {
  return pmin + (double)(n - 1) * d + b;
}
__global__ void k_basic(BasicLattice L, int64_t n, ParcelSink out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t per_cell = (int64_t)L.s * L.s * L.s;
  const int64_t cell = t / per_cell;
  const int w = (int)(t - cell * per_cell);
  const int i = (int)(cell / ((int64_t)L.Ny * L.Nz)) + 3;
  const int j = (int)((cell / L.Nz) % L.Ny) + 3;
  const int k = (int)(cell % L.Nz) + 1;
  const int ii = w / (L.s * L.s), jj = (w / L.s) % L.s, kk = w % L.s;
  const double xi = lattice_coord(L.pxmin, i, L.dx, L.bx), yj = lattice_coord(L.pymin, j, L.dy, L.by);
  const double zk = lattice_coord(L.pzmin, k, L.dz, L.bz);
  const double ddx = (lattice_coord(L.pxmin, i + 1, L.dx, L.bx) - xi) / L.s;
  const double ddy = (lattice_coord(L.pymin, j + 1, L.dy, L.by) - yj) / L.s;
  const double ddz = (lattice_coord(L.pzmin, k + 1, L.dz, L.bz) - zk) / L.s;
  out.put_xyz(t, xi + ddx / 2 + (double)ii * ddx, yj + ddy / 2 + (double)jj * ddy, zk + ddz / 2 + (double)kk * ddz);
  out.put(PMPIC_PROP_VOL, t, 1.0);
}

// a new state of n parcels whose properties `set` were written on the device:
// zero the rest over [0, n) and reset the state flags as an upload does
int finish_state(pmpic_ctx* ctx, int64_t n, const std::vector<int>& set) {
  for (int pid = 0; pid < PMPIC_NPROP; ++pid) {
    if (std::find(set.begin(), set.end(), pid) != set.end()) continue;
    int rc = prop_upload(ctx, pid, 0, n, nullptr);
    if (rc) return rc;
  }
  PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->error, 0, sizeof(int), ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->n = n;
  ctx->info.n_parcels = n;
  ctx->pending_uvw = ctx->pending_pqr = false;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->dir_ready = false;
  return 0;
}

}  // namespace

// plume_parcelsetup initialisation (plume_parcelsetup.F90:58-334), one process
int setup_plume(pmpic_ctx* ctx, const pmpic_plume_params* prm, int64_t* n_plume_out) {
  // module parameters (:30-47): default-real literals widened to double, as
  // the reference is built without -fdefault-real-8
  const double latent = 0.125;
  const double fdthetal0 = (double)0.01f;
  const double gravity = 1. / fdthetal0;
  const double glat = gravity * latent;
  const int n_pl = 4, n_bg = 2;
  const double lambda = prm->lambda, rhb = prm->H, mu = prm->mu;
  if (rhb > 1) return set_error(ctx, PMPIC_ERR_ARG, "plume set-up: relative humidity fraction must be less than 1");
  const double h_pl = std::exp(-prm->z_c);  // :94
  if (mu > 1 || mu <= rhb) return set_error(ctx, PMPIC_ERR_ARG, "plume set-up: mu must be between H and 1");
  const double h_bg = mu * h_pl;                                                           // :106
  double z_b = std::log(rhb / h_bg);                                                       // :109
  const double dbdz = glat * (h_pl - std::exp(-prm->z_m)) / (prm->z_m - prm->z_d);         // :116
  const double b_pl = dbdz * (prm->z_d - z_b);                                             // :120
  if (2. * prm->r_plume > z_b) return set_error(ctx, PMPIC_ERR_ARG, "plume set-up: plume radius is too big");
  z_b = z_b * lambda;  // :139-143
  const double r_plume = prm->r_plume * lambda;
  double e[3];
  for (int v = 0; v < 3; ++v) e[v] = prm->e_values[v] / r_plume / r_plume;  // :145

  // this process's box and the plume centre (:162-186); x_coords(n) of
  // parcel_interpolation.F90:126-136 with the halo of 2 in x and y, 0 in z
  const Geom& g = ctx->g;
  const double bx = ctx->cfg.xmin, by = ctx->cfg.ymin, bz = ctx->cfg.zmin;
  auto xcoord = [&](int n) { return g.pxmin + (double)(n - 1) * g.dx + bx; };
  auto ycoord = [&](int n) { return g.pymin + (double)(n - 1) * g.dy + by; };
  const double xmin_local = xcoord(3), xmax_local = xcoord(4 + g.Nx - 1);
  const double ymin_local = ycoord(3), ymax_local = ycoord(4 + g.Ny - 1);
  const double zmin_local = g.pzmin + 0.0 * g.dz + bz;
  const double topx = ctx->cfg.xmax - g.dx, topy = ctx->cfg.ymax - g.dy;
  const double x_c_pl = (topx + g.dx - bx) / 2 + bx;
  const double y_c_pl = (topy + g.dy - by) / 2 + by;
  const double z_c_pl = r_plume;
  if (z_c_pl + r_plume > ctx->cfg.zmax)
    return set_error(ctx, PMPIC_ERR_ARG, "plume set-up: the plume reaches above the domain top");
  const double dxplume = g.dx / n_pl, dyplume = g.dy / n_pl, dzplume = g.dz / n_pl;  // :189-191
  const double dxbg = g.dx / n_bg, dybg = g.dy / n_bg, dzbg = g.dz / n_bg;            // :246-248
  const bool in_box = xmax_local > x_c_pl - r_plume && xmin_local < x_c_pl + r_plume &&
                      ymax_local > y_c_pl - r_plume && ymin_local < y_c_pl + r_plume;  // :203-204

  // coordinate tables by repeated addition, as the loops advance x, y, z
  auto walk = [](double start, double step, int64_t count, std::vector<double>& t) {
    double v = start;
    for (int64_t i = 0; i < count; ++i) {
      t.push_back(v);
      v = v + step;
    }
  };
  const int64_t kpl = in_box ? (int64_t)std::ceil(2. * r_plume / dzplume) : 0;
  const int64_t kbg = (int64_t)(g.nzp - 1) * n_bg;
  if (kpl > (1 << 30)) return set_error(ctx, PMPIC_ERR_ARG, "plume set-up: lattice too large");
  std::vector<double> tab;
  size_t o_xpl = tab.size();
  walk(xmin_local + dxplume / 2., dxplume, (int64_t)g.Nx * n_pl, tab);
  size_t o_ypl = tab.size();
  walk(ymin_local + dyplume / 2., dyplume, (int64_t)g.Ny * n_pl, tab);
  size_t o_zpl = tab.size();
  walk(zmin_local + dzplume / 2., dzplume, kpl, tab);
  size_t o_xbg = tab.size();
  walk(xmin_local + dxbg / 2., dxbg, (int64_t)g.Nx * n_bg, tab);
  size_t o_ybg = tab.size();
  walk(ymin_local + dybg / 2., dybg, (int64_t)g.Ny * n_bg, tab);
  size_t o_zbg = tab.size();
  walk(zmin_local + dzbg / 2., dzbg, kbg, tab);
  size_t o_bbg = tab.size(), o_hbg = o_bbg + (size_t)kbg;
  tab.resize(o_hbg + (size_t)kbg);
  for (int64_t k = 0; k < kbg; ++k) {  // :274-283
    const double z = tab[o_zbg + k];
    if (z < z_b) {
      tab[o_bbg + k] = 0.;
      tab[o_hbg + k] = h_bg;
    } else {
      tab[o_bbg + k] = dbdz / lambda * (z - z_b);
      tab[o_hbg + k] = rhb * std::exp(-z / lambda);
    }
  }

  PlumeLattice L;
  L.npl = in_box ? (int64_t)g.Nx * n_pl * g.Ny * n_pl : 0;
  L.nbg = (int64_t)g.Nx * n_bg * g.Ny * n_bg;
  L.jpl = g.Ny * n_pl;
  L.jbg = g.Ny * n_bg;
  L.kpl = (int)kpl;
  L.kbg = (int)kbg;
  L.xc = x_c_pl; L.yc = y_c_pl; L.zc = z_c_pl;
  L.rr = r_plume * r_plume;
  L.b_pl = b_pl; L.h_pl = h_pl;
  L.e1 = e[0]; L.e2 = e[1]; L.e3 = e[2];
  L.vol_pl = dxplume * dyplume * dzplume;  // :200
  L.vol_bg = dxbg * dybg * dzbg;           // :250
  const int64_t ncol = L.npl + L.nbg;

  double* dtab = nullptr;
  int32_t* dcount = nullptr;
  int64_t* doff = nullptr;
  cudaError_t err = cudaMalloc(&dtab, sizeof(double) * tab.size());
  if (err == cudaSuccess) err = cudaMalloc(&dcount, sizeof(int32_t) * ncol);
  if (err == cudaSuccess) err = cudaMalloc(&doff, sizeof(int64_t) * ncol);
  int rc = 0;
  int64_t n = 0, n_plume = 0;
  if (err != cudaSuccess) rc = cuda_fail(ctx, err, "plume set-up buffers", __LINE__);
  if (!rc) {
    L.xpl = dtab + o_xpl; L.ypl = dtab + o_ypl; L.zpl = dtab + o_zpl;
    L.xbg = dtab + o_xbg; L.ybg = dtab + o_ybg; L.zbg = dtab + o_zbg;
    L.bbg = dtab + o_bbg; L.hbg = dtab + o_hbg;
    err = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, ctx->stream);
    if (err == cudaSuccess) {
      k_plume_count<<<nblk(ncol * 32, 256), 256, 0, ctx->stream>>>(L, dcount); ++ctx->nlaunch;
      err = cudaGetLastError();
    }
    // slots in the reference's loop order: an exclusive scan of the columns
    std::vector<int32_t> cnt((size_t)ncol);
    std::vector<int64_t> off((size_t)ncol);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(cnt.data(), dcount, sizeof(int32_t) * ncol, cudaMemcpyDeviceToHost, ctx->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
    if (err != cudaSuccess) rc = cuda_fail(ctx, err, "plume set-up count", __LINE__);
    if (!rc) {
      for (int64_t c = 0; c < ncol; ++c) {
        off[c] = n;
        n += cnt[c];
        if (c + 1 == L.npl) n_plume = n;
      }
      if (n > ctx->cap) rc = set_error(ctx, PMPIC_ERR_CAPACITY, "maxparcels reached (plume set-up)");  // :218-221
    }
    if (!rc) {
      err = cudaMemcpyAsync(doff, off.data(), sizeof(int64_t) * ncol, cudaMemcpyHostToDevice, ctx->stream);
      if (err == cudaSuccess) {
        k_plume_write<<<nblk(ncol * 32, 256), 256, 0, ctx->stream>>>(L, doff, sink_of(ctx)); ++ctx->nlaunch;
        err = cudaGetLastError();
      }
      if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
      if (err != cudaSuccess) rc = cuda_fail(ctx, err, "plume set-up write", __LINE__);
    }
  }
  cudaFree(dtab);
  cudaFree(dcount);
  cudaFree(doff);
  if (rc) return rc;
  rc = finish_state(ctx, n, {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_VOL});
  if (!rc && n_plume_out) *n_plume_out = n_plume;
  return rc;
}

// basic_parcelsetup initialisation (basic_parcelsetup.F90:22-134), one process
int setup_basic(pmpic_ctx* ctx, int n_per_dir) {
  if (n_per_dir <= 0) return set_error(ctx, PMPIC_ERR_ARG, "basic set-up: parcels_per_cell_dir must be positive");
  const Geom& g = ctx->g;
  const int64_t n = (int64_t)n_per_dir * n_per_dir * n_per_dir * g.ncell;  // :53-57
  if (n > ctx->cap)                                                      // :63-65
    return set_error(ctx, PMPIC_ERR_CAPACITY, "Maxparcels is not big enough for the number of parcels per cell requested");
  BasicLattice L;
  L.Nx = g.Nx; L.Ny = g.Ny; L.Nz = g.Nz; L.s = n_per_dir;
  L.pxmin = g.pxmin; L.pymin = g.pymin; L.pzmin = g.pzmin;
  L.dx = g.dx; L.dy = g.dy; L.dz = g.dz;
  L.bx = ctx->cfg.xmin; L.by = ctx->cfg.ymin; L.bz = ctx->cfg.zmin;
  if (n > 0) {
    k_basic<<<nblk(n, 256), 256, 0, ctx->stream>>>(L, n, sink_of(ctx)); ++ctx->nlaunch;
    PMPIC_CUDA(cudaGetLastError());
  }
  return finish_state(ctx, n, {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_VOL});
}

// the jittered thermal of pmpic_setup_thermal, written on the device
int setup_thermal_device(pmpic_ctx* ctx, const pmpic_thermal_params* prm) {
  const int64_t n = pmpic_setup_count(prm);
  if (n < 0) return set_error(ctx, PMPIC_ERR_ARG, "thermal set-up: bad parameters");
  if (n > ctx->cap) return set_error(ctx, PMPIC_ERR_CAPACITY, "thermal set-up: parcel count exceeds max_parcels");
  if (n > 0) {
    k_thermal<<<nblk(n, 256), 256, 0, ctx->stream>>>(*prm, thermal_geom(prm), n, sink_of(ctx)); ++ctx->nlaunch;
    PMPIC_CUDA(cudaGetLastError());
  }
  return finish_state(ctx, n, {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_VOL,
                               PMPIC_PROP_TAG});
}

}  // namespace pmpic
