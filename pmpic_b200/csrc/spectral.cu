// spectral.cu -- semi-spectral operators and the vort2vel / vorticity_tendency
// pipelines on the B200.
//
// Restates model_core/src/fft/fft_ops.F90 (wavenumbers :111-140, filter
// :176-197, diffx :204-302, diffy :305-401, diffz :419-483, laplinv :505-601,
// tridiagonal :620-656) for one GPU, plus the spectral parts of
// components/vort2vel/src/vort2vel.F90:139-320 and
// components/vorticity_tendency/src/vorticity_tendency.F90:147-265.
//
// Spectral arrays are (Nz+1) x (Ny+2) x (Nx+2), x' fastest; a column is one
// (j', i') pair over all z.  Elementwise operators are one thread per element;
// the compact z operators are one thread per column running the reference's
// Thomas recurrence with identical arithmetic (no FMA contraction), so they
// reproduce the CPU results bit for bit on identical inputs.
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace pmpic {

namespace {

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// mean flow of the zero mode (vort2vel.F90:230-241), one thread: the trapezoid
// integral and the reference's average (`1./nz` in REAL(4), 0.5*ubar(nz) added
// to every element before the sum).
// d, e: the zero-mode values of level k at d[k * stride], e[k * stride],
// multiplied by the filter's zero-mode factor *filt when filt is given (the
// filtered d = filter(a), e = filter(b) of vort2vel.F90:208-209)
__global__ void k_zmode(Geom g, const double* __restrict__ d, const double* __restrict__ e, int64_t stride,
                        const double* __restrict__ filt, double* __restrict__ zb) {
  extern __shared__ double zs[];  // e(:,1,1), d(:,1,1), then ubar, vbar
  const int nz = g.nzp;
  double* es = zs;
  double* ds = zs + nz;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {  // stage the zero-mode columns
    es[k] = filt ? e[k * stride] * filt[0] : e[k * stride];
    ds[k] = filt ? d[k * stride] * filt[0] : d[k * stride];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double* ubar = zb;
  double* vbar = zb + nz;
  const double dz = g.dz;
  double u = 0, v = 0;
  double* us = zs + 2 * nz;
  double* vs = zs + 3 * nz;
  us[0] = 0;
  vs[0] = 0;
  for (int k = 0; k < nz - 1; ++k) {
    u = u + dz / 2. * (es[k] + es[k + 1]);
    v = v - dz / 2. * (ds[k] + ds[k + 1]);
    us[k + 1] = u;
    vs[k + 1] = v;
  }
  const double inz = (double)(1.0f / (float)nz);
  double su = 0.0, sv = 0.0;
  for (int k = 0; k < nz - 1; ++k) {
    su = su + (us[k] + f4(0.5f) * us[nz - 1]);
    sv = sv + (vs[k] + f4(0.5f) * vs[nz - 1]);
  }
  double uavg = inz * su, vavg = inz * sv;
  for (int k = 0; k < nz; ++k) {
    ubar[k] = us[k] - uavg;
    vbar[k] = vs[k] - vavg;
  }
}

// FP64 horizontal sums of two FP32 grids per level, in one fixed order: the
// zero modes (kx = ky = 0) of their unscaled forward transforms, kept in FP64
// by the mixed-precision form
__global__ void __launch_bounds__(256) k_hsum2(Geom g, const float* __restrict__ p, const float* __restrict__ q,
                                               double* __restrict__ hs) {
  __shared__ double sp[256], sq[256];
  const int k = blockIdx.x;
  const int64_t m = (int64_t)g.Ny * g.Nx;
  const float* P = p + (size_t)k * m;
  const float* Q = q + (size_t)k * m;
  double a = 0.0, b = 0.0;
  for (int64_t e = threadIdx.x; e < m; e += 256) {
    a += (double)P[e];
    b += (double)Q[e];
  }
  sp[threadIdx.x] = a;
  sq[threadIdx.x] = b;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sp[threadIdx.x] += sp[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    hs[k] = sp[0];
    hs[g.nzp + k] = sq[0];
  }
}

// dt rule (vort2vel.F90:329-372, vorticity_tendency.F90:277-313), one thread
__global__ void k_dt_velocity(Geom g, DevInfo* info, double dtmax) {
  double umax = sqrt(info->umax2), vmax = sqrt(info->vmax2), wmax = sqrt(info->wmax2);
  if (umax == 0) umax = f4(1.E-15f);
  if (vmax == 0) vmax = f4(1.E-15f);
  if (wmax == 0) wmax = f4(1.E-15f);
  double Lx = (double)g.Nx * g.dx, Ly = (double)g.Ny * g.dy, Lz = (double)g.nzp * g.dz;
  double dtv = fmin(Lx / umax, fmin(Ly / vmax, Lz / wmax));
  if (dtmax > dtv) {
    info->dtm = dtv;
    info->limiter = 1;
  } else {
    info->dtm = dtmax;
    info->limiter = 0;
  }
}
__global__ void k_dt_vorticity(DevInfo* info, double prefactor, double dtmax) {
  double omax = sqrt(info->omax2);
  double dtw = (omax > 0.) ? prefactor / omax : dtmax;
  if (info->dtm > dtw) {
    info->dtm = dtw;
    info->limiter = 2;
  }
}

}  // namespace

// Host-computed Thomas factors of diffz (no bot/top, and bot/top variants).
int diffz_coef(pmpic_ctx* ctx, bool bt, std::vector<double>& out) {
  const int nz = ctx->g.nzp;
  const double a0 = 0., b0 = 1., c0 = 0.;
  const double a1 = f4div(1.f, 6.f), b1 = f4div(2.f, 3.f), c1 = f4div(1.f, 6.f);
  const double an = 0., bn = 1., cn = 0.;
  const double al = f4div(1.f, 3.f), cl = f4div(1.f, 3.f);
  std::vector<double> A(nz), B(nz), C(nz);
  A[0] = a0; B[0] = b0; C[0] = c0;
  for (int k = 1; k < nz - 1; ++k) { A[k] = a1; B[k] = b1; C[k] = c1; }
  A[nz - 1] = an; B[nz - 1] = bn; C[nz - 1] = cn;
  if (bt) { C[0] = cl; A[nz - 1] = al; }
  out.assign(3 * nz, 0.0);
  double den = B[0];
  out[nz + 0] = den;
  for (int i = 1; i < nz; ++i) {
    double cp = C[i - 1] / den;
    den = B[i] - A[i] * cp;
    if (den == 0) return set_error(ctx, PMPIC_ERR_ZERO_PIVOT, "zero pivot in tridiagonal solver (diffz)");
    out[2 * nz + i] = cp;
    out[nz + i] = den;
  }
  for (int i = 0; i < nz; ++i) out[i] = A[i];
  return 0;
}


// The Thomas factors of laplinv (fft_ops.F90:505-601, :620-656) per boundary
// form, level and wavenumber mode (a, b), from the k2 of the mode's columns:
// the pivots den(k) and the ratios cp(k) = c(k-1) / den(k-1) of the
// sequential recurrence, with the coefficients and the operation order of
// k_laplinv (FP64: the same IEEE operations, so the device's FP64 solve keeps
// its bits; FP32 form: 1/den and cp rounded to FP32).  Layout per form:
// den[nz][nmodes], then cp[nz][nmodes].  A zero pivot is the reference's
// abort (:642-645).
int laplinv_tables(pmpic_ctx* ctx, const double* k2cols) {
  const Geom& g = ctx->g;
  const int nz = g.nzp, mx = g.sx / 2, my = g.sy / 2, nmode = mx * my;
  const double f16 = f4div(1.f, 6.f), f13 = f4div(1.f, 3.f), f112 = f4div(1.f, 12.f), f56 = f4div(5.f, 6.f);
  const double dz = g.dz;
  const double i2dz2 = 2.0 / dz / dz, idz2 = 1.0 / dz / dz;
  const size_t per_form = 2 * (size_t)nz * nmode;
  std::vector<double> tab(2 * per_form, 0.0);
  for (int form = 0; form < 2; ++form) {
    double* DEN = tab.data() + form * per_form;
    double* CP = DEN + (size_t)nz * nmode;
    for (int b = 0; b < my; ++b)
      for (int a = 0; a < mx; ++a) {
        const int m = b * mx + a;
        const double kk = k2cols[(size_t)(2 * b) * g.sx + 2 * a];
        const double ai = idz2 - f112 * kk, bi = -i2dz2 - f56 * kk, ci = idz2 - f112 * kk;
        double b1, c1, an, bn;
        if (!form) {
          b1 = 1.0; c1 = 0.0; an = 0.0; bn = 1.0;
        } else {
          b1 = -idz2 - f13 * kk;
          c1 = idz2 - f16 * kk;
          an = idz2 - f16 * kk;
          bn = -idz2 - f13 * kk;
        }
        double den = b1, cprev = c1;
        DEN[m] = den;
        for (int k = 1; k < nz; ++k) {
          const double ak = k < nz - 1 ? ai : an, bk = k < nz - 1 ? bi : bn, ck = k < nz - 1 ? ci : 0.0;
          const double cp = cprev / den;
          den = bk - ak * cp;
          if (den == 0 && kk != 0)
            return set_error(ctx, PMPIC_ERR_ZERO_PIVOT, "zero pivot in tridiagonal solver (laplinv)");
          CP[(size_t)k * nmode + m] = cp;
          DEN[(size_t)k * nmode + m] = den;
          cprev = ck;
        }
      }
  }
  if (!ctx->mixed) {
    PMPIC_CUDA(cudaMalloc(&ctx->lapcp, sizeof(double) * tab.size()));
    PMPIC_CUDA(cudaMemcpy(ctx->lapcp, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    return 0;
  }
  std::vector<float> t32(tab.size());
  for (int form = 0; form < 2; ++form)
    for (size_t i = 0; i < per_form; ++i) {
      const size_t e = form * per_form + i;
      t32[e] = i < (size_t)nz * nmode ? (float)(1.0 / tab[e]) : (float)tab[e];
    }
  PMPIC_CUDA(cudaMalloc(&ctx->lapcp, sizeof(float) * t32.size()));
  PMPIC_CUDA(cudaMemcpy(ctx->lapcp, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice));
  return 0;
}

namespace f64 {
using real = double;
inline const double* tab_kx(pmpic_ctx* c) { return c->kx; }
inline const double* tab_ky(pmpic_ctx* c) { return c->ky; }
inline const double* tab_k2(pmpic_ctx* c) { return c->k2; }
inline const double* tab_filt(pmpic_ctx* c) { return c->filt; }
inline const double* tab_diffz(pmpic_ctx* c, int which) { return c->sscratch + c->g.nspec + which * 3 * c->g.nzp; }
inline void zero_mode_prepare(pmpic_ctx*) {}
// the mean flow from the columns kx = ky = 0 of the filtered a and b
// (vort2vel.F90:230-241); a, b are the unfiltered spectra
inline int zero_mode_launch(pmpic_ctx* ctx, const double* a, const double* b) {
  const Geom& g = ctx->g;
  k_zmode<<<1, 256, sizeof(double) * 4 * g.nzp, ctx->stream>>>(g, a, b, (int64_t)g.sx * g.sy, ctx->filt, ctx->zmode); ++ctx->nlaunch;
  return 0;
}
#include "spectral_impl.cuh"
}  // namespace f64

namespace f32 {
using real = float;
inline const float* tab_kx(pmpic_ctx* c) { return c->wn32; }
inline const float* tab_ky(pmpic_ctx* c) { return c->wn32 + (size_t)c->g.sx * c->g.sy; }
inline const float* tab_k2(pmpic_ctx* c) { return c->wn32 + 2 * (size_t)c->g.sx * c->g.sy; }
inline const float* tab_filt(pmpic_ctx* c) { return c->wn32 + 3 * (size_t)c->g.sx * c->g.sy; }
inline const float* tab_diffz(pmpic_ctx* c, int which) { return c->wn32 + 4 * (size_t)c->g.sx * c->g.sy + which * 3 * c->g.nzp; }
// the zero mode stays FP64: horizontal sums of the gridded p and q taken in
// FP64 before the FP32 transforms, then the FP64 mean-flow integral
inline void zero_mode_prepare(pmpic_ctx* ctx) {
  const Geom& g = ctx->g;
  k_hsum2<<<g.nzp, 256, 0, ctx->stream>>>(g, (const float*)ctx->grid[PMPIC_GRID_P], (const float*)ctx->grid[PMPIC_GRID_Q],
                                          ctx->hsum); ++ctx->nlaunch;
}
inline int zero_mode_launch(pmpic_ctx* ctx, const float*, const float*) {
  const Geom& g = ctx->g;
  k_zmode<<<1, 256, sizeof(double) * 4 * g.nzp, ctx->stream>>>(g, ctx->hsum, ctx->hsum + g.nzp, 1, nullptr, ctx->zmode); ++ctx->nlaunch;
  return 0;
}
#include "spectral_impl.cuh"
}  // namespace f32

int spectral_init(pmpic_ctx* ctx) {
  std::vector<double> c0, c1;
  int rc = diffz_coef(ctx, false, c0);
  if (rc) return rc;
  rc = diffz_coef(ctx, true, c1);
  if (rc) return rc;
  const Geom& g = ctx->g;
  double* coef = ctx->sscratch + g.nspec;
  PMPIC_CUDA(cudaMemcpy(coef, c0.data(), sizeof(double) * c0.size(), cudaMemcpyHostToDevice));
  PMPIC_CUDA(cudaMemcpy(coef + 3 * g.nzp, c1.data(), sizeof(double) * c1.size(), cudaMemcpyHostToDevice));
  // FP32 copies of the wavenumber tables and the diffz factors (mixed-precision form)
  const size_t cols = (size_t)g.sx * g.sy;
  std::vector<double> tabs(4 * cols);
  PMPIC_CUDA(cudaMemcpy(tabs.data(), ctx->kx, sizeof(double) * cols, cudaMemcpyDeviceToHost));
  PMPIC_CUDA(cudaMemcpy(tabs.data() + cols, ctx->ky, sizeof(double) * cols, cudaMemcpyDeviceToHost));
  PMPIC_CUDA(cudaMemcpy(tabs.data() + 2 * cols, ctx->k2, sizeof(double) * cols, cudaMemcpyDeviceToHost));
  PMPIC_CUDA(cudaMemcpy(tabs.data() + 3 * cols, ctx->filt, sizeof(double) * cols, cudaMemcpyDeviceToHost));
  std::vector<float> t32(4 * cols + 6 * (size_t)g.nzp);
  for (size_t i = 0; i < 4 * cols; ++i) t32[i] = (float)tabs[i];
  // diffz factors: a, the reciprocal pivots (from the FP64 recurrence), cp
  const int nz = g.nzp;
  for (int v = 0; v < 2; ++v) {
    const std::vector<double>& c = v ? c1 : c0;
    for (int i = 0; i < 3 * nz; ++i)
      t32[4 * cols + (size_t)v * 3 * nz + i] = (i >= nz && i < 2 * nz) ? (float)(1.0 / c[i]) : (float)c[i];
  }
  PMPIC_CUDA(cudaMalloc(&ctx->wn32, sizeof(float) * t32.size()));
  PMPIC_CUDA(cudaMemcpy(ctx->wn32, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice));
  PMPIC_CUDA(cudaMalloc(&ctx->hsum, sizeof(double) * 2 * g.nzp));
  return laplinv_tables(ctx, tabs.data() + 2 * cols);
}

int spec_diffx(pmpic_ctx* ctx, const double* in, double* out) { return f64::spec_diffx_impl(ctx, in, out); }
int spec_diffy(pmpic_ctx* ctx, const double* in, double* out) { return f64::spec_diffy_impl(ctx, in, out); }
int spec_filter(pmpic_ctx* ctx, const double* in, double* out) { return f64::spec_filter_impl(ctx, in, out); }
int spec_diffz(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top) {
  return f64::spec_diffz_impl(ctx, in, out, bot, top);
}
int spec_laplinv(pmpic_ctx* ctx, double* inout, bool df0) { return f64::spec_laplinv_impl(ctx, inout, df0); }

// vort2vel.F90:139-320 and vorticity_tendency.F90:147-265 in the context's precision
int vort2vel_spectral(pmpic_ctx* ctx) {
  return ctx->mixed ? f32::vort2vel_spectral_impl(ctx) : f64::vort2vel_spectral_impl(ctx);
}
int vorticity_tendency_grids(pmpic_ctx* ctx) {
  return ctx->mixed ? f32::vorticity_tendency_grids_impl(ctx) : f64::vorticity_tendency_grids_impl(ctx);
}
// maxima for the dt rule; v2v: velocity limit, vt: vorticity limit
int field_max(pmpic_ctx* ctx, bool v2v, bool vt) {
  int rc = ctx->mixed ? f32::field_max_impl(ctx, v2v, vt) : f64::field_max_impl(ctx, v2v, vt);
  if (rc) return rc;
  if (v2v) {
    k_dt_velocity<<<1, 1, 0, ctx->stream>>>(ctx->g, ctx->dinfo, ctx->cfg.dtmax); ++ctx->nlaunch;
  }
  if (vt) {
    k_dt_vorticity<<<1, 1, 0, ctx->stream>>>(ctx->dinfo, ctx->cfg.timestep_prefactor, ctx->cfg.dtmax); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
