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

// ---- elementwise spectral operators --------------------------------------------
// diffx (fft_ops.F90:266-295): out(i) = -in(i+1) kx, out(i+1) = in(i) kx
__device__ __forceinline__ double dx_of(const double* in, int64_t e, int ip, const double* kx, int col) {
  return (ip & 1) == 0 ? (-1. * in[e + 1]) * kx[col] : in[e - 1] * kx[col];
}
// diffy (fft_ops.F90:366-394)
__device__ __forceinline__ double dy_of(const double* in, int64_t e, int jp, int sx, const double* ky, int col) {
  return (jp & 1) == 0 ? (-1. * in[e + sx]) * ky[col] : in[e - sx] * ky[col];
}

struct EwIdx {
  int64_t e;
  int col, ip, jp, k;
};
__device__ __forceinline__ bool ew_index(const Geom& g, EwIdx& x) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.nspec) return false;
  int cols = g.sx * g.sy;
  x.e = e;
  x.k = (int)(e / cols);
  x.col = (int)(e - (int64_t)x.k * cols);
  x.jp = x.col / g.sx;
  x.ip = x.col - x.jp * g.sx;
  return true;
}

__global__ void k_diffx(Geom g, const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ kx) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = dx_of(in, x.e, x.ip, kx, x.col);
}
__global__ void k_diffy(Geom g, const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ ky) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = dy_of(in, x.e, x.jp, g.sx, ky, x.col);
}
__global__ void k_filter(Geom g, const double* __restrict__ in, double* __restrict__ out,
                         const double* __restrict__ filt) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = in[x.e] * filt[x.col];
}

// vort2vel.F90:158-173: f = diffx(a) + diffy(b) + (dc/dz, 2nd order with
// one-sided ends); f(:,1,1) = 0
__global__ void k_div(Geom g, const double* __restrict__ a, const double* __restrict__ b,
                      const double* __restrict__ c, double* __restrict__ f, const double* __restrict__ kx,
                      const double* __restrict__ ky, double hdzi) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  const int64_t cs = (int64_t)g.sx * g.sy;
  const int nz = g.nzp;
  double d = dx_of(a, x.e, x.ip, kx, x.col);
  double e = dy_of(b, x.e, x.jp, g.sx, ky, x.col);
  double fz;
  if (x.k == 0) {
    fz = hdzi * (4. * c[x.e + cs] - c[x.e + 2 * cs] - 3. * c[x.e]);
  } else if (x.k == nz - 1) {
    fz = hdzi * (c[x.e - 2 * cs] + 3. * c[x.e] - 4. * c[x.e - cs]);
  } else {
    fz = (c[x.e + cs] - c[x.e - cs]) * hdzi;
  }
  double v = d + e + fz;
  if (x.col == 0) v = 0.0;
  f[x.e] = v;
}

// a = a - diffx(f) (vort2vel.F90:185-188) or b = b - diffy(f) (:191-194)
__global__ void k_sub_diff(Geom g, double* __restrict__ a, const double* __restrict__ f, const double* __restrict__ kk,
                           int ydir) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  double d = ydir ? dy_of(f, x.e, x.jp, g.sx, kk, x.col) : dx_of(f, x.e, x.ip, kk, x.col);
  a[x.e] = a[x.e] - d;
}

// c = c - d; c(1,:,:) = 0 (vort2vel.F90:197-205)
__global__ void k_sub_zero0(Geom g, double* __restrict__ c, const double* __restrict__ d) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  double v = c[x.e] - d[x.e];
  if (x.k == 0) v = 0.;
  c[x.e] = v;
}

// d,e,f = filter(a,b,c) and the top/bottom planes of a and b (vort2vel.F90:208-217)
__global__ void k_filter3_bt(Geom g, const double* __restrict__ a, const double* __restrict__ b,
                             const double* __restrict__ c, double* __restrict__ d, double* __restrict__ e,
                             double* __restrict__ f, const double* __restrict__ filt, double* __restrict__ bt) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  double m = filt[x.col];
  d[x.e] = a[x.e] * m;
  e[x.e] = b[x.e] * m;
  f[x.e] = c[x.e] * m;
  const int cols = g.sx * g.sy;
  if (x.k == g.nzp - 1) {
    bt[0 * cols + x.col] = a[x.e];  // atop
    bt[2 * cols + x.col] = b[x.e];  // btop
  }
  if (x.k == 0) {
    bt[1 * cols + x.col] = a[x.e];  // abot
    bt[3 * cols + x.col] = b[x.e];  // bbot
  }
}

// Velocity components from the potentials (vort2vel.F90:254-315):
//  mode 0: f = e - diffy(c), f(:,1,1) = ubar, u_s = filter(f)
//  mode 1: f = diffx(c) - e, f(:,1,1) = vbar, v_s = filter(f)
//  mode 2: f = diffy(a) - diffx(b),             w_s = filter(f)
__global__ void k_vel(Geom g, int mode, const double* __restrict__ e, const double* __restrict__ c,
                      const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ f,
                      double* __restrict__ fs, const double* __restrict__ kx, const double* __restrict__ ky,
                      const double* __restrict__ filt, const double* __restrict__ zbar) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  double v;
  if (mode == 0) {
    v = e[x.e] - dy_of(c, x.e, x.jp, g.sx, ky, x.col);
    if (x.col == 0) v = zbar[x.k];
  } else if (mode == 1) {
    v = dx_of(c, x.e, x.ip, kx, x.col) - e[x.e];
    if (x.col == 0) v = zbar[x.k];
  } else {
    v = dy_of(a, x.e, x.jp, g.sx, ky, x.col) - dx_of(b, x.e, x.ip, kx, x.col);
  }
  f[x.e] = v;
  fs[x.e] = v * filt[x.col];
}

// mean flow of the zero mode (vort2vel.F90:230-241), one thread: the trapezoid
// integral and the reference's average (`1./nz` in REAL(4), 0.5*ubar(nz) added
// to every element before the sum).
__global__ void k_zmode(Geom g, const double* __restrict__ d, const double* __restrict__ e,
                        double* __restrict__ zb) {
  extern __shared__ double zs[];  // e(:,1,1), d(:,1,1), then ubar, vbar
  const int nz = g.nzp;
  const int64_t cs = (int64_t)g.sx * g.sy;
  double* es = zs;
  double* ds = zs + nz;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {  // stage the zero-mode columns
    es[k] = e[k * cs];
    ds[k] = d[k * cs];
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

// ---- compact z operators ----------------------------------------------------------
// diffz (fft_ops.F90:419-483).  The tridiagonal coefficients are the same for
// every column, so the Thomas factors (cp and the denominators) are computed
// once on the host with the reference's arithmetic and passed in.
__global__ void k_diffz(Geom g, const double* __restrict__ f, double* __restrict__ out,
                        const double* __restrict__ coef /* a[nz], den[nz], cp[nz] */, const double* __restrict__ bot,
                        const double* __restrict__ top, double a1) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int cols = g.sx * g.sy;
  if (col >= cols) return;
  const int nz = g.nzp;
  const int64_t cs = cols;
  const double* A = coef;
  const double* DEN = coef + nz;
  const double* CP = coef + 2 * nz;
  const double dz = g.dz;
  const bool bt = bot != nullptr;
  // forward sweep: f'(1) = d(1)/den(1); f'(i) = (d(i) - a(i) f'(i-1)) / den(i)
  double fm = f[col], f0 = f[cs + col];
  double d1 = bt ? f0 / dz - a1 * bot[col] * dz : 0.0;
  double prev = d1 / DEN[0];
  out[col] = prev;
  for (int k = 1; k < nz - 1; ++k) {
    double fp = f[(int64_t)(k + 1) * cs + col];
    double d = (fp - fm) / 2. / dz;
    prev = (d - A[k] * prev) / DEN[k];
    out[(int64_t)k * cs + col] = prev;
    fm = f0;
    f0 = fp;
  }
  {
    int k = nz - 1;
    double dn = bt ? -fm / dz + a1 * top[col] * dz : 0.0;  // fm = f(nz-1)
    prev = (dn - A[k] * prev) / DEN[k];
    out[(int64_t)k * cs + col] = prev;
  }
  // back substitution: f(i) = f(i) - cp(i+1) f(i+1)
  double nxt = prev;
  for (int k = nz - 2; k >= 0; --k) {
    double v = out[(int64_t)k * cs + col] - CP[k + 1] * nxt;
    out[(int64_t)k * cs + col] = v;
    nxt = v;
  }
}

// laplinv (fft_ops.F90:505-601), in place, one thread per column; columns with
// k2 == 0 keep their input (:567).  cp is kept in a scratch array.
__global__ void k_laplinv(Geom g, double* __restrict__ f, double* __restrict__ cpbuf, const double* __restrict__ k2,
                          int df0) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int cols = g.sx * g.sy;
  if (col >= cols) return;
  const double kk = k2[col];
  if (kk == 0) return;
  const int nz = g.nzp;
  const int64_t cs = cols;
  const double f16 = f4div(1.f, 6.f), f13 = f4div(1.f, 3.f), f112 = f4div(1.f, 12.f), f56 = f4div(5.f, 6.f);
  const double dz = g.dz;
  const double i2dz2 = 2. / dz / dz;
  const double idz2 = 1. / dz / dz;
  const double ai = idz2 - f112 * kk, bi = -i2dz2 - f56 * kk, ci = idz2 - f112 * kk;
  double b1, c1, an, bn;
  double fm, f0, fp;
  f0 = f[col];
  fp = f[cs + col];
  double d;
  if (!df0) {
    b1 = 1.; c1 = 0.; d = 0.;
    an = 0.; bn = 1.;
  } else {
    b1 = -idz2 - f13 * kk;
    c1 = idz2 - f16 * kk;
    d = f13 * f0 + f16 * fp;
    an = idz2 - f16 * kk;
    bn = -idz2 - f13 * kk;
  }
  // tridiagonal (fft_ops.F90:620-656)
  double den = b1;
  double prev = d / den;
  f[col] = prev;
  double cprev = c1;  // c(i-1)
  for (int k = 1; k < nz; ++k) {
    fm = f0;
    f0 = fp;
    double a, b, c;
    if (k < nz - 1) {
      fp = f[(int64_t)(k + 1) * cs + col];
      a = ai; b = bi; c = ci;
      d = f112 * fm + f56 * f0 + f112 * fp;
    } else {
      a = an; b = bn; c = 0.;
      d = df0 ? f13 * f0 + f16 * fm : 0.;
    }
    double cp = cprev / den;
    den = b - a * cp;
    prev = (d - a * prev) / den;
    f[(int64_t)k * cs + col] = prev;
    cpbuf[(int64_t)k * cs + col] = cp;
    cprev = c;
  }
  double nxt = prev;
  for (int k = nz - 2; k >= 0; --k) {
    double v = f[(int64_t)k * cs + col] - cpbuf[(int64_t)(k + 1) * cs + col] * nxt;
    f[(int64_t)k * cs + col] = v;
    nxt = v;
  }
}

// ---- vorticity tendency pointwise combinations (vorticity_tendency.F90:169-265)
__global__ void k_pw_add_mul(int64_t n, double* __restrict__ o, const double* __restrict__ a,
                             const double* __restrict__ b) {  // o = o + a*b
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) o[e] = o[e] + a[e] * b[e];
}
__global__ void k_pw_add_mul_sum(int64_t n, double* __restrict__ o, const double* __restrict__ r,
                                 const double* __restrict__ q, const double* __restrict__ w) {  // o = o + r*(q + w)
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) o[e] = o[e] + r[e] * (q[e] + w[e]);
}
__global__ void k_pw_neg_add_mul(int64_t n, double* __restrict__ o, const double* __restrict__ a,
                                 const double* __restrict__ b) {  // o = -o + a*b
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) o[e] = -o[e] + a[e] * b[e];
}
__global__ void k_pw_add_mul_negsum(int64_t n, double* __restrict__ o, const double* __restrict__ r,
                                    const double* __restrict__ p, const double* __restrict__ w) {  // o = o + r*(-p + w)
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) o[e] = o[e] + r[e] * (-p[e] + w[e]);
}
__global__ void k_pw_dr(int64_t n, double* __restrict__ dr, const double* __restrict__ p,
                        const double* __restrict__ q, const double* __restrict__ r, const double* __restrict__ dwdx,
                        const double* __restrict__ dwdy, const double* __restrict__ dudx,
                        const double* __restrict__ dvdy) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double v = p[e] * dwdx[e];
  v = v + q[e] * dwdy[e];
  v = v + r[e] * (-dudx[e]);
  v = v + r[e] * (-dvdy[e]);
  dr[e] = v;
}

// max of squares over the interior (vort2vel.F90:331-338,
// vorticity_tendency.F90:279-282); non-negative doubles order like their bits
__global__ void k_max_sq3(int64_t n, const double* __restrict__ u, const double* __restrict__ v,
                          const double* __restrict__ w, double* __restrict__ out3) {
  double mu = 0, mv = 0, mw = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double a = u[e], b = v[e], c = w[e];
    mu = fmax(mu, a * a);
    mv = fmax(mv, b * b);
    mw = fmax(mw, c * c);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_down_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_down_sync(0xffffffffu, mv, o));
    mw = fmax(mw, __shfl_down_sync(0xffffffffu, mw, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax((unsigned long long*)&out3[0], __double_as_longlong(mu));
    atomicMax((unsigned long long*)&out3[1], __double_as_longlong(mv));
    atomicMax((unsigned long long*)&out3[2], __double_as_longlong(mw));
  }
}
__global__ void k_max_vort(int64_t n, const double* __restrict__ p, const double* __restrict__ q,
                           const double* __restrict__ r, double* __restrict__ out) {
  double m = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double a = p[e], b = q[e], c = r[e];
    m = fmax(m, a * a + b * b + c * c);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)out, __double_as_longlong(m));
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
static int diffz_coef(pmpic_ctx* ctx, bool bt, std::vector<double>& out) {
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

static int diffz_launch(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top) {
  TimerScope ts(ctx, T_DIFFZ);
  const Geom& g = ctx->g;
  int which = bot ? 1 : 0;
  double* coef = ctx->sscratch + g.nspec;  // 2 x 3*nzp doubles after the cp scratch
  coef += which * 3 * g.nzp;
  k_diffz<<<nblk((int64_t)g.sx * g.sy, 128), 128, 0, ctx->stream>>>(g, in, out, coef, bot, top, f4div(1.f, 6.f)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

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
  return 0;
}

int spec_diffx(pmpic_ctx* ctx, const double* in, double* out) {
  k_diffx<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, ctx->kx); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_diffy(pmpic_ctx* ctx, const double* in, double* out) {
  k_diffy<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, ctx->ky); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_filter(pmpic_ctx* ctx, const double* in, double* out) {
  k_filter<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, ctx->filt); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_diffz(pmpic_ctx* ctx, const double* in, double* out, const double* bot, const double* top) {
  return diffz_launch(ctx, in, out, bot, top);
}
int spec_laplinv(pmpic_ctx* ctx, double* inout, bool df0) {
  TimerScope ts(ctx, T_LAPLINV);
  const Geom& g = ctx->g;
  k_laplinv<<<nblk((int64_t)g.sx * g.sy, 128), 128, 0, ctx->stream>>>(g, inout, ctx->sscratch, ctx->k2, df0 ? 1 : 0); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// vort2vel.F90:139-320 after the three par2grid calls (grids P, Q, R hold the
// gridded vorticity on entry; on exit they hold the corrected, filtered
// vorticity, U, V, W the velocity and u_s, v_s, w_s its filtered spectra).
int vort2vel_spectral(pmpic_ctx* ctx) {
  const Geom& g = ctx->g;
  int rc;
  double *a = ctx->sa, *b = ctx->sb, *c = ctx->sc, *d = ctx->sd, *e = ctx->se, *f = ctx->sf;
  const unsigned nb = nblk(g.nspec, 256);
  const int cols = g.sx * g.sy;
  if ((rc = fft_forward(ctx, ctx->grid[PMPIC_GRID_P], a))) return rc;
  if ((rc = fft_forward(ctx, ctx->grid[PMPIC_GRID_Q], b))) return rc;
  if ((rc = fft_forward(ctx, ctx->grid[PMPIC_GRID_R], c))) return rc;
  const double hdzi = f4div(1.f, 2.f) / g.dz;
  k_div<<<nb, 256, 0, ctx->stream>>>(g, a, b, c, f, ctx->kx, ctx->ky, hdzi); ++ctx->nlaunch;
  if ((rc = spec_laplinv(ctx, f, true))) return rc;
  k_filter<<<nb, 256, 0, ctx->stream>>>(g, f, f, ctx->filt); ++ctx->nlaunch;
  k_sub_diff<<<nb, 256, 0, ctx->stream>>>(g, a, f, ctx->kx, 0); ++ctx->nlaunch;
  k_sub_diff<<<nb, 256, 0, ctx->stream>>>(g, b, f, ctx->ky, 1); ++ctx->nlaunch;
  if ((rc = diffz_launch(ctx, f, d, nullptr, nullptr))) return rc;
  k_sub_zero0<<<nb, 256, 0, ctx->stream>>>(g, c, d); ++ctx->nlaunch;
  k_filter3_bt<<<nb, 256, 0, ctx->stream>>>(g, a, b, c, d, e, f, ctx->filt, ctx->bt); ++ctx->nlaunch;
  if ((rc = fft_backward(ctx, d, ctx->grid[PMPIC_GRID_P]))) return rc;
  if ((rc = fft_backward(ctx, e, ctx->grid[PMPIC_GRID_Q]))) return rc;
  if ((rc = fft_backward(ctx, f, ctx->grid[PMPIC_GRID_R]))) return rc;
  k_zmode<<<1, 256, sizeof(double) * 4 * g.nzp, ctx->stream>>>(g, d, e, ctx->zmode); ++ctx->nlaunch;
  if ((rc = spec_laplinv(ctx, a, false))) return rc;
  if ((rc = spec_laplinv(ctx, b, false))) return rc;
  if ((rc = spec_laplinv(ctx, c, true))) return rc;
  const double* atop = ctx->bt;
  const double* abot = ctx->bt + cols;
  const double* btop = ctx->bt + 2 * cols;
  const double* bbot = ctx->bt + 3 * cols;
  // u = dB/dz - dC/dy
  if ((rc = diffz_launch(ctx, b, e, bbot, btop))) return rc;
  k_vel<<<nb, 256, 0, ctx->stream>>>(g, 0, e, c, a, b, f, ctx->spec[PMPIC_SPEC_U], ctx->kx, ctx->ky, ctx->filt,
                                     ctx->zmode); ++ctx->nlaunch;
  if ((rc = fft_backward(ctx, f, ctx->grid[PMPIC_GRID_U]))) return rc;
  // v = dC/dx - dA/dz
  if ((rc = diffz_launch(ctx, a, e, abot, atop))) return rc;
  k_vel<<<nb, 256, 0, ctx->stream>>>(g, 1, e, c, a, b, f, ctx->spec[PMPIC_SPEC_V], ctx->kx, ctx->ky, ctx->filt,
                                     ctx->zmode + g.nzp); ++ctx->nlaunch;
  if ((rc = fft_backward(ctx, f, ctx->grid[PMPIC_GRID_V]))) return rc;
  // w = dA/dy - dB/dx
  k_vel<<<nb, 256, 0, ctx->stream>>>(g, 2, e, c, a, b, f, ctx->spec[PMPIC_SPEC_W], ctx->kx, ctx->ky, ctx->filt,
                                     ctx->zmode); ++ctx->nlaunch;
  if ((rc = fft_backward(ctx, f, ctx->grid[PMPIC_GRID_W]))) return rc;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// vorticity_tendency.F90:147-265 (grid B holds par2grid(btot) on entry).
int vorticity_tendency_grids(pmpic_ctx* ctx) {
  const Geom& g = ctx->g;
  int rc;
  double *bs = ctx->sbs, *as = ctx->sas;
  double *DP = ctx->grid[PMPIC_GRID_DP], *DQ = ctx->grid[PMPIC_GRID_DQ], *DR = ctx->grid[PMPIC_GRID_DR];
  const double *P = ctx->grid[PMPIC_GRID_P], *Q = ctx->grid[PMPIC_GRID_Q], *R = ctx->grid[PMPIC_GRID_R];
  double *dudx = ctx->gwork[0], *dwdx = ctx->gwork[1], *dvdy = ctx->gwork[2], *dwdy = ctx->gwork[3];
  double* ap = ctx->gwork[4];
  const int64_t n = g.nphys;
  const unsigned nb = nblk(n, 256);
  if ((rc = fft_forward(ctx, ctx->grid[PMPIC_GRID_B], bs))) return rc;
  if ((rc = spec_diffy(ctx, bs, as))) return rc;
  if ((rc = fft_backward(ctx, as, DP))) return rc;
  if ((rc = spec_diffx(ctx, ctx->spec[PMPIC_SPEC_U], as))) return rc;
  if ((rc = fft_backward(ctx, as, dudx))) return rc;
  k_pw_add_mul<<<nb, 256, 0, ctx->stream>>>(n, DP, P, dudx); ++ctx->nlaunch;
  if ((rc = spec_diffy(ctx, ctx->spec[PMPIC_SPEC_U], as))) return rc;
  if ((rc = fft_backward(ctx, as, ap))) return rc;
  k_pw_add_mul<<<nb, 256, 0, ctx->stream>>>(n, DP, Q, ap); ++ctx->nlaunch;
  if ((rc = spec_diffx(ctx, ctx->spec[PMPIC_SPEC_W], as))) return rc;
  if ((rc = fft_backward(ctx, as, dwdx))) return rc;
  k_pw_add_mul_sum<<<nb, 256, 0, ctx->stream>>>(n, DP, R, Q, dwdx); ++ctx->nlaunch;
  if ((rc = spec_diffx(ctx, bs, as))) return rc;
  if ((rc = fft_backward(ctx, as, DQ))) return rc;
  if ((rc = spec_diffx(ctx, ctx->spec[PMPIC_SPEC_V], as))) return rc;
  if ((rc = fft_backward(ctx, as, ap))) return rc;
  k_pw_neg_add_mul<<<nb, 256, 0, ctx->stream>>>(n, DQ, P, ap); ++ctx->nlaunch;
  if ((rc = spec_diffy(ctx, ctx->spec[PMPIC_SPEC_V], as))) return rc;
  if ((rc = fft_backward(ctx, as, dvdy))) return rc;
  k_pw_add_mul<<<nb, 256, 0, ctx->stream>>>(n, DQ, Q, dvdy); ++ctx->nlaunch;
  if ((rc = spec_diffy(ctx, ctx->spec[PMPIC_SPEC_W], as))) return rc;
  if ((rc = fft_backward(ctx, as, dwdy))) return rc;
  k_pw_add_mul_negsum<<<nb, 256, 0, ctx->stream>>>(n, DQ, R, P, dwdy); ++ctx->nlaunch;
  k_pw_dr<<<nb, 256, 0, ctx->stream>>>(n, DR, P, Q, R, dwdx, dwdy, dudx, dvdy); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// maxima for the dt rule; v2v: velocity limit, vt: vorticity limit
int field_max(pmpic_ctx* ctx, bool v2v, bool vt) {
  const Geom& g = ctx->g;
  if (v2v) {
    PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->umax2, 0, 3 * sizeof(double), ctx->stream));
    k_max_sq3<<<592, 256, 0, ctx->stream>>>(g.nphys, ctx->grid[PMPIC_GRID_U], ctx->grid[PMPIC_GRID_V],
                                            ctx->grid[PMPIC_GRID_W], &ctx->dinfo->umax2); ++ctx->nlaunch;
    k_dt_velocity<<<1, 1, 0, ctx->stream>>>(g, ctx->dinfo, ctx->cfg.dtmax); ++ctx->nlaunch;
  }
  if (vt) {
    PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->omax2, 0, sizeof(double), ctx->stream));
    k_max_vort<<<592, 256, 0, ctx->stream>>>(g.nphys, ctx->grid[PMPIC_GRID_P], ctx->grid[PMPIC_GRID_Q],
                                             ctx->grid[PMPIC_GRID_R], &ctx->dinfo->omax2); ++ctx->nlaunch;
    k_dt_vorticity<<<1, 1, 0, ctx->stream>>>(ctx->dinfo, ctx->cfg.timestep_prefactor, ctx->cfg.dtmax); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
