// spectral_impl.cuh -- the semi-spectral operators and the vort2vel /
// vorticity_tendency grid pipelines of spectral.cu, written once over the
// scalar type `real` and included by spectral.cu into one namespace per
// precision (FP64 plain path, FP32 mixed-precision form).  The namespace
// provides the tables of its precision (tab_kx, tab_ky, tab_k2, tab_filt,
// tab_diffz) and the zero-mode hooks (zero_mode_prepare, zero_mode_launch).
// Not a standalone header.

template <class P>
inline real* RP(P* p) { return reinterpret_cast<real*>(p); }

// ---- elementwise spectral operators --------------------------------------------
// The wavenumber tables are laid out like a spectral level, but kx depends on
// the x index ip alone and ky on the row jp alone: kx is read from row 0
// (kx[ip]) and ky from column 0 (ky[jp * sx]), the same values.
// diffx (fft_ops.F90:266-295): out(i) = -in(i+1) kx, out(i+1) = in(i) kx
__device__ __forceinline__ real dx_of(const real* in, int64_t e, int ip, const real* kx) {
  return (ip & 1) == 0 ? (real(-1) * in[e + 1]) * kx[ip] : in[e - 1] * kx[ip];
}
// diffy (fft_ops.F90:366-394)
__device__ __forceinline__ real dy_of(const real* in, int64_t e, int jp, int sx, const real* ky) {
  return (jp & 1) == 0 ? (real(-1) * in[e + sx]) * ky[jp * sx] : in[e - sx] * ky[jp * sx];
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

__global__ void k_diffx(Geom g, const real* __restrict__ in, real* __restrict__ out, const real* __restrict__ kx) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = dx_of(in, x.e, x.ip, kx);
}
__global__ void k_diffy(Geom g, const real* __restrict__ in, real* __restrict__ out, const real* __restrict__ ky) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = dy_of(in, x.e, x.jp, g.sx, ky);
}
__global__ void k_filter(Geom g, const real* __restrict__ in, real* __restrict__ out,
                         const real* __restrict__ filt) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  out[x.e] = in[x.e] * filt[x.col];
}

// vort2vel.F90:158-173: f = diffx(a) + diffy(b) + (dc/dz, 2nd order with
// one-sided ends); f(:,1,1) = 0
__global__ void k_div(Geom g, const real* __restrict__ a, const real* __restrict__ b,
                      const real* __restrict__ c, real* __restrict__ f, const real* __restrict__ kx,
                      const real* __restrict__ ky, real hdzi) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  const int64_t cs = (int64_t)g.sx * g.sy;
  const int nz = g.nzp;
  real d = dx_of(a, x.e, x.ip, kx);
  real e = dy_of(b, x.e, x.jp, g.sx, ky);
  real fz;
  if (x.k == 0) {
    fz = hdzi * (real(4) * c[x.e + cs] - c[x.e + 2 * cs] - real(3) * c[x.e]);
  } else if (x.k == nz - 1) {
    fz = hdzi * (c[x.e - 2 * cs] + real(3) * c[x.e] - real(4) * c[x.e - cs]);
  } else {
    fz = (c[x.e + cs] - c[x.e - cs]) * hdzi;
  }
  real v = d + e + fz;
  if (x.col == 0) v = real(0);
  f[x.e] = v;
}

// The filter and both subtractions of vort2vel.F90:179-194 in one pass:
// fo = filter(f) and a = a - diffx(fo), b = b - diffy(fo), the neighbours'
// filtered values formed as the filter forms them (f is left unfiltered; fo
// is a separate array, so no thread reads a value another one rewrote)
__global__ void k_filter_sub2(Geom g, const real* __restrict__ f, real* __restrict__ fo, real* __restrict__ a,
                              real* __restrict__ b, const real* __restrict__ kx, const real* __restrict__ ky,
                              const real* __restrict__ filt) {
  EwIdx x;
  if (!ew_index(g, x)) return;
  fo[x.e] = f[x.e] * filt[x.col];
  const real kxv = kx[x.ip], kyv = ky[x.jp * g.sx];  // (row 0, column 0: the same values)
  const real dxf = (x.ip & 1) == 0 ? (real(-1) * (f[x.e + 1] * filt[x.col + 1])) * kxv
                                   : (f[x.e - 1] * filt[x.col - 1]) * kxv;
  const real dyf = (x.jp & 1) == 0 ? (real(-1) * (f[x.e + g.sx] * filt[x.col + g.sx])) * kyv
                                   : (f[x.e - g.sx] * filt[x.col - g.sx]) * kyv;
  a[x.e] = a[x.e] - dxf;
  b[x.e] = b[x.e] - dyf;
}

// the top and bottom planes of a and b, unfiltered (vort2vel.F90:213-218)
__global__ void k_bt_planes(Geom g, const real* __restrict__ a, const real* __restrict__ b, real* __restrict__ bt) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int cols = g.sx * g.sy;
  if (col >= cols) return;
  const size_t top = (size_t)(g.nzp - 1) * cols + col;
  bt[0 * cols + col] = a[top];  // atop
  bt[1 * cols + col] = a[col];  // abot
  bt[2 * cols + col] = b[top];  // btop
  bt[3 * cols + col] = b[col];  // bbot
}

// ---- compact z operators ----------------------------------------------------------
// The z recurrences run one thread per spectral column, so only about 14 warps
// per SM are resident at 256^2 columns and a level costs the latency of its
// dependent instructions.  The Thomas factors (pivots den and ratios cp of
// fft_ops.F90:620-656) depend only on the level and, for laplinv, on the
// column's wavenumber: they are tables built once at set-up.  The FP64 path
// keeps the reference's operations bit for bit (its tables repeat the
// sequential recurrence exactly; the right-hand side is still divided by the
// pivot); the FP32 form multiplies by the reciprocal pivot (taken from the FP64
// recurrence and rounded once) and fuses the multiply-adds, so a level is two
// dependent operations.
__device__ __forceinline__ real zstep(real d, real a, real prev, real den_or_rden) {
  if constexpr (sizeof(real) == 8) return (d - a * prev) / den_or_rden;
  else return __fmaf_rn(-a, prev, d) * den_or_rden;
}
__device__ __forceinline__ real zback(real f, real cp, real nxt) {
  if constexpr (sizeof(real) == 8) return f - cp * nxt;
  else return __fmaf_rn(-cp, nxt, f);
}
__device__ __forceinline__ real zfirst(real d, real den_or_rden) {
  if constexpr (sizeof(real) == 8) return d / den_or_rden;
  else return d * den_or_rden;
}

// diffz (fft_ops.F90:419-483).  The tridiagonal coefficients are the same for
// every column, so the Thomas factors (cp and the pivots; the reciprocal
// pivots on the FP32 form) are computed once on the host with the reference's
// arithmetic and passed in.
// blockIdx.y selects one of up to two independent solves in the same launch.
struct DzBatch {
  const real* f[2];
  real* out[2];
  const real* bot[2];  // both null: no boundary values (df0 form)
  const real* top[2];
  real* sub;           // solve 0 only: c = c - diffz(f), c(1,:,:) = 0 (vort2vel.F90:196-205) in
                       // place of the final values in out
};
__global__ void k_diffz(Geom g, DzBatch zb, const real* __restrict__ coef /* a[nz], den[nz] (FP32: 1/den), cp[nz] */,
                        real a1) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int cols = g.sx * g.sy;
  if (col >= cols) return;
  const int q = blockIdx.y;  // selected without indexing the parameter arrays (no local copy)
  const real* __restrict__ f = q == 0 ? zb.f[0] : zb.f[1];
  real* __restrict__ out = q == 0 ? zb.out[0] : zb.out[1];
  const real* __restrict__ bot = q == 0 ? zb.bot[0] : zb.bot[1];
  const real* __restrict__ top = q == 0 ? zb.top[0] : zb.top[1];
  const int nz = g.nzp;
  const uint32_t cs = (uint32_t)cols;  // level offsets fit 32 bits (the spectral grid is < 2^31)
  const real* A = coef;
  const real* DEN = coef + nz;
  const real* CP = coef + 2 * nz;
  const real dz = (real)g.dz;
  const bool bt = bot != nullptr;
  // forward sweep: f'(1) = d(1)/den(1); f'(i) = (d(i) - a(i) f'(i-1)) / den(i).
  // The loads of each batch of ZB levels are issued before its recurrence, so
  // the loop waits on one memory latency per batch, not per level.
  constexpr int ZB = 8;
  real fm = f[col], f0 = f[cs + col];
  real d1 = bt ? f0 / dz - a1 * bot[col] * dz : real(0);
  real prev = zfirst(d1, DEN[0]);
  out[col] = prev;
  for (int kb = 1; kb < nz - 1; kb += ZB) {
    real fb[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u)
      if (kb + u < nz - 1) fb[u] = f[(uint32_t)(kb + u + 1) * cs + col];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int k = kb + u;
      if (k >= nz - 1) break;
      real d = (fb[u] - fm) / real(2) / dz;
      prev = zstep(d, A[k], prev, DEN[k]);
      out[(uint32_t)k * cs + col] = prev;
      fm = f0;
      f0 = fb[u];
    }
  }
  real* __restrict__ sub = q == 0 ? zb.sub : nullptr;
  {
    int k = nz - 1;
    real dn = bt ? -fm / dz + a1 * top[col] * dz : real(0);  // fm = f(nz-1)
    prev = zstep(dn, A[k], prev, DEN[k]);
    if (sub) sub[(uint32_t)k * cs + col] = sub[(uint32_t)k * cs + col] - prev;
    else out[(uint32_t)k * cs + col] = prev;
  }
  // back substitution: f(i) = f(i) - cp(i+1) f(i+1)
  real nxt = prev;
  for (int kb = nz - 2; kb >= 0; kb -= ZB) {
    real ob[ZB], sb[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u)
      if (kb - u >= 0) {
        ob[u] = out[(uint32_t)(kb - u) * cs + col];
        if (sub) sb[u] = sub[(uint32_t)(kb - u) * cs + col];  // loaded with the batch, off the chain
      }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int k = kb - u;
      if (k < 0) break;
      real v = zback(ob[u], CP[k + 1], nxt);
      if (sub) {
        sub[(uint32_t)k * cs + col] = k == 0 ? real(0) : sb[u] - v;
      } else {
        out[(uint32_t)k * cs + col] = v;
      }
      nxt = v;
    }
  }
}

// laplinv (fft_ops.F90:505-601), in place, one thread per column; columns with
// k2 == 0 keep their input (:567).  The Thomas factors of a column depend on
// its wavenumber only, shared by the four columns (2a-1..2a, 2b-1..2b) of one
// mode (a, b): tab holds, per boundary form (f0, df0), the pivots (FP32: their
// reciprocals) and then the ratios cp, each [level][mode], built at set-up
// (laplinv_tables).
// blockIdx.y selects one of up to three arrays solved in the same launch
struct LapBatch {
  real* f[3];
  int df0[3];
};
__global__ void k_laplinv(Geom g, LapBatch lb, const real* __restrict__ tab, const real* __restrict__ k2) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int cols = g.sx * g.sy;
  if (col >= cols) return;
  const int q = blockIdx.y;  // selected without indexing the parameter arrays (no local copy)
  real* __restrict__ f = q == 0 ? lb.f[0] : (q == 1 ? lb.f[1] : lb.f[2]);
  const int df0 = q == 0 ? lb.df0[0] : (q == 1 ? lb.df0[1] : lb.df0[2]);
  const real kk = k2[col];
  if (kk == 0) return;
  const int nz = g.nzp;
  const int64_t cs = cols;
  const int nmode = (g.sx >> 1) * (g.sy >> 1);
  const int jp = col / g.sx, ip = col - jp * g.sx;
  const real* __restrict__ DEN = tab + (size_t)(2 * df0) * nz * nmode + (jp >> 1) * (g.sx >> 1) + (ip >> 1);
  const real* __restrict__ CP = DEN + (size_t)nz * nmode;
  const real f16 = (real)f4div(1.f, 6.f), f13 = (real)f4div(1.f, 3.f), f112 = (real)f4div(1.f, 12.f), f56 = (real)f4div(5.f, 6.f);
  const real dz = (real)g.dz;
  const real idz2 = real(1) / dz / dz;
  const real ai = idz2 - f112 * kk;
  real an;
  real fm, f0, fp;
  f0 = f[col];
  fp = f[cs + col];
  real d;
  if (!df0) {
    d = real(0);
    an = real(0);
  } else {
    d = f13 * f0 + f16 * fp;
    an = idz2 - f16 * kk;
  }
  // tridiagonal (fft_ops.F90:620-656) with the tabulated factors
  real prev = zfirst(d, DEN[0]);
  f[col] = prev;
  // loads of each batch of ZB levels first, then its recurrence (one memory
  // latency per batch); the batch reads f above the levels it overwrites
  constexpr int ZB = sizeof(real) == 8 ? 4 : 8;  // FP64: fewer registers for the batch
  for (int kb = 1; kb < nz; kb += ZB) {
    real fb[ZB], db[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      if (kb + u < nz - 1) fb[u] = f[(int64_t)(kb + u + 1) * cs + col];
      if (kb + u < nz) db[u] = DEN[(size_t)(kb + u) * nmode];
    }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int k = kb + u;
      if (k >= nz) break;
      fm = f0;
      f0 = fp;
      real a;
      if (k < nz - 1) {
        fp = fb[u];
        a = ai;
        d = f112 * fm + f56 * f0 + f112 * fp;
      } else {
        a = an;
        d = df0 ? f13 * f0 + f16 * fm : real(0);
      }
      prev = zstep(d, a, prev, db[u]);
      f[(int64_t)k * cs + col] = prev;
    }
  }
  real nxt = prev;
  for (int kb = nz - 2; kb >= 0; kb -= ZB) {
    real fb[ZB], cb[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u)
      if (kb - u >= 0) {
        fb[u] = f[(int64_t)(kb - u) * cs + col];
        cb[u] = CP[(size_t)(kb - u + 1) * nmode];
      }
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int k = kb - u;
      if (k < 0) break;
      real v = zback(fb[u], cb[u], nxt);
      f[(int64_t)k * cs + col] = v;
      nxt = v;
    }
  }
}

// max of squares over the interior (vort2vel.F90:331-338,
// vorticity_tendency.F90:279-282); non-negative doubles order like their bits
__global__ void k_max_sq3(int64_t n, const real* __restrict__ u, const real* __restrict__ v,
                          const real* __restrict__ w, double* __restrict__ out3) {
  real mu = 0, mv = 0, mw = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    real a = u[e], b = v[e], c = w[e];
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
    atomicMax((unsigned long long*)&out3[0], __double_as_longlong((double)mu));
    atomicMax((unsigned long long*)&out3[1], __double_as_longlong((double)mv));
    atomicMax((unsigned long long*)&out3[2], __double_as_longlong((double)mw));
  }
}
__global__ void k_max_vort(int64_t n, const real* __restrict__ p, const real* __restrict__ q,
                           const real* __restrict__ r, double* __restrict__ out) {
  real m = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    real a = p[e], b = q[e], c = r[e];
    m = fmax(m, a * a + b * b + c * c);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)out, __double_as_longlong((double)m));
}

// nb (1 or 2) diffz solves of one boundary kind (all with or all without
// boundary values) in one launch
int diffz_batch_impl(pmpic_ctx* ctx, int nb, const real* const* in, real* const* out, const real* const* bot,
                     const real* const* top, real* sub = nullptr) {
  TimerScope ts(ctx, T_DIFFZ);
  const Geom& g = ctx->g;
  DzBatch zb{};
  zb.sub = sub;
  for (int q = 0; q < nb; ++q) {
    zb.f[q] = in[q];
    zb.out[q] = out[q];
    zb.bot[q] = bot ? bot[q] : nullptr;
    zb.top[q] = top ? top[q] : nullptr;
  }
  const real* coef = tab_diffz(ctx, bot ? 1 : 0);
  k_diffz<<<dim3(nblk((int64_t)g.sx * g.sy, 128), nb), 128, 0, ctx->stream>>>(g, zb, coef, (real)f4div(1.f, 6.f)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int diffz_launch_impl(pmpic_ctx* ctx, const real* in, real* out, const real* bot, const real* top) {
  return diffz_batch_impl(ctx, 1, &in, &out, bot ? &bot : nullptr, top ? &top : nullptr);
}


int spec_diffx_impl(pmpic_ctx* ctx, const real* in, real* out) {
  k_diffx<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, tab_kx(ctx)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_diffy_impl(pmpic_ctx* ctx, const real* in, real* out) {
  k_diffy<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, tab_ky(ctx)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_filter_impl(pmpic_ctx* ctx, const real* in, real* out) {
  k_filter<<<nblk(ctx->g.nspec, 256), 256, 0, ctx->stream>>>(ctx->g, in, out, tab_filt(ctx)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_diffz_impl(pmpic_ctx* ctx, const real* in, real* out, const real* bot, const real* top) {
  return diffz_launch_impl(ctx, in, out, bot, top);
}
// laplinv of na (1..3) arrays in one launch, the Thomas factors from the tables
int spec_laplinv_batch(pmpic_ctx* ctx, int na, real* const* fs, const bool* df0) {
  TimerScope ts(ctx, T_LAPLINV);
  const Geom& g = ctx->g;
  LapBatch lb{};
  for (int q = 0; q < na; ++q) {
    lb.f[q] = fs[q];
    lb.df0[q] = df0[q] ? 1 : 0;
  }
  k_laplinv<<<dim3(nblk((int64_t)g.sx * g.sy, 128), na), 128, 0, ctx->stream>>>(g, lb, RP(ctx->lapcp), tab_k2(ctx)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}
int spec_laplinv_impl(pmpic_ctx* ctx, real* inout, bool df0) { return spec_laplinv_batch(ctx, 1, &inout, &df0); }

// vort2vel.F90:139-320 after the three par2grid calls (grids P, Q, R hold the
// gridded vorticity on entry; on exit they hold the corrected, filtered
// vorticity, U, V, W the velocity and u_s, v_s, w_s its filtered spectra).
int vort2vel_spectral_impl(pmpic_ctx* ctx) {
  const Geom& g = ctx->g;
  int rc;
  real *a = RP(ctx->sa), *b = RP(ctx->sb), *c = RP(ctx->sc), *d = RP(ctx->sd), *e = RP(ctx->se), *f = RP(ctx->sf);
  real* const* G = (real* const*)ctx->grid;
  zero_mode_prepare(ctx);
  const unsigned nb = nblk(g.nspec, 256);
  const int cols = g.sx * g.sy;
  if ((rc = fft_forward(ctx, G[PMPIC_GRID_P], a))) return rc;
  if ((rc = fft_forward(ctx, G[PMPIC_GRID_Q], b))) return rc;
  if ((rc = fft_forward(ctx, G[PMPIC_GRID_R], c))) return rc;
  const real hdzi = (real)(f4div(1.f, 2.f) / g.dz);
  k_div<<<nb, 256, 0, ctx->stream>>>(g, a, b, c, f, tab_kx(ctx), tab_ky(ctx), hdzi); ++ctx->nlaunch;
  if ((rc = spec_laplinv_impl(ctx, f, true))) return rc;
  // :179-205: the filtered f (into e), a and b corrected, then c = c - diffz(filtered f)
  k_filter_sub2<<<nb, 256, 0, ctx->stream>>>(g, f, e, a, b, tab_kx(ctx), tab_ky(ctx), tab_filt(ctx)); ++ctx->nlaunch;
  {
    const real* zin[1] = {e};
    real* zout[1] = {d};
    if ((rc = diffz_batch_impl(ctx, 1, zin, zout, nullptr, nullptr, c))) return rc;
  }
  // :207-226: the top and bottom planes of a and b, then the filtered a, b, c
  // transformed back (the filter applied as the transform reads them)
  k_bt_planes<<<nblk(cols, 256), 256, 0, ctx->stream>>>(g, a, b, RP(ctx->bt)); ++ctx->nlaunch;
  SpecIn<real> F;
  F.op = SPEC_FILT;
  F.tab = tab_filt(ctx);
  const PhysOut<real> plain;
  if ((rc = fft_backward(ctx, a, G[PMPIC_GRID_P], F, plain))) return rc;
  if ((rc = fft_backward(ctx, b, G[PMPIC_GRID_Q], F, plain))) return rc;
  if ((rc = fft_backward(ctx, c, G[PMPIC_GRID_R], F, plain))) return rc;
  if ((rc = zero_mode_launch(ctx, a, b))) return rc;
  {
    real* abc[3] = {a, b, c};
    const bool df[3] = {false, false, true};
    if ((rc = spec_laplinv_batch(ctx, 3, abc, df))) return rc;
  }
  const real* atop = RP(ctx->bt);
  const real* abot = RP(ctx->bt) + cols;
  const real* btop = RP(ctx->bt) + 2 * cols;
  const real* bbot = RP(ctx->bt) + 3 * cols;
  // each velocity spectrum is formed as its inverse transform reads it, which
  // also stores the filtered copy (u_s, v_s, w_s)
  SpecIn<real> V;
  V.op = SPEC_VEL;
  V.e = e;
  V.c = c;
  V.a = a;
  V.b = b;
  V.kx = tab_kx(ctx);
  V.ky = tab_ky(ctx);
  V.filt = tab_filt(ctx);
  // dB/dz into e and dA/dz into d (:255, :284), in one launch
  {
    const real* zin[2] = {b, a};
    real* zout[2] = {e, d};
    const real* zbot[2] = {bbot, abot};
    const real* ztop[2] = {btop, atop};
    if ((rc = diffz_batch_impl(ctx, 2, zin, zout, zbot, ztop))) return rc;
  }
  // u = dB/dz - dC/dy (:251-276)
  V.vmode = 0;
  V.fs = RP(ctx->spec[PMPIC_SPEC_U]);
  V.zbar = ctx->zmode;
  if ((rc = fft_backward(ctx, nullptr, G[PMPIC_GRID_U], V, plain))) return rc;
  // v = dC/dx - dA/dz (:280-302)
  V.e = d;
  V.vmode = 1;
  V.fs = RP(ctx->spec[PMPIC_SPEC_V]);
  V.zbar = ctx->zmode + g.nzp;
  if ((rc = fft_backward(ctx, nullptr, G[PMPIC_GRID_V], V, plain))) return rc;
  // w = dA/dy - dB/dx (:306-320)
  V.vmode = 2;
  V.fs = RP(ctx->spec[PMPIC_SPEC_W]);
  V.zbar = nullptr;
  if ((rc = fft_backward(ctx, nullptr, G[PMPIC_GRID_W], V, plain))) return rc;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// vorticity_tendency.F90:147-265 (grid B holds par2grid(btot) on entry).
// Each spectral derivative is applied as its inverse transform reads it, and
// each pointwise update of dp, dq, dr as the transform writes its result, so
// no derivative spectrum or intermediate grid makes a round trip through HBM.
int vorticity_tendency_grids_impl(pmpic_ctx* ctx) {
  int rc;
  real *bs = RP(ctx->sbs);
  real* const* G = (real* const*)ctx->grid;
  real *DP = G[PMPIC_GRID_DP], *DQ = G[PMPIC_GRID_DQ], *DR = G[PMPIC_GRID_DR];
  const real *P = G[PMPIC_GRID_P], *Q = G[PMPIC_GRID_Q], *R = G[PMPIC_GRID_R];
  real *dudx = RP(ctx->gwork[0]), *dwdx = RP(ctx->gwork[1]), *dvdy = RP(ctx->gwork[2]);
  const real *us = RP(ctx->spec[PMPIC_SPEC_U]), *vs = RP(ctx->spec[PMPIC_SPEC_V]), *ws = RP(ctx->spec[PMPIC_SPEC_W]);
  SpecIn<real> DX, DY;
  DX.op = SPEC_DX;
  DX.tab = tab_kx(ctx);
  DY.op = SPEC_DY;
  DY.tab = tab_ky(ctx);
  auto epi = [](int op, int store, real* o, const real* a, const real* b) {
    PhysOut<real> E;
    E.op = op;
    E.store = store;
    E.o = o;
    E.in[0] = a;
    E.in[1] = b;
    return E;
  };
  const PhysOut<real> plain;
  if ((rc = fft_forward(ctx, G[PMPIC_GRID_B], bs))) return rc;
  // dp = db/dy + p du/dx + q du/dy + r (q + dw/dx)
  if ((rc = fft_backward(ctx, bs, DP, DY, plain))) return rc;
  if ((rc = fft_backward(ctx, us, dudx, DX, epi(PHYS_ADD_MUL, 1, DP, P, nullptr)))) return rc;
  if ((rc = fft_backward(ctx, us, nullptr, DY, epi(PHYS_ADD_MUL, 0, DP, Q, nullptr)))) return rc;
  if ((rc = fft_backward(ctx, ws, dwdx, DX, epi(PHYS_ADD_MUL_SUM, 1, DP, R, Q)))) return rc;
  // dq = -db/dx + p dv/dx + q dv/dy + r (-p + dw/dy)
  if ((rc = fft_backward(ctx, bs, DQ, DX, plain))) return rc;
  if ((rc = fft_backward(ctx, vs, nullptr, DX, epi(PHYS_NEG_ADD_MUL, 0, DQ, P, nullptr)))) return rc;
  if ((rc = fft_backward(ctx, vs, dvdy, DY, epi(PHYS_ADD_MUL, 1, DQ, Q, nullptr)))) return rc;
  // ... and, with dw/dy, dr = p dw/dx + q dw/dy - r du/dx - r dv/dy
  PhysOut<real> last = epi(PHYS_DQ_DR, 0, DQ, R, P);
  last.o2 = DR;
  last.in[2] = Q;
  last.in[3] = dwdx;
  last.in[4] = dudx;
  last.in[5] = dvdy;
  if ((rc = fft_backward(ctx, ws, nullptr, DY, last))) return rc;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// maxima for the dt rule; v2v: velocity limit, vt: vorticity limit
int field_max_impl(pmpic_ctx* ctx, bool v2v, bool vt) {
  real* const* G = (real* const*)ctx->grid;
  const Geom& g = ctx->g;
  if (v2v) {
    PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->umax2, 0, 3 * sizeof(double), ctx->stream));
    k_max_sq3<<<592, 256, 0, ctx->stream>>>(g.nphys, G[PMPIC_GRID_U], G[PMPIC_GRID_V],
                                            G[PMPIC_GRID_W], &ctx->dinfo->umax2); ++ctx->nlaunch;
  }
  if (vt) {
    PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->omax2, 0, sizeof(double), ctx->stream));
    k_max_vort<<<592, 256, 0, ctx->stream>>>(g.nphys, G[PMPIC_GRID_P], G[PMPIC_GRID_Q],
                                             G[PMPIC_GRID_R], &ctx->dinfo->omax2); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

