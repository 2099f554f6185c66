// pmpic_oracle.cpp -- TEST INFRASTRUCTURE: CPU restatement of the PMPIC hot path.
//
// This file is the parity oracle and the timed CPU baseline.  It is never part
// of the product path.  It follows the reference Fortran (EPCCed/pmpic) line by
// line for one MPI rank (so every halo exchange and parcel message is a
// self-message), in FP64, without FMA contraction (built -ffp-contract=off, the
// same arithmetic the reference gets from gfortran -O3 on x86-64), keeping the
// reference's serial loop orders wherever an integer outcome depends on them.
//
// Fortran arrays are restated 1-based and column-major: grid(k,j,i) has z
// fastest, exactly like model_core/src/grid/grids.F90 (Z=1, Y=2, X=3).
#include "pmpic_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// Single-precision Fortran literals promoted to double (e.g. `1./6.` in
// fft_ops.F90:427 is a REAL(4) constant assigned to a REAL(8) parameter).
inline double f4(float v) { return (double)v; }

// ---------------------------------------------------------------------------
// 1-based column-major 3-D array (Fortran restatement helper)
// ---------------------------------------------------------------------------
struct Grid3 {
  int n1 = 0, n2 = 0, n3 = 0;  // (k, j, i) extents
  std::vector<double> d;
  void alloc(int a, int b, int c) {
    n1 = a; n2 = b; n3 = c;
    d.assign((size_t)a * b * c, 0.0);
  }
  inline double& operator()(int k, int j, int i) {
    return d[(size_t)(k - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(i - 1))];
  }
  inline double operator()(int k, int j, int i) const {
    return d[(size_t)(k - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(i - 1))];
  }
};

// ---------------------------------------------------------------------------
// Complex FFT with FFTE's conventions (model_core/src/fft/ffte/vzfft1d.f:17-71):
// forward (IOPT=-1) unscaled, exp(-2 pi i jk/N); inverse (IOPT=+1) computed as
// conj -> forward -> conj * (1/N).  Radices 4, 2, 3, 5 (FFTE supports 2^a 3^b 5^c).
// A Stockham autosort formulation; twiddles are computed in long double.
// ---------------------------------------------------------------------------
struct FFTPlan {
  int n = 0;
  std::vector<int> radix;
  std::vector<std::vector<cplx>> tw;  // per stage: w^(p*t), p < m, t < R
};

bool factor235(int n, std::vector<int>& out) {
  out.clear();
  int m = n;
  while (m % 4 == 0) { out.push_back(4); m /= 4; }
  while (m % 2 == 0) { out.push_back(2); m /= 2; }
  while (m % 3 == 0) { out.push_back(3); m /= 3; }
  while (m % 5 == 0) { out.push_back(5); m /= 5; }
  return m == 1;
}

void make_plan(FFTPlan& pl, int n) {
  pl.n = n;
  factor235(n, pl.radix);
  pl.tw.clear();
  int len = n;
  for (int R : pl.radix) {
    int m = len / R;
    std::vector<cplx> t((size_t)m * R);
    for (int p = 0; p < m; ++p)
      for (int r = 0; r < R; ++r) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)((long long)p * r) /
                          (long double)len;
        t[(size_t)p * R + r] = cplx((double)cosl(ang), (double)sinl(ang));
      }
    pl.tw.push_back(t);
    len = m;
  }
}

// DFT of size R (R in {2,3,4,5}) on a[0..R-1] -> b[0..R-1], forward sign.
inline void small_dft(int R, const cplx* a, cplx* b) {
  if (R == 2) {
    b[0] = a[0] + a[1];
    b[1] = a[0] - a[1];
  } else if (R == 4) {
    cplx t0 = a[0] + a[2], t1 = a[0] - a[2];
    cplx t2 = a[1] + a[3], t3 = a[1] - a[3];
    cplx mi_t3(t3.imag(), -t3.real());  // -i * t3
    b[0] = t0 + t2;
    b[2] = t0 - t2;
    b[1] = t1 + mi_t3;
    b[3] = t1 - mi_t3;
  } else {
    static const long double PI_L = 3.14159265358979323846264338327950288L;
    for (int t = 0; t < R; ++t) {
      cplx s(0.0, 0.0);
      for (int r = 0; r < R; ++r) {
        long double ang = -2.0L * PI_L * (long double)((r * t) % R) / (long double)R;
        s += a[r] * cplx((double)cosl(ang), (double)sinl(ang));
      }
      b[t] = s;
    }
  }
}

// Forward transform in place (x), using y as workspace.
void fft_forward(const FFTPlan& pl, cplx* x, cplx* y) {
  int n = pl.n, s = 1, len = n;
  cplx* src = x;
  cplx* dst = y;
  cplx a[5], b[5];
  for (size_t st = 0; st < pl.radix.size(); ++st) {
    int R = pl.radix[st];
    int m = len / R;
    const std::vector<cplx>& tw = pl.tw[st];
    for (int p = 0; p < m; ++p) {
      for (int q = 0; q < s; ++q) {
        for (int r = 0; r < R; ++r) a[r] = src[q + (size_t)s * (p + r * m)];
        small_dft(R, a, b);
        for (int t = 0; t < R; ++t) dst[q + (size_t)s * (R * p + t)] = b[t] * tw[(size_t)p * R + t];
      }
    }
    std::swap(src, dst);
    s *= R;
    len = m;
  }
  if (src != x) std::memcpy(x, src, sizeof(cplx) * n);
}

// ZFFT1D(A,N,+1,B): conj, forward, conj, scale by DN=1/N (vzfft1d.f:41-46, 63-68)
void fft_inverse(const FFTPlan& pl, cplx* x, cplx* y) {
  int n = pl.n;
  for (int i = 0; i < n; ++i) x[i] = std::conj(x[i]);
  fft_forward(pl, x, y);
  double dn = 1.0 / (double)n;
  for (int i = 0; i < n; ++i) x[i] = std::conj(x[i]) * dn;
}

// ffte_r2c (ffte_mod.F90:66-89): complex forward FFT of (in, 0), keep n/2+1 terms.
void ffte_r2c(const FFTPlan& pl, const double* in, cplx* out, cplx* w1, cplx* w2) {
  int n = pl.n;
  for (int i = 0; i < n; ++i) w1[i] = cplx(in[i], 0.0);
  fft_forward(pl, w1, w2);
  for (int i = 0; i < n / 2 + 1; ++i) out[i] = w1[i];
}

// ffte_c2r (ffte_mod.F90:97-124): conjugate-symmetric fill, inverse FFT, real part.
void ffte_c2r(const FFTPlan& pl, const cplx* in, double* out, cplx* w1, cplx* w2) {
  int n = pl.n;
  for (int i = 0; i < n / 2 + 1; ++i) w1[i] = in[i];
  for (int i = n / 2 + 2; i <= n; ++i) w1[i - 1] = std::conj(in[n - i + 2 - 1]);
  fft_inverse(pl, w1, w2);
  for (int i = 0; i < n; ++i) out[i] = w1[i].real();
}

}  // namespace

// ---------------------------------------------------------------------------
// Context: the parts of model_state_type and of the module-level `save` state
// of the hot-path modules that a single rank needs.
// ---------------------------------------------------------------------------
struct orc_ctx {
  // global grid (setup_grid.F90:45-104)
  int Nx, Ny, Nz;          // cell counts; Nz+1 z points (setup_grid.F90:51)
  int nzp;                 // Nz+1
  double bottom[3], top[3], res[3];  // index 0=x, 1=y, 2=z
  double dx, dy, dz;
  // parcel_interpolation module state (parcel_interpolation.F90:29-41, 51-157)
  int nx, ny, nz;          // local extents incl. halo: Nx+4, Ny+4, Nz+1
  int hx, hy;              // halo depth 2 in x,y, 0 in z (decomposition.F90:449-451)
  double pxmin, pymin, pzmin, pxmax, pymax, pzmax;
  std::vector<double> x_coords, y_coords, z_coords;  // 1-based
  std::vector<int> is, js, ks;
  std::vector<double> delxs, delys, delzs;
  int64_t nparcels_cached = 0;
  // parcels (parcels.F90:9-38)
  int64_t maxparcels, numparcels;
  std::vector<double> prop[ORC_NPROP];
  // grids (setup_grid.F90:116-144, vorticity_tendency.F90:90-91)
  Grid3 g[ORC_NGRID];
  Grid3 gdudx, gdwdx, gdvdy, gdwdy, gap;  // vorticity_tendency work grids
  // spectral arrays (vort2vel.F90:75-84; vorticity_tendency.F90:76-77)
  Grid3 s[ORC_NSPEC];
  Grid3 sa, sb, sc, sd, se, sf, sas, sbs;
  // fft_ops wavenumbers (fft_ops.F90:111-140), per (j,i) (constant along z)
  std::vector<double> kx, ky, k2, filt;
  FFTPlan plan_x, plan_y;
  // mixing work (parcel_mixing.F90:29-31, 51-52)
  std::vector<int> npercell;   // (nz-1, ny-1, nx-1)
  Grid3 vres, bres, hres, pres, qres, rres;
  std::vector<int> keep;
  // parcel haloswap index (haloswap.F90:21)
  std::vector<int> hindex;
  // time stepping
  double dtm, dtmax, prefactor;
  int rkstep = 1, it_v2v = 0, it_vt = 0, it_split = 0, it_mix = 0;
  int rksteps = 4;
  orc_step_info info;
  int err = 0;
  std::string errmsg;
};

static int fail(orc_ctx* c, int code, const char* msg) {
  if (c->err == 0) {
    c->err = code;
    c->errmsg = msg;
  }
  return code;
}

static int g_threads = 0;

extern "C" void orc_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

// ---------------------------------------------------------------------------
// Creation: setup_grid.F90:45-104, parcel_interpolation.F90:51-157,
// fft_ops.F90:48-168, parcel_mixing.F90:46-64.
// ---------------------------------------------------------------------------
extern "C" orc_ctx* orc_create(int Nx, int Ny, int Nz, double xmin, double xmax, double ymin,
                               double ymax, double zmin, double zmax, double dtm, double dtmax,
                               double prefactor, int64_t maxp) {
  std::vector<int> f;
  if (Nx < 4 || Ny < 4 || Nz < 3 || !factor235(Nx, f) || !factor235(Ny, f)) return nullptr;
  // Only origins at zero are supported: parcel_interpolation.F90:104-106 and
  // :126-136 add global_grid%bottom twice, which is inconsistent for non-zero
  // origins; configs are run in the shifted box [0,Lx]x[0,Ly]x[0,Lz].
  if (xmin != 0.0 || ymin != 0.0 || zmin != 0.0) return nullptr;
  orc_ctx* c = new orc_ctx();
  c->Nx = Nx; c->Ny = Ny; c->Nz = Nz; c->nzp = Nz + 1;
  // setup_grid.F90:73-95
  c->dx = (xmax - xmin) / (double)Nx;
  c->dy = (ymax - ymin) / (double)Ny;
  c->dz = (zmax - zmin) / (double)(c->nzp - 1);
  c->res[0] = c->dx; c->res[1] = c->dy; c->res[2] = c->dz;
  c->bottom[0] = xmin; c->bottom[1] = ymin; c->bottom[2] = zmin;
  c->top[0] = xmax - c->dx; c->top[1] = ymax - c->dy; c->top[2] = zmax;
  // parcel_interpolation.F90:76-136 for one rank (start=1, end=N, halo 2/2/0)
  c->hx = 2; c->hy = 2;
  c->nx = Nx + 2 * c->hx;
  c->ny = Ny + 2 * c->hy;
  c->nz = c->nzp;
  int xstart = 1 - c->hx, xstop = Nx + c->hx;
  int ystart = 1 - c->hy, ystop = Ny + c->hy;
  int zstart = 1, zstop = c->nzp;
  c->pxmin = (double)(xstart - 1) * c->dx + c->bottom[0];
  c->pymin = (double)(ystart - 1) * c->dy + c->bottom[1];
  c->pzmin = (double)(zstart - 1) * c->dz + c->bottom[2];
  c->pxmax = (double)(xstop - 1) * c->dx;
  c->pymax = (double)(ystop - 1) * c->dy;
  c->pzmax = (double)(zstop - 1) * c->dz;
  c->x_coords.resize(c->nx + 1);
  c->y_coords.resize(c->ny + 1);
  c->z_coords.resize(c->nz + 1);
  for (int n = 1; n <= c->nx; ++n) c->x_coords[n] = c->pxmin + (double)(n - 1) * c->dx + c->bottom[0];
  for (int n = 1; n <= c->ny; ++n) c->y_coords[n] = c->pymin + (double)(n - 1) * c->dy + c->bottom[1];
  for (int n = 1; n <= c->nz; ++n) c->z_coords[n] = c->pzmin + (double)(n - 1) * c->dz + c->bottom[2];
  c->maxparcels = maxp;
  c->numparcels = 0;
  for (int p = 0; p < ORC_NPROP; ++p) c->prop[p].assign((size_t)maxp, 0.0);
  c->is.assign(maxp, 0); c->js.assign(maxp, 0); c->ks.assign(maxp, 0);
  c->delxs.assign(maxp, 0.0); c->delys.assign(maxp, 0.0); c->delzs.assign(maxp, 0.0);
  c->hindex.assign(maxp, 0);
  for (int gi = 0; gi < ORC_NGRID; ++gi) c->g[gi].alloc(c->nz, c->ny, c->nx);
  c->gdudx.alloc(c->nz, c->ny, c->nx); c->gdwdx.alloc(c->nz, c->ny, c->nx);
  c->gdvdy.alloc(c->nz, c->ny, c->nx); c->gdwdy.alloc(c->nz, c->ny, c->nx);
  c->gap.alloc(c->nz, c->ny, c->nx);
  int sy = Ny + 2, sx = Nx + 2;  // (n/2+1)*2 (pencilfft.F90:780)
  for (int si = 0; si < ORC_NSPEC; ++si) c->s[si].alloc(c->nzp, sy, sx);
  Grid3* w[] = {&c->sa, &c->sb, &c->sc, &c->sd, &c->se, &c->sf, &c->sas, &c->sbs};
  for (Grid3* g : w) g->alloc(c->nzp, sy, sx);
  // fft_ops.F90:111-140 (x_start = y_start = 1 on one rank)
  double lx = c->res[0] * (double)Nx;
  double ly = c->res[1] * (double)Ny;
  // `size/2.` is a REAL(4) quotient (integer / REAL(4) literal)
  const double kxm = (double)((float)Nx / 2.0f) / lx, kym = (double)((float)Ny / 2.0f) / ly;
  double ksqmax = kxm * kxm + kym * kym;
  ksqmax = ksqmax * 2.0 / 9.0;
  const double twopi = 8.0 * std::atan(1.0);
  c->kx.resize((size_t)sy * sx); c->ky.resize((size_t)sy * sx);
  c->k2.resize((size_t)sy * sx); c->filt.resize((size_t)sy * sx);
  for (int i = 1; i <= sx; ++i) {
    double xval = (double)((1 + i - 2) / 2) / lx;
    for (int j = 1; j <= sy; ++j) {
      double yval = (double)((1 + j - 2) / 2) / ly;
      size_t o = (size_t)(j - 1) + (size_t)sy * (i - 1);
      double kk = xval * xval + yval * yval;
      c->filt[o] = (kk > ksqmax) ? 0.0 : 1.0;
      c->kx[o] = xval * twopi;
      c->ky[o] = yval * twopi;
      c->k2[o] = kk * twopi * twopi;
    }
  }
  make_plan(c->plan_x, Nx);
  make_plan(c->plan_y, Ny);
  // parcel_mixing.F90:51-52
  c->npercell.assign((size_t)(c->nz - 1) * (c->ny - 1) * (c->nx - 1), 0);
  Grid3* r[] = {&c->vres, &c->bres, &c->hres, &c->pres, &c->qres, &c->rres};
  for (Grid3* g : r) g->alloc(c->nz, c->ny, c->nx);
  // rk4_integrator.F90:38-41
  c->dtm = dtm;
  c->dtmax = dtmax;
  c->prefactor = prefactor;
  std::memset(&c->info, 0, sizeof(c->info));
  c->info.dtm = dtm;
  return c;
}

extern "C" void orc_destroy(orc_ctx* c) { delete c; }

extern "C" int orc_error(const orc_ctx* c, char* msg, int len) {
  if (msg && len > 0) {
    std::snprintf(msg, (size_t)len, "%s", c->errmsg.c_str());
  }
  return c->err;
}

extern "C" int orc_set_count(orc_ctx* c, int64_t n) {
  if (n < 0 || n > c->maxparcels) return fail(c, -1, "parcel count exceeds max_parcels");
  c->numparcels = n;
  c->info.n_parcels = n;
  return 0;
}
extern "C" int64_t orc_count(const orc_ctx* c) { return c->numparcels; }

extern "C" int orc_set_prop(orc_ctx* c, int p, const double* src, int64_t n) {
  if (p < 0 || p >= ORC_NPROP || n > c->maxparcels) return -1;
  std::memcpy(c->prop[p].data(), src, sizeof(double) * (size_t)n);
  return 0;
}
extern "C" int orc_get_prop(const orc_ctx* c, int p, double* dst, int64_t n) {
  if (p < 0 || p >= ORC_NPROP || n > c->maxparcels) return -1;
  std::memcpy(dst, c->prop[p].data(), sizeof(double) * (size_t)n);
  return 0;
}

// interior of a halo grid <-> dense (Nz+1) x Ny x Nx, x fastest
static void grid_to_dense(const orc_ctx* c, const Grid3& g, double* dst) {
  for (int k = 1; k <= c->nzp; ++k)
    for (int j = 1; j <= c->Ny; ++j)
      for (int i = 1; i <= c->Nx; ++i)
        dst[(size_t)(i - 1) + (size_t)c->Nx * ((j - 1) + (size_t)c->Ny * (k - 1))] = g(k, j + c->hy, i + c->hx);
}
static void dense_to_grid(const orc_ctx* c, const double* src, Grid3& g) {
  for (int k = 1; k <= c->nzp; ++k)
    for (int j = 1; j <= c->Ny; ++j)
      for (int i = 1; i <= c->Nx; ++i)
        g(k, j + c->hy, i + c->hx) = src[(size_t)(i - 1) + (size_t)c->Nx * ((j - 1) + (size_t)c->Ny * (k - 1))];
}
static void spec_to_dense(const Grid3& s, double* dst) {
  for (int k = 1; k <= s.n1; ++k)
    for (int j = 1; j <= s.n2; ++j)
      for (int i = 1; i <= s.n3; ++i)
        dst[(size_t)(i - 1) + (size_t)s.n3 * ((j - 1) + (size_t)s.n2 * (k - 1))] = s(k, j, i);
}
static void dense_to_spec(const double* src, Grid3& s) {
  for (int k = 1; k <= s.n1; ++k)
    for (int j = 1; j <= s.n2; ++j)
      for (int i = 1; i <= s.n3; ++i)
        s(k, j, i) = src[(size_t)(i - 1) + (size_t)s.n3 * ((j - 1) + (size_t)s.n2 * (k - 1))];
}

extern "C" int orc_get_grid(const orc_ctx* c, int gi, double* dst) {
  if (gi < 0 || gi >= ORC_NGRID) return -1;
  grid_to_dense(c, c->g[gi], dst);
  return 0;
}
extern "C" int orc_set_grid(orc_ctx* c, int gi, const double* src) {
  if (gi < 0 || gi >= ORC_NGRID) return -1;
  dense_to_grid(c, src, c->g[gi]);
  return 0;
}
extern "C" int orc_get_spec(const orc_ctx* c, int si, double* dst) {
  if (si < 0 || si >= ORC_NSPEC) return -1;
  spec_to_dense(c->s[si], dst);
  return 0;
}
extern "C" void orc_get_step_info(const orc_ctx* c, orc_step_info* out) {
  *out = c->info;
  out->n_parcels = c->numparcels;
  out->error = c->err;
  std::snprintf(out->message, sizeof(out->message), "%s", c->errmsg.c_str());
}
extern "C" void orc_get_counters(const orc_ctx* c, int* v) {
  v[0] = c->it_v2v; v[1] = c->it_vt; v[2] = c->rkstep; v[3] = c->it_split; v[4] = c->it_mix;
}
extern "C" void orc_set_counters(orc_ctx* c, const int* v) {
  c->it_v2v = v[0]; c->it_vt = v[1]; c->rkstep = v[2]; c->it_split = v[3]; c->it_mix = v[4];
}
extern "C" void orc_set_dtm(orc_ctx* c, double d) { c->dtm = d; c->info.dtm = d; }

// ---------------------------------------------------------------------------
// MPIC_Haloswap.F90 for one rank.  xi = hx+1, xf = Nx+hx (local interior).
// ---------------------------------------------------------------------------
// grid2par_haloswap (MPIC_Haloswap.F90:95-184): copy first interior column/row/
// corner column into the +x / +y halo and the +x+y corner.
static void grid2par_haloswap(orc_ctx* c, Grid3& a) {
  const int xi = c->hx + 1, xf = c->Nx + c->hx, yi = c->hy + 1, yf = c->Ny + c->hy;
  // buffers are packed before any unpacking (:104-106)
  std::vector<double> left((size_t)c->nz * c->Ny), down((size_t)c->nz * c->Nx), corner(c->nz);
  for (int j = yi; j <= yf; ++j)
    for (int k = 1; k <= c->nz; ++k) left[(size_t)(k - 1) + (size_t)c->nz * (j - yi)] = a(k, j, xi);
  for (int i = xi; i <= xf; ++i)
    for (int k = 1; k <= c->nz; ++k) down[(size_t)(k - 1) + (size_t)c->nz * (i - xi)] = a(k, yi, i);
  for (int k = 1; k <= c->nz; ++k) corner[k - 1] = a(k, yi, xi);
  // receive order = send order xtag, ytag, cortag (MPI non-overtaking)
  for (int j = yi; j <= yf; ++j)
    for (int k = 1; k <= c->nz; ++k) a(k, j, xf + 1) = left[(size_t)(k - 1) + (size_t)c->nz * (j - yi)];
  for (int i = xi; i <= xf; ++i)
    for (int k = 1; k <= c->nz; ++k) a(k, yf + 1, i) = down[(size_t)(k - 1) + (size_t)c->nz * (i - xi)];
  for (int k = 1; k <= c->nz; ++k) a(k, yf + 1, xf + 1) = corner[k - 1];
}

// par2grid_haloswap (MPIC_Haloswap.F90:188-290): add the +x / +y halo and the
// +x+y corner back onto the first interior column / row / corner column.
static void par2grid_haloswap(orc_ctx* c, Grid3& a) {
  const int xi = c->hx + 1, xf = c->Nx + c->hx, yi = c->hy + 1, yf = c->Ny + c->hy;
  std::vector<double> right((size_t)c->nz * c->Ny), up((size_t)c->nz * c->Nx), corner(c->nz);
  for (int j = yi; j <= yf; ++j)
    for (int k = 1; k <= c->nz; ++k) right[(size_t)(k - 1) + (size_t)c->nz * (j - yi)] = a(k, j, xf + 1);
  for (int i = xi; i <= xf; ++i)
    for (int k = 1; k <= c->nz; ++k) up[(size_t)(k - 1) + (size_t)c->nz * (i - xi)] = a(k, yf + 1, i);
  for (int k = 1; k <= c->nz; ++k) corner[k - 1] = a(k, yf + 1, xf + 1);
  for (int j = yi; j <= yf; ++j)
    for (int k = 1; k <= c->nz; ++k) a(k, j, xi) = a(k, j, xi) + right[(size_t)(k - 1) + (size_t)c->nz * (j - yi)];
  for (int i = xi; i <= xf; ++i)
    for (int k = 1; k <= c->nz; ++k) a(k, yi, i) = a(k, yi, i) + up[(size_t)(k - 1) + (size_t)c->nz * (i - xi)];
  for (int k = 1; k <= c->nz; ++k) a(k, yi, xi) = a(k, yi, xi) + corner[k - 1];
}

// mixing_haloswap (MPIC_Haloswap.F90:294-307)
static void mixing_haloswap(orc_ctx* c, Grid3& a) {
  par2grid_haloswap(c, a);
  grid2par_haloswap(c, a);
}

// ---------------------------------------------------------------------------
// parcel_interpolation.F90
// ---------------------------------------------------------------------------
// cache_parcel_interp_weights (parcel_interpolation.F90:186-262)
static int cache_weights(orc_ctx* c) {
  const int64_t np = c->numparcels;
  c->nparcels_cached = np;
  const double* X = c->prop[ORC_X].data();
  const double* Y = c->prop[ORC_Y].data();
  const double* Z = c->prop[ORC_Z].data();
  int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (int64_t n = 0; n < np; ++n) {
    double xp = X[n], yp = Y[n], zp = Z[n];
    double fi = std::floor((xp - c->pxmin) / c->dx);
    double fj = std::floor((yp - c->pymin) / c->dy);
    double fk = std::floor((zp - c->pzmin) / c->dz);
    // (:222-227) out-of-box aborts; the NaN test also rejects non-finite positions
    if (!(fi >= 0.0 && fi + 1 < (double)c->nx) || !(fj >= 0.0 && fj + 1 < (double)c->ny) ||
        !(fk >= 0.0 && fk + 1 < (double)c->nz)) {
      bad |= 1;
      continue;
    }
    int i = (int)fi + 1, j = (int)fj + 1, k = (int)fk + 1;
    double delx = ((xp - c->pxmin) - (double)(i - 1) * c->dx) / c->dx;
    double dely = ((yp - c->pymin) - (double)(j - 1) * c->dy) / c->dy;
    double delz = ((zp - c->pzmin) - (double)(k - 1) * c->dz) / c->dz;
    // (:235-237)
    if (delx > 1.0 || delx < 0.0 || dely > 1.0 || dely < 0.0 || delz > 1.0 || delz < 0.0) {
      bad |= 2;
      continue;
    }
    c->is[n] = i; c->js[n] = j; c->ks[n] = k;
    c->delxs[n] = delx; c->delys[n] = dely; c->delzs[n] = delz;
  }
  if (bad & 1) return fail(c, -3, "parcel out of box");
  if (bad & 2) return fail(c, -3, "delx/dely/delz wrong size");
  return 0;
}

extern "C" int orc_cache_weights(orc_ctx* c, int32_t* cells) {
  int rc = cache_weights(c);
  if (rc) return rc;
  if (cells) {
    // cell id in the interior numbering used by the GPU library:
    // ((k-1)*Ny + (j-3))*Nx + (i-3), with the halo cell i = Nx+3 (j = Ny+3)
    // identified with its periodic image, interior cell i = 3 (j = 3)
    for (int64_t n = 0; n < c->numparcels; ++n) {
      int ii = (c->is[n] - 1 - c->hx) % c->Nx, jj = (c->js[n] - 1 - c->hy) % c->Ny;
      cells[n] = (int32_t)(((int64_t)(c->ks[n] - 1) * c->Ny + jj) * c->Nx + ii);
    }
  }
  return 0;
}

// grid2par (parcel_interpolation.F90:267-332)
static void grid2par(orc_ctx* c, Grid3& grid, double* var) {
  grid2par_haloswap(c, grid);
  const int64_t np = c->nparcels_cached;
#pragma omp parallel for schedule(static)
  for (int64_t n = 0; n < np; ++n) {
    double delx = c->delxs[n], dely = c->delys[n], delz = c->delzs[n];
    int i = c->is[n], j = c->js[n], k = c->ks[n];
    double c000 = grid(k, j, i);
    double c001 = grid(k, j, i + 1);
    double c010 = grid(k, j + 1, i);
    double c011 = grid(k, j + 1, i + 1);
    double c100 = grid(k + 1, j, i);
    double c101 = grid(k + 1, j, i + 1);
    double c110 = grid(k + 1, j + 1, i);
    double c111 = grid(k + 1, j + 1, i + 1);
    double c00 = c000 * (1 - delz) + c100 * delz;
    double c01 = c001 * (1 - delz) + c101 * delz;
    double c10 = c010 * (1 - delz) + c110 * delz;
    double c11 = c011 * (1 - delz) + c111 * delz;
    double c0 = c00 * (1 - dely) + c10 * dely;
    double c1 = c01 * (1 - dely) + c11 * dely;
    var[n] = c0 * (1 - delx) + c1 * delx;
  }
}

// par2grid (parcel_interpolation.F90:336-481).  The reference's OpenMP array
// reduction (:371) makes the sum order thread-count dependent; here each thread
// accumulates a private copy in parcel order and the copies are added in
// thread order.  With one thread the order is the reference's serial order.
static void par2grid(orc_ctx* c, const double* var, Grid3& grid) {
  const size_t N = (size_t)c->nz * c->ny * c->nx;
  std::vector<double> weights(N, 0.0), data(N, 0.0);
  const int64_t np = c->nparcels_cached;
  const double* VOL = c->prop[ORC_VOL].data();
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
  if (np < 100000) nt = 1;
#endif
  auto scatter = [&](int64_t n0, int64_t n1, double* W, double* D) {
    const int n1s = c->nz, n2s = c->ny;
    auto at = [&](int k, int j, int i) -> size_t {
      return (size_t)(k - 1) + (size_t)n1s * ((size_t)(j - 1) + (size_t)n2s * (size_t)(i - 1));
    };
    for (int64_t n = n0; n < n1; ++n) {
      double delx = c->delxs[n], dely = c->delys[n], delz = c->delzs[n];
      int i = c->is[n], j = c->js[n], k = c->ks[n];
      double v = VOL[n];
      double w = var[n];
      double w000 = (1 - delz) * (1 - dely) * (1 - delx) * v;
      D[at(k, j, i)] = D[at(k, j, i)] + w000 * w;
      W[at(k, j, i)] = W[at(k, j, i)] + w000;
      double w001 = (1 - delz) * (1 - dely) * (delx) * v;
      D[at(k, j, i + 1)] = D[at(k, j, i + 1)] + w001 * w;
      W[at(k, j, i + 1)] = W[at(k, j, i + 1)] + w001;
      double w010 = (1 - delz) * (dely) * (1 - delx) * v;
      D[at(k, j + 1, i)] = D[at(k, j + 1, i)] + w010 * w;
      W[at(k, j + 1, i)] = W[at(k, j + 1, i)] + w010;
      double w011 = (1 - delz) * (dely) * (delx) * v;
      D[at(k, j + 1, i + 1)] = D[at(k, j + 1, i + 1)] + w011 * w;
      W[at(k, j + 1, i + 1)] = W[at(k, j + 1, i + 1)] + w011;
      double w100 = (delz) * (1 - dely) * (1 - delx) * v;
      D[at(k + 1, j, i)] = D[at(k + 1, j, i)] + w100 * w;
      W[at(k + 1, j, i)] = W[at(k + 1, j, i)] + w100;
      double w101 = (delz) * (1 - dely) * (delx) * v;
      D[at(k + 1, j, i + 1)] = D[at(k + 1, j, i + 1)] + w101 * w;
      W[at(k + 1, j, i + 1)] = W[at(k + 1, j, i + 1)] + w101;
      double w110 = (delz) * (dely) * (1 - delx) * v;
      D[at(k + 1, j + 1, i)] = D[at(k + 1, j + 1, i)] + w110 * w;
      W[at(k + 1, j + 1, i)] = W[at(k + 1, j + 1, i)] + w110;
      double w111 = (delz) * (dely) * (delx) * v;
      D[at(k + 1, j + 1, i + 1)] = D[at(k + 1, j + 1, i + 1)] + w111 * w;
      W[at(k + 1, j + 1, i + 1)] = W[at(k + 1, j + 1, i + 1)] + w111;
    }
  };
  if (nt <= 1) {
    scatter(0, np, weights.data(), data.data());
  } else {
    std::vector<std::vector<double>> pw(nt), pd(nt);
#pragma omp parallel num_threads(nt)
    {
      int t = 0;
#ifdef _OPENMP
      t = omp_get_thread_num();
#endif
      pw[t].assign(N, 0.0);
      pd[t].assign(N, 0.0);
      int64_t n0 = np * t / nt, n1 = np * (t + 1) / nt;
      scatter(n0, n1, pw[t].data(), pd[t].data());
#pragma omp barrier
#pragma omp for schedule(static)
      for (int64_t e = 0; e < (int64_t)N; ++e) {
        double sw = 0.0, sd = 0.0;
        for (int q = 0; q < nt; ++q) { sw += pw[q][e]; sd += pd[q][e]; }
        weights[e] = sw;
        data[e] = sd;
      }
    }
  }
  Grid3 W, D;
  W.n1 = D.n1 = c->nz; W.n2 = D.n2 = c->ny; W.n3 = D.n3 = c->nx;
  W.d.swap(weights);
  D.d.swap(data);
  par2grid_haloswap(c, W);   // :451
  par2grid_haloswap(c, D);   // :452
  // :458-459 double the wall levels of grid%data, but :463-469 overwrite every
  // point of grid%data, so the doubling has no effect and is not restated.
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)N; ++e) {
    double wv = W.d[e];
    if (wv == 0.) wv = 1.;  // :466
    grid.d[e] = D.d[e] / wv;  // :467
  }
}

extern "C" int orc_par2grid(orc_ctx* c, int p, int gi) {
  if (p < 0 || p >= ORC_NPROP || gi < 0 || gi >= ORC_NGRID) return -1;
  par2grid(c, c->prop[p].data(), c->g[gi]);
  return 0;
}
extern "C" int orc_grid2par(orc_ctx* c, int gi, int p) {
  if (p < 0 || p >= ORC_NPROP || gi < 0 || gi >= ORC_NGRID) return -1;
  grid2par(c, c->g[gi], c->prop[p].data());
  return 0;
}

// ---------------------------------------------------------------------------
// Semi-spectral transforms: pencilfft.F90:151-212 on one rank.
// Forward: r2c along y of every (z, x) row (:329-342, ffte_r2c), complex ->
// interleaved reals along y (:838-864), r2c along x of every (z, y') real row
// (:372-385), interleave along x.  Result (z, Ny+2, Nx+2).
// Backward mirrors it: real -> complex along x (:872-899), c2r along x, real ->
// complex along y, c2r along y.
// ---------------------------------------------------------------------------
static void forward_3dfft(orc_ctx* c, const Grid3& src, int src_off_y, int src_off_x, Grid3& dst) {
  const int Nx = c->Nx, Ny = c->Ny, nz = c->nzp;
  const int sy = Ny + 2;
  Grid3 mid;  // (z, Ny+2, Nx)
  mid.alloc(nz, sy, Nx);
#pragma omp parallel
  {
    std::vector<double> row(std::max(Nx, Ny));
    std::vector<cplx> out(std::max(Nx, Ny) / 2 + 1), w1(std::max(Nx, Ny)), w2(std::max(Nx, Ny));
#pragma omp for collapse(2) schedule(static)
    for (int i = 1; i <= Nx; ++i)
      for (int k = 1; k <= nz; ++k) {
        for (int j = 1; j <= Ny; ++j) row[j - 1] = src(k, j + src_off_y, i + src_off_x);
        ffte_r2c(c->plan_y, row.data(), out.data(), w1.data(), w2.data());
        for (int a = 1; a <= Ny / 2 + 1; ++a) {
          mid(k, 2 * a - 1, i) = out[a - 1].real();
          mid(k, 2 * a, i) = out[a - 1].imag();
        }
      }
#pragma omp for collapse(2) schedule(static)
    for (int j = 1; j <= sy; ++j)
      for (int k = 1; k <= nz; ++k) {
        for (int i = 1; i <= Nx; ++i) row[i - 1] = mid(k, j, i);
        ffte_r2c(c->plan_x, row.data(), out.data(), w1.data(), w2.data());
        for (int b = 1; b <= Nx / 2 + 1; ++b) {
          dst(k, j, 2 * b - 1) = out[b - 1].real();
          dst(k, j, 2 * b) = out[b - 1].imag();
        }
      }
  }
}

static void backward_3dfft(orc_ctx* c, const Grid3& src, Grid3& dst, int dst_off_y, int dst_off_x) {
  const int Nx = c->Nx, Ny = c->Ny, nz = c->nzp;
  const int sy = Ny + 2;
  Grid3 mid;  // (z, Ny+2, Nx)
  mid.alloc(nz, sy, Nx);
#pragma omp parallel
  {
    std::vector<double> row(std::max(Nx, Ny));
    std::vector<cplx> in(std::max(Nx, Ny) / 2 + 1), w1(std::max(Nx, Ny)), w2(std::max(Nx, Ny));
#pragma omp for collapse(2) schedule(static)
    for (int j = 1; j <= sy; ++j)
      for (int k = 1; k <= nz; ++k) {
        for (int b = 1; b <= Nx / 2 + 1; ++b) in[b - 1] = cplx(src(k, j, 2 * b - 1), src(k, j, 2 * b));
        ffte_c2r(c->plan_x, in.data(), row.data(), w1.data(), w2.data());
        for (int i = 1; i <= Nx; ++i) mid(k, j, i) = row[i - 1];
      }
#pragma omp for collapse(2) schedule(static)
    for (int i = 1; i <= Nx; ++i)
      for (int k = 1; k <= nz; ++k) {
        for (int a = 1; a <= Ny / 2 + 1; ++a) in[a - 1] = cplx(mid(k, 2 * a - 1, i), mid(k, 2 * a, i));
        ffte_c2r(c->plan_y, in.data(), row.data(), w1.data(), w2.data());
        for (int j = 1; j <= Ny; ++j) dst(k, j + dst_off_y, i + dst_off_x) = row[j - 1];
      }
  }
}

// ---------------------------------------------------------------------------
// fft_ops.F90 on one rank (no Re/Im pair is split across ranks)
// ---------------------------------------------------------------------------
static inline size_t kidx(const orc_ctx* c, int j, int i) { return (size_t)(j - 1) + (size_t)(c->Ny + 2) * (i - 1); }

// spectral_filter (fft_ops.F90:176-197)
static void spectral_filter(orc_ctx* c, const Grid3& f, Grid3& out) {
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= f.n3; ++i)
    for (int j = 1; j <= f.n2; ++j) {
      double m = c->filt[kidx(c, j, i)];
      for (int k = 1; k <= f.n1; ++k) out(k, j, i) = f(k, j, i) * m;
    }
}

// diffx (fft_ops.F90:204-302): out(i) = -in(i+1), out(i+1) = in(i), then * kx
static void diffx(orc_ctx* c, const Grid3& in, Grid3& out) {
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= in.n3; i += 2)
    for (int j = 1; j <= in.n2; ++j)
      for (int k = 1; k <= in.n1; ++k) {
        double a = in(k, j, i), b = in(k, j, i + 1);
        out(k, j, i) = (-1. * b) * c->kx[kidx(c, j, i)];
        out(k, j, i + 1) = a * c->kx[kidx(c, j, i + 1)];
      }
}

// diffy (fft_ops.F90:305-401)
static void diffy(orc_ctx* c, const Grid3& in, Grid3& out) {
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= in.n3; ++i)
    for (int j = 1; j <= in.n2; j += 2)
      for (int k = 1; k <= in.n1; ++k) {
        double a = in(k, j, i), b = in(k, j + 1, i);
        out(k, j, i) = (-1. * b) * c->ky[kidx(c, j, i)];
        out(k, j + 1, i) = a * c->ky[kidx(c, j + 1, i)];
      }
}

// tridiagonal (fft_ops.F90:620-656).  Returns non-zero on a zero pivot (:642-645).
static int tridiagonal(int n, const double* a, const double* b, const double* cc, const double* d, double* f,
                       double* cp) {
  double denominator = b[0];
  f[0] = d[0] / denominator;
  for (int i = 2; i <= n; ++i) {
    cp[i - 1] = cc[i - 2] / denominator;
    denominator = b[i - 1] - a[i - 1] * cp[i - 1];
    if (denominator == 0) return 1;
    f[i - 1] = (d[i - 1] - a[i - 1] * f[i - 2]) / (denominator);
  }
  for (int i = n - 1; i >= 1; --i) f[i - 1] = f[i - 1] - cp[i] * f[i];
  return 0;
}

// diffz (fft_ops.F90:419-483).  Note the code (not the comment at :414-417)
// sets b(1)=b(n)=1 and c(1)=a(n)=1/3 when bot/top are given.
static int diffz(orc_ctx* c, const Grid3& f, Grid3& dfdz, const std::vector<double>* bot,
                 const std::vector<double>* top) {
  const int nz = f.n1, ny = f.n2, nx = f.n3;
  const double a0 = 0., b0 = 1., c0 = 0.;
  const double a1 = f4(1.f / 6.f), b1 = f4(2.f / 3.f), c1 = f4(1.f / 6.f);
  const double an = 0., bn = 1., cn = 0.;
  const double al = f4(1.f / 3.f), cl = f4(1.f / 3.f);
  const double dz = c->dz;
  std::vector<double> A(nz), B(nz), C(nz);
  A[0] = a0; B[0] = b0; C[0] = c0;
  for (int k = 2; k <= nz - 1; ++k) { A[k - 1] = a1; B[k - 1] = b1; C[k - 1] = c1; }
  A[nz - 1] = an; B[nz - 1] = bn; C[nz - 1] = cn;
  const bool bt = bot && top;
  if (bt) { C[0] = cl; A[nz - 1] = al; }
  int bad = 0;
#pragma omp parallel reduction(| : bad)
  {
    std::vector<double> d(nz), out(nz), cp(nz + 1);
#pragma omp for collapse(2) schedule(static)
    for (int i = 1; i <= nx; ++i)
      for (int j = 1; j <= ny; ++j) {
        if (bt) {
          size_t o = (size_t)(j - 1) + (size_t)ny * (i - 1);
          d[0] = f(2, j, i) / dz - a1 * (*bot)[o] * dz;
          d[nz - 1] = -f(nz - 1, j, i) / dz + a1 * (*top)[o] * dz;
        } else {
          d[0] = 0.0;
          d[nz - 1] = 0.0;
        }
        for (int k = 2; k <= nz - 1; ++k) d[k - 1] = (f(k + 1, j, i) - f(k - 1, j, i)) / 2. / dz;
        bad |= tridiagonal(nz, A.data(), B.data(), C.data(), d.data(), out.data(), cp.data());
        for (int k = 1; k <= nz; ++k) dfdz(k, j, i) = out[k - 1];
      }
  }
  if (bad) return fail(c, -4, "zero pivot in tridiagonal solver (diffz)");
  return 0;
}

// laplinv (fft_ops.F90:505-601), in place.  Columns with k2 == 0 are skipped
// (:567) and keep their input values.
static int laplinv(orc_ctx* c, Grid3& f, bool df0) {
  const int nx = f.n3, ny = f.n2, nz = f.n1;
  const double f16 = f4(1.f / 6.f), f13 = f4(1.f / 3.f), f112 = f4(1.f / 12.f), f56 = f4(5.f / 6.f);
  const double dz = c->dz;
  const double i2dz2 = 2. / dz / dz;
  const double idz2 = 1. / dz / dz;
  int bad = 0;
#pragma omp parallel reduction(| : bad)
  {
    std::vector<double> a(nz), b(nz), cc(nz), d(nz), out(nz), cp(nz + 1);
#pragma omp for collapse(2) schedule(static)
    for (int i = 1; i <= nx; ++i)
      for (int j = 1; j <= ny; ++j) {
        double kk = c->k2[kidx(c, j, i)];
        if (kk == 0) continue;
        if (!df0) {
          a[0] = 0.; b[0] = 1.; cc[0] = 0.; d[0] = 0.;
          a[nz - 1] = 0.; b[nz - 1] = 1.; cc[nz - 1] = 0.; d[nz - 1] = 0.;
        } else {
          a[0] = 0.;
          b[0] = -idz2 - f13 * kk;
          cc[0] = idz2 - f16 * kk;
          d[0] = f13 * f(1, j, i) + f16 * f(2, j, i);
          a[nz - 1] = idz2 - f16 * kk;
          b[nz - 1] = -idz2 - f13 * kk;
          cc[nz - 1] = 0.;
          d[nz - 1] = f13 * f(nz, j, i) + f16 * f(nz - 1, j, i);
        }
        for (int k = 2; k <= nz - 1; ++k) {
          a[k - 1] = idz2 - f112 * kk;
          b[k - 1] = -i2dz2 - f56 * kk;
          cc[k - 1] = idz2 - f112 * kk;
          d[k - 1] = f112 * f(k - 1, j, i) + f56 * f(k, j, i) + f112 * f(k + 1, j, i);
        }
        bad |= tridiagonal(nz, a.data(), b.data(), cc.data(), d.data(), out.data(), cp.data());
        for (int k = 1; k <= nz; ++k) f(k, j, i) = out[k - 1];
      }
  }
  if (bad) return fail(c, -4, "zero pivot in tridiagonal solver (laplinv)");
  return 0;
}

// dense-array wrappers for the kernel-level tests
static void dense_spec(const orc_ctx* c, Grid3& g) { g.alloc(c->nzp, c->Ny + 2, c->Nx + 2); }

extern "C" int orc_fft_forward(orc_ctx* c, const double* phys, double* spec) {
  Grid3 src, dst;
  src.alloc(c->nzp, c->Ny, c->Nx);
  for (int k = 1; k <= c->nzp; ++k)
    for (int j = 1; j <= c->Ny; ++j)
      for (int i = 1; i <= c->Nx; ++i) src(k, j, i) = phys[(size_t)(i - 1) + (size_t)c->Nx * ((j - 1) + (size_t)c->Ny * (k - 1))];
  dense_spec(c, dst);
  forward_3dfft(c, src, 0, 0, dst);
  spec_to_dense(dst, spec);
  return 0;
}
extern "C" int orc_fft_backward(orc_ctx* c, const double* spec, double* phys) {
  Grid3 src, dst;
  dense_spec(c, src);
  dense_to_spec(spec, src);
  dst.alloc(c->nzp, c->Ny, c->Nx);
  backward_3dfft(c, src, dst, 0, 0);
  for (int k = 1; k <= c->nzp; ++k)
    for (int j = 1; j <= c->Ny; ++j)
      for (int i = 1; i <= c->Nx; ++i) phys[(size_t)(i - 1) + (size_t)c->Nx * ((j - 1) + (size_t)c->Ny * (k - 1))] = dst(k, j, i);
  return 0;
}
extern "C" int orc_diffx(orc_ctx* c, const double* in, double* out) {
  Grid3 a, b; dense_spec(c, a); dense_spec(c, b);
  dense_to_spec(in, a); diffx(c, a, b); spec_to_dense(b, out);
  return 0;
}
extern "C" int orc_diffy(orc_ctx* c, const double* in, double* out) {
  Grid3 a, b; dense_spec(c, a); dense_spec(c, b);
  dense_to_spec(in, a); diffy(c, a, b); spec_to_dense(b, out);
  return 0;
}
extern "C" int orc_filter(orc_ctx* c, const double* in, double* out) {
  Grid3 a, b; dense_spec(c, a); dense_spec(c, b);
  dense_to_spec(in, a); spectral_filter(c, a, b); spec_to_dense(b, out);
  return 0;
}
extern "C" int orc_diffz(orc_ctx* c, const double* in, double* out, const double* bot, const double* top) {
  Grid3 a, b; dense_spec(c, a); dense_spec(c, b);
  dense_to_spec(in, a);
  int rc;
  if (bot && top) {
    // bot/top dense (Ny+2) x (Nx+2), x' fastest -> (j,i) column-major
    size_t sy = c->Ny + 2, sx = c->Nx + 2;
    std::vector<double> bb(sy * sx), tt(sy * sx);
    for (size_t i = 0; i < sx; ++i)
      for (size_t j = 0; j < sy; ++j) { bb[j + sy * i] = bot[i + sx * j]; tt[j + sy * i] = top[i + sx * j]; }
    rc = diffz(c, a, b, &bb, &tt);
  } else {
    rc = diffz(c, a, b, nullptr, nullptr);
  }
  spec_to_dense(b, out);
  return rc;
}
extern "C" int orc_laplinv(orc_ctx* c, double* inout, int df0) {
  Grid3 a; dense_spec(c, a);
  dense_to_spec(inout, a);
  int rc = laplinv(c, a, df0 != 0);
  spec_to_dense(a, inout);
  return rc;
}
extern "C" int orc_kx_ky_k2(orc_ctx* c, double* kx, double* ky, double* k2, double* filt) {
  size_t sy = c->Ny + 2, sx = c->Nx + 2;
  for (size_t j = 0; j < sy; ++j)
    for (size_t i = 0; i < sx; ++i) {
      size_t o = j + sy * i, d = i + sx * j;
      if (kx) kx[d] = c->kx[o];
      if (ky) ky[d] = c->ky[o];
      if (k2) k2[d] = c->k2[o];
      if (filt) filt[d] = c->filt[o];
    }
  return 0;
}

#include "pmpic_oracle_components.inc"
