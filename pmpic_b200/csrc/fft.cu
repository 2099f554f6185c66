// fft.cu -- semi-spectral 2-D real transforms (y then x) on the B200.
//
// Restates perform_forward_3dfft / perform_backwards_3dfft
// (model_core/src/fft/pencilfft.F90:151-212) for one GPU: no pencil transposes
// (the whole field is in HBM), FFTE's conventions (ffte_mod.F90:66-124,
// ffte/vzfft1d.f:41-68): forward unscaled, inverse scaled by 1/N per 1-D pass,
// complex-to-real passes ignore the imaginary parts of the zero and Nyquist
// modes (the conjugate-symmetric fill of ffte_c2r).
//
// Layouts (x fastest):  phys (Nz+1) x Ny x Nx;  mid (Nz+1) x (Ny+2) x Nx after
// the y pass (Re/Im of y-mode a interleaved at rows 2a, 2a+1);  spec
// (Nz+1) x (Ny+2) x (Nx+2) after the x pass (the reference's four reals per
// (kx, ky) mode, pencilfft.F90:838-864).
//
// Each CTA stages a batch of rows in shared memory and runs a radix-4/2/3/5
// Stockham FFT over them.  Two real rows are packed into one complex row
// (re = row A, im = row B) and separated after the transform, which halves the
// arithmetic of the reference's zero-imaginary complex transforms.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "common.cuh"

namespace pmpic {

namespace {

constexpr int FFT_THREADS = 256;

bool factor(int n, std::vector<int>& out) {
  out.clear();
  int m = n;
  while (m % 4 == 0) { out.push_back(4); m /= 4; }
  while (m % 2 == 0) { out.push_back(2); m /= 2; }
  while (m % 3 == 0) { out.push_back(3); m /= 3; }
  while (m % 5 == 0) { out.push_back(5); m /= 5; }
  return m == 1;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// forward DFT of size R in registers (exp(-2 pi i rt/R))
template <int R>
__device__ __forceinline__ void small_dft(double2* a) {
  if (R == 2) {
    double2 t0 = cadd(a[0], a[1]), t1 = csub(a[0], a[1]);
    a[0] = t0; a[1] = t1;
  } else if (R == 4) {
    double2 t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    double2 t2 = cadd(a[1], a[3]), t3 = csub(a[1], a[3]);
    double2 mt3 = make_double2(t3.y, -t3.x);  // -i * t3
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, mt3);
    a[3] = csub(t1, mt3);
  } else if (R == 3) {
    const double s3 = 0.86602540378443864676;  // sin(2pi/3)
    double2 s = cadd(a[1], a[2]), d = csub(a[1], a[2]);
    double2 b0 = cadd(a[0], s);
    double2 m = make_double2(a[0].x - 0.5 * s.x, a[0].y - 0.5 * s.y);
    double2 r = make_double2(s3 * d.y, -s3 * d.x);  // -i sin(2pi/3) d
    a[0] = b0;
    a[1] = cadd(m, r);
    a[2] = csub(m, r);
  } else if (R == 5) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    double2 t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
    double2 t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
    double2 b0 = cadd(a[0], cadd(t1, t2));
    double2 m1 = make_double2(a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y);
    double2 m2 = make_double2(a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y);
    // -i (s1 t3 + s2 t4) and -i (s2 t3 - s1 t4)
    double2 n1 = make_double2(s1 * t3.y + s2 * t4.y, -(s1 * t3.x + s2 * t4.x));
    double2 n2 = make_double2(s2 * t3.y - s1 * t4.y, -(s2 * t3.x - s1 * t4.x));
    a[0] = b0;
    a[1] = cadd(m1, n1);
    a[4] = csub(m1, n1);
    a[2] = cadd(m2, n2);
    a[3] = csub(m2, n2);
  }
}

template <int R>
__device__ __forceinline__ void stage(const double2* __restrict__ src, double2* __restrict__ dst, int n, int len,
                                      int nrows, int stride_row, const double2* __restrict__ tw) {
  const int m = len / R, s = n / len;
  const int nb = m * s;  // butterflies per row
  for (int e = threadIdx.x; e < nb * nrows; e += blockDim.x) {
    int row = e / nb, b = e - row * nb;
    int p = b / s, q = b - p * s;
    const double2* S = src + (size_t)row * stride_row;
    double2* D = dst + (size_t)row * stride_row;
    double2 a[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = S[q + s * (p + r * m)];
    small_dft<R>(a);
    D[q + s * (R * p)] = a[0];
#pragma unroll
    for (int t = 1; t < R; ++t) D[q + s * (R * p + t)] = cmul(a[t], tw[p * R + t]);
  }
}

// Forward complex FFT of nrows rows held in buf0 (stride_row); buf1 is the
// ping-pong workspace.  Returns the buffer holding the result.
__device__ double2* fft_rows(double2* buf0, double2* buf1, int nrows, int stride_row, const FftPlan& pl,
                             const double2* __restrict__ twbase) {
  double2* src = buf0;
  double2* dst = buf1;
  int len = pl.n;
  for (int st = 0; st < pl.nst; ++st) {
    const double2* tw = twbase + pl.tw_off[st];
    switch (pl.radix[st]) {
      case 4: stage<4>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 2: stage<2>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 3: stage<3>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 5: stage<5>(src, dst, pl.n, len, nrows, stride_row, tw); break;
    }
    __syncthreads();
    len /= pl.radix[st];
    double2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// ---- forward y pass: phys -> mid ------------------------------------------------
// CTA: one z level, TXF consecutive x columns (TXF/2 complex rows of length Ny).
__global__ void __launch_bounds__(FFT_THREADS) k_fwd_y(Geom g, int TXF, FftPlan pl, const double2* __restrict__ tw,
                                                       const double* __restrict__ phys, double* __restrict__ mid) {
  extern __shared__ double2 sm[];
  const int Ny = g.Ny, Nx = g.Nx;
  const int nr = TXF / 2;
  double2* b0 = sm;
  double2* b1 = sm + (size_t)nr * Ny;
  const int x0 = blockIdx.x * TXF, k = blockIdx.y;
  const double* P = phys + (size_t)k * Ny * Nx;
  for (int e = threadIdx.x; e < Ny * TXF; e += blockDim.x) {
    int j = e / TXF, x = e - j * TXF;
    double v = P[(size_t)j * Nx + x0 + x];
    double* c = (double*)&b0[(x >> 1) * Ny + j];
    c[x & 1] = v;
  }
  __syncthreads();
  double2* res = fft_rows(b0, b1, nr, Ny, pl, tw);
  double* M = mid + (size_t)k * g.sy * Nx;
  const int half = Ny / 2 + 1;
  for (int e = threadIdx.x; e < half * TXF; e += blockDim.x) {
    int a = e / TXF, x = e - a * TXF;
    int r = x >> 1;
    double2 z1 = res[r * Ny + a];
    double2 z2 = res[r * Ny + (a == 0 ? 0 : Ny - a)];
    double re, im;
    if ((x & 1) == 0) {  // A = (Z_a + conj Z_{N-a}) / 2
      re = 0.5 * (z1.x + z2.x);
      im = 0.5 * (z1.y - z2.y);
    } else {             // B = (Z_a - conj Z_{N-a}) / (2i)
      re = 0.5 * (z1.y + z2.y);
      im = -0.5 * (z1.x - z2.x);
    }
    M[(size_t)(2 * a) * Nx + x0 + x] = re;
    M[(size_t)(2 * a + 1) * Nx + x0 + x] = im;
  }
}

// ---- forward x pass: mid -> spec ------------------------------------------------
// CTA: RP pairs of consecutive rows (row = (k, j') flattened), rows of length Nx.
__global__ void __launch_bounds__(FFT_THREADS) k_fwd_x(Geom g, int RP, int64_t nrows_total, FftPlan pl,
                                                       const double2* __restrict__ tw, const double* __restrict__ mid,
                                                       double* __restrict__ spec) {
  extern __shared__ double2 sm[];
  const int Nx = g.Nx;
  double2* b0 = sm;
  double2* b1 = sm + (size_t)RP * Nx;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  for (int e = threadIdx.x; e < RP * 2 * Nx; e += blockDim.x) {
    int rr = e / Nx, i = e - rr * Nx;
    int64_t row = row0 + rr;
    double v = row < nrows_total ? mid[(size_t)row * Nx + i] : 0.0;
    double* c = (double*)&b0[(rr >> 1) * Nx + i];
    c[rr & 1] = v;
  }
  __syncthreads();
  double2* res = fft_rows(b0, b1, RP, Nx, pl, tw);
  const int half = Nx / 2 + 1;
  for (int e = threadIdx.x; e < RP * 2 * half; e += blockDim.x) {
    int rr = e / half, b = e - rr * half;
    int64_t row = row0 + rr;
    if (row >= nrows_total) continue;
    int r = rr >> 1;
    double2 z1 = res[r * Nx + b];
    double2 z2 = res[r * Nx + (b == 0 ? 0 : Nx - b)];
    double re, im;
    if ((rr & 1) == 0) {
      re = 0.5 * (z1.x + z2.x);
      im = 0.5 * (z1.y - z2.y);
    } else {
      re = 0.5 * (z1.y + z2.y);
      im = -0.5 * (z1.x - z2.x);
    }
    spec[(size_t)row * g.sx + 2 * b] = re;
    spec[(size_t)row * g.sx + 2 * b + 1] = im;
  }
}

// Build Z_k = A_k + i B_k over the full circle from two half spectra, applying
// ffte_c2r's conjugate-symmetric fill (ffte_mod.F90:108-113): for k > N/2,
// A_k = conj(A_{N-k}); the imaginary parts of modes 0 and N/2 never reach the
// real output, so they are dropped.  Stored conjugated (FFTE computes the
// inverse as conj(FFT(conj(Z)))/N, vzfft1d.f:41-46, 63-68).
__device__ __forceinline__ double2 c2r_pack(double2 A, double2 B, int k, int n) {
  // A, B are the half-spectrum values at min(k, n-k); mirrored if k > n/2
  if (k == 0 || 2 * k == n) {
    A.y = 0.0;
    B.y = 0.0;
  }
  double2 z;
  if (2 * k <= n) {
    z = make_double2(A.x - B.y, A.y + B.x);  // A + iB
  } else {
    // conj(A) + i conj(B) = (A.x + B.y) + i(-A.y + B.x)
    z = make_double2(A.x + B.y, -A.y + B.x);
  }
  return make_double2(z.x, -z.y);  // conj for the forward-transform inverse
}

// ---- inverse x pass: spec -> mid ------------------------------------------------
__global__ void __launch_bounds__(FFT_THREADS) k_inv_x(Geom g, int RP, int64_t nrows_total, FftPlan pl,
                                                       const double2* __restrict__ tw, const double* __restrict__ spec,
                                                       double* __restrict__ mid) {
  extern __shared__ double2 sm[];
  const int Nx = g.Nx;
  double2* b0 = sm;
  double2* b1 = sm + (size_t)RP * Nx;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  for (int e = threadIdx.x; e < RP * Nx; e += blockDim.x) {
    int r = e / Nx, k = e - r * Nx;
    int km = (2 * k <= Nx) ? k : Nx - k;
    int64_t ra = row0 + 2 * r, rb = ra + 1;
    double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
    if (ra < nrows_total) A = make_double2(spec[(size_t)ra * g.sx + 2 * km], spec[(size_t)ra * g.sx + 2 * km + 1]);
    if (rb < nrows_total) B = make_double2(spec[(size_t)rb * g.sx + 2 * km], spec[(size_t)rb * g.sx + 2 * km + 1]);
    b0[r * Nx + k] = c2r_pack(A, B, k, Nx);
  }
  __syncthreads();
  double2* res = fft_rows(b0, b1, RP, Nx, pl, tw);
  const double dn = 1.0 / (double)Nx;
  for (int e = threadIdx.x; e < RP * 2 * Nx; e += blockDim.x) {
    int rr = e / Nx, i = e - rr * Nx;
    int64_t row = row0 + rr;
    if (row >= nrows_total) continue;
    double2 z = res[(rr >> 1) * Nx + i];
    // conj(z) * dn: real part -> row A, imaginary part -> row B
    mid[(size_t)row * Nx + i] = (rr & 1) == 0 ? z.x * dn : -z.y * dn;
  }
}

// ---- inverse y pass: mid -> phys ------------------------------------------------
__global__ void __launch_bounds__(FFT_THREADS) k_inv_y(Geom g, int TXF, FftPlan pl, const double2* __restrict__ tw,
                                                       const double* __restrict__ mid, double* __restrict__ phys) {
  extern __shared__ double2 sm[];
  const int Ny = g.Ny, Nx = g.Nx;
  const int nr = TXF / 2;
  double2* b0 = sm;
  double2* b1 = sm + (size_t)nr * Ny;
  const int x0 = blockIdx.x * TXF, k = blockIdx.y;
  const double* M = mid + (size_t)k * g.sy * Nx;
  // stage the half spectra (Ny/2+1 modes x TXF columns) into b1 first
  const int half = Ny / 2 + 1;
  for (int e = threadIdx.x; e < half * TXF; e += blockDim.x) {
    int a = e / TXF, x = e - a * TXF;
    b1[x * half + a] = make_double2(M[(size_t)(2 * a) * Nx + x0 + x], M[(size_t)(2 * a + 1) * Nx + x0 + x]);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nr * Ny; e += blockDim.x) {
    int r = e / Ny, kk = e - r * Ny;
    int km = (2 * kk <= Ny) ? kk : Ny - kk;
    double2 A = b1[(2 * r) * half + km], B = b1[(2 * r + 1) * half + km];
    b0[r * Ny + kk] = c2r_pack(A, B, kk, Ny);
  }
  __syncthreads();
  double2* res = fft_rows(b0, b1, nr, Ny, pl, tw);
  const double dn = 1.0 / (double)Ny;
  double* P = phys + (size_t)k * Ny * Nx;
  for (int e = threadIdx.x; e < Ny * TXF; e += blockDim.x) {
    int j = e / TXF, x = e - j * TXF;
    double2 z = res[(x >> 1) * Ny + j];
    P[(size_t)j * Nx + x0 + x] = (x & 1) == 0 ? z.x * dn : -z.y * dn;
  }
}

FftPlan make_plan(int n, std::vector<double2>& tw) {
  // twiddles w^(q r) = exp(-2 pi i q r / len) of each Stockham stage, long double accuracy
  FftPlan p{};
  std::vector<int> rad;
  if (!factor(n, rad) || (int)rad.size() > FFT_MAX_STAGES) return p;
  factor(n, rad);
  p.n = n;
  p.nst = (int)rad.size();
  int len = n;
  for (int s = 0; s < p.nst; ++s) {
    int R = rad[s], m = len / R;
    p.radix[s] = R;
    p.tw_off[s] = (int)tw.size();
    for (int q = 0; q < m; ++q)
      for (int r = 0; r < R; ++r) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)((long long)q * r) /
                          (long double)len;
        tw.push_back(make_double2((double)cosl(ang), (double)sinl(ang)));
      }
    len = m;
  }
  return p;
}

int pick_txf(int nx) {
  if (nx % 16 == 0) return 16;
  if (nx % 8 == 0) return 8;
  if (nx % 4 == 0) return 4;
  return 2;
}
int pick_rp(int n) {  // complex rows per CTA for the x passes
  int rp = 4096 / n;
  if (rp < 1) rp = 1;
  if (rp > 8) rp = 8;
  return rp;
}

}  // namespace

int fft_init(pmpic_ctx* ctx) {
  std::vector<int> tmp;
  if (!factor(ctx->g.Nx, tmp) || !factor(ctx->g.Ny, tmp))
    return set_error(ctx, PMPIC_ERR_CONFIG, "nx and ny must have only the prime factors 2, 3 and 5");
  std::vector<double2> tw;
  FftPlan px = make_plan(ctx->g.Nx, tw);
  ctx->ftw_off_y = (int)tw.size();
  ctx->ftw_off_x = 0;
  FftPlan py = make_plan(ctx->g.Ny, tw);
  for (int s = 0; s < py.nst; ++s) py.tw_off[s] -= ctx->ftw_off_y;
  PMPIC_CUDA(cudaMalloc(&ctx->ftw, sizeof(double2) * tw.size()));
  PMPIC_CUDA(cudaMemcpy(ctx->ftw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice));
  ctx->plan_x = px;
  ctx->plan_y = py;
  // per device (the attribute is a property of the function on the current device)
  PMPIC_CUDA(cudaFuncSetAttribute(k_fwd_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  PMPIC_CUDA(cudaFuncSetAttribute(k_inv_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  PMPIC_CUDA(cudaFuncSetAttribute(k_fwd_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  PMPIC_CUDA(cudaFuncSetAttribute(k_inv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  return 0;
}

int fft_forward(pmpic_ctx* ctx, const double* phys, double* spec) {
  TimerScope ts(ctx, T_FFTF);
  const Geom& g = ctx->g;
  const FftPlan& px = ctx->plan_x;
  const FftPlan& py = ctx->plan_y;
  const double2* tw = (const double2*)ctx->ftw;
  int txf = pick_txf(g.Nx);
  size_t sm_y = sizeof(double2) * (size_t)(txf / 2) * g.Ny * 2;
  dim3 gy(g.Nx / txf, g.nzp);
  k_fwd_y<<<gy, FFT_THREADS, sm_y, ctx->stream>>>(g, txf, py, tw + ctx->ftw_off_y, phys, ctx->fftmid); ++ctx->nlaunch;
  int rp = pick_rp(g.Nx);
  int64_t nrows = (int64_t)g.nzp * g.sy;
  size_t sm_x = sizeof(double2) * (size_t)rp * g.Nx * 2;
  k_fwd_x<<<(unsigned)((nrows + 2 * rp - 1) / (2 * rp)), FFT_THREADS, sm_x, ctx->stream>>>(g, rp, nrows, px, tw,
                                                                                        ctx->fftmid, spec); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int fft_backward(pmpic_ctx* ctx, const double* spec, double* phys) {
  TimerScope ts(ctx, T_FFTI);
  const Geom& g = ctx->g;
  const FftPlan& px = ctx->plan_x;
  const FftPlan& py = ctx->plan_y;
  const double2* tw = (const double2*)ctx->ftw;
  int rp = pick_rp(g.Nx);
  int64_t nrows = (int64_t)g.nzp * g.sy;
  size_t sm_x = sizeof(double2) * (size_t)rp * g.Nx * 2;
  k_inv_x<<<(unsigned)((nrows + 2 * rp - 1) / (2 * rp)), FFT_THREADS, sm_x, ctx->stream>>>(g, rp, nrows, px, tw,
                                                                                        spec, ctx->fftmid); ++ctx->nlaunch;
  int txf = pick_txf(g.Nx);
  size_t half = (size_t)g.Ny / 2 + 1;
  size_t sm_y = sizeof(double2) * std::max((size_t)(txf / 2) * g.Ny * 2, (size_t)(txf / 2) * g.Ny + txf * half);
  dim3 gy(g.Nx / txf, g.nzp);
  k_inv_y<<<gy, FFT_THREADS, sm_y, ctx->stream>>>(g, txf, py, tw + ctx->ftw_off_y, ctx->fftmid, phys); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
