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

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace pmpic {

namespace {

constexpr int FFT_THREADS = 256;
constexpr int FS_THREADS = 128;

bool factor(int n, std::vector<int>& out) {
  out.clear();
  int m = n;
  while (m % 4 == 0) { out.push_back(4); m /= 4; }
  while (m % 2 == 0) { out.push_back(2); m /= 2; }
  while (m % 3 == 0) { out.push_back(3); m /= 3; }
  while (m % 5 == 0) { out.push_back(5); m /= 5; }
  return m == 1;
}

// the four-step split used for a row length (0: none)
void fs_split(int n, int& n1, int& n2) {
  n1 = n2 = 0;
  switch (n) {
    case 16: n1 = 4; n2 = 4; break;
    case 32: n1 = 8; n2 = 4; break;
    case 64: n1 = 8; n2 = 8; break;
    case 128: n1 = 16; n2 = 8; break;
    case 256: n1 = 16; n2 = 16; break;
    default: break;
  }
}

// four-step twiddles W_n^(n2 k1), [n2 * n1 + k1], long double accuracy
void fs_twiddles(FftPlan& p, std::vector<double2>& tw) {
  fs_split(p.n, p.n1, p.n2);
  p.tw4_off = (int)tw.size();
  if (!p.n1) return;
  for (int n2 = 0; n2 < p.n2; ++n2)
    for (int k1 = 0; k1 < p.n1; ++k1) {
      long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)(n2 * k1) / (long double)p.n;
      tw.push_back(make_double2((double)cosl(ang), (double)sinl(ang)));
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

// the transform kernels, once per precision
namespace f64 {
using real = double;
using real2 = double2;
__host__ __device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
#include "fft_impl.cuh"
}  // namespace f64
namespace f32 {
using real = float;
using real2 = float2;
__host__ __device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
#include "fft_impl.cuh"
}  // namespace f32

int fft_init(pmpic_ctx* ctx) {
  std::vector<int> tmp;
  if (!factor(ctx->g.Nx, tmp) || !factor(ctx->g.Ny, tmp))
    return set_error(ctx, PMPIC_ERR_CONFIG, "nx and ny must have only the prime factors 2, 3 and 5");
  std::vector<double2> tw;
  FftPlan px = make_plan(ctx->g.Nx, tw);
  fs_twiddles(px, tw);
  ctx->ftw_off_y = (int)tw.size();
  ctx->ftw_off_x = 0;
  FftPlan py = make_plan(ctx->g.Ny, tw);
  fs_twiddles(py, tw);
  for (int s = 0; s < py.nst; ++s) py.tw_off[s] -= ctx->ftw_off_y;
  py.tw4_off -= ctx->ftw_off_y;
  // the y passes of the four-step path take 16 columns per CTA
  if (ctx->g.Nx % 16 != 0) py.n1 = py.n2 = 0;
  PMPIC_CUDA(cudaMalloc(&ctx->ftw, sizeof(double2) * tw.size()));
  PMPIC_CUDA(cudaMemcpy(ctx->ftw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice));
  // the FP32 table: the same twiddles rounded once to single precision
  std::vector<float2> tw32(tw.size());
  for (size_t i = 0; i < tw.size(); ++i) tw32[i] = make_float2((float)tw[i].x, (float)tw[i].y);
  PMPIC_CUDA(cudaMalloc(&ctx->ftw32, sizeof(float2) * tw32.size()));
  PMPIC_CUDA(cudaMemcpy(ctx->ftw32, tw32.data(), sizeof(float2) * tw32.size(), cudaMemcpyHostToDevice));
  ctx->plan_x = px;
  ctx->plan_y = py;
  // per device (the attribute is a property of the function on the current device)
  PMPIC_CUDA(f64::fft_attributes());
  PMPIC_CUDA(f32::fft_attributes());
  return 0;
}

int fft_forward(pmpic_ctx* ctx, const double* phys, double* spec) {
  return f64::fft_forward_impl(ctx, phys, spec, ctx->fftmid, (const double2*)ctx->ftw);
}
int fft_backward(pmpic_ctx* ctx, const double* spec, double* phys) {
  return fft_backward(ctx, spec, phys, SpecIn<double>{}, PhysOut<double>{});
}
int fft_backward(pmpic_ctx* ctx, const double* spec, double* phys, const SpecIn<double>& si,
                 const PhysOut<double>& po) {
  return f64::fft_backward_impl(ctx, spec, phys, ctx->fftmid, (const double2*)ctx->ftw, si, po);
}
int fft_forward(pmpic_ctx* ctx, const float* phys, float* spec) {
  return f32::fft_forward_impl(ctx, phys, spec, (float*)ctx->fftmid, (const float2*)ctx->ftw32);
}
int fft_backward(pmpic_ctx* ctx, const float* spec, float* phys) {
  return fft_backward(ctx, spec, phys, SpecIn<float>{}, PhysOut<float>{});
}
int fft_backward(pmpic_ctx* ctx, const float* spec, float* phys, const SpecIn<float>& si, const PhysOut<float>& po) {
  return f32::fft_backward_impl(ctx, spec, phys, (float*)ctx->fftmid, (const float2*)ctx->ftw32, si, po);
}

}  // namespace pmpic
