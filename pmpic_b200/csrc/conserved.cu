// conserved.cu -- domain totals of volume, h * volume and b * volume over the
// parcels, by a compensated FP64 reduction, in both precision forms.
//
// The reference checks its mixing by these totals (the commented diagnostics
// of parcel_mixing.F90:87-103 and :409-418; report/report.tex:264: volume and
// h * volume conserved to 1e-13).  Each product is split exactly (the FMA gives
// its rounding error), every partial sum is a double-double (Knuth's TwoSum
// for the high part, the errors gathered in the low part), and the partials
// are combined in a fixed order: the result is the FP64 rounding of the exact
// total for any practical parcel count, and two runs give the same bits.  The
// mixed form's FP32 properties are widened exactly before the products.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace pmpic {
namespace {

constexpr int CS_THREADS = 256;

struct DD {
  double hi, lo;
};
// TwoSum: s + e == a + b exactly (no FMA contraction: this file is built with
// --fmad=false, and the explicit __fma_rn below is the only FMA)
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bv = s - a;
  e = (a - (s - bv)) + (b - bv);
}
__device__ __forceinline__ DD dd_add(DD a, double b) {
  double s, e;
  two_sum(a.hi, b, s, e);
  return {s, a.lo + e};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  double s, e;
  two_sum(a.hi, b.hi, s, e);
  return {s, (a.lo + b.lo) + e};
}
// a * b added exactly: the rounded product and its rounding error
__device__ __forceinline__ DD dd_add_prod(DD acc, double a, double b) {
  const double p = a * b;
  const double e = __fma_rn(a, b, -p);
  acc = dd_add(acc, p);
  acc.lo += e;
  return acc;
}

template <class R>
__global__ void __launch_bounds__(CS_THREADS) k_sums(int64_t n, const R* __restrict__ vol, const R* __restrict__ h,
                                                      const R* __restrict__ b, double* __restrict__ part) {
  DD s0{0.0, 0.0}, s1{0.0, 0.0}, s2{0.0, 0.0};
  const int64_t stride = (int64_t)gridDim.x * CS_THREADS;
  for (int64_t i = (int64_t)blockIdx.x * CS_THREADS + threadIdx.x; i < n; i += stride) {
    const double v = (double)vol[i];
    s0 = dd_add(s0, v);
    s1 = dd_add_prod(s1, v, (double)h[i]);
    s2 = dd_add_prod(s2, v, (double)b[i]);
  }
  // fixed-order tree over the block
  __shared__ DD red[3][CS_THREADS];
  red[0][threadIdx.x] = s0;
  red[1][threadIdx.x] = s1;
  red[2][threadIdx.x] = s2;
  __syncthreads();
  for (int w = CS_THREADS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = dd_add(red[q][threadIdx.x], red[q][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x < 3) {
    part[(size_t)blockIdx.x * 6 + 2 * threadIdx.x] = red[threadIdx.x][0].hi;
    part[(size_t)blockIdx.x * 6 + 2 * threadIdx.x + 1] = red[threadIdx.x][0].lo;
  }
}

// one warp per quantity: lane l sums the partials of blocks l, l + 32, ... in
// order, then a fixed butterfly over the lanes
__global__ void k_sums_final(int nblocks, const double* __restrict__ part, DevInfo* info) {
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (q >= 3) return;
  DD s{0.0, 0.0};
  for (int k = lane; k < nblocks; k += 32) s = dd_add(s, DD{part[(size_t)k * 6 + 2 * q], part[(size_t)k * 6 + 2 * q + 1]});
  for (int o = 16; o > 0; o >>= 1) {
    const DD t{__shfl_xor_sync(0xffffffffu, s.hi, o), __shfl_xor_sync(0xffffffffu, s.lo, o)};
    s = (lane & o) ? dd_add(t, s) : dd_add(s, t);  // the lower lane's sum first on both sides
  }
  if (lane == 0) info->sums[q] = s.hi + s.lo;
}

}  // namespace

int conserved_sums(pmpic_ctx* ctx) {
  const int64_t n = ctx->n;
  const int nb = (int)std::min<int64_t>(CS_BLOCKS, std::max<int64_t>(1, (n + CS_THREADS - 1) / CS_THREADS));
  if (ctx->mixed) {
    k_sums<float><<<nb, CS_THREADS, 0, ctx->stream>>>(n, propf(ctx, PMPIC_PROP_VOL), propf(ctx, PMPIC_PROP_H),
                                                       propf(ctx, PMPIC_PROP_B), ctx->csum);
  } else {
    k_sums<double><<<nb, CS_THREADS, 0, ctx->stream>>>(n, prop(ctx, PMPIC_PROP_VOL), prop(ctx, PMPIC_PROP_H),
                                                        prop(ctx, PMPIC_PROP_B), ctx->csum);
  }
  k_sums_final<<<1, 96, 0, ctx->stream>>>(nb, ctx->csum, ctx->dinfo);
  ctx->nlaunch += 2;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
