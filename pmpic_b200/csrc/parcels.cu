// parcels.cu -- parcel-side components on the B200: the RK4 stage update, the
// single-GPU parcel haloswap, parcel splitting and residual-grid mixing.
//
// The integer bookkeeping of the reference's serial loops (migration re-slot
// order, split child slots, mixing keep / npercell / new-parcel slots /
// backfill order) is reproduced exactly with deterministic stream compaction:
// per-block counts, an exclusive scan, and block-local ranks, so every list is
// built in ascending slot (or reference loop) order.
#include <cuda_runtime.h>

#include "common.cuh"

namespace pmpic {

int scan_excl(pmpic_ctx* ctx, const int32_t* in, int64_t n, int32_t* out);
int launch_mix_grids(pmpic_ctx* ctx, bool any_removed);
int launch_kept_corners(pmpic_ctx* ctx, const int32_t* olist, const int32_t* nnew, int64_t hnew);

namespace {

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- deterministic compaction ------------------------------------------------------
// Pred(i) -> bool over i in [0, n); list[] receives the true indices ascending.
// A CTA of 256 threads covers CCH chunks of 256 consecutive items (thread t
// takes item t of each chunk, so every load is coalesced and each thread has
// CCH independent loads in flight).  Order inside a CTA is (chunk, warp,
// lane), which is ascending item order.
constexpr int CCH = 32;              // chunks per CTA
constexpr int CITEMS = 256 * CCH;    // items per CTA
// the per-CTA counts of k_count for a direction array, accumulated by the
// kernels that classify (one ballot per warp, an atomic only where a warp
// holds a mover; a warp's items lie in one CTA range)
__device__ __forceinline__ void count_mover(int64_t t, bool moves, int32_t* __restrict__ blockcnt) {
  const unsigned b = __ballot_sync(__activemask(), moves);
  if (b && (threadIdx.x & 31) == __ffs(__activemask()) - 1) atomicAdd(&blockcnt[t / CITEMS], __popc(b));
}
template <class Pred>
__global__ void __launch_bounds__(256) k_count(Pred pr, int64_t n, int32_t* __restrict__ blockcnt) {
  __shared__ int ws[8];
  const int64_t base = (int64_t)blockIdx.x * CITEMS + threadIdx.x;
  int c = 0;
#pragma unroll 8
  for (int j = 0; j < CCH; ++j) {
    const int64_t i = base + 256 * j;
    c += (i < n && pr(i)) ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += ws[w];
    blockcnt[blockIdx.x] = t;
  }
}
template <class Pred>
__global__ void __launch_bounds__(256) k_write(Pred pr, int64_t n, const int32_t* __restrict__ blockoff,
                                               int32_t* __restrict__ list) {
  __shared__ int wc[CCH * 8];  // per (chunk, warp): count, then exclusive offset within the CTA
  // the lists are sparse (movers, splits, removals, under-populated cells):
  // a CTA whose range holds none leaves at once (blockoff has nb + 1 entries)
  if (blockoff[blockIdx.x + 1] == blockoff[blockIdx.x]) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * CITEMS + threadIdx.x;
  uint32_t mask = 0;
#pragma unroll 8
  for (int j = 0; j < CCH; ++j) {
    const int64_t i = base + 256 * j;
    const bool f = i < n && pr(i);
    mask |= (uint32_t)f << j;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wc[j * 8 + w] = __popc(b);
  }
  __syncthreads();
  if (w == 0) {  // exclusive scan of the CCH*8 counts in (chunk, warp) order, 8 per lane
    int v[8], s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      v[q] = wc[lane * 8 + q];
      s += v[q];
    }
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    int ex = incl - s;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      wc[lane * 8 + q] = ex;
      ex += v[q];
    }
  }
  __syncthreads();
  const int32_t off = blockoff[blockIdx.x];
  const unsigned lt = (1u << lane) - 1;
#pragma unroll 8
  for (int j = 0; j < CCH; ++j) {
    const bool f = (mask >> j) & 1u;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (f) list[off + wc[j * 8 + w] + __popc(b & lt)] = (int32_t)(base + 256 * j);
  }
}

struct PredKeepEq {
  const int32_t* keep;
  int v;
  __device__ bool operator()(int64_t i) const { return keep[i] == v; }
};
// the removed class (vol < vmin, parcel_mixing.F90:488), from the volumes; R the form's type
template <class R>
struct PredVolBelow {
  const R* vol;
  R vmin;
  __device__ bool operator()(int64_t i) const { return vol[i] < vmin; }
};
struct PredDirNZ {
  const int8_t* dir;
  __device__ bool operator()(int64_t i) const { return dir[i] != 0; }
};
struct PredFlag {
  const int32_t* f;
  __device__ bool operator()(int64_t i) const { return f[i] != 0; }
};
// the split criterion on an already advanced FP32 stretch (parcel_splitting.F90:76)
struct PredStretchM {
  const float* s;
  __device__ bool operator()(int64_t i) const { return s[i] > 4.f; }
};
// cell in the reference's loop order o = (i*Ny + j)*Nz + k (parcel_mixing.F90:160-162)
struct PredNewCell {
  const int32_t* npc;
  int Nx, Ny, Nz;
  __device__ bool operator()(int64_t o) const {
    int k = (int)(o % Nz);
    int j = (int)((o / Nz) % Ny);
    int i = (int)(o / ((int64_t)Nz * Ny));
    return npc[((int64_t)k * Ny + j) * Nx + i] < 3;
  }
};

// ---- packed gather grids ------------------------------------------------------------
// The RK4 pass gathers six grids (u, v, w, dp, dq, dr) at every parcel.  Parcels
// stream in z-fastest cell order while grids are x fastest, so one stage first
// repacks the six into G6[i][j][k][6] (z fastest, fields interleaved): a cell's
// four xy corners then hold their two levels and six fields in 12 consecutive
// values, and the cells of a warp (consecutive in z) share lines.
// x extent of a tile: 64 values (256-byte row segments) on the FP32 form, 32
// on the FP64 path (its tile would not fit the static shared memory)
template <class R>
struct PkT {
  static constexpr int value = sizeof(R) == 4 ? 64 : 32;
};
constexpr int PK_K = 16;  // z extent of a tile
template <class R>
__global__ void __launch_bounds__(256) k_pack(Geom g, const R* __restrict__ G0, const R* __restrict__ G1,
                                              const R* __restrict__ G2, const R* __restrict__ G3,
                                              const R* __restrict__ G4, const R* __restrict__ G5,
                                              R* __restrict__ out) {
  constexpr int NF = 6;
  constexpr int PK_T = PkT<R>::value;
  constexpr int TS = PK_K * (PK_T + 1) + 1;  // per-field tile stride, odd
  __shared__ R tile[NF * TS];
  const int i0 = blockIdx.x * PK_T, k0 = blockIdx.y * PK_K, j = blockIdx.z;
  const R* G[NF] = {G0, G1, G2, G3, G4, G5};
  const int ni = min(PK_T, g.Nx - i0), nk = min(PK_K, g.nzp - k0);
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    for (int e = threadIdx.x; e < PK_K * PK_T; e += blockDim.x) {
      const int kk = e / PK_T, ii = e - kk * PK_T;
      if (kk < nk && ii < ni) tile[f * TS + kk * (PK_T + 1) + ii] = G[f][((size_t)(k0 + kk) * g.Ny + j) * g.Nx + i0 + ii];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NF * PK_K * PK_T; e += blockDim.x) {
    const int ii = e / (NF * PK_K), r = e - ii * NF * PK_K;
    const int kk = r / NF, f = r - kk * NF;
    if (kk < nk && ii < ni)
      out[(((size_t)(i0 + ii) * g.Ny + j) * g.nzp + k0 + kk) * NF + f] = tile[f * TS + kk * (PK_T + 1) + ii];
  }
}
template <class R>
static void pack6(pmpic_ctx* ctx, const R* const* grids, R* out) {
  const Geom& g = ctx->g;
  constexpr int PK_T = PkT<R>::value;
  dim3 gr((g.Nx + PK_T - 1) / PK_T, (g.nzp + PK_K - 1) / PK_K, g.Ny);
  k_pack<R><<<gr, 256, 0, ctx->stream>>>(g, grids[0], grids[1], grids[2], grids[3], grids[4], grids[5], out);
  ++ctx->nlaunch;
}
// the six fields at the two levels of xy corner (ci, cj) of a cell of level ck:
// lo[f] at ck, hi[f] at ck+1
__device__ __forceinline__ void corner6(const Geom& g, const double* __restrict__ G6, int ci, int cj, int ck,
                                        double* lo, double* hi) {
  const double2* p = (const double2*)(G6 + (((size_t)ci * g.Ny + cj) * g.nzp + ck) * 6);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4], f = p[5];
  lo[0] = a.x; lo[1] = a.y; lo[2] = b.x; lo[3] = b.y; lo[4] = c.x; lo[5] = c.y;
  hi[0] = d.x; hi[1] = d.y; hi[2] = e.x; hi[3] = e.y; hi[4] = f.x; hi[5] = f.y;
}
__device__ __forceinline__ void corner6(const Geom& g, const float* __restrict__ G6, int ci, int cj, int ck,
                                        float* lo, float* hi) {
  const float2* p = (const float2*)(G6 + (((size_t)ci * g.Ny + cj) * g.nzp + ck) * 6);
  const float2 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4], f = p[5];
  lo[0] = a.x; lo[1] = a.y; lo[2] = b.x; lo[3] = b.y; lo[4] = c.x; lo[5] = c.y;
  hi[0] = d.x; hi[1] = d.y; hi[2] = e.x; hi[3] = e.y; hi[4] = f.x; hi[5] = f.y;
}
// grid2par (parcel_interpolation.F90:299-321) of all six packed fields: z,
// then y, then x, in the reference's operation order (FP64 path: every product
// and sum rounded as there; the FP32 form fuses each product into its sum)
template <class R>
__device__ __forceinline__ void g2p_packed(const Geom& g, const R* __restrict__ G6, int ci, int cj, int ck, R delx,
                                           R dely, R delz, R* d) {
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  const R ez = R(1) - delz, ey = R(1) - dely, ex = R(1) - delx;
  R lo[6], hi[6], c00[6], c0[6];
  // x corner i: c0 = c00 (1-dely) + c10 dely, with c.. = lower (1-delz) + upper delz
  corner6(g, G6, ci, cj, ck, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = lo[f] * ez + hi[f] * delz;
  corner6(g, G6, ci, cj1, ck, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c0[f] = c00[f] * ey + (lo[f] * ez + hi[f] * delz) * dely;
  // x corner i+1
  corner6(g, G6, ci1, cj, ck, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = lo[f] * ez + hi[f] * delz;
  corner6(g, G6, ci1, cj1, ck, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) d[f] = c0[f] * ex + (c00[f] * ey + (lo[f] * ez + hi[f] * delz) * dely) * delx;
}
// The FP32 form of the same, over a corner loader: corner(c, lo, hi) gives the
// six fields at the two levels of xy corner c = 0: (i, j), 1: (i, j+1),
// 2: (i+1, j), 3: (i+1, j+1); each product is fused into its sum
template <class Corner>
__device__ __forceinline__ void g2p_packed_f(Corner corner, float delx, float dely, float delz, float* d) {
  const float ez = 1.f - delz, ey = 1.f - dely, ex = 1.f - delx;
  float lo[6], hi[6], c00[6], c0[6];
  corner(0, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = __fmaf_rn(hi[f], delz, lo[f] * ez);
  corner(1, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c0[f] = __fmaf_rn(__fmaf_rn(hi[f], delz, lo[f] * ez), dely, c00[f] * ey);
  corner(2, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = __fmaf_rn(hi[f], delz, lo[f] * ez);
  corner(3, lo, hi);
#pragma unroll
  for (int f = 0; f < 6; ++f)
    d[f] = __fmaf_rn(__fmaf_rn(__fmaf_rn(hi[f], delz, lo[f] * ez), dely, c00[f] * ey), delx, c0[f] * ex);
}
template <>
__device__ __forceinline__ void g2p_packed<float>(const Geom& g, const float* __restrict__ G6, int ci, int cj, int ck,
                                                  float delx, float dely, float delz, float* d) {
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  g2p_packed_f(
      [&](int c, float* lo, float* hi) { corner6(g, G6, (c & 2) ? ci1 : ci, (c & 1) ? cj1 : cj, ck, lo, hi); }, delx,
      dely, delz, d);
}

// ---- staged gather window (mixed form) ---------------------------------------------
// An RK4 CTA's parcels are consecutive slots, and slots follow cell order (the
// set-up writes parcels cell by cell and they move little in a stage), so
// they sit mostly in one column of cells, in a run of levels.  The CTA copies
// the four corner columns of that run out of the packed grids into shared
// memory with bulk asynchronous copies (cp.async.bulk, completed on an
// mbarrier; no multicast) at its start, while its threads load their parcel
// state; the threads then interpolate from shared memory instead of making a
// dependent round trip to L2 after their cell ids arrive.  The window is
// placed by a hint, the cell the CTA's first parcel moved to at the previous
// stage (written by that stage; L2-resident); a parcel outside the window
// (or any parcel, if the hint is stale) gathers from the packed grids as
// before.  The values and their arithmetic are the same either way.
constexpr int GW_KW = 48;  // levels per staged corner column: 48 * 24 bytes, a multiple of 16
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// bytes (a multiple of 16) from global src to shared dst (both 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
// the barrier's first phase, with a bound on the tries (false: gave up)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, 0)) return true;
  return false;
}
// window of corner columns (i0|i0+1, j0|j0+1) around hint cell (i0, j0, k0):
// column c holds levels s[c] .. s[c] + GW_KW - 1 (s[c] is k0 or k0 - 1, whichever
// starts the copy on a 16-byte boundary); a parcel in column (i0, j0) with
// k0 <= ck <= k0 + GW_KW - 3 finds both its levels in every column
struct GatherWindow {
  int i0, j0, k0;
  int s[4];
};
__device__ __forceinline__ void window_issue(const Geom& g, const float* G6, int32_t hint, GatherWindow& w,
                                             float* S, uint64_t* bar) {
  if (hint < 0 || hint >= g.ncell) hint = 0;
  int i0, j0, k0;
  cell_decode(g, hint, i0, j0, k0);
  const int i1 = i0 + 1 == g.Nx ? 0 : i0 + 1, j1 = j0 + 1 == g.Ny ? 0 : j0 + 1;
  int64_t src[4];
  w.i0 = i0;
  w.j0 = j0;
  w.k0 = k0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int64_t base = ((int64_t)((c & 2) ? i1 : i0) * g.Ny + ((c & 1) ? j1 : j0)) * g.nzp;
    const int s0 = k0 - (int)((base + k0) & 1);  // an even point index: 24-byte records on a 16-byte boundary
    w.s[c] = s0;
    src[c] = base + s0;
  }
  // the window is written before the arrive, which releases it to the waiting threads
  mbar_expect_tx(bar, 4u * GW_KW * 24u);
  // (at most GW_KW levels past the grids' end: the pack buffer holds twice their size)
#pragma unroll
  for (int c = 0; c < 4; ++c) bulk_g2s(S + c * GW_KW * 6, G6 + src[c] * 6, GW_KW * 24u, bar);
}
// the six fields at levels lev and lev + 1 of staged corner column c
__device__ __forceinline__ void corner6_staged(const float* S, int c, int lev, float* lo, float* hi) {
  const float2* p = (const float2*)(S + (c * GW_KW + lev) * 6);
  const float2 a = p[0], b = p[1], cc = p[2], d = p[3], e = p[4], f = p[5];
  lo[0] = a.x; lo[1] = a.y; lo[2] = b.x; lo[3] = b.y; lo[4] = cc.x; lo[5] = cc.y;
  hi[0] = d.x; hi[1] = d.y; hi[2] = e.x; hi[3] = e.y; hi[4] = f.x; hi[5] = f.y;
}

// The FP64 path's window: its packed records are 48 bytes (always on a 16-byte
// boundary), so every column starts at the hint's level k0 and holds the
// levels k0 .. k0 + len - 1 that its column has (len <= GWD_KW; no copy reads
// past the grids).  The hint is the cell of the CTA's first parcel as the
// binning before the stage found it, so it is exact.
constexpr int GWD_KW = 40;  // levels per staged corner column, FP64
struct GatherWindowD {
  int i0, j0, k0, len;
};
__device__ __forceinline__ void window_issue_d(const Geom& g, const double* G6, int32_t hint, GatherWindowD& w,
                                               double* S, uint64_t* bar) {
  if (hint < 0 || hint >= g.ncell) hint = 0;
  int i0, j0, k0;
  cell_decode(g, hint, i0, j0, k0);
  const int i1 = i0 + 1 == g.Nx ? 0 : i0 + 1, j1 = j0 + 1 == g.Ny ? 0 : j0 + 1;
  const int len = min(GWD_KW, g.nzp - k0);
  w.i0 = i0;
  w.j0 = j0;
  w.k0 = k0;
  w.len = len;
  // the window is written before the arrive, which releases it to the waiting threads
  mbar_expect_tx(bar, 4u * (uint32_t)len * 48u);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int64_t base = ((int64_t)((c & 2) ? i1 : i0) * g.Ny + ((c & 1) ? j1 : j0)) * g.nzp;
    bulk_g2s(S + c * GWD_KW * 6, G6 + (base + k0) * 6, (uint32_t)len * 48u, bar);
  }
}
// grid2par of the six fields from a staged window, in the FP64 path's order
// (the same operations as g2p_packed<double>)
__device__ __forceinline__ void g2p_staged_d(const double* S, int lev, double delx, double dely, double delz,
                                             double* d) {
  const double ez = 1.0 - delz, ey = 1.0 - dely, ex = 1.0 - delx;
  double lo[6], hi[6], c00[6], c0[6];
  auto corner = [&](int c) {
    const double2* p = (const double2*)(S + (c * GWD_KW + lev) * 6);
    const double2 a = p[0], b = p[1], cc = p[2], dd = p[3], e = p[4], f = p[5];
    lo[0] = a.x; lo[1] = a.y; lo[2] = b.x; lo[3] = b.y; lo[4] = cc.x; lo[5] = cc.y;
    hi[0] = dd.x; hi[1] = dd.y; hi[2] = e.x; hi[3] = e.y; hi[4] = f.x; hi[5] = f.y;
  };
  corner(0);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = lo[f] * ez + hi[f] * delz;
  corner(1);
#pragma unroll
  for (int f = 0; f < 6; ++f) c0[f] = c00[f] * ey + (lo[f] * ez + hi[f] * delz) * dely;
  corner(2);
#pragma unroll
  for (int f = 0; f < 6; ++f) c00[f] = lo[f] * ez + hi[f] * delz;
  corner(3);
#pragma unroll
  for (int f = 0; f < 6; ++f) d[f] = c0[f] * ex + (c00[f] * ey + (lo[f] * ez + hi[f] * delz) * dely) * delx;
}

// ---- RK4 stage (rk4_integrator.F90:95-319) -----------------------------------------
// One pass per stage: the deferred grid2par gathers of vort2vel (u, v, w ->
// dxdt, dydt, dzdt, vort2vel.F90:325-327) and of vorticity_tendency (dp, dq,
// dr -> dpdt, dqdt, drdt, vorticity_tendency.F90:273-275) when pending, the
// stage update, and the first step of the following parcel haloswap: the z
// reflection (haloswap.F90:440-456) and the direction classification
// (:296-437).
struct RkPtrs {
  double* s[6];
  double* o[6];
  double* f[6];
  double* d[6];
  const double* grid[6];  // u, v, w, dp, dq, dr
  const double* g6;       // the six packed (k_pack), when both gathers are pending
  const int32_t* whint;   // per CTA: the cell of its first parcel (the binning's)
};

__device__ __forceinline__ int classify_dir(const Geom& g, double x, double y) {
  const double xmin = g.hxmin, xmax = g.hxmax, ymin = g.hymin, ymax = g.hymax;
  int d = 0;
  if (y >= ymax && x >= xmin && x < xmax) d = 1;        // N
  else if (y < ymin && x >= xmin && x < xmax) d = 5;    // S
  else if (x >= xmax && y >= ymin && y < ymax) d = 3;   // E
  else if (x < xmin && y >= ymin && y < ymax) d = 7;    // W
  else if (x >= xmax && y >= ymax) d = 2;               // NE
  else if (x < xmin && y >= ymax) d = 8;                // NW
  else if (x >= xmax && y < ymin) d = 4;                // SE
  else if (x < xmin && y < ymin) d = 6;                 // SW
  return d;
}

template <bool GU, bool GP>
__global__ void __launch_bounds__(256, 4) k_rk4(Geom g, int64_t n, RkPtrs P, int stage, const double* __restrict__ dtp,
                      const int32_t* __restrict__ cell, const double* __restrict__ del, int64_t cap,
                      int8_t* __restrict__ dir, int store_d, int32_t* __restrict__ dircnt) {
  // the staged gather window, when both gathers are pending (the step's path)
  __shared__ __align__(16) double gws[(GU && GP) ? 4 * GWD_KW * 6 : 2];
  __shared__ __align__(8) uint64_t gwbar;
  __shared__ GatherWindowD gw;
  if constexpr (GU && GP) {
    if (threadIdx.x == 0) mbar_init(&gwbar, 1);
    __syncthreads();
    if (threadIdx.x == 0) window_issue_d(g, P.g6, P.whint[blockIdx.x], gw, gws, &gwbar);
  }
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;  // (thread 0 stays: the copies complete before the CTA ends)
  bool ready = false;
  const double dt = *dtp;  // state%dtm (rk4_integrator.F90:102)
  const double dt6 = dt / 6, dt2 = dt / 2, dt3 = dt / 3;
  // every load of this parcel is issued before the first store, so none of
  // them waits behind another
  double sv[6], ov[6], fv[6], d[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    if (stage == 1) sv[v] = P.s[v][t];
    if (stage == 2 || stage == 3) ov[v] = P.o[v][t];
    if (stage >= 2) fv[v] = P.f[v][t];
    if ((v < 3 && !GU) || (v >= 3 && !GP)) d[v] = P.d[v][t];
  }
  const int32_t id = (GU || GP) ? cell[t] : -1;
  bool gathered = false;
  if ((GU || GP) && id >= 0) {  // id < 0: binning failed and reported the error
    gathered = true;
    const double delx = del[t], dely = del[cap + t], delz = del[2 * cap + t];
    const int ck = id % g.Nz, cj = (id / g.Nz) % g.Ny, ci = id / (g.Nz * g.Ny);
    const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
    const size_t r00 = ((size_t)ck * g.Ny + cj) * g.Nx, r01 = ((size_t)ck * g.Ny + cj1) * g.Nx;
    const size_t r10 = ((size_t)(ck + 1) * g.Ny + cj) * g.Nx, r11 = ((size_t)(ck + 1) * g.Ny + cj1) * g.Nx;
    if constexpr (GU && GP) {
      ready = mbar_wait_bounded(&gwbar);
      if (ready && ci == gw.i0 && cj == gw.j0 && ck >= gw.k0 && ck <= gw.k0 + gw.len - 2)
        g2p_staged_d(gws, ck - gw.k0, delx, dely, delz, d);
      else
        g2p_packed<double>(g, P.g6, ci, cj, ck, delx, dely, delz, d);
    }
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      if ((v < 3 && !GU) || (v >= 3 && !GP) || (GU && GP)) continue;
      const double* G = P.grid[v];
      // grid2par, parcel_interpolation.F90:299-321
      double c00 = G[r00 + ci] * (1 - delz) + G[r10 + ci] * delz;
      double c01 = G[r00 + ci1] * (1 - delz) + G[r10 + ci1] * delz;
      double c10 = G[r01 + ci] * (1 - delz) + G[r11 + ci] * delz;
      double c11 = G[r01 + ci1] * (1 - delz) + G[r11 + ci1] * delz;
      double c0 = c00 * (1 - dely) + c10 * dely;
      double c1 = c01 * (1 - dely) + c11 * dely;
      d[v] = c0 * (1 - delx) + c1 * delx;
    }
  } else if (GU || GP) {
#pragma unroll
    for (int v = 0; v < 6; ++v) d[v] = P.d[v][t];
  }
  double snew[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    if (stage == 1) {
      ov[v] = sv[v];
      fv[v] = sv[v] + dt6 * d[v];
      snew[v] = sv[v] + dt2 * d[v];
    } else if (stage == 2) {
      fv[v] = fv[v] + dt3 * d[v];
      snew[v] = ov[v] + dt2 * d[v];
    } else if (stage == 3) {
      fv[v] = fv[v] + dt3 * d[v];
      snew[v] = ov[v] + dt * d[v];
    } else {
      fv[v] = fv[v] + dt6 * d[v];
      snew[v] = fv[v];
    }
  }
  // parcel haloswap, first part: reflect z at the walls, classify
  double z = snew[2];
  if (z < g.pzmin) z = g.pzmin + (g.pzmin - z);
  else if (z > g.pzmax) z = g.pzmax - (z - g.pzmax);
  snew[2] = z;
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    if (store_d && gathered && ((v < 3 && GU) || (v >= 3 && GP))) P.d[v][t] = d[v];
    if (stage == 1) P.o[v][t] = ov[v];
    P.f[v][t] = fv[v];
    P.s[v][t] = snew[v];
  }
  const int dr = classify_dir(g, snew[0], snew[1]);
  dir[t] = (int8_t)dr;
  count_mover(t, dr != 0, dircnt);
  if constexpr (GU && GP) {
    if (threadIdx.x == 0 && !ready) mbar_wait_bounded(&gwbar);  // no copy in flight when the CTA ends
  }
}

// ---- parcel haloswap (parcels/haloswap.F90:109-289, one rank) -------------------------
// Reflect z at the walls (:440-456), then classify into N,NE,E,SE,S,SW,W,NW
// = 1..8 (:296-437) with the limits x_coords(3), x_coords(Nx+3) (:314-318).
__global__ void k_reflect_classify(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                                   double* __restrict__ Z, int8_t* __restrict__ dir) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double z = Z[i];
  if (z < g.pzmin) Z[i] = g.pzmin + (g.pzmin - z);
  else if (z > g.pzmax) Z[i] = g.pzmax - (z - g.pzmax);
  dir[i] = (int8_t)classify_dir(g, X[i], Y[i]);
}

// Stable partition of the ascending moved list V by direction 1..8 (single
// CTA; the moved list is short): M = the order in which the reference sends,
// receives and unpacks the parcels (dir 1..8, ascending index within a dir).
__global__ void k_partition_dirs(const int32_t* __restrict__ V, const int32_t* __restrict__ nmov,
                                 const int8_t* __restrict__ dir, int32_t* __restrict__ M) {
  __shared__ int base[9];
  __shared__ int cnt[9];
  __shared__ int wcnt[32][9];
  const int nm = *nmov;
  if (threadIdx.x < 9) cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < nm; t += blockDim.x) atomicAdd(&cnt[dir[V[t]]], 1);  // integer: order-free
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int d = 1; d <= 8; ++d) {
      base[d] = s;
      s += cnt[d];
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = 0; c0 < nm; c0 += blockDim.x) {
    int t = c0 + threadIdx.x;
    int d = (t < nm) ? dir[V[t]] : 0;
    // per-warp, per-direction counts and ranks
    int myrank = 0;
    for (int dd = 1; dd <= 8; ++dd) {
      unsigned b = __ballot_sync(0xffffffffu, d == dd);
      if (d == dd) myrank = __popc(b & ((1u << lane) - 1));
      if (lane == 0) wcnt[w][dd] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int dd = 1; dd <= 8; ++dd) {
        int s = base[dd];
        for (int q = 0; q < nw; ++q) {
          int v = wcnt[q][dd];
          wcnt[q][dd] = s;
          s += v;
        }
        base[dd] = s;
      }
    }
    __syncthreads();
    if (t < nm && d > 0) M[wcnt[w][d] + myrank] = V[t];
    __syncthreads();
  }
}

// The 29 properties carried by the haloswap buffers (haloswap.F90:35-52, :585-600).
__constant__ int c_swap_props[29] = {PMPIC_PROP_X,    PMPIC_PROP_Y,    PMPIC_PROP_Z,    PMPIC_PROP_P,
                                     PMPIC_PROP_Q,    PMPIC_PROP_R,    PMPIC_PROP_DXDT, PMPIC_PROP_DYDT,
                                     PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT, PMPIC_PROP_DRDT,
                                     PMPIC_PROP_H,    PMPIC_PROP_B,    PMPIC_PROP_VOL,  PMPIC_PROP_STRETCH,
                                     PMPIC_PROP_TAG,  PMPIC_PROP_XO,   PMPIC_PROP_YO,   PMPIC_PROP_ZO,
                                     PMPIC_PROP_XF,   PMPIC_PROP_YF,   PMPIC_PROP_ZF,   PMPIC_PROP_PO,
                                     PMPIC_PROP_QO,   PMPIC_PROP_RO,   PMPIC_PROP_PF,   PMPIC_PROP_QF,
                                     PMPIC_PROP_RF};

// gather moved parcels (with the periodic shift of their direction,
// haloswap.F90:531-559, :587-591) into the staging buffer
__global__ void k_swap_gather(Geom g, const int32_t* __restrict__ nmov, const int32_t* __restrict__ M,
                              const int8_t* __restrict__ dir, const double* __restrict__ parcels, int64_t cap,
                              double* __restrict__ buf) {
  const int nm = *nmov;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nm * 29;
       e += (int64_t)gridDim.x * blockDim.x) {
    int t = (int)(e / 29), q = (int)(e - (int64_t)t * 29);
    int src = M[t];
    int pid = c_swap_props[q];
    double v = parcels[(size_t)pid * cap + src];
    int d = dir[src];
    double xs = 0.0, ys = 0.0;
    if (d == 3 || d == 2 || d == 4) xs = g.xshift_e;
    else if (d == 7 || d == 8 || d == 6) xs = g.xshift_w;
    if (d == 1 || d == 2 || d == 8) ys = g.yshift_n;
    else if (d == 5 || d == 6 || d == 4) ys = g.yshift_s;
    if (pid == PMPIC_PROP_X || pid == PMPIC_PROP_XO || pid == PMPIC_PROP_XF) v = v + xs;
    if (pid == PMPIC_PROP_Y || pid == PMPIC_PROP_YO || pid == PMPIC_PROP_YF) v = v + ys;
    buf[e] = v;
  }
}
// unpack into the vacated slots in ascending order (haloswap.F90:695-716)
__global__ void k_swap_scatter(const int32_t* __restrict__ nmov, const int32_t* __restrict__ V,
                               const double* __restrict__ buf, double* __restrict__ parcels, int64_t cap) {
  const int nm = *nmov;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nm * 29;
       e += (int64_t)gridDim.x * blockDim.x) {
    int t = (int)(e / 29), q = (int)(e - (int64_t)t * 29);
    parcels[(size_t)c_swap_props[q] * cap + V[t]] = buf[e];
  }
}
__global__ void k_check_swapcap(const int32_t* nmov, int32_t* nclamped, int64_t swapcap, DevInfo* info) {
  int nm = *nmov;
  if (nm > swapcap) {
    atomicCAS(&info->error, 0, PMPIC_ERR_CAPACITY);
    nm = 0;  // nothing is moved; the call reports the capacity error
  }
  *nclamped = nm;
  info->n_migrated = *nmov;
}

// ---- parcel splitting (parcel_splitting.F90:64-133) -----------------------------------
__global__ void k_split_flag(int64_t n, double* __restrict__ parcels, int64_t cap, const double* __restrict__ dtp,
                             int32_t* __restrict__ flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dt = *dtp;
  const double* P = parcels + (size_t)PMPIC_PROP_P * cap;
  const double* Q = parcels + (size_t)PMPIC_PROP_Q * cap;
  const double* R = parcels + (size_t)PMPIC_PROP_R * cap;
  const double* DP = parcels + (size_t)PMPIC_PROP_DPDT * cap;
  const double* DQ = parcels + (size_t)PMPIC_PROP_DQDT * cap;
  const double* DR = parcels + (size_t)PMPIC_PROP_DRDT * cap;
  double* S = parcels + (size_t)PMPIC_PROP_STRETCH * cap;
  double ds = P[i] * DP[i] + Q[i] * DQ[i] + R[i] * DR[i];  // :68-70
  ds = pow(fabs(ds), f4div(1.f, 3.f));                      // :71
  double s = S[i] + ds * dt;                                // :73
  S[i] = s;
  flag[i] = s > 4. ? 1 : 0;                                  // :76 (stretchmax = 4)
}
// With dir given (every other parcel is inside the domain, its dir zero), the
// parent and the child are reflected at the walls and classified here, as the
// parcel haloswap that follows (:134) would do for them.
__global__ void k_split_apply(Geom g, int64_t n, const int32_t* __restrict__ list, const int32_t* __restrict__ nsplit,
                              double* __restrict__ parcels, int64_t cap, DevInfo* info, int8_t* __restrict__ dir,
                              int32_t* __restrict__ dircnt) {
  const int ns = *nsplit;
  const double pi = 4. * atan(1.0);
  const double third = f4div(1.f, 3.f);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ns; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = list[t];
    int64_t c = n + t;  // child slot: appended in index order (:94)
    if (c >= cap) {
      atomicCAS(&info->error, 0, PMPIC_ERR_CAPACITY);
      continue;
    }
    double* p = parcels;
    auto A = [&](int pid) -> double* { return p + (size_t)pid * cap; };
    double r = A(PMPIC_PROP_VOL)[i] / 4. / pi;  // :78-79
    r = pow(r, third);
    double pp = A(PMPIC_PROP_P)[i], qq = A(PMPIC_PROP_Q)[i], rr = A(PMPIC_PROP_R)[i];
    double absw = pp * pp + qq * qq + rr * rr;  // :83-84
    absw = sqrt(absw);
    double x = A(PMPIC_PROP_X)[i], y = A(PMPIC_PROP_Y)[i], z = A(PMPIC_PROP_Z)[i];
    A(PMPIC_PROP_X)[c] = x + r * pp / absw;  // :95-118
    A(PMPIC_PROP_Y)[c] = y + r * qq / absw;
    A(PMPIC_PROP_Z)[c] = z + r * rr / absw;
    A(PMPIC_PROP_P)[c] = pp;
    A(PMPIC_PROP_Q)[c] = qq;
    A(PMPIC_PROP_R)[c] = rr;
    A(PMPIC_PROP_DXDT)[c] = A(PMPIC_PROP_DXDT)[i];
    A(PMPIC_PROP_DYDT)[c] = A(PMPIC_PROP_DYDT)[i];
    A(PMPIC_PROP_DZDT)[c] = A(PMPIC_PROP_DZDT)[i];
    A(PMPIC_PROP_DPDT)[c] = A(PMPIC_PROP_DPDT)[i];
    A(PMPIC_PROP_DQDT)[c] = A(PMPIC_PROP_DQDT)[i];
    A(PMPIC_PROP_DRDT)[c] = A(PMPIC_PROP_DRDT)[i];
    A(PMPIC_PROP_H)[c] = A(PMPIC_PROP_H)[i];
    A(PMPIC_PROP_B)[c] = A(PMPIC_PROP_B)[i];
    double vol = A(PMPIC_PROP_VOL)[i];
    A(PMPIC_PROP_VOL)[c] = vol / 2;
    A(PMPIC_PROP_STRETCH)[c] = 0.;
    A(PMPIC_PROP_TAG)[c] = A(PMPIC_PROP_TAG)[i];
    A(PMPIC_PROP_X)[i] = x - r * pp / absw;  // :121-127
    A(PMPIC_PROP_Y)[i] = y - r * qq / absw;
    A(PMPIC_PROP_Z)[i] = z - r * rr / absw;
    A(PMPIC_PROP_VOL)[i] = vol / 2;
    A(PMPIC_PROP_STRETCH)[i] = 0.;
    if (dir) {
      const int64_t s2[2] = {c, i};
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int64_t m = s2[u];
        const double zz = A(PMPIC_PROP_Z)[m];
        if (zz < g.pzmin) A(PMPIC_PROP_Z)[m] = g.pzmin + (g.pzmin - zz);
        else if (zz > g.pzmax) A(PMPIC_PROP_Z)[m] = g.pzmax - (zz - g.pzmax);
        const int dr = classify_dir(g, A(PMPIC_PROP_X)[m], A(PMPIC_PROP_Y)[m]);
        dir[m] = (int8_t)dr;
        if (dr) atomicAdd(&dircnt[m / CITEMS], 1);
      }
    }
  }
}

// ---- btot (vorticity_tendency.F90:121-126) ------------------------------------------------
__global__ void k_btot(int64_t n, const double* __restrict__ B, const double* __restrict__ H,
                       const double* __restrict__ Z, double* __restrict__ BT) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BT[i] = B[i] + 12.5 * fmax(0.0, H[i] - exp(-Z[i]));
}

// ---- mixing (parcel_mixing.F90:68-431) --------------------------------------------------
// Residual grids are non-zero only at the corners of cells holding a removed
// parcel or a new one.  The cells whose corners such a residual can reach: id
// and its neighbours (periodic in x and y), marked in near (both forms).
__device__ __forceinline__ void mark_near(const Geom& g, int32_t id, uint8_t* __restrict__ near) {
  int i, j, k;
  cell_decode(g, id, i, j, k);
  for (int dk = -1; dk <= 1; ++dk) {
    const int kk = k + dk;
    if (kk < 0 || kk >= g.Nz) continue;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) near[cell_encode(g, wrap_index(i + di, g.Nx), wrap_index(j + dj, g.Ny), kk)] = 1;
  }
}
// the removed parcels' cells (FP64 path; the mixed form marks them as it uncounts them)
__global__ void k_mark_removed(Geom g, const int32_t* __restrict__ zlist, const int32_t* __restrict__ nz,
                               const int32_t* __restrict__ cell, uint8_t* __restrict__ near) {
  const int n = *nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int32_t c = cell[zlist[t]];
    if (c >= 0 && c < g.ncell) mark_near(g, c, near);
  }
}
__global__ void k_keep(int64_t n, const double* __restrict__ VOL, double vmin, int32_t* __restrict__ keep) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keep[i] = VOL[i] < vmin ? 0 : 1;  // :488, :555
}

// New parcels (:160-212): the a-th under-populated cell in loop order takes the
// a-th removed slot, or is appended after norig; keep = 2 only for slots below
// the last one (:191-193, strict <).
__global__ void k_new_parcels(Geom g, const int32_t* __restrict__ olist, const int32_t* __restrict__ nnew,
                              const int32_t* __restrict__ zlist, const int32_t* __restrict__ nzero, int64_t norig,
                              int64_t cap, int32_t* __restrict__ keep, double* __restrict__ parcels,
                              const double* __restrict__ KV, const double* __restrict__ KB,
                              const double* __restrict__ KH, const double* __restrict__ KP,
                              const double* __restrict__ KQ, const double* __restrict__ KR,
                              int32_t* __restrict__ newslot, double* __restrict__ portion,
                              uint8_t* __restrict__ near, DevInfo* info) {
  const int na = *nnew, nz0 = *nzero;
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < na; a += (int64_t)gridDim.x * blockDim.x) {
    int64_t o = olist[a];
    int k = (int)(o % g.Nz);
    int j = (int)((o / g.Nz) % g.Ny);
    int i = (int)(o / ((int64_t)g.Nz * g.Ny));
    int64_t slot = a < nz0 ? (int64_t)zlist[a] : norig + (a - nz0);
    if (slot + 2 > cap) {  // :194-199: n+1 > maxparcels after placing at n
      atomicCAS(&info->error, 0, PMPIC_ERR_CAPACITY);
      continue;
    }
    int i1 = i + 1 == g.Nx ? 0 : i + 1, j1 = j + 1 == g.Ny ? 0 : j + 1;
    // Fortran sum over the (2,2,2) section: k fastest, then j, then i
    size_t q[8] = {((size_t)k * g.Ny + j) * g.Nx + i,        ((size_t)(k + 1) * g.Ny + j) * g.Nx + i,
                   ((size_t)k * g.Ny + j1) * g.Nx + i,       ((size_t)(k + 1) * g.Ny + j1) * g.Nx + i,
                   ((size_t)k * g.Ny + j) * g.Nx + i1,       ((size_t)(k + 1) * g.Ny + j) * g.Nx + i1,
                   ((size_t)k * g.Ny + j1) * g.Nx + i1,      ((size_t)(k + 1) * g.Ny + j1) * g.Nx + i1};
    auto box = [&](const double* G) {
      double s = 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u) s = s + G[q[u]];
      return s;
    };
    double v = box(KV);
    double por = 2 * g.vmin / v;
    auto A = [&](int pid) -> double* { return parcels + (size_t)pid * cap; };
    // x_coords(I) with I = i+3 (halo-inclusive, parcel_interpolation.F90:126-136)
    double xc = g.pxmin + (double)(i + 2) * g.dx, xc1 = g.pxmin + (double)(i + 3) * g.dx;
    double yc = g.pymin + (double)(j + 2) * g.dy, yc1 = g.pymin + (double)(j + 3) * g.dy;
    double zc = g.pzmin + (double)k * g.dz, zc1 = g.pzmin + (double)(k + 1) * g.dz;
    A(PMPIC_PROP_X)[slot] = 0.5 * (xc + xc1);
    A(PMPIC_PROP_Y)[slot] = 0.5 * (yc + yc1);
    A(PMPIC_PROP_Z)[slot] = 0.5 * (zc + zc1);
    A(PMPIC_PROP_VOL)[slot] = 2 * g.vmin;
    A(PMPIC_PROP_STRETCH)[slot] = 0;
    A(PMPIC_PROP_B)[slot] = box(KB) / v;
    A(PMPIC_PROP_H)[slot] = box(KH) / v;
    A(PMPIC_PROP_P)[slot] = box(KP) / v;
    A(PMPIC_PROP_Q)[slot] = box(KQ) / v;
    A(PMPIC_PROP_R)[slot] = box(KR) / v;
    if (slot + 1 < norig) keep[slot] = 2;
    int64_t cell = ((int64_t)k * g.Ny + j) * g.Nx + i;
    newslot[cell] = (int32_t)slot;
    portion[cell] = por;
    mark_near(g, (int32_t)o, near);  // the new parcel's portion comes off its cell's corners
  }
}

// residual grids minus the new parcels' portions, then doubled at the walls
// (:202-207, :221-240)
struct ResPtrs {
  double* r[6];
  const double* k[6];
};
// A point outside the cells marked near an event keeps its residuals (+0.0,
// doubled or not), so it is left at once.
__global__ void k_residual_update(Geom g, ResPtrs RP, const int32_t* __restrict__ newslot,
                                  const double* __restrict__ portion, const uint8_t* __restrict__ near) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.nphys) return;
  int i = (int)(e % g.Nx);
  int j = (int)((e / g.Nx) % g.Ny);
  int k = (int)(e / ((int64_t)g.Nx * g.Ny));
  if (!near[cell_encode(g, i, j, k < g.Nz ? k : g.Nz - 1)]) return;
  int im = i == 0 ? g.Nx - 1 : i - 1, jm = j == 0 ? g.Ny - 1 : j - 1;
  double por[8];
  int np = 0;
  const int cis[2] = {im, i}, cjs[2] = {jm, j};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        int ck = k - 1 + c;
        if (ck < 0 || ck >= g.Nz) continue;
        int64_t cell = ((int64_t)ck * g.Ny + cjs[b]) * g.Nx + cis[a];
        if (newslot[cell] >= 0) por[np++] = portion[cell];
      }
  const bool wall = (k == 0 || k == g.Nz);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double r = RP.r[q][e];
    double kv = RP.k[q][e];
    for (int u = 0; u < np; ++u) r = r - por[u] * kv;
    if (wall) r = r * 2;
    RP.r[q][e] = r;
  }
}

// residuals onto the kept original parcels (:245-342), with the binning
// cached at the start of mixing (:80; kept parcels have not moved), the
// corners visited in the reference's order u = 0..7 (x fastest, then y, then
// z) and read from the kept volume grid and the six residual grids.
// A parcel whose cell is not marked near an event sees +0.0 residuals at all
// eight corners; when its eight corner weights are positive (so the kept
// volume there is too) every term the reference adds is +0.0: nv stays v and
// each field becomes (f v + 0) / v.  That is computed without the corners,
// with the same IEEE operations, so the bits are the reference's.  (A corner
// weight of exactly zero could meet a zero kept volume, 0/0 in the reference:
// such a parcel takes the full path.)
struct RedistGridsD {
  const double* kv;    // kept volume
  const double* r[6];  // vres, bres, hres, pres, qres, rres
};
__global__ void __launch_bounds__(256, 3) k_redistribute(Geom g, int64_t norig, const int32_t* __restrict__ keep,
                                                         double* __restrict__ parcels, int64_t cap,
                                                         const int32_t* __restrict__ cell,
                                                         const double* __restrict__ del,
                                                         const uint8_t* __restrict__ near, RedistGridsD RD) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= norig) return;
  auto A = [&](int pid) -> double* { return parcels + (size_t)pid * cap; };
  const int pids[5] = {PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
  // the state is read before the keep flag is known: one memory round trip
  // less per parcel (removed parcels are few)
  const int kp = keep ? keep[m] : 1;  // (no keep flags: no parcel was removed)
  const int32_t id = cell[m];
  const double delx = del[m], dely = del[cap + m], delz = del[2 * cap + m];
  const double v = A(PMPIC_PROP_VOL)[m];
  double s[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) s[q] = A(pids[q])[m];
  if (kp != 1 || id < 0 || id >= g.ncell) return;
#pragma unroll
  for (int q = 0; q < 5; ++q) s[q] = s[q] * v;
  // weight of corner u (:258-265, evaluated left to right as there)
  auto weight = [&](int u) {
    return ((u & 4) ? delz : 1 - delz) * ((u & 2) ? dely : 1 - dely) * ((u & 1) ? delx : 1 - delx) * v;
  };
  bool far = !near[id];
#pragma unroll
  for (int u = 0; u < 8; ++u) far = far && weight(u) > 0.0;
  if (far) {
#pragma unroll
    for (int q = 0; q < 5; ++q) A(pids[q])[m] = __dadd_rn(s[q], 0.0) / v;
    return;  // vol: v + 0 = v
  }
  const int ck = id % g.Nz, cj = (id / g.Nz) % g.Ny, ci = id / (g.Nz * g.Ny);
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  double nv = v;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int x = (u & 1) ? ci1 : ci, y = (u & 2) ? cj1 : cj, z = ck + (u >> 2);
    const size_t gi = ((size_t)z * g.Ny + y) * g.Nx + x;
    const double kv = RD.kv[gi];
    const double w = weight(u);
    const double wv = w / kv;         // the w/vol_g factor shared by b, h, p, q, r (:280-335)
    nv = nv + w * RD.r[0][gi] / kv;   // :268-276
#pragma unroll
    for (int q = 0; q < 5; ++q) s[q] = s[q] + wv * RD.r[q + 1][gi];  // :279-336
  }
  A(PMPIC_PROP_VOL)[m] = nv;
#pragma unroll
  for (int q = 0; q < 5; ++q) A(pids[q])[m] = s[q] / nv;
}

// backfill (:347-389): the t-th removed slot (ascending) receives the t-th kept
// parcel counted from the top; 11 properties are copied.
__global__ void k_backfill(const int32_t* __restrict__ zlist, const int32_t* __restrict__ nz,
                           const int32_t* __restrict__ olist, const int32_t* __restrict__ no,
                           double* __restrict__ parcels, int64_t cap, DevInfo* info) {
  const int nzero = *nz, nones = *no;
  if (blockIdx.x == 0 && threadIdx.x == 0 && nzero > nones) atomicCAS(&info->error, 0, PMPIC_ERR_BACKFILL);
  const int pids[11] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P,   PMPIC_PROP_Q,      PMPIC_PROP_R,
                        PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_VOL, PMPIC_PROP_TAG, PMPIC_PROP_STRETCH};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nzero * 11;
       e += (int64_t)gridDim.x * blockDim.x) {
    int t = (int)(e / 11), q = (int)(e - (int64_t)t * 11);
    if (t >= nones) continue;
    int dst = zlist[t], src = olist[nones - 1 - t];
    parcels[(size_t)pids[q] * cap + dst] = parcels[(size_t)pids[q] * cap + src];
  }
}

// ==== mixed-precision form ===========================================================
// The same components with FP32 fields and {cell, FP32 offset} positions
// (common.cuh): the current position as the cell id and three offsets, xo as
// a CellOff per axis, xf as the displacement from xo.  The integer bookkeeping
// (directions, lists, slots) is shared with the plain path.  Float property p
// of parcel n is ((float*)array_p)[n].
struct MPtrs {
  const float* g6;  // the six grids packed (k_pack), when both gathers are pending
  float inv[3];     // 1/dx, 1/dy, 1/dz
  int32_t* cell;    // current cell ids
  float* cur[3];    // current offsets
  CellOff* o[3];    // xo, yo, zo
  float* f[3];      // xf, yf, zf as displacements from xo (cell units)
  float* sv[3];     // p, q, r
  float* ov[3];
  float* fv[3];
  float* d[6];      // dxdt, dydt, dzdt, dpdt, dqdt, drdt
  const float* grid[6];
  int32_t* whint;   // per CTA: the cell its first parcel moved to at the last stage
};

// grid2par (parcel_interpolation.F90:299-321) of one FP32 grid at cell (i, j, k), offsets (dx, dy, dz)
__device__ __forceinline__ float g2p_f(const Geom& g, const float* __restrict__ G, int ci, int cj, int ck,
                                       float delx, float dely, float delz) {
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  const size_t r00 = ((size_t)ck * g.Ny + cj) * g.Nx, r01 = ((size_t)ck * g.Ny + cj1) * g.Nx;
  const size_t r10 = ((size_t)(ck + 1) * g.Ny + cj) * g.Nx, r11 = ((size_t)(ck + 1) * g.Ny + cj1) * g.Nx;
  const float c00 = G[r00 + ci] * (1.f - delz) + G[r10 + ci] * delz;
  const float c01 = G[r00 + ci1] * (1.f - delz) + G[r10 + ci1] * delz;
  const float c10 = G[r01 + ci] * (1.f - delz) + G[r11 + ci] * delz;
  const float c11 = G[r01 + ci1] * (1.f - delz) + G[r11 + ci1] * delz;
  const float c0 = c00 * (1.f - dely) + c10 * dely;
  const float c1 = c01 * (1.f - dely) + c11 * dely;
  return c0 * (1.f - delx) + c1 * delx;
}

__device__ __forceinline__ int classify_dir_m(const Geom& g, int i, int j) {
  const bool xl = i < 0, xh = i >= g.Nx, yl = j < 0, yh = j >= g.Ny;
  if (yh && !xl && !xh) return 1;
  if (yl && !xl && !xh) return 5;
  if (xh && !yl && !yh) return 3;
  if (xl && !yl && !yh) return 7;
  if (xh && yh) return 2;
  if (xl && yh) return 8;
  if (xh && yl) return 4;
  if (xl && yl) return 6;
  return 0;
}

// A moved position p (unwrapped x, y indices; z after the wall reflection)
// as the current position: the haloswap direction from the unwrapped indices
// (haloswap.F90:296-437), x and y wrapped by whole periods (the shift of
// :531-559; the haloswap then re-slots the parcel and shifts its xo), the
// cell id.  A z outside the grid after its reflection is reported out of box.
__device__ __forceinline__ int32_t place_m(const Geom& g, CellOff* p, int& d, DevInfo* info) {
  d = classify_dir_m(g, p[0].i, p[1].i);
  p[0].i = wrap_index(p[0].i, g.Nx);
  p[1].i = wrap_index(p[1].i, g.Ny);
  if (!(p[2].i >= 0 && p[2].i < g.Nz && p[0].f >= 0.f && p[0].f < 1.f && p[1].f >= 0.f && p[1].f < 1.f &&
        p[2].f >= 0.f && p[2].f <= 1.f)) {
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    p[0] = p[1] = p[2] = CellOff{0, 0.f};
  }
  return cell_encode(g, p[0].i, p[1].i, p[2].i);
}

// RK4 stage (rk4_integrator.F90:95-319) with the deferred gathers, the z
// reflection and the direction classification, as k_rk4; position updates in
// cell units (velocity * dt / cell size), renormalised into [0, 1).  The
// parcel is gathered at its current position; stage 1 takes that position as
// xo (:125-127); the new position is xo plus the stage's displacement, and xf
// the accumulated displacement (at stage 4 the new position is xo + xf, :303).
// The new cell id and offsets are the next binning: every parcel is counted
// in its new cell (movers too: they keep their cell as the haloswap re-slots
// them).
template <bool GU, bool GP>
__global__ void __launch_bounds__(256, 6) k_rk4_m(Geom g, int64_t n, MPtrs P, int stage, const double* __restrict__ dtp,
                        int8_t* __restrict__ dir, int32_t* __restrict__ count, DevInfo* info,
                        float* __restrict__ stretch, int store_d, int32_t* __restrict__ dircnt) {
  // the staged gather window, when both gathers are pending (the step's path)
  __shared__ __align__(16) float gws[(GU && GP) ? 4 * GW_KW * 6 : 4];
  __shared__ __align__(8) uint64_t gwbar;
  __shared__ GatherWindow gw;
  if constexpr (GU && GP) {
    if (threadIdx.x == 0) mbar_init(&gwbar, 1);
    __syncthreads();
    if (threadIdx.x == 0) window_issue(g, P.g6, P.whint[blockIdx.x], gw, gws, &gwbar);
  }
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;  // (thread 0 stays: the copies complete before the CTA ends)
  bool ready = false;
  const float dt = (float)*dtp;  // state%dtm (rk4_integrator.F90:102)
  const float dt6 = dt * (1.f / 6.f), dt2 = dt * 0.5f, dt3 = dt * (1.f / 3.f);
  const float* inv = P.inv;
  const bool need_cur = stage == 1 || GU || GP;
  int cx[3] = {0, 0, 0};
  float cf[3] = {0.f, 0.f, 0.f};
  if (need_cur) {
    cell_decode(g, P.cell[t], cx[0], cx[1], cx[2]);
#pragma unroll
    for (int v = 0; v < 3; ++v) cf[v] = P.cur[v][t];
  }
  CellOff op[3];
  float fd[3], sv[3], ov[3], fv[3], d[6];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    if (stage == 1) sv[v] = P.sv[v][t];
    if (stage >= 2) {
      op[v] = P.o[v][t];
      fd[v] = P.f[v][t];
      fv[v] = P.fv[v][t];
    }
    if (stage == 2 || stage == 3) ov[v] = P.ov[v][t];
  }
#pragma unroll
  for (int v = 0; v < 6; ++v)
    if ((v < 3 && !GU) || (v >= 3 && !GP)) d[v] = P.d[v][t];
  if constexpr (GU && GP) {
    ready = mbar_wait_bounded(&gwbar);
    if (!ready) atomicCAS(&info->error, 0, PMPIC_ERR_TIMEOUT);
    if (ready && cx[0] == gw.i0 && cx[1] == gw.j0 && cx[2] >= gw.k0 && cx[2] <= gw.k0 + GW_KW - 3)
      g2p_packed_f([&](int c, float* lo, float* hi) { corner6_staged(gws, c, cx[2] - gw.s[c], lo, hi); }, cf[0],
                   cf[1], cf[2], d);
    else
      g2p_packed<float>(g, P.g6, cx[0], cx[1], cx[2], cf[0], cf[1], cf[2], d);
  } else if (GU || GP) {
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      if ((v < 3 && !GU) || (v >= 3 && !GP)) continue;
      d[v] = g2p_f(g, P.grid[v], cx[0], cx[1], cx[2], cf[0], cf[1], cf[2]);
    }
  }
  CellOff sn[3];
  float svn[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const float dc = d[v] * inv[v];  // cell units per unit time
    const float dw = d[v + 3];
    // the FP32 form fuses each increment into its sum
    if (stage == 1) {
      op[v] = CellOff{cx[v], cf[v]};
      ov[v] = sv[v];
      fd[v] = dt6 * dc;
      fv[v] = __fmaf_rn(dt6, dw, sv[v]);
      sn[v] = co_add(op[v], dt2 * dc);
      svn[v] = __fmaf_rn(dt2, dw, sv[v]);
    } else if (stage == 2) {
      fd[v] = __fmaf_rn(dt3, dc, fd[v]);
      fv[v] = __fmaf_rn(dt3, dw, fv[v]);
      sn[v] = co_add(op[v], dt2 * dc);
      svn[v] = __fmaf_rn(dt2, dw, ov[v]);
    } else if (stage == 3) {
      fd[v] = __fmaf_rn(dt3, dc, fd[v]);
      fv[v] = __fmaf_rn(dt3, dw, fv[v]);
      sn[v] = co_add(op[v], dt * dc);
      svn[v] = __fmaf_rn(dt, dw, ov[v]);
    } else {
      fd[v] = __fmaf_rn(dt6, dc, fd[v]);
      fv[v] = __fmaf_rn(dt6, dw, fv[v]);
      sn[v] = co_add(op[v], fd[v]);
      svn[v] = fv[v];
    }
  }
  sn[2] = co_reflect(sn[2], g.Nz);
  if (stretch) {  // the split's stretch update (parcel_splitting.F90:64-73) on the final p, q, r
    float ds = svn[0] * d[3] + svn[1] * d[4] + svn[2] * d[5];
    ds = cbrtf(fabsf(ds));  // |ds|^(1/3) (parcel_splitting.F90:71); FP32 1/3 is 1/3 to 1e-8
    stretch[t] = stretch[t] + ds * dt;
  }
#pragma unroll
  for (int v = 0; v < 6; ++v)
    if (store_d && ((v < 3 && GU) || (v >= 3 && GP))) P.d[v][t] = d[v];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    if (stage == 1) {
      P.o[v][t] = op[v];
      P.ov[v][t] = ov[v];
    }
    P.f[v][t] = fd[v];
    P.fv[v][t] = fv[v];
    P.sv[v][t] = svn[v];
  }
  int dr;
  const int32_t nid = place_m(g, sn, dr, info);
  P.cell[t] = nid;
#pragma unroll
  for (int v = 0; v < 3; ++v) P.cur[v][t] = sn[v].f;
  dir[t] = (int8_t)dr;
  count_mover(t, dr != 0, dircnt);
  count_cell(nid, count);
  if constexpr (GU && GP) {
    if (threadIdx.x == 0) {
      P.whint[blockIdx.x] = nid;  // the next stage's window
      if (!ready) mbar_wait_bounded(&gwbar);  // no copy in flight when the CTA ends
    }
  }
}

// the haloswap staging of the mixed form: each property as its 8-byte slot or
// its 4-byte value, then the cell id; xo shifted by whole periods
// (haloswap.F90:531-559).  The current position was wrapped already by the
// kernel that moved it, and xf is relative to xo: neither changes.
constexpr int SWAP_M = 30;  // 29 properties + the cell id per staged parcel
__global__ void k_swap_gather_m(Geom g, const int32_t* __restrict__ nmov, const int32_t* __restrict__ M,
                                const int8_t* __restrict__ dir, const double* __restrict__ parcels, int64_t cap,
                                const int32_t* __restrict__ cell, double* __restrict__ buf) {
  const int nm = *nmov;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nm * SWAP_M;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / SWAP_M), q = (int)(e - (int64_t)t * SWAP_M);
    const int src = M[t];
    if (q == 29) {
      buf[e] = (double)cell[src];
      continue;
    }
    const int pid = c_swap_props[q];
    const double* A = parcels + (size_t)pid * cap;
    if (mixed_elem_bytes(pid) == 4) {
      buf[e] = (double)((const float*)A)[src];  // exact widening
      continue;
    }
    double v = A[src];
    if (pid == PMPIC_PROP_XO || pid == PMPIC_PROP_YO) {
      const int d = dir[src];
      int sh = 0;
      if (pid == PMPIC_PROP_XO) {
        if (d == 3 || d == 2 || d == 4) sh = -g.Nx;
        else if (d == 7 || d == 8 || d == 6) sh = g.Nx;
      } else {
        if (d == 1 || d == 2 || d == 8) sh = -g.Ny;
        else if (d == 5 || d == 6 || d == 4) sh = g.Ny;
      }
      CellOff c = *(const CellOff*)&v;
      c.i += sh;
      v = *(const double*)&c;
    }
    buf[e] = v;
  }
}
__global__ void k_swap_scatter_m(const int32_t* __restrict__ nmov, const int32_t* __restrict__ V,
                                 const double* __restrict__ buf, double* __restrict__ parcels, int64_t cap,
                                 int32_t* __restrict__ cell) {
  const int nm = *nmov;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nm * SWAP_M;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / SWAP_M), q = (int)(e - (int64_t)t * SWAP_M);
    if (q == 29) {
      cell[V[t]] = (int32_t)buf[e];
      continue;
    }
    const int pid = c_swap_props[q];
    double* A = parcels + (size_t)pid * cap;
    if (mixed_elem_bytes(pid) == 4) ((float*)A)[V[t]] = (float)buf[e];
    else A[V[t]] = buf[e];
  }
}

// splitting (parcel_splitting.F90:64-133) in FP32
__global__ void k_split_flag_m(int64_t n, double* __restrict__ parcels, int64_t cap, const double* __restrict__ dtp,
                               int32_t* __restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float dt = (float)*dtp;
  auto F = [&](int pid) { return (float*)(parcels + (size_t)pid * cap); };
  float ds = F(PMPIC_PROP_P)[i] * F(PMPIC_PROP_DPDT)[i] + F(PMPIC_PROP_Q)[i] * F(PMPIC_PROP_DQDT)[i] +
             F(PMPIC_PROP_R)[i] * F(PMPIC_PROP_DRDT)[i];
  ds = cbrtf(fabsf(ds));  // |ds|^(1/3) (parcel_splitting.F90:71); FP32 1/3 is 1/3 to 1e-8
  const float s = F(PMPIC_PROP_STRETCH)[i] + ds * dt;
  F(PMPIC_PROP_STRETCH)[i] = s;
  flag[i] = s > 4.f ? 1 : 0;
}
// The parent shifted by -r w / |w| and the child at +r w / |w| (:95-127) from
// the parent's current position, reflected, classified and wrapped as an
// RK4 stage places a parcel (place_m); their cell ids written, and with count
// given (the cell counts are current) the parent's count moved to its new
// cell and the child counted in its own.  dir and the per-block mover counts
// are for the haloswap that follows (:134).
__global__ void k_split_apply_m(Geom g, int64_t n, const int32_t* __restrict__ list, const int32_t* __restrict__ nsplit,
                                double* __restrict__ parcels, int64_t cap, DevInfo* info, int8_t* __restrict__ dir,
                                int32_t* __restrict__ dircnt, int32_t* __restrict__ cell, int32_t* __restrict__ count) {
  const int ns = *nsplit;
  const float pi = 3.14159265358979f;
  const float inv[3] = {(float)(1.0 / g.dx), (float)(1.0 / g.dy), (float)(1.0 / g.dz)};
  const int fprops[11] = {PMPIC_PROP_P,    PMPIC_PROP_Q,    PMPIC_PROP_R,    PMPIC_PROP_DXDT,
                          PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT,
                          PMPIC_PROP_DRDT, PMPIC_PROP_H,    PMPIC_PROP_B};
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ns; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = list[t];
    const int64_t c = n + t;  // child slot: appended in index order (:94)
    if (c >= cap) {
      atomicCAS(&info->error, 0, PMPIC_ERR_CAPACITY);
      continue;
    }
    auto F = [&](int pid) { return (float*)(parcels + (size_t)pid * cap); };
    const float vol = F(PMPIC_PROP_VOL)[i];
    const float r = powf(vol / 4.f / pi, 1.f / 3.f);  // :78-79
    const float pp = F(PMPIC_PROP_P)[i], qq = F(PMPIC_PROP_Q)[i], rr = F(PMPIC_PROP_R)[i];
    const float absw = sqrtf(pp * pp + qq * qq + rr * rr);
    const float w[3] = {pp / absw, qq / absw, rr / absw};
    const int32_t old = cell[i];
    int ix[3];
    cell_decode(g, old, ix[0], ix[1], ix[2]);
    CellOff pc[3], pi_[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const CellOff x = CellOff{ix[v], F(PMPIC_PROP_X + v)[i]};
      const float sh = r * w[v] * inv[v];
      pc[v] = co_add(x, sh);    // :95-118
      pi_[v] = co_add(x, -sh);  // :121-127
    }
    pc[2] = co_reflect(pc[2], g.Nz);
    pi_[2] = co_reflect(pi_[2], g.Nz);
    int dc, di;
    const int32_t nc = place_m(g, pc, dc, info), ni = place_m(g, pi_, di, info);
    dir[c] = (int8_t)dc;
    dir[i] = (int8_t)di;
    if (dc) atomicAdd(&dircnt[c / CITEMS], 1);
    if (di) atomicAdd(&dircnt[i / CITEMS], 1);
    if (count) {
      atomicSub(&count[old], 1);
      atomicAdd(&count[ni], 1);
      atomicAdd(&count[nc], 1);
    }
    cell[i] = ni;
    cell[c] = nc;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      F(PMPIC_PROP_X + v)[c] = pc[v].f;
      F(PMPIC_PROP_X + v)[i] = pi_[v].f;
    }
#pragma unroll
    for (int q = 0; q < 11; ++q) F(fprops[q])[c] = F(fprops[q])[i];
    F(PMPIC_PROP_VOL)[c] = vol / 2;
    F(PMPIC_PROP_STRETCH)[c] = 0.f;
    parcels[(size_t)PMPIC_PROP_TAG * cap + c] = parcels[(size_t)PMPIC_PROP_TAG * cap + i];
    F(PMPIC_PROP_VOL)[i] = vol / 2;
    F(PMPIC_PROP_STRETCH)[i] = 0.f;
  }
}

// btot (vorticity_tendency.F90:121-126) in FP32, z from the current cell layer and offset
__global__ void k_btot_m(Geom g, int64_t n, const float* __restrict__ B, const float* __restrict__ H,
                         const int32_t* __restrict__ cell, const float* __restrict__ FZ, float* __restrict__ BT) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int ci, cj, ck;
  cell_decode(g, cell[i], ci, cj, ck);
  const float zz = ((float)ck + FZ[i]) * (float)g.dz;
  BT[i] = B[i] + 12.5f * fmaxf(0.f, H[i] - expf(-zz));
}

// mixing (parcel_mixing.F90:68-431) in FP32
__global__ void k_keep_m(int64_t n, const float* __restrict__ VOL, float vmin, int32_t* __restrict__ keep) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keep[i] = VOL[i] < vmin ? 0 : 1;
}
__global__ void k_new_parcels_m(Geom g, const int32_t* __restrict__ olist, const int32_t* __restrict__ nnew,
                                const int32_t* __restrict__ zlist, const int32_t* __restrict__ nzero, int64_t norig,
                                int64_t cap, int32_t* __restrict__ keep, double* __restrict__ parcels,
                                const float* __restrict__ KV, const float* __restrict__ KB,
                                const float* __restrict__ KH, const float* __restrict__ KP,
                                const float* __restrict__ KQ, const float* __restrict__ KR,
                                int32_t* __restrict__ newslot, float* __restrict__ portion, float vmin,
                                int32_t* __restrict__ cell, uint8_t* __restrict__ near, DevInfo* info) {
  const int na = *nnew, nz0 = *nzero;
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < na; a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = olist[a];
    const int k = (int)(o % g.Nz);
    const int j = (int)((o / g.Nz) % g.Ny);
    const int i = (int)(o / ((int64_t)g.Nz * g.Ny));
    const int64_t slot = a < nz0 ? (int64_t)zlist[a] : norig + (a - nz0);
    if (slot + 2 > cap) {
      atomicCAS(&info->error, 0, PMPIC_ERR_CAPACITY);
      continue;
    }
    const int i1 = i + 1 == g.Nx ? 0 : i + 1, j1 = j + 1 == g.Ny ? 0 : j + 1;
    const size_t q[8] = {((size_t)k * g.Ny + j) * g.Nx + i,   ((size_t)(k + 1) * g.Ny + j) * g.Nx + i,
                         ((size_t)k * g.Ny + j1) * g.Nx + i,  ((size_t)(k + 1) * g.Ny + j1) * g.Nx + i,
                         ((size_t)k * g.Ny + j) * g.Nx + i1,  ((size_t)(k + 1) * g.Ny + j) * g.Nx + i1,
                         ((size_t)k * g.Ny + j1) * g.Nx + i1, ((size_t)(k + 1) * g.Ny + j1) * g.Nx + i1};
    auto box = [&](const float* G) {
      float s = 0.f;
#pragma unroll
      for (int u = 0; u < 8; ++u) s = s + G[q[u]];
      return s;
    };
    const float v = box(KV);
    const float por = 2.f * vmin / v;
    auto F = [&](int pid) { return (float*)(parcels + (size_t)pid * cap); };
    cell[slot] = (int32_t)o;  // the cell centre (the loop order o is the cell id)
    F(PMPIC_PROP_X)[slot] = 0.5f;
    F(PMPIC_PROP_Y)[slot] = 0.5f;
    F(PMPIC_PROP_Z)[slot] = 0.5f;
    F(PMPIC_PROP_VOL)[slot] = 2.f * vmin;
    F(PMPIC_PROP_STRETCH)[slot] = 0.f;
    F(PMPIC_PROP_B)[slot] = box(KB) / v;
    F(PMPIC_PROP_H)[slot] = box(KH) / v;
    F(PMPIC_PROP_P)[slot] = box(KP) / v;
    F(PMPIC_PROP_Q)[slot] = box(KQ) / v;
    F(PMPIC_PROP_R)[slot] = box(KR) / v;
    if (slot + 1 < norig) keep[slot] = 2;
    const int64_t gcell = ((int64_t)k * g.Ny + j) * g.Nx + i;
    newslot[gcell] = (int32_t)slot;
    portion[gcell] = por;
    mark_near(g, (int32_t)o, near);  // the new parcel's portion comes off its cell's corners
  }
}
struct ResPtrsF {
  float* r[6];
  const float* k[6];
};
// A grid point is a corner of a removed or a new parcel's cell only if its
// cell (i, j, min(k, Nz - 1)) is marked near such a cell: every other point's
// residuals are zero and stay zero (doubled at a wall or not).
__global__ void k_residual_update_m(Geom g, ResPtrsF RP, const int32_t* __restrict__ newslot,
                                    const float* __restrict__ portion, const uint8_t* __restrict__ near) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.nphys) return;
  const int i = (int)(e % g.Nx);
  const int j = (int)((e / g.Nx) % g.Ny);
  const int k = (int)(e / ((int64_t)g.Nx * g.Ny));
  if (!near[cell_encode(g, i, j, k < g.Nz ? k : g.Nz - 1)]) return;
  const int im = i == 0 ? g.Nx - 1 : i - 1, jm = j == 0 ? g.Ny - 1 : j - 1;
  float por[8];
  int np = 0;
  const int cis[2] = {im, i}, cjs[2] = {jm, j};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        const int ck = k - 1 + c;
        if (ck < 0 || ck >= g.Nz) continue;
        const int64_t cell = ((int64_t)ck * g.Ny + cjs[b]) * g.Nx + cis[a];
        if (newslot[cell] >= 0) por[np++] = portion[cell];
      }
  const bool wall = (k == 0 || k == g.Nz);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    float r = RP.r[q][e];
    const float kv = RP.k[q][e];
    for (int u = 0; u < np; ++u) r = r - por[u] * kv;
    if (wall) r = r * 2.f;
    RP.r[q][e] = r;
  }
}
// Only a kept parcel whose cell is near a mixing event can see a non-zero
// residual at its corners; the others would only re-round their properties
// (f v / v) and are left as they are (near, built by k_mix_uncount and
// k_new_parcels_m).
// The corners are read from the kept volume grid and the six residual grids
// themselves (x fastest): few parcels are near an event, so no packed copy is
// made for them.
struct RedistGrids {
  const float* kv;    // kept volume
  const float* r[6];  // vres, bres, hres, pres, qres, rres
};
__global__ void __launch_bounds__(256, 6) k_redistribute_m(Geom g, int64_t norig, const int32_t* __restrict__ keep,
                                                          double* __restrict__ parcels, int64_t cap,
                                                          const int32_t* __restrict__ cell,
                                                          const uint8_t* __restrict__ near, RedistGrids RD) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= norig) return;
  auto F = [&](int pid) { return (float*)(parcels + (size_t)pid * cap); };
  const int pids[5] = {PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
  const int kp = keep ? keep[m] : 1;  // (no keep flags: no parcel was removed)
  const int32_t id = cell[m];
  if (kp != 1) return;
  if (id < 0 || id >= g.ncell) return;  // reported by the binning
  if (!near[id]) return;
  const float delx = F(PMPIC_PROP_X)[m], dely = F(PMPIC_PROP_Y)[m], delz = F(PMPIC_PROP_Z)[m];
  const float v = F(PMPIC_PROP_VOL)[m];
  float s[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) s[q] = F(pids[q])[m];
  int ci, cj, ck;
  cell_decode(g, id, ci, cj, ck);
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
#pragma unroll
  for (int q = 0; q < 5; ++q) s[q] = s[q] * v;
  float nv = v;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int x = (u & 1) ? ci1 : ci, y = (u & 2) ? cj1 : cj, z = ck + (u >> 2);
    const size_t gi = ((size_t)z * g.Ny + y) * g.Nx + x;
    const float4 a0 = make_float4(RD.kv[gi], RD.r[0][gi], RD.r[1][gi], RD.r[2][gi]);  // (vol, vres, bres, hres)
    const float4 a1 = make_float4(RD.r[3][gi], RD.r[4][gi], RD.r[5][gi], 0.f);        // (pres, qres, rres)
    const float w = ((u & 4) ? delz : 1.f - delz) * ((u & 2) ? dely : 1.f - dely) * ((u & 1) ? delx : 1.f - delx) * v;
    const float wv = __fdividef(w, a0.x);  // the fast quotient (within 2 ulp) of the FP32 form
    nv = nv + wv * a0.y;  // :268-276
    s[0] = s[0] + wv * a0.z;
    s[1] = s[1] + wv * a0.w;
    s[2] = s[2] + wv * a1.x;
    s[3] = s[3] + wv * a1.y;
    s[4] = s[4] + wv * a1.z;
  }
  const float rnv = __fdividef(1.f, nv);
#pragma unroll
  for (int q = 0; q < 5; ++q) F(pids[q])[m] = s[q] * rnv;
  F(PMPIC_PROP_VOL)[m] = nv;
}
// The binning's cell ids and counts kept current through mixing (mixed form):
// the removed parcels leave their cells' counts first; once the final count
// is known, every slot below it whose content changed (a new parcel, or one
// moved there by the backfill: keep != 1) is binned from its position, and
// every kept parcel beyond it (dropped by the backfill) leaves its count.
__global__ void k_mix_uncount(Geom g, const int32_t* __restrict__ zlist, const int32_t* __restrict__ nz,
                              const int32_t* __restrict__ cell, int32_t* __restrict__ count,
                              uint8_t* __restrict__ near) {
  const int n = *nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int32_t c = cell[zlist[t]];
    if (c >= 0) {
      atomicSub(&count[c], 1);
      mark_near(g, c, near);  // the removed parcel's residuals land on its cell's corners
    }
  }
}
// s0: the first slot that can have changed (norig when no parcel was removed:
// then only the appended slots did)
__global__ void k_mix_recount(Geom g, int64_t s0, int64_t norig, int64_t nfinal, const int32_t* __restrict__ keep,
                              const int32_t* __restrict__ cell, int32_t* __restrict__ count, DevInfo* info) {
  const int64_t hi = norig > nfinal ? norig : nfinal;
  for (int64_t s = s0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < hi; s += (int64_t)gridDim.x * blockDim.x) {
    if (s < nfinal) {
      if (s < norig && keep[s] == 1) continue;  // unchanged
      const int32_t id = cell[s];  // written with the slot's new position
      if (id >= 0 && id < g.ncell) atomicAdd(&count[id], 1);
      else atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    } else if (keep[s] == 1) {  // s < norig: a kept parcel dropped beyond the final count
      const int32_t c = cell[s];
      if (c >= 0) atomicSub(&count[c], 1);
    }
  }
}
// backfill (:347-389) of the mixed form: the 11 properties of k_backfill and
// the cell id, the rest of the slot's current position
__global__ void k_backfill_m(const int32_t* __restrict__ zlist, const int32_t* __restrict__ nz,
                             const int32_t* __restrict__ olist, const int32_t* __restrict__ no,
                             double* __restrict__ parcels, int64_t cap, int32_t* __restrict__ cell, DevInfo* info) {
  const int nzero = *nz, nones = *no;
  if (blockIdx.x == 0 && threadIdx.x == 0 && nzero > nones) atomicCAS(&info->error, 0, PMPIC_ERR_BACKFILL);
  const int pids[11] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P,   PMPIC_PROP_Q,      PMPIC_PROP_R,
                        PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_VOL, PMPIC_PROP_TAG, PMPIC_PROP_STRETCH};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)nzero * 12;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / 12), q = (int)(e - (int64_t)t * 12);
    if (t >= nones) continue;
    const int dst = zlist[t], src = olist[nones - 1 - t];
    if (q == 11) {
      cell[dst] = cell[src];
      continue;
    }
    double* A = parcels + (size_t)pids[q] * cap;
    if (mixed_elem_bytes(pids[q]) == 4) ((float*)A)[dst] = ((const float*)A)[src];
    else A[dst] = A[src];
  }
}
// grid2par of three FP32 grids into three float properties at the current positions
__global__ void k_grid2par_m(Geom g, int64_t n, const int32_t* __restrict__ cell, const float* __restrict__ FX,
                             const float* __restrict__ FY, const float* __restrict__ FZ, const float* __restrict__ G0,
                             const float* __restrict__ G1, const float* __restrict__ G2, float* __restrict__ O0,
                             float* __restrict__ O1, float* __restrict__ O2) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int32_t id = cell[t];
  if (id < 0 || id >= g.ncell) return;  // reported by the binning
  int ci, cj, ck;
  cell_decode(g, id, ci, cj, ck);
  const float fx = FX[t], fy = FY[t], fz = FZ[t];
  O0[t] = g2p_f(g, G0, ci, cj, ck, fx, fy, fz);
  O1[t] = g2p_f(g, G1, ci, cj, ck, fx, fy, fz);
  O2[t] = g2p_f(g, G2, ci, cj, ck, fx, fy, fz);
}

// ---- test components (FP64 path) ---------------------------------------------------
// euler_integrator.F90:68-76: one explicit step of x, y, z, p, q, r
__global__ void k_euler(int64_t n, double* __restrict__ parcels, int64_t cap, const double* __restrict__ dtp) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double dt = *dtp;
  const int S[6] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
  const int D[6] = {PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT,
                    PMPIC_PROP_DRDT};
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    double* x = parcels + (size_t)S[v] * cap;
    x[t] = x[t] + parcels[(size_t)D[v] * cap + t] * dt;
  }
}
// prescribed_parcel_velocity (velocity.F90): x0, y0, r0 (:66-69) and the
// centres of the evacuating profile (:233-237) from the global grid
struct VelGeom {
  double x0, y0, r0, xc1, yc1, xc2, yc2;
};
__global__ void k_prescribed_tag(int64_t n, double* __restrict__ parcels, int64_t cap, VelGeom vg) {  // :72-84
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double tag = 0;
  if (parcels[(size_t)PMPIC_PROP_Y * cap + t] > vg.y0) tag = tag + 2;
  if (parcels[(size_t)PMPIC_PROP_X * cap + t] > vg.x0) tag = tag + 1;
  parcels[(size_t)PMPIC_PROP_TAG * cap + t] = tag;
}
__global__ void k_prescribed_velocity(int64_t n, double* __restrict__ parcels, int64_t cap, int profile,
                                      VelGeom vg) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double x = parcels[(size_t)PMPIC_PROP_X * cap + t], y = parcels[(size_t)PMPIC_PROP_Y * cap + t];
  const double x0 = vg.x0, y0 = vg.y0, r0 = vg.r0;
  double u = 0., v = 0.;
  if (profile == PMPIC_VELOCITY_SHEAR) {  // :103-111
    v = tanh((x - x0) / r0);
  } else if (profile == PMPIC_VELOCITY_CYLINDRICAL) {  // :113-129
    const double theta = atan2(y - y0, x - x0);
    const double r2 = ((x - x0) * (x - x0) + (y - y0) * (y - y0));
    const double v0 = exp(-r2 / r0 / r0 / 2) / x0 * 10;
    u = v0 * sqrt(r2) * sin(theta);
    v = -v0 * sqrt(r2) * cos(theta);
  } else if (profile == PMPIC_VELOCITY_EVACUATE) {  // :229-250
    const double r1 = sqrt((x - vg.xc1) * (x - vg.xc1) + (y - vg.yc1) * (y - vg.yc1));
    const double r2 = sqrt((x - vg.xc2) * (x - vg.xc2) + (y - vg.yc2) * (y - vg.yc2));
    u = -(x - vg.xc1) / r1 * exp(-r1 * r1 / r0 / r0 / 4) + (x - vg.xc2) / r2 * exp(-r2 * r2 / r0 / r0 / 4);
    v = -(y - vg.yc1) / r1 * exp(-r1 * r1 / r0 / r0 / 4) + (y - vg.yc2) / r2 * exp(-r2 * r2 / r0 / r0 / 4);
  } else {  // the compass directions N .. NW (:131-226)
    const int p = profile;
    u = (p == 2 || p == 3 || p == 4) ? 1. : ((p == 6 || p == 7 || p == 8) ? -1. : 0.);
    v = (p == 8 || p == 1 || p == 2) ? 1. : ((p == 4 || p == 5 || p == 6) ? -1. : 0.);
  }
  parcels[(size_t)PMPIC_PROP_DXDT * cap + t] = u;
  parcels[(size_t)PMPIC_PROP_DYDT * cap + t] = v;
  parcels[(size_t)PMPIC_PROP_DZDT * cap + t] = 0.;
}

}  // namespace

// list of i in [0,n) with pred(i), ascending; count written to *dcount (device)
template <class Pred>
static int compact(pmpic_ctx* ctx, Pred pr, int64_t n, int32_t* list, int32_t* dcount) {
  int64_t nb = (n + CITEMS - 1) / CITEMS;
  if (nb == 0) {
    PMPIC_CUDA(cudaMemsetAsync(dcount, 0, sizeof(int32_t), ctx->stream));
    return 0;
  }
  int32_t* cnt = ctx->aux2;            // nb + 1 (nb + 1 <= nbmax)
  int32_t* off = ctx->aux2 + ctx->nbmax;
  k_count<<<(unsigned)nb, 256, 0, ctx->stream>>>(pr, n, cnt); ++ctx->nlaunch;
  int rc = scan_excl(ctx, cnt, nb, off);
  if (rc) return rc;
  k_write<<<(unsigned)nb, 256, 0, ctx->stream>>>(pr, n, off, list); ++ctx->nlaunch;
  PMPIC_CUDA(cudaMemcpyAsync(dcount, off + nb, sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// the same with the per-CTA counts already in ctx->aux2 (written by the
// kernel that computed the predicate's input)
template <class Pred>
static int compact_counted(pmpic_ctx* ctx, Pred pr, int64_t n, int32_t* list, int32_t* dcount) {
  int64_t nb = (n + CITEMS - 1) / CITEMS;
  if (nb == 0) {
    PMPIC_CUDA(cudaMemsetAsync(dcount, 0, sizeof(int32_t), ctx->stream));
    return 0;
  }
  int32_t* cnt = ctx->aux2;
  int32_t* off = ctx->aux2 + ctx->nbmax;
  int rc = scan_excl(ctx, cnt, nb, off);
  if (rc) return rc;
  k_write<<<(unsigned)nb, 256, 0, ctx->stream>>>(pr, n, off, list); ++ctx->nlaunch;
  PMPIC_CUDA(cudaMemcpyAsync(dcount, off + nb, sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// small device counters live after the DevInfo block
static int32_t* dcounter(pmpic_ctx* ctx, int i) { return (int32_t*)(ctx->dinfo + 1) + i; }

// Apply deferred grid2par gathers (vort2vel.F90:325-327,
// vorticity_tendency.F90:273-275) before anything observes or changes the
// tendencies; the cached binning is valid while they are pending.
int flush_gathers(pmpic_ctx* ctx) {
  int rc = 0;
  if (ctx->mixed) {  // gathers at the current {cell, offset} positions; no binning needed
    float* const* G = (float* const*)ctx->grid;
    const int64_t n = ctx->n;
    if (ctx->pending_uvw && n > 0) {
      k_grid2par_m<<<nblk(n, 256), 256, 0, ctx->stream>>>(
          ctx->g, n, ctx->cell, curoff(ctx, 0), curoff(ctx, 1), curoff(ctx, 2), G[PMPIC_GRID_U], G[PMPIC_GRID_V],
          G[PMPIC_GRID_W], propf(ctx, PMPIC_PROP_DXDT), propf(ctx, PMPIC_PROP_DYDT), propf(ctx, PMPIC_PROP_DZDT));
      ++ctx->nlaunch;
    }
    if (ctx->pending_pqr && n > 0) {
      k_grid2par_m<<<nblk(n, 256), 256, 0, ctx->stream>>>(
          ctx->g, n, ctx->cell, curoff(ctx, 0), curoff(ctx, 1), curoff(ctx, 2), G[PMPIC_GRID_DP], G[PMPIC_GRID_DQ],
          G[PMPIC_GRID_DR], propf(ctx, PMPIC_PROP_DPDT), propf(ctx, PMPIC_PROP_DQDT), propf(ctx, PMPIC_PROP_DRDT));
      ++ctx->nlaunch;
    }
    ctx->pending_uvw = ctx->pending_pqr = false;
    PMPIC_CUDA(cudaGetLastError());
    return 0;
  }
  if (ctx->pending_uvw) {
    ctx->pending_uvw = false;
    const double* gr[3] = {ctx->grid[PMPIC_GRID_U], ctx->grid[PMPIC_GRID_V], ctx->grid[PMPIC_GRID_W]};
    double* out[3] = {prop(ctx, PMPIC_PROP_DXDT), prop(ctx, PMPIC_PROP_DYDT), prop(ctx, PMPIC_PROP_DZDT)};
    if ((rc = grid2par_multi(ctx, gr, 3, out))) return rc;
  }
  if (ctx->pending_pqr) {
    ctx->pending_pqr = false;
    const double* gr[3] = {ctx->grid[PMPIC_GRID_DP], ctx->grid[PMPIC_GRID_DQ], ctx->grid[PMPIC_GRID_DR]};
    double* out[3] = {prop(ctx, PMPIC_PROP_DPDT), prop(ctx, PMPIC_PROP_DQDT), prop(ctx, PMPIC_PROP_DRDT)};
    if ((rc = grid2par_multi(ctx, gr, 3, out))) return rc;
  }
  return 0;
}

int compute_btot(pmpic_ctx* ctx) {
  if (ctx->n == 0) return 0;
  if (ctx->mixed) {
    k_btot_m<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, propf(ctx, PMPIC_PROP_B),
                                                         propf(ctx, PMPIC_PROP_H), ctx->cell, curoff(ctx, 2),
                                                         propf(ctx, PMPIC_PROP_BTOT)); ++ctx->nlaunch;
    PMPIC_CUDA(cudaGetLastError());
    return 0;
  }
  k_btot<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, prop(ctx, PMPIC_PROP_B), prop(ctx, PMPIC_PROP_H),
                                                     prop(ctx, PMPIC_PROP_Z), prop(ctx, PMPIC_PROP_BTOT)); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// Whether the stage kernel stores the gathered tendencies (dxdt .. drdt).
// Within pmpic_step, when another stage follows in the same call with no split
// in between, they are dead: the next stage gathers them afresh before
// anything reads them, and no caller code runs in between.  Otherwise (the
// last stage, a split following, components called one at a time) they are
// stored.
static int store_tendencies(const pmpic_ctx* ctx, int stage) { return ctx->in_step && stage < 4 ? 0 : 1; }

int rk4_stage(pmpic_ctx* ctx, int stage) {
  if (ctx->n == 0) {
    ctx->pending_uvw = ctx->pending_pqr = false;
    return 0;
  }
  TimerScope ts(ctx, T_RK4K);  // the stage kernel with its grid packing
  if (ctx->mixed) {
    MPtrs P;
    const int S[6] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
    const int O[6] = {PMPIC_PROP_XO, PMPIC_PROP_YO, PMPIC_PROP_ZO, PMPIC_PROP_PO, PMPIC_PROP_QO, PMPIC_PROP_RO};
    const int F[6] = {PMPIC_PROP_XF, PMPIC_PROP_YF, PMPIC_PROP_ZF, PMPIC_PROP_PF, PMPIC_PROP_QF, PMPIC_PROP_RF};
    const int D[6] = {PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT, PMPIC_PROP_DRDT};
    const int G[6] = {PMPIC_GRID_U, PMPIC_GRID_V, PMPIC_GRID_W, PMPIC_GRID_DP, PMPIC_GRID_DQ, PMPIC_GRID_DR};
    P.cell = ctx->cell;
    for (int v = 0; v < 3; ++v) {
      P.cur[v] = curoff(ctx, v);
      P.o[v] = propc(ctx, O[v]);
      P.f[v] = propf(ctx, F[v]);
      P.sv[v] = propf(ctx, S[v + 3]);
      P.ov[v] = propf(ctx, O[v + 3]);
      P.fv[v] = propf(ctx, F[v + 3]);
    }
    for (int v = 0; v < 6; ++v) {
      P.d[v] = propf(ctx, D[v]);
      P.grid[v] = (const float*)ctx->grid[G[v]];
    }
    const bool gu = ctx->pending_uvw, gp = ctx->pending_pqr;
    P.inv[0] = (float)(1.0 / ctx->g.dx);
    P.inv[1] = (float)(1.0 / ctx->g.dy);
    P.inv[2] = (float)(1.0 / ctx->g.dz);
    P.g6 = (const float*)ctx->gpack;
    P.whint = ctx->whint;
    if (gu && gp) pack6<float>(ctx, P.grid, (float*)ctx->gpack);
    auto kern = gu ? (gp ? k_rk4_m<true, true> : k_rk4_m<true, false>) : (gp ? k_rk4_m<false, true> : k_rk4_m<false, false>);
    PMPIC_CUDA(cudaMemsetAsync(ctx->cell_count, 0, sizeof(int32_t) * (ctx->g.ncell + 1), ctx->stream));
    PMPIC_CUDA(cudaMemsetAsync(ctx->aux2, 0, sizeof(int32_t) * ctx->nbmax, ctx->stream));  // mover counts
    // within pmpic_step the last stage also advances the stretch of the split
    // that follows (the haloswap in between moves it with its parcel)
    const bool adv = ctx->split_follows && stage == 4;
    kern<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, P, stage, &ctx->dinfo->dtm, ctx->dir,
                                                     ctx->cell_count, ctx->dinfo,
                                                     adv ? propf(ctx, PMPIC_PROP_STRETCH) : nullptr,
                                                     store_tendencies(ctx, stage), ctx->aux2); ++ctx->nlaunch;
    ctx->stretch_advanced = adv;
    ctx->pending_uvw = ctx->pending_pqr = false;
    ctx->dir_ready = true;
    ctx->sorted_valid = false;
    ctx->count_ready = true;
    ctx->in_domain = false;
    ctx->btot_grid_ready = false;
    PMPIC_CUDA(cudaGetLastError());
    return 0;
  }
  RkPtrs P;
  const int S[6] = {PMPIC_PROP_X, PMPIC_PROP_Y, PMPIC_PROP_Z, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
  const int O[6] = {PMPIC_PROP_XO, PMPIC_PROP_YO, PMPIC_PROP_ZO, PMPIC_PROP_PO, PMPIC_PROP_QO, PMPIC_PROP_RO};
  const int F[6] = {PMPIC_PROP_XF, PMPIC_PROP_YF, PMPIC_PROP_ZF, PMPIC_PROP_PF, PMPIC_PROP_QF, PMPIC_PROP_RF};
  const int D[6] = {PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT, PMPIC_PROP_DPDT, PMPIC_PROP_DQDT, PMPIC_PROP_DRDT};
  const int G[6] = {PMPIC_GRID_U, PMPIC_GRID_V, PMPIC_GRID_W, PMPIC_GRID_DP, PMPIC_GRID_DQ, PMPIC_GRID_DR};
  for (int v = 0; v < 6; ++v) {
    P.s[v] = prop(ctx, S[v]);
    P.o[v] = prop(ctx, O[v]);
    P.f[v] = prop(ctx, F[v]);
    P.d[v] = prop(ctx, D[v]);
    P.grid[v] = ctx->grid[G[v]];
  }
  const bool gu = ctx->pending_uvw, gp = ctx->pending_pqr;
  if ((gu || gp) && !ctx->sorted_valid) return set_error(ctx, PMPIC_ERR_STATE, "deferred gather without binning");
  P.g6 = ctx->gpack;
  P.whint = ctx->whint;
  if (gu && gp) pack6<double>(ctx, P.grid, ctx->gpack);
  auto kern = gu ? (gp ? k_rk4<true, true> : k_rk4<true, false>) : (gp ? k_rk4<false, true> : k_rk4<false, false>);
  // the next binning stays a separate pass on this path: its six IEEE
  // divisions per parcel cost the HBM-bound stage kernel more than the
  // position reads they would save
  PMPIC_CUDA(cudaMemsetAsync(ctx->aux2, 0, sizeof(int32_t) * ctx->nbmax, ctx->stream));  // mover counts
  kern<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, P, stage, &ctx->dinfo->dtm, ctx->cell, ctx->del,
                                                   ctx->cap, ctx->dir, store_tendencies(ctx, stage), ctx->aux2); ++ctx->nlaunch;
  ctx->pending_uvw = ctx->pending_pqr = false;
  ctx->dir_ready = true;  // z reflected and directions classified
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int parcel_haloswap(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_HSWP);
  if (!ctx->dir_ready) {
    int frc = flush_gathers(ctx);
    if (frc) return frc;
  }
  const int64_t n = ctx->n;
  ctx->sorted_valid = false;
  ctx->btot_grid_ready = false;
  const bool ready = ctx->dir_ready;
  ctx->dir_ready = false;
  // mixed form: every parcel keeps its cell id (part of its position) as it
  // is re-slotted, so the cell counts stay as the kernel that moved it left them
  if (!ctx->mixed) ctx->count_ready = false;
  if (n == 0) return 0;
  if (!ready && ctx->mixed) {
    // positions of the mixed form are kept wrapped and reflected by every
    // kernel that moves them: none is outside the domain
    PMPIC_CUDA(cudaMemsetAsync(ctx->dir, 0, (size_t)n, ctx->stream));
  } else if (!ready) {
    k_reflect_classify<<<nblk(n, 256), 256, 0, ctx->stream>>>(ctx->g, n, prop(ctx, PMPIC_PROP_X),
                                                              prop(ctx, PMPIC_PROP_Y), prop(ctx, PMPIC_PROP_Z),
                                                              ctx->dir); ++ctx->nlaunch;
  }
  int32_t* V = ctx->aux;                 // vacated slots, ascending
  int32_t* M = ctx->keep;                // moved parcels in send order (keep is free outside mixing)
  int32_t* nm = dcounter(ctx, 0);
  // after an RK4 stage or a split, the kernel that classified counted the movers
  int rc = ready ? compact_counted(ctx, PredDirNZ{ctx->dir}, n, V, nm) : compact(ctx, PredDirNZ{ctx->dir}, n, V, nm);
  if (rc) return rc;
  k_partition_dirs<<<1, 1024, 0, ctx->stream>>>(V, nm, ctx->dir, M); ++ctx->nlaunch;
  // the staging buffer is bounded: on overflow nothing moves and the call
  // reports PMPIC_ERR_CAPACITY
  int32_t* nmc = dcounter(ctx, 1);
  k_check_swapcap<<<1, 1, 0, ctx->stream>>>(nm, nmc, ctx->swapcap, ctx->dinfo); ++ctx->nlaunch;
  if (ctx->mixed) {
    k_swap_gather_m<<<592, 256, 0, ctx->stream>>>(ctx->g, nmc, M, ctx->dir, ctx->parcels, ctx->cap, ctx->cell,
                                                   ctx->swapbuf); ++ctx->nlaunch;
    k_swap_scatter_m<<<592, 256, 0, ctx->stream>>>(nmc, V, ctx->swapbuf, ctx->parcels, ctx->cap, ctx->cell);
    ++ctx->nlaunch;
  } else {
    k_swap_gather<<<592, 256, 0, ctx->stream>>>(ctx->g, nmc, M, ctx->dir, ctx->parcels, ctx->cap, ctx->swapbuf); ++ctx->nlaunch;
    k_swap_scatter<<<592, 256, 0, ctx->stream>>>(nmc, V, ctx->swapbuf, ctx->parcels, ctx->cap); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  ctx->in_domain = true;  // (a staging overflow is reported as an error and ends the run)
  return 0;
}

int splitting(pmpic_ctx* ctx) {
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  const int64_t n = ctx->n;
  int32_t* flag = ctx->aux;
  int32_t* list = ctx->keep;
  int32_t* ns = dcounter(ctx, 2);
  const bool advanced = ctx->stretch_advanced;
  ctx->stretch_advanced = false;
  bool split_counted = false;
  if (n > 0) {
    int rc;
    if (advanced) {  // the RK4 stage advanced the stretch: only the criterion is left
      rc = compact(ctx, PredStretchM{propf(ctx, PMPIC_PROP_STRETCH)}, n, list, ns);
    } else {
      if (ctx->mixed)
        k_split_flag_m<<<nblk(n, 256), 256, 0, ctx->stream>>>(n, ctx->parcels, ctx->cap, &ctx->dinfo->dtm, flag);
      else
        k_split_flag<<<nblk(n, 256), 256, 0, ctx->stream>>>(n, ctx->parcels, ctx->cap, &ctx->dinfo->dtm, flag);
      ++ctx->nlaunch;
      rc = compact(ctx, PredFlag{flag}, n, list, ns);
    }
    if (rc) return rc;
    // after a haloswap only the split parcels can be outside the domain: the
    // haloswap that follows needs no pass over all parcels to find them.  The
    // mixed form's positions are always inside (kept wrapped and reflected).
    int8_t* dsplit = nullptr;
    if (ctx->in_domain || ctx->mixed) {
      PMPIC_CUDA(cudaMemsetAsync(ctx->dir, 0, (size_t)n, ctx->stream));
      PMPIC_CUDA(cudaMemsetAsync(ctx->aux2, 0, sizeof(int32_t) * ctx->nbmax, ctx->stream));  // mover counts
      dsplit = ctx->dir;
    }
    // on the mixed form the binning counts stay current through the split
    const bool keep_counts = ctx->mixed && ctx->count_ready;
    if (ctx->mixed)
      k_split_apply_m<<<592, 256, 0, ctx->stream>>>(ctx->g, n, list, ns, ctx->parcels, ctx->cap, ctx->dinfo, dsplit,
                                                    ctx->aux2, ctx->cell, keep_counts ? ctx->cell_count : nullptr);
    else
      k_split_apply<<<592, 256, 0, ctx->stream>>>(ctx->g, n, list, ns, ctx->parcels, ctx->cap, ctx->dinfo, dsplit,
                                                  ctx->aux2);
    ++ctx->nlaunch;
    ctx->dir_ready = dsplit != nullptr;
    split_counted = keep_counts;
  } else {
    PMPIC_CUDA(cudaMemsetAsync(ns, 0, sizeof(int32_t), ctx->stream));
  }
  int32_t hns = 0;
  PMPIC_CUDA(cudaMemcpyAsync(&hns, ns, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  int64_t nn = n + hns;
  ctx->count_ready = split_counted;  // else split parents moved and children were added uncounted
  if (nn > ctx->cap) return set_error(ctx, PMPIC_ERR_CAPACITY, "maxparcels reached (parcel splitting)");
  ctx->n = nn;
  ctx->info.n_split = hns;
  return parcel_haloswap(ctx);
}

static VelGeom vel_geom(const pmpic_ctx* ctx) {
  // setup_grid.F90:87-93: bottom = the domain's lower bound, top = its last grid point
  const double bx = ctx->cfg.xmin, by = ctx->cfg.ymin;
  const double tx = ctx->cfg.xmax - ctx->g.dx, ty = ctx->cfg.ymax - ctx->g.dy;
  VelGeom vg;
  vg.x0 = (tx - bx) / 2. + bx;
  vg.y0 = (ty - by) / 2. + by;
  vg.r0 = (tx - bx) / 8.;
  vg.xc1 = 0.25 * (tx - bx) + bx;
  vg.yc1 = 0.25 * (ty - by) + by;
  vg.xc2 = 0.75 * (tx - bx) + bx;
  vg.yc2 = 0.75 * (ty - by) + by;
  return vg;
}

// euler_integrator.F90:53-86 (FP64 path)
int euler_step(pmpic_ctx* ctx) {
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "euler_integrator: FP64 contexts only");
  int rc = flush_gathers(ctx);
  if (rc) return rc;
  if (ctx->n > 0) {
    k_euler<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, ctx->parcels, ctx->cap, &ctx->dinfo->dtm); ++ctx->nlaunch;
  }
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->dir_ready = false;
  PMPIC_CUDA(cudaGetLastError());
  return parcel_haloswap(ctx);  // :82
}

// prescribed_parcel_velocity timestep (velocity.F90:96-255) and its
// initialisation's quadrant tags (:72-84, one process); FP64 path
int prescribed_velocity(pmpic_ctx* ctx, int profile, bool tags) {
  if (ctx->mixed) return set_error(ctx, PMPIC_ERR_STATE, "prescribed velocity: FP64 contexts only");
  if (!tags && (profile < 0 || profile > PMPIC_VELOCITY_EVACUATE))
    return set_error(ctx, PMPIC_ERR_ARG, "prescribed velocity: unknown profile");
  int rc = flush_gathers(ctx);  // the tendencies are overwritten
  if (rc) return rc;
  if (ctx->n > 0) {
    if (tags)
      k_prescribed_tag<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, ctx->parcels, ctx->cap, vel_geom(ctx));
    else
      k_prescribed_velocity<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, ctx->parcels, ctx->cap, profile,
                                                                        vel_geom(ctx));
    ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int mixing(pmpic_ctx* ctx) {
  int frc = flush_gathers(ctx);
  if (frc) return frc;
  const Geom& g = ctx->g;
  const int64_t norig = ctx->n;
  int rc;
  // keep flags (:488) and the kept / residual grids (construct_grids :440-624)
  // (the keep flags are written only once a parcel is known to be removed: without one every
  // original parcel is kept and nothing reads them)
  if ((rc = bin_and_sort(ctx))) return rc;
  // removed slots Z (ascending), counted first: the removed-class grids need a
  // pass over the parcels only when the class is not empty
  int32_t* zlist = ctx->aux;
  int32_t* nz0 = dcounter(ctx, 3);
  if (ctx->mixed) rc = compact(ctx, PredVolBelow<float>{propf(ctx, PMPIC_PROP_VOL), (float)g.vmin}, norig, zlist, nz0);
  else rc = compact(ctx, PredVolBelow<double>{prop(ctx, PMPIC_PROP_VOL), g.vmin}, norig, zlist, nz0);
  if (rc) return rc;
  if (ctx->mixed) {  // the binning counts stay current through mixing
    PMPIC_CUDA(cudaMemsetAsync(ctx->near, 0, (size_t)g.ncell, ctx->stream));
    k_mix_uncount<<<148, 256, 0, ctx->stream>>>(g, zlist, nz0, ctx->cell, ctx->cell_count, ctx->near); ++ctx->nlaunch;
  }
  int32_t hz0 = 0;
  PMPIC_CUDA(cudaMemcpyAsync(&hz0, nz0, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (hz0 > 0 && norig > 0) {
    if (ctx->mixed)
      k_keep_m<<<nblk(norig, 256), 256, 0, ctx->stream>>>(norig, propf(ctx, PMPIC_PROP_VOL), (float)g.vmin, ctx->keep);
    else
      k_keep<<<nblk(norig, 256), 256, 0, ctx->stream>>>(norig, prop(ctx, PMPIC_PROP_VOL), g.vmin, ctx->keep);
    ++ctx->nlaunch;
  }
  if ((rc = launch_mix_grids(ctx, hz0 > 0))) return rc;
  // under-populated cells in loop order
  int32_t* olist = ctx->cell_fill;  // ncell entries; free after bin_and_sort
  int32_t* nnew = dcounter(ctx, 4);
  if ((rc = compact(ctx, PredNewCell{ctx->npercell, g.Nx, g.Ny, g.Nz}, g.ncell, olist, nnew))) return rc;
  int32_t hnew = 0;
  PMPIC_CUDA(cudaMemcpyAsync(&hnew, nnew, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  // A call that removes no parcel and adds none leaves every residual grid at
  // zero: the redistribution (:245-342) would only re-round the kept parcels'
  // properties (b v / v).  The mixed form skips it then; the FP64 path runs it,
  // as the reference does, for the bits.
  const bool events = hz0 > 0 || hnew > 0;
  if (ctx->mixed && !events) {
    const int64_t count0 = norig;
    ctx->n = count0;
    ctx->sorted_valid = true;  // no parcel moved or changed slot: the binning stands
    ctx->count_ready = true;   // and so do the counts
    ctx->in_domain = false;
    ctx->btot_grid_ready = false;
    ctx->info.n_removed = 0;
    ctx->info.n_added = 0;
    PMPIC_CUDA(cudaGetLastError());
    return 0;
  }
  PMPIC_CUDA(cudaMemsetAsync(ctx->newslot, 0xff, sizeof(int32_t) * g.ncell, ctx->stream));
  double* K[6] = {ctx->grid[PMPIC_GRID_VOL], ctx->grid[PMPIC_GRID_B], ctx->grid[PMPIC_GRID_HG],
                  ctx->grid[PMPIC_GRID_P],   ctx->grid[PMPIC_GRID_Q], ctx->grid[PMPIC_GRID_R]};
  if (ctx->mixed) {
    const float* KF[6];
    ResPtrsF RF;
    for (int q = 0; q < 6; ++q) {
      KF[q] = (const float*)K[q];
      RF.r[q] = (float*)ctx->mixres[q];
      RF.k[q] = KF[q];
    }
    float* por = (float*)ctx->newportion;
    // without removed parcels only the kept volume grid was made in full
    if (hz0 == 0 && (rc = launch_kept_corners(ctx, olist, nnew, hnew))) return rc;
    k_new_parcels_m<<<592, 256, 0, ctx->stream>>>(g, olist, nnew, zlist, nz0, norig, ctx->cap, ctx->keep, ctx->parcels,
                                                  KF[0], KF[1], KF[2], KF[3], KF[4], KF[5], ctx->newslot, por,
                                                  (float)g.vmin, ctx->cell, ctx->near, ctx->dinfo); ++ctx->nlaunch;
    k_residual_update_m<<<nblk(g.nphys, 256), 256, 0, ctx->stream>>>(g, RF, ctx->newslot, por, ctx->near);
    ++ctx->nlaunch;
    if (norig > 0) {
      RedistGrids RD;
      RD.kv = KF[0];
      for (int q = 0; q < 6; ++q) RD.r[q] = RF.r[q];
      k_redistribute_m<<<nblk(norig, 256), 256, 0, ctx->stream>>>(g, norig, hz0 > 0 ? ctx->keep : nullptr,
                                                                  ctx->parcels, ctx->cap,
                                                                  ctx->cell, ctx->near, RD);
      ++ctx->nlaunch;
    }
  } else {
    // without removed parcels only the kept volume grid was made in full
    if (hz0 == 0 && (rc = launch_kept_corners(ctx, olist, nnew, hnew))) return rc;
    PMPIC_CUDA(cudaMemsetAsync(ctx->near, 0, (size_t)g.ncell, ctx->stream));
    if (hz0 > 0) {
      k_mark_removed<<<148, 256, 0, ctx->stream>>>(g, zlist, nz0, ctx->cell, ctx->near);
      ++ctx->nlaunch;
    }
    k_new_parcels<<<592, 256, 0, ctx->stream>>>(g, olist, nnew, zlist, nz0, norig, ctx->cap, ctx->keep, ctx->parcels,
                                                K[0], K[1], K[2], K[3], K[4], K[5], ctx->newslot, ctx->newportion,
                                                ctx->near, ctx->dinfo); ++ctx->nlaunch;
    ResPtrs RP;
    for (int q = 0; q < 6; ++q) {
      RP.r[q] = ctx->mixres[q];
      RP.k[q] = K[q];
    }
    k_residual_update<<<nblk(g.nphys, 256), 256, 0, ctx->stream>>>(g, RP, ctx->newslot, ctx->newportion, ctx->near);
    ++ctx->nlaunch;
    if (norig > 0) {
      RedistGridsD RD;
      RD.kv = K[0];
      for (int q = 0; q < 6; ++q) RD.r[q] = RP.r[q];
      k_redistribute<<<nblk(norig, 256), 256, 0, ctx->stream>>>(g, norig, hz0 > 0 ? ctx->keep : nullptr,
                                                                ctx->parcels, ctx->cap,
                                                                ctx->cell, ctx->del, ctx->near, RD); ++ctx->nlaunch;
    }
  }
  const int64_t nremove = hz0, nadd = hnew;
  // count = max(n-1, numparcels_local) (:217)
  int64_t count = norig;
  if (nadd > nremove) count = norig + (nadd - nremove);
  if (nadd > 0 && nadd <= nremove) {
    // the last new parcel sits in a removed slot: count stays norig
    count = norig;
  }
  if (count == norig && nremove > 0) {
    // backfill: keep==0 slots now exclude the ones that received new parcels
    // (keep = 2), except the last slot (:191-193).  With no removed slot there
    // is no keep==0 slot and the reference's loop (:350-389) does nothing.
    int32_t* z2 = ctx->aux;
    int32_t* nz2 = dcounter(ctx, 5);
    int32_t* ones = ctx->aux2 + 2 * ctx->nbmax;
    int32_t* no = dcounter(ctx, 6);
    if ((rc = compact(ctx, PredKeepEq{ctx->keep, 0}, norig, z2, nz2))) return rc;
    if ((rc = compact(ctx, PredKeepEq{ctx->keep, 1}, norig, ones, no))) return rc;
    if (ctx->mixed)
      k_backfill_m<<<592, 256, 0, ctx->stream>>>(z2, nz2, ones, no, ctx->parcels, ctx->cap, ctx->cell, ctx->dinfo);
    else
      k_backfill<<<592, 256, 0, ctx->stream>>>(z2, nz2, ones, no, ctx->parcels, ctx->cap, ctx->dinfo);
    ++ctx->nlaunch;
    int32_t hz = 0;
    PMPIC_CUDA(cudaMemcpyAsync(&hz, nz2, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
    count = norig - hz;
  }
  if (ctx->mixed && (norig > 0 || count > 0)) {
    // with no removal every slot below norig still holds its kept parcel
    const int64_t s0 = nremove > 0 ? 0 : norig;
    const int64_t hi = std::max<int64_t>(norig, count);
    if (hi > s0) {
      k_mix_recount<<<nblk(hi - s0, 256), 256, 0, ctx->stream>>>(g, s0, norig, count, ctx->keep, ctx->cell,
                                                                 ctx->cell_count, ctx->dinfo);
      ++ctx->nlaunch;
    }
  }
  ctx->n = count;
  // without an event no parcel moved or changed slot (the FP64 redistribution
  // changes properties only): the binning made at the start still holds
  ctx->sorted_valid = nremove == 0 && nadd == 0;
  ctx->count_ready = ctx->mixed;  // the next binning starts at the scan
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->info.n_removed = nremove;
  ctx->info.n_added = nadd;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
