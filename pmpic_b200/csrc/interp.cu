// interp.cu -- parcel <-> grid interpolation on the B200.
//
// Restates model_core/src/parcels/parcel_interpolation.F90 (binning :186-262,
// grid2par :267-332, par2grid :336-481) together with the single-rank grid
// halo exchanges of MPIC_Haloswap.F90 (:95-290), which on one GPU become
// periodic index arithmetic in x and y.
//
// par2grid is deterministic and uses no floating-point atomics:
//   1. bin:   each parcel's interior cell id (bit-exact restatement of the
//             reference binning) and an integer histogram of parcels per cell;
//   2. scan:  exclusive scan of the histogram -> CSR offsets per cell;
//   3. scatter the slot indices into cell order (integer atomics only decide
//             positions inside a cell; the reduction below re-sorts each cell
//             segment by slot index, so the summation order is fixed);
//   4. reduce: one CTA per 16x16 column tile and a chunk of z levels walks the
//             cell layers upwards, each thread accumulating the eight corner
//             weights of one cell's parcels in slot order, then adding them into
//             shared-memory level accumulators in four parity phases (cells of
//             one parity class touch disjoint grid points), so every grid point
//             sums its contributions in one fixed order.
#include <cuda_runtime.h>

#include "common.cuh"

namespace pmpic {

namespace {

constexpr int TILE = 16;          // owned grid points per tile edge
constexpr int TC = TILE + 1;      // cells per tile edge incl. the low halo cell
constexpr int P2G_THREADS = 320;  // >= TC*TC = 289
constexpr int ZCHUNK = 16;        // grid levels per CTA
constexpr int MAXSEG = 32;        // cell segments sorted in registers/local memory

__global__ void k_bin_count(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                            const double* __restrict__ Z, int32_t* __restrict__ cell, int32_t* __restrict__ count,
                            DevInfo* info) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ci, cj, ck;
  double dx, dy, dz;
  if (!bin_parcel(g, X[t], Y[t], Z[t], ci, cj, ck, dx, dy, dz)) {
    cell[t] = -1;
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  int32_t id = (int32_t)(((int64_t)ck * g.Ny + cj) * g.Nx + ci);
  cell[t] = id;
  atomicAdd(&count[id], 1);
}

__global__ void k_bin_scatter(int64_t n, const int32_t* __restrict__ cell, const int32_t* __restrict__ start,
                              int32_t* __restrict__ fill, int32_t* __restrict__ sorted) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int32_t id = cell[t];
  if (id < 0) return;
  int32_t pos = start[id] + atomicAdd(&fill[id], 1);
  sorted[pos] = (int32_t)t;
}

// ---- exclusive scan of int32 counts (three-phase) ----------------------------
constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;
  }
  __syncthreads();
  int before = (warp > 0 ? sh[warp - 1] : 0);
  total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void k_scan_tiles(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ tile_sums) {
  __shared__ int sh[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  int s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q)
    if (base + q < n) s += in[base + q];
  int total;
  block_excl_scan(s, sh, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(int32_t* __restrict__ sums, int64_t ntiles, int32_t* __restrict__ grand) {
  __shared__ int sh[32];
  int carry = 0;
  for (int64_t b0 = 0; b0 < ntiles; b0 += blockDim.x) {
    int64_t i = b0 + threadIdx.x;
    int v = (i < ntiles) ? sums[i] : 0;
    int total;
    int ex = block_excl_scan(v, sh, total);
    if (i < ntiles) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int32_t* __restrict__ tile_off,
                             int32_t* __restrict__ out) {
  __shared__ int sh[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  int total;
  int ex = block_excl_scan(s, sh, total) + tile_off[blockIdx.x];
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    if (base + q < n) out[base + q] = ex;
    ex += v[q];
  }
}

// ---- par2grid reduction ----------------------------------------------------------
// MODE 0: par2grid of NQ fields (plus the weights), normalised (:463-469).
// MODE 1: parcel_mixing construct_grids for the kept class (vol >= vmin):
//         NQ = 6 unnormalised sums of (1, b, h, p, q, r) * w, doubled at the
//         walls (parcel_mixing.F90:141-152), plus npercell.
// MODE 2: the same sums for the removed class (vol < vmin), not doubled.
template <int NQ>
struct P2GArgs {
  const double* f[NQ > 0 ? NQ : 1];
  double* out[NQ > 0 ? NQ : 1];
  int32_t* npercell;
  double vmin;
};

template <int NQ, int MODE>
__global__ void __launch_bounds__(P2G_THREADS) k_par2grid(Geom g, const int32_t* __restrict__ start,
                                                          const int32_t* __restrict__ sorted,
                                                          const double* __restrict__ X, const double* __restrict__ Y,
                                                          const double* __restrict__ Z, const double* __restrict__ VOL,
                                                          P2GArgs<NQ> a) {
  constexpr int NA = MODE == 0 ? NQ + 1 : NQ;  // data fields (+ weights)
  __shared__ double acc[2][TC * TC][NA];
  const int t = threadIdx.x;
  const int x0 = blockIdx.x * TILE, y0 = blockIdx.y * TILE;
  const int L0 = blockIdx.z * ZCHUNK;
  const int L1 = min(L0 + ZCHUNK, g.nzp);
  for (int e = t; e < 2 * TC * TC * NA; e += blockDim.x) (&acc[0][0][0])[e] = 0.0;
  // this thread's cell column in the tile
  const int tx = t % TC, ty = t / TC;
  bool has_col = t < TC * TC;
  int ci = x0 - 1 + tx, cj = y0 - 1 + ty;
  if (has_col) {
    if (tx > 0 && ci >= g.Nx) has_col = false;
    if (ty > 0 && cj >= g.Ny) has_col = false;
    if (ci < 0) ci += g.Nx;
    if (cj < 0) cj += g.Ny;
  }
  const int parity = (tx & 1) | ((ty & 1) << 1);
  int cur = 0;
  __syncthreads();
  for (int ck = L0 - 1; ck <= L1 - 1; ++ck) {
    double P[8][NA];
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int q = 0; q < NA; ++q) P[c][q] = 0.0;
    if (has_col && ck >= 0 && ck < g.Nz) {
      int64_t cid = ((int64_t)ck * g.Ny + cj) * g.Nx + ci;
      int s0 = start[cid], len = start[cid + 1] - s0;
      int loc[MAXSEG];
      int nl = len <= MAXSEG ? len : 0;
      for (int u = 0; u < nl; ++u) {
        int v = sorted[s0 + u];
        int w = u - 1;
        while (w >= 0 && loc[w] > v) {
          loc[w + 1] = loc[w];
          --w;
        }
        loc[w + 1] = v;
      }
      int last = -1;
      int nkept = 0;
      for (int u = 0; u < len; ++u) {
        int n;
        if (len <= MAXSEG) {
          n = loc[u];
        } else {  // long segment: select the next larger slot index
          n = 0x7fffffff;
          for (int m = 0; m < len; ++m) {
            int v = sorted[s0 + m];
            if (v > last && v < n) n = v;
          }
          last = n;
        }
        int bi, bj, bk;
        double delx, dely, delz;
        bin_parcel(g, X[n], Y[n], Z[n], bi, bj, bk, delx, dely, delz);
        double v = VOL[n];
        if (MODE == 1 && v < a.vmin) continue;   // parcel_mixing.F90:488
        if (MODE == 2 && !(v < a.vmin)) continue;
        if (MODE == 1) ++nkept;
        // parcel_interpolation.F90:390-434: w = (1-delz)(1-dely)(1-delx) v etc.
        double ez = 1 - delz, ey = 1 - dely, ex = 1 - delx;
        double w[8];
        w[0] = ez * ey * ex * v;
        w[1] = ez * ey * delx * v;
        w[2] = ez * dely * ex * v;
        w[3] = ez * dely * delx * v;
        w[4] = delz * ey * ex * v;
        w[5] = delz * ey * delx * v;
        w[6] = delz * dely * ex * v;
        w[7] = delz * dely * delx * v;
        double fv[NQ > 0 ? NQ : 1];
#pragma unroll
        for (int q = 0; q < NQ; ++q) fv[q] = (MODE != 0 && q == 0) ? 1.0 : a.f[q][n];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
#pragma unroll
          for (int q = 0; q < NQ; ++q) P[c][q] += (MODE != 0 && q == 0) ? w[c] : w[c] * fv[q];
          if (MODE == 0) P[c][NA - 1] += w[c];
        }
      }
      if (MODE == 1 && ck >= L0 && tx > 0 && ty > 0) a.npercell[cid] = nkept;
    }
    // add corners into the level accumulators, one parity class at a time
    // corner c: dz = c>>2, dy = (c>>1)&1, dx = c&1
    for (int ph = 0; ph < 4; ++ph) {
      if (has_col && parity == ph) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          int px = tx + (c & 1), py = ty + ((c >> 1) & 1);
          if (px < TC && py < TC) {
            double* A = acc[cur ^ (c >> 2)][py * TC + px];
#pragma unroll
            for (int q = 0; q < NA; ++q) A[q] += P[c][q];
          }
        }
      }
      __syncthreads();
    }
    // level ck is complete: normalise and store owned points
    if (ck >= L0) {
      for (int e = t; e < TILE * TILE; e += blockDim.x) {
        int lx = e % TILE, ly = e / TILE;
        int gx = x0 + lx, gy = y0 + ly;
        if (gx < g.Nx && gy < g.Ny) {
          const double* A = acc[cur][(ly + 1) * TC + (lx + 1)];
          size_t o = ((size_t)ck * g.Ny + gy) * g.Nx + gx;
          if (MODE == 0) {
            double wv = A[NA - 1];
            if (wv == 0.) wv = 1.;  // parcel_interpolation.F90:466
#pragma unroll
            for (int q = 0; q < NQ; ++q) a.out[q][o] = A[q] / wv;  // :467
          } else {
            const bool wall = (MODE == 1) && (ck == 0 || ck == g.Nz);
#pragma unroll
            for (int q = 0; q < NQ; ++q) a.out[q][o] = wall ? A[q] * 2. : A[q];
          }
        }
      }
    }
    __syncthreads();
    for (int e = t; e < TC * TC * NA; e += blockDim.x) (&acc[cur][0][0])[e] = 0.0;
    cur ^= 1;
    __syncthreads();
  }
}

// ---- grid2par --------------------------------------------------------------------
template <int NG>
struct G2PArgs {
  const double* grid[NG];
  double* out[NG];
};

template <int NG>
__global__ void k_grid2par(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                           const double* __restrict__ Z, G2PArgs<NG> a, DevInfo* info) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ci, cj, ck;
  double delx, dely, delz;
  if (!bin_parcel(g, X[t], Y[t], Z[t], ci, cj, ck, delx, dely, delz)) {
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  int ci1 = ci + 1 == g.Nx ? 0 : ci + 1;  // grid2par_haloswap: periodic copy
  int cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  size_t r00 = ((size_t)ck * g.Ny + cj) * g.Nx, r01 = ((size_t)ck * g.Ny + cj1) * g.Nx;
  size_t r10 = ((size_t)(ck + 1) * g.Ny + cj) * g.Nx, r11 = ((size_t)(ck + 1) * g.Ny + cj1) * g.Nx;
#pragma unroll
  for (int q = 0; q < NG; ++q) {
    const double* G = a.grid[q];
    double c000 = G[r00 + ci], c001 = G[r00 + ci1];
    double c010 = G[r01 + ci], c011 = G[r01 + ci1];
    double c100 = G[r10 + ci], c101 = G[r10 + ci1];
    double c110 = G[r11 + ci], c111 = G[r11 + ci1];
    // parcel_interpolation.F90:309-321: z, then y, then x
    double c00 = c000 * (1 - delz) + c100 * delz;
    double c01 = c001 * (1 - delz) + c101 * delz;
    double c10 = c010 * (1 - delz) + c110 * delz;
    double c11 = c011 * (1 - delz) + c111 * delz;
    double c0 = c00 * (1 - dely) + c10 * dely;
    double c1 = c01 * (1 - dely) + c11 * dely;
    a.out[q][t] = c0 * (1 - delx) + c1 * delx;
  }
}

__global__ void k_cell_only(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                            const double* __restrict__ Z, int32_t* __restrict__ cell, DevInfo* info) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ci, cj, ck;
  double dx, dy, dz;
  if (!bin_parcel(g, X[t], Y[t], Z[t], ci, cj, ck, dx, dy, dz)) {
    cell[t] = -1;
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  cell[t] = (int32_t)(((int64_t)ck * g.Ny + cj) * g.Nx + ci);
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// exclusive scan of n int32 values; out[n] receives the total
int scan_excl(pmpic_ctx* ctx, const int32_t* in, int64_t n, int32_t* out) {
  int64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  int32_t* sums = (int32_t*)ctx->scan_tmp;
  k_scan_tiles<<<(unsigned)ntiles, SCAN_BLOCK, 0, ctx->stream>>>(in, n, sums); ++ctx->nlaunch;
  k_scan_sums<<<1, SCAN_BLOCK, 0, ctx->stream>>>(sums, ntiles, out + n); ++ctx->nlaunch;
  k_scan_apply<<<(unsigned)ntiles, SCAN_BLOCK, 0, ctx->stream>>>(in, n, sums, out); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int bin_and_sort(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_CACHE);
  const Geom& g = ctx->g;
  const int64_t n = ctx->n;
  PMPIC_CUDA(cudaMemsetAsync(ctx->cell_count, 0, sizeof(int32_t) * (g.ncell + 1), ctx->stream));
  PMPIC_CUDA(cudaMemsetAsync(ctx->cell_fill, 0, sizeof(int32_t) * g.ncell, ctx->stream));
  if (n > 0) {
    k_bin_count<<<nblk(n, 256), 256, 0, ctx->stream>>>(g, n, prop(ctx, PMPIC_PROP_X), prop(ctx, PMPIC_PROP_Y),
                                                       prop(ctx, PMPIC_PROP_Z), ctx->cell, ctx->cell_count,
                                                       ctx->dinfo); ++ctx->nlaunch;
  }
  int rc = scan_excl(ctx, ctx->cell_count, g.ncell, ctx->cell_start);
  if (rc) return rc;
  if (n > 0) {
    k_bin_scatter<<<nblk(n, 256), 256, 0, ctx->stream>>>(n, ctx->cell, ctx->cell_start, ctx->cell_fill,
                                                         ctx->sorted); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  ctx->sorted_valid = true;
  return 0;
}

template <int NQ, int MODE = 0>
static int launch_p2g(pmpic_ctx* ctx, const double* const* fields, double* const* out) {
  TimerScope ts(ctx, T_P2G);
  const Geom& g = ctx->g;
  P2GArgs<NQ> a;
  for (int q = 0; q < NQ; ++q) {
    a.f[q] = fields[q];
    a.out[q] = out[q];
  }
  a.npercell = ctx->npercell;
  a.vmin = g.vmin;
  dim3 grid((g.Nx + TILE - 1) / TILE, (g.Ny + TILE - 1) / TILE, (g.nzp + ZCHUNK - 1) / ZCHUNK);
  k_par2grid<NQ, MODE><<<grid, P2G_THREADS, 0, ctx->stream>>>(g, ctx->cell_start, ctx->sorted,
                                                              prop(ctx, PMPIC_PROP_X), prop(ctx, PMPIC_PROP_Y),
                                                              prop(ctx, PMPIC_PROP_Z), prop(ctx, PMPIC_PROP_VOL), a); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// parcel_mixing construct_grids (:440-624) + mixing_haloswap + wall doubling:
// kept grids into VOL, B, HG, P, Q, R (as the reference reuses state%vol,
// state%b, state%hg, state%p, ...), residual grids into mixres, npercell.
int launch_mix_grids(pmpic_ctx* ctx) {
  const double* f[6] = {nullptr, prop(ctx, PMPIC_PROP_B), prop(ctx, PMPIC_PROP_H),
                        prop(ctx, PMPIC_PROP_P), prop(ctx, PMPIC_PROP_Q), prop(ctx, PMPIC_PROP_R)};
  double* kept[6] = {ctx->grid[PMPIC_GRID_VOL], ctx->grid[PMPIC_GRID_B], ctx->grid[PMPIC_GRID_HG],
                     ctx->grid[PMPIC_GRID_P],   ctx->grid[PMPIC_GRID_Q], ctx->grid[PMPIC_GRID_R]};
  int rc = launch_p2g<6, 1>(ctx, f, kept);
  if (rc) return rc;
  return launch_p2g<6, 2>(ctx, f, ctx->mixres);
}

// par2grid of nf fields (1..4) with the same weights; requires bin_and_sort.
int par2grid_multi(pmpic_ctx* ctx, const double* const* fields, int nf, double* const* out, bool) {
  switch (nf) {
    case 1: return launch_p2g<1>(ctx, fields, out);
    case 2: return launch_p2g<2>(ctx, fields, out);
    case 3: return launch_p2g<3>(ctx, fields, out);
    case 4: return launch_p2g<4>(ctx, fields, out);
    default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi: 1..4 fields");
  }
}

template <int NG>
static int launch_g2p(pmpic_ctx* ctx, const double* const* grids, double* const* out) {
  TimerScope ts(ctx, T_G2P);
  const Geom& g = ctx->g;
  if (ctx->n == 0) return 0;
  G2PArgs<NG> a;
  for (int q = 0; q < NG; ++q) {
    a.grid[q] = grids[q];
    a.out[q] = out[q];
  }
  k_grid2par<NG><<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(g, ctx->n, prop(ctx, PMPIC_PROP_X),
                                                              prop(ctx, PMPIC_PROP_Y), prop(ctx, PMPIC_PROP_Z), a,
                                                              ctx->dinfo); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int grid2par_multi(pmpic_ctx* ctx, const double* const* grids, int ng, double* const* out) {
  switch (ng) {
    case 1: return launch_g2p<1>(ctx, grids, out);
    case 3: return launch_g2p<3>(ctx, grids, out);
    case 6: return launch_g2p<6>(ctx, grids, out);
    default: return set_error(ctx, PMPIC_ERR_ARG, "grid2par_multi: 1, 3 or 6 grids");
  }
}

int cell_ids(pmpic_ctx* ctx, int32_t* dcells) {
  if (ctx->n == 0) return 0;
  k_cell_only<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, prop(ctx, PMPIC_PROP_X),
                                                          prop(ctx, PMPIC_PROP_Y), prop(ctx, PMPIC_PROP_Z), dcells,
                                                          ctx->dinfo); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic
