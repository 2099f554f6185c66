// interp.cu -- parcel <-> grid interpolation on the B200.
//
// Restates model_core/src/parcels/parcel_interpolation.F90 (binning :186-262,
// grid2par :267-332, par2grid :336-481) together with the single-rank grid
// halo exchanges of MPIC_Haloswap.F90 (:95-290), which on one GPU become
// periodic index arithmetic in x and y.
//
// Binning is cached exactly like the reference's cache_parcel_interp_weights:
// per parcel the interior cell id and delx, dely, delz, computed once per
// substep with the reference's arithmetic (bit-exact) and reused by par2grid,
// grid2par and the mixing redistribution.  Cell ids here are z fastest,
// id = (i*Ny + j)*Nz + k, the order in which the set-up stores parcels
// (basic_parcelsetup.F90:90-118: x outer, z inner), so that the parcels of a
// column of cells are one contiguous run of the cell-sorted index.
//
// par2grid is deterministic and uses no floating-point atomics:
//   1. bin:     cell ids + cached offsets + an integer histogram per cell;
//   2. scan:    exclusive scan of the histogram -> CSR offsets per cell;
//   3. scatter: slot indices into cell order, then each cell segment sorted
//               by slot index, so every later sum runs in slot order;
//   4. reduce:  row pass + combine pass (see k_p2g_rows), each grid point
//               summing its contributions in one fixed order.
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "common.cuh"

namespace pmpic {

namespace {

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- binning (cache_parcel_interp_weights, parcel_interpolation.F90:186-262) ----
// (whint, when given: each block's first cell, the window hint of the FP64 RK4 stage)
__global__ void k_bin_count(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                            const double* __restrict__ Z, int32_t* __restrict__ cell, double* __restrict__ del,
                            int64_t cap, int32_t* __restrict__ count, DevInfo* info,
                            int32_t* __restrict__ whint = nullptr) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ci, cj, ck;
  double dx, dy, dz;
  if (!bin_parcel(g, X[t], Y[t], Z[t], ci, cj, ck, dx, dy, dz)) {
    cell[t] = -1;
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  int32_t id = (int32_t)(((int64_t)ci * g.Ny + cj) * g.Nz + ck);
  cell[t] = id;
  if (whint && threadIdx.x == 0) whint[blockIdx.x] = id;
  del[t] = dx;
  del[cap + t] = dy;
  del[2 * cap + t] = dz;
  count_cell(id, count);
}

// the mixed form's binning: the cell id is part of the position already; the
// pass only checks it and counts the cells
__global__ void k_bin_count_m(Geom g, int64_t n, const int32_t* __restrict__ cell, const float* __restrict__ FX,
                              const float* __restrict__ FY, const float* __restrict__ FZ,
                              int32_t* __restrict__ count, DevInfo* info) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int32_t id = cell[t];
  const float fx = FX[t], fy = FY[t], fz = FZ[t];
  if (id < 0 || id >= g.ncell || !(fx >= 0.f && fx <= 1.f) || !(fy >= 0.f && fy <= 1.f) || !(fz >= 0.f && fz <= 1.f)) {
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  count_cell(id, count);
}

// Slots into their cells' ranges.  Each thread takes SC_ITEMS slots (a block's
// slots are SC_ITEMS runs of 256, a warp's 32 consecutive slots per item).
// A cell whose slots form one contiguous run (parcels still in set-up order, or
// at rest) is placed without atomics: the warp holding part of the run knows
// the run's slots before and after its window (counted back and forward
// against the cell's count), so each slot's place is start + its rank in the
// run, the slot order.  Every other cell's slots take places from one fill
// atomic per distinct cell of a warp (issued for all items before any result
// is used, so their round trips overlap), and such a cell's segment is sorted
// by slot afterwards (its fill counter is then non-zero).  Whether a cell is
// one run is a property of the cell, so all its slots take the same path.
// The 32 slots either side of a window are loaded with the window (one
// coalesced load each, mostly L1 hits) and the run's extent there is read off
// two ballots; only a run reaching past them is followed further slot by slot.
constexpr int SC_ITEMS = 4;
// the total of counts kept current by other kernels against the parcel count
// (a mismatch would leave the cell index inconsistent: reported as an error)
__global__ void k_check_total(const int32_t* __restrict__ total, int64_t n, DevInfo* info) {
  if (*total != n) atomicCAS(&info->error, 0, PMPIC_ERR_STATE);
}
__global__ void __launch_bounds__(256) k_bin_scatter(int64_t n, const int32_t* __restrict__ cell,
                                                     const int32_t* __restrict__ count,
                                                     const int32_t* __restrict__ start, int32_t* __restrict__ fill,
                                                     int32_t* __restrict__ sorted, int64_t lim) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t t0 = (int64_t)blockIdx.x * 256 * SC_ITEMS + threadIdx.x;
  int32_t id[SC_ITEMS], prv[SC_ITEMS], nxt[SC_ITEMS], base[SC_ITEMS], st[SC_ITEMS], cnt[SC_ITEMS];
  unsigned same[SC_ITEMS];
#pragma unroll
  for (int k = 0; k < SC_ITEMS; ++k) {  // the window and the 32 slots either side (-2 outside)
    const int64_t t = t0 + 256 * k;
    id[k] = t < n ? cell[t] : -1;
    prv[k] = t - 32 >= 0 && t - 32 < n ? cell[t - 32] : -2;
    nxt[k] = t + 32 < n ? cell[t + 32] : -2;
  }
#pragma unroll
  for (int k = 0; k < SC_ITEMS; ++k) {
    same[k] = __match_any_sync(FULL, id[k]);
    const bool lead = id[k] >= 0 && lane == __ffs(same[k]) - 1;
    cnt[k] = lead ? count[id[k]] : 0;
    st[k] = id[k] >= 0 ? start[id[k]] : 0;
  }
#pragma unroll
  for (int k = 0; k < SC_ITEMS; ++k) {
    // slots of lane 0's cell just before the window, of lane 31's just after
    const unsigned bb = __ballot_sync(FULL, prv[k] == __shfl_sync(FULL, id[k], 0));
    const unsigned ba = __ballot_sync(FULL, nxt[k] == __shfl_sync(FULL, id[k], 31));
    const int nbefore = __clz(~bb);                        // from slot w0-1 down (32 when all match)
    const int nafter = ba == FULL ? 32 : __ffs(~ba) - 1;  // from slot w0+32 up
    base[k] = 0;
    const int first = __ffs(same[k]) - 1;
    if (id[k] >= 0 && lane == first) {
      // the run containing this window's slots of the cell: contiguous here,
      // extended by the cell's slots just before and after the window
      const int64_t w0 = t0 + 256 * k - lane;  // the window's first slot
      const int last = 31 - __clz(same[k]);
      const unsigned m = same[k] >> first;
      const int gsize = __popc(same[k]);
      const int c = cnt[k];
      bool run = (m & (m + 1)) == 0;
      int before = 0, after = 0;
      if (run && gsize < c) {
        if (first == 0) {
          before = min(nbefore, c - gsize);
          if (before == 32)
            for (int64_t s = w0 - 33; s >= 0 && before < c - gsize && cell[s] == id[k]; --s) ++before;
        }
        if (last == 31) {
          after = min(nafter, c - gsize - before);
          if (after == 32)
            for (int64_t s = w0 + 64; s < n && before + after < c - gsize && cell[s] == id[k]; ++s) ++after;
        }
      }
      run = run && before + gsize + after == c;
      base[k] = run ? before : atomicAdd(&fill[id[k]], gsize);
    }
  }
#pragma unroll
  for (int k = 0; k < SC_ITEMS; ++k) {
    const int32_t b = __shfl_sync(FULL, base[k], __ffs(same[k]) - 1);
    const int64_t pos = (int64_t)st[k] + b + __popc(same[k] & ((1u << lane) - 1));
    if (id[k] >= 0 && pos < lim) sorted[pos] = (int32_t)(t0 + 256 * k);  // (pos < n with exact counts)
  }
}

// Each cell's segment sorted by slot index (the integer atomics above only
// decide the order inside a cell that did not lie in one run of slots; such a
// cell's fill counter is non-zero).  A CTA takes SORT_CELLS consecutive cells,
// whose segments are one contiguous range of the index: when any of them needs
// it, the range is read into shared memory with coalesced loads, every thread
// insertion-sorts its cell's segment there (the slots are nearly in order
// already), and the range is written back.
constexpr int SORT_CELLS = 256;
constexpr int SORT_CAP = 8192;  // index entries a CTA stages (32 KB)
__global__ void __launch_bounds__(SORT_CELLS) k_sort_segments(int64_t ncell, const int32_t* __restrict__ start,
                                                              const int32_t* __restrict__ fill,
                                                              int32_t* __restrict__ sorted) {
  // staged position e sits at e + e/8: segments (~8 parcels each) start in
  // different banks for neighbouring threads
  __shared__ int32_t buf[SORT_CAP + SORT_CAP / 8];
  const int64_t c0 = (int64_t)blockIdx.x * SORT_CELLS;
  const int64_t c = c0 + threadIdx.x;
  if (!__syncthreads_or(c < ncell && fill[c] != 0)) return;  // every segment here is one run: in order
  const int64_t c1 = min(c0 + SORT_CELLS, ncell);
  const int base = start[c0], m = start[c1] - base;
  int s0 = 0, len = 0;
  if (c < ncell) {
    s0 = start[c] - base;
    len = start[c + 1] - base - s0;
  }
  auto isort = [](int32_t* s, int s0, int len, auto at) {
    for (int u = 1; u < len; ++u) {
      const int32_t v = s[at(s0 + u)];
      int w = u - 1;
      while (w >= 0 && s[at(s0 + w)] > v) {
        s[at(s0 + w + 1)] = s[at(s0 + w)];
        --w;
      }
      s[at(s0 + w + 1)] = v;
    }
  };
  auto skew = [](int e) { return e + (e >> 3); };
  if (m <= SORT_CAP) {  // uniform over the CTA
    for (int e = threadIdx.x; e < m; e += SORT_CELLS) buf[skew(e)] = sorted[base + e];
    __syncthreads();
    isort(buf, s0, len, skew);
    __syncthreads();
    for (int e = threadIdx.x; e < m; e += SORT_CELLS) sorted[base + e] = buf[skew(e)];
  } else {  // cells holding more than SORT_CAP parcels together: in place in global memory
    isort(sorted + base, s0, len, [](int e) { return e; });
  }
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
//         With BT, field NQ-1 is btot = b + 12.5 max(0, h - exp(-z)) computed
//         per parcel (vorticity_tendency.F90:121-126).
// MODE 1: parcel_mixing construct_grids for the kept class (vol >= vmin):
//         NQ = 6 unnormalised sums of (1, b, h, p, q, r) * w, doubled at the
//         walls (parcel_mixing.F90:141-152), plus npercell.
// MODE 2: the same sums for the removed class (vol < vmin), not doubled.
//
// Two passes, no atomics; every grid point sums its contributions in one fixed
// order that does not depend on timing:
//  1. k_p2g_rows: one warp per (x segment, row of cells y = cy, chunk of ZC
//     cell layers) walks the segment's columns in x order.  Cell ids are z
//     fastest, so a column chunk's parcels are one contiguous range of the
//     cell-sorted index, and with parcels stored in cell order (as the set-up
//     writes them) one contiguous range of slots: the gathers are coalesced.
//     Two lanes per cell layer (bottom and top z corner) accumulate the four
//     xy corners of their z corner over the cell's parcels in slot order.  A
//     shuffle adds the top corners of layer k-1 to the bottom corners of layer
//     k (grid level k), and a register carry adds the x-high corners of column
//     x-1 to the x-low corners of column x (grid point x).  The result, per
//     grid point and level, is the sum over the point's four cells of this
//     row, separately for the row below (y-high corners) and above (y-low
//     corners): the row partials.
//  2. k_p2g_combine: per grid point, row y-1's y-high part plus row y's y-low
//     part (and, on the bottom level of a chunk, the chunk below's top level
//     first), then the normalisation or wall doubling.
template <int NQ, class R = double>
struct P2GArgs {
  const R* f[NQ] = {};      // per-parcel fields (MODE 1/2: f[0] unused)
  R* out[NQ] = {};
  // BT: b, h and z of btot; on the mixed form z is not staged (its cell layer
  // is known from the column's layer bounds, its offset is staged as delz)
  const R* bh[3] = {};
  R* btot = nullptr;        // BT: the btot property, written as staged
  int64_t nslot = 0;        // parcel count: staged slot indices are checked against it
  int32_t* npercell = nullptr;
  double vmin = 0.0;
};

constexpr int ZC = 16;                    // cell layers per z chunk: two lanes per layer
constexpr int NLV = ZC + 1;               // grid levels a chunk contributes to
constexpr int BATCH = 128;                // sorted positions staged per batch
constexpr int SPAD = BATCH + BATCH / 16;  // staged field stride: position p sits at p + p/16
constexpr int RW = 4;                     // warps per CTA of the row pass
constexpr int XSEG = 64;                  // default columns per x segment of a warp (tunable per context)
// grid points in x per CTA of the combine pass (its staged rows fit the
// 48 KB of static shared memory)
template <class R>
struct P2GPx {
  static constexpr int value = sizeof(R) == 8 ? 16 : 32;
};

template <int NQ, int MODE, bool BT>
struct P2GLayout {
  static constexpr int NA = MODE == 0 ? NQ + 1 : NQ;  // accumulated quantities per corner
  static constexpr int NF = MODE == 0 ? NQ : NQ - 1;  // per-parcel fields staged (btot counts as one)
  static constexpr int NS = 4 + NF + (BT ? 2 : 0);    // + delx, dely, delz, vol (+ h, z for btot)
  static constexpr int RPS = 2 * NA * NLV;            // doubles of row partials per (chunk, row, column)
};

// largest row-partial record of any instantiation: MODE 1/2 with NQ = 6
constexpr int RPS_MAX = 2 * 6 * NLV;

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
// one staged value of type R
template <class R>
__device__ __forceinline__ void cp_async_r(R* smem, const R* gmem) {
  if constexpr (sizeof(R) == 8) cp_async8(smem, gmem);
  else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }


// acc + w * f: one rounding (FMA) on the FP32 form; on the FP64 path the
// product and the sum are rounded separately, as the reference computes them
__device__ __forceinline__ double madd(double w, double f, double acc) { return acc + w * f; }
__device__ __forceinline__ float madd(float w, float f, float acc) { return __fmaf_rn(w, f, acc); }

// R: the arithmetic type (double: plain path, float: mixed-precision form).
// The cell offsets delx, dely, delz of parcel n are DX[n], DY[n], DZ[n]: the
// cached binning on the plain path, the offsets of the current position on
// the mixed form (ds = 1 on both; a stride ds > 1 reads interleaved offsets).
template <int NQ, int MODE, bool BT, class R = double>
__global__ void __launch_bounds__(32 * RW, sizeof(R) == 4 ? 6 : 4) k_p2g_rows(Geom g, int nzc, int nxs, int xseg, const int32_t* __restrict__ start,
                                                     const int32_t* __restrict__ sorted, const R* __restrict__ DX,
                                                     const R* __restrict__ DY, const R* __restrict__ DZ, int ds,
                                                     const R* __restrict__ VOL, P2GArgs<NQ, R> a,
                                                     R* __restrict__ rowpart) {
  using Lay = P2GLayout<NQ, MODE, BT>;
  constexpr int NA = Lay::NA, NS = Lay::NS;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ __align__(16) R smem[RW][NS * SPAD];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t wid = (int64_t)blockIdx.x * RW + warp;
  if (wid >= (int64_t)nxs * g.Ny * nzc) return;  // the whole warp leaves together
  const int xs = (int)(wid % nxs);
  const int cy = (int)((wid / nxs) % g.Ny);
  const int zc = (int)(wid / ((int64_t)nxs * g.Ny));
  const int x_lo = xs * xseg, x_hi = min(g.Nx, x_lo + xseg);
  const int k0 = zc * ZC, nk = min(ZC, g.Nz - k0);
  const int kk = lane >> 1, cz = lane & 1;
  const bool has_cell = kk < nk;
  // after the z combination lane 0 holds level 0 (bottom corners of layer 0)
  // and odd lane 2m+1 level m+1 (top corners of layer m + bottom corners of m+1)
  const int lev = lane == 0 ? 0 : (lane >> 1) + 1;
  const bool owner = (lane == 0 || (lane & 1)) && lev <= nk;
  // row partials in two halves (y-low corners, then y-high corners), each
  // nzc * Ny * Nx records of NA * NLV values: the combine pass reads each
  // half of a row contiguously
  constexpr int SEG = Lay::RPS / 2;  // NA * NLV
  const size_t half = (size_t)nzc * g.Ny * g.Nx * SEG;
  R* out_row = rowpart + ((size_t)zc * g.Ny + cy) * (size_t)g.Nx * SEG;
  R C[2][NA];  // x-high corners of the previous column, per y corner
  auto bounds = [&](int it, int& s, int& e) {  // this lane's cell layer of column it
    int cx = x_lo + it;
    if (cx < 0) cx += g.Nx;
    const int64_t cb = ((int64_t)cx * g.Ny + cy) * g.Nz + k0;
    s = e = 0;
    if (has_cell) {
      s = start[cb + kk];
      e = start[cb + kk + 1];
    }
  };
  auto slots = [&](int b0, int nb, int* sl) {
#pragma unroll
    for (int j = 0; j < BATCH / 32; ++j) {
      const int p = lane + 32 * j;
      sl[j] = (p < nb && b0 + p < a.nslot) ? sorted[b0 + p] : -1;  // (index positions lie below the count)
    }
  };
  // the fields of a batch of parcels into shared memory, field-major, position
  // p at p + p/16 (no bank conflicts for the readers)
  auto stage = [&](R* Sb, const int* sl) {
#pragma unroll
    for (int j = 0; j < BATCH / 32; ++j) {
      const int n = sl[j];
      if (n < 0 || n >= a.nslot) continue;  // (an index entry is always a slot below the count)
      const int p = lane + 32 * j;
      R* D = Sb + p + (p >> 4);
      const size_t nd = (size_t)ds * n;
      cp_async_r(D, DX + nd);
      cp_async_r(D + SPAD, DY + nd);
      cp_async_r(D + 2 * SPAD, DZ + nd);
      cp_async_r(D + 3 * SPAD, VOL + n);
      if (MODE == 0) {
#pragma unroll
        for (int f = 0; f < (BT ? NQ - 1 : NQ); ++f) cp_async_r(D + (4 + f) * SPAD, a.f[f] + n);
        if (BT) {
          cp_async_r(D + (4 + NQ - 1) * SPAD, a.bh[0] + n);
          cp_async_r(D + (4 + NQ) * SPAD, a.bh[1] + n);
          if constexpr (sizeof(R) == 8) cp_async_r(D + (4 + NQ + 1) * SPAD, a.bh[2] + n);
        }
      } else {
#pragma unroll
        for (int f = 1; f < NQ; ++f) cp_async_r(D + (4 + f - 1) * SPAD, a.f[f] + n);
      }
    }
  };
  // btot per staged parcel (vorticity_tendency.F90:121-126), also stored as
  // the property.  On the mixed form z is (k + delz) dz, with k the cell layer
  // of the parcel's index position b0 + p among the column's layer starts LS.
  __shared__ int LS[RW][ZC + 1];
  auto btot_pass = [&](R* Sb, const int* sl, int nb, int b0) {
#pragma unroll
    for (int j = 0; j < BATCH / 32; ++j) {
      const int p = lane + 32 * j;
      if (p >= nb) continue;
      R* D = Sb + p + (p >> 4) + (4 + NQ - 1) * SPAD;
      const R bb = D[0], hh = D[SPAD];
      R bt;
      if constexpr (sizeof(R) == 8) {
        bt = bb + 12.5 * fmax(0.0, hh - exp(-D[2 * SPAD]));
      } else {  // z from its cell layer and offset, in FP32
        const int pos = b0 + p;
        int l = 0;
#pragma unroll 1
        for (int step = 8; step > 0; step >>= 1)  // the last layer start at or below pos
          if (l + step < nk && LS[warp][l + step] <= pos) l += step;
        const float zz = ((float)(k0 + l) + Sb[p + (p >> 4) + 2 * SPAD]) * (float)g.dz;
        bt = bb + 12.5f * fmaxf(0.f, hh - expf(-zz));
      }
      D[0] = bt;
      a.btot[sl[j]] = bt;  // a seed-column parcel is staged by two warps: the same value twice
    }
    __syncwarp();
  };
  // this lane's parcels (its cell layer, its z corner) among staged positions
  // b0 .. b0+nb-1, in slot order
  auto accumulate = [&](const R* Sb, int b0, int nb, int s_me, int e_me, R (&acc)[4][NA], int& nkept) {
    const int lo = max(s_me, b0) - b0, hi = min(e_me, b0 + nb) - b0;
    for (int p = lo; p < hi; ++p) {
      const R* D = Sb + p + (p >> 4);
      const R delx = D[0], dely = D[SPAD], delz = D[2 * SPAD], vv = D[3 * SPAD];
      if (MODE == 1 && vv < a.vmin) continue;  // parcel_mixing.F90:488
      if (MODE == 2 && !(vv < a.vmin)) continue;
      if (MODE == 1) ++nkept;
      // parcel_interpolation.F90:390-434: w = (1-delz)(1-dely)(1-delx) v etc.,
      // evaluated left to right as there
      const R ez = cz ? delz : R(1) - delz;
      const R zy0 = ez * (R(1) - dely), zy1 = ez * dely;
      R w[4];
      w[0] = zy0 * (R(1) - delx) * vv;
      w[1] = zy0 * delx * vv;
      w[2] = zy1 * (R(1) - delx) * vv;
      w[3] = zy1 * delx * vv;
      R fv[NA];
      if (MODE == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) fv[q] = D[(4 + q) * SPAD];
      } else {
#pragma unroll
        for (int q = 1; q < NQ; ++q) fv[q] = D[(4 + q - 1) * SPAD];
      }
#pragma unroll
      for (int ab = 0; ab < 4; ++ab) {
        if (MODE == 0) {
#pragma unroll
          for (int q = 0; q < NQ; ++q) acc[ab][q] = madd(w[ab], fv[q], acc[ab][q]);
          acc[ab][NQ] += w[ab];
        } else {
          acc[ab][0] += w[ab];
#pragma unroll
          for (int q = 1; q < NQ; ++q) acc[ab][q] = madd(w[ab], fv[q], acc[ab][q]);
        }
      }
    }
  };
  // the column's z combination, its row partials (grid point x = cx: x-high
  // corners of column cx-1, then x-low corners of column cx) and the carry
  auto finish = [&](int it, R (&acc)[4][NA], int nkept) {
    // level m+1 = top corners of layer m (odd lane 2m+1) + bottom corners of layer m+1 (lane 2m+2)
#pragma unroll
    for (int ab = 0; ab < 4; ++ab)
#pragma unroll
      for (int q = 0; q < NA; ++q) {
        const R o = __shfl_down_sync(FULL, acc[ab][q], 1);
        if ((lane & 1) && kk + 1 < nk) acc[ab][q] = acc[ab][q] + o;
      }
    if (it >= 0) {
      const int cx = x_lo + it;
      if (owner) {
        R* dst = out_row + (size_t)cx * SEG + lev;
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int q = 0; q < NA; ++q) dst[b * half + q * NLV] = C[b][q] + acc[2 * b][q];
      }
      if (MODE == 1 && cz == 0 && has_cell) a.npercell[((int64_t)(k0 + kk) * g.Ny + cy) * g.Nx + cx] = nkept;
    }
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int q = 0; q < NA; ++q) C[b][q] = acc[2 * b + 1][q];
  };
  const int last = x_hi - x_lo - 1;  // columns -1 .. last; -1 (periodic) only seeds the carry
  {
    // column it+1's bounds and first slots are loaded ahead, so a column
    // waits on one memory latency (its staged fields), not three
    R* S = smem[warp];
    int s_me, e_me;
    bounds(-1, s_me, e_me);
    int q0 = __shfl_sync(FULL, s_me, 0);
    int q1 = __shfl_sync(FULL, e_me, 2 * nk - 2);
    int pre[BATCH / 32];
    slots(q0, min(BATCH, q1 - q0), pre);
    for (int it = -1; it <= last; ++it) {
      const bool more = it + 1 <= last;
      int s_nx = 0, e_nx = 0, q0n = 0, q1n = 0;
      if (more) bounds(it + 1, s_nx, e_nx);
      R acc[4][NA];
#pragma unroll
      for (int ab = 0; ab < 4; ++ab)
#pragma unroll
        for (int q = 0; q < NA; ++q) acc[ab][q] = R(0);
      int nkept = 0;
      bool prefetched = false;
      if constexpr (BT && sizeof(R) == 4) {  // this column's layer starts for btot's z
        __syncwarp();
        if (cz == 0 && has_cell) LS[warp][kk] = s_me;
        __syncwarp();
      }
      for (int b0 = q0; b0 < q1; b0 += BATCH) {
        const int nb = min(BATCH, q1 - b0);
        __syncwarp();  // the previous batch has been read
        int slot[BATCH / 32];
        if (b0 == q0) {
#pragma unroll
          for (int j = 0; j < BATCH / 32; ++j) slot[j] = pre[j];
        } else {
          slots(b0, nb, slot);
        }
        stage(S, slot);
        if (more && b0 + BATCH >= q1) {  // the column's last batch: the next column's first slots
          q0n = __shfl_sync(FULL, s_nx, 0);
          q1n = __shfl_sync(FULL, e_nx, 2 * nk - 2);
          slots(q0n, min(BATCH, q1n - q0n), pre);
          prefetched = true;
        }
        cp_async_wait_all();
        __syncwarp();
        if constexpr (BT) btot_pass(S, slot, nb, b0);
        accumulate(S, b0, nb, s_me, e_me, acc, nkept);
      }
      if (more && !prefetched) {  // an empty column
        q0n = __shfl_sync(FULL, s_nx, 0);
        q1n = __shfl_sync(FULL, e_nx, 2 * nk - 2);
        slots(q0n, min(BATCH, q1n - q0n), pre);
      }
      finish(it, acc, nkept);
      s_me = s_nx;
      e_me = e_nx;
      q0 = q0n;
      q1 = q1n;
    }
  }
}

// per grid point: the y-high part of row y-1 plus the y-low part of row y; on
// the bottom level of a chunk the chunk below's top level comes first
template <int NQ, int MODE, class R = double>
__global__ void __launch_bounds__(256) k_p2g_combine(Geom g, int nzc, const R* __restrict__ rowpart,
                                                    P2GArgs<NQ, R> a) {
  constexpr int NA = MODE == 0 ? NQ + 1 : NQ;
  constexpr int SEG = NA * NLV;
  constexpr int TS = SEG | 1;  // odd stride: conflict-free reads by consecutive points
  constexpr int PX = P2GPx<R>::value;
  __shared__ __align__(16) R T[2][PX * TS];  // [0]: row y (y-low part), [1]: row y-1 (y-high part)
  __shared__ R Bz[2][PX * NA];               // the chunk below's top level, same rows
  const int px0 = blockIdx.x * PX, py = blockIdx.y, zc = blockIdx.z;
  const int pym = py == 0 ? g.Ny - 1 : py - 1;
  const size_t half = (size_t)nzc * g.Ny * g.Nx * SEG;  // the y-high half follows the y-low one
  const int npx = min(PX, g.Nx - px0);
  const int k0 = zc * ZC, nk = min(ZC, g.Nz - k0);
  // the CTA's records of a row are one contiguous range of npx * SEG values:
  // copied with 16-byte loads where the range is 16-byte aligned
  for (int r = 0; r < 2; ++r) {
    const int row = r == 0 ? py : pym;
    const R* src = rowpart + r * half + (((size_t)zc * g.Ny + row) * g.Nx + px0) * SEG;
    R* dst = T[r];
    const int len = npx * SEG;
    constexpr int V = 16 / sizeof(R);
    if (((uintptr_t)src & 15) == 0 && len % V == 0) {
      for (int e = threadIdx.x; e < len / V; e += blockDim.x) {
        const float4 u = __ldcs(reinterpret_cast<const float4*>(src) + e);
        if constexpr (TS == SEG) {  // unpadded: the range as it lies (T[r] is 16-byte aligned)
          reinterpret_cast<float4*>(dst)[e] = u;
        } else {
          const R* uv = reinterpret_cast<const R*>(&u);
#pragma unroll
          for (int c = 0; c < V; ++c) {
            const int f = e * V + c, pxl = f / SEG;
            dst[pxl * TS + (f - pxl * SEG)] = uv[c];
          }
        }
      }
    } else {
      for (int f = threadIdx.x; f < len; f += blockDim.x) {
        const int pxl = f / SEG;
        dst[pxl * TS + (f - pxl * SEG)] = src[f];
      }
    }
  }
  if (zc > 0) {
    for (int e = threadIdx.x; e < 2 * PX * NA; e += blockDim.x) {
      const int r = e / (PX * NA);
      const int rem = e - r * PX * NA;
      const int pxl = rem / NA, q = rem - pxl * NA;
      if (pxl >= npx) continue;
      const int row = r == 0 ? py : pym;
      Bz[r][pxl * NA + q] = rowpart[r * half + (((size_t)(zc - 1) * g.Ny + row) * g.Nx + px0 + pxl) * SEG + q * NLV + ZC];
    }
  }
  __syncthreads();
  // levels this chunk completes: its bottom nk, and the top level on the last chunk
  const int nlev = k0 + nk == g.Nz ? nk + 1 : nk;
  for (int e = threadIdx.x; e < nlev * PX; e += blockDim.x) {
    const int L = e / PX, pxl = e - L * PX;
    if (pxl >= npx) continue;
    R v[NA];
#pragma unroll
    for (int q = 0; q < NA; ++q) v[q] = T[1][pxl * TS + q * NLV + L] + T[0][pxl * TS + q * NLV + L];
    if (L == 0 && zc > 0) {
#pragma unroll
      for (int q = 0; q < NA; ++q) v[q] = (Bz[1][pxl * NA + q] + Bz[0][pxl * NA + q]) + v[q];
    }
    const int gl = k0 + L;
    const size_t o = ((size_t)gl * g.Ny + py) * g.Nx + px0 + pxl;
    if (MODE == 0) {
      R wv = v[NQ];
      if (wv == R(0)) wv = R(1);  // parcel_interpolation.F90:466
      if constexpr (sizeof(R) == 8) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) a.out[q][o] = v[q] / wv;  // :467
      } else {  // the FP32 form: one reciprocal for the point's fields
        const R rw = R(1) / wv;
#pragma unroll
        for (int q = 0; q < NQ; ++q) a.out[q][o] = v[q] * rw;
      }
    } else {
      const bool wall = (MODE == 1) && (gl == 0 || gl == g.Nz);
#pragma unroll
      for (int q = 0; q < NQ; ++q) a.out[q][o] = wall ? v[q] * R(2) : v[q];
    }
  }
}

// construct_grids (parcel_mixing.F90:440-624) with the wall doubling
// (:141-152) for b, h, p, q, r at single grid points: the eight corners of
// each new parcel's cell, on the mixed form in a mixing call that removes no
// parcel.  Mixing reads those five grids nowhere else then (the new parcels'
// box sums :174-186 and their residual portions :202-207); the kept volume
// grid is made in full.  One warp per (new cell, corner): the lanes take the
// kept parcels of the point's cells (x, then y, then z low and high, each
// cell's parcels in slot order) in turn, and a fixed shuffle tree adds their
// shares, so a point's sums do not depend on timing.  A point shared by two
// new cells is written twice with the same value.
template <class R>
struct KeptCorners {
  const R* f[5];  // b, h, p, q, r
  R* out[5];      // the B, HG, P, Q, R grids
  double vmin;
};
template <class R>
__global__ void __launch_bounds__(256) k_kept_corners(Geom g, const int32_t* __restrict__ olist,
                                                      const int32_t* __restrict__ nnew,
                                                      const int32_t* __restrict__ start,
                                                      const int32_t* __restrict__ sorted, const R* __restrict__ DX,
                                                      const R* __restrict__ DY, const R* __restrict__ DZ,
                                                      const R* __restrict__ VOL, KeptCorners<R> a) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int u = threadIdx.x >> 5;  // the corner: x low/high, then y, then z
  const int64_t e = blockIdx.x;
  if (e >= *nnew) return;  // the whole block leaves together
  int ci, cj, ck;
  cell_decode(g, olist[e], ci, cj, ck);
  const int px = wrap_index(ci + (u & 1), g.Nx), py = wrap_index(cj + ((u >> 1) & 1), g.Ny), pz = ck + (u >> 2);
  // the point's cells m = sx + 2 sy + 4 sz: cell (px-1+sx, py-1+sy, pz-1+sz),
  // of which the point is corner (1-sx, 1-sy, 1-sz); cells below z = 0 or at
  // z = Nz do not exist
  int cs[8], len[8];
  int tot = 0;
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int cz = pz - 1 + (m >> 2);
    cs[m] = 0;
    len[m] = 0;
    if (cz >= 0 && cz < g.Nz) {
      const int32_t id = cell_encode(g, wrap_index(px - 1 + (m & 1), g.Nx), wrap_index(py - 1 + ((m >> 1) & 1), g.Ny), cz);
      cs[m] = start[id];
      len[m] = start[id + 1] - cs[m];
    }
    tot += len[m];
  }
  R acc[5] = {R(0), R(0), R(0), R(0), R(0)};
  for (int t = lane; t < tot; t += 32) {
    int m = 0, off = t;
    while (off >= len[m]) off -= len[m++];  // t < tot: ends at a cell holding position t
    const int32_t n = sorted[cs[m] + off];
    const R vv = VOL[n];
    if (vv < a.vmin) continue;  // parcel_mixing.F90:488
    const R delx = DX[n], dely = DY[n], delz = DZ[n];
    // the corner's weight and products as the par2grid pass evaluates them
    const R ez = (m >> 2) ? (R(1) - delz) : delz;
    const R zy = ez * (((m >> 1) & 1) ? (R(1) - dely) : dely);
    const R w = zy * ((m & 1) ? (R(1) - delx) : delx) * vv;
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] = madd(w, a.f[q][n], acc[q]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += __shfl_xor_sync(FULL, acc[q], o);
  if (lane == 0) {
    const bool wall = pz == 0 || pz == g.Nz;
    const size_t gi = ((size_t)pz * g.Ny + py) * g.Nx + px;
#pragma unroll
    for (int q = 0; q < 5; ++q) a.out[q][gi] = wall ? acc[q] * R(2) : acc[q];
  }
}

// z-fastest cell id -> x-fastest id ((k*Ny + j)*Nx + i); -1 stays -1
__global__ void k_cell_xfast(Geom g, int64_t n, const int32_t* __restrict__ cell, int32_t* __restrict__ out) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int32_t id = cell[t];
  if (id < 0) {
    out[t] = -1;
    return;
  }
  const int ck = id % g.Nz, cj = (id / g.Nz) % g.Ny, ci = id / (g.Nz * g.Ny);
  out[t] = (int32_t)(((int64_t)ck * g.Ny + cj) * g.Nx + ci);
}

// ---- grid2par --------------------------------------------------------------------
template <int NG>
struct G2PArgs {
  const double* grid[NG];
  double* out[NG];
};

template <int NG>
__global__ void k_grid2par(Geom g, int64_t n, const int32_t* __restrict__ cell, const double* __restrict__ del,
                           int64_t cap, G2PArgs<NG> a) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int32_t id = cell[t];
  if (id < 0) return;  // binning reported the error
  const double delx = del[t], dely = del[cap + t], delz = del[2 * cap + t];
  const int ck = id % g.Nz;
  const int cj = (id / g.Nz) % g.Ny;
  const int ci = id / (g.Nz * g.Ny);
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

}  // namespace

// exclusive scan of n int32 values; out[n] receives the total
int scan_excl(pmpic_ctx* ctx, const int32_t* in, int64_t n, int32_t* out) {
  int64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  int32_t* sums = (int32_t*)ctx->scan_tmp;
  if (ntiles > 0) {
    k_scan_tiles<<<(unsigned)ntiles, SCAN_BLOCK, 0, ctx->stream>>>(in, n, sums); ++ctx->nlaunch;
  }
  k_scan_sums<<<1, SCAN_BLOCK, 0, ctx->stream>>>(sums, ntiles, out + n); ++ctx->nlaunch;
  if (ntiles > 0) {
    k_scan_apply<<<(unsigned)ntiles, SCAN_BLOCK, 0, ctx->stream>>>(in, n, sums, out); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// cache_parcel_interp_weights + the cell-ordered index: valid until positions change
int bin_and_sort(pmpic_ctx* ctx) {
  TimerScope ts(ctx, T_CACHE);
  const Geom& g = ctx->g;
  const int64_t n = ctx->n;
  PMPIC_CUDA(cudaMemsetAsync(ctx->cell_fill, 0, sizeof(int32_t) * g.ncell, ctx->stream));
  // on the mixed form, after an RK4 stage and its haloswap, a split or
  // mixing, the cell ids and counts are current already (kept by the kernels
  // that moved, added or removed parcels)
  const bool counted = ctx->count_ready;
  if (!counted) {
    PMPIC_CUDA(cudaMemsetAsync(ctx->cell_count, 0, sizeof(int32_t) * (g.ncell + 1), ctx->stream));
    if (n > 0 && ctx->mixed) {
      k_bin_count_m<<<nblk(n, 256), 256, 0, ctx->stream>>>(g, n, ctx->cell, curoff(ctx, 0), curoff(ctx, 1),
                                                           curoff(ctx, 2), ctx->cell_count, ctx->dinfo);
      ++ctx->nlaunch;
    } else if (n > 0) {
      k_bin_count<<<nblk(n, 256), 256, 0, ctx->stream>>>(g, n, prop(ctx, PMPIC_PROP_X), prop(ctx, PMPIC_PROP_Y),
                                                         prop(ctx, PMPIC_PROP_Z), ctx->cell, ctx->del, ctx->cap,
                                                         ctx->cell_count, ctx->dinfo, ctx->whint); ++ctx->nlaunch;
    }
  }
  ctx->count_ready = false;
  int rc = scan_excl(ctx, ctx->cell_count, g.ncell, ctx->cell_start);
  if (rc) return rc;
  if (counted) {  // the maintained counts must add up to the parcels
    k_check_total<<<1, 1, 0, ctx->stream>>>(ctx->cell_start + g.ncell, n, ctx->dinfo); ++ctx->nlaunch;
  }
  if (n > 0) {
    k_bin_scatter<<<nblk(n, 256 * SC_ITEMS), 256, 0, ctx->stream>>>(n, ctx->cell, ctx->cell_count, ctx->cell_start,
                                                                    ctx->cell_fill, ctx->sorted, ctx->cap); ++ctx->nlaunch;
    k_sort_segments<<<nblk(g.ncell, SORT_CELLS), SORT_CELLS, 0, ctx->stream>>>(g.ncell, ctx->cell_start,
                                                                               ctx->cell_fill, ctx->sorted);
    ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  ctx->sorted_valid = true;
  return 0;
}

// the two passes of par2grid on `st`; rowpart holds 2 * nzc * Ny * Nx records
// of P2GLayout::RPS / 2 values of type R (the y-low half, then the y-high half)
template <int NQ, int MODE, bool BT, class R = double>
static cudaError_t run_p2g(const Geom& g, const int32_t* start, const int32_t* sorted, const R* dx, const R* dy,
                           const R* dz, int ds, const R* vol, const P2GArgs<NQ, R>& a, R* rowpart, cudaStream_t st,
                           int xseg = XSEG) {
  const int nzc = (g.Nz + ZC - 1) / ZC;
  const int nxs = (g.Nx + xseg - 1) / xseg;
  const int64_t nw = (int64_t)nxs * g.Ny * nzc;
  auto rows = k_p2g_rows<NQ, MODE, BT, R>;
  cudaError_t e = cudaFuncSetAttribute(rows, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  rows<<<nblk(nw, RW), 32 * RW, 0, st>>>(g, nzc, nxs, xseg, start, sorted, dx, dy, dz, ds, vol, a, rowpart);
  dim3 gb((g.Nx + P2GPx<R>::value - 1) / P2GPx<R>::value, g.Ny, nzc);
  k_p2g_combine<NQ, MODE, R><<<gb, 256, 0, st>>>(g, nzc, rowpart, a);
  return cudaGetLastError();
}

template <int NQ, int MODE, bool BT>
static int launch_p2g(pmpic_ctx* ctx, const double* const* fields, double* const* out) {
  TimerScope ts(ctx, T_P2G);
  const Geom& g = ctx->g;
  P2GArgs<NQ> a;
  for (int q = 0; q < NQ; ++q) {
    a.f[q] = fields[q];
    a.out[q] = out[q];
  }
  a.bh[0] = prop(ctx, PMPIC_PROP_B);
  a.bh[1] = prop(ctx, PMPIC_PROP_H);
  a.bh[2] = prop(ctx, PMPIC_PROP_Z);
  a.btot = prop(ctx, PMPIC_PROP_BTOT);
  a.nslot = ctx->n;
  a.npercell = ctx->npercell;
  a.vmin = g.vmin;
  const double* del = ctx->del;
  PMPIC_CUDA((run_p2g<NQ, MODE, BT>(g, ctx->cell_start, ctx->sorted, del, del + ctx->cap, del + 2 * ctx->cap, 1,
                                    prop(ctx, PMPIC_PROP_VOL), a, ctx->rowpart, ctx->stream, ctx->p2g_xseg)));
  ctx->nlaunch += 2;
  return 0;
}

// the mixed form's par2grid: FP32 fields and accumulation, cell offsets read
// from the {cell index, offset} positions
template <int NQ, int MODE, bool BT = false>
static int launch_p2g_m(pmpic_ctx* ctx, const float* const* fields, float* const* out) {
  TimerScope ts(ctx, T_P2G);
  const Geom& g = ctx->g;
  P2GArgs<NQ, float> a{};
  for (int q = 0; q < NQ; ++q) {
    a.f[q] = fields[q];
    a.out[q] = out[q];
  }
  a.bh[0] = propf(ctx, PMPIC_PROP_B);
  a.bh[1] = propf(ctx, PMPIC_PROP_H);
  a.btot = propf(ctx, PMPIC_PROP_BTOT);
  a.nslot = ctx->n;
  a.npercell = ctx->npercell;
  a.vmin = (double)(float)g.vmin;
  // the offsets of the current positions
  PMPIC_CUDA((run_p2g<NQ, MODE, BT, float>(g, ctx->cell_start, ctx->sorted, curoff(ctx, 0), curoff(ctx, 1),
                                              curoff(ctx, 2), 1,
                                              propf(ctx, PMPIC_PROP_VOL), a, (float*)ctx->rowpart, ctx->stream,
                                              ctx->p2g_xseg)));
  ctx->nlaunch += 2;
  return 0;
}

// par2grid of nf FP32 fields on the mixed form (1, 3 or 4 fields); with btot
// the last field is btot computed from b, h, z (and stored as the property)
int par2grid_multi_m(pmpic_ctx* ctx, const float* const* fields, int nf, float* const* out, bool btot) {
  if (btot) {
    switch (nf) {
      case 1: return launch_p2g_m<1, 0, true>(ctx, fields, out);
      case 4: return launch_p2g_m<4, 0, true>(ctx, fields, out);
      default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi_m: btot with 1 or 4 fields");
    }
  }
  switch (nf) {
    case 1: return launch_p2g_m<1, 0>(ctx, fields, out);
    case 3: return launch_p2g_m<3, 0>(ctx, fields, out);
    case 4: return launch_p2g_m<4, 0>(ctx, fields, out);
    default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi_m: 1, 3 or 4 fields");
  }
}

// bytes of the row-partial buffer of a context
size_t rowpart_bytes(const Geom& g) {
  const size_t nzc = (size_t)(g.Nz + ZC - 1) / ZC;
  return sizeof(double) * nzc * (size_t)g.Ny * (size_t)g.Nx * RPS_MAX;
}

// parcel_mixing construct_grids (:440-624) + mixing_haloswap + wall doubling:
// kept grids into VOL, B, HG, P, Q, R (as the reference reuses state%vol,
// state%b, state%hg, state%p, ...), residual grids into mixres, npercell.
// With no parcel in the removed class (any_removed false) its sums are all
// +0.0, which a memset gives without a pass over the parcels, and the kept
// volume grid (and npercell) is made in full, the five other kept grids only
// where mixing reads them (launch_kept_corners).
int launch_mix_grids(pmpic_ctx* ctx, bool any_removed) {
  if (ctx->mixed) {
    const float* f[6] = {nullptr, propf(ctx, PMPIC_PROP_B), propf(ctx, PMPIC_PROP_H),
                         propf(ctx, PMPIC_PROP_P), propf(ctx, PMPIC_PROP_Q), propf(ctx, PMPIC_PROP_R)};
    float* kept[6] = {(float*)ctx->grid[PMPIC_GRID_VOL], (float*)ctx->grid[PMPIC_GRID_B],
                      (float*)ctx->grid[PMPIC_GRID_HG],  (float*)ctx->grid[PMPIC_GRID_P],
                      (float*)ctx->grid[PMPIC_GRID_Q],   (float*)ctx->grid[PMPIC_GRID_R]};
    int rc = any_removed ? launch_p2g_m<6, 1>(ctx, f, kept) : launch_p2g_m<1, 1>(ctx, f, kept);
    if (rc) return rc;
    float* res[6];
    for (int q = 0; q < 6; ++q) res[q] = (float*)ctx->mixres[q];
    if (any_removed) return launch_p2g_m<6, 2>(ctx, f, res);
    for (int q = 0; q < 6; ++q)
      PMPIC_CUDA(cudaMemsetAsync(res[q], 0, sizeof(float) * ctx->g.nphys, ctx->stream));
    return 0;
  }
  const double* f[6] = {nullptr, prop(ctx, PMPIC_PROP_B), prop(ctx, PMPIC_PROP_H),
                        prop(ctx, PMPIC_PROP_P), prop(ctx, PMPIC_PROP_Q), prop(ctx, PMPIC_PROP_R)};
  double* kept[6] = {ctx->grid[PMPIC_GRID_VOL], ctx->grid[PMPIC_GRID_B], ctx->grid[PMPIC_GRID_HG],
                     ctx->grid[PMPIC_GRID_P],   ctx->grid[PMPIC_GRID_Q], ctx->grid[PMPIC_GRID_R]};
  int rc = any_removed ? launch_p2g<6, 1, false>(ctx, f, kept) : launch_p2g<1, 1, false>(ctx, f, kept);
  if (rc) return rc;
  if (any_removed) return launch_p2g<6, 2, false>(ctx, f, ctx->mixres);
  for (int q = 0; q < 6; ++q)
    PMPIC_CUDA(cudaMemsetAsync(ctx->mixres[q], 0, sizeof(double) * ctx->g.nphys, ctx->stream));
  return 0;
}

// The kept grids B, HG, P, Q, R at the eight corners of the nnew cells in
// olist (mixed form, a mixing call without removed parcels; hnew the count,
// read back).  Requires bin_and_sort of the parcels before mixing.
int launch_kept_corners(pmpic_ctx* ctx, const int32_t* olist, const int32_t* nnew, int64_t hnew) {
  if (hnew <= 0) return 0;
  const int pf[5] = {PMPIC_PROP_B, PMPIC_PROP_H, PMPIC_PROP_P, PMPIC_PROP_Q, PMPIC_PROP_R};
  const int pg[5] = {PMPIC_GRID_B, PMPIC_GRID_HG, PMPIC_GRID_P, PMPIC_GRID_Q, PMPIC_GRID_R};
  if (ctx->mixed) {
    KeptCorners<float> k;
    for (int q = 0; q < 5; ++q) {
      k.f[q] = propf(ctx, pf[q]);
      k.out[q] = (float*)ctx->grid[pg[q]];
    }
    k.vmin = (double)(float)ctx->g.vmin;
    k_kept_corners<float><<<(unsigned)hnew, 256, 0, ctx->stream>>>(ctx->g, olist, nnew, ctx->cell_start, ctx->sorted,
                                                                  curoff(ctx, 0), curoff(ctx, 1), curoff(ctx, 2),
                                                                  propf(ctx, PMPIC_PROP_VOL), k);
  } else {
    KeptCorners<double> k;
    for (int q = 0; q < 5; ++q) {
      k.f[q] = prop(ctx, pf[q]);
      k.out[q] = ctx->grid[pg[q]];
    }
    k.vmin = ctx->g.vmin;
    const double* del = ctx->del;  // the binning made at the start of mixing
    k_kept_corners<double><<<(unsigned)hnew, 256, 0, ctx->stream>>>(ctx->g, olist, nnew, ctx->cell_start, ctx->sorted,
                                                                   del, del + ctx->cap, del + 2 * ctx->cap,
                                                                   prop(ctx, PMPIC_PROP_VOL), k);
  }
  ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// par2grid of nf fields with the same weights; with btot the last field is
// btot computed from b, h, z.  Requires bin_and_sort.
int par2grid_multi(pmpic_ctx* ctx, const double* const* fields, int nf, double* const* out, bool btot) {
  if (btot) {
    switch (nf) {
      case 1: return launch_p2g<1, 0, true>(ctx, fields, out);
      case 4: return launch_p2g<4, 0, true>(ctx, fields, out);
      default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi: btot with 1 or 4 fields");
    }
  }
  switch (nf) {
    case 1: return launch_p2g<1, 0, false>(ctx, fields, out);
    case 3: return launch_p2g<3, 0, false>(ctx, fields, out);
    case 4: return launch_p2g<4, 0, false>(ctx, fields, out);
    default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi: 1, 3 or 4 fields");
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
  k_grid2par<NG><<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(g, ctx->n, ctx->cell, ctx->del, ctx->cap, a);
  ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// grid2par of NG FP32 grids at the mixed form's current positions (cell id + offsets)
template <int NG>
__global__ void k_grid2par_mt(Geom g, int64_t n, const int32_t* __restrict__ cell, const float* __restrict__ FX,
                              const float* __restrict__ FY, const float* __restrict__ FZ, G2PArgs<NG> a,
                              DevInfo* info) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int32_t id = cell[t];
  if (id < 0 || id >= g.ncell) {  // not a cell of the grid: nothing read
    atomicCAS(&info->error, 0, PMPIC_ERR_OUT_OF_BOX);
    return;
  }
  int ci, cj, ck;
  cell_decode(g, id, ci, cj, ck);
  const int ci1 = ci + 1 == g.Nx ? 0 : ci + 1, cj1 = cj + 1 == g.Ny ? 0 : cj + 1;
  const size_t r00 = ((size_t)ck * g.Ny + cj) * g.Nx, r01 = ((size_t)ck * g.Ny + cj1) * g.Nx;
  const size_t r10 = ((size_t)(ck + 1) * g.Ny + cj) * g.Nx, r11 = ((size_t)(ck + 1) * g.Ny + cj1) * g.Nx;
  const float delx = FX[t], dely = FY[t], delz = FZ[t];
#pragma unroll
  for (int q = 0; q < NG; ++q) {
    const float* G = (const float*)a.grid[q];
    const float c00 = G[r00 + ci] * (1.f - delz) + G[r10 + ci] * delz;
    const float c01 = G[r00 + ci1] * (1.f - delz) + G[r10 + ci1] * delz;
    const float c10 = G[r01 + ci] * (1.f - delz) + G[r11 + ci] * delz;
    const float c11 = G[r01 + ci1] * (1.f - delz) + G[r11 + ci1] * delz;
    const float c0 = c00 * (1.f - dely) + c10 * dely;
    const float c1 = c01 * (1.f - dely) + c11 * dely;
    ((float*)a.out[q])[t] = c0 * (1.f - delx) + c1 * delx;
  }
}

// the mixed form's grid2par of ng FP32 grids into FP32 properties (1, 3 or 6)
int grid2par_multi_m(pmpic_ctx* ctx, const float* const* grids, int ng, float* const* out) {
  TimerScope ts(ctx, T_G2P);
  if (ctx->n == 0) return 0;
  auto run = [&](auto tag) {
    constexpr int NG = decltype(tag)::value;
    G2PArgs<NG> a;
    for (int q = 0; q < NG; ++q) {
      a.grid[q] = (const double*)grids[q];
      a.out[q] = (double*)out[q];
    }
    k_grid2par_mt<NG><<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, ctx->cell, curoff(ctx, 0),
                                                                   curoff(ctx, 1), curoff(ctx, 2), a, ctx->dinfo);
    ++ctx->nlaunch;
  };
  switch (ng) {
    case 1: run(std::integral_constant<int, 1>{}); break;
    case 3: run(std::integral_constant<int, 3>{}); break;
    case 6: run(std::integral_constant<int, 6>{}); break;
    default: return set_error(ctx, PMPIC_ERR_ARG, "grid2par_multi_m: 1, 3 or 6 grids");
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// grid2par of ng grids; requires the cached binning of the current positions
int grid2par_multi(pmpic_ctx* ctx, const double* const* grids, int ng, double* const* out) {
  if (!ctx->sorted_valid) {
    int rc = bin_and_sort(ctx);
    if (rc) return rc;
  }
  switch (ng) {
    case 1: return launch_g2p<1>(ctx, grids, out);
    case 3: return launch_g2p<3>(ctx, grids, out);
    case 6: return launch_g2p<6>(ctx, grids, out);
    default: return set_error(ctx, PMPIC_ERR_ARG, "grid2par_multi: 1, 3 or 6 grids");
  }
}

// cell ids of the current positions in the x-fastest form of the C ABI,
// ((k-1)*ny + (j-3))*nx + (i-3), into dcells (device, n entries)
int cell_ids(pmpic_ctx* ctx, int32_t* dcells) {
  int rc = bin_and_sort(ctx);
  if (rc) return rc;
  if (ctx->n > 0) {
    k_cell_xfast<<<nblk(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->n, ctx->cell, dcells); ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace pmpic

// ---- par2grid without allocation -------------------------------------------------------
// pmpic_par2grid_static: the same binning, CSR sort and par2grid reduction as
// pmpic_op_par2grid, for callers that hold no context and may not allocate
// device memory when they call: a host whose device memory is handed in full
// to its own pool allocator, or a component callback that must keep the
// device footprint fixed between steps.  Its scratch lives in one file-scope
// device array of fixed size, so a call allocates nothing; the per-device
// address of that array is looked up once, on the first call made with that
// device current.
namespace pmpic {
namespace {

constexpr int64_t SP_MAX_PARCELS = 131072;  // parcels per call
constexpr int64_t SP_MAX_CELLS = 32768;     // nx*ny*nz per call
constexpr int64_t SP_MAX_COLCHUNKS = 4096;  // ceil(nz/16)*nx*ny per call (row partials of par2grid)
constexpr int64_t SP_MAX_TILES = (SP_MAX_CELLS + SCAN_TILE - 1) / SCAN_TILE + 1;
constexpr size_t sp_round(size_t b) { return (b + 255) / 256 * 256; }
// scratch layout (byte offsets)
constexpr size_t SP_DEL = 0;                                                         // double[3][MAX_PARCELS]
constexpr size_t SP_SORTED = SP_DEL + sp_round(sizeof(double) * 3 * SP_MAX_PARCELS);  // int32[MAX_PARCELS]
constexpr size_t SP_CELL = SP_SORTED + sp_round(sizeof(int32_t) * SP_MAX_PARCELS);    // int32[MAX_PARCELS]
constexpr size_t SP_COUNT = SP_CELL + sp_round(sizeof(int32_t) * SP_MAX_PARCELS);     // int32[MAX_CELLS+1]
constexpr size_t SP_START = SP_COUNT + sp_round(sizeof(int32_t) * (SP_MAX_CELLS + 1));  // int32[MAX_CELLS+1]
constexpr size_t SP_FILL = SP_START + sp_round(sizeof(int32_t) * (SP_MAX_CELLS + 1));   // int32[MAX_CELLS]
constexpr size_t SP_TILES = SP_FILL + sp_round(sizeof(int32_t) * SP_MAX_CELLS);         // int32[MAX_TILES]
constexpr size_t SP_INFO = SP_TILES + sp_round(sizeof(int32_t) * SP_MAX_TILES);         // DevInfo
constexpr size_t SP_ROWS = SP_INFO + sp_round(sizeof(DevInfo));                         // double[MAX_COLCHUNKS][RPS]
constexpr size_t SP_BYTES = SP_ROWS + sp_round(sizeof(double) * SP_MAX_COLCHUNKS * P2GLayout<1, 0, false>::RPS);
static_assert(SP_BYTES < 8u << 20, "static par2grid scratch stays below 8 MB");

__device__ __align__(256) unsigned char g_p2g_scratch[SP_BYTES];

constexpr int SP_MAX_DEVICES = 64;
std::mutex sp_mutex;
void* sp_addr[SP_MAX_DEVICES] = {};

}  // namespace
}  // namespace pmpic

extern "C" int pmpic_par2grid_static(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                                     int64_t n, const double* x, const double* y, const double* z,
                                     const double* vol, const double* field, double* out, void* stream) {
  using namespace pmpic;
  // the smallest box pmpic_create accepts (and the oracle restates)
  if (nx < 4 || ny < 4 || nz < 3 || !(lx > 0) || !(ly > 0) || !(lz > 0) || n < 0 || !out) return PMPIC_ERR_ARG;
  if (n > 0 && (!x || !y || !z || !vol || !field)) return PMPIC_ERR_ARG;
  const int64_t ncell = (int64_t)nx * ny * nz;
  if (n > SP_MAX_PARCELS || ncell > SP_MAX_CELLS) return PMPIC_ERR_TOO_LARGE;
  if ((int64_t)((nz + ZC - 1) / ZC) * nx * ny > SP_MAX_COLCHUNKS) return PMPIC_ERR_TOO_LARGE;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SP_MAX_DEVICES) return PMPIC_ERR_CUDA;
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lk(sp_mutex);
    if (!sp_addr[dev]) {  // set-up, once per device: the array's address on this device
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_p2g_scratch) != cudaSuccess || !p) return PMPIC_ERR_CUDA;
      sp_addr[dev] = p;
    }
    base = (unsigned char*)sp_addr[dev];
  }
  double* del = (double*)(base + SP_DEL);
  int32_t* sorted = (int32_t*)(base + SP_SORTED);
  int32_t* cell = (int32_t*)(base + SP_CELL);
  int32_t* count = (int32_t*)(base + SP_COUNT);
  int32_t* cstart = (int32_t*)(base + SP_START);
  int32_t* fill = (int32_t*)(base + SP_FILL);
  int32_t* tiles = (int32_t*)(base + SP_TILES);
  DevInfo* info = (DevInfo*)(base + SP_INFO);
  double* rows = (double*)(base + SP_ROWS);
  cudaStream_t st = (cudaStream_t)stream;

  // geometry: the binning and par2grid subset of pmpic_create's (origin 0)
  Geom g{};
  g.Nx = nx; g.Ny = ny; g.Nz = nz; g.nzp = nz + 1;
  g.sx = nx + 2; g.sy = ny + 2;
  g.ncell = ncell;
  g.nphys = (int64_t)g.nzp * ny * nx;
  g.nspec = (int64_t)g.nzp * g.sy * g.sx;
  g.dx = lx / (double)nx;
  g.dy = ly / (double)ny;
  g.dz = lz / (double)nz;
  g.pxmin = (double)(-2) * g.dx;
  g.pymin = (double)(-2) * g.dy;
  g.pzmin = 0.0;
  g.pzmax = (double)nz * g.dz;

  // the counters and the error word must start at zero: cleared on every call
  if (cudaMemsetAsync(count, 0, sizeof(int32_t) * (ncell + 1), st) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (cudaMemsetAsync(fill, 0, sizeof(int32_t) * ncell, st) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (cudaMemsetAsync(info, 0, sizeof(DevInfo), st) != cudaSuccess) return PMPIC_ERR_CUDA;
  if (n > 0)
    k_bin_count<<<nblk(n, 256), 256, 0, st>>>(g, n, x, y, z, cell, del, SP_MAX_PARCELS, count, info);
  const int64_t ntiles = (ncell + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tiles<<<(unsigned)ntiles, SCAN_BLOCK, 0, st>>>(count, ncell, tiles);
  k_scan_sums<<<1, SCAN_BLOCK, 0, st>>>(tiles, ntiles, cstart + ncell);
  k_scan_apply<<<(unsigned)ntiles, SCAN_BLOCK, 0, st>>>(count, ncell, tiles, cstart);
  if (n > 0) {
    k_bin_scatter<<<nblk(n, 256 * SC_ITEMS), 256, 0, st>>>(n, cell, count, cstart, fill, sorted, SP_MAX_PARCELS);
    k_sort_segments<<<nblk(ncell, SORT_CELLS), SORT_CELLS, 0, st>>>(ncell, cstart, fill, sorted);
  }
  P2GArgs<1> a{};
  a.f[0] = field;
  a.out[0] = out;
  a.nslot = n;
  if (run_p2g<1, 0, false>(g, cstart, sorted, del, del + SP_MAX_PARCELS, del + 2 * SP_MAX_PARCELS, 1, vol, a, rows,
                           st) != cudaSuccess)
    return PMPIC_ERR_CUDA;
  int err = 0;
  if (cudaMemcpyAsync(&err, &info->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PMPIC_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return PMPIC_ERR_CUDA;
  return err;
}
