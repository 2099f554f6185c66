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
// grid2par and the mixing redistribution.
//
// par2grid is deterministic and uses no floating-point atomics:
//   1. bin:     cell ids + cached offsets + an integer histogram per cell;
//   2. scan:    exclusive scan of the histogram -> CSR offsets per cell;
//   3. scatter: slot indices into cell order, then each cell segment sorted
//               by slot index, so every later sum runs in slot order;
//   4. reduce:  one CTA per 16x8 column tile and 16 grid levels walks the
//               cell layers upwards.  A producer warp streams each layer's
//               parcels (17x9 cells incl. the low periodic halo) into a ring of
//               shared-memory buffers with cp.async gathers, handing them over
//               through mbarriers; one consumer thread per cell accumulates its
//               parcels' eight corner weights in slot order, and the cells add
//               them into the level accumulators in four parity phases (cells
//               of one parity class touch disjoint grid points), so every grid
//               point sums its contributions in one fixed order.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace pmpic {

namespace {

constexpr int TX = 16;                // owned grid points per tile in x
constexpr int TY = 8;                 // ... in y
constexpr int CX = TX + 1;            // cells per tile row incl. the low halo cell
constexpr int CY = TY + 1;
constexpr int NCELLT = CX * CY;       // 153 cells per tile layer
constexpr int P2G_CONS = 160;         // consumer threads (>= NCELLT), one per cell
constexpr int P2G_THREADS = P2G_CONS + 32;  // + one producer warp
constexpr int ZCHUNK = 16;            // grid levels per CTA
constexpr int RANKS = 2;              // in-cell ranks per staged slice
constexpr int NBUF = 4;               // staging buffers in the ring
constexpr int NTAB = 4;               // layer tables in the ring
constexpr int MAXSEG = 32;            // cell segments sorted in registers

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- binning (cache_parcel_interp_weights, parcel_interpolation.F90:186-262) ----
__global__ void k_bin_count(Geom g, int64_t n, const double* __restrict__ X, const double* __restrict__ Y,
                            const double* __restrict__ Z, int32_t* __restrict__ cell, double* __restrict__ del,
                            int64_t cap, int32_t* __restrict__ count, DevInfo* info) {
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
  del[t] = dx;
  del[cap + t] = dy;
  del[2 * cap + t] = dz;
  // neighbouring slots mostly share a cell: one atomic per distinct cell of the warp
  const unsigned act = __activemask();
  const unsigned same = __match_any_sync(act, id);
  if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&count[id], __popc(same));
}

__global__ void k_bin_scatter(int64_t n, const int32_t* __restrict__ cell, const int32_t* __restrict__ start,
                              int32_t* __restrict__ fill, int32_t* __restrict__ sorted) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int32_t id = cell[t];
  if (id < 0) return;
  // one atomic per distinct cell of the warp; lanes take consecutive places in
  // lane order (the segment is sorted by slot afterwards in any case)
  const unsigned act = __activemask();
  const unsigned same = __match_any_sync(act, id);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(same) - 1;
  int32_t base = 0;
  if (lane == leader) base = atomicAdd(&fill[id], __popc(same));
  base = __shfl_sync(same, base, leader);
  const int32_t pos = start[id] + base + __popc(same & ((1u << lane) - 1));
  sorted[pos] = (int32_t)t;
}

// each cell's segment sorted by slot index (integer atomics above only decide
// the order inside a cell)
__global__ void k_sort_segments(int64_t ncell, const int32_t* __restrict__ start, int32_t* __restrict__ sorted) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int s0 = start[c], len = start[c + 1] - s0;
  if (len < 2) return;
  int32_t* s = sorted + s0;
  if (len <= MAXSEG) {
    int loc[MAXSEG];
    for (int u = 0; u < len; ++u) {
      int v = s[u];
      int w = u - 1;
      while (w >= 0 && loc[w] > v) {
        loc[w + 1] = loc[w];
        --w;
      }
      loc[w + 1] = v;
    }
    for (int u = 0; u < len; ++u) s[u] = loc[u];
  } else {  // rare long segment: insertion sort in place
    for (int u = 1; u < len; ++u) {
      int v = s[u];
      int w = u - 1;
      while (w >= 0 && s[w] > v) {
        s[w + 1] = s[w];
        --w;
      }
      s[w + 1] = v;
    }
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
template <int NQ>
struct P2GArgs {
  const double* f[NQ];  // per-parcel fields (MODE 1/2: f[0] unused)
  double* out[NQ];
  const double* bh[3];  // b, h, z for btot
  int32_t* npercell;
  double vmin;
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <int NQ, int MODE, bool BT>
struct P2GLayout {
  static constexpr int NA = MODE == 0 ? NQ + 1 : NQ;        // accumulated quantities
  static constexpr int NF = MODE == 0 ? (BT ? NQ + 2 : NQ)  // staged per-parcel values
                                      : NQ - 1;             //   (MODE 1/2: b,h,p,q,r)
  static constexpr int NS = 4 + NF;                         // + delx, dely, delz, vol
  static constexpr int FS = RANKS * NCELLT;                 // stride between staged fields
  static constexpr size_t stage_elems = (size_t)NS * FS;    // one staging buffer
  static constexpr size_t stage_bytes = sizeof(double) * NBUF * stage_elems;
  static constexpr size_t acc_bytes = sizeof(double) * 2 * NCELLT * NA;  // two grid levels
  static constexpr size_t tab_bytes = sizeof(int) * (2 * NTAB * NCELLT + NTAB);
  static constexpr size_t bar_bytes = sizeof(uint64_t) * (2 * NBUF + NTAB) + 16;
  static constexpr size_t smem = stage_bytes + acc_bytes + tab_bytes + bar_bytes;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// arrives on b once every cp.async this thread issued before has landed
__device__ __forceinline__ void mbar_arrive_on_copies(uint64_t* b) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ull;  // 4 s: a chunk lands in microseconds
// Wait for the phase of parity `parity` of b to complete.  Gives up after
// WAIT_LIMIT_NS, or at once when *abort is set; returns false then, with *abort set.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, int parity, volatile int* abort) {
  const uint32_t a = smem_u32(b);
  unsigned long long t0 = 0;
  for (int it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 31) == 31) {
      if (*abort) return false;
      const unsigned long long now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > WAIT_LIMIT_NS) {
        *abort = 1;
        return false;
      }
    }
  }
}
__device__ __forceinline__ void cons_sync() {  // the consumer warps only
  asm volatile("bar.sync 1, %0;" ::"n"(P2G_CONS) : "memory");
}
// consumer barrier that also returns the OR of `pred` over the consumer threads
__device__ __forceinline__ bool cons_sync_or(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "n"(P2G_CONS)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One CTA per TX x TY column tile and ZCHUNK grid levels walks the cell layers
// upwards.  One producer warp streams the tile's parcels into a ring of NBUF
// shared-memory buffers; five consumer warps reduce them, one thread per cell.
//  - The chunk sequence is (layer, slice) in order: slice s of a layer holds,
//    for every cell of the tile, its parcels of in-cell rank 2s, 2s+1
//    (segments are sorted by slot, so rank order is slot order).  An empty
//    layer still takes one (empty) slice.
//  - Producer: per layer it loads the cells' CSR segments (start values one
//    layer ahead, in registers) into a ring of NTAB tables and releases each
//    table through an mbarrier; per chunk it waits until the consumers have
//    freed the buffer, issues 8-byte cp.async gathers (slot indices loaded one
//    chunk ahead, in registers) and arms the buffer's mbarrier to complete
//    when its copies have landed.  It runs up to NBUF-1 chunks ahead.
//  - Consumers: each thread accumulates its cell's eight corner weights in
//    slot order in registers; after a layer's last chunk the cells add their
//    corners into two shared level accumulators in four parity phases (cells
//    of one parity class touch disjoint points), so each grid point sums its
//    contributions in one fixed order independent of timing.
//  Every mbarrier wait is bounded: a wait that runs out sets PMPIC_ERR_TIMEOUT
//  and the CTA stops after its copies in flight have landed.
template <int NQ, int MODE, bool BT>
__global__ void __launch_bounds__(P2G_THREADS, 2)
    k_par2grid(Geom g, const int32_t* __restrict__ start, const int32_t* __restrict__ sorted,
               const double* __restrict__ del, int64_t cap, const double* __restrict__ VOL, P2GArgs<NQ> a,
               DevInfo* info) {
  using Lay = P2GLayout<NQ, MODE, BT>;
  constexpr int NA = Lay::NA, FS = Lay::FS;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* stage = (double*)smraw;                              // [NBUF][NS][RANKS][NCELLT]
  double* acc = stage + NBUF * Lay::stage_elems;               // [2 levels][NA][NCELLT points]
  int* tab_s0 = (int*)(acc + 2 * NCELLT * NA);                 // [NTAB][NCELLT]
  int* tab_len = tab_s0 + NTAB * NCELLT;                       // [NTAB][NCELLT]
  int* tab_ns = tab_len + NTAB * NCELLT;                       // [NTAB] slices of the layer
  uint64_t* bars = (uint64_t*)(((uintptr_t)(tab_ns + NTAB) + 7) & ~(uintptr_t)7);
  uint64_t* full = bars;                                       // [NBUF] copies landed
  uint64_t* empty = bars + NBUF;                               // [NBUF] consumers done
  uint64_t* tabfull = bars + 2 * NBUF;                         // [NTAB] table written
  volatile int* abort = (volatile int*)(bars + 2 * NBUF + NTAB);
  const int t = threadIdx.x;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int L0 = blockIdx.z * ZCHUNK;
  const int LAST = min(L0 + ZCHUNK, g.nzp) - 1;  // last cell layer walked
  for (int e = t; e < 2 * NCELLT * NA; e += P2G_THREADS) acc[e] = 0.0;
  if (t == 0) {
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(&full[b], 32);
      mbar_init(&empty[b], P2G_CONS);
    }
    for (int s = 0; s < NTAB; ++s) mbar_init(&tabfull[s], 32);
    *abort = 0;
  }
  __syncthreads();

  if (t >= P2G_CONS) {
    // ================================ producer warp ================================
    const int lane = t - P2G_CONS;
    const double* DX = del;
    const double* DY = del + cap;
    const double* DZ = del + 2 * cap;
    constexpr int CPL = (NCELLT + 31) / 32;  // table cells per lane
    auto fetch = [&](int ck, int* s0, int* len) {
#pragma unroll
      for (int i = 0; i < CPL; ++i) {
        const int c = lane + 32 * i;
        s0[i] = 0;
        len[i] = 0;
        if (c < NCELLT && ck >= 0 && ck < g.Nz) {
          const int tx = c % CX, ty = c / CX;
          int ci = x0 - 1 + tx, cj = y0 - 1 + ty;
          if ((tx > 0 && ci >= g.Nx) || (ty > 0 && cj >= g.Ny)) continue;
          if (ci < 0) ci += g.Nx;  // low halo cell: periodic wrap (MPIC_Haloswap.F90)
          if (cj < 0) cj += g.Ny;
          const int64_t cid = ((int64_t)ck * g.Ny + cj) * g.Nx + ci;
          s0[i] = start[cid];
          len[i] = start[cid + 1] - s0[i];
        }
      }
    };
    int ns0[CPL], nlen[CPL];  // segments of the next layer, in flight
    fetch(L0 - 1, ns0, nlen);
    constexpr int PPL = (NCELLT * RANKS + 31) / 32;  // (cell, rank) pairs per lane
    int nid[PPL];
    auto load_idx = [&](int slot, int s) {
#pragma unroll
      for (int i = 0; i < PPL; ++i) {
        const int pr = lane + 32 * i;
        nid[i] = -1;
        if (pr < NCELLT * RANKS) {
          const int c = pr / RANKS, u = s * RANKS + pr % RANKS;
          if (u < tab_len[slot * NCELLT + c]) nid[i] = sorted[tab_s0[slot * NCELLT + c] + u];
        }
      }
    };
    int k = 0;  // chunk counter
    bool ok = true;
    for (int ck = L0 - 1; ck <= LAST && ok; ++ck) {
      const int li = ck - (L0 - 1), slot = li % NTAB;
      int ns = 1;
      for (int s = 0; s < ns && ok; ++s, ++k) {
        const int b = k % NBUF;
        if (k >= NBUF && !mbar_wait(&empty[b], ((k / NBUF) - 1) & 1, abort)) {
          ok = false;
          break;
        }
        if (s == 0) {
          // this layer's table: its slot was last read for layer ck - NTAB, whose
          // chunks the consumers finished before freeing buffer b
          int m = 0;
#pragma unroll
          for (int i = 0; i < CPL; ++i) {
            const int c = lane + 32 * i;
            if (c < NCELLT) {
              tab_s0[slot * NCELLT + c] = ns0[i];
              tab_len[slot * NCELLT + c] = nlen[i];
            }
            m = max(m, nlen[i]);
          }
          m = __reduce_max_sync(0xffffffffu, m);
          ns = max(1, (m + RANKS - 1) / RANKS);
          if (lane == 0) tab_ns[slot] = ns;
          __syncwarp();
          mbar_arrive(&tabfull[slot]);
          if (ck + 1 <= LAST) fetch(ck + 1, ns0, nlen);
          load_idx(slot, 0);
        }
        double* S = stage + (size_t)b * Lay::stage_elems;
#pragma unroll
        for (int i = 0; i < PPL; ++i) {
          const int n = nid[i];
          if (n < 0) continue;
          const int pr = lane + 32 * i;
          double* D = S + (pr % RANKS) * NCELLT + pr / RANKS;
          cp_async8(D, DX + n);
          cp_async8(D + FS, DY + n);
          cp_async8(D + 2 * FS, DZ + n);
          cp_async8(D + 3 * FS, VOL + n);
          if (MODE == 0) {
#pragma unroll
            for (int qq = 0; qq < (BT ? NQ - 1 : NQ); ++qq) cp_async8(D + (4 + qq) * FS, a.f[qq] + n);
            if (BT) {
#pragma unroll
              for (int qq = 0; qq < 3; ++qq) cp_async8(D + (4 + NQ - 1 + qq) * FS, a.bh[qq] + n);
            }
          } else {
#pragma unroll
            for (int qq = 1; qq < NQ; ++qq) cp_async8(D + (4 + qq - 1) * FS, a.f[qq] + n);
          }
        }
        mbar_arrive_on_copies(&full[b]);
        if (s + 1 < ns) load_idx(slot, s + 1);  // the next chunk's indices, one chunk ahead
      }
    }
    if (!ok) atomicCAS(&info->error, 0, PMPIC_ERR_TIMEOUT);
    cp_async_wait_all();  // every copy has landed before the warp leaves
    return;
  }

  // ================================ consumer warps ================================
  const int c = t;  // this thread's cell (c < NCELLT)
  const int tx = c % CX, ty = c / CX;
  bool has_col = c < NCELLT;
  int ci = x0 - 1 + tx, cj = y0 - 1 + ty;
  if (has_col) {
    if (tx > 0 && ci >= g.Nx) has_col = false;
    if (ty > 0 && cj >= g.Ny) has_col = false;
    if (ci < 0) ci += g.Nx;
    if (cj < 0) cj += g.Ny;
  }
  const int parity = (tx & 1) | ((ty & 1) << 1);
  int cur = 0;  // level accumulator of the current layer's bottom corners
  int k = 0;
  bool ok = true;
  for (int ck = L0 - 1; ck <= LAST; ++ck) {
    const int li = ck - (L0 - 1), slot = li % NTAB;
    ok = ok && mbar_wait(&tabfull[slot], (li / NTAB) & 1, abort);
    const int ns = ok ? tab_ns[slot] : 0;
    const int mylen = (ok && c < NCELLT) ? tab_len[slot * NCELLT + c] : 0;
    double P[8][NA];
#pragma unroll
    for (int cc = 0; cc < 8; ++cc)
#pragma unroll
      for (int qq = 0; qq < NA; ++qq) P[cc][qq] = 0.0;
    int nkept = 0;
    for (int s = 0; s < ns && ok; ++s, ++k) {
      const int b = k % NBUF;
      if (!mbar_wait(&full[b], (k / NBUF) & 1, abort)) {
        ok = false;
        break;
      }
      const int nu = min(RANKS, mylen - s * RANKS);
      const double* S0 = stage + (size_t)b * Lay::stage_elems + c;
#pragma unroll
      for (int ul = 0; ul < RANKS; ++ul) {
        if (ul >= nu) break;
        const double* S = S0 + ul * NCELLT;
        const double delx = S[0], dely = S[FS], delz = S[2 * FS], vv = S[3 * FS];
        if (MODE == 1 && vv < a.vmin) continue;    // parcel_mixing.F90:488
        if (MODE == 2 && !(vv < a.vmin)) continue;
        if (MODE == 1) ++nkept;
        // parcel_interpolation.F90:390-434: w = (1-delz)(1-dely)(1-delx) v etc.
        const double ez = 1 - delz, ey = 1 - dely, ex = 1 - delx;
        double w[8];
        w[0] = ez * ey * ex * vv;
        w[1] = ez * ey * delx * vv;
        w[2] = ez * dely * ex * vv;
        w[3] = ez * dely * delx * vv;
        w[4] = delz * ey * ex * vv;
        w[5] = delz * ey * delx * vv;
        w[6] = delz * dely * ex * vv;
        w[7] = delz * dely * delx * vv;
        double fv[NQ];
        if (MODE == 0) {
#pragma unroll
          for (int qq = 0; qq < (BT ? NQ - 1 : NQ); ++qq) fv[qq] = S[(4 + qq) * FS];
          if (BT) {
            const double bb = S[(4 + NQ - 1) * FS], hh = S[(4 + NQ) * FS], zz = S[(4 + NQ + 1) * FS];
            fv[NQ - 1] = bb + 12.5 * fmax(0.0, hh - exp(-zz));  // vorticity_tendency.F90:123-124
          }
        } else {
          fv[0] = 1.0;
#pragma unroll
          for (int qq = 1; qq < NQ; ++qq) fv[qq] = S[(4 + qq - 1) * FS];
        }
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
#pragma unroll
          for (int qq = 0; qq < NQ; ++qq) P[cc][qq] += (MODE != 0 && qq == 0) ? w[cc] : w[cc] * fv[qq];
          if (MODE == 0) P[cc][NA - 1] += w[cc];
        }
      }
      mbar_arrive(&empty[b]);  // this thread's reads of buffer b are done
    }
    // uniform stop: the OR over all consumers of "a wait gave up"
    if (cons_sync_or(!ok || *abort)) break;
    if (MODE == 1 && has_col && ck >= L0 && ck < g.Nz && tx > 0 && ty > 0)
      a.npercell[((int64_t)ck * g.Ny + cj) * g.Nx + ci] = nkept;
    // corners into the level accumulators, one parity class at a time;
    // corner cc: dz = cc>>2, dy = (cc>>1)&1, dx = cc&1
    for (int ph = 0; ph < 4; ++ph) {
      if (ph) cons_sync();
      if (has_col && parity == ph) {
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int px = tx + (cc & 1), py = ty + ((cc >> 1) & 1);
          if (px < CX && py < CY) {
            double* A = acc + (size_t)(cur ^ (cc >> 2)) * NA * NCELLT + py * CX + px;
#pragma unroll
            for (int qq = 0; qq < NA; ++qq) A[qq * NCELLT] += P[cc][qq];
          }
        }
      }
    }
    cons_sync();
    // level ck is complete: normalise and store the owned points, clear the level
    for (int e = t; e < NCELLT; e += P2G_CONS) {
      double* A = acc + (size_t)cur * NA * NCELLT + e;
      const int px = e % CX, py = e / CX;
      const int gx = x0 + px - 1, gy = y0 + py - 1;
      if (ck >= L0 && px > 0 && py > 0 && gx < g.Nx && gy < g.Ny) {
        const size_t o = ((size_t)ck * g.Ny + gy) * g.Nx + gx;
        if (MODE == 0) {
          double wv = A[(NA - 1) * NCELLT];
          if (wv == 0.) wv = 1.;  // parcel_interpolation.F90:466
#pragma unroll
          for (int qq = 0; qq < NQ; ++qq) a.out[qq][o] = A[qq * NCELLT] / wv;  // :467
        } else {
          const bool wall = (MODE == 1) && (ck == 0 || ck == g.Nz);
#pragma unroll
          for (int qq = 0; qq < NQ; ++qq) a.out[qq][o] = wall ? A[qq * NCELLT] * 2. : A[qq * NCELLT];
        }
      }
#pragma unroll
      for (int qq = 0; qq < NA; ++qq) A[qq * NCELLT] = 0.0;
    }
    cur ^= 1;
    cons_sync();
  }
  if (t == 0 && *abort) atomicCAS(&info->error, 0, PMPIC_ERR_TIMEOUT);
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
  const int ci = id % g.Nx;
  const int cj = (id / g.Nx) % g.Ny;
  const int ck = id / (g.Nx * g.Ny);
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
  PMPIC_CUDA(cudaMemsetAsync(ctx->cell_count, 0, sizeof(int32_t) * (g.ncell + 1), ctx->stream));
  PMPIC_CUDA(cudaMemsetAsync(ctx->cell_fill, 0, sizeof(int32_t) * g.ncell, ctx->stream));
  if (n > 0) {
    k_bin_count<<<nblk(n, 256), 256, 0, ctx->stream>>>(g, n, prop(ctx, PMPIC_PROP_X), prop(ctx, PMPIC_PROP_Y),
                                                       prop(ctx, PMPIC_PROP_Z), ctx->cell, ctx->del, ctx->cap,
                                                       ctx->cell_count, ctx->dinfo); ++ctx->nlaunch;
  }
  int rc = scan_excl(ctx, ctx->cell_count, g.ncell, ctx->cell_start);
  if (rc) return rc;
  if (n > 0) {
    k_bin_scatter<<<nblk(n, 256), 256, 0, ctx->stream>>>(n, ctx->cell, ctx->cell_start, ctx->cell_fill,
                                                         ctx->sorted); ++ctx->nlaunch;
    k_sort_segments<<<nblk(g.ncell, 256), 256, 0, ctx->stream>>>(g.ncell, ctx->cell_start, ctx->sorted);
    ++ctx->nlaunch;
  }
  PMPIC_CUDA(cudaGetLastError());
  ctx->sorted_valid = true;
  return 0;
}

template <int NQ, int MODE, bool BT>
static int launch_p2g(pmpic_ctx* ctx, const double* const* fields, double* const* out) {
  TimerScope ts(ctx, T_P2G);
  const Geom& g = ctx->g;
  using Lay = P2GLayout<NQ, MODE, BT>;
  static_assert(Lay::smem <= 227 * 1024, "par2grid shared memory");
  P2GArgs<NQ> a;
  for (int q = 0; q < NQ; ++q) {
    a.f[q] = fields[q];
    a.out[q] = out[q];
  }
  a.bh[0] = prop(ctx, PMPIC_PROP_B);
  a.bh[1] = prop(ctx, PMPIC_PROP_H);
  a.bh[2] = prop(ctx, PMPIC_PROP_Z);
  a.npercell = ctx->npercell;
  a.vmin = g.vmin;
  auto kern = k_par2grid<NQ, MODE, BT>;
  PMPIC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::smem));
  PMPIC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
  dim3 grid((g.Nx + TX - 1) / TX, (g.Ny + TY - 1) / TY, (g.nzp + ZCHUNK - 1) / ZCHUNK);
  kern<<<grid, P2G_THREADS, Lay::smem, ctx->stream>>>(g, ctx->cell_start, ctx->sorted, ctx->del, ctx->cap,
                                                      prop(ctx, PMPIC_PROP_VOL), a, ctx->dinfo); ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

// parcel_mixing construct_grids (:440-624) + mixing_haloswap + wall doubling:
// kept grids into VOL, B, HG, P, Q, R (as the reference reuses state%vol,
// state%b, state%hg, state%p, ...), residual grids into mixres, npercell.
// With no parcel in the removed class (any_removed false) its sums are all
// +0.0, which a memset gives without a pass over the parcels.
int launch_mix_grids(pmpic_ctx* ctx, bool any_removed) {
  const double* f[6] = {nullptr, prop(ctx, PMPIC_PROP_B), prop(ctx, PMPIC_PROP_H),
                        prop(ctx, PMPIC_PROP_P), prop(ctx, PMPIC_PROP_Q), prop(ctx, PMPIC_PROP_R)};
  double* kept[6] = {ctx->grid[PMPIC_GRID_VOL], ctx->grid[PMPIC_GRID_B], ctx->grid[PMPIC_GRID_HG],
                     ctx->grid[PMPIC_GRID_P],   ctx->grid[PMPIC_GRID_Q], ctx->grid[PMPIC_GRID_R]};
  int rc = launch_p2g<6, 1, false>(ctx, f, kept);
  if (rc) return rc;
  if (any_removed) return launch_p2g<6, 2, false>(ctx, f, ctx->mixres);
  for (int q = 0; q < 6; ++q)
    PMPIC_CUDA(cudaMemsetAsync(ctx->mixres[q], 0, sizeof(double) * ctx->g.nphys, ctx->stream));
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
    default: return set_error(ctx, PMPIC_ERR_ARG, "par2grid_multi: 1 or 3 fields");
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

// cached cell ids of the current positions (ctx->cell)
int cell_ids(pmpic_ctx* ctx, int32_t* dcells) {
  (void)dcells;
  return bin_and_sort(ctx);
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
constexpr size_t SP_BYTES = SP_INFO + sp_round(sizeof(DevInfo));                        // about 4.5 MB

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
  if (nx < 1 || ny < 1 || nz < 1 || !(lx > 0) || !(ly > 0) || !(lz > 0) || n < 0 || !out) return PMPIC_ERR_ARG;
  if (n > 0 && (!x || !y || !z || !vol || !field)) return PMPIC_ERR_ARG;
  const int64_t ncell = (int64_t)nx * ny * nz;
  if (n > SP_MAX_PARCELS || ncell > SP_MAX_CELLS) return PMPIC_ERR_TOO_LARGE;
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
    k_bin_scatter<<<nblk(n, 256), 256, 0, st>>>(n, cell, cstart, fill, sorted);
    k_sort_segments<<<nblk(ncell, 256), 256, 0, st>>>(ncell, cstart, sorted);
  }
  using Lay = P2GLayout<1, 0, false>;
  auto kern = k_par2grid<1, 0, false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::smem) != cudaSuccess)
    return PMPIC_ERR_CUDA;
  P2GArgs<1> a{};
  a.f[0] = field;
  a.out[0] = out;
  dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY, (g.nzp + ZCHUNK - 1) / ZCHUNK);
  kern<<<grid, P2G_THREADS, Lay::smem, st>>>(g, cstart, sorted, del, SP_MAX_PARCELS, vol, a, info);
  if (cudaGetLastError() != cudaSuccess) return PMPIC_ERR_CUDA;
  int err = 0;
  if (cudaMemcpyAsync(&err, &info->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PMPIC_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return PMPIC_ERR_CUDA;
  return err;
}
