// parcel_setup.cpp -- host-side parcel initial conditions (new set-up component).
//
// The reference ships user-supplied set-up components (basic_parcelsetup,
// plume_parcelsetup); the jittered thermal plume here is the initial condition
// of the benchmark workloads.  It is generated on the host so that the CPU
// oracle and the GPU receive bit-identical inputs, and it is not part of the
// per-timestep path.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/pmpic_gpu.h"

namespace {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11), counter = (index lo, index hi, stream, 0), key = seed.
struct Philox {
  uint32_t k0, k1;
  static inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
  }
  void block(uint32_t c[4]) const {
    uint32_t key0 = k0, key1 = k1;
    for (int r = 0; r < 10; ++r) {
      uint32_t hi0, lo0, hi1, lo1;
      mulhilo(0xD2511F53u, c[0], hi0, lo0);
      mulhilo(0xCD9E8D57u, c[2], hi1, lo1);
      uint32_t n0 = hi1 ^ c[1] ^ key0;
      uint32_t n1 = lo1;
      uint32_t n2 = hi0 ^ c[3] ^ key1;
      uint32_t n3 = lo0;
      c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
      key0 += 0x9E3779B9u;
      key1 += 0xBB67AE85u;
    }
  }
};

// uniform double in [0,1) from two 32-bit words (53 bits)
inline double u01(uint32_t a, uint32_t b) {
  uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  v &= ((1ull << 53) - 1);
  return (double)v * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" int64_t pmpic_setup_count(const pmpic_thermal_params* p) {
  if (!p || p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->sub <= 0) return -1;
  return (int64_t)p->nx * p->ny * p->nz * p->sub * p->sub * p->sub;
}

extern "C" int pmpic_setup_thermal(const pmpic_thermal_params* prm, int64_t n, double* x, double* y,
                                   double* z, double* p, double* q, double* r, double* b, double* h,
                                   double* vol, double* stretch, double* tag) {
  int64_t total = pmpic_setup_count(prm);
  if (total < 0 || n < total) return PMPIC_ERR_ARG;
  const int nx = prm->nx, ny = prm->ny, nz = prm->nz, s = prm->sub;
  const double dx = prm->lx / nx, dy = prm->ly / ny, dz = prm->lz / nz;
  const double sdx = dx / s, sdy = dy / s, sdz = dz / s;
  const double v0 = dx * dy * dz / ((double)s * s * s);
  const double pi = 4.0 * std::atan(1.0);
  Philox ph;
  ph.k0 = (uint32_t)prm->seed;
  ph.k1 = (uint32_t)(prm->seed >> 32);
  const int64_t per_cell = (int64_t)s * s * s;
#pragma omp parallel for schedule(static)
  for (int64_t cell = 0; cell < (int64_t)nx * ny * nz; ++cell) {
    // cell order: x outer, then y, then z (basic_parcelsetup.F90:90-96)
    int i = (int)(cell / ((int64_t)ny * nz));
    int j = (int)((cell / nz) % ny);
    int k = (int)(cell % nz);
    for (int a = 0; a < s; ++a)
      for (int bb = 0; bb < s; ++bb)
        for (int cc = 0; cc < s; ++cc) {
          int64_t idx = cell * per_cell + ((int64_t)a * s + bb) * s + cc;
          uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)((uint64_t)idx >> 32), 0u, 0u};
          ph.block(ctr);
          uint32_t ctr2[4] = {(uint32_t)idx, (uint32_t)((uint64_t)idx >> 32), 1u, 0u};
          ph.block(ctr2);
          double jx = (2.0 * u01(ctr[0], ctr[1]) - 1.0) * prm->jitter;
          double jy = (2.0 * u01(ctr[2], ctr[3]) - 1.0) * prm->jitter;
          double jz = (2.0 * u01(ctr2[0], ctr2[1]) - 1.0) * prm->jitter;
          double px = i * dx + (a + 0.5 + jx) * sdx;
          double py = j * dy + (bb + 0.5 + jy) * sdy;
          double pz = k * dz + (cc + 0.5 + jz) * sdz;
          double rx = px - prm->xc, ry = py - prm->yc, rz = pz - prm->zc;
          double rr = std::sqrt(rx * rx + ry * ry + rz * rz);
          double benv = (pz > prm->z_strat) ? (pz - prm->z_strat) * prm->n2 : 0.0;
          double henv = prm->h_env0 * (1.0 - pz / prm->lz);
          double bv = benv, hv = henv;
          if (rr < prm->radius) {
            double cs = std::cos(pi * rr / (2.0 * prm->radius));
            bv = benv + prm->excess * cs * cs;
            hv = prm->h_in;
          }
          x[idx] = px; y[idx] = py; z[idx] = pz;
          if (p) p[idx] = 0.0;
          if (q) q[idx] = 0.0;
          if (r) r[idx] = 0.0;
          b[idx] = bv; h[idx] = hv; vol[idx] = v0;
          if (stretch) stretch[idx] = 0.0;
          if (tag) tag[idx] = (double)idx;
        }
  }
  return PMPIC_OK;
}
