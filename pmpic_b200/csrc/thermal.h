// thermal.h -- the jittered thermal initial condition, one parcel at a time,
// compiled for the host generator (parcel_setup.cpp) and the device one
// (setup.cu) from the same source, so both give the same parcels.
#pragma once
#include <cmath>
#include <cstdint>

#include "../../include/pmpic_gpu.h"

#ifdef __CUDACC__
#define PMPIC_HD __host__ __device__ __forceinline__
#else
#define PMPIC_HD inline
#endif

namespace pmpic {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11), counter = (index lo, index hi, stream, 0), key = seed.
PMPIC_HD void philox_block(uint32_t k0, uint32_t k1, uint32_t c[4]) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// uniform double in [0,1) from two 32-bit words (53 bits)
PMPIC_HD double philox_u01(uint32_t a, uint32_t b) {
  uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  v &= ((1ull << 53) - 1);
  return (double)v * (1.0 / 9007199254740992.0);
}

// spacings of the sub-lattice, computed once on the host
struct ThermalGeom {
  double dx, dy, dz, sdx, sdy, sdz, v0, pi;
};
inline ThermalGeom thermal_geom(const pmpic_thermal_params* p) {
  ThermalGeom g;
  const int s = p->sub;
  g.dx = p->lx / p->nx; g.dy = p->ly / p->ny; g.dz = p->lz / p->nz;
  g.sdx = g.dx / s; g.sdy = g.dy / s; g.sdz = g.dz / s;
  g.v0 = g.dx * g.dy * g.dz / ((double)s * s * s);
  g.pi = 4.0 * std::atan(1.0);
  return g;
}

struct ThermalParcel {
  double x, y, z, b, h;
};

// Parcel idx: cell by cell (x outer, then y, then z) and, inside a cell, sub-
// lattice point by point (x outer, z inner), the order of
// basic_parcelsetup.F90:90-118.
PMPIC_HD ThermalParcel thermal_parcel(const pmpic_thermal_params& prm, const ThermalGeom& g, int64_t idx) {
  const int s = prm.sub;
  const int64_t per_cell = (int64_t)s * s * s;
  const int64_t cell = idx / per_cell;
  const int w = (int)(idx - cell * per_cell);
  const int i = (int)(cell / ((int64_t)prm.ny * prm.nz));
  const int j = (int)((cell / prm.nz) % prm.ny);
  const int k = (int)(cell % prm.nz);
  const int a = w / (s * s), bb = (w / s) % s, cc = w % s;
  uint32_t c1[4] = {(uint32_t)idx, (uint32_t)((uint64_t)idx >> 32), 0u, 0u};
  uint32_t c2[4] = {(uint32_t)idx, (uint32_t)((uint64_t)idx >> 32), 1u, 0u};
  const uint32_t k0 = (uint32_t)prm.seed, k1 = (uint32_t)(prm.seed >> 32);
  philox_block(k0, k1, c1);
  philox_block(k0, k1, c2);
  const double jx = (2.0 * philox_u01(c1[0], c1[1]) - 1.0) * prm.jitter;
  const double jy = (2.0 * philox_u01(c1[2], c1[3]) - 1.0) * prm.jitter;
  const double jz = (2.0 * philox_u01(c2[0], c2[1]) - 1.0) * prm.jitter;
  ThermalParcel p;
  p.x = i * g.dx + (a + 0.5 + jx) * g.sdx;
  p.y = j * g.dy + (bb + 0.5 + jy) * g.sdy;
  p.z = k * g.dz + (cc + 0.5 + jz) * g.sdz;
  const double rx = p.x - prm.xc, ry = p.y - prm.yc, rz = p.z - prm.zc;
  const double rr = sqrt(rx * rx + ry * ry + rz * rz);
  const double benv = (p.z > prm.z_strat) ? (p.z - prm.z_strat) * prm.n2 : 0.0;
  p.b = benv;
  p.h = prm.h_env0 * (1.0 - p.z / prm.lz);
  if (rr < prm.radius) {
    const double cs = cos(g.pi * rr / (2.0 * prm.radius));
    p.b = benv + prm.excess * cs * cs;
    p.h = prm.h_in;
  }
  return p;
}

}  // namespace pmpic
