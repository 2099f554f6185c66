// parcel_setup.cpp -- host-side parcel initial conditions (new set-up component).
//
// The reference ships user-supplied set-up components (basic_parcelsetup,
// plume_parcelsetup); the jittered thermal plume here is the initial condition
// of the benchmark workloads.  This host generator gives the CPU oracle its
// inputs; setup.cu writes the same parcels on the device from the same
// per-parcel formula (thermal.h).  Neither is part of the per-timestep path.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "thermal.h"

extern "C" int64_t pmpic_setup_count(const pmpic_thermal_params* p) {
  if (!p || p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->sub <= 0) return -1;
  return (int64_t)p->nx * p->ny * p->nz * p->sub * p->sub * p->sub;
}

extern "C" int pmpic_setup_thermal(const pmpic_thermal_params* prm, int64_t n, double* x, double* y,
                                   double* z, double* p, double* q, double* r, double* b, double* h,
                                   double* vol, double* stretch, double* tag) {
  int64_t total = pmpic_setup_count(prm);
  if (total < 0 || n < total) return PMPIC_ERR_ARG;
  const pmpic::ThermalGeom g = pmpic::thermal_geom(prm);
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < total; ++idx) {
    const pmpic::ThermalParcel c = pmpic::thermal_parcel(*prm, g, idx);
    x[idx] = c.x; y[idx] = c.y; z[idx] = c.z;
    if (p) p[idx] = 0.0;
    if (q) q[idx] = 0.0;
    if (r) r[idx] = 0.0;
    b[idx] = c.b; h[idx] = c.h; vol[idx] = g.v0;
    if (stretch) stretch[idx] = 0.0;
    if (tag) tag[idx] = (double)idx;
  }
  return PMPIC_OK;
}
