// dump.cu -- parcel and grid dumps in the reference's binary stream format, and
// the parcel restart reader, so that the reference's post-processing tools and
// its restart path read and write the same files as this library.
//
// Parcel dump (writebinary.F90:149-199, "parcels_<rank>_<num>.dat"): stream,
// native byte order: time (real*8); the rank's domain x_coords(first),
// x_coords(last+1), y likewise, z_coords(first), z_coords(last) (6 real*8);
// numparcels (integer*8); then x, y, z, p, q, r, dxdt, dydt, dzdt, dpdt, dqdt,
// drdt, h, b, vol, stretch, tag, each numparcels real*8 (qvalues: qnum = 0).
// Grid dump (writebinary.F90:201-299, "grids_<rank>_<num>.dat"): time; x_coords
// of the first and last interior points, y likewise, z of the first and last
// level (6 real*8); the sizes nx, ny, nz+1 (3 integer*4); then u, v, w, p, q,
// r, b, hg, hgliq, vol, each (nz+1)*ny*nx real*8 with z fastest, then y, then x.
// Before the grids are written, p, q, r, b and h are gridded afresh from the
// parcels (par2grid with a fresh binning), hgliq = max(0, hg - exp(-z)) and
// b = b + 12.5 hgliq.
// NetCDF files (writenetcdf.F90:182-439, "grids_<num>.nc" and
// "parcels_<rank>_<num>.nc"): the same grids and parcel properties with the
// writer's dimensions, variables and attributes, in the NetCDF classic
// 64-bit-offset format (the reference writes NetCDF-4 through libnetcdf,
// which this build does not link; netCDF readers open either format).
// Restart (readfromfile_parcelsetup.F90:26-321): every parcel of the file whose
// x and y lie in this domain ([xmin, xmax), [ymin, ymax)) is taken, in file
// order; several files (one per rank of the run that wrote them) are read by
// appending.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <ctime>
#include <vector>

#include "common.cuh"
#include "netcdf_classic.h"

using namespace pmpic;

namespace {

const int kDumpProps[17] = {PMPIC_PROP_X,    PMPIC_PROP_Y,    PMPIC_PROP_Z,    PMPIC_PROP_P,       PMPIC_PROP_Q,
                            PMPIC_PROP_R,    PMPIC_PROP_DXDT, PMPIC_PROP_DYDT, PMPIC_PROP_DZDT,    PMPIC_PROP_DPDT,
                            PMPIC_PROP_DQDT, PMPIC_PROP_DRDT, PMPIC_PROP_H,    PMPIC_PROP_B,       PMPIC_PROP_VOL,
                            PMPIC_PROP_STRETCH, PMPIC_PROP_TAG};

constexpr int64_t CHUNK = (int64_t)1 << 22;  // values per host transfer

struct File {
  FILE* f = nullptr;
  explicit File(FILE* p) : f(p) {}
  ~File() {
    if (f) fclose(f);
  }
};

// one grid in the dump's order (z fastest, then y, then x), widened to FP64;
// mode 1: hgliq = max(0, hg - exp(-z)); mode 2: b + 12.5 hgliq (hg in h)
template <class R>
__global__ void k_dump_field(Geom g, const R* __restrict__ src, const R* __restrict__ h, int mode,
                             double* __restrict__ dst) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.nphys) return;
  const int k = (int)(e % g.nzp);
  const int j = (int)((e / g.nzp) % g.Ny);
  const int i = (int)(e / ((int64_t)g.nzp * g.Ny));
  const size_t o = ((size_t)k * g.Ny + j) * g.Nx + i;
  double v = (double)src[o];
  if (mode) {
    const double zc = g.pzmin + (double)k * g.dz;  // z_coords(k+1)
    const double hgliq = fmax(0.0, (double)h[o] - exp(-zc));
    v = mode == 1 ? hgliq : v + 12.5 * hgliq;
  }
  dst[e] = v;
}

}  // namespace

// p, q, r, b and h gridded afresh into the work grids (writebinary.F90:205-211;
// writenetcdf.F90:182-211), then the ten dump fields u, v, w, p, q, r,
// b (+12.5 hgliq), hg, hgliq, vol handed to emit(values, count) one at a time
// as FP64 host arrays, z fastest.  The model's own grids, which a step in
// progress may still use, are untouched.
template <class Emit>
int dump_grid_fields(pmpic_ctx* ctx, Emit&& emit) {
  int rc;
  const Geom& g = ctx->g;
  if (!ctx->sorted_valid && (rc = bin_and_sort(ctx))) return rc;
  double* W[5] = {ctx->gwork[0], ctx->gwork[1], ctx->gwork[2], ctx->gwork[3], ctx->gwork[4]};  // p q r b h
  if (ctx->mixed) {
    const float* f4[4] = {propf(ctx, PMPIC_PROP_P), propf(ctx, PMPIC_PROP_Q), propf(ctx, PMPIC_PROP_R),
                          propf(ctx, PMPIC_PROP_B)};
    float* o4[4] = {(float*)W[0], (float*)W[1], (float*)W[2], (float*)W[3]};
    const float* f1[1] = {propf(ctx, PMPIC_PROP_H)};
    float* o1[1] = {(float*)W[4]};
    if ((rc = par2grid_multi_m(ctx, f4, 4, o4)) || (rc = par2grid_multi_m(ctx, f1, 1, o1))) return rc;
  } else {
    const double* f4[4] = {prop(ctx, PMPIC_PROP_P), prop(ctx, PMPIC_PROP_Q), prop(ctx, PMPIC_PROP_R),
                           prop(ctx, PMPIC_PROP_B)};
    const double* f1[1] = {prop(ctx, PMPIC_PROP_H)};
    if ((rc = par2grid_multi(ctx, f4, 4, W, false)) || (rc = par2grid_multi(ctx, f1, 1, W + 4, false))) return rc;
  }
  if ((rc = sync_info(ctx))) return rc;
  const double* src[10] = {ctx->grid[PMPIC_GRID_U], ctx->grid[PMPIC_GRID_V], ctx->grid[PMPIC_GRID_W], W[0], W[1], W[2],
                           W[3], W[4], W[4], ctx->grid[PMPIC_GRID_VOL]};
  const int mode[10] = {0, 0, 0, 0, 0, 0, 2, 0, 1, 0};
  double* stage = ctx->sscratch;  // nspec >= nphys doubles, free between operators
  std::vector<double> host((size_t)g.nphys);
  const unsigned nb = (unsigned)((g.nphys + 255) / 256);
  for (int q = 0; q < 10; ++q) {
    if (ctx->mixed)
      k_dump_field<float><<<nb, 256, 0, ctx->stream>>>(g, (const float*)src[q], (const float*)W[4], mode[q], stage);
    else
      k_dump_field<double><<<nb, 256, 0, ctx->stream>>>(g, src[q], W[4], mode[q], stage);
    ++ctx->nlaunch;
    PMPIC_CUDA(cudaGetLastError());
    PMPIC_CUDA(cudaMemcpyAsync(host.data(), stage, sizeof(double) * g.nphys, cudaMemcpyDeviceToHost, ctx->stream));
    PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!emit(host.data(), g.nphys)) return PMPIC_ERR_ARG;
  }
  return 0;
}

// ---- NetCDF files (writenetcdf.F90) -----------------------------------------
namespace {

// the global attributes of write_out_global_attributes (:443-454): the title
// and the creation time as day/month/year hour:minute:second, unpadded
void nc_global_atts(NcClassicWriter& w) {
  w.global_text("title", "MONC checkpoint file");
  std::time_t t = std::time(nullptr);
  std::tm lt{};
  localtime_r(&t, &lt);
  char buf[64];
  std::snprintf(buf, sizeof buf, "%d/%d/%d %d:%d:%d", lt.tm_mday, lt.tm_mon + 1, lt.tm_year + 1900, lt.tm_hour,
                lt.tm_min, lt.tm_sec);
  w.global_text("created", buf);
}

const char* const kNcGridFields[10] = {"u", "v", "w", "p", "q", "r", "b", "hg", "hgliq", "vol"};

// write_ncgrid_file (:225-308) for one process: dimensions time, z, y, x; the
// 1-D coordinate variables; the ten fields over (time, x, y, z) (the Fortran
// (z, y, x, time)); timestep and dtm.  Writes the header and the fixed data
// before the fields; the caller adds the ten fields, then finishes with
// nc_grid_tail.
bool nc_grid_head(NcClassicWriter& w, const char* path, int Nx, int Ny, int nzp, double dx, double dy, double dz,
                  double time) {
  nc_global_atts(w);
  const int dt = w.dim("time", 1), dzid = w.dim("z", nzp), dyid = w.dim("y", Ny), dxid = w.dim("x", Nx);
  w.var("time", NcClassicWriter::NC_DOUBLE, {dt}, "-");
  w.var("z", NcClassicWriter::NC_DOUBLE, {dzid}, "-");
  w.var("y", NcClassicWriter::NC_DOUBLE, {dyid}, "-");
  w.var("x", NcClassicWriter::NC_DOUBLE, {dxid}, "-");
  for (const char* f : kNcGridFields) w.var(f, NcClassicWriter::NC_DOUBLE, {dt, dxid, dyid, dzid}, "-");
  w.var("timestep", NcClassicWriter::NC_INT, {}, "");
  w.var("dtm", NcClassicWriter::NC_DOUBLE, {}, "");
  if (!w.begin(path, 0)) return false;
  // coordinates (:254-263): bottom + resolution * (i - 1.0) for z, (i - 0.5)
  // for y and x, with the default-real literal (i - 1.0 in single precision)
  std::vector<double> a((size_t)std::max(nzp, std::max(Ny, Nx)));
  bool ok = w.fixed_doubles(&time, 1);
  for (int i = 1; i <= nzp; ++i) a[i - 1] = 0.0 + dz * (double)((float)i - 1.0f);
  ok = ok && w.fixed_doubles(a.data(), nzp);
  for (int i = 1; i <= Ny; ++i) a[i - 1] = 0.0 + dy * (double)((float)i - 0.5f);
  ok = ok && w.fixed_doubles(a.data(), Ny);
  for (int i = 1; i <= Nx; ++i) a[i - 1] = 0.0 + dx * (double)((float)i - 0.5f);
  return ok && w.fixed_doubles(a.data(), Nx);
}
bool nc_grid_tail(NcClassicWriter& w, int32_t timestep, double dtm) {
  return w.fixed_int(timestep) && w.fixed_doubles(&dtm, 1) && w.end();
}

const char* const kNcParcelVars[17] = {"x",    "y",    "z",    "p", "q", "r",   "dxdt",   "dydt", "dzdt",
                                       "dpdt", "dqdt", "drdt", "h", "b", "vol", "stetch", "tag"};

// write_parcels_to_file (:310-439) for one process: dimensions time and the
// unlimited nparcel; time, the record variables parcel (1..n) and the 17
// properties (the reference's key "stetch" for stretch; qnum = 0 q-values),
// the scalars x_start .. z_end (the local domain's index bounds: 3, Nx+3,
// 3, Ny+3, 1, Nz+1 on one process), timestep and dtm.  Writes everything but
// the records.
bool nc_parcel_head(NcClassicWriter& w, const char* path, int Nx, int Ny, int Nz, int64_t n, double time,
                    int32_t timestep, double dtm) {
  nc_global_atts(w);
  const int dt = w.dim("time", 1), dp = w.dim("nparcel", 0);
  w.var("time", NcClassicWriter::NC_DOUBLE, {dt}, "-");
  w.var("parcel", NcClassicWriter::NC_DOUBLE, {dp}, "-");
  for (const char* v : kNcParcelVars) w.var(v, NcClassicWriter::NC_DOUBLE, {dp}, "-");
  const char* bounds[6] = {"x_start", "y_start", "z_start", "x_end", "y_end", "z_end"};
  for (const char* b : bounds) w.var(b, NcClassicWriter::NC_DOUBLE, {}, "");
  w.var("timestep", NcClassicWriter::NC_INT, {}, "");
  w.var("dtm", NcClassicWriter::NC_DOUBLE, {}, "");
  if (!w.begin(path, n)) return false;
  const double bv[6] = {3.0, 3.0, 1.0, (double)Nx + 3.0, (double)Ny + 3.0, (double)Nz + 1.0};
  return w.fixed_doubles(&time, 1) && w.fixed_doubles(bv, 6) && w.fixed_int(timestep) && w.fixed_doubles(&dtm, 1);
}

}  // namespace

extern "C" {

int pmpic_write_parcels(pmpic_ctx* ctx, const char* path, double time) {
  if (!ctx || !path) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = flush_gathers(ctx);  // the tendencies are part of the dump
  if (rc) return rc;
  File fo(std::fopen(path, "wb"));
  if (!fo.f) return set_error(ctx, PMPIC_ERR_ARG, std::string("cannot open ") + path);
  const Geom& g = ctx->g;
  const int64_t n = ctx->n;
  const double hdr[7] = {time, 0.0, (double)g.Nx * g.dx, 0.0, (double)g.Ny * g.dy, 0.0, (double)g.Nz * g.dz};
  bool ok = std::fwrite(hdr, sizeof(double), 7, fo.f) == 7;
  ok = ok && std::fwrite(&n, sizeof(int64_t), 1, fo.f) == 1;
  std::vector<double> buf((size_t)std::min<int64_t>(std::max<int64_t>(n, 1), CHUNK));
  for (int q = 0; q < 17 && ok; ++q) {
    for (int64_t c0 = 0; c0 < n && ok; c0 += CHUNK) {
      const int64_t len = std::min<int64_t>(CHUNK, n - c0);
      if ((rc = prop_download(ctx, kDumpProps[q], c0, len, buf.data()))) return rc;
      PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
      ok = std::fwrite(buf.data(), sizeof(double), (size_t)len, fo.f) == (size_t)len;
    }
  }
  if (!ok) return set_error(ctx, PMPIC_ERR_ARG, std::string("write failed: ") + path);
  return PMPIC_OK;
}

int pmpic_read_parcels(pmpic_ctx* ctx, const char* path, int append, double* time) {
  if (!ctx || !path) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  File fi(std::fopen(path, "rb"));
  if (!fi.f) return set_error(ctx, PMPIC_ERR_ARG, std::string("cannot open ") + path);
  double hdr[7];
  int64_t nin = 0;
  if (std::fread(hdr, sizeof(double), 7, fi.f) != 7 || std::fread(&nin, sizeof(int64_t), 1, fi.f) != 1 || nin < 0)
    return set_error(ctx, PMPIC_ERR_ARG, std::string("not a parcel dump: ") + path);
  if (time) *time = hdr[0];
  int rc = flush_gathers(ctx);
  if (rc) return rc;
  const Geom& g = ctx->g;
  const double xmin = 0.0, xmax = (double)g.Nx * g.dx, ymin = 0.0, ymax = (double)g.Ny * g.dy;
  // which parcels of the file belong to this domain (readfromfile_parcelsetup.F90:205-214)
  std::vector<double> x((size_t)nin), y((size_t)nin);
  if (std::fread(x.data(), sizeof(double), (size_t)nin, fi.f) != (size_t)nin ||
      std::fread(y.data(), sizeof(double), (size_t)nin, fi.f) != (size_t)nin)
    return set_error(ctx, PMPIC_ERR_ARG, std::string("truncated parcel dump: ") + path);
  std::vector<int64_t> keep;
  keep.reserve((size_t)nin);
  for (int64_t t = 0; t < nin; ++t)
    if (x[t] < xmax && x[t] >= xmin && y[t] < ymax && y[t] >= ymin) keep.push_back(t);
  x.clear();
  y.clear();
  const int64_t n0 = append ? ctx->n : 0;
  const int64_t nk = (int64_t)keep.size();
  if (n0 + nk > ctx->cap) return set_error(ctx, PMPIC_ERR_CAPACITY, "parcel count exceeds max_parcels");
  std::vector<double> col((size_t)nin), sel((size_t)nk);
  const long data0 = (long)(7 * sizeof(double) + sizeof(int64_t));
  for (int q = 0; q < 17; ++q) {
    if (std::fseek(fi.f, data0 + (long)((int64_t)q * nin * (int64_t)sizeof(double)), SEEK_SET) != 0 ||
        std::fread(col.data(), sizeof(double), (size_t)nin, fi.f) != (size_t)nin)
      return set_error(ctx, PMPIC_ERR_ARG, std::string("truncated parcel dump: ") + path);
    for (int64_t t = 0; t < nk; ++t) sel[t] = col[keep[t]];
    if ((rc = prop_upload(ctx, kDumpProps[q], n0, nk, sel.data()))) return rc;
    PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));  // sel is reused
  }
  // the RK4 arrays and btot of the new slots start at zero, as after set-up
  const int zero[] = {PMPIC_PROP_BTOT, PMPIC_PROP_XO, PMPIC_PROP_YO, PMPIC_PROP_ZO, PMPIC_PROP_XF, PMPIC_PROP_YF,
                      PMPIC_PROP_ZF,   PMPIC_PROP_PO, PMPIC_PROP_QO, PMPIC_PROP_RO, PMPIC_PROP_PF, PMPIC_PROP_QF,
                      PMPIC_PROP_RF};
  for (int pid : zero)
    if ((rc = prop_upload(ctx, pid, n0, nk, nullptr))) return rc;
  PMPIC_CUDA(cudaMemsetAsync(&ctx->dinfo->error, 0, sizeof(int), ctx->stream));
  PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->n = n0 + nk;
  ctx->info.n_parcels = ctx->n;
  ctx->sorted_valid = false;
  ctx->count_ready = false;
  ctx->in_domain = false;
  ctx->btot_grid_ready = false;
  ctx->dir_ready = false;
  return PMPIC_OK;
}

int pmpic_write_grids(pmpic_ctx* ctx, const char* path, double time) {
  if (!ctx || !path) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  const Geom& g = ctx->g;
  File fo(std::fopen(path, "wb"));
  if (!fo.f) return set_error(ctx, PMPIC_ERR_ARG, std::string("cannot open ") + path);
  const double hdr[7] = {time, 0.0, (double)(g.Nx - 1) * g.dx, 0.0, (double)(g.Ny - 1) * g.dy, 0.0,
                         (double)g.Nz * g.dz};
  const int32_t sz[3] = {g.Nx, g.Ny, g.nzp};
  bool ok = std::fwrite(hdr, sizeof(double), 7, fo.f) == 7 && std::fwrite(sz, sizeof(int32_t), 3, fo.f) == 3;
  int rc = ok ? dump_grid_fields(ctx, [&](const double* v, int64_t n) {
    return std::fwrite(v, sizeof(double), (size_t)n, fo.f) == (size_t)n;
  }) : PMPIC_ERR_ARG;
  if (rc == PMPIC_ERR_ARG) return set_error(ctx, PMPIC_ERR_ARG, std::string("write failed: ") + path);
  return rc;
}

int pmpic_write_grids_netcdf(pmpic_ctx* ctx, const char* path, double time, int32_t timestep) {
  if (!ctx || !path) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  const Geom& g = ctx->g;
  NcClassicWriter w;
  if (!nc_grid_head(w, path, g.Nx, g.Ny, g.nzp, g.dx, g.dy, g.dz, time))
    return set_error(ctx, PMPIC_ERR_ARG, std::string("cannot write ") + path);
  int rc = dump_grid_fields(ctx, [&](const double* v, int64_t n) { return w.fixed_doubles(v, n); });
  if (!rc && !nc_grid_tail(w, timestep, ctx->dtm)) rc = PMPIC_ERR_ARG;
  if (rc == PMPIC_ERR_ARG) return set_error(ctx, PMPIC_ERR_ARG, std::string("write failed: ") + path);
  return rc;
}

int pmpic_write_parcels_netcdf(pmpic_ctx* ctx, const char* path, double time, int32_t timestep) {
  if (!ctx || !path) return PMPIC_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = flush_gathers(ctx);  // the tendencies are part of the file
  if (rc) return rc;
  const Geom& g = ctx->g;
  const int64_t n = ctx->n;
  NcClassicWriter w;
  if (!nc_parcel_head(w, path, g.Nx, g.Ny, g.Nz, n, time, timestep, ctx->dtm))
    return set_error(ctx, PMPIC_ERR_ARG, std::string("cannot write ") + path);
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(n, 1), (int64_t)1 << 18);
  std::vector<double> cols(18 * (size_t)chunk);
  std::vector<const double*> ptr(18);
  for (int q = 0; q < 18; ++q) ptr[q] = cols.data() + (size_t)q * chunk;
  bool ok = true;
  for (int64_t c0 = 0; c0 < n && ok; c0 += chunk) {
    const int64_t len = std::min<int64_t>(chunk, n - c0);
    for (int64_t i = 0; i < len; ++i) cols[i] = (double)(c0 + i + 1);  // parcel = 1..n
    for (int q = 0; q < 17; ++q)
      if ((rc = prop_download(ctx, kDumpProps[q], c0, len, cols.data() + (size_t)(q + 1) * chunk))) return rc;
    PMPIC_CUDA(cudaStreamSynchronize(ctx->stream));
    ok = w.records(ptr, len);
  }
  if (!ok || !w.end()) return set_error(ctx, PMPIC_ERR_ARG, std::string("write failed: ") + path);
  return PMPIC_OK;
}

int pmpic_netcdf_write_grids(const char* path, int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                             double time, int32_t timestep, double dtm, const double* const* fields) {
  if (!path || !fields || nx <= 0 || ny <= 0 || nz <= 0) return PMPIC_ERR_ARG;
  for (int q = 0; q < 10; ++q)
    if (!fields[q]) return PMPIC_ERR_ARG;
  const int64_t np = (int64_t)(nz + 1) * ny * nx;
  NcClassicWriter w;
  bool ok = nc_grid_head(w, path, nx, ny, nz + 1, lx / (double)nx, ly / (double)ny, lz / (double)nz, time);
  for (int q = 0; q < 10 && ok; ++q) ok = w.fixed_doubles(fields[q], np);
  ok = ok && nc_grid_tail(w, timestep, dtm);
  return ok ? PMPIC_OK : PMPIC_ERR_ARG;
}

int pmpic_netcdf_write_parcels(const char* path, int32_t nx, int32_t ny, int32_t nz, int64_t n, double time,
                               int32_t timestep, double dtm, const double* const* props) {
  if (!path || !props || n < 0) return PMPIC_ERR_ARG;
  for (int q = 0; q < 17; ++q)
    if (!props[q] && n > 0) return PMPIC_ERR_ARG;
  NcClassicWriter w;
  bool ok = nc_parcel_head(w, path, nx, ny, nz, n, time, timestep, dtm);
  const int64_t chunk = (int64_t)1 << 18;
  std::vector<double> idx((size_t)std::min<int64_t>(std::max<int64_t>(n, 1), chunk));
  std::vector<const double*> ptr(18);
  for (int64_t c0 = 0; c0 < n && ok; c0 += chunk) {
    const int64_t len = std::min<int64_t>(chunk, n - c0);
    for (int64_t i = 0; i < len; ++i) idx[i] = (double)(c0 + i + 1);
    ptr[0] = idx.data();
    for (int q = 0; q < 17; ++q) ptr[q + 1] = props[q] + c0;
    ok = w.records(ptr, len);
  }
  ok = ok && w.end();
  return ok ? PMPIC_OK : PMPIC_ERR_ARG;
}

}  // extern "C"
