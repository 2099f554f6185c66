// netcdf_classic.h -- a streaming writer of NetCDF classic files in the
// 64-bit-offset variant (CDF-2), written from the published format
// specification (Unidata, "The NetCDF Classic Format Specification"): a
// header of dimensions, global attributes and variables with their byte
// offsets, then the fixed-size variables' data one after another, then the
// record section (one record = every record variable's slab in turn).  All
// numbers are big-endian.  Host code; the caller writes the data in file
// order: fixed variables in definition order, then whole records.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace pmpic {

class NcClassicWriter {
 public:
  enum Type { NC_CHAR = 2, NC_INT = 4, NC_DOUBLE = 6 };

  // a dimension; length 0 marks the record (unlimited) dimension
  int dim(const std::string& name, int64_t len) {
    dims_.push_back({name, len});
    return (int)dims_.size() - 1;
  }
  void global_text(const std::string& name, const std::string& value) { gatts_.push_back({name, value}); }
  // a variable over dimension ids (slowest first), with a "units" text
  // attribute unless units is empty
  int var(const std::string& name, Type type, const std::vector<int>& dimids, const std::string& units) {
    Var v;
    v.name = name;
    v.type = type;
    v.dimids = dimids;
    v.units = units;
    v.record = !dimids.empty() && dims_[dimids[0]].len == 0;
    int64_t n = 1;
    for (size_t d = v.record ? 1 : 0; d < dimids.size(); ++d) n *= dims_[dimids[d]].len;
    v.vsize = pad4(n * (type == NC_DOUBLE ? 8 : type == NC_INT ? 4 : 1));
    vars_.push_back(v);
    return (int)vars_.size() - 1;
  }

  // write the header for numrecs records; false if the file cannot be written
  // or a variable is too large for the format (vsize must fit in 32 bits)
  bool begin(const char* path, int64_t numrecs) {
    numrecs_ = numrecs;
    if (numrecs < 0 || numrecs > INT32_MAX) return fail();
    for (const Var& v : vars_)
      if (v.vsize > (int64_t)UINT32_MAX - 3) return fail();
    f_ = std::fopen(path, "wb");
    if (!f_) return false;
    // two passes: sizes first, then the offsets are known
    std::vector<uint8_t> h;
    header(h);
    int64_t off = (int64_t)h.size();
    for (Var& v : vars_)
      if (!v.record) {
        v.begin = off;
        off += v.vsize;
      }
    recsize_ = 0;
    for (Var& v : vars_)
      if (v.record) {
        v.begin = off + recsize_;
        recsize_ += v.vsize;
      }
    h.clear();
    header(h);
    return put(h.data(), h.size());
  }
  // data of the next fixed variable (in definition order)
  bool fixed_doubles(const double* x, int64_t n) { return doubles(x, n); }
  bool fixed_int(int32_t x) {
    uint8_t b[4];
    be32(b, (uint32_t)x);
    return put(b, 4);
  }
  // one slab of n consecutive records for record variables that are all
  // scalar doubles per record: cols[v][r] is variable v of record r
  bool records(const std::vector<const double*>& cols, int64_t n) {
    buf_.resize((size_t)n * cols.size() * 8);
    uint8_t* p = buf_.data();
    for (int64_t r = 0; r < n; ++r)
      for (const double* c : cols) {
        uint64_t u;
        std::memcpy(&u, &c[r], 8);
        be64(p, u);
        p += 8;
      }
    return put(buf_.data(), buf_.size());
  }
  bool end() {
    bool ok = f_ && !bad_;
    if (f_) ok = (std::fclose(f_) == 0) && ok;
    f_ = nullptr;
    return ok;
  }
  ~NcClassicWriter() {
    if (f_) std::fclose(f_);
  }

 private:
  struct Dim {
    std::string name;
    int64_t len;
  };
  struct Att {
    std::string name, value;
  };
  struct Var {
    std::string name;
    Type type;
    std::vector<int> dimids;
    std::string units;
    bool record = false;
    int64_t vsize = 0, begin = 0;
  };
  static int64_t pad4(int64_t n) { return (n + 3) & ~(int64_t)3; }
  static void be32(uint8_t* b, uint32_t v) {
    b[0] = (uint8_t)(v >> 24); b[1] = (uint8_t)(v >> 16); b[2] = (uint8_t)(v >> 8); b[3] = (uint8_t)v;
  }
  static void be64(uint8_t* b, uint64_t v) {
    be32(b, (uint32_t)(v >> 32));
    be32(b + 4, (uint32_t)v);
  }
  static void u32(std::vector<uint8_t>& h, uint32_t v) {
    uint8_t b[4];
    be32(b, v);
    h.insert(h.end(), b, b + 4);
  }
  static void u64(std::vector<uint8_t>& h, uint64_t v) {
    uint8_t b[8];
    be64(b, v);
    h.insert(h.end(), b, b + 8);
  }
  static void name(std::vector<uint8_t>& h, const std::string& s) {
    u32(h, (uint32_t)s.size());
    h.insert(h.end(), s.begin(), s.end());
    while (h.size() % 4) h.push_back(0);
  }
  static void text_att(std::vector<uint8_t>& h, const Att& a) {
    name(h, a.name);
    u32(h, NC_CHAR);
    name(h, a.value);  // nelems, the characters, zero padding
  }
  void header(std::vector<uint8_t>& h) const {
    const char magic[4] = {'C', 'D', 'F', 2};
    h.insert(h.end(), magic, magic + 4);
    u32(h, (uint32_t)numrecs_);
    const uint32_t NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12;
    if (dims_.empty()) { u32(h, 0); u32(h, 0); }
    else {
      u32(h, NC_DIMENSION);
      u32(h, (uint32_t)dims_.size());
      for (const Dim& d : dims_) {
        name(h, d.name);
        u32(h, (uint32_t)d.len);
      }
    }
    if (gatts_.empty()) { u32(h, 0); u32(h, 0); }
    else {
      u32(h, NC_ATTRIBUTE);
      u32(h, (uint32_t)gatts_.size());
      for (const Att& a : gatts_) text_att(h, a);
    }
    if (vars_.empty()) { u32(h, 0); u32(h, 0); }
    else {
      u32(h, NC_VARIABLE);
      u32(h, (uint32_t)vars_.size());
      for (const Var& v : vars_) {
        name(h, v.name);
        u32(h, (uint32_t)v.dimids.size());
        for (int d : v.dimids) u32(h, (uint32_t)d);
        if (v.units.empty()) { u32(h, 0); u32(h, 0); }
        else {
          u32(h, NC_ATTRIBUTE);
          u32(h, 1);
          text_att(h, Att{"units", v.units});
        }
        u32(h, (uint32_t)v.type);
        u32(h, (uint32_t)v.vsize);
        u64(h, (uint64_t)v.begin);
      }
    }
  }
  bool doubles(const double* x, int64_t n) {
    const int64_t chunk = 1 << 16;
    for (int64_t c0 = 0; c0 < n; c0 += chunk) {
      const int64_t len = n - c0 < chunk ? n - c0 : chunk;
      buf_.resize((size_t)len * 8);
      for (int64_t i = 0; i < len; ++i) {
        uint64_t u;
        std::memcpy(&u, &x[c0 + i], 8);
        be64(&buf_[(size_t)i * 8], u);
      }
      if (!put(buf_.data(), buf_.size())) return false;
    }
    return true;
  }
  bool put(const void* p, size_t n) {
    if (bad_ || !f_) return false;
    if (n && std::fwrite(p, 1, n, f_) != n) bad_ = true;
    return !bad_;
  }
  bool fail() {
    bad_ = true;
    return false;
  }
  std::vector<Dim> dims_;
  std::vector<Att> gatts_;
  std::vector<Var> vars_;
  std::vector<uint8_t> buf_;
  FILE* f_ = nullptr;
  bool bad_ = false;
  int64_t numrecs_ = 0, recsize_ = 0;
};

}  // namespace pmpic
