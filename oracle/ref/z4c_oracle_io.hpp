// Record-file I/O shared by the reference-oracle problem generator and the
// operator driver (test infrastructure only).
//
// A record file is a sequence of records:
//   char[8]  "Z4CREC01"
//   int32    name length, then the name bytes
//   int32    dtype (0 = float64, 1 = int32)
//   int32    ndim, then int64 dims[ndim]
//   payload  row-major, little endian
// tests/golden/z4cio.py reads and writes the same format.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace z4c_oracle {

struct Record {
  std::string name;
  int dtype = 0;
  std::vector<std::int64_t> dims;
  std::vector<double> f64;
  std::vector<std::int32_t> i32;
  std::int64_t size() const {
    std::int64_t n = 1;
    for (auto d : dims) n *= d;
    return n;
  }
};

class Writer {
 public:
  explicit Writer(const std::string& path) {
    fp_ = std::fopen(path.c_str(), "wb");
    if (!fp_) throw std::runtime_error("cannot open " + path);
  }
  ~Writer() { if (fp_) std::fclose(fp_); }
  void header(const std::string& name, int dtype,
              const std::vector<std::int64_t>& dims) {
    std::fwrite("Z4CREC01", 1, 8, fp_);
    std::int32_t nl = static_cast<std::int32_t>(name.size());
    std::fwrite(&nl, 4, 1, fp_);
    std::fwrite(name.data(), 1, name.size(), fp_);
    std::int32_t dt = dtype, nd = static_cast<std::int32_t>(dims.size());
    std::fwrite(&dt, 4, 1, fp_);
    std::fwrite(&nd, 4, 1, fp_);
    std::fwrite(dims.data(), 8, dims.size(), fp_);
  }
  void f64(const std::string& name, const std::vector<std::int64_t>& dims,
           const double* data) {
    header(name, 0, dims);
    std::int64_t n = 1;
    for (auto d : dims) n *= d;
    std::fwrite(data, 8, n, fp_);
  }
  void i32(const std::string& name, const std::vector<std::int64_t>& dims,
           const std::int32_t* data) {
    header(name, 1, dims);
    std::int64_t n = 1;
    for (auto d : dims) n *= d;
    std::fwrite(data, 4, n, fp_);
  }
 private:
  std::FILE* fp_ = nullptr;
};

inline std::vector<Record> read_all(const std::string& path) {
  std::FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) throw std::runtime_error("cannot open " + path);
  std::vector<Record> out;
  char magic[8];
  while (std::fread(magic, 1, 8, fp) == 8) {
    if (std::memcmp(magic, "Z4CREC01", 8) != 0)
      throw std::runtime_error("bad record magic in " + path);
    Record r;
    std::int32_t nl, dt, nd;
    if (std::fread(&nl, 4, 1, fp) != 1) break;
    r.name.resize(nl);
    if (std::fread(&r.name[0], 1, nl, fp) != static_cast<size_t>(nl)) break;
    if (std::fread(&dt, 4, 1, fp) != 1 || std::fread(&nd, 4, 1, fp) != 1) break;
    r.dtype = dt;
    r.dims.resize(nd);
    if (std::fread(r.dims.data(), 8, nd, fp) != static_cast<size_t>(nd)) break;
    const std::int64_t n = r.size();
    if (dt == 0) {
      r.f64.resize(n);
      if (std::fread(r.f64.data(), 8, n, fp) != static_cast<size_t>(n)) break;
    } else {
      r.i32.resize(n);
      if (std::fread(r.i32.data(), 4, n, fp) != static_cast<size_t>(n)) break;
    }
    out.push_back(std::move(r));
  }
  std::fclose(fp);
  return out;
}

inline const Record& find(const std::vector<Record>& recs,
                          const std::string& name) {
  for (const auto& r : recs)
    if (r.name == name) return r;
  throw std::runtime_error("record not found: " + name);
}

}  // namespace z4c_oracle
