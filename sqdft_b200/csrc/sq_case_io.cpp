// Writer for the named-array case container described in sq_case.h.
#include "sq_case.h"

#include <cstring>

namespace sqb {

CaseWriter::CaseWriter(const std::string &path) {
  f_ = std::fopen(path.c_str(), "wb");
  if (f_) std::fwrite("SQBCASE1", 1, 8, f_);
}

CaseWriter::~CaseWriter() { close(); }

void CaseWriter::record(const char *name, int dtype, const void *data, size_t elem,
                        const std::vector<int64_t> &dims) {
  if (!f_) return;
  char nm[48];
  std::memset(nm, 0, sizeof(nm));
  std::strncpy(nm, name, sizeof(nm) - 1);
  int32_t hdr[2] = {dtype, (int32_t)dims.size()};
  std::fwrite(nm, 1, sizeof(nm), f_);
  std::fwrite(hdr, sizeof(int32_t), 2, f_);
  size_t n = 1;
  for (int64_t d : dims) {
    std::fwrite(&d, sizeof(int64_t), 1, f_);
    n *= (size_t)d;
  }
  if (n) std::fwrite(data, elem, n, f_);
}

void CaseWriter::f64(const char *name, const double *data, std::vector<int64_t> dims) {
  record(name, 1, data, sizeof(double), dims);
}

void CaseWriter::i32(const char *name, const int *data, std::vector<int64_t> dims) {
  record(name, 2, data, sizeof(int), dims);
}

void CaseWriter::close() {
  if (!f_) return;
  record("__end__", 2, nullptr, sizeof(int), {0});
  std::fclose(f_);
  f_ = nullptr;
}

}  // namespace sqb
