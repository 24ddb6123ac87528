// Named-array container for the inputs and outputs of one SQ step.
//
// A "case" holds exactly what ClenshawCurtisSpectralQuadrature (sq.cpp:377),
// NonlocalProjectors (nonlocal.cpp:317) and ForcesNonLocal (forces.cpp:318)
// read from DS_SQ (ds_sq.h:128-238): grid parameters, the Veff block with its
// Rcut halo, the replica atoms of every type (ds_sq.h:26-30) and the radial
// pseudopotential tables with their spline derivatives (ds_sq.h:76-102).
// Outputs of a reference run (rho, rho_pj, Ci, chi, zee, lambda_f, Ebs, Eent,
// fnloc) use the same container.
//
// File layout: the 8-byte magic "SQBCASE1", then records of
//   char name[48] | int32 dtype | int32 ndim | int64 dims[ndim] | data
// with dtype 1 = float64, 2 = int32, 3 = float32, terminated by a record
// named "__end__".  Little-endian, no padding.  sqdft_b200/case.py reads it.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace sqb {

class CaseWriter {
 public:
  explicit CaseWriter(const std::string &path);
  ~CaseWriter();
  bool ok() const { return f_ != nullptr; }
  void f64(const char *name, const double *data, std::vector<int64_t> dims);
  void i32(const char *name, const int *data, std::vector<int64_t> dims);
  void f64s(const char *name, double v) { f64(name, &v, {1}); }
  void i32s(const char *name, int v) { i32(name, &v, {1}); }
  void close();

 private:
  void record(const char *name, int dtype, const void *data, size_t elem, const std::vector<int64_t> &dims);
  FILE *f_ = nullptr;
};

}  // namespace sqb
