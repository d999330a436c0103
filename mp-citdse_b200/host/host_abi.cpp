// host_abi.cpp -- C entry points of the host I/O layer (libmpc_host.so): the
// HDF5 subset of h5lite.hpp, for tools and tests that prepare or inspect the
// tdse input files (energies "En"/"En_CI", dipoles "d_if"/"CI_dip").
#include <cstdio>
#include <string>
#include <vector>

#include "h5lite.hpp"

namespace {
thread_local std::string g_err;
int fail(const std::exception& e) {
  g_err = e.what();
  return -1;
}
}  // namespace

extern "C" {

int mpc_host_last_error(char* buf, size_t len) {
  if (!buf || !len) return -1;
  std::snprintf(buf, len, "%s", g_err.c_str());
  return 0;
}

// Writes nsets float64 datasets at the root group of `path`; dataset i has
// rank ranks[i] (1 or 2), its dims taken in order from `dims`.
int mpc_h5_write(const char* path, int nsets, const char* const* names, const int* ranks,
                 const long long* dims, const double* const* data) {
  try {
    std::vector<h5::NamedArray> sets;
    int k = 0;
    for (int i = 0; i < nsets; ++i) {
      h5::NamedArray a;
      a.name = names[i];
      for (int r = 0; r < ranks[i]; ++r) a.dims.push_back((uint64_t)dims[k++]);
      a.data = data[i];
      sets.push_back(a);
    }
    h5::write(path, sets);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// rank and dims (up to 2) of a dataset
int mpc_h5_dims(const char* path, const char* name, int* rank, long long* dims) {
  try {
    const h5::Dataset d = h5::read(path, name);
    *rank = (int)d.dims.size();
    for (size_t i = 0; i < d.dims.size() && i < 2; ++i) dims[i] = (long long)d.dims[i];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// top-left rows x cols block (rows entries for a 1-D dataset) into out
int mpc_h5_read_block(const char* path, const char* name, long long rows, long long cols,
                      double* out) {
  try {
    const std::vector<double> v = h5::read_block(path, name, (uint64_t)rows, (uint64_t)cols);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
}
