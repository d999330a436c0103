// h5lite.hpp -- the subset of the HDF5 file format the tdse inputs use.
//
// The reference reads its energies and dipole blocks with the HDF5 C++ API
// (tdrd::readEnergies / readDipoles, src/tdse/td_read.cpp:50-120): one
// dataset per file at the root group ("En", "d_if", "En_CI", "CI_dip"), IEEE
// float64, 1-D or 2-D, written by H5Cpp with default properties.  libhdf5 is
// not a dependency here, so this file implements, from the published HDF5
// File Format Specification (version 3.0):
//   reading  - superblock versions 0, 1, 2 and 3; object headers version 1
//              and 2; root-group lookup through a symbol table (v1 B-tree +
//              local heap + symbol nodes) or compact link messages;
//              dataspace messages v1/v2; floating-point datatype (8 bytes,
//              either byte order); data layout v3 (contiguous and compact);
//   writing  - superblock v0, v1 object headers, a symbol-table root group
//              and contiguous float64 datasets (the layout HDF5 writes with
//              its default, earliest-format settings).
// Unsupported features (chunked or filtered storage, dense link storage,
// other types) raise h5::Error.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace h5 {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Dataset {
  std::vector<uint64_t> dims;
  std::vector<double> data;  // row-major (C order)
};

// Reads dataset `name` from the root group of `path`.
Dataset read(const std::string& path, const std::string& name);

// Reads only the top-left sub-block [rows x cols] of a 2-D dataset (or the
// first `rows` entries of a 1-D one, cols ignored), as the reference's
// hyperslab selections do.
std::vector<double> read_block(const std::string& path, const std::string& name, uint64_t rows,
                               uint64_t cols);

// Writes a file holding the given float64 datasets at the root group.
struct NamedArray {
  std::string name;
  std::vector<uint64_t> dims;
  const double* data;
};
void write(const std::string& path, const std::vector<NamedArray>& sets);

}  // namespace h5
