// H5Cpp.h stand-in -- TEST INFRASTRUCTURE ONLY.
//
// The subset of the HDF5 C++ API that the reference's src/pes/pes.cpp calls
// (H5File, DataSet, DataSpace with one-dimensional hyperslabs, PredType,
// the int attribute "N"), over an in-memory table of files that the checker's
// driver fills before it calls pes::genPES1e / genPES2e: file name ->
// dataset name -> float64 values.  No HDF5 file is read or written.  The
// attribute "N" reads as the length of the file's "En" dataset, which is what
// the reference's h1e stores there (the number of states in the file).
#pragma once
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

typedef unsigned long long hsize_t;
#define H5F_ACC_RDONLY 0u
enum H5S_seloper_t { H5S_SELECT_SET = 0 };

namespace h5shim {
using File = std::map<std::string, std::vector<double>>;
inline std::map<std::string, File>& files() {
  static std::map<std::string, File> table;
  return table;
}
}  // namespace h5shim

namespace H5 {

struct PredType {
  int is_int;
  static const PredType NATIVE_DOUBLE, NATIVE_INT32, NATIVE_INT;
};
inline const PredType PredType::NATIVE_DOUBLE{0};
inline const PredType PredType::NATIVE_INT32{1};
inline const PredType PredType::NATIVE_INT{1};

struct DataSpace {
  hsize_t extent = 0;
  hsize_t offset = 0, count = 0;
  bool selected = false;
  DataSpace() = default;
  DataSpace(int rank, const hsize_t* dims, const hsize_t* /*maxdims*/) {
    if (rank != 1) throw std::runtime_error("H5 stand-in: rank-1 spaces only");
    extent = dims[0];
  }
  void setExtentSimple(int rank, const hsize_t* dims, const hsize_t* /*maxdims*/ = nullptr) {
    if (rank != 1) throw std::runtime_error("H5 stand-in: rank-1 spaces only");
    extent = dims[0];
  }
  void selectHyperslab(int /*op*/, const hsize_t* cnt, const hsize_t* off,
                       const hsize_t* stride = nullptr, const hsize_t* block = nullptr) {
    if ((stride && stride[0] != 1) || (block && block[0] != 1))
      throw std::runtime_error("H5 stand-in: unit stride and block only");
    offset = off[0];
    count = cnt[0];
    selected = true;
  }
  hsize_t getSimpleExtentNpoints() const { return extent; }
};

struct Attribute {
  double value = 0.0;
  void read(const PredType& t, void* out) const {
    if (t.is_int)
      *static_cast<int*>(out) = static_cast<int>(value);
    else
      *static_cast<double*>(out) = value;
  }
};

struct DataSet {
  const std::vector<double>* data = nullptr;
  DataSpace getSpace() const {
    DataSpace s;
    s.extent = data->size();
    return s;
  }
  void read(void* out, const PredType& /*t*/) const {
    std::memcpy(out, data->data(), sizeof(double) * data->size());
  }
  void read(void* out, const PredType& /*t*/, const DataSpace& /*mem*/,
            const DataSpace& file) const {
    const hsize_t off = file.selected ? file.offset : 0;
    const hsize_t cnt = file.selected ? file.count : data->size();
    if (off + cnt > data->size()) throw std::runtime_error("H5 stand-in: read past the dataset");
    std::memcpy(out, data->data() + off, sizeof(double) * cnt);
  }
  void close() {}
};

struct H5File {
  const h5shim::File* file = nullptr;
  std::string name;
  H5File(const std::string& nm, unsigned /*flags*/) : name(nm) {
    auto it = h5shim::files().find(nm);
    if (it == h5shim::files().end()) throw std::runtime_error("H5 stand-in: no file " + nm);
    file = &it->second;
  }
  DataSet openDataSet(const std::string& ds) const {
    auto it = file->find(ds);
    if (it == file->end()) throw std::runtime_error("H5 stand-in: no dataset " + ds + " in " + name);
    DataSet d;
    d.data = &it->second;
    return d;
  }
  Attribute openAttribute(const std::string& a) const {
    if (a != "N") throw std::runtime_error("H5 stand-in: no attribute " + a);
    Attribute at;
    at.value = (double)openDataSet("En").data->size();
    return at;
  }
  void close() {}
};

}  // namespace H5
