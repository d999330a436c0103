// yaml-cpp stand-in -- TEST INFRASTRUCTURE ONLY.  The checker calls the
// reference's pes::genPES1e / genPES2e directly with their arguments, never
// pes::readConfig, which is the one user of this API in src/pes/pes.cpp; the
// types exist so that the file compiles.
#pragma once
#include <stdexcept>
#include <string>

namespace YAML {
struct Node {
  Node operator[](const std::string&) const { return Node(); }
  template <class T>
  T as() const {
    throw std::runtime_error("yaml stand-in: configuration reading is not available");
  }
};
inline Node LoadFile(const std::string&) { return Node(); }
}  // namespace YAML
