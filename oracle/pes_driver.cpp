/*
 * pes_driver.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference's own src/pes/pes.cpp (pes::genPES1e, genPES2e,
 * src/pes/pes.cpp:48-262) as it lies in the reference tree, against the
 * stand-ins in ref_shim/ (H5Cpp.h: an in-memory file table; yaml-cpp and
 * lapacke: declarations only), and exposes one C entry point:
 *
 *   ref_pes  - fills the in-memory files the way the reference's inputs lie
 *              in dat/ (1e: <pot><l>.h5:/En per block; 2e: <pot>0.h5:/En
 *              holding the lowest 1e energy, and <pot>CI<L>.h5:/En_CI per
 *              block), then calls genPES1e / genPES2e on the coefficients.
 *              The spectra land in the reference's own output files
 *              (<prefix>_pes<L>.dat and, with s_flag, <prefix>_pes.dat);
 *              what it prints (ground population, norm, yield, excited
 *              population, 16 digits) is returned in `out`.
 */
#include "pes.cpp"

#include <sstream>

extern "C" int ref_pes(int electrons, int s_flag, int L_max, const int* state_sz,
                       const int* file_sz, const double* file_eig, double e0_1e,
                       const double* ct, const char* prefix, char* out, size_t outlen) {
  auto& files = h5shim::files();
  files.clear();
  const std::string pot = "mem";
  std::vector<int> sz(state_sz, state_sz + L_max + 1);
  long long ctsz = 0, off = 0;
  for (int L = 0; L <= L_max; ++L) {
    ctsz += sz[L];
    std::vector<double> e(file_eig + off, file_eig + off + file_sz[L]);
    off += file_sz[L];
    if (electrons == 1)
      files[pot + std::to_string(L) + ".h5"]["En"] = e;
    else
      files[pot + "CI" + std::to_string(L) + ".h5"]["En_CI"] = e;
  }
  if (electrons == 2) files[pot + "0.h5"]["En"] = std::vector<double>{e0_1e};
  std::vector<std::complex<double>> c(ctsz);
  for (long long i = 0; i < ctsz; ++i) c[i] = std::complex<double>(ct[2 * i], ct[2 * i + 1]);
  std::ostringstream cap;
  std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
  int rc = 0;
  try {
    if (electrons == 1)
      rc = pes::genPES1e(pot, s_flag != 0, L_max, sz, c, prefix);
    else
      rc = pes::genPES2e(pot, s_flag != 0, L_max, sz, c, prefix);
  } catch (const std::exception& e) {
    std::cout.rdbuf(old);
    std::snprintf(out, outlen, "error: %s", e.what());
    return -1;
  }
  std::cout.rdbuf(old);
  std::snprintf(out, outlen, "%s", cap.str().c_str());
  return rc;
}
