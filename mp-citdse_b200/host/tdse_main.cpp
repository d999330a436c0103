// tdse_main.cpp -- drop-in `tdse` executable: the reference's command line,
// input files and output files, with the propagation on the GPU through
// libmpc_tdse.so.
//
// Mirrors src/tdse/tdse_main.cpp (flags :25-66, settings copy and overwrite
// prompt :70-94, 1e/2e file names :96-128, ground or restart start :148-160,
// step count :162-163, pulse choice :166-198), tdrd::readConfig /
// readEnergies / readDipoles / readInitCt (src/tdse/td_read.cpp:3-143) and the
// file output of tdse::propV / propL (src/tdse/tdse.cpp:150-222): the same
// names, headers, number formats and 10 % checkpoints.  Differences: fewer
// than 10 steps does not divide by zero (dumps every step); an unknown gauge
// or missing -e is reported instead of silently doing nothing.
// Addition: -p also writes every coefficient dump as <pot>_ct_<t>.h5
// (datasets "ct" [size x 2] and "t" [1], full float64), and -s accepts such a
// file: a restart from it continues bit for bit, where the 6-digit text dump
// and the time parsed from its file name lose precision.
#include <getopt.h>
#include <unistd.h>

#include <cmath>
#include <complex>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mpc_tdse.h"
#include "h5lite.hpp"
#include "yaml_lite.hpp"

namespace {

// A named region on a profiler's timeline (load / propagate / output).
struct Range {
  bool open = true;
  explicit Range(const char* name) { nvtxRangePushA(name); }
  void end() {
    if (open) nvtxRangePop();
    open = false;
  }
  ~Range() { end(); }
};

constexpr double kEvAu = 1. / 27.211396181;  // conv::En_ev_au_ (src/include/au.hpp:30-31)

struct Config {
  std::string pot;
  int L_max = 0;
  char gauge = 'v';
  std::vector<int> state_sz;
  double dt = 0.0;
  std::string shape;
  double w = 0.0, Io = 0.0, cepd = 0.0;
  int cycles = 0;
};

Config read_config(const std::string& file, const std::string& base, const std::string& option) {
  const yl::Doc y = yl::Doc::load(file);
  Config c;
  std::cout << "Global Settings:" << std::endl;
  c.pot = y.str("Global_Settings", "potential");
  std::cout << "  Core Potential:                       " << c.pot << std::endl;
  c.L_max = y.integer(base, option);
  std::cout << "  max l/L:                              " << c.L_max << std::endl;
  const std::string g = y.str("Global_Settings", "gauge");
  if (g.size() != 1) throw yl::Error("yaml: gauge must be one character");
  c.gauge = g[0];
  std::cout << "  Gauge type ('l' length/'v' velocity): " << c.gauge << std::endl;
  std::cout << "Propagator Settings:" << std::endl;
  c.state_sz = y.int_list("Propagator_Settings", "states_in_l");
  if ((int)c.state_sz.size() != c.L_max + 1)
    throw yl::Error("yaml: states_in_l must have L_max + 1 entries");
  std::cout << "  states per l/L:          ";
  for (int v : c.state_sz) std::cout << v << " ";
  std::cout << std::endl;
  c.dt = y.num("Propagator_Settings", "dt");
  std::cout << "  timestep dt:                          " << c.dt << std::endl;
  std::cout << "Field Parameters:" << std::endl;
  c.shape = y.str("Field_Parameters", "shape");
  std::cout << "  envelope shape:                       " << c.shape << std::endl;
  c.w = y.num("Field_Parameters", "w");
  std::cout << "  photon energy:                        " << c.w << std::endl;
  c.Io = y.num("Field_Parameters", "Io");
  std::cout << "  Peak intensity:                       " << c.Io << std::endl;
  c.cepd = y.num("Field_Parameters", "cepd");
  std::cout << "  phase shift:                          " << c.cepd << std::endl;
  c.cycles = y.integer("Field_Parameters", "cycles");
  std::cout << "  number of cycles:                     " << c.cycles << std::endl;
  return c;
}

void write_ct(const std::string& prefix, double t, const std::vector<double>& ct) {
  std::fstream f(prefix + "_ct_" + std::to_string(t) + ".dat", std::ios::out);
  f << "#Index, Re(c(t)), Im(c(t))\n";
  for (size_t k = 0; k < ct.size(); k += 2) f << k / 2 << "  " << ct[k] << "  " << ct[k + 1] << "\n";
}

// Full-precision dump: the coefficients and the exact time.
void write_ct_h5(const std::string& prefix, double t, const std::vector<double>& ct) {
  const uint64_t n = ct.size() / 2;
  h5::write(prefix + "_ct_" + std::to_string(t) + ".h5",
            {{"ct", {n, 2}, ct.data()}, {"t", {1}, &t}});
}

bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

// tdrd::readInitCt: lines of "index re im", leading blanks and # lines skipped
void read_init_ct(const std::string& file, int ct_sz, std::vector<double>& ct) {
  std::ifstream fl(file);
  if (!fl) throw std::runtime_error("cannot open " + file);
  std::string temp;
  int i = 0;
  while (i < ct_sz * 2) {
    if (!std::getline(fl, temp)) throw std::runtime_error(file + ": too few coefficients");
    temp = std::regex_replace(temp, std::regex("^ +"), "");
    if (!temp.empty() && temp[0] == '#') continue;
    std::istringstream iss(temp);
    int idx;
    double re, im;
    iss >> idx >> re >> im;
    ct[i] = re;
    ct[i + 1] = im;
    i += 2;
  }
}

int check(int rc) {
  if (rc != MPC_OK) {
    char msg[1024];
    mpc_last_error(msg, sizeof msg);
    throw std::runtime_error(std::string("libmpc_tdse: ") + msg);
  }
  return rc;
}

int run(int argc, char* argv[]) {
  std::string opt_file, out_dir, init_ct = "ground";
  int e_num = 0, pop_n = 0, pop_l = 0;
  bool h5_dumps = false;
  for (;;) {
    switch (getopt(argc, argv, "he:f:o:s:n:l:p")) {
      case 'h':
        std::cout << "Program for propagating either the 1- or 2-e^- tdse\n"
                  << "-e <1 or 2> the number of electrons in the tdse\n"
                  << "-f <path> yaml input file with the input settings\n"
                  << "-o <path> output directory for the coefficient files\n"
                  << "-s <path> file with the start coefficients\n"
                  << "-n <int> primary quantum number of state to track\n"
                  << "-l <int> angular quantum number of state to track\n"
                  << "-p also write full-precision <pot>_ct_<t>.h5 dumps (-s accepts them)\n";
        return -1;
      case 'e':
        e_num = std::stoi(optarg);
        if (e_num != 1 && e_num != 2) {
          std::cout << "Invalid number of electrons, use 1 or 2\n";
          return -1;
        }
        continue;
      case 'f': opt_file = optarg; continue;
      case 'o': out_dir = optarg; continue;
      case 's': init_ct = optarg; continue;
      case 'n':
        pop_n = std::stoi(optarg);
        if (pop_n < 1) {
          std::cout << "Invalid primary quantum number -n, use int > 0\n";
          return -1;
        }
        --pop_n;
        continue;
      case 'l': pop_l = std::stoi(optarg); continue;
      case 'p': h5_dumps = true; continue;
    }
    break;
  }
  if (e_num == 0) {
    std::cout << "Invalid number of electrons, use 1 or 2\n";
    return -1;
  }
  namespace fs = std::filesystem;
  if (!fs::exists(out_dir)) fs::create_directory(out_dir);
  const std::string set_file = out_dir + "/settings.yaml";
  fs::copy_options cpopt = fs::copy_options::none;
  if (fs::exists(set_file) && init_ct == "ground") {
    char ovw = 'n';
    std::cout << "File " << set_file << " exists. Overwrite? [y/n]\n";
    std::cin >> ovw;
    if (ovw == 'y') {
      cpopt = fs::copy_options::update_existing;
    } else {
      std::cout << out_dir << " contians old data, please choose a different output"
                << " directory!\n";
      return -1;
    }
  }
  fs::copy_file(opt_file, set_file, cpopt);
  const std::string base = (e_num == 1) ? "Basis_Settings" : "Global_Settings";
  const std::string option = (e_num == 1) ? "l_max" : "L_max";
  const Config cf = read_config(opt_file, base, option);
  std::string en_pot, en_set, dip_pot, dip_set;
  if (e_num == 1) {
    en_pot = "dat/" + cf.pot;
    en_set = "En";
    dip_pot = "dat/" + cf.pot;
    dip_set = "d_if";
  } else {
    en_pot = "dat/" + cf.pot + "CI";
    en_set = "En_CI";
    dip_pot = "dat/" + cf.pot + "CI_";
    dip_set = "CI_dip";
    for (int L = 0; L <= cf.L_max; ++L)
      fs::copy_file("dat/cfg-" + std::to_string(L) + ".inp",
                    out_dir + "/cfg-" + std::to_string(L) + ".inp", cpopt);
  }
  const std::string prefix = out_dir + "/" + cf.pot;
  if (cf.gauge != 'l' && cf.gauge != 'v') {
    std::cout << "Invalid gauge, use 'l' or 'v'\n";
    return -1;
  }
  if (cf.shape != "sine" && cf.shape != "gaussian") {
    std::cout << "Invalid envelope shape, use \"sine\" or \"gaussian\"\n";
    return -1;
  }

  // tdrd::readEnergies / readDipoles: the top-left state_sz blocks
  std::vector<int> offs{0};
  std::vector<double> eig, dip;
  Range load_range("tdse: load inputs");
  for (int L = 0; L <= cf.L_max; ++L) {
    const auto e = h5::read_block(en_pot + std::to_string(L) + ".h5", en_set, cf.state_sz[L], 0);
    eig.insert(eig.end(), e.begin(), e.end());
    offs.push_back(offs.back() + cf.state_sz[L]);
  }
  for (int L = 0; L < cf.L_max; ++L) {
    const auto d = h5::read_block(dip_pot + std::to_string(L) + std::to_string(L + 1) + cf.gauge + ".h5",
                                  dip_set, cf.state_sz[L], cf.state_sz[L + 1]);
    dip.insert(dip.end(), d.begin(), d.end());
  }
  const int ct_sz = offs.back();
  std::vector<double> ct(2 * (size_t)ct_sz, 0.0);
  ct[0] = 1.0;
  double t = 0.0;
  if (init_ct != "ground" && ends_with(init_ct, ".h5")) {
    const h5::Dataset c = h5::read(init_ct, "ct");
    const h5::Dataset tt = h5::read(init_ct, "t");
    if (c.dims.size() != 2 || c.dims[1] != 2 || c.dims[0] < (uint64_t)ct_sz || tt.data.empty())
      throw std::runtime_error(init_ct + ": expected ct [>= " + std::to_string(ct_sz) +
                               " x 2] and t");
    std::copy(c.data.begin(), c.data.begin() + 2 * (size_t)ct_sz, ct.begin());
    t = tt.data[0];
    std::cout << "Start time (a.u.): " << t << "\n";
  } else if (init_ct != "ground") {
    const std::string fln = fs::path(init_ct).filename();
    const auto t_start = fln.find_first_of("0123456789");
    t = std::stod(fln.substr(t_start));
    std::cout << "Start time (a.u.): " << t << "\n";
    read_init_ct(init_ct, ct_sz, ct);
  }
  load_range.end();
  const double tau = mpc_period(cf.w * kEvAu, cf.cycles);
  const int steps = (tau - t) / cf.dt;
  double auIo, auw;
  check(mpc_to_au(cf.Io, cf.w, &auIo, &auw));
  mpc_pulse pulse;
  check(mpc_pulse_setup(cf.shape == "sine" ? 0 : 1, cf.gauge, auIo, auw, 0.0, cf.cycles, tau, &pulse));

  int device = 0;
  if (const char* d = std::getenv("MPC_DEVICE")) device = std::atoi(d);
  mpc_ctx* ctx = nullptr;
  check(mpc_ctx_create(cf.L_max, cf.state_sz.data(), eig.data(), dip.data(), cf.gauge, device, &ctx));
  const int pop_index = offs[pop_l] + pop_n;

  // output of tdse::propV / propL (src/tdse/tdse.cpp:150-222)
  const int print = steps / 10 > 0 ? steps / 10 : 1;
  write_ct(prefix, t, ct);
  if (h5_dumps) write_ct_h5(prefix, t, ct);
  std::fstream field_fl(prefix + "_field.dat", std::ios::out);
  field_fl << "#time (a.u.), field (A(t) or E(t)) (a.u.)\n";
  std::fstream f_pop(prefix + "_pop" + std::to_string(pop_n + 1) + std::to_string(pop_l) + ".dat",
                     std::ios::out);
  f_pop << "#time (a.u.), population\n";
  f_pop << std::setprecision(16) << t << " "
        << std::norm(std::complex<double>(ct[2 * pop_index], ct[2 * pop_index + 1])) << "\n";
  check(mpc_state_set(ctx, ct.data()));
  std::vector<double> pop, fld;
  int st = 0;
  while (st < steps) {
    const int n = (st == 0) ? 1 : std::min(print, steps - st);
    {
      Range r("tdse: propagate");
      check(mpc_advance(ctx, &pulse, t, cf.dt, n, pop_index));
    }
    Range out_range("tdse: output");
    pop.resize(n + 1);
    fld.resize(n);
    check(mpc_history_get(ctx, n, pop.data(), fld.data(), nullptr));
    for (int j = 0; j < n; ++j) {
      field_fl << t + cf.dt << " " << fld[j] << "\n";
      t += cf.dt;
      f_pop << std::setprecision(16) << t << " " << pop[j + 1] << "\n";
    }
    st += n;
    if ((st - 1) % print == 0) {
      std::cout << fld[n - 1] << "\n";
      check(mpc_state_get(ctx, ct.data()));
      write_ct(prefix, t, ct);
      if (h5_dumps) write_ct_h5(prefix, t, ct);
    }
  }
  check(mpc_state_get(ctx, ct.data()));
  write_ct(prefix, t, ct);
  if (h5_dumps) write_ct_h5(prefix, t, ct);
  mpc_ctx_destroy(ctx);
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  try {
    return run(argc, argv);
  } catch (const std::exception& e) {
    std::cerr << "tdse: " << e.what() << "\n";
    return -1;
  }
}
