/*
 * ref_driver.cpp -- C entry points into the reference's own tdse code.
 * TEST INFRASTRUCTURE ONLY.
 *
 * This translation unit compiles the reference's src/tdse/tdse.cpp in place
 * (it is #included from the reference tree by the recipe in oracle/Makefile,
 * never copied) together with the stand-in odeint and CBLAS headers under
 * ref_shim/.  It exposes:
 *   ref_rhs        - MatVecV / MatVecL::operator() (src/tdse/tdse.cpp:14-73,
 *                    :85-143) at a given field value;
 *   ref_propagate  - tdse::propV / propL (src/tdse/tdse.cpp:146-310) set up as
 *                    the reference's main does (src/tdse/tdse_main.cpp:162-192:
 *                    tau from the period, steps = int((tau - t0)/dt), CEP 0);
 *   ref_field      - the reference's pulse functions (src/tdse/pulse.cpp).
 */
#include "tdse.cpp"

#include <cstring>

extern "C" {
int refshim_override_field = 0;
double refshim_field = 0.0;
int refshim_capture = 0;
double *refshim_capture_buf = nullptr;
int refshim_set_blas(const char *path, int threads);
}

namespace {
struct Blocks {
  std::vector<int> state_sz, offs;
  stvupt eig, dip;
  int ct_sz = 0;
};

void load(Blocks &b, int L_max, const int *n, const double *eig,
          const double *dip) {
  b.offs.push_back(0);
  const double *e = eig;
  const double *d = dip;
  for (int L = 0; L <= L_max; ++L) {
    b.state_sz.push_back(n[L]);
    b.ct_sz += n[L];
    b.offs.push_back(b.ct_sz);
    b.eig.push_back(std::make_unique<std::vector<double>>(e, e + n[L]));
    e += n[L];
    if (L < L_max) {
      size_t sz = (size_t)n[L] * n[L + 1];
      b.dip.push_back(std::make_unique<std::vector<double>>(d, d + sz));
      d += sz;
    }
  }
}

template <class MV> void fill(MV &mv, Blocks &b, int L_max) {
  mv.L_max = L_max;
  mv.state_sz = b.state_sz;
  mv.offs = b.offs;
  for (int L = 0; L < L_max; ++L) {
    mv.eig.push_back(b.eig[L]->data());
    mv.dipole.push_back(b.dip[L]->data());
  }
  mv.eig.push_back(b.eig[L_max]->data());
}

void setup(int shape, char gauge, double Io_W, double w_eV, int cycles,
           double cepd, pulse::params &pars, fieldFcn &f) {
  double auIo, auw;
  pulse::toAU(Io_W, w_eV, auIo, auw);
  double tau = pulse::period(w_eV * conv::En_ev_au_, cycles);
  if (shape == 0) {
    if (gauge == 'v') { pulse::sineASetup(auIo, auw, cepd, cycles, pars); f = pulse::sineAA; }
    else { pulse::sineESetup(auIo, auw, cepd, cycles, pars); f = pulse::sineEE; }
  } else {
    if (gauge == 'v') pulse::gaussASetup(auIo, auw, tau, cycles, cepd, pars);
    else pulse::gaussESetup(auIo, auw, tau, cycles, cepd, pars);
    f = pulse::gauss;
  }
}
} // namespace

extern "C" {

int ref_set_blas(const char *path, int threads) {
  return refshim_set_blas(path, threads);
}

int ref_rhs(int L_max, const int *n, const double *eig, const double *dip,
            char gauge, double F, const double *x, double *dxdt) {
  Blocks b;
  load(b, L_max, n, eig, dip);
  std::vector<double> xs(x, x + 2 * b.ct_sz), out(2 * b.ct_sz);
  if (gauge == 'v') {
    MatVecV mv; fill(mv, b, L_max); mv.field = F; mv(xs, out, 0.0);
  } else {
    MatVecL mv; fill(mv, b, L_max); mv.field = F; mv(xs, out, 0.0);
  }
  std::memcpy(dxdt, out.data(), sizeof(double) * out.size());
  return 0;
}

/* Steps the reference's main would take (src/tdse/tdse_main.cpp:162-163). */
int ref_steps(double w_eV, int cycles, double t0, double dt) {
  double tau = pulse::period(w_eV * conv::En_ev_au_, cycles);
  int steps = (tau - t0) / dt;
  return steps;
}

double ref_field(int shape, char gauge, double Io_W, double w_eV, int cycles,
                 double cepd, double t) {
  pulse::params pars;
  fieldFcn f;
  setup(shape, gauge, Io_W, w_eV, cycles, cepd, pars, f);
  return f(pars, t);
}

/* Runs tdse::propV/propL for `steps` steps (steps >= 10, as the reference's
 * progress print divides by steps/10).  ct is in/out.  Files go to prefix. */
int ref_propagate(int L_max, const int *n, const double *eig, const double *dip,
                  char gauge, int shape, double Io_W, double w_eV, int cycles,
                  double t0, double dt, int steps, int pop_n, int pop_l,
                  const char *prefix, double *ct) {
  if (steps < 10) return -1;
  Blocks b;
  load(b, L_max, n, eig, dip);
  pulse::params pars;
  fieldFcn f;
  setup(shape, gauge, Io_W, w_eV, cycles, 0.0, pars, f);
  std::vector<double> c(ct, ct + 2 * b.ct_sz);
  refshim_override_field = 0;
  refshim_capture = 0;
  std::streambuf *old = std::cout.rdbuf(nullptr);
  if (gauge == 'v')
    tdse::propV(prefix, L_max, t0, dt, steps, pop_n, pop_l, f, pars, b.ct_sz,
                b.offs, b.state_sz, b.eig, b.dip, c);
  else
    tdse::propL(prefix, L_max, t0, dt, steps, pop_n, pop_l, f, pars, b.ct_sz,
                b.offs, b.state_sz, b.eig, b.dip, c);
  std::cout.rdbuf(old);
  std::memcpy(ct, c.data(), sizeof(double) * c.size());
  return 0;
}
}
