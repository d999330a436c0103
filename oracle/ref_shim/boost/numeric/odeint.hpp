/*
 * Stand-in for <boost/numeric/odeint.hpp> -- TEST INFRASTRUCTURE ONLY.
 *
 * boost is not installed here, so the reference's src/tdse/tdse.cpp is built
 * against this header instead.  It provides exactly the one type tdse.cpp
 * uses, runge_kutta_fehlberg78<state_type>, with the one call it makes,
 * do_step(sys, x, t, dt) (src/tdse/tdse.cpp:171,190,254,273): a single fixed
 * 13-stage step of Fehlberg's 7(8) pair, propagating the 8th-order solution,
 * with stage inputs summed x + (dt*a_s0)*k_0 + (dt*a_s1)*k_1 + ... left to
 * right.  The tableau is rkf78_tableau.h (Fehlberg, NASA TR R-287, 1968).
 *
 * Two hooks let the test driver reach the reference's own right-hand side:
 *   refshim_override_field: if set, the system's `field` member is replaced
 *     by refshim_field before the step;
 *   refshim_capture: if set, the step stores f(x) into refshim_capture_buf
 *     and leaves x unchanged.
 */
#ifndef REFSHIM_ODEINT_HPP_
#define REFSHIM_ODEINT_HPP_
#include <cstddef>
#include <memory> /* boost/odeint pulls this in; the reference relies on it */
#include <vector>

#include "../../../rkf78_tableau.h"

extern "C" {
extern int refshim_override_field;
extern double refshim_field;
extern int refshim_capture;
extern double *refshim_capture_buf;
}

namespace boost {
namespace numeric {
namespace odeint {

template <class State> class runge_kutta_fehlberg78 {
public:
  template <class System>
  void do_step(System &sys, State &x, double t, double dt) {
    const std::size_t m = x.size();
    for (int s = 0; s < 13; ++s) k_[s].resize(m);
    tmp_.resize(m);
    if (refshim_override_field) sys.field = refshim_field;
    sys(x, k_[0], t);
    if (refshim_capture) {
      for (std::size_t i = 0; i < m; ++i) refshim_capture_buf[i] = k_[0][i];
      return;
    }
    for (int s = 1; s < 13; ++s) {
      tmp_ = x;
      for (int e = 0; e < RKF78_NA; ++e) {
        if (RKF78_A[e].s != s) continue;
        const double c = dt * (RKF78_A[e].p / RKF78_A[e].q);
        const State &kj = k_[RKF78_A[e].j];
        for (std::size_t i = 0; i < m; ++i) tmp_[i] = tmp_[i] + c * kj[i];
      }
      sys(tmp_, k_[s], t + dt * (RKF78_C[s][0] / RKF78_C[s][1]));
    }
    tmp_ = x;
    for (int j = 0; j < 13; ++j) {
      const double b = RKF78_B8[j][0] / RKF78_B8[j][1];
      if (b == 0.0) continue;
      const double c = dt * b;
      for (std::size_t i = 0; i < m; ++i) tmp_[i] = tmp_[i] + c * k_[j][i];
    }
    x.swap(tmp_);
  }

private:
  State k_[13];
  State tmp_;
};

} // namespace odeint
} // namespace numeric
} // namespace boost
#endif
