// batch_types.h -- per-pulse column state of the batched propagation, shared
// by the streamed (batch.cu) and shared-memory-resident (batch_resident.cu)
// kernels, and the device-side pulse shapes they evaluate.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/mpc_tdse.h"

struct mpc_ctx;

namespace mpc {

// The field E(t) (or A(t)) of one pulse: pulse::sineEE / sineAA / sineAE /
// sineEA / gauss, src/tdse/pulse.cpp:10-97, zero outside the pulse.
__device__ inline double dev_field(const mpc_pulse& p, double t) {
  const double Eo = p.Eo, w = p.w, cepd = p.cepd, a = p.a, b = p.b;
  switch (p.kind) {
    case MPC_FIELD_SINE_EE:
    case MPC_FIELD_SINE_AA: {
      const double s = sin(a * t);
      return (double)(t >= 0.0 && t <= M_PI / a) * Eo * s * s * sin(w * t + cepd);
    }
    case MPC_FIELD_SINE_AE: {
      const double Wt = a * t, s = sin(Wt), wtc = w * t + cepd;
      return (double)(t >= 0.0 && t <= M_PI / a) * Eo *
             (w * s * s * cos(wtc) + a * sin(2 * Wt) * sin(wtc));
    }
    case MPC_FIELD_SINE_EA: {
      const double WpP = w + 2.0 * a, WpN = w - 2.0 * a;
      return (double)(t >= 0.0 && t <= M_PI / a) * 0.5 * Eo *
             (((1.0 - cos(w * t + cepd)) / w) -
              0.5 * ((1.0 - cos(WpP * t)) / WpP + (1.0 - cos(WpN * t)) / WpN));
    }
    case MPC_FIELD_GAUSS: {
      const double td = t - 0.5 * b;
      return (double)(t >= 0.0 && t <= b) * Eo * exp(-td * td / (a * a)) * sin(w * t + cepd);
    }
  }
  return 0.0;
}

// Per-pulse-column state.
struct ColState {
  mpc_pulse* pulse;
  double* t;
  double* t_end;
  double* h;       // proposed next step
  double* hatt;    // step of the current attempt
  int* last;       // the attempt ends the pulse
  int* done;
  int* accepted;   // 1 if the last attempt was accepted
  int* nacc;
  int* nrej;
  int* natt;
  int* pulse_id;   // column -> pulse index
  double* nrm;
  int* retired;    // set when the pulse finishes; cleared once its state is out
  int* nsteps;     // fixed-step mode: the pulse's step count
};

// Fixed-step mode (the reference's semantics, tdse::propV / propL,
// src/tdse/tdse.cpp:186-215): every attempt is one step of dt with the field
// F(t + dt) frozen for the 13 stages, always accepted unless the norm is not
// finite, then t += dt and x /= ||x||; a pulse retires after nsteps steps.
// Optional per-pulse histories (indexed by pulse id, rows hist_ld apart):
// pop_hist[id][k] = |x_k[pop_index]|^2 after step k (entry 0 is the host's),
// norm_hist[id][k-1] = ||x_new|| before the renormalisation of step k.
struct FixedStep {
  int on;
  double dt;
  int pop_index;
  long long hist_ld;
  double* pop_hist;
  double* norm_hist;
};

// Per-pulse results, indexed by pulse id (columns move; these do not).
struct PulseResults {
  int* nacc;
  int* nrej;
  double* t;
  int* status;     // 0 finished at t_end, 2 gave up after max_attempts
};

// Arguments of one persistent launch of the resident batched kernel.
struct BatchResLaunch {
  ColState c;
  PulseResults res;
  double2* X;       // current (normalised) states [n][ldc]
  double2* XN;      // candidate x_new [n][ldc]
  double2* Y0;      // stage inputs, ping-pong [n][ldc]
  double2* Y1;
  double2* out;     // final states [pulse][n]
  int ldc;
  int ncol;
  int max_attempts;
  double rtol, atol, dt_max;
  FixedStep fx;
};

}  // namespace mpc

// Largest pulse count (1, 2, 4 or 8) the resident batched kernel takes for
// this context, or 0 when the system's coupling does not fit on chip.
int mpc_batch_res_pmax(mpc_ctx* c);
// Runs attempts of the ncol <= P active columns until every one is done or
// fewer than `exit_below` remain active.
int mpc_batch_res_run(mpc_ctx* c, const mpc::BatchResLaunch& l, int P, int exit_below);
void mpc_batch_res_free(mpc_ctx* c);
