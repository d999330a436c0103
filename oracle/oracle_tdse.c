/*
 * oracle_tdse.c -- CPU restatement of MP-CITDSE's `tdse` propagation.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py).  Nothing in the product library links or calls it.
 *
 * What it restates (paths relative to the MP-CITDSE source tree):
 *   - the right-hand side dc/dt of the velocity gauge, MatVecV::operator()
 *     src/tdse/tdse.cpp:14-73, and of the length gauge, MatVecL::operator()
 *     src/tdse/tdse.cpp:85-143.  The four strided dgemv calls per dipole
 *     block are restated with the same operand orientation (column-major view
 *     of the row-major [n_L x n_{L+1}] block, lda = n_{L+1}), the same alpha
 *     signs, the same beta (0 for the L-1 coupling, 1 for the L+1 coupling)
 *     and the same order of the diagonal update;
 *   - one fixed step of boost::odeint's runge_kutta_fehlberg78 called as
 *     rkf.do_step(sys, x, t, dt) (src/tdse/tdse.cpp:171,190): 13 stages, the
 *     8th-order weights, no error estimate.  odeint is not vendored by the
 *     reference; its published algorithm is Fehlberg's 7(8) pair (NASA TR
 *     R-287, 1968), whose tableau is restated below.  Stage inputs are summed
 *     as x + (dt*a_s0)*k_0 + (dt*a_s1)*k_1 + ... left to right;
 *   - the step loop of tdse::propV / tdse::propL (src/tdse/tdse.cpp:186-215,
 *     :269-298): the field F(t+dt) is frozen for the whole step, then
 *     t += dt, then c /= ||c||_2 (cblas_dznrm2, :194-198), then the tracked
 *     population |c_k|^2 (:200-204);
 *   - the pulse shapes and set-up routines of src/tdse/pulse.cpp:3-97 and the
 *     unit constants of src/include/au.hpp:30-32, and the step count of
 *     src/tdse/tdse_main.cpp:162-163.
 *
 * What it adds that the reference does not have (own semantics, used to check
 * the new GPU modes): an adaptive RKF78 driver with the embedded 7th-order
 * error estimate and a per-pulse step controller, a per-stage ("continuous")
 * field mode, a piecewise-cubic control perturbation of E(t), and the discrete
 * adjoint of the fixed-step propagation.
 *
 * Arithmetic note: built with -ffp-contract=off so that every product and sum
 * is rounded separately; results are compared against the GPU within the
 * tolerances written in the tests, not bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXB 64
#define NST 13
#include "rkf78_tableau.h"

/* ------------------------------------------------------------------------ */
/* Fehlberg 7(8) tableau (NASA TR R-287, 1968).                              */
/* ------------------------------------------------------------------------ */
static double RK_A[NST][NST];
static double RK_B8[NST], RK_B7[NST], RK_C[NST];
static int rk_ready = 0;

static void rk_init(void) {
  if (rk_ready) return;
  memset(RK_A, 0, sizeof RK_A);
  for (int s = 0; s < NST; ++s) RK_C[s] = RKF78_C[s][0] / RKF78_C[s][1];
  for (int e = 0; e < RKF78_NA; ++e)
    RK_A[RKF78_A[e].s][RKF78_A[e].j] = RKF78_A[e].p / RKF78_A[e].q;
  for (int s = 0; s < NST; ++s) {
    RK_B8[s] = RKF78_B8[s][0] / RKF78_B8[s][1];
    RK_B7[s] = RKF78_B7[s][0] / RKF78_B7[s][1];
  }
  rk_ready = 1;
}

/* Exported for tests: copy the tableau out (A row-major 13x13, b8, b7, c). */
void orc_tableau(double *A, double *b8, double *b7, double *c) {
  rk_init();
  memcpy(A, RK_A, sizeof RK_A);
  memcpy(b8, RK_B8, sizeof RK_B8);
  memcpy(b7, RK_B7, sizeof RK_B7);
  memcpy(c, RK_C, sizeof RK_C);
}

/* ------------------------------------------------------------------------ */
/* Optional external CBLAS (e.g. OpenBLAS) for the timed CPU baseline.       */
/* ------------------------------------------------------------------------ */
typedef void (*cblas_dgemv_fn)(int, int, int, int, double, const double *, int,
                               const double *, int, double, double *, int);
typedef double (*cblas_dznrm2_fn)(int, const void *, int);
static cblas_dgemv_fn ext_dgemv = NULL;
static cblas_dznrm2_fn ext_dznrm2 = NULL;

void orc_use_blas(void *dgemv_fn, void *dznrm2_fn) {
  ext_dgemv = (cblas_dgemv_fn)dgemv_fn;
  ext_dznrm2 = (cblas_dznrm2_fn)dznrm2_fn;
}

/* y := alpha*op(A)*x + beta*y with A column-major MxN (BLAS dgemv semantics,
 * beta restricted to 0 or 1 as the reference uses it).  op = A (trans=0) or
 * A^T (trans=1). */
static void dgemv_cm(int trans, int M, int N, double alpha, const double *A,
                     int lda, const double *x, int incx, double beta,
                     double *y, int incy) {
  if (ext_dgemv) {
    ext_dgemv(102, trans ? 112 : 111, M, N, alpha, A, lda, x, incx, beta, y,
              incy);
    return;
  }
  if (!trans) {
    for (int i = 0; i < M; ++i) {
      double acc = 0.0;
      for (int j = 0; j < N; ++j) acc += A[(size_t)j * lda + i] * x[(size_t)j * incx];
      double *yi = &y[(size_t)i * incy];
      *yi = (beta == 0.0) ? alpha * acc : *yi + alpha * acc;
    }
  } else {
    for (int j = 0; j < N; ++j) {
      const double *col = &A[(size_t)j * lda];
      double acc = 0.0;
      for (int i = 0; i < M; ++i) acc += col[i] * x[(size_t)i * incx];
      double *yj = &y[(size_t)j * incy];
      *yj = (beta == 0.0) ? alpha * acc : *yj + alpha * acc;
    }
  }
}

static double znrm2(int n, const double *x) {
  if (ext_dznrm2) return ext_dznrm2(n, x, 1);
  double s = 0.0;
  for (int i = 0; i < 2 * n; ++i) s += x[i] * x[i];
  return sqrt(s);
}

/* ------------------------------------------------------------------------ */
/* The blocked system.                                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
  int L_max;
  int n[ORC_MAXB];
  int offs[ORC_MAXB + 1];
  int ntot;
  const double *eig;               /* flat, ntot */
  const double *dip[ORC_MAXB];     /* block L: row-major n[L] x n[L+1] */
  char gauge;
} sys_t;

static int sys_init(sys_t *s, int L_max, const int *n, const double *eig,
                    const double *dip, char gauge) {
  if (L_max < 1 || L_max >= ORC_MAXB) return -1;
  if (gauge != 'l' && gauge != 'v') return -2;
  s->L_max = L_max;
  s->gauge = gauge;
  s->offs[0] = 0;
  for (int L = 0; L <= L_max; ++L) {
    if (n[L] <= 0) return -3;
    s->n[L] = n[L];
    s->offs[L + 1] = s->offs[L] + n[L];
  }
  s->ntot = s->offs[L_max + 1];
  s->eig = eig;
  size_t o = 0;
  for (int L = 0; L < L_max; ++L) {
    s->dip[L] = dip + o;
    o += (size_t)n[L] * n[L + 1];
  }
  return 0;
}

/* dxdt = f(x) with the field frozen at F.  Follows MatVecV::operator()
 * (src/tdse/tdse.cpp:14-73) for gauge 'v' and MatVecL::operator()
 * (src/tdse/tdse.cpp:85-143) for gauge 'l'.
 *
 * Wiring of the coupling terms per gauge (component 0 = Re, 1 = Im):
 *   velocity: Re <- Re and Im <- Im, alpha = +F from block L-1 (NoTrans on
 *             D_{L-1}) and alpha = -F from block L+1 (Trans on D_L);
 *   length:   Im <- Re with alpha = -F, Re <- Im with alpha = +F, for both
 *             neighbours. */
static void rhs(const sys_t *s, double F, const double *x, double *dxdt) {
  const int Lm = s->L_max;
  int dst[2], src[2];
  double a_lo[2], a_up[2];
  if (s->gauge == 'v') {
    dst[0] = 0; src[0] = 0; a_lo[0] = F; a_up[0] = -F;
    dst[1] = 1; src[1] = 1; a_lo[1] = F; a_up[1] = -F;
  } else {
    dst[0] = 1; src[0] = 0; a_lo[0] = -F; a_up[0] = -F;
    dst[1] = 0; src[1] = 1; a_lo[1] = F;  a_up[1] = F;
  }
  for (int L = 0; L <= Lm; ++L) {
    const int o = 2 * s->offs[L];
    const int nl = s->n[L];
    const double *e = s->eig + s->offs[L];
    if (L > 0) {
      /* D_{L-1}^T x_{L-1} -> block L (cblas NoTrans, beta = 0) */
      const int om = 2 * s->offs[L - 1];
      for (int p = 0; p < 2; ++p)
        dgemv_cm(0, nl, s->n[L - 1], a_lo[p], s->dip[L - 1], nl,
                 &x[om + src[p]], 2, 0.0, &dxdt[o + dst[p]], 2);
      for (int i = 0; i < nl; ++i) {
        const int i2 = o + 2 * i;
        dxdt[i2 + 1] = -e[i] * x[i2] + dxdt[i2 + 1];
        dxdt[i2] = e[i] * x[i2 + 1] + dxdt[i2];
      }
    } else {
      for (int i = 0; i < nl; ++i) {
        const int i2 = o + 2 * i;
        dxdt[i2 + 1] = -e[i] * x[i2];
        dxdt[i2] = e[i] * x[i2 + 1];
      }
    }
    if (L < Lm) {
      /* D_L x_{L+1} -> block L (cblas Trans, beta = 1) */
      const int op = 2 * s->offs[L + 1];
      for (int p = 0; p < 2; ++p)
        dgemv_cm(1, s->n[L + 1], nl, a_up[p], s->dip[L], s->n[L + 1],
                 &x[op + src[p]], 2, 1.0, &dxdt[o + dst[p]], 2);
    }
  }
}

/* Stage input y = x + sum_j (h*a_j)*k_j, left to right, zero terms skipped
 * (adding 0*k_j leaves a finite sum unchanged). */
static void stage_sum(int m, const double *x, double *const *k,
                      const double *coef, double h, double *y) {
  for (int i = 0; i < m; ++i) y[i] = x[i];
  for (int j = 0; j < NST; ++j) {
    if (coef[j] == 0.0) continue;
    const double c = h * coef[j];
    const double *kj = k[j];
    for (int i = 0; i < m; ++i) y[i] = y[i] + c * kj[i];
  }
}

typedef struct {
  double *k[NST];
  double *y;
  double *buf;
} work_t;

static int work_alloc(work_t *w, int m) {
  w->buf = (double *)malloc(sizeof(double) * (size_t)m * (NST + 1));
  if (!w->buf) return -1;
  for (int s = 0; s < NST; ++s) w->k[s] = w->buf + (size_t)s * m;
  w->y = w->buf + (size_t)NST * m;
  return 0;
}

/* Fields per stage: Fs[s] for s = 0..12. */
static void rk78_stages(const sys_t *s, const double *Fs, double h,
                        const double *x, work_t *w) {
  const int m = 2 * s->ntot;
  rhs(s, Fs[0], x, w->k[0]);
  for (int st = 1; st < NST; ++st) {
    stage_sum(m, x, w->k, RK_A[st], h, w->y);
    rhs(s, Fs[st], w->y, w->k[st]);
  }
}

/* ------------------------------------------------------------------------ */
/* Pulses: src/tdse/pulse.cpp:3-97, src/include/au.hpp:30-32.                */
/* kind: 0 sineEE, 1 sineAA, 2 sineAE, 3 sineEA, 4 gauss.                    */
/* pars: {Eo, w, cepd, a, b} as pulse::params (src/tdse/include/pulse.hpp:20)*/
/* ------------------------------------------------------------------------ */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

void orc_units(double *ev_au, double *wcm2_au) {
  *ev_au = 1. / 27.211396181;
  *wcm2_au = (1. / 3.509338) * 1.e-16;
}

double orc_period(double w, int cycles) { return cycles * 2.0 * M_PI / w; }

/* shape: 0 sine (E- or A-defined per gauge), 1 gaussian.  gauge 'l' sets up
 * an E-defined pulse, 'v' an A-defined one (src/tdse/tdse_main.cpp:166-192).
 * Io, w in atomic units. */
void orc_pulse_setup(int shape, char gauge, double Io, double w, double cepd,
                     int cycles, double tau, double *pars) {
  double Eo = (gauge == 'v') ? sqrt(Io) / w : sqrt(Io);
  if (shape == 0) {
    pars[0] = Eo;
    pars[1] = w;
    pars[2] = (gauge == 'v') ? cepd * (2.0 * M_PI / w) : cepd * (2 * M_PI / w);
    pars[3] = w / (2.0 * cycles);
    pars[4] = 0.0;
  } else {
    const double width = 0.58870501125773734549;
    double To = 2 * M_PI / w;
    int cycles_fwhm = 2 + (int)(cycles / 10);
    pars[0] = Eo;
    pars[1] = w;
    pars[2] = cepd;
    pars[3] = 0.5 * To * cycles_fwhm / width;
    pars[4] = tau;
  }
}

double orc_field(int kind, const double *p, double t) {
  const double Eo = p[0], w = p[1], cepd = p[2], a = p[3], b = p[4];
  switch (kind) {
  case 0: /* sineEE */
  case 1: { /* sineAA */
    double sinWt = sin(a * t);
    return (double)(t >= 0.0 && t <= M_PI / a) * Eo * sinWt * sinWt *
           sin(w * t + cepd);
  }
  case 2: { /* sineAE */
    double Wt = a * t;
    double sinWt = sin(Wt);
    double wtc = w * t + cepd;
    return (double)(t >= 0.0 && t <= M_PI / a) * Eo *
           (w * sinWt * sinWt * cos(wtc) + a * sin(2 * Wt) * sin(wtc));
  }
  case 3: { /* sineEA */
    double WpP = w + 2.0 * a;
    double WpN = w - 2.0 * a;
    return (double)(t >= 0.0 && t <= M_PI / a) * 0.5 * Eo *
           (((1.0 - cos(w * t + cepd)) / w) -
            0.5 * ((1.0 - cos(WpP * t)) / WpP + (1.0 - cos(WpN * t)) / WpN));
  }
  case 4: { /* gauss */
    double td = t - 0.5 * b;
    return (double)(t >= 0.0 && t <= b) * Eo * exp(-td * td / (a * a)) *
           sin(w * t + cepd);
  }
  }
  return 0.0;
}

/* ------------------------------------------------------------------------ */
/* Piecewise-cubic control perturbation (own semantics, no reference).       */
/* dE(t) = sum_k u_k * phi((t - t_k)/g), t_k = k*g, g = T/(K-1), with phi the */
/* Catmull-Rom (Keys a = -1/2) cubic convolution kernel; samples outside     */
/* [0, K-1] are zero.                                                        */
/* ------------------------------------------------------------------------ */
static double keys_phi(double s) {
  double x = fabs(s);
  if (x < 1.0) return (1.5 * x - 2.5) * x * x + 1.0;
  if (x < 2.0) return ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0;
  return 0.0;
}

double orc_control_eval(int K, const double *u, double T, double t) {
  if (K < 2 || t < 0.0 || t > T) return 0.0;
  const double g = T / (double)(K - 1);
  const double q = t / g;
  int i0 = (int)floor(q);
  double acc = 0.0;
  for (int k = i0 - 1; k <= i0 + 2; ++k) {
    if (k < 0 || k >= K) continue;
    acc += u[k] * keys_phi(q - (double)k);
  }
  return acc;
}

/* weights w[0..3] and first index of the 4 samples that shape dE(t) */
static int control_weights(int K, double T, double t, double *wts) {
  const double g = T / (double)(K - 1);
  const double q = t / g;
  int i0 = (int)floor(q);
  for (int j = 0; j < 4; ++j) {
    int k = i0 - 1 + j;
    wts[j] = (t < 0.0 || t > T || k < 0 || k >= K) ? 0.0 : keys_phi(q - (double)k);
  }
  return i0 - 1;
}

/* ------------------------------------------------------------------------ */
/* Exported entry points.                                                    */
/* ------------------------------------------------------------------------ */

/* One right-hand-side evaluation (MatVecV/MatVecL::operator()).
 * eig: flat [ntot]; dip: blocks back to back, each row-major n[L] x n[L+1];
 * x, dxdt: interleaved complex [2*ntot]. */
int orc_rhs(int L_max, const int *n, const double *eig, const double *dip,
            char gauge, double F, const double *x, double *dxdt) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  rhs(&s, F, x, dxdt);
  return 0;
}

/* One rkf.do_step(sys, x, t, dt) with the field frozen at F (in place). */
int orc_rk78_step(int L_max, const int *n, const double *eig,
                  const double *dip, char gauge, double F, double dt,
                  double *x) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  rk_init();
  work_t w;
  const int m = 2 * s.ntot;
  if (work_alloc(&w, m)) return -10;
  double Fs[NST];
  for (int i = 0; i < NST; ++i) Fs[i] = F;
  rk78_stages(&s, Fs, dt, x, &w);
  stage_sum(m, x, w.k, RK_B8, dt, w.y);
  memcpy(x, w.y, sizeof(double) * m);
  free(w.buf);
  return 0;
}

/* The propagation loop of tdse::propV/propL (src/tdse/tdse.cpp:186-215).
 * field_kind / pars: pulse (see orc_field).  If K > 0 the field is
 * F = base(t) + dE(t) with the control perturbation of K samples u over
 * [0, T].  pop_index: flat index of the tracked coefficient.  Outputs (each
 * optional): pop_out[steps+1] (|c|^2 at t0 and after every step),
 * field_out[steps], norm_out[steps] (norm before renormalisation). */
int orc_propagate(int L_max, const int *n, const double *eig,
                  const double *dip, char gauge, int field_kind,
                  const double *pars, int K, const double *u, double T,
                  double t0, double dt, int steps, int pop_index, double *x,
                  double *pop_out, double *field_out, double *norm_out) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  rk_init();
  work_t w;
  const int m = 2 * s.ntot;
  if (work_alloc(&w, m)) return -10;
  double t = t0;
  const int pi2 = 2 * pop_index;
  if (pop_out) pop_out[0] = x[pi2] * x[pi2] + x[pi2 + 1] * x[pi2 + 1];
  double Fs[NST];
  for (int st = 0; st < steps; ++st) {
    double F = orc_field(field_kind, pars, t + dt);
    if (K > 0) F += orc_control_eval(K, u, T, t + dt);
    if (field_out) field_out[st] = F;
    for (int i = 0; i < NST; ++i) Fs[i] = F;
    rk78_stages(&s, Fs, dt, x, &w);
    stage_sum(m, x, w.k, RK_B8, dt, w.y);
    memcpy(x, w.y, sizeof(double) * m);
    t += dt;
    double nrm = znrm2(s.ntot, x);
    for (int i = 0; i < m; ++i) x[i] /= nrm;
    if (norm_out) norm_out[st] = nrm;
    if (pop_out) pop_out[st + 1] = x[pi2] * x[pi2] + x[pi2 + 1] * x[pi2 + 1];
  }
  free(w.buf);
  return 0;
}

/* Adaptive RKF78 (own semantics).  Per attempted step of size h:
 *   stage fields F_s = field(t + c_s h)   (field_mode 1, continuous) or
 *                F_s = field(t + h)        (field_mode 0, frozen as the
 *                                           reference's fixed-step loop);
 *   x_new = x + sum (h*b8_j) k_j;  e = sum (h*(b8_j-b7_j)) k_j;
 *   err = max_i |e_i| / (atol + rtol*max(|x_i|, |x_new_i|))  (complex moduli);
 *   accept if err <= 1: t += h (t = t_end on the final step), x = x_new/||x_new||;
 *   factor = safety * err^(-1/8) clamped to [facmin, facmax] (facmax if
 *   err == 0), with err^(-1/8) computed as 1/sqrt(sqrt(sqrt(err))); the next
 *   h = min(h*factor, dt_max, t_end - t).
 * stats[0] accepted, [1] rejected, [2] final t, [3] next h.
 * Returns 0, or 1 if max_steps attempts were used before t_end. */
int orc_propagate_adaptive(int L_max, const int *n, const double *eig,
                           const double *dip, char gauge, int field_kind,
                           const double *pars, double t0, double t_end,
                           double h0, double dt_max, double rtol, double atol,
                           int field_mode, int max_attempts, double *x,
                           double *stats) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  rk_init();
  work_t w;
  const int m = 2 * s.ntot;
  if (work_alloc(&w, m)) return -10;
  double *xn = (double *)malloc(sizeof(double) * m);
  double *e = (double *)malloc(sizeof(double) * m);
  double D[NST];
  for (int j = 0; j < NST; ++j) D[j] = RK_B8[j] - RK_B7[j];
  const double safety = 0.9, facmin = 0.2, facmax = 5.0;
  double t = t0, h = h0;
  int acc = 0, rej = 0, attempts = 0, ret = 0;
  double Fs[NST];
  while (t < t_end) {
    if (attempts >= max_attempts) { ret = 1; break; }
    ++attempts;
    int last = 0;
    if (h >= t_end - t) { h = t_end - t; last = 1; }
    for (int st = 0; st < NST; ++st)
      Fs[st] = orc_field(field_kind, pars, field_mode ? t + RK_C[st] * h : t + h);
    rk78_stages(&s, Fs, h, x, &w);
    stage_sum(m, x, w.k, RK_B8, h, xn);
    for (int i = 0; i < m; ++i) e[i] = 0.0;
    for (int j = 0; j < NST; ++j) {
      if (D[j] == 0.0) continue;
      const double c = h * D[j];
      for (int i = 0; i < m; ++i) e[i] = e[i] + c * w.k[j][i];
    }
    double err = 0.0;
    for (int i = 0; i < s.ntot; ++i) {
      double ax = sqrt(x[2 * i] * x[2 * i] + x[2 * i + 1] * x[2 * i + 1]);
      double an = sqrt(xn[2 * i] * xn[2 * i] + xn[2 * i + 1] * xn[2 * i + 1]);
      double ae = sqrt(e[2 * i] * e[2 * i] + e[2 * i + 1] * e[2 * i + 1]);
      double sc = atol + rtol * (ax > an ? ax : an);
      double r = ae / sc;
      if (r > err) err = r;
    }
    double fac;
    if (err == 0.0) fac = facmax;
    else {
      fac = safety / sqrt(sqrt(sqrt(err)));
      if (fac < facmin) fac = facmin;
      if (fac > facmax) fac = facmax;
    }
    if (err <= 1.0) {
      t = last ? t_end : t + h;
      double nrm = znrm2(s.ntot, xn);
      for (int i = 0; i < m; ++i) x[i] = xn[i] / nrm;
      ++acc;
      h = h * fac;
      if (h > dt_max) h = dt_max;
    } else {
      ++rej;
      if (fac > 1.0) fac = 1.0;
      h = h * fac;
    }
  }
  if (stats) {
    stats[0] = acc;
    stats[1] = rej;
    stats[2] = t;
    stats[3] = h;
  }
  free(xn);
  free(e);
  free(w.buf);
  return ret;
}

/* ------------------------------------------------------------------------ */
/* Discrete adjoint of the fixed-step propagation (own semantics).           */
/*                                                                           */
/* Forward per step n: F_n = base(t_n+dt) + dE(t_n+dt); y_s, k_s = M(F_n) y_s */
/* (M = -i(H0 + F S) length, -i H0 + F K velocity); z_n = x_n + h sum b_j k_j;*/
/* x_{n+1} = z_n / ||z_n||.  Objective J(x_N): target < 0 -> the yield       */
/* above the threshold, 1 - sum_{eig<thr} |x_i|^2 (thr = 0 unless            */
/* orc_set_yield_threshold changed it), evaluated as sum_{eig>=thr} |x_i|^2  */
/* (||x_N|| = 1) with the seed 2 x on those states; else |x_target|^2.       */
/* Reverse (real inner product Re<u,v>, M^T = M^dagger = -M):               */
/*   zbar = (lam - x_{n+1} Re<x_{n+1},lam>) / ||z_n||                        */
/*   kbar_s = h b_s zbar + sum_{s'>s} h a_{s's} ybar_{s'}  (s = 12..0)       */
/*   ybar_s = -M kbar_s;  dJ/dF_n += -Re<M1 kbar_s, y_s>,  M1 = dM/dF        */
/*   lam_n = zbar + sum_s ybar_s                                             */
/* dJ/du_k = sum_n dJ/dF_n * phi((t_n + dt)/g - k).                          */
/* ------------------------------------------------------------------------ */

static double g_yield_thr = 0.0;
void orc_set_yield_threshold(double thr) { g_yield_thr = thr; }

/* M1 v (coupling at unit field), with a zero diagonal. */
static void coupling(const sys_t *s, const double *v, double *out, double *zero_eig) {
  sys_t z = *s;
  z.eig = zero_eig;
  rhs(&z, 1.0, v, out);
}

int orc_objective_gradient(int L_max, const int *n, const double *eig, const double *dip,
                           char gauge, int field_kind, const double *pars, int K,
                           const double *u, double T, double t0, double dt, int steps,
                           int target, const double *x0, double *J, double *grad_u,
                           double *Fbar_out, double *xN) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  rk_init();
  const int m = 2 * s.ntot;
  const size_t per = (size_t)m;
  double *X = (double *)malloc(sizeof(double) * per * (steps + 1));
  double *Ys = (double *)malloc(sizeof(double) * per * (size_t)steps * NST);
  double *nrm = (double *)malloc(sizeof(double) * steps);
  double *Fn = (double *)malloc(sizeof(double) * steps);
  double *tn = (double *)malloc(sizeof(double) * steps);
  double *zero = (double *)calloc(s.ntot, sizeof(double));
  work_t w;
  if (!X || !Ys || !nrm || !Fn || !tn || !zero || work_alloc(&w, m)) return -10;
  memcpy(X, x0, sizeof(double) * per);
  double t = t0;
  for (int st = 0; st < steps; ++st) {
    double F = orc_field(field_kind, pars, t + dt);
    if (K > 0) F += orc_control_eval(K, u, T, t + dt);
    Fn[st] = F;
    tn[st] = t + dt;
    const double *x = X + per * st;
    double *ys = Ys + per * (size_t)st * NST;
    /* stages, keeping every stage input */
    memcpy(ys, x, sizeof(double) * per);
    rhs(&s, F, ys, w.k[0]);
    for (int q = 1; q < NST; ++q) {
      stage_sum(m, x, w.k, RK_A[q], dt, ys + per * q);
      rhs(&s, F, ys + per * q, w.k[q]);
    }
    double *xn = X + per * (st + 1);
    stage_sum(m, x, w.k, RK_B8, dt, xn);
    double nr = znrm2(s.ntot, xn);
    for (int i = 0; i < m; ++i) xn[i] /= nr;
    nrm[st] = nr;
    t += dt;
  }
  const double *xf = X + per * steps;
  double *lam = (double *)calloc(per, sizeof(double));
  double *zb = (double *)malloc(sizeof(double) * per);
  double *kb = (double *)malloc(sizeof(double) * per);
  double *yb = (double *)malloc(sizeof(double) * per * NST);
  double *w1 = (double *)malloc(sizeof(double) * per);
  double Jv = 0.0;
  if (target < 0) {
    double b = 0.0;
    for (int i = 0; i < s.ntot; ++i)
      if (eig[i] >= g_yield_thr) {
        b += xf[2 * i] * xf[2 * i] + xf[2 * i + 1] * xf[2 * i + 1];
        lam[2 * i] = 2.0 * xf[2 * i];
        lam[2 * i + 1] = 2.0 * xf[2 * i + 1];
      }
    Jv = b;
  } else {
    Jv = xf[2 * target] * xf[2 * target] + xf[2 * target + 1] * xf[2 * target + 1];
    lam[2 * target] = 2.0 * xf[2 * target];
    lam[2 * target + 1] = 2.0 * xf[2 * target + 1];
  }
  if (xN) memcpy(xN, xf, sizeof(double) * per);
  for (int st = steps - 1; st >= 0; --st) {
    const double *x1 = X + per * (st + 1);
    const double *ys = Ys + per * (size_t)st * NST;
    double d = 0.0;
    for (int i = 0; i < m; ++i) d += x1[i] * lam[i];
    for (int i = 0; i < m; ++i) zb[i] = (lam[i] - x1[i] * d) / nrm[st];
    const double F = Fn[st];
    double fb = 0.0;
    for (int q = NST - 1; q >= 0; --q) {
      /* kbar_q = h b_q zbar + sum_{q'>q} h a_{q'q} ybar_{q'} */
      for (int i = 0; i < m; ++i) kb[i] = (dt * RK_B8[q]) * zb[i];
      for (int qq = q + 1; qq < NST; ++qq) {
        const double c = dt * RK_A[qq][q];
        if (c == 0.0) continue;
        for (int i = 0; i < m; ++i) kb[i] += c * yb[per * qq + i];
      }
      coupling(&s, kb, w1, zero); /* M1 kbar */
      double *ybq = yb + per * q;
      for (int i = 0; i < s.ntot; ++i) {
        const double e = eig[i];
        const double vr = kb[2 * i], vi = kb[2 * i + 1];
        const double mr = e * vi + F * w1[2 * i], mi = -e * vr + F * w1[2 * i + 1];
        ybq[2 * i] = -mr;
        ybq[2 * i + 1] = -mi;
        fb -= w1[2 * i] * ys[per * q + 2 * i] + w1[2 * i + 1] * ys[per * q + 2 * i + 1];
      }
    }
    for (int i = 0; i < m; ++i) {
      double a = zb[i];
      for (int q = 0; q < NST; ++q) a += yb[per * q + i];
      lam[i] = a;
    }
    if (Fbar_out) Fbar_out[st] = fb;
    if (grad_u && K > 0) {
      double wts[4];
      int k0 = control_weights(K, T, tn[st], wts);
      for (int j = 0; j < 4; ++j)
        if (wts[j] != 0.0) grad_u[k0 + j] += fb * wts[j];
    }
  }
  *J = Jv;
  free(X); free(Ys); free(nrm); free(Fn); free(tn); free(zero); free(w.buf);
  free(lam); free(zb); free(kb); free(yb); free(w1);
  return 0;
}

/* Objective only (same forward as orc_objective_gradient). */
int orc_objective(int L_max, const int *n, const double *eig, const double *dip, char gauge,
                  int field_kind, const double *pars, int K, const double *u, double T,
                  double t0, double dt, int steps, int target, const double *x0, double *J) {
  sys_t s;
  int rc = sys_init(&s, L_max, n, eig, dip, gauge);
  if (rc) return rc;
  const int m = 2 * s.ntot;
  double *x = (double *)malloc(sizeof(double) * m);
  memcpy(x, x0, sizeof(double) * m);
  rc = orc_propagate(L_max, n, eig, dip, gauge, field_kind, pars, K, u, T, t0, dt, steps, 0, x,
                     NULL, NULL, NULL);
  double Jv = 0.0;
  if (target < 0) {
    double b = 0.0;
    for (int i = 0; i < s.ntot; ++i)
      if (eig[i] >= g_yield_thr) b += x[2 * i] * x[2 * i] + x[2 * i + 1] * x[2 * i + 1];
    Jv = b;
  } else {
    Jv = x[2 * target] * x[2 * target] + x[2 * target + 1] * x[2 * target + 1];
  }
  *J = Jv;
  free(x);
  return rc;
}
