// combine.cuh -- per-element epilogue of one RKF78 stage and the per-step
// renormalisation.
//
// k_stage_combine: for every state i (block L, local row r)
//   Q = sum_strips RP_L[strip][r]                  (D_L y_{L+1}, if L < L_max)
//   P = sum_slots  CP[slot][r mod 256]             (D_{L-1}^T y_{L-1}, if L > 0)
//   (4 lanes per state, each summing every 4th strip / slot, then a fixed
//   xor-shuffle tree: the order is fixed, so results repeat bit for bit)
//   k_s[i] per gauge, in the reference's order of operations
//   (src/tdse/tdse.cpp:14-73 velocity, :85-143 length):
//     length:   Im: ((-e*Re y) + (-F)*P.re) + (-F)*Q.re
//               Re: (( e*Im y) + ( F)*P.im) + ( F)*Q.im
//     velocity: Re: (( e*Im y) + ( F)*P.re) + (-F)*Q.re
//               Im: ((-e*Re y) + ( F)*P.im) + (-F)*Q.im
//   then the next stage input y_{s+1} = x + sum_{j<=s} (dt*a_{s+1,j}) k_j, or
//   for the last stage x_new = x + sum_j (dt*b_j) k_j with a per-CTA partial of
//   ||x_new||^2.  Products and sums are rounded separately (no contraction),
//   left to right, as the CPU restatement does.
//   Horner form (a.horner; the frozen-field step as the method's stability
//   polynomial R(z) = sum_m G_m z^m, degree 12): the input is v_{m+1} scaled
//   by vscale (G_12 for the first product, else 1) and the output
//   v_m = dt * M(F) (vscale v_{m+1}) + G_m x, v_0 = x_new; k is not stored.
// k_renorm: ||x_new|| from the per-CTA partials in a fixed order, then
//   x = x_new / ||x_new|| element by element (c /= ||c||, src/tdse/tdse.cpp:
//   194-198) and the tracked population |x[pop]|^2 (:200-204).
#pragma once
#include "dev_util.cuh"
#include "plan.h"

namespace mpc {

struct CombineArgs {
  const double2* x;        // state at the start of the step
  const double2* y;        // stage input y_s
  double2* k;              // k[13][ntot]
  double2* out;            // y_{s+1}, or x_new after the last stage
  const double* eps;       // H0 diagonal
  const double2* RP;
  const double2* CP;
  const int* strip_slot0;  // CP slots of global strip g: [strip_slot0[g], strip_slot0[g+1])
  const double* Ftab;      // field per step
  double* norm_part;       // last stage: per-CTA sum of |x_new|^2
  int step;
  int stage;               // 0..12
  int gauge;               // 0 length, 1 velocity
  int ncoef;               // non-zero weights of the next combination
  int coef_j[kNumStages];
  double coef[kNumStages]; // dt * a_{s+1,j}  (or dt * b_j)
  int horner;              // 1: one Horner product (stage 12: the last, with norm partials)
  double vscale, hg, hstep;
  Geometry g;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

__global__ void __launch_bounds__(kCombineThreads)
    k_stage_combine(const __grid_constant__ CombineArgs a) {
  const Geometry& g = a.g;
  pdl_trigger();
  pdl_wait();
  // kCombineLanes consecutive threads share one coefficient: they split its
  // partial sums (strip s and slot s handled by lane s mod kCombineLanes) and
  // reduce them with a fixed shuffle tree; lane 0 finishes the coefficient.
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = gt / kCombineLanes;
  const int q = gt % kCombineLanes;
  const bool valid = i < g.ntot;
  int L = 0, r = 0;
  double2 Q = make_double2(0.0, 0.0), P = make_double2(0.0, 0.0);
  if (valid) {
    while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
    r = i - g.state_off[L];
    if (L < g.nblk) {
      const BlockGeom& b = g.blk[L];
      const double2* rp = a.RP + b.rp_off + r;
#pragma unroll 4
      for (int s = q; s < b.nstrips; s += kCombineLanes) {
        const double2 v = rp[s * (long long)b.nrow];
        Q.x = dadd(Q.x, v.x);
        Q.y = dadd(Q.y, v.y);
      }
    }
    if (L > 0) {
      const BlockGeom& b = g.blk[L - 1];
      const int gs = b.strip0 + r / kStripW;
      const int c = r % kStripW;
      const int s1 = a.strip_slot0[gs + 1];
      for (int sl = a.strip_slot0[gs] + q; sl < s1; sl += kCombineLanes) {
        const double2 v = a.CP[(long long)sl * kStripW + c];
        P.x = dadd(P.x, v.x);
        P.y = dadd(P.y, v.y);
      }
    }
  }
#pragma unroll
  for (int o = 1; o < kCombineLanes; o <<= 1) {
    Q.x = dadd(Q.x, __shfl_xor_sync(0xffffffffu, Q.x, o));
    Q.y = dadd(Q.y, __shfl_xor_sync(0xffffffffu, Q.y, o));
    P.x = dadd(P.x, __shfl_xor_sync(0xffffffffu, P.x, o));
    P.y = dadd(P.y, __shfl_xor_sync(0xffffffffu, P.y, o));
  }
  double nsq = 0.0;
  if (valid && q == 0 && a.horner) {
    const double F = a.Ftab[a.step];
    const double e = a.eps[i];
    const double vs = a.vscale;
    const double2 yr = a.y[i];
    const double2 xi = a.x[i];
    const double2 y = make_double2(dmul(vs, yr.x), dmul(vs, yr.y));
    P = make_double2(dmul(vs, P.x), dmul(vs, P.y));
    Q = make_double2(dmul(vs, Q.x), dmul(vs, Q.y));
    double kre = dmul(e, y.y);
    double kim = dmul(-e, y.x);
    if (a.gauge == 0) {
      if (L > 0) { kim = dadd(kim, dmul(-F, P.x)); kre = dadd(kre, dmul(F, P.y)); }
      if (L < g.nblk) { kim = dadd(kim, dmul(-F, Q.x)); kre = dadd(kre, dmul(F, Q.y)); }
    } else {
      if (L > 0) { kre = dadd(kre, dmul(F, P.x)); kim = dadd(kim, dmul(F, P.y)); }
      if (L < g.nblk) { kre = dadd(kre, dmul(-F, Q.x)); kim = dadd(kim, dmul(-F, Q.y)); }
    }
    const double2 o = make_double2(dadd(dmul(a.hstep, kre), dmul(a.hg, xi.x)),
                                   dadd(dmul(a.hstep, kim), dmul(a.hg, xi.y)));
    a.out[i] = o;
    nsq = dadd(dmul(o.x, o.x), dmul(o.y, o.y));
  } else if (valid && q == 0) {
    const double F = a.Ftab[a.step];
    const double e = a.eps[i];
    const double2 y = a.y[i];
    double kre = dmul(e, y.y);
    double kim = dmul(-e, y.x);
    if (a.gauge == 0) {
      if (L > 0) { kim = dadd(kim, dmul(-F, P.x)); kre = dadd(kre, dmul(F, P.y)); }
      if (L < g.nblk) { kim = dadd(kim, dmul(-F, Q.x)); kre = dadd(kre, dmul(F, Q.y)); }
    } else {
      if (L > 0) { kre = dadd(kre, dmul(F, P.x)); kim = dadd(kim, dmul(F, P.y)); }
      if (L < g.nblk) { kre = dadd(kre, dmul(-F, Q.x)); kim = dadd(kim, dmul(-F, Q.y)); }
    }
    const long long n = g.ntot;
    a.k[a.stage * n + i] = make_double2(kre, kim);
    // load every earlier k_j first, then sum left to right
    double2 kj[kNumStages];
#pragma unroll
    for (int m = 0; m < kNumStages; ++m)
      if (m < a.ncoef) {
        const int j = a.coef_j[m];
        kj[m] = (j == a.stage) ? make_double2(kre, kim) : a.k[j * n + i];
      }
    double2 acc = a.x[i];
#pragma unroll
    for (int m = 0; m < kNumStages; ++m)
      if (m < a.ncoef) {
        const double c = a.coef[m];
        acc.x = dadd(acc.x, dmul(c, kj[m].x));
        acc.y = dadd(acc.y, dmul(c, kj[m].y));
      }
    a.out[i] = acc;
    nsq = dadd(dmul(acc.x, acc.x), dmul(acc.y, acc.y));
  }
  if (a.stage == kNumStages - 1) {
    // fixed-shape block reduction of |x_new|^2
    __shared__ double sh[kCombineThreads / 32];
    for (int o = 16; o > 0; o >>= 1) nsq += __shfl_xor_sync(0xffffffffu, nsq, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = nsq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = sh[0];
      for (int w = 1; w < kCombineThreads / 32; ++w) s += sh[w];
      a.norm_part[blockIdx.x] = s;
    }
  }
}

struct RenormArgs {
  double2* x;              // out: normalised state
  const double2* xnew;     // in
  const double* norm_part;
  int nparts;
  int ntot;
  int pop_index;
  int step;
  int hist_base;           // history index = step - hist_base
  double* pop_hist;        // [steps+1], entry step+1 written
  double* norm_hist;       // [steps]
  unsigned* status;
};

__global__ void __launch_bounds__(kCombineThreads) k_renorm(const __grid_constant__ RenormArgs a) {
  __shared__ double nrm_sh;
  pdl_trigger();
  pdl_wait();
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int p = threadIdx.x; p < a.nparts; p += 32) s += a.norm_part[p];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) nrm_sh = sqrt(s);
  }
  __syncthreads();
  const double nrm = nrm_sh;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (a.norm_hist) a.norm_hist[a.step - a.hist_base] = nrm;
    if (!(nrm > 0.0) || !isfinite(nrm)) atomicOr(a.status, ST_NONFINITE);
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ntot) {
    const double2 v = a.xnew[i];
    const double2 o = make_double2(v.x / nrm, v.y / nrm);
    a.x[i] = o;
    if (i == a.pop_index && a.pop_hist)
      a.pop_hist[a.step - a.hist_base + 1] = dadd(dmul(o.x, o.x), dmul(o.y, o.y));
  }
}

}  // namespace mpc
