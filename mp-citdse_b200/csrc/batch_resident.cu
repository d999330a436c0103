// batch_resident.cu -- batched adaptive RKF78 for a few pulses on a system
// whose coupling fits in the GPU's shared memory: one persistent cooperative
// launch runs every attempted step of every pulse.
//
// When a batch has narrowed to at most 8 pulses, the streamed GEMM path
// (batch.cu) is bound by per-launch latency rather than by work.  This kernel
// takes over instead.  Each of G CTAs (one per SM) owns a contiguous range of
// rows of one state block L and keeps their coupling rows in shared memory
// for the whole run (column r of D_{L-1} and row r of D_L, the latter
// negated in the velocity gauge), as the single-pulse resident kernel does.
// Per stage a CTA loads the stage input of the two blocks its rows couple to
// for all P pulse columns (L2), forms the coupling sums for all its rows at
// once (each window element is read once from shared memory and applied to
// every row held in registers), writes k_s and the next stage input, and
// meets the other CTAs at a grid barrier: 13 barriers per attempted step.
//
// In fixed-step mode (the reference's semantics) an attempt is the frozen-
// field step as the 12 Horner products of its stability polynomial, one
// barrier each, instead of the 13 stages.
// Step control needs no extra barrier: after the last stage every CTA
// reduces the per-CTA norm and error partials in the same fixed order and
// makes the same accept / reject decision for every pulse (the decision
// logic is that of the streamed path's controller).  An accepted x_new is
// divided by its norm where it is read (by every CTA, identically), and the
// owning CTA stores the divided rows into X at the next stage 0.
// Pulses that finish write their final state out; the launch ends when all
// are done or fewer than `exit_below` remain active, so that the host can
// compact the columns and continue with a narrower launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "batch_types.h"
#include "ctx.h"
#include "dev_util.cuh"
#include "plan.h"
#include "rkf78.h"

using namespace mpc;

namespace {

constexpr int QT = 256;          // threads per CTA
constexpr int QW = QT / 32;      // warps per CTA
constexpr int kRowGroup = 16;    // rows accumulated in registers per pass over the window
constexpr int kMaxP = 8;         // widest launch (pulse columns)

__constant__ double q_A[13][13];
__constant__ double q_B8[13];
__constant__ double q_G[13];     // the stability polynomial's coefficients
__constant__ double q_E[13];     // b8 - b7
__constant__ double q_C[13];

struct CtaPart {
  int L;           // state block of the CTA's rows
  int row0, row1;  // global rows [row0, row1)
};

struct BrArgs {
  const double* D;
  const double* eps;
  double2* X;
  double2* XN;
  double2* Y0;
  double2* Y1;
  double2* out;
  ColState c;
  PulseResults res;
  const CtaPart* part;
  double* red_nrm;    // [G][kMaxP]
  double* red_err;    // [G][kMaxP]
  unsigned* bar;      // 64-bit arrival counter (two words), cleared per launch
  unsigned* status;
  int ldc, ncol, ntot;
  int exit_below, max_attempts, gauge;
  double rtol, atol, dt_max;
  FixedStep fx;       // fixed-step mode (the reference's semantics)
  BarrierCfg bc;
  Geometry g;
};

// Grid barrier on a monotonic 64-bit arrival counter (cleared before each
// launch): the CTA's e-th barrier completes when the counter reaches
// e * gridDim.x.  Bounded wait: returns false (status raised) on timeout.
__device__ bool br_sync(const BrArgs& a, unsigned long long& epoch, int* s_dead) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(a.bar);
    if (!grid_arrive_wait(ctr, (epoch + 1) * gridDim.x + a.bc.skew, a.status, a.bc.wait_ns))
      *s_dead = 1;
    epoch += 1;
  }
  __syncthreads();
  return *s_dead == 0;
}

__device__ __forceinline__ double nanmax(double m, double e) {
  return (m != m) ? m : ((e != e) ? e : fmax(m, e));
}

__device__ __forceinline__ double2 scaled(double2 v, double nrm) {
  return make_double2(v.x / nrm, v.y / nrm);
}

// Shared-memory bytes of one CTA's tables at width P.
__host__ __device__ inline size_t br_smem(int Kc, int nrows, int P) {
  const int RP = (nrows + 1) & ~1;
  return 8 * (size_t)Kc * RP + 16 * (size_t)Kc * P + 16 * (size_t)kNumStages * nrows * P +
         2 * 16 * (size_t)nrows * P + 8 * (size_t)QW * kRowGroup * P * 2 +
         2 * 8 * (size_t)nrows * P;
}

template <int P>
__global__ void __launch_bounds__(QT, 1) k_batch_res(const __grid_constant__ BrArgs a) {
  extern __shared__ __align__(16) unsigned char qsm[];
  const Geometry& g = a.g;
  const int cta = blockIdx.x, G = gridDim.x;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const CtaPart pt = a.part[cta];
  const int L = pt.L, row0 = pt.row0, nrows = pt.row1 - pt.row0;
  const int nlo = L > 0 ? g.state_off[L] - g.state_off[L - 1] : 0;
  const int nup = L < g.nblk ? g.state_off[L + 2] - g.state_off[L + 1] : 0;
  const int Kc = nlo + nup;
  const int RP = (nrows + 1) & ~1;
  const int lo0 = L > 0 ? g.state_off[L - 1] : 0;
  const int up0 = L < g.nblk ? g.state_off[L + 1] : 0;
  const int rloc0 = row0 - g.state_off[L];
  const int ldc = a.ldc, ncol = a.ncol;

  double* crow = reinterpret_cast<double*>(qsm);            // [Kc][RP]
  double2* win = reinterpret_cast<double2*>(crow + (size_t)Kc * RP);  // [Kc][P]
  double2* ksm = win + (size_t)Kc * P;                       // [13][nrows][P]
  double2* xsm = ksm + (size_t)kNumStages * nrows * P;       // [nrows][P]
  double2* ysm = xsm + (size_t)nrows * P;                    // [nrows][P]
  double* wred = reinterpret_cast<double*>(ysm + (size_t)nrows * P);  // [QW][kRowGroup][P][2]
  double* rnrm = wred + QW * kRowGroup * P * 2;              // [nrows][P]
  double* rerr = rnrm + (size_t)nrows * P;                   // [nrows][P]

  __shared__ mpc_pulse s_pulse[P];
  __shared__ double s_t[P], s_tend[P], s_h[P], s_hatt[P], s_nrm[P], s_nsum[P], s_err[P];
  __shared__ double s_F[kNumStages][P];
  __shared__ int s_last[P], s_done[P], s_acc[P], s_nacc[P], s_nrej[P], s_natt[P], s_pid[P],
      s_ret[P], s_nsteps[P];
  __shared__ int s_exit, s_dead;

  // ---- coupling rows, once ----
  if (L > 0) {  // crow[k][li] = D_{L-1}[k][r]
    const BlockGeom& b = g.blk[L - 1];
    for (int e = tid; e < nlo * RP; e += QT) {
      const int k = e / RP, li = e % RP;
      crow[e] = li < nrows ? a.D[b.d_off + (long long)k * b.pitch + rloc0 + li] : 0.0;
    }
  }
  if (L < g.nblk) {  // crow[nlo + k][li] = sg * D_L[r][k]
    const BlockGeom& b = g.blk[L];
    const double sg = (a.gauge == 1) ? -1.0 : 1.0;
    for (int e = tid; e < RP * nup; e += QT) {
      const int li = e / nup, k = e % nup;
      crow[(size_t)(nlo + k) * RP + li] =
          li < nrows ? sg * a.D[b.d_off + (long long)(rloc0 + li) * b.pitch + k] : 0.0;
    }
  }
  // ---- column state (identical copy in every CTA) ----
  if (tid < P) {
    const int q = tid;
    if (q < ncol) {
      s_pulse[q] = a.c.pulse[q];
      s_t[q] = a.c.t[q];
      s_tend[q] = a.c.t_end[q];
      s_h[q] = a.c.h[q];
      s_done[q] = a.c.done[q];
      s_nacc[q] = a.c.nacc[q];
      s_nrej[q] = a.c.nrej[q];
      s_natt[q] = a.c.natt[q];
      s_pid[q] = a.c.pulse_id[q];
      s_nsteps[q] = a.c.nsteps[q];
    } else {
      s_pulse[q] = mpc_pulse{};
      s_t[q] = s_tend[q] = s_h[q] = 0.0;
      s_done[q] = 3;  // padding column
      s_nacc[q] = s_nrej[q] = s_natt[q] = 0;
      s_pid[q] = -1;
      s_nsteps[q] = 0;
    }
    s_nrm[q] = 1.0;
    s_hatt[q] = 0.0;
    s_last[q] = 0;
    s_acc[q] = 0;
    s_ret[q] = 0;
  }
  if (tid == 0) s_dead = 0;
  for (int e = tid; e < nrows * P; e += QT) {
    const int li = e / P, q = e % P;
    xsm[e] = q < ncol ? __ldcg(a.X + (long long)(row0 + li) * ldc + q) : make_double2(0.0, 0.0);
  }
  unsigned long long epoch = 0;
  __syncthreads();

  const int qc = tid % P;           // this thread's column in the coupling loop
  const int kt0 = tid / P;          // its first window row
  constexpr int KSTEP = QT / P;

  while (true) {
    if (tid == 0) {
      int act = 0;
      for (int q = 0; q < P; ++q) act += s_done[q] == 0;
      s_exit = (act == 0 || act < a.exit_below) ? 1 : 0;
    }
    __syncthreads();
    if (s_exit) break;
    // the attempt's step (capped at the time left) and its 13 stage fields
    if (tid < P) {
      const int q = tid;
      if (s_done[q]) {
        s_hatt[q] = 0.0;
      } else if (a.fx.on) {  // one step of dt
        s_hatt[q] = a.fx.dt;
        s_last[q] = (s_nacc[q] + 1 >= s_nsteps[q]) ? 1 : 0;
      } else {
        double h = s_h[q];
        const double rem = s_tend[q] - s_t[q];
        int last = 0;
        if (h >= rem) {
          h = rem;
          last = 1;
        }
        s_hatt[q] = h;
        s_last[q] = last;
      }
    }
    __syncthreads();
    for (int e = tid; e < kNumStages * P; e += QT) {
      const int s = e / P, q = e % P;
      // F(t + c_s h); in fixed-step mode F(t + dt) frozen for every stage
      const double ts = a.fx.on ? s_t[q] + a.fx.dt : s_t[q] + q_C[s] * s_hatt[q];
      s_F[s][q] = s_done[q] ? 0.0 : dev_field(s_pulse[q], ts);
    }
    __syncthreads();

    // fixed-step mode: the frozen-field step as the 12 Horner products of its
    // stability polynomial (v_12 = G_12 x, v_m = h M(F) v_{m+1} + G_m x,
    // x_new = v_0), one grid barrier each; otherwise the 13 stages
    const int nst = a.fx.on ? 12 : kNumStages;
    for (int s = 0; s < nst; ++s) {
      // ---- stage input: the coupled blocks' rows and this CTA's own rows ----
      if (s == 0) {
        for (int e = tid; e < Kc * P; e += QT) {
          const int k = e / P, q = e % P;
          const int row = k < nlo ? lo0 + k : up0 + (k - nlo);
          const long long idx = (long long)row * ldc + q;
          double2 v = make_double2(0.0, 0.0);
          if (q < ncol) v = s_acc[q] ? scaled(__ldcg(a.XN + idx), s_nrm[q]) : __ldcg(a.X + idx);
          win[e] = v;
        }
        for (int e = tid; e < nrows * P; e += QT) {
          const int li = e / P, q = e % P;
          if (q < ncol && s_acc[q]) {
            const long long idx = (long long)(row0 + li) * ldc + q;
            const double2 v = scaled(__ldcg(a.XN + idx), s_nrm[q]);
            xsm[e] = v;
            a.X[idx] = v;
          }
          ysm[e] = xsm[e];
        }
      } else {
        const double2* Yin = (s & 1) ? a.Y1 : a.Y0;
        for (int e = tid; e < Kc * P; e += QT) {
          const int k = e / P, q = e % P;
          const int row = k < nlo ? lo0 + k : up0 + (k - nlo);
          win[e] = q < ncol ? __ldcg(Yin + (long long)row * ldc + q) : make_double2(0.0, 0.0);
        }
        for (int e = tid; e < nrows * P; e += QT) {
          const int li = e / P, q = e % P;
          ysm[e] = q < ncol ? __ldcg(Yin + (long long)(row0 + li) * ldc + q)
                            : make_double2(0.0, 0.0);
        }
      }
      __syncthreads();
      const bool last_stage = (s == nst - 1);
      double2* Yout = ((s + 1) & 1) ? a.Y1 : a.Y0;
      // ---- coupling sums W[li][q] = sum_k crow[k][li] win[k][q], then k_s ----
      for (int rg = 0; rg < nrows; rg += kRowGroup) {
        double ar[kRowGroup], ai[kRowGroup];
#pragma unroll
        for (int r = 0; r < kRowGroup; ++r) ar[r] = ai[r] = 0.0;
        const int rmax = RP - rg;  // rows of this group present in crow (even)
        for (int k = kt0; k < Kc; k += KSTEP) {
          const double2 y = win[k * P + qc];
          const double* cr = crow + (size_t)k * RP + rg;
#pragma unroll
          for (int r = 0; r < kRowGroup; r += 2) {
            if (r < rmax) {
              const double2 d = *reinterpret_cast<const double2*>(cr + r);
              ar[r] = fma(d.x, y.x, ar[r]);
              ai[r] = fma(d.x, y.y, ai[r]);
              ar[r + 1] = fma(d.y, y.x, ar[r + 1]);
              ai[r + 1] = fma(d.y, y.y, ai[r + 1]);
            }
          }
        }
        // lanes of a warp holding the same column: fixed xor tree
#pragma unroll
        for (int o = P; o < 32; o <<= 1)
#pragma unroll
          for (int r = 0; r < kRowGroup; ++r) {
            ar[r] += __shfl_xor_sync(0xffffffffu, ar[r], o);
            ai[r] += __shfl_xor_sync(0xffffffffu, ai[r], o);
          }
        if (lane < P) {
#pragma unroll
          for (int r = 0; r < kRowGroup; ++r) {
            wred[((warp * kRowGroup + r) * P + lane) * 2 + 0] = ar[r];
            wred[((warp * kRowGroup + r) * P + lane) * 2 + 1] = ai[r];
          }
        }
        __syncthreads();
        const int nr = min(kRowGroup, nrows - rg);
        for (int e = tid; e < nr * P; e += QT) {
          const int r = e / P, q = e % P, li = rg + r;
          double wre = 0.0, wim = 0.0;
#pragma unroll
          for (int w = 0; w < QW; ++w) {  // warps in a fixed order
            wre += wred[((w * kRowGroup + r) * P + q) * 2 + 0];
            wim += wred[((w * kRowGroup + r) * P + q) * 2 + 1];
          }
          const int i = row0 + li;
          const double ev = a.eps[i];
          double2 y = ysm[li * P + q];
          const double F = s_F[s][q];
          if (a.fx.on && s == 0) {   // v_12 = G_12 x: its coupling G_12 (D x)
            const double vs = q_G[12];
            y = make_double2(vs * y.x, vs * y.y);
            wre *= vs;
            wim *= vs;
          }
          double kre, kim;
          if (a.gauge == 0) {
            kre = fma(F, wim, ev * y.y);
            kim = -fma(F, wre, ev * y.x);
          } else {
            kre = fma(F, wre, ev * y.y);
            kim = fma(F, wim, -ev * y.x);
          }
          const double2 x = xsm[li * P + q];
          const double hq = s_hatt[q];
          if (a.fx.on) {   // v_{11-s} = h M(F) v + G_{11-s} x
            const double gm = q_G[11 - s];
            const double2 o = make_double2(fma(hq, kre, gm * x.x), fma(hq, kim, gm * x.y));
            if (!last_stage) {
              if (q < ncol) Yout[(long long)i * ldc + q] = o;
            } else {
              rerr[li * P + q] = 0.0;
              rnrm[li * P + q] = o.x * o.x + o.y * o.y;
              if (q < ncol) a.XN[(long long)i * ldc + q] = o;
            }
            continue;
          }
          ksm[((size_t)s * nrows + li) * P + q] = make_double2(kre, kim);
          double2 o = x;
          if (!last_stage) {
#pragma unroll
            for (int j = 0; j < kNumStages; ++j) {
              const double cj = q_A[s + 1][j];
              if (j > s || cj == 0.0) continue;
              const double2 kj = (j == s) ? make_double2(kre, kim)
                                          : ksm[((size_t)j * nrows + li) * P + q];
              const double cf = hq * cj;
              o.x = fma(cf, kj.x, o.x);
              o.y = fma(cf, kj.y, o.y);
            }
            if (q < ncol) Yout[(long long)i * ldc + q] = o;
          } else {
            double2 er = make_double2(0.0, 0.0);
#pragma unroll
            for (int j = 0; j < kNumStages; ++j) {
              const double bj = q_B8[j], ej = q_E[j];
              if (bj == 0.0 && ej == 0.0) continue;
              const double2 kj = (j == s) ? make_double2(kre, kim)
                                          : ksm[((size_t)j * nrows + li) * P + q];
              if (bj != 0.0) {
                o.x = fma(hq * bj, kj.x, o.x);
                o.y = fma(hq * bj, kj.y, o.y);
              }
              if (ej != 0.0) {
                er.x = fma(hq * ej, kj.x, er.x);
                er.y = fma(hq * ej, kj.y, er.y);
              }
            }
            const double ax = sqrt(x.x * x.x + x.y * x.y), an = sqrt(o.x * o.x + o.y * o.y);
            const double ae = sqrt(er.x * er.x + er.y * er.y);
            rerr[li * P + q] = ae / (a.atol + a.rtol * fmax(ax, an));
            rnrm[li * P + q] = o.x * o.x + o.y * o.y;
            if (q < ncol) a.XN[(long long)i * ldc + q] = o;
          }
        }
        __syncthreads();
      }
      if (last_stage && tid < P) {
        // this CTA's partials per column, rows in order
        double ns = 0.0, em = 0.0;
        for (int li = 0; li < nrows; ++li) {
          ns += rnrm[li * P + tid];
          em = nanmax(em, rerr[li * P + tid]);
        }
        a.red_nrm[cta * kMaxP + tid] = ns;
        a.red_err[cta * kMaxP + tid] = em;
      }
      if (!br_sync(a, epoch, &s_dead)) break;
    }
    if (s_dead) break;

    // ---- step control: every CTA reduces the partials in the same order ----
    if (warp < P) {
      const int q = warp;
      double ns = 0.0, em = 0.0;
      for (int c = lane; c < G; c += 32) {
        ns += __ldcg(a.red_nrm + c * kMaxP + q);
        em = nanmax(em, __ldcg(a.red_err + c * kMaxP + q));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ns += __shfl_xor_sync(0xffffffffu, ns, o);
        em = nanmax(em, __shfl_xor_sync(0xffffffffu, em, o));
      }
      if (lane == 0) {
        s_nsum[q] = ns;
        s_err[q] = em;
      }
    }
    __syncthreads();
    if (tid < P && a.fx.on) {
      // fixed-step mode: accept every finite step, t += dt, retire after
      // nsteps steps
      const int q = tid;
      s_acc[q] = 0;
      if (!s_done[q]) {
        const double nrm = sqrt(s_nsum[q]);
        s_natt[q] += 1;
        if (nrm > 0.0 && isfinite(nrm)) {
          s_t[q] = s_t[q] + a.fx.dt;
          s_nacc[q] += 1;
          s_acc[q] = 1;
          s_nrm[q] = nrm;
          if (cta == 0 && a.fx.norm_hist)
            a.fx.norm_hist[(long long)s_pid[q] * a.fx.hist_ld + s_nacc[q] - 1] = nrm;
          if (s_nacc[q] >= s_nsteps[q]) s_done[q] = 1;
        } else {
          if (cta == 0) atomicOr(a.status, ST_NONFINITE);
          s_done[q] = 2;
        }
        s_ret[q] = s_done[q] ? 1 : 0;
      }
    } else if (tid < P) {
      const int q = tid;
      s_acc[q] = 0;
      if (!s_done[q]) {
        const double err = s_err[q];
        const double nrm = sqrt(s_nsum[q]);
        const double hh = s_hatt[q];
        const double safety = 0.9, facmin = 0.2, facmax = 5.0;
        double fac;
        if (err == 0.0) {
          fac = facmax;
        } else {
          fac = safety / sqrt(sqrt(sqrt(err)));
          fac = fmin(fmax(fac, facmin), facmax);
        }
        s_natt[q] += 1;
        const bool ok = (err <= 1.0) && (nrm > 0.0) && isfinite(nrm);
        if (ok) {
          s_t[q] = s_last[q] ? s_tend[q] : s_t[q] + hh;
          s_nacc[q] += 1;
          s_acc[q] = 1;
          s_nrm[q] = nrm;
          double hn = hh * fac;
          if (hn > a.dt_max) hn = a.dt_max;
          s_h[q] = hn;
          if (s_last[q]) s_done[q] = 1;
        } else {
          s_nrej[q] += 1;
          s_h[q] = hh * fmin(fac, 1.0);
        }
        if (!s_done[q] && (s_natt[q] >= a.max_attempts ||
                           s_h[q] < 1e-13 * fmax(1.0, fabs(s_tend[q]))))
          s_done[q] = 2;
        s_ret[q] = s_done[q] ? 1 : 0;
      }
    }
    __syncthreads();
    // fixed-step population history: the CTA owning pop_index
    if (a.fx.pop_hist && tid < P && s_acc[tid] && a.fx.pop_index >= row0 &&
        a.fx.pop_index < row0 + nrows) {
      const double2 v =
          scaled(__ldcg(a.XN + (long long)a.fx.pop_index * ldc + tid), s_nrm[tid]);
      a.fx.pop_hist[(long long)s_pid[tid] * a.fx.hist_ld + s_nacc[tid]] =
          __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    }
    // pulses that finished: final state out (own rows), counters by CTA 0
    for (int e = tid; e < nrows * P; e += QT) {
      const int li = e / P, q = e % P;
      if (!s_ret[q]) continue;
      const long long idx = (long long)(row0 + li) * ldc + q;
      const double2 v = s_acc[q] ? scaled(__ldcg(a.XN + idx), s_nrm[q]) : xsm[e];
      a.out[(long long)s_pid[q] * a.ntot + row0 + li] = v;
    }
    if (cta == 0 && tid < P && s_ret[tid]) {
      const int id = s_pid[tid];
      a.res.nacc[id] = s_nacc[tid];
      a.res.nrej[id] = s_nrej[tid];
      a.res.t[id] = s_t[tid];
      a.res.status[id] = (s_done[tid] == 2) ? 2 : 0;
    }
    __syncthreads();
    if (tid < P) s_ret[tid] = 0;
    __syncthreads();
  }
  if (s_dead) return;
  // ---- leave X holding every column's current state; column state back ----
  for (int e = tid; e < nrows * P; e += QT) {
    const int li = e / P, q = e % P;
    if (q < ncol && s_acc[q]) {
      const long long idx = (long long)(row0 + li) * ldc + q;
      a.X[idx] = scaled(__ldcg(a.XN + idx), s_nrm[q]);
    }
  }
  if (cta == 0 && tid < ncol && tid < P) {
    const int q = tid;
    a.c.t[q] = s_t[q];
    a.c.h[q] = s_h[q];
    a.c.done[q] = s_done[q];
    a.c.nacc[q] = s_nacc[q];
    a.c.nrej[q] = s_nrej[q];
    a.c.natt[q] = s_natt[q];
    a.c.nrm[q] = s_nrm[q];
    a.c.accepted[q] = 0;
    a.c.retired[q] = 0;
  }
}

template <int P>
const void* br_kernel() {
  return reinterpret_cast<const void*>(&k_batch_res<P>);
}

const void* br_kernel_for(int P) {
  switch (P) {
    case 1: return br_kernel<1>();
    case 2: return br_kernel<2>();
    case 4: return br_kernel<4>();
    default: return br_kernel<8>();
  }
}

}  // namespace

struct mpc_batch_res_state {
  bool tried = false;
  int pmax = 0;
  int G = 0;
  size_t smem[kMaxP + 1] = {};
  CtaPart* part = nullptr;
  double* red = nullptr;    // [2][G][kMaxP]
  unsigned* bar = nullptr;
};

namespace {

// CTAs per state block in proportion to its size, rows split evenly inside
// the block, so that every CTA's rows couple to the same two blocks.
bool plan_parts(const Geometry& g, int G, std::vector<CtaPart>& parts) {
  const int nb = g.nstate_blk;
  if (nb > G) return false;
  std::vector<int> cnt(nb);
  int used = 0;
  for (int L = 0; L < nb; ++L) {
    const int nL = g.state_off[L + 1] - g.state_off[L];
    cnt[L] = std::max(1, (int)((long long)G * nL / g.ntot));
    used += cnt[L];
  }
  while (used < G) {  // one more CTA to the block with the most rows per CTA
    int best = 0;
    double br = -1.0;
    for (int L = 0; L < nb; ++L) {
      const double r = (double)(g.state_off[L + 1] - g.state_off[L]) / cnt[L];
      if (r > br) { br = r; best = L; }
    }
    ++cnt[best];
    ++used;
  }
  while (used > G) {  // one fewer from the block with the fewest rows per CTA
    int best = -1;
    double br = 1e300;
    for (int L = 0; L < nb; ++L) {
      if (cnt[L] <= 1) continue;
      const double r = (double)(g.state_off[L + 1] - g.state_off[L]) / cnt[L];
      if (r < br) { br = r; best = L; }
    }
    if (best < 0) return false;
    --cnt[best];
    --used;
  }
  parts.clear();
  for (int L = 0; L < nb; ++L) {
    const int o = g.state_off[L], nL = g.state_off[L + 1] - o;
    for (int j = 0; j < cnt[L]; ++j)
      parts.push_back({L, o + (int)((long long)nL * j / cnt[L]),
                       o + (int)((long long)nL * (j + 1) / cnt[L])});
  }
  for (const CtaPart& p : parts)
    if (p.row1 <= p.row0) return false;
  return true;
}

}  // namespace

int mpc_batch_res_pmax(mpc_ctx* c) {
  if (!c->batch_res) c->batch_res = new mpc_batch_res_state();
  mpc_batch_res_state* r = c->batch_res;
  if (r->tried) return r->pmax;
  r->tried = true;
  if (std::getenv("MPC_NO_RESIDENT")) return 0;
  int coop = 0, optin = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (!coop) return 0;
  const int G = c->num_sms;
  std::vector<CtaPart> parts;
  if (!plan_parts(c->g, G, parts)) return 0;
  const size_t static_bytes = 4096;  // column state and flags (static shared)
  int pmax = 0;
  for (int P = 1; P <= kMaxP; P *= 2) {
    size_t need = 0;
    for (const CtaPart& p : parts) {
      const int L = p.L;
      const int Kc = (L > 0 ? c->g.state_off[L] - c->g.state_off[L - 1] : 0) +
                     (L < c->g.nblk ? c->g.state_off[L + 2] - c->g.state_off[L + 1] : 0);
      need = std::max(need, br_smem(Kc, p.row1 - p.row0, P));
    }
    if (need + static_bytes > (size_t)optin) break;
    const void* k = br_kernel_for(P);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need) !=
        cudaSuccess)
      break;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, QT, need) != cudaSuccess ||
        per_sm < 1)
      break;
    r->smem[P] = need;
    pmax = P;
  }
  cudaGetLastError();
  if (pmax == 0) return 0;
  double A[13][13], B8[13], E[13], Cn[13];
  for (int i = 0; i < 13; ++i) {
    for (int j = 0; j < 13; ++j) A[i][j] = rkf78::A[i][j];
    B8[i] = rkf78::B8[i];
    E[i] = rkf78::B8[i] - rkf78::B7[i];
    Cn[i] = rkf78::C[i];
  }
  if (cudaMemcpyToSymbol(q_A, A, sizeof A) != cudaSuccess ||
      cudaMemcpyToSymbol(q_B8, B8, sizeof B8) != cudaSuccess ||
      cudaMemcpyToSymbol(q_G, rkf78::G, sizeof rkf78::G) != cudaSuccess ||
      cudaMemcpyToSymbol(q_E, E, sizeof E) != cudaSuccess ||
      cudaMemcpyToSymbol(q_C, Cn, sizeof Cn) != cudaSuccess ||
      cudaMalloc(&r->part, sizeof(CtaPart) * G) != cudaSuccess ||
      cudaMalloc(&r->red, sizeof(double) * 2 * G * kMaxP) != cudaSuccess ||
      cudaMalloc(&r->bar, sizeof(unsigned) * 2) != cudaSuccess ||
      cudaMemcpy(r->part, parts.data(), sizeof(CtaPart) * G, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  r->G = G;
  r->pmax = pmax;
  return pmax;
}

int mpc_batch_res_run(mpc_ctx* c, const BatchResLaunch& l, int P, int exit_below) {
  mpc_batch_res_state* r = c->batch_res;
  if (!r || P < 1 || P > r->pmax || l.ncol > P || l.ncol < 1)
    return mpc_fail(MPC_ERR_ARG, "resident batched launch of %d columns at width %d", l.ncol, P);
  BrArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.X = l.X;
  a.XN = l.XN;
  a.Y0 = l.Y0;
  a.Y1 = l.Y1;
  a.out = l.out;
  a.c = l.c;
  a.res = l.res;
  a.part = r->part;
  a.red_nrm = r->red;
  a.red_err = r->red + (size_t)r->G * kMaxP;
  a.bar = r->bar;
  a.status = c->d_status;
  a.ldc = l.ldc;
  a.ncol = l.ncol;
  a.ntot = c->g.ntot;
  a.exit_below = exit_below;
  a.max_attempts = l.max_attempts;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.rtol = l.rtol;
  a.atol = l.atol;
  a.dt_max = l.dt_max;
  a.fx = l.fx;
  a.bc = mpc_barrier_cfg(c);
  a.g = c->g;
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream));  // arrival counter
  void* args[] = {&a};
  ProfScope ps(c, MPC_KERNEL_RESIDENT);
  CK(cudaLaunchCooperativeKernel(br_kernel_for(P), dim3(r->G), dim3(QT), args, r->smem[P],
                                 c->stream));
  ++c->launches;
  return MPC_OK;
}

void mpc_batch_res_free(mpc_ctx* c) {
  if (!c || !c->batch_res) return;
  mpc_batch_res_state* r = c->batch_res;
  cudaFree(r->part);
  cudaFree(r->red);
  cudaFree(r->bar);
  delete r;
  c->batch_res = nullptr;
}
