// resident.cu -- the fixed-step propagation for systems whose coupling fits
// in the GPU's shared memory: one persistent cooperative launch for all steps.
//
// Each of G CTAs (one per SM) owns a contiguous range of basis states (rows)
// and keeps, for each of its rows r of block L, the row's two coupling
// segments in shared memory for the whole run:
//   D_{L-1}[:, r]  (column r of the lower block: D_{L-1}^T y_{L-1}) and
//   D_L[r, :]      (row r of the upper block: D_L y_{L+1}), negated in the
//                  velocity gauge (K = [[0, -D],[D^T, 0]]),
// so a stage's coupling for its rows is complete inside the CTA: no partial
// sums cross CTAs.  Its k_s vectors stay in shared memory too.  Per stage the
// CTA reads the stage vector of the blocks its rows couple to (L2), forms k_s
// and the next stage input for its rows, writes that input, and meets the
// other CTAs at a grid barrier.  The norm after the last stage is reduced
// from per-CTA partials in a fixed order by every CTA, and the division
// x_new / ||x_new|| is applied when the next step reads the vector, so one
// barrier per stage suffices (13 per step).
// Same arithmetic semantics as the streaming path (tdse::propV / propL,
// src/tdse/tdse.cpp:186-215): F frozen at t+dt, 8th-order RKF78, c /= ||c||.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "ctx.h"
#include "dev_util.cuh"
#include "plan.h"
#include "rkf78.h"

using namespace mpc;

namespace {

constexpr int RTHREADS = 256;
constexpr int RWARPS = RTHREADS / 32;
constexpr int kMaxRowsPerCta = 96;

__constant__ double r_A[13][13];
__constant__ double r_B8[13];

struct ResArgs {
  const double* D;         // padded device layout (pitch per block)
  const double* eps;
  const double* Ftab;      // field per step
  double2* Y[2];           // stage inputs y_1..y_12, ping-pong
  double2* XN;             // x_new (unnormalised) after each step; x at entry
  double2* xout;           // normalised state at the end
  double* norm_part;       // [G]
  unsigned* bar;           // 64-bit arrival counter (two words), cleared per launch
  unsigned* status;
  double* pop_hist;        // [steps+1] (entry 0 written too)
  double* norm_hist;       // [steps]
  int pop_index;
  int steps;
  int gauge;               // 0 length, 1 velocity
  int first_is_normalised; // XN at entry holds a normalised x (norm 1)
  double dt;
  // optional outputs of the adjoint's passes (null when unused); slots are
  // vpitch complex apart
  double2* seg_x;          // x_n at the start of every step (normalised)
  double2* seg_y;          // stage inputs: slot step*13 + s holds y_s, s = 1..12
  double2* ckpt;           // x every ckpt_every steps: slot k holds x after k*ckpt_every
  int ckpt_every;
  long long vpitch;
  BarrierCfg bc;
  Geometry g;
};

// Grid barrier on a monotonic 64-bit arrival counter (cleared before each
// launch): the CTA's e-th barrier completes when the counter reaches
// e * gridDim.x, so the last arrival releases everyone with its one atomic
// (no reset, no second word).  Bounded wait; returns false (status raised) if
// it timed out.
__device__ bool bar_sync(unsigned* bar, unsigned* status, const BarrierCfg& bc,
                         unsigned long long& epoch, bool& dead) {
  __syncthreads();
  __shared__ int timed_out;
  if (threadIdx.x == 0) {
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(bar);
    timed_out =
        grid_arrive_wait(ctr, (epoch + 1) * gridDim.x + bc.skew, status, bc.wait_ns) ? 0 : 1;
    epoch += 1;
  }
  __syncthreads();
  if (timed_out) dead = true;
  return !dead;
}

__device__ bool grid_sync(const ResArgs& a, unsigned long long& epoch, bool& dead) {
  return bar_sync(a.bar, a.status, a.bc, epoch, dead);
}

__device__ __forceinline__ double2 ld_cg(const double2* p) { return __ldcg(p); }

// The stage-vector window [wlo, whi) this CTA's rows [row0, row1) couple to.
__device__ void row_window(const Geometry& g, int row0, int row1, int& wlo, int& whi) {
  int Llo = 0;
  while (Llo + 1 < g.nstate_blk && row0 >= g.state_off[Llo + 1]) ++Llo;
  int Lhi = Llo;
  while (Lhi + 1 < g.nstate_blk && row1 - 1 >= g.state_off[Lhi + 1]) ++Lhi;
  wlo = g.state_off[max(Llo - 1, 0)];
  whi = g.state_off[min(Lhi + 2, g.nstate_blk)];
}

// Loads, once, each row's two coupling segments: column r of D_{L-1}, then
// row r of D_L (negated in the velocity gauge); roff[li] is row li's offset.
__device__ void load_rows(const Geometry& g, const double* D, int gauge, int row0, int nrows,
                          int* roff, double* crow) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  if (threadIdx.x == 0) {
    int o = 0;
    for (int li = 0; li < nrows; ++li) {
      const int i = row0 + li;
      int L = 0;
      while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
      roff[li] = o;
      o += (L > 0 ? g.state_off[L] - g.state_off[L - 1] : 0) +
           (L < g.nblk ? g.state_off[L + 2] - g.state_off[L + 1] : 0);
    }
    roff[nrows] = o;
  }
  __syncthreads();
  for (int li = warp; li < nrows; li += nwarps) {
    const int i = row0 + li;
    int L = 0;
    while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
    const int r = i - g.state_off[L];
    double* dst = crow + roff[li];
    int o = 0;
    if (L > 0) {
      const BlockGeom& b = g.blk[L - 1];  // column r of D_{L-1}
      for (int k = lane; k < b.nrow; k += 32) dst[k] = D[b.d_off + (long long)k * b.pitch + r];
      o = b.nrow;
    }
    if (L < g.nblk) {
      const BlockGeom& b = g.blk[L];      // row r of D_L
      const double sg = (gauge == 1) ? -1.0 : 1.0;
      for (int k = lane; k < b.ncol; k += 32) dst[o + k] = sg * D[b.d_off + (long long)r * b.pitch + k];
    }
  }
}

// Coupling of row i (block L) with the window: W = sum_k crow[k] y_k over the
// coupled blocks, lanes striding k, then a fixed xor tree (all lanes hold W).
__device__ __forceinline__ void row_coupling(const Geometry& g, const double* cr,
                                             const double2* ywin, int wlo, int L, int lane,
                                             double& wr, double& wi) {
  wr = 0.0;
  wi = 0.0;
  int o = 0;
  if (L > 0) {
    const int nlo = g.state_off[L] - g.state_off[L - 1];
    const double2* yl = ywin + (g.state_off[L - 1] - wlo);
    for (int k = lane; k < nlo; k += 32) {
      const double d = cr[k];
      const double2 y = yl[k];
      wr = fma(d, y.x, wr);
      wi = fma(d, y.y, wi);
    }
    o = nlo;
  }
  if (L < g.nblk) {
    const int nup = g.state_off[L + 2] - g.state_off[L + 1];
    const double2* yu = ywin + (g.state_off[L + 1] - wlo);
    for (int k = lane; k < nup; k += 32) {
      const double d = cr[o + k];
      const double2 y = yu[k];
      wr = fma(d, y.x, wr);
      wi = fma(d, y.y, wi);
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    wr += __shfl_xor_sync(0xffffffffu, wr, off);
    wi += __shfl_xor_sync(0xffffffffu, wi, off);
  }
}

__global__ void __launch_bounds__(RTHREADS, 1) k_prop_resident(const __grid_constant__ ResArgs a) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const Geometry& g = a.g;
  const int G = gridDim.x, c = blockIdx.x;
  const int row0 = (int)((long long)g.ntot * c / G);
  const int row1 = (int)((long long)g.ntot * (c + 1) / G);
  const int nrows = row1 - row0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // the stage-vector window this CTA's rows couple to
  int wlo, whi;
  row_window(g, row0, row1, wlo, whi);
  const int wlen = whi - wlo;

  // shared layout: [row offsets (int, kMaxRowsPerCta+1)] [ywin (double2, wlen)]
  // [k (double2, 13 x nrows)] [x (double2, nrows)] [coupling rows (double)]
  int* roff = reinterpret_cast<int*>(rsm);
  double2* ywin = reinterpret_cast<double2*>(rsm + 16 * ((4 * (kMaxRowsPerCta + 1) + 15) / 16));
  double2* ksm = ywin + wlen;
  double2* xsm = ksm + kNumStages * nrows;
  double* crow = reinterpret_cast<double*>(xsm + nrows);
  __shared__ double red[RWARPS];
  __shared__ double nrm_sh;

  // ---- load the coupling rows once ----
  load_rows(g, a.D, a.gauge, row0, nrows, roff, crow);
  unsigned long long epoch = 0;
  bool dead = false;
  __syncthreads();

  const double h = a.dt;
  for (int step = 0; step < a.steps && !dead; ++step) {
    const double F = a.Ftab[step];
    for (int s = 0; s < kNumStages; ++s) {
      // ---- the stage input window ----
      if (s == 0) {
        // x = x_new / ||x_new|| (the previous step's result), or the entry x
        if (threadIdx.x < 32) {
          double sum = 0.0;
          if (step > 0 || !a.first_is_normalised) {
            for (int p = threadIdx.x; p < G; p += 32) sum += __ldcg(a.norm_part + p);
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
          } else {
            sum = 1.0;
          }
          if (threadIdx.x == 0) nrm_sh = (step > 0 || !a.first_is_normalised) ? sqrt(sum) : 1.0;
        }
        __syncthreads();
        const double nrm = nrm_sh;
        const bool divide = step > 0 || !a.first_is_normalised;
        for (int k = threadIdx.x; k < wlen; k += RTHREADS) {
          const double2 v = ld_cg(a.XN + wlo + k);
          ywin[k] = divide ? make_double2(v.x / nrm, v.y / nrm) : v;
        }
        __syncthreads();
        const bool to_ckpt = a.ckpt && step > 0 && step % a.ckpt_every == 0;
        for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
          const double2 v = ywin[row0 + li - wlo];
          xsm[li] = v;
          if (a.seg_x) a.seg_x[a.vpitch * step + row0 + li] = v;
          if (to_ckpt) a.ckpt[a.vpitch * (step / a.ckpt_every) + row0 + li] = v;
        }
        if (c == 0 && threadIdx.x == 0 && step > 0 && a.norm_hist) a.norm_hist[step - 1] = nrm;
        if (threadIdx.x == 0 && a.pop_index >= row0 && a.pop_index < row1) {
          const double2 v = ywin[a.pop_index - wlo];
          a.pop_hist[step] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
        }
      } else {
        const double2* Yin = a.seg_y ? a.seg_y + a.vpitch * (step * 13LL + s) : a.Y[s & 1];
        for (int k = threadIdx.x; k < wlen; k += RTHREADS) ywin[k] = ld_cg(Yin + wlo + k);
      }
      __syncthreads();
      // ---- k_s for this CTA's rows: one warp per row ----
      for (int li = warp; li < nrows; li += RWARPS) {
        const int i = row0 + li;
        int L = 0;
        while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
        double wr, wi;
        row_coupling(g, crow + roff[li], ywin, wlo, L, lane, wr, wi);
        if (lane == 0) {
          const double e = a.eps[i];
          const double2 y = ywin[i - wlo];
          double kre, kim;
          if (a.gauge == 0) {  // -i (e y + F W)
            kre = __dadd_rn(__dmul_rn(e, y.y), __dmul_rn(F, wi));
            kim = __dadd_rn(__dmul_rn(-e, y.x), __dmul_rn(-F, wr));
          } else {             // -i e y + F W
            kre = __dadd_rn(__dmul_rn(e, y.y), __dmul_rn(F, wr));
            kim = __dadd_rn(__dmul_rn(-e, y.x), __dmul_rn(F, wi));
          }
          ksm[s * nrows + li] = make_double2(kre, kim);
        }
      }
      __syncthreads();
      // ---- next stage input (or x_new) for this CTA's rows ----
      double nsq = 0.0;
      const bool last = (s == kNumStages - 1);
      for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
        double2 acc = xsm[li];
        for (int j = 0; j <= s; ++j) {
          const double cj = last ? r_B8[j] : r_A[s + 1][j];
          if (cj == 0.0) continue;
          const double cf = h * cj;
          const double2 kj = ksm[j * nrows + li];
          acc.x = __dadd_rn(acc.x, __dmul_rn(cf, kj.x));
          acc.y = __dadd_rn(acc.y, __dmul_rn(cf, kj.y));
        }
        if (last) {
          a.XN[row0 + li] = acc;
          nsq += __dadd_rn(__dmul_rn(acc.x, acc.x), __dmul_rn(acc.y, acc.y));
        } else if (a.seg_y) {
          a.seg_y[a.vpitch * (step * 13LL + s + 1) + row0 + li] = acc;
        } else {
          a.Y[(s + 1) & 1][row0 + li] = acc;
        }
      }
      if (last) {
        for (int o = 16; o > 0; o >>= 1) nsq += __shfl_xor_sync(0xffffffffu, nsq, o);
        if (lane == 0) red[warp] = nsq;
        __syncthreads();
        if (threadIdx.x == 0) {
          double t = red[0];
          for (int w = 1; w < RWARPS; ++w) t += red[w];
          a.norm_part[c] = t;
        }
      }
      if (!grid_sync(a, epoch, dead)) break;
    }
  }
  if (dead) return;
  // final state: x = x_new / ||x_new||, the last norm and population
  if (threadIdx.x < 32) {
    double sum = 0.0;
    for (int p = threadIdx.x; p < G; p += 32) sum += __ldcg(a.norm_part + p);
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (threadIdx.x == 0) nrm_sh = sqrt(sum);
  }
  __syncthreads();
  const double nrm = nrm_sh;
  if (a.steps > 0) {
    if (c == 0 && threadIdx.x == 0) {
      if (a.norm_hist) a.norm_hist[a.steps - 1] = nrm;
      if (!(nrm > 0.0) || !isfinite(nrm)) atomicOr(a.status, ST_NONFINITE);
    }
    for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
      const double2 v = ld_cg(a.XN + row0 + li);
      const double2 o = make_double2(v.x / nrm, v.y / nrm);
      a.xout[row0 + li] = o;
      if (row0 + li == a.pop_index)
        a.pop_hist[a.steps] = __dadd_rn(__dmul_rn(o.x, o.x), __dmul_rn(o.y, o.y));
    }
  }
}

// ---------------------------------------------------------------------------
// The adjoint sweep of one checkpoint segment on the resident layout (the
// reverse pass of the objective gradient, adjoint.cu): per step n, backwards,
//   d = Re<x_{n+1}, lam>            (per-CTA partials, a grid barrier, then the
//                                    same fixed-order sum in every CTA)
//   zbar = (lam - x_{n+1} d) / ||z_n||,   kbar_12 = h b_12 zbar
//   for s = 12 .. 0:  ybar_s = -M(F_n) kbar_s   (the coupling of kbar_s: the
//     same shared-memory rows and window as the forward, one barrier per stage)
//     dJ/dF_n += -Re<M1 kbar_s, y_s>
//     kbar_{s-1} = h b_{s-1} zbar + sum_{j>=s} h a_{j,s-1} ybar_j, or after
//     stage 0 lam_n = zbar + sum_j ybar_j.
// lam lives in shared memory for the CTA's rows (no other CTA reads it);
// kbar is exchanged through a ping-pong pair in global memory.
struct AdjResArgs {
  const double* D;
  const double* eps;
  const double* Ftab;      // field of local step j at Ftab[j]
  const double2* seg_x;    // x_j, j = 0..len (normalised), vpitch apart
  const double2* seg_y;    // y_s of step j at slot j*13 + s, s = 1..12
  const double* seg_n;     // ||z_j||
  double2* lam;            // in: lambda after the segment; out: before it
  double2* kb[2];          // kbar ping-pong [ntot]
  double* part;            // [G] partials of the inner product
  double* fpart;           // [len][G] per-CTA dJ/dF of each step
  unsigned* bar;           // 64-bit arrival counter (two words), cleared per launch
  unsigned* status;
  int len;
  int gauge;
  double dt;
  long long vpitch;
  BarrierCfg bc;
  Geometry g;
};

__constant__ double r_At[13][13];  // a_{j,s} at [s][j]

__global__ void __launch_bounds__(RTHREADS, 1) k_adj_resident(const __grid_constant__ AdjResArgs a) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const Geometry& g = a.g;
  const int G = gridDim.x, c = blockIdx.x;
  const int row0 = (int)((long long)g.ntot * c / G);
  const int row1 = (int)((long long)g.ntot * (c + 1) / G);
  const int nrows = row1 - row0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int wlo, whi;
  row_window(g, row0, row1, wlo, whi);
  const int wlen = whi - wlo;
  // shared layout: [row offsets] [window (double2, wlen)] [ybar (double2, 13 x nrows)]
  // [zbar (double2, nrows)] [lam (double2, nrows)] [dJ/dF per row (double, nrows)]
  // [coupling rows (double)]
  int* roff = reinterpret_cast<int*>(rsm);
  double2* ywin = reinterpret_cast<double2*>(rsm + 16 * ((4 * (kMaxRowsPerCta + 1) + 15) / 16));
  double2* ybs = ywin + wlen;
  double2* zbs = ybs + kNumStages * nrows;
  double2* lams = zbs + nrows;
  double* frow = reinterpret_cast<double*>(lams + nrows);
  double* crow = frow + ((nrows + 1) & ~1);
  __shared__ double red[RWARPS];
  __shared__ double d_sh;

  load_rows(g, a.D, a.gauge, row0, nrows, roff, crow);
  for (int li = threadIdx.x; li < nrows; li += RTHREADS) lams[li] = ld_cg(a.lam + row0 + li);
  unsigned long long epoch = 0;
  bool dead = false;
  __syncthreads();

  const double h = a.dt;
  const long long vp = a.vpitch;
  for (int j = a.len - 1; j >= 0 && !dead; --j) {
    const double F = a.Ftab[j];
    const double2* x1 = a.seg_x + vp * (j + 1);
    // ---- d = Re<x_{n+1}, lam> ----
    double v = 0.0;
    for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
      const double2 x = ld_cg(x1 + row0 + li), l = lams[li];
      v += __dadd_rn(__dmul_rn(x.x, l.x), __dmul_rn(x.y, l.y));
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = red[0];
      for (int w = 1; w < RWARPS; ++w) t += red[w];
      a.part[c] = t;
    }
    if (!bar_sync(a.bar, a.status, a.bc, epoch, dead)) break;
    if (threadIdx.x < 32) {
      double t = 0.0;
      for (int p = threadIdx.x; p < G; p += 32) t += __ldcg(a.part + p);
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) d_sh = t;
    }
    __syncthreads();
    // ---- zbar and kbar_12 ----
    {
      const double d = d_sh, nz = __ldcg(a.seg_n + j), hb = h * r_B8[kNumStages - 1];
      for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
        const double2 l = lams[li], x = ld_cg(x1 + row0 + li);
        const double2 z = make_double2((l.x - x.x * d) / nz, (l.y - x.y * d) / nz);
        zbs[li] = z;
        a.kb[0][row0 + li] = make_double2(hb * z.x, hb * z.y);
        frow[li] = 0.0;
      }
    }
    if (!bar_sync(a.bar, a.status, a.bc, epoch, dead)) break;
    double fcta = 0.0;
    for (int s = kNumStages - 1; s >= 0; --s) {
      const double2* kin = a.kb[s & 1];
      for (int k = threadIdx.x; k < wlen; k += RTHREADS) ywin[k] = ld_cg(kin + wlo + k);
      __syncthreads();
      for (int li = warp; li < nrows; li += RWARPS) {
        const int i = row0 + li;
        int L = 0;
        while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
        double wr, wi;
        row_coupling(g, crow + roff[li], ywin, wlo, L, lane, wr, wi);
        if (lane == 0) {
          const double e = a.eps[i];
          const double2 kv = ywin[i - wlo];
          // M1 kbar: -i W (length) or W (velocity, signs in the rows)
          const double2 m1 = (a.gauge == 0) ? make_double2(wi, -wr) : make_double2(wr, wi);
          // ybar_s = -M kbar = -(-i e kbar + F M1 kbar)
          const double2 yb = make_double2(-(__dmul_rn(e, kv.y) + __dmul_rn(F, m1.x)),
                                          -(__dmul_rn(-e, kv.x) + __dmul_rn(F, m1.y)));
          ybs[s * nrows + li] = yb;
          const double2 y = (s == 0) ? ld_cg(a.seg_x + vp * j + i)
                                     : ld_cg(a.seg_y + vp * (j * 13LL + s) + i);
          frow[li] = -(__dmul_rn(m1.x, y.x) + __dmul_rn(m1.y, y.y));
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {  // this stage's dJ/dF, rows in order
        double t = 0.0;
        for (int li = 0; li < nrows; ++li) t += frow[li];
        fcta += t;
      }
      double2* kout = a.kb[(s + 1) & 1];
      for (int li = threadIdx.x; li < nrows; li += RTHREADS) {
        if (s > 0) {
          const double cb = h * r_B8[s - 1];
          const double2 z = zbs[li];
          double2 o = make_double2(__dmul_rn(cb, z.x), __dmul_rn(cb, z.y));
          for (int sp = s; sp < kNumStages; ++sp) {
            const double cf = r_At[s - 1][sp];
            if (cf == 0.0) continue;
            const double2 w = ybs[sp * nrows + li];
            const double cc = h * cf;
            o.x = __dadd_rn(o.x, __dmul_rn(cc, w.x));
            o.y = __dadd_rn(o.y, __dmul_rn(cc, w.y));
          }
          kout[row0 + li] = o;
        } else {
          double2 o = zbs[li];
          for (int sp = 0; sp < kNumStages; ++sp) {
            const double2 w = ybs[sp * nrows + li];
            o.x = __dadd_rn(o.x, w.x);
            o.y = __dadd_rn(o.y, w.y);
          }
          lams[li] = o;
        }
      }
      if (s > 0 && !bar_sync(a.bar, a.status, a.bc, epoch, dead)) break;
      __syncthreads();
    }
    if (dead) break;
    if (threadIdx.x == 0) a.fpart[(long long)j * G + c] = fcta;
  }
  if (dead) return;
  __syncthreads();
  for (int li = threadIdx.x; li < nrows; li += RTHREADS) a.lam[row0 + li] = lams[li];
}

// dJ/dF_n = sum over CTAs of the step's partials, in CTA order.
__global__ void k_adj_res_fbar(const double* fpart, int len, int G, double* fbar) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= len) return;
  double t = 0.0;
  for (int p = 0; p < G; ++p) t += fpart[(long long)j * G + p];
  fbar[j] = t;
}

// ---------------------------------------------------------------------------
// The whole reverse pass of the objective gradient in one persistent launch,
// with the recompute of checkpoint segment a-1 running concurrently with the
// adjoint sweep of segment a.  The two are independent -- the sweep of a
// needs only segment a's stored states, stage inputs and norms; the
// recompute of a-1 only the checkpoint at its start -- and both are bound by
// grid-barrier latency, so they share the barriers: each CTA runs its
// recompute on warps 0-7 (the forward group) and its sweep on warps 8-15
// (the adjoint group), both over the CTA's own rows with the same
// shared-memory coupling rows, and one grid barrier ends each tick.
// A step slot is 14 ticks: the forward group does stage s at tick s (13
// stages, tick 13 idle); the adjoint group does, per step n (backwards),
//   tick 0    stage 0 of step n+1 (ybar_0, lambda_{n+1} = zbar + sum ybar,
//             its dJ/dF), then the partials of Re<x_{n+1}, lambda>;
//   tick 1    d, zbar = (lambda - x_{n+1} d) / ||z_n||, kbar_12;
//   tick 1+k  stage 13-k (k = 1..12): ybar_s, dJ/dF partial, kbar_{s-1},
// and after the segment's last slot one more tick finishes stage 0 of its
// first step (and the forward group normalises its last x_new).  Iteration
// it recomputes segment nseg-1-it and sweeps segment nseg-it; segments
// alternate between two buffer sets, so a sweep always reads the set that
// the previous iteration's recompute wrote.  Arithmetic per row is that of
// k_prop_resident and k_adj_resident (same order of operations), so the
// gradient is the same as theirs run one after the other.
struct FusedArgs {
  const double* D;
  const double* eps;
  const double* Ftab;      // field of global step n at Ftab[n]
  const double2* ckpt;     // checkpoint k (x after k*ckpt_every steps), vpitch apart
  double2* segX[2];        // per buffer set: x_j, j = 0..len (normalised)
  double2* segY[2];        // per buffer set: y_s of step j at slot j*13 + s
  double* segN[2];         // per buffer set: ||z_j||
  double2* XN;             // forward group: x_new of the current step [ntot]
  double* part_f;          // [G] norm partials (forward group)
  double2* lam;            // in: lambda_N; out: lambda_0
  double2* kb[2];          // kbar ping-pong [ntot]
  double* part_a;          // [G] partials of Re<x, lambda> (adjoint group)
  double* fpart;           // [steps][G] per-CTA dJ/dF of every step
  unsigned* bar;           // 64-bit arrival counter, cleared per launch
  unsigned* status;
  int steps, ckpt_every, nseg;
  int gauge;
  double dt;
  long long vpitch;
  BarrierCfg bc;
  Geometry g;
};

__device__ __forceinline__ void group_sync(int grp) { named_bar_sync(1 + grp, RTHREADS); }

__global__ void __launch_bounds__(2 * RTHREADS, 1) k_adj_fused(const __grid_constant__ FusedArgs a) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const Geometry& g = a.g;
  const int G = gridDim.x, c = blockIdx.x;
  const int row0 = (int)((long long)g.ntot * c / G);
  const int row1 = (int)((long long)g.ntot * (c + 1) / G);
  const int nrows = row1 - row0;
  const int grp = threadIdx.x >= RTHREADS ? 1 : 0;   // 0: recompute, 1: sweep
  const int tg = threadIdx.x - grp * RTHREADS;
  const int warp = tg >> 5, lane = tg & 31;
  int wlo, whi;
  row_window(g, row0, row1, wlo, whi);
  const int wlen = whi - wlo;
  // shared layout: [row offsets] [forward window] [k (13 x nrows)] [x (nrows)]
  // [adjoint window] [ybar (13 x nrows)] [zbar] [lambda] [dJ/dF per row]
  // [coupling rows]
  int* roff = reinterpret_cast<int*>(rsm);
  double2* ywin = reinterpret_cast<double2*>(rsm + 16 * ((4 * (kMaxRowsPerCta + 1) + 15) / 16));
  double2* ksm = ywin + wlen;
  double2* xsm = ksm + kNumStages * nrows;
  double2* awin = xsm + nrows;
  double2* ybs = awin + wlen;
  double2* zbs = ybs + kNumStages * nrows;
  double2* lams = zbs + nrows;
  double* frow = reinterpret_cast<double*>(lams + nrows);
  double* crow = frow + ((nrows + 1) & ~1);
  __shared__ double redf[RWARPS], reda[RWARPS];
  __shared__ double nrm_sh, d_sh, fcta_sh;

  load_rows(g, a.D, a.gauge, row0, nrows, roff, crow);
  if (grp == 1)
    for (int li = tg; li < nrows; li += RTHREADS) lams[li] = ld_cg(a.lam + row0 + li);
  if (threadIdx.x == 0) fcta_sh = 0.0;
  unsigned long long epoch = 0;
  bool dead = false;
  __syncthreads();

  const double h = a.dt;
  const long long vp = a.vpitch;
  const int K = a.ckpt_every;

  // stage 0 of adjoint step j (global step n0 + j) of the segment in set `set`:
  // ybar_0 from the kbar_0 window, lambda_j = zbar + sum_s ybar_s, the step's
  // dJ/dF (all 13 stages, rows in order) into fpart.
  auto adj_stage0 = [&](int set, int n0, int j) {
    const double F = a.Ftab[n0 + j];
    const double2* kin = a.kb[0];
    for (int k = tg; k < wlen; k += RTHREADS) awin[k] = ld_cg(kin + wlo + k);
    group_sync(1);
    for (int li = warp; li < nrows; li += RWARPS) {
      const int i = row0 + li;
      int L = 0;
      while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
      double wr, wi;
      row_coupling(g, crow + roff[li], awin, wlo, L, lane, wr, wi);
      if (lane == 0) {
        const double e = a.eps[i];
        const double2 kv = awin[i - wlo];
        const double2 m1 = (a.gauge == 0) ? make_double2(wi, -wr) : make_double2(wr, wi);
        const double2 yb = make_double2(-(__dmul_rn(e, kv.y) + __dmul_rn(F, m1.x)),
                                        -(__dmul_rn(-e, kv.x) + __dmul_rn(F, m1.y)));
        ybs[li] = yb;
        const double2 y = ld_cg(a.segX[set] + vp * j + i);
        frow[li] = -(__dmul_rn(m1.x, y.x) + __dmul_rn(m1.y, y.y));
      }
    }
    group_sync(1);
    if (tg == 0) {
      double t = 0.0;
      for (int li = 0; li < nrows; ++li) t += frow[li];
      a.fpart[(long long)(n0 + j) * G + c] = fcta_sh + t;
      fcta_sh = 0.0;
    }
    for (int li = tg; li < nrows; li += RTHREADS) {
      double2 o = zbs[li];
      for (int sp = 0; sp < kNumStages; ++sp) {
        const double2 w = ybs[sp * nrows + li];
        o.x = __dadd_rn(o.x, w.x);
        o.y = __dadd_rn(o.y, w.y);
      }
      lams[li] = o;
    }
    group_sync(1);
  };

  for (int it = 0; it <= a.nseg && !dead; ++it) {
    const int rseg = a.nseg - 1 - it;   // recomputed segment (forward group)
    const int aseg = a.nseg - it;       // swept segment (adjoint group)
    const int lenF = rseg >= 0 ? min(K, a.steps - rseg * K) : 0;
    const int lenA = aseg <= a.nseg - 1 ? min(K, a.steps - aseg * K) : 0;
    const int fset = rseg & 1, aset = aseg & 1;
    const int slots = max(lenF, lenA);
    for (int slot = 0; slot < slots && !dead; ++slot) {
      for (int tick = 0; tick < 14; ++tick) {
        if (grp == 0 && slot < lenF && tick < kNumStages) {
          // ---------------- recompute: stage `tick` of step `slot` ----------------
          const int j = slot, st = tick;
          const int n0 = rseg * K;
          const double F = a.Ftab[n0 + j];
          double2* sx = a.segX[fset];
          double2* sy = a.segY[fset];
          if (st == 0) {
            if (j > 0) {
              if (tg < 32) {
                double sum = 0.0;
                for (int p = tg; p < G; p += 32) sum += __ldcg(a.part_f + p);
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                if (tg == 0) nrm_sh = sqrt(sum);
              }
              group_sync(0);
            }
            const double nrm = j > 0 ? nrm_sh : 1.0;
            const double2* src = j > 0 ? a.XN : a.ckpt + vp * rseg;
            for (int k = tg; k < wlen; k += RTHREADS) {
              const double2 v = ld_cg(src + wlo + k);
              ywin[k] = j > 0 ? make_double2(v.x / nrm, v.y / nrm) : v;
            }
            group_sync(0);
            for (int li = tg; li < nrows; li += RTHREADS) {
              const double2 v = ywin[row0 + li - wlo];
              xsm[li] = v;
              sx[vp * j + row0 + li] = v;
            }
            if (c == 0 && tg == 0 && j > 0) a.segN[fset][j - 1] = nrm;
          } else {
            const double2* yin = sy + vp * (j * 13LL + st);
            for (int k = tg; k < wlen; k += RTHREADS) ywin[k] = ld_cg(yin + wlo + k);
          }
          group_sync(0);
          for (int li = warp; li < nrows; li += RWARPS) {
            const int i = row0 + li;
            int L = 0;
            while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
            double wr, wi;
            row_coupling(g, crow + roff[li], ywin, wlo, L, lane, wr, wi);
            if (lane == 0) {
              const double e = a.eps[i];
              const double2 y = ywin[i - wlo];
              double kre, kim;
              if (a.gauge == 0) {
                kre = __dadd_rn(__dmul_rn(e, y.y), __dmul_rn(F, wi));
                kim = __dadd_rn(__dmul_rn(-e, y.x), __dmul_rn(-F, wr));
              } else {
                kre = __dadd_rn(__dmul_rn(e, y.y), __dmul_rn(F, wr));
                kim = __dadd_rn(__dmul_rn(-e, y.x), __dmul_rn(F, wi));
              }
              ksm[st * nrows + li] = make_double2(kre, kim);
            }
          }
          group_sync(0);
          const bool last = (st == kNumStages - 1);
          double nsq = 0.0;
          for (int li = tg; li < nrows; li += RTHREADS) {
            double2 acc = xsm[li];
            for (int jj = 0; jj <= st; ++jj) {
              const double cj = last ? r_B8[jj] : r_A[st + 1][jj];
              if (cj == 0.0) continue;
              const double cf = h * cj;
              const double2 kj = ksm[jj * nrows + li];
              acc.x = __dadd_rn(acc.x, __dmul_rn(cf, kj.x));
              acc.y = __dadd_rn(acc.y, __dmul_rn(cf, kj.y));
            }
            if (last) {
              a.XN[row0 + li] = acc;
              nsq += __dadd_rn(__dmul_rn(acc.x, acc.x), __dmul_rn(acc.y, acc.y));
            } else {
              sy[vp * (j * 13LL + st + 1) + row0 + li] = acc;
            }
          }
          if (last) {
            for (int o = 16; o > 0; o >>= 1) nsq += __shfl_xor_sync(0xffffffffu, nsq, o);
            if (lane == 0) redf[warp] = nsq;
            group_sync(0);
            if (tg == 0) {
              double t = redf[0];
              for (int w = 1; w < RWARPS; ++w) t += redf[w];
              a.part_f[c] = t;
            }
          }
        } else if (grp == 1 && slot < lenA) {
          // ---------------- sweep: phase `tick` of step lenA-1-slot ----------------
          const int j = lenA - 1 - slot;
          const int n0 = aseg * K;
          const double2* x1 = a.segX[aset] + vp * (j + 1);
          if (tick == 0) {
            if (slot > 0) adj_stage0(aset, n0, j + 1);
            double v = 0.0;
            for (int li = tg; li < nrows; li += RTHREADS) {
              const double2 x = ld_cg(x1 + row0 + li), l = lams[li];
              v += __dadd_rn(__dmul_rn(x.x, l.x), __dmul_rn(x.y, l.y));
            }
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) reda[warp] = v;
            group_sync(1);
            if (tg == 0) {
              double t = reda[0];
              for (int w = 1; w < RWARPS; ++w) t += reda[w];
              a.part_a[c] = t;
            }
          } else if (tick == 1) {
            if (tg < 32) {
              double t = 0.0;
              for (int p = tg; p < G; p += 32) t += __ldcg(a.part_a + p);
              for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
              if (tg == 0) d_sh = t;
            }
            group_sync(1);
            const double d = d_sh, nz = __ldcg(a.segN[aset] + j),
                         hb = h * r_B8[kNumStages - 1];
            for (int li = tg; li < nrows; li += RTHREADS) {
              const double2 l = lams[li], x = ld_cg(x1 + row0 + li);
              const double2 z = make_double2((l.x - x.x * d) / nz, (l.y - x.y * d) / nz);
              zbs[li] = z;
              a.kb[0][row0 + li] = make_double2(hb * z.x, hb * z.y);
            }
          } else {
            const int st = 14 - tick;   // 12 .. 1
            const double F = a.Ftab[n0 + j];
            const double2* kin = a.kb[st & 1];
            for (int k = tg; k < wlen; k += RTHREADS) awin[k] = ld_cg(kin + wlo + k);
            group_sync(1);
            for (int li = warp; li < nrows; li += RWARPS) {
              const int i = row0 + li;
              int L = 0;
              while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
              double wr, wi;
              row_coupling(g, crow + roff[li], awin, wlo, L, lane, wr, wi);
              if (lane == 0) {
                const double e = a.eps[i];
                const double2 kv = awin[i - wlo];
                const double2 m1 = (a.gauge == 0) ? make_double2(wi, -wr) : make_double2(wr, wi);
                const double2 yb = make_double2(-(__dmul_rn(e, kv.y) + __dmul_rn(F, m1.x)),
                                                -(__dmul_rn(-e, kv.x) + __dmul_rn(F, m1.y)));
                ybs[st * nrows + li] = yb;
                const double2 y = ld_cg(a.segY[aset] + vp * (j * 13LL + st) + i);
                frow[li] = -(__dmul_rn(m1.x, y.x) + __dmul_rn(m1.y, y.y));
              }
            }
            group_sync(1);
            if (tg == 0) {
              double t = 0.0;
              for (int li = 0; li < nrows; ++li) t += frow[li];
              fcta_sh += t;
            }
            double2* kout = a.kb[(st + 1) & 1];
            const double cb = h * r_B8[st - 1];
            for (int li = tg; li < nrows; li += RTHREADS) {
              const double2 z = zbs[li];
              double2 o = make_double2(__dmul_rn(cb, z.x), __dmul_rn(cb, z.y));
              for (int sp = st; sp < kNumStages; ++sp) {
                const double cf = r_At[st - 1][sp];
                if (cf == 0.0) continue;
                const double2 w = ybs[sp * nrows + li];
                const double cc = h * cf;
                o.x = __dadd_rn(o.x, __dmul_rn(cc, w.x));
                o.y = __dadd_rn(o.y, __dmul_rn(cc, w.y));
              }
              kout[row0 + li] = o;
            }
          }
        }
        if (!bar_sync(a.bar, a.status, a.bc, epoch, dead)) break;
      }
    }
    if (dead) break;
    // ---- closing tick: the forward group's last normalisation, the adjoint
    // group's stage 0 of the segment's first step ----
    if (grp == 0 && lenF > 0) {
      if (tg < 32) {
        double sum = 0.0;
        for (int p = tg; p < G; p += 32) sum += __ldcg(a.part_f + p);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (tg == 0) nrm_sh = sqrt(sum);
      }
      group_sync(0);
      const double nrm = nrm_sh;
      if (c == 0 && tg == 0) {
        a.segN[fset][lenF - 1] = nrm;
        if (!(nrm > 0.0) || !isfinite(nrm)) atomicOr(a.status, ST_NONFINITE);
      }
      for (int li = tg; li < nrows; li += RTHREADS) {
        const double2 v = ld_cg(a.XN + row0 + li);
        a.segX[fset][vp * lenF + row0 + li] = make_double2(v.x / nrm, v.y / nrm);
      }
    } else if (grp == 1 && lenA > 0) {
      adj_stage0(aset, aseg * K, 0);
    }
    if (!bar_sync(a.bar, a.status, a.bc, epoch, dead)) break;
  }
  if (dead) return;
  if (grp == 1)
    for (int li = tg; li < nrows; li += RTHREADS) a.lam[row0 + li] = lams[li];
}

size_t resident_smem(const Geometry& g, int G, int* max_rows) {
  size_t best = 0;
  int mr = 0;
  for (int c = 0; c < G; ++c) {
    const int row0 = (int)((long long)g.ntot * c / G), row1 = (int)((long long)g.ntot * (c + 1) / G);
    const int nrows = row1 - row0;
    mr = std::max(mr, nrows);
    int Llo = 0;
    while (Llo + 1 < g.nstate_blk && row0 >= g.state_off[Llo + 1]) ++Llo;
    int Lhi = Llo;
    while (Lhi + 1 < g.nstate_blk && row1 - 1 >= g.state_off[Lhi + 1]) ++Lhi;
    const int wlen = g.state_off[std::min(Lhi + 2, g.nstate_blk)] - g.state_off[std::max(Llo - 1, 0)];
    size_t cr = 0;
    for (int i = row0; i < row1; ++i) {
      int L = 0;
      while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
      cr += (L > 0 ? g.state_off[L] - g.state_off[L - 1] : 0) +
            (L < g.nblk ? g.state_off[L + 2] - g.state_off[L + 1] : 0);
    }
    const size_t bytes = 16 * ((4 * (kMaxRowsPerCta + 1) + 15) / 16) + 16 * (size_t)wlen +
                         16 * (size_t)kNumStages * nrows + 16 * (size_t)nrows + 8 * cr;
    best = std::max(best, bytes);
  }
  *max_rows = mr;
  return best;
}

// Shared memory of the fused reverse-pass kernel: the resident layout plus a
// second window and the adjoint group's per-row vectors.
size_t fused_smem(const Geometry& g, int G) {
  size_t best = 0;
  for (int c = 0; c < G; ++c) {
    const int row0 = (int)((long long)g.ntot * c / G), row1 = (int)((long long)g.ntot * (c + 1) / G);
    const int nrows = row1 - row0;
    int Llo = 0;
    while (Llo + 1 < g.nstate_blk && row0 >= g.state_off[Llo + 1]) ++Llo;
    int Lhi = Llo;
    while (Lhi + 1 < g.nstate_blk && row1 - 1 >= g.state_off[Lhi + 1]) ++Lhi;
    const int wlen = g.state_off[std::min(Lhi + 2, g.nstate_blk)] - g.state_off[std::max(Llo - 1, 0)];
    size_t cr = 0;
    for (int i = row0; i < row1; ++i) {
      int L = 0;
      while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
      cr += (L > 0 ? g.state_off[L] - g.state_off[L - 1] : 0) +
            (L < g.nblk ? g.state_off[L + 2] - g.state_off[L + 1] : 0);
    }
    const size_t bytes = 16 * ((4 * (kMaxRowsPerCta + 1) + 15) / 16) + 2 * 16 * (size_t)wlen +
                         2 * 16 * (size_t)kNumStages * nrows + 3 * 16 * (size_t)nrows +
                         8 * (size_t)((nrows + 1) & ~1) + 8 * cr;
    best = std::max(best, bytes);
  }
  return best;
}

}  // namespace

struct mpc_resident_state {
  int G = 0;
  size_t smem = 0;
  size_t smem_adj = 0;
  bool adj_ok = false;      // the adjoint sweep kernel fits as well
  double2* kb = nullptr;    // [2][ntot] kbar ping-pong of the adjoint sweep
  double* fpart = nullptr;  // [fpart_cap][G]
  int fpart_cap = 0;
  double2* Y0 = nullptr;
  double2* Y1 = nullptr;
  double2* XN = nullptr;
  double* part = nullptr;
  unsigned* bar = nullptr;  // 64-bit arrival counter
  bool ok = false;
  int fused = -1;           // the fused reverse pass fits (-1: not checked yet)
  size_t smem_fused = 0;
  double* part_a = nullptr; // [G] the fused kernel's adjoint-group partials
};

// Sets up the resident path if the system fits; returns true when usable.
bool mpc_resident_setup(mpc_ctx* c) {
  if (c->resident) return c->resident->ok;
  mpc_resident_state* r = new mpc_resident_state();
  c->resident = r;
  if (std::getenv("MPC_NO_RESIDENT")) return false;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
  if (!coop) return false;
  const int G = c->num_sms;
  int max_rows = 0;
  const size_t smem = resident_smem(c->g, G, &max_rows);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (max_rows > kMaxRowsPerCta || smem + 2048 > (size_t)optin) return false;
  if (cudaFuncSetAttribute(k_prop_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return false;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prop_resident, RTHREADS, smem) !=
          cudaSuccess ||
      per_sm < 1)
    return false;
  double A[13][13], B8[13];
  for (int i = 0; i < 13; ++i) {
    B8[i] = rkf78::B8[i];
    for (int j = 0; j < 13; ++j) A[i][j] = rkf78::A[i][j];
  }
  double At[13][13];
  for (int i = 0; i < 13; ++i)
    for (int j = 0; j < 13; ++j) At[i][j] = rkf78::A[j][i];
  if (cudaMemcpyToSymbol(r_A, A, sizeof A) != cudaSuccess ||
      cudaMemcpyToSymbol(r_B8, B8, sizeof B8) != cudaSuccess ||
      cudaMemcpyToSymbol(r_At, At, sizeof At) != cudaSuccess)
    return false;
  // the adjoint sweep: two more vectors and a double per row
  const size_t smem_adj = smem + 24 * (size_t)max_rows + 16;
  int per_sm_adj = 0;
  if (smem_adj + 2048 <= (size_t)optin &&
      cudaFuncSetAttribute(k_adj_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem_adj) == cudaSuccess &&
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_adj, k_adj_resident, RTHREADS,
                                                    smem_adj) == cudaSuccess &&
      per_sm_adj >= 1) {
    r->smem_adj = smem_adj;
    r->adj_ok = true;
  }
  cudaGetLastError();
  const size_t n = c->g.ntot;
  if (cudaMalloc(&r->Y0, sizeof(double2) * n) != cudaSuccess ||
      cudaMalloc(&r->Y1, sizeof(double2) * n) != cudaSuccess ||
      cudaMalloc(&r->XN, sizeof(double2) * n) != cudaSuccess ||
      cudaMalloc(&r->part, sizeof(double) * G) != cudaSuccess ||
      cudaMalloc(&r->bar, sizeof(unsigned) * 2) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream);
  r->G = G;
  r->smem = smem;
  r->ok = true;
  return true;
}

void mpc_resident_free(mpc_ctx* c) {
  if (!c || !c->resident) return;
  mpc_resident_state* r = c->resident;
  cudaFree(r->kb);
  cudaFree(r->fpart);
  cudaFree(r->Y0);
  cudaFree(r->Y1);
  cudaFree(r->XN);
  cudaFree(r->part);
  cudaFree(r->part_a);
  cudaFree(r->bar);
  delete r;
  c->resident = nullptr;
}

// Runs `steps` steps of the fixed-step loop on the state in c->d_x with the
// field table already in c->d_Ftab; histories into c->d_pop / c->d_nrm.
int mpc_resident_run(mpc_ctx* c, double dt, int steps, int pop_index) {
  mpc_resident_state* r = c->resident;
  ResArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.Ftab = c->d_Ftab;
  a.Y[0] = r->Y0;
  a.Y[1] = r->Y1;
  a.XN = r->XN;
  a.xout = c->d_x;
  a.norm_part = r->part;
  a.bar = r->bar;
  a.status = c->d_status;
  a.pop_hist = c->d_pop;
  a.norm_hist = c->d_nrm;
  a.pop_index = pop_index;
  a.steps = steps;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.first_is_normalised = 1;
  a.dt = dt;
  a.bc = mpc_barrier_cfg(c);
  a.g = c->g;
  CK(cudaMemcpyAsync(r->XN, c->d_x, sizeof(double2) * c->g.ntot, cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream));  // arrival counter
  void* args[] = {&a};
  ProfScope ps(c, MPC_KERNEL_RESIDENT);
  CK(cudaLaunchCooperativeKernel((const void*)k_prop_resident, dim3(r->G), dim3(RTHREADS), args,
                                 r->smem, c->stream));
  return MPC_OK;
}

// The fixed-step loop from x_in (device, normalised or as given) for `steps`
// steps with the field table Ftab, result (normalised) into x_out; optional
// outputs for the objective gradient: seg_x / seg_y / norm_hist (every step's
// state, stage inputs and norm) and ckpt (the state every ckpt_every steps),
// slots vpitch complex apart.
int mpc_resident_forward_ex(mpc_ctx* c, const double2* x_in, double2* x_out, const double* Ftab,
                            double dt, int steps, double2* seg_x, double2* seg_y,
                            double* norm_hist, double2* ckpt, int ckpt_every, long long vpitch) {
  mpc_resident_state* r = c->resident;
  ResArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.Ftab = Ftab;
  a.Y[0] = r->Y0;
  a.Y[1] = r->Y1;
  a.XN = r->XN;
  a.xout = x_out;
  a.norm_part = r->part;
  a.bar = r->bar;
  a.status = c->d_status;
  a.pop_hist = nullptr;
  a.norm_hist = norm_hist;
  a.pop_index = -1;
  a.steps = steps;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.first_is_normalised = 1;
  a.dt = dt;
  a.seg_x = seg_x;
  a.seg_y = seg_y;
  a.ckpt = ckpt;
  a.ckpt_every = ckpt_every > 0 ? ckpt_every : 1;
  a.vpitch = vpitch;
  a.bc = mpc_barrier_cfg(c);
  a.g = c->g;
  CK(cudaMemcpyAsync(r->XN, x_in, sizeof(double2) * c->g.ntot, cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream));
  void* args[] = {&a};
  ProfScope ps(c, MPC_KERNEL_RESIDENT);
  CK(cudaLaunchCooperativeKernel((const void*)k_prop_resident, dim3(r->G), dim3(RTHREADS), args,
                                 r->smem, c->stream));
  ++c->launches;
  return MPC_OK;
}

bool mpc_resident_adjoint_ok(mpc_ctx* c) { return c->resident && c->resident->adj_ok; }

// The adjoint sweep of one segment of len steps (see k_adj_resident); lam in
// and out (device, ntot), dJ/dF of the segment's steps into fbar [len].
int mpc_resident_adjoint(mpc_ctx* c, const double* Ftab, double dt, int len,
                         const double2* seg_x, const double2* seg_y, const double* seg_n,
                         double2* lam, double* fbar, long long vpitch) {
  mpc_resident_state* r = c->resident;
  if (!r || !r->adj_ok) return mpc_fail(MPC_ERR_ARG, "resident adjoint unavailable");
  if (!r->kb) CK(cudaMalloc(&r->kb, sizeof(double2) * 2 * (size_t)c->g.ntot));
  if (r->fpart_cap < len) {
    cudaFree(r->fpart);
    r->fpart = nullptr;
    CK(cudaMalloc(&r->fpart, sizeof(double) * (size_t)len * r->G));
    r->fpart_cap = len;
  }
  AdjResArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.Ftab = Ftab;
  a.seg_x = seg_x;
  a.seg_y = seg_y;
  a.seg_n = seg_n;
  a.lam = lam;
  a.kb[0] = r->kb;
  a.kb[1] = r->kb + c->g.ntot;
  a.part = r->part;
  a.fpart = r->fpart;
  a.bar = r->bar;
  a.status = c->d_status;
  a.len = len;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.dt = dt;
  a.vpitch = vpitch;
  a.bc = mpc_barrier_cfg(c);
  a.g = c->g;
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream));
  void* args[] = {&a};
  {
    ProfScope ps(c, MPC_KERNEL_RESIDENT);
    CK(cudaLaunchCooperativeKernel((const void*)k_adj_resident, dim3(r->G), dim3(RTHREADS), args,
                                   r->smem_adj, c->stream));
  }
  k_adj_res_fbar<<<(len + 127) / 128, 128, 0, c->stream>>>(r->fpart, len, r->G, fbar);
  CK(cudaGetLastError());
  c->launches += 2;
  return MPC_OK;
}

// The whole reverse pass in one persistent launch (k_adj_fused): segment
// nseg-1 is recomputed from its checkpoint, then every iteration sweeps one
// segment while recomputing the one before it, into the other buffer set;
// lam in (lambda_N) and out (lambda_0); dJ/dF of every step into fbar
// [steps].  Returns MPC_ERR_ARG (nothing launched) when the kernel does not
// fit on this system, so the caller can take the per-segment path.
bool mpc_resident_fused_ok(mpc_ctx* c) {
  mpc_resident_state* r = c->resident;
  if (!r || !r->ok || !r->adj_ok) return false;
  if (r->fused >= 0) return r->fused == 1;
  r->fused = 0;
  if (std::getenv("MPC_NO_FUSED_ADJOINT")) return false;
  const size_t smem = fused_smem(c->g, r->G);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  int per_sm = 0;
  if (smem + 2048 <= (size_t)optin &&
      cudaFuncSetAttribute(k_adj_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) == cudaSuccess &&
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_fused, 2 * RTHREADS, smem) ==
          cudaSuccess &&
      per_sm >= 1 && cudaMalloc(&r->part_a, sizeof(double) * r->G) == cudaSuccess) {
    r->smem_fused = smem;
    r->fused = 1;
  }
  cudaGetLastError();
  return r->fused == 1;
}

int mpc_resident_backward_fused(mpc_ctx* c, const double2* ckpts, int steps, int ckpt_every,
                                const double* Ftab, double dt, double2* const* segX,
                                double2* const* segY, double* const* segN, double2* lam,
                                double* fbar, long long vpitch) {
  mpc_resident_state* r = c->resident;
  if (!mpc_resident_fused_ok(c)) return mpc_fail(MPC_ERR_ARG, "fused reverse pass unavailable");
  if (!r->kb) CK(cudaMalloc(&r->kb, sizeof(double2) * 2 * (size_t)c->g.ntot));
  if (r->fpart_cap < steps) {
    cudaFree(r->fpart);
    r->fpart = nullptr;
    CK(cudaMalloc(&r->fpart, sizeof(double) * (size_t)steps * r->G));
    r->fpart_cap = steps;
  }
  FusedArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.Ftab = Ftab;
  a.ckpt = ckpts;
  for (int k = 0; k < 2; ++k) {
    a.segX[k] = segX[k];
    a.segY[k] = segY[k];
    a.segN[k] = segN[k];
  }
  a.XN = r->XN;
  a.part_f = r->part;
  a.lam = lam;
  a.kb[0] = r->kb;
  a.kb[1] = r->kb + c->g.ntot;
  a.part_a = r->part_a;
  a.fpart = r->fpart;
  a.bar = r->bar;
  a.status = c->d_status;
  a.steps = steps;
  a.ckpt_every = ckpt_every;
  a.nseg = (steps + ckpt_every - 1) / ckpt_every;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.dt = dt;
  a.vpitch = vpitch;
  a.bc = mpc_barrier_cfg(c);
  a.g = c->g;
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned) * 2, c->stream));
  void* args[] = {&a};
  {
    ProfScope ps(c, MPC_KERNEL_RESIDENT);
    CK(cudaLaunchCooperativeKernel((const void*)k_adj_fused, dim3(r->G), dim3(2 * RTHREADS), args,
                                   r->smem_fused, c->stream));
  }
  k_adj_res_fbar<<<(steps + 127) / 128, 128, 0, c->stream>>>(r->fpart, steps, r->G, fbar);
  CK(cudaGetLastError());
  c->launches += 2;
  return MPC_OK;
}
