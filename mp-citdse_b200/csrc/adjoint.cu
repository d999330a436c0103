// adjoint.cu -- gradient of an objective of the final state with respect to
// control samples of E(t), by the discrete adjoint of the fixed-step
// propagation (the reference has no gradients; this is new).
//
// Forward (as tdse::propL / propV, src/tdse/tdse.cpp:186-215): per step n the
// field F_n = base(t_n + dt) + dE(t_n + dt) is frozen, the 13 RKF78 stages
// give z_n = x_n + h sum_j b_j k_j, and x_{n+1} = z_n / ||z_n||.  The control
// perturbation dE(t) = sum_k u_k phi((t - t_k)/g) is piecewise cubic
// (Catmull-Rom / Keys a = -1/2 kernel) over K samples on [0, T].
// Objective J(x_N): the yield above a threshold, 1 - sum_{E_i < thr} |x_i|^2
// (thr = 0: ionisation of a 1e system, double ionisation of a 2e system whose
// energies are given relative to the doubly-charged ion; thr = the ion's
// ground-state energy: single ionisation), or the population |x_target|^2.
// Since every step renormalises, ||x_N|| = 1 and the yield is evaluated as
// sum_{E_i >= thr} |x_i|^2, which keeps small yields (double ionisation,
// ~1e-6) free of the cancellation in 1 - (1 - J); its seed 2 x on those states
// differs from -2 x on the others by 2 x_N, which the adjoint of the
// normalisation removes.
//
// Reverse mode.  The generator M(F) = -i(H0 + F S) (length) or -i H0 + F K
// (velocity) is anti-Hermitian, so for the real inner product Re<u, v> its
// transpose is -M(F): the adjoint of one step is the step's stage structure
// transposed and run backwards with the same right-hand-side kernels:
//   zbar   = (lam - x_{n+1} Re<x_{n+1}, lam>) / ||z_n||
//   kbar_s = h b_s zbar + sum_{s'>s} h a_{s's} ybar_{s'}     (s = 12 .. 0)
//   ybar_s = -M(F_n) kbar_s
//   dJ/dF_n += -Re<M1 kbar_s, y_s>,  M1 = dM/dF (anti-Hermitian too)
//   lam_n  = zbar + sum_s ybar_s
// and dJ/du_k = sum_n dJ/dF_n phi((t_n + dt - t_k)/g).
// Memory: the forward keeps x every `ckpt` steps; the reverse pass re-runs
// each segment forward from its checkpoint, keeping the segment's states,
// stage inputs y_s and norms, then walks it backwards.  Cost: one forward,
// one recomputed forward, one adjoint sweep (about 3 forwards).  When the
// couplings fit in shared memory (the resident path) each pass is one
// persistent launch (resident.cu: the forward with checkpoint / segment
// outputs, and k_adj_resident for the sweep); otherwise the streamed kernels
// below run step by step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"
#include "dev_util.cuh"
#include "plan.h"
#include "rkf78.h"

using namespace mpc;

namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }

// per-CTA partials of Re<a, b>
__global__ void k_adj_dot(const double2* a, const double2* b, double* part, int ntot) {
  pdl_trigger();
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < ntot) {
    const double2 x = a[i], y = b[i];
    v = da(dm(x.x, y.x), dm(x.y, y.y));
  }
  __shared__ double sh[8];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = sh[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    part[blockIdx.x] = s;
  }
}

// zbar = (lam - x1 * d) / nrm with d = sum(part) (fixed order); also the
// first adjoint stage input v = h b_12 zbar.
__global__ void k_adj_zbar(const double2* lam, const double2* x1, const double* part, int nparts,
                           const double* nrm, double2* zbar, double2* v, double hb12, int ntot) {
  pdl_trigger();
  pdl_wait();
  __shared__ double d_sh;
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int p = threadIdx.x; p < nparts; p += 32) s += part[p];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) d_sh = s;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  const double d = d_sh, nr = *nrm;
  const double2 l = lam[i], x = x1[i];
  const double2 z = make_double2((l.x - x.x * d) / nr, (l.y - x.y * d) / nr);
  zbar[i] = z;
  v[i] = make_double2(hb12 * z.x, hb12 * z.y);
}

struct AdjCombineArgs {
  double2* v;              // in: kbar_s; out: kbar_{s-1}
  const double2* ys;       // forward stage input y_s of this step
  const double2* zbar;
  double2* ybar;           // [13][ntot]: ybar_s slots
  double2* lam;            // out (s == 0): lam_n
  const double* eps;
  const double2* RP;
  const double2* CP;
  const int* strip_slot0;
  const double* Ftab;
  double* fpart;           // [13][nblocks] partials of dJ/dF
  int step;
  int stage;
  int gauge;
  double h;
  Geometry g;
};

__constant__ double c_At[13][13];   // a_{s', s}: row s, column s'
__constant__ double c_b8[13];

__global__ void __launch_bounds__(kCombineThreads) k_adj_combine(const __grid_constant__ AdjCombineArgs a) {
  pdl_trigger();
  pdl_wait();
  const Geometry& g = a.g;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = gt / kCombineLanes, q = gt % kCombineLanes;
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
        const double2 w = rp[s * (long long)b.nrow];
        Q.x = da(Q.x, w.x);
        Q.y = da(Q.y, w.y);
      }
    }
    if (L > 0) {
      const BlockGeom& b = g.blk[L - 1];
      const int gs = b.strip0 + r / kStripW, c = r % kStripW;
      const int s1 = a.strip_slot0[gs + 1];
      for (int sl = a.strip_slot0[gs] + q; sl < s1; sl += kCombineLanes) {
        const double2 w = a.CP[(long long)sl * kStripW + c];
        P.x = da(P.x, w.x);
        P.y = da(P.y, w.y);
      }
    }
  }
#pragma unroll
  for (int o = 1; o < kCombineLanes; o <<= 1) {
    Q.x = da(Q.x, __shfl_xor_sync(0xffffffffu, Q.x, o));
    Q.y = da(Q.y, __shfl_xor_sync(0xffffffffu, Q.y, o));
    P.x = da(P.x, __shfl_xor_sync(0xffffffffu, P.x, o));
    P.y = da(P.y, __shfl_xor_sync(0xffffffffu, P.y, o));
  }
  double fp = 0.0;
  if (valid && q == 0) {
    const long long n = g.ntot;
    const int s = a.stage;
    const double F = a.Ftab[a.step];
    const double e = a.eps[i];
    const double2 v = a.v[i];
    // M1 v: length -i (P + Q), velocity (P - Q)
    double2 m1;
    if (a.gauge == 0) {
      const double sr = (L > 0 ? P.x : 0.0) + (L < g.nblk ? Q.x : 0.0);
      const double si = (L > 0 ? P.y : 0.0) + (L < g.nblk ? Q.y : 0.0);
      m1 = make_double2(si, -sr);
    } else {
      m1 = make_double2((L > 0 ? P.x : 0.0) - (L < g.nblk ? Q.x : 0.0),
                        (L > 0 ? P.y : 0.0) - (L < g.nblk ? Q.y : 0.0));
    }
    // ybar_s = -M v = -(-i e v + F M1 v)
    const double2 yb = make_double2(-(dm(e, v.y) + dm(F, m1.x)), -(dm(-e, v.x) + dm(F, m1.y)));
    a.ybar[s * n + i] = yb;
    const double2 y = a.ys[i];
    fp = -(dm(m1.x, y.x) + dm(m1.y, y.y));
    if (s > 0) {
      // kbar_{s-1} = h b_{s-1} zbar + sum_{s' >= s} h a_{s', s-1} ybar_{s'}
      const double2 z = a.zbar[i];
      const double cb = a.h * c_b8[s - 1];
      double2 o = make_double2(dm(cb, z.x), dm(cb, z.y));
      for (int sp = s; sp < kNumStages; ++sp) {
        const double cf = c_At[s - 1][sp];
        if (cf == 0.0) continue;
        const double2 w = (sp == s) ? yb : a.ybar[sp * n + i];
        const double c = a.h * cf;
        o.x = da(o.x, dm(c, w.x));
        o.y = da(o.y, dm(c, w.y));
      }
      a.v[i] = o;
    } else {
      // lam_n = zbar + sum_s ybar_s
      double2 o = a.zbar[i];
      for (int sp = 0; sp < kNumStages; ++sp) {
        const double2 w = (sp == 0) ? yb : a.ybar[sp * n + i];
        o.x = da(o.x, w.x);
        o.y = da(o.y, w.y);
      }
      a.lam[i] = o;
    }
  }
  __shared__ double sh[kCombineThreads / 32];
  for (int o = 16; o > 0; o >>= 1) fp += __shfl_xor_sync(0xffffffffu, fp, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = fp;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = sh[0];
    for (int w = 1; w < kCombineThreads / 32; ++w) s += sh[w];
    a.fpart[a.stage * gridDim.x + blockIdx.x] = s;
  }
}

// dJ/dF_n = sum over stages and CTAs of the partials (fixed order).
__global__ void k_adj_fbar(const double* fpart, int nblocks, double* fbar_n) {
  pdl_trigger();
  pdl_wait();
  if (threadIdx.x >= 32) return;
  double s = 0.0;
  for (int p = threadIdx.x; p < kNumStages * nblocks; p += 32) s += fpart[p];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *fbar_n = s;
}

// lam_N = dJ/dx_N: yield -> 2 x on the states at or above the threshold;
// target -> 2 x_t.
__global__ void k_adj_seed(const double2* x, const double* eps, double2* lam, int target,
                           double thr, int ntot) {
  pdl_trigger();
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  const double2 v = x[i];
  double2 o = make_double2(0.0, 0.0);
  if (target < 0) {
    if (eps[i] >= thr) o = make_double2(2.0 * v.x, 2.0 * v.y);
  } else if (i == target) {
    o = make_double2(2.0 * v.x, 2.0 * v.y);
  }
  lam[i] = o;
}

}  // namespace

static double keys_phi(double s) {
  const double x = std::fabs(s);
  if (x < 1.0) return (1.5 * x - 2.5) * x * x + 1.0;
  if (x < 2.0) return ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0;
  return 0.0;
}

// dE(t) and the 4 weights it takes from the samples (first index in *k0)
double mpc_control_at(int K, const double* u, double T, double t, int* k0, double* w) {
  for (int j = 0; j < 4; ++j) w[j] = 0.0;
  *k0 = 0;
  if (K < 2 || t < 0.0 || t > T) return 0.0;
  const double gsp = T / (double)(K - 1);
  const double qq = t / gsp;
  const int i0 = (int)std::floor(qq);
  *k0 = i0 - 1;
  double acc = 0.0;
  for (int j = 0; j < 4; ++j) {
    const int k = i0 - 1 + j;
    if (k < 0 || k >= K) continue;
    w[j] = keys_phi(qq - (double)k);
    acc += u[k] * w[j];
  }
  return acc;
}

struct mpc_adjoint_state {
  int steps = 0, ckpt = 0, nseg = 0, target = -1, K = 0;
  double dt = 0.0, T = 0.0, t0 = 0.0;
  mpc_pulse pulse{};
  std::vector<double> u, F, tn;
  double2* ckpts = nullptr;   // [nseg + 1][ntot]
  double2* segX = nullptr;    // [ckpt + 1][ntot]
  double2* segY = nullptr;    // [ckpt][13][ntot]  (slot 0 unused: y_0 = x_n)
  double* segN = nullptr;     // [ckpt]
  // a second segment buffer set for the fused reverse pass (recompute of one
  // segment while the previous one is swept), allocated on first use
  double2* segX2 = nullptr;
  double2* segY2 = nullptr;
  double* segN2 = nullptr;
  double2* lam = nullptr;
  double2* zbar = nullptr;
  double2* v = nullptr;
  double2* ybar = nullptr;    // [13][ntot]
  double* part = nullptr;
  double* fpart = nullptr;    // [13][nblocks]
  double* fbar = nullptr;     // [steps]
  size_t cap_ckpt = 0, cap_seg = 0, cap_steps = 0;
  std::vector<void*> allocs;
  bool have_forward = false;
  bool resident = false;      // both passes on the shared-memory-resident kernels
  bool last_kept = false;     // the streamed forward kept the last segment's states
};

namespace {

template <class T>
int aalloc(mpc_adjoint_state* a, T** p, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  a->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return MPC_OK;
}

int ensure_adjoint(mpc_ctx* c, int steps, int ckpt) {
  static bool consts[64] = {};  // per device: the transposed tableau in constant memory
  if (c->device < 0 || c->device >= 64) return mpc_fail(MPC_ERR_ARG, "device %d", c->device);
  if (!consts[c->device]) {
    double At[13][13], b8[13];
    for (int s = 0; s < 13; ++s) {
      b8[s] = rkf78::B8[s];
      for (int sp = 0; sp < 13; ++sp) At[s][sp] = rkf78::A[sp][s];
    }
    CK(cudaMemcpyToSymbol(c_At, At, sizeof At));
    CK(cudaMemcpyToSymbol(c_b8, b8, sizeof b8));
    consts[c->device] = true;
  }
  const int nseg = (steps + ckpt - 1) / ckpt;
  const size_t n = c->g.ntot + kVecPad;
  mpc_adjoint_state* a = c->adj;
  if (a && a->cap_ckpt >= (size_t)nseg + 1 && a->cap_seg >= (size_t)ckpt &&
      a->cap_steps >= (size_t)steps)
    return MPC_OK;
  mpc_adjoint_free(c);
  a = new mpc_adjoint_state();
  c->adj = a;
  int rc;
  if ((rc = aalloc(a, &a->ckpts, n * (nseg + 1))) || (rc = aalloc(a, &a->segX, n * (ckpt + 1))) ||
      (rc = aalloc(a, &a->segY, n * (size_t)ckpt * kNumStages)) ||
      (rc = aalloc(a, &a->segN, ckpt)) || (rc = aalloc(a, &a->lam, n)) ||
      (rc = aalloc(a, &a->zbar, n)) || (rc = aalloc(a, &a->v, n)) ||
      (rc = aalloc(a, &a->ybar, n * kNumStages)) || (rc = aalloc(a, &a->part, c->combine_grid)) ||
      (rc = aalloc(a, &a->fpart, (size_t)kNumStages * c->combine_grid)) ||
      (rc = aalloc(a, &a->fbar, steps)))
    return rc;
  // zero the padded tails the streaming kernel may read
  CK(cudaMemsetAsync(a->ckpts, 0, sizeof(double2) * n * (nseg + 1), c->stream));
  CK(cudaMemsetAsync(a->segX, 0, sizeof(double2) * n * (ckpt + 1), c->stream));
  CK(cudaMemsetAsync(a->segY, 0, sizeof(double2) * n * (size_t)ckpt * kNumStages, c->stream));
  CK(cudaMemsetAsync(a->v, 0, sizeof(double2) * n, c->stream));
  a->cap_ckpt = nseg + 1;
  a->cap_seg = ckpt;
  a->cap_steps = steps;
  return MPC_OK;
}

// One forward step from x (stage inputs into ys[1..12], x_new into ys[13]),
// renormalised into x_next, norm into *nrm_slot.
int fwd_step(mpc_ctx* c, int step, double dt, const double2* x, double2* const* ys,
             double2* x_next, double* nrm_slot) {
  int rc;
  for (int s = 0; s < kNumStages; ++s) {
    const double2* yin = (s == 0) ? x : ys[s];
    if ((rc = mpc_launch_stream(c, yin))) return rc;
    if ((rc = mpc_launch_combine_x(c, x, s, step, dt, yin, ys[s + 1], s == kNumStages - 1, false)))
      return rc;
  }
  return mpc_launch_renorm_to(c, x_next, ys[13], step, 0, nullptr, nrm_slot, step);
}

}  // namespace

void mpc_adjoint_free(mpc_ctx* c) {
  if (!c || !c->adj) return;
  for (void* p : c->adj->allocs) cudaFree(p);
  delete c->adj;
  c->adj = nullptr;
}

extern "C" {

int mpc_objective(mpc_ctx* c, const mpc_pulse* p, int K, const double* u, double T, double t0,
                  double dt, int steps, int target, int ckpt_every, const double* ct0,
                  double* J) {
  NvtxRange nvtx_("mpc_objective (forward)");
  if (!c || !p || !ct0 || !J || steps <= 0 || !(dt > 0.0) || (K > 0 && !u) || K == 1)
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  if (target >= c->g.ntot) return mpc_fail(MPC_ERR_ARG, "target out of range");
  if (ckpt_every <= 0) ckpt_every = 64;
  if (dt * c->eps_max > kRk78ImagStability)
    return mpc_fail(MPC_ERR_UNSTABLE, "dt*max|E| = %.4g exceeds the RKF78 stability bound",
                    dt * c->eps_max);
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = ensure_adjoint(c, steps, ckpt_every))) return rc;
  mpc_adjoint_state* a = c->adj;
  a->steps = steps;
  a->ckpt = ckpt_every;
  a->nseg = (steps + ckpt_every - 1) / ckpt_every;
  a->target = target;
  a->K = K;
  a->T = T;
  a->t0 = t0;
  a->dt = dt;
  a->pulse = *p;
  a->u.assign(u, u + (K > 0 ? K : 0));
  // field table as the reference's loop accumulates t (t += dt)
  a->F.resize(steps);
  a->tn.resize(steps);
  double t = t0;
  int k0;
  double w[4];
  for (int st = 0; st < steps; ++st) {
    a->tn[st] = t + dt;
    a->F[st] = mpc_field(p, t + dt) + (K > 0 ? mpc_control_at(K, u, T, t + dt, &k0, w) : 0.0);
    t += dt;
  }
  if ((rc = mpc_fill_field_table(c, a->F.data(), steps))) return rc;
  const size_t n = c->g.ntot + kVecPad;
  const size_t nb = sizeof(double2) * c->g.ntot;
  CK(cudaMemcpyAsync(a->ckpts, ct0, nb, cudaMemcpyHostToDevice, c->stream));
  // forward, keeping a checkpoint every ckpt steps (ping-pong through segX)
  double2* ys[14];
  for (int s = 1; s <= 13; ++s) ys[s] = a->segY + n * (s - 1);  // scratch: slots of step 0
  ys[0] = nullptr;
  const double2* x = a->ckpts;
  a->resident = mpc_use_resident(c) && mpc_resident_adjoint_ok(c);
  if (a->resident) {
    // one persistent launch; it stores the checkpoints as it passes them
    if ((rc = mpc_resident_forward_ex(c, a->ckpts, a->ckpts + n * a->nseg, c->d_Ftab, dt, steps,
                                      nullptr, nullptr, nullptr, a->ckpts, ckpt_every,
                                      (long long)n)))
      return rc;
  } else {
    // the last segment keeps every state, stage input and norm as the reverse
    // pass's recompute would, so the reverse pass starts sweeping at once
    const int n0_last = (a->nseg - 1) * ckpt_every;
    for (int st = 0; st < n0_last; ++st) {
      double2* xn = ((st + 1) % ckpt_every == 0)
                        ? a->ckpts + n * ((st + 1) / ckpt_every)
                        : a->segX + n * ((st & 1) ? 0 : 1);
      if ((rc = fwd_step(c, st, dt, x, ys, xn, a->segN))) return rc;
      x = xn;
    }
    CK(cudaMemcpyAsync(a->segX, a->ckpts + n * (a->nseg - 1), sizeof(double2) * n,
                       cudaMemcpyDeviceToDevice, c->stream));
    for (int j = 0; j < steps - n0_last; ++j) {
      double2* yj[14];
      yj[0] = nullptr;
      for (int s = 1; s < kNumStages; ++s) yj[s] = a->segY + n * ((size_t)j * kNumStages + s);
      yj[13] = a->segY + n * ((size_t)j * kNumStages);  // slot 0 holds x_new (y_0 = x_n)
      if ((rc = fwd_step(c, n0_last + j, dt, a->segX + n * j, yj, a->segX + n * (j + 1),
                         a->segN + j)))
        return rc;
    }
    CK(cudaMemcpyAsync(a->ckpts + n * a->nseg, a->segX + n * (steps - n0_last),
                       sizeof(double2) * n, cudaMemcpyDeviceToDevice, c->stream));
  }
  a->last_kept = !a->resident;
  // objective on the host from x_N
  std::vector<double> xN(2 * c->g.ntot), eps(c->g.ntot);
  CK(cudaMemcpyAsync(xN.data(), a->ckpts + n * a->nseg, nb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(eps.data(), c->d_eps, sizeof(double) * c->g.ntot, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  unsigned st = 0;
  CK(cudaMemcpy(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream);
    return mpc_fail(MPC_ERR_DEVICE, "kernel status 0x%x during the forward pass", st);
  }
  if (target < 0) {
    double y = 0.0;
    for (int i = 0; i < c->g.ntot; ++i)
      if (eps[i] >= c->yield_thr) y += xN[2 * i] * xN[2 * i] + xN[2 * i + 1] * xN[2 * i + 1];
    *J = y;
  } else {
    *J = xN[2 * target] * xN[2 * target] + xN[2 * target + 1] * xN[2 * target + 1];
  }
  a->have_forward = true;
  return MPC_OK;
}

int mpc_objective_threshold(mpc_ctx* c, double thr) {
  if (!c || !std::isfinite(thr)) return mpc_fail(MPC_ERR_ARG, "bad argument");
  c->yield_thr = thr;
  if (c->adj) c->adj->have_forward = false;
  mpc_badj_invalidate(c);
  return MPC_OK;
}

int mpc_objective_backward(mpc_ctx* c, double* grad_u, double* dJdF) {
  NvtxRange nvtx_("mpc_objective_backward");
  if (!c || !c->adj || !c->adj->have_forward)
    return mpc_fail(MPC_ERR_ARG, "mpc_objective_backward needs a preceding mpc_objective");
  CK(cudaSetDevice(c->device));
  mpc_adjoint_state* a = c->adj;
  const int steps = a->steps, ckpt = a->ckpt, nseg = a->nseg;
  const double dt = a->dt;
  const size_t n = c->g.ntot + kVecPad;
  const int ntot = c->g.ntot;
  const int nbk = (ntot + 255) / 256;
  int rc;
  k_adj_seed<<<nbk, 256, 0, c->stream>>>(a->ckpts + n * nseg, c->d_eps, a->lam, a->target,
                                    c->yield_thr, ntot);
  CK(cudaGetLastError());
  AdjCombineArgs ac{};
  ac.v = a->v;
  ac.zbar = a->zbar;
  ac.ybar = a->ybar;
  ac.lam = a->lam;
  ac.eps = c->d_eps;
  ac.RP = c->d_RP;
  ac.CP = c->d_CP;
  ac.strip_slot0 = c->d_strip_slot0;
  ac.Ftab = c->d_Ftab;
  ac.fpart = a->fpart;
  ac.gauge = (c->gauge == 'l') ? 0 : 1;
  ac.h = dt;
  ac.g = c->g;
  if (a->resident && mpc_resident_fused_ok(c)) {
    // one persistent launch: each segment's recompute runs concurrently with
    // the sweep of the segment after it
    if (!a->segX2) {
      if ((rc = aalloc(a, &a->segX2, n * (ckpt + 1))) ||
          (rc = aalloc(a, &a->segY2, n * (size_t)ckpt * kNumStages)) ||
          (rc = aalloc(a, &a->segN2, ckpt)))
        return rc;
    }
    double2* sx[2] = {a->segX, a->segX2};
    double2* sy[2] = {a->segY, a->segY2};
    double* sn[2] = {a->segN, a->segN2};
    if ((rc = mpc_resident_backward_fused(c, a->ckpts, steps, ckpt, c->d_Ftab, dt, sx, sy, sn,
                                          a->lam, a->fbar, (long long)n)))
      return rc;
  }
  for (int seg = nseg - 1; seg >= 0 && !(a->resident && mpc_resident_fused_ok(c)); --seg) {
    const int n0 = seg * ckpt;
    const int len = std::min(ckpt, steps - n0);
    if (a->resident) {
      // recompute the segment (states, stage inputs, norms), then its sweep
      if ((rc = mpc_resident_forward_ex(c, a->ckpts + n * seg, a->segX + n * len,
                                        c->d_Ftab + n0, dt, len, a->segX, a->segY, a->segN,
                                        nullptr, 0, (long long)n)) ||
          (rc = mpc_resident_adjoint(c, c->d_Ftab + n0, dt, len, a->segX, a->segY, a->segN,
                                     a->lam, a->fbar + n0, (long long)n)))
        return rc;
      continue;
    }
    // recompute the segment, keeping states, stage inputs and norms (the
    // forward kept the last one)
    const bool kept = a->last_kept && seg == nseg - 1;
    if (!kept)
      CK(cudaMemcpyAsync(a->segX, a->ckpts + n * seg, sizeof(double2) * n,
                         cudaMemcpyDeviceToDevice, c->stream));
    for (int j = 0; j < len && !kept; ++j) {
      double2* ys[14];
      ys[0] = nullptr;
      for (int s = 1; s < kNumStages; ++s) ys[s] = a->segY + n * ((size_t)j * kNumStages + s);
      ys[13] = a->segY + n * ((size_t)j * kNumStages);  // slot 0 holds x_new (y_0 = x_n)
      if ((rc = fwd_step(c, n0 + j, dt, a->segX + n * j, ys, a->segX + n * (j + 1),
                         a->segN + j)))
        return rc;
    }
    // the recomputed end state must be the next checkpoint (it is, bit for
    // bit, since the kernels are deterministic); walk back through the segment
    for (int j = len - 1; j >= 0; --j) {
      const int stp = n0 + j;
      const double2* x1 = a->segX + n * (j + 1);
      CK(mpc_launch_pdl(k_adj_dot, dim3(nbk), dim3(256), 0, c->stream, (const double2*)x1,
                        (const double2*)a->lam, a->part, ntot));
      CK(mpc_launch_pdl(k_adj_zbar, dim3(nbk), dim3(256), 0, c->stream, (const double2*)a->lam,
                        x1, (const double*)a->part, nbk, (const double*)(a->segN + j), a->zbar,
                        a->v, dt * rkf78::B8[kNumStages - 1], ntot));
      for (int s = kNumStages - 1; s >= 0; --s) {
        if ((rc = mpc_launch_stream(c, a->v))) return rc;
        ac.ys = (s == 0) ? a->segX + n * j : a->segY + n * ((size_t)j * kNumStages + s);
        ac.step = stp;
        ac.stage = s;
        ProfScope ps(c, MPC_KERNEL_COMBINE);
        CK(mpc_launch_pdl(k_adj_combine, dim3(c->combine_grid), dim3(kCombineThreads), 0,
                          c->stream, ac));
      }
      CK(mpc_launch_pdl(k_adj_fbar, dim3(1), dim3(32), 0, c->stream, (const double*)a->fpart,
                        c->combine_grid, a->fbar + stp));
    }
  }
  a->last_kept = false;  // the sweep overwrote the kept segment: a repeat recomputes it
  std::vector<double> fb(steps);
  CK(cudaMemcpyAsync(fb.data(), a->fbar, sizeof(double) * steps, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  unsigned st = 0;
  CK(cudaMemcpy(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream);
    return mpc_fail(MPC_ERR_DEVICE, "kernel status 0x%x during the adjoint pass", st);
  }
  if (dJdF) std::copy(fb.begin(), fb.end(), dJdF);
  if (grad_u && a->K > 0) {
    std::fill(grad_u, grad_u + a->K, 0.0);
    for (int stp = steps - 1; stp >= 0; --stp) {
      int k0;
      double w[4];
      mpc_control_at(a->K, a->u.data(), a->T, a->tn[stp], &k0, w);
      for (int j = 0; j < 4; ++j)
        if (w[j] != 0.0) grad_u[k0 + j] += fb[stp] * w[j];
    }
  }
  return MPC_OK;
}

int mpc_objective_gradient(mpc_ctx* c, const mpc_pulse* p, int K, const double* u, double T,
                           double t0, double dt, int steps, int target, int ckpt_every,
                           const double* ct0, double* J, double* grad_u, double* dJdF) {
  int rc = mpc_objective(c, p, K, u, T, t0, dt, steps, target, ckpt_every, ct0, J);
  if (rc) return rc;
  return mpc_objective_backward(c, grad_u, dJdF);
}

int mpc_adjoint(mpc_ctx* c, const mpc_pulse* p, int K, const double* u, double T, double t0,
                double dt, int steps, int target, int ckpt_every, const double* ct0, double* J,
                double* grad_u, double* dJdF) {
  return mpc_objective_gradient(c, p, K, u, T, t0, dt, steps, target, ckpt_every, ct0, J, grad_u,
                                dJdF);
}

}  // extern "C"
