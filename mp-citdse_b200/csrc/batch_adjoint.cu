// batch_adjoint.cu -- objective and gradient for B pulses at once: the
// fixed-step propagation and its discrete adjoint on the batched stage GEMM
// (the reference has no gradients and one pulse per run; this is new).
//
// Semantics are those of the single-pulse objective (adjoint.cu), per pulse:
// per step n the field F_{n,b} = base_b(t_n + dt) + dE_b(t_n + dt) is frozen
// over the 13 stages, z = x_n + h sum_j b_j k_j (8th-order weights) and
// x_{n+1} = z / ||z|| (tdse::propL / propV, src/tdse/tdse.cpp:186-215); J_b is
// a function of x_N (yield above a threshold, or one population); dJ_b/du_b
// comes from the discrete adjoint with checkpoints every `ckpt` steps and
// each segment recomputed.  All pulses share t0, dt and the step count; each
// has its own pulse, K controls and control window T_b.
//
// Per step the forward is 13 stage GEMMs (MODE 0, one field per step) and a
// norm pair; the adjoint step is a column inner product for zbar, 13 stage
// GEMMs (MODE 1: ybar_s = -M kbar_s, the dJ/dF partials and kbar_{s-1} fused
// into the store) and the dJ/dF reduction.  The couplings are read once per
// stage for all B pulses, so the FP64 tensor pipe, not HBM, bounds the pass.
// Every reduction runs in a fixed order: results repeat bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "batch_stage.cuh"
#include "batch_types.h"
#include "ctx.h"

using namespace mpc;

namespace {

constexpr int kDotRows = 64;  // rows per partial of a column inner product

// [B][n] (user layout) -> [n][ldc]
__global__ void k_fb_load(double2* X, const double2* in, int ntot, int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  X[(long long)i * ldc + q] = in[(long long)q * ntot + i];
}

// per column: ||x_new|| from the stage kernel's row-tile partials, in order
__global__ void k_fb_norm(const double* normpart, int nrt, int ldc, int ncol, double* nrm) {
  pdl_trigger();
  pdl_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ncol) return;
  double s = 0.0;
  for (int r = 0; r < nrt; ++r) s += normpart[(long long)r * ldc + q];
  nrm[q] = sqrt(s);
}

__global__ void k_fb_scale(const double2* XN, const double* nrm, double2* X, int ntot, int ncol,
                           int ldc) {
  pdl_trigger();
  pdl_wait();
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  const long long idx = (long long)i * ldc + q;
  const double2 v = XN[idx];
  X[idx] = make_double2(v.x / nrm[q], v.y / nrm[q]);
}

// lambda_N = dJ/dx_N per column: yield -> 2 x on states at or above thr;
// target -> 2 x_t
__global__ void k_fb_seed(const double2* x, const double* eps, double2* lam, int target,
                          double thr, int ntot, int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  const long long idx = (long long)i * ldc + q;
  const double2 v = x[idx];
  double2 o = make_double2(0.0, 0.0);
  if (target < 0 ? eps[i] >= thr : i == target) o = make_double2(2.0 * v.x, 2.0 * v.y);
  lam[idx] = o;
}

// Re<x, lam> per column: one partial per kDotRows rows (rows in order)
__global__ void k_fb_dot(const double2* x, const double2* lam, double* part, int ntot, int ncol,
                         int ldc) {
  pdl_trigger();
  pdl_wait();
  const int q = blockIdx.y * blockDim.x + threadIdx.x;
  if (q >= ncol) return;
  const int r0 = blockIdx.x * kDotRows, r1 = min(r0 + kDotRows, ntot);
  double s = 0.0;
  for (int i = r0; i < r1; ++i) {
    const long long idx = (long long)i * ldc + q;
    const double2 a = x[idx], b = lam[idx];
    s += fma(a.x, b.x, a.y * b.y);
  }
  part[(long long)blockIdx.x * ldc + q] = s;
}

__global__ void k_fb_colsum(const double* part, int nchunk, int ldc, int ncol, double* out) {
  pdl_trigger();
  pdl_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ncol) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += part[(long long)c * ldc + q];
  out[q] = s;
}

// zbar = (lam - x1 Re<x1, lam>) / ||z_n||; kbar_12 = h b_12 zbar
__global__ void k_fb_zbar(const double2* lam, const double2* x1, const double* dot,
                          const double* nrm, double2* zbar, double2* kb12, double hb12, int ntot,
                          int ncol, int ldc) {
  pdl_trigger();
  pdl_wait();
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  const long long idx = (long long)i * ldc + q;
  const double2 l = lam[idx], x = x1[idx];
  const double r = dot[q], nz = nrm[q];
  const double2 z = make_double2((l.x - x.x * r) / nz, (l.y - x.y * r) / nz);
  zbar[idx] = z;
  kb12[idx] = make_double2(hb12 * z.x, hb12 * z.y);
}

// dJ/dF_n per column: stages, then row tiles, in order
__global__ void k_fb_fbar(const double* fpart, int nrt, int ldc, int ncol, double* fbar) {
  pdl_trigger();
  pdl_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ncol) return;
  double s = 0.0;
  for (int st = 0; st < kNumStages; ++st)
    for (int r = 0; r < nrt; ++r) s += fpart[((long long)st * nrt + r) * ldc + q];
  fbar[q] = s;
}

}  // namespace

struct mpc_badj_state {
  // problem
  int B = 0, ldc = 0, steps = 0, ckpt = 0, nseg = 0, K = 0, target = -1, nrt = 0, nchunk = 0;
  double dt = 0.0;
  std::vector<double> T, u, tn;
  bool have_forward = false;
  // device buffers ([n][ldc] complex unless noted)
  double2* ckpts = nullptr;  // [nseg + 1]
  double2* segX = nullptr;   // [ckpt + 1]
  double2* segY = nullptr;   // [ckpt][12]: stage inputs y_1 .. y_12
  double2* XN = nullptr;
  double2* Ks = nullptr;     // [13]: k_s (forward) or ybar_s (adjoint)
  double2* Zbar = nullptr;
  double2* KB[2] = {nullptr, nullptr};  // kbar ping-pong; KB[1] holds lambda between steps
  double* Ftab = nullptr;    // [steps][ldc]
  double* h = nullptr;       // [ldc]
  double* normpart = nullptr;  // [nrt][ldc]
  double* segN = nullptr;    // [ckpt][ldc]
  double* fpart = nullptr;   // [13][nrt][ldc]
  double* fbar = nullptr;    // [steps][ldc]
  double* dpart = nullptr;   // [nchunk][ldc]
  double* dsum = nullptr;    // [ldc]
  unsigned long long* err = nullptr;  // [ldc] (the forward kernel's error slot, unused)
  double* ws = nullptr;      // split-variant workspace of the stage GEMM
  int* cnt = nullptr;
  // allocation sizes
  size_t cap_slab = 0, cap_ckpt = 0, cap_seg = 0, cap_steps = 0;
  std::vector<void*> allocs;
};

namespace {

void badj_release(mpc_badj_state* a) {
  for (void* p : a->allocs) cudaFree(p);
  a->allocs.clear();
  a->cap_slab = a->cap_ckpt = a->cap_seg = a->cap_steps = 0;
}

template <class T>
int fballoc(mpc_badj_state* a, T** p, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  a->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return MPC_OK;
}

int ensure_badj(mpc_ctx* c, int B, int steps, int ckpt) {
  if (!c->badj) c->badj = new mpc_badj_state();
  mpc_badj_state* a = c->badj;
  const int ldc = (B + 31) / 32 * 32;
  const Geometry& g = c->g;
  int nrt = 0;
  for (int L = 0; L < g.nstate_blk; ++L)
    nrt += (g.state_off[L + 1] - g.state_off[L] + BM - 1) / BM;
  const int nchunk = (g.ntot + kDotRows - 1) / kDotRows;
  const int nseg = (steps + ckpt - 1) / ckpt;
  const size_t slab = (size_t)g.ntot * ldc;
  if (a->cap_slab >= slab && a->ldc == ldc && a->cap_ckpt >= (size_t)nseg + 1 &&
      a->cap_seg >= (size_t)ckpt && a->cap_steps >= (size_t)steps) {
    a->nrt = nrt;
    a->nchunk = nchunk;
    return MPC_OK;
  }
  badj_release(a);
  int rc;
  if ((rc = fballoc(a, &a->ckpts, slab * (nseg + 1))) || (rc = fballoc(a, &a->segX, slab * (ckpt + 1))) ||
      (rc = fballoc(a, &a->segY, slab * 12 * (size_t)ckpt)) || (rc = fballoc(a, &a->XN, slab)) ||
      (rc = fballoc(a, &a->Ks, slab * kNumStages)) || (rc = fballoc(a, &a->Zbar, slab)) ||
      (rc = fballoc(a, &a->KB[0], slab)) || (rc = fballoc(a, &a->KB[1], slab)) ||
      (rc = fballoc(a, &a->Ftab, (size_t)steps * ldc)) || (rc = fballoc(a, &a->h, ldc)) ||
      (rc = fballoc(a, &a->normpart, (size_t)nrt * ldc)) ||
      (rc = fballoc(a, &a->segN, (size_t)ckpt * ldc)) ||
      (rc = fballoc(a, &a->fpart, (size_t)kNumStages * nrt * ldc)) ||
      (rc = fballoc(a, &a->fbar, (size_t)steps * ldc)) ||
      (rc = fballoc(a, &a->dpart, (size_t)nchunk * ldc)) || (rc = fballoc(a, &a->dsum, ldc)) ||
      (rc = fballoc(a, &a->err, ldc)) ||
      (rc = fballoc(a, &a->ws, split_ws_doubles(nrt, ldc))) ||
      (rc = fballoc(a, &a->cnt, split_cnt_ints(nrt, ldc)))) {
    badj_release(a);
    return rc;
  }
  // columns beyond the batch stay zero (finite) in every buffer they are read from
  CK(cudaMemsetAsync(a->ckpts, 0, sizeof(double2) * slab * (nseg + 1), c->stream));
  CK(cudaMemsetAsync(a->segX, 0, sizeof(double2) * slab * (ckpt + 1), c->stream));
  CK(cudaMemsetAsync(a->segY, 0, sizeof(double2) * slab * 12 * (size_t)ckpt, c->stream));
  CK(cudaMemsetAsync(a->XN, 0, sizeof(double2) * slab, c->stream));
  CK(cudaMemsetAsync(a->Ks, 0, sizeof(double2) * slab * kNumStages, c->stream));
  CK(cudaMemsetAsync(a->Zbar, 0, sizeof(double2) * slab, c->stream));
  CK(cudaMemsetAsync(a->KB[0], 0, sizeof(double2) * slab, c->stream));
  CK(cudaMemsetAsync(a->KB[1], 0, sizeof(double2) * slab, c->stream));
  CK(cudaMemsetAsync(a->cnt, 0, sizeof(int) * split_cnt_ints(nrt, ldc), c->stream));
  a->ldc = ldc;
  a->nrt = nrt;
  a->nchunk = nchunk;
  a->cap_slab = slab;
  a->cap_ckpt = nseg + 1;
  a->cap_seg = ckpt;
  a->cap_steps = steps;
  return MPC_OK;
}

StageArgs fb_args(mpc_ctx* c, int stage, int step) {
  mpc_badj_state* a = c->badj;
  StageArgs s{};
  s.D = c->d_D;
  s.eps = c->d_eps;
  s.K = a->Ks;
  s.Fs = a->Ftab + (size_t)step * a->ldc;
  s.fs_stride = 0;  // one field for all 13 stages of the step
  s.h = a->h;
  s.err = a->err;
  s.normpart = a->normpart;
  s.rtol = 1.0;
  s.atol = 1.0;
  s.stage = stage;
  s.gauge = (c->gauge == 'l') ? 0 : 1;
  s.ncol = a->B;
  s.ldc = a->ldc;
  s.nrowtiles = a->nrt;
  s.want_k_only = 0;
  s.fpart = a->fpart;
  s.ws = a->ws;
  s.cnt = a->cnt;
  s.g = c->g;
  return s;
}

template <int MODE>
int fb_launch(mpc_ctx* c, const StageArgs& s) {
  ProfScope ps(c, MPC_KERNEL_BATCH_STAGE);
  ++c->launches;
  CK(launch_variant<MODE>(c->stream, mpc_batch_variant(c, s.ncol), s));
  return MPC_OK;
}

// One forward step from x: stage inputs y_1..y_12 into ys[0..11], x_new into
// XN, x_out = x_new / ||x_new||, the norms into nrm_out [ldc].
int fb_step(mpc_ctx* c, int step, const double2* x, double2* ys, double2* x_out, double* nrm_out) {
  mpc_badj_state* a = c->badj;
  const size_t slab = (size_t)c->g.ntot * a->ldc;
  int rc;
  for (int s = 0; s < kNumStages; ++s) {
    StageArgs st = fb_args(c, s, step);
    st.X = x;
    st.Yin = (s == 0) ? x : ys + slab * (s - 1);
    st.Yout = (s < kNumStages - 1) ? ys + slab * s : a->XN;
    if ((rc = fb_launch<0>(c, st))) return rc;
  }
  const int n = c->g.ntot, B = a->B;
  ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
  CK(mpc_launch_pdl(k_fb_norm, dim3(blocks_for(B, 128)), dim3(128), 0, c->stream,
                    (const double*)a->normpart, a->nrt, a->ldc, B, nrm_out));
  CK(mpc_launch_pdl(k_fb_scale, dim3(blocks_for((long long)n * B, 256)), dim3(256), 0, c->stream,
                    (const double2*)a->XN, (const double*)nrm_out, x_out, n, B, a->ldc));
  c->launches += 2;
  return MPC_OK;
}

int check_device_status(mpc_ctx* c, const char* where) {
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st) {
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
    return mpc_fail(MPC_ERR_DEVICE, "kernel status 0x%x during the %s", st, where);
  }
  return MPC_OK;
}

// Device bytes of the batched objective's buffers for a checkpoint interval.
size_t badj_bytes(const mpc_ctx* c, int B, int steps, int ckpt) {
  const size_t ldc = (B + 31) / 32 * 32, slab = 16 * (size_t)c->g.ntot * ldc;
  int nrt = 0;
  for (int L = 0; L < c->g.nstate_blk; ++L)
    nrt += (c->g.state_off[L + 1] - c->g.state_off[L] + BM - 1) / BM;
  const size_t nseg = (steps + ckpt - 1) / ckpt;
  return slab * (nseg + 1 + (ckpt + 1) + 12 * (size_t)ckpt + 1 + kNumStages + 3) +
         8 * ldc * (2 * (size_t)steps + (size_t)ckpt + (size_t)(kNumStages + 1) * nrt +
                    (size_t)c->g.ntot / kDotRows + 4);
}

// ckpt_every <= 0: the longest interval whose buffers fit in 85 % of the free
// device memory (all steps kept when they fit: no recomputation at all).
int auto_ckpt(mpc_ctx* c, int B, int steps, int* ckpt) {
  if (c->badj) badj_release(c->badj);
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  const double budget = 0.85 * (double)free_b;
  int k = steps;
  while (k > 1 && (double)badj_bytes(c, B, steps, k) > budget) k = (k + 1) / 2;
  if ((double)badj_bytes(c, B, steps, k) > budget)
    return mpc_fail(MPC_ERR_NOMEM, "the batched objective needs %.3g GB, %.3g GB free",
                    badj_bytes(c, B, steps, k) / 1e9, free_b / 1e9);
  *ckpt = k;
  return MPC_OK;
}

}  // namespace

void mpc_badj_invalidate(mpc_ctx* c) {
  if (c && c->badj) c->badj->have_forward = false;
}

void mpc_badj_free(mpc_ctx* c) {
  if (!c || !c->badj) return;
  badj_release(c->badj);
  delete c->badj;
  c->badj = nullptr;
}

extern "C" {

int mpc_batch_objective(mpc_ctx* c, int B, const mpc_pulse* pulses, int K, const double* u,
                        const double* T, double t0, double dt, int steps, int target,
                        int ckpt_every, const double* ct0, double* J) {
  NvtxRange nvtx_("mpc_batch_objective (forward)");
  if (!c || !pulses || !ct0 || !J || B <= 0 || steps <= 0 || !(dt > 0.0) || K == 1 ||
      (K > 0 && (!u || !T)))
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  if (target >= c->g.ntot) return mpc_fail(MPC_ERR_ARG, "target out of range");
  if (dt * c->eps_max > kRk78ImagStability)
    return mpc_fail(MPC_ERR_UNSTABLE, "dt*max|E| = %.4g exceeds the RKF78 stability bound",
                    dt * c->eps_max);
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = stage_setup(c->device))) return rc;
  if (ckpt_every <= 0 && (rc = auto_ckpt(c, B, steps, &ckpt_every))) return rc;
  if ((rc = ensure_badj(c, B, steps, ckpt_every))) return rc;
  mpc_badj_state* a = c->badj;
  a->have_forward = false;
  a->B = B;
  a->steps = steps;
  a->ckpt = ckpt_every;
  a->nseg = (steps + ckpt_every - 1) / ckpt_every;
  a->K = K > 0 ? K : 0;
  a->target = target;
  a->dt = dt;
  a->T.assign(B, 0.0);
  a->u.assign((size_t)B * a->K, 0.0);
  if (a->K) {
    std::copy(T, T + B, a->T.begin());
    std::copy(u, u + (size_t)B * a->K, a->u.begin());
  }
  // field table, t accumulated as the reference's loop does (t += dt)
  const int ldc = a->ldc, n = c->g.ntot;
  std::vector<double> F((size_t)steps * ldc, 0.0);
  a->tn.resize(steps);
  double t = t0;
  for (int st = 0; st < steps; ++st) {
    a->tn[st] = t + dt;
    for (int b = 0; b < B; ++b) {
      int k0;
      double w[4];
      F[(size_t)st * ldc + b] =
          mpc_field(&pulses[b], t + dt) +
          (a->K ? mpc_control_at(a->K, a->u.data() + (size_t)b * a->K, a->T[b], t + dt, &k0, w)
                : 0.0);
    }
    t += dt;
  }
  std::vector<double> hv(ldc, dt);
  CK(cudaMemcpyAsync(a->Ftab, F.data(), sizeof(double) * F.size(), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(a->h, hv.data(), sizeof(double) * ldc, cudaMemcpyHostToDevice, c->stream));
  const size_t slab = (size_t)n * ldc;
  CK(cudaMemcpyAsync(a->XN, ct0, sizeof(double2) * (size_t)n * B, cudaMemcpyHostToDevice,
                     c->stream));
  k_fb_load<<<blocks_for((long long)n * B, 256), 256, 0, c->stream>>>(a->ckpts, a->XN, n, B, ldc);
  CK(cudaGetLastError());
  ++c->launches;
  // forward, a checkpoint every ckpt steps (ping-pong through XN's
  // neighbours otherwise); the last segment is run straight into the segment
  // buffers, so that the backward pass need not recompute it
  const int nlast = (a->nseg - 1) * ckpt_every;
  const double2* x = a->ckpts;
  for (int st = 0; st < nlast; ++st) {
    double2* xn = ((st + 1) % ckpt_every == 0)
                      ? a->ckpts + slab * ((st + 1) / ckpt_every)
                      : a->KB[st & 1];
    if ((rc = fb_step(c, st, x, a->segY, xn, a->segN))) return rc;
    x = xn;
  }
  CK(cudaMemcpyAsync(a->segX, a->ckpts + slab * (a->nseg - 1), sizeof(double2) * slab,
                     cudaMemcpyDeviceToDevice, c->stream));
  for (int st = nlast; st < steps; ++st) {
    const int j = st - nlast;
    if ((rc = fb_step(c, st, a->segX + slab * j, a->segY + slab * 12 * (size_t)j,
                      a->segX + slab * (j + 1), a->segN + (size_t)j * ldc)))
      return rc;
  }
  CK(cudaMemcpyAsync(a->ckpts + slab * a->nseg, a->segX + slab * (steps - nlast),
                     sizeof(double2) * slab, cudaMemcpyDeviceToDevice, c->stream));
  // objective per pulse from x_N
  std::vector<double2> xN(slab);
  std::vector<double> eps(n);
  CK(cudaMemcpyAsync(xN.data(), a->ckpts + slab * a->nseg, sizeof(double2) * slab,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(eps.data(), c->d_eps, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  if ((rc = check_device_status(c, "batched forward pass"))) return rc;
  for (int b = 0; b < B; ++b) {
    double y = 0.0;
    if (target < 0) {
      for (int i = 0; i < n; ++i)
        if (eps[i] >= c->yield_thr) {
          const double2 v = xN[(size_t)i * ldc + b];
          y += v.x * v.x + v.y * v.y;
        }
    } else {
      const double2 v = xN[(size_t)target * ldc + b];
      y = v.x * v.x + v.y * v.y;
    }
    J[b] = y;
  }
  a->have_forward = true;
  return MPC_OK;
}

int mpc_batch_objective_info(mpc_ctx* c, int* ckpt_every, int* segments, double* device_bytes) {
  if (!c || !c->badj || !c->badj->have_forward)
    return mpc_fail(MPC_ERR_ARG, "mpc_batch_objective_info needs a preceding mpc_batch_objective");
  const mpc_badj_state* a = c->badj;
  if (ckpt_every) *ckpt_every = a->ckpt;
  if (segments) *segments = a->nseg;
  if (device_bytes) *device_bytes = (double)badj_bytes(c, a->B, a->steps, a->ckpt);
  return MPC_OK;
}

int mpc_batch_objective_backward(mpc_ctx* c, double* grad_u, double* dJdF) {
  NvtxRange nvtx_("mpc_batch_objective_backward");
  if (!c || !c->badj || !c->badj->have_forward)
    return mpc_fail(MPC_ERR_ARG, "mpc_batch_objective_backward needs a preceding "
                                 "mpc_batch_objective");
  CK(cudaSetDevice(c->device));
  mpc_badj_state* a = c->badj;
  const int B = a->B, ldc = a->ldc, n = c->g.ntot, steps = a->steps, ckpt = a->ckpt;
  const size_t slab = (size_t)n * ldc;
  const int eb = blocks_for((long long)n * B, 256);
  int rc;
  k_fb_seed<<<eb, 256, 0, c->stream>>>(a->ckpts + slab * a->nseg, c->d_eps, a->KB[1], a->target,
                                       c->yield_thr, n, B, ldc);
  CK(cudaGetLastError());
  ++c->launches;
  const double hb12 = a->dt * rkf78::B8[kNumStages - 1];
  for (int seg = a->nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * ckpt;
    const int len = std::min(ckpt, steps - n0);
    // recompute the segment (the last one is still resident from the
    // forward pass): states, stage inputs and norms
    if (seg < a->nseg - 1) {
      CK(cudaMemcpyAsync(a->segX, a->ckpts + slab * seg, sizeof(double2) * slab,
                         cudaMemcpyDeviceToDevice, c->stream));
      for (int j = 0; j < len; ++j)
        if ((rc = fb_step(c, n0 + j, a->segX + slab * j, a->segY + slab * 12 * (size_t)j,
                          a->segX + slab * (j + 1), a->segN + (size_t)j * ldc)))
          return rc;
    }
    // walk back through it
    for (int j = len - 1; j >= 0; --j) {
      const int stp = n0 + j;
      const double2* x1 = a->segX + slab * (j + 1);
      {
        ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
        CK(mpc_launch_pdl(k_fb_dot, dim3(a->nchunk, blocks_for(B, 64)), dim3(64), 0, c->stream,
                          x1, (const double2*)a->KB[1], a->dpart, n, B, ldc));
        CK(mpc_launch_pdl(k_fb_colsum, dim3(blocks_for(B, 128)), dim3(128), 0, c->stream,
                          (const double*)a->dpart, a->nchunk, ldc, B, a->dsum));
        CK(mpc_launch_pdl(k_fb_zbar, dim3(eb), dim3(256), 0, c->stream, (const double2*)a->KB[1],
                          x1, (const double*)a->dsum, (const double*)(a->segN + (size_t)j * ldc),
                          a->Zbar, a->KB[0], hb12, n, B, ldc));
        c->launches += 3;
      }
      for (int s = kNumStages - 1; s >= 0; --s) {
        StageArgs st = fb_args(c, s, stp);
        st.Yin = a->KB[(kNumStages - 1 - s) & 1];
        st.Yout = a->KB[(kNumStages - s) & 1];
        st.Ys = (s == 0) ? a->segX + slab * j : a->segY + slab * (12 * (size_t)j + (s - 1));
        st.Zbar = a->Zbar;
        if ((rc = fb_launch<1>(c, st))) return rc;
      }
      {
        ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
        CK(mpc_launch_pdl(k_fb_fbar, dim3(blocks_for(B, 128)), dim3(128), 0, c->stream,
                          (const double*)a->fpart, a->nrt, ldc, B, a->fbar + (size_t)stp * ldc));
        ++c->launches;
      }
    }
  }
  std::vector<double> fb((size_t)steps * ldc);
  CK(cudaMemcpyAsync(fb.data(), a->fbar, sizeof(double) * fb.size(), cudaMemcpyDeviceToHost,
                     c->stream));
  if ((rc = check_device_status(c, "batched adjoint pass"))) return rc;
  if (dJdF)
    for (int b = 0; b < B; ++b)
      for (int st = 0; st < steps; ++st) dJdF[(size_t)b * steps + st] = fb[(size_t)st * ldc + b];
  if (grad_u && a->K > 0) {
    std::fill(grad_u, grad_u + (size_t)B * a->K, 0.0);
    for (int b = 0; b < B; ++b) {
      double* gb = grad_u + (size_t)b * a->K;
      const double* ub = a->u.data() + (size_t)b * a->K;
      for (int st = steps - 1; st >= 0; --st) {
        int k0;
        double w[4];
        mpc_control_at(a->K, ub, a->T[b], a->tn[st], &k0, w);
        for (int q = 0; q < 4; ++q)
          if (w[q] != 0.0) gb[k0 + q] += fb[(size_t)st * ldc + b] * w[q];
      }
    }
  }
  return MPC_OK;
}

int mpc_batch_objective_gradient(mpc_ctx* c, int B, const mpc_pulse* pulses, int K,
                                 const double* u, const double* T, double t0, double dt,
                                 int steps, int target, int ckpt_every, const double* ct0,
                                 double* J, double* grad_u, double* dJdF) {
  int rc = mpc_batch_objective(c, B, pulses, K, u, T, t0, dt, steps, target, ckpt_every, ct0, J);
  if (rc) return rc;
  return mpc_batch_objective_backward(c, grad_u, dJdF);
}

}  // extern "C"
