// batch.cu -- many pulses in one propagation: batched adaptive RKF78.
//
// The reference propagates one pulse per process (tdse::propV / propL,
// src/tdse/tdse.cpp:146-310) with a fixed step.  Here B pulses -- each with
// its own field, duration, step size and accept/reject history -- advance
// together.  The state of all pulses is one matrix X [n][B] (row = basis
// state, complex column = pulse), so every right-hand side is a real GEMM of
// the block-tridiagonal coupling (the dipole blocks) with the [n x 2B] stage
// matrix, run on the FP64 tensor cores (mma.sync m16n8k8 .f64), with the RK
// stage epilogue fused into the GEMM's store.
//
// Per attempted step (all active pulses at once):
//   13 x k_batch_stage   (GEMM + epilogue: k_s, next stage input; the last
//                         stage also forms x_new, the embedded 7th-order
//                         error and per-pulse norm partials)
//    1 x k_batch_control (per pulse: accept/reject, next step, stage fields)
//    1 x k_batch_apply   (accepted pulses: x = x_new / ||x_new||; retired
//                         pulses write their final state out)
// Retired pulses' columns are compacted away so the GEMM narrows.
// Step control and error norm are those of the CPU oracle's adaptive driver:
//   err = max_i |e_i| / (atol + rtol*max(|x_i|, |x_new_i|)),
//   factor = clamp(0.9 * err^(-1/8), 0.2, 5) with err^(-1/8) as
//   1/sqrt(sqrt(sqrt(err))), stage fields F(t + c_s h) (continuous field).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "batch_stage.cuh"
#include "batch_tma.cuh"
#include "batch_types.h"
#include "ctx.h"
#include "dev_util.cuh"
#include "plan.h"
#include "rkf78.h"

using namespace mpc;

namespace {

struct ControlArgs {
  ColState c;
  PulseResults res;
  double* Fs;                 // [13][ldc]
  unsigned long long* err;
  const double* normpart;
  int nrowtiles;
  int ncol, ldc;
  int mode;                   // 0: start, 1: after an attempt
  double h0, dt_max;
  int max_attempts;
  FixedStep fx;               // fixed-step mode (the reference's semantics)
  unsigned* status;
  // fixed-step mode: the step's unnormalised x_new [n][ldc] (the next step's
  // first product normalises it); a pulse that finishes is written out here
  const double2* XN;
  double2* out;               // [B][n] final states (user layout)
  int ntot;
};

// The next attempt's step: h capped at the time left (the final step lands
// exactly on t_end).
__device__ void prepare_step(const ControlArgs& a, int q) {
  const ColState& c = a.c;
  if (c.done[q]) {
    c.hatt[q] = 0.0;
    return;
  }
  if (a.fx.on) {  // one step of dt; the pulse ends after nsteps of them
    c.hatt[q] = a.fx.dt;
    c.last[q] = (c.nacc[q] + 1 >= c.nsteps[q]) ? 1 : 0;
    return;
  }
  double h = c.h[q];
  const double rem = c.t_end[q] - c.t[q];
  int last = 0;
  if (h >= rem) {
    h = rem;
    last = 1;
  }
  c.hatt[q] = h;
  c.last[q] = last;
}

__device__ void retire(const ControlArgs& a, int q) {
  const ColState& c = a.c;
  const int id = c.pulse_id[q];
  a.res.nacc[id] = c.nacc[q];
  a.res.nrej[id] = c.nrej[q];
  a.res.t[id] = c.t[q];
  a.res.status[id] = (c.done[q] == 2) ? 2 : 0;
  c.retired[q] = 1;
}

// Per pulse: 16 threads.  Thread 0 accepts or rejects the last attempt and
// sets the next step; then threads 0..12 evaluate the 13 stage fields
// F(t + c_s h) in parallel.
constexpr int kCtlLanes = 16;

__global__ void k_batch_control(const __grid_constant__ ControlArgs a) {
  pdl_trigger();
  pdl_wait();
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) / kCtlLanes;
  const int lane = threadIdx.x % kCtlLanes;
  const ColState& c = a.c;
  if (q < a.ncol && lane == 0 && a.fx.on) {
    // fixed-step mode: accept every step whose norm is finite, t += dt as the
    // reference's loop does, retire after nsteps steps.  The state stays
    // unnormalised in XN with its norm in c.nrm (the next step's first
    // product divides); the _pop entry and a finished pulse's final state are
    // formed here, dividing as the reference's c /= ||c|| does.
    c.retired[q] = 0;
    if (a.mode == 0) {
      c.h[q] = a.fx.dt;
      c.done[q] = (c.nsteps[q] <= 0) ? 1 : 0;
      c.accepted[q] = 0;
      c.nrm[q] = 1.0;   // XN holds the normalised start state
      a.err[q] = 0ull;
      if (c.done[q]) retire(a, q);
      prepare_step(a, q);
    } else {
      c.accepted[q] = 0;
      if (!c.done[q]) {
        a.err[q] = 0ull;
        double ns = 0.0;
        for (int r = 0; r < a.nrowtiles; ++r) ns += a.normpart[(long long)r * a.ldc + q];
        const double nrm = sqrt(ns);
        c.natt[q] += 1;
        if (nrm > 0.0 && isfinite(nrm)) {
          c.t[q] = c.t[q] + a.fx.dt;
          c.nacc[q] += 1;
          c.accepted[q] = 1;
          c.nrm[q] = nrm;
          const long long id = c.pulse_id[q];
          if (a.fx.norm_hist) a.fx.norm_hist[id * a.fx.hist_ld + c.nacc[q] - 1] = nrm;
          if (a.fx.pop_hist) {
            const double2 v = a.XN[(long long)a.fx.pop_index * a.ldc + q];
            const double2 o = make_double2(v.x / nrm, v.y / nrm);
            a.fx.pop_hist[id * a.fx.hist_ld + c.nacc[q]] =
                __dadd_rn(__dmul_rn(o.x, o.x), __dmul_rn(o.y, o.y));
          }
          if (c.nacc[q] >= c.nsteps[q]) c.done[q] = 1;
        } else {
          atomicOr(a.status, ST_NONFINITE);
          c.done[q] = 2;
        }
        if (c.done[q]) retire(a, q);
        prepare_step(a, q);
      }
    }
  } else if (q < a.ncol && lane == 0) {
    if (a.mode == 0) {
      c.h[q] = a.h0;
      c.done[q] = (c.t[q] >= c.t_end[q]) ? 1 : 0;
      c.accepted[q] = 0;
      c.retired[q] = 0;
      a.err[q] = 0ull;
      if (c.done[q]) retire(a, q);
      prepare_step(a, q);
    } else {
      c.accepted[q] = 0;
      if (!c.done[q]) {
        const double err = __longlong_as_double((long long)a.err[q]);
        a.err[q] = 0ull;
        double ns = 0.0;
        for (int r = 0; r < a.nrowtiles; ++r) ns += a.normpart[(long long)r * a.ldc + q];
        const double nrm = sqrt(ns);
        const double hh = c.hatt[q];
        const double safety = 0.9, facmin = 0.2, facmax = 5.0;
        double fac;
        if (err == 0.0) {
          fac = facmax;
        } else {
          fac = safety / sqrt(sqrt(sqrt(err)));
          fac = fmin(fmax(fac, facmin), facmax);
        }
        c.natt[q] += 1;
        const bool ok = (err <= 1.0) && (nrm > 0.0) && isfinite(nrm);
        if (ok) {
          c.t[q] = c.last[q] ? c.t_end[q] : c.t[q] + hh;
          c.nacc[q] += 1;
          c.accepted[q] = 1;
          c.nrm[q] = nrm;
          double hn = hh * fac;
          if (hn > a.dt_max) hn = a.dt_max;
          c.h[q] = hn;
          if (c.last[q]) c.done[q] = 1;
        } else {
          c.nrej[q] += 1;
          c.h[q] = hh * fmin(fac, 1.0);
        }
        // give up after max_attempts, or when rejections have shrunk the step
        // to nothing (a non-finite error keeps rejecting)
        if (!c.done[q] && (c.natt[q] >= a.max_attempts ||
                           c.h[q] < 1e-13 * fmax(1.0, fabs(c.t_end[q]))))
          c.done[q] = 2;
        if (c.done[q]) retire(a, q);
        prepare_step(a, q);
      }
    }
  }
  __syncthreads();
  if (a.fx.on && q < a.ncol && c.retired[q]) {
    // fixed-step mode: the finished pulse's final state out, by its lanes
    const double nrm = c.nrm[q];
    const long long id = c.pulse_id[q];
    for (int i = lane; i < a.ntot; i += kCtlLanes) {
      const double2 v = a.XN[(long long)i * a.ldc + q];
      a.out[id * a.ntot + i] = make_double2(v.x / nrm, v.y / nrm);
    }
  }
  if (q < a.ncol && lane < kNumStages) {
    // stage fields F(t + c_s h); in fixed-step mode F(t + dt) for every stage
    const double ts = a.fx.on ? c.t[q] + a.fx.dt : c.t[q] + c_C[lane] * c.hatt[q];
    const double F = c.done[q] ? 0.0 : dev_field(c.pulse[q], ts);
    a.Fs[lane * a.ldc + q] = F;
  }
}

struct ApplyArgs {
  double2* X;
  const double2* Xn;
  ColState c;
  double2* out;     // [B][n] final states (user layout)
  int ntot, ncol, ldc;
  FixedStep fx;     // fixed-step mode: the population history
};

__global__ void k_batch_apply(const __grid_constant__ ApplyArgs a) {
  pdl_trigger();
  pdl_wait();
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long tot = (long long)a.ntot * a.ncol;
  if (e >= tot) return;
  const int i = (int)(e / a.ncol), q = (int)(e % a.ncol);
  const long long idx = (long long)i * a.ldc + q;
  double2 o;
  if (a.c.accepted[q]) {
    const double2 v = a.Xn[idx];
    const double nrm = a.c.nrm[q];
    o = make_double2(v.x / nrm, v.y / nrm);
    a.X[idx] = o;
    if (a.fx.pop_hist && i == a.fx.pop_index)
      a.fx.pop_hist[(long long)a.c.pulse_id[q] * a.fx.hist_ld + a.c.nacc[q]] =
          __dadd_rn(__dmul_rn(o.x, o.x), __dmul_rn(o.y, o.y));
  } else {
    if (!a.c.retired[q]) return;
    o = a.X[idx];
  }
  if (a.c.retired[q]) a.out[(long long)a.c.pulse_id[q] * a.ntot + i] = o;
}

// Clears the retired flags once apply has written the states out.
__global__ void k_batch_clear_retired(int* retired, int ncol) {
  pdl_trigger();
  pdl_wait();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < ncol) retired[q] = 0;
}

// X = XN / nrm per column (fixed-step mode, before the resident tail takes
// the batch over).
__global__ void k_batch_normalize(double2* X, const double2* XN, const double* nrm, int ntot,
                                  int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  const long long idx = (long long)i * ldc + q;
  const double2 v = XN[idx];
  X[idx] = make_double2(v.x / nrm[q], v.y / nrm[q]);
}

// X columns in from the user layout [B][n].
__global__ void k_batch_load(double2* X, const double2* in, int ntot, int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  X[(long long)i * ldc + q] = in[(long long)q * ntot + i];
}

// Compaction: column q of the new layout takes column map[q] of the old.
__global__ void k_batch_gather_cols(double2* dst, const double2* src, const int* map, int ntot,
                                    int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  dst[(long long)i * ldc + q] = src[(long long)i * ldc + map[q]];
}

// K slabs of a single RHS evaluation out to the user layout [B][n].
__global__ void k_batch_store_k0(double2* out, const double2* K, int ntot, int ncol, int ldc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)ntot * ncol) return;
  const int i = (int)(e / ncol), q = (int)(e % ncol);
  out[(long long)q * ntot + i] = K[(long long)i * ldc + q];
}

template <class T>
__global__ void k_gather_scalar(T* dst, const T* src, const int* map, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[map[q]];
}

}  // namespace

struct mpc_batch_state {
  int ldc = 0;        // allocated pulse columns
  int nrowtiles = 0;
  double2* X = nullptr;
  double2* Y[2] = {nullptr, nullptr};
  double2* K = nullptr;
  double2* out = nullptr;   // [ldc][n] user layout
  double* Fs = nullptr;
  unsigned long long* err = nullptr;
  double* normpart = nullptr;
  int* map = nullptr;
  double* ws = nullptr;     // split-variant workspace
  int* cnt = nullptr;       // split-variant arrival counters (kept at zero)
  unsigned* hcnt = nullptr; // persistent Horner launch: ticket + per-column progress
  size_t hcnt_n = 0;
  void* scratch = nullptr;  // compaction staging for per-column scalars
  ColState c{};
  PulseResults res{};
  std::vector<void*> allocs;
  // autotuned stage-GEMM variant per width bucket (bucket j: up to 2^j pulses)
  std::vector<int> tile;
  std::vector<double> tile_us;
  // fixed-step steps, per width bucket: -1 one launch per Horner product
  // (on the right-hand-side tuner's variant), kPlanPerProduct + v one launch
  // per product on variant v, v >= 0 the persistent launch on variant v,
  // kPlanTma + s one TMA-fed launch per product on TMA shape s;
  // microseconds per step of the choice
  std::vector<int> hplan;
  std::vector<double> hplan_us;
  // TMA tensor maps of the TMA-fed Horner products
  std::vector<CUtensorMap> maps;
  CUtensorMap ymaps[kNumTmaShapes][2];
  bool tma_ok = false;
};

namespace {
constexpr int kPlanTma = 100;
constexpr int kPlanPerProduct = 200;
}

namespace {

template <class T>
int balloc(mpc_batch_state* b, T** p, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  b->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return MPC_OK;
}

int ensure_batch(mpc_ctx* c, int B) {
  int rc0;
  if ((rc0 = stage_setup(c->device))) return rc0;
  const int ldc = (B + kColAlign - 1) / kColAlign * kColAlign;
  if (c->batch && c->batch->ldc >= ldc) return MPC_OK;
  mpc_batch_free(c);
  mpc_batch_state* b = new mpc_batch_state();
  c->batch = b;
  b->ldc = ldc;
  const Geometry& g = c->g;
  int nrt = 0;
  for (int L = 0; L < g.nstate_blk; ++L)
    nrt += (g.state_off[L + 1] - g.state_off[L] + BM - 1) / BM;
  b->nrowtiles = nrt;
  b->hcnt_n = 1 + 12 * (size_t)((2 * ldc + 15) / 16) * kMaxBlocks;
  const size_t nel = (size_t)g.ntot * ldc;
  int rc;
  ColState& s = b->c;
  if ((rc = balloc(b, &b->X, nel)) || (rc = balloc(b, &b->Y[0], nel)) ||
      (rc = balloc(b, &b->Y[1], nel)) || (rc = balloc(b, &b->K, nel * kNumStages)) ||
      (rc = balloc(b, &b->out, nel)) || (rc = balloc(b, &b->Fs, (size_t)kNumStages * ldc)) ||
      (rc = balloc(b, &b->err, ldc)) || (rc = balloc(b, &b->normpart, (size_t)nrt * ldc)) ||
      (rc = balloc(b, &b->map, ldc)) ||
      (rc = balloc(b, &b->ws, split_ws_doubles(nrt, ldc))) ||
      (rc = balloc(b, &b->cnt, split_cnt_ints(nrt, ldc))) ||
      (rc = balloc(b, &b->hcnt, 1 + 12 * (size_t)((2 * ldc + 15) / 16) * kMaxBlocks)) ||
      (rc = balloc(b, reinterpret_cast<char**>(&b->scratch), sizeof(mpc_pulse) * ldc)) ||
      (rc = balloc(b, &s.pulse, ldc)) || (rc = balloc(b, &s.t, ldc)) ||
      (rc = balloc(b, &s.t_end, ldc)) || (rc = balloc(b, &s.h, ldc)) ||
      (rc = balloc(b, &s.hatt, ldc)) || (rc = balloc(b, &s.last, ldc)) ||
      (rc = balloc(b, &s.done, ldc)) || (rc = balloc(b, &s.accepted, ldc)) ||
      (rc = balloc(b, &s.nacc, ldc)) || (rc = balloc(b, &s.nrej, ldc)) ||
      (rc = balloc(b, &s.natt, ldc)) || (rc = balloc(b, &s.pulse_id, ldc)) ||
      (rc = balloc(b, &s.nrm, ldc)) || (rc = balloc(b, &s.retired, ldc)) ||
      (rc = balloc(b, &s.nsteps, ldc)) ||
      (rc = balloc(b, &b->res.nacc, ldc)) || (rc = balloc(b, &b->res.nrej, ldc)) ||
      (rc = balloc(b, &b->res.t, ldc)) || (rc = balloc(b, &b->res.status, ldc)))
    return rc;
  // tensor maps of the TMA-fed Horner products: the coupling blocks in both
  // box shapes and the two product buffers (the library's pitches and
  // allocations satisfy TMA's 16-byte rules)
  {
    static bool attrs_set[64] = {};
    if (c->device >= 0 && c->device < 64 && !attrs_set[c->device]) {
      CK(set_tma_attrs());
      attrs_set[c->device] = true;
    }
    const int nblk = g.nblk;
    std::vector<CUtensorMap>& maps = b->maps;
    maps.assign(2 * kTmaMaxBlocks, CUtensorMap{});
    bool ok = nblk >= 1 && nblk <= kTmaMaxBlocks;
    for (int L = 0; ok && L < nblk; ++L) {
      const BlockGeom& bg = g.blk[L];
      const double* base = c->d_D + bg.d_off;
      ok = mpc_encode_map_grouped(&maps[L], base, bg.ncol, bg.nrow, 8ull * bg.pitch, BK,
                                  BM / 16) == MPC_OK &&
           mpc_encode_map_grouped(&maps[kTmaMaxBlocks + L], base, bg.ncol, bg.nrow,
                                  8ull * bg.pitch, BM, BK / 16) == MPC_OK;
    }
    // the product buffers, once per column tile width of the TMA shapes
    for (int sh = 0; ok && sh < kNumTmaShapes; ++sh)
      for (int i = 0; ok && i < 2; ++i)
        ok = mpc_encode_map_grouped(&b->ymaps[sh][i], b->Y[i], 2ull * ldc, g.ntot, 16ull * ldc,
                                    BK, kTmaShapes[sh].bn / 16) == MPC_OK;
    b->tma_ok = ok;
  }
  CK(cudaMemsetAsync(b->X, 0, nel * sizeof(double2), c->stream));
  CK(cudaMemsetAsync(b->cnt, 0, split_cnt_ints(nrt, ldc) * sizeof(int), c->stream));
  CK(cudaMemsetAsync(b->Y[0], 0, nel * sizeof(double2), c->stream));
  CK(cudaMemsetAsync(b->Y[1], 0, nel * sizeof(double2), c->stream));
  CK(cudaMemsetAsync(b->K, 0, nel * kNumStages * sizeof(double2), c->stream));
  return MPC_OK;
}

StageArgs stage_args(mpc_ctx* c, int s, int ncol, double rtol, double atol, bool k_only) {
  mpc_batch_state* b = c->batch;
  StageArgs a{};
  a.D = c->d_D;
  a.eps = c->d_eps;
  a.X = b->X;
  a.Yin = (s == 0) ? b->X : b->Y[s & 1];
  a.K = b->K;
  a.Yout = b->Y[(s + 1) & 1];
  a.Fs = b->Fs;
  a.h = b->c.hatt;
  a.err = b->err;
  a.normpart = b->normpart;
  a.rtol = rtol;
  a.atol = atol;
  a.stage = s;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.ncol = ncol;
  a.ldc = b->ldc;
  a.nrowtiles = b->nrowtiles;
  a.want_k_only = k_only ? 1 : 0;
  a.fs_stride = b->ldc;
  a.ws = b->ws;
  a.cnt = b->cnt;
  a.nrm = b->c.nrm;
  a.Xw = b->X;
  a.g = c->g;
  return a;
}

int launch_stage(mpc_ctx* c, const StageArgs& a) {
  ProfScope ps(c, MPC_KERNEL_BATCH_STAGE);
  ++c->launches;
  CK(launch_variant<0>(c->stream, mpc_batch_variant(c, a.ncol), a));
  return MPC_OK;
}

// How a fixed step of ncol pulses runs: -1 one launch per Horner product,
// else the persistent launch (k_batch_horner) on tile variant v.  The
// fixed-step tuner's choice when it ran; otherwise persistent on the tuned
// variant when a product has enough tiles to fill the GPU.
int horner_plan(mpc_ctx* c, int ncol) {
  if (c->no_persist) return -1;
  const mpc_batch_state* b = c->batch;
  if (c->force_tma > 0 && b->tma_ok) return kPlanTma + std::min(c->force_tma - 1, kNumTmaShapes - 1);
  if (c->force_persist) return mpc_batch_variant(c, ncol);
  if (c->forced_variant >= 0 && c->forced_variant < kNumVariants)
    return kPlanPerProduct + c->forced_variant;
  const int j = width_bucket(ncol);
  if (j < (int)b->hplan.size()) return b->hplan[j];
  const int v = mpc_batch_variant(c, ncol);
  const int bn = horner_tile_bn(v);
  const int ncolt = (2 * ncol + bn - 1) / bn;
  return (long long)ncolt * b->nrowtiles >= c->num_sms ? v : -1;
}


int launch_horner_persistent_v(mpc_ctx* c, int ncol, int v) {
  mpc_batch_state* b = c->batch;
  const int bn = horner_tile_bn(v);
  HornerArgs h{};
  h.a = stage_args(c, 0, ncol, 1.0, 1.0, false);
  h.Y[0] = b->Y[0];
  h.Y[1] = b->Y[1];
  h.ticket = b->hcnt;
  h.done = b->hcnt + 1;
  h.status = c->d_status;
  const BarrierCfg bc = mpc_barrier_cfg(c);
  h.wait_ns = bc.wait_ns;
  h.skew = (unsigned)bc.skew;
  h.ncolt = (2 * ncol + bn - 1) / bn;
  const int items = 12 * h.ncolt * b->nrowtiles;
  CK(cudaMemsetAsync(b->hcnt, 0, sizeof(unsigned) * (1 + 12 * (size_t)h.ncolt * c->g.nstate_blk),
                     c->stream));
  ProfScope ps(c, MPC_KERNEL_BATCH_STAGE);
  ++c->launches;
  CK(launch_horner_variant(c->stream, v, h, c->num_sms, items));
  return MPC_OK;
}


// Product p = 0 .. 11 of a fixed-step (frozen-field) step evaluated as the
// stability polynomial by Horner's rule: v_12 = G[12] x, then
// v_m = h M(F) v_{m+1} + G[m] x for m = 11 .. 0, and v_0 = x_new.  Product p
// forms v_{11-p}; the same ping-pong buffers as the stage form, so x_new
// lands in Y[0].
int launch_horner(mpc_ctx* c, int p, int ncol, int v = -1) {
  StageArgs a = stage_args(c, p, ncol, 1.0, 1.0, false);
  if (p == 0) a.Yin = c->batch->Y[0];   // the previous step's unnormalised x_new
  a.hg = rkf78::G[11 - p];
  a.vscale = (p == 0) ? rkf78::G[12] : 1.0;
  a.hlast = (p == 11) ? 1 : 0;
  ProfScope ps(c, MPC_KERNEL_BATCH_STAGE);
  ++c->launches;
  CK(launch_variant<2>(c->stream, v >= 0 ? v : mpc_batch_variant(c, a.ncol), a));
  return MPC_OK;
}

// Product p of a fixed step as the TMA-fed launch on TMA tile shape `shape`.
int launch_horner_tma(mpc_ctx* c, int p, int ncol, int shape) {
  mpc_batch_state* b = c->batch;
  HornerTmaArgs h{};
  h.a = stage_args(c, p, ncol, 1.0, 1.0, false);
  for (size_t i = 0; i < b->maps.size(); ++i) h.maps[i] = b->maps[i];
  h.maps[2 * kTmaMaxBlocks] = b->ymaps[shape][0];
  h.maps[2 * kTmaMaxBlocks + 1] = b->ymaps[shape][1];
  h.Y[0] = b->Y[0];
  h.Y[1] = b->Y[1];
  h.status = c->d_status;
  h.wait_ns = c->wait_limit_ns;
  const int bn = kTmaShapes[shape].bn;
  h.ncolt = (2 * ncol + bn - 1) / bn;
  h.p = p;
  ProfScope ps(c, MPC_KERNEL_BATCH_STAGE);
  ++c->launches;
  CK(launch_horner_tma_shape(c->stream, shape, h, c->num_sms));
  return MPC_OK;
}

// The 12 products of one fixed step of ncol pulses, run as plan says.
int launch_horner_plan(mpc_ctx* c, int ncol, int plan) {
  int rc;
  if (plan >= kPlanPerProduct) {
    for (int p = 0; p < 12; ++p)
      if ((rc = launch_horner(c, p, ncol, plan - kPlanPerProduct))) return rc;
    return MPC_OK;
  }
  if (plan >= kPlanTma) {
    for (int p = 0; p < 12; ++p)
      if ((rc = launch_horner_tma(c, p, ncol, plan - kPlanTma))) return rc;
    return MPC_OK;
  }
  if (plan >= 0) return launch_horner_persistent_v(c, ncol, plan);
  for (int p = 0; p < 12; ++p)
    if ((rc = launch_horner(c, p, ncol))) return rc;
  return MPC_OK;
}

int launch_horner_step(mpc_ctx* c, int ncol) {
  return launch_horner_plan(c, ncol, horner_plan(c, ncol));
}

// Kernel launches of one fixed step (its products and the controller).
long long horner_step_launches(mpc_ctx* c, int ncol) {
  const int plan = horner_plan(c, ncol);
  return (plan >= 0 && plan < kPlanTma) ? 2 : 13;
}

// Times every variant on a single right-hand side (stage 0, k only) at
// widths 1, 2, 4, ... up to max_cols pulses and keeps the fastest per width.
// Every variant sums in the same order, so the choice affects speed only.
int autotune(mpc_ctx* c, int max_cols) {
  mpc_batch_state* b = c->batch;
  const int top = width_bucket(std::min(std::max(max_cols, 1), b->ldc));
  std::vector<int> tile(top + 1);
  std::vector<double> us((size_t)(top + 1) * kNumVariants);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = MPC_OK;
  for (int j = 0; j <= top && rc == MPC_OK; ++j) {
    const int w = std::min(1 << j, b->ldc);
    const StageArgs a = stage_args(c, 0, w, 0.0, 0.0, true);
    double best = 1e300;
    for (int v = 0; v < kNumVariants && rc == MPC_OK; ++v) {
      cudaError_t e = cudaSuccess;
      for (int r = 0; r < 2 && e == cudaSuccess; ++r) e = launch_variant<0>(c->stream, v, a);
      if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
      const int reps = 5;
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = launch_variant<0>(c->stream, v, a);
      if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        rc = mpc_fail(MPC_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
        break;
      }
      c->launches += 2 + reps;
      const double t = 1000.0 * ms / reps;
      us[(size_t)j * kNumVariants + v] = t;
      if (t < best) {
        best = t;
        tile[j] = v;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->tile = tile;
  b->tile_us = us;
  return MPC_OK;
}

// The fixed-step tuner: at widths 1, 2, 4, ... up to max_cols pulses, times
// one whole step's 12 Horner products as one launch per product (on the
// tuned variant) and as the persistent launch on each unsplit tile shape,
// and keeps the fastest.  Every candidate computes the same tiles in the same
// order, so the choice changes speed only.  Runs on the batch's work
// buffers before the propagation loads its states.
int autotune_horner(mpc_ctx* c, int max_cols) {
  mpc_batch_state* b = c->batch;
  const int top = width_bucket(std::min(std::max(max_cols, 1), b->ldc));
  std::vector<int> plan(top + 1, -1);
  std::vector<double> plan_us(top + 1, 0.0);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // one launch per product on every tile variant (the right-hand-side
  // tuner's choice need not suit the Horner epilogue), the persistent launch
  // on every unsplit variant, the TMA-fed launches
  std::vector<int> cands = {0, 1, 2, 3, 4};
  for (int v = 0; v < kNumVariants; ++v) cands.push_back(kPlanPerProduct + v);
  if (b->tma_ok && !c->no_tma)
    for (int sh = 0; sh < kNumTmaShapes; ++sh) cands.push_back(kPlanTma + sh);
  int rc = MPC_OK;
  const long long l0 = c->launches;
  for (int j = 0; j <= top && rc == MPC_OK; ++j) {
    const int w = std::min(1 << j, b->ldc);
    double best = 1e300;
    for (int v : cands) {
      auto step = [&]() -> int { return launch_horner_plan(c, w, v); };
      for (int r = 0; r < 2 && rc == MPC_OK; ++r) rc = step();
      if (rc) break;
      CK(cudaEventRecord(e0, c->stream));
      const int reps = 3;
      for (int r = 0; r < reps && rc == MPC_OK; ++r) rc = step();
      if (rc) break;
      CK(cudaEventRecord(e1, c->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      const double t = 1000.0 * ms / reps;
      if (t < best) {
        best = t;
        plan[j] = v;
        plan_us[j] = t;
      }
    }
  }
  c->launches = l0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->hplan = plan;
  b->hplan_us = plan_us;
  return MPC_OK;
}

}  // namespace

int mpc_batch_variant(mpc_ctx* c, int ncol) {
  if (c->forced_variant >= 0 && c->forced_variant < kNumVariants) return c->forced_variant;
  if (c->batch) {
    const std::vector<int>& t = c->batch->tile;
    const int j = width_bucket(ncol);
    if (j < (int)t.size()) return t[j];
  }
  return default_variant(ncol);
}

void mpc_batch_free(mpc_ctx* c) {
  if (!c || !c->batch) return;
  for (void* p : c->batch->allocs) cudaFree(p);
  delete c->batch;
  c->batch = nullptr;
}

extern "C" {

int mpc_batch_rhs(mpc_ctx* c, int B, const double* F, const double* x, double* dxdt) {
  if (!c || !F || !x || !dxdt || B <= 0) return mpc_fail(MPC_ERR_ARG, "bad argument");
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = ensure_batch(c, B))) return rc;
  mpc_batch_state* b = c->batch;
  const int n = c->g.ntot;
  CK(cudaMemcpyAsync(b->out, x, sizeof(double2) * (size_t)n * B, cudaMemcpyHostToDevice,
                     c->stream));
  k_batch_load<<<blocks_for((long long)n * B, 256), 256, 0, c->stream>>>(b->X, b->out, n, B, b->ldc);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(b->Fs, F, sizeof(double) * B, cudaMemcpyHostToDevice, c->stream));
  if ((rc = launch_stage(c, stage_args(c, 0, B, 0.0, 0.0, true)))) return rc;
  k_batch_store_k0<<<blocks_for((long long)n * B, 256), 256, 0, c->stream>>>(b->out, b->K, n, B,
                                                                            b->ldc);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dxdt, b->out, sizeof(double2) * (size_t)n * B, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MPC_OK;
}

int mpc_propagate_adaptive(mpc_ctx* c, const mpc_pulse* pulse, double t0, double t_end,
                           double h0, double dt_max, double rtol, double atol, int max_attempts,
                           double* ct, int* accepted, int* rejected, double* t_final) {
  if (!pulse || !ct) return mpc_fail(MPC_ERR_ARG, "bad argument");
  return mpc_batch_propagate(c, 1, pulse, &t0, &t_end, h0, dt_max, rtol, atol, max_attempts, ct,
                             accepted, rejected, t_final);
}

int mpc_propagate_batch(mpc_ctx* c, int B, const mpc_pulse* pulses, const double* t0,
                        const double* t_end, double h0, double dt_max, double rtol, double atol,
                        int max_attempts, double* ct, int* accepted, int* rejected,
                        double* t_final) {
  return mpc_batch_propagate(c, B, pulses, t0, t_end, h0, dt_max, rtol, atol, max_attempts, ct,
                             accepted, rejected, t_final);
}

int mpc_batch_fixed_plan(mpc_ctx* c, double* table, int cap) {
  if (!c || (table && cap < 0)) return mpc_fail(MPC_ERR_ARG, "bad argument");
  if (!c->batch || c->batch->hplan.empty()) return 0;
  const mpc_batch_state* b = c->batch;
  const int rows = (int)b->hplan.size();
  for (int j = 0; table && j < rows && j < cap; ++j) {
    const int v = b->hplan[j];
    table[5 * j + 0] = std::min(1 << j, b->ldc);
    if (v >= kPlanPerProduct) {
      const TileVariant& tv = kVariants[v - kPlanPerProduct];
      table[5 * j + 1] = tv.split ? 3 : 0;
      table[5 * j + 2] = tv.bn;
      table[5 * j + 3] = tv.nst;
    } else if (v >= kPlanTma) {
      table[5 * j + 1] = 2;
      table[5 * j + 2] = kTmaShapes[v - kPlanTma].bn;
      table[5 * j + 3] = kTmaShapes[v - kPlanTma].ns;
    } else {
      const int vv = v >= 0 ? v : mpc_batch_variant(c, std::min(1 << j, b->ldc));
      table[5 * j + 1] = v >= 0 ? 1 : 0;
      table[5 * j + 2] = kVariants[vv].bn;
      table[5 * j + 3] = v >= 0 ? (kVariants[vv].nst >= 6 ? 3 : 2) : kVariants[vv].nst;
    }
    table[5 * j + 4] = b->hplan_us[j];
  }
  return rows;
}

int mpc_batch_autotune(mpc_ctx* c, int B, double* table, int cap) {
  if (!c || B <= 0 || (table && cap < 0)) return mpc_fail(MPC_ERR_ARG, "bad argument");
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = ensure_batch(c, B))) return rc;
  if ((rc = autotune(c, B))) return rc;
  const mpc_batch_state* b = c->batch;
  const int rows = (int)b->tile.size();
  for (int j = 0; table && j < rows && j < cap; ++j) {
    const int v = b->tile[j];
    table[5 * j + 0] = std::min(1 << j, b->ldc);
    table[5 * j + 1] = kVariants[v].bn;
    table[5 * j + 2] = kVariants[v].nst;
    table[5 * j + 3] = kVariants[v].split;
    table[5 * j + 4] = b->tile_us[(size_t)j * kNumVariants + v];
  }
  return rows;
}

}  // extern "C"

namespace {

// The batched driver shared by the adaptive entry point and the fixed-step
// one (fx->on: the reference's semantics; nsteps[B] the per-pulse step
// counts, t_end unused).
int batch_run(mpc_ctx* c, int B, const mpc_pulse* pulses, const double* t0, const double* t_end,
              double h0, double dt_max, double rtol, double atol, int max_attempts, double* ct,
              int* accepted, int* rejected, double* t_final, FixedStep fx, const int* nsteps) {
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = ensure_batch(c, B))) return rc;
  mpc_batch_state* b = c->batch;
  ColState& s = b->c;
  const int n = c->g.ntot;
  const int ldc = b->ldc;

  if (fx.on && c->force_tma > 0 && !b->tma_ok)
    return mpc_fail(MPC_ERR_CUDA, "MPC_FORCE_TMA: the TMA tensor maps could not be set up");
  // the fixed-step tuner times Horner steps on the work buffers (the first
  // product writes X): it runs before the states are loaded, on unit norms
  if (b->tile.empty() && !std::getenv("MPC_NO_AUTOTUNE") && (rc = autotune(c, B))) return rc;
  if (fx.on && b->hplan.empty() && !c->no_persist && !c->force_persist && !c->force_tma &&
      !std::getenv("MPC_NO_AUTOTUNE")) {
    std::vector<double> ones(ldc, 1.0);
    CK(cudaMemcpyAsync(s.nrm, ones.data(), sizeof(double) * ldc, cudaMemcpyHostToDevice,
                       c->stream));
    if ((rc = autotune_horner(c, B))) return rc;
  }

  // per-column start state
  std::vector<int> ids(B);
  for (int i = 0; i < B; ++i) ids[i] = i;
  std::vector<int> zeros(B, 0);
  CK(cudaMemcpyAsync(s.pulse, pulses, sizeof(mpc_pulse) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.t, t0, sizeof(double) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.t_end, t_end, sizeof(double) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.pulse_id, ids.data(), sizeof(int) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.nacc, zeros.data(), sizeof(int) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.nrej, zeros.data(), sizeof(int) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.natt, zeros.data(), sizeof(int) * B, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s.nsteps, fx.on ? nsteps : zeros.data(), sizeof(int) * B,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(b->out, ct, sizeof(double2) * (size_t)n * B, cudaMemcpyHostToDevice,
                     c->stream));
  k_batch_load<<<blocks_for((long long)n * B, 256), 256, 0, c->stream>>>(b->X, b->out, n, B, ldc);
  CK(cudaGetLastError());
  // fixed-step mode: the state lives unnormalised in Y[0] (norm 1 at start)
  if (fx.on)
    CK(cudaMemcpyAsync(b->Y[0], b->X, sizeof(double2) * (size_t)n * ldc, cudaMemcpyDeviceToDevice,
                       c->stream));

  ControlArgs ca{};
  ca.c = s;
  ca.res = b->res;
  ca.Fs = b->Fs;
  ca.err = b->err;
  ca.normpart = b->normpart;
  ca.nrowtiles = b->nrowtiles;
  ca.ldc = ldc;
  ca.h0 = h0;
  ca.dt_max = dt_max;
  ca.max_attempts = max_attempts > 0 ? max_attempts : 1000000000;
  ca.fx = fx;
  ca.status = c->d_status;
  ca.XN = b->Y[0];
  ca.out = b->out;
  ca.ntot = n;
  ApplyArgs aa{};
  aa.X = b->X;
  aa.Xn = b->Y[1];
  aa.c = s;
  aa.out = b->out;
  aa.ntot = n;
  aa.ldc = ldc;
  aa.fx = fx;
  if (fx.on) aa.Xn = b->Y[0];  // the Horner products leave x_new in Y[0]

  int ncol = B;
  ca.ncol = ncol;
  ca.mode = 0;
  k_batch_control<<<blocks_for((long long)ncol * kCtlLanes, 128), 128, 0, c->stream>>>(ca);
  CK(cudaGetLastError());
  ca.mode = 1;
  // pulses with nothing to do are retired by the start: write their states
  // out (the control kernel itself does in fixed-step mode)
  if (!fx.on) {
    aa.ncol = ncol;
    k_batch_apply<<<blocks_for((long long)n * ncol, 256), 256, 0, c->stream>>>(aa);
    k_batch_clear_retired<<<blocks_for(ncol, 128), 128, 0, c->stream>>>(s.retired, ncol);
    CK(cudaGetLastError());
    c->launches += 2;
  }
  c->launches += 1;

  // Few pulses left on a system whose coupling fits on chip: the persistent
  // resident kernel takes over (unless the streamed path was asked for).
  const int pres = (c->path == MPC_PATH_STREAMING) ? 0 : mpc_batch_res_pmax(c);

  std::vector<int> done_h(B), map_h(B);
  // fixed-step mode: every active pulse takes one step per attempt, so the
  // host knows when the next one finishes -- the attempts up to then run
  // without reading the done flags in between
  std::vector<int> colpid(B), steps_h(nsteps ? nsteps : zeros.data(),
                                      (nsteps ? nsteps : zeros.data()) + B);
  for (int q = 0; q < B; ++q) colpid[q] = q;
  long long steps_done = 0;
  auto width = [](int nc) {
    return 2 * nc <= 16 ? 16 : (2 * nc <= 128 ? (2 * nc + 31) / 32 * 32 : (2 * nc + 63) / 64 * 64);
  };
  // active columns -> map_h[0 .. act)
  auto scan = [&](int* act) -> int {
    CK(cudaMemcpyAsync(done_h.data(), s.done, sizeof(int) * ncol, cudaMemcpyDeviceToHost,
                       c->stream));
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (st) {
      CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
      return mpc_fail(MPC_ERR_DEVICE, "kernel status 0x%x in the batched propagation", st);
    }
    int k = 0;
    for (int q = 0; q < ncol; ++q)
      if (!done_h[q]) map_h[k++] = q;
    *act = k;
    return MPC_OK;
  };
  // Compaction: the active columns move to the front of X and of every
  // per-column array (the results of retired pulses are already out).
  // (in fixed-step mode the GEMM path keeps the state unnormalised in Y[0];
  // the resident tail keeps it normalised in X)
  bool state_in_y0 = fx.on;
  auto compact = [&](int act) -> int {
    CK(cudaMemcpyAsync(b->map, map_h.data(), sizeof(int) * act, cudaMemcpyHostToDevice,
                       c->stream));
    const int gb = blocks_for((long long)n * act, 256);
    if (state_in_y0) {  // the state is the unnormalised Y[0]; Y[1] is free between steps
      k_batch_gather_cols<<<gb, 256, 0, c->stream>>>(b->Y[1], b->Y[0], b->map, n, act, ldc);
      CK(cudaMemcpyAsync(b->Y[0], b->Y[1], sizeof(double2) * (size_t)n * ldc,
                         cudaMemcpyDeviceToDevice, c->stream));
    } else {
      k_batch_gather_cols<<<gb, 256, 0, c->stream>>>(b->Y[0], b->X, b->map, n, act, ldc);
      CK(cudaMemcpyAsync(b->X, b->Y[0], sizeof(double2) * (size_t)n * ldc,
                         cudaMemcpyDeviceToDevice, c->stream));
    }
    const int sb = blocks_for(act, 128);
#define GATHER(field, T)                                                                    \
  k_gather_scalar<T><<<sb, 128, 0, c->stream>>>(reinterpret_cast<T*>(b->scratch), s.field,  \
                                               b->map, act);                               \
  CK(cudaMemcpyAsync(s.field, b->scratch, sizeof(T) * act, cudaMemcpyDeviceToDevice, c->stream));
    GATHER(pulse, mpc_pulse)
    GATHER(t, double)
    GATHER(t_end, double)
    GATHER(h, double)
    GATHER(hatt, double)
    GATHER(last, int)
    GATHER(done, int)
    GATHER(accepted, int)
    GATHER(nacc, int)
    GATHER(nrej, int)
    GATHER(natt, int)
    GATHER(pulse_id, int)
    GATHER(nrm, double)
    GATHER(retired, int)
    GATHER(nsteps, int)
    {
      std::vector<int> cp(act);
      for (int k = 0; k < act; ++k) cp[k] = colpid[map_h[k]];
      std::copy(cp.begin(), cp.end(), colpid.begin());
    }
    for (int st = 0; st < kNumStages; ++st) {
      k_gather_scalar<double><<<sb, 128, 0, c->stream>>>(reinterpret_cast<double*>(b->scratch),
                                                         b->Fs + st * ldc, b->map, act);
      CK(cudaMemcpyAsync(b->Fs + st * ldc, b->scratch, sizeof(double) * act,
                         cudaMemcpyDeviceToDevice, c->stream));
    }
#undef GATHER
    CK(cudaGetLastError());
    c->launches += 16;
    ncol = act;
    return MPC_OK;
  };

  // One attempted step of every active pulse: 13 stage GEMMs, the step
  // controller, the accepted-state update and the retirement flags.
  auto launch_attempt = [&]() -> int {
    if (fx.on) {  // frozen field: the 12 products of the stability polynomial
      if ((rc = launch_horner_step(c, ncol))) return rc;
    } else {
      for (int st = 0; st < kNumStages; ++st)
        if ((rc = launch_stage(c, stage_args(c, st, ncol, rtol, atol, false)))) return rc;
    }
    ca.ncol = ncol;
    aa.ncol = ncol;
    {
      ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
      CK(mpc_launch_pdl(k_batch_control, dim3(blocks_for((long long)ncol * kCtlLanes, 128)),
                        dim3(128), 0, c->stream, ca));
    }
    c->launches += 1;
    if (fx.on) return MPC_OK;  // renormalisation in the next step's first product
    {
      ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
      CK(mpc_launch_pdl(k_batch_apply, dim3(blocks_for((long long)n * ncol, 256)), dim3(256), 0,
                        c->stream, aa));
    }
    {
      ProfScope ps(c, MPC_KERNEL_BATCH_OTHER);
      CK(mpc_launch_pdl(k_batch_clear_retired, dim3(blocks_for(ncol, 128)), dim3(128), 0,
                        c->stream, s.retired, ncol));
    }
    c->launches += 2;
    return MPC_OK;
  };
  // Attempts run in groups of check_every between reads of the done flags;
  // a group is captured once per active width as a CUDA graph and replayed
  // (not while profiling, whose per-launch events stay outside graphs).
  const int check_every = 8;
  bool use_graph = !c->profiling && !std::getenv("MPC_NO_GRAPH");
  cudaGraphExec_t gexec = nullptr;
  int g_ncol = -1;
  auto drop_graph = [&]() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    g_ncol = -1;
  };
  auto run_group = [&]() -> int {
    if (use_graph && g_ncol != ncol) {
      drop_graph();
      cudaGraph_t graph = nullptr;
      bool ok = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      const long long l0 = c->launches;
      int lrc = MPC_OK;
      for (int k = 0; ok && k < check_every && lrc == MPC_OK; ++k) lrc = launch_attempt();
      if (ok) ok = cudaStreamEndCapture(c->stream, &graph) == cudaSuccess && lrc == MPC_OK;
      if (ok) ok = cudaGraphInstantiate(&gexec, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      c->launches = l0;
      if (!ok) {  // capture unavailable: plain launches from here on
        cudaGetLastError();
        gexec = nullptr;
        use_graph = false;
      } else {
        g_ncol = ncol;
      }
    }
    if (use_graph) {
      CK(cudaGraphLaunch(gexec, c->stream));
      c->launches += (fx.on ? horner_step_launches(c, ncol) : 16LL) * check_every;
      return MPC_OK;
    }
    for (int k = 0; k < check_every; ++k)
      if ((rc = launch_attempt())) return rc;
    return MPC_OK;
  };

  for (;;) {
    int act = 0;
    if ((rc = scan(&act))) break;
    if (act == 0) break;
    if (pres && act <= pres) {
      if (act < ncol && (rc = compact(act))) break;
      if (fx.on) {  // the resident kernel takes normalised states in X
        k_batch_normalize<<<blocks_for((long long)n * ncol, 256), 256, 0, c->stream>>>(
            b->X, b->Y[0], s.nrm, n, ncol, ldc);
        CK(cudaGetLastError());
        ++c->launches;
        state_in_y0 = false;
      }
      BatchResLaunch l{};
      l.c = s;
      l.res = b->res;
      l.X = b->X;
      l.XN = b->K;  // k slab 0 (unused by the resident kernel)
      l.Y0 = b->Y[0];
      l.Y1 = b->Y[1];
      l.out = b->out;
      l.ldc = ldc;
      l.max_attempts = ca.max_attempts;
      l.rtol = rtol;
      l.atol = atol;
      l.dt_max = dt_max;
      l.fx = fx;
      while (true) {
        int P = 1;
        while (P < ncol) P *= 2;
        l.ncol = ncol;
        if ((rc = mpc_batch_res_run(c, l, P, P > 1 ? P / 2 + 1 : 0))) break;
        if ((rc = scan(&act))) break;
        if (act == 0) break;
        if (act < ncol && (rc = compact(act))) break;
      }
      break;
    }
    // compact when the GEMM can drop a column tile or use a narrower one
    if (width(act) < width(ncol) && (rc = compact(act))) break;
    if (fx.on) {
      // run up to the next pulse's last step: whole graph groups, then single
      // attempts, then look at the done flags again
      long long until = -1;   // a finished pulse has no steps left
      for (int q = 0; q < ncol; ++q) {
        const long long left = (long long)steps_h[colpid[q]] - steps_done;
        if (left > 0 && (until < 0 || left < until)) until = left;
      }
      if (until <= 0) until = 1;
      for (long long k = 0; k + check_every <= until && rc == MPC_OK; k += check_every)
        rc = run_group();
      for (long long k = until - until % check_every; k < until && rc == MPC_OK; ++k)
        rc = launch_attempt();
      if (rc) break;
      steps_done += until;
      continue;
    }
    if ((rc = run_group())) break;
  }
  drop_graph();
  if (rc) return rc;
  // per-pulse results (indexed by pulse id) and final states
  std::vector<int> na(B), nr(B), stt(B);
  std::vector<double> tf(B);
  CK(cudaMemcpyAsync(na.data(), b->res.nacc, sizeof(int) * B, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(nr.data(), b->res.nrej, sizeof(int) * B, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(tf.data(), b->res.t, sizeof(double) * B, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(stt.data(), b->res.status, sizeof(int) * B, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaMemcpyAsync(ct, b->out, sizeof(double2) * (size_t)n * B, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int gave_up = 0;
  for (int i = 0; i < B; ++i) {
    if (accepted) accepted[i] = na[i];
    if (rejected) rejected[i] = nr[i];
    if (t_final) t_final[i] = tf[i];
    gave_up += stt[i] == 2;
  }
  if (gave_up)
    return mpc_fail(MPC_ERR_DEVICE,
                    fx.on ? "%d pulse(s) stopped on a non-finite norm"
                          : "%d pulse(s) stopped after max_attempts step attempts",
                    gave_up);
  return MPC_OK;
}

}  // namespace

extern "C" {

int mpc_batch_propagate(mpc_ctx* c, int B, const mpc_pulse* pulses, const double* t0,
                        const double* t_end, double h0, double dt_max, double rtol, double atol,
                        int max_attempts, double* ct, int* accepted, int* rejected,
                        double* t_final) {
  NvtxRange nvtx_("mpc_batch_propagate");
  if (!c || !pulses || !t0 || !t_end || !ct || B <= 0)
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  if (!(h0 > 0.0) || !(dt_max > 0.0) || !(rtol >= 0.0) || !(atol >= 0.0) || rtol + atol <= 0.0)
    return mpc_fail(MPC_ERR_ARG, "bad step-control parameters");
  if (h0 * c->eps_max > kRk78ImagStability * 4.0 || dt_max * c->eps_max > kRk78ImagStability)
    return mpc_fail(MPC_ERR_UNSTABLE,
                    "dt_max*max|E| = %.4g exceeds the RKF78 imaginary-axis stability bound %.4g",
                    dt_max * c->eps_max, kRk78ImagStability);
  FixedStep fx{};
  return batch_run(c, B, pulses, t0, t_end, h0, dt_max, rtol, atol, max_attempts, ct, accepted,
                   rejected, t_final, fx, nullptr);
}

int mpc_batch_advance(mpc_ctx* c, int B, const mpc_pulse* pulses, const double* t0, double dt,
                      const int* steps, int pop_index, double* ct, double* pop_out,
                      double* norm_out) {
  NvtxRange nvtx_("mpc_batch_advance");
  if (!c || !pulses || !t0 || !steps || !ct || B <= 0)
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  if (!(dt > 0.0)) return mpc_fail(MPC_ERR_ARG, "dt must be > 0");
  if (pop_index < 0 || pop_index >= c->g.ntot) return mpc_fail(MPC_ERR_ARG, "pop_index out of range");
  int max_steps = 0;
  for (int b = 0; b < B; ++b) {
    if (steps[b] < 0) return mpc_fail(MPC_ERR_ARG, "steps[%d] < 0", b);
    max_steps = std::max(max_steps, steps[b]);
  }
  if (dt * c->eps_max > kRk78ImagStability)
    return mpc_fail(MPC_ERR_UNSTABLE,
                    "dt*max|E| = %.4g exceeds the RKF78 imaginary-axis stability bound %.4g",
                    dt * c->eps_max, kRk78ImagStability);
  CK(cudaSetDevice(c->device));
  FixedStep fx{};
  fx.on = 1;
  fx.dt = dt;
  fx.pop_index = pop_index;
  fx.hist_ld = (long long)max_steps + 1;
  double* dpop = nullptr;
  double* dnrm = nullptr;
  auto release = [&]() {
    if (dpop) cudaFree(dpop);
    if (dnrm) cudaFree(dnrm);
  };
  if (pop_out && cudaMalloc(&dpop, sizeof(double) * (size_t)B * fx.hist_ld) != cudaSuccess) {
    cudaGetLastError();
    return mpc_fail(MPC_ERR_NOMEM, "population history of %d x %lld", B, fx.hist_ld);
  }
  if (norm_out && cudaMalloc(&dnrm, sizeof(double) * (size_t)B * fx.hist_ld) != cudaSuccess) {
    cudaGetLastError();
    release();
    return mpc_fail(MPC_ERR_NOMEM, "norm history of %d x %lld", B, fx.hist_ld);
  }
  fx.pop_hist = dpop;
  fx.norm_hist = dnrm;
  std::vector<double> t_end(B), pop0(B);
  for (int b = 0; b < B; ++b) {
    t_end[b] = t0[b] + steps[b] * dt;
    // entry 0 of the history: the start state, as the reference writes it
    // before its loop
    const double* x = ct + 2 * (size_t)b * c->g.ntot + 2 * (size_t)pop_index;
    pop0[b] = x[0] * x[0] + x[1] * x[1];
  }
  // the error-norm tolerances are unused in fixed-step mode (every finite
  // step is accepted); 1 keeps the stage epilogue's ratio finite
  int rc = batch_run(c, B, pulses, t0, t_end.data(), dt, dt, 1.0, 1.0, 0, ct, nullptr, nullptr,
                     nullptr, fx, steps);
  if (rc == MPC_OK && (dpop || dnrm)) {
    std::vector<double> h((size_t)B * fx.hist_ld);
    const size_t ld = (size_t)fx.hist_ld;
    if (dpop) {
      if (cudaMemcpy(h.data(), dpop, sizeof(double) * h.size(), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
        rc = mpc_fail(MPC_ERR_CUDA, "history copy failed");
      for (int b = 0; rc == MPC_OK && b < B; ++b) {
        pop_out[b * ld] = pop0[b];
        for (int k = 1; k <= steps[b]; ++k) pop_out[b * ld + k] = h[b * ld + k];
      }
    }
    if (dnrm && rc == MPC_OK) {
      if (cudaMemcpy(h.data(), dnrm, sizeof(double) * h.size(), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
        rc = mpc_fail(MPC_ERR_CUDA, "history copy failed");
      for (int b = 0; rc == MPC_OK && b < B; ++b)
        for (int k = 0; k < steps[b]; ++k) norm_out[b * (ld - 1) + k] = h[b * ld + k];
    }
  }
  release();
  return rc;
}

}  // extern "C"
