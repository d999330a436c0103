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
  unsigned* bar_count;
  unsigned* bar_gen;
  unsigned* status;
  double* pop_hist;        // [steps+1] (entry 0 written too)
  double* norm_hist;       // [steps]
  int pop_index;
  int steps;
  int gauge;               // 0 length, 1 velocity
  int first_is_normalised; // XN at entry holds a normalised x (norm 1)
  double dt;
  Geometry g;
};

// Grid barrier on a counter and a generation word; bounded wait.  Returns
// false if it timed out (status raised).
__device__ bool grid_sync(const ResArgs& a, unsigned& gen, bool& dead) {
  __syncthreads();
  __shared__ int timed_out;
  if (threadIdx.x == 0) {
    timed_out = 0;
    __threadfence();
    const unsigned g0 = gen;
    if (atomicAdd(a.bar_count, 1u) == gridDim.x - 1) {
      atomicExch(a.bar_count, 0u);
      __threadfence();
      atomicAdd(a.bar_gen, 1u);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      unsigned it = 0;
      while (*(volatile unsigned*)a.bar_gen == g0) {
        if ((++it & 1023u) == 0 && globaltimer_ns() - t0 > kWaitLimitNs) {
          atomicOr(a.status, ST_WAIT_TIMEOUT);
          timed_out = 1;
          break;
        }
      }
    }
    __threadfence();
    gen = g0 + 1;
  }
  __syncthreads();
  if (timed_out) dead = true;
  return !dead;
}

__device__ __forceinline__ double2 ld_cg(const double2* p) { return __ldcg(p); }

__global__ void __launch_bounds__(RTHREADS, 1) k_prop_resident(const __grid_constant__ ResArgs a) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const Geometry& g = a.g;
  const int G = gridDim.x, c = blockIdx.x;
  const int row0 = (int)((long long)g.ntot * c / G);
  const int row1 = (int)((long long)g.ntot * (c + 1) / G);
  const int nrows = row1 - row0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // blocks touched by this CTA's rows and the stage-vector window they couple to
  int Llo = 0;
  while (Llo + 1 < g.nstate_blk && row0 >= g.state_off[Llo + 1]) ++Llo;
  int Lhi = Llo;
  while (Lhi + 1 < g.nstate_blk && row1 - 1 >= g.state_off[Lhi + 1]) ++Lhi;
  const int wlo = g.state_off[max(Llo - 1, 0)];
  const int whi = g.state_off[min(Lhi + 2, g.nstate_blk)];
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
  for (int li = warp; li < nrows; li += RWARPS) {
    const int i = row0 + li;
    int L = 0;
    while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
    const int r = i - g.state_off[L];
    double* dst = crow + roff[li];
    int o = 0;
    if (L > 0) {
      const BlockGeom& b = g.blk[L - 1];  // column r of D_{L-1}
      for (int k = lane; k < b.nrow; k += 32) dst[k] = a.D[b.d_off + (long long)k * b.pitch + r];
      o = b.nrow;
    }
    if (L < g.nblk) {
      const BlockGeom& b = g.blk[L];      // row r of D_L
      const double sg = (a.gauge == 1) ? -1.0 : 1.0;
      for (int k = lane; k < b.ncol; k += 32) dst[o + k] = sg * a.D[b.d_off + (long long)r * b.pitch + k];
    }
  }
  unsigned gen = *(volatile unsigned*)a.bar_gen;
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
        for (int li = threadIdx.x; li < nrows; li += RTHREADS) xsm[li] = ywin[row0 + li - wlo];
        if (c == 0 && threadIdx.x == 0 && step > 0) a.norm_hist[step - 1] = nrm;
        if (threadIdx.x == 0 && a.pop_index >= row0 && a.pop_index < row1) {
          const double2 v = ywin[a.pop_index - wlo];
          a.pop_hist[step] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
        }
      } else {
        const double2* Yin = a.Y[s & 1];
        for (int k = threadIdx.x; k < wlen; k += RTHREADS) ywin[k] = ld_cg(Yin + wlo + k);
      }
      __syncthreads();
      // ---- k_s for this CTA's rows: one warp per row ----
      for (int li = warp; li < nrows; li += RWARPS) {
        const int i = row0 + li;
        int L = 0;
        while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
        const double* cr = crow + roff[li];
        double wr = 0.0, wi = 0.0;
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
      if (!grid_sync(a, gen, dead)) break;
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
      a.norm_hist[a.steps - 1] = nrm;
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

}  // namespace

struct mpc_resident_state {
  int G = 0;
  size_t smem = 0;
  double2* Y0 = nullptr;
  double2* Y1 = nullptr;
  double2* XN = nullptr;
  double* part = nullptr;
  unsigned* bar = nullptr;  // [0] count, [1] generation
  bool ok = false;
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
  if (cudaMemcpyToSymbol(r_A, A, sizeof A) != cudaSuccess ||
      cudaMemcpyToSymbol(r_B8, B8, sizeof B8) != cudaSuccess)
    return false;
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
  cudaFree(r->Y0);
  cudaFree(r->Y1);
  cudaFree(r->XN);
  cudaFree(r->part);
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
  a.bar_count = r->bar;
  a.bar_gen = r->bar + 1;
  a.status = c->d_status;
  a.pop_hist = c->d_pop;
  a.norm_hist = c->d_nrm;
  a.pop_index = pop_index;
  a.steps = steps;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.first_is_normalised = 1;
  a.dt = dt;
  a.g = c->g;
  CK(cudaMemcpyAsync(r->XN, c->d_x, sizeof(double2) * c->g.ntot, cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaMemsetAsync(r->bar, 0, sizeof(unsigned), c->stream));  // arrival count
  void* args[] = {&a};
  ProfScope ps(c, MPC_KERNEL_RESIDENT);
  CK(cudaLaunchCooperativeKernel((const void*)k_prop_resident, dim3(r->G), dim3(RTHREADS), args,
                                 r->smem, c->stream));
  return MPC_OK;
}
