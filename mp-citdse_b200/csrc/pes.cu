// pes.cu -- photoelectron spectra and populations of a propagated state,
// computed on the GPU from the coefficients (the reference's downstream
// `pes` program, src/pes/pes.cpp:48-262, which reads them back from 6-digit
// text files).
//
// 1e (pes::genPES1e): the grid is the l = 1 energies E1[k]; state i >= 1 of
//   block l adds |c_i|^2 * 2 / (dn + dp) to bin k (1 <= k <= n0 - 2,
//   dn = |E1[k] - E1[k-1]|, dp = |E1[k+1] - E1[k]|) when
//   E1[k] - dn/2 < E_i < E1[k] + dp/2, and |c_i|^2 to the yield if E1[k] > 0;
//   the summed spectrum adds the blocks.
// 2e (pes::genPES2e): per L, state 1 <= i <= n_L - 2 with E_i > threshold
//   has density |c_i|^2 * 2 / (E_{i+1} - E_{i-1}) at E_i - threshold and adds
//   to the yield; every such state except the global ground state adds to
//   the excited population.  The summed spectrum (pes -s, mpc_pes_summed)
//   bins every state i >= 1 of every block onto the L = 1 energies as in 1e
//   (bins 1 <= k <= n1 - 1, whose upper neighbour for k = n1 - 1 is the first
//   energy of L = 2, as the reference indexes its concatenated energies; with
//   L_max = 1 there is no such energy and the bins stop at n1 - 2).
// Sums run in a fixed order (one thread per bin or state, then one CTA), so
// results repeat bit for bit.
#include <cuda_runtime.h>

#include <vector>

#include "ctx.h"

using namespace mpc;

namespace {

struct PesArgs {
  const double2* c;
  const double* eps;
  double* pes;       // [nblocks][ngrid]
  double* yield_c;   // [ntot] per-state yield contribution
  double* exc_c;     // [ntot] per-state excitation contribution
  double* stats;     // [4] ground, norm, yield, excitation
  int electrons;
  double threshold;
  int ngrid;         // columns of pes
  Geometry g;
};

__device__ __forceinline__ double nsq(double2 v) { return v.x * v.x + v.y * v.y; }

// one thread per (block, grid slot)
__global__ void k_pes(const __grid_constant__ PesArgs a) {
  const Geometry& g = a.g;
  const int L = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.ngrid) return;
  const int o = g.state_off[L], nL = g.state_off[L + 1] - o;
  double out = 0.0;
  if (a.electrons == 1) {
    // bins on the l = 1 energies; the reference loops k over 1 .. n0 - 2
    const int n0 = g.state_off[1] - g.state_off[0];
    const double* E1 = a.eps + g.state_off[1];
    if (k >= 1 && k <= n0 - 2) {
      const double dn = fabs(E1[k] - E1[k - 1]), dp = fabs(E1[k + 1] - E1[k]);
      const double lo = E1[k] - 0.5 * dn, hi = E1[k] + 0.5 * dp;
      for (int i = 1; i < nL; ++i) {
        const double e = a.eps[o + i];
        if (e > lo && e < hi) out += nsq(a.c[o + i]) * 2.0 / (dn + dp);
      }
    }
  } else {
    // per-state density at E_i - threshold
    if (k >= 1 && k <= nL - 2) {
      const double e = a.eps[o + k];
      if (e - a.threshold > 0.0) out = nsq(a.c[o + k]) * 2.0 / (a.eps[o + k + 1] - a.eps[o + k - 1]);
    }
  }
  a.pes[(long long)L * a.ngrid + k] = out;
}

// per-state contributions to the yield and excitation
__global__ void k_pes_contrib(const __grid_constant__ PesArgs a) {
  const Geometry& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.ntot) return;
  int L = 0;
  while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
  const int o = g.state_off[L], r = i - o, nL = g.state_off[L + 1] - o;
  const double p = nsq(a.c[i]);
  double y = 0.0, x = 0.0;
  if (a.electrons == 1) {
    const int n0 = g.state_off[1] - g.state_off[0];
    const double* E1 = a.eps + g.state_off[1];
    if (r >= 1) {
      const double e = a.eps[i];
      for (int k = 1; k <= n0 - 2; ++k) {  // first bin that holds the state
        const double dn = fabs(E1[k] - E1[k - 1]), dp = fabs(E1[k + 1] - E1[k]);
        if (e > E1[k] - 0.5 * dn && e < E1[k] + 0.5 * dp) {
          y = (E1[k] > 0.0) ? p : 0.0;
          break;
        }
      }
    }
  } else {
    if (r >= 1 && r <= nL - 2) {
      if (a.eps[i] - a.threshold > 0.0) y = p;
      if (i > 0) x = p;
    }
  }
  a.yield_c[i] = y;
  a.exc_c[i] = x;
}

__global__ void k_pes_stats(const __grid_constant__ PesArgs a) {
  __shared__ double sh[3][32];
  double nrm = 0.0, y = 0.0, x = 0.0;
  for (int i = threadIdx.x; i < a.g.ntot; i += blockDim.x) {
    nrm += nsq(a.c[i]);
    y += a.yield_c[i];
    x += a.exc_c[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
    x += __shfl_xor_sync(0xffffffffu, x, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = nrm;
    sh[1][threadIdx.x >> 5] = y;
    sh[2][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s0 += sh[0][w];
      s1 += sh[1][w];
      s2 += sh[2][w];
    }
    a.stats[0] = nsq(a.c[0]);
    a.stats[1] = s0;
    a.stats[2] = s1;
    a.stats[3] = s2;
  }
}

// The summed spectrum, one thread per bin k of the L = 1 grid.  Per bin the
// states are visited in the reference's order (block by block, state by
// state); the bins are disjoint intervals, so a state's first matching bin
// is its only one.
__global__ void k_pes_summed(const __grid_constant__ PesArgs a, double* grid, int n1) {
  const Geometry& g = a.g;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n1) return;
  const double* E1 = a.eps + g.state_off[1];
  double out = 0.0;
  if (a.electrons == 1) {
    const int n0 = g.state_off[1] - g.state_off[0];
    if (k >= 1 && k <= n0 - 2) {
      const double dn = fabs(E1[k] - E1[k - 1]), dp = fabs(E1[k + 1] - E1[k]);
      const double lo = E1[k] - 0.5 * dn, hi = E1[k] + 0.5 * dp;
      for (int L = 0; L < g.nstate_blk; ++L) {  // the block's spectrum, then the sum
        const int o = g.state_off[L], nL = g.state_off[L + 1] - o;
        double pl = 0.0;
        for (int i = 1; i < nL; ++i) {
          const double e = a.eps[o + i];
          if (e > lo && e < hi) pl += nsq(a.c[o + i]) * 2.0 / (dn + dp);
        }
        out += pl;
      }
    }
    grid[k] = E1[k];
  } else {
    const int kmax = g.nstate_blk > 2 ? n1 - 1 : n1 - 2;
    if (k >= 1 && k <= kmax) {
      // E1[k + 1] is the first L = 2 energy for k = n1 - 1 (contiguous eps)
      const double dn = fabs(E1[k] - E1[k - 1]), dp = fabs(E1[k + 1] - E1[k]);
      const double lo = E1[k] - 0.5 * dn, hi = E1[k] + 0.5 * dp;
      for (int L = 0; L < g.nstate_blk; ++L) {
        const int o = g.state_off[L], nL = g.state_off[L + 1] - o;
        for (int i = 1; i < nL; ++i) {
          const double e = a.eps[o + i];
          if (e > lo && e < hi) out += nsq(a.c[o + i]) * 2.0 / (dn + dp);
        }
      }
    }
    grid[k] = E1[k] - a.threshold;
  }
  a.pes[k] = out;
}

}  // namespace

extern "C" int mpc_pes_summed(mpc_ctx* c, int electrons, double threshold, const double* ct,
                              double* grid, double* pes, int ngrid) {
  if (!c || !grid || !pes || (electrons != 1 && electrons != 2))
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  const Geometry& g = c->g;
  if (g.nstate_blk < 2) return mpc_fail(MPC_ERR_ARG, "the summed spectrum needs block 1");
  const int n1 = g.state_off[2] - g.state_off[1];
  if (ngrid < n1) return mpc_fail(MPC_ERR_ARG, "ngrid must be at least n_1 (%d)", n1);
  CK(cudaSetDevice(c->device));
  double *d_pes = nullptr, *d_grid = nullptr;
  CK(cudaMallocAsync(&d_pes, sizeof(double) * n1, c->stream));
  CK(cudaMallocAsync(&d_grid, sizeof(double) * n1, c->stream));
  if (ct)
    CK(cudaMemcpyAsync(c->d_y, ct, sizeof(double2) * g.ntot, cudaMemcpyHostToDevice, c->stream));
  PesArgs a{};
  a.c = ct ? c->d_y : c->d_x;
  a.eps = c->d_eps;
  a.pes = d_pes;
  a.electrons = electrons;
  a.threshold = threshold;
  a.ngrid = n1;
  a.g = g;
  k_pes_summed<<<(n1 + 127) / 128, 128, 0, c->stream>>>(a, d_grid, n1);
  CK(cudaGetLastError());
  c->launches += 1;
  CK(cudaMemcpyAsync(pes, d_pes, sizeof(double) * n1, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(grid, d_grid, sizeof(double) * n1, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(d_pes, c->stream));
  CK(cudaFreeAsync(d_grid, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = n1; k < ngrid; ++k) pes[k] = grid[k] = 0.0;
  return MPC_OK;
}

extern "C" int mpc_pes(mpc_ctx* c, int electrons, double threshold, const double* ct, double* pes,
                       int ngrid, double* stats) {
  NvtxRange nvtx_("mpc_pes");
  if (!c || !pes || !stats || (electrons != 1 && electrons != 2))
    return mpc_fail(MPC_ERR_ARG, "bad argument");
  const Geometry& g = c->g;
  int need = 0;
  for (int L = 0; L < g.nstate_blk; ++L) need = std::max(need, g.state_off[L + 1] - g.state_off[L]);
  if (ngrid < need) return mpc_fail(MPC_ERR_ARG, "ngrid must be at least the largest block (%d)", need);
  if (electrons == 1 && g.nstate_blk < 2) return mpc_fail(MPC_ERR_ARG, "1e spectra need l = 1");
  CK(cudaSetDevice(c->device));
  const size_t n = g.ntot;
  double *d_pes = nullptr, *d_y = nullptr, *d_x = nullptr, *d_st = nullptr;
  double2* d_c = c->d_x;
  CK(cudaMallocAsync(&d_pes, sizeof(double) * (size_t)g.nstate_blk * ngrid, c->stream));
  CK(cudaMallocAsync(&d_y, sizeof(double) * n, c->stream));
  CK(cudaMallocAsync(&d_x, sizeof(double) * n, c->stream));
  CK(cudaMallocAsync(&d_st, sizeof(double) * 4, c->stream));
  if (ct) CK(cudaMemcpyAsync(c->d_y, ct, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream));
  PesArgs a{};
  a.c = ct ? c->d_y : d_c;
  a.eps = c->d_eps;
  a.pes = d_pes;
  a.yield_c = d_y;
  a.exc_c = d_x;
  a.stats = d_st;
  a.electrons = electrons;
  a.threshold = threshold;
  a.ngrid = ngrid;
  a.g = g;
  k_pes<<<dim3((ngrid + 127) / 128, g.nstate_blk), 128, 0, c->stream>>>(a);
  k_pes_contrib<<<(int)((n + 255) / 256), 256, 0, c->stream>>>(a);
  k_pes_stats<<<1, 1024, 0, c->stream>>>(a);
  CK(cudaGetLastError());
  c->launches += 3;
  CK(cudaMemcpyAsync(pes, d_pes, sizeof(double) * (size_t)g.nstate_blk * ngrid,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(stats, d_st, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(d_pes, c->stream));
  CK(cudaFreeAsync(d_y, c->stream));
  CK(cudaFreeAsync(d_x, c->stream));
  CK(cudaFreeAsync(d_st, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MPC_OK;
}
