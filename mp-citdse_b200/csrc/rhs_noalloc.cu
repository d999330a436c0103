// rhs_noalloc.cu -- one right-hand-side evaluation that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host framework whose caching
// allocator already owns the device memory (a raw cudaMalloc there can fail
// or fragment the pool, so every buffer must come from the framework), a
// solver plugin loaded into a simulation code that forbids allocation after
// start-up, or a time-critical loop where cudaMalloc/cudaFree would add
// milliseconds and an implicit device synchronisation.  For them,
// mpc_rhs_noalloc evaluates dxdt = f(x) on caller-owned device buffers and
// keeps its only scratch -- the row and column partials of the dipole pass --
// in the file-scope array below.
//
// The array is MPC_NOALLOC_SCRATCH_BYTES (16 MiB) and lives on every GPU that
// loads the library until the process exits.  Every call shares it and it
// keeps the last call's contents, so calls whose kernels overlap on the GPU
// (different streams, or different host threads, on the same device) race;
// serialise them.  Each call writes every scratch entry it later reads, so no
// entry has to start at zero.
//
// In host code `g_scratch` is only a host-side stand-in for the device array,
// not a device address: the address is obtained with cudaGetSymbolAddress on
// the first call on each device (with that device current) and cached
// together with the identity of the CUDA context it belongs to.  When the
// current context of the device changes (after cudaDeviceReset, or when the
// caller makes another context current), the module is loaded anew in that
// context and the address is looked up again.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/mpc_tdse.h"
#include "plan.h"

int mpc_internal_fail(int code, const char* msg);  // mpc_tdse.cu

namespace mpc {
namespace {

static __device__ __align__(256) unsigned char g_scratch[MPC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr int kMaxCtas = 160;
constexpr int kMaxStripsNA = 256;
constexpr int kThreadsNA = kConsumerWarps * 32;

struct DirectArgs {
  const double* D;       // caller's dipole blocks, back to back, row-major, unpadded
  const double2* x;
  double2* RP;
  double2* CP;
  Geometry g;            // pitch = ncol, d_off = offset of block L in D
  int cta_slot0[kMaxCtas];
};

struct EpiArgs {
  const double2* x;
  const double* eig;
  double2* dxdt;
  const double2* RP;
  const double2* CP;
  double F;
  int gauge;             // 0 length, 1 velocity
  Geometry g;
  int strip_slot0[kMaxStripsNA + 1];
};

// The dipole pass of k_rhs_stream with the tiles read straight from global
// memory (the caller's rows need not be 16-byte aligned, so no TMA).
__global__ void __launch_bounds__(kThreadsNA, 1) k_rhs_direct(const __grid_constant__ DirectArgs a) {
  __shared__ double2 red[kConsumerWarps * kStripW];
  const Geometry& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t_begin = (int)((long long)g.ntiles * blockIdx.x / gridDim.x);
  const int t_end = (int)((long long)g.ntiles * (blockIdx.x + 1) / gridDim.x);
  double2 ycol[8], cacc[8];
  int cur_b = -1, cur_s = -1;
  int slot = a.cta_slot0[blockIdx.x] - 1;

  auto flush = [&]() {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      red[warp * kStripW + 64 * j + 2 * lane] = cacc[2 * j];
      red[warp * kStripW + 64 * j + 2 * lane + 1] = cacc[2 * j + 1];
    }
    __syncthreads();
    double2 acc = red[threadIdx.x];
    for (int w = 1; w < kConsumerWarps; ++w) {
      const double2 v = red[w * kStripW + threadIdx.x];
      acc.x += v.x;
      acc.y += v.y;
    }
    a.CP[(long long)slot * kStripW + threadIdx.x] = acc;
    __syncthreads();
  };

  for (int t = t_begin; t < t_end; ++t) {
    int b, s, rt;
    decode_tile(g, t, b, s, rt);
    const BlockGeom& bg = g.blk[b];
    if (b != cur_b || s != cur_s) {
      if (cur_b >= 0) flush();
      ++slot;
      cur_b = b;
      cur_s = s;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = s * kStripW + 64 * j + 2 * lane + e;
          ycol[2 * j + e] = (c < bg.ncol) ? a.x[bg.col_off + c] : make_double2(0.0, 0.0);
          cacc[2 * j + e] = make_double2(0.0, 0.0);
        }
    }
    const int r0 = rt * kTileR + 2 * warp;
    const bool ok0 = r0 < bg.nrow, ok1 = r0 + 1 < bg.nrow;
    const double2 yr0 = ok0 ? a.x[bg.row_off + r0] : make_double2(0.0, 0.0);
    const double2 yr1 = ok1 ? a.x[bg.row_off + r0 + 1] : make_double2(0.0, 0.0);
    const double* D0 = a.D + bg.d_off + (long long)r0 * bg.ncol;
    const double* D1 = D0 + bg.ncol;
    double2 ra = make_double2(0.0, 0.0), rb = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = s * kStripW + 64 * j + 2 * lane;
      double2 d0, d1;
      d0.x = (ok0 && c < bg.ncol) ? __ldg(D0 + c) : 0.0;
      d0.y = (ok0 && c + 1 < bg.ncol) ? __ldg(D0 + c + 1) : 0.0;
      d1.x = (ok1 && c < bg.ncol) ? __ldg(D1 + c) : 0.0;
      d1.y = (ok1 && c + 1 < bg.ncol) ? __ldg(D1 + c + 1) : 0.0;
      const double2 c0 = ycol[2 * j], c1 = ycol[2 * j + 1];
      ra.x = fma(d0.x, c0.x, ra.x); ra.x = fma(d0.y, c1.x, ra.x);
      ra.y = fma(d0.x, c0.y, ra.y); ra.y = fma(d0.y, c1.y, ra.y);
      rb.x = fma(d1.x, c0.x, rb.x); rb.x = fma(d1.y, c1.x, rb.x);
      rb.y = fma(d1.x, c0.y, rb.y); rb.y = fma(d1.y, c1.y, rb.y);
      double2& q0 = cacc[2 * j];
      double2& q1 = cacc[2 * j + 1];
      q0.x = fma(d0.x, yr0.x, q0.x); q0.x = fma(d1.x, yr1.x, q0.x);
      q0.y = fma(d0.x, yr0.y, q0.y); q0.y = fma(d1.x, yr1.y, q0.y);
      q1.x = fma(d0.y, yr0.x, q1.x); q1.x = fma(d1.y, yr1.x, q1.x);
      q1.y = fma(d0.y, yr0.y, q1.y); q1.y = fma(d1.y, yr1.y, q1.y);
    }
    const bool hi16 = (lane & 16) != 0;
    const double s0 = hi16 ? ra.x : rb.x, s1 = hi16 ? ra.y : rb.y;
    const double k0 = hi16 ? rb.x : ra.x, k1 = hi16 ? rb.y : ra.y;
    const double w0 = k0 + __shfl_xor_sync(0xffffffffu, s0, 16);
    const double w1 = k1 + __shfl_xor_sync(0xffffffffu, s1, 16);
    const bool hi8 = (lane & 8) != 0;
    double z = (hi8 ? w1 : w0) + __shfl_xor_sync(0xffffffffu, hi8 ? w0 : w1, 8);
    z += __shfl_xor_sync(0xffffffffu, z, 4);
    z += __shfl_xor_sync(0xffffffffu, z, 2);
    z += __shfl_xor_sync(0xffffffffu, z, 1);
    if ((lane & 7) == 0) {
      const int r = r0 + (hi16 ? 1 : 0);
      if (r < bg.nrow)
        reinterpret_cast<double*>(a.RP + bg.rp_off + (long long)s * bg.nrow + r)[hi8 ? 1 : 0] = z;
    }
  }
  if (cur_b >= 0) flush();
}

// dxdt = f(x) from the partials, in the reference's order of operations.
__global__ void __launch_bounds__(256) k_rhs_direct_epilogue(const __grid_constant__ EpiArgs a) {
  const Geometry& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.ntot) return;
  int L = 0;
  while (L + 1 < g.nstate_blk && i >= g.state_off[L + 1]) ++L;
  const int r = i - g.state_off[L];
  double2 Q = make_double2(0.0, 0.0), P = make_double2(0.0, 0.0);
  if (L < g.nblk) {
    const BlockGeom& b = g.blk[L];
    const double2* rp = a.RP + b.rp_off + r;
    Q = rp[0];
    for (int s = 1; s < b.nstrips; ++s) {
      const double2 v = rp[(long long)s * b.nrow];
      Q.x = __dadd_rn(Q.x, v.x);
      Q.y = __dadd_rn(Q.y, v.y);
    }
  }
  if (L > 0) {
    const BlockGeom& b = g.blk[L - 1];
    const int gs = b.strip0 + r / kStripW, c = r % kStripW;
    const int s0 = a.strip_slot0[gs], s1 = a.strip_slot0[gs + 1];
    P = a.CP[(long long)s0 * kStripW + c];
    for (int sl = s0 + 1; sl < s1; ++sl) {
      const double2 v = a.CP[(long long)sl * kStripW + c];
      P.x = __dadd_rn(P.x, v.x);
      P.y = __dadd_rn(P.y, v.y);
    }
  }
  const double F = a.F, e = a.eig[i];
  const double2 y = a.x[i];
  double kre = __dmul_rn(e, y.y), kim = __dmul_rn(-e, y.x);
  if (a.gauge == 0) {
    if (L > 0) { kim = __dadd_rn(kim, __dmul_rn(-F, P.x)); kre = __dadd_rn(kre, __dmul_rn(F, P.y)); }
    if (L < g.nblk) { kim = __dadd_rn(kim, __dmul_rn(-F, Q.x)); kre = __dadd_rn(kre, __dmul_rn(F, Q.y)); }
  } else {
    if (L > 0) { kre = __dadd_rn(kre, __dmul_rn(F, P.x)); kim = __dadd_rn(kim, __dmul_rn(F, P.y)); }
    if (L < g.nblk) { kre = __dadd_rn(kre, __dmul_rn(-F, Q.x)); kim = __dadd_rn(kim, __dmul_rn(-F, Q.y)); }
  }
  a.dxdt[i] = make_double2(kre, kim);
}

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// Identity of the calling thread's current CUDA context (0 when none is
// current yet), through the driver entry points the runtime exposes.
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked = false;
  if (!looked) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
    cudaGetLastError();
    looked = true;
  }
  CUcontext cu = nullptr;
  if (!get_cur || get_cur(&cu) != CUDA_SUCCESS || !cu) return 0;
  unsigned long long id = 0;
  if (get_id && get_id(cu, &id) == CUDA_SUCCESS) return id + 1;
  return (unsigned long long)(uintptr_t)cu;
}

// Look up the device address of g_scratch (with device `dev` current) and the
// SM count on the first call in each CUDA context; both are cached until the
// device's current context changes.
int device_setup(int dev, void** scratch, int* sms) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  const unsigned long long ctx = current_ctx_id();
  if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      char m[256];
      std::snprintf(m, sizeof m, "cudaGetSymbolAddress(g_scratch) failed: %s",
                    cudaGetErrorString(e));
      return mpc_internal_fail(MPC_ERR_CUDA, m);
    }
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || n <= 0)
      return mpc_internal_fail(MPC_ERR_CUDA, "cannot read the SM count");
    g_num_sms[dev] = n;
    g_scratch_addr[dev] = p;
    // the symbol lookup made the device's primary context current if none was
    g_scratch_ctx[dev] = ctx ? ctx : current_ctx_id();
  }
  *scratch = g_scratch_addr[dev];
  *sms = g_num_sms[dev];
  return MPC_OK;
}

}  // namespace
}  // namespace mpc

using namespace mpc;

extern "C" int mpc_rhs_noalloc(int L_max, const int* state_sz, const double* d_eig,
                               const double* d_dip, char gauge, double F, const double* d_x,
                               double* d_dxdt, void* stream) {
  if (!state_sz || !d_eig || !d_dip || !d_x || !d_dxdt)
    return mpc_internal_fail(MPC_ERR_ARG, "mpc_rhs_noalloc: null argument");
  if (L_max < 1 || L_max >= kMaxBlocks)
    return mpc_internal_fail(MPC_ERR_ARG, "mpc_rhs_noalloc: L_max out of range");
  if (gauge != 'l' && gauge != 'v')
    return mpc_internal_fail(MPC_ERR_ARG, "mpc_rhs_noalloc: gauge must be 'l' or 'v'");
  for (int L = 0; L <= L_max; ++L)
    if (state_sz[L] <= 0) return mpc_internal_fail(MPC_ERR_ARG, "mpc_rhs_noalloc: state_sz <= 0");
  // the kernels read and write x / dxdt as 16-byte complex pairs and the
  // energies / dipoles as doubles: a misaligned view is refused here, before
  // any launch, instead of faulting on the device
  if (((uintptr_t)d_x | (uintptr_t)d_dxdt) & 15u)
    return mpc_internal_fail(MPC_ERR_ARG,
                             "mpc_rhs_noalloc: d_x and d_dxdt must be 16-byte aligned");
  if (((uintptr_t)d_eig | (uintptr_t)d_dip) & 7u)
    return mpc_internal_fail(MPC_ERR_ARG,
                             "mpc_rhs_noalloc: d_eig and d_dip must be 8-byte aligned");

  // geometry on the stack (nothing is allocated, on the host either)
  DirectArgs da;
  EpiArgs ea;
  Geometry& g = da.g;
  g = Geometry{};
  g.nblk = L_max;
  g.nstate_blk = L_max + 1;
  long long tot = 0;
  g.state_off[0] = 0;
  for (int L = 0; L <= L_max; ++L) {
    tot += state_sz[L];
    if (tot > (1LL << 30)) return mpc_internal_fail(MPC_ERR_ARG, "mpc_rhs_noalloc: too many states");
    g.state_off[L + 1] = (int)tot;
  }
  g.ntot = (int)tot;
  long long tiles = 0, strips = 0, rp = 0, doff = 0;
  for (int L = 0; L < L_max; ++L) {
    BlockGeom& b = g.blk[L];
    b.nrow = state_sz[L];
    b.ncol = state_sz[L + 1];
    b.row_off = g.state_off[L];
    b.col_off = g.state_off[L + 1];
    b.pitch = b.ncol;
    b.nstrips = (b.ncol + kStripW - 1) / kStripW;
    b.nrtiles = (b.nrow + kTileR - 1) / kTileR;
    b.tile0 = (int)tiles;
    b.strip0 = (int)strips;
    b.d_off = doff;
    b.rp_off = rp;
    tiles += (long long)b.nstrips * b.nrtiles;
    strips += b.nstrips;
    rp += (long long)b.nstrips * b.nrow;
    doff += (long long)b.nrow * b.ncol;
  }
  if (strips > kMaxStripsNA)
    return mpc_internal_fail(MPC_ERR_ARG,
                             "mpc_rhs_noalloc: more than 256 column strips (sum over blocks "
                             "L>=1 of ceil(n_L/256)); use mpc_rhs");
  g.ntiles = (int)tiles;
  g.nstrips = (int)strips;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return mpc_internal_fail(MPC_ERR_CUDA, "mpc_rhs_noalloc: no current CUDA device");
  void* scratch = nullptr;
  int sms = 0;
  int rc = device_setup(dev, &scratch, &sms);
  if (rc) return rc;

  int G = sms < g.ntiles ? sms : g.ntiles;
  if (G > kMaxCtas) G = kMaxCtas;
  // column-partial slots: one per (CTA, strip) pair the CTA touches
  int slot = 0;
  for (int s = 0; s <= kMaxStripsNA; ++s) ea.strip_slot0[s] = -1;
  for (int cta = 0; cta < G; ++cta) {
    const int t0 = (int)((long long)g.ntiles * cta / G);
    const int t1 = (int)((long long)g.ntiles * (cta + 1) / G);
    da.cta_slot0[cta] = slot;
    int last = -1;
    for (int t = t0; t < t1; ++t) {
      int b, s, rt;
      decode_tile(g, t, b, s, rt);
      const int gs = g.blk[b].strip0 + s;
      if (gs != last) {
        if (ea.strip_slot0[gs] < 0) ea.strip_slot0[gs] = slot;
        ++slot;
        last = gs;
      }
    }
  }
  ea.strip_slot0[g.nstrips] = slot;
  const unsigned long long need =
      16ull * (unsigned long long)rp + 16ull * (unsigned long long)slot * kStripW;
  if (need > MPC_NOALLOC_SCRATCH_BYTES) {
    char m[256];
    std::snprintf(m, sizeof m,
                  "mpc_rhs_noalloc: this system needs %llu bytes of scratch, more than the "
                  "%u-byte static maximum; use mpc_rhs",
                  need, (unsigned)MPC_NOALLOC_SCRATCH_BYTES);
    return mpc_internal_fail(MPC_ERR_ARG, m);
  }
  double2* RP = static_cast<double2*>(scratch);
  double2* CP = RP + rp;

  da.D = d_dip;
  da.x = reinterpret_cast<const double2*>(d_x);
  da.RP = RP;
  da.CP = CP;
  ea.x = da.x;
  ea.eig = d_eig;
  ea.dxdt = reinterpret_cast<double2*>(d_dxdt);
  ea.RP = RP;
  ea.CP = CP;
  ea.F = F;
  ea.gauge = (gauge == 'l') ? 0 : 1;
  ea.g = g;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_rhs_direct<<<G, kThreadsNA, 0, st>>>(da);
  k_rhs_direct_epilogue<<<(g.ntot + 255) / 256, 256, 0, st>>>(ea);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char m[256];
    std::snprintf(m, sizeof m, "mpc_rhs_noalloc: launch failed: %s", cudaGetErrorString(e));
    return mpc_internal_fail(MPC_ERR_CUDA, m);
  }
  return MPC_OK;
}
