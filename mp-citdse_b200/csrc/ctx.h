// ctx.h -- the context object shared by the library's translation units,
// and its error helpers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/mpc_tdse.h"
#include "dev_util.cuh"
#include "plan.h"
#include "stream_types.h"

// Records `fmt` as the calling thread's last error and returns `code`.
int mpc_fail(int code, const char* fmt, ...);
int mpc_internal_fail(int code, const char* msg);
// A 2-D FP64 tensor map for TMA loads (mpc_tdse.cu).
int mpc_encode_map_2d(CUtensorMap* m, const void* base, unsigned long long inner,
                      unsigned long long outer, unsigned long long row_bytes, unsigned box_inner,
                      unsigned box_outer, bool swizzle128);
// A 3-D FP64 tensor map over [rows][cols] viewed as 16-column groups
// (mpc_tdse.cu).
int mpc_encode_map_grouped(CUtensorMap* m, const void* base, unsigned long long cols,
                           unsigned long long rows, unsigned long long row_bytes,
                           unsigned box_rows, unsigned box_groups);

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return mpc_fail(e_ == cudaErrorMemoryAllocation ? MPC_ERR_NOMEM : MPC_ERR_CUDA,    \
                      "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                      __LINE__);                                                         \
  } while (0)

struct mpc_batch_state;

struct mpc_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  char gauge = 'l';
  mpc::Geometry g{};
  std::vector<int> n;
  double eps_max = 0.0;

  // device buffers
  double* d_eps = nullptr;
  double* d_D = nullptr;
  double2* d_x = nullptr;
  double2* d_y = nullptr;
  double2* d_v = nullptr;   // Horner products' second buffer (zero tail like d_x, d_y)
  double2* d_k = nullptr;
  double2* d_RP = nullptr;
  double2* d_CP = nullptr;
  int* d_cta_slot0 = nullptr;
  int* d_strip_slot0 = nullptr;
  double* d_norm_part = nullptr;
  unsigned* d_status = nullptr;
  double* d_Ftab = nullptr;
  double* d_pop = nullptr;
  double* d_nrm = nullptr;
  int hist_cap = 0;

  // profiling: event pairs per kernel kind, and a launch counter
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[6];
  std::vector<cudaEvent_t> ev_pool;
  long long launches = 0;

  int stream_grid = 0;
  int combine_grid = 0;
  mpc::TmapSet tmaps{};
  mpc::StreamArgs sargs{};
  std::vector<void*> allocs;

  mpc_batch_state* batch = nullptr;  // batched-propagation work space (batch.cu)
  struct mpc_adjoint_state* adj = nullptr;  // adjoint work space (adjoint.cu)
  struct mpc_resident_state* resident = nullptr;  // resident path (resident.cu)
  struct mpc_batch_res_state* batch_res = nullptr;  // resident batched path (batch_resident.cu)
  struct mpc_badj_state* badj = nullptr;  // batched objective / adjoint (batch_adjoint.cu)
  int path = 0;  // 0 automatic, 1 streaming, 2 resident (MPC_PATH_*)
  double yield_thr = 0.0;  // yield objective: 1 - sum over states below this energy
  // MPC_BATCH_VARIANT=v at context creation pins the stage-GEMM tile variant
  // (tests check that every variant gives the same bits); -1: tuned/default
  int forced_variant = -1;
  // MPC_NO_PERSIST=1 at context creation: the batched fixed step as one launch
  // per Horner product instead of the persistent launch
  bool no_persist = false;
  // MPC_FORCE_PERSIST=1 at context creation: the persistent launch at every
  // width (tests of that path; it is correct at any width, not always faster)
  bool force_persist = false;
  // MPC_FORCE_TMA=s at context creation: the batched fixed step as the
  // TMA-fed product launches on TMA tile shape s - 1 at every width (tests);
  // MPC_NO_TMA=1: the fixed-step tuner leaves the TMA-fed launches out
  int force_tma = 0;
  bool no_tma = false;
  // MPC_STAGE_FORM=1 at context creation: the streamed single-pulse steps as
  // 13 stages instead of the 12 Horner products of the stability polynomial
  bool stage_form = false;
  // grid-barrier wait limit of the persistent kernels (mpc_ctx_set_wait_limit)
  unsigned long long wait_limit_ns = 2000000000ull;
  // the next persistent launch gets an unreachable barrier target
  // (mpc_ctx_inject_barrier_timeout); cleared when that launch is set up
  bool inject_barrier_timeout = false;
};

// Barrier settings for the next persistent launch on c (consumes a pending
// injected barrier timeout).
mpc::BarrierCfg mpc_barrier_cfg(mpc_ctx* c);

// Launch with programmatic stream serialization (see mpc_tdse.cu).
bool mpc_pdl_enabled();
template <typename... KArgs, typename... Args>
cudaError_t mpc_launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = mpc_pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// An NVTX range for the duration of a scope (a named region on a profiler's
// timeline; no cost without a profiler attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Event bracket for profiling one launch of kernel kind `kind`.
struct ProfScope {
  mpc_ctx* c;
  int kind;
  cudaEvent_t b = nullptr;
  ProfScope(mpc_ctx* c_, int k);
  ~ProfScope();
};

void mpc_batch_free(mpc_ctx* c);
void mpc_adjoint_free(mpc_ctx* c);
bool mpc_resident_setup(mpc_ctx* c);
void mpc_resident_free(mpc_ctx* c);
void mpc_batch_res_free(mpc_ctx* c);
void mpc_badj_free(mpc_ctx* c);
void mpc_badj_invalidate(mpc_ctx* c);  // a setting changed: backward needs a new forward
// Stage-GEMM variant for ncol active pulses: autotuned if the context's
// batched path has been tuned, else the default (batch.cu).
int mpc_batch_variant(mpc_ctx* c, int ncol);
int mpc_resident_run(mpc_ctx* c, double dt, int steps, int pop_index);
bool mpc_use_resident(mpc_ctx* c);  // the resident path applies (set-up done, not disabled)
bool mpc_resident_adjoint_ok(mpc_ctx* c);
int mpc_resident_forward_ex(mpc_ctx* c, const double2* x_in, double2* x_out, const double* Ftab,
                            double dt, int steps, double2* seg_x, double2* seg_y,
                            double* norm_hist, double2* ckpt, int ckpt_every, long long vpitch);
int mpc_resident_adjoint(mpc_ctx* c, const double* Ftab, double dt, int len,
                         const double2* seg_x, const double2* seg_y, const double* seg_n,
                         double2* lam, double* fbar, long long vpitch);
// The fused reverse pass (recompute of one segment concurrent with the sweep
// of the next, one persistent launch; resident.cu).
bool mpc_resident_fused_ok(mpc_ctx* c);
int mpc_resident_backward_fused(mpc_ctx* c, const double2* ckpts, int steps, int ckpt_every,
                                const double* Ftab, double dt, double2* const* segX,
                                double2* const* segY, double* const* segN, double2* lam,
                                double* fbar, long long vpitch);

// Launch helpers of the single-pulse path (mpc_tdse.cu), used by adjoint.cu.
int mpc_launch_stream(mpc_ctx* c, const double2* y);
int mpc_launch_combine_x(mpc_ctx* c, const double2* x, int stage, int step, double dt,
                         const double2* y, double2* out, bool final_weights, bool no_sum);
int mpc_launch_renorm_to(mpc_ctx* c, double2* x_out, const double2* xnew, int step, int pop_index,
                         double* pop_hist, double* norm_hist, int hist_base);
int mpc_fill_field_table(mpc_ctx* c, const double* F, int steps);

// The control perturbation dE(t) = sum_k u_k phi(t/g - k), g = T/(K-1), phi
// the Keys (a = -1/2) cubic kernel, zero outside [0, T]; w[0..3] receive the
// weights of samples k0 .. k0+3 (adjoint.cu).
double mpc_control_at(int K, const double* u, double T, double t, int* k0, double* w);
