// mpc_tdse.cu -- host side of libmpc_tdse.so: context set-up, the planner for
// the streaming right-hand side, launch sequences, and the C ABI declared in
// include/mpc_tdse.h.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpc_tdse.h"
#include "combine.cuh"
#include "ctx.h"
#include "plan.h"
#include "rhs_stream.cuh"
#include "rkf78.h"

using namespace mpc;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int mpc_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// error reporting for the other translation units of the library
int mpc_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encode(EncodeTiledFn* fn) {
  static EncodeTiledFn cached = nullptr;
  if (!cached) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p)
      return fail(MPC_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cached = reinterpret_cast<EncodeTiledFn>(p);
  }
  *fn = cached;
  return MPC_OK;
}

}  // namespace

// A 2-D FP64 tensor map for TMA loads of [outer][inner] elements, rows
// row_bytes apart, boxes of box_inner x box_outer; swizzle128: the 128-byte
// swizzle (box_inner * 8 must then be 128).
int mpc_encode_map_2d(CUtensorMap* m, const void* base, unsigned long long inner,
                      unsigned long long outer, unsigned long long row_bytes, unsigned box_inner,
                      unsigned box_outer, bool swizzle128) {
  EncodeTiledFn enc = nullptr;
  int rc;
  if ((rc = get_encode(&enc))) return rc;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MPC_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MPC_OK;
}

// A 3-D FP64 tensor map over a row-major [rows][cols] matrix (rows
// row_bytes apart) viewed as [cols / 16 groups][rows][16]: boxes of
// {16, box_rows, box_groups} with the 128-byte swizzle.  Columns past cols
// in the last group read the row padding (the caller keeps it zero).
int mpc_encode_map_grouped(CUtensorMap* m, const void* base, unsigned long long cols,
                           unsigned long long rows, unsigned long long row_bytes,
                           unsigned box_rows, unsigned box_groups) {
  EncodeTiledFn enc = nullptr;
  int rc;
  if ((rc = get_encode(&enc))) return rc;
  cuuint64_t dims[3] = {16, (cuuint64_t)rows, (cuuint64_t)((cols + 15) / 16)};
  cuuint64_t strides[2] = {(cuuint64_t)row_bytes, 128};
  cuuint32_t box[3] = {16, (cuuint32_t)box_rows, (cuuint32_t)box_groups};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MPC_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MPC_OK;
}

namespace {

template <class T>
int dalloc(mpc_ctx* c, T** p, size_t count) {
  void* q = nullptr;
  if (count == 0) count = 1;
  CK(cudaMalloc(&q, count * sizeof(T)));
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return MPC_OK;
}

void free_all(mpc_ctx* c) {
  for (void* p : c->allocs) cudaFree(p);
  c->allocs.clear();
}

// Fills the geometry, the tile->CTA split and the CP slot tables.
void plan_geometry(mpc_ctx* c, const int* n, int L_max, std::vector<int>& cta_slot0,
                   std::vector<int>& strip_slot0, int& nslots, long long& rp_total,
                   long long& d_total) {
  Geometry& g = c->g;
  g.nblk = L_max;
  g.nstate_blk = L_max + 1;
  g.state_off[0] = 0;
  for (int L = 0; L <= L_max; ++L) g.state_off[L + 1] = g.state_off[L] + n[L];
  g.ntot = g.state_off[L_max + 1];
  int tile = 0, strip = 0;
  rp_total = 0;
  d_total = 0;
  for (int L = 0; L < L_max; ++L) {
    BlockGeom& b = g.blk[L];
    b.nrow = n[L];
    b.ncol = n[L + 1];
    b.row_off = g.state_off[L];
    b.col_off = g.state_off[L + 1];
    b.pitch = (b.ncol + 31) / 32 * 32;
    b.nstrips = (b.ncol + kStripW - 1) / kStripW;
    b.nrtiles = (b.nrow + kTileR - 1) / kTileR;
    b.tile0 = tile;
    b.strip0 = strip;
    b.d_off = d_total;
    b.rp_off = rp_total;
    tile += b.nstrips * b.nrtiles;
    strip += b.nstrips;
    d_total += (long long)b.nrow * b.pitch;
    rp_total += (long long)b.nstrips * b.nrow;
  }
  g.ntiles = tile;
  g.nstrips = strip;
  const int G = std::min(c->num_sms, g.ntiles);
  c->stream_grid = G;
  cta_slot0.assign(G, 0);
  strip_slot0.assign(g.nstrips + 1, -1);
  int slot = 0;
  for (int cta = 0; cta < G; ++cta) {
    const int t0 = (int)((long long)g.ntiles * cta / G);
    const int t1 = (int)((long long)g.ntiles * (cta + 1) / G);
    cta_slot0[cta] = slot;
    int last = -1;
    for (int t = t0; t < t1; ++t) {
      int b, s, rt;
      decode_tile(g, t, b, s, rt);
      const int gs = g.blk[b].strip0 + s;
      if (gs != last) {
        if (strip_slot0[gs] < 0) strip_slot0[gs] = slot;
        ++slot;
        last = gs;
      }
    }
  }
  strip_slot0[g.nstrips] = slot;
  nslots = slot;
  c->combine_grid = (g.ntot * kCombineLanes + kCombineThreads - 1) / kCombineThreads;
}

int ensure_hist(mpc_ctx* c, int steps) {
  if (steps + 1 <= c->hist_cap) return MPC_OK;
  int cap = std::max(steps + 1, 2 * c->hist_cap);
  // history buffers are replaced, not tracked in allocs
  if (c->d_Ftab) cudaFree(c->d_Ftab);
  if (c->d_pop) cudaFree(c->d_pop);
  if (c->d_nrm) cudaFree(c->d_nrm);
  c->d_Ftab = c->d_pop = c->d_nrm = nullptr;
  c->hist_cap = 0;
  CK(cudaMalloc(&c->d_Ftab, sizeof(double) * cap));
  CK(cudaMalloc(&c->d_pop, sizeof(double) * cap));
  CK(cudaMalloc(&c->d_nrm, sizeof(double) * cap));
  c->hist_cap = cap;
  return MPC_OK;
}

// --- profiling ---------------------------------------------------------------
cudaEvent_t pool_get(mpc_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

}  // namespace

ProfScope::ProfScope(mpc_ctx* c_, int k) : c(c_), kind(k) {
  ++c->launches;
  if (c->profiling) {
    b = pool_get(c);
    cudaEventRecord(b, c->stream);
  }
}

ProfScope::~ProfScope() {
  if (b) {
    cudaEvent_t e = pool_get(c);
    cudaEventRecord(e, c->stream);
    c->ev[kind].emplace_back(b, e);
  }
}

namespace {

// --- launch sequences -------------------------------------------------------

// MPC_NO_PDL=1 in the environment turns programmatic dependent launch off
// (plain stream order), a debugging aid.
}  // namespace

bool mpc_pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("MPC_NO_PDL");
    return !(e && e[0] == '1');
  }();
  return on;
}

namespace {

}  // namespace

int mpc_launch_stream(mpc_ctx* c, const double2* y) {
  c->sargs.y = y;
  ProfScope ps(c, MPC_KERNEL_RHS_STREAM);
  CK(mpc_launch_pdl(k_rhs_stream, dim3(c->stream_grid), dim3(kStreamThreads), kStreamSmem,
                    c->stream, c->sargs, c->tmaps));
  return MPC_OK;
}

// stage s: k_s = f(y_s); out = x + sum coef*k.  coefs: the row of the next
// combination (a_{s+1,*}, or b for s == 12), multiplied by dt.
int mpc_launch_combine_x(mpc_ctx* c, const double2* x, int stage, int step, double dt,
                         const double2* y, double2* out, bool final_weights, bool no_sum) {
  CombineArgs a{};
  a.x = x;
  a.y = y;
  a.k = c->d_k;
  a.out = out;
  a.eps = c->d_eps;
  a.RP = c->d_RP;
  a.CP = c->d_CP;
  a.strip_slot0 = c->d_strip_slot0;
  a.Ftab = c->d_Ftab;
  a.norm_part = c->d_norm_part;
  a.step = step;
  a.stage = stage;
  a.gauge = (c->gauge == 'l') ? 0 : 1;
  a.ncoef = 0;
  if (!no_sum) {
    const double* row = final_weights ? rkf78::B8 : rkf78::A[stage + 1];
    for (int j = 0; j <= stage; ++j) {
      if (row[j] == 0.0) continue;
      a.coef_j[a.ncoef] = j;
      a.coef[a.ncoef] = dt * row[j];
      ++a.ncoef;
    }
  }
  a.g = c->g;
  ProfScope ps(c, MPC_KERNEL_COMBINE);
  CK(mpc_launch_pdl(k_stage_combine, dim3(c->combine_grid), dim3(kCombineThreads), 0, c->stream, a));
  return MPC_OK;
}

int mpc_launch_renorm_to(mpc_ctx* c, double2* x_out, const double2* xnew, int step, int pop_index,
                         double* pop_hist, double* norm_hist, int hist_base) {
  RenormArgs r{};
  r.x = x_out;
  r.xnew = xnew;
  r.norm_part = c->d_norm_part;
  r.nparts = c->combine_grid;
  r.ntot = c->g.ntot;
  r.pop_index = pop_index;
  r.step = step;
  r.hist_base = hist_base;
  r.pop_hist = pop_hist;
  r.norm_hist = norm_hist;
  r.status = c->d_status;
  ProfScope ps(c, MPC_KERNEL_RENORM);
  CK(mpc_launch_pdl(k_renorm, dim3(c->combine_grid), dim3(kCombineThreads), 0, c->stream, r));
  return MPC_OK;
}

namespace {

int launch_stream(mpc_ctx* c, const double2* y) { return mpc_launch_stream(c, y); }

int launch_combine(mpc_ctx* c, int stage, int step, double dt, const double2* y, double2* out,
                   bool final_weights, bool no_sum) {
  return mpc_launch_combine_x(c, c->d_x, stage, step, dt, y, out, final_weights, no_sum);
}

int launch_renorm(mpc_ctx* c, int step, int pop_index) {
  RenormArgs r{};
  r.x = c->d_x;
  r.xnew = c->d_y;
  r.norm_part = c->d_norm_part;
  r.nparts = c->combine_grid;
  r.ntot = c->g.ntot;
  r.pop_index = pop_index;
  r.step = step;
  r.pop_hist = c->d_pop;
  r.norm_hist = c->d_nrm;
  r.status = c->d_status;
  ProfScope ps(c, MPC_KERNEL_RENORM);
  CK(mpc_launch_pdl(k_renorm, dim3(c->combine_grid), dim3(kCombineThreads), 0, c->stream, r));
  return MPC_OK;
}

// One RKF78 step of the state in d_x with field Ftab[step]; result in d_y
// (not renormalised).
int rk78_step_dev(mpc_ctx* c, int step, double dt) {
  int rc;
  for (int s = 0; s < kNumStages; ++s) {
    const double2* ys = (s == 0) ? c->d_x : c->d_y;
    if ((rc = launch_stream(c, ys))) return rc;
    if ((rc = launch_combine(c, s, step, dt, ys, c->d_y, s == kNumStages - 1, false))) return rc;
  }
  return MPC_OK;
}

// One fixed step of the state in d_x with field Ftab[step] as the 12 Horner
// products of the RKF78 stability polynomial (the same step: with the field
// frozen the system is linear and autonomous, and R(hM)x is what the 13
// stages form), each a dipole stream and a combine pass: one stream pass per
// step fewer than the stage form.  Result in d_y (not renormalised).
int horner_step_dev(mpc_ctx* c, int step, double dt) {
  int rc;
  for (int p = 0; p < 12; ++p) {
    // d_x -> d_v -> d_y -> d_v -> ... -> d_y (p = 11)
    const double2* in = (p == 0) ? c->d_x : ((p - 1) % 2 == 1 ? c->d_y : c->d_v);
    double2* out = (p % 2 == 1) ? c->d_y : c->d_v;
    if ((rc = launch_stream(c, in))) return rc;
    CombineArgs a{};
    a.x = c->d_x;
    a.y = in;
    a.k = c->d_k;
    a.out = out;
    a.eps = c->d_eps;
    a.RP = c->d_RP;
    a.CP = c->d_CP;
    a.strip_slot0 = c->d_strip_slot0;
    a.Ftab = c->d_Ftab;
    a.norm_part = c->d_norm_part;
    a.step = step;
    a.stage = (p == 11) ? kNumStages - 1 : 0;   // the last product forms the norm partials
    a.gauge = (c->gauge == 'l') ? 0 : 1;
    a.horner = 1;
    a.vscale = (p == 0) ? rkf78::G[12] : 1.0;
    a.hg = rkf78::G[11 - p];
    a.hstep = dt;
    a.g = c->g;
    ProfScope ps(c, MPC_KERNEL_COMBINE);
    CK(mpc_launch_pdl(k_stage_combine, dim3(c->combine_grid), dim3(kCombineThreads), 0,
                      c->stream, a));
  }
  return MPC_OK;
}

__global__ void k_pop_init(const double2* x, int pop_index, double* pop) {
  const double2 v = x[pop_index];
  pop[0] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
}

int check_status(mpc_ctx* c) {
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof st, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st) {
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
    return fail(MPC_ERR_DEVICE, "kernel status 0x%x (%s%s%s)", st,
                (st & ST_WAIT_TIMEOUT) ? "wait timeout " : "",
                (st & ST_NONFINITE) ? "non-finite norm " : "",
                (st & ST_BAD_LAUNCH) ? "bad launch " : "");
  }
  return MPC_OK;
}

double host_field(const mpc_pulse& p, double t) {
  const double Eo = p.Eo, w = p.w, cepd = p.cepd, a = p.a, b = p.b;
  switch (p.kind) {
    case MPC_FIELD_SINE_EE:
    case MPC_FIELD_SINE_AA: {
      const double sinWt = std::sin(a * t);
      return (double)(t >= 0.0 && t <= M_PI / a) * Eo * sinWt * sinWt * std::sin(w * t + cepd);
    }
    case MPC_FIELD_SINE_AE: {
      const double Wt = a * t;
      const double sinWt = std::sin(Wt);
      const double wtc = w * t + cepd;
      return (double)(t >= 0.0 && t <= M_PI / a) * Eo *
             (w * sinWt * sinWt * std::cos(wtc) + a * std::sin(2 * Wt) * std::sin(wtc));
    }
    case MPC_FIELD_SINE_EA: {
      const double WpP = w + 2.0 * a, WpN = w - 2.0 * a;
      return (double)(t >= 0.0 && t <= M_PI / a) * 0.5 * Eo *
             (((1.0 - std::cos(w * t + cepd)) / w) -
              0.5 * ((1.0 - std::cos(WpP * t)) / WpP + (1.0 - std::cos(WpN * t)) / WpN));
    }
    case MPC_FIELD_GAUSS: {
      const double td = t - 0.5 * b;
      return (double)(t >= 0.0 && t <= b) * Eo * std::exp(-td * td / (a * a)) *
             std::sin(w * t + cepd);
    }
  }
  return 0.0;
}

int fill_fields(mpc_ctx* c, const mpc_pulse* p, double t0, double dt, int steps,
                std::vector<double>& F) {
  F.resize(steps > 0 ? steps : 1);
  double t = t0;
  double fmax = 0.0;
  for (int st = 0; st < steps; ++st) {
    F[st] = host_field(*p, t + dt);
    fmax = std::max(fmax, std::fabs(F[st]));
    t += dt;
  }
  if (dt * c->eps_max > kRk78ImagStability)
    return fail(MPC_ERR_UNSTABLE,
                "dt*max|E| = %.4g exceeds the RKF78 imaginary-axis stability bound %.4g",
                dt * c->eps_max, kRk78ImagStability);
  CK(cudaMemcpyAsync(c->d_Ftab, F.data(), sizeof(double) * steps, cudaMemcpyHostToDevice,
                     c->stream));
  return MPC_OK;
}

bool use_resident(mpc_ctx* c) {
  if (c->path == MPC_PATH_STREAMING) return false;
  return mpc_resident_setup(c);
}

int run_steps(mpc_ctx* c, double dt, int steps, int pop_index) {
  int rc;
  if (steps > 0 && use_resident(c)) return mpc_resident_run(c, dt, steps, pop_index);
  ++c->launches;
  k_pop_init<<<1, 1, 0, c->stream>>>(c->d_x, pop_index, c->d_pop);
  CK(cudaGetLastError());
  for (int st = 0; st < steps; ++st) {
    if ((rc = c->stage_form ? rk78_step_dev(c, st, dt) : horner_step_dev(c, st, dt))) return rc;
    if ((rc = launch_renorm(c, st, pop_index))) return rc;
  }
  return MPC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
int mpc_fill_field_table(mpc_ctx* c, const double* F, int steps) {
  int rc;
  if ((rc = ensure_hist(c, steps))) return rc;
  CK(cudaMemcpyAsync(c->d_Ftab, F, sizeof(double) * steps, cudaMemcpyHostToDevice, c->stream));
  return MPC_OK;
}

bool mpc_use_resident(mpc_ctx* c) { return use_resident(c); }

mpc::BarrierCfg mpc_barrier_cfg(mpc_ctx* c) {
  mpc::BarrierCfg b{c->wait_limit_ns, 0ull};
  if (c->inject_barrier_timeout) {
    b.skew = 1;  // one arrival more than the grid can make: no barrier completes
    c->inject_barrier_timeout = false;
  }
  return b;
}

extern "C" {

int mpc_version(void) { return 100; }

int mpc_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return MPC_ERR_ARG;
  std::snprintf(buf, len, "%s", g_err.c_str());
  return MPC_OK;
}

int mpc_to_au(double Io_Wcm2, double w_eV, double* Io_au, double* w_au) {
  if (!Io_au || !w_au) return fail(MPC_ERR_ARG, "null output");
  *Io_au = Io_Wcm2 * ((1. / 3.509338) * 1.e-16);
  *w_au = w_eV * (1. / 27.211396181);
  return MPC_OK;
}

double mpc_period(double w_au, int cycles) { return cycles * 2.0 * M_PI / w_au; }

int mpc_pulse_setup(int shape, char gauge, double Io, double w, double cepd, int cycles,
                    double tau, mpc_pulse* out) {
  if (!out) return fail(MPC_ERR_ARG, "null output");
  if (gauge != 'l' && gauge != 'v') return fail(MPC_ERR_ARG, "gauge must be 'l' or 'v'");
  if (cycles <= 0 || !(w > 0.0) || !(Io >= 0.0)) return fail(MPC_ERR_ARG, "bad pulse parameters");
  const double Eo = (gauge == 'v') ? std::sqrt(Io) / w : std::sqrt(Io);
  out->Eo = Eo;
  out->w = w;
  if (shape == 0) {
    out->kind = (gauge == 'v') ? MPC_FIELD_SINE_AA : MPC_FIELD_SINE_EE;
    out->cepd = (gauge == 'v') ? cepd * (2.0 * M_PI / w) : cepd * (2 * M_PI / w);
    out->a = w / (2.0 * cycles);
    out->b = 0.0;
  } else if (shape == 1) {
    const double width = 0.58870501125773734549;
    const double To = 2 * M_PI / w;
    const int cycles_fwhm = 2 + int(cycles / 10);
    out->kind = MPC_FIELD_GAUSS;
    out->cepd = cepd;
    out->a = 0.5 * To * cycles_fwhm / width;
    out->b = tau;
  } else {
    return fail(MPC_ERR_ARG, "shape must be 0 (sine) or 1 (gaussian)");
  }
  return MPC_OK;
}

double mpc_field(const mpc_pulse* p, double t) { return p ? host_field(*p, t) : 0.0; }

int mpc_ctx_create(int L_max, const int* state_sz, const double* eig, const double* dip,
                   char gauge, int device, mpc_ctx** out) {
  NvtxRange nvtx_("mpc_ctx_create (upload)");
  if (!out) return fail(MPC_ERR_ARG, "null output");
  *out = nullptr;
  if (L_max < 1 || L_max >= kMaxBlocks)
    return fail(MPC_ERR_ARG, "L_max must be in [1, %d]", kMaxBlocks - 1);
  if (!state_sz || !eig || !dip) return fail(MPC_ERR_ARG, "null input array");
  if (gauge != 'l' && gauge != 'v') return fail(MPC_ERR_ARG, "gauge must be 'l' or 'v'");
  long long tot = 0;
  for (int L = 0; L <= L_max; ++L) {
    if (state_sz[L] <= 0) return fail(MPC_ERR_ARG, "state_sz[%d] = %d", L, state_sz[L]);
    tot += state_sz[L];
  }
  if (tot > (1LL << 28)) return fail(MPC_ERR_ARG, "too many states");
  for (long long i = 0; i < tot; ++i)
    if (!std::isfinite(eig[i])) return fail(MPC_ERR_ARG, "non-finite energy at %lld", i);

  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MPC_ERR_ARG, "no CUDA device %d", device);
  CK(cudaSetDevice(device));

  mpc_ctx* c = new mpc_ctx();
  c->device = device;
  if (const char* v = std::getenv("MPC_BATCH_VARIANT")) c->forced_variant = std::atoi(v);
  c->no_persist = std::getenv("MPC_NO_PERSIST") != nullptr;
  c->force_persist = std::getenv("MPC_FORCE_PERSIST") != nullptr;
  if (const char* ft = std::getenv("MPC_FORCE_TMA")) c->force_tma = std::max(0, std::atoi(ft));
  c->no_tma = std::getenv("MPC_NO_TMA") != nullptr;
  c->stage_form = std::getenv("MPC_STAGE_FORM") != nullptr;
  c->gauge = gauge;
  c->n.assign(state_sz, state_sz + L_max + 1);
  CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
  for (long long i = 0; i < tot; ++i) c->eps_max = std::max(c->eps_max, std::fabs(eig[i]));

  std::vector<int> cta_slot0, strip_slot0;
  int nslots = 0;
  long long rp_total = 0, d_total = 0;
  plan_geometry(c, state_sz, L_max, cta_slot0, strip_slot0, nslots, rp_total, d_total);
  const Geometry& g = c->g;

  int rc = MPC_OK;
  auto bail = [&](int code) {
    free_all(c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MPC_ERR_CUDA, "cudaStreamCreate failed"));
  if ((rc = dalloc(c, &c->d_eps, g.ntot)) || (rc = dalloc(c, &c->d_D, d_total)) ||
      (rc = dalloc(c, &c->d_x, g.ntot + kVecPad)) || (rc = dalloc(c, &c->d_y, g.ntot + kVecPad)) ||
      (rc = dalloc(c, &c->d_v, g.ntot + kVecPad)) ||
      (rc = dalloc(c, &c->d_k, (size_t)kNumStages * g.ntot)) ||
      (rc = dalloc(c, &c->d_RP, rp_total)) ||
      (rc = dalloc(c, &c->d_CP, (size_t)nslots * kStripW)) ||
      (rc = dalloc(c, &c->d_cta_slot0, cta_slot0.size())) ||
      (rc = dalloc(c, &c->d_strip_slot0, strip_slot0.size())) ||
      (rc = dalloc(c, &c->d_norm_part, c->combine_grid)) || (rc = dalloc(c, &c->d_status, 1)))
    return bail(rc);

  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  };
  if (up(c->d_eps, eig, sizeof(double) * g.ntot) != cudaSuccess ||
      up(c->d_cta_slot0, cta_slot0.data(), sizeof(int) * cta_slot0.size()) != cudaSuccess ||
      up(c->d_strip_slot0, strip_slot0.data(), sizeof(int) * strip_slot0.size()) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(c->d_x, 0, sizeof(double2) * (g.ntot + kVecPad)) != cudaSuccess ||
      cudaMemset(c->d_y, 0, sizeof(double2) * (g.ntot + kVecPad)) != cudaSuccess ||
      cudaMemset(c->d_v, 0, sizeof(double2) * (g.ntot + kVecPad)) != cudaSuccess ||
      cudaMemset(c->d_D, 0, sizeof(double) * d_total) != cudaSuccess)
    return bail(fail(MPC_ERR_CUDA, "upload failed"));
  const double* src = dip;
  for (int L = 0; L < L_max; ++L) {
    const BlockGeom& b = g.blk[L];
    for (long long i = 0; i < (long long)b.nrow * b.ncol; ++i)
      if (!std::isfinite(src[i]))
        return bail(fail(MPC_ERR_ARG, "non-finite dipole element in block %d", L));
    if (cudaMemcpy2D(c->d_D + b.d_off, sizeof(double) * b.pitch, src, sizeof(double) * b.ncol,
                     sizeof(double) * b.ncol, b.nrow, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(MPC_ERR_CUDA, "dipole upload failed"));
    src += (long long)b.nrow * b.ncol;
  }

  EncodeTiledFn enc = nullptr;
  if ((rc = get_encode(&enc))) return bail(rc);
  for (int L = 0; L < L_max; ++L) {
    const BlockGeom& b = g.blk[L];
    cuuint64_t dims[2] = {(cuuint64_t)b.ncol, (cuuint64_t)b.nrow};
    cuuint64_t strides[1] = {(cuuint64_t)b.pitch * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)kStripW, (cuuint32_t)kTileR};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&c->tmaps.m[L], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, c->d_D + b.d_off, dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return bail(fail(MPC_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for block %d", (int)r, L));
  }
  if (cudaFuncSetAttribute(k_rhs_stream, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kStreamSmem) != cudaSuccess)
    return bail(fail(MPC_ERR_CUDA, "cannot reserve %d B of shared memory", kStreamSmem));

  c->sargs.RP = c->d_RP;
  c->sargs.CP = c->d_CP;
  c->sargs.cta_slot0 = c->d_cta_slot0;
  c->sargs.status = c->d_status;
  c->sargs.g = c->g;
  {
    // dipole bytes kept in L2 across the passes of a step (MPC_L2_KEEP_MB
    // overrides): the rest streams through with an evict-first hint.  40 MB
    // of the 126 MB L2: on the 547 MB He CI couplings 0 / 24 / 32 / 40 / 48 /
    // 64 / 128 MB gave 856-868 / 869 / 872-893 / 876 / 876 / 883 / 863
    // pulse-steps/s (two boxes)
    double keep_mb = 40.0;
    if (const char* e = std::getenv("MPC_L2_KEEP_MB")) keep_mb = std::atof(e);
    const double dbytes = 8.0 * (double)d_total;
    c->sargs.keep_frac =
        dbytes > 0.0 ? (float)std::min(1.0, std::max(0.0, keep_mb * 1048576.0 / dbytes)) : 0.0f;
  }
  if ((rc = ensure_hist(c, 1024))) return bail(rc);
  *out = c;
  return MPC_OK;
}

int mpc_ctx_destroy(mpc_ctx* c) {
  if (!c) return MPC_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  mpc_batch_free(c);
  mpc_adjoint_free(c);
  mpc_resident_free(c);
  mpc_batch_res_free(c);
  mpc_badj_free(c);
  free_all(c);
  for (auto& v : c->ev)
    for (auto& pr : v) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->d_Ftab) cudaFree(c->d_Ftab);
  if (c->d_pop) cudaFree(c->d_pop);
  if (c->d_nrm) cudaFree(c->d_nrm);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MPC_OK;
}

int mpc_ctx_size(const mpc_ctx* c) { return c ? c->g.ntot : MPC_ERR_ARG; }

int mpc_ctx_set_wait_limit(mpc_ctx* c, double seconds) {
  if (!c || !(seconds >= 1e-6) || !(seconds <= 60.0))
    return fail(MPC_ERR_ARG, "wait limit must be in [1e-6, 60] s");
  c->wait_limit_ns = (unsigned long long)(seconds * 1e9);
  return MPC_OK;
}

int mpc_ctx_inject_barrier_timeout(mpc_ctx* c) {
  if (!c) return fail(MPC_ERR_ARG, "null argument");
  c->inject_barrier_timeout = true;
  return MPC_OK;
}

int mpc_ctx_set_path(mpc_ctx* c, int path) {
  if (!c || path < 0 || path > 2) return fail(MPC_ERR_ARG, "bad path");
  CK(cudaSetDevice(c->device));
  if (path == MPC_PATH_RESIDENT && !mpc_resident_setup(c))
    return fail(MPC_ERR_ARG, "the system's coupling rows do not fit in shared memory");
  c->path = path;
  return MPC_OK;
}

int mpc_ctx_get_path(mpc_ctx* c) {
  if (!c) return MPC_ERR_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return MPC_ERR_CUDA;
  return use_resident(c) ? MPC_PATH_RESIDENT : MPC_PATH_STREAMING;
}

int mpc_ctx_stream(const mpc_ctx* c, void** stream) {
  if (!c || !stream) return fail(MPC_ERR_ARG, "null argument");
  *stream = c->stream;
  return MPC_OK;
}

int mpc_rhs(mpc_ctx* c, double F, const double* x, double* dxdt) {
  if (!c || !x || !dxdt) return fail(MPC_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const size_t bytes = sizeof(double2) * c->g.ntot;
  CK(cudaMemcpyAsync(c->d_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_Ftab, &F, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc;
  if ((rc = launch_stream(c, c->d_x))) return rc;
  if ((rc = launch_combine(c, 0, 0, 0.0, c->d_x, c->d_y, false, true))) return rc;
  CK(cudaMemcpyAsync(dxdt, c->d_k, bytes, cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

int mpc_rk78_step(mpc_ctx* c, double F, double dt, double* x) {
  if (!c || !x) return fail(MPC_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const size_t bytes = sizeof(double2) * c->g.ntot;
  CK(cudaMemcpyAsync(c->d_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_Ftab, &F, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc;
  if ((rc = rk78_step_dev(c, 0, dt))) return rc;
  CK(cudaMemcpyAsync(x, c->d_y, bytes, cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

int mpc_state_set(mpc_ctx* c, const double* ct) {
  if (!c || !ct) return fail(MPC_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->d_x, ct, sizeof(double2) * c->g.ntot, cudaMemcpyHostToDevice,
                     c->stream));
  return MPC_OK;
}

int mpc_state_get(mpc_ctx* c, double* ct) {
  if (!c || !ct) return fail(MPC_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(ct, c->d_x, sizeof(double2) * c->g.ntot, cudaMemcpyDeviceToHost,
                     c->stream));
  return check_status(c);
}

int mpc_advance(mpc_ctx* c, const mpc_pulse* p, double t0, double dt, int steps,
                int pop_index) {
  NvtxRange nvtx_("mpc_advance");
  if (!c || !p) return fail(MPC_ERR_ARG, "null argument");
  if (steps < 0) return fail(MPC_ERR_ARG, "steps < 0");
  if (pop_index < 0 || pop_index >= c->g.ntot) return fail(MPC_ERR_ARG, "pop_index out of range");
  if (!(dt > 0.0)) return fail(MPC_ERR_ARG, "dt must be > 0");
  CK(cudaSetDevice(c->device));
  int rc;
  if ((rc = ensure_hist(c, steps))) return rc;
  std::vector<double> F;
  if ((rc = fill_fields(c, p, t0, dt, steps, F))) return rc;
  return run_steps(c, dt, steps, pop_index);
}

}  // extern "C"

namespace {

// Enqueues the copies of the last run's histories (no wait).
int history_copy(mpc_ctx* c, int steps, double* pop_out, double* field_out, double* norm_out) {
  if (steps < 0 || steps + 1 > c->hist_cap) return fail(MPC_ERR_ARG, "steps out of range");
  CK(cudaSetDevice(c->device));
  if (pop_out)
    CK(cudaMemcpyAsync(pop_out, c->d_pop, sizeof(double) * (steps + 1), cudaMemcpyDeviceToHost,
                       c->stream));
  if (field_out && steps > 0)
    CK(cudaMemcpyAsync(field_out, c->d_Ftab, sizeof(double) * steps, cudaMemcpyDeviceToHost,
                       c->stream));
  if (norm_out && steps > 0)
    CK(cudaMemcpyAsync(norm_out, c->d_nrm, sizeof(double) * steps, cudaMemcpyDeviceToHost,
                       c->stream));
  return MPC_OK;
}

}  // namespace

extern "C" {

int mpc_history_get(mpc_ctx* c, int steps, double* pop_out, double* field_out,
                    double* norm_out) {
  if (!c) return fail(MPC_ERR_ARG, "null argument");
  int rc;
  if ((rc = history_copy(c, steps, pop_out, field_out, norm_out))) return rc;
  return check_status(c);
}

int mpc_propagate(mpc_ctx* c, const mpc_pulse* p, double t0, double dt, int steps,
                  int pop_index, double* ct, double* pop_out, double* field_out,
                  double* norm_out) {
  NvtxRange nvtx_("mpc_propagate");
  if (!c || !p || !ct) return fail(MPC_ERR_ARG, "null argument");
  int rc;
  if ((rc = mpc_state_set(c, ct))) return rc;
  if ((rc = mpc_advance(c, p, t0, dt, steps, pop_index))) return rc;
  // the histories and the state come back behind one wait (mpc_state_get's)
  if ((rc = history_copy(c, steps, pop_out, field_out, norm_out))) return rc;
  return mpc_state_get(c, ct);
}

int mpc_profile_enable(mpc_ctx* c, int on) {
  if (!c) return fail(MPC_ERR_ARG, "null argument");
  c->profiling = on != 0;
  return MPC_OK;
}

int mpc_profile_read(mpc_ctx* c, int kind, double* total_ms, long long* launches) {
  if (!c || kind < 0 || kind > 5 || !total_ms || !launches)
    return fail(MPC_ERR_ARG, "bad argument");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  double tot = 0.0;
  for (auto& pr : c->ev[kind]) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
    tot += ms;
    c->ev_pool.push_back(pr.first);
    c->ev_pool.push_back(pr.second);
  }
  *total_ms = tot;
  *launches = (long long)c->ev[kind].size();
  c->ev[kind].clear();
  return MPC_OK;
}

long long mpc_launch_count(const mpc_ctx* c) { return c ? c->launches : 0; }

int mpc_sync(mpc_ctx* c) {
  if (!c) return fail(MPC_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  return check_status(c);
}

}  // extern "C"
