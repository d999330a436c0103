// batch_stage.cuh -- the stage GEMM of the batched propagation, shared by the
// batched adaptive path (batch.cu) and the batched adjoint (batch_adjoint.cu).
//
// The state of B pulses is one matrix [n][ldc] (row = basis state, complex
// column = pulse), so one right-hand side for all pulses is a real GEMM of
// the block-tridiagonal coupling (the dipole blocks) with the [n x 2B] stage
// matrix on the FP64 tensor cores (mma.sync m16n8k8 .f64), with an epilogue
// fused into its store:
//   MODE 0 (forward): k_s = M(F) y_s, the next stage input (or, after the last
//     stage, x_new, the embedded error and per-pulse norm partials);
//   MODE 1 (adjoint): ybar_s = -M(F) kbar_s, the partial of dJ/dF =
//     -Re<M1 kbar_s, y_s>, and the next adjoint stage input kbar_{s-1} (or,
//     after stage 0, lambda_n = zbar + sum_s ybar_s).
// Each translation unit that includes this header owns its own constant
// tables and kernel instantiations and sets them up with stage_setup().
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

#include "ctx.h"
#include "dev_util.cuh"
#include "plan.h"
#include "rkf78.h"

namespace {

using namespace mpc;

constexpr int BM = 64, BK = 32, BTHREADS = 256;
constexpr int LDA_P = BM + 4;   // A stored [k][m] (transposed block), pitch in doubles
constexpr int LDA_Q = BK + 4;   // A stored [m][k]
constexpr int A_STAGE = (BK * LDA_P > BM * LDA_Q) ? BK * LDA_P : BM * LDA_Q;
constexpr int kColAlign = 32;   // pulse columns are allocated in multiples of this

// Column-tile shapes (real columns = 2 x pulses).  8 warps in a WGM x WGN
// grid, each owning WMT x WNT tiles of m16n8; BM = WGM*WMT*16 = 64 rows.
// The narrowest tile covering the active pulses is used, so that a batch
// whose pulses have mostly retired does not pay for empty columns.
template <int BN_> struct Tile;
// Every variant sums the coupling in the same order (see the kernel), so
// the autotuner's choice never changes the numbers.
template <> struct Tile<64> { static constexpr int WGM = 2, WGN = 4, WMT = 2, WNT = 2; };
template <> struct Tile<32> { static constexpr int WGM = 2, WGN = 4, WMT = 2, WNT = 1; };
template <> struct Tile<16> { static constexpr int WGM = 4, WGN = 2, WMT = 1, WNT = 1; };
template <int BN_> constexpr int b_stage() { return BK * (BN_ + 4); }
// NST_ cp.async stages: 3 for the wide tile (two CTAs per SM), 6 for the
// narrow ones (small grids: more loads in flight per CTA instead)
template <int BN_, int NST_> constexpr int batch_smem() {
  return NST_ * (A_STAGE + b_stage<BN_>()) * 8;
}
// Unsplit variants with narrow tiles pair each P chunk with the Q chunk of
// the same index in one ring slot (see stage_tile): NST_ chunk slots become
// 2 (NST_ = 3) or 3 (NST_ = 6) slots of two chunks.
template <int BN_, int SPLIT_> constexpr bool paired() { return SPLIT_ == 0 && BN_ <= 32; }
template <int NST_> constexpr int pair_slots() { return NST_ >= 6 ? 3 : 2; }
template <int BN_, int NST_, int SPLIT_> constexpr int stage_smem() {
  return paired<BN_, SPLIT_>() ? pair_slots<NST_>() * 2 * (A_STAGE + b_stage<BN_>()) * 8
                               : batch_smem<BN_, NST_>();
}

__constant__ double c_A[13][13];
__constant__ double c_B8[13];
__constant__ double c_E[13];   // b8 - b7
__constant__ double c_C[13];

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = smem_u32(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(sz)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// D (16x8, f64) += A (16x8) * B (8x8); fragments as in the PTX ISA for
// m16n8k8 .f64: a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]},
// b = {B[t][g], B[t+4][g]}, c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]}
// with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void dmma16x8x8(double* c, const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

struct StageArgs {
  const double* D;
  const double* eps;
  const double2* X;      // x, [n][ldc]
  const double2* Yin;    // y_s (X for s = 0)
  double2* K;            // k[13][n][ldc]
  double2* Yout;         // y_{s+1}, or x_new for s = 12
  const double* Fs;      // stage fields: Fs[s * fs_stride + q]
  const double* h;       // [ldc] attempt step
  unsigned long long* err;  // [ldc] bits of the max error ratio
  double* normpart;      // [nrowtiles][ldc]
  double rtol, atol;
  int stage;
  int gauge;             // 0 length, 1 velocity
  int ncol;              // active pulse columns
  int ldc;               // allocated pulse columns (row pitch of X, Y, K in complex)
  int nrowtiles;
  int want_k_only;       // 1: stop after storing k_s (single RHS evaluations)
  int fs_stride;         // ldc (a field per stage) or 0 (one field per step)
  // MODE 2 (a frozen-field step as its stability polynomial, by Horner's
  // rule): Yout = h M(F) (vscale Yin) + hg X; the last product (hlast) also
  // forms the per-pulse norm partials of x_new = Yout
  double hg;
  double vscale;
  int hlast;
  // the first product takes the previous step's unnormalised x_new (Yin) and
  // its norm per pulse (nrm), forms x = x_new / ||x_new|| on the fly and
  // stores it (Xw) for the step's later products
  const double* nrm;
  double2* Xw;
  // adjoint stages (MODE 1): Yin = kbar_s, K = ybar slabs, Yout = kbar_{s-1}
  // (or lambda_n after stage 0)
  const double2* Ys;     // the forward stage input y_s
  const double2* Zbar;   // zbar of the step
  double* fpart;         // [13][nrowtiles][ldc] partials of dJ/dF
  // split variants: the P and Q halves of a tile run in two CTAs; the second
  // to finish adds the first one's partial (workspace) and runs the epilogue
  double* ws;            // [row tiles x column tiles][2][BM x BN]
  int* cnt;              // [row tiles x column tiles] arrivals (left at zero)
  Geometry g;
};


// One BK-deep chunk of the tile product from shared memory into acc: the A
// operand is D_{L-1}^T (IS_P, stored k-major) or D_L (stored m-major).  The
// velocity gauge's minus sign on the D_L term is applied once to its
// accumulated sum: negation commutes exactly with every rounding, so
// sign * sum(D y) has the bits of sum((sign D) y), without a multiply between
// each fragment load and its DMMA.
// Only the chunk's first nks 8-deep k-steps hold coupling (the rest of the
// last chunk of a block is zero fill) and only this warp's first mt_lim
// 16-row m-tiles hold rows of the block: the rest would add exact zeros or
// rows that are never stored, so they are skipped (warp-uniform branches).
template <int BN, bool IS_P, bool FULL>
__device__ __forceinline__ void chunk_mma_body(const double* As, const double* Bs, int wm, int wn,
                                          int gq, int tq, int nks, int mt_lim,
                                          double (&acc)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  constexpr int WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
  constexpr int LDB = BN + 4;
#pragma unroll
  for (int ks = 0; ks < BK / 8; ++ks) {
    if (!FULL && ks >= nks) break;
    double af[WMT][4], bf[WNT][2];
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
      const int m = wm * (WMT * 16) + mt * 16 + gq;
      const int k = ks * 8 + tq;
      if constexpr (IS_P) {
        af[mt][0] = As[k * LDA_P + m];
        af[mt][1] = As[k * LDA_P + m + 8];
        af[mt][2] = As[(k + 4) * LDA_P + m];
        af[mt][3] = As[(k + 4) * LDA_P + m + 8];
      } else {
        af[mt][0] = As[m * LDA_Q + k];
        af[mt][1] = As[(m + 8) * LDA_Q + k];
        af[mt][2] = As[m * LDA_Q + k + 4];
        af[mt][3] = As[(m + 8) * LDA_Q + k + 4];
      }
    }
#pragma unroll
    for (int nt = 0; nt < WNT; ++nt) {
      const int n = wn * (WNT * 8) + nt * 8 + gq;
      const int k = ks * 8 + tq;
      bf[nt][0] = Bs[k * LDB + n];
      bf[nt][1] = Bs[(k + 4) * LDB + n];
    }
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
#pragma unroll
      for (int nt = 0; nt < WNT; ++nt) dmma16x8x8(acc[mt][nt], af[mt], bf[nt]);
    }
  }
}

// A whole chunk on a warp whose m-tiles all hold rows (the usual case) runs
// without the skip branches, so its fragment loads schedule ahead of the DMMAs.
template <int BN, bool IS_P>
__device__ __forceinline__ void chunk_mma(const double* As, const double* Bs, int wm, int wn,
                                          int gq, int tq, int nks, int mt_lim,
                                          double (&acc)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  if (nks == BK / 8 && mt_lim == Tile<BN>::WMT)
    chunk_mma_body<BN, IS_P, true>(As, Bs, wm, wn, gq, tq, nks, mt_lim, acc);
  else
    chunk_mma_body<BN, IS_P, false>(As, Bs, wm, wn, gq, tq, nks, mt_lim, acc);
}

// One output tile of a stage (or Horner product): tile index `bid` (the
// block index of the one-launch-per-stage kernel below, or a work item of the
// persistent kernel), shared-memory ring `bsm`.
// The fields that change from one stage (or Horner product) to the next;
// the rest of StageArgs is shared by all of a step's launches.
struct ProdSel {
  const double2* Yin;
  double2* Yout;
  int stage;
  double hg, vscale;
  int hlast;
};

__device__ __forceinline__ ProdSel prod_sel(const StageArgs& a) {
  return ProdSel{a.Yin, a.Yout, a.stage, a.hg, a.vscale, a.hlast};
}

// A P chunk and a Q chunk of the same index together: per 8-deep k-step the
// P product goes into accP and the Q product into accQ, so each warp keeps
// twice as many independent DMMA accumulations in flight as with one chunk
// at a time, with each accumulator's terms in the same order as before.
template <int BN, bool FULL>
__device__ __forceinline__ void pair_mma_body(const double* AsP, const double* BsP, const double* AsQ,
                                         const double* BsQ, int wm, int wn, int gq, int tq,
                                         int nksP, int nksQ, int mt_lim,
                                         double (&accP)[Tile<BN>::WMT][Tile<BN>::WNT][4],
                                         double (&accQ)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  constexpr int WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
  constexpr int LDB = BN + 4;
#pragma unroll
  for (int ks = 0; ks < BK / 8; ++ks) {
    const int k = ks * 8 + tq;
    if (FULL || ks < nksP) {
      double af[WMT][4], bf[WNT][2];
#pragma unroll
      for (int mt = 0; mt < WMT; ++mt) {
        if (!FULL && mt >= mt_lim) break;
        const int m = wm * (WMT * 16) + mt * 16 + gq;
        af[mt][0] = AsP[k * LDA_P + m];
        af[mt][1] = AsP[k * LDA_P + m + 8];
        af[mt][2] = AsP[(k + 4) * LDA_P + m];
        af[mt][3] = AsP[(k + 4) * LDA_P + m + 8];
      }
#pragma unroll
      for (int nt = 0; nt < WNT; ++nt) {
        const int n = wn * (WNT * 8) + nt * 8 + gq;
        bf[nt][0] = BsP[k * LDB + n];
        bf[nt][1] = BsP[(k + 4) * LDB + n];
      }
#pragma unroll
      for (int mt = 0; mt < WMT; ++mt) {
        if (!FULL && mt >= mt_lim) break;
#pragma unroll
        for (int nt = 0; nt < WNT; ++nt) dmma16x8x8(accP[mt][nt], af[mt], bf[nt]);
      }
    }
    if (FULL || ks < nksQ) {
      double af[WMT][4], bf[WNT][2];
#pragma unroll
      for (int mt = 0; mt < WMT; ++mt) {
        if (!FULL && mt >= mt_lim) break;
        const int m = wm * (WMT * 16) + mt * 16 + gq;
        af[mt][0] = AsQ[m * LDA_Q + k];
        af[mt][1] = AsQ[(m + 8) * LDA_Q + k];
        af[mt][2] = AsQ[m * LDA_Q + k + 4];
        af[mt][3] = AsQ[(m + 8) * LDA_Q + k + 4];
      }
#pragma unroll
      for (int nt = 0; nt < WNT; ++nt) {
        const int n = wn * (WNT * 8) + nt * 8 + gq;
        bf[nt][0] = BsQ[k * LDB + n];
        bf[nt][1] = BsQ[(k + 4) * LDB + n];
      }
#pragma unroll
      for (int mt = 0; mt < WMT; ++mt) {
        if (!FULL && mt >= mt_lim) break;
#pragma unroll
        for (int nt = 0; nt < WNT; ++nt) dmma16x8x8(accQ[mt][nt], af[mt], bf[nt]);
      }
    }
  }
}

template <int BN>
__device__ __forceinline__ void pair_mma(const double* AsP, const double* BsP, const double* AsQ,
                                         const double* BsQ, int wm, int wn, int gq, int tq,
                                         int nksP, int nksQ, int mt_lim,
                                         double (&accP)[Tile<BN>::WMT][Tile<BN>::WNT][4],
                                         double (&accQ)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  if (nksP == BK / 8 && nksQ == BK / 8 && mt_lim == Tile<BN>::WMT)
    pair_mma_body<BN, true>(AsP, BsP, AsQ, BsQ, wm, wn, gq, tq, nksP, nksQ, mt_lim, accP, accQ);
  else
    pair_mma_body<BN, false>(AsP, BsP, AsQ, BsQ, wm, wn, gq, tq, nksP, nksQ, mt_lim, accP, accQ);
}

template <int BN, int NSTB, int MODE, int SPLIT>
__device__ __forceinline__ void stage_tile(const StageArgs& a, const ProdSel& ps, const int bid,
                                           double* bsm) {
  constexpr int WGM = Tile<BN>::WGM, WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
  constexpr int LDB = BN + 4;
  constexpr int B_STAGE = b_stage<BN>();
  constexpr int WM_TILES = WMT, WN_TILES = WNT;
  static_assert(Tile<BN>::WGM * Tile<BN>::WGN * 32 == BTHREADS, "8 warps");
  static_assert(WGM * WMT * 16 == BM && Tile<BN>::WGN * WNT * 8 == BN, "tile shape");
  const Geometry& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int wm = warp % WGM, wn = warp / WGM;

  // Block index = (row tile, column tile[, k half]) with the column tile and
  // k half varying fastest: CTAs that read the same coupling rows run side by
  // side and share them through L2.
  const int ncolt = (2 * a.ncol + BN - 1) / BN;
  const int zk = SPLIT ? (bid & 1) : 0;
  const int tp = SPLIT ? (bid >> 1) : bid;  // tile pair
  const int rtile = tp / ncolt;
  // row tile -> state block L and first local row r0
  int L = 0, rt = rtile;
  while (true) {
    const int nt = (g.state_off[L + 1] - g.state_off[L] + BM - 1) / BM;
    if (rt < nt || L + 1 >= g.nstate_blk) break;
    rt -= nt;
    ++L;
  }
  const int nL = g.state_off[L + 1] - g.state_off[L];
  const int r0 = rt * BM;
  const int c0 = (tp % ncolt) * BN;         // first real column
  const int ncr = 2 * a.ncol;               // real columns in use
  const int ldr = 2 * a.ldc;                // real row pitch of X / Y
  const bool hasP = L > 0, hasQ = L < g.nblk;
  const int KP = hasP ? g.state_off[L] - g.state_off[L - 1] : 0;
  const int KQ = hasQ ? g.state_off[L + 2] - g.state_off[L + 1] : 0;
  const int nchP = (KP + BK - 1) / BK, nchQ = (KQ + BK - 1) / BK;
  const int nch = nchP + nchQ;
  const double qsign = (a.gauge == 1) ? -1.0 : 1.0;
  // this warp's m-tiles that hold rows of block L
  const int wrows = nL - r0 - wm * (Tile<BN>::WMT * 16);
  const int mt_lim = wrows <= 0 ? 0 : min(Tile<BN>::WMT, (wrows + 15) / 16);

  pdl_wait();
  const double* Yin = reinterpret_cast<const double*>(ps.Yin);

  // Each thread's cp.async assignments are fixed for the whole K loop, so
  // their source pointers and bounds are set up once; a chunk only adds its
  // k offset.
  constexpr int A_PER = BK * (BM / 2) / BTHREADS;       // 16-B copies of A per thread
  constexpr int BPR = BN / 2;                            // 16-B copies per B row
  constexpr int B_ROWS = BTHREADS / BPR;                 // B rows per pass
  constexpr int B_PER = (BK + B_ROWS - 1) / B_ROWS;
  const int tid = threadIdx.x;
  const int p_mm = 2 * (tid % (BM / 2)), p_kk0 = tid / (BM / 2);   // P: kk = p_kk0 + 8 i
  const int q_kk = 2 * (tid % (BK / 2)), q_mm0 = tid / (BK / 2);   // Q: mm = q_mm0 + 16 i
  const int b_nn = 2 * (tid % BPR), b_kk0 = tid / BPR;
  const bool p_mv = r0 + p_mm < nL;
  const bool b_nv = c0 + b_nn < ncr;
  const long long pitchP = hasP ? g.blk[L - 1].pitch : 0;
  const long long pitchQ = hasQ ? g.blk[L].pitch : 0;
  const double* p_base = hasP ? a.D + g.blk[L - 1].d_off + r0 + p_mm : a.D;
  const double* q_base = hasQ ? a.D + g.blk[L].d_off + (long long)(r0 + q_mm0) * pitchQ + q_kk : a.D;
  const int yrowP = hasP ? g.state_off[L - 1] : 0, yrowQ = hasQ ? g.state_off[L + 1] : 0;

  auto load_chunk = [&](int ch, double* As) {
    double* Bs = As + A_STAGE;
    const bool isP = ch < nchP;
    const int k0 = (isP ? ch : ch - nchP) * BK;
    const int nK = isP ? KP : KQ;
    const int yrow0 = isP ? yrowP : yrowQ;
    if (isP) {
      // A = D_{L-1}^T : D_{L-1}[k0+kk][r0+mm] -> As[kk][mm]
#pragma unroll
      for (int i = 0; i < A_PER; ++i) {
        const int kk = p_kk0 + (BTHREADS / (BM / 2)) * i;
        const bool v = p_mv && (k0 + kk < nK);
        cp_async16(As + kk * LDA_P + p_mm, v ? p_base + (long long)(k0 + kk) * pitchP : a.D, v);
      }
    } else {
      // A = D_L : D_L[r0+mm][k0+kk] -> As[mm][kk]
#pragma unroll
      for (int i = 0; i < A_PER; ++i) {
        const int mm = q_mm0 + (BTHREADS / (BK / 2)) * i;
        const bool v = (r0 + mm < nL) && (k0 + q_kk < nK);
        cp_async16(As + mm * LDA_Q + q_kk,
                   v ? q_base + (long long)((BTHREADS / (BK / 2)) * i) * pitchQ + k0 : a.D, v);
      }
    }
    // B = Y rows of the coupled block: Bs[kk][nn]
#pragma unroll
    for (int i = 0; i < B_PER; ++i) {
      const int kk = b_kk0 + B_ROWS * i;
      if (kk < BK) {
        const bool v = b_nv && (k0 + kk < nK);
        cp_async16(Bs + kk * LDB + b_nn, v ? Yin + (long long)(yrow0 + k0 + kk) * ldr + c0 + b_nn : Yin, v);
      }
    }
  };

  // The coupling's two halves accumulate separately -- P (D_{L-1}^T y_{L-1})
  // and Q (+-D_L y_{L+1}), chunks in order within each -- and are added once,
  // P + Q, at the end: the same association whether one CTA does both or two
  // CTAs split them, so every variant gives the same bits.
  double accP[WM_TILES][WN_TILES][4], accQ[WM_TILES][WN_TILES][4];
#pragma unroll
  for (int i = 0; i < WM_TILES; ++i)
#pragma unroll
    for (int j = 0; j < WN_TILES; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) accP[i][j][v] = accQ[i][j][v] = 0.0;

  if constexpr (paired<BN, SPLIT>()) {
    // slot i holds P chunk i (first half) and Q chunk i (second half)
    constexpr int NSP = pair_slots<NSTB>();
    constexpr int CH = A_STAGE + B_STAGE;
    const int nsup = max(nchP, nchQ);
    auto load_pair = [&](int i, int slot) {
      double* base = bsm + slot * 2 * CH;
      if (i < nchP) load_chunk(i, base);
      if (i < nchQ) load_chunk(nchP + i, base + CH);
    };
    for (int p = 0; p < NSP - 1; ++p) {
      if (p < nsup) load_pair(p, p);
      cp_commit();
    }
    for (int i = 0; i < nsup; ++i) {
      cp_wait<NSP - 2>();
      __syncthreads();
      {
        const int nx = i + NSP - 1;
        if (nx < nsup) load_pair(nx, nx % NSP);
        cp_commit();
      }
      const double* base = bsm + (i % NSP) * 2 * CH;
      // valid k-steps: the coupled blocks' columns left from k0 = i * BK
      const int nksP = i < nchP ? min(BK / 8, (KP - i * BK + 7) / 8) : 0;
      const int nksQ = i < nchQ ? min(BK / 8, (KQ - i * BK + 7) / 8) : 0;
      pair_mma<BN>(base, base + A_STAGE, base + CH, base + CH + A_STAGE, wm, wn, gq, tq, nksP,
                   nksQ, mt_lim, accP, accQ);
    }
    cp_wait<0>();
  } else {
    const int ch0 = (SPLIT && zk == 1) ? nchP : 0;
    const int ch1 = (SPLIT && zk == 0) ? nchP : nch;
    const int nmine = ch1 - ch0;
    for (int p = 0; p < NSTB - 1; ++p) {
      if (p < nmine) load_chunk(ch0 + p, bsm + p * (A_STAGE + B_STAGE));
      cp_commit();
    }
    // this CTA's P chunks come first (local indices [0, nPm)), then its Q chunks
    const int nPm = (SPLIT && zk == 1) ? 0 : nchP;
    for (int ci = 0; ci < nmine; ++ci) {
      cp_wait<NSTB - 2>();
      __syncthreads();
      {
        const int nx = ci + NSTB - 1;
        if (nx < nmine) load_chunk(ch0 + nx, bsm + (nx % NSTB) * (A_STAGE + B_STAGE));
        cp_commit();
      }
      const double* As = bsm + (ci % NSTB) * (A_STAGE + B_STAGE);
      const double* Bs = As + A_STAGE;
      // valid k-steps of this chunk: the coupled block's columns left from k0
      const int chg = ch0 + ci;
      const int krem = (chg < nchP) ? KP - chg * BK : KQ - (chg - nchP) * BK;
      const int nks = min(BK / 8, (krem + 7) / 8);
      if (ci < nPm)
        chunk_mma<BN, true>(As, Bs, wm, wn, gq, tq, nks, mt_lim, accP);
      else
        chunk_mma<BN, false>(As, Bs, wm, wn, gq, tq, nks, mt_lim, accQ);
    }
    cp_wait<0>();
  }
  if constexpr (SPLIT) {
    // publish this half, then the tile's second arrival takes over
    constexpr int NACC = WM_TILES * WN_TILES * 4;
    constexpr int kWsPerCta = BM * BN;  // one CTA's partial tile
    static_assert(NACC * BTHREADS == kWsPerCta, "workspace slot");
    const int z = zk;
    double* mine = a.ws + ((long long)tp * 2 + z) * kWsPerCta;
#pragma unroll
    for (int i = 0; i < WM_TILES; ++i)
#pragma unroll
      for (int j = 0; j < WN_TILES; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v)
          mine[((i * WN_TILES + j) * 4 + v) * BTHREADS + tid] = z ? accQ[i][j][v] : accP[i][j][v];
    __threadfence();
    __syncthreads();
    __shared__ int s_last;
    if (tid == 0) {
      const int old = atomicAdd(a.cnt + tp, 1);
      s_last = (old == 1);
      if (s_last) a.cnt[tp] = 0;  // ready for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const double* other = a.ws + ((long long)tp * 2 + (1 - z)) * kWsPerCta;
#pragma unroll
    for (int i = 0; i < WM_TILES; ++i)
#pragma unroll
      for (int j = 0; j < WN_TILES; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double o = __ldcg(other + ((i * WN_TILES + j) * 4 + v) * BTHREADS + tid);
          if (z) accP[i][j][v] = o;
          else accQ[i][j][v] = o;
        }
  }
  double acc[WM_TILES][WN_TILES][4];
#pragma unroll
  for (int i = 0; i < WM_TILES; ++i)
#pragma unroll
    for (int j = 0; j < WN_TILES; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = accP[i][j][v] + qsign * accQ[i][j][v];

  if constexpr (MODE == 2) {
    // ---------------- Horner epilogue (fixed step, frozen field) ----------------
    __shared__ double red_h[BM / 16][BN / 2];
#pragma unroll
    for (int nt = 0; nt < WN_TILES; ++nt) {
      const int q = (c0 + wn * (WNT * 8) + nt * 8) / 2 + tq;  // pulse column
      const bool qv = q < a.ncol;
      double nsum[WM_TILES];
#pragma unroll
      for (int mt = 0; mt < WM_TILES; ++mt) nsum[mt] = 0.0;
      const double F = qv ? a.Fs[q] : 0.0;
      const double hq = qv ? a.h[q] : 0.0;
      const double nq = (qv && ps.stage == 0) ? a.nrm[q] : 1.0;
      const double vs = ps.vscale, gm = ps.hg;
      // every operand of the thread's elements first, so that their loads are
      // in flight together (the stores below may alias them as far as the
      // compiler knows, which would otherwise order each element's loads
      // after the previous element's stores)
      double2 yv[WM_TILES][2], xv[WM_TILES][2];
      double ev[WM_TILES][2];
#pragma unroll
      for (int mt = 0; mt < WM_TILES; ++mt)
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const int r = r0 + wm * (WMT * 16) + mt * 16 + gq + 8 * hr;
          yv[mt][hr] = xv[mt][hr] = make_double2(0.0, 0.0);
          ev[mt][hr] = 0.0;
          if (!qv || r >= nL) continue;
          const long long i = g.state_off[L] + r;
          const long long idx = i * a.ldc + q;
          yv[mt][hr] = ps.Yin[idx];
          if (ps.stage != 0) xv[mt][hr] = a.X[idx];
          ev[mt][hr] = a.eps[i];
        }
#pragma unroll
      for (int mt = 0; mt < WM_TILES; ++mt)
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const int r = r0 + wm * (WMT * 16) + mt * 16 + gq + 8 * hr;
          if (!qv || r >= nL) continue;
          const long long i = g.state_off[L] + r;
          const long long idx = i * a.ldc + q;
          double wre, wim;
          double2 v, x;
          if (ps.stage == 0) {
            // x = x_new / ||x_new|| (the reference's c /= ||c||), its coupling
            // D x = (D x_new) / ||x_new||
            const double2 z = yv[mt][hr];
            x = make_double2(z.x / nq, z.y / nq);
            a.Xw[idx] = x;
            wre = vs * (acc[mt][nt][2 * hr] / nq);
            wim = vs * (acc[mt][nt][2 * hr + 1] / nq);
            v = make_double2(vs * x.x, vs * x.y);
          } else {
            wre = vs * acc[mt][nt][2 * hr];
            wim = vs * acc[mt][nt][2 * hr + 1];
            const double2 v0 = yv[mt][hr];
            v = make_double2(vs * v0.x, vs * v0.y);
            x = xv[mt][hr];
          }
          const double e = ev[mt][hr];
          double kre, kim;  // M(F) v, formed as the stage form forms k
          if (a.gauge == 0) {
            kre = fma(F, wim, e * v.y);
            kim = -fma(F, wre, e * v.x);
          } else {
            kre = fma(F, wre, e * v.y);
            kim = fma(F, wim, -e * v.x);
          }
          const double2 o = make_double2(fma(hq, kre, gm * x.x), fma(hq, kim, gm * x.y));
          ps.Yout[idx] = o;
          if (ps.hlast) nsum[mt] += o.x * o.x + o.y * o.y;
        }
      if (ps.hlast) {
#pragma unroll
        for (int o = 4; o < 32; o <<= 1)
#pragma unroll
          for (int mt = 0; mt < WM_TILES; ++mt)
            nsum[mt] += __shfl_xor_sync(0xffffffffu, nsum[mt], o);
        const int col = wn * (WNT * 4) + nt * 4 + tq;
        if (gq == 0) {
#pragma unroll
          for (int mt = 0; mt < WM_TILES; ++mt) red_h[wm * WMT + mt][col] = nsum[mt];
        }
      }
    }
    if (ps.hlast) {
      __syncthreads();
      if (threadIdx.x < BN / 2) {
        const int q = c0 / 2 + threadIdx.x;
        if (q < a.ncol) {
          double ns = red_h[0][threadIdx.x];
#pragma unroll
          for (int m = 1; m < BM / 16; ++m) ns += red_h[m][threadIdx.x];
          a.normpart[(long long)rtile * a.ldc + q] = ns;
        }
      }
    }
    return;
  }

  if constexpr (MODE == 1) {
    // ---------------- adjoint epilogue ----------------
    const int s = ps.stage;
    const long long nld = (long long)g.ntot * a.ldc;
    __shared__ double red_f[BM / 16][BN / 2];
#pragma unroll
    for (int nt = 0; nt < WN_TILES; ++nt) {
      const int q = (c0 + wn * (WNT * 8) + nt * 8) / 2 + tq;  // pulse column
      const bool qv = q < a.ncol;
      double fsum[WM_TILES];
#pragma unroll
      for (int mt = 0; mt < WM_TILES; ++mt) fsum[mt] = 0.0;
      const double F = qv ? a.Fs[s * a.fs_stride + q] : 0.0;
      const double hq = qv ? a.h[q] : 0.0;
#pragma unroll
      for (int mt = 0; mt < WM_TILES; ++mt)
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const int r = r0 + wm * (WMT * 16) + mt * 16 + gq + 8 * hr;
          if (!qv || r >= nL) continue;
          const long long i = g.state_off[L] + r;
          const long long idx = i * a.ldc + q;
          const double wre = acc[mt][nt][2 * hr], wim = acc[mt][nt][2 * hr + 1];
          const double2 kb = ps.Yin[idx];
          const double e = a.eps[i];
          // M(F) kbar (formed as the forward forms k) and M1 kbar = dM/dF kbar
          double gre, gim, mre, mim;
          if (a.gauge == 0) {
            gre = fma(F, wim, e * kb.y);
            gim = -fma(F, wre, e * kb.x);
            mre = wim;
            mim = -wre;
          } else {
            gre = fma(F, wre, e * kb.y);
            gim = fma(F, wim, -e * kb.x);
            mre = wre;
            mim = wim;
          }
          const double2 yb = make_double2(-gre, -gim);  // ybar_s = -M kbar_s
          a.K[s * nld + idx] = yb;
          const double2 y = a.Ys[idx];
          fsum[mt] -= fma(mre, y.x, mim * y.y);         // -Re<M1 kbar_s, y_s>
          const double2 zb = a.Zbar[idx];
          double2 o;
          if (s > 0) {
            // kbar_{s-1} = h b_{s-1} zbar + sum_{j >= s} h a_{j, s-1} ybar_j
            const double cb = hq * c_B8[s - 1];
            o = make_double2(cb * zb.x, cb * zb.y);
#pragma unroll
            for (int j = 1; j < kNumStages; ++j) {
              const double cj = c_A[j][s - 1];
              if (j < s || cj == 0.0) continue;
              const double2 ybj = (j == s) ? yb : a.K[j * nld + idx];
              const double cf = hq * cj;
              o.x = fma(cf, ybj.x, o.x);
              o.y = fma(cf, ybj.y, o.y);
            }
          } else {
            // lambda_n = zbar + sum_j ybar_j
            o = zb;
#pragma unroll
            for (int j = 0; j < kNumStages; ++j) {
              const double2 ybj = (j == 0) ? yb : a.K[j * nld + idx];
              o.x += ybj.x;
              o.y += ybj.y;
            }
          }
          ps.Yout[idx] = o;
        }
#pragma unroll
      for (int o = 4; o < 32; o <<= 1)
#pragma unroll
        for (int mt = 0; mt < WM_TILES; ++mt)
          fsum[mt] += __shfl_xor_sync(0xffffffffu, fsum[mt], o);
      const int col = wn * (WNT * 4) + nt * 4 + tq;
      if (gq == 0) {
#pragma unroll
        for (int mt = 0; mt < WM_TILES; ++mt) red_f[wm * WMT + mt][col] = fsum[mt];
      }
    }
    __syncthreads();
    if (threadIdx.x < BN / 2) {
      const int q = c0 / 2 + threadIdx.x;
      if (q < a.ncol) {
        double fs = red_f[0][threadIdx.x];
#pragma unroll
        for (int m = 1; m < BM / 16; ++m) fs += red_f[m][threadIdx.x];
        a.fpart[((long long)s * a.nrowtiles + rtile) * a.ldc + q] = fs;
      }
    }
    return;
  }

  // ---------------- fused RK epilogue ----------------
  const int s = ps.stage;
  const long long nld = (long long)g.ntot * a.ldc;  // complex elements per k slab
  const bool last = (s == kNumStages - 1);
  // norm partials per 16-row m-tile, summed over the tile's rows by a fixed
  // tree and over the row tile's four m-tiles in order: the same association
  // for every tile shape
  __shared__ double red_n[BM / 16][BN / 2];
  __shared__ double red_e[WGM][BN / 2];
#pragma unroll
  for (int nt = 0; nt < WN_TILES; ++nt) {
    const int q = (c0 + wn * (WNT * 8) + nt * 8) / 2 + tq;  // pulse column
    const bool qv = q < a.ncol;
    double nsum[WM_TILES], emax = 0.0;
#pragma unroll
    for (int mt = 0; mt < WM_TILES; ++mt) nsum[mt] = 0.0;
    const double F = qv ? a.Fs[s * a.fs_stride + q] : 0.0;
    const double hq = qv ? a.h[q] : 0.0;
#pragma unroll
    for (int mt = 0; mt < WM_TILES; ++mt)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int r = r0 + wm * (WMT * 16) + mt * 16 + gq + 8 * hr;
        if (!qv || r >= nL) continue;
        const long long i = g.state_off[L] + r;
        const long long idx = i * a.ldc + q;
        const double wre = acc[mt][nt][2 * hr], wim = acc[mt][nt][2 * hr + 1];
        const double2 y = ps.Yin[idx];
        const double e = a.eps[i];
        double kre, kim;
        if (a.gauge == 0) {
          kre = fma(F, wim, e * y.y);
          kim = -fma(F, wre, e * y.x);
        } else {
          kre = fma(F, wre, e * y.y);
          kim = fma(F, wim, -e * y.x);
        }
        a.K[s * nld + idx] = make_double2(kre, kim);
        if (a.want_k_only) continue;
        const double2 x = a.X[idx];
        double2 o = x;
        if (!last) {
#pragma unroll
          for (int j = 0; j < kNumStages; ++j) {
            const double cj = c_A[s + 1][j];
            if (j > s || cj == 0.0) continue;
            const double2 kj = (j == s) ? make_double2(kre, kim) : a.K[j * nld + idx];
            const double cf = hq * cj;
            o.x = fma(cf, kj.x, o.x);
            o.y = fma(cf, kj.y, o.y);
          }
        } else {
          double2 er = make_double2(0.0, 0.0);
#pragma unroll
          for (int j = 0; j < kNumStages; ++j) {
            const double bj = c_B8[j], ej = c_E[j];
            if (bj == 0.0 && ej == 0.0) continue;
            const double2 kj = (j == s) ? make_double2(kre, kim) : a.K[j * nld + idx];
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
          const double ratio = ae / (a.atol + a.rtol * fmax(ax, an));
          emax = fmax(emax, ratio);
          if (!(ratio == ratio)) emax = ratio;  // keep a NaN
          nsum[mt] += o.x * o.x + o.y * o.y;
        }
        ps.Yout[idx] = o;
      }
    if (last && !a.want_k_only) {
      // per pulse and m-tile: this thread's two rows, then the 8 lanes
      // sharing tq (fixed xor tree)
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
#pragma unroll
        for (int mt = 0; mt < WM_TILES; ++mt)
          nsum[mt] += __shfl_xor_sync(0xffffffffu, nsum[mt], o);
        const double oe = __shfl_xor_sync(0xffffffffu, emax, o);
        emax = (oe != oe) ? oe : fmax(emax, oe);
      }
      const int col = wn * (WNT * 4) + nt * 4 + tq;  // pulse slot within the CTA
      if (gq == 0) {
#pragma unroll
        for (int mt = 0; mt < WM_TILES; ++mt) red_n[wm * WMT + mt][col] = nsum[mt];
        red_e[wm][col] = emax;
      }
    }
  }
  if (last && !a.want_k_only) {
    __syncthreads();
    if (threadIdx.x < BN / 2) {
      const int q = c0 / 2 + threadIdx.x;
      if (q < a.ncol) {
        double ns = red_n[0][threadIdx.x], em = red_e[0][threadIdx.x];
#pragma unroll
        for (int m = 1; m < BM / 16; ++m) ns += red_n[m][threadIdx.x];
#pragma unroll
        for (int w = 1; w < WGM; ++w) {
          const double e = red_e[w][threadIdx.x];
          em = (em != em) ? em : ((e != e) ? e : fmax(em, e));
        }
        a.normpart[(long long)rtile * a.ldc + q] = ns;
        atomicMax(&a.err[q], (unsigned long long)__double_as_longlong(em));
      }
    }
  }
}


template <int BN, int NSTB, int MODE, int SPLIT>
__global__ void __launch_bounds__(BTHREADS, 2) k_batch_stage(const __grid_constant__ StageArgs a) {
  extern __shared__ __align__(16) double bsm[];
  pdl_trigger();
  stage_tile<BN, NSTB, MODE, SPLIT>(a, prod_sel(a), (int)blockIdx.x, bsm);
}

// The 12 Horner products of one fixed step in one persistent launch.  Work
// items are (product p, column tile c, row tile r), handed out in that order
// by an atomic ticket; an item waits until product p-1 has finished every row
// tile of the three blocks its rows couple to (L-1, L, L+1) in the same
// column tile -- its GEMM operand rows and its own rows -- then runs the tile
// exactly as the one-launch-per-product kernel would.  Pulse columns never
// depend on each other, so the CTAs flow from one product into the next
// without a grid-wide barrier: the last partial wave of one product overlaps
// the first tiles of the next.  An item only waits for items with smaller
// tickets, all of them already taken by running CTAs, so the launch needs no
// co-residency guarantee.  Waits are bounded (the context's limit); one that
// runs out raises the status word and ends the CTA, and the others then run
// out of their own waits.  Item p's writes go to Y[(p+1)&1]; the rows it
// overwrites were last read by product p-1 items that it waited for.
struct HornerArgs {
  StageArgs a;            // X, Y, D, fields, steps; the per-product fields are set here
  const double2* Y[2];    // ping-pong of the products (Y[1] first)
  unsigned* ticket;       // work counter, zero at launch
  unsigned* done;         // [12][ncolt][nstate_blk] finished row tiles, zero at launch
  unsigned* status;
  unsigned long long wait_ns;
  unsigned skew;          // 0; 1 when a test injects a dependency that cannot complete
  int ncolt;              // column tiles
};

__constant__ double c_G[13];   // the stability polynomial's coefficients

template <int BN, int NSTB>
__global__ void __launch_bounds__(BTHREADS, 2) k_batch_horner(const __grid_constant__ HornerArgs h) {
  extern __shared__ __align__(16) double bsm[];
  __shared__ int s_item, s_dead;
  const Geometry& g = h.a.g;
  const int nrt = h.a.nrowtiles, ncolt = h.ncolt;
  const int per = nrt * ncolt, total = 12 * per;
  if (threadIdx.x == 0) s_dead = 0;
  for (;;) {
    __syncthreads();   // the previous tile's shared-memory reads are over
    if (threadIdx.x == 0) {
      s_item = (int)atomicAdd(h.ticket, 1u);
      // another CTA's wait ran out: its items will never finish, stop now
      if (*(volatile unsigned*)h.status & ST_WAIT_TIMEOUT) s_dead = 1;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= total || s_dead) break;
    const int p = item / per, w = item % per;
    const int ct = w / nrt, rtile = w % nrt;   // column tile outer: products flow per column
    int L = 0, rt = rtile;
    while (true) {
      const int nt = (g.state_off[L + 1] - g.state_off[L] + BM - 1) / BM;
      if (rt < nt || L + 1 >= g.nstate_blk) break;
      rt -= nt;
      ++L;
    }
    if (p > 0 && threadIdx.x == 0) {
      const unsigned* dn = h.done + ((size_t)(p - 1) * ncolt + ct) * g.nstate_blk;
      const unsigned long long t0 = globaltimer_ns();
      for (int Ld = max(L - 1, 0); Ld <= min(L + 1, g.nstate_blk - 1) && !s_dead; ++Ld) {
        const unsigned need =
            (unsigned)((g.state_off[Ld + 1] - g.state_off[Ld] + BM - 1) / BM) + h.skew;
        for (unsigned it = 0;; ++it) {
          unsigned v;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(dn + Ld) : "memory");
          if (v >= need) break;
          if ((it & 255u) == 255u) {
            if (globaltimer_ns() - t0 > h.wait_ns) {
              atomicOr(h.status, ST_WAIT_TIMEOUT);
              s_dead = 1;
              break;
            }
            if (*(volatile unsigned*)h.status & ST_WAIT_TIMEOUT) {  // another CTA gave up
              s_dead = 1;
              break;
            }
          }
        }
      }
    }
    __syncthreads();
    if (s_dead) break;
    ProdSel ps;
    ps.stage = p;
    ps.Yin = h.Y[p & 1];   // p = 0: the previous step's unnormalised x_new in Y[0]
    ps.Yout = const_cast<double2*>(h.Y[(p + 1) & 1]);
    ps.hg = c_G[11 - p];
    ps.vscale = (p == 0) ? c_G[12] : 1.0;
    ps.hlast = (p == 11) ? 1 : 0;
    stage_tile<BN, NSTB, 2, 0>(h.a, ps, rtile * ncolt + ct, bsm);
    __syncthreads();   // every thread's stores of the tile are issued
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(h.done + ((size_t)p * ncolt + ct) * g.nstate_blk + L, 1u);
    }
  }
}

// Stage-GEMM variants: pulse-column tile width (real columns), cp.async
// pipeline depth, and whether the P and Q halves of a tile run in two CTAs
// (split; the second to finish adds the first one's partial).  Variant v is
// index v here (MPC_BATCH_VARIANT pins one).  Three-stage variants fit two
// CTAs per SM.
struct TileVariant {
  int bn, nst, split;
};
constexpr TileVariant kVariants[] = {{16, 3, 0}, {16, 6, 0}, {32, 3, 0}, {32, 6, 0}, {64, 3, 0},
                                     {16, 6, 1}, {32, 6, 1}, {32, 3, 1}, {64, 3, 1}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

inline int width_bucket(int ncol) {
  int j = 0;
  while ((1 << j) < ncol) ++j;
  return j;
}

// Before tuning: the narrowest tile that covers the pulses.
inline int default_variant(int ncol) {
  const int ncr = 2 * ncol;
  return ncr <= 16 ? 1 : (ncr <= 128 ? 3 : 4);
}

template <int BN, int NST, int MODE, int SPLIT>
cudaError_t launch_tile(cudaStream_t st, const StageArgs& a) {
  const int ncolt = (2 * a.ncol + BN - 1) / BN;
  return mpc_launch_pdl(k_batch_stage<BN, NST, MODE, SPLIT>,
                        dim3(a.nrowtiles * ncolt * (SPLIT ? 2 : 1)), dim3(BTHREADS),
                        stage_smem<BN, NST, SPLIT>(), st, a);
}

template <int MODE>
cudaError_t launch_variant(cudaStream_t st, int v, const StageArgs& a) {
  switch (v) {
    case 0: return launch_tile<16, 3, MODE, 0>(st, a);
    case 1: return launch_tile<16, 6, MODE, 0>(st, a);
    case 2: return launch_tile<32, 3, MODE, 0>(st, a);
    case 3: return launch_tile<32, 6, MODE, 0>(st, a);
    case 4: return launch_tile<64, 3, MODE, 0>(st, a);
    case 5: return launch_tile<16, 6, MODE, 1>(st, a);
    case 6: return launch_tile<32, 6, MODE, 1>(st, a);
    case 7: return launch_tile<32, 3, MODE, 1>(st, a);
    default: return launch_tile<64, 3, MODE, 1>(st, a);
  }
}

// The persistent Horner launch for tile variant v (its column width and ring
// depth; a k-split variant runs unsplit): grid = min(work items, resident
// CTAs), counters cleared on the stream first.
template <int BN, int NST>
cudaError_t launch_horner_tile(cudaStream_t st, const HornerArgs& h, int sms, int items) {
  static int per_sm = 0;   // resident CTAs per SM (the same on every B200)
  if (per_sm == 0) {
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_batch_horner<BN, NST>, BTHREADS, stage_smem<BN, NST, 0>());
    if (e != cudaSuccess) {
      per_sm = 0;
      return e;
    }
  }
  const int grid = std::max(1, std::min(items, std::max(per_sm, 1) * sms));
  // plain stream order: the counters' clear right before must be complete
  k_batch_horner<BN, NST><<<grid, BTHREADS, stage_smem<BN, NST, 0>(), st>>>(h);
  return cudaGetLastError();
}

inline int horner_tile_bn(int v) { return kVariants[v].bn; }

inline cudaError_t launch_horner_variant(cudaStream_t st, int v, const HornerArgs& h, int sms,
                                         int items) {
  switch (v) {
    case 0: return launch_horner_tile<16, 3>(st, h, sms, items);
    case 1:
    case 5: return launch_horner_tile<16, 6>(st, h, sms, items);
    case 2:
    case 7: return launch_horner_tile<32, 3>(st, h, sms, items);
    case 3:
    case 6: return launch_horner_tile<32, 6>(st, h, sms, items);
    default: return launch_horner_tile<64, 3>(st, h, sms, items);
  }
}

// Workspace of the split variants for nrowtiles row tiles and ldc pulse
// columns: two BM x BN partial tiles per tile pair, at most 2 ldc + 64 real
// columns of tiles whatever BN is; the finest column tiling (16) sets the
// number of arrival counters.
inline size_t split_ws_doubles(int nrowtiles, int ldc) {
  return (size_t)nrowtiles * (2 * ldc + 64) * 2 * BM;
}
inline size_t split_cnt_ints(int nrowtiles, int ldc) {
  return (size_t)nrowtiles * ((2 * ldc + 15) / 16);
}

template <int MODE>
cudaError_t set_stage_attrs() {
  cudaError_t e;
#define MPC_STAGE_ATTR(BN, NST, SPLIT)                                                   \
  if ((e = cudaFuncSetAttribute(k_batch_stage<BN, NST, MODE, SPLIT>,                     \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                                stage_smem<BN, NST, SPLIT>())) != cudaSuccess)           \
    return e;
  MPC_STAGE_ATTR(16, 3, 0)
  MPC_STAGE_ATTR(16, 6, 0)
  MPC_STAGE_ATTR(32, 3, 0)
  MPC_STAGE_ATTR(32, 6, 0)
  MPC_STAGE_ATTR(64, 3, 0)
  MPC_STAGE_ATTR(16, 6, 1)
  MPC_STAGE_ATTR(32, 6, 1)
  MPC_STAGE_ATTR(32, 3, 1)
  MPC_STAGE_ATTR(64, 3, 1)
#undef MPC_STAGE_ATTR
  if (MODE == 2) {
#define MPC_HORNER_ATTR(BN, NST)                                                          \
  if ((e = cudaFuncSetAttribute(k_batch_horner<BN, NST>,                                  \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                                stage_smem<BN, NST, 0>())) != cudaSuccess)               \
    return e;
    MPC_HORNER_ATTR(16, 3)
    MPC_HORNER_ATTR(16, 6)
    MPC_HORNER_ATTR(32, 3)
    MPC_HORNER_ATTR(32, 6)
    MPC_HORNER_ATTR(64, 3)
#undef MPC_HORNER_ATTR
  }
  return cudaSuccess;
}

// This translation unit's tableau constants and kernel attributes, once per
// device.
inline int stage_setup(int device) {
  static bool done[64] = {};
  if (device < 0 || device >= 64) return mpc_fail(MPC_ERR_ARG, "device %d", device);
  if (done[device]) return MPC_OK;
  double A[13][13], B8[13], E[13], Cn[13];
  for (int i = 0; i < 13; ++i) {
    for (int j = 0; j < 13; ++j) A[i][j] = rkf78::A[i][j];
    B8[i] = rkf78::B8[i];
    E[i] = rkf78::B8[i] - rkf78::B7[i];
    Cn[i] = rkf78::C[i];
  }
  CK(cudaMemcpyToSymbol(c_A, A, sizeof A));
  CK(cudaMemcpyToSymbol(c_B8, B8, sizeof B8));
  CK(cudaMemcpyToSymbol(c_E, E, sizeof E));
  CK(cudaMemcpyToSymbol(c_C, Cn, sizeof Cn));
  CK(cudaMemcpyToSymbol(c_G, rkf78::G, sizeof rkf78::G));
  CK(set_stage_attrs<0>());
  CK(set_stage_attrs<1>());
  CK(set_stage_attrs<2>());
  done[device] = true;
  return MPC_OK;
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace
