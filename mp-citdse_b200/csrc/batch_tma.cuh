// batch_tma.cuh -- the Horner products of the batched fixed step (the
// frozen-field RKF78 step as its degree-12 stability polynomial) with their
// operand tiles moved by the Tensor Memory Accelerator.
//
// One output tile per CTA.  The CTA's eight warps share a ring of NS
// shared-memory slots, each guarded by a pair of mbarriers ("full": the
// slot's TMA loads have landed; "empty": all eight warps are done with it).
// A chunk is two cp.async.bulk.tensor instructions: the BK-deep coupling
// tile as one 3-D box (D_{L-1} k-major as {16, 32, 4}, or D_L m-major as
// {16, 64, 2}: 16-double column groups as the outer dimension) and the
// state tile ({16, 32, BN / 16} of Y).  The first NS coupling tiles are
// requested before the programmatic-launch wait (the couplings are
// constant), their state tiles right after it; chunk j + NS is requested by
// warp j % 8 once every warp is done with chunk j, so the issuing duty
// rotates.  The K loop holds fragment loads, DMMAs (mma.sync m16n8k8 .f64)
// and one mbarrier arrival per warp and chunk -- no copy address arithmetic
// and no CTA-wide barrier; rings deep enough for one CTA per SM take a P and
// a Q chunk together (two independent accumulations per fragment).  The
// epilogue is stage_tile<.., 2, ..>'s Horner epilogue.
//
// Every box row is one 128-byte line and lands with the 128-byte TMA
// swizzle (16-byte chunk c of line r stored at chunk c ^ (r & 7)).  The DMMA
// fragment layouts read such a tile conflict-free once the rows of each
// 16-row m-tile and the columns of each 8-column n-tile are assigned to
// fragment rows and columns in a fixed permuted order (frag_row, frag_col):
// every half-warp fragment load then covers the 32 banks exactly once, for
// the k-major and the m-major coupling tiles and for the state tile alike.
// The permutation only relabels which fragment slot holds which row or
// column: every output element is the same sum over k in the same order,
// so the results have the bits of the cp.async kernels.
//
// The norm partials of the last product are summed over the tile's rows in
// the same fixed tree as stage_tile's (per 16-row m-tile: row pairs g,
// g + 8, then a butterfly over g; then the four m-tiles in order), here
// through shared memory since a lane's rows are permuted.
//
// Waits are bounded: a ring wait that runs past the context's limit raises
// ST_WAIT_TIMEOUT and marks the CTA dead (later waits return at once, the
// loop runs out on garbage that the raised status voids), and a dead CTA
// waits for the copies it issued before it exits.
#pragma once

namespace {

constexpr int kTmaConsumerWarps = BTHREADS / 32;
constexpr int kTmaConsumerThreads = BTHREADS;
constexpr int kTmaBarId = 1;   // named barrier of the epilogue (all warps)

// Row of a 16-row m-tile held by fragment row g (0..15).
__device__ __forceinline__ int frag_row(int g) {
  return (int)((0x9a56b874de12fc30ull >> (4 * g)) & 15ull);
}
// Column of a 16-column box held by fragment column g (0..7) of the box's
// n-tile nb (0, 1).  Fragment column pairs (2t, 2t + 1) stay adjacent and
// even-aligned: the real and imaginary part of one pulse.
__device__ __forceinline__ int frag_col(int nb, int g) {
  return 4 * nb + (g & 1) + 8 * ((g >> 1) & 1) + 2 * (g >> 2);
}
// Offset (doubles) of element (line r, column c) of a 128-byte-wide box
// stored with the 128-byte swizzle at a 1024-byte aligned base.
__device__ __forceinline__ int swz(int r, int c) {
  return r * 16 + ((((c >> 1) ^ (r & 7))) << 1) + (c & 1);
}

// Waits for phase `parity` of a ring barrier; gives up after limit_ns
// (raising ST_WAIT_TIMEOUT and marking the CTA dead), or at once when the
// CTA is already dead.
// (the waiting threads sleep in the try_wait rather than poll the barrier:
// a ring barrier has 256 waiters and the copy engine's completions to take)
__device__ __forceinline__ bool ring_wait(uint64_t* bar, uint32_t parity, volatile int* dead,
                                          unsigned* status, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    if (mbar_try_wait_sleep(bar, parity, 100000u)) return true;
    if (*dead) return false;
    if (globaltimer_ns() - t0 > limit_ns) {
      *dead = 1;
      atomicOr(status, ST_WAIT_TIMEOUT);
      return false;
    }
  }
}

// Coupling blocks the TMA-fed launch takes (its tensor maps travel in the
// kernel parameters).
constexpr int kTmaMaxBlocks = 8;

struct HornerTmaArgs {
  // 3-D views (16-double column groups as the outer dimension) with the
  // 128-byte swizzle: D_L as [n_L][n_{L+1}] in {16, 32, 4} boxes (index L:
  // the k-major A tile of block L + 1), in {16, 64, 2} boxes (kTmaMaxBlocks
  // + L: the m-major A tile of block L); Y[0], Y[1] as [ntot][2 ldc] in
  // {16, 32, BN / 16} boxes (2 kTmaMaxBlocks + 0, 1)
  CUtensorMap maps[2 * kTmaMaxBlocks + 2];
  StageArgs a;                // X, Xw, nrm, D, eps, fields, steps, normpart, geometry
  const double2* Y[2];        // ping-pong of the products
  unsigned* status;
  unsigned long long wait_ns;
  int ncolt;                  // column tiles
  int p;                      // the product of this launch (0 .. 11)
};

// One tile's geometry: row tile -> state block L, first row r0, block rows
// nL; the coupled blocks' extents and chunk counts.
struct TmaTileGeom {
  int L, r0, nL, c0, KP, KQ, nchP, nchQ;
};

template <int BN>
__device__ __forceinline__ TmaTileGeom tma_tile_geom(const Geometry& g, int rtile, int ct) {
  TmaTileGeom t;
  int L = 0, rt = rtile;
  while (true) {
    const int nt = (g.state_off[L + 1] - g.state_off[L] + BM - 1) / BM;
    if (rt < nt || L + 1 >= g.nstate_blk) break;
    rt -= nt;
    ++L;
  }
  t.L = L;
  t.nL = g.state_off[L + 1] - g.state_off[L];
  t.r0 = rt * BM;
  t.c0 = ct * BN;
  t.KP = L > 0 ? g.state_off[L] - g.state_off[L - 1] : 0;
  t.KQ = L < g.nblk ? g.state_off[L + 2] - g.state_off[L + 1] : 0;
  t.nchP = (t.KP + BK - 1) / BK;
  t.nchQ = (t.KQ + BK - 1) / BK;
  return t;
}

// One BK-deep chunk from a swizzled slot into acc.  oA[mt][0/1]: the
// thread's offsets of fragment rows g and g + 8 at k-step 0 (P: k-major
// tile, Q: m-major tile); oB[nt]: the state tile offset of its column.
template <int BN, bool IS_P, bool FULL>
__device__ __forceinline__ void tma_chunk_mma(const double* As, const double* Bs,
                                              const int (&oA)[Tile<BN>::WMT][2],
                                              const int (&oB)[Tile<BN>::WNT], int nks, int mt_lim,
                                              double (&acc)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  constexpr int WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
#pragma unroll
  for (int ks = 0; ks < BK / 8; ++ks) {
    if (!FULL && ks >= nks) break;
    double af[WMT][4], bf[WNT][2];
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
      if constexpr (IS_P) {
        // line k = 8 ks + t (+4), column m: k + 4 flips chunk bit 2
        const int o0 = oA[mt][0] + ks * 128, o1 = oA[mt][1] + ks * 128;
        af[mt][0] = As[o0];
        af[mt][1] = As[o1];
        af[mt][2] = As[(o0 ^ 8) + 64];
        af[mt][3] = As[(o1 ^ 8) + 64];
      } else {
        // line m, column k = 8 ks + t (+4) in box ks / 2: odd ks flips
        // chunk bit 2, k + 4 flips chunk bit 1
        const int base = (ks >> 1) * 1024, x = (ks & 1) ? 8 : 0;
        af[mt][0] = As[base + (oA[mt][0] ^ x)];
        af[mt][1] = As[base + (oA[mt][1] ^ x)];
        af[mt][2] = As[base + (oA[mt][0] ^ x ^ 4)];
        af[mt][3] = As[base + (oA[mt][1] ^ x ^ 4)];
      }
    }
#pragma unroll
    for (int nt = 0; nt < WNT; ++nt) {
      const int o = oB[nt] + ks * 128;
      bf[nt][0] = Bs[o];
      bf[nt][1] = Bs[(o ^ 8) + 64];
    }
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
#pragma unroll
      for (int nt = 0; nt < WNT; ++nt) dmma16x8x8(acc[mt][nt], af[mt], bf[nt]);
    }
  }
}

template <int BN, bool IS_P>
__device__ __forceinline__ void tma_chunk(const double* As, const double* Bs,
                                          const int (&oA)[Tile<BN>::WMT][2],
                                          const int (&oB)[Tile<BN>::WNT], int nks, int mt_lim,
                                          double (&acc)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  if (nks == BK / 8 && mt_lim == Tile<BN>::WMT)
    tma_chunk_mma<BN, IS_P, true>(As, Bs, oA, oB, nks, mt_lim, acc);
  else
    tma_chunk_mma<BN, IS_P, false>(As, Bs, oA, oB, nks, mt_lim, acc);
}

// A P chunk and a Q chunk of the same index together (two slots): per
// k-step the P product into accP and the Q product into accQ, so each warp
// has twice the independent DMMA accumulations in flight; each
// accumulator's terms in the same order as chunk by chunk.
template <int BN, bool FULL>
__device__ __forceinline__ void tma_pair_mma(const double* AsP, const double* BsP,
                                             const double* AsQ, const double* BsQ,
                                             const int (&oP)[Tile<BN>::WMT][2],
                                             const int (&oQ)[Tile<BN>::WMT][2],
                                             const int (&oB)[Tile<BN>::WNT], int nksP, int nksQ,
                                             int mt_lim,
                                             double (&accP)[Tile<BN>::WMT][Tile<BN>::WNT][4],
                                             double (&accQ)[Tile<BN>::WMT][Tile<BN>::WNT][4]) {
  constexpr int WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
#pragma unroll
  for (int ks = 0; ks < BK / 8; ++ks) {
    const bool doP = FULL || ks < nksP, doQ = FULL || ks < nksQ;
    double afP[WMT][4], afQ[WMT][4], bfP[WNT][2], bfQ[WNT][2];
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
      if (doP) {
        const int o0 = oP[mt][0] + ks * 128, o1 = oP[mt][1] + ks * 128;
        afP[mt][0] = AsP[o0];
        afP[mt][1] = AsP[o1];
        afP[mt][2] = AsP[(o0 ^ 8) + 64];
        afP[mt][3] = AsP[(o1 ^ 8) + 64];
      }
      if (doQ) {
        const int base = (ks >> 1) * 1024, x = (ks & 1) ? 8 : 0;
        afQ[mt][0] = AsQ[base + (oQ[mt][0] ^ x)];
        afQ[mt][1] = AsQ[base + (oQ[mt][1] ^ x)];
        afQ[mt][2] = AsQ[base + (oQ[mt][0] ^ x ^ 4)];
        afQ[mt][3] = AsQ[base + (oQ[mt][1] ^ x ^ 4)];
      }
    }
#pragma unroll
    for (int nt = 0; nt < WNT; ++nt) {
      const int o = oB[nt] + ks * 128;
      if (doP) {
        bfP[nt][0] = BsP[o];
        bfP[nt][1] = BsP[(o ^ 8) + 64];
      }
      if (doQ) {
        bfQ[nt][0] = BsQ[o];
        bfQ[nt][1] = BsQ[(o ^ 8) + 64];
      }
    }
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt) {
      if (!FULL && mt >= mt_lim) break;
#pragma unroll
      for (int nt = 0; nt < WNT; ++nt) {
        if (doP) dmma16x8x8(accP[mt][nt], afP[mt], bfP[nt]);
        if (doQ) dmma16x8x8(accQ[mt][nt], afQ[mt], bfQ[nt]);
      }
    }
  }
}

template <int BN>
constexpr int tma_slot_doubles() {
  return BM * BK + BK * BN;
}
template <int BN, int NS>
constexpr int tma_smem() {
  return NS * tma_slot_doubles<BN>() * 8 + 1024;   // + alignment slack
}

// Chunk j of a tile (P chunks of D_{L-1}^T, Q chunks of D_L): P0, Q0, P1,
// Q1, ..., the longer half's remaining chunks last.
__device__ __forceinline__ void tma_chunk_of(int j, int nchP, int nchQ, int& i, bool& isP) {
  const int both = min(nchP, nchQ);
  if (j < 2 * both) {
    i = j >> 1;
    isP = (j & 1) == 0;
  } else {
    i = both + (j - 2 * both);
    isP = nchP > nchQ;
  }
}

// Rings small enough for two CTAs per SM (128 registers a thread) run the
// chunks one at a time; the deeper rings (one CTA per SM, registers to
// spare) pair them.
template <int BN, int NS>
constexpr bool tma_two_per_sm() {
  return tma_smem<BN, NS>() <= 100 * 1024;
}

// Product h.p of a fixed step, one tile per CTA: blockIdx.x = row tile x
// column tiles + column tile (CTAs that read the same coupling rows run side
// by side).  Chunk j lands in slot j % NS; the first NS are issued up front,
// then chunk j + NS by warp j % 8 once all eight warps are done with chunk j
// (the issuing duty rotates, so no warp carries more than an eighth of it).
// Per chunk two TMA instructions: the coupling tile and the state tile, each
// one 3-D box.
template <int BN, int NS>
__global__ void __launch_bounds__(BTHREADS, (tma_two_per_sm<BN, NS>() ? 2 : 1))
    k_horner_tma(const __grid_constant__ HornerTmaArgs h) {
  constexpr bool PAIR = !tma_two_per_sm<BN, NS>();
  constexpr int WGM = Tile<BN>::WGM, WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
  constexpr int SLOT = tma_slot_doubles<BN>();
  constexpr uint32_t SLOT_TX = SLOT * 8;
  static_assert(NS >= 2, "ring");
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  __shared__ __align__(8) uint64_t full[NS], empty[NS];
  __shared__ int s_dead, s_issued;
  __shared__ double red[BM][BN / 2];
  double* ring =
      reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(tsm_raw) + 1023) & ~uintptr_t(1023));
  const StageArgs& a = h.a;
  const Geometry& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = h.p;
  const int ncolt = h.ncolt;
  const int w = blockIdx.x;
  const TmaTileGeom t = tma_tile_geom<BN>(g, w / ncolt, w % ncolt);
  const int nch = t.nchP + t.nchQ;
  // (a half the tile does not have is never loaded: its map may be unset)
  const CUtensorMap* mapP = &h.maps[max(t.L - 1, 0)];
  const CUtensorMap* mapQ = &h.maps[kTmaMaxBlocks + min(t.L, kTmaMaxBlocks - 1)];
  const CUtensorMap* mapY = &h.maps[2 * kTmaMaxBlocks + (p & 1)];
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kTmaConsumerWarps);
    }
    s_dead = 0;
    s_issued = 0;
    fence_mbar_init();
    if (t.nchP) prefetch_tmap(mapP);
    if (t.nchQ) prefetch_tmap(mapQ);
    prefetch_tmap(mapY);
  }
  __syncthreads();
  pdl_trigger();

  // chunk j into its slot (whose previous chunk is done): its coupling tile,
  // its state tile, or both
  auto issue_part = [&](int j, bool coupling, bool state) {
    const int slot = j % NS;
    double* As = ring + slot * SLOT;
    double* Bs = As + BM * BK;
    int i;
    bool isP;
    tma_chunk_of(j, t.nchP, t.nchQ, i, isP);
    const int k0 = i * BK;
    if (coupling) {
      mbar_arrive_expect_tx(&full[slot], SLOT_TX);
      if (isP)
        tma_load_3d(As, mapP, &full[slot], 0, k0, t.r0 / 16);
      else
        tma_load_3d(As, mapQ, &full[slot], 0, t.r0, k0 / 16);
    }
    if (state) {
      const int yrow = (isP ? g.state_off[t.L - 1] : g.state_off[t.L + 1]) + k0;
      tma_load_3d(Bs, mapY, &full[slot], 0, yrow, t.c0 / 16);
      atomicMax(&s_issued, j + 1);
    }
  };
  auto issue = [&](int j) { issue_part(j, true, true); };
  // the couplings are constant: the first NS coupling tiles load while the
  // previous product finishes; the state tiles only after it has
  const int npre = min(NS, nch);
  if (threadIdx.x == 0)
    for (int j = 0; j < npre; ++j) issue_part(j, true, false);
  pdl_wait();   // the previous product's Y, the step's fields and norms
  if (threadIdx.x == 0)
    for (int j = 0; j < npre; ++j) issue_part(j, false, true);
  __syncwarp();   // (warp-synchronous instructions follow: reconverge warp 0)

  const int wm = warp % WGM, wn = warp / WGM;
  const int gq = lane >> 2, tq = lane & 3;
  const double qsign = (a.gauge == 1) ? -1.0 : 1.0;
  // fragment offsets
  int oP[WMT][2], oQ[WMT][2], oB[WNT];
#pragma unroll
  for (int mt = 0; mt < WMT; ++mt) {
    const int mtile = wm * WMT + mt;
#pragma unroll
    for (int hr = 0; hr < 2; ++hr) {
      const int rr = frag_row(gq + 8 * hr);
      oP[mt][hr] = mtile * 512 + swz(tq, rr);
      oQ[mt][hr] = swz(16 * mtile + rr, tq);
    }
  }
#pragma unroll
  for (int nt = 0; nt < WNT; ++nt) {
    const int j = wn * WNT + nt;
    oB[nt] = (j >> 1) * 512 + swz(tq, frag_col(j & 1, gq));
  }
  const int wrows = t.nL - t.r0 - wm * (WMT * 16);
  const int mt_lim = wrows <= 0 ? 0 : min(WMT, (wrows + 15) / 16);
  double accP[WMT][WNT][4], accQ[WMT][WNT][4];
#pragma unroll
  for (int i = 0; i < WMT; ++i)
#pragma unroll
    for (int j = 0; j < WNT; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) accP[i][j][v] = accQ[i][j][v] = 0.0;

  // chunk j is done with: release its slot and, on this warp's turn,
  // refill it with chunk j + NS
  auto release = [&](int j) {
    const int slot = j % NS;
    if (lane == 0) {
      mbar_arrive(&empty[slot]);
      if (warp == j % kTmaConsumerWarps && j + NS < nch &&
          ring_wait(&empty[slot], (uint32_t)(j / NS) & 1u, &s_dead, h.status, h.wait_ns))
        issue(j + NS);
    }
  };
  // (a wait that gives up leaves garbage; the raised status fails the call)
  auto acquire = [&](int j) {
    ring_wait(&full[j % NS], (uint32_t)(j / NS) & 1u, &s_dead, h.status, h.wait_ns);
  };
  const int both = min(t.nchP, t.nchQ);
  for (int j = 0; j < nch;) {
    if (PAIR && j < 2 * both) {
      // P chunk i in slot j, Q chunk i in slot j + 1
      const int i = j >> 1;
      acquire(j);
      acquire(j + 1);
      __syncwarp();
      const double* AsP = ring + (j % NS) * SLOT;
      const double* AsQ = ring + ((j + 1) % NS) * SLOT;
      const int nksP = min(BK / 8, (t.KP - i * BK + 7) / 8);
      const int nksQ = min(BK / 8, (t.KQ - i * BK + 7) / 8);
      if (nksP == BK / 8 && nksQ == BK / 8 && mt_lim == WMT)
        tma_pair_mma<BN, true>(AsP, AsP + BM * BK, AsQ, AsQ + BM * BK, oP, oQ, oB, nksP, nksQ,
                               mt_lim, accP, accQ);
      else
        tma_pair_mma<BN, false>(AsP, AsP + BM * BK, AsQ, AsQ + BM * BK, oP, oQ, oB, nksP, nksQ,
                                mt_lim, accP, accQ);
      __syncwarp();
      release(j);
      release(j + 1);
      __syncwarp();
      j += 2;
    } else {
      int i;
      bool isP;
      tma_chunk_of(j, t.nchP, t.nchQ, i, isP);
      acquire(j);
      __syncwarp();
      const double* As = ring + (j % NS) * SLOT;
      const double* Bs = As + BM * BK;
      const int nks = min(BK / 8, ((isP ? t.KP : t.KQ) - i * BK + 7) / 8);
      if (isP)
        tma_chunk<BN, true>(As, Bs, oP, oB, nks, mt_lim, accP);
      else
        tma_chunk<BN, false>(As, Bs, oQ, oB, nks, mt_lim, accQ);
      __syncwarp();
      release(j);
      __syncwarp();
      ++j;
    }
  }

  // ---------------- Horner epilogue (stage_tile<.., 2, ..>'s) ----------------
  const ProdSel ps{h.Y[p & 1], const_cast<double2*>(h.Y[(p + 1) & 1]), p, c_G[11 - p],
                   (p == 0) ? c_G[12] : 1.0, (p == 11) ? 1 : 0};
  const int rtile = w / ncolt;
  const int L = t.L, nL = t.nL, r0 = t.r0, c0 = t.c0;
#pragma unroll
  for (int nt = 0; nt < WNT; ++nt) {
    const int j = wn * WNT + nt;
    const int col = 16 * (j >> 1) + 4 * (j & 1) + 2 * (tq >> 1) + 8 * (tq & 1);
    const int q = (c0 + col) / 2;   // pulse column
    const bool qv = q < a.ncol;
    const double F = qv ? a.Fs[q] : 0.0;
    const double hq = qv ? a.h[q] : 0.0;
    const double nq = (qv && ps.stage == 0) ? a.nrm[q] : 1.0;
    const double vs = ps.vscale, gm = ps.hg;
    // operands of the thread's elements first: their loads in flight together
    double2 yv[WMT][2], xv[WMT][2];
    double ev[WMT][2];
#pragma unroll
    for (int mt = 0; mt < WMT; ++mt)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int r = r0 + 16 * (wm * WMT + mt) + frag_row(gq + 8 * hr);
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
    for (int mt = 0; mt < WMT; ++mt)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int rl = 16 * (wm * WMT + mt) + frag_row(gq + 8 * hr);
        const int r = r0 + rl;
        double nv = 0.0;
        if (qv && r < nL) {
          const double accr = accP[mt][nt][2 * hr] + qsign * accQ[mt][nt][2 * hr];
          const double acci = accP[mt][nt][2 * hr + 1] + qsign * accQ[mt][nt][2 * hr + 1];
          const long long i = g.state_off[L] + r;
          const long long idx = i * a.ldc + q;
          double wre, wim;
          double2 v, x;
          if (ps.stage == 0) {
            // x = x_new / ||x_new||, D x = (D x_new) / ||x_new||
            const double2 z = yv[mt][hr];
            x = make_double2(z.x / nq, z.y / nq);
            a.Xw[idx] = x;
            wre = vs * (accr / nq);
            wim = vs * (acci / nq);
            v = make_double2(vs * x.x, vs * x.y);
          } else {
            wre = vs * accr;
            wim = vs * acci;
            const double2 v0 = yv[mt][hr];
            v = make_double2(vs * v0.x, vs * v0.y);
            x = xv[mt][hr];
          }
          const double e = ev[mt][hr];
          double kre, kim;
          if (a.gauge == 0) {
            kre = fma(F, wim, e * v.y);
            kim = -fma(F, wre, e * v.x);
          } else {
            kre = fma(F, wre, e * v.y);
            kim = fma(F, wim, -e * v.x);
          }
          const double2 o = make_double2(fma(hq, kre, gm * x.x), fma(hq, kim, gm * x.y));
          ps.Yout[idx] = o;
          nv = o.x * o.x + o.y * o.y;
        }
        if (ps.hlast) red[rl][col / 2] = nv;
      }
  }
  if (ps.hlast) {
    named_bar_sync(kTmaBarId, kTmaConsumerThreads);
    const int tid = threadIdx.x;
    if (tid < BN / 2) {
      const int q = c0 / 2 + tid;
      if (q < a.ncol) {
        // per m-tile: s_g = (0 + v_g) + v_{g+8}, then the butterfly over g
        double ns = 0.0;
#pragma unroll
        for (int m = 0; m < BM / 16; ++m) {
          double sg[8];
#pragma unroll
          for (int gg = 0; gg < 8; ++gg)
            sg[gg] = (0.0 + red[16 * m + gg][tid]) + red[16 * m + gg + 8][tid];
          const double tm = ((sg[0] + sg[1]) + (sg[2] + sg[3])) + ((sg[4] + sg[5]) + (sg[6] + sg[7]));
          ns = (m == 0) ? tm : ns + tm;
        }
        a.normpart[(long long)rtile * a.ldc + q] = ns;
      }
    }
  }
  // a CTA that gave up: the copies it issued land before its shared memory
  // goes away
  __syncthreads();
  if (threadIdx.x == 0 && s_dead) {
    const int issued = s_issued;
    for (int j = max(0, issued - NS); j < issued; ++j) {
      int never = 0;
      ring_wait(&full[j % NS], (uint32_t)(j / NS) & 1u, &never, h.status, h.wait_ns);
    }
  }
}

template <int BN, int NS>
cudaError_t launch_horner_tma_tile(cudaStream_t st, const HornerTmaArgs& h, int sms) {
  (void)sms;
  const int grid = h.a.nrowtiles * h.ncolt;   // one tile per CTA
  return mpc_launch_pdl(k_horner_tma<BN, NS>, dim3(grid), dim3(BTHREADS), tma_smem<BN, NS>(),
                        st, h);
}

// TMA tile shapes: {column tile width, ring slots}.  {32, 4} fits two CTAs
// per SM; the deeper rings, one.
struct TmaShape {
  int bn, ns;
};
constexpr TmaShape kTmaShapes[] = {{32, 4}, {64, 6}, {16, 8}, {32, 8}};
constexpr int kNumTmaShapes = sizeof(kTmaShapes) / sizeof(kTmaShapes[0]);

inline cudaError_t launch_horner_tma_shape(cudaStream_t st, int shape, const HornerTmaArgs& h,
                                           int sms) {
  switch (shape) {
    case 0: return launch_horner_tma_tile<32, 4>(st, h, sms);
    case 1: return launch_horner_tma_tile<64, 6>(st, h, sms);
    case 2: return launch_horner_tma_tile<16, 8>(st, h, sms);
    default: return launch_horner_tma_tile<32, 8>(st, h, sms);
  }
}

inline cudaError_t set_tma_attrs() {
  cudaError_t e;
#define MPC_TMA_ATTR(BN, NS)                                                                \
  if ((e = cudaFuncSetAttribute(k_horner_tma<BN, NS>,                                     \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                                tma_smem<BN, NS>())) != cudaSuccess)                     \
    return e;
  MPC_TMA_ATTR(32, 4)
  MPC_TMA_ATTR(64, 6)
  MPC_TMA_ATTR(16, 8)
  MPC_TMA_ATTR(32, 8)
#undef MPC_TMA_ATTR
  return cudaSuccess;
}

}  // namespace
