// batch_tma.cuh -- the Horner products of the batched fixed step (the
// frozen-field RKF78 step as its degree-12 stability polynomial) with their
// operand tiles moved by the Tensor Memory Accelerator.
//
// The CTA's eight warps share a ring of shared-memory slots, each guarded by
// a pair of mbarriers ("full": the slot's TMA loads have landed; "empty":
// all eight warps are done with it).  One lane issues, per BK-deep chunk,
// the coupling tile (four 16 x 32 boxes of D_{L-1}, k-major, or two 64 x 16
// boxes of D_L, m-major) and the state tile (16-column boxes of 32 Y rows)
// with cp.async.bulk.tensor, completing on the slot's full barrier; it runs
// NS - 1 chunks ahead, into the next tile while the current one's epilogue
// runs.  The K loop holds no copy instructions, copy address arithmetic or
// CTA-wide barrier: fragment loads, DMMAs (mma.sync m16n8k8 .f64) and one
// mbarrier arrival per warp and chunk.  The epilogue is stage_tile<.., 2,
// ..>'s Horner epilogue.
//
// Every box is one 128-byte line wide and lands with the 128-byte TMA
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
// ST_WAIT_TIMEOUT and marks the CTA dead (later waits return at once); the
// warps agree by a barrier reduction to stop at the next tile, and the
// issuing lane waits for its copies in flight before the CTA exits.
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

// Consumer barrier with an OR over the participating threads' predicates.
__device__ __forceinline__ bool consumers_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(kTmaBarId), "n"(kTmaConsumerThreads)
      : "memory");
  return r != 0;
}

// Waits for phase `parity` of a ring barrier; gives up after limit_ns
// (raising ST_WAIT_TIMEOUT and marking the CTA dead), or at once when the
// CTA is already dead.
__device__ __forceinline__ bool ring_wait(uint64_t* bar, uint32_t parity, volatile int* dead,
                                          unsigned* status, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 63u) {
      if (*dead) return false;
      if (globaltimer_ns() - t0 > limit_ns) {
        *dead = 1;
        atomicOr(status, ST_WAIT_TIMEOUT);
        return false;
      }
    }
  }
}

struct HornerTmaArgs {
  StageArgs a;                // X, Xw, nrm, D, eps, fields, steps, normpart, geometry
  const CUtensorMap* maps;    // [2 nblk + 2], 64-byte aligned in device memory: D_L as
                              // [n_L][n_{L+1}] with 16 x 32 boxes (L < nblk), D_L with
                              // 16 x 64 boxes (nblk + L), Y[0] and Y[1] as
                              // [ntot][2 ldc] with 16 x 32 boxes
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

template <int BN>
constexpr int tma_slot_doubles() {
  return BM * BK + BK * BN;
}
template <int BN, int NS>
constexpr int tma_smem() {
  return NS * tma_slot_doubles<BN>() * 8 + 1024;   // + alignment slack
}

// The issuing lane's position in the CTA's chunk sequence: tiles w =
// blockIdx.x, blockIdx.x + gridDim.x, ...; per tile, chunk i of the P half
// then of the Q half, for i = 0, 1, ... (a half with no chunk i is skipped).
struct TmaCursor {
  TmaTileGeom t;
  int w, i, half;
  uint32_t it;   // chunks (and the end marker) issued so far
  bool ended;
};

template <int BN>
__device__ __forceinline__ void cursor_seek(TmaCursor& cu, const Geometry& g, int ncolt, int per) {
  // from (i, half) forward to the next chunk that exists, across tiles; each
  // pass moves half, i or w forward, so this ends
  for (;;) {
    if (cu.w >= per) return;
    if (cu.half >= 2) {
      cu.half = 0;
      ++cu.i;
    }
    const int nsup = max(cu.t.nchP, cu.t.nchQ);
    if (cu.i >= nsup) {
      cu.i = 0;
      cu.half = 0;
      cu.w += gridDim.x;
      if (cu.w < per) cu.t = tma_tile_geom<BN>(g, cu.w / ncolt, cu.w % ncolt);
      continue;
    }
    if (cu.half == 0 ? cu.i < cu.t.nchP : cu.i < cu.t.nchQ) return;
    ++cu.half;
  }
}

// Product h.p of a fixed step for every tile: blockIdx.x, blockIdx.x +
// gridDim.x, ... of the product's row tile x column tile grid (column tile
// fastest: CTAs that read the same coupling rows run side by side).  Lane 0
// of warp 0 issues the copies: the first NS - 1 chunks up front, then one
// chunk into the slot of chunk c - 1 each time its warp has finished chunk c
// (so it waits, if at all, only for warps a whole chunk behind).
template <int BN, int NS>
__global__ void __launch_bounds__(BTHREADS, (BN <= 32 ? 2 : 1))
    k_horner_tma(const __grid_constant__ HornerTmaArgs h) {
  constexpr int WGM = Tile<BN>::WGM, WMT = Tile<BN>::WMT, WNT = Tile<BN>::WNT;
  constexpr int SLOT = tma_slot_doubles<BN>();
  constexpr uint32_t SLOT_TX = SLOT * 8;
  static_assert(NS >= 2, "ring");
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  __shared__ __align__(8) uint64_t full[NS], empty[NS];
  __shared__ int meta[NS];
  __shared__ int s_dead;
  __shared__ double red[BM][BN / 2];
  double* ring =
      reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(tsm_raw) + 1023) & ~uintptr_t(1023));
  const StageArgs& a = h.a;
  const Geometry& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = h.p;
  const int ncolt = h.ncolt;
  const int per = a.nrowtiles * ncolt;
  const bool issuer = threadIdx.x == 0;
  if (issuer) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kTmaConsumerWarps);
    }
    s_dead = 0;
    fence_mbar_init();
  }
  __syncthreads();
  pdl_trigger();
  pdl_wait();   // the previous product's Y, the step's fields and norms

  // ---------------- issuing lane ----------------
  TmaCursor cu;
  cu.w = blockIdx.x;
  cu.i = 0;
  cu.half = 0;
  cu.it = 0;
  cu.ended = false;
  const CUtensorMap* mapY = h.maps + 2 * g.nblk + (p & 1);
  auto issue_next = [&]() {
    if (cu.ended || cu.w >= per) return;
    const uint32_t slot = cu.it % NS;
    if (!ring_wait(&empty[slot], ((cu.it / NS) & 1) ^ 1, &s_dead, h.status, h.wait_ns)) {
      cu.ended = true;
      return;
    }
    double* As = ring + slot * SLOT;
    double* Bs = As + BM * BK;
    const int k0 = cu.i * BK;
    meta[slot] = cu.w;
    mbar_arrive_expect_tx(&full[slot], SLOT_TX);
    if (cu.half == 0) {
      const CUtensorMap* mp = h.maps + (cu.t.L - 1);
#pragma unroll
      for (int b = 0; b < BM / 16; ++b)
        tma_load_2d(As + b * 512, mp, &full[slot], cu.t.r0 + 16 * b, k0);
    } else {
      const CUtensorMap* mq = h.maps + g.nblk + cu.t.L;
#pragma unroll
      for (int j = 0; j < BK / 16; ++j)
        tma_load_2d(As + j * 1024, mq, &full[slot], k0 + 16 * j, cu.t.r0);
    }
    const int yrow = (cu.half == 0 ? g.state_off[cu.t.L - 1] : g.state_off[cu.t.L + 1]) + k0;
#pragma unroll
    for (int j = 0; j < BN / 16; ++j)
      tma_load_2d(Bs + j * 512, mapY, &full[slot], cu.t.c0 + 16 * j, yrow);
    ++cu.it;
    ++cu.half;
    cursor_seek<BN>(cu, g, ncolt, per);
  };
  if (issuer) {
    if (cu.w < per) cu.t = tma_tile_geom<BN>(g, cu.w / ncolt, cu.w % ncolt);
    cursor_seek<BN>(cu, g, ncolt, per);
    for (int k = 0; k < NS - 1; ++k) issue_next();
  }
  __syncwarp();   // (warp-synchronous instructions follow: reconverge warp 0)

  // ---------------- consumers (every warp) ----------------
  const int wm = warp % WGM, wn = warp / WGM;
  const int gq = lane >> 2, tq = lane & 3;
  const double qsign = (a.gauge == 1) ? -1.0 : 1.0;
  // fragment offsets, fixed for the whole launch
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
  uint32_t it = 0;
  for (int w = blockIdx.x; w < per; w += gridDim.x) {
    // the slot's tile must be this one (a mismatch would be a defect of the
    // issue order: reported, never run)
    const uint32_t slot0 = it % NS;
    const bool got = ring_wait(&full[slot0], (it / NS) & 1, &s_dead, h.status, h.wait_ns);
    __syncwarp();
    const bool bad = got && meta[slot0] != w;
    if (bad) atomicOr(h.status, ST_BAD_LAUNCH);
    if (consumers_any(!got || bad)) break;
    const TmaTileGeom t = tma_tile_geom<BN>(g, w / ncolt, w % ncolt);
    const int wrows = t.nL - t.r0 - wm * (WMT * 16);
    const int mt_lim = wrows <= 0 ? 0 : min(WMT, (wrows + 15) / 16);
    double accP[WMT][WNT][4], accQ[WMT][WNT][4];
#pragma unroll
    for (int i = 0; i < WMT; ++i)
#pragma unroll
      for (int j = 0; j < WNT; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) accP[i][j][v] = accQ[i][j][v] = 0.0;
    const int nsup = max(t.nchP, t.nchQ);
    bool first = true;
    for (int i = 0; i < nsup; ++i) {
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const bool isP = half == 0;
        if (isP ? i >= t.nchP : i >= t.nchQ) continue;
        const uint32_t slot = it % NS;
        // (a wait that gives up leaves garbage in this tile; the raised
        // status fails the call and the next tile's vote stops the CTA)
        if (!first) ring_wait(&full[slot], (it / NS) & 1, &s_dead, h.status, h.wait_ns);
        __syncwarp();
        first = false;
        const double* As = ring + slot * SLOT;
        const double* Bs = As + BM * BK;
        const int krem = (isP ? t.KP : t.KQ) - i * BK;
        const int nks = min(BK / 8, (krem + 7) / 8);
        if (isP)
          tma_chunk<BN, true>(As, Bs, oP, oB, nks, mt_lim, accP);
        else
          tma_chunk<BN, false>(As, Bs, oQ, oB, nks, mt_lim, accQ);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
        ++it;
        if (issuer) issue_next();
        __syncwarp();
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
      const double vs = ps.vscale, gm = ps.hg;
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
              const double nq = a.nrm[q];
              const double2 z = ps.Yin[idx];
              x = make_double2(z.x / nq, z.y / nq);
              a.Xw[idx] = x;
              wre = vs * (accr / nq);
              wim = vs * (acci / nq);
              v = make_double2(vs * x.x, vs * x.y);
            } else {
              wre = vs * accr;
              wim = vs * acci;
              const double2 v0 = ps.Yin[idx];
              v = make_double2(vs * v0.x, vs * v0.y);
              x = a.X[idx];
            }
            const double e = a.eps[i];
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
            double s[8];
#pragma unroll
            for (int gg = 0; gg < 8; ++gg)
              s[gg] = (0.0 + red[16 * m + gg][tid]) + red[16 * m + gg + 8][tid];
            const double tm = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
            ns = (m == 0) ? tm : ns + tm;
          }
          a.normpart[(long long)rtile * a.ldc + q] = ns;
        }
      }
      // red is rewritten by the next tile only after this barrier
      named_bar_sync(kTmaBarId, kTmaConsumerThreads);
    }
  }
  // drain (a CTA that gave up): the copies of the last slots issued land
  // before the CTA's shared memory goes away
  if (issuer) {
    const uint32_t first = cu.it > (uint32_t)NS ? cu.it - NS : 0u;
    for (uint32_t j = first; j < cu.it; ++j) {
      int never = 0;   // wait even when the CTA is dead, still bounded
      ring_wait(&full[j % NS], (j / NS) & 1, &never, h.status, h.wait_ns);
    }
  }
  __syncwarp();
  __syncthreads();
}

template <int BN, int NS>
cudaError_t launch_horner_tma_tile(cudaStream_t st, const HornerTmaArgs& h, int sms) {
  static int per_sm = 0;   // resident CTAs per SM (the same on every B200)
  if (per_sm == 0) {
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_horner_tma<BN, NS>, BTHREADS, tma_smem<BN, NS>());
    if (e != cudaSuccess) {
      per_sm = 0;
      return e;
    }
  }
  const int items = h.a.nrowtiles * h.ncolt;
  const int grid = std::max(1, std::min(items, std::max(per_sm, 1) * sms));
  return mpc_launch_pdl(k_horner_tma<BN, NS>, dim3(grid), dim3(BTHREADS), tma_smem<BN, NS>(),
                        st, h);
}

// TMA tile shapes: {column tile width, ring slots}.
struct TmaShape {
  int bn, ns;
};
constexpr TmaShape kTmaShapes[] = {{32, 4}, {64, 6}};
constexpr int kNumTmaShapes = sizeof(kTmaShapes) / sizeof(kTmaShapes[0]);

inline cudaError_t launch_horner_tma_shape(cudaStream_t st, int shape, const HornerTmaArgs& h,
                                           int sms) {
  return shape == 0 ? launch_horner_tma_tile<32, 4>(st, h, sms)
                    : launch_horner_tma_tile<64, 6>(st, h, sms);
}

inline cudaError_t set_tma_attrs() {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_horner_tma<32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tma_smem<32, 4>())) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(k_horner_tma<64, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              tma_smem<64, 6>());
}

}  // namespace
