// rhs_stream.cuh -- the dipole-coupling pass of one right-hand-side
// evaluation, streaming every dipole block through shared memory once.
//
// Replaces the 4 strided cblas_dgemv calls per dipole block of
// MatVecV/MatVecL::operator() (src/tdse/tdse.cpp:28-68, :99-139), which read
// each block four times (Re/Im x D/D^T).  Here each element D[r][c] of block
// L is read once from HBM and used twice:
//   row partial  P_row[r] += D[r][c] * y_{L+1}[c]   (D_L y_{L+1} -> block L)
//   col partial  P_col[c] += D[r][c] * y_L[r]       (D_L^T y_L   -> block L+1)
// with y complex and D real, 4 DFMA per element.
//
// Layout: one persistent CTA per SM.  Warp 8 is the producer: one lane
// issues 2-D TMA loads of 16x256 tiles (with an L2 evict-first hint: the
// blocks are streamed once per pass) plus a 1-D bulk copy of the tile's 16
// stage-vector rows into a kStages-deep shared-memory ring (full/empty
// mbarriers).  Warps 0-7 consume: warp w takes rows 2w and 2w+1
// of each tile; lane l holds the 8 columns {64j + 2l, 64j + 2l + 1}, j<4, of
// the current strip.
//   - Row partials are complete for the strip after a 6-shuffle
//     reduce-scatter across the warp; they are staged in shared memory (two
//     buffers of kRpRows rows) and written to RP[strip][row] by one bulk
//     store per run of consecutive rows.
//   - Column partials accumulate in registers while the CTA walks down a
//     strip; when the strip (or the CTA's range) ends, the 8 warps' partials
//     are summed in shared memory (warp order 0..7) and stored as one slot
//     CP[slot][0..255].
// Every output is written by exactly one thread in a fixed order, so repeated
// runs give identical bits.
#pragma once
#include <cuda.h>

#include "dev_util.cuh"
#include "plan.h"
#include "stream_types.h"

namespace mpc {


__device__ __forceinline__ double2 ld_y(const double2* y, int idx) {
  return __ldg(y + idx);
}

__global__ void __launch_bounds__(kStreamThreads, 1)
    k_rhs_stream(const __grid_constant__ StreamArgs a, const __grid_constant__ TmapSet tm) {
  extern __shared__ __align__(1024) unsigned char smem[];
  double* tiles = reinterpret_cast<double*>(smem);
  double2* yrows = reinterpret_cast<double2*>(smem + kStages * kTileBytes);
  double2* red = reinterpret_cast<double2*>(smem + kStages * (kTileBytes + kYRowBytes));
  double2* rpbuf =
      reinterpret_cast<double2*>(smem + kStages * (kTileBytes + kYRowBytes) + kRedBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * (kTileBytes + kYRowBytes) +
                                               kRedBytes + kRpStageBytes);
  uint64_t* empty = full + kStages;

  const Geometry& g = a.g;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int t_begin = (int)((long long)g.ntiles * blockIdx.x / gridDim.x);
  const int t_end = (int)((long long)g.ntiles * (blockIdx.x + 1) / gridDim.x);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();
  pdl_trigger();
  if (t_begin >= t_end) {
    pdl_wait();
    return;
  }

  if (warp == kConsumerWarps) {
    // ---------------- producer ----------------
    if (lane != 0) {
      pdl_wait();
      return;
    }
    const uint64_t stream_policy = make_evict_first_policy();
    const uint64_t keep_policy = make_evict_last_policy();
    const int keep_end = t_begin + (int)(a.keep_frac * (float)(t_end - t_begin));
    // The dipole blocks do not change between launches: the first ring's
    // worth of tiles is requested before waiting for the previous kernel;
    // their stage-vector rows (written by that kernel) only after it.
    const int pre = (t_end - t_begin < kStages) ? (t_end - t_begin) : kStages;
    for (int i = 0; i < pre; ++i) {
      int b, s, rt;
      decode_tile(g, t_begin + i, b, s, rt);
      mbar_arrive_expect_tx(&full[i], kTileBytes + kYRowBytes);
      tma_load_2d_hint(tiles + i * (kTileR * kStripW), &tm.m[b], &full[i], s * kStripW,
                       rt * kTileR, t_begin + i < keep_end ? keep_policy : stream_policy);
    }
    pdl_wait();
    int issued = 0;
    for (int t = t_begin; t < t_end; ++t, ++issued) {
      const int stage = issued % kStages;
      const int round = issued / kStages;
      int b, s, rt;
      decode_tile(g, t, b, s, rt);
      if (issued >= pre) {
        if (!mbar_wait_bounded(&empty[stage], (round - 1) & 1, a.status)) break;
        mbar_arrive_expect_tx(&full[stage], kTileBytes + kYRowBytes);
        tma_load_2d_hint(tiles + stage * (kTileR * kStripW), &tm.m[b], &full[stage],
                         s * kStripW, rt * kTileR, t < keep_end ? keep_policy : stream_policy);
      }
      // the tile's 16 rows of the stage vector (the vector carries a zeroed
      // tail of kVecPad entries, so the last tile never reads past it)
      bulk_load(yrows + stage * kTileR, a.y + g.blk[b].row_off + rt * kTileR, kYRowBytes,
                &full[stage]);
    }
    // Do not leave while a load is in flight: wait until every issued tile
    // was released by the consumers, or, if they gave up, until it landed.
    for (int i = (issued > kStages ? issued - kStages : 0); i < issued; ++i) {
      const int stage = i % kStages;
      const int round = i / kStages;
      if (!mbar_wait_bounded(&empty[stage], round & 1, a.status))
        mbar_wait_bounded(&full[stage], round & 1, a.status);
    }
    return;
  }

  // ---------------- consumers ----------------
  pdl_wait();
  double2 ycol[8];
  double2 cacc[8];
  int cur_b = -1, cur_s = -1;
  int slot = a.cta_slot0[blockIdx.x] - 1;
  const int ctid = threadIdx.x;  // 0..255 among consumers

  auto flush_cols = [&](int b) {
    // warp partials -> shared, then a fixed-order sum over warps
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      red[warp * kStripW + 64 * j + 2 * lane] = cacc[2 * j];
      red[warp * kStripW + 64 * j + 2 * lane + 1] = cacc[2 * j + 1];
    }
    named_bar_sync(1, kConsumerWarps * 32);
    double2 acc = red[ctid];
#pragma unroll
    for (int w = 1; w < kConsumerWarps; ++w) {
      const double2 v = red[w * kStripW + ctid];
      acc.x += v.x;
      acc.y += v.y;
    }
    a.CP[(long long)slot * kStripW + ctid] = acc;
    named_bar_sync(1, kConsumerWarps * 32);
    (void)b;
  };

  // Row partials of the current run of consecutive rows [seg_r0, seg_r0 +
  // seg_n) of strip seg_s of block seg_b, staged in rpbuf[rp_cur]; flushed by
  // one bulk store when the run ends or the buffer is full.  The store of
  // the other buffer must have read its rows before that buffer is reused.
  int rp_cur = 0, seg_b = -1, seg_s = 0, seg_r0 = 0, seg_n = 0;
  auto flush_rows = [&]() {
    if (seg_n == 0) return;
    fence_proxy_async_smem();
    named_bar_sync(2, kConsumerWarps * 32);
    if (ctid == 0) {
      const BlockGeom& sb = g.blk[seg_b];
      const int nv = min(seg_n, sb.nrow - seg_r0);  // rows past the block's end are not stored
      bulk_store(a.RP + sb.rp_off + (long long)seg_s * sb.nrow + seg_r0, rpbuf + rp_cur * kRpRows,
                 (uint32_t)nv * 16u);
      bulk_commit();
      bulk_wait_read<1>();
    }
    named_bar_sync(2, kConsumerWarps * 32);
    rp_cur ^= 1;
    seg_n = 0;
  };

  // After a timed-out wait the warp keeps walking its tiles without reading
  // shared memory, so that every consumer warp still reaches each named
  // barrier; the raised status makes the host discard the result.
  bool dead = false;
  int it = 0;
  for (int t = t_begin; t < t_end; ++t, ++it) {
    int b, s, rt;
    decode_tile(g, t, b, s, rt);
    const BlockGeom& bg = g.blk[b];
    if (b != seg_b || s != seg_s || seg_n == kRpRows || rt * kTileR != seg_r0 + seg_n) {
      flush_rows();
      seg_b = b;
      seg_s = s;
      seg_r0 = rt * kTileR;
    }
    const int rp_local = rt * kTileR - seg_r0;  // this tile's first row in the buffer
    seg_n += kTileR;
    if (b != cur_b || s != cur_s) {
      if (cur_b >= 0) flush_cols(cur_b);
      ++slot;
      cur_b = b;
      cur_s = s;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = s * kStripW + 64 * j + 2 * lane + e;
          ycol[2 * j + e] = (c < bg.ncol) ? ld_y(a.y, bg.col_off + c) : make_double2(0.0, 0.0);
          cacc[2 * j + e] = make_double2(0.0, 0.0);
        }
      }
    }
    const int stage = it % kStages;
    const int round = it / kStages;
    if (!dead && !mbar_wait_bounded(&full[stage], round & 1, a.status)) dead = true;
    // rows past the block's end meet zero-filled dipole rows, so their
    // (finite) stage-vector entries contribute nothing
    const double2 yr0 = dead ? make_double2(0.0, 0.0) : yrows[stage * kTileR + 2 * warp];
    const double2 yr1 = dead ? make_double2(0.0, 0.0) : yrows[stage * kTileR + 2 * warp + 1];
    const double* T = tiles + stage * (kTileR * kStripW);
    const double* T0 = T + (2 * warp) * kStripW + 2 * lane;
    const double* T1 = T0 + kStripW;
    double2 ra = make_double2(0.0, 0.0), rb = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double2 d0 = dead ? make_double2(0.0, 0.0) : *reinterpret_cast<const double2*>(T0 + 64 * j);
      const double2 d1 = dead ? make_double2(0.0, 0.0) : *reinterpret_cast<const double2*>(T1 + 64 * j);
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
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[stage]);

    // reduce-scatter of (ra.x, ra.y, rb.x, rb.y) over the 32 lanes:
    // lane 0 -> ra.x, lane 8 -> ra.y, lane 16 -> rb.x, lane 24 -> rb.y
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
      double* rp = reinterpret_cast<double*>(rpbuf + rp_cur * kRpRows + rp_local + 2 * warp +
                                             (hi16 ? 1 : 0));
      rp[hi8 ? 1 : 0] = z;
    }
  }
  if (cur_b >= 0) flush_cols(cur_b);
  flush_rows();
  if (ctid == 0) bulk_wait<0>();  // the last stores complete before the grid does
}

}  // namespace mpc
