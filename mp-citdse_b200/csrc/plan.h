// plan.h -- geometry shared by the host planner and the kernels.
//
// Dipole block L couples angular-momentum block L (rows, n_L states) to block
// L+1 (columns, n_{L+1} states).  On the device each block is stored
// row-major with a padded pitch (a multiple of 32 doubles, 256 B) so that
// 2-D TMA can address it; the padding is never read (tensor-map extents are
// the true sizes, out-of-range elements arrive as zeros).
//
// The streaming right-hand side cuts every block into tiles of kTileR rows
// by kStripW columns.  Tiles are numbered block by block, and inside a block
// strip by strip (a strip is kStripW consecutive columns), going down the
// strip, so that consecutive tiles share their columns.  CTA c of G takes the
// contiguous tile range [T*c/G, T*(c+1)/G).
#pragma once
#include <cstdint>

namespace mpc {

constexpr int kMaxBlocks = 16;      // angular-momentum blocks L = 0..15
constexpr int kStripW = 256;        // tile width (columns, doubles)
constexpr int kTileR = 16;          // tile height (rows)
constexpr int kStages = 4;          // TMA ring depth
constexpr int kConsumerWarps = 8;   // warps that compute; one more issues TMA
constexpr int kStreamThreads = (kConsumerWarps + 1) * 32;
constexpr int kTileBytes = kTileR * kStripW * 8;
constexpr int kYRowBytes = kTileR * 16;          // the tile's stage-vector rows
constexpr int kRedBytes = kConsumerWarps * kStripW * 16;
constexpr int kRpRows = 512;        // row partials staged per bulk store
constexpr int kRpStageBytes = 2 * kRpRows * 16;
constexpr int kStreamSmem =
    kStages * (kTileBytes + kYRowBytes) + kRedBytes + kRpStageBytes + 2 * kStages * 8;
constexpr int kVecPad = kTileR;     // zeroed tail of every stage vector (row bulk copies)
constexpr int kNumStages = 13;      // RKF78 stages
constexpr int kCombineThreads = 256;
constexpr int kCombineLanes = 4;    // threads cooperating on one coefficient

struct BlockGeom {
  int nrow, ncol;        // n_L, n_{L+1}
  int row_off, col_off;  // state offsets of block L and block L+1
  int pitch;             // device row pitch in doubles
  int nstrips;           // ceil(ncol / kStripW)
  int nrtiles;           // ceil(nrow / kTileR)
  int tile0;             // first global tile number of this block
  int strip0;            // first global strip number of this block
  long long d_off;       // element offset of the block in the dipole buffer
  long long rp_off;      // complex offset of the block's row partials:
                         //   RP[rp_off + strip*nrow + row]
};

struct Geometry {
  int nblk;                    // number of dipole blocks (= L_max)
  int nstate_blk;              // number of state blocks (= L_max + 1)
  int ntot;                    // total states
  int ntiles;                  // total tiles over all dipole blocks
  int nstrips;                 // total strips over all dipole blocks
  int state_off[kMaxBlocks + 1];
  BlockGeom blk[kMaxBlocks];
};

// Locates global tile t: block b, strip s, row tile rt.
__host__ __device__ inline void decode_tile(const Geometry& g, int t, int& b, int& s, int& rt) {
  b = 0;
  while (b + 1 < g.nblk && t >= g.blk[b + 1].tile0) ++b;
  const int loc = t - g.blk[b].tile0;
  s = loc / g.blk[b].nrtiles;
  rt = loc - s * g.blk[b].nrtiles;
}

}  // namespace mpc
