// Internal interface of the blockSize-64 topology encoder (not part of the C ABI).
#pragma once
#include "tsz_codec.h"

namespace tsz {

struct Enc64Args {
  const float *data;            // the field, 16-byte aligned
  unsigned long long n;
  double inv;                   // 1 / (double)eb
  Geom g;
  unsigned char *out;           // payload base (stream + 8)
  unsigned long long out_cap;
  unsigned long long *blk_off;  // per-block payload offsets (optional)
  TileDesc *desc;               // zeroed, one per tile
  unsigned *tile_ctr;           // zeroed
  unsigned long long tile_lo;   // tiles [tile_lo, tile_hi) of this launch (tile_hi 0: all)
  unsigned long long tile_hi;
  int *err;                     // status word
  unsigned long long *total;    // [payload bytes, cps, extrema]
  uint2 *cp_out;                // critical-point pairs {value code, extremum index or ~0}
  unsigned long long cp_cap;
  int spin_limit;               // look-back polls before giving up (0: default)
  unsigned long long base;      // global index of local element 0 (a slab of a larger field; 0 otherwise):
                                // tiles, blocks and outputs are local, classification and loads use
                                // base + local through data (indexed by global element)
};

// The fused topology encoder with pairs output applies to blockSize 64 and a
// 16-byte aligned field; its tiles are the general encoder's (2048 elements).
bool enc64_applies(const EncArgs &a, int mode);
// Launches it over the tiles of a (persistent grid sized by occupancy).
cudaError_t launch_enc64_from(const EncArgs &a, cudaStream_t s, int sm_count);
cudaError_t launch_enc64_args(const Enc64Args &a, cudaStream_t s, int sm_count);
unsigned long long enc64_tiles(unsigned long long n);

// Bounded-wait checks (tests): a look-back whose predecessor never
// publishes, and a grid barrier that one CTA never reaches.  Each returns 0
// when the probe ran, with the status word it ended with and its device time.
int selftest_lookback(int spin_limit, int *status, float *ms);
int selftest_grid_barrier(int spin_limit, int *status, float *ms);

}  // namespace tsz
