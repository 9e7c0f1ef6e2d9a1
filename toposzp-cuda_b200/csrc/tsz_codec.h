// Internal interface of the codec kernels (not part of the C ABI).
#pragma once
#include "tsz_common.cuh"

namespace tsz {

// kEncIntTypes: int values with per-element 2-bit tags (pre-quantized fields)
// kEncQuant: a float field quantized, no tags (the plain codec's blocks)
enum EncMode { kEncClassify = 0, kEncTypes = 1, kEncInts = 2, kEncIntTypes = 3, kEncQuant = 4 };

// whether the blocks of a mode carry 2-bit tags
__host__ __device__ constexpr bool mode_tags(int mode) { return mode != kEncInts && mode != kEncQuant; }
enum CpMode { kCpNone = 0, kCpRecords = 1, kCpPairs = 2 };

struct EncArgs {
  const float *data;            // float field (kEncClassify / kEncTypes / kEncQuant)
  const int *ints;              // int values (kEncInts / kEncIntTypes)
  const unsigned char *types;   // per-element types 0..3 (kEncTypes / kEncIntTypes)
  unsigned long long n;
  int B;
  float eb;
  double inv;
  Geom g;                       // geometry for in-kernel classification
  unsigned char *out;           // payload base (stream + 8-byte header)
  unsigned long long out_cap;
  unsigned long long *blk_off;  // per-block payload offsets (optional)
  TileDesc *desc;               // zeroed, one per tile
  unsigned *tile_ctr;           // zeroed
  unsigned long long tile_lo;   // tiles [tile_lo, tile_hi) of this launch (tile_hi 0: all)
  unsigned long long tile_hi;
  int *err;                     // status word
  unsigned long long *total;    // [payload bytes, cps, extrema]
  int cp_mode;                  // CpMode (kEncClassify only)
  void *cp_out;                 // CriticalPoint / CriticalPoint3D records or uint2 pairs
  unsigned long long cp_cap;
  unsigned img_stride;          // octet encoder: bytes of one of its two tile images (0: one image, no pipelining)
};

struct DecArgs {
  const unsigned char *payload; // stream payload (after the offset table)
  unsigned long long payload_len;
  const unsigned long long *blk_off;  // per-block payload offsets
  unsigned long long n;
  int B;
  float eb;
  float *out_f;                 // decoded floats (topology stream)
  int *out_i;                   // decoded ints (sort-position stream)
  int *fn_i;                    // 2-bit tags as int (optional)
  unsigned char *fn_u8;         // 2-bit tags as bytes (optional)
  int *err;
  unsigned long long *ext_count;  // optional: number of type-1/2 tags
  unsigned long long img_cap;   // set by the launcher
  int cpu_layout;               // OpenMP layout: a one-element block carries its (zero) bit-count byte
};

// bytes of one block in the CUDA layout, or in the OpenMP layout (cpu), where
// a one-element block also carries a bit-count byte
__host__ __device__ __forceinline__ uint32_t block_bytes_layout(uint32_t n, uint32_t bc, bool tags, bool cpu) {
  return (cpu && n == 1u) ? 5u + (tags ? 1u : 0u) : block_bytes(n, bc, tags);
}

int enc_tile_blocks(int B);   // codec blocks per encoder tile (look-back granularity)
int octet_group(int B);       // lanes per codec block in the octet kernels (B <= 256)
int kmax_for(int B);
int bpw_for(int kmax);
int tile_blocks_for(int B);
size_t enc_smem_bytes(int B, bool tags);
size_t dec_smem_bytes(int B, bool tags);
cudaError_t launch_encode(int mode, const EncArgs &a, cudaStream_t s, int grid);
cudaError_t launch_decode(bool tags, DecArgs a, cudaStream_t s);

}  // namespace tsz
