// Internal operators shared by the API layer (not part of the C ABI).
#pragma once
#include "tsz_codec.h"
#include "tsz_runtime.h"

namespace tsz {

// Geometry from extents (nd = 2: rows, cols; nd = 3: d1, d2, d3).
Geom make_geom(int nd, long long a, long long b, long long c);

// Largest element count a field may have (2^40): larger products, and
// products of the extents that overflow, are rejected as invalid geometry.
constexpr unsigned long long kMaxElements = 1ull << 40;

// Validates a C-ABI geometry (nd 2 or 3, positive extents, element count
// below kMaxElements without overflow) and fills the kernel geometry.
bool geom_elements(const szp_b200_geom &g, unsigned long long *n, Geom *out);

// Largest topology stream (header, blocks with tags, slack) of n elements.
size_t topo_stream_bound(unsigned long long n, int B);

// Block size inside the reference's range [1, 257]; sets the error otherwise.
bool valid_block_size(int B, const char *fn);

// Types (1..3) of a critical-point list into a zeroed byte-per-element array:
// records of `stride` ints (x, y, type, ... in 2D; x, y, z, type, ... in 3D),
// points outside the grid or with other types skipped.  Enqueued on s.
cudaError_t launch_mark_types(const int *d_cps, int stride, long long count, const Geom &g, unsigned long long n,
                              unsigned char *d_types, cudaStream_t s);

// Runs one encoder pass on ctx->stream and waits for it.
//   out: payload destination (stream base + 8); the 8-byte header is written here too.
//   totals_out (host): payload bytes, cps, extrema.
int encode_pass(szp_b200_ctx *ctx, int mode, const float *d_data, const int *d_ints,
                const unsigned char *d_types, unsigned long long n, int B, float eb,
                const Geom &g, unsigned char *d_stream, unsigned long long stream_cap,
                unsigned long long *d_blk_off, int cp_mode, void *d_cp, unsigned long long cp_cap,
                unsigned long long totals_out[3]);

// Dense rank of every extremum inside its quantization bin.
//   pairs[k] = (orderable value code, extremum index or kNoExtremum), k < K
//   writes sp[e] for every extremum e < E.  bins come from the value
//   (bin = quant_bin(value, eb)); mode_given_bins = true uses bins[k] instead.
int rank_positions(szp_b200_ctx *ctx, const uint2 *d_pairs, const int *d_bins,
                   unsigned long long K, unsigned long long E, float eb, int *d_sp);

// Post-processing of a decoded field in place (serial raster semantics of the
// reference drivers).  types: u8 per element (or int when types_i != null).
int postprocess(szp_b200_ctx *ctx, float *d_data, const float *d_orig,
                const unsigned char *d_types_u8, const int *d_types_i, const int *d_sp,
                unsigned long long n_sp, const Geom &g, float eb, int axis_stencil,
                int *restored_out);

size_t rank_scratch_bytes(unsigned long long K, int sm_count);

// Ranks of F segments in one pass (h_seg_K: records per segment, host);
// bins disjoint across segments.
int rank_positions_seg(szp_b200_ctx *ctx, const uint2 *d_pairs, const int *d_bins,
                       const unsigned long long *h_seg_K, int F, int *d_sp);
size_t rank_scratch_bytes_seg(unsigned long long K, int F, int sm_count);
size_t post_scratch_bytes(unsigned long long n);
int compact_extrema(szp_b200_ctx *ctx, const int *d_cps, int stride, unsigned long long K, int *d_sp,
                    unsigned long long *E_out);
unsigned long long *post_words(szp_b200_ctx *ctx, unsigned long long n);
int postprocess_with(szp_b200_ctx *ctx, float *d_data, const float *d_orig, unsigned char *d_T,
                     unsigned long long *d_S, TileDesc *desc, const int *d_sp,
                     unsigned long long n_sp, const Geom &g, float eb, int axis_stencil,
                     int *restored_out);

// Block offsets of a single-chunk stream, parsed on the device (enqueued on
// ctx->stream, no sync).  d_payload: the bytes after the 8-byte offset table,
// buf_len of them.  Element count n, or read on the device from d_n when it is
// not null.  ref_bound adds the reference's validation bound (8n+1024 with
// tags, 4n+4 without) to the buffer bound.  Writes the first ceil(n/B)
// payload offsets to d_offs and d_status[0] = payload length + 1 on success
// (0 when the walk failed), d_status[1] = nonzero on a malformed block.
size_t parse_scratch_bytes(unsigned long long buf_len, int B, bool tags);
// cpu: the OpenMP layout, whose one-element blocks carry a bit-count byte.
int parse_stream(szp_b200_ctx *ctx, Arena &A, const unsigned char *d_payload, unsigned long long buf_len,
                 unsigned long long n, const unsigned long long *d_n, int B, bool tags, bool ref_bound,
                 unsigned long long *d_offs, unsigned long long *d_status, bool cpu = false);

// Fused decompression (+ post-processing) of device streams; d_topo / d_sort
// point 8 bytes before their payloads.  With d_blk_index null the block
// offsets are parsed on the device (single-chunk streams).  cpu_layout: the
// topology stream's one-element blocks carry a bit-count byte (OpenMP layout).
// sort_count: entries of the sort-position stream when the caller knows it
// (a container header), else one per extremum tag.
int decompress_dev_impl(szp_b200_ctx *ctx, const unsigned char *d_topo, size_t topo_bytes,
                        const unsigned char *d_sort, size_t sort_bytes,
                        const uint64_t *d_blk_index, szp_b200_geom geom, float absErrBound,
                        int blockSize, float *d_out, unsigned char *d_types, int postprocess,
                        bool ref_bound, bool *parse_failed, cudaEvent_t sort_ready = nullptr,
                        bool cpu_layout = false, unsigned long long sort_count = ~0ull);

// Grows a workspace so that compressing or decompressing (with
// post-processing) a field of n elements allocates nothing more.
int ctx_reserve_for(szp_b200_ctx *ctx, unsigned long long n, int B);

}  // namespace tsz
