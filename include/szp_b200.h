/*
 * szp_b200.h -- C ABI of the B200-native TopoSZp topology path.
 *
 * Part 1 re-exports the reference's topology entry points with identical
 * names, argument lists, struct layouts and byte-stream layout, so a caller
 * linked against the reference CUDA library can relink against
 * libtoposzp_b200.so unchanged.  Host pointers in, malloc'd host buffers out
 * (release them with free()), exactly as in the reference.
 *
 * Deviation: where the reference calls exit(EXIT_FAILURE) (bad blockSize or
 * dimensions, any CUDA error), these functions return NULL / a zero count and
 * record a message that szp_b200_last_error() returns.
 *
 * Part 2 adds device-pointer entry points (fused compress / decompress /
 * post-processing on a caller stream) that have no counterpart in the
 * reference.
 */
#ifndef SZP_B200_H
#define SZP_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SZP_B200_API __attribute__((visibility("default")))
#else
#define SZP_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* ABI structs (SZp/include/szp_float.h:20-25, SZp/include/szp_topology_3d.h:22-27) */
/* ------------------------------------------------------------------ */
#ifndef _szp_Float_H
typedef struct {
    int x, y;
    int type;            /* 1 max, 2 min, 3 saddle */
    int quantized_bin;
    int sort_position;
} CriticalPoint;
#endif

#ifndef _SZP_TOPOLOGY_3D_H
typedef struct {
    int x, y, z;
    int type;
    int quantized_bin;
    int sort_position;
} CriticalPoint3D;
#endif

/* ------------------------------------------------------------------ */
/* Part 1: reference entry points                                      */
/* ------------------------------------------------------------------ */

/* replaces SZp/include/szp_cuda_topology.cuh:23-24 (szp_cuda_topology.cu:78) */
SZP_B200_API CriticalPoint *szp_cuda_find_critical_points(float *data, size_t *outCount,
                                              int rows, int cols, float absErrBound);

/* replaces SZp/include/szp_cuda_topology.cuh:30-32 (szp_cuda_topology.cu:195) */
SZP_B200_API void szp_cuda_sort_critical_points_by_original_data(CriticalPoint *critical_points,
                                                     size_t critical_count,
                                                     float *data, int cols);

/* replaces SZp/include/szp_cuda_topology.cuh:38-40 (szp_cuda_topology.cu:424) */
SZP_B200_API unsigned char *szp_cuda_compress_sort_positions(CriticalPoint *critical_points,
                                                 size_t critical_count,
                                                 size_t *outSize, int blockSize);

/* replaces SZp/include/szp_cuda_topology.cuh:46-50 (szp_cuda_topology.cu:683) */
SZP_B200_API unsigned char *szp_cuda_float_compress_randomaccess_topology_preserved(
    float *oriData, size_t *outSize, float absErrBound,
    size_t nbEle, int blockSize,
    CriticalPoint *critical_points, int critical_count,
    int rows, int cols);

/* replaces SZp/include/szp_cuda_topology_3d.cuh:16-18 (szp_cuda_topology_3d.cu:175) */
SZP_B200_API CriticalPoint3D *szp_cuda_find_critical_points_3d(float *data, size_t *outCount,
                                                    int d1, int d2, int d3,
                                                    float absErrBound);

/* replaces SZp/include/szp_cuda_topology_3d.cuh:20-22 (szp_cuda_topology_3d.cu:321) */
SZP_B200_API void szp_cuda_sort_critical_points_3d(CriticalPoint3D *critical_points,
                                       size_t critical_count,
                                       float *data, int d2, int d3);

/* replaces SZp/include/szp_cuda_topology_3d.cuh:24-26 (szp_cuda_topology_3d.cu:529) */
SZP_B200_API unsigned char *szp_cuda_compress_sort_positions_3d(CriticalPoint3D *critical_points,
                                                     size_t critical_count,
                                                     size_t *outSize, int blockSize);

/* replaces SZp/include/szp_cuda_topology_3d.cuh:28-32 (szp_cuda_topology_3d.cu:958) */
SZP_B200_API unsigned char *szp_cuda_float_compress_topology_3d(
    float *oriData, size_t *outSize, float absErrBound,
    size_t nbEle, int blockSize,
    CriticalPoint3D *critical_points, int critical_count,
    int d1, int d2, int d3);

/* replaces SZp/include/szp_cuda_topology_3d.cuh:34-38 (szp_cuda_topology_3d.cu:1066):
 * fp64 field, double quantization, three saddle-repair passes in q-space,
 * the fp32 path's stream format ([u64 0][blocks with 2-bit tags]). */
SZP_B200_API unsigned char *szp_cuda_double_compress_topology_3d(
    double *oriData, size_t *outSize, double absErrBound,
    size_t nbEle, int blockSize,
    CriticalPoint3D *critical_points, int critical_count,
    int d1, int d2, int d3);

/* replaces SZp/include/szp_cuda_decompress.cuh:63-65 (szp_cuda_decompress.cu:1074) */
SZP_B200_API void szp_cuda_float_decompress_randomaccess_topology_preserved(
    float **newData, size_t nbEle, float absErrBound, int blockSize,
    unsigned char *cmpBytes, int **FN);

/* replaces SZp/include/szp_cuda_decompress.cuh:71-72 (szp_cuda_decompress.cu:1165) */
SZP_B200_API int *szp_cuda_decompress_sort_positions(
    unsigned char *cmpBytes, size_t critical_count, int blockSize);

/* Plain (non-topology) codec.  Compressed stream: [T eb][u64 0][body], T the
 * element type; the decompressors take the stream after its T header, as the
 * reference's do.  blockSize 1..1025. */
/* replaces SZp/include/szp_cuda_compress.cuh:22 (szp_cuda_compress.cu:718) */
SZP_B200_API unsigned char *szp_cuda_float_compress_randomaccess(float *oriData, size_t *outSize,
                                                                 float absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:26 */
SZP_B200_API void szp_cuda_float_compress_randomaccess_arg(unsigned char *output, float *oriData, size_t *outSize,
                                                           float absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:30 */
SZP_B200_API unsigned char *szp_cuda_double_compress_randomaccess(double *oriData, size_t *outSize,
                                                                  double absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:34 */
SZP_B200_API void szp_cuda_double_compress_randomaccess_arg(unsigned char *output, double *oriData,
                                                            size_t *outSize, double absErrBound, size_t nbEle,
                                                            int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:40 */
SZP_B200_API unsigned char *szp_cuda_float_compress_threadblock(float *oriData, size_t *outSize,
                                                                float absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:44 */
SZP_B200_API void szp_cuda_float_compress_threadblock_arg(unsigned char *output, float *oriData, size_t *outSize,
                                                          float absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:48 */
SZP_B200_API unsigned char *szp_cuda_double_compress_threadblock(double *oriData, size_t *outSize,
                                                                 double absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:52 */
SZP_B200_API void szp_cuda_double_compress_threadblock_arg(unsigned char *output, double *oriData,
                                                           size_t *outSize, double absErrBound, size_t nbEle,
                                                           int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:58: q[0], q[i] - q[i-1] (malloc'd) */
SZP_B200_API int *szp_cuda_float_direct_predict_quantization(float *oriData, size_t *outSize, float absErrBound,
                                                             size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_compress.cuh:62 (the same result) */
SZP_B200_API int *szp_cuda_float_threadblock_predict_quantization(float *oriData, size_t *outSize,
                                                                  float absErrBound, size_t nbEle, int blockSize);
/* replaces SZp/include/szp_cuda_decompress.cuh:23 (szp_cuda_decompress.cu:990) */
SZP_B200_API float *szp_cuda_float_decompress_randomaccess(size_t nbEle, float absErrBound, int blockSize,
                                                           unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:27 */
SZP_B200_API void szp_cuda_float_decompress_randomaccess_arg(float *newData, size_t nbEle, float absErrBound,
                                                             int blockSize, unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:31 */
SZP_B200_API double *szp_cuda_double_decompress_randomaccess(size_t nbEle, double absErrBound, int blockSize,
                                                             unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:35 */
SZP_B200_API void szp_cuda_double_decompress_randomaccess_arg(double *newData, size_t nbEle, double absErrBound,
                                                              int blockSize, unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:43 */
SZP_B200_API float *szp_cuda_float_decompress_threadblock(size_t nbEle, float absErrBound, int blockSize,
                                                          unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:47 */
SZP_B200_API void szp_cuda_float_decompress_threadblock_arg(float *newData, size_t nbEle, float absErrBound,
                                                            int blockSize, unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:51 */
SZP_B200_API double *szp_cuda_double_decompress_threadblock(size_t nbEle, double absErrBound, int blockSize,
                                                            unsigned char *cmpBytes);
/* replaces SZp/include/szp_cuda_decompress.cuh:55 */
SZP_B200_API void szp_cuda_double_decompress_threadblock_arg(double *newData, size_t nbEle, double absErrBound,
                                                             int blockSize, unsigned char *cmpBytes);

/* ------------------------------------------------------------------ */
/* Part 2: additions (no reference counterpart)                        */
/* ------------------------------------------------------------------ */

/* Message of the last failure on this thread ("" when none). */
SZP_B200_API const char *szp_b200_last_error(void);

/* Library version string. */
SZP_B200_API const char *szp_b200_version(void);

/* Opaque, reusable device workspace (scratch buffers, stream, events). */
typedef struct szp_b200_ctx szp_b200_ctx;

/* Create / destroy a workspace on the current device.  stream may be 0. */
SZP_B200_API szp_b200_ctx *szp_b200_ctx_create(void *cuda_stream);
SZP_B200_API void szp_b200_ctx_destroy(szp_b200_ctx *ctx);

/* Device time of each stage of the last call on this workspace, measured
 * with CUDA events on the workspace stream.  Fills up to max entries and
 * returns how many stages the call had. */
SZP_B200_API int szp_b200_ctx_stage_times(szp_b200_ctx *ctx, const char **names, float *ms, int max);

/* Number of kernels this workspace has launched since it was created. */
SZP_B200_API unsigned long long szp_b200_ctx_launches(szp_b200_ctx *ctx);

/* Geometry of a field: nd = 2 (dims[0] rows, dims[1] cols) or nd = 3. */
typedef struct {
    int nd;
    int dims[3];
} szp_b200_geom;

/* Result of a fused compression, all sizes in bytes. */
typedef struct {
    size_t topo_bytes;      /* topology stream, header included */
    size_t sort_bytes;      /* sort-position stream, header included (0 if no extrema) */
    size_t cp_count;        /* critical points */
    size_t extrema_count;   /* maxima + minima */
} szp_b200_sizes;

/* Upper bounds of the two streams for n elements (for sizing buffers). */
SZP_B200_API size_t szp_b200_topo_bound(size_t n, int blockSize);
SZP_B200_API size_t szp_b200_sort_bound(size_t n, int blockSize);

/* Fused compression of a device-resident field: classify, rank, pack.
 *   d_data        device float[n]
 *   d_topo        device buffer >= szp_b200_topo_bound(n, B)
 *   d_sort        device buffer >= szp_b200_sort_bound(n, B)
 *   d_blk_index   optional device uint64[2 * ceil(n/B)]: payload offset of
 *                 every topology block, followed by the offsets of the
 *                 sort-position blocks; szp_b200_topo_decompress_dev reuses it
 * Synchronous on the workspace stream.  Returns 0 on success. */
SZP_B200_API int szp_b200_topo_compress_dev(szp_b200_ctx *ctx, const float *d_data,
                               szp_b200_geom geom, float absErrBound, int blockSize,
                               unsigned char *d_topo, unsigned char *d_sort,
                               uint64_t *d_blk_index, szp_b200_sizes *sizes);

/* Fused decompression + post-processing of device-resident streams.
 *   d_blk_index   block index written by szp_b200_topo_compress_dev, or NULL:
 *                 the block offsets of both streams are then parsed on the
 *                 device from the stream bytes (single-chunk streams, offset
 *                 table [0], as szp_cuda_* and szp_b200_* compressors write)
 *   d_topo/d_sort any alignment for blockSize <= 256, 4-byte aligned above
 *   d_out         device float[n] (output)
 *   d_types       optional device uint8[n] (2-bit tags, output)
 *   postprocess   0: raw decode only; 1: stencils + enforcement + RBF;
 *                 2: as 1 plus the 3D axis-pattern saddle stencil */
SZP_B200_API int szp_b200_topo_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_topo,
                                 size_t topo_bytes, const unsigned char *d_sort,
                                 size_t sort_bytes, const uint64_t *d_blk_index,
                                 szp_b200_geom geom, float absErrBound, int blockSize,
                                 float *d_out, unsigned char *d_types, int postprocess);

/* Host-buffer forms of the two calls above: the field and the streams live
 * in host memory (pinned memory gives full copy bandwidth); device staging
 * is kept in the workspace.  The decompressor finds the block offsets from
 * the stream bytes alone, as the reference decoder does. */
SZP_B200_API int szp_b200_topo_compress_host(szp_b200_ctx *ctx, const float *h_data,
                                szp_b200_geom geom, float absErrBound, int blockSize,
                                unsigned char *h_topo, size_t topo_cap,
                                unsigned char *h_sort, size_t sort_cap,
                                szp_b200_sizes *sizes);
SZP_B200_API int szp_b200_topo_decompress_host(szp_b200_ctx *ctx, const unsigned char *h_topo,
                                  size_t topo_bytes, const unsigned char *h_sort,
                                  size_t sort_bytes, szp_b200_geom geom, float absErrBound,
                                  int blockSize, float *h_out, int postprocess);

/* Post-processing of an already decoded field in place (device pointers).
 *   d_orig   raw decoded values (read only)
 *   d_types  int per element (FN) as returned by the reference decoder
 *   d_sp     decoded sort positions (E entries), may be NULL when E == 0 */
SZP_B200_API int szp_b200_topo_postprocess_dev(szp_b200_ctx *ctx, float *d_data, const float *d_orig,
                                  const int *d_types, const int *d_sp, size_t n_sp,
                                  szp_b200_geom geom, float absErrBound, int axis_stencil);

/* Topology report of a decompressed field against the original (device
 * pointers, both float[n]); the counts of the reference drivers' checks
 * (example/test_cuda_topology.cu:540-602, 636-660, 800-868 and
 * example/test_cuda_topology_3d.cu:636-730).  A critical point is
 * preserved when the decompressed field classifies the same point with the
 * same type; lost when it is a regular point there; changed otherwise; new
 * when the decompressed field has a critical point where the original has
 * none.  pairs / violations: adjacent interior pairs (+1 along each axis,
 * both points interior) whose original values differ, and those whose order
 * changed; [0] all, [1] at least one critical point, [2] both critical
 * points, [3] at least one extremum.  The reference accepts a run at
 * max_err <= 2 eb with more than 90 % of the critical points preserved.
 * Arrays indexed by type hold the total at [0] and type t at [t]. */
typedef struct {
    uint64_t orig_cps[4];
    uint64_t dec_cps[4];
    uint64_t preserved, lost, changed, new_cps;
    uint64_t lost_by_type[4];
    uint64_t pairs[4];
    uint64_t violations[4];
    uint64_t over_1eb;      /* |error| > 1.01 eb */
    uint64_t over_2eb;      /* |error| > 2 eb */
    double max_err;
} szp_b200_topo_report;

/* Synchronous on the workspace stream.  Returns 0 on success. */
SZP_B200_API int szp_b200_topo_check(szp_b200_ctx *ctx, const float *d_orig, const float *d_dec,
                                     szp_b200_geom geom, float absErrBound,
                                     szp_b200_topo_report *report);

/* ------------------------------------------------------------------ */
/* .SZp container and the OpenMP stream layouts                        */
/* ------------------------------------------------------------------ */
/* The container the reference's CPU drivers write and read
 * (example/testfloat_compress_fastmode1_topology.cc:105-125,
 * example/testfloat_decompress_fastmode1_topology.cc:720-805):
 *   [topology stream][sort-position stream][u64 topology size][u64 sort size]
 * with the streams in the reference's OpenMP layout
 * (SZp/src/szp_float.cc:522-865, 999-1318; SZp/src/szp_topology_3d.cc:253-632):
 *   topology       [u64 offset x T][blocks]
 *   sort positions [u64 E][u64 offset x T][blocks]   (absent when E == 0)
 * T = the writer's thread count; a one-element block carries its (zero)
 * bit-count byte.  Device pointers; synchronous on the workspace stream. */

/* Bytes a container of n elements may need with `threads` chunks. */
SZP_B200_API size_t szp_b200_container_bound(size_t n, int blockSize, int threads);

/* Container from the CUDA-layout streams of szp_b200_topo_compress_dev (the
 * bytes the reference's CPU compressor writes with `threads` OpenMP threads,
 * 1..128, for the same critical-point order).  extrema: sizes.extrema_count.
 * blockSize <= 256.  Returns 0 on success. */
SZP_B200_API int szp_b200_container_from_streams_dev(szp_b200_ctx *ctx, const unsigned char *d_topo,
                                                     size_t topo_bytes, const unsigned char *d_sort,
                                                     size_t sort_bytes, szp_b200_geom geom, int blockSize,
                                                     size_t extrema, int threads, unsigned char *d_out,
                                                     size_t out_cap, size_t *out_bytes);

/* Decompression (+ post-processing, as szp_b200_topo_decompress_dev) of a
 * container written by the reference's CPU path with any thread count, or
 * by the call above.  The thread counts of both streams are detected by the
 * reference's rule (SZp/include/szp_detect_threads.h:153-190, 282-309), every
 * chunk walked by the device parser.  blockSize <= 256. */
SZP_B200_API int szp_b200_container_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_in, size_t in_bytes,
                                                   szp_b200_geom geom, float absErrBound, int blockSize,
                                                   float *d_out, unsigned char *d_types, int postprocess);

/* The fp64 3D compression on device memory: d_data (nd 3 geometry), the
 * critical points on the device (d_cps, critical_count records; null when 0),
 * `passes` saddle-repair passes (the reference runs 3; 0..64).  Writes the
 * stream to d_out (out_cap >= szp_b200_topo_bound(n, blockSize)) and its
 * length to *out_len; with d_q non-null the repaired integers go there
 * (n ints) instead of workspace scratch.  Returns 0, or -1 with
 * szp_b200_last_error(). */
SZP_B200_API int szp_b200_double_compress_topology_3d_dev(szp_b200_ctx *ctx, const double *d_data,
                                                          szp_b200_geom geom, double absErrBound,
                                                          int blockSize, const CriticalPoint3D *d_cps,
                                                          size_t critical_count, int passes,
                                                          unsigned char *d_out, size_t out_cap,
                                                          size_t *out_len, int *d_q);
/* Device scratch the call above takes from the workspace. */
SZP_B200_API size_t szp_b200_f64_topo_scratch_bytes(size_t n, size_t critical_count, int blockSize);

/* Plain codec on device memory.  Bound of the whole stream ([T eb][u64 0]
 * [body]; is_double selects T), compression of n elements into d_out (random
 * access, or threadblock when threadblock != 0), and random-access
 * decompression of a single-chunk stream (d_in: the stream after its T header,
 * in_len bytes; block offsets parsed on the device).  Return 0 / -1. */
SZP_B200_API size_t szp_b200_plain_bound(size_t n, int blockSize, int is_double, int threadblock);
SZP_B200_API int szp_b200_plain_compress_dev(szp_b200_ctx *ctx, const void *d_data, int is_double, size_t n,
                                             double absErrBound, int blockSize, int threadblock,
                                             unsigned char *d_out, size_t out_cap, size_t *out_len);
SZP_B200_API int szp_b200_plain_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_in, size_t in_len,
                                               int is_double, size_t n, double absErrBound, int blockSize,
                                               void *d_out);

/* One field split across devices (no reference counterpart; the exchange
 * steps run in the host layer, toposzp-cuda_b200/shard.py).  A slab
 * [begin, end) of the field (block-aligned: begin and end multiples of 64, or
 * end == n), held in d_slab from global element begin - halo_lo on (halo_lo a
 * multiple of 4 covering min(begin, one plane + 1 -- one row + 1 in 2D), and
 * the buffer reaching min(n, end + the same)), encodes into its topology
 * blocks (no header; offsets relative to the slab) and its critical-point
 * pairs {order-preserving value code, slab-local extremum index or ~0} in
 * raster order.  blockSize 64.  Concatenated in slab order, the blocks of all
 * slabs are the single-device topology payload. */
typedef struct {
    size_t payload_bytes;   /* topology blocks of the slab */
    size_t cp_count;        /* critical points of the slab */
    size_t extrema_count;   /* maxima + minima of the slab */
} szp_b200_slab_sizes;
SZP_B200_API int szp_b200_topo_encode_slab_dev(szp_b200_ctx *ctx, const float *d_slab, size_t halo_lo,
                                               szp_b200_geom geom, float absErrBound, int blockSize,
                                               size_t begin, size_t end, unsigned char *d_payload,
                                               size_t payload_cap, void *d_pairs, size_t pairs_cap,
                                               szp_b200_slab_sizes *sizes);
/* Quantization bin (the reference's qbin of the value) of K pairs. */
SZP_B200_API int szp_b200_pair_bins_dev(szp_b200_ctx *ctx, const void *d_pairs, size_t K, float absErrBound,
                                        int *d_bins);
/* Sort positions (dense rank of the value among the pairs of its bin) of the
 * E extrema among K pairs, written at each pair's extremum index. */
SZP_B200_API int szp_b200_rank_pairs_dev(szp_b200_ctx *ctx, const void *d_pairs, size_t K, size_t E,
                                         float absErrBound, int *d_sp);
/* [u64 0][blocks] of n ints (the sort-position stream format). */
SZP_B200_API int szp_b200_encode_ints_dev(szp_b200_ctx *ctx, const int *d_vals, size_t n, int blockSize,
                                          unsigned char *d_out, size_t out_cap, size_t *out_bytes);

/* Bounded-wait self-test (no reference counterpart).  Every device wait of
 * the library gives up after a poll limit and reports an error instead of
 * hanging; this runs one such wait that can never be satisfied, with a short
 * limit (spin_limit polls, 1 .. 2^20), and returns the status it ended with:
 *   which = 0: a tile look-back whose predecessor never publishes
 *              (expected status 1, look-back timeout);
 *   which = 1: a grid barrier that one CTA never reaches
 *              (expected status 5, wait timeout).
 * *ms is the probe kernel's device time.  Returns 0 when the probe ran. */
SZP_B200_API int szp_b200_selftest_bounded_wait(int which, int spin_limit, int *status, float *ms);

/* ------------------------------------------------------------------ */
/* Batched compression (no reference counterpart)                      */
/* ------------------------------------------------------------------ */

/* One field of a batch.  errBound is absolute, or relative to the field's
 * value range when rel != 0 (bound = errBound * (max - min) in float, as the
 * reference's szp_rel_to_abs_float).  Buffers are device memory sized with
 * szp_b200_topo_bound / szp_b200_sort_bound. */
typedef struct {
    const float *d_data;
    szp_b200_geom geom;
    float errBound;
    int rel;
    unsigned char *d_topo;
    size_t topo_cap;
    unsigned char *d_sort;
    size_t sort_cap;
    szp_b200_sizes sizes;   /* out */
    float abs_eb;           /* out: the absolute bound the field was coded with */
} szp_b200_batch_field;

/* A batch compressor on a stream (0: its own stream) for one blockSize
 * (at most 256).  Each call compresses any number of fields of any shapes
 * with one persistent launch per codec pass (a device tile work-queue over
 * all fields), replayed from captured CUDA graphs; the streams are the same
 * bytes as szp_b200_topo_compress_dev gives per field.  The encoders' CTA
 * shape (threads per CTA, CTAs per SM) is autotuned on the first batch. */
typedef struct szp_b200_batch szp_b200_batch;
SZP_B200_API szp_b200_batch *szp_b200_batch_create(void *cuda_stream, int blockSize);
SZP_B200_API void szp_b200_batch_destroy(szp_b200_batch *b);

/* use_graphs: replay captured CUDA graphs (1, default) or launch directly (0).
 * autotune: 0 keep the current shapes, 1 tune once (default), 2 tune again. */
SZP_B200_API int szp_b200_batch_configure(szp_b200_batch *b, int use_graphs, int autotune);

/* Compresses count fields; fills each field's sizes and abs_eb.  Synchronous.
 * Returns 0 on success. */
SZP_B200_API int szp_b200_batch_compress(szp_b200_batch *b, szp_b200_batch_field *fields, int count);

/* Sizes the batch's device and pinned buffers and its workspace for any batch
 * of at most max_fields fields of at most max_elements elements in total, so
 * that such batches allocate nothing (buffer growth frees memory, which waits
 * for the whole device).  Returns 0 on success. */
SZP_B200_API int szp_b200_batch_reserve(szp_b200_batch *b, int max_fields, size_t max_elements);

/* Chosen shapes: shape[0..3] = topology encoder threads per CTA, CTAs per SM,
 * sort-position encoder threads per CTA, CTAs per SM; ms[] = the autotuner's
 * timings of the topology-encoder candidates.  Returns 1 once tuned. */
SZP_B200_API int szp_b200_batch_tuning(szp_b200_batch *b, int *shape, float *ms, int max);

/* The batch's workspace (stage times, launch counter). */
SZP_B200_API szp_b200_ctx *szp_b200_batch_ctx(szp_b200_batch *b);

/* ------------------------------------------------------------------ */
/* Request server with continuous batching (no reference counterpart)  */
/* ------------------------------------------------------------------ */

#define SZP_B200_OP_COMPRESS 0
#define SZP_B200_OP_DECOMPRESS 1

typedef struct {
    int slots;            /* concurrent workers: one stream + workspace + batch compressor each */
    int max_batch;        /* compressions merged into one batched launch */
    int blockSize;        /* blockSize of the compressions (at most 256) */
    size_t hbm_budget;    /* estimated device bytes admitted at once (0: 120 GiB); one merged
                             launch takes at most hbm_budget / slots */
} szp_b200_server_config;

/* One request; it must stay alive and untouched until done != 0.  All
 * buffers are device memory owned by the caller.
 *   compress:   d_data in; d_topo / d_sort out with topo_bytes / sort_bytes
 *               their capacities; errBound absolute, or relative when rel
 *   decompress: d_topo / d_sort in with topo_bytes / sort_bytes their stream
 *               lengths (block offsets parsed on the device); d_out out;
 *               errBound absolute; postprocess as szp_b200_topo_decompress_dev */
typedef struct {
    int op;
    int blockSize;
    szp_b200_geom geom;
    float errBound;
    int rel;
    int postprocess;
    const float *d_data;
    float *d_out;
    unsigned char *d_topo;
    size_t topo_bytes;
    unsigned char *d_sort;
    size_t sort_bytes;
    szp_b200_sizes sizes;     /* out (compress) */
    float abs_eb;             /* out (compress) */
    int status;               /* out: 0 ok, -1 failed (message), 1 pending */
    int done;                 /* out: set when the request has finished */
    double t_arrival;         /* server clock, seconds: arrival (set on submit when 0) */
    double t_start;           /* out: taken by a worker */
    double t_done;            /* out: finished */
    char message[96];         /* out: error text */
} szp_b200_request;

typedef struct {
    unsigned long long submitted, completed, failed;
    unsigned long long batches, batched_requests;   /* batched compress launches, requests in them */
    size_t max_inflight_bytes;                      /* peak admitted working set */
    int max_concurrent;                             /* peak requests in flight */
} szp_b200_server_stats_t;

typedef struct szp_b200_server szp_b200_server;
SZP_B200_API szp_b200_server *szp_b200_server_create(const szp_b200_server_config *cfg);
SZP_B200_API void szp_b200_server_destroy(szp_b200_server *s);
SZP_B200_API double szp_b200_server_now(szp_b200_server *s);
/* Grows every worker's device workspace for requests of up to max_elements
 * elements, and its batch compressor for the largest merged launch (up to
 * max_batch fields of 2^24 elements in total), so that serving them allocates
 * nothing (an allocation while other workers run would stall the device for
 * all of them).  A relative-bound compression of more than 2^24 elements runs
 * as a batch of one and still grows its worker's batch compressor the first
 * time.  Call it while no request is in flight.  Returns 0 on success. */
SZP_B200_API int szp_b200_server_reserve(szp_b200_server *s, size_t max_elements);
SZP_B200_API int szp_b200_server_submit(szp_b200_server *s, szp_b200_request *r);
/* 0 when r finished within timeout_s, 1 on timeout */
SZP_B200_API int szp_b200_server_wait(szp_b200_server *s, szp_b200_request *r, double timeout_s);
/* 0 when every submitted request finished within timeout_s, 1 on timeout */
SZP_B200_API int szp_b200_server_drain(szp_b200_server *s, double timeout_s);
/* Submits reqs[i] at arrival_s[i] seconds after the call (NULL: all at once),
 * then drains. */
SZP_B200_API int szp_b200_server_run_trace(szp_b200_server *s, szp_b200_request *reqs, int n,
                                           const double *arrival_s, double timeout_s);
SZP_B200_API int szp_b200_server_stats(szp_b200_server *s, szp_b200_server_stats_t *st);

/* Topology stream of a device-resident field without any allocation (no
 * counterpart in the reference).  For callers that may not let a library
 * allocate device memory: code inside a framework that owns every device
 * allocation, and latency-critical paths where cudaMalloc/cudaFree would
 * synchronise the device.  Writes the same bytes as the topology stream of
 * szp_b200_topo_compress_dev (header included) into d_topo (topo_cap bytes,
 * szp_b200_topo_bound(n, B) always suffices) and its length to *topo_bytes.
 * Its only scratch is a fixed 4 MiB device array inside the library: fields
 * needing more than 131072 tile descriptors (more than 268,435,456 elements
 * at blockSize 64) are rejected with an error.  The first call on each
 * device resolves that array's address; make it before any stream capture
 * begins.  Calls on one device share the array: overlapping calls race, so
 * serialise them.  Synchronous on cuda_stream (0 = legacy default stream).
 * Returns 0 on success, -1 with szp_b200_last_error() set otherwise. */
SZP_B200_API int szp_b200_topo_encode_noalloc(const float *d_data, szp_b200_geom geom,
                                 float absErrBound, int blockSize,
                                 unsigned char *d_topo, size_t topo_cap,
                                 size_t *topo_bytes, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* SZP_B200_H */
