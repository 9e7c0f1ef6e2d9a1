/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the TopoSZp topology-preserving compression path,
 * used as the parity checker for the CUDA library.  Nothing in the product
 * library links, loads or calls this code; only tests, the smoke check and
 * the CPU-baseline leg of the benchmark do.
 *
 * Layout conventions follow the reference's CUDA path (one offset-table entry
 * of value 0, no anchor-only tail byte); a "cpu_layout" switch reproduces the
 * reference's OpenMP layout at one thread so the restatement can be pinned
 * against the reference CPU library built from its own sources.
 */
#ifndef TOPOSZP_ORACLE_H
#define TOPOSZP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int x, y, type, quantized_bin, sort_position; } ora_cp2;
typedef struct { int x, y, z, type, quantized_bin, sort_position; } ora_cp3;

/* quantization, bit-count and block-size rules */
int      ora_quantize(float x, double inv);
unsigned ora_bitcount(unsigned maxmag);
size_t   ora_block_bytes(size_t n, unsigned bc, int with_tags, int cpu_layout);

/* critical points (raster order) */
size_t ora_find_cp_2d(const float *data, int rows, int cols, float eb, ora_cp2 *out);
size_t ora_find_cp_3d(const float *data, int d1, int d2, int d3, float eb, ora_cp3 *out);
int    ora_classify_2d(const float *data, int cols, int i, int j);
int    ora_classify_3d(const float *data, int d2, int d3, int x, int y, int z);

/* dense rank of the value inside its quantization bin */
void ora_sort_cp_2d(ora_cp2 *cp, size_t k, const float *data, int cols);
void ora_sort_cp_3d(ora_cp3 *cp, size_t k, const float *data, int d2, int d3);

/* types from a CP list into u8[n] */
void ora_mark_types_2d(const ora_cp2 *cp, size_t k, int rows, int cols, uint8_t *types);
void ora_mark_types_3d(const ora_cp3 *cp, size_t k, int d1, int d2, int d3, uint8_t *types);

/* extrema sort positions in list order; returns the extrema count */
size_t ora_extract_sp_2d(const ora_cp2 *cp, size_t k, int *sp);
size_t ora_extract_sp_3d(const ora_cp3 *cp, size_t k, int *sp);

/* encoders: return the total byte count written to out (including header) */
size_t ora_encode_topo(const float *data, size_t n, float eb, int B,
                       const uint8_t *types, int cpu_layout, uint8_t *out);
size_t ora_encode_ints(const int *v, size_t n, int B, int cpu_layout, uint8_t *out);
size_t ora_double_compress_topo_3d(const double *d, size_t n, double eb, int B, const uint8_t *types,
                                   int d1, int d2, int d3, int passes, int *q_out, uint8_t *out);
size_t ora_topo_bound(size_t n, int B);
size_t ora_ints_bound(size_t n, int B);

/* decoders: return 0 on success, negative on a malformed stream.
 * *used receives the number of stream bytes consumed (header included). */
int ora_decode_topo(const uint8_t *s, size_t len, size_t n, float eb, int B,
                    float *out, int *fn, size_t *used);
int ora_decode_ints(const uint8_t *s, size_t len, size_t n, int B, int *out, size_t *used);
size_t ora_plain_compress(const void *d, int dbl, size_t n, double eb, int B, int tb, uint8_t *out);
size_t ora_plain_bound(size_t n, int B, int dbl);
int ora_plain_decompress_ra(const uint8_t *s, size_t len, size_t n, double eb, int B, int dbl, void *out,
                            size_t *used);
int ora_plain_decompress_tb(const uint8_t *s, size_t len, size_t n, double eb, int B, int dbl, void *out,
                            size_t *used);

/* post-processing (serial raster semantics of the reference CUDA drivers) */
int ora_post_2d(float *data, const float *orig, const int *fn, const int *sp,
                size_t n_sp, int rows, int cols, float eb, int *restored);
int ora_post_3d(float *data, const float *orig, const int *fn, const int *sp,
                size_t n_sp, int d1, int d2, int d3, float eb, int axis_stencil,
                int *restored);

/* individual passes, exposed for finer-grained tests */
void ora_stencils_2d(float *data, const float *orig, const int *fn, const int *sp,
                     size_t n_sp, int rows, int cols, float eb);
void ora_enforce_2d(float *data, const float *orig, const int *fn, int rows, int cols,
                    float eps, float eb);
int  ora_rbf_2d(float *data, const float *orig, const int *fn, int rows, int cols,
                float eps, float eb);
void ora_stencils_3d(float *data, const float *orig, const int *fn, const int *sp,
                     size_t n_sp, int d1, int d2, int d3, float eb);
void ora_enforce_3d(float *data, const float *orig, const int *fn, int d1, int d2, int d3,
                    float eps, float eb);
int  ora_rbf_3d(float *data, const float *orig, const int *fn, int d1, int d2, int d3,
                float eps, float eb);
int  ora_axis_saddles_3d(float *data, const float *orig, const int *fn,
                         int d1, int d2, int d3, float eb);

/* relative error bound -> absolute (float arithmetic) */
float ora_rel_to_abs(const float *data, size_t n, float rel);

#ifdef __cplusplus
}
#endif
#endif
