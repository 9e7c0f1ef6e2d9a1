/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Plain-C restatement of the TopoSZp topology path.  Every function names the
 * reference file:line whose behaviour it restates (paths relative to the
 * reference project root).  Build with -ffp-contract=off: the reference's
 * post-processing is host code compiled without FMA contraction, and the
 * parity target is its exact float/double rounding.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* scalar rules                                                        */
/* ------------------------------------------------------------------ */

/* (int)((double)x * inv) as the CUDA path evaluates it
 * (SZp/src/szp_cuda_topology.cu:547,592): truncation toward zero, values
 * beyond the int range saturate, and NaN converts to INT_MIN -- the outputs
 * of the reference's own CUDA build on sm_100a for +-inf, +-1e300, values just
 * outside the range and NaN (the special_20x21x22 case of
 * tests/golden/f64_topo.json).  For values inside the int range this is
 * identical to the host cast (SZp/src/szp_float.cc:1212). */
static int trunc_sat(double v)
{
    if (v != v) return (-2147483647 - 1);
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (-2147483647 - 1);
    return (int)v;
}

int ora_quantize(float x, double inv) { return trunc_sat((double)x * inv); }

/* qbin = (int)((center + eb) * inv): float add first, then the double
 * multiply (SZp/src/szp_cuda_topology.cu:67, SZp/src/szp_float.cc:76). */
static int quant_bin(float c, float eb, double inv)
{
    volatile float s = c + eb;
    return trunc_sat((double)s * inv);
}

/* bc = floor(log2f((float)max)) + 1, 0 when all deltas vanish
 * (SZp/src/szp_cuda_topology.cu:558,619; SZp/src/szp_float.cc:1243). */
unsigned ora_bitcount(unsigned m)
{
    if (m == 0) return 0;
    return (unsigned)floorf(log2f((float)m)) + 1u;
}

static size_t magnitude_bytes(size_t cnt, unsigned bc)
{
    size_t fb = bc / 8, rem = bc % 8;
    size_t len = fb * cnt;
    if (rem) len += (rem * cnt - 1) / 8 + 1;
    return len;
}

/* Size of one compressed block of n elements (Appendix-A layout).  The CUDA
 * layout omits the bit-count byte for n == 1 (SZp/src/szp_cuda_topology.cu:
 * 546-567); the OpenMP layout always writes it (SZp/src/szp_float.cc:1239). */
size_t ora_block_bytes(size_t n, unsigned bc, int with_tags, int cpu_layout)
{
    size_t s = 4;
    if (n > 1 || cpu_layout) s += 1;
    if (n > 1 && bc) s += (n - 1 + 7) / 8 + magnitude_bytes(n - 1, bc);
    if (with_tags) s += (2 * n + 7) / 8;
    return s;
}

/* ------------------------------------------------------------------ */
/* critical points                                                     */
/* ------------------------------------------------------------------ */

/* 4-neighbour classification (SZp/src/szp_cuda_topology.cu:50-64,
 * example/test_cuda_topology.cu:56-68). */
static int cls2(float c, float up, float dn, float lf, float rt)
{
    if (c > up && c > dn && c > lf && c > rt) return 1;
    if (c < up && c < dn && c < lf && c < rt) return 2;
    if ((c < up && c < dn && c > lf && c > rt) || (c > up && c > dn && c < lf && c < rt))
        return 3;
    return 0;
}

int ora_classify_2d(const float *d, int cols, int i, int j)
{
    size_t c = (size_t)i * cols + j;
    return cls2(d[c], d[c - cols], d[c + cols], d[c - 1], d[c + 1]);
}

/* 6-neighbour classification (SZp/src/szp_cuda_topology_3d.cu:126-160,
 * example/test_cuda_topology_3d.cu:52-73). */
static int cls3(float c, float xm, float xp, float ym, float yp, float zm, float zp)
{
    if (c > xm && c > xp && c > ym && c > yp && c > zm && c > zp) return 1;
    if (c < xm && c < xp && c < ym && c < yp && c < zm && c < zp) return 2;
    int hi = (c > xm && c > xp) + (c > ym && c > yp) + (c > zm && c > zp);
    int lo = (c < xm && c < xp) + (c < ym && c < yp) + (c < zm && c < zp);
    return (hi >= 1 && lo >= 1) ? 3 : 0;
}

int ora_classify_3d(const float *d, int d2, int d3, int x, int y, int z)
{
    size_t pl = (size_t)d2 * d3;
    size_t c = (size_t)x * pl + (size_t)y * d3 + z;
    return cls3(d[c], d[c - pl], d[c + pl], d[c - d3], d[c + d3], d[c - 1], d[c + 1]);
}

/* Interior cells in raster order; the reference's OpenMP finder produces this
 * order at one thread (SZp/src/szp_float.cc:28-120). */
size_t ora_find_cp_2d(const float *d, int rows, int cols, float eb, ora_cp2 *out)
{
    if (!d || rows <= 2 || cols <= 2) return 0;
    double inv = 1.0 / (double)eb;
    size_t k = 0;
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            int t = ora_classify_2d(d, cols, i, j);
            if (!t) continue;
            ora_cp2 c = {i, j, t, quant_bin(d[(size_t)i * cols + j], eb, inv), 0};
            out[k++] = c;
        }
    return k;
}

/* (SZp/src/szp_topology_3d.cc:30-129) */
size_t ora_find_cp_3d(const float *d, int d1, int d2, int d3, float eb, ora_cp3 *out)
{
    if (!d || d1 <= 2 || d2 <= 2 || d3 <= 2) return 0;
    double inv = 1.0 / (double)eb;
    size_t pl = (size_t)d2 * d3, k = 0;
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                int t = ora_classify_3d(d, d2, d3, x, y, z);
                if (!t) continue;
                float c = d[(size_t)x * pl + (size_t)y * d3 + z];
                ora_cp3 r = {x, y, z, t, quant_bin(c, eb, inv), 0};
                out[k++] = r;
            }
    return k;
}

/* ------------------------------------------------------------------ */
/* sort positions: dense rank of the value among the CPs of one bin    */
/* (SZp/src/szp_float.cc:137-509; SZp/src/szp_cuda_topology.cu:139-272) */
/* ------------------------------------------------------------------ */

typedef struct { int bin; float val; size_t idx; } rank_item;

static int rank_cmp(const void *a, const void *b)
{
    const rank_item *p = (const rank_item *)a, *q = (const rank_item *)b;
    if (p->bin != q->bin) return p->bin < q->bin ? -1 : 1;
    if (p->val < q->val) return -1;
    if (p->val > q->val) return 1;
    return (p->idx < q->idx) ? -1 : (p->idx > q->idx);
}

static void dense_rank(rank_item *it, size_t k, int *pos_out_by_idx)
{
    qsort(it, k, sizeof(*it), rank_cmp);
    int r = 0;
    for (size_t i = 0; i < k; i++) {
        if (i == 0 || it[i].bin != it[i - 1].bin) r = 0;
        else if (it[i].val != it[i - 1].val) r++;
        pos_out_by_idx[it[i].idx] = r;
    }
}

void ora_sort_cp_2d(ora_cp2 *cp, size_t k, const float *d, int cols)
{
    if (!cp || !k || !d) return;
    rank_item *it = (rank_item *)malloc(k * sizeof(*it));
    int *pos = (int *)malloc(k * sizeof(int));
    for (size_t i = 0; i < k; i++) {
        it[i].bin = cp[i].quantized_bin;
        it[i].val = d[(size_t)cp[i].x * cols + cp[i].y];
        it[i].idx = i;
    }
    dense_rank(it, k, pos);
    for (size_t i = 0; i < k; i++) cp[i].sort_position = pos[i];
    free(it); free(pos);
}

void ora_sort_cp_3d(ora_cp3 *cp, size_t k, const float *d, int d2, int d3)
{
    if (!cp || !k || !d) return;
    rank_item *it = (rank_item *)malloc(k * sizeof(*it));
    int *pos = (int *)malloc(k * sizeof(int));
    size_t pl = (size_t)d2 * d3;
    for (size_t i = 0; i < k; i++) {
        it[i].bin = cp[i].quantized_bin;
        it[i].val = d[(size_t)cp[i].x * pl + (size_t)cp[i].y * d3 + cp[i].z];
        it[i].idx = i;
    }
    dense_rank(it, k, pos);
    for (size_t i = 0; i < k; i++) cp[i].sort_position = pos[i];
    free(it); free(pos);
}

/* (SZp/src/szp_cuda_topology.cu:513-528; SZp/src/szp_float.cc:1043-1064) */
void ora_mark_types_2d(const ora_cp2 *cp, size_t k, int rows, int cols, uint8_t *ty)
{
    for (size_t i = 0; i < k; i++) {
        int x = cp[i].x, y = cp[i].y, t = cp[i].type;
        if (x < 0 || x >= rows || y < 0 || y >= cols) continue;
        if (t >= 1 && t <= 3) ty[(size_t)x * cols + y] = (uint8_t)t;
    }
}

/* (SZp/src/szp_cuda_topology_3d.cu:602-618) */
void ora_mark_types_3d(const ora_cp3 *cp, size_t k, int d1, int d2, int d3, uint8_t *ty)
{
    size_t pl = (size_t)d2 * d3;
    for (size_t i = 0; i < k; i++) {
        int x = cp[i].x, y = cp[i].y, z = cp[i].z, t = cp[i].type;
        if (x < 0 || x >= d1 || y < 0 || y >= d2 || z < 0 || z >= d3) continue;
        if (t >= 1 && t <= 3) ty[(size_t)x * pl + (size_t)y * d3 + z] = (uint8_t)t;
    }
}

/* extrema only, in list order (SZp/src/szp_cuda_topology.cu:436-449) */
size_t ora_extract_sp_2d(const ora_cp2 *cp, size_t k, int *sp)
{
    size_t e = 0;
    for (size_t i = 0; i < k; i++)
        if (cp[i].type == 1 || cp[i].type == 2) sp[e++] = cp[i].sort_position;
    return e;
}

size_t ora_extract_sp_3d(const ora_cp3 *cp, size_t k, int *sp)
{
    size_t e = 0;
    for (size_t i = 0; i < k; i++)
        if (cp[i].type == 1 || cp[i].type == 2) sp[e++] = cp[i].sort_position;
    return e;
}

/* ------------------------------------------------------------------ */
/* block encoder                                                       */
/* ------------------------------------------------------------------ */

/* One block: int32 anchor, bit count, MSB-first sign bits, "Jiajun"
 * magnitudes (full bytes little-endian per value, then the remaining bits
 * MSB-first and contiguous), then 2-bit tags MSB-first.
 * (SZp/src/szp_cuda_topology.cu:577-680; SZp/src/szp_TypeManager.cc:13-102,
 *  837-861, 1079-1176.) */
static size_t encode_block(const int *q, size_t n, const uint8_t *tags, int cpu_layout,
                           uint8_t *o)
{
    uint8_t *p = o;
    unsigned int a = (unsigned int)q[0];
    p[0] = (uint8_t)a; p[1] = (uint8_t)(a >> 8); p[2] = (uint8_t)(a >> 16); p[3] = (uint8_t)(a >> 24);
    p += 4;
    size_t cnt = n > 1 ? n - 1 : 0;
    unsigned maxm = 0;
    unsigned *mag = NULL;
    uint8_t *neg = NULL;
    if (cnt) {
        mag = (unsigned *)malloc(cnt * sizeof(unsigned));
        neg = (uint8_t *)malloc(cnt);
        for (size_t j = 0; j < cnt; j++) {
            unsigned ud = (unsigned)q[j + 1] - (unsigned)q[j];
            int d = (int)ud;
            neg[j] = d < 0;
            mag[j] = d < 0 ? 0u - ud : ud;
            if (mag[j] > maxm) maxm = mag[j];
        }
    }
    unsigned bc = ora_bitcount(maxm);
    if (n > 1 || cpu_layout) *p++ = (uint8_t)bc;
    if (cnt && bc) {
        size_t sb = (cnt + 7) / 8;
        memset(p, 0, sb);
        for (size_t j = 0; j < cnt; j++)
            if (neg[j]) p[j / 8] |= (uint8_t)(1u << (7 - j % 8));
        p += sb;
        unsigned fb = bc / 8, rem = bc % 8;
        for (size_t j = 0; j < cnt; j++) {
            unsigned v = mag[j] >> rem;
            for (unsigned t = 0; t < fb; t++) { *p++ = (uint8_t)(v & 0xFF); v >>= 8; }
        }
        if (rem) {
            size_t rb = (rem * cnt - 1) / 8 + 1;
            memset(p, 0, rb);
            unsigned mask = (1u << rem) - 1u;
            for (size_t j = 0; j < cnt; j++) {
                unsigned v = mag[j] & mask;
                for (unsigned b = 0; b < rem; b++) {
                    size_t bit = j * rem + b;
                    if ((v >> (rem - 1 - b)) & 1u) p[bit / 8] |= (uint8_t)(1u << (7 - bit % 8));
                }
            }
            p += rb;
        }
    }
    if (tags) {
        size_t tb = (2 * n + 7) / 8;
        memset(p, 0, tb);
        for (size_t j = 0; j < n; j++)
            p[j / 4] |= (uint8_t)((tags[j] & 3u) << (6 - 2 * (j % 4)));
        p += tb;
    }
    free(mag); free(neg);
    return (size_t)(p - o);
}

size_t ora_topo_bound(size_t n, int B)
{
    size_t nb = (n + B - 1) / B;
    return 8 + nb * ora_block_bytes((size_t)B, 33, 1, 1) + 64;
}

size_t ora_ints_bound(size_t n, int B)
{
    size_t nb = (n + B - 1) / B;
    return 16 + nb * ora_block_bytes((size_t)B, 33, 0, 1) + 64;
}

/* CUDA layout: [u64 0][blocks] (SZp/src/szp_cuda_topology.cu:746-762).
 * OpenMP layout at one thread: the same header, plus the tail bit-count byte
 * (SZp/src/szp_float.cc:1239-1253, 1277-1286). */
size_t ora_encode_topo(const float *data, size_t n, float eb, int B, const uint8_t *types,
                       int cpu_layout, uint8_t *out)
{
    double inv = 1.0 / (double)eb;
    memset(out, 0, 8);
    size_t off = 8;
    int *q = (int *)malloc((size_t)B * sizeof(int));
    uint8_t *tg = (uint8_t *)malloc((size_t)B);
    for (size_t s = 0; s < n; s += (size_t)B) {
        size_t m = (n - s < (size_t)B) ? n - s : (size_t)B;
        for (size_t j = 0; j < m; j++) {
            q[j] = ora_quantize(data[s + j], inv);
            tg[j] = types ? types[s + j] : 0;
        }
        off += encode_block(q, m, tg, cpu_layout, out + off);
    }
    free(q); free(tg);
    return off;
}

/* CUDA layout: [u64 0][blocks] (SZp/src/szp_cuda_topology.cu:480-496).
 * OpenMP layout at one thread: [u64 count][u64 0][blocks]
 * (SZp/src/szp_float.cc:607-621, 839-849). */
size_t ora_encode_ints(const int *v, size_t n, int B, int cpu_layout, uint8_t *out)
{
    size_t off = 0;
    if (cpu_layout) {
        unsigned long long c = n;
        memcpy(out, &c, 8);
        off = 8;
    }
    memset(out + off, 0, 8);
    off += 8;
    for (size_t s = 0; s < n; s += (size_t)B) {
        size_t m = (n - s < (size_t)B) ? n - s : (size_t)B;
        off += encode_block(v + s, m, NULL, cpu_layout, out + off);
    }
    return off;
}

/* ------------------------------------------------------------------ */
/* fp64 3D topology compression                                        */
/* ------------------------------------------------------------------ */

/* Integer arithmetic of the saddle repair wraps (c - 1 at INT_MIN). */
static int wrap_add(int a, int d) { return (int)((unsigned)a + (unsigned)d); }

/* One repair pass over the interior saddles (type 3), all reads from the
 * snapshot src, writes into dst (SZp/src/szp_cuda_topology_3d.cu:736-826).
 * A saddle that is still high along one axis and low along another keeps its
 * value; otherwise c, c - 1, c + 1 are tried in that order, and the first
 * that is high along >= 1 axis, low along >= 1 axis and leaves every
 * neighbouring maximum above it and every neighbouring minimum below it is
 * written.  Interior: 1 <= x <= d1-2 (y, z alike); a grid with an axis below
 * 3 has none.  Points whose +x neighbour lies at or beyond n are skipped. */
static void fix_saddles_pass(const int *src, int *dst, const uint8_t *ty, size_t n, int d1, int d2, int d3)
{
    if (d1 < 3 || d2 < 3 || d3 < 3) return;
    const size_t pl = (size_t)d2 * d3;
    const long long st[6] = {-(long long)pl, (long long)pl, -(long long)d3, (long long)d3, -1, 1};
    for (int x = 1; x <= d1 - 2; x++)
        for (int y = 1; y <= d2 - 2; y++)
            for (int z = 1; z <= d3 - 2; z++) {
                size_t p = (size_t)x * pl + (size_t)y * d3 + z;
                if (p + pl >= n || ty[p] != 3) continue;
                int c = src[p], v[6], hi[3], lo[3];
                for (int k = 0; k < 6; k++) v[k] = src[(size_t)((long long)p + st[k])];
                int nh = 0, nl = 0;
                for (int a = 0; a < 3; a++) {
                    hi[a] = v[2 * a] > v[2 * a + 1] ? v[2 * a] : v[2 * a + 1];
                    lo[a] = v[2 * a] < v[2 * a + 1] ? v[2 * a] : v[2 * a + 1];
                    nh += c > hi[a];
                    nl += c < lo[a];
                }
                if (nh >= 1 && nl >= 1) continue;
                const int tries[3] = {0, -1, 1};
                for (int t = 0; t < 3; t++) {
                    int tv = wrap_add(c, tries[t]);
                    int th = 0, tl = 0;
                    for (int a = 0; a < 3; a++) { th += tv > hi[a]; tl += tv < lo[a]; }
                    if (th < 1 || tl < 1) continue;
                    int ok = 1;
                    for (int k = 0; k < 6; k++) {
                        uint8_t tk = ty[(size_t)((long long)p + st[k])];
                        if (tk == 1 && v[k] <= tv) ok = 0;
                        if (tk == 2 && v[k] >= tv) ok = 0;
                    }
                    if (ok) { dst[p] = tv; break; }
                }
            }
}

/* q = (int)(x * (1/eb)) in double (SZp/src/szp_cuda_topology_3d.cu:641-646),
 * `passes` snapshot repair passes (three in the reference, :1125-1145), then
 * the topology block layout over the ints with the 2-bit tags
 * (:836-958, header :1171-1174): [u64 0][blocks].  Writes q after repair to
 * q_out when it is not NULL. */
size_t ora_double_compress_topo_3d(const double *d, size_t n, double eb, int B, const uint8_t *types,
                                   int d1, int d2, int d3, int passes, int *q_out, uint8_t *out)
{
    double inv = 1.0 / eb;
    int *q = (int *)malloc(n * sizeof(int));
    int *src = (int *)malloc(n * sizeof(int));
    for (size_t i = 0; i < n; i++) q[i] = trunc_sat(d[i] * inv);
    for (int p = 0; p < passes; p++) {
        memcpy(src, q, n * sizeof(int));
        fix_saddles_pass(src, q, types, n, d1, d2, d3);
    }
    memset(out, 0, 8);
    size_t off = 8;
    for (size_t s = 0; s < n; s += (size_t)B) {
        size_t m = (n - s < (size_t)B) ? n - s : (size_t)B;
        off += encode_block(q + s, m, types + s, 0, out + off);
    }
    if (q_out) memcpy(q_out, q, n * sizeof(int));
    free(q); free(src);
    return off;
}

/* ------------------------------------------------------------------ */
/* decoder                                                             */
/* ------------------------------------------------------------------ */

static unsigned rd_u32(const uint8_t *p)
{
    return (unsigned)p[0] | ((unsigned)p[1] << 8) | ((unsigned)p[2] << 16) | ((unsigned)p[3] << 24);
}

static unsigned long long rd_u64(const uint8_t *p)
{
    unsigned long long v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}

/* one Jiajun value (SZp/src/szp_cuda_decompress.cu:91-138) */
static unsigned extract_mag(const uint8_t *m, size_t idx, size_t cnt, unsigned bc)
{
    unsigned fb = bc >> 3, rem = bc & 7;
    unsigned v = 0;
    if (rem) {
        size_t bit = idx * rem;
        const uint8_t *r = m + fb * cnt;
        for (unsigned b = 0; b < rem; b++, bit++)
            v = (v << 1) | ((r[bit >> 3] >> (7 - (bit & 7))) & 1u);
    }
    if (fb) {
        unsigned full = 0;
        for (unsigned t = 0; t < fb; t++) full |= (unsigned)m[idx * fb + t] << (8 * t);
        v |= full << rem;
    }
    return v;
}

/* walk of one block (SZp/src/szp_cuda_decompress.cu:443-473) */
static int block_span(const uint8_t *s, size_t pos, size_t lim, size_t n, int tags,
                      size_t *next)
{
    if (pos + 4 > lim) return -1;
    size_t p = pos + 4;
    if (n > 1) {
        if (p >= lim) return -1;
        unsigned bc = s[p++];
        if (bc > 32) return -1;
        if (bc) p += (n - 1 + 7) / 8 + magnitude_bytes(n - 1, bc);
        if (p > lim) return -1;
    }
    if (tags) p += (2 * n + 7) / 8;
    if (p > lim) return -1;
    *next = p;
    return 0;
}

/* Offset-table thread-count detection and block walk
 * (SZp/src/szp_cuda_decompress.cu:339-477, 233-328). */
static int find_layout(const uint8_t *s, size_t len, size_t n, int B, int tags,
                       unsigned *T_out)
{
    size_t nb = (n + B - 1) / B;
    size_t maxc = tags ? 8ull * n + 1024 : 4ull * n + 4;
    size_t lim = len < maxc ? len : maxc;
    unsigned T = 1;
    if (len >= 8 && rd_u64(s) == 0) {
        for (unsigned t = 1; t <= 128; t++) {
            int ok = 1;
            if ((size_t)8 * t > len) break;
            for (unsigned k = 1; k < t; k++) {
                unsigned long long ok_ = rd_u64(s + 8 * k), pk = rd_u64(s + 8 * (k - 1));
                if (ok_ > maxc || ok_ < pk) { ok = 0; break; }
            }
            if (!ok) break;
            /* validate: walk every chunk */
            size_t hdr = (size_t)8 * t;
            int valid = 1;
            if (tags) {
                size_t bpt = (nb + t - 1) / t;
                for (unsigned c = 0; c < t && valid; c++) {
                    size_t pos = hdr + (size_t)rd_u64(s + 8 * c);
                    if (pos >= lim) { valid = 0; break; }
                    size_t b1 = (c + 1) * bpt < nb ? (c + 1) * bpt : nb;
                    for (size_t b = c * bpt; b < b1; b++) {
                        size_t e0 = b * B, m = (n - e0 < (size_t)B) ? n - e0 : (size_t)B;
                        if (block_span(s, pos, lim, m, 1, &pos)) { valid = 0; break; }
                    }
                }
            } else {
                size_t tbs = n / t;
                for (unsigned c = 0; c < t && valid; c++) {
                    size_t lo = c * tbs, hi = (c == t - 1) ? n : (c + 1) * tbs;
                    size_t pos = hdr + (size_t)rd_u64(s + 8 * c);
                    if (pos >= lim) { valid = 0; break; }
                    for (size_t i = lo; i < hi; i += (size_t)B) {
                        size_t m = (i + B > hi) ? hi - i : (size_t)B;
                        if (block_span(s, pos, lim, m, 0, &pos)) { valid = 0; break; }
                    }
                }
            }
            if (valid) { T = t; break; }
        }
    }
    *T_out = T;
    return 0;
}

/* (SZp/src/szp_cuda_decompress.cu:673-741, 1074-1161) */
int ora_decode_topo(const uint8_t *s, size_t len, size_t n, float eb, int B, float *out,
                    int *fn, size_t *used)
{
    /* len is the readable buffer size; the reference interface carries no
     * stream length, so only the thread-count detection applies its own
     * bound (8n + 1024) and the walk itself stops at the buffer end */
    unsigned T;
    find_layout(s, len, n, B, 1, &T);
    size_t nb = (n + B - 1) / B, hdr = (size_t)8 * T, bpt = (nb + T - 1) / T;
    size_t end = hdr;
    for (unsigned c = 0; c < T; c++) {
        size_t pos = hdr + (size_t)rd_u64(s + 8 * c);
        size_t b1 = (c + 1) * bpt < nb ? (c + 1) * bpt : nb;
        for (size_t b = c * bpt; b < b1; b++) {
            size_t e0 = b * B, m = (n - e0 < (size_t)B) ? n - e0 : (size_t)B;
            size_t nxt;
            if (block_span(s, pos, len, m, 1, &nxt)) return -1;
            int prior = (int)rd_u32(s + pos);
            size_t p = pos + 4;
            out[e0] = (float)prior * eb;
            if (m > 1) {
                unsigned bc = s[p++];
                size_t cnt = m - 1;
                if (!bc) {
                    for (size_t j = 0; j < cnt; j++) out[e0 + 1 + j] = (float)prior * eb;
                } else {
                    const uint8_t *sg = s + p;
                    const uint8_t *mg = sg + (cnt + 7) / 8;
                    for (size_t j = 0; j < cnt; j++) {
                        unsigned mg_ = extract_mag(mg, j, cnt, bc);
                        int neg = (sg[j >> 3] >> (7 - (j & 7))) & 1;
                        prior = (int)((unsigned)prior + (neg ? 0u - mg_ : mg_));
                        out[e0 + 1 + j] = (float)prior * eb;
                    }
                    p += (cnt + 7) / 8 + magnitude_bytes(cnt, bc);
                }
            }
            if (fn)
                for (size_t j = 0; j < m; j++)
                    fn[e0 + j] = (s[p + j / 4] >> (6 - 2 * (j % 4))) & 3;
            pos = nxt;
            if (pos > end) end = pos;
        }
    }
    if (used) *used = end;
    return 0;
}

/* (SZp/src/szp_cuda_decompress.cu:749-804, 1165-1235) */
int ora_decode_ints(const uint8_t *s, size_t len, size_t n, int B, int *out, size_t *used)
{
    unsigned T;
    find_layout(s, len, n, B, 0, &T);
    size_t hdr = (size_t)8 * T, tbs = n / T, end = hdr;
    for (unsigned c = 0; c < T; c++) {
        size_t lo = c * tbs, hi = (c == T - 1) ? n : (c + 1) * tbs;
        size_t pos = hdr + (size_t)rd_u64(s + 8 * c);
        for (size_t i = lo; i < hi; i += (size_t)B) {
            size_t m = (i + B > hi) ? hi - i : (size_t)B;
            size_t nxt;
            if (block_span(s, pos, len, m, 0, &nxt)) return -1;
            int prior = (int)rd_u32(s + pos);
            size_t p = pos + 4;
            out[i] = prior;
            if (m > 1) {
                unsigned bc = s[p++];
                size_t cnt = m - 1;
                const uint8_t *sg = s + p;
                const uint8_t *mg = sg + (cnt + 7) / 8;
                for (size_t j = 0; j < cnt; j++) {
                    if (bc) {
                        unsigned mg_ = extract_mag(mg, j, cnt, bc);
                        int neg = (sg[j >> 3] >> (7 - (j & 7))) & 1;
                        prior = (int)((unsigned)prior + (neg ? 0u - mg_ : mg_));
                    }
                    out[i + 1 + j] = prior;
                }
            }
            pos = nxt;
            if (pos > end) end = pos;
        }
    }
    if (used) *used = end;
    return 0;
}

/* ------------------------------------------------------------------ */
/* plain (non-topology) codec: random-access and threadblock modes,    */
/* float and double (SZp/src/szp_cuda_compress.cu:122-360, 384-802;   */
/* SZp/src/szp_cuda_decompress.cu:176-328, 480-665, 810-1070)          */
/* ------------------------------------------------------------------ */

static int quant_elem(const void *d, int dbl, size_t i, double inv)
{
    return dbl ? trunc_sat(((const double *)d)[i] * inv) : trunc_sat((double)((const float *)d)[i] * inv);
}

/* [bit count][sign bits][magnitudes] of the cnt deltas q[j+1] - q[j]; the
 * bit-count byte is always written, the rest only when it is not 0
 * (SZp/src/szp_cuda_compress.cu:296-357). */
static size_t encode_deltas(const int *q, size_t cnt, uint8_t *o)
{
    uint8_t *p = o;
    unsigned maxm = 0;
    for (size_t j = 0; j < cnt; j++) {
        unsigned ud = (unsigned)q[j + 1] - (unsigned)q[j];
        unsigned m = (int)ud < 0 ? 0u - ud : ud;
        if (m > maxm) maxm = m;
    }
    unsigned bc = ora_bitcount(maxm);
    *p++ = (uint8_t)bc;
    if (!bc) return 1;
    size_t sb = (cnt + 7) / 8;
    memset(p, 0, sb);
    for (size_t j = 0; j < cnt; j++) {
        unsigned ud = (unsigned)q[j + 1] - (unsigned)q[j];
        if ((int)ud < 0) p[j / 8] |= (uint8_t)(1u << (7 - j % 8));
    }
    p += sb;
    unsigned fb = bc / 8, rem = bc % 8;
    for (size_t j = 0; j < cnt; j++) {
        unsigned ud = (unsigned)q[j + 1] - (unsigned)q[j];
        unsigned v = ((int)ud < 0 ? 0u - ud : ud) >> rem;
        for (unsigned t = 0; t < fb; t++) { *p++ = (uint8_t)(v & 0xFF); v >>= 8; }
    }
    if (rem) {
        size_t rb = (rem * cnt + 7) / 8;
        memset(p, 0, rb);
        for (size_t j = 0; j < cnt; j++) {
            unsigned ud = (unsigned)q[j + 1] - (unsigned)q[j];
            unsigned v = ((int)ud < 0 ? 0u - ud : ud) & ((1u << rem) - 1u);
            for (unsigned b = 0; b < rem; b++) {
                size_t bit = j * rem + b;
                if ((v >> (rem - 1 - b)) & 1u) p[bit / 8] |= (uint8_t)(1u << (7 - bit % 8));
            }
        }
        p += rb;
    }
    return (size_t)(p - o);
}

/* Compressed stream of the CUDA plain compressors: [T eb][u64 0][body]
 * (T float or double; one chunk).  Random access (tb == 0): blocks of B
 * elements, each [i32 anchor][bit count if the block has > 1 element][signs]
 * [magnitudes] (:122-243, 384-474).  Threadblock (tb == 1): [i32 q0], then
 * blocks of B deltas over elements 1 .. n-1, each [bit count][signs]
 * [magnitudes], deltas chained across blocks (:245-357, 550-607).  q =
 * (int)(x * (1/eb)) in double, inv = 1.0 / (double)eb.  eb carries the
 * caller's float bound exactly when dbl == 0. */
size_t ora_plain_compress(const void *d, int dbl, size_t n, double eb, int B, int tb, uint8_t *out)
{
    size_t es = dbl ? 8 : 4;
    if (dbl) memcpy(out, &eb, 8);
    else { float f = (float)eb; memcpy(out, &f, 4); }
    memset(out + es, 0, 8);
    size_t off = es + 8;
    double inv = 1.0 / eb;
    int *q = (int *)malloc(((size_t)B + 1) * sizeof(int));
    if (!tb) {
        for (size_t s = 0; s < n; s += (size_t)B) {
            size_t m = (n - s < (size_t)B) ? n - s : (size_t)B;
            for (size_t j = 0; j < m; j++) q[j] = quant_elem(d, dbl, s + j, inv);
            off += encode_block(q, m, NULL, 0, out + off);
        }
    } else if (n) {
        int prior = quant_elem(d, dbl, 0, inv);
        memcpy(out + off, &prior, 4);
        off += 4;
        for (size_t i = 1; i < n; i += (size_t)B) {
            size_t m = (n - i < (size_t)B) ? n - i : (size_t)B;
            q[0] = prior;
            for (size_t j = 0; j < m; j++) q[j + 1] = quant_elem(d, dbl, i + j, inv);
            off += encode_deltas(q, m, out + off);
            prior = q[m];
        }
    }
    free(q);
    return off;
}

size_t ora_plain_bound(size_t n, int B, int dbl)
{
    size_t nb = (n + B - 1) / B + 1;
    return (dbl ? 8 : 4) + 8 + 4 + nb * ora_block_bytes((size_t)B + 1, 32, 0, 1) + 64;
}

static void store_deq(void *out, int dbl, size_t i, int q, double eb)
{
    if (dbl) ((double *)out)[i] = (double)q * eb;
    else ((float *)out)[i] = (float)q * (float)eb;
}

/* Random-access decompression of s = the stream after its T eb header, as
 * the reference API receives it: thread-count detection and walk as for the
 * sort-position stream (:176-328), values (T)q * eb (:523-595). */
int ora_plain_decompress_ra(const uint8_t *s, size_t len, size_t n, double eb, int B, int dbl, void *out,
                            size_t *used)
{
    int *q = (int *)malloc((n ? n : 1) * sizeof(int));
    int rc = ora_decode_ints(s, len, n, B, q, used);
    if (!rc)
        for (size_t i = 0; i < n; i++) store_deq(out, dbl, i, q[i], eb);
    free(q);
    return rc;
}

/* Threadblock decompression (:480-518, 597-665, 905-984).  Thread count:
 * the largest t <= 256 whose first t offsets are non-decreasing and at most
 * 4n + 4, stopping at the first t that is not (1 when the first offset is
 * not 0); each chunk [lo, hi) of n / t elements is [i32 q0][blocks of B
 * deltas].  A detected table whose chunks do not walk inside 4n + 4 bytes is
 * read as one chunk (the reference decodes past its buffer there); -1 when
 * that does not walk either. */
int ora_plain_decompress_tb(const uint8_t *s, size_t len, size_t n, double eb, int B, int dbl, void *out,
                            size_t *used)
{
    size_t maxc = 4 * n + 4, lim = len < maxc ? len : maxc;
    unsigned T = 0;
    for (unsigned t = 1; t <= 256; t++) {
        if ((size_t)8 * t > len || rd_u64(s) != 0) break;
        int ok = 1;
        for (unsigned k = 1; k < t; k++) {
            unsigned long long a = rd_u64(s + 8 * k), b = rd_u64(s + 8 * (k - 1));
            if (a > maxc || a < b) { ok = 0; break; }
        }
        if (!ok) break;
        if ((size_t)8 * t + 5 <= maxc) T = t;
    }
    if (T == 0) T = 1;
    for (int attempt = 0; attempt < 2; attempt++) {
        size_t hdr = (size_t)8 * T, tbs = n / T, end = hdr;
        int bad = 0;
        /* a multi-chunk table must walk inside 4n + 4 bytes; one chunk is
         * walked as far as the buffer goes, as the reference walks it */
        lim = T > 1 ? (len < maxc ? len : maxc) : len;
        for (unsigned c = 0; c < T && !bad; c++) {
            size_t lo = c * tbs, hi = (c == T - 1) ? n : (c + 1) * tbs;
            if (lo >= hi) continue;
            size_t pos = hdr + (size_t)rd_u64(s + 8 * c);
            if (pos + 4 > lim) { bad = 1; break; }
            int prior = (int)rd_u32(s + pos);
            pos += 4;
            store_deq(out, dbl, lo, prior, eb);
            for (size_t i = lo + 1; i < hi; i += (size_t)B) {
                size_t m = (i + B > hi) ? hi - i : (size_t)B;
                if (pos >= lim) { bad = 1; break; }
                unsigned bc = s[pos++];
                if (bc > 32) { bad = 1; break; }
                const uint8_t *sg = s + pos, *mg = sg + (m + 7) / 8;
                if (bc) pos += (m + 7) / 8 + magnitude_bytes(m, bc);
                if (pos > lim) { bad = 1; break; }
                for (size_t j = 0; j < m; j++) {
                    if (bc) {
                        unsigned v = extract_mag(mg, j, m, bc);
                        int neg = (sg[j >> 3] >> (7 - (j & 7))) & 1;
                        prior = (int)((unsigned)prior + (neg ? 0u - v : v));
                    }
                    store_deq(out, dbl, i + j, prior, eb);
                }
            }
            if (pos > end) end = pos;
        }
        if (!bad) { if (used) *used = end; return 0; }
        if (T == 1) return -1;
        T = 1;
    }
    return -1;
}

/* ------------------------------------------------------------------ */
/* 2D post-processing (example/test_cuda_topology.cu:117-326, :493-531) */
/* ------------------------------------------------------------------ */

void ora_stencils_2d(float *d, const float *orig, const int *fn, const int *sp,
                     size_t n_sp, int rows, int cols, float eb)
{
    static const int nb[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    size_t k = 0;
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            size_t c = (size_t)i * cols + j;
            int t = fn[c];
            if (t != 1 && t != 2) continue;
            int s = (k < n_sp) ? sp[k] : 0;
            float hi = orig[c] + eb, lo = orig[c] - eb;
            float m = d[c], target;
            for (int q = 0; q < 4; q++) {
                float v = d[(size_t)(i + nb[q][0]) * cols + (j + nb[q][1])];
                if (t == 1 ? (v > m) : (v < m)) m = v;
            }
            if (t == 1) {
                target = m * (1.0f + ((float)s * FLT_EPSILON));
            } else if (s == 0) {
                target = m * (1.0f - FLT_EPSILON);
            } else {
                target = m * (1.0f - ((1.0f / (float)s) * FLT_EPSILON));
            }
            if (target > hi) target = hi;
            if (target < lo) target = lo;
            d[c] = target;
            k++;
        }
}

void ora_enforce_2d(float *d, const float *orig, const int *fn, int rows, int cols,
                    float eps, float eb)
{
    float soft = 0.25f * eps;
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            size_t c = (size_t)i * cols + j;
            float hi = orig[c] + eb * 0.999f, lo = orig[c] - eb * 0.999f;
            float n = d[c - cols], s = d[c + cols], w = d[c - 1], e = d[c + 1];
            if (fn[c] == 1) {
                float t = fmaxf(fmaxf(n, s), fmaxf(w, e)) + soft;
                if (t > hi) t = hi;
                if (t < lo) t = lo;
                if (d[c] < t) d[c] = t;
            } else if (fn[c] == 2) {
                float t = fminf(fminf(n, s), fminf(w, e)) - soft;
                if (t < lo) t = lo;
                if (t > hi) t = hi;
                if (d[c] > t) d[c] = t;
            }
        }
}

static float saddle_center_clamp(float cand, float n, float s, float w, float e, float eps)
{
    float lo = fminf(fmaxf(n, s), fmaxf(w, e)) - 0.25f * eps;
    float hi = fmaxf(fminf(n, s), fminf(w, e)) + 0.25f * eps;
    if (lo > hi) {
        float mid = 0.5f * (lo + hi);
        lo = mid - 0.25f * eps;
        hi = mid + 0.25f * eps;
    }
    if (cand < lo) cand = lo;
    if (cand > hi) cand = hi;
    return cand;
}

static int cls4_eps(float c, float n, float s, float w, float e, float eps)
{
    if (c > n + eps && c > s + eps && c > w + eps && c > e + eps) return 1;
    if (c < n - eps && c < s - eps && c < w - eps && c < e - eps) return 2;
    int vh = (c > n + eps) && (c > s + eps), vl = (c < n - eps) && (c < s - eps);
    int hh = (c > w + eps) && (c > e + eps), hl = (c < w - eps) && (c < e - eps);
    return ((vh && hl) || (vl && hh)) ? 3 : 0;
}

static int cls4_at(const float *d, int cols, int i, int j, float eps)
{
    size_t c = (size_t)i * cols + j;
    return cls4_eps(d[c], d[c - cols], d[c + cols], d[c - 1], d[c + 1], eps);
}

int ora_rbf_2d(float *d, const float *orig, const int *fn, int rows, int cols,
               float eps, float eb)
{
    size_t N = (size_t)rows * cols;
    uint8_t *lock = (uint8_t *)calloc(N, 1), *cand_mask = (uint8_t *)calloc(N, 1);
    size_t ncand = 0;
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            int t = fn[(size_t)i * cols + j];
            if (t != 1 && t != 2) continue;
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++) {
                    int ii = i + a, jj = j + b;
                    if (ii > 0 && ii < rows - 1 && jj > 0 && jj < cols - 1)
                        lock[(size_t)ii * cols + jj] = 1;
                }
        }
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            size_t c = (size_t)i * cols + j;
            if (fn[c] == 3 && ora_classify_2d(d, cols, i, j) != 3) { cand_mask[c] = 1; ncand++; }
        }
    int restored = 0;
    if (!ncand) { free(lock); free(cand_mask); return 0; }
    double s2 = 0.8 * 0.8, w[9];
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            w[(a + 1) * 3 + (b + 1)] = exp(-((double)a * a + b * b) / (2.0 * s2));
    for (int i = 1; i < rows - 1; i++)
        for (int j = 1; j < cols - 1; j++) {
            size_t c = (size_t)i * cols + j;
            if (!cand_mask[c] || fn[c] != 3) continue;
            double num = 0, den = 0;
            for (int a = -1; a <= 1; a++) {
                int ii = i + a;
                if (ii < 0 || ii >= rows) continue;
                for (int b = -1; b <= 1; b++) {
                    int jj = j + b;
                    if (jj < 0 || jj >= cols) continue;
                    double ww = w[(a + 1) * 3 + (b + 1)];
                    if (lock[(size_t)ii * cols + jj]) ww *= 0.4;
                    num += ww * d[(size_t)ii * cols + jj];
                    den += ww;
                }
            }
            if (den <= 0) continue;
            float old = d[c];
            float lo = orig[c] - eb * 0.999f, hi = orig[c] + eb * 0.999f;
            float cand = (float)(num / den);
            cand = saddle_center_clamp(cand, d[c - cols], d[c + cols], d[c - 1], d[c + 1], eps);
            if (cand < lo) cand = lo;
            if (cand > hi) cand = hi;
            float step = cand - old, alpha = 1.0f;
            for (int it = 0; it < 10; it++) {
                float trial = old + alpha * step;
                if (trial < lo) trial = lo;
                if (trial > hi) trial = hi;
                float saved = d[c];
                d[c] = trial;
                int bad = 0;
                if (i - 1 >= 1 && fn[c - cols] == 0 && cls4_at(d, cols, i - 1, j, eps) != 0) bad = 1;
                if (!bad && i + 1 < rows - 1 && fn[c + cols] == 0 && cls4_at(d, cols, i + 1, j, eps) != 0) bad = 1;
                if (!bad && j - 1 >= 1 && fn[c - 1] == 0 && cls4_at(d, cols, i, j - 1, eps) != 0) bad = 1;
                if (!bad && j + 1 < cols - 1 && fn[c + 1] == 0 && cls4_at(d, cols, i, j + 1, eps) != 0) bad = 1;
                if (!bad && cls4_at(d, cols, i, j, eps) != 3) bad = 1;
                if (bad) { d[c] = saved; alpha *= 0.5f; }
                else { restored++; break; }
            }
        }
    free(lock); free(cand_mask);
    return restored;
}

int ora_post_2d(float *d, const float *orig, const int *fn, const int *sp, size_t n_sp,
                int rows, int cols, float eb, int *restored)
{
    if (rows < 3 || cols < 3) { if (restored) *restored = 0; return 0; }
    if (sp && n_sp > 0) ora_stencils_2d(d, orig, fn, sp, n_sp, rows, cols, eb);
    float eps = fmaxf(1e-6f, 0.1f * eb);
    ora_enforce_2d(d, orig, fn, rows, cols, eps, eb);
    int r = ora_rbf_2d(d, orig, fn, rows, cols, eps, eb);
    if (restored) *restored = r;
    return 0;
}

/* ------------------------------------------------------------------ */
/* 3D post-processing (example/test_cuda_topology_3d.cu:75-434, :600-631) */
/* ------------------------------------------------------------------ */

void ora_stencils_3d(float *d, const float *orig, const int *fn, const int *sp,
                     size_t n_sp, int d1, int d2, int d3, float eb)
{
    size_t pl = (size_t)d2 * d3, k = 0;
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                size_t c = (size_t)x * pl + (size_t)y * d3 + z;
                int t = fn[c];
                if (t != 1 && t != 2) continue;
                int s = (k < n_sp) ? sp[k] : 0;
                float hi = orig[c] + eb * 0.999f, lo = orig[c] - eb * 0.999f;
                float xm = d[c - pl], xp = d[c + pl], ym = d[c - d3], yp = d[c + d3];
                float zm = d[c - 1], zp = d[c + 1], target;
                if (t == 1) {
                    float m = fmaxf(fmaxf(xm, xp), fmaxf(fmaxf(ym, yp), fmaxf(zm, zp)));
                    target = m * (1.0f + (float)s * FLT_EPSILON);
                } else {
                    float m = fminf(fminf(xm, xp), fminf(fminf(ym, yp), fminf(zm, zp)));
                    target = (s == 0) ? m * (1.0f - FLT_EPSILON)
                                      : m * (1.0f - (1.0f / (float)s) * FLT_EPSILON);
                }
                if (target > hi) target = hi;
                if (target < lo) target = lo;
                d[c] = target;
                k++;
            }
}

void ora_enforce_3d(float *d, const float *orig, const int *fn, int d1, int d2, int d3,
                    float eps, float eb)
{
    float soft = 0.25f * eps;
    size_t pl = (size_t)d2 * d3;
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                size_t c = (size_t)x * pl + (size_t)y * d3 + z;
                int t = fn[c];
                if (t != 1 && t != 2) continue;
                float hi = orig[c] + eb * 0.999f, lo = orig[c] - eb * 0.999f;
                float xm = d[c - pl], xp = d[c + pl], ym = d[c - d3], yp = d[c + d3];
                float zm = d[c - 1], zp = d[c + 1];
                if (t == 1) {
                    float v = fmaxf(fmaxf(xm, xp), fmaxf(fmaxf(ym, yp), fmaxf(zm, zp))) + soft;
                    if (v > hi) v = hi;
                    if (v < lo) v = lo;
                    if (d[c] < v) d[c] = v;
                } else {
                    float v = fminf(fminf(xm, xp), fminf(fminf(ym, yp), fminf(zm, zp))) - soft;
                    if (v < lo) v = lo;
                    if (v > hi) v = hi;
                    if (d[c] > v) d[c] = v;
                }
            }
}

static int regular_neighbours_stay_3d(const float *d, const int *fn, int d1, int d2, int d3,
                                      int x, int y, int z)
{
    size_t pl = (size_t)d2 * d3, c = (size_t)x * pl + (size_t)y * d3 + z;
    if (x - 1 >= 1 && fn[c - pl] == 0 && ora_classify_3d(d, d2, d3, x - 1, y, z) != 0) return 0;
    if (x + 1 < d1 - 1 && fn[c + pl] == 0 && ora_classify_3d(d, d2, d3, x + 1, y, z) != 0) return 0;
    if (y - 1 >= 1 && fn[c - d3] == 0 && ora_classify_3d(d, d2, d3, x, y - 1, z) != 0) return 0;
    if (y + 1 < d2 - 1 && fn[c + d3] == 0 && ora_classify_3d(d, d2, d3, x, y + 1, z) != 0) return 0;
    if (z - 1 >= 1 && fn[c - 1] == 0 && ora_classify_3d(d, d2, d3, x, y, z - 1) != 0) return 0;
    if (z + 1 < d3 - 1 && fn[c + 1] == 0 && ora_classify_3d(d, d2, d3, x, y, z + 1) != 0) return 0;
    return 1;
}

int ora_rbf_3d(float *d, const float *orig, const int *fn, int d1, int d2, int d3,
               float eps, float eb)
{
    (void)eps;
    size_t pl = (size_t)d2 * d3, N = (size_t)d1 * pl;
    uint8_t *lock = (uint8_t *)calloc(N, 1), *cand_mask = (uint8_t *)calloc(N, 1);
    size_t ncand = 0;
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                int t = fn[(size_t)x * pl + (size_t)y * d3 + z];
                if (t != 1 && t != 2) continue;
                for (int a = -1; a <= 1; a++)
                    for (int b = -1; b <= 1; b++)
                        for (int g = -1; g <= 1; g++) {
                            int xx = x + a, yy = y + b, zz = z + g;
                            if (xx >= 1 && xx < d1 - 1 && yy >= 1 && yy < d2 - 1 &&
                                zz >= 1 && zz < d3 - 1)
                                lock[(size_t)xx * pl + (size_t)yy * d3 + zz] = 1;
                        }
            }
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                size_t c = (size_t)x * pl + (size_t)y * d3 + z;
                if (fn[c] == 3 && ora_classify_3d(d, d2, d3, x, y, z) != 3) { cand_mask[c] = 1; ncand++; }
            }
    int restored = 0;
    if (!ncand) { free(lock); free(cand_mask); return 0; }
    double s2 = 0.8 * 0.8, w[27];
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int g = -1; g <= 1; g++)
                w[(a + 1) * 9 + (b + 1) * 3 + (g + 1)] =
                    exp(-(double)(a * a + b * b + g * g) / (2.0 * s2));
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                size_t c = (size_t)x * pl + (size_t)y * d3 + z;
                if (!cand_mask[c] || fn[c] != 3) continue;
                double num = 0, den = 0;
                for (int a = -1; a <= 1; a++) {
                    int xx = x + a;
                    if (xx < 0 || xx >= d1) continue;
                    for (int b = -1; b <= 1; b++) {
                        int yy = y + b;
                        if (yy < 0 || yy >= d2) continue;
                        for (int g = -1; g <= 1; g++) {
                            int zz = z + g;
                            if (zz < 0 || zz >= d3) continue;
                            size_t q = (size_t)xx * pl + (size_t)yy * d3 + zz;
                            double ww = w[(a + 1) * 9 + (b + 1) * 3 + (g + 1)];
                            if (lock[q]) ww *= 0.4;
                            num += ww * d[q];
                            den += ww;
                        }
                    }
                }
                if (den <= 0) continue;
                float old = d[c];
                float lo = orig[c] - eb * 0.999f, hi = orig[c] + eb * 0.999f;
                float cand = (float)(num / den);
                if (cand < lo) cand = lo;
                if (cand > hi) cand = hi;
                float step = cand - old, alpha = 1.0f;
                for (int it = 0; it < 10; it++) {
                    float trial = old + alpha * step;
                    if (trial < lo) trial = lo;
                    if (trial > hi) trial = hi;
                    float saved = d[c];
                    d[c] = trial;
                    int bad = ora_classify_3d(d, d2, d3, x, y, z) != 3;
                    if (!bad && !regular_neighbours_stay_3d(d, fn, d1, d2, d3, x, y, z)) bad = 1;
                    if (bad) { d[c] = saved; alpha *= 0.5f; }
                    else { restored++; break; }
                }
            }
    free(lock); free(cand_mask);
    return restored;
}

/* Axis-pattern saddle repair: defined in the reference driver but not
 * invoked there (example/test_cuda_topology_3d.cu:187-314); here an opt-in
 * stage run after the RBF pass. */
int ora_axis_saddles_3d(float *d, const float *orig, const int *fn, int d1, int d2, int d3,
                        float eb)
{
    size_t pl = (size_t)d2 * d3;
    int restored = 0;
    for (int x = 1; x < d1 - 1; x++)
        for (int y = 1; y < d2 - 1; y++)
            for (int z = 1; z < d3 - 1; z++) {
                size_t c = (size_t)x * pl + (size_t)y * d3 + z;
                if (fn[c] != 3) continue;
                if (ora_classify_3d(d, d2, d3, x, y, z) == 3) continue;
                float hi = orig[c] + eb * 0.999f, lo = orig[c] - eb * 0.999f;
                float nb[6] = {d[c - pl], d[c + pl], d[c - d3], d[c + d3], d[c - 1], d[c + 1]};
                int fixed = 0;
                for (int pat = 1; pat <= 6 && !fixed; pat++) {
                    float hthr = -1e30f, lthr = 1e30f;
                    for (int ax = 0; ax < 3; ax++) {
                        float pmax = fmaxf(nb[2 * ax], nb[2 * ax + 1]);
                        float pmin = fminf(nb[2 * ax], nb[2 * ax + 1]);
                        if ((pat >> ax) & 1) { if (pmax > hthr) hthr = pmax; }
                        else { if (pmin < lthr) lthr = pmin; }
                    }
                    if (hthr >= lthr) continue;
                    float target = 0.5f * (hthr + lthr);
                    float nudge = (lthr - hthr) * 0.01f;
                    if (nudge < FLT_EPSILON) nudge = FLT_EPSILON;
                    if (target <= hthr) target = hthr + nudge;
                    if (target >= lthr) target = lthr - nudge;
                    if (target <= hthr || target >= lthr) continue;
                    if (target > hi || target < lo) continue;
                    float saved = d[c];
                    d[c] = target;
                    int bad = ora_classify_3d(d, d2, d3, x, y, z) != 3;
                    if (!bad && !regular_neighbours_stay_3d(d, fn, d1, d2, d3, x, y, z)) bad = 1;
                    if (bad) d[c] = saved;
                    else { restored++; fixed = 1; }
                }
            }
    return restored;
}

int ora_post_3d(float *d, const float *orig, const int *fn, const int *sp, size_t n_sp,
                int d1, int d2, int d3, float eb, int axis_stencil, int *restored)
{
    if (d1 < 3 || d2 < 3 || d3 < 3) { if (restored) *restored = 0; return 0; }
    if (sp && n_sp > 0) ora_stencils_3d(d, orig, fn, sp, n_sp, d1, d2, d3, eb);
    float eps = fmaxf(1e-6f, 0.1f * eb);
    ora_enforce_3d(d, orig, fn, d1, d2, d3, eps, eb);
    int r = ora_rbf_3d(d, orig, fn, d1, d2, d3, eps, eb);
    if (axis_stencil) r += ora_axis_saddles_3d(d, orig, fn, d1, d2, d3, eb);
    if (restored) *restored = r;
    return 0;
}

/* (SZp/include/szp_errbound.h:34-53) */
float ora_rel_to_abs(const float *d, size_t n, float rel)
{
    float mn = d[0], mx = d[0];
    for (size_t i = 1; i < n; i++) {
        if (d[i] < mn) mn = d[i];
        if (d[i] > mx) mx = d[i];
    }
    float r = mx - mn;
    if (r <= 0) r = FLT_EPSILON;
    return rel * r;
}
