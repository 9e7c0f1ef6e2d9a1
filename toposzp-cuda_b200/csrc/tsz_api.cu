// C ABI: the reference's topology entry points (host pointers, malloc'd
// results) and the device-pointer additions.
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "tsz_enc64.h"
#include "tsz_ops.h"

namespace tsz {

__global__ void mark_types_kernel(const int *__restrict__ cps, int stride, long long count, int nd,
                                  long long d1, long long d2, long long d3, unsigned long long n,
                                  unsigned char *__restrict__ types) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int *r = cps + (long long)stride * i;
  long long flat;
  int t;
  if (nd == 2) {
    int x = r[0], y = r[1];
    t = r[2];
    if (x < 0 || x >= d2 || y < 0 || y >= d3) return;
    flat = (long long)x * d3 + y;
  } else {
    int x = r[0], y = r[1], z = r[2];
    t = r[3];
    if (x < 0 || x >= d1 || y < 0 || y >= d2 || z < 0 || z >= d3) return;
    flat = (long long)x * d2 * d3 + (long long)y * d3 + z;
  }
  if (t >= 1 && t <= 3 && (unsigned long long)flat < n) types[flat] = (unsigned char)t;
}

Geom make_geom(int nd, long long a, long long b, long long c) {
  Geom g;
  g.nd = nd;
  if (nd == 2) { g.d1 = 1; g.d2 = a; g.d3 = b; }
  else { g.d1 = a; g.d2 = b; g.d3 = c; }
  g.plane = g.d2 * g.d3;
  g.m_d3 = magic_u64((unsigned long long)(g.d3 > 0 ? g.d3 : 1));
  g.m_plane = magic_u64((unsigned long long)(g.plane > 0 ? g.plane : 1));
  return g;
}

bool geom_elements(const szp_b200_geom &g, unsigned long long *n, Geom *out) {
  unsigned long long p = 1;
  if (g.nd != 2 && g.nd != 3) return false;
  for (int i = 0; i < g.nd; i++) {
    if (g.dims[i] <= 0) return false;
    if (__builtin_mul_overflow(p, (unsigned long long)g.dims[i], &p)) return false;
  }
  // the product of the extents must not wrap, and flat indices +- one plane
  // stay far inside 64 bits
  if (p >= kMaxElements) return false;
  *out = (g.nd == 2) ? make_geom(2, g.dims[0], g.dims[1], 1) : make_geom(3, g.dims[0], g.dims[1], g.dims[2]);
  *n = p;
  return true;
}

static size_t stream_bound(unsigned long long n, int B, bool tags);

int ctx_reserve_for(szp_b200_ctx *ctx, unsigned long long n, int B) {
  DeviceGuard dg(ctx);
  if (!ctx || n == 0 || B <= 0) { set_error("ctx_reserve_for: invalid arguments"); return -1; }
  const unsigned long long nb = (n + B - 1) / B;
  // the largest scratch of a fused compression and of a fused decompression
  // with post-processing and device stream parsing
  const size_t comp = a256(n * 8) + a256(n * 4) + a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) * 2 +
                      rank_scratch_bytes(n, ctx->sm_count) + 8192;
  const size_t dec = post_scratch_bytes(n) + a256(n * 4) + a256(n) + 8192 + a256(2 * nb * 8) +
                     parse_scratch_bytes(stream_bound(n, B, true) - 8, B, true) +
                     parse_scratch_bytes(stream_bound(n, B, false) - 8, B, false);
  if (!ctx->scratch.reserve(comp > dec ? comp : dec)) return -1;
  return post_words(ctx, n) ? 0 : -1;
}

static bool check_block_size(int B, const char *fn) {
  if (B <= 0 || B > kMaxBlockSize) {
    set_error("%s: blockSize %d out of range [1, %d]", fn, B, kMaxBlockSize);
    return false;
  }
  return true;
}

static size_t stream_bound(unsigned long long n, int B, bool tags) {
  unsigned long long nb = (n + B - 1) / B;
  return 8 + nb * (size_t)max_block_bytes((uint32_t)B, tags) + 64;
}

size_t topo_stream_bound(unsigned long long n, int B) { return stream_bound(n, B, true); }

bool valid_block_size(int B, const char *fn) { return check_block_size(B, fn); }

cudaError_t launch_mark_types(const int *d_cps, int stride, long long count, const Geom &g, unsigned long long n,
                              unsigned char *d_types, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((count + 255) / 256);
  mark_types_kernel<<<blocks, 256, 0, s>>>(d_cps, stride, count, g.nd, g.d1, g.d2, g.d3, n, d_types);
  return cudaGetLastError();
}

int encode_pass(szp_b200_ctx *ctx, int mode, const float *d_data, const int *d_ints,
                const unsigned char *d_types, unsigned long long n, int B, float eb,
                const Geom &g, unsigned char *d_stream, unsigned long long stream_cap,
                unsigned long long *d_blk_off, int cp_mode, void *d_cp, unsigned long long cp_cap,
                unsigned long long totals_out[3]) {
  cudaStream_t s = ctx->stream;
  const unsigned long long nb = (n + B - 1) / B;
  const int TB = enc_tile_blocks(B);
  const unsigned long long ntiles = (nb + TB - 1) / TB;
  TileDesc *desc = ctx->scratch.take<TileDesc>(ntiles + 1);
  if (!desc) { set_error("scratch arena too small for tile descriptors"); return -1; }
  unsigned long long *w = ctx->d_words;  // [0..2] totals, [3] tile counter, [4] err
  if (cuda_fail(cudaMemsetAsync(desc, 0, (ntiles + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(w, 0, 8 * sizeof(unsigned long long), s), "memset"))
    return -1;
  if (d_stream && cuda_fail(cudaMemsetAsync(d_stream, 0, 8, s), "memset")) return -1;
  EncArgs a{};
  a.data = d_data;
  a.ints = d_ints;
  a.types = d_types;
  a.n = n;
  a.B = B;
  a.eb = eb;
  a.inv = 1.0 / (double)eb;
  a.g = g;
  a.out = d_stream ? d_stream + 8 : nullptr;
  a.out_cap = d_stream ? (stream_cap > 8 ? stream_cap - 8 : 0) : 0;
  a.blk_off = d_blk_off;
  a.desc = desc;
  a.tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  a.err = reinterpret_cast<int *>(w + 4);
  a.total = w;
  a.cp_mode = cp_mode;
  a.cp_out = d_cp;
  a.cp_cap = cp_cap;
  int grid = (int)std::min<unsigned long long>(ntiles, (unsigned long long)ctx->sm_count * 8ull);
  if (grid < 1) grid = 1;
  if (cuda_fail(enc64_applies(a, mode) ? launch_enc64_from(a, s, ctx->sm_count) : launch_encode(mode, a, s, grid),
                "encode launch"))
    return -1;
  ctx->launches += 1;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 8 * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, s), "D2H totals") ||
      cuda_fail(cudaStreamSynchronize(s), "encode"))
    return -1;
  int err = (int)(ctx->h_words[4] & 0xffffffffu);
  if (err) { set_error("encoder reported status %d", err); return -1; }
  totals_out[0] = ctx->h_words[0];
  totals_out[1] = ctx->h_words[1];
  totals_out[2] = ctx->h_words[2];
  return 0;
}

// Topology encode of a field that is still on its way from the host: the copy
// runs in parts on the copy stream and the encoder runs one launch per part,
// over the tiles whose reads (the tile, and one plane -- one row in 2D --
// beyond it) the copied data already covers.  Tiles leave the launches in
// order, so the look-back of a launch only meets completed tiles of earlier
// launches.  Same results as one encode_pass over the whole field.  With
// h_out set, the stream goes to the host part by part on the copy stream as
// the launches finish (the caller waits for the copy stream).
static int encode_topo_chunked(szp_b200_ctx *ctx, const float *h_src, float *d_data, unsigned long long n, int B,
                               float eb, const Geom &g, unsigned char *d_stream, unsigned long long stream_cap,
                               unsigned long long *d_blk_off, void *d_cp, unsigned long long cp_cap,
                               unsigned long long totals_out[3], unsigned char *h_out, size_t out_cap) {
  cudaStream_t s = ctx->stream;
  cudaStream_t cs = copy_stream(ctx);
  if (!cs) return -1;
  const int K = 8;
  const unsigned long long nb = (n + B - 1) / B;
  const unsigned long long TB = (unsigned long long)enc_tile_blocks(B);
  const unsigned long long TE = TB * (unsigned long long)B;   // elements per tile
  const unsigned long long ntiles = (nb + TB - 1) / TB;
  const unsigned long long halo = (g.nd == 3 ? (unsigned long long)g.plane : (unsigned long long)g.d3) + 1;
  unsigned long long cut[K + 1];
  cut[0] = 0;
  for (int k = 1; k < K; k++) cut[k] = std::min<unsigned long long>(n, (n / K * k) / TE * TE);
  cut[K] = n;
  for (int k = 0; k < K; k++) {
    if (!ctx->chunk_ev[k] && cuda_fail(cudaEventCreateWithFlags(&ctx->chunk_ev[k], cudaEventDisableTiming), "event"))
      return -1;
    if (cut[k + 1] > cut[k] &&
        cuda_fail(cudaMemcpyAsync(d_data + cut[k], h_src + cut[k], (cut[k + 1] - cut[k]) * 4, cudaMemcpyHostToDevice,
                                  cs), "H2D field"))
      return -1;
    if (cuda_fail(cudaEventRecord(ctx->chunk_ev[k], cs), "event")) return -1;
  }
  TileDesc *desc = ctx->scratch.take<TileDesc>(ntiles + 1);
  if (!desc) { set_error("scratch arena too small for tile descriptors"); return -1; }
  unsigned long long *w = ctx->d_words;  // [0..2] totals, [3] tile counter, [4] err
  if (cuda_fail(cudaMemsetAsync(desc, 0, (ntiles + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(w, 0, 8 * sizeof(unsigned long long), s), "memset") ||
      cuda_fail(cudaMemsetAsync(d_stream, 0, 8, s), "memset"))
    return -1;
  EncArgs a{};
  a.data = d_data;
  a.n = n;
  a.B = B;
  a.eb = eb;
  a.inv = 1.0 / (double)eb;
  a.g = g;
  a.out = d_stream + 8;
  a.out_cap = stream_cap > 8 ? stream_cap - 8 : 0;
  a.blk_off = d_blk_off;
  a.tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  a.err = reinterpret_cast<int *>(w + 4);
  a.total = w;
  a.desc = desc;
  a.cp_mode = kCpPairs;
  a.cp_out = d_cp;
  a.cp_cap = cp_cap;
  unsigned long long done = 0;
  int parts = 0;
  for (int k = 0; k < K; k++) {
    if (cuda_fail(cudaStreamWaitEvent(s, ctx->chunk_ev[k], 0), "wait")) return -1;
    // tiles whose reads end inside [0, cut[k+1])
    unsigned long long upto = ntiles;
    if (k < K - 1) upto = cut[k + 1] > halo ? std::min<unsigned long long>(ntiles, (cut[k + 1] - halo) / TE) : 0;
    if (upto <= done) continue;
    a.tile_lo = done;
    a.tile_hi = upto;
    if (cuda_fail(cudaMemsetAsync(w + 3, 0, 8, s), "memset")) return -1;
    const int grid = (int)std::min<unsigned long long>(upto - done, (unsigned long long)ctx->sm_count * 8ull);
    if (cuda_fail(enc64_applies(a, kEncClassify) ? launch_enc64_from(a, s, ctx->sm_count)
                                                 : launch_encode(kEncClassify, a, s, grid),
                  "encode launch"))
      return -1;
    ctx->launches += 1;
    done = upto;
    if (h_out && upto < ntiles) {
      // stream bytes through the launch's last tile: its inclusive status word
      if (!ctx->part_ev[parts] &&
          cuda_fail(cudaEventCreateWithFlags(&ctx->part_ev[parts], cudaEventDisableTiming), "event"))
        return -1;
      if (cuda_fail(cudaMemcpyAsync(ctx->h_words + 32 + parts, &desc[upto - 1].status, 8, cudaMemcpyDeviceToHost,
                                    s), "D2H") ||
          cuda_fail(cudaEventRecord(ctx->part_ev[parts], s), "event"))
        return -1;
      parts++;
    }
  }
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
                "D2H totals"))
    return -1;
  // as each launch finishes, its part of the stream leaves for the host on a
  // stream of its own (the copy stream still carries the field's later parts)
  cudaStream_t ds = h_out ? d2h_stream(ctx) : nullptr;
  if (h_out && !ds) return -1;
  unsigned long long sent = 0;   // stream bytes (header included) already queued
  for (int p = 0; p < parts; p++) {
    if (cuda_fail(cudaEventSynchronize(ctx->part_ev[p]), "encode")) return -1;
    const unsigned long long st = ctx->h_words[32 + p];
    if ((st >> kStatShift) != 2ull) break;   // not an inclusive prefix: left to the final copy
    const unsigned long long upto_bytes = 8 + (st & kByteMask);
    if (upto_bytes > out_cap || upto_bytes > stream_cap) break;
    if (upto_bytes > sent &&
        cuda_fail(cudaMemcpyAsync(h_out + sent, d_stream + sent, upto_bytes - sent, cudaMemcpyDeviceToHost, ds),
                  "D2H stream"))
      return -1;
    sent = upto_bytes > sent ? upto_bytes : sent;
  }
  if (cuda_fail(cudaStreamSynchronize(s), "encode")) return -1;
  const int err = (int)(ctx->h_words[4] & 0xffffffffu);
  if (err) { set_error("encoder reported status %d", err); return -1; }
  if (h_out) {
    const unsigned long long total = 8 + ctx->h_words[0];
    if (total > out_cap) { set_error("topology output buffer too small (%llu bytes needed)", total); return -1; }
    if (total > sent &&
        cuda_fail(cudaMemcpyAsync(h_out + sent, d_stream + sent, total - sent, cudaMemcpyDeviceToHost, ds),
                  "D2H stream"))
      return -1;
  }
  totals_out[0] = ctx->h_words[0];
  totals_out[1] = ctx->h_words[1];
  totals_out[2] = ctx->h_words[2];
  return 0;
}

// ---------------------------------------------------------------------------
// host-side walk of a foreign stream: the reference's offset-table thread-count
// detection and block walk (SZp/src/szp_cuda_decompress.cu:233-328, 339-477).
// The reference interface carries no stream length, so the length is
// discovered here (and the copy to the device sized from it).
// ---------------------------------------------------------------------------
static inline unsigned long long rd64(const unsigned char *p) {
  unsigned long long v;
  memcpy(&v, p, 8);
  return v;
}

static bool span_one(const unsigned char *s, unsigned long long pos, unsigned long long lim,
                     unsigned long long len, bool tags, bool check, unsigned long long *next) {
  if (check && pos + 4 > lim) return false;
  unsigned long long p = pos + 4;
  if (len > 1) {
    if (check && p >= lim) return false;
    unsigned bc = s[p++];
    if (bc > 32) return false;
    if (bc) p += (len - 2) / 8 + 1 + mag_bytes((uint32_t)(len - 1), bc);
    if (check && p > lim) return false;
  }
  if (tags) p += (2 * len + 7) / 8;
  if (check && p > lim) return false;
  *next = p;
  return true;
}

// Fills per-block payload offsets (relative to the end of the offset table);
// returns false on a malformed stream.
// buf_len bounds every read when the caller knows the stream length (the
// reference interface does not: ~0 then, as in the reference).
static bool walk_stream(const unsigned char *s, unsigned long long n, int B, bool tags,
                        std::vector<unsigned long long> &offs, unsigned long long &hdr,
                        unsigned long long &payload_len, unsigned long long buf_len = ~0ull) {
  const unsigned long long nb = (n + B - 1) / B;
  const unsigned long long maxc = std::min<unsigned long long>(tags ? 8ull * n + 1024 : 4ull * n + 4, buf_len);
  const bool bounded = buf_len != ~0ull;
  if (buf_len < 8) return false;
  unsigned T = 1;
  if (rd64(s) == 0) {
    for (unsigned t = 1; t <= 128; t++) {
      if (8ull * t > buf_len) break;
      bool ok = true;
      for (unsigned k = 1; k < t; k++) {
        unsigned long long a = rd64(s + 8 * k), b = rd64(s + 8 * (k - 1));
        if (a > maxc || a < b) { ok = false; break; }
      }
      if (!ok) break;
      const unsigned long long h = 8ull * t;
      bool valid = true;
      if (tags) {
        const unsigned long long bpt = (nb + t - 1) / t;
        for (unsigned c = 0; c < t && valid; c++) {
          unsigned long long pos = h + rd64(s + 8 * c);
          if (pos >= maxc) { valid = false; break; }
          unsigned long long b1 = std::min<unsigned long long>((c + 1) * bpt, nb);
          for (unsigned long long b = c * bpt; b < b1; b++) {
            unsigned long long e0 = b * B, m = std::min<unsigned long long>(B, n - e0);
            if (!span_one(s, pos, maxc, m, true, true, &pos)) { valid = false; break; }
          }
        }
      } else {
        const unsigned long long tbs = n / t;
        for (unsigned c = 0; c < t && valid; c++) {
          unsigned long long lo = c * tbs, hi = (c == t - 1) ? n : (c + 1) * tbs;
          unsigned long long pos = h + rd64(s + 8 * c);
          if (pos >= maxc) { valid = false; break; }
          for (unsigned long long i = lo; i < hi; i += B) {
            unsigned long long m = std::min<unsigned long long>(B, hi - i);
            if (!span_one(s, pos, maxc, m, false, true, &pos)) { valid = false; break; }
          }
        }
      }
      if (valid) { T = t; break; }
    }
  }
  // Deviation: the reference accepts a multi-chunk table whose chunks overlap
  // (possible when a one-chunk stream exceeds its validation bound, e.g. a
  // sort-position stream with blockSize 1) and then decodes garbage.  Chunks
  // that start before their predecessor ends mean the stream is one chunk.
  if (T > 1) {
    unsigned long long prev_end = 0;
    const unsigned long long h = 8ull * T;
    bool overlap = false;
    for (unsigned c = 0; c < T && !overlap; c++) {
      unsigned long long pos = h + rd64(s + 8 * c);
      if (pos < prev_end) { overlap = true; break; }
      if (tags) {
        const unsigned long long bpt = (nb + T - 1) / T;
        unsigned long long b1 = std::min<unsigned long long>((c + 1) * bpt, nb);
        for (unsigned long long b = c * bpt; b < b1; b++) {
          unsigned long long e0 = b * B, m = std::min<unsigned long long>(B, n - e0);
          if (!span_one(s, pos, buf_len, m, true, bounded, &pos)) { overlap = true; break; }
        }
      } else {
        const unsigned long long tbs = n / T;
        unsigned long long lo = c * tbs, hi = (c == T - 1) ? n : (c + 1) * tbs;
        for (unsigned long long i = lo; i < hi; i += B) {
          unsigned long long m = std::min<unsigned long long>(B, hi - i);
          if (!span_one(s, pos, buf_len, m, false, bounded, &pos)) { overlap = true; break; }
        }
      }
      prev_end = pos;
    }
    if (overlap) T = 1;
  }
  hdr = 8ull * T;
  offs.resize(nb);
  unsigned long long end = hdr;
  if (tags) {
    const unsigned long long bpt = (nb + T - 1) / T;
    for (unsigned c = 0; c < T; c++) {
      unsigned long long pos = hdr + rd64(s + 8 * c);
      unsigned long long b1 = std::min<unsigned long long>((c + 1) * bpt, nb);
      for (unsigned long long b = c * bpt; b < b1; b++) {
        unsigned long long e0 = b * B, m = std::min<unsigned long long>(B, n - e0);
        offs[b] = pos - hdr;
        if (!span_one(s, pos, buf_len, m, true, bounded, &pos)) return false;
        if (pos > end) end = pos;
      }
    }
  } else {
    const unsigned long long tbs = n / T;
    unsigned long long b = 0;
    for (unsigned c = 0; c < T; c++) {
      unsigned long long lo = c * tbs, hi = (c == T - 1) ? n : (c + 1) * tbs;
      unsigned long long pos = hdr + rd64(s + 8 * c);
      for (unsigned long long i = lo; i < hi && b < nb; i += B, b++) {
        unsigned long long m = std::min<unsigned long long>(B, hi - i);
        offs[b] = pos - hdr;
        if (!span_one(s, pos, buf_len, m, false, bounded, &pos)) return false;
        if (pos > end) end = pos;
      }
    }
  }
  payload_len = end - hdr;
  return true;
}

// ---------------------------------------------------------------------------
// shared host paths
// ---------------------------------------------------------------------------

// H2D of a host field + types from a CP list + encode; returns a malloc'd stream.
static unsigned char *compress_host_path(const char *fn, const float *h_data, size_t *outSize,
                                         float eb, size_t n, int B, const int *h_cps, int count,
                                         int stride, int nd, long long d1, long long d2,
                                         long long d3) {
  *outSize = 0;
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  const size_t cap = stream_bound(n, B, true);
  const size_t cps_bytes = (h_cps && count > 0) ? (size_t)count * stride * sizeof(int) : 0;
  const unsigned long long nb = (n + B - 1) / B;
  const size_t need = a256(n * 4) + a256(n) + a256(cap) + a256(cps_bytes) +
                      a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) + 4096;
  if (!ctx->scratch.reserve(need)) return nullptr;
  float *d_data = ctx->scratch.take<float>(n);
  unsigned char *d_types = ctx->scratch.take<unsigned char>(n);
  unsigned char *d_stream = ctx->scratch.take<unsigned char>(cap);
  int *d_cps = cps_bytes ? ctx->scratch.take<int>((size_t)count * stride) : nullptr;
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_data, h_data, n * 4, cudaMemcpyHostToDevice, s), "H2D data") ||
      cuda_fail(cudaMemsetAsync(d_types, 0, n, s), "memset types"))
    return nullptr;
  if (d_cps) {
    if (cuda_fail(cudaMemcpyAsync(d_cps, h_cps, cps_bytes, cudaMemcpyHostToDevice, s), "H2D cps"))
      return nullptr;
    const unsigned blocks = (unsigned)((count + 255) / 256);
    Geom g = make_geom(nd, d1, d2, d3);
    mark_types_kernel<<<blocks, 256, 0, s>>>(d_cps, stride, count, nd, g.d1, g.d2, g.d3, n, d_types);
    ctx->launches += 1;
    if (cuda_fail(cudaGetLastError(), "mark types")) return nullptr;
  }
  unsigned long long tot[3];
  Geom g = make_geom(nd, d1, d2, d3);
  if (encode_pass(ctx, kEncTypes, d_data, nullptr, d_types, n, B, eb, g, d_stream, cap, nullptr,
                  kCpNone, nullptr, 0, tot))
    return nullptr;
  const size_t total = 8 + tot[0];
  unsigned char *out = (unsigned char *)malloc(total);
  if (!out) { set_error("%s: host allocation failed", fn); return nullptr; }
  if (cuda_fail(cudaMemcpyAsync(out, d_stream, total, cudaMemcpyDeviceToHost, s), "D2H stream") ||
      cuda_fail(cudaStreamSynchronize(s), "sync")) {
    free(out);
    return nullptr;
  }
  *outSize = total;
  return out;
}

static void *find_host_path(const float *h_data, size_t *outCount, int nd, long long d1,
                            long long d2, long long d3, float eb) {
  *outCount = 0;
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  Geom g = make_geom(nd, d1, d2, d3);
  const unsigned long long n = (unsigned long long)(g.d1 * g.d2 * g.d3);
  const unsigned long long interior =
      (nd == 2) ? (unsigned long long)(d1 - 2) * (d2 - 2)
                : (unsigned long long)(d1 - 2) * (d2 - 2) * (d3 - 2);
  const int rec = (nd == 2) ? 5 : 6;
  const int B = 64;
  const unsigned long long nb = (n + B - 1) / B;
  const size_t need = a256(n * 4) + a256(interior * rec * 4) +
                      a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) + 4096;
  if (!ctx->scratch.reserve(need)) return nullptr;
  float *d_data = ctx->scratch.take<float>(n);
  int *d_rec = ctx->scratch.take<int>(interior * rec);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_data, h_data, n * 4, cudaMemcpyHostToDevice, s), "H2D data"))
    return nullptr;
  unsigned long long tot[3];
  if (encode_pass(ctx, kEncClassify, d_data, nullptr, nullptr, n, B, eb, g, nullptr, 0, nullptr,
                  kCpRecords, d_rec, interior, tot))
    return nullptr;
  const unsigned long long k = tot[1];
  if (k == 0) return nullptr;
  void *out = malloc(k * rec * 4);
  if (!out) { set_error("host allocation failed"); return nullptr; }
  if (cuda_fail(cudaMemcpyAsync(out, d_rec, k * rec * 4, cudaMemcpyDeviceToHost, s), "D2H cps") ||
      cuda_fail(cudaStreamSynchronize(s), "sync")) {
    free(out);
    return nullptr;
  }
  *outCount = k;
  return out;
}

}  // namespace tsz

using namespace tsz;

// ---------------------------------------------------------------------------
// reference entry points
// ---------------------------------------------------------------------------
extern "C" {

CriticalPoint *szp_cuda_find_critical_points(float *data, size_t *outCount, int rows, int cols,
                                              float absErrBound) {
  clear_error();
  if (!data || rows <= 2 || cols <= 2) { *outCount = 0; return nullptr; }
  return (CriticalPoint *)find_host_path(data, outCount, 2, rows, cols, 1, absErrBound);
}

CriticalPoint3D *szp_cuda_find_critical_points_3d(float *data, size_t *outCount, int d1, int d2,
                                                   int d3, float absErrBound) {
  clear_error();
  if (!data || d1 <= 2 || d2 <= 2 || d3 <= 2) { *outCount = 0; return nullptr; }
  return (CriticalPoint3D *)find_host_path(data, outCount, 3, d1, d2, d3, absErrBound);
}

unsigned char *szp_cuda_float_compress_randomaccess_topology_preserved(
    float *oriData, size_t *outSize, float absErrBound, size_t nbEle, int blockSize,
    CriticalPoint *critical_points, int critical_count, int rows, int cols) {
  clear_error();
  if (absErrBound <= 0.0f || !oriData || nbEle == 0) { *outSize = 0; return nullptr; }
  *outSize = 0;
  if (!check_block_size(blockSize, "szp_cuda_float_compress_randomaccess_topology_preserved"))
    return nullptr;
  if (rows <= 0 || cols <= 0) {
    set_error("invalid dimensions %d x %d", rows, cols);
    return nullptr;
  }
  return compress_host_path("szp_cuda_float_compress_randomaccess_topology_preserved", oriData,
                            outSize, absErrBound, nbEle, blockSize,
                            reinterpret_cast<const int *>(critical_points), critical_count, 5, 2,
                            rows, cols, 1);
}

unsigned char *szp_cuda_float_compress_topology_3d(float *oriData, size_t *outSize,
                                                   float absErrBound, size_t nbEle, int blockSize,
                                                   CriticalPoint3D *critical_points,
                                                   int critical_count, int d1, int d2, int d3) {
  clear_error();
  if (absErrBound <= 0.0f || !oriData || nbEle == 0) { *outSize = 0; return nullptr; }
  *outSize = 0;
  if (!check_block_size(blockSize, "szp_cuda_float_compress_topology_3d")) return nullptr;
  if (d1 <= 0 || d2 <= 0 || d3 <= 0) {
    set_error("invalid dimensions %d x %d x %d", d1, d2, d3);
    return nullptr;
  }
  return compress_host_path("szp_cuda_float_compress_topology_3d", oriData, outSize, absErrBound,
                            nbEle, blockSize, reinterpret_cast<const int *>(critical_points),
                            critical_count, 6, 3, d1, d2, d3);
}

void szp_cuda_float_decompress_randomaccess_topology_preserved(float **newData, size_t nbEle,
                                                               float absErrBound, int blockSize,
                                                               unsigned char *cmpBytes, int **FN) {
  clear_error();
  *newData = nullptr;
  *FN = nullptr;
  if (!cmpBytes || nbEle == 0) return;
  if (!check_block_size(blockSize, "szp_cuda_float_decompress_randomaccess_topology_preserved"))
    return;
  std::vector<unsigned long long> offs;
  unsigned long long hdr = 0, plen = 0;
  if (!walk_stream(cmpBytes, nbEle, blockSize, true, offs, hdr, plen)) {
    set_error("malformed topology stream");
    return;
  }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return;
  const size_t nb = offs.size();
  const size_t need = a256(plen + 16) + a256(nb * 8) + a256(nbEle * 4) * 2 + 4096;
  if (!ctx->scratch.reserve(need)) return;
  unsigned char *d_pay = ctx->scratch.take<unsigned char>(plen + 16);
  unsigned long long *d_off = ctx->scratch.take<unsigned long long>(nb);
  float *d_out = ctx->scratch.take<float>(nbEle);
  int *d_fn = ctx->scratch.take<int>(nbEle);
  cudaStream_t s = ctx->stream;
  float *h_out = (float *)malloc(nbEle * sizeof(float));
  int *h_fn = (int *)calloc(nbEle, sizeof(int));
  if (!h_out || !h_fn) { free(h_out); free(h_fn); set_error("host allocation failed"); return; }
  int *w_err = reinterpret_cast<int *>(ctx->d_words + 4);
  DecArgs a{};
  a.payload = d_pay;
  a.payload_len = plen;
  a.blk_off = d_off;
  a.n = nbEle;
  a.B = blockSize;
  a.eb = absErrBound;
  a.out_f = d_out;
  a.fn_i = d_fn;
  a.err = w_err;
  bool bad =
      cuda_fail(cudaMemsetAsync(ctx->d_words, 0, 8 * 8, s), "memset") ||
      cuda_fail(cudaMemcpyAsync(d_pay, cmpBytes + hdr, plen, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(cudaMemcpyAsync(d_off, offs.data(), nb * 8, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(launch_decode(true, a, s), "decode") || !(++ctx->launches) ||
      cuda_fail(cudaMemcpyAsync(ctx->h_words, ctx->d_words, 8 * 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaMemcpyAsync(h_out, d_out, nbEle * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaMemcpyAsync(h_fn, d_fn, nbEle * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "sync");
  if (!bad && (ctx->h_words[4] & 0xffffffffu)) {
    set_error("decoder reported malformed stream");
    bad = true;
  }
  if (bad) { free(h_out); free(h_fn); return; }
  *newData = h_out;
  *FN = h_fn;
}

int *szp_cuda_decompress_sort_positions(unsigned char *cmpBytes, size_t critical_count,
                                        int blockSize) {
  clear_error();
  if (!cmpBytes || critical_count == 0) return nullptr;
  if (!check_block_size(blockSize, "szp_cuda_decompress_sort_positions")) return nullptr;
  std::vector<unsigned long long> offs;
  unsigned long long hdr = 0, plen = 0;
  if (!walk_stream(cmpBytes, critical_count, blockSize, false, offs, hdr, plen)) {
    set_error("malformed sort-position stream");
    return nullptr;
  }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  const size_t nb = offs.size();
  const size_t need = a256(plen + 16) + a256(nb * 8) + a256(critical_count * 4) + 4096;
  if (!ctx->scratch.reserve(need)) return nullptr;
  unsigned char *d_pay = ctx->scratch.take<unsigned char>(plen + 16);
  unsigned long long *d_off = ctx->scratch.take<unsigned long long>(nb);
  int *d_out = ctx->scratch.take<int>(critical_count);
  cudaStream_t s = ctx->stream;
  int *h_out = (int *)malloc(critical_count * sizeof(int));
  if (!h_out) { set_error("host allocation failed"); return nullptr; }
  DecArgs a{};
  a.payload = d_pay;
  a.payload_len = plen;
  a.blk_off = d_off;
  a.n = critical_count;
  a.B = blockSize;
  a.out_i = d_out;
  a.err = reinterpret_cast<int *>(ctx->d_words + 4);
  bool bad =
      cuda_fail(cudaMemsetAsync(ctx->d_words, 0, 8 * 8, s), "memset") ||
      cuda_fail(cudaMemcpyAsync(d_pay, cmpBytes + hdr, plen, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(cudaMemcpyAsync(d_off, offs.data(), nb * 8, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(launch_decode(false, a, s), "decode") || !(++ctx->launches) ||
      cuda_fail(cudaMemcpyAsync(ctx->h_words, ctx->d_words, 8 * 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaMemcpyAsync(h_out, d_out, critical_count * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "sync");
  if (!bad && (ctx->h_words[4] & 0xffffffffu)) {
    set_error("decoder reported malformed stream");
    bad = true;
  }
  if (bad) { free(h_out); return nullptr; }
  return h_out;
}

size_t szp_b200_topo_bound(size_t n, int blockSize) {
  if (blockSize <= 0 || blockSize > kMaxBlockSize) return 0;
  return stream_bound(n, blockSize, true);
}

size_t szp_b200_sort_bound(size_t n, int blockSize) {
  if (blockSize <= 0 || blockSize > kMaxBlockSize) return 0;
  return stream_bound(n, blockSize, false);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// device-pointer entry points
// ---------------------------------------------------------------------------
namespace tsz {

static bool geom_ok(const szp_b200_geom &g, unsigned long long *n, Geom *out) {
  return geom_elements(g, n, out);
}

}  // namespace tsz

extern "C" {

}  // extern "C"

namespace tsz {

// Fused compression.  With h_topo set, the topology stream is copied to the
// host on the workspace's copy stream as soon as it is complete, overlapping
// the rank and sort-position stages (the caller waits for the copy stream).
static int compress_dev_impl(szp_b200_ctx *ctx, const float *d_data, szp_b200_geom geom, float absErrBound,
                             int blockSize, unsigned char *d_topo, unsigned char *d_sort, uint64_t *d_blk_index,
                             szp_b200_sizes *sizes, unsigned char *h_topo, size_t topo_cap,
                             const float *h_src = nullptr) {
  if (!ctx || !d_data || !d_topo || !d_sort || !sizes) { set_error("null argument"); return -1; }
  if (!(absErrBound > 0.0f)) { set_error("error bound must be positive"); return -1; }
  if (!check_block_size(blockSize, "szp_b200_topo_compress_dev")) return -1;
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const int B = blockSize;
  const unsigned long long nb = (n + B - 1) / B;
  const unsigned long long kcap = n;
  const size_t need = a256(kcap * 8) + a256(n * 4) + a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) * 2 +
                      rank_scratch_bytes(kcap, ctx->sm_count) + 8192;
  if (!ctx->scratch.reserve(need)) return -1;
  Arena &A = ctx->scratch;
  uint2 *pairs = A.take<uint2>(kcap);
  int *sp = A.take<int>(n);
  unsigned long long tot[3];
  tl_begin(ctx);
  // a field still on the host (h_src) is copied in parts that overlap the encoder
  const bool chunked = h_src && B <= 256 && n >= (1ull << 24);
  if (h_src && !chunked &&
      cuda_fail(cudaMemcpyAsync(const_cast<float *>(d_data), h_src, n * 4, cudaMemcpyHostToDevice, ctx->stream),
                "H2D field"))
    return -1;
  if (chunked ? encode_topo_chunked(ctx, h_src, const_cast<float *>(d_data), n, B, absErrBound, g, d_topo,
                                    stream_bound(n, B, true), reinterpret_cast<unsigned long long *>(d_blk_index),
                                    pairs, kcap, tot, h_topo, topo_cap)
              : encode_pass(ctx, kEncClassify, d_data, nullptr, nullptr, n, B, absErrBound, g, d_topo,
                            stream_bound(n, B, true), reinterpret_cast<unsigned long long *>(d_blk_index),
                            kCpPairs, pairs, kcap, tot))
    return -1;
  tl_mark(ctx, "encode_topo");
  sizes->topo_bytes = 8 + tot[0];
  sizes->cp_count = tot[1];
  sizes->extrema_count = tot[2];
  sizes->sort_bytes = 0;
  if (h_topo && !chunked) {
    // the encoder has finished (encode_pass waited for it): copy now
    if (sizes->topo_bytes > topo_cap) {
      set_error("topology output buffer too small (%zu bytes needed)", sizes->topo_bytes);
      return -1;
    }
    cudaStream_t cs = copy_stream(ctx);
    if (!cs || cuda_fail(cudaMemcpyAsync(h_topo, d_topo, sizes->topo_bytes, cudaMemcpyDeviceToHost, cs), "D2H"))
      return -1;
  }
  const unsigned long long K = tot[1], E = tot[2];
  if (E == 0) return 0;
  if (rank_positions(ctx, pairs, nullptr, K, E, absErrBound, sp)) return -1;
  tl_mark(ctx, "rank");
  unsigned long long st[3];
  if (encode_pass(ctx, kEncInts, nullptr, sp, nullptr, E, B, absErrBound, g, d_sort,
                  stream_bound(E, B, false),
                  d_blk_index ? reinterpret_cast<unsigned long long *>(d_blk_index) + nb : nullptr,
                  kCpNone, nullptr, 0, st))
    return -1;
  tl_mark(ctx, "encode_sort");
  sizes->sort_bytes = 8 + st[0];
  return 0;
}

}  // namespace tsz

extern "C" {

int szp_b200_topo_compress_dev(szp_b200_ctx *ctx, const float *d_data, szp_b200_geom geom,
                               float absErrBound, int blockSize, unsigned char *d_topo,
                               unsigned char *d_sort, uint64_t *d_blk_index,
                               szp_b200_sizes *sizes) {
  clear_error();
  DeviceGuard dg(ctx);
  return compress_dev_impl(ctx, d_data, geom, absErrBound, blockSize, d_topo, d_sort, d_blk_index, sizes, nullptr,
                           0);
}

}  // extern "C"

namespace tsz {

// Fused decompression (+ post-processing) of device-resident streams.  With
// d_blk_index == nullptr the block offsets of both streams are parsed on the
// device; ref_bound selects the reference's validation bound for that parse
// and *parse_failed reports a stream that is not a valid single-chunk stream.
int decompress_dev_impl(szp_b200_ctx *ctx, const unsigned char *d_topo, size_t topo_bytes,
                        const unsigned char *d_sort, size_t sort_bytes,
                        const uint64_t *d_blk_index, szp_b200_geom geom, float absErrBound,
                        int blockSize, float *d_out, unsigned char *d_types, int postprocess,
                        bool ref_bound, bool *parse_failed, cudaEvent_t sort_ready, bool cpu_layout,
                        unsigned long long sort_count) {
  if (parse_failed) *parse_failed = false;
  if (!ctx || !d_topo || !d_out) { set_error("null argument"); return -1; }
  if (!check_block_size(blockSize, "szp_b200_topo_decompress_dev")) return -1;
  if (topo_bytes < 8) { set_error("topology stream too short"); return -1; }
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const int B = blockSize;
  const unsigned long long nb = (n + B - 1) / B;
  const bool post = postprocess != 0;
  const bool parse = d_blk_index == nullptr;
  const bool have_sort = d_sort && sort_bytes > 8;
  size_t need = (post ? post_scratch_bytes(n) + a256(n * 4) : 0) + a256(n) + 8192;
  if (parse)
    need += a256(2 * nb * 8) + parse_scratch_bytes(topo_bytes - 8, B, true) +
            (post && have_sort ? parse_scratch_bytes(sort_bytes - 8, B, false) : 0);
  if (!ctx->scratch.reserve(need)) return -1;
  Arena &A = ctx->scratch;
  int *sp = post ? A.take<int>(n) : nullptr;
  unsigned char *T = d_types ? d_types : A.take<unsigned char>(n);
  unsigned long long *idx = parse ? A.take<unsigned long long>(2 * nb)
                                  : reinterpret_cast<unsigned long long *>(const_cast<uint64_t *>(d_blk_index));
  cudaStream_t s = ctx->stream;
  unsigned long long *w = ctx->d_words;  // [16..17] topology parse status, [18..19] sort parse status
  if (cuda_fail(cudaMemsetAsync(w, 0, 64, s), "memset")) return -1;
  tl_begin(ctx);
  if (parse) {
    if (parse_stream(ctx, A, d_topo + 8, topo_bytes - 8, n, nullptr, B, true, ref_bound, idx, w + 16))
      return -1;
    tl_mark(ctx, "parse_topo");
  }
  DecArgs a{};
  a.payload = d_topo + 8;
  a.payload_len = topo_bytes - 8;
  a.blk_off = idx;
  a.n = n;
  a.B = B;
  a.eb = absErrBound;
  a.out_f = d_out;
  a.fn_u8 = T;
  a.err = reinterpret_cast<int *>(w + 4);
  a.ext_count = w + 6;
  a.cpu_layout = cpu_layout ? 1 : 0;
  if (cpu_layout && B > 256) { set_error("the OpenMP stream layout is read for blockSize <= 256"); return -1; }
  if (cuda_fail(launch_decode(true, a, s), "decode")) return -1;
  ctx->launches += 1;
  tl_mark(ctx, "decode_topo");
  // the sort stream may still be on its way to the device (host-buffer path)
  if (sort_ready && post && have_sort && cuda_fail(cudaStreamWaitEvent(s, sort_ready, 0), "wait")) return -1;
  if (parse && post && have_sort) {
    // the sort stream holds one value per extremum: its element count is the
    // decoder's count of type-1/2 tags, read on the device
    if (parse_stream(ctx, A, d_sort + 8, sort_bytes - 8, 0, w + 6, B, false, ref_bound, idx + nb, w + 18))
      return -1;
    tl_mark(ctx, "parse_sort");
  }
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 20 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
                "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "decode"))
    return -1;
  if (parse && (ctx->h_words[16] == 0 || ctx->h_words[17] != 0)) {
    if (parse_failed) *parse_failed = true;
    set_error("topology stream is not a valid single-chunk stream (pass the block index from "
              "szp_b200_topo_compress_dev, or use the host-buffer entry point)");
    return -1;
  }
  if (ctx->h_words[4] & 0xffffffffu) { set_error("decoder reported malformed stream"); return -1; }
  if (!post) return 0;
  // sort positions: one per extremum tag, unless the caller knows the count
  const unsigned long long E = sort_count != ~0ull ? sort_count : ctx->h_words[6];
  const int *spp = nullptr;
  if (E > 0 && have_sort) {
    if (parse && (ctx->h_words[18] == 0 || ctx->h_words[19] != 0)) {
      if (parse_failed) *parse_failed = true;
      set_error("sort-position stream is not a valid single-chunk stream");
      return -1;
    }
    DecArgs b{};
    b.payload = d_sort + 8;
    b.payload_len = sort_bytes - 8;
    b.blk_off = idx + nb;
    b.n = E;
    b.B = B;
    b.out_i = sp;
    b.err = reinterpret_cast<int *>(w + 4);
    if (cuda_fail(launch_decode(false, b, s), "decode sort")) return -1;
    ctx->launches += 1;
    tl_mark(ctx, "decode_sort");
    spp = sp;
  }
  unsigned long long *S = post_words(ctx, n);
  const unsigned long long ntiles = (n + 2047) / 2048;
  TileDesc *desc = A.take<TileDesc>(ntiles + 1);
  if (!S || !desc) { set_error("scratch arena too small for post-processing"); return -1; }
  int restored = 0;
  // d_out holds the raw decoded field: the list build gathers the raw values
  // of the candidates from it before any pass updates it in place
  return postprocess_with(ctx, d_out, d_out, T, S, desc, spp, spp ? E : 0, g, absErrBound,
                          postprocess == 2, &restored);
}

}  // namespace tsz

extern "C" {

int szp_b200_topo_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_topo, size_t topo_bytes,
                                 const unsigned char *d_sort, size_t sort_bytes,
                                 const uint64_t *d_blk_index, szp_b200_geom geom, float absErrBound,
                                 int blockSize, float *d_out, unsigned char *d_types,
                                 int postprocess) {
  clear_error();
  DeviceGuard dg(ctx);
  return decompress_dev_impl(ctx, d_topo, topo_bytes, d_sort, sort_bytes, d_blk_index, geom, absErrBound,
                             blockSize, d_out, d_types, postprocess, false, nullptr);
}

int szp_b200_topo_postprocess_dev(szp_b200_ctx *ctx, float *d_data, const float *d_orig,
                                  const int *d_types, const int *d_sp, size_t n_sp,
                                  szp_b200_geom geom, float absErrBound, int axis_stencil) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_data || !d_orig || !d_types) { set_error("null argument"); return -1; }
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  if (!ctx->scratch.reserve(post_scratch_bytes(n) + 8192)) return -1;
  int restored = 0;
  return postprocess(ctx, d_data, d_orig, nullptr, d_types, d_sp, d_sp ? n_sp : 0, g, absErrBound,
                     axis_stencil, &restored);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sort-position stream of an arbitrary CP list (extrema in list order)
// ---------------------------------------------------------------------------
namespace tsz {

static unsigned char *compress_sp_host(const int *h_cps, int stride, size_t K, size_t *outSize,
                                       int B, const char *fn) {
  *outSize = 0;
  if (!check_block_size(B, fn)) return nullptr;
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  const size_t cap = stream_bound(K, B, false);
  const size_t need = a256(K * stride * 4) + a256(K * 4) + a256(cap) +
                      a256((K / 2048 + 2) * sizeof(TileDesc)) +
                      a256((K / B / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) + 8192;
  if (!ctx->scratch.reserve(need)) return nullptr;
  Arena &A = ctx->scratch;
  int *d_cps = A.take<int>(K * stride);
  int *d_sp = A.take<int>(K);
  unsigned char *d_stream = A.take<unsigned char>(cap);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_cps, h_cps, K * stride * 4, cudaMemcpyHostToDevice, s), "H2D"))
    return nullptr;
  unsigned long long E = 0;
  if (compact_extrema(ctx, d_cps, stride, K, d_sp, &E)) return nullptr;
  if (E == 0) return nullptr;
  unsigned long long tot[3];
  Geom g = make_geom(2, 1, 1, 1);
  if (encode_pass(ctx, kEncInts, nullptr, d_sp, nullptr, E, B, 1.0f, g, d_stream, cap, nullptr,
                  kCpNone, nullptr, 0, tot))
    return nullptr;
  const size_t total = 8 + tot[0];
  unsigned char *out = (unsigned char *)malloc(total);
  if (!out) { set_error("host allocation failed"); return nullptr; }
  if (cuda_fail(cudaMemcpyAsync(out, d_stream, total, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "sync")) {
    free(out);
    return nullptr;
  }
  *outSize = total;
  return out;
}

}  // namespace tsz

extern "C" {

unsigned char *szp_cuda_compress_sort_positions(CriticalPoint *critical_points,
                                                 size_t critical_count, size_t *outSize,
                                                 int blockSize) {
  clear_error();
  if (!critical_points || critical_count == 0) { *outSize = 0; return nullptr; }
  return compress_sp_host(reinterpret_cast<const int *>(critical_points), 5, critical_count,
                          outSize, blockSize, "szp_cuda_compress_sort_positions");
}

unsigned char *szp_cuda_compress_sort_positions_3d(CriticalPoint3D *critical_points,
                                                    size_t critical_count, size_t *outSize,
                                                    int blockSize) {
  clear_error();
  if (!critical_points || critical_count == 0) { *outSize = 0; return nullptr; }
  return compress_sp_host(reinterpret_cast<const int *>(critical_points), 6, critical_count,
                          outSize, blockSize, "szp_cuda_compress_sort_positions_3d");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// host-buffer fused entry points (device staging kept in the workspace)
// ---------------------------------------------------------------------------
extern "C" {

int szp_b200_topo_compress_host(szp_b200_ctx *ctx, const float *h_data, szp_b200_geom geom,
                                float absErrBound, int blockSize, unsigned char *h_topo,
                                size_t topo_cap, unsigned char *h_sort, size_t sort_cap,
                                szp_b200_sizes *sizes) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !h_data || !h_topo || !h_sort || !sizes) { set_error("null argument"); return -1; }
  if (!check_block_size(blockSize, "szp_b200_topo_compress_host")) return -1;
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const size_t tb = stream_bound(n, blockSize, true), sb = stream_bound(n, blockSize, false);
  if (!ctx->io.reserve(a256(n * 4) + a256(tb) + a256(sb) + 4096)) return -1;
  float *d_data = ctx->io.take<float>(n);
  unsigned char *d_topo = ctx->io.take<unsigned char>(tb);
  unsigned char *d_sort = ctx->io.take<unsigned char>(sb);
  cudaStream_t s = ctx->stream;
  // the field is copied in parts that overlap the encoder; the topology
  // stream goes to the host while the rank and sort stages run
  const int rc = compress_dev_impl(ctx, d_data, geom, absErrBound, blockSize, d_topo, d_sort, nullptr, sizes,
                                   h_topo, topo_cap, h_data);
  cudaStream_t cs = ctx->copy_stream, ds = ctx->d2h_stream;
  if (rc) {
    if (cs) cudaStreamSynchronize(cs);
    if (ds) cudaStreamSynchronize(ds);
    return -1;
  }
  if (sizes->sort_bytes > sort_cap) {
    if (cs) cudaStreamSynchronize(cs);
    if (ds) cudaStreamSynchronize(ds);
    set_error("sort-position output buffer too small (%zu bytes needed)", sizes->sort_bytes);
    return -1;
  }
  if ((sizes->sort_bytes &&
       cuda_fail(cudaMemcpyAsync(h_sort, d_sort, sizes->sort_bytes, cudaMemcpyDeviceToHost, s), "D2H")) ||
      cuda_fail(cudaStreamSynchronize(s), "sync") || (cs && cuda_fail(cudaStreamSynchronize(cs), "sync")) ||
      (ds && cuda_fail(cudaStreamSynchronize(ds), "sync")))
    return -1;
  return 0;
}

// Host-walk form: the reference's thread-count detection and serial block
// walk on the host (multi-chunk offset tables and the other cases the device
// parser leaves to it).
static int decompress_host_walk(szp_b200_ctx *ctx, const unsigned char *h_topo, size_t topo_bytes,
                                const unsigned char *h_sort, size_t sort_bytes, szp_b200_geom geom,
                                float absErrBound, int blockSize, float *h_out, int postprocess) {
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const int B = blockSize;
  const unsigned long long nb = (n + B - 1) / B;
  // block offsets of the topology stream from its bytes (the reference's walk)
  std::vector<unsigned long long> offs;
  unsigned long long hdr = 0, plen = 0;
  if (!walk_stream(h_topo, n, B, true, offs, hdr, plen, topo_bytes) || hdr + plen > topo_bytes) {
    set_error("malformed topology stream");
    return -1;
  }
  // the extrema count is the number of type-1/2 tags; it sizes the sort stream
  if (!ctx->io.reserve(a256(topo_bytes + 16) + a256(sort_bytes + 16) + a256(2 * nb * 8) + a256(n * 4) + 4096))
    return -1;
  unsigned char *d_topo = ctx->io.take<unsigned char>(topo_bytes + 16);
  unsigned char *d_sort = ctx->io.take<unsigned char>(sort_bytes + 16);
  unsigned long long *d_idx = ctx->io.take<unsigned long long>(2 * nb);
  float *d_out = ctx->io.take<float>(n);
  cudaStream_t s = ctx->stream;
  // a multi-chunk offset table is folded into the payload offsets
  std::vector<unsigned char> rebased;
  const unsigned char *src = h_topo;
  size_t src_bytes = topo_bytes;
  if (hdr != 8) {
    rebased.assign(8 + plen, 0);
    memcpy(rebased.data() + 8, h_topo + hdr, plen);
    src = rebased.data();
    src_bytes = 8 + plen;
  }
  if (cuda_fail(cudaMemcpyAsync(d_topo, src, src_bytes, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(cudaMemcpyAsync(d_idx, offs.data(), nb * 8, cudaMemcpyHostToDevice, s), "H2D"))
    return -1;
  size_t sbytes = 0;
  if (postprocess && h_sort && sort_bytes > 8) {
    // count extrema from the tags on the host-side copy: decode tags only
    // through the device decoder (raw pass) to learn E
    if (szp_b200_topo_decompress_dev(ctx, d_topo, src_bytes, nullptr, 0, reinterpret_cast<const uint64_t *>(d_idx), geom, absErrBound, B,
                                     d_out, nullptr, 0))
      return -1;
  }
  unsigned long long E = 0;
  if (postprocess && h_sort && sort_bytes > 8) {
    // ext count of the raw pass is in the status words
    E = ctx->h_words[6];
    std::vector<unsigned long long> soffs;
    unsigned long long shdr = 0, splen = 0;
    if (E > 0) {
      if (!walk_stream(h_sort, E, B, false, soffs, shdr, splen, sort_bytes) || shdr + splen > sort_bytes) {
        set_error("malformed sort-position stream");
        return -1;
      }
      std::vector<unsigned char> srb(8 + splen, 0);
      memcpy(srb.data() + 8, h_sort + shdr, splen);
      if (cuda_fail(cudaMemcpyAsync(d_sort, srb.data(), 8 + splen, cudaMemcpyHostToDevice, s), "H2D") ||
          cuda_fail(cudaMemcpyAsync(d_idx + nb, soffs.data(), soffs.size() * 8, cudaMemcpyHostToDevice, s),
                    "H2D") ||
          cuda_fail(cudaStreamSynchronize(s), "sync"))
        return -1;
      sbytes = 8 + splen;
    }
  }
  if (szp_b200_topo_decompress_dev(ctx, d_topo, src_bytes, sbytes ? d_sort : nullptr, sbytes, reinterpret_cast<const uint64_t *>(d_idx), geom,
                                   absErrBound, B, d_out, nullptr, postprocess))
    return -1;
  if (cuda_fail(cudaMemcpyAsync(h_out, d_out, n * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "sync"))
    return -1;
  return 0;
}

int szp_b200_topo_decompress_host(szp_b200_ctx *ctx, const unsigned char *h_topo, size_t topo_bytes,
                                  const unsigned char *h_sort, size_t sort_bytes, szp_b200_geom geom,
                                  float absErrBound, int blockSize, float *h_out, int postprocess) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !h_topo || !h_out) { set_error("null argument"); return -1; }
  if (!check_block_size(blockSize, "szp_b200_topo_decompress_host")) return -1;
  unsigned long long n;
  Geom g;
  if (!geom_ok(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  // A single-chunk stream (offset table [0]) is parsed on the device; anything
  // the device parser rejects goes through the reference's host detection.
  if (topo_bytes > 8 && rd64(h_topo) == 0) {
    const size_t sbytes = (h_sort && sort_bytes > 8) ? sort_bytes : 0;
    if (!ctx->io.reserve(a256(topo_bytes) + a256(sbytes + 16) + a256(n * 4) + 4096)) return -1;
    unsigned char *d_topo = ctx->io.take<unsigned char>(topo_bytes);
    unsigned char *d_sort = ctx->io.take<unsigned char>(sbytes + 16);
    float *d_out = ctx->io.take<float>(n);
    cudaStream_t s = ctx->stream;
    // the sort stream travels on the copy stream while the topology stream is
    // parsed and decoded
    cudaStream_t cs = sbytes ? copy_stream(ctx) : nullptr;
    if (sbytes && !cs) return -1;
    if (cuda_fail(cudaMemcpyAsync(d_topo, h_topo, topo_bytes, cudaMemcpyHostToDevice, s), "H2D") ||
        (sbytes && (cuda_fail(cudaMemcpyAsync(d_sort, h_sort, sbytes, cudaMemcpyHostToDevice, cs), "H2D") ||
                    cuda_fail(cudaEventRecord(ctx->copy_ev, cs), "event"))))
      return -1;
    bool parse_failed = false;
    const int rc = decompress_dev_impl(ctx, d_topo, topo_bytes, sbytes ? d_sort : nullptr, sbytes, nullptr, geom,
                                       absErrBound, blockSize, d_out, nullptr, postprocess, true, &parse_failed,
                                       sbytes ? ctx->copy_ev : nullptr);
    if (cs) cudaStreamSynchronize(cs);
    if (rc == 0) {
      if (cuda_fail(cudaMemcpyAsync(h_out, d_out, n * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
          cuda_fail(cudaStreamSynchronize(s), "sync"))
        return -1;
      return 0;
    }
    if (!parse_failed) return -1;
    clear_error();
  }
  return decompress_host_walk(ctx, h_topo, topo_bytes, h_sort, sort_bytes, geom, absErrBound, blockSize,
                              h_out, postprocess);
}

}  // extern "C"
