// The .SZp container of the reference's CPU drivers and the OpenMP stream
// layouts inside it, written and read on the device.
//
// Container (example/testfloat_compress_fastmode1_topology.cc:105-125, read
// back at example/testfloat_decompress_fastmode1_topology.cc:720-805):
//   [topology stream][sort-position stream][u64 topology size][u64 sort size]
// OpenMP layouts (SZp/src/szp_float.cc:1170-1302, :522-865;
// SZp/src/szp_topology_3d.cc:253-416):
//   topology:       [u64 offset x T][blocks]        T = writer's thread count
//   sort positions: [u64 E][u64 offset x T][blocks] E = extrema
// Thread t writes blocks [t*ceil(nb/T), (t+1)*ceil(nb/T)) contiguously and
// its table entry is where they start (relative to the end of the table), so
// the block payload is the single-chunk payload; the one difference in the
// blocks is that the OpenMP writer gives a one-element block its (zero)
// bit-count byte (SZp/src/szp_float.cc:1239-1242), which the CUDA layout omits.
//
// Reading follows the reference's thread-count detection
// (SZp/include/szp_detect_threads.h:153-190 for the sort positions, :282-309
// for the topology): the first candidate T whose table is non-decreasing and
// bounded and whose every chunk walks inside the validation bound.  Each
// candidate's chunks are walked by the device parser, one chunk at a time,
// not by a serial walk on the host.
#include <algorithm>
#include <vector>

#include "tsz_ops.h"

namespace tsz {

constexpr int kMaxTableThreads = 128;

// table entry t: where chunk t's blocks start (the payload length when the
// chunk is empty), as a little-endian u64 at any byte alignment
// (every: blockSize 1, where every earlier block gained its bit-count byte)
__global__ void chunk_table_kernel(const unsigned long long *__restrict__ offs, unsigned long long nb, int T,
                                   unsigned long long payload_len, bool every, unsigned char *__restrict__ dst) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const unsigned long long bpt = (nb + T - 1) / T;
  const unsigned long long b = (unsigned long long)t * bpt;
  const unsigned long long v = b < nb ? offs[b] + (every ? b : 0ull) : payload_len;
#pragma unroll
  for (int k = 0; k < 8; k++) dst[8 * t + k] = (unsigned char)(v >> (8 * k));
}

__global__ void put_u64_kernel(unsigned char *__restrict__ dst, unsigned long long v) {
  if (threadIdx.x < 8) dst[threadIdx.x] = (unsigned char)(v >> (8 * threadIdx.x));
}

__global__ void add_base_kernel(const unsigned long long *__restrict__ in, unsigned long long n,
                                unsigned long long base, unsigned long long *__restrict__ out) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] + base;
}

// One-element blocks in the OpenMP layout: [anchor][bit count 0][tags].
// Block b (CUDA offset offs[b]) lands at offs[b] + (one-element blocks
// before it): b itself for blockSize 1, 0 for the last block otherwise.
__global__ void one_blocks_kernel(const unsigned char *__restrict__ src, const unsigned long long *__restrict__ offs,
                                  unsigned long long b0, unsigned long long b1, bool every, bool tags,
                                  unsigned char *__restrict__ dst) {
  const unsigned long long b = b0 + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= b1) return;
  const unsigned long long o = offs[b];
  const unsigned long long d = o + (every ? b : 0ull);
  for (int k = 0; k < 4; k++) dst[d + k] = src[o + k];
  dst[d + 4] = 0;
  if (tags) dst[d + 5] = src[o + 4];
}

// Copies a CUDA-layout payload into the OpenMP layout (see one_blocks_kernel).
static int cpu_payload(cudaStream_t s, const unsigned char *src, unsigned long long len,
                       const unsigned long long *offs, unsigned long long n, int B, bool tags, unsigned char *dst) {
  const unsigned long long nb = (n + B - 1) / B;
  if (nb == 0) return 0;
  if (B == 1) {
    one_blocks_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(src, offs, 0, nb, true, tags, dst);
    return cuda_fail(cudaGetLastError(), "layout kernel") ? -1 : 0;
  }
  if (n % B != 1) return cuda_fail(cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToDevice, s), "copy") ? -1 : 0;
  // every block but the last as it is, then the one-element last block
  unsigned long long last = 0;
  if (cuda_fail(cudaMemcpyAsync(&last, offs + nb - 1, 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "layout"))
    return -1;
  if (last && cuda_fail(cudaMemcpyAsync(dst, src, last, cudaMemcpyDeviceToDevice, s), "copy")) return -1;
  one_blocks_kernel<<<1, 32, 0, s>>>(src, offs, nb - 1, nb, false, tags, dst);
  return cuda_fail(cudaGetLastError(), "layout kernel") ? -1 : 0;
}

static unsigned long long ones_of(unsigned long long n, int B) {
  if (n == 0) return 0;
  return B == 1 ? n : (n % B == 1 ? 1ull : 0ull);
}

// Parses the block offsets of one chunk of a stream on the device: blocks
// [b0, b0 + nbc) starting at payload offset off (relative to pay), within
// lim bytes of pay.  Offsets go to d_offs[b0 ..] (relative to pay).
static int parse_chunk(szp_b200_ctx *ctx, Arena &A, const unsigned char *pay, unsigned long long lim,
                       unsigned long long off, unsigned long long b0, unsigned long long nbc, unsigned long long n,
                       int B, bool tags, unsigned long long *d_offs, unsigned long long *d_status, bool *ok) {
  *ok = false;
  if (nbc == 0) { *ok = true; return 0; }
  if (off >= lim) return 0;
  const unsigned long long e0 = b0 * (unsigned long long)B;
  const unsigned long long ne = std::min<unsigned long long>(n, (b0 + nbc) * (unsigned long long)B) - e0;
  const size_t mark = A.used;
  unsigned long long *tmp = A.take<unsigned long long>(nbc);
  if (!tmp) { set_error("scratch arena too small for the chunk parser"); return -1; }
  // the reference's walk reads a bit count only for blocks of more than one
  // element (SZp/include/szp_detect_threads.h:64-101, 238-275); with
  // blockSize 1, where every block has one element and carries the byte, the
  // walk follows the blocks as written
  if (parse_stream(ctx, A, pay + off, lim - off, ne, nullptr, B, tags, false, tmp, d_status, B == 1)) return -1;
  unsigned long long st[2] = {0, 0};
  if (cuda_fail(cudaMemcpyAsync(st, d_status, 16, cudaMemcpyDeviceToHost, ctx->stream), "D2H") ||
      cuda_fail(cudaStreamSynchronize(ctx->stream), "chunk parse"))
    return -1;
  if (st[0] != 0 && st[1] == 0) {
    *ok = true;
    add_base_kernel<<<(unsigned)((nbc + 255) / 256), 256, 0, ctx->stream>>>(tmp, nbc, off, d_offs + b0);
    if (cuda_fail(cudaGetLastError(), "offsets")) return -1;
    ctx->launches += 1;
  }
  A.used = mark;
  return 0;
}

// Thread count and block offsets of an OpenMP-layout stream by the
// reference's detection rule.  cmp: the stream (its offset table first),
// len: its bytes, n: elements; first_try: 1 for the topology stream, 2 for
// the sort positions (whose detection assumes one thread unless a larger
// count validates).  Writes the payload-relative offsets of every block to
// d_offs and returns T (0 when no candidate, not even one thread, walks).
static int detect_chunks(szp_b200_ctx *ctx, Arena &A, const unsigned char *cmp, unsigned long long len,
                         unsigned long long n, int B, bool tags, int first_try, unsigned long long *d_offs,
                         unsigned long long *d_status) {
  cudaStream_t s = ctx->stream;
  const unsigned long long nb = (n + B - 1) / B;
  const unsigned long long maxc = tags ? 8ull * n + 1024ull : 4ull * n + 4ull;
  const unsigned long long bound = std::min(maxc, len);
  const int tmax = (int)std::min<unsigned long long>(kMaxTableThreads, len / 8);
  if (tmax < 1) return 0;
  std::vector<unsigned long long> tab(tmax);
  if (cuda_fail(cudaMemcpyAsync(tab.data(), cmp, (size_t)tmax * 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "table"))
    return -1;
  auto try_T = [&](int T, unsigned long long bound, bool *ok) -> int {
    *ok = false;
    const unsigned long long hdr = (unsigned long long)T * 8;
    if (hdr >= bound) return 0;
    const unsigned long long bpt = (nb + T - 1) / T;
    for (int t = 0; t < T; t++) {
      const unsigned long long b0 = (unsigned long long)t * bpt;
      if (b0 >= nb) break;
      const unsigned long long nbc = std::min(bpt, nb - b0);
      bool cok = false;
      if (parse_chunk(ctx, A, cmp + hdr, bound - hdr, tab[t], b0, nbc, n, B, tags, d_offs, d_status, &cok)) return -1;
      if (!cok) return 0;
    }
    *ok = true;
    return 0;
  };
  if (tab[0] == 0) {
    for (int T = first_try; T <= tmax; T++) {
      bool valid = true;
      for (int k = 1; k < T; k++)
        if (tab[k] > maxc || tab[k] < tab[k - 1]) { valid = false; break; }
      if (!valid) break;
      bool ok = false;
      if (try_T(T, bound, &ok)) return -1;
      if (ok) return T;
    }
  }
  // No candidate validated: the reference then takes one thread without a
  // walk (so a single chunk longer than its validation bound is read as
  // well); here that chunk is walked inside the stream's own length.
  bool ok = false;
  if (try_T(1, len, &ok)) return -1;
  return ok ? 1 : 0;
}

}  // namespace tsz

using namespace tsz;

extern "C" {

size_t szp_b200_container_bound(size_t n, int blockSize, int threads) {
  if (blockSize <= 0 || threads <= 0) return 0;
  return szp_b200_topo_bound(n, blockSize) + szp_b200_sort_bound(n, blockSize) + (size_t)threads * 16 +
         2 * ((n + blockSize - 1) / blockSize) + 64;
}

int szp_b200_container_from_streams_dev(szp_b200_ctx *ctx, const unsigned char *d_topo, size_t topo_bytes,
                                        const unsigned char *d_sort, size_t sort_bytes, szp_b200_geom geom,
                                        int blockSize, size_t extrema, int threads, unsigned char *d_out,
                                        size_t out_cap, size_t *out_bytes) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_topo || !d_out || !out_bytes) { set_error("null argument"); return -1; }
  *out_bytes = 0;
  if (threads < 1 || threads > kMaxTableThreads) { set_error("threads must lie in [1, 128]"); return -1; }
  if (blockSize <= 0 || blockSize > 256) { set_error("blockSize must lie in [1, 256]"); return -1; }
  if (topo_bytes < 8 || (extrema && (!d_sort || sort_bytes < 8))) { set_error("stream too short"); return -1; }
  unsigned long long n;
  Geom g;
  if (!geom_elements(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const int B = blockSize, T = threads;
  const unsigned long long E = extrema;
  const unsigned long long nb = (n + B - 1) / B, nbs = (E + B - 1) / B;
  const unsigned long long tp = topo_bytes - 8, sp = E ? sort_bytes - 8 : 0;
  const unsigned long long tp_cpu = tp + ones_of(n, B), sp_cpu = E ? sp + ones_of(E, B) : 0;
  const unsigned long long topo_size = 8ull * T + tp_cpu;
  const unsigned long long sort_size = E ? 8ull + 8ull * T + sp_cpu : 0;
  const unsigned long long total = topo_size + sort_size + 16;
  if (total > out_cap) { set_error("container buffer too small (%llu bytes needed)", total); return -1; }
  const size_t need = a256(nb * 8) + a256(nbs * 8) + parse_scratch_bytes(tp, B, true) +
                      (E ? parse_scratch_bytes(sp, B, false) : 0) + 8192;
  if (!ctx->scratch.reserve(need)) return -1;
  Arena &A = ctx->scratch;
  unsigned long long *offs = A.take<unsigned long long>(nb), *offs_s = A.take<unsigned long long>(nbs ? nbs : 1);
  cudaStream_t s = ctx->stream;
  unsigned long long *w = ctx->d_words;
  if (parse_stream(ctx, A, d_topo + 8, tp, n, nullptr, B, true, false, offs, w + 16)) return -1;
  if (E && parse_stream(ctx, A, d_sort + 8, sp, E, nullptr, B, false, false, offs_s, w + 18)) return -1;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words + 16, w + 16, 32, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "parse"))
    return -1;
  if (ctx->h_words[16] == 0 || ctx->h_words[17] != 0 || (E && (ctx->h_words[18] == 0 || ctx->h_words[19] != 0))) {
    set_error("the streams are not valid single-chunk streams");
    return -1;
  }
  // topology: table, payload
  chunk_table_kernel<<<1, 128, 0, s>>>(offs, nb, T, tp_cpu, B == 1, d_out);
  if (cpu_payload(s, d_topo + 8, tp, offs, n, B, true, d_out + 8ull * T)) return -1;
  // sort positions: extrema count, table, payload
  unsigned char *so = d_out + topo_size;
  if (E) {
    put_u64_kernel<<<1, 32, 0, s>>>(so, E);
    chunk_table_kernel<<<1, 128, 0, s>>>(offs_s, nbs, T, sp_cpu, B == 1, so + 8);
    if (cpu_payload(s, d_sort + 8, sp, offs_s, E, B, false, so + 8 + 8ull * T)) return -1;
  }
  put_u64_kernel<<<1, 32, 0, s>>>(d_out + topo_size + sort_size, topo_size);
  put_u64_kernel<<<1, 32, 0, s>>>(d_out + topo_size + sort_size + 8, sort_size);
  ctx->launches += 3 + (E ? 2 : 0);
  if (cuda_fail(cudaGetLastError(), "container kernels") || cuda_fail(cudaStreamSynchronize(s), "container"))
    return -1;
  *out_bytes = total;
  return 0;
}

int szp_b200_container_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_in, size_t in_bytes,
                                      szp_b200_geom geom, float absErrBound, int blockSize, float *d_out,
                                      unsigned char *d_types, int postprocess) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_in || !d_out) { set_error("null argument"); return -1; }
  if (blockSize <= 0 || blockSize > 256) { set_error("blockSize must lie in [1, 256]"); return -1; }
  unsigned long long n;
  Geom g;
  if (!geom_elements(geom, &n, &g)) { set_error("invalid geometry"); return -1; }
  const int B = blockSize;
  const unsigned long long nb = (n + B - 1) / B;
  cudaStream_t s = ctx->stream;
  // footer, validated as the reference's reader does; otherwise the whole
  // buffer is a topology stream
  unsigned long long topo_size = in_bytes, sort_size = 0;
  if (in_bytes >= 16) {
    unsigned long long ft[2];
    if (cuda_fail(cudaMemcpyAsync(ft, d_in + in_bytes - 16, 16, cudaMemcpyDeviceToHost, s), "D2H") ||
        cuda_fail(cudaStreamSynchronize(s), "footer"))
      return -1;
    if (ft[0] > 0 && ft[0] + ft[1] + 16 <= in_bytes + 16 && ft[0] < in_bytes && ft[0] + ft[1] <= in_bytes) {
      topo_size = ft[0];
      sort_size = ft[1];
    }
  }
  unsigned long long E = 0;
  const unsigned char *sort_cmp = nullptr;
  unsigned long long sort_len = 0;
  if (sort_size >= 16) {
    if (cuda_fail(cudaMemcpyAsync(&E, d_in + topo_size, 8, cudaMemcpyDeviceToHost, s), "D2H") ||
        cuda_fail(cudaStreamSynchronize(s), "sort header"))
      return -1;
    sort_cmp = d_in + topo_size + 8;
    sort_len = sort_size - 8;
    if (E > n) { set_error("sort-position stream counts %llu extrema for %llu elements", E, n); return -1; }
  }
  const unsigned long long nbs = (E + B - 1) / B;
  const size_t need = a256((nb + nbs + 1) * 8) + parse_scratch_bytes(topo_size, B, true) +
                      (E ? parse_scratch_bytes(sort_len, B, false) : 0) + a256(nb * 8) + 16384;
  // the decompression reserves its own scratch: keep the index in the io arena
  if (!ctx->io.reserve(a256((nb + nbs + 1) * 8) + 256)) return -1;
  unsigned long long *idx = ctx->io.take<unsigned long long>(nb + nbs + 1);
  if (!ctx->scratch.reserve(need)) return -1;
  unsigned long long *w = ctx->d_words;
  const int Tt = detect_chunks(ctx, ctx->scratch, d_in, topo_size, n, B, true, 1, idx, w + 16);
  if (Tt < 0) return -1;
  if (Tt == 0) { set_error("topology stream: no thread count walks inside the stream"); return -1; }
  int Ts = 0;
  if (E) {
    ctx->scratch.reset();
    Ts = detect_chunks(ctx, ctx->scratch, sort_cmp, sort_len, E, B, false, 2, idx + nb, w + 18);
    if (Ts < 0) return -1;
    if (Ts == 0) { set_error("sort-position stream: no thread count walks inside the stream"); return -1; }
  }
  // decompress with the index; the streams are passed 8 bytes before their
  // payloads (after the tables)
  const unsigned char *tptr = d_in + 8ull * Tt - 8;
  const unsigned long long tbytes = topo_size - 8ull * Tt + 8;
  const unsigned char *sptr = E ? sort_cmp + 8ull * Ts - 8 : nullptr;
  const unsigned long long sbytes = E ? sort_len - 8ull * Ts + 8 : 0;
  return decompress_dev_impl(ctx, tptr, tbytes, sptr, sbytes, reinterpret_cast<const uint64_t *>(idx), geom,
                             absErrBound, B, d_out, d_types, postprocess, false, nullptr, nullptr, true, E);
}

}  // extern "C"
