// Plain (non-topology) SZp codec: random-access and threadblock modes, float
// and double, compress and decompress, behind the reference's entry points
// (SZp/include/szp_cuda_compress.cuh:22-64, szp_cuda_decompress.cuh:23-57;
// SZp/src/szp_cuda_compress.cu:122-802, szp_cuda_decompress.cu:176-665,
// 810-1070).
//
// Stream of the compressors: [T eb][u64 0][body], one chunk.
//   random access: blocks of B elements, each [i32 anchor q0][bit count, when
//     the block has more than one element][sign bits][magnitudes]
//   threadblock:   [i32 q0], then blocks of B deltas over elements 1 .. n-1,
//     each [bit count][sign bits][magnitudes]; deltas chain across blocks
// q = (int)(x * (1/eb)) in double; bit count floor(log2f(max |delta|)) + 1;
// magnitudes: bc / 8 full bytes per delta (little-endian, upper bits), then
// the bc % 8 lower bits of every delta, MSB-first and contiguous.  The
// decompressors receive the stream after its T header and detect the
// offset-table thread count as the reference does (streams of the reference's
// OpenMP compressors carry T chunks).
//
// Work on the device: one warp per compression block (B <= 1025, so up to
// 1025 deltas, the threadblock mode's B: 33 per lane).  Compression is two passes over the input -- a
// size pass (quantize, deltas, max), a device-wide scan of the 64-bit block
// sizes, a packing pass that stages the magnitudes and sign ballots of its
// block in shared memory and writes every byte of the block once, lane-
// strided (signs from the ballot words, full bytes per delta, remainder bytes
// gathered from the staged magnitudes).  Decompression decodes a block per
// warp, deltas lane-parallel and a warp prefix sum for the values; the
// threadblock mode adds a per-block delta-sum pass and a scan for the carry
// of each block inside its chunk.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "tsz_ops.h"
#include "tsz_scan.cuh"

namespace tsz {

constexpr int kPlainThreads = 256;
constexpr int kPlainWarps = kPlainThreads / 32;
constexpr int kPlainMaxBlock = 1025;     // reference limit SZP_CUDA_MAX_BLOCK + 1
// deltas of one block: B - 1 in the random-access mode, B in the threadblock
// mode (its blocks carry no anchor)
constexpr int kPlainMaxDeltas = kPlainMaxBlock;
constexpr int kPlainChunks = (kPlainMaxDeltas + 31) / 32;

template <class T>
__device__ __forceinline__ int plain_quant(T x, double inv) { return (int)__dmul_rn((double)x, inv); }

__device__ __forceinline__ float plain_deq(int q, float eb) { return __fmul_rn(__int2float_rn(q), eb); }
__device__ __forceinline__ double plain_deq(int q, double eb) { return __dmul_rn((double)q, eb); }

// One compression block of the compressor's grid: deltas over the element
// pairs (e0 + d, e0 + d + 1), d < cnt; `anchor`: the block starts with q of e0.
struct PlainBlock {
  unsigned long long e0;
  unsigned cnt;
  bool anchor;
};

__device__ __forceinline__ PlainBlock plain_block(unsigned long long b, unsigned long long n, int B, int tb) {
  PlainBlock k;
  k.e0 = b * (unsigned long long)B;
  if (!tb) {
    const unsigned long long m = n - k.e0 < (unsigned long long)B ? n - k.e0 : (unsigned long long)B;
    k.cnt = (unsigned)(m - 1);
    k.anchor = true;
  } else {
    const unsigned long long m = n - 1 - k.e0 < (unsigned long long)B ? n - 1 - k.e0 : (unsigned long long)B;
    k.cnt = (unsigned)m;
    k.anchor = false;
  }
  return k;
}

__host__ __device__ __forceinline__ unsigned long long plain_mag_bytes(unsigned cnt, unsigned bc) {
  const unsigned fb = bc >> 3, rem = bc & 7;
  return (unsigned long long)fb * cnt + (rem ? ((unsigned long long)rem * cnt + 7) / 8 : 0);
}

// bytes of one block of `cnt` deltas with bit count bc
__host__ __device__ __forceinline__ unsigned long long plain_block_bytes(bool anchor, unsigned cnt, unsigned bc) {
  unsigned long long s = anchor ? 4 : 0;
  if (anchor && cnt == 0) return s;
  s += 1;
  if (bc) s += (cnt + 7) / 8 + plain_mag_bytes(cnt, bc);
  return s;
}

// Deltas of chunk k (d = 32k + lane) of a block: q of the pair's second
// element, its delta's magnitude and sign.  qc: q of element e0 + 32k (the
// carry from the previous chunk, or the block's first element).
template <class T>
__device__ __forceinline__ void plain_chunk(const T *__restrict__ x, const PlainBlock &k, int c, double inv, int &qc,
                                            unsigned &mag, bool &neg, bool &in) {
  const int lane = threadIdx.x & 31;
  const unsigned d = 32u * c + lane;
  in = d < k.cnt;
  const int q = in ? plain_quant(__ldg(x + k.e0 + d + 1), inv) : 0;
  int qp = __shfl_up_sync(0xffffffffu, q, 1);
  if (lane == 0) qp = qc;
  const unsigned ud = (unsigned)q - (unsigned)qp;
  neg = in && (int)ud < 0;
  mag = in ? (neg ? 0u - ud : ud) : 0u;
  qc = __shfl_sync(0xffffffffu, q, 31);
}

template <class T>
__global__ void __launch_bounds__(kPlainThreads) plain_size_kernel(const T *__restrict__ x, unsigned long long n,
                                                                   int B, int tb, double inv,
                                                                   unsigned long long nblocks,
                                                                   unsigned long long *__restrict__ sizes) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long b = (unsigned long long)blockIdx.x * kPlainWarps + warp; b < nblocks;
       b += (unsigned long long)gridDim.x * kPlainWarps) {
    const PlainBlock k = plain_block(b, n, B, tb);
    int qc = plain_quant(__ldg(x + k.e0), inv);
    unsigned maxm = 0;
    for (int c = 0; 32u * c < k.cnt; c++) {
      unsigned mag;
      bool neg, in;
      plain_chunk(x, k, c, inv, qc, mag, neg, in);
      maxm = mag > maxm ? mag : maxm;
    }
    maxm = __reduce_max_sync(0xffffffffu, maxm);
    if (lane == 0) sizes[b] = plain_block_bytes(k.anchor, k.cnt, bitcount(maxm));
  }
}

// body: where the blocks go (after the threadblock mode's leading q0).
template <class T>
__global__ void __launch_bounds__(kPlainThreads) plain_pack_kernel(const T *__restrict__ x, unsigned long long n,
                                                                   int B, int tb, double inv,
                                                                   unsigned long long nblocks,
                                                                   const unsigned long long *__restrict__ offs,
                                                                   unsigned char *__restrict__ body) {
  __shared__ unsigned s_mag[kPlainWarps][kPlainMaxDeltas];
  __shared__ unsigned s_sgn[kPlainWarps][kPlainChunks];
  // every index below stays inside the warp's rows: d < cnt <= kPlainMaxDeltas,
  // chunk c < ceil(cnt / 32) <= kPlainChunks, sign byte t < ceil(cnt / 8) so t / 4 < kPlainChunks
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned *mg = s_mag[warp];
  unsigned *sg = s_sgn[warp];
  for (unsigned long long b = (unsigned long long)blockIdx.x * kPlainWarps + warp; b < nblocks;
       b += (unsigned long long)gridDim.x * kPlainWarps) {
    const PlainBlock k = plain_block(b, n, B, tb);
    const int q0 = plain_quant(__ldg(x + k.e0), inv);
    int qc = q0;
    unsigned maxm = 0;
    for (int c = 0; 32u * c < k.cnt; c++) {
      unsigned mag;
      bool neg, in;
      plain_chunk(x, k, c, inv, qc, mag, neg, in);
      if (in) mg[32 * c + lane] = mag;
      const unsigned w = __ballot_sync(0xffffffffu, neg);
      if (lane == 0) sg[c] = w;
      maxm = mag > maxm ? mag : maxm;
    }
    maxm = __reduce_max_sync(0xffffffffu, maxm);
    const unsigned bc = bitcount(maxm);
    __syncwarp();
    unsigned char *p = body + offs[b];
    if (k.anchor) {
      if (lane < 4) p[lane] = (unsigned char)((unsigned)q0 >> (8 * lane));
      p += 4;
      if (k.cnt == 0) { __syncwarp(); continue; }
    } else if (b == 0 && lane < 4) {
      body[lane - 4 + 0] = (unsigned char)((unsigned)q0 >> (8 * lane));   // q0 before the first block
    }
    if (lane == 0) p[0] = (unsigned char)bc;
    p += 1;
    if (bc) {
      const unsigned cnt = k.cnt;
      const unsigned sb = (cnt + 7) / 8;
      for (unsigned t = lane; t < sb; t += 32)
        p[t] = (unsigned char)(__brev((sg[t >> 2] >> (8 * (t & 3))) & 0xffu) >> 24);
      p += sb;
      const unsigned fb = bc >> 3, rem = bc & 7;
      if (fb) {
        for (unsigned i = lane; i < cnt * fb; i += 32) {
          const unsigned d = i / fb, j = i - d * fb;
          p[i] = (unsigned char)((mg[d] >> rem) >> (8 * j));
        }
        p += (unsigned long long)fb * cnt;
      }
      if (rem) {
        const unsigned bits = rem * cnt, rb = (bits + 7) / 8, mask = (1u << rem) - 1u;
        for (unsigned t = lane; t < rb; t += 32) {
          unsigned byte = 0;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const unsigned pos = 8 * t + i;
            if (pos < bits) {
              const unsigned d = pos / rem, bi = pos - d * rem;
              byte |= (((mg[d] & mask) >> (rem - 1 - bi)) & 1u) << (7 - i);
            }
          }
          p[t] = (unsigned char)byte;
        }
      }
    }
    __syncwarp();
  }
}

// q0 of a threadblock stream with no deltas (n == 1)
template <class T>
__global__ void plain_q0_kernel(const T *__restrict__ x, double inv, unsigned char *__restrict__ at) {
  if (threadIdx.x < 4) at[threadIdx.x] = (unsigned char)((unsigned)plain_quant(x[0], inv) >> (8 * threadIdx.x));
}

// ---------------------------------------------------------------------------
// decompression
// ---------------------------------------------------------------------------

// A block of a stream being decoded: payload offset, the element its first
// delta (or anchor) lands on, its delta count, and (threadblock mode) its
// chunk.
struct PlainDesc {
  unsigned long long off;
  unsigned long long start;
  unsigned cnt;
  unsigned chunk;
};

// Chunk of a threadblock stream: its anchor, the element the anchor lands on,
// and the index of its first block.
struct PlainChunk {
  unsigned long long lo;
  unsigned first_block;
  int anchor;
};

__device__ __forceinline__ unsigned plain_extract(const unsigned char *__restrict__ mg, unsigned d, unsigned cnt,
                                                  unsigned bc) {
  const unsigned fb = bc >> 3, rem = bc & 7;
  unsigned v = 0;
  if (rem) {
    const unsigned char *r = mg + (unsigned long long)fb * cnt;
    const unsigned start = d * rem, byte0 = start >> 3, off = start & 7;
    if (off + rem <= 8) {
      v = ((unsigned)r[byte0] >> (8 - off - rem)) & ((1u << rem) - 1u);
    } else {
      const unsigned w = ((unsigned)r[byte0] << 8) | r[byte0 + 1];
      v = (w >> (16 - off - rem)) & ((1u << rem) - 1u);
    }
  }
  if (fb) {
    const unsigned char *f = mg + (unsigned long long)d * fb;
    unsigned full = 0;
    for (unsigned t = 0; t < fb; t++) full |= (unsigned)f[t] << (8 * t);
    v |= full << rem;
  }
  return v;
}

// signed delta d of a block with bit count bc (as an unsigned, wrapping)
__device__ __forceinline__ unsigned plain_delta(const unsigned char *__restrict__ sg, unsigned d, unsigned cnt,
                                                unsigned bc) {
  const unsigned char *mg = sg + (cnt + 7) / 8;
  const unsigned mag = plain_extract(mg, d, cnt, bc);
  const bool neg = (sg[d >> 3] >> (7 - (d & 7))) & 1u;
  return neg ? 0u - mag : mag;
}

__device__ __forceinline__ unsigned warp_incl_add(unsigned v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

__device__ __forceinline__ int plain_rd32(const unsigned char *p) {
  return (int)((unsigned)p[0] | ((unsigned)p[1] << 8) | ((unsigned)p[2] << 16) | ((unsigned)p[3] << 24));
}

// random access: block = [anchor][bc][signs][magnitudes]; cnt deltas after the anchor
// Blocks from descriptors, or (desc null) the compressors' single-chunk grid
// with payload offsets offs[b].
template <class T>
__global__ void __launch_bounds__(kPlainThreads) plain_decode_ra_kernel(const unsigned char *__restrict__ pay,
                                                                        const PlainDesc *__restrict__ desc,
                                                                        const unsigned long long *__restrict__ offs,
                                                                        unsigned long long n, int B,
                                                                        unsigned long long nblocks, T eb,
                                                                        T *__restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long b = (unsigned long long)blockIdx.x * kPlainWarps + warp; b < nblocks;
       b += (unsigned long long)gridDim.x * kPlainWarps) {
    PlainDesc k;
    if (desc) {
      k = desc[b];
    } else {
      k.off = offs[b];
      k.start = b * (unsigned long long)B;
      k.cnt = (unsigned)((n - k.start < (unsigned long long)B ? n - k.start : (unsigned long long)B) - 1);
      k.chunk = 0;
    }
    const unsigned char *p = pay + k.off;
    const int a = plain_rd32(p);
    if (lane == 0) out[k.start] = plain_deq(a, eb);
    if (k.cnt == 0) continue;
    const unsigned bc = p[4];
    const unsigned char *sg = p + 5;
    unsigned carry = (unsigned)a;
    for (unsigned c = 0; 32u * c < k.cnt; c++) {
      const unsigned d = 32u * c + lane;
      const unsigned dl = (d < k.cnt && bc) ? plain_delta(sg, d, k.cnt, bc) : 0u;
      const unsigned v = carry + warp_incl_add(dl);
      if (d < k.cnt) out[k.start + 1 + d] = plain_deq((int)v, eb);
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// threadblock, pass 1: the delta sum (mod 2^32) of every block
__global__ void __launch_bounds__(kPlainThreads) plain_tb_sums_kernel(const unsigned char *__restrict__ pay,
                                                                      const PlainDesc *__restrict__ desc,
                                                                      unsigned long long nblocks,
                                                                      unsigned *__restrict__ sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long b = (unsigned long long)blockIdx.x * kPlainWarps + warp; b < nblocks;
       b += (unsigned long long)gridDim.x * kPlainWarps) {
    const PlainDesc k = desc[b];
    const unsigned char *p = pay + k.off;
    const unsigned bc = p[0];
    unsigned s = 0;
    if (bc)
      for (unsigned d = lane; d < k.cnt; d += 32) s += plain_delta(p + 1, d, k.cnt, bc);
    s = __reduce_add_sync(0xffffffffu, s);
    if (lane == 0) sums[b] = s;
  }
}

// threadblock, pass 2: values from the chunk anchor + the exclusive sum of
// the chunk's earlier blocks (pre: exclusive scan of the sums over all blocks)
template <class T>
__global__ void __launch_bounds__(kPlainThreads) plain_tb_decode_kernel(const unsigned char *__restrict__ pay,
                                                                        const PlainDesc *__restrict__ desc,
                                                                        unsigned long long nblocks,
                                                                        const PlainChunk *__restrict__ chunks,
                                                                        const unsigned *__restrict__ pre, T eb,
                                                                        T *__restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long b = (unsigned long long)blockIdx.x * kPlainWarps + warp; b < nblocks;
       b += (unsigned long long)gridDim.x * kPlainWarps) {
    const PlainDesc k = desc[b];
    const PlainChunk ch = chunks[k.chunk];
    const unsigned char *p = pay + k.off;
    const unsigned bc = p[0];
    unsigned carry = (unsigned)ch.anchor + (pre[b] - pre[ch.first_block]);
    for (unsigned c = 0; 32u * c < k.cnt; c++) {
      const unsigned d = 32u * c + lane;
      const unsigned dl = (d < k.cnt && bc) ? plain_delta(p + 1, d, k.cnt, bc) : 0u;
      const unsigned v = carry + warp_incl_add(dl);
      if (d < k.cnt) out[k.start + d] = plain_deq((int)v, eb);
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

template <class T>
__global__ void plain_tb_anchor_kernel(const PlainChunk *__restrict__ chunks, unsigned nchunks, T eb,
                                       T *__restrict__ out) {
  const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nchunks && chunks[c].lo != ~0ull) out[chunks[c].lo] = plain_deq(chunks[c].anchor, eb);
}

// direct / threadblock predict quantization: q[0], q[i] - q[i-1]
__global__ void plain_predict_kernel(const float *__restrict__ x, unsigned long long n, double inv,
                                     int *__restrict__ out) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const int q = plain_quant(x[i], inv);
    out[i] = i ? (int)((unsigned)q - (unsigned)plain_quant(x[i - 1], inv)) : q;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static inline unsigned long long prd64(const unsigned char *p) {
  unsigned long long v;
  memcpy(&v, p, 8);
  return v;
}

static unsigned long long plain_nblocks(unsigned long long n, int B, int tb) {
  if (!tb) return (n + B - 1) / B;
  return n > 1 ? (n - 1 + B - 1) / B : 0;
}

static size_t plain_body_bound(unsigned long long n, int B, int tb) {
  return (tb ? 4 : 0) + plain_nblocks(n, B, tb) * (size_t)plain_block_bytes(!tb, (unsigned)B, 32) + 64;
}

// Walk of one block from pos; lim bounds the reads (~0: unbounded, as the
// reference's interface carries no stream length).
static bool plain_span(const unsigned char *s, unsigned long long pos, unsigned long long lim, bool anchor,
                       unsigned cnt, unsigned long long *next) {
  const bool chk = lim != ~0ull;
  unsigned long long p = pos;
  if (anchor) {
    if (chk && p + 4 > lim) return false;
    p += 4;
    if (cnt == 0) { *next = p; return true; }
  }
  if (chk && p >= lim) return false;
  const unsigned bc = s[p++];
  if (bc > 32) return false;
  if (bc) p += (cnt + 7) / 8 + plain_mag_bytes(cnt, bc);
  if (chk && p > lim) return false;
  *next = p;
  return true;
}

struct PlainLayout {
  std::vector<PlainDesc> desc;
  std::vector<PlainChunk> chunks;
  unsigned long long hdr = 0, end = 0;
};

// Walks the chunks of a T-chunk table; fills the layout when it is not null.
static bool plain_walk(const unsigned char *s, unsigned long long n, int B, int tb, unsigned T,
                       unsigned long long lim, PlainLayout *L) {
  const unsigned long long hdr = 8ull * T, tbs = n / T;
  unsigned long long end = hdr;
  if (L) { L->desc.clear(); L->chunks.clear(); }
  for (unsigned c = 0; c < T; c++) {
    const unsigned long long lo = c * tbs, hi = (c == T - 1) ? n : (c + 1) * tbs;
    unsigned long long pos = hdr + prd64(s + 8 * c);
    if (lim != ~0ull && pos >= lim) return false;
    if (!tb) {
      for (unsigned long long i = lo; i < hi; i += B) {
        const unsigned m = (unsigned)std::min<unsigned long long>(B, hi - i);
        if (L) L->desc.push_back(PlainDesc{pos - hdr, i, m - 1, c});
        if (!plain_span(s, pos, lim, true, m - 1, &pos)) return false;
      }
    } else {
      PlainChunk ch{~0ull, (unsigned)(L ? L->desc.size() : 0), 0};
      if (lo < hi) {
        if (lim != ~0ull && pos + 4 > lim) return false;
        int a;
        memcpy(&a, s + pos, 4);
        ch.lo = lo;
        ch.anchor = a;
        pos += 4;
        for (unsigned long long i = lo + 1; i < hi; i += B) {
          const unsigned cnt = (unsigned)std::min<unsigned long long>(B, hi - i);
          if (L) L->desc.push_back(PlainDesc{pos - hdr, i, cnt, c});
          if (!plain_span(s, pos, lim, false, cnt, &pos)) return false;
        }
      }
      if (L) L->chunks.push_back(ch);
    }
    end = std::max(end, pos);
  }
  if (L) { L->hdr = hdr; L->end = end; }
  return true;
}

// Offset-table thread count as the reference detects it: random access
// (SZp/src/szp_cuda_decompress.cu:233-276) the first t in 1..128 whose
// offsets are non-decreasing and at most 4n + 4 and whose chunks all walk
// inside 4n + 4 bytes, else 1; threadblock (:486-518) the largest t <= 256
// whose first t offsets are non-decreasing and at most 4n + 4, stopping at the
// first t that is not (1 when the first offset is not 0).  Deviation: a
// detected threadblock table whose chunks do not walk inside 4n + 4 bytes
// (the reference then decodes past its buffer) is read as one chunk.
static unsigned plain_detect(const unsigned char *s, unsigned long long n, int B, int tb) {
  const unsigned long long maxc = 4ull * n + 4;
  unsigned T = 0;
  if (prd64(s) == 0) {
    for (unsigned t = 1; t <= (tb ? 256u : 128u); t++) {
      bool ok = true;
      for (unsigned k = 1; k < t; k++) {
        const unsigned long long a = prd64(s + 8 * k), b = prd64(s + 8 * (k - 1));
        if (a > maxc || a < b) { ok = false; break; }
      }
      if (!ok) break;
      if (!tb) {
        if (plain_walk(s, n, B, 0, t, maxc, nullptr)) { T = t; break; }
      } else if (8ull * t + 5 <= maxc) {
        T = t;
      }
    }
  }
  if (T == 0) T = 1;
  if (tb && T > 1 && !plain_walk(s, n, B, 1, T, maxc, nullptr)) T = 1;
  return T;
}


static unsigned plain_grid(szp_b200_ctx *ctx, unsigned long long nb) {
  const unsigned long long g = (nb + kPlainWarps - 1) / kPlainWarps;
  return (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>(g, (unsigned long long)ctx->sm_count * 16));
}

static size_t plain_stream_bound(unsigned long long n, int B, int tb, size_t tsize) {
  return tsize + 8 + plain_body_bound(n, B, tb);
}

static size_t plain_compress_scratch(unsigned long long n, int B, int tb) {
  const unsigned long long nb = plain_nblocks(n, B, tb);
  const size_t two_pass = a256((nb + 1) * 8) + a256(scan_parts(nb + 1) * 8);
  const size_t fused = B <= kMaxBlockSize ? a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) : 0;
  return std::max(two_pass, fused) + 1024;
}

// Random-access float streams with blockSize <= 257 go through the fused
// single-pass encoder (quantize-without-tags mode) and the octet decoder; the
// block layout is the one the sort-position stream uses.
template <class T>
static bool plain_fused(int B, int tb) {
  return std::is_same<T, float>::value && !tb && B <= kMaxBlockSize;
}

// The whole stream [T eb][u64 0][body] of d_data into d_out (device), on
// ctx->stream; waits for the body size.  Scratch: plain_compress_scratch.
template <class T>
static int plain_compress_impl(szp_b200_ctx *ctx, const T *d_data, unsigned long long n, T eb, int B, int tb,
                               unsigned char *d_out, unsigned long long out_cap, unsigned long long *out_len) {
  cudaStream_t s = ctx->stream;
  const unsigned long long nb = plain_nblocks(n, B, tb);
  const double inv = 1.0 / (double)eb;
  const unsigned long long hdr = sizeof(T) + 8, lead = tb ? 4 : 0;
  if (plain_fused<T>(B, tb)) {
    // [T eb] from the host, then the encoder's [u64 0][blocks] right behind it
    memcpy(ctx->h_words + 16, &eb, sizeof(T));
    if (out_cap < hdr ||
        cuda_fail(cudaMemcpyAsync(d_out, ctx->h_words + 16, sizeof(T), cudaMemcpyHostToDevice, s), "H2D header"))
      return out_cap < hdr ? (set_error("plain output buffer too small"), -1) : -1;
    unsigned long long tot[3];
    const Geom g = make_geom(2, 1, (long long)n, 1);
    if (encode_pass(ctx, kEncQuant, reinterpret_cast<const float *>(d_data), nullptr, nullptr, n, B, (float)eb, g,
                    d_out + sizeof(T), out_cap - sizeof(T), nullptr, kCpNone, nullptr, 0, tot))
      return -1;
    *out_len = hdr + tot[0];
    return 0;
  }
  unsigned long long *sizes = ctx->scratch.take<unsigned long long>(nb + 1);
  unsigned long long *part = ctx->scratch.take<unsigned long long>(scan_parts(nb + 1));
  if (!sizes || !part) { set_error("scratch arena too small"); return -1; }
  // one extra zero item: its exclusive prefix is the body size
  if (cuda_fail(cudaMemsetAsync(sizes + nb, 0, 8, s), "memset")) return -1;
  if (nb) {
    plain_size_kernel<T><<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(d_data, n, B, tb, inv, nb, sizes);
    if (cuda_fail(cudaGetLastError(), "plain size launch")) return -1;
    ctx->launches += 1;
  }
  if (cuda_fail(device_scan<unsigned long long, OpAdd>(sizes, sizes, nb + 1, part, false, s), "scan")) return -1;
  ctx->launches += 3;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, sizes + nb, 8, cudaMemcpyDeviceToHost, s), "D2H size") ||
      cuda_fail(cudaStreamSynchronize(s), "plain size"))
    return -1;
  const unsigned long long len = hdr + lead + ctx->h_words[0];
  if (len > out_cap) { set_error("plain stream needs %llu bytes, output holds %llu", len, out_cap); return -1; }
  memcpy(ctx->h_words, &eb, sizeof(T));
  memset(reinterpret_cast<unsigned char *>(ctx->h_words) + sizeof(T), 0, 8);
  if (cuda_fail(cudaMemcpyAsync(d_out, ctx->h_words, hdr, cudaMemcpyHostToDevice, s), "H2D header")) return -1;
  if (nb) {
    plain_pack_kernel<T><<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(d_data, n, B, tb, inv, nb, sizes,
                                                                       d_out + hdr + lead);
    if (cuda_fail(cudaGetLastError(), "plain pack launch")) return -1;
    ctx->launches += 1;
  } else if (tb) {
    plain_q0_kernel<T><<<1, 32, 0, s>>>(d_data, inv, d_out + hdr);
    if (cuda_fail(cudaGetLastError(), "plain q0 launch")) return -1;
    ctx->launches += 1;
  }
  // the header copy read h_words: finish before it is reused
  if (cuda_fail(cudaStreamSynchronize(s), "plain pack")) return -1;
  *out_len = len;
  return 0;
}

// Random-access decode of a single-chunk payload whose block offsets are on
// the device: the octet decoder for float streams (blockSize <= 256, or 257
// on a 4-byte aligned payload), the warp-per-block decoder otherwise.
template <class T>
static int plain_decode_offsets(szp_b200_ctx *ctx, const unsigned char *pay, unsigned long long pay_len,
                                const unsigned long long *offs, unsigned long long n, int B, T eb, T *d_out) {
  cudaStream_t s = ctx->stream;
  const unsigned long long nb = (n + B - 1) / B;
  if (plain_fused<T>(B, 0) && (B <= 256 || (reinterpret_cast<uintptr_t>(pay) & 3u) == 0)) {
    DecArgs a{};
    a.payload = pay;
    a.payload_len = pay_len;
    a.blk_off = offs;
    a.n = n;
    a.B = B;
    a.eb = (float)eb;
    a.out_f = reinterpret_cast<float *>(d_out);
    a.err = reinterpret_cast<int *>(ctx->d_words + 4);
    if (cuda_fail(cudaMemsetAsync(ctx->d_words + 4, 0, 8, s), "memset") ||
        cuda_fail(launch_decode(false, a, s), "plain decode launch"))
      return -1;
    ctx->launches += 1;
    if (cuda_fail(cudaMemcpyAsync(ctx->h_words + 4, ctx->d_words + 4, 8, cudaMemcpyDeviceToHost, s), "D2H status") ||
        cuda_fail(cudaStreamSynchronize(s), "plain decode"))
      return -1;
    if (ctx->h_words[4] & 0xffffffffu) { set_error("malformed plain stream (status %llu)", ctx->h_words[4]); return -1; }
    return 0;
  }
  plain_decode_ra_kernel<T><<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(pay, nullptr, offs, n, B, nb, eb, d_out);
  if (cuda_fail(cudaGetLastError(), "plain decode launch")) return -1;
  ctx->launches += 1;
  return cuda_fail(cudaStreamSynchronize(s), "plain decode") ? -1 : 0;
}

// Random-access decode of a single-chunk stream on the device (block offsets
// parsed on the device).  d_in: the stream after its T header.
template <class T>
static int plain_decompress_dev_impl(szp_b200_ctx *ctx, const unsigned char *d_in, unsigned long long in_len,
                                     unsigned long long n, T eb, int B, T *d_out) {
  cudaStream_t s = ctx->stream;
  const unsigned long long nb = (n + B - 1) / B;
  if (in_len < 8) { set_error("plain stream shorter than its offset table"); return -1; }
  const unsigned long long buf = in_len - 8;
  if (!ctx->scratch.reserve(a256(nb * 8) + a256(16) + parse_scratch_bytes(buf, B, false) + 4096)) return -1;
  unsigned long long *offs = ctx->scratch.take<unsigned long long>(nb);
  unsigned long long *st = ctx->scratch.take<unsigned long long>(2);
  if (!offs || !st) { set_error("scratch arena too small"); return -1; }
  if (cuda_fail(cudaMemsetAsync(st, 0, 16, s), "memset")) return -1;
  if (parse_stream(ctx, ctx->scratch, d_in + 8, buf, n, nullptr, B, false, false, offs, st)) return -1;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, st, 16, cudaMemcpyDeviceToHost, s), "D2H status") ||
      cuda_fail(cudaStreamSynchronize(s), "plain parse"))
    return -1;
  if (ctx->h_words[0] == 0 || ctx->h_words[1]) { set_error("malformed plain stream"); return -1; }
  return plain_decode_offsets<T>(ctx, d_in + 8, buf, offs, n, B, eb, d_out);
}

static bool plain_block_ok(int B, const char *fn) {
  if (B >= 1 && B <= kPlainMaxBlock) return true;
  set_error("%s: blockSize %d out of range [1, %d]", fn, B, kPlainMaxBlock);
  return false;
}

// reference API: host field in, malloc'd (or caller's) stream out
template <class T>
static unsigned char *plain_compress_host(const char *fn, const T *h, size_t *outSize, T eb, size_t n, int B, int tb,
                                          unsigned char *arg_out) {
  clear_error();
  if (outSize) *outSize = 0;
  if (!outSize || !h || n == 0 || eb <= 0) return nullptr;
  if (!plain_block_ok(B, fn)) return nullptr;
  if (n >= kMaxElements) { set_error("%s: too many elements", fn); return nullptr; }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  const size_t cap = plain_stream_bound(n, B, tb, sizeof(T));
  if (!ctx->scratch.reserve(a256(n * sizeof(T)) + a256(cap) + plain_compress_scratch(n, B, tb))) return nullptr;
  T *d_data = ctx->scratch.take<T>(n);
  unsigned char *d_stream = ctx->scratch.take<unsigned char>(cap);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_data, h, n * sizeof(T), cudaMemcpyHostToDevice, s), "H2D field")) return nullptr;
  unsigned long long len = 0;
  if (plain_compress_impl<T>(ctx, d_data, n, eb, B, tb, d_stream, cap, &len)) return nullptr;
  unsigned char *out = arg_out ? arg_out : (unsigned char *)malloc(len);
  if (!out) { set_error("%s: host allocation failed", fn); return nullptr; }
  if (cuda_fail(cudaMemcpyAsync(out, d_stream, len, cudaMemcpyDeviceToHost, s), "D2H stream") ||
      cuda_fail(cudaStreamSynchronize(s), "sync")) {
    if (!arg_out) free(out);
    return nullptr;
  }
  *outSize = len;
  return out;
}

// reference API: stream after its T header in, values out (host)
template <class T>
static void plain_decompress_host(const char *fn, T *h_out, size_t n, T eb, int B, const unsigned char *cmp, int tb) {
  clear_error();
  if (!cmp || n == 0 || !h_out) return;
  if (!plain_block_ok(B, fn)) return;
  if (n >= kMaxElements) { set_error("%s: too many elements", fn); return; }
  const unsigned Tn = plain_detect(cmp, n, B, tb);
  PlainLayout L;
  if (!plain_walk(cmp, n, B, tb, Tn, ~0ull, &L)) { set_error("%s: malformed stream", fn); return; }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return;
  const unsigned long long nb = L.desc.size(), nc = L.chunks.size();
  const size_t need = a256(L.end + 16) + a256(nb * sizeof(PlainDesc) + 16) + a256(nc * sizeof(PlainChunk) + 16) +
                      2 * a256((nb + 1) * 4) + a256(scan_parts(nb + 1) * 4) + a256(n * sizeof(T)) + 4096;
  if (!ctx->scratch.reserve(need)) return;
  unsigned char *d_s = ctx->scratch.take<unsigned char>(L.end + 16);
  PlainDesc *d_desc = ctx->scratch.take<PlainDesc>(nb + 1);
  PlainChunk *d_ch = ctx->scratch.take<PlainChunk>(nc + 1);
  unsigned *d_sums = ctx->scratch.take<unsigned>(nb + 1);
  unsigned *d_part = ctx->scratch.take<unsigned>(scan_parts(nb + 1));
  T *d_out = ctx->scratch.take<T>(n);
  cudaStream_t s = ctx->stream;
  const bool one_chunk_ra = !tb && Tn == 1;
  if (cuda_fail(cudaMemcpyAsync(d_s, cmp, L.end, cudaMemcpyHostToDevice, s), "H2D stream") ||
      (nb && !one_chunk_ra &&
       cuda_fail(cudaMemcpyAsync(d_desc, L.desc.data(), nb * sizeof(PlainDesc), cudaMemcpyHostToDevice, s),
                 "H2D blocks")) ||
      (nc && cuda_fail(cudaMemcpyAsync(d_ch, L.chunks.data(), nc * sizeof(PlainChunk), cudaMemcpyHostToDevice, s),
                       "H2D chunks")))
    return;
  const unsigned char *pay = d_s + L.hdr;
  if (one_chunk_ra) {
    // one chunk: the compressors' regular block grid, payload offsets only
    unsigned long long *d_off = reinterpret_cast<unsigned long long *>(d_desc);
    std::vector<unsigned long long> offs(nb);
    for (unsigned long long b = 0; b < nb; b++) offs[b] = L.desc[b].off;
    if ((nb && cuda_fail(cudaMemcpyAsync(d_off, offs.data(), nb * 8, cudaMemcpyHostToDevice, s), "H2D offsets")) ||
        plain_decode_offsets<T>(ctx, pay, L.end - L.hdr, d_off, n, B, eb, d_out))
      return;
  } else if (!tb) {
    plain_decode_ra_kernel<T><<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(pay, d_desc, nullptr, n, B, nb, eb, d_out);
    if (cuda_fail(cudaGetLastError(), "plain decode launch")) return;
    ctx->launches += 1;
  } else {
    if (nc) {
      plain_tb_anchor_kernel<T><<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(d_ch, (unsigned)nc, eb, d_out);
      ctx->launches += 1;
    }
    if (nb) {
      plain_tb_sums_kernel<<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(pay, d_desc, nb, d_sums);
      if (cuda_fail(cudaGetLastError(), "plain sums launch") ||
          cuda_fail(device_scan_u32<OpAdd>(d_sums, d_sums, nb, d_part, false, s), "scan"))
        return;
      plain_tb_decode_kernel<T><<<plain_grid(ctx, nb), kPlainThreads, 0, s>>>(pay, d_desc, nb, d_ch, d_sums, eb, d_out);
      ctx->launches += 5;
    }
    if (cuda_fail(cudaGetLastError(), "plain decode launch")) return;
  }
  if (cuda_fail(cudaMemcpyAsync(h_out, d_out, n * sizeof(T), cudaMemcpyDeviceToHost, s), "D2H values")) return;
  cuda_fail(cudaStreamSynchronize(s), "plain decode");
}

static int *plain_predict_host(const float *h, float eb, size_t n) {
  clear_error();
  if (!h || n == 0) return nullptr;
  if (n >= kMaxElements) { set_error("too many elements"); return nullptr; }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  if (!ctx->scratch.reserve(a256(n * 4) * 2 + 1024)) return nullptr;
  float *d_x = ctx->scratch.take<float>(n);
  int *d_q = ctx->scratch.take<int>(n);
  cudaStream_t s = ctx->stream;
  int *out = (int *)malloc(n * sizeof(int));
  if (!out) { set_error("host allocation failed"); return nullptr; }
  const double inv = 1.0 / (double)eb;
  if (cuda_fail(cudaMemcpyAsync(d_x, h, n * 4, cudaMemcpyHostToDevice, s), "H2D field")) { free(out); return nullptr; }
  const unsigned grid = (unsigned)std::min<unsigned long long>((n + 255) / 256, (unsigned long long)ctx->sm_count * 16);
  plain_predict_kernel<<<grid, 256, 0, s>>>(d_x, n, inv, d_q);
  ctx->launches += 1;
  if (cuda_fail(cudaGetLastError(), "predict launch") ||
      cuda_fail(cudaMemcpyAsync(out, d_q, n * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "predict")) {
    free(out);
    return nullptr;
  }
  return out;
}

}  // namespace tsz

using namespace tsz;

extern "C" {

// ---- reference entry points (SZp/include/szp_cuda_compress.cuh:22-64) ----
unsigned char *szp_cuda_float_compress_randomaccess(float *oriData, size_t *outSize, float absErrBound, size_t nbEle,
                                                    int blockSize) {
  return plain_compress_host<float>("szp_cuda_float_compress_randomaccess", oriData, outSize, absErrBound, nbEle,
                                    blockSize, 0, nullptr);
}
void szp_cuda_float_compress_randomaccess_arg(unsigned char *output, float *oriData, size_t *outSize,
                                              float absErrBound, size_t nbEle, int blockSize) {
  if (!output) { if (outSize) *outSize = 0; return; }
  plain_compress_host<float>("szp_cuda_float_compress_randomaccess_arg", oriData, outSize, absErrBound, nbEle,
                             blockSize, 0, output);
}
unsigned char *szp_cuda_double_compress_randomaccess(double *oriData, size_t *outSize, double absErrBound,
                                                     size_t nbEle, int blockSize) {
  return plain_compress_host<double>("szp_cuda_double_compress_randomaccess", oriData, outSize, absErrBound, nbEle,
                                     blockSize, 0, nullptr);
}
void szp_cuda_double_compress_randomaccess_arg(unsigned char *output, double *oriData, size_t *outSize,
                                               double absErrBound, size_t nbEle, int blockSize) {
  if (!output) { if (outSize) *outSize = 0; return; }
  plain_compress_host<double>("szp_cuda_double_compress_randomaccess_arg", oriData, outSize, absErrBound, nbEle,
                              blockSize, 0, output);
}
unsigned char *szp_cuda_float_compress_threadblock(float *oriData, size_t *outSize, float absErrBound, size_t nbEle,
                                                   int blockSize) {
  return plain_compress_host<float>("szp_cuda_float_compress_threadblock", oriData, outSize, absErrBound, nbEle,
                                    blockSize, 1, nullptr);
}
void szp_cuda_float_compress_threadblock_arg(unsigned char *output, float *oriData, size_t *outSize,
                                             float absErrBound, size_t nbEle, int blockSize) {
  if (!output) { if (outSize) *outSize = 0; return; }
  plain_compress_host<float>("szp_cuda_float_compress_threadblock_arg", oriData, outSize, absErrBound, nbEle,
                             blockSize, 1, output);
}
unsigned char *szp_cuda_double_compress_threadblock(double *oriData, size_t *outSize, double absErrBound,
                                                    size_t nbEle, int blockSize) {
  return plain_compress_host<double>("szp_cuda_double_compress_threadblock", oriData, outSize, absErrBound, nbEle,
                                     blockSize, 1, nullptr);
}
void szp_cuda_double_compress_threadblock_arg(unsigned char *output, double *oriData, size_t *outSize,
                                              double absErrBound, size_t nbEle, int blockSize) {
  if (!output) { if (outSize) *outSize = 0; return; }
  plain_compress_host<double>("szp_cuda_double_compress_threadblock_arg", oriData, outSize, absErrBound, nbEle,
                              blockSize, 1, output);
}
int *szp_cuda_float_direct_predict_quantization(float *oriData, size_t *outSize, float absErrBound, size_t nbEle,
                                                int blockSize) {
  (void)outSize;
  (void)blockSize;
  return plain_predict_host(oriData, absErrBound, nbEle);
}
int *szp_cuda_float_threadblock_predict_quantization(float *oriData, size_t *outSize, float absErrBound,
                                                     size_t nbEle, int blockSize) {
  (void)outSize;
  (void)blockSize;
  return plain_predict_host(oriData, absErrBound, nbEle);
}

// ---- reference entry points (SZp/include/szp_cuda_decompress.cuh:23-57) ----
float *szp_cuda_float_decompress_randomaccess(size_t nbEle, float absErrBound, int blockSize, unsigned char *cmpBytes) {
  float *out = (float *)calloc(nbEle ? nbEle : 1, sizeof(float));
  if (out) plain_decompress_host<float>("szp_cuda_float_decompress_randomaccess", out, nbEle, absErrBound, blockSize,
                                        cmpBytes, 0);
  return out;
}
void szp_cuda_float_decompress_randomaccess_arg(float *newData, size_t nbEle, float absErrBound, int blockSize,
                                                unsigned char *cmpBytes) {
  plain_decompress_host<float>("szp_cuda_float_decompress_randomaccess_arg", newData, nbEle, absErrBound, blockSize,
                               cmpBytes, 0);
}
double *szp_cuda_double_decompress_randomaccess(size_t nbEle, double absErrBound, int blockSize,
                                                unsigned char *cmpBytes) {
  double *out = (double *)calloc(nbEle ? nbEle : 1, sizeof(double));
  if (out) plain_decompress_host<double>("szp_cuda_double_decompress_randomaccess", out, nbEle, absErrBound,
                                         blockSize, cmpBytes, 0);
  return out;
}
void szp_cuda_double_decompress_randomaccess_arg(double *newData, size_t nbEle, double absErrBound, int blockSize,
                                                 unsigned char *cmpBytes) {
  plain_decompress_host<double>("szp_cuda_double_decompress_randomaccess_arg", newData, nbEle, absErrBound,
                                blockSize, cmpBytes, 0);
}
float *szp_cuda_float_decompress_threadblock(size_t nbEle, float absErrBound, int blockSize, unsigned char *cmpBytes) {
  float *out = (float *)calloc(nbEle ? nbEle : 1, sizeof(float));
  if (out) plain_decompress_host<float>("szp_cuda_float_decompress_threadblock", out, nbEle, absErrBound, blockSize,
                                        cmpBytes, 1);
  return out;
}
void szp_cuda_float_decompress_threadblock_arg(float *newData, size_t nbEle, float absErrBound, int blockSize,
                                               unsigned char *cmpBytes) {
  plain_decompress_host<float>("szp_cuda_float_decompress_threadblock_arg", newData, nbEle, absErrBound, blockSize,
                               cmpBytes, 1);
}
double *szp_cuda_double_decompress_threadblock(size_t nbEle, double absErrBound, int blockSize,
                                               unsigned char *cmpBytes) {
  double *out = (double *)calloc(nbEle ? nbEle : 1, sizeof(double));
  if (out) plain_decompress_host<double>("szp_cuda_double_decompress_threadblock", out, nbEle, absErrBound,
                                         blockSize, cmpBytes, 1);
  return out;
}
void szp_cuda_double_decompress_threadblock_arg(double *newData, size_t nbEle, double absErrBound, int blockSize,
                                                unsigned char *cmpBytes) {
  plain_decompress_host<double>("szp_cuda_double_decompress_threadblock_arg", newData, nbEle, absErrBound,
                                blockSize, cmpBytes, 1);
}

// ---- device-pointer additions ----
SZP_B200_API size_t szp_b200_plain_bound(size_t n, int blockSize, int is_double, int threadblock) {
  if (n == 0 || blockSize < 1 || blockSize > kPlainMaxBlock) return 0;
  return plain_stream_bound(n, blockSize, threadblock ? 1 : 0, is_double ? 8 : 4);
}

SZP_B200_API int szp_b200_plain_compress_dev(szp_b200_ctx *ctx, const void *d_data, int is_double, size_t n,
                                             double absErrBound, int blockSize, int threadblock,
                                             unsigned char *d_out, size_t out_cap, size_t *out_len) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_data || !d_out || !out_len) { set_error("szp_b200_plain_compress_dev: null argument"); return -1; }
  *out_len = 0;
  if (n == 0 || n >= kMaxElements) { set_error("szp_b200_plain_compress_dev: element count out of range"); return -1; }
  if (!(absErrBound > 0)) { set_error("szp_b200_plain_compress_dev: error bound must be > 0"); return -1; }
  if (!plain_block_ok(blockSize, "szp_b200_plain_compress_dev")) return -1;
  const int tb = threadblock ? 1 : 0;
  if (!ctx->scratch.reserve(plain_compress_scratch(n, blockSize, tb))) return -1;
  unsigned long long len = 0;
  const int rc = is_double
      ? plain_compress_impl<double>(ctx, static_cast<const double *>(d_data), n, absErrBound, blockSize, tb, d_out,
                                    out_cap, &len)
      : plain_compress_impl<float>(ctx, static_cast<const float *>(d_data), n, (float)absErrBound, blockSize, tb,
                                   d_out, out_cap, &len);
  if (rc) return -1;
  *out_len = len;
  return 0;
}

SZP_B200_API int szp_b200_plain_decompress_dev(szp_b200_ctx *ctx, const unsigned char *d_in, size_t in_len,
                                               int is_double, size_t n, double absErrBound, int blockSize,
                                               void *d_out) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_in || !d_out) { set_error("szp_b200_plain_decompress_dev: null argument"); return -1; }
  if (n == 0 || n >= kMaxElements) { set_error("szp_b200_plain_decompress_dev: element count out of range"); return -1; }
  if (!plain_block_ok(blockSize, "szp_b200_plain_decompress_dev")) return -1;
  return is_double ? plain_decompress_dev_impl<double>(ctx, d_in, in_len, n, absErrBound, blockSize,
                                                       static_cast<double *>(d_out))
                   : plain_decompress_dev_impl<float>(ctx, d_in, in_len, n, (float)absErrBound, blockSize,
                                                      static_cast<float *>(d_out));
}

}  // extern "C"
