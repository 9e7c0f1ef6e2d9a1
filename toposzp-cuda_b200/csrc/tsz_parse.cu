// Block offsets of a compressed stream, found on the device from the stream
// bytes alone.
//
// The streams carry no block index: a block's length follows from its bit
// count byte, so block k+1 starts where block k ends and the reference finds
// the offsets with one serial walk (SZp/src/szp_cuda_decompress.cu:233-328
// and its thread-count detection, :400-418).  Here the walk is parallel and
// exact:
//   1. The payload is cut into segments of kSegBytes.  A block that starts in
//      segment j-1 ends less than M bytes into segment j (M = largest valid
//      block), so the first block start in segment j lies in [jS, jS + M).
//      For every segment and every such entry e, one thread walks the blocks
//      that start inside the segment and records (blocks started, exit entry
//      into the next segment) -- a transfer function of the segment.
//   2. Transfer functions are composed kGroup at a time, level by level, up
//      to a single function; entry 0 of the payload is then pushed back down
//      the levels, giving every segment its true entry and the global index
//      of its first block.
//   3. One thread per segment re-walks from its true entry and writes the
//      offsets of the first nb blocks; the thread that reaches block nb-1
//      sizes it with its own element count and records the payload length.
// Validation matches the reference's single-chunk check: every bit count is
// at most 32 and the last block ends inside min(buffer, validation bound).
// A walk that meets a bit count above 32 or the buffer end stops ("stuck");
// such a chain is reported as a failed parse unless it is past block nb-1.
#include "tsz_common.cuh"
#include "tsz_ops.h"
#include "tsz_runtime.h"

namespace tsz {

constexpr unsigned long long kSegBytes = 16384;
constexpr int kGroup = 32;
constexpr unsigned kStuck = 0xFFFFu;   // exit entry of a walk that stopped

// packed transfer value: (blocks started << 16) | exit entry
__device__ __forceinline__ unsigned long long tv_pack(unsigned long long c, unsigned x) {
  return (c << 16) | x;
}

struct ParseGeom {
  const unsigned char *p;      // payload (after the 8-byte offset table)
  unsigned long long len;      // payload bytes present in the buffer
  int B;
  bool tags;
  unsigned full_tag;           // tag bytes of a full block
  unsigned M;                  // largest valid block (bit count 32)
  bool cpu;                    // OpenMP layout: one-element blocks carry a bit-count byte
};

// length of a full block (B elements) from its bit count; 0 = invalid
__device__ __forceinline__ unsigned full_block_len(const ParseGeom &g, unsigned bc) {
  if (g.B == 1) return 4u + (g.cpu ? 1u : 0u) + g.full_tag;
  if (bc > 32u) return 0u;
  unsigned s = 5u + g.full_tag;
  if (bc) s += (unsigned)((g.B - 2) >> 3) + 1u + mag_bytes((unsigned)g.B - 1u, bc);
  return s;
}

// 1. per-segment transfer functions
__global__ void __launch_bounds__(256) parse_seg_kernel(ParseGeom g, unsigned long long nseg,
                                                        unsigned long long *tab) {
  const unsigned long long j = blockIdx.x;
  if (j >= nseg) return;
  const unsigned long long s0 = j * kSegBytes, s1 = s0 + kSegBytes;
  for (unsigned e = threadIdx.x; e < g.M; e += blockDim.x) {
    unsigned long long p = s0 + e, c = 0;
    unsigned x = kStuck;
    while (true) {
      if (p >= s1) { x = (unsigned)(p - s1); break; }
      c++;
      unsigned len;
      if (g.B == 1) {
        len = 4u + (g.cpu ? 1u : 0u) + g.full_tag;
      } else {
        if (p + 4 >= g.len) break;   // bit count byte outside the buffer
        len = full_block_len(g, __ldg(g.p + p + 4));
        if (!len) break;             // bit count above 32
      }
      p += len;
    }
    tab[j * g.M + e] = tv_pack(c, x);
  }
}

// 2a. compose kGroup consecutive functions of one level into one
__global__ void __launch_bounds__(256) parse_up_kernel(const unsigned long long *in, unsigned long long nin,
                                                       unsigned M, unsigned long long *out) {
  const unsigned long long grp = blockIdx.x;
  for (unsigned e = threadIdx.x; e < M; e += blockDim.x) {
    unsigned long long c = 0;
    unsigned x = e;
    for (int k = 0; k < kGroup; k++) {
      const unsigned long long i = grp * kGroup + k;
      if (i >= nin) break;
      const unsigned long long t = in[i * M + x];
      c += t >> 16;
      x = (unsigned)(t & 0xFFFFu);
      if (x == kStuck) break;
    }
    out[grp * M + e] = tv_pack(c, x);
  }
}

// 2b. push (entry, first block index) down one level: one thread per group
__global__ void parse_down_kernel(const unsigned long long *tab, unsigned long long nin, unsigned M,
                                  const unsigned long long *ent_up, unsigned long long ngroups,
                                  unsigned long long *ent) {
  const unsigned long long grp = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if (grp >= ngroups) return;
  const unsigned long long eu = ent_up[grp];
  unsigned long long base = eu >> 16;
  unsigned x = (unsigned)(eu & 0xFFFFu);
  for (int k = 0; k < kGroup; k++) {
    const unsigned long long i = grp * kGroup + k;
    if (i >= nin) break;
    ent[i] = tv_pack(base, x);
    if (x == kStuck) continue;
    const unsigned long long t = tab[i * M + x];
    base += t >> 16;
    x = (unsigned)(t & 0xFFFFu);
  }
}

// 3. offsets of the blocks that start in each segment
struct ParseOut {
  unsigned long long *offs;          // [nb]
  unsigned long long *status;        // [0] payload length + 1 once block nb-1 is sized, [1] error
  unsigned long long n;              // elements (when n_dev is null)
  const unsigned long long *n_dev;   // elements, read on the device (optional)
  unsigned long long maxc;           // validation bound of the whole stream (when n_dev is null)
  bool ref_bound;                    // also bound by the reference's 8n+1024 / 4n+4 limit
};

__global__ void parse_write_kernel(ParseGeom g, unsigned long long nseg, const unsigned long long *ent,
                                   ParseOut o) {
  const unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if (j >= nseg) return;
  const unsigned long long n = o.n_dev ? *o.n_dev : o.n;
  if (n == 0) {
    if (j == 0) o.status[0] = 1;     // empty stream: nothing to walk
    return;
  }
  const unsigned long long nb = (n + g.B - 1) / g.B;
  const unsigned long long nlast = n - (nb - 1) * g.B;
  const unsigned long long maxc =
      !o.ref_bound ? ~0ull : (o.n_dev ? (g.tags ? 8ull * n + 1024ull : 4ull * n + 4ull) : o.maxc);
  // validation bound in payload coordinates (the offset table is 8 bytes)
  const unsigned long long lim = (maxc > 8 ? (maxc - 8 < g.len ? maxc - 8 : g.len) : 0);
  const unsigned long long e = ent[j];
  unsigned x = (unsigned)(e & 0xFFFFu);
  if (x == kStuck) return;
  unsigned long long idx = e >> 16;
  const unsigned long long s1 = (j + 1) * kSegBytes;
  unsigned long long p = j * kSegBytes + x;
  while (p < s1 && idx < nb) {
    o.offs[idx] = p;
    const unsigned long long len = (idx == nb - 1) ? nlast : (unsigned long long)g.B;
    unsigned long long q;
    if (len > 1) {
      if (p + 4 >= lim) { atomicExch(o.status + 1, 1ull); return; }
      const unsigned bc = __ldg(g.p + p + 4);
      if (bc > 32u) { atomicExch(o.status + 1, 2ull); return; }
      q = p + block_bytes((unsigned)len, bc, g.tags);
    } else {
      q = p + 4 + (g.cpu ? 1 : 0) + (g.tags ? 1 : 0);
    }
    if (idx == nb - 1) {
      if (q > lim) { atomicExch(o.status + 1, 3ull); return; }
      o.status[0] = q + 1;
      return;
    }
    p = q;
    idx++;
  }
}

static unsigned parse_M(int B, bool tags) { return block_bytes((unsigned)B, 32u, tags) + (B == 1 ? 1u : 0u); }

static void parse_levels(unsigned long long nseg, unsigned long long *cnt, int *nlev) {
  int L = 0;
  unsigned long long c = nseg;
  cnt[L++] = c;
  while (c > 1) {
    c = (c + kGroup - 1) / kGroup;
    cnt[L++] = c;
  }
  *nlev = L;
}

size_t parse_scratch_bytes(unsigned long long buf_len, int B, bool tags) {
  const unsigned M = parse_M(B, tags);
  const unsigned long long nseg = buf_len ? (buf_len + kSegBytes - 1) / kSegBytes : 1;
  unsigned long long cnt[16];
  int L;
  parse_levels(nseg, cnt, &L);
  size_t s = 0;
  for (int l = 0; l < L; l++) s += a256(cnt[l] * M * 8) + a256(cnt[l] * 8);
  return s + 1024;
}

int parse_stream(szp_b200_ctx *ctx, Arena &A, const unsigned char *d_payload, unsigned long long buf_len,
                 unsigned long long n, const unsigned long long *d_n, int B, bool tags, bool ref_bound,
                 unsigned long long *d_offs, unsigned long long *d_status, bool cpu) {
  cudaStream_t s = ctx->stream;
  ParseGeom g;
  g.cpu = cpu;
  g.p = d_payload;
  g.len = buf_len;
  g.B = B;
  g.tags = tags;
  g.full_tag = tags ? (2u * (unsigned)B + 7u) / 8u : 0u;
  g.M = parse_M(B, tags);
  const unsigned long long nseg = buf_len ? (buf_len + kSegBytes - 1) / kSegBytes : 1;
  unsigned long long cnt[16];
  int L;
  parse_levels(nseg, cnt, &L);
  unsigned long long *tab[16], *ent[16];
  for (int l = 0; l < L; l++) {
    tab[l] = A.take<unsigned long long>(cnt[l] * g.M);
    ent[l] = A.take<unsigned long long>(cnt[l]);
    if (!tab[l] || !ent[l]) { set_error("scratch arena too small for the stream parser"); return -1; }
  }
  if (cuda_fail(cudaMemsetAsync(d_status, 0, 2 * sizeof(unsigned long long), s), "memset") ||
      cuda_fail(cudaMemsetAsync(ent[L - 1], 0, cnt[L - 1] * 8, s), "memset"))
    return -1;
  parse_seg_kernel<<<(unsigned)nseg, 256, 0, s>>>(g, nseg, tab[0]);
  for (int l = 1; l < L; l++)
    parse_up_kernel<<<(unsigned)cnt[l], 256, 0, s>>>(tab[l - 1], cnt[l - 1], g.M, tab[l]);
  // the top level holds one group whose entry is payload offset 0, block 0
  for (int l = L - 2; l >= 0; l--)
    parse_down_kernel<<<(unsigned)((cnt[l + 1] + 127) / 128), 128, 0, s>>>(tab[l], cnt[l], g.M, ent[l + 1],
                                                                          cnt[l + 1], ent[l]);
  ParseOut o;
  o.offs = d_offs;
  o.status = d_status;
  o.n = n;
  o.n_dev = d_n;
  o.maxc = tags ? 8ull * n + 1024ull : 4ull * n + 4ull;
  o.ref_bound = ref_bound;
  parse_write_kernel<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(g, nseg, ent[0], o);
  ctx->launches += 2 + 2 * (L - 1);
  return cuda_fail(cudaGetLastError(), "stream parser launch") ? -1 : 0;
}

}  // namespace tsz
