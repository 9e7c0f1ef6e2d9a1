// Sort positions: dense rank of a critical point's value among the distinct
// values of all critical points in the same quantization bin
// (SZp/src/szp_float.cc:137-509; SZp/src/szp_cuda_topology.cu:139-272).
//
// No comparison sort of all K points.  Instead:
//   1. bucket the points by  bin mod NB  (matrix histogram -> column scan ->
//      scatter; the order inside a bucket is irrelevant because ties share a
//      rank);
//   2. rank every bucket inside one CTA: the bins of a bucket are slots, each
//      slot gets a shared-memory bitmap over its [min code, max code] range,
//      every point sets the bit of its value code, and the dense rank is the
//      popcount of the bits below its own code;
//   3. buckets whose slots do not fit (bins spanning huge code ranges, e.g.
//      values next to zero, or too many bins) fall back to a device-wide LSD
//      radix sort on (bin, code) followed by a segmented distinct count.
#include <algorithm>
#include <vector>

#include "tsz_ops.h"
#include "tsz_lookback.cuh"
#include "tsz_scan.cuh"

namespace tsz {

constexpr int kRankThreads = 512;
constexpr int kMaxSlots = 256;
constexpr int kBitmapWords = 5120;   // 20 KB bitmap + 20 KB prefix per CTA

// A bucketed record is the critical-point pair itself ({value code, extremum
// index}).  Its bin is recomputed from the code, or, when the caller supplies
// bins (batches, whose bins carry per-field offsets, or a given CP list), read
// from a bin array permuted together with the records.
struct BinSrc {
  const int *bins;   // bins in record order, or nullptr
  float eb;
  double inv;
  __device__ __forceinline__ int operator()(const uint2 &r, unsigned long long i) const {
    return bins ? bins[i] : quant_bin(code_float(r.x), eb, inv);
  }
};

// A chunk of records that belongs to one segment (one field of a batch):
// records [k0, k1) use buckets bbase .. bbase + NB - 1.
struct SegChunk {
  unsigned long long k0, k1;
  unsigned long long bbase;
};

// exclusive scan of one value per thread over a CTA of T threads; the total
// goes to *total; s_w holds T/32 words and may be reused after the return
template <int T>
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned *s_w, unsigned *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  unsigned wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < T / 32; w++) {
    const unsigned x = s_w[w];
    if (w < warp) wpre += x;
    tot += x;
  }
  __syncthreads();
  *total = tot;
  return wpre + inc - v;
}

// ---- 1a. per-CTA bucket histogram over a contiguous chunk -----------------
// (seg != nullptr: CTA c takes chunk seg[c] instead of the c-th uniform chunk)
constexpr int kHistThreads = 512;
constexpr int kHistUnroll = 4;

__global__ void __launch_bounds__(kHistThreads)
bucket_hist_kernel(const uint2 *__restrict__ pairs, BinSrc bin_of, unsigned long long K, int logNB,
                   unsigned long long chunk, unsigned *__restrict__ M, const SegChunk *__restrict__ seg = nullptr) {
  extern __shared__ unsigned sh[];
  const int NB = 1 << logNB;
  for (int b = threadIdx.x; b < NB; b += blockDim.x) sh[b] = 0;
  __syncthreads();
  const unsigned long long c0 = seg ? seg[blockIdx.x].k0 : blockIdx.x * chunk;
  const unsigned long long c1 = seg ? seg[blockIdx.x].k1 : ((c0 + chunk < K) ? c0 + chunk : K);
  for (unsigned long long k = c0 + threadIdx.x; k < c1; k += (unsigned long long)kHistUnroll * kHistThreads) {
    uint2 r[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; u++) {
      const unsigned long long j = k + (unsigned long long)u * kHistThreads;
      if (j < c1) r[u] = pairs[j];
    }
#pragma unroll
    for (int u = 0; u < kHistUnroll; u++) {
      const unsigned long long j = k + (unsigned long long)u * kHistThreads;
      if (j < c1) atomicAdd(&sh[(unsigned)bin_of(r[u], j) & (unsigned)(NB - 1)], 1u);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < NB; b += blockDim.x) M[(size_t)blockIdx.x * NB + b] = sh[b];
}

// ---- 1b. column scan: M[g][b] <- exclusive prefix over g; tot[b] ----------
// rows g0 .. g1-1 of column b, eight loads in flight
__device__ __forceinline__ unsigned colscan_rows(unsigned *__restrict__ M, unsigned g0, unsigned g1, int NB, int b) {
  unsigned run = 0;
  unsigned g = g0;
  for (; g + 8 <= g1; g += 8) {
    unsigned v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = M[(size_t)(g + u) * NB + b];
#pragma unroll
    for (int u = 0; u < 8; u++) { M[(size_t)(g + u) * NB + b] = run; run += v[u]; }
  }
  for (; g < g1; g++) {
    const unsigned v = M[(size_t)g * NB + b];
    M[(size_t)g * NB + b] = run;
    run += v;
  }
  return run;
}

__global__ void bucket_colscan_kernel(unsigned *__restrict__ M, int G, int NB, unsigned *__restrict__ tot) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= NB) return;
  tot[b] = colscan_rows(M, 0, (unsigned)G, NB, b);
}

// segmented column scan: bucket b of segment f scans the rows (chunks)
// crow[f] .. crow[f+1]-1; its totals go to tot[f * NB + b]
__global__ void bucket_colscan_seg_kernel(unsigned *__restrict__ M, const unsigned *__restrict__ crow, int F,
                                          int NB, unsigned *__restrict__ tot) {
  const long long gb = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gb >= (long long)F * NB) return;
  const int f = (int)(gb / NB), b = (int)(gb % NB);
  tot[gb] = colscan_rows(M, crow[f], crow[f + 1], NB, b);
}

// ---- 1c. exclusive scan of bucket totals (one CTA) -------------------------
__global__ void bucket_start_kernel(const unsigned *__restrict__ tot, int NB,
                                    unsigned long long *__restrict__ start) {
  __shared__ unsigned long long part[1024];
  const int per = (NB + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per;
  unsigned long long s = 0;
  for (int i = 0; i < per; i++) if (b0 + i < NB) s += tot[b0 + i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    unsigned long long v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned long long run = part[threadIdx.x] - s;
  for (int i = 0; i < per; i++)
    if (b0 + i < NB) { start[b0 + i] = run; run += tot[b0 + i]; }
  if (threadIdx.x == blockDim.x - 1) start[NB] = part[threadIdx.x];
}

// ---- 1d. scatter into buckets, coalesced ---------------------------------
// Each CTA walks its chunk in sub-chunks of kSub records: the records are
// counting-sorted by bucket in shared memory, then written out in that order,
// so every bucket's records of a sub-chunk form one contiguous run in global
// memory (consecutive threads store consecutive addresses).  The next
// sub-chunk's records are loaded while the current one is written out.
constexpr int kSub = 4096;
constexpr int kScatterThreads = 512;
constexpr int kScatterPer = kSub / kScatterThreads;

__host__ __device__ constexpr size_t scatter_smem(int NB) {
  return (size_t)NB * 16 + (size_t)kSub * 12;
}

__global__ void __launch_bounds__(kScatterThreads)
bucket_scatter_sorted_kernel(const uint2 *__restrict__ pairs, BinSrc bin_of, unsigned long long K, int logNB,
                             unsigned long long chunk, const unsigned *__restrict__ M,
                             const unsigned long long *__restrict__ start_all, uint2 *__restrict__ recs,
                             int *__restrict__ rbins, const SegChunk *__restrict__ seg = nullptr) {
  extern __shared__ unsigned long long smx[];
  const int NB = 1 << logNB;
  unsigned long long *base = smx;                              // next global position per bucket
  unsigned *hist = reinterpret_cast<unsigned *>(base + NB);    // per sub-chunk counts
  unsigned *off = hist + NB;                                   // per sub-chunk exclusive offsets
  uint2 *stage = reinterpret_cast<uint2 *>(off + NB);          // kSub staged records
  int *sbin = reinterpret_cast<int *>(stage + kSub);           // their bins
  __shared__ unsigned s_w[kScatterThreads / 32];
  const unsigned long long c0 = seg ? seg[blockIdx.x].k0 : blockIdx.x * chunk;
  const unsigned long long c1 = seg ? seg[blockIdx.x].k1 : ((c0 + chunk < K) ? c0 + chunk : K);
  const unsigned long long *start = start_all + (seg ? seg[blockIdx.x].bbase : 0ull);
  for (int b = threadIdx.x; b < NB; b += blockDim.x) {
    base[b] = start[b] + M[(size_t)blockIdx.x * NB + b];
    hist[b] = 0;
  }
  uint2 pr[kScatterPer];
#pragma unroll
  for (int u = 0; u < kScatterPer; u++) {
    const unsigned long long k = c0 + threadIdx.x + u * kScatterThreads;
    if (k < c1) pr[u] = pairs[k];
  }
  __syncthreads();
  for (unsigned long long sub = c0; sub < c1; sub += kSub) {
    const int cnt = (int)((c1 - sub) < (unsigned long long)kSub ? (c1 - sub) : kSub);
    // bucket and in-bucket slot of each record (slot order within a bucket is irrelevant)
    int bn[kScatterPer];
    unsigned slot[kScatterPer];
#pragma unroll
    for (int u = 0; u < kScatterPer; u++) {
      const int i = threadIdx.x + u * kScatterThreads;
      if (i < cnt) {
        bn[u] = bin_of(pr[u], sub + i);
        slot[u] = atomicAdd(&hist[(unsigned)bn[u] & (unsigned)(NB - 1)], 1u);
      }
    }
    __syncthreads();
    // exclusive scan of hist -> off (NB <= 4 * kScatterThreads)
    {
      const int per = (NB + kScatterThreads - 1) / kScatterThreads;
      const int b0 = threadIdx.x * per;
      unsigned sum = 0, total;
      for (int i = 0; i < per; i++) if (b0 + i < NB) sum += hist[b0 + i];
      unsigned r = block_excl_scan<kScatterThreads>(sum, s_w, &total);
      for (int i = 0; i < per; i++)
        if (b0 + i < NB) { off[b0 + i] = r; r += hist[b0 + i]; }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kScatterPer; u++) {
      const int i = threadIdx.x + u * kScatterThreads;
      if (i < cnt) {
        const unsigned pos = off[(unsigned)bn[u] & (unsigned)(NB - 1)] + slot[u];
        stage[pos] = pr[u];
        sbin[pos] = bn[u];
      }
    }
    __syncthreads();
    // next sub-chunk in flight during the write-out
    if (sub + kSub < c1) {
#pragma unroll
      for (int u = 0; u < kScatterPer; u++) {
        const unsigned long long k = sub + kSub + threadIdx.x + u * kScatterThreads;
        if (k < c1) pr[u] = pairs[k];
      }
    }
    // write in staged (bucket) order: global = base[b] + (i - off[b])
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int bv = sbin[i];
      const unsigned b = (unsigned)bv & (unsigned)(NB - 1);
      const unsigned long long g = base[b] + (unsigned)(i - off[b]);
      recs[g] = stage[i];
      if (rbins) rbins[g] = bv;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < NB; b += blockDim.x) {
      base[b] += hist[b];
      hist[b] = 0;
    }
    __syncthreads();
  }
}

// ---- 2. per-bucket bitmap rank ---------------------------------------------
// Records are read in three passes (bin bounds, bitmap, ranks), kRankUnroll
// loads in flight per thread.
constexpr int kRankUnroll = 4;

__global__ void __launch_bounds__(kRankThreads)
bucket_rank_kernel(const uint2 *__restrict__ recs, BinSrc bin_of, const unsigned long long *__restrict__ start,
                   int logNB, int *__restrict__ out, unsigned *__restrict__ fb_list,
                   unsigned *__restrict__ fb_count) {
  __shared__ unsigned s_min[kMaxSlots], s_max[kMaxSlots], s_wbase[kMaxSlots + 1];
  __shared__ unsigned bm[kBitmapWords];
  __shared__ unsigned pref[kBitmapWords];
  __shared__ unsigned s_w[kRankThreads / 32];
  __shared__ int s_bmin, s_bmax;
  const unsigned b = blockIdx.x;
  const unsigned long long r0 = start[b], r1 = start[b + 1];
  if (r1 == r0) return;
  const unsigned long long cnt = r1 - r0;
  constexpr unsigned long long kStep = (unsigned long long)kRankUnroll * kRankThreads;
  // bins of this bucket are b + k * NB; slot = k mod kMaxSlots is one-to-one
  // whenever the bucket's bins span fewer than kMaxSlots values of k
  for (int sl = threadIdx.x; sl < kMaxSlots; sl += blockDim.x) { s_min[sl] = 0xffffffffu; s_max[sl] = 0u; }
  if (threadIdx.x == 0) { s_bmin = 0x7fffffff; s_bmax = (int)0x80000000; }
  __syncthreads();
  int lmin = 0x7fffffff, lmax = (int)0x80000000;
  for (unsigned long long i = threadIdx.x; i < cnt; i += kStep) {
    uint2 r[kRankUnroll];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++)
      if (i + u * kRankThreads < cnt) r[u] = recs[r0 + i + u * kRankThreads];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++) {
      if (i + u * kRankThreads >= cnt) continue;
      const int bn = bin_of(r[u], r0 + i + u * kRankThreads);
      lmin = min(lmin, bn);
      lmax = max(lmax, bn);
      const int sl = (bn >> logNB) & (kMaxSlots - 1);
      atomicMin(&s_min[sl], r[u].x);
      atomicMax(&s_max[sl], r[u].x);
    }
  }
  atomicMin(&s_bmin, lmin);
  atomicMax(&s_bmax, lmax);
  __syncthreads();
  const long long span = ((long long)s_bmax >> logNB) - ((long long)s_bmin >> logNB);
  if (span + 1 > kMaxSlots) {
    if (threadIdx.x == 0) fb_list[atomicAdd(fb_count, 1u)] = b;
    return;
  }
  // bitmap words of every slot, laid out by an exclusive scan over the slots
  {
    unsigned wv = 0;
    if (threadIdx.x < kMaxSlots && s_max[threadIdx.x] >= s_min[threadIdx.x])
      wv = ((s_max[threadIdx.x] - s_min[threadIdx.x]) >> 5) + 1;
    // a slot wider than the bitmap saturates so that the sum cannot wrap
    if (wv > kBitmapWords + 1) wv = kBitmapWords + 1;
    unsigned total;
    const unsigned wb = block_excl_scan<kRankThreads>(wv, s_w, &total);
    if (total > kBitmapWords) {
      if (threadIdx.x == 0) fb_list[atomicAdd(fb_count, 1u)] = b;
      return;
    }
    if (threadIdx.x < kMaxSlots) s_wbase[threadIdx.x] = wb;
    if (threadIdx.x == 0) s_wbase[kMaxSlots] = total;
  }
  __syncthreads();
  const unsigned W = s_wbase[kMaxSlots];
  for (unsigned w = threadIdx.x; w < W; w += blockDim.x) bm[w] = 0u;
  __syncthreads();
  for (unsigned long long i = threadIdx.x; i < cnt; i += kStep) {
    uint2 r[kRankUnroll];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++)
      if (i + u * kRankThreads < cnt) r[u] = recs[r0 + i + u * kRankThreads];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++) {
      if (i + u * kRankThreads >= cnt) continue;
      const int sl = (bin_of(r[u], r0 + i + u * kRankThreads) >> logNB) & (kMaxSlots - 1);
      const unsigned pos = r[u].x - s_min[sl];
      atomicOr(&bm[s_wbase[sl] + (pos >> 5)], 1u << (pos & 31));
    }
  }
  __syncthreads();
  // exclusive prefix popcount over the bitmap words (each thread owns a run)
  {
    const unsigned per = (W + blockDim.x - 1) / blockDim.x;
    const unsigned w0 = threadIdx.x * per;
    unsigned sm = 0, total;
    for (unsigned i = 0; i < per; i++) if (w0 + i < W) sm += __popc(bm[w0 + i]);
    unsigned run = block_excl_scan<kRankThreads>(sm, s_w, &total);
    for (unsigned i = 0; i < per; i++)
      if (w0 + i < W) { pref[w0 + i] = run; run += __popc(bm[w0 + i]); }
  }
  __syncthreads();
  for (unsigned long long i = threadIdx.x; i < cnt; i += kStep) {
    uint2 r[kRankUnroll];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++)
      if (i + u * kRankThreads < cnt) r[u] = recs[r0 + i + u * kRankThreads];
#pragma unroll
    for (int u = 0; u < kRankUnroll; u++) {
      if (i + u * kRankThreads >= cnt || r[u].y == kNoExtremum) continue;
      const int sl = (bin_of(r[u], r0 + i + u * kRankThreads) >> logNB) & (kMaxSlots - 1);
      const unsigned pos = r[u].x - s_min[sl];
      const unsigned w = s_wbase[sl] + (pos >> 5);
      const unsigned below = __popc(bm[w] & ((1u << (pos & 31)) - 1u));
      out[r[u].y] = (int)(pref[w] - pref[s_wbase[sl]] + below);
    }
  }
}

// ---- 2b. buckets the bitmap cannot hold, up to kSortCap records: sorted ----
// in shared memory by (bin, code) (bitonic), then ranked by a segmented scan
// (a new bin restarts at 0, every new distinct code adds 1).  Larger buckets
// go on to the device-wide fallback.
constexpr int kSortCap = 8192;
constexpr int kSortThreads = 1024;

__global__ void __launch_bounds__(kSortThreads)
bucket_sort_rank_kernel(const uint2 *__restrict__ recs, BinSrc bin_of, const unsigned long long *__restrict__ start,
                        const unsigned *__restrict__ fb_list, const unsigned *__restrict__ fb_count,
                        int *__restrict__ out, unsigned *__restrict__ fb2_list, unsigned *__restrict__ fb2_count) {
  extern __shared__ unsigned long long sk[];
  unsigned *sd = reinterpret_cast<unsigned *>(sk + kSortCap);
  __shared__ unsigned s_flag[kSortThreads];
  __shared__ unsigned s_val[kSortThreads];
  if (blockIdx.x >= *fb_count) return;
  const unsigned b = fb_list[blockIdx.x];
  const unsigned long long r0 = start[b], r1 = start[b + 1];
  const unsigned cnt = (unsigned)(r1 - r0);
  if (r1 - r0 > (unsigned long long)kSortCap) {
    if (threadIdx.x == 0) fb2_list[atomicAdd(fb2_count, 1u)] = b;
    return;
  }
  unsigned P = 1;
  while (P < cnt) P <<= 1;
  for (unsigned i = threadIdx.x; i < P; i += blockDim.x) {
    if (i < cnt) {
      const uint2 r = recs[r0 + i];
      sk[i] = ((unsigned long long)((unsigned)bin_of(r, r0 + i) ^ 0x80000000u) << 32) | r.x;
      sd[i] = r.y;
    } else {
      sk[i] = ~0ull;
      sd[i] = kNoExtremum;
    }
  }
  __syncthreads();
  for (unsigned k = 2; k <= P; k <<= 1) {
    for (unsigned j = k >> 1; j > 0; j >>= 1) {
      for (unsigned i = threadIdx.x; i < P; i += blockDim.x) {
        const unsigned ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = sk[i], c = sk[ixj];
          if ((a > c) == ((i & k) == 0)) {
            sk[i] = c;
            sk[ixj] = a;
            const unsigned t = sd[i];
            sd[i] = sd[ixj];
            sd[ixj] = t;
          }
        }
      }
      __syncthreads();
    }
  }
  // each thread owns a contiguous run of the sorted records
  const unsigned per = (cnt + blockDim.x - 1) / blockDim.x;
  const unsigned i0 = threadIdx.x * per, i1 = min(i0 + per, cnt);
  unsigned flag = 0, val = 0;
  for (unsigned i = i0; i < i1; i++) {
    const bool st = (i == 0) || (sk[i] >> 32) != (sk[i - 1] >> 32);
    if (st) { flag = 1; val = 0; }
    else if ((unsigned)sk[i] != (unsigned)sk[i - 1]) val++;
  }
  s_flag[threadIdx.x] = flag;
  s_val[threadIdx.x] = val;
  __syncthreads();
  // inclusive segmented scan over threads: (f1, v1) then (f2, v2) -> (f1|f2, f2 ? v2 : v1 + v2)
  for (unsigned o = 1; o < blockDim.x; o <<= 1) {
    unsigned pf = 0, pv = 0;
    if (threadIdx.x >= o) { pf = s_flag[threadIdx.x - o]; pv = s_val[threadIdx.x - o]; }
    __syncthreads();
    if (threadIdx.x >= o && !s_flag[threadIdx.x]) { s_val[threadIdx.x] += pv; s_flag[threadIdx.x] = pf; }
    __syncthreads();
  }
  unsigned run = threadIdx.x ? s_val[threadIdx.x - 1] : 0u;
  for (unsigned i = i0; i < i1; i++) {
    const bool st = (i == 0) || (sk[i] >> 32) != (sk[i - 1] >> 32);
    if (st) run = 0;
    else if ((unsigned)sk[i] != (unsigned)sk[i - 1]) run++;
    if (sd[i] != kNoExtremum) out[sd[i]] = (int)run;
  }
}

static size_t sort_rank_smem() { return (size_t)kSortCap * 12; }

// ---- 3. fallback: device-wide LSD radix sort on (bin, code) ---------------
// gather the records of the failed buckets into a contiguous list
__global__ void fb_gather_count_kernel(const unsigned *__restrict__ fb_list, unsigned nfb,
                                       const unsigned long long *__restrict__ start,
                                       unsigned long long *__restrict__ fb_len) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nfb) fb_len[i] = start[fb_list[i] + 1] - start[fb_list[i]];
}

__global__ void fb_gather_kernel(const unsigned *__restrict__ fb_list, unsigned nfb,
                                 const unsigned long long *__restrict__ start,
                                 const unsigned long long *__restrict__ fb_off,
                                 const uint2 *__restrict__ recs, BinSrc bin_of, bool code_keys,
                                 unsigned long long *__restrict__ key,
                                 unsigned *__restrict__ val) {
  for (unsigned f = blockIdx.x; f < nfb; f += gridDim.x) {
    const unsigned long long r0 = start[fb_list[f]], r1 = start[fb_list[f] + 1];
    const unsigned long long o = fb_off[f];
    for (unsigned long long i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const uint2 r = recs[i];
      key[o + (i - r0)] = code_keys ? (unsigned long long)r.x
                                    : (((unsigned long long)((unsigned)bin_of(r, i) ^ 0x80000000u) << 32) | r.x);
      val[o + (i - r0)] = r.y;
    }
  }
}

constexpr int kRadixTile = 2048;   // items per tile (8 per thread)

__global__ void radix_hist_kernel(const unsigned long long *__restrict__ key, unsigned long long n,
                                  int shift, unsigned *__restrict__ H, unsigned ntiles) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kRadixTile;
  for (int i = threadIdx.x; i < kRadixTile; i += 256) {
    const unsigned long long k = t0 + i;
    if (k < n) atomicAdd(&h[(key[k] >> shift) & 255u], 1u);
  }
  __syncthreads();
  H[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];  // digit-major
}

// stable scatter: items of a tile are ranked in order, 256 at a time
__global__ void radix_scatter_kernel(const unsigned long long *__restrict__ key,
                                     const unsigned *__restrict__ val, unsigned long long n,
                                     int shift, const unsigned *__restrict__ H, unsigned ntiles,
                                     unsigned long long *__restrict__ key2,
                                     unsigned *__restrict__ val2) {
  __shared__ unsigned base[256];
  __shared__ unsigned wcnt[8][256];
  base[threadIdx.x] = H[(size_t)threadIdx.x * ntiles + blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kRadixTile;
  for (int c = 0; c < kRadixTile; c += 256) {
    for (int w = 0; w < 8; w++) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const unsigned long long k = t0 + c + threadIdx.x;
    const bool in = k < n;
    unsigned long long kv = in ? key[k] : 0ull;
    const unsigned d = in ? (unsigned)((kv >> shift) & 255u) : 256u + (unsigned)warp;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank_in_warp = __popc(peers & ((1u << lane) - 1u));
    const int leader = __ffs(peers) - 1;
    if (in && lane == leader) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    unsigned before = 0;
    if (in) {
      for (int w = 0; w < warp; w++) before += wcnt[w][d];
      const unsigned pos = base[d] + before + rank_in_warp;
      key2[pos] = kv;
      val2[pos] = val[k];
    }
    __syncthreads();
    // advance the per-digit base by this chunk's totals
    unsigned tot = 0;
    for (int w = 0; w < 8; w++) tot += wcnt[w][threadIdx.x];
    base[threadIdx.x] += tot;
    __syncthreads();
  }
}

// Dense rank inside bins of the sorted fallback list, in parallel:
//   A[i] = 1 where a new distinct key starts; D = inclusive sum of A
//   H[i] = D[i] where a new bin starts (else 0); Dh = inclusive max of H
//   rank[i] = D[i] - Dh[i]  (distinct keys of the bin before key i)
// Keys are (bin, code) pairs, or codes alone when the bins follow from the
// codes (a bin is a monotone function of the value).
__device__ __forceinline__ unsigned long long fb_bin(unsigned long long k, bool code_keys, float eb, double inv) {
  return code_keys ? (unsigned long long)(unsigned)quant_bin(code_float((unsigned)k), eb, inv) : (k >> 32);
}

__global__ void fb_distinct_kernel(const unsigned long long *__restrict__ key, unsigned long long n,
                                   unsigned *__restrict__ A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

__global__ void fb_heads_kernel(const unsigned long long *__restrict__ key, unsigned long long n,
                                const unsigned *__restrict__ D, bool code_keys, float eb, double inv,
                                unsigned *__restrict__ H) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool head = i == 0 || fb_bin(key[i], code_keys, eb, inv) != fb_bin(key[i - 1], code_keys, eb, inv);
  H[i] = head ? D[i] : 0u;
}

__global__ void fb_out_kernel(const unsigned *__restrict__ val, unsigned long long n, const unsigned *__restrict__ D,
                              const unsigned *__restrict__ Dh, int *__restrict__ out) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && val[i] != kNoExtremum) out[val[i]] = (int)(D[i] - Dh[i]);
}

static int rank_fallback(szp_b200_ctx *ctx, const uint2 *recs, BinSrc bin_of, const unsigned long long *start,
                         const unsigned *fb_list, unsigned nfb, int *d_sp);

// bucket stages shared by the single-field and segmented drivers, launched
// after the histogram matrix M and the bucket starts exist
static int rank_buckets(szp_b200_ctx *ctx, const uint2 *d_pairs, BinSrc src, unsigned long long K, int logNB,
                        unsigned nbk, unsigned C, unsigned long long chunk, const unsigned *M,
                        const unsigned long long *start, const SegChunk *d_chunks, int *d_sp) {
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->scratch;
  uint2 *recs = A.take<uint2>(K);
  int *rbins = src.bins ? A.take<int>(K) : nullptr;
  unsigned *fb_list = A.take<unsigned>(nbk);
  unsigned *fb2_list = A.take<unsigned>(nbk);
  unsigned *fb_cnt = A.take<unsigned>(4);
  if (!recs || (src.bins && !rbins) || !fb_list || !fb2_list || !fb_cnt) {
    set_error("scratch arena too small for the rank stage");
    return -1;
  }
  const size_t ssm = scatter_smem(1 << logNB);
  cudaFuncSetAttribute(bucket_scatter_sorted_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm);
  bucket_scatter_sorted_kernel<<<C, kScatterThreads, ssm, s>>>(d_pairs, src, K, logNB, chunk, M, start, recs,
                                                               rbins, d_chunks);
  // past the scatter, bins (when given) are read in record order
  const BinSrc rsrc = {rbins, src.eb, src.inv};
  if (cuda_fail(cudaMemsetAsync(fb_cnt, 0, 16, s), "memset")) return -1;
  bucket_rank_kernel<<<nbk, kRankThreads, 0, s>>>(recs, rsrc, start, logNB, d_sp, fb_list, fb_cnt);
  cudaFuncSetAttribute(bucket_sort_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sort_rank_smem());
  bucket_sort_rank_kernel<<<nbk, kSortThreads, sort_rank_smem(), s>>>(recs, rsrc, start, fb_list, fb_cnt, d_sp,
                                                                      fb2_list, fb_cnt + 1);
  ctx->launches += 3;
  if (cuda_fail(cudaGetLastError(), "rank kernels")) return -1;
  unsigned nfb = 0;
  if (cuda_fail(cudaMemcpyAsync(&nfb, fb_cnt + 1, 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "rank"))
    return -1;
  if (nfb == 0) return 0;
  return rank_fallback(ctx, recs, rsrc, start, fb2_list, nfb, d_sp);
}

int rank_positions(szp_b200_ctx *ctx, const uint2 *d_pairs, const int *d_bins,
                   unsigned long long K, unsigned long long E, float eb, int *d_sp) {
  if (K == 0) return 0;
  (void)E;
  cudaStream_t s = ctx->stream;
  const BinSrc src = {d_bins, eb, 1.0 / (double)eb};
  // 2^9 buckets keep each bucket's bins (slots) within the shared bitmap for
  // typical fields while giving the coalesced scatter long runs
  int logNB = 6;
  while (logNB < 9 && (K >> logNB) > 2048) logNB++;
  const int NB = 1 << logNB;
  int G = ctx->sm_count * 2;
  unsigned long long chunk = (K + G - 1) / G;
  if (chunk < 4096) { chunk = 4096; G = (int)((K + chunk - 1) / chunk); }
  Arena &A = ctx->scratch;
  unsigned *M = A.take<unsigned>((size_t)G * NB);
  unsigned *tot = A.take<unsigned>(NB);
  unsigned long long *start = A.take<unsigned long long>(NB + 1);
  if (!M || !tot || !start) {
    set_error("scratch arena too small for the rank stage");
    return -1;
  }
  const size_t hsm = (size_t)NB * 4;
  bucket_hist_kernel<<<G, kHistThreads, hsm, s>>>(d_pairs, src, K, logNB, chunk, M);
  bucket_colscan_kernel<<<(NB + 255) / 256, 256, 0, s>>>(M, G, NB, tot);
  bucket_start_kernel<<<1, 1024, 0, s>>>(tot, NB, start);
  ctx->launches += 3;
  return rank_buckets(ctx, d_pairs, src, K, logNB, (unsigned)NB, (unsigned)G, chunk, M, start, nullptr, d_sp);
}

// Buckets that did not fit the bitmap rank: their records are gathered and
// ranked after a device-wide LSD radix sort on (bin, code) -- on the code
// alone when the bins follow from the codes -- and a parallel segmented
// distinct count.
static int rank_fallback(szp_b200_ctx *ctx, const uint2 *recs, BinSrc bin_of, const unsigned long long *start,
                         const unsigned *fb_list, unsigned nfb, int *d_sp) {
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->scratch;
  unsigned long long *fb_len = A.take<unsigned long long>(nfb + 1);
  if (!fb_len) { set_error("scratch arena too small for the rank fallback"); return -1; }
  fb_gather_count_kernel<<<(nfb + 255) / 256, 256, 0, s>>>(fb_list, nfb, start, fb_len);
  std::vector<unsigned long long> h_len(nfb);
  if (cuda_fail(cudaMemcpyAsync(h_len.data(), fb_len, nfb * 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "fallback"))
    return -1;
  std::vector<unsigned long long> h_off(nfb);
  unsigned long long nf = 0;
  for (unsigned i = 0; i < nfb; i++) { h_off[i] = nf; nf += h_len[i]; }
  unsigned long long *fb_off = A.take<unsigned long long>(nfb);
  unsigned long long *k1 = A.take<unsigned long long>(nf), *k2 = A.take<unsigned long long>(nf);
  unsigned *v1 = A.take<unsigned>(nf), *v2 = A.take<unsigned>(nf);
  const unsigned ntiles = (unsigned)((nf + kRadixTile - 1) / kRadixTile);
  unsigned *H = A.take<unsigned>((size_t)256 * ntiles);
  const unsigned long long hn = (unsigned long long)256 * ntiles;
  unsigned *part = A.take<unsigned>(scan_parts(hn > nf ? hn : nf));
  if (!fb_off || !k1 || !k2 || !v1 || !v2 || !H || !part) {
    set_error("scratch arena too small for the rank fallback");
    return -1;
  }
  const bool code_keys = bin_of.bins == nullptr;
  cudaMemcpyAsync(fb_off, h_off.data(), nfb * 8, cudaMemcpyHostToDevice, s);
  fb_gather_kernel<<<std::min(nfb, 4096u), 256, 0, s>>>(fb_list, nfb, start, fb_off, recs, bin_of, code_keys, k1,
                                                          v1);
  const int bits = code_keys ? 32 : 64;
  for (int shift = 0; shift < bits; shift += 8) {
    radix_hist_kernel<<<ntiles, 256, 0, s>>>(k1, nf, shift, H, ntiles);
    if (cuda_fail(device_scan_u32<OpAdd>(H, H, hn, part, false, s), "scan")) return -1;
    radix_scatter_kernel<<<ntiles, 256, 0, s>>>(k1, v1, nf, shift, H, ntiles, k2, v2);
    std::swap(k1, k2);
    std::swap(v1, v2);
  }
  // k2 / v2 are free now: D in the key storage of k2, Dh beside it
  unsigned *D = reinterpret_cast<unsigned *>(k2);
  unsigned *Dh = D + nf;
  const unsigned g = (unsigned)((nf + 255) / 256);
  fb_distinct_kernel<<<g, 256, 0, s>>>(k1, nf, D);
  if (cuda_fail(device_scan_u32<OpAdd>(D, D, nf, part, true, s), "scan")) return -1;
  fb_heads_kernel<<<g, 256, 0, s>>>(k1, nf, D, code_keys, bin_of.eb, bin_of.inv, Dh);
  if (cuda_fail(device_scan_u32<OpMax>(Dh, Dh, nf, part, true, s), "scan")) return -1;
  fb_out_kernel<<<g, 256, 0, s>>>(v1, nf, D, Dh, d_sp);
  ctx->launches += 3 + (bits / 8) * 5 + 9;
  if (cuda_fail(cudaGetLastError(), "fallback kernels") ||
      cuda_fail(cudaStreamSynchronize(s), "fallback"))
    return -1;
  return 0;
}

// Ranks of many segments (fields of a batch) in one pass: every segment gets
// its own NB buckets and chunks never straddle segments, so records of
// different segments never share a bucket.  bins must be disjoint across
// segments (the fallback sorts all failing buckets together by bin).
int rank_positions_seg(szp_b200_ctx *ctx, const uint2 *d_pairs, const int *d_bins,
                       const unsigned long long *h_seg_K, int F, int *d_sp) {
  unsigned long long K = 0;
  for (int f = 0; f < F; f++) K += h_seg_K[f];
  if (K == 0) return 0;
  cudaStream_t s = ctx->stream;
  const int logNB = 9, NB = 1 << logNB;
  unsigned long long chunk = std::max<unsigned long long>(4096, (K + 2 * ctx->sm_count - 1) / (2 * ctx->sm_count));
  std::vector<SegChunk> chunks;
  std::vector<unsigned> crow(F + 1);
  unsigned long long k = 0;
  for (int f = 0; f < F; f++) {
    crow[f] = (unsigned)chunks.size();
    const unsigned long long k1 = k + h_seg_K[f];
    for (unsigned long long c = k; c < k1; c += chunk)
      chunks.push_back({c, std::min(c + chunk, k1), (unsigned long long)f * NB});
    k = k1;
  }
  crow[F] = (unsigned)chunks.size();
  const unsigned C = (unsigned)chunks.size();
  const unsigned long long nbk = (unsigned long long)F * NB;
  Arena &A = ctx->scratch;
  SegChunk *d_chunks = A.take<SegChunk>(C);
  unsigned *d_crow = A.take<unsigned>(F + 1);
  unsigned *M = A.take<unsigned>((size_t)C * NB);
  unsigned *tot = A.take<unsigned>(nbk);
  unsigned long long *start = A.take<unsigned long long>(nbk + 1);
  if (!d_chunks || !d_crow || !M || !tot || !start) {
    set_error("scratch arena too small for the batched rank stage");
    return -1;
  }
  if (cuda_fail(cudaMemcpyAsync(d_chunks, chunks.data(), C * sizeof(SegChunk), cudaMemcpyHostToDevice, s),
                "H2D chunks") ||
      cuda_fail(cudaMemcpyAsync(d_crow, crow.data(), (F + 1) * sizeof(unsigned), cudaMemcpyHostToDevice, s),
                "H2D chunk rows"))
    return -1;
  const BinSrc src = {d_bins, 1.0f, 1.0};
  const size_t hsm = (size_t)NB * 4;
  bucket_hist_kernel<<<C, kHistThreads, hsm, s>>>(d_pairs, src, K, logNB, chunk, M, d_chunks);
  bucket_colscan_seg_kernel<<<(unsigned)((nbk + 255) / 256), 256, 0, s>>>(M, d_crow, F, NB, tot);
  bucket_start_kernel<<<1, 1024, 0, s>>>(tot, (int)nbk, start);
  ctx->launches += 3;
  return rank_buckets(ctx, d_pairs, src, K, logNB, (unsigned)nbk, C, chunk, M, start, d_chunks, d_sp);
}

size_t rank_scratch_bytes_seg(unsigned long long K, int F, int sm_count) {
  const size_t NB = 512;
  const unsigned long long chunk = std::max<unsigned long long>(4096, (K + 2 * sm_count - 1) / (2 * sm_count));
  const size_t C = (size_t)(K / chunk) + (size_t)F + 1;
  const size_t nbk = (size_t)F * NB;
  const size_t fb = a256(K * 8) * 2 + a256(K * 4) * 2 + a256(256 * ((K + kRadixTile - 1) / kRadixTile) * 4) +
                    a256(scan_parts(256 * ((K + kRadixTile - 1) / kRadixTile) + K) * 4);
  return a256(C * sizeof(SegChunk)) + a256((F + 1) * 4) + a256(C * NB * 4) + a256(nbk * 4) +
         a256((nbk + 1) * 8) + a256(K * 8) + a256(K * 4) + a256(nbk * 4) * 2 + a256(16) + fb + a256(nbk * 8) + 8192;
}

size_t rank_scratch_bytes(unsigned long long K, int sm_count) {
  int logNB = 6;
  while (logNB < 9 && (K >> logNB) > 2048) logNB++;
  const size_t NB = (size_t)1 << logNB;
  const size_t G = (size_t)sm_count * 2 + 1;
  // fallback worst case: all K records (two key/value ping-pong buffers + histogram)
  const size_t fb = a256(K * 8) * 2 + a256(K * 4) * 2 + a256(256 * ((K + kRadixTile - 1) / kRadixTile) * 4) +
                    a256(scan_parts(256 * ((K + kRadixTile - 1) / kRadixTile) + K) * 4);
  // records (8 B) and, for given bins, their permuted bins (4 B)
  return a256(G * NB * 4) + a256(NB * 4) + a256((NB + 1) * 8) + a256(K * 8) + a256(K * 4) +
         a256(NB * 4) * 3 + a256(16) + fb + a256((NB + 1) * 8) * 2 + 4096;
}

// ---------------------------------------------------------------------------
// extrema compaction in list order (for the reference's sort-position
// compression of an arbitrary CP list, SZp/src/szp_cuda_topology.cu:436-449)
// ---------------------------------------------------------------------------
__global__ void extrema_compact_kernel(const int *__restrict__ cps, int stride, int type_field,
                                       unsigned long long K, TileDesc *desc, unsigned *tile_ctr,
                                       int *err, int *__restrict__ sp,
                                       unsigned long long *__restrict__ total) {
  __shared__ long long s_tile;
  __shared__ unsigned s_w[8];
  __shared__ unsigned long long s_base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int T = 2048;
  const long long ntiles = (long long)((K + T - 1) / T);
  while (true) {
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) break;
    // each thread owns 8 consecutive items
    const unsigned long long i0 = (unsigned long long)tile * T + threadIdx.x * 8;
    unsigned flags = 0, c = 0;
    for (int u = 0; u < 8; u++) {
      const unsigned long long i = i0 + u;
      if (i < K) {
        const int t = cps[(size_t)i * stride + type_field];
        if (t == 1 || t == 2) { flags |= 1u << u; c++; }
      }
    }
    unsigned incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    unsigned wpre = 0, ttot = 0;
    for (int w = 0; w < 8; w++) { if (w < warp) wpre += s_w[w]; ttot += s_w[w]; }
    if (warp == 0) {
      Prefix pf = lookback(desc, tile, 0, ttot, err);
      if (lane == 0) {
        s_base = pf.cnt;
        if (tile == ntiles - 1) *total = pf.cnt + ttot;
      }
    }
    __syncthreads();
    unsigned long long o = s_base + wpre + incl - c;
    for (int u = 0; u < 8; u++)
      if (flags & (1u << u)) sp[o++] = cps[(size_t)(i0 + u) * stride + 4 + (stride == 6 ? 1 : 0)];
    __syncthreads();
  }
}

int compact_extrema(szp_b200_ctx *ctx, const int *d_cps, int stride, unsigned long long K,
                    int *d_sp, unsigned long long *E_out) {
  cudaStream_t s = ctx->stream;
  const unsigned long long ntiles = (K + 2047) / 2048;
  TileDesc *desc = ctx->scratch.take<TileDesc>(ntiles + 1);
  if (!desc) { set_error("scratch arena too small"); return -1; }
  unsigned long long *w = ctx->d_words;
  if (cuda_fail(cudaMemsetAsync(desc, 0, (ntiles + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(w, 0, 64, s), "memset"))
    return -1;
  const int grid = (int)std::min<unsigned long long>(ntiles, (unsigned long long)ctx->sm_count * 8);
  extrema_compact_kernel<<<grid, 256, 0, s>>>(d_cps, stride, stride == 6 ? 3 : 2, K, desc,
                                              reinterpret_cast<unsigned *>(w + 3),
                                              reinterpret_cast<int *>(w + 4), d_sp, w);
  ctx->launches += 1;
  if (cuda_fail(cudaGetLastError(), "compact") ||
      cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 64, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "compact"))
    return -1;
  if (ctx->h_words[4] & 0xffffffffu) { set_error("compaction status %d", (int)ctx->h_words[4]); return -1; }
  *E_out = ctx->h_words[0];
  return 0;
}

// ---------------------------------------------------------------------------
// API sort of an arbitrary CP list: every CP gets its rank
// ---------------------------------------------------------------------------
__global__ void cp_pairs_kernel(const int *__restrict__ cps, int stride, unsigned long long K,
                                const float *__restrict__ data, long long d2, long long d3,
                                uint2 *__restrict__ pairs, int *__restrict__ bins) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K) return;
  const int *r = cps + (size_t)i * stride;
  unsigned long long flat;
  int bin;
  if (stride == 5) { flat = (unsigned long long)(long long)r[0] * d3 + (long long)r[1]; bin = r[3]; }
  else {
    flat = (unsigned long long)(long long)r[0] * d2 * d3 + (unsigned long long)((long long)r[1] * d3) +
           (long long)r[2];
    bin = r[4];
  }
  pairs[i] = make_uint2(float_code(data[flat]), (unsigned)i);
  bins[i] = bin;
}

__global__ void cp_store_rank_kernel(int *__restrict__ cps, int stride, unsigned long long K,
                                     const int *__restrict__ rank) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K) cps[(size_t)i * stride + stride - 1] = rank[i];
}

int sort_cp_list_host(int *h_cps, int stride, unsigned long long K, const float *h_data,
                      long long d2, long long d3) {
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return -1;
  // extent of the data the list refers to (the reference copies data[0..max_flat])
  unsigned long long max_flat = 0;
  for (unsigned long long i = 0; i < K; i++) {
    const int *r = h_cps + (size_t)i * stride;
    unsigned long long f = (stride == 5)
                               ? (unsigned long long)((long long)r[0] * d3 + r[1])
                               : (unsigned long long)((long long)r[0] * d2 * d3 + (long long)r[1] * d3 + r[2]);
    if (f > max_flat) max_flat = f;
  }
  if (max_flat >= (1ull << 40)) { set_error("critical point coordinates out of range"); return -1; }
  const size_t need = a256((max_flat + 1) * 4) + a256(K * stride * 4) + a256(K * 8) + a256(K * 4) * 2 +
                      rank_scratch_bytes(K, ctx->sm_count);
  if (!ctx->scratch.reserve(need)) return -1;
  Arena &A = ctx->scratch;
  float *d_data = A.take<float>(max_flat + 1);
  int *d_cps = A.take<int>(K * stride);
  uint2 *d_pairs = A.take<uint2>(K);
  int *d_bins = A.take<int>(K);
  int *d_rank = A.take<int>(K);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_data, h_data, (max_flat + 1) * 4, cudaMemcpyHostToDevice, s), "H2D") ||
      cuda_fail(cudaMemcpyAsync(d_cps, h_cps, K * stride * 4, cudaMemcpyHostToDevice, s), "H2D"))
    return -1;
  const unsigned blocks = (unsigned)((K + 255) / 256);
  cp_pairs_kernel<<<blocks, 256, 0, s>>>(d_cps, stride, K, d_data, d2, d3, d_pairs, d_bins);
  if (rank_positions(ctx, d_pairs, d_bins, K, K, 1.0f, d_rank)) return -1;
  cp_store_rank_kernel<<<blocks, 256, 0, s>>>(d_cps, stride, K, d_rank);
  ctx->launches += 2;
  if (cuda_fail(cudaMemcpyAsync(h_cps, d_cps, K * stride * 4, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "sort"))
    return -1;
  return 0;
}

}  // namespace tsz

extern "C" {

void szp_cuda_sort_critical_points_by_original_data(CriticalPoint *critical_points,
                                                     size_t critical_count, float *data, int cols) {
  tsz::clear_error();
  if (!critical_points || critical_count == 0 || !data) return;
  tsz::sort_cp_list_host(reinterpret_cast<int *>(critical_points), 5, critical_count, data, 1, cols);
}

void szp_cuda_sort_critical_points_3d(CriticalPoint3D *critical_points, size_t critical_count,
                                      float *data, int d2, int d3) {
  tsz::clear_error();
  if (!critical_points || critical_count == 0 || !data) return;
  tsz::sort_cp_list_host(reinterpret_cast<int *>(critical_points), 6, critical_count, data, d2, d3);
}

}  // extern "C"
