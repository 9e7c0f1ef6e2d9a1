// Batched compression: many fields of uneven dims, sizes and error bounds per
// call, with one persistent launch per codec pass.
//
// Stage A (one CUDA graph, replayed per batch):
//   upload the field table -> init -> min/max of the relative-bound fields ->
//   absolute bounds -> ONE persistent topology-encoder launch over a device
//   tile work-queue spanning every field -> per-field CP / extremum prefix ->
//   gather all fields' CP pairs into one list with field-disjoint bins ->
//   results to pinned host memory.
// Rank: one pass of the bucket/bitmap rank over the whole batch (bins of
//   different fields never meet: each field's bins are shifted into its own
//   range).  Should the shifted ranges not fit in 31 bits, fields are ranked
//   one by one instead.
// Stage C (one CUDA graph): upload the sort-stream table -> ONE persistent
//   launch of the integer encoder over all fields' sort positions.
// The streams are byte-identical to the per-field calls.
//
// The encoder's CTA shape (warps per CTA, hence codec blocks per tile) and the
// persistent grid (CTAs per SM) are chosen by an autotuner that times the
// candidates on the first batch; the format's blockSize is never tuned.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstring>
#include <mutex>
#include <vector>

#include "tsz_codec2.cuh"
#include "tsz_ops.h"
#include "tsz_runtime.h"

namespace tsz {

struct BatchFieldDev {
  const float *data;
  unsigned long long n;
  unsigned long long pairs_off;   // first CP-pair slot of this field
  unsigned long long chunk0;      // first min/max chunk of this field
  float err;                      // absolute bound, or the relative factor
  int rel;
  unsigned char *topo;            // topology stream (offset table included)
};

// header of the uploaded tables
struct BatchHdr {
  unsigned nf;
  unsigned pad;
  unsigned long long nchunks;     // min/max chunks over all relative-bound fields
};

constexpr unsigned long long kMinMaxChunk = 1ull << 16;
constexpr int kAuxThreads = 256;

// ---- table layout (host pinned copy and device copy are identical) ----
struct TableLayout {
  size_t hdr, fields, args, tstart, bytes;
  void make(int cap) {
    size_t o = 0;
    hdr = o; o += a256(sizeof(BatchHdr));
    fields = o; o += a256(sizeof(BatchFieldDev) * (size_t)cap);
    args = o; o += a256(sizeof(EncArgs) * (size_t)cap);
    tstart = o; o += a256(8 * ((size_t)cap + 1));
    bytes = o;
  }
};

// ---- results layout (device -> pinned host in one copy) ----
struct ResultLayout {
  size_t totals, kbase, ebase, eb, flags, bytes;
  void make(int cap) {
    size_t o = 0;
    totals = o; o += a256(24 * (size_t)cap);
    kbase = o; o += a256(8 * ((size_t)cap + 1));
    ebase = o; o += a256(8 * ((size_t)cap + 1));
    eb = o; o += a256(4 * (size_t)cap);
    flags = o; o += a256(8 * 8);   // [0] bin overflow, [1] encoder status, [2] bad bound
    bytes = o;
  }
};

__device__ __forceinline__ int last_le(const unsigned long long *a, int n, unsigned long long v) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a[mid] <= v) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void batch_init_kernel(const BatchHdr *hdr, const BatchFieldDev *fields, unsigned *minmax,
                                  int *binmm) {
  const unsigned nf = hdr->nf;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    minmax[2 * f] = 0xFFFFFFFFu;
    minmax[2 * f + 1] = 0u;
    binmm[2 * f] = INT_MAX;
    binmm[2 * f + 1] = INT_MIN;
    unsigned char *t = fields[f].topo;
    for (int i = 0; i < 8; i++) t[i] = 0;   // offset table of a single-chunk stream
  }
}

// min / max (as order-preserving codes) of every relative-bound field
__global__ void __launch_bounds__(kAuxThreads) batch_minmax_kernel(const BatchHdr *hdr,
                                                                   const BatchFieldDev *fields,
                                                                   unsigned *minmax) {
  __shared__ unsigned s_mn[kAuxThreads / 32], s_mx[kAuxThreads / 32];
  const unsigned nf = hdr->nf;
  const unsigned long long nch = hdr->nchunks;
  for (unsigned long long c = blockIdx.x; c < nch; c += gridDim.x) {
    // field owning chunk c: last field with chunk0 <= c among relative-bound fields
    int lo = 0, hi = (int)nf - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (fields[mid].chunk0 <= c) lo = mid; else hi = mid - 1;
    }
    // (a field without chunks shares chunk0 with the next field, which owns c)
    const BatchFieldDev &fd = fields[lo];
    const unsigned long long b0 = (c - fd.chunk0) * kMinMaxChunk;
    const unsigned long long b1 = min(fd.n, b0 + kMinMaxChunk);
    unsigned mn = 0xFFFFFFFFu, mx = 0u;
    for (unsigned long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
      const unsigned v = float_code(__ldg(fd.data + i));
      mn = min(mn, v);
      mx = max(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) { s_mn[threadIdx.x >> 5] = mn; s_mx[threadIdx.x >> 5] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < kAuxThreads / 32; w++) { mn = min(mn, s_mn[w]); mx = max(mx, s_mx[w]); }
      atomicMin(&minmax[2 * lo], mn);
      atomicMax(&minmax[2 * lo + 1], mx);
    }
    __syncthreads();
  }
}

// absolute bound of every field: a relative bound is err * (max - min) in
// float, FLT_EPSILON standing in for an empty range (szp_rel_to_abs_float,
// SZp/include/szp_errbound.h:34-101)
__global__ void batch_eb_kernel(const BatchHdr *hdr, const BatchFieldDev *fields, const unsigned *minmax,
                                EncArgs *args, float *eb_out, unsigned long long *flags) {
  const unsigned nf = hdr->nf;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    float eb = fields[f].err;
    if (fields[f].rel) {
      const float mn = code_float(minmax[2 * f]), mx = code_float(minmax[2 * f + 1]);
      float r = __fsub_rn(mx, mn);
      if (r <= 0.0f) r = FLT_EPSILON;
      eb = __fmul_rn(fields[f].err, r);
    }
    if (!(eb > 0.0f) || isinf(eb)) atomicExch(flags + 2, 1ull);
    args[f].eb = eb;
    args[f].inv = 1.0 / (double)eb;
    eb_out[f] = eb;
  }
}

// exclusive prefix of the per-field CP and extremum counts (one CTA)
__global__ void batch_plan_kernel(const BatchHdr *hdr, const unsigned long long *totals,
                                  unsigned long long *kbase, unsigned long long *ebase) {
  __shared__ unsigned long long s_k[1024], s_e[1024];
  __shared__ unsigned long long s_ck, s_ce;
  const unsigned nf = hdr->nf;
  if (threadIdx.x == 0) { s_ck = 0; s_ce = 0; }
  __syncthreads();
  for (unsigned c0 = 0; c0 < nf; c0 += blockDim.x) {
    const unsigned f = c0 + threadIdx.x;
    const unsigned long long k = f < nf ? totals[3 * f + 1] : 0ull, e = f < nf ? totals[3 * f + 2] : 0ull;
    s_k[threadIdx.x] = k;
    s_e[threadIdx.x] = e;
    __syncthreads();
    for (unsigned o = 1; o < blockDim.x; o <<= 1) {
      const unsigned long long a = threadIdx.x >= o ? s_k[threadIdx.x - o] : 0ull;
      const unsigned long long b = threadIdx.x >= o ? s_e[threadIdx.x - o] : 0ull;
      __syncthreads();
      s_k[threadIdx.x] += a;
      s_e[threadIdx.x] += b;
      __syncthreads();
    }
    if (f < nf) {
      kbase[f] = s_ck + s_k[threadIdx.x] - k;
      ebase[f] = s_ce + s_e[threadIdx.x] - e;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) { s_ck += s_k[threadIdx.x]; s_ce += s_e[threadIdx.x]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { kbase[nf] = s_ck; ebase[nf] = s_ce; }
}

// all fields' CP pairs into one list: extremum destinations made global and
// bins computed with each field's bound; per-field bin range reduced
__global__ void __launch_bounds__(kAuxThreads) batch_gather_kernel(
    const BatchHdr *hdr, const BatchFieldDev *fields, const EncArgs *args, const uint2 *pairs,
    const unsigned long long *kbase, const unsigned long long *ebase, uint2 *pairs_all, int *bins,
    int *binmm) {
  const int nf = (int)hdr->nf;
  const unsigned long long K = kbase[nf];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long k0 = (unsigned long long)blockIdx.x * blockDim.x; k0 < K; k0 += stride) {
    const unsigned long long k = k0 + threadIdx.x;
    const bool in = k < K;
    int f = 0, bin = 0;
    if (in) {
      f = last_le(kbase, nf, k);
      const uint2 p = pairs[fields[f].pairs_off + (k - kbase[f])];
      bin = quant_bin(code_float(p.x), args[f].eb, args[f].inv);
      pairs_all[k] = make_uint2(p.x, p.y == kNoExtremum ? kNoExtremum : (uint32_t)(p.y + ebase[f]));
      bins[k] = bin;
    }
    const unsigned act = __ballot_sync(0xffffffffu, in);
    const int f0 = __shfl_sync(0xffffffffu, f, 0);
    const bool same = __all_sync(0xffffffffu, !in || f == f0);
    if (same) {
      int mn = in ? bin : INT_MAX, mx = in ? bin : INT_MIN;
      for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      }
      if ((threadIdx.x & 31) == 0 && act) {
        atomicMin(&binmm[2 * f0], mn);
        atomicMax(&binmm[2 * f0 + 1], mx);
      }
    } else if (in) {
      atomicMin(&binmm[2 * f], bin);
      atomicMax(&binmm[2 * f + 1], bin);
    }
  }
}

// field-disjoint bin ranges: field f's bins move to [base_f, base_f + range_f)
__global__ void batch_offsets_kernel(const BatchHdr *hdr, const unsigned long long *totals, const int *binmm,
                                     long long *off, unsigned long long *flags) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const unsigned nf = hdr->nf;
  long long base = 0;
  bool over = false;
  for (unsigned f = 0; f < nf; f++) {
    off[f] = 0;
    if (totals[3 * f + 1] == 0) continue;
    off[f] = base - (long long)binmm[2 * f];
    base += (long long)binmm[2 * f + 1] - (long long)binmm[2 * f] + 1;
    if (base > (long long)INT_MAX) over = true;
  }
  flags[0] = over ? 1ull : 0ull;
}

__global__ void __launch_bounds__(kAuxThreads) batch_apply_kernel(const BatchHdr *hdr,
                                                                  const unsigned long long *kbase,
                                                                  const long long *off,
                                                                  const unsigned long long *flags, int *bins) {
  if (flags[0]) return;   // ranges overflow: fields are ranked one by one
  const int nf = (int)hdr->nf;
  const unsigned long long K = kbase[nf];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += stride) {
    const int f = last_le(kbase, nf, k);
    bins[k] = (int)((long long)bins[k] + off[f]);
  }
}

// offset table of every non-empty sort-position stream
__global__ void batch_sort_header_kernel(const BatchHdr *hdr, const EncArgs *args) {
  const unsigned nf = hdr->nf;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    if (args[f].n == 0) continue;
    unsigned char *t = args[f].out - 8;
    for (int i = 0; i < 8; i++) t[i] = 0;
  }
}

// ---- encoder launch for a (mode, warps) choice ----
template <int MODE, int WARPS>
static size_t batch_smem(int B) {
  const int tb = WARPS * (32 / octet_group(B));
  return enc2_total_smem(B, MODE != kEncInts, MODE == kEncClassify, WARPS, tb);
}

// prepare == true sets the kernel's shared-memory limit (outside any stream
// capture); prepare == false launches it
template <int MODE, int G, int WARPS>
static cudaError_t launch_batch_g(const EncArgs *args, const unsigned long long *tstart, const unsigned *nf,
                                  unsigned *queue, int B, int grid, cudaStream_t s, bool prepare) {
  auto k = encode2_batch_kernel<MODE, G, WARPS>;
  const size_t sm = batch_smem<MODE, WARPS>(B);
  if (prepare) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k<<<grid, WARPS * 32, sm, s>>>(args, tstart, nf, queue);
  return cudaGetLastError();
}

template <int MODE, int WARPS>
static cudaError_t launch_batch_w(const EncArgs *args, const unsigned long long *tstart, const unsigned *nf,
                                  unsigned *queue, int B, int grid, cudaStream_t s, bool prepare) {
  switch (octet_group(B)) {
    case 1: return launch_batch_g<MODE, 1, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
    case 2: return launch_batch_g<MODE, 2, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
    case 4: return launch_batch_g<MODE, 4, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
    case 8: return launch_batch_g<MODE, 8, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
    case 16: return launch_batch_g<MODE, 16, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
    default: return launch_batch_g<MODE, 32, WARPS>(args, tstart, nf, queue, B, grid, s, prepare);
  }
}

static cudaError_t launch_batch_encode(int mode, int warps, const EncArgs *args, const unsigned long long *tstart,
                                       const unsigned *nf, unsigned *queue, int B, int grid, cudaStream_t s,
                                       bool prepare = false) {
  if (mode == kEncClassify)
    return warps == 4 ? launch_batch_w<kEncClassify, 4>(args, tstart, nf, queue, B, grid, s, prepare)
                      : launch_batch_w<kEncClassify, 8>(args, tstart, nf, queue, B, grid, s, prepare);
  return warps == 4 ? launch_batch_w<kEncInts, 4>(args, tstart, nf, queue, B, grid, s, prepare)
                    : launch_batch_w<kEncInts, 8>(args, tstart, nf, queue, B, grid, s, prepare);
}

static int tile_blocks_w(int B, int warps) { return warps * (32 / octet_group(B)); }

struct EncTune {
  int warps = 8;
  int ctas_per_sm = 8;
};

// tuned shapes per (device, blockSize, mode), shared by every batch object
static std::mutex g_tune_mu;
static std::vector<std::pair<long long, EncTune>> g_tune_cache;
static long long tune_key(int dev, int B, int mode) { return ((long long)dev << 20) | ((long long)B << 4) | mode; }

}  // namespace tsz

using namespace tsz;

struct szp_b200_batch {
  szp_b200_ctx *ctx = nullptr;
  int B = 64;
  bool use_graphs = true;
  int autotune = 1;
  bool tuned = false;
  EncTune tune[2];          // [0] topology encoder, [1] sort-position encoder
  float tune_ms[2][16] = {};
  int tune_count[2] = {0, 0};
  // capacity
  int cap_f = 0;
  unsigned long long cap_tiles = 0, cap_pairs = 0, cap_itiles = 0;
  TableLayout tl;
  ResultLayout rl;
  unsigned char *h_tab = nullptr, *h_itab = nullptr, *h_res = nullptr, *h_ires = nullptr;
  unsigned char *d_tab = nullptr, *d_itab = nullptr, *d_res = nullptr, *d_ires = nullptr;
  TileDesc *d_desc = nullptr, *d_idesc = nullptr;
  unsigned *d_minmax = nullptr, *d_queue = nullptr;
  int *d_binmm = nullptr;
  long long *d_off = nullptr;
  uint2 *d_pairs = nullptr, *d_pairs_all = nullptr;
  int *d_bins = nullptr, *d_sp = nullptr;
  unsigned long long *d_dummy = nullptr;
  cudaGraphExec_t graph_a = nullptr, graph_c = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace tsz {

static void batch_free_buffers(szp_b200_batch *b) {
  if (b->graph_a) cudaGraphExecDestroy(b->graph_a);
  if (b->graph_c) cudaGraphExecDestroy(b->graph_c);
  b->graph_a = b->graph_c = nullptr;
  cudaFreeHost(b->h_tab); cudaFreeHost(b->h_itab); cudaFreeHost(b->h_res); cudaFreeHost(b->h_ires);
  b->h_tab = b->h_itab = b->h_res = b->h_ires = nullptr;
  void *dv[] = {b->d_tab, b->d_itab, b->d_res, b->d_ires, b->d_desc, b->d_idesc, b->d_minmax, b->d_queue,
                b->d_binmm, b->d_off, b->d_pairs, b->d_pairs_all, b->d_bins, b->d_sp, b->d_dummy};
  for (void *p : dv) if (p) cudaFree(p);
  b->d_tab = b->d_itab = b->d_res = b->d_ires = nullptr;
  b->d_desc = b->d_idesc = nullptr;
  b->d_minmax = b->d_queue = nullptr;
  b->d_binmm = nullptr;
  b->d_off = nullptr;
  b->d_pairs = b->d_pairs_all = nullptr;
  b->d_bins = b->d_sp = nullptr;
  b->d_dummy = nullptr;
  b->cap_f = 0;
  b->cap_tiles = b->cap_pairs = b->cap_itiles = 0;
}

template <class T> static bool dalloc(T **p, size_t count) {
  if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    set_error("device allocation of %zu bytes failed", count * sizeof(T));
    return false;
  }
  return true;
}

// grows the batch buffers to hold nf fields, `tiles` topology tiles (at the
// smallest tile shape), `pairs` CP slots and `itiles` sort-stream tiles
static bool batch_reserve(szp_b200_batch *b, int nf, unsigned long long tiles, unsigned long long pairs,
                          unsigned long long itiles) {
  if (nf <= b->cap_f && tiles <= b->cap_tiles && pairs <= b->cap_pairs && itiles <= b->cap_itiles) return true;
  const int cf = std::max(nf, b->cap_f + b->cap_f / 2);
  const unsigned long long ct = std::max(tiles, b->cap_tiles + b->cap_tiles / 4);
  const unsigned long long cp = std::max(pairs, b->cap_pairs + b->cap_pairs / 4);
  const unsigned long long ci = std::max(itiles, b->cap_itiles + b->cap_itiles / 4);
  cudaStreamSynchronize(b->ctx->stream);
  batch_free_buffers(b);
  b->tl.make(cf);
  b->rl.make(cf);
  if (cuda_fail(cudaMallocHost(&b->h_tab, b->tl.bytes), "cudaMallocHost") ||
      cuda_fail(cudaMallocHost(&b->h_itab, b->tl.bytes), "cudaMallocHost") ||
      cuda_fail(cudaMallocHost(&b->h_res, b->rl.bytes), "cudaMallocHost") ||
      cuda_fail(cudaMallocHost(&b->h_ires, b->rl.bytes), "cudaMallocHost"))
    return false;
  memset(b->h_tab, 0, b->tl.bytes);
  memset(b->h_itab, 0, b->tl.bytes);
  if (!dalloc(&b->d_tab, b->tl.bytes) || !dalloc(&b->d_itab, b->tl.bytes) || !dalloc(&b->d_res, b->rl.bytes) ||
      !dalloc(&b->d_ires, b->rl.bytes) || !dalloc(&b->d_desc, ct + cf + 1) || !dalloc(&b->d_idesc, ci + cf + 1) ||
      !dalloc(&b->d_minmax, 2 * (size_t)cf) || !dalloc(&b->d_queue, 8) || !dalloc(&b->d_binmm, 2 * (size_t)cf) ||
      !dalloc(&b->d_off, (size_t)cf) || !dalloc(&b->d_pairs, cp) || !dalloc(&b->d_pairs_all, cp) ||
      !dalloc(&b->d_bins, cp) || !dalloc(&b->d_sp, cp) || !dalloc(&b->d_dummy, 8))
    return false;
  b->cap_f = cf;
  b->cap_tiles = ct;
  b->cap_pairs = cp;
  b->cap_itiles = ci;
  return true;
}

static int persistent_grid(szp_b200_batch *b, const EncTune &t) {
  return std::max(1, b->ctx->sm_count * t.ctas_per_sm);
}

// Stage A on stream s (captured into a graph, or run directly)
static int enqueue_stage_a(szp_b200_batch *b, cudaStream_t s) {
  const TableLayout &T = b->tl;
  const ResultLayout &R = b->rl;
  const BatchHdr *hdr = reinterpret_cast<const BatchHdr *>(b->d_tab + T.hdr);
  const BatchFieldDev *fields = reinterpret_cast<const BatchFieldDev *>(b->d_tab + T.fields);
  EncArgs *args = reinterpret_cast<EncArgs *>(b->d_tab + T.args);
  const unsigned long long *tstart = reinterpret_cast<const unsigned long long *>(b->d_tab + T.tstart);
  unsigned long long *totals = reinterpret_cast<unsigned long long *>(b->d_res + R.totals);
  unsigned long long *kbase = reinterpret_cast<unsigned long long *>(b->d_res + R.kbase);
  unsigned long long *ebase = reinterpret_cast<unsigned long long *>(b->d_res + R.ebase);
  float *eb_out = reinterpret_cast<float *>(b->d_res + R.eb);
  unsigned long long *flags = reinterpret_cast<unsigned long long *>(b->d_res + R.flags);
  const int aux_grid = b->ctx->sm_count * 4;
  if (cuda_fail(cudaMemcpyAsync(b->d_tab, b->h_tab, T.bytes, cudaMemcpyHostToDevice, s), "H2D batch table") ||
      cuda_fail(cudaMemsetAsync(b->d_res, 0, R.bytes, s), "memset") ||
      cuda_fail(cudaMemsetAsync(b->d_desc, 0, (b->cap_tiles + b->cap_f + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(b->d_queue, 0, 8 * sizeof(unsigned), s), "memset"))
    return -1;
  batch_init_kernel<<<(b->cap_f + 255) / 256, 256, 0, s>>>(hdr, fields, b->d_minmax, b->d_binmm);
  batch_minmax_kernel<<<aux_grid, kAuxThreads, 0, s>>>(hdr, fields, b->d_minmax);
  batch_eb_kernel<<<(b->cap_f + 255) / 256, 256, 0, s>>>(hdr, fields, b->d_minmax, args, eb_out, flags);
  if (cuda_fail(cudaGetLastError(), "batch setup kernels")) return -1;
  if (cuda_fail(launch_batch_encode(kEncClassify, b->tune[0].warps, args, tstart, &hdr->nf, b->d_queue, b->B,
                                    persistent_grid(b, b->tune[0]), s),
                "batched topology encoder"))
    return -1;
  batch_plan_kernel<<<1, 1024, 0, s>>>(hdr, totals, kbase, ebase);
  batch_gather_kernel<<<aux_grid, kAuxThreads, 0, s>>>(hdr, fields, args, b->d_pairs, kbase, ebase,
                                                       b->d_pairs_all, b->d_bins, b->d_binmm);
  batch_offsets_kernel<<<1, 32, 0, s>>>(hdr, totals, b->d_binmm, b->d_off, flags);
  batch_apply_kernel<<<aux_grid, kAuxThreads, 0, s>>>(hdr, kbase, b->d_off, flags, b->d_bins);
  if (cuda_fail(cudaGetLastError(), "batch gather kernels") ||
      cuda_fail(cudaMemcpyAsync(b->h_res, b->d_res, R.bytes, cudaMemcpyDeviceToHost, s), "D2H batch results"))
    return -1;
  return 0;
}

// Stage C on stream s
static int enqueue_stage_c(szp_b200_batch *b, cudaStream_t s) {
  const TableLayout &T = b->tl;
  const ResultLayout &R = b->rl;
  const BatchHdr *hdr = reinterpret_cast<const BatchHdr *>(b->d_itab + T.hdr);
  const EncArgs *args = reinterpret_cast<const EncArgs *>(b->d_itab + T.args);
  const unsigned long long *tstart = reinterpret_cast<const unsigned long long *>(b->d_itab + T.tstart);
  if (cuda_fail(cudaMemcpyAsync(b->d_itab, b->h_itab, T.bytes, cudaMemcpyHostToDevice, s), "H2D sort table") ||
      cuda_fail(cudaMemsetAsync(b->d_ires, 0, R.bytes, s), "memset") ||
      cuda_fail(cudaMemsetAsync(b->d_idesc, 0, (b->cap_itiles + b->cap_f + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(b->d_queue + 4, 0, 4 * sizeof(unsigned), s), "memset"))
    return -1;
  batch_sort_header_kernel<<<(b->cap_f + 255) / 256, 256, 0, s>>>(hdr, args);
  if (cuda_fail(launch_batch_encode(kEncInts, b->tune[1].warps, args, tstart, &hdr->nf, b->d_queue + 4, b->B,
                                    persistent_grid(b, b->tune[1]), s),
                "batched sort-position encoder") ||
      cuda_fail(cudaMemcpyAsync(b->h_ires, b->d_ires, R.bytes, cudaMemcpyDeviceToHost, s), "D2H sort results"))
    return -1;
  return 0;
}

static int run_stage(szp_b200_batch *b, int which) {
  cudaStream_t s = b->ctx->stream;
  cudaGraphExec_t &ge = which == 0 ? b->graph_a : b->graph_c;
  if (cuda_fail(launch_batch_encode(which == 0 ? kEncClassify : kEncInts, b->tune[which].warps, nullptr, nullptr,
                                    nullptr, nullptr, b->B, 1, s, true),
                "encoder attributes"))
    return -1;
  b->ctx->launches += which == 0 ? 8 : 2;
  if (!b->use_graphs) {
    return which == 0 ? enqueue_stage_a(b, s) : enqueue_stage_c(b, s);
  }
  if (!ge) {
    cudaGraph_t g = nullptr;
    if (cuda_fail(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
    const int rc = which == 0 ? enqueue_stage_a(b, s) : enqueue_stage_c(b, s);
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc || cuda_fail(e, "end capture")) {
      if (g) cudaGraphDestroy(g);
      return -1;
    }
    const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (cuda_fail(ei, "graph instantiate")) { ge = nullptr; return -1; }
  }
  return cuda_fail(cudaGraphLaunch(ge, s), "graph launch") ? -1 : 0;
}

static void drop_graphs(szp_b200_batch *b) {
  if (b->graph_a) cudaGraphExecDestroy(b->graph_a);
  if (b->graph_c) cudaGraphExecDestroy(b->graph_c);
  b->graph_a = b->graph_c = nullptr;
}

struct FieldPlan {
  unsigned long long n, nb, interior;
  Geom g;
};

// fills the topology table for the current tile shape
static void fill_topo_table(szp_b200_batch *b, const szp_b200_batch_field *fs, int nf,
                            const std::vector<FieldPlan> &plan) {
  const TableLayout &T = b->tl;
  BatchHdr *hdr = reinterpret_cast<BatchHdr *>(b->h_tab + T.hdr);
  BatchFieldDev *fd = reinterpret_cast<BatchFieldDev *>(b->h_tab + T.fields);
  EncArgs *args = reinterpret_cast<EncArgs *>(b->h_tab + T.args);
  unsigned long long *tstart = reinterpret_cast<unsigned long long *>(b->h_tab + T.tstart);
  const ResultLayout &R = b->rl;
  unsigned long long *totals = reinterpret_cast<unsigned long long *>(b->d_res + R.totals);
  unsigned long long *flags = reinterpret_cast<unsigned long long *>(b->d_res + R.flags);
  const int TB = tile_blocks_w(b->B, b->tune[0].warps);
  unsigned long long t = 0, p = 0, ch = 0;
  for (int f = 0; f < nf; f++) {
    const FieldPlan &P = plan[f];
    fd[f].data = fs[f].d_data;
    fd[f].n = P.n;
    fd[f].pairs_off = p;
    fd[f].chunk0 = ch;
    fd[f].err = fs[f].errBound;
    fd[f].rel = fs[f].rel ? 1 : 0;
    fd[f].topo = fs[f].d_topo;
    if (fs[f].rel) ch += (P.n + kMinMaxChunk - 1) / kMinMaxChunk;
    const unsigned long long nt = (P.nb + TB - 1) / TB;
    EncArgs a{};
    a.data = fs[f].d_data;
    a.n = P.n;
    a.B = b->B;
    a.eb = fs[f].errBound;
    a.inv = 1.0 / (double)fs[f].errBound;
    a.g = P.g;
    a.out = fs[f].d_topo + 8;
    a.out_cap = fs[f].topo_cap - 8;
    a.desc = b->d_desc + t + f;
    a.tile_ctr = reinterpret_cast<unsigned *>(b->d_dummy);
    a.err = reinterpret_cast<int *>(flags + 1);
    a.total = totals + 3 * f;
    a.cp_mode = kCpPairs;
    a.cp_out = b->d_pairs + p;
    a.cp_cap = P.interior;
    args[f] = a;
    tstart[f] = t;
    t += nt;
    p += P.interior;
  }
  tstart[nf] = t;
  hdr->nf = (unsigned)nf;
  hdr->nchunks = ch;
}

static void fill_sort_table(szp_b200_batch *b, const szp_b200_batch_field *fs, int nf,
                            const unsigned long long *ebase, const unsigned long long *E) {
  const TableLayout &T = b->tl;
  BatchHdr *hdr = reinterpret_cast<BatchHdr *>(b->h_itab + T.hdr);
  EncArgs *args = reinterpret_cast<EncArgs *>(b->h_itab + T.args);
  unsigned long long *tstart = reinterpret_cast<unsigned long long *>(b->h_itab + T.tstart);
  const ResultLayout &R = b->rl;
  unsigned long long *totals = reinterpret_cast<unsigned long long *>(b->d_ires + R.totals);
  unsigned long long *flags = reinterpret_cast<unsigned long long *>(b->d_ires + R.flags);
  const int TB = tile_blocks_w(b->B, b->tune[1].warps);
  unsigned long long t = 0;
  for (int f = 0; f < nf; f++) {
    const unsigned long long nb = (E[f] + b->B - 1) / b->B;
    const unsigned long long nt = (nb + TB - 1) / TB;
    EncArgs a{};
    a.ints = b->d_sp + ebase[f];
    a.n = E[f];
    a.B = b->B;
    a.eb = 1.0f;
    a.inv = 1.0;
    a.g = make_geom(2, 1, 1, 1);
    a.out = E[f] ? fs[f].d_sort + 8 : nullptr;
    a.out_cap = E[f] ? fs[f].sort_cap - 8 : 0;
    a.desc = b->d_idesc + t + f;
    a.tile_ctr = reinterpret_cast<unsigned *>(b->d_dummy);
    a.err = reinterpret_cast<int *>(flags + 1);
    a.total = totals + 3 * f;
    a.cp_mode = kCpNone;
    args[f] = a;
    tstart[f] = t;
    t += nt;
  }
  tstart[nf] = t;
  hdr->nf = (unsigned)nf;
  hdr->nchunks = 0;
}

// Autotuner: times every candidate shape of one encoder on the current batch
// (the streams do not depend on the shape) and keeps the fastest.
static int autotune_encoder(szp_b200_batch *b, int which, const szp_b200_batch_field *fs, int nf,
                            const std::vector<FieldPlan> &plan, const unsigned long long *ebase,
                            const unsigned long long *E) {
  static const EncTune cands[] = {{4, 4}, {4, 8}, {4, 12}, {4, 16}, {8, 2}, {8, 3}, {8, 4}, {8, 8}};
  const int nc = (int)(sizeof(cands) / sizeof(cands[0]));
  cudaStream_t s = b->ctx->stream;
  float best = 1e30f;
  EncTune bt = b->tune[which];
  b->tune_count[which] = nc;
  for (int c = 0; c < nc; c++) {
    b->tune[which] = cands[c];
    if (which == 0) fill_topo_table(b, fs, nf, plan);
    else fill_sort_table(b, fs, nf, ebase, E);
    unsigned char *h = which == 0 ? b->h_tab : b->h_itab;
    unsigned char *d = which == 0 ? b->d_tab : b->d_itab;
    const TableLayout &T = b->tl;
    const EncArgs *args = reinterpret_cast<const EncArgs *>(d + T.args);
    const unsigned long long *tstart = reinterpret_cast<const unsigned long long *>(d + T.tstart);
    const BatchHdr *hdr = reinterpret_cast<const BatchHdr *>(d + T.hdr);
    float ms_best = 1e30f;
    if (cuda_fail(launch_batch_encode(which == 0 ? kEncClassify : kEncInts, cands[c].warps, nullptr, nullptr,
                                      nullptr, nullptr, b->B, 1, s, true),
                  "encoder attributes"))
      return -1;
    for (int rep = 0; rep < 3; rep++) {
      if (cuda_fail(cudaMemcpyAsync(d, h, T.bytes, cudaMemcpyHostToDevice, s), "H2D") ||
          cuda_fail(cudaMemsetAsync(which == 0 ? b->d_res : b->d_ires, 0, b->rl.bytes, s), "memset") ||
          cuda_fail(cudaMemsetAsync(which == 0 ? (void *)b->d_desc : (void *)b->d_idesc, 0,
                                    ((which == 0 ? b->cap_tiles : b->cap_itiles) + b->cap_f + 1) * sizeof(TileDesc),
                                    s),
                    "memset") ||
          cuda_fail(cudaMemsetAsync(b->d_queue, 0, 8 * sizeof(unsigned), s), "memset"))
        return -1;
      if (which == 0) {
        // the relative bounds are resolved once before the timed encoder run
        const BatchFieldDev *fields = reinterpret_cast<const BatchFieldDev *>(d + T.fields);
        batch_init_kernel<<<(b->cap_f + 255) / 256, 256, 0, s>>>(hdr, fields, b->d_minmax, b->d_binmm);
        batch_minmax_kernel<<<b->ctx->sm_count * 4, kAuxThreads, 0, s>>>(hdr, fields, b->d_minmax);
        batch_eb_kernel<<<(b->cap_f + 255) / 256, 256, 0, s>>>(
            hdr, fields, b->d_minmax, const_cast<EncArgs *>(args),
            reinterpret_cast<float *>(b->d_res + b->rl.eb),
            reinterpret_cast<unsigned long long *>(b->d_res + b->rl.flags));
      }
      cudaEventRecord(b->ev0, s);
      if (cuda_fail(launch_batch_encode(which == 0 ? kEncClassify : kEncInts, cands[c].warps, args, tstart, &hdr->nf,
                                        b->d_queue + (which == 0 ? 0 : 4), b->B, persistent_grid(b, cands[c]), s),
                    "autotune launch"))
        return -1;
      cudaEventRecord(b->ev1, s);
      if (cuda_fail(cudaEventSynchronize(b->ev1), "autotune")) return -1;
      float ms = 0;
      cudaEventElapsedTime(&ms, b->ev0, b->ev1);
      if (rep > 0) ms_best = std::min(ms_best, ms);
    }
    b->tune_ms[which][c] = ms_best;
    if (ms_best < best) { best = ms_best; bt = cands[c]; }
  }
  b->tune[which] = bt;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const long long key = tune_key(b->ctx->device, b->B, which);
  for (auto &kv : g_tune_cache) if (kv.first == key) { kv.second = bt; return 0; }
  g_tune_cache.push_back({key, bt});
  return 0;
}

static unsigned long long interior_of(const Geom &g) {
  if (g.nd == 2) return (g.d2 > 2 && g.d3 > 2) ? (unsigned long long)(g.d2 - 2) * (g.d3 - 2) : 0ull;
  return (g.d1 > 2 && g.d2 > 2 && g.d3 > 2) ? (unsigned long long)(g.d1 - 2) * (g.d2 - 2) * (g.d3 - 2) : 0ull;
}

}  // namespace tsz

extern "C" {

szp_b200_batch *szp_b200_batch_create(void *cuda_stream, int blockSize) {
  clear_error();
  if (blockSize <= 0 || blockSize > 256) {
    set_error("szp_b200_batch_create: blockSize %d out of range [1, 256]", blockSize);
    return nullptr;
  }
  auto *b = new szp_b200_batch();
  b->ctx = szp_b200_ctx_create(cuda_stream);
  if (!b->ctx) { delete b; return nullptr; }
  b->B = blockSize;
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (int m = 0; m < 2; m++)
    for (auto &kv : g_tune_cache)
      if (kv.first == tune_key(b->ctx->device, blockSize, m)) { b->tune[m] = kv.second; b->tuned = true; }
  return b;
}

void szp_b200_batch_destroy(szp_b200_batch *b) {
  if (!b) return;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  batch_free_buffers(b);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  szp_b200_ctx_destroy(b->ctx);
  delete b;
}

int szp_b200_batch_configure(szp_b200_batch *b, int use_graphs, int autotune) {
  clear_error();
  if (!b) { set_error("null batch"); return -1; }
  b->use_graphs = use_graphs != 0;
  b->autotune = autotune;
  if (autotune > 1) b->tuned = false;   // tune again on the next batch
  drop_graphs(b);
  return 0;
}

int szp_b200_batch_tuning(szp_b200_batch *b, int *shape, float *ms, int max) {
  clear_error();
  if (!b || !shape) { set_error("null argument"); return -1; }
  shape[0] = b->tune[0].warps * 32;
  shape[1] = b->tune[0].ctas_per_sm;
  shape[2] = b->tune[1].warps * 32;
  shape[3] = b->tune[1].ctas_per_sm;
  if (ms)
    for (int i = 0; i < max && i < 16; i++) ms[i] = i < b->tune_count[0] ? b->tune_ms[0][i] : 0.f;
  return b->tuned ? 1 : 0;
}

szp_b200_ctx *szp_b200_batch_ctx(szp_b200_batch *b) { return b ? b->ctx : nullptr; }

int szp_b200_batch_reserve(szp_b200_batch *b, int max_fields, size_t max_elements) {
  DeviceGuard dg(b ? b->ctx : nullptr);
  clear_error();
  if (!b || max_fields <= 0 || max_elements == 0) { set_error("szp_b200_batch_reserve: invalid arguments"); return -1; }
  // bounds over any max_fields fields of max_elements elements in total
  // (the sums szp_b200_batch_compress forms): blocks <= N / B + F, and a
  // field's interior points (CP slots) <= its elements
  const unsigned long long F = (unsigned long long)max_fields, N = max_elements, B = (unsigned long long)b->B;
  const unsigned long long tb_min = (unsigned long long)tile_blocks_w(b->B, 4);
  const unsigned long long blocks = N / B + F;
  const unsigned long long tiles = blocks / tb_min + 2 * F + 1;
  const unsigned long long itiles = N / B / tb_min + 3 * F + 1;
  const int oldcap = b->cap_f;
  const unsigned long long oldt = b->cap_tiles, oldp = b->cap_pairs, oldi = b->cap_itiles;
  if (!batch_reserve(b, max_fields, tiles, N, itiles)) return -1;
  if (b->cap_f != oldcap || b->cap_tiles != oldt || b->cap_pairs != oldp || b->cap_itiles != oldi) drop_graphs(b);
  szp_b200_ctx *ctx = b->ctx;
  if (!ctx->scratch.reserve(std::max(rank_scratch_bytes(N, ctx->sm_count),
                                     rank_scratch_bytes_seg(N, max_fields, ctx->sm_count)) + 8192))
    return -1;
  return cuda_fail(cudaStreamSynchronize(ctx->stream), "batch reserve") ? -1 : 0;
}

int szp_b200_batch_compress(szp_b200_batch *b, szp_b200_batch_field *fs, int count) {
  DeviceGuard dg(b ? b->ctx : nullptr);
  clear_error();
  if (!b || (!fs && count)) { set_error("null argument"); return -1; }
  if (count <= 0) return 0;
  const int B = b->B;
  std::vector<FieldPlan> plan(count);
  unsigned long long tiles = 0, pairs = 0, itiles = 0;
  const int tb_min = tile_blocks_w(B, 4);
  for (int f = 0; f < count; f++) {
    unsigned long long n;
    Geom g;
    const szp_b200_geom &gg = fs[f].geom;
    if (!fs[f].d_data || !fs[f].d_topo || !fs[f].d_sort) { set_error("field %d: null pointer", f); return -1; }
    if (!geom_elements(gg, &n, &g)) { set_error("field %d: invalid geometry", f); return -1; }
    if (!(fs[f].errBound > 0.0f)) { set_error("field %d: error bound must be positive", f); return -1; }
    if (fs[f].topo_cap < 8 || fs[f].sort_cap < 8) { set_error("field %d: output buffer too small", f); return -1; }
    plan[f].n = n;
    plan[f].nb = (n + B - 1) / B;
    plan[f].g = g;
    plan[f].interior = interior_of(g);
    tiles += (plan[f].nb + tb_min - 1) / tb_min;
    pairs += plan[f].interior;
    itiles += (std::min(plan[f].interior, n) / B + 1 + tb_min - 1) / tb_min + 1;
    fs[f].sizes.topo_bytes = fs[f].sizes.sort_bytes = fs[f].sizes.cp_count = fs[f].sizes.extrema_count = 0;
  }
  const int oldcap = b->cap_f;
  const unsigned long long oldt = b->cap_tiles, oldp = b->cap_pairs, oldi = b->cap_itiles;
  if (!batch_reserve(b, count, tiles, pairs, itiles)) return -1;
  if (b->cap_f != oldcap || b->cap_tiles != oldt || b->cap_pairs != oldp || b->cap_itiles != oldi) drop_graphs(b);
  szp_b200_ctx *ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  if (b->autotune == 1 && !b->tuned) {
    // shapes already tuned on this device by another batch object
    std::lock_guard<std::mutex> lk(g_tune_mu);
    int found = 0;
    for (int m = 0; m < 2; m++)
      for (auto &kv : g_tune_cache)
        if (kv.first == tune_key(ctx->device, B, m)) { b->tune[m] = kv.second; found++; }
    if (found == 2) { b->tuned = true; drop_graphs(b); }
  }
  const bool tune_now = b->autotune && !b->tuned;
  tl_begin(ctx);
  if (tune_now) {
    if (autotune_encoder(b, 0, fs, count, plan, nullptr, nullptr)) return -1;
    drop_graphs(b);
  }
  fill_topo_table(b, fs, count, plan);
  if (run_stage(b, 0)) return -1;
  tl_mark(ctx, "batch_encode_topo");
  if (cuda_fail(cudaStreamSynchronize(s), "batch stage A")) return -1;
  const ResultLayout &R = b->rl;
  const unsigned long long *totals = reinterpret_cast<const unsigned long long *>(b->h_res + R.totals);
  const unsigned long long *kbase = reinterpret_cast<const unsigned long long *>(b->h_res + R.kbase);
  const unsigned long long *ebase = reinterpret_cast<const unsigned long long *>(b->h_res + R.ebase);
  const float *ebv = reinterpret_cast<const float *>(b->h_res + R.eb);
  const unsigned long long *flags = reinterpret_cast<const unsigned long long *>(b->h_res + R.flags);
  if (flags[2]) { set_error("a relative error bound resolved to a non-positive or infinite bound"); return -1; }
  if (flags[1] & 0xffffffffull) {
    set_error("batched encoder reported status %d%s", (int)(flags[1] & 0xffffffffull),
              (flags[1] & 0xffffffffull) == kErrOutputOverflow ? " (a topology buffer is too small)" : "");
    return -1;
  }
  const unsigned long long Ktot = kbase[count], Etot = ebase[count];
  if (Etot >= 0xFFFFFFFFull) { set_error("too many extrema in one batch"); return -1; }
  std::vector<unsigned long long> E(count), eb_copy(count);
  for (int f = 0; f < count; f++) {
    fs[f].sizes.topo_bytes = 8 + totals[3 * f];
    fs[f].sizes.cp_count = totals[3 * f + 1];
    fs[f].sizes.extrema_count = totals[3 * f + 2];
    fs[f].abs_eb = ebv[f];
    E[f] = totals[3 * f + 2];
  }
  std::vector<unsigned long long> eb_base(ebase, ebase + count + 1);
  // ranks of the whole batch
  if (Etot > 0) {
    if (!ctx->scratch.reserve(std::max(rank_scratch_bytes(Ktot, ctx->sm_count),
                                       rank_scratch_bytes_seg(Ktot, count, ctx->sm_count)) + 8192))
      return -1;
    if (!flags[0]) {
      std::vector<unsigned long long> Kf(count);
      for (int f = 0; f < count; f++) Kf[f] = totals[3 * f + 1];
      if (rank_positions_seg(ctx, b->d_pairs_all, b->d_bins, Kf.data(), count, b->d_sp)) return -1;
    } else {
      for (int f = 0; f < count; f++) {
        const unsigned long long Kf = totals[3 * f + 1];
        if (!E[f]) continue;
        ctx->scratch.reset();
        if (rank_positions(ctx, b->d_pairs_all + kbase[f], nullptr, Kf, E[f], ebv[f], b->d_sp)) return -1;
      }
    }
  }
  tl_mark(ctx, "batch_rank");
  // sort-position streams of the whole batch
  if (Etot > 0) {
    if (tune_now) {
      if (autotune_encoder(b, 1, fs, count, plan, eb_base.data(), E.data())) return -1;
      drop_graphs(b);
    }
    fill_sort_table(b, fs, count, eb_base.data(), E.data());
    if (run_stage(b, 1)) return -1;
    if (cuda_fail(cudaStreamSynchronize(s), "batch stage C")) return -1;
    const unsigned long long *it = reinterpret_cast<const unsigned long long *>(b->h_ires + R.totals);
    const unsigned long long *ifl = reinterpret_cast<const unsigned long long *>(b->h_ires + R.flags);
    if (ifl[1] & 0xffffffffull) {
      set_error("batched sort-position encoder reported status %d", (int)(ifl[1] & 0xffffffffull));
      return -1;
    }
    for (int f = 0; f < count; f++) fs[f].sizes.sort_bytes = E[f] ? 8 + it[3 * f] : 0;
  }
  tl_mark(ctx, "batch_encode_sort");
  if (tune_now) b->tuned = true;
  return 0;
}

}  // extern "C"
